/*
 * santoku.tsetlin.capi on B200: the Lua C module of the reference
 * (lib/santoku/tsetlin/capi.c:1790-1803) as a thin binding over the C ABI
 * of libtsetlin_b200.so (include/tsetlin_b200.h).  Module name, functions,
 * methods, table keys, argument order and return values are the
 * reference's, so `require("santoku.tsetlin")` code runs unchanged:
 *
 *   create(type, tbl)           capi.c:701-716
 *   load(data, from_string)     capi.c:1751-1772
 *   align                       capi.c:1801-1802
 *   m:train(tbl)                capi.c:1484-1507
 *   m:predict(problems, n) / m:predict(problems, dim_offsets, n)
 *                               capi.c:1088-1110
 *   m:persist(path?)            capi.c:1538-1562
 *   m:checkpoint(cvec)          capi.c:1564-1576
 *   m:restore(cvec)             capi.c:1578-1588
 *   m:reconfigure(tbl)          capi.c:1590-1673
 *   m:restrict(ivec)            capi.c:752-901
 *   m:type()                    capi.c:1774-1788
 *   m:destroy() / __gc          capi.c:725-750
 *
 * Samples, labels and codes are santoku-matrix cvec / ivec userdata, read
 * and created through santoku-matrix's own accessors (tk_cvec_peek,
 * tk_ivec_peek, tk_cvec_create, tk_ivec_create, tk_cvec_ensure), as the
 * reference does.  Two optional create keys have no counterpart in the
 * reference: `device` (CUDA ordinal, default 0) and `seed` (key of the
 * Philox draws, default 0).  Errors of the library are raised as Lua errors
 * carrying tm_last_error().
 *
 * Build (beside the santoku and santoku-matrix headers of the host's Lua
 * rocks):
 *   cc -O2 -fPIC -shared -I<lua include> -I<santoku include> -I<repo>/include \
 *      santoku_tsetlin_capi.c -L<dir of libtsetlin_b200.so> -ltsetlin_b200 \
 *      -o santoku/tsetlin/capi.so
 */
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <lauxlib.h>
#include <lua.h>

#include <santoku/cvec.h>
#include <santoku/ivec.h>

#include "tsetlin_b200.h"

#define TM_LUA_MT "santoku_tsetlin" /* the reference's metatable name, capi.c:39 */

typedef struct {
  tm_machine *m;
} tm_lua_box;

#if LUA_VERSION_NUM < 502
static void tm_lua_setfuncs(lua_State *L, const luaL_Reg *r) {
  for (; r->name; r++) {
    lua_pushcfunction(L, r->func);
    lua_setfield(L, -2, r->name);
  }
}
static int tm_lua_absindex(lua_State *L, int i) {
  return (i > 0 || i <= LUA_REGISTRYINDEX) ? i : lua_gettop(L) + i + 1;
}
#else
static void tm_lua_setfuncs(lua_State *L, const luaL_Reg *r) { luaL_setfuncs(L, r, 0); }
static int tm_lua_absindex(lua_State *L, int i) { return lua_absindex(L, i); }
#endif

static int tm_lua_fail(lua_State *L) { return luaL_error(L, "%s", tm_last_error()); }

static tm_machine *tm_lua_check(lua_State *L, int i) {
  tm_lua_box *b = (tm_lua_box *)luaL_checkudata(L, i, TM_LUA_MT);
  if (!b->m) luaL_error(L, "tsetlin machine already destroyed");
  return b->m;
}

/* ---- table fields ------------------------------------------------------ */
static int tm_lua_has(lua_State *L, int t, const char *k) {
  lua_getfield(L, t, k);
  const int has = !lua_isnil(L, -1);
  lua_pop(L, 1);
  return has;
}

static double tm_lua_number(lua_State *L, int t, const char *who, const char *k, int required,
                            double dflt) {
  lua_getfield(L, t, k);
  if (lua_isnil(L, -1)) {
    lua_pop(L, 1);
    if (required) luaL_error(L, "%s: %s is required", who, k);
    return dflt;
  }
  if (!lua_isnumber(L, -1)) luaL_error(L, "%s: %s must be a number", who, k);
  const double v = lua_tonumber(L, -1);
  lua_pop(L, 1);
  return v;
}

static uint32_t tm_lua_unsigned(lua_State *L, int t, const char *who, const char *k, int required,
                                uint32_t dflt) {
  const double v = tm_lua_number(L, t, who, k, required, (double)dflt);
  if (v < 0 || v > 4294967295.0 || v != (double)(uint32_t)v)
    luaL_error(L, "%s: %s must be an unsigned integer", who, k);
  return (uint32_t)v;
}

static int tm_lua_bool(lua_State *L, int t, const char *k) {
  lua_getfield(L, t, k);
  const int v = lua_toboolean(L, -1);
  lua_pop(L, 1);
  return v;
}

/* field k of table t as a cvec / ivec (left on the stack until the caller pops) */
static tk_cvec_t *tm_lua_cvec_field(lua_State *L, int t, const char *k) {
  lua_getfield(L, t, k);
  return tk_cvec_peek(L, -1, k);
}

static tk_ivec_t *tm_lua_ivec_field(lua_State *L, int t, const char *k) {
  lua_getfield(L, t, k);
  return tk_ivec_peek(L, -1, k);
}

static void tm_lua_push_machine(lua_State *L, tm_machine *m) {
  tm_lua_box *b = (tm_lua_box *)lua_newuserdata(L, sizeof(tm_lua_box));
  b->m = m;
  luaL_getmetatable(L, TM_LUA_MT);
  lua_setmetatable(L, -2);
}

/* ---- create (capi.c:627-716) ------------------------------------------- */
static int tm_lua_create(lua_State *L) {
  const char *type = luaL_checkstring(L, 1);
  luaL_checktype(L, 2, LUA_TTABLE);
  tm_params p;
  tm_params_init(&p);
  const char *who;
  if (!strcmp(type, "classifier")) {
    who = "create classifier";
    p.type = TM_CLASSIFIER;
    p.classes = tm_lua_unsigned(L, 2, who, "classes", 1, 0);
  } else if (!strcmp(type, "encoder")) {
    who = "create encoder";
    p.type = TM_ENCODER;
    p.classes = tm_lua_unsigned(L, 2, who, "hidden", 1, 0);
  } else {
    return luaL_error(L, "unexpected tsetlin machine type in create");
  }
  p.individualized = tm_lua_bool(L, 2, "individualized");
  tk_ivec_t *fo = NULL;
  if (p.individualized) {
    fo = tm_lua_ivec_field(L, 2, "feat_offsets");
    if (fo->n != (size_t)p.classes + 1)
      return luaL_error(L, "%s: feat_offsets must have classes + 1 elements", who);
    p.feat_offsets = fo->a;
  } else {
    p.features = tm_lua_unsigned(L, 2, who, p.type == TM_CLASSIFIER ? "features" : "visible", 1, 0);
  }
  p.clauses = tm_lua_unsigned(L, 2, who, "clauses", 1, 0);
  p.clause_tolerance = tm_lua_unsigned(L, 2, who, "clause_tolerance", 1, 0);
  p.clause_maximum = tm_lua_unsigned(L, 2, who, "clause_maximum", 1, 0);
  p.state_bits = tm_lua_unsigned(L, 2, who, "state", 0, 8);
  p.include_bits = tm_lua_unsigned(L, 2, who, "include_bits", 0, 1);
  p.target = tm_lua_number(L, 2, who, "target", 0, -1.0);
  p.negative = tm_lua_number(L, 2, who, "negative", 0, -1.0);
  p.specificity = tm_lua_number(L, 2, who, "specificity", 1, 0.0);
  p.reusable = tm_lua_bool(L, 2, "reusable");
  p.seed = (uint64_t)tm_lua_number(L, 2, who, "seed", 0, 0.0);
  p.device = (int32_t)tm_lua_number(L, 2, who, "device", 0, 0.0);
  tm_machine *m = NULL;
  if (tm_create(&p, &m) != TM_OK) return tm_lua_fail(L);
  if (fo) lua_pop(L, 1);
  tm_lua_push_machine(L, m);
  return 1;
}

/* ---- load (capi.c:1751-1772) ------------------------------------------- */
static int tm_lua_load(lua_State *L) {
  lua_settop(L, 3);
  size_t len = 0;
  const char *data = luaL_checklstring(L, 1, &len);
  const int from_string = lua_type(L, 2) == LUA_TBOOLEAN && lua_toboolean(L, 2);
  const int device = lua_isnumber(L, 3) ? (int)lua_tointeger(L, 3) : 0;
  tm_machine *m = NULL;
  if (tm_load((const uint8_t *)data, len, from_string, device, &m) != TM_OK) return tm_lua_fail(L);
  tm_lua_push_machine(L, m);
  return 1;
}

/* ---- train (capi.c:1112-1507) ------------------------------------------ */
typedef struct {
  lua_State *L;
  int fn;
} tm_lua_each;

/* capi.c:1168-1182: each(epoch); an error is printed and stops training,
 * `false` stops training. */
static int tm_lua_each_cb(void *user, uint32_t epoch) {
  tm_lua_each *e = (tm_lua_each *)user;
  lua_State *L = e->L;
  lua_pushvalue(L, e->fn);
  lua_pushinteger(L, (lua_Integer)epoch);
  if (lua_pcall(L, 1, 1, 0) != 0) {
    fprintf(stderr, "Error in Lua callback: %s\n", lua_tostring(L, -1));
    lua_pop(L, 1);
    return 1;
  }
  const int stop = lua_type(L, -1) == LUA_TBOOLEAN && !lua_toboolean(L, -1);
  lua_pop(L, 1);
  return stop;
}

static int tm_lua_train(lua_State *L) {
  lua_settop(L, 2);
  tm_machine *m = tm_lua_check(L, 1);
  luaL_checktype(L, 2, LUA_TTABLE);
  uint64_t info[TM_INFO_N];
  if (tm_get_info(m, info) != TM_OK) return tm_lua_fail(L);
  const int classifier = info[0] == TM_CLASSIFIER, ind = info[16] != 0;
  tm_train_args a;
  memset(&a, 0, sizeof a);
  a.samples = tm_lua_unsigned(L, 2, "train", "samples", 1, 0);
  a.iterations = tm_lua_unsigned(L, 2, "train", "iterations", 1, 0);
  if (classifier) {
    a.problems = (const uint8_t *)tm_lua_cvec_field(L, 2, "problems")->a;
    a.solutions = tm_lua_ivec_field(L, 2, "solutions")->a;
  } else {
    a.problems = (const uint8_t *)tm_lua_cvec_field(L, 2, "sentences")->a;
    a.codes = (const uint8_t *)tm_lua_cvec_field(L, 2, "codes")->a;
  }
  if (ind) a.dim_offsets = tm_lua_ivec_field(L, 2, "dim_offsets")->a;
  tm_lua_each each;
  if (tm_lua_has(L, 2, "each")) {
    lua_getfield(L, 2, "each");
    each.L = L;
    each.fn = tm_lua_absindex(L, -1);
    a.each = tm_lua_each_cb;
    a.each_user = &each;
  }
  if (tm_train(m, &a) != TM_OK) return tm_lua_fail(L);
  lua_settop(L, 1);
  return 0;
}

/* ---- predict (capi.c:903-1110) ----------------------------------------- */
static int tm_lua_predict(lua_State *L) {
  tm_machine *m = tm_lua_check(L, 1);
  uint64_t info[TM_INFO_N];
  if (tm_get_info(m, info) != TM_OK) return tm_lua_fail(L);
  const int classifier = info[0] == TM_CLASSIFIER, ind = info[16] != 0;
  tk_cvec_t *problems = tk_cvec_peek(L, 2, "problems");
  const int64_t *dim_offsets = NULL;
  uint64_t n;
  if (ind) {
    dim_offsets = tk_ivec_peek(L, 3, "dim_offsets")->a;
    n = (uint64_t)luaL_checkinteger(L, 4);
  } else {
    n = (uint64_t)luaL_checkinteger(L, 3);
  }
  if (classifier) {
    tk_ivec_t *out = tk_ivec_create(L, n, 0, 0);
    if (tm_predict(m, (const uint8_t *)problems->a, dim_offsets, n, out->a, NULL, 0) != TM_OK)
      return tm_lua_fail(L);
  } else {
    tk_cvec_t *out = tk_cvec_create(L, n * info[12], 0, 0); /* class_chunks bytes per sample */
    if (tm_predict(m, (const uint8_t *)problems->a, dim_offsets, n, NULL, (uint8_t *)out->a, 0) !=
        TM_OK)
      return tm_lua_fail(L);
  }
  return 1;
}

/* ---- persist / checkpoint / restore (capi.c:1538-1588) ----------------- */
static int tm_lua_persist(lua_State *L) {
  lua_settop(L, 2);
  tm_machine *m = tm_lua_check(L, 1);
  if (lua_isnil(L, 2)) {
    uint8_t *data = NULL;
    uint64_t len = 0;
    if (tm_persist_buf(m, &data, &len) != TM_OK) return tm_lua_fail(L);
    lua_pushlstring(L, (const char *)data, (size_t)len);
    tm_free(data);
    return 1;
  }
  if (tm_persist(m, luaL_checkstring(L, 2)) != TM_OK) return tm_lua_fail(L);
  return 0;
}

static int tm_lua_checkpoint(lua_State *L) {
  lua_settop(L, 2);
  tm_machine *m = tm_lua_check(L, 1);
  tk_cvec_t *cp = tk_cvec_peek(L, 2, "checkpoint");
  uint64_t size = 0;
  if (tm_checkpoint(m, NULL, 0, &size) != TM_OK) return tm_lua_fail(L);
  if (tk_cvec_ensure(cp, size) != 0) return luaL_error(L, "failed to resize checkpoint buffer");
  cp->n = size;
  if (tm_checkpoint(m, (uint8_t *)cp->a, size, &size) != TM_OK) return tm_lua_fail(L);
  return 0;
}

static int tm_lua_restore(lua_State *L) {
  lua_settop(L, 2);
  tm_machine *m = tm_lua_check(L, 1);
  tk_cvec_t *cp = tk_cvec_peek(L, 2, "checkpoint");
  if (tm_restore(m, (const uint8_t *)cp->a, cp->n) != TM_OK) return tm_lua_fail(L);
  return 0;
}

/* ---- reconfigure / restrict / type / destroy ---------------------------- */
static int tm_lua_reconfigure(lua_State *L) {
  lua_settop(L, 2);
  tm_machine *m = tm_lua_check(L, 1);
  luaL_checktype(L, 2, LUA_TTABLE);
  tm_reconfig r;
  r.clauses = tm_lua_unsigned(L, 2, "reconfigure", "clauses", 1, 0);
  r.clause_tolerance = tm_lua_unsigned(L, 2, "reconfigure", "clause_tolerance", 1, 0);
  r.clause_maximum = tm_lua_unsigned(L, 2, "reconfigure", "clause_maximum", 1, 0);
  r.include_bits = tm_lua_has(L, 2, "include_bits")
                       ? (int64_t)tm_lua_unsigned(L, 2, "reconfigure", "include_bits", 1, 0)
                       : -1;
  r.target = tm_lua_number(L, 2, "reconfigure", "target", 0, -1.0);
  r.specificity = tm_lua_number(L, 2, "reconfigure", "specificity", 1, 0.0);
  if (tm_reconfigure(m, &r) != TM_OK) return tm_lua_fail(L);
  return 0;
}

static int tm_lua_restrict(lua_State *L) {
  lua_settop(L, 2);
  tm_machine *m = tm_lua_check(L, 1);
  tk_ivec_t *dims = tk_ivec_peek(L, 2, "selected_dims");
  if (tm_restrict(m, dims->a, dims->n) != TM_OK) return tm_lua_fail(L);
  return 0;
}

static int tm_lua_type(lua_State *L) {
  tm_machine *m = tm_lua_check(L, 1);
  lua_pushstring(L, tm_type(m) == TM_CLASSIFIER ? "classifier" : "encoder");
  return 1;
}

static int tm_lua_destroy(lua_State *L) {
  tm_lua_box *b = (tm_lua_box *)luaL_checkudata(L, 1, TM_LUA_MT);
  if (b->m) tm_destroy(b->m);
  b->m = NULL;
  return 0;
}

static const luaL_Reg tm_lua_methods[] = {
    {"train", tm_lua_train},         {"predict", tm_lua_predict},
    {"destroy", tm_lua_destroy},     {"restrict", tm_lua_restrict},
    {"persist", tm_lua_persist},     {"checkpoint", tm_lua_checkpoint},
    {"restore", tm_lua_restore},     {"reconfigure", tm_lua_reconfigure},
    {"type", tm_lua_type},           {NULL, NULL},
};

static const luaL_Reg tm_lua_fns[] = {
    {"create", tm_lua_create},
    {"load", tm_lua_load},
    {NULL, NULL},
};

int luaopen_santoku_tsetlin_capi(lua_State *L) {
  if (luaL_newmetatable(L, TM_LUA_MT)) {
    lua_newtable(L);
    tm_lua_setfuncs(L, tm_lua_methods);
    lua_setfield(L, -2, "__index");
    lua_pushcfunction(L, tm_lua_destroy);
    lua_setfield(L, -2, "__gc");
  }
  lua_pop(L, 1);
  lua_newtable(L);
  tm_lua_setfuncs(L, tm_lua_fns);
  lua_pushinteger(L, (lua_Integer)tm_align());
  lua_setfield(L, -2, "align");
  return 1;
}
