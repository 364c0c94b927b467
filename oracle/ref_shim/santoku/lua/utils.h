/*
 * Minimal stand-ins for the santoku rock's Lua helper declarations, so that
 * the reference's lib/santoku/tsetlin/capi.c compiles as plain C for the
 * reference-code harness (ref_harness.c).  TEST INFRASTRUCTURE ONLY.
 *
 * Only the arithmetic of capi.c is exercised.  Every Lua entry point below
 * aborts if reached: the harness drives the reference's static functions
 * directly and never goes through the Lua bindings.
 */
#ifndef TM_REF_SHIM_LUA_UTILS_H
#define TM_REF_SHIM_LUA_UTILS_H

#include <math.h>
#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <santoku/cvec.h>

typedef struct lua_State lua_State;
typedef int (*lua_CFunction)(lua_State *);
typedef struct luaL_Reg { const char *name; lua_CFunction func; } luaL_Reg;

#define LUA_TNIL 0
#define LUA_TBOOLEAN 1

static inline void tm_shim_unreachable(const char *f) {
  fprintf(stderr, "reference shim: %s is not available in the harness\n", f);
  abort();
}

static inline void lua_getfield(lua_State *L, int i, const char *k) { (void)L; (void)i; (void)k; tm_shim_unreachable("lua_getfield"); }
static inline void lua_pop(lua_State *L, int n) { (void)L; (void)n; tm_shim_unreachable("lua_pop"); }
static inline void lua_settop(lua_State *L, int n) { (void)L; (void)n; tm_shim_unreachable("lua_settop"); }
static inline int lua_type(lua_State *L, int i) { (void)L; (void)i; tm_shim_unreachable("lua_type"); return 0; }
static inline int lua_toboolean(lua_State *L, int i) { (void)L; (void)i; tm_shim_unreachable("lua_toboolean"); return 0; }
static inline void lua_pushinteger(lua_State *L, long long v) { (void)L; (void)v; tm_shim_unreachable("lua_pushinteger"); }
static inline const char *lua_tostring(lua_State *L, int i) { (void)L; (void)i; tm_shim_unreachable("lua_tostring"); return NULL; }
static inline void lua_pushvalue(lua_State *L, int i) { (void)L; (void)i; tm_shim_unreachable("lua_pushvalue"); }
static inline int lua_pcall(lua_State *L, int a, int r, int e) { (void)L; (void)a; (void)r; (void)e; tm_shim_unreachable("lua_pcall"); return 0; }
static inline void lua_remove(lua_State *L, int i) { (void)L; (void)i; tm_shim_unreachable("lua_remove"); }
static inline void lua_insert(lua_State *L, int i) { (void)L; (void)i; tm_shim_unreachable("lua_insert"); }
static inline void lua_pushstring(lua_State *L, const char *s) { (void)L; (void)s; tm_shim_unreachable("lua_pushstring"); }
static inline void lua_setfield(lua_State *L, int i, const char *k) { (void)L; (void)i; (void)k; tm_shim_unreachable("lua_setfield"); }
static inline void lua_pushlstring(lua_State *L, const char *s, size_t n) { (void)L; (void)s; (void)n; tm_shim_unreachable("lua_pushlstring"); }
static inline void lua_newtable(lua_State *L) { (void)L; tm_shim_unreachable("lua_newtable"); }
static inline void *luaL_checkudata(lua_State *L, int i, const char *t) { (void)L; (void)i; (void)t; tm_shim_unreachable("luaL_checkudata"); return NULL; }
static inline const char *luaL_checkstring(lua_State *L, int i) { (void)L; (void)i; tm_shim_unreachable("luaL_checkstring"); return NULL; }
static inline const char *luaL_checklstring(lua_State *L, int i, size_t *n) { (void)L; (void)i; (void)n; tm_shim_unreachable("luaL_checklstring"); return NULL; }
static inline int luaL_error(lua_State *L, const char *fmt, ...) { (void)L; fprintf(stderr, "reference error: %s\n", fmt); abort(); return 0; }

static inline void tk_lua_verror(lua_State *L, int n, ...) { (void)L; (void)n; tm_shim_unreachable("tk_lua_verror"); }
static inline unsigned int tk_lua_fcheckunsigned(lua_State *L, int i, const char *c, const char *f) { (void)L; (void)i; (void)c; (void)f; tm_shim_unreachable("tk_lua_fcheckunsigned"); return 0; }
static inline unsigned int tk_lua_foptunsigned(lua_State *L, int i, const char *c, const char *f, unsigned int d) { (void)L; (void)i; (void)c; (void)f; (void)d; tm_shim_unreachable("tk_lua_foptunsigned"); return 0; }
static inline double tk_lua_foptposdouble(lua_State *L, int i, const char *c, const char *f, double d) { (void)L; (void)i; (void)c; (void)f; (void)d; tm_shim_unreachable("tk_lua_foptposdouble"); return 0; }
static inline double tk_lua_fcheckposdouble(lua_State *L, int i, const char *c, const char *f) { (void)L; (void)i; (void)c; (void)f; tm_shim_unreachable("tk_lua_fcheckposdouble"); return 0; }
static inline bool tk_lua_foptboolean(lua_State *L, int i, const char *c, const char *f, bool d) { (void)L; (void)i; (void)c; (void)f; (void)d; tm_shim_unreachable("tk_lua_foptboolean"); return false; }
static inline int tk_lua_ftype(lua_State *L, int i, const char *f) { (void)L; (void)i; (void)f; tm_shim_unreachable("tk_lua_ftype"); return 0; }
static inline int tk_lua_absindex(lua_State *L, int i) { (void)L; (void)i; tm_shim_unreachable("tk_lua_absindex"); return 0; }
static inline unsigned int tk_lua_checkunsigned(lua_State *L, int i, const char *m) { (void)L; (void)i; (void)m; tm_shim_unreachable("tk_lua_checkunsigned"); return 0; }
static inline const char *tk_lua_checkstring(lua_State *L, int i, const char *m) { (void)L; (void)i; (void)m; tm_shim_unreachable("tk_lua_checkstring"); return NULL; }
static inline void tk_lua_register(lua_State *L, luaL_Reg *r, int n) { (void)L; (void)r; (void)n; tm_shim_unreachable("tk_lua_register"); }
#define tk_lua_newuserdata(L, T, mt, fns, gc) ((T *)(tm_shim_unreachable("tk_lua_newuserdata"), (void *)0))

/* Memory and stdio helpers: plain libc. */
static inline void *tk_malloc(lua_State *L, size_t n) { (void)L; return malloc(n ? n : 1); }
static inline void *tk_realloc(lua_State *L, void *p, size_t n) { (void)L; return realloc(p, n ? n : 1); }
static inline void *tk_malloc_aligned(lua_State *L, size_t n, size_t a) {
  (void)L;
  void *p = NULL;
  size_t al = a < sizeof(void *) ? sizeof(void *) : a;
  if (posix_memalign(&p, al, n ? n : 1)) return NULL;
  return p;
}
static inline void tk_lua_fwrite(lua_State *L, const void *p, size_t s, size_t n, FILE *f) { (void)L; if (fwrite(p, s, n, f) != n) tm_shim_unreachable("fwrite"); }
static inline void tk_lua_fread(lua_State *L, void *p, size_t s, size_t n, FILE *f) { (void)L; if (fread(p, s, n, f) != n) tm_shim_unreachable("fread"); }
static inline FILE *tk_lua_fopen(lua_State *L, const char *p, const char *m) { (void)L; return fopen(p, m); }
static inline void tk_lua_fclose(lua_State *L, FILE *f) { (void)L; fclose(f); }
static inline FILE *tk_lua_tmpfile(lua_State *L) { (void)L; return tmpfile(); }
static inline FILE *tk_lua_fmemopen(lua_State *L, char *d, size_t n, const char *m) { (void)L; return fmemopen(d, n, m); }
static inline char *tk_lua_fslurp(lua_State *L, FILE *f, size_t *len) {
  (void)L;
  long end = ftell(f);
  char *d = malloc(end > 0 ? (size_t)end : 1);
  rewind(f);
  *len = fread(d, 1, (size_t)end, f);
  return d;
}

/* The reference's generator lives in the un-vendored santoku rock; the
 * harness supplies these (ref_harness.c). */
static void tk_fast_seed(uint64_t s);
static uint64_t tk_fast_random(void);
static bool tk_fast_chance(double p);

#endif
