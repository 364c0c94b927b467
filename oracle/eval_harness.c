/*
 * Evaluator harness.  TEST INFRASTRUCTURE ONLY, built only where the
 * reference tree exists (oracle/Makefile, target `ref`), output in _ref/.
 *
 * The reference's evaluator module (lib/santoku/tsetlin/evaluator/capi.c)
 * includes santoku's container headers and the graph, ANN and index code,
 * which are absent here; the two metrics the library computes on the device
 * -- tm_class_accuracy (evaluator/capi.c:119-202) and tm_encoding_accuracy
 * (:497-574) -- use none of that.  The Makefile copies those two functions
 * out of the reference file, as they lie, into _ref/eval_funcs.c at build
 * time (with #line directives back to the reference file), and this file
 * compiles them with the reference's own compiler flags against a small
 * stand-in for the Lua C API: arguments sit in a fake Lua stack, and the
 * tables the functions build are recorded so that their numbers can be read
 * back.  Nothing else of the reference is compiled here.
 *
 *   ref_eval_class_accuracy(pred, expected, n, classes, out[3 + 3 classes])
 *     out = precision, recall, f1, then (precision, recall, f1) per class
 *   ref_eval_encoding_accuracy(pred, expected, n, hidden, out[4 + hidden])
 *     out = mean_hamming, ber_min, ber_max, ber_std, then the per-bit rates
 */
#include <math.h>
#include <stdarg.h>
#include <stdatomic.h>
#include <stdbool.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ---- santoku-matrix vectors (the fields the two functions read) -------- */
#define TK_CVEC_BITS 8
#define TK_CVEC_BITS_BYTES(n) (((n) + TK_CVEC_BITS - 1) / TK_CVEC_BITS)
#define TK_CVEC_BITS_BYTE(n) ((n) / TK_CVEC_BITS)
#define TK_CVEC_BITS_BIT(n) ((n) % TK_CVEC_BITS)

typedef struct { size_t n; size_t m; char *a; } tk_cvec_t;
typedef struct { size_t n; size_t m; int64_t *a; } tk_ivec_t;

/* ---- a stand-in Lua state ----------------------------------------------- */
enum { EV_NIL, EV_NUM, EV_INT, EV_PTR, EV_TAB };

typedef struct {
  int kind;
  double num;
  int64_t ival;
  void *ptr;
  int tab;
} ev_slot;

/* A table: named number fields, and integer keys 1..n holding numbers or
 * tables. */
#define EV_FIELDS 8
typedef struct {
  const char *name[EV_FIELDS];
  ev_slot field[EV_FIELDS];
  int nfield;
  ev_slot *item;
  int64_t nitem;
} ev_table;

#define EV_STACK 32
typedef struct lua_State {
  ev_slot st[EV_STACK];
  int top;
  ev_table *tab;
  int ntab, captab;
  void *udata[4];
  int nudata;
} lua_State;

static void ev_die(const char *what) {
  fprintf(stderr, "evaluator harness: %s\n", what);
  abort();
}

static ev_slot *ev_at(lua_State *L, int i) {
  const int k = i > 0 ? i - 1 : L->top + i;
  if (k < 0 || k >= L->top) ev_die("stack index out of range");
  return &L->st[k];
}

static void ev_push(lua_State *L, ev_slot s) {
  if (L->top >= EV_STACK) ev_die("stack overflow");
  L->st[L->top++] = s;
}

static void lua_settop(lua_State *L, int n) {
  while (L->top < n) ev_push(L, (ev_slot){.kind = EV_NIL});
  L->top = n;
}

static void lua_newtable(lua_State *L) {
  if (L->ntab == L->captab) {
    L->captab = L->captab ? 2 * L->captab : 16;
    L->tab = realloc(L->tab, (size_t)L->captab * sizeof(ev_table));
    if (!L->tab) ev_die("out of memory");
  }
  memset(&L->tab[L->ntab], 0, sizeof(ev_table));
  ev_push(L, (ev_slot){.kind = EV_TAB, .tab = L->ntab++});
}

static void lua_pushnumber(lua_State *L, double v) { ev_push(L, (ev_slot){.kind = EV_NUM, .num = v}); }

static void lua_pushinteger(lua_State *L, int64_t v) {
  ev_push(L, (ev_slot){.kind = EV_INT, .ival = v});
}

static void *lua_newuserdata(lua_State *L, size_t n) {
  if (L->nudata == 4) ev_die("too many userdata");
  void *p = malloc(n ? n : 1);
  if (!p) ev_die("out of memory");
  L->udata[L->nudata++] = p;
  ev_push(L, (ev_slot){.kind = EV_PTR, .ptr = p});
  return p;
}

static ev_table *ev_table_at(lua_State *L, int i) {
  ev_slot *s = ev_at(L, i);
  if (s->kind != EV_TAB) ev_die("not a table");
  return &L->tab[s->tab];
}

static void lua_setfield(lua_State *L, int i, const char *k) {
  ev_table *t = ev_table_at(L, i);
  if (t->nfield == EV_FIELDS) ev_die("too many fields");
  t->name[t->nfield] = k;
  t->field[t->nfield++] = L->st[L->top - 1];
  L->top--;
}

static void lua_settable(lua_State *L, int i) {
  ev_table *t = ev_table_at(L, i);
  const ev_slot key = L->st[L->top - 2], val = L->st[L->top - 1];
  if (key.kind != EV_INT || key.ival != t->nitem + 1) ev_die("keys must be 1, 2, ...");
  t->item = realloc(t->item, (size_t)(t->nitem + 1) * sizeof(ev_slot));
  if (!t->item) ev_die("out of memory");
  t->item[t->nitem++] = val;
  L->top -= 2;
}

static void lua_replace(lua_State *L, int i) {
  *ev_at(L, i) = L->st[L->top - 1];
  L->top--;
}

/* ---- the santoku helpers the two functions call -------------------------- */
static tk_ivec_t *tk_ivec_peek(lua_State *L, int i, const char *name) {
  (void)name;
  return (tk_ivec_t *)ev_at(L, i)->ptr;
}

static tk_cvec_t *tk_cvec_peekopt(lua_State *L, int i) { return (tk_cvec_t *)ev_at(L, i)->ptr; }

static const char *tk_lua_checkustring(lua_State *L, int i, const char *name) {
  (void)L, (void)i, (void)name;
  ev_die("string arguments are not staged by this harness");
  return NULL;
}

static uint64_t tk_lua_checkunsigned(lua_State *L, int i, const char *name) {
  (void)name;
  ev_slot *s = ev_at(L, i);
  if (s->kind != EV_INT || s->ival < 0) ev_die("expected an unsigned integer");
  return (uint64_t)s->ival;
}

static void tk_lua_verror(lua_State *L, int n, ...) {
  (void)L, (void)n;
  ev_die("the reference raised an argument error");
}

static void *tk_malloc(lua_State *L, size_t n) {
  (void)L;
  void *p = malloc(n ? n : 1);
  if (!p) ev_die("out of memory");
  return p;
}

#include TM_REF_EVAL

/* ---- entry points ---------------------------------------------------------- */
static void ev_open(lua_State *L) { memset(L, 0, sizeof *L); }

static void ev_close(lua_State *L) {
  for (int i = 0; i < L->ntab; i++) free(L->tab[i].item);
  free(L->tab);
  for (int i = 0; i < L->nudata; i++) free(L->udata[i]);
}

static double ev_field(const ev_table *t, const char *k) {
  for (int i = 0; i < t->nfield; i++)
    if (!strcmp(t->name[i], k)) {
      if (t->field[i].kind != EV_NUM) ev_die("field is not a number");
      return t->field[i].num;
    }
  ev_die("field missing");
  return 0;
}

static const ev_table *ev_subtable(const lua_State *L, const ev_table *t, const char *k) {
  for (int i = 0; i < t->nfield; i++)
    if (!strcmp(t->name[i], k) && t->field[i].kind == EV_TAB) return &L->tab[t->field[i].tab];
  ev_die("table field missing");
  return NULL;
}

int ref_eval_class_accuracy(const int64_t *pred, const int64_t *expected, uint32_t n,
                            uint32_t classes, double *out) {
  lua_State L;
  ev_open(&L);
  tk_ivec_t p = {n, n, (int64_t *)pred}, e = {n, n, (int64_t *)expected};
  ev_push(&L, (ev_slot){.kind = EV_PTR, .ptr = &p});
  ev_push(&L, (ev_slot){.kind = EV_PTR, .ptr = &e});
  lua_pushinteger(&L, n);
  lua_pushinteger(&L, classes);
  tm_class_accuracy(&L);
  const ev_table *r = ev_table_at(&L, 1);
  out[0] = ev_field(r, "precision");
  out[1] = ev_field(r, "recall");
  out[2] = ev_field(r, "f1");
  const ev_table *cls = ev_subtable(&L, r, "classes");
  if (cls->nitem != classes) ev_die("class count");
  for (uint32_t c = 0; c < classes; c++) {
    if (cls->item[c].kind != EV_TAB) ev_die("class entry");
    const ev_table *t = &L.tab[cls->item[c].tab];
    out[3 + 3 * c] = ev_field(t, "precision");
    out[4 + 3 * c] = ev_field(t, "recall");
    out[5 + 3 * c] = ev_field(t, "f1");
  }
  ev_close(&L);
  return 0;
}

int ref_eval_encoding_accuracy(const uint8_t *pred, const uint8_t *expected, uint32_t n,
                               uint32_t hidden, double *out) {
  lua_State L;
  ev_open(&L);
  const size_t bytes = (size_t)n * TK_CVEC_BITS_BYTES(hidden);
  tk_cvec_t p = {bytes, bytes, (char *)pred}, e = {bytes, bytes, (char *)expected};
  ev_push(&L, (ev_slot){.kind = EV_PTR, .ptr = &p});
  ev_push(&L, (ev_slot){.kind = EV_PTR, .ptr = &e});
  lua_pushinteger(&L, n);
  lua_pushinteger(&L, hidden);
  tm_encoding_accuracy(&L);
  const ev_table *r = ev_table_at(&L, 1);
  out[0] = ev_field(r, "mean_hamming");
  out[1] = ev_field(r, "ber_min");
  out[2] = ev_field(r, "ber_max");
  out[3] = ev_field(r, "ber_std");
  const ev_table *bits = ev_subtable(&L, r, "bits");
  if (bits->nitem != hidden) ev_die("bit count");
  for (uint32_t j = 0; j < hidden; j++) {
    if (bits->item[j].kind != EV_NUM) ev_die("bit entry");
    out[4 + j] = bits->item[j].num;
  }
  ev_close(&L);
  return 0;
}
