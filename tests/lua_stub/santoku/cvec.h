/* Declarations of the santoku-matrix byte-vector accessors the binding uses,
 * with the argument lists of their call sites in the reference
 * (lib/santoku/tsetlin/capi.c:1083, 1118, 1568-1572).  santoku-matrix is not
 * installed here; test infrastructure only. */
#ifndef TM_TEST_SANTOKU_CVEC_H
#define TM_TEST_SANTOKU_CVEC_H
#include <stddef.h>
#include <stdint.h>
#include "lua.h"

#define TK_CVEC_BITS 8
typedef struct { size_t n; size_t m; char *a; } tk_cvec_t;

tk_cvec_t *tk_cvec_peek(lua_State *L, int i, const char *name);
tk_cvec_t *tk_cvec_create(lua_State *L, size_t n, char *data, tk_cvec_t *src);
int tk_cvec_ensure(tk_cvec_t *v, size_t n);
#endif
