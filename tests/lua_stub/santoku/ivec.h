/* Declarations of the santoku-matrix int64-vector accessors the binding
 * uses, with the argument lists of their call sites in the reference
 * (lib/santoku/tsetlin/capi.c:1120, 1293, 754).  Test infrastructure only. */
#ifndef TM_TEST_SANTOKU_IVEC_H
#define TM_TEST_SANTOKU_IVEC_H
#include <stddef.h>
#include <stdint.h>
#include "lua.h"

typedef struct { size_t n; size_t m; int64_t *a; } tk_ivec_t;

tk_ivec_t *tk_ivec_peek(lua_State *L, int i, const char *name);
tk_ivec_t *tk_ivec_create(lua_State *L, size_t n, int64_t *data, tk_ivec_t *src);
#endif
