/*
 * Stand-ins for the santoku-matrix vector declarations used by the
 * reference's capi.c / automata.h (reference-code harness only).
 */
#ifndef TM_REF_SHIM_CVEC_H
#define TM_REF_SHIM_CVEC_H

#include <stdint.h>
#include <stddef.h>

#define TK_CVEC_BITS 8
#define TK_CVEC_BITS_BYTES(n) (((n) + TK_CVEC_BITS - 1) / TK_CVEC_BITS)
#define TK_CVEC_BITS_BYTE(n) ((n) / TK_CVEC_BITS)
#define TK_CVEC_BITS_BIT(n) ((n) % TK_CVEC_BITS)

typedef struct lua_State lua_State;

typedef struct { size_t n; size_t m; char *a; } tk_cvec_t;
typedef struct { size_t n; size_t m; int64_t *a; } tk_ivec_t;

void tm_shim_abort(const char *f);
#define tk_cvec_peek(L, i, name) ((tk_cvec_t *)(tm_shim_abort("tk_cvec_peek"), (void *)0))
#define tk_ivec_peek(L, i, name) ((tk_ivec_t *)(tm_shim_abort("tk_ivec_peek"), (void *)0))
#define tk_cvec_create(L, n, a, b) ((tk_cvec_t *)(tm_shim_abort("tk_cvec_create"), (void *)0))
#define tk_ivec_create(L, n, a, b) ((tk_ivec_t *)(tm_shim_abort("tk_ivec_create"), (void *)0))
#define tk_cvec_ensure(v, n) (tm_shim_abort("tk_cvec_ensure"), 0)

/* santoku-matrix's bit helper, restated from its use at capi.c:103-109:
 * over the first `bits` bits, *pa = popcount(a), *pn = popcount(a & ~b). */
static inline void tk_cvec_bits_popcount_andnot_serial(const uint8_t *a, const uint8_t *b,
                                                       uint64_t bits, uint64_t *pa,
                                                       uint64_t *pn) {
  uint64_t la = 0, ln = 0, nb = bits / 8;
  for (uint64_t i = 0; i < nb; i++) {
    la += (uint64_t)__builtin_popcount(a[i]);
    ln += (uint64_t)__builtin_popcount((uint8_t)(a[i] & ~b[i]));
  }
  if (bits % 8) {
    uint8_t m = (uint8_t)((1u << (bits % 8)) - 1);
    la += (uint64_t)__builtin_popcount(a[nb] & m);
    ln += (uint64_t)__builtin_popcount((uint8_t)(a[nb] & ~b[nb] & m));
  }
  *pa = la;
  *pn = ln;
}

#endif
