// Semirings of the QDB scan kernels and the reference's child fold orders.
//
// CYK: f32 adds with __fadd_rn (no contraction) and the reference's max
// `a >= b ? a : b` (src/cm_nohmm.rs:108-114).  Inside: i32 wrapping adds and
// ILogsum (src/cp9.rs:65-75) from a u16 table in shared memory.
// reduce_c follows reduce_c_order (src/cm_nohmm.rs:187-242): the integer
// ILogsum fold is not associative, so the order is the reference's.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace cmx {
namespace dev {

constexpr int INFTY_D = 987654321;
constexpr float IMPOSSIBLE_D = -1.0e36f;

template <bool INS>
struct Sem;

template <>
struct Sem<false> {  // CYK: f32, ESL_MAX
    typedef float T;
    static constexpr bool ORDERED = false;
    __device__ static __forceinline__ T zero() { return IMPOSSIBLE_D; }
    __device__ static __forceinline__ T add(T a, T b) { return __fadd_rn(a, b); }
    __device__ static __forceinline__ T comb(T a, T b, const uint16_t *, int) { return a >= b ? a : b; }
    __device__ static __forceinline__ T ld(const uint32_t *p) { return __uint_as_float(*p); }
    __device__ static __forceinline__ T ldg(const uint32_t *p) { return __uint_as_float(__ldg(p)); }
    __device__ static __forceinline__ void st(uint32_t *p, T x) { *p = __float_as_uint(x); }
    __device__ static __forceinline__ uint32_t u(T x) { return __float_as_uint(x); }
    __device__ static __forceinline__ float bits(T x) { return x; }
};

template <>
struct Sem<true> {  // Inside: i32 wrapping adds, ILogsum
    typedef int32_t T;
    static constexpr bool ORDERED = true;
    __device__ static __forceinline__ T zero() { return -INFTY_D; }
    __device__ static __forceinline__ T add(T a, T b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
    // ILogsum (src/cp9.rs:65-75): max + tbl[max-min], written without
    // branches.  The table is stored up to its last nonzero entry plus one
    // zero entry, tbl[nz] = 0; the two cases where the rule adds nothing --
    // min at or below -INFTY, and max-min >= LOGSUM_TBL (beyond nz the table
    // is 0 anyway) -- index that zero entry.
    __device__ static __forceinline__ T comb(T a, T b, const uint16_t *tbl, int nz) {
        const int32_t mx = max(max(a, b), -INFTY_D);
        const int32_t mn = min(a, b);
        const uint32_t diff = (uint32_t)mx - (uint32_t)mn;
        const uint32_t idx = mn <= -INFTY_D ? (uint32_t)nz : min(diff, (uint32_t)nz);
        return (int32_t)((uint32_t)mx + (uint32_t)tbl[idx]);
    }
    __device__ static __forceinline__ T ld(const uint32_t *p) { return (int32_t)*p; }
    __device__ static __forceinline__ T ldg(const uint32_t *p) { return (int32_t)__ldg(p); }
    __device__ static __forceinline__ void st(uint32_t *p, T x) { *p = (uint32_t)x; }
    __device__ static __forceinline__ uint32_t u(T x) { return (uint32_t)x; }
    __device__ static __forceinline__ float bits(T x) {
        return x == -INFTY_D ? IMPOSSIBLE_D : (float)((double)x / 1000.0);
    }
};

template <class S>
__device__ __forceinline__ typename S::T reduce_c(int cnum, const typename S::T *t, typename S::T init,
                                                  const uint16_t *tb, int nz) {
    typedef typename S::T T;
    T s;
    if (!S::ORDERED) {
        // CYK: max selects one operand exactly, so any bracketing returns the
        // same value; a tree shortens the dependency chain.
        T a = init, b = cnum > 0 ? t[0] : init, c = cnum > 1 ? t[1] : init;
        T d = cnum > 2 ? t[2] : init, e = cnum > 3 ? t[3] : init, f = cnum > 4 ? t[4] : init;
        T g = cnum > 5 ? t[5] : init;
        T ab = S::comb(a, b, tb, nz), cd = S::comb(c, d, tb, nz), ef = S::comb(e, f, tb, nz);
        return S::comb(S::comb(ab, cd, tb, nz), S::comb(ef, g, tb, nz), tb, nz);
    }
    switch (cnum) {
    case 1: s = S::comb(init, t[0], tb, nz); break;
    case 2: s = S::comb(S::comb(t[1], init, tb, nz), t[0], tb, nz); break;
    case 3: s = S::comb(S::comb(S::comb(t[2], t[1], tb, nz), init, tb, nz), t[0], tb, nz); break;
    case 4:
        s = S::comb(t[3], t[2], tb, nz);
        s = S::comb(s, init, tb, nz);
        s = S::comb(s, t[1], tb, nz);
        s = S::comb(s, t[0], tb, nz);
        break;
    case 5:
        s = S::comb(t[4], t[3], tb, nz);
        s = S::comb(s, init, tb, nz);
        s = S::comb(s, t[1], tb, nz);
        s = S::comb(s, t[2], tb, nz);
        s = S::comb(s, t[0], tb, nz);
        break;
    case 6:
        s = S::comb(t[5], init, tb, nz);
        s = S::comb(s, t[4], tb, nz);
        s = S::comb(s, t[3], tb, nz);
        s = S::comb(s, t[2], tb, nz);
        s = S::comb(s, t[1], tb, nz);
        s = S::comb(s, t[0], tb, nz);
        break;
    default:  // cnum is 1..6 for every non-B, non-E state of a CM
        s = init;
    }
    return s;
}

// reduce_c_order with the self term t[0] left out: the IL step is then
// comb(c, x + t0) (t[0] is combined last for every cnum).
template <class S>
__device__ __forceinline__ typename S::T reduce_c_noself(int cnum, const typename S::T *t, typename S::T init,
                                                         const uint16_t *tb, int nz) {
    typedef typename S::T T;
    T s;
    switch (cnum) {
    case 1: s = init; break;
    case 2: s = S::comb(t[1], init, tb, nz); break;
    case 3: s = S::comb(S::comb(t[2], t[1], tb, nz), init, tb, nz); break;
    case 4:
        s = S::comb(t[3], t[2], tb, nz);
        s = S::comb(s, init, tb, nz);
        s = S::comb(s, t[1], tb, nz);
        break;
    case 5:
        s = S::comb(t[4], t[3], tb, nz);
        s = S::comb(s, init, tb, nz);
        s = S::comb(s, t[1], tb, nz);
        s = S::comb(s, t[2], tb, nz);
        break;
    case 6:
        s = S::comb(t[5], init, tb, nz);
        s = S::comb(s, t[4], tb, nz);
        s = S::comb(s, t[3], tb, nz);
        s = S::comb(s, t[2], tb, nz);
        s = S::comb(s, t[1], tb, nz);
        break;
    default:  // cnum is 1..6 for every non-B, non-E state of a CM
        s = init;
    }
    return s;
}

}  // namespace dev
}  // namespace cmx
