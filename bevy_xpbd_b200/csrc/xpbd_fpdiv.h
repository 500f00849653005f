// Three correctly rounded quotients a_k / b sharing one divisor, from one correctly rounded reciprocal.
//
// Method (Markstein's theorem, P. Markstein, "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Develop. 34(1), 1990; also Muller et al., Handbook of Floating-Point Arithmetic, ch. 4):
// with y = RN(1/b) and q = RN(a·y) (within one ulp of a/b), the remainder r = a − b·q is exactly representable and
// one fused multiply-add gives it exactly; then RN(q + r·y) = RN(a/b). The three quotients therefore cost one
// reciprocal and three multiply + two FMA steps instead of three divisions, bit-identical to a / b.
//
// The theorem needs every value in the normal range. The fast path is taken when 2^-60 <= |b| <= 2^60 and each a is
// zero or 2^-60 <= |a| (then q, y and r stay far from underflow and overflow); anything else — tiny or huge
// operands, infinities, NaN — goes through the ordinary division. A zero numerator returns q = a·y, which carries
// the sign rule of a / b. `xpbd_selftest_division` compares this against the division on random operands.
#pragma once
#include <cuda_runtime.h>

namespace xpbd {

__device__ __forceinline__ bool fpdiv_num_ok(float a) {
    const float m = fabsf(a);
    return ((m >= 0x1p-60f) & (m <= 0x1p60f)) | (a == 0.0f);
}

__device__ __forceinline__ float fpdiv_step(float a, float b, float y) {
    const float q = __fmul_rn(a, y);
    const float r = __fmaf_rn(-b, q, a);
    return a == 0.0f ? q : __fmaf_rn(r, y, q);
}

// The shared-reciprocal quotients for the components of a vector divided by its own computed length b = |a| (so
// |a_k| <= b·(1 + 2^-23) and no quotient can overflow), without a fallback branch: returns whether they are the
// correctly rounded ones, so the caller recomputes the rare failing case with fpdiv3. The range test reduces to
// 2^-60 <= b <= 2^60 and every a_k zero or >= 2^-60 in magnitude, evaluated on the bit patterns — (bits << 1) - 1
// wraps zero to the top, so one unsigned minimum over the three components tests "zero or exponent >= 67" at once.
__device__ __forceinline__ bool fpdiv3_by_length_fast(float ax, float ay, float az, float b, float& qx, float& qy,
                                                      float& qz) {
    const float y = __frcp_rn(b);
    qx = fpdiv_step(ax, b, y);
    qy = fpdiv_step(ay, b, y);
    qz = fpdiv_step(az, b, y);
    const uint32_t mx = (__float_as_uint(ax) << 1) - 1u, my = (__float_as_uint(ay) << 1) - 1u,
                   mz = (__float_as_uint(az) << 1) - 1u;
    const uint32_t mn = min(mx, min(my, mz));
    const bool b_ok = ((__float_as_uint(b) & 0x7FFFFFFFu) - (67u << 23)) < (120u << 23);  // 2^-60 <= |b| < 2^60
    return b_ok & (mn >= (67u << 24) - 1u);
}

// The bare shared-reciprocal quotients, for callers that have established the theorem's conditions beforehand. The
// Jacobi row kernel does so once per pass for the whole grid: when every coordinate of every particle is 0 or has a
// magnitude in [2^-37, 2^58] (see coord_outside_fast_range), every nonzero difference of two coordinates is a
// multiple of 2^-60 (so |a_k| >= 2^-60), every length of a used term is in [1e-8, 2^60), and the quotients are in
// [2^-120, 1 + 2^-23] — all normal, so the result is RN(a_k / b).
// A zero numerator gives a zero of either sign here (the remainder step runs for it too, saving the select): RN(a_k / b)
// up to the sign of a zero. Its caller multiplies the quotient into a term that is added to a sum started at +0, where
// a zero of either sign leaves the sum unchanged, so the result is the same bits.
__device__ __forceinline__ void fpdiv3_unchecked(float ax, float ay, float az, float b, float& qx, float& qy,
                                                 float& qz) {
    const float y = __frcp_rn(b);
    const float px = __fmul_rn(ax, y), py = __fmul_rn(ay, y), pz = __fmul_rn(az, y);
    qx = __fmaf_rn(__fmaf_rn(-b, px, ax), y, px);
    qy = __fmaf_rn(__fmaf_rn(-b, py, ay), y, py);
    qz = __fmaf_rn(__fmaf_rn(-b, pz, az), y, pz);
}

// True when a coordinate breaks the fpdiv3_unchecked invariant: nonzero and below 2^-37 in magnitude, above 2^58,
// or not a number.
__device__ __forceinline__ bool coord_outside_fast_range(float c) {
    const float m = fabsf(c);
    return ((m < 0x1p-37f) & (m != 0.0f)) | !(m <= 0x1p58f);
}

// {ax, ay, az} / b with y = RN(1/b) computed beforehand (2^-60 <= b <= 2^60, e.g. a constraint count), each
// correctly rounded: the shared-reciprocal steps when the numerators pass the range test, else the division.
__device__ __forceinline__ void fpdiv3_rcp(float ax, float ay, float az, float b, float y, float& qx, float& qy,
                                           float& qz) {
    if (fpdiv_num_ok(ax) && fpdiv_num_ok(ay) && fpdiv_num_ok(az)) {
        qx = fpdiv_step(ax, b, y);
        qy = fpdiv_step(ay, b, y);
        qz = fpdiv_step(az, b, y);
    } else {
        qx = __fdiv_rn(ax, b);
        qy = __fdiv_rn(ay, b);
        qz = __fdiv_rn(az, b);
    }
}

// {ax, ay, az} / b, each correctly rounded.
__device__ __forceinline__ void fpdiv3(float ax, float ay, float az, float b, float& qx, float& qy, float& qz) {
    const float mb = fabsf(b);
    if (mb >= 0x1p-60f && mb <= 0x1p60f && fpdiv_num_ok(ax) && fpdiv_num_ok(ay) && fpdiv_num_ok(az)) {
        const float y = __frcp_rn(b);
        qx = fpdiv_step(ax, b, y);
        qy = fpdiv_step(ay, b, y);
        qz = fpdiv_step(az, b, y);
    } else {
        qx = __fdiv_rn(ax, b);
        qy = __fdiv_rn(ay, b);
        qz = __fdiv_rn(az, b);
    }
}

}  // namespace xpbd
