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
    return (m >= 0x1p-60f && m <= 0x1p60f) || a == 0.0f;
}

__device__ __forceinline__ float fpdiv_step(float a, float b, float y) {
    const float q = __fmul_rn(a, y);
    const float r = __fmaf_rn(-b, q, a);
    return a == 0.0f ? q : __fmaf_rn(r, y, q);
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
