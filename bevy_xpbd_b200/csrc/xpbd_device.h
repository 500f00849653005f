// Device helpers shared by the solver kernels: the reference's FP32 vector operations with correctly rounded
// intrinsics (no contraction into FMA), the safety clamps, predict and the post-velocity update.
//   clamp_correction   xpbd_cpu.rs:28-36
//   predict_particle   xpbd_cpu.rs:38-65     (WGSL predict_copy_sim_to_jac, cloth_sim_jacobi.wgsl:85-121)
//   finalize_particle  xpbd_cpu.rs:393-409   (WGSL post_velocity :220-233)
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "xpbd_fpdiv.h"
#include "xpbd_internal.h"

namespace xpbd {

constexpr float kCorrectionCap = 0.28f;  // JACOBI_CORRECTION_CAP, cloth_compute.rs:82
constexpr float kMaxSpeed = 12.0f;       // PREDICT_MAX_SPEED, cloth_compute.rs:84
constexpr float kGrabMaxPull = 0.065f;   // GRAB_MAX_PULL_PER_SUBSTEP, cloth_compute.rs:86
constexpr unsigned kFull = 0xFFFFFFFFu;

struct F3 {
    float x, y, z;
};
__device__ __forceinline__ F3 f3(float4 a) { return {a.x, a.y, a.z}; }
__device__ __forceinline__ F3 add3(F3 a, F3 b) { return {__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)}; }
__device__ __forceinline__ F3 sub3(F3 a, F3 b) { return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)}; }
__device__ __forceinline__ F3 mul3(F3 a, float s) { return {__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s)}; }
__device__ __forceinline__ F3 div3(F3 a, float s) {  // correctly rounded, one shared reciprocal (xpbd_fpdiv.h)
    F3 q;
    fpdiv3(a.x, a.y, a.z, s, q.x, q.y, q.z);
    return q;
}
__device__ __forceinline__ F3 neg3(F3 a) { return {-a.x, -a.y, -a.z}; }
// glam dot: (x*x' + y*y') + z*z'; length = sqrt(dot)
__device__ __forceinline__ float dot3(F3 a, F3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ float len3(F3 a) { return __fsqrt_rn(dot3(a, a)); }
__device__ __forceinline__ bool finite3(F3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }

// Compliance of incidence k: the cloth's palette entry named by the record's top four bits, or, when some cloth of
// the batch has more than 16 distinct compliance values, the per-incidence array.
__device__ __forceinline__ float inc_compliance(const XpbdWorld& W, const float* pal, uint2 rec, uint32_t k) {
    return W.inc_comp ? W.inc_comp[k] : pal[rec.x >> 28];
}

__device__ __forceinline__ void set_status(int* status, int flag) {
    if ((*(volatile int*)status & flag) == 0) atomicOr(status, flag);
}

// clamp_correction, xpbd_cpu.rs:28-36. When |dx|² <= 0x3da0902d (the largest float not above 0.28f²), sqrt(|dx|²)
// <= 0.28f holds exactly, so the reference does not clamp and the square root can be skipped: same bits, cheaper.
__device__ __forceinline__ F3 clamp_correction(F3 dx) {
    const float d = dot3(dx, dx);
    if (d <= __uint_as_float(0x3da0902du)) return dx;
    const float ml = __fsqrt_rn(d);
    if (ml > kCorrectionCap && ml > 0.0f) return mul3(dx, __fdiv_rn(kCorrectionCap, ml));
    return dx;
}

// predict_particle, xpbd_cpu.rs:38-65 (callers handle inv_mass <= 0)
// `wind` (extension, may be null): after gravity, v += (wind − v) · (drag · dt).
__device__ __forceinline__ F3 predict_particle(uint32_t i, F3 sim, F3& vel, const XpbdDevParams& P,
                                               const XpbdWind* wind = nullptr) {
    F3 g = {P.gravity[0], P.gravity[1], P.gravity[2]};
    F3 v = add3(vel, mul3(g, P.dt));
    if (wind) v = add3(v, mul3(sub3(F3{wind->vel[0], wind->vel[1], wind->vel[2]}, v), __fmul_rn(wind->drag, P.dt)));
    const float v2 = dot3(v, v);
    if (v2 >= 144.0f) {  // below 12² the reference's speed = sqrt(v2) cannot exceed 12: skip the root
        const float speed = __fsqrt_rn(v2);
        if (speed > kMaxSpeed && speed > 0.0f) v = mul3(v, __fdiv_rn(kMaxSpeed, speed));
    }
    F3 pos = add3(sim, mul3(v, P.dt));
    if (P.grab_active != 0u && (int32_t)i == P.grab_idx) {
        F3 tgt = {P.grab_target[0], P.grab_target[1], P.grab_target[2]};
        F3 pull = mul3(sub3(tgt, pos), P.grab_stiffness);
        float pl = len3(pull);
        if (pl > kGrabMaxPull && pl > 0.0f) pull = mul3(pull, __fdiv_rn(kGrabMaxPull, pl));
        pos = add3(pos, pull);
    }
    vel = v;
    return pos;
}

// Per-cloth grab (extension of the reference's single grab, xpbd_cpu.rs:56-63): the same pull, applied after
// predict_particle to the cloth's grabbed vertex.
__device__ __forceinline__ F3 apply_cloth_grab(const XpbdWorld& W, uint32_t i, F3 pos) {
    if (*W.grab_count == 0u) return pos;
    const XpbdGrab g = W.grabs[W.row_cloth[i]];
    if (g.idx != (int32_t)i) return pos;
    F3 pull = mul3(sub3(F3{g.target[0], g.target[1], g.target[2]}, pos), g.stiffness);
    const float pl = len3(pull);
    if (pl > kGrabMaxPull && pl > 0.0f) pull = mul3(pull, __fdiv_rn(kGrabMaxPull, pl));
    return add3(pos, pull);
}
__device__ __forceinline__ F3 predict_w(const XpbdWorld& W, uint32_t i, F3 sim, F3& vel, const XpbdDevParams& P) {
    XpbdWind wind;
    const XpbdWind* wp = nullptr;
    if (*W.wind_count != 0u) {
        wind = W.winds[W.row_cloth[i]];
        if (wind.drag > 0.0f) wp = &wind;
    }
    return apply_cloth_grab(W, i, predict_particle(i, sim, vel, P, wp));
}

// xpbd_substep_post_velocity, xpbd_cpu.rs:393-409, for an unpinned particle: ground plane (extension), then
// v = ((x - prev) * inv_dt) * exp(-k dt). Returns the (possibly clamped) new position.
__device__ __forceinline__ F3 finalize_particle(F3 xn, F3 xo, F3& vel, const XpbdDevParams& P, int* status) {
    if (P.ground_enabled != 0u && xn.y < P.ground_y) xn.y = P.ground_y;
    vel = mul3(mul3(sub3(xn, xo), P.inv_dt), P.damp);
    if (!finite3(xn) || !finite3(vel)) set_status(status, XPBD_DEV_NONFINITE);
    return xn;
}

}  // namespace xpbd
