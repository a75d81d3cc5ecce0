// rpl_weno32.cuh -- packed FP32 WENO5-JS faces shared by the FP32 stage kernels (rpl_tile32.cu,
// rpl_xyw.cu). Every value is a float2 holding two adjacent kappa bins, so the arithmetic issues as
// packed FP32 pairs (FFMA2/FADD2/FMUL2, sm_100); every kernel that uses these forms reconstructs a face
// with the same operations in the same order, so their results agree bit for bit.
#pragma once
#include <cuda_runtime.h>

#include "rpl_device.cuh"

namespace rpl {
namespace w32 {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, f2(-1.0f), a); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float rcpf(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float2 rcp2(float2 a) { return make_float2(rcpf(a.x), rcpf(a.y)); }
__device__ __forceinline__ float2 sel2(bool px, bool py, float2 a, float2 b) {
    return make_float2(px ? a.x : b.x, py ? a.y : b.y);
}

// Nonlinear part of one WENO5 face given the shared quantities of its stencil (see weno5d in
// rpl_stage.cu). Every smoothness indicator is carried as 4*beta: with G0 = D1 + 2 d2, G1 = d2 + d3,
// G2 = D3 - 2 d3 and A'_c = 4(13/12 D_c^2 + eps), t'_k = G_k^2 + A'_k = 4 (eps + beta_k) exactly as the
// reference's indicators, scaled. The weights d_k / t_k^2 are formed as u_k = 1/t'_k^2 with the
// linear weights (0.1, 0.6, 0.3) scaled by 10 (they and the factor 16 cancel in the normalisation):
// returns s2 + sum(w_k u_k) / (u0 + 6 u1 + 3 u2), w_k = 10 d_k (v_k - s2).
__device__ __forceinline__ float2 weno_face2(float2 d1, float2 d2, float2 d3, float2 d4, float2 D1, float2 D2,
                                             float2 D3, float2 A1, float2 A2, float2 A3, float2 s2) {
    const float2 G0 = fma2(f2(2.0f), d2, D1);
    const float2 G1 = add2(d2, d3);
    const float2 G2 = fma2(f2(-2.0f), d3, D3);
    const float2 t0 = fma2(G0, G0, A1), t1 = fma2(G1, G1, A2), t2 = fma2(G2, G2, A3);
    const float2 u0 = rcp2(mul2(t0, t0)), u1 = rcp2(mul2(t1, t1)), u2 = rcp2(mul2(t2, t2));
    const float2 den = fma2(f2(3.0f), u2, fma2(f2(6.0f), u1, u0));
    const float2 w0 = fma2(f2(5.0f / 6.0f), d2, mul2(f2(-1.0f / 3.0f), d1));
    const float2 e3 = add2(d3, d3);
    const float2 w1 = add2(e3, d2);
    const float2 w2 = fma2(f2(-0.5f), d4, e3);
    const float2 num = fma2(w2, u2, fma2(w1, u1, mul2(w0, u0)));
    return fma2(num, rcp2(den), s2);
}

// A'_c = 4 (13/12 D_c^2 + eps)
__device__ __forceinline__ float2 areg(float2 D) {
    return fma2(mul2(f2(13.0f / 3.0f), D), D, f2((float)(4.0 * RPL_WENO_EPS)));
}

// value at the face between s2 and s3 of the oriented stencil s0..s4
__device__ __forceinline__ float2 weno5_2(float2 s0, float2 s1, float2 s2, float2 s3, float2 s4) {
    const float2 d1 = sub2(s1, s0), d2 = sub2(s2, s1), d3 = sub2(s3, s2), d4 = sub2(s4, s3);
    const float2 D1 = sub2(d2, d1), D2 = sub2(d3, d2), D3 = sub2(d4, d3);
    return weno_face2(d1, d2, d3, d4, D1, D2, D3, areg(D1), areg(D2), areg(D3), s2);
}

// both faces of the cell s3 from s0..s5 oriented upwind -> downwind: lo (s2|s3), hi (s3|s4)
__device__ __forceinline__ void weno5_pair2(float2 s0, float2 s1, float2 s2, float2 s3, float2 s4, float2 s5,
                                            float2& lo, float2& hi) {
    const float2 d1 = sub2(s1, s0), d2 = sub2(s2, s1), d3 = sub2(s3, s2), d4 = sub2(s4, s3), d5 = sub2(s5, s4);
    const float2 D1 = sub2(d2, d1), D2 = sub2(d3, d2), D3 = sub2(d4, d3), D4 = sub2(d5, d4);
    const float2 A1 = areg(D1), A2 = areg(D2), A3 = areg(D3), A4 = areg(D4);
    lo = weno_face2(d1, d2, d3, d4, D1, D2, D3, A1, A2, A3, s2);
    hi = weno_face2(d2, d3, d4, d5, D2, D3, D4, A2, A3, A4, s3);
}

// Four adjacent kappa bins as two packed pairs, and the packed forms used on them.
struct Q {                            // four adjacent kappa bins
    float2 a, b;
};
__device__ __forceinline__ Q ldq(const float* p) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    return {make_float2(v.x, v.y), make_float2(v.z, v.w)};
}
__device__ __forceinline__ Q ldgq(const float* p) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    return {make_float2(v.x, v.y), make_float2(v.z, v.w)};
}
__device__ __forceinline__ void stq(float* p, Q q) {
    *reinterpret_cast<float4*>(p) = make_float4(q.a.x, q.a.y, q.b.x, q.b.y);
}
__device__ __forceinline__ Q qz() { return {f2(0.f), f2(0.f)}; }
__device__ __forceinline__ Q qadd(Q x, Q y) { return {add2(x.a, y.a), add2(x.b, y.b)}; }
__device__ __forceinline__ Q qsub(Q x, Q y) { return {sub2(x.a, y.a), sub2(x.b, y.b)}; }
__device__ __forceinline__ Q qmul(Q x, Q y) { return {mul2(x.a, y.a), mul2(x.b, y.b)}; }
__device__ __forceinline__ Q qmuls(Q x, float s) { return {mul2(x.a, f2(s)), mul2(x.b, f2(s))}; }
__device__ __forceinline__ Q qweno(Q s0, Q s1, Q s2, Q s3, Q s4) {
    return {weno5_2(s0.a, s1.a, s2.a, s3.a, s4.a), weno5_2(s0.b, s1.b, s2.b, s3.b, s4.b)};
}
// kappa flux of one bin, c (F_hi - F_lo) with the face flux of the top bin (top) or of the bottom bin
// (bottom) taken as zero: both products and the difference rounded separately, so that every kernel
// gets the same bits however the compiler would otherwise contract them.
__device__ __forceinline__ float kflux(bool top, bool bottom, float c, float hi, float lo) {
    return __fsub_rn(top ? 0.f : __fmul_rn(c, hi), bottom ? 0.f : __fmul_rn(c, lo));
}

}  // namespace w32
}  // namespace rpl
