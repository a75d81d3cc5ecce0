// rpl_src32.cuh -- FP32 evaluation of the source bundle for the precision form: wind input with the
// wave-supported stress cap (pressure_correlation.jl:109-151, precomputed_sources.jl:269-326) and
// local-saturation whitecapping (local_saturation.jl:30-47), split into per-cell constants (wind),
// per-kappa constants (bin) and a cheap per-cell-bin part. Branch-free: invalid cases are masked.
#pragma once

#include <cuda_runtime.h>

#include "rpl_internal.h"

namespace rpl {

// per (i,j): u*, log(z1) with z1 = alpha0 u*^2 / g, cos/sin of the wind direction, wind-on flag,
// stress factor (written by the stress kernel of each stage)
struct Cell32 {
    float ustar, logz1, cu, su, on, factor, pad0, pad1;
};

// per kappa bin: log k, 1/C = k/sigma, sigma, sigma k^3 / B_r, -C_ds sigma^q
struct Bin32 {
    float logk, invC, sigma, skB, dsK, pad0, pad1, pad2;
};

__device__ __forceinline__ Cell32 load_cell32(const float* rec) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(rec));
    const float4 b = __ldg(reinterpret_cast<const float4*>(rec) + 1);
    return Cell32{a.x, a.y, a.z, a.w, b.x, b.y, 0.f, 0.f};
}

__device__ __forceinline__ Bin32 load_bin32(const float* rec) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(rec));
    const float4 b = __ldg(reinterpret_cast<const float4*>(rec) + 1);
    return Bin32{a.x, a.y, a.z, a.w, b.x, 0.f, 0.f, 0.f};
}

// x^e for x >= 0, e > 0 as exp2(e log2 x) (relative error a few FP32 ulps times e |log2 x|).
__device__ __forceinline__ float pow_pos32(float x, float e) { return exp2f(e * log2f(x)); }

// Raw Janssen growth rate of one bin (direction cos/sin cth, sth), 0 outside the growth window.
template <class P>
__device__ __forceinline__ float wind_rate32(const P& p, const Cell32& c, const Bin32& b, float cth,
                                             float sth, float& cos_tu) {
    cos_tu = fmaf(cth, c.cu, sth * c.su);
    const float inv_age = fmaf(c.ustar, b.invC, p.z_alpha32);
    const float Z = (b.logk + c.logz1) + p.von_karman32 / (inv_age * cos_tu);
    const bool valid = c.on > 0.5f && cos_tu > 0.0f && Z < 0.0f;
    const float Zc = valid ? Z : 0.0f;
    const float Z2 = Zc * Zc;
    const float cp = (p.p_in == 2.0) ? cos_tu * cos_tu : pow_pos32(fmaxf(cos_tu, 0.0f), (float)p.p_in);
    const float rate = p.wind_K32 * expf(Zc) * (Z2 * Z2) * (inv_age * inv_age) * cp * b.sigma;
    return valid ? rate : 0.0f;
}

// Source tendency of one cell-bin with action a: wind growth (stress-capped) minus whitecapping.
template <class P>
__device__ __forceinline__ float source32(const P& p, const Cell32& c, const Bin32& b, float cth, float sth,
                                          float a) {
    float g = 0.0f;
    if (p.has_wind) {
        float cos_tu;
        const float r = wind_rate32(p, c, b, cth, sth, cos_tu);
        g = (p.stress_cap ? r * c.factor : r) * a;
    }
    if (p.has_diss) {
        float ov = fmaf(a, b.skB, -1.0f);
        const bool valid = a > 0.0f && ov > 0.0f;
        ov = fminf(fmaxf(ov, 0.0f), 1e6f);
        const float op = (p.ds_p == 2.0) ? ov * ov : pow_pos32(ov, (float)p.ds_p);
        g -= valid ? b.dsK * op * a : 0.0f;
    }
    return g;
}

// Source rate of one cell-bin, g / a for the g of source32 (the learned source's training target):
// the stress-capped wind growth rate minus the whitecapping rate at action a.
template <class P>
__device__ __forceinline__ float rate32(const P& p, const Cell32& c, const Bin32& b, float cth, float sth, float a) {
    float r = 0.0f;
    if (p.has_wind) {
        float cos_tu;
        const float w = wind_rate32(p, c, b, cth, sth, cos_tu);
        r = p.stress_cap ? w * c.factor : w;
    }
    if (p.has_diss) {
        float ov = fmaf(a, b.skB, -1.0f);
        const bool valid = a > 0.0f && ov > 0.0f;
        ov = fminf(fmaxf(ov, 0.0f), 1e6f);
        const float op = (p.ds_p == 2.0) ? ov * ov : pow_pos32(ov, (float)p.ds_p);
        r -= valid ? b.dsK * op : 0.0f;
    }
    return r;
}

}  // namespace rpl
