// rpl_device.cuh -- device arithmetic shared by the stage kernels: WENO5 reconstruction,
// refraction velocities, source rates. Each function cites the reference lines it computes.
#pragma once

#include <cuda_runtime.h>
#include <float.h>
#include <stdint.h>

#include "rpl_internal.h"

namespace rpl {

// WENO5 epsilon: 1e4 * eps(Float64) (wave_current_refraction.jl:43). The FP32 path keeps the
// FP64 value so its weights track the FP64 solution (the reference's Float32 eps, 1.19e-3, would
// switch the scheme to nearly linear weights wherever beta < 1e-3).
#define RPL_WENO_EPS (10000.0 * DBL_EPSILON)

// ---------------------------------------------------------------- Q kernel (FP64)
// CDF of the vertical kernel Q (q_kernel.jl:77-85): F(z) = (e^{2mu(s-1)} - e^{-2mu(s+1)}) /
// (1 - e^{-4mu}), s = clamp((z+d)/d, 0, 1), mu = kappa*d; F = s when |mu| < small_mu.
// exact_form = 1 evaluates the exponents as the reference does (2mu*s - 2mu); exact_form = 0
// evaluates them as 2*kappa*z_c and -2*kappa*(z_c + 2d) with z_c = clamp(z, -d, 0), which avoids
// the cancellation of 2mu*s - 2mu when kappa*d is large.
__device__ __forceinline__ double q_cdf(double kappa, double z, double d, double small_mu, int exact_form) {
    const double mu = kappa * d;
    const double sgn = mu < 0.0 ? -1.0 : 1.0;
    const double m = fabs(mu) < small_mu ? sgn * small_mu : mu;
    double s = (z + d) / d;
    s = s < 0.0 ? 0.0 : (s > 1.0 ? 1.0 : s);
    double e1, e2;
    if (exact_form) {
        const double a = 2.0 * m * s, b = 2.0 * m;
        e1 = a - b;
        e2 = -a - b;
    } else {
        const double kq = m / d;  // kappa, or the safe-mu kappa
        double zc = z < -d ? -d : (z > 0.0 ? 0.0 : z);
        e1 = 2.0 * kq * zc;
        e2 = -2.0 * kq * (zc + 2.0 * d);
    }
    const double fd = (exp(e1) - exp(e2)) / (1.0 - exp(-4.0 * m));
    return fabs(mu) < small_mu ? s : fd;
}

// d F / d kappa (q_kernel.jl:94-109).
__device__ __forceinline__ double q_cdf_dk(double kappa, double z, double d, double small_mu) {
    const double mu = kappa * d;
    const double sgn = mu < 0.0 ? -1.0 : 1.0;
    const double m = fabs(mu) < small_mu ? sgn * small_mu : mu;
    double s = (z + d) / d;
    s = s < 0.0 ? 0.0 : (s > 1.0 ? 1.0 : s);
    const double small_val = d * (4.0 * mu * s * (s * s - 1.0) / 3.0);
    const double a = exp(-2.0 * m * (1.0 - s));
    const double b = exp(-2.0 * m * (1.0 + s));
    const double e = exp(-4.0 * m);
    const double num = a - b, den = 1.0 - e;
    const double dnum = -2.0 * (1.0 - s) * a + 2.0 * (1.0 + s) * b;
    const double dden = 4.0 * e;
    const double fd = d * (dnum * den - num * dden) / (den * den);
    return fabs(mu) < small_mu ? small_val : fd;
}

template <typename T> __device__ __forceinline__ T relu(T x) {
    // max(0, x) with NaN propagation (Julia semantics), -0 -> +0.
    return (x != x) ? x : (x > T(0) ? x : T(0));
}

__device__ __forceinline__ int wrap(int i, int N) { return i < 0 ? i + N : (i >= N ? i - N : i); }
__device__ __forceinline__ int clampi(int i, int N) { return i < 0 ? 0 : (i >= N ? N - 1 : i); }

// Jiang-Shu WENO5 left-biased value at i+1/2 from (i-2 .. i+2)
// (wave_current_refraction.jl:41-55), written in the reference's evaluation order.
template <typename T>
__device__ __forceinline__ T weno5(T fm2, T fm1, T f0, T fp1, T fp2) {
    const T eps = T(RPL_WENO_EPS);
    const T v0 = T(1.0 / 3.0) * fm2 - T(7.0 / 6.0) * fm1 + T(11.0 / 6.0) * f0;
    const T v1 = -T(1.0 / 6.0) * fm1 + T(5.0 / 6.0) * f0 + T(1.0 / 3.0) * fp1;
    const T v2 = T(1.0 / 3.0) * f0 + T(5.0 / 6.0) * fp1 - T(1.0 / 6.0) * fp2;
    const T a0 = fm2 - T(2) * fm1 + f0, b0 = fm2 - T(4) * fm1 + T(3) * f0;
    const T a1 = fm1 - T(2) * f0 + fp1, b1 = fm1 - fp1;
    const T a2 = f0 - T(2) * fp1 + fp2, b2 = T(3) * f0 - T(4) * fp1 + fp2;
    const T beta0 = T(13.0 / 12.0) * (a0 * a0) + T(0.25) * (b0 * b0);
    const T beta1 = T(13.0 / 12.0) * (a1 * a1) + T(0.25) * (b1 * b1);
    const T beta2 = T(13.0 / 12.0) * (a2 * a2) + T(0.25) * (b2 * b2);
    const T q0 = eps + beta0, q1 = eps + beta1, q2 = eps + beta2;
    const T al0 = T(0.1) / (q0 * q0);
    const T al1 = T(0.6) / (q1 * q1);
    const T al2 = T(0.3) / (q2 * q2);
    const T sum = al0 + al1 + al2;
    return (al0 * v0 + al1 * v1 + al2 * v2) / sum;
}

// Upwinded face value at i+1/2 (wave_current_refraction.jl:57-64): the stencil is mirrored for
// negative cell-centre velocity; without a full stencil the first-order upwind value is used.
template <typename T>
__device__ __forceinline__ T weno_face(T im2, T im1, T i0, T ip1, T ip2, T ip3, T vel, bool has) {
    const bool pos = vel >= T(0);
    const T a = pos ? im2 : ip3, b = pos ? im1 : ip2, c = pos ? i0 : ip1;
    const T d = pos ? ip1 : i0, e = pos ? ip2 : im1;
    const T w = weno5(a, b, c, d, e);
    return has ? w : c;
}

// Raw Janssen growth rate (pressure_correlation.jl:109-136 / precomputed_sources.jl:269-280).
// theta is the bin direction, k its wavenumber; all FP64.
__device__ __forceinline__ double jp_rate(double k, double theta, double theta_u, double u_star,
                                          const StageParams& p) {
    const double sigma = sqrt(p.wind_g * k), C = sigma / k;
    const double cos_tu = cos(theta - theta_u);
    if (!(cos_tu > 0.0)) return 0.0;
    const double z1 = p.alpha0 * (u_star * u_star) / p.wind_g;
    if (!(z1 > 0.0)) return 0.0;
    const double inv_age = u_star / C + p.z_alpha;
    const double Z = log(k * z1) + p.von_karman / (inv_age * cos_tu);
    if (Z >= 0.0) return 0.0;
    const double Z2 = Z * Z;
    const double cp = (p.p_in == 2.0) ? cos_tu * cos_tu : pow(cos_tu, p.p_in);
    return p.rho_ratio * (p.beta_max / (p.von_karman * p.von_karman)) * exp(Z) * (Z2 * Z2) *
           (inv_age * inv_age) * cp * sigma;
}

// positive - damping * N of the source bundle at one unit (precomputed_sources.jl:396-439,
// pressure_correlation.jl:145-156, local_saturation.jl:30-47, Sources.jl:430-434).
__device__ __forceinline__ double source_term(const StageParams& p, int64_t cell, int m, int n,
                                              double a) {
    double positive = 0.0, damping = 0.0;
    const double kap = p.kappa[m];
    const double kx = kap * p.cosp[n], ky = kap * p.sinp[n];
    const double k = hypot(kx, ky);
    if (p.has_wind) {
        const double U = p.wind_U10[cell], u_star = p.wind_ustar[cell];
        if (U > 0.0 && u_star > 0.0 && k > 0.0) {
            const double raw = jp_rate(k, atan2(ky, kx), p.wind_theta[cell], u_star, p);
            if (raw > 0.0) {
                const double rate = p.stress_cap ? raw * p.stress_factor[cell] : raw;
                if (rate >= 0.0) positive += rate * a;
                else damping += -rate;
            }
        }
    }
    if (p.has_diss && a > 0.0 && k > 0.0) {
        const double sigma = sqrt(p.ds_g * k);
        const double B = a * sigma * (k * k * k);
        double ov = B / p.B_r - 1.0;
        ov = ov > 0.0 ? ov : 0.0;
        if (ov > 0.0) {
            ov = ov < 1e6 ? ov : 1e6;
            const double sq = (p.sigma_power == 1.0) ? sigma : pow(sigma, p.sigma_power);
            const double op = (p.ds_p == 2.0) ? ov * ov : pow(ov, p.ds_p);
            const double rate = -p.C_ds * sq * op;
            if (rate >= 0.0) damping += rate;
            else positive += -rate * a;
        }
    }
    return positive - damping * a;
}

}  // namespace rpl
