/*
 * ripple_oracle.cpp -- TEST INFRASTRUCTURE ONLY (see ripple_oracle.h).
 *
 * A plain FP64 CPU restatement of the reference's time-step path. Every function
 * cites the reference file:line it follows. Arithmetic is written in the
 * reference's evaluation order and compiled with -ffp-contract=off, so no FMA
 * contraction changes its rounding (Julia does not contract either).
 * OpenMP parallelises over independent output points only; every result is the
 * same for any thread count.
 */
#include "ripple_oracle.h"

#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

inline double clamp01(double s) { return s < 0.0 ? 0.0 : (s > 1.0 ? 1.0 : s); }

/* Julia max(0, x): NaN propagates, -0.0 becomes +0.0. */
inline double relu(double x) { return (x != x) ? x : (x > 0.0 ? x : 0.0); }

inline int64_t periodic(int64_t i, int64_t N) { return i < 0 ? i + N : (i >= N ? i - N : i); }
inline int64_t clamp_idx(int64_t i, int64_t N) { return i < 0 ? 0 : (i >= N ? N - 1 : i); }

/* src/Coupling/wave_current_refraction.jl:41-55 (Jiang-Shu WENO5, eps = 1e4*eps(FT)). */
inline double weno5(double fm2, double fm1, double f0, double fp1, double fp2) {
    const double eps = 10000.0 * DBL_EPSILON;
    const double v0 = (1.0 / 3.0) * fm2 - (7.0 / 6.0) * fm1 + (11.0 / 6.0) * f0;
    const double v1 = -(1.0 / 6.0) * fm1 + (5.0 / 6.0) * f0 + (1.0 / 3.0) * fp1;
    const double v2 = (1.0 / 3.0) * f0 + (5.0 / 6.0) * fp1 - (1.0 / 6.0) * fp2;
    const double a0 = fm2 - 2.0 * fm1 + f0, b0 = fm2 - 4.0 * fm1 + 3.0 * f0;
    const double a1 = fm1 - 2.0 * f0 + fp1, b1 = fm1 - fp1;
    const double a2 = f0 - 2.0 * fp1 + fp2, b2 = 3.0 * f0 - 4.0 * fp1 + fp2;
    const double beta0 = (13.0 / 12.0) * (a0 * a0) + (1.0 / 4.0) * (b0 * b0);
    const double beta1 = (13.0 / 12.0) * (a1 * a1) + (1.0 / 4.0) * (b1 * b1);
    const double beta2 = (13.0 / 12.0) * (a2 * a2) + (1.0 / 4.0) * (b2 * b2);
    const double q0 = eps + beta0, q1 = eps + beta1, q2 = eps + beta2;
    const double al0 = (1.0 / 10.0) / (q0 * q0);
    const double al1 = (6.0 / 10.0) / (q1 * q1);
    const double al2 = (3.0 / 10.0) / (q2 * q2);
    const double sum = al0 + al1 + al2;
    return (al0 * v0 + al1 * v1 + al2 * v2) / sum;
}

/* src/Coupling/wave_current_refraction.jl:57-64 */
inline double weno_face(double im2, double im1, double i0, double ip1, double ip2, double ip3,
                        double vel, bool has_stencil) {
    const bool pos = vel >= 0.0;
    const double wv = pos ? weno5(im2, im1, i0, ip1, ip2) : weno5(ip3, ip2, ip1, i0, im1);
    const double fo = pos ? i0 : ip1;
    return has_stencil ? wv : fo;
}

/* src/Physics/Packages/precomputed_sources.jl:269-280 */
inline double jp_rate(double k, double sigma, double C, double theta, double theta_u, double u_star,
                      double rho_ratio, double beta_max, double z_alpha, double p_in, double alpha0,
                      double kvk, double g) {
    const double cos_tu = std::cos(theta - theta_u);
    if (!(cos_tu > 0.0)) return 0.0;
    const double z1 = alpha0 * (u_star * u_star) / g;
    if (!(z1 > 0.0)) return 0.0;
    const double inv_age = u_star / C + z_alpha;
    const double Z = std::log(k * z1) + kvk / (inv_age * cos_tu);
    if (Z >= 0.0) return 0.0;
    return rho_ratio * (beta_max / (kvk * kvk)) * std::exp(Z) * std::pow(Z, 4.0) *
           (inv_age * inv_age) * std::pow(cos_tu, p_in) * sigma;
}

}  // namespace

extern "C" {

/* ------------------------------------------------------------------ Q kernel */

/* src/Coupling/q_kernel.jl:7-16 (host twin; depth <= 0 throws there, NaN here) */
double ora_q_value(double kappa, double z, double depth, double small_mu) {
    if (depth <= 0.0) return NAN;
    const double mu = kappa * depth;
    if (std::fabs(mu) < small_mu) return 1.0 / depth;
    const double s = (z + depth) / depth;
    const double b = 2.0 * mu;
    const double a = b * s;
    const double ratio = (std::exp(a - b) + std::exp(-a - b)) / (1.0 - std::exp(-2.0 * b));
    return (2.0 * mu / depth) * ratio;
}

/* src/Coupling/q_kernel.jl:18-27 */
double ora_q_cdf(double kappa, double z, double depth, double small_mu) {
    if (depth <= 0.0) return NAN;
    const double mu = kappa * depth;
    const double s = clamp01((z + depth) / depth);
    if (std::fabs(mu) < small_mu) return s;
    const double a = 2.0 * mu * s;
    const double b = 2.0 * mu;
    return (std::exp(a - b) - std::exp(-a - b)) / (1.0 - std::exp(-2.0 * b));
}

/* src/Coupling/q_kernel.jl:29-32 */
double ora_q_cell_integral(double kappa, double z1, double z2, double depth, double small_mu) {
    const double lo = z1 < z2 ? z1 : z2, hi = z1 < z2 ? z2 : z1;
    return ora_q_cdf(kappa, hi, depth, small_mu) - ora_q_cdf(kappa, lo, depth, small_mu);
}

/* src/Coupling/q_kernel.jl:34-52 */
double ora_q_cdf_kappa_derivative(double kappa, double z, double depth, double small_mu) {
    if (depth <= 0.0) return NAN;
    const double mu = kappa * depth;
    const double s = clamp01((z + depth) / depth);
    if (std::fabs(mu) < small_mu) return depth * (4.0 * mu * s * (s * s - 1.0) / 3.0);
    const double a = std::exp(-2.0 * mu * (1.0 - s));
    const double b = std::exp(-2.0 * mu * (1.0 + s));
    const double e = std::exp(-4.0 * mu);
    const double num = a - b, den = 1.0 - e;
    const double dnum = -2.0 * (1.0 - s) * a + 2.0 * (1.0 + s) * b;
    const double dden = 4.0 * e;
    const double dF = (dnum * den - num * dden) / (den * den);
    return depth * dF;
}

/* src/Coupling/q_kernel.jl:54-58 */
double ora_q_cell_integral_kappa_derivative(double kappa, double z1, double z2, double depth,
                                            double small_mu) {
    const double lo = z1 < z2 ? z1 : z2, hi = z1 < z2 ? z2 : z1;
    return ora_q_cdf_kappa_derivative(kappa, hi, depth, small_mu) -
           ora_q_cdf_kappa_derivative(kappa, lo, depth, small_mu);
}

/* src/Coupling/q_kernel.jl:60-63,77-85 (kernel form: safe mu, branch-free select) */
double ora_q_cdf_kernel(double kappa, double z, double depth, double small_mu) {
    const double mu = kappa * depth;
    const double sgn = mu < 0.0 ? -1.0 : 1.0;
    const double m = std::fabs(mu) < small_mu ? sgn * small_mu : mu;
    const double s = clamp01((z + depth) / depth);
    const double a = 2.0 * m * s;
    const double b = 2.0 * m;
    const double fd = (std::exp(a - b) - std::exp(-a - b)) / (1.0 - std::exp(-2.0 * b));
    return std::fabs(mu) < small_mu ? s : fd;
}

/* src/Coupling/q_kernel.jl:87-92 */
double ora_q_cell_integral_kernel(double kappa, double z1, double z2, double depth, double small_mu) {
    const double lo = z1 < z2 ? z1 : z2, hi = z1 < z2 ? z2 : z1;
    return ora_q_cdf_kernel(kappa, hi, depth, small_mu) - ora_q_cdf_kernel(kappa, lo, depth, small_mu);
}

/* src/Coupling/q_kernel.jl:94-116 */
static double q_cdf_kappa_derivative_kernel(double kappa, double z, double depth, double small_mu) {
    const double mu = kappa * depth;
    const double sgn = mu < 0.0 ? -1.0 : 1.0;
    const double m = std::fabs(mu) < small_mu ? sgn * small_mu : mu;
    const double s = clamp01((z + depth) / depth);
    const double small_val = depth * (4.0 * mu * s * (s * s - 1.0) / 3.0);
    const double a = std::exp(-2.0 * m * (1.0 - s));
    const double b = std::exp(-2.0 * m * (1.0 + s));
    const double e = std::exp(-4.0 * m);
    const double num = a - b, den = 1.0 - e;
    const double dnum = -2.0 * (1.0 - s) * a + 2.0 * (1.0 + s) * b;
    const double dden = 4.0 * e;
    const double fd = depth * (dnum * den - num * dden) / (den * den);
    return std::fabs(mu) < small_mu ? small_val : fd;
}

double ora_q_cell_integral_kappa_derivative_kernel(double kappa, double z1, double z2, double depth,
                                                   double small_mu) {
    const double lo = z1 < z2 ? z1 : z2, hi = z1 < z2 ? z2 : z1;
    return q_cdf_kappa_derivative_kernel(kappa, hi, depth, small_mu) -
           q_cdf_kappa_derivative_kernel(kappa, lo, depth, small_mu);
}

/* src/Coupling/doppler_velocity.jl:45-82: U[i,j,m] = sum_k uL[i,j,k] * Qcell(kappa_m, z_k, z_k+1, d_ij),
 * sequential in k. derivative=1 gives dU/dkappa (doppler_velocity.jl:64-82). */
void ora_doppler_velocity(int64_t Nx, int64_t Ny, int64_t Nz, int64_t Nk, const double* u,
                          const double* v, const double* depth_field, double depth_scalar,
                          const double* kappa, const double* zfaces, double small_mu,
                          int32_t derivative, double* Ux, double* Uy) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int64_t m = 0; m < Nk; ++m)
        for (int64_t j = 0; j < Ny; ++j)
            for (int64_t i = 0; i < Nx; ++i) {
                const double d = depth_field ? depth_field[i + Nx * j] : depth_scalar;
                double ax = 0.0, ay = 0.0;
                for (int64_t k = 0; k < Nz; ++k) {
                    const double w =
                        derivative ? ora_q_cell_integral_kappa_derivative_kernel(kappa[m], zfaces[k],
                                                                                zfaces[k + 1], d, small_mu)
                                   : ora_q_cell_integral_kernel(kappa[m], zfaces[k], zfaces[k + 1], d,
                                                                small_mu);
                    const int64_t c = i + Nx * (j + Ny * k);
                    ax += u[c] * w;
                    ay += v[c] * w;
                }
                Ux[i + Nx * (j + Ny * m)] = ax;
                Uy[i + Nx * (j + Ny * m)] = ay;
            }
}

/* src/Coupling/wave_current_refraction.jl:7-19 (periodic centred differences) */
void ora_current_gradients(int64_t Nx, int64_t Ny, int64_t Nk, const double* Ux, const double* Uy,
                           double dx_inv, double dy_inv, double* Uxx, double* Uxy, double* Uyx,
                           double* Uyy) {
    for (int64_t k = 0; k < Nk; ++k)
        for (int64_t j = 0; j < Ny; ++j)
            for (int64_t i = 0; i < Nx; ++i) {
                const int64_t ip = i == Nx - 1 ? 0 : i + 1, im = i == 0 ? Nx - 1 : i - 1;
                const int64_t jp = j == Ny - 1 ? 0 : j + 1, jm = j == 0 ? Ny - 1 : j - 1;
                const int64_t o = Nx * Ny * k;
                const int64_t c = i + Nx * j + o;
                Uxx[c] = (Ux[ip + Nx * j + o] - Ux[im + Nx * j + o]) * (dx_inv / 2.0);
                Uxy[c] = (Ux[i + Nx * jp + o] - Ux[i + Nx * jm + o]) * (dy_inv / 2.0);
                Uyx[c] = (Uy[ip + Nx * j + o] - Uy[im + Nx * j + o]) * (dx_inv / 2.0);
                Uyy[c] = (Uy[i + Nx * jp + o] - Uy[i + Nx * jm + o]) * (dy_inv / 2.0);
            }
}

/* -------------------------------------------------------- pseudomomentum self-coupling */

/* src/CoordinateGrids/polar_wavevector_grid.jl:73-99,107-110 (spectral_first_moment_measures):
 * kx = (k2^3 - k1^3)/3 * (sin p2 - sin p1), ky = (k2^3 - k1^3)/3 * (cos p1 - cos p2), (Nk,Np) m fastest. */
void ora_first_moment_measures(int64_t Nk, int64_t Np, const double* kf, const double* pf, double* kx,
                               double* ky) {
    for (int64_t n = 0; n < Np; ++n)
        for (int64_t m = 0; m < Nk; ++m) {
            const double k1 = kf[m], k2 = kf[m + 1], p1 = pf[n], p2 = pf[n + 1];
            const double radial = (k2 * k2 * k2 - k1 * k1 * k1) / 3.0;
            kx[m + Nk * n] = radial * (std::sin(p2) - std::sin(p1));
            ky[m + Nk * n] = radial * (std::cos(p1) - std::cos(p2));
        }
}

/* src/Coupling/pseudomomentum.jl:68-121: overlap[t,s] = sum_k Qcell(kappa_t) * Qcell(kappa_s) / |dz_k| and
 * derivative_overlap[t,s] = sum_k dQcell/dkappa(kappa_t) * Qcell(kappa_s) / |dz_k|, sequential in k, with the
 * host Q forms (q_kernel.jl:18-58). depth_field NULL: (Nk,Nk) tables, target fastest; else per-column tables
 * (Nx,Ny,Nk,Nk), x fastest. */
void ora_pm_overlap_tables(int64_t Nx, int64_t Ny, int64_t Nk, const double* kappa, int64_t Nz,
                           const double* zf, const double* depth_field, double depth_scalar, double small_mu,
                           double* overlap, double* doverlap) {
    const int64_t cols = depth_field ? Nx * Ny : 1;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < cols; ++c) {
        const double d = depth_field ? depth_field[c] : depth_scalar;
        for (int64_t sm = 0; sm < Nk; ++sm)
            for (int64_t tm = 0; tm < Nk; ++tm) {
                double total = 0.0, dtotal = 0.0;
                for (int64_t k = 0; k < Nz; ++k) {
                    const double z1 = zf[k], z2 = zf[k + 1], dz = std::fabs(z2 - z1);
                    const double sw = ora_q_cell_integral(kappa[sm], z1, z2, d, small_mu);
                    const double tw = ora_q_cell_integral(kappa[tm], z1, z2, d, small_mu);
                    const double td = ora_q_cell_integral_kappa_derivative(kappa[tm], z1, z2, d, small_mu);
                    total += tw * sw / dz;
                    dtotal += td * sw / dz;
                }
                const int64_t e = tm + Nk * sm;
                overlap[c + cols * e] = total;
                doverlap[c + cols * e] = dtotal;
            }
    }
}

/* src/Coupling/pseudomomentum.jl:123-138,316-342: per (i,j,t) U = sum over n (outer) and source s (inner)
 * of overlap[t,s] * N[i,j,s,n] * kx_measure[s,n] (ky for Uy, derivative_overlap for dU/dkappa). N and the
 * outputs x fastest; per_cell selects the (Nx,Ny,Nk,Nk) tables. */
void ora_pm_doppler_velocity(int64_t Nx, int64_t Ny, int64_t Nk, int64_t Np, const double* N, int32_t per_cell,
                             const double* overlap, const double* doverlap, const double* kx, const double* ky,
                             double* Ux, double* Uy, double* dUx, double* dUy) {
    const int64_t P = Nx * Ny, cols = per_cell ? P : 1;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < P; ++c) {
        const int64_t tc = per_cell ? c : 0;
        for (int64_t tm = 0; tm < Nk; ++tm) {
            double ax = 0.0, ay = 0.0, dax = 0.0, day = 0.0;
            for (int64_t n = 0; n < Np; ++n)
                for (int64_t sm = 0; sm < Nk; ++sm) {
                    const double a = N[c + P * (sm + Nk * n)];
                    const double q = overlap[tc + cols * (tm + Nk * sm)];
                    const double dq = doverlap ? doverlap[tc + cols * (tm + Nk * sm)] : 0.0;
                    ax += q * a * kx[sm + Nk * n];
                    ay += q * a * ky[sm + Nk * n];
                    dax += dq * a * kx[sm + Nk * n];
                    day += dq * a * ky[sm + Nk * n];
                }
            const int64_t o = c + P * tm;
            if (Ux) Ux[o] = ax;
            if (Uy) Uy[o] = ay;
            if (dUx) dUx[o] = dax;
            if (dUy) dUy[o] = day;
        }
    }
}

/* src/Coupling/pseudomomentum.jl:173-210,380-410 (compute_pseudomomentum_cell_integrals / _averages):
 * p[i,j,k] = sum over n (outer), m (inner) of Qcell_kernel(kappa_m, z_k, z_k+1, d) * N * k_measure, divided
 * by |dz_k| when cell_average. Outputs (Nx,Ny,Nz) x fastest. */
void ora_pm_cells(int64_t Nx, int64_t Ny, int64_t Nk, int64_t Np, const double* N, int64_t Nz, const double* zf,
                  const double* depth_field, double depth_scalar, const double* kappa, const double* kx,
                  const double* ky, double small_mu, int32_t cell_average, double* px, double* py) {
    const int64_t P = Nx * Ny;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < P; ++c) {
        const double d = depth_field ? depth_field[c] : depth_scalar;
        for (int64_t k = 0; k < Nz; ++k) {
            const double z1 = zf[k], z2 = zf[k + 1];
            double ax = 0.0, ay = 0.0;
            for (int64_t n = 0; n < Np; ++n)
                for (int64_t m = 0; m < Nk; ++m) {
                    const double q = ora_q_cell_integral_kernel(kappa[m], z1, z2, d, small_mu);
                    const double a = N[c + P * (m + Nk * n)];
                    ax += q * a * kx[m + Nk * n];
                    ay += q * a * ky[m + Nk * n];
                }
            const double scale = cell_average ? 1.0 / std::fabs(z2 - z1) : 1.0;
            px[c + P * k] = ax * scale;
            py[c + P * k] = ay * scale;
        }
    }
}

/* -------------------------------------------------------- spectral grid */

/* src/CoordinateGrids/spectral_grids.jl:4-27 */
void ora_lower_bounded_faces(int64_t N, const double* c, double lower, double* f) {
    if (N == 1) {
        f[0] = c[0] - 0.5;
        f[1] = c[0] + 0.5;
    } else {
        for (int64_t i = 1; i < N; ++i) f[i] = (c[i - 1] + c[i]) / 2.0;
        f[0] = c[0] - (f[1] - c[0]);
        f[N] = c[N - 1] + (c[N - 1] - f[N - 1]);
    }
    if (f[0] < lower) f[0] = lower;
}

/* src/CoordinateGrids/polar_wavevector_grid.jl:34-37 */
void ora_uniform_periodic_faces(int64_t N, const double* c, double* f) {
    const double dphi = N == 1 ? 2.0 * M_PI : 2.0 * M_PI / (double)N;
    for (int64_t i = 0; i <= N; ++i) f[i] = c[0] - dphi / 2.0 + (double)i * dphi;
}

/* src/CoordinateGrids/polar_wavevector_grid.jl:44-47 */
void ora_polar_weights(int64_t Nk, int64_t Np, const double* kf, const double* pf, double* w) {
    for (int64_t n = 0; n < Np; ++n)
        for (int64_t m = 0; m < Nk; ++m)
            w[m + Nk * n] = ((kf[m + 1] * kf[m + 1] - kf[m] * kf[m]) / 2.0) * (pf[n + 1] - pf[n]);
}

/* src/Models/transport.jl:61-70 (cell-averaged deep-water c_g) */
void ora_group_velocity_deep(int64_t Nk, int64_t Np, const double* kf, const double* pf,
                             const double* w, double g, double* cg_x, double* cg_y) {
    for (int64_t n = 0; n < Np; ++n)
        for (int64_t m = 0; m < Nk; ++m) {
            const double k1 = kf[m], k2 = kf[m + 1], p1 = pf[n], p2 = pf[n + 1];
            const double radial = (std::pow(k2, 1.5) - std::pow(k1, 1.5)) / 1.5;
            const double ax = std::sin(p2) - std::sin(p1);
            const double ay = std::cos(p1) - std::cos(p2);
            const double scale = std::sqrt(g) / (2.0 * w[m + Nk * n]);
            cg_x[m + Nk * n] = scale * radial * ax;
            cg_y[m + Nk * n] = scale * radial * ay;
        }
}

/* src/Models/transport.jl:72-83 (cell-centre finite-depth c_g); depth_field != NULL gives the
 * (Nx,Ny,Nk,Np) table of transport.jl:114-125, else the (Nk,Np) table of :126-135. */
void ora_group_velocity_finite(int64_t Nx, int64_t Ny, int64_t Nk, int64_t Np, const double* kappa,
                               const double* phi, const double* depth_field, double depth_scalar,
                               double g, double* cg_x, double* cg_y) {
    const int64_t ncol = depth_field ? Nx * Ny : 1;
#pragma omp parallel for schedule(static)
    for (int64_t n = 0; n < Np; ++n)
        for (int64_t m = 0; m < Nk; ++m)
            for (int64_t c = 0; c < ncol; ++c) {
                const double kx = kappa[m] * std::cos(phi[n]), ky = kappa[m] * std::sin(phi[n]);
                const double k = kappa[m];
                const double h = depth_field ? depth_field[c] : depth_scalar;
                const double mu = k * h;
                const double cp = std::sqrt(g * std::tanh(mu) / k);
                const double gf = (1.0 + 2.0 * mu / std::sinh(2.0 * mu)) / 2.0;
                const double cg = gf * cp;
                cg_x[c + ncol * (m + Nk * n)] = cg * kx / k;
                cg_y[c + ncol * (m + Nk * n)] = cg * ky / k;
            }
}

/* ---------------------------------------------------------------- winds */

/* src/Physics/shared/drag.jl:77-86 (BulkWindDrag{:linear}) */
double ora_friction_velocity_linear(double U10) {
    const double cd = (0.8 + 0.065 * U10) * 1e-3;
    return U10 * std::sqrt(cd > 0.0 ? cd : 0.0);
}

/* src/Forcing/winds.jl:139-152 (LinearStormTrack) */
void ora_storm_center(const ora_holland* w, double t, double* cx, double* cy) {
    const int64_t n = w->n_track;
    if (n <= 0) { *cx = w->center_x[0]; *cy = w->center_y[0]; return; }
    if (t <= w->track_t[0]) { *cx = w->center_x[0]; *cy = w->center_y[0]; return; }
    if (t >= w->track_t[n - 1]) { *cx = w->center_x[n - 1]; *cy = w->center_y[n - 1]; return; }
    int64_t up = 0;
    while (w->track_t[up] < t) ++up;
    const int64_t lo = up - 1;
    const double wt = (t - w->track_t[lo]) / (w->track_t[up] - w->track_t[lo]);
    *cx = (1.0 - wt) * w->center_x[lo] + wt * w->center_x[up];
    *cy = (1.0 - wt) * w->center_y[lo] + wt * w->center_y[up];
}

/* src/Forcing/winds.jl:255-265,295-309 (Holland profile, inflow angle, rotation, background) */
void ora_holland_velocity(const ora_holland* w, double x, double y, double t, double* vx, double* vy) {
    double cx, cy;
    ora_storm_center(w, t, &cx, &cy);
    const double dx = x - cx, dy = y - cy;
    const double r = std::hypot(dx, dy);
    if (r == 0.0) { *vx = w->background_x; *vy = w->background_y; return; }
    const double scaled = w->rmax / r;
    const double shape = std::pow(scaled, w->shape_parameter);
    const double e = shape * std::exp(1.0 - shape);
    double speed = w->vmax * std::sqrt(e > 0.0 ? e : 0.0);
    if (r > w->radius) {
        const double dd = w->radius - w->rmax;
        const double ulp = std::nextafter(w->radius, INFINITY) - w->radius; /* Julia eps(radius) */
        const double decay = dd > ulp ? dd : ulp;
        speed *= std::exp(-(r - w->radius) / decay);
    }
    const double s = (double)w->rotation;
    const double tx = -s * dy / r, ty = s * dx / r;
    const double rx = dx / r, ry = dy / r;
    const double ci = std::cos(w->inflow_angle), si = std::sin(w->inflow_angle);
    *vx = speed * (ci * tx - si * rx) + w->background_x;
    *vy = speed * (ci * ty - si * ry) + w->background_y;
}

/* Per-(i,j) wind at time t: src/Physics/WindInput/pressure_correlation.jl:54-63 and the host
 * loop of src/Physics/Packages/precomputed_sources.jl:337-347. */
void ora_wind_fields(const ora_model* M, double t, double* U10, double* theta, double* ustar) {
    for (int64_t j = 0; j < M->Ny; ++j)
        for (int64_t i = 0; i < M->Nx; ++i) {
            const int64_t c = i + M->Nx * j;
            double U = 0.0, th = 0.0;
            if (M->wind_kind == ORA_WIND_UNIFORM) {
                U = M->wind_speed;
                th = M->wind_direction;
            } else if (M->wind_kind == ORA_WIND_HOLLAND) {
                double vx, vy;
                ora_holland_velocity(&M->holland, M->xnodes[i], M->ynodes[j], t, &vx, &vy);
                U = std::hypot(vx, vy);
                th = std::atan2(vy, vx);
            } else if (M->wind_kind == ORA_WIND_FIELD) {
                U = M->wind_U10[c];
                th = M->wind_theta[c];
            }
            U10[c] = U;
            theta[c] = th;
            ustar[c] = ora_friction_velocity_linear(U);
        }
}

/* src/Physics/Packages/precomputed_sources.jl:282-326 (stress cap, eps = 0.4), loop n outer m inner */
void ora_stress_factor(const ora_model* M, const double* N, double t, double* factor) {
    const int64_t Nx = M->Nx, Ny = M->Ny, Nk = M->Nk, Np = M->Np;
    std::vector<double> U10(Nx * Ny), th(Nx * Ny), us(Nx * Ny);
    ora_wind_fields(M, t, U10.data(), th.data(), us.data());
    const double g = M->gravity;
    const double rho_w_g = M->rho_water * g, rho_air = M->rho_air, ratio = M->rho_air / M->rho_water;
    const double eps = 0.4;
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < Ny; ++j)
        for (int64_t i = 0; i < Nx; ++i) {
            const int64_t c = i + Nx * j;
            const double U = U10[c], u_star = us[c];
            if (U > 0.0 && u_star > 0.0) {
                const double tu = th[c];
                const double tau_max = rho_air * (u_star * u_star);
                double twx = 0.0, twy = 0.0;
                for (int64_t n = 0; n < Np; ++n)
                    for (int64_t m = 0; m < Nk; ++m) {
                        const double a = N[i + Nx * (j + Ny * (m + Nk * n))];
                        if (a > 0.0) {
                            const double k = M->kappa[m];
                            if (k > 0.0) {
                                const double sigma = std::sqrt(g * k), C = sigma / k;
                                const double theta = M->phi[n];
                                const double rate = jp_rate(k, sigma, C, theta, tu, u_star, ratio, M->beta_max,
                                                            M->z_alpha, M->p_in, M->alpha0, M->von_karman, g);
                                if (rate > 0.0) {
                                    const double mflux = rate * a / C * M->weights[m + Nk * n] * rho_w_g;
                                    twx += mflux * std::cos(theta);
                                    twy += mflux * std::sin(theta);
                                }
                            }
                        }
                    }
                const double par = twx * std::cos(tu) + twy * std::sin(tu);
                const double eff = par > 0.0 ? par : 0.0;
                factor[c] = (eff > eps * tau_max && tau_max > 0.0) ? eps * tau_max / eff : 1.0;
            } else {
                factor[c] = 1.0;
            }
        }
}

/* ------------------------------------------------------------ tendencies */

/* src/Coupling/wave_current_refraction.jl:74-151 (fused Doppler transport + refraction) */
static void refraction_tendency(const ora_model* M, const double* N, double* G) {
    const int64_t Nx = M->Nx, Ny = M->Ny, Nk = M->Nk, Np = M->Np;
    const double dx_inv = 1.0 / M->dx, dy_inv = 1.0 / M->dy;
    const double dk_inv = 1.0 / (M->kappa_faces[1] - M->kappa_faces[0]);  /* first(coordinate_spacings) */
    const double dp_inv = 1.0 / (M->phi_faces[1] - M->phi_faces[0]);
    const int64_t P = Nx * Ny, S = P * Nk;
#pragma omp parallel for collapse(2) schedule(static)
    for (int64_t n = 0; n < Np; ++n)
        for (int64_t m = 0; m < Nk; ++m) {
            const double kap = M->kappa[m];
            const double cph = std::cos(M->phi[n]), sph = std::sin(M->phi[n]);
            for (int64_t j = 0; j < Ny; ++j)
                for (int64_t i = 0; i < Nx; ++i) {
                    const int64_t c3 = i + Nx * (j + Ny * m);
                    const double Uxc = M->Ux[c3], Uyc = M->Uy[c3];
                    const double Uxx = M->Uxx[c3], Uxy = M->Uxy[c3], Uyx = M->Uyx[c3], Uyy = M->Uyy[c3];
                    const double ck = -kap * (cph * cph * Uxx + cph * sph * (Uyx + Uxy) + sph * sph * Uyy);
                    const double cp = cph * sph * (Uxx - Uyy) + sph * sph * Uyx - cph * cph * Uxy;
                    const int64_t tc = M->cg_per_cell ? i + Nx * (j + Ny * (m + Nk * n)) : m + Nk * n;
                    const double ux = M->cg_x[tc] + Uxc, uy = M->cg_y[tc] + Uyc;
                    const double* col = N + S * n + P * m + Nx * j;  /* row j of bin (m,n) */
                    /* x */
                    const double x_m3 = col[periodic(i - 3, Nx)], x_m2 = col[periodic(i - 2, Nx)],
                                 x_m1 = col[periodic(i - 1, Nx)], x_0 = col[i],
                                 x_p1 = col[periodic(i + 1, Nx)], x_p2 = col[periodic(i + 2, Nx)],
                                 x_p3 = col[periodic(i + 3, Nx)];
                    const double Nxp = weno_face(x_m2, x_m1, x_0, x_p1, x_p2, x_p3, ux, true);
                    const double Nxm = weno_face(x_m3, x_m2, x_m1, x_0, x_p1, x_p2, ux, true);
                    const double fx = ux * (Nxp - Nxm) * dx_inv;
                    /* y */
                    const double* bin = N + S * n + P * m;
                    const double y_m3 = bin[i + Nx * periodic(j - 3, Ny)], y_m2 = bin[i + Nx * periodic(j - 2, Ny)],
                                 y_m1 = bin[i + Nx * periodic(j - 1, Ny)], y_0 = bin[i + Nx * j],
                                 y_p1 = bin[i + Nx * periodic(j + 1, Ny)], y_p2 = bin[i + Nx * periodic(j + 2, Ny)],
                                 y_p3 = bin[i + Nx * periodic(j + 3, Ny)];
                    const double Nyp = weno_face(y_m2, y_m1, y_0, y_p1, y_p2, y_p3, uy, true);
                    const double Nym = weno_face(y_m3, y_m2, y_m1, y_0, y_p1, y_p2, uy, true);
                    const double fy = uy * (Nyp - Nym) * dy_inv;
                    /* kappa (bounded, no-flux outer faces, first-order fallback) */
                    const bool hp = (m - 2 >= 0) && (m + 3 <= Nk - 1);
                    const bool hm = (m - 3 >= 0) && (m + 2 <= Nk - 1);
                    const double* pt = N + S * n + i + Nx * j;
                    const double k_m3 = pt[P * clamp_idx(m - 3, Nk)], k_m2 = pt[P * clamp_idx(m - 2, Nk)],
                                 k_m1 = pt[P * clamp_idx(m - 1, Nk)], k_0 = pt[P * m],
                                 k_p1 = pt[P * clamp_idx(m + 1, Nk)], k_p2 = pt[P * clamp_idx(m + 2, Nk)],
                                 k_p3 = pt[P * clamp_idx(m + 3, Nk)];
                    const double Nkp = weno_face(k_m2, k_m1, k_0, k_p1, k_p2, k_p3, ck, hp);
                    const double Nkm = weno_face(k_m3, k_m2, k_m1, k_0, k_p1, k_p2, ck, hm);
                    const double fkp = (m == Nk - 1) ? 0.0 : ck * Nkp;
                    const double fkm = (m == 0) ? 0.0 : ck * Nkm;
                    const double fk = (fkp - fkm) * dk_inv;
                    /* phi (periodic) */
                    const double* pm = N + P * m + i + Nx * j;
                    const double p_m3 = pm[S * periodic(n - 3, Np)], p_m2 = pm[S * periodic(n - 2, Np)],
                                 p_m1 = pm[S * periodic(n - 1, Np)], p_0 = pm[S * n],
                                 p_p1 = pm[S * periodic(n + 1, Np)], p_p2 = pm[S * periodic(n + 2, Np)],
                                 p_p3 = pm[S * periodic(n + 3, Np)];
                    const double Npp = weno_face(p_m2, p_m1, p_0, p_p1, p_p2, p_p3, cp, true);
                    const double Npm = weno_face(p_m3, p_m2, p_m1, p_0, p_p1, p_p2, cp, true);
                    const double fp = cp * (Npp - Npm) * dp_inv;
                    G[i + Nx * (j + Ny * (m + Nk * n))] = -(fx + fy + fk + fp);
                }
        }
}

/* src/Models/intrinsic_transport.jl:14-68 (periodic x,y; the gate tendencies.jl:43-50 admits only
 * periodic grids into this kernel) */
static void intrinsic_tendency(const ora_model* M, const double* N, double* G) {
    const int64_t Nx = M->Nx, Ny = M->Ny, Nk = M->Nk, Np = M->Np;
    const double dx_inv = 1.0 / M->dx, dy_inv = 1.0 / M->dy;
    const int64_t P = Nx * Ny;
#pragma omp parallel for collapse(2) schedule(static)
    for (int64_t n = 0; n < Np; ++n)
        for (int64_t m = 0; m < Nk; ++m)
            for (int64_t j = 0; j < Ny; ++j)
                for (int64_t i = 0; i < Nx; ++i) {
                    const int64_t tc = M->cg_per_cell ? i + Nx * (j + Ny * (m + Nk * n)) : m + Nk * n;
                    const double ux = M->cg_x[tc], uy = M->cg_y[tc];
                    const double* bin = N + P * (m + Nk * n);
                    const double* col = bin + Nx * j;
                    const double x_m3 = col[periodic(i - 3, Nx)], x_m2 = col[periodic(i - 2, Nx)],
                                 x_m1 = col[periodic(i - 1, Nx)], x_0 = col[i],
                                 x_p1 = col[periodic(i + 1, Nx)], x_p2 = col[periodic(i + 2, Nx)],
                                 x_p3 = col[periodic(i + 3, Nx)];
                    const double Nxp = weno_face(x_m2, x_m1, x_0, x_p1, x_p2, x_p3, ux, true);
                    const double Nxm = weno_face(x_m3, x_m2, x_m1, x_0, x_p1, x_p2, ux, true);
                    const double fx = ux * (Nxp - Nxm) * dx_inv;
                    const double y_m3 = bin[i + Nx * periodic(j - 3, Ny)], y_m2 = bin[i + Nx * periodic(j - 2, Ny)],
                                 y_m1 = bin[i + Nx * periodic(j - 1, Ny)], y_0 = bin[i + Nx * j],
                                 y_p1 = bin[i + Nx * periodic(j + 1, Ny)], y_p2 = bin[i + Nx * periodic(j + 2, Ny)],
                                 y_p3 = bin[i + Nx * periodic(j + 3, Ny)];
                    const double Nyp = weno_face(y_m2, y_m1, y_0, y_p1, y_p2, y_p3, uy, true);
                    const double Nym = weno_face(y_m3, y_m2, y_m1, y_0, y_p1, y_p2, uy, true);
                    const double fy = uy * (Nyp - Nym) * dy_inv;
                    G[i + Nx * (j + Ny * (m + Nk * n))] = -(fx + fy);
                }
}

/* Source tendency of PrecomputedSources(wind_input=PressureCorrelationInput,
 * dissipation=LocalSaturationDissipation) added to G:
 *   src/Models/tendencies.jl:34-36,91-93 (G += source_tendency),
 *   src/Physics/Packages/precomputed_sources.jl:396-417,436-439 (split bundle),
 *   src/Physics/WindInput/pressure_correlation.jl:109-151 (raw rate x stress factor),
 *   src/Physics/Dissipation/local_saturation.jl:30-47,
 *   src/Sources/Sources.jl:430-434 (split_growth_rate / split_damping_rate). */
static void add_sources(const ora_model* M, const double* N, double t, double* G) {
    const int64_t Nx = M->Nx, Ny = M->Ny, Nk = M->Nk, Np = M->Np;
    const bool wind = M->wind_kind != ORA_WIND_NONE;
    std::vector<double> factor, U10, th, us;
    if (wind) {
        factor.resize(Nx * Ny);
        U10.resize(Nx * Ny); th.resize(Nx * Ny); us.resize(Nx * Ny);
        ora_stress_factor(M, N, t, factor.data());
        ora_wind_fields(M, t, U10.data(), th.data(), us.data());
    }
    const double g = M->gravity;
#pragma omp parallel for collapse(2) schedule(static)
    for (int64_t n = 0; n < Np; ++n)
        for (int64_t m = 0; m < Nk; ++m) {
            const double kx = M->kappa[m] * std::cos(M->phi[n]);
            const double ky = M->kappa[m] * std::sin(M->phi[n]);
            const double k = std::hypot(kx, ky);
            for (int64_t j = 0; j < Ny; ++j)
                for (int64_t i = 0; i < Nx; ++i) {
                    const int64_t c = i + Nx * j, u = c + Nx * Ny * (m + Nk * n);
                    const double a = N[u];
                    double positive = 0.0, damping = 0.0;
                    if (wind) {
                        double raw = 0.0;
                        const double U = U10[c], u_star = us[c];
                        if (U > 0.0 && u_star > 0.0 && k > 0.0) {
                            const double sigma = std::sqrt(g * k), C = sigma / k;
                            const double theta = std::atan2(ky, kx);
                            raw = jp_rate(k, sigma, C, theta, th[c], u_star, M->rho_air / M->rho_water,
                                          M->beta_max, M->z_alpha, M->p_in, M->alpha0, M->von_karman, g);
                        }
                        if (raw > 0.0) {
                            const double rate = raw * factor[c];
                            double p, l;
                            if (rate >= 0.0) { p = rate * a; l = 0.0; } else { p = 0.0; l = -rate; }
                            positive += p;
                            damping += l;
                        }
                    }
                    if (M->has_dissipation) {
                        double p = 0.0, l = 0.0;
                        if (a > 0.0 && k > 0.0) {
                            const double sg = M->ds_gravity;
                            const double sigma = std::sqrt(sg * k);
                            const double B = a * sigma * (k * k * k);
                            double ov = B / M->B_r - 1.0;
                            ov = ov > 0.0 ? ov : 0.0;
                            if (ov > 0.0) {
                                ov = ov < 1e6 ? ov : 1e6;
                                const double rate = -M->C_ds * std::pow(sigma, M->sigma_power) * std::pow(ov, M->ds_p);
                                if (rate >= 0.0) { p = 0.0; l = rate; } else { p = -rate * a; l = 0.0; }
                            }
                        }
                        positive += p;
                        damping += l;
                    }
                    G[u] += positive - damping * a;
                }
        }
}

/* ------------------------------------------------------ SourceTermSet terms */

/* Sources.jl:1394-1400 */
static double cosine_power_antiderivative(double a, int power) {
    if (power == 0) return a;
    if (power == 1) return std::sin(a);
    return std::sin(a) * std::pow(std::cos(a), power - 1) / power +
           (double)(power - 1) / power * cosine_power_antiderivative(a, power - 2);
}

/* Sources.jl:1402-1421: integral of max(cos, 0)^power over [a1, a2] */
double ora_positive_cosine_power_integral(double a1, double a2, int power) {
    if (a2 < a1) return -ora_positive_cosine_power_integral(a2, a1, power);
    if (power == 0) return a2 - a1;
    const double period = 2.0 * M_PI;
    const int64_t lo = (int64_t)std::floor((a1 - M_PI / 2) / period) - 1;
    const int64_t hi = (int64_t)std::ceil((a2 + M_PI / 2) / period) + 1;
    double integral = 0.0;
    for (int64_t q = lo; q <= hi; ++q) {
        const double shift = q * period;
        const double left = std::max(a1, shift - M_PI / 2), right = std::min(a2, shift + M_PI / 2);
        if (!(right > left)) continue;
        integral += cosine_power_antiderivative(right - shift, power) - cosine_power_antiderivative(left - shift, power);
    }
    return integral;
}

/* Sources.jl:1423-1434 (polar grid): the cell average of max(cos(phi - direction), 0)^power */
double ora_wind_directional_weight(const ora_model* M, int64_t n, double direction, int power) {
    if (power == 0) return 1.0;
    const double p1 = M->phi_faces[n], p2 = M->phi_faces[n + 1];
    return ora_positive_cosine_power_integral(p1 - direction, p2 - direction, power) / (p2 - p1);
}

/* finite_volume_integration.jl:24-27,29-33,86-88: radial-power average kappa^power over the cell */
double ora_radial_power_average(const ora_model* M, int64_t m, int64_t n, double power) {
    const double k1 = M->kappa_faces[m], k2 = M->kappa_faces[m + 1];
    const double p1 = M->phi_faces[n], p2 = M->phi_faces[n + 1];
    const double meas = (p2 - p1) * (std::pow(k2, power + 2.0) - std::pow(k1, power + 2.0)) / (power + 2.0);
    return meas / M->weights[m + M->Nk * n];
}

static double term_value(double v, const double* field, int64_t c) { return field ? field[c] : v; }

/* Source tendency of the SourceTermSet terms added to G (tendencies.jl:34-36: G += source_tendency; the
 * set sums its terms in order, Sources.jl:443-449). Per-(i,j) integrals as the reference computes them
 * per call: local_zeroth_moment (Sources.jl:1471-1480, n outer m inner, every bin), and for
 * MeanSpectrumWhitecapping the p-th means over bins with N > 0 and k > 0 (mean_spectrum.jl:43-82). */
static void add_source_terms(const ora_model* M, const double* N, double* G) {
    const int64_t Nx = M->Nx, Ny = M->Ny, Nk = M->Nk, Np = M->Np, P = Nx * Ny;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < P; ++c) {
        // per-(i,j) integrals
        double m0 = 0.0;
        for (int64_t n = 0; n < Np; ++n)
            for (int64_t m = 0; m < Nk; ++m) m0 += N[c + P * (m + Nk * n)] * M->weights[m + Nk * n];
        std::vector<double> kbar(M->n_terms, 0.0), sbar(M->n_terms, 0.0);
        for (int32_t t = 0; t < M->n_terms; ++t) {
            const ora_term& T = M->terms[t];
            if (T.kind != ORA_TERM_MEAN_SPECTRUM) continue;
            const double p = T.p[3];
            double nk = 0.0, dk = 0.0, ns = 0.0, ds = 0.0;
            for (int64_t n = 0; n < Np; ++n)
                for (int64_t m = 0; m < Nk; ++m) {
                    const double a = N[c + P * (m + Nk * n)];
                    if (a <= 0.0) continue;
                    const double w = M->weights[m + Nk * n];
                    const double kx = M->kappa[m] * std::cos(M->phi[n]), ky = M->kappa[m] * std::sin(M->phi[n]);
                    const double k = std::hypot(kx, ky);
                    if (k <= 0.0) continue;
                    nk += a * w * std::pow(k, p);
                    dk += a * w;
                    ns += a * w * std::pow(std::sqrt(T.gravity * k), p);
                    ds += a * w;
                }
            kbar[t] = dk > 0.0 ? std::pow(nk / dk, 1.0 / p) : 0.0;
            sbar[t] = ds > 0.0 ? std::pow(ns / ds, 1.0 / p) : 0.0;
        }
        for (int64_t n = 0; n < Np; ++n)
            for (int64_t m = 0; m < Nk; ++m) {
                const int64_t u = c + P * (m + Nk * n);
                const double a = N[u];
                const double kx = M->kappa[m] * std::cos(M->phi[n]), ky = M->kappa[m] * std::sin(M->phi[n]);
                const double k = std::hypot(kx, ky);
                double total = 0.0;
                for (int32_t t = 0; t < M->n_terms; ++t) {
                    const ora_term& T = M->terms[t];
                    double positive = 0.0, damping = 0.0;
                    bool growth = true;   // split_growth_rate of `rate`, else split_damping_rate
                    double rate = 0.0;
                    switch (T.kind) {
                        case ORA_TERM_EXPONENTIAL_WIND:  // Sources.jl:492-496
                            rate = term_value(T.rate, T.rate_field, c) *
                                   ora_wind_directional_weight(M, n, T.direction, (int)T.p[0]);
                            break;
                        case ORA_TERM_WAVE_AGE_WIND: {  // Sources.jl:522-554
                            const double kr = M->kappa[m];   // radial_wavenumber (polar_wavevector_grid.jl:70)
                            if (kr <= 0.0) break;
                            const double al =
                                k == 0.0 ? 0.0 : std::max((kx * std::cos(T.direction) + ky * std::sin(T.direction)) / k, 0.0);
                            if (al == 0.0) break;
                            const double speed = term_value(T.speed, T.speed_field, c);
                            const double inv_age = speed * al / std::sqrt(T.gravity / kr);
                            const double excess = std::max(inv_age - T.p[0], 0.0);
                            rate = term_value(T.rate, T.rate_field, c) * std::pow(excess, T.p[1]) * std::pow(al, T.p[2]);
                            break;
                        }
                        case ORA_TERM_WHITECAPPING: {  // Sources.jl:588-598, 568-573
                            growth = false;
                            const double excess = std::max(m0 / T.p[0] - 1.0, 0.0);
                            const double weighting = T.p[2] == 0.0 ? 1.0
                                                                   : ora_radial_power_average(M, m, n, T.p[2]) /
                                                                         std::pow(T.p[3], T.p[2]);
                            rate = term_value(T.rate, T.rate_field, c) * std::pow(excess, T.p[1]) * weighting;
                            break;
                        }
                        case ORA_TERM_MEAN_SPECTRUM: {  // mean_spectrum.jl:90-111
                            growth = false;
                            if (!(m0 > 0.0) || !(kbar[t] > 0.0) || !(k > 0.0)) break;
                            const double alpha = m0 * kbar[t] * kbar[t];
                            const double ratio = k / kbar[t];
                            const double bracket = T.p[1] * ratio + T.p[2] * ratio * ratio;
                            rate = -T.p[0] * alpha * alpha * sbar[t] * bracket;
                            break;
                        }
                        default:
                            break;
                    }
                    if (growth) {
                        if (rate >= 0.0) positive = rate * a; else damping = -rate;
                    } else {
                        if (rate >= 0.0) damping = rate; else positive = -rate * a;
                    }
                    total += positive - damping * a;
                }
                G[u] += total;
            }
    }
}

/* src/Models/tendencies.jl:28-41,82-101 (dispatch) */
void ora_tendency(const ora_model* M, const double* N, double t, int32_t with_sources, double* G) {
    const int64_t total = M->Nx * M->Ny * M->Nk * M->Np;
    if (M->transport == ORA_TRANSPORT_REFRACTION && M->pm_mode) {
        /* PseudomomentumVelocities: the coupling is refreshed from the stage's action before every
         * tendency (tendencies.jl:103-107, current_coupling.jl:140-143), then the gradients
         * (wave_current_refraction.jl:21-39) and the fused refraction tendency. */
        const int64_t c3 = M->Nx * M->Ny * M->Nk;
        std::vector<double> U(6 * c3);
        ora_pm_doppler_velocity(M->Nx, M->Ny, M->Nk, M->Np, N, M->pm_per_cell, M->pm_overlap, nullptr, M->pm_kx,
                                M->pm_ky, U.data(), U.data() + c3, nullptr, nullptr);
        ora_current_gradients(M->Nx, M->Ny, M->Nk, U.data(), U.data() + c3, 1.0 / M->dx, 1.0 / M->dy,
                              U.data() + 2 * c3, U.data() + 3 * c3, U.data() + 4 * c3, U.data() + 5 * c3);
        ora_model Mc = *M;
        Mc.Ux = U.data();
        Mc.Uy = U.data() + c3;
        Mc.Uxx = U.data() + 2 * c3;
        Mc.Uxy = U.data() + 3 * c3;
        Mc.Uyx = U.data() + 4 * c3;
        Mc.Uyy = U.data() + 5 * c3;
        refraction_tendency(&Mc, N, G);
    } else if (M->transport == ORA_TRANSPORT_REFRACTION) refraction_tendency(M, N, G);
    else if (M->transport == ORA_TRANSPORT_INTRINSIC) intrinsic_tendency(M, N, G);
    else std::memset(G, 0, sizeof(double) * total);
    if (with_sources && (M->wind_kind != ORA_WIND_NONE || M->has_dissipation)) add_sources(M, N, t, G);
    if (with_sources && M->n_terms > 0) add_source_terms(M, N, G);
}

/* src/Models/propagation_smoothing.jl:60-109 (_spatial_averaging_kernel!), :117-158 (tables),
 * :163-199 (apply). Index arithmetic is 1-based like the reference so the bilinear weights round the
 * same way; a corner that one periodic wrap does not bring into range is clamped (the reference would
 * read its halo there; with a CFL-limited dt the corners stay within one cell). */
void ora_spatial_averaging(const ora_model* M, double* N, double dt) { ora_spatial_averaging_at(M, N, dt, 0); }

/* The same with the model's rows at rows y_offset + 1 .. y_offset + Ny of a larger grid (a slab of a
 * y-decomposed domain): corner positions and bilinear weights are computed at the larger grid's row
 * indices, so they round as in the undecomposed run. */
void ora_spatial_averaging_at(const ora_model* M, double* N, double dt, int64_t y_offset) {
    const int64_t Nx = M->Nx, Ny = M->Ny, Nk = M->Nk, Np = M->Np, P = Nx * Ny;
    const double g = 9.81;
    std::vector<double> cg(Nk), dcg(Nk), cs(Np), sn(Np);
    for (int64_t m = 0; m < Nk; ++m) cg[m] = 1.0 / 2.0 * std::sqrt(g / M->kappa[m]);
    for (int64_t m = 0; m < Nk; ++m) {
        const double lo = m == 0 ? cg[0] : 1.0 / 2.0 * std::sqrt(g / M->kappa[m - 1]);
        const double hi = m == Nk - 1 ? cg[Nk - 1] : 1.0 / 2.0 * std::sqrt(g / M->kappa[m + 1]);
        dcg[m] = std::fabs(lo - hi) / 2.0;
    }
    for (int64_t n = 0; n < Np; ++n) {
        cs[n] = std::cos(M->phi[n]);
        sn[n] = std::sin(M->phi[n]);
    }
    const double dphi = M->phi_faces[1] - M->phi_faces[0];
    const double dx_inv = 1.0 / M->dx, dy_inv = 1.0 / M->dy;
    const double as = M->gse_alpha_s, an = M->gse_alpha_n;
    auto wrap = [](int64_t i, int64_t n, int32_t periodic) {
        if (periodic) i = i < 1 ? i + n : (i > n ? i - n : i);
        return i < 1 ? (int64_t)1 : (i > n ? n : i);
    };
    std::vector<double> out((size_t)(P * Nk * Np));
#pragma omp parallel for collapse(2) schedule(static)
    for (int64_t n = 0; n < Np; ++n)
        for (int64_t m = 0; m < Nk; ++m) {
            const double Ls = as * dcg[m] * dt, Ln = an * cg[m] * dphi * dt;
            const double Ls_x = Ls * cs[n] * dx_inv, Ls_y = Ls * sn[n] * dy_inv;
            const double Ln_x = -Ln * sn[n] * dx_inv, Ln_y = Ln * cs[n] * dy_inv;
            const double* plane = N + P * (m + Nk * n);
            for (int64_t j = 1; j <= Ny; ++j)
                for (int64_t i = 1; i <= Nx; ++i) {
                    double acc = 0.0;
                    for (int s1 = -1; s1 <= 1; s1 += 2)
                        for (int s2 = -1; s2 <= 1; s2 += 2) {
                            const double di = s1 * Ls_x + s2 * Ln_x, dj = s1 * Ls_y + s2 * Ln_y;
                            const double ir = (double)i + di, jr = (double)(j + y_offset) + dj;
                            const double fi = std::floor(ir), fj = std::floor(jr);
                            const int64_t i0 = (int64_t)fi, j0 = (int64_t)fj - y_offset;
                            const double wi = ir - (double)i0, wj = jr - fj;
                            const int64_t i0c = wrap(i0, Nx, M->periodic_x), i1c = wrap(i0 + 1, Nx, M->periodic_x);
                            const int64_t j0c = wrap(j0, Ny, M->periodic_y), j1c = wrap(j0 + 1, Ny, M->periodic_y);
                            const double f00 = plane[(i0c - 1) + Nx * (j0c - 1)], f10 = plane[(i1c - 1) + Nx * (j0c - 1)];
                            const double f01 = plane[(i0c - 1) + Nx * (j1c - 1)], f11 = plane[(i1c - 1) + Nx * (j1c - 1)];
                            acc += (1.0 - wi) * (1.0 - wj) * f00 + wi * (1.0 - wj) * f10 + (1.0 - wi) * wj * f01 +
                                   wi * wj * f11;
                        }
                    out[(size_t)((i - 1) + Nx * (j - 1) + P * (m + Nk * n))] = acc / 4.0;
                }
        }
    std::memcpy(N, out.data(), sizeof(double) * out.size());
}

/* src/Models/time_step.jl:138-152,168 (SSP-RK3 with max(0,.) after every stage kernel) */
void ora_rk3_step(const ora_model* M, double* N, double dt, int64_t nsteps, double* t) {
    const int64_t total = M->Nx * M->Ny * M->Nk * M->Np;
    std::vector<double> N0(total), G(total);
    const double a2 = 0.75, b2 = 0.25, a3 = 1.0 / 3.0, b3 = 2.0 / 3.0;
    for (int64_t s = 0; s < nsteps; ++s) {
        std::memcpy(N0.data(), N, sizeof(double) * total);
        ora_tendency(M, N, *t, 1, G.data());
#pragma omp parallel for schedule(static)
        for (int64_t u = 0; u < total; ++u) N[u] = relu(N[u] + dt * G[u]);
        ora_tendency(M, N, *t, 1, G.data());
#pragma omp parallel for schedule(static)
        for (int64_t u = 0; u < total; ++u) {
            const double stage = relu(N[u] + dt * G[u]);
            N[u] = relu(a2 * N0[u] + b2 * stage);
        }
        ora_tendency(M, N, *t, 1, G.data());
#pragma omp parallel for schedule(static)
        for (int64_t u = 0; u < total; ++u) {
            const double stage = relu(N[u] + dt * G[u]);
            N[u] = relu(a3 * N0[u] + b3 * stage);
        }
        if (M->gse) ora_spatial_averaging(M, N, dt);  /* time_step.jl:168 */
        *t += dt;
    }
}

/* --------------------------------------------------------- diagnostics */

/* src/Diagnostics/moments.jl:33-37,100-123; diagnostic_operations.jl:56-165,480-509;
 * bulk_statistics.jl:9,87-91; moment measures polar_wavevector_grid.jl:73-115.
 * Per-(i,j) sums run n outer, m inner like the reference kernels. The total action uses a
 * Neumaier-compensated sum over (i,j) of m0·Δx(i)·Δy(j) with each cell's own widths. Any output
 * pointer may be NULL. */
void ora_diagnostics(const ora_model* M, const double* N, double* m0, double* hs, double* krms,
                     double* mean_dir, double* total_action) {
    const int64_t Nx = M->Nx, Ny = M->Ny, Nk = M->Nk, Np = M->Np;
    std::vector<double> mux(Nk * Np), muy(Nk * Np), trace(Nk * Np);
    for (int64_t n = 0; n < Np; ++n)
        for (int64_t m = 0; m < Nk; ++m) {
            const double k1 = M->kappa_faces[m], k2 = M->kappa_faces[m + 1];
            const double p1 = M->phi_faces[n], p2 = M->phi_faces[n + 1];
            const double r1 = (k2 * k2 * k2 - k1 * k1 * k1) / 3.0;
            mux[m + Nk * n] = r1 * (std::sin(p2) - std::sin(p1));
            muy[m + Nk * n] = r1 * (std::cos(p1) - std::cos(p2));
            const double r2 = (std::pow(k2, 4.0) - std::pow(k1, 4.0)) / 4.0;
            const double dp = p2 - p1, s2 = std::sin(2.0 * p2) - std::sin(2.0 * p1);
            const double cc = dp / 2.0 + s2 / 4.0, ss = dp / 2.0 - s2 / 4.0;
            trace[m + Nk * n] = r2 * cc + r2 * ss;
        }
    std::vector<double> col(Nx * Ny);
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < Ny; ++j)
        for (int64_t i = 0; i < Nx; ++i) {
            double s0 = 0.0, sx = 0.0, sy = 0.0, st = 0.0;
            for (int64_t n = 0; n < Np; ++n)
                for (int64_t m = 0; m < Nk; ++m) {
                    const double a = N[i + Nx * (j + Ny * (m + Nk * n))];
                    s0 += a * M->weights[m + Nk * n];
                    sx += a * mux[m + Nk * n];
                    sy += a * muy[m + Nk * n];
                    st += a * trace[m + Nk * n];
                }
            const int64_t c = i + Nx * j;
            col[c] = s0;
            if (m0) m0[c] = s0;
            if (hs) hs[c] = 4.0 * std::sqrt(s0);
            if (krms) krms[c] = std::sqrt(s0 == 0.0 ? 0.0 : st / s0);
            if (mean_dir) mean_dir[c] = std::atan2(sy, sx);
        }
    if (total_action) {
        double sum = 0.0, comp = 0.0;
        for (int64_t c = 0; c < Nx * Ny; ++c) {
            const double ddx = M->xspacings ? M->xspacings[c % Nx] : M->dx;
            const double ddy = M->yspacings ? M->yspacings[c / Nx] : M->dy;
            const double v = col[c] * ddx * ddy;   /* diagnostic_operations.jl:502: acc * Δx * Δy */
            const double tsum = sum + v;
            if (std::fabs(sum) >= std::fabs(v)) comp += (sum - tsum) + v;
            else comp += (v - tsum) + sum;
            sum = tsum;
        }
        *total_action = sum + comp;
    }
}

int ora_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void ora_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

}  // extern "C"
