// rpl_setup.cu -- set-up and per-step auxiliary kernels: Q-transform Doppler velocity and its
// kappa derivative, periodic current gradients, finite-depth group speed field, wind fields and
// the wave-supported stress cap, diagnostics reductions, dtype conversion.
#include <cuda_runtime.h>
#include <float.h>

#include <algorithm>

#include "rpl_device.cuh"
#include "rpl_internal.h"
#include "rpl_src32.cuh"

namespace rpl {

namespace {

// Q weight of vertical cell k for ring m at column depth d (q_kernel.jl:87-116): F(z_k+1) - F(z_k), or
// with derivative the same difference of dF/dkappa.
__device__ __forceinline__ double q_weight(double kap, double lo, double hi, double d, double small_mu,
                                           int exact_form, int derivative) {
    return derivative ? q_cdf_dk(kap, hi, d, small_mu) - q_cdf_dk(kap, lo, d, small_mu)
                      : q_cdf(kap, hi, d, small_mu, exact_form) - q_cdf(kap, lo, d, small_mu, exact_form);
}

// Q weights W[k,m] and Wd[k,m] of one constant projection depth, (Nz, Nk) with m fastest.
__global__ void q_table_kernel(int64_t Nz, int64_t Nk, const double* __restrict__ zf, double d,
                               const double* __restrict__ kappa, double small_mu, int exact_form,
                               double* __restrict__ W, double* __restrict__ Wd) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= Nz * Nk) return;
    const int64_t k = t / Nk, m = t - k * Nk;
    const double kap = kappa[m], lo = zf[k], hi = zf[k + 1];
    W[t] = q_weight(kap, lo, hi, d, small_mu, exact_form, 0);
    Wd[t] = q_weight(kap, lo, hi, d, small_mu, exact_form, 1);
}

// Per-column Q weights of a depth field, column-contiguous (Nz, Nk) blocks with m fastest, stored as TW.
// One warp per column, lanes over the rings; each lane walks the faces once (a face's F serves the two
// cells that share it).
template <typename TW>
__global__ void q_column_table_kernel(int64_t P, int64_t Nz, int64_t Nk, const double* __restrict__ zf,
                                      const double* __restrict__ qdepth, const double* __restrict__ kappa,
                                      double small_mu, int exact_form, TW* __restrict__ W) {
    const int lane = threadIdx.x & 31;
    const int64_t col = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (col >= P) return;
    const double d = qdepth[col];
    TW* w = W + col * Nz * Nk;
    for (int64_t m = lane; m < Nk; m += 32) {
        const double kap = kappa[m];
        double F0 = q_cdf(kap, zf[0], d, small_mu, exact_form);
        for (int64_t k = 0; k < Nz; ++k) {
            const double F1 = q_cdf(kap, zf[k + 1], d, small_mu, exact_form);
            w[k * Nk + m] = (TW)(F1 - F0);
            F0 = F1;
        }
    }
}

// U[i,j,m] = sum_k uL[i,j,k] * W_m[k] (doppler_velocity.jl:45-62; with derivative the dF/dkappa
// weights of :64-82), sequential in k like the reference. One warp per (i,j) column, lanes over the
// kappa rings (chunks of 32); u, v are warp-uniform loads; U is written in device order c*Nk + m
// (coalesced). The weights come from a shared (Nz, Nk)
// table (W, col_stride 0), a per-column table (col_stride Nz*Nk), or are evaluated here (W null; each
// face once). z faces are strictly increasing (checked by the caller).
template <typename TW>
__global__ void doppler_kernel(int64_t Nx, int64_t Ny, int64_t Nz, int64_t Nk,
                               const double* __restrict__ u, const double* __restrict__ v,
                               const double* __restrict__ zf, const double* __restrict__ qdepth,
                               double qdepth_const, const double* __restrict__ kappa, double small_mu,
                               int exact_form, int derivative, const TW* __restrict__ W, int64_t col_stride,
                               double* __restrict__ Ux, double* __restrict__ Uy) {
    const int lane = threadIdx.x & 31;
    const int64_t col = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t P = Nx * Ny;
    if (col >= P) return;
    const double d = qdepth ? qdepth[col] : qdepth_const;
    for (int64_t m0 = 0; m0 < Nk; m0 += 32) {
        const int64_t m = m0 + lane;
        const bool active = m < Nk;
        const int64_t mm = active ? m : Nk - 1;
        double ax = 0.0, ay = 0.0;
        if (W) {
            const TW* w = W + col * col_stride + mm;
#pragma unroll 4
            for (int64_t k = 0; k < Nz; ++k) {
                const double wk = (double)__ldg(w + k * Nk);
                ax += __ldg(u + col + P * k) * wk;
                ay += __ldg(v + col + P * k) * wk;
            }
        } else {
            const double kap = kappa[mm];
            double F0 = derivative ? q_cdf_dk(kap, zf[0], d, small_mu) : q_cdf(kap, zf[0], d, small_mu, exact_form);
            for (int64_t k = 0; k < Nz; ++k) {
                const double z1 = zf[k + 1];
                const double F1 = derivative ? q_cdf_dk(kap, z1, d, small_mu) : q_cdf(kap, z1, d, small_mu, exact_form);
                const double wk = F1 - F0;
                ax += __ldg(u + col + P * k) * wk;
                ay += __ldg(v + col + P * k) * wk;
                F0 = F1;
            }
        }
        if (active) {
            Ux[col * Nk + m] = ax;
            Uy[col * Nk + m] = ay;
        }
    }
}

// Periodic centred differences of Ux, Uy (wave_current_refraction.jl:7-19).
__global__ void gradients_kernel(int64_t Nx, int64_t Ny, int64_t Nk, const double* __restrict__ Ux,
                                 const double* __restrict__ Uy, double dx_inv, double dy_inv,
                                 double* __restrict__ Uxx, double* __restrict__ Uxy,
                                 double* __restrict__ Uyx, double* __restrict__ Uyy) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= Nx * Ny * Nk) return;
    const int64_t i = t % Nx, j = (t / Nx) % Ny, k = t / (Nx * Ny);
    const int64_t ip = i == Nx - 1 ? 0 : i + 1, im = i == 0 ? Nx - 1 : i - 1;
    const int64_t jp = j == Ny - 1 ? 0 : j + 1, jm = j == 0 ? Ny - 1 : j - 1;
    const int64_t o = Nx * Ny * k;
    Uxx[t] = (Ux[ip + Nx * j + o] - Ux[im + Nx * j + o]) * (dx_inv / 2.0);
    Uxy[t] = (Ux[i + Nx * jp + o] - Ux[i + Nx * jm + o]) * (dy_inv / 2.0);
    Uyx[t] = (Uy[ip + Nx * j + o] - Uy[im + Nx * j + o]) * (dx_inv / 2.0);
    Uyy[t] = (Uy[i + Nx * jp + o] - Uy[i + Nx * jm + o]) * (dy_inv / 2.0);
}

// Cell-centre finite-depth group speed per (i,j,m) (transport.jl:72-83 without the direction):
// cg = (1 + 2mu/sinh(2mu))/2 * sqrt(g tanh(mu)/k), mu = k d.
__global__ void cg_field_kernel(int64_t Nx, int64_t Ny, int64_t Nk, const double* __restrict__ depth,
                                const double* __restrict__ kappa, double g, double* __restrict__ cg) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= Nx * Ny * Nk) return;
    const int64_t c = t % (Nx * Ny), m = t / (Nx * Ny);
    const double k = kappa[m], h = depth[c];
    const double mu = k * h;
    const double cp = sqrt(g * tanh(mu) / k);
    const double gf = (1.0 + 2.0 * mu / sinh(2.0 * mu)) / 2.0;
    cg[t] = gf * cp;
}

struct WindArgs {
    int kind, rotation, drag_form;
    double speed, direction;
    double vmax, rmax, radius, shape, inflow, bx, by, cx, cy;  // cx, cy: storm centre at t
    double alpha0, g;                                            // Charnock constant, gravity
};

__device__ __forceinline__ double friction_velocity(double U, int form) {
    double cd;
    if (form == 0) cd = (0.8 + 0.065 * U) * 1e-3;  // drag.jl:77-78
    else {
        cd = (8.058 + 0.967 * U - 0.016 * (U * U)) * 1e-4;  // drag.jl:80-83
        cd = cd > 4e-4 ? cd : 4e-4;
    }
    return U * sqrt(cd > 0.0 ? cd : 0.0);
}

// Per-(i,j) wind speed, direction and friction velocity at one time (winds.jl:255-315,
// pressure_correlation.jl:54-63, drag.jl:85-86).
__global__ void wind_kernel(int64_t Nx, int64_t Ny, const double* __restrict__ xn, const double* __restrict__ yn,
                            WindArgs w, double* __restrict__ U10, double* __restrict__ theta,
                            double* __restrict__ ustar, float* __restrict__ cell32) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= Nx * Ny) return;
    double U = 0.0, th = 0.0;
    if (w.kind == RPL_WIND_UNIFORM) {
        U = w.speed;
        th = w.direction;
    } else if (w.kind == RPL_WIND_HOLLAND) {
        const double dx = xn[c % Nx] - w.cx, dy = yn[c / Nx] - w.cy;
        const double r = hypot(dx, dy);
        double vx = w.bx, vy = w.by;
        if (r != 0.0) {
            const double scaled = w.rmax / r;
            const double shape = pow(scaled, w.shape);
            const double e = shape * exp(1.0 - shape);
            double speed = w.vmax * sqrt(e > 0.0 ? e : 0.0);
            if (r > w.radius) {
                const double dd = w.radius - w.rmax;
                const double ulp = nextafter(w.radius, INFINITY) - w.radius;
                speed *= exp(-(r - w.radius) / (dd > ulp ? dd : ulp));
            }
            const double s = (double)w.rotation;
            const double tx = -s * dy / r, ty = s * dx / r, rx = dx / r, ry = dy / r;
            const double ci = cos(w.inflow), si = sin(w.inflow);
            vx = speed * (ci * tx - si * rx) + w.bx;
            vy = speed * (ci * ty - si * ry) + w.by;
        }
        U = hypot(vx, vy);
        th = atan2(vy, vx);
    } else if (w.kind == RPL_WIND_FIELD) {
        U = U10[c];
        th = theta[c];
    }
    const double us = friction_velocity(U, w.drag_form);
    U10[c] = U;
    theta[c] = th;
    ustar[c] = us;
    // FP32 per-cell wind constants (rpl_src32.cuh); the stress kernel fills slot 5
    const double z1 = w.alpha0 * (us * us) / w.g;
    const bool on = U > 0.0 && us > 0.0 && z1 > 0.0;
    float4* rec = reinterpret_cast<float4*>(cell32 + 8 * c);
    rec[0] = make_float4(on ? (float)us : 0.0f, on ? (float)log(z1) : 0.0f, (float)cos(th), (float)sin(th));
    reinterpret_cast<float*>(rec + 1)[0] = on ? 1.0f : 0.0f;
}

// Wave-supported stress cap per (i,j) (precomputed_sources.jl:282-326): tau_w along the wind from
// the current spectrum; factor = min(1, 0.4 tau_max / tau_w). Loop n outer, m inner as the reference.
template <typename T>
__global__ void stress_kernel(const T* __restrict__ N, StageParams p, double rho_w_g, double rho_air,
                              double* __restrict__ factor) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t P = p.Nx * p.Ny;
    if (c >= P) return;
    const double U = p.wind_U10[c], u_star = p.wind_ustar[c];
    double f = 1.0;
    if (U > 0.0 && u_star > 0.0) {
        const double tu = p.wind_theta[c];
        const double tau_max = rho_air * (u_star * u_star);
        double twx = 0.0, twy = 0.0;
        for (int n = 0; n < p.Np; ++n) {
            const double cth = p.cosp[n], sth = p.sinp[n];
            for (int m = 0; m < p.Nk; ++m) {
                const double a = (double)N[((int64_t)n * P + c) * p.Nk + m];
                const double k = p.kappa[m];
                if (a > 0.0 && k > 0.0) {
                    const double theta = p.phi[n];
                    const double rate = jp_rate(k, theta, tu, u_star, p);
                    if (rate > 0.0) {
                        const double sigma = sqrt(p.wind_g * k), C = sigma / k;
                        const double mflux = rate * a / C * p.weights[m + p.Nk * n] * rho_w_g;
                        twx += mflux * cth;
                        twy += mflux * sth;
                    }
                }
            }
        }
        const double par = twx * cos(tu) + twy * sin(tu);
        const double eff = par > 0.0 ? par : 0.0;
        f = (eff > 0.4 * tau_max && tau_max > 0.0) ? 0.4 * tau_max / eff : 1.0;
    }
    factor[c] = f;
}

// Neumaier compensated accumulation.
__device__ __forceinline__ void kadd(double& s, double& c, double v) {
    const double t = s + v;
    if (fabs(s) >= fabs(v)) c += (s - t) + v;
    else c += (v - t) + s;
    s = t;
}

// Per-(i,j) spectral sums (diagnostic_operations.jl:56-165): m0 = sum N w, Hs = 4 sqrt(m0),
// kappa_rms = sqrt(sum N trace / m0) (0 when m0 = 0), mean direction = atan(sum N mu_y, sum N mu_x).
// Exact error of s + v folded into the compensation c (Knuth's two-sum: branch-free, and the same error
// term as the branch form of kadd).
__device__ __forceinline__ void tadd(double& s, double& c, double v) {
    const double t = s + v;
    const double bp = t - s;
    c += (s - (t - bp)) + (v - bp);
    s = t;
}

// Per-(i,j) moments (moments.jl:33-37,100-123): one warp per column, lanes over the kappa rings
// (coalesced reads of each direction's kappa column); per lane, FP64 sums of blocks of 4 directions
// folded into compensated totals, then a fixed-order compensated butterfly over the lanes
// (deterministic). The error stays within a few units in the last place of the sum of |terms|.
// ALL = false computes m0 alone (for the total action), with the same arithmetic for m0.
template <typename T, bool ALL>
__global__ void __launch_bounds__(256)
diag_kernel(const T* __restrict__ N, int64_t Nx, int64_t Ny, int64_t Nk, int64_t Np,
            const double* __restrict__ tabs, double* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int64_t c = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t P = Nx * Ny;
    if (c >= P) return;
    const int64_t nb = Nk * Np;
    const double* w = tabs;
    const double* mux = tabs + nb;
    const double* muy = tabs + 2 * nb;
    const double* tr = tabs + 3 * nb;
    double s0 = 0, c0 = 0, sx = 0, cx = 0, sy = 0, cy = 0, st = 0, ct = 0;
    const int64_t stride = P * Nk;  // between directions
    const int nk = (int)Nk, np = (int)Np;
    for (int m = lane; m < nk; m += 32) {
        const T* p = N + c * Nk + m;
        // chunks of CH directions: the chunk's loads are issued together (memory-level parallelism), then
        // its blocks of DB directions are summed with FMAs and each block sum is folded into the
        // compensated totals, block by block in direction order
        constexpr int DB = 4, CH = 3 * DB;
        for (int n0 = 0; n0 < np; n0 += CH, p += CH * stride) {
            T a[CH];
#pragma unroll
            for (int k = 0; k < CH; ++k) a[k] = n0 + k < np ? p[k * stride] : T(0);
#pragma unroll
            for (int q = 0; q < CH; q += DB) {
                if (n0 + q >= np) break;
                double b0 = 0.0, bx = 0.0, by = 0.0, bt = 0.0;
#pragma unroll
                for (int k = q; k < q + DB; ++k) {
                    const int b = n0 + k < np ? m + nk * (n0 + k) : m;  // a[k] = 0 past the last direction
                    const double ak = (double)a[k];
                    b0 = fma(ak, __ldg(w + b), b0);
                    if (ALL) {
                        bx = fma(ak, __ldg(mux + b), bx);
                        by = fma(ak, __ldg(muy + b), by);
                        bt = fma(ak, __ldg(tr + b), bt);
                    }
                }
                tadd(s0, c0, b0);
                if (ALL) {
                    tadd(sx, cx, bx);
                    tadd(sy, cy, by);
                    tadd(st, ct, bt);
                }
            }
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        double so = __shfl_down_sync(0xffffffffu, s0, off), co = __shfl_down_sync(0xffffffffu, c0, off);
        tadd(s0, c0, so);
        c0 += co;
        if (ALL) {
            so = __shfl_down_sync(0xffffffffu, sx, off), co = __shfl_down_sync(0xffffffffu, cx, off);
            tadd(sx, cx, so);
            cx += co;
            so = __shfl_down_sync(0xffffffffu, sy, off), co = __shfl_down_sync(0xffffffffu, cy, off);
            tadd(sy, cy, so);
            cy += co;
            so = __shfl_down_sync(0xffffffffu, st, off), co = __shfl_down_sync(0xffffffffu, ct, off);
            tadd(st, ct, so);
            ct += co;
        }
    }
    if (lane == 0) {
        const double m0 = s0 + c0;
        out[c] = m0;
        if (ALL) {
            const double mx = sx + cx, my = sy + cy, mt = st + ct;
            out[P + c] = 4.0 * sqrt(m0);
            out[2 * P + c] = sqrt(m0 == 0.0 ? 0.0 : mt / m0);
            out[3 * P + c] = atan2(my, mx);
        }
    }
}

// Total action = sum_ij m0 dx dy with a compensated, deterministic two-level reduction.
// Total action: compensated sum over (i,j) of m0(i,j)·Δx(i)·Δy(j), each cell with its own widths
// (diagnostic_operations.jl:492-503, bulk_statistics.jl:87-91).
__global__ void total_kernel(const double* __restrict__ m0, int64_t Nx, int64_t P, const double* __restrict__ xsp,
                             const double* __restrict__ ysp, double* __restrict__ total) {
    __shared__ double ss[1024], cc[1024];
    double s = 0.0, c = 0.0;
    const int64_t Ny = P / Nx;
    for (int64_t j = 0; j < Ny; ++j)
        for (int64_t i = threadIdx.x; i < Nx; i += blockDim.x) kadd(s, c, m0[j * Nx + i] * xsp[i] * ysp[j]);
    ss[threadIdx.x] = s;
    cc[threadIdx.x] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        double S = 0.0, C = 0.0;
        for (unsigned k = 0; k < blockDim.x; ++k) {
            kadd(S, C, ss[k]);
            C += cc[k];
        }
        *total = S + C;
    }
}

template <typename T>
__global__ void nonfinite_kernel(const T* __restrict__ x, int64_t n, unsigned int* err) {
    bool bad = false;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        bad |= !isfinite(x[t]);
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(err, 2u);
}

inline unsigned blocks_for(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

}  // namespace

cudaError_t launch_q_table(const Handle& h, int64_t Nz, const double* d_zf, double qdepth_const, double small_mu,
                           double* W, double* Wd, cudaStream_t s) {
    const int64_t n = Nz * h.desc.Nk;
    const int exact_form = h.precision == RPL_FP64 ? 1 : 0;
    q_table_kernel<<<blocks_for(n, 256), 256, 0, s>>>(Nz, h.desc.Nk, d_zf, qdepth_const, h.d_kappa, small_mu,
                                                      exact_form, W, Wd);
    return cudaGetLastError();
}

cudaError_t launch_q_column_table(const Handle& h, cudaStream_t s) {
    const int64_t P = h.cells;
    const int exact_form = h.precision == RPL_FP64 ? 1 : 0;
    if (h.q_col_f32)
        q_column_table_kernel<float><<<blocks_for(P * 32, 256), 256, 0, s>>>(
            P, h.q_Nz, h.desc.Nk, h.d_qz, h.d_qdepth, h.d_kappa, h.q_small_mu, exact_form, (float*)h.d_qcol);
    else
        q_column_table_kernel<double><<<blocks_for(P * 32, 256), 256, 0, s>>>(
            P, h.q_Nz, h.desc.Nk, h.d_qz, h.d_qdepth, h.d_kappa, h.q_small_mu, exact_form, (double*)h.d_qcol);
    return cudaGetLastError();
}

cudaError_t launch_doppler(const Handle& h, const double* d_u, const double* d_v, int derivative, double* Ux,
                           double* Uy, cudaStream_t s) {
    const rpl_desc& d = h.desc;
    const int64_t cols = d.Nx * d.Ny, Nz = h.q_Nz, tab = Nz * d.Nk;
    const int exact_form = h.precision == RPL_FP64 ? 1 : 0;
    const unsigned blocks = blocks_for(cols * 32, 256);
    if (h.d_qW) {  // constant projection depth: shared tables
        doppler_kernel<double><<<blocks, 256, 0, s>>>(d.Nx, d.Ny, Nz, d.Nk, d_u, d_v, h.d_qz, nullptr, h.q_const,
                                                      h.d_kappa, h.q_small_mu, exact_form, derivative,
                                                      h.d_qW + (derivative ? tab : 0), 0, Ux, Uy);
    } else if (h.d_qcol && !derivative) {  // depth field with cached per-column weights
        if (h.q_col_f32)
            doppler_kernel<float><<<blocks, 256, 0, s>>>(d.Nx, d.Ny, Nz, d.Nk, d_u, d_v, h.d_qz, h.d_qdepth, 0.0,
                                                         h.d_kappa, h.q_small_mu, exact_form, 0,
                                                         (const float*)h.d_qcol, tab, Ux, Uy);
        else
            doppler_kernel<double><<<blocks, 256, 0, s>>>(d.Nx, d.Ny, Nz, d.Nk, d_u, d_v, h.d_qz, h.d_qdepth, 0.0,
                                                          h.d_kappa, h.q_small_mu, exact_form, 0,
                                                          (const double*)h.d_qcol, tab, Ux, Uy);
    } else {  // depth field, weights evaluated per column
        doppler_kernel<double><<<blocks, 256, 0, s>>>(d.Nx, d.Ny, Nz, d.Nk, d_u, d_v, h.d_qz, h.d_qdepth, 0.0,
                                                      h.d_kappa, h.q_small_mu, exact_form, derivative, nullptr, 0,
                                                      Ux, Uy);
    }
    return cudaGetLastError();
}

cudaError_t launch_gradients(const Handle& h, cudaStream_t s) {
    const rpl_desc& d = h.desc;
    const int64_t c3 = d.Nx * d.Ny * d.Nk;
    gradients_kernel<<<blocks_for(c3, 256), 256, 0, s>>>(
        d.Nx, d.Ny, d.Nk, h.d_coupling, h.d_coupling + c3, 1.0 / d.dx, 1.0 / d.dy, h.d_coupling + 4 * c3,
        h.d_coupling + 5 * c3, h.d_coupling + 6 * c3, h.d_coupling + 7 * c3);
    return cudaGetLastError();
}

cudaError_t launch_cg_field(const Handle& h, cudaStream_t s) {
    const rpl_desc& d = h.desc;
    const int64_t c3 = d.Nx * d.Ny * d.Nk;
    cg_field_kernel<<<blocks_for(c3, 256), 256, 0, s>>>(d.Nx, d.Ny, d.Nk, h.d_depth, h.d_kappa, d.gravity,
                                                         h.d_cgmag);
    return cudaGetLastError();
}

cudaError_t launch_wind(const Handle& h, double t, cudaStream_t s) {
    const rpl_desc& d = h.desc;
    const int64_t P = d.Nx * d.Ny;
    WindArgs w{};
    w.kind = h.src.wind_kind;
    w.rotation = h.src.rotation;
    w.drag_form = h.src.drag_form;
    w.speed = h.src.wind_speed;
    w.direction = h.src.wind_direction;
    w.vmax = h.src.vmax; w.rmax = h.src.rmax; w.radius = h.src.radius; w.shape = h.src.shape_parameter;
    w.inflow = h.src.inflow_angle; w.bx = h.src.background_x; w.by = h.src.background_y;
    // Storm centre on the LinearStormTrack at t (winds.jl:139-152), host side.
    const int64_t n = (int64_t)h.track_t.size();
    if (n == 0) {
        w.cx = h.track_x.empty() ? 0.0 : h.track_x[0];
        w.cy = h.track_y.empty() ? 0.0 : h.track_y[0];
    } else if (t <= h.track_t[0]) {
        w.cx = h.track_x[0]; w.cy = h.track_y[0];
    } else if (t >= h.track_t[n - 1]) {
        w.cx = h.track_x[n - 1]; w.cy = h.track_y[n - 1];
    } else {
        int64_t up = 0;
        while (h.track_t[up] < t) ++up;
        const int64_t lo = up - 1;
        const double wt = (t - h.track_t[lo]) / (h.track_t[up] - h.track_t[lo]);
        w.cx = (1.0 - wt) * h.track_x[lo] + wt * h.track_x[up];
        w.cy = (1.0 - wt) * h.track_y[lo] + wt * h.track_y[up];
    }
    // xnodes / ynodes live after the wind arrays in the same allocation
    const double* xn = h.d_wind + 4 * P;
    const double* yn = xn + d.Nx;
    w.alpha0 = h.src.alpha0;
    w.g = h.src.wind_gravity;
    wind_kernel<<<blocks_for(P, 256), 256, 0, s>>>(d.Nx, d.Ny, xn, yn, w, h.d_wind, h.d_wind + P,
                                                    h.d_wind + 2 * P, h.d_cell32);
    return cudaGetLastError();
}

// FP32 form of stress_kernel: one warp per (i,j), lane m over kappa bins m, m+32, ...; each lane sums
// its bins over the direction ring in FP32, then the warp reduces. Writes the factor to the FP32 cell
// record (slot 5) and to the FP64 factor field.
__global__ void stress32_kernel(const float* __restrict__ N, StageParams p, float rho_w_g, float rho_air,
                                float* cell32, double* __restrict__ factor, const unsigned int* __restrict__ only) {
    const int64_t c = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int64_t P = p.Nx * p.Ny;
    if (c >= P) return;  // uniform per warp
    if (only && only[c] == 0) return;  // learned source: only cells that fall back need the cap
    const float* r = cell32 + 8 * c;
    const Cell32 q{r[0], r[1], r[2], r[3], r[4], 1.0f, 0.0f, 0.0f};
    float f = 1.0f;
    if (q.on > 0.5f) {
        float twx = 0.0f, twy = 0.0f;
        for (int m = lane; m < (int)p.Nk; m += 32) {
            const Bin32 b = load_bin32(p.bin32 + 8 * m);
            for (int n = 0; n < (int)p.Np; ++n) {
                const float2 cs = __ldg(p.cs32 + n);
                const float a = __ldg(N + ((int64_t)n * P + c) * p.Nk + m);
                float cos_tu;
                const float rate = wind_rate32(p, q, b, cs.x, cs.y, cos_tu);
                const float mf = a > 0.0f ? rate * a * b.invC * __ldg(p.w32 + m + p.Nk * n) : 0.0f;
                twx = fmaf(mf, cs.x, twx);
                twy = fmaf(mf, cs.y, twy);
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            twx += __shfl_xor_sync(0xffffffffu, twx, o);
            twy += __shfl_xor_sync(0xffffffffu, twy, o);
        }
        const float par = fmaf(twx, q.cu, twy * q.su) * rho_w_g;
        const float tau_max = rho_air * (q.ustar * q.ustar);
        const float eff = fmaxf(par, 0.0f);
        f = (eff > 0.4f * tau_max && tau_max > 0.0f) ? 0.4f * tau_max / eff : 1.0f;
    }
    if (lane == 0) {
        cell32[8 * c + 5] = f;
        factor[c] = (double)f;
    }
}

cudaError_t launch_stress_factor(const Handle& h, const void* Nin, cudaStream_t s, const unsigned int* only) {
    const rpl_desc& d = h.desc;
    const int64_t P = d.Nx * d.Ny;
    StageParams p = make_params(h, 1.0, 1);
    const double rho_w_g = h.src.rho_water * h.src.wind_gravity;
    if (h.precision == RPL_FP64)
        stress_kernel<double><<<blocks_for(P, 128), 128, 0, s>>>((const double*)Nin, p, rho_w_g, h.src.rho_air,
                                                                 h.d_wind + 3 * P);
    else
        stress32_kernel<<<blocks_for(P * 32, 256), 256, 0, s>>>((const float*)Nin, p, (float)rho_w_g,
                                                                (float)h.src.rho_air, h.d_cell32, h.d_wind + 3 * P, only);
    return cudaGetLastError();
}

cudaError_t launch_diagnostics(const Handle& h, const void* Nin, cudaStream_t s, bool moments) {
    const rpl_desc& d = h.desc;
    const int64_t P = d.Nx * d.Ny;
    const unsigned blocks = blocks_for(P * 32, 256);
    if (h.precision == RPL_FP64) {
        if (moments)
            diag_kernel<double, true><<<blocks, 256, 0, s>>>((const double*)Nin, d.Nx, d.Ny, d.Nk, d.Np, h.d_weights,
                                                             h.d_diag);
        else
            diag_kernel<double, false><<<blocks, 256, 0, s>>>((const double*)Nin, d.Nx, d.Ny, d.Nk, d.Np,
                                                              h.d_weights, h.d_diag);
    } else {
        if (moments)
            diag_kernel<float, true><<<blocks, 256, 0, s>>>((const float*)Nin, d.Nx, d.Ny, d.Nk, d.Np, h.d_weights,
                                                            h.d_diag);
        else
            diag_kernel<float, false><<<blocks, 256, 0, s>>>((const float*)Nin, d.Nx, d.Ny, d.Nk, d.Np, h.d_weights,
                                                             h.d_diag);
    }
    total_kernel<<<1, 1024, 0, s>>>(h.d_diag, d.Nx, P, h.d_spacing, h.d_spacing + d.Nx, h.d_diag + 4 * P);
    return cudaGetLastError();
}

cudaError_t launch_scan_nonfinite(const Handle& h, const void* buf, cudaStream_t s) {
    const unsigned blocks = (unsigned)std::min<int64_t>(blocks_for(h.units, 256), 148 * 32);
    if (h.precision == RPL_FP64)
        nonfinite_kernel<double><<<blocks, 256, 0, s>>>((const double*)buf, h.units, h.d_err);
    else
        nonfinite_kernel<float><<<blocks, 256, 0, s>>>((const float*)buf, h.units, h.d_err);
    return cudaGetLastError();
}

}  // namespace rpl
