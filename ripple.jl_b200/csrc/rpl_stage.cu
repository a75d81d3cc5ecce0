// rpl_stage.cu -- fused RK3 stage kernels: tendency (Doppler transport + refraction, or intrinsic
// transport) + sources + stage combine + max(0, .) clamp in one pass over the state.
//
// Reference: src/Coupling/wave_current_refraction.jl:74-151 (tendency),
// src/Models/intrinsic_transport.jl:14-68, src/Models/tendencies.jl:28-41,82-101 (dispatch, sources),
// src/Models/time_step.jl:67-74,98-105,138-152 (stage update with clamp).
//
// State layout (device): x fastest, (i,j,m,n) at i + Nx*(j + Ny*(m + Nk*n)).
// Launch order: the block index enumerates the Nk*Np spectral bins fastest and the (32 x 8) spatial
// tiles slowest, so the blocks resident at one time cover every bin of a few spatial tiles and the
// kappa/phi neighbours of a bin are read from L2 rather than HBM.
#include <cuda_runtime.h>

#include "rpl_device.cuh"
#include "rpl_internal.h"

namespace rpl {

namespace {

constexpr int TX = 32, TY = 8;

template <typename T>
__device__ __forceinline__ T tendency_at(const T* __restrict__ N, const StageParams& p, int i, int j,
                                         int m, int n) {
    const int Nx = (int)p.Nx, Ny = (int)p.Ny, Nk = (int)p.Nk, Np = (int)p.Np;
    const int64_t P = (int64_t)Nx * Ny, S = P * Nk;
    const int64_t c3 = (int64_t)i + (int64_t)Nx * (j + (int64_t)Ny * m);
    const T* bin = N + S * n + P * m;
    const T* row = bin + (int64_t)Nx * j;
    T ux, uy;
    if (p.cg_per_cell) {
        const double cg = p.cg_mag[c3];
        ux = T(cg * p.cg_x[m + Nk * n]);
        uy = T(cg * p.cg_y[m + Nk * n]);
    } else {
        ux = T(p.cg_x[m + Nk * n]);
        uy = T(p.cg_y[m + Nk * n]);
    }
    T ck = T(0), cp = T(0);
    if (p.transport == RPL_TRANSPORT_REFRACTION) {
        const T kap = T(p.kappa[m]);
        const T c = T(p.cosp[n]), s = T(p.sinp[n]);
        const T Uxx = T(p.Uxx[c3]), Uxy = T(p.Uxy[c3]), Uyx = T(p.Uyx[c3]), Uyy = T(p.Uyy[c3]);
        ck = -kap * (c * c * Uxx + c * s * (Uyx + Uxy) + s * s * Uyy);
        cp = c * s * (Uxx - Uyy) + s * s * Uyx - c * c * Uxy;
        ux = ux + T(p.Ux[c3]);
        uy = uy + T(p.Uy[c3]);
    }
    // x (periodic)
    const T x_m3 = row[wrap(i - 3, Nx)], x_m2 = row[wrap(i - 2, Nx)], x_m1 = row[wrap(i - 1, Nx)];
    const T x_0 = row[i];
    const T x_p1 = row[wrap(i + 1, Nx)], x_p2 = row[wrap(i + 2, Nx)], x_p3 = row[wrap(i + 3, Nx)];
    const T Nxp = weno_face(x_m2, x_m1, x_0, x_p1, x_p2, x_p3, ux, true);
    const T Nxm = weno_face(x_m3, x_m2, x_m1, x_0, x_p1, x_p2, ux, true);
    const T fx = ux * (Nxp - Nxm) * T(p.dx_inv);
    // y (periodic)
    const T y_m3 = bin[i + (int64_t)Nx * wrap(j - 3, Ny)], y_m2 = bin[i + (int64_t)Nx * wrap(j - 2, Ny)];
    const T y_m1 = bin[i + (int64_t)Nx * wrap(j - 1, Ny)];
    const T y_p1 = bin[i + (int64_t)Nx * wrap(j + 1, Ny)], y_p2 = bin[i + (int64_t)Nx * wrap(j + 2, Ny)];
    const T y_p3 = bin[i + (int64_t)Nx * wrap(j + 3, Ny)];
    const T Nyp = weno_face(y_m2, y_m1, x_0, y_p1, y_p2, y_p3, uy, true);
    const T Nym = weno_face(y_m3, y_m2, y_m1, x_0, y_p1, y_p2, uy, true);
    const T fy = uy * (Nyp - Nym) * T(p.dy_inv);
    if (p.transport != RPL_TRANSPORT_REFRACTION) return -(fx + fy);
    // kappa (bounded: clamped indices, first-order near the ends, no flux through the outer faces)
    const T* pt = N + S * n + (int64_t)i + (int64_t)Nx * j;
    const T k_m3 = pt[P * clampi(m - 3, Nk)], k_m2 = pt[P * clampi(m - 2, Nk)];
    const T k_m1 = pt[P * clampi(m - 1, Nk)];
    const T k_p1 = pt[P * clampi(m + 1, Nk)], k_p2 = pt[P * clampi(m + 2, Nk)];
    const T k_p3 = pt[P * clampi(m + 3, Nk)];
    const bool hp = (m - 2 >= 0) && (m + 3 <= Nk - 1);
    const bool hm = (m - 3 >= 0) && (m + 2 <= Nk - 1);
    const T Nkp = weno_face(k_m2, k_m1, x_0, k_p1, k_p2, k_p3, ck, hp);
    const T Nkm = weno_face(k_m3, k_m2, k_m1, x_0, k_p1, k_p2, ck, hm);
    const T fkp = (m == Nk - 1) ? T(0) : ck * Nkp;
    const T fkm = (m == 0) ? T(0) : ck * Nkm;
    const T fk = (fkp - fkm) * T(p.dk_inv);
    // phi (periodic)
    const T* pm = N + P * m + (int64_t)i + (int64_t)Nx * j;
    const T p_m3 = pm[S * wrap(n - 3, Np)], p_m2 = pm[S * wrap(n - 2, Np)], p_m1 = pm[S * wrap(n - 1, Np)];
    const T p_p1 = pm[S * wrap(n + 1, Np)], p_p2 = pm[S * wrap(n + 2, Np)], p_p3 = pm[S * wrap(n + 3, Np)];
    const T Npp = weno_face(p_m2, p_m1, x_0, p_p1, p_p2, p_p3, cp, true);
    const T Npm = weno_face(p_m3, p_m2, p_m1, x_0, p_p1, p_p2, cp, true);
    const T fp = cp * (Npp - Npm) * T(p.dp_inv);
    return -(fx + fy + fk + fp);
}

__device__ __forceinline__ void block_coords(const StageParams& p, int& i, int& j, int& m, int& n) {
    const unsigned nbins = (unsigned)(p.Nk * p.Np);
    const unsigned bin = blockIdx.x % nbins, tile = blockIdx.x / nbins;
    const unsigned tiles_x = (unsigned)((p.Nx + TX - 1) / TX);
    i = (int)((tile % tiles_x) * TX + threadIdx.x);
    j = (int)((tile / tiles_x) * TY + threadIdx.y);
    m = (int)(bin % (unsigned)p.Nk);
    n = (int)(bin / (unsigned)p.Nk);
}

template <typename T>
__global__ void __launch_bounds__(TX* TY) stage_kernel(const T* __restrict__ Nin, const T* N0, T* Nout,
                                                       StageParams p) {
    int i, j, m, n;
    block_coords(p, i, j, m, n);
    if (i >= p.Nx || j >= p.Ny) return;
    const int64_t u = (int64_t)i + p.Nx * ((int64_t)j + p.Ny * ((int64_t)m + p.Nk * n));
    T G = (p.transport == RPL_TRANSPORT_NONE) ? T(0) : tendency_at<T>(Nin, p, i, j, m, n);
    const T a = Nin[u];
    if (p.has_wind || p.has_diss) G = G + T(source_term(p, (int64_t)i + p.Nx * (int64_t)j, m, n, (double)a));
    const T st = relu(a + T(p.dt) * G);
    T out;
    if (p.stage == 1) out = st;
    else out = relu(T(p.a) * N0[u] + T(p.b) * st);
    if (!isfinite(out)) atomicOr(p.err, 1u);
    Nout[u] = out;
}

template <typename T>
__global__ void __launch_bounds__(TX* TY) tendency_kernel(const T* __restrict__ Nin, double* __restrict__ G,
                                                          StageParams p) {
    int i, j, m, n;
    block_coords(p, i, j, m, n);
    if (i >= p.Nx || j >= p.Ny) return;
    const int64_t u = (int64_t)i + p.Nx * ((int64_t)j + p.Ny * ((int64_t)m + p.Nk * n));
    T g = (p.transport == RPL_TRANSPORT_NONE) ? T(0) : tendency_at<T>(Nin, p, i, j, m, n);
    if (p.has_wind || p.has_diss) g = g + T(source_term(p, (int64_t)i + p.Nx * (int64_t)j, m, n, (double)Nin[u]));
    G[u] = (double)g;
}

dim3 stage_grid(const Handle& h) {
    const int64_t tiles = ((h.desc.Nx + TX - 1) / TX) * ((h.desc.Ny + TY - 1) / TY);
    return dim3((unsigned)(tiles * h.desc.Nk * h.desc.Np));
}

}  // namespace

StageParams make_params(const Handle& h, double dt, int stage) {
    StageParams p{};
    const rpl_desc& d = h.desc;
    p.Nx = d.Nx; p.Ny = d.Ny; p.Nk = d.Nk; p.Np = d.Np;
    p.dx_inv = 1.0 / d.dx;
    p.dy_inv = 1.0 / d.dy;
    p.dk_inv = 1.0 / (h.kappa_faces[1] - h.kappa_faces[0]);
    p.dp_inv = 1.0 / (h.phi_faces[1] - h.phi_faces[0]);
    p.dt = dt;
    p.stage = stage;
    p.a = stage == 2 ? 0.75 : (stage == 3 ? 1.0 / 3.0 : 0.0);
    p.b = stage == 2 ? 0.25 : (stage == 3 ? 2.0 / 3.0 : 1.0);
    p.transport = d.transport;
    p.cg_per_cell = h.d_cgmag != nullptr;
    p.kappa = h.d_kappa; p.phi = h.d_phi; p.weights = h.d_weights;
    p.cosp = h.d_cos; p.sinp = h.d_sin;
    p.cg_x = h.d_cgx; p.cg_y = h.d_cgy; p.cg_mag = h.d_cgmag;
    const int64_t c3 = d.Nx * d.Ny * d.Nk;
    if (h.d_coupling) {
        p.Ux = h.d_coupling; p.Uy = h.d_coupling + c3;
        p.Uxx = h.d_coupling + 4 * c3; p.Uxy = h.d_coupling + 5 * c3;
        p.Uyx = h.d_coupling + 6 * c3; p.Uyy = h.d_coupling + 7 * c3;
    }
    p.has_wind = h.has_sources && h.src.wind_kind != RPL_WIND_NONE;
    p.stress_cap = h.has_sources && h.src.stress_cap;
    p.has_diss = h.has_sources && h.src.has_dissipation;
    if (h.d_wind) {
        const int64_t c2 = d.Nx * d.Ny;
        p.wind_U10 = h.d_wind; p.wind_theta = h.d_wind + c2; p.wind_ustar = h.d_wind + 2 * c2;
        p.stress_factor = h.d_wind + 3 * c2;
    }
    p.rho_ratio = h.src.rho_air / h.src.rho_water;
    p.beta_max = h.src.beta_max; p.z_alpha = h.src.z_alpha; p.p_in = h.src.p_in;
    p.alpha0 = h.src.alpha0; p.von_karman = h.src.von_karman; p.wind_g = h.src.wind_gravity;
    p.C_ds = h.src.C_ds; p.B_r = h.src.B_r; p.ds_p = h.src.ds_p; p.sigma_power = h.src.sigma_power;
    p.ds_g = h.src.ds_gravity;
    p.err = h.d_err;
    return p;
}

cudaError_t launch_stage(const Handle& h, const StageParams& p, const void* Nin, const void* N0,
                         void* Nout, cudaStream_t s) {
    const dim3 grid = stage_grid(h), block(TX, TY);
    if (h.precision == RPL_FP64)
        stage_kernel<double><<<grid, block, 0, s>>>((const double*)Nin, (const double*)N0, (double*)Nout, p);
    else
        stage_kernel<float><<<grid, block, 0, s>>>((const float*)Nin, (const float*)N0, (float*)Nout, p);
    return cudaGetLastError();
}

cudaError_t launch_tendency(const Handle& h, const StageParams& p, const void* Nin, double* G,
                            cudaStream_t s) {
    const dim3 grid = stage_grid(h), block(TX, TY);
    if (h.precision == RPL_FP64)
        tendency_kernel<double><<<grid, block, 0, s>>>((const double*)Nin, G, p);
    else
        tendency_kernel<float><<<grid, block, 0, s>>>((const float*)Nin, G, p);
    return cudaGetLastError();
}

}  // namespace rpl
