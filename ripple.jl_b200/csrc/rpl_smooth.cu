// rpl_smooth.cu -- SpatialAveraging, the Garden-Sprinkler-Effect alleviation of Tolman (2002) that the
// reference applies after every time step (src/Models/propagation_smoothing.jl:20-199,
// src/Models/time_step.jl:168).
//
// Each spectral bin's physical field is replaced by the mean of four bilinear interpolations at the
// corners of a rectangle of half-widths L_s = alpha_s |dc_g| dt along the bin's direction and
// L_n = alpha_n c_g dphi dt across it. When the smoothing is on, the RK3 stage 3 writes its result into
// the free stage buffer A and smooth_kernel writes A -> N, so the step needs no extra copy and the
// state pointers never change (a captured step stays valid).
//
// When every corner lies within one cell of its target (any step that respects the CFL limit), the
// four samples form a 3 x 3 stencil whose weights depend on the bin only: smooth_weights_kernel builds
// them once per dt, and smooth_kernel walks strips of cells along x with the 3 x 3 neighbourhood in
// registers (three new kappa-contiguous loads and nine FMAs per output); HBM sees about one read and
// one write of the state (the neighbouring rows come from L2). Bins whose corners reach further take the
// reference's per-corner bilinear path. Corner positions are FP64 for both precisions.
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "rpl_internal.h"

namespace rpl {

namespace {

constexpr int STRIP = 32;  // cells along x per thread
constexpr int ROWS = 8;    // y rows per block (threadIdx.y)

// 1-based index wrap like the reference (_gse_periodic / _gse_clamp), then a clamp so a corner beyond
// one period never leaves the array.
__device__ __forceinline__ int gse_index(int i, int N, bool periodic) {
    if (periodic) i = i < 1 ? i + N : (i > N ? i - N : i);
    return i < 1 ? 1 : (i > N ? N : i);
}

// Corner offsets of bin (m, n) in cells (propagation_smoothing.jl:72-86), in FP64: corner q = (s1, s2)
// with s1, s2 in {-1, +1}, q = 2 * (s1 > 0) + (s2 > 0).
struct Corners {
    double di[4], dj[4];
};

__device__ __forceinline__ Corners corners(const double* __restrict__ tab, int Nk, int Np, int m, int n,
                                           double dphi, double as, double an, double dt, double dx_inv,
                                           double dy_inv) {
    const double cg = tab[m], dcg = tab[Nk + m], cs = tab[2 * Nk + n], sn = tab[2 * Nk + Np + n];
    const double Ls = as * dcg * dt, Ln = an * cg * dphi * dt;
    const double Ls_x = Ls * cs * dx_inv, Ls_y = Ls * sn * dy_inv;
    const double Ln_x = -Ln * sn * dx_inv, Ln_y = Ln * cs * dy_inv;
    Corners k;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const double s1 = q < 2 ? -1.0 : 1.0, s2 = (q & 1) ? 1.0 : -1.0;
        k.di[q] = s1 * Ls_x + s2 * Ln_x;
        k.dj[q] = s1 * Ls_y + s2 * Ln_y;
    }
    return k;
}

// Per-bin 3 x 3 stencil of the averaging when every corner lies within one cell of the target (then
// each corner's bilinear sample uses only the 3 x 3 neighbourhood): W[(b + 1) * 3 + (a + 1)] is the
// weight of cell (i + a, j + b), the four samples' weights already divided by 4. Layout: weights
// (n * 9 + q) * Nk + m in T, flag[n * Nk + m] = 1 where a corner reaches further (general path).
template <typename T>
__global__ void smooth_weights_kernel(int Nk, int Np, const double* __restrict__ tab, double dphi, double as,
                                      double an, double dt, double dx_inv, double dy_inv, T* __restrict__ W,
                                      int* __restrict__ flag) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= Nk * Np) return;
    const int n = t / Nk, m = t - n * Nk;
    const Corners k = corners(tab, Nk, Np, m, n, dphi, as, an, dt, dx_inv, dy_inv);
    double w[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    int far = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const double fi = floor(k.di[q]), fj = floor(k.dj[q]);
        const double wi = k.di[q] - fi, wj = k.dj[q] - fj;
        const bool near = fi >= -1.0 && fi <= 0.0 && fj >= -1.0 && fj <= 0.0;
        far |= !near;
        if (near) {
            const int a = (int)fi + 1, b = (int)fj + 1;  // 0 or 1
            w[b * 3 + a] += (1.0 - wi) * (1.0 - wj) / 4.0;
            w[b * 3 + a + 1] += wi * (1.0 - wj) / 4.0;
            w[(b + 1) * 3 + a] += (1.0 - wi) * wj / 4.0;
            w[(b + 1) * 3 + a + 1] += wi * wj / 4.0;
        }
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) W[((int64_t)n * 9 + q) * Nk + m] = (T)w[q];
    flag[n * Nk + m] = far;
}

// Block (32 lanes over kappa, ROWS rows), grid (x strips, row groups, directions). Each thread walks a
// strip of STRIP cells along x for its ring m (chunks of 32 rings) and row j, keeping the 3 x 3
// neighbourhood in registers: near bins take 3 new kappa-contiguous loads and 9 FMAs per output; far
// bins (a corner beyond one cell) take the reference's four bilinear samples with FP64 positions.
template <typename T>
__global__ void __launch_bounds__(32 * ROWS)
smooth_kernel(const T* __restrict__ Nin, T* __restrict__ Nout, int Nx, int Ny, int Nk, int Np,
              const T* __restrict__ W, const int* __restrict__ flag, const double* __restrict__ tab, double dphi,
              double as, double an, double dt, double dx_inv, double dy_inv, int periodic_x, int periodic_y,
              int j_lo, int j_hi, int y_offset) {
    const int j = j_lo + blockIdx.y * ROWS + threadIdx.y + 1;  // 1-based like the reference, rows [j_lo, j_hi)
    if (j > j_hi) return;
    const int n = blockIdx.z;
    const int i_first = blockIdx.x * STRIP + 1, i_last = min(i_first + STRIP - 1, Nx);
    const int64_t P = (int64_t)Nx * Ny;
    const T* base = Nin + (int64_t)n * P * Nk;
    T* out = Nout + (int64_t)n * P * Nk;
    const int jm = gse_index(j - 1, Ny, periodic_y), jp = gse_index(j + 1, Ny, periodic_y);
    const int64_t rowoff[3] = {(int64_t)(jm - 1) * Nx * Nk, (int64_t)(j - 1) * Nx * Nk, (int64_t)(jp - 1) * Nx * Nk};
    for (int m = threadIdx.x; m < Nk; m += 32) {
        if (flag[n * Nk + m]) {
            const Corners k = corners(tab, Nk, Np, m, n, dphi, as, an, dt, dx_inv, dy_inv);
            for (int i = i_first; i <= i_last; ++i) {
                T acc = T(0);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    // rows at their index in the larger grid of a decomposition slab (y_offset), so the
                    // weights round as in the undecomposed model
                    const double ir = (double)i + k.di[q], jr = (double)(j + y_offset) + k.dj[q];
                    const double fi = floor(ir), fj = floor(jr);
                    const int i0 = (int)fi, j0 = (int)fj - y_offset;
                    const T wi = (T)(ir - fi), wj = (T)(jr - fj);
                    const int i0c = gse_index(i0, Nx, periodic_x), i1c = gse_index(i0 + 1, Nx, periodic_x);
                    const int j0c = gse_index(j0, Ny, periodic_y), j1c = gse_index(j0 + 1, Ny, periodic_y);
                    const T f00 = __ldg(base + ((int64_t)(j0c - 1) * Nx + (i0c - 1)) * Nk + m);
                    const T f10 = __ldg(base + ((int64_t)(j0c - 1) * Nx + (i1c - 1)) * Nk + m);
                    const T f01 = __ldg(base + ((int64_t)(j1c - 1) * Nx + (i0c - 1)) * Nk + m);
                    const T f11 = __ldg(base + ((int64_t)(j1c - 1) * Nx + (i1c - 1)) * Nk + m);
                    const T one = T(1);
                    acc += (one - wi) * (one - wj) * f00 + wi * (one - wj) * f10 + (one - wi) * wj * f01 +
                           wi * wj * f11;
                }
                out[((int64_t)(j - 1) * Nx + (i - 1)) * Nk + m] = acc / T(4);
            }
            continue;
        }
        T w[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) w[q] = __ldg(W + ((int64_t)n * 9 + q) * Nk + m);
        // window columns: a = 0 (i-1), 1 (i), 2 (i+1); rows b = 0 (j-1), 1 (j), 2 (j+1)
        T f[3][3];
        const int cl = gse_index(i_first - 1, Nx, periodic_x) - 1, cc = i_first - 1;
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            f[b][0] = __ldg(base + rowoff[b] + (int64_t)cl * Nk + m);
            f[b][1] = __ldg(base + rowoff[b] + (int64_t)cc * Nk + m);
        }
#pragma unroll 4
        for (int i = i_first; i <= i_last; ++i) {
            const int cr = gse_index(i + 1, Nx, periodic_x) - 1;
#pragma unroll
            for (int b = 0; b < 3; ++b) f[b][2] = __ldg(base + rowoff[b] + (int64_t)cr * Nk + m);
            T acc = T(0);
#pragma unroll
            for (int b = 0; b < 3; ++b)
#pragma unroll
                for (int a = 0; a < 3; ++a) acc += w[b * 3 + a] * f[b][a];
            out[((int64_t)(j - 1) * Nx + (i - 1)) * Nk + m] = acc;
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                f[b][0] = f[b][1];
                f[b][1] = f[b][2];
            }
        }
    }
}

// propagation_smoothing.jl:117-158: deep-water c_g = sqrt(g / kappa) / 2 with g = 9.81, its half-
// difference to the neighbouring rings, cos and sin of the directions (FP64; the reference's FP32 models
// take the corner positions in FP64 too, through its Float64 1/dx).
std::vector<double> smooth_tables(const Handle& h) {
    const int64_t Nk = h.desc.Nk, Np = h.desc.Np;
    const double g = 9.81;
    std::vector<double> tab(2 * Nk + 2 * Np);
    for (int64_t m = 0; m < Nk; ++m) tab[m] = 1.0 / 2.0 * std::sqrt(g / h.kappa[m]);
    for (int64_t m = 0; m < Nk; ++m) {
        const double lo = m == 0 ? tab[0] : 1.0 / 2.0 * std::sqrt(g / h.kappa[m - 1]);
        const double hi = m == Nk - 1 ? tab[Nk - 1] : 1.0 / 2.0 * std::sqrt(g / h.kappa[m + 1]);
        tab[Nk + m] = std::fabs(lo - hi) / 2.0;
    }
    for (int64_t n = 0; n < Np; ++n) {
        tab[2 * Nk + n] = std::cos(h.phi[n]);
        tab[2 * Nk + Np + n] = std::sin(h.phi[n]);
    }
    return tab;
}

template <typename T>
cudaError_t launch_smooth_t(Handle& h, const void* Nin, void* Nout, double dt, int64_t j_lo, int64_t j_hi,
                            int64_t y_offset, cudaStream_t s) {
    const rpl_desc& d = h.desc;
    const int Nk = (int)d.Nk, Np = (int)d.Np;
    const double* tab = (const double*)h.d_smooth;
    T* W = (T*)(tab + 2 * Nk + 2 * Np);
    int* flag = (int*)(W + (int64_t)9 * Nk * Np);
    const double dphi = h.phi_faces[1] - h.phi_faces[0];
    if (dt != h.smooth_dt) {  // per-bin stencils for this dt
        smooth_weights_kernel<T><<<(unsigned)((Nk * Np + 127) / 128), 128, 0, s>>>(
            Nk, Np, tab, dphi, h.smooth_as, h.smooth_an, dt, 1.0 / d.dx, 1.0 / d.dy, W, flag);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        h.smooth_dt = dt;
    }
    const dim3 grid((unsigned)((d.Nx + STRIP - 1) / STRIP), (unsigned)((j_hi - j_lo + ROWS - 1) / ROWS), (unsigned)Np);
    smooth_kernel<T><<<grid, dim3(32, ROWS), 0, s>>>((const T*)Nin, (T*)Nout, (int)d.Nx, (int)d.Ny, Nk, Np, W, flag,
                                                     tab, dphi, h.smooth_as, h.smooth_an, dt, 1.0 / d.dx,
                                                     1.0 / d.dy, d.periodic_x, d.periodic_y, (int)j_lo, (int)j_hi,
                                                     (int)y_offset);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_smooth(Handle& h, const void* Nin, void* Nout, double dt, int64_t j_lo, int64_t j_hi,
                          int64_t y_offset, cudaStream_t s) {
    if (h.precision == RPL_FP64) return launch_smooth_t<double>(h, Nin, Nout, dt, j_lo, j_hi, y_offset, s);
    return launch_smooth_t<float>(h, Nin, Nout, dt, j_lo, j_hi, y_offset, s);
}

void free_smooth(Handle* h) {
    if (h->d_smooth) {
        cudaFree(h->d_smooth);
        h->bytes -= h->smooth_bytes;
    }
    h->d_smooth = nullptr;
    h->smooth_bytes = 0;
    h->smooth = false;
}

}  // namespace rpl

extern "C" int rpl_set_propagation_smoothing(rpl_handle* hh, int32_t kind, double alpha_s, double alpha_n) {
    using rpl::Handle;
    auto fail = [](int code, const std::string& msg) {
        rpl::set_last_error(msg);
        return code;
    };
    if (!hh) return fail(RPL_ERR_ARGUMENT, "null handle");
    Handle* h = reinterpret_cast<Handle*>(hh);
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return fail(RPL_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    if (kind != 0 && kind != 1) return fail(RPL_ERR_ARGUMENT, "unknown propagation smoothing");
    e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return fail(RPL_ERR_CUDA, std::string("rpl_set_propagation_smoothing: ") + cudaGetErrorString(e));
    rpl::free_smooth(h);
    if (kind == 0) return RPL_OK;
    if (!std::isfinite(alpha_s) || !std::isfinite(alpha_n) || alpha_s < 0.0 || alpha_n < 0.0)
        return fail(RPL_ERR_ARGUMENT, "SpatialAveraging needs finite alpha_s, alpha_n >= 0");
    if (h->desc.Nx >= 0x7fffffff || h->desc.Ny >= 0x7fffffff || h->desc.Ny > 65535 * 8 || h->desc.Np > 65535)
        return fail(RPL_ERR_UNSUPPORTED, "SpatialAveraging supports Ny <= 524280 and Np <= 65535");
    for (int64_t m = 0; m < h->desc.Nk; ++m)
        if (!(h->kappa[m] > 0.0)) return fail(RPL_ERR_ARGUMENT, "SpatialAveraging needs kappa > 0");
    // FP64 tables, then the per-bin stencils (9 per bin, state type) and far flags (int per bin)
    const size_t elem = h->precision == RPL_FP64 ? 8 : 4;
    const int64_t Nk = h->desc.Nk, Np = h->desc.Np, ntab = 2 * Nk + 2 * Np;
    const int64_t bytes = ntab * 8 + 9 * Nk * Np * (int64_t)elem + Nk * Np * 4;
    if (h->desc.memory_limit_bytes > 0 && h->bytes + bytes > h->desc.memory_limit_bytes)
        return fail(RPL_ERR_OOM, "SpatialAveraging tables would exceed the memory limit");
    e = cudaMalloc(&h->d_smooth, bytes);
    if (e != cudaSuccess) {
        h->d_smooth = nullptr;
        cudaGetLastError();
        return fail(RPL_ERR_OOM, "SpatialAveraging tables: device allocation failed");
    }
    {
        const std::vector<double> tab = rpl::smooth_tables(*h);
        e = cudaMemcpy(h->d_smooth, tab.data(), ntab * 8, cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {
        cudaFree(h->d_smooth);
        h->d_smooth = nullptr;
        return fail(RPL_ERR_CUDA, std::string("rpl_set_propagation_smoothing: ") + cudaGetErrorString(e));
    }
    h->smooth_bytes = bytes;
    h->bytes += bytes;
    h->smooth_as = alpha_s;
    h->smooth_an = alpha_n;
    h->smooth_dt = -1.0;  // stencils are built at the first step
    h->smooth = true;
    return RPL_OK;
}
