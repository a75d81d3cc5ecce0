// rpl_pm.cu -- PseudomomentumVelocities: the waves' own pseudomomentum as the Lagrangian-mean current
// that Doppler-shifts them (src/Coupling/current_coupling.jl:41-118,140-143,
// src/Coupling/pseudomomentum.jl:68-138,316-342, src/Coupling/lagrangian_velocities.jl:294-311).
//
// Set-up builds the vertical overlap tables of the Q transform once (one Nk x Nk pair for a constant
// projection depth, one pair per (i,j) column for a depth field; FP32 copies for FP32 models). Before
// every RK3 stage (and every stand-alone tendency) the Doppler velocity is refreshed from the stage's
// input action (dU/dkappa, which the stage kernels do not read, follows on request):
//   pm_velocity_kernel  one warp per (i,j) column: first moments M_s = sum_n N[s,n] k_measure[s,n]
//                       for every source ring s (lanes over s, coalesced kappa-contiguous reads of the
//                       state), then U_t = sum_s overlap[t,s] M_s and dU/dkappa_t with the derivative
//                       table (lanes over targets t); written kappa-fastest per column.
//   coef_from_U_kernel  (rpl_layout.cu) the periodic centred gradients of Ux, Uy
//                       (wave_current_refraction.jl:7-19) fused with the write of the stage kernels'
//                       coefficient records.
// The caller-order coupling arrays (rpl_get_coupling) are produced on request only.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>

#include "rpl_device.cuh"
#include "rpl_internal.h"

namespace rpl {

namespace {

constexpr int PM_WARPS = 8;     // columns per block of the velocity kernel
constexpr int PM_MAX_NK = 256;  // per-warp moments in shared memory: 2 * Nk doubles

// Overlap tables of one projection column per block (pseudomomentum.jl:68-121):
//   O[t,s]  = sum_k Qcell(kappa_t) Qcell(kappa_s) / |dz_k|
//   Od[t,s] = sum_k dQcell/dkappa(kappa_t) Qcell(kappa_s) / |dz_k|
// sequential in k like the reference. Cell integrals of a chunk of kc vertical cells are staged in
// shared memory; each table element is owned by one thread across all chunks. Table layout per
// column: element (t, s) at s * Nk + t.
__global__ void pm_overlap_kernel(int Nk, int64_t Nz, int kc_max, const double* __restrict__ zf,
                                  const double* __restrict__ kappa, const double* __restrict__ depth,
                                  double depth_const, double small_mu, int exact_form, double* __restrict__ O,
                                  double* __restrict__ Od) {
    extern __shared__ double sm[];
    double* W = sm;                           // kc_max x Nk cell integrals
    double* Wd = W + (int64_t)kc_max * Nk;    // kc_max x Nk kappa derivatives
    double* dz = Wd + (int64_t)kc_max * Nk;   // kc_max
    const int64_t col = blockIdx.x;
    const double d = depth ? depth[col] : depth_const;
    const int64_t n2 = (int64_t)Nk * Nk;
    double* o = O + col * n2;
    double* od = Od + col * n2;
    for (int64_t e = threadIdx.x; e < n2; e += blockDim.x) {
        o[e] = 0.0;
        od[e] = 0.0;
    }
    for (int64_t k0 = 0; k0 < Nz; k0 += kc_max) {
        const int kc = (int)min((int64_t)kc_max, Nz - k0);
        __syncthreads();
        for (int e = threadIdx.x; e < kc * Nk; e += blockDim.x) {
            const int k = e / Nk, m = e - k * Nk;
            const double z1 = zf[k0 + k], z2 = zf[k0 + k + 1];
            const double lo = fmin(z1, z2), hi = fmax(z1, z2);
            const double kap = kappa[m];
            W[e] = q_cdf(kap, hi, d, small_mu, exact_form) - q_cdf(kap, lo, d, small_mu, exact_form);
            Wd[e] = q_cdf_dk(kap, hi, d, small_mu) - q_cdf_dk(kap, lo, d, small_mu);
        }
        for (int k = threadIdx.x; k < kc; k += blockDim.x) dz[k] = fabs(zf[k0 + k + 1] - zf[k0 + k]);
        __syncthreads();
        for (int64_t e = threadIdx.x; e < n2; e += blockDim.x) {
            const int s = (int)(e / Nk), t = (int)(e - (int64_t)s * Nk);
            double a = o[e], b = od[e];
            for (int k = 0; k < kc; ++k) {
                const double sw = W[k * Nk + s];
                a += W[k * Nk + t] * sw / dz[k];
                b += Wd[k * Nk + t] * sw / dz[k];
            }
            o[e] = a;
            od[e] = b;
        }
    }
}

// Doppler velocity of the pseudomomentum (pseudomomentum.jl:316-342), one warp per (i,j) column.
// N: device layout (n*P + c)*Nk + m. kx, ky: (Nk, Np) first-moment measures, m fastest. O: the overlap
// table (or the derivative overlap, for dU/dkappa), one Nk x Nk table (per_cell = 0) or one per column.
// Ux, Uy: c3 doubles each in device order c*Nk + t. A is the arithmetic type: double for FP64 models
// and for dU/dkappa, float for the per-stage refresh of FP32 models.
template <typename T, typename A>
__global__ void __launch_bounds__(PM_WARPS * 32)
pm_velocity_kernel(const T* __restrict__ N, int64_t P, int Nk, int Np, const A* __restrict__ kx,
                   const A* __restrict__ ky, const A* __restrict__ O, int per_cell, double* __restrict__ Ux,
                   double* __restrict__ Uy) {
    extern __shared__ __align__(16) unsigned char pm_smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t c = (int64_t)blockIdx.x * PM_WARPS + w;
    if (c >= P) return;  // uniform per warp; the kernel has no block-wide barrier
    A* mx = reinterpret_cast<A*>(pm_smem) + (int64_t)w * 2 * Nk;
    A* my = mx + Nk;
    for (int s = lane; s < Nk; s += 32) {
        A ax = 0, ay = 0;
#pragma unroll 6
        for (int n = 0; n < Np; ++n) {
            const A a = (A)N[((int64_t)n * P + c) * Nk + s];
            ax += a * __ldg(kx + s + (int64_t)Nk * n);
            ay += a * __ldg(ky + s + (int64_t)Nk * n);
        }
        mx[s] = ax;
        my[s] = ay;
    }
    __syncwarp();
    const A* o = per_cell ? O + c * (int64_t)Nk * Nk : O;
    for (int t = lane; t < Nk; t += 32) {
        A ux = 0, uy = 0;
#pragma unroll 8
        for (int s = 0; s < Nk; ++s) {
            const A q = __ldg(o + (int64_t)s * Nk + t);
            ux += q * mx[s];
            uy += q * my[s];
        }
        Ux[c * Nk + t] = (double)ux;
        Uy[c * Nk + t] = (double)uy;
    }
}

// FP32 copy of a table.
__global__ void to_f32_kernel(const double* __restrict__ a, int64_t n, float* __restrict__ b) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) b[t] = (float)a[t];
}

inline unsigned blocks_for(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

int overlap_chunk(int Nk) { return std::max(1, std::min(32, 2048 / Nk)); }

}  // namespace

cudaError_t launch_pm_refresh(Handle& h, const void* Nin, cudaStream_t s, bool with_derivative) {
    const rpl_desc& d = h.desc;
    const int Nk = (int)d.Nk, Np = (int)d.Np;
    const int64_t P = h.cells, c3 = P * Nk;
    const unsigned blocks = blocks_for(P, PM_WARPS);
    if (h.precision == RPL_FP64)
        pm_velocity_kernel<double, double><<<blocks, PM_WARPS * 32, (size_t)PM_WARPS * 2 * Nk * 8, s>>>(
            (const double*)Nin, P, Nk, Np, h.d_pm_moments, h.d_pm_moments + (int64_t)Nk * Np, h.d_pm_overlap,
            h.pm_cols > 1, h.d_U, h.d_U + c3);
    else
        pm_velocity_kernel<float, float><<<blocks, PM_WARPS * 32, (size_t)PM_WARPS * 2 * Nk * 4, s>>>(
            (const float*)Nin, P, Nk, Np, h.d_pm_moments32, h.d_pm_moments32 + (int64_t)Nk * Np, h.d_pm_overlap32,
            h.pm_cols > 1, h.d_U, h.d_U + c3);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = launch_coef_from_U(h, s);
    if (e != cudaSuccess) return e;
    h.pm_ready = true;
    h.pm_last_in = Nin;  // a state buffer that only the next step overwrites
    h.dU_stale = true;
    if (with_derivative) {
        e = launch_pm_derivative(h, s);
        if (e == cudaSuccess) h.dU_stale = false;
    }
    return e;
}

cudaError_t launch_pm_derivative(const Handle& h, cudaStream_t s) {
    const rpl_desc& d = h.desc;
    const int Nk = (int)d.Nk, Np = (int)d.Np;
    const int64_t P = h.cells, c3 = P * Nk;
    if (!h.pm_ready) return cudaMemsetAsync(h.d_U + 2 * c3, 0, 2 * c3 * sizeof(double), s);
    const unsigned blocks = blocks_for(P, PM_WARPS);
    const size_t smem = (size_t)PM_WARPS * 2 * Nk * 8;
    const double* Od = h.d_pm_overlap + h.pm_cols * (int64_t)Nk * Nk;
    if (h.precision == RPL_FP64)
        pm_velocity_kernel<double, double><<<blocks, PM_WARPS * 32, smem, s>>>(
            (const double*)h.pm_last_in, P, Nk, Np, h.d_pm_moments, h.d_pm_moments + (int64_t)Nk * Np, Od,
            h.pm_cols > 1, h.d_U + 2 * c3, h.d_U + 3 * c3);
    else
        pm_velocity_kernel<float, double><<<blocks, PM_WARPS * 32, smem, s>>>(
            (const float*)h.pm_last_in, P, Nk, Np, h.d_pm_moments, h.d_pm_moments + (int64_t)Nk * Np, Od,
            h.pm_cols > 1, h.d_U + 2 * c3, h.d_U + 3 * c3);
    return cudaGetLastError();
}

void free_pm(Handle* h) {
    const int64_t Nk = h->desc.Nk, Np = h->desc.Np;
    if (h->d_pm_overlap) h->bytes -= 2 * h->pm_cols * Nk * Nk * 8;
    if (h->d_pm_moments) h->bytes -= 2 * Nk * Np * 8;
    if (h->d_pm_overlap32) h->bytes -= h->pm_cols * Nk * Nk * 4 + 2 * Nk * Np * 4;
    for (double* p : {h->d_pm_overlap, h->d_pm_moments})
        if (p) cudaFree(p);
    for (float* p : {h->d_pm_overlap32, h->d_pm_moments32})
        if (p) cudaFree(p);
    h->d_pm_overlap = h->d_pm_moments = nullptr;
    h->d_pm_overlap32 = h->d_pm_moments32 = nullptr;
    h->pm_last_in = nullptr;
    h->pm = h->pm_ready = false;
    h->pm_cols = 0;
}

}  // namespace rpl

namespace {

int pm_fail(int code, const std::string& msg) {
    rpl::set_last_error(msg);
    return code;
}

bool finite_range(const double* a, int64_t n) {
    for (int64_t i = 0; i < n; ++i)
        if (!std::isfinite(a[i])) return false;
    return true;
}

}  // namespace

extern "C" int rpl_set_pseudomomentum(rpl_handle* hh, int64_t Nz, const double* z_faces, int32_t q_depth_kind,
                                      double q_depth_constant, const double* q_depth_field, double small_mu) {
    using rpl::Handle;
    if (!hh) return pm_fail(RPL_ERR_ARGUMENT, "null handle");
    Handle* h = reinterpret_cast<Handle*>(hh);
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return pm_fail(RPL_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    const rpl_desc& d = h->desc;
    if (d.transport != RPL_TRANSPORT_REFRACTION)
        return pm_fail(RPL_ERR_STATE, "pseudomomentum velocities need RPL_TRANSPORT_REFRACTION");
    if (d.Nk > rpl::PM_MAX_NK)
        return pm_fail(RPL_ERR_UNSUPPORTED, "pseudomomentum coupling supports up to 256 kappa rings");
    if (Nz < 1 || !z_faces) return pm_fail(RPL_ERR_ARGUMENT, "pseudomomentum coupling needs Nz >= 1 and z faces");
    if (!(small_mu >= 0.0)) return pm_fail(RPL_ERR_ARGUMENT, "small_mu must be non-negative");
    if (!finite_range(z_faces, Nz + 1)) return pm_fail(RPL_ERR_NONFINITE, "non-finite z faces");
    for (int64_t k = 0; k < Nz; ++k)
        if (!(z_faces[k + 1] > z_faces[k])) return pm_fail(RPL_ERR_ARGUMENT, "z faces must be strictly increasing");
    const int64_t P = h->cells, Nk = d.Nk, Np = d.Np, c3 = P * Nk;
    int64_t cols = 1;
    if (q_depth_kind == RPL_DEPTH_CONSTANT) {
        if (!(q_depth_constant > 0.0) || !std::isfinite(q_depth_constant))
            return pm_fail(RPL_ERR_ARGUMENT, "depth must be positive");
    } else if (q_depth_kind == RPL_DEPTH_FIELD) {
        if (!q_depth_field) return pm_fail(RPL_ERR_ARGUMENT, "null Q depth field");
        for (int64_t c = 0; c < P; ++c)
            if (!(q_depth_field[c] > 0.0) || !std::isfinite(q_depth_field[c]))
                return pm_fail(RPL_ERR_ARGUMENT, "depth values must be positive");
        cols = P;
    } else {
        return pm_fail(RPL_ERR_ARGUMENT, "Q-transform depth must be constant or a field");
    }
    const bool f32 = h->precision == RPL_FP32;
    const int64_t table_bytes = 2 * cols * Nk * Nk * 8, moment_bytes = 2 * Nk * Np * 8;
    const int64_t f32_bytes = f32 ? cols * Nk * Nk * 4 + 2 * Nk * Np * 4 : 0;
    const int64_t extra = table_bytes + moment_bytes + f32_bytes + (h->d_coupling ? 0 : 8 * c3 * 8) +
                          (h->d_U ? 0 : 4 * c3 * 8);
    if (d.memory_limit_bytes > 0 && h->bytes + extra > d.memory_limit_bytes)
        return pm_fail(RPL_ERR_OOM, "pseudomomentum tables need " + std::to_string(extra) +
                                        " more device bytes, above the memory limit");
    cudaStream_t s = h->stream;
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return pm_fail(RPL_ERR_CUDA, std::string("rpl_set_pseudomomentum: ") + cudaGetErrorString(e));
    // previous tables (another Q grid) and prescribed currents go; the coupling buffers stay allocated
    rpl::free_pm(h);
    rpl::free_currents(h);
    if (!h->d_coupling) {
        e = cudaMalloc(&h->d_coupling, 8 * c3 * sizeof(double));
        if (e != cudaSuccess) return pm_fail(RPL_ERR_OOM, "pseudomomentum coupling: device allocation failed");
        h->bytes += 8 * c3 * 8;
    }
    if (!h->d_U) {
        e = cudaMalloc(&h->d_U, 4 * c3 * sizeof(double));
        if (e != cudaSuccess) return pm_fail(RPL_ERR_OOM, "pseudomomentum coupling: device allocation failed");
        h->bytes += 4 * c3 * 8;
    }
    e = cudaMalloc(&h->d_pm_overlap, table_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_pm_moments, moment_bytes);
    if (e == cudaSuccess && f32) e = cudaMalloc(&h->d_pm_overlap32, cols * Nk * Nk * 4);
    if (e == cudaSuccess && f32) e = cudaMalloc(&h->d_pm_moments32, 2 * Nk * Np * 4);
    if (e == cudaSuccess) {
        h->bytes += table_bytes + moment_bytes + f32_bytes;
        h->pm_cols = cols;
    } else {
        for (double* p : {h->d_pm_overlap, h->d_pm_moments})
            if (p) cudaFree(p);
        for (float* p : {h->d_pm_overlap32, h->d_pm_moments32})
            if (p) cudaFree(p);
        h->d_pm_overlap = h->d_pm_moments = nullptr;
        h->d_pm_overlap32 = h->d_pm_moments32 = nullptr;
        cudaGetLastError();
        return pm_fail(RPL_ERR_OOM, "pseudomomentum tables: device allocation failed");
    }

    // first-moment measures (polar_wavevector_grid.jl:73-99,107-110), (Nk, Np) m fastest
    std::vector<double> mom(2 * Nk * Np);
    for (int64_t n = 0; n < Np; ++n)
        for (int64_t m = 0; m < Nk; ++m) {
            const double k1 = h->kappa_faces[m], k2 = h->kappa_faces[m + 1];
            const double p1 = h->phi_faces[n], p2 = h->phi_faces[n + 1];
            const double radial = (k2 * k2 * k2 - k1 * k1 * k1) / 3.0;
            mom[m + Nk * n] = radial * (std::sin(p2) - std::sin(p1));
            mom[Nk * Np + m + Nk * n] = radial * (std::cos(p1) - std::cos(p2));
        }
    double *dz = nullptr, *dq = nullptr;
    e = cudaMalloc(&dz, (Nz + 1) * 8);
    if (e == cudaSuccess && cols > 1) e = cudaMalloc(&dq, P * 8);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dz, z_faces, (Nz + 1) * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && dq) e = cudaMemcpyAsync(dq, q_depth_field, P * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->d_pm_moments, mom.data(), moment_bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        const int kc = rpl::overlap_chunk((int)Nk);
        const size_t smem = ((size_t)2 * kc * Nk + kc) * sizeof(double);
        const int exact_form = h->precision == RPL_FP64 ? 1 : 0;
        rpl::pm_overlap_kernel<<<(unsigned)cols, 256, smem, s>>>((int)Nk, Nz, kc, dz, h->d_kappa, dq,
                                                                 q_depth_constant, small_mu, exact_form,
                                                                 h->d_pm_overlap, h->d_pm_overlap + cols * Nk * Nk);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && f32) {
        const int64_t n = cols * Nk * Nk, nm = 2 * Nk * Np;
        rpl::to_f32_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(h->d_pm_overlap, n, h->d_pm_overlap32);
        rpl::to_f32_kernel<<<(unsigned)((nm + 255) / 256), 256, 0, s>>>(h->d_pm_moments, nm, h->d_pm_moments32);
        e = cudaGetLastError();
    }
    // the coupling starts at zero like the reference's caches (current_coupling.jl:103-107)
    if (e == cudaSuccess) e = cudaMemsetAsync(h->d_coupling, 0, 8 * c3 * sizeof(double), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->d_U, 0, 4 * c3 * sizeof(double), s);
    if (e == cudaSuccess) {
        h->currents_set = true;
        e = rpl::launch_coef(*h, s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (dz) cudaFree(dz);
    if (dq) cudaFree(dq);
    if (e != cudaSuccess) {
        h->currents_set = false;
        rpl::free_pm(h);
        return pm_fail(RPL_ERR_CUDA, std::string("rpl_set_pseudomomentum: ") + cudaGetErrorString(e));
    }
    h->pm = true;
    return RPL_OK;
}

extern "C" int rpl_update_coupling(rpl_handle* hh) {
    using rpl::Handle;
    if (!hh) return pm_fail(RPL_ERR_ARGUMENT, "null handle");
    Handle* h = reinterpret_cast<Handle*>(hh);
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return pm_fail(RPL_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    if (!h->pm) return RPL_OK;  // prescribed currents are static: rpl_set_currents already applied them
    e = rpl::launch_pm_refresh(*h, h->N, h->stream, true);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return pm_fail(RPL_ERR_CUDA, std::string("rpl_update_coupling: ") + cudaGetErrorString(e));
    return RPL_OK;
}
