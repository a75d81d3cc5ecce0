// rpl_static.cu -- rpl_diagnostics_static: the spectral diagnostics of a wave-action array that
// the caller already holds on the device, computed without allocating any memory.
//
// Who needs it: code that must not call cudaMalloc at the moment it wants the diagnostics, e.g.
// a host framework whose device memory is all owned by its own pool allocator (Julia's CUDA.jl
// pool, PyTorch's caching allocator), or work enqueued while that framework captures a stream into
// a CUDA graph, where allocating through the runtime is not permitted. Such a caller passes device
// pointers for the action, the spectral measures and every output, and this file supplies the only
// scratch the reduction needs (per-block partial sums of the total action) from a fixed array that
// is part of the loaded library.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "rpl_internal.h"

namespace {

// Largest horizontal grid the fixed scratch supports: one partial per block of 256 columns.
constexpr int kColumnsPerBlock = 256;
constexpr int64_t kMaxBlocks = RPL_STATIC_MAX_COLUMNS / kColumnsPerBlock;

// Block partials (sum, compensation) of the total action: 2 * 16384 doubles = 256 KiB. Every GPU
// that loads librpl.so holds this array until the process exits.
static __device__ __align__(256) double g_static_partials[2 * kMaxBlocks];

// Device address of g_static_partials per device ordinal, looked up once per device.
constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double* g_scratch[kMaxDevices] = {};

__device__ __forceinline__ void kadd(double& s, double& c, double v) {
    const double t = s + v;
    if (fabs(s) >= fabs(v)) c += (s - t) + v;
    else c += (v - t) + s;
    s = t;
}

// Per-(i,j) Kahan-compensated sums over the spectral bins (one sequential loop per column; the
// handle-based diagnostics sum in another order, so the two agree to a few ulps, not bit for bit),
// then one compensated partial of m0 * dx * dy per block, written to its own slot of the scratch.
template <typename T>
__global__ void __launch_bounds__(kColumnsPerBlock)
    static_diag_kernel(const T* __restrict__ N, int64_t P, int64_t nb, const double* __restrict__ tabs,
                       double area, double* m0o, double* hso, double* krmso, double* mdiro,
                       double* __restrict__ partials) {
    __shared__ double cell[kColumnsPerBlock];
    const int64_t c = (int64_t)blockIdx.x * kColumnsPerBlock + threadIdx.x;
    double m0 = 0.0;
    if (c < P) {
        const double* w = tabs;
        const double* mux = tabs + nb;
        const double* muy = tabs + 2 * nb;
        const double* tr = tabs + 3 * nb;
        double s0 = 0, c0 = 0, sx = 0, cx = 0, sy = 0, cy = 0, st = 0, ct = 0;
        for (int64_t b = 0; b < nb; ++b) {
            const double a = (double)N[c + P * b];
            kadd(s0, c0, a * w[b]);
            kadd(sx, cx, a * mux[b]);
            kadd(sy, cy, a * muy[b]);
            kadd(st, ct, a * tr[b]);
        }
        m0 = s0 + c0;
        const double mx = sx + cx, my = sy + cy, mt = st + ct;
        if (m0o) m0o[c] = m0;
        if (hso) hso[c] = 4.0 * sqrt(m0);
        if (krmso) krmso[c] = sqrt(m0 == 0.0 ? 0.0 : mt / m0);
        if (mdiro) mdiro[c] = atan2(my, mx);
    }
    cell[threadIdx.x] = m0 * area;
    __syncthreads();
    if (threadIdx.x == 0) {
        double S = 0.0, C = 0.0;
        for (int k = 0; k < kColumnsPerBlock; ++k) kadd(S, C, cell[k]);
        partials[2 * blockIdx.x] = S;
        partials[2 * blockIdx.x + 1] = C;
    }
}

// Sums the partials written by this call (slots 0 .. nblocks-1) in a fixed order.
__global__ void static_total_kernel(const double* __restrict__ partials, int64_t nblocks, double* total) {
    __shared__ double ss[1024], cc[1024];
    double s = 0.0, c = 0.0;
    for (int64_t k = threadIdx.x; k < nblocks; k += blockDim.x) {
        kadd(s, c, partials[2 * k]);
        c += partials[2 * k + 1];
    }
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

int fail(int code, const std::string& msg) {
    rpl::set_last_error(msg);
    return code;
}

// The device address of the scratch array on the current device. The first call on each device
// resolves it with cudaGetSymbolAddress (which may also load the library's module onto that
// device), so that first call belongs before any stream capture begins.
int scratch_on_current_device(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(RPL_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(RPL_ERR_UNSUPPORTED, "device ordinal beyond 63");
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch[dev]) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_static_partials);
        if (e != cudaSuccess || !ptr)
            return fail(RPL_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_scratch[dev] = (double*)ptr;
    }
    *out = g_scratch[dev];
    return RPL_OK;
}

}  // namespace

extern "C" int rpl_diagnostics_static(const void* N, int32_t dtype, int64_t Nx, int64_t Ny, int64_t Nk,
                                      int64_t Np, const double* measures, double dx, double dy, double* m0,
                                      double* hs, double* krms, double* mean_dir, double* total, void* stream) {
    if (!N || !measures) return fail(RPL_ERR_ARGUMENT, "null action or measures pointer");
    if (dtype != RPL_F64 && dtype != RPL_F32) return fail(RPL_ERR_ARGUMENT, "unknown dtype");
    if (Nx < 1 || Ny < 1 || Nk < 1 || Np < 1) return fail(RPL_ERR_ARGUMENT, "grid sizes must be positive");
    if (!(dx > 0.0) || !(dy > 0.0)) return fail(RPL_ERR_ARGUMENT, "grid spacings must be positive");
    // bounds checked before any product is formed, so no size can overflow into an accepted one
    if (Nx > RPL_STATIC_MAX_COLUMNS / Ny)
        return fail(RPL_ERR_ARGUMENT, "rpl_diagnostics_static supports at most " +
                                          std::to_string((long long)RPL_STATIC_MAX_COLUMNS) +
                                          " horizontal cells (Nx*Ny); got Nx = " + std::to_string((long long)Nx) +
                                          ", Ny = " + std::to_string((long long)Ny));
    if (Nk > INT32_MAX / Np) return fail(RPL_ERR_ARGUMENT, "Nk*Np must stay below 2^31 spectral bins");
    const int64_t P = Nx * Ny;
    double* partials = nullptr;
    int st = scratch_on_current_device(&partials);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t nblocks = (P + kColumnsPerBlock - 1) / kColumnsPerBlock;
    const double area = dx * dy;
    if (dtype == RPL_F64)
        static_diag_kernel<double><<<(unsigned)nblocks, kColumnsPerBlock, 0, s>>>(
            (const double*)N, P, Nk * Np, measures, area, m0, hs, krms, mean_dir, partials);
    else
        static_diag_kernel<float><<<(unsigned)nblocks, kColumnsPerBlock, 0, s>>>(
            (const float*)N, P, Nk * Np, measures, area, m0, hs, krms, mean_dir, partials);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && total) {
        static_total_kernel<<<1, 1024, 0, s>>>(partials, nblocks, total);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return fail(RPL_ERR_CUDA, std::string("rpl_diagnostics_static: ") + cudaGetErrorString(e));
    return RPL_OK;
}
