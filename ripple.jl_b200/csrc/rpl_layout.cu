// rpl_layout.cu -- conversions between the caller's layout and the device layout of the state,
// and the per-(i,j,kappa) coefficient records the stage kernels read.
//
// Caller layout (RPL_LAYOUT_XFAST, the reference's flat_data interior): (i,j,m,n) at
//   c + P*(m + Nk*n),   c = i + Nx*j, P = Nx*Ny.
// Device layout of the state: kappa fastest, one contiguous spectral column slice per (i,j,n):
//   (n*P + c)*Nk + m.
// For each direction bin n this is the transpose of an Nk x P matrix, done in 32 x 32 tiles
// through shared memory so both sides are read and written in full 128-byte lines.
#include <cuda_runtime.h>

#include "rpl_internal.h"

namespace rpl {

namespace {

constexpr int TILE = 32, ROWS = 8;

// src: rows m0 .. m0+mc-1 of slices n0 .. n0+nc-1 in caller layout, starting at (n0, m0)
// dst: device layout, whole array
template <typename S, typename D>
__global__ void to_device_kernel(const S* __restrict__ src, D* __restrict__ dst, int64_t P, int64_t Nk,
                                 int64_t n0, int64_t m0, int64_t mc, int64_t src_slice_stride) {
    __shared__ D tile[TILE][TILE + 1];
    const int64_t c0 = (int64_t)blockIdx.x * TILE, mb = (int64_t)blockIdx.y * TILE;
    const int64_t n = n0 + blockIdx.z;
    const S* s = src + (int64_t)blockIdx.z * src_slice_stride;
    for (int r = threadIdx.y; r < TILE; r += ROWS) {
        const int64_t m = mb + r, c = c0 + threadIdx.x;
        if (m < mc && c < P) tile[r][threadIdx.x] = (D)s[m * P + c];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < TILE; r += ROWS) {
        const int64_t c = c0 + r, m = mb + threadIdx.x;
        if (m < mc && c < P) dst[(n * P + c) * Nk + m0 + m] = tile[threadIdx.x][r];
    }
}

template <typename S, typename D>
__global__ void from_device_kernel(const S* __restrict__ src, D* __restrict__ dst, int64_t P, int64_t Nk,
                                   int64_t n0, int64_t m0, int64_t mc, int64_t dst_slice_stride) {
    __shared__ D tile[TILE][TILE + 1];
    const int64_t c0 = (int64_t)blockIdx.x * TILE, mb = (int64_t)blockIdx.y * TILE;
    const int64_t n = n0 + blockIdx.z;
    D* d = dst + (int64_t)blockIdx.z * dst_slice_stride;
    for (int r = threadIdx.y; r < TILE; r += ROWS) {
        const int64_t c = c0 + r, m = mb + threadIdx.x;
        if (m < mc && c < P) tile[r][threadIdx.x] = (D)src[(n * P + c) * Nk + m0 + m];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < TILE; r += ROWS) {
        const int64_t m = mb + r, c = c0 + threadIdx.x;
        if (m < mc && c < P) d[m * P + c] = tile[threadIdx.x][r];
    }
}

// Coefficient record per (i,j,m), device order (j*Nx + i)*Nk + m, 8 doubles:
// Ux, Uy, Ux_x, Ux_y, Uy_x, Uy_y, c_g magnitude (depth field; else 0), kappa.
__global__ void coef_kernel(int64_t Nx, int64_t Ny, int64_t Nk, const double* __restrict__ coupling,
                            const double* __restrict__ cgmag, const double* __restrict__ kappa,
                            double* __restrict__ coef) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t P = Nx * Ny, c3 = P * Nk;
    if (t >= c3) return;
    const int64_t m = t % Nk, c = t / Nk;     // device order
    const int64_t x = c + P * m;              // caller order of the coupling arrays
    double* r = coef + 8 * t;
    if (coupling) {
        r[0] = coupling[x];
        r[1] = coupling[c3 + x];
        r[2] = coupling[4 * c3 + x];
        r[3] = coupling[5 * c3 + x];
        r[4] = coupling[6 * c3 + x];
        r[5] = coupling[7 * c3 + x];
    } else {
        r[0] = r[1] = r[2] = r[3] = r[4] = r[5] = 0.0;
    }
    r[6] = cgmag ? cgmag[x] : 0.0;
    r[7] = kappa[m];
}

constexpr int COEF_THREADS = 256;

// Coefficient records (Ux, Uy, Ux_x, Ux_y, Uy_x, Uy_y; fields 6 and 7 are kept) from the device-order
// velocity, with the periodic centred gradients of wave_current_refraction.jl:7-19. A block's 256
// records are assembled in shared memory and written back whole with 16-byte stores, so every DRAM
// sector is written in full.
__global__ void __launch_bounds__(COEF_THREADS)
coef_from_U_kernel(int64_t Nx, int64_t Ny, int Nk, const double* __restrict__ U, double dx_inv, double dy_inv,
                   double* __restrict__ coef) {
    __shared__ double2 rec[COEF_THREADS * 4];
    const int64_t P = Nx * Ny, c3 = P * Nk;
    const int64_t t0 = (int64_t)blockIdx.x * COEF_THREADS, t = t0 + threadIdx.x;
    if (t < c3) {
        const int64_t c = t / Nk, m = t - c * Nk;
        const int64_t j = c / Nx, i = c - j * Nx;
        const int64_t ip = i == Nx - 1 ? 0 : i + 1, im = i == 0 ? Nx - 1 : i - 1;
        const int64_t jp = j == Ny - 1 ? 0 : j + 1, jm = j == 0 ? Ny - 1 : j - 1;
        const int64_t xp = (j * Nx + ip) * Nk + m, xm = (j * Nx + im) * Nk + m;
        const int64_t yp = (jp * Nx + i) * Nk + m, ym = (jm * Nx + i) * Nk + m;
        const double* Uy = U + c3;
        double2* r = rec + threadIdx.x * 4;
        r[0] = make_double2(U[t], Uy[t]);
        r[1] = make_double2((U[xp] - U[xm]) * (dx_inv / 2.0), (U[yp] - U[ym]) * (dy_inv / 2.0));
        r[2] = make_double2((Uy[xp] - Uy[xm]) * (dx_inv / 2.0), (Uy[yp] - Uy[ym]) * (dy_inv / 2.0));
        r[3] = *reinterpret_cast<const double2*>(coef + 8 * t + 6);
    }
    __syncthreads();
    const int n = (int)(min((int64_t)COEF_THREADS, c3 - t0) * 4);
    double2* out = reinterpret_cast<double2*>(coef + 8 * t0);
    for (int k = threadIdx.x; k < n; k += COEF_THREADS) out[k] = rec[k];
}

// Device-order velocity -> the caller-order coupling arrays Ux, Uy, dUx/dkappa, dUy/dkappa (x fastest).
__global__ void export_U_kernel(int64_t P, int Nk, const double* __restrict__ U, double* __restrict__ out) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t c3 = P * Nk;
    if (t >= c3) return;
    const int64_t c = t / Nk, m = t - c * Nk;
    const int64_t x = c + P * m;
#pragma unroll
    for (int a = 0; a < 4; ++a) out[a * c3 + x] = U[a * c3 + t];
}

template <typename S, typename D>
cudaError_t to_dev(const void* src, void* dst, const Handle& h, int64_t n0, int64_t nc, int64_t m0, int64_t mc,
                   cudaStream_t s) {
    const int64_t P = h.cells, Nk = h.desc.Nk;
    dim3 grid((unsigned)((P + TILE - 1) / TILE), (unsigned)((mc + TILE - 1) / TILE), (unsigned)nc);
    to_device_kernel<S, D><<<grid, dim3(TILE, ROWS), 0, s>>>((const S*)src, (D*)dst, P, Nk, n0, m0, mc, Nk * P);
    return cudaGetLastError();
}

template <typename S, typename D>
cudaError_t from_dev(const void* src, void* dst, const Handle& h, int64_t n0, int64_t nc, int64_t m0, int64_t mc,
                     cudaStream_t s) {
    const int64_t P = h.cells, Nk = h.desc.Nk;
    dim3 grid((unsigned)((P + TILE - 1) / TILE), (unsigned)((mc + TILE - 1) / TILE), (unsigned)nc);
    from_device_kernel<S, D><<<grid, dim3(TILE, ROWS), 0, s>>>((const S*)src, (D*)dst, P, Nk, n0, m0, mc, Nk * P);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_to_device_layout(const Handle& h, const void* src, int src_dtype, void* dst, int dst_dtype,
                                    int64_t n0, int64_t nc, int64_t m0, int64_t mc, cudaStream_t s) {
    if (src_dtype == RPL_F64 && dst_dtype == RPL_F64) return to_dev<double, double>(src, dst, h, n0, nc, m0, mc, s);
    if (src_dtype == RPL_F64 && dst_dtype == RPL_F32) return to_dev<double, float>(src, dst, h, n0, nc, m0, mc, s);
    if (src_dtype == RPL_F32 && dst_dtype == RPL_F64) return to_dev<float, double>(src, dst, h, n0, nc, m0, mc, s);
    return to_dev<float, float>(src, dst, h, n0, nc, m0, mc, s);
}

cudaError_t launch_from_device_layout(const Handle& h, const void* src, int src_dtype, void* dst, int dst_dtype,
                                      int64_t n0, int64_t nc, int64_t m0, int64_t mc, cudaStream_t s) {
    if (src_dtype == RPL_F64 && dst_dtype == RPL_F64) return from_dev<double, double>(src, dst, h, n0, nc, m0, mc, s);
    if (src_dtype == RPL_F64 && dst_dtype == RPL_F32) return from_dev<double, float>(src, dst, h, n0, nc, m0, mc, s);
    if (src_dtype == RPL_F32 && dst_dtype == RPL_F64) return from_dev<float, double>(src, dst, h, n0, nc, m0, mc, s);
    return from_dev<float, float>(src, dst, h, n0, nc, m0, mc, s);
}

cudaError_t launch_coef(const Handle& h, cudaStream_t s) {
    const rpl_desc& d = h.desc;
    const int64_t c3 = d.Nx * d.Ny * d.Nk;
    coef_kernel<<<(unsigned)((c3 + 255) / 256), 256, 0, s>>>(d.Nx, d.Ny, d.Nk, h.currents_set ? h.d_coupling : nullptr,
                                                             h.d_cgmag, h.d_kappa, h.d_coef);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? launch_vel32(h, s) : e;
}

cudaError_t launch_coef_from_U(const Handle& h, cudaStream_t s) {
    const rpl_desc& d = h.desc;
    const int64_t c3 = d.Nx * d.Ny * d.Nk;
    coef_from_U_kernel<<<(unsigned)((c3 + COEF_THREADS - 1) / COEF_THREADS), COEF_THREADS, 0, s>>>(
        d.Nx, d.Ny, (int)d.Nk, h.d_U, 1.0 / d.dx, 1.0 / d.dy, h.d_coef);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? launch_vel32(h, s) : e;
}

cudaError_t launch_export_U(const Handle& h, cudaStream_t s) {
    const int64_t c3 = h.cells * h.desc.Nk;
    export_U_kernel<<<(unsigned)((c3 + 255) / 256), 256, 0, s>>>(h.cells, (int)h.desc.Nk, h.d_U, h.d_coupling);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_gradients(h, s);
}

}  // namespace rpl
