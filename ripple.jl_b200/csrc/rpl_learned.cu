// rpl_learned.cu -- the learned source inside the RK3 stage, and its training data.
//
// Per stage (rpl_api.cu launch_step): the feature kernel turns the stage input into network rows (per
// cell: the Nk*Np BF16 log-action features in bin order m + Nk n, and 4 extras) and flags every cell
// with an input outside the training bounds; the stress cap runs for flagged cells only; the network
// (rpl_mlp.cu) writes the per-bin outputs y; with a trust gate (rpl_set_learned_gate) cells whose network
// rates are stiff are flagged too; the stress cap runs for flagged cells; the tile kernel adds
// N * target_scale * sinh(y), or the plain FP32 sources for flagged cells. rpl_learned_sample writes the same rows plus the plain sources'
// rates as targets, in the network's output form asinh(rate / target_scale) (relative accuracy uniform
// over the rates' decades). Reference for the replaced terms: precomputed_sources.jl:396-439,
// pressure_correlation.jl:109-156, local_saturation.jl:30-47.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "rpl_internal.h"
#include "rpl_mlp.h"
#include "rpl_src32.cuh"

using bf16 = __nv_bfloat16;

namespace rpl {

namespace {

int lfail(int code, const std::string& msg) {
    set_last_error(msg);
    return code;
}

struct RowArgs {
    const float* N;         // device layout: ((n * P + c) * Nk + m)
    int64_t P;
    int Nk, Np;
    float shift, inv_scale, floor, inv_target;
    const double* U10;      // (P) wind speed, direction
    const double* theta;
    const double* depth;    // (P) depth field, or NULL with depth_const
    double depth_const;
    bf16* X;                // (rows x Nk*Np)
    float* E;               // (rows x 4)
    float* T;               // (rows x Nk*Np) targets (sample only)
    unsigned int* flag;     // (P) out-of-bounds flags (stage only)
    const float* lo;        // Nk*Np + 4 bounds (stage only)
    const float* hi;
};

// One warp per (cell, direction plane): lane m < Nk holds bin (m, n). SAMPLE: also the target rates.
template <bool SAMPLE>
__global__ void rows_kernel(const RowArgs a, const StageParams p) {
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= a.P * a.Np) return;  // uniform per warp
    const int64_t c = w / a.Np;
    const int n = (int)(w % a.Np);
    const int nb = a.Nk * a.Np;
    bool bad = false;
    if (lane < a.Nk) {
        const float v = __ldg(a.N + ((int64_t)n * a.P + c) * a.Nk + lane);
        const float x = (logf(fmaxf(v, a.floor)) - a.shift) * a.inv_scale;
        const int b = n * a.Nk + lane;
        a.X[c * nb + b] = __float2bfloat16_rn(x);
        if (SAMPLE) {
            const Cell32 q = load_cell32(p.cell32 + 8 * c);
            const Bin32 bn = load_bin32(p.bin32 + 8 * lane);
            const float2 cs = __ldg(p.cs32 + n);
            a.T[c * nb + b] = asinhf(rate32(p, q, bn, cs.x, cs.y, v) * a.inv_target);
        } else {
            bad = !(x >= a.lo[b] && x <= a.hi[b]);
        }
    }
    if (n == 0 && lane < 4) {
        const double U = a.U10[c], th = a.theta[c];
        const double d = a.depth ? a.depth[c] : a.depth_const;
        const float e = lane == 0 ? (float)(U / 30.0)
                                  : lane == 1 ? (float)sin(th) : lane == 2 ? (float)cos(th) : (float)(log10(d) / 4.0);
        a.E[c * 4 + lane] = e;
        if (!SAMPLE) bad = bad || !(e >= a.lo[nb + lane] && e <= a.hi[nb + lane]);
    }
    if (!SAMPLE && __any_sync(0xffffffffu, bad) && lane == 0) atomicOr(a.flag + c, 1u);
}

// Trust gate of the network: one warp per cell over its bins; a cell whose network rate would change any
// bin by more than `gate` of itself in one step (|lscale sinh(y)| * dt > gate) is flagged and takes the
// plain sources instead. Stiff cells are where a rate error compounds fastest from step to step.
__global__ void gate_kernel(const float* __restrict__ Y, int64_t P, int nb, float lscale, float limit,
                            unsigned int* flag) {
    const int64_t c = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (c >= P) return;  // uniform per warp
    float big = 0.0f;
    for (int b = lane; b < nb; b += 32) big = fmaxf(big, fabsf(__ldg(Y + c * nb + b)));
    for (int o = 16; o > 0; o >>= 1) big = fmaxf(big, __shfl_xor_sync(0xffffffffu, big, o));
    if (lane == 0 && lscale * sinhf(big) > limit) atomicOr(flag + c, 2u);
}

// Cells of this stage that take the plain sources, added to count[0]; count[1] counts the cells.
__global__ void count_kernel(const unsigned int* __restrict__ flag, int64_t P, unsigned long long* count) {
    unsigned long long k = 0;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < P; c += (int64_t)gridDim.x * blockDim.x)
        k += flag[c] != 0u;
    for (int o = 16; o > 0; o >>= 1) k += __shfl_xor_sync(0xffffffffu, k, o);
    if ((threadIdx.x & 31) == 0 && k) atomicAdd(count, k);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(count + 1, (unsigned long long)P);
}

RowArgs row_args(const Handle& h, const rpl_mlp_desc& md, const void* Nin) {
    RowArgs a{};
    a.N = (const float*)Nin;
    a.P = h.cells;
    a.Nk = (int)h.desc.Nk;
    a.Np = (int)h.desc.Np;
    a.shift = md.feature_shift;
    a.inv_scale = 1.0f / md.feature_scale;
    a.floor = md.log_floor;
    a.inv_target = 1.0f / md.target_scale;
    a.U10 = h.d_wind;
    a.theta = h.d_wind + h.cells;
    a.depth = h.desc.depth_kind == RPL_DEPTH_FIELD ? h.d_depth : nullptr;
    a.depth_const = h.desc.depth_kind == RPL_DEPTH_CONSTANT ? h.desc.depth_constant : 1e4;
    return a;
}

unsigned blocks_for_warps(int64_t warps) { return (unsigned)((warps * 32 + 255) / 256); }

int check_learned_handle(const Handle& h, const rpl_mlp* m) {
    if (h.precision != RPL_FP32) return lfail(RPL_ERR_UNSUPPORTED, "the learned source runs on FP32 models");
    if (!h.has_sources || h.src.wind_kind == RPL_WIND_NONE)
        return lfail(RPL_ERR_STATE, "the learned source stands in for wind-input sources; set them first");
    if (h.desc.Nk > 32 || h.desc.Nk * h.desc.Np != mlp_nbins(m))
        return lfail(RPL_ERR_ARGUMENT, "the network's nbins must equal Nk * Np (Nk <= 32)");
    if (!tile32_supported(h) || h.force_column_kernel)
        return lfail(RPL_ERR_UNSUPPORTED, "the learned source needs the FP32 tile kernel");
    return RPL_OK;
}

}  // namespace

cudaError_t launch_learned_stage_prep(const Handle& h, const void* Nin, double dt, cudaStream_t s) {
    const rpl_mlp_desc& md = mlp_desc(h.learned);
    RowArgs a = row_args(h, md, Nin);
    a.X = (bf16*)h.d_lx;
    a.E = h.d_le;
    a.flag = h.d_lflag;
    a.lo = h.d_lbounds;
    a.hi = h.d_lbounds + (mlp_nbins(h.learned) + 4);
    cudaError_t e = cudaMemsetAsync(h.d_lflag, 0, h.cells * sizeof(unsigned int), s);
    if (e != cudaSuccess) return e;
    const StageParams p = make_params(h, 1.0, 1);
    rows_kernel<false><<<blocks_for_warps(h.cells * h.desc.Np), 256, 0, s>>>(a, p);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int nb = mlp_nbins(h.learned);
    const float* ylo = h.lclamp ? h.d_lbounds + 2 * (nb + 4) : nullptr;
    e = mlp_forward(h.learned, (const bf16*)h.d_lx, nb, h.d_le, h.lrows, h.d_lr, nb, false, s, h.d_err, ylo,
                    ylo ? ylo + nb : nullptr);
    if (e != cudaSuccess) return e;
    if (h.lgate > 0.0) {
        gate_kernel<<<blocks_for_warps(h.cells), 256, 0, s>>>(h.d_lr, h.cells, nb, md.target_scale,
                                                              (float)(h.lgate / dt), h.d_lflag);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    count_kernel<<<148, 256, 0, s>>>(h.d_lflag, h.cells, h.d_lcount);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    // the stress cap of the plain sources, for the cells that take them
    if (h.src.stress_cap) e = launch_stress_factor(h, Nin, s, h.d_lflag);
    return e;
}

void free_learned(Handle* h) {
    void* ps[] = {h->d_lx, h->d_le, h->d_lr, h->d_lflag, h->d_lbounds, h->d_lcount};
    for (void* p : ps)
        if (p) cudaFree(p);
    h->d_lcount = nullptr;
    h->d_lx = nullptr;
    h->d_le = h->d_lr = h->d_lbounds = nullptr;
    h->d_lflag = nullptr;
    h->learned = nullptr;
    h->lrows = 0;
}

}  // namespace rpl

using rpl::Handle;

extern "C" {

int rpl_learned_sample(rpl_handle* hh, const rpl_mlp* m, void* X, float* E, float* T) {
    if (!hh || !m || !X || !E || !T) return rpl::lfail(RPL_ERR_ARGUMENT, "null argument");
    Handle* h = reinterpret_cast<Handle*>(hh);
    int st = rpl::check_learned_handle(*h, m);
    if (st) return st;
    cudaError_t e = cudaSetDevice(h->device);
    cudaStream_t s = h->stream;
    if (e == cudaSuccess) e = rpl::launch_wind(*h, h->time, s);
    if (e == cudaSuccess && h->src.stress_cap) e = rpl::launch_stress_factor(*h, h->N, s);
    if (e == cudaSuccess) {
        rpl::RowArgs a = rpl::row_args(*h, rpl::mlp_desc(m), h->N);
        a.X = (bf16*)X;
        a.E = E;
        a.T = T;
        const rpl::StageParams p = rpl::make_params(*h, 1.0, 1);
        rpl::rows_kernel<true><<<rpl::blocks_for_warps(h->cells * h->desc.Np), 256, 0, s>>>(a, p);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return rpl::lfail(RPL_ERR_CUDA, std::string("rpl_learned_sample: ") + cudaGetErrorString(e));
    return RPL_OK;
}

int rpl_set_learned_source(rpl_handle* hh, rpl_mlp* m, const float* lo, const float* hi, const float* ylo,
                           const float* yhi) {
    if (!hh) return rpl::lfail(RPL_ERR_ARGUMENT, "null handle");
    Handle* h = reinterpret_cast<Handle*>(hh);
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return rpl::lfail(RPL_ERR_CUDA, "cudaSetDevice");
    cudaStreamSynchronize(h->stream);
    rpl::free_learned(h);
    if (!m) return RPL_OK;
    int st = rpl::check_learned_handle(*h, m);
    if (st) return st;
    if (!lo || !hi) return rpl::lfail(RPL_ERR_ARGUMENT, "input bounds lo, hi are required");
    const int nb = rpl::mlp_nbins(m);
    for (int i = 0; i < nb + 4; ++i)
        if (!(lo[i] <= hi[i])) return rpl::lfail(RPL_ERR_ARGUMENT, "input bounds need lo <= hi");
    if ((ylo == nullptr) != (yhi == nullptr)) return rpl::lfail(RPL_ERR_ARGUMENT, "give both output bounds or neither");
    if (ylo)
        for (int i = 0; i < nb; ++i)
            if (!(ylo[i] <= yhi[i])) return rpl::lfail(RPL_ERR_ARGUMENT, "output bounds need ylo <= yhi");
    const int64_t rows = (h->cells + 127) / 128 * 128;
    const size_t nbound = (size_t)2 * (nb + 4) + 2 * nb;  // input lo, hi, output lo, hi
    const size_t need = rows * nb * (2 + 4) + rows * 16 + h->cells * 4 + nbound * 4;
    if (h->desc.memory_limit_bytes > 0 && h->bytes + (int64_t)need > h->desc.memory_limit_bytes)
        return rpl::lfail(RPL_ERR_OOM, "the learned source's buffers would exceed memory_limit_bytes");
    auto al = [&](auto** p, size_t bytes) { return cudaMalloc((void**)p, bytes); };
    if ((e = al(&h->d_lx, rows * nb * 2)) != cudaSuccess || (e = al(&h->d_le, rows * 16)) != cudaSuccess ||
        (e = al(&h->d_lr, rows * nb * 4)) != cudaSuccess ||
        (e = al(&h->d_lflag, h->cells * sizeof(unsigned int))) != cudaSuccess ||
        (e = al(&h->d_lbounds, nbound * 4)) != cudaSuccess || (e = al(&h->d_lcount, 16)) != cudaSuccess) {
        rpl::free_learned(h);
        return rpl::lfail(e == cudaErrorMemoryAllocation ? RPL_ERR_OOM : RPL_ERR_CUDA, "learned-source buffers");
    }
    std::vector<float> b(nbound, 0.0f);
    std::copy(lo, lo + nb + 4, b.begin());
    std::copy(hi, hi + nb + 4, b.begin() + nb + 4);
    if (ylo) {
        std::copy(ylo, ylo + nb, b.begin() + 2 * (nb + 4));
        std::copy(yhi, yhi + nb, b.begin() + 2 * (nb + 4) + nb);
    }
    if ((e = cudaMemsetAsync(h->d_lx, 0, rows * nb * 2, h->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(h->d_le, 0, rows * 16, h->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(h->d_lflag, 0, h->cells * sizeof(unsigned int), h->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(h->d_lcount, 0, 16, h->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(h->d_lbounds, b.data(), b.size() * 4, cudaMemcpyHostToDevice, h->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(h->stream)) != cudaSuccess) {
        rpl::free_learned(h);
        return rpl::lfail(RPL_ERR_CUDA, "learned-source set-up");
    }
    h->learned = m;
    h->lrows = rows;
    h->lclamp = ylo != nullptr;
    return RPL_OK;
}

int rpl_set_learned_gate(rpl_handle* hh, double max_rate_dt) {
    if (!hh) return rpl::lfail(RPL_ERR_ARGUMENT, "null handle");
    if (!(max_rate_dt >= 0.0) || !std::isfinite(max_rate_dt))
        return rpl::lfail(RPL_ERR_ARGUMENT, "the gate must be a finite value >= 0 (0: no gate)");
    reinterpret_cast<Handle*>(hh)->lgate = max_rate_dt;
    return RPL_OK;
}

int rpl_learned_outputs(rpl_handle* hh, float* Y) {
    if (!hh || !Y) return rpl::lfail(RPL_ERR_ARGUMENT, "null argument");
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h->learned) return rpl::lfail(RPL_ERR_STATE, "no learned source is set");
    cudaSetDevice(h->device);
    const size_t bytes = (size_t)h->cells * rpl::mlp_nbins(h->learned) * sizeof(float);
    cudaError_t e = cudaMemcpyAsync(Y, h->d_lr, bytes, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return rpl::lfail(RPL_ERR_CUDA, "rpl_learned_outputs");
    return RPL_OK;
}

int rpl_learned_fallback_totals(rpl_handle* hh, int64_t* fallback_cell_stages, int64_t* cell_stages) {
    if (!hh || !fallback_cell_stages || !cell_stages) return rpl::lfail(RPL_ERR_ARGUMENT, "null argument");
    Handle* h = reinterpret_cast<Handle*>(hh);
    *fallback_cell_stages = *cell_stages = 0;
    if (!h->learned) return RPL_OK;
    cudaSetDevice(h->device);
    unsigned long long v[2] = {0, 0};
    cudaError_t e = cudaMemcpyAsync(v, h->d_lcount, 16, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return rpl::lfail(RPL_ERR_CUDA, "rpl_learned_fallback_totals");
    *fallback_cell_stages = (int64_t)v[0];
    *cell_stages = (int64_t)v[1];
    return RPL_OK;
}

int rpl_learned_fallback_cells(rpl_handle* hh, int64_t* count) {
    if (!hh || !count) return rpl::lfail(RPL_ERR_ARGUMENT, "null argument");
    Handle* h = reinterpret_cast<Handle*>(hh);
    *count = 0;
    if (!h->learned) return RPL_OK;
    cudaSetDevice(h->device);
    std::vector<unsigned int> f(h->cells);
    cudaError_t e = cudaMemcpyAsync(f.data(), h->d_lflag, h->cells * 4, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return rpl::lfail(RPL_ERR_CUDA, "rpl_learned_fallback_cells");
    int64_t c = 0;
    for (unsigned int v : f) c += v != 0;
    *count = c;
    return RPL_OK;
}

}  // extern "C"
