// rpl_mlp.cu -- the learned-source MLP: parameters, forward and backward passes on the tensor-core GEMM
// (rpl_gemm.cu), Adam, and the C-ABI entry points rpl_mlp_* / rpl_gemm_bf16.
//
// Network: x (nbins BF16 features) and e (4 FP32 extras) -> z1 = W1 x + W1e e + b1 -> h1 = GELU(z1)
// (GELU in its tanh form, see rpl_gemm.cu)
// -> h2 = GELU(W2 h1 + b2) -> h3 = GELU(W3 h2 + b3) -> y = W4 h3 + b4 (nbins, FP32). Rows are cells.
// Forward GEMMs keep activations in BF16 (and, when training, their transposes and the FP32
// pre-activations); backward: dY = 2 (y - t) / (B nbins), dW_l = dZ_l^T H_{l-1} and
// dZ_{l-1} = (dZ_l W_l) * GELU'(z_{l-1}) on the same GEMM, gradients in FP32, Adam on FP32 masters, then
// BF16 copies (and transposes for the backward products) refreshed.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <new>
#include <string>
#include <vector>

#include "rpl_internal.h"
#include "rpl_mlp.h"

using bf16 = __nv_bfloat16;

namespace {

int mfail(int code, const std::string& msg) {
    rpl::set_last_error(msg);
    return code;
}
int mcuda(cudaError_t e, const char* what) {
    return mfail(e == cudaErrorMemoryAllocation ? RPL_ERR_OOM : RPL_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
#define MLP_CUDA(call)                                  \
    do {                                                \
        cudaError_t e_ = (call);                        \
        if (e_ != cudaSuccess) return mcuda(e_, #call); \
    } while (0)

// ---- small kernels ----

// 32 x 32 tiles: X[r][c] = src row rows[r] (or r0 + r), col c; Xt[c][r] (optional, row stride ldt).
__global__ void gather_bf16_kernel(const bf16* __restrict__ src, int64_t lds, const int32_t* __restrict__ rows,
                                   int64_t r0, int n, int cols, bf16* __restrict__ dst, int64_t ldd,
                                   bf16* __restrict__ dstT, int64_t ldt) {
    __shared__ bf16 tile[32][33];
    const int c0 = blockIdx.x * 32, rb = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = rb + k, c = c0 + threadIdx.x;
        bf16 v = __float2bfloat16_rn(0.0f);
        if (r < n && c < cols) {
            const int64_t sr = rows ? (int64_t)rows[r] : r0 + r;
            v = src[sr * lds + c];
            dst[(int64_t)r * ldd + c] = v;
        }
        tile[k][threadIdx.x] = v;
    }
    if (!dstT) return;
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c = c0 + k, r = rb + threadIdx.x;
        if (c < cols && r < n) dstT[(int64_t)c * ldt + r] = tile[threadIdx.x][k];
    }
}

__global__ void gather_f32_kernel(const float* __restrict__ src, int64_t lds, const int32_t* __restrict__ rows,
                                  int n, int cols, float* __restrict__ dst, int64_t ldd) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)n * cols) return;
    const int r = (int)(t / cols), c = (int)(t % cols);
    dst[(int64_t)r * ldd + c] = src[(int64_t)rows[r] * lds + c];
}

// Loss and output gradient over 32 x 32 tiles: d = y - t, loss += d^2, dY = bf16(2 d / count), dYt = dY^T.
__global__ void loss_grad_kernel(const float* __restrict__ Y, const float* __restrict__ T, int n, int cols,
                                 float inv_count, bf16* __restrict__ dY, bf16* __restrict__ dYt, int64_t ldt,
                                 double* __restrict__ loss) {
    __shared__ bf16 tile[32][33];
    __shared__ float red[256];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    float acc = 0.0f;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        bf16 g = __float2bfloat16_rn(0.0f);
        if (r < n && c < cols) {
            const float d = Y[(int64_t)r * cols + c] - T[(int64_t)r * cols + c];
            acc += d * d;
            g = __float2bfloat16_rn(2.0f * d * inv_count);
            dY[(int64_t)r * cols + c] = g;
        }
        tile[k][threadIdx.x] = g;
    }
    const int tid = threadIdx.y * 32 + threadIdx.x;
    red[tid] = acc;
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if (c < cols && r < n) dYt[(int64_t)c * ldt + r] = tile[threadIdx.x][k];
    }
    for (int s = 128; s > 0; s >>= 1) {
        __syncthreads();
        if (tid < s) red[tid] += red[tid + s];
    }
    if (tid == 0) atomicAdd(loss, (double)red[0]);
}

constexpr int RED_ROWS = 512;  // rows per block of the column reductions

// g[c] += sum_r D[r][c] over this block's RED_ROWS rows (bias gradients; g zeroed before). Blocks of
// 32 columns x 8 row lanes, one atomic add per column and block.
__global__ void colsum_kernel(const bf16* __restrict__ D, int n, int cols, float* __restrict__ g) {
    __shared__ float red[8][33];
    const int c = blockIdx.x * 32 + threadIdx.x;
    const int r0 = blockIdx.y * RED_ROWS, r1 = min(n, r0 + RED_ROWS);
    float s = 0.0f;
    if (c < cols)
        for (int r = r0 + threadIdx.y; r < r1; r += 8) s += __bfloat162float(D[(int64_t)r * cols + c]);
    red[threadIdx.y][threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.y == 0 && c < cols) {
        float t = 0.0f;
        for (int k = 0; k < 8; ++k) t += red[k][threadIdx.x];
        atomicAdd(g + c, t);
    }
}

// g[h][e] += sum_r dZ[r][h] E[r][e] over this block's rows (gradient of the extra-input weights).
__global__ void extra_grad_kernel(const bf16* __restrict__ dZ, const float* __restrict__ E, int n, int hd,
                                  float* __restrict__ g) {
    __shared__ float red[8][4][33];
    const int h = blockIdx.x * 32 + threadIdx.x;
    const int r0 = blockIdx.y * RED_ROWS, r1 = min(n, r0 + RED_ROWS);
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
    if (h < hd)
        for (int r = r0 + threadIdx.y; r < r1; r += 8) {
            const float d = __bfloat162float(dZ[(int64_t)r * hd + h]);
            const float4 e = *reinterpret_cast<const float4*>(E + (int64_t)r * 4);
            s0 = fmaf(d, e.x, s0);
            s1 = fmaf(d, e.y, s1);
            s2 = fmaf(d, e.z, s2);
            s3 = fmaf(d, e.w, s3);
        }
    red[threadIdx.y][0][threadIdx.x] = s0;
    red[threadIdx.y][1][threadIdx.x] = s1;
    red[threadIdx.y][2][threadIdx.x] = s2;
    red[threadIdx.y][3][threadIdx.x] = s3;
    __syncthreads();
    if (threadIdx.y < 4 && h < hd) {
        float t = 0.0f;
        for (int k = 0; k < 8; ++k) t += red[k][threadIdx.y][threadIdx.x];
        atomicAdd(g + h * 4 + threadIdx.y, t);
    }
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1,
                            float* __restrict__ m2, int64_t n, float lr, float c1, float c2) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float gi = g[t];
    const float a = 0.9f * m1[t] + 0.1f * gi;
    const float b = 0.999f * m2[t] + 0.001f * gi * gi;
    m1[t] = a;
    m2[t] = b;
    p[t] -= lr * (a * c1) / (sqrtf(b * c2) + 1e-8f);
}

// BF16 copy W (rows x cols) and optionally its transpose Wt (cols x rows), 32 x 32 tiles.
__global__ void refresh_kernel(const float* __restrict__ W, int rows, int cols, bf16* __restrict__ Wb,
                               bf16* __restrict__ Wt) {
    __shared__ bf16 tile[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        bf16 v = __float2bfloat16_rn(0.0f);
        if (r < rows && c < cols) {
            v = __float2bfloat16_rn(W[(int64_t)r * cols + c]);
            Wb[(int64_t)r * cols + c] = v;
        }
        tile[k][threadIdx.x] = v;
    }
    if (!Wt) return;
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if (c < cols && r < rows) Wt[(int64_t)c * rows + r] = tile[threadIdx.x][k];
    }
}

uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // namespace

struct rpl_mlp {
    rpl_mlp_desc d{};
    cudaStream_t stream = nullptr;
    bool own_stream = true;
    int nb = 0, hd = 0, R = 0;
    int64_t np = 0, oW1 = 0, oW1e = 0, ob1 = 0, oW2 = 0, ob2 = 0, oW3 = 0, ob3 = 0, oW4 = 0, ob4 = 0;
    float *P = nullptr, *G = nullptr, *M1 = nullptr, *M2 = nullptr;
    bf16 *W1b = nullptr, *W2b = nullptr, *W3b = nullptr, *W4b = nullptr, *W2t = nullptr, *W3t = nullptr, *W4t = nullptr;
    bf16 *X = nullptr, *Xt = nullptr, *H1 = nullptr, *H1t = nullptr, *H2 = nullptr, *H2t = nullptr, *H3 = nullptr,
         *H3t = nullptr, *dY = nullptr, *dYt = nullptr, *dZ3 = nullptr, *dZ3t = nullptr, *dZ2 = nullptr,
         *dZ2t = nullptr, *dZ1 = nullptr, *dZ1t = nullptr;
    float *E = nullptr, *Z1 = nullptr, *Z2 = nullptr, *Z3 = nullptr, *Y = nullptr, *T = nullptr;
    double* d_loss = nullptr;
    unsigned int* d_err = nullptr;
    int64_t step = 0;
    std::vector<void*> allocs;
};

namespace rpl {

int mlp_nbins(const rpl_mlp* m) { return m->nb; }
const rpl_mlp_desc& mlp_desc(const rpl_mlp* m) { return m->d; }

// 256-column tiles when N allows them and they still give every SM a tile; else 128.
static int pick_bn(int M, int N) { return (N % 256 == 0 && (M / 128) * (N / 256) >= 148) ? 256 : 128; }

static cudaError_t gemm(rpl_mlp* m, GemmArgs g, cudaStream_t s) {
    g.err = m->d_err;
    const int bn = pick_bn(g.M, g.N);
    if (!gemm_shape_ok(g, bn)) return cudaErrorInvalidValue;
    return launch_gemm(g, bn, s);
}

// Forward over n rows (n % 128 == 0) of X (row stride ldx) / E, output rows of Y (row stride ldy). With
// `train` (n <= R) the pre-activations and transposed activations for the backward pass are kept.
cudaError_t mlp_forward(rpl_mlp* m, const bf16* X, int64_t ldx, const float* E, int64_t n, float* Y, int64_t ldy,
                        bool train, cudaStream_t s, unsigned int* err, const float* ylo, const float* yhi) {
    const int nb = m->nb, hd = m->hd, R = m->R;
    auto run = [&](GemmArgs g) {
        g.err = err ? err : m->d_err;
        const int bn = pick_bn(g.M, g.N);
        if (!gemm_shape_ok(g, bn)) return cudaErrorInvalidValue;
        return launch_gemm(g, bn, s);
    };
    for (int64_t r0 = 0; r0 < n; r0 += R) {
        const int rows = (int)std::min<int64_t>(R, n - r0);
        GemmArgs g{};
        g.M = rows;
        g.epi = EPI_BIAS_GELU;
        // layer 1
        g.A = X + r0 * ldx; g.lda = ldx; g.B = m->W1b; g.ldb = nb; g.K = nb; g.N = hd;
        g.bias = m->P + m->ob1; g.extra = E + r0 * 4; g.wextra = m->P + m->oW1e;
        g.out_f32 = train ? m->Z1 : nullptr; g.ldo = hd;
        g.out_bf16 = m->H1; g.ldh = hd; g.out_bf16_t = train ? m->H1t : nullptr; g.ldt = R;
        cudaError_t e = run(g);
        if (e != cudaSuccess) return e;
        // layers 2 and 3
        g.extra = nullptr; g.wextra = nullptr; g.K = hd;
        g.A = m->H1; g.lda = hd; g.B = m->W2b; g.ldb = hd; g.bias = m->P + m->ob2;
        g.out_f32 = train ? m->Z2 : nullptr; g.out_bf16 = m->H2; g.out_bf16_t = train ? m->H2t : nullptr;
        if ((e = run(g)) != cudaSuccess) return e;
        g.A = m->H2; g.B = m->W3b; g.bias = m->P + m->ob3;
        g.out_f32 = train ? m->Z3 : nullptr; g.out_bf16 = m->H3; g.out_bf16_t = train ? m->H3t : nullptr;
        if ((e = run(g)) != cudaSuccess) return e;
        // output layer
        GemmArgs o{};
        o.M = rows; o.epi = EPI_BIAS; o.A = m->H3; o.lda = hd; o.B = m->W4b; o.ldb = hd; o.K = hd; o.N = nb;
        o.bias = m->P + m->ob4; o.out_f32 = Y + r0 * ldy; o.ldo = ldy; o.clamp_lo = ylo; o.clamp_hi = yhi;
        if ((e = run(o)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace rpl

namespace {

cudaError_t refresh(rpl_mlp* m, cudaStream_t s) {
    const dim3 blk(32, 8);
    auto go = [&](const float* W, int rows, int cols, bf16* Wb, bf16* Wt) {
        dim3 grid((cols + 31) / 32, (rows + 31) / 32);
        refresh_kernel<<<grid, blk, 0, s>>>(W, rows, cols, Wb, Wt);
    };
    go(m->P + m->oW1, m->hd, m->nb, m->W1b, nullptr);
    go(m->P + m->oW2, m->hd, m->hd, m->W2b, m->W2t);
    go(m->P + m->oW3, m->hd, m->hd, m->W3b, m->W3t);
    go(m->P + m->oW4, m->nb, m->hd, m->W4b, m->W4t);
    return cudaGetLastError();
}

// Gradient of the batch `rows` into m->G (and the loss into m->d_loss).
int batch_gradient(rpl_mlp* m, const bf16* X, const float* E, const float* T, const int32_t* rows, int B) {
    cudaStream_t s = m->stream;
    const int nb = m->nb, hd = m->hd, R = m->R;
    const dim3 blk(32, 8);
    MLP_CUDA(cudaMemsetAsync(m->d_loss, 0, sizeof(double), s));
    gather_bf16_kernel<<<dim3((nb + 31) / 32, (B + 31) / 32), blk, 0, s>>>(X, nb, rows, 0, B, nb, m->X, nb, m->Xt, R);
    gather_f32_kernel<<<(unsigned)(((int64_t)B * 4 + 255) / 256), 256, 0, s>>>(E, 4, rows, B, 4, m->E, 4);
    gather_f32_kernel<<<(unsigned)(((int64_t)B * nb + 255) / 256), 256, 0, s>>>(T, nb, rows, B, nb, m->T, nb);
    MLP_CUDA(cudaGetLastError());
    MLP_CUDA(rpl::mlp_forward(m, m->X, nb, m->E, B, m->Y, nb, true, s, nullptr));
    loss_grad_kernel<<<dim3((nb + 31) / 32, (B + 31) / 32), blk, 0, s>>>(m->Y, m->T, B, nb, 1.0f / ((float)B * nb), m->dY,
                                                                        m->dYt, R, m->d_loss);
    MLP_CUDA(cudaGetLastError());
    using rpl::GemmArgs;
    auto wgrad = [&](const bf16* At, const bf16* Bt, int M, int N, float* out) {
        GemmArgs g{};
        g.A = At; g.lda = R; g.B = Bt; g.ldb = R; g.M = M; g.N = N; g.K = B; g.epi = rpl::EPI_F32;
        g.out_f32 = out; g.ldo = N;
        return rpl::gemm(m, g, s);
    };
    auto dgrad = [&](const bf16* D, int Din, const bf16* Wt, const float* pre, bf16* dZ, bf16* dZt) {
        GemmArgs g{};
        g.A = D; g.lda = Din; g.B = Wt; g.ldb = Din; g.M = B; g.N = hd; g.K = Din; g.epi = rpl::EPI_GELU_BWD;
        g.pre = pre; g.ldp = hd; g.out_bf16 = dZ; g.ldh = hd; g.out_bf16_t = dZt; g.ldt = R;
        return rpl::gemm(m, g, s);
    };
    float* G = m->G;
    MLP_CUDA(cudaMemsetAsync(G, 0, m->np * sizeof(float), s));  // the reductions below accumulate
    const dim3 rblk(32, 8);
    auto rgrid = [&](int cols) { return dim3((cols + 31) / 32, (B + RED_ROWS - 1) / RED_ROWS); };
    MLP_CUDA(wgrad(m->dYt, m->H3t, nb, hd, G + m->oW4));
    colsum_kernel<<<rgrid(nb), rblk, 0, s>>>(m->dY, B, nb, G + m->ob4);
    MLP_CUDA(dgrad(m->dY, nb, m->W4t, m->Z3, m->dZ3, m->dZ3t));
    MLP_CUDA(wgrad(m->dZ3t, m->H2t, hd, hd, G + m->oW3));
    colsum_kernel<<<rgrid(hd), rblk, 0, s>>>(m->dZ3, B, hd, G + m->ob3);
    MLP_CUDA(dgrad(m->dZ3, hd, m->W3t, m->Z2, m->dZ2, m->dZ2t));
    MLP_CUDA(wgrad(m->dZ2t, m->H1t, hd, hd, G + m->oW2));
    colsum_kernel<<<rgrid(hd), rblk, 0, s>>>(m->dZ2, B, hd, G + m->ob2);
    MLP_CUDA(dgrad(m->dZ2, hd, m->W2t, m->Z1, m->dZ1, m->dZ1t));
    MLP_CUDA(wgrad(m->dZ1t, m->Xt, hd, nb, G + m->oW1));
    colsum_kernel<<<rgrid(hd), rblk, 0, s>>>(m->dZ1, B, hd, G + m->ob1);
    extra_grad_kernel<<<rgrid(hd), rblk, 0, s>>>(m->dZ1, m->E, B, hd, G + m->oW1e);
    MLP_CUDA(cudaGetLastError());
    return RPL_OK;
}

int check_err_word(rpl_mlp* m) {
    unsigned int w = 0;
    MLP_CUDA(cudaMemcpyAsync(&w, m->d_err, sizeof(w), cudaMemcpyDeviceToHost, m->stream));
    MLP_CUDA(cudaStreamSynchronize(m->stream));
    if (w) {
        MLP_CUDA(cudaMemsetAsync(m->d_err, 0, sizeof(unsigned int), m->stream));
        return mfail(RPL_ERR_DEVICE, "a tensor-core GEMM gave up waiting for its MMAs");
    }
    return RPL_OK;
}

int check_batch(const rpl_mlp* m, const void* X, const float* E, const float* T, const int32_t* rows, int B) {
    if (!m) return mfail(RPL_ERR_ARGUMENT, "null network");
    if (!X || !E || !T || !rows) return mfail(RPL_ERR_ARGUMENT, "X, E, T and rows must be device pointers");
    if (B <= 0 || B % 128 || B > m->R) return mfail(RPL_ERR_ARGUMENT, "batch must be a positive multiple of 128 <= rows");
    if (((uintptr_t)E & 15u) != 0) return mfail(RPL_ERR_ARGUMENT, "E must be 16-byte aligned");
    return RPL_OK;
}

void destroy_mlp(rpl_mlp* m) {
    for (void* p : m->allocs) cudaFree(p);
    if (m->own_stream && m->stream) cudaStreamDestroy(m->stream);
    delete m;
}

}  // namespace

extern "C" {

int rpl_mlp_create(const rpl_mlp_desc* d, rpl_mlp** out) {
    if (!out) return mfail(RPL_ERR_ARGUMENT, "out must not be NULL");
    *out = nullptr;
    if (!d || d->abi_version != RPL_ABI_VERSION) return mfail(RPL_ERR_ARGUMENT, "rpl_mlp_desc abi_version mismatch");
    if (d->nbins <= 0 || d->nbins % 128) return mfail(RPL_ERR_ARGUMENT, "nbins must be a positive multiple of 128");
    if (d->hidden <= 0 || d->hidden % 256) return mfail(RPL_ERR_ARGUMENT, "hidden must be a positive multiple of 256");
    if (d->rows <= 0 || d->rows % 128) return mfail(RPL_ERR_ARGUMENT, "rows must be a positive multiple of 128");
    if (!(d->feature_scale > 0.f) || !(d->target_scale > 0.f) || !(d->log_floor > 0.f))
        return mfail(RPL_ERR_ARGUMENT, "feature_scale, target_scale and log_floor must be positive");
    cudaError_t err = cudaSetDevice(d->device);
    if (err != cudaSuccess) return mcuda(err, "cudaSetDevice");
    rpl_mlp* m = new (std::nothrow) rpl_mlp();
    if (!m) return mfail(RPL_ERR_OOM, "host allocation failed");
    m->d = *d;
    m->nb = d->nbins;
    m->hd = d->hidden;
    m->R = d->rows;
    const int64_t nb = m->nb, hd = m->hd, R = m->R;
    m->oW1 = 0;
    m->oW1e = m->oW1 + hd * nb;
    m->ob1 = m->oW1e + hd * 4;
    m->oW2 = m->ob1 + hd;
    m->ob2 = m->oW2 + hd * hd;
    m->oW3 = m->ob2 + hd;
    m->ob3 = m->oW3 + hd * hd;
    m->oW4 = m->ob3 + hd;
    m->ob4 = m->oW4 + nb * hd;
    m->np = m->ob4 + nb;
    auto fail_out = [&](int code) {
        destroy_mlp(m);
        return code;
    };
    if ((err = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return fail_out(mcuda(err, "cudaStreamCreate"));
    auto alloc = [&](auto** p, size_t count) {
        cudaError_t e = cudaMalloc((void**)p, count * sizeof(**p));
        if (e == cudaSuccess) m->allocs.push_back((void*)*p);
        return e;
    };
    const cudaError_t es[] = {
        alloc(&m->P, m->np), alloc(&m->G, m->np), alloc(&m->M1, m->np), alloc(&m->M2, m->np),
        alloc(&m->W1b, hd * nb), alloc(&m->W2b, hd * hd), alloc(&m->W3b, hd * hd), alloc(&m->W4b, nb * hd),
        alloc(&m->W2t, hd * hd), alloc(&m->W3t, hd * hd), alloc(&m->W4t, hd * nb),
        alloc(&m->X, R * nb), alloc(&m->Xt, nb * R), alloc(&m->H1, R * hd), alloc(&m->H1t, hd * R),
        alloc(&m->H2, R * hd), alloc(&m->H2t, hd * R), alloc(&m->H3, R * hd), alloc(&m->H3t, hd * R),
        alloc(&m->dY, R * nb), alloc(&m->dYt, nb * R), alloc(&m->dZ3, R * hd), alloc(&m->dZ3t, hd * R),
        alloc(&m->dZ2, R * hd), alloc(&m->dZ2t, hd * R), alloc(&m->dZ1, R * hd), alloc(&m->dZ1t, hd * R),
        alloc(&m->E, R * 4), alloc(&m->Z1, R * hd), alloc(&m->Z2, R * hd), alloc(&m->Z3, R * hd),
        alloc(&m->Y, R * nb), alloc(&m->T, R * nb), alloc(&m->d_loss, 1), alloc(&m->d_err, 1)};
    for (cudaError_t e : es)
        if (e != cudaSuccess) return fail_out(mcuda(e, "cudaMalloc"));
    // Glorot-uniform weights from a seeded generator, zero biases; the output layer starts small.
    std::vector<float> p(m->np, 0.0f);
    uint64_t s = d->seed;
    auto fill = [&](int64_t off, int64_t rows, int64_t cols, float gain) {
        const float a = gain * std::sqrt(6.0f / (float)(rows + cols));
        for (int64_t i = 0; i < rows * cols; ++i)
            p[off + i] = a * (2.0f * (float)((splitmix(s) >> 11) * (1.0 / 9007199254740992.0)) - 1.0f);
    };
    fill(m->oW1, hd, nb, 1.0f);
    fill(m->oW1e, hd, 4, 1.0f);
    fill(m->oW2, hd, hd, 1.0f);
    fill(m->oW3, hd, hd, 1.0f);
    fill(m->oW4, nb, hd, 0.1f);
    if ((err = cudaMemcpyAsync(m->P, p.data(), m->np * 4, cudaMemcpyHostToDevice, m->stream)) != cudaSuccess ||
        (err = cudaMemsetAsync(m->M1, 0, m->np * 4, m->stream)) != cudaSuccess ||
        (err = cudaMemsetAsync(m->M2, 0, m->np * 4, m->stream)) != cudaSuccess ||
        (err = cudaMemsetAsync(m->d_err, 0, 4, m->stream)) != cudaSuccess ||
        (err = refresh(m, m->stream)) != cudaSuccess || (err = cudaStreamSynchronize(m->stream)) != cudaSuccess)
        return fail_out(mcuda(err, "network initialisation"));
    *out = m;
    return RPL_OK;
}

int rpl_mlp_destroy(rpl_mlp* m) {
    if (!m) return RPL_OK;
    cudaSetDevice(m->d.device);
    cudaStreamSynchronize(m->stream);
    destroy_mlp(m);
    return RPL_OK;
}

int rpl_mlp_set_stream(rpl_mlp* m, void* stream) {
    if (!m) return mfail(RPL_ERR_ARGUMENT, "null network");
    MLP_CUDA(cudaSetDevice(m->d.device));
    MLP_CUDA(cudaStreamSynchronize(m->stream));
    if (m->own_stream) cudaStreamDestroy(m->stream);
    m->stream = (cudaStream_t)stream;  // NULL: the legacy default stream
    m->own_stream = false;
    return RPL_OK;
}

int rpl_mlp_param_count(const rpl_mlp* m, int64_t* count) {
    if (!m || !count) return mfail(RPL_ERR_ARGUMENT, "null argument");
    *count = m->np;
    return RPL_OK;
}

int rpl_mlp_get_params(rpl_mlp* m, float* host) {
    if (!m || !host) return mfail(RPL_ERR_ARGUMENT, "null argument");
    MLP_CUDA(cudaSetDevice(m->d.device));
    MLP_CUDA(cudaMemcpyAsync(host, m->P, m->np * 4, cudaMemcpyDeviceToHost, m->stream));
    MLP_CUDA(cudaStreamSynchronize(m->stream));
    return RPL_OK;
}

int rpl_mlp_set_params(rpl_mlp* m, const float* host) {
    if (!m || !host) return mfail(RPL_ERR_ARGUMENT, "null argument");
    for (int64_t i = 0; i < m->np; ++i)
        if (!std::isfinite(host[i])) return mfail(RPL_ERR_NONFINITE, "non-finite parameter");
    MLP_CUDA(cudaSetDevice(m->d.device));
    MLP_CUDA(cudaMemcpyAsync(m->P, host, m->np * 4, cudaMemcpyHostToDevice, m->stream));
    MLP_CUDA(cudaMemsetAsync(m->M1, 0, m->np * 4, m->stream));
    MLP_CUDA(cudaMemsetAsync(m->M2, 0, m->np * 4, m->stream));
    m->step = 0;
    MLP_CUDA(refresh(m, m->stream));
    MLP_CUDA(cudaStreamSynchronize(m->stream));
    return RPL_OK;
}

int rpl_mlp_gradients(rpl_mlp* m, const void* X, const float* E, const float* T, const int32_t* rows, int32_t B,
                      float* grads, double* loss) {
    int st = check_batch(m, X, E, T, rows, B);
    if (st) return st;
    MLP_CUDA(cudaSetDevice(m->d.device));
    if ((st = batch_gradient(m, (const bf16*)X, E, T, rows, B))) return st;
    double l = 0.0;
    if (grads) MLP_CUDA(cudaMemcpyAsync(grads, m->G, m->np * 4, cudaMemcpyDeviceToHost, m->stream));
    MLP_CUDA(cudaMemcpyAsync(&l, m->d_loss, sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    if ((st = check_err_word(m))) return st;
    if (loss) *loss = l / ((double)B * m->nb);
    return RPL_OK;
}

int rpl_mlp_train_step(rpl_mlp* m, const void* X, const float* E, const float* T, const int32_t* rows, int32_t B,
                       float lr, double* loss) {
    int st = check_batch(m, X, E, T, rows, B);
    if (st) return st;
    if (!(lr > 0.f)) return mfail(RPL_ERR_ARGUMENT, "learning rate must be positive");
    MLP_CUDA(cudaSetDevice(m->d.device));
    if ((st = batch_gradient(m, (const bf16*)X, E, T, rows, B))) return st;
    m->step += 1;
    const float c1 = (float)(1.0 / (1.0 - std::pow(0.9, (double)m->step)));
    const float c2 = (float)(1.0 / (1.0 - std::pow(0.999, (double)m->step)));
    adam_kernel<<<(unsigned)((m->np + 255) / 256), 256, 0, m->stream>>>(m->P, m->G, m->M1, m->M2, m->np, lr, c1, c2);
    MLP_CUDA(cudaGetLastError());
    MLP_CUDA(refresh(m, m->stream));
    if (loss) {
        double l = 0.0;
        MLP_CUDA(cudaMemcpyAsync(&l, m->d_loss, sizeof(double), cudaMemcpyDeviceToHost, m->stream));
        if ((st = check_err_word(m))) return st;
        *loss = l / ((double)B * m->nb);
    }
    return RPL_OK;
}

int rpl_mlp_forward(rpl_mlp* m, const void* X, const float* E, int64_t n, float* Y) {
    if (!m || !X || !E || !Y) return mfail(RPL_ERR_ARGUMENT, "null argument");
    if (n <= 0 || n % 128) return mfail(RPL_ERR_ARGUMENT, "rows must be a positive multiple of 128");
    MLP_CUDA(cudaSetDevice(m->d.device));
    MLP_CUDA(rpl::mlp_forward(m, (const bf16*)X, m->nb, E, n, Y, m->nb, false, m->stream, nullptr));
    return check_err_word(m);
}

int rpl_gemm_bf16(const void* A, const void* B, float* C, int32_t M, int32_t N, int32_t K, void* stream) {
    return rpl_gemm_bf16_bounded(A, B, C, M, N, K, 0u, stream);
}

int rpl_gemm_bf16_bounded(const void* A, const void* B, float* C, int32_t M, int32_t N, int32_t K,
                          uint32_t wait_limit, void* stream) {
    rpl::GemmArgs g{};
    g.A = (const bf16*)A; g.lda = K; g.B = (const bf16*)B; g.ldb = K; g.M = M; g.N = N; g.K = K;
    g.epi = rpl::EPI_F32; g.out_f32 = C; g.ldo = N;
    g.wait_limit = wait_limit;
    const int bn = (N % 256 == 0 && (M / 128) * (N / 256) >= 148) ? 256 : 128;
    if (!rpl::gemm_shape_ok(g, bn)) return mfail(RPL_ERR_ARGUMENT, "GEMM shape or alignment not supported");
    unsigned int* err = nullptr;
    MLP_CUDA(cudaMalloc((void**)&err, sizeof(unsigned int)));
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(unsigned int), s);
    g.err = err;
    if (e == cudaSuccess) e = rpl::launch_gemm(g, bn, s);
    unsigned int w = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&w, err, sizeof(w), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(err);
    if (e != cudaSuccess) return mcuda(e, "rpl_gemm_bf16");
    if (w) return mfail(RPL_ERR_DEVICE, "the GEMM gave up waiting on a barrier (bounded wait ran out)");
    return RPL_OK;
}

}  // extern "C"
