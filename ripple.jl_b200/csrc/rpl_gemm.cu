// rpl_gemm.cu -- BF16 x BF16 -> FP32 GEMM on the sm_100a tensor cores (tcgen05.mma, accumulators in
// tensor memory) with the fused epilogues the learned-source MLP needs.
//
// C[M x N] = A[M x K] * B[N x K]^T, A and B row-major with K contiguous ("K-major" operands).
// One CTA of 128 threads owns a 128 x BN output tile. K advances in blocks of 64: every thread copies
// its share of the A and B blocks into shared memory with cp.async, 128-byte swizzled so the tensor core
// reads them through K-major descriptors; STAGES blocks are in flight. Thread 0 issues the four
// K = 16 MMAs of a block into the TMEM accumulator and commits them to the block's mbarrier; a stage is
// refilled only after that mbarrier reports the MMAs which read it complete. Every wait is bounded: on
// timeout the kernel sets bit 4 of the error word, drains its copies, frees its TMEM and returns.
// Requirements (checked by the host): M % 128 == 0, N % BN == 0, K % 64 == 0, 16-byte aligned rows.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "rpl_mlp.h"
#include "rpl_umma.cuh"

namespace rpl {

namespace {

constexpr int BM = 128, BK = 64, THREADS = 128;
constexpr uint32_t WAIT_LIMIT = 1u << 24;

template <int BN, int STAGES>
struct GemmSmem {
    static constexpr int A_BYTES = BM * BK * 2;
    static constexpr int B_BYTES = BN * BK * 2;
    static constexpr int STAGE = A_BYTES + B_BYTES;  // a multiple of 1024
    static constexpr int TOTAL = STAGES * STAGE + 1024 /* alignment slack */;
};

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
    const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
    return cdf + z * pdf;
}

template <int BN, int STAGES, int EPI>
__global__ void __launch_bounds__(THREADS, 1) gemm_kernel(const GemmArgs g) {
    using S = GemmSmem<BN, STAGES>;
    extern __shared__ uint8_t smem_raw[];
    __shared__ uint64_t bars[STAGES];
    __shared__ uint32_t s_tmem;
    __shared__ int s_bad;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    const int KB = g.K / BK;
    const uint32_t base = (umma::smem_u32(smem_raw) + 1023u) & ~1023u;

    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) umma::mbar_init(umma::smem_u32(&bars[s]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_bad = 0;
    }
    if (warp == 0) umma::tmem_alloc(umma::smem_u32(&s_tmem), BN);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = s_tmem;

    auto load = [&](int s, int kb) {
        const uint32_t sa = base + s * S::STAGE, sb = sa + S::A_BYTES;
        const int k0 = kb * BK;
#pragma unroll 4
        for (int q = tid; q < BM * 8; q += THREADS) {
            const int r = q >> 3, c = q & 7;
            umma::cp_async16(sa + r * 128 + ((c ^ (r & 7)) << 4), g.A + (int64_t)(m0 + r) * g.lda + k0 + c * 8);
        }
#pragma unroll 4
        for (int q = tid; q < BN * 8; q += THREADS) {
            const int r = q >> 3, c = q & 7;
            umma::cp_async16(sb + r * 128 + ((c ^ (r & 7)) << 4), g.B + (int64_t)(n0 + r) * g.ldb + k0 + c * 8);
        }
    };

    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < KB) load(s, s);
        umma::cp_async_commit();
    }
    constexpr uint32_t IDESC = umma::idesc_bf16_f32(BM, BN);
    for (int kb = 0; kb < KB; ++kb) {
        const int s = kb % STAGES;
        umma::cp_async_wait<STAGES - 2>();
        umma::fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            umma::fence_after_sync();
            const uint32_t sa = base + s * S::STAGE, sb = sa + S::A_BYTES;
#pragma unroll
            for (int k = 0; k < BK / 16; ++k)
                umma::mma_bf16(tmem, umma::kmajor_sw128_desc(sa + 32 * k), umma::kmajor_sw128_desc(sb + 32 * k), IDESC,
                               (kb > 0 || k > 0) ? 1u : 0u);
            umma::mma_commit(umma::smem_u32(&bars[s]));
            // the stage refilled below was read by the MMAs of block kb - 1
            if (kb >= 1 && kb + STAGES - 1 < KB) {
                const int j = kb - 1;
                if (!umma::mbar_wait_bounded(umma::smem_u32(&bars[j % STAGES]), (uint32_t)((j / STAGES) & 1),
                                             WAIT_LIMIT))
                    s_bad = 1;
            }
        }
        __syncthreads();
        if (s_bad) break;
        if (kb + STAGES - 1 < KB) load((kb + STAGES - 1) % STAGES, kb + STAGES - 1);
        umma::cp_async_commit();
    }
    if (tid == 0 && !s_bad && KB > 0) {
        const int j = KB - 1;
        if (!umma::mbar_wait_bounded(umma::smem_u32(&bars[j % STAGES]), (uint32_t)((j / STAGES) & 1), WAIT_LIMIT))
            s_bad = 1;
    }
    umma::cp_async_wait<0>();
    __syncthreads();
    umma::fence_after_sync();
    const bool bad = s_bad != 0;
    if (bad) {
        if (tid == 0 && g.err) atomicOr(g.err, 4u);
    } else {
        // epilogue: warp w holds rows 32w .. 32w+31 of the tile in TMEM lanes 32w .. 32w+31
        const int row = m0 + warp * 32 + lane;
        const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
        float ex[4] = {0.f, 0.f, 0.f, 0.f};
        if (EPI == EPI_BIAS_GELU && g.extra) {
#pragma unroll
            for (int e = 0; e < 4; ++e) ex[e] = g.extra[(int64_t)row * 4 + e];
        }
        for (int c0 = 0; c0 < BN; c0 += 16) {
            float v[16];
            umma::tmem_ld16(trow + c0, v);
            const int col = n0 + c0;
            if (EPI == EPI_F32) {
                float4* o = reinterpret_cast<float4*>(g.out_f32 + (int64_t)row * g.ldo + col);
#pragma unroll
                for (int i = 0; i < 4; ++i) o[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
            } else if (EPI == EPI_BIAS) {
                float4* o = reinterpret_cast<float4*>(g.out_f32 + (int64_t)row * g.ldo + col);
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    o[i] = make_float4(v[4 * i] + g.bias[col + 4 * i], v[4 * i + 1] + g.bias[col + 4 * i + 1],
                                       v[4 * i + 2] + g.bias[col + 4 * i + 2], v[4 * i + 3] + g.bias[col + 4 * i + 3]);
            } else {
                __nv_bfloat16 h[16];
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    float z = v[i];
                    if (EPI == EPI_BIAS_GELU) {
                        z += g.bias[col + i];
                        if (g.wextra) {
                            const float* we = g.wextra + (int64_t)(col + i) * 4;
                            z = fmaf(ex[0], we[0], fmaf(ex[1], we[1], fmaf(ex[2], we[2], fmaf(ex[3], we[3], z))));
                        }
                        if (g.out_f32) g.out_f32[(int64_t)row * g.ldo + col + i] = z;
                        z = gelu(z);
                    } else {  // EPI_GELU_BWD: upstream gradient times GELU'(pre-activation)
                        z *= gelu_grad(g.pre[(int64_t)row * g.ldp + col + i]);
                    }
                    h[i] = __float2bfloat16_rn(z);
                }
                if (g.out_bf16) {
                    uint4* o = reinterpret_cast<uint4*>(g.out_bf16 + (int64_t)row * g.ldh + col);
                    o[0] = *reinterpret_cast<const uint4*>(&h[0]);
                    o[1] = *reinterpret_cast<const uint4*>(&h[8]);
                }
                if (g.out_bf16_t) {
#pragma unroll
                    for (int i = 0; i < 16; ++i) g.out_bf16_t[(int64_t)(col + i) * g.ldt + row] = h[i];
                }
            }
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        umma::fence_after_sync();
        umma::tmem_dealloc(tmem, BN);
    }
}

template <int BN, int STAGES, int EPI>
cudaError_t launch_bn(const GemmArgs& g, cudaStream_t s) {
    using S = GemmSmem<BN, STAGES>;
    auto k = gemm_kernel<BN, STAGES, EPI>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, S::TOTAL);
    if (e != cudaSuccess) return e;
    dim3 grid(g.M / BM, g.N / BN);
    k<<<grid, THREADS, S::TOTAL, s>>>(g);
    return cudaGetLastError();
}

template <int EPI>
cudaError_t launch_epi(const GemmArgs& g, int bn, cudaStream_t s) {
    if (bn == 256) return launch_bn<256, 4, EPI>(g, s);
    return launch_bn<128, 4, EPI>(g, s);
}

}  // namespace

bool gemm_shape_ok(const GemmArgs& g, int bn) {
    auto al16 = [](const void* p) { return ((uintptr_t)p & 15u) == 0; };
    if (g.M <= 0 || g.N <= 0 || g.K <= 0 || g.M % BM || g.K % BK || (bn != 128 && bn != 256) || g.N % bn) return false;
    if (!g.A || !g.B || !al16(g.A) || !al16(g.B) || g.lda % 8 || g.ldb % 8 || g.lda < g.K || g.ldb < g.K) return false;
    switch (g.epi) {
        case EPI_F32:
        case EPI_BIAS:
            return g.out_f32 && al16(g.out_f32) && g.ldo % 4 == 0 && g.ldo >= g.N && (g.epi == EPI_F32 || g.bias);
        case EPI_BIAS_GELU:
            return g.bias && (g.out_bf16 || g.out_bf16_t) && (!g.out_bf16 || (al16(g.out_bf16) && g.ldh % 8 == 0)) &&
                   (!g.out_f32 || g.ldo >= g.N) && (!g.out_bf16_t || g.ldt >= g.M);
        case EPI_GELU_BWD:
            return g.pre && g.ldp >= g.N && (g.out_bf16 || g.out_bf16_t) &&
                   (!g.out_bf16 || (al16(g.out_bf16) && g.ldh % 8 == 0)) && (!g.out_bf16_t || g.ldt >= g.M);
        default:
            return false;
    }
}

cudaError_t launch_gemm(const GemmArgs& g, int bn, cudaStream_t s) {
    switch (g.epi) {
        case EPI_F32: return launch_epi<EPI_F32>(g, bn, s);
        case EPI_BIAS: return launch_epi<EPI_BIAS>(g, bn, s);
        case EPI_BIAS_GELU: return launch_epi<EPI_BIAS_GELU>(g, bn, s);
        default: return launch_epi<EPI_GELU_BWD>(g, bn, s);
    }
}

}  // namespace rpl
