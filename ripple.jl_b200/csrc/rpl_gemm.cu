// rpl_gemm.cu -- BF16 x BF16 -> FP32 GEMM on the sm_100a tensor cores (tcgen05.mma, accumulators in
// tensor memory) with the fused epilogues the learned-source MLP needs.
//
// C[M x N] = A[M x K] * B[N x K]^T, A and B row-major with K contiguous ("K-major" operands).
// A persistent, warp-specialised kernel: one CTA per SM walks the 128 x BN output tiles (tile t and
// t + gridDim.x, ...). Its warps split the work:
//   warp 0 (producer, one thread): TMA-loads (no multicast) 64-wide K blocks of A and B into a
//     STAGES-deep ring of shared-memory stages, 128-byte swizzled by the tensor maps so the tensor core
//     reads them through K-major descriptors; each stage's `full` barrier completes on the bytes landed;
//   warp 1 (MMA, one thread): waits `full`, issues the block's four K = 16 tcgen05.mma into one of two
//     TMEM accumulators (double buffered across tiles), commits the stage's `empty` barrier (the producer
//     refills it) and, after a tile's last block, the accumulator's `acc_full` barrier;
//   warps 2-17 (epilogue, four per TMEM lane quadrant warp % 4, each taking a quarter of the columns):
//     wait `acc_full`, read their lanes with tcgen05.ld, apply the fused epilogue, store, and arrive on
//     `acc_empty` so the MMA warp may reuse that accumulator -- the epilogue of one tile overlaps the
//     MMAs of the next.
// Every wait is bounded (GemmArgs::wait_limit polls, default 2^24) and checks a shared abort flag: a wait
// that gives up sets bit 4 of the error word and the flag, every role then leaves its loop; the producer
// waits (bounded) for the TMA loads it issued to land and the MMA thread for its issued MMAs to finish,
// so nothing writes shared or tensor memory after the CTA frees them; then TMEM is freed and the kernel
// returns. Requirements (checked by the host): M % 128 == 0, N % BN == 0, K % 64 == 0, 16-byte
// aligned rows.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <mutex>

#include "rpl_mlp.h"
#include "rpl_umma.cuh"

namespace rpl {

namespace {

constexpr int BM = 128, BK = 64, STAGES = 4;
constexpr int MMA_WARP = 1;
constexpr int EPI_WARP0 = 2, EPI_WARPS = 16;   // warps 2-17
constexpr int EPILOGUE = EPI_WARPS * 32;
constexpr int THREADS = (EPI_WARP0 + EPI_WARPS) * 32;
constexpr uint32_t WAIT_LIMIT = 1u << 24;   // default polls per barrier wait
constexpr uint32_t DRAIN_LIMIT = 1u << 24;  // polls per wait for work in flight after an abort

template <int BN>
struct GemmSmem {
    static constexpr int A_BYTES = BM * BK * 2;
    static constexpr int B_BYTES = BN * BK * 2;
    static constexpr int STAGE = A_BYTES + B_BYTES;  // a multiple of 1024
    static constexpr int TOTAL = STAGES * STAGE + 1024 /* alignment slack */;
};

// The network's activation: GELU in its tanh form, 0.5 z (1 + tanh(c (z + a z^3))), c = sqrt(2/pi),
// a = 0.044715, with the hardware tanh (tanh.approx.f32, relative error ~5e-4, below BF16 rounding).
__device__ __forceinline__ float tanh_fast(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
constexpr float GELU_C = 0.7978845608028654f, GELU_A = 0.044715f;
__device__ __forceinline__ float gelu(float z) {
    const float t = tanh_fast(GELU_C * fmaf(GELU_A * z, z * z, z));
    return 0.5f * z * (1.0f + t);
}
__device__ __forceinline__ float gelu_grad(float z) {
    const float z2 = z * z;
    const float t = tanh_fast(GELU_C * fmaf(GELU_A * z, z2, z));
    return fmaf(0.5f * z * fmaf(-t, t, 1.0f), GELU_C * fmaf(3.0f * GELU_A, z2, 1.0f), 0.5f * (1.0f + t));
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Bounded wait (`limit` polls) that also gives up once another role has aborted.
__device__ __forceinline__ bool wait_phase(uint32_t bar, uint32_t parity, volatile int* abort_flag, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i) {
        if (umma::mbar_try_wait(bar, parity)) return true;
        if (*abort_flag) return false;
    }
    *abort_flag = 1;
    return false;
}

// Fused epilogue of COLS accumulator columns for the thread holding row `row`: reads its TMEM lane
// starting at TMEM address `trow`, writes output columns n0 .. n0 + COLS - 1.
template <int COLS, int EPI>
__device__ __forceinline__ void epilogue_cols(const GemmArgs& g, uint32_t trow, int row, int n0) {
    float ex[4] = {0.f, 0.f, 0.f, 0.f};
    if (EPI == EPI_BIAS_GELU && g.extra) {
#pragma unroll
        for (int e = 0; e < 4; ++e) ex[e] = g.extra[(int64_t)row * 4 + e];
    }
    for (int c0 = 0; c0 < COLS; c0 += 16) {
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
            for (int i = 0; i < 16; ++i) v[i] += g.bias[col + i];
            if (g.clamp_lo) {
#pragma unroll
                for (int i = 0; i < 16; ++i) v[i] = fminf(fmaxf(v[i], g.clamp_lo[col + i]), g.clamp_hi[col + i]);
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) o[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
        } else {
            __nv_bfloat16 h[16];
            float u[16];
            if (EPI == EPI_BIAS_GELU) {
                const float4* bp = reinterpret_cast<const float4*>(g.bias + col);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const float4 bb = __ldg(bp + i);
                    u[4 * i] = bb.x; u[4 * i + 1] = bb.y; u[4 * i + 2] = bb.z; u[4 * i + 3] = bb.w;
                }
            } else {
                const float4* pp = reinterpret_cast<const float4*>(g.pre + (int64_t)row * g.ldp + col);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const float4 q = pp[i];
                    u[4 * i] = q.x; u[4 * i + 1] = q.y; u[4 * i + 2] = q.z; u[4 * i + 3] = q.w;
                }
            }
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                float z = v[i];
                if (EPI == EPI_BIAS_GELU) {
                    z += u[i];
                    if (g.wextra) {
                        const float4 we = __ldg(reinterpret_cast<const float4*>(g.wextra) + col + i);
                        z = fmaf(ex[0], we.x, fmaf(ex[1], we.y, fmaf(ex[2], we.z, fmaf(ex[3], we.w, z))));
                    }
                    if (g.out_f32) g.out_f32[(int64_t)row * g.ldo + col + i] = z;
                    z = gelu(z);
                } else {  // EPI_GELU_BWD: upstream gradient times GELU'(pre-activation)
                    z *= gelu_grad(u[i]);
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

template <int BN, int EPI>
__global__ void __launch_bounds__(THREADS, 1)
    gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, const GemmArgs g) {
    using S = GemmSmem<BN>;
    extern __shared__ uint8_t smem_raw[];
    __shared__ uint64_t full_bar[STAGES], empty_bar[STAGES], acc_full[2], acc_empty[2], drain_bar;
    __shared__ uint32_t s_tmem;
    __shared__ int s_abort;
    volatile int* abort_flag = &s_abort;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tiles_n = g.N / BN, tiles = (g.M / BM) * tiles_n;
    const int KB = g.K / BK;
    const uint32_t base = (umma::smem_u32(smem_raw) + 1023u) & ~1023u;
    const uint32_t limit = g.wait_limit ? g.wait_limit : WAIT_LIMIT;
    int64_t last_use[STAGES];  // producer thread: per stage, the fill count of its last issued load (-1: none)
#pragma unroll
    for (int q = 0; q < STAGES; ++q) last_use[q] = -1;

    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            umma::mbar_init(umma::smem_u32(&full_bar[s]), 1);
            umma::mbar_init(umma::smem_u32(&empty_bar[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            umma::mbar_init(umma::smem_u32(&acc_full[b]), 1);
            umma::mbar_init(umma::smem_u32(&acc_empty[b]), EPILOGUE);
        }
        umma::mbar_init(umma::smem_u32(&drain_bar), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    if (warp == MMA_WARP) umma::tmem_alloc(umma::smem_u32(&s_tmem), 2 * BN);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = s_tmem;

    if (warp == 0) {
        // ---- producer (one thread): TMA loads ----
        if (lane == 0) {
            int64_t gcount = 0;  // K blocks issued by this CTA so far
            for (int t = blockIdx.x; t < tiles && !*abort_flag; t += gridDim.x) {
                const int m0 = (t / tiles_n) * BM, n0 = (t % tiles_n) * BN;
                for (int kb = 0; kb < KB; ++kb, ++gcount) {
                    const int s = (int)(gcount % STAGES);
                    const int64_t use = gcount / STAGES;
                    if (use > 0 &&
                        !wait_phase(umma::smem_u32(&empty_bar[s]), (uint32_t)((use - 1) & 1), abort_flag, limit))
                        break;
                    const uint32_t sa = base + s * S::STAGE, sb = sa + S::A_BYTES;
                    const uint32_t bar = umma::smem_u32(&full_bar[s]);
                    umma::mbar_arrive_expect_tx(bar, (uint32_t)S::STAGE);
                    umma::tma_load_2d(sa, &tmA, kb * BK, m0, bar);
                    umma::tma_load_2d(sb, &tmB, kb * BK, n0, bar);
#pragma unroll
                    for (int q = 0; q < STAGES; ++q)
                        if (q == s) last_use[q] = use;
                }
            }
        }
        __syncwarp();
    } else if (warp == MMA_WARP) {
        // ---- MMA issue (one thread) ----
        if (lane == 0) {
            constexpr uint32_t IDESC = umma::idesc_bf16_f32(BM, BN);
            int64_t gcount = 0;
            int local = 0;
            for (int t = blockIdx.x; t < tiles && !*abort_flag; t += gridDim.x, ++local) {
                const int b = local & 1, ub = local >> 1;
                if (ub > 0 && !wait_phase(umma::smem_u32(&acc_empty[b]), (uint32_t)((ub - 1) & 1), abort_flag, limit)) break;
                umma::fence_after_sync();
                const uint32_t acc = tmem + (uint32_t)(b * BN);
                bool ok = true;
                for (int kb = 0; kb < KB; ++kb, ++gcount) {
                    const int s = (int)(gcount % STAGES);
                    if (!wait_phase(umma::smem_u32(&full_bar[s]), (uint32_t)((gcount / STAGES) & 1), abort_flag, limit)) {
                        ok = false;
                        break;
                    }
                    umma::fence_after_sync();
                    const uint32_t sa = base + s * S::STAGE, sb = sa + S::A_BYTES;
#pragma unroll
                    for (int k = 0; k < BK / 16; ++k)
                        umma::mma_bf16(acc, umma::kmajor_sw128_desc(sa + 32 * k), umma::kmajor_sw128_desc(sb + 32 * k),
                                       IDESC, (kb > 0 || k > 0) ? 1u : 0u);
                    umma::mma_commit(umma::smem_u32(&empty_bar[s]));
                }
                if (!ok) break;
                umma::mma_commit(umma::smem_u32(&acc_full[b]));
            }
        }
        __syncwarp();
    } else {
        // ---- epilogue (warps 2-17: TMEM lane quadrant warp % 4, column quarter (warp - 2) / 4) ----
        const int quad = warp & 3, part = (warp - EPI_WARP0) >> 2;
        int local = 0;
        for (int t = blockIdx.x; t < tiles && !*abort_flag; t += gridDim.x, ++local) {
            const int b = local & 1;
            if (!wait_phase(umma::smem_u32(&acc_full[b]), (uint32_t)((local >> 1) & 1), abort_flag, limit)) break;
            umma::fence_after_sync();
            const int m0 = (t / tiles_n) * BM, n0 = (t % tiles_n) * BN;
            const uint32_t trow = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(b * BN + part * (BN / 4));
            epilogue_cols<BN / 4, EPI>(g, trow, m0 + quad * 32 + lane, n0 + part * (BN / 4));
            umma::fence_before_sync();
            mbar_arrive(umma::smem_u32(&acc_empty[b]));
        }
    }
    umma::fence_before_sync();
    __syncthreads();  // every role has left its loop; the abort flag is final
    if (*abort_flag) {
        if (warp == 0 && lane == 0) {
            // every TMA load still in flight lands before the CTA releases its shared memory
#pragma unroll
            for (int q = 0; q < STAGES; ++q)
                if (last_use[q] >= 0)
                    umma::mbar_wait_bounded(umma::smem_u32(&full_bar[q]), (uint32_t)(last_use[q] & 1), DRAIN_LIMIT);
        }
        if (warp == MMA_WARP && lane == 0) {
            // every MMA issued so far (and its barrier arrivals) completes before TMEM is freed
            umma::mma_commit(umma::smem_u32(&drain_bar));
            umma::mbar_wait_bounded(umma::smem_u32(&drain_bar), 0u, DRAIN_LIMIT);
        }
        if (tid == 0 && g.err) atomicOr(g.err, 4u);
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == MMA_WARP) {
        umma::fence_after_sync();
        umma::tmem_dealloc(tmem, 2 * BN);
    }
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// The driver's tensor-map encoder, looked up once through the runtime (no link against libcuda).
EncodeTiled encoder() {
    static std::once_flag once;
    static EncodeTiled fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    });
    return fn;
}

// Tensor map of a row-major BF16 matrix (rows x K, row stride ld elements): boxes of 64 K values x
// box_rows rows, 128-byte swizzle (the layout the K-major UMMA descriptors read).
bool encode(CUtensorMap* m, const __nv_bfloat16* base, int64_t rows, int64_t K, int64_t ld, int box_rows) {
    EncodeTiled fn = encoder();
    if (!fn) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int BN, int EPI>
cudaError_t launch_bn(const GemmArgs& g, cudaStream_t s) {
    using S = GemmSmem<BN>;
    auto k = gemm_kernel<BN, EPI>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, S::TOTAL);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    alignas(64) CUtensorMap ta, tb;
    if (!encode(&ta, g.A, g.M, g.K, g.lda, BM) || !encode(&tb, g.B, g.N, g.K, g.ldb, BN))
        return cudaErrorInvalidValue;
    const int tiles = (g.M / BM) * (g.N / BN);
    k<<<tiles < sms ? tiles : sms, THREADS, S::TOTAL, s>>>(ta, tb, g);
    return cudaGetLastError();
}

template <int EPI>
cudaError_t launch_epi(const GemmArgs& g, int bn, cudaStream_t s) {
    if (bn == 256) return launch_bn<256, EPI>(g, s);
    return launch_bn<128, EPI>(g, s);
}

}  // namespace

bool gemm_shape_ok(const GemmArgs& g, int bn) {
    auto al16 = [](const void* p) { return ((uintptr_t)p & 15u) == 0; };
    if (g.M <= 0 || g.N <= 0 || g.K <= 0 || g.M % BM || g.K % BK || (bn != 128 && bn != 256) || g.N % bn) return false;
    if (!g.A || !g.B || !al16(g.A) || !al16(g.B) || g.lda % 8 || g.ldb % 8 || g.lda < g.K || g.ldb < g.K) return false;
    switch (g.epi) {
        case EPI_F32:
        case EPI_BIAS:
            return g.out_f32 && al16(g.out_f32) && g.ldo % 4 == 0 && g.ldo >= g.N && (g.epi == EPI_F32 || g.bias) &&
                   (!g.clamp_lo) == (!g.clamp_hi);
        case EPI_BIAS_GELU:
            return g.bias && al16(g.bias) && (!g.wextra || al16(g.wextra)) && (g.out_bf16 || g.out_bf16_t) && (!g.out_bf16 || (al16(g.out_bf16) && g.ldh % 8 == 0)) &&
                   (!g.out_f32 || g.ldo >= g.N) && (!g.out_bf16_t || g.ldt >= g.M);
        case EPI_GELU_BWD:
            return g.pre && al16(g.pre) && g.ldp % 4 == 0 && g.ldp >= g.N && (g.out_bf16 || g.out_bf16_t) &&
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
