// The learned stage's dense layers on the 5th-generation tensor cores
// (tcgen05): D[m][n] = sum_k A(m,k) B(n,k), BF16 operands staged in shared
// memory, FP32 accumulation in tensor memory (TMEM).
//
// One CTA of 4 warps per 128 x 64 output tile (and per chunk of the
// reduction for the weight gradient).  Per 64-wide slice of the reduction the
// threads load A (128 x 64) and B (64 x 64) from FP32 global memory, round
// them to BF16 and store them in the canonical K-major layout without
// swizzle (8 x 8 core matrices of 128 contiguous bytes; the two core
// matrices of one 16-wide MMA step 128 bytes apart, row groups 1024 bytes
// apart); one thread issues four tcgen05.mma (M = 128, N = 64, K = 16) into
// the TMEM accumulator and commits them to the stage's mbarrier.  Two stages:
// the threads fill one while the tensor core reads the other, and wait on a
// stage's mbarrier before they refill it.  The epilogue reads the
// accumulator with tcgen05.ld (warp w reads TMEM lanes 32w..32w+31, one
// output row per thread) and writes Z (+ bias, ReLU), dX or the weight-
// gradient partials.  Every output element is one accumulator's sum over the
// reduction in a fixed order: results are deterministic.
//
// The mbarrier waits are bounded (2 s on %globaltimer): on expiry the CTA
// sets err[0], leaves the loop, frees its TMEM and returns.
#include <cuda_bf16.h>

#include "ofea_internal.cuh"
#include "tc_gemm.cuh"

namespace ofea {
namespace {

constexpr int kTM = 128, kTN = 64, kTK = 64, kTcThreads = 128;
constexpr uint32_t kTmemCols = 64;
constexpr size_t kTcSmem = 2 * (kTM + kTN) * kTK * sizeof(__nv_bfloat16);  // 48 KB
// kind::f16 instruction descriptor: D F32 (bits 4-5 = 1), A and B BF16 (bits
// 7-9 = 1, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at bit 17,
// M >> 4 at bit 24.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kTN >> 3) << 17) |
                            ((uint32_t)(kTM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Element offset of (row, k) in a K-major tile of kTK columns.
__device__ __forceinline__ int kmaj(int row, int k) {
    return ((row >> 3) * (kTK / 8) + (k >> 3)) * 64 + (row & 7) * 8 + (k & 7);
}

// Shared-memory matrix descriptor: start address, leading (K-direction core
// matrix) and stride (8-row group) byte offsets, version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for the mbarrier phase `parity` to complete, at most limit_ns.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, unsigned long long limit_ns) {
    const unsigned long long t0 = now_ns();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (now_ns() - t0 > limit_ns) return false;
    }
}

// Stage rows [r0, r0 + ROWS) x reduction [k0, k0 + kTK) of an operand as
// BF16 into the K-major tile.  Entries outside [0, R) x [k0, kend) are zero.
// Every load of the slice is issued before the first conversion (the
// thread's values are in registers), so the loads' latencies overlap.
template <int ROWS>
__device__ __forceinline__ void stage(__nv_bfloat16 *tile, const TcOperand &op, int r0, int R, long k0,
                                      long kend) {
    constexpr int kV = ROWS * kTK / 4 / kTcThreads;  // float4 groups per thread
    constexpr int kS = ROWS * kTK / kTcThreads;      // scalars per thread
    if (op.ks == 1 && (op.ms & 3) == 0 && (reinterpret_cast<uintptr_t>(op.p) & 15) == 0) {
        // contiguous along the reduction, rows 16-byte aligned: four k per
        // thread as one 16-byte load, stored as four adjacent BF16 of a core row
        float4 v[kV];
#pragma unroll
        for (int q = 0; q < kV; ++q) {
            const int idx = threadIdx.x + q * kTcThreads;
            const int rr = idx / (kTK / 4), kk = 4 * (idx % (kTK / 4));
            const long r = r0 + rr, k = k0 + kk;
            v[q] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (r < R) {
                const float *src = op.p + r * op.ms + k;
                if (k + 3 < kend) {
                    v[q] = *reinterpret_cast<const float4 *>(src);
                } else {
                    if (k < kend) v[q].x = src[0];
                    if (k + 1 < kend) v[q].y = src[1];
                    if (k + 2 < kend) v[q].z = src[2];
                }
            }
        }
#pragma unroll
        for (int q = 0; q < kV; ++q) {
            const int idx = threadIdx.x + q * kTcThreads;
            const int rr = idx / (kTK / 4), kk = 4 * (idx % (kTK / 4));
            __nv_bfloat162 lo = __floats2bfloat162_rn(v[q].x, v[q].y), hi = __floats2bfloat162_rn(v[q].z, v[q].w);
            uint2 packed;
            packed.x = *reinterpret_cast<uint32_t *>(&lo);
            packed.y = *reinterpret_cast<uint32_t *>(&hi);
            *reinterpret_cast<uint2 *>(tile + kmaj(rr, kk)) = packed;
        }
    } else {
        // scalar loads, 32 per thread in flight; consecutive threads take
        // consecutive addresses
        const bool along_k = op.ks == 1;
        constexpr int kH = kS < 32 ? kS : 32;
#pragma unroll
        for (int h = 0; h < kS; h += kH) {
            float v[kH];
#pragma unroll
            for (int q = 0; q < kH; ++q) {
                const int idx = threadIdx.x + (h + q) * kTcThreads;
                const int rr = along_k ? idx / kTK : idx % ROWS, kk = along_k ? idx % kTK : idx / ROWS;
                const long r = r0 + rr, k = k0 + kk;
                v[q] = (r < R && k < kend) ? op.p[r * op.ms + k * op.ks] : 0.f;
            }
#pragma unroll
            for (int q = 0; q < kH; ++q) {
                const int idx = threadIdx.x + (h + q) * kTcThreads;
                const int rr = along_k ? idx / kTK : idx % ROWS, kk = along_k ? idx % kTK : idx / ROWS;
                tile[kmaj(rr, kk)] = __float2bfloat16_rn(v[q]);
            }
        }
    }
}

__global__ void __launch_bounds__(kTcThreads) k_tc_gemm(int M, int N, long Kred, long kchunk, TcOperand A,
                                                        TcOperand B, TcEpilogue epi, int *err) {
    // two stages of A (128 x 64) and B (64 x 64) BF16 tiles, 1024-byte aligned
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    __nv_bfloat16 *const stages = reinterpret_cast<__nv_bfloat16 *>(tc_smem);
    constexpr int kStage = (kTM + kTN) * kTK;  // elements per stage: A then B
    __shared__ __align__(8) unsigned long long mbar[2];
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * kTM, n0 = blockIdx.y * kTN;
    const long kb = (long)blockIdx.z * kchunk, ke = min(Kred, kb + kchunk);
    const uint32_t bar0 = smem_u32(&mbar[0]);  // stage b's mbarrier at bar0 + 8 b
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar0), "r"(1));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar0 + 8u), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    unsigned parity = 0u, pending = 0u;  // bit b: stage b's next phase, stage b has MMAs in flight
    bool ok = true, any = false;
    // slice i goes to stage i % 2: its staging overlaps the MMAs of slice
    // i - 1; before a stage is refilled, the MMAs that read it (slice i - 2)
    // must be complete
    int i = 0;
    for (long k0 = kb; k0 < ke; k0 += kTK, ++i) {
        const int b = i & 1;
        if (pending >> b & 1u) {
            const bool mine = mbar_wait(bar0 + 8u * b, parity >> b & 1u, 2000000000ull);
            parity ^= 1u << b;
            pending &= ~(1u << b);
            ok = __syncthreads_and(mine) != 0;
            if (!ok) break;
        }
        __nv_bfloat16 *sA = stages + b * kStage, *sB = sA + kTM * kTK;
        stage<kTM>(sA, A, m0, M, k0, ke);
        stage<kTN>(sB, B, n0, N, k0, ke);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the tiles, to the tensor core's proxy
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
#pragma unroll
            for (int j = 0; j < kTK / 16; ++j) {
                const uint64_t da = smem_desc(a0 + 256u * j, 128u, 1024u);
                const uint64_t db = smem_desc(b0 + 256u * j, 128u, 1024u);
                const uint32_t acc = (any || j > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                    ::"r"(tmem), "l"(da), "l"(db), "r"(kIdesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(bar0 + 8u * b) : "memory");
        }
        pending |= 1u << b;
        any = true;
    }
    // the MMAs still in flight
    for (int b = 0; b < 2 && ok; ++b)
        if (pending >> b & 1u) {
            const bool mine = mbar_wait(bar0 + 8u * b, parity >> b & 1u, 2000000000ull);
            ok = __syncthreads_and(mine) != 0;
        }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!ok) {
        if (tid == 0) atomicExch(err, 1);
    } else {
        const int m = m0 + 32 * warp + lane;
#pragma unroll
        for (int c0 = 0; c0 < kTN; c0 += 16) {
            uint32_t v[16];
            if (any) {
                const uint32_t addr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0;
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                    "%12, %13, %14, %15}, [%16];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                      "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                      "=r"(v[14]), "=r"(v[15])
                    : "r"(addr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            } else {
#pragma unroll
                for (int i = 0; i < 16; ++i) v[i] = 0u;  // an empty reduction chunk
            }
            if (m < M) {
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int n = n0 + c0 + i;
                    if (n >= N) break;
                    const float x = __uint_as_float(v[i]);
                    if (epi.mode == kTcForward) {
                        const float z = x + epi.bias[n];
                        epi.out[(long)m * N + n] = z;
                        if (epi.out2) epi.out2[(long)m * N + n] = z > 0.f ? z : 0.f;
                    } else if (epi.mode == kTcRowMajor) {
                        epi.out[(long)m * N + n] = x;
                    } else {  // kTcTransposedPartial: out[z][n][m]
                        epi.out[(long)blockIdx.z * epi.zstride + (long)n * M + m] = x;
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

}  // namespace

void tc_gemm(cudaStream_t s, int M, int N, long Kred, long kchunk, const TcOperand &A, const TcOperand &B,
             const TcEpilogue &epi, int *err) {
    if (M <= 0 || N <= 0) return;
    if (kchunk <= 0) kchunk = Kred;
    const long nz = Kred > 0 ? (Kred + kchunk - 1) / kchunk : 1;
    dim3 grid((M + kTM - 1) / kTM, (N + kTN - 1) / kTN, (unsigned)nz);
    // two 24 KB stages: at most 4 CTAs per SM, so their TMEM (64 columns
    // each) always fits the SM's 512 columns and no allocation has to wait
    // for another CTA to finish
    OFEA_CUDA(cudaFuncSetAttribute(k_tc_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem));
    k_tc_gemm<<<grid, kTcThreads, kTcSmem, s>>>(M, N, Kred, kchunk, A, B, epi, err);
    OFEA_CHECK_LAUNCH();
}

}  // namespace ofea
