// Batched reanalysis: many design variants (each an assembled context on one
// GPU) times up to kMaxBatchRhs load cases each, solved by ONE persistent
// cooperative kernel launched from a CUDA graph.  The reference solves such
// batches variant by variant with a kept SuperLU factor and dgstrs per load
// case (src/solver/solver_superlu.cpp:31-94, the CA reanalysis of
// src/ca_analysis.cpp:148-248).
//
// Layout in HBM: the variants' DOF are concatenated (variant v starts at
// dof0[v]) and every vector is load-case interleaved, x[(dof0 + d) * NP + j]
// (NP = the NR load cases padded to a power of two >= 4): the load cases of
// one DOF are one contiguous run.  Matrices stay where their contexts keep
// them (BSELL-32, FP64 and BF16 copies); a table of per-variant
// descriptors points at them.
//
// Algorithm per (variant, load case): the MIXED method of solve.cu, FP64
// flexible CG with the FP32 two-level V(1,1) preconditioner of precond.cu, or
// PCG64 (FP64 CG, block Jacobi).  The kernel runs every variant in lock step
// through phases separated by grid barriers.  In the matrix phases a CTA owns
// one slice (32 block rows) of some variant at a time: it stages the slice's
// BSELL slots in shared memory (cp.async, double-buffered), and its
// threads take (block row, load case) pairs, JW lanes per row, so each matrix
// value is read from HBM once for all load cases and every gather of x is one
// contiguous run of load cases.  The restriction takes one aggregate per
// CTA; other phases take (coarse row) or (variant, load case) items per warp.
// The outer SpMM multiplies the preconditioned residual z, not p: q = K z +
// beta q_old equals K p (p = z + beta p_old), and gathering z (FP32 for
// MIXED) instead of p_old and z cuts the gathered bytes by 3x (MIXED) or 2x
// (PCG64).  Any drift of q from K p is caught by the true FP64 residual that
// the host checks after the kernel.
// Per-(variant, load case) scalars come from per-slice partial sums reduced
// in a fixed order: results are bitwise reproducible.  Converged load cases
// stop updating; the kernel ends when none is left or at max_iter.
//
// Every wait at a grid barrier is bounded (time limit on %globaltimer): on
// expiry the kernel records an error and every CTA returns.
#include <cuda/atomic>
#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <type_traits>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <type_traits>
#include <vector>

#include "precond.cuh"
#include "sell.cuh"
#include "solver_common.cuh"

namespace ofea {

constexpr int kMaxBatchRhs = 32;

// Per-variant descriptor (device copy).
struct BVar {
    int nfree, nslice, slice0, na, m, agg0, crow0, n;
    long dof0;  // first DOF of the variant in the batch (its vectors start at dof0 * NR)
    long c0;    // first coarse entry of the variant (times NR)
    const int *sl_ptr, *scols;
    const double *sv64, *Dinv;
    const __nv_bfloat16 *sv16;
    const float *Dinv32;
    const int *agg_of, *agg_ptr, *agg_nodes, *node_of_free;
    const double *xyz, *centroid;
    const float *Einv32;
    double inv_scale;
    float wsm, pad2;
};

struct GridSync {
    unsigned count, gen;
    int err, pad;
};

struct BArgs {
    int V, NR, nslices, naggs, ncrows, max_iter, extra_arrivals;
    unsigned long long limit_ns;
    double rtol;
    const BVar *var;
    const int *slice_var, *agg_var, *crow_var;
    const double *f;
    double *u, *r, *p0, *p1, *q, *z64;
    float *b32, *x32, *t32, *zA, *zB, *cvec, *evec;
    double *pa, *pb;                                    // partials [slice][NR]
    double *ff, *tol2, *rz, *alpha, *beta;              // [V * NR]
    int *live, *iters, *status, *live_cnt;              // [V * NR], live_cnt[3]
    GridSync *gs;
    unsigned long long *trace;  // NULL, or %globaltimer at the start and after each grid barrier (CTA 0)
    int trace_cap;
};

namespace {

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid barrier for a cooperative launch.  Returns false when the batch has
// failed (a wait ran out here or elsewhere): the caller returns.
__device__ bool grid_barrier(GridSync *gs, unsigned nblocks, unsigned long long limit_ns) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> gen(gs->gen), cnt(gs->count);
        cuda::atomic_ref<int, cuda::thread_scope_device> err(gs->err);
        const unsigned g = gen.load(cuda::memory_order_acquire);
        __threadfence();
        const unsigned arrived = cnt.fetch_add(1u, cuda::memory_order_acq_rel) + 1u;
        if (arrived == nblocks) {
            cnt.store(0u, cuda::memory_order_relaxed);
            gen.fetch_add(1u, cuda::memory_order_release);
        } else {
            const unsigned long long t0 = global_ns();
            while (gen.load(cuda::memory_order_acquire) == g) {
                if (err.load(cuda::memory_order_relaxed) != 0) break;
                if (global_ns() - t0 > limit_ns) {
                    err.store(1, cuda::memory_order_relaxed);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        s_ok = err.load(cuda::memory_order_relaxed) == 0;
    }
    __syncthreads();
    return s_ok != 0;
}

// Entry (node i, component c, load case j) of a variant in a batch vector
// whose load-case stride is NP (NR rounded up; padding entries stay zero).
template <int NP>
__device__ __forceinline__ long vidx(const BVar &B, long i, int c, int j) {
    return (B.dof0 + 3 * i + c) * NP + j;
}

// RL consecutive load cases of one DOF as one vector access (the offset is
// a multiple of RL: aligned).
template <class V, int RL>
__device__ __forceinline__ void ldv(const V *p, V (&o)[RL]) {
    if constexpr (sizeof(V) * RL == 32) {
        using T = typename std::conditional<sizeof(V) == 8, double2, float4>::type;
        const T a = reinterpret_cast<const T *>(p)[0], b = reinterpret_cast<const T *>(p)[1];
        std::memcpy(&o[0], &a, 16);
        std::memcpy(&o[RL / 2], &b, 16);
    } else if constexpr (sizeof(V) * RL == 16) {
        using T = typename std::conditional<sizeof(V) == 8, double2, float4>::type;
        const T a = *reinterpret_cast<const T *>(p);
        std::memcpy(&o[0], &a, 16);
    } else if constexpr (sizeof(V) * RL == 8 && sizeof(V) == 4) {
        const float2 a = *reinterpret_cast<const float2 *>(p);
        o[0] = a.x;
        o[1] = a.y;
    } else {
#pragma unroll
        for (int q = 0; q < RL; ++q) o[q] = p[q];
    }
}
template <class V, int RL>
__device__ __forceinline__ void stv(V *p, const V (&o)[RL]) {
    if constexpr (sizeof(V) * RL == 32) {
        using T = typename std::conditional<sizeof(V) == 8, double2, float4>::type;
        T a, b;
        std::memcpy(&a, &o[0], 16);
        std::memcpy(&b, &o[RL / 2], 16);
        reinterpret_cast<T *>(p)[0] = a;
        reinterpret_cast<T *>(p)[1] = b;
    } else if constexpr (sizeof(V) * RL == 16) {
        using T = typename std::conditional<sizeof(V) == 8, double2, float4>::type;
        T a;
        std::memcpy(&a, &o[0], 16);
        *reinterpret_cast<T *>(p) = a;
    } else if constexpr (sizeof(V) * RL == 8 && sizeof(V) == 4) {
        *reinterpret_cast<float2 *>(p) = make_float2(o[0], o[1]);
    } else {
#pragma unroll
        for (int q = 0; q < RL; ++q) p[q] = o[q];
    }
}

// Thread roles in the CTA that owns one slice: LW = NP / RL lanes per block
// row, each carrying RL consecutive load cases; 32 / LW rows per warp.
template <int NP, int RL>
struct Lanes {
    static constexpr int kLW = NP / RL;
    static constexpr int kRowsPerWarp = 32 / kLW;
    static constexpr int kWarps = kSlice / kRowsPerWarp;
    __device__ static int row() { return (threadIdx.x >> 5) * kRowsPerWarp + (threadIdx.x & 31) / kLW; }
    __device__ static int j0() { return (threadIdx.x & (kLW - 1)) * RL; }
};

// Shared-memory stage of a slice's BSELL slots: two buffers of kKC slots
// (values in FP64 or BF16, then columns), filled with cp.async while the
// other buffer is consumed.
constexpr int kKC = 8;
struct __align__(128) Stage {
    double v[2][kKC * 9 * kSlice];  // BF16 values use the first quarter of each buffer
    int col[2][kKC * kSlice];
    double red[32][32];             // [warp][load case] partial sums
};
static_assert(sizeof(Stage::v) >= 6 * 32 * 32 * sizeof(float), "the restriction's per-warp sums fit in the stage");

// Bulk prefetch of [p, p + bytes) from HBM into L2 (no data returned, no
// completion to wait for).  p and bytes are multiples of 16 (the BSELL slot
// blocks and the slices' vector runs are); issued in pieces of at most 32 KB.
__device__ __forceinline__ void l2_prefetch(const void *p, long bytes) {
    const size_t g = __cvta_generic_to_global(p);
    for (long o = 0; o < bytes; o += 32768) {
        const unsigned nb = (unsigned)min(32768L, bytes - o);
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(g + o), "r"(nb) : "memory");
    }
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Start copying slots [k0, k0 + kc) of the slice at S into buffer b (16-byte
// pieces: every chunk is a multiple of 16 bytes at a 16-byte-aligned offset).
template <class ST>
__device__ __forceinline__ void stage_chunk(Stage &st, int b, long S, int k0, int kc, const int *__restrict__ scols,
                                            const ST *__restrict__ svals) {
    const char *gv = reinterpret_cast<const char *>(svals + (S + k0) * 9L * kSlice);
    char *sv = reinterpret_cast<char *>(st.v[b]);
    const int nv = kc * 9 * kSlice * (int)sizeof(ST) / 16;
    for (int i = threadIdx.x; i < nv; i += blockDim.x) cp_async16(sv + 16 * i, gv + 16 * i);
    const char *gc = reinterpret_cast<const char *>(scols + (S + k0) * (long)kSlice);
    char *sc = reinterpret_cast<char *>(st.col[b]);
    const int nc = kc * kSlice * 4 / 16;
    for (int i = threadIdx.x; i < nc; i += blockDim.x) cp_async16(sc + 16 * i, gc + 16 * i);
    cp_async_commit();
}

// A staged matrix value in the arithmetic type V.
template <class V, class ST>
__device__ __forceinline__ V staged_val(const ST &a) {
    if constexpr (std::is_same<ST, __nv_bfloat16>::value) return (V)__bfloat162float(a);
    else return (V)a;
}

// y[c][q] = (K x)_(row, c) for this thread's RL load cases.  The slice's
// slots (stored as ST: FP64, or BF16 read into FP32 arithmetic) stream
// through shared memory kKC at a time, double-buffered, shared by every load
// case; each staged value feeds RL FMAs.  xf(col, c, out[RL]) loads the
// operand.  Called by all threads of the CTA (rows beyond nfree read
// padding: column 0, value 0).
template <class V, class ST, int NP, int RL, class XF>
__device__ __forceinline__ void spmm_slice(Stage &st, long S, int W, const int *__restrict__ scols,
                                           const ST *__restrict__ svals, XF xf, V (&y)[3][RL]) {
    const int r = Lanes<NP, RL>::row();
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int q = 0; q < RL; ++q) y[c][q] = 0;
    const int nch = (W + kKC - 1) / kKC;
    __syncthreads();  // both buffers are free
    if (nch > 0) stage_chunk<ST>(st, 0, S, 0, min(kKC, W), scols, svals);
    for (int ch = 0; ch < nch; ++ch) {
        const int b = ch & 1, k0 = ch * kKC, kc = min(kKC, W - k0);
        if (ch + 1 < nch) {
            stage_chunk<ST>(st, b ^ 1, S, k0 + kKC, min(kKC, W - k0 - kKC), scols, svals);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const ST *sv = reinterpret_cast<const ST *>(st.v[b]);
        // A full chunk runs without per-slot guards, so the compiler can
        // hoist its gathers (measured 13 % faster per batched solve).
        auto run = [&](auto full_t) {
            constexpr bool FULL = decltype(full_t)::value;
#pragma unroll
            for (int k2 = 0; k2 < kKC; k2 += 2) {
                V x[2][3][RL];
#pragma unroll
                for (int u = 0; u < 2; ++u)
                    if (FULL || k2 + u < kc) {
                        const int col = st.col[b][(k2 + u) * kSlice + r];
                        xf(col, 0, x[u][0]);
                        xf(col, 1, x[u][1]);
                        xf(col, 2, x[u][2]);
                    }
#pragma unroll
                for (int u = 0; u < 2; ++u)
                    if (FULL || k2 + u < kc) {
                        const ST *v = sv + (k2 + u) * 9 * kSlice + r;
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            const V a0 = staged_val<V>(v[(3 * c) * kSlice]),
                                    a1 = staged_val<V>(v[(3 * c + 1) * kSlice]),
                                    a2 = staged_val<V>(v[(3 * c + 2) * kSlice]);
#pragma unroll
                            for (int q = 0; q < RL; ++q)
                                y[c][q] = fma(a0, x[u][0][q], fma(a1, x[u][1][q], fma(a2, x[u][2][q], y[c][q])));
                        }
                    }
            }
        };
        if (kc == kKC) run(std::true_type{});
        else run(std::false_type{});
        __syncthreads();  // buffer b is consumed before it is refilled
    }
}

// Sums of p[q] over the CTA's 32 rows for each of this thread's load cases,
// stored as P[gsl * NR + j] for j < NR (fixed order: lanes, then warps).
template <int NP, int RL>
__device__ __forceinline__ void slice_partial(Stage &st, double (&p)[RL], double *P, int gsl, int NR) {
    constexpr int LW = Lanes<NP, RL>::kLW;
#pragma unroll
    for (int q = 0; q < RL; ++q)
#pragma unroll
        for (int off = LW; off < 32; off <<= 1) p[q] += __shfl_xor_sync(0xffffffffu, p[q], off);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane < LW)
#pragma unroll
        for (int q = 0; q < RL; ++q) st.red[w][lane * RL + q] = p[q];
    __syncthreads();
    if ((int)threadIdx.x < NR) {
        double s = 0;
        for (int ww = 0; ww < Lanes<NP, RL>::kWarps; ++ww) s += st.red[ww][threadIdx.x];
        P[(long)gsl * NR + threadIdx.x] = s;
    }
}

// Reduce phase: one warp per (variant, load case); f(v, j, sum_pa, sum_pb).
template <class F>
__device__ __forceinline__ void for_pairs(const BArgs &a, bool two, F f) {
    const int warps = blockDim.x / 32, w = threadIdx.x / 32, lane = threadIdx.x & 31;
    for (int it = blockIdx.x * warps + w; it < a.V * a.NR; it += gridDim.x * warps) {
        const int v = it / a.NR, j = it % a.NR;
        const BVar B = a.var[v];
        double sa = 0, sb = 0;
        for (int s = lane; s < B.nslice; s += 32) {
            sa += a.pa[(long)(B.slice0 + s) * a.NR + j];
            if (two) sb += a.pb[(long)(B.slice0 + s) * a.NR + j];
        }
        sa = warp_sum(sa);
        sb = warp_sum(sb);
        if (lane == 0) f(v, j, sa, sb);
    }
}

}  // namespace

// The persistent batched solver.  MIXED: FP64 FCG + FP32 V-cycle; else PCG64.
// One CTA per slice item (grid-stride); NP / RL lanes per block row, RL load
// cases per lane.  The PCG64 instances are held to 3 (RL <= 2) or 2 CTAs per
// SM worth of registers and MIXED with RL = 2 to 2 (measured faster than the
// compiler's choice); the other MIXED ones keep theirs (bounds spill and
// measured slower).
constexpr int batch_min_ctas(int threads, int rl, bool mixed) {
    return mixed ? (rl == 2 ? 2 : 1) : ((rl <= 2 ? 3 : 2) * threads <= 2048 ? (rl <= 2 ? 3 : 2) : 2048 / threads);
}
template <int NP, int RL, bool MIXED>
__global__ void __launch_bounds__(32 * (NP / RL), batch_min_ctas(32 * (NP / RL), RL, MIXED)) k_batch_solve(BArgs a) {
    __shared__ Stage st;
    using LN = Lanes<NP, RL>;
    const unsigned nb = gridDim.x + a.extra_arrivals;
    const int NR = a.NR;
    const int r = LN::row(), j0 = LN::j0();
    const bool tracer = a.trace != nullptr && blockIdx.x == 0 && threadIdx.x == 0;
    int tn = 0;
    if (tracer && tn < a.trace_cap) a.trace[tn++] = global_ns();
    auto sync = [&]() {
        const bool ok = grid_barrier(a.gs, nb, a.limit_ns);
        if (tracer && tn < a.trace_cap) a.trace[tn++] = global_ns();
        return ok;
    };
    auto X = [&](const BVar &B, int row, int c) { return vidx<NP>(B, row, c, j0); };
    // CTA-level loop over slices: f(B, v, gsl, ls, row, live[RL], any).
    // pf(Bn, lsn), run by thread 0 as each slice starts, prefetches into L2
    // what f will read of the CTA's next slice (its HBM latency then overlaps
    // this slice's work).
    auto for_slices_pf = [&](auto pf, auto f) {
        for (int gsl = blockIdx.x; gsl < a.nslices; gsl += gridDim.x) {
            if (threadIdx.x == 0 && gsl + (int)gridDim.x < a.nslices) {
                const int gn = gsl + (int)gridDim.x;
                const BVar &Bn = a.var[a.slice_var[gn]];
                pf(Bn, gn - Bn.slice0);
            }
            const int v = a.slice_var[gsl];
            const BVar B = a.var[v];
            const int ls = gsl - B.slice0;
            const int row = ls * kSlice + r;
            bool live[RL];
            bool any = false;
#pragma unroll
            for (int q = 0; q < RL; ++q) {
                live[q] = j0 + q < NR && a.live[v * NR + j0 + q] != 0;
                any |= live[q];
            }
            f(B, v, gsl, ls, row, live, any);
        }
    };
    auto for_slices = [&](auto f) { for_slices_pf([](const BVar &, int) {}, f); };
    // Prefetch pieces for a slice lsn of variant Bn: the rows' runs of a batch
    // vector (esize bytes per entry), the rows' inverse diagonal blocks (FP32
    // or FP64; a partial last slice is rounded down to 16 bytes).  Used by
    // the vector phases only: in the matrix phases the prefetch measured
    // slower (thread 0's descriptor loads delay the CTA's staging barrier,
    // and K prefetched ahead competes with the gathered columns in L2).
    auto pf_rows = [&](const BVar &Bn, int lsn, const void *base, int esize) {
        const int row0 = lsn * kSlice, rows = min(kSlice, Bn.nfree - row0);
        if (rows > 0)
            l2_prefetch(static_cast<const char *>(base) + (Bn.dof0 + 3L * row0) * NP * esize,
                        3L * rows * NP * esize);
    };
    auto pf_dinv = [&](const BVar &Bn, int lsn) {
        const int row0 = lsn * kSlice, rows = min(kSlice, Bn.nfree - row0);
        if (MIXED) {
            if (rows > 0) l2_prefetch(Bn.Dinv32 + 9L * row0, (36L * rows) & ~15L);
        } else {
            if (rows > 0) l2_prefetch(Bn.Dinv + 9L * row0, (72L * rows) & ~15L);
        }
    };

    // ---- init: r = f - K u, partials ||r||^2 (pa), ||f||^2 (pb); start of M(r)
    for_slices([&](const BVar &B, int v, int gsl, int ls, int row, const bool (&)[RL], bool) {
        const int S = B.sl_ptr[ls], W = B.sl_ptr[ls + 1] - S;
        double y[3][RL];
        spmm_slice<double, double, NP, RL>(st, S, W, B.scols, B.sv64,
                                   [&](int k, int c, double (&o)[RL]) { ldv<double, RL>(a.u + vidx<NP>(B, k, c, j0), o); }, y);
        double prr[RL] = {}, pff[RL] = {};
        if (row < B.nfree) {
            double rv[3][RL];
            for (int c = 0; c < 3; ++c) {
                double fv[RL];
                ldv<double, RL>(a.f + X(B, row, c), fv);
#pragma unroll
                for (int q = 0; q < RL; ++q) {
                    rv[c][q] = fv[q] - y[c][q];
                    prr[q] += rv[c][q] * rv[c][q];
                    pff[q] += fv[q] * fv[q];
                }
                stv<double, RL>(a.r + X(B, row, c), rv[c]);
            }
            if (MIXED) {
                float b[3][RL], x[3][RL];
#pragma unroll
                for (int q = 0; q < RL; ++q) {
                    float bb[3], xx[3];
                    for (int c = 0; c < 3; ++c) bb[c] = (float)rv[c][q];
                    block3_apply(B.Dinv32 + 9L * row, bb, xx);
                    for (int c = 0; c < 3; ++c) {
                        b[c][q] = bb[c];
                        x[c][q] = B.wsm * xx[c];
                    }
                }
                for (int c = 0; c < 3; ++c) {
                    stv<float, RL>(a.b32 + X(B, row, c), b[c]);
                    stv<float, RL>(a.x32 + X(B, row, c), x[c]);
                }
            } else {
                double z[3][RL];
#pragma unroll
                for (int q = 0; q < RL; ++q) {
                    double rr[3], zz[3];
                    for (int c = 0; c < 3; ++c) rr[c] = rv[c][q];
                    block3_apply(B.Dinv + 9L * row, rr, zz);
                    for (int c = 0; c < 3; ++c) z[c][q] = zz[c];
                }
                for (int c = 0; c < 3; ++c) stv<double, RL>(a.z64 + X(B, row, c), z[c]);
            }
        }
        slice_partial<NP, RL>(st, prr, a.pa, gsl, NR);
        slice_partial<NP, RL>(st, pff, a.pb, gsl, NR);
    });
    if (!sync()) return;
    for_pairs(a, true, [&](int v, int jj, double rr, double ff) {
        const int vj = v * NR + jj;
        a.ff[vj] = ff;
        const double t = 0.5 * a.rtol;
        a.tol2[vj] = t * t * ff;
        a.live[vj] = (ff > 0.0 && rr > a.tol2[vj] && isfinite(rr)) ? 1 : 0;
        a.iters[vj] = 0;
        a.status[vj] = isfinite(rr) ? OFEA_OK : OFEA_ERR_BREAKDOWN;
        a.beta[vj] = 0.0;
    });
    if (!sync()) return;

    // MIXED preconditioner z_new = M(r) from b32 / x32 (pre-smoothed by the
    // phase before); partials r.z_new (pa), r.z_old (pb).  Inlined at both
    // call sites: a call would put every captured local on the stack.
    auto precondition = [&](float *znew, const float *zold) __attribute__((always_inline)) -> bool {
        // t = b - K32 x
        for_slices([&](const BVar &B, int v, int gsl, int ls, int row, const bool (&live)[RL], bool any) {
            const int S = B.sl_ptr[ls], W = B.sl_ptr[ls + 1] - S;
            float y[3][RL];
            spmm_slice<float, __nv_bfloat16, NP, RL>(st, S, W, B.scols, B.sv16,
                                      [&](int k, int c, float (&o)[RL]) { ldv<float, RL>(a.x32 + vidx<NP>(B, k, c, j0), o); }, y);
            if (any && row < B.nfree)
                for (int c = 0; c < 3; ++c) {
                    float bv[RL], t[RL];
                    ldv<float, RL>(a.b32 + X(B, row, c), bv);
#pragma unroll
                    for (int q = 0; q < RL; ++q) t[q] = bv[q] - y[c][q];
                    stv<float, RL>(a.t32 + X(B, row, c), t);
                }
        });
        if (!sync()) return false;
        // c = Z^T t: CTA per aggregate, NP lanes per node (one load case
        // each), G = threads / NP nodes side by side and 4 nodes per thread in
        // flight; per-warp sums, then a fixed-order sum over the warps.
        {
            constexpr int JW = NP, kU = 4;
            const int G = blockDim.x / JW, sub = threadIdx.x / JW, jj = threadIdx.x % JW;
            const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
            float *red = reinterpret_cast<float *>(st.v);  // [warp][6][JW]: 6 * 32 * 32 floats at most
            for (int ga = blockIdx.x; ga < a.naggs; ga += gridDim.x) {
                const int v = a.agg_var[ga];
                const BVar B = a.var[v];
                const int I = ga - B.agg0;
                const bool live = jj < NR && a.live[v * NR + jj] != 0;
                float acc[6] = {0, 0, 0, 0, 0, 0};
                if (live) {
                    const float cx = (float)B.centroid[3L * I], cy = (float)B.centroid[3L * I + 1],
                                cz = (float)B.centroid[3L * I + 2];
                    const float sc = (float)B.inv_scale;
                    auto add = [&](int node, float tx, float ty, float tz) {
                        const float dx = ((float)B.xyz[3L * node] - cx) * sc;
                        const float dy = ((float)B.xyz[3L * node + 1] - cy) * sc;
                        const float dz = ((float)B.xyz[3L * node + 2] - cz) * sc;
                        acc[0] += tx;
                        acc[1] += ty;
                        acc[2] += tz;
                        acc[3] += -dz * ty + dy * tz;
                        acc[4] += dz * tx - dx * tz;
                        acc[5] += -dy * tx + dx * ty;
                    };
                    const int e = B.agg_ptr[I + 1];
                    int idx = B.agg_ptr[I] + sub;
                    for (; idx + (kU - 1) * G < e; idx += kU * G) {
                        int rr[kU], node[kU];
                        float t[kU][3];
#pragma unroll
                        for (int u = 0; u < kU; ++u) rr[u] = B.agg_nodes[idx + u * G];
#pragma unroll
                        for (int u = 0; u < kU; ++u) {
                            node[u] = B.node_of_free[rr[u]];
#pragma unroll
                            for (int c = 0; c < 3; ++c) t[u][c] = a.t32[vidx<NP>(B, rr[u], c, jj)];
                        }
#pragma unroll
                        for (int u = 0; u < kU; ++u) add(node[u], t[u][0], t[u][1], t[u][2]);
                    }
                    for (; idx < e; idx += G) {
                        const int rr = B.agg_nodes[idx];
                        add(B.node_of_free[rr], a.t32[vidx<NP>(B, rr, 0, jj)], a.t32[vidx<NP>(B, rr, 1, jj)],
                            a.t32[vidx<NP>(B, rr, 2, jj)]);
                    }
                }
#pragma unroll
                for (int k = 0; k < 6; ++k) {
#pragma unroll
                    for (int off = JW; off < 32; off <<= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], off);
                }
                if (lane < JW)
#pragma unroll
                    for (int k = 0; k < 6; ++k) red[(w * 6 + k) * JW + lane] = acc[k];
                __syncthreads();
                if ((int)threadIdx.x < 6 * JW) {
                    const int k = threadIdx.x / JW, j = threadIdx.x % JW;
                    float sum = 0.f;
                    for (int ww = 0; ww < nw; ++ww) sum += red[(ww * 6 + k) * JW + j];
                    if (j < NR && a.live[v * NR + j] != 0) a.cvec[(B.c0 + 6L * I + k) * NP + j] = sum;
                }
                __syncthreads();
            }
        }
        if (!sync()) return false;
        // e = E^-1 c: warp per coarse row, NP lanes per load case group
        {
            constexpr int JW = NP, RPW = 32 / NP;
            const int warps = blockDim.x / 32, w = threadIdx.x / 32, lane = threadIdx.x & 31;
            const int sub = lane / JW, jj = lane % JW;
            for (int gr = blockIdx.x * warps + w; gr < a.ncrows; gr += gridDim.x * warps) {
                const int v = a.crow_var[gr];
                const BVar B = a.var[v];
                const bool live = jj < NR && a.live[v * NR + jj] != 0;
                const int i = gr - B.crow0, m = B.m;
                const float *row = B.Einv32 + (long)i * m;
                float acc = 0.f;
                if (live)
                    for (int k = sub; k < m; k += RPW) acc = fmaf(__ldg(row + k), a.cvec[(B.c0 + k) * NP + jj], acc);
#pragma unroll
                for (int off = JW; off < 32; off <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
                if (sub == 0 && live) a.evec[(B.c0 + i) * NP + jj] = acc;
            }
        }
        if (!sync()) return false;
        // x += Z e
        for_slices_pf(
            [&](const BVar &Bn, int lsn) {
                pf_rows(Bn, lsn, a.x32, 4);
            },
            [&](const BVar &B, int v, int gsl, int ls, int row, const bool (&live)[RL], bool any) {
            if (!any || row >= B.nfree) return;
            const int I = B.agg_of[row], node = B.node_of_free[row];
            const float dx = (float)((B.xyz[3L * node] - B.centroid[3L * I]) * B.inv_scale);
            const float dy = (float)((B.xyz[3L * node + 1] - B.centroid[3L * I + 1]) * B.inv_scale);
            const float dz = (float)((B.xyz[3L * node + 2] - B.centroid[3L * I + 2]) * B.inv_scale);
            float e[6][RL], x[3][RL];
            for (int k = 0; k < 6; ++k) ldv<float, RL>(a.evec + (B.c0 + 6L * I + k) * NP + j0, e[k]);
            for (int c = 0; c < 3; ++c) ldv<float, RL>(a.x32 + X(B, row, c), x[c]);
#pragma unroll
            for (int q = 0; q < RL; ++q) {
                x[0][q] += e[0][q] + dz * e[4][q] - dy * e[5][q];
                x[1][q] += e[1][q] - dz * e[3][q] + dx * e[5][q];
                x[2][q] += e[2][q] + dy * e[3][q] - dx * e[4][q];
            }
            for (int c = 0; c < 3; ++c) stv<float, RL>(a.x32 + X(B, row, c), x[c]);
        });
        if (!sync()) return false;
        // post-smoothing: z_new = x + w Dinv32 (b - K32 x); partials r.z_new, r.z_old
        for_slices([&](const BVar &B, int v, int gsl, int ls, int row, const bool (&live)[RL], bool any) {
            const int S = B.sl_ptr[ls], W = B.sl_ptr[ls + 1] - S;
            float y[3][RL];
            spmm_slice<float, __nv_bfloat16, NP, RL>(st, S, W, B.scols, B.sv16,
                                      [&](int k, int c, float (&o)[RL]) { ldv<float, RL>(a.x32 + vidx<NP>(B, k, c, j0), o); }, y);
            double pn[RL] = {}, po[RL] = {};
            if (any && row < B.nfree) {
                float res[3][RL], xv[3][RL], zn[3][RL], zo[3][RL];
                double rv[3][RL];
                for (int c = 0; c < 3; ++c) {
                    float bv[RL];
                    ldv<float, RL>(a.b32 + X(B, row, c), bv);
                    ldv<float, RL>(a.x32 + X(B, row, c), xv[c]);
                    ldv<double, RL>(a.r + X(B, row, c), rv[c]);
                    if (zold) ldv<float, RL>(zold + X(B, row, c), zo[c]);
#pragma unroll
                    for (int q = 0; q < RL; ++q) res[c][q] = bv[q] - y[c][q];
                }
#pragma unroll
                for (int q = 0; q < RL; ++q) {
                    float rr[3], cor[3];
                    for (int c = 0; c < 3; ++c) rr[c] = res[c][q];
                    block3_apply(B.Dinv32 + 9L * row, rr, cor);
                    for (int c = 0; c < 3; ++c) {
                        zn[c][q] = xv[c][q] + B.wsm * cor[c];
                        if (live[q]) {
                            pn[q] += rv[c][q] * (double)zn[c][q];
                            if (zold) po[q] += rv[c][q] * (double)zo[c][q];
                        }
                    }
                }
                for (int c = 0; c < 3; ++c) stv<float, RL>(znew + X(B, row, c), zn[c]);
            }
            slice_partial<NP, RL>(st, pn, a.pa, gsl, NR);
            slice_partial<NP, RL>(st, po, a.pb, gsl, NR);
        });
        return sync();
    };

    float *zcur = a.zA, *znext = a.zB;
    if (MIXED) {
        if (!precondition(zcur, nullptr)) return;
    } else {
        // PCG64: partials r.z with z64 = Dinv r
        for_slices([&](const BVar &B, int v, int gsl, int ls, int row, const bool (&)[RL], bool) {
            double p[RL] = {};
            if (row < B.nfree)
                for (int c = 0; c < 3; ++c) {
                    double rv[RL], zv[RL];
                    ldv<double, RL>(a.r + X(B, row, c), rv);
                    ldv<double, RL>(a.z64 + X(B, row, c), zv);
#pragma unroll
                    for (int q = 0; q < RL; ++q) p[q] += rv[q] * zv[q];
                }
            slice_partial<NP, RL>(st, p, a.pa, gsl, NR);
        });
        if (!sync()) return;
    }
    for_pairs(a, false, [&](int v, int jj, double rz, double) { a.rz[v * NR + jj] = rz; });
    if (!sync()) return;

    for (int k = 0; k < a.max_iter; ++k) {
        double *pnew = (k & 1) ? a.p1 : a.p0;
        const double *pold = (k & 1) ? a.p0 : a.p1;
        // live_cnt[k % 3] counts the load cases still running after iteration k;
        // slot (k + 1) % 3 was last read two barriers ago at least
        if (blockIdx.x == 0 && threadIdx.x == 0) a.live_cnt[(k + 1) % 3] = 0;
        // A: p = z + beta p_old, q = K64 z + beta q_old (= K64 p), partial p.q
        for_slices([&](const BVar &B, int v, int gsl, int ls, int row, const bool (&live)[RL], bool any) {
            const int S = B.sl_ptr[ls], W = B.sl_ptr[ls + 1] - S;
            double bt[RL];
#pragma unroll
            for (int q = 0; q < RL; ++q) bt[q] = live[q] ? a.beta[v * NR + j0 + q] : 0.0;
            auto zval = [&](long d, double (&o)[RL]) {
                if (MIXED) {
                    float zf[RL];
                    ldv<float, RL>(zcur + d, zf);
#pragma unroll
                    for (int q = 0; q < RL; ++q) o[q] = (double)zf[q];
                } else {
                    ldv<double, RL>(a.z64 + d, o);
                }
            };
            double y[3][RL];
            spmm_slice<double, double, NP, RL>(st, S, W, B.scols, B.sv64,
                                       [&](int kk, int c, double (&o)[RL]) { zval(vidx<NP>(B, kk, c, j0), o); }, y);
            double ppq[RL] = {};
            if (any && row < B.nfree)
                for (int c = 0; c < 3; ++c) {
                    const long d = X(B, row, c);
                    double zn[RL], po[RL], qo[RL], pn[RL], qn[RL];
                    zval(d, zn);
                    ldv<double, RL>(pold + d, po);
                    ldv<double, RL>(a.q + d, qo);
#pragma unroll
                    for (int q = 0; q < RL; ++q) {
                        pn[q] = fma(bt[q], po[q], zn[q]);
                        qn[q] = bt[q] != 0.0 ? fma(bt[q], qo[q], y[c][q]) : y[c][q];
                        if (live[q]) ppq[q] += pn[q] * qn[q];
                    }
                    stv<double, RL>(pnew + d, pn);
                    stv<double, RL>(a.q + d, qn);
                }
            slice_partial<NP, RL>(st, ppq, a.pa, gsl, NR);
        });
        if (!sync()) return;
        for_pairs(a, false, [&](int v, int jj, double pq, double) {
            const int vj = v * NR + jj;
            if (!a.live[vj]) return;
            if (!(pq > 0.0) || !isfinite(pq)) {
                a.live[vj] = 0;
                a.status[vj] = OFEA_ERR_BREAKDOWN;
                a.iters[vj] = k;
                return;
            }
            a.alpha[vj] = a.rz[vj] / pq;
        });
        if (!sync()) return;
        // B: u += alpha p, r -= alpha q, partial ||r||^2; start of M(r)
        for_slices_pf(
            [&](const BVar &Bn, int lsn) {
                pf_rows(Bn, lsn, a.u, 8);
                pf_rows(Bn, lsn, pnew, 8);
                pf_rows(Bn, lsn, a.q, 8);
                pf_rows(Bn, lsn, a.r, 8);
                pf_dinv(Bn, lsn);
            },
            [&](const BVar &B, int v, int gsl, int ls, int row, const bool (&live)[RL], bool any) {
            double prr[RL] = {}, prz[RL] = {};
            if (any && row < B.nfree) {
                double al[RL];
#pragma unroll
                for (int q = 0; q < RL; ++q) al[q] = live[q] ? a.alpha[v * NR + j0 + q] : 0.0;
                double rv[3][RL];
                for (int c = 0; c < 3; ++c) {
                    const long d = X(B, row, c);
                    double uu[RL], pp[RL], qq[RL];
                    ldv<double, RL>(a.u + d, uu);
                    ldv<double, RL>(pnew + d, pp);
                    ldv<double, RL>(a.q + d, qq);
                    ldv<double, RL>(a.r + d, rv[c]);
#pragma unroll
                    for (int q = 0; q < RL; ++q)
                        if (live[q]) {
                            uu[q] = fma(al[q], pp[q], uu[q]);
                            rv[c][q] = fma(-al[q], qq[q], rv[c][q]);
                            prr[q] += rv[c][q] * rv[c][q];
                        }
                    stv<double, RL>(a.u + d, uu);
                    stv<double, RL>(a.r + d, rv[c]);
                }
                if (MIXED) {
                    float b[3][RL], x[3][RL];
#pragma unroll
                    for (int q = 0; q < RL; ++q) {
                        float bb[3], xx[3];
                        for (int c = 0; c < 3; ++c) bb[c] = (float)rv[c][q];
                        block3_apply(B.Dinv32 + 9L * row, bb, xx);
                        for (int c = 0; c < 3; ++c) {
                            b[c][q] = bb[c];
                            x[c][q] = B.wsm * xx[c];
                        }
                    }
                    for (int c = 0; c < 3; ++c) {
                        stv<float, RL>(a.b32 + X(B, row, c), b[c]);
                        stv<float, RL>(a.x32 + X(B, row, c), x[c]);
                    }
                } else {
                    double z[3][RL];
#pragma unroll
                    for (int q = 0; q < RL; ++q) {
                        double rr[3], zz[3];
                        for (int c = 0; c < 3; ++c) rr[c] = rv[c][q];
                        block3_apply(B.Dinv + 9L * row, rr, zz);
                        for (int c = 0; c < 3; ++c) {
                            z[c][q] = zz[c];
                            if (live[q]) prz[q] += rr[c] * zz[c];
                        }
                    }
                    for (int c = 0; c < 3; ++c) stv<double, RL>(a.z64 + X(B, row, c), z[c]);
                }
            }
            slice_partial<NP, RL>(st, prr, a.pa, gsl, NR);
            if (!MIXED) slice_partial<NP, RL>(st, prz, a.pb, gsl, NR);
        });
        if (!sync()) return;
        for_pairs(a, !MIXED, [&](int v, int jj, double rr, double rz) {
            const int vj = v * NR + jj;
            if (!a.live[vj]) return;
            a.iters[vj] = k + 1;
            if (!isfinite(rr)) {
                a.live[vj] = 0;
                a.status[vj] = OFEA_ERR_BREAKDOWN;
                return;
            }
            if (rr <= a.tol2[vj]) {
                a.live[vj] = 0;
                return;
            }
            if (k + 1 >= a.max_iter) {
                a.live[vj] = 0;
                a.status[vj] = OFEA_ERR_NOT_CONVERGED;
                return;
            }
            if (!MIXED) {
                a.beta[vj] = rz / a.rz[vj];
                a.rz[vj] = rz;
            }
            atomicAdd(&a.live_cnt[k % 3], 1);
        });
        if (!sync()) return;
        if (*(volatile int *)&a.live_cnt[k % 3] == 0) break;
        if (MIXED) {
            if (!precondition(znext, zcur)) return;
            for_pairs(a, true, [&](int v, int jj, double rzn, double rzo) {
                const int vj = v * NR + jj;
                if (!a.live[vj]) return;
                a.beta[vj] = (rzn - rzo) / a.rz[vj];
                a.rz[vj] = rzn;
            });
            if (!sync()) return;
            float *tz = zcur;
            zcur = znext;
            znext = tz;
        }
    }
}

// Host order (load case j at j * n, DOF d) to the batch's interleaved order
// (d * NP + j) for one variant (and back); padding load cases stay zero.
__global__ void k_interleave(long n, int nrhs, int NP, const double *__restrict__ src, double *__restrict__ dst) {
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < n * nrhs; g += (long)gridDim.x * blockDim.x) {
        const long j = g / n, d = g % n;
        dst[d * NP + j] = src[g];
    }
}
__global__ void k_deinterleave(long n, int nrhs, int NP, const double *__restrict__ src, double *__restrict__ dst) {
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < n * nrhs; g += (long)gridDim.x * blockDim.x) {
        const long j = g / n, d = g % n;
        dst[g] = src[d * NP + j];
    }
}

// True FP64 residual partials per (slice, load case): ||f - K u||^2 (pa), ||f||^2 (pb).
template <int NP, int RL>
__global__ void __launch_bounds__(32 * (NP / RL)) k_batch_residual(BArgs a) {
    __shared__ Stage st;
    using LN = Lanes<NP, RL>;
    const int NR = a.NR, j0 = LN::j0(), r = LN::row();
    for (int gsl = blockIdx.x; gsl < a.nslices; gsl += gridDim.x) {
        const BVar B = a.var[a.slice_var[gsl]];
        const int ls = gsl - B.slice0, row = ls * kSlice + r;
        const int S = B.sl_ptr[ls], W = B.sl_ptr[ls + 1] - S;
        double y[3][RL];
        spmm_slice<double, double, NP, RL>(st, S, W, B.scols, B.sv64,
                                   [&](int k, int c, double (&o)[RL]) { ldv<double, RL>(a.u + vidx<NP>(B, k, c, j0), o); }, y);
        double prr[RL] = {}, pff[RL] = {};
        if (row < B.nfree)
            for (int c = 0; c < 3; ++c) {
                double fv[RL];
                ldv<double, RL>(a.f + vidx<NP>(B, row, c, j0), fv);
#pragma unroll
                for (int q = 0; q < RL; ++q) {
                    const double rv = fv[q] - y[c][q];
                    prr[q] += rv * rv;
                    pff[q] += fv[q] * fv[q];
                }
            }
        slice_partial<NP, RL>(st, prr, a.pa, gsl, NR);
        slice_partial<NP, RL>(st, pff, a.pb, gsl, NR);
    }
}

// Per (variant, load case): rel = sqrt(rr / ff).
__global__ void k_batch_rel(BArgs a, double *rel) {
    for_pairs(a, true, [&](int v, int j, double rr, double ff) {
        rel[v * a.NR + j] = ff > 0.0 ? sqrt(rr / ff) : 0.0;
    });
}

// A bounded wait that nothing releases: one extra arrival is expected at
// the first barrier, so every CTA's wait runs out after limit_ns and the
// kernel reports the failure (used to test the failure path).
__global__ void k_barrier_probe(GridSync *gs, unsigned extra, unsigned long long limit_ns, int *out) {
    const bool ok = grid_barrier(gs, gridDim.x + extra, limit_ns);
    if (blockIdx.x == 0 && threadIdx.x == 0) *out = ok ? 1 : 0;
}

// ------------------------------------------------------------------ host --

namespace {

struct TuneCfg {
    int rl = 2, ctas_per_sm = 1;
    double ms_per_iter = 0.0;
};

// Load-case stride of the batch vectors: NR rounded up to a power of two >= 4.
int np_for(int NR) { return NR <= 4 ? 4 : NR <= 8 ? 8 : NR <= 16 ? 16 : 32; }
int threads_for(int np, int rl) { return 32 * (np / rl); }

template <int NP, int RL>
const void *solve_inst(bool mixed) {
    return mixed ? (const void *)k_batch_solve<NP, RL, true> : (const void *)k_batch_solve<NP, RL, false>;
}
template <int NP>
const void *solve_np(int rl, bool mixed) {
    switch (rl) {
        case 1: return solve_inst<NP, 1>(mixed);
        case 2: return solve_inst<NP, 2>(mixed);
        case 4: return solve_inst<NP, 4>(mixed);
    }
    fail(OFEA_ERR_INVALID_ARG, "unsupported load cases per lane");
}
const void *solve_kernel_raw(int np, int rl, bool mixed) {
    switch (np) {
        case 4: return solve_np<4>(rl, mixed);
        case 8: return solve_np<8>(rl, mixed);
        case 16: return solve_np<16>(rl, mixed);
        case 32: return solve_np<32>(rl, mixed);
    }
    fail(OFEA_ERR_INVALID_ARG, "unsupported load-case stride");
}
// Kernel instance for (NP, RL, mixed), with the shared-memory carveout at its
// maximum so that several CTAs' slot stages fit on an SM.
const void *solve_kernel(int np, int rl, bool mixed) {
    const void *fn = solve_kernel_raw(np, rl, mixed);
    OFEA_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                   (int)cudaSharedmemCarveoutMaxShared));
    return fn;
}
template <int NP>
const void *residual_np(int rl) {
    switch (rl) {
        case 1: return (const void *)k_batch_residual<NP, 1>;
        case 2: return (const void *)k_batch_residual<NP, 2>;
        case 4: return (const void *)k_batch_residual<NP, 4>;
    }
    fail(OFEA_ERR_INVALID_ARG, "unsupported load cases per lane");
}
const void *residual_kernel(int np, int rl) {
    switch (np) {
        case 4: return residual_np<4>(rl);
        case 8: return residual_np<8>(rl);
        case 16: return residual_np<16>(rl);
        case 32: return residual_np<32>(rl);
    }
    fail(OFEA_ERR_INVALID_ARG, "unsupported load-case stride");
}

// ---- the on-disk tuning cache: one JSON object per line inside "entries"
std::mutex g_tune_mu;

std::string tune_path() {
    if (const char *p = std::getenv("OFEA_TUNE_FILE")) return p;
    const char *home = std::getenv("HOME");
    return std::string(home ? home : ".") + "/.cache/openfea_b200_tune.json";
}

std::map<std::string, TuneCfg> tune_load(const std::string &path) {
    std::map<std::string, TuneCfg> out;
    std::ifstream in(path);
    std::string line;
    auto num = [](const std::string &l, const char *k, double dflt) {
        const std::string key = std::string("\"") + k + "\": ";
        const size_t p = l.find(key);
        return p == std::string::npos ? dflt : std::strtod(l.c_str() + p + key.size(), nullptr);
    };
    while (std::getline(in, line)) {
        const size_t p = line.find("\"key\": \"");
        if (p == std::string::npos) continue;
        const size_t b = p + 8, e = line.find('"', b);
        if (e == std::string::npos) continue;
        TuneCfg t;
        t.rl = (int)num(line, "rl", 2);
        t.ctas_per_sm = (int)num(line, "ctas_per_sm", 1);
        t.ms_per_iter = num(line, "ms_per_iter", 0);
        out[line.substr(b, e - b)] = t;
    }
    return out;
}

void tune_store(const std::string &path, const std::string &key, const TuneCfg &t) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto all = tune_load(path);
    all[key] = t;
    const size_t slash = path.rfind('/');
    if (slash != std::string::npos && slash > 0) mkdir(path.substr(0, slash).c_str(), 0755);  // one level (~/.cache)
    std::ofstream o(path);
    if (!o) return;  // the cache is an optimisation: an unwritable path is not an error
    o << "{\n  \"entries\": [\n";
    size_t i = 0;
    for (const auto &kv : all) {
        char buf[512];
        std::snprintf(buf, sizeof(buf),
                      "    {\"key\": \"%s\", \"rl\": %d, \"ctas_per_sm\": %d, \"ms_per_iter\": %.6f}%s\n",
                      kv.first.c_str(), kv.second.rl, kv.second.ctas_per_sm,
                      kv.second.ms_per_iter, ++i < all.size() ? "," : "");
        o << buf;
    }
    o << "  ]\n}\n";
}

}  // namespace

// ---- the batch plan

}  // namespace ofea

struct ofea_batch {
    int device = 0, V = 0, NR = 0, NP = 4, num_sms = 148;
    cudaStream_t stream = nullptr;
    std::vector<ofea_ctx *> ctx;
    std::vector<long> dof0, c0;
    long ndof = 0, ncoarse = 0;
    int nslices = 0, naggs = 0, ncrows = 0;
    bool mixed_ready = false, have_rhs = false;
    ofea::DevBuf<ofea::BVar> var;
    ofea::DevBuf<int> slice_var, agg_var, crow_var;
    ofea::DevBuf<double> f, u, r, p0, p1, q, z64, pa, pb, ff, tol2, rz, alpha, beta, rel, stage;
    ofea::DevBuf<float> b32, x32, t32, zA, zB, cvec, evec;
    ofea::DevBuf<int> live, iters, status, live_cnt;
    ofea::DevBuf<ofea::GridSync> gs;
    ofea::DevBuf<unsigned long long> trace;  // per-phase timestamps when tracing (trace_cap > 0)
    ofea::HostBuf<double> bounce[2];          // page-locked blocks between the callers' arrays and the device
    int trace_cap = 0;
    std::map<int, ofea::TuneCfg> tuned;  // by method
    // the captured graph of one launch and what it was captured for
    cudaGraphExec_t exec = nullptr;
    std::string exec_key;
    ~ofea_batch() {
        if (exec) cudaGraphExecDestroy(exec);
    }
};

namespace ofea {

namespace {

std::string device_name(int dev) {
    cudaDeviceProp p{};
    if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) return "gpu";
    return p.name;
}

// Descriptor table; with `mixed` also the coarse levels' pointers and offsets.
void build_desc(ofea_batch *b, bool mixed) {
    std::vector<BVar> d(b->V);
    std::vector<int> sv, av, cv;
    long c0 = 0;
    int slice0 = 0, agg0 = 0, crow0 = 0;
    b->c0.assign(b->V, 0);
    for (int v = 0; v < b->V; ++v) {
        ofea_ctx *c = b->ctx[v];
        BVar &B = d[v];
        std::memset(&B, 0, sizeof(B));
        B.nfree = c->nfree;
        B.n = c->n;
        B.nslice = (c->nfree + kSlice - 1) / kSlice;
        B.slice0 = slice0;
        B.dof0 = b->dof0[v];
        B.sl_ptr = c->sl_ptr.p;
        B.scols = c->scols.p;
        B.sv64 = c->sv64.p;
        B.Dinv = c->Dinv.p;
        B.sv16 = c->sv16.p;
        B.Dinv32 = c->Dinv32.p;
        for (int s = 0; s < B.nslice; ++s) sv.push_back(v);
        slice0 += B.nslice;
        if (mixed) {
            const Coarse &C = c->coarse;
            B.na = C.na;
            B.m = C.m;
            B.agg0 = agg0;
            B.crow0 = crow0;
            B.c0 = c0;
            b->c0[v] = c0;
            B.agg_of = C.agg_of.p;
            B.agg_ptr = C.agg_ptr.p;
            B.agg_nodes = C.agg_nodes.p;
            B.node_of_free = c->node_of_free.p;
            B.xyz = c->xyz.p;
            B.centroid = C.centroid.p;
            B.Einv32 = C.Einv32.p;
            B.inv_scale = C.inv_scale;
            B.wsm = smoother_weight(c, kBatchSmootherDamping);
            for (int a = 0; a < C.na; ++a) av.push_back(v);
            for (int i = 0; i < C.m; ++i) cv.push_back(v);
            agg0 += C.na;
            crow0 += C.m;
            c0 += C.m;
        }
    }
    b->nslices = slice0;
    b->naggs = agg0;
    b->ncrows = crow0;
    b->ncoarse = c0;
    cudaStream_t s = b->stream;
    b->var.upload(d.data(), d.size(), s);
    b->slice_var.upload(sv.data(), sv.size(), s);
    if (mixed) {
        b->agg_var.upload(av.data(), av.size(), s);
        b->crow_var.upload(cv.data(), cv.size(), s);
    }
    const size_t NR = b->NR;
    b->pa.ensure(std::max<size_t>(1, (size_t)b->nslices * NR));
    b->pb.ensure(std::max<size_t>(1, (size_t)b->nslices * NR));
    OFEA_CUDA(cudaStreamSynchronize(s));
}

void prepare(ofea_batch *b, bool mixed) {
    if (mixed && !b->mixed_ready) {
        for (ofea_ctx *c : b->ctx) {
            setup_coarse(c, c->coarse_nodes);
            coarse_dense_inverse(c);
            OFEA_CUDA(cudaStreamSynchronize(c->stream));
        }
        build_desc(b, true);
        const size_t n = (size_t)b->ndof * b->NP, nc = std::max<size_t>(1, (size_t)b->ncoarse * b->NP);
        b->b32.ensure(n);
        b->x32.ensure(n);
        b->t32.ensure(n);
        b->zA.ensure(n);
        b->zB.ensure(n);
        b->cvec.ensure(nc);
        b->evec.ensure(nc);
        for (auto *buf : {&b->b32, &b->x32, &b->t32, &b->zA, &b->zB})
            OFEA_CUDA(cudaMemsetAsync(buf->p, 0, sizeof(float) * n, b->stream));
        OFEA_CUDA(cudaMemsetAsync(b->cvec.p, 0, sizeof(float) * nc, b->stream));
        OFEA_CUDA(cudaMemsetAsync(b->evec.p, 0, sizeof(float) * nc, b->stream));
        b->mixed_ready = true;
    }
    if (!mixed && !b->z64.p) {
        b->z64.ensure((size_t)b->ndof * b->NP);
        OFEA_CUDA(cudaMemsetAsync(b->z64.p, 0, sizeof(double) * b->ndof * b->NP, b->stream));
    }
}

BArgs make_args(ofea_batch *b, bool mixed, const TuneCfg &t, int max_iter, double rtol) {
    BArgs a{};
    a.V = b->V;
    a.NR = b->NR;
    a.nslices = b->nslices;
    a.naggs = mixed ? b->naggs : 0;
    a.ncrows = mixed ? b->ncrows : 0;
    a.max_iter = max_iter;
    a.extra_arrivals = 0;
    a.limit_ns = 5000000000ull;  // 5 s: far above any phase
    a.rtol = rtol;
    a.var = b->var.p;
    a.slice_var = b->slice_var.p;
    a.agg_var = b->agg_var.p;
    a.crow_var = b->crow_var.p;
    a.f = b->f.p;
    a.u = b->u.p;
    a.r = b->r.p;
    a.p0 = b->p0.p;
    a.p1 = b->p1.p;
    a.q = b->q.p;
    a.z64 = b->z64.p;
    a.b32 = b->b32.p;
    a.x32 = b->x32.p;
    a.t32 = b->t32.p;
    a.zA = b->zA.p;
    a.zB = b->zB.p;
    a.cvec = b->cvec.p;
    a.evec = b->evec.p;
    a.pa = b->pa.p;
    a.pb = b->pb.p;
    a.ff = b->ff.p;
    a.tol2 = b->tol2.p;
    a.rz = b->rz.p;
    a.alpha = b->alpha.p;
    a.beta = b->beta.p;
    a.live = b->live.p;
    a.iters = b->iters.p;
    a.status = b->status.p;
    a.live_cnt = b->live_cnt.p;
    a.gs = b->gs.p;
    a.trace = b->trace_cap > 0 ? b->trace.p : nullptr;
    a.trace_cap = b->trace_cap;
    return a;
}

int grid_of(ofea_batch *b, const void *fn, const TuneCfg &t) {
    int occ = 0;
    OFEA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, threads_for(b->NP, t.rl), 0));
    if (occ < 1) fail(OFEA_ERR_CAPACITY, "batched solver kernel does not fit on an SM");
    return b->num_sms * std::min(occ, t.ctas_per_sm);
}

// Enqueue one launch: reset of the per-launch state + the cooperative kernel.
void enqueue(ofea_batch *b, const BArgs &a, const TuneCfg &t, bool mixed) {
    cudaStream_t s = b->stream;
    const size_t n = (size_t)b->ndof * b->NP;
    OFEA_CUDA(cudaMemsetAsync(b->p0.p, 0, sizeof(double) * n, s));
    OFEA_CUDA(cudaMemsetAsync(b->p1.p, 0, sizeof(double) * n, s));
    OFEA_CUDA(cudaMemsetAsync(b->gs.p, 0, sizeof(GridSync), s));
    OFEA_CUDA(cudaMemsetAsync(b->live_cnt.p, 0, sizeof(int) * 3, s));
    if (a.trace) OFEA_CUDA(cudaMemsetAsync(a.trace, 0, sizeof(unsigned long long) * a.trace_cap, s));
    const void *fn = solve_kernel(b->NP, t.rl, mixed);
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid_of(b, fn, t));
    cfg.blockDim = dim3(threads_for(b->NP, t.rl));
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void *args[] = {(void *)&a};
    OFEA_CUDA(cudaLaunchKernelExC(&cfg, fn, args));
}

// True FP64 residuals per (variant, load case) into b->rel.
void residuals(ofea_batch *b, const TuneCfg &t) {
    BArgs a = make_args(b, false, t, 0, 0.0);
    cudaStream_t s = b->stream;
    const void *fn = residual_kernel(b->NP, t.rl);
    const int G = std::min(kMaxGrid, b->num_sms * 4);
    void *args[] = {(void *)&a};
    OFEA_CUDA(cudaLaunchKernel(fn, dim3(G), dim3(threads_for(b->NP, t.rl)), args, 0, s));
    k_batch_rel<<<std::max(1, std::min(kMaxGrid, (b->V * b->NR + 7) / 8)), 256, 0, s>>>(a, b->rel.p);
    OFEA_CHECK_LAUNCH();
}

std::string tune_key(ofea_batch *b, bool mixed) {
    // problem class: device, method, load cases, rows rounded to 2 significant digits
    long rows = (long)b->nslices * kSlice;
    long scale = 1;
    while (rows / scale >= 100) scale *= 10;
    std::ostringstream k;
    k << device_name(b->device) << "|" << (mixed ? "mixed" : "pcg64") << "|nrhs=" << b->NR
      << "|rows~" << (rows / scale) * scale << "|variants=" << b->V;
    return k.str();
}

// Times a few iterations of every candidate and keeps the fastest; the
// result is cached in the batch and on disk (OFEA_TUNE_FILE or
// ~/.cache/openfea_b200_tune.json), keyed by device and problem class.
TuneCfg autotune(ofea_batch *b, bool mixed, double rtol) {
    const std::string key = tune_key(b, mixed);
    const std::string path = tune_path();
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto all = tune_load(path);
        auto it = all.find(key);
        if (it != all.end()) {
            TuneCfg t = it->second;
            if ((t.rl == 1 || t.rl == 2 || t.rl == 4) && t.rl <= b->NP && t.ctas_per_sm >= 1 && t.ctas_per_sm <= 32)
                return t;
        }
    }
    std::vector<TuneCfg> cand;
    for (int rl : {1, 2, 4}) {
        int occ = 0;
        OFEA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, solve_kernel(b->NP, rl, mixed),
                                                                threads_for(b->NP, rl), 0));
        std::vector<int> cps{1, 2, 4, occ};
        std::sort(cps.begin(), cps.end());
        cps.erase(std::unique(cps.begin(), cps.end()), cps.end());
        for (int c : cps)
            if (c >= 1 && c <= occ) cand.push_back(TuneCfg{rl, c, 0.0});
    }
    // per-iteration time = (t(long) - t(short)) / (long - short): the init
    // phases and the launch cancel out
    const int it_short = 4, it_long = 20;
    cudaEvent_t e0, e1;
    OFEA_CUDA(cudaEventCreate(&e0));
    OFEA_CUDA(cudaEventCreate(&e1));
    TuneCfg best;
    double best_ms = 1e300;
    cudaStream_t s = b->stream;
    auto time_launch = [&](const TuneCfg &t, int iters) {
        double ms_min = 1e300;
        for (int rep = 0; rep < 3; ++rep) {
            OFEA_CUDA(cudaMemsetAsync(b->u.p, 0, sizeof(double) * b->ndof * b->NP, s));
            BArgs a = make_args(b, mixed, t, iters, rtol);
            OFEA_CUDA(cudaEventRecord(e0, s));
            enqueue(b, a, t, mixed);
            OFEA_CUDA(cudaEventRecord(e1, s));
            OFEA_CUDA(cudaEventSynchronize(e1));
            float ms = 0;
            OFEA_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            GridSync g{};
            OFEA_CUDA(cudaMemcpy(&g, b->gs.p, sizeof(g), cudaMemcpyDeviceToHost));
            if (g.err) fail(OFEA_ERR_TIMEOUT, "batched solver: a grid-barrier wait ran out while tuning");
            ms_min = std::min(ms_min, (double)ms);
        }
        return ms_min;
    };
    const bool verbose = std::getenv("OFEA_TUNE_VERBOSE") != nullptr;
    for (TuneCfg &t : cand) {
        t.ms_per_iter = std::max(0.0, time_launch(t, it_long) - time_launch(t, it_short)) / (it_long - it_short);
        if (verbose)
            std::fprintf(stderr, "ofea tune %s: rl %d ctas/SM %d -> %.4f ms per iteration\n", key.c_str(), t.rl,
                         t.ctas_per_sm, t.ms_per_iter);
        if (t.ms_per_iter < best_ms) {
            best_ms = t.ms_per_iter;
            best = t;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    tune_store(path, key, best);
    return best;
}

}  // namespace

ofea_batch *batch_create(ofea_ctx *const *ctxs, int nv, int nrhs) {
    if (!ctxs || nv < 1) fail(OFEA_ERR_INVALID_ARG, "batch: no variants");
    if (nrhs < 1 || nrhs > kMaxBatchRhs)
        fail(OFEA_ERR_CAPACITY, "batch: 1 to " + std::to_string(kMaxBatchRhs) + " load cases per variant");
    auto b = std::make_unique<ofea_batch>();
    b->V = nv;
    b->NR = nrhs;
    b->NP = np_for(nrhs);
    for (int v = 0; v < nv; ++v) {
        ofea_ctx *c = ctxs[v];
        if (!c) fail(OFEA_ERR_INVALID_ARG, "batch: NULL context");
        if (!c->K_ok || !c->sell_ok) fail(OFEA_ERR_STATE, "batch: variant " + std::to_string(v) + " not assembled");
        OFEA_CUDA(cudaSetDevice(c->device));
        ensure_sv16(c);  // BF16 planes of the V-cycle SpMMs (a fused assembly leaves them to be derived)
        OFEA_CUDA(cudaStreamSynchronize(c->stream));
        if (c->device != ctxs[0]->device) fail(OFEA_ERR_INVALID_ARG, "batch: variants on different GPUs");
        b->ctx.push_back(c);
    }
    b->device = ctxs[0]->device;
    b->num_sms = ctxs[0]->num_sms;
    b->stream = ctxs[0]->stream;
    OFEA_CUDA(cudaSetDevice(b->device));
    int coop = 0;
    OFEA_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, b->device));
    if (!coop) fail(OFEA_ERR_NO_DEVICE, "batch: the GPU does not support cooperative launches");
    long d0 = 0;
    for (ofea_ctx *c : b->ctx) {
        b->dof0.push_back(d0);
        d0 += c->n;
    }
    b->ndof = d0;
    const size_t n = std::max<size_t>(1, (size_t)b->ndof * b->NP), vj = (size_t)nv * nrhs;
    for (auto *buf : {&b->f, &b->u, &b->r, &b->p0, &b->p1, &b->q}) buf->ensure(n);
    for (auto *buf : {&b->ff, &b->tol2, &b->rz, &b->alpha, &b->beta, &b->rel}) buf->ensure(vj);
    for (auto *buf : {&b->live, &b->iters, &b->status}) buf->ensure(vj);
    b->live_cnt.ensure(3);
    b->gs.ensure(1);
    OFEA_CUDA(cudaMemsetAsync(b->f.p, 0, sizeof(double) * n, b->stream));
    OFEA_CUDA(cudaMemsetAsync(b->u.p, 0, sizeof(double) * n, b->stream));
    build_desc(b.get(), false);
    return b.release();
}

void batch_destroy(ofea_batch *b) {
    if (!b) return;
    cudaSetDevice(b->device);
    delete b;
}

namespace {

// dst <- src (host memory, bytes), split over the host pool's chunks when large.
void host_copy(void *dst, const void *src, size_t bytes) {
    if (bytes < (size_t(4) << 20)) {
        std::memcpy(dst, src, bytes);
        return;
    }
    const long units = (long)(bytes / 64);
    host_for_chunks([&](int k) {
        const size_t a = (size_t)chunk_begin(units, k) * 64;
        const size_t e = k + 1 == kHostChunks ? bytes : (size_t)chunk_begin(units, k + 1) * 64;
        std::memcpy(static_cast<char *>(dst) + a, static_cast<const char *>(src) + a, e - a);
    });
}

// Two events for the bounce blocks, destroyed on every exit.
struct EventPair {
    cudaEvent_t e[2] = {nullptr, nullptr};
    EventPair() {
        for (auto &x : e) OFEA_CUDA(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
    }
    ~EventPair() {
        for (auto &x : e)
            if (x) cudaEventDestroy(x);
    }
};

}  // namespace

// The callers' arrays are pageable: each variant goes through one of two
// page-locked bounce blocks, the host copy of one variant (over the host
// pool's chunks) overlapping the DMA of the other.
void batch_set_rhs(ofea_batch *b, const double *const *f) {
    OFEA_CUDA(cudaSetDevice(b->device));
    cudaStream_t s = b->stream;
    size_t maxn = 1;
    for (int v = 0; v < b->V; ++v) {
        if (!f[v]) fail(OFEA_ERR_INVALID_ARG, "batch: NULL load array");
        maxn = std::max(maxn, (size_t)b->ctx[v]->n * b->NR);
    }
    b->stage.ensure((size_t)b->ndof * b->NR);
    for (auto &h : b->bounce) h.ensure(maxn);
    EventPair ev;
    for (int v = 0; v < b->V; ++v) {
        const long n = b->ctx[v]->n;
        const int k = v & 1;
        double *dst = b->stage.p + b->dof0[v] * b->NR;
        if (v >= 2) OFEA_CUDA(cudaEventSynchronize(ev.e[k]));  // the DMA out of this block (variant v - 2) is done
        host_copy(b->bounce[k].p, f[v], sizeof(double) * n * b->NR);
        OFEA_CUDA(cudaMemcpyAsync(dst, b->bounce[k].p, sizeof(double) * n * b->NR, cudaMemcpyHostToDevice, s));
        OFEA_CUDA(cudaEventRecord(ev.e[k], s));
        k_interleave<<<std::max(1, std::min(kMaxGrid, (int)((n * b->NR + 255) / 256))), 256, 0, s>>>(
            n, b->NR, b->NP, dst, b->f.p + b->dof0[v] * b->NP);
        OFEA_CHECK_LAUNCH();
    }
    OFEA_CUDA(cudaStreamSynchronize(s));
    b->have_rhs = true;
}

void batch_get_solution(ofea_batch *b, double *const *u) {
    OFEA_CUDA(cudaSetDevice(b->device));
    cudaStream_t s = b->stream;
    size_t maxn = 1;
    for (int v = 0; v < b->V; ++v) {
        if (!u[v]) fail(OFEA_ERR_INVALID_ARG, "batch: NULL solution array");
        maxn = std::max(maxn, (size_t)b->ctx[v]->n * b->NR);
    }
    b->stage.ensure((size_t)b->ndof * b->NR);
    for (auto &h : b->bounce) h.ensure(maxn);
    for (int v = 0; v < b->V; ++v) {
        const long n = b->ctx[v]->n;
        k_deinterleave<<<std::max(1, std::min(kMaxGrid, (int)((n * b->NR + 255) / 256))), 256, 0, s>>>(
            n, b->NR, b->NP, b->u.p + b->dof0[v] * b->NP, b->stage.p + b->dof0[v] * b->NR);
        OFEA_CHECK_LAUNCH();
    }
    EventPair ev;
    for (int v = 0; v <= b->V; ++v) {
        if (v < b->V) {  // block v & 1 was last read by the host copy of variant v - 2, already done
            const long n = b->ctx[v]->n;
            OFEA_CUDA(cudaMemcpyAsync(b->bounce[v & 1].p, b->stage.p + b->dof0[v] * b->NR, sizeof(double) * n * b->NR,
                                      cudaMemcpyDeviceToHost, s));
            OFEA_CUDA(cudaEventRecord(ev.e[v & 1], s));
        }
        if (v > 0) {
            const int w = v - 1;
            OFEA_CUDA(cudaEventSynchronize(ev.e[w & 1]));
            host_copy(u[w], b->bounce[w & 1].p, sizeof(double) * b->ctx[w]->n * b->NR);
        }
    }
}

void batch_tuning(ofea_batch *b, int method, int *rl, int *threads, int *ctas_per_sm, double *ms_per_iter) {
    const bool mixed = method == OFEA_SOLVER_MIXED;
    OFEA_CUDA(cudaSetDevice(b->device));
    prepare(b, mixed);
    auto it = b->tuned.find(method);
    if (it == b->tuned.end()) it = b->tuned.emplace(method, autotune(b, mixed, 1e-8)).first;
    const TuneCfg &t = it->second;
    if (rl) *rl = t.rl;
    if (threads) *threads = threads_for(b->NP, t.rl);
    if (ctas_per_sm) *ctas_per_sm = t.ctas_per_sm;
    if (ms_per_iter) *ms_per_iter = t.ms_per_iter;
}

// Solves all (variant, load case) pairs on the resident right-hand sides.
// One graph launch per attempt; a pair whose true FP64 residual misses rtol
// after the kernel (recurrence drift) is resumed from its u by the next
// attempt.  stats: one per variant (worst load case).
void batch_solve(ofea_batch *b, const ofea_solve_opts &o, ofea_solve_stats *stats, ofea_solve_stats *case_stats) {
    if (o.method != OFEA_SOLVER_MIXED && o.method != OFEA_SOLVER_PCG64)
        fail(OFEA_ERR_UNKNOWN_SOLVER, "batch: method must be OFEA_SOLVER_PCG64 or OFEA_SOLVER_MIXED");
    if (!b->have_rhs) fail(OFEA_ERR_STATE, "batch: no load cases set");
    if (!(o.rtol > 0) || o.max_iter < 1) fail(OFEA_ERR_INVALID_ARG, "batch: bad rtol / max_iter");
    const bool mixed = o.method == OFEA_SOLVER_MIXED;
    OFEA_CUDA(cudaSetDevice(b->device));
    prepare(b, mixed);
    batch_tuning(b, o.method, nullptr, nullptr, nullptr, nullptr);
    const TuneCfg t = b->tuned[o.method];
    cudaStream_t s = b->stream;
    const int VJ = b->V * b->NR;
    std::vector<int> iters_tot(VJ, 0), hit(VJ), hst(VJ);
    std::vector<double> hrel(VJ);
    cudaEvent_t e0, e1;
    OFEA_CUDA(cudaEventCreate(&e0));
    OFEA_CUDA(cudaEventCreate(&e1));
    OFEA_CUDA(cudaMemsetAsync(b->u.p, 0, sizeof(double) * b->ndof * b->NP, s));
    OFEA_CUDA(cudaEventRecord(e0, s));
    int attempts = 0, launches = 0, remaining = o.max_iter;
    bool failed_barrier = false;
    for (; attempts < 4 && remaining > 0; ++attempts) {
        BArgs a = make_args(b, mixed, t, remaining, o.rtol);
        std::ostringstream k;
        k << o.method << "/" << t.rl << "/" << t.ctas_per_sm << "/" << remaining << "/"
          << o.rtol << "/" << b->trace_cap;
        if (o.use_graph) {
            if (!b->exec || b->exec_key != k.str()) {
                if (b->exec) {
                    cudaGraphExecDestroy(b->exec);
                    b->exec = nullptr;
                }
                cudaGraph_t g = nullptr;
                OFEA_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
                try {
                    enqueue(b, a, t, mixed);
                } catch (...) {
                    cudaStreamEndCapture(s, &g);
                    if (g) cudaGraphDestroy(g);
                    throw;
                }
                OFEA_CUDA(cudaStreamEndCapture(s, &g));
                cudaError_t e = cudaGraphInstantiate(&b->exec, g, 0);
                cudaGraphDestroy(g);
                if (e != cudaSuccess) fail_cuda(e, "cudaGraphInstantiate(batched solve)", __FILE__, __LINE__);
                b->exec_key = k.str();
            }
            OFEA_CUDA(cudaGraphLaunch(b->exec, s));
        } else {
            enqueue(b, a, t, mixed);
        }
        ++launches;
        residuals(b, t);
        launches += 2;
        GridSync g{};
        OFEA_CUDA(cudaMemcpyAsync(&g, b->gs.p, sizeof(g), cudaMemcpyDeviceToHost, s));
        OFEA_CUDA(cudaMemcpyAsync(hit.data(), b->iters.p, sizeof(int) * VJ, cudaMemcpyDeviceToHost, s));
        OFEA_CUDA(cudaMemcpyAsync(hst.data(), b->status.p, sizeof(int) * VJ, cudaMemcpyDeviceToHost, s));
        OFEA_CUDA(cudaMemcpyAsync(hrel.data(), b->rel.p, sizeof(double) * VJ, cudaMemcpyDeviceToHost, s));
        OFEA_CUDA(cudaStreamSynchronize(s));
        if (g.err) {
            failed_barrier = true;
            break;
        }
        int most = 0;
        bool again = false;
        for (int i = 0; i < VJ; ++i) {
            iters_tot[i] += hit[i];
            most = std::max(most, hit[i]);
            if (hst[i] == OFEA_OK && !(hrel[i] <= o.rtol)) again = true;
        }
        remaining -= std::max(most, 1);
        if (!again) break;
    }
    OFEA_CUDA(cudaEventRecord(e1, s));
    OFEA_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    OFEA_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (failed_barrier) fail(OFEA_ERR_TIMEOUT, "batched solver: a grid-barrier wait ran out");
    if (stats) {
        for (int v = 0; v < b->V; ++v) {
            ofea_solve_stats &st = stats[v];
            st = ofea_solve_stats{};
            int worst = OFEA_OK;
            for (int j = 0; j < b->NR; ++j) {
                const int i = v * b->NR + j;
                st.iterations = std::max(st.iterations, iters_tot[i]);
                st.rel_residual = std::max(st.rel_residual, hrel[i]);
                int sj = hst[i];
                if (sj == OFEA_OK && !(hrel[i] <= o.rtol)) sj = OFEA_ERR_NOT_CONVERGED;
                if (sj != OFEA_OK) worst = sj;
            }
            st.status = worst;
            st.refinements = attempts;
            st.seconds = ms * 1e-3;
            st.kernel_launches = launches;
        }
    }
    if (case_stats)  // one entry per (variant, load case), load cases of a variant adjacent
        for (int i = 0; i < VJ; ++i) {
            ofea_solve_stats &st = case_stats[i];
            st = ofea_solve_stats{};
            st.status = hst[i];
            if (st.status == OFEA_OK && !(hrel[i] <= o.rtol)) st.status = OFEA_ERR_NOT_CONVERGED;
            st.iterations = iters_tot[i];
            st.rel_residual = hrel[i];
            st.refinements = attempts;
            st.seconds = ms * 1e-3;
            st.kernel_launches = launches;
        }
}

// A cooperative launch whose barrier expects one CTA more than it has: every
// wait runs out after limit_ms and the kernel reports it (*released = 0).
// Phase trace of the solver kernel: with max_phases > 0 every later launch
// records %globaltimer at its start and after each grid barrier (CTA 0,
// thread 0; at most max_phases barriers); 0 turns it off.
void batch_set_trace(ofea_batch *b, int max_phases) {
    if (max_phases < 0 || max_phases > (1 << 20)) fail(OFEA_ERR_INVALID_ARG, "batch: max_phases must be 0..2^20");
    OFEA_CUDA(cudaSetDevice(b->device));
    if (max_phases > 0) {
        b->trace.ensure((size_t)max_phases + 1);
        OFEA_CUDA(cudaMemsetAsync(b->trace.p, 0, sizeof(unsigned long long) * (max_phases + 1), b->stream));
    }
    b->trace_cap = max_phases > 0 ? max_phases + 1 : 0;
}

// Durations (ms) between consecutive records of the last traced launch, in
// barrier order; *count = how many there are (up to cap are written).
void batch_phase_times(ofea_batch *b, double *ms, int cap, int *count) {
    *count = 0;
    if (b->trace_cap == 0) fail(OFEA_ERR_STATE, "batch: tracing is off (ofea_batch_set_trace)");
    OFEA_CUDA(cudaSetDevice(b->device));
    std::vector<unsigned long long> t(b->trace_cap);
    OFEA_CUDA(cudaMemcpyAsync(t.data(), b->trace.p, sizeof(unsigned long long) * t.size(), cudaMemcpyDeviceToHost,
                              b->stream));
    OFEA_CUDA(cudaStreamSynchronize(b->stream));
    int n = 0;
    while (n + 1 < (int)t.size() && t[n] != 0 && t[n + 1] != 0) {
        if (ms && n < cap) ms[n] = (double)(t[n + 1] - t[n]) * 1e-6;
        ++n;
    }
    *count = n;
}

void barrier_probe(ofea_ctx *c, int limit_ms, int *released) {
    DevBuf<GridSync> gs;
    DevBuf<int> out;
    gs.ensure(1);
    out.ensure(1);
    cudaStream_t s = c->stream;
    OFEA_CUDA(cudaMemsetAsync(gs.p, 0, sizeof(GridSync), s));
    OFEA_CUDA(cudaMemsetAsync(out.p, 0xff, sizeof(int), s));
    unsigned extra = 1;
    unsigned long long lim = (unsigned long long)limit_ms * 1000000ull;
    void *args[] = {(void *)&gs.p, (void *)&extra, (void *)&lim, (void *)&out.p};
    OFEA_CUDA(cudaLaunchCooperativeKernel((const void *)k_barrier_probe, dim3(c->num_sms), dim3(64), args, 0, s));
    int h = -1;
    OFEA_CUDA(cudaMemcpyAsync(&h, out.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    OFEA_CUDA(cudaStreamSynchronize(s));
    *released = h;
}

}  // namespace ofea
