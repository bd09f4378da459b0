// On-device preconditioned conjugate gradients: the B200 replacement of the
// direct solves behind solution_api / solution_nl_api
// (src/linear_solution.cpp:17-137, MKL Pardiso / SuperLU dgssv).
//
// K is block-CSR with 3x3 blocks (one column index per 9 values).  The SpMV is
// a warp per block row; 27 lanes hold one (block-in-triple, entry) pair each,
// so a step streams 3 consecutive blocks (216 B FP64 / 108 B FP32) and the row
// sums reduce with 4 shuffles.  Each iteration is two fused kernels:
//   A: p <- z + beta p (neighbour values formed on the fly, owner writes p),
//      q = K p, per-CTA partial of p.q
//   B: u += alpha p, r -= alpha q, z = Dinv r (3x3 block-Jacobi), partials of
//      r.z and r.r
// Scalars (alpha, beta, convergence) are formed redundantly and identically
// by every CTA from the previous kernel's partials, in a fixed order: results
// are bitwise reproducible and no extra launches or host round trips are
// needed.  Iteration counters and flags live in device memory, so a chunk of
// iterations can be captured once as a CUDA graph and replayed; the host polls
// a pinned copy of the flags between chunks.
//
// MIXED: the same iteration in FP32 (values, vectors, inner dot products and
// their accumulation) plus a third kernel U that performs a reliable update
// when ||r32|| has dropped by ru_delta since the last one: the FP64 true
// residual r = f - K (x64 + x32) is formed from the FP64 matrix and replaces
// r32; x64 += x32 follows in the next A.  Convergence is only ever declared on
// that FP64 true residual.
#include <algorithm>
#include <chrono>
#include <cmath>

#include "ofea_internal.cuh"

namespace ofea {

// ---------------------------------------------------------------- helpers --

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block sum, result in every thread, fixed order.
template <class T>
__device__ __forceinline__ T block_sum(T v, T *sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    T s = 0;
#pragma unroll
    for (int w = 0; w < kWarpsPerBlock; ++w) s += sh[w];
    return s;
}

template <class T>
__device__ __forceinline__ T sum_partials(const T *P, int cnt, T *sh) {
    T s = 0;
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) s += P[i];
    return block_sum(s, sh);
}

// One block row of y = K x with 27 active lanes (sub = lane/9 picks every third
// block, e = lane%9 the entry).  Returns y_i in lane 3i (i = 0..2).
template <class V, class XF>
__device__ __forceinline__ V bsr3_row(int rb, int deg, const int *__restrict__ cols,
                                      const V *__restrict__ Kb, XF x) {
    const int lane = threadIdx.x & 31;
    const int sub = lane / 9, e = lane - 9 * sub, j = e % 3;
    V acc = 0;
    if (lane < 27) {
        const V *kv = Kb + 9L * rb + e;
        const int *cp = cols + rb;
        int p = sub;
        for (; p + 6 < deg; p += 9) {
            int c0 = cp[p], c1 = cp[p + 3], c2 = cp[p + 6];
            V k0 = kv[9L * p], k1 = kv[9L * (p + 3)], k2 = kv[9L * (p + 6)];
            V x0 = x(3 * c0 + j), x1 = x(3 * c1 + j), x2 = x(3 * c2 + j);
            acc = fma(k0, x0, acc);
            acc = fma(k1, x1, acc);
            acc = fma(k2, x2, acc);
        }
        for (; p < deg; p += 3) acc = fma(kv[9L * p], x(3 * cp[p] + j), acc);
    }
    V t1 = __shfl_down_sync(0xffffffffu, acc, 1);
    V t2 = __shfl_down_sync(0xffffffffu, acc, 2);
    acc = acc + t1 + t2;  // valid where j == 0
    V s1 = __shfl_down_sync(0xffffffffu, acc, 9);
    V s2 = __shfl_down_sync(0xffffffffu, acc, 18);
    return acc + s1 + s2;  // valid at lanes 0, 3, 6
}

__device__ __forceinline__ void block3_apply(const double *D, const double *v, double *o) {
    o[0] = D[0] * v[0] + D[1] * v[1] + D[2] * v[2];
    o[1] = D[3] * v[0] + D[4] * v[1] + D[5] * v[2];
    o[2] = D[6] * v[0] + D[7] * v[1] + D[8] * v[2];
}
__device__ __forceinline__ void block3_apply(const float *D, const float *v, float *o) {
    o[0] = D[0] * v[0] + D[1] * v[1] + D[2] * v[2];
    o[1] = D[3] * v[0] + D[4] * v[1] + D[5] * v[2];
    o[2] = D[6] * v[0] + D[7] * v[1] + D[8] * v[2];
}

// Device-resident solver state.
struct Flags {
    int done;    // 1: stop (converged, breakdown)
    int status;  // OFEA_OK / OFEA_ERR_BREAKDOWN
    int itA;     // iteration index read by A (written by B)
    int itB;     // iteration index read by B, U (written by A)
    int iters;   // completed iterations
    int updates; // reliable updates performed
    int pad[2];
};

// The stop flag is written by CTA 0 of some kernels while other CTAs of the
// same kernel may be starting: read it once per CTA and broadcast, so every
// thread of a CTA takes the same path before any barrier.
__device__ __forceinline__ bool cta_done(const Flags *fl) {
    __shared__ int s_done;
    if (threadIdx.x == 0) s_done = *(volatile const int *)&fl->done;
    __syncthreads();
    return s_done != 0;
}

// Partial arrays (per-CTA), offsets into one double buffer.
struct Parts {
    double *pq, *rz0, *rz1, *rr, *rrU, *ff;
    float *pq32, *rz32_0, *rz32_1, *rrB32;
    double *rref;  // [2]
    int G;         // CTAs of every reducing kernel
};

// ------------------------------------------------------------ plain SpMV --

__global__ void __launch_bounds__(kBlock) k_spmv64(int nfree, const int *__restrict__ rowptr,
                                                   const int *__restrict__ cols,
                                                   const double *__restrict__ Kb,
                                                   const double *__restrict__ x,
                                                   double *__restrict__ y) {
    const int lane = threadIdx.x & 31;
    const int nwarps = gridDim.x * kWarpsPerBlock;
    for (int r = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5); r < nfree; r += nwarps) {
        int rb = rowptr[r], deg = rowptr[r + 1] - rb;
        double v = bsr3_row(rb, deg, cols, Kb, [&](int k) { return x[k]; });
        if (lane < 9 && lane % 3 == 0) y[3L * r + lane / 3] = v;
    }
}

void spmv64(ofea_ctx *c, const double *d_x, double *d_y) {
    k_spmv64<<<grid_for(c, c->nfree, kWarpsPerBlock), kBlock, 0, c->stream>>>(
        c->nfree, c->rowptr.p, c->cols.p, c->Kb.p, d_x, d_y);
    OFEA_CHECK_LAUNCH();
}

// -------------------------------------------------------------- PCG FP64 --

// r = f - K u, z = Dinv r, partials r.z -> rz0, r.r -> rr, f.f -> ff.
__global__ void __launch_bounds__(kBlock) k_residual64(
    int nfree, const int *__restrict__ rowptr, const int *__restrict__ cols,
    const double *__restrict__ Kb, const double *__restrict__ Dinv, const double *__restrict__ f,
    const double *__restrict__ u, double *__restrict__ r, double *__restrict__ z, Parts P) {
    __shared__ double sh[kWarpsPerBlock];
    __shared__ double sr[kWarpsPerBlock][3];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = gridDim.x * kWarpsPerBlock;
    double prz = 0, prr = 0, pff = 0;
    for (int rw = blockIdx.x * kWarpsPerBlock + warp; rw < nfree; rw += nwarps) {
        int rb = rowptr[rw], deg = rowptr[rw + 1] - rb;
        double v = bsr3_row(rb, deg, cols, Kb, [&](int k) { return u[k]; });
        if (lane < 9 && lane % 3 == 0) {
            int i = lane / 3;
            double fi = f[3L * rw + i];
            double ri = fi - v;
            r[3L * rw + i] = ri;
            sr[warp][i] = ri;
            prr += ri * ri;
            pff += fi * fi;
        }
        __syncwarp();
        if (lane == 0) {
            double zz[3];
            block3_apply(Dinv + 9L * rw, sr[warp], zz);
            for (int i = 0; i < 3; ++i) {
                z[3L * rw + i] = zz[i];
                prz += sr[warp][i] * zz[i];
            }
        }
        __syncwarp();
    }
    double a = block_sum(prz, sh);
    double b = block_sum(prr, sh);
    double cf = block_sum(pff, sh);
    if (threadIdx.x == 0) {
        P.rz0[blockIdx.x] = a;
        P.rr[blockIdx.x] = b;
        P.ff[blockIdx.x] = cf;
    }
}

// Iteration kernel A (see file comment).  tol2 = (rtol ||f||)^2.
__global__ void __launch_bounds__(kBlock) k_pcg64_A(
    int nfree, const int *__restrict__ rowptr, const int *__restrict__ cols,
    const double *__restrict__ Kb, const double *__restrict__ z, const double *__restrict__ pA,
    double *__restrict__ pB, double *__restrict__ q, Parts P, Flags *fl, double tol2) {
    __shared__ double sh[kWarpsPerBlock];
    if (cta_done(fl)) return;
    const int k = fl->itA;
    const double *Pcur = (k & 1) ? P.rz1 : P.rz0;   // rz^(k)
    const double *Pprev = (k & 1) ? P.rz0 : P.rz1;  // rz^(k-1)
    double rr = sum_partials(P.rr, P.G, sh);
    double rz = sum_partials(Pcur, P.G, sh);
    double rzp = k > 0 ? sum_partials(Pprev, P.G, sh) : 1.0;
    if (rr <= tol2) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            fl->done = 1;
            fl->iters = k;
        }
        return;
    }
    const double beta = k > 0 ? rz / rzp : 0.0;
    // ping-pong: p_old = pA (k even) or pB; written to the other
    const double *pold = (k & 1) ? pB : pA;
    double *pnew = (k & 1) ? const_cast<double *>(pA) : pB;
    const int lane = threadIdx.x & 31;
    const int nwarps = gridDim.x * kWarpsPerBlock;
    double ppq = 0;
    for (int rw = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5); rw < nfree; rw += nwarps) {
        int rb = rowptr[rw], deg = rowptr[rw + 1] - rb;
        double v = bsr3_row(rb, deg, cols, Kb, [&](int kk) { return fma(beta, pold[kk], z[kk]); });
        if (lane < 9 && lane % 3 == 0) {
            long d = 3L * rw + lane / 3;
            double pn = fma(beta, pold[d], z[d]);
            pnew[d] = pn;
            q[d] = v;
            ppq += pn * v;
        }
    }
    double s = block_sum(ppq, sh);
    if (threadIdx.x == 0) P.pq[blockIdx.x] = s;
    if (blockIdx.x == 0 && threadIdx.x == 0) fl->itB = k;
}

__global__ void __launch_bounds__(kBlock) k_pcg64_B(
    int nfree, const double *__restrict__ Dinv, const double *__restrict__ pA,
    const double *__restrict__ pB, const double *__restrict__ q, double *__restrict__ u,
    double *__restrict__ r, double *__restrict__ z, Parts P, Flags *fl) {
    __shared__ double sh[kWarpsPerBlock];
    if (cta_done(fl)) return;
    const int k = fl->itB;
    const double *Pcur = (k & 1) ? P.rz1 : P.rz0;
    double *Pnext = (k & 1) ? P.rz0 : P.rz1;
    double pq = sum_partials(P.pq, P.G, sh);
    double rz = sum_partials(Pcur, P.G, sh);
    if (!(pq > 0.0) || !isfinite(pq)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            fl->done = 1;
            fl->status = OFEA_ERR_BREAKDOWN;
            fl->iters = k;
        }
        return;
    }
    const double alpha = rz / pq;
    const double *p = (k & 1) ? pA : pB;  // p^(k) = pnew of A(k)
    double prz = 0, prr = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nfree; i += gridDim.x * blockDim.x) {
        double rv[3], zz[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            long d = 3L * i + c;
            u[d] = fma(alpha, p[d], u[d]);
            rv[c] = fma(-alpha, q[d], r[d]);
            r[d] = rv[c];
        }
        block3_apply(Dinv + 9L * i, rv, zz);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            z[3L * i + c] = zz[c];
            prz += rv[c] * zz[c];
            prr += rv[c] * rv[c];
        }
    }
    double a = block_sum(prz, sh);
    double b = block_sum(prr, sh);
    if (threadIdx.x == 0) {
        Pnext[blockIdx.x] = a;
        P.rr[blockIdx.x] = b;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        fl->itA = k + 1;
        fl->iters = k + 1;
    }
}

// ------------------------------------------------------------- MIXED FP32 --

// Init: r64 = f - K64 x64; r32 = r64; z32 = Dinv32 r32; partials.
__global__ void __launch_bounds__(kBlock) k_mx_init(
    int nfree, const int *__restrict__ rowptr, const int *__restrict__ cols,
    const double *__restrict__ Kb, const float *__restrict__ Dinv32, const double *__restrict__ f,
    const double *__restrict__ x64, float *__restrict__ r32, float *__restrict__ z32, Parts P) {
    __shared__ double sh[kWarpsPerBlock];
    __shared__ float shf[kWarpsPerBlock];
    __shared__ float sr[kWarpsPerBlock][3];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = gridDim.x * kWarpsPerBlock;
    double prr = 0, pff = 0;
    float prz = 0;
    for (int rw = blockIdx.x * kWarpsPerBlock + warp; rw < nfree; rw += nwarps) {
        int rb = rowptr[rw], deg = rowptr[rw + 1] - rb;
        double v = bsr3_row(rb, deg, cols, Kb, [&](int k) { return x64[k]; });
        if (lane < 9 && lane % 3 == 0) {
            int i = lane / 3;
            double fi = f[3L * rw + i];
            double ri = fi - v;
            r32[3L * rw + i] = (float)ri;
            sr[warp][i] = (float)ri;
            prr += ri * ri;
            pff += fi * fi;
        }
        __syncwarp();
        if (lane == 0) {
            float zz[3];
            block3_apply(Dinv32 + 9L * rw, sr[warp], zz);
            for (int i = 0; i < 3; ++i) {
                z32[3L * rw + i] = zz[i];
                prz += sr[warp][i] * zz[i];
            }
        }
        __syncwarp();
    }
    double b = block_sum(prr, sh);
    double cf = block_sum(pff, sh);
    float a = block_sum(prz, shf);
    if (threadIdx.x == 0) {
        P.rz32_0[blockIdx.x] = a;
        P.rrU[blockIdx.x] = b;
        P.rrB32[blockIdx.x] = (float)b;
        P.ff[blockIdx.x] = cf;
    }
}

// Single CTA: rref[0] = ||r64|| after init.
__global__ void k_mx_init_ref(Parts P) {
    __shared__ double sh[kWarpsPerBlock];
    double rr = sum_partials(P.rrU, P.G, sh);
    if (threadIdx.x == 0) P.rref[0] = sqrt(rr);
}

// The reliable-update decision of iteration k, identical wherever evaluated.
__device__ __forceinline__ bool mx_update_due(const Parts &P, int k, double ftol, double delta,
                                              float *shf) {
    float rrB = sum_partials(P.rrB32, P.G, shf);
    double rn = sqrt((double)rrB);
    double ref = P.rref[k & 1];
    return rn < delta * ref || rn <= ftol;
}

__global__ void __launch_bounds__(kBlock) k_mx_A(
    int nfree, const int *__restrict__ rowptr, const int *__restrict__ cols,
    const float *__restrict__ Kb32, const float *__restrict__ z32, const float *__restrict__ pA,
    float *__restrict__ pB, float *__restrict__ q32, double *__restrict__ x64,
    float *__restrict__ x32, Parts P, Flags *fl, double ftol, double delta) {
    __shared__ double sh[kWarpsPerBlock];
    __shared__ float shf[kWarpsPerBlock];
    if (cta_done(fl)) return;
    const int k = fl->itA;
    // 1. did U(k-1) perform a reliable update?  (same decision U took)
    bool upd = false;
    double rr64 = 0;
    if (k > 0) {
        upd = mx_update_due(P, k - 1, ftol, delta, shf);
        if (upd) {
            for (long d = blockIdx.x * (long)blockDim.x + threadIdx.x; d < 3L * nfree;
                 d += (long)gridDim.x * blockDim.x) {
                x64[d] += (double)x32[d];
                x32[d] = 0.0f;
            }
            rr64 = sum_partials(P.rrU, P.G, sh);
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            P.rref[k & 1] = upd ? sqrt(rr64) : P.rref[(k - 1) & 1];
            if (upd) fl->updates += 1;
        }
        if (upd && sqrt(rr64) <= ftol) {
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                fl->done = 1;
                fl->iters = k;
            }
            return;
        }
    }
    const float *Pcur = (k & 1) ? P.rz32_1 : P.rz32_0;
    const float *Pprev = (k & 1) ? P.rz32_0 : P.rz32_1;
    float rz = sum_partials(Pcur, P.G, shf);
    float rzp = k > 0 ? sum_partials(Pprev, P.G, shf) : 1.0f;
    const float beta = k > 0 ? rz / rzp : 0.0f;
    const float *pold = (k & 1) ? pB : pA;
    float *pnew = (k & 1) ? const_cast<float *>(pA) : pB;
    const int lane = threadIdx.x & 31;
    const int nwarps = gridDim.x * kWarpsPerBlock;
    float ppq = 0;
    for (int rw = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5); rw < nfree; rw += nwarps) {
        int rb = rowptr[rw], deg = rowptr[rw + 1] - rb;
        float v = bsr3_row(rb, deg, cols, Kb32, [&](int kk) { return fmaf(beta, pold[kk], z32[kk]); });
        if (lane < 9 && lane % 3 == 0) {
            long d = 3L * rw + lane / 3;
            float pn = fmaf(beta, pold[d], z32[d]);
            pnew[d] = pn;
            q32[d] = v;
            ppq += pn * v;
        }
    }
    float s = block_sum(ppq, shf);
    if (threadIdx.x == 0) P.pq32[blockIdx.x] = s;
    if (blockIdx.x == 0 && threadIdx.x == 0) fl->itB = k;
}

__global__ void __launch_bounds__(kBlock) k_mx_B(
    int nfree, const float *__restrict__ Dinv32, const float *__restrict__ pA,
    const float *__restrict__ pB, const float *__restrict__ q32, float *__restrict__ x32,
    float *__restrict__ r32, float *__restrict__ z32, Parts P, Flags *fl) {
    __shared__ float shf[kWarpsPerBlock];
    if (cta_done(fl)) return;
    const int k = fl->itB;
    const float *Pcur = (k & 1) ? P.rz32_1 : P.rz32_0;
    float *Pnext = (k & 1) ? P.rz32_0 : P.rz32_1;
    float pq = sum_partials(P.pq32, P.G, shf);
    float rz = sum_partials(Pcur, P.G, shf);
    if (!(pq > 0.0f) || !isfinite(pq)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            fl->done = 1;
            fl->status = OFEA_ERR_BREAKDOWN;
            fl->iters = k;
        }
        return;
    }
    const float alpha = rz / pq;
    const float *p = (k & 1) ? pA : pB;
    float prz = 0, prr = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nfree; i += gridDim.x * blockDim.x) {
        float rv[3], zz[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            long d = 3L * i + c;
            x32[d] = fmaf(alpha, p[d], x32[d]);
            rv[c] = fmaf(-alpha, q32[d], r32[d]);
            r32[d] = rv[c];
        }
        block3_apply(Dinv32 + 9L * i, rv, zz);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            z32[3L * i + c] = zz[c];
            prz += rv[c] * zz[c];
            prr += rv[c] * rv[c];
        }
    }
    float a = block_sum(prz, shf);
    float b = block_sum(prr, shf);
    if (threadIdx.x == 0) {
        Pnext[blockIdx.x] = a;
        P.rrB32[blockIdx.x] = b;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        fl->itA = k + 1;
        fl->iters = k + 1;
    }
}

// Reliable update (when due): r64 = f - K64 (x64 + x32), r32 = r64, z32, partials.
__global__ void __launch_bounds__(kBlock) k_mx_U(
    int nfree, const int *__restrict__ rowptr, const int *__restrict__ cols,
    const double *__restrict__ Kb, const float *__restrict__ Dinv32, const double *__restrict__ f,
    const double *__restrict__ x64, const float *__restrict__ x32, float *__restrict__ r32,
    float *__restrict__ z32, Parts P, Flags *fl, double ftol, double delta) {
    __shared__ double sh[kWarpsPerBlock];
    __shared__ float shf[kWarpsPerBlock];
    __shared__ float sr[kWarpsPerBlock][3];
    if (cta_done(fl)) return;
    const int k = fl->itB;
    if (!mx_update_due(P, k, ftol, delta, shf)) return;
    float *Pnext = (k & 1) ? P.rz32_0 : P.rz32_1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = gridDim.x * kWarpsPerBlock;
    double prr = 0;
    float prz = 0;
    for (int rw = blockIdx.x * kWarpsPerBlock + warp; rw < nfree; rw += nwarps) {
        int rb = rowptr[rw], deg = rowptr[rw + 1] - rb;
        double v = bsr3_row(rb, deg, cols, Kb, [&](int kk) { return x64[kk] + (double)x32[kk]; });
        if (lane < 9 && lane % 3 == 0) {
            int i = lane / 3;
            double ri = f[3L * rw + i] - v;
            r32[3L * rw + i] = (float)ri;
            sr[warp][i] = (float)ri;
            prr += ri * ri;
        }
        __syncwarp();
        if (lane == 0) {
            float zz[3];
            block3_apply(Dinv32 + 9L * rw, sr[warp], zz);
            for (int i = 0; i < 3; ++i) {
                z32[3L * rw + i] = zz[i];
                prz += sr[warp][i] * zz[i];
            }
        }
        __syncwarp();
    }
    double b = block_sum(prr, sh);
    float a = block_sum(prz, shf);
    if (threadIdx.x == 0) {
        Pnext[blockIdx.x] = a;
        P.rrU[blockIdx.x] = b;
    }
}

// x64 += x32 (used when the loop stops on max_iter with a pending correction).
__global__ void k_mx_flush(long n, double *__restrict__ x64, float *__restrict__ x32) {
    for (long d = blockIdx.x * (long)blockDim.x + threadIdx.x; d < n; d += (long)gridDim.x * blockDim.x) {
        x64[d] += (double)x32[d];
        x32[d] = 0.0f;
    }
}

// Single CTA: final scalar reductions into out[0..] (FP64).
__global__ void k_final_norms(Parts P, double *out) {
    __shared__ double sh[kWarpsPerBlock];
    double rr = sum_partials(P.rr, P.G, sh);
    double ff = sum_partials(P.ff, P.G, sh);
    if (threadIdx.x == 0) {
        out[0] = rr;
        out[1] = ff;
    }
}

// ------------------------------------------------------------------- host --

namespace {

struct Workspace {
    Parts P;
    Flags *fl;
    double *scal;  // device scalars [4]
};

Workspace setup(ofea_ctx *c, int G) {
    SolverWork &w = c->w;
    // doubles: pq, rz0, rz1, rr, rrU, ff (6 G) + rref 2 + scal 4; floats: 4 G
    size_t nd = 6 * (size_t)kMaxGrid + 8 + 2 * (size_t)kMaxGrid;  // floats packed as doubles
    w.partials.ensure(nd);
    w.flags.ensure(sizeof(Flags) / sizeof(int));
    double *b = w.partials.p;
    Workspace ws;
    ws.P.pq = b;
    ws.P.rz0 = b + kMaxGrid;
    ws.P.rz1 = b + 2 * kMaxGrid;
    ws.P.rr = b + 3 * kMaxGrid;
    ws.P.rrU = b + 4 * kMaxGrid;
    ws.P.ff = b + 5 * kMaxGrid;
    ws.P.rref = b + 6 * kMaxGrid;
    ws.scal = b + 6 * kMaxGrid + 2;
    float *fb = reinterpret_cast<float *>(b + 6 * kMaxGrid + 8);
    ws.P.pq32 = fb;
    ws.P.rz32_0 = fb + kMaxGrid;
    ws.P.rz32_1 = fb + 2 * kMaxGrid;
    ws.P.rrB32 = fb + 3 * kMaxGrid;
    ws.P.G = G;
    ws.fl = reinterpret_cast<Flags *>(w.flags.p);
    OFEA_CUDA(cudaMemsetAsync(w.partials.p, 0, nd * sizeof(double), c->stream));
    OFEA_CUDA(cudaMemsetAsync(w.flags.p, 0, sizeof(Flags), c->stream));
    w.hflags.ensure(sizeof(Flags) / sizeof(int));
    w.hscal.ensure(4);
    return ws;
}

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Runs `chunk(iters)` repeatedly (optionally as a captured graph) until the
// device flags say done, max_iter is reached or the time budget runs out.
template <class ChunkFn>
void drive(ofea_ctx *c, const ofea_solve_opts &o, Workspace &ws, int per_chunk, ChunkFn chunk,
           Flags &hf, long long &launches, int kernels_per_iter, bool &timed_out) {
    cudaStream_t s = c->stream;
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    if (o.use_graph) {
        OFEA_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        chunk(per_chunk);
        cudaError_t e = cudaStreamEndCapture(s, &graph);
        if (e != cudaSuccess) fail_cuda(e, "cudaStreamEndCapture", __FILE__, __LINE__);
        e = cudaGraphInstantiate(&exec, graph, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(graph);
            fail_cuda(e, "cudaGraphInstantiate", __FILE__, __LINE__);
        }
    }
    const double t0 = now_s();
    int launched = 0;
    timed_out = false;
    Flags *h = reinterpret_cast<Flags *>(c->w.hflags.p);
    try {
        while (true) {
            if (exec)
                OFEA_CUDA(cudaGraphLaunch(exec, s));
            else
                chunk(per_chunk);
            launched += per_chunk;
            launches += (long long)per_chunk * kernels_per_iter;
            OFEA_CUDA(cudaMemcpyAsync(h, ws.fl, sizeof(Flags), cudaMemcpyDeviceToHost, s));
            OFEA_CUDA(cudaStreamSynchronize(s));
            if (h->done || launched >= o.max_iter) break;
            if (o.time_budget_s > 0 && now_s() - t0 > o.time_budget_s) {
                timed_out = true;
                break;
            }
        }
    } catch (...) {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        throw;
    }
    hf = *h;
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
}

}  // namespace

void solve_device(ofea_ctx *c, const double *d_f, double *d_u, const ofea_solve_opts &o,
                  ofea_solve_stats &st) {
    cudaStream_t s = c->stream;
    const int n = c->n, nf = c->nfree;
    if (n == 0) {
        st.status = OFEA_OK;
        return;
    }
    const int G = std::min(kMaxGrid, c->num_sms * (2048 / kBlock));
    Workspace ws = setup(c, G);
    SolverWork &w = c->w;
    cudaEvent_t e0, e1;
    OFEA_CUDA(cudaEventCreate(&e0));
    OFEA_CUDA(cudaEventCreate(&e1));
    OFEA_CUDA(cudaEventRecord(e0, s));
    int per_chunk = o.check_every > 0 ? o.check_every : 16;
    per_chunk = std::max(1, std::min(per_chunk, o.max_iter));
    long long launches = 0;
    Flags hf{};
    bool timed_out = false;
    double rel = 0;
    int total_iters = 0, refinements = 0;

    if (o.method == OFEA_SOLVER_PCG64) {
        w.r.ensure(n);
        w.z.ensure(n);
        w.q.ensure(n);
        w.p0.ensure(n);
        w.p1.ensure(n);
        for (int restart = 0; restart < 8; ++restart) {
            OFEA_CUDA(cudaMemsetAsync(w.p0.p, 0, sizeof(double) * n, s));
            OFEA_CUDA(cudaMemsetAsync(w.p1.p, 0, sizeof(double) * n, s));
            OFEA_CUDA(cudaMemsetAsync(ws.fl, 0, sizeof(Flags), s));
            k_residual64<<<G, kBlock, 0, s>>>(nf, c->rowptr.p, c->cols.p, c->Kb.p, c->Dinv.p, d_f,
                                               d_u, w.r.p, w.z.p, ws.P);
            OFEA_CHECK_LAUNCH();
            k_final_norms<<<1, kBlock, 0, s>>>(ws.P, ws.scal);
            OFEA_CUDA(cudaMemcpyAsync(w.hscal.p, ws.scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
            OFEA_CUDA(cudaStreamSynchronize(s));
            launches += 2;
            double rr = w.hscal.p[0], ff = w.hscal.p[1];
            if (ff == 0.0) {
                OFEA_CUDA(cudaMemsetAsync(d_u, 0, sizeof(double) * n, s));
                rel = 0;
                break;
            }
            rel = std::sqrt(rr / ff);
            if (rel <= o.rtol || total_iters >= o.max_iter || timed_out) break;
            ++refinements;
            // recursive residual target a little below rtol, true residual re-checked
            const double tol2 = (0.5 * o.rtol) * (0.5 * o.rtol) * ff;
            ofea_solve_opts oo = o;
            oo.max_iter = o.max_iter - total_iters;
            auto chunk = [&](int iters) {
                for (int it = 0; it < iters; ++it) {
                    k_pcg64_A<<<G, kBlock, 0, s>>>(nf, c->rowptr.p, c->cols.p, c->Kb.p, w.z.p, w.p0.p,
                                                   w.p1.p, w.q.p, ws.P, ws.fl, tol2);
                    k_pcg64_B<<<G, kBlock, 0, s>>>(nf, c->Dinv.p, w.p0.p, w.p1.p, w.q.p, d_u, w.r.p,
                                                   w.z.p, ws.P, ws.fl);
                }
                OFEA_CHECK_LAUNCH();
            };
            drive(c, oo, ws, per_chunk, chunk, hf, launches, 2, timed_out);
            total_iters += hf.iters;
            if (hf.status == OFEA_ERR_BREAKDOWN) break;
        }
    } else if (o.method == OFEA_SOLVER_MIXED) {
        if (!c->K32_ok) build_fp32_copy(c);
        w.r32.ensure(n);
        w.z32.ensure(n);
        w.q32.ensure(n);
        w.p32a.ensure(n);
        w.p32b.ensure(n);
        w.x32.ensure(n);
        w.r.ensure(n);
        w.z.ensure(n);
        const double delta = o.ru_delta > 0 ? o.ru_delta : 0.1;
        for (int restart = 0; restart < 8; ++restart) {
            OFEA_CUDA(cudaMemsetAsync(w.p32a.p, 0, sizeof(float) * n, s));
            OFEA_CUDA(cudaMemsetAsync(w.p32b.p, 0, sizeof(float) * n, s));
            OFEA_CUDA(cudaMemsetAsync(w.x32.p, 0, sizeof(float) * n, s));
            OFEA_CUDA(cudaMemsetAsync(ws.fl, 0, sizeof(Flags), s));
            k_mx_init<<<G, kBlock, 0, s>>>(nf, c->rowptr.p, c->cols.p, c->Kb.p, c->Dinv32.p, d_f, d_u,
                                           w.r32.p, w.z32.p, ws.P);
            OFEA_CHECK_LAUNCH();
            k_mx_init_ref<<<1, kBlock, 0, s>>>(ws.P);
            // ||f||^2 and ||r||^2 for the host
            OFEA_CUDA(cudaMemcpyAsync(ws.P.rr, ws.P.rrU, sizeof(double) * G, cudaMemcpyDeviceToDevice, s));
            k_final_norms<<<1, kBlock, 0, s>>>(ws.P, ws.scal);
            OFEA_CUDA(cudaMemcpyAsync(w.hscal.p, ws.scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
            OFEA_CUDA(cudaStreamSynchronize(s));
            launches += 3;
            double rr = w.hscal.p[0], ff = w.hscal.p[1];
            if (ff == 0.0) {
                OFEA_CUDA(cudaMemsetAsync(d_u, 0, sizeof(double) * n, s));
                rel = 0;
                break;
            }
            rel = std::sqrt(rr / ff);
            if (rel <= o.rtol || total_iters >= o.max_iter || timed_out) break;
            ++refinements;
            const double ftol = o.rtol * std::sqrt(ff);
            ofea_solve_opts oo = o;
            oo.max_iter = o.max_iter - total_iters;
            auto chunk = [&](int iters) {
                for (int it = 0; it < iters; ++it) {
                    k_mx_A<<<G, kBlock, 0, s>>>(nf, c->rowptr.p, c->cols.p, c->Kb32.p, w.z32.p, w.p32a.p,
                                                w.p32b.p, w.q32.p, d_u, w.x32.p, ws.P, ws.fl, ftol, delta);
                    k_mx_B<<<G, kBlock, 0, s>>>(nf, c->Dinv32.p, w.p32a.p, w.p32b.p, w.q32.p, w.x32.p,
                                                w.r32.p, w.z32.p, ws.P, ws.fl);
                    k_mx_U<<<G, kBlock, 0, s>>>(nf, c->rowptr.p, c->cols.p, c->Kb.p, c->Dinv32.p, d_f, d_u,
                                                w.x32.p, w.r32.p, w.z32.p, ws.P, ws.fl, ftol, delta);
                }
                OFEA_CHECK_LAUNCH();
            };
            drive(c, oo, ws, per_chunk, chunk, hf, launches, 3, timed_out);
            total_iters += hf.iters;
            refinements += hf.updates;
            k_mx_flush<<<grid_for(c, n, kBlock), kBlock, 0, s>>>(n, d_u, w.x32.p);
            OFEA_CHECK_LAUNCH();
            launches += 1;
            if (hf.status == OFEA_ERR_BREAKDOWN) break;
        }
    } else {
        fail(OFEA_ERR_UNKNOWN_SOLVER, "unknown solver method " + std::to_string(o.method));
    }
    OFEA_CUDA(cudaEventRecord(e1, s));
    OFEA_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    OFEA_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    st.iterations = total_iters;
    st.refinements = refinements;
    st.rel_residual = rel;
    st.seconds = ms * 1e-3;
    st.kernel_launches = launches;
    if (hf.status == OFEA_ERR_BREAKDOWN)
        st.status = OFEA_ERR_BREAKDOWN;
    else if (!(rel <= o.rtol))
        st.status = timed_out ? OFEA_ERR_TIMEOUT : OFEA_ERR_NOT_CONVERGED;
    else
        st.status = OFEA_OK;
}

void profile_kernels(ofea_ctx *c, int method, int reps, double *ms, double *bytes) {
    cudaStream_t s = c->stream;
    const int n = c->n, nf = c->nfree;
    const int G = std::min(kMaxGrid, c->num_sms * (2048 / kBlock));
    Workspace ws = setup(c, G);
    SolverWork &w = c->w;
    // iteration 1 with beta != 0 paths; the vectors hold the last solve's state
    Flags f0{};
    f0.itA = 1;
    f0.itB = 1;
    OFEA_CUDA(cudaMemcpyAsync(ws.fl, &f0, sizeof(Flags), cudaMemcpyHostToDevice, s));
    double one = 1.0;
    for (int i = 0; i < G; ++i) {
        OFEA_CUDA(cudaMemcpyAsync(ws.P.pq + i, &one, sizeof(double), cudaMemcpyHostToDevice, s));
        OFEA_CUDA(cudaMemcpyAsync(ws.P.rz0 + i, &one, sizeof(double), cudaMemcpyHostToDevice, s));
        OFEA_CUDA(cudaMemcpyAsync(ws.P.rz1 + i, &one, sizeof(double), cudaMemcpyHostToDevice, s));
        OFEA_CUDA(cudaMemcpyAsync(ws.P.rr + i, &one, sizeof(double), cudaMemcpyHostToDevice, s));
    }
    std::vector<float> onesf(4 * kMaxGrid, 1.0f);
    OFEA_CUDA(cudaMemcpyAsync(ws.P.pq32, onesf.data(), sizeof(float) * 4 * kMaxGrid, cudaMemcpyHostToDevice, s));
    const double nnzv = 9.0 * c->nnzb;
    cudaEvent_t e0, e1, e2;
    OFEA_CUDA(cudaEventCreate(&e0));
    OFEA_CUDA(cudaEventCreate(&e1));
    OFEA_CUDA(cudaEventCreate(&e2));
    if (method == OFEA_SOLVER_PCG64) {
        if (!w.z.p || w.z.n < (size_t)n || !w.p1.p) fail(OFEA_ERR_STATE, "run a GPU_PCG solve first");
        double tol2 = -1.0;  // never converged: every launch does the full work
        OFEA_CUDA(cudaEventRecord(e0, s));
        for (int i = 0; i < reps; ++i)
            k_pcg64_A<<<G, kBlock, 0, s>>>(nf, c->rowptr.p, c->cols.p, c->Kb.p, w.z.p, w.p0.p, w.p1.p,
                                           w.q.p, ws.P, ws.fl, tol2);
        OFEA_CUDA(cudaEventRecord(e1, s));
        for (int i = 0; i < reps; ++i)
            k_pcg64_B<<<G, kBlock, 0, s>>>(nf, c->Dinv.p, w.p0.p, w.p1.p, w.q.p, w.u.p ? w.u.p : w.t.p,
                                           w.r.p, w.z.p, ws.P, ws.fl);
        OFEA_CUDA(cudaEventRecord(e2, s));
        bytes[0] = 8 * nnzv + 4.0 * c->nnzb + 4.0 * (nf + 1) + 8.0 * n * 4;  // K, cols, rowptr, z, p_old, p_new, q
        bytes[1] = 72.0 * nf + 8.0 * n * 7;  // Dinv; u r/w, r r/w, p, q, z
    } else {
        if (!w.z32.p || w.z32.n < (size_t)n || !c->K32_ok) fail(OFEA_ERR_STATE, "run a GPU_MIXED solve first");
        OFEA_CUDA(cudaEventRecord(e0, s));
        for (int i = 0; i < reps; ++i)
            k_mx_A<<<G, kBlock, 0, s>>>(nf, c->rowptr.p, c->cols.p, c->Kb32.p, w.z32.p, w.p32a.p, w.p32b.p,
                                        w.q32.p, w.t.p, w.x32.p, ws.P, ws.fl, -1.0, 0.0);
        OFEA_CUDA(cudaEventRecord(e1, s));
        for (int i = 0; i < reps; ++i)
            k_mx_B<<<G, kBlock, 0, s>>>(nf, c->Dinv32.p, w.p32a.p, w.p32b.p, w.q32.p, w.x32.p, w.r32.p,
                                        w.z32.p, ws.P, ws.fl);
        OFEA_CUDA(cudaEventRecord(e2, s));
        bytes[0] = 4 * nnzv + 4.0 * c->nnzb + 4.0 * (nf + 1) + 4.0 * n * 4;
        bytes[1] = 36.0 * nf + 4.0 * n * 7;  // Dinv32; x r/w, r r/w, p, q, z
    }
    OFEA_CHECK_LAUNCH();
    OFEA_CUDA(cudaEventSynchronize(e2));
    float a = 0, b = 0;
    OFEA_CUDA(cudaEventElapsedTime(&a, e0, e1));
    OFEA_CUDA(cudaEventElapsedTime(&b, e1, e2));
    ms[0] = a / reps;
    ms[1] = b / reps;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
}

}  // namespace ofea
