// On-device Krylov solvers: the B200 replacement of the direct solves behind
// solution_api / solution_nl_api (src/linear_solution.cpp:17-137, MKL Pardiso /
// SuperLU dgssv).
//
// PCG64 (plain): FP64 conjugate gradients with 3x3 block-Jacobi.  Two fused
// kernels per iteration over the BSELL-32 matrix (sell.cuh):
//   A: p <- z + beta p (neighbour values formed on the fly, the owner writes
//      p), q = K p, per-CTA partial of p.q
//   B: u += alpha p, r -= alpha q, z = Dinv r, partials of r.z and r.r
//
// MIXED: FP64 flexible CG (Polak-Ribiere beta) whose preconditioner is the
// FP32 two-level V(1,1) cycle of precond.cu.  FP64: K for the outer SpMV, the
// residual recursion r -= alpha K p, the update u += alpha p and every outer
// reduction.  FP32 with FP32 accumulation: the smoother's and the residual's
// SpMV, the block-Jacobi smoother, the restriction and the coarse GEMV.
// Kernels per iteration: A, B (+ pre-smoothing), residual, restriction, GEMV,
// prolongation, post-smoothing (+ the r.z dots).
//
// Scalars (alpha, beta, convergence) are formed redundantly and identically
// by every CTA from the previous kernel's partials, in a fixed order: results
// are bitwise reproducible and no host round trip is needed per iteration.
// Iteration counters and flags live in device memory, so a chunk of
// iterations is captured once as a CUDA graph and replayed; the host polls a
// pinned copy of the flags between chunks.  Convergence is confirmed on a
// freshly computed FP64 residual f - K u before a solve returns.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <functional>

#include "precond.cuh"
#include "sell.cuh"
#include "solver_common.cuh"

namespace ofea {

// The BSELL SpMV kernels are latency bound (a gather per block): they are
// compiled for full occupancy (8 CTAs of 256 threads per SM, 32 registers),
// measured on the B200 at 79 % of HBM peak for the FP64 outer SpMV against
// 69 % at the 48 registers the compiler picks on its own.
constexpr int kSpmvCtas = 2048 / kBlock;

// ---------------------------------------------------------- plain SpMV --

__global__ void __launch_bounds__(kBlock, kSpmvCtas) k_spmv64(int nfree, const int *__restrict__ sl_ptr,
                                                   const int *__restrict__ scols,
                                                   const double *__restrict__ sv64,
                                                   const double *__restrict__ x,
                                                   double *__restrict__ y) {
    for_each_sell_row(nfree, sl_ptr, [&](int r, long S, int t, int W) {
        double v[3];
        sell_row<double, 2>(S, t, W, scols, sv64, [&](int k) { return x[k]; }, v[0], v[1], v[2]);
        for (int i = 0; i < 3; ++i) y[3L * r + i] = v[i];
    });
}

static int sell_grid(const ofea_ctx *c) {
    return grid_for(c, (c->nfree + kSlice - 1) / kSlice, kBlock / kSlice);
}

void spmv64(ofea_ctx *c, const double *d_x, double *d_y) {
    k_spmv64<<<sell_grid(c), kBlock, 0, c->stream>>>(c->nfree, c->sl_ptr.p, c->scols.p, c->sv64.p, d_x, d_y);
    OFEA_CHECK_LAUNCH();
}

// ------------------------------------------------------------ PCG FP64 --

// r = f - K u, z = Dinv r; partials r.z -> rz0, r.r -> rr, f.f -> ff.
__global__ void __launch_bounds__(kBlock, kSpmvCtas) k_residual64(
    int nfree, const int *__restrict__ sl_ptr, const int *__restrict__ scols,
    const double *__restrict__ sv64, const double *__restrict__ Dinv, const double *__restrict__ f,
    const double *__restrict__ u, double *__restrict__ r, double *__restrict__ z, Parts P) {
    __shared__ double sh[kWarpsPerBlock];
    double prz = 0, prr = 0, pff = 0;
    for_each_sell_row(nfree, sl_ptr, [&](int rw, long S, int t, int W) {
        double y[3], rv[3], zz[3];
        sell_row<double, 2>(S, t, W, scols, sv64, [&](int k) { return u[k]; }, y[0], y[1], y[2]);
        for (int i = 0; i < 3; ++i) {
            const double fi = f[3L * rw + i];
            rv[i] = fi - y[i];
            r[3L * rw + i] = rv[i];
            prr += rv[i] * rv[i];
            pff += fi * fi;
        }
        block3_apply(Dinv + 9L * rw, rv, zz);
        for (int i = 0; i < 3; ++i) {
            z[3L * rw + i] = zz[i];
            prz += rv[i] * zz[i];
        }
    });
    double a = block_sum(prz, sh);
    double b = block_sum(prr, sh);
    double cf = block_sum(pff, sh);
    if (threadIdx.x == 0) {
        P.rz0[blockIdx.x] = a;
        P.rr[blockIdx.x] = b;
        P.ff[blockIdx.x] = cf;
    }
}

// Iteration kernel A: p = z + beta p_old, q = K p as K z + beta q_old, partial
// p.q.  tol2 = (target ||r||)^2.
__global__ void __launch_bounds__(kBlock, kSpmvCtas) k_pcg64_A(
    int nfree, const int *__restrict__ sl_ptr, const int *__restrict__ scols,
    const double *__restrict__ sv64, const double *__restrict__ z, double *__restrict__ pA,
    double *__restrict__ pB, double *__restrict__ q, Parts P, Flags *fl, double tol2) {
    __shared__ double sh[kWarpsPerBlock];
    if (cta_done(fl)) return;
    const int k = fl->itA;
    const double *Pcur = (k & 1) ? P.rz1 : P.rz0;   // rz^(k)
    const double *Pprev = (k & 1) ? P.rz0 : P.rz1;  // rz^(k-1)
    const double rr = sum_partials(P.rr, P.G, sh);
    const double rz = sum_partials(Pcur, P.G, sh);
    const double rzp = k > 0 ? sum_partials(Pprev, P.G, sh) : 1.0;
    if (rr <= tol2) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            fl->done = 1;
            fl->iters = k;
        }
        return;
    }
    const double beta = k > 0 ? rz / rzp : 0.0;
    const double *pold = (k & 1) ? pB : pA;
    double *pnew = (k & 1) ? pA : pB;
    double ppq = 0;
    for_each_sell_row(nfree, sl_ptr, [&](int rw, long S, int t, int W) {
        double y[3];
        sell_row<double, 2>(S, t, W, scols, sv64, [&](int kk) { return z[kk]; }, y[0], y[1], y[2]);
        for (int i = 0; i < 3; ++i) {
            const long d = 3L * rw + i;
            const double pn = fma(beta, pold[d], z[d]);
            const double qn = fma(beta, q[d], y[i]);  // K p = K z + beta K p_old
            pnew[d] = pn;
            q[d] = qn;
            ppq += pn * qn;
        }
    });
    const double s = block_sum(ppq, sh);
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
    const double pq = sum_partials(P.pq, P.G, sh);
    const double rz = sum_partials(Pcur, P.G, sh);
    if (!(pq > 0.0) || !isfinite(pq)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            fl->done = 1;
            fl->status = OFEA_ERR_BREAKDOWN;
            fl->iters = k;
        }
        return;
    }
    const double alpha = rz / pq;
    const double *p = (k & 1) ? pA : pB;  // written by A(k)
    double prz = 0, prr = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nfree; i += gridDim.x * blockDim.x) {
        double rv[3], zz[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const long d = 3L * i + c;
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
    const double a = block_sum(prz, sh);
    const double b = block_sum(prr, sh);
    if (threadIdx.x == 0) {
        Pnext[blockIdx.x] = a;
        P.rr[blockIdx.x] = b;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        fl->itA = k + 1;
        fl->iters = k + 1;
    }
}

// --------------------------------------------------- MIXED: FP64 FCG --

// Outer A: beta (Polak-Ribiere) from the post-smoothing partials,
// p <- double(z_k) + beta p, q = K64 p as K64 z + beta q (the SpMV gathers z
// alone; drift of q from K p is caught by the FP64 true-residual check),
// partial p.q.
__global__ void __launch_bounds__(kBlock, kSpmvCtas) k_fcg_A(
    int nfree, const int *__restrict__ sl_ptr, const int *__restrict__ scols,
    const double *__restrict__ sv64, const float *__restrict__ zA, const float *__restrict__ zB,
    double *__restrict__ pA, double *__restrict__ pB, double *__restrict__ q, Parts P, Flags *fl,
    double tol2) {
    __shared__ double sh[kWarpsPerBlock];
    if (cta_done(fl)) return;
    const int k = fl->itA;
    const double rr = sum_partials(P.rr, P.G, sh);
    if (rr <= tol2) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            fl->done = 1;
            fl->iters = k;
        }
        return;
    }
    double beta = 0.0;
    if (k > 0) {
        const double rz = sum_partials((k & 1) ? P.rz1 : P.rz0, P.G, sh);   // r_k . z_k
        const double rzp = sum_partials((k & 1) ? P.rz0 : P.rz1, P.G, sh);  // r_{k-1} . z_{k-1}
        const double rzo = sum_partials(P.rzo, P.G, sh);                    // r_k . z_{k-1}
        beta = (rz - rzo) / rzp;
    }
    const float *z = (k & 1) ? zB : zA;
    const double *pold = (k & 1) ? pB : pA;
    double *pnew = (k & 1) ? pA : pB;
    double ppq = 0;
    for_each_sell_row(nfree, sl_ptr, [&](int rw, long S, int t, int W) {
        double y[3];
        sell_row<double, 2>(S, t, W, scols, sv64, [&](int kk) { return (double)z[kk]; }, y[0], y[1], y[2]);
        for (int i = 0; i < 3; ++i) {
            const long d = 3L * rw + i;
            const double pn = fma(beta, pold[d], (double)z[d]);
            const double qn = fma(beta, q[d], y[i]);  // K p = K z + beta K p_old
            pnew[d] = pn;
            q[d] = qn;
            ppq += pn * qn;
        }
    });
    const double s = block_sum(ppq, sh);
    if (threadIdx.x == 0) P.pq[blockIdx.x] = s;
    if (blockIdx.x == 0 && threadIdx.x == 0) fl->itB = k;
}

// Outer B: u += alpha p, r -= alpha q (FP64), ||r||^2, then the start of the
// preconditioner: b32 = float(r), x32 = w Dinv32 b32 (pre-smoothing).
__global__ void __launch_bounds__(kBlock) k_fcg_B(
    int nfree, const float *__restrict__ Dinv32, float w, const double *__restrict__ pA,
    const double *__restrict__ pB, const double *__restrict__ q, double *__restrict__ u,
    double *__restrict__ r, float *__restrict__ b32, float *__restrict__ x32, Parts P, Flags *fl) {
    __shared__ double sh[kWarpsPerBlock];
    if (cta_done(fl)) return;
    const int k = fl->itB;
    const double pq = sum_partials(P.pq, P.G, sh);
    const double rz = sum_partials((k & 1) ? P.rz1 : P.rz0, P.G, sh);
    if (!(pq > 0.0) || !isfinite(pq)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            fl->done = 1;
            fl->status = OFEA_ERR_BREAKDOWN;
            fl->iters = k;
        }
        return;
    }
    const double alpha = rz / pq;
    const double *p = (k & 1) ? pA : pB;
    double prr = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nfree; i += gridDim.x * blockDim.x) {
        float b[3], x[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const long d = 3L * i + c;
            u[d] = fma(alpha, p[d], u[d]);
            const double rv = fma(-alpha, q[d], r[d]);
            r[d] = rv;
            prr += rv * rv;
            b[c] = (float)rv;
        }
        block3_apply(Dinv32 + 9L * i, b, x);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            b32[3L * i + c] = b[c];
            x32[3L * i + c] = w * x[c];
        }
    }
    const double s = block_sum(prr, sh);
    if (threadIdx.x == 0) P.rr[blockIdx.x] = s;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        fl->itA = k + 1;
        fl->iters = k + 1;
    }
}

// Init for MIXED: r = f - K64 u (FP64), ||r||^2, ||f||^2, b32, x32 pre-smoothing.
__global__ void __launch_bounds__(kBlock, kSpmvCtas) k_fcg_init(
    int nfree, const int *__restrict__ sl_ptr, const int *__restrict__ scols,
    const double *__restrict__ sv64, const float *__restrict__ Dinv32, float w,
    const double *__restrict__ f, const double *__restrict__ u, double *__restrict__ r,
    float *__restrict__ b32, float *__restrict__ x32, Parts P) {
    __shared__ double sh[kWarpsPerBlock];
    double prr = 0, pff = 0;
    for_each_sell_row(nfree, sl_ptr, [&](int rw, long S, int t, int W) {
        double y[3];
        float b[3], x[3];
        sell_row<double, 2>(S, t, W, scols, sv64, [&](int k) { return u[k]; }, y[0], y[1], y[2]);
        for (int i = 0; i < 3; ++i) {
            const double fi = f[3L * rw + i];
            const double rv = fi - y[i];
            r[3L * rw + i] = rv;
            prr += rv * rv;
            pff += fi * fi;
            b[i] = (float)rv;
        }
        block3_apply(Dinv32 + 9L * rw, b, x);
        for (int i = 0; i < 3; ++i) {
            b32[3L * rw + i] = b[i];
            x32[3L * rw + i] = w * x[i];
        }
    });
    const double b = block_sum(prr, sh);
    const double cf = block_sum(pff, sh);
    if (threadIdx.x == 0) {
        P.rr[blockIdx.x] = b;
        P.ff[blockIdx.x] = cf;
    }
}

// Post-smoothing and the end of the preconditioner:
// z_{k+1} = x + w Dinv32 (b32 - K32 x); partials r.z_{k+1} and r.z_k (FP64).
// k = itB (itB = -1 for the initial application).
__global__ void __launch_bounds__(kBlock, kSpmvCtas) k_fcg_post(
    int nfree, const int *__restrict__ sl_ptr, const int *__restrict__ scols,
    const int *__restrict__ sl_g, const __nv_bfloat16 *__restrict__ svg, const float *__restrict__ Dinv32, float w,
    const float *__restrict__ b32, const float *__restrict__ x32, const double *__restrict__ r,
    float *__restrict__ zA, float *__restrict__ zB, Parts P, Flags *fl) {
    __shared__ double sh[kWarpsPerBlock];
    if (cta_done(fl)) return;
    const int k = fl->itB;
    float *znew = ((k + 1) & 1) ? zB : zA;
    const float *zold = ((k + 1) & 1) ? zA : zB;
    double *Pnext = ((k + 1) & 1) ? P.rz1 : P.rz0;
    double prz = 0, przo = 0;
    for_each_sell_row(nfree, sl_ptr, [&](int rw, long S, int t, int W) {
        float y[3], d[3], o[3];
        sell_row_g4(S, sl_g[rw / kSlice], t, W, scols, svg, [&](int kk) { return x32[kk]; }, y[0], y[1], y[2]);
        for (int i = 0; i < 3; ++i) d[i] = b32[3L * rw + i] - y[i];
        block3_apply(Dinv32 + 9L * rw, d, o);
        for (int i = 0; i < 3; ++i) {
            const long dd = 3L * rw + i;
            const float zn = fmaf(w, o[i], x32[dd]);
            const double rv = r[dd];
            prz += rv * (double)zn;
            przo += rv * (double)zold[dd];
            znew[dd] = zn;
        }
    });
    const double a = block_sum(prz, sh);
    const double b = block_sum(przo, sh);
    if (threadIdx.x == 0) {
        Pnext[blockIdx.x] = a;
        P.rzo[blockIdx.x] = b;
    }
}

// Single CTA: final reductions of rr and ff into out[0..1].
__global__ void k_final_norms(Parts P, double *out) {
    __shared__ double sh[kWarpsPerBlock];
    const double rr = sum_partials(P.rr, P.G, sh);
    const double ff = sum_partials(P.ff, P.G, sh);
    if (threadIdx.x == 0) {
        out[0] = rr;
        out[1] = ff;
    }
}

__global__ void k_set_itB(Flags *fl, int v) { fl->itB = v; }

// ------------------------------------------------------------------- host --

void setup_marks_clear(ofea_ctx *c) {
    for (auto &m : c->setup_marks) cudaEventDestroy(m.second);
    c->setup_marks.clear();
}

void setup_mark(ofea_ctx *c, const char *phase) {
    if (!c->setup_trace) return;
    cudaEvent_t e = nullptr;
    OFEA_CUDA(cudaEventCreate(&e));
    c->setup_marks.emplace_back(phase, e);
    OFEA_CUDA(cudaEventRecord(e, c->stream));
}

namespace {

struct Workspace {
    Parts P;
    Flags *fl;
    double *scal;  // device scalars [4]
};

Workspace setup(ofea_ctx *c, int G) {
    SolverWork &w = c->w;
    const size_t nd = 6 * (size_t)kMaxGrid + 8;
    w.partials.ensure(nd);
    w.flags.ensure(sizeof(Flags) / sizeof(int));
    double *b = w.partials.p;
    Workspace ws;
    ws.P.pq = b;
    ws.P.rz0 = b + kMaxGrid;
    ws.P.rz1 = b + 2 * kMaxGrid;
    ws.P.rzo = b + 3 * kMaxGrid;
    ws.P.rr = b + 4 * kMaxGrid;
    ws.P.ff = b + 5 * kMaxGrid;
    ws.scal = b + 6 * kMaxGrid;
    ws.P.G = G;
    ws.fl = reinterpret_cast<Flags *>(w.flags.p);
    OFEA_CUDA(cudaMemsetAsync(w.partials.p, 0, nd * sizeof(double), c->stream));
    OFEA_CUDA(cudaMemsetAsync(w.flags.p, 0, sizeof(Flags), c->stream));
    w.hflags.ensure(2 * sizeof(Flags) / sizeof(int));  // two slots: drive() reads one chunk's flags while the next runs
    w.hscal.ensure(4);
    return ws;
}

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Replays `chunk(iters)` (as a captured CUDA graph when requested) until the
// device flags say done, max_iter is reached or the time budget runs out.
// Without per-chunk host work the next chunk is enqueued before the flags of
// the one before it are read, so the GPU does not wait for the host's round
// trip; a chunk that starts after the solve stopped returns at once in every
// kernel (the stop flag), and the flags are read again after the last one.
// There the first chunk is launched directly and the graph is captured and
// instantiated while the GPU runs it.
template <class ChunkFn>
void drive(ofea_ctx *c, const ofea_solve_opts &o, Workspace &ws, int per_chunk, ChunkFn chunk,
           Flags &hf, long long &launches, int kernels_per_iter, bool &timed_out, double t_start,
           const std::function<void()> &after_chunk) {
    cudaStream_t s = c->stream;
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    auto make_graph = [&]() {
        if (!o.use_graph || exec) return;
        OFEA_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        try {
            chunk(per_chunk);
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(s, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        cudaError_t e = cudaStreamEndCapture(s, &graph);
        if (e != cudaSuccess) fail_cuda(e, "cudaStreamEndCapture", __FILE__, __LINE__);
        e = cudaGraphInstantiate(&exec, graph, 0);
        if (e != cudaSuccess) fail_cuda(e, "cudaGraphInstantiate", __FILE__, __LINE__);
    };
    int launched = 0;
    Flags *h = reinterpret_cast<Flags *>(c->w.hflags.p);  // two slots
    cudaEvent_t ev[2] = {nullptr, nullptr};
    auto launch_chunk = [&]() {
        if (exec)
            OFEA_CUDA(cudaGraphLaunch(exec, s));
        else
            chunk(per_chunk);
        launched += per_chunk;
        launches += (long long)per_chunk * kernels_per_iter;
    };
    auto over_budget = [&]() { return o.time_budget_s > 0 && now_s() - t_start > o.time_budget_s; };
    try {
        if (!after_chunk) {
            for (auto &e : ev) OFEA_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            int k = 0;
            launch_chunk();
            OFEA_CUDA(cudaMemcpyAsync(&h[0], ws.fl, sizeof(Flags), cudaMemcpyDeviceToHost, s));
            OFEA_CUDA(cudaEventRecord(ev[0], s));
            make_graph();
            while (true) {
                const bool more = launched < o.max_iter;
                if (more) {  // slot k ^ 1 was read two chunks ago
                    launch_chunk();
                    OFEA_CUDA(cudaMemcpyAsync(&h[k ^ 1], ws.fl, sizeof(Flags), cudaMemcpyDeviceToHost, s));
                    OFEA_CUDA(cudaEventRecord(ev[k ^ 1], s));
                }
                OFEA_CUDA(cudaEventSynchronize(ev[k]));
                if (h[k].done || !more) break;
                if (over_budget()) {
                    timed_out = true;
                    break;
                }
                k ^= 1;
            }
            OFEA_CUDA(cudaMemcpyAsync(&h[0], ws.fl, sizeof(Flags), cudaMemcpyDeviceToHost, s));
            OFEA_CUDA(cudaStreamSynchronize(s));
        } else {
            make_graph();
            while (true) {
                launch_chunk();
                OFEA_CUDA(cudaMemcpyAsync(h, ws.fl, sizeof(Flags), cudaMemcpyDeviceToHost, s));
                OFEA_CUDA(cudaStreamSynchronize(s));
                if (h->done || launched >= o.max_iter) break;
                after_chunk();
                if (over_budget()) {
                    timed_out = true;
                    break;
                }
            }
        }
    } catch (...) {
        for (auto &e : ev)
            if (e) cudaEventDestroy(e);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        throw;
    }
    for (auto &e : ev)
        if (e) cudaEventDestroy(e);
    hf = *h;
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
}

int solver_grid(const ofea_ctx *c) { return std::min(kMaxGrid, c->num_sms * (2048 / kBlock)); }

// Clears the context's V-cycle stop flag when the solve's iterations end
// (normally or by an exception).
struct StopFlagScope {
    ofea_ctx *c;
    ~StopFlagScope() { c->vc_stop = nullptr; }
};

}  // namespace

// Damping of the block-Jacobi smoother: omega = damping / lmax, lmax the power
// iteration's estimate of lambda_max(D^-1 K).  The V(1,1) cycle stays
// positive definite while omega lmax < 2 (with margin for the estimate,
// which lies below lambda_max).
float smoother_weight(const ofea_ctx *c, double damping) { return (float)(damping / c->coarse.lmax); }

void solve_device(ofea_ctx *c, const double *d_f, double *d_u, const ofea_solve_opts &o,
                  ofea_solve_stats &st, const std::function<void(const double *)> &on_chunk) {
    cudaStream_t s = c->stream;
    const int n = c->n, nf = c->nfree;
    if (n == 0) {
        st.status = OFEA_OK;
        return;
    }
    const double t_start = now_s();
    const int G = solver_grid(c);
    Workspace ws = setup(c, G);
    SolverWork &w = c->w;
    cudaEvent_t e0, e1;
    OFEA_CUDA(cudaEventCreate(&e0));
    OFEA_CUDA(cudaEventCreate(&e1));
    OFEA_CUDA(cudaEventRecord(e0, s));
    // default poll interval: a preconditioned iteration is long and its solves
    // short (a poll every 4 iterations wastes fewer iterations after
    // convergence than it costs in host round trips); plain PCG polls every 16
    const bool precond = o.method == OFEA_SOLVER_MIXED || o.method == OFEA_SOLVER_LEARNED;
    int per_chunk = o.check_every > 0 ? o.check_every : (precond ? 4 : 16);
    per_chunk = std::max(1, std::min(per_chunk, o.max_iter));
    long long launches = 0;
    Flags hf{};
    bool timed_out = false;
    double rel = 0;
    int total_iters = 0, restarts = 0;
    w.r.ensure(n);
    w.q.ensure(n);
    w.p0.ensure(n);
    w.p1.ensure(n);
    const bool learned = o.method == OFEA_SOLVER_LEARNED;
    const bool mixed = o.method == OFEA_SOLVER_MIXED || learned;
    float setup_ms = 0.f;
    if (mixed) {
        const bool had = c->coarse.K_ok;
        cudaEvent_t es;
        OFEA_CUDA(cudaEventCreate(&es));
        setup_marks_clear(c);
        setup_mark(c, "start");
        if (learned) {
            if (!c->learned.have_weights) fail(OFEA_ERR_STATE, "train or load the learned stage first");
            setup_learned_solver(c);
        } else {
            setup_coarse(c, c->coarse_nodes);
        }
        OFEA_CUDA(cudaEventRecord(es, s));
        OFEA_CUDA(cudaEventSynchronize(es));
        OFEA_CUDA(cudaEventElapsedTime(&setup_ms, e0, es));
        cudaEventDestroy(es);
        if (!had) launches += 4 + 4 * ((c->coarse.m + 31) / 32) + 14;
        w.b32.ensure(n);
        w.x32.ensure(n);
        w.t32.ensure(n);
        w.z32a.ensure(n);
        w.z32b.ensure(n);
    } else {
        w.z.ensure(n);
    }
    const float wsm = mixed ? smoother_weight(c, kSmootherDamping) : 0.f;
    for (int attempt = 0; attempt < 8; ++attempt) {
        OFEA_CUDA(cudaMemsetAsync(w.p0.p, 0, sizeof(double) * n, s));
        OFEA_CUDA(cudaMemsetAsync(w.p1.p, 0, sizeof(double) * n, s));
        OFEA_CUDA(cudaMemsetAsync(w.q.p, 0, sizeof(double) * n, s));  // q = K p is kept by recurrence
        OFEA_CUDA(cudaMemsetAsync(ws.fl, 0, sizeof(Flags), s));
        if (mixed) {
            OFEA_CUDA(cudaMemsetAsync(w.z32a.p, 0, sizeof(float) * n, s));
            OFEA_CUDA(cudaMemsetAsync(w.z32b.p, 0, sizeof(float) * n, s));
            k_fcg_init<<<G, kBlock, 0, s>>>(nf, c->sl_ptr.p, c->scols.p, c->sv64.p, c->Dinv32.p, wsm, d_f,
                                            d_u, w.r.p, w.b32.p, w.x32.p, ws.P);
        } else {
            k_residual64<<<G, kBlock, 0, s>>>(nf, c->sl_ptr.p, c->scols.p, c->sv64.p, c->Dinv.p, d_f, d_u,
                                               w.r.p, w.z.p, ws.P);
        }
        OFEA_CHECK_LAUNCH();
        k_final_norms<<<1, kBlock, 0, s>>>(ws.P, ws.scal);
        OFEA_CUDA(cudaMemcpyAsync(w.hscal.p, ws.scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
        OFEA_CUDA(cudaStreamSynchronize(s));
        launches += 2;
        const double rr = w.hscal.p[0], ff = w.hscal.p[1];
        if (ff == 0.0) {
            OFEA_CUDA(cudaMemsetAsync(d_u, 0, sizeof(double) * n, s));
            rel = 0;
            break;
        }
        rel = std::sqrt(rr / ff);
        if (!std::isfinite(rel)) {
            hf.status = OFEA_ERR_BREAKDOWN;
            break;
        }
        if (rel <= o.rtol || total_iters >= o.max_iter || timed_out) break;
        if (attempt > 0) ++restarts;
        // recursive residual target a little below rtol; the true residual is re-checked
        const double tol2 = (0.5 * o.rtol) * (0.5 * o.rtol) * ff;
        ofea_solve_opts oo = o;
        oo.max_iter = o.max_iter - total_iters;
        if (mixed) {
            // the V-cycle kernels of this attempt return at once once the
            // solve has stopped (the flag is cleared at every attempt)
            c->vc_stop = &ws.fl->done;
            const StopFlagScope stop_scope{c};
            // initial preconditioner application z_0 = M(r_0)
            k_set_itB<<<1, 1, 0, s>>>(ws.fl, -1);
            vc_resid(c, w.b32.p, w.x32.p, w.t32.p);
            if (learned) learned_coarse_correct(c, w.t32.p, w.x32.p);
            else coarse_correct(c, w.t32.p, w.x32.p);
            k_fcg_post<<<G, kBlock, 0, s>>>(nf, c->sl_ptr.p, c->scols.p, c->sl_g.p, c->sv16g.p, c->Dinv32.p, wsm, w.b32.p,
                                            w.x32.p, w.r.p, w.z32a.p, w.z32b.p, ws.P, ws.fl);
            OFEA_CHECK_LAUNCH();
            launches += learned ? 12 : 6;
            auto chunk = [&](int iters) {
                for (int it = 0; it < iters; ++it) {
                    k_fcg_A<<<G, kBlock, 0, s>>>(nf, c->sl_ptr.p, c->scols.p, c->sv64.p, w.z32a.p, w.z32b.p,
                                                 w.p0.p, w.p1.p, w.q.p, ws.P, ws.fl, tol2);
                    k_fcg_B<<<G, kBlock, 0, s>>>(nf, c->Dinv32.p, wsm, w.p0.p, w.p1.p, w.q.p, d_u, w.r.p,
                                                 w.b32.p, w.x32.p, ws.P, ws.fl);
                    vc_resid(c, w.b32.p, w.x32.p, w.t32.p);
                    if (learned) learned_coarse_correct(c, w.t32.p, w.x32.p);
                    else coarse_correct(c, w.t32.p, w.x32.p);
                    k_fcg_post<<<G, kBlock, 0, s>>>(nf, c->sl_ptr.p, c->scols.p, c->sl_g.p, c->sv16g.p, c->Dinv32.p, wsm,
                                                    w.b32.p, w.x32.p, w.r.p, w.z32a.p, w.z32b.p, ws.P, ws.fl);
                }
                OFEA_CHECK_LAUNCH();
            };
            drive(c, oo, ws, per_chunk, chunk, hf, launches, learned ? 13 : 7, timed_out, t_start, {});
        } else {
            auto chunk = [&](int iters) {
                for (int it = 0; it < iters; ++it) {
                    k_pcg64_A<<<G, kBlock, 0, s>>>(nf, c->sl_ptr.p, c->scols.p, c->sv64.p, w.z.p, w.p0.p,
                                                   w.p1.p, w.q.p, ws.P, ws.fl, tol2);
                    k_pcg64_B<<<G, kBlock, 0, s>>>(nf, c->Dinv.p, w.p0.p, w.p1.p, w.q.p, d_u, w.r.p, w.z.p,
                                                   ws.P, ws.fl);
                }
                OFEA_CHECK_LAUNCH();
            };
            std::function<void()> after;
            if (on_chunk) after = [&] { on_chunk(w.r.p); };
            drive(c, oo, ws, per_chunk, chunk, hf, launches, 2, timed_out, t_start, after);
        }
        total_iters += hf.iters;
        if (hf.status == OFEA_ERR_BREAKDOWN) break;
    }
    OFEA_CUDA(cudaEventRecord(e1, s));
    OFEA_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    OFEA_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    st.iterations = total_iters;
    st.refinements = restarts;
    st.rel_residual = rel;
    st.seconds = ms * 1e-3;
    st.setup_seconds = setup_ms * 1e-3;
    st.kernel_launches = launches;
    if (hf.status == OFEA_ERR_BREAKDOWN)
        st.status = OFEA_ERR_BREAKDOWN;
    else if (!(rel <= o.rtol))
        st.status = timed_out ? OFEA_ERR_TIMEOUT : OFEA_ERR_NOT_CONVERGED;
    else
        st.status = OFEA_OK;
    if (learned && st.status != OFEA_OK) {
        // The learned stage is judged by the FP64 true residual: it missed the
        // target, so plain FP64 PCG restarts from zero and finishes the solve.
        ofea_solve_opts plain = o;
        plain.method = OFEA_SOLVER_PCG64;
        ofea_solve_stats st2{};
        OFEA_CUDA(cudaMemsetAsync(d_u, 0, sizeof(double) * n, s));
        solve_device(c, d_f, d_u, plain, st2, {});
        st2.iterations += st.iterations;
        st2.seconds += st.seconds;
        st2.setup_seconds += st.setup_seconds;
        st2.kernel_launches += st.kernel_launches;
        st2.rejected_learned = 1;
        st = st2;
    }
}

// Times the per-iteration kernels in isolation on the current state (after a
// solve of the same method): ms[0]/bytes[0] = the FP64 SpMV kernel (A),
// ms[1]/bytes[1] = B for PCG64, the FP32 post-smoothing SpMV for MIXED.
void profile_kernels(ofea_ctx *c, int method, int reps, double *ms, double *bytes) {
    cudaStream_t s = c->stream;
    const int n = c->n, nf = c->nfree;
    const int G = solver_grid(c);
    Workspace ws = setup(c, G);
    SolverWork &w = c->w;
    Flags f0{};
    f0.itA = 1;
    f0.itB = 1;
    OFEA_CUDA(cudaMemcpyAsync(ws.fl, &f0, sizeof(Flags), cudaMemcpyHostToDevice, s));
    std::vector<double> ones(5 * kMaxGrid, 1.0);
    OFEA_CUDA(cudaMemcpyAsync(ws.P.pq, ones.data(), sizeof(double) * 5 * kMaxGrid, cudaMemcpyHostToDevice, s));
    const double nnzv = 9.0 * c->sell_len * kSlice;  // stored values incl. padding
    const double nblk = (double)c->sell_len * kSlice;
    cudaEvent_t e0, e1, e2;
    OFEA_CUDA(cudaEventCreate(&e0));
    OFEA_CUDA(cudaEventCreate(&e1));
    OFEA_CUDA(cudaEventCreate(&e2));
    const double tol2 = -1.0;  // never converged: every launch does the full work
    if (method == OFEA_SOLVER_PCG64) {
        if (!w.z.p || w.z.n < (size_t)n) fail(OFEA_ERR_STATE, "run a GPU_PCG solve first");
        double *u = w.t.p;
        OFEA_CUDA(cudaEventRecord(e0, s));
        for (int i = 0; i < reps; ++i)
            k_pcg64_A<<<G, kBlock, 0, s>>>(nf, c->sl_ptr.p, c->scols.p, c->sv64.p, w.z.p, w.p0.p, w.p1.p,
                                           w.q.p, ws.P, ws.fl, tol2);
        OFEA_CUDA(cudaEventRecord(e1, s));
        for (int i = 0; i < reps; ++i)
            k_pcg64_B<<<G, kBlock, 0, s>>>(nf, c->Dinv.p, w.p0.p, w.p1.p, w.q.p, u, w.r.p, w.z.p, ws.P, ws.fl);
        OFEA_CUDA(cudaEventRecord(e2, s));
        // K values + columns + slice pointers, z, p_old and q_old read, p_new and q written
        bytes[0] = 8 * nnzv + 4 * nblk + 4.0 * ((nf + 31) / 32 + 1) + 8.0 * n * 5;
        bytes[1] = 72.0 * nf + 8.0 * n * 7;  // Dinv; u r/w, r r/w, p, q, z
    } else {
        if (!w.z32a.p || w.z32a.n < (size_t)n) fail(OFEA_ERR_STATE, "run a GPU_MIXED solve first");
        const float wsm = smoother_weight(c, kSmootherDamping);
        OFEA_CUDA(cudaEventRecord(e0, s));
        for (int i = 0; i < reps; ++i)
            k_fcg_A<<<G, kBlock, 0, s>>>(nf, c->sl_ptr.p, c->scols.p, c->sv64.p, w.z32a.p, w.z32b.p, w.p0.p,
                                         w.p1.p, w.q.p, ws.P, ws.fl, tol2);
        OFEA_CUDA(cudaEventRecord(e1, s));
        for (int i = 0; i < reps; ++i)
            k_fcg_post<<<G, kBlock, 0, s>>>(nf, c->sl_ptr.p, c->scols.p, c->sl_g.p, c->sv16g.p, c->Dinv32.p, wsm, w.b32.p,
                                            w.x32.p, w.r.p, w.z32a.p, w.z32b.p, ws.P, ws.fl);
        OFEA_CUDA(cudaEventRecord(e2, s));
        // FP64 K + columns + slice pointers, z (FP32), p_old and q_old read, p_new and q written
        bytes[0] = 8 * nnzv + 4 * nblk + 4.0 * ((nf + 31) / 32 + 1) + 4.0 * n + 8.0 * n * 4;
        // BF16 K + columns, x32 and b32 read, Dinv32, r (FP64) and z_old read, z_new written
        bytes[1] = 2 * nnzv + 4 * nblk + 4.0 * n * 2 + 36.0 * nf + 8.0 * n + 4.0 * n * 2;
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
