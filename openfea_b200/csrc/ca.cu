// Combined-approximations (CA) reanalysis on the device.
//
// The reference (src/ca_analysis.cpp) reanalyses a modified structure from
// the factorised original one: ΔK from the modified elements
// (ca_get_delt_stiffness, :18-30, ca_fill_CSR_sparse_mat :52-145), the basis
// r_0 = u_0, r_i = -K0^-1 ΔK r_(i-1) by re-solving with the kept SuperLU
// factor (ca_build_rom, :146-178), a thin SVD of the basis (ca_SVD, :180-207)
// and the Galerkin system V^T K V y = V^T f of the modified K (ca_solve,
// :209-250, ca_reduced_K :262-283, ca_reduced_F :303-311), u = V y.
//
// Here both models are assembled contexts on the same nodes, elements and
// free numbering (a deleted element has E = 0 in the modified model), so
// ΔK r = K r - K0 r is two device SpMVs and K0^-1 is the device solver.  The
// basis is orthonormalised in FP64 from the eigen-decomposition of its Gram
// matrix (the SVD's U = V W Λ^-1/2, computed twice); the Galerkin solution
// depends only on the span, so this matches the reference's FP32 SVD up to
// that SVD's rounding.  The tall-skinny products are device kernels; the
// n_basis x n_basis algebra is host code.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>

#include "ofea_internal.cuh"

namespace ofea {

namespace {

constexpr int kCaBlock = 256;

// out = a - b
__global__ void k_ca_sub(long n, const double *__restrict__ a, const double *__restrict__ b, double *__restrict__ out) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        out[i] = a[i] - b[i];
}

// Block partial sums of X[:, pi] . Y[:, pj] for every pair (pi, pj) =
// pairs[blockIdx.y]; columns of length n at stride n.  part[pair * gridDim.x
// + block]; the host adds them in block order (reproducible).
__global__ void k_ca_dots(long n, const double *__restrict__ X, const double *__restrict__ Y,
                          const int2 *__restrict__ pairs, double *__restrict__ part) {
    __shared__ double sh[kCaBlock / 32];
    const int2 pr = pairs[blockIdx.y];
    const double *x = X + (long)pr.x * n, *y = Y + (long)pr.y * n;
    double s = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        s = fma(x[i], y[i], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kCaBlock / 32; ++w) t += sh[w];
        part[(long)blockIdx.y * gridDim.x + blockIdx.x] = t;
    }
}

// Y[:, j] = sum_k X[:, k] C[k + p * j]  (X: p columns, Y: q columns, stride n)
__global__ void k_ca_combine(long n, const double *__restrict__ X, int p, const double *__restrict__ C, int q,
                             double *__restrict__ Y) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        double x[kCaMaxBasis];
        for (int k = 0; k < p; ++k) x[k] = X[(long)k * n + i];
        for (int j = 0; j < q; ++j) {
            double s = 0.0;
            for (int k = 0; k < p; ++k) s = fma(x[k], C[k + p * j], s);
            Y[(long)j * n + i] = s;
        }
    }
}

struct CaWork {
    int grid = 296;
    cudaStream_t s = nullptr;
    DevBuf<int2> pairs;
    DevBuf<double> part, coef;
    std::vector<double> hpart;

    // G[i][j] = X[:, i] . Y[:, j] for i < p, j < q (sym: X == Y, only i <= j computed)
    std::vector<double> dots(long n, const double *X, int p, const double *Y, int q, bool sym) {
        std::vector<int2> pr;
        for (int i = 0; i < p; ++i)
            for (int j = sym ? i : 0; j < q; ++j) pr.push_back(make_int2(i, j));
        pairs.ensure(pr.size());
        part.ensure(pr.size() * (size_t)grid);
        OFEA_CUDA(cudaMemcpyAsync(pairs.p, pr.data(), sizeof(int2) * pr.size(), cudaMemcpyHostToDevice, s));
        k_ca_dots<<<dim3(grid, (unsigned)pr.size()), kCaBlock, 0, s>>>(n, X, Y, pairs.p, part.p);
        OFEA_CHECK_LAUNCH();
        hpart.resize(pr.size() * (size_t)grid);
        OFEA_CUDA(cudaMemcpyAsync(hpart.data(), part.p, sizeof(double) * hpart.size(), cudaMemcpyDeviceToHost, s));
        OFEA_CUDA(cudaStreamSynchronize(s));
        std::vector<double> G((size_t)p * q, 0.0);
        for (size_t k = 0; k < pr.size(); ++k) {
            double t = 0.0;
            for (int b = 0; b < grid; ++b) t += hpart[k * grid + b];
            G[(size_t)pr[k].x * q + pr[k].y] = t;
            if (sym) G[(size_t)pr[k].y * q + pr[k].x] = t;
        }
        return G;
    }

    // Y = X C, C p x q column-major on the host
    void combine(long n, const double *X, int p, const std::vector<double> &C, int q, double *Y) {
        coef.ensure(C.size());
        OFEA_CUDA(cudaMemcpyAsync(coef.p, C.data(), sizeof(double) * C.size(), cudaMemcpyHostToDevice, s));
        k_ca_combine<<<grid, kCaBlock, 0, s>>>(n, X, p, coef.p, q, Y);
        OFEA_CHECK_LAUNCH();
    }
};

// Eigen-decomposition of the symmetric m x m matrix A (row-major) by cyclic
// Jacobi rotations: A = W diag(lam) W^T, W column-major in w[k + m * j].
void sym_eigen(std::vector<double> A, int m, std::vector<double> &lam, std::vector<double> &w) {
    w.assign((size_t)m * m, 0.0);
    for (int i = 0; i < m; ++i) w[i + m * i] = 1.0;
    auto a = [&](int i, int j) -> double & { return A[(size_t)i * m + j]; };
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, diag = 0.0;
        for (int i = 0; i < m; ++i) {
            diag += a(i, i) * a(i, i);
            for (int j = i + 1; j < m; ++j) off += a(i, j) * a(i, j);
        }
        if (off <= 1e-32 * diag || off == 0.0) break;
        for (int p = 0; p < m; ++p)
            for (int q = p + 1; q < m; ++q) {
                const double apq = a(p, q);
                if (apq == 0.0) continue;
                const double theta = (a(q, q) - a(p, p)) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
                for (int k = 0; k < m; ++k) {  // A <- A J (columns p, q)
                    const double akp = a(k, p), akq = a(k, q);
                    a(k, p) = c * akp - sn * akq;
                    a(k, q) = sn * akp + c * akq;
                }
                for (int k = 0; k < m; ++k) {  // A <- J^T A (rows p, q)
                    const double apk = a(p, k), aqk = a(q, k);
                    a(p, k) = c * apk - sn * aqk;
                    a(q, k) = sn * apk + c * aqk;
                }
                for (int k = 0; k < m; ++k) {
                    const double wkp = w[k + m * p], wkq = w[k + m * q];
                    w[k + m * p] = c * wkp - sn * wkq;
                    w[k + m * q] = sn * wkp + c * wkq;
                }
            }
    }
    lam.resize(m);
    for (int i = 0; i < m; ++i) lam[i] = a(i, i);
}

// Solves A y = b (m x m row-major) by Gaussian elimination with partial
// pivoting; false if A is singular to working precision.
bool dense_solve(std::vector<double> A, std::vector<double> b, int m, std::vector<double> &y) {
    for (int k = 0; k < m; ++k) {
        int piv = k;
        for (int i = k + 1; i < m; ++i)
            if (std::fabs(A[(size_t)i * m + k]) > std::fabs(A[(size_t)piv * m + k])) piv = i;
        if (!(std::fabs(A[(size_t)piv * m + k]) > 0.0)) return false;
        if (piv != k) {
            for (int j = 0; j < m; ++j) std::swap(A[(size_t)k * m + j], A[(size_t)piv * m + j]);
            std::swap(b[k], b[piv]);
        }
        for (int i = k + 1; i < m; ++i) {
            const double l = A[(size_t)i * m + k] / A[(size_t)k * m + k];
            for (int j = k; j < m; ++j) A[(size_t)i * m + j] -= l * A[(size_t)k * m + j];
            b[i] -= l * b[k];
        }
    }
    y.assign(m, 0.0);
    for (int i = m - 1; i >= 0; --i) {
        double s = b[i];
        for (int j = i + 1; j < m; ++j) s -= A[(size_t)i * m + j] * y[j];
        y[i] = s / A[(size_t)i * m + i];
    }
    return true;
}

// Orthonormal basis of span(V[:, 0..p)) into U (same stride); returns its
// size.  Columns are scaled to unit norm, then U = V W Λ^-1/2 from the Gram
// matrix V^T V = W Λ W^T (directions with λ < 1e-13 λ_max are dropped), twice.
int orthonormalise(CaWork &cw, long n, double *V, int p, double *U, double *tmp) {
    double *src = V;
    int m = p;
    for (int pass = 0; pass < 2; ++pass) {
        std::vector<double> G = cw.dots(n, src, m, src, m, true);
        // scale to unit columns (folded into the combination coefficients)
        std::vector<double> d(m);
        for (int i = 0; i < m; ++i) d[i] = G[(size_t)i * m + i] > 0 ? 1.0 / std::sqrt(G[(size_t)i * m + i]) : 0.0;
        std::vector<double> Gs((size_t)m * m);
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j) Gs[(size_t)i * m + j] = d[i] * G[(size_t)i * m + j] * d[j];
        std::vector<double> lam, W;
        sym_eigen(Gs, m, lam, W);
        const double lmax = *std::max_element(lam.begin(), lam.end());
        if (!(lmax > 0)) return 0;
        std::vector<int> keep;
        for (int j = 0; j < m; ++j)
            if (lam[j] > 1e-13 * lmax) keep.push_back(j);
        const int q = (int)keep.size();
        std::vector<double> C((size_t)m * q);
        for (int jj = 0; jj < q; ++jj) {
            const int j = keep[jj];
            const double s = 1.0 / std::sqrt(lam[j]);
            for (int k = 0; k < m; ++k) C[k + (size_t)m * jj] = d[k] * W[k + (size_t)m * j] * s;
        }
        double *dst = pass == 0 ? tmp : U;
        cw.combine(n, src, m, C, q, dst);
        src = dst;
        m = q;
    }
    return m;
}

double now_seconds() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

}  // namespace

void ca_reanalysis(ofea_ctx *base, ofea_ctx *mod, const double *h_f, const double *h_u0, int nb,
                   const ofea_solve_opts &o, double *h_u, ofea_ca_stats *stats) {
    const double t0 = now_seconds();
    const long n = base->n;
    cudaStream_t s = base->stream;
    CaWork cw;
    cw.s = s;
    cw.grid = 2 * std::max(1, base->num_sms);
    DevBuf<double> V, U, T, f, t0v, t1v, x;
    V.ensure((size_t)n * nb);
    U.ensure((size_t)n * nb);
    T.ensure((size_t)n * nb);
    f.ensure(n);
    t0v.ensure(n);
    t1v.ensure(n);
    x.ensure(n);
    cudaEvent_t ev;
    OFEA_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    auto join = [&](cudaStream_t from, cudaStream_t to) {  // `to` waits for the work queued on `from`
        OFEA_CUDA(cudaEventRecord(ev, from));
        OFEA_CUDA(cudaStreamWaitEvent(to, ev, 0));
    };
    int iters = 0;
    auto solve0 = [&](const double *rhs, double *out) {  // out = K0^-1 rhs
        OFEA_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * n, s));
        ofea_solve_stats st{};
        solve_device(base, rhs, out, o, st);
        iters += st.iterations;
        if (st.status != OFEA_OK)
            fail(st.status, "CA reanalysis: a solve with the original K did not converge");
    };
    OFEA_CUDA(cudaMemcpyAsync(f.p, h_f, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    // r_0 = u_0
    if (h_u0) OFEA_CUDA(cudaMemcpyAsync(V.p, h_u0, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    else solve0(f.p, V.p);
    // r_i = -K0^-1 (K r_(i-1) - K0 r_(i-1))
    for (int i = 1; i < nb; ++i) {
        const double *r = V.p + (long)(i - 1) * n;
        join(s, mod->stream);
        spmv64(mod, r, t1v.p);
        spmv64(base, r, t0v.p);
        join(mod->stream, s);
        k_ca_sub<<<cw.grid, kCaBlock, 0, s>>>(n, t0v.p, t1v.p, t0v.p);  // K0 r - K r = -ΔK r
        OFEA_CHECK_LAUNCH();
        solve0(t0v.p, V.p + (long)i * n);
    }
    // orthonormal basis, reduced system of the modified K, u = U y
    const int m = orthonormalise(cw, n, V.p, nb, U.p, T.p);
    if (m == 0) fail(OFEA_ERR_BREAKDOWN, "CA reanalysis: the basis is zero");
    join(s, mod->stream);
    for (int j = 0; j < m; ++j) spmv64(mod, U.p + (long)j * n, T.p + (long)j * n);
    join(mod->stream, s);
    std::vector<double> KR = cw.dots(n, U.p, m, T.p, m, false);
    for (int i = 0; i < m; ++i)  // symmetrise (K is symmetric; rounding is not)
        for (int j = i + 1; j < m; ++j) {
            const double a = 0.5 * (KR[(size_t)i * m + j] + KR[(size_t)j * m + i]);
            KR[(size_t)i * m + j] = KR[(size_t)j * m + i] = a;
        }
    OFEA_CUDA(cudaMemcpyAsync(x.p, f.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    std::vector<double> fr = cw.dots(n, U.p, m, x.p, 1, false);
    std::vector<double> y;
    if (!dense_solve(KR, fr, m, y)) fail(OFEA_ERR_BREAKDOWN, "CA reanalysis: the reduced matrix is singular");
    cw.combine(n, U.p, m, y, 1, x.p);
    // true relative residual of the CA solution on the modified K
    join(s, mod->stream);
    spmv64(mod, x.p, t1v.p);
    join(mod->stream, s);
    k_ca_sub<<<cw.grid, kCaBlock, 0, s>>>(n, f.p, t1v.p, t0v.p);
    OFEA_CHECK_LAUNCH();
    std::vector<double> rr = cw.dots(n, t0v.p, 1, t0v.p, 1, true), ff = cw.dots(n, f.p, 1, f.p, 1, true);
    OFEA_CUDA(cudaMemcpyAsync(h_u, x.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    OFEA_CUDA(cudaStreamSynchronize(s));
    cudaEventDestroy(ev);
    if (stats) {
        stats->status = OFEA_OK;
        stats->basis_requested = nb;
        stats->basis_used = m;
        stats->solve_iterations = iters;
        stats->rel_residual = ff[0] > 0 ? std::sqrt(rr[0] / ff[0]) : 0.0;
        stats->seconds = now_seconds() - t0;
    }
}

}  // namespace ofea
