// Learned coarse-correction stage of the LEARNED solver.
//
// Level: the nested aggregates of build_aggregation_fine (cells half as wide
// as the exact coarse level's), each with six rigid-body modes Z2, and the
// Galerkin operator E2 = Z2^T K Z2 (6 x 6 blocks between neighbouring cells).
// The exact correction of that level is what an extra multigrid level would
// add to the V-cycle; factoring E2 is too costly, so the stage applies a
// learned linear approximation of its inverse:
//
//   input   c  = Z2^T t - E2 P e1      (the level-2 residual with the exact
//                                      level-1 correction e1 taken out; P e1
//                                      is e1 in level-2 modes)
//   scaled  x  = D^-1/2 c,  Ehat = D^-1/2 E2 D^-1/2,  D = diag E2
//   stage   y  = s * M(s * x),   M = sum_k c_k (B Ehat)^(k-1) B,  k = 1..3
//           B  = the inverse of Ehat's diagonal 6x6 blocks (block Jacobi)
//   output  x_fine += Z2 D^-1/2 y
//
// M is a polynomial in the block-Jacobi-preconditioned operator with global
// coefficients c_k; s (6 per aggregate) are scalings set by a graph network
// from per-aggregate features (log stiffness, neighbour count, log diag B):
//
//   h0 = relu(W0 f + b0)                                    (64 wide)
//   4 layers: a_I = [h_I, mean_J h_J, mean_J dx h_J, mean_J dy h_J, mean_J dz h_J]
//             over the existing ones of the 26 neighbour cells J,
//             h = relu(W a + b)                              (320 -> 64)
//   s = exp((Wd h + bd) / 2)
//
// The stage is linear and symmetric in x for any weights, so the outer
// flexible CG sees a fixed SPD-like preconditioner; the network is evaluated
// once per matrix.  Training (on the GPU, these kernels): inputs are the
// level-2 residuals, built as above, of plain-PCG iterates on the current
// matrix; the loss is the energy
//   L(y) = (1/2 y^T Ehat y - y^T x) / (6 na),
// whose minimiser is the exact correction Ehat^-1 x, so no inverse and no
// displacement targets are needed.  c starts at the energy-optimal constants
// (a 3 x 3 least-squares fit over the samples), the network at s ~ 1; Adam,
// FP32 weights and FP32 accumulation.  Every reduction runs in a fixed order:
// training is deterministic.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <random>

#include "precond.cuh"
#include "tc_gemm.cuh"
#include "sell.cuh"
#include "solver_common.cuh"

namespace ofea {

constexpr int kF = 64;        // hidden width
constexpr int kNFeat = 8;     // per-aggregate input features
constexpr int kOut = 6;       // log-scalings, one per rigid mode
constexpr int kTerms = 3;     // polynomial terms of M
constexpr int kA = 5 * kF;    // aggregated features per layer
constexpr int kLayers = 4;

Learned::Layout Learned::layout() {
    Layout L;
    size_t o = 0;
    L.W0 = o; o += (size_t)kF * kNFeat;
    L.b0 = o; o += kF;
    for (int l = 0; l < kLayers; ++l) {
        L.W[l] = o; o += (size_t)kF * kA;
        L.b[l] = o; o += kF;
    }
    L.Wd = o; o += (size_t)kOut * kF;
    L.bd = o; o += kOut;
    L.c0 = o; o += kTerms;
    L.total = o;
    return L;
}

namespace {

__device__ __forceinline__ int slot_dx(int s) { return s / 9 - 1; }
__device__ __forceinline__ int slot_dy(int s) { return (s / 3) % 3 - 1; }
__device__ __forceinline__ int slot_dz(int s) { return s % 3 - 1; }

// ------------------------------------------------------------ level data --

// Eb[I][slot][36] from the Galerkin blocks (nchunk = 1: a masked copy).
__global__ void k_e2_blocks(int na, int nchunk, const int *__restrict__ nbr, const double *__restrict__ part,
                            double *__restrict__ Eb) {
    const long total = (long)na * 27 * 36;
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < total; g += (long)gridDim.x * blockDim.x) {
        const int I = (int)(g / (27 * 36)), v = (int)(g % (27 * 36)), slot = v / 36;
        double s = 0.0;
        if (nbr[27L * I + slot] >= 0)
            for (int ch = 0; ch < nchunk; ++ch) s += part[((long)I * nchunk + ch) * (27 * 36) + v];
        Eb[g] = s;
    }
}

// Jacobi scaling: dsq = sqrt(diag E2), Ehat = D^-1/2 E2 D^-1/2 (FP32), and
// the per-aggregate stiffness feature log(mean diag).
__global__ void k_e2_scale(int na, const double *__restrict__ Eb, float *__restrict__ dsq,
                           float *__restrict__ feat) {
    for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < na; I += gridDim.x * blockDim.x) {
        double mean = 0.0;
        for (int k = 0; k < 6; ++k) {
            const double d = Eb[(27L * I + 13) * 36 + 7 * k];
            dsq[6L * I + k] = d > 0 ? (float)sqrt(d) : 0.f;
            mean += d > 0 ? d : 0.0;
        }
        feat[I] = (float)log(mean / 6.0 + 1e-300);
    }
}
__global__ void k_e2_hat(int na, const int *__restrict__ nbr, const double *__restrict__ Eb,
                         const float *__restrict__ dsq, float *__restrict__ Ehat) {
    const long total = (long)na * 27 * 36;
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < total; g += (long)gridDim.x * blockDim.x) {
        const int I = (int)(g / (27 * 36)), v = (int)(g % (27 * 36)), slot = v / 36, k = (v % 36) / 6,
                  l = v % 6;
        const int J = nbr[27L * I + slot];
        float e = 0.f;
        if (J >= 0) {
            const float a = dsq[6L * I + k], b = dsq[6L * J + l];
            e = (a > 0 && b > 0) ? (float)(Eb[g] / ((double)a * (double)b)) : 0.f;
        }
        Ehat[g] = e;
    }
}


// B_I = inverse of the diagonal block Ehat[I, 13] (SPD, unit diagonal), by
// Gauss-Jordan in FP64 without pivoting; thread per aggregate.
__global__ void k_block_inv6(int na, const float *__restrict__ Ehat, float *__restrict__ Binv) {
    for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < na; I += gridDim.x * blockDim.x) {
        double a[6][12];
        const float *e = Ehat + (27L * I + 13) * 36;
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 6; ++j) {
                a[i][j] = e[6 * i + j];
                a[i][6 + j] = i == j ? 1.0 : 0.0;
            }
        bool ok = true;
        for (int k = 0; k < 6; ++k) {
            const double p = a[k][k];
            if (!(p > 0.0)) {
                ok = false;
                break;
            }
            const double ip = 1.0 / p;
            for (int j = 0; j < 12; ++j) a[k][j] *= ip;
            for (int i = 0; i < 6; ++i) {
                if (i == k) continue;
                const double f = a[i][k];
                for (int j = 0; j < 12; ++j) a[i][j] -= f * a[k][j];
            }
        }
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 6; ++j) Binv[36L * I + 6 * i + j] = ok ? (float)a[i][6 + j] : (i == j ? 1.f : 0.f);
    }
}

// Network input per aggregate: [centred log stiffness, neighbour count / 26, log diag B (6)].
__global__ void k_node_features(int na, const float *__restrict__ feat, const float *__restrict__ invdeg,
                                const float *__restrict__ Binv, float *__restrict__ X0) {
    for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < na; I += gridDim.x * blockDim.x) {
        float *x = X0 + (long)kNFeat * I;
        x[0] = feat[I];
        x[1] = invdeg[I] > 0.f ? 1.f / (26.f * invdeg[I]) : 0.f;
        for (int k = 0; k < 6; ++k) x[2 + k] = logf(fmaxf(Binv[36L * I + 7 * k], 1e-30f));
    }
}

// ----------------------------------------------------------------- layers --

// Bias-gradient partials: part[s][O*K + o] = sum over the rows of chunk s of
// dZ[r][o], rows in order (the weight part of each partial comes from the
// tensor-core product); summed afterwards in chunk order (deterministic).
__global__ void k_bias_partials(long R, int O, int K, long chunk, const float *__restrict__ dZ,
                                float *__restrict__ part) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (o >= O) return;
    const long rb = s * chunk, re = min(R, rb + chunk);
    float acc = 0.f;
    for (long r = rb; r < re; ++r) acc += dZ[r * O + o];
    part[(long)s * (O * K + O) + O * K + o] = acc;
}

// grad[j] = sum_s part[s][j] (fixed order), scattered to the W / b offsets.
__global__ void k_wgrad_sum(int S, int O, int K, const float *__restrict__ part, float *__restrict__ gW,
                            float *__restrict__ gb) {
    const int nout = O * K + O;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nout; j += gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int q = 0; q < S; ++q) s += part[(long)q * nout + j];
        if (j < O * K) gW[j] = s;
        else gb[j - O * K] = s;
    }
}

// a = [h, mean h_J, mean dx h_J, mean dy h_J, mean dz h_J] over the existing
// neighbours J of I (invdeg = 1 / their count): means keep every layer's
// activations at the scale of its input.
__global__ void k_gnn_aggregate(long R, int na, const int *__restrict__ nbr, const float *__restrict__ invdeg,
                                const float *__restrict__ H, float *__restrict__ A) {
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < R * kF; g += (long)gridDim.x * blockDim.x) {
        const long r = g / kF;
        const int f = (int)(g % kF);
        const int I = (int)(r % na);
        const long base = r - I;  // sample offset
        float s = 0.f, sx = 0.f, sy = 0.f, sz = 0.f;
        for (int sl = 0; sl < 27; ++sl) {
            if (sl == 13) continue;
            const int J = nbr[27L * I + sl];
            if (J < 0) continue;
            const float h = H[(base + J) * kF + f];
            s += h;
            sx += slot_dx(sl) * h;
            sy += slot_dy(sl) * h;
            sz += slot_dz(sl) * h;
        }
        const float w = invdeg[I];
        float *a = A + r * kA;
        a[f] = H[r * kF + f];
        a[kF + f] = w * s;
        a[2 * kF + f] = w * sx;
        a[3 * kF + f] = w * sy;
        a[4 * kF + f] = w * sz;
    }
}

// dH from dA: the transpose of k_gnn_aggregate (neighbour J sees I at the
// opposite slot, offset negated, weighted by J's invdeg).  Gather form: no atomics.
__global__ void k_gnn_aggregate_bwd(long R, int na, const int *__restrict__ nbr, const float *__restrict__ invdeg,
                                    const float *__restrict__ dA, const float *__restrict__ Z,
                                    float *__restrict__ dZ) {
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < R * kF; g += (long)gridDim.x * blockDim.x) {
        const long r = g / kF;
        const int f = (int)(g % kF);
        const int I = (int)(r % na);
        const long base = r - I;
        float d = dA[r * kA + f];
        for (int sl = 0; sl < 27; ++sl) {
            if (sl == 13) continue;
            const int J = nbr[27L * I + sl];
            if (J < 0) continue;
            // offset of I seen from J is -(dx,dy,dz) of slot sl
            const float *aJ = dA + (base + J) * kA;
            d += invdeg[J] * (aJ[kF + f] - slot_dx(sl) * aJ[2 * kF + f] - slot_dy(sl) * aJ[3 * kF + f] -
                              slot_dz(sl) * aJ[4 * kF + f]);
        }
        // relu backward of the layer that produced h: dZ = dH (Z > 0)
        dZ[g] = Z[g] > 0.f ? d : 0.f;
    }
}

// invdeg[I] = 1 / (number of existing neighbours of I), 0 for none.
__global__ void k_invdeg(int na, const int *__restrict__ nbr, float *__restrict__ invdeg) {
    for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < na; I += gridDim.x * blockDim.x) {
        int n = 0;
        for (int sl = 0; sl < 27; ++sl) n += (sl != 13 && nbr[27L * I + sl] >= 0);
        invdeg[I] = n > 0 ? 1.f / n : 0.f;
    }
}

__global__ void k_relu_bwd(long n, const float *__restrict__ dH, const float *__restrict__ Z, float *__restrict__ dZ) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        dZ[i] = Z[i] > 0.f ? dH[i] : 0.f;
}

__global__ void k_adam(long n, float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// ----------------------------------------------------- the level-2 input --

// Level-1 correction e1 (6 per parent aggregate) expressed in the modes of
// child aggregate J: a rigid motion (T, theta) about the parent centroid is
// (T + theta x delta, ratio theta) about the child's, delta = s1 (c_J - c_P),
// ratio = s1 / s2 (the modes' length scales).  pdel = (delta, ratio).
__device__ __forceinline__ void child_coeffs(int J, const int *__restrict__ parent, const float *__restrict__ pdel,
                                             const float *__restrict__ e1, float g[6]) {
    const float *e = e1 + 6L * parent[J];
    const float dx = pdel[4L * J], dy = pdel[4L * J + 1], dz = pdel[4L * J + 2], ratio = pdel[4L * J + 3];
    g[0] = e[0] + e[4] * dz - e[5] * dy;
    g[1] = e[1] + e[5] * dx - e[3] * dz;
    g[2] = e[2] + e[3] * dy - e[4] * dx;
    g[3] = ratio * e[3];
    g[4] = ratio * e[4];
    g[5] = ratio * e[5];
}

// t[a] += sum_b e[6a + b] v[b] for one 6 x 6 FP32 block e (16-byte aligned:
// blocks are 144 bytes apart), loaded as nine 16-byte words before the
// first product; the sums run in the order a, then b = 0..5.
__device__ __forceinline__ void block6_apply(const float *__restrict__ e, const float (&v)[6], float (&t)[6]) {
    float w[36];
    const float4 *e4 = reinterpret_cast<const float4 *>(e);
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const float4 x = __ldg(e4 + q);
        w[4 * q] = x.x;
        w[4 * q + 1] = x.y;
        w[4 * q + 2] = x.z;
        w[4 * q + 3] = x.w;
    }
#pragma unroll
    for (int a = 0; a < 6; ++a)
#pragma unroll
        for (int b = 0; b < 6; ++b) t[a] = fmaf(w[6 * a + b], v[b], t[a]);
}

// Scaled level-2 residual with the exact level-1 correction taken out:
//   S_I = D_I^-1/2 (c2 - E2 P e1)_I = c2_I / dsq_I - sum_s Ehat[I,s] (dsq o P e1)_J(s).
// Warp per aggregate, lane s < 27 handles neighbour slot s.
// FIRST: also the stage's first term on S (as k_poly_first with x = S):
// v1 = B (sc * S) into v1, c_1 v1 into out.
template <bool FIRST>
__global__ void __launch_bounds__(kBlock) k_lrn_shift(int na, const int *__restrict__ nbr,
                                                      const float *__restrict__ Ehat, const float *__restrict__ dsq,
                                                      const int *__restrict__ parent, const float *__restrict__ pdel,
                                                      const float *__restrict__ e1, const float *__restrict__ c2,
                                                      float *__restrict__ S, const float *__restrict__ Binv = nullptr,
                                                      const float *__restrict__ sc = nullptr,
                                                      const float *__restrict__ coef = nullptr,
                                                      float *__restrict__ v1 = nullptr, float *__restrict__ out = nullptr,
                                                      const int *__restrict__ stop = nullptr) {
    if (vc_stopped(stop)) return;
    const int lane = threadIdx.x & 31;
    for (int I = (blockIdx.x * blockDim.x + threadIdx.x) / 32; I < na; I += gridDim.x * blockDim.x / 32) {
        float v[6] = {0, 0, 0, 0, 0, 0};
        const int J = lane < 27 ? nbr[27L * I + lane] : -1;
        if (J >= 0) {
            float g[6];
            child_coeffs(J, parent, pdel, e1, g);
            for (int l = 0; l < 6; ++l) g[l] *= dsq[6L * J + l];
            block6_apply(Ehat + (27L * I + lane) * 36, g, v);
        }
        for (int k = 0; k < 6; ++k) v[k] = warp_sum(v[k]);
        float Sv = 0.f;
        if (lane < 6) {
            float vk = v[0];
            for (int k = 1; k < 6; ++k)
                if (lane == k) vk = v[k];
            const float d = dsq[6L * I + lane];
            Sv = d > 0.f ? c2[6L * I + lane] / d - vk : 0.f;
            S[6L * I + lane] = Sv;
        }
        if (FIRST) {
            const float uu = lane < 6 ? (sc ? sc[6L * I + lane] * Sv : Sv) : 0.f;
            float u[6];
#pragma unroll
            for (int l = 0; l < 6; ++l) u[l] = __shfl_sync(0xffffffffu, uu, l);
            if (lane < 6) {
                const float *B = Binv + 36L * I;
                float w = 0.f;
                for (int l = 0; l < 6; ++l) w = fmaf(B[6 * lane + l], u[l], w);
                v1[6L * I + lane] = w;
                out[6L * I + lane] = coef[0] * w;
            }
        }
    }
}

// sigma = RMS of S (one CTA, fixed order).
__global__ void __launch_bounds__(kBlock) k_gnn_sigma(int na, const float *__restrict__ S, double *__restrict__ out) {
    __shared__ double sh[kWarpsPerBlock];
    double acc = 0.0;
    for (int i = threadIdx.x; i < 6 * na; i += blockDim.x) acc += (double)S[i] * S[i];
    const double s = block_sum(acc, sh);
    if (threadIdx.x == 0) out[0] = sqrt(s / (6.0 * na)) + 1e-300;
}

// Dataset sample: the normalised rows S / sigma.
__global__ void k_gnn_sample(int na, const float *__restrict__ S, const double *__restrict__ sigma,
                             float *__restrict__ out) {
    const float is = (float)(1.0 / sigma[0]);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 6 * na; i += gridDim.x * blockDim.x) out[i] = S[i] * is;
}

__global__ void k_f64_to_f32(long n, const double *__restrict__ a, float *__restrict__ b) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}




// ------------------------------------------------ coarse level from level 2 --

// E1 = P^T E2 P: the coarse Galerkin matrix from the nested level's blocks
// (Z1 = Z2 P exactly, P the map of a parent's rigid modes into its
// children's).  36 threads per (parent I, neighbour slot S), one per entry of
// the 6 x 6 block; sums over child pairs in a fixed order.
__device__ __forceinline__ double pmat(const float *pd, int p, int k) {
    // P[p][k] of a child with (delta, ratio) = pd
    const double dx = pd[0], dy = pd[1], dz = pd[2], ro = pd[3];
    if (p < 3) {
        if (k < 3) return p == k ? 1.0 : 0.0;
        // translation rows: T2 = T1 + theta1 x delta
        const int t = k - 3;  // theta component
        if (p == 0) return t == 1 ? dz : t == 2 ? -dy : 0.0;
        if (p == 1) return t == 2 ? dx : t == 0 ? -dz : 0.0;
        return t == 0 ? dy : t == 1 ? -dx : 0.0;
    }
    return k == p ? ro : 0.0;
}

__global__ void k_e1_from_e2(int na1, int m1, const int *__restrict__ nbr1, const int *__restrict__ children,
                             const int *__restrict__ cell2, const float *__restrict__ pdel,
                             const double *__restrict__ Eb, double *__restrict__ E1) {
    const int k = threadIdx.x / 6, l = threadIdx.x % 6;
    for (int item = blockIdx.x; item < na1 * 27; item += gridDim.x) {
        const int I = item / 27, S = item % 27;
        const int J = nbr1[27L * I + S];
        if (J < 0 || threadIdx.x >= 36) continue;
        double acc = 0.0;
        for (int ca = 0; ca < 8; ++ca) {
            const int a = children[8L * I + ca];
            if (a < 0) continue;
            for (int cb = 0; cb < 8; ++cb) {
                const int b = children[8L * J + cb];
                if (b < 0) continue;
                const int dx = cell2[3 * b] - cell2[3 * a], dy = cell2[3 * b + 1] - cell2[3 * a + 1],
                          dz = cell2[3 * b + 2] - cell2[3 * a + 2];
                if (dx < -1 || dx > 1 || dy < -1 || dy > 1 || dz < -1 || dz > 1) continue;
                const double *E = Eb + ((long)a * 27 + (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1)) * 36;
                const float *pa = pdel + 4L * a, *pb = pdel + 4L * b;
                for (int p = 0; p < 6; ++p) {
                    const double pak = pmat(pa, p, k);
                    if (pak == 0.0) continue;
                    double t = 0.0;
                    for (int q = 0; q < 6; ++q) t += E[6 * p + q] * pmat(pb, q, l);
                    acc += pak * t;
                }
            }
        }
        E1[(6L * I + k) * m1 + 6L * J + l] = acc;
    }
}

// -------------------------------------------------------- the stage M --

// Rows r = b * na + I of a batch of coarse vectors (6 floats per row).
// First term: u = s * x (s may be null: ones), v1 = B u, out = c_1 v1.
__global__ void k_poly_first(long R, int na, const float *__restrict__ Binv, const float *__restrict__ s,
                             const float *__restrict__ x, const float *__restrict__ c, float *__restrict__ v1,
                             float *__restrict__ out) {
    for (long r = blockIdx.x * (long)blockDim.x + threadIdx.x; r < R; r += (long)gridDim.x * blockDim.x) {
        const int I = (int)(r % na);
        float u[6];
        for (int k = 0; k < 6; ++k) u[k] = s ? s[6L * I + k] * x[6 * r + k] : x[6 * r + k];
        const float *B = Binv + 36L * I;
        for (int k = 0; k < 6; ++k) {
            float v = 0.f;
            for (int l = 0; l < 6; ++l) v = fmaf(B[6 * k + l], u[l], v);
            v1[6 * r + k] = v;
            if (out) out[6 * r + k] = c[0] * v;
        }
    }
}

// Next term: vout = B (Ehat vin), out += c_k vout.  Warp per row: lane
// s < 27 takes neighbour slot s, the 6-vector is reduced across the warp.
__global__ void __launch_bounds__(kBlock) k_poly_next(long R, int na, const int *__restrict__ nbr,
                                                      const float *__restrict__ Ehat, const float *__restrict__ Binv,
                                                      const float *__restrict__ c, int k, const float *__restrict__ vin,
                                                      float *__restrict__ vout, float *__restrict__ out,
                                                      const int *__restrict__ stop) {
    if (vc_stopped(stop)) return;
    const int lane = threadIdx.x & 31;
    for (long r = (blockIdx.x * (long)blockDim.x + threadIdx.x) / 32; r < R;
         r += (long)gridDim.x * blockDim.x / 32) {
        const int I = (int)(r % na);
        const long base = r - I;
        float t[6] = {0, 0, 0, 0, 0, 0};
        const int J = lane < 27 ? nbr[27L * I + lane] : -1;
        if (J >= 0) {
            const float2 *v2 = reinterpret_cast<const float2 *>(vin + 6 * (base + J));
            const float2 x0 = v2[0], x1 = v2[1], x2 = v2[2];
            const float v[6] = {x0.x, x0.y, x1.x, x1.y, x2.x, x2.y};
            block6_apply(Ehat + (27L * I + lane) * 36, v, t);
        }
        for (int a = 0; a < 6; ++a) t[a] = warp_sum(t[a]);
        if (lane < 6) {
            const float *B = Binv + 36L * I + 6 * lane;
            float v = 0.f;
            for (int b = 0; b < 6; ++b) v = fmaf(B[b], t[b], v);
            vout[6 * r + lane] = v;
            if (out) out[6 * r + lane] += c[k] * v;
        }
    }
}

// Energy of y = s * wv: d = (Ehat y - x) / (6 na) and per-CTA loss partials
// (1/2 y . Ehat y - y . x) / (6 na).  Warp per row as in k_poly_next.
__global__ void __launch_bounds__(kBlock) k_poly_energy(long R, int na, const int *__restrict__ nbr,
                                                        const float *__restrict__ Ehat, const float *__restrict__ s,
                                                        const float *__restrict__ wv, const float *__restrict__ x,
                                                        float *__restrict__ d, double *__restrict__ lossp) {
    __shared__ double sh[kWarpsPerBlock];
    const int lane = threadIdx.x & 31;
    const float inv = 1.0f / (6.0f * na);
    double acc = 0.0;
    for (long r = (blockIdx.x * (long)blockDim.x + threadIdx.x) / 32; r < R;
         r += (long)gridDim.x * blockDim.x / 32) {
        const int I = (int)(r % na);
        const long base = r - I;
        float t[6] = {0, 0, 0, 0, 0, 0};
        const int J = lane < 27 ? nbr[27L * I + lane] : -1;
        if (J >= 0) {
            float y[6];
            for (int b = 0; b < 6; ++b) y[b] = s[6L * J + b] * wv[6 * (base + J) + b];
            block6_apply(Ehat + (27L * I + lane) * 36, y, t);
        }
        for (int a = 0; a < 6; ++a) t[a] = warp_sum(t[a]);
        if (lane < 6) {
            float ey = t[0];
            for (int a = 1; a < 6; ++a)
                if (lane == a) ey = t[a];
            const float y = s[6L * I + lane] * wv[6 * r + lane], xv = x[6 * r + lane];
            d[6 * r + lane] = (ey - xv) * inv;
            acc += (0.5 * (double)y * ey - (double)y * xv) * inv;
        }
    }
    const double tot = block_sum(acc, sh);
    if (threadIdx.x == 0) lossp[blockIdx.x] = tot;
}

// Gradient of the network's output Y (s = exp(Y/2)), summed over the batch
// in order:  dL/ds = sum_b d * wv + x * md  (md = M(s * d)),  dY = dL/ds * s / 2.
__global__ void k_poly_grad_s(int na, int B, const float *__restrict__ s, const float *__restrict__ d,
                              const float *__restrict__ wv, const float *__restrict__ x,
                              const float *__restrict__ md, float *__restrict__ dY) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 6 * na; i += gridDim.x * blockDim.x) {
        float g = 0.f;
        for (int b = 0; b < B; ++b) {
            const long q = 6L * na * b + i;
            g = fmaf(d[q], wv[q], g);
            g = fmaf(x[q], md[q], g);
        }
        dY[i] = 0.5f * g * s[i];
    }
}

// Per-CTA partials of dL/dc_k = sum (s * d) . v_k, k = 1..3.
__global__ void __launch_bounds__(kBlock) k_poly_grad_c(long R, int na, const float *__restrict__ s,
                                                        const float *__restrict__ d, const float *__restrict__ v1,
                                                        const float *__restrict__ v2, const float *__restrict__ v3,
                                                        double *__restrict__ part) {
    __shared__ double sh[kWarpsPerBlock];
    double a1 = 0, a2 = 0, a3 = 0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < 6 * R; i += (long)gridDim.x * blockDim.x) {
        const double sd = (double)s[i % (6L * na)] * d[i];
        a1 += sd * v1[i];
        a2 += sd * v2[i];
        a3 += sd * v3[i];
    }
    a1 = block_sum(a1, sh);
    a2 = block_sum(a2, sh);
    a3 = block_sum(a3, sh);
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x] = a1;
        part[3 * blockIdx.x + 1] = a2;
        part[3 * blockIdx.x + 2] = a3;
    }
}

__global__ void __launch_bounds__(kBlock) k_poly_grad_c_sum(int G, const double *__restrict__ part,
                                                            float *__restrict__ gc) {
    __shared__ double sh[kWarpsPerBlock];
    for (int k = 0; k < kTerms; ++k) {
        double a = 0;
        for (int i = threadIdx.x; i < G; i += blockDim.x) a += part[3 * i + k];
        a = block_sum(a, sh);
        if (threadIdx.x == 0) gc[k] = (float)a;
    }
}

// Gram partials for the least-squares start of c: H_kl = v_k . Ehat v_l,
// g_k = v_k . x (per CTA, 9 + 3 values).  Warp per row.
__global__ void __launch_bounds__(kBlock) k_poly_gram(long R, int na, const int *__restrict__ nbr,
                                                      const float *__restrict__ Ehat, const float *__restrict__ v1,
                                                      const float *__restrict__ v2, const float *__restrict__ v3,
                                                      const float *__restrict__ x, double *__restrict__ part) {
    __shared__ double sh[kWarpsPerBlock];
    const int lane = threadIdx.x & 31;
    const float *V[3] = {v1, v2, v3};
    double acc[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (long r = (blockIdx.x * (long)blockDim.x + threadIdx.x) / 32; r < R;
         r += (long)gridDim.x * blockDim.x / 32) {
        const int I = (int)(r % na);
        const long base = r - I;
        const int J = lane < 27 ? nbr[27L * I + lane] : -1;
        for (int l = 0; l < 3; ++l) {
            float t[6] = {0, 0, 0, 0, 0, 0};
            if (J >= 0) {
                const float *e = Ehat + (27L * I + lane) * 36;
                const float *v = V[l] + 6 * (base + J);
                for (int a = 0; a < 6; ++a)
                    for (int b = 0; b < 6; ++b) t[a] = fmaf(e[6 * a + b], v[b], t[a]);
            }
            for (int a = 0; a < 6; ++a) t[a] = warp_sum(t[a]);
            if (lane == 0)
                for (int k = 0; k < 3; ++k)
                    for (int a = 0; a < 6; ++a) acc[3 * k + l] += (double)V[k][6 * r + a] * t[a];
        }
        if (lane == 0)
            for (int k = 0; k < 3; ++k)
                for (int a = 0; a < 6; ++a) acc[9 + k] += (double)V[k][6 * r + a] * x[6 * r + a];
    }
    for (int q = 0; q < 12; ++q) {
        const double tot = block_sum(acc[q], sh);
        if (threadIdx.x == 0) part[12L * blockIdx.x + q] = tot;
    }
}

// s = exp(Y / 2).
__global__ void k_scales(int n, const float *__restrict__ Y, float *__restrict__ s) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s[i] = expf(0.5f * Y[i]);
}

// Both coarse corrections in level-2 modes: g = D^-1/2 (s * wv) + P e1,
// written over c2 (one prolongation then adds Z2 g = Z1 e1 + Z2 D^-1/2 y).
__global__ void k_poly_out_e1(int na, const float *__restrict__ s, const float *__restrict__ wv,
                              const float *__restrict__ dsq, const int *__restrict__ parent,
                              const float *__restrict__ pdel, const float *__restrict__ e1, float *__restrict__ g,
                              const int *__restrict__ stop) {
    if (vc_stopped(stop)) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 6 * na; i += gridDim.x * blockDim.x) {
        const int J = i / 6, l = i % 6;
        float pe[6];
        child_coeffs(J, parent, pdel, e1, pe);
        const float d = dsq[i];
        g[i] = (d > 0.f ? s[i] * wv[i] / d : 0.f) + pe[l];
    }
}

// c1 = P^T c2: the coarse level's residual from its children's (row k of
// each child's mode map transposed), children summed in table order; every
// load of the eight children is issued before the first sum.
__global__ void k_restrict_parent(int na1, const int *__restrict__ children, const float *__restrict__ pdel,
                                  const float *__restrict__ c2, float *__restrict__ c1, const int *__restrict__ stop) {
    if (vc_stopped(stop)) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 6 * na1; i += gridDim.x * blockDim.x) {
        const int P = i / 6, k = i % 6;
        int J[8];
        float g[8][3], dl[8][4];
#pragma unroll
        for (int ch = 0; ch < 8; ++ch) J[ch] = children[8L * P + ch];
#pragma unroll
        for (int ch = 0; ch < 8; ++ch) {
            const int j = J[ch] < 0 ? 0 : J[ch];
            // the three values row k combines, and the offsets they are weighted by
            const int a0 = k < 3 ? k : (k == 3 ? 1 : 0), a1 = k < 3 ? k : (k == 5 ? 1 : 2);
            g[ch][0] = c2[6L * j + a0];
            g[ch][1] = c2[6L * j + a1];
            g[ch][2] = c2[6L * j + k];
            dl[ch][0] = pdel[4L * j];
            dl[ch][1] = pdel[4L * j + 1];
            dl[ch][2] = pdel[4L * j + 2];
            dl[ch][3] = pdel[4L * j + 3];
        }
        float acc = 0.f;
#pragma unroll
        for (int ch = 0; ch < 8; ++ch) {
            if (J[ch] < 0) continue;
            const float dx = dl[ch][0], dy = dl[ch][1], dz = dl[ch][2], ratio = dl[ch][3];
            float v;
            switch (k) {
                case 0: case 1: case 2: v = g[ch][2]; break;
                case 3: v = -dz * g[ch][0] + dy * g[ch][1] + ratio * g[ch][2]; break;   // g1, g2, g3
                case 4: v = dz * g[ch][0] - dx * g[ch][1] + ratio * g[ch][2]; break;    // g0, g2, g4
                default: v = -dy * g[ch][0] + dx * g[ch][1] + ratio * g[ch][2]; break;  // g0, g1, g5
            }
            acc += v;
        }
        c1[i] = acc;
    }
}

int tiles(long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

// --------------------------------------------------------------- host --

void Learned::init_weights(unsigned seed) {
    const Layout L = layout();
    std::vector<float> w(L.total, 0.f);
    std::mt19937 rng(seed);
    auto fill = [&](size_t off, int rows, int cols, float gain) {
        std::normal_distribution<float> nd(0.f, gain / std::sqrt((float)cols));
        for (size_t i = 0; i < (size_t)rows * cols; ++i) w[off + i] = nd(rng);
    };
    fill(L.W0, kF, kNFeat, std::sqrt(2.f));
    for (int l = 0; l < kLayers; ++l) fill(L.W[l], kF, kA, std::sqrt(2.f));
    fill(L.Wd, kOut, kF, 0.01f);
    w[L.c0] = 1.f;  // block Jacobi until fitted
    host_w = w;
    uploaded = false;
    have_weights = true;
    fitted = false;
    trained_steps = 0;
}

// Level-2 aggregation, E2 blocks, scaling, block-Jacobi inverses and node
// features for the current K.
void setup_learned_level(ofea_ctx *c) {
    Coarse &C2 = c->coarse2;
    Learned &N = c->learned;
    geometry_join(c);
    if (!c->coarse.geom_ok) fail(OFEA_ERR_STATE, "coarse level missing");
    if (!C2.geom_ok) {
        build_aggregation_fine(c);
        N.links_ok = false;
    }
    if (!N.links_ok) {
        // parent aggregate of every child and the change of mode origin/scale
        const Coarse &C1 = c->coarse;
        const int na2 = C2.na;
        std::vector<int> par(na2);
        std::vector<float> pd(4L * na2);
        const double ratio = C1.inv_scale / C2.inv_scale;
        for (int J = 0; J < na2; ++J) {
            int pc[3];
            for (int d = 0; d < 3; ++d) pc[d] = C1.ext[d] > 0 ? C2.agg_cell_h[3L * J + d] / 2 : 0;
            const int P = C1.cell_agg_h[((long)pc[0] * C1.nc[1] + pc[1]) * C1.nc[2] + pc[2]];
            if (P < 0) fail(OFEA_ERR_STATE, "learned level not nested in the coarse level");
            par[J] = P;
            for (int d = 0; d < 3; ++d)
                pd[4L * J + d] = (float)((C2.centroid_h[3L * J + d] - C1.centroid_h[3L * P + d]) * C1.inv_scale);
            pd[4L * J + 3] = (float)ratio;
        }
        std::vector<int> ch(8L * C1.na, -1), nch(C1.na, 0);
        for (int J = 0; J < na2; ++J) {
            const int P = par[J];
            if (nch[P] >= 8) fail(OFEA_ERR_STATE, "learned level: more than 8 children in a coarse cell");
            ch[8L * P + nch[P]++] = J;
        }
        N.parent.upload(par.data(), na2, c->stream);
        N.children.upload(ch.data(), ch.size(), c->stream);
        N.pdel.upload(pd.data(), pd.size(), c->stream);
        N.invdeg.ensure(na2);
        k_invdeg<<<grid_for(c, na2, kBlock), kBlock, 0, c->stream>>>(na2, C2.nbr.p, N.invdeg.p);
        OFEA_CHECK_LAUNCH();
        OFEA_CUDA(cudaStreamSynchronize(c->stream));
        N.links_ok = true;
    }
    if (C2.K_ok) return;
    cudaStream_t s = c->stream;
    const int na = C2.na;
    const int nchunk = 1;
    OFEA_CUDA(cudaMemsetAsync(c->err_flag.p, 0, sizeof(int), s));
    setup_mark(c, "geometry");
    coarse_E_partials(c, C2, nchunk);
    setup_mark(c, "galerkin_level2");
    N.Eb.ensure((size_t)na * 27 * 36);
    N.Ehat.ensure((size_t)na * 27 * 36);
    N.dsq.ensure((size_t)6 * na);
    N.feat.ensure(na);
    k_e2_blocks<<<grid_for(c, (long)na * 27 * 36, kBlock), kBlock, 0, s>>>(na, nchunk, C2.nbr.p, C2.part.p, N.Eb.p);
    k_e2_scale<<<grid_for(c, na, kBlock), kBlock, 0, s>>>(na, N.Eb.p, N.dsq.p, N.feat.p);
    k_e2_hat<<<grid_for(c, (long)na * 27 * 36, kBlock), kBlock, 0, s>>>(na, C2.nbr.p, N.Eb.p, N.dsq.p, N.Ehat.p);
    OFEA_CHECK_LAUNCH();
    // centre the stiffness feature on its mean (host, na values)
    std::vector<float> f(na);
    OFEA_CUDA(cudaMemcpyAsync(f.data(), N.feat.p, sizeof(float) * na, cudaMemcpyDeviceToHost, s));
    OFEA_CUDA(cudaMemcpyAsync(c->herr.p, c->err_flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    OFEA_CUDA(cudaStreamSynchronize(s));
    if (c->herr.p[0]) fail(OFEA_ERR_CAPACITY, "learned level: cells smaller than the element couplings");
    setup_mark(c, "level2_blocks");
    double mean = 0;
    for (float v : f) mean += v;
    mean /= std::max(na, 1);
    for (float &v : f) v = (float)(v - mean);
    N.feat.upload(f.data(), na, s);
    N.Binv.ensure(36L * na);
    N.X0.ensure((size_t)kNFeat * na);
    k_block_inv6<<<grid_for(c, na, 128), 128, 0, s>>>(na, N.Ehat.p, N.Binv.p);
    k_node_features<<<grid_for(c, na, kBlock), kBlock, 0, s>>>(na, N.feat.p, N.invdeg.p, N.Binv.p, N.X0.p);
    OFEA_CHECK_LAUNCH();
    C2.cvec.ensure(6L * na);
    N.shifted.ensure(6L * na);
    N.sigma.ensure(4);
    N.scale.ensure(6L * na);
    setup_mark(c, "level2_inverse_features");
    C2.K_ok = true;
}


// Both coarse levels for the LEARNED solver: the nested level's Galerkin
// blocks are assembled from K, and, when the coarse level's E is missing, it
// is formed from them (E1 = P^T E2 P) instead of a second pass over K.
void setup_learned_levels(ofea_ctx *c) {
    setup_coarse_geometry(c, c->coarse_nodes);
    const bool need_e1 = !c->coarse.K_ok;
    setup_learned_level(c);
    if (need_e1) {
        Coarse &C1 = c->coarse;
        double *E = coarse_begin_E(c);
        k_e1_from_e2<<<std::min(C1.na * 27, c->num_sms * 16), 64, 0, c->stream>>>(
            C1.na, C1.m, C1.nbr.p, c->learned.children.p, c->coarse2.agg_cell.p, c->learned.pdel.p,
            c->learned.Eb.p, E);
        OFEA_CHECK_LAUNCH();
        setup_mark(c, "e1_from_e2");
        coarse_finish(c);
    }
}

static void ensure_rows(ofea_ctx *c, long Rp) {
    Learned &N = c->learned;
    const long R = c->coarse2.na;  // network rows: one per aggregate
    if (!N.Z0.p || N.Z0.n < (size_t)(R * kF)) {
        N.Z0.ensure(R * kF);
        for (int l = 0; l <= kLayers; ++l) N.H[l].ensure(R * kF);
        for (int l = 0; l < kLayers; ++l) {
            N.A[l].ensure(R * kA);
            N.Zl[l].ensure(R * kF);
        }
        N.Y.ensure(R * kOut);
        N.dY.ensure(R * kOut);
        N.dH.ensure(R * kF);
        N.dZ.ensure(R * kF);
        N.dA.ensure(R * kA);
    }
    if (N.cap_rows >= Rp && N.pv[0].p) return;
    for (auto &b : N.pv) b.ensure(6 * Rp);
    N.batch_src.ensure(6 * Rp);
    N.cap_rows = Rp;
}

static void upload_weights(ofea_ctx *c) {
    Learned &N = c->learned;
    const size_t n = Learned::layout().total;
    if (!N.have_weights) N.init_weights(1234u);
    if (N.uploaded && N.w.p) return;
    N.w.upload(N.host_w.data(), n, c->stream);
    N.g.ensure(n);
    if (!N.m.p || N.m.n < n) {
        N.m.ensure(n);
        N.v.ensure(n);
        OFEA_CUDA(cudaMemsetAsync(N.m.p, 0, sizeof(float) * n, c->stream));
        OFEA_CUDA(cudaMemsetAsync(N.v.p, 0, sizeof(float) * n, c->stream));
    }
    N.uploaded = true;
}

// The flag a tensor-core product sets when one of its waits ran out.
static void tc_flag(ofea_ctx *c) {
    Learned &N = c->learned;
    if (!N.tc_err.p) {
        N.tc_err.ensure(1);
        OFEA_CUDA(cudaMemsetAsync(N.tc_err.p, 0, sizeof(int), c->stream));
    }
}

// A tensor-core product whose wait ran out leaves the flag set: fail the call.
static void check_tc(ofea_ctx *c) {
    Learned &N = c->learned;
    if (!N.tc_err.p) return;
    int h = 0;
    OFEA_CUDA(cudaMemcpyAsync(&h, N.tc_err.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    OFEA_CUDA(cudaStreamSynchronize(c->stream));
    if (h) {
        OFEA_CUDA(cudaMemsetAsync(N.tc_err.p, 0, sizeof(int), c->stream));
        fail(OFEA_ERR_TIMEOUT, "learned stage: a tensor-core product's wait ran out");
    }
}

// Network forward over the aggregates (input: the node features), scalings s.
static void gnn_forward(ofea_ctx *c, cudaStream_t s) {
    Learned &N = c->learned;
    const Learned::Layout L = Learned::layout();
    const long R = c->coarse2.na;
    const int na = (int)R;
    const float *w = N.w.p;
    const int G = grid_for(c, R * kF, kBlock);
    tc_flag(c);
    // Z = X W^T + b on the tensor cores (BF16 operands, FP32 accumulation)
    auto dense = [&](int O, int K, const float *X, size_t offW, size_t offb, float *Z, float *H) {
        tc_gemm(s, (int)R, O, K, 0, TcOperand{X, K, 1}, TcOperand{w + offW, K, 1},
                TcEpilogue{kTcForward, Z, H, w + offb, 0}, N.tc_err.p);
    };
    dense(kF, kNFeat, N.X0.p, L.W0, L.b0, N.Z0.p, N.H[0].p);
    for (int l = 0; l < kLayers; ++l) {
        k_gnn_aggregate<<<G, kBlock, 0, s>>>(R, na, c->coarse2.nbr.p, N.invdeg.p, N.H[l].p, N.A[l].p);
        dense(kF, kA, N.A[l].p, L.W[l], L.b[l], N.Zl[l].p, N.H[l + 1].p);
    }
    dense(kOut, kF, N.H[kLayers].p, L.Wd, L.bd, N.Y.p, nullptr);
    k_scales<<<grid_for(c, 6 * R, kBlock), kBlock, 0, s>>>((int)(6 * R), N.Y.p, N.scale.p);
    OFEA_CHECK_LAUNCH();
}

// Network backward from dY (in N.dY), parameter gradient into N.g (all but c).
static void gnn_backward(ofea_ctx *c) {
    Learned &N = c->learned;
    const Learned::Layout L = Learned::layout();
    cudaStream_t s = c->stream;
    const long R = c->coarse2.na;
    const int na = (int)R;
    const float *w = N.w.p;
    float *g = N.g.p;
    const long chunk = 256;
    const int S = (int)((R + chunk - 1) / chunk);
    N.part.ensure((size_t)S * (kF * kA + kF));
    tc_flag(c);
    // weight gradient dZ^T X on the tensor cores, one partial per chunk of
    // rows (output transposed: k_in is the tile's M), the bias sums beside it;
    // partials summed in chunk order
    auto wgrad = [&](int O, int K, const float *dZ, const float *X, size_t offW, size_t offb) {
        const int nout = O * K + O;
        tc_gemm(s, K, O, R, chunk, TcOperand{X, 1, K}, TcOperand{dZ, 1, O},
                TcEpilogue{kTcTransposedPartial, N.part.p, nullptr, nullptr, (long)nout}, N.tc_err.p);
        k_bias_partials<<<dim3(tiles(O, 64), S), 64, 0, s>>>(R, O, K, chunk, dZ, N.part.p);
        k_wgrad_sum<<<tiles(nout, 256), 256, 0, s>>>(S, O, K, N.part.p, g + offW, g + offb);
    };
    // dX = dZ W on the tensor cores
    auto bwd_data = [&](int O, int K, const float *dZ, size_t offW, float *dX) {
        tc_gemm(s, (int)R, K, O, 0, TcOperand{dZ, O, 1}, TcOperand{w + offW, 1, K},
                TcEpilogue{kTcRowMajor, dX, nullptr, nullptr, 0}, N.tc_err.p);
    };
    wgrad(kOut, kF, N.dY.p, N.H[kLayers].p, L.Wd, L.bd);
    bwd_data(kOut, kF, N.dY.p, L.Wd, N.dH.p);
    const int Gf = grid_for(c, R * kF, kBlock);
    k_relu_bwd<<<Gf, kBlock, 0, s>>>(R * kF, N.dH.p, N.Zl[kLayers - 1].p, N.dZ.p);
    for (int l = kLayers - 1; l >= 0; --l) {
        wgrad(kF, kA, N.dZ.p, N.A[l].p, L.W[l], L.b[l]);
        bwd_data(kF, kA, N.dZ.p, L.W[l], N.dA.p);
        const float *Zprev = l > 0 ? N.Zl[l - 1].p : N.Z0.p;
        k_gnn_aggregate_bwd<<<Gf, kBlock, 0, s>>>(R, na, c->coarse2.nbr.p, N.invdeg.p, N.dA.p, Zprev, N.dZ.p);
    }
    wgrad(kF, kNFeat, N.dZ.p, N.X0.p, L.W0, L.b0);
    OFEA_CHECK_LAUNCH();
}

// The stage's terms after the first (pv[0] and its share of out present).
static void apply_M_rest(ofea_ctx *c, long Rp, const float *coef, float *out) {
    Learned &N = c->learned;
    const Coarse &C2 = c->coarse2;
    const int na = C2.na;
    const int Gw = grid_for(c, 32 * Rp, kBlock);
    for (int k = 1; k < kTerms; ++k)
        k_poly_next<<<Gw, kBlock, 0, c->stream>>>(Rp, na, C2.nbr.p, N.Ehat.p, N.Binv.p, coef, k, N.pv[k - 1].p,
                                                  N.pv[k].p, out, c->vc_stop);
    OFEA_CHECK_LAUNCH();
}

// out = M(s * x) over Rp rows; the basis v_k lands in pv[0..2].  s and c may be null.
static void apply_M(ofea_ctx *c, long Rp, const float *s_, const float *x, const float *coef, float *out) {
    Learned &N = c->learned;
    const int na = c->coarse2.na;
    k_poly_first<<<grid_for(c, Rp, kBlock), kBlock, 0, c->stream>>>(Rp, na, N.Binv.p, s_, x, coef, N.pv[0].p, out);
    apply_M_rest(c, Rp, coef, out);
}

// Loss and full gradient (N.g) of a batch of Bsz samples already in N.batch_src.
static void loss_and_grad(ofea_ctx *c, int Bsz) {
    Learned &N = c->learned;
    const Learned::Layout L = Learned::layout();
    const Coarse &C2 = c->coarse2;
    cudaStream_t s = c->stream;
    const int na = C2.na;
    const long Rp = (long)Bsz * na;
    const float *coef = N.w.p + L.c0;
    gnn_forward(c, c->stream);
    float *wv = N.pv[3].p, *d = N.pv[4].p, *md = N.pv[5].p;
    // y = s * M(s x): basis v_k of the first chain kept in pv[6..8]
    apply_M(c, Rp, N.scale.p, N.batch_src.p, coef, wv);
    for (int k = 0; k < kTerms; ++k)
        OFEA_CUDA(cudaMemcpyAsync(N.pv[6 + k].p, N.pv[k].p, sizeof(float) * 6 * Rp, cudaMemcpyDeviceToDevice, s));
    const int Ge = std::min(kMaxGrid, grid_for(c, 32 * Rp, kBlock));
    N.lossp.ensure(kMaxGrid);
    N.nlossp = Ge;
    k_poly_energy<<<Ge, kBlock, 0, s>>>(Rp, na, C2.nbr.p, N.Ehat.p, N.scale.p, wv, N.batch_src.p, d, N.lossp.p);
    OFEA_CHECK_LAUNCH();
    apply_M(c, Rp, N.scale.p, d, coef, md);
    k_poly_grad_s<<<grid_for(c, 6L * na, kBlock), kBlock, 0, s>>>(na, Bsz, N.scale.p, d, wv, N.batch_src.p, md,
                                                                  N.dY.p);
    const int Gc = std::min(kMaxGrid, grid_for(c, 6 * Rp, kBlock));
    N.cpart.ensure(3L * kMaxGrid);
    k_poly_grad_c<<<Gc, kBlock, 0, s>>>(Rp, na, N.scale.p, d, N.pv[6].p, N.pv[7].p, N.pv[8].p, N.cpart.p);
    k_poly_grad_c_sum<<<1, kBlock, 0, s>>>(Gc, N.cpart.p, N.g.p + L.c0);
    OFEA_CHECK_LAUNCH();
    gnn_backward(c);
}

static double read_loss(ofea_ctx *c) {
    Learned &N = c->learned;
    std::vector<double> h(N.nlossp);
    OFEA_CUDA(cudaMemcpyAsync(h.data(), N.lossp.p, sizeof(double) * N.nlossp, cudaMemcpyDeviceToHost, c->stream));
    OFEA_CUDA(cudaStreamSynchronize(c->stream));
    double s = 0;
    for (double v : h) s += v;
    return s;
}

// Network input of the learned level for a fine-level vector t (FP32): the
// level-1 correction e1 = E1^-1 Z1^T t, the level-2 restriction c2 = Z2^T t,
// then S = D^-1/2 (c2 - E2 P e1) (the training samples' inputs).
static void learned_input(ofea_ctx *c, const float *t) {
    Coarse &C1 = c->coarse;
    Coarse &C2 = c->coarse2;
    Learned &N = c->learned;
    cudaStream_t s = c->stream;
    const int na = C2.na;
    restrict_level(c, C1, t, C1.cvec.p);
    coarse_gemv(c, C1.cvec.p, C1.evec.p);
    restrict_level(c, C2, t, C2.cvec.p);
    k_lrn_shift<false><<<grid_for(c, 32L * na, kBlock), kBlock, 0, s>>>(na, C2.nbr.p, N.Ehat.p, N.dsq.p, N.parent.p,
                                                                  N.pdel.p, C1.evec.p, C2.cvec.p, N.shifted.p);
    OFEA_CHECK_LAUNCH();
}

// One training sample from a device FP64 residual r (n entries).
void learned_add_sample(ofea_ctx *c, const double *d_r) {
    Coarse &C2 = c->coarse2;
    Learned &N = c->learned;
    if (N.nsamples >= N.max_samples) return;
    cudaStream_t s = c->stream;
    const int na = C2.na;
    N.r32.ensure(c->n);
    k_f64_to_f32<<<grid_for(c, c->n, kBlock), kBlock, 0, s>>>(c->n, d_r, N.r32.p);
    learned_input(c, N.r32.p);
    k_gnn_sigma<<<1, kBlock, 0, s>>>(na, N.shifted.p, N.sigma.p);
    k_gnn_sample<<<grid_for(c, 6L * na, kBlock), kBlock, 0, s>>>(na, N.shifted.p, N.sigma.p,
                                                                 N.data.p + (size_t)N.nsamples * 6 * na);
    OFEA_CHECK_LAUNCH();
    N.nsamples++;
}



void learned_begin_dataset(ofea_ctx *c, int max_samples) {
    Learned &N = c->learned;
    N.max_samples = max_samples;
    N.nsamples = 0;
    N.data.ensure((size_t)max_samples * 6 * c->coarse2.na);
}

// The energy-optimal constant coefficients c over all samples (s = 1): the
// 3 x 3 system H c = g, H_kl = sum v_k . Ehat v_l, g_k = sum v_k . x.
static void fit_coefficients(ofea_ctx *c, int chunk) {
    Learned &N = c->learned;
    const Learned::Layout L = Learned::layout();
    const int na = c->coarse2.na;
    cudaStream_t s = c->stream;
    double H[3][3] = {}, g[3] = {};
    std::vector<double> hp;
    N.cpart.ensure(12L * kMaxGrid);
    for (int b0 = 0; b0 < N.nsamples; b0 += chunk) {
        const int nb = std::min(chunk, N.nsamples - b0);
        const long Rp = (long)nb * na;
        const float *x = N.data.p + (size_t)b0 * 6 * na;
        apply_M(c, Rp, nullptr, x, nullptr, nullptr);
        const int G = std::min(kMaxGrid, grid_for(c, 32 * Rp, kBlock));
        k_poly_gram<<<G, kBlock, 0, s>>>(Rp, na, c->coarse2.nbr.p, N.Ehat.p, N.pv[0].p, N.pv[1].p, N.pv[2].p, x,
                                         N.cpart.p);
        OFEA_CHECK_LAUNCH();
        hp.resize(12L * G);
        OFEA_CUDA(cudaMemcpyAsync(hp.data(), N.cpart.p, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, s));
        OFEA_CUDA(cudaStreamSynchronize(s));
        for (int q = 0; q < G; ++q) {
            for (int k = 0; k < 3; ++k)
                for (int l = 0; l < 3; ++l) H[k][l] += hp[12L * q + 3 * k + l];
            for (int k = 0; k < 3; ++k) g[k] += hp[12L * q + 9 + k];
        }
    }
    // symmetrise, then Gaussian elimination with partial pivoting (3 x 3)
    double A[3][4];
    for (int k = 0; k < 3; ++k) {
        for (int l = 0; l < 3; ++l) A[k][l] = 0.5 * (H[k][l] + H[l][k]);
        A[k][3] = g[k];
    }
    for (int k = 0; k < 3; ++k) {
        int p = k;
        for (int i = k + 1; i < 3; ++i)
            if (std::fabs(A[i][k]) > std::fabs(A[p][k])) p = i;
        for (int j = 0; j < 4; ++j) std::swap(A[k][j], A[p][j]);
        if (!(std::fabs(A[k][k]) > 0)) return;  // degenerate: keep the current coefficients
        for (int i = 0; i < 3; ++i) {
            if (i == k) continue;
            const double f = A[i][k] / A[k][k];
            for (int j = k; j < 4; ++j) A[i][j] -= f * A[k][j];
        }
    }
    float cf[3];
    for (int k = 0; k < 3; ++k) {
        cf[k] = (float)(A[k][3] / A[k][k]);
        if (!std::isfinite(cf[k])) return;
    }
    for (int k = 0; k < 3; ++k) N.host_w[L.c0 + k] = cf[k];
    OFEA_CUDA(cudaMemcpyAsync(N.w.p + L.c0, cf, sizeof(cf), cudaMemcpyHostToDevice, s));
    OFEA_CUDA(cudaStreamSynchronize(s));
    N.fitted = true;
}

// Adam training on the collected samples.  loss0 / loss1: the energy loss of
// the first batch before the first step and after the last.
void learned_train(ofea_ctx *c, int steps, int batch, float lr, unsigned seed, double *loss0, double *loss1) {
    Learned &N = c->learned;
    if (N.nsamples < 1) fail(OFEA_ERR_STATE, "no training samples");
    upload_weights(c);
    const int na = c->coarse2.na;
    const int B = std::min(batch, N.nsamples);
    ensure_rows(c, (long)B * na);
    if (!N.fitted) fit_coefficients(c, B);
    std::mt19937 rng(seed);
    const size_t n = Learned::layout().total;
    cudaStream_t s = c->stream;
    double first = 0, last = 0;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    std::vector<int> idx(N.nsamples), first_batch;
    auto load_batch = [&](const int *ids) {
        for (int b = 0; b < B; ++b)
            OFEA_CUDA(cudaMemcpyAsync(N.batch_src.p + (size_t)b * 6 * na, N.data.p + (size_t)ids[b] * 6 * na,
                                      sizeof(float) * 6 * na, cudaMemcpyDeviceToDevice, s));
    };
    for (int it = 0; it < steps; ++it) {
        // batch: B distinct samples
        for (int i = 0; i < N.nsamples; ++i) idx[i] = i;
        for (int i = 0; i < B; ++i) std::swap(idx[i], idx[i + rng() % (N.nsamples - i)]);
        load_batch(idx.data());
        loss_and_grad(c, B);
        if (it == 0) {
            first = read_loss(c);
            first_batch.assign(idx.begin(), idx.begin() + B);
        }
        ++N.trained_steps;
        const float c1 = 1.f - std::pow(b1, (float)N.trained_steps);
        const float c2 = 1.f - std::pow(b2, (float)N.trained_steps);
        k_adam<<<grid_for(c, (long)n, kBlock), kBlock, 0, s>>>((long)n, N.w.p, N.g.p, N.m.p, N.v.p, lr, b1, b2,
                                                              eps, c1, c2);
        OFEA_CHECK_LAUNCH();
    }
    if (steps > 0) {
        load_batch(first_batch.data());
        loss_and_grad(c, B);
        last = read_loss(c);
    }
    // keep the host copy in step with the device weights
    N.host_w.resize(n);
    OFEA_CUDA(cudaMemcpyAsync(N.host_w.data(), N.w.p, sizeof(float) * n, cudaMemcpyDeviceToHost, s));
    OFEA_CUDA(cudaStreamSynchronize(s));
    N.inference_ready = false;
    check_tc(c);
    if (loss0) *loss0 = first;
    if (loss1) *loss1 = last;
}

// Loss and full parameter gradient for given inputs (B x na x 6, host).
void learned_gradient(ofea_ctx *c, const float *h_x, int B, double *loss, float *h_grad) {
    Learned &N = c->learned;
    upload_weights(c);
    const int na = c->coarse2.na;
    const long Rp = (long)B * na;
    ensure_rows(c, Rp);
    OFEA_CUDA(cudaMemcpyAsync(N.batch_src.p, h_x, sizeof(float) * 6 * Rp, cudaMemcpyHostToDevice, c->stream));
    loss_and_grad(c, B);
    *loss = read_loss(c);
    const size_t n = Learned::layout().total;
    OFEA_CUDA(cudaMemcpyAsync(h_grad, N.g.p, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
    OFEA_CUDA(cudaStreamSynchronize(c->stream));
    check_tc(c);
}

// The coarse part of the LEARNED V-cycle: x += Z1 e1 + Z2 D^-1/2 y with
// e1 = E1^-1 Z1^T t (the exact level) and y = s * M(s * D^-1/2 (c2 - E2 P e1))
// (the learned stage), c2 = Z2^T t.  One restriction and one prolongation
// pass over the fine vector serve both levels (Z1 = Z2 P): c1 = P^T c2, and
// the level-1 correction joins the stage's output in level-2 modes.
void learned_coarse_correct(ofea_ctx *c, const float *t, float *x) {
    Coarse &C1 = c->coarse;
    Coarse &C2 = c->coarse2;
    Learned &N = c->learned;
    const Learned::Layout L = Learned::layout();
    cudaStream_t s = c->stream;
    const int na = C2.na;
    restrict_level(c, C2, t, C2.cvec.p);
    k_restrict_parent<<<grid_for(c, 6L * C1.na, 128), 128, 0, s>>>(C1.na, N.children.p, N.pdel.p, C2.cvec.p,
                                                                 C1.cvec.p, c->vc_stop);
    coarse_gemv(c, C1.cvec.p, C1.evec.p);
    // the shifted residual and the stage's first term in one launch, then the
    // stage's other terms
    float *wv = N.pv[3].p;
    const float *coef = N.w.p + L.c0;
    k_lrn_shift<true><<<grid_for(c, 32L * na, kBlock), kBlock, 0, s>>>(
        na, C2.nbr.p, N.Ehat.p, N.dsq.p, N.parent.p, N.pdel.p, C1.evec.p, C2.cvec.p, N.shifted.p, N.Binv.p,
        N.scale.p, coef, N.pv[0].p, wv, c->vc_stop);
    apply_M_rest(c, na, coef, wv);
    k_poly_out_e1<<<grid_for(c, 6L * na, kBlock), kBlock, 0, s>>>(na, N.scale.p, wv, N.dsq.p, N.parent.p,
                                                                   N.pdel.p, C1.evec.p, C2.cvec.p, c->vc_stop);
    prolong_level(c, C2, C2.cvec.p, x);
    OFEA_CHECK_LAUNCH();
}

// The LEARNED solver's per-K set-up: both coarse levels as in
// setup_learned_levels, with the network's scalings evaluated on the side
// stream beside the coarse level's E1 = P^T E2 P and its factor (the network
// reads the nested level's features alone); the context stream waits for it.
void setup_learned_solver(ofea_ctx *c) {
    Learned &N = c->learned;
    setup_coarse_geometry(c, c->coarse_nodes);
    const bool need_e1 = !c->coarse.K_ok;
    setup_learned_level(c);
    upload_weights(c);
    ensure_rows(c, c->coarse2.na);
    tc_flag(c);
    if (!c->side_stream) OFEA_CUDA(cudaStreamCreateWithFlags(&c->side_stream, cudaStreamNonBlocking));
    cudaEvent_t fork = nullptr, join = nullptr;
    OFEA_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    OFEA_CUDA(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
    bool forked = false;
    try {
        OFEA_CUDA(cudaEventRecord(fork, c->stream));
        OFEA_CUDA(cudaStreamWaitEvent(c->side_stream, fork, 0));
        forked = true;
        gnn_forward(c, c->side_stream);
        OFEA_CUDA(cudaEventRecord(join, c->side_stream));
        if (need_e1) {
            Coarse &C1 = c->coarse;
            double *E = coarse_begin_E(c);
            k_e1_from_e2<<<std::min(C1.na * 27, c->num_sms * 16), 64, 0, c->stream>>>(
                C1.na, C1.m, C1.nbr.p, N.children.p, c->coarse2.agg_cell.p, N.pdel.p, N.Eb.p, E);
            OFEA_CHECK_LAUNCH();
            setup_mark(c, "e1_from_e2");
            coarse_finish(c);
        }
        OFEA_CUDA(cudaStreamWaitEvent(c->stream, join, 0));
    } catch (...) {
        if (forked) {  // nothing on the context stream may overtake the side stream's work
            cudaEventRecord(join, c->side_stream);
            cudaStreamWaitEvent(c->stream, join, 0);
        }
        cudaEventDestroy(fork);
        cudaEventDestroy(join);
        throw;
    }
    cudaEventDestroy(fork);
    cudaEventDestroy(join);
    setup_mark(c, "network_join");
    N.inference_ready = true;
}

}  // namespace ofea
