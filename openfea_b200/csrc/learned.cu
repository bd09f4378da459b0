// Learned coarse-correction stage of the LEARNED solver.
//
// Level: the nested aggregates of build_aggregation_fine (cells half as wide
// as the exact coarse level's), each with six rigid-body modes Z2.  The
// Galerkin correction of that level, E2^-1 Z2^T t, is what an exact extra
// level would add to the V-cycle; it is too costly to factor, so a small
// graph network approximates it:
//
//   x_I = D_I^-1/2 c_I / sigma  (c = Z2^T t, D = diag E2, sigma its RMS),
//   plus the feature log(mean diag E2_II) - its mean
//   h0  = relu(W0 x + b0)                                   (64 wide)
//   4 layers: a_I = [h_I, sum_J h_J, sum_J dx h_J, sum_J dy h_J, sum_J dz h_J]
//             over the 26 neighbour cells J (offsets dx, dy, dz in {-1,0,1}),
//             h  = relu(W a + b)                             (320 -> 64)
//   y   = Wd h + bd;  correction g_I = sigma D_I^-1/2 y_I,  x += Z2 g.
//
// Training (on the GPU, these kernels): inputs are the restricted residuals
// of plain-PCG iterates on the current matrix, the loss is the energy
//   L(y) = (1/2 y^T Ehat y - y^T x) / (6 na),  Ehat = D^-1/2 E2 D^-1/2,
// whose minimiser is the exact Galerkin correction, so no inverse and no
// displacement targets are needed; Adam, FP32 weights and FP32 accumulation.
// Weight gradients are reduced in a fixed order: training is deterministic.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <random>

#include "precond.cuh"
#include "sell.cuh"
#include "solver_common.cuh"

namespace ofea {

constexpr int kF = 64;        // hidden width
constexpr int kIn = 7;        // 6 scaled residual components + stiffness feature
constexpr int kOut = 6;
constexpr int kA = 5 * kF;    // aggregated features per layer
constexpr int kLayers = 4;

Learned::Layout Learned::layout() {
    Layout L;
    size_t o = 0;
    L.W0 = o; o += (size_t)kF * kIn;
    L.b0 = o; o += kF;
    for (int l = 0; l < kLayers; ++l) {
        L.W[l] = o; o += (size_t)kF * kA;
        L.b[l] = o; o += kF;
    }
    L.Wd = o; o += (size_t)kOut * kF;
    L.bd = o; o += kOut;
    L.total = o;
    return L;
}

namespace {

__device__ __forceinline__ int slot_dx(int s) { return s / 9 - 1; }
__device__ __forceinline__ int slot_dy(int s) { return (s / 3) % 3 - 1; }
__device__ __forceinline__ int slot_dz(int s) { return s % 3 - 1; }

// ------------------------------------------------------------ level data --

// Eb[I][slot][36] from the chunk partials of k_coarse_E_chunks (fixed order).
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
__global__ void k_e2_scale(int na, const int *__restrict__ nbr, const double *__restrict__ Eb,
                           float *__restrict__ dsq, float *__restrict__ Ehat, float *__restrict__ feat) {
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

// ----------------------------------------------------------------- layers --

// x (R x kIn) from normalised scaled residuals (rows of `src`, kOut wide) and
// the stiffness feature of the row's aggregate.
__global__ void k_gnn_input(long R, int na, const float *__restrict__ src, const float *__restrict__ feat,
                            float *__restrict__ X) {
    for (long r = blockIdx.x * (long)blockDim.x + threadIdx.x; r < R; r += (long)gridDim.x * blockDim.x) {
        const int I = (int)(r % na);
        for (int k = 0; k < kOut; ++k) X[r * kIn + k] = src[r * kOut + k];
        X[r * kIn + 6] = feat[I];
    }
}

// Z = X W^T + b (R x O, X is R x K, W is O x K), H = relu(Z) when H != null.
// 64 x 64 tiles, K in chunks of 16, 256 threads with 4 x 4 outputs each.
__global__ void __launch_bounds__(256) k_dense(long R, int O, int K, const float *__restrict__ X,
                                               const float *__restrict__ W, const float *__restrict__ b,
                                               float *__restrict__ Z, float *__restrict__ H) {
    __shared__ float sX[64][17], sW[64][17];
    const long r0 = (long)blockIdx.y * 64;
    const int o0 = blockIdx.x * 64;
    const int tr = threadIdx.x / 16, tc = threadIdx.x % 16;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += 16) {
        for (int v = threadIdx.x; v < 64 * 16; v += 256) {
            const int i = v / 16, k = v % 16;
            sX[i][k] = (r0 + i < R && k0 + k < K) ? X[(r0 + i) * K + k0 + k] : 0.f;
            sW[i][k] = (o0 + i < O && k0 + k < K) ? W[(long)(o0 + i) * K + k0 + k] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            float xa[4], wb[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) xa[a] = sX[tr * 4 + a][k];
#pragma unroll
            for (int q = 0; q < 4; ++q) wb[q] = sW[tc * 4 + q][k];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[a][q] = fmaf(xa[a], wb[q], acc[a][q]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const long r = r0 + tr * 4 + a;
        if (r >= R) continue;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int o = o0 + tc * 4 + q;
            if (o >= O) continue;
            const float z = acc[a][q] + b[o];
            Z[r * O + o] = z;
            if (H) H[r * O + o] = z > 0.f ? z : 0.f;
        }
    }
}

// dX = dZ W  (R x K from R x O times O x K), same tiling.
__global__ void __launch_bounds__(256) k_dense_bwd_data(long R, int O, int K, const float *__restrict__ dZ,
                                                        const float *__restrict__ W, float *__restrict__ dX) {
    __shared__ float sD[64][17], sW[16][65];
    const long r0 = (long)blockIdx.y * 64;
    const int k0 = blockIdx.x * 64;
    const int tr = threadIdx.x / 16, tc = threadIdx.x % 16;
    float acc[4][4] = {};
    for (int o0 = 0; o0 < O; o0 += 16) {
        for (int v = threadIdx.x; v < 64 * 16; v += 256) {
            const int i = v / 16, o = v % 16;
            sD[i][o] = (r0 + i < R && o0 + o < O) ? dZ[(r0 + i) * O + o0 + o] : 0.f;
            const int oo = v / 64, kk = v % 64;
            sW[oo][kk] = (o0 + oo < O && k0 + kk < K) ? W[(long)(o0 + oo) * K + k0 + kk] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int o = 0; o < 16; ++o) {
            float da[4], wb[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) da[a] = sD[tr * 4 + a][o];
#pragma unroll
            for (int q = 0; q < 4; ++q) wb[q] = sW[o][tc * 4 + q];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[a][q] = fmaf(da[a], wb[q], acc[a][q]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const long r = r0 + tr * 4 + a;
        if (r >= R) continue;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = k0 + tc * 4 + q;
            if (k < K) dX[r * K + k] = acc[a][q];
        }
    }
}

// Weight gradient partials: part[s][o*K + k] = sum over rows of chunk s of
// dZ[r][o] X[r][k], part[s][O*K + o] = sum dZ[r][o] (bias).  One thread per
// output, rows in order: summed afterwards in chunk order (deterministic).
__global__ void __launch_bounds__(256) k_wgrad(long R, int O, int K, long chunk, const float *__restrict__ dZ,
                                               const float *__restrict__ X, float *__restrict__ part) {
    const int nout = O * K + O;
    const int s = blockIdx.y;
    const long rb = s * chunk, re = min(R, rb + chunk);
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nout; j += gridDim.x * blockDim.x) {
        float acc = 0.f;
        if (j < O * K) {
            const int o = j / K, k = j % K;
            for (long r = rb; r < re; ++r) acc = fmaf(dZ[r * O + o], X[r * K + k], acc);
        } else {
            const int o = j - O * K;
            for (long r = rb; r < re; ++r) acc += dZ[r * O + o];
        }
        part[(long)s * nout + j] = acc;
    }
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

// a = [h, sum h_J, sum dx h_J, sum dy h_J, sum dz h_J] over the neighbours.
__global__ void k_gnn_aggregate(long R, int na, const int *__restrict__ nbr, const float *__restrict__ H,
                                float *__restrict__ A) {
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
        float *a = A + r * kA;
        a[f] = H[r * kF + f];
        a[kF + f] = s;
        a[2 * kF + f] = sx;
        a[3 * kF + f] = sy;
        a[4 * kF + f] = sz;
    }
}

// dH from dA: the transpose of k_gnn_aggregate (neighbour J sees I at the
// opposite slot, offset negated).  Gather form: no atomics.
__global__ void k_gnn_aggregate_bwd(long R, int na, const int *__restrict__ nbr, const float *__restrict__ dA,
                                    const float *__restrict__ Z, float *__restrict__ dZ) {
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
            d += aJ[kF + f] - slot_dx(sl) * aJ[2 * kF + f] - slot_dy(sl) * aJ[3 * kF + f] -
                 slot_dz(sl) * aJ[4 * kF + f];
        }
        // relu backward of the layer that produced h: dZ = dH (Z > 0)
        dZ[g] = Z[g] > 0.f ? d : 0.f;
    }
}

__global__ void k_relu_bwd(long n, const float *__restrict__ dH, const float *__restrict__ Z, float *__restrict__ dZ) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        dZ[i] = Z[i] > 0.f ? dH[i] : 0.f;
}

// Energy loss gradient dY = (Ehat Y - x) / (6 na) and per-CTA loss partials.
__global__ void __launch_bounds__(kBlock) k_gnn_energy(long R, int na, const int *__restrict__ nbr,
                                                       const float *__restrict__ Ehat, const float *__restrict__ X,
                                                       const float *__restrict__ Y, float *__restrict__ dY,
                                                       double *__restrict__ lossp) {
    __shared__ double sh[kWarpsPerBlock];
    const float inv = 1.0f / (6.0f * na);
    double acc = 0.0;
    for (long r = blockIdx.x * (long)blockDim.x + threadIdx.x; r < R; r += (long)gridDim.x * blockDim.x) {
        const int I = (int)(r % na);
        const long base = r - I;
        float ey[6] = {0, 0, 0, 0, 0, 0};
        for (int sl = 0; sl < 27; ++sl) {
            const int J = nbr[27L * I + sl];
            if (J < 0) continue;
            const float *e = Ehat + (27L * I + sl) * 36;
            const float *y = Y + (base + J) * kOut;
            for (int k = 0; k < 6; ++k)
                for (int l = 0; l < 6; ++l) ey[k] = fmaf(e[6 * k + l], y[l], ey[k]);
        }
        for (int k = 0; k < 6; ++k) {
            const float y = Y[r * kOut + k], x = X[r * kIn + k];
            dY[r * kOut + k] = (ey[k] - x) * inv;
            acc += (0.5 * (double)y * ey[k] - (double)y * x) * inv;
        }
    }
    const double s = block_sum(acc, sh);
    if (threadIdx.x == 0) lossp[blockIdx.x] = s;
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

// ----------------------------------------------------- inference helpers --

// sigma^2 partials of the Jacobi-scaled restricted residual c/dsq.
__global__ void __launch_bounds__(kBlock) k_gnn_sigma(int na, const float *__restrict__ c,
                                                      const float *__restrict__ dsq, double *__restrict__ out) {
    __shared__ double sh[kWarpsPerBlock];
    double acc = 0.0;
    for (int i = threadIdx.x; i < 6 * na; i += blockDim.x) {
        const float d = dsq[i];
        const double v = d > 0.f ? (double)c[i] / d : 0.0;
        acc += v * v;
    }
    const double s = block_sum(acc, sh);
    if (threadIdx.x == 0) out[0] = sqrt(s / (6.0 * na)) + 1e-300;
}

// Network input from the restricted residual: x = c / (dsq sigma), + feature.
__global__ void k_gnn_input_c(int na, const float *__restrict__ c, const float *__restrict__ dsq,
                              const float *__restrict__ feat, const double *__restrict__ sigma,
                              float *__restrict__ X) {
    const float is = (float)(1.0 / sigma[0]);
    for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < na; I += gridDim.x * blockDim.x) {
        for (int k = 0; k < 6; ++k) {
            const float d = dsq[6L * I + k];
            X[(long)I * kIn + k] = d > 0.f ? c[6L * I + k] / d * is : 0.f;
        }
        X[(long)I * kIn + 6] = feat[I];
    }
}

// Coarse correction g = sigma D^-1/2 y, written over c (used as evec by the prolongation).
__global__ void k_gnn_output(int na, const float *__restrict__ Y, const float *__restrict__ dsq,
                             const double *__restrict__ sigma, float *__restrict__ g) {
    const float sg = (float)sigma[0];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 6 * na; i += gridDim.x * blockDim.x) {
        const float d = dsq[i];
        g[i] = d > 0.f ? sg * Y[i] / d : 0.f;
    }
}

// Dataset sample: restricted residual c (FP32, 6 na) -> normalised scaled rows.
__global__ void k_gnn_sample(int na, const float *__restrict__ c, const float *__restrict__ dsq,
                             const double *__restrict__ sigma, float *__restrict__ out) {
    const float is = (float)(1.0 / sigma[0]);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 6 * na; i += gridDim.x * blockDim.x) {
        const float d = dsq[i];
        out[i] = d > 0.f ? c[i] / d * is : 0.f;
    }
}

__global__ void k_f64_to_f32(long n, const double *__restrict__ a, float *__restrict__ b) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
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
    fill(L.W0, kF, kIn, std::sqrt(2.f));
    for (int l = 0; l < kLayers; ++l) fill(L.W[l], kF, kA, std::sqrt(2.f));
    fill(L.Wd, kOut, kF, 0.1f);
    host_w = w;
    uploaded = false;
    have_weights = true;
    trained_steps = 0;
}

// Level-2 aggregation + E2 blocks + scaling for the current K.
void setup_learned_level(ofea_ctx *c) {
    Coarse &C2 = c->coarse2;
    Learned &N = c->learned;
    if (!c->coarse.geom_ok) fail(OFEA_ERR_STATE, "coarse level missing");
    if (!C2.geom_ok) build_aggregation_fine(c);
    if (C2.K_ok) return;
    cudaStream_t s = c->stream;
    const int na = C2.na;
    const int nchunk = (C2.max_agg + 63) / 64;
    C2.part.ensure((size_t)na * nchunk * 27 * 36);
    OFEA_CUDA(cudaMemsetAsync(c->err_flag.p, 0, sizeof(int), s));
    coarse_E_partials(c, C2, nchunk);
    N.Eb.ensure((size_t)na * 27 * 36);
    N.Ehat.ensure((size_t)na * 27 * 36);
    N.dsq.ensure((size_t)6 * na);
    N.feat.ensure(na);
    k_e2_blocks<<<grid_for(c, (long)na * 27 * 36, kBlock), kBlock, 0, s>>>(na, nchunk, C2.nbr.p, C2.part.p, N.Eb.p);
    k_e2_scale<<<grid_for(c, na, kBlock), kBlock, 0, s>>>(na, C2.nbr.p, N.Eb.p, N.dsq.p, N.Ehat.p, N.feat.p);
    k_e2_hat<<<grid_for(c, (long)na * 27 * 36, kBlock), kBlock, 0, s>>>(na, C2.nbr.p, N.Eb.p, N.dsq.p, N.Ehat.p);
    OFEA_CHECK_LAUNCH();
    // centre the stiffness feature on its mean (host, na values)
    std::vector<float> f(na);
    OFEA_CUDA(cudaMemcpyAsync(f.data(), N.feat.p, sizeof(float) * na, cudaMemcpyDeviceToHost, s));
    OFEA_CUDA(cudaMemcpyAsync(c->herr.p, c->err_flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    OFEA_CUDA(cudaStreamSynchronize(s));
    if (c->herr.p[0]) fail(OFEA_ERR_CAPACITY, "learned level: cells smaller than the element couplings");
    double mean = 0;
    for (float v : f) mean += v;
    mean /= std::max(na, 1);
    for (float &v : f) v = (float)(v - mean);
    N.feat.upload(f.data(), na, s);
    C2.cvec.ensure(6L * na);
    N.sigma.ensure(4);
    C2.K_ok = true;
}

static void ensure_rows(ofea_ctx *c, long R) {
    Learned &N = c->learned;
    if (N.cap_rows >= R && N.X.p) return;
    N.X.ensure(R * kIn);
    N.Z0.ensure(R * kF);
    for (int l = 0; l <= kLayers; ++l) N.H[l].ensure(R * kF);
    for (int l = 0; l < kLayers; ++l) {
        N.A[l].ensure(R * kA);
        N.Zl[l].ensure(R * kF);
    }
    N.Y.ensure(R * kOut);
    N.Yz.ensure(R * kOut);
    N.dY.ensure(R * kOut);
    N.dH.ensure(R * kF);
    N.dZ.ensure(R * kF);
    N.dA.ensure(R * kA);
    N.cap_rows = R;
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

// Forward pass over R = B * na rows whose inputs are in N.X.
static void forward(ofea_ctx *c, long R, int na) {
    Learned &N = c->learned;
    const Learned::Layout L = Learned::layout();
    cudaStream_t s = c->stream;
    const float *w = N.w.p;
    const int G = grid_for(c, R * kF, kBlock);
    k_dense<<<dim3(tiles(kF, 64), tiles(R, 64)), 256, 0, s>>>(R, kF, kIn, N.X.p, w + L.W0, w + L.b0, N.Z0.p, N.H[0].p);
    for (int l = 0; l < kLayers; ++l) {
        k_gnn_aggregate<<<G, kBlock, 0, s>>>(R, na, c->coarse2.nbr.p, N.H[l].p, N.A[l].p);
        k_dense<<<dim3(tiles(kF, 64), tiles(R, 64)), 256, 0, s>>>(R, kF, kA, N.A[l].p, w + L.W[l], w + L.b[l],
                                                                 N.Zl[l].p, N.H[l + 1].p);
    }
    k_dense<<<dim3(1, tiles(R, 64)), 256, 0, s>>>(R, kOut, kF, N.H[kLayers].p, w + L.Wd, w + L.bd, N.Y.p, nullptr);
    OFEA_CHECK_LAUNCH();
}

// Loss gradient at N.Y, backward pass, parameter gradient in N.g.  Returns
// nothing; loss partials in N.lossp (G of them).
static void backward(ofea_ctx *c, long R, int na) {
    Learned &N = c->learned;
    const Learned::Layout L = Learned::layout();
    cudaStream_t s = c->stream;
    const float *w = N.w.p;
    float *g = N.g.p;
    const int G = std::min(kMaxGrid, grid_for(c, R, kBlock));
    N.lossp.ensure(kMaxGrid);
    N.nlossp = G;
    k_gnn_energy<<<G, kBlock, 0, s>>>(R, na, c->coarse2.nbr.p, N.Ehat.p, N.X.p, N.Y.p, N.dY.p, N.lossp.p);
    const long chunk = 2048;
    const int S = (int)((R + chunk - 1) / chunk);
    N.part.ensure((size_t)S * (kF * kA + kF));
    auto wgrad = [&](int O, int K, const float *dZ, const float *X, size_t offW, size_t offb) {
        const int nout = O * K + O;
        k_wgrad<<<dim3(tiles(nout, 256), S), 256, 0, s>>>(R, O, K, chunk, dZ, X, N.part.p);
        k_wgrad_sum<<<tiles(nout, 256), 256, 0, s>>>(S, O, K, N.part.p, g + offW, g + offb);
    };
    // decoder
    wgrad(kOut, kF, N.dY.p, N.H[kLayers].p, L.Wd, L.bd);
    k_dense_bwd_data<<<dim3(tiles(kF, 64), tiles(R, 64)), 256, 0, s>>>(R, kOut, kF, N.dY.p, w + L.Wd, N.dH.p);
    const int Gf = grid_for(c, R * kF, kBlock);
    k_relu_bwd<<<Gf, kBlock, 0, s>>>(R * kF, N.dH.p, N.Zl[kLayers - 1].p, N.dZ.p);
    for (int l = kLayers - 1; l >= 0; --l) {
        wgrad(kF, kA, N.dZ.p, N.A[l].p, L.W[l], L.b[l]);
        k_dense_bwd_data<<<dim3(tiles(kA, 64), tiles(R, 64)), 256, 0, s>>>(R, kF, kA, N.dZ.p, w + L.W[l], N.dA.p);
        const float *Zprev = l > 0 ? N.Zl[l - 1].p : N.Z0.p;
        k_gnn_aggregate_bwd<<<Gf, kBlock, 0, s>>>(R, na, c->coarse2.nbr.p, N.dA.p, Zprev, N.dZ.p);
    }
    wgrad(kF, kIn, N.dZ.p, N.X.p, L.W0, L.b0);
    OFEA_CHECK_LAUNCH();
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

// One restricted residual sample from a device FP64 vector r (n entries).
void learned_add_sample(ofea_ctx *c, const double *d_r) {
    Coarse &C2 = c->coarse2;
    Learned &N = c->learned;
    if (N.nsamples >= N.max_samples) return;
    cudaStream_t s = c->stream;
    const int na = C2.na;
    N.r32.ensure(c->n);
    k_f64_to_f32<<<grid_for(c, c->n, kBlock), kBlock, 0, s>>>(c->n, d_r, N.r32.p);
    restrict_level(c, C2, N.r32.p, C2.cvec.p);
    k_gnn_sigma<<<1, kBlock, 0, s>>>(na, C2.cvec.p, N.dsq.p, N.sigma.p);
    k_gnn_sample<<<grid_for(c, 6L * na, kBlock), kBlock, 0, s>>>(na, C2.cvec.p, N.dsq.p, N.sigma.p,
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

// Adam training on the collected samples.  Returns (first, last) epoch loss.
void learned_train(ofea_ctx *c, int steps, int batch, float lr, unsigned seed, double *loss0, double *loss1) {
    Learned &N = c->learned;
    if (N.nsamples < 1) fail(OFEA_ERR_STATE, "no training samples");
    upload_weights(c);
    const int na = c->coarse2.na;
    const int B = std::min(batch, N.nsamples);
    const long R = (long)B * na;
    ensure_rows(c, R);
    N.batch_src.ensure(R * kOut);
    std::mt19937 rng(seed);
    const size_t n = Learned::layout().total;
    cudaStream_t s = c->stream;
    double first = 0, last = 0;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int it = 0; it < steps; ++it) {
        // batch: B distinct samples
        std::vector<int> idx(N.nsamples);
        for (int i = 0; i < N.nsamples; ++i) idx[i] = i;
        for (int i = 0; i < B; ++i) std::swap(idx[i], idx[i + rng() % (N.nsamples - i)]);
        for (int b = 0; b < B; ++b)
            OFEA_CUDA(cudaMemcpyAsync(N.batch_src.p + (size_t)b * 6 * na, N.data.p + (size_t)idx[b] * 6 * na,
                                      sizeof(float) * 6 * na, cudaMemcpyDeviceToDevice, s));
        k_gnn_input<<<grid_for(c, R, kBlock), kBlock, 0, s>>>(R, na, N.batch_src.p, N.feat.p, N.X.p);
        forward(c, R, na);
        backward(c, R, na);
        ++N.trained_steps;
        const float c1 = 1.f - std::pow(b1, (float)N.trained_steps);
        const float c2 = 1.f - std::pow(b2, (float)N.trained_steps);
        k_adam<<<grid_for(c, (long)n, kBlock), kBlock, 0, s>>>((long)n, N.w.p, N.g.p, N.m.p, N.v.p, lr, b1, b2,
                                                              eps, c1, c2);
        OFEA_CHECK_LAUNCH();
        if (it == 0) first = read_loss(c);
        if (it == steps - 1) last = read_loss(c);
    }
    // keep the host copy in step with the device weights
    N.host_w.resize(n);
    OFEA_CUDA(cudaMemcpyAsync(N.host_w.data(), N.w.p, sizeof(float) * n, cudaMemcpyDeviceToHost, s));
    OFEA_CUDA(cudaStreamSynchronize(s));
    if (loss0) *loss0 = first;
    if (loss1) *loss1 = last;
}

// Loss and full parameter gradient for given normalised inputs (B x na x 6, host).
void learned_gradient(ofea_ctx *c, const float *h_x, int B, double *loss, float *h_grad) {
    Learned &N = c->learned;
    upload_weights(c);
    const int na = c->coarse2.na;
    const long R = (long)B * na;
    ensure_rows(c, R);
    N.batch_src.upload(h_x, R * kOut, c->stream);
    k_gnn_input<<<grid_for(c, R, kBlock), kBlock, 0, c->stream>>>(R, na, N.batch_src.p, N.feat.p, N.X.p);
    forward(c, R, na);
    backward(c, R, na);
    *loss = read_loss(c);
    const size_t n = Learned::layout().total;
    OFEA_CUDA(cudaMemcpyAsync(h_grad, N.g.p, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
    OFEA_CUDA(cudaStreamSynchronize(c->stream));
}

// Inference inside the V-cycle: x += Z2 g(Z2^T t).
void learned_apply(ofea_ctx *c, const float *t, float *x) {
    Coarse &C2 = c->coarse2;
    Learned &N = c->learned;
    cudaStream_t s = c->stream;
    const int na = C2.na;
    restrict_level(c, C2, t, C2.cvec.p);
    k_gnn_sigma<<<1, kBlock, 0, s>>>(na, C2.cvec.p, N.dsq.p, N.sigma.p);
    k_gnn_input_c<<<grid_for(c, na, kBlock), kBlock, 0, s>>>(na, C2.cvec.p, N.dsq.p, N.feat.p, N.sigma.p, N.X.p);
    forward(c, na, na);
    k_gnn_output<<<grid_for(c, 6L * na, kBlock), kBlock, 0, s>>>(na, N.Y.p, N.dsq.p, N.sigma.p, C2.cvec.p);
    prolong_level(c, C2, C2.cvec.p, x);
    OFEA_CHECK_LAUNCH();
}

void learned_prepare_inference(ofea_ctx *c) {
    upload_weights(c);
    ensure_rows(c, c->coarse2.na);
}

}  // namespace ofea
