// Element integration and assembly on the device: the B200 replacement of
// assamble_stiffness::fill_CSR_sparse_mat (src/assemble.cpp:95-151) and
// assamble_nl_stiffness::fill_CSR_sparse_mat (src/nl_assemble.cpp:94-166).
//
// Stage 1 (integration, FP64): one warp-group (128 threads) integrates a batch
// of elements: node coordinates are staged in shared memory, each thread
// computes the Jacobian of one Gauss point redundantly and the physical shape
// function gradients of one node, then one 3x3 nodal block of Ke per thread.
// The nodal-block form of B^T D B used here (isotropic D, engineering shear,
// strain order [xx, yy, zz, xy, yz, zx], src/Elements/C3D8.cpp:21-35) is
//   K_ab[i][j] = sum_q w_q det_q (lam g_a[i] g_b[j] + mu g_a[j] g_b[i]
//                                 + delta_ij mu g_a.g_b)
// with g_a = J^-1 dN_a at Gauss point q; for C3D8 the 2x2x2 rule with weight
// 1 (src/Elements/C3D8_Gauss.cpp:80-107), for C3D4 one point, weight 1/6 and
// the signed determinant (src/Elements/C3D4_hammer.cpp:61-72).  Element
// matrices go to a scratch buffer with coalesced stores.
//
// Stage 2 (assembly): one warp per free node owns its block row of K, walks
// the node's incident elements in ascending order and adds their block rows
// through the precomputed slot map in shared memory, then writes the row once:
// no atomics, coalesced, bitwise reproducible.
#include <algorithm>
#include <cmath>

#include <mutex>

#include "ofea_internal.cuh"
#include "sell.cuh"

namespace ofea {

// dN/d(r,s,t) of the 8-node brick at the 8 Gauss points, [q][dim][node]
// (node order src/Elements/C3D8_Gauss.cpp:27-52, points :84-92).
__constant__ double c_hex_dN[8 * 3 * 8];

// Per-device constant table (192 doubles), uploaded once per device: the
// first integration or stress call on a device writes it, later calls only
// check a flag.
static void upload_hex_table() {
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static bool done[kMaxDevices] = {};
    int dev = 0;
    OFEA_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) fail(OFEA_ERR_INVALID_ARG, "device index too large");
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev]) return;
    const int sr[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
    const int ss[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
    const int st[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
    double g = 1.0 / std::sqrt(3.0), t[192];
    for (int q = 0; q < 8; ++q) {
        double r = sr[q] * g, s = ss[q] * g, u = st[q] * g;
        for (int a = 0; a < 8; ++a) {
            t[(q * 3 + 0) * 8 + a] = 0.125 * sr[a] * (1.0 + ss[a] * s) * (1.0 + st[a] * u);
            t[(q * 3 + 1) * 8 + a] = 0.125 * ss[a] * (1.0 + sr[a] * r) * (1.0 + st[a] * u);
            t[(q * 3 + 2) * 8 + a] = 0.125 * st[a] * (1.0 + sr[a] * r) * (1.0 + ss[a] * s);
        }
    }
    OFEA_CUDA(cudaMemcpyToSymbol(c_hex_dN, t, sizeof(t)));
    done[dev] = true;
}

struct Lame {
    double lam, mu, fac;
};
// Same expressions as build_cons_mat (src/Elements/C3D8.cpp:23-27).
__device__ __forceinline__ Lame lame(double E, double nu) {
    double fac = (E * (1.0 - nu)) / ((1.0 + nu) * (1.0 - 2.0 * nu));
    return {fac * nu / (1.0 - nu), fac * (1.0 - 2.0 * nu) / (2.0 * (1.0 - nu)), fac};
}

// Determinant in the reference's expression (C3D8_Gauss.cpp:58-63) and the
// cofactor inverse.
__device__ __forceinline__ double det_sarrus(const double *J) {
    return J[0] * J[4] * J[8] + J[1] * J[5] * J[6] + J[2] * J[3] * J[7] - J[2] * J[4] * J[6] -
           J[5] * J[7] * J[0] - J[8] * J[1] * J[3];
}
__device__ __forceinline__ void inv3(const double *J, double *Ji) {
    double c00 = J[4] * J[8] - J[5] * J[7];
    double c01 = J[5] * J[6] - J[3] * J[8];
    double c02 = J[3] * J[7] - J[4] * J[6];
    double id = 1.0 / (J[0] * c00 + J[1] * c01 + J[2] * c02);
    Ji[0] = c00 * id;
    Ji[1] = (J[2] * J[7] - J[1] * J[8]) * id;
    Ji[2] = (J[1] * J[5] - J[2] * J[4]) * id;
    Ji[3] = c01 * id;
    Ji[4] = (J[0] * J[8] - J[2] * J[6]) * id;
    Ji[5] = (J[2] * J[3] - J[0] * J[5]) * id;
    Ji[6] = c02 * id;
    Ji[7] = (J[1] * J[6] - J[0] * J[7]) * id;
    Ji[8] = (J[0] * J[4] - J[1] * J[3]) * id;
}

// Jacobian of the 8-node brick at Gauss point q from its node coordinates
// X[8][3], the physical gradients g_a[d] = sum_i Jinv[d][i] dN_i(a), stored
// to out[a * sa + d * sd] as they are formed, and the point's weight det J
// (Gauss weight 1), returned.  Every linear C3D8 path evaluates the point
// through this function, so they give the same bits.
__device__ __forceinline__ double hex_point(const double *X, int q, double *out, int sa, int sd) {
    const double *dN = c_hex_dN + q * 24;
    double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 2
    for (int b = 0; b < 8; ++b) {  // J_ij = sum_b dN_i(b) X_bj, b ascending
        const double x0 = X[3 * b], x1 = X[3 * b + 1], x2 = X[3 * b + 2];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double dn = dN[i * 8 + b];
            J[3 * i] = fma(dn, x0, J[3 * i]);
            J[3 * i + 1] = fma(dn, x1, J[3 * i + 1]);
            J[3 * i + 2] = fma(dn, x2, J[3 * i + 2]);
        }
    }
    double Ji[9];
    inv3(J, Ji);
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int d = 0; d < 3; ++d)
            out[a * sa + d * sd] = fma(Ji[3 * d + 2], dN[16 + a], fma(Ji[3 * d + 1], dN[8 + a], Ji[3 * d] * dN[a]));
    return det_sarrus(J);
}

// One Gauss point of T = sum_q w g_u g_v^T (w on the u side).
__device__ __forceinline__ void lin_T_step(double *T, double w, const double *gu, const double *gv) {
    const double a0 = w * gu[0], a1 = w * gu[1], a2 = w * gu[2];
    T[0] = fma(a0, gv[0], T[0]);
    T[1] = fma(a0, gv[1], T[1]);
    T[2] = fma(a0, gv[2], T[2]);
    T[3] = fma(a1, gv[0], T[3]);
    T[4] = fma(a1, gv[1], T[4]);
    T[5] = fma(a1, gv[2], T[5]);
    T[6] = fma(a2, gv[0], T[6]);
    T[7] = fma(a2, gv[1], T[7]);
    T[8] = fma(a2, gv[2], T[8]);
}

// Linear elastic block from T: K_uv = lam T + mu T^T + mu tr(T) I, operation
// order fixed (explicit FMAs) so every assembly path gives the same bits.
__device__ __forceinline__ void lin_block(const double *T, double lam, double mu, double *k) {
    const double md = mu * (T[0] + T[4] + T[8]);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            k[3 * i + j] = fma(lam, T[3 * i + j], i == j ? fma(mu, T[3 * j + i], md) : mu * T[3 * j + i]);
}

// Block-Jacobi inverse of one diagonal block; false (and the identity) for a
// block without a positive determinant.
__device__ __forceinline__ bool jacobi_inverse(const double *A, double *Ai) {
    const double det = A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
                       A[2] * (A[3] * A[7] - A[4] * A[6]);
    if (!(det > 0.0) || !isfinite(det)) {
#pragma unroll
        for (int i = 0; i < 9; ++i) Ai[i] = (i % 4 == 0) ? 1.0 : 0.0;
        return false;
    }
    inv3(A, Ai);
    return true;
}

// Linear nodal block accumulation: k += w (lam ga gb^T + mu gb ga^T + mu (ga.gb) I).
__device__ __forceinline__ void add_block_lin(double *k, const double *ga, const double *gb,
                                              double wl, double wm) {
    double d = ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double v = wl * ga[i] * gb[j] + wm * ga[j] * gb[i];
            if (i == j) v += wm * d;
            k[3 * i + j] += v;
        }
}

// Total-Lagrangian quantities of one integration point from F:
// S = D E_GL (Voigt [xx,yy,zz,xy,yz,zx], engineering shear as the reference's
// Gl_vec, src/Elements/C3D8_Gauss.cpp:164-172) and C = F F^T.
__device__ __forceinline__ void tl_point(const double *F, const Lame &L, double *S, double *C) {
    double Eg[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double s = F[i] * F[j] + F[3 + i] * F[3 + j] + F[6 + i] * F[6 + j];  // (F^T F)_ij
            Eg[3 * i + j] = 0.5 * (s - (i == j ? 1.0 : 0.0));
        }
    double e0 = Eg[0], e1 = Eg[4], e2 = Eg[8];
    double fa = L.lam;
    S[0] = L.fac * e0 + fa * e1 + fa * e2;
    S[1] = fa * e0 + L.fac * e1 + fa * e2;
    S[2] = fa * e0 + fa * e1 + L.fac * e2;
    S[3] = L.mu * (2.0 * Eg[1]);
    S[4] = L.mu * (2.0 * Eg[5]);
    S[5] = L.mu * (2.0 * Eg[2]);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            C[3 * i + j] = F[3 * i] * F[3 * j] + F[3 * i + 1] * F[3 * j + 1] + F[3 * i + 2] * F[3 * j + 2];
}

// Smat g with Smat = [[S0,S3,S5],[S3,S1,S4],[S5,S4,S2]].
__device__ __forceinline__ void smat_vec(const double *S, const double *g, double *o) {
    o[0] = S[0] * g[0] + S[3] * g[1] + S[5] * g[2];
    o[1] = S[3] * g[0] + S[1] * g[1] + S[4] * g[2];
    o[2] = S[5] * g[0] + S[4] * g[1] + S[2] * g[2];
}

// Tangent nodal block: k += w (lam pa pb^T + mu pb pa^T + mu (ga.gb) C + (ga.S gb) I),
// p = F g, which equals (B_L^T D B_L + B_NL^T SIG B_NL)_ab of the reference
// (src/Elements/C3D8_Gauss.cpp:174-264).
__device__ __forceinline__ void add_block_nl(double *k, const double *ga, const double *gb,
                                             const double *pa, const double *pb, const double *C,
                                             const double *S, double w, const Lame &L) {
    double d = ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2];
    double sg[3];
    smat_vec(S, gb, sg);
    double geo = ga[0] * sg[0] + ga[1] * sg[1] + ga[2] * sg[2];
    double wl = w * L.lam, wm = w * L.mu, wc = w * L.mu * d;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double v = wl * pa[i] * pb[j] + wm * pb[i] * pa[j] + wc * C[3 * i + j];
            if (i == j) v += w * geo;
            k[3 * i + j] += v;
        }
}

// ------------------------------------------------------------------ C3D8 --

constexpr int kHexPerCta = 2;  // 64 threads per element: (q,a) then (a,b)

template <bool NL>
__global__ void __launch_bounds__(128) k_hex_integrate(
    int ne8, const int *__restrict__ topo8, const double *__restrict__ xyz,
    const double *__restrict__ E8, double nu, const int *__restrict__ free_map,
    const double *__restrict__ u, double *__restrict__ Ke, double *__restrict__ Fe) {
    __shared__ double sX[kHexPerCta][24];
    __shared__ double sU[kHexPerCta][24];       // [a][c]
    __shared__ double sG[kHexPerCta][8 * 3 * 8];  // [q][d][a]
    __shared__ double sP[kHexPerCta][NL ? 8 * 3 * 8 : 1];
    __shared__ double sW[kHexPerCta][8];
    __shared__ double sS[kHexPerCta][NL ? 8 * 6 : 1];
    __shared__ double sC[kHexPerCta][NL ? 8 * 9 : 1];
    __shared__ double sF[kHexPerCta][NL ? 8 * 9 : 1];
    __shared__ double sK[kHexPerCta][576];
    const int le = threadIdx.x >> 6, t = threadIdx.x & 63;
    for (long base = (long)blockIdx.x * kHexPerCta; base < ne8; base += (long)gridDim.x * kHexPerCta) {
        const long e = base + le;
        const bool act = e < ne8;
        if (act && t < 24) {
            int a = t / 3, cc = t - 3 * a;
            int node = topo8[8 * e + a];
            sX[le][t] = xyz[3L * node + cc];
            if (NL) {
                int f = free_map[node];
                sU[le][t] = f >= 0 ? u[3L * f + cc] : 0.0;
            }
        }
        __syncthreads();
        Lame L{0, 0, 0};
        if (act) L = lame(E8[e], nu);
        if (act) {
            // thread (q, a): Jacobian at q (redundant over a), gradient of node a
            const int q = t >> 3, a = t & 7;
            const double *dN = c_hex_dN + q * 24;
            double J[9];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    double s = 0;
#pragma unroll
                    for (int b = 0; b < 8; ++b) s += dN[i * 8 + b] * sX[le][3 * b + j];
                    J[3 * i + j] = s;
                }
            double Ji[9];
            inv3(J, Ji);
            double g[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                g[d] = Ji[3 * d] * dN[a] + Ji[3 * d + 1] * dN[8 + a] + Ji[3 * d + 2] * dN[16 + a];
                sG[le][(q * 3 + d) * 8 + a] = g[d];
            }
            if (a == 0) sW[le][q] = det_sarrus(J);  // Gauss weight 1
            if (NL) {
                // F = I + sum_b u_b (x) g_b needs every node's gradient: recompute
                // them from Ji here (8 x 9 FMA) rather than wait for sG.
                double F[9];
#pragma unroll
                for (int i = 0; i < 9; ++i) F[i] = (i % 4 == 0) ? 1.0 : 0.0;
#pragma unroll
                for (int b = 0; b < 8; ++b) {
                    double gb[3];
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        gb[d] = Ji[3 * d] * dN[b] + Ji[3 * d + 1] * dN[8 + b] + Ji[3 * d + 2] * dN[16 + b];
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int j = 0; j < 3; ++j) F[3 * i + j] += sU[le][3 * b + i] * gb[j];
                }
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    sP[le][(q * 3 + i) * 8 + a] = F[3 * i] * g[0] + F[3 * i + 1] * g[1] + F[3 * i + 2] * g[2];
                if (a == 0) {
                    double S[6], C[9];
                    tl_point(F, L, S, C);
#pragma unroll
                    for (int i = 0; i < 6; ++i) sS[le][6 * q + i] = S[i];
#pragma unroll
                    for (int i = 0; i < 9; ++i) {
                        sC[le][9 * q + i] = C[i];
                        sF[le][9 * q + i] = F[i];
                    }
                }
            }
        }
        __syncthreads();
        if (act) {
            // thread (a, b): block K_ab summed over the Gauss points
            const int a = t >> 3, b = t & 7;
            double k[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            double fa[3] = {0, 0, 0};
#pragma unroll 2
            for (int q = 0; q < 8; ++q) {
                double ga[3], gb[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    ga[d] = sG[le][(q * 3 + d) * 8 + a];
                    gb[d] = sG[le][(q * 3 + d) * 8 + b];
                }
                double w = sW[le][q];
                if (!NL) {
                    add_block_lin(k, ga, gb, w * L.lam, w * L.mu);
                } else {
                    double pa[3], pb[3];
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        pa[d] = sP[le][(q * 3 + d) * 8 + a];
                        pb[d] = sP[le][(q * 3 + d) * 8 + b];
                    }
                    add_block_nl(k, ga, gb, pa, pb, &sC[le][9 * q], &sS[le][6 * q], w, L);
                    if (b == 0) {
                        // f_a += w F (Smat g_a)  (= B_L^T S, C3D8_Gauss.cpp:257)
                        double sg[3];
                        smat_vec(&sS[le][6 * q], ga, sg);
                        const double *F = &sF[le][9 * q];
#pragma unroll
                        for (int i = 0; i < 3; ++i)
                            fa[i] += w * (F[3 * i] * sg[0] + F[3 * i + 1] * sg[1] + F[3 * i + 2] * sg[2]);
                    }
                }
            }
#pragma unroll
            for (int i = 0; i < 9; ++i) sK[le][(a * 8 + b) * 9 + i] = k[i];
            if (NL && b == 0)
#pragma unroll
                for (int i = 0; i < 3; ++i) Fe[24 * e + 3 * a + i] = fa[i];
        }
        __syncthreads();
        // coalesced store of the batch's element matrices
        for (int v = threadIdx.x; v < kHexPerCta * 576; v += blockDim.x) {
            int l2 = v / 576;
            long e2 = base + l2;
            if (e2 < ne8) Ke[576 * e2 + (v - 576 * l2)] = sK[l2][v - 576 * l2];
        }
        __syncthreads();
    }
}

// Linear C3D8 element blocks, kLinHex elements per CTA of 128 threads.
// Phase 1, thread (element, q): J at Gauss point q, det J (the weight) and
// the gradients of all 8 shape functions, once per point.  Phase 2, thread
// per upper block (a <= b) of an element: T = sum_q w g_a g_b^T and
// d = sum_q w g_a . g_b, then K_ab = lam T + mu T^T + mu d I and
// K_ba = K_ab^T (the same sums, so Ke is exactly symmetric): the nodal-block
// form of B^T D B with 36 of the 64 blocks computed.
constexpr int kLinHex = 16;

__global__ void __launch_bounds__(128) k_hex_integrate_lin(int ne8, const int *__restrict__ topo8,
                                                           const double *__restrict__ xyz,
                                                           const double *__restrict__ E8, double nu,
                                                           double *__restrict__ Ke) {
    __shared__ double sX[kLinHex][25];  // odd stride: the 16 elements of a warp hit distinct banks
    __shared__ double sG[kLinHex][8][8][4];  // [element][q][a][d], d padded to 4
    __shared__ double sW[kLinHex][8];
    const int tid = threadIdx.x;
    for (long base = (long)blockIdx.x * kLinHex; base < ne8; base += (long)gridDim.x * kLinHex) {
        const int nel = (int)min((long)kLinHex, ne8 - base);
        for (int v = tid; v < nel * 24; v += 128) {
            const int le = v / 24, t = v % 24, a = t / 3, cc = t - 3 * a;
            sX[le][t] = xyz[3L * topo8[8 * (base + le) + a] + cc];
        }
        __syncthreads();
        {
            const int q = tid >> 4, le = tid & 15;  // a warp shares two Gauss points (constant-cache broadcasts)
            if (le < nel) {
                sW[le][q] = hex_point(sX[le], q, &sG[le][q][0][0], 4, 1);
            }
        }
        __syncthreads();
        for (int v = tid; v < nel * 36; v += 128) {
            const int le = v / 36;
            int pr = v % 36, a = 0;  // pr -> (a, b), a <= b, row by row
            while (pr >= 8 - a) {
                pr -= 8 - a;
                ++a;
            }
            const int b = a + pr;
            double T[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
            for (int q = 0; q < 8; ++q) lin_T_step(T, sW[le][q], sG[le][q][a], sG[le][q][b]);
            const Lame L = lame(E8[base + le], nu);
            double kab[9];
            lin_block(T, L.lam, L.mu, kab);
            double *ke = Ke + 576L * (base + le);
#pragma unroll
            for (int i = 0; i < 9; ++i) ke[(a * 8 + b) * 9 + i] = kab[i];
            if (b != a)
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) ke[(b * 8 + a) * 9 + 3 * i + j] = kab[3 * j + i];
        }
        __syncthreads();
    }
}

// ------------------------------------------------- fused linear assembly --
// Linear C3D8 meshes: integration and assembly in one pass, no element
// matrices in HBM.  One CTA per BSELL slice (32 block rows, sell.cuh) at a
// time, one CTA per SM:
//   * the slice's incident elements (sorted and de-duplicated once per
//     pattern: se_ptr/se_list, and inc_loc = an incidence's position in that
//     list) have their node coordinates and Lame constants staged in shared
//     memory, and each row's incidences (position, local node, the slots of
//     the element's 8 nodes) form a small table there;
//   * chunk by chunk (ascending element order) thread (element, q) writes the
//     8 shape-function gradients and det J of its Gauss point to shared memory;
//   * thread (warp k, lane t) owns slot k of row t: it walks the row's
//     incidences in ascending element order and adds the element block that
//     lands in slot k to 9 registers.  The block is formed from the gradients
//     exactly as k_hex_integrate_lin forms it (upper block, transposed for
//     b < a) and the sums run in the gather's order, so K carries the same
//     bits as the two-pass assembly;
//   * the slice is written once: FP64 planes (coalesced), the grouped BF16
//     copy through shared memory, and the diagonal block's inverse.
// The block sums read 56 gradient doubles from shared memory per block: the
// kernel is bound by shared-memory bandwidth, so slot loads that differ
// between warps (1 to 8 blocks per row) do not idle the SM.  Meshes it does
// not cover (tetrahedra, nodes in more than 8 elements, rows wider than 27
// blocks, slices touching more than kFuMaxElem elements) take the two-pass
// path.
constexpr int kFuMaxW = 27;               // widest slice: 27 blocks
constexpr int kFuNW = kFuMaxW;            // warps per CTA: warp k owns slot k
constexpr int kFuThreads = 32 * kFuNW;
constexpr int kFuRowInc = 8;              // incident elements per node
constexpr int kFuMaxElem = 192;           // distinct elements per slice
constexpr int kFuChunk = 96;              // elements whose gradients are in shared memory at once
constexpr int kFuGS = 8 * 3 * 8 + 8 + 1;  // per element: g[a][d][q], det J [q]; odd stride
constexpr int kFuXS = 25;                 // coordinate doubles per element (odd stride)
constexpr size_t kFuSmem = sizeof(double) * (kFuMaxElem * kFuXS + kFuMaxElem * 2 + kFuChunk * kFuGS);

// Block K_ab of an element from its gradients in shared memory (layout of
// k_hex_assemble_fused): the upper block (a <= b) as k_hex_integrate_lin
// computes it, transposed for b < a.
__device__ __forceinline__ void fused_block(const double *G, int a, int b, double lam, double mu, double *kab) {
    const bool sw = a > b;
    const int u = sw ? b : a, v = sw ? a : b;
    double T[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 1
    for (int q = 0; q < 8; ++q) {
        const double gu[3] = {G[(3 * u) * 8 + q], G[(3 * u + 1) * 8 + q], G[(3 * u + 2) * 8 + q]};
        const double gv[3] = {G[(3 * v) * 8 + q], G[(3 * v + 1) * 8 + q], G[(3 * v + 2) * 8 + q]};
        lin_T_step(T, G[192 + q], gu, gv);
    }
    double k[9];
    lin_block(T, lam, mu, k);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) kab[3 * i + j] = sw ? k[3 * j + i] : k[3 * i + j];
}

__global__ void __launch_bounds__(kFuThreads, 1) k_hex_assemble_fused(
    int nfree, const int *__restrict__ node_of_free, const int *__restrict__ inc_ptr,
    const int *__restrict__ inc, const uint16_t *__restrict__ slot, const uint16_t *__restrict__ inc_loc,
    const int *__restrict__ se_ptr, const int *__restrict__ se_list, const int *__restrict__ topo8,
    const double *__restrict__ xyz, const double *__restrict__ E8, double nu, const int *__restrict__ diag_pos,
    const int *__restrict__ sl_ptr, const int *__restrict__ sl_g, double *__restrict__ sv64,
    __nv_bfloat16 *__restrict__ svg, double *__restrict__ Dinv, float *__restrict__ Dinv32, int *__restrict__ err) {
    extern __shared__ double fsm[];
    double *sX = fsm;                      // [kFuMaxElem][kFuXS] node coordinates
    double *sL = sX + kFuMaxElem * kFuXS;  // [kFuMaxElem][2]  lam, mu
    double *sG = sL + kFuMaxElem * 2;      // [kFuChunk][kFuGS] gradients, then the BF16 staging
    // row t's incidences: position in the slice's list, local node, and the
    // slots of the element's 8 nodes as bytes (0xFF: fixed node)
    __shared__ unsigned long long s_sl[kSlice][kFuRowInc];
    __shared__ uint16_t s_loc[kSlice][kFuRowInc];
    __shared__ unsigned char s_a[kSlice][kFuRowInc];
    __shared__ int s_ninc[kSlice];
    const int tid = threadIdx.x, lane = tid & 31, k = tid >> 5;
    const int nslice = (nfree + kSlice - 1) / kSlice;
    for (int s = blockIdx.x; s < nslice; s += gridDim.x) {
        const int e0 = se_ptr[s], nes = se_ptr[s + 1] - e0;
        const long S = sl_ptr[s];
        const int W = sl_ptr[s + 1] - (int)S;
        __syncthreads();  // the previous slice is written out
        for (int v = tid; v < nes * 24; v += kFuThreads) {
            const int le = v / 24, t = v - 24 * le, a = t / 3, d = t - 3 * a;
            sX[le * kFuXS + t] = xyz[3L * topo8[8L * se_list[e0 + le] + a] + d];
        }
        for (int le = tid; le < nes; le += kFuThreads) {
            const Lame L = lame(E8[se_list[e0 + le]], nu);
            sL[2 * le] = L.lam;
            sL[2 * le + 1] = L.mu;
        }
        if (tid < kSlice * kFuRowInc) {
            const int t = tid / kFuRowInc, i = tid % kFuRowInc, r = s * kSlice + t;
            int n = 0;
            if (r < nfree) {
                const int node = node_of_free[r], p0 = inc_ptr[node];
                n = inc_ptr[node + 1] - p0;
                if (i < n) {
                    const uint4 raw = __ldg(reinterpret_cast<const uint4 *>(slot) + (p0 + i));
                    const unsigned w4[4] = {raw.x, raw.y, raw.z, raw.w};
                    unsigned long long by = 0;
#pragma unroll
                    for (int b = 0; b < 8; ++b) {
                        const unsigned kk = (w4[b >> 1] >> (16 * (b & 1))) & 0xFFFFu;
                        by |= (unsigned long long)(kk < (unsigned)kFuMaxW ? kk : 0xFFu) << (8 * b);
                    }
                    s_sl[t][i] = by;
                    s_loc[t][i] = inc_loc[p0 + i];
                    s_a[t][i] = (unsigned char)(inc[p0 + i] & 7);
                }
            }
            if (i == 0) s_ninc[t] = n;
        }
        const int r = s * kSlice + lane;
        int cur = 0;  // next incidence of row `lane`
        double acc[9];
#pragma unroll
        for (int e = 0; e < 9; ++e) acc[e] = 0.0;
        for (int c0 = 0; c0 < nes; c0 += kFuChunk) {
            const int nel = min(kFuChunk, nes - c0);
            __syncthreads();  // staging done; the previous chunk's gradients consumed
            if (tid < kFuChunk * 8) {  // q-major: a warp shares its Gauss point (constant-cache broadcasts)
                const int q = tid / kFuChunk, le = tid - q * kFuChunk;
                if (le < nel) {
                    double *G = sG + le * kFuGS;
                    G[192 + q] = hex_point(sX + kFuXS * (c0 + le), q, G + q, 24, 8);
                }
            }
            __syncthreads();
            if (k < W) {
                const int ninc = s_ninc[lane], chunk_hi = c0 + nel;
                const unsigned kk4 = (unsigned)k * 0x01010101u;
                for (; cur < ninc; ++cur) {
                    const int loc = s_loc[lane][cur];
                    if (loc >= chunk_hi) break;
                    if (loc < c0) continue;  // ascending by construction; never read outside the chunk
                    const unsigned long long by = s_sl[lane][cur];
                    const unsigned m0 = __vcmpeq4((unsigned)by, kk4), m1 = __vcmpeq4((unsigned)(by >> 32), kk4);
                    if ((m0 | m1) == 0u) continue;
                    const int b = m0 ? (__ffs(m0) - 1) >> 3 : 4 + ((__ffs(m1) - 1) >> 3);
                    double kab[9];
                    fused_block(sG + (loc - c0) * kFuGS, s_a[lane][cur], b, sL[2 * loc], sL[2 * loc + 1], kab);
#pragma unroll
                    for (int e = 0; e < 9; ++e) acc[e] += kab[e];
                }
            }
        }
        __syncthreads();  // every chunk consumed: sG becomes the BF16 staging area
        __nv_bfloat16 *sB = reinterpret_cast<__nv_bfloat16 *>(sG);  // [W][9][32]
        const int dp = r < nfree ? diag_pos[r] : -1;
        if (k < W) {
#pragma unroll
            for (int e = 0; e < 9; ++e) {
                sv64[((S + k) * 9 + e) * kSlice + lane] = acc[e];
                sB[(k * 9 + e) * kSlice + lane] = __double2bfloat16(acc[e]);
            }
        }
        // block-Jacobi: the owner of the diagonal slot inverts it; a free node
        // outside every element (empty row) gets the identity and the flag
        if (k == dp || (r < nfree && dp < 0 && k == 0)) {
            if (k != dp)
#pragma unroll
                for (int e = 0; e < 9; ++e) acc[e] = 0.0;
            double Ai[9];
            if (!jacobi_inverse(acc, Ai)) atomicExch(err, 1);
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                Dinv[9L * r + i] = Ai[i];
                Dinv32[9L * r + i] = (float)Ai[i];
            }
        }
        __syncthreads();
        const long G = sl_g[s];
        const int ng = (W + 3) / 4;
        uint2 *svg2 = reinterpret_cast<uint2 *>(svg);
        for (int v = tid; v < ng * 9 * kSlice; v += kFuThreads) {
            const int g = v / (9 * kSlice), rem = v - g * 9 * kSlice, e = rem / kSlice, t = rem - e * kSlice;
            unsigned h[2] = {0u, 0u};
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int kk = 4 * g + u;
                if (kk < W) h[u >> 1] |= (unsigned)__bfloat16_as_ushort(sB[(kk * 9 + e) * kSlice + t]) << (16 * (u & 1));
            }
            svg2[((G + g) * 9 + e) * kSlice + t] = make_uint2(h[0], h[1]);
        }
    }
}

// Per pattern: the sorted distinct elements of every slice's rows (pass 0
// counts them, pass 1 writes them and every incidence's position in its
// slice's list).  One CTA per slice, a bitonic sort of the slice's <= 256
// incidences.  stats[0]: a node in more than kFuRowInc elements, stats[1]:
// the widest slice, stats[2]: the most elements of a slice.
constexpr int kSeThreads = kSlice * kFuRowInc;  // one thread per incidence of a slice

template <bool FILL>
__global__ void __launch_bounds__(kSeThreads) k_slice_elements(
    int nfree, const int *__restrict__ node_of_free, const int *__restrict__ inc_ptr, const int *__restrict__ inc,
    const int *__restrict__ sl_ptr, const int *__restrict__ se_ptr, int *__restrict__ se_cnt,
    int *__restrict__ se_list, uint16_t *__restrict__ inc_loc, int *__restrict__ stats) {
    __shared__ int key[kSeThreads];
    __shared__ int rowbeg[kSlice + 1];
    __shared__ int rownode[kSlice];
    __shared__ int wsum[kSeThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nslice = (nfree + kSlice - 1) / kSlice;
    for (int s = blockIdx.x; s < nslice; s += gridDim.x) {
        if (warp == 0) {
            const int r = s * kSlice + lane;
            const int node = r < nfree ? node_of_free[r] : -1;
            int cnt = node >= 0 ? inc_ptr[node + 1] - inc_ptr[node] : 0;
            if (cnt > kFuRowInc) {
                atomicExch(stats, 1);
                cnt = kFuRowInc;
            }
            int v = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, v, o);
                if (lane >= o) v += t;
            }
            rownode[lane] = node;
            rowbeg[lane + 1] = v;
            if (lane == 0) rowbeg[0] = 0;
            if (!FILL && lane == 0) atomicMax(stats + 1, sl_ptr[s + 1] - sl_ptr[s]);
        }
        __syncthreads();
        const int total = rowbeg[kSlice];
        int p = -1;
        if (tid < total) {
            int row = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1)
                if (row + step < kSlice && rowbeg[row + step] <= tid) row += step;
            p = inc_ptr[rownode[row]] + (tid - rowbeg[row]);
            key[tid] = inc[p] >> 3;
        } else {
            key[tid] = 0x7FFFFFFF;
        }
        __syncthreads();
        for (int k = 2; k <= kSeThreads; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1) {
                const int ixj = tid ^ j;
                if (ixj > tid) {
                    const int x = key[tid], y = key[ixj];
                    if ((x > y) == ((tid & k) == 0)) {
                        key[tid] = y;
                        key[ixj] = x;
                    }
                }
                __syncthreads();
            }
        const int kv = key[tid];
        const int flag = tid < total && (tid == 0 || key[tid - 1] != kv);
        // block scan of the flags: rank of each distinct element
        const unsigned bal = __ballot_sync(0xffffffffu, flag);
        if (lane == 0) wsum[warp] = __popc(bal);
        __syncthreads();
        int before = 0, count = 0;
        for (int w = 0; w < kSeThreads / 32; ++w) {
            if (w < warp) before += wsum[w];
            count += wsum[w];
        }
        const int rank = before + __popc(bal & ((1u << lane) - 1u));
        if (!FILL) {
            if (tid == 0) {
                se_cnt[s] = count;
                atomicMax(stats + 2, count);
            }
        } else {
            __syncthreads();  // every thread has read key[] for its flag
            if (flag) {
                se_list[se_ptr[s] + rank] = kv;
                key[rank] = kv;  // compacted in place: rank <= tid, and every key is read
            }
            __syncthreads();
            if (p >= 0) {
                const int g = inc[p] >> 3;
                int lo = 0, hi = count - 1;  // g is in key[0..count)
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (key[mid] < g) lo = mid + 1;
                    else hi = mid;
                }
                inc_loc[p] = (uint16_t)lo;
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ C3D4 --// ------------------------------------------------------------------ C3D4 --

constexpr int kTetPerCta = 8;  // 16 threads per element: (a,b)

template <bool NL>
__global__ void __launch_bounds__(128) k_tet_integrate(
    int ne4, const int *__restrict__ topo4, const double *__restrict__ xyz,
    const double *__restrict__ E4, double nu, const int *__restrict__ free_map,
    const double *__restrict__ u, double *__restrict__ Ke, double *__restrict__ Fe) {
    __shared__ double sX[kTetPerCta][12];
    __shared__ double sU[kTetPerCta][12];
    __shared__ double sK[kTetPerCta][144];
    const int le = threadIdx.x >> 4, t = threadIdx.x & 15;
    for (long base = (long)blockIdx.x * kTetPerCta; base < ne4; base += (long)gridDim.x * kTetPerCta) {
        const long e = base + le;
        const bool act = e < ne4;
        if (act && t < 12) {
            int a = t / 3, cc = t - 3 * a;
            int node = topo4[4 * e + a];
            sX[le][t] = xyz[3L * node + cc];
            if (NL) {
                int f = free_map[node];
                sU[le][t] = f >= 0 ? u[3L * f + cc] : 0.0;
            }
        }
        __syncthreads();
        if (act) {
            const int a = t >> 2, b = t & 3;
            const double *X = sX[le];
            // dN/d(rst) = [[-1,1,0,0],[-1,0,1,0],[-1,0,0,1]] (C3D4_hammer.cpp:26-28)
            double J[9];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) J[3 * i + j] = X[3 * (i + 1) + j] - X[j];
            double Ji[9];
            inv3(J, Ji);
            double G[4][3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                G[0][d] = -(Ji[3 * d] + Ji[3 * d + 1] + Ji[3 * d + 2]);
                G[1][d] = Ji[3 * d];
                G[2][d] = Ji[3 * d + 1];
                G[3][d] = Ji[3 * d + 2];
            }
            const double w = (1.0 / 6.0) * det_sarrus(J);  // signed, no abs (C3D4_hammer.cpp:70)
            const Lame L = lame(E4[e], nu);
            double k[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            if (!NL) {
                add_block_lin(k, G[a], G[b], w * L.lam, w * L.mu);
            } else {
                const double *U = sU[le];
                double F[9];
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        double s = (i == j) ? 1.0 : 0.0;
#pragma unroll
                        for (int c2 = 0; c2 < 4; ++c2) s += U[3 * c2 + i] * G[c2][j];
                        F[3 * i + j] = s;
                    }
                double S[6], C[9], pa[3], pb[3];
                tl_point(F, L, S, C);
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    pa[i] = F[3 * i] * G[a][0] + F[3 * i + 1] * G[a][1] + F[3 * i + 2] * G[a][2];
                    pb[i] = F[3 * i] * G[b][0] + F[3 * i + 1] * G[b][1] + F[3 * i + 2] * G[b][2];
                }
                add_block_nl(k, G[a], G[b], pa, pb, C, S, w, L);
                if (b == 0) {
                    double sg[3];
                    smat_vec(S, G[a], sg);
#pragma unroll
                    for (int i = 0; i < 3; ++i)
                        Fe[12 * e + 3 * a + i] = w * (F[3 * i] * sg[0] + F[3 * i + 1] * sg[1] + F[3 * i + 2] * sg[2]);
                }
            }
#pragma unroll
            for (int i = 0; i < 9; ++i) sK[le][(a * 4 + b) * 9 + i] = k[i];
        }
        __syncthreads();
        for (int v = threadIdx.x; v < kTetPerCta * 144; v += blockDim.x) {
            int l2 = v / 144;
            long e2 = base + l2;
            if (e2 < ne4) Ke[144 * e2 + (v - 144 * l2)] = sK[l2][v - 144 * l2];
        }
        __syncthreads();
    }
}

// -------------------------------------------------------------- assembly --

constexpr int kRowCap = 64;    // blocks accumulated in shared memory per warp
constexpr int kIncBatch = 8;   // incidences whose loads are in flight together

// The solver copy of K (BSELL-32, sell.cuh) that the owning warp writes with
// its row: slice layout of the current pattern and the three value arrays.
struct SellOut {
    const int *sl_ptr, *sl_g;
    double *sv64;
    __nv_bfloat16 *sv16, *svg;
};

// One warp per free node (block row).  Rows wider than kRowCap accumulate in
// global memory instead (still owned by the warp).  The warp also writes its
// row into the solver's BSELL copies (the separate fill pass is gone).

template <bool WITH_F>
__global__ void __launch_bounds__(kBlock) k_gather_assemble(
    int nfree, int ne8, const int *__restrict__ node_of_free, const int *__restrict__ inc_ptr,
    const int *__restrict__ inc, const uint16_t *__restrict__ slot, const int *__restrict__ rowptr,
    const double *__restrict__ Ke, double *__restrict__ Kb, const double *__restrict__ Fe,
    double *__restrict__ fint, SellOut so) {
    __shared__ double s_acc[kWarpsPerBlock][kRowCap * 9];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long ke8 = 576L * ne8;
    const int nwarps = gridDim.x * kWarpsPerBlock;
    for (int r = blockIdx.x * kWarpsPerBlock + warp; r < nfree; r += nwarps) {
        const int rb = rowptr[r], deg = rowptr[r + 1] - rb;
        const bool in_smem = deg <= kRowCap;
        double *acc = in_smem ? s_acc[warp] : Kb + 9L * rb;
        for (int v = lane; v < 9 * deg; v += 32) acc[v] = 0.0;
        __syncwarp();
        const int node = node_of_free[r];
        double fsum = 0.0;
        const int kb = inc_ptr[node], kend = inc_ptr[node + 1];
        // incidences in batches of kIncBatch: every load of a batch is issued
        // before the first sum, then the sums run in ascending incidence order
        for (int k0 = kb; k0 < kend; k0 += kIncBatch) {
            const int nk = min(kIncBatch, kend - k0);
            const int my_inc = lane < nk ? inc[k0 + lane] : 0;
            double val[kIncBatch][3];
            int sl[kIncBatch][3];
#pragma unroll
            for (int j = 0; j < kIncBatch; ++j) {
                const int ga = __shfl_sync(0xffffffffu, my_inc, j);
                const int g = ga >> 3, a = ga & 7;
                const bool hex = g < ne8;
                const int nv = hex ? 72 : 36;
                const double *row = hex ? Ke + 576L * g + 72 * a : Ke + ke8 + 144L * (g - ne8) + 36 * a;
#pragma unroll
                for (int t = 0; t < 3; ++t) {
                    const int v = lane + 32 * t;
                    const bool ok = j < nk && v < nv;
                    sl[j][t] = ok ? (int)slot[8L * (k0 + j) + v / 9] : (int)kNoSlot;
                    val[j][t] = ok ? row[v] : 0.0;
                }
                if (WITH_F && lane < 3 && j < nk)
                    fsum += hex ? Fe[24L * g + 3 * a + lane] : Fe[24L * ne8 + 12L * (g - ne8) + 3 * a + lane];
            }
#pragma unroll
            for (int j = 0; j < kIncBatch; ++j) {
#pragma unroll
                for (int t = 0; t < 3; ++t) {
                    const int v = lane + 32 * t;
                    if (sl[j][t] != kNoSlot) acc[9 * sl[j][t] + v % 9] += val[j][t];
                }
                __syncwarp();
            }
        }
        if (in_smem) {
            double *out = Kb + 9L * rb;
            for (int v = lane; v < 9 * deg; v += 32) out[v] = acc[v];
        }
        if (WITH_F && lane < 3) fint[3L * r + lane] = fsum;
        // the same row in the solver's layout (as k_fill_sell writes it):
        // slots up to the slice width, padding slots zero; FP64 and BF16
        // planes, then the BF16 copy grouped by four slots
        {
            const int sl = r / kSlice, t = r % kSlice;
            const long S = so.sl_ptr[sl];
            const int W = so.sl_ptr[sl + 1] - (int)S;
            for (int v = lane; v < 9 * W; v += 32) {
                const int k = v / 9, e = v - 9 * k;
                const double x = k < deg ? acc[v] : 0.0;
                so.sv64[((S + k) * 9 + e) * kSlice + t] = x;
                so.sv16[((S + k) * 9 + e) * kSlice + t] = __double2bfloat16(x);
            }
            const long G = so.sl_g[sl];
            uint2 *svg2 = reinterpret_cast<uint2 *>(so.svg);
            for (int p = lane; p < 9 * ((W + 3) / 4); p += 32) {
                const int g = p / 9, e = p - 9 * g;
                unsigned h[2] = {0u, 0u};
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int k = 4 * g + u;
                    const double x = k < deg ? acc[9 * k + e] : 0.0;
                    h[u >> 1] |= (unsigned)__bfloat16_as_ushort(__double2bfloat16(x)) << (16 * (u & 1));
                }
                svg2[((G + g) * 9 + e) * kSlice + t] = make_uint2(h[0], h[1]);
            }
        }
        __syncwarp();
    }
}

// Block-Jacobi: invert each diagonal 3x3 block (FP64, and an FP32 copy).
__global__ void k_block_jacobi(int nfree, const int *__restrict__ diag_pos, KBlocks K,
                               double *__restrict__ Dinv, float *__restrict__ Dinv32,
                               int *__restrict__ err) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nfree; r += gridDim.x * blockDim.x) {
        const int dp = diag_pos[r];
        double A[9], Ai[9];
        if (dp >= 0) {
#pragma unroll
            for (int i = 0; i < 9; ++i) A[i] = K.at(r, dp, i);
        } else {  // free node outside every element: K has an empty row
#pragma unroll
            for (int i = 0; i < 9; ++i) A[i] = 0.0;
        }
        if (!jacobi_inverse(A, Ai)) atomicExch(err, 1);
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            Dinv[9L * r + i] = Ai[i];
            Dinv32[9L * r + i] = (float)Ai[i];
        }
    }
}

// Block-CSR values from the FP64 BSELL copy (for callers that read K in CSR
// after a fused assembly, which writes only the solver's copy).
__global__ void k_sell_to_kb(int nfree, const int *__restrict__ rowptr, const int *__restrict__ sl_ptr,
                             const double *__restrict__ sv64, double *__restrict__ Kb) {
    for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < 9L * nfree; v += (long)gridDim.x * blockDim.x) {
        const int r = (int)(v / 9), e = (int)(v - 9L * r);
        const long S = sl_ptr[r / kSlice];
        const int rb = rowptr[r], deg = rowptr[r + 1] - rb, t = r % kSlice;
        for (int k = 0; k < deg; ++k) Kb[9L * (rb + k) + e] = sv64[((S + k) * 9 + e) * kSlice + t];
    }
}

// BF16 plane copy from the FP64 planes (the batched engine's operand).
__global__ void k_sv64_to_sv16(long len, const double *__restrict__ sv64, __nv_bfloat16 *__restrict__ sv16) {
    for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < len; v += (long)gridDim.x * blockDim.x)
        sv16[v] = __double2bfloat16(sv64[v]);
}

static void integrate(ofea_ctx *c, bool nl, const double *d_u) {
    upload_hex_table();
    cudaStream_t s = c->stream;
    size_t ke_len = 576L * c->ne8 + 144L * c->ne4;
    c->Ke.ensure(ke_len);
    if (nl) c->Fe.ensure(24L * c->ne8 + 12L * c->ne4 + 1);
    double *Fe8 = nl ? c->Fe.p : nullptr;
    double *Fe4 = nl ? c->Fe.p + 24L * c->ne8 : nullptr;
    if (c->ne8 > 0) {
        int g = grid_for(c, (c->ne8 + kHexPerCta - 1) / kHexPerCta, 1);
        g = std::min(g, c->num_sms * 8);
        if (nl)
            k_hex_integrate<true><<<g, 128, 0, s>>>(c->ne8, c->topo8.p, c->xyz.p, c->E8.p, c->nu,
                                                    c->free_map.p, d_u, c->Ke.p, Fe8);
        else
            k_hex_integrate_lin<<<std::min(grid_for(c, (c->ne8 + kLinHex - 1) / kLinHex, 1), c->num_sms * 16),
                                  128, 0, s>>>(c->ne8, c->topo8.p, c->xyz.p, c->E8.p, c->nu, c->Ke.p);
        OFEA_CHECK_LAUNCH();
    }
    if (c->ne4 > 0) {
        int g = grid_for(c, (c->ne4 + kTetPerCta - 1) / kTetPerCta, 1);
        g = std::min(g, c->num_sms * 12);
        double *Ke4 = c->Ke.p + 576L * c->ne8;
        if (nl)
            k_tet_integrate<true><<<g, 128, 0, s>>>(c->ne4, c->topo4.p, c->xyz.p, c->E4.p, c->nu,
                                                    c->free_map.p, d_u, Ke4, Fe4);
        else
            k_tet_integrate<false><<<g, 128, 0, s>>>(c->ne4, c->topo4.p, c->xyz.p, c->E4.p, c->nu,
                                                     nullptr, nullptr, Ke4, nullptr);
        OFEA_CHECK_LAUNCH();
    }
    c->ke_ok = true;
}

static void gather(ofea_ctx *c, bool with_f, double *d_fint) {
    c->Kb.ensure((size_t)std::max<long long>(9 * c->nnzb, 1));
    if (!c->sell_layout_ok) build_sell_layout(c);
    const SellOut so{c->sl_ptr.p, c->sl_g.p, c->sv64.p, c->sv16.p, c->sv16g.p};
    int gw = grid_for(c, c->nfree, kWarpsPerBlock);
    if (with_f)
        k_gather_assemble<true><<<gw, kBlock, 0, c->stream>>>(
            c->nfree, c->ne8, c->node_of_free.p, c->inc_ptr.p, c->inc.p, c->slot.p, c->rowptr.p,
            c->Ke.p, c->Kb.p, c->Fe.p, d_fint, so);
    else
        k_gather_assemble<false><<<gw, kBlock, 0, c->stream>>>(
            c->nfree, c->ne8, c->node_of_free.p, c->inc_ptr.p, c->inc.p, c->slot.p, c->rowptr.p,
            c->Ke.p, c->Kb.p, nullptr, nullptr, so);
    OFEA_CHECK_LAUNCH();
    c->K_ok = true;
    c->kb_ok = true;
    c->asm_path = 1;
    c->sell_ok = true;  // written by the gather, BF16 planes included
    c->sv16_ok = true;
    c->jacobi_fresh = false;
    c->coarse.K_ok = false;
    c->coarse2.K_ok = false;
}

// Slice element lists of the current pattern (one host sync, once per
// pattern); se_state 1 when the fused assembly covers the mesh, -1 if not.
static void build_slice_elements(ofea_ctx *c) {
    c->se_state = -1;
    if (c->ne4 != 0 || c->ne8 == 0 || c->nfree == 0 || c->fused_off) return;
    if (!c->sell_layout_ok) build_sell_layout(c);
    cudaStream_t s = c->stream;
    const int nslice = (c->nfree + kSlice - 1) / kSlice;
    const int tmp_len = nslice / 1024 + 4;
    c->scratch_i.ensure((size_t)nslice + 1 + tmp_len + 4);
    int *cnt = c->scratch_i.p, *tmp = cnt + nslice + 1, *stats = tmp + tmp_len;
    c->se_ptr.ensure((size_t)nslice + 1);
    OFEA_CUDA(cudaMemsetAsync(stats, 0, 4 * sizeof(int), s));
    const int g = std::min(nslice, c->num_sms * 8);
    k_slice_elements<false><<<g, kSeThreads, 0, s>>>(c->nfree, c->node_of_free.p, c->inc_ptr.p, c->inc.p,
                                                     c->sl_ptr.p, nullptr, cnt, nullptr, nullptr, stats);
    OFEA_CHECK_LAUNCH();
    const long long total = exclusive_scan(cnt, c->se_ptr.p, nslice, s, tmp, tmp_len);
    c->herr.ensure(4);
    OFEA_CUDA(cudaMemcpyAsync(c->herr.p, stats, 3 * sizeof(int), cudaMemcpyDeviceToHost, s));
    OFEA_CUDA(cudaStreamSynchronize(s));
    if (c->herr.p[0] != 0 || c->herr.p[1] > kFuMaxW || c->herr.p[2] > kFuMaxElem) return;
    c->se_list.ensure((size_t)std::max<long long>(total, 1));
    c->inc_loc.ensure((size_t)std::max<long>(8L * c->ne8, 1));
    k_slice_elements<true><<<g, kSeThreads, 0, s>>>(c->nfree, c->node_of_free.p, c->inc_ptr.p, c->inc.p,
                                                    c->sl_ptr.p, c->se_ptr.p, nullptr, c->se_list.p,
                                                    c->inc_loc.p, stats);
    OFEA_CHECK_LAUNCH();
    c->se_state = 1;
}

// Fused linear assembly when the mesh allows it; false leaves K untouched.
static bool assemble_linear_fused(ofea_ctx *c) {
    if (c->se_state == 0) build_slice_elements(c);
    if (c->se_state != 1 || c->fused_off) return false;
    upload_hex_table();
    cudaStream_t s = c->stream;
    c->Dinv.ensure((size_t)9 * std::max(c->nfree, 1));
    c->Dinv32.ensure((size_t)9 * std::max(c->nfree, 1));
    OFEA_CUDA(cudaMemsetAsync(c->err_flag.p, 0, sizeof(int), s));
    OFEA_CUDA(cudaFuncSetAttribute(k_hex_assemble_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFuSmem));
    const int nslice = (c->nfree + kSlice - 1) / kSlice;
    const int g = std::min(nslice, c->num_sms);
    k_hex_assemble_fused<<<g, kFuThreads, kFuSmem, s>>>(
        c->nfree, c->node_of_free.p, c->inc_ptr.p, c->inc.p, c->slot.p, c->inc_loc.p, c->se_ptr.p, c->se_list.p,
        c->topo8.p, c->xyz.p, c->E8.p, c->nu, c->diag_pos.p, c->sl_ptr.p, c->sl_g.p, c->sv64.p, c->sv16g.p,
        c->Dinv.p, c->Dinv32.p, c->err_flag.p);
    OFEA_CHECK_LAUNCH();
    c->K_ok = true;
    c->asm_path = 0;
    c->sell_ok = true;
    c->kb_ok = false;        // block CSR on demand (ensure_kb)
    c->sv16_ok = false;      // BF16 planes on demand (ensure_sv16)
    c->ke_ok = false;        // element matrices on demand (ensure_element_matrices)
    c->jacobi_fresh = true;  // Dinv written by the kernel
    c->coarse.K_ok = false;
    c->coarse2.K_ok = false;
    return true;
}

void assemble_linear(ofea_ctx *c) {
    if (assemble_linear_fused(c)) return;
    integrate(c, false, nullptr);
    gather(c, false, nullptr);
}

void assemble_nl(ofea_ctx *c, const double *d_u, double *d_fint) {
    integrate(c, true, d_u);
    gather(c, true, d_fint);
}

void build_block_jacobi(ofea_ctx *c) {
    c->Dinv.ensure((size_t)9 * std::max(c->nfree, 1));
    c->Dinv32.ensure((size_t)9 * std::max(c->nfree, 1));
    OFEA_CUDA(cudaMemsetAsync(c->err_flag.p, 0, sizeof(int), c->stream));
    k_block_jacobi<<<grid_for(c, c->nfree, kBlock), kBlock, 0, c->stream>>>(
        c->nfree, c->diag_pos.p, kblocks(c), c->Dinv.p, c->Dinv32.p, c->err_flag.p);
    OFEA_CHECK_LAUNCH();
}

void ensure_kb(ofea_ctx *c) {
    if (c->kb_ok) return;
    c->Kb.ensure((size_t)std::max<long long>(9 * c->nnzb, 1));
    k_sell_to_kb<<<grid_for(c, 9L * c->nfree, kBlock), kBlock, 0, c->stream>>>(c->nfree, c->rowptr.p, c->sl_ptr.p,
                                                                              c->sv64.p, c->Kb.p);
    OFEA_CHECK_LAUNCH();
    c->kb_ok = true;
}

void ensure_sv16(ofea_ctx *c) {
    if (c->sv16_ok) return;
    const long len = 9L * std::max<long long>(c->sell_len, 1) * kSlice;
    k_sv64_to_sv16<<<grid_for(c, len, kBlock), kBlock, 0, c->stream>>>(len, c->sv64.p, c->sv16.p);
    OFEA_CHECK_LAUNCH();
    c->sv16_ok = true;
}

void ensure_element_matrices(ofea_ctx *c) {
    if (c->ke_ok) return;
    integrate(c, false, nullptr);  // the fused assembly left none: the linear ones it summed
}

// --------------------------------------------------------- stress recovery --
// simulation_post::get_cauchy_stress_3d (src/post_process.cpp:79-167): seven
// values per element (xx yy zz xy yz xz and the von Mises expression of
// :103-109 applied to them), then per node the mean over its incident
// elements.  Mode 0 is the reference's quantity: for C3D4 the engineering
// strain B u that its get_stress_node_hammer returns as "stress"
// (src/Elements/C3D4_hammer.cpp:219-226, the D product commented out); for
// C3D8, which has no get_stress_node (the base-class stub leaves the values
// unset), zero.  Mode 1 is the Cauchy stress D B u (C3D8: the mean over its
// eight Gauss points).  Element values are stored by unified id g (hexes,
// then tets).

__device__ __forceinline__ void strain_from_grads(const double (*g)[3], const double (*U)[3], int nn, double *e) {
    for (int k = 0; k < 6; ++k) e[k] = 0.0;
    for (int a = 0; a < nn; ++a) {
        e[0] += g[a][0] * U[a][0];
        e[1] += g[a][1] * U[a][1];
        e[2] += g[a][2] * U[a][2];
        e[3] += g[a][1] * U[a][0] + g[a][0] * U[a][1];
        e[4] += g[a][2] * U[a][1] + g[a][1] * U[a][2];
        e[5] += g[a][2] * U[a][0] + g[a][0] * U[a][2];
    }
}

__device__ __forceinline__ void stress_from_strain(const Lame &L, const double *e, double *s) {
    const double tr = e[0] + e[1] + e[2];
    for (int k = 0; k < 3; ++k) s[k] = L.lam * tr + 2.0 * L.mu * e[k];
    for (int k = 3; k < 6; ++k) s[k] = L.mu * e[k];
}

__device__ __forceinline__ double mises_ref(const double *s) {
    return sqrt(0.5 * ((s[0] - s[1]) * (s[0] - s[1]) + (s[1] - s[2]) * (s[1] - s[2]) + (s[2] - s[0]) * (s[2] - s[0]) +
                       6.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5])));
}

// Gathers the element's coordinates and displacements (fixed DOF: 0).
template <int NN>
__device__ __forceinline__ void gather_elem(const int *t, const double *xyz, const int *free_map, const double *u,
                                            double (*X)[3], double (*U)[3]) {
    for (int a = 0; a < NN; ++a) {
        const int node = t[a], f = free_map[node];
        for (int d = 0; d < 3; ++d) {
            X[a][d] = xyz[3L * node + d];
            U[a][d] = f >= 0 ? u[3L * f + d] : 0.0;
        }
    }
}

__global__ void k_tet_stress(int ne4, int ne8, const int *__restrict__ topo4, const double *__restrict__ xyz,
                             const double *__restrict__ E4, double nu, const int *__restrict__ free_map,
                             const double *__restrict__ u, int mode, double *__restrict__ out) {
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < ne4; e += (long)gridDim.x * blockDim.x) {
        double X[4][3], U[4][3];
        gather_elem<4>(topo4 + 4 * e, xyz, free_map, u, X, U);
        // J = dN/d(r,s,t) X with dN rows (-1 1 0 0), (-1 0 1 0), (-1 0 0 1)
        double J[9];
        for (int i = 0; i < 3; ++i)
            for (int d = 0; d < 3; ++d) J[3 * i + d] = X[i + 1][d] - X[0][d];
        double Ji[9];
        inv3(J, Ji);
        double g[4][3];
        for (int i = 0; i < 3; ++i) {
            g[0][i] = -(Ji[3 * i] + Ji[3 * i + 1] + Ji[3 * i + 2]);
            for (int a = 1; a < 4; ++a) g[a][i] = Ji[3 * i + a - 1];
        }
        double eps[6], s[7];
        strain_from_grads(g, U, 4, eps);
        if (mode == 1) stress_from_strain(lame(E4[e], nu), eps, s);
        else
            for (int k = 0; k < 6; ++k) s[k] = eps[k];
        s[6] = mises_ref(s);
        for (int k = 0; k < 7; ++k) out[(ne8 + e) * 7 + k] = s[k];
    }
}

__global__ void k_hex_stress(int ne8, const int *__restrict__ topo8, const double *__restrict__ xyz,
                             const double *__restrict__ E8, double nu, const int *__restrict__ free_map,
                             const double *__restrict__ u, int mode, double *__restrict__ out) {
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < ne8; e += (long)gridDim.x * blockDim.x) {
        double s[7] = {0, 0, 0, 0, 0, 0, 0};
        if (mode == 1) {
            double X[8][3], U[8][3];
            gather_elem<8>(topo8 + 8 * e, xyz, free_map, u, X, U);
            const Lame L = lame(E8[e], nu);
            for (int q = 0; q < 8; ++q) {
                const double *dN = c_hex_dN + q * 24;
                double J[9];
                for (int i = 0; i < 3; ++i)
                    for (int d = 0; d < 3; ++d) {
                        double v = 0;
                        for (int b = 0; b < 8; ++b) v += dN[i * 8 + b] * X[b][d];
                        J[3 * i + d] = v;
                    }
                double Ji[9];
                inv3(J, Ji);
                double g[8][3];
                for (int a = 0; a < 8; ++a)
                    for (int i = 0; i < 3; ++i)
                        g[a][i] = Ji[3 * i] * dN[a] + Ji[3 * i + 1] * dN[8 + a] + Ji[3 * i + 2] * dN[16 + a];
                double eps[6], sq[6];
                strain_from_grads(g, U, 8, eps);
                stress_from_strain(L, eps, sq);
                for (int k = 0; k < 6; ++k) s[k] += 0.125 * sq[k];
            }
            s[6] = mises_ref(s);
        }
        for (int k = 0; k < 7; ++k) out[e * 7 + k] = s[k];
    }
}

// node[k * nd + i] = mean over node i's incident elements (ascending g) of
// their value k; 0 for a node on no element.
__global__ void k_node_mean(int nd, const int *__restrict__ inc_ptr, const int *__restrict__ inc,
                            const double *__restrict__ elem, double *__restrict__ node) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nd; i += (long)gridDim.x * blockDim.x) {
        const int b = inc_ptr[i], cnt = inc_ptr[i + 1] - b;
        double acc[7] = {0, 0, 0, 0, 0, 0, 0};
        for (int j = 0; j < cnt; ++j) {
            const long g = inc[b + j] >> 3;
            for (int k = 0; k < 7; ++k) acc[k] += elem[g * 7 + k];
        }
        for (int k = 0; k < 7; ++k) node[k * (long)nd + i] = cnt > 0 ? acc[k] / cnt : 0.0;
    }
}

void stress_recovery(ofea_ctx *c, const double *d_u, int mode, double *d_elem, double *d_node) {
    cudaStream_t s = c->stream;
    upload_hex_table();
    if (c->ne8 > 0)
        k_hex_stress<<<grid_for(c, c->ne8, kBlock), kBlock, 0, s>>>(c->ne8, c->topo8.p, c->xyz.p, c->E8.p, c->nu,
                                                                     c->free_map.p, d_u, mode, d_elem);
    if (c->ne4 > 0)
        k_tet_stress<<<grid_for(c, c->ne4, kBlock), kBlock, 0, s>>>(c->ne4, c->ne8, c->topo4.p, c->xyz.p, c->E4.p,
                                                                     c->nu, c->free_map.p, d_u, mode, d_elem);
    k_node_mean<<<grid_for(c, c->nd, kBlock), kBlock, 0, s>>>(c->nd, c->inc_ptr.p, c->inc.p, d_elem, d_node);
    OFEA_CHECK_LAUNCH();
}

}  // namespace ofea
