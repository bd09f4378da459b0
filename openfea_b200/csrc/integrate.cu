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
    __shared__ double sX[kLinHex][24];
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
            const int le = tid >> 3, q = tid & 7;
            if (le < nel) {
                const double *dN = c_hex_dN + q * 24;
                double J[9];
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        double acc = 0;
#pragma unroll
                        for (int b = 0; b < 8; ++b) acc += dN[i * 8 + b] * sX[le][3 * b + j];
                        J[3 * i + j] = acc;
                    }
                double Ji[9];
                inv3(J, Ji);
                sW[le][q] = det_sarrus(J);  // Gauss weight 1
#pragma unroll
                for (int a = 0; a < 8; ++a)
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        sG[le][q][a][d] = Ji[3 * d] * dN[a] + Ji[3 * d + 1] * dN[8 + a] + Ji[3 * d + 2] * dN[16 + a];
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
            double T[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, d = 0;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const double w = sW[le][q];
                const double ga0 = w * sG[le][q][a][0], ga1 = w * sG[le][q][a][1], ga2 = w * sG[le][q][a][2];
                const double gb0 = sG[le][q][b][0], gb1 = sG[le][q][b][1], gb2 = sG[le][q][b][2];
                T[0] = fma(ga0, gb0, T[0]);
                T[1] = fma(ga0, gb1, T[1]);
                T[2] = fma(ga0, gb2, T[2]);
                T[3] = fma(ga1, gb0, T[3]);
                T[4] = fma(ga1, gb1, T[4]);
                T[5] = fma(ga1, gb2, T[5]);
                T[6] = fma(ga2, gb0, T[6]);
                T[7] = fma(ga2, gb1, T[7]);
                T[8] = fma(ga2, gb2, T[8]);
            }
            d = T[0] + T[4] + T[8];
            const Lame L = lame(E8[base + le], nu);
            double kab[9];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) kab[3 * i + j] = L.lam * T[3 * i + j] + L.mu * T[3 * j + i] + (i == j ? L.mu * d : 0.0);
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

// ------------------------------------------------------------------ C3D4 --

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
__global__ void k_block_jacobi(int nfree, const int *__restrict__ rowptr,
                               const int *__restrict__ diag_pos, const double *__restrict__ Kb,
                               double *__restrict__ Dinv, float *__restrict__ Dinv32,
                               int *__restrict__ err) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nfree; r += gridDim.x * blockDim.x) {
        const int dp = diag_pos[r];
        double A[9], Ai[9];
        if (dp >= 0) {
            const double *D = Kb + 9L * (rowptr[r] + dp);
#pragma unroll
            for (int i = 0; i < 9; ++i) A[i] = D[i];
        } else {  // free node outside every element: K has an empty row
#pragma unroll
            for (int i = 0; i < 9; ++i) A[i] = 0.0;
        }
        double det = A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
                     A[2] * (A[3] * A[7] - A[4] * A[6]);
        if (!(det > 0.0) || !isfinite(det)) {
            atomicExch(err, 1);
#pragma unroll
            for (int i = 0; i < 9; ++i) Ai[i] = (i % 4 == 0) ? 1.0 : 0.0;
        } else {
            inv3(A, Ai);
        }
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            Dinv[9L * r + i] = Ai[i];
            Dinv32[9L * r + i] = (float)Ai[i];
        }
    }
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
    c->sell_ok = true;  // written by the gather
    c->coarse.K_ok = false;
    c->coarse2.K_ok = false;
}

void assemble_linear(ofea_ctx *c) {
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
        c->nfree, c->rowptr.p, c->diag_pos.p, c->Kb.p, c->Dinv.p, c->Dinv32.p, c->err_flag.p);
    OFEA_CHECK_LAUNCH();
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
