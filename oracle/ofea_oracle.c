/* ofea_oracle.c - CPU restatement of OpenFEA's implicit-static hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see ofea_oracle.h).  Plain C, no dependencies.
 * Parity is pinned: tests/test_oracle.py checks every function here against
 * the reference's own routines compiled in oracle/_ref and against the golden
 * VTK output shipped with the reference (sample_model/CA/cadcae_o.vtk).
 *
 * The element routines below deliberately follow the reference's DENSE form
 * (explicit B matrices, B^T D B products), not the structured nodal-block
 * form the GPU kernels use, so that the two are independent derivations.
 */
#include "ofea_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ BCs -- */

static int cmp_int(const void *a, const void *b) {
    int x = *(const int *)a, y = *(const int *)b;
    return (x > y) - (x < y);
}

/* src/set_bc.cpp:20-43: sort fixed ids ascending, walk all nodes; a node that
 * equals the current fixed id gets -1, every other node the next free index. */
int orc_build_free_index(int nd, int nfix, const int *fix_ids, int *free_map) {
    if (nfix <= 0) return -1;
    int *s = (int *)malloc(sizeof(int) * (size_t)nfix);
    memcpy(s, fix_ids, sizeof(int) * (size_t)nfix);
    qsort(s, (size_t)nfix, sizeof(int), cmp_int);
    for (int k = 0; k < nfix; ++k) {
        if (s[k] < 1 || s[k] > nd || (k > 0 && s[k] == s[k - 1])) {
            free(s);
            return -1;
        }
    }
    int next = 0, c = 0;
    for (int i = 0; i < nd; ++i) {
        if (i == s[c] - 1) {
            free_map[i] = -1;
            if (c < nfix - 1) ++c;
        } else {
            free_map[i] = next++;
        }
    }
    free(s);
    return nd - nfix;
}

/* ------------------------------------------------------------ elements -- */

void orc_cons_mat(double E, double nu, double D[36]) {
    /* src/Elements/C3D8.cpp:23-34 */
    double fac = (E * (1.0 - nu)) / ((1.0 + nu) * (1.0 - 2.0 * nu));
    double fa = fac * nu / (1.0 - nu);
    double fb = fac * (1.0 - 2.0 * nu) / (2.0 * (1.0 - nu));
    memset(D, 0, 36 * sizeof(double));
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) D[6 * i + j] = (i == j) ? fac : fa;
    D[6 * 3 + 3] = fb;
    D[6 * 4 + 4] = fb;
    D[6 * 5 + 5] = fb;
}

/* 3x3 helpers (row-major). */
static double det3_sarrus(const double J[9]) {
    /* the reference's determinant expression (C3D8_Gauss.cpp:58-63) */
    return J[0] * J[4] * J[8] + J[1] * J[5] * J[6] + J[2] * J[3] * J[7] - J[2] * J[4] * J[6] -
           J[5] * J[7] * J[0] - J[8] * J[1] * J[3];
}
static void inv3(const double J[9], double Ji[9]) {
    /* cofactor inverse (the reference calls Eigen's 3x3 inverse) */
    double c00 = J[4] * J[8] - J[5] * J[7];
    double c01 = J[5] * J[6] - J[3] * J[8];
    double c02 = J[3] * J[7] - J[4] * J[6];
    double det = J[0] * c00 + J[1] * c01 + J[2] * c02;
    double id = 1.0 / det;
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

/* Shape-function derivatives in (r,s,t) for the 8-node brick, 3 x 8,
 * node order of src/Elements/C3D8_Gauss.cpp:27-52. */
static void hex_dN(double r, double s, double t, double dN[24]) {
    static const double sr[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
    static const double ss[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
    static const double st[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
    for (int a = 0; a < 8; ++a) {
        dN[0 * 8 + a] = 0.125 * sr[a] * (1.0 + ss[a] * s) * (1.0 + st[a] * t);
        dN[1 * 8 + a] = 0.125 * ss[a] * (1.0 + sr[a] * r) * (1.0 + st[a] * t);
        dN[2 * 8 + a] = 0.125 * st[a] * (1.0 + sr[a] * r) * (1.0 + ss[a] * s);
    }
}
/* Gauss points in the order of src/Elements/C3D8_Gauss.cpp:84-92. */
static void hex_gp(int i, double *r, double *s, double *t) {
    static const double sr[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
    static const double ss[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
    static const double st[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
    double g = 1.0 / sqrt(3.0);
    *r = sr[i] * g;
    *s = ss[i] * g;
    *t = st[i] * g;
}
/* Tet derivatives, src/Elements/C3D4_hammer.cpp:26-28. */
static void tet_dN(double dN[12]) {
    static const double d[12] = {-1, 1, 0, 0, -1, 0, 1, 0, -1, 0, 0, 1};
    memcpy(dN, d, sizeof(d));
}

/* J = dN * X (3 x npe by npe x 3), g = J^-1 dN (3 x npe); returns Sarrus det. */
static double grad_N(int npe, const double *dN, const double *X, double *g) {
    double J[9] = {0}, Ji[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0;
            for (int a = 0; a < npe; ++a) s += dN[i * npe + a] * X[3 * a + j];
            J[3 * i + j] = s;
        }
    inv3(J, Ji);
    for (int i = 0; i < 3; ++i)
        for (int a = 0; a < npe; ++a) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += Ji[3 * i + k] * dN[k * npe + a];
            g[i * npe + a] = s;
        }
    return det3_sarrus(J);
}

/* Linear B (6 x 3npe), src/Elements/C3D8_Gauss.cpp:64-75. */
static void build_B(int npe, const double *g, double *B) {
    int m = 3 * npe;
    memset(B, 0, sizeof(double) * 6 * (size_t)m);
    for (int a = 0; a < npe; ++a) {
        double gx = g[0 * npe + a], gy = g[1 * npe + a], gz = g[2 * npe + a];
        B[0 * m + 3 * a] = gx;
        B[1 * m + 3 * a + 1] = gy;
        B[2 * m + 3 * a + 2] = gz;
        B[3 * m + 3 * a] = gy;
        B[3 * m + 3 * a + 1] = gx;
        B[4 * m + 3 * a + 1] = gz;
        B[4 * m + 3 * a + 2] = gy;
        B[5 * m + 3 * a] = gz;
        B[5 * m + 3 * a + 2] = gx;
    }
}

/* K += c * B^T D B  (B 6 x m), in the reference's association (B^T D) B. */
static void add_BtDB(int m, const double *B, const double *D, double c, double *K) {
    double *BtD = (double *)malloc(sizeof(double) * 6 * (size_t)m);
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < 6; ++j) {
            double s = 0;
            for (int k = 0; k < 6; ++k) s += B[k * m + i] * D[6 * k + j];
            BtD[6 * i + j] = s;
        }
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) {
            double s = 0;
            for (int k = 0; k < 6; ++k) s += BtD[6 * i + k] * B[k * m + j];
            K[i * m + j] += c * s;
        }
    free(BtD);
}

double orc_c3d8_ke(const double *X, double E, double nu, double *Ke) {
    double D[36], dN[24], g[24], B[6 * 24], det = 0;
    orc_cons_mat(E, nu, D);
    memset(Ke, 0, sizeof(double) * 576);
    for (int q = 0; q < 8; ++q) {
        double r, s, t;
        hex_gp(q, &r, &s, &t);
        hex_dN(r, s, t, dN);
        det = grad_N(8, dN, X, g);
        build_B(8, g, B);
        add_BtDB(24, B, D, 1.0 * det, Ke); /* weight 1 (C3D8_Gauss.cpp:93,105) */
    }
    return det;
}

double orc_c3d4_ke(const double *X, double E, double nu, double *Ke) {
    double D[36], dN[12], g[12], B[6 * 12];
    orc_cons_mat(E, nu, D);
    memset(Ke, 0, sizeof(double) * 144);
    tet_dN(dN);
    double det = grad_N(4, dN, X, g);
    build_B(4, g, B);
    /* Ke = (B^T D B), then scaled by weight*det (C3D4_hammer.cpp:68-70); no abs(det). */
    add_BtDB(12, B, D, 1.0, Ke);
    for (int i = 0; i < 144; ++i) Ke[i] = (1.0 / 6.0) * det * Ke[i];
    return det;
}

/* One integration point of the Total-Lagrangian tangent (reference dense form,
 * src/Elements/C3D8_Gauss.cpp:110-217 / C3D4_hammer.cpp:75-152). */
static void nl_point(int npe, const double *g, const double *u_el, const double *D, double c,
                     double *Ke, double *fint) {
    int m = 3 * npe;
    double F[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = (i == j) ? 1.0 : 0.0;
            for (int a = 0; a < npe; ++a) s += u_el[i * npe + a] * g[j * npe + a];
            F[3 * i + j] = s;
        }
    double Eg[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += F[3 * k + i] * F[3 * k + j];
            Eg[3 * i + j] = 0.5 * (s - (i == j ? 1.0 : 0.0));
        }
    double ev[6] = {Eg[0], Eg[4], Eg[8], 2.0 * Eg[1], 2.0 * Eg[5], 2.0 * Eg[2]};
    double S[6];
    for (int i = 0; i < 6; ++i) {
        double s = 0;
        for (int k = 0; k < 6; ++k) s += D[6 * i + k] * ev[k];
        S[i] = s;
    }
    double *BL = (double *)calloc(6 * (size_t)m, sizeof(double));
    double *BN = (double *)calloc(9 * (size_t)m, sizeof(double));
    for (int a = 0; a < npe; ++a) {
        double gx = g[0 * npe + a], gy = g[1 * npe + a], gz = g[2 * npe + a];
        for (int k = 0; k < 3; ++k) {
            int col = 3 * a + k;
            BL[0 * m + col] = F[3 * k + 0] * gx;
            BL[1 * m + col] = F[3 * k + 1] * gy;
            BL[2 * m + col] = F[3 * k + 2] * gz;
            BL[3 * m + col] = F[3 * k + 0] * gy + F[3 * k + 1] * gx;
            BL[4 * m + col] = F[3 * k + 1] * gz + F[3 * k + 2] * gy;
            BL[5 * m + col] = F[3 * k + 0] * gz + F[3 * k + 2] * gx;
            BN[(3 * k + 0) * m + col] = gx;
            BN[(3 * k + 1) * m + col] = gy;
            BN[(3 * k + 2) * m + col] = gz;
        }
    }
    /* SIG = blockdiag(Smat, Smat, Smat), Smat = [[S0,S3,S5],[S3,S1,S4],[S5,S4,S2]] */
    double Sm[9] = {S[0], S[3], S[5], S[3], S[1], S[4], S[5], S[4], S[2]};
    for (int i = 0; i < m; ++i) {
        double s = 0;
        for (int k = 0; k < 6; ++k) s += BL[k * m + i] * S[k];
        fint[i] += c * s;
    }
    add_BtDB(m, BL, D, c, Ke);
    /* + c * BN^T SIG BN */
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) {
            double s = 0;
            for (int blk = 0; blk < 3; ++blk)
                for (int p = 0; p < 3; ++p)
                    for (int q = 0; q < 3; ++q)
                        s += BN[(3 * blk + p) * m + i] * Sm[3 * p + q] * BN[(3 * blk + q) * m + j];
            Ke[i * m + j] += c * s;
        }
    free(BL);
    free(BN);
}

void orc_c3d8_nl(const double *X, const double *u_el, double E, double nu, double *Ke,
                 double *fint) {
    double D[36], dN[24], g[24];
    orc_cons_mat(E, nu, D);
    memset(Ke, 0, sizeof(double) * 576);
    memset(fint, 0, sizeof(double) * 24);
    for (int q = 0; q < 8; ++q) {
        double r, s, t;
        hex_gp(q, &r, &s, &t);
        hex_dN(r, s, t, dN);
        double det = grad_N(8, dN, X, g);
        nl_point(8, g, u_el, D, 1.0 * det, Ke, fint);
    }
}

void orc_c3d4_nl(const double *X, const double *u_el, double E, double nu, double *Ke,
                 double *fint) {
    double D[36], dN[12], g[12];
    orc_cons_mat(E, nu, D);
    memset(Ke, 0, sizeof(double) * 144);
    memset(fint, 0, sizeof(double) * 12);
    tet_dN(dN);
    double det = grad_N(4, dN, X, g);
    nl_point(4, g, u_el, D, (1.0 / 6.0) * det, Ke, fint);
}

/* ------------------------------------------------------------- pattern -- */

static int npe_of(int t) { return t == 1 ? 8 : 4; }

/* Node adjacency over free nodes (sorted unique neighbour lists).  Output:
 * nptr (nfree+1) and nidx, both malloc'ed. */
static void node_adjacency(int nd, int ne, const int *topo, const int *etype,
                           const int *free_map, int nfree, int **nptr_out, int **nidx_out) {
    int *cnt = (int *)calloc((size_t)nd + 1, sizeof(int));
    for (int e = 0; e < ne; ++e)
        for (int a = 0; a < npe_of(etype[e]); ++a) cnt[topo[8 * e + a] - 1 + 1]++;
    for (int i = 0; i < nd; ++i) cnt[i + 1] += cnt[i];
    int *inc = (int *)malloc(sizeof(int) * (size_t)(cnt[nd] > 0 ? cnt[nd] : 1));
    int *cur = (int *)malloc(sizeof(int) * (size_t)nd);
    memcpy(cur, cnt, sizeof(int) * (size_t)nd);
    for (int e = 0; e < ne; ++e)
        for (int a = 0; a < npe_of(etype[e]); ++a) inc[cur[topo[8 * e + a] - 1]++] = e;
    int *nptr = (int *)calloc((size_t)nfree + 1, sizeof(int));
    int cap = 1024, *buf = (int *)malloc(sizeof(int) * (size_t)cap);
    /* pass 1: counts; pass 2: fill */
    int *nidx = NULL;
    for (int pass = 0; pass < 2; ++pass) {
        for (int i = 0; i < nd; ++i) {
            int r = free_map[i];
            if (r < 0) continue;
            int m = 0;
            for (int k = cnt[i]; k < cnt[i + 1]; ++k) {
                int e = inc[k];
                for (int b = 0; b < npe_of(etype[e]); ++b) {
                    int s = free_map[topo[8 * e + b] - 1];
                    if (s < 0) continue;
                    if (m == cap) {
                        cap *= 2;
                        buf = (int *)realloc(buf, sizeof(int) * (size_t)cap);
                    }
                    buf[m++] = s;
                }
            }
            qsort(buf, (size_t)m, sizeof(int), cmp_int);
            int u = 0;
            for (int k = 0; k < m; ++k)
                if (k == 0 || buf[k] != buf[k - 1]) buf[u++] = buf[k];
            if (pass == 0)
                nptr[r + 1] = u;
            else
                memcpy(nidx + nptr[r], buf, sizeof(int) * (size_t)u);
        }
        if (pass == 0) {
            for (int r = 0; r < nfree; ++r) nptr[r + 1] += nptr[r];
            nidx = (int *)malloc(sizeof(int) * (size_t)(nptr[nfree] > 0 ? nptr[nfree] : 1));
        }
    }
    free(buf);
    free(cur);
    free(inc);
    free(cnt);
    *nptr_out = nptr;
    *nidx_out = nidx;
}

/* The reference inserts, for every element, every (row, col) pair of its free
 * DOFs into a per-column std::set (src/assemble.cpp:25-53).  With whole-node
 * constraints this is the node adjacency expanded to 3x3 blocks, columns in
 * DOF order 3*s + c with rows ascending. */
long long orc_pattern_count(int nd, int ne, const int *topo, const int *etype,
                            const int *free_map, int n, int *col_ptr) {
    int nfree = n / 3, *nptr, *nidx;
    node_adjacency(nd, ne, topo, etype, free_map, nfree, &nptr, &nidx);
    col_ptr[0] = 0;
    long long tot = 0;
    for (int r = 0; r < nfree; ++r) {
        int deg = nptr[r + 1] - nptr[r];
        for (int c = 0; c < 3; ++c) {
            tot += 3LL * deg;
            col_ptr[3 * r + c + 1] = (int)tot;
        }
    }
    free(nptr);
    free(nidx);
    return tot;
}

void orc_pattern_fill(int nd, int ne, const int *topo, const int *etype, const int *free_map,
                      int n, const int *col_ptr, int *row_idx) {
    int nfree = n / 3, *nptr, *nidx;
    node_adjacency(nd, ne, topo, etype, free_map, nfree, &nptr, &nidx);
    for (int r = 0; r < nfree; ++r)
        for (int c = 0; c < 3; ++c) {
            int p = col_ptr[3 * r + c];
            for (int k = nptr[r]; k < nptr[r + 1]; ++k)
                for (int cc = 0; cc < 3; ++cc) row_idx[p++] = 3 * nidx[k] + cc;
        }
    free(nptr);
    free(nidx);
}

/* ---------------------------------------------------------------- fill -- */

/* Element DOFs and coordinates (assamble_stiffness::build_ele_dofs_coors,
 * src/assemble.cpp:153-174). */
static int ele_gather(const double *xyz, const int *topo, const int *etype, const int *free_map,
                      int e, int *dofs, double *X) {
    int npe = npe_of(etype[e]);
    for (int a = 0; a < npe; ++a) {
        int node = topo[8 * e + a] - 1;
        int f = free_map[node];
        /* 3*(-1)+c is negative for a fixed node, as in the reference */
        dofs[3 * a] = 3 * f;
        dofs[3 * a + 1] = 3 * f + 1;
        dofs[3 * a + 2] = 3 * f + 2;
        for (int c = 0; c < 3; ++c) X[3 * a + c] = xyz[3 * node + c];
    }
    return npe;
}

/* Scatter-add with the reference's linear slot search (src/assemble.cpp:128-148):
 * column jj = dofs[mm], row ii = dofs[nn], value Ke(mm, nn). */
static void scatter(int m, const int *dofs, const double *Ke, const int *col_ptr,
                    const int *row_idx, double *val) {
    for (int mm = 0; mm < m; ++mm) {
        int jj = dofs[mm];
        if (jj < 0) continue;
        for (int nn = 0; nn < m; ++nn) {
            int ii = dofs[nn];
            if (ii < 0) continue;
            int t = col_ptr[jj];
            while (row_idx[t] < ii) ++t;
            val[t] += Ke[mm * m + nn];
        }
    }
}

void orc_fill(int nd, const double *xyz, int ne, const int *topo, const int *etype,
              const int *free_map, const double *E_elem, double E0, double nu,
              const int *col_ptr, const int *row_idx, double *val) {
    (void)nd;
    double Ke[576], X[24];
    int dofs[24];
    for (int e = 0; e < ne; ++e) {
        int npe = ele_gather(xyz, topo, etype, free_map, e, dofs, X);
        double E = E_elem ? E_elem[e] : E0;
        if (npe == 8)
            orc_c3d8_ke(X, E, nu, Ke);
        else
            orc_c3d4_ke(X, E, nu, Ke);
        scatter(3 * npe, dofs, Ke, col_ptr, row_idx, val);
    }
}

void orc_nl_fill(int nd, const double *xyz, int ne, const int *topo, const int *etype,
                 const int *free_map, const double *E_elem, double E0, double nu,
                 const double *u, const int *col_ptr, const int *row_idx, double *val,
                 double *f_int) {
    (void)nd;
    double Ke[576], X[24], ue[24], fe[24];
    int dofs[24];
    int n = 0;
    /* n is not passed; val length is col_ptr[n].  Zero what the reference
     * zeroes: K (nl_assemble.cpp:98) and f_int (cae.cpp:222). */
    for (int i = 0; i < nd; ++i)
        if (free_map[i] >= 0) n += 3;
    memset(val, 0, sizeof(double) * (size_t)col_ptr[n]);
    memset(f_int, 0, sizeof(double) * (size_t)n);
    for (int e = 0; e < ne; ++e) {
        int npe = ele_gather(xyz, topo, etype, free_map, e, dofs, X);
        /* item_ele_dis (3 x npe), zero on constrained DOFs (nl_assemble.cpp:118-134) */
        for (int a = 0; a < npe; ++a)
            for (int c = 0; c < 3; ++c) ue[c * npe + a] = dofs[3 * a + c] >= 0 ? u[dofs[3 * a + c]] : 0.0;
        double E = E_elem ? E_elem[e] : E0;
        if (npe == 8)
            orc_c3d8_nl(X, ue, E, nu, Ke, fe);
        else
            orc_c3d4_nl(X, ue, E, nu, Ke, fe);
        for (int mm = 0; mm < 3 * npe; ++mm)
            if (dofs[mm] >= 0) f_int[dofs[mm]] += fe[mm];
        scatter(3 * npe, dofs, Ke, col_ptr, row_idx, val);
    }
}

/* --------------------------------------------------------------- solve -- */

void orc_spmv(int n, const int *col_ptr, const int *row_idx, const double *val, const double *x,
              double *y) {
    /* K symmetric: row i of K equals column i. */
    for (int i = 0; i < n; ++i) {
        double s = 0;
        for (int k = col_ptr[i]; k < col_ptr[i + 1]; ++k) s += val[k] * x[row_idx[k]];
        y[i] = s;
    }
}

static double dot(int n, const double *a, const double *b) {
    double s = 0;
    for (int i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

int orc_pcg(int n, const int *col_ptr, const int *row_idx, const double *val, const double *f,
            double *u, double rtol, int max_iter, int *iters, double *rel_res) {
    double *r = (double *)malloc(sizeof(double) * (size_t)n);
    double *z = (double *)malloc(sizeof(double) * (size_t)n);
    double *p = (double *)malloc(sizeof(double) * (size_t)n);
    double *q = (double *)malloc(sizeof(double) * (size_t)n);
    double *dinv = (double *)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; ++i) {
        double d = 0;
        for (int k = col_ptr[i]; k < col_ptr[i + 1]; ++k)
            if (row_idx[k] == i) d = val[k];
        dinv[i] = d != 0 ? 1.0 / d : 1.0;
        u[i] = 0;
    }
    double fn = sqrt(dot(n, f, f));
    int it = 0, status = 1;
    double rr = 0;
    if (fn == 0) {
        *iters = 0;
        *rel_res = 0;
        free(r); free(z); free(p); free(q); free(dinv);
        return 0;
    }
    /* restarted from the recomputed residual until it meets rtol */
    while (it < max_iter) {
        orc_spmv(n, col_ptr, row_idx, val, u, q);
        for (int i = 0; i < n; ++i) r[i] = f[i] - q[i];
        rr = sqrt(dot(n, r, r));
        if (rr <= rtol * fn) {
            status = 0;
            break;
        }
        for (int i = 0; i < n; ++i) z[i] = dinv[i] * r[i], p[i] = z[i];
        double rz = dot(n, r, z);
        while (it < max_iter) {
            orc_spmv(n, col_ptr, row_idx, val, p, q);
            double pq = dot(n, p, q);
            if (!(pq > 0)) {
                status = 2; /* breakdown: K not positive definite */
                goto done;
            }
            double alpha = rz / pq;
            for (int i = 0; i < n; ++i) u[i] += alpha * p[i], r[i] -= alpha * q[i];
            ++it;
            if (sqrt(dot(n, r, r)) <= 0.5 * rtol * fn) break;
            for (int i = 0; i < n; ++i) z[i] = dinv[i] * r[i];
            double rz2 = dot(n, r, z);
            double beta = rz2 / rz;
            rz = rz2;
            for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
        }
    }
done:
    orc_spmv(n, col_ptr, row_idx, val, u, q);
    for (int i = 0; i < n; ++i) r[i] = f[i] - q[i];
    rr = sqrt(dot(n, r, r));
    *iters = it;
    *rel_res = rr / fn;
    if (status != 2 && rr <= rtol * fn) status = 0;
    free(r); free(z); free(p); free(q); free(dinv);
    return status;
}

void orc_full_displacement(int nd, const int *free_map, const double *u, double *u_full) {
    for (int i = 0; i < nd; ++i) {
        int r = free_map[i];
        for (int c = 0; c < 3; ++c) u_full[3 * i + c] = r >= 0 ? u[3 * r + c] : 0.0;
    }
}
