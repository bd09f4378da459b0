/* ofea_oracle.h - CPU restatement of OpenFEA's implicit-static hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker of the GPU path: it is
 * loaded by tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline
 * leg, never by the product.  It is pinned against the reference's own code
 * compiled into oracle/_ref/libofea_ref.so and against the reference's golden
 * output sample_model/CA/cadcae_o.vtk (tests/test_oracle.py).
 *
 * Conventions follow the reference (citations are paths in the OpenFEA tree):
 *   - node ids in `topo` are 1-based, 8 slots per element (C3D4 uses the first
 *     4), like data_management::node_topos_ (src/include/data_management.h:49);
 *   - etype 0 = C3D4, 1 = C3D8 (ELE_TYPES, src/include/data_management.h:76);
 *   - free_map[node] = free-node index or -1 (resort_free_nodes_,
 *     src/set_bc.cpp:20-43); DOF = 3*free_map[node] + component;
 *   - K is stored as the reference stores it: compressed columns (col_ptr n+1,
 *     row_idx nnz sorted ascending per column, val nnz) - src/assemble.cpp:54-75.
 */
#ifndef OFEA_ORACLE_H
#define OFEA_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* set_BCs::build_free_index (src/set_bc.cpp:20-43).  Returns the number of
 * free nodes (nd - nfix, as the reference counts them), or -1 when fix_ids is
 * empty, has duplicates or ids outside 1..nd (inputs on which the reference's
 * loop is undefined). */
int orc_build_free_index(int nd, int nfix, const int *fix_ids, int *free_map);

/* Isotropic constitutive matrix, 6x6 row-major, strain order
 * [xx, yy, zz, xy, yz, zx] (hex_ele_elastic::build_cons_mat, src/Elements/C3D8.cpp:21-35). */
void orc_cons_mat(double E, double nu, double D[36]);

/* Element stiffness, reference dense form.  coords npe x 3 row-major,
 * Ke (3 npe)^2 row-major, DOF order 3*node + component.
 * C3D8: 2x2x2 Gauss (src/Elements/C3D8_Gauss.cpp:19-107).
 * C3D4: one-point rule, weight 1/6, signed det (src/Elements/C3D4_hammer.cpp:20-72).
 * Returns the (last) Jacobian determinant. */
double orc_c3d8_ke(const double *coords, double E, double nu, double *Ke);
double orc_c3d4_ke(const double *coords, double E, double nu, double *Ke);

/* Total-Lagrangian tangent K_T = B_L^T D B_L + B_NL^T SIG B_NL and internal
 * force f = B_L^T S, u_el 3 x npe (component-major, like nl_assemble's
 * item_ele_dis, src/nl_assemble.cpp:118-134).
 * C3D8: src/Elements/C3D8_Gauss.cpp:110-266; C3D4: src/Elements/C3D4_hammer.cpp:75-182. */
void orc_c3d8_nl(const double *coords, const double *u_el, double E, double nu, double *Ke,
                 double *fint);
void orc_c3d4_nl(const double *coords, const double *u_el, double E, double nu, double *Ke,
                 double *fint);

/* assamble_stiffness::build_CSR (src/assemble.cpp:19-77), in two calls:
 * count fills col_ptr (n+1) and returns nnz; fill writes row_idx (nnz). */
long long orc_pattern_count(int nd, int ne, const int *topo, const int *etype,
                            const int *free_map, int n, int *col_ptr);
void orc_pattern_fill(int nd, int ne, const int *topo, const int *etype, const int *free_map,
                      int n, const int *col_ptr, int *row_idx);

/* assamble_stiffness::fill_CSR_sparse_mat (src/assemble.cpp:95-151), element
 * order and slot search as the reference.  E_elem may be NULL (E0 for all). */
void orc_fill(int nd, const double *xyz, int ne, const int *topo, const int *etype,
              const int *free_map, const double *E_elem, double E0, double nu,
              const int *col_ptr, const int *row_idx, double *val);

/* assamble_nl_stiffness::fill_CSR_sparse_mat (src/nl_assemble.cpp:94-166):
 * zeroes val, accumulates K_T and f_int (f_int is zeroed here, as
 * implict_analysis does before each call, src/cae.cpp:222). */
void orc_nl_fill(int nd, const double *xyz, int ne, const int *topo, const int *etype,
                 const int *free_map, const double *E_elem, double E0, double nu,
                 const double *u, const int *col_ptr, const int *row_idx, double *val,
                 double *f_int);

/* y = K x for the symmetric K stored by columns (the reference treats its CSC
 * arrays as CSR when handing them to the solvers; K is symmetric). */
void orc_spmv(int n, const int *col_ptr, const int *row_idx, const double *val, const double *x,
              double *y);

/* Jacobi-preconditioned CG in FP64 on K (symmetric), stopping when
 * ||f - K u||_2 / ||f||_2 <= rtol (recomputed residual).  Returns 0 on
 * convergence, 1 when max_iter is reached, 2 on breakdown (p.Kp <= 0).  Stand-in for the reference's direct solvers
 * (src/linear_solution.cpp:17-64) at sizes where LU is slow; the pinned
 * solution at small sizes is the reference's own SuperLU path. */
int orc_pcg(int n, const int *col_ptr, const int *row_idx, const double *val, const double *f,
            double *u, double rtol, int max_iter, int *iters, double *rel_res);

/* simulation_post::reset_displacement (src/post_process.cpp:18-39). */
void orc_full_displacement(int nd, const int *free_map, const double *u, double *u_full);

#ifdef __cplusplus
}
#endif
#endif
