// Test infrastructure only: a C-callable harness around the reference's OWN
// hot-path code (compiled from the reference tree by oracle/Makefile into
// oracle/_ref/libofea_ref.so).  Nothing in the product links this file.
//
// It drives, unchanged, the reference functions the GPU path replaces:
//   ReadInfo::read_*            src/data2cae.cpp:18-446        (.inp reader)
//   set_BCs::build_free_index   src/set_bc.cpp:20-43           (DOF numbering)
//   set_BCs::build_single_load  src/set_bc.cpp:46-77           (load vector)
//   assamble_stiffness::build_CSR / fill_CSR_sparse_mat  src/assemble.cpp:19-151
//   assamble_nl_stiffness::build_CSR / fill_CSR_sparse_mat src/nl_assemble.cpp:18-166
//   solution_api(..., "SuperLU_func")  src/linear_solution.cpp:17-64
//   element routines  src/Elements/C3D8_Gauss.cpp, src/Elements/C3D4_hammer.cpp
//
// The one loop written here is ref_model_fill_per_element(): the reference has
// one material per element TYPE (src/data_managrment.cpp:20-26), so for
// per-element Young's modulus it repeats fill_CSR_sparse_mat's loop
// (src/assemble.cpp:106-149) calling set_matrial()+build_cons_mat() before each
// element, so every element matrix still comes from the reference's routines.
#include <chrono>
#include <cstdio>
#include <string>
#include <vector>

#include "include/assemble.h"
#include "include/data2cae.h"
#include "include/data_management.h"
#include "include/linear_solution.h"
#include "include/nl_assemble.h"
#include "include/post_process.h"
#include "include/set_bcs.h"

#include <Eigen/IterativeLinearSolvers>
#include <Eigen/SparseCore>

using namespace CAE;

namespace {
// Eigen CG + IC solver of the scale oracle on a model's K.  K is symmetric,
// so the reference's CSC arrays are read as CSR, which lets Eigen's SpMV use
// OpenMP threads (the IC triangular solves are serial).
struct CgIc {
    typedef Eigen::SparseMatrix<double, Eigen::RowMajor, int> SpR;
    Eigen::Map<const SpR> K;
    Eigen::ConjugateGradient<SpR, Eigen::Lower | Eigen::Upper,
                             Eigen::IncompleteCholesky<double, Eigen::Lower, Eigen::NaturalOrdering<int>>>
        cg;
    CgIc(int n, assamble_stiffness &A)
        : K(n, n, (int)A.nz_val_.size(), A.col_idx_.data(), A.row_idx_.data(), A.nz_val_.data()) {}
};

struct RefModel {
    data_management data;
    elastic_mat mat{};
    assamble_stiffness lin;
    assamble_nl_stiffness nl;
    std::vector<double> E_elem;  // empty -> one material for all elements
    double t_csr = 0, t_fill = 0, t_solve = 0;
    CgIc *cgic = nullptr;
    ~RefModel() { delete cgic; }
};

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void register_types(RefModel *m) {
    for (int t : m->data.ele_class_) {
        std::string name = (t == 0) ? "C3D4" : "C3D8";
        m->data.add_ele(name);
    }
}
}  // namespace

extern "C" {

// Build a model from arrays.  topo: ne x 8, 1-based node ids (tets use the
// first 4); etype: 0 = C3D4, 1 = C3D8 (ELE_TYPES, data_management.h:76);
// fix_ids: 1-based fixed node ids (whole-node ENCASTRE); E_elem may be NULL.
void *ref_model_create(int nd, const double *xyz, int ne, const int *topo, const int *etype,
                       const double *E_elem, double E0, double nu, int nfix, const int *fix_ids) {
    RefModel *m = new RefModel();
    data_management &d = m->data;
    d.nd_ = nd;
    d.ne_ = ne;
    d.coords_.assign(nd, std::vector<double>(3));
    for (int i = 0; i < nd; ++i)
        for (int c = 0; c < 3; ++c) d.coords_[i][c] = xyz[3 * i + c];
    d.node_topos_.assign(ne, std::vector<int>(8, 0));
    d.ele_list_idx_.resize(ne);
    for (int e = 0; e < ne; ++e) {
        d.ele_list_idx_[e] = etype[e];
        d.ele_class_.insert(etype[e]);
        int npe = etype[e] == 1 ? 8 : 4;
        for (int a = 0; a < npe; ++a) d.node_topos_[e][a] = topo[8 * e + a];
    }
    register_types(m);
    d.dis_bc_set_.assign(fix_ids, fix_ids + nfix);
    m->mat.young_modulus = E0;
    m->mat.poisson_ratio = nu;
    m->mat.density = 0.0;
    if (E_elem) m->E_elem.assign(E_elem, E_elem + ne);
    set_BCs bcs;
    bcs.build_free_index(d);
    int nfree = d.nd_ - (int)d.dis_bc_set_.size();
    d.single_load_vec_.assign(3 * nfree, 0.0);
    return m;
}

// Parse an Abaqus .inp with the reference reader exactly as
// CAE_process::pre_info does (src/cae.cpp:168-195), then build_free_index and
// build_single_load (src/cae.cpp:200-206).  E/nu override the file's *Elastic
// when override_mat != 0 (the golden CA model has no *Elastic line).
void *ref_model_from_inp(const char *path, int override_mat, double E0, double nu) {
    RefModel *m = new RefModel();
    ReadInfo info{std::string(path)};
    info.read_ele_node_num(m->data);
    info.read_geo_mesh(m->data);
    info.read_load_bcs("Set-load", "Cload", m->data);
    info.read_dis_bcs("Set-fix", m->data);
    m->mat.young_modulus = 0;
    m->mat.poisson_ratio = 0;
    m->mat.density = 0;
    info.read_mat(m->mat);
    if (override_mat) {
        m->mat.young_modulus = E0;
        m->mat.poisson_ratio = nu;
    }
    set_BCs bcs;
    bcs.build_free_index(m->data);
    bcs.build_single_load(m->data);
    return m;
}

void ref_model_destroy(void *h) { delete (RefModel *)h; }

// Sizes and parsed arrays (for checking the product's own .inp reader).
void ref_model_sizes(void *h, int *nd, int *ne, int *nfree_dof) {
    RefModel *m = (RefModel *)h;
    *nd = m->data.nd_;
    *ne = m->data.ne_;
    *nfree_dof = 3 * (m->data.nd_ - (int)m->data.dis_bc_set_.size());
}
void ref_model_mesh(void *h, double *xyz, int *topo, int *etype, int *free_map, double *f,
                    double *E_nu) {
    RefModel *m = (RefModel *)h;
    data_management &d = m->data;
    for (int i = 0; i < d.nd_; ++i)
        for (int c = 0; c < 3; ++c) xyz[3 * i + c] = d.coords_[i][c];
    for (int e = 0; e < d.ne_; ++e) {
        etype[e] = d.ele_list_idx_[e];
        for (int a = 0; a < 8; ++a) topo[8 * e + a] = d.node_topos_[e][a];
    }
    for (int i = 0; i < d.nd_; ++i) free_map[i] = d.resort_free_nodes_[i];
    for (size_t i = 0; i < d.single_load_vec_.size(); ++i) f[i] = d.single_load_vec_[i];
    E_nu[0] = m->mat.young_modulus;
    E_nu[1] = m->mat.poisson_ratio;
}

void ref_model_set_load(void *h, const double *f) {
    RefModel *m = (RefModel *)h;
    for (size_t i = 0; i < m->data.single_load_vec_.size(); ++i) m->data.single_load_vec_[i] = f[i];
}

// build_CSR + fill_CSR_sparse_mat (src/assemble.cpp:19-151).  Returns nnz.
long long ref_model_assemble(void *h) {
    RefModel *m = (RefModel *)h;
    double t0 = now_s();
    m->lin.build_CSR(m->data);
    double t1 = now_s();
    if (m->E_elem.empty()) {
        m->lin.fill_CSR_sparse_mat(m->data, m->mat);
    } else {
        // fill_CSR_sparse_mat's loop with one material per element.
        assamble_stiffness &A = m->lin;
        data_management &d = m->data;
        A.nz_val_.assign(A.num_nz_val_, 0.0);
        std::vector<int> dofs;
        Eigen::MatrixXd xe, Ke;
        for (int e = 0; e < d.ne_; ++e) {
            int map_idx = d.ele_map_list_[d.ele_list_idx_[e]];
            ele_base *ele = d.ele_list_[map_idx];
            int npe = ele->nnode_;
            elastic_mat me = m->mat;
            me.young_modulus = m->E_elem[e];
            ele->set_matrial(me);
            ele->build_cons_mat();
            xe.resize(npe, 3);
            A.build_ele_dofs_coors(dofs, xe, d, e, npe);
            Ke.resize(3 * npe, 3 * npe);
            ele->build_ele_stiff_mat(xe, Ke);
            int nd = (int)dofs.size();
            for (int mm = 0; mm < nd; ++mm) {
                int jj = dofs[mm];
                if (jj < 0) continue;
                for (int nn = 0; nn < nd; ++nn) {
                    int ii = dofs[nn];
                    if (ii < 0) continue;
                    int t = A.col_idx_[jj];
                    while (A.row_idx_[t] < ii) ++t;
                    A.nz_val_[t] += Ke(mm, nn);
                }
            }
        }
    }
    double t2 = now_s();
    m->t_csr = t1 - t0;
    m->t_fill = t2 - t1;
    return (long long)m->lin.num_nz_val_;
}

// CSC arrays of the assembled K (col_ptr n+1, row_idx nnz, val nnz).
void ref_model_get_csc(void *h, int *col_ptr, int *row_idx, double *val) {
    RefModel *m = (RefModel *)h;
    std::copy(m->lin.col_idx_.begin(), m->lin.col_idx_.end(), col_ptr);
    std::copy(m->lin.row_idx_.begin(), m->lin.row_idx_.end(), row_idx);
    std::copy(m->lin.nz_val_.begin(), m->lin.nz_val_.end(), val);
}

// solution_api(..., "SuperLU_func") (src/linear_solution.cpp:19-22) on the
// current load vector; u gets the free-DOF displacement (single_dis_vec_).
int ref_model_solve(void *h, double *u) {
    RefModel *m = (RefModel *)h;
    data_management &d = m->data;
    int n = (int)d.single_load_vec_.size();
    d.single_dis_vec_.assign(n, 0.0);
    // superlu_solver_func solves in place in F (solver_superlu.cpp:160-162);
    // keep the caller-visible load intact.
    std::vector<double> keep = d.single_load_vec_;
    double t0 = now_s();
    bool ok = solution_api(m->lin, d, "SuperLU_func");
    m->t_solve = now_s() - t0;
    d.single_load_vec_ = keep;
    for (int i = 0; i < n; ++i) u[i] = d.single_dis_vec_[i];
    return ok ? 0 : -1;
}

// reset_displacement (src/post_process.cpp:18-39): full 3*nd field.
void ref_model_full_displacement(void *h, double *u_full) {
    RefModel *m = (RefModel *)h;
    simulation_post post;
    post.reset_displacement(m->data);
    for (int i = 0; i < 3 * m->data.nd_; ++i) u_full[i] = m->data.single_full_dis_vec_[i];
}

void ref_model_times(void *h, double *t3) {
    RefModel *m = (RefModel *)h;
    t3[0] = m->t_csr;
    t3[1] = m->t_fill;
    t3[2] = m->t_solve;
}

// Many load cases on one factor, as the reference's reanalysis does:
// solution_api(..., "SuperLU_class") factors K and solves load case 0
// (src/linear_solution.cpp:23-39, superlu_solution_1st keeps L and U), then
// superlu_solution_next re-solves every further load case with that factor
// (src/solver/solver_superlu.cpp:76-94, called so by src/ca_analysis.cpp:164);
// the last call frees the factor.  F and U: nrhs x n, row-major.
int ref_model_solve_multi(void *h, int nrhs, const double *F, double *U) {
    RefModel *m = (RefModel *)h;
    data_management &d = m->data;
    int n = (int)d.single_load_vec_.size();
    if (nrhs < 1) return -1;
    std::vector<double> keep = d.single_load_vec_;
    double t0 = now_s();
    d.single_load_vec_.assign(F, F + n);
    d.single_dis_vec_.assign(n, 0.0);
    bool ok = solution_api(m->lin, d, "SuperLU_class");
    for (int i = 0; i < n; ++i) U[i] = d.single_dis_vec_[i];
    for (int j = 1; j < nrhs && ok; ++j) {
        std::vector<double> b(F + (size_t)j * n, F + (size_t)(j + 1) * n), x(n, 0.0);
        ok = d.item_superlu.superlu_solution_next(b, x, j == nrhs - 1);
        for (int i = 0; i < n; ++i) U[(size_t)j * n + i] = x[i];
    }
    if (nrhs == 1 && ok) {  // free the factor that superlu_solution_1st kept
        std::vector<double> b(n, 0.0), x(n, 0.0);
        d.item_superlu.superlu_solution_next(b, x, true);
    }
    m->t_solve = now_s() - t0;
    d.single_load_vec_ = keep;
    return ok ? 0 : -1;
}

// The scale oracle where a direct factor does not fit in time: the vendored
// Eigen 3.4.0 ConjugateGradient (FP64) with its IncompleteCholesky
// preconditioner (Lin-More modified IC, externals/eigen-3.4.0/Eigen/src/
// IterativeLinearSolvers/IncompleteCholesky.h) on the reference-assembled K,
// in the reference's own node-interleaved numbering (natural ordering: fewer
// iterations than AMD here, 101 against 165 on a 40x10x10 cantilever).
// ref_model_cg_ic_setup factors once; each ref_model_cg_ic_run is one CG
// solve with that factor.

// IC set-up on the current K; returns its seconds, or a negative value.
double ref_model_cg_ic_setup(void *h, int threads) {
    RefModel *m = (RefModel *)h;
    assamble_stiffness &A = m->lin;
    if (A.col_idx_.empty()) return -1.0;
#ifdef _OPENMP
    Eigen::setNbThreads(threads > 0 ? threads : 1);
#else
    (void)threads;
#endif
    const int n = (int)A.col_idx_.size() - 1;
    const double t0 = now_s();
    delete m->cgic;
    m->cgic = new CgIc(n, A);
    m->cgic->cg.compute(m->cgic->K);
    if (m->cgic->cg.info() != Eigen::Success) return -2.0;
    return now_s() - t0;
}

// One CG solve with the factor of ref_model_cg_ic_setup, started from u:
// stops at ||f - K u|| <= tol ||f|| (Eigen's recursive residual) or after
// maxit iterations.  out[0..3] = iterations, Eigen's residual estimate, the
// FP64 true relative residual, CG seconds.
int ref_model_cg_ic_run(void *h, const double *f, double *u, double tol, int maxit, double *out) {
    RefModel *m = (RefModel *)h;
    CgIc *s = m->cgic;
    if (!s) return -1;
    const int n = (int)s->K.rows();
    Eigen::Map<const Eigen::VectorXd> b(f, n);
    Eigen::Map<Eigen::VectorXd> x(u, n);
    s->cg.setTolerance(tol);
    s->cg.setMaxIterations(maxit);
    const double t0 = now_s();
    Eigen::VectorXd x0 = x;
    x = s->cg.solveWithGuess(b, x0);
    const double t1 = now_s();
    Eigen::VectorXd r = b - s->K * x;
    out[0] = (double)s->cg.iterations();
    out[1] = s->cg.error();
    out[2] = r.norm() / b.norm();
    out[3] = t1 - t0;
    return 0;
}

// Geometric-nonlinear tangent: assamble_nl_stiffness::build_CSR (once) +
// fill_CSR_sparse_mat(u) (src/nl_assemble.cpp:18-166).  f_int accumulates
// into a zeroed vector as implict_analysis does (src/cae.cpp:222-223).
long long ref_model_nl_assemble(void *h, const double *u, double *f_int) {
    RefModel *m = (RefModel *)h;
    data_management &d = m->data;
    int n = (int)d.single_load_vec_.size();
    if (m->nl.col_idx.empty()) m->nl.build_CSR(d);
    std::vector<double> uu(u, u + n), fi(n, 0.0);
    if (m->E_elem.empty()) {
        m->nl.fill_CSR_sparse_mat(d, m->mat, uu, fi);
    } else {
        // nl fill_CSR_sparse_mat's loop (src/nl_assemble.cpp:97-164) with one
        // material per element, element routines still the reference's.
        assamble_nl_stiffness &A = m->nl;
        A.nz_val.assign(A.num_nz_val, 0.0);
        std::vector<int> dofs;
        Eigen::MatrixXd xe, ue, Ke, fe;
        for (int e = 0; e < d.ne_; ++e) {
            int map_idx = d.ele_map_list_[d.ele_list_idx_[e]];
            ele_base *ele = d.ele_list_[map_idx];
            int npe = ele->nnode_;
            elastic_mat me = m->mat;
            me.young_modulus = m->E_elem[e];
            ele->set_matrial(me);
            ele->build_cons_mat();
            xe.resize(npe, 3);
            A.build_ele_dofs_coors(dofs, xe, d, e, npe);
            ue.setZero(3, npe);
            for (int a = 0; a < npe; ++a)
                for (int c = 0; c < 3; ++c)
                    if (dofs[3 * a + c] >= 0) ue(c, a) = uu[dofs[3 * a + c]];
            Ke.resize(3 * npe, 3 * npe);
            fe.resize(3 * npe, 1);
            ele->build_ele_nl_stiff_mat(xe, ue, Ke, fe);
            int ndf = (int)dofs.size();
            for (int mm = 0; mm < ndf; ++mm) {
                int jj = dofs[mm];
                if (jj < 0) continue;
                fi[jj] += fe(mm, 0);
                for (int nn = 0; nn < ndf; ++nn) {
                    int ii = dofs[nn];
                    if (ii < 0) continue;
                    int t = A.col_idx[jj];
                    while (A.row_idx[t] < ii) ++t;
                    A.nz_val[t] += Ke(mm, nn);
                }
            }
        }
    }
    for (int i = 0; i < n; ++i) f_int[i] = fi[i];
    return (long long)m->nl.num_nz_val;
}
void ref_model_nl_get_csc(void *h, int *col_ptr, int *row_idx, double *val) {
    RefModel *m = (RefModel *)h;
    std::copy(m->nl.col_idx.begin(), m->nl.col_idx.end(), col_ptr);
    std::copy(m->nl.row_idx.begin(), m->nl.row_idx.end(), row_idx);
    std::copy(m->nl.nz_val.begin(), m->nl.nz_val.end(), val);
}
// solution_nl_api(..., "SuperLU_func") (src/linear_solution.cpp:66-74).
int ref_model_nl_solve(void *h, const double *b, double *x) {
    RefModel *m = (RefModel *)h;
    int n = (int)m->data.single_load_vec_.size();
    std::vector<double> bb(b, b + n), xx(n, 0.0);
    bool ok = solution_nl_api(m->nl, m->data, bb, xx, "SuperLU_func");
    for (int i = 0; i < n; ++i) x[i] = xx[i];
    return ok ? 0 : -1;
}

// Element routines, called directly.  type 0 = C3D4 (4 nodes), 1 = C3D8 (8).
// coords: npe x 3 row-major.  Ke: (3 npe)^2 row-major.
void ref_element_ke(int type, const double *coords, double E, double nu, double *Ke) {
    std::string name = type == 1 ? "C3D8" : "C3D4";
    ele_base *ele = GetFactory<ele_baseFactory>::instance()->create_class(name);
    elastic_mat mat{E, nu, 0.0};
    ele->set_matrial(mat);
    ele->build_cons_mat();
    int npe = ele->nnode_;
    Eigen::MatrixXd xe(npe, 3), K(3 * npe, 3 * npe);
    for (int a = 0; a < npe; ++a)
        for (int c = 0; c < 3; ++c) xe(a, c) = coords[3 * a + c];
    ele->build_ele_stiff_mat(xe, K);
    for (int i = 0; i < 3 * npe; ++i)
        for (int j = 0; j < 3 * npe; ++j) Ke[i * 3 * npe + j] = K(i, j);
    delete ele;
}
// u_el: 3 x npe (row c = component, column a = node), as nl_assemble gathers it.
void ref_element_nl(int type, const double *coords, const double *u_el, double E, double nu,
                    double *Ke, double *fint) {
    std::string name = type == 1 ? "C3D8" : "C3D4";
    ele_base *ele = GetFactory<ele_baseFactory>::instance()->create_class(name);
    elastic_mat mat{E, nu, 0.0};
    ele->set_matrial(mat);
    ele->build_cons_mat();
    int npe = ele->nnode_;
    Eigen::MatrixXd xe(npe, 3), ue(3, npe), K(3 * npe, 3 * npe), f(3 * npe, 1);
    for (int a = 0; a < npe; ++a)
        for (int c = 0; c < 3; ++c) {
            xe(a, c) = coords[3 * a + c];
            ue(c, a) = u_el[c * npe + a];
        }
    ele->build_ele_nl_stiff_mat(xe, ue, K, f);
    for (int i = 0; i < 3 * npe; ++i) {
        fint[i] = f(i, 0);
        for (int j = 0; j < 3 * npe; ++j) Ke[i * 3 * npe + j] = K(i, j);
    }
    delete ele;
}

}  // extern "C"
