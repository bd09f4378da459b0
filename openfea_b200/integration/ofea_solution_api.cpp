// Reference-side binding of the B200 solver into OpenFEA's own solve entry
// points (src/include/linear_solution.h:27-29).  This file is compiled into
// the reference program, next to its src/linear_solution.cpp, against the
// reference's headers and include/ofea_gpu.h, and linked with libofea_gpu.so.
//
// It adds the solver strings "GPU_PCG", "GPU_MIXED" and "GPU_LEARNED" beside
// the reference's "SuperLU_func" / "SuperLU_class" / "Pardiso_func" /
// "Pardiso_class" (src/linear_solution.cpp:19-62).  The reference's CPU
// dispatch is kept under another name by compiling linear_solution.cpp with
//     -Dsolution_api=solution_api_cpu -Dsolution_nl_api=solution_nl_api_cpu
// (or, equivalently, by pasting the two GPU branches below into its if/else
// chains); every other string goes to it unchanged.
//
// The GPU branch receives exactly what the CPU solvers receive: K as the
// assembler's CSC arrays (assamble_stiffness::col_idx_ / row_idx_ / nz_val_,
// or assamble_nl_stiffness::col_idx / row_idx / nz_val for the Newton
// tangent, src/include/assemble.h:41-43), the right-hand side, and the model
// (coords_ and resort_free_nodes_ for the coarse levels' rigid-body modes).
// Like the reference it writes the displacement into single_dis_vec_ (linear)
// or x (Newton increment) and returns false on failure; it never exits.
//
// gpu_implicit_analysis() is the other binding point: it replaces the
// CPU assembly and the solve of CAE_process::implict_analysis together.
//
// Settings (environment, read on first use): OFEA_DEVICE (GPU index, 0),
// OFEA_RTOL (relative FP64 residual, 1e-10: a direct solve's accuracy),
// OFEA_LEARNED_WEIGHTS (weight file for GPU_LEARNED; without it the stage is
// trained on the first matrix it sees).
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "include/linear_solution.h"
#include "ofea_gpu.h"

namespace CAE {

bool solution_api_cpu(assamble_stiffness &item_ass, data_management &item_cae_data, string solver_type);
bool solution_nl_api_cpu(assamble_nl_stiffness &item_ass, data_management &item_cae_data, vector<double> &b,
                         vector<double> &x, string solver_type);

namespace {

int gpu_method(const string &s) {
    if (s == "GPU_PCG") return OFEA_SOLVER_PCG64;
    if (s == "GPU_MIXED") return OFEA_SOLVER_MIXED;
    if (s == "GPU_LEARNED") return OFEA_SOLVER_LEARNED;
    return -1;
}

bool report(int rc, const char *what) {
    if (rc == OFEA_OK) return true;
    std::fprintf(stderr, "%s: %s (%s)\n", what, ofea_status_string(rc), ofea_last_error());
    return false;
}

// One context per host thread, created on first use and kept: later solves
// reuse its device buffers.
ofea_ctx *thread_context() {
    static thread_local ofea_ctx *ctx = nullptr;
    if (!ctx) {
        const char *dev = std::getenv("OFEA_DEVICE");
        if (!report(ofea_ctx_create(&ctx, dev ? std::atoi(dev) : 0), "ofea_ctx_create")) ctx = nullptr;
    }
    return ctx;
}

bool gpu_solve(vector<int> &col_idx, vector<int> &row_idx, vector<double> &nz_val, data_management &d,
               const vector<double> &b, vector<double> &x, int method) {
    ofea_ctx *ctx = thread_context();
    if (!ctx) return false;
    const int n = (int)col_idx.size() - 1;
    if (n <= 0 || (int)b.size() != n) {
        std::fprintf(stderr, "GPU solve: K has %d columns, the right-hand side %zu values\n", n, b.size());
        return false;
    }
    std::vector<double> xyz(3 * (size_t)d.nd_);
    for (int i = 0; i < d.nd_; ++i)
        for (int c = 0; c < 3; ++c) xyz[3 * (size_t)i + c] = d.coords_[i][c];
    if (!report(ofea_matrix_upload_csc(ctx, d.nd_, xyz.data(), d.resort_free_nodes_.data(), n, col_idx.data(),
                                       row_idx.data(), nz_val.data()),
                "ofea_matrix_upload_csc"))
        return false;
    if (method == OFEA_SOLVER_LEARNED) {
        static thread_local bool have_weights = false;
        if (!have_weights) {
            const char *path = std::getenv("OFEA_LEARNED_WEIGHTS");
            int rc = path ? ofea_learned_load(ctx, path) : ofea_learned_train(ctx, nullptr, nullptr, nullptr);
            if (!report(rc, path ? "ofea_learned_load" : "ofea_learned_train")) return false;
            have_weights = true;
        }
    }
    ofea_solve_opts opts;
    ofea_solve_opts_default(&opts);
    opts.method = method;
    const char *rtol = std::getenv("OFEA_RTOL");
    opts.rtol = rtol ? std::atof(rtol) : 1e-10;
    ofea_solve_stats st;
    x.assign(n, 0.0);
    return report(ofea_solve(ctx, b.data(), x.data(), 1, &opts, &st), "ofea_solve");
}

}  // namespace

// The whole linear analysis on the GPU, for CAE_process::implict_analysis
// (src/cae.cpp:259-275): in place of build_CSR + fill_CSR_sparse_mat +
// solution_api, the mesh goes to the device, which builds the pattern,
// assembles K and solves; single_dis_vec_ receives u as before.
bool gpu_implicit_analysis(data_management &d, elastic_mat &mat, string solver_type) {
    const int method = gpu_method(solver_type);
    ofea_ctx *ctx = method < 0 ? nullptr : thread_context();
    if (!ctx) return false;
    std::vector<double> xyz(3 * (size_t)d.nd_);
    for (int i = 0; i < d.nd_; ++i)
        for (int c = 0; c < 3; ++c) xyz[3 * (size_t)i + c] = d.coords_[i][c];
    std::vector<int> topo(8 * (size_t)d.ne_), etype(d.ne_);
    for (int e = 0; e < d.ne_; ++e) {
        etype[e] = d.ele_list_idx_[e];  // ELE_TYPES: 0 C3D4, 1 C3D8
        for (int a = 0; a < 8; ++a) topo[8 * (size_t)e + a] = d.node_topos_[e][a];  // 1-based, as read
    }
    int n = 0;
    long long nnz = 0;
    if (!report(ofea_mesh_upload(ctx, d.nd_, xyz.data(), d.ne_, topo.data(), etype.data(), nullptr,
                                 mat.young_modulus, mat.poisson_ratio, d.resort_free_nodes_.data()),
                "ofea_mesh_upload") ||
        !report(ofea_assemble_pattern(ctx, &n, &nnz), "ofea_assemble_pattern") ||
        !report(ofea_assemble_linear(ctx), "ofea_assemble_linear"))
        return false;
    if (method == OFEA_SOLVER_LEARNED) {
        const char *path = std::getenv("OFEA_LEARNED_WEIGHTS");
        int rc = path ? ofea_learned_load(ctx, path) : ofea_learned_train(ctx, nullptr, nullptr, nullptr);
        if (!report(rc, path ? "ofea_learned_load" : "ofea_learned_train")) return false;
    }
    ofea_solve_opts opts;
    ofea_solve_opts_default(&opts);
    opts.method = method;
    const char *rtol = std::getenv("OFEA_RTOL");
    opts.rtol = rtol ? std::atof(rtol) : 1e-10;
    ofea_solve_stats st;
    d.single_dis_vec_.assign(n, 0.0);
    return report(ofea_solve(ctx, d.single_load_vec_.data(), d.single_dis_vec_.data(), 1, &opts, &st),
                  "ofea_solve");
}

bool solution_api(assamble_stiffness &item_ass, data_management &item_cae_data, string solver_type) {
    const int method = gpu_method(solver_type);
    if (method < 0) return solution_api_cpu(item_ass, item_cae_data, solver_type);
    return gpu_solve(item_ass.col_idx_, item_ass.row_idx_, item_ass.nz_val_, item_cae_data,
                     item_cae_data.single_load_vec_, item_cae_data.single_dis_vec_, method);
}

bool solution_nl_api(assamble_nl_stiffness &item_ass, data_management &item_cae_data, vector<double> &b,
                     vector<double> &x, string solver_type) {
    const int method = gpu_method(solver_type);
    if (method < 0) return solution_nl_api_cpu(item_ass, item_cae_data, b, x, solver_type);
    return gpu_solve(item_ass.col_idx, item_ass.row_idx, item_ass.nz_val, item_cae_data, b, x, method);
}

}  // namespace CAE
