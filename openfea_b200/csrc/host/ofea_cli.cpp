// ofea_cli: OpenFEA's implicit-static driver (CAE_process::Init / Solve /
// implict_analysis, src/cae.cpp:18-301) with the assembly and the linear
// solves running on the GPU through the C ABI.
//
//   ofea_cli -i model.inp [-o out.vtk] [-imp] [-nl] [-solver GPU_PCG|GPU_MIXED|GPU_LEARNED]
//            [-weights gnn.bin] [-save-weights gnn.bin] [-rtol 1e-8] [-E <Young> -nu <Poisson>]
//            [-ca CA_info.txt -mesh-m mesh_m.inp [-nbasis 4] [-o-ca out_ca.vtk]]
//            [-stress reference|cauchy|none]
//
// The VTK carries the nodal stress fields S_xx .. S_Mises as the reference's
// driver writes them (get_cauchy_stress_3d, src/cae.cpp:286-290): by default
// its own numbers (for C3D4 the engineering strain it labels stress, for C3D8
// zero); -stress cauchy writes the Cauchy stress instead, -stress none no
// fields.
//
// -ca runs the combined-approximations reanalysis after the linear analysis
// (CAE_process::CA_pre_process + CA_ReAnalysis, src/cae.cpp:303-375): the
// change file's deleted elements get E = 0 and its coordinates are used for
// the modified model, which is assembled as a second context; the CA
// solution goes to the modified model's nodes (mesh_m.inp) and its VTK.
//
// GPU_LEARNED loads the learned stage's weights from -weights, or trains it
// on the model's own K (plain-PCG residuals of a seeded random load) when no
// file is given; -save-weights keeps the trained weights for later runs.
//
// -E/-nu override the file's material (the reference's code_test cases set it
// in code for models without *Elastic, src/main.cpp:121-135).  The output VTK
// name defaults to the input name with .vtk (src/cae.cpp:108-110).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../../include/ofea_gpu.h"
#include "../../../include/ofea_host.h"

namespace {

double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int die(const char *what, int rc) {
    std::fprintf(stderr, "ofea_cli: %s failed: %s (%s)\n", what, ofea_status_string(rc), ofea_last_error());
    return 2;
}

// The CA reanalysis of the analysed model (ctx, u) from the change file:
// the modified model on the same elements and numbering (deleted elements
// E = 0, the change file's coordinates), assembled as a second context.
int reanalyse(const std::string &info, const std::string &mesh_m, const std::string &out_ca, int nbasis,
              ofea_ctx *ctx, int nd, int ne, const std::vector<int> &topo, const std::vector<int> &etype,
              double E, double nu, const std::vector<int> &fm, const std::vector<double> &f,
              const std::vector<double> &u, const ofea_solve_opts &opts) {
    int rc, ndc = 0, nc = 0;
    if ((rc = ofea_ca_info_read(info.c_str(), &ndc, &nc, nullptr, nullptr, nullptr, nullptr, nullptr)))
        return die("reading the CA change file", rc);
    if (ndc != nd) {
        std::fprintf(stderr, "ofea_cli: the change file has %d nodes, the model %d\n", ndc, nd);
        return 2;
    }
    std::vector<double> xyz_m(3L * nd);
    std::vector<int> kind(nc), cet(nc), ctopo(8L * nc), node_map(nd);
    ofea_ca_info_read(info.c_str(), &ndc, &nc, xyz_m.data(), kind.data(), cet.data(), ctopo.data(),
                      node_map.data());
    std::printf("the number node set after modifying is: %d\nthe number of changed element is: %d\n", nd, nc);
    // each changed element among the model's elements (same node set)
    std::map<std::vector<int>, int> by_nodes;
    for (int e = 0; e < ne; ++e) {
        std::vector<int> k;
        for (int j = 0; j < 8; ++j)
            if (topo[8L * e + j] > 0) k.push_back(topo[8L * e + j] - 1);
        std::sort(k.begin(), k.end());
        by_nodes.emplace(k, e);
    }
    std::vector<double> E_m(ne, E);
    for (int c = 0; c < nc; ++c) {
        std::vector<int> k;
        for (int j = 0; j < 8; ++j)
            if (ctopo[8L * c + j] >= 0) k.push_back(ctopo[8L * c + j]);
        std::sort(k.begin(), k.end());
        auto it = by_nodes.find(k);
        if (it == by_nodes.end()) {
            std::fprintf(stderr, "ofea_cli: changed element %d is not an element of the model (added elements "
                                 "must be in the model's mesh)\n", c);
            return 2;
        }
        if (kind[c] == 0) E_m[it->second] = 0.0;
    }
    ofea_ctx *cm = nullptr;
    if ((rc = ofea_ctx_create(&cm, 0))) return die("ofea_ctx_create", rc);
    if ((rc = ofea_mesh_upload(cm, nd, xyz_m.data(), ne, topo.data(), etype.data(), E_m.data(), E, nu, fm.data())))
        return die("ofea_mesh_upload (modified model)", rc);
    int n_chk;
    long long nnz;
    if ((rc = ofea_assemble_pattern(cm, &n_chk, &nnz))) return die("ofea_assemble_pattern (modified model)", rc);
    if ((rc = ofea_assemble_linear(cm))) return die("ofea_assemble_linear (modified model)", rc);
    std::vector<double> uca(f.size());
    ofea_ca_stats cs{};
    if ((rc = ofea_ca_reanalysis(ctx, cm, f.data(), u.data(), nbasis, &opts, uca.data(), &cs)))
        return die("ofea_ca_reanalysis", rc);
    std::printf("CA reanalysis: %d of %d basis vectors, %d solver iterations, relative residual %.3e, %.4f s\n",
                cs.basis_used, cs.basis_requested, cs.solve_iterations, cs.rel_residual, cs.seconds);
    ofea_ctx_destroy(cm);
    // reset_ca_displacement (src/post_process.cpp:42-75): onto the modified model's nodes
    std::vector<double> uf(3L * nd);
    ofea_full_displacement(nd, fm.data(), uca.data(), uf.data());
    ofea_model *mm = nullptr;
    if ((rc = ofea_inp_read(mesh_m.c_str(), &mm))) return die("reading the modified mesh", rc);
    int ndm, nem, nfm, nlm;
    ofea_model_sizes(mm, &ndm, &nem, &nfm, &nlm);
    std::vector<double> xm(3L * ndm);
    std::vector<int> tm(8L * nem), em(nem), fxm(nfm), lm(nlm);
    ofea_model_arrays(mm, xm.data(), tm.data(), em.data(), fxm.data(), lm.data());
    ofea_model_free(mm);
    std::vector<double> un(3L * ndm, 0.0);
    for (int i = 0; i < nd; ++i) {
        const int j = node_map[i];
        if (j < 0) continue;
        if (j >= ndm) {
            std::fprintf(stderr, "ofea_cli: the node map points past the modified mesh's %d nodes\n", ndm);
            return 2;
        }
        for (int c = 0; c < 3; ++c) un[3L * j + c] = uf[3L * i + c];
    }
    if ((rc = ofea_write_vtk(out_ca.c_str(), ndm, xm.data(), nem, tm.data(), em.data(), un.data(), 1.0)))
        return die("writing the CA VTK file", rc);
    return 0;
}

}  // namespace

int main(int argc, char **argv) {
    std::string in, out, solver = "GPU_PCG", weights, save_weights, ca_info, mesh_m, out_ca;
    int nbasis = 4;
    std::string stress = "reference";
    bool nl = false;
    double rtol = 1e-8, E_over = -1, nu_over = -1;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        if (a == "-i" && i + 1 < argc) in = argv[++i];
        else if (a == "-o" && i + 1 < argc) out = argv[++i];
        else if (a == "-nl") nl = true;
        else if (a == "-imp") {}
        else if (a == "-solver" && i + 1 < argc) solver = argv[++i];
        else if (a == "-rtol" && i + 1 < argc) rtol = std::atof(argv[++i]);
        else if (a == "-weights" && i + 1 < argc) weights = argv[++i];
        else if (a == "-save-weights" && i + 1 < argc) save_weights = argv[++i];
        else if (a == "-E" && i + 1 < argc) E_over = std::atof(argv[++i]);
        else if (a == "-nu" && i + 1 < argc) nu_over = std::atof(argv[++i]);
        else if (a == "-ca" && i + 1 < argc) ca_info = argv[++i];
        else if (a == "-mesh-m" && i + 1 < argc) mesh_m = argv[++i];
        else if (a == "-nbasis" && i + 1 < argc) nbasis = std::atoi(argv[++i]);
        else if (a == "-o-ca" && i + 1 < argc) out_ca = argv[++i];
        else if (a == "-stress" && i + 1 < argc) stress = argv[++i];
        else if (argc == 2) in = a;
        else if (a == "-exp" || a == "-sfem" || a == "-re") {
            std::fprintf(stderr, "ofea_cli: %s is not part of the GPU implicit-static path\n", a.c_str());
            return 2;
        }
    }
    if (in.size() < 5 || in.substr(in.size() - 4) != ".inp") {
        std::fprintf(stderr, "Please enter the correct path to the input file ending in .inp\n");
        return 2;
    }
    if (out.empty()) out = in.substr(0, in.size() - 4) + ".vtk";
    if (!ca_info.empty() && (nl || mesh_m.empty())) {
        std::fprintf(stderr, "ofea_cli: -ca needs -mesh-m and the linear analysis (no -nl)\n");
        return 2;
    }
    if (out_ca.empty()) out_ca = in.substr(0, in.size() - 4) + "_ca.vtk";
    if (stress != "reference" && stress != "cauchy" && stress != "none") {
        std::fprintf(stderr, "ofea_cli: -stress must be reference, cauchy or none\n");
        return 2;
    }
    ofea_solve_opts opts;
    ofea_solve_opts_default(&opts);
    opts.rtol = rtol;
    if (solver == "GPU_PCG") opts.method = OFEA_SOLVER_PCG64;
    else if (solver == "GPU_MIXED") opts.method = OFEA_SOLVER_MIXED;
    else if (solver == "GPU_LEARNED") opts.method = OFEA_SOLVER_LEARNED;
    else {
        std::fprintf(stderr, "Please check your flag of solver !!!\n");
        return 2;
    }

    ofea_model *m = nullptr;
    int rc = ofea_inp_read(in.c_str(), &m);
    if (rc) return die("reading the .inp file", rc);
    int nd, ne, nfix, nload;
    ofea_model_sizes(m, &nd, &ne, &nfix, &nload);
    std::vector<double> xyz(3L * nd);
    std::vector<int> topo(8L * ne), etype(ne), fix(nfix), load(nload);
    ofea_model_arrays(m, xyz.data(), topo.data(), etype.data(), fix.data(), load.data());
    double E, nu, rho;
    int has_el, dof;
    double val;
    ofea_model_material(m, &E, &nu, &rho, &has_el);
    ofea_model_cload(m, &dof, &val);
    ofea_model_free(m);
    if (E_over > 0) E = E_over;
    if (nu_over >= 0) nu = nu_over;
    if (!has_el && E_over <= 0) {
        std::fprintf(stderr, "ofea_cli: the model has no *Elastic; pass -E and -nu\n");
        return 2;
    }
    std::printf("the number of element is: %d\nthe number of node is: %d\n", ne, nd);

    std::vector<int> fm(nd);
    int nfree = 0;
    if ((rc = ofea_build_free_index(nd, nfix, fix.data(), fm.data(), &nfree))) return die("build_free_index", rc);
    const int n = 3 * nfree;
    std::vector<double> f(n), u(n, 0.0);
    if ((rc = ofea_build_single_load(nd, fm.data(), nload, load.data(), dof, val, f.data())))
        return die("build_single_load", rc);

    ofea_ctx *ctx = nullptr;
    if ((rc = ofea_ctx_create(&ctx, 0))) return die("ofea_ctx_create", rc);
    double t0 = now();
    if ((rc = ofea_mesh_upload(ctx, nd, xyz.data(), ne, topo.data(), etype.data(), nullptr, E, nu, fm.data())))
        return die("ofea_mesh_upload", rc);
    int n_chk;
    long long nnz;
    if ((rc = ofea_assemble_pattern(ctx, &n_chk, &nnz))) return die("ofea_assemble_pattern", rc);
    std::printf("The CSR index has been built (n = %d, nnz = %lld)\n", n_chk, nnz);
    ofea_solve_stats st{};
    // the learned stage needs weights before its first solve
    auto prepare_learned = [&]() -> int {
        if (opts.method != OFEA_SOLVER_LEARNED) return OFEA_OK;
        int r;
        if (!weights.empty()) {
            if ((r = ofea_learned_load(ctx, weights.c_str()))) return die("ofea_learned_load", r);
        } else {
            ofea_learn_stats ls{};
            if ((r = ofea_learned_train(ctx, nullptr, nullptr, &ls))) return die("ofea_learned_train", r);
            std::printf("learned stage trained: %d samples, %d steps, %.3f s\n", ls.samples, ls.steps, ls.seconds);
            weights = "(trained)";
        }
        if (!save_weights.empty() && (r = ofea_learned_save(ctx, save_weights.c_str())))
            return die("ofea_learned_save", r);
        return OFEA_OK;
    };
    if (!nl) {
        if ((rc = ofea_assemble_linear(ctx))) return die("ofea_assemble_linear", rc);
        if ((rc = prepare_learned())) return rc;
        rc = ofea_solve(ctx, f.data(), u.data(), 1, &opts, &st);
        std::printf("solve: %s, %d iterations, relative residual %.3e, %.4f s on the GPU\n",
                    ofea_status_string(st.status), st.iterations, st.rel_residual, st.seconds);
        if (rc) return die("ofea_solve", rc);
    } else {
        // Newton loop of implict_analysis (src/cae.cpp:209-253), same stopping
        // rule: ||f - f_int||_2 / (3 n_free_nodes) < 1e-6, at most 100 passes.
        std::vector<double> fint(n), r(n), du(n);
        double res = 1.0;
        int loop = 0;
        while (res > 1.0e-6 && loop < 100) {
            if ((rc = ofea_assemble_nl(ctx, u.data(), fint.data()))) return die("ofea_assemble_nl", rc);
            if (loop == 0 && (rc = prepare_learned())) return rc;
            for (int i = 0; i < n; ++i) r[i] = f[i] - fint[i];
            rc = ofea_solve(ctx, r.data(), du.data(), 1, &opts, &st);
            if (rc) return die("ofea_solve", rc);
            res = 0;
            for (int i = 0; i < n; ++i) {
                u[i] += du[i];
                res += r[i] * r[i];
            }
            res = std::sqrt(res) / (3.0 * nfree);
            ++loop;
            std::printf("this is loop %d, and res is %g\n", loop, res);
        }
        std::printf("the loop is over\n");
    }
    std::printf("It took %g s to compute full analysis\n", now() - t0);
    std::vector<double> uf(3L * nd);
    ofea_full_displacement(nd, fm.data(), u.data(), uf.data());
    std::vector<double> node_stress;
    if (stress != "none") {
        node_stress.resize(7L * nd);
        const int mode = stress == "cauchy" ? OFEA_STRESS_CAUCHY : OFEA_STRESS_REFERENCE;
        if ((rc = ofea_stress(ctx, u.data(), mode, nullptr, node_stress.data()))) return die("ofea_stress", rc);
        std::printf("the nodal stress has been smoothed.\n");
    }
    if ((rc = ofea_write_vtk_stress(out.c_str(), nd, xyz.data(), ne, topo.data(), etype.data(), uf.data(), 1.0,
                                    node_stress.empty() ? nullptr : node_stress.data())))
        return die("writing the VTK file", rc);
    if (!ca_info.empty()) {
        if ((rc = reanalyse(ca_info, mesh_m, out_ca, nbasis, ctx, nd, ne, topo, etype, E, nu, fm, f, u, opts)))
            return rc;
    }
    ofea_ctx_destroy(ctx);
    return 0;
}
