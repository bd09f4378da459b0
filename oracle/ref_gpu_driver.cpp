// Test infrastructure only: the reference's own analysis flow with the GPU
// solver bound in through openfea_b200/integration/ofea_solution_api.cpp,
// built by oracle/Makefile into oracle/_ref/ref_gpu_driver from the
// reference's sources.  It checks that binding end to end: the reference
// reads the .inp, numbers the DOFs, assembles K on the CPU, hands K to
// solution_api(..., solver) exactly as CAE_process::implict_analysis does
// (src/cae.cpp:197-275), then recovers stress and writes its VTK
// (src/cae.cpp:277-286).  The one thing restated here is that driver's
// sequence of calls: the reference hard-codes its solver string
// ("Pardiso_class", src/cae.cpp:232,274), which this driver takes from the
// command line instead.
//
//   ref_gpu_driver -i model.inp -o out.vtk -solver GPU_PCG [-nl] [-gpu-assembly] [-E 2.1e5 -nu 0.3]
//
// -E / -nu override the file's *Elastic (the shipped CA sample has none).
// -gpu-assembly runs the linear analysis through gpu_implicit_analysis (the
// binding that also moves build_CSR + fill_CSR_sparse_mat to the device).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "include/assemble.h"
#include "include/data2cae.h"
#include "include/data2vtk.h"
#include "include/data_management.h"
#include "include/linear_solution.h"
#include "include/nl_assemble.h"
#include "include/post_process.h"
#include "include/set_bcs.h"

namespace CAE {
bool gpu_implicit_analysis(data_management &d, elastic_mat &mat, string solver_type);
}

using namespace CAE;

int main(int argc, char **argv) {
    std::string in, out, solver = "GPU_PCG";
    bool nl = false, override_mat = false, gpu_assembly = false;
    double E = 0, nu = 0;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        if (a == "-i" && i + 1 < argc) in = argv[++i];
        else if (a == "-o" && i + 1 < argc) out = argv[++i];
        else if (a == "-solver" && i + 1 < argc) solver = argv[++i];
        else if (a == "-nl") nl = true;
        else if (a == "-gpu-assembly") gpu_assembly = true;
        else if (a == "-E" && i + 1 < argc) E = std::atof(argv[++i]), override_mat = true;
        else if (a == "-nu" && i + 1 < argc) nu = std::atof(argv[++i]), override_mat = true;
        else {
            std::fprintf(stderr, "usage: %s -i model.inp -o out.vtk -solver NAME [-nl] [-E e -nu v]\n", argv[0]);
            return 2;
        }
    }
    if (in.empty() || out.empty()) return 2;
    data_management data;
    elastic_mat mat{};
    // CAE_process::pre_info (src/cae.cpp:168-195)
    ReadInfo info(in);
    info.read_ele_node_num(data);
    info.read_geo_mesh(data);
    info.read_load_bcs("Set-load", "Cload", data);
    info.read_dis_bcs("Set-fix", data);
    info.read_mat(mat);
    if (override_mat) {
        mat.young_modulus = E;
        mat.poisson_ratio = nu;
    }
    data.NLFEA = nl;
    // CAE_process::implict_analysis (src/cae.cpp:197-286)
    set_BCs bcs;
    bcs.build_free_index(data);
    bcs.build_single_load(data);
    const int n = 3 * (data.nd_ - (int)data.dis_bc_set_.size());
    if (nl) {
        assamble_nl_stiffness assam;
        assam.build_CSR(data);
        std::vector<double> u(n, 0.0), fint(n, 0.0), res(n, 0.0);
        double res_norm = 1.0;
        int loop = 0;
        while (res_norm > data.res_lmit && loop < 100) {
            std::fill(fint.begin(), fint.end(), 0.0);
            assam.fill_CSR_sparse_mat(data, mat, u, fint);
            for (int i = 0; i < n; ++i) res[i] = data.single_load_vec_[i] - fint[i];
            std::vector<double> du(n, 0.0);
            if (!solution_nl_api(assam, data, res, du, solver)) return 1;
            res_norm = 0.0;
            for (int i = 0; i < n; ++i) {
                u[i] += du[i];
                res_norm += res[i] * res[i];
            }
            res_norm = std::sqrt(res_norm) / n;
            ++loop;
            std::printf("newton %d residual %.6e\n", loop, res_norm);
        }
        data.single_dis_vec_ = u;
    } else if (gpu_assembly) {
        if (!gpu_implicit_analysis(data, mat, solver)) return 1;
    } else {
        assamble_stiffness assam;
        assam.build_CSR(data);
        assam.fill_CSR_sparse_mat(data, mat);
        data.single_dis_vec_.resize(n);
        if (!solution_api(assam, data, solver)) return 1;
    }
    simulation_post post;
    post.reset_displacement(data);
    post.get_cauchy_stress_3d(data);
    data_process output;
    output.export_dis_2_vtk(data, out, 1.0);
    std::printf("solved n=%d with %s -> %s\n", n, solver.c_str(), out.c_str());
    return 0;
}
