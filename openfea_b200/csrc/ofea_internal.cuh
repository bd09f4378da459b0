// Internal definitions shared by the CUDA translation units of libofea_gpu.
//
// Device data layout (all in HBM, resident for the life of the context):
//   xyz        double[3*nd]            node coordinates
//   topo8      int[8*ne8]              C3D8 connectivity (0-based), elements in caller order
//   topo4      int[4*ne4]              C3D4 connectivity
//   E8, E4     double[ne8], [ne4]      Young's modulus per element
//   free_map   int[nd]                 node -> free index or -1
//   node_of_free int[nfree]            free index -> node
//   inc_ptr    int[nd+1], inc int[..]  node -> incident elements, packed g*8+local, sorted
//              (g = unified element id: hexes 0..ne8-1, then tets ne8..ne8+ne4-1)
//   rowptr     int[nfree+1], cols int[nnzb]   block (3x3) CSR pattern, columns sorted
//   slot       uint16[8*len(inc)]      for incidence k and local node b: block
//                                      position within the row, 0xFFFF if b is fixed
//   Kb         double[9*nnzb]          K values, block-row-major, 3x3 blocks row-major
//                                      (derived from sv64 on demand after a fused assembly)
//   sl_ptr, scols, sv64, sv16          the solver's copy of K in BSELL-32 (sell.cuh),
//                                      FP64 values and a BF16 rounding
//   se_ptr, se_list, inc_loc           per BSELL slice the sorted elements of its rows, and
//                                      each incidence's position in them (fused assembly)
//   Ke         double[576*ne8 + 144*ne4]  element matrices (scratch of the two-pass assembly):
//                                      element g, block (a,b), entries 3x3 row-major
//   Dinv       double[9*nfree]         inverted diagonal blocks (block-Jacobi), + FP32 copy
//   coarse                             aggregates, E = Z^T K Z and its FP32 inverse (precond.cu)
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "host_pool.cuh"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <functional>
#include <future>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/ofea_gpu.h"

namespace ofea {

struct Failure {
    int code;
    std::string msg;
};

[[noreturn]] void fail(int code, const std::string &msg);
[[noreturn]] void fail_cuda(cudaError_t e, const char *what, const char *file, int line);
void set_last_error(const std::string &msg);

#define OFEA_CUDA(call)                                                   \
    do {                                                                  \
        cudaError_t e_ = (call);                                          \
        if (e_ != cudaSuccess) ::ofea::fail_cuda(e_, #call, __FILE__, __LINE__); \
    } while (0)

#define OFEA_CHECK_LAUNCH() OFEA_CUDA(cudaGetLastError())

// Device memory of the library's buffers comes from a per-device cache
// (devmem.cu): dev_free waits for the device and keeps the block, dev_alloc
// reuses a fitting one or calls cudaMalloc; dev_trim frees the cached blocks.
void *dev_alloc(size_t bytes, size_t *got, int *device);
void dev_free(void *p, size_t bytes, int device);
void dev_trim();

template <class T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    size_t bytes = 0;  // size of the block held
    int dev = 0;       // the GPU it lives on
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) dev_free(p, bytes, dev);
        p = nullptr;
        n = 0;
        bytes = 0;
    }
    // Grow-only allocation; contents are not preserved on growth.
    void ensure(size_t count) {
        if (count <= n && p) return;
        release();
        const size_t want = std::max(count, size_t(1)) * sizeof(T);
        if (want / sizeof(T) < count) fail(OFEA_ERR_OOM, "allocation size overflows");
        p = static_cast<T *>(dev_alloc(want, &bytes, &dev));
        n = count;
    }
    void upload(const T *h, size_t count, cudaStream_t s) {
        ensure(count);
        if (count) OFEA_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
};

// Pinned host scratch.  Blocks come from a per-process cache (devmem.cu):
// cudaMallocHost takes milliseconds, and a fresh context would otherwise pay
// it for every small flag buffer.
void *pinned_take(size_t bytes);
void pinned_give(void *p, size_t bytes);

template <class T>
struct HostBuf {
    T *p = nullptr;
    size_t n = 0;
    HostBuf() = default;
    HostBuf(const HostBuf &) = delete;
    HostBuf &operator=(const HostBuf &) = delete;
    ~HostBuf() {
        if (p) pinned_give(p, n * sizeof(T));
    }
    void ensure(size_t count) {
        if (count <= n && p) return;
        if (p) pinned_give(p, n * sizeof(T));
        p = nullptr;
        n = 0;
        p = static_cast<T *>(pinned_take(count * sizeof(T)));
        n = count;
    }
};

constexpr int kBlock = 256;          // threads per CTA for streaming kernels
constexpr int kWarpsPerBlock = kBlock / 32;
constexpr uint16_t kNoSlot = 0xFFFF;

// Solver workspace (vectors of n or nfree*9 entries).
struct SolverWork {
    DevBuf<double> r, z, q, p0, p1, u, f, t;  // FP64
    DevBuf<float> b32, x32, t32, z32a, z32b;    // FP32 preconditioner vectors
    DevBuf<double> partials;   // reduction partials (several arrays of kMaxGrid)
    DevBuf<int> flags;         // [0]=done [1]=iters [2]=status
    HostBuf<int> hflags;
    HostBuf<double> hscal;
};

constexpr int kMaxGrid = 4096;  // upper bound on CTAs of any reducing kernel

// Coarse space of the two-level preconditioner (precond.cu).
struct Coarse {
    bool geom_ok = false, K_ok = false;
    int target = 0, na = 0, m = 0, max_agg = 0, band = 0;  // band: max |J - I| of neighbouring aggregates
    int nc[3] = {1, 1, 1};
    double lo[3] = {0, 0, 0}, ext[3] = {0, 0, 0};
    double inv_scale = 1.0, lmax = 0.0;
    DevBuf<int> agg_of, agg_ptr, agg_nodes, agg_cell, cell_agg, nbr;
    DevBuf<double> centroid, E, S, P, diag0, pp, part;
    DevBuf<float> Einv32, cvec, evec, pw;
    DevBuf<float> agg_off;  // [nfree][4] in aggregate order: offset from the centroid (cell units), row
    DevBuf<float> row_off;  // [nfree][4] in row order: the same offset, aggregate
    DevBuf<unsigned long long> row_cell;  // [nfree] in row order: the aggregate's cell, 21 bits per axis
    DevBuf<int> nof;                      // [nfree] node of each free row (input of the transfer offsets)
    // the coarse solve as a block LDL^T factor (precond.cu): S_k, L_ik and the
    // FP32 array F (U = diag(S) V below, V^T above); dense_ok: Einv32 holds the
    // dense inverse (the Gauss-Jordan path, or formed from F on demand)
    bool factored = false, dense_ok = false;
    int nbw = 0, ldf = 0;  // block half-bandwidth; row stride of F (m rounded up to 4)
    DevBuf<double> Sb, Lb;
    DevBuf<float> F32, zvec;
    std::vector<int> agg_cell_h, cell_agg_h;  // host copies (nesting of the learned level)
    std::vector<double> centroid_h;
};

// Learned coarse-correction stage (learned.cu): network weights, Adam state,
// per-K data of the nested level and activation buffers.
struct Learned {
    bool links_ok = false;  // parent / children tables of the nested level
    struct Layout {
        size_t W0, b0, W[4], b[4], Wd, bd, c0, total;
    };
    static Layout layout();
    void init_weights(unsigned seed);
    std::vector<float> host_w;
    bool have_weights = false, uploaded = false, fitted = false, inference_ready = false;
    int trained_steps = 0;
    DevBuf<float> w, g, m, v, part;              // weights, gradient, Adam moments, wgrad partials
    DevBuf<double> Eb, sigma, lossp, cpart;      // E2 blocks, sample RMS, loss / coefficient partials
    DevBuf<float> Ehat, dsq, feat, pdel, shifted, invdeg, Binv, X0, scale;
    DevBuf<int> parent, children;
    DevBuf<float> Z0, H[5], A[4], Zl[4], Y, dY, dH, dZ, dA;  // network activations (one row per aggregate)
    DevBuf<float> pv[9];                                      // stage vectors (rows of a batch)
    DevBuf<float> batch_src, r32, data;
    DevBuf<int> tc_err;  // set by a tensor-core product whose wait ran out
    long cap_rows = 0;
    int nlossp = 0, nsamples = 0, max_samples = 0;
};

}  // namespace ofea

struct ofea_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaStream_t side_stream = nullptr;  // the coarse inversion's lookahead; the network beside the coarse factor (owned)
    cudaStream_t aux_stream = nullptr;   // power iteration beside the coarse inversion (owned)
    cudaStream_t geo_stream = nullptr;   // uploads of the coarse geometry (owned)
    // During a preconditioned solve's iterations: the solve's stop flag on the
    // device (its V-cycle kernels return at once once it is set); else null.
    const int *vc_stop = nullptr;
    std::future<void> geom_job;          // coarse geometry built in the background after the pattern
    // mesh
    int nd = 0, ne = 0, ne8 = 0, ne4 = 0, nfree = 0, n = 0;
    double E0 = 0, nu = 0;
    ofea::HVec<int> elem_type;     // caller order
    ofea::HVec<int> elem_local;    // caller element -> index within its type
    ofea::HVec<double> xyz_h;      // host copies for the coarse-space setup
    ofea::HVec<int> fm_h, topo_h;  // topo_h: ne x 8, 0-based
    ofea::DevBuf<double> xyz, E8, E4;
    ofea::DevBuf<int> topo8, topo4, free_map, node_of_free;
    bool mesh_ok = false;
    // K uploaded as CSC arrays (ofea_matrix_upload_csc): no elements, and the
    // widest node coupling per direction stands in for the element extent
    bool matrix_only = false;
    double coupling_ext[3] = {0, 0, 0};
    // pattern
    ofea::DevBuf<int> inc_ptr, inc, rowptr, cols, diag_pos;
    ofea::DevBuf<uint16_t> slot;
    long long nnzb = 0;
    int max_deg = 0;
    bool pattern_ok = false;
    // values
    ofea::DevBuf<double> Kb, Ke, Fe, Dinv, u_nl, f_int;
    ofea::DevBuf<float> Dinv32;
    bool K_ok = false, jacobi_ok = false;
    // what the last assembly left current besides the solver copy: the fused
    // linear assembly writes only sv64, sv16g and Dinv; Kb, sv16 and Ke are
    // derived on demand (ensure_kb, ensure_sv16, ensure_element_matrices)
    bool kb_ok = false, sv16_ok = false, ke_ok = false, jacobi_fresh = false;
    int asm_path = 1;  // 0: the fused assembly made K, 1: the two-pass assembly or a CSC upload
    // per-slice element lists of the fused assembly (integrate.cu), per pattern:
    // se_state 0 not built, 1 built, -1 the mesh takes the two-pass assembly
    ofea::DevBuf<int> se_ptr, se_list;
    ofea::DevBuf<uint16_t> inc_loc;
    int se_state = 0;
    bool fused_off = false;  // ofea_set_assembly_path(ctx, 1): always the two-pass assembly
    // solver layout of K (sell.cuh): BSELL-32, FP64 and BF16 values
    ofea::DevBuf<int> sl_ptr, scols;
    ofea::DevBuf<double> sv64;
    ofea::DevBuf<__nv_bfloat16> sv16;  // BF16 copy (plane layout) for the batched solver's V-cycle
    ofea::DevBuf<int> sl_g;            // slot-group offsets of the grouped BF16 copy (sell.cuh)
    ofea::DevBuf<__nv_bfloat16> sv16g; // grouped BF16 copy for the single-matrix V-cycle SpMVs
    long long sell_len = 0;
    bool sell_ok = false;         // values of the solver copy current
    bool sell_layout_ok = false;  // slice pointers, columns and buffers for the current pattern
    ofea::Coarse coarse;      // exact coarse level
    ofea::Coarse coarse2;     // nested finer level of the learned stage
    ofea::Learned learned;
    int coarse_nodes = 1000;  // target free nodes per aggregate
    int coarse_solver = 0;    // 0: block LDL^T factor where the band allows, 1: dense inverse
    ofea::SolverWork w;
    ofea::DevBuf<int> scratch_i;
    ofea::DevBuf<int> err_flag;
    ofea::HostBuf<int> herr;
    // set-up trace (ofea_set_setup_trace): events recorded on the context
    // stream at the phase boundaries of the last preconditioner set-up
    bool setup_trace = false;
    std::vector<std::pair<const char *, cudaEvent_t>> setup_marks;
};

namespace ofea {
// pattern.cu
void build_pattern(ofea_ctx *c);
// csc.cu
void upload_csc(ofea_ctx *c, int n, const int *col_ptr, const int *row_idx, const double *val);
// integrate.cu
void assemble_linear(ofea_ctx *c);
void assemble_nl(ofea_ctx *c, const double *d_u, double *d_fint);
void build_block_jacobi(ofea_ctx *c);
void ensure_kb(ofea_ctx *c);
void ensure_sv16(ofea_ctx *c);
void ensure_element_matrices(ofea_ctx *c);
void stress_recovery(ofea_ctx *c, const double *d_u, int mode, double *d_elem, double *d_node);
// sell.cu
void build_sell_layout(ofea_ctx *c);
void build_sell(ofea_ctx *c);
// solve.cu
void spmv64(ofea_ctx *c, const double *d_x, double *d_y);
void solve_device(ofea_ctx *c, const double *d_f, double *d_u, const ofea_solve_opts &o,
                  ofea_solve_stats &st, const std::function<void(const double *)> &on_chunk = {});
void profile_kernels(ofea_ctx *c, int method, int reps, double *ms, double *bytes);
// set-up trace: setup_mark records an event named `phase` (the phase that
// ends there) when tracing is on; setup_marks_clear drops the last set-up's
void setup_mark(ofea_ctx *c, const char *phase);
void setup_marks_clear(ofea_ctx *c);
// learned.cu
void setup_learned_level(ofea_ctx *c);
void setup_learned_levels(ofea_ctx *c);
void geometry_start(ofea_ctx *c);
void geometry_join(ofea_ctx *c);
void setup_learned_solver(ofea_ctx *c);
void learned_coarse_correct(ofea_ctx *c, const float *t, float *x);
// Batched persistent solver (batched.cu).
ofea_batch *batch_create(ofea_ctx *const *ctxs, int nv, int nrhs);
void batch_destroy(ofea_batch *b);
void batch_set_rhs(ofea_batch *b, const double *const *f);
void batch_get_solution(ofea_batch *b, double *const *u);
void batch_solve(ofea_batch *b, const ofea_solve_opts &o, ofea_solve_stats *stats,
                 ofea_solve_stats *case_stats = nullptr);
void batch_tuning(ofea_batch *b, int method, int *rl, int *threads, int *ctas_per_sm, double *ms_per_iter);
void batch_set_trace(ofea_batch *b, int max_phases);
void batch_phase_times(ofea_batch *b, double *ms, int cap, int *count);
void barrier_probe(ofea_ctx *c, int limit_ms, int *released);
void learned_begin_dataset(ofea_ctx *c, int max_samples);
void learned_add_sample(ofea_ctx *c, const double *d_r);
void learned_train(ofea_ctx *c, int steps, int batch, float lr, unsigned seed, double *loss0, double *loss1);
void learned_gradient(ofea_ctx *c, const float *h_x, int B, double *loss, float *h_grad);
// ca.cu
constexpr int kCaMaxBasis = OFEA_CA_MAX_BASIS;
void ca_reanalysis(ofea_ctx *base, ofea_ctx *mod, const double *h_f, const double *h_u0, int nb,
                   const ofea_solve_opts &o, double *h_u, ofea_ca_stats *stats);
// noalloc.cu
void noalloc_prepare(int device);
void residual_norms_noalloc(ofea_ctx *c, int nrhs, const double *d_f, const double *d_u,
                            double *d_norms);
// pattern.cu (scan)
long long exclusive_scan(const int *d_in, int *d_out, int n, cudaStream_t s, int *d_tmp,
                         int tmp_len);
int grid_for(const ofea_ctx *c, long long work_items, int per_block);
}  // namespace ofea
