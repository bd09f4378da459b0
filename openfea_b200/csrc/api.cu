// C ABI entry points (include/ofea_gpu.h).  Every function catches internal
// failures and returns a status code; nothing throws or exits across the ABI.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <fstream>
#include <memory>
#include <mutex>
#include <random>

#include "host_pool.cuh"
#include "ofea_internal.cuh"
#include "precond.cuh"
#include "tc_gemm.cuh"

namespace ofea {

thread_local std::string g_last_error;

void set_last_error(const std::string &msg) { g_last_error = msg; }

[[noreturn]] void fail(int code, const std::string &msg) { throw Failure{code, msg}; }

[[noreturn]] void fail_cuda(cudaError_t e, const char *what, const char *file, int line) {
    int code = (e == cudaErrorMemoryAllocation) ? OFEA_ERR_OOM
               : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? OFEA_ERR_NO_DEVICE
                                                                              : OFEA_ERR_CUDA;
    cudaGetLastError();
    throw Failure{code, std::string(what) + ": " + cudaGetErrorString(e) + " (" + file + ":" +
                            std::to_string(line) + ")"};
}

template <class F>
int guarded(F f) {
    try {
        f();
        return OFEA_OK;
    } catch (const Failure &e) {
        set_last_error(e.msg);
        return e.code;
    } catch (const std::bad_alloc &) {
        set_last_error("host allocation failed");
        return OFEA_ERR_OOM;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return OFEA_ERR_INVALID_ARG;
    }
}

static void use_device(ofea_ctx *c) { OFEA_CUDA(cudaSetDevice(c->device)); }

static void need(bool cond, int code, const char *msg) {
    if (!cond) fail(code, msg);
}

static const char *const kNoElements =
    "the context holds a matrix loaded by ofea_matrix_upload_csc, without elements";

}  // namespace ofea

using namespace ofea;

extern "C" {

const char *ofea_version(void) { return "ofea_gpu 0.1.0 (sm_100a)"; }

const char *ofea_status_string(int s) {
    switch (s) {
        case OFEA_OK: return "ok";
        case OFEA_ERR_INVALID_ARG: return "invalid argument";
        case OFEA_ERR_CUDA: return "CUDA error";
        case OFEA_ERR_OOM: return "out of device memory";
        case OFEA_ERR_NOT_CONVERGED: return "not converged";
        case OFEA_ERR_TIMEOUT: return "time budget exceeded";
        case OFEA_ERR_STATE: return "call out of order";
        case OFEA_ERR_CAPACITY: return "mesh exceeds a kernel limit";
        case OFEA_ERR_BREAKDOWN: return "CG breakdown (K not positive definite)";
        case OFEA_ERR_NO_DEVICE: return "no CUDA device";
        case OFEA_ERR_IO: return "I/O error";
        case OFEA_ERR_UNKNOWN_SOLVER: return "unknown solver";
        case OFEA_ERR_REJECTED: return "learned stage rejected";
        default: return "unknown status";
    }
}

const char *ofea_last_error(void) { return g_last_error.c_str(); }

void ofea_solve_opts_default(ofea_solve_opts *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->method = OFEA_SOLVER_PCG64;
    o->rtol = 1e-8;
    o->max_iter = 100000;
    o->time_budget_s = 0;
    o->check_every = 0;  // by method
    o->ru_delta = 0.1;
    o->use_graph = 1;
}

// The context's own stream gets the highest priority: while the coarse
// inversion's side stream runs a large update, the context stream's short
// serial kernels take the next free SM instead of queueing behind it.
static void create_ctx_stream(ofea_ctx *c) {
    int least = 0, greatest = 0;
    OFEA_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    OFEA_CUDA(cudaStreamCreateWithPriority(&c->stream, cudaStreamNonBlocking, greatest));
    c->own_stream = true;
}

int ofea_ctx_create(ofea_ctx **out, int device) {
    return guarded([&] {
        need(out != nullptr, OFEA_ERR_INVALID_ARG, "out is NULL");
        *out = nullptr;
        int count = 0;
        cudaError_t e = cudaGetDeviceCount(&count);
        if (e != cudaSuccess || count == 0) {
            cudaGetLastError();
            fail(OFEA_ERR_NO_DEVICE, "no CUDA device visible");
        }
        need(device >= 0 && device < count, OFEA_ERR_INVALID_ARG, "device out of range");
        ofea_ctx *c = new ofea_ctx();
        c->device = device;
        try {
            OFEA_CUDA(cudaSetDevice(device));
            OFEA_CUDA(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device));
            create_ctx_stream(c);
            noalloc_prepare(device);
            c->err_flag.ensure(4);
            c->herr.ensure(4);
        } catch (...) {
            delete c;
            throw;
        }
        *out = c;
    });
}

int ofea_ctx_destroy(ofea_ctx *c) {
    return guarded([&] {
        if (!c) return;
        cudaSetDevice(c->device);
        try {
            geometry_join(c);
        } catch (...) {  // a failed background geometry has nothing left to release
        }
        if (c->stream) cudaStreamSynchronize(c->stream);
        for (cudaStream_t x : {c->side_stream, c->aux_stream, c->geo_stream})
            if (x) {
                cudaStreamSynchronize(x);
                cudaStreamDestroy(x);
            }
        setup_marks_clear(c);
        if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
        delete c;
    });
}

int ofea_ctx_set_stream(ofea_ctx *c, void *stream) {
    return guarded([&] {
        need(c != nullptr, OFEA_ERR_INVALID_ARG, "ctx is NULL");
        use_device(c);
        OFEA_CUDA(cudaStreamSynchronize(c->stream));
        if (c->own_stream) cudaStreamDestroy(c->stream);
        if (stream) {
            c->stream = (cudaStream_t)stream;
            c->own_stream = false;
        } else {
            create_ctx_stream(c);
        }
    });
}

static void split_modulus(ofea_ctx *c, const double *E_elem, double E0, HVec<double> &E8,
                          HVec<double> &E4) {
    E8.assign(c->ne8, E0);
    E4.assign(c->ne4, E0);
    if (E_elem)
        for (int e = 0; e < c->ne; ++e) {
            double v = E_elem[e];
            need(std::isfinite(v), OFEA_ERR_INVALID_ARG, "non-finite Young's modulus");
            (c->elem_type[e] == 1 ? E8 : E4)[c->elem_local[e]] = v;
        }
}

// The DOF numbering and coordinates shared by both ways of loading a model:
// free_map numbers the free nodes 0..nfree-1 (resort_free_nodes_), every
// coordinate is finite.  Keeps the host copies the coarse levels are built from.
static void check_nodes(ofea_ctx *c, int nd, const double *xyz, const int *free_map) {
    int nfree = 0;
    HVec<char> seen(nd, 0);
    for (int i = 0; i < nd; ++i) {
        int f = free_map[i];
        need(f >= -1 && f < nd, OFEA_ERR_INVALID_ARG, "free_map entry out of range");
        if (f >= 0) {
            need(!seen[f], OFEA_ERR_INVALID_ARG, "free_map is not a numbering");
            seen[f] = 1;
            ++nfree;
        }
    }
    for (int i = 0; i < nfree; ++i)
        need(seen[i], OFEA_ERR_INVALID_ARG, "free_map must number free nodes 0..nfree-1");
    std::vector<char> finite(kHostChunks, 1);
    c->xyz_h.resize(3L * nd);
    c->fm_h.resize(nd);
    host_for_chunks([&](int k) {  // checks and the host copies, chunk by chunk
        const long i0 = chunk_begin(3L * nd, k), i1 = chunk_begin(3L * nd, k + 1);
        for (long i = i0; i < i1; ++i)
            if (!std::isfinite(xyz[i])) finite[k] = 0;
        std::copy(xyz + i0, xyz + i1, c->xyz_h.data() + i0);
        std::copy(free_map + chunk_begin(nd, k), free_map + chunk_begin(nd, k + 1), c->fm_h.data() + chunk_begin(nd, k));
    });
    for (int k = 0; k < kHostChunks; ++k) need(finite[k] != 0, OFEA_ERR_INVALID_ARG, "non-finite coordinate");
    c->nfree = nfree;
    c->n = 3 * nfree;
}

int ofea_mesh_upload(ofea_ctx *c, int nd, const double *xyz, int ne, const int *topo,
                     const int *etype, const double *E_elem, double E0, double nu,
                     const int *free_map) {
    return guarded([&] {
        need(c != nullptr, OFEA_ERR_INVALID_ARG, "ctx is NULL");
        need(nd > 0 && ne > 0 && xyz && topo && etype && free_map, OFEA_ERR_INVALID_ARG,
             "empty mesh or NULL array");
        need(ne < (1 << 28), OFEA_ERR_CAPACITY, "more than 2^28 elements");
        need(std::isfinite(E0) && std::isfinite(nu) && nu > -1.0 && nu < 0.5, OFEA_ERR_INVALID_ARG,
             "invalid material (nu must be in (-1, 0.5))");
        use_device(c);
        geometry_join(c);
        c->mesh_ok = c->pattern_ok = c->K_ok = c->sell_ok = false;
        c->matrix_only = false;
        c->coarse.geom_ok = c->coarse.K_ok = false;
        c->coarse2.geom_ok = c->coarse2.K_ok = false;
        c->learned.links_ok = false;
        c->nd = nd;
        c->ne = ne;
        c->E0 = E0;
        c->nu = nu;
        // the nodes first: their host copies are then copied to the device
        // while the element passes run (page-locked blocks: asynchronous DMA)
        check_nodes(c, nd, xyz, free_map);
        cudaStream_t s = c->stream;
        c->xyz.upload(c->xyz_h.data(), 3L * nd, s);
        c->free_map.upload(c->fm_h.data(), nd, s);
        // pass 1 (chunks of elements): checks, per-chunk counts by type and
        // the host copy of the types; the error reported is the first one in
        // element order
        struct Scan {
            long n8 = 0, n4 = 0;
            const char *why = nullptr;
        };
        std::vector<Scan> sc(kHostChunks);
        c->elem_type.resize(ne);
        host_for_chunks([&](int k) {
            Scan &r = sc[k];
            for (long e = chunk_begin(ne, k); e < chunk_begin(ne, k + 1); ++e) {
                const int t = etype[e];
                c->elem_type[e] = t;
                if (t != 0 && t != 1) {
                    r.why = "element type must be 0 (C3D4) or 1 (C3D8)";
                    return;
                }
                const int npe = t == 1 ? 8 : 4;
                for (int a = 0; a < npe; ++a) {
                    const int v = topo[8L * e + a];
                    if (v < 1 || v > nd) {
                        r.why = "node id out of range 1..nd in topo";
                        return;
                    }
                    for (int b = 0; b < a; ++b)
                        if (topo[8L * e + b] == v) {
                            r.why = "element repeats a node";
                            return;
                        }
                }
                if (E_elem && !std::isfinite(E_elem[e])) {
                    r.why = "non-finite Young's modulus";
                    return;
                }
                (t == 1 ? r.n8 : r.n4)++;
            }
        });
        std::vector<long> o8(kHostChunks + 1, 0), o4(kHostChunks + 1, 0);
        for (int k = 0; k < kHostChunks; ++k)
            if (sc[k].why) OFEA_CUDA(cudaStreamSynchronize(s));  // the node copies have left the host blocks
        for (int k = 0; k < kHostChunks; ++k) {
            need(sc[k].why == nullptr, OFEA_ERR_INVALID_ARG, sc[k].why);
            o8[k + 1] = o8[k] + sc[k].n8;
            o4[k + 1] = o4[k] + sc[k].n4;
        }
        // pass 2: 0-based device connectivity and modulus per type, element ->
        // position, host copy of the connectivity
        HVec<int> t8(8L * o8[kHostChunks]), t4(4L * o4[kHostChunks]);
        HVec<double> E8(o8[kHostChunks]), E4(o4[kHostChunks]);
        c->elem_local.resize(ne);
        c->topo_h.resize(8L * ne);
        host_for_chunks([&](int k) {
            long p8 = o8[k], p4 = o4[k];
            for (long e = chunk_begin(ne, k); e < chunk_begin(ne, k + 1); ++e) {
                const bool hex = etype[e] == 1;
                const long p = hex ? p8++ : p4++;
                int *dst = hex ? &t8[8 * p] : &t4[4 * p];
                (hex ? E8 : E4)[p] = E_elem ? E_elem[e] : E0;
                c->elem_local[e] = (int)p;
                for (int a = 0; a < (hex ? 8 : 4); ++a) dst[a] = topo[8L * e + a] - 1;
                for (int a = 0; a < 8; ++a) c->topo_h[8L * e + a] = topo[8L * e + a] > 0 ? topo[8L * e + a] - 1 : 0;
            }
        });
        c->ne8 = (int)o8[kHostChunks];
        c->ne4 = (int)o4[kHostChunks];
        c->topo8.upload(t8.data(), t8.size(), s);
        c->topo4.upload(t4.data(), t4.size(), s);
        c->E8.upload(E8.data(), E8.size(), s);
        c->E4.upload(E4.data(), E4.size(), s);
        OFEA_CUDA(cudaStreamSynchronize(s));
        c->mesh_ok = true;
        // the coarse levels' geometry depends on the mesh alone: it is built on
        // a host thread while the caller builds the pattern and assembles K
        // (every user of it joins the job first)
        geometry_start(c);
    });
}

int ofea_mesh_set_modulus(ofea_ctx *c, const double *E_elem, double E0) {
    return guarded([&] {
        need(c != nullptr, OFEA_ERR_INVALID_ARG, "ctx is NULL");
        need(c->mesh_ok, OFEA_ERR_STATE, "no mesh uploaded");
        use_device(c);
        HVec<double> E8, E4;
        split_modulus(c, E_elem, E0, E8, E4);
        c->E0 = E0;
        c->E8.upload(E8.data(), E8.size(), c->stream);
        c->E4.upload(E4.data(), E4.size(), c->stream);
        OFEA_CUDA(cudaStreamSynchronize(c->stream));
        c->K_ok = c->sell_ok = false;
        c->coarse.K_ok = false;
        c->coarse2.K_ok = false;
    });
}

int ofea_assemble_pattern(ofea_ctx *c, int *n, long long *nnz) {
    return guarded([&] {
        need(c != nullptr, OFEA_ERR_INVALID_ARG, "ctx is NULL");
        need(c->mesh_ok, OFEA_ERR_STATE, "no mesh uploaded");
        need(!c->matrix_only, OFEA_ERR_STATE, kNoElements);
        use_device(c);
        build_pattern(c);  // the coarse geometry, started by the mesh upload, may still be in flight
        if (n) *n = c->n;
        if (nnz) *nnz = 9 * c->nnzb;
    });
}

static void after_assembly(ofea_ctx *c) {
    if (!c->jacobi_fresh) build_block_jacobi(c);  // the fused assembly inverts the diagonal itself
    c->jacobi_fresh = false;
    if (!c->sell_ok) build_sell(c);  // the assembly kernels write it themselves
    OFEA_CUDA(cudaMemcpyAsync(c->herr.p, c->err_flag.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    OFEA_CUDA(cudaStreamSynchronize(c->stream));
    c->jacobi_ok = c->herr.p[0] == 0;
}

int ofea_assemble_linear(ofea_ctx *c) {
    return guarded([&] {
        need(c != nullptr, OFEA_ERR_INVALID_ARG, "ctx is NULL");
        need(c->pattern_ok, OFEA_ERR_STATE, "ofea_assemble_pattern first");
        need(!c->matrix_only, OFEA_ERR_STATE, kNoElements);
        use_device(c);
        assemble_linear(c);
        after_assembly(c);
    });
}

int ofea_assemble_nl(ofea_ctx *c, const double *u, double *f_int) {
    return guarded([&] {
        need(c != nullptr && u != nullptr, OFEA_ERR_INVALID_ARG, "NULL argument");
        need(c->pattern_ok, OFEA_ERR_STATE, "ofea_assemble_pattern first");
        need(!c->matrix_only, OFEA_ERR_STATE, kNoElements);
        use_device(c);
        c->u_nl.upload(u, c->n, c->stream);
        c->f_int.ensure(std::max(c->n, 1));
        assemble_nl(c, c->u_nl.p, c->f_int.p);
        if (f_int)
            OFEA_CUDA(cudaMemcpyAsync(f_int, c->f_int.p, sizeof(double) * c->n, cudaMemcpyDeviceToHost,
                                      c->stream));
        after_assembly(c);
    });
}

int ofea_matrix_upload_csc(ofea_ctx *c, int nd, const double *xyz, const int *free_map, int n,
                           const int *col_ptr, const int *row_idx, const double *val) {
    return guarded([&] {
        need(c != nullptr, OFEA_ERR_INVALID_ARG, "ctx is NULL");
        need(nd > 0 && xyz && free_map && n > 0 && col_ptr && row_idx && val, OFEA_ERR_INVALID_ARG,
             "empty model or NULL array");
        use_device(c);
        geometry_join(c);
        c->mesh_ok = c->pattern_ok = c->K_ok = c->sell_ok = false;
        c->coarse.geom_ok = c->coarse.K_ok = false;
        c->coarse2.geom_ok = c->coarse2.K_ok = false;
        c->learned.links_ok = false;
        c->matrix_only = true;
        c->nd = nd;
        c->ne = c->ne8 = c->ne4 = 0;
        c->elem_type.clear();
        c->elem_local.clear();
        c->topo_h.clear();
        check_nodes(c, nd, xyz, free_map);
        need(n == c->n, OFEA_ERR_INVALID_ARG, "n must be 3 x (free nodes of free_map)");
        need(col_ptr[0] == 0, OFEA_ERR_INVALID_ARG, "col_ptr[0] must be 0");
        for (int j = 0; j < n; ++j)
            need(col_ptr[j + 1] >= col_ptr[j], OFEA_ERR_INVALID_ARG, "col_ptr must be non-decreasing");
        need(col_ptr[n] % 9 == 0, OFEA_ERR_INVALID_ARG, "nnz must be a multiple of 9 (3x3 blocks)");
        cudaStream_t s = c->stream;
        c->xyz.upload(xyz, 3L * nd, s);
        c->free_map.upload(free_map, nd, s);
        upload_csc(c, n, col_ptr, row_idx, val);
        // the widest coupling per direction (the coarse cells must be wider),
        // over the block pattern, which the checks above have validated
        std::vector<int> node_of(c->nfree);
        for (int i = 0; i < nd; ++i)
            if (free_map[i] >= 0) node_of[free_map[i]] = i;
        double ext[kHostChunks][3] = {};
        host_for_chunks([&](int k) {
            for (long I = chunk_begin(c->nfree, k); I < chunk_begin(c->nfree, k + 1); ++I) {
                const double *xi = &xyz[3L * node_of[I]];
                for (int t = col_ptr[3 * I]; t < col_ptr[3 * I + 1]; t += 3) {
                    const double *xj = &xyz[3L * node_of[row_idx[t] / 3]];
                    for (int d = 0; d < 3; ++d) ext[k][d] = std::max(ext[k][d], std::fabs(xj[d] - xi[d]));
                }
            }
        });
        for (int d = 0; d < 3; ++d) {
            c->coupling_ext[d] = 0;
            for (int k = 0; k < kHostChunks; ++k) c->coupling_ext[d] = std::max(c->coupling_ext[d], ext[k][d]);
        }
        c->mesh_ok = true;
        c->pattern_ok = true;
        c->K_ok = true;
        c->kb_ok = true;
        c->asm_path = 1;
        c->jacobi_fresh = false;
        c->sell_ok = c->sell_layout_ok = false;
        after_assembly(c);
        geometry_start(c);
    });
}

int ofea_get_csr(ofea_ctx *c, int *rowptr, int *col, double *val) {
    return guarded([&] {
        need(c != nullptr, OFEA_ERR_INVALID_ARG, "ctx is NULL");
        need(c->pattern_ok, OFEA_ERR_STATE, "no pattern");
        need(val == nullptr || c->K_ok, OFEA_ERR_STATE, "K not assembled");
        use_device(c);
        const int nf = c->nfree;
        std::vector<int> brp(nf + 1), bcol(c->nnzb);
        std::vector<double> bval(val ? 9 * c->nnzb : 0);
        if (val) ensure_kb(c);
        OFEA_CUDA(cudaMemcpyAsync(brp.data(), c->rowptr.p, sizeof(int) * (nf + 1), cudaMemcpyDeviceToHost, c->stream));
        OFEA_CUDA(cudaMemcpyAsync(bcol.data(), c->cols.p, sizeof(int) * c->nnzb, cudaMemcpyDeviceToHost, c->stream));
        if (val)
            OFEA_CUDA(cudaMemcpyAsync(bval.data(), c->Kb.p, sizeof(double) * 9 * c->nnzb,
                                      cudaMemcpyDeviceToHost, c->stream));
        OFEA_CUDA(cudaStreamSynchronize(c->stream));
        // scalar row 3r+i: for each block (r, s): columns 3s+j, j = 0..2
        long pos = 0;
        if (rowptr) rowptr[0] = 0;
        for (int r = 0; r < nf; ++r) {
            int b0 = brp[r], b1 = brp[r + 1];
            for (int i = 0; i < 3; ++i) {
                for (int b = b0; b < b1; ++b)
                    for (int j = 0; j < 3; ++j) {
                        if (col) col[pos] = 3 * bcol[b] + j;
                        if (val) val[pos] = bval[9L * b + 3 * i + j];
                        ++pos;
                    }
                if (rowptr) rowptr[3 * r + i + 1] = (int)pos;
            }
        }
    });
}

int ofea_get_element_matrices(ofea_ctx *c, int first, int count, double *Ke) {
    return guarded([&] {
        need(c != nullptr && Ke != nullptr, OFEA_ERR_INVALID_ARG, "NULL argument");
        need(c->K_ok && !c->matrix_only, OFEA_ERR_STATE, "no assembly yet");
        need(first >= 0 && count >= 0 && first + count <= c->ne, OFEA_ERR_INVALID_ARG, "range");
        use_device(c);
        ensure_element_matrices(c);
        std::vector<double> blk(576);
        double *out = Ke;
        for (int e = first; e < first + count; ++e) {
            bool hex = c->elem_type[e] == 1;
            int npe = hex ? 8 : 4, m = 3 * npe;
            size_t off = hex ? 576L * c->elem_local[e] : 576L * c->ne8 + 144L * c->elem_local[e];
            OFEA_CUDA(cudaMemcpyAsync(blk.data(), c->Ke.p + off, sizeof(double) * m * m,
                                      cudaMemcpyDeviceToHost, c->stream));
            OFEA_CUDA(cudaStreamSynchronize(c->stream));
            // device layout [a][b][i][j] -> row-major (3a+i, 3b+j)
            for (int a = 0; a < npe; ++a)
                for (int b = 0; b < npe; ++b)
                    for (int i = 0; i < 3; ++i)
                        for (int j = 0; j < 3; ++j)
                            out[(3 * a + i) * m + 3 * b + j] = blk[((a * npe + b) * 9) + 3 * i + j];
            out += m * m;
        }
    });
}

int ofea_spmv(ofea_ctx *c, const double *x, double *y) {
    return guarded([&] {
        need(c != nullptr && x && y, OFEA_ERR_INVALID_ARG, "NULL argument");
        need(c->K_ok, OFEA_ERR_STATE, "K not assembled");
        use_device(c);
        c->w.t.ensure(std::max(c->n, 1));
        c->w.q.ensure(std::max(c->n, 1));
        OFEA_CUDA(cudaMemcpyAsync(c->w.t.p, x, sizeof(double) * c->n, cudaMemcpyHostToDevice, c->stream));
        spmv64(c, c->w.t.p, c->w.q.p);
        OFEA_CUDA(cudaMemcpyAsync(y, c->w.q.p, sizeof(double) * c->n, cudaMemcpyDeviceToHost, c->stream));
        OFEA_CUDA(cudaStreamSynchronize(c->stream));
    });
}

static std::string fmt_e(double v) {
    char b[32];
    std::snprintf(b, sizeof(b), "%.3e", v);
    return b;
}

static void check_solve_ready(ofea_ctx *c, const ofea_solve_opts &o) {
    need(c->K_ok, OFEA_ERR_STATE, "K not assembled");
    need(o.rtol > 0 && o.max_iter > 0, OFEA_ERR_INVALID_ARG, "rtol and max_iter must be positive");
    if (o.method != OFEA_SOLVER_PCG64 && o.method != OFEA_SOLVER_MIXED && o.method != OFEA_SOLVER_LEARNED)
        fail(OFEA_ERR_UNKNOWN_SOLVER, "unknown solver method");
    if (!c->jacobi_ok) fail(OFEA_ERR_BREAKDOWN, "a diagonal block of K is not positive definite");
}

int ofea_set_assembly_path(ofea_ctx *c, int path) {
    return guarded([&] {
        need(c != nullptr, OFEA_ERR_INVALID_ARG, "ctx is NULL");
        need(path == 0 || path == 1, OFEA_ERR_INVALID_ARG, "assembly path must be 0 (automatic) or 1 (two-pass)");
        c->fused_off = path == 1;
    });
}

int ofea_get_assembly_path(ofea_ctx *c, int *path) {
    return guarded([&] {
        need(c != nullptr && path != nullptr, OFEA_ERR_INVALID_ARG, "NULL argument");
        need(c->K_ok, OFEA_ERR_STATE, "K not assembled");
        *path = c->asm_path;
    });
}

int ofea_set_coarse_nodes(ofea_ctx *c, int nodes) {
    return guarded([&] {
        need(c != nullptr, OFEA_ERR_INVALID_ARG, "ctx is NULL");
        need(nodes >= 8 && nodes <= 1000000, OFEA_ERR_INVALID_ARG, "nodes per aggregate must be 8..1e6");
        geometry_join(c);
        if (nodes != c->coarse_nodes) {
            c->coarse_nodes = nodes;
            c->coarse.geom_ok = c->coarse.K_ok = false;
            c->coarse2.geom_ok = c->coarse2.K_ok = false;
        c->learned.links_ok = false;
        }
    });
}

int ofea_set_coarse_solver(ofea_ctx *c, int method) {
    return guarded([&] {
        need(c != nullptr, OFEA_ERR_INVALID_ARG, "ctx is NULL");
        need(method == 0 || method == 1, OFEA_ERR_INVALID_ARG, "coarse solver must be 0 (factor) or 1 (dense)");
        geometry_join(c);
        if (method != c->coarse_solver) {
            c->coarse_solver = method;
            c->coarse.K_ok = false;
            c->coarse2.K_ok = false;
        }
    });
}

int ofea_coarse_apply(ofea_ctx *c, const double *cv, double *y, int *m_out, int *factored) {
    return guarded([&] {
        need(c != nullptr, OFEA_ERR_INVALID_ARG, "ctx is NULL");
        use_device(c);
        Coarse &C = c->coarse;
        need(C.K_ok, OFEA_ERR_STATE, "no coarse level: run a MIXED or LEARNED solve first");
        const int m = C.m;
        if (m_out) *m_out = m;
        if (factored) *factored = C.factored ? 1 : 0;
        if (!cv || !y) return;
        std::vector<float> h(m);
        for (int i = 0; i < m; ++i) h[i] = (float)cv[i];
        DevBuf<float> dc, de;
        dc.upload(h.data(), m, c->stream);
        de.ensure(m);
        coarse_gemv(c, dc.p, de.p);
        OFEA_CUDA(cudaMemcpyAsync(h.data(), de.p, sizeof(float) * m, cudaMemcpyDeviceToHost, c->stream));
        OFEA_CUDA(cudaStreamSynchronize(c->stream));
        for (int i = 0; i < m; ++i) y[i] = h[i];
    });
}

int ofea_trim_device_memory(void) {
    return guarded([&] {
        dev_trim();
        host_cache_trim();
    });
}

int ofea_precond_reset(ofea_ctx *c) {
    return guarded([&] {
        need(c != nullptr, OFEA_ERR_INVALID_ARG, "ctx is NULL");
        geometry_join(c);
        c->coarse.K_ok = false;
        c->coarse2.K_ok = false;
    });
}

int ofea_solve_device(ofea_ctx *c, const double *d_f, double *d_u, const ofea_solve_opts *opts,
                      ofea_solve_stats *stats) {
    ofea_solve_stats st{};
    int rc = guarded([&] {
        need(c != nullptr && d_f && d_u, OFEA_ERR_INVALID_ARG, "NULL argument");
        ofea_solve_opts o;
        if (opts)
            o = *opts;
        else
            ofea_solve_opts_default(&o);
        check_solve_ready(c, o);
        use_device(c);
        OFEA_CUDA(cudaMemsetAsync(d_u, 0, sizeof(double) * c->n, c->stream));
        solve_device(c, d_f, d_u, o, st);
        if (st.status != OFEA_OK)
            set_last_error(std::string("solve: ") + ofea_status_string(st.status) +
                           ", relative residual " + fmt_e(st.rel_residual));
    });
    if (rc != OFEA_OK) st.status = rc;
    if (stats) *stats = st;
    return st.status;
}

int ofea_solve(ofea_ctx *c, const double *f, double *u, int nrhs, const ofea_solve_opts *opts,
               ofea_solve_stats *stats) {
    int worst = OFEA_OK;
    int rc = guarded([&] {
        need(c != nullptr && f && u && nrhs > 0, OFEA_ERR_INVALID_ARG, "NULL argument or nrhs < 1");
        ofea_solve_opts o;
        if (opts)
            o = *opts;
        else
            ofea_solve_opts_default(&o);
        check_solve_ready(c, o);
        use_device(c);
        const int n = c->n;
        if (nrhs > 1 && nrhs <= OFEA_BATCH_MAX_RHS && o.method != OFEA_SOLVER_LEARNED) {
            // several load cases on one K: one persistent launch for all of
            // them (the batched engine with one variant), K read once per
            // iteration for every load case
            std::unique_ptr<ofea_batch, void (*)(ofea_batch *)> b(batch_create(&c, 1, nrhs), batch_destroy);
            const double *fp[1] = {f};
            double *up[1] = {u};
            std::vector<ofea_solve_stats> cs(nrhs);
            batch_set_rhs(b.get(), fp);
            batch_solve(b.get(), o, nullptr, cs.data());
            batch_get_solution(b.get(), up);
            for (int k = 0; k < nrhs; ++k) {
                if (stats) stats[k] = cs[k];
                if (cs[k].status != OFEA_OK && worst == OFEA_OK) {
                    worst = cs[k].status;
                    set_last_error(std::string("solve: ") + ofea_status_string(cs[k].status) +
                                   ", relative residual " + fmt_e(cs[k].rel_residual));
                }
            }
            return;
        }
        c->w.f.ensure(std::max(n, 1));
        c->w.u.ensure(std::max(n, 1));
        // the caller's vectors pass through a page-locked block of the host
        // cache (copied on the host pool's threads, then one DMA each way)
        HVec<double> stage(std::max(n, 1));
        for (int k = 0; k < nrhs; ++k) {
            ofea_solve_stats st{};
            host_for_chunks([&](int q) {
                std::copy(f + (long)k * n + chunk_begin(n, q), f + (long)k * n + chunk_begin(n, q + 1),
                          stage.data() + chunk_begin(n, q));
            });
            OFEA_CUDA(cudaMemcpyAsync(c->w.f.p, stage.data(), sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
            OFEA_CUDA(cudaMemsetAsync(c->w.u.p, 0, sizeof(double) * n, c->stream));
            try {
                solve_device(c, c->w.f.p, c->w.u.p, o, st);
            } catch (...) {
                cudaStreamSynchronize(c->stream);  // no copy reads the staging block after it is released
                throw;
            }
            OFEA_CUDA(cudaMemcpyAsync(stage.data(), c->w.u.p, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
            OFEA_CUDA(cudaStreamSynchronize(c->stream));
            host_for_chunks([&](int q) {
                std::copy(stage.data() + chunk_begin(n, q), stage.data() + chunk_begin(n, q + 1),
                          u + (long)k * n + chunk_begin(n, q));
            });
            if (stats) stats[k] = st;
            if (st.status != OFEA_OK && worst == OFEA_OK) {
                worst = st.status;
                set_last_error(std::string("solve: ") + ofea_status_string(st.status) +
                               ", relative residual " + fmt_e(st.rel_residual));
            }
        }
    });
    if (rc != OFEA_OK) {
        if (stats) stats[0].status = rc;
        return rc;
    }
    return worst;
}

void ofea_learn_opts_default(ofea_learn_opts *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->sample_iters = 600;
    o->sample_every = 4;
    o->steps = 400;
    o->batch = 16;
    o->lr = 1e-3f;
    o->seed = 1234u;
}

static void prepare_learned_level(ofea_ctx *c) {
    need(c->K_ok, OFEA_ERR_STATE, "K not assembled");
    use_device(c);
    setup_learned_levels(c);
}

int ofea_learned_train(ofea_ctx *c, const double *f, const ofea_learn_opts *opts, ofea_learn_stats *stats) {
    return guarded([&] {
        need(c != nullptr, OFEA_ERR_INVALID_ARG, "ctx is NULL");
        ofea_learn_opts o;
        if (opts) o = *opts;
        else ofea_learn_opts_default(&o);
        need(o.sample_iters > 0 && o.sample_every > 0 && o.steps >= 0 && o.batch > 0 && o.lr > 0,
             OFEA_ERR_INVALID_ARG, "bad training options");
        const auto t0 = std::chrono::steady_clock::now();
        prepare_learned_level(c);
        Learned &N = c->learned;
        if (o.reset || !N.have_weights) N.init_weights(o.seed);
        const int n = c->n;
        c->w.f.ensure(std::max(n, 1));
        c->w.u.ensure(std::max(n, 1));
        std::vector<double> hf(n);
        if (f) {
            std::copy(f, f + n, hf.begin());
        } else {
            std::mt19937 rng(o.seed);
            std::normal_distribution<double> nd(0.0, 1.0);
            for (double &v : hf) v = nd(rng);
        }
        OFEA_CUDA(cudaMemcpyAsync(c->w.f.p, hf.data(), sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
        OFEA_CUDA(cudaMemsetAsync(c->w.u.p, 0, sizeof(double) * n, c->stream));
        learned_begin_dataset(c, o.sample_iters / o.sample_every + 2);
        ofea_solve_opts so;
        ofea_solve_opts_default(&so);
        so.method = OFEA_SOLVER_PCG64;
        so.rtol = 1e-14;  // run the full sampling budget
        so.max_iter = o.sample_iters;
        so.check_every = o.sample_every;
        ofea_solve_stats st{};
        solve_device(c, c->w.f.p, c->w.u.p, so, st, [&](const double *r) { learned_add_sample(c, r); });
        double l0 = 0, l1 = 0;
        if (o.steps > 0) learned_train(c, o.steps, o.batch, o.lr, o.seed, &l0, &l1);
        if (stats) {
            stats->samples = N.nsamples;
            stats->steps = o.steps;
            stats->loss_first = l0;
            stats->loss_last = l1;
            stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        }
    });
}

int ofea_learned_get_weights(ofea_ctx *c, float *w, long long *count) {
    return guarded([&] {
        need(c != nullptr && count != nullptr, OFEA_ERR_INVALID_ARG, "NULL argument");
        const size_t n = Learned::layout().total;
        *count = (long long)n;
        if (!w) return;
        Learned &N = c->learned;
        if (!N.have_weights) N.init_weights(1234u);
        std::copy(N.host_w.begin(), N.host_w.end(), w);
    });
}

int ofea_learned_set_weights(ofea_ctx *c, const float *w, long long count) {
    return guarded([&] {
        need(c != nullptr && w != nullptr, OFEA_ERR_INVALID_ARG, "NULL argument");
        need(count == (long long)Learned::layout().total, OFEA_ERR_INVALID_ARG, "weight count mismatch");
        Learned &N = c->learned;
        N.host_w.assign(w, w + count);
        N.have_weights = true;
        N.fitted = true;  // the caller's coefficients are kept by later training
        N.uploaded = false;
    });
}

int ofea_learned_save(ofea_ctx *c, const char *path) {
    return guarded([&] {
        need(c != nullptr && path != nullptr, OFEA_ERR_INVALID_ARG, "NULL argument");
        need(c->learned.have_weights, OFEA_ERR_STATE, "no weights");
        std::ofstream o(path, std::ios::binary);
        if (!o) fail(OFEA_ERR_IO, std::string("cannot write ") + path);
        const long long n = (long long)c->learned.host_w.size();
        o.write("OFEAGNN1", 8);
        o.write(reinterpret_cast<const char *>(&n), sizeof(n));
        o.write(reinterpret_cast<const char *>(c->learned.host_w.data()), sizeof(float) * n);
        if (!o) fail(OFEA_ERR_IO, std::string("cannot write ") + path);
    });
}

int ofea_learned_load(ofea_ctx *c, const char *path) {
    return guarded([&] {
        need(c != nullptr && path != nullptr, OFEA_ERR_INVALID_ARG, "NULL argument");
        std::ifstream in(path, std::ios::binary);
        if (!in) fail(OFEA_ERR_IO, std::string("cannot read ") + path);
        char magic[8];
        long long n = 0;
        in.read(magic, 8);
        in.read(reinterpret_cast<char *>(&n), sizeof(n));
        if (!in || std::memcmp(magic, "OFEAGNN1", 8) != 0 || n != (long long)Learned::layout().total)
            fail(OFEA_ERR_IO, std::string("not a weight file of this network: ") + path);
        std::vector<float> w(n);
        in.read(reinterpret_cast<char *>(w.data()), sizeof(float) * n);
        if (!in) fail(OFEA_ERR_IO, std::string("truncated weight file: ") + path);
        c->learned.host_w = std::move(w);
        c->learned.have_weights = true;
        c->learned.fitted = true;
        c->learned.uploaded = false;
    });
}

int ofea_learned_level(ofea_ctx *c, int *na, int *nbr, float *Ehat, float *feat) {
    return guarded([&] {
        need(c != nullptr && na != nullptr, OFEA_ERR_INVALID_ARG, "NULL argument");
        prepare_learned_level(c);
        const Coarse &C2 = c->coarse2;
        *na = C2.na;
        cudaStream_t s = c->stream;
        if (nbr) OFEA_CUDA(cudaMemcpyAsync(nbr, C2.nbr.p, sizeof(int) * 27 * C2.na, cudaMemcpyDeviceToHost, s));
        if (Ehat)
            OFEA_CUDA(cudaMemcpyAsync(Ehat, c->learned.Ehat.p, sizeof(float) * 27 * 36 * C2.na,
                                      cudaMemcpyDeviceToHost, s));
        if (feat)
            OFEA_CUDA(cudaMemcpyAsync(feat, c->learned.X0.p, sizeof(float) * OFEA_LEARN_NFEAT * C2.na,
                                      cudaMemcpyDeviceToHost, s));
        OFEA_CUDA(cudaStreamSynchronize(s));
    });
}

int ofea_learned_gradient(ofea_ctx *c, const float *x, int batch, double *loss, float *grad) {
    return guarded([&] {
        need(c != nullptr && x && loss && grad && batch > 0, OFEA_ERR_INVALID_ARG, "bad argument");
        prepare_learned_level(c);
        learned_gradient(c, x, batch, loss, grad);
    });
}

int ofea_residual_norms_noalloc(ofea_ctx *c, int nrhs, const double *d_f, const double *d_u,
                                double *d_norms) {
    return guarded([&] {
        need(c != nullptr && d_f && d_u && d_norms, OFEA_ERR_INVALID_ARG, "NULL argument");
        need(c->K_ok && c->sell_ok, OFEA_ERR_STATE, "K not assembled (or its solver copy not built)");
        OFEA_CUDA(cudaSetDevice(c->device));
        residual_norms_noalloc(c, nrhs, d_f, d_u, d_norms);
    });
}

int ofea_tc_matmul(int device, int M, int N, int K, const float *A, const float *B, float *D) {
    return guarded([&] {
        need(A && B && D && M > 0 && N > 0 && K > 0, OFEA_ERR_INVALID_ARG, "bad argument");
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
            cudaGetLastError();
            fail(OFEA_ERR_NO_DEVICE, "no CUDA device visible");
        }
        need(device >= 0 && device < count, OFEA_ERR_INVALID_ARG, "device out of range");
        OFEA_CUDA(cudaSetDevice(device));
        cudaStream_t s = nullptr;
        OFEA_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        try {
            DevBuf<float> dA, dB, dD;
            DevBuf<int> err;
            dA.upload(A, (size_t)M * K, s);
            dB.upload(B, (size_t)N * K, s);
            dD.ensure((size_t)M * N);
            err.ensure(1);
            OFEA_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), s));
            tc_gemm(s, M, N, K, 0, TcOperand{dA.p, K, 1}, TcOperand{dB.p, K, 1},
                    TcEpilogue{kTcRowMajor, dD.p, nullptr, nullptr, 0}, err.p);
            int herr = 0;
            OFEA_CUDA(cudaMemcpyAsync(D, dD.p, sizeof(float) * M * N, cudaMemcpyDeviceToHost, s));
            OFEA_CUDA(cudaMemcpyAsync(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
            OFEA_CUDA(cudaStreamSynchronize(s));
            if (herr) fail(OFEA_ERR_TIMEOUT, "tensor-core product: a wait inside the kernel ran out");
        } catch (...) {
            cudaStreamDestroy(s);
            throw;
        }
        cudaStreamDestroy(s);
    });
}

int ofea_batch_create(ofea_batch **out, ofea_ctx *const *ctxs, int n_variants, int nrhs) {
    return guarded([&] {
        need(out != nullptr && ctxs != nullptr, OFEA_ERR_INVALID_ARG, "NULL argument");
        *out = nullptr;
        *out = batch_create(ctxs, n_variants, nrhs);
    });
}

int ofea_batch_destroy(ofea_batch *b) {
    return guarded([&] { batch_destroy(b); });
}

int ofea_batch_set_rhs(ofea_batch *b, const double *const *f) {
    return guarded([&] {
        need(b != nullptr && f != nullptr, OFEA_ERR_INVALID_ARG, "NULL argument");
        batch_set_rhs(b, f);
    });
}

int ofea_batch_solve_resident(ofea_batch *b, const ofea_solve_opts *opts, ofea_solve_stats *stats) {
    return guarded([&] {
        need(b != nullptr, OFEA_ERR_INVALID_ARG, "NULL batch");
        ofea_solve_opts o;
        if (opts) o = *opts;
        else ofea_solve_opts_default(&o);
        batch_solve(b, o, stats);
    });
}

int ofea_batch_get_solution(ofea_batch *b, double *const *u) {
    return guarded([&] {
        need(b != nullptr && u != nullptr, OFEA_ERR_INVALID_ARG, "NULL argument");
        batch_get_solution(b, u);
    });
}

int ofea_batch_solve(ofea_batch *b, const double *const *f, double *const *u, const ofea_solve_opts *opts,
                     ofea_solve_stats *stats) {
    int rc = ofea_batch_set_rhs(b, f);
    if (rc != OFEA_OK) return rc;
    rc = ofea_batch_solve_resident(b, opts, stats);
    if (rc != OFEA_OK) return rc;
    return ofea_batch_get_solution(b, u);
}

int ofea_batch_tuning(ofea_batch *b, int method, int *rl, int *threads, int *ctas_per_sm, double *ms) {
    return guarded([&] {
        need(b != nullptr, OFEA_ERR_INVALID_ARG, "NULL batch");
        need(method == OFEA_SOLVER_PCG64 || method == OFEA_SOLVER_MIXED, OFEA_ERR_UNKNOWN_SOLVER, "method");
        batch_tuning(b, method, rl, threads, ctas_per_sm, ms);
    });
}

int ofea_batch_set_trace(ofea_batch *b, int max_phases) {
    return guarded([&] {
        need(b != nullptr, OFEA_ERR_INVALID_ARG, "NULL batch");
        batch_set_trace(b, max_phases);
    });
}

int ofea_batch_phase_times(ofea_batch *b, double *ms, int cap, int *count) {
    return guarded([&] {
        need(b != nullptr && count != nullptr && cap >= 0, OFEA_ERR_INVALID_ARG, "bad argument");
        batch_phase_times(b, ms, cap, count);
    });
}

int ofea_solve_batched(ofea_ctx *const *ctxs, int n_variants, const double *const *f, double *const *u, int nrhs,
                       const ofea_solve_opts *opts, ofea_solve_stats *stats) {
    ofea_batch *b = nullptr;
    int rc = ofea_batch_create(&b, ctxs, n_variants, nrhs);
    if (rc != OFEA_OK) return rc;
    rc = ofea_batch_solve(b, f, u, opts, stats);
    ofea_batch_destroy(b);
    return rc;
}

int ofea_check_barrier_timeout(ofea_ctx *c, int limit_ms, int *released) {
    return guarded([&] {
        need(c != nullptr && released != nullptr, OFEA_ERR_INVALID_ARG, "NULL argument");
        need(limit_ms >= 1 && limit_ms <= 10000, OFEA_ERR_INVALID_ARG, "limit_ms must be 1..10000");
        use_device(c);
        barrier_probe(c, limit_ms, released);
    });
}

int ofea_stress(ofea_ctx *c, const double *u, int mode, double *elem, double *node) {
    return guarded([&] {
        need(c != nullptr && u != nullptr, OFEA_ERR_INVALID_ARG, "NULL argument");
        need(mode == OFEA_STRESS_REFERENCE || mode == OFEA_STRESS_CAUCHY, OFEA_ERR_INVALID_ARG,
             "mode must be OFEA_STRESS_REFERENCE or OFEA_STRESS_CAUCHY");
        need(c->pattern_ok, OFEA_ERR_STATE, "no pattern (ofea_assemble_pattern)");
        need(!c->matrix_only, OFEA_ERR_STATE, kNoElements);
        use_device(c);
        cudaStream_t s = c->stream;
        DevBuf<double> du, de, dn;
        du.ensure(std::max(c->n, 1));
        de.ensure(7L * std::max(c->ne, 1));
        dn.ensure(7L * c->nd);
        OFEA_CUDA(cudaMemcpyAsync(du.p, u, sizeof(double) * c->n, cudaMemcpyHostToDevice, s));
        stress_recovery(c, du.p, mode, de.p, dn.p);
        if (node) OFEA_CUDA(cudaMemcpyAsync(node, dn.p, sizeof(double) * 7L * c->nd, cudaMemcpyDeviceToHost, s));
        std::vector<double> h;
        if (elem) {
            h.resize(7L * c->ne);
            OFEA_CUDA(cudaMemcpyAsync(h.data(), de.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s));
        }
        OFEA_CUDA(cudaStreamSynchronize(s));
        if (elem)  // unified id (hexes, then tets) -> caller order
            for (int e = 0; e < c->ne; ++e) {
                const long g = c->elem_type[e] == 1 ? c->elem_local[e] : (long)c->ne8 + c->elem_local[e];
                std::copy(h.begin() + 7 * g, h.begin() + 7 * g + 7, elem + 7L * e);
            }
    });
}

int ofea_ca_reanalysis(ofea_ctx *base, ofea_ctx *mod, const double *f, const double *u0, int n_basis,
                       const ofea_solve_opts *opts, double *u, ofea_ca_stats *stats) {
    int rc = guarded([&] {
        need(base != nullptr && mod != nullptr && f != nullptr && u != nullptr, OFEA_ERR_INVALID_ARG,
             "NULL argument");
        need(n_basis >= 1 && n_basis <= OFEA_CA_MAX_BASIS, OFEA_ERR_INVALID_ARG, "n_basis must be 1..32");
        need(base != mod, OFEA_ERR_INVALID_ARG, "base and modified are the same context");
        need(base->device == mod->device, OFEA_ERR_INVALID_ARG, "base and modified are on different GPUs");
        need(base->K_ok && base->sell_ok && mod->K_ok && mod->sell_ok, OFEA_ERR_STATE, "K not assembled");
        need(base->n == mod->n && base->nnzb == mod->nnzb && base->fm_h == mod->fm_h &&
                 base->topo_h == mod->topo_h && base->elem_type == mod->elem_type,
             OFEA_ERR_INVALID_ARG, "base and modified differ in nodes, elements or free numbering");
        ofea_solve_opts o;
        if (opts) o = *opts;
        else ofea_solve_opts_default(&o);
        check_solve_ready(base, o);
        use_device(base);
        ca_reanalysis(base, mod, f, u0, n_basis, o, u, stats);
    });
    if (rc != OFEA_OK && stats) stats->status = rc;
    return rc;
}

int ofea_profile_solver_kernels(ofea_ctx *c, int method, int reps, double *ms, double *bytes) {
    return guarded([&] {
        need(c != nullptr && ms && bytes && reps > 0, OFEA_ERR_INVALID_ARG, "bad argument");
        need(c->K_ok, OFEA_ERR_STATE, "K not assembled");
        need(method == OFEA_SOLVER_PCG64 || method == OFEA_SOLVER_MIXED, OFEA_ERR_UNKNOWN_SOLVER,
             "method");
        use_device(c);
        c->w.t.ensure(std::max(c->n, 1));
        profile_kernels(c, method, reps, ms, bytes);
    });
}

int ofea_set_setup_trace(ofea_ctx *c, int on) {
    return guarded([&] {
        need(c != nullptr, OFEA_ERR_INVALID_ARG, "ctx is NULL");
        use_device(c);
        c->setup_trace = on != 0;
        if (!on) setup_marks_clear(c);
    });
}

int ofea_setup_phase_times(ofea_ctx *c, double *ms, int cap, int *count, char *names, int names_len) {
    return guarded([&] {
        need(c != nullptr && count != nullptr && cap >= 0 && names_len >= 0, OFEA_ERR_INVALID_ARG,
             "bad argument");
        use_device(c);
        const auto &mk = c->setup_marks;
        const int n = mk.empty() ? 0 : (int)mk.size() - 1;
        *count = n;
        std::string joined;
        for (int i = 0; i < n; ++i) {
            if (ms && i < cap) {
                OFEA_CUDA(cudaEventSynchronize(mk[i + 1].second));
                float t = 0.f;
                OFEA_CUDA(cudaEventElapsedTime(&t, mk[i].second, mk[i + 1].second));
                ms[i] = t;
            }
            if (i) joined += ',';
            joined += mk[i + 1].first;
        }
        if (names && names_len > 0) {
            const size_t k = std::min(joined.size(), (size_t)names_len - 1);
            std::copy(joined.begin(), joined.begin() + k, names);
            names[k] = '\0';
        }
    });
}

}  // extern "C"
