// Two-level preconditioner of the mixed-precision solver.
//
//   M(r) = V(1,1) cycle in FP32:  x0 = w D^-1 b            (pre-smoothing, damped block Jacobi)
//                                 t  = b - K32 x0
//                                 x1 = x0 + Z E^-1 Z^T t   (coarse correction)
//                                 z  = x1 + w D^-1 (b - K32 x1)   (post-smoothing)
// with b = float(r), D the 3x3 diagonal blocks, w = 1.5 / lmax (lmax the
// power iteration's estimate of lambda_max(D^-1 K)), and Z the rigid-body modes of node
// aggregates: the free nodes are binned into a grid of cells of about
// `coarse_nodes` nodes; each non-empty cell I is an aggregate with six modes
// (three translations, three rotations about its centroid, scaled by the
// cell size).  E = Z^T K Z (FP64, 6 x 6 blocks between neighbouring cells) is
// banded in cell order; it is factored on the device as a block LDL^T (one
// thread-block cluster) and applied as two FP32 triangular GEMVs, or, where
// the band is too wide, inverted by blocked Gauss-Jordan and applied as one
// FP32 GEMV.
//
// The smoother's SpMV reads a BF16 rounding of K into FP32 arithmetic; that
// is accurate for the high-frequency error the smoother damps, and the smooth
// modes that the rounding of K would corrupt are carried by the
// exact FP64 coarse operator, so the FP64 outer iteration keeps the iteration
// count of an all-FP64 preconditioner.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <functional>
#include <future>
#include <mutex>
#include <numeric>
#include <thread>

#include <unistd.h>

#include "host_pool.cuh"
#include "precond.cuh"
#include "sell.cuh"
#include "solver_common.cuh"

namespace ofea {

// ---------------------------------------------------------- aggregation --

// Worker threads of host_for_chunks (host_pool.cuh), started on first use and
// kept (never torn down: process exit ends them).  run(w) calls w on every
// worker and on the caller and returns when all have returned; calls are
// serialised.
class HostPool {
public:
    explicit HostPool(int workers) : workers_(workers) {
        for (int t = 0; t < workers; ++t) std::thread([this] { loop(); }).detach();
    }
    void run(const std::function<void()> &w) {
        std::lock_guard<std::mutex> serial(run_mu_);
        {
            std::lock_guard<std::mutex> lk(mu_);
            work_ = &w;
            busy_ = workers_;
            ++gen_;
        }
        go_.notify_all();
        w();
        std::unique_lock<std::mutex> lk(mu_);
        done_.wait(lk, [&] { return busy_ == 0; });
    }

private:
    void loop() {
        unsigned seen = 0;
        for (;;) {
            const std::function<void()> *w;
            {
                std::unique_lock<std::mutex> lk(mu_);
                go_.wait(lk, [&] { return gen_ != seen; });
                seen = gen_;
                w = work_;
            }
            (*w)();
            std::lock_guard<std::mutex> lk(mu_);
            if (--busy_ == 0) done_.notify_all();
        }
    }
    std::mutex run_mu_, mu_;
    std::condition_variable go_, done_;
    const std::function<void()> *work_ = nullptr;
    unsigned gen_ = 0;
    int busy_ = 0, workers_;
};

// The pool of this process (a forked child inherits the object but not the
// threads, so it starts its own).
static HostPool &host_pool() {
    static std::mutex mu;
    static HostPool *p = nullptr;
    static pid_t owner = 0;
    std::lock_guard<std::mutex> lk(mu);
    if (!p || owner != getpid()) {
        p = new HostPool((int)std::min<unsigned>(kHostChunks, std::max(1u, std::thread::hardware_concurrency())) - 1);
        owner = getpid();
    }
    return *p;
}

void host_for_chunks(const std::function<void(int)> &f) {
    std::atomic<int> next(0);
    const std::function<void()> work = [&] {
        for (int k; (k = next.fetch_add(1)) < kHostChunks;) f(k);
    };
    host_pool().run(work);
}

// Offsets of the free rows from their aggregates' centroids (cell units,
// FP64 rounded to FP32): agg_off in aggregate order with the row index,
// row_off in row order with the aggregate index; row_cell in row order: the
// aggregate's cell (x | y << 21 | z << 42).
constexpr int kCellBits = 21;
constexpr unsigned long long kCellMask = (1ull << kCellBits) - 1;
__global__ void k_transfer_offsets(int nf, const int *__restrict__ agg_nodes, const int *__restrict__ agg_of,
                                   const int *__restrict__ nof, const double *__restrict__ xyz,
                                   const double *__restrict__ centroid, const int *__restrict__ agg_cell, double isc,
                                   float4 *__restrict__ agg_off, float4 *__restrict__ row_off,
                                   unsigned long long *__restrict__ row_cell) {
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nf; idx += gridDim.x * blockDim.x) {
        const int r = agg_nodes[idx], a = agg_of[r], node = nof[r];
        const float dx = (float)((xyz[3L * node] - centroid[3L * a]) * isc);
        const float dy = (float)((xyz[3L * node + 1] - centroid[3L * a + 1]) * isc);
        const float dz = (float)((xyz[3L * node + 2] - centroid[3L * a + 2]) * isc);
        agg_off[idx] = make_float4(dx, dy, dz, __int_as_float(r));
        row_off[r] = make_float4(dx, dy, dz, __int_as_float(a));
        row_cell[r] = (unsigned long long)agg_cell[3L * a] | ((unsigned long long)agg_cell[3L * a + 1] << kCellBits) |
                      ((unsigned long long)agg_cell[3L * a + 2] << (2 * kCellBits));
    }
}

// Bins the free nodes into the nc[0] x nc[1] x nc[2] cell grid over [lo, lo+ext]
// and fills C's aggregate arrays (non-empty cells in cell order, nodes in
// ascending free index, centroids, the cell -> aggregate table and, for the
// learned level, the 27-slot neighbour table).
static void bin_nodes(ofea_ctx *c, Coarse &C, const int nc[3], const double lo[3], const double ext[3]) {
    const int nd = c->nd, nf = c->nfree;
    const auto &X = c->xyz_h;
    const auto &fm = c->fm_h;
    HVec<int> nof(nf);
    host_for_chunks([&](int k) {
        for (long i = chunk_begin(nd, k); i < chunk_begin(nd, k + 1); ++i)
            if (fm[i] >= 0) nof[fm[i]] = (int)i;
    });
    for (int d = 0; d < 3; ++d) C.nc[d] = nc[d];
    const long ncell = (long)nc[0] * nc[1] * nc[2];
    // cell of every free row and per-chunk counts per cell
    HVec<int> cell_of(nf);
    std::vector<std::vector<int>> ccnt(kHostChunks);
    host_for_chunks([&](int k) {
        std::vector<int> &cnt = ccnt[k];
        cnt.assign(ncell, 0);
        for (long r = chunk_begin(nf, k); r < chunk_begin(nf, k + 1); ++r) {
            const int node = nof[r];
            int ci[3];
            for (int d = 0; d < 3; ++d) {
                ci[d] = ext[d] > 0 ? (int)std::floor((X[3L * node + d] - lo[d]) / ext[d] * nc[d]) : 0;
                ci[d] = std::min(std::max(ci[d], 0), nc[d] - 1);
            }
            cell_of[r] = (ci[0] * nc[1] + ci[1]) * nc[2] + ci[2];
            cnt[cell_of[r]]++;
        }
    });
    std::vector<int> cell_agg(ncell, -1), agg_cell3;
    std::vector<int> ptr(1, 0);
    int na = 0;
    for (long cl = 0; cl < ncell; ++cl) {
        int tot = 0;
        for (int k = 0; k < kHostChunks; ++k) tot += ccnt[k][cl];
        if (tot > 0) {
            cell_agg[cl] = na++;
            agg_cell3.push_back((int)(cl / ((long)nc[1] * nc[2])));
            agg_cell3.push_back((int)((cl / nc[2]) % nc[1]));
            agg_cell3.push_back((int)(cl % nc[2]));
            ptr.push_back(ptr.back() + tot);
        }
    }
    // chunk k's first slot in aggregate a: ptr[a] + rows of a in chunks < k
    // (rows stay in ascending order within each aggregate)
    std::vector<std::vector<int>> cur(kHostChunks, std::vector<int>(na));
    for (int a = 0; a < na; ++a) {
        const long cl = ((long)agg_cell3[3 * a] * nc[1] + agg_cell3[3 * a + 1]) * nc[2] + agg_cell3[3 * a + 2];
        int o = ptr[a];
        for (int k = 0; k < kHostChunks; ++k) {
            cur[k][a] = o;
            o += ccnt[k][cl];
        }
    }
    HVec<int> agg_of(nf), nodes(nf);
    std::vector<std::vector<double>> csum(kHostChunks);
    host_for_chunks([&](int k) {
        std::vector<int> &pos = cur[k];
        std::vector<double> &cs = csum[k];
        cs.assign(3L * na, 0.0);
        for (long r = chunk_begin(nf, k); r < chunk_begin(nf, k + 1); ++r) {
            const int a = cell_agg[cell_of[r]];
            agg_of[r] = a;
            nodes[pos[a]++] = (int)r;
            for (int d = 0; d < 3; ++d) cs[3L * a + d] += X[3L * nof[r] + d];
        }
    });
    std::vector<double> cen(3L * na, 0.0);
    for (int k = 0; k < kHostChunks; ++k)
        for (long j = 0; j < 3L * na; ++j) cen[j] += csum[k][j];
    for (int a = 0; a < na; ++a)
        for (int d = 0; d < 3; ++d) cen[3L * a + d] /= (ptr[a + 1] - ptr[a]);
    double scale = 0;
    for (int d = 0; d < 3; ++d) scale = std::max(scale, ext[d] > 0 ? ext[d] / nc[d] : 0.0);
    C.inv_scale = scale > 0 ? 1.0 / scale : 1.0;
    C.na = na;
    C.m = 6 * na;
    C.max_agg = 0;
    for (int a = 0; a < na; ++a) C.max_agg = std::max(C.max_agg, ptr[a + 1] - ptr[a]);
    // neighbour table: slot (dx+1)*9 + (dy+1)*3 + (dz+1), -1 where the cell is empty/outside
    std::vector<int> nbr(27L * na, -1);
    int band = 0;  // largest |J - I| over neighbouring aggregates
    for (int a = 0; a < na; ++a)
        for (int sl = 0; sl < 27; ++sl) {
            const int x = agg_cell3[3 * a] + sl / 9 - 1, y = agg_cell3[3 * a + 1] + (sl / 3) % 3 - 1,
                      z = agg_cell3[3 * a + 2] + sl % 3 - 1;
            if (x < 0 || y < 0 || z < 0 || x >= nc[0] || y >= nc[1] || z >= nc[2]) continue;
            const int J = cell_agg[((long)x * nc[1] + y) * nc[2] + z];
            nbr[27L * a + sl] = J;
            if (J >= 0) band = std::max(band, std::abs(J - a));
        }
    C.band = band;
    if (!c->geo_stream) OFEA_CUDA(cudaStreamCreateWithFlags(&c->geo_stream, cudaStreamNonBlocking));
    cudaStream_t st = c->geo_stream;  // its own stream: may run beside the assembly (geometry_start)
    C.agg_of.upload(agg_of.data(), nf, st);
    C.agg_ptr.upload(ptr.data(), na + 1, st);
    C.agg_nodes.upload(nodes.data(), nf, st);
    C.agg_cell.upload(agg_cell3.data(), agg_cell3.size(), st);
    C.cell_agg.upload(cell_agg.data(), ncell, st);
    C.centroid.upload(cen.data(), cen.size(), st);
    C.nbr.upload(nbr.data(), nbr.size(), st);
    // per free row its offset from the aggregate's centroid in cell units
    // (FP64, rounded to FP32), in aggregate order with the row (agg_off, the
    // restriction's coalesced reads) and in row order with the aggregate
    // (row_off, the prolongation's); formed on the device from the node
    // coordinates already there
    C.nof.upload(nof.data(), nf, st);
    C.agg_off.ensure(4L * std::max(nf, 1));
    C.row_off.ensure(4L * std::max(nf, 1));
    C.row_cell.ensure(std::max(nf, 1));
    for (int d = 0; d < 3; ++d)
        if (nc[d] > (int)kCellMask) fail(OFEA_ERR_CAPACITY, "coarse level: more than 2^21 cells along an axis");
    k_transfer_offsets<<<std::max(1, std::min((nf + 255) / 256, c->num_sms * 16)), 256, 0, st>>>(
        nf, C.agg_nodes.p, C.agg_of.p, C.nof.p, c->xyz.p, C.centroid.p, C.agg_cell.p, C.inv_scale,
        reinterpret_cast<float4 *>(C.agg_off.p), reinterpret_cast<float4 *>(C.row_off.p), C.row_cell.p);
    OFEA_CHECK_LAUNCH();
    OFEA_CUDA(cudaStreamSynchronize(st));
    C.agg_cell_h = std::move(agg_cell3);
    C.cell_agg_h = std::move(cell_agg);
    C.centroid_h = std::move(cen);
    C.geom_ok = true;  // K_ok is false already: every change of the geometry resets it first
}

void build_aggregation(ofea_ctx *c, int target_nodes) {
    Coarse &C = c->coarse;
    const int nd = c->nd, nf = c->nfree;
    const auto &X = c->xyz_h;
    const auto &fm = c->fm_h;
    // box of the free nodes and the largest element extent per direction
    // (cells must be at least 2.5x wider so that every K coupling stays
    // between neighbouring cells; the nested level, half as wide, then still
    // spans an element); min and max do not depend on the combining order
    double clo[kHostChunks][3], chi[kHostChunks][3], cem[kHostChunks][3];
    host_for_chunks([&](int k) {
        double l[3] = {1e300, 1e300, 1e300}, h[3] = {-1e300, -1e300, -1e300}, em[3] = {0, 0, 0};
        for (long i = chunk_begin(nd, k); i < chunk_begin(nd, k + 1); ++i)
            if (fm[i] >= 0)
                for (int d = 0; d < 3; ++d) {
                    l[d] = std::min(l[d], X[3L * i + d]);
                    h[d] = std::max(h[d], X[3L * i + d]);
                }
        for (long e = chunk_begin(c->ne, k); e < chunk_begin(c->ne, k + 1); ++e) {
            const int *t = &c->topo_h[8L * e];
            const int npe = c->elem_type[e] == 1 ? 8 : 4;
            for (int d = 0; d < 3; ++d) {
                double a = 1e300, b = -1e300;
                for (int q = 0; q < npe; ++q) {
                    a = std::min(a, X[3L * t[q] + d]);
                    b = std::max(b, X[3L * t[q] + d]);
                }
                em[d] = std::max(em[d], b - a);
            }
        }
        if (c->matrix_only)  // no elements: the widest coupling of K
            for (int d = 0; d < 3; ++d) em[d] = c->coupling_ext[d];
        for (int d = 0; d < 3; ++d) {  // written once per chunk (no shared cache lines in the loops)
            clo[k][d] = l[d];
            chi[k][d] = h[d];
            cem[k][d] = em[d];
        }
    });
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300}, emax[3] = {0, 0, 0};
    for (int k = 0; k < kHostChunks; ++k)
        for (int d = 0; d < 3; ++d) {
            lo[d] = std::min(lo[d], clo[k][d]);
            hi[d] = std::max(hi[d], chi[k][d]);
            emax[d] = std::max(emax[d], cem[k][d]);
        }
    double ext[3], vol = 1.0;
    int flat = 0;
    for (int d = 0; d < 3; ++d) {
        ext[d] = hi[d] - lo[d];
        if (ext[d] > 0) vol *= ext[d];
        else ++flat;
    }
    const double target = std::max(8, target_nodes);
    double s = std::pow(vol * target / std::max(nf, 1), 1.0 / std::max(1, 3 - flat));
    int nc[3];
    for (int d = 0; d < 3; ++d) {
        if (!(ext[d] > 0)) {
            nc[d] = 1;
            continue;
        }
        double cell = std::max(s, 2.5 * emax[d]);
        nc[d] = std::max(1, (int)std::lround(ext[d] / cell));
    }
    for (int d = 0; d < 3; ++d) {
        C.lo[d] = lo[d];
        C.ext[d] = ext[d];
    }
    bin_nodes(c, C, nc, lo, ext);
}

// The learned level: the same box, twice as many cells per direction, so each
// coarse cell is the union of 2 x 2 x 2 of these.
void build_aggregation_fine(ofea_ctx *c) {
    const Coarse &C = c->coarse;
    int nc[3];
    for (int d = 0; d < 3; ++d) nc[d] = C.ext[d] > 0 ? 2 * C.nc[d] : 1;
    bin_nodes(c, c->coarse2, nc, C.lo, C.ext);
}

// ------------------------------------------------------- coarse matrix --



// Stage 2: E entries from the chunk partials, fixed chunk order.
// Galerkin blocks E[I][s] = sum over nodes i of I and row blocks K_ij with
// aggregate(j) in neighbour slot s of Z_i^T K_ij Z_j (6 x 6, row-major), for
// every aggregate I of a level, with the rows' offsets of the V-cycle's
// transfers (agg_off, row_off: FP64 offsets rounded to FP32, so E is the
// exact Galerkin operator of the Z the V-cycle applies).  One CTA per
// aggregate; warp w takes the aggregate's nodes w, w + kGW, ... in order;
// lane t takes block t of the node's row (32 at a time), finds the slot of
// j's aggregate from j's packed cell (row_cell) and forms
// W = K_ij Z_j (3 x 6).  Lanes whose
// blocks land in the same slot are summed in lane order (match_any, then 32
// broadcast shuffles, or a shuffle tree when the whole warp shares one slot),
// the group's first lane adds Z_i^T W to its warp's accumulator, and the
// warps' accumulators are summed in warp order: deterministic.
constexpr int kGW = 4;  // warps per CTA

__device__ __forceinline__ void cross_e(int t, const double d[3], double z[3]) {
    // e_t x d
    if (t == 0) { z[0] = 0.0; z[1] = -d[2]; z[2] = d[1]; }
    else if (t == 1) { z[0] = d[2]; z[1] = 0.0; z[2] = -d[0]; }
    else { z[0] = -d[1]; z[1] = d[0]; z[2] = 0.0; }
}

__global__ void __launch_bounds__(kGW * 32) k_galerkin_blocks(
    int na, const int *__restrict__ agg_ptr, const float4 *__restrict__ agg_off, const float4 *__restrict__ row_off,
    const unsigned long long *__restrict__ row_cell, const int *__restrict__ agg_cell, const int *__restrict__ rowptr,
    const int *__restrict__ cols, KBlocks KB, double *__restrict__ Eb, int *__restrict__ err) {
    extern __shared__ double gsm[];
    double (*acc)[27 * 36] = reinterpret_cast<double (*)[27 * 36]>(gsm);                  // [kGW][27 * 36]
    double (*stage)[32][18] = reinterpret_cast<double (*)[32][18]>(gsm + kGW * 27 * 36);  // [kGW][32][18]
    __shared__ unsigned smask[kGW][32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int I = blockIdx.x; I < na; I += gridDim.x) {
        for (int v = threadIdx.x; v < kGW * 27 * 36; v += blockDim.x) (&acc[0][0])[v] = 0.0;
        __syncthreads();
        const int cx = agg_cell[3 * I], cy = agg_cell[3 * I + 1], cz = agg_cell[3 * I + 2];
        const int idx_end = agg_ptr[I + 1];
        int idx = agg_ptr[I] + w;
        // The warp's rows are walked with the next row's offset and pattern
        // range already in flight (loaded one row ahead): per row only the
        // lanes' column loads and their dependent loads remain on the chain.
        float4 oi = make_float4(0.f, 0.f, 0.f, 0.f), on = oi;  // current and next row: offset from the centroid, row
        int rb = 0, re = 0;
        if (idx < idx_end) {
            oi = agg_off[idx];
            rb = rowptr[__float_as_int(oi.w)];
            re = rowptr[__float_as_int(oi.w) + 1];
            if (idx + kGW < idx_end) on = agg_off[idx + kGW];
        }
        for (; idx < idx_end; idx += kGW) {
            const int i = __float_as_int(oi.w);
            const double di[3] = {oi.x, oi.y, oi.z};
            const int deg = re - rb;
            int rbn = 0, ren = 0;
            float4 onn = on;
            if (idx + kGW < idx_end) {
                rbn = rowptr[__float_as_int(on.w)];
                ren = rowptr[__float_as_int(on.w) + 1];
                if (idx + 2 * kGW < idx_end) onn = agg_off[idx + 2 * kGW];
            }
            for (int c0 = 0; c0 < deg; c0 += 32) {
                const int k = c0 + lane;
                double v[18];
#pragma unroll
                for (int e = 0; e < 18; ++e) v[e] = 0.0;
                int slot = -2;  // lanes past the row form their own group
                if (k < deg) {
                    const int j = cols[rb + k];
                    const float4 oj = row_off[j];
                    const unsigned long long pc = row_cell[j];
                    const int dx = (int)(pc & kCellMask) - cx, dy = (int)((pc >> kCellBits) & kCellMask) - cy,
                              dz = (int)(pc >> (2 * kCellBits)) - cz;
                    if (dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1 && dz >= -1 && dz <= 1) {
                        slot = (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1);
                    } else {
                        atomicExch(err, 1);
                        slot = -1;
                    }
                    const double dj[3] = {oj.x, oj.y, oj.z};
                    double K[9];
#pragma unroll
                    for (int e = 0; e < 9; ++e) K[e] = KB.at(i, k, e);
                    // W[:, l] = K e_l (l < 3), K (e_(l-3) x dj) (l >= 3); v[r * 6 + l]
#pragma unroll
                    for (int r = 0; r < 3; ++r)
#pragma unroll
                        for (int l = 0; l < 3; ++l) v[r * 6 + l] = K[3 * r + l];
#pragma unroll
                    for (int t = 0; t < 3; ++t) {
                        double z[3];
                        cross_e(t, dj, z);
#pragma unroll
                        for (int r = 0; r < 3; ++r) v[r * 6 + 3 + t] = K[3 * r] * z[0] + K[3 * r + 1] * z[1] + K[3 * r + 2] * z[2];
                    }
                }
                const unsigned mask = __match_any_sync(0xffffffffu, slot);
                const int leader = __ffs(mask) - 1;
                double W[18];
                if (__all_sync(0xffffffffu, mask == 0xffffffffu)) {
                    // one slot for the whole warp: tree sum
#pragma unroll
                    for (int e = 0; e < 18; ++e) {
                        double x = v[e];
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
                        W[e] = x;
                    }
                } else {
                    // several slots: the lanes' values go to shared memory, the
                    // (group, component) sums are spread over the lanes, each
                    // summed in ascending lane order and written back into its
                    // leader's row (groups are disjoint, so no other sum reads it)
#pragma unroll
                    for (int e = 0; e < 18; ++e) stage[w][lane][e] = v[e];
                    smask[w][lane] = mask;
                    __syncwarp();
                    const unsigned leaders = __ballot_sync(0xffffffffu, lane == leader);
                    const int ntask = __popc(leaders) * 18;
                    for (int task = lane; task < ntask; task += 32) {
                        const int gi = task / 18, e = task - 18 * gi;
                        const int L = (int)__fns(leaders, 0, gi + 1);
                        unsigned gm = smask[w][L];
                        double x = 0.0;
                        while (gm) {
                            const int t = __ffs(gm) - 1;
                            gm &= gm - 1;
                            x += stage[w][t][e];
                        }
                        stage[w][L][e] = x;
                    }
                    __syncwarp();
#pragma unroll
                    for (int e = 0; e < 18; ++e) W[e] = stage[w][lane][e];
                    __syncwarp();  // the stage is read before the next chunk overwrites it
                }
                if (lane == leader && slot >= 0) {
                    // E[k][l] += Z_i[:, k] . W[:, l]
                    double *a = acc[w] + slot * 36;
#pragma unroll
                    for (int kk = 0; kk < 3; ++kk)
#pragma unroll
                        for (int l = 0; l < 6; ++l) a[kk * 6 + l] += W[kk * 6 + l];
#pragma unroll
                    for (int t = 0; t < 3; ++t) {
                        double z[3];
                        cross_e(t, di, z);
#pragma unroll
                        for (int l = 0; l < 6; ++l)
                            a[(3 + t) * 6 + l] += z[0] * W[l] + z[1] * W[6 + l] + z[2] * W[12 + l];
                    }
                }
                __syncwarp();
            }
            oi = on;
            on = onn;
            rb = rbn;
            re = ren;
        }
        __syncthreads();
        for (int v = threadIdx.x; v < 27 * 36; v += blockDim.x) {
            double sum = 0.0;
#pragma unroll
            for (int q = 0; q < kGW; ++q) sum += acc[q][v];
            Eb[(long)I * 27 * 36 + v] = sum;
        }
        __syncthreads();
    }
}

__global__ void k_coarse_E_sum(int na, int nchunk_max, const int *__restrict__ agg_cell,
                               const int *__restrict__ cell_agg, int ncx, int ncy, int ncz, int m,
                               const double *__restrict__ part, double *__restrict__ E) {
    const long total = (long)na * 27 * 36;
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < total; g += (long)gridDim.x * blockDim.x) {
        const int I = (int)(g / (27 * 36));
        const int v = (int)(g % (27 * 36));
        const int slot = v / 36, e = v % 36, kk = e / 6, ll = e % 6;
        const int x = agg_cell[3 * I] + slot / 9 - 1, y = agg_cell[3 * I + 1] + (slot / 3) % 3 - 1,
                  z = agg_cell[3 * I + 2] + slot % 3 - 1;
        if (x < 0 || y < 0 || z < 0 || x >= ncx || y >= ncy || z >= ncz) continue;
        const int J = cell_agg[((long)x * ncy + y) * ncz + z];
        if (J < 0) continue;
        double s = 0.0;
        for (int ch = 0; ch < nchunk_max; ++ch) s += part[((long)I * nchunk_max + ch) * (27 * 36) + v];
        E[(6L * I + kk) * m + 6L * J + ll] = s;
    }
}

// --------------------------------------------- blocked Gauss-Jordan inverse --
//
// In-place inverse of the SPD matrix A (m x m, row-major) without pivoting,
// panel width kGJ.  For the diagonal block J (indices j0 .. j0+bb-1):
//   S = A_JJ^-1; P = A_{:,J} (saved);
//   A_{J,k} <- S A_{J,k}            for k outside J     (row panel)
//   A_{i,k} <- A_{i,k} - P_i A_{J,k} for i, k outside J (rank-bb update)
//   A_{i,J} <- -P_i S               for i outside J;  A_JJ <- S.
// A pivot that vanishes (a degenerate aggregate) drops its direction: its
// row and column of the result are zero.

constexpr int kGJ = 64;

// Inverse of the diagonal block A_JJ -> S (kGJ x kGJ, padded with zeros
// beyond bb) by one CTA of 256 threads: thread (ti, tj) keeps the entries
// (ti + 16 u, tj + 16 v), u, v = 0..3, in registers.  Pivot p: the holders of
// row p and column p publish them to shared memory (two buffers, so one
// barrier per pivot), then every thread applies the Gauss-Jordan step to its
// 16 entries: a_rc -= a_rp a_pc / a_pp, row p scaled by 1 / a_pp, column p by
// -1 / a_pp, a_pp <- 1 / a_pp.  A pivot that vanishes against the original
// diagonal (a degenerate aggregate) drops its direction: the step runs with
// 1 / a_pp replaced by 0, which zeroes row and column p and leaves the rest.
constexpr int kGjT = 16;  // threads per row / column of the thread grid

// The diagonal-block step of both coarse inversions: A_JJ (rows and columns
// j0..j0+bb of the m x m row-major A) -> its inverse S (kGJ x kGJ row-major,
// zero beyond bb), by the CTA's kGjT x kGjT threads; thread (ti, tj) holds
// the 4 x 4 block of rows 4 ti .. 4 ti + 3 and columns 4 tj .. 4 tj + 3.
// Pivot p = 4 pb + pp (pp unrolled, so every register index is fixed): the
// holders of row p and column p publish them to shared memory and zero them
// in their registers, the holder of a_pp publishes d = 1 / a_pp (0 for a
// vanishing pivot), one barrier, then every entry takes the same update
// a_rc <- a_rc - cr_r rc_c with cr_r = a_rp d (r != p), cr_p = -d,
// rc_c = a_pc (c != p), rc_p = 1, which gives a_rc - a_rp a_pc d off row and
// column p, a_pc d on row p, -a_rp d on column p and d at (p, p).
__device__ __forceinline__ void gj_block_inverse(int m, int j0, int bb, const double *__restrict__ A,
                                                 double *__restrict__ S, const double *__restrict__ diag0,
                                                 double (*srow)[kGJ], double (*scol)[kGJ], double *sthr,
                                                 double *sd) {
    const int tid = threadIdx.x, ti = tid / kGjT, tj = tid % kGjT;
    double a[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int r = 4 * ti + u, c = 4 * tj + v;
            a[u][v] = (r < bb && c < bb) ? __ldcg(A + (long)(j0 + r) * m + j0 + c) : 0.0;
        }
    if (tid < kGJ) sthr[tid] = tid < bb ? 1e-12 * __ldcg(diag0 + j0 + tid) : 0.0;
    __syncthreads();
    const int npb = (bb + 3) / 4;  // pivots beyond bb (zero rows) only drop their direction
#pragma unroll 1
    for (int pb = 0; pb < npb; ++pb) {
#pragma unroll
        for (int pp = 0; pp < 4; ++pp) {
            const int p = 4 * pb + pp, buf = pp & 1;
            const bool rowp = ti == pb, colp = tj == pb;
            if (rowp && colp) sd[buf] = a[pp][pp] > sthr[p] ? 1.0 / a[pp][pp] : 0.0;
            if (colp)
#pragma unroll
                for (int u = 0; u < 4; ++u) scol[buf][4 * ti + u] = a[u][pp];
            if (rowp)
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    srow[buf][kGjT * v + tj] = a[pp][v];  // column 4 tj + v, stored lane-contiguous
                    a[pp][v] = 0.0;
                }
            if (colp)
#pragma unroll
                for (int u = 0; u < 4; ++u) a[u][pp] = 0.0;
            __syncthreads();
            const double d = sd[buf];
            double cr[4], rc[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) cr[u] = scol[buf][4 * ti + u] * d;
            if (rowp) cr[pp] = -d;
#pragma unroll
            for (int v = 0; v < 4; ++v) rc[v] = srow[buf][kGjT * v + tj];
            if (colp) rc[pp] = 1.0;
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) a[u][v] = fma(-cr[u], rc[v], a[u][v]);
        }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) S[(4 * ti + u) * kGJ + 4 * tj + v] = a[u][v];
}

__global__ void __launch_bounds__(kGjT * kGjT) k_gj_diag(int m, int j0, int bb, const double *__restrict__ A,
                                                         double *__restrict__ S, const double *__restrict__ diag0) {
    __shared__ double srow[2][kGJ], scol[2][kGJ], sthr[kGJ], sd[2];
    gj_block_inverse(m, j0, bb, A, S, diag0, srow, scol, sthr, sd);
}

// Column panel, one warp per row i: P_i = A_{i,J} (saved for the update),
// A_{i,J} <- -P_i S (i outside J) or S (i inside J).
__global__ void __launch_bounds__(256) k_gj_panel(int m, int lim, int j0, int bb, double *__restrict__ A,
                                                  const double *__restrict__ S, double *__restrict__ P) {
    __shared__ double sS[kGJ][kGJ];
    for (int v = threadIdx.x; v < kGJ * kGJ; v += blockDim.x) sS[v / kGJ][v % kGJ] = S[v];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) / 32; i < lim; i += gridDim.x * blockDim.x / 32) {
        const bool in = i >= j0 && i < j0 + bb;
        double p0 = lane < bb ? A[(long)i * m + j0 + lane] : 0.0;
        double p1 = lane + 32 < bb ? A[(long)i * m + j0 + lane + 32] : 0.0;
        P[(long)i * kGJ + lane] = p0;
        P[(long)i * kGJ + lane + 32] = p1;
        double o0 = 0.0, o1 = 0.0;
        if (in) {
            o0 = sS[i - j0][lane];
            o1 = sS[i - j0][lane + 32];
        } else {
            for (int q = 0; q < 32; ++q) {
                const double pq = __shfl_sync(0xffffffffu, p0, q);
                o0 -= pq * sS[q][lane];
                o1 -= pq * sS[q][lane + 32];
            }
            for (int q = 0; q < 32; ++q) {
                const double pq = __shfl_sync(0xffffffffu, p1, q);
                o0 -= pq * sS[q + 32][lane];
                o1 -= pq * sS[q + 32][lane + 32];
            }
        }
        if (lane < bb) A[(long)i * m + j0 + lane] = o0;
        if (lane + 32 < bb) A[(long)i * m + j0 + lane + 32] = o1;
    }
}

// Row panel: A_{J,k} <- S A_{J,k} for k outside J; one CTA per 32 columns.
__global__ void __launch_bounds__(256) k_gj_rows(int m, int lim, int j0, int bb, double *__restrict__ A,
                                                 const double *__restrict__ S) {
    __shared__ double sS[kGJ][kGJ];  // read as broadcasts: no padding needed
    __shared__ double sR[kGJ][32];
    for (int v = threadIdx.x; v < kGJ * kGJ; v += blockDim.x) sS[v / kGJ][v % kGJ] = S[v];
    for (int k0 = blockIdx.x * 32; k0 < lim; k0 += gridDim.x * 32) {
        __syncthreads();
        for (int v = threadIdx.x; v < kGJ * 32; v += blockDim.x) {
            const int j = v / 32, kk = v % 32, k = k0 + kk;
            sR[j][kk] = (j < bb && k < lim) ? A[(long)(j0 + j) * m + k] : 0.0;
        }
        __syncthreads();
        // thread: column kk = tid % 32, rows i = tid / 32 + 8 q
        const int kk = threadIdx.x % 32, k = k0 + kk;
        const bool skip = k >= lim || (k >= j0 && k < j0 + bb);
        for (int q = 0; q < kGJ / 8; ++q) {
            const int i = threadIdx.x / 32 + 8 * q;
            if (i >= bb || skip) continue;
            double s = 0.0;
            for (int j = 0; j < bb; ++j) s = fma(sS[i][j], sR[j][kk], s);
            A[(long)(j0 + i) * m + k] = s;
        }
    }
}

// Rank-bb update of the outside block: A_ik -= P_i . A_{J,k}, 64 x 64 tiles,
// 256 threads with 4 x 4 outputs each; dynamic shared memory (66 KB).
// mode 0: every tile (2D grid); 2: every tile outside tile row and column
// `cross` (the next panel's rows and columns; 2D grid); 1: only those, on a
// 1D grid of 2 nt - 1 blocks (nt tiles per side): row `cross` first, then
// column `cross` without the shared tile.
__global__ void __launch_bounds__(256) k_gj_update(int m, int lim, int j0, int bb, double *__restrict__ A,
                                                   const double *__restrict__ P, int mode, int cross) {
    extern __shared__ double smem[];
    double (*sP)[kGJ + 1] = reinterpret_cast<double (*)[kGJ + 1]>(smem);             // [64][65]
    double (*sR)[64 + 1] = reinterpret_cast<double (*)[64 + 1]>(smem + 64 * (kGJ + 1));  // [64][65]
    int ty = blockIdx.y, tx = blockIdx.x;
    if (mode == 1) {
        const int nt = (lim + 63) / 64, b = blockIdx.x;
        if (b < nt) {
            ty = cross;
            tx = b;
        } else {
            const int q = b - nt;
            ty = q < cross ? q : q + 1;
            tx = cross;
        }
    } else if (mode == 2 && (ty == cross || tx == cross)) {
        return;
    }
    const int i0 = ty * 64, k0 = tx * 64;
    if (i0 >= j0 && i0 + 64 <= j0 + bb) return;  // every row of the tile is in J: nothing to update
    const int tr = threadIdx.x / 16, tc = threadIdx.x % 16;
    for (int v = threadIdx.x; v < 64 * kGJ; v += 256) {
        const int ii = v / kGJ, jj = v % kGJ;
        sP[ii][jj] = (i0 + ii < lim && jj < bb) ? P[(long)(i0 + ii) * kGJ + jj] : 0.0;
        const int jr = v / 64, kk = v % 64;
        sR[jr][kk] = (jr < bb && k0 + kk < lim) ? A[(long)(j0 + jr) * m + k0 + kk] : 0.0;
    }
    __syncthreads();
    double acc[4][4] = {};
    for (int j = 0; j < bb; ++j) {
        double pv[4], rv[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) pv[a] = sP[tr * 4 + a][j];
#pragma unroll
        for (int b = 0; b < 4; ++b) rv[b] = sR[j][tc * 4 + b];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] = fma(pv[a], rv[b], acc[a][b]);
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int i = i0 + tr * 4 + a;
        if (i >= lim || (i >= j0 && i < j0 + bb)) continue;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int k = k0 + tc * 4 + b;
            if (k >= lim || (k >= j0 && k < j0 + bb)) continue;
            A[(long)i * m + k] -= acc[a][b];
        }
    }
}

__global__ void k_diag_of(int m, const double *__restrict__ A, double *__restrict__ d) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
        d[i] = fabs(A[(long)i * m + i]);
}

__global__ void k_round_f32(long n, const double *__restrict__ a, float *__restrict__ b) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

// ------------------------------------------------ banded block LDL^T factor --
// The coarse solve of a banded E (half-bandwidth hb, so block half-bandwidth
// bw = floor((hb + 63) / 64) in 64 x 64 blocks) as a block LDL^T factor
// instead of the dense inverse:
//   for k = 0 .. nb-1:  S_k = (A_kk)^-1                  (gj_block_inverse)
//                       L_ik = A_ik S_k                  (k < i <= k + bw)
//                       A_ij -= L_ik A_jk^T              (k < j <= i <= k + bw)
// so A = L D L^T with L unit block-lower and D^-1 = diag(S_k); then, with
// V = L^-1 (unit block-lower, dense below the diagonal),
//   A^-1 = V^T diag(S) V,   V_ij = -sum_{l = max(j, i - bw)}^{i-1} L_il V_lj.
// The FP32 array F (m x m) keeps U = diag(S) V in its block-lower triangle
// (diagonal blocks: S_k) and V^T in its strict block-upper triangle, and
// A^-1 c = V^T (U c): two triangular GEMVs reading F once.  A vanishing pivot
// of a diagonal block drops its direction (zero row and column of S_k, hence
// of L's column and of the result), as in the dense Gauss-Jordan inverse.
// Flops: nb steps of (bw + 1)(bw + 2)/2 tile products for the factor and
// about nb^2 bw / 2 for V (about a tenth of the dense inverse at m = 3000,
// hb = 191), and the factor's serial chain is nb short steps of one cluster
// instead of nb multi-kernel panels.
constexpr int kLdlCluster = 8;   // CTAs of the factor's one thread-block cluster
constexpr int kLdlMaxBw = 8;     // widest block band factored (wider: dense inverse)
constexpr int kLdlLd = kGJ + 1;  // shared-memory tile row stride (odd: no bank conflicts)
constexpr int kVuCols = 16;      // columns of V per CTA of k_ldl_vu
static_assert(kLdlMaxBw <= kLdlCluster, "one L tile per CTA of the factor's cluster");

__device__ __forceinline__ void cluster_arrive() {
    __threadfence();  // this CTA's global writes are visible to the cluster's other CTAs
    asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}

__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory"); }

__device__ __forceinline__ void cluster_sync_all() {
    cluster_arrive();
    cluster_wait();
}

__device__ __forceinline__ unsigned cluster_rank() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
    return r;
}

// sT[r][c] = G[(r0 + r) * ld + c0 + c] (zero outside rows < rmax, cols < cmax);
// transposed: sT[c][r].  By the CTA's 256 threads, all sixteen loads of a
// thread issued before the first store.  Loads bypass L1: other CTAs of the
// cluster wrote these tiles during the kernel.
template <bool TRANS>
__device__ __forceinline__ void ldl_load_tile(double (*sT)[kLdlLd], const double *__restrict__ G, long ld, int r0,
                                              int c0, int rmax, int cmax) {
    constexpr int kPer = kGJ * kGJ / 256;
    double x[kPer];
#pragma unroll
    for (int t = 0; t < kPer; ++t) {
        const int v = threadIdx.x + 256 * t, r = v / kGJ, c = v % kGJ;
        x[t] = (r0 + r < rmax && c0 + c < cmax) ? __ldcg(G + (long)(r0 + r) * ld + c0 + c) : 0.0;
    }
#pragma unroll
    for (int t = 0; t < kPer; ++t) {
        const int v = threadIdx.x + 256 * t, r = v / kGJ, c = v % kGJ;
        if (TRANS) sT[c][r] = x[t];
        else sT[r][c] = x[t];
    }
}

// acc[u][v] = sum_q sX[ti + 16u][q] sY[q][tj + 16v]  (thread (ti, tj) of 16 x 16)
__device__ __forceinline__ void ldl_tile_product(const double (*sX)[kLdlLd], const double (*sY)[kLdlLd],
                                                 double (&acc)[4][4]) {
    const int ti = threadIdx.x / kGjT, tj = threadIdx.x % kGjT;
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = 0.0;
#pragma unroll 4
    for (int q = 0; q < kGJ; ++q) {
        double x[4], y[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) x[u] = sX[ti + kGjT * u][q];
#pragma unroll
        for (int v = 0; v < 4; ++v) y[v] = sY[q][tj + kGjT * v];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[u][v] = fma(x[u], y[v], acc[u][v]);
    }
}

// Update tile A_ij -= L_ik A_jk^T of step k (L_ik is tile a of step k's L
// tiles), by the CTA's 256 threads; the tile's old values are loaded before
// the product so their latency overlaps it.
__device__ __forceinline__ void ldl_update_tile(int m, int k, int bw, int a, int i, int j, double *__restrict__ A,
                                                const double *__restrict__ Lb, double (*sX)[kLdlLd],
                                                double (*sY)[kLdlLd]) {
    const int ti = threadIdx.x / kGjT, tj = threadIdx.x % kGjT;
    ldl_load_tile<false>(sX, Lb + ((long)k * bw + a) * kGJ * kGJ, kGJ, 0, 0, kGJ, kGJ);
    ldl_load_tile<true>(sY, A, m, kGJ * j, kGJ * k, m, m);
    double old[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int r = kGJ * i + ti + kGjT * u, c = kGJ * j + tj + kGjT * v;
            old[u][v] = (r < m && c < m) ? __ldcg(A + (long)r * m + c) : 0.0;
        }
    __syncthreads();
    double acc[4][4];
    ldl_tile_product(sX, sY, acc);
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int r = kGJ * i + ti + kGjT * u, c = kGJ * j + tj + kGjT * v;
            if (r < m && c < m) A[(long)r * m + c] = old[u][v] - acc[u][v];
        }
    __syncthreads();
}

// The factor: one cluster of kLdlCluster CTAs of kGjT^2 threads.  A (m x m,
// symmetric, band hb) is updated in place in its block-lower band; S_k go to
// Sb [nb][64][64], L_ik to Lb [nb][bw][64][64] (tile k + 1 + t at t).
// Step k: CTA t computes L tile t (one each: bw <= kLdlMaxBw = kLdlCluster);
// CTA 0 then goes on, without waiting for the others, to the next diagonal
// tile A_{k+1,k+1} -= L_{k+1,k} A_{k+1,k}^T (its own L tile) and that tile's
// inverse S_{k+1}, while CTAs 1.. wait for every L tile and update the rest
// of the trailing band; one cluster barrier ends the step.  The serial chain
// per step is one L tile, one update tile and one diagonal-block inverse.
__global__ void __cluster_dims__(kLdlCluster, 1, 1) __launch_bounds__(kGjT * kGjT)
    k_ldl_band(int m, int nb, int bw, double *__restrict__ A, double *__restrict__ Sb, double *__restrict__ Lb,
               const double *__restrict__ diag0) {
    extern __shared__ double ldl_sm[];
    double (*sX)[kLdlLd] = reinterpret_cast<double (*)[kLdlLd]>(ldl_sm);
    double (*sY)[kLdlLd] = reinterpret_cast<double (*)[kLdlLd]>(ldl_sm + kGJ * kLdlLd);
    __shared__ double srow[2][kGJ], scol[2][kGJ], sthr[kGJ], sd[2];
    const int rank = (int)cluster_rank();
    const int ti = threadIdx.x / kGjT, tj = threadIdx.x % kGjT;
    if (rank == 0) gj_block_inverse(m, 0, min(kGJ, m), A, Sb, diag0, srow, scol, sthr, sd);
    cluster_sync_all();
    for (int k = 0; k < nb; ++k) {
        const int j0 = kGJ * k;
        const double *Sk = Sb + (long)k * kGJ * kGJ;
        const int nl = min(bw, nb - 1 - k);
        if (nl == 0) break;  // the last step: nothing below the diagonal
        if (rank < nl) {  // L_ik = A_ik S_k, i = k + 1 + rank
            ldl_load_tile<false>(sX, A, m, kGJ * (k + 1 + rank), j0, m, m);
            ldl_load_tile<false>(sY, Sk, kGJ, 0, 0, kGJ, kGJ);
            __syncthreads();
            double acc[4][4];
            ldl_tile_product(sX, sY, acc);
            double *L = Lb + ((long)k * bw + rank) * kGJ * kGJ;
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) L[(ti + kGjT * u) * kGJ + tj + kGjT * v] = acc[u][v];
            __syncthreads();
        }
        cluster_arrive();  // the L tiles are written
        if (rank == 0) {
            // tile p = 0 (the next diagonal block) needs only CTA 0's own L tile
            ldl_update_tile(m, k, bw, 0, k + 1, k + 1, A, Lb, sX, sY);
            const int j1 = kGJ * (k + 1);
            gj_block_inverse(m, j1, min(kGJ, m - j1), A, Sb + (long)(k + 1) * kGJ * kGJ, diag0, srow, scol, sthr,
                             sd);
            cluster_wait();
        } else {
            cluster_wait();
            // update tiles p = a (a + 1) / 2 + b (b <= a < nl), p >= 1
            for (int p = rank; p < nl * (nl + 1) / 2; p += kLdlCluster - 1) {
                int a = 0;
                while ((a + 1) * (a + 2) / 2 <= p) ++a;
                const int b = p - a * (a + 1) / 2;
                ldl_update_tile(m, k, bw, a, k + 1 + a, k + 1 + b, A, Lb, sX, sY);
            }
        }
        cluster_sync_all();
    }
}

// V and U of the factor into F: CTA (block column j, strip s) walks block rows
// i = j .. nb-1 with the last bw + 1 blocks of its kVuCols columns of V in
// shared memory (FP64).  The tiles it multiplies form one sequence (for each
// i: L_il for l = max(j, i - bw) .. i - 1, then S_i); the next tile's loads
// are in flight while the current one is multiplied (two shared buffers).
__global__ void __launch_bounds__(256) k_ldl_vu(int m, int ldf, int nb, int bw, const double *__restrict__ Sb,
                                                const double *__restrict__ Lb, float *__restrict__ F) {
    extern __shared__ double vu_sm[];
    constexpr int SW = kGJ / kVuCols;  // strips per block column
    constexpr int kPer = kGJ * kGJ / 256;
    double (*ring)[kGJ][kVuCols + 1] = reinterpret_cast<double (*)[kGJ][kVuCols + 1]>(vu_sm + 2 * kGJ * kLdlLd);
    const int j = blockIdx.x / SW, s = blockIdx.x % SW, c0 = kGJ * j + kVuCols * s;
    if (j >= nb || c0 >= m) return;  // the whole CTA leaves together
    const int tr = threadIdx.x / kVuCols, tc = threadIdx.x % kVuCols;  // rows tr + 16 u, column tc
    const int R = bw + 1;
    for (int v = threadIdx.x; v < kGJ * kVuCols; v += blockDim.x) {  // V_jj = I
        const int r = v / kVuCols, c = v % kVuCols;
        ring[j % R][r][c] = r == kVuCols * s + c ? 1.0 : 0.0;
    }
    // tile (i, l): L_il for l < i, S_i for l == i
    auto tile = [&](int i, int l) -> const double * {
        return l < i ? Lb + ((long)l * bw + (i - l - 1)) * kGJ * kGJ : Sb + (long)i * kGJ * kGJ;
    };
    double x[kPer];
    auto fetch = [&](const double *G) {
#pragma unroll
        for (int t = 0; t < kPer; ++t) x[t] = G[threadIdx.x + 256 * t];
    };
    int i = j, l = j, buf = 0;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    fetch(tile(i, l));
    for (;;) {
#pragma unroll
        for (int t = 0; t < kPer; ++t) {
            const int v = threadIdx.x + 256 * t;
            vu_sm[buf * kGJ * kLdlLd + (v / kGJ) * kLdlLd + v % kGJ] = x[t];
        }
        __syncthreads();
        int ni = i, nl = l + 1;
        if (l == i) {
            ni = i + 1;
            nl = max(j, ni - bw);
        }
        const bool more = ni < nb;
        if (more) fetch(tile(ni, nl));  // in flight during this tile's product
        const double(*X)[kLdlLd] = reinterpret_cast<const double(*)[kLdlLd]>(vu_sm + buf * kGJ * kLdlLd);
        if (l < i) {  // acc += L_il V_lj
            const double(*Vl)[kVuCols + 1] = ring[l % R];
#pragma unroll 8
            for (int q = 0; q < kGJ; ++q) {
                const double y = Vl[q][tc];
#pragma unroll
                for (int u = 0; u < 4; ++u) acc[u] = fma(X[tr + 16 * u][q], y, acc[u]);
            }
        } else {
            if (i > j) {  // V_ij = -acc; the slot's last reader (V_{i-bw-1,j}) is done
#pragma unroll
                for (int u = 0; u < 4; ++u) ring[i % R][tr + 16 * u][tc] = -acc[u];
                __syncthreads();
            }
            const double(*Vi)[kVuCols + 1] = ring[i % R];
            double u4[4] = {0.0, 0.0, 0.0, 0.0};  // U_ij = S_i V_ij
#pragma unroll 8
            for (int q = 0; q < kGJ; ++q) {
                const double y = Vi[q][tc];
#pragma unroll
                for (int u = 0; u < 4; ++u) u4[u] = fma(X[tr + 16 * u][q], y, u4[u]);
            }
            const int col = c0 + tc;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int row = kGJ * i + tr + 16 * u;
                if (row < m && col < m) F[(long)row * ldf + col] = (float)u4[u];
                acc[u] = 0.0;
            }
            if (i > j)  // V_ij^T into the block-upper triangle, 64 consecutive floats per column of V
                for (int v = threadIdx.x; v < kGJ * kVuCols; v += blockDim.x) {
                    const int r = v % kGJ, cc = v / kGJ, row = kGJ * i + r;
                    if (row < m && c0 + cc < m) F[(long)(c0 + cc) * ldf + row] = (float)Vi[r][cc];
                }
        }
        if (!more) break;
        i = ni;
        l = nl;
        buf ^= 1;
    }
}

// Dot product of a row of F (16-byte aligned, ldf a multiple of 4) with v over
// columns [lo, hi), lo a multiple of 4: float4 loads, four in flight per lane,
// per-lane partial sums combined in a fixed order.
__device__ __forceinline__ float coarse_row_dot(const float *__restrict__ row, const float *__restrict__ v, int lo,
                                                int hi, int lane) {
    const float4 *r4 = reinterpret_cast<const float4 *>(row);
    const float4 *v4 = reinterpret_cast<const float4 *>(v);
    const int n4 = hi / 4;
    float s[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    int j = lo / 4 + lane;
    for (; j + 96 < n4; j += 128) {
        float4 a[4], x[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            a[u] = r4[j + 32 * u];
            x[u] = v4[j + 32 * u];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            s[u] = fmaf(a[u].x, x[u].x, fmaf(a[u].y, x[u].y, fmaf(a[u].z, x[u].z, fmaf(a[u].w, x[u].w, s[u]))));
    }
    for (; j < n4; j += 32) {
        const float4 a = r4[j], x = v4[j];
        s[0] = fmaf(a.x, x.x, fmaf(a.y, x.y, fmaf(a.z, x.z, fmaf(a.w, x.w, s[0]))));
    }
    for (int t = 4 * n4 + lane; t < hi; t += 32) s[0] = fmaf(row[t], v[t], s[0]);  // tail: hi = m, m % 4 != 0
    return warp_sum((s[0] + s[1]) + (s[2] + s[3]));
}

// z = U c: row r over the columns of its own and earlier blocks.
__global__ void __launch_bounds__(kBlock) k_coarse_apply_lower(int m, int ldf, const float *__restrict__ F,
                                                               const float *__restrict__ cvec,
                                                               float *__restrict__ z, const int *__restrict__ stop) {
    if (vc_stopped(stop)) return;
    const int lane = threadIdx.x & 31;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) / 32; i < m; i += gridDim.x * blockDim.x / 32) {
        const float s = coarse_row_dot(F + (long)i * ldf, cvec, 0, min(m, kGJ * (i / kGJ + 1)), lane);
        if (lane == 0) z[i] = s;
    }
}

// e = V^T z: z_r plus row r over the columns of later blocks.
__global__ void __launch_bounds__(kBlock) k_coarse_apply_upper(int m, int ldf, const float *__restrict__ F,
                                                               const float *__restrict__ z,
                                                               float *__restrict__ evec, const int *__restrict__ stop) {
    if (vc_stopped(stop)) return;
    const int lane = threadIdx.x & 31;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) / 32; i < m; i += gridDim.x * blockDim.x / 32) {
        const int lo = min(m, kGJ * (i / kGJ + 1));
        const float s = lo < m ? coarse_row_dot(F + (long)i * ldf, z, lo, m, lane) : 0.0f;
        if (lane == 0) evec[i] = z[i] + s;
    }
}

// The dense inverse V^T U from the factor (for the batched solver, which
// applies a dense inverse): entry (r, c) = [blk(r) >= blk(c)] F[r][c] +
// sum over q >= max(64 (blk(r) + 1), 64 blk(c)) of F[r][q] F[q][c].
__global__ void __launch_bounds__(kBlock) k_dense_from_factor(int m, int ldf, const float *__restrict__ F,
                                                              float *__restrict__ Einv) {
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < (long)m * m; e += (long)gridDim.x * blockDim.x) {
        const int r = (int)(e / m), c = (int)(e % m), br = r / kGJ, bc = c / kGJ;
        float s = br >= bc ? F[(long)r * ldf + c] : 0.0f;
        for (int q = kGJ * max(br + 1, bc); q < m; ++q) s = fmaf(F[(long)r * ldf + q], F[(long)q * ldf + c], s);
        Einv[e] = s;
    }
}

// hb: half-bandwidth of A (A_ik = 0 for |i - k| > hb).  Before panel J is
// processed, rows and columns beyond j0 + bb + hb are still untouched band
// (their entries in the panel's rows and columns are zero), so every step
// works on the leading (j0 + bb + hb)^2 window only: about a third of the
// dense work for a narrow band.
//
// Lookahead: of panel J's update only the next panel's rows and columns (the
// "cross") are needed by the next panel's diagonal, column and row steps, and
// those steps touch neither the rest of J's update nor its column panel P.
// So the update runs in two launches, the cross on the context's stream and
// the rest on a side stream, where it overlaps the next panel's three
// serial steps; P alternates between two buffers.  Every entry gets the
// same arithmetic as in order, so the inverse is the same.
static void invert_spd(ofea_ctx *c, double *A, int m, int hb) {
    Coarse &C = c->coarse;
    cudaStream_t s = c->stream;
    if (!c->side_stream) OFEA_CUDA(cudaStreamCreateWithFlags(&c->side_stream, cudaStreamNonBlocking));
    cudaStream_t s2 = c->side_stream;
    C.S.ensure(kGJ * kGJ);
    C.P.ensure(2 * (size_t)m * kGJ);
    C.diag0.ensure(m);
    k_diag_of<<<grid_for(c, m, kBlock), kBlock, 0, s>>>(m, A, C.diag0.p);
    OFEA_CHECK_LAUNCH();
    const size_t upd_smem = sizeof(double) * (64 * (kGJ + 1) + kGJ * 65);
    OFEA_CUDA(cudaFuncSetAttribute(k_gj_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)upd_smem));
    cudaEvent_t cross_done = nullptr, rest_done = nullptr;
    OFEA_CUDA(cudaEventCreateWithFlags(&cross_done, cudaEventDisableTiming));
    OFEA_CUDA(cudaEventCreateWithFlags(&rest_done, cudaEventDisableTiming));
    bool rest_pending = false;
    for (int j0 = 0, it = 0; j0 < m; j0 += kGJ, ++it) {
        const int bb = std::min(kGJ, m - j0);
        const int lim = (int)std::min<long>(m, (long)j0 + bb + hb);
        dim3 tiles((lim + 63) / 64, (lim + 63) / 64);
        double *P = C.P.p + (size_t)(it & 1) * m * kGJ;
        k_gj_diag<<<1, kGjT * kGjT, 0, s>>>(m, j0, bb, A, C.S.p, C.diag0.p);
        k_gj_panel<<<grid_for(c, (long)lim * 32, 256), 256, 0, s>>>(m, lim, j0, bb, A, C.S.p, P);
        k_gj_rows<<<std::max(1, std::min((lim + 31) / 32, c->num_sms * 4)), 256, 0, s>>>(m, lim, j0, bb, A, C.S.p);
        if (rest_pending) OFEA_CUDA(cudaStreamWaitEvent(s, rest_done, 0));  // the previous panel's update is complete
        if (j0 + bb < m) {
            const int cross = (j0 + bb) / 64;
            k_gj_update<<<2 * tiles.x - 1, 256, upd_smem, s>>>(m, lim, j0, bb, A, P, 1, cross);
            OFEA_CUDA(cudaEventRecord(cross_done, s));
            OFEA_CUDA(cudaStreamWaitEvent(s2, cross_done, 0));
            k_gj_update<<<tiles, 256, upd_smem, s2>>>(m, lim, j0, bb, A, P, 2, cross);
            OFEA_CUDA(cudaEventRecord(rest_done, s2));
            rest_pending = true;
        } else {
            k_gj_update<<<tiles, 256, upd_smem, s>>>(m, lim, j0, bb, A, P, 0, -1);
            rest_pending = false;
        }
    }
    OFEA_CHECK_LAUNCH();
    cudaEventDestroy(cross_done);
    cudaEventDestroy(rest_done);
}

// The block LDL^T factor of the banded A (block half-bandwidth bw <= kLdlMaxBw)
// and its FP32 apply array C.F32 (k_ldl_band, k_ldl_vu).
static void factor_band(ofea_ctx *c, double *A, int m, int bw) {
    Coarse &C = c->coarse;
    cudaStream_t s = c->stream;
    const int nb = (m + kGJ - 1) / kGJ;
    C.nbw = bw;
    C.Sb.ensure((size_t)nb * kGJ * kGJ);
    C.Lb.ensure(std::max<size_t>(1, (size_t)nb * bw * kGJ * kGJ));
    C.ldf = (m + 3) & ~3;  // rows 16-byte aligned for the apply's float4 loads
    C.F32.ensure((size_t)m * C.ldf);
    C.zvec.ensure(std::max(m, 1));
    C.diag0.ensure(m);
    k_diag_of<<<grid_for(c, m, kBlock), kBlock, 0, s>>>(m, A, C.diag0.p);
    OFEA_CHECK_LAUNCH();
    const int band_smem = (int)(sizeof(double) * 2 * kGJ * kLdlLd);
    OFEA_CUDA(cudaFuncSetAttribute(k_ldl_band, cudaFuncAttributeMaxDynamicSharedMemorySize, band_smem));
    k_ldl_band<<<kLdlCluster, kGjT * kGjT, band_smem, s>>>(m, nb, bw, A, C.Sb.p, C.Lb.p, C.diag0.p);
    OFEA_CHECK_LAUNCH();
    setup_mark(c, "coarse_ldl_band");
    const int vu_smem = (int)(sizeof(double) * (2 * kGJ * kLdlLd + (size_t)(bw + 1) * kGJ * (kVuCols + 1)));
    OFEA_CUDA(cudaFuncSetAttribute(k_ldl_vu, cudaFuncAttributeMaxDynamicSharedMemorySize, vu_smem));
    k_ldl_vu<<<nb * (kGJ / kVuCols), 256, vu_smem, s>>>(m, C.ldf, nb, bw, C.Sb.p, C.Lb.p, C.F32.p);
    OFEA_CHECK_LAUNCH();
    setup_mark(c, "coarse_ldl_vu");
}

void coarse_dense_inverse(ofea_ctx *c) {
    Coarse &C = c->coarse;
    if (!C.K_ok) fail(OFEA_ERR_STATE, "coarse level missing");
    if (C.dense_ok) return;
    const int m = C.m;
    C.Einv32.ensure((size_t)m * m);
    k_dense_from_factor<<<grid_for(c, (long)m * m, kBlock), kBlock, 0, c->stream>>>(m, C.ldf, C.F32.p, C.Einv32.p);
    OFEA_CHECK_LAUNCH();
    C.dense_ok = true;
}

// ----------------------------------------------------- lambda_max(D^-1 K) --

// w = Dinv32 K32 (v * sc), sc = 1/||v|| from the previous partials.
__global__ void __launch_bounds__(kBlock, 2048 / kBlock) k_power(int nfree, const int *__restrict__ sl_ptr,
                                                  const int *__restrict__ scols,
                                                  const int *__restrict__ sl_g, const __nv_bfloat16 *__restrict__ svg,
                                                  const float *__restrict__ Dinv32,
                                                  const float *__restrict__ v, float *__restrict__ w,
                                                  const double *__restrict__ Pin, int Gin,
                                                  double *__restrict__ Pout, int first) {
    __shared__ double sh[kWarpsPerBlock];
    double nrm2 = first ? 1.0 : sum_partials(Pin, Gin, sh);
    const float sc = (float)(1.0 / sqrt(nrm2));
    double acc = 0.0;
    for_each_sell_row(nfree, sl_ptr, [&](int r, long S, int t, int W) {
        float y[3];
        sell_row_g4(S, sl_g[r / kSlice], t, W, scols, svg, [&](int k) { return v[k] * sc; }, y[0], y[1], y[2]);
        float o[3];
        block3_apply(Dinv32 + 9L * r, y, o);
        for (int i = 0; i < 3; ++i) {
            w[3L * r + i] = o[i];
            acc += (double)o[i] * o[i];
        }
    });
    double s = block_sum(acc, sh);
    if (threadIdx.x == 0) Pout[blockIdx.x] = s;
}

__global__ void k_hash_vec(long n, float *v) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        unsigned h = (unsigned)(i * 2654435761u) ^ 0x9e3779b9u;
        h ^= h >> 15;
        h *= 2246822519u;
        h ^= h >> 13;
        v[i] = 0.5f + (float)(h & 0xffff) / 65536.0f;
    }
}

// lambda_max(D^-1 K) by `steps` power-iteration SpMVs, enqueued on stream a
// (buffers allocated first, on the host); lambda_max_read returns it once
// the context stream has waited for a.
static void lambda_max_launch(ofea_ctx *c, int steps, cudaStream_t a) {
    const int n = c->n;
    const int G = std::min(kMaxGrid, c->num_sms * (2048 / kBlock));
    Coarse &C = c->coarse;
    C.pw.ensure(2L * std::max(n, 1));
    C.pp.ensure(2L * kMaxGrid);
    float *v = C.pw.p, *w = C.pw.p + n;
    k_hash_vec<<<grid_for(c, n, kBlock), kBlock, 0, a>>>(n, v);
    for (int k = 0; k < steps; ++k) {
        double *Pin = C.pp.p + (k & 1) * kMaxGrid, *Pout = C.pp.p + ((k + 1) & 1) * kMaxGrid;
        k_power<<<G, kBlock, 0, a>>>(c->nfree, c->sl_ptr.p, c->scols.p, c->sl_g.p, c->sv16g.p, c->Dinv32.p, v, w,
                                     Pin, G, Pout, k == 0);
        std::swap(v, w);
    }
    OFEA_CHECK_LAUNCH();
}

static double lambda_max_read(ofea_ctx *c, int steps) {
    const int G = std::min(kMaxGrid, c->num_sms * (2048 / kBlock));
    std::vector<double> h(G);
    OFEA_CUDA(cudaMemcpyAsync(h.data(), c->coarse.pp.p + (steps & 1) * kMaxGrid, sizeof(double) * G,
                              cudaMemcpyDeviceToHost, c->stream));
    OFEA_CUDA(cudaStreamSynchronize(c->stream));
    double nrm2 = 0;
    for (double x : h) nrm2 += x;
    return std::sqrt(nrm2);
}

// ------------------------------------------------------------ setup entry --

void coarse_E_partials(ofea_ctx *c, Coarse &C, int nchunk) {
    if (nchunk != 1) fail(OFEA_ERR_STATE, "Galerkin blocks are assembled in one pass");
    C.part.ensure((size_t)C.na * 27 * 36);
    const int gsm_bytes = (int)(sizeof(double) * kGW * (27 * 36 + 32 * 18));
    OFEA_CUDA(cudaFuncSetAttribute(k_galerkin_blocks, cudaFuncAttributeMaxDynamicSharedMemorySize, gsm_bytes));
    k_galerkin_blocks<<<std::max(1, C.na), kGW * 32, gsm_bytes, c->stream>>>(
        C.na, C.agg_ptr.p, reinterpret_cast<const float4 *>(C.agg_off.p),
        reinterpret_cast<const float4 *>(C.row_off.p), C.row_cell.p, C.agg_cell.p, c->rowptr.p, c->cols.p, kblocks(c),
        C.part.p, c->err_flag.p);
    OFEA_CHECK_LAUNCH();
}

// The geometry of both levels depends on the mesh only: after the pattern it
// is built on a background host thread while the caller assembles K; every
// user of it joins the job first (a failure surfaces there).
// Device buffers the geometry job writes are released here, on the caller's
// thread, so that the job only allocates: a free waits for the whole device
// (dev_free), and a device-wide wait on a background thread would invalidate
// a CUDA graph that the caller's thread may be capturing at that moment (a
// PCG64 solve does not join the job).
static void release_geometry(Coarse &C) {
    for (DevBuf<int> *b : {&C.agg_of, &C.agg_ptr, &C.agg_nodes, &C.agg_cell, &C.cell_agg, &C.nbr, &C.nof}) b->release();
    C.centroid.release();
    C.agg_off.release();
    C.row_off.release();
    C.row_cell.release();
    C.geom_ok = C.K_ok = false;
}

void geometry_start(ofea_ctx *c) {
    geometry_join(c);
    release_geometry(c->coarse);
    release_geometry(c->coarse2);
    const int target = c->coarse_nodes;
    c->geom_job = std::async(std::launch::async, [c, target] {
        OFEA_CUDA(cudaSetDevice(c->device));
        c->coarse.target = target;
        build_aggregation(c, target);
        build_aggregation_fine(c);
    });
}

void geometry_join(ofea_ctx *c) {
    if (c->geom_job.valid()) c->geom_job.get();
}

void setup_coarse_geometry(ofea_ctx *c, int target_nodes) {
    geometry_join(c);
    Coarse &C = c->coarse;
    if (!C.geom_ok || C.target != target_nodes) {
        C.target = target_nodes;
        build_aggregation(c, target_nodes);
    }
}

double *coarse_begin_E(ofea_ctx *c) {
    Coarse &C = c->coarse;
    const int m = C.m;
    C.E.ensure((size_t)m * m);
    C.cvec.ensure(std::max(m, 1));
    C.evec.ensure(std::max(m, 1));
    OFEA_CUDA(cudaMemsetAsync(C.E.p, 0, sizeof(double) * m * m, c->stream));
    return C.E.p;
}

// The power iteration for the smoother's interval reads only K and D^-1: it
// runs on an auxiliary stream while the coarse inverse runs on the context
// stream (and its side stream), and is joined before its result is read.
void coarse_finish(ofea_ctx *c) {
    Coarse &C = c->coarse;
    cudaStream_t s = c->stream;
    const int m = C.m;
    constexpr int kPowerSteps = 10;
    if (!c->aux_stream) OFEA_CUDA(cudaStreamCreateWithFlags(&c->aux_stream, cudaStreamNonBlocking));
    cudaEvent_t fork = nullptr, join = nullptr;
    OFEA_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    OFEA_CUDA(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
    OFEA_CUDA(cudaEventRecord(fork, s));
    OFEA_CUDA(cudaStreamWaitEvent(c->aux_stream, fork, 0));
    lambda_max_launch(c, kPowerSteps, c->aux_stream);
    OFEA_CUDA(cudaEventRecord(join, c->aux_stream));
    const int hb = 6 * C.band + 5, nb = (m + kGJ - 1) / kGJ;
    const int bw = std::min(nb - 1, (hb + kGJ - 1) / kGJ);
    C.factored = c->coarse_solver == 0 && bw <= kLdlMaxBw;
    C.dense_ok = !C.factored;
    if (C.factored) {
        factor_band(c, C.E.p, m, bw);
    } else {
        invert_spd(c, C.E.p, m, hb);
        setup_mark(c, "coarse_inverse");
        C.Einv32.ensure((size_t)m * m);
        k_round_f32<<<grid_for(c, (long)m * m, kBlock), kBlock, 0, s>>>((long)m * m, C.E.p, C.Einv32.p);
        OFEA_CHECK_LAUNCH();
        setup_mark(c, "coarse_round_f32");
    }
    OFEA_CUDA(cudaStreamWaitEvent(s, join, 0));
    C.lmax = lambda_max_read(c, kPowerSteps);
    setup_mark(c, "lambda_max_join");
    cudaEventDestroy(fork);
    cudaEventDestroy(join);
    C.K_ok = true;
}

void setup_coarse(ofea_ctx *c, int target_nodes) {
    Coarse &C = c->coarse;
    setup_coarse_geometry(c, target_nodes);
    if (C.K_ok) return;
    cudaStream_t s = c->stream;
    const int m = C.m;
    coarse_begin_E(c);
    OFEA_CUDA(cudaMemsetAsync(c->err_flag.p, 0, sizeof(int), s));
    const int nchunk = 1;
    setup_mark(c, "geometry");
    coarse_E_partials(c, C, nchunk);
    setup_mark(c, "galerkin_level1");
    k_coarse_E_sum<<<grid_for(c, (long)C.na * 27 * 36, kBlock), kBlock, 0, s>>>(
        C.na, nchunk, C.agg_cell.p, C.cell_agg.p, C.nc[0], C.nc[1], C.nc[2], m, C.part.p, C.E.p);
    OFEA_CHECK_LAUNCH();
    OFEA_CUDA(cudaMemcpyAsync(c->herr.p, c->err_flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    OFEA_CUDA(cudaStreamSynchronize(s));
    if (c->herr.p[0]) fail(OFEA_ERR_CAPACITY, "coarse cells smaller than the element couplings");
    setup_mark(c, "coarse_E_sum");
    coarse_finish(c);
}

// ---------------------------------------------------------- V-cycle kernels --

// t = b - K32 x (x complete), per row.
__global__ void __launch_bounds__(kBlock, 2048 / kBlock) k_vc_resid(int nfree, const int *__restrict__ sl_ptr,
                                                     const int *__restrict__ scols,
                                                     const int *__restrict__ sl_g, const __nv_bfloat16 *__restrict__ svg,
                                                     const float *__restrict__ b,
                                                     const float *__restrict__ x, float *__restrict__ t,
                                                     const int *__restrict__ stop) {
    if (vc_stopped(stop)) return;
    for_each_sell_row(nfree, sl_ptr, [&](int r, long S, int tt, int W) {
        float y[3];
        sell_row_g4(S, sl_g[r / kSlice], tt, W, scols, svg, [&](int k) { return x[k]; }, y[0], y[1], y[2]);
        for (int i = 0; i < 3; ++i) t[3L * r + i] = b[3L * r + i] - y[i];
    });
}

// cvec_I = Z_I^T t (6 values per aggregate): one CTA of NT threads per
// aggregate, the rows' offsets and indices read in aggregate order (agg_off),
// sums in a fixed order (per thread, then warps).
template <int NT>
__global__ void __launch_bounds__(NT) k_restrict(int na, const int *__restrict__ agg_ptr,
                                                 const float4 *__restrict__ off, const float *__restrict__ t,
                                                 float *__restrict__ cvec, const int *__restrict__ stop) {
    constexpr int NW = NT / 32;
    __shared__ float sh[6][NW];
    if (vc_stopped(stop)) return;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int I = blockIdx.x; I < na; I += gridDim.x) {
        float a[6] = {0, 0, 0, 0, 0, 0};
        for (int idx = agg_ptr[I] + threadIdx.x; idx < agg_ptr[I + 1]; idx += NT) {
            const float4 o = off[idx];
            const int r = __float_as_int(o.w);
            const float dx = o.x, dy = o.y, dz = o.z;
            const float tx = t[3L * r], ty = t[3L * r + 1], tz = t[3L * r + 2];
            a[0] += tx;
            a[1] += ty;
            a[2] += tz;
            a[3] += -dz * ty + dy * tz;  // (e_x x d) . t
            a[4] += dz * tx - dx * tz;   // (e_y x d) . t
            a[5] += -dy * tx + dx * ty;  // (e_z x d) . t
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            a[k] = warp_sum(a[k]);
            if (lane == 0) sh[k][w] = a[k];
        }
        __syncthreads();
        if (threadIdx.x < 6) {
            float v = 0.f;
#pragma unroll
            for (int q = 0; q < NW; ++q) v += sh[threadIdx.x][q];
            cvec[6 * I + threadIdx.x] = v;
        }
        __syncthreads();
    }
}

// e = Einv32 c: one warp per row.
__global__ void __launch_bounds__(kBlock) k_coarse_gemv(int m, const float *__restrict__ Ainv,
                                                        const float *__restrict__ cvec,
                                                        float *__restrict__ evec, const int *__restrict__ stop) {
    if (vc_stopped(stop)) return;
    const int lane = threadIdx.x & 31;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) / 32; i < m; i += gridDim.x * blockDim.x / 32) {
        const float *row = Ainv + (long)i * m;
        float s = 0.0f;
        for (int j = lane; j < m; j += 32) s = fmaf(row[j], cvec[j], s);
        s = warp_sum(s);
        if (lane == 0) evec[i] = s;
    }
}

// x_r += Z_r e_I(r), per free row: the row's offset from its aggregate's
// centroid and the aggregate from row_off (one 16-byte load).
__global__ void k_prolong(int nfree, const float4 *__restrict__ roff, const float *__restrict__ evec,
                          float *__restrict__ x, const int *__restrict__ stop) {
    if (vc_stopped(stop)) return;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nfree; r += gridDim.x * blockDim.x) {
        const float4 o = roff[r];
        const int I = __float_as_int(o.w);
        const float dx = o.x, dy = o.y, dz = o.z;
        const float *e = evec + 6L * I;
        x[3L * r] += e[0] + dz * e[4] - dy * e[5];
        x[3L * r + 1] += e[1] - dz * e[3] + dx * e[5];
        x[3L * r + 2] += e[2] + dy * e[3] - dx * e[4];
    }
}

void restrict_level(ofea_ctx *c, const Coarse &C, const float *t, float *cvec) {
    const int g = std::min(C.na, c->num_sms * 16);
    const float4 *off = reinterpret_cast<const float4 *>(C.agg_off.p);
    // 128 threads for aggregates of a few hundred rows (the nested level), 256 beyond
    if (C.max_agg <= 512)
        k_restrict<128><<<g, 128, 0, c->stream>>>(C.na, C.agg_ptr.p, off, t, cvec, c->vc_stop);
    else
        k_restrict<256><<<g, 256, 0, c->stream>>>(C.na, C.agg_ptr.p, off, t, cvec, c->vc_stop);
    OFEA_CHECK_LAUNCH();
}

void prolong_level(ofea_ctx *c, const Coarse &C, const float *g, float *x) {
    k_prolong<<<grid_for(c, c->nfree, kBlock), kBlock, 0, c->stream>>>(
        c->nfree, reinterpret_cast<const float4 *>(C.row_off.p), g, x, c->vc_stop);
    OFEA_CHECK_LAUNCH();
}

void coarse_gemv(ofea_ctx *c, const float *cvec, float *evec) {
    Coarse &C = c->coarse;
    const int g = grid_for(c, (long)C.m * 32, kBlock);
    if (C.factored) {
        k_coarse_apply_lower<<<g, kBlock, 0, c->stream>>>(C.m, C.ldf, C.F32.p, cvec, C.zvec.p, c->vc_stop);
        k_coarse_apply_upper<<<g, kBlock, 0, c->stream>>>(C.m, C.ldf, C.F32.p, C.zvec.p, evec, c->vc_stop);
    } else {
        k_coarse_gemv<<<g, kBlock, 0, c->stream>>>(C.m, C.Einv32.p, cvec, evec, c->vc_stop);
    }
    OFEA_CHECK_LAUNCH();
}

void coarse_correct(ofea_ctx *c, const float *t, float *x) {
    Coarse &C = c->coarse;
    restrict_level(c, C, t, C.cvec.p);
    coarse_gemv(c, C.cvec.p, C.evec.p);
    prolong_level(c, C, C.evec.p, x);
}

void vc_resid(ofea_ctx *c, const float *b, const float *x, float *t) {
    k_vc_resid<<<grid_for(c, (c->nfree + 31) / 32, kWarpsPerBlock), kBlock, 0, c->stream>>>(
        c->nfree, c->sl_ptr.p, c->scols.p, c->sl_g.p, c->sv16g.p, b, x, t, c->vc_stop);
    OFEA_CHECK_LAUNCH();
}

}  // namespace ofea
