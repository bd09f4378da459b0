// Sparsity pattern of K on the device: the B200 replacement of
// assamble_stiffness::build_CSR (src/assemble.cpp:19-77).
//
// The reference inserts every (row, col) DOF pair of every element into a
// per-column std::set.  With whole-node constraints that pattern is the free
// node adjacency expanded to 3x3 blocks, so it is built here at node level:
//   1. node -> element incidence lists (counting sort + per-node sort, so the
//      result does not depend on atomic ordering);
//   2. one warp per free node collects the free nodes of its incident elements,
//      de-duplicates and ranks them in shared memory -> sorted block row;
//   3. the same pass writes the element-to-slot map: for incidence k (element g
//      seen from its local node a) and every local node b, the position of
//      node b in the row, which turns assembly into owner-computes gathers
//      with no atomics.
#include "ofea_internal.cuh"

namespace ofea {

// ------------------------------------------------------------------ scan --

__device__ __forceinline__ int warp_incl_scan(int v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Inclusive block scan of one value per thread (kBlock threads).
__device__ __forceinline__ int block_incl_scan(int v, int *sh /*[kWarpsPerBlock]*/, int *total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int s = warp_incl_scan(v);
    if (lane == 31) sh[warp] = s;
    __syncthreads();
    if (warp == 0) {
        int w = lane < kWarpsPerBlock ? sh[lane] : 0;
        w = warp_incl_scan(w);
        if (lane < kWarpsPerBlock) sh[lane] = w;
    }
    __syncthreads();
    if (warp > 0) s += sh[warp - 1];
    *total = sh[kWarpsPerBlock - 1];
    __syncthreads();
    return s;
}

constexpr int kScanItems = 4;  // per thread
constexpr int kScanTile = kBlock * kScanItems;

__global__ void __launch_bounds__(kBlock) k_scan_tiles(const int *__restrict__ in, int n,
                                                       int *__restrict__ tile_sums) {
    __shared__ int sh[kWarpsPerBlock];
    long base = (long)blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (base + k < n) s += in[base + k];
    int tot;
    block_incl_scan(s, sh, &tot);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

// Single CTA: exclusive scan of the tile sums in place; total -> tile_sums[nt].
__global__ void __launch_bounds__(kBlock) k_scan_sums(int *__restrict__ tile_sums, int nt) {
    __shared__ int sh[kWarpsPerBlock];
    int carry = 0;
    for (int b = 0; b < nt; b += kBlock) {
        int i = b + threadIdx.x;
        int v = i < nt ? tile_sums[i] : 0;
        int tot;
        int s = block_incl_scan(v, sh, &tot);
        if (i < nt) tile_sums[i] = carry + s - v;
        carry += tot;
    }
    if (threadIdx.x == 0) tile_sums[nt] = carry;
}

__global__ void __launch_bounds__(kBlock) k_scan_apply(const int *__restrict__ in, int n,
                                                       const int *__restrict__ tile_sums,
                                                       int *__restrict__ out) {
    __shared__ int sh[kWarpsPerBlock];
    long base = (long)blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    int v[kScanItems], s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < n ? in[base + k] : 0;
        s += v[k];
    }
    int tot;
    int incl = block_incl_scan(s, sh, &tot);
    int run = tile_sums[blockIdx.x] + incl - s;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = tile_sums[gridDim.x];
}

// out[0..n] = exclusive scan of in[0..n-1], out[n] = total.  d_tmp needs
// ceil(n / kScanTile) + 1 ints.  Returns the total (synchronises the stream).
long long exclusive_scan(const int *d_in, int *d_out, int n, cudaStream_t s, int *d_tmp,
                         int tmp_len) {
    int nt = (n + kScanTile - 1) / kScanTile;
    if (nt < 1) nt = 1;
    if (nt + 1 > tmp_len) fail(OFEA_ERR_INVALID_ARG, "scan scratch too small");
    k_scan_tiles<<<nt, kBlock, 0, s>>>(d_in, n, d_tmp);
    OFEA_CHECK_LAUNCH();
    k_scan_sums<<<1, kBlock, 0, s>>>(d_tmp, nt);
    OFEA_CHECK_LAUNCH();
    k_scan_apply<<<nt, kBlock, 0, s>>>(d_in, n, d_tmp, d_out);
    OFEA_CHECK_LAUNCH();
    int total = 0;
    OFEA_CUDA(cudaMemcpyAsync(&total, d_out + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    OFEA_CUDA(cudaStreamSynchronize(s));
    return total;
}

int grid_for(const ofea_ctx *c, long long work_items, int per_block) {
    long long g = (work_items + per_block - 1) / per_block;
    long long cap = (long long)c->num_sms * 16;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

// ------------------------------------------------------------- incidence --

// Visits every (element, local node) of both element types; g is the unified
// element id (hexes first).
template <class F>
__device__ __forceinline__ void for_each_corner(long i, int ne8, const int *topo8,
                                                const int *topo4, F f) {
    long n8 = 8L * ne8;
    if (i < n8) {
        f((int)(i >> 3), (int)(i & 7), topo8[i]);
    } else {
        long j = i - n8;
        f(ne8 + (int)(j >> 2), (int)(j & 3), topo4[j]);
    }
}

__global__ void k_count_incidence(long ncorner, int ne8, const int *__restrict__ topo8,
                                  const int *__restrict__ topo4, int *__restrict__ cnt) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < ncorner;
         i += (long)gridDim.x * blockDim.x)
        for_each_corner(i, ne8, topo8, topo4, [&](int, int, int node) { atomicAdd(&cnt[node], 1); });
}

__global__ void k_fill_incidence(long ncorner, int ne8, const int *__restrict__ topo8,
                                 const int *__restrict__ topo4, const int *__restrict__ inc_ptr,
                                 int *__restrict__ cursor, int *__restrict__ inc) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < ncorner;
         i += (long)gridDim.x * blockDim.x)
        for_each_corner(i, ne8, topo8, topo4, [&](int g, int a, int node) {
            int pos = inc_ptr[node] + atomicAdd(&cursor[node], 1);
            inc[pos] = g * 8 + a;
        });
}

// Sort each node's incidence list ascending (element id, then local index):
// the assembly sums contributions in this order, so K is bitwise reproducible.
__global__ void k_sort_incidence(int nd, const int *__restrict__ inc_ptr, int *__restrict__ inc) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nd; i += gridDim.x * blockDim.x) {
        int b = inc_ptr[i], e = inc_ptr[i + 1];
        for (int k = b + 1; k < e; ++k) {
            int v = inc[k], m = k - 1;
            while (m >= b && inc[m] > v) {
                inc[m + 1] = inc[m];
                --m;
            }
            inc[m + 1] = v;
        }
    }
}

__global__ void k_node_of_free(int nd, const int *__restrict__ free_map, int *__restrict__ nof) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nd; i += gridDim.x * blockDim.x) {
        int f = free_map[i];
        if (f >= 0) nof[f] = i;
    }
}

// ------------------------------------------------------------- adjacency --

constexpr int kCandCap = 512;  // candidate (element, node) pairs per free node

// One warp per free node r.  PASS 0: deg[r] = number of distinct free
// neighbours.  PASS 1: sorted columns, diagonal position and slot map.
template <int PASS>
__global__ void __launch_bounds__(kBlock) k_adjacency(
    int nfree, int ne8, const int *__restrict__ topo8, const int *__restrict__ topo4,
    const int *__restrict__ free_map, const int *__restrict__ node_of_free,
    const int *__restrict__ inc_ptr, const int *__restrict__ inc, int *__restrict__ deg,
    const int *__restrict__ rowptr, int *__restrict__ cols, int *__restrict__ diag_pos,
    uint16_t *__restrict__ slot, int *__restrict__ err, int *__restrict__ max_deg) {
    __shared__ int s_cand[kWarpsPerBlock][kCandCap];  // free index of candidate, -1 fixed
    __shared__ int s_where[kWarpsPerBlock][kCandCap]; // k*8+b of the candidate
    __shared__ bool s_first[kWarpsPerBlock][kCandCap];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int *cand = s_cand[warp];
    int *where = s_where[warp];
    bool *isfirst = s_first[warp];
    const int nwarps = gridDim.x * kWarpsPerBlock;
    for (int r = blockIdx.x * kWarpsPerBlock + warp; r < nfree; r += nwarps) {
        const int node = node_of_free[r];
        const int kb = inc_ptr[node], ke = inc_ptr[node + 1];
        // collect candidates (uniform loop over incidences)
        int m = 0;
        bool overflow = false;
        for (int k = kb; k < ke; ++k) {
            int g = inc[k] >> 3;
            int npe = g < ne8 ? 8 : 4;
            if (m + npe > kCandCap) {
                overflow = true;
                break;
            }
            if (lane < npe) {
                int nb = g < ne8 ? topo8[8L * g + lane] : topo4[4L * (g - ne8) + lane];
                cand[m + lane] = free_map[nb];
                where[m + lane] = k * 8 + lane;
            }
            m += npe;
        }
        __syncwarp();
        if (overflow) {
            if (lane == 0) {
                atomicExch(err, OFEA_ERR_CAPACITY);
                if (PASS == 0) deg[r] = 0;
            }
            continue;
        }
        // first occurrences, then ranks, by pairwise comparison (m is small:
        // 64 for a structured hex node, ~100 for a tet node)
        for (int c = lane; c < m; c += 32) {
            int v = cand[c];
            bool first = v >= 0;
            for (int o = 0; o < c && first; ++o) first = cand[o] != v;
            isfirst[c] = first;
        }
        __syncwarp();
        int my_unique = 0;
        for (int c = lane; c < m; c += 32) {
            int v = cand[c];
            bool first = isfirst[c];
            if (PASS == 0) {
                my_unique += first;
            } else {
                int rank = 0;
                for (int o = 0; o < m; ++o) rank += (isfirst[o] && cand[o] < v);
                int k = where[c] >> 3, b = where[c] & 7;
                slot[8L * k + b] = v >= 0 ? (uint16_t)rank : kNoSlot;
                if (first) cols[rowptr[r] + rank] = v;
                if (v == r && first) diag_pos[r] = rank;
            }
        }
        if (PASS == 0) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) my_unique += __shfl_xor_sync(0xffffffffu, my_unique, o);
            if (lane == 0) {
                deg[r] = my_unique;
                atomicMax(max_deg, my_unique);
                if (my_unique >= kNoSlot) atomicExch(err, OFEA_ERR_CAPACITY);
            }
        }
        __syncwarp();
    }
}

void build_pattern(ofea_ctx *c) {
    cudaStream_t s = c->stream;
    const long ncorner = 8L * c->ne8 + 4L * c->ne4;
    const int nd = c->nd, nfree = c->nfree;
    int tmp_len = (int)((std::max<long>(nd, nfree) + kScanTile - 1) / kScanTile) + 2;
    c->scratch_i.ensure((size_t)std::max(nd, nfree) + 1 + tmp_len);
    int *cnt = c->scratch_i.p;                 // nd (+1)
    int *tmp = c->scratch_i.p + std::max(nd, nfree) + 1;
    c->err_flag.ensure(4);
    OFEA_CUDA(cudaMemsetAsync(c->err_flag.p, 0, 4 * sizeof(int), s));

    // 1. incidence lists
    c->inc_ptr.ensure((size_t)nd + 1);
    c->inc.ensure((size_t)std::max<long>(ncorner, 1));
    OFEA_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * ((size_t)nd + 1), s));
    int g = grid_for(c, ncorner, kBlock);
    k_count_incidence<<<g, kBlock, 0, s>>>(ncorner, c->ne8, c->topo8.p, c->topo4.p, cnt);
    OFEA_CHECK_LAUNCH();
    exclusive_scan(cnt, c->inc_ptr.p, nd, s, tmp, tmp_len);
    OFEA_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * ((size_t)nd + 1), s));
    k_fill_incidence<<<g, kBlock, 0, s>>>(ncorner, c->ne8, c->topo8.p, c->topo4.p, c->inc_ptr.p,
                                          cnt, c->inc.p);
    OFEA_CHECK_LAUNCH();
    k_sort_incidence<<<grid_for(c, nd, kBlock), kBlock, 0, s>>>(nd, c->inc_ptr.p, c->inc.p);
    OFEA_CHECK_LAUNCH();
    c->node_of_free.ensure((size_t)std::max(nfree, 1));
    k_node_of_free<<<grid_for(c, nd, kBlock), kBlock, 0, s>>>(nd, c->free_map.p, c->node_of_free.p);
    OFEA_CHECK_LAUNCH();

    // 2. block rows: degrees, pointers
    int *deg = cnt;  // reuse (nfree entries)
    c->rowptr.ensure((size_t)nfree + 1);
    c->diag_pos.ensure((size_t)std::max(nfree, 1));
    c->slot.ensure((size_t)std::max<long>(8L * ncorner, 1));
    int gw = grid_for(c, nfree, kWarpsPerBlock);
    int *max_deg = c->err_flag.p + 1;
    k_adjacency<0><<<gw, kBlock, 0, s>>>(nfree, c->ne8, c->topo8.p, c->topo4.p, c->free_map.p,
                                         c->node_of_free.p, c->inc_ptr.p, c->inc.p, deg, nullptr,
                                         nullptr, nullptr, nullptr, c->err_flag.p, max_deg);
    OFEA_CHECK_LAUNCH();
    long long nnzb = exclusive_scan(deg, c->rowptr.p, nfree, s, tmp, tmp_len);
    c->herr.ensure(4);
    OFEA_CUDA(cudaMemcpyAsync(c->herr.p, c->err_flag.p, 4 * sizeof(int), cudaMemcpyDeviceToHost, s));
    OFEA_CUDA(cudaStreamSynchronize(s));
    if (c->herr.p[0] != 0)
        fail(OFEA_ERR_CAPACITY, "a node touches more than 512 element corners or has >= 65535 neighbours");
    if (nnzb * 9 >= (1LL << 31)) fail(OFEA_ERR_CAPACITY, "nnz exceeds the 32-bit index range");
    c->nnzb = nnzb;
    c->max_deg = c->herr.p[1];
    c->cols.ensure((size_t)std::max<long long>(nnzb, 1));
    // slot entries of rows owned by fixed nodes stay unused; clear for determinism.
    // diag_pos stays -1 for a free node that no element touches (empty row).
    OFEA_CUDA(cudaMemsetAsync(c->slot.p, 0xFF, sizeof(uint16_t) * 8 * (size_t)ncorner, s));
    OFEA_CUDA(cudaMemsetAsync(c->diag_pos.p, 0xFF, sizeof(int) * (size_t)std::max(nfree, 1), s));
    k_adjacency<1><<<gw, kBlock, 0, s>>>(nfree, c->ne8, c->topo8.p, c->topo4.p, c->free_map.p,
                                         c->node_of_free.p, c->inc_ptr.p, c->inc.p, nullptr,
                                         c->rowptr.p, c->cols.p, c->diag_pos.p, c->slot.p,
                                         c->err_flag.p, max_deg);
    OFEA_CHECK_LAUNCH();
    OFEA_CUDA(cudaStreamSynchronize(s));
    c->pattern_ok = true;
    c->K_ok = false;
    c->sell_ok = false;
    c->sell_layout_ok = false;
    c->se_state = 0;
    c->coarse.K_ok = false;  // the coarse geometry depends on the mesh alone: it stays
    c->coarse2.K_ok = false;
    c->learned.links_ok = false;
}

}  // namespace ofea
