// Conversion of the assembled block-CSR K into the solver's BSELL-32 layout
// (sell.cuh): FP64 values, a BF16 copy in the same plane layout and a BF16
// copy grouped by four slots (sell_row_g4).  Runs once per assembly.
#include <algorithm>

#include "sell.cuh"

namespace ofea {

__global__ void k_slice_width(int nfree, const int *__restrict__ rowptr, int *__restrict__ width) {
    const int nslice = (nfree + kSlice - 1) / kSlice;
    const int lane = threadIdx.x & 31;
    for (int s = (blockIdx.x * blockDim.x + threadIdx.x) / 32; s < nslice;
         s += gridDim.x * blockDim.x / 32) {
        int r = s * kSlice + lane;
        int d = r < nfree ? rowptr[r + 1] - rowptr[r] : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) d = max(d, __shfl_xor_sync(0xffffffffu, d, o));
        if (lane == 0) width[s] = d;
    }
}

// Pattern part of the layout: the slots' block columns (padding: the row's
// own column, row 0 past the last row).  Once per pattern.
__global__ void k_fill_scols(int nfree, const int *__restrict__ rowptr, const int *__restrict__ cols,
                             const int *__restrict__ sl_ptr, int *__restrict__ scols) {
    const int nslice = (nfree + kSlice - 1) / kSlice;
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < (long)nslice * kSlice;
         g += (long)gridDim.x * blockDim.x) {
        const int s = (int)(g / kSlice), t = (int)(g % kSlice);
        const int r = s * kSlice + t;
        const long S = sl_ptr[s];
        const int W = sl_ptr[s + 1] - (int)S;
        const int rb = r < nfree ? rowptr[r] : 0;
        const int deg = r < nfree ? rowptr[r + 1] - rb : 0;
        for (int k = 0; k < W; ++k) scols[(S + k) * kSlice + t] = k < deg ? cols[rb + k] : (r < nfree ? r : 0);
    }
}

// Values: FP64 and BF16 planes, and the grouped BF16 copy, from block-CSR K.
__global__ void k_fill_sell(int nfree, const int *__restrict__ rowptr, const double *__restrict__ Kb,
                            const int *__restrict__ sl_ptr, double *__restrict__ sv64,
                            __nv_bfloat16 *__restrict__ sv16, const int *__restrict__ sl_g,
                            __nv_bfloat16 *__restrict__ svg) {
    const int nslice = (nfree + kSlice - 1) / kSlice;
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < (long)nslice * kSlice;
         g += (long)gridDim.x * blockDim.x) {
        const int s = (int)(g / kSlice), t = (int)(g % kSlice);
        const int r = s * kSlice + t;
        const long S = sl_ptr[s];
        const int W = sl_ptr[s + 1] - (int)S;
        const int rb = r < nfree ? rowptr[r] : 0;
        const int deg = r < nfree ? rowptr[r + 1] - rb : 0;
        const long G = sl_g[s];
        uint2 *svg2 = reinterpret_cast<uint2 *>(svg);
        for (int g = 0; g < (W + 3) / 4; ++g) {
            unsigned h[9][2] = {};  // the group's four BF16 values per plane, two per word
            for (int u = 0; u < 4; ++u) {
                const int k = 4 * g + u;
                const bool real = k < deg;
#pragma unroll
                for (int e = 0; e < 9; ++e) {
                    const double v = real ? Kb[9L * (rb + k) + e] : 0.0;
                    const __nv_bfloat16 bv = __double2bfloat16(v);
                    if (k < W) {
                        sv64[((S + k) * 9 + e) * kSlice + t] = v;
                        sv16[((S + k) * 9 + e) * kSlice + t] = bv;
                    }
                    h[e][u >> 1] |= (unsigned)__bfloat16_as_ushort(bv) << (16 * (u & 1));
                }
            }
#pragma unroll
            for (int e = 0; e < 9; ++e) svg2[((G + g) * 9 + e) * kSlice + t] = make_uint2(h[e][0], h[e][1]);
        }
    }
}

__global__ void k_group_width(int nslice, const int *__restrict__ sl_ptr, int *__restrict__ gw) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nslice; s += gridDim.x * blockDim.x)
        gw[s] = (sl_ptr[s + 1] - sl_ptr[s] + 3) / 4;
}

void build_sell_layout(ofea_ctx *c) {
    cudaStream_t s = c->stream;
    const int nslice = (c->nfree + kSlice - 1) / kSlice;
    c->sl_ptr.ensure((size_t)nslice + 1);
    int tmp_len = nslice / 1024 + 4;
    c->scratch_i.ensure((size_t)nslice + 1 + tmp_len);
    int *width = c->scratch_i.p;
    k_slice_width<<<grid_for(c, (long)nslice * 32, kBlock), kBlock, 0, s>>>(c->nfree, c->rowptr.p, width);
    OFEA_CHECK_LAUNCH();
    long long tot = exclusive_scan(width, c->sl_ptr.p, nslice, s, width + nslice + 1, tmp_len);
    c->sell_len = tot;
    size_t slots = (size_t)std::max<long long>(tot, 1) * kSlice;
    c->scols.ensure(slots);
    c->sv64.ensure(9 * slots);
    c->sv16.ensure(9 * slots);
    // slot groups of four per slice for the grouped BF16 copy
    c->sl_g.ensure((size_t)nslice + 1);
    k_group_width<<<grid_for(c, nslice, kBlock), kBlock, 0, s>>>(nslice, c->sl_ptr.p, width);
    OFEA_CHECK_LAUNCH();
    const long long groups = exclusive_scan(width, c->sl_g.p, nslice, s, width + nslice + 1, tmp_len);
    c->sv16g.ensure((size_t)std::max<long long>(groups, 1) * 9 * kSlice * 4);
    k_fill_scols<<<grid_for(c, (long)nslice * kSlice, kBlock), kBlock, 0, s>>>(c->nfree, c->rowptr.p, c->cols.p,
                                                                              c->sl_ptr.p, c->scols.p);
    OFEA_CHECK_LAUNCH();
    c->sell_layout_ok = true;
}

void build_sell(ofea_ctx *c) {
    if (!c->sell_layout_ok) build_sell_layout(c);
    cudaStream_t s = c->stream;
    const int nslice = (c->nfree + kSlice - 1) / kSlice;
    k_fill_sell<<<grid_for(c, (long)nslice * kSlice, kBlock), kBlock, 0, s>>>(
        c->nfree, c->rowptr.p, c->Kb.p, c->sl_ptr.p, c->sv64.p, c->sv16.p, c->sl_g.p, c->sv16g.p);
    OFEA_CHECK_LAUNCH();
    c->sell_ok = true;
    c->sv16_ok = true;
}

}  // namespace ofea
