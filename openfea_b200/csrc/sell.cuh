// Sliced-ELL storage of the 3x3-block matrix (BSELL-32) and its SpMV row.
//
// Slice s holds block rows 32s .. 32s+31; its width W_s is the largest block
// count of those rows.  For slot k < W_s and lane t (row 32s+t):
//   column  scols[(S_s + k) * 32 + t]
//   entry e svals[((S_s + k) * 9 + e) * 32 + t]      e = 3 i + j of the 3x3 block
// with S_s = sl_ptr[s].  Rows shorter than W_s are padded with their own
// column and zero values.  One thread owns one block row (3 DOF rows): every
// value load of a warp is one coalesced 256 B (FP64) / 128 B (FP32) line, the
// 9 planes of a slot and several slots are in flight at once, and for
// structured node orderings neighbouring threads gather neighbouring x.
#pragma once
#include <type_traits>

#include "ofea_internal.cuh"

namespace ofea {

constexpr int kSlice = 32;

// Matrix values are stored as ST and used as V (BF16 storage, FP32 arithmetic).
template <class V, class ST>
__device__ __forceinline__ V sell_val(const ST *p) {
    if constexpr (std::is_same<ST, __nv_bfloat16>::value) return (V)__bfloat162float(__ldg(p));
    else return (V)__ldg(p);
}

// y_i (i = 0..2) of block row (slice base S, lane t, width W); x(k) returns
// entry k of the operand vector.
template <class V, int UNROLL, class XF, class ST = V>
__device__ __forceinline__ void sell_row(long S, int t, int W, const int *__restrict__ scols,
                                         const ST *__restrict__ svals, XF x, V &y0, V &y1, V &y2) {
    y0 = 0;
    y1 = 0;
    y2 = 0;
    const int *cp = scols + S * kSlice + t;
    const ST *vp = svals + S * 9 * kSlice + t;
    int k = 0;
    for (; k + UNROLL <= W; k += UNROLL) {
        int c[UNROLL];
        V v[UNROLL][9];
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
            c[u] = __ldg(cp + (long)(k + u) * kSlice);
#pragma unroll
            for (int e = 0; e < 9; ++e) v[u][e] = sell_val<V>(vp + ((long)(k + u) * 9 + e) * kSlice);
        }
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
            V x0 = x(3 * c[u]), x1 = x(3 * c[u] + 1), x2 = x(3 * c[u] + 2);
            y0 = fma(v[u][0], x0, fma(v[u][1], x1, fma(v[u][2], x2, y0)));
            y1 = fma(v[u][3], x0, fma(v[u][4], x1, fma(v[u][5], x2, y1)));
            y2 = fma(v[u][6], x0, fma(v[u][7], x1, fma(v[u][8], x2, y2)));
        }
    }
    for (; k < W; ++k) {
        int c = __ldg(cp + (long)k * kSlice);
        V v[9];
#pragma unroll
        for (int e = 0; e < 9; ++e) v[e] = sell_val<V>(vp + ((long)k * 9 + e) * kSlice);
        V x0 = x(3 * c), x1 = x(3 * c + 1), x2 = x(3 * c + 2);
        y0 = fma(v[0], x0, fma(v[1], x1, fma(v[2], x2, y0)));
        y1 = fma(v[3], x0, fma(v[4], x1, fma(v[5], x2, y1)));
        y2 = fma(v[6], x0, fma(v[7], x1, fma(v[8], x2, y2)));
    }
}

// The same row (FP32 arithmetic) from the grouped BF16 copy: slot groups of
// four, group g of slice s at G_s + g with G_s = sl_g[s]; for group g, plane
// e and lane t the four slots' values are side by side,
//   svg[(((G_s + g) * 9 + e) * 32 + t) * 4 + (k % 4)],
// zero beyond W.  One 4-byte load per plane brings two slots (the plane
// layout needs two 2-byte loads); the slots are summed in the same order and
// FMA nesting as sell_row<float, 4>, so the result is the same.
template <class XF>
__device__ __forceinline__ void sell_row_g4(long S, long G, int t, int W, const int *__restrict__ scols,
                                            const __nv_bfloat16 *__restrict__ svg, XF x, float &y0, float &y1,
                                            float &y2) {
    y0 = 0.f;
    y1 = 0.f;
    y2 = 0.f;
    const int *cp = scols + S * kSlice + t;
    const unsigned *vp = reinterpret_cast<const unsigned *>(svg) + (G * 9 * kSlice + t) * 2;
    for (int k = 0; k < W; k += 2) {  // k even: slots k, k + 1 are half (k / 2) & 1 of group k / 4
        const int c0 = __ldg(cp + (long)k * kSlice);
        const bool two = k + 1 < W;
        const int c1 = two ? __ldg(cp + (long)(k + 1) * kSlice) : 0;
        unsigned raw[9];
#pragma unroll
        for (int e = 0; e < 9; ++e) raw[e] = __ldg(vp + ((long)(k >> 2) * 9 + e) * kSlice * 2 + ((k >> 1) & 1));
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            if (u == 1 && !two) break;
            float v[9];
#pragma unroll
            for (int e = 0; e < 9; ++e)  // BF16 -> FP32 is exact
                v[e] = __uint_as_float(u ? (raw[e] & 0xFFFF0000u) : (raw[e] << 16));
            const int c = u ? c1 : c0;
            const float x0 = x(3 * c), x1 = x(3 * c + 1), x2 = x(3 * c + 2);
            y0 = fmaf(v[0], x0, fmaf(v[1], x1, fmaf(v[2], x2, y0)));
            y1 = fmaf(v[3], x0, fmaf(v[4], x1, fmaf(v[5], x2, y1)));
            y2 = fmaf(v[6], x0, fmaf(v[7], x1, fmaf(v[8], x2, y2)));
        }
    }
}

// Iterate over this thread's block rows: f(r, S, t, W) for each row r < nfree.
template <class F>
__device__ __forceinline__ void for_each_sell_row(int nfree, const int *__restrict__ sl_ptr, F f) {
    const int nslice = (nfree + kSlice - 1) / kSlice;
    const int t = threadIdx.x & (kSlice - 1);
    const int slices_per_cta = blockDim.x / kSlice;
    for (int s = blockIdx.x * slices_per_cta + (threadIdx.x / kSlice); s < nslice;
         s += gridDim.x * slices_per_cta) {
        const int r = s * kSlice + t;
        if (r >= nfree) continue;
        const int S = sl_ptr[s], W = sl_ptr[s + 1] - S;
        f(r, (long)S, t, W);
    }
}

// Read access to block (r, k) of K: block CSR when it is current, else the
// FP64 BSELL copy (all a fused assembly writes).
struct KBlocks {
    const double *Kb;  // null: read sv64
    const int *rowptr, *sl_ptr;
    const double *sv64;
    __device__ __forceinline__ double at(int r, int k, int e) const {
        if (Kb) return Kb[9L * (rowptr[r] + k) + e];
        return sv64[((long)(sl_ptr[r / kSlice] + k) * 9 + e) * kSlice + (r % kSlice)];
    }
};

inline KBlocks kblocks(const ofea_ctx *c) {
    return KBlocks{c->kb_ok ? c->Kb.p : nullptr, c->rowptr.p, c->sl_ptr.p, c->sv64.p};
}

void build_sell(ofea_ctx *c);

}  // namespace ofea
