// K handed over already assembled, as the reference's solution_api receives it
// (src/linear_solution.cpp:17-64): the CSC arrays col_idx_ (n+1 column
// pointers), row_idx_ (sorted row ids) and nz_val_ of assamble_stiffness
// (src/include/assemble.h:41-43), or col_idx / row_idx / nz_val of
// assamble_nl_stiffness for the Newton tangent.
//
// K is symmetric, so column j of the CSC arrays is row j.  Every free node has
// all three DOFs free (whole-node boundary conditions, src/set_bc.cpp:20-43)
// and build_CSR inserts every DOF pair of an element, so the scalar pattern is
// the 3x3 block pattern expanded: scalar column 3I+r lists, for each block
// neighbour J of node I in ascending order, the rows 3J, 3J+1, 3J+2.  One warp
// per block row checks that structure and writes the block-CSR pattern and
// the block-row-major values the solver reads; a violation sets a flag and
// the upload fails.
#include "ofea_internal.cuh"

namespace ofea {

long long exclusive_scan(const int *d_in, int *d_out, int n, cudaStream_t s, int *d_tmp, int tmp_len);

namespace {

// err[0] = 1: a column is not 3x3-block structured; err[1]: maximum block degree.
__global__ void __launch_bounds__(kBlock) k_csc_to_blocks(int nfree, const int *__restrict__ col_ptr,
                                                          const int *__restrict__ row_idx,
                                                          const double *__restrict__ val,
                                                          int *__restrict__ rowptr, int *__restrict__ cols,
                                                          int *__restrict__ diag_pos, double *__restrict__ Kb,
                                                          int *__restrict__ err) {
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * kWarpsPerBlock;
    for (int I = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5); I < nfree; I += warps) {
        const int c0 = col_ptr[3 * I], c1 = col_ptr[3 * I + 1], c2 = col_ptr[3 * I + 2], c3 = col_ptr[3 * I + 3];
        const int len = c1 - c0;
        bool bad = (len % 3) != 0 || (c2 - c1) != len || (c3 - c2) != len || (c0 % 9) != 0;
        if (__any_sync(0xffffffffu, bad)) {
            if (lane == 0) atomicExch(err, 1);
            continue;
        }
        const int nb = len / 3, base = c0 / 9;
        if (lane == 0) {
            rowptr[I] = base;
            if (I == nfree - 1) rowptr[nfree] = c3 / 9;
            atomicMax(err + 1, nb);
        }
        // block columns: ascending, in range, the same three rows in all three columns
        for (int b = lane; b < nb; b += 32) {
            const int r0 = row_idx[c0 + 3 * b];
            const int J = r0 / 3;
            bool ok = r0 >= 0 && (r0 % 3) == 0 && J < nfree;
            if (ok && b > 0) ok = row_idx[c0 + 3 * b - 3] < r0;
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int k = 0; k < 3; ++k) ok = ok && row_idx[col_ptr[3 * I + r] + 3 * b + k] == r0 + k;
            if (!ok) atomicExch(err, 1);
            cols[base + b] = J;
            if (J == I) diag_pos[I] = b;
        }
        // values: block b, entry (r, k) = K(3I + r, 3J + k) = column 3I + r, row 3J + k
        double *out = Kb + 9L * base;
        for (int t = lane; t < 9 * nb; t += 32) {
            const int b = t / 9, rk = t - 9 * b, r = rk / 3, k = rk - 3 * r;
            out[t] = val[col_ptr[3 * I + r] + 3 * b + k];
        }
    }
}

__global__ void k_free_nodes(int nd, const int *__restrict__ free_map, int *__restrict__ nof) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nd; i += gridDim.x * blockDim.x) {
        const int f = free_map[i];
        if (f >= 0) nof[f] = i;
    }
}

}  // namespace

void upload_csc(ofea_ctx *c, int n, const int *col_ptr, const int *row_idx, const double *val) {
    cudaStream_t s = c->stream;
    const int nf = c->nfree;
    const long long nnz = col_ptr[n];
    // scratch copies of the caller's arrays (from the device cache; freed at return)
    DevBuf<int> dcp, dri;
    DevBuf<double> dval;
    dcp.upload(col_ptr, (size_t)n + 1, s);
    dri.upload(row_idx, (size_t)std::max<long long>(nnz, 1), s);
    dval.upload(val, (size_t)std::max<long long>(nnz, 1), s);
    const long long nnzb = nnz / 9;
    c->rowptr.ensure((size_t)nf + 1);
    c->cols.ensure((size_t)std::max<long long>(nnzb, 1));
    c->diag_pos.ensure((size_t)std::max(nf, 1));
    c->Kb.ensure((size_t)std::max<long long>(9 * nnzb, 1));
    c->node_of_free.ensure((size_t)std::max(nf, 1));
    OFEA_CUDA(cudaMemsetAsync(c->diag_pos.p, 0xFF, sizeof(int) * (size_t)std::max(nf, 1), s));
    OFEA_CUDA(cudaMemsetAsync(c->err_flag.p, 0, 4 * sizeof(int), s));
    k_csc_to_blocks<<<grid_for(c, nf, kWarpsPerBlock), kBlock, 0, s>>>(nf, dcp.p, dri.p, dval.p, c->rowptr.p,
                                                                       c->cols.p, c->diag_pos.p, c->Kb.p,
                                                                       c->err_flag.p);
    OFEA_CHECK_LAUNCH();
    k_free_nodes<<<grid_for(c, c->nd, kBlock), kBlock, 0, s>>>(c->nd, c->free_map.p, c->node_of_free.p);
    OFEA_CHECK_LAUNCH();
    OFEA_CUDA(cudaMemcpyAsync(c->herr.p, c->err_flag.p, 4 * sizeof(int), cudaMemcpyDeviceToHost, s));
    OFEA_CUDA(cudaStreamSynchronize(s));
    if (c->herr.p[0] != 0)
        fail(OFEA_ERR_INVALID_ARG,
             "K is not 3x3-block structured (every free node's three columns must list the same "
             "block rows, each as three consecutive rows, ascending)");
    c->nnzb = nnzb;
    c->max_deg = c->herr.p[1];
}

}  // namespace ofea
