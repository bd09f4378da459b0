// Coarse space and V-cycle of the two-level preconditioner (precond.cu).
#pragma once
#include "ofea_internal.cuh"

namespace ofea {

// A V-cycle kernel launched among a solve's iterations returns at once when
// the solve has stopped (the iterations a chunk runs past convergence cost
// only their launches).  stop is null outside a solve.  Read once per CTA and
// broadcast: every thread takes the same path before any barrier.
__device__ __forceinline__ bool vc_stopped(const int *stop) {
    if (stop == nullptr) return false;
    __shared__ int s_stop;
    if (threadIdx.x == 0) s_stop = *(volatile const int *)stop;
    __syncthreads();
    return s_stop != 0;
}

void build_aggregation(ofea_ctx *c, int target_nodes);
void build_aggregation_fine(ofea_ctx *c);
// Aggregation (once per mesh), E = Z^T K Z, its inverse and lambda_max(D^-1 K)
// (once per K).
void setup_coarse(ofea_ctx *c, int target_nodes);
// The same in parts: the aggregation only; a zeroed dense E to fill (returns
// it); inversion, FP32 copy and lambda_max of a filled E.
void setup_coarse_geometry(ofea_ctx *c, int target_nodes);
double *coarse_begin_E(ofea_ctx *c);
void coarse_finish(ofea_ctx *c);
// Damping weight of the block-Jacobi smoother (needs setup_coarse's lmax).
float smoother_weight(const ofea_ctx *c, double damping);
// omega lmax of the single-matrix solves and of the batched solver, each the
// value that took the fewest outer iterations on its workload: the 1.56M-DOF
// cantilever, LEARNED / MIXED, 1.3: 51 / 69, 1.4: 51 / 67, 1.5: 51 / 65,
// 1.6: 52 / 64, 1.76: 56 / 71, 1.9: MIXED does not converge; the 64 SIMP
// variants of the batched reanalysis, 1.4: 86, 1.5: 83, 1.6: 81, 1.76: 78.
constexpr double kSmootherDamping = 1.5;
constexpr double kBatchSmootherDamping = 1.76;
// x += Z E^-1 Z^T t  (FP32 vectors of n entries)
// evec = E^-1 cvec (FP32 GEMV with the coarse level's inverse)
void coarse_gemv(ofea_ctx *c, const float *cvec, float *evec);
// Einv32 = the dense FP32 inverse of E (formed from the factor when the
// coarse solve is factored); for the batched solver, which applies it densely.
void coarse_dense_inverse(ofea_ctx *c);
void coarse_correct(ofea_ctx *c, const float *t, float *x);
// t = b - K32 x
void vc_resid(ofea_ctx *c, const float *b, const float *x, float *t);
// Level-generic pieces (also used by the learned level):
// cvec = Z^T t, x += Z g, and the Galerkin blocks of Z^T K Z into C.part
// ([aggregate][27 neighbour slots][6 x 6]; nchunk must be 1).
void restrict_level(ofea_ctx *c, const Coarse &C, const float *t, float *cvec);
void prolong_level(ofea_ctx *c, const Coarse &C, const float *g, float *x);
void coarse_E_partials(ofea_ctx *c, Coarse &C, int nchunk);

}  // namespace ofea
