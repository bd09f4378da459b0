// Coarse space and V-cycle of the two-level preconditioner (precond.cu).
#pragma once
#include "ofea_internal.cuh"

namespace ofea {

void build_aggregation(ofea_ctx *c, int target_nodes);
// Aggregation (once per mesh), E = Z^T K Z, its inverse and lambda_max(D^-1 K)
// (once per K).
void setup_coarse(ofea_ctx *c, int target_nodes);
// x += Z E^-1 Z^T t  (FP32 vectors of n entries)
void coarse_correct(ofea_ctx *c, const float *t, float *x);
// t = b - K32 x
void vc_resid(ofea_ctx *c, const float *b, const float *x, float *t);

}  // namespace ofea
