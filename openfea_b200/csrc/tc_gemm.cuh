// Tensor-core (tcgen05) products of the learned stage's dense layers
// (tc_gemm.cu): D[m][n] = sum over k of A(m,k) B(n,k), BF16 operands, FP32
// accumulation.
#pragma once
#include <cuda_runtime.h>

namespace ofea {

// Element (row, k) of an FP32 operand at p[row * ms + k * ks].
struct TcOperand {
    const float *p;
    long ms, ks;
};

constexpr int kTcForward = 0;            // out[m][n] = D + bias[n], out2 = relu(out) when not null
constexpr int kTcRowMajor = 1;           // out[m][n] = D
constexpr int kTcTransposedPartial = 2;  // out[z * zstride + n * M + m] = D of reduction chunk z

struct TcEpilogue {
    int mode;
    float *out, *out2;
    const float *bias;
    long zstride;
};

// M x N outputs, reduction length Kred; with kchunk > 0 the reduction is
// split into chunks of kchunk (one partial per chunk, kTcTransposedPartial).
// err[0] is set to 1 when a wait inside the kernel ran out.
void tc_gemm(cudaStream_t s, int M, int N, long Kred, long kchunk, const TcOperand &A, const TcOperand &B,
             const TcEpilogue &epi, int *err);

}  // namespace ofea
