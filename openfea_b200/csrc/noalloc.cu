// Residual norms computed without allocating any device memory.
//
// Some callers cannot let a library allocate: applications that reserve the
// whole GPU memory up front for their own pool allocator, and latency-critical
// loops in which cudaMalloc / cudaFree are unacceptable because they may
// synchronize the device.  For them ofea_residual_norms_noalloc() computes
// ||f - K u||_2 and ||f||_2 for up to kMaxRhs load cases using only the
// caller's buffers, the context's assembled K, and the file-scope scratch
// array below for the per-CTA partial sums.
//
// The scratch array (kMaxRhs * 2 * kMaxCtas doubles = 512 KB) exists on every
// GPU that loads this library, for as long as the process lives.  Its device
// address is looked up, and the two kernels loaded, when a context is created
// on a device (noalloc_prepare), so the entry point allocates nothing.  Every call
// shares it and it keeps the last call's contents; each call overwrites every
// partial it later reads, so nothing needs clearing.  Calls whose work
// overlaps on the same GPU (other streams or contexts of the device) race on
// the array: the caller must order them.
#include <algorithm>
#include <mutex>

#include "sell.cuh"
#include "solver_common.cuh"

namespace ofea {
namespace {

constexpr int kMaxRhs = 16;     // load cases per call
constexpr int kMaxCtas = 2048;  // CTAs of the partial-sum kernel
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_residual_scratch[kMaxRhs * 2 * kMaxCtas];

// Device address of g_residual_scratch per device, looked up once per device.
std::mutex g_mu;
double *g_scratch_addr[kMaxDevices] = {};

double *scratch_address(int device) {
    if (device < 0 || device >= kMaxDevices) fail(OFEA_ERR_INVALID_ARG, "device index too large");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_residual_scratch);
        if (e != cudaSuccess) fail_cuda(e, "cudaGetSymbolAddress(g_residual_scratch)", __FILE__, __LINE__);
        g_scratch_addr[device] = static_cast<double *>(p);
    }
    return g_scratch_addr[device];
}

// Partials of ||f - K u||^2 and ||f||^2 of load case blockIdx.y.
__global__ void __launch_bounds__(kBlock) k_residual_partials(
    int nfree, long n, const int *__restrict__ sl_ptr, const int *__restrict__ scols,
    const double *__restrict__ sv64, const double *__restrict__ F, const double *__restrict__ U,
    double *__restrict__ scratch) {
    __shared__ double sh[kWarpsPerBlock];
    const double *f = F + n * blockIdx.y;
    const double *u = U + n * blockIdx.y;
    double prr = 0, pff = 0;
    for_each_sell_row(nfree, sl_ptr, [&](int rw, long S, int t, int W) {
        double y[3];
        sell_row<double, 2>(S, t, W, scols, sv64, [&](int k) { return u[k]; }, y[0], y[1], y[2]);
        for (int i = 0; i < 3; ++i) {
            const double fi = f[3L * rw + i];
            const double rv = fi - y[i];
            prr += rv * rv;
            pff += fi * fi;
        }
    });
    const double a = block_sum(prr, sh);
    const double b = block_sum(pff, sh);
    if (threadIdx.x == 0) {
        scratch[(2L * blockIdx.y) * kMaxCtas + blockIdx.x] = a;
        scratch[(2L * blockIdx.y + 1) * kMaxCtas + blockIdx.x] = b;
    }
}

// One CTA per load case: fixed-order sums of the partials, square roots.
__global__ void __launch_bounds__(kBlock) k_residual_final(int G, const double *__restrict__ scratch,
                                                           double *__restrict__ norms) {
    __shared__ double sh[kWarpsPerBlock];
    const int k = blockIdx.x;
    const double rr = sum_partials(scratch + 2L * k * kMaxCtas, G, sh);
    const double ff = sum_partials(scratch + (2L * k + 1) * kMaxCtas, G, sh);
    if (threadIdx.x == 0) {
        norms[2 * k] = sqrt(rr);
        norms[2 * k + 1] = sqrt(ff);
    }
}

}  // namespace

// Looks up the scratch array's address on `device` and loads the entry
// point's two kernels there (CUDA loads modules and kernels lazily, which
// allocates device memory); run when a context is created on that device, so
// the entry point itself allocates nothing, from its first call on.
void noalloc_prepare(int device) {
    scratch_address(device);
    cudaFuncAttributes a;
    OFEA_CUDA(cudaFuncGetAttributes(&a, k_residual_partials));
    OFEA_CUDA(cudaFuncGetAttributes(&a, k_residual_final));
}

void residual_norms_noalloc(ofea_ctx *c, int nrhs, const double *d_f, const double *d_u,
                            double *d_norms) {
    if (nrhs < 1 || nrhs > kMaxRhs)
        fail(OFEA_ERR_CAPACITY, "ofea_residual_norms_noalloc takes 1 to " + std::to_string(kMaxRhs) +
                                    " load cases per call, got " + std::to_string(nrhs));
    double *scratch = scratch_address(c->device);
    // the same CTA count and row order as the solver's residual kernels
    const int G = std::min(kMaxCtas, std::min(kMaxGrid, c->num_sms * (2048 / kBlock)));
    k_residual_partials<<<dim3(G, nrhs), kBlock, 0, c->stream>>>(c->nfree, (long)c->n, c->sl_ptr.p,
                                                                   c->scols.p, c->sv64.p, d_f, d_u, scratch);
    OFEA_CHECK_LAUNCH();
    k_residual_final<<<nrhs, kBlock, 0, c->stream>>>(G, scratch, d_norms);
    OFEA_CHECK_LAUNCH();
}

}  // namespace ofea
