// noalloc.cu -- residual RMS norms without any device allocation.
//
// Same quantity as the norms the engine records in its history (solverCalcRes, solver.c:867-892:
// res[k] = sqrt(sum_i R[k][i]^2 / Nelem)), for a caller that holds the residual in its own device memory
// and cannot let the library allocate: applications that give the solver a fixed device-memory budget
// managed by their own allocator, or that must not call cudaMalloc/cudaFree because those calls
// synchronize the device and would stall their other streams.
//
// The per-block partial sums live in a file-scope __device__ array (g_norm_scratch): every GPU that loads
// the library holds it (192 KiB) until the process exits. Host code reaches it only through the address
// returned by cudaGetSymbolAddress, looked up once per device on the first call made with that device
// current and cached for the life of the process: after a cudaDeviceReset the device's module is loaded
// again at another address, so the entry point must not be used across a device reset. Calls share the
// array: two calls whose kernels overlap on a GPU race on it. Each call writes every partial it later reads,
// so nothing has to be cleared between calls.
#include <cuda_runtime.h>
#include <math.h>
#include <mutex>
#include "csu_gpu.h"

extern "C" void csu_set_error(const char* fmt, ...);

namespace {

constexpr int NA_BLOCK = 256;                       // threads per block
constexpr int NA_PER_THREAD = 8;                    // cells per thread
constexpr int NA_CHUNK = NA_BLOCK * NA_PER_THREAD;  // cells per block
constexpr int NA_MAX_BLOCKS = 4096;                 // partial sums the scratch holds
constexpr int NA_MAX_VARS = 6;

static __device__ __align__(256) double g_norm_scratch[NA_MAX_BLOCKS * NA_MAX_VARS];

constexpr int NA_MAX_DEVICES = 64;
double* g_scratch_ptr[NA_MAX_DEVICES] = {nullptr};
std::mutex g_scratch_mu;

__device__ __forceinline__ double na_warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// partial sums of R^2 per variable over a contiguous chunk of cells
__global__ void __launch_bounds__(NA_BLOCK) k_norm_partial(const double* __restrict__ R, int nvar, int nc,
                                                           double* __restrict__ scratch)
{
    __shared__ double sh[NA_MAX_VARS][NA_BLOCK / 32];
    double acc[NA_MAX_VARS];
#pragma unroll
    for (int k = 0; k < NA_MAX_VARS; k++) acc[k] = 0.0;
    const int base = blockIdx.x * NA_CHUNK;
#pragma unroll
    for (int i = 0; i < NA_PER_THREAD; i++) {
        int c = base + i * NA_BLOCK + threadIdx.x;
        if (c < nc) {
#pragma unroll
            for (int k = 0; k < NA_MAX_VARS; k++) {
                if (k < nvar) {
                    double r = R[(size_t)k * nc + c];
                    acc[k] += r * r;
                }
            }
        }
    }
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NA_MAX_VARS; k++) {
        double v = na_warp_sum(acc[k]);
        if (lane == 0) sh[k][w] = v;
    }
    __syncthreads();
    if (threadIdx.x < nvar) {
        double s = 0.0;
        for (int j = 0; j < NA_BLOCK / 32; j++) s += sh[threadIdx.x][j];
        scratch[(size_t)blockIdx.x * NA_MAX_VARS + threadIdx.x] = s;
    }
}

// one block: sums the partials in a fixed order and writes the RMS norms
__global__ void __launch_bounds__(NA_BLOCK) k_norm_final(const double* __restrict__ scratch, int nblocks, int nvar,
                                                         int nc, double* __restrict__ res)
{
    __shared__ double sh[NA_MAX_VARS][NA_BLOCK / 32];
    double acc[NA_MAX_VARS];
#pragma unroll
    for (int k = 0; k < NA_MAX_VARS; k++) acc[k] = 0.0;
    int per = (nblocks + NA_BLOCK - 1) / NA_BLOCK;
    int lo = threadIdx.x * per, hi = min(nblocks, lo + per);
    for (int b = lo; b < hi; b++)
#pragma unroll
        for (int k = 0; k < NA_MAX_VARS; k++)
            if (k < nvar) acc[k] += scratch[(size_t)b * NA_MAX_VARS + k];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NA_MAX_VARS; k++) {
        double v = na_warp_sum(acc[k]);
        if (lane == 0) sh[k][w] = v;
    }
    __syncthreads();
    if (threadIdx.x < nvar) {
        double s = 0.0;
        for (int j = 0; j < NA_BLOCK / 32; j++) s += sh[threadIdx.x][j];
        res[threadIdx.x] = sqrt(s / nc);
    }
}

} // namespace

extern "C" int csu_residual_norms_noalloc(const double* R, int nvar, int ncells, double* res, void* stream)
{
    if (!R || !res || nvar < 1 || nvar > NA_MAX_VARS || ncells < 1) {
        csu_set_error("csu_residual_norms_noalloc: need device R and res, 1 <= nvar <= %d, ncells >= 1",
                      NA_MAX_VARS);
        return CSU_ERR_INPUT;
    }
    long long nblocks = ((long long)ncells + NA_CHUNK - 1) / NA_CHUNK;
    if (nblocks > NA_MAX_BLOCKS) {
        csu_set_error("csu_residual_norms_noalloc: %d cells exceed the limit of %d cells of its fixed scratch",
                      ncells, NA_MAX_BLOCKS * NA_CHUNK);
        return CSU_ERR_INPUT;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        csu_set_error("csu_residual_norms_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
        return CSU_ERR_NO_DEVICE;
    }
    if (dev < 0 || dev >= NA_MAX_DEVICES) {
        csu_set_error("csu_residual_norms_noalloc: device %d beyond the %d supported", dev, NA_MAX_DEVICES);
        return CSU_ERR_UNSUPPORTED;
    }
    double* scratch;
    {
        std::lock_guard<std::mutex> lock(g_scratch_mu);
        if (!g_scratch_ptr[dev]) {
            // host code may not use g_norm_scratch's own name as a device address
            e = cudaGetSymbolAddress((void**)&g_scratch_ptr[dev], g_norm_scratch);
            if (e != cudaSuccess) {
                g_scratch_ptr[dev] = nullptr;
                csu_set_error("csu_residual_norms_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
                return CSU_ERR_CUDA;
            }
        }
        scratch = g_scratch_ptr[dev];
    }
    // an error left by the caller's earlier work is reported as such, not as a failure of these launches
    e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        csu_set_error("csu_residual_norms_noalloc: an earlier CUDA error is pending: %s", cudaGetErrorString(e));
        return CSU_ERR_CUDA;
    }
    cudaStream_t s = (cudaStream_t)stream;
    k_norm_partial<<<(unsigned)nblocks, NA_BLOCK, 0, s>>>(R, nvar, ncells, scratch);
    k_norm_final<<<1, NA_BLOCK, 0, s>>>(scratch, (int)nblocks, nvar, ncells, res);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        csu_set_error("csu_residual_norms_noalloc: launch: %s", cudaGetErrorString(e));
        return CSU_ERR_CUDA;
    }
    return CSU_OK;
}
