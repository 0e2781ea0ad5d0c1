// Residual norm of a 7-point operator that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code that runs while a host
// application is recording a CUDA graph of its own, solvers embedded under a
// fixed device-memory budget that the host application owns, or plugins that
// must not change the device heap of the program that loads them.  For them
// this entry point takes every input and output from the caller and keeps its
// only scratch -- one partial sum per thread block plus a completion counter
// -- in a file-scope device array that is part of the library image.  Every
// GPU that loads the library holds that array (about 32 KiB) until the
// process exits.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/lsstag_b200.h"

namespace {

constexpr int kBlock = 256;
constexpr int kCellsPerThread = 16;
constexpr long long kCellsPerBlock = (long long)kBlock * kCellsPerThread;
constexpr int kMaxBlocks = 4096;                       // scratch slots
constexpr long long kMaxCells = kCellsPerBlock * kMaxBlocks;   // 16,777,216 cells (256^3)
constexpr int kMaxDevices = 64;

// scratch: kMaxBlocks partial sums, then the completion counter
__device__ __align__(256) double g_noalloc_scratch[kMaxBlocks + 32];

struct DeviceSlot {
    bool ready = false;
    double* scratch = nullptr;   // device address of g_noalloc_scratch on that device
};
DeviceSlot g_slots[kMaxDevices];
std::mutex g_slots_mutex;

__global__ void __launch_bounds__(kBlock) k_residual_norm_noalloc(int N, int M, int K, const double* __restrict__ planes,
                                                                   const double* __restrict__ x,
                                                                   const double* __restrict__ b,
                                                                   double* __restrict__ r, double* scratch,
                                                                   double* norm2)
{
    const long long n = (long long)N * M * K;
    const long long NM = (long long)N * M;
    const long long base = (long long)blockIdx.x * kCellsPerBlock;
    double s = 0.0;
    for (int k = 0; k < kCellsPerThread; k++) {
        const long long i = base + (long long)k * kBlock + threadIdx.x;
        if (i >= n) break;
        const int iz = (int)(i / NM);
        const long long rem = i - (long long)iz * NM;
        const int iy = (int)(rem / N);
        const int ix = (int)(rem - (long long)iy * N);
        double acc = planes[3 * n + i] * x[i];
        if (iz > 0) acc += planes[i] * x[i - NM];
        if (iy > 0) acc += planes[n + i] * x[i - N];
        if (ix > 0) acc += planes[2 * n + i] * x[i - 1];
        if (ix < N - 1) acc += planes[4 * n + i] * x[i + 1];
        if (iy < M - 1) acc += planes[5 * n + i] * x[i + N];
        if (iz < K - 1) acc += planes[6 * n + i] * x[i + NM];
        const double v = b[i] - acc;
        if (r) r[i] = v;
        s += v * v;
    }
    // block sum, then the last block adds the partials in block order
    __shared__ double sh[kBlock / 32];
    __shared__ bool last;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    unsigned int* counter = (unsigned int*)(scratch + kMaxBlocks);
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kBlock / 32; w++) t += sh[w];
        scratch[blockIdx.x] = t;
        __threadfence();
        last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double acc = 0.0;
    for (int bk = threadIdx.x; bk < (int)gridDim.x; bk += kBlock) acc += ((volatile double*)scratch)[bk];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kBlock / 32; w++) t += sh[w];
        *norm2 = t;
        *counter = 0u;
    }
}

}  // namespace

extern "C" int lsg_residual_norm_noalloc(int N, int M, int K, const double* planes, const double* x,
                                         const double* b, double* r, double* norm2, void* stream)
{
    if (N < 1 || M < 1 || K < 1 || !planes || !x || !b || !norm2) return LSG_ERR_ARG;
    // compare before multiplying all three: N*M*K of three large ints can
    // overflow 64 bits, M*K (< 2^62) cannot
    const long long MK = (long long)M * K;
    if (MK > kMaxCells || (long long)N > kMaxCells / MK) {
        fprintf(stderr,
                "lsg_residual_norm_noalloc: a %d x %d x %d grid exceeds the fixed scratch capacity of %lld cells "
                "(%d blocks of %lld cells)\n",
                N, M, K, kMaxCells, kMaxBlocks, kCellsPerBlock);
        return LSG_ERR_ARG;
    }
    const long long n = (long long)N * MK;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return LSG_ERR_CUDA;
    double* scratch = nullptr;
    {
        // once per device, with that device current: the device address of the
        // static array (host code cannot use the symbol itself as a pointer)
        std::lock_guard<std::mutex> lock(g_slots_mutex);
        DeviceSlot& slot = g_slots[dev];
        if (!slot.ready) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) return LSG_ERR_CUDA;
            slot.scratch = (double*)p;
            slot.ready = true;
        }
        scratch = slot.scratch;
    }
    cudaStream_t s = (cudaStream_t)stream;
    // the completion counter must start at zero
    if (cudaMemsetAsync(scratch + kMaxBlocks, 0, sizeof(unsigned int), s) != cudaSuccess) return LSG_ERR_CUDA;
    const int blocks = (int)((n + kCellsPerBlock - 1) / kCellsPerBlock);
    k_residual_norm_noalloc<<<blocks, kBlock, 0, s>>>(N, M, K, planes, x, b, r, scratch, norm2);
    if (cudaGetLastError() != cudaSuccess) return LSG_ERR_CUDA;
    return LSG_OK;
}
