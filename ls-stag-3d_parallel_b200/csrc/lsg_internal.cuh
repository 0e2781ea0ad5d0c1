// Internal declarations of the B200 pressure-Poisson solver library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>
#include <vector>

#include "../../include/lsstag_b200.h"

namespace lsg {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
struct Error {
    int code;
    std::string msg;
};

#define LSG_CUDA(call)                                                                    \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            throw ::lsg::Error{LSG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

// every kernel launch of the library is followed by this check, which also
// counts launches (reported per solve in lsg_stats.kernel_launches)
extern thread_local long long g_launches;
#define LSG_CHECK_LAUNCH()              \
    do {                                \
        ::lsg::g_launches++;            \
        LSG_CUDA(cudaGetLastError());   \
    } while (0)

#define LSG_REQUIRE(cond, code, text)                  \
    do {                                               \
        if (!(cond)) throw ::lsg::Error{(code), (text)}; \
    } while (0)

// ---------------------------------------------------------------------------
// per-call temporaries: stream-ordered allocations from a context's own memory
// pool, released on the context's stream when they go out of scope.  The
// pool keeps freed memory (release threshold: never), so a call that repeats
// every time step reuses its blocks instead of a cudaMalloc / cudaFree pair
// (cudaFree synchronises the device).
// ---------------------------------------------------------------------------
template <typename T>
struct TmpBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    cudaMemPool_t pool = nullptr;
    TmpBuf(cudaStream_t stream, cudaMemPool_t mp) : s(stream), pool(mp) {}
    TmpBuf(const TmpBuf&) = delete;
    TmpBuf& operator=(const TmpBuf&) = delete;
    ~TmpBuf() { release(); }
    void alloc(size_t count)
    {
        if (count == n && p) return;
        release();
        if (count == 0) return;
        cudaError_t e = cudaMallocFromPoolAsync((void**)&p, count * sizeof(T), pool, s);
        if (e != cudaSuccess) {
            p = nullptr;
            throw Error{LSG_ERR_NOMEM, std::string("stream-ordered allocation of ") +
                                           std::to_string(count * sizeof(T)) + " bytes: " + cudaGetErrorString(e)};
        }
        n = count;
    }
    void release()
    {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
        n = 0;
    }
    size_t bytes() const { return n * sizeof(T); }
};

// ---------------------------------------------------------------------------
// device buffers
// ---------------------------------------------------------------------------
template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept
    {
        if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DevBuf() { release(); }
    void alloc(size_t count)
    {
        if (count == n && p) return;
        release();
        if (count == 0) return;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            throw Error{LSG_ERR_NOMEM, std::string("cudaMalloc of ") + std::to_string(count * sizeof(T)) +
                                           " bytes: " + cudaGetErrorString(e)};
        }
        n = count;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    size_t bytes() const { return n * sizeof(T); }
};

// ---------------------------------------------------------------------------
// grids and stencils
// ---------------------------------------------------------------------------
struct Dims {
    int N = 0, M = 0, K = 0;
    long long n() const { return (long long)N * M * K; }
};

// Offsets of the fine-level 7-point operator, in the reference's CSR column
// order (b, s, w, p, e, n, t).
constexpr int kFineOffsets = 7;

// A box stencil operator on one grid level: coef[o * n + cell] multiplies the
// neighbour (x+ox, y+oy, z+oz).  Offsets outside the grid carry 0.
template <typename T>
struct Stencil {
    Dims d;
    int rx = 0, ry = 0, rz = 0;   // radius per dimension
    int noff = 0;                 // number of offsets
    std::vector<int> off;         // 3 * noff host copy (ox, oy, oz)
    DevBuf<int> d_off;            // 3 * noff on the device
    int center = -1;              // index of (0,0,0)
    DevBuf<T> coef;               // noff * n
};

// Line tridiagonal of one direction, stored per natural cell index:
//   lo[i] couples cell i to the previous cell of its line (0 at line start)
//   dinv[i] inverse pivot, up[i] (scaled) coupling to the next cell.
template <typename T>
struct LineFactor {
    DevBuf<T> lo, dinv, up;
};

// Multigrid level (precision T).
template <typename T>
struct Level {
    Dims d;
    Stencil<T> A;
    LineFactor<T> line[3];        // x, y, z
    bool oddN = false, oddM = false, oddK = false;   // parity of THIS level (fine side of the transfer)
    bool agglomerate = false;     // restriction to the next level is the 1/8 agglomeration
    DevBuf<T> r, c, ch;           // residual / right-hand side, correction, accumulated solution
};

struct CoarseLU {
    int n = 0;
    std::vector<double> L, U, scale;  // row-major n x n
    std::vector<int> perm;
    DevBuf<double> dL, dU, dscale;
    DevBuf<int> dperm;
};

template <typename T>
struct Hierarchy {
    std::vector<Level<T>> lev;    // lev[0] fine ... lev[L] coarsest
    CoarseLU lu;
    DevBuf<double> coarse_rhs, coarse_sol;
};

// ---------------------------------------------------------------------------
// reductions: deterministic two-stage (block partials + last-block sum)
// ---------------------------------------------------------------------------
struct Reducer {
    static constexpr int kMaxBlocks = 2048;   // default grid cap of the one-thread-per-cell kernels
    static constexpr int kCapBlocks = 8192;   // most blocks any reducing launch may use
    static constexpr int kSlots = 4;
    DevBuf<double> partial;       // kCapBlocks * kSlots
    DevBuf<unsigned int> counter; // one per concurrent reduction site
    void init()
    {
        partial.alloc((size_t)kCapBlocks * kSlots);
        counter.alloc(64);
        LSG_CUDA(cudaMemset(counter.p, 0, counter.bytes()));
    }
};

// FGMRES device-side scalars (one struct, device memory).
struct KrylovScalars {
    double H[64 * 65];      // column-major Hessenberg entries h[i + j*65]
    double cs[64], sn[64], y[64];
    double norm_r;          // running |gamma|
    double normW2;          // ||w||^2 of the latest Arnoldi vector
    double invNormW;        // 1 / ||w||
    double bnorm2;
    int it;
    int done;               // 1 converged / capped
    int breakdown;
    int pad;
};

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
inline int grid_for(long long n, int block, int max_blocks = 148 * 16)
{
    long long g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > max_blocks) g = max_blocks;
    return (int)g;
}

}  // namespace lsg
