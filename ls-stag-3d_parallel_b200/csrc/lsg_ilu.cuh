// ILU(0) of the 7-point operator and its level-scheduled triangular solves.
//
// For a 7-point pattern in natural order (with N, M >= 3) the reference's
// general row-by-row ILU(0) (ilu_decomposition_sparse_matrix.h:63-119)
// reduces to
//     L_kj = A_kj / U_jj            j in {b, s, w}  (|U_jj| clamped at 1e-12)
//     U_kk = A_kk - (L_kb A_bk + L_ks A_sk + L_kw A_wk)   (clamped at 1e-16)
//     U_kj = A_kj                   j in {e, n, t}
// so only the pivots U_kk need computing; they depend on the three upstream
// neighbours, i.e. on the previous hyperplane x + y + z = const.  The
// triangular solves sweep the same hyperplanes
// (ILUDecomposition7pStencilMatrix::DirectGauss/InverseGauss,
// ilu_decomposition_7p_stencil_matrix.h:90-134), one launch per hyperplane,
// all captured in one CUDA graph.
#pragma once

#include "lsg_kernels.cuh"

namespace lsg {

// cell of hyperplane `level` handled by thread t: (x, y) enumerate the plane
// rows, z = level - x - y.
__device__ __forceinline__ bool plane_cell(int level, long long t, int N, int M, int K, long long& i)
{
    const int x = (int)(t % N);
    const int y = (int)(t / N);
    if (y >= M) return false;
    const int z = level - x - y;
    if (z < 0 || z >= K) return false;
    i = (long long)z * N * M + (long long)y * N + x;
    return true;
}

// Pivots of one hyperplane.  A: 7 planes b s w p e n t; U: pivot array.
__global__ void k_ilu_pivots(int level, int N, int M, int K, const double* __restrict__ A, double* __restrict__ U)
{
    const long long n = (long long)N * M * K;
    const int NM = N * M;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)N * M;
         t += (long long)gridDim.x * blockDim.x) {
        long long i;
        if (!plane_cell(level, t, N, M, K, i)) continue;
        const int x = (int)(t % N), y = (int)(t / N), z = level - x - y;
        double aux = 0.0;
        // lower entries in column order b (i-NM), s (i-N), w (i-1)
        if (z > 0) {
            double u = U[i - NM];
            if (fabs(u) < 1e-12) u = (u < 0.0) ? -1e-12 : 1e-12;
            aux += (A[i] / u) * A[6 * n + i - NM];
        }
        if (y > 0) {
            double u = U[i - N];
            if (fabs(u) < 1e-12) u = (u < 0.0) ? -1e-12 : 1e-12;
            aux += (A[n + i] / u) * A[5 * n + i - N];
        }
        if (x > 0) {
            double u = U[i - 1];
            if (fabs(u) < 1e-12) u = (u < 0.0) ? -1e-12 : 1e-12;
            aux += (A[2 * n + i] / u) * A[4 * n + i - 1];
        }
        double cur = A[3 * n + i] - aux;
        if (fabs(cur) < 1e-16) cur = (cur < 0.0) ? -1e-16 : 1e-16;
        U[i] = cur;
    }
}

// L planes (b, s, w) from the pivots: L_kj = A_kj / clamp(U_jj).
__global__ void k_ilu_lower(int N, int M, int K, const double* __restrict__ A, const double* __restrict__ U,
                            double* __restrict__ Lp)
{
    const long long n = (long long)N * M * K;
    const int NM = N * M;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        cell_xyz(i, N, NM, x, y, z);
        double lb = 0, ls = 0, lw = 0;
        if (z > 0) {
            double u = U[i - NM];
            if (fabs(u) < 1e-12) u = (u < 0.0) ? -1e-12 : 1e-12;
            lb = A[i] / u;
        }
        if (y > 0) {
            double u = U[i - N];
            if (fabs(u) < 1e-12) u = (u < 0.0) ? -1e-12 : 1e-12;
            ls = A[n + i] / u;
        }
        if (x > 0) {
            double u = U[i - 1];
            if (fabs(u) < 1e-12) u = (u < 0.0) ? -1e-12 : 1e-12;
            lw = A[2 * n + i] / u;
        }
        Lp[i] = lb;
        Lp[n + i] = ls;
        Lp[2 * n + i] = lw;
    }
}

// forward sweep of one hyperplane: y = b - (L_b y_b + L_s y_s + L_w y_w)
__global__ void k_ilu_fwd(int level, int N, int M, int K, const double* __restrict__ Lp, const double* __restrict__ b,
                          double* __restrict__ y)
{
    const long long n = (long long)N * M * K;
    const int NM = N * M;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)N * M;
         t += (long long)gridDim.x * blockDim.x) {
        long long i;
        if (!plane_cell(level, t, N, M, K, i)) continue;
        const int x = (int)(t % N), yy = (int)(t / N), z = level - x - yy;
        double aux = b[i];
        if (z > 0) aux -= Lp[i] * y[i - NM];
        if (yy > 0) aux -= Lp[n + i] * y[i - N];
        if (x > 0) aux -= Lp[2 * n + i] * y[i - 1];
        y[i] = aux;
    }
}

// backward sweep of one hyperplane: x = (y - (U_e x_e + U_n x_n + U_t x_t)) / U_p
__global__ void k_ilu_bwd(int level, int N, int M, int K, const double* __restrict__ A, const double* __restrict__ U,
                          const double* __restrict__ y, double* __restrict__ xo)
{
    const long long n = (long long)N * M * K;
    const int NM = N * M;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)N * M;
         t += (long long)gridDim.x * blockDim.x) {
        long long i;
        if (!plane_cell(level, t, N, M, K, i)) continue;
        const int x = (int)(t % N), yy = (int)(t / N), z = level - x - yy;
        double aux = y[i];
        if (x < N - 1) aux -= A[4 * n + i] * xo[i + 1];
        if (yy < M - 1) aux -= A[5 * n + i] * xo[i + N];
        if (z < K - 1) aux -= A[6 * n + i] * xo[i + NM];
        xo[i] = aux / U[i];
    }
}

// Both triangular sweeps of one ILU(0) application in one cooperative launch
// (every CTA resident): the hyperplanes of the forward sweep, then those of
// the backward sweep, each thread owning the (x, y) columns t, t + T, ...
// (at most CMAX) for every plane, with the arithmetic of k_ilu_fwd /
// k_ilu_bwd (so the same bits) and a grid-wide barrier between consecutive
// planes instead of a kernel boundary.  A plane's operands that do not
// depend on the previous plane (b or y, the factor entries, the pivot) are
// loaded before the barrier that ends the previous plane, so after it only
// the neighbours just written remain to fetch (through L2, __ldcg: other
// CTAs wrote them).  The barrier counts arrivals on bar[0] (zeroed before
// the launch) and gives up after one second, setting *err.
__device__ __forceinline__ bool ilu_grid_barrier(unsigned int* bar, unsigned int target, int* err)
{
    __syncthreads();
    __shared__ int ok;
    if (threadIdx.x == 0) {
        // arrive (release: this CTA's stores first), then poll with acquire
        // loads; every 256 polls look at the clock and at the error flag
        asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(bar) : "memory");
        ok = 1;
        unsigned long long t0 = 0;
        for (unsigned it = 0;; it++) {
            unsigned int v;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(bar) : "memory");
            if (v >= target) break;
            if ((it & 255) == 0) {
                unsigned long long now;
                asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
                if (it == 0) t0 = now;
                else if (now - t0 > 1000000000ull || *(volatile int*)err != 0) {
                    atomicExch(err, 1);
                    ok = 0;
                    break;
                }
            }
        }
    }
    __syncthreads();
    return ok != 0;
}

template <int CMAX>
__global__ void __launch_bounds__(256, CMAX == 4 ? 3 : (CMAX == 2 ? 4 : 5)) k_ilu_sweep_coop(int N, int M, int K, const double* __restrict__ Lp,
                                                         const double* __restrict__ A, const double* __restrict__ U,
                                                         const double* __restrict__ b, double* y, double* xo,
                                                         unsigned int* bar, int* err)
{
    const long long n = (long long)N * M * K;
    const int NM = N * M;
    const int planes = N + M + K - 2;
    const int T = gridDim.x * blockDim.x;                 // T * CMAX >= N * M (host)
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    // the (x, y) columns of this thread, fixed for every plane
    int cx[CMAX], cy[CMAX];
#pragma unroll
    for (int k = 0; k < CMAX; k++) {
        const int t = tid + k * T;
        cy[k] = t < NM ? t / N : M;                        // y = M: no column
        cx[k] = t < NM ? t - cy[k] * N : 0;
    }
    // operands of a plane that do not depend on the previous plane, loaded
    // before the barrier that ends the previous plane
    double p0[CMAX], p1[CMAX], p2[CMAX], p3[CMAX], p4[CMAX];
    long long ci[CMAX];
    bool act[CMAX];
    auto cell = [&](int level, int k) {
        const int z = level - cx[k] - cy[k];
        act[k] = cy[k] < M && z >= 0 && z < K;
        ci[k] = act[k] ? (long long)z * NM + (long long)cy[k] * N + cx[k] : 0;
        return z;
    };
    auto fwd_operands = [&](int level) {
#pragma unroll
        for (int k = 0; k < CMAX; k++) {
            const int z = cell(level, k);
            if (act[k]) {
                const long long i = ci[k];
                p0[k] = b[i];
                p1[k] = z > 0 ? Lp[i] : 0.0;
                p2[k] = cy[k] > 0 ? Lp[n + i] : 0.0;
                p3[k] = cx[k] > 0 ? Lp[2 * n + i] : 0.0;
            }
        }
    };
    auto bwd_operands = [&](int level) {
#pragma unroll
        for (int k = 0; k < CMAX; k++) {
            const int z = cell(level, k);
            if (act[k]) {
                const long long i = ci[k];
                p0[k] = __ldcg(y + i);
                p1[k] = cx[k] < N - 1 ? A[4 * n + i] : 0.0;
                p2[k] = cy[k] < M - 1 ? A[5 * n + i] : 0.0;
                p3[k] = z < K - 1 ? A[6 * n + i] : 0.0;
                p4[k] = U[i];
            }
        }
    };
    unsigned int target = 0;
    fwd_operands(0);
    for (int level = 0; level < planes; level++) {
#pragma unroll
        for (int k = 0; k < CMAX; k++) {
            if (!act[k]) continue;
            const long long i = ci[k];
            const int z = level - cx[k] - cy[k];
            double aux = p0[k];
            if (z > 0) aux -= p1[k] * __ldcg(y + i - NM);
            if (cy[k] > 0) aux -= p2[k] * __ldcg(y + i - N);
            if (cx[k] > 0) aux -= p3[k] * __ldcg(y + i - 1);
            y[i] = aux;
        }
        if (level + 1 < planes) fwd_operands(level + 1);
        target += gridDim.x;
        if (!ilu_grid_barrier(bar, target, err)) return;
    }
    bwd_operands(planes - 1);
    for (int level = planes - 1; level >= 0; level--) {
#pragma unroll
        for (int k = 0; k < CMAX; k++) {
            if (!act[k]) continue;
            const long long i = ci[k];
            const int z = level - cx[k] - cy[k];
            double aux = p0[k];
            if (cx[k] < N - 1) aux -= p1[k] * __ldcg(xo + i + 1);
            if (cy[k] < M - 1) aux -= p2[k] * __ldcg(xo + i + N);
            if (z < K - 1) aux -= p3[k] * __ldcg(xo + i + NM);
            xo[i] = aux / p4[k];
        }
        if (level > 0) {
            bwd_operands(level - 1);
            target += gridDim.x;
            if (!ilu_grid_barrier(bar, target, err)) return;
        }
    }
}

}  // namespace lsg
