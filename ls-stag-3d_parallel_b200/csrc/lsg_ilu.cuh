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

// Grid-wide barrier of the cooperative ILU sweep (every CTA resident):
// arrivals are counted on bar[0] (zeroed before the launch); it gives up
// after one second, setting *err.  Values other CTAs wrote before the
// barrier are read after it through L2 (__ldcg).
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

// Position of cell (x, y, z) in the hyperplane order: planes l = x + y + z in
// turn, inside a plane by z, then y (x = l - y - z).  start[l] is the first
// position of plane l, rowstart[l K + z] the first of its row z.
__device__ __forceinline__ int ilu_hpos(int x, int y, int z, int N, int K, const int* __restrict__ start,
                                        const int* __restrict__ rowstart)
{
    const int l = x + y + z;
    const int ymin = max(0, l - z - (N - 1));
    return start[l] + rowstart[(long long)l * K + z] + (y - ymin);
}

// The factors and neighbour positions in hyperplane order: perm[p] = i for
// the cell i at position p; fac = L_b, L_s, L_w, U_e, U_n, U_t, U_p (7 arrays
// of n); nbr = the positions of the cells below (z-1, y-1, x-1) and above
// (x+1, y+1, z+1), -1 outside the grid (6 arrays of n).
__global__ void k_ilu_perm_build(int N, int M, int K, const int* __restrict__ start, const int* __restrict__ rowstart,
                                 const double* __restrict__ Lp, const double* __restrict__ A,
                                 const double* __restrict__ U, int* __restrict__ perm, double* __restrict__ fac,
                                 int* __restrict__ nbr)
{
    const long long n = (long long)N * M * K;
    const int NM = N * M;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        cell_xyz(i, N, NM, x, y, z);
        const int p = ilu_hpos(x, y, z, N, K, start, rowstart);
        perm[p] = (int)i;
        fac[p] = Lp[i];
        fac[n + p] = Lp[n + i];
        fac[2 * n + p] = Lp[2 * n + i];
        fac[3 * n + p] = A[4 * n + i];
        fac[4 * n + p] = A[5 * n + i];
        fac[5 * n + p] = A[6 * n + i];
        fac[6 * n + p] = U[i];
        nbr[p] = z > 0 ? ilu_hpos(x, y, z - 1, N, K, start, rowstart) : -1;
        nbr[n + p] = y > 0 ? ilu_hpos(x, y - 1, z, N, K, start, rowstart) : -1;
        nbr[2 * n + p] = x > 0 ? ilu_hpos(x - 1, y, z, N, K, start, rowstart) : -1;
        nbr[3 * n + p] = x < N - 1 ? ilu_hpos(x + 1, y, z, N, K, start, rowstart) : -1;
        nbr[4 * n + p] = y < M - 1 ? ilu_hpos(x, y + 1, z, N, K, start, rowstart) : -1;
        nbr[5 * n + p] = z < K - 1 ? ilu_hpos(x, y, z + 1, N, K, start, rowstart) : -1;
    }
}

// Both triangular sweeps of one ILU(0) application in one cooperative launch
// over the hyperplane-ordered factors (k_ilu_perm_build): the cells of a
// plane are contiguous, so every stream of a plane is read coalesced, and
// their neighbours in the previous plane lie close together.  Each thread
// takes positions t, t + T, ... (at most CMAX) of every plane, with the
// arithmetic of k_ilu_fwd / k_ilu_bwd (the same bits); b is gathered and x
// scattered through perm inside the sweeps.  A plane's operands that do not
// depend on the previous plane are loaded before the barrier that ends it.
template <int CMAX>
__global__ void __launch_bounds__(256) k_ilu_sweep_perm(int planes, long long n, const int* __restrict__ start,
                                                         const int* __restrict__ perm, const double* __restrict__ fac,
                                                         const int* __restrict__ nbr, const double* __restrict__ b,
                                                         double* yp, double* xp, double* __restrict__ x,
                                                         unsigned int* bar, int* err, int withhold)
{
    // withhold >= 0 (the wait-limit self-test only): that CTA leaves before its
    // first barrier arrival, so the others' first wait runs out
    if ((int)blockIdx.x == withhold) return;
    const int T = gridDim.x * blockDim.x;                 // T * CMAX >= the largest plane (host)
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    int pos[CMAX], n0[CMAX], n1[CMAX], n2[CMAX];
    double v0[CMAX], v1[CMAX], v2[CMAX], v3[CMAX], v4[CMAX];
    auto fwd_operands = [&](int level) {
        const int s0 = start[level], cnt = start[level + 1] - s0;
#pragma unroll
        for (int k = 0; k < CMAX; k++) {
            const int q = tid + k * T;
            pos[k] = q < cnt ? s0 + q : -1;
            if (pos[k] >= 0) {
                const int p = pos[k];
                v0[k] = b[perm[p]];
                v1[k] = fac[p];
                v2[k] = fac[n + p];
                v3[k] = fac[2 * n + p];
                n0[k] = nbr[p];
                n1[k] = nbr[n + p];
                n2[k] = nbr[2 * n + p];
            }
        }
    };
    auto bwd_operands = [&](int level) {
        const int s0 = start[level], cnt = start[level + 1] - s0;
#pragma unroll
        for (int k = 0; k < CMAX; k++) {
            const int q = tid + k * T;
            pos[k] = q < cnt ? s0 + q : -1;
            if (pos[k] >= 0) {
                const int p = pos[k];
                v0[k] = __ldcg(yp + p);
                v1[k] = fac[3 * n + p];
                v2[k] = fac[4 * n + p];
                v3[k] = fac[5 * n + p];
                v4[k] = fac[6 * n + p];
                n0[k] = nbr[3 * n + p];
                n1[k] = nbr[4 * n + p];
                n2[k] = nbr[5 * n + p];
            }
        }
    };
    unsigned int target = 0;
    fwd_operands(0);
    for (int level = 0; level < planes; level++) {
#pragma unroll
        for (int k = 0; k < CMAX; k++) {
            if (pos[k] < 0) continue;
            double aux = v0[k];
            if (n0[k] >= 0) aux -= v1[k] * __ldcg(yp + n0[k]);
            if (n1[k] >= 0) aux -= v2[k] * __ldcg(yp + n1[k]);
            if (n2[k] >= 0) aux -= v3[k] * __ldcg(yp + n2[k]);
            yp[pos[k]] = aux;
        }
        if (level + 1 < planes) fwd_operands(level + 1);
        target += gridDim.x;
        if (!ilu_grid_barrier(bar, target, err)) return;
    }
    bwd_operands(planes - 1);
    for (int level = planes - 1; level >= 0; level--) {
#pragma unroll
        for (int k = 0; k < CMAX; k++) {
            if (pos[k] < 0) continue;
            double aux = v0[k];
            if (n0[k] >= 0) aux -= v1[k] * __ldcg(xp + n0[k]);
            if (n1[k] >= 0) aux -= v2[k] * __ldcg(xp + n1[k]);
            if (n2[k] >= 0) aux -= v3[k] * __ldcg(xp + n2[k]);
            const double v = aux / v4[k];
            xp[pos[k]] = v;
            x[perm[pos[k]]] = v;
        }
        if (level > 0) {
            bwd_operands(level - 1);
            target += gridDim.x;
            if (!ilu_grid_barrier(bar, target, err)) return;
        }
    }
}

}  // namespace lsg
