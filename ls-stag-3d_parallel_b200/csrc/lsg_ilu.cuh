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

}  // namespace lsg
