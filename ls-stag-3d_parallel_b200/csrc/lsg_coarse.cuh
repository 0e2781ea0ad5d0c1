// The smallest multigrid levels in one kernel.
//
// On levels of a few hundred cells every V-cycle operation (restriction,
// 27-point residual update, line solve, prolongation) is a kernel launch of a
// few microseconds for almost no data.  k_vcycle_tail runs the lower part of
// the cycle (MultiGridSolver::solve, multigrid_solver.h:48-75, from level l0
// down to the coarsest solve and back up through the smoothing of level l0) in
// one CTA of 1024 threads, phases separated by __syncthreads(); the level data
// stays in the SM's L1.  Each phase performs the same arithmetic, in the same
// order, as the stand-alone kernel it replaces (k_restrict, k_coarse_solve,
// k_prolong, k_apply27z, k_tdma_strided), so both paths give the same iterates.
// Larger levels stay separate launches: there one CTA is bound by the latency
// of its own sequential line recurrences.
#pragma once

#include "lsg_kernels.cuh"

namespace lsg {

constexpr int kTailThreads = 1024;
constexpr int kTailMaxCells = 512;      // levels fused into the tail kernel hold at most this many cells
constexpr int kTailMaxLevels = 12;

template <typename T>
struct TailLevel {
    int N, M, K;
    const int* cls;
    const T* dict28;                    // 27-point rows, stride 28 (z, y, x box order)
    const T* lo[3];
    const T* dinv[3];
    const T* up[3];
    T* r;
    T* c;
    T* ch;
    // transfer tables between this level (fine side) and the next coarser one
    PTab px, py, pz;
    RTab rx, ry, rz;
    int agg;
};

template <typename T>
struct TailArgs {
    TailLevel<T> lev[kTailMaxLevels];   // levels l0 .. L (index 0 = level l0)
    int nlev;                           // number of levels including the coarsest
    // coarsest dense LU (LUDecompositionSparseMatrix)
    int nc;
    const double* L;
    const double* U;
    const double* scale;
    const int* perm;
    double* work;
    int n_post;
    int zquirk;
    T omega;
};

// coarse = R fine (k_restrict)
template <typename T>
__device__ __forceinline__ void tail_restrict(const TailLevel<T>& f, const TailLevel<T>& c)
{
    const int nc = c.N * c.M * c.K, NMc = c.N * c.M, NM = f.N * f.M;
    for (int I = threadIdx.x; I < nc; I += blockDim.x) {
        const int Z = I / NMc, rem = I - Z * NMc, Y = rem / c.N, X = rem - Y * c.N;
        T acc = 0;
        if (f.agg) {
            const int f0 = (2 * Z) * NM + (2 * Y) * f.N + 2 * X;
            const T w = (T)0.125;
            acc += w * f.r[f0];
            acc += w * f.r[f0 + 1];
            acc += w * f.r[f0 + f.N];
            acc += w * f.r[f0 + f.N + 1];
            acc += w * f.r[f0 + NM];
            acc += w * f.r[f0 + NM + 1];
            acc += w * f.r[f0 + NM + f.N];
            acc += w * f.r[f0 + NM + f.N + 1];
        } else {
            for (int a = 0; a < 4; a++) {
                const int fz = f.rz.f[4 * Z + a];
                if (fz < 0) continue;
                const float wz = f.rz.w[4 * Z + a];
                for (int b = 0; b < 4; b++) {
                    const int fy = f.ry.f[4 * Y + b];
                    if (fy < 0) continue;
                    const float wy = f.ry.w[4 * Y + b];
                    for (int q = 0; q < 4; q++) {
                        const int fx = f.rx.f[4 * X + q];
                        if (fx < 0) continue;
                        acc += (T)(wz * wy * f.rx.w[4 * X + q]) * f.r[fz * NM + fy * f.N + fx];
                    }
                }
            }
        }
        c.r[I] = acc;
    }
}

// fine ch = P coarse ch, fine c = ch (k_prolong)
template <typename T>
__device__ __forceinline__ void tail_prolong(const TailLevel<T>& f, const TailLevel<T>& c)
{
    const int n = f.N * f.M * f.K, NM = f.N * f.M, NMc = c.N * c.M;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int z = i / NM, rem = i - z * NM, y = rem / f.N, x = rem - y * f.N;
        T acc = 0;
        for (int a = 0; a < 2; a++) {
            const float wz = f.pz.w[2 * z + a];
            const int oz = f.pz.c[2 * z + a] * NMc;
            for (int b = 0; b < 2; b++) {
                const float wy = f.py.w[2 * y + b];
                const int oy = f.py.c[2 * y + b] * c.N;
                for (int q = 0; q < 2; q++) {
                    const float wx = f.px.w[2 * x + q];
                    if (wz != 0.f && wy != 0.f && wx != 0.f)
                        acc += (T)(wz * wy * wx) * c.ch[oz + oy + f.px.c[2 * x + q]];
                }
            }
        }
        f.ch[i] = acc;
        f.c[i] = acc;
    }
}

// r -= A c with the 27-point box rows (k_apply27z, MODE 0)
template <typename T>
__device__ __forceinline__ void tail_resid27(const TailLevel<T>& v)
{
    const int n = v.N * v.M * v.K, NM = v.N * v.M;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int z = i / NM, rem = i - z * NM, y = rem / v.N, x = rem - y * v.N;
        const T* a = v.dict28 + (size_t)v.cls[i] * 28;
        T acc = 0;
#pragma unroll
        for (int dz = -1; dz <= 1; dz++) {
            const bool zin = z + dz >= 0 && z + dz < v.K;
#pragma unroll
            for (int dy = -1; dy <= 1; dy++)
#pragma unroll
                for (int dx = -1; dx <= 1; dx++) {
                    const bool ok = zin && x + dx >= 0 && x + dx < v.N && y + dy >= 0 && y + dy < v.M;
                    const T xv = ok ? v.c[i + dz * NM + dy * v.N + dx] : (T)0;
                    acc += a[(dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)] * xv;
                }
        }
        v.r[i] = v.r[i] - acc;
    }
}

// c = omega T_d^-1 r, ch += c, one thread per line (k_tdma_strided)
template <typename T>
__device__ __forceinline__ void tail_lines(const TailLevel<T>& v, int d, bool zquirk, T omega)
{
    const int L = d == 0 ? v.N : (d == 1 ? v.M : v.K);
    const int nl = d == 0 ? v.M * v.K : (d == 1 ? v.N * v.K : v.N * v.M);
    const int st = d == 0 ? 1 : (d == 1 ? v.N : v.N * v.M);
    const T* lo = v.lo[d];
    const T* dinv = v.dinv[d];
    const T* up = v.up[d];
    for (int l = threadIdx.x; l < nl; l += blockDim.x) {
        int i0;
        if (d == 0) {
            i0 = l * v.N;
        } else if (d == 1) {
            const int z = l / v.N;
            i0 = z * v.N * v.M + (l - z * v.N);
        } else {
            i0 = l;
        }
        T rhs0 = v.r[i0];
        if (d == 2 && zquirk) {
            const int y = l / v.N, x = l - y * v.N;
            rhs0 = v.r[y * v.N * v.K + x];            // reference z-line quirk
        }
        T yv = 0;
        for (int t = 0; t < L; t++) {
            const int i = i0 + t * st;
            const T rv = t == 0 ? rhs0 : v.r[i];
            yv = (t == 0) ? rv * dinv[i] : (rv - lo[i] * yv) * dinv[i];
            v.c[i] = yv;
        }
        T xv = 0;
        for (int t = L - 1; t >= 0; t--) {
            const int i = i0 + t * st;
            const T y = v.c[i];
            xv = (t == L - 1) ? y : y - up[i] * xv;
            const T cv = omega * xv;
            v.c[i] = cv;
            v.ch[i] = v.ch[i] + cv;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kTailThreads) k_vcycle_tail(const TailArgs<T>* __restrict__ argp)
{
    const TailArgs<T>& A = *argp;
    const int last = A.nlev - 1;
    for (int l = 0; l < last; l++) {
        tail_restrict<T>(A.lev[l], A.lev[l + 1]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        // coarsest solve (k_coarse_solve)
        const TailLevel<T>& c = A.lev[last];
        const int n = A.nc;
        double* y = A.work;
        double* z = A.work + n;
        for (int i = 0; i < n; i++) {
            double aux = A.scale[A.perm[i]] * (double)c.r[A.perm[i]];
            for (int j = 0; j < i; j++) aux -= A.L[i * n + j] * y[j];
            y[i] = aux;
        }
        for (int i = n - 1; i >= 0; i--) {
            double aux = y[i];
            for (int j = i + 1; j < n; j++) aux -= A.U[i * n + j] * z[j];
            z[i] = aux / A.U[i * n + i];
        }
        for (int i = 0; i < n; i++) c.ch[i] = (T)(A.scale[i] * z[i]);
    }
    __syncthreads();
    for (int l = last - 1; l >= 0; l--) {
        const TailLevel<T>& v = A.lev[l];
        tail_prolong<T>(v, A.lev[l + 1]);
        __syncthreads();
        for (int it = 0; it < A.n_post; it++) {
            for (int q = 0; q < 3; q++) {
                tail_resid27<T>(v);
                __syncthreads();
                tail_lines<T>(v, 2 - q, A.zquirk != 0, A.omega);   // z, y, x
                __syncthreads();
            }
        }
    }
}

}  // namespace lsg
