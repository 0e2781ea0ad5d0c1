// Device kernels of the B200 pressure-Poisson solver.
//
// Every kernel is bandwidth bound (<= 0.25 flop/B); they are written for
// coalesced, vectorisable streaming of the SoA coefficient planes with the
// stencil neighbours served from L1/L2, and for deterministic reductions
// (block partials summed by the last block in a fixed order).
#pragma once

#include "lsg_internal.cuh"

namespace lsg {

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------
struct OffList {
    int n;
    int center;
    signed char o[125][3];
};

// Cell coordinates of a flat index (x fastest).  Grids hold fewer than 2^31
// cells, so 32-bit unsigned division suffices.
__device__ __forceinline__ void cell_xyz(long long i, int N, int NM, int& x, int& y, int& z)
{
    const unsigned u = (unsigned)i;
    z = (int)(u / (unsigned)NM);
    const unsigned r = u - (unsigned)z * (unsigned)NM;
    y = (int)(r / (unsigned)N);
    x = (int)(r - (unsigned)y * (unsigned)N);
}

// Division by a run-time invariant d >= 1 of numerators below 2^31 by one
// multiply-high and shifts (Granlund & Montgomery, "Division by invariant
// integers using multiplication", PLDI 1994, fig. 4.1):
//   l = ceil(log2 d),  m = floor(2^32 (2^l - d) / d) + 1,
//   t = mulhi(m, n),   q = (t + ((n - t) >> min(l,1))) >> max(l-1,0).
// Built once per thread, used for every cell the thread visits.
struct FDiv {
    unsigned d, m;
    int s1, s2;
    __device__ explicit FDiv(unsigned dd) : d(dd)
    {
        int l = 0;
        while (l < 31 && (1u << l) < dd) l++;
        m = (unsigned)((((unsigned long long)((1ull << l) - dd)) << 32) / dd + 1);
        s1 = l < 1 ? l : 1;
        s2 = l - 1 > 0 ? l - 1 : 0;
    }
    __device__ __forceinline__ unsigned div(unsigned n) const
    {
        const unsigned t = __umulhi(m, n);
        return (t + ((n - t) >> s1)) >> s2;
    }
};

struct CellIndex {
    FDiv dN, dNM;
    __device__ CellIndex(int N, int NM) : dN((unsigned)N), dNM((unsigned)NM) {}
    __device__ __forceinline__ void xyz(long long i, int& x, int& y, int& z) const
    {
        const unsigned u = (unsigned)i;
        const unsigned zz = dNM.div(u);
        const unsigned r = u - zz * dNM.d;
        const unsigned yy = dN.div(r);
        z = (int)zz;
        y = (int)yy;
        x = (int)(r - yy * dN.d);
    }
};

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block + grid reduction of NS values.  Every block writes its
// partial sums; the last block to finish adds them in block order and writes
// out[s].  Blocks of 1-3 dimensions with a multiple of 32 threads (<= 1024),
// grids of 1-3 dimensions; blocks and threads are taken in linear order.
template <int NS>
__device__ void grid_reduce(double (&v)[NS], double* partial, unsigned int* counter, double* out)
{
    __shared__ double sh[32][NS];
    __shared__ bool last;
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthr = blockDim.x * blockDim.y * blockDim.z;
    const unsigned bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    const unsigned nblk = gridDim.x * gridDim.y * gridDim.z;
    const int lane = tid & 31, wid = tid >> 5, nw = nthr >> 5;
#pragma unroll
    for (int s = 0; s < NS; s++) {
        double t = warp_sum(v[s]);
        if (lane == 0) sh[wid][s] = t;
    }
    __syncthreads();
    if (tid == 0) {
#pragma unroll
        for (int s = 0; s < NS; s++) {
            double t = 0.0;
            for (int w = 0; w < nw; w++) t += sh[w][s];
            partial[(size_t)bid * NS + s] = t;
        }
        __threadfence();
        unsigned int prev = atomicAdd(counter, 1u);
        last = (prev == nblk - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // partials read past L1 (__ldcg), two blocks per step so loads overlap
    double acc[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) acc[s] = 0.0;
    int b = tid;
    for (; b + nthr < (int)nblk; b += 2 * nthr) {
#pragma unroll
        for (int s = 0; s < NS; s++) {
            const double p0 = __ldcg(partial + (size_t)b * NS + s);
            const double p1 = __ldcg(partial + (size_t)(b + nthr) * NS + s);
            acc[s] += p0 + p1;
        }
    }
    for (; b < (int)nblk; b += nthr) {
#pragma unroll
        for (int s = 0; s < NS; s++) acc[s] += __ldcg(partial + (size_t)b * NS + s);
    }
#pragma unroll
    for (int s = 0; s < NS; s++) {
        double t = warp_sum(acc[s]);
        if (lane == 0) sh[wid][s] = t;
    }
    __syncthreads();
    if (tid == 0) {
#pragma unroll
        for (int s = 0; s < NS; s++) {
            double t = 0.0;
            for (int w = 0; w < nw; w++) t += sh[w][s];
            out[s] = t;
        }
        *counter = 0u;
    }
}

// ---------------------------------------------------------------------------
// operator assembly
// ---------------------------------------------------------------------------

// Scatter the reference's CSR rows into the 7 coefficient planes (b, s, w, p,
// e, n, t).  Entries of one row with the same column add up, like the CSR
// product does.  err[0] = 1 + first bad row when an entry is not one of the
// six face neighbours or the cell itself.
__global__ void k_csr_to_stencil7(int N, int M, int K, const int* __restrict__ rowptr,
                                  const int* __restrict__ col, const double* __restrict__ val,
                                  double* __restrict__ coef, int* err)
{
    const long long n = (long long)N * M * K;
    const int NM = N * M;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        cell_xyz(i, N, NM, x, y, z);
        for (int e = rowptr[i]; e < rowptr[i + 1]; e++) {
            const long long j = col[e];
            int slot = -1;
            if (j >= 0 && j < n) {
                int jx, jy, jz;
                cell_xyz(j, N, NM, jx, jy, jz);
                const int dx = jx - x, dy = jy - y, dz = jz - z;
                if (dx == 0 && dy == 0 && dz == -1) slot = 0;
                else if (dx == 0 && dy == -1 && dz == 0) slot = 1;
                else if (dx == -1 && dy == 0 && dz == 0) slot = 2;
                else if (dx == 0 && dy == 0 && dz == 0) slot = 3;
                else if (dx == 1 && dy == 0 && dz == 0) slot = 4;
                else if (dx == 0 && dy == 1 && dz == 0) slot = 5;
                else if (dx == 0 && dy == 0 && dz == 1) slot = 6;
            }
            if (slot < 0) {
                atomicCAS(err, 0, (int)(i + 1));
                continue;
            }
            coef[(size_t)slot * n + i] += val[e];
        }
    }
}

template <typename Tout, typename Tin>
__global__ void k_convert(long long n, const Tin* __restrict__ a, Tout* __restrict__ b)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        b[i] = (Tout)a[i];
}

// ---------------------------------------------------------------------------
// stencil applies
// ---------------------------------------------------------------------------

// Fine 7-point residual update  r -= A x  (mode 0),  y = A x  (mode 1).
template <typename T, int MODE>
__global__ void __launch_bounds__(256) k_apply7(int N, int M, int K, const T* __restrict__ coef,
                                                 const T* __restrict__ x, T* __restrict__ r)
{
    const long long n = (long long)N * M * K;
    const int NM = N * M;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int ix, iy, iz;
        cell_xyz(i, N, NM, ix, iy, iz);
        T acc = coef[3 * n + i] * x[i];
        if (iz > 0) acc += coef[i] * x[i - NM];
        if (iy > 0) acc += coef[n + i] * x[i - N];
        if (ix > 0) acc += coef[2 * n + i] * x[i - 1];
        if (ix < N - 1) acc += coef[4 * n + i] * x[i + 1];
        if (iy < M - 1) acc += coef[5 * n + i] * x[i + N];
        if (iz < K - 1) acc += coef[6 * n + i] * x[i + NM];
        if (MODE == 0) r[i] -= acc;
        else r[i] = acc;
    }
}

// Box-stencil (coarse Galerkin operator) residual update r -= A x (mode 0)
// or y = A x (mode 1).
template <typename T, int MODE>
__global__ void __launch_bounds__(256) k_applybox(int N, int M, int K, OffList ol, const T* __restrict__ coef,
                                                   const T* __restrict__ x, T* __restrict__ r)
{
    const long long n = (long long)N * M * K;
    const int NM = N * M;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int ix, iy, iz;
        cell_xyz(i, N, NM, ix, iy, iz);
        T acc = 0;
        for (int o = 0; o < ol.n; o++) {
            const int jx = ix + ol.o[o][0], jy = iy + ol.o[o][1], jz = iz + ol.o[o][2];
            if (jx < 0 || jx >= N || jy < 0 || jy >= M || jz < 0 || jz >= K) continue;
            acc += coef[(size_t)o * n + i] * x[i + ol.o[o][0] + (long long)ol.o[o][1] * N + (long long)ol.o[o][2] * NM];
        }
        if (MODE == 0) r[i] -= acc;
        else r[i] = acc;
    }
}

// 27-point box stencil (radius 1 in every dimension, the Galerkin operator of
// the even-even-even and odd-odd-odd coarsenings): offsets unrolled, plane
// q = ((dz+1)*3 + (dy+1))*3 + (dx+1).
template <typename T, int MODE>
__global__ void __launch_bounds__(256) k_apply27(int N, int M, int K, const T* __restrict__ coef,
                                                  const T* __restrict__ x, T* __restrict__ r)
{
    const long long n = (long long)N * M * K;
    const int NM = N * M;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int ix, iy, iz;
        cell_xyz(i, N, NM, ix, iy, iz);
        T acc = 0;
        const bool interior = ix > 0 && ix < N - 1 && iy > 0 && iy < M - 1 && iz > 0 && iz < K - 1;
        if (interior) {
#pragma unroll
            for (int dz = -1; dz <= 1; dz++)
#pragma unroll
                for (int dy = -1; dy <= 1; dy++)
#pragma unroll
                    for (int dx = -1; dx <= 1; dx++) {
                        const int q = ((dz + 1) * 3 + (dy + 1)) * 3 + (dx + 1);
                        acc += coef[(size_t)q * n + i] * x[i + dx + (long long)dy * N + (long long)dz * NM];
                    }
        } else {
#pragma unroll
            for (int dz = -1; dz <= 1; dz++)
#pragma unroll
                for (int dy = -1; dy <= 1; dy++)
#pragma unroll
                    for (int dx = -1; dx <= 1; dx++) {
                        const int jx = ix + dx, jy = iy + dy, jz = iz + dz;
                        if (jx < 0 || jx >= N || jy < 0 || jy >= M || jz < 0 || jz >= K) continue;
                        const int q = ((dz + 1) * 3 + (dy + 1)) * 3 + (dx + 1);
                        acc += coef[(size_t)q * n + i] * x[i + dx + (long long)dy * N + (long long)dz * NM];
                    }
        }
        if (MODE == 0) r[i] -= acc;
        else r[i] = acc;
    }
}

// ---------------------------------------------------------------------------
// row-dictionary operators: cls[i] indexes a table of the distinct
// coefficient rows (row-major, NOFF values per row).  Bit-identical rows share
// one entry, so a level whose rows are mostly uniform streams 4 bytes of
// operator per cell instead of NOFF coefficients; the table stays in L1/L2.
// ---------------------------------------------------------------------------
template <typename T, int MODE>
__global__ void __launch_bounds__(256) k_apply7d(int N, int M, int K, const int* __restrict__ cls,
                                                  const T* __restrict__ dict, const T* __restrict__ x,
                                                  T* __restrict__ r)
{
    const long long n = (long long)N * M * K;
    const int NM = N * M;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int ix, iy, iz;
        cell_xyz(i, N, NM, ix, iy, iz);
        const T* a = dict + (size_t)cls[i] * 7;
        T acc = a[3] * x[i];
        if (iz > 0) acc += a[0] * x[i - NM];
        if (iy > 0) acc += a[1] * x[i - N];
        if (ix > 0) acc += a[2] * x[i - 1];
        if (ix < N - 1) acc += a[4] * x[i + 1];
        if (iy < M - 1) acc += a[5] * x[i + N];
        if (iz < K - 1) acc += a[6] * x[i + NM];
        if (MODE == 0) r[i] -= acc;
        else r[i] = acc;
    }
}

template <typename T, int MODE>
__global__ void __launch_bounds__(256) k_apply27d(int N, int M, int K, const int* __restrict__ cls,
                                                   const T* __restrict__ dict, const T* __restrict__ x,
                                                   T* __restrict__ r)
{
    const long long n = (long long)N * M * K;
    const int NM = N * M;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int ix, iy, iz;
        cell_xyz(i, N, NM, ix, iy, iz);
        const T* a = dict + (size_t)cls[i] * 27;
        T acc = 0;
        const bool interior = ix > 0 && ix < N - 1 && iy > 0 && iy < M - 1 && iz > 0 && iz < K - 1;
        if (interior) {
#pragma unroll
            for (int dz = -1; dz <= 1; dz++)
#pragma unroll
                for (int dy = -1; dy <= 1; dy++)
#pragma unroll
                    for (int dx = -1; dx <= 1; dx++) {
                        const int q = ((dz + 1) * 3 + (dy + 1)) * 3 + (dx + 1);
                        acc += a[q] * x[i + dx + (long long)dy * N + (long long)dz * NM];
                    }
        } else {
#pragma unroll
            for (int dz = -1; dz <= 1; dz++)
#pragma unroll
                for (int dy = -1; dy <= 1; dy++)
#pragma unroll
                    for (int dx = -1; dx <= 1; dx++) {
                        const int jx = ix + dx, jy = iy + dy, jz = iz + dz;
                        if (jx < 0 || jx >= N || jy < 0 || jy >= M || jz < 0 || jz >= K) continue;
                        const int q = ((dz + 1) * 3 + (dy + 1)) * 3 + (dx + 1);
                        acc += a[q] * x[i + dx + (long long)dy * N + (long long)dz * NM];
                    }
        }
        if (MODE == 0) r[i] -= acc;
        else r[i] = acc;
    }
}

// z-marching variants: a 32 x 8 thread tile covers (x, y); each thread walks a
// chunk of ZC planes, keeping the z-neighbours of its column in registers.
// No integer division; rows of the same class hit the same L1 lines.
// z planes per thread: long chunks on big levels (register reuse), short
// ones on coarse levels (parallelism).
inline int zchunk_for(long long n) { return n >= (8LL << 20) ? 16 : (n >= (1LL << 20) ? 4 : 2); }

// 7-point apply marching along z: a thread owns one (x, y) column of a
// z-chunk and keeps x at z-1, z, z+1 in registers.  The loads of U z-steps
// (class index, r, the four lateral neighbours and the next plane) are all
// issued before the arithmetic of those steps, so each thread has U cells of
// loads in flight.  Terms are summed p, b, s, w, e, n, t.
template <typename T, int MODE>
__global__ void __launch_bounds__(256) k_apply7z(int N, int M, int K, int zc, const int* __restrict__ cls,
                                                  const T* __restrict__ dict, const T* __restrict__ x,
                                                  T* __restrict__ r)
{
    constexpr int U = 4;
    const int ix = blockIdx.x * 32 + threadIdx.x;
    const int iy = blockIdx.y * 8 + threadIdx.y;
    if (ix >= N || iy >= M) return;
    const int NM = N * M;                                  // grids hold fewer than 2^31 cells
    const int z0 = blockIdx.z * zc;
    const int z1 = min(z0 + zc, K);
    int i = ix + N * iy + NM * z0;
    T xm = (z0 > 0) ? x[i - NM] : (T)0;
    T xc = x[i];
    const bool hasw = ix > 0, hase = ix < N - 1, hass = iy > 0, hasn = iy < M - 1;
    for (int zb = z0; zb < z1; zb += U, i += U * NM) {
        int cl[U];
        T rv[U], xs[U], xw[U], xe[U], xn[U], xp[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int z = zb + u;
            const int ii = (z < z1) ? i + u * NM : i;       // steps past the chunk reload a valid cell
            cl[u] = cls[ii];
            rv[u] = (MODE == 0) ? r[ii] : (T)0;
            xs[u] = hass ? x[ii - N] : (T)0;
            xw[u] = hasw ? x[ii - 1] : (T)0;
            xe[u] = hase ? x[ii + 1] : (T)0;
            xn[u] = hasn ? x[ii + N] : (T)0;
            xp[u] = (z < K - 1) ? x[ii + NM] : (T)0;
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (zb + u < z1) {
                const T* a = dict + (size_t)cl[u] * 7;
                T acc = a[3] * xc;
                acc += a[0] * xm;          // zero coefficient below the bottom wall
                if (hass) acc += a[1] * xs[u];
                if (hasw) acc += a[2] * xw[u];
                if (hase) acc += a[4] * xe[u];
                if (hasn) acc += a[5] * xn[u];
                acc += a[6] * xp[u];
                const int ii = i + u * NM;
                if (MODE == 0) r[ii] = rv[u] - acc;
                else r[ii] = acc;
                xm = xc;
                xc = xp[u];
            }
        }
    }
}

// Row of 27 coefficients stored with stride 28, read as 16-byte vectors.
template <typename T>
__device__ __forceinline__ void load_row28(const T* __restrict__ p, T (&a)[28])
{
    if constexpr (sizeof(T) == 4) {
        const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
        for (int k = 0; k < 7; k++) {
            const float4 v = __ldg(q + k);
            a[4 * k] = v.x;
            a[4 * k + 1] = v.y;
            a[4 * k + 2] = v.z;
            a[4 * k + 3] = v.w;
        }
    } else {
        const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
        for (int k = 0; k < 14; k++) {
            const double2 v = __ldg(q + k);
            a[2 * k] = v.x;
            a[2 * k + 1] = v.y;
        }
    }
}

// 27-point apply (Galerkin levels) marching along z.  dict28 holds each
// distinct row with stride 28 (the 27 box coefficients in z, y, x order and a
// zero), so a row is seven (FP32) or fourteen (FP64) vector loads.  The row
// stays in registers from one z-step to the next and a warp reloads only
// when one of its cells changes class (the kernel is bound by load
// instructions, and along z most columns keep their class).
template <typename T, int MODE>
__global__ void __launch_bounds__(256) k_apply27z(int N, int M, int K, int zc, const int* __restrict__ cls,
                                                   const T* __restrict__ dict28, const T* __restrict__ x,
                                                   T* __restrict__ r)
{
    const int ix = blockIdx.x * 32 + threadIdx.x;
    const int iy = blockIdx.y * 8 + threadIdx.y;
    if (ix >= N || iy >= M) return;
    const int NM = N * M;                                  // grids hold fewer than 2^31 cells
    const int z0 = blockIdx.z * zc;
    const int z1 = min(z0 + zc, K);
    const int col = ix + N * iy;
    bool ok[9];
    int off[9];
#pragma unroll
    for (int dy = -1; dy <= 1; dy++)
#pragma unroll
        for (int dx = -1; dx <= 1; dx++) {
            const int q = (dy + 1) * 3 + (dx + 1);
            ok[q] = (ix + dx >= 0) && (ix + dx < N) && (iy + dy >= 0) && (iy + dy < M);
            off[q] = dx + dy * N;
        }
    // plane values of the 3x3 column neighbourhood at z-1, z, z+1
    T pm[9], pc[9], pp[9];
    auto load_plane = [&](int z, T* p) {
        const bool zin = z >= 0 && z < K;
#pragma unroll
        for (int q = 0; q < 9; q++) p[q] = (zin && ok[q]) ? x[col + NM * z + off[q]] : (T)0;
    };
    load_plane(z0 - 1, pm);
    load_plane(z0, pc);
    int cn = cls[col + NM * z0];
    T rn = (MODE == 0) ? r[col + NM * z0] : (T)0;
    T a[28];
    int cprev = -1;
    const unsigned active = __activemask();               // lanes past the grid edge returned above
    for (int z = z0; z < z1; z++) {
        const int i = col + NM * z;
        const int cl = cn;
        const T rv = rn;
        load_plane(z + 1, pp);
        if (z + 1 < z1) {                                  // next step's class and residual, one step ahead
            cn = cls[i + NM];
            if (MODE == 0) rn = r[i + NM];
        }
        if (__any_sync(active, cl != cprev)) {
            if (cl != cprev) load_row28(dict28 + (size_t)cl * 28, a);
            cprev = cl;
        }
        T acc = 0;
#pragma unroll
        for (int q = 0; q < 9; q++) acc += a[q] * pm[q];
#pragma unroll
        for (int q = 0; q < 9; q++) acc += a[9 + q] * pc[q];
#pragma unroll
        for (int q = 0; q < 9; q++) acc += a[18 + q] * pp[q];
        if (MODE == 0) r[i] = rv - acc;
        else r[i] = acc;
#pragma unroll
        for (int q = 0; q < 9; q++) {
            pm[q] = pc[q];
            pc[q] = pp[q];
        }
    }
}

__global__ void k_pad_rows(long long nrows, int w, int wpad, const double* __restrict__ src, double* __restrict__ dst)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nrows * wpad;
         e += (long long)gridDim.x * blockDim.x) {
        const long long row = e / wpad;
        const int k = (int)(e - row * wpad);
        dst[e] = k < w ? src[row * w + k] : 0.0;
    }
}

template <typename T, int MODE>
__global__ void __launch_bounds__(256) k_applyboxd(int N, int M, int K, OffList ol, const int* __restrict__ cls,
                                                    const T* __restrict__ dict, const T* __restrict__ x,
                                                    T* __restrict__ r)
{
    const long long n = (long long)N * M * K;
    const int NM = N * M;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int ix, iy, iz;
        cell_xyz(i, N, NM, ix, iy, iz);
        const T* a = dict + (size_t)cls[i] * ol.n;
        T acc = 0;
        for (int o = 0; o < ol.n; o++) {
            const int jx = ix + ol.o[o][0], jy = iy + ol.o[o][1], jz = iz + ol.o[o][2];
            if (jx < 0 || jx >= N || jy < 0 || jy >= M || jz < 0 || jz >= K) continue;
            acc += a[o] * x[i + ol.o[o][0] + (long long)ol.o[o][1] * N + (long long)ol.o[o][2] * NM];
        }
        if (MODE == 0) r[i] -= acc;
        else r[i] = acc;
    }
}

// ---------------------------------------------------------------------------
// transfers (structured tensor-product operators, one 1-D table per axis)
// ---------------------------------------------------------------------------
// Prolongation table per fine index f: two (coarse index, weight) pairs.
struct PTab {
    const int* c;      // 2 per fine index
    const float* w;    // 2 per fine index (exact binary fractions)
};
// Restriction table per coarse index: up to 4 (fine index, weight) pairs.
struct RTab {
    const int* f;      // 4 per coarse index, -1 = unused
    const float* w;
};

// ch = P cHH and c = ch  (the prolongation plus the copy c.copy(m_ch) of
// MultiGridSolver::solve, multigrid_solver.h:65-66)
template <typename T, int ZC, bool ADD = false>
__global__ void __launch_bounds__(256) k_prolong(int N, int M, int K, int Nc, int Mc, PTab px, PTab py, PTab pz,
                                                 const T* __restrict__ coarse, T* __restrict__ ch, T* __restrict__ c)
{
    // block (32, 8) over (x, y); each thread ZC consecutive z.  All gathers of
    // the ZC cells are issued before any is summed (unused table slots hold
    // index 0 and weight 0, so every address is valid); the sum skips zero
    // weights and runs in the row order of P (z, y, x ascending).
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    if (x >= N || y >= M) return;
    const int z0 = blockIdx.z * ZC;
    const int NMc = Nc * Mc;
    float wx[2], wy[2];
    int ox[2], oy[2];
#pragma unroll
    for (int q = 0; q < 2; q++) {
        wx[q] = px.w[2 * x + q];
        ox[q] = px.c[2 * x + q];
        wy[q] = py.w[2 * y + q];
        oy[q] = py.c[2 * y + q] * Nc;
    }
    T g[ZC][8];
    float wz[ZC][2];
#pragma unroll
    for (int u = 0; u < ZC; u++) {
        const int z = min(z0 + u, K - 1);
#pragma unroll
        for (int a = 0; a < 2; a++) {
            wz[u][a] = pz.w[2 * z + a];
            const int oz = pz.c[2 * z + a] * NMc;
#pragma unroll
            for (int b = 0; b < 2; b++)
#pragma unroll
                for (int q = 0; q < 2; q++) g[u][4 * a + 2 * b + q] = coarse[oz + oy[b] + ox[q]];
        }
    }
#pragma unroll
    for (int u = 0; u < ZC; u++) {
        const int z = z0 + u;
        if (z >= K) break;
        T acc = 0;
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
            for (int b = 0; b < 2; b++)
#pragma unroll
                for (int q = 0; q < 2; q++)
                    if (wz[u][a] != 0.f && wy[b] != 0.f && wx[q] != 0.f)
                        acc += (T)(wz[u][a] * wy[b] * wx[q]) * g[u][4 * a + 2 * b + q];
        const int i = x + N * (y + M * z);                 // grids hold fewer than 2^31 cells
        if (ADD) {
            ch[i] += acc;                                  // correction added to the smoothed iterate
        } else {
            ch[i] = acc;
            if (c) c[i] = acc;                             // null: the one copy the fused smoother starts from
        }
    }
}

// coarse = R fine.  agglomerate: 1/8 of the 2x2x2 block (even-even-even
// class, summed in the reference's CSR order); otherwise R = P^T via tables.
template <typename T>
__global__ void k_restrict(int Nc, int Mc, int Kc, int N, int M, bool agglomerate, RTab rx, RTab ry, RTab rz,
                           const T* __restrict__ fine, T* __restrict__ coarse)
{
    const long long nc = (long long)Nc * Mc * Kc;
    const int NMc = Nc * Mc, NM = N * M;
    const CellIndex ci(Nc, NMc);
    for (long long I = blockIdx.x * (long long)blockDim.x + threadIdx.x; I < nc;
         I += (long long)gridDim.x * blockDim.x) {
        int X, Y, Z;
        ci.xyz(I, X, Y, Z);
        T acc = 0;
        if (agglomerate) {
            const long long f0 = (long long)(2 * Z) * NM + (2 * Y) * N + 2 * X;
            const T w = (T)0.125;
            acc += w * fine[f0];
            acc += w * fine[f0 + 1];
            acc += w * fine[f0 + N];
            acc += w * fine[f0 + N + 1];
            acc += w * fine[f0 + NM];
            acc += w * fine[f0 + NM + 1];
            acc += w * fine[f0 + NM + N];
            acc += w * fine[f0 + NM + N + 1];
        } else {
            for (int a = 0; a < 4; a++) {
                const int fz = rz.f[4 * Z + a];
                if (fz < 0) continue;
                const float wz = rz.w[4 * Z + a];
                for (int b = 0; b < 4; b++) {
                    const int fy = ry.f[4 * Y + b];
                    if (fy < 0) continue;
                    const float wy = ry.w[4 * Y + b];
                    for (int q = 0; q < 4; q++) {
                        const int fx = rx.f[4 * X + q];
                        if (fx < 0) continue;
                        acc += (T)(wz * wy * rx.w[4 * X + q]) * fine[(long long)fz * NM + fy * N + fx];
                    }
                }
            }
        }
        coarse[I] = acc;
    }
}

// Galerkin coarse operator A_H = R A P for one coarse cell per thread.  The
// box of the coarse stencil is (2rx+1)(2ry+1)(2rz+1), offsets ordered
// z-major, then y, then x (all in [-r, r]).  A is a box/offset-list stencil
// on the fine level.  Accumulation is in FP64.
__global__ void k_galerkin(int N, int M, int K, OffList fol, const double* __restrict__ Af, int Nc, int Mc,
                           int Kc, int crx, int cry, int crz, bool agglomerate, PTab px, PTab py, PTab pz,
                           RTab rx, RTab ry, RTab rz, double* __restrict__ Ac)
{
    const long long n = (long long)N * M * K;
    const long long nc = (long long)Nc * Mc * Kc;
    const int NMc = Nc * Mc;
    const int bx = 2 * crx + 1, by = 2 * cry + 1;
    const int nbox = bx * by * (2 * crz + 1);
    for (long long I = blockIdx.x * (long long)blockDim.x + threadIdx.x; I < nc;
         I += (long long)gridDim.x * blockDim.x) {
        int X, Y, Z;
        cell_xyz(I, Nc, NMc, X, Y, Z);
        double box[125];
        for (int q = 0; q < nbox; q++) box[q] = 0.0;
        // support of row I of R: 1-D lists
        int fxl[4], fyl[4], fzl[4];
        double wxl[4], wyl[4], wzl[4];
        int nx = 0, ny = 0, nz = 0;
        if (agglomerate) {
            fxl[0] = 2 * X; fxl[1] = 2 * X + 1; wxl[0] = wxl[1] = 0.5; nx = 2;
            fyl[0] = 2 * Y; fyl[1] = 2 * Y + 1; wyl[0] = wyl[1] = 0.5; ny = 2;
            fzl[0] = 2 * Z; fzl[1] = 2 * Z + 1; wzl[0] = wzl[1] = 0.5; nz = 2;
        } else {
            for (int a = 0; a < 4; a++) {
                if (rx.f[4 * X + a] >= 0) { fxl[nx] = rx.f[4 * X + a]; wxl[nx++] = rx.w[4 * X + a]; }
                if (ry.f[4 * Y + a] >= 0) { fyl[ny] = ry.f[4 * Y + a]; wyl[ny++] = ry.w[4 * Y + a]; }
                if (rz.f[4 * Z + a] >= 0) { fzl[nz] = rz.f[4 * Z + a]; wzl[nz++] = rz.w[4 * Z + a]; }
            }
        }
        for (int a = 0; a < nz; a++)
            for (int b = 0; b < ny; b++)
                for (int q = 0; q < nx; q++) {
                    const int fx = fxl[q], fy = fyl[b], fz = fzl[a];
                    const double rw = wzl[a] * wyl[b] * wxl[q];
                    const long long f = (long long)fz * N * M + (long long)fy * N + fx;
                    for (int o = 0; o < fol.n; o++) {
                        const int gx = fx + fol.o[o][0], gy = fy + fol.o[o][1], gz = fz + fol.o[o][2];
                        if (gx < 0 || gx >= N || gy < 0 || gy >= M || gz < 0 || gz >= K) continue;
                        const double a_fg = Af[(size_t)o * n + f];
                        if (a_fg == 0.0) continue;
                        const double ra = rw * a_fg;
                        for (int s = 0; s < 2; s++) {
                            const float wz = pz.w[2 * gz + s];
                            if (wz == 0.f) continue;
                            const int dz = pz.c[2 * gz + s] - Z;
                            for (int t = 0; t < 2; t++) {
                                const float wy = py.w[2 * gy + t];
                                if (wy == 0.f) continue;
                                const int dy = py.c[2 * gy + t] - Y;
                                for (int u = 0; u < 2; u++) {
                                    const float wx = px.w[2 * gx + u];
                                    if (wx == 0.f) continue;
                                    const int dx = px.c[2 * gx + u] - X;
                                    const int q2 = ((dz + crz) * by + (dy + cry)) * bx + (dx + crx);
                                    box[q2] += ra * ((double)wz * (double)wy * (double)wx);
                                }
                            }
                        }
                    }
                }
        for (int q = 0; q < nbox; q++) Ac[(size_t)q * nc + I] = box[q];
    }
}

// ---------------------------------------------------------------------------
// ADLJ line splitting
// ---------------------------------------------------------------------------
// Raw line tridiagonals (natural layout): for each stencil neighbour whose
// flat column equals i-NM, i-N, i-1, i, i+1, i+N, i+NM the value goes to the
// matching slot, exactly as SmootherADLJ::_k_build matches CSR columns
// (smoother_adlj.h:40-86).  lo_d[i] = coupling to the previous cell of the
// d-line of i, up_d[i] = to the next one, dg = diagonal (shared).
__global__ void k_adlj_extract(int N, int M, int K, OffList ol, const double* __restrict__ A,
                               double* __restrict__ dg, double* __restrict__ xlo, double* __restrict__ xup,
                               double* __restrict__ ylo, double* __restrict__ yup,
                               double* __restrict__ zlo, double* __restrict__ zup)
{
    const long long n = (long long)N * M * K;
    const int NM = N * M;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int ix, iy, iz;
        cell_xyz(i, N, NM, ix, iy, iz);
        double d = 0, xl = 0, xu = 0, yl = 0, yu = 0, zl = 0, zu = 0;
        for (int o = 0; o < ol.n; o++) {
            const int jx = ix + ol.o[o][0], jy = iy + ol.o[o][1], jz = iz + ol.o[o][2];
            if (jx < 0 || jx >= N || jy < 0 || jy >= M || jz < 0 || jz >= K) continue;
            const long long delta = ol.o[o][0] + (long long)ol.o[o][1] * N + (long long)ol.o[o][2] * NM;
            const double v = A[(size_t)o * n + i];
            if (delta == -NM) zl = v;
            else if (delta == -N) yl = v;
            else if (delta == -1) xl = v;
            else if (delta == 0) d = v;
            else if (delta == 1) xu = v;
            else if (delta == N) yu = v;
            else if (delta == NM) zu = v;
        }
        dg[i] = d;
        xlo[i] = xl; xup[i] = xu;
        ylo[i] = yl; yup[i] = yu;
        zlo[i] = zl; zup[i] = zu;
    }
}

__global__ void k_absmax(long long n, const double* __restrict__ a, double* partial, unsigned int* counter,
                         double* out)
{
    double m = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        m = fmax(m, fabs(a[i]));
    // max-reduce through the same partial buffer
    __shared__ double sh[32];
    __shared__ bool last;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t = fmax(t, sh[w]);
        partial[blockIdx.x] = t;
        __threadfence();
        last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double t = 0.0;
        for (int b = 0; b < (int)gridDim.x; b++) t = fmax(t, ((volatile double*)partial)[b]);
        *out = t;
        *counter = 0u;
    }
}

// Geometry of the lines of one direction in natural indexing:
//   cell of line l at position t = start(l) + t * stride
struct LineGeom {
    int N, M, K;
    int dir;        // 0 x, 1 y, 2 z
    __host__ __device__ long long nlines() const { return dir == 0 ? (long long)M * K : (dir == 1 ? (long long)N * K : (long long)N * M); }
    __host__ __device__ int len() const { return dir == 0 ? N : (dir == 1 ? M : K); }
};

__device__ __forceinline__ long long line_start(const LineGeom& g, long long l)
{
    if (g.dir == 0) return l * g.N;                                        // l = y + M z
    if (g.dir == 1) {                                                      // l = x + N z
        const long long z = l / g.N, x = l - z * g.N;
        return z * (long long)g.N * g.M + x;
    }
    return l;                                                              // l = x + N y
}
__device__ __forceinline__ long long line_stride(const LineGeom& g)
{
    return g.dir == 0 ? 1 : (g.dir == 1 ? g.N : (long long)g.N * g.M);
}

// Per-line LU of the line tridiagonals (TriDiagonalMatrix::triLU,
// tridiagonal_matrix.h:45-67) when no coupling crosses line ends: each line
// starts afresh.  dinv <- inverse pivots (0 below tiny), up <- up * dinv.
__global__ void k_trilu_lines(LineGeom g, const double* __restrict__ tinyp, const double* __restrict__ lo,
                              double* __restrict__ dinv, double* __restrict__ up)
{
    const long long nl = g.nlines();
    const int L = g.len();
    const long long st = line_stride(g);
    const double tiny = *tinyp;
    for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < nl;
         l += (long long)gridDim.x * blockDim.x) {
        long long i = line_start(g, l);
        double aux = dinv[i];
        double dprev = (fabs(aux) < tiny) ? 0.0 : 1.0 / aux;
        dinv[i] = dprev;
        for (int t = 1; t < L; t++) {
            const long long ip = i;
            i += st;
            const double e = up[ip] * dprev;
            up[ip] = e;
            aux = dinv[i] - lo[i] * e;
            dprev = (fabs(aux) < tiny) ? 0.0 : 1.0 / aux;
            dinv[i] = dprev;
        }
        up[i] *= dprev;   // coupling across the line end (zero unless aliased)
    }
}

// Serial LU over the whole direction order, for levels whose line ends are
// coupled (a dimension too small for the stencil, see k_adlj_extract).
__global__ void k_trilu_serial(LineGeom g, const double* __restrict__ tinyp, const double* __restrict__ lo,
                               double* __restrict__ dinv, double* __restrict__ up)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const double tiny = *tinyp;
    const long long nl = g.nlines();
    const int L = g.len();
    const long long st = line_stride(g);
    double dprev = 0.0;
    long long ip = -1;
    for (long long l = 0; l < nl; l++) {
        long long i = line_start(g, l);
        for (int t = 0; t < L; t++, i += st) {
            double aux = dinv[i];
            if (ip >= 0) {
                const double e = up[ip] * dprev;
                up[ip] = e;
                aux -= lo[i] * e;
            }
            dprev = (fabs(aux) < tiny) ? 0.0 : 1.0 / aux;
            dinv[i] = dprev;
            ip = i;
        }
    }
}

// Flags coupling across line ends: lo(start of line l+1) * up(end of line l).
__global__ void k_line_coupling(LineGeom g, const double* __restrict__ lo, const double* __restrict__ up,
                                int* flag)
{
    const long long nl = g.nlines();
    const int L = g.len();
    const long long st = line_stride(g);
    for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l + 1 < nl;
         l += (long long)gridDim.x * blockDim.x) {
        const long long iend = line_start(g, l) + (long long)(L - 1) * st;
        const long long inext = line_start(g, l + 1);
        if (lo[inext] != 0.0 && up[iend] != 0.0) atomicOr(flag, 1);
    }
}

// ---------------------------------------------------------------------------
// ADLJ line solves:  c = omega * T^{-1} r ;  ch += c
// ---------------------------------------------------------------------------

// y- and z-lines: one thread per line, neighbouring threads on neighbouring x
// (coalesced).  The forward sweep stores into c, the backward sweep finishes
// it in place.  quirk_first >= 0: natural index base of the z-line first
// right-hand side as the reference reads it (y*N*K + x), see header.
// The sweeps run in chunks of U cells: all loads of a chunk are issued before
// its dependent recurrence, so each thread keeps 3U loads in flight (the
// recurrence itself is latency bound, one FMA chain per line).
template <typename T>
__global__ void __launch_bounds__(128) k_tdma_strided(LineGeom g, bool zquirk, const T* __restrict__ lo,
                                                       const T* __restrict__ dinv, const T* __restrict__ up,
                                                       const T* __restrict__ r, T* __restrict__ c,
                                                       T* __restrict__ ch, T omega)
{
    constexpr int U = 8;
    const long long nl = g.nlines();
    const int L = g.len();
    const long long st = line_stride(g);
    for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < nl;
         l += (long long)gridDim.x * blockDim.x) {
        const long long i0 = line_start(g, l);
        T rhs0;
        if (zquirk) {
            // line l = x + N*y; the reference reads right_member[y*N*K + x]
            const long long y = l / g.N, x = l - y * g.N;
            rhs0 = r[y * (long long)g.N * g.K + x];
        } else {
            rhs0 = r[i0];
        }
        // forward: y_t = (r_t - lo_t y_{t-1}) * dinv_t, stored in c.  The loads
        // of chunk k+1 are issued before the recurrence of chunk k.
        T yv = 0;
        T rr[U], ll[U], dd[U], rn[U], ln[U], dn[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (u < L) {
                const long long i = i0 + (long long)u * st;
                rn[u] = (u == 0) ? rhs0 : r[i];
                ln[u] = lo[i];
                dn[u] = dinv[i];
            }
        }
        for (int t0 = 0; t0 < L; t0 += U) {
#pragma unroll
            for (int u = 0; u < U; u++) {
                rr[u] = rn[u];
                ll[u] = ln[u];
                dd[u] = dn[u];
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int t = t0 + U + u;
                if (t < L) {
                    const long long i = i0 + (long long)t * st;
                    rn[u] = r[i];
                    ln[u] = lo[i];
                    dn[u] = dinv[i];
                }
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int t = t0 + u;
                if (t < L) {
                    yv = (t == 0) ? rr[u] * dd[u] : (rr[u] - ll[u] * yv) * dd[u];
                    c[i0 + (long long)t * st] = yv;
                }
            }
        }
        // backward: x_t = y_t - up_t x_{t+1};  c = omega x ; ch += c
        T xv = 0;
        T yy[U], uu[U], hh[U], yn[U], un[U], hn[U];
        const int tl = L - 1;
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int t = tl - u;
            if (t >= 0) {
                const long long i = i0 + (long long)t * st;
                yn[u] = (u == 0) ? yv : c[i];
                un[u] = up[i];
                hn[u] = ch[i];
            }
        }
        for (int t1 = tl; t1 >= 0; t1 -= U) {
#pragma unroll
            for (int u = 0; u < U; u++) {
                yy[u] = yn[u];
                uu[u] = un[u];
                hh[u] = hn[u];
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int t = t1 - U - u;
                if (t >= 0) {
                    const long long i = i0 + (long long)t * st;
                    yn[u] = c[i];
                    un[u] = up[i];
                    hn[u] = ch[i];
                }
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int t = t1 - u;
                if (t >= 0) {
                    xv = (t == tl) ? yy[u] : yy[u] - uu[u] * xv;
                    const T cv = omega * xv;
                    const long long i = i0 + (long long)t * st;
                    c[i] = cv;
                    ch[i] = hh[u] + cv;
                }
            }
        }
    }
}

// Inclusive scan of the segment maps y = A + B y_in along the segment index
// (threadIdx.y) of each line (threadIdx.x), Kogge-Stone in shared memory
// with two buffers: log2(S) steps.  REV scans from the last segment down
// (backward recurrence).  Returns the composed map of the segments before
// this one (exclusive), as (A, B).
template <typename T, bool REV>
__device__ __forceinline__ void seg_scan(T& a, T& b, T* sA, T* sB)
{
    const int W = blockDim.x, S = blockDim.y;
    const int w = threadIdx.x, sg = threadIdx.y;
    const int q = REV ? S - 1 - sg : sg;                  // position along the scan
    int cur = 0;
    sA[sg * W + w] = a;
    sB[sg * W + w] = b;
    __syncthreads();
    for (int off = 1; off < S; off <<= 1) {
        T na = a, nb = b;
        if (q >= off) {
            const int src = (REV ? sg + off : sg - off) * W + w;
            const T pa = sA[cur * W * S + src], pb = sB[cur * W * S + src];
            na = a + b * pa;
            nb = b * pb;
        }
        a = na;
        b = nb;
        cur ^= 1;
        sA[cur * W * S + sg * W + w] = a;
        sB[cur * W * S + sg * W + w] = b;
        __syncthreads();
    }
    // exclusive: the inclusive result of the neighbour before this segment
    if (q == 0) {
        a = 0;
        b = 1;
    } else {
        const int src = (REV ? sg + 1 : sg - 1) * W + w;
        a = sA[cur * W * S + src];
        b = sB[cur * W * S + src];
    }
}

// y- and z-lines, segmented.  A CTA holds W neighbouring lines (consecutive
// x, so each warp load is a contiguous row piece) split into S = ceil(L/SEG)
// segments, one thread per (line, segment).  Every thread issues all loads of
// its segment (r, lo, dinv, up, ch) before any arithmetic, so the whole line
// is one memory round trip.  Within a segment the forward recurrence
//   y_t = (r_t - lo_t y_{t-1}) dinv_t
// is kept as affine maps of the value entering the segment, y_t = A_t + B_t y_in,
// and the backward one x_t = y_t - up_t x_{t+1} as x_t = G_t + H_t x_out; the
// S segment maps of a line are composed through shared memory by log-step
// scans (SCAN), or by each thread walking the maps before its own.  Shared
// memory: 4 W S values.
template <typename T, int SEG, int MAXT, int MINB, bool SCAN = true>
__global__ void __launch_bounds__(MAXT, MINB) k_tdma_seg(LineGeom g, bool zquirk, const T* __restrict__ lo,
                                                         const T* __restrict__ dinv, const T* __restrict__ up,
                                                         const T* __restrict__ r, T* __restrict__ c,
                                                         T* __restrict__ ch, T omega)
{
    extern __shared__ __align__(16) unsigned char seg_smem[];
    const int W = blockDim.x, S = blockDim.y;
    T* sA = reinterpret_cast<T*>(seg_smem);
    T* sB = sA + W * S;
    const int w = threadIdx.x, sg = threadIdx.y;
    const int L = g.len();
    const long long st = line_stride(g);
    const int gx = (g.N + W - 1) / W;
    const int row = blockIdx.x / gx;                       // z for y-lines, y for z-lines
    const int x = (blockIdx.x - row * gx) * W + w;
    const bool valid = x < g.N;
    const int xs = valid ? x : g.N - 1;                    // idle lanes load a valid line, store nothing
    const long long i0 = line_start(g, (long long)row * g.N + xs);
    const int t0 = sg * SEG;
    T rv[SEG], lv[SEG], dv[SEG], uv[SEG], hv[SEG];
#pragma unroll
    for (int u = 0; u < SEG; u++) {
        const int t = min(t0 + u, L - 1);
        const long long i = i0 + (long long)t * st;
        rv[u] = r[i];
        lv[u] = lo[i];
        dv[u] = dinv[i];
        uv[u] = up[i];
        hv[u] = ch[i];
    }
    if (zquirk && sg == 0) rv[0] = r[(long long)row * g.N * g.K + xs];   // reference z-line quirk (y*N*K + x)
    // forward, relative to y_in
    T a = 0, b = 1;
#pragma unroll
    for (int u = 0; u < SEG; u++) {
        const int t = t0 + u;
        if (t < L) {
            if (t == 0) {
                a = rv[u] * dv[u];
                b = 0;
            } else {
                a = (rv[u] - lv[u] * a) * dv[u];
                b = -(lv[u] * b) * dv[u];
            }
        }
        rv[u] = a;
        lv[u] = b;
    }
    T yin = 0;
    if constexpr (SCAN) {
        seg_scan<T, false>(a, b, sA, sA + 2 * W * S);
        yin = a;
    } else {
        sA[sg * W + w] = a;
        sB[sg * W + w] = b;
        __syncthreads();
        for (int q = 0; q < sg; q++) yin = sA[q * W + w] + sB[q * W + w] * yin;
    }
    __syncthreads();
    // backward, relative to x_out
    T gg = 0, hh = 1;
#pragma unroll
    for (int u = SEG - 1; u >= 0; u--) {
        const int t = t0 + u;
        if (t < L) {
            const T yv = rv[u] + lv[u] * yin;
            if (t == L - 1) {
                gg = yv;
                hh = 0;
            } else {
                gg = yv - uv[u] * gg;
                hh = -(uv[u] * hh);
            }
        }
        rv[u] = gg;
        lv[u] = hh;
    }
    T xo = 0;
    if constexpr (SCAN) {
        seg_scan<T, true>(gg, hh, sA, sA + 2 * W * S);
        xo = gg;
    } else {
        sA[sg * W + w] = gg;
        sB[sg * W + w] = hh;
        __syncthreads();
        for (int q = S - 1; q > sg; q--) xo = sA[q * W + w] + sB[q * W + w] * xo;
    }
    if (valid) {
#pragma unroll
        for (int u = 0; u < SEG; u++) {
            const int t = t0 + u;
            if (t < L) {
                const long long i = i0 + (long long)t * st;
                const T cv = omega * (rv[u] + lv[u] * xo);
                c[i] = cv;
                ch[i] = hv[u] + cv;
            }
        }
    }
}

// x-lines of power-of-two length L = P * SEG (P <= 32 lanes per line): every
// thread owns SEG consecutive cells of a line and reads them with 16-byte
// vector loads (all loads before any arithmetic, one memory round trip).  The
// segment maps y = A + B y_in (forward) and x = G + H x_out (backward) are
// chained across the P lanes of a line by warp shuffle scans of width P, so a
// line costs one scan each way instead of one per 32 cells, and the forward
// values never leave registers.
template <typename T, int SEG>
__device__ __forceinline__ void load_seg(const T* __restrict__ p, T (&v)[SEG])
{
    if constexpr (sizeof(T) == 4) {
        static_assert(SEG % 4 == 0, "FP32 segments are whole float4s");
#pragma unroll
        for (int k = 0; k < SEG / 4; k++) {
            const float4 q = *reinterpret_cast<const float4*>(p + 4 * k);
            v[4 * k] = q.x;
            v[4 * k + 1] = q.y;
            v[4 * k + 2] = q.z;
            v[4 * k + 3] = q.w;
        }
    } else {
        static_assert(SEG % 2 == 0, "FP64 segments are whole double2s");
#pragma unroll
        for (int k = 0; k < SEG / 2; k++) {
            const double2 q = *reinterpret_cast<const double2*>(p + 2 * k);
            v[2 * k] = q.x;
            v[2 * k + 1] = q.y;
        }
    }
}

template <typename T, int SEG>
__device__ __forceinline__ void store_seg(T* __restrict__ p, const T (&v)[SEG])
{
    if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (int k = 0; k < SEG / 4; k++)
            *reinterpret_cast<float4*>(p + 4 * k) = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
    } else {
#pragma unroll
        for (int k = 0; k < SEG / 2; k++) *reinterpret_cast<double2*>(p + 2 * k) = make_double2(v[2 * k], v[2 * k + 1]);
    }
}

template <typename T, int SEG>
__global__ void __launch_bounds__(256) k_tdma_xseg(int L, int P, long long nlines, const T* __restrict__ lo,
                                                    const T* __restrict__ dinv, const T* __restrict__ up,
                                                    const T* __restrict__ r, T* __restrict__ c, T* __restrict__ ch,
                                                    T omega)
{
    // whole warps stay in the loop so every shuffle has its full group
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long line = tid / P;
    const int q = (int)(tid - line * P);
    const bool valid = line < nlines;
    const long long base = (valid ? line : 0) * L + (long long)q * SEG;
    T rv[SEG], lv[SEG], dv[SEG], uv[SEG], hv[SEG];
    load_seg<T, SEG>(r + base, rv);
    load_seg<T, SEG>(lo + base, lv);
    load_seg<T, SEG>(dinv + base, dv);
    load_seg<T, SEG>(up + base, uv);
    load_seg<T, SEG>(ch + base, hv);
    // forward: y_t = (r_t - lo_t y_{t-1}) dinv_t relative to the segment input
    T a = 0, b = 1;
#pragma unroll
    for (int u = 0; u < SEG; u++) {
        if (q == 0 && u == 0) {
            a = rv[0] * dv[0];
            b = 0;
        } else {
            a = (rv[u] - lv[u] * a) * dv[u];
            b = -(lv[u] * b) * dv[u];
        }
        rv[u] = a;
        lv[u] = b;
    }
    // inclusive scan of the segment maps over the P lanes of the line
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        if (o >= P) break;
        const T a2 = __shfl_up_sync(0xffffffffu, a, o, P);
        const T b2 = __shfl_up_sync(0xffffffffu, b, o, P);
        if (q >= o) {
            a = a + b * a2;
            b = b * b2;
        }
    }
    T yin = __shfl_up_sync(0xffffffffu, a, 1, P);
    if (q == 0) yin = 0;
    // backward: x_t = y_t - up_t x_{t+1} relative to the segment output
    T g = 0, hh = 1;
#pragma unroll
    for (int u = SEG - 1; u >= 0; u--) {
        const T yv = rv[u] + lv[u] * yin;
        if (q == P - 1 && u == SEG - 1) {
            g = yv;
            hh = 0;
        } else {
            g = yv - uv[u] * g;
            hh = -(uv[u] * hh);
        }
        rv[u] = g;
        lv[u] = hh;
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        if (o >= P) break;
        const T g2 = __shfl_down_sync(0xffffffffu, g, o, P);
        const T h2 = __shfl_down_sync(0xffffffffu, hh, o, P);
        if (q + o < P) {
            g = g + hh * g2;
            hh = hh * h2;
        }
    }
    T xout = __shfl_down_sync(0xffffffffu, g, 1, P);
    if (q == P - 1) xout = 0;
    if (!valid) return;
#pragma unroll
    for (int u = 0; u < SEG; u++) {
        const T cv = omega * (rv[u] + lv[u] * xout);
        rv[u] = cv;
        hv[u] = hv[u] + cv;
    }
    store_seg<T, SEG>(c + base, rv);
    store_seg<T, SEG>(ch + base, hv);
}

// x-lines: one warp per line.  The forward recurrence y_t = D_t r_t -
// D_t lo_t y_{t-1} and the backward one x_t = y_t - up_t x_{t+1} are affine;
// each round of 32 consecutive cells is solved by a warp scan of affine maps
// (a, b) o (a', b') = (a + b a', b b'), carrying the last value between rounds.
template <typename T>
__global__ void __launch_bounds__(256) k_tdma_xwarp(int N, long long nlines, const T* __restrict__ lo,
                                                     const T* __restrict__ dinv, const T* __restrict__ up,
                                                     const T* __restrict__ r, T* __restrict__ c,
                                                     T* __restrict__ ch, T omega)
{
    const int lane = threadIdx.x & 31;
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const int rounds = (N + 31) >> 5;
    for (long long l = warp; l < nlines; l += nwarps) {
        const long long base = l * N;
        T carry = 0;
        // forward, with the next round's loads issued before this round's scan
        T nr = 0, nd = 1, nl = 0;
        if (lane < N) {
            nr = r[base + lane];
            nd = dinv[base + lane];
            nl = lo[base + lane];
        }
        for (int rd = 0; rd < rounds; rd++) {
            const int t = rd * 32 + lane;
            const T rv = nr, D = nd, lv = nl;
            const int tn = t + 32;
            if (tn < N) {
                nr = r[base + tn];
                nd = dinv[base + tn];
                nl = lo[base + tn];
            }
            T a = 0, b = 1;
            if (t < N) {
                a = rv * D;
                b = (t == 0) ? (T)0 : -lv * D;
            }
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const T a2 = __shfl_up_sync(0xffffffffu, a, o);
                const T b2 = __shfl_up_sync(0xffffffffu, b, o);
                if (lane >= o) {
                    a = a + b * a2;
                    b = b * b2;
                }
            }
            const T yv = a + b * carry;
            if (t < N) c[base + t] = yv;
            carry = __shfl_sync(0xffffffffu, yv, 31);
        }
        __syncwarp();
        carry = 0;
        T ny = 0, nu = 0, nh = 0;
        {
            const int t = N - 1 - lane;
            if (t >= 0) {
                ny = c[base + t];
                nu = up[base + t];
                nh = ch[base + t];
            }
        }
        for (int rd = 0; rd < rounds; rd++) {
            const int t = N - 1 - (rd * 32 + lane);
            const T yv = ny, uv = nu, hv = nh;
            const int tn = t - 32;
            if (tn >= 0) {
                ny = c[base + tn];
                nu = up[base + tn];
                nh = ch[base + tn];
            }
            T a = 0, b = 1;
            if (t >= 0) {
                a = yv;
                b = (t == N - 1) ? (T)0 : -uv;
            }
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const T a2 = __shfl_up_sync(0xffffffffu, a, o);
                const T b2 = __shfl_up_sync(0xffffffffu, b, o);
                if (lane >= o) {
                    a = a + b * a2;
                    b = b * b2;
                }
            }
            const T xv = a + b * carry;
            carry = __shfl_sync(0xffffffffu, xv, 31);
            if (t >= 0) {
                const T cv = omega * xv;
                c[base + t] = cv;
                ch[base + t] = hv + cv;
            }
        }
    }
}

// Coarsest-grid solve with the stored scaled/permuted LU factors
// (LUDecompositionSparseMatrix DirectGauss/InverseGauss,
// lu_decomposition_sparse_matrix.h:238-259): one thread, n is tiny.
template <typename T>
__global__ void k_coarse_solve(int n, const double* __restrict__ L, const double* __restrict__ U,
                               const double* __restrict__ scale, const int* __restrict__ perm,
                               const T* __restrict__ b, T* __restrict__ ch, double* __restrict__ work)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double* y = work;
    double* z = work + n;
    for (int i = 0; i < n; i++) {
        double aux = scale[perm[i]] * (double)b[perm[i]];
        for (int j = 0; j < i; j++) aux -= L[i * n + j] * y[j];
        y[i] = aux;
    }
    for (int i = n - 1; i >= 0; i--) {
        double aux = y[i];
        for (int j = i + 1; j < n; j++) aux -= U[i * n + j] * z[j];
        z[i] = aux / U[i * n + i];
    }
    for (int i = 0; i < n; i++) ch[i] = (T)(scale[i] * z[i]);
}

}  // namespace lsg

namespace lsg {

// ---------------------------------------------------------------------------
// Cut-cell Laplace operator from the geometry (restatement of
// LaplaceDiscreteOperator::calcLap, laplace_discrete_operator.h:107-686, and
// fixPointFlow :809-821).  Face coefficient  a_f = (theta_f dS_f)^2 / M_f
// with the face fraction of the shared face (west/south/bottom read from the
// neighbour's east/north/top), 1/M from the staggered x/y/z grids; a fully
// fluid cell uses dS_f^2 / M_f; the faces on the box walls named by a
// boundary cell type are absent; diagonal = -(a_b + a_s + a_w + a_e + a_n +
// a_t) summed in that order; a solid cell has only PLUS_TINY on the diagonal;
// the two pinned rows become identity rows.  Planes: b s w p e n t.
// Cell type codes (cut_cells.h): SolidCell 0, FluidCell 11111111, box
// boundary types -2 .. -27.
// ---------------------------------------------------------------------------
__host__ __device__ inline int absent_faces(int type)
{
    // bit 0 b, 1 s, 2 w, 3 e, 4 n, 5 t
    constexpr int B = 1, S = 2, W = 4, E = 8, Nn = 16, T = 32;
    switch (type) {
    case -2: return T;
    case -3: return B;
    case -4: return Nn;
    case -5: return S;
    case -6: return E;
    case -7: return W;
    case -8: return T | Nn;
    case -9: return T | S;
    case -10: return T | E;
    case -11: return T | W;
    case -12: return B | Nn;
    case -13: return B | S;
    case -14: return B | E;
    case -15: return B | W;
    case -16: return Nn | E;
    case -17: return Nn | W;
    case -18: return S | E;
    case -19: return S | W;
    case -20: return T | Nn | E;
    case -21: return T | Nn | W;
    case -22: return T | S | E;
    case -23: return T | S | W;
    case -24: return B | Nn | E;
    case -25: return B | Nn | W;
    case -26: return B | S | E;
    case -27: return B | S | W;
    default: return 0;
    }
}

__global__ void k_laplace_from_geometry(int N, int M, int K, const int* __restrict__ type,
                                        const double* __restrict__ theta, const double* __restrict__ delta,
                                        const double* __restrict__ inv_mx, const double* __restrict__ inv_my,
                                        const double* __restrict__ inv_mz, long long pin0, long long pin1,
                                        double* __restrict__ planes)
{
    const long long n = (long long)N * M * K;
    const long long NM = (long long)N * M;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        double a[7] = {0, 0, 0, 0, 0, 0, 0};
        const int ty = type[i];
        if (i == pin0 || i == pin1) {
            a[3] = 1.0;
        } else if (ty == 0) {
            a[3] = 1e-16;                                   // PLUS_TINY
        } else {
            const int iz = (int)(i / NM);
            const long long rem = i - (long long)iz * NM;
            const int iy = (int)(rem / N);
            const long long numX = i - iy - (long long)iz * M;   // x-grid cell east of i
            const long long numY = i - (long long)iz * N;        // y-grid cell north of i
            const double dx = delta[3 * i], dy = delta[3 * i + 1], dz = delta[3 * i + 2];
            const double dyz = dy * dz, dxz = dx * dz, dxy = dx * dy;
            const int miss = absent_faces(ty);
            const bool fluid = (ty == 11111111);
            double ab = 0, as = 0, aw = 0, ae = 0, an = 0, at = 0;
            auto coef = [&](double th, double ds, double inv) {
                const double aux = fluid ? ds : th * ds;
                return aux * aux * inv;
            };
            if (!(miss & 1)) ab = coef(theta[3 * (i - NM) + 2], dxy, inv_mz[i - NM]);
            if (!(miss & 2)) as = coef(theta[3 * (i - N) + 1], dxz, inv_my[numY - N]);
            if (!(miss & 4)) aw = coef(theta[3 * (i - 1)], dyz, inv_mx[numX - 1]);
            if (!(miss & 8)) ae = coef(theta[3 * i], dyz, inv_mx[numX]);
            if (!(miss & 16)) an = coef(theta[3 * i + 1], dxz, inv_my[numY]);
            if (!(miss & 32)) at = coef(theta[3 * i + 2], dxy, inv_mz[i]);
            double dg = 0.0;
            bool first = true;
            const double vals[6] = {ab, as, aw, ae, an, at};
#pragma unroll
            for (int f = 0; f < 6; f++) {
                if (miss & (1 << f)) continue;
                dg = first ? -vals[f] : dg - vals[f];
                first = false;
            }
            a[0] = ab; a[1] = as; a[2] = aw; a[3] = dg; a[4] = ae; a[5] = an; a[6] = at;
        }
#pragma unroll
        for (int s = 0; s < 7; s++) planes[(size_t)s * n + i] = a[s];
    }
}

}  // namespace lsg

namespace lsg {

// ---------------------------------------------------------------------------
// Multi-colour point Gauss-Seidel (the red-black smoother variant; no
// counterpart in the reference, whose smoother is ADLJ).  One launch per
// colour updates every cell of that colour in place,
//   x_i = (b_i - sum_{j != i} a_ij x_j) * dinv_i,
// dinv_i = 1 / a_ii, or 0 on rows whose pivot is below the level's tiny
// threshold (solid and sealed cells keep their value).  Cells of one colour
// never couple: 7-point rows use the parity of x + y + z (red-black), 27-point
// box rows the parities of x, y and z (8 colours).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_gs_dinv(long long n, const double* __restrict__ diag, const double* __restrict__ tinyp,
                          T* __restrict__ dinv)
{
    const double tiny = *tinyp;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double d = diag[i];
        dinv[i] = (T)(fabs(d) < tiny ? 0.0 : 1.0 / d);
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_gs_rb7(int N, int M, int K, int color, const int* __restrict__ cls,
                                                const T* __restrict__ dict, const T* __restrict__ dinv,
                                                const T* __restrict__ b, T* __restrict__ x)
{
    const int xh = blockIdx.x * 32 + threadIdx.x;
    const int iy = blockIdx.y * 8 + threadIdx.y;
    const int iz = blockIdx.z;
    const int ix = 2 * xh + ((iy + iz + color) & 1);
    if (ix >= N || iy >= M) return;
    const int NM = N * M;
    const int i = ix + N * iy + NM * iz;
    const T di = dinv[i];
    if (di == (T)0) return;
    const T* a = dict + (size_t)cls[i] * 7;
    T acc = b[i];
    if (iz > 0) acc -= a[0] * x[i - NM];
    if (iy > 0) acc -= a[1] * x[i - N];
    if (ix > 0) acc -= a[2] * x[i - 1];
    if (ix < N - 1) acc -= a[4] * x[i + 1];
    if (iy < M - 1) acc -= a[5] * x[i + N];
    if (iz < K - 1) acc -= a[6] * x[i + NM];
    x[i] = acc * di;
}

template <typename T>
__global__ void __launch_bounds__(256) k_gs_box27(int N, int M, int K, int color, const int* __restrict__ cls,
                                                  const T* __restrict__ dict28, const T* __restrict__ dinv,
                                                  const T* __restrict__ b, T* __restrict__ x)
{
    const int ix = 2 * (blockIdx.x * 32 + threadIdx.x) + (color & 1);
    const int iy = 2 * (blockIdx.y * 8 + threadIdx.y) + ((color >> 1) & 1);
    const int iz = 2 * blockIdx.z + ((color >> 2) & 1);
    if (ix >= N || iy >= M || iz >= K) return;
    const int NM = N * M;
    const int i = ix + N * iy + NM * iz;
    const T di = dinv[i];
    if (di == (T)0) return;
    T a[28];
    load_row28(dict28 + (size_t)cls[i] * 28, a);
    T acc = b[i];
#pragma unroll
    for (int dz = -1; dz <= 1; dz++)
#pragma unroll
        for (int dy = -1; dy <= 1; dy++)
#pragma unroll
            for (int dx = -1; dx <= 1; dx++) {
                if (dx == 0 && dy == 0 && dz == 0) continue;
                const bool ok = ix + dx >= 0 && ix + dx < N && iy + dy >= 0 && iy + dy < M && iz + dz >= 0 &&
                                iz + dz < K;
                if (ok) acc -= a[(dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)] * x[i + dz * NM + dy * N + dx];
            }
    x[i] = acc * di;
}

// damped point Jacobi for levels with wider (mixed-parity) stencils:
// x += 0.8 dinv (b - A x), with t = b - A x computed by the caller
template <typename T>
__global__ void k_jacobi_update(long long n, const T* __restrict__ dinv, const T* __restrict__ t, T* __restrict__ x)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        x[i] += (T)0.8 * dinv[i] * t[i];
}

template <typename T>
__global__ void k_sub_from(long long n, const T* __restrict__ b, T* __restrict__ t)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        t[i] = b[i] - t[i];
}

}  // namespace lsg
