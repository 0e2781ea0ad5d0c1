// FP64 Krylov kernels: fused SpMV/residual + reductions, modified
// Gram-Schmidt steps, Givens rotations and the solution update of FGMRES
// (Base/Solvers/FGMRES/fgmres_interface.h:78-168), and the fused vector
// updates of BiCGStab (Base/Solvers/BiCGStab/bicgstab_interface.h:39-111).
// The Hessenberg/Givens bookkeeping lives in device memory (KrylovScalars) so
// that no per-dot host round trip is needed.
#pragma once

#include "lsg_kernels.cuh"

namespace lsg {

// w = b - A x  and  out[0] = ||w||^2   (setProductWithResidual,
// real_valued_mesh_function.h:203-211, 245-256)
__global__ void __launch_bounds__(256) k_residual7(int N, int M, int K, const int* __restrict__ cls, const double* __restrict__ dict,
                                                    const double* __restrict__ x, const double* __restrict__ b,
                                                    double* __restrict__ w, double* partial,
                                                    unsigned int* counter, double* out)
{
    const long long n = (long long)N * M * K;
    const int NM = N * M;
    double s[1] = {0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int ix, iy, iz;
        cell_xyz(i, N, NM, ix, iy, iz);
        const double* a = dict + (size_t)cls[i] * 7;
        double acc = a[3] * x[i];
        if (iz > 0) acc += a[0] * x[i - NM];
        if (iy > 0) acc += a[1] * x[i - N];
        if (ix > 0) acc += a[2] * x[i - 1];
        if (ix < N - 1) acc += a[4] * x[i + 1];
        if (iy < M - 1) acc += a[5] * x[i + N];
        if (iz < K - 1) acc += a[6] * x[i + NM];
        const double v = b[i] - acc;
        w[i] = v;
        s[0] += v * v;
    }
    grid_reduce<1>(s, partial, counter, out);
}

// w = A z  and  H[0,j] = (w, v0)   (z in FP64, or FP32 widened exactly)
template <typename Tz>
__global__ void __launch_bounds__(256) k_spmv_dot7(int N, int M, int K, const int* __restrict__ cls, const double* __restrict__ dict,
                                                    const Tz* __restrict__ z, const double* __restrict__ v0,
                                                    double* __restrict__ w, double* partial,
                                                    unsigned int* counter, double* out)
{
    const long long n = (long long)N * M * K;
    const int NM = N * M;
    double s[1] = {0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int ix, iy, iz;
        cell_xyz(i, N, NM, ix, iy, iz);
        const double* a = dict + (size_t)cls[i] * 7;
        double acc = a[3] * (double)z[i];
        if (iz > 0) acc += a[0] * (double)z[i - NM];
        if (iy > 0) acc += a[1] * (double)z[i - N];
        if (ix > 0) acc += a[2] * (double)z[i - 1];
        if (ix < N - 1) acc += a[4] * (double)z[i + 1];
        if (iy < M - 1) acc += a[5] * (double)z[i + N];
        if (iz < K - 1) acc += a[6] * (double)z[i + NM];
        w[i] = acc;
        s[0] += acc * v0[i];
    }
    grid_reduce<1>(s, partial, counter, out);
}

// One modified Gram-Schmidt step fused with the next dot:
//   w -= h_prev * vprev ;  out = (w, vnext)   (vnext == w gives ||w||^2)
__global__ void __launch_bounds__(256) k_mgs_step(long long n, const double* __restrict__ hprev,
                                                   const double* __restrict__ vprev,
                                                   const double* __restrict__ vnext, double* __restrict__ w,
                                                   bool norm_only, double* partial, unsigned int* counter,
                                                   double* out)
{
    const double h = *hprev;
    double s[1] = {0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double v = w[i] - h * vprev[i];
        w[i] = v;
        s[0] += norm_only ? v * v : v * vnext[i];
    }
    grid_reduce<1>(s, partial, counter, out);
}

// v = w / ||w||  (copyTo(curV, normW), mesh_function.h:256-260) and the
// preconditioner right-hand side in its precision.
template <typename T>
__global__ void k_scale_copy(long long n, const double* __restrict__ w, const double* __restrict__ invnorm,
                             double* __restrict__ v, T* __restrict__ rhs)
{
    const double s = *invnorm;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double t = w[i] * s;
        v[i] = t;
        rhs[i] = (T)t;
    }
}

// Givens update of Hessenberg column j and the residual estimate
// (fgmres_interface.h:103-135).  Runs on one thread.
__global__ void k_givens(KrylovScalars* ks, int j, int ldh, double eps, int max_it, volatile int* host_flag,
                         volatile double* host_norm)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double* H = ks->H + (size_t)j * ldh;
    double curH = H[0];
    for (int i = 0; i < j; i++) {
        const double c = ks->cs[i], s = ks->sn[i];
        const double nextH = H[i + 1];
        H[i] = c * curH - s * nextH;
        curH = s * curH + c * nextH;
    }
    const double normW = sqrt(ks->normW2);
    const double curC0 = curH * curH + normW * normW;
    const double curA = sqrt(curC0);
    double curC = 1.0 / curA;
    const double curS = -normW * curC;
    curC *= curH;
    H[j] = curA;
    ks->y[j] = curC * ks->norm_r;
    ks->norm_r *= curS;
    const double g = fabs(ks->norm_r);
    ks->invNormW = 1.0 / normW;
    int done = 0;
    if ((g > eps) && (ks->it < max_it)) {
        ks->cs[j] = curC;
        ks->sn[j] = curS;
        ks->it++;            // the inner loop's  it++
    } else {
        done = 1;
        ks->norm_r = g;
    }
    if (!(curA > 0.0) || isnan(g)) ks->breakdown = 1;
    ks->done = done;
    *host_norm = g;
    __threadfence_system();
    *host_flag = done ? 2 : 1;
}

// Back substitution of the triangular Hessenberg (solUpdate,
// fgmres_interface.h:153-168): coefficients of  x += sum_k coef_k z_k.
__global__ void k_backsub(KrylovScalars* ks, int last, int ldh, double* coef)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double y[64];
    for (int k = 0; k <= last; k++) y[k] = ks->y[k];
    for (int k = last; k >= 0; k--) {
        const double* Hk = ks->H + (size_t)k * ldh;
        const double curY = y[k] / Hk[k];
        for (int i = k - 1; i >= 0; i--) y[i] -= curY * Hk[i];
        coef[k] = curY;
    }
}

// x += sum_k coef_k z_k over nz basis vectors (stride n).
template <typename Tz>
__global__ void __launch_bounds__(256) k_multi_axpy(long long n, long long ld, int nz, const double* __restrict__ coef,
                                                     const Tz* __restrict__ Z, double* __restrict__ x)
{
    __shared__ double cf[64];
    if (threadIdx.x < nz) cf[threadIdx.x] = coef[threadIdx.x];
    __syncthreads();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        double acc = x[i];
        // the reference adds z_last first and z_0 last
        for (int k = nz - 1; k >= 0; k--) acc += (double)Z[(size_t)k * ld + i] * cf[k];
        x[i] = acc;
    }
}

// ---------------------------------------------------------------------------
// BiCGStab helpers
// ---------------------------------------------------------------------------
// out = { (a, b), (c, d) } two dots in one pass
__global__ void __launch_bounds__(256) k_dot2(long long n, const double* __restrict__ a, const double* __restrict__ b,
                                               const double* __restrict__ c, const double* __restrict__ d,
                                               double* partial, unsigned int* counter, double* out)
{
    double s[2] = {0.0, 0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        s[0] += a[i] * b[i];
        s[1] += c[i] * d[i];
    }
    grid_reduce<2>(s, partial, counter, out);
}

// BiCGStab device scalars: sc[0] = (rr, r), sc[1] = (rr, nu), sc[2] = (t, s),
// sc[3] = (t, t), sc[4] = (rr, r_new), sc[5] = ||r_new||^2.
//
// nu = A y ;  sc[0] = (rr, r) ; sc[1] = (rr, nu)
__global__ void __launch_bounds__(256) k_bicg_nu(int N, int M, int K, const int* __restrict__ cls, const double* __restrict__ dict,
                                                  const double* __restrict__ y, double* __restrict__ nu,
                                                  const double* __restrict__ rr, const double* __restrict__ r,
                                                  double* partial, unsigned int* counter, double* sc)
{
    const long long n = (long long)N * M * K;
    const int NM = N * M;
    double s[2] = {0.0, 0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int ix, iy, iz;
        cell_xyz(i, N, NM, ix, iy, iz);
        const double* a = dict + (size_t)cls[i] * 7;
        double acc = a[3] * y[i];
        if (iz > 0) acc += a[0] * y[i - NM];
        if (iy > 0) acc += a[1] * y[i - N];
        if (ix > 0) acc += a[2] * y[i - 1];
        if (ix < N - 1) acc += a[4] * y[i + 1];
        if (iy < M - 1) acc += a[5] * y[i + N];
        if (iz < K - 1) acc += a[6] * y[i + NM];
        nu[i] = acc;
        s[0] += rr[i] * r[i];
        s[1] += rr[i] * acc;
    }
    grid_reduce<2>(s, partial, counter, sc);
}

// alpha = sc0/sc1 ; nu *= alpha ; s = r - nu   (setDiffWithScale,
// mesh_function.h:116-121)
__global__ void k_bicg_s(long long n, const double* __restrict__ sc, double* __restrict__ nu,
                         const double* __restrict__ r, double* __restrict__ sv)
{
    const double alpha = sc[0] / sc[1];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double v = nu[i] * alpha;
        nu[i] = v;
        sv[i] = r[i] - v;
    }
}

// t = A z ; sc[2] = (t, s) ; sc[3] = (t, t)
__global__ void __launch_bounds__(256) k_bicg_t(int N, int M, int K, const int* __restrict__ cls, const double* __restrict__ dict,
                                                 const double* __restrict__ z, double* __restrict__ t,
                                                 const double* __restrict__ sv, double* partial,
                                                 unsigned int* counter, double* sc2)
{
    const long long n = (long long)N * M * K;
    const int NM = N * M;
    double s[2] = {0.0, 0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int ix, iy, iz;
        cell_xyz(i, N, NM, ix, iy, iz);
        const double* a = dict + (size_t)cls[i] * 7;
        double acc = a[3] * z[i];
        if (iz > 0) acc += a[0] * z[i - NM];
        if (iy > 0) acc += a[1] * z[i - N];
        if (ix > 0) acc += a[2] * z[i - 1];
        if (ix < N - 1) acc += a[4] * z[i + 1];
        if (iy < M - 1) acc += a[5] * z[i + N];
        if (iz < K - 1) acc += a[6] * z[i + NM];
        t[i] = acc;
        s[0] += acc * sv[i];
        s[1] += acc * acc;
    }
    grid_reduce<2>(s, partial, counter, sc2);
}

// solUpd (bicgstab_interface.h:39-48): y *= alpha; z *= w; x += y + z;
// t *= w; r = s - t ; sc[4] = (rr, r)
__global__ void __launch_bounds__(256) k_bicg_upd(long long n, const double* __restrict__ sc, double* __restrict__ y,
                                                   double* __restrict__ z, double* __restrict__ x,
                                                   double* __restrict__ t, double* __restrict__ r,
                                                   const double* __restrict__ sv, const double* __restrict__ rr,
                                                   double* partial, unsigned int* counter, double* sc4)
{
    const double alpha = sc[0] / sc[1];
    const double w = sc[2] / sc[3];
    double s[1] = {0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double yv = y[i] * alpha;
        const double zv = z[i] * w;
        x[i] += yv + zv;
        const double tv = t[i] * w;
        const double rv = sv[i] - tv;
        r[i] = rv;
        s[0] += rr[i] * rv;
    }
    grid_reduce<1>(s, partial, counter, sc4);
}

// pUpd (bicgstab_interface.h:49-56): coef = w/alpha; beta = (rr,r)/(vs coef);
// p = r + (p - nu coef) beta ; sc[5] = ||r||^2
__global__ void __launch_bounds__(256) k_bicg_p(long long n, const double* __restrict__ sc, double* __restrict__ p,
                                                 const double* __restrict__ nu, const double* __restrict__ r,
                                                 double* partial, unsigned int* counter, double* sc5)
{
    const double alpha = sc[0] / sc[1];
    const double w = sc[2] / sc[3];
    const double coef = w / alpha;
    const double vs = sc[0] * coef;
    const double beta = sc[4] / vs;
    double s[1] = {0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double cur = (p[i] - nu[i] * coef) * beta;
        const double rv = r[i];
        p[i] = rv + cur;
        s[0] += rv * rv;
    }
    grid_reduce<1>(s, partial, counter, sc5);
}

}  // namespace lsg

namespace lsg {

// ---------------------------------------------------------------------------
// Low-synchronisation MGS (inverse compact WY form).  For the basis
// V = [v_0 .. v_j] the MGS coefficients satisfy (I + L) h = V^T w with L the
// strictly lower part of V^T V; both right-hand sides come from one pass.
// ---------------------------------------------------------------------------
constexpr int kGsMaxVec = 64;

// Block-level sum of nv values per thread into partial[block * stride + q];
// the last block sums the partials in block order into out[q].
__device__ void grid_reduce_n(double* vals, int nv, double* partial, int stride, unsigned int* counter,
                              double* out)
{
    __shared__ double sh[32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int q = 0; q < nv; q++) {
        double t = warp_sum(vals[q]);
        if (lane == 0) sh[wid] = t;
        __syncthreads();
        if (threadIdx.x == 0) {
            double u = 0.0;
            for (int w = 0; w < nw; w++) u += sh[w];
            partial[(size_t)blockIdx.x * stride + q] = u;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        __threadfence();
        last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int q = wid; q < nv; q += nw) {
        double acc = 0.0;
        for (int b = lane; b < (int)gridDim.x; b += 32) acc += ((volatile double*)partial)[(size_t)b * stride + q];
        acc = warp_sum(acc);
        if (lane == 0) out[q] = acc;
    }
    __syncthreads();
    if (threadIdx.x == 0) *counter = 0u;
}

// One pass over V[0..j] and w:  s[k] = (v_k, w), k <= j;  g[k] = (v_k, v_j), k < j.
// out = s[0..j], g[0..j-1] (2j+1 values).
template <int NV>
__global__ void __launch_bounds__(256) k_gs_dots(long long n, long long ld, int j, const double* __restrict__ V,
                                                  const double* __restrict__ w, double* partial,
                                                  unsigned int* counter, double* out)
{
    double sacc[NV], gacc[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) {
        sacc[k] = 0.0;
        gacc[k] = 0.0;
    }
    const double* vj = V + (size_t)j * ld;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double wi = w[i], vji = vj[i];
#pragma unroll
        for (int k = 0; k < NV; k++) {
            if (k <= j) {
                const double vk = (k == j) ? vji : V[(size_t)k * ld + i];
                sacc[k] += vk * wi;
                if (k < j) gacc[k] += vk * vji;
            }
        }
    }
    double vals[2 * NV];
    int nv = 0;
#pragma unroll
    for (int k = 0; k < NV; k++)
        if (k <= j) vals[nv++] = sacc[k];
#pragma unroll
    for (int k = 0; k < NV; k++)
        if (k < j) vals[nv++] = gacc[k];
    grid_reduce_n(vals, nv, partial, 2 * kGsMaxVec, counter, out);
}

// Triangular correction on one thread: store row j of L (from g), solve
// (I + L) h = s, write h into Hessenberg column j.
__global__ void k_gs_tri(KrylovScalars* ks, int j, int ldh, const double* __restrict__ sg, double* __restrict__ Lrows)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double* s = sg;
    const double* g = sg + (j + 1);
    for (int k = 0; k < j; k++) Lrows[(size_t)j * kGsMaxVec + k] = g[k];
    double* H = ks->H + (size_t)j * ldh;
    for (int i = 0; i <= j; i++) {
        double h = s[i];
        for (int k = 0; k < i; k++) h -= Lrows[(size_t)i * kGsMaxVec + k] * H[k];
        H[i] = h;
    }
}

// w -= sum_k h_k v_k (k <= j) and ||w||^2.
template <int NV>
__global__ void __launch_bounds__(256) k_gs_update(long long n, long long ld, int j, const double* __restrict__ V,
                                                    const double* __restrict__ h, double* __restrict__ w,
                                                    double* partial, unsigned int* counter, double* out)
{
    __shared__ double hs[NV];
    if (threadIdx.x < NV) hs[threadIdx.x] = (threadIdx.x <= j) ? h[threadIdx.x] : 0.0;
    __syncthreads();
    double s[1] = {0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        double acc = w[i];
#pragma unroll
        for (int k = 0; k < NV; k++)
            if (k <= j) acc -= hs[k] * V[(size_t)k * ld + i];
        w[i] = acc;
        s[0] += acc * acc;
    }
    grid_reduce<1>(s, partial, counter, out);
}

}  // namespace lsg
