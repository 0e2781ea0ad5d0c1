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
    const CellIndex ci(N, NM);
    double s[1] = {0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int ix, iy, iz;
        ci.xyz(i, ix, iy, iz);
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
    const CellIndex ci(N, NM);
    double s[1] = {0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int ix, iy, iz;
        ci.xyz(i, ix, iy, iz);
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

// Krylov 7-point products on the fine grid, marching along z like k_apply7z
// (U z-steps of loads in flight per thread) and fused with one dot product:
//   MODE 0:  w = A z,      out = (w, v)      (Arnoldi: first MGS coefficient)
//   MODE 1:  w = v - A z,  out = (w, w)      (residual and its squared norm)
// z is FP64, or FP32 widened exactly.  Terms are summed p, b, s, w, e, n, t.
template <typename Tz, int MODE>
__global__ void __launch_bounds__(256, 3) k_krylov7z(int N, int M, int K, int zc, const int* __restrict__ cls,
                                                   const double* __restrict__ dict, const Tz* __restrict__ z,
                                                   const double* __restrict__ v, double* __restrict__ w,
                                                   double* partial, unsigned int* counter, double* out)
{
    constexpr int U = sizeof(Tz) == 4 ? 8 : 4;            // z-steps of DRAM loads in flight per thread
    double s[1] = {0.0};
    const int ix = blockIdx.x * 32 + threadIdx.x;
    const int iy = blockIdx.y * 8 + threadIdx.y;
    if (ix < N && iy < M) {
        const int NM = N * M;                              // grids hold fewer than 2^31 cells
        const int z0 = blockIdx.z * zc;
        const int z1 = min(z0 + zc, K);
        int i = ix + N * iy + NM * z0;
        Tz xm = (z0 > 0) ? z[i - NM] : (Tz)0;
        Tz xc = z[i];
        const bool hasw = ix > 0, hase = ix < N - 1, hass = iy > 0, hasn = iy < M - 1;
        for (int zb = z0; zb < z1; zb += U, i += U * NM) {
            // the streams from DRAM (class, v, next plane) for U steps first;
            // the four lateral neighbours were just read by the adjacent
            // threads and come from L1 inside the step
            int cl[U];
            double vv[U];
            Tz xp[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int zz = zb + u;
                const int ii = (zz < z1) ? i + u * NM : i;
                cl[u] = cls[ii];
                vv[u] = v[ii];
                xp[u] = (zz < K - 1) ? z[ii + NM] : (Tz)0;
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                if (zb + u < z1) {
                    const int ii = i + u * NM;
                    const double* a = dict + (size_t)cl[u] * 7;
                    double acc = a[3] * (double)xc;
                    acc += a[0] * (double)xm;
                    if (hass) acc += a[1] * (double)z[ii - N];
                    if (hasw) acc += a[2] * (double)z[ii - 1];
                    if (hase) acc += a[4] * (double)z[ii + 1];
                    if (hasn) acc += a[5] * (double)z[ii + N];
                    acc += a[6] * (double)xp[u];
                    if (MODE == 0) {
                        w[ii] = acc;
                        s[0] += acc * vv[u];
                    } else {
                        const double t = vv[u] - acc;
                        w[ii] = t;
                        s[0] += t * t;
                    }
                    xm = xc;
                    xc = xp[u];
                }
            }
        }
    }
    grid_reduce<1>(s, partial, counter, out);
}

// The same Krylov products with the z planes staged in shared memory (the
// kernel the solve launches; k_krylov7z stays for timing comparisons): a CTA
// marches a 32 x 8 (x, y) tile along z with the tile's planes z-1, z, z+1 and
// their one-cell halo (34 x 10 values) in a ring of three shared buffers, each
// plane read once per CTA by two coalesced loads per thread issued one plane
// ahead; the seven neighbours of a cell then come from shared memory instead
// of four lateral gathers per cell through L1.  Row class and v stream from
// DRAM one step ahead.  Values outside the grid are staged as 0.  Same
// summation order and neighbour guards as k_krylov7z.
template <typename Tz, int MODE>
__global__ void __launch_bounds__(256) k_krylov7s(int N, int M, int K, int zc, const int* __restrict__ cls,
                                                   const double* __restrict__ dict, const Tz* __restrict__ z,
                                                   const double* __restrict__ v, double* __restrict__ w,
                                                   double* partial, unsigned int* counter, double* out)
{
    constexpr int TW = 34, TH = 10, TP = TW * TH;
    __shared__ Tz sp[3][TP];
    double s[1] = {0.0};
    const int tid = threadIdx.y * 32 + threadIdx.x;
    const int ix = blockIdx.x * 32 + threadIdx.x;
    const int iy = blockIdx.y * 8 + threadIdx.y;
    const bool own = ix < N && iy < M;
    const int NM = N * M;                                  // grids hold fewer than 2^31 cells
    const int z0 = blockIdx.z * zc;
    const int z1 = min(z0 + zc, K);
    const int gx0 = blockIdx.x * 32 - 1, gy0 = blockIdx.y * 8 - 1;
    int goff[2];
    bool gin[2];
#pragma unroll
    for (int q = 0; q < 2; q++) {
        const int e = tid + 256 * q;
        const int ly = e / TW, lx = e - ly * TW;
        const int gx = gx0 + lx, gy = gy0 + ly;
        gin[q] = (e < TP) && gx >= 0 && gx < N && gy >= 0 && gy < M;
        goff[q] = gx + N * gy;
    }
    auto fetch = [&](int zz, Tz (&t)[2]) {
        const bool zin = zz >= 0 && zz < K;
#pragma unroll
        for (int q = 0; q < 2; q++) t[q] = (zin && gin[q]) ? z[goff[q] + NM * zz] : (Tz)0;
    };
    auto stage = [&](int slot, const Tz (&t)[2]) {
        sp[slot][tid] = t[0];
        if (tid + 256 < TP) sp[slot][tid + 256] = t[1];
    };
    Tz t[2];
    fetch(z0 - 1, t);
    stage(0, t);
    fetch(z0, t);
    stage(1, t);
    fetch(z0 + 1, t);
    const int col = ix + N * iy;
    int cn = own ? cls[col + NM * z0] : 0;
    double vn = own ? v[col + NM * z0] : 0.0;
    const bool hasw = ix > 0, hase = ix < N - 1, hass = iy > 0, hasn = iy < M - 1;
    int sm = 0, sc = 1, sn = 2;
    const int c0 = (threadIdx.y + 1) * TW + threadIdx.x + 1;
    for (int zz = z0; zz < z1; zz++) {
        stage(sn, t);
        __syncthreads();
        if (zz + 2 <= z1) fetch(zz + 2, t);
        const int cl = cn;
        const double vv = vn;
        if (own && zz + 1 < z1) {
            cn = cls[col + NM * (zz + 1)];
            vn = v[col + NM * (zz + 1)];
        }
        if (own) {
            const double* a = dict + (size_t)cl * 7;
            const Tz* pc = sp[sc];
            double acc = a[3] * (double)pc[c0];
            acc += a[0] * (double)sp[sm][c0];
            if (hass) acc += a[1] * (double)pc[c0 - TW];
            if (hasw) acc += a[2] * (double)pc[c0 - 1];
            if (hase) acc += a[4] * (double)pc[c0 + 1];
            if (hasn) acc += a[5] * (double)pc[c0 + TW];
            acc += a[6] * (double)sp[sn][c0];
            const int i = col + NM * zz;
            if (MODE == 0) {
                w[i] = acc;
                s[0] += acc * vv;
            } else {
                const double r = vv - acc;
                w[i] = r;
                s[0] += r * r;
            }
        }
        __syncthreads();
        const int tt = sm;
        sm = sc;
        sc = sn;
        sn = tt;
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
    const CellIndex ci(N, NM);
    double s[2] = {0.0, 0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int ix, iy, iz;
        ci.xyz(i, ix, iy, iz);
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
    const CellIndex ci(N, NM);
    double s[2] = {0.0, 0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int ix, iy, iz;
        ci.xyz(i, ix, iy, iz);
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

// One pass over V[0..j] and w for the low-synchronisation Gram-Schmidt:
// s_k = (v_k, w) for k <= j and g_k = (v_k, v_j) for k < j; out = s_0..s_j,
// g_0..g_{j-1}.  A block is 32 lanes (consecutive cells) by one warp per group
// of four basis vectors: each warp streams only its own vectors, while w and
// v_j are shared by the warps of the block through L1.  Per-block sums go to
// partial[block][q]; the last block to finish adds them in block order.
__global__ void __launch_bounds__(512) k_gs_dots2(long long n, long long ld, int j, const double* __restrict__ V,
                                                  const double* __restrict__ w, double* partial,
                                                  unsigned int* counter, double* out)
{
    constexpr int VW = 4;
    const int lane = threadIdx.x, grp = threadIdx.y;
    const int k0 = grp * VW;
    const int nk = max(0, min(VW, j + 1 - k0));
    double sa[VW], ga[VW];
#pragma unroll
    for (int q = 0; q < VW; q++) {
        sa[q] = 0.0;
        ga[q] = 0.0;
    }
    const double* vj = V + (size_t)j * ld;
    // each block streams one contiguous range of cells, 128 per warp step
    // (four 32-cell pieces, all loads of a step issued before the sums)
    const long long chunk = ((n + gridDim.x - 1) / gridDim.x + 127) / 128 * 128;
    const long long beg = (long long)blockIdx.x * chunk, end = min(n, beg + chunk);
    for (long long i0 = beg + lane; i0 < end; i0 += 128) {
        double wv[4], vv[4], av[VW][4];
#pragma unroll
        for (int p = 0; p < 4; p++) {
            const long long i = i0 + 32 * p;
            const bool in = i < end;
            wv[p] = in ? w[i] : 0.0;
            vv[p] = in ? vj[i] : 0.0;
#pragma unroll
            for (int q = 0; q < VW; q++) av[q][p] = (in && q < nk) ? V[(size_t)(k0 + q) * ld + i] : 0.0;
        }
#pragma unroll
        for (int p = 0; p < 4; p++)
#pragma unroll
            for (int q = 0; q < VW; q++) {
                sa[q] += av[q][p] * wv[p];
                ga[q] += av[q][p] * vv[p];
            }
    }
    const int pstride = 2 * kGsMaxVec;
#pragma unroll
    for (int q = 0; q < VW; q++) {
        sa[q] = warp_sum(sa[q]);
        ga[q] = warp_sum(ga[q]);
    }
    if (lane == 0) {
        for (int q = 0; q < nk; q++) {
            const int k = k0 + q;
            partial[(size_t)blockIdx.x * pstride + k] = sa[q];
            if (k < j) partial[(size_t)blockIdx.x * pstride + j + 1 + k] = ga[q];
        }
        __threadfence();
    }
    __shared__ bool last;
    __syncthreads();
    if (lane == 0 && grp == 0) last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    // final sums: one warp per value, four independent L2 loads in flight per lane
    const int nv = 2 * j + 1;
    for (int q = grp; q < nv; q += blockDim.y) {
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
        int b = lane;
        for (; b + 96 < (int)gridDim.x; b += 128) {
            a0 += __ldcg(partial + (size_t)b * pstride + q);
            a1 += __ldcg(partial + (size_t)(b + 32) * pstride + q);
            a2 += __ldcg(partial + (size_t)(b + 64) * pstride + q);
            a3 += __ldcg(partial + (size_t)(b + 96) * pstride + q);
        }
        for (; b < (int)gridDim.x; b += 32) a0 += __ldcg(partial + (size_t)b * pstride + q);
        const double acc = warp_sum((a0 + a1) + (a2 + a3));
        if (lane == 0) out[q] = acc;
    }
    __syncthreads();
    if (lane == 0 && grp == 0) *counter = 0u;
}

// w -= sum_{k<=j} h_k v_k and ||w||^2, the basis vectors read four at a time.
__global__ void __launch_bounds__(256) k_gs_update2(long long n, long long ld, int j, const double* __restrict__ V,
                                                    const double* __restrict__ h, double* __restrict__ w,
                                                    double* partial, unsigned int* counter, double* out)
{
    __shared__ double hs[kGsMaxVec];
    for (int t = threadIdx.x; t <= j; t += blockDim.x) hs[t] = h[t];
    __syncthreads();
    double s[1] = {0.0};
    const long long chunk = ((n + gridDim.x - 1) / gridDim.x + blockDim.x - 1) / blockDim.x * blockDim.x;
    const long long beg = (long long)blockIdx.x * chunk, end = min(n, beg + chunk);
    for (long long i = beg + threadIdx.x; i < end; i += blockDim.x) {
        double acc = w[i];
        int k = 0;
        for (; k + 4 <= j + 1; k += 4) {
            const double v0 = V[(size_t)k * ld + i], v1 = V[(size_t)(k + 1) * ld + i];
            const double v2 = V[(size_t)(k + 2) * ld + i], v3 = V[(size_t)(k + 3) * ld + i];
            acc -= hs[k] * v0;
            acc -= hs[k + 1] * v1;
            acc -= hs[k + 2] * v2;
            acc -= hs[k + 3] * v3;
        }
        for (; k <= j; k++) acc -= hs[k] * V[(size_t)k * ld + i];
        w[i] = acc;
        s[0] += acc * acc;
    }
    grid_reduce<1>(s, partial, counter, out);
}

}  // namespace lsg
