// ADLJ direction steps with the residual formed inside the line solve.
//
// SmootherADLJInterface::solve (smoother_adlj_interface.h:66-77) runs, per
// direction d of the sweep order z, y, x:
//     r -= A c ;   c = omega T_d^{-1} r ;   ch += c
// starting from c = ch = P c_H (the prolonged coarse correction) and r = b
// (the level's right-hand side).  By induction r = b - A ch before every
// direction, so the step is the line-Jacobi update
//     ch' = ch + omega T_d^{-1} (b - A ch)
// computed here by one kernel per direction: each thread forms the residual
// of its cells from b, the row class and the current iterate (its line
// neighbours from registers, the lateral ones through L1/L2), then runs the
// segmented Thomas recurrence of k_tdma_seg / k_tdma_xseg on it.  The line
// tridiagonal is read from the operator's own rows (lo, up = the row's
// couplings along d) and the stored inverse pivots dinv_d (the factorisation
// of TriDiagonalMatrix::triLU, tridiagonal_matrix.h:45-67), with the LU's
// scaled upper diagonal formed as up * dinv.  The iterate is read from one
// buffer and written to another (every line reads its lateral neighbours'
// old values, as the Jacobi step requires).
//
// Per cell and direction this streams b, the iterate, the row class and
// dinv_d and writes the new iterate: 4w + 4 bytes (w the element size)
// against 10w + 4 for the separate residual update and line solve (r, c read
// and r written; r, lo, dinv, up, ch read and c, ch written).
//
// The operator is the fine 7-point stencil in the row-dictionary form: dict
// holds each distinct row as (b, s, w, p, e, n, t), cls[i] its index.
#pragma once

#include "lsg_kernels.cuh"

namespace lsg {

// b - A x at flat cell q with row class c, every neighbour read from memory
// (the z-line quirk's right-hand side cell).  Terms summed p, b, s, w, e, n, t.
template <typename T, int RS>
__device__ __forceinline__ T resid7_at_class(int N, int M, int K, long long q, int c, const T* __restrict__ dict,
                                             const T* __restrict__ b, const T* __restrict__ x)
{
    const int NM = N * M;
    const int qz = (int)(q / NM);
    const int rem = (int)(q - (long long)qz * NM);
    const int qy = rem / N, qx = rem - qy * N;
    const T* a = dict + (size_t)c * RS;
    T acc = a[3] * x[q];
    if (qz > 0) acc += a[0] * x[q - NM];
    if (qy > 0) acc += a[1] * x[q - N];
    if (qx > 0) acc += a[2] * x[q - 1];
    if (qx < N - 1) acc += a[4] * x[q + 1];
    if (qy < M - 1) acc += a[5] * x[q + N];
    if (qz < K - 1) acc += a[6] * x[q + NM];
    return b[q] - acc;
}

template <typename T, int RS>
__device__ __forceinline__ T resid7_at(int N, int M, int K, long long q, const int* __restrict__ cls,
                                       const T* __restrict__ dict, const T* __restrict__ b,
                                       const T* __restrict__ x)
{
    return resid7_at_class<T, RS>(N, M, K, q, cls[q], dict, b, x);
}

// y-lines (DIR 1) and z-lines (DIR 2), segmented like k_tdma_seg: a CTA holds
// W neighbouring lines (consecutive x) split into S = ceil(L/SEG) segments,
// one thread per (line, segment).  Phase 1 loads the segment's row classes,
// right-hand sides, pivots and iterate values (plus the iterate just before
// and after the segment); phase 2 forms the residuals with the four lateral
// neighbours (coalesced loads, mostly L1/L2 hits); then the affine segment
// maps of the forward and backward recurrences are composed across the
// segments: by log-step scans in shared memory when VAR & 1 (the solve's
// form), else by each thread walking the maps before its own (timing
// comparison).  VAR & 2: the line splits into whole segments (L = S SEG),
// so no cell lies past its end and the line-end guards go.  zquirk (DIR 2):
// the first right-hand side of the z-line
// (x, y) is the residual at cell y*N*K + x, where the reference reads it
// (smoother_adlj_z.h:54-58).  Shared memory: 4 W S values.
template <typename T, int DIR, int SEG, int MAXT, int MINB, int VAR>
__global__ void __launch_bounds__(MAXT, MINB)
    k_adlj_fused_seg(int N, int M, int K, bool zquirk, const int* __restrict__ cls, const T* __restrict__ dict,
                     const T* __restrict__ dinv, const T* __restrict__ b, const T* __restrict__ xin,
                     T* __restrict__ xout, T omega)
{
    static_assert(DIR == 1 || DIR == 2, "y- or z-lines");
    constexpr bool LOGSCAN = (VAR & 1) != 0;
    constexpr bool EXACT = (VAR & 2) != 0;                 // L = S * SEG: no cell past the line end
    extern __shared__ __align__(16) unsigned char fseg_smem[];
    const int W = blockDim.x, S = blockDim.y;
    T* sA = reinterpret_cast<T*>(fseg_smem);               // 2 buffers of W*S each
    T* sB = sA + 2 * W * S;
    const int w = threadIdx.x, sg = threadIdx.y;
    const int NM = N * M;                                  // grids hold fewer than 2^31 cells
    const int L = DIR == 1 ? M : K;
    const int st = DIR == 1 ? N : NM;                      // stride along the line
    const int rows = DIR == 1 ? K : M;                     // the other cross direction
    const int sb = DIR == 1 ? NM : N;                      // its stride
    const int gx = (N + W - 1) / W;
    const int row = blockIdx.x / gx;                       // z of a y-line, y of a z-line
    const int x = (blockIdx.x - row * gx) * W + w;
    const bool valid = x < N;
    const int xs = valid ? x : N - 1;                      // idle lanes load a valid line, store nothing
    const int i0 = DIR == 1 ? row * NM + xs : row * N + xs;
    const int t0 = sg * SEG;
    const bool hw = xs > 0, he = xs < N - 1, hm = row > 0, hp = row < rows - 1;
    // the z-line quirk's cell y*N*K + x: its row class is read now, so the
    // residual there (after phase 2) starts from a class already in hand
    int qcl = 0;
    if (DIR == 2 && zquirk && sg == 0) qcl = cls[(long long)row * N * K + xs];
    // phase 1: the segment's own streams
    int cl[SEG];
    T rv[SEG], dv[SEG], xc[SEG];
#pragma unroll
    for (int u = 0; u < SEG; u++) {
        const int t = EXACT ? t0 + u : min(t0 + u, L - 1);
        const int i = i0 + t * st;
        cl[u] = cls[i];
        rv[u] = b[i];
        dv[u] = dinv[i];
        xc[u] = xin[i];
    }
    const T xprev = t0 > 0 ? xin[i0 + (t0 - 1) * st] : (T)0;
    const T xnext = t0 + SEG < L ? xin[i0 + (t0 + SEG) * st] : (T)0;
    // phase 2: residuals; lv <- lower coupling, uv <- scaled upper coupling
    T lv[SEG], uv[SEG];
#pragma unroll
    for (int u = 0; u < SEG; u++) {
        const int t = t0 + u;
        lv[u] = 0;
        uv[u] = 0;
        if (EXACT || t < L) {
            const int i = i0 + t * st;
            const T* a = dict + (size_t)cl[u] * 7;
            const T xw = hw ? xin[i - 1] : (T)0;
            const T xe = he ? xin[i + 1] : (T)0;
            const T xm = hm ? xin[i - sb] : (T)0;
            const T xq = hp ? xin[i + sb] : (T)0;
            const T xa = u == 0 ? xprev : xc[u > 0 ? u - 1 : 0];           // previous along the line
            const T xb = u == SEG - 1 ? xnext : xc[u < SEG - 1 ? u + 1 : 0];   // next along the line
            const bool ha = t > 0, hb = t < L - 1;
            T acc = a[3] * xc[u];
            if (DIR == 1) {
                if (hm) acc += a[0] * xm;                  // z - 1
                if (ha) acc += a[1] * xa;                  // y - 1
                if (hw) acc += a[2] * xw;
                if (he) acc += a[4] * xe;
                if (hb) acc += a[5] * xb;                  // y + 1
                if (hp) acc += a[6] * xq;                  // z + 1
                lv[u] = a[1];
                uv[u] = a[5] * dv[u];
            } else {
                if (ha) acc += a[0] * xa;                  // z - 1
                if (hm) acc += a[1] * xm;                  // y - 1
                if (hw) acc += a[2] * xw;
                if (he) acc += a[4] * xe;
                if (hp) acc += a[5] * xq;                  // y + 1
                if (hb) acc += a[6] * xb;                  // z + 1
                lv[u] = a[0];
                uv[u] = a[6] * dv[u];
            }
            rv[u] = rv[u] - acc;
        }
    }
    if (DIR == 2 && zquirk && sg == 0)
        rv[0] = resid7_at_class<T, 7>(N, M, K, (long long)row * N * K + xs, qcl, dict, b, xin);
    // forward, relative to y_in
    T fa = 0, fb = 1;
#pragma unroll
    for (int u = 0; u < SEG; u++) {
        const int t = t0 + u;
        if (EXACT || t < L) {
            if (t == 0) {
                fa = rv[u] * dv[u];
                fb = 0;
            } else {
                fa = (rv[u] - lv[u] * fa) * dv[u];
                fb = -(lv[u] * fb) * dv[u];
            }
        }
        rv[u] = fa;
        lv[u] = fb;
    }
    T yin = 0;
    if constexpr (LOGSCAN) {
        seg_scan<T, false>(fa, fb, sA, sB);
        yin = fa;                                          // y entering this segment (line start: 0)
    } else {
        sA[sg * W + w] = fa;
        sB[sg * W + w] = fb;
        __syncthreads();
        for (int q = 0; q < sg; q++) yin = sA[q * W + w] + sB[q * W + w] * yin;
    }
    __syncthreads();                                       // the shared buffers are reused below
    // backward, relative to x_out
    T gg = 0, hh = 1;
#pragma unroll
    for (int u = SEG - 1; u >= 0; u--) {
        const int t = t0 + u;
        if (EXACT || t < L) {
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
    if constexpr (LOGSCAN) {
        seg_scan<T, true>(gg, hh, sA, sB);
        xo = gg;                                           // x leaving the next segment (line end: 0)
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
            if (EXACT || t < L) {
                const T cv = omega * (rv[u] + lv[u] * xo);
                xout[i0 + t * st] = xc[u] + cv;
            }
        }
    }
}

// x-lines of length N = P * SEG (P a power of two <= 32), as k_tdma_xseg:
// every thread owns SEG consecutive cells of a line, read with 16-byte vector
// loads (b, iterate, pivots, row classes, and the four lateral rows y +- 1,
// z +- 1 of the iterate), the x neighbours across segment ends come from the
// adjacent lanes by shuffles, and the segment maps are chained across the P
// lanes of a line by warp scans.
template <typename T, int SEG>
__global__ void __launch_bounds__(256) k_adlj_fused_xseg(int N, int M, int K, int P, const int* __restrict__ cls,
                                                          const T* __restrict__ dict, const T* __restrict__ dinv,
                                                          const T* __restrict__ b, const T* __restrict__ xin,
                                                          T* __restrict__ xout, T omega)
{
    static_assert(SEG % 4 == 0, "row classes are read as int4");
    const long long nlines = (long long)M * K;
    // whole warps stay in the kernel so every shuffle has its full group
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long line = tid / P;
    const int q = (int)(tid - line * P);
    const bool valid = line < nlines;
    const int ln = valid ? (int)line : 0;                  // line = y + M z
    const int z = ln / M, y = ln - z * M;
    const int NM = N * M;
    const int base = ln * N + q * SEG;
    T bv[SEG], xc[SEG], dv[SEG], zm[SEG], ym[SEG], yp[SEG], zp[SEG];
    int cl[SEG];
#pragma unroll
    for (int k = 0; k < SEG / 4; k++) {
        const int4 c4 = *reinterpret_cast<const int4*>(cls + base + 4 * k);
        cl[4 * k] = c4.x;
        cl[4 * k + 1] = c4.y;
        cl[4 * k + 2] = c4.z;
        cl[4 * k + 3] = c4.w;
    }
    load_seg<T, SEG>(b + base, bv);
    load_seg<T, SEG>(xin + base, xc);
    load_seg<T, SEG>(dinv + base, dv);
    const bool hzm = z > 0, hym = y > 0, hyp = y < M - 1, hzp = z < K - 1;
    // lateral rows (a row outside the grid is read from this one and not used)
    load_seg<T, SEG>(xin + (hzm ? base - NM : base), zm);
    load_seg<T, SEG>(xin + (hym ? base - N : base), ym);
    load_seg<T, SEG>(xin + (hyp ? base + N : base), yp);
    load_seg<T, SEG>(xin + (hzp ? base + NM : base), zp);
    const T xl = __shfl_up_sync(0xffffffffu, xc[SEG - 1], 1, P);     // last cell of lane q-1
    const T xr = __shfl_down_sync(0xffffffffu, xc[0], 1, P);         // first cell of lane q+1
    T lv[SEG], uv[SEG];
#pragma unroll
    for (int u = 0; u < SEG; u++) {
        const int xx = q * SEG + u;
        const T* a = dict + (size_t)cl[u] * 7;
        T acc = a[3] * xc[u];
        if (hzm) acc += a[0] * zm[u];
        if (hym) acc += a[1] * ym[u];
        if (xx > 0) acc += a[2] * (u == 0 ? xl : xc[u > 0 ? u - 1 : 0]);
        if (xx < N - 1) acc += a[4] * (u == SEG - 1 ? xr : xc[u < SEG - 1 ? u + 1 : 0]);
        if (hyp) acc += a[5] * yp[u];
        if (hzp) acc += a[6] * zp[u];
        bv[u] = bv[u] - acc;
        lv[u] = a[2];
        uv[u] = a[4] * dv[u];
    }
    // forward: y_t = (r_t - lo_t y_{t-1}) dinv_t relative to the segment input
    T fa = 0, fb = 1;
#pragma unroll
    for (int u = 0; u < SEG; u++) {
        if (q == 0 && u == 0) {
            fa = bv[0] * dv[0];
            fb = 0;
        } else {
            fa = (bv[u] - lv[u] * fa) * dv[u];
            fb = -(lv[u] * fb) * dv[u];
        }
        bv[u] = fa;
        lv[u] = fb;
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        if (o >= P) break;
        const T a2 = __shfl_up_sync(0xffffffffu, fa, o, P);
        const T b2 = __shfl_up_sync(0xffffffffu, fb, o, P);
        if (q >= o) {
            fa = fa + fb * a2;
            fb = fb * b2;
        }
    }
    T yin = __shfl_up_sync(0xffffffffu, fa, 1, P);
    if (q == 0) yin = 0;
    // backward: x_t = y_t - up_t x_{t+1} relative to the segment output
    T g = 0, hh = 1;
#pragma unroll
    for (int u = SEG - 1; u >= 0; u--) {
        const T yv = bv[u] + lv[u] * yin;
        if (q == P - 1 && u == SEG - 1) {
            g = yv;
            hh = 0;
        } else {
            g = yv - uv[u] * g;
            hh = -(uv[u] * hh);
        }
        bv[u] = g;
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
    T xo = __shfl_down_sync(0xffffffffu, g, 1, P);
    if (q == P - 1) xo = 0;
    if (!valid) return;
#pragma unroll
    for (int u = 0; u < SEG; u++) xc[u] = xc[u] + omega * (bv[u] + lv[u] * xo);
    store_seg<T, SEG>(xout + base, xc);
}

}  // namespace lsg
