// Pressure projection of the time step on the GPU: the divergence right-hand
// side of the pressure equation and the velocity/pressure update, computed
// from the cut-cell geometry without assembling the reference's CSR operators.
//
// The reference evaluates these products on the CPU as separate IEEE multiply
// and add operations, so the kernels use __dmul_rn / __dadd_rn (no fused
// multiply-add) in the reference's order and reproduce its results bit for
// bit.
#pragma once

#include "lsg_kernels.cuh"

namespace lsg {

// CellTypes families (Base/LS_STAG_Mesh/cut_cells.h:142-167) by which border
// of the domain a cell lies on.
__device__ __forceinline__ bool fam_e(int t) { return t == -6 || t == -16 || t == -18 || t == -10 || t == -14 || t == -20 || t == -22 || t == -24 || t == -26; }
__device__ __forceinline__ bool fam_w(int t) { return t == -7 || t == -17 || t == -19 || t == -11 || t == -15 || t == -21 || t == -23 || t == -25 || t == -27; }
__device__ __forceinline__ bool fam_n(int t) { return t == -4 || t == -16 || t == -17 || t == -8 || t == -12 || t == -20 || t == -21 || t == -24 || t == -25; }
__device__ __forceinline__ bool fam_s(int t) { return t == -5 || t == -18 || t == -19 || t == -9 || t == -13 || t == -22 || t == -23 || t == -26 || t == -27; }
__device__ __forceinline__ bool fam_t(int t) { return t == -2 || t == -8 || t == -9 || t == -10 || t == -11 || t == -20 || t == -21 || t == -22 || t == -23; }
__device__ __forceinline__ bool fam_b(int t) { return t == -3 || t == -12 || t == -13 || t == -14 || t == -15 || t == -24 || t == -25 || t == -26 || t == -27; }

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// b = Dx u + flux + Dy v + Dz w (PoissonDiscreteEquation::recalcRightMember,
// DiscreteEquations/poisson_discrete_equation.h:145-159):
//   aux = Dx u;  b = (aux + flux) + Dy v;  b += Dz w;  b[pin0] = b[pin1] = 0,
// each product summed from its initial value in the row's column order
// (RealValuedMeshFunction::mvProd, real_valued_mesh_function.h:81-106).  The
// rows are DivergenceDiscreteOperatorX/Y/Z::calcD*
// (DiscreteOperators/Divergence/divergence_discrete_operator_x.h:119-159,
// _y.h:92-121, _z.h:86-111): -theta dS on the lower face, +theta dS on the
// upper face, one face on a domain-border cell, one zero entry on a solid
// cell.  The cell types must be consistent with the grid (border families on
// the border layers); lsg_set_matrix_geometry checks that before any launch.
__global__ void __launch_bounds__(256) k_projection_rhs(int N, int M, int K, const int* __restrict__ type,
                                                        const double* __restrict__ theta,
                                                        const double* __restrict__ delta,
                                                        const double* __restrict__ flux, const double* __restrict__ u,
                                                        const double* __restrict__ v, const double* __restrict__ w,
                                                        long long pin0, long long pin1, double* __restrict__ b)
{
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= N || y >= M) return;
    const long long NM = (long long)N * M;
    const long long i = x + (long long)N * y + NM * z;
    const int t = type[i];
    const double dx = delta[3 * i], dy = delta[3 * i + 1], dz = delta[3 * i + 2];
    const long long numX = i - y - (long long)z * M;          // x-face east of the cell
    const long long numY = i - (long long)z * N;              // y-face north of the cell
    // Dx u (divergence_discrete_operator_x.h:119-159)
    double aux;
    if (t == 0) {
        aux = add(0.0, mul(0.0, u[x == 0 ? numX : numX - 1]));
    } else if (fam_e(t)) {
        aux = add(0.0, mul(mul(mul(-theta[3 * (i - 1)], dy), dz), u[numX - 1]));
    } else if (fam_w(t)) {
        aux = add(0.0, mul(mul(mul(theta[3 * i], dy), dz), u[numX]));
    } else {
        const double dyz = mul(dy, dz);
        aux = add(add(0.0, mul(mul(-theta[3 * (i - 1)], dyz), u[numX - 1])), mul(mul(theta[3 * i], dyz), u[numX]));
    }
    // (aux + flux) + Dy v (divergence_discrete_operator_y.h:92-121)
    double r = add(aux, flux[i]);
    if (t == 0) {
        r = add(r, mul(0.0, v[y == 0 ? numY : numY - N]));
    } else if (fam_n(t)) {
        r = add(r, mul(mul(mul(-theta[3 * (i - N) + 1], dx), dz), v[numY - N]));
    } else if (fam_s(t)) {
        r = add(r, mul(mul(mul(theta[3 * i + 1], dx), dz), v[numY]));
    } else {
        const double dxz = mul(dx, dz);
        r = add(add(r, mul(mul(-theta[3 * (i - N) + 1], dxz), v[numY - N])), mul(mul(theta[3 * i + 1], dxz), v[numY]));
    }
    // + Dz w (divergence_discrete_operator_z.h:86-111)
    double q;
    if (t == 0) {
        q = add(0.0, mul(0.0, w[z == 0 ? i : i - NM]));
    } else if (fam_b(t)) {
        q = add(0.0, mul(mul(mul(theta[3 * i + 2], dx), dy), w[i]));
    } else if (fam_t(t)) {
        q = add(0.0, mul(mul(mul(-theta[3 * (i - NM) + 2], dx), dy), w[i - NM]));
    } else {
        const double dxy = mul(dx, dy);
        q = add(add(0.0, mul(mul(-theta[3 * (i - NM) + 2], dxy), w[i - NM])), mul(mul(theta[3 * i + 2], dxy), w[i]));
    }
    r = add(r, q);
    if (i == pin0 || i == pin1) r = 0.0;
    b[i] = r;
}

// Velocity update on one staggered grid (SetSolutions::correction,
// Base/set_solutions.h:215-237, with GradientDiscreteOperatorX/Y/Z::calc,
// DiscreteOperators/Gradient/gradient_discrete_operator_x.h:58-77, _y.h:52-74,
// _z.h:45-62):  out = (G phi) * inv_vof + pred, where the staggered cell f
// between base cells P and E = P + step carries (+c at P, -c at E),
// c = (theta_P[comp] * d1_P) * d2_P, and a solid staggered cell one zero
// entry at P.  dir 0: x-grid (N-1)MK, 1: y-grid N(M-1)K, 2: z-grid NM(K-1).
__global__ void __launch_bounds__(256) k_projection_velocity(int dir, int N, int M, int K, const int* __restrict__ stype,
                                                             const double* __restrict__ theta,
                                                             const double* __restrict__ delta,
                                                             const double* __restrict__ inv_vof,
                                                             const double* __restrict__ phi,
                                                             const double* __restrict__ pred,
                                                             double* __restrict__ out)
{
    const int Ns = N - (dir == 0), Ms = M - (dir == 1);     // blockIdx.z runs over the K - (dir == 2) layers
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= Ns || y >= Ms) return;
    const long long f = x + (long long)Ns * (y + (long long)Ms * z);
    const long long p = x + (long long)N * (y + (long long)M * z);      // base cell below the face
    const long long step = dir == 0 ? 1 : (dir == 1 ? N : (long long)N * M);
    double g;
    if (stype[f] == 0) {
        g = add(0.0, mul(0.0, phi[p]));
    } else {
        // d1, d2: the two cell sizes across the face (y, z for x; x, z for y; x, y for z)
        const double d1 = delta[3 * p + (dir == 0 ? 1 : 0)];
        const double d2 = delta[3 * p + (dir == 2 ? 1 : 2)];
        const double c = mul(mul(theta[3 * p + dir], d1), d2);
        g = add(add(0.0, mul(c, phi[p])), mul(-c, phi[p + step]));
    }
    out[f] = add(mul(g, inv_vof[f]), pred[f]);
}

// Outflow clamp at the east boundary (SetSolutions::corrOutFlow,
// Base/set_solutions.h:87-106) over y in [1, M-1), z in [1, K-1): where the
// last two x-faces of a row carry backflow (u < 0) they are reset to vbase and
// the matching v and w faces to zero.
__global__ void k_outflow_east(int N, int M, int K, double vbase, double* __restrict__ u, double* __restrict__ v,
                               double* __restrict__ w)
{
    const int y = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int z = 1 + blockIdx.y;
    if (y >= M - 1 || z >= K - 1) return;
    const long long NM = (long long)N * M;
    const long long num = (long long)(y + 1) * N - 1 + z * NM;
    long long num2 = num - y - 1 - (long long)z * M;
    const long long num3 = num - (long long)z * N;
    if (u[num2] < 0.0) {
        u[num2] = vbase;
        v[num3] = 0.0;
        w[num] = 0.0;
    }
    num2--;
    if (u[num2] < 0.0) {
        u[num2] = vbase;
        v[num3 - 1] = 0.0;
        w[num - 1] = 0.0;
    }
}

// Anti-backflow clamp on the bottom and top z-face layers
// (SetSolutions::corrOutFlowTB, Base/set_solutions.h:111-118) over
// x in [1, N), y in [1, M).
__global__ void k_outflow_tb(int N, int M, int K, double* __restrict__ w)
{
    const int x = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int y = 1 + blockIdx.y;
    if (x >= N || y >= M) return;
    const long long num = x + (long long)y * N;
    const long long top = num + (long long)(K - 2) * N * M;
    if (w[num] > 0.0) w[num] = 0.0;
    if (w[top] < 0.0) w[top] = 0.0;
}

// p += phi * coef (prediction.p *= coef; current.p += prediction.p).
__global__ void k_pressure_update(long long n, double coef, const double* __restrict__ phi, double* __restrict__ p)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        p[i] = add(p[i], mul(phi[i], coef));
}

// Source term of the pressure equation, LaplaceDiscreteOperator::flux after
// initMeshParams + calcFlux for a flow task with fixed bodies
// (DiscreteOperators/WithFlux/Sym/laplace_discrete_operator.h:47-83,
// :687-808).  One thread per cell applies, in the reference's order:
//   ibFlux (x in [1, N-2], y in [1, M-2]): 0 on fluid and solid cells; on cut
//     cells -V_ib . (theta jump) dS over the cut faces (B/T border cells only
//     when a face is cut, their z term left out; TW/TE/BW/BE edges untouched);
//   initFlux: -U_W(y, z) dS at x = 0, U_E dS at x = N-1 (dS of the row's first
//     cell);  addFluxNSp: -V_S dx dz at y = 0, +V_N dx dz at y = M-1 (dx of the
//     y = 0 cell, dz of the layer's first cell);  addFluxTBp: -W_B theta_z dx dy
//     at z = 0, +W_T theta_z dx dy at z = K-1 (dx of the z = 0 cell, dy of the
//     row's first cell);
//   setBaseFlux: x = N-1 overwritten by u(last x-face) dy dz (outflow).
// (A cut-cell type on the bottom layer has no face below; its index is
// clamped to the cell itself so that inconsistent input cannot read outside
// the arrays.)
__global__ void __launch_bounds__(256) k_laplace_flux(int N, int M, int K, const int* __restrict__ type,
                                                      const int* __restrict__ side, const double* __restrict__ theta,
                                                      const double* __restrict__ delta,
                                                      const double* __restrict__ vib, const double* __restrict__ u_w,
                                                      double U_E, double V_S, double V_N, double W_B, double W_T,
                                                      const double* __restrict__ ux, double* __restrict__ flux)
{
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= N || y >= M) return;
    const long long NM = (long long)N * M;
    const long long i = x + (long long)N * y + NM * z;
    double f = 0.0;
    if (y >= 1 && y <= M - 2 && x >= 1 && x <= N - 2) {
        const int t = type[i];
        const double dx = delta[3 * i], dy = delta[3 * i + 1], dz = delta[3 * i + 2];
        const double vx = vib[3 * i], vy = vib[3 * i + 1], vz = vib[3 * i + 2];
        if (t == 0 || t == 11111111) {
            f = 0.0;
        } else if (t == -3 || t == -2) {                       // B_Border, T_Border
            bool cut = false;
#pragma unroll
            for (int c = 0; c < 3; c++) cut |= side[3 * i + c] > 0 && side[3 * i + c] < 1111;
            f = cut ? mul(add(mul(mul(vx, sub(theta[3 * (i - 1)], theta[3 * i])), dy),
                              mul(mul(vy, sub(theta[3 * (i - N) + 1], theta[3 * i + 1])), dx)),
                          dz)
                    : 0.0;
        } else if (t == -11 || t == -10 || t == -15 || t == -14) {   // TW, TE, BW, BE edges: untouched
        } else {
            f = add(mul(add(mul(mul(vx, sub(theta[3 * (i - 1)], theta[3 * i])), dy),
                            mul(mul(vy, sub(theta[3 * (i - N) + 1], theta[3 * i + 1])), dx)),
                        dz),
                    mul(mul(mul(vz, sub(theta[3 * (z > 0 ? i - NM : i) + 2], theta[3 * i + 2])), dx), dy));
        }
    }
    const long long row0 = (long long)N * y + NM * z;          // first cell of the x-row
    if (x == 0 || x == N - 1) {
        const double dyz = mul(delta[3 * row0 + 1], delta[3 * row0 + 2]);
        f = (x == 0) ? mul(-u_w[y + (long long)z * M], dyz) : mul(U_E, dyz);
    }
    if (y == 0 || y == M - 1) {
        const double dz0 = delta[3 * (NM * z) + 2];
        const double coef = mul(delta[3 * (x + NM * z)], dz0);
        if (y == 0) f = sub(f, mul(coef, V_S));
        if (y == M - 1) f = add(f, mul(coef, V_N));
    }
    if (z == 0 || z == K - 1) {
        const long long b0 = (long long)N * y;                  // (x, y, 0) and its row start
        const double coef = mul(delta[3 * b0 + 1], delta[3 * (b0 + x)]);
        if (z == 0) f = sub(f, mul(mul(coef, theta[3 * i + 2]), W_B));
        if (z == K - 1) f = add(f, mul(mul(coef, theta[3 * i + 2]), W_T));
    }
    if (x == N - 1) f = mul(mul(ux[i - 1 - y - (long long)z * M], delta[3 * i + 1]), delta[3 * i + 2]);
    flux[i] = f;
}

// Pressure gradient on one staggered grid, out = G p (the rows of
// k_projection_velocity without the update): GradientDiscreteOperatorX/Y/Z
// applied by RealValuedMeshFunction::mvProd.
__global__ void __launch_bounds__(256) k_gradient_apply(int dir, int N, int M, int K, const int* __restrict__ stype,
                                                        const double* __restrict__ theta,
                                                        const double* __restrict__ delta,
                                                        const double* __restrict__ p, double* __restrict__ out)
{
    const int Ns = N - (dir == 0), Ms = M - (dir == 1);     // blockIdx.z runs over the K - (dir == 2) layers
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= Ns || y >= Ms) return;
    const long long f = x + (long long)Ns * (y + (long long)Ms * z);
    const long long P = x + (long long)N * (y + (long long)M * z);
    const long long step = dir == 0 ? 1 : (dir == 1 ? N : (long long)N * M);
    if (stype[f] == 0) {
        out[f] = add(0.0, mul(0.0, p[P]));
    } else {
        const double d1 = delta[3 * P + (dir == 0 ? 1 : 0)];
        const double d2 = delta[3 * P + (dir == 2 ? 1 : 2)];
        const double c = mul(mul(theta[3 * P + dir], d1), d2);
        out[f] = add(add(0.0, mul(c, p[P])), mul(-c, p[P + step]));
    }
}

// Right-hand side of one momentum equation for a fixed-body flow,
// HelmholtzDiscreteEquation::recalcRightMember (DiscreteEquations/
// helmholtz_discrete_equation.h:91-95, :213-254), one thread per staggered
// cell: aux = flux2 + C u summed in the CSR row order of the convective
// operator (ConvectiveDiscreteOperator*, rebuilt by the caller each step),
// right = ((-2 u + 0.5 u_prev) VOF) coef2 - ((G p + flux) + prev_aux) + 2 aux;
// aux is returned as the next step's prev_aux (Adams-Bashforth history).
// Without a CSR (rowptr == NULL) flux2 already holds flux2 + C u.
__global__ void __launch_bounds__(256) k_momentum_rhs(long long n, const int* __restrict__ rowptr,
                                                      const int* __restrict__ col, const double* __restrict__ val,
                                                      const double* __restrict__ flux2, const double* __restrict__ u,
                                                      const double* __restrict__ uprev,
                                                      const double* __restrict__ vof,
                                                      const double* __restrict__ hflux,
                                                      const double* __restrict__ prev_aux,
                                                      const double* __restrict__ gp, double coef2,
                                                      double* __restrict__ right, double* __restrict__ aux_out)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        double aux = flux2[i];
        if (rowptr)
            for (int e = rowptr[i]; e < rowptr[i + 1]; e++) aux = add(aux, mul(val[e], u[col[e]]));
        double r = mul(mul(add(mul(-2.0, u[i]), mul(0.5, uprev[i])), vof[i]), coef2);
        r = sub(r, add(add(gp[i], hflux[i]), prev_aux[i]));
        r = add(r, mul(aux, 2.0));
        right[i] = r;
        aux_out[i] = aux;
    }
}

// Convective operator of momentum component d applied from the geometry,
// out = init + C(U) v on the d-grid (ConvectiveDiscreteOperatorX/Y/Z::calcConv*,
// DiscreteOperators/WithFlux/SkewSym/convective_discrete_operator_x.h:49-366,
// _y.h, _z.h, in the form of their generic cut-cell rows).  For the staggered
// cell f between base cells P and Q = P + step_d, faces B, S, W, E, N, T:
//   along d:  -/+ 0.25 A (theta_d(P) U_d[f] + theta_d(P - step_d | Q) U_d[f -/+ stride_d]),
//             A = the product of P's two cell sizes across d;
//   across d (direction e):  -/+ 0.25 h (delta_d(P) theta_e(.) U_e[face of P] + delta_d(Q) theta_e(.) U_e[face of Q]),
//             h = P's cell size in the third direction, the faces below (theta of
//             the cells below) or above P and Q;
// faces absent for the staggered cell's type are left out, solid cells give
// init.  With zquirk the z operator reads the x-velocity with M + 1 cells per
// row, as the reference does (calcConvZ launched with M3,
// convective_discrete_operator_z.h:772-773): its x-face indices are shifted
// back by P's layer index.  Products and sums in the reference's order without
// fused multiply-adds, so out is bit-identical to init + (its CSR) v.
__device__ __forceinline__ long long face_index(int e, int N, int M, int x, int y, int z)
{
    const int Ne = N - (e == 0), Me = M - (e == 1);
    return x + (long long)Ne * (y + (long long)Me * z);
}

__global__ void __launch_bounds__(256) k_convective_apply(int d, int N, int M, int K, const int* __restrict__ stype,
                                                          const double* __restrict__ theta,
                                                          const double* __restrict__ delta,
                                                          const double* __restrict__ Ux, const double* __restrict__ Uy,
                                                          const double* __restrict__ Uz, const double* __restrict__ v,
                                                          const double* __restrict__ init, bool zquirk,
                                                          double* __restrict__ out)
{
    const int Nd = N - (d == 0), Md = M - (d == 1);
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= Nd || y >= Md) return;
    const long long f = x + (long long)Nd * (y + (long long)Md * z);
    double acc = init ? init[f] : 0.0;
    const int t = stype[f];
    if (t != 0) {
        const long long NM = (long long)N * M;
        const long long step[3] = {1, N, NM};
        const long long P = x + (long long)N * (y + (long long)M * z), Q = P + step[d];
        const int qx = x + (d == 0), qy = y + (d == 1), qz = z + (d == 2);
        const double* U[3] = {Ux, Uy, Uz};
        const long long dstride = d == 0 ? 1 : (d == 1 ? Nd : (long long)Nd * Md);
        const long long cols[6] = {-(long long)Nd * Md, -Nd, -1, 1, Nd, (long long)Nd * Md};
        const int fdir[6] = {2, 1, 0, 0, 1, 2};
        const int miss = absent_faces(t);
        const double tx = mul(theta[3 * P + d], U[d][f]);
#pragma unroll
        for (int k = 0; k < 6; k++) {
            if (miss & (1 << k)) continue;
            const bool upper = k >= 3;
            const int e = fdir[k];
            double coef;
            if (e == d) {
                const int o0 = d == 0 ? 1 : 0, o1 = d == 2 ? 1 : 2;
                const double area = mul(delta[3 * P + o0], delta[3 * P + o1]);
                const double th2 = upper ? theta[3 * Q + d] : theta[3 * (P - step[d]) + d];
                const double u2 = upper ? U[d][f + dstride] : U[d][f - dstride];
                coef = mul(mul(upper ? 0.25 : -0.25, area), add(tx, mul(th2, u2)));
            } else {
                const int third = 3 - d - e;
                const double h = delta[3 * P + third];
                const long long pc = upper ? P : P - step[e], qc = upper ? Q : Q - step[e];
                // coordinates of the two cells whose e-faces are used
                const int px = x - (!upper && e == 0), py = y - (!upper && e == 1), pz = z - (!upper && e == 2);
                const int cx = qx - (!upper && e == 0), cy = qy - (!upper && e == 1), cz = qz - (!upper && e == 2);
                const long long shift = (zquirk && d == 2 && e == 0) ? z : 0;
                const long long fp = face_index(e, N, M, px, py, pz) - shift;
                const long long fq = face_index(e, N, M, cx, cy, cz) - shift;
                const double a = mul(mul(delta[3 * P + d], theta[3 * pc + e]), U[e][fp]);
                const double b = mul(mul(delta[3 * Q + d], theta[3 * qc + e]), U[e][fq]);
                coef = mul(mul(upper ? 0.25 : -0.25, h), add(a, b));
            }
            acc = add(acc, mul(coef, v[f + cols[k]]));
        }
    }
    out[f] = acc;
}

// Transposed Jacobian of the convective term out = init + C(U) v
// (k_convective_apply): out is bilinear in (U, v), so for a cotangent lam on
// the d-grid
//   v_bar[f + col_k]  += lam_f coef_k(U)
//   U_bar[e][face]    += lam_f v[f + col_k] dcoef_k/dU_e[face]
// for every face k of every non-solid row f, with the same face model,
// absent faces and z-operator x-velocity indexing as the forward kernel.
// Contributions of neighbouring rows meet in one unknown, so they are added
// with atomics (their order is not fixed).  The outputs accumulate; for the
// momentum equation's own velocity (v = U_d) pass the same buffer for v_bar
// and U_bar[d].
__global__ void __launch_bounds__(256) k_convective_adjoint(int d, int N, int M, int K, const int* __restrict__ stype,
                                                            const double* __restrict__ theta,
                                                            const double* __restrict__ delta,
                                                            const double* __restrict__ Ux,
                                                            const double* __restrict__ Uy,
                                                            const double* __restrict__ Uz,
                                                            const double* __restrict__ v,
                                                            const double* __restrict__ lam, bool zquirk,
                                                            double* Ux_bar, double* Uy_bar, double* Uz_bar,
                                                            double* v_bar)
{
    const int Nd = N - (d == 0), Md = M - (d == 1);
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= Nd || y >= Md) return;
    const long long f = x + (long long)Nd * (y + (long long)Md * z);
    const int t = stype[f];
    const double lf = lam[f];
    if (t == 0 || lf == 0.0) return;
    const long long NM = (long long)N * M;
    const long long step[3] = {1, N, NM};
    const long long P = x + (long long)N * (y + (long long)M * z), Q = P + step[d];
    const int qx = x + (d == 0), qy = y + (d == 1), qz = z + (d == 2);
    const double* U[3] = {Ux, Uy, Uz};
    double* Ub[3] = {Ux_bar, Uy_bar, Uz_bar};
    const long long dstride = d == 0 ? 1 : (d == 1 ? Nd : (long long)Nd * Md);
    const long long cols[6] = {-(long long)Nd * Md, -Nd, -1, 1, Nd, (long long)Nd * Md};
    const int fdir[6] = {2, 1, 0, 0, 1, 2};
    const int miss = absent_faces(t);
    for (int k = 0; k < 6; k++) {
        if (miss & (1 << k)) continue;
        const bool upper = k >= 3;
        const int e = fdir[k];
        const double sgn = upper ? 0.25 : -0.25;
        const double vk = v[f + cols[k]];
        const double lv = lf * vk;
        double coef;
        if (e == d) {
            const int o0 = d == 0 ? 1 : 0, o1 = d == 2 ? 1 : 2;
            const double area = delta[3 * P + o0] * delta[3 * P + o1];
            const double th1 = theta[3 * P + d];
            const double th2 = upper ? theta[3 * Q + d] : theta[3 * (P - step[d]) + d];
            const long long f2 = upper ? f + dstride : f - dstride;
            coef = sgn * area * (th1 * U[d][f] + th2 * U[d][f2]);
            atomicAdd(Ub[d] + f, lv * sgn * area * th1);
            atomicAdd(Ub[d] + f2, lv * sgn * area * th2);
        } else {
            const int third = 3 - d - e;
            const double h = delta[3 * P + third];
            const long long pc = upper ? P : P - step[e], qc = upper ? Q : Q - step[e];
            const int px = x - (!upper && e == 0), py = y - (!upper && e == 1), pz = z - (!upper && e == 2);
            const int cx = qx - (!upper && e == 0), cy = qy - (!upper && e == 1), cz = qz - (!upper && e == 2);
            const long long shift = (zquirk && d == 2 && e == 0) ? z : 0;
            const long long fp = face_index(e, N, M, px, py, pz) - shift;
            const long long fq = face_index(e, N, M, cx, cy, cz) - shift;
            const double ca = sgn * h * delta[3 * P + d] * theta[3 * pc + e];
            const double cb = sgn * h * delta[3 * Q + d] * theta[3 * qc + e];
            coef = ca * U[e][fp] + cb * U[e][fq];
            atomicAdd(Ub[e] + fp, lv * ca);
            atomicAdd(Ub[e] + fq, lv * cb);
        }
        atomicAdd(v_bar + f + cols[k], lf * coef);
    }
}

// ---------------------------------------------------------------------------
// Adjoint of the projection (outflow clamps off):
//   b = Pi (Dx u + Dy v + Dz w + flux),  A phi = b,
//   u' = u + S_x Gx phi (likewise v, w),  p' = p + coef phi,
// Pi zeroing the pinned rows and S = diag(inv_vof).  Given the cotangents
// (u'_bar, v'_bar, w'_bar, p'_bar):
//   phi_bar = Gx^T S_x u'_bar + Gy^T S_y v'_bar + Gz^T S_z w'_bar + coef p'_bar,
//   A^T lambda = phi_bar,  b_bar = Pi lambda,
//   u_bar = u'_bar + Dx^T b_bar (likewise v, w),  flux_bar = b_bar,  p_bar = p'_bar.
// The transposed operators are applied from the geometry like the forward ones.
// ---------------------------------------------------------------------------

// face coefficient of the gradient row of the staggered cell whose lower base
// cell is P (GradientDiscreteOperator*::calc): c = (theta_P[dir] d1_P) d2_P
__device__ __forceinline__ double grad_coef(int dir, const double* __restrict__ theta, const double* __restrict__ delta,
                                            long long P)
{
    const double d1 = delta[3 * P + (dir == 0 ? 1 : 0)];
    const double d2 = delta[3 * P + (dir == 2 ? 1 : 2)];
    return theta[3 * P + dir] * d1 * d2;
}

// phi_bar at every base cell: sum over the cell's faces of +-c S u'_bar, plus coef p'_bar
__global__ void __launch_bounds__(256) k_projection_adjoint_phi(int N, int M, int K, const int* __restrict__ xtype,
                                                                const int* __restrict__ ytype,
                                                                const int* __restrict__ ztype,
                                                                const double* __restrict__ theta,
                                                                const double* __restrict__ delta,
                                                                const double* __restrict__ inv_x,
                                                                const double* __restrict__ inv_y,
                                                                const double* __restrict__ inv_z,
                                                                const double* __restrict__ ub,
                                                                const double* __restrict__ vb,
                                                                const double* __restrict__ wb,
                                                                const double* __restrict__ pb, double coef,
                                                                double* __restrict__ phib)
{
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= N || y >= M) return;
    const long long NM = (long long)N * M;
    const long long i = x + (long long)N * y + NM * z;
    double acc = coef * pb[i];
    // x-faces: east (P = i) and west (P = i - 1); x-grid index numX = i - y - z M
    const long long fx = i - y - (long long)z * M;
    // inv_* == nullptr: unit weights (the plain transposed gradient)
    auto w = [](const double* __restrict__ inv, long long f) { return inv ? inv[f] : 1.0; };
    if (x < N - 1 && xtype[fx] != 0) acc += grad_coef(0, theta, delta, i) * w(inv_x, fx) * ub[fx];
    if (x > 0 && xtype[fx - 1] != 0) acc -= grad_coef(0, theta, delta, i - 1) * w(inv_x, fx - 1) * ub[fx - 1];
    // y-faces: north (P = i) and south (P = i - N); y-grid index i - z N
    const long long fy = i - (long long)z * N;
    if (y < M - 1 && ytype[fy] != 0) acc += grad_coef(1, theta, delta, i) * w(inv_y, fy) * vb[fy];
    if (y > 0 && ytype[fy - N] != 0) acc -= grad_coef(1, theta, delta, i - N) * w(inv_y, fy - N) * vb[fy - N];
    // z-faces: top (P = i) and bottom (P = i - NM); z-grid index i
    if (z < K - 1 && ztype[i] != 0) acc += grad_coef(2, theta, delta, i) * w(inv_z, i) * wb[i];
    if (z > 0 && ztype[i - NM] != 0) acc -= grad_coef(2, theta, delta, i - NM) * w(inv_z, i - NM) * wb[i - NM];
    phib[i] = acc;
}

// divergence entry of base cell P's row for its upper face (dir) and of cell
// E's row for its lower face, as DivergenceDiscreteOperatorX/Y/Z::calcD* build
// them (solid rows hold a zero; upper face: +theta_P dS on W/S/B-border rows
// and interior rows; lower face: -theta_P dS on E/N/T-border and interior rows)
__device__ __forceinline__ double div_upper(int dir, int t, const double* __restrict__ theta,
                                            const double* __restrict__ delta, long long P)
{
    if (t == 0) return 0.0;
    const double d0 = delta[3 * P], d1 = delta[3 * P + 1], d2 = delta[3 * P + 2];
    const double th = theta[3 * P + dir];
    if (dir == 0) return fam_w(t) ? th * d1 * d2 : th * (d1 * d2);
    if (dir == 1) return fam_s(t) ? th * d0 * d2 : th * (d0 * d2);
    return fam_b(t) ? th * d0 * d1 : th * (d0 * d1);
}
__device__ __forceinline__ double div_lower(int dir, int t, const double* __restrict__ theta,
                                            const double* __restrict__ delta, long long E, long long P)
{
    if (t == 0) return 0.0;
    const double d0 = delta[3 * E], d1 = delta[3 * E + 1], d2 = delta[3 * E + 2];
    const double th = -theta[3 * P + dir];
    if (dir == 0) return fam_e(t) ? th * d1 * d2 : th * (d1 * d2);
    if (dir == 1) return fam_n(t) ? th * d0 * d2 : th * (d0 * d2);
    return fam_t(t) ? th * d0 * d1 : th * (d0 * d1);
}

// u_bar = u'_bar + D^T b_bar on one staggered grid; b_bar is lambda with the
// pinned rows zeroed
__global__ void __launch_bounds__(256) k_projection_adjoint_vel(int dir, int N, int M, int K,
                                                                const int* __restrict__ type,
                                                                const double* __restrict__ theta,
                                                                const double* __restrict__ delta,
                                                                const double* __restrict__ lambda, long long pin0,
                                                                long long pin1, const double* __restrict__ outbar,
                                                                double* __restrict__ inbar)
{
    const int Ns = N - (dir == 0), Ms = M - (dir == 1);
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= Ns || y >= Ms) return;
    const long long f = x + (long long)Ns * (y + (long long)Ms * z);
    const long long P = x + (long long)N * (y + (long long)M * z);
    const long long E = P + (dir == 0 ? 1 : (dir == 1 ? N : (long long)N * M));
    const double bP = (P == pin0 || P == pin1) ? 0.0 : lambda[P];
    const double bE = (E == pin0 || E == pin1) ? 0.0 : lambda[E];
    inbar[f] = outbar[f] + div_upper(dir, type[P], theta, delta, P) * bP +
               div_lower(dir, type[E], theta, delta, E, P) * bE;
}

// flux_bar = lambda with the pinned rows zeroed
__global__ void k_pin_zero_copy(long long n, long long pin0, long long pin1, const double* __restrict__ lambda,
                                double* __restrict__ out)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = (i == pin0 || i == pin1) ? 0.0 : lambda[i];
}

// The adjoint right-hand side restricted to the rows the forward solve can
// excite.  Solid rows (a decoupled 1e-16 diagonal) and empty rows (cut cells
// whose faces are all closed) see a zero right-hand side in every forward
// projection, and no velocity reads their pressure, so the forward map does
// not depend on the pressure cotangent there; dropping it keeps a
// 1e16-scaled component out of the transposed Krylov solve.
__global__ void k_adjoint_live_rows(long long n, const int* __restrict__ type, const double* __restrict__ A7,
                                    double* __restrict__ v)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        bool live = type[i] != 0;
        if (live) {
            bool any = false;
#pragma unroll
            for (int s = 0; s < 7; s++) any = any || (A7[(size_t)s * n + i] != 0.0);
            live = any;
        }
        if (!live) v[i] = 0.0;
    }
}

// Cotangent algebra of one momentum equation in the reverse sweep of the
// time steps (the transposes of HelmholtzDiscreteEquation::recalcRightMember's
// BDF2 / Adams-Bashforth terms, helmholtz_discrete_equation.h:213-254), for
// r = the transposed momentum solve's solution on the fluid faces (0 on solid
// faces):
//   fb += vof r          forcing cotangent (forcing enters as vof f)
//   ub += (-2 c2) vof r  current velocity (the 2 u^n / dt mass term)
//   upb = (c2 / 2) vof r previous velocity (the -u^{n-1} / (2 dt) term)
//   pab = -r             Adams-Bashforth history a^{n-1}
//   cb += 2 r            convective term of this step
__global__ void k_momentum_cotangents(long long n, const int* __restrict__ stype, const double* __restrict__ vof,
                                      const double* __restrict__ rsol, double c2, double* __restrict__ r,
                                      double* __restrict__ fb, double* __restrict__ ub, double* __restrict__ upb,
                                      double* __restrict__ pab, double* __restrict__ cb)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double rv = (stype[i] != 0) ? rsol[i] : 0.0;
        const double v = vof[i];
        r[i] = rv;
        fb[i] += ((stype[i] != 0) ? v : 0.0) * rv;
        ub[i] += ((-2.0 * c2) * v) * rv;
        upb[i] = ((0.5 * c2) * v) * rv;
        pab[i] = -rv;
        cb[i] += 2.0 * rv;
    }
}

// out = in on the staggered grid's fluid faces, 0 on its solid faces
__global__ void k_fluid_faces(long long n, const int* __restrict__ stype, const double* __restrict__ in,
                              double* __restrict__ out)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = (stype[i] != 0) ? in[i] : 0.0;
}

// Transpose of the outflow clamps of SetSolutions::correction
// (Base/set_solutions.h:87-118, :297-304): the clamps overwrite entries with
// constants, so their transpose zeroes the cotangents of those entries.  q =
// the velocities before the clamps decides which: per interior (y, z) row of
// the east outflow (y in 1..M-2, z in 1..K-2), if the x-face value at the
// row's last or next-to-last face is negative, that x-face and the matching
// y- and z-faces; a bottom z-face (k = 0) with positive and a top one
// (k = K-2) with negative velocity.  out holds a copy of the cotangents; the
// two kernels zero the clamped entries in place.
__global__ void k_clamp_transpose_east(int N, int M, int K, const double* __restrict__ qx, double* __restrict__ ox,
                                       double* __restrict__ oy, double* __restrict__ oz)
{
    const long long rows = (long long)(M - 2) * (K - 2);
    const int NM = N * M;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < 2 * rows;
         e += (long long)gridDim.x * blockDim.x) {
        const int sh = (int)(e / rows);
        const long long r = e - sh * rows;
        const int zz = 1 + (int)(r / (M - 2)), yy = 1 + (int)(r % (M - 2));
        const int num = (yy + 1) * N - 1 + zz * NM;         // last base cell of the row
        const int num2 = num - yy - 1 - zz * M;             // its x-face
        const int num3 = num - zz * N;                      // its y-face
        if (qx[num2 - sh] < 0.0) {
            ox[num2 - sh] = 0.0;
            oy[num3 - sh] = 0.0;
            oz[num - sh] = 0.0;
        }
    }
}

__global__ void k_clamp_transpose_tb(int N, int M, int K, const double* __restrict__ qz, double* __restrict__ oz)
{
    const long long faces = (long long)(N - 1) * (M - 1);
    const int NM = N * M;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < faces;
         e += (long long)gridDim.x * blockDim.x) {
        const int yy = 1 + (int)(e / (N - 1)), xx = 1 + (int)(e % (N - 1));
        const int nb = xx + yy * N, nt = nb + (K - 2) * NM;
        if (qz[nb] > 0.0) oz[nb] = 0.0;
        if (qz[nt] < 0.0) oz[nt] = 0.0;
    }
}

// dst[di[e]] += coef[e] * src[si[e]] * (src2 ? src2[s2i[e]] : 1): the
// boundary source terms' transposes (index sets built once on the host).
// FP64 atomic adds: entries that share a destination add in an unspecified
// order.
__global__ void k_scatter_add(long long count, double* dst, const long long* __restrict__ di,
                              const double* __restrict__ src, const long long* __restrict__ si,
                              const double* __restrict__ coef, const double* __restrict__ src2,
                              const long long* __restrict__ s2i)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count;
         e += (long long)gridDim.x * blockDim.x) {
        double v = coef[e] * src[si[e]];
        if (src2) v *= src2[s2i[e]];
        atomicAdd(dst + di[e], v);
    }
}

__global__ void k_axpy(long long n, double alpha, const double* __restrict__ x, double* __restrict__ y)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] += alpha * x[i];
}

}  // namespace lsg
