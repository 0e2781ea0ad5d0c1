// Momentum (Helmholtz) operators assembled on the GPU from the cut-cell
// geometry: K_d = -(coef) M_d + nu * (cut-cell Laplacian on the staggered
// d-grid) with the box-boundary, immersed-boundary and outflow terms of
// HelmholtzDiscreteOperatorX/Y/Z::calcHelm* (DiscreteOperators/WithFlux/Sym/
// helmholtz_discrete_operator_x.h:98-686, _y.h:92-…, _z.h:90-…) and
// addPlusOutFlow/setPlusOutFlow* (helmholtz_discrete_operator_base.h:50-58,
// _x.h:732-737, _y.h:736-742, _z.h:726-732).
//
// The reference writes one formula block per cell type (fluid, solid, six
// borders, twelve edges, eight corners, cut cells); here every row comes from
// one face model of the staggered cell:
//   * lateral face (direction l != d, lower or upper): coefficient
//       nu dperp (theta_l(Q) da + theta_l(Q+up) da') alpha_r(Q) / (t_d dl + theta_d(nb) dl(nb)),
//     Q the cell owning the face, nb the neighbour across it, r the third
//     direction; for a fluid cell (dperp nu (da' + da)) / (dl + theta_d(nb) dl(nb));
//   * axial face: nu t_d (dl1 dl2)^2 / V of the base cell on that side
//     (nu (dl1 dl2)^2 / V for a fluid cell), entry scaled by the neighbour's
//     theta_d;
//   * cut cells (and some borders, below) drop a lateral face whose edge
//     fraction alpha is below 1e-5 and add the immersed-boundary term of
//     that direction pair instead.
// The per-type differences of the reference are flags of that model:
//   * a face on the box side is not an entry; on the outflow side (E) the
//     coefficient stays in the diagonal, on the inflow side (W) it is dropped;
//   * walls: lateral N/S walls of the x and z operators and T/B walls of the
//     x and y operators (the latter only for tasks other than flows) add the
//     upper lateral numerator at the cell over t_d dl; the N/S walls of the y
//     operator keep the axial coefficient without the t_d factor, the T/B
//     walls of the z operator (non-flow tasks) keep it with the factor;
//   * T/B borders of all three operators gate their lateral faces like cut
//     cells; the immersed-boundary terms they add follow the reference's
//     conditions (x: T adds the z pair when alpha_y(P) or the b face is
//     gated, B when the t face is; y: only the face it keeps; z: both pairs);
//   * y-operator edges and corners with a T/B wall evaluate the wall term
//     after the reference has overwritten dx by dx dz, and its TE/TW/BE/BW
//     edges after dyy has become nu t_y (dx dz)^2 (values reproduced).
// Fluid and cut-cell rows use the reference's operation order (bitwise); the
// box-boundary rows agree to rounding (their diagonal sums are taken in the
// cut-cell order).
#pragma once

#include "lsg_kernels.cuh"

namespace lsg {

struct HelmGeom {
    int N, M, K;                   // base grid
    int d;                         // 0 x, 1 y, 2 z operator
    const int* stype;              // staggered cell types
    const double* theta;           // 3n
    const double* alpha;           // 3n
    const double* delta;           // 3n
    const double* inv_vof;         // n (base cells)
    const double* vof;             // staggered cell volumes
    const double* dib_en;          // 3n immersed-boundary distances
    const double* dib_ws;
    const double* dib_nb;
    const double* dib_st;
    const double* inv_dib_ne;      // 3n inverse distances
    const double* inv_dib_tn;
    double nu, coef;
    int is_flow;
    double* planes;                // 7 * ns: b s w p e n t
};

__device__ __forceinline__ double h_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double h_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double h_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double h_div(double a, double b) { return __ddiv_rn(a, b); }

// immersed-boundary term of operator d for the lateral pair in direction l
__device__ __forceinline__ double helm_ib(const HelmGeom& g, int l, long long P, long long up)
{
    const double* A;
    const double* B;
    const double* I;
    int c, ci;
    if (g.d == 0) {
        A = g.dib_en; B = g.dib_ws; I = g.inv_dib_ne;
        c = (l == 1) ? 1 : 0;
        ci = (l == 1) ? 1 : 2;
    } else if (g.d == 1) {
        if (l == 0) { A = g.dib_en; B = g.dib_ws; I = g.inv_dib_ne; c = 2; ci = 0; }
        else { A = g.dib_nb; B = g.dib_st; I = g.inv_dib_tn; c = 0; ci = 2; }
    } else {
        A = g.dib_st; B = g.dib_nb; I = g.inv_dib_tn;
        c = (l == 0) ? 2 : 1;
        ci = (l == 0) ? 0 : 1;
    }
    return h_mul(h_mul(g.nu, h_add(A[3 * P + c], B[3 * (P + up) + c])), I[3 * P + ci]);
}

__global__ void __launch_bounds__(256) k_helmholtz_from_geometry(HelmGeom g)
{
    const int d = g.d;
    const int N = g.N, M = g.M;
    const long long NM = (long long)N * M;
    const int Ns = N - (d == 0), Ms = M - (d == 1), Ks = g.K - (d == 2);
    const long long ns = (long long)Ns * Ms * Ks;
    const long long step[3] = {1, N, NM};
    const long long up = step[d];
    const int l0 = d == 0 ? 1 : 0, l1 = d == 2 ? 1 : 2;      // lateral directions, lower first
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ns;
         i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % Ns);
        const long long rest = i / Ns;
        const int y = (int)(rest % Ms), z = (int)(rest / Ms);
        const long long P = x + (long long)N * (y + (long long)M * z);
        const int t = g.stype[i];
        double e[7] = {0, 0, 0, 0, 0, 0, 0};
        if (t == 0) {
            e[3] = 1e-16;                                      // PLUS_TINY
        } else {
            const int miss = absent_faces(t);
            // face bits of absent_faces by (axis, side)
            auto bit = [](int ax, int side) {
                return ax == 0 ? (side < 0 ? 4 : 8) : (ax == 1 ? (side < 0 ? 2 : 16) : (side < 0 ? 1 : 32));
            };
            const bool fluid = (t == 11111111);
            const bool cut = t > 0 && !fluid;
            const bool tb_border = (t == -2 || t == -3);
            const bool gating = cut || tb_border;
            const double* th = g.theta;
            const double* de = g.delta;
            const double* al = g.alpha;
            const double ta = th[3 * P + d];
            const double da = de[3 * P + d], da2 = de[3 * (P + up) + d];
            double kl[3][2] = {{0, 0}, {0, 0}, {0, 0}};
            bool gated[3][2] = {{false, false}, {false, false}, {false, false}};
            for (int q = 0; q < 2; q++) {
                const int l = q == 0 ? l0 : l1;
                const int r = 3 - d - l;
                const long long sl = step[l];
                const double dperp = de[3 * P + r];
                for (int s = 0; s < 2; s++) {
                    const int side = s == 0 ? -1 : 1;
                    const bool on_box = (miss & bit(l, side)) != 0;
                    // the outflow face (E) stays in the diagonal of the y and z operators
                    if (on_box && !(l == 0 && side > 0)) continue;
                    const long long Q = side < 0 ? P - sl : P;
                    const long long nb = side < 0 ? P - sl : P + sl;
                    const double den_n = h_mul(th[3 * nb + d], de[3 * nb + l]);
                    if (fluid) {
                        const double aux = h_mul(dperp, h_mul(g.nu, h_add(da2, da)));
                        kl[l][s] = h_div(aux, h_add(de[3 * P + l], den_n));
                    } else {
                        const double a = al[3 * Q + r];
                        if (gating && a < 1e-5) {
                            gated[l][s] = true;
                            continue;
                        }
                        const double aux = h_mul(dperp, g.nu);
                        const double num =
                            h_mul(h_mul(aux, h_add(h_mul(th[3 * Q + l], da), h_mul(th[3 * (Q + up) + l], da2))), a);
                        kl[l][s] = h_div(num, h_add(h_mul(ta, de[3 * P + l]), den_n));
                    }
                }
            }
            // axial coefficients
            const double A = h_mul(de[3 * P + l0], de[3 * P + l1]);
            const double f0 = fluid ? h_mul(h_mul(g.nu, A), A) : h_mul(h_mul(h_mul(g.nu, ta), A), A);
            const double kax_lo = h_mul(f0, g.inv_vof[P]);
            const double kax_hi = h_mul(f0, g.inv_vof[P + up]);
            // immersed-boundary terms
            double ib = 0.0;
            const bool ib_l0 = gated[l0][0] || gated[l0][1];
            // the x operator's T border also adds the z pair when alpha_y of the cell is below 1e-5
            const bool ib_l1 = gated[l1][0] || gated[l1][1] || (d == 0 && t == -2 && al[3 * P + 1] < 1e-5);
            if (ib_l0) ib = helm_ib(g, l0, P, up);
            if (ib_l1) ib = h_add(ib, helm_ib(g, l1, P, up));
            // entries
            const bool lo_box = (miss & bit(d, -1)) != 0, hi_box = (miss & bit(d, 1)) != 0;
            if (!lo_box) e[d == 0 ? 2 : (d == 1 ? 1 : 0)] = h_mul(kax_lo, th[3 * (P - up) + d]);
            if (!hi_box) e[d == 0 ? 4 : (d == 1 ? 5 : 6)] = h_mul(kax_hi, th[3 * (P + up) + d]);
            const int slot_lo[3] = {2, 1, 0}, slot_hi[3] = {4, 5, 6};
            for (int q = 0; q < 2; q++) {
                const int l = q == 0 ? l0 : l1;
                if (!(miss & bit(l, -1))) e[slot_lo[l]] = kl[l][0];
                if (!(miss & bit(l, 1))) e[slot_hi[l]] = kl[l][1];
            }
            // diagonal
            double dg = -h_mul(g.coef, g.vof[i]);
            if (fluid) {
                // CSR order b s w e n t (the reference's fluid rows)
                const double kk[6] = {d == 2 ? kax_lo : kl[2][0], d == 1 ? kax_lo : kl[1][0],
                                      d == 0 ? kax_lo : kl[0][0], d == 0 ? kax_hi : kl[0][1],
                                      d == 1 ? kax_hi : kl[1][1], d == 2 ? kax_hi : kl[2][1]};
                const int fb[6] = {1, 2, 4, 8, 16, 32};
                for (int f = 0; f < 6; f++)
                    if (!(miss & fb[f])) dg = h_sub(dg, kk[f]);
            } else {
                // lateral lower faces, the axial pair, lateral upper faces, then
                // walls and immersed-boundary terms (the reference's cut-cell order)
                dg = h_sub(dg, kl[l1][0]);
                dg = h_sub(dg, kl[l0][0]);
                double ax = 0.0;
                bool any_ax = false;
                double ax_plain = 0.0;
                for (int s = 0; s < 2; s++) {
                    const int side = s == 0 ? -1 : 1;
                    const double kv = s == 0 ? kax_lo : kax_hi;
                    if (!(miss & bit(d, side))) {
                        ax = any_ax ? h_add(ax, kv) : kv;
                        any_ax = true;
                    } else if (d == 0 && side > 0) {
                        ax = any_ax ? h_add(ax, kv) : kv;         // outflow face of the x operator
                        any_ax = true;
                    } else if (d == 1) {
                        ax_plain = h_add(ax_plain, kv);            // y: N/S wall keeps the coefficient
                    } else if (d == 2 && !g.is_flow) {
                        ax = any_ax ? h_add(ax, kv) : kv;          // z: T/B wall of a non-flow task
                        any_ax = true;
                    }
                }
                if (any_ax) dg = h_sub(dg, h_mul(ax, ta));
                dg = h_sub(dg, kl[l0][1]);
                dg = h_sub(dg, kl[l1][1]);
                dg = h_sub(dg, ax_plain);
                // lateral walls
                for (int q = 0; q < 2; q++) {
                    const int l = q == 0 ? l0 : l1;
                    const int r = 3 - d - l;
                    for (int s = 0; s < 2; s++) {
                        const int side = s == 0 ? -1 : 1;
                        if (!(miss & bit(l, side))) continue;
                        const bool ns_wall = (l == 1) && (d == 0 || d == 2);
                        const bool tb_wall = (l == 2) && (d == 0 || d == 1) && !g.is_flow;
                        if (!ns_wall && !tb_wall) continue;
                        const bool checked = !(d == 2 && (t == -4 || t == -5));
                        if (checked && !(ta > 1e-5)) continue;
                        double dr = de[3 * P + r];
                        double d2 = da2;
                        if (d == 1 && l == 2 && t <= -8) {
                            dr = h_mul(dr, de[3 * P + 2]);
                            if (t == -10 || t == -11 || t == -14 || t == -15) d2 = h_mul(h_mul(h_mul(g.nu, ta), dr), dr);
                        }
                        const double num = h_mul(h_mul(h_mul(dr, g.nu),
                                                       h_add(h_mul(th[3 * P + l], da), h_mul(th[3 * (P + up) + l], d2))),
                                                 al[3 * P + r]);
                        dg = h_sub(dg, h_div(num, h_mul(ta, de[3 * P + l])));
                    }
                }
                dg = h_sub(dg, ib);
            }
            if (g.is_flow && (miss & 8)) {
                // convective outflow on the last cell of each row
                double po;
                if (d == 0) {
                    const long long Pb = P + 1;
                    po = h_div(h_mul(h_mul(g.nu, de[3 * Pb + 1]), de[3 * Pb + 2]), de[3 * Pb]);
                } else if (d == 1) {
                    po = h_div(h_mul(h_mul(g.nu, h_add(de[3 * P + 1], de[3 * (P + N) + 1])), de[3 * P + 2]), de[3 * P]);
                } else {
                    po = h_div(h_mul(h_mul(g.nu, h_add(de[3 * P + 2], de[3 * (P + NM) + 2])), de[3 * P + 1]), de[3 * P]);
                }
                dg = h_add(dg, po);
            }
            e[3] = dg;
        }
        for (int f = 0; f < 7; f++) g.planes[(size_t)f * ns + i] = e[f];
    }
}

}  // namespace lsg

namespace lsg {

// Source term of the momentum operator of direction d as build() leaves it
// (initInFlowFlux: inFlowFluxHelm*, addFluxNS*, addFluxTB*,
// helmholtz_discrete_operator_x.h:50-96 and :750-758, _y.h, _z.h), one thread
// per staggered cell: the inflow value on x = 0 is assigned, then the S/N
// wall terms and the B/T wall terms (non-solid cells) are added, in that
// order.  The T/B terms are present for flow tasks too (the reference builds
// them before it marks the operator as having an outflow).  The reference's
// index choices are kept: the N-row terms use the S row's dx and dz, the x
// operator's N coefficient reads dy at base index (N-1)(M-1)+zNM, the y
// operator's T coefficient reads dz at base (y, y, K-1).
// With ib != 0 the immersed-boundary term (ibFluxHelmX/Y/Z, :687-731) is then
// written over rows 1 .. Ms-2: cut cells, and T/B borders with a cut face,
// get it; every other cell of those rows gets 0.
struct HelmFluxArgs {
    HelmGeom g;
    const int* side_type;         // 3n (ib only)
    const double* vib;            // 3n (ib only)
    const double* vyx;
    const double* vzy;
    const double* u_w;            // x-inflow profile, M*K
    double bc[18];                // U_W U_E U_S U_N U_B U_T, V_*, W_*
    int ib;
    double* flux;
};

__device__ __forceinline__ bool helm_cut_face(const int* sd, long long P)
{
    const int a = sd[3 * P], b = sd[3 * P + 1], c = sd[3 * P + 2];
    return (a > 0 && a < 1111) || (b > 0 && b < 1111) || (c > 0 && c < 1111);
}

__global__ void __launch_bounds__(256) k_helmholtz_flux(HelmFluxArgs a)
{
    const HelmGeom& g = a.g;
    const int d = g.d;
    const int N = g.N, M = g.M, K = g.K;
    const long long NM = (long long)N * M;
    const int Ns = N - (d == 0), Ms = M - (d == 1), Ks = K - (d == 2);
    const long long nsm = (long long)Ns * Ms, ns = nsm * Ks;
    const double* de = g.delta;
    const double nu = g.nu;
    const double S_ = a.bc[6 * d + 2], N_ = a.bc[6 * d + 3], B_ = a.bc[6 * d + 4], T_ = a.bc[6 * d + 5];
    const double W_ = a.bc[6 * d];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ns;
         i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % Ns);
        const long long rest = i / Ns;
        const int y = (int)(rest % Ms), z = (int)(rest / Ms);
        const long long P = x + (long long)N * (y + (long long)M * z);
        const int t = g.stype[i];
        double f = 0.0;
        if (x == 0) {
            if (d == 0)
                f = h_div(h_mul(a.u_w[y + (long long)z * M], h_mul(h_mul(nu, de[3 * P + 2]), de[3 * P + 1])), de[3 * P]);
            else if (d == 1)
                f = h_div(h_mul(W_, h_mul(h_mul(nu, de[3 * P + 2]), h_add(de[3 * P + 1], de[3 * (P + N) + 1]))),
                          de[3 * P]);
            else
                f = h_div(h_mul(W_, h_mul(h_mul(nu, de[3 * P + 1]), h_add(de[3 * P + 2], de[3 * (P + NM) + 2]))),
                          de[3 * P]);
        }
        if (y == 0 || y == Ms - 1) {
            const long long b0 = (long long)z * NM;
            const bool north = (y == Ms - 1);
            double coef;
            if (d == 0) {
                const long long q = north ? (nsm * z + nsm - Ns) + (long long)z * M : b0;
                coef = h_div(h_mul(h_mul(nu, north ? N_ : S_), de[3 * b0 + 2]), de[3 * q + 1]);
            } else if (d == 1) {
                const long long q = north ? b0 + (long long)N * (M - 2) : b0;
                coef = h_div(h_mul(h_mul(nu, north ? N_ : S_), de[3 * b0 + 2]), de[3 * q + 1]);
            } else {
                const double dzz = h_add(de[3 * b0 + 2], de[3 * (b0 + NM) + 2]);
                const long long q = north ? b0 + NM - N : b0;
                coef = h_div(h_mul(h_mul(nu, north ? N_ : S_), dzz), de[3 * q + 1]);
            }
            const double c = d == 0 ? h_add(de[3 * (b0 + x)], de[3 * (b0 + x + 1)]) : de[3 * (b0 + x)];
            f = h_add(f, h_mul(c, coef));
        }
        if ((z == 0 || z == Ks - 1) && t != 0) {
            const long long b0 = (long long)N * y;
            const bool top = (z == Ks - 1);
            double coef;
            if (d == 0) {
                coef = h_div(h_mul(h_mul(nu, top ? T_ : B_), de[3 * b0 + 1]),
                             de[3 * (top ? b0 + (long long)(K - 1) * NM : b0) + 2]);
            } else if (d == 1) {
                const double dyy = h_add(de[3 * b0 + 1], de[3 * (b0 + N) + 1]);
                const long long numT = (long long)(Ks - 1) * nsm + (long long)y * Ns;
                coef = h_div(h_mul(h_mul(nu, top ? T_ : B_), dyy),
                             de[3 * (top ? numT + y + (long long)(K - 1) * N : b0) + 2]);
            } else {
                coef = h_div(h_mul(h_mul(nu, top ? T_ : B_), de[3 * b0 + 1]),
                             de[3 * (top ? b0 + (long long)(K - 2) * NM : b0) + 2]);
            }
            const double c = d == 0 ? h_add(de[3 * (b0 + x)], de[3 * (b0 + x + 1)]) : de[3 * (b0 + x)];
            f = h_add(f, h_mul(c, coef));
        }
        if (a.ib && y >= 1 && y <= Ms - 2) {
            const long long up = d == 0 ? 1 : (d == 1 ? N : NM);
            bool cut = t > 0 && t < 11111111;
            if (t == -2 || t == -3) cut = helm_cut_face(a.side_type, P) || (d != 2 && helm_cut_face(a.side_type, P + up));
            const double* th = g.theta;
            const double* al = g.alpha;
            const double ta = th[3 * P + d];
            if (!cut || ta < 1e-5) {
                f = 0.0;
            } else {
                const long long bnum = z ? NM : 0;
                double a2, ib = 0.0, lo;
                if (d == 0) {
                    a2 = h_mul(de[3 * P + 1], de[3 * P + 2]);
                    if (al[3 * P + 2] < 1e-5 || al[3 * (P - N) + 2] < 1e-5)
                        ib = h_mul(h_mul(h_add(g.dib_en[3 * P + 1], g.dib_ws[3 * (P + 1) + 1]), g.inv_dib_ne[3 * P + 1]),
                                   a.vyx[3 * P]);
                    if (al[3 * P + 1] < 1e-5 || al[3 * (P - bnum) + 1] < 1e-5)
                        ib = h_add(ib, h_mul(h_mul(h_add(g.dib_en[3 * P], g.dib_ws[3 * (P + 1)]), g.inv_dib_ne[3 * P + 2]),
                                             a.vzy[3 * P]));
                    lo = th[3 * (P - 1)];
                } else if (d == 1) {
                    a2 = h_mul(de[3 * P], de[3 * P + 2]);
                    if (al[3 * P + 2] < 1e-5 || al[3 * (P - 1) + 2] < 1e-5)
                        ib = h_mul(h_mul(h_add(g.dib_en[3 * P + 2], g.dib_ws[3 * (P + N) + 2]), g.inv_dib_ne[3 * P]),
                                   a.vyx[3 * P + 1]);
                    if (al[3 * P] < 1e-5 || al[3 * (P - bnum)] < 1e-5)
                        ib = h_add(ib, h_mul(h_mul(h_add(g.dib_nb[3 * P], g.dib_st[3 * (P + N)]), g.inv_dib_tn[3 * P + 2]),
                                             a.vzy[3 * P + 1]));
                    lo = th[3 * (P - N) + 1];
                } else {
                    a2 = h_mul(de[3 * P], de[3 * P + 1]);
                    if (al[3 * P + 1] < 1e-5 || al[3 * (P - 1) + 1] < 1e-5)
                        ib = h_mul(h_mul(h_add(g.dib_st[3 * P + 2], g.dib_nb[3 * (P + NM) + 2]), g.inv_dib_tn[3 * P]),
                                   a.vyx[3 * P + 2]);
                    if (al[3 * P] < 1e-5 || al[3 * (P - N)] < 1e-5)
                        ib = h_add(ib, h_mul(h_mul(h_add(g.dib_st[3 * P + 1], g.dib_nb[3 * (P + NM) + 1]),
                                                   g.inv_dib_tn[3 * P + 1]),
                                             a.vzy[3 * P + 2]));
                    lo = th[3 * (P - bnum) + 2];
                }
                const double hi_t = h_mul(h_mul(h_sub(ta, th[3 * (P + up) + d]), a.vib[3 * (P + up) + d]), g.inv_vof[P + up]);
                const double lo_t = h_mul(h_mul(h_sub(lo, ta), a.vib[3 * P + d]), g.inv_vof[P]);
                f = h_mul(nu, h_add(ib, h_mul(h_mul(h_mul(ta, a2), a2), h_sub(hi_t, lo_t))));
            }
        }
        a.flux[i] = f;
    }
}

}  // namespace lsg

namespace lsg {

// Boundary source term of the z convective operator as the time step
// recomputes it (ConvectiveDiscreteOperatorZ::baseFlux,
// convective_discrete_operator_z.h:748-757: baseFluxz, addFluxNSz,
// addFluxTBOutZ), one thread per z-grid cell, in the reference's order
// (inflow / outflow value assigned, then the S/N and B/T terms added).  The
// outflow value uses the row's first cell's sizes, as the reference does.
// The x and y operators' source terms are 0 in the reference (their
// baseFluxX/baseFluxY never run), so no kernel exists for them.
struct ConvFluxArgs {
    int N, M, K;
    const double* theta;
    const double* delta;
    const double* ux;
    const double* uz;
    const double* u_w;
    double W_W, VW_S, VW_N;       // W_W, W_S * V_S, W_N * V_N
    double* flux;
};

__global__ void __launch_bounds__(256) k_convective_flux_z(ConvFluxArgs a)
{
    const int N = a.N, M = a.M, Ks = a.K - 1;
    const long long NM = (long long)N * M, ns = NM * Ks;
    const double* de = a.delta;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ns;
         i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % N);
        const long long rest = i / N;
        const int y = (int)(rest % M), z = (int)(rest / M);
        double f = 0.0;
        if (x == 0 || x == N - 1) {
            const long long numF = (long long)N * y + NM * z;       // the row's first cell
            const long long numW = y + (long long)z * M;
            const double dz = de[3 * numF + 2], dy = de[3 * numF + 1], dzz = de[3 * (numF + NM) + 2];
            if (x == 0) {
                f = h_mul(h_mul(h_mul(-0.25, h_add(h_mul(a.u_w[numW], dz), h_mul(a.u_w[numW + M], dzz))), a.W_W), dy);
            } else {
                const long long last = numF + N - 1, num2 = last - numW - 1;
                f = h_mul(h_mul(h_mul(0.25, a.uz[last]),
                                h_add(h_mul(a.ux[num2], dz), h_mul(a.ux[num2 + (long long)(N - 1) * M], dzz))),
                          dy);
            }
        }
        if (y == 0 || y == M - 1) {
            const long long b0 = (long long)z * NM;
            const double dzz = h_mul(0.25, h_add(de[3 * b0 + 2], de[3 * (b0 + NM) + 2]));
            const double coef = h_mul(de[3 * (b0 + x)], dzz);
            f = (y == 0) ? h_sub(f, h_mul(coef, a.VW_S)) : h_add(f, h_mul(coef, a.VW_N));
        }
        if (z == 0 || z == Ks - 1) {
            const double w = a.uz[i];
            const double t = h_mul(h_mul(h_mul(h_mul(h_mul(0.5, de[3 * i]), de[3 * i + 1]), a.theta[3 * i + 2]), w), w);
            f = (z == 0) ? h_sub(f, t) : h_add(f, t);
        }
        a.flux[i] = f;
    }
}

}  // namespace lsg
