// Aerodynamic loads on the immersed boundary: per-cut-cell forces, their
// sums, moments, and the adjoint of a weighted force sum.
//
// LoadsCalculator::calc (Base/loads_calculator.h:79-1269) gives every cut cell
// a force made of a pressure / normal-stress part and, per cell type, up to
// six tangential shear terms ("quad" terms) of the form
//     S * (v_ib - u) * (1 / delta_ib),
// a face area S (delta_ib_max), an immersed-boundary velocity from v_ib_yx or
// v_ib_zy, a velocity of the staggered grid, and an inverse wall distance
// (inv_delta_ib_ne or inv_delta_ib_tn).  Every term is taken either at the
// cell or one cell behind along the velocity's own axis, or is the sum of
// both; calculate() (:1366-1377) then sums the forces, scales them to
// coefficients and low-pass filters the moments (:1327-1341).
//
// Here the per-type choices are one descriptor byte per shear term, decoded
// on the host once per cut-cell list (lsg_loads_set) together with every
// geometric value the cell reads, packed structure-of-arrays; the per-call
// kernel reads those records coalesced and gathers only the velocities,
// pressure and immersed-boundary velocities.  The arithmetic follows the
// reference expression by expression with round-to-nearest intrinsics (no
// contraction), so per-cell forces and moments are bitwise equal to the
// reference's; the sums are deterministic tree reductions.
#pragma once

#include "lsg_kernels.cuh"

namespace lsg {

// ---------------------------------------------------------------------------
// cell-type descriptors (host)
// ---------------------------------------------------------------------------
namespace loads_desc {
// one byte per shear term, terms in the order uy uz vx vz wx wy
// (the velocity component, then the derivative direction)
constexpr uint8_t Q = 1;       // the term exists for this type
constexpr uint8_t PAIR = 2;    // S * ((v-u) d [behind] + (v-u) d [at the cell])
constexpr uint8_t INNER = 4;   // single term grouped S * ((v-u) * d) instead of (S * (v-u)) * d
constexpr uint8_t BACK = 8;    // single term taken one cell behind along the velocity's axis
constexpr uint8_t TN = 16;     // inverse distance from inv_delta_ib_tn (else inv_delta_ib_ne)
constexpr uint8_t NEG = 32;    // area taken with a minus sign
constexpr uint8_t DHERE = 64;  // BACK term whose inverse distance is still read at the cell
                               // (TNW_Tetrahedron's v_z term, loads_calculator.h:139-140)
struct Row {
    int code;                  // CellTypes value (LS_STAG_Mesh/cut_cells.h:26-168)
    uint8_t slot[6];
};
// The 94 types with shear terms (loads_calculator.h:127-1263); every other
// cell type contributes its pressure / normal-stress part only.
static const Row kRows[] = {
    {        1, {Q, Q, Q|BACK, Q|BACK|DHERE|TN, Q|BACK|TN, Q|BACK|TN}},   // TNW_Tetrahedron
    {       10, {Q|BACK, Q|BACK, Q|BACK, Q|BACK|TN, Q|BACK|TN, Q|BACK|TN}},   // TNE_Tetrahedron
    {       11, {Q|PAIR, Q|PAIR, 0, Q|BACK|TN, 0, Q|BACK|TN}},   // TN_Pentahedron
    {      100, {Q|BACK, Q|BACK, Q, Q|TN, Q|BACK|TN, Q|BACK|TN}},   // TSE_Tetrahedron
    {      110, {0, Q|INNER|BACK, Q|PAIR, Q|PAIR|TN, Q|BACK|TN, 0}},   // TE_Pentahedron
    {      111, {0, Q|PAIR|TN, 0, Q|PAIR|TN, 0, 0}},   // TNTE_Hexahedron5
    {     1000, {Q, Q, Q, Q|TN, Q|BACK|TN, Q|BACK|TN}},   // TSW_Tetrahedron
    {     1001, {0, Q|INNER, Q|PAIR, Q|PAIR|TN, Q|BACK|TN, 0}},   // TW_Pentahedron
    {     1011, {0, Q|PAIR|TN, 0, Q|PAIR|TN, 0, 0}},   // TNTW_Hexahedron5
    {     1100, {Q|PAIR, Q|PAIR, 0, Q|INNER|TN, 0, Q|INNER|BACK|TN}},   // TS_Pentahedron
    {     1101, {0, Q|PAIR|TN, 0, Q|PAIR|TN, 0, 0}},   // TSTW_Hexahedron5
    {     1110, {0, Q|PAIR|TN, 0, Q|PAIR|TN, 0, 0}},   // TSTE_Hexahedron5
    {     1111, {0, Q|PAIR|TN, 0, Q|PAIR|TN, 0, 0}},   // T_Hexahedron4
    {    10000, {Q, Q, Q|BACK, Q|BACK|TN, Q|TN, Q|TN}},   // BNW_Tetrahedron
    {    10001, {Q, 0, Q|BACK, 0, Q|PAIR|TN, Q|PAIR|TN}},   // NW_Pentahedron
    {    10011, {Q|PAIR, 0, 0, 0, 0, Q|PAIR|TN}},   // TNNW_Hexahedron5
    {    11001, {0, 0, Q|PAIR, 0, Q|PAIR|TN, 0}},   // TWNW_Hexahedron5
    {    11011, {Q|BACK, Q|BACK, Q, Q|TN, Q|TN, Q|TN}},   // TNW_Heptahedron6
    {    11111, {0, Q|BACK, 0, Q|TN, Q|TN, Q|TN}},   // TNTW_Heptahedron5
    {   100000, {Q|BACK, Q|BACK, Q|BACK, Q|BACK|TN, Q|TN, Q|TN}},   // BNE_Tetrahedron
    {   100010, {Q|BACK, 0, Q|BACK, 0, Q|PAIR|TN, Q|PAIR|TN}},   // NE_Pentahedron
    {   100011, {Q|PAIR, 0, 0, 0, 0, Q|PAIR|TN}},   // TNNE_Hexahedron5
    {   100110, {0, 0, Q|PAIR, 0, Q|PAIR|TN, 0}},   // TENE_Hexahedron5
    {   100111, {Q, Q, Q, Q|TN, Q|TN, Q|TN}},   // TNE_Heptahedron6
    {   101111, {0, Q, 0, Q|TN, Q|TN, Q|TN}},   // TNTE_Heptahedron5
    {   110000, {Q|PAIR, Q|PAIR, 0, Q|INNER|BACK|TN, 0, Q|INNER|TN}},   // BN_Pentahedron
    {   110001, {Q|PAIR, 0, 0, 0, 0, Q|PAIR|TN}},   // BNNW_Hexahedron5
    {   110010, {Q|PAIR, 0, 0, 0, 0, Q|PAIR|TN}},   // BNNE_Hexahedron5
    {   110011, {Q|PAIR, 0, 0, 0, 0, Q|PAIR|TN}},   // N_Hexahedron4
    {   110111, {Q, 0, Q, Q|TN, 0, Q|TN}},   // TNNE_Heptahedron5
    {   111011, {Q|BACK, 0, Q, Q|TN, 0, Q|TN}},   // TNNW_Heptahedron5
    {   111111, {0, 0, 0, Q|TN, 0, Q|TN}},   // TN_Heptahedron4
    {  1000000, {Q|BACK, Q|BACK, Q, Q|TN, Q|TN, Q|TN}},   // BSE_Tetrahedron
    {  1000100, {Q|BACK, 0, Q, 0, Q|PAIR|TN, Q|PAIR|TN}},   // SE_Pentahedron
    {  1000110, {0, 0, Q|PAIR, 0, Q|PAIR|TN, 0}},   // TESE_Hexahedron5
    {  1001100, {Q|PAIR, 0, 0, 0, 0, Q|PAIR|TN}},   // TSSE_Hexahedron5
    {  1001110, {Q, Q, Q|BACK, Q|BACK|TN, Q|TN, Q|TN}},   // TSE_Heptahedron6
    {  1001111, {0, Q, 0, Q|BACK|TN, Q|TN, Q|TN}},   // TSTE_Heptahedron5
    {  1100000, {0, Q|INNER|BACK, Q|PAIR, Q|PAIR|TN, Q|TN, 0}},   // BE_Pentahedron
    {  1100010, {0, 0, Q|PAIR, 0, Q|PAIR|TN, 0}},   // BENE_Hexahedron5
    {  1100100, {0, 0, Q|PAIR, 0, Q|PAIR|TN, 0}},   // BESE_Hexahedron5
    {  1100110, {0, 0, Q|PAIR, 0, Q|PAIR|TN, 0}},   // E_Hexahedron4
    {  1100111, {Q, Q, Q, 0, Q|TN, 0}},   // TENE_Heptahedron5
    {  1101110, {Q, Q, Q|BACK, 0, Q|TN, 0}},   // TESE_Heptahedron5
    {  1101111, {0, Q, 0, 0, Q|TN, 0}},   // TE_Heptahedron4
    {  1110000, {0, Q|PAIR|TN, 0, Q|PAIR|TN, 0, 0}},   // BNBE_Hexahedron5
    {  1110010, {Q, Q, Q, Q|TN, Q|BACK|TN, Q|BACK|TN}},   // BNE_Heptahedron6
    {  1110011, {Q, 0, Q, Q|TN, 0, Q|BACK|TN}},   // BNNE_Heptahedron5
    {  1110110, {Q, Q, Q, 0, Q|BACK|TN, 0}},   // BENE_Heptahedron5
    {  1110111, {Q, 0, Q, 0, 0, 0}},   // NE_Heptahedron4
    { 10000000, {Q, Q, Q, Q|TN, Q|TN, Q|TN}},   // BSW_Tetrahedron
    { 10001000, {Q, 0, Q, 0, Q|PAIR|TN, Q|PAIR|TN}},   // SW_Pentahedron
    { 10001001, {0, 0, Q|PAIR, 0, Q|PAIR|TN, 0}},   // TWSW_Hexahedron5
    { 10001100, {Q|PAIR, 0, 0, 0, 0, Q|PAIR|TN}},   // TSSW_Hexahedron5
    { 10001101, {Q|BACK, Q|BACK, Q|BACK, Q|BACK|TN, Q|TN, Q|TN}},   // TSW_Heptahedron6
    { 10001111, {0, Q|BACK, 0, Q|BACK|TN, Q|TN, Q|TN}},   // TSTW_Heptahedron5
    { 10010000, {0, Q|INNER, Q|PAIR, Q|PAIR|TN, Q|TN, 0}},   // BW_Pentahedron
    { 10010001, {0, 0, Q|PAIR, 0, Q|PAIR|TN, 0}},   // BWNW_Hexahedron5
    { 10011000, {0, 0, Q|PAIR, 0, Q|PAIR|TN, 0}},   // BWSW_Hexahedron5
    { 10011001, {0, 0, Q|PAIR, 0, Q|PAIR|TN, 0}},   // W_Hexahedron4
    { 10011011, {Q|BACK, Q|BACK, Q, 0, Q|TN, 0}},   // TWNW_Heptahedron5
    { 10011101, {Q|BACK, Q|BACK, Q|BACK, 0, Q|TN, 0}},   // TWSW_Heptahedron5
    { 10011111, {0, Q|BACK, 0, 0, Q|TN, 0}},   // TW_Heptahedron4
    { 10110000, {0, Q|PAIR|TN, 0, Q|PAIR|TN, 0, 0}},   // BNBW_Hexahedron5
    { 10110001, {Q|BACK, Q|BACK, Q, Q|TN, Q|BACK|TN, Q|BACK|TN}},   // BNW_Heptahedron6
    { 10110011, {Q|BACK, 0, Q, Q|TN, 0, Q|BACK|TN}},   // BNNW_Heptahedron5
    { 10111001, {Q|BACK, Q|BACK, Q, 0, Q|BACK|TN, 0}},   // BWNW_Heptahedron5
    { 10111011, {Q|BACK, 0, Q, 0, 0, 0}},   // NW_Heptahedron4
    { 11000000, {Q|PAIR, Q|PAIR, 0, Q|INNER|TN, 0, Q|INNER|TN}},   // BS_Pentahedron
    { 11000100, {Q|PAIR, 0, 0, 0, 0, Q|PAIR|TN}},   // BSSE_Hexahedron5
    { 11001000, {Q|PAIR, 0, 0, 0, 0, Q|PAIR|TN}},   // BSSW_Hexahedron5
    { 11001100, {Q|PAIR, 0, 0, 0, 0, Q|PAIR|TN}},   // S_Hexahedron4
    { 11001101, {Q|BACK, 0, Q|BACK, Q|BACK|TN, 0, Q|TN}},   // TSSW_Heptahedron5
    { 11001110, {Q, 0, Q|BACK, Q|BACK|TN, 0, Q|TN}},   // TSSE_Heptahedron5
    { 11001111, {0, 0, 0, Q|BACK|TN, 0, Q|TN}},   // TS_Heptahedron4
    { 11010000, {0, Q|PAIR|TN, 0, Q|PAIR|TN, 0, 0}},   // BSBW_Hexahedron5
    { 11011000, {Q|BACK, Q|BACK, Q|BACK, Q|BACK|TN, Q|BACK|TN, Q|BACK|TN}},   // BSW_Heptahedron6
    { 11011001, {Q|BACK, Q|BACK, Q|BACK, 0, Q|BACK|TN, 0}},   // BWSW_Heptahedron5
    { 11011100, {Q|BACK, 0, Q|BACK, Q|BACK|TN, 0, Q|BACK|TN}},   // BSSW_Heptahedron5
    { 11011101, {Q|BACK|NEG, 0, Q|BACK|NEG, 0, 0, 0}},   // SW_Heptahedron4
    { 11100000, {0, Q|PAIR|TN, 0, Q|PAIR|TN, 0, 0}},   // BSBE_Hexahedron5
    { 11100100, {Q, Q, Q|BACK, Q|BACK|TN, Q|BACK|TN, Q|BACK|TN}},   // BSE_Heptahedron6
    { 11100110, {Q, Q, Q|BACK, 0, Q|BACK|TN, 0}},   // BESE_Heptahedron5
    { 11101100, {Q, 0, Q|BACK, Q|BACK|TN, 0, Q|BACK|TN}},   // BSSE_Heptahedron5
    { 11101110, {Q|NEG, 0, Q|BACK, 0, 0, 0}},   // SE_Heptahedron4
    { 11110000, {0, Q|PAIR|TN, 0, Q|PAIR|TN, 0, 0}},   // B_Hexahedron4
    { 11110001, {0, Q|BACK, 0, Q|TN, Q|BACK|TN, Q|BACK|TN}},   // BNBW_Heptahedron5
    { 11110010, {0, Q, 0, Q|TN, Q|BACK|TN, Q|BACK|TN}},   // BNBE_Heptahedron5
    { 11110011, {0, 0, 0, Q|TN, 0, Q|BACK|TN}},   // BN_Heptahedron4
    { 11110100, {0, Q|TN, 0, Q|BACK|TN, Q|BACK|TN, Q|BACK|TN}},   // BSBE_Heptahedron5
    { 11110110, {0, Q, 0, 0, Q|BACK|TN, 0}},   // BE_Heptahedron4
    { 11111000, {0, Q|BACK, 0, Q|BACK|TN, Q|BACK|TN, Q|BACK|TN}},   // BSBW_Heptahedron5
    { 11111001, {0, Q|BACK, 0, 0, Q|BACK|TN, 0}},   // BW_Heptahedron4
    { 11111100, {0, 0, 0, Q|BACK|TN, 0, Q|BACK|TN}},   // BS_Heptahedron4
};
constexpr int kRowCount = (int)(sizeof(kRows) / sizeof(kRows[0]));
inline const uint8_t* find(int code)
{
    int lo = 0, hi = kRowCount - 1;
    while (lo <= hi) {
        const int mid = (lo + hi) / 2;
        if (kRows[mid].code == code) return kRows[mid].slot;
        if (kRows[mid].code < code) lo = mid + 1;
        else hi = mid - 1;
    }
    return nullptr;
}
// velocity component of each term (0 u, 1 v, 2 w), the face-area component
// it uses (delta_ib_max.x = S_xy, .y = S_xz, .z = S_yz) and the component of
// the inverse-distance array
__host__ __device__ constexpr int vel_of(int s) { return s >> 1; }
__host__ __device__ constexpr int area_of(int s) { return s == 0 || s == 5 ? 1 : (s == 2 || s == 4 ? 2 : 0); }
__host__ __device__ constexpr int dist_of(int s) { return s == 0 || s == 5 ? 1 : (s == 1 || s == 3 ? 2 : 0); }
}  // namespace loads_desc

// packed per-cut-cell geometry, structure of arrays: field f of cell i at
// g[f * count + i]
enum LoadsField : int {
    LF_TX = 0, LF_TY, LF_TZ,      // theta at the cell
    LF_TXX, LF_TYY, LF_TZZ,       // theta.x at i-1, theta.y at j-1, theta.z at k-1
    LF_DX, LF_DY, LF_DZ,          // delta
    LF_VV,                        // 1 / VOF of the base cell
    LF_S0, LF_S1, LF_S2,          // delta_ib_max (S_xy, S_xz, S_yz)
    LF_D = 13,                    // 12 values: per term, inverse distance at the cell, then behind
    LF_NX = 25, LF_NY, LF_NZ,     // node coordinates (moment arm)
    LF_COUNT = 28
};

struct LoadsArgs {
    int count, N, NM;
    const double* g;              // LF_COUNT * count
    const int* idx;               // 3 * count: num, numX, numY
    const unsigned long long* desc;   // 6 descriptor bytes per cell
    const double* ux;
    const double* uy;
    const double* uz;
    const double* p;
    const double* vib;            // 3n, xyz interleaved
    const double* vyx;
    const double* vzy;
    const double* nu_cell;        // n or null
    double nu;
    double cx, cy, cz;            // moment centre
    double* fx;                   // per-cell forces or null
    double* fy;
    double* fz;
    double* partial;
    unsigned int* counter;
    double* sums;                 // 6: Fx Fy Fz Mz Mx My
};

__device__ __forceinline__ double l_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double l_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double l_sub(double a, double b) { return __dsub_rn(a, b); }

// one shear term (the "quad" expressions of loads_calculator.h:127-1263)
__device__ __forceinline__ double loads_term(unsigned b, double S, double vh, double uh, double dh, double vb,
                                             double ub, double db)
{
    using namespace loads_desc;
    if (!(b & Q)) return 0.0;
    const double s = (b & NEG) ? -S : S;
    if (b & PAIR) return l_mul(s, l_add(l_mul(l_sub(vb, ub), db), l_mul(l_sub(vh, uh), dh)));
    const bool back = (b & BACK) != 0;
    const double v = back ? vb : vh, u = back ? ub : uh, d = back ? db : dh;
    return (b & INNER) ? l_mul(s, l_mul(l_sub(v, u), d)) : l_mul(l_mul(s, l_sub(v, u)), d);
}

// LoadsCalculator::calc + calcMoment/X/Y + the sums of calculate()
__global__ void __launch_bounds__(256) k_loads(LoadsArgs a)
{
    using namespace loads_desc;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    const int cnt = a.count;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        const double* g = a.g + i;
#define G(f) __ldg(g + (size_t)(f) * cnt)
        const int num = a.idx[i], numX = a.idx[cnt + i], numY = a.idx[2 * cnt + i];
        const unsigned long long ds = a.desc[i];
        const double nu = a.nu_cell ? a.nu_cell[num] : a.nu;
        const double tx = G(LF_TX), ty = G(LF_TY), tz = G(LF_TZ);
        const double txx = G(LF_TXX), tyy = G(LF_TYY), tzz = G(LF_TZZ);
        const double dx = G(LF_DX), dy = G(LF_DY), dz = G(LF_DZ), VV = G(LF_VV);
        const double u0 = a.ux[numX], u1 = a.ux[numX - 1];
        const double v0 = a.uy[numY], v1 = a.uy[numY - a.N];
        const double w0 = a.uz[num], w1 = a.uz[num - a.NM];
        const double P = a.p[num];
        const double* vib = a.vib + 3 * (size_t)num;
        const double nx = l_sub(txx, tx), ny = l_sub(tyy, ty), nz = l_sub(tzz, tz);
        const double ax = l_mul(dy, dz), ay = l_mul(dx, dz), az = l_mul(dx, dy);
        const double dux = l_mul(l_mul(l_add(l_sub(l_mul(tx, u0), l_mul(txx, u1)), l_mul(nx, vib[0])), VV), ax);
        const double dvy = l_mul(l_mul(l_add(l_sub(l_mul(ty, v0), l_mul(tyy, v1)), l_mul(ny, vib[1])), VV), ay);
        const double dwz = l_mul(l_mul(l_add(l_sub(l_mul(tz, w0), l_mul(tzz, w1)), l_mul(nz, vib[2])), VV), az);
        const double bx = l_mul(l_mul(nx, ax), l_sub(P, l_mul(nu, dux)));
        const double by = l_mul(l_mul(ny, ay), l_sub(P, l_mul(nu, dvy)));
        const double bz = l_mul(l_mul(nz, az), l_sub(P, l_mul(nu, dwz)));
        double q[6];
        const int step[3] = {1, a.N, a.NM};
        const double uh[3] = {u0, v0, w0}, ub[3] = {u1, v1, w1};
#pragma unroll
        for (int s = 0; s < 6; s++) {
            const unsigned b = (unsigned)(ds >> (8 * s)) & 0xffu;
            if (!(b & Q)) { q[s] = 0.0; continue; }
            const int c = vel_of(s);
            const double* V = (s & 1) ? a.vzy : a.vyx;      // uy vx wx: v_ib_yx; uz vz wy: v_ib_zy
            const double vh = V[3 * (size_t)num + c];
            const double vb = V[3 * (size_t)(num - step[c]) + c];
            q[s] = loads_term(b, G(LF_S0 + area_of(s)), vh, uh[c], G(LF_D + 2 * s), vb, ub[c], G(LF_D + 2 * s + 1));
        }
        const double Fx = l_sub(bx, l_mul(nu, l_add(q[0], q[1])));
        const double Fy = l_sub(by, l_mul(nu, l_add(q[2], q[3])));
        const double Fz = l_sub(bz, l_mul(nu, l_add(q[4], q[5])));
        if (a.fx) { a.fx[i] = Fx; a.fy[i] = Fy; a.fz[i] = Fz; }
        const double rx = l_sub(G(LF_NX), a.cx), ry = l_sub(G(LF_NY), a.cy), rz = l_sub(G(LF_NZ), a.cz);
#undef G
        acc[0] += Fx;
        acc[1] += Fy;
        acc[2] += Fz;
        acc[3] += l_sub(l_mul(rx, Fy), l_mul(ry, Fx));      // M_z (calcMoment)
        acc[4] += l_sub(l_mul(ry, Fz), l_mul(rz, Fy));      // M_x (calcMomentX)
        acc[5] += l_sub(l_mul(rz, Fx), l_mul(rx, Fz));      // M_y (calcMomentY)
    }
    grid_reduce<6>(acc, a.partial, a.counter, a.sums);
}

// Gradient of J = w . (sum Fx, sum Fy, sum Fz) with respect to the pressure
// and the three velocity fields.  The forces are affine in those fields, so
// the gradient depends on the geometry, nu and w only.  Contributions of
// neighbouring cut cells to one unknown are added with atomics (the order of
// those few additions is not fixed).
struct LoadsAdjArgs {
    int count, N, NM;
    const double* g;
    const int* idx;
    const unsigned long long* desc;
    const double* nu_cell;
    double nu;
    double w[3];
    double* gux;
    double* guy;
    double* guz;
    double* gp;
};

__global__ void __launch_bounds__(256) k_loads_adjoint(LoadsAdjArgs a)
{
    using namespace loads_desc;
    const int cnt = a.count;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        const double* g = a.g + i;
#define G(f) g[(size_t)(f) * cnt]
        const int num = a.idx[i], numX = a.idx[cnt + i], numY = a.idx[2 * cnt + i];
        const unsigned long long ds = a.desc[i];
        const double nu = a.nu_cell ? a.nu_cell[num] : a.nu;
        const double t[3] = {G(LF_TX), G(LF_TY), G(LF_TZ)};
        const double tb[3] = {G(LF_TXX), G(LF_TYY), G(LF_TZZ)};
        const double dx = G(LF_DX), dy = G(LF_DY), dz = G(LF_DZ), VV = G(LF_VV);
        const double area[3] = {dy * dz, dx * dz, dx * dy};
        double* gu[3] = {a.gux, a.guy, a.guz};
        const int ih[3] = {numX, numY, num};
        const int stepU[3] = {1, a.N, a.NM};
        double gp = 0.0;
        for (int c = 0; c < 3; c++) {
            // F_c = n A (P - nu (t u_h - tb u_b + n vib) VV A) - nu (q + q')
            const double nA = (tb[c] - t[c]) * area[c];
            gp += a.w[c] * nA;
            const double k = a.w[c] * nA * nu * VV * area[c];
            double gh = -k * t[c], gb = k * tb[c];
            for (int s = 2 * c; s < 2 * c + 2; s++) {
                const unsigned b = (unsigned)(ds >> (8 * s)) & 0xffu;
                if (!(b & Q)) continue;
                const double S = ((b & NEG) ? -1.0 : 1.0) * G(LF_S0 + area_of(s)) * a.w[c] * nu;
                // -nu dq/du = nu S d per product
                if (b & PAIR) {
                    gh += S * G(LF_D + 2 * s);
                    gb += S * G(LF_D + 2 * s + 1);
                } else if (b & BACK) {
                    gb += S * G(LF_D + 2 * s + 1);
                } else {
                    gh += S * G(LF_D + 2 * s);
                }
            }
            atomicAdd(gu[c] + ih[c], gh);
            atomicAdd(gu[c] + ih[c] - stepU[c], gb);
        }
        atomicAdd(a.gp + num, gp);
#undef G
    }
}

// ---------------------------------------------------------------------------
// moment filter (ButterworthLowPassFilter, Base/butterworth_low_pass_filter.h:
// a second-order recursive low-pass filter whose coefficients follow from the
// time step, a cut-off frequency (5) and a suppression level (3 dB); a sample
// that jumps by more than 10 from a previous one above 1e-5 in magnitude is
// replaced by the previous sample)
// ---------------------------------------------------------------------------
struct LoadsFilter {
    double b0 = 0, b1 = 0, b2 = 0, a0 = 0, a1 = 0;
    double x1 = 0, x2 = 0, y1 = 0, y2 = 0;       // previous inputs / outputs
    void init(double dt, double cutoff = 5.0, double suppression = 3.0)
    {
        const double pi = 3.14159265358979323846;
        const double r = pow(10.0, -0.025 * suppression);      // amplitude at the cut-off, square root
        const double r2 = r * r;
        const double xi = pow(1 - r2 * r2, 0.25) / (r * tan(dt * cutoff * pi));
        const double xi2 = xi * xi;
        const double c = 1.0 + xi2, s = xi * 1.4142135623730951;
        const double g = 1.0 / (c + s);
        b0 = b2 = g;
        a1 = (c - s) * g;
        b1 = 2.0 * g;
        a0 = b1 * (1.0 - xi2);
        x1 = x2 = y1 = y2 = 0;
    }
    double step(double v)
    {
        if (fabs(v - x1) > 10.0 && fabs(x1) > 1e-5) v = x1;
        const double y = b0 * v + b1 * x1 + b2 * x2 - (a0 * y1 + a1 * y2);
        y2 = y1;
        y1 = y;
        x2 = x1;
        x1 = v;
        return y;
    }
};

}  // namespace lsg
