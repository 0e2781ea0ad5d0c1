// Mesh build of the flow task on the GPU: level set -> edge fractions alpha
// -> face and cell types -> face fractions theta -> cell volumes -> staggered
// types, volumes and inverse volumes.
//
// Restates, for a uniform grid, the reference's flow-task mesh build
// (BaseTaskDescription::buildMesh, base_task_description.h:330-371):
//   level set            FlowSphereTaskDescription::calcLevelSetSphere
//                        (flow_sphere_task_description.h:57-74), several
//                        bodies merged by max (phi > 0 inside);
//   alpha                FlowTaskDescription::calcAlpha (flow_task_description.h:102-136)
//                        with BuildAlpha / bottomBuildAlpha / topBuildAlpha and
//                        the in-place oscillation fix checkOscLS
//                        (ls_stag_uniform_mesh.h:2906-2963);
//   types                calcTypeOfCells (flow_task_description.h:175-230) with
//                        TypeOfSide / TypeOfCell / bottom- / topTypeOfCell
//                        (ls_stag_uniform_mesh.h:2969-2977, :3624-3675);
//   theta                calcTheta (flow_task_description.h:138-173) with
//                        getThetaZ / BuildTheta / tbBuildTheta (:1652-1837);
//   volumes              kernel v (:1838-2714), inverse (ls_stag_base_mesh_params.h:77-85);
//   staggered grids      cvu / cvv / cvw (:108-136), mx / my / mz (:2804-2826).
//
// Everything is FP64 and bit-identical to the reference: every sum and
// product is written as an explicit IEEE operation in the reference's order
// (no contraction into fused multiply-adds).  The per-cell functions are
// __host__ __device__ so that the same code also runs on the host.
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#define LSG_MHD __host__ __device__ __forceinline__
#else
#define LSG_MHD inline
#include <cmath>
#endif

namespace lsg {
namespace mesh {

constexpr double kEq = 1e-5;            // EQ_DOUBLE (ls_stag_real_constants.h:28)
constexpr double kThetaZero = 0.05;     // THETA_EQ_ZERO
constexpr double kTiny = 1e-12;         // EQ_TINY_DOUBLE
constexpr double kPlusTiny = 1e-16;     // PLUS_TINY
constexpr double kThird = 1.0 / 3.0;    // ONE_THIRD

// side types (cut_sides.h:27-44): one decimal digit per face corner, 1 = fluid
constexpr int kSolidSide = 0, kFluidSide = 1111;
// cell types (cut_cells.h:26-168): cut cells carry the codes of their top and
// bottom faces (top * 10000 + bottom); the box's borders are negative
constexpr int kSolid = 0, kFluid = 11111111;
enum BoxType {
    T_Border = -2, B_Border = -3, N_Border = -4, S_Border = -5, E_Border = -6, W_Border = -7,
    TN_Edge = -8, TS_Edge = -9, TE_Edge = -10, TW_Edge = -11, BN_Edge = -12, BS_Edge = -13,
    BE_Edge = -14, BW_Edge = -15, NE_Edge = -16, NW_Edge = -17, SE_Edge = -18, SW_Edge = -19,
    TNE_Corner = -20, TNW_Corner = -21, TSE_Corner = -22, TSW_Corner = -23,
    BNE_Corner = -24, BNW_Corner = -25, BSE_Corner = -26, BSW_Corner = -27
};

// ---------------------------------------------------------------------------
// IEEE operations in the written order
// ---------------------------------------------------------------------------
LSG_MHD double add(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
LSG_MHD double sub(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
LSG_MHD double mul(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
LSG_MHD double dvd(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __ddiv_rn(a, b);
#else
    return a / b;
#endif
}
LSG_MHD double sqr_root(double a)
{
#ifdef __CUDA_ARCH__
    return __dsqrt_rn(a);
#else
    return std::sqrt(a);
#endif
}

// ---------------------------------------------------------------------------
// level set
// ---------------------------------------------------------------------------
// A body record of kBodyWords doubles: kind (0 sphere, 1 ellipsoid), centre
// (3), sphere radius, ellipsoid semi-axes (3), ellipsoid rotation (3x3, row
// major; body frame = R (x - c)).
constexpr int kBodyWords = 17;

// phi of one body at point (x, y, z), > 0 inside.  Sphere: the reference's
// rad - |x - c| (calcLevelSetSphere).  Ellipsoid: (1 - s) min(a), with s the
// ellipsoid norm of the point in the body frame (zero on the surface, > 0
// inside, scaled like a distance near the surface).
LSG_MHD double body_phi(const double* b, double x, double y, double z)
{
    const double qx = sub(x, b[1]), qy = sub(y, b[2]), qz = sub(z, b[3]);
    if (b[0] == 0.0) return sub(b[4], sqr_root(add(add(mul(qx, qx), mul(qy, qy)), mul(qz, qz))));
    const double* R = b + 8;
    const double bx = add(add(mul(R[0], qx), mul(R[1], qy)), mul(R[2], qz));
    const double by = add(add(mul(R[3], qx), mul(R[4], qy)), mul(R[5], qz));
    const double bz = add(add(mul(R[6], qx), mul(R[7], qy)), mul(R[8], qz));
    const double ux = dvd(bx, b[5]), uy = dvd(by, b[6]), uz = dvd(bz, b[7]);
    const double s = sqr_root(add(add(mul(ux, ux), mul(uy, uy)), mul(uz, uz)));
    const double a01 = (b[6] < b[5]) ? b[6] : b[5];
    const double amin = (b[7] < a01) ? b[7] : a01;
    return mul(sub(1.0, s), amin);
}

// One x-row of the level-set block: phi at the upper cell corners, the
// reference's point walk (corner = node + delta / 2 at the first cell, then
// x += delta.x cell by cell; node = (i + 1/2) h).
LSG_MHD void levelset_row(int j, int k, int N, int M, int hs, int hf, const double h[3], int nb, const double* bodies,
                          double* phi)
{
    const long long row = (long long)N * j + (long long)N * M * k;
    double x = add(mul((double)hs + 0.5, h[0]), 0.0);
    x = add(x, mul(0.5, h[0]));
    const double y = add(add(mul((double)j + 0.5, h[1]), 0.0), mul(0.5, h[1]));
    const double z = add(add(mul((double)k + 0.5, h[2]), 0.0), mul(0.5, h[2]));
    for (int i = hs; i < hf; i++) {
        double f = -1e300;
        for (int q = 0; q < nb; q++) {
            const double v = body_phi(bodies + q * kBodyWords, x, y, z);
            f = (f < v) ? v : f;           // std::max(f, v)
        }
        phi[row + i] = f;
        x = add(x, h[0]);
    }
}

// ---------------------------------------------------------------------------
// oscillation fix and edge fractions
// ---------------------------------------------------------------------------
// The reference walks the block cell by cell (x fastest, then y, then z) and
// replaces, in place, a corner value f > EQ whose two neighbours along an
// axis are both negative by their mean (checkOscLS).  The walk reads the
// already-walked neighbours (-x, -y, -z) after their own fix and the
// forward ones (+x, +y, +z) before theirs.  cur holds the walked values
// (initially phi0); the function returns the fixed value of cell c given
// them, so iterating it to a fixed point over the block reproduces the walk.
LSG_MHD double osc_fixed(long long c, bool zcheck, long long N, long long NM, const double* phi0, const double* cur)
{
    double f = phi0[c];
    const double fw = cur[c - 1], fs = cur[c - N];
    if (f > kEq && fw < 0 && phi0[c + 1] < 0) f = mul(0.5, add(fw, phi0[c + 1]));
    if (f > kEq && fs < 0 && phi0[c + N] < 0) f = mul(0.5, add(fs, phi0[c + N]));
    if (zcheck) {
        const double fb = cur[c - NM];
        if (f > kEq && fb < 0 && phi0[c + NM] < 0) f = mul(0.5, add(fb, phi0[c + NM]));
    }
    return f;
}

// linear zero crossing of phi between the corner and its neighbour corner
LSG_MHD double edge_fraction(double f, double fn)
{
    if (mul(f, fn) < 0) return (f > 0) ? dvd(fn, sub(fn, f)) : dvd(f, sub(f, fn));
    return (f > -fn) ? 0.0 : 1.0;
}

// alpha of a block cell from the fixed level set (BuildAlpha; the bottom and
// top layers have no z neighbour: alpha.z = 0 inside the body, 1 outside)
LSG_MHD void alpha_cell(long long c, int k, int K, long long N, long long NM, const double* phi, double* alpha)
{
    const double f = phi[c];
    alpha[3 * c] = edge_fraction(f, phi[c - 1]);
    alpha[3 * c + 1] = edge_fraction(f, phi[c - N]);
    alpha[3 * c + 2] = (k > 0 && k < K - 1) ? edge_fraction(f, phi[c - NM]) : ((f > 0.0) ? 0.0 : 1.0);
}

// ---------------------------------------------------------------------------
// face and cell types
// ---------------------------------------------------------------------------
LSG_MHD int side_type(double p, double pw, double psw, double ps)
{
    int t = (ps < kEq) ? 1 : 0;
    if (psw < kEq) t += 10;
    if (pw < kEq) t += 100;
    if (p < kEq) t += 1000;
    return t;
}

// the box classification of a cell that is not a cut cell (calcTypeOfCells'
// walks outside the level-set block, calcTypeOfCellBaseBox's layout)
LSG_MHD int box_type(int i, int j, int k, int N, int M, int K)
{
    const int ix = (i == 0) ? 0 : ((i == N - 1) ? 2 : 1);
    const int iy = (j == 0) ? 0 : ((j == M - 1) ? 2 : 1);
    const int iz = (k == 0) ? 0 : ((k == K - 1) ? 2 : 1);
    // rows (south, middle, north) x columns (west, middle, east) of each layer
    if (iz == 0) {
        if (iy == 0) return ix == 0 ? BSW_Corner : (ix == 1 ? BS_Edge : BSE_Corner);
        if (iy == 1) return ix == 0 ? BW_Edge : (ix == 1 ? B_Border : BE_Edge);
        return ix == 0 ? BNW_Corner : (ix == 1 ? BN_Edge : BNE_Corner);
    }
    if (iz == 1) {
        if (iy == 0) return ix == 0 ? SW_Edge : (ix == 1 ? S_Border : SE_Edge);
        if (iy == 1) return ix == 0 ? W_Border : (ix == 1 ? kFluid : E_Border);
        return ix == 0 ? NW_Edge : (ix == 1 ? N_Border : NE_Edge);
    }
    if (iy == 0) return ix == 0 ? TSW_Corner : (ix == 1 ? TS_Edge : TSE_Corner);
    if (iy == 1) return ix == 0 ? TW_Edge : (ix == 1 ? T_Border : TE_Edge);
    return ix == 0 ? TNW_Corner : (ix == 1 ? TN_Edge : TNE_Corner);
}

// types of a block cell from the fixed level set: side types (east, north,
// top faces) and the cell type (TypeOfCell; bottom- / topTypeOfCell on the
// first and last layer, where the missing layer repeats the cell's own)
LSG_MHD void types_cell(long long c, int k, int K, long long N, long long NM, const double* phi, int* side, int* type)
{
    const double p = phi[c], pw = phi[c - 1], ps = phi[c - N], psw = phi[c - N - 1];
    if (k == 0 || k == K - 1) {
        const int tt = side_type(p, pw, psw, ps);
        side[3 * c] = side_type(p, ps, ps, p);
        side[3 * c + 1] = side_type(p, pw, pw, p);
        side[3 * c + 2] = tt;
        type[c] = (tt == kSolidSide) ? kSolid : ((k == 0) ? (int)B_Border : (int)T_Border);
        return;
    }
    const double pb = phi[c - NM], psb = phi[c - N - NM], pbw = phi[c - NM - 1], pswb = phi[c - N - 1 - NM];
    const int tt = side_type(p, pw, psw, ps);
    side[3 * c] = side_type(p, ps, psb, pb);
    side[3 * c + 1] = side_type(p, pw, pbw, pb);
    side[3 * c + 2] = tt;
    type[c] = tt * 10000 + side_type(pb, pbw, pswb, psb);
}

// ---------------------------------------------------------------------------
// face fractions
// ---------------------------------------------------------------------------
// Fraction of a face of side type st from the edge fractions of its edges:
// p0, p1 along its first in-plane edge direction at this cell and one cell
// back, q0, q1 along the second (getThetaZ / BuildTheta: trapezoids, pentagons,
// triangles of the marching-squares shapes; 0 below THETA_EQ_ZERO)
LSG_MHD double face_fraction(int st, double p0, double p1, double q0, double q1)
{
    double t;
    switch (st) {
    case kFluidSide: return 1.0;
    case kSolidSide: return 0.0;
    case 11: case 1100: t = mul(0.5, add(p0, p1)); break;                          // N, S trapezoids
    case 1001: case 110: t = mul(0.5, add(q0, q1)); break;                         // W, E trapezoids
    case 1011: t = sub(1.0, mul(mul(0.5, sub(1.0, p1)), sub(1.0, q0))); break;    // NW pentagon
    case 111: t = sub(1.0, mul(mul(0.5, sub(1.0, p0)), sub(1.0, q0))); break;     // NE pentagon
    case 1101: t = sub(1.0, mul(mul(0.5, sub(1.0, p1)), sub(1.0, q1))); break;    // SW pentagon
    case 1110: t = sub(1.0, mul(mul(0.5, sub(1.0, p0)), sub(1.0, q1))); break;    // SE pentagon
    case 1: t = mul(mul(0.5, p0), q1); break;                                      // NW triangle
    case 10: t = mul(mul(0.5, p1), q1); break;                                     // NE triangle
    case 1000: t = mul(mul(0.5, p0), q0); break;                                   // SW triangle
    case 100: t = mul(mul(0.5, p1), q0); break;                                    // SE triangle
    default: return 1.0;                                                           // ambiguous corner pattern
    }
    return (t < kThetaZero) ? 0.0 : t;
}

LSG_MHD void theta_cell(long long c, int k, int K, long long N, long long NM, const int* side, const double* alpha,
                        double* theta)
{
    const double* a = alpha + 3 * c;
    // top face: first direction alpha.y (this cell, x - 1), second alpha.x (this cell, y - 1)
    const double tz = face_fraction(side[3 * c + 2], a[1], a[1 - 3], a[0], a[-3 * N]);
    if (k == 0 || k == K - 1) {
        const double tx = a[1], ty = a[0];
        theta[3 * c] = (tx < kThetaZero) ? 0.0 : tx;
        theta[3 * c + 1] = (ty < kThetaZero) ? 0.0 : ty;
        theta[3 * c + 2] = tz;
        return;
    }
    // east face: alpha.z (this cell, y - 1), alpha.y (this cell, z - 1)
    theta[3 * c] = face_fraction(side[3 * c], a[2], a[2 - 3 * N], a[1], a[1 - 3 * NM]);
    // north face: alpha.z (this cell, x - 1), alpha.x (this cell, z - 1)
    theta[3 * c + 1] = face_fraction(side[3 * c + 1], a[2], a[2 - 3], a[0], a[-3 * NM]);
    theta[3 * c + 2] = tz;
}

// ---------------------------------------------------------------------------
// cell volumes (kernel v): one descriptor per cell type.  An operand byte is
// component (0..2) + 4 * back-offset mask (1: x - 1, 2: y - 1, 4: z - 1) of
// the alpha or theta array; the shapes and their operand orders follow the
// reference's volume formulas case by case.
// ---------------------------------------------------------------------------
enum VofKind : unsigned char {
    VOF_FULL = 0,     // fullV
    VOF_TBORDER,      // fullV * theta_z (bottom / top border cells)
    VOF_SOLID,        // 0
    VOF_TETRA,        // alpha[o0] * theta[o1] * fullV / 3
    VOF_HEPTA3,       // (3 - (1 - alpha[o0]) (1 - theta[o1])) * fullV / 3
    VOF_AVG,          // (theta[o0] + theta[o1]) * fullV / 2
    VOF_HEX5,         // pentagonal hexahedra: alpha[o0], theta[o1] scaled, alpha[o2], theta[o3]
    VOF_HEPTA5,       // pentagonal heptahedra: theta[o0], alpha[o1], alpha[o2], theta[o3]
    VOF_HEPTA6        // hexagonal heptahedra: theta[o0], two (alpha, alpha) pairs, theta[o5]
};
struct VofDesc {
    int code;
    unsigned char kind;
    unsigned char op[6];
};
constexpr int kVofRows = 106;
#define LSG_VOF_ROWS \
    { \
    {-3, VOF_TBORDER, {2, 0, 0, 0, 0, 0}},        {-2, VOF_TBORDER, {2, 0, 0, 0, 0, 0}}, \
    {0, VOF_SOLID, {0, 0, 0, 0, 0, 0}},           {1, VOF_TETRA, {24, 0, 0, 0, 0, 0}}, \
    {10, VOF_TETRA, {24, 4, 0, 0, 0, 0}},         {11, VOF_AVG, {0, 4, 0, 0, 0, 0}}, \
    {100, VOF_TETRA, {16, 4, 0, 0, 0, 0}},        {110, VOF_AVG, {1, 9, 0, 0, 0, 0}}, \
    {111, VOF_HEX5, {16, 1, 1, 9, 0, 0}},         {1000, VOF_TETRA, {16, 0, 0, 0, 0, 0}}, \
    {1001, VOF_AVG, {1, 9, 0, 0, 0, 0}},          {1011, VOF_HEX5, {16, 1, 5, 9, 0, 0}}, \
    {1100, VOF_AVG, {0, 4, 0, 0, 0, 0}},          {1101, VOF_HEX5, {24, 9, 5, 1, 0, 0}}, \
    {1110, VOF_HEX5, {24, 9, 1, 1, 0, 0}},        {1111, VOF_AVG, {0, 4, 0, 0, 0, 0}}, \
    {10000, VOF_TETRA, {8, 0, 0, 0, 0, 0}},       {10001, VOF_AVG, {2, 18, 0, 0, 0, 0}}, \
    {10011, VOF_HEX5, {14, 4, 8, 0, 0, 0}},       {11001, VOF_HEX5, {1, 2, 2, 18, 0, 0}}, \
    {11011, VOF_HEPTA6, {0, 2, 16, 1, 8, 4}},     {11111, VOF_HEPTA5, {9, 8, 5, 1, 0, 0}}, \
    {100000, VOF_TETRA, {8, 4, 0, 0, 0, 0}},      {100010, VOF_AVG, {2, 18, 0, 0, 0, 0}}, \
    {100011, VOF_HEX5, {10, 0, 8, 4, 0, 0}},      {100110, VOF_HEX5, {5, 2, 6, 18, 0, 0}}, \
    {100111, VOF_HEPTA6, {4, 6, 16, 5, 8, 0}},    {101111, VOF_HEPTA5, {9, 8, 1, 1, 0, 0}}, \
    {110000, VOF_AVG, {0, 4, 0, 0, 0, 0}},        {110001, VOF_HEX5, {14, 4, 24, 0, 0, 0}}, \
    {110010, VOF_HEX5, {10, 0, 24, 4, 0, 0}},     {110011, VOF_AVG, {0, 4, 0, 0, 0, 0}}, \
    {110111, VOF_HEPTA5, {4, 6, 16, 0, 0, 0}},    {111011, VOF_HEPTA5, {0, 2, 18, 4, 0, 0}}, \
    {111111, VOF_AVG, {0, 4, 0, 0, 0, 0}},        {1000000, VOF_TETRA, {0, 4, 0, 0, 0, 0}}, \
    {1000100, VOF_AVG, {2, 18, 0, 0, 0, 0}},      {1000110, VOF_HEX5, {5, 2, 14, 18, 0, 0}}, \
    {1001100, VOF_HEX5, {2, 0, 0, 4, 0, 0}},      {1001110, VOF_HEPTA6, {4, 14, 24, 5, 0, 0}}, \
    {1001111, VOF_HEPTA5, {1, 0, 5, 9, 0, 0}},    {1100000, VOF_AVG, {1, 9, 0, 0, 0, 0}}, \
    {1100010, VOF_HEX5, {21, 18, 6, 2, 0, 0}},    {1100100, VOF_HEX5, {21, 18, 14, 2, 0, 0}}, \
    {1100110, VOF_AVG, {1, 9, 0, 0, 0, 0}},       {1100111, VOF_HEPTA5, {18, 17, 10, 2, 0, 0}}, \
    {1101110, VOF_HEPTA5, {18, 17, 2, 2, 0, 0}},  {1101111, VOF_AVG, {1, 9, 0, 0, 0, 0}}, \
    {1110000, VOF_HEX5, {0, 1, 1, 9, 0, 0}},      {1110010, VOF_HEPTA6, {4, 6, 0, 21, 24, 0}}, \
    {1110011, VOF_HEPTA5, {4, 6, 0, 0, 0, 0}},    {1110110, VOF_HEPTA5, {2, 1, 10, 18, 0, 0}}, \
    {1110111, VOF_AVG, {2, 18, 0, 0, 0, 0}},      {1111111, VOF_HEPTA3, {0, 0, 0, 0, 0, 0}}, \
    {10000000, VOF_TETRA, {0, 0, 0, 0, 0, 0}},    {10001000, VOF_AVG, {2, 18, 0, 0, 0, 0}}, \
    {10001001, VOF_HEX5, {1, 2, 10, 18, 0, 0}},   {10001100, VOF_HEX5, {6, 4, 0, 0, 0, 0}}, \
    {10001101, VOF_HEPTA6, {0, 10, 24, 1, 0, 4}}, {10001111, VOF_HEPTA5, {1, 0, 1, 9, 0, 0}}, \
    {10010000, VOF_AVG, {1, 9, 0, 0, 0, 0}},      {10010001, VOF_HEX5, {17, 18, 2, 2, 0, 0}}, \
    {10011000, VOF_HEX5, {17, 18, 10, 2, 0, 0}},  {10011001, VOF_AVG, {1, 9, 0, 0, 0, 0}}, \
    {10011011, VOF_HEPTA5, {18, 21, 14, 2, 0, 0}}, {10011101, VOF_HEPTA5, {18, 21, 6, 2, 0, 0}}, \
    {10011111, VOF_AVG, {1, 9, 0, 0, 0, 0}},      {10110000, VOF_HEX5, {0, 1, 5, 9, 0, 0}}, \
    {10110001, VOF_HEPTA6, {0, 2, 0, 17, 24, 4}}, {10110011, VOF_HEPTA5, {0, 2, 0, 4, 0, 0}}, \
    {10111001, VOF_HEPTA5, {2, 5, 14, 18, 0, 0}}, {10111011, VOF_AVG, {2, 18, 0, 0, 0, 0}}, \
    {10111111, VOF_HEPTA3, {0, 4, 0, 0, 0, 0}},   {11000000, VOF_AVG, {0, 4, 0, 0, 0, 0}}, \
    {11000100, VOF_HEX5, {2, 0, 16, 4, 0, 0}},    {11001000, VOF_HEX5, {6, 4, 16, 0, 0, 0}}, \
    {11001100, VOF_AVG, {0, 4, 0, 0, 0, 0}},      {11001101, VOF_HEPTA5, {0, 10, 24, 4, 0, 0}}, \
    {11001110, VOF_HEPTA5, {4, 14, 24, 0, 0, 0}}, {11001111, VOF_AVG, {0, 4, 0, 0, 0, 0}}, \
    {11010000, VOF_HEX5, {8, 9, 5, 1, 0, 0}},     {11011000, VOF_HEPTA6, {0, 10, 16, 17, 8, 4}}, \
    {11011001, VOF_HEPTA5, {2, 5, 6, 18, 0, 0}},  {11011100, VOF_HEPTA5, {0, 10, 8, 4, 0, 0}}, \
    {11011101, VOF_AVG, {2, 18, 0, 0, 0, 0}},     {11011111, VOF_HEPTA3, {8, 4, 0, 0, 0, 0}}, \
    {11100000, VOF_HEX5, {8, 9, 1, 1, 0, 0}},     {11100100, VOF_HEPTA6, {4, 14, 8, 21, 16, 0}}, \
    {11100110, VOF_HEPTA5, {2, 1, 2, 18, 0, 0}},  {11101100, VOF_HEPTA5, {4, 14, 8, 0, 0, 0}}, \
    {11101110, VOF_AVG, {2, 18, 0, 0, 0, 0}},     {11101111, VOF_HEPTA3, {8, 0, 0, 0, 0, 0}}, \
    {11110000, VOF_AVG, {0, 4, 0, 0, 0, 0}},      {11110001, VOF_HEPTA5, {9, 24, 17, 1, 0, 0}}, \
    {11110010, VOF_HEPTA5, {9, 24, 21, 1, 0, 0}}, {11110011, VOF_AVG, {0, 4, 0, 0, 0, 0}}, \
    {11110100, VOF_HEPTA5, {1, 16, 21, 9, 0, 0}}, {11110110, VOF_AVG, {1, 9, 0, 0, 0, 0}}, \
    {11110111, VOF_HEPTA3, {16, 0, 0, 0, 0, 0}},  {11111000, VOF_HEPTA5, {1, 16, 17, 9, 0, 0}}, \
    {11111001, VOF_AVG, {1, 9, 0, 0, 0, 0}},      {11111011, VOF_HEPTA3, {16, 4, 0, 0, 0, 0}}, \
    {11111100, VOF_AVG, {0, 4, 0, 0, 0, 0}},      {11111101, VOF_HEPTA3, {24, 4, 0, 0, 0, 0}}, \
    {11111110, VOF_HEPTA3, {24, 0, 0, 0, 0, 0}},  {11111111, VOF_FULL, {0, 0, 0, 0, 0, 0}}, \
    }
static const VofDesc kVofHost[kVofRows] = LSG_VOF_ROWS;
#ifdef __CUDACC__
__constant__ VofDesc kVofDev[kVofRows] = LSG_VOF_ROWS;
#endif
#undef LSG_VOF_ROWS

LSG_MHD const VofDesc* vof_table()
{
#ifdef __CUDA_ARCH__
    return kVofDev;
#else
    return kVofHost;
#endif
}

// the descriptor of a cell type, or nullptr (types without a formula keep the
// full volume: the fluid cell, the side and edge borders, the corners)
LSG_MHD const VofDesc* vof_desc(int code)
{
    const VofDesc* t = vof_table();
    int lo = 0, hi = kVofRows - 1;
    while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        if (t[mid].code == code) return t + mid;
        if (t[mid].code < code) lo = mid + 1;
        else hi = mid - 1;
    }
    return nullptr;
}

// value of operand byte o of a 3-component array at cell c
LSG_MHD double opnd(const double* a, long long c, unsigned char o, long long N, long long NM)
{
    const int m = o >> 2;
    const long long cc = c - ((m & 1) ? 1 : 0) - ((m & 2) ? N : 0) - ((m & 4) ? NM : 0);
    return a[3 * cc + (o & 3)];
}

// 1 - (1 + 2 b) c^2 / 3 with c = (1 - a) / a (pentagonal hexahedra)
LSG_MHD double hex5_factor(double a, double b)
{
    const double coef = dvd(sub(1.0, a), a);
    return sub(1.0, mul(mul(mul(add(1.0, mul(2.0, b)), coef), coef), kThird));
}

LSG_MHD double volume_cell(long long c, int type, long long N, long long NM, const double* delta, const double* theta,
                           const double* alpha)
{
    const double fullV = mul(mul(delta[3 * c], delta[3 * c + 1]), delta[3 * c + 2]);
    double vol = fullV;
    const VofDesc* d = vof_desc(type);
    if (d) {
        const unsigned char* o = d->op;
        switch (d->kind) {
        case VOF_TBORDER: vol = mul(vol, opnd(theta, c, o[0], N, NM)); break;
        case VOF_SOLID: vol = 0.0; break;
        case VOF_TETRA:
            vol = mul(mul(mul(opnd(alpha, c, o[0], N, NM), opnd(theta, c, o[1], N, NM)), fullV), kThird);
            break;
        case VOF_HEPTA3:
            vol = mul(mul(sub(3.0, mul(sub(1.0, opnd(alpha, c, o[0], N, NM)), sub(1.0, opnd(theta, c, o[1], N, NM)))),
                          fullV),
                      kThird);
            break;
        case VOF_AVG: vol = mul(mul(add(opnd(theta, c, o[0], N, NM), opnd(theta, c, o[1], N, NM)), fullV), 0.5); break;
        case VOF_HEX5: {
            const double den = opnd(alpha, c, o[0], N, NM);
            double t2 = opnd(theta, c, o[1], N, NM);
            if (den > kEq) t2 = mul(t2, hex5_factor(den, opnd(alpha, c, o[2], N, NM)));
            vol = mul(mul(add(opnd(theta, c, o[3], N, NM), t2), fullV), 0.5);
            break;
        }
        case VOF_HEPTA5: {
            const double tx = opnd(theta, c, o[0], N, NM);
            double a = opnd(alpha, c, o[1], N, NM);
            const double den = sub(1.0, a);
            double term = 0.0;
            if (den > kEq) {
                a = dvd(a, den);
                term = mul(mul(mul(mul(sub(1.0, tx), sub(3.0, mul(2.0, opnd(alpha, c, o[2], N, NM)))), a), a), kThird);
            }
            vol = mul(mul(add(add(opnd(theta, c, o[3], N, NM), tx), term), fullV), 0.5);
            break;
        }
        case VOF_HEPTA6: {
            const double tx = opnd(theta, c, o[0], N, NM);
            double term = 0.0;
            double a = opnd(alpha, c, o[1], N, NM);
            double den = sub(1.0, a);
            if (den > kEq) {
                a = dvd(a, den);
                term = mul(mul(sub(3.0, mul(2.0, opnd(alpha, c, o[2], N, NM))), a), a);
            }
            a = opnd(alpha, c, o[3], N, NM);
            den = sub(1.0, a);
            if (den > kEq) {
                a = dvd(a, den);
                term = add(term, mul(mul(sub(3.0, mul(2.0, opnd(alpha, c, o[4], N, NM))), a), a));
            }
            vol = mul(mul(add(add(opnd(theta, c, o[5], N, NM), tx), mul(mul(sub(1.0, tx), term), kThird)), fullV), 0.5);
            break;
        }
        default: break;
        }
    }
    return add(vol, kPlusTiny);
}

LSG_MHD double inverse_volume(double v) { return (v < kTiny) ? 0.0 : dvd(1.0, v); }

// staggered cell type between base cells c (west / south / bottom) and e
// (cvu / cvv / cvw): solid if the shared face is closed, else the smaller code
LSG_MHD int staggered_type(int tc, int te, double face_theta)
{
    return (face_theta < kEq) ? kSolid : ((te < tc) ? te : tc);
}

// ---------------------------------------------------------------------------
// immersed-boundary face areas (calcDeltaIB, ls_stag_uniform_mesh.h:186-1650):
// per cell five coordinate triples -- delta_ib_en, _ws, _nb, _st and _max,
// the areas of the cut surface seen from the east/north, west/south,
// north/bottom and south/top sides -- from theta and delta.  The reference
// writes one block of assignments per cell type (and, for the bottom and
// top border cells, per top-face side type); each block is restated here as a
// short program for a stack machine: push theta (component, back-offset mask
// 1 = x-1, 2 = y-1, 4 = z-1), push delta (component), push a constant, load or
// store a local, add / subtract / multiply / absolute value / negate in the
// block's own order, write one output component, or copy one output triple
// into another.  Types without a block keep their arrays untouched (0).
// ---------------------------------------------------------------------------
enum DibOp : unsigned char {
    DIB_END = 0, DIB_T, DIB_D, DIB_C, DIB_LD, DIB_ST, DIB_ADD, DIB_SUB, DIB_MUL, DIB_ABS, DIB_NEG, DIB_OUT, DIB_COPY
};
struct DibCase {
    int type;      // cell type
    int side_z;    // top-face side type (bottom / top border cells), else -1
    int at;        // offset of the program in the code blob
};
constexpr int kDibCases = 156;
constexpr int kDibCode = 13094;
#define LSG_DIB_TABLE { \
    {-27, -1, 0}, {-26, -1, 46}, {-25, -1, 92}, \
    {-24, -1, 138}, {-23, -1, 184}, {-22, -1, 230}, \
    {-21, -1, 276}, {-20, -1, 322}, {-19, -1, 368}, \
    {-18, -1, 406}, {-17, -1, 444}, {-16, -1, 482}, \
    {-15, -1, 520}, {-14, -1, 558}, {-13, -1, 596}, \
    {-12, -1, 634}, {-11, -1, 672}, {-10, -1, 710}, \
    {-9, -1, 748}, {-8, -1, 786}, {-7, -1, 824}, \
    {-6, -1, 854}, {-5, -1, 884}, {-4, -1, 914}, \
    {-3, 0, 944}, {-3, 1, 966}, {-3, 10, 1024}, \
    {-3, 11, 1082}, {-3, 100, 1142}, {-3, 110, 1200}, \
    {-3, 111, 1260}, {-3, 1000, 1354}, {-3, 1001, 1412}, \
    {-3, 1011, 1472}, {-3, 1100, 1576}, {-3, 1101, 1636}, \
    {-3, 1110, 1730}, {-3, 1111, 1834}, {-2, 0, 1856}, \
    {-2, 1, 1878}, {-2, 10, 1936}, {-2, 11, 1994}, \
    {-2, 100, 2054}, {-2, 110, 2112}, {-2, 111, 2172}, \
    {-2, 1000, 2266}, {-2, 1001, 2324}, {-2, 1011, 2384}, \
    {-2, 1100, 2488}, {-2, 1101, 2548}, {-2, 1110, 2642}, \
    {-2, 1111, 2746}, {0, -1, 2768}, {1, -1, 2814}, \
    {10, -1, 2884}, {11, -1, 2954}, {100, -1, 3042}, \
    {110, -1, 3112}, {111, -1, 3200}, {1000, -1, 3294}, \
    {1001, -1, 3364}, {1011, -1, 3452}, {1100, -1, 3546}, \
    {1101, -1, 3634}, {1110, -1, 3728}, {1111, -1, 3822}, \
    {10000, -1, 3912}, {10001, -1, 3982}, {10011, -1, 4070}, \
    {11001, -1, 4164}, {11011, -1, 4258}, {11111, -1, 4358}, \
    {100000, -1, 4456}, {100010, -1, 4526}, {100011, -1, 4614}, \
    {100110, -1, 4708}, {100111, -1, 4802}, {101111, -1, 4902}, \
    {110000, -1, 5000}, {110001, -1, 5088}, {110010, -1, 5182}, \
    {110011, -1, 5276}, {110111, -1, 5366}, {111011, -1, 5464}, \
    {111111, -1, 5562}, {1000000, -1, 5706}, {1000100, -1, 5776}, \
    {1000110, -1, 5864}, {1001100, -1, 5958}, {1001110, -1, 6052}, \
    {1001111, -1, 6152}, {1100000, -1, 6250}, {1100010, -1, 6338}, \
    {1100100, -1, 6432}, {1100110, -1, 6526}, {1100111, -1, 6616}, \
    {1101110, -1, 6714}, {1101111, -1, 6812}, {1110000, -1, 6956}, \
    {1110010, -1, 7050}, {1110011, -1, 7150}, {1110110, -1, 7248}, \
    {1110111, -1, 7346}, {1111111, -1, 7490}, {10000000, -1, 7612}, \
    {10001000, -1, 7682}, {10001001, -1, 7770}, {10001100, -1, 7864}, \
    {10001101, -1, 7958}, {10001111, -1, 8058}, {10010000, -1, 8156}, \
    {10010001, -1, 8244}, {10011000, -1, 8338}, {10011001, -1, 8432}, \
    {10011011, -1, 8522}, {10011101, -1, 8620}, {10011111, -1, 8718}, \
    {10110000, -1, 8862}, {10110001, -1, 8956}, {10110011, -1, 9056}, \
    {10111001, -1, 9154}, {10111011, -1, 9252}, {10111111, -1, 9396}, \
    {11000000, -1, 9518}, {11000100, -1, 9606}, {11001000, -1, 9700}, \
    {11001100, -1, 9794}, {11001101, -1, 9884}, {11001110, -1, 9982}, \
    {11001111, -1, 10080}, {11010000, -1, 10214}, {11011000, -1, 10308}, \
    {11011001, -1, 10408}, {11011100, -1, 10506}, {11011101, -1, 10604}, \
    {11011111, -1, 10738}, {11100000, -1, 10850}, {11100100, -1, 10944}, \
    {11100110, -1, 11044}, {11101100, -1, 11142}, {11101110, -1, 11240}, \
    {11101111, -1, 11384}, {11110000, -1, 11506}, {11110001, -1, 11596}, \
    {11110010, -1, 11694}, {11110011, -1, 11792}, {11110100, -1, 11926}, \
    {11110110, -1, 12024}, {11110111, -1, 12168}, {11111000, -1, 12280}, \
    {11111001, -1, 12378}, {11111011, -1, 12522}, {11111100, -1, 12644}, \
    {11111101, -1, 12788}, {11111110, -1, 12910}, {11111111, -1, 13032}, \
}
#define LSG_DIB_CODE { \
    3, 0, 2, 0, 8, 0, 2, 1, 8, 0, 11, 0, 3, 0, 2, 0, 8, 0, 2, 2, 8, 0, 11, 1, \
    3, 0, 2, 1, 8, 0, 2, 2, 8, 0, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 3, 0, \
    2, 0, 8, 0, 2, 1, 8, 0, 11, 0, 3, 0, 2, 0, 8, 0, 2, 2, 8, 0, 11, 1, 3, 0, \
    2, 1, 8, 0, 2, 2, 8, 0, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 3, 0, 2, 0, \
    8, 0, 2, 1, 8, 0, 11, 0, 3, 0, 2, 0, 8, 0, 2, 2, 8, 0, 11, 1, 3, 0, 2, 1, \
    8, 0, 2, 2, 8, 0, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 3, 0, 2, 0, 8, 0, \
    2, 1, 8, 0, 11, 0, 3, 0, 2, 0, 8, 0, 2, 2, 8, 0, 11, 1, 3, 0, 2, 1, 8, 0, \
    2, 2, 8, 0, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 3, 0, 2, 0, 8, 0, 2, 1, \
    8, 0, 11, 0, 3, 0, 2, 0, 8, 0, 2, 2, 8, 0, 11, 1, 3, 0, 2, 1, 8, 0, 2, 2, \
    8, 0, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 3, 0, 2, 0, 8, 0, 2, 1, 8, 0, \
    11, 0, 3, 0, 2, 0, 8, 0, 2, 2, 8, 0, 11, 1, 3, 0, 2, 1, 8, 0, 2, 2, 8, 0, \
    11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 3, 0, 2, 0, 8, 0, 2, 1, 8, 0, 11, 0, \
    3, 0, 2, 0, 8, 0, 2, 2, 8, 0, 11, 1, 3, 0, 2, 1, 8, 0, 2, 2, 8, 0, 11, 2, \
    12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 3, 0, 2, 0, 8, 0, 2, 1, 8, 0, 11, 0, 3, 0, \
    2, 0, 8, 0, 2, 2, 8, 0, 11, 1, 3, 0, 2, 1, 8, 0, 2, 2, 8, 0, 11, 2, 12, 8, \
    12, 16, 12, 24, 12, 32, 0, 0, 3, 1, 11, 0, 3, 0, 2, 0, 8, 0, 2, 2, 8, 0, 11, 1, \
    3, 0, 2, 1, 8, 0, 2, 2, 8, 0, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 3, 1, \
    11, 0, 3, 0, 2, 0, 8, 0, 2, 2, 8, 0, 11, 1, 3, 0, 2, 1, 8, 0, 2, 2, 8, 0, \
    11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 3, 1, 11, 0, 3, 0, 2, 0, 8, 0, 2, 2, \
    8, 0, 11, 1, 3, 0, 2, 1, 8, 0, 2, 2, 8, 0, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, \
    0, 0, 3, 1, 11, 0, 3, 0, 2, 0, 8, 0, 2, 2, 8, 0, 11, 1, 3, 0, 2, 1, 8, 0, \
    2, 2, 8, 0, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 3, 0, 2, 0, 8, 0, 2, 1, \
    8, 0, 11, 0, 3, 1, 11, 1, 3, 0, 2, 1, 8, 0, 2, 2, 8, 0, 11, 2, 12, 8, 12, 16, \
    12, 24, 12, 32, 0, 0, 3, 0, 2, 0, 8, 0, 2, 1, 8, 0, 11, 0, 3, 1, 11, 1, 3, 0, \
    2, 1, 8, 0, 2, 2, 8, 0, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 3, 0, 2, 0, \
    8, 0, 2, 1, 8, 0, 11, 0, 3, 0, 2, 0, 8, 0, 2, 2, 8, 0, 11, 1, 3, 1, 11, 2, \
    12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 3, 0, 2, 0, 8, 0, 2, 1, 8, 0, 11, 0, 3, 0, \
    2, 0, 8, 0, 2, 2, 8, 0, 11, 1, 3, 1, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, \
    3, 0, 2, 0, 8, 0, 2, 1, 8, 0, 11, 0, 3, 1, 11, 1, 3, 0, 2, 1, 8, 0, 2, 2, \
    8, 0, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 3, 0, 2, 0, 8, 0, 2, 1, 8, 0, \
    11, 0, 3, 1, 11, 1, 3, 0, 2, 1, 8, 0, 2, 2, 8, 0, 11, 2, 12, 8, 12, 16, 12, 24, \
    12, 32, 0, 0, 3, 0, 2, 0, 8, 0, 2, 1, 8, 0, 11, 0, 3, 0, 2, 0, 8, 0, 2, 2, \
    8, 0, 11, 1, 3, 1, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 3, 0, 2, 0, 8, 0, \
    2, 1, 8, 0, 11, 0, 3, 0, 2, 0, 8, 0, 2, 2, 8, 0, 11, 1, 3, 1, 11, 2, 12, 8, \
    12, 16, 12, 24, 12, 32, 0, 0, 3, 1, 11, 0, 3, 1, 11, 1, 3, 0, 2, 1, 8, 0, 2, 2, \
    8, 0, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 3, 1, 11, 0, 3, 1, 11, 1, 3, 0, \
    2, 1, 8, 0, 2, 2, 8, 0, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 3, 1, 11, 0, \
    3, 0, 2, 0, 8, 0, 2, 2, 8, 0, 11, 1, 3, 1, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, \
    0, 0, 3, 1, 11, 0, 3, 0, 2, 0, 8, 0, 2, 2, 8, 0, 11, 1, 3, 1, 11, 2, 12, 8, \
    12, 16, 12, 24, 12, 32, 0, 0, 3, 1, 11, 0, 3, 1, 11, 1, 3, 1, 11, 2, 12, 8, 12, 16, \
    12, 24, 12, 32, 0, 0, 2, 2, 5, 0, 3, 0, 1, 9, 8, 0, 2, 0, 8, 0, 4, 0, 8, 0, \
    5, 1, 3, 0, 1, 0, 8, 0, 2, 1, 8, 0, 4, 0, 8, 0, 5, 2, 3, 1, 11, 0, 4, 1, \
    11, 1, 4, 2, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 2, 5, 0, 3, 0, 1, 9, \
    8, 0, 2, 0, 8, 0, 4, 0, 8, 0, 5, 1, 3, 0, 1, 4, 8, 0, 2, 1, 8, 0, 4, 0, \
    8, 0, 5, 2, 3, 1, 11, 0, 4, 1, 11, 1, 4, 2, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, \
    0, 0, 2, 2, 5, 0, 3, 0, 2, 0, 8, 0, 4, 0, 8, 0, 5, 1, 3, 0, 1, 4, 1, 0, \
    7, 0, 9, 0, 8, 0, 2, 1, 8, 0, 4, 0, 8, 0, 5, 2, 3, 1, 11, 0, 4, 1, 11, 1, \
    4, 2, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 2, 5, 0, 3, 0, 1, 1, 8, 0, \
    2, 0, 8, 0, 4, 0, 8, 0, 5, 1, 3, 0, 1, 4, 8, 0, 2, 1, 8, 0, 4, 0, 8, 0, \
    5, 2, 3, 1, 11, 0, 4, 1, 11, 1, 4, 2, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, \
    2, 2, 5, 0, 3, 0, 1, 9, 1, 1, 7, 0, 9, 0, 8, 0, 2, 0, 8, 0, 4, 0, 8, 0, \
    5, 1, 3, 0, 2, 1, 8, 0, 4, 0, 8, 0, 5, 2, 3, 1, 11, 0, 4, 1, 11, 1, 4, 2, \
    11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 2, 5, 0, 3, 2, 1, 1, 7, 0, 2, 0, \
    8, 0, 4, 0, 8, 0, 5, 1, 3, 0, 4, 1, 8, 0, 5, 2, 3, 2, 1, 0, 7, 0, 2, 1, \
    8, 0, 4, 0, 8, 0, 5, 3, 3, 0, 4, 3, 8, 0, 5, 4, 3, 1, 11, 0, 4, 1, 11, 1, \
    4, 3, 11, 2, 3, 1, 11, 3, 3, 1, 11, 4, 3, 1, 11, 5, 3, 1, 11, 6, 4, 2, 11, 7, \
    4, 4, 11, 8, 12, 26, 12, 32, 0, 0, 2, 2, 5, 0, 3, 0, 1, 1, 8, 0, 2, 0, 8, 0, \
    4, 0, 8, 0, 5, 1, 3, 0, 1, 0, 8, 0, 2, 1, 8, 0, 4, 0, 8, 0, 5, 2, 3, 1, \
    11, 0, 4, 1, 11, 1, 4, 2, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 2, 5, 0, \
    3, 0, 1, 9, 1, 1, 7, 0, 9, 0, 8, 0, 2, 0, 8, 0, 4, 0, 8, 0, 5, 1, 3, 0, \
    2, 1, 8, 0, 4, 0, 8, 0, 5, 2, 3, 1, 11, 0, 4, 1, 11, 1, 4, 2, 11, 2, 12, 8, \
    12, 16, 12, 24, 12, 32, 0, 0, 2, 2, 5, 0, 3, 2, 1, 1, 7, 0, 2, 0, 8, 0, 4, 0, \
    8, 0, 5, 1, 3, 0, 4, 1, 8, 0, 5, 2, 3, 2, 1, 4, 7, 0, 2, 1, 8, 0, 4, 0, \
    8, 0, 5, 3, 3, 0, 4, 3, 8, 0, 5, 4, 3, 1, 11, 0, 3, 1, 11, 1, 4, 3, 11, 2, \
    3, 1, 11, 3, 4, 1, 11, 4, 3, 1, 11, 5, 3, 1, 11, 6, 4, 2, 11, 7, 4, 4, 11, 8, \
    12, 26, 3, 1, 11, 12, 4, 1, 11, 13, 4, 3, 11, 14, 0, 0, 2, 2, 5, 0, 3, 0, 2, 0, \
    8, 0, 4, 0, 8, 0, 5, 1, 3, 0, 1, 4, 1, 0, 7, 0, 9, 0, 8, 0, 2, 1, 8, 0, \
    4, 0, 8, 0, 5, 2, 3, 1, 11, 0, 4, 1, 11, 1, 4, 2, 11, 2, 12, 8, 12, 16, 12, 24, \
    12, 32, 0, 0, 2, 2, 5, 0, 3, 2, 1, 9, 7, 0, 2, 0, 8, 0, 4, 0, 8, 0, 5, 1, \
    3, 0, 4, 1, 8, 0, 5, 2, 3, 2, 1, 4, 7, 0, 2, 1, 8, 0, 4, 0, 8, 0, 5, 3, \
    3, 0, 4, 3, 8, 0, 5, 4, 3, 1, 11, 0, 3, 1, 11, 1, 3, 1, 11, 2, 3, 1, 11, 3, \
    4, 1, 11, 4, 4, 3, 11, 5, 3, 1, 11, 6, 4, 2, 11, 7, 4, 4, 11, 8, 12, 26, 12, 33, \
    0, 0, 2, 2, 5, 0, 3, 2, 1, 9, 7, 0, 2, 0, 8, 0, 4, 0, 8, 0, 5, 1, 3, 0, \
    4, 1, 8, 0, 5, 2, 3, 2, 1, 0, 7, 0, 2, 1, 8, 0, 4, 0, 8, 0, 5, 3, 3, 0, \
    4, 3, 8, 0, 5, 4, 3, 1, 11, 0, 4, 1, 11, 1, 3, 1, 11, 2, 3, 1, 11, 3, 3, 1, \
    11, 4, 4, 3, 11, 5, 3, 1, 11, 6, 4, 2, 11, 7, 4, 4, 11, 8, 12, 26, 3, 1, 11, 12, \
    4, 1, 11, 13, 4, 3, 11, 14, 0, 0, 3, 1, 11, 0, 3, 1, 11, 1, 3, 1, 11, 2, 12, 8, \
    12, 16, 12, 24, 12, 32, 0, 0, 3, 1, 11, 0, 3, 1, 11, 1, 3, 1, 11, 2, 12, 8, 12, 16, \
    12, 24, 12, 32, 0, 0, 2, 2, 5, 0, 3, 0, 1, 9, 8, 0, 2, 0, 8, 0, 4, 0, 8, 0, \
    5, 1, 3, 0, 1, 0, 8, 0, 2, 1, 8, 0, 4, 0, 8, 0, 5, 2, 3, 1, 11, 0, 4, 1, \
    11, 1, 4, 2, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 2, 5, 0, 3, 0, 1, 9, \
    8, 0, 2, 0, 8, 0, 4, 0, 8, 0, 5, 1, 3, 0, 1, 4, 8, 0, 2, 1, 8, 0, 4, 0, \
    8, 0, 5, 2, 3, 1, 11, 0, 4, 1, 11, 1, 4, 2, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, \
    0, 0, 2, 2, 5, 0, 3, 0, 2, 0, 8, 0, 4, 0, 8, 0, 5, 1, 3, 0, 1, 4, 1, 0, \
    7, 0, 9, 0, 8, 0, 2, 1, 8, 0, 4, 0, 8, 0, 5, 2, 3, 1, 11, 0, 4, 1, 11, 1, \
    4, 2, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 2, 5, 0, 3, 0, 1, 1, 8, 0, \
    2, 0, 8, 0, 4, 0, 8, 0, 5, 1, 3, 0, 1, 4, 8, 0, 2, 1, 8, 0, 4, 0, 8, 0, \
    5, 2, 3, 1, 11, 0, 4, 1, 11, 1, 4, 2, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, \
    2, 2, 5, 0, 3, 0, 1, 9, 1, 1, 7, 0, 9, 0, 8, 0, 2, 0, 8, 0, 4, 0, 8, 0, \
    5, 1, 3, 0, 2, 1, 8, 0, 4, 0, 8, 0, 5, 2, 3, 1, 11, 0, 4, 1, 11, 1, 4, 2, \
    11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 2, 5, 0, 3, 2, 1, 1, 7, 0, 2, 0, \
    8, 0, 4, 0, 8, 0, 5, 1, 3, 0, 4, 1, 8, 0, 5, 2, 3, 2, 1, 0, 7, 0, 2, 1, \
    8, 0, 4, 0, 8, 0, 5, 3, 3, 0, 4, 3, 8, 0, 5, 4, 3, 1, 11, 0, 4, 1, 11, 1, \
    4, 3, 11, 2, 3, 1, 11, 3, 3, 1, 11, 4, 3, 1, 11, 5, 3, 1, 11, 6, 4, 2, 11, 7, \
    4, 4, 11, 8, 12, 26, 12, 32, 0, 0, 2, 2, 5, 0, 3, 0, 1, 1, 8, 0, 2, 0, 8, 0, \
    4, 0, 8, 0, 5, 1, 3, 0, 1, 0, 8, 0, 2, 1, 8, 0, 4, 0, 8, 0, 5, 2, 3, 1, \
    11, 0, 4, 1, 11, 1, 4, 2, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 2, 5, 0, \
    3, 0, 1, 9, 1, 1, 7, 0, 9, 0, 8, 0, 2, 0, 8, 0, 4, 0, 8, 0, 5, 1, 3, 0, \
    2, 1, 8, 0, 4, 0, 8, 0, 5, 2, 3, 1, 11, 0, 4, 1, 11, 1, 4, 2, 11, 2, 12, 8, \
    12, 16, 12, 24, 12, 32, 0, 0, 2, 2, 5, 0, 3, 2, 1, 1, 7, 0, 2, 0, 8, 0, 4, 0, \
    8, 0, 5, 1, 3, 0, 4, 1, 8, 0, 5, 2, 3, 2, 1, 4, 7, 0, 2, 1, 8, 0, 4, 0, \
    8, 0, 5, 3, 3, 0, 4, 3, 8, 0, 5, 4, 3, 1, 11, 0, 3, 1, 11, 1, 4, 3, 11, 2, \
    3, 1, 11, 3, 4, 1, 11, 4, 3, 1, 11, 5, 3, 1, 11, 6, 4, 2, 11, 7, 4, 4, 11, 8, \
    12, 26, 3, 1, 11, 12, 4, 1, 11, 13, 4, 3, 11, 14, 0, 0, 2, 2, 5, 0, 3, 0, 2, 0, \
    8, 0, 4, 0, 8, 0, 5, 1, 3, 0, 1, 4, 1, 0, 7, 0, 9, 0, 8, 0, 2, 1, 8, 0, \
    4, 0, 8, 0, 5, 2, 3, 1, 11, 0, 4, 1, 11, 1, 4, 2, 11, 2, 12, 8, 12, 16, 12, 24, \
    12, 32, 0, 0, 2, 2, 5, 0, 3, 2, 1, 9, 7, 0, 2, 0, 8, 0, 4, 0, 8, 0, 5, 1, \
    3, 0, 4, 1, 8, 0, 5, 2, 3, 2, 1, 4, 7, 0, 2, 1, 8, 0, 4, 0, 8, 0, 5, 3, \
    3, 0, 4, 3, 8, 0, 5, 4, 3, 1, 11, 0, 3, 1, 11, 1, 3, 1, 11, 2, 3, 1, 11, 3, \
    4, 1, 11, 4, 4, 3, 11, 5, 3, 1, 11, 6, 4, 2, 11, 7, 4, 4, 11, 8, 12, 26, 12, 33, \
    0, 0, 2, 2, 5, 0, 3, 2, 1, 9, 7, 0, 2, 0, 8, 0, 4, 0, 8, 0, 5, 1, 3, 0, \
    4, 1, 8, 0, 5, 2, 3, 2, 1, 0, 7, 0, 2, 1, 8, 0, 4, 0, 8, 0, 5, 3, 3, 0, \
    4, 3, 8, 0, 5, 4, 3, 1, 11, 0, 4, 1, 11, 1, 3, 1, 11, 2, 3, 1, 11, 3, 3, 1, \
    11, 4, 4, 3, 11, 5, 3, 1, 11, 6, 4, 2, 11, 7, 4, 4, 11, 8, 12, 26, 3, 1, 11, 12, \
    4, 1, 11, 13, 4, 3, 11, 14, 0, 0, 3, 1, 11, 0, 3, 1, 11, 1, 3, 1, 11, 2, 12, 8, \
    12, 16, 12, 24, 12, 32, 0, 0, 3, 0, 2, 1, 8, 0, 2, 2, 8, 0, 11, 0, 3, 0, 2, 0, \
    8, 0, 2, 2, 8, 0, 11, 1, 3, 0, 2, 0, 8, 0, 2, 1, 8, 0, 11, 2, 12, 8, 12, 16, \
    12, 24, 12, 32, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 18, 8, 0, \
    4, 0, 8, 0, 4, 1, 8, 0, 11, 0, 3, 0, 1, 9, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, \
    11, 1, 3, 0, 1, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 11, 2, 12, 8, 12, 16, 12, 24, \
    12, 32, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 18, 8, 0, 4, 0, \
    8, 0, 4, 1, 8, 0, 11, 0, 3, 0, 1, 9, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 11, 1, \
    3, 0, 1, 4, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, \
    0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 8, 0, 4, 0, 8, 0, \
    4, 2, 8, 0, 5, 3, 3, 0, 1, 4, 1, 0, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, \
    8, 0, 5, 4, 3, 0, 1, 18, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, \
    4, 3, 11, 1, 4, 4, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 0, 5, 0, 2, 1, \
    5, 1, 2, 2, 5, 2, 3, 0, 1, 18, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 11, 0, 3, 0, \
    1, 1, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 11, 1, 3, 0, 1, 4, 8, 0, 4, 1, 8, 0, \
    4, 2, 8, 0, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, \
    2, 2, 5, 2, 3, 0, 1, 9, 1, 1, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, \
    5, 3, 3, 0, 1, 4, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 8, 0, \
    4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 8, \
    12, 16, 12, 24, 12, 32, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, \
    1, 1, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 4, 1, 0, \
    7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 8, 0, 4, 0, \
    8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, \
    12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 18, 8, 0, \
    4, 0, 8, 0, 4, 1, 8, 0, 11, 0, 3, 0, 1, 1, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, \
    11, 1, 3, 0, 1, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 11, 2, 12, 8, 12, 16, 12, 24, \
    12, 32, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 1, 1, 7, 0, \
    9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 0, 8, 0, 4, 1, 8, 0, \
    4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, \
    11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 0, 5, 0, \
    2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 1, 1, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, \
    4, 2, 8, 0, 5, 3, 3, 0, 1, 0, 1, 4, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, \
    8, 0, 5, 4, 3, 0, 1, 18, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, \
    4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, \
    5, 1, 2, 2, 5, 2, 3, 0, 1, 1, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, \
    1, 4, 1, 0, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, \
    8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, \
    12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, \
    1, 1, 1, 9, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 0, \
    1, 4, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 8, 0, \
    4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, \
    12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 1, \
    1, 9, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 4, 1, 0, \
    7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 8, 0, 4, 0, \
    8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, \
    12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 1, 1, \
    7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 4, 1, 0, 7, 0, \
    9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 4, 0, 8, 0, 4, 1, 8, 0, \
    5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, \
    2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 2, 8, 0, 4, 0, 8, 0, 4, 1, \
    8, 0, 11, 0, 3, 0, 1, 9, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 11, 1, 3, 0, 1, 0, \
    8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 0, \
    5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, \
    5, 3, 3, 0, 1, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 1, 2, \
    7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, \
    4, 4, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, \
    5, 2, 3, 0, 1, 9, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 0, 1, 4, \
    7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 1, 2, 7, 0, \
    9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, \
    11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, \
    3, 0, 1, 9, 1, 1, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, \
    1, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 1, 2, 7, 0, 9, 0, \
    8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, \
    12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, \
    1, 9, 1, 1, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 0, \
    1, 4, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 1, 2, \
    7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, \
    4, 4, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, \
    5, 2, 3, 0, 1, 1, 1, 9, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, \
    3, 0, 1, 4, 1, 0, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, \
    3, 2, 1, 2, 7, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, \
    11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, \
    2, 2, 5, 2, 3, 0, 1, 2, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 11, 0, 3, 0, 1, 9, \
    8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 11, 1, 3, 0, 1, 4, 8, 0, 4, 1, 8, 0, 4, 2, \
    8, 0, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, \
    5, 2, 3, 0, 1, 9, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 4, 8, 0, \
    4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 1, 2, 7, 0, 9, 0, 8, 0, 4, 0, \
    8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 8, 12, 16, \
    12, 24, 12, 32, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 8, 0, \
    4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 4, 1, 0, 7, 0, 9, 0, 8, 0, 4, 1, \
    8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 1, 2, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, \
    4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, \
    12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 1, 1, 7, 0, \
    9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 4, 8, 0, 4, 1, 8, 0, \
    4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 1, 2, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, \
    8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, \
    0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 1, 1, 7, 0, 9, 0, \
    8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 4, 1, 0, 7, 0, 9, 0, 8, 0, \
    4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 1, 2, 7, 0, 9, 0, 8, 0, 4, 0, \
    8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 8, 12, 16, \
    12, 24, 12, 32, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 1, 1, 9, \
    7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 0, 1, 4, 7, 0, \
    9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 3, 2, 1, 2, 7, 0, 8, 0, \
    4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, \
    12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, \
    8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 4, 1, 0, 7, 0, 9, 0, 8, 0, \
    4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 2, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, \
    5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, \
    2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 8, 0, 4, 0, 8, 0, 4, 2, \
    8, 0, 5, 3, 3, 0, 1, 0, 1, 4, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, \
    5, 4, 3, 0, 1, 2, 1, 18, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, \
    4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, \
    5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, \
    5, 3, 3, 0, 1, 4, 1, 0, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, \
    3, 0, 1, 2, 1, 18, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, \
    11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, \
    2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 4, \
    1, 0, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 1, 2, \
    7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, \
    4, 4, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, \
    5, 2, 3, 0, 3, 2, 1, 9, 7, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, \
    1, 0, 1, 4, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 2, \
    1, 18, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, \
    11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, \
    2, 2, 5, 2, 3, 0, 3, 2, 1, 9, 7, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, \
    3, 0, 1, 4, 1, 0, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, \
    1, 2, 1, 18, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, \
    4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, \
    5, 1, 2, 2, 5, 2, 3, 0, 1, 4, 1, 0, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, \
    8, 0, 5, 3, 3, 2, 1, 1, 7, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 4, 4, \
    8, 0, 5, 5, 3, 2, 1, 2, 7, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 6, 3, 0, 4, 6, \
    8, 0, 5, 7, 4, 7, 11, 0, 4, 5, 11, 1, 4, 3, 11, 2, 4, 7, 11, 3, 4, 5, 11, 4, \
    4, 3, 11, 5, 4, 6, 11, 6, 3, 1, 11, 7, 4, 3, 11, 8, 3, 1, 11, 9, 4, 4, 11, 10, \
    4, 3, 11, 11, 4, 6, 11, 12, 4, 4, 11, 13, 4, 3, 11, 14, 0, 0, 2, 0, 5, 0, 2, 1, \
    5, 1, 2, 2, 5, 2, 3, 0, 1, 2, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 11, 0, 3, 0, \
    1, 1, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 11, 1, 3, 0, 1, 4, 8, 0, 4, 1, 8, 0, \
    4, 2, 8, 0, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, \
    2, 2, 5, 2, 3, 0, 1, 1, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 4, \
    8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 1, 2, 7, 0, 9, 0, 8, 0, \
    4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 8, \
    12, 16, 12, 24, 12, 32, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 1, \
    1, 9, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 4, 8, 0, \
    4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 1, 2, 7, 0, 9, 0, 8, 0, 4, 0, \
    8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, \
    12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 1, 8, 0, \
    4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 4, 1, 0, 7, 0, 9, 0, 8, 0, 4, 1, \
    8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 1, 2, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, \
    4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, \
    12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 1, 1, 9, 7, 0, \
    9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 4, 1, 0, 7, 0, 9, 0, \
    8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 1, 2, 7, 0, 9, 0, 8, 0, \
    4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 8, \
    12, 16, 12, 24, 12, 32, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, \
    1, 1, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 0, 1, 4, \
    7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 3, 2, 1, 2, 7, 0, \
    8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, \
    12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, \
    1, 9, 1, 1, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 4, \
    8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 2, 8, 0, 4, 0, 8, 0, 4, 1, \
    8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, \
    0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 1, 1, 7, 0, 9, 0, \
    8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 4, 8, 0, 4, 1, 8, 0, 4, 2, \
    8, 0, 5, 4, 3, 0, 1, 2, 1, 18, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, \
    5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, \
    2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 1, 1, 9, 7, 0, 9, 0, 8, 0, \
    4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 4, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, \
    5, 4, 3, 0, 1, 2, 1, 18, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, \
    4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, \
    5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 1, 1, 7, 0, 9, 0, 8, 0, 4, 0, \
    8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, \
    1, 2, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, \
    11, 1, 4, 4, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, \
    2, 2, 5, 2, 3, 0, 1, 1, 1, 9, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, \
    5, 3, 3, 0, 3, 2, 1, 0, 7, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, \
    1, 2, 1, 18, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, \
    4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, \
    5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 1, 1, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, \
    8, 0, 5, 3, 3, 0, 3, 2, 1, 0, 7, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, \
    3, 0, 1, 2, 1, 18, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, \
    11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, \
    2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 1, 1, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, \
    4, 2, 8, 0, 5, 3, 3, 2, 1, 0, 7, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, \
    4, 4, 8, 0, 5, 5, 3, 2, 1, 2, 7, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 6, 3, 0, \
    4, 6, 8, 0, 5, 7, 4, 6, 11, 0, 4, 3, 11, 1, 4, 5, 11, 2, 3, 1, 11, 3, 4, 3, \
    11, 4, 4, 5, 11, 5, 4, 7, 11, 6, 4, 3, 11, 7, 3, 1, 11, 8, 4, 7, 11, 9, 4, 3, \
    11, 10, 4, 4, 11, 11, 4, 6, 11, 12, 4, 3, 11, 13, 4, 4, 11, 14, 0, 0, 2, 0, 5, 0, \
    2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 1, 1, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, \
    4, 2, 8, 0, 5, 3, 3, 0, 1, 4, 1, 0, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, \
    8, 0, 5, 4, 3, 0, 1, 2, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, \
    4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, \
    5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 1, 1, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, \
    8, 0, 5, 3, 3, 0, 1, 4, 1, 0, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, \
    5, 4, 3, 0, 1, 2, 1, 18, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, \
    4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 0, \
    5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 3, 2, 1, 9, 7, 0, 8, 0, 4, 0, 8, 0, \
    4, 2, 8, 0, 5, 3, 3, 0, 1, 0, 1, 4, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, \
    8, 0, 5, 4, 3, 0, 1, 18, 1, 2, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, \
    5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, \
    2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 1, 1, 9, 7, 0, 9, 0, 8, 0, \
    4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 3, 2, 1, 0, 7, 0, 8, 0, 4, 1, 8, 0, \
    4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 1, 2, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, \
    8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, \
    0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 18, 1, 2, 7, 0, 9, 0, \
    8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 3, 3, 2, 1, 1, 7, 0, 4, 0, 8, 0, 4, 2, \
    8, 0, 5, 4, 3, 0, 4, 4, 8, 0, 5, 5, 3, 2, 1, 0, 7, 0, 4, 1, 8, 0, 4, 2, \
    8, 0, 5, 6, 3, 0, 4, 6, 8, 0, 5, 7, 4, 3, 11, 0, 4, 4, 11, 1, 4, 6, 11, 2, \
    4, 3, 11, 3, 3, 1, 11, 4, 3, 1, 11, 5, 4, 3, 11, 6, 4, 5, 11, 7, 4, 7, 11, 8, \
    4, 3, 11, 9, 4, 5, 11, 10, 4, 7, 11, 11, 4, 3, 11, 12, 4, 4, 11, 13, 4, 6, 11, 14, \
    0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 2, 1, 1, 7, 0, 4, 0, 8, 0, \
    4, 2, 8, 0, 5, 3, 3, 2, 1, 0, 7, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 2, \
    1, 2, 7, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, \
    11, 2, 3, 1, 11, 3, 3, 1, 11, 4, 3, 1, 11, 5, 4, 5, 11, 6, 3, 1, 11, 7, 3, 1, \
    11, 8, 3, 1, 11, 9, 4, 3, 11, 10, 4, 4, 11, 11, 3, 1, 11, 12, 3, 1, 11, 13, 3, 1, \
    11, 14, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 2, 8, 0, 4, 0, \
    8, 0, 4, 1, 8, 0, 11, 0, 3, 0, 1, 1, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 11, 1, \
    3, 0, 1, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, \
    0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 1, 8, 0, 4, 0, 8, 0, \
    4, 2, 8, 0, 5, 3, 3, 0, 1, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, \
    1, 18, 1, 2, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, \
    4, 3, 11, 1, 4, 4, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 0, 5, 0, 2, 1, \
    5, 1, 2, 2, 5, 2, 3, 0, 1, 1, 1, 9, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, \
    8, 0, 5, 3, 3, 0, 1, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, \
    1, 2, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, \
    11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, \
    2, 2, 5, 2, 3, 0, 1, 1, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 0, \
    1, 4, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 1, 2, \
    7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, \
    4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, \
    5, 2, 3, 0, 1, 1, 1, 9, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, \
    3, 0, 1, 0, 1, 4, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, \
    1, 18, 1, 2, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, \
    4, 3, 11, 1, 4, 4, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 0, 5, 0, 2, 1, \
    5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 1, 1, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, \
    8, 0, 5, 3, 3, 0, 1, 4, 1, 0, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, \
    5, 4, 3, 0, 3, 2, 1, 2, 7, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, \
    11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, \
    2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 1, 1, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, \
    4, 2, 8, 0, 5, 3, 3, 0, 1, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, \
    1, 2, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, \
    11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, \
    3, 0, 1, 9, 1, 1, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, \
    1, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 2, 1, 18, 7, 0, 9, 0, \
    8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, \
    12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, \
    1, 1, 1, 9, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 0, \
    8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 2, 1, 18, 7, 0, 9, 0, 8, 0, \
    4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, \
    12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, \
    1, 1, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 4, 1, 8, 0, \
    4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 1, 2, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, \
    8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, \
    0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 1, 1, 9, 7, 0, 9, 0, \
    8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 3, 2, 1, 4, 7, 0, 8, 0, 4, 1, \
    8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 2, 1, 18, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, \
    4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, \
    12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 1, 1, 7, 0, \
    9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 3, 2, 1, 4, 7, 0, 8, 0, \
    4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 2, 1, 18, 7, 0, 9, 0, 8, 0, 4, 0, \
    8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, \
    12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 1, 1, \
    7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 2, 1, 4, 7, 0, 4, 1, \
    8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 4, 4, 8, 0, 5, 5, 3, 2, 1, 2, 7, 0, 4, 0, \
    8, 0, 4, 1, 8, 0, 5, 6, 3, 0, 4, 6, 8, 0, 5, 7, 3, 1, 11, 0, 4, 3, 11, 1, \
    4, 5, 11, 2, 4, 6, 11, 3, 4, 3, 11, 4, 4, 5, 11, 5, 4, 7, 11, 6, 4, 3, 11, 7, \
    3, 1, 11, 8, 4, 7, 11, 9, 4, 3, 11, 10, 4, 4, 11, 11, 4, 6, 11, 12, 4, 3, 11, 13, \
    4, 4, 11, 14, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 1, 1, \
    7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 0, 1, 4, 7, 0, \
    9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 2, 8, 0, 4, 0, 8, 0, \
    4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, \
    12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 1, 1, 7, 0, \
    9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 0, 1, 4, 7, 0, 9, 0, \
    8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 2, 1, 18, 7, 0, 9, 0, 8, 0, \
    4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 8, \
    12, 16, 12, 24, 12, 32, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 3, 2, \
    1, 9, 7, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 4, 1, 0, 7, 0, \
    9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 1, 2, 7, 0, 9, 0, \
    8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, \
    12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, \
    1, 1, 1, 9, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 3, 2, \
    1, 4, 7, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 1, 2, 7, 0, \
    9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, \
    11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, \
    3, 0, 1, 18, 1, 2, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 3, 3, 2, \
    1, 1, 7, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 4, 4, 8, 0, 5, 5, 3, 2, \
    1, 4, 7, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 6, 3, 0, 4, 6, 8, 0, 5, 7, 4, 3, \
    11, 0, 3, 1, 11, 1, 4, 6, 11, 2, 4, 3, 11, 3, 4, 4, 11, 4, 3, 1, 11, 5, 4, 3, \
    11, 6, 4, 5, 11, 7, 4, 7, 11, 8, 4, 3, 11, 9, 4, 5, 11, 10, 4, 7, 11, 11, 4, 3, \
    11, 12, 4, 4, 11, 13, 4, 6, 11, 14, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, \
    3, 2, 1, 1, 7, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 2, 1, 4, 7, 0, 4, 1, \
    8, 0, 4, 2, 8, 0, 5, 4, 3, 2, 1, 2, 7, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, \
    3, 1, 11, 0, 3, 1, 11, 1, 4, 4, 11, 2, 4, 5, 11, 3, 4, 3, 11, 4, 3, 1, 11, 5, \
    4, 5, 11, 6, 3, 1, 11, 7, 3, 1, 11, 8, 3, 1, 11, 9, 4, 3, 11, 10, 4, 4, 11, 11, \
    3, 1, 11, 12, 3, 1, 11, 13, 3, 1, 11, 14, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, \
    5, 2, 3, 0, 1, 1, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 4, 1, 0, \
    7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 2, 8, 0, 4, 0, \
    8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 8, 12, 16, \
    12, 24, 12, 32, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 1, 8, 0, \
    4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 4, 1, 0, 7, 0, 9, 0, 8, 0, 4, 1, \
    8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 2, 1, 18, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, \
    4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, \
    12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 1, 8, 0, 4, 0, \
    8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 0, 1, 4, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, \
    4, 2, 8, 0, 5, 4, 3, 0, 1, 2, 1, 18, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, \
    8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, \
    0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 4, 0, 8, 0, 4, 2, 8, 0, \
    5, 3, 3, 0, 1, 4, 1, 0, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, \
    3, 0, 1, 18, 1, 2, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, \
    11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 0, 5, 0, \
    2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 3, 2, 1, 1, 7, 0, 8, 0, 4, 0, 8, 0, 4, 2, \
    8, 0, 5, 3, 3, 0, 1, 4, 1, 0, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, \
    5, 4, 3, 0, 1, 2, 1, 18, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, \
    4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, \
    5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 3, 2, 1, 1, 7, 0, 8, 0, 4, 0, 8, 0, \
    4, 2, 8, 0, 5, 3, 3, 0, 1, 0, 1, 4, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, \
    8, 0, 5, 4, 3, 0, 1, 2, 1, 18, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, \
    5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, \
    2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 4, 1, 0, 7, 0, 9, 0, 8, 0, \
    4, 1, 8, 0, 4, 2, 8, 0, 5, 3, 3, 2, 1, 9, 7, 0, 4, 0, 8, 0, 4, 2, 8, 0, \
    5, 4, 3, 0, 4, 4, 8, 0, 5, 5, 3, 2, 1, 2, 7, 0, 4, 0, 8, 0, 4, 1, 8, 0, \
    5, 6, 3, 0, 4, 6, 8, 0, 5, 7, 4, 7, 11, 0, 4, 5, 11, 1, 4, 3, 11, 2, 4, 7, \
    11, 3, 4, 5, 11, 4, 4, 3, 11, 5, 3, 1, 11, 6, 3, 1, 11, 7, 4, 3, 11, 8, 4, 6, \
    11, 9, 4, 4, 11, 10, 4, 3, 11, 11, 12, 35, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, \
    5, 2, 3, 0, 1, 1, 1, 9, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, \
    3, 0, 1, 0, 1, 4, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, \
    1, 2, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, \
    11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, \
    3, 0, 1, 1, 1, 9, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, \
    1, 0, 1, 4, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 2, \
    1, 18, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, \
    11, 1, 4, 4, 11, 2, 12, 8, 12, 16, 12, 24, 12, 32, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, \
    2, 2, 5, 2, 3, 0, 1, 9, 1, 1, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, \
    5, 3, 3, 0, 3, 2, 1, 4, 7, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, \
    1, 18, 1, 2, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, \
    4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, \
    5, 1, 2, 2, 5, 2, 3, 0, 3, 2, 1, 1, 7, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, \
    5, 3, 3, 0, 1, 4, 1, 0, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, \
    3, 0, 1, 18, 1, 2, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, \
    11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, \
    2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 18, 1, 2, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, \
    4, 1, 8, 0, 5, 3, 3, 2, 1, 9, 7, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, \
    4, 4, 8, 0, 5, 5, 3, 2, 1, 4, 7, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 6, 3, 0, \
    4, 6, 8, 0, 5, 7, 4, 3, 11, 0, 3, 1, 11, 1, 3, 1, 11, 2, 4, 3, 11, 3, 4, 4, \
    11, 4, 4, 6, 11, 5, 4, 3, 11, 6, 4, 5, 11, 7, 4, 7, 11, 8, 4, 3, 11, 9, 4, 5, \
    11, 10, 4, 7, 11, 11, 12, 33, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 2, \
    1, 9, 7, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 2, 1, 4, 7, 0, 4, 1, 8, 0, \
    4, 2, 8, 0, 5, 4, 3, 2, 1, 2, 7, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 3, 1, \
    11, 0, 3, 1, 11, 1, 3, 1, 11, 2, 4, 5, 11, 3, 4, 3, 11, 4, 4, 4, 11, 5, 3, 1, \
    11, 6, 3, 1, 11, 7, 3, 1, 11, 8, 12, 25, 3, 1, 11, 12, 3, 1, 11, 13, 3, 1, 11, 14, \
    0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 1, 1, 9, 7, 0, 9, 0, \
    8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 4, 1, 0, 7, 0, 9, 0, 8, 0, \
    4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 2, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, \
    5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, \
    2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 1, 1, 9, 7, 0, 9, 0, 8, 0, \
    4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 4, 1, 0, 7, 0, 9, 0, 8, 0, 4, 1, \
    8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 2, 1, 18, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, \
    4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 8, 12, 16, 12, 24, \
    12, 32, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 1, 1, 7, 0, \
    9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 3, 2, 1, 0, 7, 0, 8, 0, \
    4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 1, 2, 7, 0, 9, 0, 8, 0, 4, 0, \
    8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, \
    12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 3, 2, 1, 1, \
    7, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 0, 1, 4, 7, 0, 9, 0, \
    8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 1, 18, 1, 2, 7, 0, 9, 0, 8, 0, \
    4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, \
    12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 18, \
    1, 2, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 3, 3, 2, 1, 9, 7, 0, \
    4, 0, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 4, 4, 8, 0, 5, 5, 3, 2, 1, 0, 7, 0, \
    4, 1, 8, 0, 4, 2, 8, 0, 5, 6, 3, 0, 4, 6, 8, 0, 5, 7, 4, 3, 11, 0, 4, 4, \
    11, 1, 3, 1, 11, 2, 4, 3, 11, 3, 3, 1, 11, 4, 4, 6, 11, 5, 4, 3, 11, 6, 4, 5, \
    11, 7, 4, 7, 11, 8, 4, 3, 11, 9, 4, 5, 11, 10, 4, 7, 11, 11, 4, 3, 11, 12, 4, 4, \
    11, 13, 4, 6, 11, 14, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 2, 1, 9, \
    7, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 2, 1, 0, 7, 0, 4, 1, 8, 0, 4, 2, \
    8, 0, 5, 4, 3, 2, 1, 2, 7, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, \
    4, 3, 11, 1, 3, 1, 11, 2, 3, 1, 11, 3, 3, 1, 11, 4, 4, 4, 11, 5, 3, 1, 11, 6, \
    3, 1, 11, 7, 3, 1, 11, 8, 4, 5, 11, 9, 4, 3, 11, 10, 4, 4, 11, 11, 3, 1, 11, 12, \
    3, 1, 11, 13, 3, 1, 11, 14, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, \
    1, 9, 1, 1, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 4, \
    1, 0, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 4, 0, 8, 0, \
    4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 8, 12, 16, 12, 24, \
    12, 32, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 1, 1, 9, 7, 0, \
    9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 4, 1, 0, 7, 0, 9, 0, \
    8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 3, 2, 1, 18, 7, 0, 8, 0, 4, 0, \
    8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, \
    12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 1, 1, 9, \
    7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 0, 1, 4, 7, 0, \
    9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 3, 2, 1, 18, 7, 0, 8, 0, \
    4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, \
    12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 4, \
    1, 0, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 3, 3, 2, 1, 1, 7, 0, \
    4, 0, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, 4, 4, 8, 0, 5, 5, 3, 2, 1, 18, 7, 0, \
    4, 0, 8, 0, 4, 1, 8, 0, 5, 6, 3, 0, 4, 6, 8, 0, 5, 7, 4, 7, 11, 0, 4, 5, \
    11, 1, 4, 3, 11, 2, 4, 7, 11, 3, 4, 5, 11, 4, 4, 3, 11, 5, 4, 6, 11, 6, 4, 4, \
    11, 7, 4, 3, 11, 8, 3, 1, 11, 9, 3, 1, 11, 10, 4, 3, 11, 11, 12, 34, 0, 0, 2, 0, \
    5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 1, 1, 7, 0, 9, 0, 8, 0, 4, 0, \
    8, 0, 4, 2, 8, 0, 5, 3, 3, 0, 1, 0, 1, 4, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, \
    4, 2, 8, 0, 5, 4, 3, 0, 3, 2, 1, 18, 7, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, \
    5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, \
    2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 1, 1, 7, 0, 9, 0, 8, 0, \
    4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 2, 1, 0, 7, 0, 4, 1, 8, 0, 4, 2, 8, 0, \
    5, 4, 3, 0, 4, 4, 8, 0, 5, 5, 3, 2, 1, 18, 7, 0, 4, 0, 8, 0, 4, 1, 8, 0, \
    5, 6, 3, 0, 4, 6, 8, 0, 5, 7, 4, 6, 11, 0, 4, 3, 11, 1, 4, 5, 11, 2, 3, 1, \
    11, 3, 4, 3, 11, 4, 4, 5, 11, 5, 4, 7, 11, 6, 4, 3, 11, 7, 4, 4, 11, 8, 4, 7, \
    11, 9, 4, 3, 11, 10, 3, 1, 11, 11, 4, 6, 11, 12, 4, 3, 11, 13, 4, 4, 11, 14, 0, 0, \
    2, 0, 5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 2, 1, 1, 7, 0, 4, 0, 8, 0, 4, 2, \
    8, 0, 5, 3, 3, 2, 1, 0, 7, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 2, 1, 18, \
    7, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 4, 4, 11, 2, \
    3, 1, 11, 3, 3, 1, 11, 4, 3, 1, 11, 5, 12, 16, 3, 1, 11, 9, 3, 1, 11, 10, 3, 1, \
    11, 11, 3, 1, 11, 12, 3, 1, 11, 13, 3, 1, 11, 14, 0, 0, 2, 0, 5, 0, 2, 1, 5, 1, \
    2, 2, 5, 2, 3, 0, 1, 9, 1, 1, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, 8, 0, \
    5, 3, 3, 0, 1, 4, 1, 0, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, \
    3, 0, 3, 2, 1, 18, 7, 0, 8, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, \
    4, 3, 11, 1, 4, 4, 11, 2, 12, 32, 12, 8, 12, 16, 12, 24, 0, 0, 2, 0, 5, 0, 2, 1, \
    5, 1, 2, 2, 5, 2, 3, 0, 1, 9, 1, 1, 7, 0, 9, 0, 8, 0, 4, 0, 8, 0, 4, 2, \
    8, 0, 5, 3, 3, 2, 1, 4, 7, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 2, 1, 18, \
    7, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 3, 0, 4, 4, 8, 0, 5, 6, 3, 0, 4, 5, \
    8, 0, 5, 7, 3, 1, 11, 0, 4, 3, 11, 1, 4, 6, 11, 2, 4, 5, 11, 3, 4, 3, 11, 4, \
    4, 6, 11, 5, 4, 7, 11, 6, 4, 3, 11, 7, 4, 4, 11, 8, 4, 7, 11, 9, 4, 3, 11, 10, \
    3, 1, 11, 11, 4, 5, 11, 12, 4, 3, 11, 13, 4, 4, 11, 14, 0, 0, 2, 0, 5, 0, 2, 1, \
    5, 1, 2, 2, 5, 2, 3, 2, 1, 1, 7, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, 3, 2, \
    1, 4, 7, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 2, 1, 18, 7, 0, 4, 0, 8, 0, \
    4, 1, 8, 0, 5, 5, 3, 1, 11, 0, 3, 1, 11, 1, 4, 4, 11, 2, 4, 5, 11, 3, 4, 3, \
    11, 4, 3, 1, 11, 5, 4, 5, 11, 6, 4, 3, 11, 7, 4, 4, 11, 8, 3, 1, 11, 9, 3, 1, \
    11, 10, 3, 1, 11, 11, 3, 1, 11, 12, 3, 1, 11, 13, 3, 1, 11, 14, 0, 0, 2, 0, 5, 0, \
    2, 1, 5, 1, 2, 2, 5, 2, 3, 0, 1, 4, 1, 0, 7, 0, 9, 0, 8, 0, 4, 1, 8, 0, \
    4, 2, 8, 0, 5, 3, 3, 2, 1, 9, 7, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 4, 3, 0, \
    4, 4, 8, 0, 5, 5, 3, 2, 1, 18, 7, 0, 4, 0, 8, 0, 4, 1, 8, 0, 5, 6, 3, 0, \
    4, 6, 8, 0, 5, 7, 4, 7, 11, 0, 4, 5, 11, 1, 4, 3, 11, 2, 4, 7, 11, 3, 4, 5, \
    11, 4, 4, 3, 11, 5, 3, 1, 11, 6, 4, 4, 11, 7, 4, 3, 11, 8, 4, 6, 11, 9, 3, 1, \
    11, 10, 4, 3, 11, 11, 4, 6, 11, 12, 4, 4, 11, 13, 4, 3, 11, 14, 0, 0, 2, 0, 5, 0, \
    2, 1, 5, 1, 2, 2, 5, 2, 3, 2, 1, 9, 7, 0, 4, 0, 8, 0, 4, 2, 8, 0, 5, 3, \
    3, 2, 1, 4, 7, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 2, 1, 18, 7, 0, 4, 0, \
    8, 0, 4, 1, 8, 0, 5, 5, 3, 1, 11, 0, 3, 1, 11, 1, 3, 1, 11, 2, 4, 5, 11, 3, \
    4, 3, 11, 4, 4, 4, 11, 5, 3, 1, 11, 6, 4, 3, 11, 7, 4, 4, 11, 8, 4, 5, 11, 9, \
    3, 1, 11, 10, 3, 1, 11, 11, 3, 1, 11, 12, 3, 1, 11, 13, 3, 1, 11, 14, 0, 0, 2, 0, \
    5, 0, 2, 1, 5, 1, 2, 2, 5, 2, 3, 2, 1, 9, 7, 0, 4, 0, 8, 0, 4, 2, 8, 0, \
    5, 3, 3, 2, 1, 0, 7, 0, 4, 1, 8, 0, 4, 2, 8, 0, 5, 4, 3, 2, 1, 18, 7, 0, \
    4, 0, 8, 0, 4, 1, 8, 0, 5, 5, 4, 5, 11, 0, 4, 3, 11, 1, 3, 1, 11, 2, 3, 1, \
    11, 3, 3, 1, 11, 4, 4, 4, 11, 5, 3, 1, 11, 6, 4, 3, 11, 7, 4, 4, 11, 8, 4, 5, \
    11, 9, 3, 1, 11, 10, 3, 1, 11, 11, 3, 1, 11, 12, 3, 1, 11, 13, 3, 1, 11, 14, 0, 0, \
    3, 1, 11, 0, 3, 1, 11, 1, 3, 1, 11, 2, 3, 1, 11, 3, 3, 1, 11, 4, 3, 1, 11, 5, \
    3, 1, 11, 6, 3, 1, 11, 7, 3, 1, 11, 8, 3, 1, 11, 9, 3, 1, 11, 10, 3, 1, 11, 11, \
    3, 1, 11, 12, 3, 1, 11, 13, 3, 1, 11, 14, 0, 0, \
}
static const DibCase kDibCaseHost[kDibCases] = LSG_DIB_TABLE;
static const unsigned char kDibCodeHost[kDibCode] = LSG_DIB_CODE;
static const double kDibConstHost[3] = {0.5, 0.0, 1.0};
#ifdef __CUDACC__
__constant__ DibCase kDibCaseDev[kDibCases] = LSG_DIB_TABLE;
__device__ const unsigned char kDibCodeDev[kDibCode] = LSG_DIB_CODE;
__constant__ double kDibConstDev[3] = {0.5, 0.0, 1.0};
#endif
#undef LSG_DIB_TABLE
#undef LSG_DIB_CODE

// out: the cell's five triples (en, ws, nb, st, max), left as given when the
// type has no block
LSG_MHD void dib_cell(long long c, int type, int side_z, long long N, long long NM, const double* theta,
                      const double* delta, double (&out)[15])
{
#ifdef __CUDA_ARCH__
    const DibCase* cs = kDibCaseDev;
    const unsigned char* code = kDibCodeDev;
    const double* kc = kDibConstDev;
#else
    const DibCase* cs = kDibCaseHost;
    const unsigned char* code = kDibCodeHost;
    const double* kc = kDibConstHost;
#endif
    const int sz = (type == B_Border || type == T_Border) ? side_z : -1;
    int lo = 0, hi = kDibCases - 1, at = -1;
    while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        const int cmp = (cs[mid].type != type) ? (cs[mid].type < type ? -1 : 1) : (cs[mid].side_z < sz ? -1 :
                                                                                   (cs[mid].side_z > sz ? 1 : 0));
        if (cmp == 0) {
            at = cs[mid].at;
            break;
        }
        if (cmp < 0) lo = mid + 1;
        else hi = mid - 1;
    }
    if (at < 0) return;
    double st[8], loc[8];
    int sp = 0;
    for (const unsigned char* p = code + at;; p += 2) {
        const unsigned char op = p[0], a = p[1];
        switch (op) {
        case DIB_END: return;
        case DIB_T: st[sp++] = opnd(theta, c, a, N, NM); break;
        case DIB_D: st[sp++] = delta[3 * c + a]; break;
        case DIB_C: st[sp++] = kc[a]; break;
        case DIB_LD: st[sp++] = loc[a]; break;
        case DIB_ST: loc[a] = st[--sp]; break;
        case DIB_ADD: sp--; st[sp - 1] = add(st[sp - 1], st[sp]); break;
        case DIB_SUB: sp--; st[sp - 1] = sub(st[sp - 1], st[sp]); break;
        case DIB_MUL: sp--; st[sp - 1] = mul(st[sp - 1], st[sp]); break;
        case DIB_ABS: st[sp - 1] = fabs(st[sp - 1]); break;
        case DIB_NEG: st[sp - 1] = -st[sp - 1]; break;
        case DIB_OUT: out[a] = st[--sp]; break;
        case DIB_COPY: {
            const int d = a >> 3, s = a & 7;
            for (int q = 0; q < 3; q++) out[3 * d + q] = out[3 * s + q];
            break;
        }
        default: return;
        }
    }
}

// inverse distances to the cut surface (calcInvBaseDeltaIb,
// ls_stag_uniform_mesh.h:3395-3620) across the east, north and top faces:
// for each face, by its side type, the edge fractions of its two in-plane
// directions P and Q at the cell and one cell back give 2 / delta next to a
// closed edge of a fluid face, 3 / (alpha delta) on triangles, and
// 3 (a1 + a2) / ((a1 (a1 + a2) + a2 a2) delta) on trapezoids.  Returns the
// two values of the face (P direction, Q direction).
LSG_MHD void inv_dib_face(int st, const double* alpha, long long c, int cp, long long bp, int cq, long long bq,
                          const double* d, int dp, int dq, double& outp, double& outq)
{
    const double pc = alpha[3 * c + cp], pb = alpha[3 * bp + cp];
    const double qc = alpha[3 * c + cq], qb = alpha[3 * bq + cq];
    auto tri = [&](double a, int di, double& o) {
        if (a > kEq) o = dvd(3.0, mul(a, d[di]));
    };
    auto trap = [&](double a1, double a2, int di, double& o) {
        const double s = add(a1, a2);
        const double den = add(mul(a1, s), mul(a2, a2));
        if (den > kEq) o = dvd(mul(3.0, s), mul(den, d[di]));
    };
    switch (st) {
    case kFluidSide:
        if (pc < kEq || pb < kEq) outq = dvd(2.0, d[dq]);
        if (qc < kEq || qb < kEq) outp = dvd(2.0, d[dp]);
        break;
    case 10: tri(pb, dp, outp); tri(qb, dq, outq); break;       // NE triangle
    case 1: tri(pb, dp, outp); tri(qc, dq, outq); break;        // NW triangle
    case 100: tri(pc, dp, outp); tri(qb, dq, outq); break;      // SE triangle
    case 1000: tri(pc, dp, outp); tri(qc, dq, outq); break;     // SW triangle
    case 1001: case 110: trap(pb, pc, dp, outp); break;         // W, E trapezoids
    case 1100: case 11: trap(qb, qc, dq, outq); break;          // S, N trapezoids
    default: break;
    }
}

// inv_dib_ne = (x_N, y_E, z_E), inv_dib_tn = (x_T, y_T, z_N); zero outside
// the bottom / top borders and the cut cells
LSG_MHD void inv_dib_cell(long long c, int type, const int* side, const double* alpha, const double* delta,
                          long long N, long long NM, double* ne, double* tn)
{
    double xN = 0, yE = 0, zE = 0, zN = 0, xT = 0, yT = 0;
    if (type > N_Border && type < kFluid && type != kSolid) {
        const long long nb = (c < NM) ? c : c - NM;
        const double* d = delta + 3 * c;
        inv_dib_face(side[3 * c], alpha, c, 1, nb, 2, c - N, d, 1, 2, yE, zE);        // east face: P = y, Q = z
        inv_dib_face(side[3 * c + 1], alpha, c, 0, nb, 2, c - 1, d, 0, 2, xN, zN);    // north face: P = x, Q = z
        inv_dib_face(side[3 * c + 2], alpha, c, 0, c - N, 1, c - 1, d, 0, 1, xT, yT); // top face: P = x, Q = y
    }
    ne[3 * c] = xN;
    ne[3 * c + 1] = yE;
    ne[3 * c + 2] = zE;
    tn[3 * c] = xT;
    tn[3 * c + 1] = yT;
    tn[3 * c + 2] = zN;
}

// ---------------------------------------------------------------------------
// kernels (one thread per cell unless stated; the level-set block is
// [hs, hf) x [vs, vf) x [0, K))
// ---------------------------------------------------------------------------
#ifdef __CUDACC__
struct Block {
    int hs, hf, vs, vf;
};

// every cell outside the block as the flow task's walks leave it: level set
// 0, alpha and theta 1, fluid faces, the box classification, cell sizes h
__global__ void __launch_bounds__(256) k_mesh_init(int N, int M, int K, double hx, double hy, double hz, double* phi0,
                                                   double* alpha, double* theta, double* delta, int* side, int* type)
{
    const long long n = (long long)N * M * K;
    const long long NM = (long long)N * M;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(c / NM);
        const long long r = c - (long long)k * NM;
        const int j = (int)(r / N), i = (int)(r - (long long)j * N);
        phi0[c] = 0.0;
        for (int q = 0; q < 3; q++) {
            alpha[3 * c + q] = 1.0;
            theta[3 * c + q] = 1.0;
            side[3 * c + q] = kFluidSide;
        }
        delta[3 * c] = hx;
        delta[3 * c + 1] = hy;
        delta[3 * c + 2] = hz;
        type[c] = box_type(i, j, k, N, M, K);
    }
}

// one thread per x-row (j, k) of the block
__global__ void __launch_bounds__(128) k_mesh_levelset(int N, int M, int K, Block b, double hx, double hy, double hz,
                                                       int nb, const double* __restrict__ bodies, double* phi0)
{
    const int rows = b.vf - b.vs;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)rows * K) return;
    const int k = (int)(t / rows), j = b.vs + (int)(t - (long long)k * rows);
    const double h[3] = {hx, hy, hz};
    levelset_row(j, k, N, M, b.hs, b.hf, h, nb, bodies, phi0);
}

// a caller's level set: the block's values, zero elsewhere
__global__ void __launch_bounds__(256) k_mesh_phi_block(int N, int M, int K, Block b, const double* __restrict__ in,
                                                        double* phi0)
{
    const long long n = (long long)N * M * K, NM = (long long)N * M;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(c / NM);
        const long long r = c - (long long)k * NM;
        const int j = (int)(r / N), i = (int)(r - (long long)j * N);
        phi0[c] = (i >= b.hs && i < b.hf && j >= b.vs && j < b.vf) ? in[c] : 0.0;
        (void)k;
    }
}

// cell index of the t-th block cell
__device__ __forceinline__ bool block_cell(long long t, int N, int M, int K, Block b, long long& c, int& k)
{
    const int bx = b.hf - b.hs, by = b.vf - b.vs;
    const long long per = (long long)bx * by;
    if (t >= per * K) return false;
    k = (int)(t / per);
    const long long r = t - (long long)k * per;
    const int j = b.vs + (int)(r / bx), i = b.hs + (int)(r - (long long)(r / bx) * bx);
    c = i + (long long)N * j + (long long)N * M * k;
    return true;
}

// one fixed-point sweep of the oscillation fix; *changed counts cells whose
// value moved (bitwise)
__global__ void __launch_bounds__(256) k_mesh_osc(int N, int M, int K, Block b, const double* __restrict__ phi0,
                                                  const double* __restrict__ cur, double* __restrict__ nxt,
                                                  unsigned int* changed)
{
    long long c;
    int k;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (!block_cell(t, N, M, K, b, c, k)) return;
    const double v = osc_fixed(c, k > 0 && k < K - 1, N, (long long)N * M, phi0, cur);
    if (__double_as_longlong(v) != __double_as_longlong(cur[c])) atomicAdd(changed, 1u);
    nxt[c] = v;
}

__global__ void __launch_bounds__(256) k_mesh_alpha_types(int N, int M, int K, Block b, const double* __restrict__ phi,
                                                          double* alpha, int* side, int* type)
{
    long long c;
    int k;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (!block_cell(t, N, M, K, b, c, k)) return;
    alpha_cell(c, k, K, N, (long long)N * M, phi, alpha);
    types_cell(c, k, K, N, (long long)N * M, phi, side, type);
}

__global__ void __launch_bounds__(256) k_mesh_theta(int N, int M, int K, Block b, const int* __restrict__ side,
                                                    const double* __restrict__ alpha, double* theta)
{
    long long c;
    int k;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (!block_cell(t, N, M, K, b, c, k)) return;
    theta_cell(c, k, K, N, (long long)N * M, side, alpha, theta);
}

__global__ void __launch_bounds__(256) k_mesh_volume(int N, int M, int K, const int* __restrict__ type,
                                                     const double* __restrict__ delta, const double* __restrict__ theta,
                                                     const double* __restrict__ alpha, double* vof, double* inv_vof)
{
    const long long n = (long long)N * M * K, NM = (long long)N * M;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const double v = volume_cell(c, type[c], N, NM, delta, theta, alpha);
        vof[c] = v;
        inv_vof[c] = inverse_volume(v);
    }
}

// the three staggered grids' types, volumes M = (V_P + V_E) / 2 and 1 / M
__global__ void __launch_bounds__(256) k_mesh_staggered(int N, int M, int K, const int* __restrict__ type,
                                                        const double* __restrict__ theta,
                                                        const double* __restrict__ vof, int* tx, int* ty, int* tz,
                                                        double* vx, double* vy, double* vz, double* ix, double* iy,
                                                        double* iz)
{
    const long long n = (long long)N * M * K, NM = (long long)N * M;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(c / NM);
        const long long r = c - (long long)k * NM;
        const int j = (int)(r / N), i = (int)(r - (long long)j * N);
        if (i < N - 1) {
            const long long s = c - j - (long long)k * M;      // x-grid index
            tx[s] = staggered_type(type[c], type[c + 1], theta[3 * c]);
            const double m = mul(0.5, add(vof[c], vof[c + 1]));
            vx[s] = m;
            ix[s] = inverse_volume(m);
        }
        if (j < M - 1) {
            const long long s = c - (long long)k * N;          // y-grid index
            ty[s] = staggered_type(type[c], type[c + N], theta[3 * c + 1]);
            const double m = mul(0.5, add(vof[c], vof[c + N]));
            vy[s] = m;
            iy[s] = inverse_volume(m);
        }
        if (k < K - 1) {
            tz[c] = staggered_type(type[c], type[c + NM], theta[3 * c + 2]);
            const double m = mul(0.5, add(vof[c], vof[c + NM]));
            vz[c] = m;
            iz[c] = inverse_volume(m);
        }
    }
}
// immersed-boundary face areas and inverse distances of every cell
__global__ void __launch_bounds__(256) k_mesh_ib(int N, int M, int K, const int* __restrict__ type,
                                                 const int* __restrict__ side, const double* __restrict__ theta,
                                                 const double* __restrict__ alpha, const double* __restrict__ delta,
                                                 double* en, double* ws, double* nb, double* st, double* mx,
                                                 double* ne, double* tn)
{
    const long long n = (long long)N * M * K, NM = (long long)N * M;
    double* arr[5] = {en, ws, nb, st, mx};
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        double o[15];
#pragma unroll
        for (int q = 0; q < 15; q++) o[q] = 0.0;
        dib_cell(c, type[c], side[3 * c + 2], N, NM, theta, delta, o);
#pragma unroll
        for (int a = 0; a < 5; a++)
#pragma unroll
            for (int q = 0; q < 3; q++) arr[a][3 * c + q] = o[3 * a + q];
        inv_dib_cell(c, type[c], side, alpha, delta, N, NM, ne, tn);
    }
}
#endif  // __CUDACC__

}  // namespace mesh
}  // namespace lsg
