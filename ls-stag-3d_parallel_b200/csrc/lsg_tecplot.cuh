// Tecplot solution file of the reference's SolTecplotPrinter::printField
// (Base/TecplotPrinters/sol_tecplot_printer.h:254-355), host code.
//
// The printer walks the (N+2) x (M+2) x (K+2) point grid layer by layer
// (bottom plane, the K cell layers, top plane), row by row (south wall, the
// rows, north wall) and point by point (west boundary, the cells, east
// boundary), carrying running indices into the base grid (num), the x-grid
// (num2), the y-grid (num3), the inflow profile (numW) and the node array
// (cur); the pressure of a point is the base-grid value last read, and a
// point is printed with ostream's default formatting of a double, which is
// printf's %g.  The walk below keeps those indices and that order, so the
// bytes equal the reference's file.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <thread>
#include <vector>

namespace lsg {

struct TecplotSol {
    int N, M, K, NM, NMK, xN, yM, zK;
    const double *nd, *de, *th, *u, *v, *w, *p, *uw;
    const int* ct;
    double U_W, U_E, U_S, U_N, U_B, U_T, V_W, V_E, V_S, V_N, V_B, V_T, W_W, W_E, W_S, W_N, W_B, W_T;
    bool flow;
    long long num = 0, num2 = 0, num3 = 0, numW = 0, cur = 0;
    double tx = 0, ty = 0, tz = 0, tP = 0, Ux = 0, Uy = 0, Uz = 0;
    std::string out;
    bool emit = true;   // false: the walk only advances the indices (the dry pass)

    static constexpr int kSolid = 0, kFluid = 11111111;
    static constexpr double kEq = 1e-5;   // EQ_DOUBLE (Base/ls_stag_real_constants.h)

    void setP() { tP = p[num]; }
    void node()
    {
        if (!emit) return;
        const double U = std::sqrt(Ux * Ux + Uy * Uy + Uz * Uz);
        char buf[256];
        const int len = std::snprintf(buf, sizeof buf, "%g %g %g %g %g %g %g %g\n", tx, ty, tz, tP, Ux, Uy, Uz, U);
        out.append(buf, (size_t)len);
    }
    double X(long long c) const { return nd[3 * c]; }
    double Y(long long c) const { return nd[3 * c + 1]; }
    double Z(long long c) const { return nd[3 * c + 2]; }

    void wall(double V, double U, double W)                      // PrintWall
    {
        tx = 0.0;
        setP();
        Ux = U;
        Uy = V;
        Uz = W;
        node();
        for (int i = 0; i < N; i++, num++, cur++) {
            tx = X(cur);
            setP();
            node();
        }
        tx += 0.5 * de[3 * (num - 1)];
        node();
    }
    void wall_plane(double V, double U, double W)                // PrintWallPlane
    {
        ty = 0.0;
        wall(V, U, W);
        num -= N;
        cur -= N;
        for (int ii = 0; ii < M; ii++) {
            tx = 0.0;
            ty = Y(cur);
            wall(V, U, W);
        }
        num -= N;
        cur -= N;
        ty += 0.5 * de[3 * num + 1];
        wall(V, U, W);
    }
    void west(double V, double W, double W2)                     // PrintWest
    {
        ty = Y(cur);
        tx = 0.0;
        setP();
        Ux = uw ? uw[numW] : 0.0;
        Uy = V_W;
        Uz = W_W;
        node();
        tx = X(cur);
        Ux = uw ? 0.5 * (u[num2] + uw[numW]) : 0.0;
        Uy = 0.5 * (v[num3] + V);
        Uz = 0.5 * (W2 + W);
        node();
        num++;
        numW++;
        num3++;
        cur++;
        num2++;
    }
    void east(double V, double W, double W2)                     // PrintEast
    {
        tx = X(cur);
        setP();
        Ux = flow ? u[num2 - 1] : 0.5 * (u[num2 - 1] + U_E);
        Uy = 0.5 * (v[num3] + V);
        Uz = 0.5 * (W2 + W);
        node();
        tx += 0.5 * de[3 * num];
        if (!flow) {
            Ux = U_E;
            Uy = V_E;
            Uz = W_E;
        }
        node();
        num++;
        num3++;
        cur++;
    }
    void edge(double V, double W, double W2)                     // PrintEdge
    {
        west(V, W, W2);
        for (int i = 1; i < xN; i++, num++, cur++, num2++, num3++) {
            tx = X(cur);
            setP();
            Ux = 0.5 * (u[num2] + u[num2 - 1]);
            Uy = 0.5 * (v[num3] + V);
            Uz = 0.5 * (W2 + W);
            node();
        }
        east(V, W, W2);
    }
    static double cell_value(double ta, double va, double tb, double vb)   // cellValue
    {
        const double s = ta + tb;
        return (s > kEq) ? ((ta * va + tb * vb) / s) : 0.0;
    }
    // the cells of one row; layer 0 bottom (w below = W_B, both apertures
    // theta_z of the cell), 1 interior, 2 top (w above = W_T, w below at num - NM)
    void interior_row(int layer)
    {
        for (int i = 1; i < xN; i++, num++, num2++, num3++, cur++) {
            tx = X(cur);
            setP();
            const int t = ct[num];
            double wa, wb, ta, tb;
            if (layer == 0) {
                wa = w[num];
                wb = W_B;
                ta = tb = th[3 * num + 2];
            } else if (layer == 1) {
                wa = w[num];
                wb = w[num - NM];
                ta = th[3 * num + 2];
                tb = th[3 * (num - NM) + 2];
            } else {
                wa = w[num - NM];
                wb = W_T;
                ta = tb = th[3 * num + 2];
            }
            if (t == kSolid) {
                Ux = Uy = Uz = 0.0;
            } else if (t == kFluid) {
                Ux = 0.5 * (u[num2] + u[num2 - 1]);
                Uy = 0.5 * (v[num3] + v[num3 - N]);
                Uz = 0.5 * (wa + wb);
            } else {
                Ux = cell_value(th[3 * num], u[num2], th[3 * (num - 1)], u[num2 - 1]);
                Uy = cell_value(th[3 * num + 1], v[num3], th[3 * (num - N) + 1], v[num3 - N]);
                Uz = cell_value(ta, wa, tb, wb);
            }
            node();
        }
    }
    void layer_b(bool asB)                                       // printWallLayerB
    {
        num = num2 = num3 = numW = 0;
        cur = 0;
        ty = 0.0;
        tz = asB ? 0.0 : Z(cur);
        wall(V_S, U_S, W_S);
        num = 0;
        cur = 0;
        edge(V_S, W_B, w[num]);
        for (int j = 1; j < yM; j++) {
            west(v[num3 - N], W_B, w[num]);
            num2 = num - j;
            num3 = num;
            interior_row(0);
            east(v[num3 - N], W_B, w[num]);
        }
        num3 -= N;
        edge(V_N, W_B, w[num]);
        num -= N;
        cur -= N;
        tx = 0.0;
        ty += 0.5 * de[3 * num + 1];
        wall(V_N, U_N, W_N);
    }
    void layer_t(bool asT)                                       // printWallLayerT
    {
        if (asT) {
            const long long nT = (long long)NMK - NM;
            ty = 0.0;
            tz = Z(nT) + 0.5 * de[3 * nT + 2];
        } else {
            ty = 0.0;
            tz = Z(cur);
        }
        wall(V_S, U_S, W_S);
        num -= N;
        cur -= N;
        edge(V_S, w[num - NM], W_T);
        for (int j = 1; j < yM; j++) {
            west(v[num3 - N], w[num - NM], W_T);
            num2 = num - (j + (long long)zK * M);
            num3 = num - (long long)zK * N;
            interior_row(2);
            east(v[num3 - N], w[num - NM], W_T);
        }
        num3 -= N;
        edge(V_N, w[num - NM], W_T);
        num -= N;
        cur -= N;
        tx = 0.0;
        ty += 0.5 * de[3 * num + 1];
        wall(V_N, U_N, W_N);
    }
    // the walk after the header is K + 2 segments, one per printed layer:
    // 0 the bottom plane, 1 the first cell layer, 2 .. K-1 the interior
    // layers, K the last cell layer, K + 1 the top plane; each starts from
    // the running indices the previous one left (the top plane from those
    // the last cell layer started with)
    void segment(int sg)
    {
        if (sg == 0) {
            if (flow)
                layer_b(true);
            else
                wall_plane(V_B, U_B, W_B);
        } else if (sg == 1) {
            layer_b(false);
        } else if (sg <= zK) {
            const int k = sg - 1;
            ty = 0.0;
            tz = Z(cur);
            wall(V_S, U_S, W_S);
            num -= N;
            cur -= N;
            edge(V_S, w[num - NM], w[num]);
            for (int j = 1; j < yM; j++) {
                west(v[num3 - N], w[num - NM], w[num]);
                num2 = num - (j + (long long)k * M);
                num3 = num - (long long)k * N;
                interior_row(1);
                east(v[num3 - N], w[num - NM], w[num]);
            }
            num3 -= N;
            edge(V_N, w[num - NM], w[num]);
            num -= N;
            cur -= N;
            tx = 0.0;
            ty += 0.5 * de[3 * num + 1];
            wall(V_N, U_N, W_N);
        } else if (sg == zK + 1) {
            layer_t(false);
        } else if (flow) {
            layer_t(true);
        } else {
            const long long nT = (long long)NMK - NM;
            tz = Z(nT) + 0.5 * de[3 * nT + 2];
            wall_plane(V_T, U_T, W_T);
        }
    }
    struct State {
        long long num, num2, num3, numW, cur;
        double tx, ty, tz, tP, Ux, Uy, Uz;
    };
    State state() const { return {num, num2, num3, numW, cur, tx, ty, tz, tP, Ux, Uy, Uz}; }
    void set_state(const State& q)
    {
        num = q.num;
        num2 = q.num2;
        num3 = q.num3;
        numW = q.numW;
        cur = q.cur;
        tx = q.tx;
        ty = q.ty;
        tz = q.tz;
        tP = q.tP;
        Ux = q.Ux;
        Uy = q.Uy;
        Uz = q.Uz;
    }
    static std::string header(int N, int M, int K)
    {
        std::string h = "TITLE     = \"Velocity Vectors\" \n";
        h += "VARIABLES = \"x\" \n";
        for (const char* name : {"y", "z", "P", "SPD_x", "SPD_y", "SPD_z", "SPD"}) {
            h += "\"";
            h += name;
            h += "\"\n";
        }
        h += "ZONE T=\"Data\" \n";
        char buf[96];
        std::snprintf(buf, sizeof buf, "I=%d, J=%d, K=%d, F=POINT\n", N + 2, M + 2, K + 2);
        h += buf;
        return h;
    }
};

// The file's bytes: a dry pass records the running indices at the start of
// every segment, then groups of consecutive segments are formatted on up
// to `threads` threads and joined in order (the same bytes as one walk).
inline std::string tecplot_sol_text(const TecplotSol& proto, int threads)
{
    const int nseg = proto.K + 2;
    std::vector<TecplotSol::State> start((size_t)nseg + 1);
    TecplotSol dry = proto;
    dry.emit = false;
    dry.tx = dry.ty = dry.tz = 0.0;
    dry.num = dry.cur = 0;
    for (int sg = 0; sg < nseg; sg++) {
        start[(size_t)sg] = dry.state();
        if (sg == nseg - 1) dry.set_state(start[(size_t)nseg - 2]);   // the top plane restarts from the last layer
        dry.segment(sg);
    }
    start[(size_t)nseg - 1] = start[(size_t)nseg - 2];
    const int nt = std::max(1, std::min(threads, nseg));
    std::vector<std::string> parts((size_t)nt);
    auto work = [&](int t) {
        const int s0 = (int)((long long)nseg * t / nt), s1 = (int)((long long)nseg * (t + 1) / nt);
        TecplotSol w = proto;
        w.emit = true;
        w.out.clear();
        w.out.reserve((size_t)(s1 - s0) * (w.N + 2) * (w.M + 2) * 72);
        for (int sg = s0; sg < s1; sg++) {
            w.set_state(start[(size_t)sg]);
            w.segment(sg);
        }
        parts[(size_t)t] = std::move(w.out);
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; t++) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
    std::string out = TecplotSol::header(proto.N, proto.M, proto.K);
    size_t total = out.size();
    for (const auto& s : parts) total += s.size();
    out.reserve(total);
    for (const auto& s : parts) out += s;
    return out;
}

// the file's bytes for host arrays (bc: U_W U_E U_S U_N U_B U_T, V_W .. V_T, W_W .. W_T)
inline std::string tecplot_sol_bytes(int N, int M, int K, const double* nodes, const double* delta,
                                     const double* theta, const int* celltype, const double* u, const double* v,
                                     const double* w, const double* p, const double* u_w, const double* bc, bool flow)
{
    TecplotSol t;
    t.N = N;
    t.M = M;
    t.K = K;
    t.NM = N * M;
    t.NMK = N * M * K;
    t.xN = N - 1;
    t.yM = M - 1;
    t.zK = K - 1;
    t.nd = nodes;
    t.de = delta;
    t.th = theta;
    t.ct = celltype;
    t.u = u;
    t.v = v;
    t.w = w;
    t.p = p;
    t.uw = u_w;
    double* f[18] = {&t.U_W, &t.U_E, &t.U_S, &t.U_N, &t.U_B, &t.U_T, &t.V_W, &t.V_E, &t.V_S,
                     &t.V_N, &t.V_B, &t.V_T, &t.W_W, &t.W_E, &t.W_S, &t.W_N, &t.W_B, &t.W_T};
    for (int i = 0; i < 18; i++) *f[i] = bc[i];
    t.flow = flow;
    const unsigned hc = std::thread::hardware_concurrency();
    return tecplot_sol_text(t, (int)std::min(hc ? hc : 1u, 16u));
}

}  // namespace lsg
