/*
 * ref_harness.cpp -- TEST INFRASTRUCTURE (the oracle), never part of the product.
 *
 * Drives the reference LS-STAG-3D CPU/OpenMP code (compiled from its own
 * headers by oracle/build_ref.sh) on the synthetic cases the product is
 * measured on, and dumps everything the parity tests compare against:
 *   geometry (cell types, theta, delta, VOF, 1/M_x,y,z), the Laplace CSR
 *   (laplace_discrete_operator.h:107-686, fixPoint :809-821), the right-hand
 *   side, the multigrid hierarchy (coarse_grid.h:93-106: P, R, A_H, ADLJ
 *   factors, coarse LU), one V-cycle (multigrid_solver.h:48-75), one
 *   MG-FGMRES solve (fgmres_interface.h:78-142) and one ILU(0)-BiCGStab
 *   solve (bicgstab_interface.h:76-111).
 *
 * Geometry: a uniform staggered grid built through the reference's own zoned
 * mesh (ls_stag_mesh.h) with a single zone, and the reference's level-set
 * machinery (FlowTaskDescription::buildBaseMesh, flow_task_description.h).
 * The level set is evaluated exactly like calcLevelSetSphere
 * (flow_sphere_task_description.h:57-74): at the upper cell corner, phi > 0
 * inside a body; several bodies are merged by max (i.e. min of |x-c|-r).
 *
 * Usage: ref_harness <config.txt> <outdir>
 * The config is a whitespace separated key/value list written by
 * oracle/ref_runner.py.  Every dumped array is raw little-endian binary with
 * a line in <outdir>/manifest.txt: "<name> <dtype> <count>".
 */
#include "stdafx.h"
#include "TimeSteppingMethod/time_stepping_method_interface.h"
#include "Base/Solvers/BiCGStab/ilu_bicgstab.h"
#include <chrono>
#include <fstream>
#include <filesystem>
#include <map>
#include <random>
#include <sstream>
#include <vector>

using namespace LS_STAG;

namespace {

struct Body {
    int kind = 0;          // 0 sphere, 1 ellipsoid
    double c[3] = {0, 0, 0};
    double r = 0.0;        // sphere radius
    double ax[3] = {1, 1, 1};   // ellipsoid semi-axes
    double rot[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};  // body frame = rot * (x - c)
    double phi(double x, double y, double z) const
    {
        const double qx = x - c[0], qy = y - c[1], qz = z - c[2];
        if (kind == 0) return r - sqrt(qx * qx + qy * qy + qz * qz);
        const double bx = rot[0] * qx + rot[1] * qy + rot[2] * qz;
        const double by = rot[3] * qx + rot[4] * qy + rot[5] * qz;
        const double bz = rot[6] * qx + rot[7] * qy + rot[8] * qz;
        const double s = sqrt((bx / ax[0]) * (bx / ax[0]) + (by / ax[1]) * (by / ax[1]) +
                              (bz / ax[2]) * (bz / ax[2]));
        // scaled distance-like function, zero on the surface, > 0 inside
        const double amin = std::min(ax[0], std::min(ax[1], ax[2]));
        return (1.0 - s) * amin;
    }
    void bbox(double lo[3], double hi[3]) const
    {
        const double e = (kind == 0) ? r : std::max(ax[0], std::max(ax[1], ax[2]));
        for (int d = 0; d < 3; d++) { lo[d] = c[d] - e; hi[d] = c[d] + e; }
    }
};

struct Config {
    std::map<std::string, std::string> kv;
    std::vector<Body> bodies;
    double get(const std::string& k, double d) const
    {
        auto it = kv.find(k);
        return it == kv.end() ? d : atof(it->second.c_str());
    }
    std::string gets(const std::string& k, const std::string& d) const
    {
        auto it = kv.find(k);
        return it == kv.end() ? d : it->second;
    }
};

Config readConfig(const char* path)
{
    Config c;
    std::ifstream in(path);
    std::string key;
    while (in >> key) {
        if (key == "body") {
            Body b;
            in >> b.kind >> b.c[0] >> b.c[1] >> b.c[2];
            if (b.kind == 0) in >> b.r;
            else {
                in >> b.ax[0] >> b.ax[1] >> b.ax[2];
                for (int i = 0; i < 9; i++) in >> b.rot[i];
            }
            c.bodies.push_back(b);
        } else {
            std::string v;
            in >> v;
            c.kv[key] = v;
        }
    }
    return c;
}

/* Uniform-grid flow task over bodies given by level sets.  Subclasses the
   reference FlowTaskDescription exactly like FlowSphereTaskDescription does
   (flow_sphere_task_description.h:41-153), replacing the zoned step table
   with one zone of step h in every direction. */
struct HarnessTask : FlowTaskDescription {
    LSSTAGMesh mesh;
    int gN, gM, gK;
    double hx, hy, hz;
    std::vector<Body> bodies;
    HarnessTask()
        : FlowTaskDescription(AIRFOIL_SPHERE, MOTION_NO, (LSSTAGUniformMesh*)&mesh, sizeof(HarnessTask)),
          gN(8), gM(8), gK(8), hx(1), hy(1), hz(1)
    {
        discontin = 0;
        ibCount = 1;
        useNNM = 0;
        needXYMesh = 0;
        useTM = 0;
        continueSolveTask = 0;
        PeriodPrintSol = 1e30;
        PeriodPrintRotor = 0.0;
        PeriodSaveState = 1e30;
    }
    double loadsCoef() const { return fcoef; }
    void calcNodesCount() override
    {
        mesh.baseMesh.N = gN;
        mesh.baseMesh.M = gM;
        mesh.baseMesh.K = gK;
    }
    void initMeshParams() override
    {
        FlowTaskDescription::initMeshParams();
        for (int k = 0; k < LSSTAGMesh::ZONES_COUNT; k++) mesh.zone[k].set(0, 0, 0);
        mesh.zone[3].x = gN;  // ZONE_ORDER_X[3] = 0 -> deltaCurZone[0].x
        mesh.zone[2].y = gM;  // deltaOrder[0][2] = 0 -> deltaCurZone[0].y
        mesh.zone[2].z = gK;
        for (int d = 0; d < LSSTAGMesh::DELTA_COUNT; d++) mesh.deltaCurZone[d].set(hx, hy, hz);
        mesh.maxCountCutCells = gN * gM * gK;
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (const Body& b : bodies) {
            double l[3], h[3];
            b.bbox(l, h);
            for (int d = 0; d < 3; d++) { lo[d] = std::min(lo[d], l[d]); hi[d] = std::max(hi[d], h[d]); }
        }
        // LS block as in FlowSphereTaskDescription::initMeshParams, kept >= 5
        // cells from the walls: buildBaseMesh widens it by 3 and the row walks
        // of calcTypeOfCells (flow_task_description.h) need >= 2 plain cells
        // on each side of the widened block.  Bodies must lie inside it.
        mesh.hs = std::max(5, (int)floor(lo[0] / hx));
        mesh.hf = std::min(gN - 5, (int)floor(hi[0] / hx) + 1);
        mesh.vs = std::max(5, (int)floor(lo[1] / hy));
        mesh.vf = std::min(gM - 5, (int)floor(hi[1] / hy) + 1);
        H_BASE = 1.0;
    }
    void buildLS(const int zs, const int zf, const int vs, const int vf, const int hs, const int hf) override
    {
        const int N = mesh.baseMesh.N, NM = N * mesh.baseMesh.M;
        for (int k = zs; k < zf; k++)
            for (int j = vs; j < vf; j++) {
                // same point walk as calcLevelSetSphere: corner = node + delta/2, then += delta.x
                int num = NM * k + N * j + hs;
                coordinate p = mesh.nodes[num];
                coordinate* d = mesh.delta + num;
                p.add(0.5 * d->x, 0.5 * d->y, 0.5 * d->z);
                for (int end = NM * k + N * j + hf; num < end; num++) {
                    double f = -1e300;
                    for (const Body& b : bodies) f = std::max(f, b.phi(p.x, p.y, p.z));
                    mesh.phi[num] = f;
                    d++;
                    p.x += d->x;
                }
            }
        // the level set as evaluated, before calcAlpha's oscillation fix
        // (checkOscLS, ls_stag_uniform_mesh.h:2906-2916) edits it in place
        const long n = (long)N * mesh.baseMesh.M * mesh.baseMesh.K;
        phi_ls.assign(mesh.phi, mesh.phi + n);
    }
    std::vector<double> phi_ls;
    // the block FlowTaskDescription::buildBaseMesh walks (its hs_loc .. vf_loc:
    // the level-set block widened by 3 cells, flow_task_description.h:388-398)
    void lsBlock(int b[4]) const { b[0] = mesh.hs - 3; b[1] = mesh.hf + 3; b[2] = mesh.vs - 3; b[3] = mesh.vf + 3; }
};

/* The momentum operators with their immersed-boundary source term made
   callable (ibFlux is run by the reference only for moving bodies). */
struct HelmXProbe : HelmholtzDiscreteOperatorX {
    void runIbFlux() { ibRecalcFlux = true; calcFlux(); }
};
struct HelmYProbe : HelmholtzDiscreteOperatorY {
    void runIbFlux() { ibRecalcFlux = true; calcFlux(); }
};
struct HelmZProbe : HelmholtzDiscreteOperatorZ {
    void runIbFlux() { ibRecalcFlux = true; calcFlux(); }
};

struct Dumper {
    std::string dir;
    std::ofstream man;
    explicit Dumper(const std::string& d) : dir(d), man(d + "/manifest.txt") {}
    template <typename T>
    void put(const std::string& name, const T* p, long n, const char* dt)
    {
        std::ofstream f(dir + "/" + name + ".bin", std::ios::binary);
        f.write((const char*)p, sizeof(T) * n);
        man << name << " " << dt << " " << n << "\n";
        man.flush();
    }
    void d(const std::string& name, const double* p, long n) { put(name, p, n, "f8"); }
    void i(const std::string& name, const int* p, long n) { put(name, p, n, "i4"); }
    void csr(const std::string& name, SparseMatrix* A)
    {
        const int n = A->NMK;
        const int nnz = A->Number[n];
        i(name + "_rowptr", A->Number, n + 1);
        i(name + "_col", A->Portrait, nnz);
        d(name + "_val", A->Cell, nnz);
        int dims[4] = {A->m_N, A->m_M, A->m_K, A->NMK};
        i(name + "_dims", dims, 4);
    }
    void scalar(const std::string& name, double v) { d(name, &v, 1); }
};

double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

/* Same accessors as the reference's private members need: MultiGridSolver
   exposes grids/LU publicly through CoarseGridsHierarchy. */
void dumpHierarchy(Dumper& out, MultiGridSolver& mg)
{
    int nl = mg.numMG;
    out.i("mg_nlev", &nl, 1);
    for (int l = 0; l < nl; l++) {
        CoarseGrid& g = mg.grids[l];
        std::string p = "mg" + std::to_string(l) + "_";
        out.csr(p + "P", &g.P);
        out.csr(p + "R", (SparseMatrix*)&g.R);
        out.csr(p + "AH", (SparseMatrix*)&g.AH);
        int par[3] = {g.oddN, g.oddM, g.oddK};
        out.i(p + "odd", par, 3);
        const int n = g.m_A->NMK;
        SmootherADLJ& s = g.ADLJ;
        out.d(p + "xc", s.ADLJ_x.c, n - 1);
        out.d(p + "xd", s.ADLJ_x.d, n);
        out.d(p + "xe", s.ADLJ_x.e, n - 1);
        out.d(p + "yc", s.ADLJ_y.c, n - 1);
        out.d(p + "yd", s.ADLJ_y.d, n);
        out.d(p + "ye", s.ADLJ_y.e, n - 1);
        out.d(p + "zc", s.ADLJ_z.c, n - 1);
        out.d(p + "zd", s.ADLJ_z.d, n);
        out.d(p + "ze", s.ADLJ_z.e, n - 1);
    }
}

/* Reference solvers on an operator given as seven coefficient planes
   (b, s, w, p, e, n, t of the reference's CSR order; raw f8 file of 7*n
   values) and a right-hand side: the CPU-baseline mode.  The CSR holds every
   in-grid neighbour (explicit zeros included), like the reference's portrait
   for fluid rows (sym_discrete_operator.h). */
int solvePlanes(const Config& cfg, const std::string& outdir)
{
    const int N = (int)cfg.get("N", 0), M = (int)cfg.get("M", 0), K = (int)cfg.get("K", 0);
    const long n = (long)N * M * K;
    std::vector<double> planes(7 * n), b(n);
    {
        std::ifstream f(cfg.gets("planes_in", ""), std::ios::binary);
        f.read((char*)planes.data(), sizeof(double) * 7 * n);
        std::ifstream g(cfg.gets("rhs", ""), std::ios::binary);
        g.read((char*)b.data(), sizeof(double) * n);
        if (!f || !g) { fprintf(stderr, "cannot read planes/rhs\n"); return 3; }
    }
    const int NM = N * M;
    const int offs[7] = {-NM, -N, -1, 0, 1, N, NM};
    SparseMatrix* A = new SparseMatrix;
    A->set(N, M, K, (int)n);
    std::vector<int> cols;
    std::vector<double> vals;
    cols.reserve(7 * n);
    vals.reserve(7 * n);
    A->Number[0] = 0;
    for (long i = 0; i < n; i++) {
        const int z = (int)(i / NM), y = (int)((i - (long)z * NM) / N), x = (int)(i - (long)z * NM - (long)y * N);
        const bool ok[7] = {z > 0, y > 0, x > 0, true, x < N - 1, y < M - 1, z < K - 1};
        for (int s = 0; s < 7; s++)
            if (ok[s]) { cols.push_back((int)(i + offs[s])); vals.push_back(planes[(size_t)s * n + i]); }
        A->Number[i + 1] = (int)cols.size();
    }
    A->resize();
    A->maxElemCount = A->elemCount;
    A->reserve();
    std::copy(cols.begin(), cols.end(), A->Portrait);
    std::copy(vals.begin(), vals.end(), A->Cell);
    HarnessTask* task = new HarnessTask;
    task->FGMRES_RESTART_NUM = (int)cfg.get("restart", 30);
    task->MAX_ITER = (int)cfg.get("max_it", 200);
    task->n_post = (int)cfg.get("n_post", BaseTaskDescription::DEFAULT_N_POST);
    double bnorm = 0.0;
    for (long i = 0; i < n; i++) bnorm += b[i] * b[i];
    bnorm = sqrt(bnorm);
    task->eps = cfg.get("abs_tol", cfg.get("rel_tol", 1e-10) * bnorm);
    Dumper out(outdir);
    out.scalar("eps", task->eps);
    const int reps = (int)cfg.get("repeats", 1);
    std::vector<double> x(n, 0.0);
    const char* names[2] = {"fgmres", "bicgstab"};
    for (int which = 0; which < 2; which++) {
        if (!(int)cfg.get(names[which], which == 0 ? 1 : 0)) continue;
        IterativeSolverInterface* s = which == 0 ? (IterativeSolverInterface*)new MGFGMRES
                                                 : (IterativeSolverInterface*)new ILUBiCGStab;
        double tset = now_s();
        s->set(A, b.data(), x.data(), task);
        tset = now_s() - tset;
        s->eps = task->eps;
        std::vector<double> ts;
        int iters = 0;
        for (int r = 0; r < reps; r++) {
            std::fill(x.begin(), x.end(), 0.0);
            double t1 = now_s();
            iters = s->solve();
            ts.push_back(now_s() - t1);
        }
        std::string p = names[which];
        out.d(p + "_x", x.data(), n);
        out.i(p + "_it", &iters, 1);
        out.scalar(p + "_norm_r", s->norm_r);
        out.d(p + "_time_s", ts.data(), (long)ts.size());
        out.scalar(p + "_setup_s", tset);
    }
    int nthreads = omp_get_max_threads();
    out.i("omp_threads", &nthreads, 1);
    return 0;
}

template <typename T>
bool readRaw(const Config& cfg, const std::string& key, std::vector<T>& v, long cnt)
{
    v.assign(cnt, T(0));
    const std::string path = cfg.gets(key, "");
    if (path.empty()) return false;
    std::ifstream f(path, std::ios::binary);
    f.read((char*)v.data(), sizeof(T) * cnt);
    return (bool)f;
}

/* The reference's per-cut-cell load kernel (LoadsCalculator::calc,
   loads_calculator.h:79-1269) and its moment kernels (:1270-1291) evaluated
   on arrays read from files: every cut-cell type is exercised on seeded
   inputs, independently of which types a geometry happens to produce.  Also
   runs the moment filter (ButterworthLowPassFilter, butterworth_low_pass_filter.h)
   on a given signal. */
int loadsProbe(const Config& cfg, const std::string& outdir)
{
    const int N = (int)cfg.get("N", 0), M = (int)cfg.get("M", 0), K = (int)cfg.get("K", 0);
    const long n = (long)N * M * K;
    const int count = (int)cfg.get("count", 0);
    std::vector<int> type, cells;
    std::vector<double> theta, delta, vib, vibyx, vibzy, dne, dtn, dmax, nodes, invv, p, ux, uy, uz, nucell, cc;
    bool ok = readRaw(cfg, "lp_type", type, n) && readRaw(cfg, "lp_cells", cells, count) &&
              readRaw(cfg, "lp_theta", theta, 3 * n) && readRaw(cfg, "lp_delta", delta, 3 * n) &&
              readRaw(cfg, "lp_vib", vib, 3 * n) && readRaw(cfg, "lp_vibyx", vibyx, 3 * n) &&
              readRaw(cfg, "lp_vibzy", vibzy, 3 * n) && readRaw(cfg, "lp_dne", dne, 3 * n) &&
              readRaw(cfg, "lp_dtn", dtn, 3 * n) && readRaw(cfg, "lp_dmax", dmax, 3 * n) &&
              readRaw(cfg, "lp_nodes", nodes, 3 * n) && readRaw(cfg, "lp_center", cc, 3) &&
              readRaw(cfg, "lp_invv", invv, n) && readRaw(cfg, "lp_p", p, n) &&
              readRaw(cfg, "lp_ux", ux, (long)(N - 1) * M * K) && readRaw(cfg, "lp_uy", uy, (long)N * (M - 1) * K) &&
              readRaw(cfg, "lp_uz", uz, (long)N * M * (K - 1));
    if (!ok) { fprintf(stderr, "cannot read loads probe inputs\n"); return 3; }
    const bool haveNu = readRaw(cfg, "lp_nucell", nucell, n);
    const double nu = cfg.get("nu", 0.01);
    std::vector<tripletInt> list(count);
    for (int i = 0; i < count; i++) {
        const int num = cells[i], k = num / (N * M), j = (num - k * N * M) / N;
        list[i].set(num - j - k * M, num - k * N, num);      // BaseTaskDescription::addCutCell
    }
    std::vector<double> fx(count), fy(count), fz(count), mz(count), mx(count), my(count);
    auto C = [](std::vector<double>& v) { return (coordinate*)v.data(); };
    for (int i = 0; i < count; i++)
        LoadsCalculator::_k_calc(i, (const CellTypes*)type.data(), list.data(), fx.data(), fy.data(), fz.data(),
                                 C(vib), C(vibyx), C(vibzy), C(delta), C(dne), C(dtn), C(dmax), C(theta),
                                 ux.data(), uy.data(), uz.data(), p.data(), invv.data(),
                                 haveNu ? nucell.data() : nullptr, nu, N, M, N * M);
    for (int i = 0; i < count; i++) {
        mz[i] = LoadsCalculator::_k_calcMoment(i, C(nodes), list.data(), fx.data(), fy.data(), C(cc));
        mx[i] = LoadsCalculator::_k_calcMomentX(i, C(nodes), list.data(), fy.data(), fz.data(), C(cc));
        my[i] = LoadsCalculator::_k_calcMomentY(i, C(nodes), list.data(), fx.data(), fz.data(), C(cc));
    }
    Dumper out(outdir);
    out.d("fx", fx.data(), count);
    out.d("fy", fy.data(), count);
    out.d("fz", fz.data(), count);
    out.d("mz", mz.data(), count);
    out.d("mx", mx.data(), count);
    out.d("my", my.data(), count);
    const int ns = (int)cfg.get("filter_len", 0);
    if (ns > 0) {
        std::vector<double> sig;
        if (!readRaw(cfg, "filter_in", sig, ns)) { fprintf(stderr, "cannot read filter input\n"); return 3; }
        ButterworthLowPassFilter flt;
        flt.init(cfg.get("dt", 0.01), DEFAULT_CUT_OFF_FREQUENCY, DEFAULT_SUPPRESSION_LEVEL);
        std::vector<double> res(ns);
        for (int i = 0; i < ns; i++) res[i] = flt.getValue(sig[i]);
        out.d("filter_out", res.data(), ns);
    }
    return 0;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 3) {
        fprintf(stderr, "usage: %s config outdir\n", argv[0]);
        return 2;
    }
    Config cfg = readConfig(argv[1]);
    const std::string outdir = argv[2];
    const int threads = (int)cfg.get("threads", 0);
    if (threads > 0) omp_set_num_threads(threads);
    if (!cfg.gets("planes_in", "").empty()) return solvePlanes(cfg, outdir);
    if ((int)cfg.get("loads_probe", 0)) return loadsProbe(cfg, outdir);

    HarnessTask* task = new HarnessTask;
    task->gN = (int)cfg.get("N", 16);
    task->gM = (int)cfg.get("M", 16);
    task->gK = (int)cfg.get("K", 16);
    task->hx = cfg.get("hx", 1.0 / task->gN);
    task->hy = cfg.get("hy", 1.0 / task->gM);
    task->hz = cfg.get("hz", 1.0 / task->gK);
    task->bodies = cfg.bodies;
    task->Re = cfg.get("Re", 100.0);
    task->t = cfg.get("dt", 0.01);
    task->T_end = cfg.get("T_end", 1.0);
    task->nu = task->V_BASE * task->L_BASE / task->Re;
    task->FGMRES_RESTART_NUM_P = (int)cfg.get("restart", 30);
    task->MAX_ITER = (int)cfg.get("max_it", 200);
    task->n_post = (int)cfg.get("n_post", BaseTaskDescription::DEFAULT_N_POST);
    task->outputDirectoryFull = outdir + "/";

    Dumper out(outdir);
    double curTime = 0.0;
    int it = 1;
    double t0 = now_s();
    task->init(&curTime);
    SetSolutions* sol = new SetSolutions;
    // print_sol: the solution printer (SolTecplotPrinter, set up by
    // SetSolutions::init) prints on its first call
    if ((int)cfg.get("print_sol", 0)) task->PeriodPrintSol = task->t;
    sol->init(task, &it);
    task->initSol(&(sol->current), &(sol->prediction), &(sol->previous));
    if ((int)cfg.get("flux_perturb", 0)) {
        // nonzero boundary and immersed-boundary velocities, so that every term
        // of the Laplace source (inflow profile, outflow, N/S and T/B walls,
        // immersed boundary) contributes; all inputs are dumped below
        LSSTAGUniformMesh* mm = task->m_mesh;
        const long nb = (long)mm->baseMesh.N * mm->baseMesh.M * mm->baseMesh.K;
        for (long j = 0; j < (long)mm->baseMesh.M * mm->baseMesh.K; j++) task->pU_W[j] = 1.0 + 0.1 * sin(0.37 * j);
        task->U_E = 0.9;
        task->V_S = 0.05;
        task->V_N = -0.07;
        task->W_B = 0.03;
        task->W_T = -0.02;
        for (long i = 0; i < nb; i++)
            mm->v_ib[i].set(0.1 * sin(0.11 * i), 0.1 * cos(0.13 * i), 0.05 * sin(0.17 * i));
        for (long i = 0; i < (long)mm->xMesh.NMK; i++) mm->m_Ux[i] = 1.0 + 0.2 * sin(0.29 * i);
    }
    if ((int)cfg.get("mesh_dump", 0)) {
        // the whole mesh build of the flow task (BaseTaskDescription::buildMesh,
        // base_task_description.h:330-371): level set as evaluated, level set
        // after the oscillation fix, edge fractions alpha, face types, cell
        // types, face fractions theta, cell volumes, staggered types, volumes
        // and inverse volumes, with the level-set block the walks used
        LSSTAGUniformMesh* mm = task->m_mesh;
        const int N = mm->baseMesh.N, M = mm->baseMesh.M, K = mm->baseMesh.K;
        const long n = (long)N * M * K;
        const long ns[3] = {(long)mm->xMesh.NMK, (long)mm->yMesh.NMK, (long)mm->zMesh.NMK};
        int dd[3] = {N, M, K};
        out.i("dims", dd, 3);
        int blk[4];
        task->lsBlock(blk);
        out.i("ls_block", blk, 4);
        double hh[3] = {task->hx, task->hy, task->hz};
        out.d("h", hh, 3);
        out.d("phi_ls", task->phi_ls.data(), n);
        out.d("phi", mm->phi, n);
        out.d("alpha", (const double*)mm->alpha, 3 * n);
        out.i("side_type", (const int*)mm->baseSideTypes, 3 * n);
        out.i("celltype", (const int*)mm->baseMesh.typeOfCell, n);
        out.d("theta", (const double*)mm->theta, 3 * n);
        out.d("delta", (const double*)mm->delta, 3 * n);
        out.d("nodes", (const double*)mm->nodes, 3 * n);
        out.d("vof", mm->baseMesh.VOF, n);
        out.d("inv_vof", mm->baseMesh.inv_VOF, n);
        out.i("xtype", (const int*)mm->xMesh.typeOfCell, ns[0]);
        out.i("ytype", (const int*)mm->yMesh.typeOfCell, ns[1]);
        out.i("ztype", (const int*)mm->zMesh.typeOfCell, ns[2]);
        out.d("vof_x", mm->xMesh.VOF, ns[0]);
        out.d("vof_y", mm->yMesh.VOF, ns[1]);
        out.d("vof_z", mm->zMesh.VOF, ns[2]);
        out.d("inv_mx", mm->xMesh.inv_VOF, ns[0]);
        out.d("inv_my", mm->yMesh.inv_VOF, ns[1]);
        out.d("inv_mz", mm->zMesh.inv_VOF, ns[2]);
        out.d("dib_en", (const double*)mm->delta_ib_en, 3 * n);
        out.d("dib_ws", (const double*)mm->delta_ib_ws, 3 * n);
        out.d("dib_nb", (const double*)mm->delta_ib_nb, 3 * n);
        out.d("dib_st", (const double*)mm->delta_ib_st, 3 * n);
        out.d("dib_max", (const double*)mm->delta_ib_max, 3 * n);
        out.d("inv_dib_ne", (const double*)mm->inv_delta_ib_ne, 3 * n);
        out.d("inv_dib_tn", (const double*)mm->inv_delta_ib_tn, 3 * n);
        return 0;
    }
    if ((int)cfg.get("flow_steps", 0) || (int)cfg.get("flow_setup", 0)) {
        // whole time steps of the flow task as TimeSteppingMethodInterface::init
        // and ::step run them (time_stepping_method_interface.h:150-214: the
        // three momentum equations, the pressure equation, the projection),
        // with every input of the GPU path and the state after each step
        // dumped; no start-up pressure scaling (tScaleP < 0), solver
        // tolerance task_eps (absolute)
        LSSTAGUniformMesh* mm = task->m_mesh;
        const int N = mm->baseMesh.N, M = mm->baseMesh.M, K = mm->baseMesh.K;
        const long n = (long)N * M * K;
        const long ns[3] = {(long)mm->xMesh.NMK, (long)mm->yMesh.NMK, (long)mm->zMesh.NMK};
        task->tScaleP = -1.0;
        task->eps = cfg.get("task_eps", task->eps);
        PoissonDiscreteEquation* pE = new PoissonDiscreteEquation;   // not destroyed (see below)
        pE->set(task, &(sol->prediction.p));
        mm->U_ib = pE->m_A->flux;
        HelmholtzDiscreteEquationX* uE = new HelmholtzDiscreteEquationX;
        HelmholtzDiscreteEquationY* vE = new HelmholtzDiscreteEquationY;
        HelmholtzDiscreteEquationZ* wE = new HelmholtzDiscreteEquationZ;
        uE->set(task, &(sol->prediction.u));
        vE->set(task, &(sol->prediction.v));
        wE->set(task, &(sol->prediction.w));
        sol->set((SparseMatrix*)(uE->m_grad), (SparseMatrix*)(vE->m_grad), (SparseMatrix*)(wE->m_grad), uE->coef);
        int dd[3] = {N, M, K};
        out.i("dims", dd, 3);
        out.i("celltype", (const int*)mm->baseMesh.typeOfCell, n);
        out.i("xtype", (const int*)mm->xMesh.typeOfCell, ns[0]);
        out.i("ytype", (const int*)mm->yMesh.typeOfCell, ns[1]);
        out.i("ztype", (const int*)mm->zMesh.typeOfCell, ns[2]);
        out.i("side_type", (const int*)mm->baseSideTypes, 3 * n);
        out.d("theta", (const double*)mm->theta, 3 * n);
        out.d("alpha", (const double*)mm->alpha, 3 * n);
        out.d("delta", (const double*)mm->delta, 3 * n);
        out.d("inv_vof", mm->baseMesh.inv_VOF, n);
        out.d("vof_x", mm->xMesh.VOF, ns[0]);
        out.d("vof_y", mm->yMesh.VOF, ns[1]);
        out.d("vof_z", mm->zMesh.VOF, ns[2]);
        out.d("inv_mx", mm->xMesh.inv_VOF, ns[0]);
        out.d("inv_my", mm->yMesh.inv_VOF, ns[1]);
        out.d("inv_mz", mm->zMesh.inv_VOF, ns[2]);
        out.d("dib_en", (const double*)mm->delta_ib_en, 3 * n);
        out.d("dib_ws", (const double*)mm->delta_ib_ws, 3 * n);
        out.d("dib_nb", (const double*)mm->delta_ib_nb, 3 * n);
        out.d("dib_st", (const double*)mm->delta_ib_st, 3 * n);
        out.d("inv_dib_ne", (const double*)mm->inv_delta_ib_ne, 3 * n);
        out.d("inv_dib_tn", (const double*)mm->inv_delta_ib_tn, 3 * n);
        out.d("vib", (const double*)mm->v_ib, 3 * n);
        out.d("vibyx", (const double*)mm->v_ib_yx, 3 * n);
        out.d("vibzy", (const double*)mm->v_ib_zy, 3 * n);
        out.d("u_w", task->pU_W, (long)M * K);
        double bc[18] = {task->U_W, task->U_E, task->U_S, task->U_N, task->U_B, task->U_T,
                         task->V_W, task->V_E, task->V_S, task->V_N, task->V_B, task->V_T,
                         task->W_W, task->W_E, task->W_S, task->W_N, task->W_B, task->W_T};
        out.d("bc", bc, 18);
        int pins[2] = {pE->A.fixPointNum, pE->A.fixPointFlowNum};
        out.i("pins", pins, 2);
        double par[8] = {task->nu, uE->coef, 1.0 / task->t, task->COEF_INTEGR_TIME, task->t, task->eps,
                         task->V_BASE, (double)task->MAX_ITER};
        out.d("nu_coef_coef2_integr_dt_eps_vbase_maxit", par, 8);
        int rs[2] = {task->FGMRES_RESTART_NUM, task->FGMRES_RESTART_NUM_P};
        out.i("restart_mom_p", rs, 2);
        double *cu, *cv, *cw, *cp, *pu, *pv, *pw, *pp;
        sol->current.getCopy(cu, cv, cw, cp);
        sol->prediction.getCopy(pu, pv, pw, pp);
        out.d("u_0", cu, ns[0]);
        out.d("v_0", cv, ns[1]);
        out.d("w_0", cw, ns[2]);
        out.d("p_0", cp, n);
        const int steps = (int)cfg.get("flow_steps", 0);
        std::vector<double> step_s;
        for (int s = 1; s <= steps; s++) {
            const double t_step = now_s();
            curTime += task->t;
            sol->init();
            task->rebuildMesh();
            pE->m_A->calcFlux();
            const std::string k = std::to_string(s);
            const bool dump = !(int)cfg.get("flow_no_dump", 0);   // timing runs write nothing inside the step
            if (dump) out.d("lflux_" + k, pE->A.flux, n);
            uE->solve();
            vE->solve();
            wE->solve();
            pE->solve();
            if (dump) {
                out.d("us_" + k, pu, ns[0]);
                out.d("vs_" + k, pv, ns[1]);
                out.d("ws_" + k, pw, ns[2]);
                out.d("phi_" + k, pp, n);
            }
            int its[4] = {uE->solver.it, vE->solver.it, wE->solver.it, pE->solver.it};
            out.i("its_" + k, its, 4);
            sol->correction();
            step_s.push_back(now_s() - t_step);
            if (s < steps) it++;
            if (!dump) continue;
            out.d("u_" + k, cu, ns[0]);
            out.d("v_" + k, cv, ns[1]);
            out.d("w_" + k, cw, ns[2]);
            out.d("p_" + k, cp, n);
        }
        out.d("step_s", step_s.data(), (long)step_s.size());
        if ((int)cfg.get("save_state", 0)) {
            // the reference's own continue-state file (SetSolutions::saveState,
            // set_solutions.h:318-337), returned byte for byte
            sol->saveState();
            std::string found;
            for (const auto& e : std::filesystem::directory_iterator(outdir))
                if (e.path().filename().string().rfind("continueSolveTask__", 0) == 0) found = e.path().string();
            std::ifstream sf(found, std::ios::binary);
            std::vector<char> bytes((std::istreambuf_iterator<char>(sf)), std::istreambuf_iterator<char>());
            out.put("state_bytes", (const unsigned char*)bytes.data(), (long)bytes.size(), "u1");
            int itc = it;
            out.i("state_it", &itc, 1);
            out.scalar("state_time", curTime);
        }
        if ((int)cfg.get("print_sol", 0)) {
            // the reference's own Tecplot solution file (SetSolutions::print ->
            // SolTecplotPrinter::printField, sol_tecplot_printer.h:254-355) of
            // the current state, returned byte for byte
            sol->print();
            std::string found;
            for (const auto& e : std::filesystem::directory_iterator(outdir)) {
                const std::string nm = e.path().filename().string();
                if (nm.find("Sol") != std::string::npos && nm.rfind("continueSolveTask", 0) != 0 && nm.size() > 4 &&
                    nm.substr(nm.size() - 4) == ".dat")
                    found = e.path().string();
            }
            std::ifstream sf(found, std::ios::binary);
            std::vector<char> bytes((std::istreambuf_iterator<char>(sf)), std::istreambuf_iterator<char>());
            out.put("sol_bytes", (const unsigned char*)bytes.data(), (long)bytes.size(), "u1");
            LSSTAGUniformMesh* pm = task->m_mesh;
            out.d("nodes", (const double*)pm->nodes, 3L * pm->baseMesh.N * pm->baseMesh.M * pm->baseMesh.K);
        }
        int nthreads = omp_get_max_threads();
        out.i("omp_threads", &nthreads, 1);
        return 0;
    }
    if ((int)cfg.get("helm", 0)) {
        // the momentum operators as the time step builds them
        // (HelmholtzDiscreteOperatorX/Y/Z::init -> build: calcFlux, calcHelm*,
        // the outflow terms), optionally on seeded geometry arrays: face and
        // edge fractions (some alpha exactly 0, so that the immersed-boundary
        // branches run on every cell type), cell volumes and the
        // immersed-boundary distances are replaced, the cell types are kept
        LSSTAGUniformMesh* mm = task->m_mesh;
        const int N = mm->baseMesh.N, M = mm->baseMesh.M, K = mm->baseMesh.K;
        const long n = (long)N * M * K;
        const long ns[3] = {(long)mm->xMesh.NMK, (long)mm->yMesh.NMK, (long)mm->zMesh.NMK};
        if ((int)cfg.get("helm_random", 0)) {
            std::mt19937_64 rng((unsigned long long)cfg.get("seed", 1));
            std::uniform_real_distribution<double> U(0.0, 1.0);
            auto frac = [&](double pz, double p1) {
                const double r = U(rng);
                if (r < pz) return 0.0;
                if (r < pz + p1) return 1.0;
                return 0.05 + 0.95 * U(rng);
            };
            for (long i = 0; i < n; i++) {
                mm->theta[i].set(frac(0.0, 0.2), frac(0.0, 0.2), frac(0.0, 0.2));
                mm->alpha[i].set(frac(0.15, 0.2), frac(0.15, 0.2), frac(0.15, 0.2));
                mm->baseMesh.inv_VOF[i] = 0.5 + 1.5 * U(rng);
                coordinate* arr[6] = {mm->delta_ib_en, mm->delta_ib_ws, mm->delta_ib_nb, mm->delta_ib_st,
                                      mm->inv_delta_ib_ne, mm->inv_delta_ib_tn};
                for (int a = 0; a < 6; a++) arr[a][i].set(0.1 + U(rng), 0.1 + U(rng), 0.1 + U(rng));
            }
            double* vofs[3] = {mm->xMesh.VOF, mm->yMesh.VOF, mm->zMesh.VOF};
            for (int d = 0; d < 3; d++)
                for (long i = 0; i < ns[d]; i++) vofs[d][i] = 0.2 + 0.8 * U(rng);
            // cell sizes, boundary velocities and immersed-boundary velocities too
            const double hx = task->hx, hy = task->hy, hz = task->hz;
            for (long i = 0; i < n; i++) {
                mm->delta[i].set(hx * (0.5 + U(rng)), hy * (0.5 + U(rng)), hz * (0.5 + U(rng)));
                mm->v_ib[i].set(U(rng) - 0.5, U(rng) - 0.5, U(rng) - 0.5);
                mm->v_ib_yx[i].set(U(rng) - 0.5, U(rng) - 0.5, U(rng) - 0.5);
                mm->v_ib_zy[i].set(U(rng) - 0.5, U(rng) - 0.5, U(rng) - 0.5);
            }
            for (long j = 0; j < (long)M * K; j++) task->pU_W[j] = 0.5 + U(rng);
            double* bcs[18] = {&task->U_W, &task->U_E, &task->U_S, &task->U_N, &task->U_B, &task->U_T,
                               &task->V_W, &task->V_E, &task->V_S, &task->V_N, &task->V_B, &task->V_T,
                               &task->W_W, &task->W_E, &task->W_S, &task->W_N, &task->W_B, &task->W_T};
            for (int b = 0; b < 18; b++) *bcs[b] = U(rng) - 0.5;
        }
        // the operators of a task that is not a flow (no outflow terms, walls on T/B)
        if ((int)cfg.get("helm_noflow", 0)) task->id = BaseTaskDescription::TASK_UNKNOWN;
        HelmXProbe* kx = new HelmXProbe;   // not destroyed (see below)
        HelmYProbe* ky = new HelmYProbe;
        HelmZProbe* kz = new HelmZProbe;
        kx->init(task, &mm->xMesh);
        ky->init(task, &mm->yMesh);
        kz->init(task, &mm->zMesh);
        int dd[3] = {N, M, K};
        out.i("dims", dd, 3);
        out.csr("Kx", (SparseMatrix*)kx);
        out.csr("Ky", (SparseMatrix*)ky);
        out.csr("Kz", (SparseMatrix*)kz);
        out.d("hflux_x", kx->flux, ns[0]);
        out.d("hflux_y", ky->flux, ns[1]);
        out.d("hflux_z", kz->flux, ns[2]);
        if ((int)cfg.get("helm_conv", 0)) {
            // the convective operators' boundary source term (baseFlux of
            // ConvectiveDiscreteOperatorX/Y/Z, built by init -> build -> calcFlux
            // for flow tasks) on seeded velocities
            std::mt19937_64 rng2((unsigned long long)cfg.get("seed", 1) + 17);
            std::uniform_real_distribution<double> U2(-1.0, 1.0);
            double* cur[3] = {mm->m_Ux, mm->m_Uy, mm->m_Uz};
            for (int d = 0; d < 3; d++)
                for (long i = 0; i < ns[d]; i++) cur[d][i] = U2(rng2);
            ConvectiveDiscreteOperatorX* cx = new ConvectiveDiscreteOperatorX;   // not destroyed (see below)
            ConvectiveDiscreteOperatorY* cy = new ConvectiveDiscreteOperatorY;
            ConvectiveDiscreteOperatorZ* cz = new ConvectiveDiscreteOperatorZ;
            cx->init(task, &mm->xMesh);
            cy->init(task, &mm->yMesh);
            cz->init(task, &mm->zMesh);
            cx->recalc();
            cy->recalc();
            cz->recalc();
            out.d("cflux_x", cx->flux, ns[0]);
            out.d("cflux_y", cy->flux, ns[1]);
            out.d("cflux_z", cz->flux, ns[2]);
            out.d("ux", mm->m_Ux, ns[0]);
            out.d("uy", mm->m_Uy, ns[1]);
            out.d("uz", mm->m_Uz, ns[2]);
        }
        if ((int)cfg.get("helm_ibflux", 0)) {
            // the immersed-boundary part of the source term, which the time
            // step recomputes for moving bodies (ibFluxHelmX/Y/Z), applied
            // over the boundary flux above
            kx->runIbFlux();
            ky->runIbFlux();
            kz->runIbFlux();
            out.d("hflux_ib_x", kx->flux, ns[0]);
            out.d("hflux_ib_y", ky->flux, ns[1]);
            out.d("hflux_ib_z", kz->flux, ns[2]);
        }
        out.i("xtype", (const int*)mm->xMesh.typeOfCell, ns[0]);
        out.i("ytype", (const int*)mm->yMesh.typeOfCell, ns[1]);
        out.i("ztype", (const int*)mm->zMesh.typeOfCell, ns[2]);
        out.i("celltype", (const int*)mm->baseMesh.typeOfCell, n);
        out.i("side_type", (const int*)mm->baseSideTypes, 3 * n);
        out.d("theta", (const double*)mm->theta, 3 * n);
        out.d("alpha", (const double*)mm->alpha, 3 * n);
        out.d("delta", (const double*)mm->delta, 3 * n);
        out.d("inv_vof", mm->baseMesh.inv_VOF, n);
        out.d("vof_x", mm->xMesh.VOF, ns[0]);
        out.d("vof_y", mm->yMesh.VOF, ns[1]);
        out.d("vof_z", mm->zMesh.VOF, ns[2]);
        out.d("dib_en", (const double*)mm->delta_ib_en, 3 * n);
        out.d("dib_ws", (const double*)mm->delta_ib_ws, 3 * n);
        out.d("dib_nb", (const double*)mm->delta_ib_nb, 3 * n);
        out.d("dib_st", (const double*)mm->delta_ib_st, 3 * n);
        out.d("inv_dib_ne", (const double*)mm->inv_delta_ib_ne, 3 * n);
        out.d("inv_dib_tn", (const double*)mm->inv_delta_ib_tn, 3 * n);
        out.d("vib", (const double*)mm->v_ib, 3 * n);
        out.d("vibyx", (const double*)mm->v_ib_yx, 3 * n);
        out.d("vibzy", (const double*)mm->v_ib_zy, 3 * n);
        out.d("u_w", task->pU_W, (long)M * K);
        double par[4] = {task->nu, task->COEF_INTEGR_TIME, (double)(task->id == BaseTaskDescription::TASK_FLOW), task->t};
        out.d("nu_coef_isflow_dt", par, 4);
        // U_W U_E U_S U_N U_B U_T, V_W V_E V_S V_N V_B V_T, W_W W_E W_S W_N W_B W_T
        double bc[18] = {task->U_W, task->U_E, task->U_S, task->U_N, task->U_B, task->U_T,
                         task->V_W, task->V_E, task->V_S, task->V_N, task->V_B, task->V_T,
                         task->W_W, task->W_E, task->W_S, task->W_N, task->W_B, task->W_T};
        out.d("bc", bc, 18);
        return 0;
    }
    if ((int)cfg.get("loads", 0)) {
        // LoadsCalculator::calculate (loads_calculator.h:1366-1377) over the
        // cut cells the mesh build listed (BaseTaskDescription::addCutCell,
        // base_task_description.h:127-132), on seeded velocities, pressure and
        // immersed-boundary velocities (velocities stay zero inside the bodies)
        LSSTAGUniformMesh* mm = task->m_mesh;
        const int N = mm->baseMesh.N, M = mm->baseMesh.M, K = mm->baseMesh.K;
        const long n = (long)N * M * K;
        double* cur[3] = {mm->m_Ux, mm->m_Uy, mm->m_Uz};
        const long ns[3] = {(long)mm->xMesh.NMK, (long)mm->yMesh.NMK, (long)mm->zMesh.NMK};
        const CellTypes* st[3] = {mm->xMesh.typeOfCell, mm->yMesh.typeOfCell, mm->zMesh.typeOfCell};
        for (int d = 0; d < 3; d++)
            for (long i = 0; i < ns[d]; i++)
                cur[d][i] = (st[d][i] == SolidCell) ? 0.0 : (d == 0 ? 1.0 : 0.0) + 0.2 * sin(0.07 * i + d);
        for (long i = 0; i < n; i++) {
            mm->m_P[i] = 0.3 * sin(0.013 * i);
            mm->v_ib[i].set(0.02 * sin(0.11 * i), 0.02 * cos(0.13 * i), 0.01 * sin(0.17 * i));
            mm->v_ib_yx[i].set(0.02 * cos(0.19 * i), 0.01 * sin(0.23 * i), 0.02 * cos(0.29 * i));
            mm->v_ib_zy[i].set(0.01 * sin(0.31 * i), 0.02 * cos(0.37 * i), 0.01 * cos(0.41 * i));
        }
        LoadsCalculator& L = task->m_loads[0];
        L.initSol();
        L.calculate();
        const int cnt = L.countCutCells;
        std::vector<int> cells(cnt);
        for (int i = 0; i < cnt; i++) cells[i] = L.OnAirfoil[i].z;
        int dd[3] = {N, M, K};
        out.i("dims", dd, 3);
        out.i("cells", cells.data(), cnt);
        out.d("fx", L.ForceX, cnt);
        out.d("fy", L.ForceY, cnt);
        out.d("fz", L.ForceZ, cnt);
        double sc[9] = {L.F_aer_x, L.F_aer_y, L.F_aer_z, L.C_d, L.C_y, L.C_z,
                        L.moment_aer, L.moment_x_aer, L.moment_y_aer};
        out.d("sums", sc, 9);
        double par[3] = {task->nu, task->loadsCoef(), task->t};
        out.d("nu_fcoef_dt", par, 3);
        out.i("celltype", (const int*)mm->baseMesh.typeOfCell, n);
        out.d("theta", (const double*)mm->theta, 3 * n);
        out.d("delta", (const double*)mm->delta, 3 * n);
        out.d("inv_vof", mm->baseMesh.inv_VOF, n);
        out.d("dmax", (const double*)mm->delta_ib_max, 3 * n);
        out.d("dne", (const double*)mm->inv_delta_ib_ne, 3 * n);
        out.d("dtn", (const double*)mm->inv_delta_ib_tn, 3 * n);
        out.d("vib", (const double*)mm->v_ib, 3 * n);
        out.d("vibyx", (const double*)mm->v_ib_yx, 3 * n);
        out.d("vibzy", (const double*)mm->v_ib_zy, 3 * n);
        out.d("nodes", (const double*)mm->nodes, 3 * n);
        out.d("center", (const double*)mm->cur_C, 3);
        out.d("ux", mm->m_Ux, ns[0]);
        out.d("uy", mm->m_Uy, ns[1]);
        out.d("uz", mm->m_Uz, ns[2]);
        out.d("p", mm->m_P, n);
        return 0;
    }
    if ((int)cfg.get("operator_only", 0)) {
        // the Laplace operator alone (LaplaceDiscreteOperator::init + build), without
        // the pressure equation's solver set-up, whose multigrid hierarchy does not
        // fit host memory on the largest grids
        LaplaceDiscreteOperator* Aop = new LaplaceDiscreteOperator;   // not destroyed (see below)
        Aop->init(task, &task->m_mesh->baseMesh);
        LSSTAGUniformMesh* mm = task->m_mesh;
        int dd[3] = {mm->baseMesh.N, mm->baseMesh.M, mm->baseMesh.K};
        out.i("dims", dd, 3);
        out.csr("A", (SparseMatrix*)Aop);
        int pp[2] = {Aop->fixPointNum, Aop->fixPointFlowNum};
        out.i("pins", pp, 2);
        return 0;
    }
    PoissonDiscreteEquation* pEq = new PoissonDiscreteEquation;
    pEq->set(task, &(sol->prediction.p));
    double t_setup = now_s() - t0;

    LSSTAGUniformMesh* m = task->m_mesh;
    const int N = m->baseMesh.N, M = m->baseMesh.M, K = m->baseMesh.K;
    const long n = (long)N * M * K;
    int dims[3] = {N, M, K};
    out.i("dims", dims, 3);
    out.scalar("t_setup_s", t_setup);

    const int dumpGeom = (int)cfg.get("dump_geometry", 1);
    if (dumpGeom) {
        out.i("celltype", (const int*)m->baseMesh.typeOfCell, n);
        out.d("theta", (const double*)m->theta, 3 * n);
        out.d("alpha", (const double*)m->alpha, 3 * n);
        out.d("delta", (const double*)m->delta, 3 * n);
        out.d("phi", m->phi, n);
        out.d("vof", m->baseMesh.VOF, n);
        out.d("inv_mx", m->xMesh.inv_VOF, (long)m->xMesh.NMK);
        out.d("inv_my", m->yMesh.inv_VOF, (long)m->yMesh.NMK);
        out.d("inv_mz", m->zMesh.inv_VOF, (long)m->zMesh.NMK);
        out.d("flux", pEq->A.flux, n);
        // inputs of the Laplace source term (LaplaceDiscreteOperator::initFlux,
        // ibFlux, setBaseFlux): face types, immersed-boundary velocity,
        // boundary velocities and the x-velocity used for the outflow
        out.i("side_type", (const int*)m->baseSideTypes, 3 * n);
        out.d("vib", (const double*)m->v_ib, 3 * n);
        out.d("u_w", task->pU_W, (long)M * K);
        double bc[5] = {task->U_E, task->V_S, task->V_N, task->W_B, task->W_T};
        out.d("bc_ue_vs_vn_wb_wt", bc, 5);
        out.d("ux0", m->m_Ux, (long)m->xMesh.NMK);
    }
    // projection operators: divergence rows on the base grid
    // (poisson_discrete_equation.h Dx/Dy/Dz), gradient rows on the staggered
    // grids (GradientDiscreteOperatorX/Y/Z as the momentum equations build
    // them, helmholtz_discrete_equation.h set()), staggered cell types
    GradientDiscreteOperatorX* gx = nullptr;   // not destroyed (see below)
    GradientDiscreteOperatorY* gy = nullptr;
    GradientDiscreteOperatorZ* gz = nullptr;
    const bool wantProj = (int)cfg.get("dump_projection", 0) || (int)cfg.get("projection", 0);
    if (wantProj) {
        gx = new GradientDiscreteOperatorX;
        gy = new GradientDiscreteOperatorY;
        gz = new GradientDiscreteOperatorZ;
        gx->initMeshParams(&m->xMesh, m);
        gy->initMeshParams(&m->yMesh, m);
        gz->initMeshParams(&m->zMesh, m);
    }
    if ((int)cfg.get("dump_projection", 0)) {
        out.i("xtype", (const int*)m->xMesh.typeOfCell, (long)m->xMesh.NMK);
        out.i("ytype", (const int*)m->yMesh.typeOfCell, (long)m->yMesh.NMK);
        out.i("ztype", (const int*)m->zMesh.typeOfCell, (long)m->zMesh.NMK);
        out.csr("Dx", (SparseMatrix*)&pEq->Dx);
        out.csr("Dy", (SparseMatrix*)&pEq->Dy);
        out.csr("Dz", (SparseMatrix*)&pEq->Dz);
        out.csr("Gx", (SparseMatrix*)gx);
        out.csr("Gy", (SparseMatrix*)gy);
        out.csr("Gz", (SparseMatrix*)gz);
    }
    SparseMatrix* A = (SparseMatrix*)&pEq->A;
    if ((int)cfg.get("dump_matrix", 1)) out.csr("A", A);
    int pins[2] = {pEq->A.fixPointNum, pEq->A.fixPointFlowNum};
    out.i("pins", pins, 2);

    // Right-hand side: read from file when given (written by the runner).
    std::vector<double> b(n, 0.0);
    const std::string rhsPath = cfg.gets("rhs", "");
    if (rhsPath.empty()) return 0;
    {
        std::ifstream f(rhsPath, std::ios::binary);
        f.read((char*)b.data(), sizeof(double) * n);
        if (!f) { fprintf(stderr, "cannot read rhs %s\n", rhsPath.c_str()); return 3; }
    }
    double bnorm = 0.0;
    for (long i = 0; i < n; i++) bnorm += b[i] * b[i];
    bnorm = sqrt(bnorm);
    const double rel = cfg.get("rel_tol", 1e-10);
    const double eps = cfg.get("abs_tol", rel * bnorm);
    out.scalar("eps", eps);

    // --- one pressure projection of the time step (TimeSteppingMethod::step:
    //     pEq.solve() then sol.correction()) on predicted velocities read from
    //     files: the right-hand side (PoissonDiscreteEquation::recalcRightMember),
    //     the MG-FGMRES pressure correction and the corrected fields ---
    // --- the momentum equations as the time step builds them
    //     (TimeSteppingMethod::init: uEq/vEq/wEq.set): the Helmholtz operators
    //     K (HelmholtzDiscreteOperatorX/Y/Z), the convective operators C
    //     (ConvectiveDiscreteOperatorX/Y/Z, recalculated on the initial
    //     velocity) and one solve of each K with the momentum solver
    //     (ILUFGMRES) on a right-hand side read from a file ---
    if ((int)cfg.get("momentum", 0)) {
        HelmholtzDiscreteEquationX* ux = new HelmholtzDiscreteEquationX;   // not destroyed (see below)
        HelmholtzDiscreteEquationY* vy = new HelmholtzDiscreteEquationY;
        HelmholtzDiscreteEquationZ* wz = new HelmholtzDiscreteEquationZ;
        ux->set(task, &(sol->prediction.u));
        vy->set(task, &(sol->prediction.v));
        wz->set(task, &(sol->prediction.w));
        HelmholtzDiscreteEquation* eq[3] = {ux, vy, wz};
        const char* nm[3] = {"x", "y", "z"};
        const double meps = cfg.get("mom_rel_tol", 1e-10);
        for (int d = 0; d < 3; d++) {
            HelmholtzDiscreteEquation* e = eq[d];
            const long ne = e->m_A->NMK;
            out.csr(std::string("K") + nm[d], (SparseMatrix*)e->m_A);
            out.csr(std::string("C") + nm[d], (SparseMatrix*)e->m_conv);
            std::vector<double> rhs(ne, 0.0);
            std::ifstream f(cfg.gets(std::string("mom_rhs_") + nm[d], ""), std::ios::binary);
            f.read((char*)rhs.data(), sizeof(double) * ne);
            if (!f) {
                fprintf(stderr, "cannot read momentum rhs %s\n", nm[d]);
                return 3;
            }
            double bn = 0.0;
            for (double v : rhs) bn += v * v;
            std::copy(rhs.begin(), rhs.end(), e->m_right);
            std::fill(e->m_sol, e->m_sol + ne, 0.0);
            e->solver.eps = meps * sqrt(bn);
            int mit = e->solver.solve();
            out.d(std::string("mom_x_") + nm[d], e->m_sol, ne);
            out.i(std::string("mom_it_") + nm[d], &mit, 1);
            out.scalar(std::string("mom_eps_") + nm[d], e->solver.eps);
        }
        int rs = task->FGMRES_RESTART_NUM, mi = task->MAX_ITER;
        out.i("mom_restart", &rs, 1);
        out.i("mom_max_it", &mi, 1);
        if ((int)cfg.get("mom_step", 0)) {
            // one momentum step of each equation (HelmholtzDiscreteEquation::
            // solve: recalcRightMember + ILUFGMRES) on perturbed current and
            // previous velocities and pressure.  The state left by set() (the
            // convective product C(u0) u0 + flux2 as the previous term) is
            // dumped first, then the inputs, the right-hand side and solution.
            LSSTAGUniformMesh* mm = task->m_mesh;
            double* cur[3] = {mm->m_Ux, mm->m_Uy, mm->m_Uz};
            double* prv[3] = {mm->m_prevUx, mm->m_prevUy, mm->m_prevUz};
            const double* vofs[3] = {mm->xMesh.VOF, mm->yMesh.VOF, mm->zMesh.VOF};
            for (int d = 0; d < 3; d++) {
                HelmholtzDiscreteEquation* e = eq[d];
                const long ne = e->m_A->NMK;
                out.csr(std::string("C0") + nm[d], (SparseMatrix*)e->m_conv);
                out.d(std::string("flux2_0") + nm[d], e->m_conv->flux, ne);
                out.d(std::string("u0") + nm[d], cur[d], ne);
            }
            const CellTypes* stype[3] = {mm->xMesh.typeOfCell, mm->yMesh.typeOfCell, mm->zMesh.typeOfCell};
            for (int d = 0; d < 3; d++) {
                const long ne = eq[d]->m_A->NMK;
                for (long i = 0; i < ne; i++) {
                    if (stype[d][i] == SolidCell) continue;     // velocities stay zero inside the bodies
                    cur[d][i] += 0.05 * sin(0.07 * i + d);
                    prv[d][i] = cur[d][i] - 0.01 * cos(0.05 * i + 2 * d);
                }
            }
            for (long i = 0; i < n; i++) mm->m_P[i] = 0.3 * sin(0.013 * i);
            out.d("mstep_p", mm->m_P, n);
            for (int d = 0; d < 3; d++) {
                HelmholtzDiscreteEquation* e = eq[d];
                const long ne = e->m_A->NMK;
                out.d(std::string("mstep_u_") + nm[d], cur[d], ne);
                out.d(std::string("mstep_uprev_") + nm[d], prv[d], ne);
                out.d(std::string("mstep_vof_") + nm[d], vofs[d], ne);
                std::fill(e->m_sol, e->m_sol + ne, 0.0);
                e->solver.eps = 1e-10;
                e->solve();
                out.csr(std::string("C1") + nm[d], (SparseMatrix*)e->m_conv);
                out.d(std::string("flux2_1") + nm[d], e->m_conv->flux, ne);
                out.d(std::string("mstep_hflux_") + nm[d], e->m_A->flux, ne);
                out.d(std::string("mstep_rhs_") + nm[d], e->m_right, ne);
                out.d(std::string("mstep_sol_") + nm[d], e->m_sol, ne);
                int it = e->solver.it;
                out.i(std::string("mstep_it_") + nm[d], &it, 1);
                out.csr(std::string("K1") + nm[d], (SparseMatrix*)e->m_A);
            }
            double c2 = 1.0 / task->t;
            out.scalar("mstep_coef2", c2);
        }
        return 0;
    }
    if ((int)cfg.get("projection", 0)) {
        task->tScaleP = -1.0;                     // no start-up pressure scaling
        const double coefP = 1.5 / task->t;       // HelmholtzDiscreteEquation::coef (BDF2)
        sol->set((SparseMatrix*)gx, (SparseMatrix*)gy, (SparseMatrix*)gz, coefP);
        double *pu, *pv, *pw, *pp, *cu, *cv, *cw, *cp;
        sol->prediction.getCopy(pu, pv, pw, pp);
        sol->current.getCopy(cu, cv, cw, cp);
        auto readv = [&](const char* key, double* dst, long cnt) {
            std::ifstream f(cfg.gets(key, ""), std::ios::binary);
            f.read((char*)dst, sizeof(double) * cnt);
            return (bool)f;
        };
        if (!readv("proj_u", pu, m->xMesh.NMK) || !readv("proj_v", pv, m->yMesh.NMK) ||
            !readv("proj_w", pw, m->zMesh.NMK) || !readv("proj_p", cp, n)) {
            fprintf(stderr, "cannot read projection inputs\n");
            return 3;
        }
        std::fill(pp, pp + n, 0.0);
        pEq->solver.eps = eps;
        pEq->solve();
        out.d("proj_b", pEq->m_right, n);
        out.d("proj_phi", pp, n);
        int pit = pEq->solver.it;
        out.i("proj_it", &pit, 1);
        sol->correction();
        out.d("proj_u_out", cu, m->xMesh.NMK);
        out.d("proj_v_out", cv, m->yMesh.NMK);
        out.d("proj_w_out", cw, m->zMesh.NMK);
        out.d("proj_p_out", cp, n);
        out.scalar("proj_coef", coefP);
        out.scalar("proj_vbase", task->V_BASE);
        return 0;
    }
    const int reps = (int)cfg.get("repeats", 1);
    // --- one V-cycle of the reference multigrid (a standalone instance with
    //     the same task parameters as the MGFGMRES preconditioner) ---
    if ((int)cfg.get("dump_mg", 0)) {
        // heap-allocated and intentionally not destroyed: the reference's
        // hierarchy destructors are not safe for a second instance.
        MultiGridSolver* mg = new MultiGridSolver;
        mg->set(A, task);
        dumpHierarchy(out, *mg);
        std::vector<double> x(n, 0.0);
        mg->solve(b.data(), x.data());
        out.d("vcycle_x", x.data(), n);
    }
    // --- MG-FGMRES ---
    if ((int)cfg.get("fgmres", 1)) {
        auto& s = pEq->solver;       // MGFGMRES, or the B200 adapter in the drop-in build
        s.eps = eps;
        std::vector<double> ts;
        for (int r = 0; r < reps; r++) {
            std::copy(b.begin(), b.end(), pEq->m_right);
            std::fill(pEq->m_sol, pEq->m_sol + n, 0.0);
            double t1 = now_s();
            int iters = s.solve();
            ts.push_back(now_s() - t1);
            if (r == reps - 1) {
                out.d("fgmres_x", pEq->m_sol, n);
                out.i("fgmres_it", &iters, 1);
                out.scalar("fgmres_norm_r", s.norm_r);
            }
        }
        out.d("fgmres_time_s", ts.data(), (long)ts.size());
    }
    // --- ILU(0)-BiCGStab (bicgstab_interface.h / ilu_bicgstab.h) ---
    if ((int)cfg.get("bicgstab", 0)) {
        ILUBiCGStab& s = *new ILUBiCGStab;  // not destroyed (see above)
        std::vector<double> x(n, 0.0), bb(b);
        double tset = now_s();
        s.set(A, bb.data(), x.data(), task);
        tset = now_s() - tset;
        s.eps = eps;
        std::vector<double> ts;
        for (int r = 0; r < reps; r++) {
            std::fill(x.begin(), x.end(), 0.0);
            double t1 = now_s();
            int iters = s.solve();
            ts.push_back(now_s() - t1);
            if (r == reps - 1) {
                out.d("bicgstab_x", x.data(), n);
                out.i("bicgstab_it", &iters, 1);
                out.scalar("bicgstab_norm_r", s.norm_r);
            }
        }
        out.d("bicgstab_time_s", ts.data(), (long)ts.size());
        out.scalar("bicgstab_setup_s", tset);
    }
    int nthreads = omp_get_max_threads();
    out.i("omp_threads", &nthreads, 1);
    return 0;
}
