// Host orchestration and C ABI of the B200 pressure-Poisson solver.
//
// Replaces the reference's MGFGMRES / ILUBiCGStab solvers
// (Base/Solvers/FGMRES/mg_fgmres.h, Base/Solvers/BiCGStab/ilu_bicgstab.h)
// behind IterativeSolverInterface (Base/Solvers/iterative_solver_interface.h).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <thread>

#include "lsg_adlj_fused.cuh"
#include "lsg_dict.cuh"
#include "lsg_coarse.cuh"
#include "lsg_ilu.cuh"
#include "lsg_krylov.cuh"
#include "lsg_helmholtz.cuh"
#include "lsg_loads.cuh"
#include "lsg_mesh.cuh"
#include "lsg_projection.cuh"
#include "lsg_tecplot.cuh"

namespace lsg {

thread_local long long g_launches = 0;   // per host thread: solves on different contexts may run concurrently

// ---------------------------------------------------------------------------
// host-side tables and helpers
// ---------------------------------------------------------------------------
static int grid_levels(int N, int M, int K)
{
    // CoarseGridsHierarchy::GridLevels (coarse_grids_hierarchy.h:73-81)
    double aux = (double)std::min(std::min(N, M), K);
    int n = 0;
    while (aux > 2.0) {
        aux *= 0.5;
        n++;
    }
    return n;
}

static int coarse_count(int nf, bool& odd)
{
    // CoarseGrid::nodesCount (coarse_grid.h:62-69)
    odd = std::fmod((double)nf, 2.0) > 1e-5;
    return odd ? (nf + 1) / 2 : nf / 2;
}

// 1-D prolongation table: for each fine index two (coarse, weight) pairs.
static void prolong_table(int nf, std::vector<int>& c, std::vector<float>& w)
{
    bool odd;
    const int nc = coarse_count(nf, odd);
    c.assign(2 * nf, 0);
    w.assign(2 * nf, 0.f);
    for (int f = 0; f < nf; f++) {
        const int I = f / 2;
        int c0 = 0, c1 = 0;
        float w0 = 0.f, w1 = 0.f;
        if (odd) {
            if (f % 2 == 0) { c0 = I; w0 = 1.f; }
            else { c0 = I; w0 = 0.5f; c1 = I + 1; w1 = 0.5f; }
        } else {
            if (f == 0) { c0 = 0; w0 = 1.f; }
            else if (f == nf - 1) { c0 = nc - 1; w0 = 1.f; }
            else if (f % 2 == 0) { c0 = I - 1; w0 = 0.25f; c1 = I; w1 = 0.75f; }
            else { c0 = I; w0 = 0.75f; c1 = I + 1; w1 = 0.25f; }
        }
        c[2 * f] = c0; w[2 * f] = w0;
        c[2 * f + 1] = c1; w[2 * f + 1] = w1;
    }
}

// 1-D restriction table R = P^T: for each coarse index up to 4 (fine, w).
static void restrict_table(int nf, std::vector<int>& f4, std::vector<float>& w4)
{
    bool odd;
    const int nc = coarse_count(nf, odd);
    std::vector<int> pc;
    std::vector<float> pw;
    prolong_table(nf, pc, pw);
    f4.assign(4 * nc, -1);
    w4.assign(4 * nc, 0.f);
    std::vector<int> cnt(nc, 0);
    for (int f = 0; f < nf; f++)
        for (int a = 0; a < 2; a++) {
            if (pw[2 * f + a] == 0.f) continue;
            const int I = pc[2 * f + a];
            f4[4 * I + cnt[I]] = f;
            w4[4 * I + cnt[I]] = pw[2 * f + a];
            cnt[I]++;
        }
}

// Radius of the Galerkin coarse stencil in one dimension.
static int coarse_radius(int rf, bool odd, bool agglomerate)
{
    std::vector<int> rs, ps;
    if (agglomerate) rs = {0, 1};
    else if (odd) rs = {-1, 0, 1};
    else rs = {-1, 0, 1, 2};
    if (odd) ps = {-1, 0, 1};
    else ps = {-1, 0, 1, 2};
    int rc = 0;
    for (int sr : rs)
        for (int a = -rf; a <= rf; a++)
            for (int sp : ps) {
                const int v = sr + a - sp;
                if (v % 2 == 0) rc = std::max(rc, std::abs(v / 2));
            }
    return rc;
}

static OffList make_offlist(const std::vector<int>& off)
{
    OffList ol;
    std::memset(&ol, 0, sizeof(ol));
    ol.n = (int)off.size() / 3;
    ol.center = -1;
    for (int o = 0; o < ol.n; o++) {
        for (int d = 0; d < 3; d++) ol.o[o][d] = (signed char)off[3 * o + d];
        if (off[3 * o] == 0 && off[3 * o + 1] == 0 && off[3 * o + 2] == 0) ol.center = o;
    }
    return ol;
}

static const int kFine7[21] = {0, 0, -1, 0, -1, 0, -1, 0, 0, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 1};

// ---------------------------------------------------------------------------
// multigrid level storage (FP64 master copy; FP32 shadow for mixed precision)
// ---------------------------------------------------------------------------
struct TransferTabs {
    DevBuf<int> pc[3];
    DevBuf<float> pw[3];
    DevBuf<int> rf[3];
    DevBuf<float> rw[3];
    PTab P(int d) const { return PTab{pc[d].p, pw[d].p}; }
    RTab R(int d) const { return RTab{rf[d].p, rw[d].p}; }
};

template <typename T>
struct LevelT {
    Dims d;
    std::vector<int> off;     // 3 * noff
    OffList ol;
    const T* A = nullptr;     // noff * n coefficient planes (setup; FP64 master only)
    DevBuf<T> Aown;
    // solve-time operator: per-cell row class + table of distinct rows
    const int* cls = nullptr;
    DevBuf<int> clsown;
    const T* dict = nullptr;
    DevBuf<T> dictown;
    DevBuf<T> dict28;         // 27-point levels: rows padded to stride 28 for vector loads
    int nclass = 0;
    DevBuf<T> lo[3], dinv[3], up[3];
    DevBuf<T> gsdinv;         // Gauss-Seidel smoother: 1 / a_ii, 0 below the tiny pivot threshold
    DevBuf<T> r, c, ch;
};

struct MGData {
    int L = 0;                // coarse levels
    std::vector<Dims> dims;   // L + 1
    std::vector<TransferTabs> tabs;   // L (level l -> l+1)
    std::vector<bool> agg;            // L
    std::vector<LevelT<double>> l64;  // L + 1 (operators, factors for l < L)
    std::vector<LevelT<float>> l32;
    // coarsest LU
    int nc = 0;
    DevBuf<double> dL, dU, dscale, dwork;
    DevBuf<int> dperm;
    bool fp32 = false;
    // lower part of the cycle fused into k_vcycle_tail from level tail_l0 on
    // (-1: every level runs as separate kernels)
    int tail_l0 = -1;
    DevBuf<TailArgs<double>> tail64;
    DevBuf<TailArgs<float>> tail32;
    // the ADLJ V-cycle as one CUDA graph per precision (instantiated on first
    // use; it reads level 0's r and leaves the correction in level 0's ch)
    cudaGraphExec_t cycle64 = nullptr, cycle32 = nullptr;
    long long cycle64_nodes = 0, cycle32_nodes = 0;   // kernels per replay (launch accounting)
};

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
// an asynchronous Tecplot write (lsg_tecplot_sol_async): pinned host copies
// of u | v | w | p and the thread that formats and writes the file
struct TecplotAsync {
    std::thread th;
    int status = 0;
    double* pinned = nullptr;
    size_t pinned_len = 0;
    ~TecplotAsync()
    {
        if (th.joinable()) th.join();
        if (pinned) cudaFreeHost(pinned);
    }
};

struct Context {
    int device = 0;
    cudaStream_t s = nullptr;
    cudaMemPool_t pool = nullptr;   // per-call temporaries (TmpBuf)
    std::string err;
    Dims d;
    long long n = 0;
    DevBuf<double> A7;        // fine operator, 7 planes (b s w p e n t)
    DevBuf<int> cls0;         // fine operator as row classes + distinct rows
    DevBuf<double> dict0;
    int nclass0 = 0;
    bool have_matrix = false, have_setup = false;
    double matrix_ms = 0.0, setup_ms = 0.0;   // wall time of the last lsg_set_matrix_* / lsg_setup
    lsg_options opt;
    MGData mg;
    Reducer red;
    DevBuf<double> scal;      // misc device scalars (64)
    // Krylov storage
    int restart = 0;
    long long ldv = 0;        // stride between basis vectors (n padded off a power of two)
    DevBuf<double> V, Z, w, xd, bd, coefs, t1, t2, t3, t4;
    DevBuf<KrylovScalars> ks;
    int* hflag = nullptr;
    double* hnorm = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    DevBuf<float> Z32;        // FP32 preconditioned basis (FP32 multigrid)
    DevBuf<double> gs_partial, gs_sg, gs_L;   // low-synchronisation Gram-Schmidt
    // ILU(0)
    DevBuf<double> iluL, iluU;        // 3 lower planes (b s w) / 4 planes (p e n t), U diagonal = plane 0
    bool have_ilu = false;
    // the level-scheduled ILU(0) solves as one CUDA graph (instantiated on
    // first use, reading ilu_in and writing ilu_out)
    cudaGraphExec_t ilu_exec = nullptr;
    long long ilu_nodes = 0;
    DevBuf<double> ilu_in, ilu_out;
    // the one-launch ILU sweep (k_ilu_sweep_perm): factors, neighbour
    // positions and work vectors in hyperplane order, the plane offsets, its
    // barrier counter, the flag its bounded barrier sets when it gives up,
    // its grid size and positions per thread
    DevBuf<int> ilu_start, ilu_rowstart, ilu_perm, ilu_nbr;
    DevBuf<double> ilu_fac, ilu_yp, ilu_xp;
    int ilu_planes = 0, ilu_maxplane = 0;
    DevBuf<unsigned int> ilu_bar;
    DevBuf<int> ilu_err;
    int ilu_blocks = 0;
    int ilu_cmax = 0;
    double bytes = 0;
    int vcycles = 0;
    bool own_stream = true;
    // adjoint: a second solver state for the transposed operator, built on
    // first use and dropped whenever the operator changes
    std::unique_ptr<Context> adj;
    std::unique_ptr<TecplotAsync> tec;
    // cut-cell geometry kept on the device by lsg_set_matrix_geometry (the
    // projection kernels read it); staggered cell types from
    // lsg_set_staggered_types
    struct Geometry {
        DevBuf<int> type, stype[3];
        DevBuf<double> theta, delta, inv[3];
        long long pin0 = -1, pin1 = -1;
        bool have = false, have_stypes = false;
    } geo;
    // the mesh built on the device by lsg_mesh_build (the flow task's mesh
    // build: level set to staggered inverse volumes)
    struct Mesh {
        int N = 0, M = 0, K = 0;
        DevBuf<double> phi_ls, phi, alpha, theta, delta, vof, inv_vof, svof[3], sinv[3];
        DevBuf<double> dib[5], inv_dib_ne, inv_dib_tn;   // immersed-boundary areas, inverse distances
        DevBuf<int> side, type, stype[3];
        int osc_sweeps = 0;
        bool have = false;
    } mesh;
    // cut-cell loads: packed per-cut-cell records from lsg_loads_set, the
    // reduction scratch, and the state of the three moment filters
    struct Loads {
        int N = 0, M = 0, K = 0, count = 0;
        DevBuf<double> g;
        DevBuf<int> idx;
        DevBuf<unsigned long long> desc;
        DevBuf<double> partial, sums;
        DevBuf<unsigned int> counter;
        double center[3] = {0, 0, 0};
        double fcoef = 0;
        LoadsFilter filt[3];
        bool have = false;
    } loads;
};

}  // namespace lsg

struct lsg_ctx {
    lsg::Context c;
};

namespace lsg {

static void ilu_apply(Context& C, const double* b, double* x);
static void ilu_graph_release(Context& C);
static void ilu_check(Context& C);

// ---------------------------------------------------------------------------
// row dictionary of an operator given as noff coefficient planes
// ---------------------------------------------------------------------------
__global__ void k_planes_to_rows(int noff, long long n, const double* __restrict__ planes, double* __restrict__ rows)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        for (int o = 0; o < noff; o++) rows[i * noff + o] = planes[(size_t)o * n + i];
}

// Host build of the same dictionary (serial first-seen dedup); taken only
// when the device build meets two different rows with one 64-bit hash.
static int build_dict_host(cudaStream_t s, const double* planes, int noff, long long n, DevBuf<int>& cls,
                           DevBuf<double>& dict)
{
    DevBuf<double> rows;
    rows.alloc((size_t)noff * n);
    k_planes_to_rows<<<grid_for(n, 256), 256, 0, s>>>(noff, n, planes, rows.p);
    LSG_CHECK_LAUNCH();
    std::vector<double> h((size_t)noff * n);
    LSG_CUDA(cudaMemcpyAsync(h.data(), rows.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    LSG_CUDA(cudaStreamSynchronize(s));
    rows.release();
    std::vector<int> hc(n);
    std::vector<long long> first;        // row index of each class
    size_t cap = 1 << 12;
    std::vector<int> slot(cap, -1);
    const size_t rowbytes = (size_t)noff * sizeof(double);
    auto hash_row = [&](long long i) {
        const uint64_t* w = (const uint64_t*)(h.data() + (size_t)i * noff);
        uint64_t x = 0x9E3779B97F4A7C15ull;
        for (int o = 0; o < noff; o++) {
            x ^= w[o] + 0x9E3779B97F4A7C15ull + (x << 6) + (x >> 2);
            x *= 0xBF58476D1CE4E5B9ull;
            x ^= x >> 31;
        }
        return x;
    };
    for (long long i = 0; i < n; i++) {
        if (first.size() * 2 >= cap) {
            cap *= 2;
            slot.assign(cap, -1);
            for (size_t c = 0; c < first.size(); c++) {
                size_t q = hash_row(first[c]) & (cap - 1);
                while (slot[q] >= 0) q = (q + 1) & (cap - 1);
                slot[q] = (int)c;
            }
        }
        size_t q = hash_row(i) & (cap - 1);
        const double* ri = h.data() + (size_t)i * noff;
        int id = -1;
        while (slot[q] >= 0) {
            const int c = slot[q];
            if (std::memcmp(ri, h.data() + (size_t)first[c] * noff, rowbytes) == 0) {
                id = c;
                break;
            }
            q = (q + 1) & (cap - 1);
        }
        if (id < 0) {
            id = (int)first.size();
            first.push_back(i);
            slot[q] = id;
        }
        hc[i] = id;
    }
    const int nclass = (int)first.size();
    std::vector<double> hd((size_t)nclass * noff);
    for (int c = 0; c < nclass; c++)
        std::memcpy(hd.data() + (size_t)c * noff, h.data() + (size_t)first[c] * noff, rowbytes);
    cls.alloc(n);
    dict.alloc(hd.size());
    LSG_CUDA(cudaMemcpyAsync(cls.p, hc.data(), n * sizeof(int), cudaMemcpyHostToDevice, s));
    LSG_CUDA(cudaMemcpyAsync(dict.p, hd.data(), hd.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    LSG_CUDA(cudaStreamSynchronize(s));
    return nclass;
}

// Assign every row a class id (first-seen order) and collect the distinct
// rows; rows are compared bit for bit, so the format is lossless.  Built on
// the device (lsg_dict.cuh); the result equals the host build's.
static int build_dict(cudaStream_t s, const double* planes, int noff, long long n, DevBuf<int>& cls,
                      DevBuf<double>& dict)
{
    LSG_REQUIRE(n >= 1 && n < 0x7F7F7F7FLL, LSG_ERR_ARG, "row count out of range for the dictionary build");
    unsigned long long cap = 1;
    while (cap < 2ull * (unsigned long long)n) cap <<= 1;
    int nclass = 0, flag = 0;
    DevBuf<int> repidx, number, tiles, out;
    const long long ntiles = (n + kDictTile - 1) / kDictTile;
    {
        DevBuf<unsigned long long> keys;
        DevBuf<int> rep;
        keys.alloc(cap);
        rep.alloc(cap);
        repidx.alloc(n);
        number.alloc(n);
        tiles.alloc(ntiles);
        out.alloc(2);
        LSG_CUDA(cudaMemsetAsync(keys.p, 0xFF, cap * sizeof(unsigned long long), s));
        LSG_CUDA(cudaMemsetAsync(rep.p, 0x7F, cap * sizeof(int), s));     // 0x7F7F7F7F > every row index
        LSG_CUDA(cudaMemsetAsync(out.p, 0, 2 * sizeof(int), s));
        k_dict_insert<<<grid_for(n, 256), 256, 0, s>>>(noff, n, planes, keys.p, rep.p, cap - 1);
        LSG_CHECK_LAUNCH();
        k_dict_lookup<<<grid_for(n, 256), 256, 0, s>>>(noff, n, planes, keys.p, rep.p, cap - 1, repidx.p, number.p,
                                                       out.p);
        LSG_CHECK_LAUNCH();
        k_dict_tile_count<<<(unsigned)ntiles, kDictTile, 0, s>>>(n, number.p, tiles.p);
        LSG_CHECK_LAUNCH();
        k_dict_scan_tiles<<<1, kDictTile, 0, s>>>((int)ntiles, tiles.p, out.p + 1);
        LSG_CHECK_LAUNCH();
        int h[2];
        LSG_CUDA(cudaMemcpyAsync(h, out.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
        LSG_CUDA(cudaStreamSynchronize(s));
        flag = h[0];
        nclass = h[1];
    }
    if (flag) return build_dict_host(s, planes, noff, n, cls, dict);
    dict.alloc((size_t)nclass * noff);
    cls.alloc(n);
    k_dict_number<<<(unsigned)ntiles, kDictTile, 0, s>>>(noff, n, planes, tiles.p, number.p, dict.p);
    LSG_CHECK_LAUNCH();
    k_dict_classes<<<grid_for(n, 256), 256, 0, s>>>(n, repidx.p, number.p, cls.p);
    LSG_CHECK_LAUNCH();
    LSG_CUDA(cudaStreamSynchronize(s));
    return nclass;
}

// ---------------------------------------------------------------------------
// multigrid setup
// ---------------------------------------------------------------------------
static void upload_tabs(TransferTabs& t, const Dims& f, cudaStream_t s)
{
    const int nf[3] = {f.N, f.M, f.K};
    for (int d = 0; d < 3; d++) {
        std::vector<int> pc, rf;
        std::vector<float> pw, rw;
        prolong_table(nf[d], pc, pw);
        restrict_table(nf[d], rf, rw);
        t.pc[d].alloc(pc.size());
        t.pw[d].alloc(pw.size());
        t.rf[d].alloc(rf.size());
        t.rw[d].alloc(rw.size());
        LSG_CUDA(cudaMemcpyAsync(t.pc[d].p, pc.data(), pc.size() * sizeof(int), cudaMemcpyHostToDevice, s));
        LSG_CUDA(cudaMemcpyAsync(t.pw[d].p, pw.data(), pw.size() * sizeof(float), cudaMemcpyHostToDevice, s));
        LSG_CUDA(cudaMemcpyAsync(t.rf[d].p, rf.data(), rf.size() * sizeof(int), cudaMemcpyHostToDevice, s));
        LSG_CUDA(cudaMemcpyAsync(t.rw[d].p, rw.data(), rw.size() * sizeof(float), cudaMemcpyHostToDevice, s));
    }
}

// Scaled partial-pivoting dense LU of the coarsest operator, a restatement
// of LUDecompositionSparseMatrix::initScalePerm/calcLU
// (Base/SparseMatrix/Decomposition/lu_decomposition_sparse_matrix.h:66-215).
// A is row-major dense; first_col0[i] tells whether the first stored CSR
// entry of row i is in column 0 (the first pivot search only looks there).
static void coarse_lu(int n, const std::vector<double>& A, const std::vector<char>& first_col0,
                      std::vector<double>& L, std::vector<double>& U, std::vector<double>& scale,
                      std::vector<int>& perm)
{
    L.assign((size_t)n * n, 0.0);
    U.assign((size_t)n * n, 0.0);
    scale.assign(n, 1.0);
    perm.resize(n);
    double maxabs = 0.0;
    for (int i = 0; i < n; i++) {
        const double dg = std::fabs(A[(size_t)i * n + i]);
        scale[i] = (dg > 1e-5) ? 1.0 / std::sqrt(dg) : 1.0;
        perm[i] = i;
        for (int j = 0; j < n; j++) maxabs = std::max(maxabs, std::fabs(A[(size_t)i * n + j]));
    }
    const double tiny = 1e-13 * maxabs;
    double maxv = 0.0;
    int piv = 0;
    for (int i = 0; i < n; i++) {
        if (!first_col0[i]) continue;
        const double v = std::fabs(A[(size_t)i * n] * scale[i] * scale[0]);
        if (v > maxv) { maxv = v; piv = i; }
    }
    if (piv != 0) std::swap(perm[0], perm[piv]);
    {
        const int p0 = perm[0];
        for (int j = 0; j < n; j++) U[j] = A[(size_t)p0 * n + j] * scale[p0] * scale[j];
        double u00 = U[0];
        if (std::fabs(u00) < tiny) u00 = (u00 < 0) ? -tiny : tiny;
        U[0] = u00;
        const double inv = scale[0] / u00;
        for (int k = 1; k < n; k++) L[(size_t)k * n] = A[(size_t)perm[k] * n] * scale[perm[k]] * inv;
        L[0] = 1.0;
    }
    std::vector<double> col(n, 0.0);
    for (int i = 1; i < n; i++) {
        maxv = 0.0;
        piv = i;
        const double si = scale[i];
        for (int k = i; k < n; k++) {
            double s = 0.0;
            for (int t = 0; t < i; t++) s += L[(size_t)k * n + t] * U[(size_t)t * n + i];
            const double val = A[(size_t)perm[k] * n + i] * scale[perm[k]] * si - s;
            col[k] = val;
            if (std::fabs(val) > maxv) { maxv = std::fabs(val); piv = k; }
        }
        if (piv != i) {
            std::swap(perm[i], perm[piv]);
            for (int t = 0; t < i; t++) std::swap(L[(size_t)i * n + t], L[(size_t)piv * n + t]);
            std::swap(col[i], col[piv]);
        }
        const int pi = perm[i];
        const double sp = scale[pi];
        for (int j = i; j < n; j++) {
            double s = 0.0;
            for (int t = 0; t < i; t++) s += L[(size_t)i * n + t] * U[(size_t)t * n + j];
            U[(size_t)i * n + j] = A[(size_t)pi * n + j] * sp * scale[j] - s;
        }
        double uii = U[(size_t)i * n + i];
        if (std::fabs(uii) < tiny) uii = (uii < 0) ? -tiny : tiny;
        U[(size_t)i * n + i] = uii;
        const double inv = 1.0 / uii;
        for (int k = i + 1; k < n; k++) L[(size_t)k * n + i] = col[k] * inv;
        L[(size_t)i * n + i] = 1.0;
    }
}

template <typename T>
static void alloc_vectors(LevelT<T>& lv)
{
    const long long n = lv.d.n();
    lv.r.alloc(n);
    lv.c.alloc(n);
    lv.ch.alloc(n);
}

// First level from which the rest of the cycle fits the one-CTA tail kernel:
// every level from there down holds at most kTailMaxCells cells, and every
// smoothed one is a 27-point Galerkin level.
static int tail_first_level(const MGData& mg)
{
    const int L = mg.L;
    if (L < 2) return -1;
    int l0 = -1;
    for (int l = L - 1; l >= 1; l--) {
        const LevelT<double>& lv = mg.l64[l];
        if (lv.d.n() > kTailMaxCells || lv.ol.n != 27 || !lv.dict28.p) break;
        l0 = l;
    }
    if (l0 >= 0 && L - l0 + 1 > kTailMaxLevels) return -1;
    return l0;
}

template <typename T>
static void fill_tail(const MGData& mg, const std::vector<LevelT<T>>& lev, int l0, const Context& C, TailArgs<T>& A)
{
    std::memset(&A, 0, sizeof(A));
    const int L = mg.L;
    A.nlev = L - l0 + 1;
    for (int l = l0; l <= L; l++) {
        TailLevel<T>& t = A.lev[l - l0];
        const LevelT<T>& lv = lev[l];
        t.N = lv.d.N;
        t.M = lv.d.M;
        t.K = lv.d.K;
        t.cls = lv.cls;
        t.dict28 = lv.dict28.p;
        for (int d = 0; d < 3; d++) {
            t.lo[d] = lv.lo[d].p;
            t.dinv[d] = lv.dinv[d].p;
            t.up[d] = lv.up[d].p;
        }
        t.r = const_cast<T*>(lv.r.p);
        t.c = const_cast<T*>(lv.c.p);
        t.ch = const_cast<T*>(lv.ch.p);
        if (l < L) {
            const TransferTabs& tb = mg.tabs[l];
            t.px = tb.P(0);
            t.py = tb.P(1);
            t.pz = tb.P(2);
            t.rx = tb.R(0);
            t.ry = tb.R(1);
            t.rz = tb.R(2);
            t.agg = mg.agg[l] ? 1 : 0;
        }
    }
    A.nc = mg.nc;
    A.L = mg.dL.p;
    A.U = mg.dU.p;
    A.scale = mg.dscale.p;
    A.perm = mg.dperm.p;
    A.work = mg.dwork.p;
    A.n_post = C.opt.n_post;
    A.zquirk = C.opt.zline_reference != 0;
    A.omega = (T)C.opt.omega;
}

static void tail_setup(Context& C)
{
    MGData& mg = C.mg;
    mg.tail_l0 = C.opt.smoother == LSG_SMOOTHER_ADLJ ? tail_first_level(mg) : -1;
    if (mg.tail_l0 < 0) return;
    TailArgs<double> a64;
    fill_tail<double>(mg, mg.l64, mg.tail_l0, C, a64);
    mg.tail64.alloc(1);
    LSG_CUDA(cudaMemcpyAsync(mg.tail64.p, &a64, sizeof(a64), cudaMemcpyHostToDevice, C.s));
    if (mg.fp32) {
        TailArgs<float> a32;
        fill_tail<float>(mg, mg.l32, mg.tail_l0, C, a32);
        mg.tail32.alloc(1);
        LSG_CUDA(cudaMemcpyAsync(mg.tail32.p, &a32, sizeof(a32), cudaMemcpyHostToDevice, C.s));
    }
    LSG_CUDA(cudaStreamSynchronize(C.s));    // the host copies of the arguments go out of scope
}

static void vcycle_graphs_release(MGData& mg);

static void mg_setup(Context& C)
{
    vcycle_graphs_release(C.mg);           // the hierarchy's buffers are rebuilt below
    MGData& mg = C.mg;
    const lsg_options& o = C.opt;
    cudaStream_t s = C.s;
    int L = grid_levels(C.d.N, C.d.M, C.d.K);
    if (o.max_levels > 0) L = std::min(L, o.max_levels);
    LSG_REQUIRE(L >= 1, LSG_ERR_ARG, "grid too small for a multigrid hierarchy (min dimension <= 2)");
    mg.L = L;
    mg.dims.assign(L + 1, Dims());
    mg.tabs.clear();
    mg.tabs.resize(L);
    mg.agg.assign(L, false);
    mg.l64.clear();
    mg.l64.resize(L + 1);
    mg.dims[0] = C.d;
    mg.l64[0].d = C.d;
    mg.l64[0].off.assign(kFine7, kFine7 + 21);
    mg.l64[0].ol = make_offlist(mg.l64[0].off);
    mg.l64[0].A = C.A7.p;
    mg.l64[0].cls = C.cls0.p;
    mg.l64[0].dict = C.dict0.p;
    mg.l64[0].nclass = C.nclass0;
    std::vector<int> rad = {1, 1, 1};
    for (int l = 0; l < L; l++) {
        const Dims f = mg.dims[l];
        bool oN, oM, oK;
        Dims c;
        c.N = coarse_count(f.N, oN);
        c.M = coarse_count(f.M, oM);
        c.K = coarse_count(f.K, oK);
        mg.dims[l + 1] = c;
        const bool agg = !oN && !oM && !oK;
        mg.agg[l] = agg;
        upload_tabs(mg.tabs[l], f, s);
        const int crx = coarse_radius(rad[0], oN, agg), cry = coarse_radius(rad[1], oM, agg),
                  crz = coarse_radius(rad[2], oK, agg);
        LSG_REQUIRE((2 * crx + 1) * (2 * cry + 1) * (2 * crz + 1) <= 125, LSG_ERR_ARG, "coarse stencil too wide");
        LevelT<double>& cl = mg.l64[l + 1];
        cl.d = c;
        cl.off.clear();
        for (int dz = -crz; dz <= crz; dz++)
            for (int dy = -cry; dy <= cry; dy++)
                for (int dx = -crx; dx <= crx; dx++) {
                    cl.off.push_back(dx);
                    cl.off.push_back(dy);
                    cl.off.push_back(dz);
                }
        cl.ol = make_offlist(cl.off);
        cl.Aown.alloc((size_t)cl.ol.n * c.n());
        cl.A = cl.Aown.p;
        const TransferTabs& t = mg.tabs[l];
        k_galerkin<<<grid_for(c.n(), 128), 128, 0, s>>>(f.N, f.M, f.K, mg.l64[l].ol, mg.l64[l].A, c.N, c.M, c.K, crx,
                                                        cry, crz, agg, t.P(0), t.P(1), t.P(2), t.R(0), t.R(1), t.R(2),
                                                        cl.Aown.p);
        LSG_CHECK_LAUNCH();
        cl.nclass = build_dict(s, cl.A, cl.ol.n, c.n(), cl.clsown, cl.dictown);
        cl.cls = cl.clsown.p;
        cl.dict = cl.dictown.p;
        if (cl.ol.n == 27) {
            cl.dict28.alloc((size_t)cl.nclass * 28);
            k_pad_rows<<<grid_for((long long)cl.nclass * 28, 256), 256, 0, s>>>(cl.nclass, 27, 28, cl.dict, cl.dict28.p);
            LSG_CHECK_LAUNCH();
        }
        rad = {crx, cry, crz};
    }
    // ADLJ line factors of every smoothed level
    double* tinyp = C.scal.p;
    int* flag = (int*)(C.scal.p + 8);
    for (int l = 0; l < L; l++) {
        LevelT<double>& lv = mg.l64[l];
        const long long n = lv.d.n();
        for (int d = 0; d < 3; d++) {
            lv.lo[d].alloc(n);
            lv.dinv[d].alloc(n);
            lv.up[d].alloc(n);
        }
        k_adlj_extract<<<grid_for(n, 256), 256, 0, s>>>(lv.d.N, lv.d.M, lv.d.K, lv.ol, lv.A, lv.dinv[0].p, lv.lo[0].p,
                                                       lv.up[0].p, lv.lo[1].p, lv.up[1].p, lv.lo[2].p, lv.up[2].p);
        LSG_CHECK_LAUNCH();
        LSG_CUDA(cudaMemcpyAsync(lv.dinv[1].p, lv.dinv[0].p, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        LSG_CUDA(cudaMemcpyAsync(lv.dinv[2].p, lv.dinv[0].p, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        // tiny = max(1e-5 * max|d|, 1e-12)   (tridiagonal_matrix.h:49-57)
        k_absmax<<<grid_for(n, 256, Reducer::kMaxBlocks), 256, 0, s>>>(n, lv.dinv[0].p, C.red.partial.p,
                                                                      C.red.counter.p, tinyp);
        LSG_CHECK_LAUNCH();
        double maxabs = 0.0;
        LSG_CUDA(cudaMemcpyAsync(&maxabs, tinyp, sizeof(double), cudaMemcpyDeviceToHost, s));
        LSG_CUDA(cudaStreamSynchronize(s));
        double tiny = 1e-5 * maxabs;
        if (tiny < 1e-12) tiny = 1e-12;
        LSG_CUDA(cudaMemcpyAsync(tinyp, &tiny, sizeof(double), cudaMemcpyHostToDevice, s));
        if (o.smoother == LSG_SMOOTHER_RBGS) {           // point pivots from the diagonal, before the line LU
            lv.gsdinv.alloc(n);
            k_gs_dinv<double><<<grid_for(n, 256), 256, 0, s>>>(n, lv.dinv[0].p, tinyp, lv.gsdinv.p);
            LSG_CHECK_LAUNCH();
        }
        for (int d = 0; d < 3; d++) {
            LineGeom g{lv.d.N, lv.d.M, lv.d.K, d};
            LSG_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s));
            k_line_coupling<<<grid_for(g.nlines(), 256), 256, 0, s>>>(g, lv.lo[d].p, lv.up[d].p, flag);
            LSG_CHECK_LAUNCH();
            int coupled = 0;
            LSG_CUDA(cudaMemcpyAsync(&coupled, flag, sizeof(int), cudaMemcpyDeviceToHost, s));
            LSG_CUDA(cudaStreamSynchronize(s));
            if (coupled)
                k_trilu_serial<<<1, 1, 0, s>>>(g, tinyp, lv.lo[d].p, lv.dinv[d].p, lv.up[d].p);
            else
                k_trilu_lines<<<grid_for(g.nlines(), 128), 128, 0, s>>>(g, tinyp, lv.lo[d].p, lv.dinv[d].p, lv.up[d].p);
            LSG_CHECK_LAUNCH();
        }
        alloc_vectors(lv);
    }
    alloc_vectors(mg.l64[L]);
    // coarsest dense LU on the host
    {
        LevelT<double>& cl = mg.l64[L];
        const int nc = (int)cl.d.n();
        LSG_REQUIRE(nc <= 4096, LSG_ERR_ARG, "coarsest level too large for the dense LU");
        const int no = cl.ol.n;
        std::vector<double> box((size_t)no * nc);
        LSG_CUDA(cudaMemcpyAsync(box.data(), cl.A, box.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
        LSG_CUDA(cudaStreamSynchronize(s));
        std::vector<double> A((size_t)nc * nc, 0.0);
        std::vector<char> first0(nc, 0);
        const int N = cl.d.N, M = cl.d.M, K = cl.d.K, NM = N * M;
        for (int i = 0; i < nc; i++) {
            const int z = i / NM, y = (i - z * NM) / N, x = i - z * NM - y * N;
            int firstcol = nc;
            for (int q = 0; q < no; q++) {
                const int jx = x + cl.off[3 * q], jy = y + cl.off[3 * q + 1], jz = z + cl.off[3 * q + 2];
                if (jx < 0 || jx >= N || jy < 0 || jy >= M || jz < 0 || jz >= K) continue;
                const int j = jx + jy * N + jz * NM;
                A[(size_t)i * nc + j] += box[(size_t)q * nc + i];
                firstcol = std::min(firstcol, j);   // structural pattern (sorted CSR)
            }
            first0[i] = (firstcol == 0);
        }
        // the reference's pivot clamp (1e-13 max|A|) keeps any nonzero
        // coarsest matrix factorable; a zero or non-finite one is not
        double amax = 0.0;
        bool finite = true;
        for (const double v : A) {
            finite = finite && std::isfinite(v);
            amax = std::max(amax, std::fabs(v));
        }
        LSG_REQUIRE(finite && amax > 0.0, LSG_ERR_SINGULAR,
                    "coarsest multigrid operator is zero or holds NaN/Inf: no LU factorisation");
        std::vector<double> Lh, Uh, sc;
        std::vector<int> pm;
        coarse_lu(nc, A, first0, Lh, Uh, sc, pm);
        mg.nc = nc;
        mg.dL.alloc(Lh.size());
        mg.dU.alloc(Uh.size());
        mg.dscale.alloc(nc);
        mg.dperm.alloc(nc);
        mg.dwork.alloc(2 * (size_t)nc);
        LSG_CUDA(cudaMemcpyAsync(mg.dL.p, Lh.data(), Lh.size() * 8, cudaMemcpyHostToDevice, s));
        LSG_CUDA(cudaMemcpyAsync(mg.dU.p, Uh.data(), Uh.size() * 8, cudaMemcpyHostToDevice, s));
        LSG_CUDA(cudaMemcpyAsync(mg.dscale.p, sc.data(), sc.size() * 8, cudaMemcpyHostToDevice, s));
        LSG_CUDA(cudaMemcpyAsync(mg.dperm.p, pm.data(), pm.size() * sizeof(int), cudaMemcpyHostToDevice, s));
        LSG_CUDA(cudaStreamSynchronize(s));
    }
    // FP32 shadow hierarchy
    mg.fp32 = (o.mg_precision == LSG_FP32);
    mg.l32.clear();
    if (mg.fp32) {
        mg.l32.resize(L + 1);
        for (int l = 0; l <= L; l++) {
            LevelT<double>& a = mg.l64[l];
            LevelT<float>& b = mg.l32[l];
            b.d = a.d;
            b.off = a.off;
            b.ol = a.ol;
            const long long n = a.d.n();
            b.cls = a.cls;
            b.nclass = a.nclass;
            const long long nd = (long long)a.nclass * a.ol.n;
            b.dictown.alloc(nd);
            b.dict = b.dictown.p;
            k_convert<float, double><<<grid_for(nd, 256), 256, 0, s>>>(nd, a.dict, b.dictown.p);
            LSG_CHECK_LAUNCH();
            if (a.ol.n == 27) {
                const long long n28 = (long long)a.nclass * 28;
                b.dict28.alloc(n28);
                k_convert<float, double><<<grid_for(n28, 256), 256, 0, s>>>(n28, a.dict28.p, b.dict28.p);
                LSG_CHECK_LAUNCH();
            }
            if (l < L && a.gsdinv.p) {
                b.gsdinv.alloc(n);
                k_convert<float, double><<<grid_for(n, 256), 256, 0, s>>>(n, a.gsdinv.p, b.gsdinv.p);
                LSG_CHECK_LAUNCH();
            }
            if (l < L) {
                for (int d = 0; d < 3; d++) {
                    b.lo[d].alloc(n);
                    b.dinv[d].alloc(n);
                    b.up[d].alloc(n);
                    k_convert<float, double><<<grid_for(n, 256), 256, 0, s>>>(n, a.lo[d].p, b.lo[d].p);
                    k_convert<float, double><<<grid_for(n, 256), 256, 0, s>>>(n, a.dinv[d].p, b.dinv[d].p);
                    k_convert<float, double><<<grid_for(n, 256), 256, 0, s>>>(n, a.up[d].p, b.up[d].p);
                    LSG_CHECK_LAUNCH();
                }
            }
            alloc_vectors(b);
        }
    }
    tail_setup(C);
    LSG_CUDA(cudaStreamSynchronize(s));
}

// ---------------------------------------------------------------------------
// V-cycle (MultiGridSolver::solve, multigrid_solver.h:48-75).
// Input: right-hand side already in lev[0].r.  Output: lev[0].ch.
// ---------------------------------------------------------------------------
template <typename T>
static void apply_resid(const LevelT<T>& lv, const T* x, T* r, cudaStream_t s, int mode, int zc27 = 0)
{
    const long long n = lv.d.n();
    // 27-point levels of a million cells or more march 8 z-planes a thread (the
    // two planes loaded ahead of each chunk weigh less; 14.9 against 16.5 us
    // at 128^3 in FP32, measured)
    const int zc = lv.ol.n == 27 ? (zc27 > 0 ? zc27 : (n >= (1LL << 20) ? 8 : zchunk_for(n))) : zchunk_for(n);
    const dim3 zb(32, 8), zg((lv.d.N + 31) / 32, (lv.d.M + 7) / 8, (lv.d.K + zc - 1) / zc);
    if (lv.ol.n == 7 && lv.off[0] == 0 && lv.off[2] == -1) {
        if (mode == 0)
            k_apply7z<T, 0><<<zg, zb, 0, s>>>(lv.d.N, lv.d.M, lv.d.K, zc, lv.cls, lv.dict, x, r);
        else
            k_apply7z<T, 1><<<zg, zb, 0, s>>>(lv.d.N, lv.d.M, lv.d.K, zc, lv.cls, lv.dict, x, r);
    } else if (lv.ol.n == 27 && lv.dict28.p) {
        if (mode == 0)
            k_apply27z<T, 0><<<zg, zb, 0, s>>>(lv.d.N, lv.d.M, lv.d.K, zc, lv.cls, lv.dict28.p, x, r);
        else
            k_apply27z<T, 1><<<zg, zb, 0, s>>>(lv.d.N, lv.d.M, lv.d.K, zc, lv.cls, lv.dict28.p, x, r);
    } else {
        if (mode == 0)
            k_applyboxd<T, 0><<<grid_for(n, 256), 256, 0, s>>>(lv.d.N, lv.d.M, lv.d.K, lv.ol, lv.cls, lv.dict, x, r);
        else
            k_applyboxd<T, 1><<<grid_for(n, 256), 256, 0, s>>>(lv.d.N, lv.d.M, lv.d.K, lv.ol, lv.cls, lv.dict, x, r);
    }
    LSG_CHECK_LAUNCH();
}

template <typename T>
static void line_solve(const LevelT<T>& lv, int d, bool zquirk, T omega, cudaStream_t s, T* ch = nullptr,
                       int form = 0)
{
    const bool walk = form == 1;
    if (!ch) ch = const_cast<T*>(lv.ch.p);
    const Dims& g = lv.d;
    if (d == 0) {
        const long long nl = (long long)g.M * g.K;
        // whole lines per warp with 16-byte aligned segments: lengths SEG * P,
        // P a power of two <= 32 (SEG 8: 8..256, SEG 12: 12..384)
        auto xseg_p = [&](int seg) {
            if (g.N % seg) return 0;
            const int P = g.N / seg;
            return (P <= 32 && (P & (P - 1)) == 0) ? P : 0;
        };
        const bool aligned = ((reinterpret_cast<uintptr_t>(ch) | reinterpret_cast<uintptr_t>(lv.c.p)) & 15) == 0;
        const int P8 = xseg_p(8), P12 = xseg_p(12);
        if (aligned && P8) {
            const long long threads = nl * P8;
            k_tdma_xseg<T, 8><<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(
                g.N, P8, nl, lv.lo[0].p, lv.dinv[0].p, lv.up[0].p, lv.r.p, lv.c.p, ch, omega);
        } else if (aligned && P12) {
            const long long threads = nl * P12;
            k_tdma_xseg<T, 12><<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(
                g.N, P12, nl, lv.lo[0].p, lv.dinv[0].p, lv.up[0].p, lv.r.p, lv.c.p, ch, omega);
        } else {
            const int blocks = grid_for(nl * 32, 256, 148 * 64);
            k_tdma_xwarp<T><<<blocks, 256, 0, s>>>(g.N, nl, lv.lo[0].p, lv.dinv[0].p, lv.up[0].p, lv.r.p, lv.c.p,
                                                   ch, omega);
        }
    } else {
        LineGeom lg{g.N, g.M, g.K, d};
        constexpr int MAXT = sizeof(T) == 4 ? 512 : 256;
        const int L = lg.len();
        const long long rows = d == 1 ? g.K : g.M;
        // W lines per CTA (as many as fit MAXT threads, at most 32: one warp
        // row of x) times S segments; the segment chain is sequential, so in
        // FP32 longer segments (12 cells) are used where 8-cell ones would
        // give more than 32 of them.  In FP64 the 12-cell segments need 166
        // registers a thread, and at 384^3 the strided solve measured faster.
        auto pick_w = [&](int S) {
            int W = 8;
            while (W < 32 && 2 * W * S <= MAXT) W *= 2;
            return W;
        };
        const int S8 = (L + 7) / 8, S12 = (L + 11) / 12, S4 = (L + 3) / 4;
        // FP64 z-lines: 4-cell segments in 512-thread CTAs (59 registers, two
        // CTAs per SM instead of one 126-register CTA of 8-cell segments:
        // 246 against 276 us at 256^3, measured); form 2 forces them
        const bool seg4 = (form == 2 || (form == 0 && sizeof(T) == 8 && d == 2)) && 8 * S4 <= 512;
        if (seg4) {
            const long long blocks = (long long)((g.N + 7) / 8) * rows;
            k_tdma_seg<T, 4, 512, 2><<<(unsigned)blocks, dim3(8, S4), 4 * (size_t)8 * S4 * sizeof(T), s>>>(
                lg, d == 2 && zquirk, lv.lo[d].p, lv.dinv[d].p, lv.up[d].p, lv.r.p, lv.c.p, ch, omega);
        } else if (8 * S8 <= MAXT && (S8 <= 32 || 8 * S12 > MAXT)) {
            const int W = pick_w(S8);
            const long long blocks = (long long)((g.N + W - 1) / W) * rows;
            if (walk)
                k_tdma_seg<T, 8, MAXT, 2, false><<<(unsigned)blocks, dim3(W, S8), 4 * (size_t)W * S8 * sizeof(T), s>>>(
                    lg, d == 2 && zquirk, lv.lo[d].p, lv.dinv[d].p, lv.up[d].p, lv.r.p, lv.c.p, ch, omega);
            else
                k_tdma_seg<T, 8, MAXT, 2><<<(unsigned)blocks, dim3(W, S8), 4 * (size_t)W * S8 * sizeof(T), s>>>(
                    lg, d == 2 && zquirk, lv.lo[d].p, lv.dinv[d].p, lv.up[d].p, lv.r.p, lv.c.p, ch, omega);
        } else if (sizeof(T) == 4 && 8 * S12 <= MAXT) {
            const int W = pick_w(S12);
            const long long blocks = (long long)((g.N + W - 1) / W) * rows;
            k_tdma_seg<T, 12, MAXT, 1><<<(unsigned)blocks, dim3(W, S12), 4 * (size_t)W * S12 * sizeof(T), s>>>(
                lg, d == 2 && zquirk, lv.lo[d].p, lv.dinv[d].p, lv.up[d].p, lv.r.p, lv.c.p, ch, omega);
        } else {
            k_tdma_strided<T><<<grid_for(lg.nlines(), 128, 148 * 64), 128, 0, s>>>(
                lg, d == 2 && zquirk, lv.lo[d].p, lv.dinv[d].p, lv.up[d].p, lv.r.p, lv.c.p, ch, omega);
        }
    }
    LSG_CHECK_LAUNCH();
}

// y/z-line shapes of the segmented kernels: 8-cell segments (two CTAs of
// MAXT threads per SM) where a line has at most 32 of them or 12-cell ones
// would not fit either, else 12-cell segments (FP32 only); 0 = neither.
template <typename T>
static int seg_cells(int L)
{
    constexpr int MAXT = sizeof(T) == 4 ? 512 : 256;
    const int S8 = (L + 7) / 8, S12 = (L + 11) / 12;
    if (8 * S8 <= MAXT && (S8 <= 32 || 8 * S12 > MAXT)) return 8;
    if (sizeof(T) == 4 && 8 * S12 <= MAXT) return 12;
    return 0;
}

// Segment length of the fused x-line step: N = SEG * P with P <= 32 lanes, P a
// power of two, 8-cell segments where they fit (lines of 8..256), else 12-cell
// ones (12..384), else 16-cell ones (16..512); 0 = none.
static int xseg_cells(int N)
{
    for (int seg : {8, 12, 16}) {
        if (N % seg) continue;
        const int P = N / seg;
        if (P <= 32 && (P & (P - 1)) == 0) return seg;
    }
    return 0;
}

// Whether a level with these dimensions and stencil runs the fused ADLJ
// direction steps: the fine 7-point stencil (offsets b, s, w, p, e, n, t),
// x-lines of 8-, 12- or 16-cell segments on P <= 32 lanes (P a power of two),
// y- and z-lines in the segmented kernel's shapes.
template <typename T>
static bool adlj_fused_level(const Dims& g, int noff, const std::vector<int>& off, const lsg_options& o)
{
    if (o.smoother != LSG_SMOOTHER_ADLJ) return false;
    if (!(o.adlj_schedule == LSG_ADLJ_FUSED || (o.adlj_schedule == LSG_ADLJ_AUTO && sizeof(T) == 4))) return false;
    if (noff != 7 || off.size() < 3 || off[0] != 0 || off[1] != 0 || off[2] != -1) return false;
    if (g.N < 2 || g.M < 2 || g.K < 2 || !xseg_cells(g.N)) return false;
    return seg_cells<T>(g.M) != 0 && seg_cells<T>(g.K) != 0;
}

// The fused y (DIR 1) or z (DIR 2) step in the form VAR of k_adlj_fused_seg:
// W lines x S segments per CTA of at most MAXT threads.  FP32 y-lines of more
// than 32 8-cell segments keep 8-cell segments while they fit (at 384^3: 558
// against 868 us with 12-cell ones; z-lines the other way, 587 against 830 us).
template <typename T, int DIR, int VAR>
static void launch_fused_seg(const LevelT<T>& lv, bool zq, T omega, cudaStream_t s, const T* dinv, const T* xin,
                             T* xout)
{
    constexpr int MAXT = sizeof(T) == 4 ? 512 : 256;
    const Dims& g = lv.d;
    const int L = DIR == 1 ? g.M : g.K;
    const long long rows = DIR == 1 ? g.K : g.M;
    const int seg = (sizeof(T) == 4 && DIR == 1 && 8 * ((L + 7) / 8) <= MAXT) ? 8 : seg_cells<T>(L);
    const int S = (L + seg - 1) / seg;
    int W = 8;                                             // lanes per line row: a divisor of 32
    while (W < 32 && 2 * W * S <= MAXT) W *= 2;
    const unsigned blocks = (unsigned)((long long)((g.N + W - 1) / W) * rows);
    const dim3 blk(W, S);
    const size_t sm = 4 * (size_t)W * S * sizeof(T);       // scan buffers
    const T* dict = lv.dict;
    if (seg == 8) {
        k_adlj_fused_seg<T, DIR, 8, MAXT, 2, VAR><<<blocks, blk, sm, s>>>(g.N, g.M, g.K, zq, lv.cls, dict, dinv,
                                                                         lv.r.p, xin, xout, omega);
    } else {
        if constexpr (sizeof(T) == 4)
            k_adlj_fused_seg<T, DIR, 12, MAXT, 1, VAR><<<blocks, blk, sm, s>>>(g.N, g.M, g.K, zq, lv.cls, dict,
                                                                              dinv, lv.r.p, xin, xout, omega);
        else
            throw Error{LSG_ERR_STATE, "no fused line kernel for this line length"};
    }
}

// One fused ADLJ direction step on level lv:  xout = xin + omega T_d^{-1} (b - A xin),
// b = the level's right-hand side (lv.r, left unchanged).  scan: the y/z
// kernel composes its segment maps by log-step scans (the solve's form;
// false: each thread walks them, kept for timing comparisons).
template <typename T>
static void adlj_fused_step(const LevelT<T>& lv, int d, bool zquirk, T omega, cudaStream_t s, const T* xin, T* xout,
                            bool scan = true)
{
    const Dims& g = lv.d;
    const T* b = lv.r.p;
    const T* dinv = lv.dinv[d].p;
    if (d == 0) {
        const int seg = xseg_cells(g.N);
        const int P = g.N / seg;
        const long long threads = (long long)g.M * g.K * P;
        if (seg == 8)
            k_adlj_fused_xseg<T, 8><<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(g.N, g.M, g.K, P, lv.cls,
                                                                                    lv.dict, dinv, b, xin, xout, omega);
        else if (seg == 12)
            k_adlj_fused_xseg<T, 12><<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(g.N, g.M, g.K, P, lv.cls,
                                                                                     lv.dict, dinv, b, xin, xout,
                                                                                     omega);
        else
            k_adlj_fused_xseg<T, 16><<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(g.N, g.M, g.K, P, lv.cls,
                                                                                     lv.dict, dinv, b, xin, xout,
                                                                                     omega);
    } else {
        const bool zq = d == 2 && zquirk;
        if (scan) {
            // y-lines that split into whole segments drop the line-end guards
            // (256^3 FP32: 112 against 131 us; the z step measured 140
            // against 135 us that way and keeps them)
            const int L = g.M;
            const int sgl = (sizeof(T) == 4 && 8 * ((L + 7) / 8) <= 512) ? 8 : seg_cells<T>(L);
            if (d == 1) {
                if (L % sgl == 0) launch_fused_seg<T, 1, 3>(lv, false, omega, s, dinv, xin, xout);
                else launch_fused_seg<T, 1, 1>(lv, false, omega, s, dinv, xin, xout);
            } else {
                launch_fused_seg<T, 2, 1>(lv, zq, omega, s, dinv, xin, xout);
            }
        } else {
            if (d == 1) launch_fused_seg<T, 1, 0>(lv, false, omega, s, dinv, xin, xout);
            else launch_fused_seg<T, 2, 0>(lv, zq, omega, s, dinv, xin, xout);
        }
    }
    LSG_CHECK_LAUNCH();
}

// One smoothing sweep of the multi-colour Gauss-Seidel variant on level lv:
// colours in increasing order (forward) or decreasing order (backward, for
// the post-smoothing of a symmetric cycle).
template <typename T>
static void gs_sweep(const LevelT<T>& lv, const T* b, T* x, bool backward, cudaStream_t s)
{
    const Dims& d = lv.d;
    if (lv.ol.n == 7 && lv.off[0] == 0 && lv.off[2] == -1) {
        const dim3 g((d.N / 2 + 1 + 31) / 32, (d.M + 7) / 8, d.K);
        for (int q = 0; q < 2; q++) {
            k_gs_rb7<T><<<g, dim3(32, 8), 0, s>>>(d.N, d.M, d.K, backward ? 1 - q : q, lv.cls, lv.dict,
                                                  lv.gsdinv.p, b, x);
            LSG_CHECK_LAUNCH();
        }
    } else if (lv.ol.n == 27 && lv.dict28.p) {
        const dim3 g(((d.N + 1) / 2 + 31) / 32, ((d.M + 1) / 2 + 7) / 8, (d.K + 1) / 2);
        for (int q = 0; q < 8; q++) {
            k_gs_box27<T><<<g, dim3(32, 8), 0, s>>>(d.N, d.M, d.K, backward ? 7 - q : q, lv.cls, lv.dict28.p,
                                                    lv.gsdinv.p, b, x);
            LSG_CHECK_LAUNCH();
        }
    } else {
        // wider stencils (mixed-parity coarsening): one damped Jacobi step
        T* t = const_cast<T*>(lv.c.p);
        const long long n = d.n();
        apply_resid<T>(lv, x, t, s, 1);                 // t = A x
        k_sub_from<T><<<grid_for(n, 256), 256, 0, s>>>(n, b, t);
        LSG_CHECK_LAUNCH();
        k_jacobi_update<T><<<grid_for(n, 256), 256, 0, s>>>(n, lv.gsdinv.p, t, x);
        LSG_CHECK_LAUNCH();
    }
}

// V(n_pre, n_post) cycle with the multi-colour Gauss-Seidel smoother (the
// red-black variant): on the way down each level starts from zero, is
// pre-smoothed, and restricts its residual; the coarsest level is solved by
// the dense LU; on the way up the prolonged correction is added and
// post-smoothed.  Same hierarchy, transfers and coarsest solve as the
// reference-shaped cycle.
template <typename T>
static void vcycle_rb(Context& C, std::vector<LevelT<T>>& lev, T* ch0)
{
    MGData& mg = C.mg;
    cudaStream_t s = C.s;
    const int L = mg.L;
    const int npre = C.opt.n_pre, npost = C.opt.n_post;
    for (int l = 0; l < L; l++) {
        LevelT<T>& lv = lev[l];
        const Dims& f = lv.d;
        const Dims& c = lev[l + 1].d;
        T* x = (l == 0 && ch0) ? ch0 : lv.ch.p;
        const T* res = lv.r.p;
        if (npre > 0) {
            LSG_CUDA(cudaMemsetAsync(x, 0, f.n() * sizeof(T), s));
            for (int it = 0; it < npre; it++) gs_sweep<T>(lv, lv.r.p, x, false, s);
            // residual r - A x into c
            LSG_CUDA(cudaMemcpyAsync(lv.c.p, lv.r.p, f.n() * sizeof(T), cudaMemcpyDeviceToDevice, s));
            apply_resid<T>(lv, x, lv.c.p, s, 0);
            res = lv.c.p;
        }
        const TransferTabs& t = mg.tabs[l];
        k_restrict<T><<<grid_for(c.n(), 256), 256, 0, s>>>(c.N, c.M, c.K, f.N, f.M, mg.agg[l], t.R(0), t.R(1), t.R(2),
                                                          res, lev[l + 1].r.p);
        LSG_CHECK_LAUNCH();
    }
    k_coarse_solve<T><<<1, 32, 0, s>>>(mg.nc, mg.dL.p, mg.dU.p, mg.dscale.p, mg.dperm.p, lev[L].r.p, lev[L].ch.p,
                                       mg.dwork.p);
    LSG_CHECK_LAUNCH();
    for (int l = L - 1; l >= 0; l--) {
        LevelT<T>& lv = lev[l];
        const Dims& f = lv.d;
        const TransferTabs& t = mg.tabs[l];
        T* x = (l == 0 && ch0) ? ch0 : lv.ch.p;
        constexpr int PZ = 4;
        const dim3 pg((f.N + 31) / 32, (f.M + 7) / 8, (f.K + PZ - 1) / PZ);
        if (npre > 0) {
            k_prolong<T, PZ, true><<<pg, dim3(32, 8), 0, s>>>(f.N, f.M, f.K, lev[l + 1].d.N, lev[l + 1].d.M, t.P(0),
                                                              t.P(1), t.P(2), lev[l + 1].ch.p, x, lv.c.p);
        } else {
            k_prolong<T, PZ><<<pg, dim3(32, 8), 0, s>>>(f.N, f.M, f.K, lev[l + 1].d.N, lev[l + 1].d.M, t.P(0), t.P(1),
                                                        t.P(2), lev[l + 1].ch.p, x, lv.c.p);
        }
        LSG_CHECK_LAUNCH();
        for (int it = 0; it < npost; it++) gs_sweep<T>(lv, lv.r.p, x, true, s);
    }
    C.vcycles++;
}

// ch0: where the finest-level correction (the preconditioned vector) goes;
// nullptr = the level's own buffer.
template <typename T>
static void vcycle(Context& C, std::vector<LevelT<T>>& lev, T* ch0 = nullptr)
{
    if (C.opt.smoother == LSG_SMOOTHER_RBGS) {
        vcycle_rb<T>(C, lev, ch0);
        return;
    }
    MGData& mg = C.mg;
    cudaStream_t s = C.s;
    const int L = mg.L;
    const int lt = mg.tail_l0;              // levels lt..L run inside k_vcycle_tail
    for (int l = 0; l < (lt >= 0 ? lt : L); l++) {
        const Dims& f = lev[l].d;
        const Dims& c = lev[l + 1].d;
        const TransferTabs& t = mg.tabs[l];
        k_restrict<T><<<grid_for(c.n(), 256), 256, 0, s>>>(c.N, c.M, c.K, f.N, f.M, mg.agg[l], t.R(0), t.R(1), t.R(2),
                                                          lev[l].r.p, lev[l + 1].r.p);
        LSG_CHECK_LAUNCH();
    }
    if (lt >= 0) {
        if constexpr (sizeof(T) == 8) k_vcycle_tail<double><<<1, kTailThreads, 0, s>>>(mg.tail64.p);
        else k_vcycle_tail<float><<<1, kTailThreads, 0, s>>>(mg.tail32.p);
    } else {
        k_coarse_solve<T><<<1, 32, 0, s>>>(mg.nc, mg.dL.p, mg.dU.p, mg.dscale.p, mg.dperm.p, lev[L].r.p, lev[L].ch.p,
                                           mg.dwork.p);
    }
    LSG_CHECK_LAUNCH();
    const T omega = (T)C.opt.omega;
    const bool zq = C.opt.zline_reference != 0;
    for (int l = (lt >= 0 ? lt : L) - 1; l >= 0; l--) {
        LevelT<T>& lv = lev[l];
        const Dims& f = lv.d;
        const TransferTabs& t = mg.tabs[l];
        T* chl = (l == 0 && ch0) ? ch0 : lv.ch.p;
        const int order[3] = {2, 1, 0};           // SmootherADLJ::solve: z, y, x
        const int steps = 3 * C.opt.n_post;
        const bool aligned = ((reinterpret_cast<uintptr_t>(chl) | reinterpret_cast<uintptr_t>(lv.c.p) |
                               reinterpret_cast<uintptr_t>(lv.r.p) | reinterpret_cast<uintptr_t>(lv.cls)) & 15) == 0;
        const bool fused = steps > 0 && aligned && adlj_fused_level<T>(f, lv.ol.n, lv.off, C.opt);
        // the fused steps alternate the iterate between c and chl, starting from
        // the buffer that makes the last step write chl: the prolongation fills
        // that one only; the reference schedule needs P c_H in both
        T* buf[2] = {chl, lv.c.p};
        int cur = steps % 2;
        constexpr int PZ = 4;
        const dim3 pg((f.N + 31) / 32, (f.M + 7) / 8, (f.K + PZ - 1) / PZ);
        if (fused)
            k_prolong<T, PZ><<<pg, dim3(32, 8), 0, s>>>(f.N, f.M, f.K, lev[l + 1].d.N, lev[l + 1].d.M, t.P(0), t.P(1),
                                                        t.P(2), lev[l + 1].ch.p, buf[cur], nullptr);
        else
            k_prolong<T, PZ><<<pg, dim3(32, 8), 0, s>>>(f.N, f.M, f.K, lev[l + 1].d.N, lev[l + 1].d.M, t.P(0), t.P(1),
                                                        t.P(2), lev[l + 1].ch.p, chl, lv.c.p);
        LSG_CHECK_LAUNCH();
        if (fused) {
            for (int it = 0; it < C.opt.n_post; it++)
                for (int q = 0; q < 3; q++) {
                    adlj_fused_step<T>(lv, order[q], zq, omega, s, buf[cur], buf[cur ^ 1]);
                    cur ^= 1;
                }
        } else {
            for (int it = 0; it < C.opt.n_post; it++)
                for (int q = 0; q < 3; q++) {
                    apply_resid<T>(lv, lv.c.p, lv.r.p, s, 0);        // calcRes: r -= A c
                    line_solve<T>(lv, order[q], zq, omega, s, chl);  // c = omega T^-1 r ; ch += c
                }
        }
    }
    C.vcycles++;
}

static void vcycle_graphs_release(MGData& mg)
{
    if (mg.cycle64) cudaGraphExecDestroy(mg.cycle64);
    if (mg.cycle32) cudaGraphExecDestroy(mg.cycle32);
    mg.cycle64 = mg.cycle32 = nullptr;
}

// One ADLJ V-cycle replayed from a CUDA graph: the cycle's launches (about 20
// per level above the tail kernel) only touch the hierarchy's own buffers, so
// they are captured once and submitted as one unit, which removes the host
// submission gaps of the small coarse-level kernels.  The correction is left
// in level 0's ch; ch0 (if given) receives a copy.  Contexts on the legacy
// default stream and the Gauss-Seidel cycle run the launches directly.
template <typename T>
static void vcycle_run(Context& C, std::vector<LevelT<T>>& lev, T* ch0)
{
    if (!C.s || C.opt.smoother == LSG_SMOOTHER_RBGS) {
        vcycle<T>(C, lev, ch0);
        return;
    }
    cudaGraphExec_t& exec = sizeof(T) == 8 ? C.mg.cycle64 : C.mg.cycle32;
    if (!exec) {
        cudaGraph_t graph = nullptr;
        LSG_CUDA(cudaStreamBeginCapture(C.s, cudaStreamCaptureModeThreadLocal));
        Error captured{LSG_OK, ""};
        try {
            vcycle<T>(C, lev, nullptr);
        } catch (const Error& e) {
            captured = e;
        }
        const cudaError_t cap_err = cudaStreamEndCapture(C.s, &graph);
        if (captured.code != LSG_OK) {
            if (graph) cudaGraphDestroy(graph);
            throw captured;
        }
        LSG_CUDA(cap_err);
        size_t nodes = 0;
        cudaGraphGetNodes(graph, nullptr, &nodes);
        (sizeof(T) == 8 ? C.mg.cycle64_nodes : C.mg.cycle32_nodes) = (long long)nodes;
        const cudaError_t inst_err = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (inst_err != cudaSuccess) exec = nullptr;
        LSG_CUDA(inst_err);
        C.vcycles--;                       // the capture only recorded the cycle
    }
    LSG_CUDA(cudaGraphLaunch(exec, C.s));
    // launch accounting counts the kernels the replay runs
    ::lsg::g_launches += sizeof(T) == 8 ? C.mg.cycle64_nodes : C.mg.cycle32_nodes;
    C.vcycles++;
    if (ch0)
        LSG_CUDA(cudaMemcpyAsync(ch0, lev[0].ch.p, (size_t)lev[0].d.n() * sizeof(T), cudaMemcpyDeviceToDevice, C.s));
}

// Algorithmic bytes of one V-cycle with element size w (documented model).
static double vcycle_bytes(const MGData& mg, const lsg_options& o, double w)
{
    double b = 0;
    for (int l = 0; l <= mg.L; l++) {
        const double n = (double)mg.dims[l].n();
        if (l < mg.L) {
            b += (1.0 + 0.125) * w * n;                      // restriction read fine + write coarse
            const LevelT<double>& lp = mg.l64[l];
            const bool fused_l = o.smoother == LSG_SMOOTHER_ADLJ && o.n_post > 0 &&
                                 (w == 4.0 ? adlj_fused_level<float>(mg.dims[l], lp.ol.n, lp.off, o)
                                           : adlj_fused_level<double>(mg.dims[l], lp.ol.n, lp.off, o));
            // prolongation: read coarse, write ch and c (one of them ahead of
            // the fused smoother; ch read and written in the Gauss-Seidel cycle)
            b += (0.125 + (fused_l ? 1.0 : 2.0)) * w * n;
            if (o.smoother == LSG_SMOOTHER_RBGS) {
                // full colour sweep: b, x read, x written, row class 4 B; pre-smoothed
                // levels also form their residual (copy 2w + apply 3w + 4)
                b += (o.n_pre + o.n_post) * (3.0 * w + 4.0) * n;
                if (o.n_pre > 0) b += (5.0 * w + 4.0) * n;
            } else {
                // per direction, fused step: b, iterate, dinv read, iterate written,
                // row class 4 B (the distinct-row table is L2 resident); otherwise
                // residual (r rw, c; row class) + line solve (r, lo, dinv, up, ch
                // read; c, ch written)
                const LevelT<double>& lv = mg.l64[l];
                const bool fused = w == 4.0 ? adlj_fused_level<float>(mg.dims[l], lv.ol.n, lv.off, o)
                                            : adlj_fused_level<double>(mg.dims[l], lv.ol.n, lv.off, o);
                b += 3.0 * o.n_post * (fused ? 4.0 * w + 4.0 : (3.0 * w + 4.0) + 7.0 * w) * n;
            }
        }
    }
    return b;
}

// ---------------------------------------------------------------------------
// preconditioner application z = M^{-1} v  (v FP64 on the device)
// ---------------------------------------------------------------------------
static void precond_apply(Context& C, const double* v, double* z)
{
    cudaStream_t s = C.s;
    const long long n = C.n;
    if (C.opt.precond == LSG_PC_NONE) {
        LSG_CUDA(cudaMemcpyAsync(z, v, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        return;
    }
    if (C.opt.precond == LSG_PC_ILU0) {
        ilu_apply(C, v, z);
        return;
    }
    if (C.mg.fp32) {
        auto& lev = C.mg.l32;
        k_convert<float, double><<<grid_for(n, 256), 256, 0, s>>>(n, v, lev[0].r.p);
        LSG_CHECK_LAUNCH();
        vcycle_run<float>(C, lev, nullptr);
        k_convert<double, float><<<grid_for(n, 256), 256, 0, s>>>(n, lev[0].ch.p, z);
        LSG_CHECK_LAUNCH();
    } else {
        auto& lev = C.mg.l64;
        LSG_CUDA(cudaMemcpyAsync(lev[0].r.p, v, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        vcycle_run<double>(C, lev, nullptr);
        LSG_CUDA(cudaMemcpyAsync(z, lev[0].ch.p, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
}

// ---------------------------------------------------------------------------
// FGMRES (FGMRESInterface::solve, fgmres_interface.h:78-142)
// ---------------------------------------------------------------------------
static void launch_givens(Context& C, int j)
{
    k_givens<<<1, 32, 0, C.s>>>(C.ks.p, j, 65, C.opt.eps, C.opt.max_it, C.hflag, C.hnorm);
    LSG_CHECK_LAUNCH();
}

// Low-synchronisation MGS for Arnoldi step j: one pass for V^T w and the new
// row of V^T V, a triangular correction, one update pass (with ||w||^2).
// Fine-grid Krylov product fused with one dot (k_krylov7s, z planes staged in
// shared memory): MODE 0 w = A z, out = (w, v); MODE 1 w = v - A z,
// out = ||w||^2.  The z-chunk is at least 8 planes (each CTA stages two planes
// beyond its chunk) and doubles until the grid has at most 4096 blocks; wider
// grids use the one-thread-per-cell kernels.
template <typename Tz, int MODE>
static void krylov7(Context& C, const Tz* z, const double* v, double* w, double* out)
{
    const Dims& d = C.d;
    const long long gx = (d.N + 31) / 32, gy = (d.M + 7) / 8;
    constexpr long long cap = 4096;
    if (gx * gy <= cap) {
        int zc = std::max(zchunk_for(C.n), 8);
        while (gx * gy * ((d.K + zc - 1) / zc) > cap) zc *= 2;
        const dim3 grid((unsigned)gx, (unsigned)gy, (unsigned)((d.K + zc - 1) / zc));
        k_krylov7s<Tz, MODE><<<grid, dim3(32, 8), 0, C.s>>>(d.N, d.M, d.K, zc, C.cls0.p, C.dict0.p, z, v, w,
                                                             C.red.partial.p, C.red.counter.p, out);
    } else {
        const int gb = grid_for(C.n, 256, Reducer::kMaxBlocks);
        if constexpr (MODE == 0)
            k_spmv_dot7<Tz><<<gb, 256, 0, C.s>>>(d.N, d.M, d.K, C.cls0.p, C.dict0.p, z, v, w, C.red.partial.p,
                                                 C.red.counter.p, out);
        else
            k_residual7<<<gb, 256, 0, C.s>>>(d.N, d.M, d.K, C.cls0.p, C.dict0.p, z, v, w, C.red.partial.p,
                                             C.red.counter.p, out);
    }
    LSG_CHECK_LAUNCH();
}

static void gs_lowsync(Context& C, int j, int gb, double* Hj)
{
    const long long n = C.n;
    // about 32 resident warps per SM whatever the number of vector groups
    const int groups = (j + 4) / 4;
    const int gd = (int)std::min<long long>((n + 127) / 128, std::max(148, 148 * 32 / groups));
    k_gs_dots2<<<gd, dim3(32, (j + 4) / 4), 0, C.s>>>(n, C.ldv, j, C.V.p, C.w.p, C.gs_partial.p, C.red.counter.p,
                                                      C.gs_sg.p);
    LSG_CHECK_LAUNCH();
    k_gs_tri<<<1, 32, 0, C.s>>>(C.ks.p, j, 65, C.gs_sg.p, C.gs_L.p);
    LSG_CHECK_LAUNCH();
    k_gs_update2<<<gb, 256, 0, C.s>>>(n, C.ldv, j, C.V.p, Hj, C.w.p, C.red.partial.p, C.red.counter.p,
                                      &C.ks.p->normW2);
    LSG_CHECK_LAUNCH();
}

static int fgmres(Context& C, double* x, const double* b, lsg_stats* st)
{
    cudaStream_t s = C.s;
    const long long n = C.n;
    const int m = C.restart;
    const int gb = grid_for(n, 256, Reducer::kMaxBlocks);
    double* part = C.red.partial.p;
    unsigned int* cnt = C.red.counter.p;
    KrylovScalars* ks = C.ks.p;
    const double w8 = 8.0;
    double bytes = 0;
    // norm_r = ||b - A x||  ; w = b - A x
    krylov7<double, 1>(C, x, b, C.w.p, &ks->normW2);
    bytes += (3 * w8 + 4) * n;
    double nrm2 = 0;
    LSG_CUDA(cudaMemcpyAsync(&nrm2, &ks->normW2, sizeof(double), cudaMemcpyDeviceToHost, s));
    LSG_CUDA(cudaStreamSynchronize(s));
    double norm_r = std::sqrt(nrm2);
    int it = 0;
    int status = LSG_OK;
    // a NaN or Inf in b, x or the operator: no iteration can help (the
    // reference would iterate to MAX_ITER on NaNs and report nothing)
    if (!std::isfinite(norm_r)) status = LSG_BREAKDOWN;
    else if (norm_r > C.opt.eps) {
        it = 1;
        // initialise device scalars: norm_r, invNormW = 1/norm_r, it
        KrylovScalars h;
        std::memset(&h, 0, sizeof(h));
        h.norm_r = norm_r;
        h.invNormW = 1.0 / norm_r;
        h.it = 1;
        LSG_CUDA(cudaMemcpyAsync(ks, &h, sizeof(h), cudaMemcpyHostToDevice, s));
        bool finished = false;
        while (!finished) {
            int jlast = m - 1;
            for (int j = 0; j < m; j++) {
                double* vj = C.V.p + (size_t)j * C.ldv;
                double* zj = C.Z.p + (size_t)j * C.ldv;
                // v_j = w / ||w|| (also the preconditioner input)
                const bool z32 = C.mg.fp32 && C.opt.precond == LSG_PC_MG;
                float* zj32 = z32 ? C.Z32.p + (size_t)j * C.ldv : nullptr;
                if (z32) {
                    // the FP32 cycle writes z_j directly; it is kept in FP32
                    // (exactly representable in FP64, so the Arnoldi relation
                    // w = A z_j below holds for the stored z_j)
                    k_scale_copy<float><<<grid_for(n, 256), 256, 0, s>>>(n, C.w.p, &ks->invNormW, vj, C.mg.l32[0].r.p);
                    LSG_CHECK_LAUNCH();
                    vcycle_run<float>(C, C.mg.l32, zj32);
                    bytes += (8 + 8 + 4) * (double)n + vcycle_bytes(C.mg, C.opt, 4.0);
                } else {
                    k_scale_copy<double><<<grid_for(n, 256), 256, 0, s>>>(n, C.w.p, &ks->invNormW, vj, C.t1.p);
                    LSG_CHECK_LAUNCH();
                    precond_apply(C, C.t1.p, zj);
                    bytes += 24.0 * n + (C.opt.precond == LSG_PC_MG ? vcycle_bytes(C.mg, C.opt, 8.0) + 32.0 * n : 0);
                }
                // w = A z_j ; H[0,j] = (w, v_0)
                double* Hj = ks->H + (size_t)j * 65;
                if (z32) krylov7<float, 0>(C, zj32, C.V.p, C.w.p, Hj);
                else krylov7<double, 0>(C, zj, C.V.p, C.w.p, Hj);
                bytes += (3 * w8 + 4) * n;
                if (C.opt.gram_schmidt == LSG_GS_LOWSYNC) {
                    gs_lowsync(C, j, gb, Hj);
                    bytes += (2.0 * j + 5.0) * w8 * n;
                } else {
                    // modified Gram-Schmidt: w -= h_i v_i ; h_{i+1} = (w, v_{i+1}); last: ||w||^2
                    for (int i = 1; i <= j + 1; i++) {
                        const bool last = (i == j + 1);
                        k_mgs_step<<<gb, 256, 0, s>>>(n, Hj + (i - 1), C.V.p + (size_t)(i - 1) * C.ldv,
                                                     last ? C.w.p : C.V.p + (size_t)i * C.ldv, C.w.p, last, part, cnt,
                                                     last ? &ks->normW2 : Hj + i);
                        LSG_CHECK_LAUNCH();
                        bytes += (last ? 3 : 4) * w8 * n;
                    }
                }
                launch_givens(C, j);
                LSG_CUDA(cudaStreamSynchronize(s));
                const int flag = *(volatile int*)C.hflag;
                if (flag == 2) {
                    jlast = j;
                    finished = true;
                    break;
                }
            }
            // x += Z y   (solUpdate)
            k_backsub<<<1, 32, 0, s>>>(ks, jlast, 65, C.coefs.p);
            LSG_CHECK_LAUNCH();
            if (C.mg.fp32 && C.opt.precond == LSG_PC_MG)
                k_multi_axpy<float><<<grid_for(n, 256), 256, 0, s>>>(n, C.ldv, jlast + 1, C.coefs.p, C.Z32.p, x);
            else
                k_multi_axpy<double><<<grid_for(n, 256), 256, 0, s>>>(n, C.ldv, jlast + 1, C.coefs.p, C.Z.p, x);
            LSG_CHECK_LAUNCH();
            bytes += (jlast + 3) * w8 * n;
            const bool refine = (C.opt.mg_precision == LSG_FP32 && C.opt.precond == LSG_PC_MG);
            if (!finished || refine) {
                // w = b - A x: the next cycle's first direction
                // (fgmres_interface.h:136-138)
                krylov7<double, 1>(C, x, b, C.w.p, C.scal.p + 16);
                bytes += (3 * w8 + 4) * n;
                KrylovScalars hs;
                double tr2 = 0;
                LSG_CUDA(cudaMemcpyAsync(&hs, ks, sizeof(hs), cudaMemcpyDeviceToHost, s));
                LSG_CUDA(cudaMemcpyAsync(&tr2, C.scal.p + 16, sizeof(double), cudaMemcpyDeviceToHost, s));
                LSG_CUDA(cudaStreamSynchronize(s));
                // FP64 reference semantics restart with the implicit norm |gamma|;
                // with the FP32 preconditioner the restart is an iterative
                // refinement step from the true FP64 residual, and the solve only
                // ends when that true residual meets eps.
                double g = refine ? std::sqrt(tr2) : std::fabs(hs.norm_r);
                if (finished) {
                    if (!(g > C.opt.eps) || !(hs.it < C.opt.max_it) || hs.breakdown) {
                        hs.norm_r = g;
                        LSG_CUDA(cudaMemcpyAsync(ks, &hs, sizeof(hs), cudaMemcpyHostToDevice, s));
                        break;
                    }
                    finished = false;
                    hs.it++;
                }
                hs.norm_r = g;
                hs.invNormW = 1.0 / g;
                hs.done = 0;
                LSG_CUDA(cudaMemcpyAsync(ks, &hs, sizeof(hs), cudaMemcpyHostToDevice, s));
            }
        }
        KrylovScalars hs;
        LSG_CUDA(cudaMemcpyAsync(&hs, ks, sizeof(hs), cudaMemcpyDeviceToHost, s));
        LSG_CUDA(cudaStreamSynchronize(s));
        it = hs.it;
        norm_r = hs.norm_r;
        if (hs.breakdown) status = LSG_BREAKDOWN;
        else if (!(norm_r <= C.opt.eps)) status = LSG_NOT_CONVERGED;
    }
    ilu_check(C);
    if (st) {
        st->iterations = it;
        st->norm_r = norm_r;
        st->status = status;
    }
    C.bytes += bytes;
    return status;
}

}  // namespace lsg

namespace lsg {

// ---------------------------------------------------------------------------
// adjoint pieces: transposed stencil, operator-coefficient gradient
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool nbr7(int s, int x, int y, int z, int N, int M, int K, long long& off, long long NM)
{
    switch (s) {
    case 0: off = -NM; return z > 0;
    case 1: off = -N; return y > 0;
    case 2: off = -1; return x > 0;
    case 3: off = 0; return true;
    case 4: off = 1; return x < N - 1;
    case 5: off = N; return y < M - 1;
    default: off = NM; return z < K - 1;
    }
}

// AT[s][i] = A[6-s][i + off_s]: row i of A^T holds column i of A (the
// neighbour's coefficient pointing back, b<->t, s<->n, w<->e).
__global__ void k_transpose7(int N, int M, int K, const double* __restrict__ A, double* __restrict__ AT)
{
    const long long n = (long long)N * M * K;
    const long long NM = (long long)N * M;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        cell_xyz(i, N, (int)NM, x, y, z);
        for (int sl = 0; sl < 7; sl++) {
            long long off;
            const bool ok = nbr7(sl, x, y, z, N, M, K, off, NM);
            AT[(size_t)sl * n + i] = ok ? A[(size_t)(6 - sl) * n + i + off] : 0.0;
        }
    }
}

// grad[s][i] = -lambda_i x_{i+off_s}: dJ/dA for J(x(A)) with A^T lambda = dJ/dx
__global__ void k_operator_grad7(int N, int M, int K, const double* __restrict__ lam, const double* __restrict__ x,
                                 double* __restrict__ grad)
{
    const long long n = (long long)N * M * K;
    const long long NM = (long long)N * M;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int xx, y, z;
        cell_xyz(i, N, (int)NM, xx, y, z);
        for (int sl = 0; sl < 7; sl++) {
            long long off;
            const bool ok = nbr7(sl, xx, y, z, N, M, K, off, NM);
            grad[(size_t)sl * n + i] = ok ? -lam[i] * x[i + off] : 0.0;
        }
    }
}

// ---------------------------------------------------------------------------
// ILU(0): pivots by hyperplane sweeps, level-scheduled solves in a CUDA graph
// ---------------------------------------------------------------------------

static void ilu_setup(Context& C)
{
    const Dims& d = C.d;
    LSG_REQUIRE(d.N >= 3 && d.M >= 3 && d.K >= 3, LSG_ERR_ARG, "ILU(0) needs N, M, K >= 3");
    const long long n = C.n;
    ilu_graph_release(C);              // factors and work buffers may move
    C.iluU.alloc(n);
    C.iluL.alloc(3 * n);
    const int planes = d.N + d.M + d.K - 2;
    const int blocks = grid_for((long long)d.N * d.M, 256);
    for (int lv = 0; lv < planes; lv++) {
        k_ilu_pivots<<<blocks, 256, 0, C.s>>>(lv, d.N, d.M, d.K, C.A7.p, C.iluU.p);
    }
    LSG_CHECK_LAUNCH();
    k_ilu_lower<<<grid_for(n, 256), 256, 0, C.s>>>(d.N, d.M, d.K, C.A7.p, C.iluU.p, C.iluL.p);
    LSG_CHECK_LAUNCH();
    // the factors in hyperplane order for the one-launch sweep (grids of fewer
    // than 2^31 cells): plane offsets and row offsets on the host, the rest
    // on the device
    C.ilu_blocks = 0;
    C.ilu_planes = 0;
    if (n < (1LL << 31) && C.s) {
        const int P = planes, N = d.N, M = d.M, K = d.K;
        std::vector<int> start(P + 1, 0), rowstart((size_t)P * K, 0);
        int maxplane = 0;
        for (int l = 0; l < P; l++) {
            long long acc = 0;
            for (int z = 0; z < K; z++) {
                rowstart[(size_t)l * K + z] = (int)acc;
                const int lz = l - z;
                if (lz < 0) continue;
                const int ylo = std::max(0, lz - (N - 1)), yhi = std::min(M - 1, lz);
                if (yhi >= ylo) acc += yhi - ylo + 1;
            }
            start[l + 1] = start[l] + (int)acc;
            maxplane = std::max(maxplane, (int)acc);
        }
        LSG_REQUIRE(start[P] == n, LSG_ERR_STATE, "hyperplane count mismatch");
        C.ilu_planes = P;
        C.ilu_maxplane = maxplane;
        C.ilu_start.alloc(P + 1);
        C.ilu_rowstart.alloc((size_t)P * K);
        C.ilu_perm.alloc(n);
        C.ilu_nbr.alloc(6 * (size_t)n);
        C.ilu_fac.alloc(7 * (size_t)n);
        C.ilu_yp.alloc(n);
        C.ilu_xp.alloc(n);
        LSG_CUDA(cudaMemcpyAsync(C.ilu_start.p, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice,
                                 C.s));
        LSG_CUDA(cudaMemcpyAsync(C.ilu_rowstart.p, rowstart.data(), rowstart.size() * sizeof(int),
                                 cudaMemcpyHostToDevice, C.s));
        k_ilu_perm_build<<<grid_for(n, 256), 256, 0, C.s>>>(N, M, K, C.ilu_start.p, C.ilu_rowstart.p, C.iluL.p,
                                                            C.A7.p, C.iluU.p, C.ilu_perm.p, C.ilu_fac.p,
                                                            C.ilu_nbr.p);
        LSG_CHECK_LAUNCH();
    }
    LSG_CUDA(cudaStreamSynchronize(C.s));
    C.have_ilu = true;
}

// x = U^{-1} L^{-1} b ; uses C.t4 for the intermediate
static void ilu_sweeps(Context& C, const double* b, double* x)
{
    const Dims& d = C.d;
    const int planes = d.N + d.M + d.K - 2;
    const int blocks = grid_for((long long)d.N * d.M, 256);
    double* y = C.t4.p;
    for (int lv = 0; lv < planes; lv++)
        k_ilu_fwd<<<blocks, 256, 0, C.s>>>(lv, d.N, d.M, d.K, C.iluL.p, b, y);
    for (int lv = planes - 1; lv >= 0; lv--)
        k_ilu_bwd<<<blocks, 256, 0, C.s>>>(lv, d.N, d.M, d.K, C.A7.p, C.iluU.p, y, x);
}

static void ilu_graph_release(Context& C)
{
    if (C.ilu_exec) cudaGraphExecDestroy(C.ilu_exec);
    C.ilu_exec = nullptr;
}

// Both sweeps of one ILU(0) application as one cooperative launch
// (k_ilu_sweep_perm over the hyperplane-ordered factors: a grid barrier
// between hyperplanes instead of a kernel boundary, one launch instead of
// 2 (N + M + K - 2)).  The grid covers the largest plane with at most a third
// of the CTAs that fit on the GPU at once, so the three momentum equations'
// solves still run side by side.  false = not available (the caller replays
// the per-plane graph).
static bool ilu_coop(Context& C, const double* b, double* x, int withhold = -1)
{
    if (C.ilu_blocks == 0) {
        int dev = 0, sms = 0, coop = 0, per_sm[3] = {0, 0, 0};
        LSG_CUDA(cudaGetDevice(&dev));
        LSG_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
        LSG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        LSG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[0], k_ilu_sweep_perm<1>, 256, 0));
        LSG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[1], k_ilu_sweep_perm<2>, 256, 0));
        LSG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[2], k_ilu_sweep_perm<4>, 256, 0));
        // the fewest positions per thread (1, 2 or 4) for which the grid, as
        // wide as the largest plane, fits a third of the CTAs the GPU holds
        const long long cols = C.ilu_maxplane;
        C.ilu_cmax = 0;
        for (int q = 0; q < 3 && !C.ilu_cmax; q++) {
            const int c = 1 << q;
            if ((cols + 256LL * c - 1) / (256LL * c) <= (long long)sms * per_sm[q] / 3) C.ilu_cmax = c;
        }
        const long long need = C.ilu_cmax ? (cols + 256LL * C.ilu_cmax - 1) / (256LL * C.ilu_cmax) : 0;
        C.ilu_blocks = (coop && C.ilu_cmax && C.ilu_planes > 0) ? (int)std::max(1LL, need) : -1;
        if (C.ilu_blocks > 0) {
            C.ilu_bar.alloc(1);
            C.ilu_err.alloc(1);
            LSG_CUDA(cudaMemsetAsync(C.ilu_err.p, 0, sizeof(int), C.s));
        }
    }
    if (C.ilu_blocks < 0) return false;
    LSG_CUDA(cudaMemsetAsync(C.ilu_bar.p, 0, sizeof(unsigned int), C.s));
    int planes = C.ilu_planes;
    long long nn = C.n;
    const int* start = C.ilu_start.p;
    const int* perm = C.ilu_perm.p;
    const double* fac = C.ilu_fac.p;
    const int* nbr = C.ilu_nbr.p;
    double* yp = C.ilu_yp.p;
    double* xp = C.ilu_xp.p;
    unsigned int* bar = C.ilu_bar.p;
    int* err = C.ilu_err.p;
    void* args[] = {&planes, &nn, (void*)&start, (void*)&perm, (void*)&fac, (void*)&nbr, (void*)&b, &yp, &xp, &x,
                    &bar, &err, &withhold};
    const void* fn = C.ilu_cmax == 1   ? (const void*)k_ilu_sweep_perm<1>
                     : C.ilu_cmax == 2 ? (const void*)k_ilu_sweep_perm<2>
                                       : (const void*)k_ilu_sweep_perm<4>;
    LSG_CUDA(cudaLaunchCooperativeKernel(fn, dim3(C.ilu_blocks), dim3(256), args, 0, C.s));
    LSG_CHECK_LAUNCH();
    return true;
}

// Raises the failure of a cooperative ILU sweep whose barrier gave up.
static void ilu_check(Context& C)
{
    if (C.opt.precond != LSG_PC_ILU0 || C.ilu_blocks <= 0) return;
    int e = 0;
    LSG_CUDA(cudaMemcpyAsync(&e, C.ilu_err.p, sizeof(int), cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    if (e) {
        LSG_CUDA(cudaMemsetAsync(C.ilu_err.p, 0, sizeof(int), C.s));
        throw Error{LSG_ERR_CUDA, "an ILU sweep's grid barrier gave up waiting"};
    }
}

// The 2 (N + M + K - 2) hyperplane launches of one application are replayed
// as one CUDA graph: b is copied into a fixed input buffer, the graph runs,
// the result is copied out (two device copies of n values against hundreds
// of launch submissions).  A context on the legacy default stream launches
// the sweeps directly.
static void ilu_apply(Context& C, const double* b, double* x)
{
    if (!C.s) {
        ilu_sweeps(C, b, x);
        LSG_CHECK_LAUNCH();
        return;
    }
    if (ilu_coop(C, b, x)) return;
    const long long n = C.n;
    if (!C.ilu_exec) {
        C.ilu_in.alloc(n);
        C.ilu_out.alloc(n);
        cudaGraph_t graph = nullptr;
        LSG_CUDA(cudaStreamBeginCapture(C.s, cudaStreamCaptureModeThreadLocal));
        ilu_sweeps(C, C.ilu_in.p, C.ilu_out.p);
        const cudaError_t launch_err = cudaGetLastError();
        const cudaError_t cap_err = cudaStreamEndCapture(C.s, &graph);
        LSG_CUDA(launch_err);
        LSG_CUDA(cap_err);
        size_t nodes = 0;
        cudaGraphGetNodes(graph, nullptr, &nodes);
        C.ilu_nodes = (long long)nodes;
        const cudaError_t inst_err = cudaGraphInstantiate(&C.ilu_exec, graph, 0);
        cudaGraphDestroy(graph);
        if (inst_err != cudaSuccess) C.ilu_exec = nullptr;
        LSG_CUDA(inst_err);
    }
    LSG_CUDA(cudaMemcpyAsync(C.ilu_in.p, b, n * sizeof(double), cudaMemcpyDeviceToDevice, C.s));
    LSG_CUDA(cudaGraphLaunch(C.ilu_exec, C.s));
    ::lsg::g_launches += C.ilu_nodes;
    LSG_CUDA(cudaMemcpyAsync(x, C.ilu_out.p, n * sizeof(double), cudaMemcpyDeviceToDevice, C.s));
}

// ---------------------------------------------------------------------------
// BiCGStab (BiCGStabInterface::solve, bicgstab_interface.h:76-111)
// ---------------------------------------------------------------------------
static int bicgstab(Context& C, double* x, const double* b, lsg_stats* st)
{
    cudaStream_t s = C.s;
    const long long n = C.n;
    const Dims& d = C.d;
    const int gb = grid_for(n, 256, Reducer::kMaxBlocks);
    double* part = C.red.partial.p;
    unsigned int* cnt = C.red.counter.p;
    double* sc = C.scal.p + 24;   // 8 scalars
    double* r = C.w.p;
    double* rr = C.V.p;
    double* p = C.V.p + C.ldv;
    double* y = C.Z.p;
    double* z = C.Z.p + C.ldv;
    double* nu = C.t1.p;
    double* sv = C.t2.p;
    double* t = C.t3.p;
    double bytes = 0;
    int it = 1;
    krylov7<double, 1>(C, x, b, r, sc + 5);
    bytes += 80.0 * n;
    double nr2 = 0;
    LSG_CUDA(cudaMemcpyAsync(&nr2, sc + 5, 8, cudaMemcpyDeviceToHost, s));
    LSG_CUDA(cudaStreamSynchronize(s));
    double norm_r = std::sqrt(nr2);
    int status = LSG_OK;
    if (!std::isfinite(norm_r)) status = LSG_BREAKDOWN;
    else if (norm_r > C.opt.eps) {
        LSG_CUDA(cudaMemcpyAsync(rr, r, n * 8, cudaMemcpyDeviceToDevice, s));
        LSG_CUDA(cudaMemcpyAsync(p, r, n * 8, cudaMemcpyDeviceToDevice, s));
        do {
            precond_apply(C, p, y);
            k_bicg_nu<<<gb, 256, 0, s>>>(d.N, d.M, d.K, C.cls0.p, C.dict0.p, y, nu, rr, r, part, cnt, sc);
            LSG_CHECK_LAUNCH();
            k_bicg_s<<<grid_for(n, 256), 256, 0, s>>>(n, sc, nu, r, sv);
            LSG_CHECK_LAUNCH();
            precond_apply(C, sv, z);
            k_bicg_t<<<gb, 256, 0, s>>>(d.N, d.M, d.K, C.cls0.p, C.dict0.p, z, t, sv, part, cnt, sc + 2);
            LSG_CHECK_LAUNCH();
            k_bicg_upd<<<gb, 256, 0, s>>>(n, sc, y, z, x, t, r, sv, rr, part, cnt, sc + 4);
            LSG_CHECK_LAUNCH();
            k_bicg_p<<<gb, 256, 0, s>>>(n, sc, p, nu, r, part, cnt, sc + 5);
            LSG_CHECK_LAUNCH();
            LSG_CUDA(cudaMemcpyAsync(&nr2, sc + 5, 8, cudaMemcpyDeviceToHost, s));
            LSG_CUDA(cudaStreamSynchronize(s));
            norm_r = std::sqrt(nr2);
            it++;
            bytes += 8.0 * n * (10 + 4 + 10 + 10 + 5) + (C.opt.precond == LSG_PC_ILU0 ? 2 * 8.0 * n * 12 : 0.0);
            if (!std::isfinite(norm_r)) {
                status = LSG_BREAKDOWN;
                break;
            }
        } while (norm_r > C.opt.eps && it < C.opt.max_it);
        if (status == LSG_OK && !(norm_r <= C.opt.eps)) status = LSG_NOT_CONVERGED;
    }
    ilu_check(C);
    if (st) {
        st->iterations = it;
        st->norm_r = norm_r;
        st->status = status;
    }
    C.bytes += bytes;
    return status;
}

static void krylov_alloc(Context& C)
{
    const long long n = C.n;
    const int m = std::max(2, std::min(C.opt.restart, 64));
    C.restart = m;
    // vectors n*8 bytes apart alias in the memory system when n is a power of
    // two; an odd multiple of 256 bytes of padding spreads them
    C.ldv = ((n + 31) / 32) * 32 + 96;
    const long long ldv = C.ldv;
    C.V.alloc((size_t)m * ldv);
    if (C.opt.mg_precision == LSG_FP32 && C.opt.precond == LSG_PC_MG && C.opt.method == LSG_METHOD_FGMRES) {
        C.Z.alloc(2 * ldv);        // BiCGStab-sized scratch only
        C.Z32.alloc((size_t)m * ldv);
    } else {
        C.Z.alloc((size_t)std::max(m, 2) * ldv);
        C.Z32.release();
    }
    C.w.alloc(n);
    C.t1.alloc(n);
    C.t2.alloc(n);
    C.t3.alloc(n);
    C.t4.alloc(n);
    C.xd.alloc(n);
    C.bd.alloc(n);
    C.coefs.alloc(64);
    if (C.opt.gram_schmidt == LSG_GS_LOWSYNC) {
        C.gs_partial.alloc((size_t)148 * 32 * 2 * kGsMaxVec);
        C.gs_sg.alloc(2 * kGsMaxVec);
        C.gs_L.alloc((size_t)kGsMaxVec * kGsMaxVec);
    }
}

static double true_residual(Context& C, const double* x, const double* b)
{
    krylov7<double, 1>(C, x, b, C.t1.p, C.scal.p + 40);
    double r2 = 0;
    LSG_CUDA(cudaMemcpyAsync(&r2, C.scal.p + 40, 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return std::sqrt(r2);
}

static int solve_device(Context& C, const double* b, double* x, lsg_stats* st)
{
    LSG_REQUIRE(C.have_setup, LSG_ERR_STATE, "lsg_setup must be called before solving");
    C.bytes = 0;
    C.vcycles = 0;
    const long long l0 = g_launches;
    LSG_CUDA(cudaEventRecord(C.ev0, C.s));
    int rc;
    if (C.opt.method == LSG_METHOD_BICGSTAB) rc = bicgstab(C, x, b, st);
    else rc = fgmres(C, x, b, st);
    LSG_CUDA(cudaEventRecord(C.ev1, C.s));
    LSG_CUDA(cudaEventSynchronize(C.ev1));
    float ms = 0;
    LSG_CUDA(cudaEventElapsedTime(&ms, C.ev0, C.ev1));
    if (st) {
        st->ms = ms;
        st->bytes = C.bytes;
        st->vcycles = C.vcycles;
        st->kernel_launches = g_launches - l0;
        st->true_residual = true_residual(C, x, b);
    }
    return rc;
}

static void context_init(Context& C, int device, cudaStream_t stream)
{
    C.device = device;
    LSG_CUDA(cudaSetDevice(device));
    if (stream) {
        C.s = stream;
        C.own_stream = false;
    } else {
        LSG_CUDA(cudaStreamCreateWithFlags(&C.s, cudaStreamNonBlocking));
        C.own_stream = true;
    }
    LSG_CUDA(cudaEventCreate(&C.ev0));
    LSG_CUDA(cudaEventCreate(&C.ev1));
    {
        cudaMemPoolProps props;
        std::memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        LSG_CUDA(cudaMemPoolCreate(&C.pool, &props));
        uint64_t keep = UINT64_MAX;          // freed blocks stay with the pool
        LSG_CUDA(cudaMemPoolSetAttribute(C.pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    C.red.init();
    C.scal.alloc(64);
    LSG_CUDA(cudaMemset(C.scal.p, 0, C.scal.bytes()));
    C.ks.alloc(1);
    LSG_CUDA(cudaHostAlloc((void**)&C.hflag, 64, cudaHostAllocMapped));
    C.hnorm = (double*)((char*)C.hflag + 8);
    lsg_default_options(&C.opt);
}

// Frees what the DevBuf members do not own; returns the stream to destroy.
static cudaStream_t context_release(Context& C)
{
    if (C.adj) {
        context_release(*C.adj);
        C.adj.reset();
    }
    if (C.s) cudaStreamSynchronize(C.s);
    ilu_graph_release(C);
    vcycle_graphs_release(C.mg);
    if (C.hflag) cudaFreeHost(C.hflag);
    C.hflag = nullptr;
    if (C.ev0) cudaEventDestroy(C.ev0);
    if (C.ev1) cudaEventDestroy(C.ev1);
    C.ev0 = C.ev1 = nullptr;
    if (C.pool) cudaMemPoolDestroy(C.pool);
    C.pool = nullptr;
    return C.own_stream ? C.s : nullptr;
}

// The transposed operator's solver state, with the forward solver's options.
static Context& adjoint_context(Context& C)
{
    LSG_REQUIRE(C.have_setup, LSG_ERR_STATE, "lsg_setup must be called before the adjoint");
    if (!C.adj) {
        std::unique_ptr<Context> a(new Context);
        context_init(*a, C.device, C.s);
        a->d = C.d;
        a->n = C.n;
        a->A7.alloc(7 * C.n);
        k_transpose7<<<grid_for(C.n, 256), 256, 0, C.s>>>(C.d.N, C.d.M, C.d.K, C.A7.p, a->A7.p);
        LSG_CHECK_LAUNCH();
        a->nclass0 = build_dict(C.s, a->A7.p, 7, C.n, a->cls0, a->dict0);
        a->have_matrix = true;
        C.adj = std::move(a);
    }
    Context& A = *C.adj;
    if (!A.have_setup || std::memcmp(&A.opt, &C.opt, sizeof(lsg_options)) != 0) {
        A.opt = C.opt;
        if (A.opt.precond == LSG_PC_MG) mg_setup(A);
        if (A.opt.precond == LSG_PC_ILU0) ilu_setup(A);
        krylov_alloc(A);
        A.have_setup = true;
    }
    return A;
}

}  // namespace lsg

// ===========================================================================
// C ABI
// ===========================================================================
using namespace lsg;

#define LSG_API_BEGIN \
    try {
#define LSG_API_END(ctxp)                                   \
    }                                                       \
    catch (const lsg::Error& e)                             \
    {                                                       \
        if (ctxp) (ctxp)->c.err = e.msg;                     \
        return e.code;                                      \
    }                                                       \
    catch (const std::exception& e)                         \
    {                                                       \
        if (ctxp) (ctxp)->c.err = e.what();                  \
        return LSG_ERR_ARG;                                 \
    }

extern "C" {

void lsg_default_options(lsg_options* o)
{
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->method = LSG_METHOD_FGMRES;
    o->precond = LSG_PC_MG;
    o->mg_precision = LSG_FP64;
    o->smoother = LSG_SMOOTHER_ADLJ;
    o->n_pre = 0;
    o->n_post = 3;
    o->max_levels = 0;
    o->restart = 30;
    o->max_it = 200;
    o->zline_reference = 1;
    o->eps = 1e-5;
    o->omega = 0.805;
}

const char* lsg_version(void) { return "lsstag_b200 1.0 (sm_100a)"; }

int lsg_create(int device, lsg_ctx** out)
{
    if (!out) return LSG_ERR_ARG;
    *out = nullptr;
    lsg_ctx* h = new (std::nothrow) lsg_ctx;
    if (!h) return LSG_ERR_NOMEM;
    try {
        context_init(h->c, device, nullptr);
    } catch (const lsg::Error& e) {
        fprintf(stderr, "lsg_create: %s\n", e.msg.c_str());
        cudaStream_t s = context_release(h->c);
        delete h;
        if (s) cudaStreamDestroy(s);
        return e.code;
    }
    *out = h;
    return LSG_OK;
}

int lsg_destroy(lsg_ctx* h)
{
    if (!h) return LSG_OK;
    cudaSetDevice(h->c.device);
    cudaStream_t s = context_release(h->c);
    delete h;   // DevBuf destructors free device memory
    if (s) cudaStreamDestroy(s);
    return LSG_OK;
}

const char* lsg_last_error(const lsg_ctx* h) { return h ? h->c.err.c_str() : "null context"; }

// Wall time of an entry point into *out (host clock; the entry points below
// end with a stream synchronisation).
struct WallTimer {
    double& out;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    explicit WallTimer(double& o) : out(o) {}
    ~WallTimer() { out = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count(); }
};

static int set_matrix_impl(lsg_ctx* h, int N, int M, int K, const int* rowptr, const int* col, const double* val,
                           long long nnz, bool host)
{
    Context& C = h->c;
    WallTimer wt(C.matrix_ms);
    LSG_REQUIRE(N >= 1 && M >= 1 && K >= 1, LSG_ERR_ARG, "grid dimensions must be positive");
    LSG_REQUIRE(rowptr && col && val, LSG_ERR_ARG, "null CSR pointer");
    C.geo.have = C.geo.have_stypes = false;    // geometry of an earlier operator no longer applies
    LSG_CUDA(cudaSetDevice(C.device));
    const long long n = (long long)N * M * K;
    LSG_REQUIRE(n < (1LL << 31), LSG_ERR_ARG, "grid too large for 32-bit CSR indices");
    TmpBuf<int> drp(C.s, C.pool), dcol(C.s, C.pool);
    TmpBuf<double> dval(C.s, C.pool);
    const int* prp = rowptr;
    const int* pcol = col;
    const double* pval = val;
    if (host) {
        nnz = rowptr[n];
        LSG_REQUIRE(nnz >= 0, LSG_ERR_ARG, "negative nnz");
        drp.alloc(n + 1);
        dcol.alloc(nnz > 0 ? nnz : 1);
        dval.alloc(nnz > 0 ? nnz : 1);
        LSG_CUDA(cudaMemcpyAsync(drp.p, rowptr, (n + 1) * sizeof(int), cudaMemcpyHostToDevice, C.s));
        LSG_CUDA(cudaMemcpyAsync(dcol.p, col, nnz * sizeof(int), cudaMemcpyHostToDevice, C.s));
        LSG_CUDA(cudaMemcpyAsync(dval.p, val, nnz * sizeof(double), cudaMemcpyHostToDevice, C.s));
        prp = drp.p;
        pcol = dcol.p;
        pval = dval.p;
    }
    C.d.N = N;
    C.d.M = M;
    C.d.K = K;
    C.n = n;
    C.A7.alloc(7 * n);
    LSG_CUDA(cudaMemsetAsync(C.A7.p, 0, C.A7.bytes(), C.s));
    int* err = (int*)(C.scal.p + 8);
    LSG_CUDA(cudaMemsetAsync(err, 0, sizeof(int), C.s));
    k_csr_to_stencil7<<<grid_for(n, 256), 256, 0, C.s>>>(N, M, K, prp, pcol, pval, C.A7.p, err);
    LSG_CHECK_LAUNCH();
    int e = 0;
    LSG_CUDA(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    if (e != 0) {
        C.have_matrix = false;
        throw Error{LSG_ERR_PATTERN, "row " + std::to_string(e - 1) +
                                         " holds an entry that is not the cell or one of its six face neighbours"};
    }
    C.nclass0 = build_dict(C.s, C.A7.p, 7, n, C.cls0, C.dict0);
    if (C.adj) {
        context_release(*C.adj);
        C.adj.reset();
    }
    C.have_matrix = true;
    C.have_setup = false;
    return LSG_OK;
}

int lsg_set_matrix_csr(lsg_ctx* h, int N, int M, int K, const int* rowptr, const int* col, const double* val)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    return set_matrix_impl(h, N, M, K, rowptr, col, val, -1, true);
    LSG_API_END(h)
}

int lsg_set_matrix_csr_device(lsg_ctx* h, int N, int M, int K, const int* rowptr, const int* col,
                              const double* val, long long nnz)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    return set_matrix_impl(h, N, M, K, rowptr, col, val, nnz, false);
    LSG_API_END(h)
}

int lsg_set_matrix_stencil7(lsg_ctx* h, int N, int M, int K, const double* planes)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    WallTimer wt(C.matrix_ms);
    LSG_REQUIRE(N >= 1 && M >= 1 && K >= 1, LSG_ERR_ARG, "grid dimensions must be positive");
    LSG_REQUIRE(planes, LSG_ERR_ARG, "null planes");
    C.geo.have = C.geo.have_stypes = false;    // geometry of an earlier operator no longer applies
    LSG_CUDA(cudaSetDevice(C.device));
    const long long n = (long long)N * M * K;
    LSG_REQUIRE(n < (1LL << 31), LSG_ERR_ARG, "grid too large");
    C.d.N = N;
    C.d.M = M;
    C.d.K = K;
    C.n = n;
    C.A7.alloc(7 * n);
    LSG_CUDA(cudaMemcpyAsync(C.A7.p, planes, 7 * n * sizeof(double), cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    C.nclass0 = build_dict(C.s, C.A7.p, 7, n, C.cls0, C.dict0);
    if (C.adj) {
        context_release(*C.adj);
        C.adj.reset();
    }
    C.have_matrix = true;
    C.have_setup = false;
    return LSG_OK;
    LSG_API_END(h)
}

// Every face a row reads must exist: a cell whose type keeps a face (fluid,
// cut or border family without that face) may not lie on the matching domain
// border.  Checked on the host before the geometry reaches any kernel.
static void check_cell_types(int N, int M, int K, const int* t)
{
    const long long NM = (long long)N * M;
    for (int z = 0; z < K; z++)
        for (int y = 0; y < M; y++)
            for (int x = 0; x < N; x++) {
                const long long i = x + N * (long long)y + NM * z;
                if (t[i] == 0) continue;
                const int miss = absent_faces(t[i]);
                const bool ok = ((miss & 1) || z > 0) && ((miss & 2) || y > 0) && ((miss & 4) || x > 0) &&
                                ((miss & 8) || x < N - 1) && ((miss & 16) || y < M - 1) && ((miss & 32) || z < K - 1);
                if (!ok) {
                    char buf[160];
                    std::snprintf(buf, sizeof buf, "cell type %d at (%d, %d, %d) keeps a face outside the grid", t[i], x,
                                  y, z);
                    throw Error{LSG_ERR_ARG, buf};
                }
            }
}

// The Laplace operator from the context's geometry (C.geo type, theta,
// delta, inverse staggered volumes), the row dictionary, and the context's
// operator state.
static void assemble_laplace(Context& C, int N, int M, int K, long long pin0, long long pin1)
{
    Context::Geometry& g = C.geo;
    const long long n = (long long)N * M * K;
    g.pin0 = pin0;
    g.pin1 = pin1;
    C.d.N = N;
    C.d.M = M;
    C.d.K = K;
    C.n = n;
    C.A7.alloc(7 * n);
    k_laplace_from_geometry<<<grid_for(n, 256), 256, 0, C.s>>>(N, M, K, g.type.p, g.theta.p, g.delta.p, g.inv[0].p,
                                                              g.inv[1].p, g.inv[2].p, pin0, pin1, C.A7.p);
    LSG_CHECK_LAUNCH();
    LSG_CUDA(cudaStreamSynchronize(C.s));
    C.nclass0 = build_dict(C.s, C.A7.p, 7, n, C.cls0, C.dict0);
    if (C.adj) {
        context_release(*C.adj);
        C.adj.reset();
    }
    g.have = true;
    C.have_matrix = true;
    C.have_setup = false;
}

int lsg_set_matrix_geometry(lsg_ctx* h, int N, int M, int K, const int* celltype, const double* theta,
                            const double* delta, const double* inv_mx, const double* inv_my, const double* inv_mz,
                            long long pin0, long long pin1)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    WallTimer wt(C.matrix_ms);
    LSG_REQUIRE(N >= 2 && M >= 2 && K >= 2, LSG_ERR_ARG, "grid dimensions must be >= 2");
    LSG_REQUIRE(celltype && theta && delta && inv_mx && inv_my && inv_mz, LSG_ERR_ARG, "null geometry array");
    const long long n = (long long)N * M * K;
    LSG_REQUIRE(n < (1LL << 31), LSG_ERR_ARG, "grid too large");
    LSG_REQUIRE(pin0 >= -1 && pin0 < n && pin1 >= -1 && pin1 < n, LSG_ERR_ARG, "pinned row outside the grid");
    check_cell_types(N, M, K, celltype);
    LSG_CUDA(cudaSetDevice(C.device));
    const long long nx = (long long)(N - 1) * M * K, ny = (long long)N * (M - 1) * K, nz = (long long)N * M * (K - 1);
    Context::Geometry& g = C.geo;
    g.have = false;
    g.have_stypes = false;
    g.type.alloc(n);
    g.theta.alloc(3 * n);
    g.delta.alloc(3 * n);
    g.inv[0].alloc(nx);
    g.inv[1].alloc(ny);
    g.inv[2].alloc(nz);
    LSG_CUDA(cudaMemcpyAsync(g.type.p, celltype, n * sizeof(int), cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(g.theta.p, theta, 3 * n * 8, cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(g.delta.p, delta, 3 * n * 8, cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(g.inv[0].p, inv_mx, nx * 8, cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(g.inv[1].p, inv_my, ny * 8, cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(g.inv[2].p, inv_mz, nz * 8, cudaMemcpyHostToDevice, C.s));
    assemble_laplace(C, N, M, K, pin0, pin1);
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_set_matrix_helmholtz(lsg_ctx* h, int dir, int N, int M, int K, const int* stype, const double* theta,
                             const double* alpha, const double* delta, const double* inv_vof, const double* vof,
                             const double* delta_ib_en, const double* delta_ib_ws, const double* delta_ib_nb,
                             const double* delta_ib_st, const double* inv_delta_ib_ne, const double* inv_delta_ib_tn,
                             double nu, double coef, int is_flow)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    WallTimer wt(C.matrix_ms);
    LSG_REQUIRE(dir >= 0 && dir <= 2, LSG_ERR_ARG, "dir must be 0 (x), 1 (y) or 2 (z)");
    LSG_REQUIRE(N >= 3 && M >= 3 && K >= 3, LSG_ERR_ARG, "grid must be at least 3 cells in every direction");
    LSG_REQUIRE(stype && theta && alpha && delta && inv_vof && vof && delta_ib_en && delta_ib_ws && delta_ib_nb &&
                    delta_ib_st && inv_delta_ib_ne && inv_delta_ib_tn,
                LSG_ERR_ARG, "null geometry array");
    const long long n = (long long)N * M * K;
    LSG_REQUIRE(n < (1LL << 31), LSG_ERR_ARG, "grid too large");
    const int Ns = N - (dir == 0), Ms = M - (dir == 1), Ks = K - (dir == 2);
    const long long ns = (long long)Ns * Ms * Ks;
    // a face kept by a staggered cell's type must lie inside the staggered grid
    check_cell_types(Ns, Ms, Ks, stype);
    C.geo.have = C.geo.have_stypes = false;    // geometry of an earlier operator no longer applies
    LSG_CUDA(cudaSetDevice(C.device));
    TmpBuf<int> dt(C.s, C.pool);
    TmpBuf<double> dth(C.s, C.pool), dal(C.s, C.pool), dde(C.s, C.pool), dinv(C.s, C.pool), dvof(C.s, C.pool), den(C.s, C.pool), dws(C.s, C.pool), dnb(C.s, C.pool), dst(C.s, C.pool), dne(C.s, C.pool), dtn(C.s, C.pool);
    dt.alloc(ns);
    LSG_CUDA(cudaMemcpyAsync(dt.p, stype, ns * sizeof(int), cudaMemcpyHostToDevice, C.s));
    const double* src3[9] = {theta, alpha, delta, delta_ib_en, delta_ib_ws, delta_ib_nb, delta_ib_st,
                             inv_delta_ib_ne, inv_delta_ib_tn};
    TmpBuf<double>* dst3[9] = {&dth, &dal, &dde, &den, &dws, &dnb, &dst, &dne, &dtn};
    for (int a = 0; a < 9; a++) {
        dst3[a]->alloc(3 * n);
        LSG_CUDA(cudaMemcpyAsync(dst3[a]->p, src3[a], 3 * n * 8, cudaMemcpyHostToDevice, C.s));
    }
    dinv.alloc(n);
    dvof.alloc(ns);
    LSG_CUDA(cudaMemcpyAsync(dinv.p, inv_vof, n * 8, cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(dvof.p, vof, ns * 8, cudaMemcpyHostToDevice, C.s));
    C.d.N = Ns;
    C.d.M = Ms;
    C.d.K = Ks;
    C.n = ns;
    C.A7.alloc(7 * ns);
    HelmGeom g;
    g.N = N;
    g.M = M;
    g.K = K;
    g.d = dir;
    g.stype = dt.p;
    g.theta = dth.p;
    g.alpha = dal.p;
    g.delta = dde.p;
    g.inv_vof = dinv.p;
    g.vof = dvof.p;
    g.dib_en = den.p;
    g.dib_ws = dws.p;
    g.dib_nb = dnb.p;
    g.dib_st = dst.p;
    g.inv_dib_ne = dne.p;
    g.inv_dib_tn = dtn.p;
    g.nu = nu;
    g.coef = coef;
    g.is_flow = is_flow ? 1 : 0;
    g.planes = C.A7.p;
    k_helmholtz_from_geometry<<<grid_for(ns, 256), 256, 0, C.s>>>(g);
    LSG_CHECK_LAUNCH();
    LSG_CUDA(cudaStreamSynchronize(C.s));
    C.nclass0 = build_dict(C.s, C.A7.p, 7, ns, C.cls0, C.dict0);
    if (C.adj) {
        context_release(*C.adj);
        C.adj.reset();
    }
    C.have_matrix = true;
    C.have_setup = false;
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_helmholtz_flux(lsg_ctx* h, int dir, int N, int M, int K, const int* stype, const double* delta,
                       const double* u_w, const double* bc, double nu, int ib, const int* side_type,
                       const double* theta, const double* alpha, const double* inv_vof, const double* delta_ib_en,
                       const double* delta_ib_ws, const double* delta_ib_nb, const double* delta_ib_st,
                       const double* inv_delta_ib_ne, const double* inv_delta_ib_tn, const double* vib,
                       const double* vib_yx, const double* vib_zy, double* flux)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(dir >= 0 && dir <= 2, LSG_ERR_ARG, "dir must be 0 (x), 1 (y) or 2 (z)");
    LSG_REQUIRE(N >= 3 && M >= 3 && K >= 3, LSG_ERR_ARG, "grid must be at least 3 cells in every direction");
    LSG_REQUIRE(stype && delta && u_w && bc && flux, LSG_ERR_ARG, "null argument");
    LSG_REQUIRE(!ib || (side_type && theta && alpha && inv_vof && delta_ib_en && delta_ib_ws && delta_ib_nb &&
                        delta_ib_st && inv_delta_ib_ne && inv_delta_ib_tn && vib && vib_yx && vib_zy),
                LSG_ERR_ARG, "null immersed-boundary argument");
    const long long n = (long long)N * M * K;
    LSG_REQUIRE(n < (1LL << 31), LSG_ERR_ARG, "grid too large");
    const int Ns = N - (dir == 0), Ms = M - (dir == 1), Ks = K - (dir == 2);
    const long long ns = (long long)Ns * Ms * Ks;
    LSG_CUDA(cudaSetDevice(C.device));
    TmpBuf<int> dt(C.s, C.pool), dsd(C.s, C.pool);
    TmpBuf<double> dde(C.s, C.pool), duw(C.s, C.pool), dout(C.s, C.pool), dth(C.s, C.pool), dal(C.s, C.pool), dinv(C.s, C.pool), den(C.s, C.pool), dws(C.s, C.pool), dnb(C.s, C.pool), dst(C.s, C.pool), dne(C.s, C.pool), dtn(C.s, C.pool), dv(C.s, C.pool), dyx(C.s, C.pool), dzy(C.s, C.pool);
    dt.alloc(ns);
    dde.alloc(3 * n);
    duw.alloc((size_t)M * K);
    dout.alloc(ns);
    LSG_CUDA(cudaMemcpyAsync(dt.p, stype, ns * sizeof(int), cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(dde.p, delta, 3 * n * 8, cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(duw.p, u_w, (size_t)M * K * 8, cudaMemcpyHostToDevice, C.s));
    HelmFluxArgs a;
    memset(&a, 0, sizeof(a));
    a.g.N = N;
    a.g.M = M;
    a.g.K = K;
    a.g.d = dir;
    a.g.stype = dt.p;
    a.g.delta = dde.p;
    a.g.nu = nu;
    if (ib) {
        dsd.alloc(3 * n);
        LSG_CUDA(cudaMemcpyAsync(dsd.p, side_type, 3 * n * sizeof(int), cudaMemcpyHostToDevice, C.s));
        const double* src3[11] = {theta, alpha, delta_ib_en, delta_ib_ws, delta_ib_nb, delta_ib_st,
                                  inv_delta_ib_ne, inv_delta_ib_tn, vib, vib_yx, vib_zy};
        TmpBuf<double>* dst3[11] = {&dth, &dal, &den, &dws, &dnb, &dst, &dne, &dtn, &dv, &dyx, &dzy};
        for (int q = 0; q < 11; q++) {
            dst3[q]->alloc(3 * n);
            LSG_CUDA(cudaMemcpyAsync(dst3[q]->p, src3[q], 3 * n * 8, cudaMemcpyHostToDevice, C.s));
        }
        dinv.alloc(n);
        LSG_CUDA(cudaMemcpyAsync(dinv.p, inv_vof, n * 8, cudaMemcpyHostToDevice, C.s));
        a.g.theta = dth.p;
        a.g.alpha = dal.p;
        a.g.inv_vof = dinv.p;
        a.g.dib_en = den.p;
        a.g.dib_ws = dws.p;
        a.g.dib_nb = dnb.p;
        a.g.dib_st = dst.p;
        a.g.inv_dib_ne = dne.p;
        a.g.inv_dib_tn = dtn.p;
        a.side_type = dsd.p;
        a.vib = dv.p;
        a.vyx = dyx.p;
        a.vzy = dzy.p;
    }
    a.u_w = duw.p;
    for (int q = 0; q < 18; q++) a.bc[q] = bc[q];
    a.ib = ib ? 1 : 0;
    a.flux = dout.p;
    k_helmholtz_flux<<<grid_for(ns, 256), 256, 0, C.s>>>(a);
    LSG_CHECK_LAUNCH();
    LSG_CUDA(cudaMemcpyAsync(flux, dout.p, ns * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

static void convective_flux_run(Context& C, int dir, int N, int M, int K, const double* theta, const double* delta,
                                const double* ux, const double* uz, const double* u_w, const double* bc, double* flux)
{
    const int Ns = N - (dir == 0), Ms = M - (dir == 1), Ks = K - (dir == 2);
    const long long ns = (long long)Ns * Ms * Ks;
    if (dir != 2) {
        // the reference's x and y convective operators keep a zero source term
        LSG_CUDA(cudaMemsetAsync(flux, 0, ns * 8, C.s));
        return;
    }
    ConvFluxArgs a;
    a.N = N;
    a.M = M;
    a.K = K;
    a.theta = theta;
    a.delta = delta;
    a.ux = ux;
    a.uz = uz;
    a.u_w = u_w;
    a.W_W = bc[12];
    a.VW_S = bc[14] * bc[8];
    a.VW_N = bc[15] * bc[9];
    a.flux = flux;
    k_convective_flux_z<<<grid_for(ns, 256), 256, 0, C.s>>>(a);
    LSG_CHECK_LAUNCH();
}

int lsg_convective_flux_device(lsg_ctx* h, int dir, int N, int M, int K, const double* theta, const double* delta,
                               const double* ux, const double* uy, const double* uz, const double* u_w,
                               const double* bc, double* flux)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(dir >= 0 && dir <= 2, LSG_ERR_ARG, "dir must be 0 (x), 1 (y) or 2 (z)");
    LSG_REQUIRE(N >= 3 && M >= 3 && K >= 3, LSG_ERR_ARG, "grid must be at least 3 cells in every direction");
    LSG_REQUIRE(flux && bc && (dir != 2 || (theta && delta && ux && uz && u_w)), LSG_ERR_ARG, "null argument");
    (void)uy;
    LSG_CUDA(cudaSetDevice(C.device));
    convective_flux_run(C, dir, N, M, K, theta, delta, ux, uz, u_w, bc, flux);
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_convective_flux(lsg_ctx* h, int dir, int N, int M, int K, const double* theta, const double* delta,
                        const double* ux, const double* uy, const double* uz, const double* u_w, const double* bc,
                        double* flux)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(dir >= 0 && dir <= 2, LSG_ERR_ARG, "dir must be 0 (x), 1 (y) or 2 (z)");
    LSG_REQUIRE(N >= 3 && M >= 3 && K >= 3, LSG_ERR_ARG, "grid must be at least 3 cells in every direction");
    LSG_REQUIRE(flux && bc && (dir != 2 || (theta && delta && ux && uz && u_w)), LSG_ERR_ARG, "null argument");
    (void)uy;
    const long long n = (long long)N * M * K;
    LSG_REQUIRE(n < (1LL << 31), LSG_ERR_ARG, "grid too large");
    const int Ns = N - (dir == 0), Ms = M - (dir == 1), Ks = K - (dir == 2);
    const long long ns = (long long)Ns * Ms * Ks;
    LSG_CUDA(cudaSetDevice(C.device));
    TmpBuf<double> dth(C.s, C.pool), dde(C.s, C.pool), dux(C.s, C.pool), duz(C.s, C.pool), duw(C.s, C.pool), dout(C.s, C.pool);
    dout.alloc(ns);
    if (dir == 2) {
        const long long nx = (long long)(N - 1) * M * K, nz = (long long)N * M * (K - 1);
        dth.alloc(3 * n);
        dde.alloc(3 * n);
        dux.alloc(nx);
        duz.alloc(nz);
        duw.alloc((size_t)M * K);
        LSG_CUDA(cudaMemcpyAsync(dth.p, theta, 3 * n * 8, cudaMemcpyHostToDevice, C.s));
        LSG_CUDA(cudaMemcpyAsync(dde.p, delta, 3 * n * 8, cudaMemcpyHostToDevice, C.s));
        LSG_CUDA(cudaMemcpyAsync(dux.p, ux, nx * 8, cudaMemcpyHostToDevice, C.s));
        LSG_CUDA(cudaMemcpyAsync(duz.p, uz, nz * 8, cudaMemcpyHostToDevice, C.s));
        LSG_CUDA(cudaMemcpyAsync(duw.p, u_w, (size_t)M * K * 8, cudaMemcpyHostToDevice, C.s));
    }
    convective_flux_run(C, dir, N, M, K, dth.p, dde.p, dux.p, duz.p, duw.p, bc, dout.p);
    LSG_CUDA(cudaMemcpyAsync(flux, dout.p, ns * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_set_staggered_types(lsg_ctx* h, const int* xtype, const int* ytype, const int* ztype)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.geo.have, LSG_ERR_STATE, "no geometry set (lsg_set_matrix_geometry)");
    LSG_REQUIRE(xtype && ytype && ztype, LSG_ERR_ARG, "null type array");
    LSG_CUDA(cudaSetDevice(C.device));
    const Dims& d = C.d;
    const long long cnt[3] = {(long long)(d.N - 1) * d.M * d.K, (long long)d.N * (d.M - 1) * d.K,
                              (long long)d.N * d.M * (d.K - 1)};
    const int* src[3] = {xtype, ytype, ztype};
    // as for the base grid: a face kept by a staggered cell's type must lie inside its grid
    for (int k = 0; k < 3; k++) {
        const int Nd = d.N - (k == 0), Md = d.M - (k == 1), Kd = d.K - (k == 2);
        check_cell_types(Nd, Md, Kd, src[k]);
    }
    for (int k = 0; k < 3; k++) {
        C.geo.stype[k].alloc(cnt[k]);
        LSG_CUDA(cudaMemcpyAsync(C.geo.stype[k].p, src[k], cnt[k] * sizeof(int), cudaMemcpyHostToDevice, C.s));
    }
    LSG_CUDA(cudaStreamSynchronize(C.s));
    C.geo.have_stypes = true;
    return LSG_OK;
    LSG_API_END(h)
}

// ---------------------------------------------------------------------------
// mesh build on the device (level set -> ... -> staggered inverse volumes)
// ---------------------------------------------------------------------------
int lsg_mesh_build(lsg_ctx* h, int N, int M, int K, const double* hstep, const int* block, int n_bodies,
                   const double* bodies, const double* phi, double* ms)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(N >= 4 && M >= 4 && K >= 3, LSG_ERR_ARG, "grid must be at least 4 x 4 x 3 cells");
    LSG_REQUIRE(hstep && block, LSG_ERR_ARG, "null cell size or block");
    LSG_REQUIRE(hstep[0] > 0 && hstep[1] > 0 && hstep[2] > 0, LSG_ERR_ARG, "cell sizes must be positive");
    const long long n = (long long)N * M * K;
    LSG_REQUIRE(n < (1LL << 31), LSG_ERR_ARG, "grid too large");
    const mesh::Block b{block[0], block[1], block[2], block[3]};
    // the walks read one corner value back and one ahead along x and y: the
    // block keeps off the box's first and last column and row
    LSG_REQUIRE(b.hs >= 1 && b.hs < b.hf && b.hf <= N - 1 && b.vs >= 1 && b.vs < b.vf && b.vf <= M - 1, LSG_ERR_ARG,
                "level-set block must satisfy 1 <= hs < hf <= N-1 and 1 <= vs < vf <= M-1");
    LSG_REQUIRE(phi || (n_bodies > 0 && bodies), LSG_ERR_ARG, "need a level set (phi) or at least one body");
    if (!phi) {
        for (int q = 0; q < n_bodies; q++) {
            const double* bq = bodies + (size_t)q * mesh::kBodyWords;
            LSG_REQUIRE(bq[0] == 0.0 || bq[0] == 1.0, LSG_ERR_ARG, "body kind must be 0 (sphere) or 1 (ellipsoid)");
            LSG_REQUIRE(bq[0] == 0.0 ? bq[4] > 0 : (bq[5] > 0 && bq[6] > 0 && bq[7] > 0), LSG_ERR_ARG,
                        "body radius / semi-axes must be positive");
        }
    }
    LSG_CUDA(cudaSetDevice(C.device));
    Context::Mesh& m = C.mesh;
    m.have = false;
    m.N = N;
    m.M = M;
    m.K = K;
    const long long ns[3] = {(long long)(N - 1) * M * K, (long long)N * (M - 1) * K, (long long)N * M * (K - 1)};
    m.phi_ls.alloc(n);
    m.phi.alloc(n);
    m.alpha.alloc(3 * n);
    m.theta.alloc(3 * n);
    m.delta.alloc(3 * n);
    m.vof.alloc(n);
    m.inv_vof.alloc(n);
    m.side.alloc(3 * n);
    m.type.alloc(n);
    for (int d = 0; d < 3; d++) {
        m.svof[d].alloc(ns[d]);
        m.sinv[d].alloc(ns[d]);
        m.stype[d].alloc(ns[d]);
    }
    for (int a = 0; a < 5; a++) m.dib[a].alloc(3 * n);
    m.inv_dib_ne.alloc(3 * n);
    m.inv_dib_tn.alloc(3 * n);
    cudaEvent_t e0, e1;
    LSG_CUDA(cudaEventCreate(&e0));
    LSG_CUDA(cudaEventCreate(&e1));
    struct Ev {
        cudaEvent_t a, b;
        ~Ev() { cudaEventDestroy(a); cudaEventDestroy(b); }
    } ev{e0, e1};
    LSG_CUDA(cudaEventRecord(e0, C.s));
    const int gsz = grid_for(n, 256);
    mesh::k_mesh_init<<<gsz, 256, 0, C.s>>>(N, M, K, hstep[0], hstep[1], hstep[2], m.phi_ls.p, m.alpha.p, m.theta.p,
                                      m.delta.p, m.side.p, m.type.p);
    LSG_CHECK_LAUNCH();
    TmpBuf<double> scratch(C.s, C.pool);
    if (phi) {
        scratch.alloc(n);
        LSG_CUDA(cudaMemcpyAsync(scratch.p, phi, n * 8, cudaMemcpyHostToDevice, C.s));
        mesh::k_mesh_phi_block<<<gsz, 256, 0, C.s>>>(N, M, K, b, scratch.p, m.phi_ls.p);
        LSG_CHECK_LAUNCH();
    } else {
        TmpBuf<double> db(C.s, C.pool);
        db.alloc((size_t)n_bodies * mesh::kBodyWords);
        LSG_CUDA(cudaMemcpyAsync(db.p, bodies, (size_t)n_bodies * mesh::kBodyWords * 8, cudaMemcpyHostToDevice, C.s));
        const long long rows = (long long)(b.vf - b.vs) * K;
        mesh::k_mesh_levelset<<<(unsigned)((rows + 127) / 128), 128, 0, C.s>>>(N, M, K, b, hstep[0], hstep[1], hstep[2],
                                                                          n_bodies, db.p, m.phi_ls.p);
        LSG_CHECK_LAUNCH();
        LSG_CUDA(cudaStreamSynchronize(C.s));   // db is released on return of this scope
    }
    // oscillation fix: fixed-point sweeps of the reference's walk until no
    // value moves; each sweep settles at least the next cell of every chain of
    // edits, so the count is bounded by the longest chain (a few cells)
    LSG_CUDA(cudaMemcpyAsync(m.phi.p, m.phi_ls.p, n * 8, cudaMemcpyDeviceToDevice, C.s));
    if (!scratch.p) scratch.alloc(n);
    LSG_CUDA(cudaMemcpyAsync(scratch.p, m.phi_ls.p, n * 8, cudaMemcpyDeviceToDevice, C.s));
    unsigned int* changed = (unsigned int*)(C.scal.p + 8);
    const long long bcells = (long long)(b.hf - b.hs) * (b.vf - b.vs) * K;
    const unsigned bgrid = (unsigned)((bcells + 255) / 256);
    const long long max_sweeps = bcells + 1;
    double* cur = m.phi.p;
    double* nxt = scratch.p;
    m.osc_sweeps = 0;
    for (;;) {
        LSG_REQUIRE(m.osc_sweeps < max_sweeps, LSG_ERR_STATE, "level-set oscillation fix did not settle");
        LSG_CUDA(cudaMemsetAsync(changed, 0, sizeof(unsigned int), C.s));
        mesh::k_mesh_osc<<<bgrid, 256, 0, C.s>>>(N, M, K, b, m.phi_ls.p, cur, nxt, changed);
        LSG_CHECK_LAUNCH();
        unsigned int hc = 0;
        LSG_CUDA(cudaMemcpyAsync(&hc, changed, sizeof(hc), cudaMemcpyDeviceToHost, C.s));
        LSG_CUDA(cudaStreamSynchronize(C.s));
        m.osc_sweeps++;
        std::swap(cur, nxt);
        if (hc == 0) break;
    }
    if (cur != m.phi.p)                                   // keep the settled values in m.phi
        LSG_CUDA(cudaMemcpyAsync(m.phi.p, cur, n * 8, cudaMemcpyDeviceToDevice, C.s));
    mesh::k_mesh_alpha_types<<<bgrid, 256, 0, C.s>>>(N, M, K, b, m.phi.p, m.alpha.p, m.side.p, m.type.p);
    LSG_CHECK_LAUNCH();
    mesh::k_mesh_theta<<<bgrid, 256, 0, C.s>>>(N, M, K, b, m.side.p, m.alpha.p, m.theta.p);
    LSG_CHECK_LAUNCH();
    mesh::k_mesh_volume<<<gsz, 256, 0, C.s>>>(N, M, K, m.type.p, m.delta.p, m.theta.p, m.alpha.p, m.vof.p, m.inv_vof.p);
    LSG_CHECK_LAUNCH();
    mesh::k_mesh_staggered<<<gsz, 256, 0, C.s>>>(N, M, K, m.type.p, m.theta.p, m.vof.p, m.stype[0].p, m.stype[1].p,
                                           m.stype[2].p, m.svof[0].p, m.svof[1].p, m.svof[2].p, m.sinv[0].p,
                                           m.sinv[1].p, m.sinv[2].p);
    LSG_CHECK_LAUNCH();
    mesh::k_mesh_ib<<<gsz, 256, 0, C.s>>>(N, M, K, m.type.p, m.side.p, m.theta.p, m.alpha.p, m.delta.p, m.dib[0].p,
                                          m.dib[1].p, m.dib[2].p, m.dib[3].p, m.dib[4].p, m.inv_dib_ne.p,
                                          m.inv_dib_tn.p);
    LSG_CHECK_LAUNCH();
    LSG_CUDA(cudaEventRecord(e1, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    float t = 0;
    LSG_CUDA(cudaEventElapsedTime(&t, e0, e1));
    if (ms) *ms = t;
    m.have = true;
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_mesh_get(lsg_ctx* h, int field, void* out)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    Context::Mesh& m = C.mesh;
    LSG_REQUIRE(m.have, LSG_ERR_STATE, "no mesh built (lsg_mesh_build)");
    LSG_REQUIRE(out, LSG_ERR_ARG, "null output");
    const void* src = nullptr;
    size_t bytes = 0;
    const long long n = (long long)m.N * m.M * m.K;
    const long long ns[3] = {(long long)(m.N - 1) * m.M * m.K, (long long)m.N * (m.M - 1) * m.K,
                             (long long)m.N * m.M * (m.K - 1)};
    switch (field) {
    case LSG_MESH_PHI_LS: src = m.phi_ls.p; bytes = n * 8; break;
    case LSG_MESH_PHI: src = m.phi.p; bytes = n * 8; break;
    case LSG_MESH_ALPHA: src = m.alpha.p; bytes = 3 * n * 8; break;
    case LSG_MESH_SIDE_TYPE: src = m.side.p; bytes = 3 * n * 4; break;
    case LSG_MESH_CELL_TYPE: src = m.type.p; bytes = n * 4; break;
    case LSG_MESH_THETA: src = m.theta.p; bytes = 3 * n * 8; break;
    case LSG_MESH_DELTA: src = m.delta.p; bytes = 3 * n * 8; break;
    case LSG_MESH_VOF: src = m.vof.p; bytes = n * 8; break;
    case LSG_MESH_INV_VOF: src = m.inv_vof.p; bytes = n * 8; break;
    case LSG_MESH_XTYPE: case LSG_MESH_YTYPE: case LSG_MESH_ZTYPE: {
        const int d = field - LSG_MESH_XTYPE;
        src = m.stype[d].p;
        bytes = ns[d] * 4;
        break;
    }
    case LSG_MESH_VOF_X: case LSG_MESH_VOF_Y: case LSG_MESH_VOF_Z: {
        const int d = field - LSG_MESH_VOF_X;
        src = m.svof[d].p;
        bytes = ns[d] * 8;
        break;
    }
    case LSG_MESH_INV_MX: case LSG_MESH_INV_MY: case LSG_MESH_INV_MZ: {
        const int d = field - LSG_MESH_INV_MX;
        src = m.sinv[d].p;
        bytes = ns[d] * 8;
        break;
    }
    case LSG_MESH_DIB_EN: case LSG_MESH_DIB_WS: case LSG_MESH_DIB_NB: case LSG_MESH_DIB_ST: case LSG_MESH_DIB_MAX:
        src = m.dib[field - LSG_MESH_DIB_EN].p;
        bytes = 3 * n * 8;
        break;
    case LSG_MESH_INV_DIB_NE: src = m.inv_dib_ne.p; bytes = 3 * n * 8; break;
    case LSG_MESH_INV_DIB_TN: src = m.inv_dib_tn.p; bytes = 3 * n * 8; break;
    default: throw Error{LSG_ERR_ARG, "unknown mesh field"};
    }
    LSG_CUDA(cudaSetDevice(C.device));
    LSG_CUDA(cudaMemcpyAsync(out, src, bytes, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_mesh_osc_sweeps(const lsg_ctx* h)
{
    if (!h || !h->c.mesh.have) return LSG_ERR_STATE;
    return h->c.mesh.osc_sweeps;
}

int lsg_set_matrix_mesh(lsg_ctx* h, long long pin0, long long pin1)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    WallTimer wt(C.matrix_ms);
    Context::Mesh& m = C.mesh;
    LSG_REQUIRE(m.have, LSG_ERR_STATE, "no mesh built (lsg_mesh_build)");
    const long long n = (long long)m.N * m.M * m.K;
    LSG_REQUIRE(pin0 >= -1 && pin0 < n && pin1 >= -1 && pin1 < n, LSG_ERR_ARG, "pinned row outside the grid");
    LSG_CUDA(cudaSetDevice(C.device));
    const long long ns[3] = {(long long)(m.N - 1) * m.M * m.K, (long long)m.N * (m.M - 1) * m.K,
                             (long long)m.N * m.M * (m.K - 1)};
    Context::Geometry& g = C.geo;
    g.have = false;
    g.have_stypes = false;
    g.type.alloc(n);
    g.theta.alloc(3 * n);
    g.delta.alloc(3 * n);
    LSG_CUDA(cudaMemcpyAsync(g.type.p, m.type.p, n * 4, cudaMemcpyDeviceToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(g.theta.p, m.theta.p, 3 * n * 8, cudaMemcpyDeviceToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(g.delta.p, m.delta.p, 3 * n * 8, cudaMemcpyDeviceToDevice, C.s));
    for (int d = 0; d < 3; d++) {
        g.inv[d].alloc(ns[d]);
        g.stype[d].alloc(ns[d]);
        LSG_CUDA(cudaMemcpyAsync(g.inv[d].p, m.sinv[d].p, ns[d] * 8, cudaMemcpyDeviceToDevice, C.s));
        LSG_CUDA(cudaMemcpyAsync(g.stype[d].p, m.stype[d].p, ns[d] * 4, cudaMemcpyDeviceToDevice, C.s));
    }
    assemble_laplace(C, m.N, m.M, m.K, pin0, pin1);
    g.have_stypes = true;
    return LSG_OK;
    LSG_API_END(h)
}

static void projection_rhs(Context& C, const double* u, const double* v, const double* w, const double* flux, double* b)
{
    const Dims& d = C.d;
    const Context::Geometry& g = C.geo;
    k_projection_rhs<<<dim3((d.N + 31) / 32, (d.M + 7) / 8, d.K), dim3(32, 8), 0, C.s>>>(
        d.N, d.M, d.K, g.type.p, g.theta.p, g.delta.p, flux, u, v, w, g.pin0, g.pin1, b);
    LSG_CHECK_LAUNCH();
}

static void projection_correct(Context& C, const double* phi, const double* const pred[3], double* const out[3],
                               double* p, double coef, double vbase, bool outflow)
{
    const Dims& d = C.d;
    const Context::Geometry& g = C.geo;
    for (int dir = 0; dir < 3; dir++) {
        const int Ns = d.N - (dir == 0), Ms = d.M - (dir == 1), Ks = d.K - (dir == 2);
        k_projection_velocity<<<dim3((Ns + 31) / 32, (Ms + 7) / 8, Ks), dim3(32, 8), 0, C.s>>>(
            dir, d.N, d.M, d.K, g.stype[dir].p, g.theta.p, g.delta.p, g.inv[dir].p, phi, pred[dir], out[dir]);
        LSG_CHECK_LAUNCH();
    }
    if (outflow) {
        if (d.M > 2 && d.K > 2) {
            k_outflow_east<<<dim3((d.M - 2 + 127) / 128, d.K - 2), 128, 0, C.s>>>(d.N, d.M, d.K, vbase, out[0], out[1],
                                                                                 out[2]);
            LSG_CHECK_LAUNCH();
        }
        k_outflow_tb<<<dim3((d.N - 1 + 127) / 128, d.M - 1), 128, 0, C.s>>>(d.N, d.M, d.K, out[2]);
        LSG_CHECK_LAUNCH();
    }
    k_pressure_update<<<grid_for(C.n, 256), 256, 0, C.s>>>(C.n, coef, phi, p);
    LSG_CHECK_LAUNCH();
}

int lsg_projection_rhs_device(lsg_ctx* h, const double* u, const double* v, const double* w, const double* flux,
                              double* b)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.geo.have, LSG_ERR_STATE, "no geometry set (lsg_set_matrix_geometry)");
    LSG_REQUIRE(u && v && w && flux && b, LSG_ERR_ARG, "null field");
    LSG_CUDA(cudaSetDevice(C.device));
    projection_rhs(C, u, v, w, flux, b);
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_projection_rhs(lsg_ctx* h, const double* u, const double* v, const double* w, const double* flux, double* b)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.geo.have, LSG_ERR_STATE, "no geometry set (lsg_set_matrix_geometry)");
    LSG_REQUIRE(u && v && w && flux && b, LSG_ERR_ARG, "null field");
    LSG_CUDA(cudaSetDevice(C.device));
    const Dims& d = C.d;
    const long long n = C.n, cnt[3] = {(long long)(d.N - 1) * d.M * d.K, (long long)d.N * (d.M - 1) * d.K,
                                       (long long)d.N * d.M * (d.K - 1)};
    TmpBuf<double> du(C.s, C.pool), dv(C.s, C.pool), dw(C.s, C.pool), df(C.s, C.pool), db(C.s, C.pool);
    du.alloc(cnt[0]);
    dv.alloc(cnt[1]);
    dw.alloc(cnt[2]);
    df.alloc(n);
    db.alloc(n);
    LSG_CUDA(cudaMemcpyAsync(du.p, u, cnt[0] * 8, cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(dv.p, v, cnt[1] * 8, cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(dw.p, w, cnt[2] * 8, cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(df.p, flux, n * 8, cudaMemcpyHostToDevice, C.s));
    projection_rhs(C, du.p, dv.p, dw.p, df.p, db.p);
    LSG_CUDA(cudaMemcpyAsync(b, db.p, n * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

static void laplace_flux(Context& C, const int* side, const double* vib, const double* u_w, const double* bc,
                         const double* ux, double* flux)
{
    const Dims& d = C.d;
    const Context::Geometry& g = C.geo;
    k_laplace_flux<<<dim3((d.N + 31) / 32, (d.M + 7) / 8, d.K), dim3(32, 8), 0, C.s>>>(
        d.N, d.M, d.K, g.type.p, side, g.theta.p, g.delta.p, vib, u_w, bc[0], bc[1], bc[2], bc[3], bc[4], ux, flux);
    LSG_CHECK_LAUNCH();
}

int lsg_laplace_flux_device(lsg_ctx* h, const int* side_type, const double* vib, const double* u_w, const double* bc,
                            const double* ux, double* flux)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.geo.have, LSG_ERR_STATE, "no geometry set (lsg_set_matrix_geometry)");
    LSG_REQUIRE(side_type && vib && u_w && bc && ux && flux, LSG_ERR_ARG, "null argument");
    LSG_CUDA(cudaSetDevice(C.device));
    laplace_flux(C, side_type, vib, u_w, bc, ux, flux);
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_laplace_flux(lsg_ctx* h, const int* side_type, const double* vib, const double* u_w, const double* bc,
                     const double* ux, double* flux)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.geo.have, LSG_ERR_STATE, "no geometry set (lsg_set_matrix_geometry)");
    LSG_REQUIRE(side_type && vib && u_w && bc && ux && flux, LSG_ERR_ARG, "null argument");
    LSG_CUDA(cudaSetDevice(C.device));
    const Dims& d = C.d;
    const long long n = C.n, nx = (long long)(d.N - 1) * d.M * d.K, nmk = (long long)d.M * d.K;
    TmpBuf<int> ds(C.s, C.pool);
    TmpBuf<double> dv(C.s, C.pool), dw(C.s, C.pool), dux(C.s, C.pool), df(C.s, C.pool);
    ds.alloc(3 * n);
    dv.alloc(3 * n);
    dw.alloc(nmk);
    dux.alloc(nx);
    df.alloc(n);
    LSG_CUDA(cudaMemcpyAsync(ds.p, side_type, 3 * n * sizeof(int), cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(dv.p, vib, 3 * n * 8, cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(dw.p, u_w, nmk * 8, cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(dux.p, ux, nx * 8, cudaMemcpyHostToDevice, C.s));
    laplace_flux(C, ds.p, dv.p, dw.p, bc, dux.p, df.p);
    LSG_CUDA(cudaMemcpyAsync(flux, df.p, n * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_momentum_rhs(lsg_ctx* h, int dir, const int* rowptr, const int* col, const double* val, const double* flux2,
                     const double* u, const double* uprev, const double* vof, const double* hflux, const double* p,
                     const double* prev_aux, double coef2, double* right, double* aux)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.geo.have && C.geo.have_stypes, LSG_ERR_STATE,
                "geometry and staggered types needed (lsg_set_matrix_geometry, lsg_set_staggered_types)");
    LSG_REQUIRE(dir >= 0 && dir <= 2, LSG_ERR_ARG, "dir must be 0 (x), 1 (y) or 2 (z)");
    // rowptr == NULL: flux2 already holds the convective term flux2 + C u
    // (lsg_convective_apply with init = flux2)
    LSG_REQUIRE((!rowptr || (col && val)) && flux2 && u && uprev && vof && hflux && p && prev_aux && right && aux,
                LSG_ERR_ARG, "null argument");
    LSG_CUDA(cudaSetDevice(C.device));
    const Dims& d = C.d;
    const int Ns = d.N - (dir == 0), Ms = d.M - (dir == 1), Ks = d.K - (dir == 2);
    const long long ns = (long long)Ns * Ms * Ks, n = C.n;
    const long long nnz = rowptr ? rowptr[ns] : 0;
    if (rowptr) {
        LSG_REQUIRE(rowptr[0] == 0 && nnz >= 0, LSG_ERR_ARG, "bad CSR row pointer");
        for (long long i = 0; i < ns; i++)
            LSG_REQUIRE(rowptr[i] <= rowptr[i + 1], LSG_ERR_ARG, "CSR row pointer not monotone");
        for (long long e = 0; e < nnz; e++)
            LSG_REQUIRE(col[e] >= 0 && col[e] < ns, LSG_ERR_ARG, "CSR column outside the staggered grid");
    }
    TmpBuf<int> drp(C.s, C.pool), dcol(C.s, C.pool);
    TmpBuf<double> dval(C.s, C.pool), dflux2(C.s, C.pool), du(C.s, C.pool), dup(C.s, C.pool), dvof(C.s, C.pool), dhf(C.s, C.pool), dp(C.s, C.pool), dprev(C.s, C.pool), dgp(C.s, C.pool), dr(C.s, C.pool), da(C.s, C.pool);
    if (rowptr) {
        drp.alloc(ns + 1);
        dcol.alloc(std::max<long long>(nnz, 1));
        dval.alloc(std::max<long long>(nnz, 1));
    }
    for (TmpBuf<double>* b : {&dflux2, &du, &dup, &dvof, &dhf, &dprev, &dgp, &dr, &da}) b->alloc(ns);
    dp.alloc(n);
    if (rowptr) {
        LSG_CUDA(cudaMemcpyAsync(drp.p, rowptr, (ns + 1) * sizeof(int), cudaMemcpyHostToDevice, C.s));
        if (nnz) {
            LSG_CUDA(cudaMemcpyAsync(dcol.p, col, nnz * sizeof(int), cudaMemcpyHostToDevice, C.s));
            LSG_CUDA(cudaMemcpyAsync(dval.p, val, nnz * 8, cudaMemcpyHostToDevice, C.s));
        }
    }
    const double* hsrc[6] = {flux2, u, uprev, vof, hflux, prev_aux};
    TmpBuf<double>* dst[6] = {&dflux2, &du, &dup, &dvof, &dhf, &dprev};
    for (int k = 0; k < 6; k++) LSG_CUDA(cudaMemcpyAsync(dst[k]->p, hsrc[k], ns * 8, cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(dp.p, p, n * 8, cudaMemcpyHostToDevice, C.s));
    const Context::Geometry& g = C.geo;
    k_gradient_apply<<<dim3((Ns + 31) / 32, (Ms + 7) / 8, Ks), dim3(32, 8), 0, C.s>>>(
        dir, d.N, d.M, d.K, g.stype[dir].p, g.theta.p, g.delta.p, dp.p, dgp.p);
    LSG_CHECK_LAUNCH();
    k_momentum_rhs<<<grid_for(ns, 256), 256, 0, C.s>>>(ns, drp.p, dcol.p, dval.p, dflux2.p, du.p, dup.p, dvof.p, dhf.p,
                                                       dprev.p, dgp.p, coef2, dr.p, da.p);
    LSG_CHECK_LAUNCH();
    LSG_CUDA(cudaMemcpyAsync(right, dr.p, ns * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaMemcpyAsync(aux, da.p, ns * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_momentum_rhs_device(lsg_ctx* h, int dir, const double* conv, const double* u, const double* uprev,
                            const double* vof, const double* hflux, const double* p, const double* prev_aux,
                            double coef2, double* right, double* aux, double* gp_work)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.geo.have && C.geo.have_stypes, LSG_ERR_STATE,
                "geometry and staggered types needed (lsg_set_matrix_geometry, lsg_set_staggered_types)");
    LSG_REQUIRE(dir >= 0 && dir <= 2, LSG_ERR_ARG, "dir must be 0 (x), 1 (y) or 2 (z)");
    LSG_REQUIRE(conv && u && uprev && vof && hflux && p && prev_aux && right && aux && gp_work, LSG_ERR_ARG,
                "null argument");
    LSG_CUDA(cudaSetDevice(C.device));
    const Dims& d = C.d;
    const int Ns = d.N - (dir == 0), Ms = d.M - (dir == 1), Ks = d.K - (dir == 2);
    const long long ns = (long long)Ns * Ms * Ks;
    const Context::Geometry& g = C.geo;
    k_gradient_apply<<<dim3((Ns + 31) / 32, (Ms + 7) / 8, Ks), dim3(32, 8), 0, C.s>>>(
        dir, d.N, d.M, d.K, g.stype[dir].p, g.theta.p, g.delta.p, p, gp_work);
    LSG_CHECK_LAUNCH();
    k_momentum_rhs<<<grid_for(ns, 256), 256, 0, C.s>>>(ns, nullptr, nullptr, nullptr, conv, u, uprev, vof, hflux,
                                                       prev_aux, gp_work, coef2, right, aux);
    LSG_CHECK_LAUNCH();
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

static void convective_apply(Context& C, int dir, const double* ux, const double* uy, const double* uz, const double* v,
                             const double* init, double* out, bool zquirk)
{
    const Dims& d = C.d;
    const Context::Geometry& g = C.geo;
    const int Ns = d.N - (dir == 0), Ms = d.M - (dir == 1), Ks = d.K - (dir == 2);
    k_convective_apply<<<dim3((Ns + 31) / 32, (Ms + 7) / 8, Ks), dim3(32, 8), 0, C.s>>>(
        dir, d.N, d.M, d.K, g.stype[dir].p, g.theta.p, g.delta.p, ux, uy, uz, v, init, zquirk, out);
    LSG_CHECK_LAUNCH();
}

int lsg_convective_adjoint_device(lsg_ctx* h, int dir, const double* ux, const double* uy, const double* uz,
                                  const double* v, const double* lam, double* ux_bar, double* uy_bar, double* uz_bar,
                                  double* v_bar, int zconv_reference)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.geo.have && C.geo.have_stypes, LSG_ERR_STATE,
                "geometry and staggered types needed (lsg_set_matrix_geometry, lsg_set_staggered_types)");
    LSG_REQUIRE(dir >= 0 && dir <= 2, LSG_ERR_ARG, "dir must be 0 (x), 1 (y) or 2 (z)");
    LSG_REQUIRE(ux && uy && uz && v && lam && ux_bar && uy_bar && uz_bar && v_bar, LSG_ERR_ARG, "null argument");
    LSG_CUDA(cudaSetDevice(C.device));
    const Dims& d = C.d;
    const Context::Geometry& g = C.geo;
    const int Ns = d.N - (dir == 0), Ms = d.M - (dir == 1), Ks = d.K - (dir == 2);
    k_convective_adjoint<<<dim3((Ns + 31) / 32, (Ms + 7) / 8, Ks), dim3(32, 8), 0, C.s>>>(
        dir, d.N, d.M, d.K, g.stype[dir].p, g.theta.p, g.delta.p, ux, uy, uz, v, lam, zconv_reference != 0, ux_bar,
        uy_bar, uz_bar, v_bar);
    LSG_CHECK_LAUNCH();
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_convective_adjoint(lsg_ctx* h, int dir, const double* ux, const double* uy, const double* uz,
                           const double* v, const double* lam, double* ux_bar, double* uy_bar, double* uz_bar,
                           double* v_bar, int zconv_reference)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.geo.have && C.geo.have_stypes, LSG_ERR_STATE,
                "geometry and staggered types needed (lsg_set_matrix_geometry, lsg_set_staggered_types)");
    LSG_REQUIRE(dir >= 0 && dir <= 2, LSG_ERR_ARG, "dir must be 0 (x), 1 (y) or 2 (z)");
    LSG_REQUIRE(ux && uy && uz && v && lam && ux_bar && uy_bar && uz_bar && v_bar, LSG_ERR_ARG, "null argument");
    LSG_CUDA(cudaSetDevice(C.device));
    const Dims& d = C.d;
    const long long cnt[3] = {(long long)(d.N - 1) * d.M * d.K, (long long)d.N * (d.M - 1) * d.K,
                              (long long)d.N * d.M * (d.K - 1)};
    TmpBuf<double> du[3] = {TmpBuf<double>(C.s, C.pool), TmpBuf<double>(C.s, C.pool), TmpBuf<double>(C.s, C.pool)}, db[3] = {TmpBuf<double>(C.s, C.pool), TmpBuf<double>(C.s, C.pool), TmpBuf<double>(C.s, C.pool)}, dv(C.s, C.pool), dl(C.s, C.pool), dvb(C.s, C.pool);
    const double* hu[3] = {ux, uy, uz};
    for (int e = 0; e < 3; e++) {
        du[e].alloc(cnt[e]);
        db[e].alloc(cnt[e]);
        LSG_CUDA(cudaMemcpyAsync(du[e].p, hu[e], cnt[e] * 8, cudaMemcpyHostToDevice, C.s));
        LSG_CUDA(cudaMemsetAsync(db[e].p, 0, cnt[e] * 8, C.s));
    }
    dv.alloc(cnt[dir]);
    dl.alloc(cnt[dir]);
    dvb.alloc(cnt[dir]);
    LSG_CUDA(cudaMemcpyAsync(dv.p, v, cnt[dir] * 8, cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(dl.p, lam, cnt[dir] * 8, cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemsetAsync(dvb.p, 0, cnt[dir] * 8, C.s));
    const Context::Geometry& g = C.geo;
    const int Ns = d.N - (dir == 0), Ms = d.M - (dir == 1), Ks = d.K - (dir == 2);
    k_convective_adjoint<<<dim3((Ns + 31) / 32, (Ms + 7) / 8, Ks), dim3(32, 8), 0, C.s>>>(
        dir, d.N, d.M, d.K, g.stype[dir].p, g.theta.p, g.delta.p, du[0].p, du[1].p, du[2].p, dv.p, dl.p,
        zconv_reference != 0, db[0].p, db[1].p, db[2].p, dvb.p);
    LSG_CHECK_LAUNCH();
    double* hb[3] = {ux_bar, uy_bar, uz_bar};
    for (int e = 0; e < 3; e++) LSG_CUDA(cudaMemcpyAsync(hb[e], db[e].p, cnt[e] * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaMemcpyAsync(v_bar, dvb.p, cnt[dir] * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_convective_apply_device(lsg_ctx* h, int dir, const double* ux, const double* uy, const double* uz,
                                const double* v, const double* init, double* out, int zconv_reference)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.geo.have && C.geo.have_stypes, LSG_ERR_STATE,
                "geometry and staggered types needed (lsg_set_matrix_geometry, lsg_set_staggered_types)");
    LSG_REQUIRE(dir >= 0 && dir <= 2, LSG_ERR_ARG, "dir must be 0 (x), 1 (y) or 2 (z)");
    LSG_REQUIRE(ux && uy && uz && v && out, LSG_ERR_ARG, "null argument");
    LSG_CUDA(cudaSetDevice(C.device));
    convective_apply(C, dir, ux, uy, uz, v, init, out, zconv_reference != 0);
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_convective_apply(lsg_ctx* h, int dir, const double* ux, const double* uy, const double* uz, const double* v,
                         const double* init, double* out, int zconv_reference)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.geo.have && C.geo.have_stypes, LSG_ERR_STATE,
                "geometry and staggered types needed (lsg_set_matrix_geometry, lsg_set_staggered_types)");
    LSG_REQUIRE(dir >= 0 && dir <= 2, LSG_ERR_ARG, "dir must be 0 (x), 1 (y) or 2 (z)");
    LSG_REQUIRE(ux && uy && uz && v && out, LSG_ERR_ARG, "null argument");
    LSG_CUDA(cudaSetDevice(C.device));
    const Dims& d = C.d;
    const long long cnt[3] = {(long long)(d.N - 1) * d.M * d.K, (long long)d.N * (d.M - 1) * d.K,
                              (long long)d.N * d.M * (d.K - 1)};
    const double* hu[3] = {ux, uy, uz};
    TmpBuf<double> du[3] = {TmpBuf<double>(C.s, C.pool), TmpBuf<double>(C.s, C.pool), TmpBuf<double>(C.s, C.pool)}, dv(C.s, C.pool), di(C.s, C.pool), dout(C.s, C.pool);
    for (int k = 0; k < 3; k++) {
        du[k].alloc(cnt[k]);
        LSG_CUDA(cudaMemcpyAsync(du[k].p, hu[k], cnt[k] * 8, cudaMemcpyHostToDevice, C.s));
    }
    dv.alloc(cnt[dir]);
    dout.alloc(cnt[dir]);
    LSG_CUDA(cudaMemcpyAsync(dv.p, v, cnt[dir] * 8, cudaMemcpyHostToDevice, C.s));
    if (init) {
        di.alloc(cnt[dir]);
        LSG_CUDA(cudaMemcpyAsync(di.p, init, cnt[dir] * 8, cudaMemcpyHostToDevice, C.s));
    }
    convective_apply(C, dir, du[0].p, du[1].p, du[2].p, dv.p, init ? di.p : nullptr, dout.p, zconv_reference != 0);
    LSG_CUDA(cudaMemcpyAsync(out, dout.p, cnt[dir] * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_projection_correct_device(lsg_ctx* h, const double* phi, const double* us, const double* vs, const double* ws,
                                  double* u, double* v, double* w, double* p, double coef, double vbase, int outflow)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.geo.have && C.geo.have_stypes, LSG_ERR_STATE,
                "geometry and staggered types needed (lsg_set_matrix_geometry, lsg_set_staggered_types)");
    LSG_REQUIRE(phi && us && vs && ws && u && v && w && p, LSG_ERR_ARG, "null field");
    LSG_CUDA(cudaSetDevice(C.device));
    const double* pred[3] = {us, vs, ws};
    double* out[3] = {u, v, w};
    projection_correct(C, phi, pred, out, p, coef, vbase, outflow != 0);
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_projection_correct(lsg_ctx* h, const double* phi, const double* us, const double* vs, const double* ws,
                           double* u, double* v, double* w, double* p, double coef, double vbase, int outflow)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.geo.have && C.geo.have_stypes, LSG_ERR_STATE,
                "geometry and staggered types needed (lsg_set_matrix_geometry, lsg_set_staggered_types)");
    LSG_REQUIRE(phi && us && vs && ws && u && v && w && p, LSG_ERR_ARG, "null field");
    LSG_CUDA(cudaSetDevice(C.device));
    const Dims& d = C.d;
    const long long n = C.n, cnt[3] = {(long long)(d.N - 1) * d.M * d.K, (long long)d.N * (d.M - 1) * d.K,
                                       (long long)d.N * d.M * (d.K - 1)};
    TmpBuf<double> dphi(C.s, C.pool), dp(C.s, C.pool), dpred[3] = {TmpBuf<double>(C.s, C.pool), TmpBuf<double>(C.s, C.pool), TmpBuf<double>(C.s, C.pool)}, dout[3] = {TmpBuf<double>(C.s, C.pool), TmpBuf<double>(C.s, C.pool), TmpBuf<double>(C.s, C.pool)};
    dphi.alloc(n);
    dp.alloc(n);
    const double* hpred[3] = {us, vs, ws};
    double* hout[3] = {u, v, w};
    LSG_CUDA(cudaMemcpyAsync(dphi.p, phi, n * 8, cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(dp.p, p, n * 8, cudaMemcpyHostToDevice, C.s));
    const double* pred[3];
    double* out[3];
    for (int k = 0; k < 3; k++) {
        dpred[k].alloc(cnt[k]);
        dout[k].alloc(cnt[k]);
        LSG_CUDA(cudaMemcpyAsync(dpred[k].p, hpred[k], cnt[k] * 8, cudaMemcpyHostToDevice, C.s));
        pred[k] = dpred[k].p;
        out[k] = dout[k].p;
    }
    projection_correct(C, dphi.p, pred, out, dp.p, coef, vbase, outflow != 0);
    for (int k = 0; k < 3; k++)
        LSG_CUDA(cudaMemcpyAsync(hout[k], dout[k].p, cnt[k] * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaMemcpyAsync(p, dp.p, n * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_get_matrix_stencil7(lsg_ctx* h, double* planes)
{
    if (!h || !planes) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.have_matrix, LSG_ERR_STATE, "no operator set");
    LSG_CUDA(cudaSetDevice(C.device));
    LSG_CUDA(cudaMemcpyAsync(planes, C.A7.p, 7 * C.n * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_set_tolerance(lsg_ctx* h, double eps)
{
    if (!h) return LSG_ERR_ARG;
    if (!(eps >= 0.0)) return LSG_ERR_ARG;
    h->c.opt.eps = eps;
    return LSG_OK;
}

int lsg_setup(lsg_ctx* h, const lsg_options* opts)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    WallTimer wt(C.setup_ms);
    LSG_REQUIRE(C.have_matrix, LSG_ERR_STATE, "lsg_set_matrix_csr must be called before lsg_setup");
    LSG_CUDA(cudaSetDevice(C.device));
    ilu_graph_release(C);                  // work buffers are (re)allocated below
    if (opts) C.opt = *opts;
    LSG_REQUIRE(C.opt.method == LSG_METHOD_FGMRES || C.opt.method == LSG_METHOD_BICGSTAB, LSG_ERR_ARG, "bad method");
    LSG_REQUIRE(C.opt.precond >= 0 && C.opt.precond <= 2, LSG_ERR_ARG, "bad preconditioner");
    LSG_REQUIRE(C.opt.restart >= 1 && C.opt.restart <= 64, LSG_ERR_ARG, "restart must be in [1, 64]");
    LSG_REQUIRE(C.opt.max_it >= 1, LSG_ERR_ARG, "max_it must be >= 1");
    LSG_REQUIRE(C.opt.n_post >= 0 && C.opt.n_post <= 16, LSG_ERR_ARG, "n_post must be in [0, 16]");
    LSG_REQUIRE(C.opt.smoother == LSG_SMOOTHER_ADLJ || C.opt.smoother == LSG_SMOOTHER_RBGS, LSG_ERR_ARG,
                "smoother not supported");
    LSG_REQUIRE(C.opt.n_pre >= 0 && C.opt.n_post >= 0 && (C.opt.smoother == LSG_SMOOTHER_RBGS || C.opt.n_pre == 0),
                LSG_ERR_ARG, "pre-smoothing needs the Gauss-Seidel smoother (the ADLJ cycle is V(0, n_post))");
    LSG_REQUIRE(C.opt.adlj_schedule >= LSG_ADLJ_AUTO && C.opt.adlj_schedule <= LSG_ADLJ_FUSED, LSG_ERR_ARG,
                "bad ADLJ schedule");
    C.have_setup = false;
    if (C.opt.precond == LSG_PC_MG) mg_setup(C);
    if (C.opt.precond == LSG_PC_ILU0) ilu_setup(C);
    krylov_alloc(C);
    LSG_CUDA(cudaStreamSynchronize(C.s));
    C.have_setup = true;
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_row_classes(lsg_ctx* h, int level, int* cls, double* dict, int* nclass, int* noff)
{
    if (!h || !nclass || !noff) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.have_matrix, LSG_ERR_STATE, "no operator");
    const int* c = nullptr;
    const double* d = nullptr;
    long long n = 0;
    if (level == 0) {
        c = C.cls0.p;
        d = C.dict0.p;
        n = C.n;
        *nclass = C.nclass0;
        *noff = 7;
    } else {
        LSG_REQUIRE(C.have_setup && C.opt.precond == LSG_PC_MG && level >= 1 && level <= C.mg.L, LSG_ERR_ARG,
                    "level out of range (needs the multigrid setup)");
        const LevelT<double>& lv = C.mg.l64[level];
        c = lv.cls;
        d = lv.dict;
        n = lv.d.n();
        *nclass = lv.nclass;
        *noff = lv.ol.n;
    }
    LSG_CUDA(cudaSetDevice(C.device));
    if (cls) LSG_CUDA(cudaMemcpyAsync(cls, c, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, C.s));
    if (dict)
        LSG_CUDA(cudaMemcpyAsync(dict, d, (size_t)*nclass * *noff * sizeof(double), cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_setup_times(const lsg_ctx* h, double* matrix_ms, double* setup_ms)
{
    if (!h || !matrix_ms || !setup_ms) return LSG_ERR_ARG;
    *matrix_ms = h->c.matrix_ms;
    *setup_ms = h->c.setup_ms;
    return LSG_OK;
}

int lsg_solve_device(lsg_ctx* h, const double* b, double* x, lsg_stats* st)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(b && x, LSG_ERR_ARG, "null vector");
    LSG_CUDA(cudaSetDevice(C.device));
    if (st) std::memset(st, 0, sizeof(*st));
    return solve_device(C, b, x, st);
    LSG_API_END(h)
}

int lsg_solve(lsg_ctx* h, const double* b, double* x, lsg_stats* st)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(b && x, LSG_ERR_ARG, "null vector");
    LSG_REQUIRE(C.have_setup, LSG_ERR_STATE, "lsg_setup must be called before solving");
    LSG_CUDA(cudaSetDevice(C.device));
    if (st) std::memset(st, 0, sizeof(*st));
    const size_t bytes = (size_t)C.n * sizeof(double);
    LSG_CUDA(cudaMemcpyAsync(C.bd.p, b, bytes, cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(C.xd.p, x, bytes, cudaMemcpyHostToDevice, C.s));
    const int rc = solve_device(C, C.bd.p, C.xd.p, st);
    LSG_CUDA(cudaMemcpyAsync(x, C.xd.p, bytes, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return rc;
    LSG_API_END(h)
}

int lsg_apply(lsg_ctx* h, const double* x, double* y)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.have_matrix, LSG_ERR_STATE, "no operator set");
    LSG_REQUIRE(x && y, LSG_ERR_ARG, "null vector");
    LSG_CUDA(cudaSetDevice(C.device));
    const long long n = C.n;
    TmpBuf<double> dx(C.s, C.pool), dy(C.s, C.pool);
    dx.alloc(n);
    dy.alloc(n);
    LSG_CUDA(cudaMemcpyAsync(dx.p, x, n * 8, cudaMemcpyHostToDevice, C.s));
    k_apply7d<double, 1><<<grid_for(n, 256), 256, 0, C.s>>>(C.d.N, C.d.M, C.d.K, C.cls0.p, C.dict0.p, dx.p, dy.p);
    LSG_CHECK_LAUNCH();
    LSG_CUDA(cudaMemcpyAsync(y, dy.p, n * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_precond_apply(lsg_ctx* h, const double* b, double* x)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.have_setup, LSG_ERR_STATE, "lsg_setup must be called first");
    LSG_REQUIRE(b && x, LSG_ERR_ARG, "null vector");
    LSG_CUDA(cudaSetDevice(C.device));
    const long long n = C.n;
    LSG_CUDA(cudaMemcpyAsync(C.bd.p, b, n * 8, cudaMemcpyHostToDevice, C.s));
    precond_apply(C, C.bd.p, C.xd.p);
    LSG_CUDA(cudaMemcpyAsync(x, C.xd.p, n * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_mg_num_levels(const lsg_ctx* h)
{
    if (!h || !h->c.have_setup || h->c.opt.precond != LSG_PC_MG) return LSG_ERR_STATE;
    return h->c.mg.L;
}

int lsg_mg_level_dims(const lsg_ctx* h, int level, int dims[3])
{
    if (!h || !dims) return LSG_ERR_ARG;
    const Context& C = h->c;
    if (!C.have_setup || C.opt.precond != LSG_PC_MG) return LSG_ERR_STATE;
    if (level < 0 || level > C.mg.L) return LSG_ERR_ARG;
    dims[0] = C.mg.dims[level].N;
    dims[1] = C.mg.dims[level].M;
    dims[2] = C.mg.dims[level].K;
    return LSG_OK;
}

int lsg_mg_level_csr(lsg_ctx* h, int level, int* rowptr, int* col, double* val, long long* nnz)
{
    if (!h || !nnz) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.have_setup && C.opt.precond == LSG_PC_MG, LSG_ERR_STATE, "no multigrid hierarchy");
    LSG_REQUIRE(level >= 0 && level <= C.mg.L, LSG_ERR_ARG, "bad level");
    const LevelT<double>& lv = C.mg.l64[level];
    const long long n = lv.d.n();
    const int no = lv.ol.n;
    std::vector<double> box((size_t)no * n);
    LSG_CUDA(cudaMemcpyAsync(box.data(), lv.A, box.size() * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    const int N = lv.d.N, M = lv.d.M, K = lv.d.K, NM = N * M;
    std::vector<std::pair<long long, double>> row;
    long long cntnz = 0;
    for (long long i = 0; i < n; i++) {
        const int z = (int)(i / NM), y = (int)((i - (long long)z * NM) / N), x = (int)(i - (long long)z * NM - (long long)y * N);
        row.clear();
        for (int q = 0; q < no; q++) {
            const int jx = x + lv.off[3 * q], jy = y + lv.off[3 * q + 1], jz = z + lv.off[3 * q + 2];
            if (jx < 0 || jx >= N || jy < 0 || jy >= M || jz < 0 || jz >= K) continue;
            const double v = box[(size_t)q * n + i];
            if (level == 0 && v == 0.0 && !(lv.off[3 * q] == 0 && lv.off[3 * q + 1] == 0 && lv.off[3 * q + 2] == 0)) continue;
            row.push_back({jx + (long long)jy * N + (long long)jz * NM, v});
        }
        std::sort(row.begin(), row.end());
        if (rowptr) rowptr[i] = (int)cntnz;
        if (col)
            for (auto& e : row) {
                col[cntnz] = (int)e.first;
                val[cntnz] = e.second;
                cntnz++;
            }
        else
            cntnz += (long long)row.size();
    }
    if (rowptr) rowptr[n] = (int)cntnz;
    *nnz = cntnz;
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_mg_level_tridiag(lsg_ctx* h, int level, char dir, double* c, double* d, double* e)
{
    if (!h || !c || !d || !e) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.have_setup && C.opt.precond == LSG_PC_MG, LSG_ERR_STATE, "no multigrid hierarchy");
    LSG_REQUIRE(level >= 0 && level < C.mg.L, LSG_ERR_ARG, "level has no smoother");
    const int di = (dir == 'x') ? 0 : (dir == 'y') ? 1 : (dir == 'z') ? 2 : -1;
    LSG_REQUIRE(di >= 0, LSG_ERR_ARG, "dir must be 'x', 'y' or 'z'");
    const LevelT<double>& lv = C.mg.l64[level];
    const long long n = lv.d.n();
    std::vector<double> lo(n), dv(n), up(n);
    LSG_CUDA(cudaMemcpyAsync(lo.data(), lv.lo[di].p, n * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaMemcpyAsync(dv.data(), lv.dinv[di].p, n * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaMemcpyAsync(up.data(), lv.up[di].p, n * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    // map natural -> the direction's storage order (SmootherADLJy::initOrder,
    // smoother_adlj_y.h:51-59; SmootherADLJz::initOrderZ, smoother_adlj_z.h:34-43)
    const int N = lv.d.N, M = lv.d.M, K = lv.d.K;
    long long pos = 0;
    auto nat = [&](long long q) -> long long {
        if (di == 0) return q;
        if (di == 1) {   // q = z*N*M + x*M + y
            const long long z = q / ((long long)N * M), r = q - z * N * M, x = r / M, y = r - x * M;
            return x + N * (y + M * z);
        }
        const long long y = q / ((long long)N * K), r = q - y * N * K, x = r / K, z = r - x * K;   // q = y*N*K + x*K + z
        return x + N * (y + M * z);
    };
    for (pos = 0; pos < n; pos++) {
        const long long i = nat(pos);
        d[pos] = dv[i];
        if (pos + 1 < n) {
            e[pos] = up[i];
            c[pos] = lo[nat(pos + 1)];
        }
    }
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_apply_transpose(lsg_ctx* h, const double* x, double* y)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.have_matrix, LSG_ERR_STATE, "no operator set");
    LSG_REQUIRE(x && y, LSG_ERR_ARG, "null vector");
    LSG_CUDA(cudaSetDevice(C.device));
    const long long n = C.n;
    TmpBuf<double> AT(C.s, C.pool), dx(C.s, C.pool), dy(C.s, C.pool);
    AT.alloc(7 * n);
    dx.alloc(n);
    dy.alloc(n);
    k_transpose7<<<grid_for(n, 256), 256, 0, C.s>>>(C.d.N, C.d.M, C.d.K, C.A7.p, AT.p);
    LSG_CHECK_LAUNCH();
    LSG_CUDA(cudaMemcpyAsync(dx.p, x, n * 8, cudaMemcpyHostToDevice, C.s));
    k_apply7<double, 1><<<grid_for(n, 256), 256, 0, C.s>>>(C.d.N, C.d.M, C.d.K, AT.p, dx.p, dy.p);
    LSG_CHECK_LAUNCH();
    LSG_CUDA(cudaMemcpyAsync(y, dy.p, n * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_projection_adjoint(lsg_ctx* h, const double* ubar_out, const double* vbar_out, const double* wbar_out,
                           const double* pbar_out, double coef, double* ubar, double* vbar, double* wbar,
                           double* fluxbar, lsg_stats* st)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.geo.have && C.geo.have_stypes, LSG_ERR_STATE,
                "geometry and staggered types needed (lsg_set_matrix_geometry, lsg_set_staggered_types)");
    LSG_REQUIRE(ubar_out && vbar_out && wbar_out && pbar_out && ubar && vbar && wbar && fluxbar, LSG_ERR_ARG,
                "null field");
    LSG_CUDA(cudaSetDevice(C.device));
    Context& A = adjoint_context(C);
    if (st) std::memset(st, 0, sizeof(*st));
    const Dims& d = C.d;
    const Context::Geometry& g = C.geo;
    const long long n = C.n, cnt[3] = {(long long)(d.N - 1) * d.M * d.K, (long long)d.N * (d.M - 1) * d.K,
                                       (long long)d.N * d.M * (d.K - 1)};
    const double* hout[3] = {ubar_out, vbar_out, wbar_out};
    double* hin[3] = {ubar, vbar, wbar};
    TmpBuf<double> dout[3] = {TmpBuf<double>(C.s, C.pool), TmpBuf<double>(C.s, C.pool), TmpBuf<double>(C.s, C.pool)}, din[3] = {TmpBuf<double>(C.s, C.pool), TmpBuf<double>(C.s, C.pool), TmpBuf<double>(C.s, C.pool)}, dp(C.s, C.pool), df(C.s, C.pool);
    for (int k = 0; k < 3; k++) {
        dout[k].alloc(cnt[k]);
        din[k].alloc(cnt[k]);
        LSG_CUDA(cudaMemcpyAsync(dout[k].p, hout[k], cnt[k] * 8, cudaMemcpyHostToDevice, C.s));
    }
    dp.alloc(n);
    df.alloc(n);
    LSG_CUDA(cudaMemcpyAsync(dp.p, pbar_out, n * 8, cudaMemcpyHostToDevice, C.s));
    const dim3 blk(32, 8);
    k_projection_adjoint_phi<<<dim3((d.N + 31) / 32, (d.M + 7) / 8, d.K), blk, 0, C.s>>>(
        d.N, d.M, d.K, g.stype[0].p, g.stype[1].p, g.stype[2].p, g.theta.p, g.delta.p, g.inv[0].p, g.inv[1].p,
        g.inv[2].p, dout[0].p, dout[1].p, dout[2].p, dp.p, coef, A.bd.p);
    LSG_CHECK_LAUNCH();
    k_adjoint_live_rows<<<grid_for(n, 256), 256, 0, C.s>>>(n, g.type.p, C.A7.p, A.bd.p);
    LSG_CHECK_LAUNCH();
    LSG_CUDA(cudaMemsetAsync(A.xd.p, 0, n * 8, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    const int rc = solve_device(A, A.bd.p, A.xd.p, st);
    for (int dir = 0; dir < 3; dir++) {
        const int Ns = d.N - (dir == 0), Ms = d.M - (dir == 1), Ks = d.K - (dir == 2);
        k_projection_adjoint_vel<<<dim3((Ns + 31) / 32, (Ms + 7) / 8, Ks), blk, 0, C.s>>>(
            dir, d.N, d.M, d.K, g.type.p, g.theta.p, g.delta.p, A.xd.p, g.pin0, g.pin1, dout[dir].p, din[dir].p);
        LSG_CHECK_LAUNCH();
        LSG_CUDA(cudaMemcpyAsync(hin[dir], din[dir].p, cnt[dir] * 8, cudaMemcpyDeviceToHost, C.s));
    }
    k_pin_zero_copy<<<grid_for(n, 256), 256, 0, C.s>>>(n, g.pin0, g.pin1, A.xd.p, df.p);
    LSG_CHECK_LAUNCH();
    LSG_CUDA(cudaMemcpyAsync(fluxbar, df.p, n * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return rc;
    LSG_API_END(h)
}

int lsg_projection_adjoint_device(lsg_ctx* h, const double* ubar_out, const double* vbar_out,
                                  const double* wbar_out, const double* pbar_out, double coef, double* ubar,
                                  double* vbar, double* wbar, double* fluxbar, lsg_stats* st)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.geo.have && C.geo.have_stypes, LSG_ERR_STATE,
                "geometry and staggered types needed (lsg_set_matrix_geometry, lsg_set_staggered_types)");
    LSG_REQUIRE(ubar_out && vbar_out && wbar_out && pbar_out && ubar && vbar && wbar && fluxbar, LSG_ERR_ARG,
                "null field");
    LSG_CUDA(cudaSetDevice(C.device));
    Context& A = adjoint_context(C);
    if (st) std::memset(st, 0, sizeof(*st));
    const Dims& d = C.d;
    const Context::Geometry& g = C.geo;
    const long long n = C.n;
    const double* dout[3] = {ubar_out, vbar_out, wbar_out};
    double* din[3] = {ubar, vbar, wbar};
    const dim3 blk(32, 8);
    k_projection_adjoint_phi<<<dim3((d.N + 31) / 32, (d.M + 7) / 8, d.K), blk, 0, C.s>>>(
        d.N, d.M, d.K, g.stype[0].p, g.stype[1].p, g.stype[2].p, g.theta.p, g.delta.p, g.inv[0].p, g.inv[1].p,
        g.inv[2].p, dout[0], dout[1], dout[2], pbar_out, coef, A.bd.p);
    LSG_CHECK_LAUNCH();
    k_adjoint_live_rows<<<grid_for(n, 256), 256, 0, C.s>>>(n, g.type.p, C.A7.p, A.bd.p);
    LSG_CHECK_LAUNCH();
    LSG_CUDA(cudaMemsetAsync(A.xd.p, 0, n * 8, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    const int rc = solve_device(A, A.bd.p, A.xd.p, st);
    for (int dir = 0; dir < 3; dir++) {
        const int Ns = d.N - (dir == 0), Ms = d.M - (dir == 1), Ks = d.K - (dir == 2);
        k_projection_adjoint_vel<<<dim3((Ns + 31) / 32, (Ms + 7) / 8, Ks), blk, 0, C.s>>>(
            dir, d.N, d.M, d.K, g.type.p, g.theta.p, g.delta.p, A.xd.p, g.pin0, g.pin1, dout[dir], din[dir]);
        LSG_CHECK_LAUNCH();
    }
    k_pin_zero_copy<<<grid_for(n, 256), 256, 0, C.s>>>(n, g.pin0, g.pin1, A.xd.p, fluxbar);
    LSG_CHECK_LAUNCH();
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return rc;
    LSG_API_END(h)
}

int lsg_momentum_cotangents_device(lsg_ctx* h, int dir, const double* vof, const double* rsol, double coef2,
                                   double* r, double* fbar, double* ubar, double* uprevbar, double* histbar,
                                   double* convbar)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.geo.have && C.geo.have_stypes, LSG_ERR_STATE,
                "geometry and staggered types needed (lsg_set_matrix_geometry, lsg_set_staggered_types)");
    LSG_REQUIRE(dir >= 0 && dir <= 2, LSG_ERR_ARG, "dir must be 0, 1 or 2");
    LSG_REQUIRE(vof && rsol && r && fbar && ubar && uprevbar && histbar && convbar, LSG_ERR_ARG, "null field");
    LSG_CUDA(cudaSetDevice(C.device));
    const Dims& d = C.d;
    const long long ns = (long long)(d.N - (dir == 0)) * (d.M - (dir == 1)) * (d.K - (dir == 2));
    k_momentum_cotangents<<<grid_for(ns, 256), 256, 0, C.s>>>(ns, C.geo.stype[dir].p, vof, rsol, coef2, r, fbar,
                                                                ubar, uprevbar, histbar, convbar);
    LSG_CHECK_LAUNCH();
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_fluid_faces_device(lsg_ctx* h, int dir, const double* in, double* out)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.geo.have && C.geo.have_stypes, LSG_ERR_STATE,
                "geometry and staggered types needed (lsg_set_matrix_geometry, lsg_set_staggered_types)");
    LSG_REQUIRE(dir >= 0 && dir <= 2, LSG_ERR_ARG, "dir must be 0, 1 or 2");
    LSG_REQUIRE(in && out, LSG_ERR_ARG, "null field");
    LSG_CUDA(cudaSetDevice(C.device));
    const Dims& d = C.d;
    const long long ns = (long long)(d.N - (dir == 0)) * (d.M - (dir == 1)) * (d.K - (dir == 2));
    k_fluid_faces<<<grid_for(ns, 256), 256, 0, C.s>>>(ns, C.geo.stype[dir].p, in, out);
    LSG_CHECK_LAUNCH();
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_clamp_transpose_device(lsg_ctx* h, const double* qx, const double* qz, const double* bx, const double* by,
                               const double* bz, double* ox, double* oy, double* oz)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.have_matrix, LSG_ERR_STATE, "no grid (set an operator first)");
    LSG_REQUIRE(qx && qz && bx && by && bz && ox && oy && oz, LSG_ERR_ARG, "null field");
    LSG_CUDA(cudaSetDevice(C.device));
    const Dims& d = C.d;
    LSG_REQUIRE(d.N >= 2 && d.M >= 3 && d.K >= 3, LSG_ERR_ARG, "grid too small for the outflow clamps");
    const long long nx = (long long)(d.N - 1) * d.M * d.K, ny = (long long)d.N * (d.M - 1) * d.K,
                    nz = (long long)d.N * d.M * (d.K - 1);
    if (ox != bx) LSG_CUDA(cudaMemcpyAsync(ox, bx, nx * sizeof(double), cudaMemcpyDeviceToDevice, C.s));
    if (oy != by) LSG_CUDA(cudaMemcpyAsync(oy, by, ny * sizeof(double), cudaMemcpyDeviceToDevice, C.s));
    if (oz != bz) LSG_CUDA(cudaMemcpyAsync(oz, bz, nz * sizeof(double), cudaMemcpyDeviceToDevice, C.s));
    const long long rows = 2LL * (d.M - 2) * (d.K - 2);
    k_clamp_transpose_east<<<grid_for(rows, 256), 256, 0, C.s>>>(d.N, d.M, d.K, qx, ox, oy, oz);
    LSG_CHECK_LAUNCH();
    const long long faces = (long long)(d.N - 1) * (d.M - 1);
    k_clamp_transpose_tb<<<grid_for(faces, 256), 256, 0, C.s>>>(d.N, d.M, d.K, qz, oz);
    LSG_CHECK_LAUNCH();
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_scatter_add_device(lsg_ctx* h, long long count, double* dst, const long long* dst_idx, const double* src,
                           const long long* src_idx, const double* coef, const double* src2,
                           const long long* src2_idx)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(count >= 0, LSG_ERR_ARG, "negative count");
    if (count == 0) return LSG_OK;
    LSG_REQUIRE(dst && dst_idx && src && src_idx && coef && (!src2 || src2_idx), LSG_ERR_ARG, "null array");
    LSG_CUDA(cudaSetDevice(C.device));
    k_scatter_add<<<grid_for(count, 256), 256, 0, C.s>>>(count, dst, dst_idx, src, src_idx, coef, src2, src2_idx);
    LSG_CHECK_LAUNCH();
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_axpy_device(lsg_ctx* h, long long n, double alpha, const double* x, double* y)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(n >= 0 && x && y, LSG_ERR_ARG, "bad vector");
    LSG_CUDA(cudaSetDevice(C.device));
    if (n > 0) {
        k_axpy<<<grid_for(n, 256), 256, 0, C.s>>>(n, alpha, x, y);
        LSG_CHECK_LAUNCH();
    }
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_gradient_transpose_device(lsg_ctx* h, const double* gx, const double* gy, const double* gz, double* out)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.geo.have && C.geo.have_stypes, LSG_ERR_STATE,
                "geometry and staggered types needed (lsg_set_matrix_geometry, lsg_set_staggered_types)");
    LSG_REQUIRE(gx && gy && gz && out, LSG_ERR_ARG, "null field");
    LSG_CUDA(cudaSetDevice(C.device));
    const Dims& d = C.d;
    const Context::Geometry& g = C.geo;
    TmpBuf<double> dzero(C.s, C.pool);
    dzero.alloc(C.n);
    LSG_CUDA(cudaMemsetAsync(dzero.p, 0, C.n * 8, C.s));
    k_projection_adjoint_phi<<<dim3((d.N + 31) / 32, (d.M + 7) / 8, d.K), dim3(32, 8), 0, C.s>>>(
        d.N, d.M, d.K, g.stype[0].p, g.stype[1].p, g.stype[2].p, g.theta.p, g.delta.p, nullptr, nullptr, nullptr, gx,
        gy, gz, dzero.p, 0.0, out);
    LSG_CHECK_LAUNCH();
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_gradient_transpose(lsg_ctx* h, const double* gx, const double* gy, const double* gz, double* out)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.geo.have && C.geo.have_stypes, LSG_ERR_STATE,
                "geometry and staggered types needed (lsg_set_matrix_geometry, lsg_set_staggered_types)");
    LSG_REQUIRE(gx && gy && gz && out, LSG_ERR_ARG, "null field");
    LSG_CUDA(cudaSetDevice(C.device));
    const Dims& d = C.d;
    const Context::Geometry& g = C.geo;
    const long long n = C.n, cnt[3] = {(long long)(d.N - 1) * d.M * d.K, (long long)d.N * (d.M - 1) * d.K,
                                       (long long)d.N * d.M * (d.K - 1)};
    const double* hin[3] = {gx, gy, gz};
    TmpBuf<double> din[3] = {TmpBuf<double>(C.s, C.pool), TmpBuf<double>(C.s, C.pool), TmpBuf<double>(C.s, C.pool)}, dzero(C.s, C.pool), dout(C.s, C.pool);
    for (int k = 0; k < 3; k++) {
        din[k].alloc(cnt[k]);
        LSG_CUDA(cudaMemcpyAsync(din[k].p, hin[k], cnt[k] * 8, cudaMemcpyHostToDevice, C.s));
    }
    dzero.alloc(n);
    dout.alloc(n);
    LSG_CUDA(cudaMemsetAsync(dzero.p, 0, n * 8, C.s));
    k_projection_adjoint_phi<<<dim3((d.N + 31) / 32, (d.M + 7) / 8, d.K), dim3(32, 8), 0, C.s>>>(
        d.N, d.M, d.K, g.stype[0].p, g.stype[1].p, g.stype[2].p, g.theta.p, g.delta.p, nullptr, nullptr, nullptr,
        din[0].p, din[1].p, din[2].p, dzero.p, 0.0, dout.p);
    LSG_CHECK_LAUNCH();
    LSG_CUDA(cudaMemcpyAsync(out, dout.p, n * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_tecplot_sol_write(const char* path, int N, int M, int K, const double* nodes, const double* delta,
                          const double* theta, const int* celltype, const double* u, const double* v,
                          const double* w, const double* p, const double* u_w, const double* bc, int flow)
{
    if (!path || N < 2 || M < 2 || K < 3 || !nodes || !delta || !theta || !celltype || !u || !v || !w || !p || !bc)
        return LSG_ERR_ARG;
    try {
        const std::string s = tecplot_sol_bytes(N, M, K, nodes, delta, theta, celltype, u, v, w, p, u_w, bc,
                                                flow != 0);
        FILE* f = std::fopen(path, "wb");
        if (!f) return LSG_ERR_ARG;
        const size_t wr = std::fwrite(s.data(), 1, s.size(), f);
        const int cl = std::fclose(f);
        return (wr == s.size() && cl == 0) ? LSG_OK : LSG_ERR_ARG;
    } catch (const std::bad_alloc&) {
        return LSG_ERR_NOMEM;
    }
}

int lsg_tecplot_sol_async(lsg_ctx* h, const char* path, const double* nodes, const double* delta,
                          const double* theta, const int* celltype, const double* u, const double* v,
                          const double* w, const double* p, const double* u_w, const double* bc, int flow)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.geo.have, LSG_ERR_STATE, "a context holding the base grid's geometry is needed "
                                           "(lsg_set_matrix_geometry)");
    LSG_REQUIRE(path && nodes && delta && theta && celltype && u && v && w && p && bc, LSG_ERR_ARG, "null argument");
    LSG_REQUIRE(C.d.N >= 2 && C.d.M >= 2 && C.d.K >= 3, LSG_ERR_ARG, "grid too small for the printer");
    LSG_CUDA(cudaSetDevice(C.device));
    if (!C.tec) C.tec.reset(new TecplotAsync);
    TecplotAsync& T = *C.tec;
    if (T.th.joinable()) T.th.join();                      // one write in flight per context
    const int N = C.d.N, M = C.d.M, K = C.d.K;
    const size_t n = (size_t)C.n, c0 = (size_t)(N - 1) * M * K, c1 = (size_t)N * (M - 1) * K,
                 c2 = (size_t)N * M * (K - 1);
    const size_t len = c0 + c1 + c2 + n;
    if (T.pinned_len < len) {
        if (T.pinned) cudaFreeHost(T.pinned);
        T.pinned = nullptr;
        T.pinned_len = 0;
        LSG_CUDA(cudaMallocHost(&T.pinned, len * sizeof(double)));
        T.pinned_len = len;
    }
    double* hp = T.pinned;
    LSG_CUDA(cudaMemcpyAsync(hp, u, c0 * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaMemcpyAsync(hp + c0, v, c1 * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaMemcpyAsync(hp + c0 + c1, w, c2 * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaMemcpyAsync(hp + c0 + c1 + c2, p, n * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));                  // the caller may overwrite the fields on return
    std::vector<double> vn(nodes, nodes + 3 * n), vd(delta, delta + 3 * n), vt(theta, theta + 3 * n);
    std::vector<int> vc(celltype, celltype + n);
    std::vector<double> vw;
    if (u_w) vw.assign(u_w, u_w + (size_t)M * K);
    std::vector<double> vb(bc, bc + 18);
    const std::string sp(path);
    const bool fl = flow != 0;
    // the status stays sticky: an error of an earlier write that nobody
    // collected with lsg_tecplot_wait survives this new write
    TecplotAsync* tp = &T;
    T.th = std::thread([tp, N, M, K, hp, c0, c1, c2, sp, fl, vn = std::move(vn), vd = std::move(vd),
                        vt = std::move(vt), vc = std::move(vc), vw = std::move(vw), vb = std::move(vb)]() {
        try {
            const std::string s = tecplot_sol_bytes(N, M, K, vn.data(), vd.data(), vt.data(), vc.data(), hp, hp + c0,
                                                    hp + c0 + c1, hp + c0 + c1 + c2,
                                                    vw.empty() ? nullptr : vw.data(), vb.data(), fl);
            FILE* f = std::fopen(sp.c_str(), "wb");
            if (!f) {
                tp->status = LSG_ERR_ARG;
                return;
            }
            const size_t wr = std::fwrite(s.data(), 1, s.size(), f);
            if (std::fclose(f) != 0 || wr != s.size()) tp->status = LSG_ERR_ARG;
        } catch (const std::bad_alloc&) {
            tp->status = LSG_ERR_NOMEM;
        } catch (...) {
            // nothing may escape a std::thread (it would end the process)
            tp->status = LSG_ERR_ARG;
        }
    });
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_tecplot_wait(lsg_ctx* h)
{
    if (!h) return LSG_ERR_ARG;
    if (!h->c.tec) return LSG_OK;
    TecplotAsync& T = *h->c.tec;
    if (T.th.joinable()) T.th.join();
    const int st = T.status;
    T.status = LSG_OK;       // collected: the next write starts clean
    return st;
}

int lsg_solve_adjoint(lsg_ctx* h, const double* g, double* lambda, lsg_stats* st)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(g && lambda, LSG_ERR_ARG, "null vector");
    LSG_CUDA(cudaSetDevice(C.device));
    Context& A = adjoint_context(C);
    if (st) std::memset(st, 0, sizeof(*st));
    const size_t bytes = (size_t)A.n * sizeof(double);
    LSG_CUDA(cudaMemcpyAsync(A.bd.p, g, bytes, cudaMemcpyHostToDevice, A.s));
    LSG_CUDA(cudaMemcpyAsync(A.xd.p, lambda, bytes, cudaMemcpyHostToDevice, A.s));
    const int rc = solve_device(A, A.bd.p, A.xd.p, st);
    LSG_CUDA(cudaMemcpyAsync(lambda, A.xd.p, bytes, cudaMemcpyDeviceToHost, A.s));
    LSG_CUDA(cudaStreamSynchronize(A.s));
    return rc;
    LSG_API_END(h)
}

int lsg_operator_gradient(lsg_ctx* h, const double* lambda, const double* x, double* grad)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.have_matrix, LSG_ERR_STATE, "no operator set");
    LSG_REQUIRE(lambda && x && grad, LSG_ERR_ARG, "null vector");
    LSG_CUDA(cudaSetDevice(C.device));
    const long long n = C.n;
    TmpBuf<double> dl(C.s, C.pool), dx(C.s, C.pool), dg(C.s, C.pool);
    dl.alloc(n);
    dx.alloc(n);
    dg.alloc(7 * n);
    LSG_CUDA(cudaMemcpyAsync(dl.p, lambda, n * 8, cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(dx.p, x, n * 8, cudaMemcpyHostToDevice, C.s));
    k_operator_grad7<<<grid_for(n, 256), 256, 0, C.s>>>(C.d.N, C.d.M, C.d.K, dl.p, dx.p, dg.p);
    LSG_CHECK_LAUNCH();
    LSG_CUDA(cudaMemcpyAsync(grad, dg.p, 7 * n * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_selftest_wait_limit(lsg_ctx* h)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.have_setup && C.opt.precond == LSG_PC_ILU0, LSG_ERR_STATE, "needs lsg_setup with ILU(0)");
    LSG_CUDA(cudaSetDevice(C.device));
    LSG_CUDA(cudaMemsetAsync(C.t1.p, 0, C.n * sizeof(double), C.s));
    if (C.ilu_blocks == 0) ilu_coop(C, C.t1.p, C.t2.p);   // sizes the sweep (a normal run)
    LSG_REQUIRE(C.ilu_blocks >= 2, LSG_ERR_STATE, "the self-test needs a one-launch sweep of two CTAs or more");
    LSG_CUDA(cudaStreamSynchronize(C.s));
    ilu_coop(C, C.t1.p, C.t2.p, 0);                // CTA 0 withholds its first arrival
    ilu_check(C);                                  // throws: the others' wait ran out
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_profile_kernel(lsg_ctx* h, int which, int reps, double* ms_per_launch, double* bytes_per_launch)
{
    if (!h || !ms_per_launch || !bytes_per_launch || reps < 1) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.have_setup && C.opt.precond == LSG_PC_MG, LSG_ERR_STATE, "needs the multigrid setup");
    LSG_CUDA(cudaSetDevice(C.device));
    const bool f32 = C.mg.fp32;
    const double w = f32 ? 4.0 : 8.0;
    const long long n = C.n;
    auto launch = [&]() {
        if (which >= 0 && which <= 2) {
            if (f32) line_solve<float>(C.mg.l32[0], which, C.opt.zline_reference != 0, (float)C.opt.omega, C.s);
            else line_solve<double>(C.mg.l64[0], which, C.opt.zline_reference != 0, C.opt.omega, C.s);
        } else if (which == 3) {
            if (f32) apply_resid<float>(C.mg.l32[0], C.mg.l32[0].c.p, C.mg.l32[0].r.p, C.s, 0);
            else apply_resid<double>(C.mg.l64[0], C.mg.l64[0].c.p, C.mg.l64[0].r.p, C.s, 0);
        } else if (which == 5) {
            LSG_REQUIRE(C.mg.L >= 2, LSG_ERR_STATE, "no smoothed coarse level");
            if (f32) apply_resid<float>(C.mg.l32[1], C.mg.l32[1].c.p, C.mg.l32[1].r.p, C.s, 0);
            else apply_resid<double>(C.mg.l64[1], C.mg.l64[1].c.p, C.mg.l64[1].r.p, C.s, 0);
        } else if (which == 4) {
            krylov7<double, 0>(C, C.Z.p, C.V.p, C.w.p, C.scal.p + 48);
        } else if (which == 6) {
            LSG_REQUIRE(f32 && C.Z32.p, LSG_ERR_STATE, "needs the FP32 multigrid");
            krylov7<float, 0>(C, C.Z32.p, C.V.p, C.w.p, C.scal.p + 48);
        } else if (which == 8) {
            LSG_REQUIRE(f32 && C.Z32.p, LSG_ERR_STATE, "needs the FP32 multigrid");
            const Dims& d = C.d;
            const long long gx = (d.N + 31) / 32, gy = (d.M + 7) / 8;
            LSG_REQUIRE(gx * gy <= 4096, LSG_ERR_STATE, "grid too wide for the z-marching kernel");
            int zc = zchunk_for(n);
            while (gx * gy * ((d.K + zc - 1) / zc) > 4096) zc *= 2;
            const dim3 grid((unsigned)gx, (unsigned)gy, (unsigned)((d.K + zc - 1) / zc));
            k_krylov7z<float, 0><<<grid, dim3(32, 8), 0, C.s>>>(d.N, d.M, d.K, zc, C.cls0.p, C.dict0.p, C.Z32.p,
                                                                  C.V.p, C.w.p, C.red.partial.p, C.red.counter.p,
                                                                  C.scal.p + 48);
            LSG_CHECK_LAUNCH();
        } else if (which == 7) {
            LSG_REQUIRE(f32 && C.Z32.p, LSG_ERR_STATE, "needs the FP32 multigrid");
            const Dims& d = C.d;
            k_spmv_dot7<float><<<grid_for(n, 256, Reducer::kMaxBlocks), 256, 0, C.s>>>(
                d.N, d.M, d.K, C.cls0.p, C.dict0.p, C.Z32.p, C.V.p, C.w.p, C.red.partial.p, C.red.counter.p,
                C.scal.p + 48);
            LSG_CHECK_LAUNCH();
        } else if (which >= 14 && which <= 17) {
            // the reference-schedule y/z line solve with the segment maps walked
            // (14/15) or with 4-cell segments (16/17)
            const int form = which <= 15 ? 1 : 2;
            const int d = 1 + (which - 14) % 2;
            if (f32) line_solve<float>(C.mg.l32[0], d, C.opt.zline_reference != 0, (float)C.opt.omega, C.s,
                                       nullptr, form);
            else line_solve<double>(C.mg.l64[0], d, C.opt.zline_reference != 0, C.opt.omega, C.s, nullptr, form);
        } else if (which == 18 || which == 19) {
            // the first coarse level's residual update with 8 / 16 z-planes per thread
            LSG_REQUIRE(C.mg.L >= 2, LSG_ERR_STATE, "no smoothed coarse level");
            const int zc = which == 18 ? 8 : 16;
            if (f32) apply_resid<float>(C.mg.l32[1], C.mg.l32[1].c.p, C.mg.l32[1].r.p, C.s, 0, zc);
            else apply_resid<double>(C.mg.l64[1], C.mg.l64[1].c.p, C.mg.l64[1].r.p, C.s, 0, zc);
        } else if (which >= 9 && which <= 13) {
            // 9/10/11: the solve's x/y/z steps; 12/13: y/z with the segment maps
            // walked by each thread instead of scanned
            const int d = which <= 11 ? which - 9 : which - 11;
            const bool scan = which <= 11;
            const bool zq = C.opt.zline_reference != 0;
            if (f32) {
                const LevelT<float>& lv = C.mg.l32[0];
                LSG_REQUIRE(adlj_fused_level<float>(lv.d, lv.ol.n, lv.off, C.opt), LSG_ERR_STATE,
                            "the finest level does not run the fused ADLJ steps");
                adlj_fused_step<float>(lv, d, zq, (float)C.opt.omega, C.s, lv.ch.p, lv.c.p, scan);
            } else {
                const LevelT<double>& lv = C.mg.l64[0];
                LSG_REQUIRE(adlj_fused_level<double>(lv.d, lv.ol.n, lv.off, C.opt), LSG_ERR_STATE,
                            "the finest level does not run the fused ADLJ steps");
                adlj_fused_step<double>(lv, d, zq, C.opt.omega, C.s, lv.ch.p, lv.c.p, scan);
            }
        } else {
            throw Error{LSG_ERR_ARG, "unknown kernel id"};
        }
    };
    double bytes;
    if (which >= 14 && which <= 17) bytes = 7.0 * w * n;
    else if (which == 18 || which == 19) bytes = (3.0 * w + 4.0) * (double)C.mg.dims[1].n();
    else if (which >= 9) bytes = (4.0 * w + 4.0) * n; // b, iterate, dinv read; iterate written; row class
    else if (which <= 2) bytes = 7.0 * w * n;         // r, lo, dinv, up, ch read; c, ch written
    else if (which == 3) bytes = (3.0 * w + 4.0) * n; // c, r read/write, row class
    else if (which == 5) bytes = (3.0 * w + 4.0) * (double)C.mg.dims[1].n();
    else if (which >= 6) bytes = (4.0 + 8.0 + 8.0 + 4.0) * n;   // FP32 z, v0 read, w written, row class
    else bytes = (3.0 * 8.0 + 4.0) * n;               // z, v0 read, w written, row class
    // defined inputs for the timed launches
    if (which == 5 || which == 18 || which == 19) {
        const long long n1 = C.mg.dims[1].n();
        if (f32) {
            LSG_CUDA(cudaMemsetAsync(C.mg.l32[1].r.p, 0, n1 * 4, C.s));
            LSG_CUDA(cudaMemsetAsync(C.mg.l32[1].c.p, 0, n1 * 4, C.s));
        } else {
            LSG_CUDA(cudaMemsetAsync(C.mg.l64[1].r.p, 0, n1 * 8, C.s));
            LSG_CUDA(cudaMemsetAsync(C.mg.l64[1].c.p, 0, n1 * 8, C.s));
        }
    }
    if (f32) {
        LSG_CUDA(cudaMemsetAsync(C.mg.l32[0].r.p, 0, n * 4, C.s));
        LSG_CUDA(cudaMemsetAsync(C.mg.l32[0].c.p, 0, n * 4, C.s));
        LSG_CUDA(cudaMemsetAsync(C.mg.l32[0].ch.p, 0, n * 4, C.s));
    } else {
        LSG_CUDA(cudaMemsetAsync(C.mg.l64[0].r.p, 0, n * 8, C.s));
        LSG_CUDA(cudaMemsetAsync(C.mg.l64[0].c.p, 0, n * 8, C.s));
        LSG_CUDA(cudaMemsetAsync(C.mg.l64[0].ch.p, 0, n * 8, C.s));
    }
    if (which == 4) {
        LSG_CUDA(cudaMemsetAsync(C.Z.p, 0, n * 8, C.s));
        LSG_CUDA(cudaMemsetAsync(C.V.p, 0, n * 8, C.s));
    }
    if (which >= 6 && which <= 8) {
        LSG_CUDA(cudaMemsetAsync(C.Z32.p, 0, n * 4, C.s));
        LSG_CUDA(cudaMemsetAsync(C.V.p, 0, n * 8, C.s));
    }
    launch();
    LSG_CUDA(cudaEventRecord(C.ev0, C.s));
    for (int r = 0; r < reps; r++) launch();
    LSG_CUDA(cudaEventRecord(C.ev1, C.s));
    LSG_CUDA(cudaEventSynchronize(C.ev1));
    float ms = 0;
    LSG_CUDA(cudaEventElapsedTime(&ms, C.ev0, C.ev1));
    *ms_per_launch = ms / reps;
    *bytes_per_launch = bytes;
    return LSG_OK;
    LSG_API_END(h)
}


// ---------------------------------------------------------------------------
// cut-cell loads (LoadsCalculator, Base/loads_calculator.h)
// ---------------------------------------------------------------------------
int lsg_loads_set(lsg_ctx* h, int N, int M, int K, int count, const int* cells, const int* celltype,
                  const double* theta, const double* delta, const double* inv_vof, const double* delta_ib_max,
                  const double* inv_delta_ib_ne, const double* inv_delta_ib_tn, const double* nodes,
                  const double* center, double fcoef, double dt)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(N >= 3 && M >= 3 && K >= 3, LSG_ERR_ARG, "grid must be at least 3 cells in every direction");
    LSG_REQUIRE((long long)N * M * K < (1LL << 31), LSG_ERR_ARG, "grid too large for 32-bit cell indices");
    LSG_REQUIRE(count >= 0, LSG_ERR_ARG, "negative cut-cell count");
    LSG_REQUIRE(center && (count == 0 || (cells && celltype && theta && delta && inv_vof && delta_ib_max &&
                                          inv_delta_ib_ne && inv_delta_ib_tn && nodes)),
                LSG_ERR_ARG, "null argument");
    LSG_REQUIRE(dt > 0, LSG_ERR_ARG, "time step must be positive (moment filter)");
    LSG_CUDA(cudaSetDevice(C.device));
    using namespace loads_desc;
    const int NM = N * M;
    const long long n = (long long)NM * K;
    std::vector<double> g((size_t)LF_COUNT * count);
    std::vector<int> idx(3 * (size_t)count);
    std::vector<unsigned long long> desc(count, 0ull);
    auto put = [&](int f, int i, double v) { g[(size_t)f * count + i] = v; };
    for (int i = 0; i < count; i++) {
        const int num = cells[i];
        LSG_REQUIRE(num >= 0 && num < n, LSG_ERR_ARG, "cut cell index outside the grid");
        const int k = num / NM, j = (num - k * NM) / N, x = num - k * NM - j * N;
        LSG_REQUIRE(x >= 1 && x <= N - 2 && j >= 1 && j <= M - 2 && k >= 1 && k <= K - 2, LSG_ERR_ARG,
                    "cut cell on the outer layer of the grid (its loads read the neighbours on both sides)");
        idx[i] = num;
        idx[count + i] = num - j - k * M;      // x-grid index (BaseTaskDescription::addCutCell)
        idx[2 * count + i] = num - k * N;      // y-grid index
        const double* t = theta + 3 * (size_t)num;
        put(LF_TX, i, t[0]);
        put(LF_TY, i, t[1]);
        put(LF_TZ, i, t[2]);
        put(LF_TXX, i, theta[3 * (size_t)(num - 1)]);
        put(LF_TYY, i, theta[3 * (size_t)(num - N) + 1]);
        put(LF_TZZ, i, theta[3 * (size_t)(num - NM) + 2]);
        for (int c = 0; c < 3; c++) {
            put(LF_DX + c, i, delta[3 * (size_t)num + c]);
            put(LF_S0 + c, i, delta_ib_max[3 * (size_t)num + c]);
            put(LF_NX + c, i, nodes[3 * (size_t)num + c]);
        }
        put(LF_VV, i, inv_vof[num]);
        const uint8_t* sl = find(celltype[num]);
        unsigned long long dsc = 0;
        for (int s = 0; s < 6; s++) {
            const unsigned b = sl ? sl[s] : 0u;
            double dh = 0.0, db = 0.0;
            if (b & Q) {
                const int c = vel_of(s);
                const int step = c == 0 ? 1 : (c == 1 ? N : NM);
                const double* D = (b & TN) ? inv_delta_ib_tn : inv_delta_ib_ne;
                dh = D[3 * (size_t)num + dist_of(s)];
                db = (b & DHERE) ? dh : D[3 * (size_t)(num - step) + dist_of(s)];
            }
            put(LF_D + 2 * s, i, dh);
            put(LF_D + 2 * s + 1, i, db);
            dsc |= (unsigned long long)b << (8 * s);
        }
        desc[i] = dsc;
    }
    Context::Loads& L = C.loads;
    L.have = false;
    L.N = N;
    L.M = M;
    L.K = K;
    L.count = count;
    if (count > 0) {
        L.g.alloc(g.size());
        L.idx.alloc(idx.size());
        L.desc.alloc(desc.size());
        LSG_CUDA(cudaMemcpyAsync(L.g.p, g.data(), g.size() * 8, cudaMemcpyHostToDevice, C.s));
        LSG_CUDA(cudaMemcpyAsync(L.idx.p, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice, C.s));
        LSG_CUDA(cudaMemcpyAsync(L.desc.p, desc.data(), desc.size() * 8, cudaMemcpyHostToDevice, C.s));
    }
    L.partial.alloc(1024 * 6);
    L.sums.alloc(8);
    if (!L.counter.p) {
        L.counter.alloc(1);
        LSG_CUDA(cudaMemsetAsync(L.counter.p, 0, sizeof(unsigned int), C.s));
    }
    for (int c = 0; c < 3; c++) {
        L.center[c] = center[c];
        L.filt[c].init(dt);
    }
    L.fcoef = fcoef;
    LSG_CUDA(cudaStreamSynchronize(C.s));
    L.have = true;
    return LSG_OK;
    LSG_API_END(h)
}

static void loads_run(Context& C, const double* ux, const double* uy, const double* uz, const double* p,
                      const double* vib, const double* vib_yx, const double* vib_zy, const double* nu_cell,
                      double nu, double* fx, double* fy, double* fz, lsg_loads_result* out)
{
    Context::Loads& L = C.loads;
    memset(out, 0, sizeof(*out));
    out->count = L.count;
    if (L.count == 0) return;     // calculate() leaves everything untouched without cut cells
    LoadsArgs a;
    a.count = L.count;
    a.N = L.N;
    a.NM = L.N * L.M;
    a.g = L.g.p;
    a.idx = L.idx.p;
    a.desc = L.desc.p;
    a.ux = ux;
    a.uy = uy;
    a.uz = uz;
    a.p = p;
    a.vib = vib;
    a.vyx = vib_yx;
    a.vzy = vib_zy;
    a.nu_cell = nu_cell;
    a.nu = nu;
    a.cx = L.center[0];
    a.cy = L.center[1];
    a.cz = L.center[2];
    a.fx = fx;
    a.fy = fy;
    a.fz = fz;
    a.partial = L.partial.p;
    a.counter = L.counter.p;
    a.sums = L.sums.p;
    const int grid = grid_for(L.count, 256, 1024);
    k_loads<<<grid, 256, 0, C.s>>>(a);
    LSG_CHECK_LAUNCH();
    double s[6];
    LSG_CUDA(cudaMemcpyAsync(s, L.sums.p, sizeof(s), cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    for (int c = 0; c < 3; c++) {
        out->force[c] = s[c];
        out->coef[c] = s[c] * L.fcoef;
        out->moment_raw[c] = s[3 + c];
        out->moment[c] = L.filt[c].step(s[3 + c]);
    }
}

int lsg_loads_calculate_device(lsg_ctx* h, const double* ux, const double* uy, const double* uz, const double* p,
                               const double* vib, const double* vib_yx, const double* vib_zy,
                               const double* nu_cell, double nu, double* forces, lsg_loads_result* out)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.loads.have, LSG_ERR_STATE, "no cut-cell list set (lsg_loads_set)");
    LSG_REQUIRE(ux && uy && uz && p && vib && vib_yx && vib_zy && out, LSG_ERR_ARG, "null argument");
    LSG_CUDA(cudaSetDevice(C.device));
    const int cnt = C.loads.count;
    loads_run(C, ux, uy, uz, p, vib, vib_yx, vib_zy, nu_cell, nu, forces, forces ? forces + cnt : nullptr,
              forces ? forces + 2 * (size_t)cnt : nullptr, out);
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_loads_calculate(lsg_ctx* h, const double* ux, const double* uy, const double* uz, const double* p,
                        const double* vib, const double* vib_yx, const double* vib_zy, const double* nu_cell,
                        double nu, double* forces, lsg_loads_result* out)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    Context::Loads& L = C.loads;
    LSG_REQUIRE(L.have, LSG_ERR_STATE, "no cut-cell list set (lsg_loads_set)");
    LSG_REQUIRE(ux && uy && uz && p && vib && vib_yx && vib_zy && out, LSG_ERR_ARG, "null argument");
    LSG_CUDA(cudaSetDevice(C.device));
    const long long N = L.N, M = L.M, K = L.K, n = N * M * K;
    const long long nx = (N - 1) * M * K, ny = N * (M - 1) * K, nz = N * M * (K - 1);
    TmpBuf<double> du(C.s, C.pool), dv(C.s, C.pool), dw(C.s, C.pool), dp(C.s, C.pool), dvib(C.s, C.pool), dyx(C.s, C.pool), dzy(C.s, C.pool), dnu(C.s, C.pool), df(C.s, C.pool);
    du.alloc(nx);
    dv.alloc(ny);
    dw.alloc(nz);
    dp.alloc(n);
    dvib.alloc(3 * n);
    dyx.alloc(3 * n);
    dzy.alloc(3 * n);
    LSG_CUDA(cudaMemcpyAsync(du.p, ux, nx * 8, cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(dv.p, uy, ny * 8, cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(dw.p, uz, nz * 8, cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(dp.p, p, n * 8, cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(dvib.p, vib, 3 * n * 8, cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(dyx.p, vib_yx, 3 * n * 8, cudaMemcpyHostToDevice, C.s));
    LSG_CUDA(cudaMemcpyAsync(dzy.p, vib_zy, 3 * n * 8, cudaMemcpyHostToDevice, C.s));
    if (nu_cell) {
        dnu.alloc(n);
        LSG_CUDA(cudaMemcpyAsync(dnu.p, nu_cell, n * 8, cudaMemcpyHostToDevice, C.s));
    }
    const size_t cnt = (size_t)L.count;
    if (forces && cnt) df.alloc(3 * cnt);
    loads_run(C, du.p, dv.p, dw.p, dp.p, dvib.p, dyx.p, dzy.p, nu_cell ? dnu.p : nullptr, nu, df.p,
              df.p ? df.p + cnt : nullptr, df.p ? df.p + 2 * cnt : nullptr, out);
    if (forces && cnt) {
        LSG_CUDA(cudaMemcpyAsync(forces, df.p, 3 * cnt * 8, cudaMemcpyDeviceToHost, C.s));
        LSG_CUDA(cudaStreamSynchronize(C.s));
    }
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_loads_reset_filter(lsg_ctx* h, double dt)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    LSG_REQUIRE(dt > 0, LSG_ERR_ARG, "time step must be positive");
    for (int c = 0; c < 3; c++) h->c.loads.filt[c].init(dt);
    return LSG_OK;
    LSG_API_END(h)
}

static void loads_adjoint_run(Context& C, const double* w, const double* nu_cell, double nu, double* gux,
                              double* guy, double* guz, double* gp)
{
    Context::Loads& L = C.loads;
    const long long N = L.N, M = L.M, K = L.K, n = N * M * K;
    LSG_CUDA(cudaMemsetAsync(gux, 0, (N - 1) * M * K * 8, C.s));
    LSG_CUDA(cudaMemsetAsync(guy, 0, N * (M - 1) * K * 8, C.s));
    LSG_CUDA(cudaMemsetAsync(guz, 0, N * M * (K - 1) * 8, C.s));
    LSG_CUDA(cudaMemsetAsync(gp, 0, n * 8, C.s));
    if (L.count == 0) return;
    LoadsAdjArgs a;
    a.count = L.count;
    a.N = L.N;
    a.NM = L.N * L.M;
    a.g = L.g.p;
    a.idx = L.idx.p;
    a.desc = L.desc.p;
    a.nu_cell = nu_cell;
    a.nu = nu;
    for (int c = 0; c < 3; c++) a.w[c] = w[c];
    a.gux = gux;
    a.guy = guy;
    a.guz = guz;
    a.gp = gp;
    k_loads_adjoint<<<grid_for(L.count, 256, 1024), 256, 0, C.s>>>(a);
    LSG_CHECK_LAUNCH();
}

int lsg_loads_adjoint_device(lsg_ctx* h, const double* weight, const double* nu_cell, double nu, double* g_ux,
                             double* g_uy, double* g_uz, double* g_p)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    LSG_REQUIRE(C.loads.have, LSG_ERR_STATE, "no cut-cell list set (lsg_loads_set)");
    LSG_REQUIRE(weight && g_ux && g_uy && g_uz && g_p, LSG_ERR_ARG, "null argument");
    LSG_CUDA(cudaSetDevice(C.device));
    loads_adjoint_run(C, weight, nu_cell, nu, g_ux, g_uy, g_uz, g_p);
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

int lsg_loads_adjoint(lsg_ctx* h, const double* weight, const double* nu_cell, double nu, double* g_ux,
                      double* g_uy, double* g_uz, double* g_p)
{
    if (!h) return LSG_ERR_ARG;
    LSG_API_BEGIN
    Context& C = h->c;
    Context::Loads& L = C.loads;
    LSG_REQUIRE(L.have, LSG_ERR_STATE, "no cut-cell list set (lsg_loads_set)");
    LSG_REQUIRE(weight && g_ux && g_uy && g_uz && g_p, LSG_ERR_ARG, "null argument");
    LSG_CUDA(cudaSetDevice(C.device));
    const long long N = L.N, M = L.M, K = L.K, n = N * M * K;
    const long long nx = (N - 1) * M * K, ny = N * (M - 1) * K, nz = N * M * (K - 1);
    TmpBuf<double> gx(C.s, C.pool), gy(C.s, C.pool), gz(C.s, C.pool), gpd(C.s, C.pool), dnu(C.s, C.pool);
    gx.alloc(nx);
    gy.alloc(ny);
    gz.alloc(nz);
    gpd.alloc(n);
    if (nu_cell) {
        dnu.alloc(n);
        LSG_CUDA(cudaMemcpyAsync(dnu.p, nu_cell, n * 8, cudaMemcpyHostToDevice, C.s));
    }
    loads_adjoint_run(C, weight, nu_cell ? dnu.p : nullptr, nu, gx.p, gy.p, gz.p, gpd.p);
    LSG_CUDA(cudaMemcpyAsync(g_ux, gx.p, nx * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaMemcpyAsync(g_uy, gy.p, ny * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaMemcpyAsync(g_uz, gz.p, nz * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaMemcpyAsync(g_p, gpd.p, n * 8, cudaMemcpyDeviceToHost, C.s));
    LSG_CUDA(cudaStreamSynchronize(C.s));
    return LSG_OK;
    LSG_API_END(h)
}

}  // extern "C"
