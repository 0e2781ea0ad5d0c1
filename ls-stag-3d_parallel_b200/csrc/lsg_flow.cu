// Native fixed-body flow time step over the library's own entry points: the
// counterpart of TimeSteppingMethodInterface::step
// (TimeSteppingMethod/time_stepping_method_interface.h:180-214) for a flow
// past bodies that do not move, in the reference's order:
//   1. the pressure operator's source term from the current x-velocity
//      (LaplaceDiscreteOperator::calcFlux);
//   2. per momentum component: the convective operator of the current
//      velocities with its source term, the right-hand side with the
//      Adams-Bashforth history (HelmholtzDiscreteEquation::recalcRightMember),
//      and the ILU(0)-FGMRES solve started from the current velocity; the
//      three solves are independent and run concurrently, one host thread
//      and one context (stream) each;
//   3. b = D u* + flux and the pressure MG-FGMRES solve from 0
//      (PoissonDiscreteEquation), optionally to a tolerance relative to ||b||;
//   4. the projection (SetSolutions::correction) and the buffer rotation.
// The state lives in device memory owned by the stepper; every step's work
// is device work issued through the public entry points (each ends with its
// stream synchronised, which orders the phases across contexts).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <utility>

#include "../../include/lsstag_b200.h"

namespace {

struct Buf {
    double* p = nullptr;
    size_t n = 0;
    ~Buf() { if (p) cudaFree(p); }
    bool alloc(size_t count)
    {
        n = count;
        return cudaMalloc(&p, count * sizeof(double)) == cudaSuccess;
    }
};

// ||x||_2 of a device vector: per-block partial sums, then one block adds
// them in block order (deterministic).
__global__ void k_sumsq(long long n, const double* __restrict__ x, double* partial)
{
    __shared__ double sh[256];
    double s = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        s += x[i] * x[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

__global__ void k_sum_partials(int nb, const double* __restrict__ partial, double* out)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int b = 0; b < nb; b++) s += partial[b];
        *out = s;
    }
}

constexpr int kNormBlocks = 592;   // 4 x 148 SMs

}  // namespace

struct lsg_flow {
    lsg_flow_desc d{};
    std::string err;
    long long n = 0, ns[3] = {0, 0, 0};
    int* side_type = nullptr;
    Buf vib, u_w, theta, delta, vof[3], hflux[3];
    Buf u[3], uprev[3], unew[3], us[3], p, prev_aux[3], aux[3], gp[3], conv[3], flux2[3], right[3];
    Buf flux_lap, b, phi, partial;
    cudaStream_t s = nullptr;
    bool have_state = false;
    ~lsg_flow()
    {
        if (side_type) cudaFree(side_type);
        if (s) cudaStreamDestroy(s);
    }
};

namespace {

int fail(lsg_flow* f, int code, const std::string& what)
{
    if (f) f->err = what;
    return code;
}

// Status of an entry point call on context c; the context's message is kept.
int check(lsg_flow* f, lsg_ctx* c, int rc, const char* what)
{
    if (rc < 0) return fail(f, rc, std::string(what) + ": " + lsg_last_error(c));
    return rc;
}

bool copy_in(Buf& dst, const double* src, size_t n, cudaStream_t s)
{
    if (!dst.alloc(n)) return false;
    return cudaMemcpyAsync(dst.p, src, n * sizeof(double), cudaMemcpyDefault, s) == cudaSuccess;
}

}  // namespace

extern "C" {

int lsg_flow_create(const lsg_flow_desc* d, lsg_flow** out)
{
    if (!d || !out) return LSG_ERR_ARG;
    *out = nullptr;
    if (d->N < 2 || d->M < 2 || d->K < 2 || !d->pres || !d->psolve || !d->mom[0] || !d->mom[1] || !d->mom[2])
        return LSG_ERR_ARG;
    if (!d->side_type || !d->vib || !d->u_w || !d->theta || !d->delta) return LSG_ERR_ARG;
    for (int k = 0; k < 3; k++)
        if (!d->vof[k] || !d->hflux[k]) return LSG_ERR_ARG;
    if (!(d->p_rel_tol >= 0.0)) return LSG_ERR_ARG;
    lsg_flow* f = new (std::nothrow) lsg_flow;
    if (!f) return LSG_ERR_NOMEM;
    f->d = *d;
    const long long N = d->N, M = d->M, K = d->K;
    f->n = N * M * K;
    f->ns[0] = (N - 1) * M * K;
    f->ns[1] = N * (M - 1) * K;
    f->ns[2] = N * M * (K - 1);
    if (d->device >= 0 && cudaSetDevice(d->device) != cudaSuccess) {
        delete f;
        return LSG_ERR_CUDA;
    }
    bool ok = cudaStreamCreateWithFlags(&f->s, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && cudaMalloc(&f->side_type, 3 * (size_t)f->n * sizeof(int)) == cudaSuccess &&
         cudaMemcpyAsync(f->side_type, d->side_type, 3 * (size_t)f->n * sizeof(int), cudaMemcpyDefault, f->s) ==
             cudaSuccess;
    ok = ok && copy_in(f->vib, d->vib, 3 * (size_t)f->n, f->s) && copy_in(f->u_w, d->u_w, (size_t)M * K, f->s) &&
         copy_in(f->theta, d->theta, 3 * (size_t)f->n, f->s) && copy_in(f->delta, d->delta, 3 * (size_t)f->n, f->s);
    for (int k = 0; k < 3 && ok; k++) {
        const size_t m = (size_t)f->ns[k];
        ok = copy_in(f->vof[k], d->vof[k], m, f->s) && copy_in(f->hflux[k], d->hflux[k], m, f->s);
        for (Buf* b : {&f->u[k], &f->uprev[k], &f->unew[k], &f->us[k], &f->prev_aux[k], &f->aux[k], &f->gp[k],
                       &f->conv[k], &f->flux2[k], &f->right[k]})
            ok = ok && b->alloc(m);
    }
    ok = ok && f->p.alloc(f->n) && f->flux_lap.alloc(f->n) && f->b.alloc(f->n) && f->phi.alloc(f->n) &&
         f->partial.alloc(kNormBlocks + 1);
    ok = ok && cudaStreamSynchronize(f->s) == cudaSuccess;
    if (!ok) {
        delete f;
        return LSG_ERR_NOMEM;
    }
    *out = f;
    return LSG_OK;
}

int lsg_flow_destroy(lsg_flow* f)
{
    delete f;
    return LSG_OK;
}

const char* lsg_flow_last_error(const lsg_flow* f) { return f ? f->err.c_str() : "null flow"; }

int lsg_flow_set_state(lsg_flow* f, const double* const u[3], const double* const uprev[3], const double* p,
                       const double* const prev_aux[3])
{
    if (!f || !u || !uprev || !p) return LSG_ERR_ARG;
    const lsg_flow_desc& d = f->d;
    for (int k = 0; k < 3; k++) {
        const size_t bytes = (size_t)f->ns[k] * sizeof(double);
        if (!u[k] || !uprev[k]) return fail(f, LSG_ERR_ARG, "null velocity");
        if (cudaMemcpyAsync(f->u[k].p, u[k], bytes, cudaMemcpyDefault, f->s) != cudaSuccess ||
            cudaMemcpyAsync(f->uprev[k].p, uprev[k], bytes, cudaMemcpyDefault, f->s) != cudaSuccess)
            return fail(f, LSG_ERR_CUDA, "state copy");
    }
    if (cudaMemcpyAsync(f->p.p, p, (size_t)f->n * sizeof(double), cudaMemcpyDefault, f->s) != cudaSuccess ||
        cudaStreamSynchronize(f->s) != cudaSuccess)
        return fail(f, LSG_ERR_CUDA, "state copy");
    if (prev_aux) {
        for (int k = 0; k < 3; k++) {
            if (!prev_aux[k]) return fail(f, LSG_ERR_ARG, "null history");
            if (cudaMemcpyAsync(f->prev_aux[k].p, prev_aux[k], (size_t)f->ns[k] * sizeof(double), cudaMemcpyDefault,
                                f->s) != cudaSuccess)
                return fail(f, LSG_ERR_CUDA, "state copy");
        }
        if (cudaStreamSynchronize(f->s) != cudaSuccess) return fail(f, LSG_ERR_CUDA, "state copy");
    } else {
        // HelmholtzDiscreteEquation::set: history = flux2 + C(u) u of the state
        for (int k = 0; k < 3; k++) {
            int rc = check(f, d.mom[k],
                           lsg_convective_flux_device(d.mom[k], k, d.N, d.M, d.K, f->theta.p, f->delta.p, f->u[0].p,
                                                      f->u[1].p, f->u[2].p, f->u_w.p, d.bc, f->flux2[k].p),
                           "convective source term");
            if (rc < 0) return rc;
            rc = check(f, d.pres,
                       lsg_convective_apply_device(d.pres, k, f->u[0].p, f->u[1].p, f->u[2].p, f->u[k].p,
                                                   f->flux2[k].p, f->prev_aux[k].p, d.zconv_reference),
                       "convective operator");
            if (rc < 0) return rc;
        }
    }
    f->have_state = true;
    return LSG_OK;
}

int lsg_flow_step(lsg_flow* f, int its[4])
{
    if (!f) return LSG_ERR_ARG;
    if (!f->have_state) return fail(f, LSG_ERR_STATE, "lsg_flow_set_state must be called before lsg_flow_step");
    const lsg_flow_desc& d = f->d;
    int rc = check(f, d.pres,
                   lsg_laplace_flux_device(d.pres, f->side_type, f->vib.p, f->u_w.p, d.bc_lap, f->u[0].p,
                                           f->flux_lap.p),
                   "pressure source term");
    if (rc < 0) return rc;
    for (int k = 0; k < 3; k++) {
        rc = check(f, d.mom[k],
                   lsg_convective_flux_device(d.mom[k], k, d.N, d.M, d.K, f->theta.p, f->delta.p, f->u[0].p,
                                              f->u[1].p, f->u[2].p, f->u_w.p, d.bc, f->flux2[k].p),
                   "convective source term");
        if (rc < 0) return rc;
        rc = check(f, d.pres,
                   lsg_convective_apply_device(d.pres, k, f->u[0].p, f->u[1].p, f->u[2].p, f->u[k].p, f->flux2[k].p,
                                               f->conv[k].p, d.zconv_reference),
                   "convective operator");
        if (rc < 0) return rc;
        rc = check(f, d.pres,
                   lsg_momentum_rhs_device(d.pres, k, f->conv[k].p, f->u[k].p, f->uprev[k].p, f->vof[k].p,
                                           f->hflux[k].p, f->p.p, f->prev_aux[k].p, d.coef2, f->right[k].p,
                                           f->aux[k].p, f->gp[k].p),
                   "momentum right-hand side");
        if (rc < 0) return rc;
        std::swap(f->prev_aux[k].p, f->aux[k].p);
        if (cudaMemcpyAsync(f->us[k].p, f->u[k].p, (size_t)f->ns[k] * sizeof(double), cudaMemcpyDeviceToDevice,
                            f->s) != cudaSuccess)
            return fail(f, LSG_ERR_CUDA, "copy of the velocity");
    }
    if (cudaStreamSynchronize(f->s) != cudaSuccess) return fail(f, LSG_ERR_CUDA, "copy of the velocity");
    // the three momentum systems are independent given the current state
    lsg_stats st[4];
    std::memset(st, 0, sizeof(st));
    int mrc[3] = {0, 0, 0};
    {
        std::thread th[3];
        for (int k = 0; k < 3; k++)
            th[k] = std::thread([&, k]() { mrc[k] = lsg_solve_device(d.mom[k], f->right[k].p, f->us[k].p, &st[k]); });
        for (auto& t : th) t.join();
    }
    for (int k = 0; k < 3; k++) {
        rc = check(f, d.mom[k], mrc[k], "momentum solve");
        if (rc < 0) return rc;
    }
    rc = check(f, d.pres,
               lsg_projection_rhs_device(d.pres, f->us[0].p, f->us[1].p, f->us[2].p, f->flux_lap.p, f->b.p),
               "pressure right-hand side");
    if (rc < 0) return rc;
    if (cudaMemsetAsync(f->phi.p, 0, (size_t)f->n * sizeof(double), f->s) != cudaSuccess)
        return fail(f, LSG_ERR_CUDA, "pressure correction reset");
    if (d.p_rel_tol > 0.0) {
        k_sumsq<<<kNormBlocks, 256, 0, f->s>>>(f->n, f->b.p, f->partial.p);
        k_sum_partials<<<1, 32, 0, f->s>>>(kNormBlocks, f->partial.p, f->partial.p + kNormBlocks);
        double ss = 0.0;
        if (cudaMemcpyAsync(&ss, f->partial.p + kNormBlocks, sizeof(double), cudaMemcpyDeviceToHost, f->s) !=
                cudaSuccess ||
            cudaStreamSynchronize(f->s) != cudaSuccess)
            return fail(f, LSG_ERR_CUDA, "norm of the pressure right-hand side");
        rc = check(f, d.psolve, lsg_set_tolerance(d.psolve, d.p_rel_tol * std::sqrt(ss)), "pressure tolerance");
        if (rc < 0) return rc;
    } else if (cudaStreamSynchronize(f->s) != cudaSuccess) {
        return fail(f, LSG_ERR_CUDA, "pressure correction reset");
    }
    rc = check(f, d.psolve, lsg_solve_device(d.psolve, f->b.p, f->phi.p, &st[3]), "pressure solve");
    if (rc < 0) return rc;
    rc = check(f, d.pres,
               lsg_projection_correct_device(d.pres, f->phi.p, f->us[0].p, f->us[1].p, f->us[2].p, f->unew[0].p,
                                             f->unew[1].p, f->unew[2].p, f->p.p, d.coef, d.vbase, 1),
               "projection");
    if (rc < 0) return rc;
    // previous <- current, current <- corrected
    for (int k = 0; k < 3; k++) {
        double* t = f->uprev[k].p;
        f->uprev[k].p = f->u[k].p;
        f->u[k].p = f->unew[k].p;
        f->unew[k].p = t;
    }
    if (its)
        for (int k = 0; k < 4; k++) its[k] = st[k].iterations;
    int worst = LSG_OK;
    for (int k = 0; k < 4; k++)
        if (st[k].status != LSG_OK && worst == LSG_OK) worst = st[k].status;
    return worst;
}

int lsg_flow_state(lsg_flow* f, double* const u[3], double* p, double* const uprev[3])
{
    if (!f) return LSG_ERR_ARG;
    for (int k = 0; k < 3; k++) {
        const size_t bytes = (size_t)f->ns[k] * sizeof(double);
        if (u && u[k] && cudaMemcpyAsync(u[k], f->u[k].p, bytes, cudaMemcpyDefault, f->s) != cudaSuccess)
            return fail(f, LSG_ERR_CUDA, "state copy");
        if (uprev && uprev[k] && cudaMemcpyAsync(uprev[k], f->uprev[k].p, bytes, cudaMemcpyDefault, f->s) != cudaSuccess)
            return fail(f, LSG_ERR_CUDA, "state copy");
    }
    if (p && cudaMemcpyAsync(p, f->p.p, (size_t)f->n * sizeof(double), cudaMemcpyDefault, f->s) != cudaSuccess)
        return fail(f, LSG_ERR_CUDA, "state copy");
    if (cudaStreamSynchronize(f->s) != cudaSuccess) return fail(f, LSG_ERR_CUDA, "state copy");
    return LSG_OK;
}

}  // extern "C"
