/*
 * lsstag_b200_adapter.hpp -- reference-side adapter: the B200 solver behind
 * LS-STAG-3D's own solver interface.
 *
 * Include this header inside the reference tree (after its
 * Base/Solvers/iterative_solver_interface.h) and add one branch to the
 * solver ladder of PoissonDiscreteEquation
 * (DiscreteEquations/poisson_discrete_equation.h:167-209):
 *
 *     #if defined(LS_STAG_USE_B200)
 *         B200MGFGMRES solver;
 *     #elif defined(LS_STAG_USE_CUDA)
 *         ...the reference's ladder unchanged...
 *
 * B200MGFGMRES implements IterativeSolverInterface
 * (Base/Solvers/iterative_solver_interface.h:31-73) over the C ABI of
 * include/lsstag_b200.h:
 *   set()                     lsg_set_matrix_csr (the equation's own CSR,
 *                             SparseMatrix Number/Portrait/Cell) + lsg_setup
 *                             (MG hierarchy), as MGFGMRES::set
 *                             (mg_fgmres.h:40-52) builds its multigrid;
 *   rebuildPreconditioner()   the operator again + lsg_setup (mg_fgmres.h:40-44);
 *   solve()                   lsg_solve on the equation's right-hand side and
 *                             solution arrays (updated in place), sets the
 *                             public it / norm_r the time step logs
 *                             (time_stepping_method_interface.h:205-206).
 * The reference's CPU build passes host arrays; its CUDA build keeps the CSR
 * and the vectors in device memory (Base/MeshFunctions/array.h), for which
 * the *_device entry points are used (LS_STAG_USE_CUDA).
 *
 * B200ILUBiCGStab is the same with BiCGStab + ILU(0) (ilu_bicgstab.h:33-64).
 *
 * Differences a maintainer sees: errors throw std::runtime_error with the
 * library's message (the reference aborts or runs on silently); a capped
 * solve sets status() to LSG_NOT_CONVERGED (the reference returns the count
 * silently); with mg_precision = LSG_FP32 the FP32 multigrid runs inside
 * FP64 FGMRES and the solve stops only once the FP64 true residual meets eps.
 */
#ifndef LSSTAG_B200_ADAPTER_HPP
#define LSSTAG_B200_ADAPTER_HPP

#include <stdexcept>
#include <string>

#include "lsstag_b200.h"

namespace LS_STAG {

template <int Method, int Precond>
struct B200Solver : IterativeSolverInterface {
    B200Solver() { lsg_default_options(&opt_); }
    ~B200Solver() override
    {
        if (ctx_) lsg_destroy(ctx_);
    }
    B200Solver(const B200Solver&) = delete;
    B200Solver& operator=(const B200Solver&) = delete;

    /* multigrid arithmetic: LSG_FP64 (the reference's) or LSG_FP32 */
    int mg_precision = LSG_FP64;
    /* CUDA device of the context */
    int device = 0;

    void set(SparseMatrix* A, double* b, double* x, BaseTaskDescription* task) override
    {
        IterativeSolverInterface::set(A, b, x, task);   // m_A, m_rightM, m_sol, eps, max_it, NM
        if (!ctx_ && lsg_create(device, &ctx_) != LSG_OK) throw std::runtime_error("lsg_create failed");
        lsg_default_options(&opt_);
        opt_.method = Method;
        opt_.precond = Precond;
        opt_.mg_precision = mg_precision;
        opt_.restart = (Method == LSG_METHOD_FGMRES) ? task->FGMRES_RESTART_NUM : opt_.restart;
        opt_.max_it = task->MAX_ITER;
        opt_.n_post = task->n_post;
        opt_.eps = eps;
        upload();
        check(lsg_setup(ctx_, &opt_));
    }
    void rebuildPreconditioner() override
    {
        upload();
        check(lsg_setup(ctx_, &opt_));
    }
    int solve() override
    {
        if (opt_.eps != eps) {          // the equation may set eps between solves
            opt_.eps = eps;
            check(lsg_setup(ctx_, &opt_));
        }
        lsg_stats st;
#ifdef LS_STAG_USE_CUDA
        const int rc = lsg_solve_device(ctx_, m_rightM, m_sol, &st);
#else
        const int rc = lsg_solve(ctx_, m_rightM, m_sol, &st);
#endif
        check(rc);
        it = st.iterations;
        norm_r = st.norm_r;
        status_ = st.status;
        return it;
    }
    /* LSG_OK, LSG_NOT_CONVERGED or LSG_BREAKDOWN of the last solve */
    int status() const { return status_; }

  private:
    void upload()
    {
#ifdef LS_STAG_USE_CUDA
        check(lsg_set_matrix_csr_device(ctx_, m_A->m_N, m_A->m_M, m_A->m_K, m_A->Number, m_A->Portrait, m_A->Cell,
                                        m_A->elemCount));
#else
        check(lsg_set_matrix_csr(ctx_, m_A->m_N, m_A->m_M, m_A->m_K, m_A->Number, m_A->Portrait, m_A->Cell));
#endif
    }
    void check(int rc) const
    {
        if (rc < 0) throw std::runtime_error(std::string("lsstag_b200: ") + lsg_last_error(ctx_));
    }
    lsg_ctx* ctx_ = nullptr;
    lsg_options opt_;
    int status_ = LSG_OK;
};

using B200MGFGMRES = B200Solver<LSG_METHOD_FGMRES, LSG_PC_MG>;
using B200ILUBiCGStab = B200Solver<LSG_METHOD_BICGSTAB, LSG_PC_ILU0>;

}  // namespace LS_STAG

#endif /* LSSTAG_B200_ADAPTER_HPP */
