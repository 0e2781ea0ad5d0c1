/*
 * lsstag_b200.h -- C ABI of the B200 (sm_100a) pressure-Poisson projection
 * solver for LS-STAG-3D.
 *
 * The library replaces the reference's iterative solvers for the pressure
 * correction system: the drop-in point is the reference's
 *     IterativeSolverInterface::set(SparseMatrix* A, double* b, double* x,
 *                                   BaseTaskDescription* task)   (Base/Solvers/iterative_solver_interface.h:46-55)
 *     IterativeSolverInterface::solve()                          (:45, FGMRES fgmres_interface.h:78-142,
 *                                                                  BiCGStab bicgstab_interface.h:76-111)
 *     IterativeSolverInterface::rebuildPreconditioner()          (:38, mg_fgmres.h:40-44, ilu_bicgstab.h:50-54)
 * An adapter class implementing that interface calls, in order,
 *     lsg_set_matrix_csr (set: the operator the equation assembled),
 *     lsg_setup          (set / rebuildPreconditioner: MG hierarchy or ILU(0)),
 *     lsg_solve          (solve: x updated in place, returns iterations).
 *
 * Conventions
 *   - cells are numbered  i + N*(j + M*k)  (x fastest), as in the reference;
 *   - the operator is given as the reference's CSR (Number/Portrait/Cell,
 *     Base/SparseMatrix/sparse_matrix.h:220-228), 32-bit indices, FP64 values;
 *     every row may hold only the cell itself and its six face neighbours;
 *   - host pointers unless the function name ends in _device;
 *   - every call returns an lsg status; 0 is success, > 0 a solver outcome,
 *     < 0 an error (lsg_last_error gives the text);
 *   - one context per device and per operator; a context is not thread safe;
 *     all work of a context runs on its own CUDA stream.
 */
#ifndef LSSTAG_B200_H
#define LSSTAG_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define LSG_OK 0
#define LSG_NOT_CONVERGED 1   /* iteration cap reached (reference: silent MAX_ITER) */
#define LSG_BREAKDOWN 2       /* zero/NaN norm met by a reduction */
#define LSG_ERR_ARG (-1)
#define LSG_ERR_CUDA (-2)
#define LSG_ERR_NOMEM (-3)
#define LSG_ERR_STATE (-4)    /* call order violated (e.g. solve before setup) */
#define LSG_ERR_PATTERN (-5)  /* operator entry outside the 7-point stencil */
#define LSG_ERR_SINGULAR (-6)

/* lsg_options.method */
#define LSG_METHOD_FGMRES 0
#define LSG_METHOD_BICGSTAB 1
/* lsg_options.precond */
#define LSG_PC_MG 0
#define LSG_PC_ILU0 1
#define LSG_PC_NONE 2
/* lsg_options.mg_precision */
#define LSG_FP64 0
#define LSG_FP32 1
/* lsg_options.gram_schmidt */
#define LSG_GS_MGS 0
#define LSG_GS_LOWSYNC 1
/* lsg_options.smoother */
#define LSG_SMOOTHER_ADLJ 0   /* reference: damped z,y,x line Jacobi */
#define LSG_SMOOTHER_RBGS 1   /* red-black point Gauss-Seidel (new variant) */
#define LSG_ADLJ_AUTO 0       /* fused for the FP32 cycle, the reference's schedule for the FP64 cycle */
#define LSG_ADLJ_REFERENCE 1  /* the reference's schedule: r -= A c, then the line solve */
#define LSG_ADLJ_FUSED 2      /* ADLJ direction step as one kernel (residual formed in the line solve) */

typedef struct lsg_options {
    int method;          /* LSG_METHOD_*; reference default FGMRES */
    int precond;         /* LSG_PC_*; reference default MG */
    int mg_precision;    /* LSG_FP64 (reference) or LSG_FP32 (mixed precision) */
    int smoother;        /* LSG_SMOOTHER_* */
    int n_pre;           /* pre-smoothing sweeps (reference 0) */
    int n_post;          /* post-smoothing sweeps (reference 3) */
    int max_levels;      /* coarse levels; <= 0: the reference's GridLevels rule */
    int restart;         /* FGMRES restart length (reference FGMRES_RESTART_NUM_P) */
    int max_it;          /* iteration cap (reference MAX_ITER = 200) */
    int zline_reference; /* 1: z-line smoother reads its first right-hand side
                            where the reference does (smoother_adlj_z.h:54-58) */
    double eps;          /* absolute stopping tolerance (reference semantics) */
    double omega;        /* ADLJ damping (reference 0.805) */
    int gram_schmidt;    /* LSG_GS_MGS: modified Gram-Schmidt, one pass per basis
                            vector (reference, fgmres_interface.h:97-102);
                            LSG_GS_LOWSYNC: the same MGS projections computed as
                            h = (I + L)^{-1} V^T w with L the strictly lower part of
                            V^T V (inverse compact WY form), two passes per step */
    int adlj_schedule;   /* LSG_ADLJ_FUSED: every ADLJ direction step
                            ch' = ch + omega T_d^{-1} (b - A ch) as one kernel on
                            levels with the 7-point stencil (other levels keep
                            the separate kernels); LSG_ADLJ_REFERENCE: the
                            reference's r -= A c, c = omega T_d^{-1} r, ch += c
                            (smoother_adlj_interface.h:66-77) everywhere.  The
                            two are equal in exact arithmetic (r = b - A ch
                            before every direction) and differ by rounding.
                            LSG_ADLJ_AUTO (default): fused in the FP32 cycle,
                            the reference's schedule in the FP64 cycle. */
    int reserved[6];
} lsg_options;

typedef struct lsg_stats {
    int iterations;       /* reference IterativeSolverInterface::it */
    int status;           /* LSG_OK / LSG_NOT_CONVERGED / LSG_BREAKDOWN */
    double norm_r;        /* reference norm_r: implicit residual at exit */
    double true_residual; /* ||b - A x||_2 recomputed in FP64 at exit */
    double ms;            /* device time of the solve (CUDA events) */
    double bytes;         /* algorithmic HBM bytes the solve moved */
    int vcycles;          /* preconditioner applications */
    int pad;
    long long kernel_launches; /* CUDA kernels this library launched in the solve */
    int reserved[4];
} lsg_stats;

typedef struct lsg_ctx lsg_ctx;

/* Fill *o with the reference defaults (MG-FGMRES, FP64, ADLJ V(0,3),
   omega 0.805, restart 30, max_it 200, eps 1e-5). */
void lsg_default_options(lsg_options* o);

/* Create a context on CUDA device `device`.  Replaces the construction of
   MGFGMRES / ILUBiCGStab (mg_fgmres.h:33-52, ilu_bicgstab.h:33-64). */
int lsg_create(int device, lsg_ctx** out);
int lsg_destroy(lsg_ctx* ctx);
/* Text of the last error of this context (static storage of the context). */
const char* lsg_last_error(const lsg_ctx* ctx);

/* Set the operator: the reference's CSR of the N x M x K cell-centred
   Laplace operator (LaplaceDiscreteOperator, laplace_discrete_operator.h:107-686
   with the pinned rows of fixPoint :809-821).  Replaces the matrix half of
   IterativeSolverInterface::set (iterative_solver_interface.h:46-55). */
int lsg_set_matrix_csr(lsg_ctx* ctx, int N, int M, int K, const int* rowptr, const int* col,
                       const double* val);
/* Same with device pointers (the reference's CUDA build keeps its CSR in
   device memory, Base/MeshFunctions/array.h). */
int lsg_set_matrix_csr_device(lsg_ctx* ctx, int N, int M, int K, const int* rowptr, const int* col,
                              const double* val, long long nnz);

/* Set the operator from its seven coefficient planes, the structured form of
   the same CSR: planes[s*n + i] is row i's coefficient toward the cell at
   offset s = 0..6 = (0,0,-1), (0,-1,0), (-1,0,0), (0,0,0), (1,0,0), (0,1,0),
   (0,0,1)  (the column order b, s, w, p, e, n, t of the reference's CSR,
   laplace_discrete_operator.h:130-136).  Coefficients toward cells outside
   the grid must be 0.  Host pointer, 7*N*M*K doubles. */
int lsg_set_matrix_stencil7(lsg_ctx* ctx, int N, int M, int K, const double* planes);

/* Assemble the operator on the GPU from the cut-cell geometry, the
   restatement of LaplaceDiscreteOperator::calcLap + fixPoint
   (laplace_discrete_operator.h:107-686, :809-821): celltype[n] (CellTypes
   codes, cut_cells.h:26-168), theta/delta[3n] (per-cell x,y,z face fractions
   and cell sizes, the reference's coord<double> layout), inv_mx/my/mz the
   inverse staggered masses on the x-grid ((N-1)MK), y-grid (N(M-1)K) and
   z-grid (NM(K-1)) (LSSTAGUniformMesh xMesh/yMesh/zMesh inv_VOF), pin0/pin1
   the two rows made identity (N-1 and NM-1 for the flow task).  Host
   pointers.  The result is bit-identical to the reference's CSR values. */
int lsg_set_matrix_geometry(lsg_ctx* ctx, int N, int M, int K, const int* celltype, const double* theta,
                            const double* delta, const double* inv_mx, const double* inv_my, const double* inv_mz,
                            long long pin0, long long pin1);
/* Copy the current operator out as seven planes (layout of
   lsg_set_matrix_stencil7).  Host pointer, 7*N*M*K doubles. */
int lsg_get_matrix_stencil7(lsg_ctx* ctx, double* planes);

/* ---- pressure projection of the time step -----------------------------
   Both calls use the geometry given to lsg_set_matrix_geometry (kept on the
   device).  Fields: u on the x-grid ((N-1)MK), v on the y-grid (N(M-1)K), w on
   the z-grid (NM(K-1)), base-grid fields (flux, b, phi, p) NMK, x fastest.
   Results equal the reference's bit for bit. */

/* Source term of the pressure equation, LaplaceDiscreteOperator::flux after
   initMeshParams + calcFlux for a flow task with fixed bodies
   (DiscreteOperators/WithFlux/Sym/laplace_discrete_operator.h:47-83, :687-808):
   immersed-boundary term on cut cells, inflow profile, N/S and T/B wall
   velocities, outflow from u.  side_type[3n] (the cell's e, n, t face types,
   LSSTAGUniformMesh baseSideTypes, cut_sides.h SideTypes codes), vib[3n] (the
   immersed-boundary velocity, v_ib), u_w[M*K] (inflow profile pU_W, index
   y + M z), bc = {U_E, V_S, V_N, W_B, W_T} (host memory in both variants),
   ux the x-grid velocity; flux[n] out.  Host pointers. */
int lsg_laplace_flux(lsg_ctx* ctx, const int* side_type, const double* vib, const double* u_w, const double* bc,
                     const double* ux, double* flux);
/* Same with device pointers (bc stays a host array of five values). */
int lsg_laplace_flux_device(lsg_ctx* ctx, const int* side_type, const double* vib, const double* u_w,
                            const double* bc, const double* ux, double* flux);

/* Right-hand side of one momentum equation (dir 0: u on the x-grid, 1: v,
   2: w) for a fixed-body flow, HelmholtzDiscreteEquation::recalcRightMember
   (DiscreteEquations/helmholtz_discrete_equation.h:91-95, :213-254):
     aux   = flux2 + C u   (C the convective operator of this step in the
                            reference's CSR form, flux2 its source term),
     right = ((-2 u + 0.5 u_prev) VOF) coef2 - ((G p + flux) + prev_aux) + 2 aux,
   with G the pressure gradient applied from the geometry, flux the Helmholtz
   operator's source term, coef2 = 1/dt; aux is returned as the next step's
   prev_aux.  Bit-identical to the reference.  With rowptr == NULL (col and
   val unused) flux2 already holds flux2 + C u, as lsg_convective_apply
   returns it from the geometry.  Host pointers (staggered-grid vectors, p on
   the base grid). */
int lsg_momentum_rhs(lsg_ctx* ctx, int dir, const int* rowptr, const int* col, const double* val,
                     const double* flux2, const double* u, const double* uprev, const double* vof,
                     const double* hflux, const double* p, const double* prev_aux, double coef2, double* right,
                     double* aux);

/* Device form of lsg_momentum_rhs without a CSR: conv holds flux2 + C u
   (lsg_convective_apply_device with init = flux2), gp_work is a scratch
   vector of the staggered grid (receives G p); right and aux as there; aux
   may alias nothing else.  Device pointers. */
int lsg_momentum_rhs_device(lsg_ctx* ctx, int dir, const double* conv, const double* u, const double* uprev,
                            const double* vof, const double* hflux, const double* p, const double* prev_aux,
                            double coef2, double* right, double* aux, double* gp_work);

/* Convective operator of momentum component dir (0 x, 1 y, 2 z) applied
   from the geometry: out = init + C(u) v on the dir-grid, C the operator
   ConvectiveDiscreteOperatorX/Y/Z::calcConv* builds from the velocity
   (ux, uy, uz) (DiscreteOperators/WithFlux/SkewSym/convective_discrete_operator_x.h:49-366,
   _y.h, _z.h); init may be NULL (zero).  zconv_reference = 1 reproduces the
   reference's x-velocity indexing in the z operator (M + 1 cells per row,
   calcConvZ launched with M3 at convective_discrete_operator_z.h:772-773);
   0 uses the grid's own row length.  Bit-identical to init + (the
   reference's CSR) v.  Host pointers. */
int lsg_convective_apply(lsg_ctx* ctx, int dir, const double* ux, const double* uy, const double* uz,
                         const double* v, const double* init, double* out, int zconv_reference);
/* Same on device pointers. */
int lsg_convective_apply_device(lsg_ctx* ctx, int dir, const double* ux, const double* uy, const double* uz,
                                const double* v, const double* init, double* out, int zconv_reference);

/* The momentum operator of direction dir (0 x, 1 y, 2 z) assembled on the
   GPU from the cut-cell geometry and set as the context's operator (a 7-point
   operator on the staggered grid of N-1 x M x K, N x M-1 x K or N x M x K-1
   cells), replacing HelmholtzDiscreteOperatorX/Y/Z::build/calcElem
   (DiscreteOperators/WithFlux/Sym/helmholtz_discrete_operator_x.h:98-686,
   _y.h:92-…, _z.h:90-…) with the outflow terms of addPlusOutFlow
   (helmholtz_discrete_operator_base.h:50-58).  stype are the staggered cell
   types; theta, alpha, delta, delta_ib_en/ws/nb/st, inv_delta_ib_ne/tn (3n,
   xyz interleaved) and inv_vof (n) describe the N x M x K base grid; vof are
   the staggered cell volumes (the reference's M_x/M_y/M_z); nu the
   viscosity, coef the time-integration coefficient (COEF_INTEGR_TIME, 1.5/dt
   for BDF2); is_flow selects the flow-task boundary conditions (outflow on
   E, slip T/B walls).  Entries agree with the reference to rounding (fluid
   and cut-cell rows bitwise); read back with lsg_get_matrix_stencil7, solve
   with lsg_setup (ILU(0) preconditioner) + lsg_solve.  Host pointers. */
int lsg_set_matrix_helmholtz(lsg_ctx* ctx, int dir, int N, int M, int K, const int* stype, const double* theta,
                             const double* alpha, const double* delta, const double* inv_vof, const double* vof,
                             const double* delta_ib_en, const double* delta_ib_ws, const double* delta_ib_nb,
                             const double* delta_ib_st, const double* inv_delta_ib_ne, const double* inv_delta_ib_tn,
                             double nu, double coef, int is_flow);

/* Source term of the momentum operator of direction dir as build() leaves
   it (HelmholtzDiscreteOperatorX/Y/Z::initInFlowFlux: inFlowFluxHelm*,
   addFluxNS*, addFluxTB*; helmholtz_discrete_operator_x.h:50-96, :750-758,
   _y.h, _z.h): the inflow value on the x = 0 cells, then the S/N and B/T wall
   terms.  bc = (U_W U_E U_S U_N U_B U_T, V_W V_E V_S V_N V_B V_T, W_W W_E
   W_S W_N W_B W_T), u_w the x-inflow profile (M*K, the reference's pU_W).
   With ib != 0 the immersed-boundary term (ibFluxHelmX/Y/Z, :687-731, run by
   the reference for moving bodies) is written over rows 1 .. Ms-2 as the
   reference does; the arrays after `ib` are then required (NULL allowed
   otherwise).  Bitwise equal to the reference.  Host pointers; flux holds
   the staggered grid's cells. */
int lsg_helmholtz_flux(lsg_ctx* ctx, int dir, int N, int M, int K, const int* stype, const double* delta,
                       const double* u_w, const double* bc, double nu, int ib, const int* side_type,
                       const double* theta, const double* alpha, const double* inv_vof, const double* delta_ib_en,
                       const double* delta_ib_ws, const double* delta_ib_nb, const double* delta_ib_st,
                       const double* inv_delta_ib_ne, const double* inv_delta_ib_tn, const double* vib,
                       const double* vib_yx, const double* vib_zy, double* flux);

/* Source term of the convective operator of direction dir as the time step
   recomputes it (SkewSymDiscreteOperator::recalc -> calcFlux -> baseFlux,
   skew_sym_discrete_operator.h:244-249, :290-294), the flux2 input of
   lsg_momentum_rhs.  For z: ConvectiveDiscreteOperatorZ::baseFlux
   (convective_discrete_operator_z.h:748-757: inflow W_W with the x-inflow
   profile, outflow from ux and uz, S/N walls W_S*V_S, W_N*V_N, B/T outflow
   terms from uz), bitwise.  For x and y the reference's operators never run
   their baseFluxX/baseFluxY (they do not override baseFlux), so the term is
   0, reproduced.  theta, delta (3n) on the N x M x K base grid, ux/uz the
   x/z-grid velocities, u_w the x-inflow profile (M*K), bc as for
   lsg_helmholtz_flux.  Host pointers. */
int lsg_convective_flux(lsg_ctx* ctx, int dir, int N, int M, int K, const double* theta, const double* delta,
                        const double* ux, const double* uy, const double* uz, const double* u_w, const double* bc,
                        double* flux);
/* Same on device pointers (bc on the host). */
int lsg_convective_flux_device(lsg_ctx* ctx, int dir, int N, int M, int K, const double* theta, const double* delta,
                               const double* ux, const double* uy, const double* uz, const double* u_w,
                               const double* bc, double* flux);

/* ---- loads on the immersed boundary (LoadsCalculator, loads_calculator.h) ---- */

typedef struct lsg_loads_result {
    double force[3];       /* F_aer_x, F_aer_y, F_aer_z: sums of the per-cut-cell forces */
    double coef[3];        /* C_d, C_y, C_z = force * fcoef */
    double moment_raw[3];  /* sums of the per-cell moments M_z, M_x, M_y (calcMoment, calcMomentX/Y) */
    double moment[3];      /* the same after the moment low-pass filters
                              (moment_aer, moment_x_aer, moment_y_aer) */
    int count;             /* number of cut cells */
} lsg_loads_result;

/* The cut-cell list and the geometry the loads read, replacing
   LoadsCalculator::set + the OnAirfoil list (loads_calculator.h:1298-1333;
   BaseTaskDescription::addCutCell, base_task_description.h:127-132).  cells
   holds the base-grid indices of the cut cells in the order the forces are
   reported; the x/y-grid indices follow from them.  celltype, inv_vof (n)
   and theta, delta, delta_ib_max, inv_delta_ib_ne, inv_delta_ib_tn, nodes
   (3n, xyz interleaved, the reference's coordinate arrays) describe the
   N x M x K base grid; center is the moment centre (cur_C).  fcoef scales
   forces to coefficients; dt initialises the moment filters
   (ButterworthLowPassFilter::init with the reference defaults).  A cut cell
   on the outer layer of the grid is rejected.  Host pointers; the packed
   records stay on the device until the next call. */
int lsg_loads_set(lsg_ctx* ctx, int N, int M, int K, int count, const int* cells, const int* celltype,
                  const double* theta, const double* delta, const double* inv_vof, const double* delta_ib_max,
                  const double* inv_delta_ib_ne, const double* inv_delta_ib_tn, const double* nodes,
                  const double* center, double fcoef, double dt);
/* LoadsCalculator::calculate (loads_calculator.h:1366-1377, calc :79-1269):
   per-cut-cell forces, their sums and coefficients, the moments and one step
   of the moment filters.  ux, uy, uz are the staggered velocity grids, p the
   pressure, vib / vib_yx / vib_zy the immersed-boundary velocities (3n);
   nu_cell (n) replaces nu per cell when not NULL.  forces (3 * count: all x,
   then all y, then all z) may be NULL.  Per-cell forces and moments are
   bitwise equal to the reference's; the sums differ from its OpenMP sums by
   summation order only.  With no cut cells nothing is computed (as in the
   reference) and the filters do not advance.  Host pointers. */
int lsg_loads_calculate(lsg_ctx* ctx, const double* ux, const double* uy, const double* uz, const double* p,
                        const double* vib, const double* vib_yx, const double* vib_zy, const double* nu_cell,
                        double nu, double* forces, lsg_loads_result* out);
/* Same on device pointers (forces a device pointer or NULL; out on the host). */
int lsg_loads_calculate_device(lsg_ctx* ctx, const double* ux, const double* uy, const double* uz, const double* p,
                               const double* vib, const double* vib_yx, const double* vib_zy,
                               const double* nu_cell, double nu, double* forces, lsg_loads_result* out);
/* Restart the three moment filters with time step dt. */
int lsg_loads_reset_filter(lsg_ctx* ctx, double dt);
/* Gradient of J = weight[0] F_aer_x + weight[1] F_aer_y + weight[2] F_aer_z
   with respect to ux, uy, uz and p (the forces are affine in them, so the
   gradient depends on the geometry, nu and the weights only): the adjoint
   of the loads for drag-based objectives.  No reference counterpart (the
   reference has no adjoint).  Outputs are overwritten.  Host pointers. */
int lsg_loads_adjoint(lsg_ctx* ctx, const double* weight, const double* nu_cell, double nu, double* g_ux,
                      double* g_uy, double* g_uz, double* g_p);
/* Same on device pointers (weight on the host). */
int lsg_loads_adjoint_device(lsg_ctx* ctx, const double* weight, const double* nu_cell, double nu,
                             double* g_ux, double* g_uy, double* g_uz, double* g_p);

/* Transposed Jacobian of the convective term out = init + C(U) v of
   lsg_convective_apply: for a cotangent lam on the dir-grid, the gradients
   of <lam, C(U) v> with respect to the three velocity grids (ux_bar, uy_bar,
   uz_bar) and to v (v_bar).  No reference counterpart (the reference has no
   adjoint); it is the nonlinear part of the momentum step's adjoint.  Host
   pointers, outputs overwritten. */
int lsg_convective_adjoint(lsg_ctx* ctx, int dir, const double* ux, const double* uy, const double* uz,
                           const double* v, const double* lam, double* ux_bar, double* uy_bar, double* uz_bar,
                           double* v_bar, int zconv_reference);
/* Same on device pointers; the outputs accumulate (zero them first; for the
   equation's own velocity v = U_dir the same buffer may serve as v_bar and
   the dir component of U_bar). */
int lsg_convective_adjoint_device(lsg_ctx* ctx, int dir, const double* ux, const double* uy, const double* uz,
                                  const double* v, const double* lam, double* ux_bar, double* uy_bar, double* uz_bar,
                                  double* v_bar, int zconv_reference);

/* Staggered cell types (LSSTAGUniformMesh xMesh/yMesh/zMesh typeOfCell),
   needed by the staggered-grid entry points below.  Checked on the host like
   the base types (a kept face must lie inside the grid).  Host pointers. */
int lsg_set_staggered_types(lsg_ctx* ctx, const int* xtype, const int* ytype, const int* ztype);

/* b = Dx u + Dy v + Dz w + flux with b[pin0] = b[pin1] = 0: the right-hand
   side of the pressure equation, PoissonDiscreteEquation::recalcRightMember
   (DiscreteEquations/poisson_discrete_equation.h:145-159) with the divergence
   operators DivergenceDiscreteOperatorX/Y/Z
   (DiscreteOperators/Divergence/divergence_discrete_operator_x.h:119-159,
   _y.h:92-121, _z.h:86-111) applied from the geometry.  Host pointers. */
int lsg_projection_rhs(lsg_ctx* ctx, const double* u, const double* v, const double* w, const double* flux,
                       double* b);
/* Same on device pointers (the context's device, its stream). */
int lsg_projection_rhs_device(lsg_ctx* ctx, const double* u, const double* v, const double* w, const double* flux,
                              double* b);

/* Velocity and pressure update after the pressure solve, SetSolutions::
   correction (Base/set_solutions.h:215-237): u = inv_VOF_x (Gx phi) + us
   (gradient GradientDiscreteOperatorX/Y/Z, DiscreteOperators/Gradient/
   gradient_discrete_operator_x.h:58-77, _y.h:52-74, _z.h:45-62), likewise v, w;
   with outflow != 0 the east outflow and bottom/top backflow clamps
   (corrOutFlow / corrOutFlowTB, :87-118, :297-304; vbase = V_BASE); then
   p += phi * coef (coef = 1.5/dt for the BDF2 step).  phi is not modified
   (the reference scales its copy in place).  Host pointers; u/v/w are outputs
   and may alias us/vs/ws. */
int lsg_projection_correct(lsg_ctx* ctx, const double* phi, const double* us, const double* vs, const double* ws,
                           double* u, double* v, double* w, double* p, double coef, double vbase, int outflow);
/* Adjoint of the projection step without the outflow clamps (the linear map
   (u*, v*, w*, flux, p) -> (u, v, w, p) of lsg_projection_rhs, the pressure
   solve and lsg_projection_correct with outflow = 0): given the cotangents of
   the outputs, returns those of the inputs,
     phi_bar = Gx^T S_x ubar_out + Gy^T S_y vbar_out + Gz^T S_z wbar_out + coef pbar_out,
               set to 0 on solid rows and on empty rows (cut cells whose
               faces are all closed): the forward solve never excites them
               and no velocity reads their pressure,
     A^T lambda = phi_bar (lsg_solve_adjoint's solver),  b_bar = lambda with the pins zeroed,
     ubar = ubar_out + Dx^T b_bar (likewise v, w),  fluxbar = b_bar,
   the pressure cotangent passing through unchanged.  No counterpart in the
   reference (the adjoint of its projection step).  Host pointers; st
   receives the adjoint solve's statistics (may be NULL). */
int lsg_projection_adjoint(lsg_ctx* ctx, const double* ubar_out, const double* vbar_out, const double* wbar_out,
                           const double* pbar_out, double coef, double* ubar, double* vbar, double* wbar,
                           double* fluxbar, lsg_stats* st);
/* out = Gx^T gx + Gy^T gy + Gz^T gz on the base grid: the transpose of the
   pressure gradient GradientDiscreteOperatorX/Y/Z
   (DiscreteOperators/Gradient/gradient_discrete_operator_x.h:58-77, _y.h:52-74,
   _z.h:45-62) applied from the geometry, as lsg_projection_adjoint applies it
   with unit weights.  It is the pressure cotangent of the G p term of the
   momentum right-hand side (lsg_momentum_rhs).  No reference counterpart.
   Host pointers (staggered-grid inputs). */
int lsg_gradient_transpose(lsg_ctx* ctx, const double* gx, const double* gy, const double* gz, double* out);
/* Same on device pointers (the context's device; the call returns when the
   result is written). */
int lsg_gradient_transpose_device(lsg_ctx* ctx, const double* gx, const double* gy, const double* gz, double* out);
/* Reverse sweep of the time steps, per momentum equation dir (device
   pointers on the dir staggered grid, a context holding the geometry and
   the staggered types): with r = rsol on fluid faces and 0 on solid ones
   (written to r),
     fbar += vof r,  ubar += (-2 coef2) vof r,  uprevbar = (coef2 / 2) vof r,
     histbar = -r,   convbar += 2 r,
   the cotangents of the forcing, the current and previous velocity, the
   Adams-Bashforth history and the convective term, given the transposed
   momentum solve's solution rsol (coef2 = 1/dt): the transpose of the BDF2 /
   Adams-Bashforth right-hand side of HelmholtzDiscreteEquation
   (helmholtz_discrete_equation.h:213-254).  No reference counterpart. */
int lsg_momentum_cotangents_device(lsg_ctx* ctx, int dir, const double* vof, const double* rsol, double coef2,
                                   double* r, double* fbar, double* ubar, double* uprevbar, double* histbar,
                                   double* convbar);
/* out = in on the fluid faces of staggered grid dir, 0 on its solid faces
   (device pointers; in and out may alias). */
int lsg_fluid_faces_device(lsg_ctx* ctx, int dir, const double* in, double* out);
/* Transpose of the outflow clamps of SetSolutions::correction
   (Base/set_solutions.h:87-118, :297-304) for the adjoint sweep: o = b with
   the entries the clamps overwrite set to 0, decided from qx, qz (the x- and
   z-velocities before the clamps): per interior (y, z) row of the east
   outflow whose last or next-to-last x-face is negative, that x-face and
   the matching y- and z-faces; bottom z-faces with positive and top ones
   with negative velocity.  o may equal b.  Device pointers; needs the
   context's grid (an operator). */
int lsg_clamp_transpose_device(lsg_ctx* ctx, const double* qx, const double* qz, const double* bx,
                               const double* by, const double* bz, double* ox, double* oy, double* oz);
/* dst[dst_idx[e]] += coef[e] * src[src_idx[e]] * (src2 ? src2[src2_idx[e]] : 1)
   for e < count: the boundary source terms' transposes of the adjoint sweep
   (index sets built once by the caller).  FP64 atomic adds: entries sharing
   a destination add in an unspecified order.  Device pointers. */
int lsg_scatter_add_device(lsg_ctx* ctx, long long count, double* dst, const long long* dst_idx,
                           const double* src, const long long* src_idx, const double* coef,
                           const double* src2, const long long* src2_idx);
/* y += alpha x on device vectors of n doubles. */
int lsg_axpy_device(lsg_ctx* ctx, long long n, double alpha, const double* x, double* y);
/* lsg_projection_adjoint on device pointers; outputs must not alias inputs. */
int lsg_projection_adjoint_device(lsg_ctx* ctx, const double* ubar_out, const double* vbar_out,
                                  const double* wbar_out, const double* pbar_out, double coef, double* ubar,
                                  double* vbar, double* wbar, double* fluxbar, lsg_stats* st);
/* Same on device pointers. */
int lsg_projection_correct_device(lsg_ctx* ctx, const double* phi, const double* us, const double* vs,
                                  const double* ws, double* u, double* v, double* w, double* p, double coef,
                                  double vbase, int outflow);

/* Build the preconditioner for the current operator (multigrid hierarchy:
   MultiGridSolver::set multigrid_solver.h:76-101 / CoarseGrid::set
   coarse_grid.h:93-106; or ILU(0): ILUDecompositionSparseMatrix::decompose
   ilu_decomposition_sparse_matrix.h:138-148).  Call again after
   lsg_set_matrix_csr to rebuild (rebuildPreconditioner). */
int lsg_setup(lsg_ctx* ctx, const lsg_options* opts);
/* Wall times (host clock, ms) of the context's last lsg_set_matrix_* call
   (operator upload or assembly and the row-dictionary build, both on the
   device) and of its last lsg_setup (Galerkin products and dictionaries of
   the coarse levels, line factorisations, coarsest LU, FP32 copies, Krylov
   buffers).  The reference rebuilds the same in
   IterativeSolverInterface::set / rebuildPreconditioner
   (iterative_solver_interface.h:46-70, coarse_grid.h:93-106). */
int lsg_setup_times(const lsg_ctx* ctx, double* matrix_ms, double* setup_ms);
/* The row dictionary of multigrid level `level` (0 = the operator itself,
   needs an operator; 1..lsg_mg_num_levels() need lsg_setup): *nclass
   distinct rows of *noff coefficients (7, or 27 on Galerkin levels) in
   first-seen row order, and each row's index into them.  cls (n ints) and
   dict (nclass * noff doubles) may be null to query the sizes first. */
int lsg_row_classes(lsg_ctx* ctx, int level, int* cls, double* dict, int* nclass, int* noff);

/* Solve A x = b; x holds the initial guess on entry and the solution on exit
   (IterativeSolverInterface::solve).  Host buffers of N*M*K doubles.
   The first preconditioner application after lsg_setup records the
   multigrid V-cycle (or the ILU(0) sweeps) as a CUDA graph on the
   context's own stream and later ones replay it; make that first solve
   outside any stream capture of the caller's. */
int lsg_solve(lsg_ctx* ctx, const double* b, double* x, lsg_stats* stats);
/* Same with device buffers (no host copies). */
int lsg_solve_device(lsg_ctx* ctx, const double* b, double* x, lsg_stats* stats);

/* y = A x with the stored operator (RealValuedMeshFunction::mvProd,
   real_valued_mesh_function.h:81-88).  Host buffers. */
int lsg_apply(lsg_ctx* ctx, const double* x, double* y);
/* x = M^{-1} b: one application of the configured preconditioner
   (MultiGridSolver::solve multigrid_solver.h:48-75 or the ILU(0) solves).
   Host buffers; for the FP32 multigrid the result is the FP32 cycle rounded
   to FP64. */
int lsg_precond_apply(lsg_ctx* ctx, const double* b, double* x);

/* Adjoint (no counterpart in the reference, which has no adjoint; built for
   gradient-based use of the pressure solve).
   lsg_apply_transpose: y = A^T x, the transposed cut-cell stencil (row i of
     A^T holds column i of A).
   lsg_solve_adjoint: A^T lambda = g with the same method, preconditioner
     construction and options as the forward solve, applied to A^T (the
     multigrid hierarchy is rebuilt from A^T on first use); lambda holds the
     initial guess on entry.  For J(x) with A x = b, dJ/db = lambda when
     g = dJ/dx.
   lsg_operator_gradient: grad[s*n + i] = -lambda_i x_{i + off_s} = dJ/dA for
     the seven planes of lsg_set_matrix_stencil7 (0 toward outside cells).
   Host buffers. */
/* Tecplot solution file, byte for byte the file SolTecplotPrinter::printField
   writes (Base/TecplotPrinters/sol_tecplot_printer.h:254-355, header of
   BaseTecplotPrinter::init base_tecplot_printer.h:35-60): the (N+2) x (M+2)
   x (K+2) points (walls, boundary rows, cell centres) with x y z P SPD_x
   SPD_y SPD_z SPD in ostream's default format.  nodes: the cell-centre
   coordinates (3 N M K, xyz interleaved, LSSTAGUniformMesh m_nodes); delta,
   theta: as lsg_set_matrix_geometry; celltype: base cell types; u, v, w, p
   the staggered velocities and the pressure; u_w the inflow profile (M K,
   the task's pU_W; NULL: none); bc the 18 boundary velocities U_W U_E U_S
   U_N U_B U_T V_W .. V_T W_W .. W_T; flow != 0 for a flow task (outflow
   east, the B and T planes repeat the first and last layer).
   lsg_tecplot_sol_write: host arrays, no context, no device work.
   lsg_tecplot_sol_async: u, v, w, p on the device of a context holding the
   base grid's geometry; the call copies them to pinned host memory (the
   caller may overwrite them on return; they must be complete when the call
   is made) and returns while a host thread formats and writes the file;
   lsg_tecplot_wait joins that thread and returns its status.  One write in
   flight per context (a second call waits for the first).  The status is
   sticky: the first failure of any write since the last lsg_tecplot_wait is
   what lsg_tecplot_wait returns, and that call clears it. */
int lsg_tecplot_sol_write(const char* path, int N, int M, int K, const double* nodes, const double* delta,
                          const double* theta, const int* celltype, const double* u, const double* v,
                          const double* w, const double* p, const double* u_w, const double* bc, int flow);
int lsg_tecplot_sol_async(lsg_ctx* ctx, const char* path, const double* nodes, const double* delta,
                          const double* theta, const int* celltype, const double* u, const double* v,
                          const double* w, const double* p, const double* u_w, const double* bc, int flow);
int lsg_tecplot_wait(lsg_ctx* ctx);

int lsg_apply_transpose(lsg_ctx* ctx, const double* x, double* y);
int lsg_solve_adjoint(lsg_ctx* ctx, const double* g, double* lambda, lsg_stats* stats);
int lsg_operator_gradient(lsg_ctx* ctx, const double* lambda, const double* x, double* grad);

/* Multigrid introspection for parity checks.  Level 0 is the fine grid. */
int lsg_mg_num_levels(const lsg_ctx* ctx);  /* coarse levels (GridLevels), or < 0 */
int lsg_mg_level_dims(const lsg_ctx* ctx, int level, int dims[3]);
/* Level operator as CSR with columns sorted (rowptr n+1, col/val nnz).
   Call with col == NULL to get *nnz only. */
int lsg_mg_level_csr(lsg_ctx* ctx, int level, int* rowptr, int* col, double* val, long long* nnz);
/* Factored line tridiagonal of `dir` ('x', 'y', 'z') on `level` in the
   reference's storage order (TriDiagonalMatrix c, d, e after triLU,
   tridiagonal_matrix.h:45-67): c and e hold n-1 values, d holds n. */
int lsg_mg_level_tridiag(lsg_ctx* ctx, int level, char dir, double* c, double* d, double* e);

/* Time one kernel of the solve path on the context's stream with CUDA
   events (after a warm-up launch): `which` = 0/1/2 the finest-level x/y/z
   line solve of the multigrid smoother, 3 the finest-level residual update
   r -= A c, 4 the FP64 operator apply fused with a dot product (Krylov),
   5 the residual update of the first coarse level (Galerkin stencil),
   6 the operator apply fused with a dot product on an FP32 preconditioned
   vector (the Krylov product of the FP32-multigrid solve, z planes staged in
   shared memory), 7 the same product by the one-thread-per-cell kernel the
   solve uses on wide grids, 8 the same product by the register z-marching
   kernel (no staging; for comparison), 9/10/11 the fused ADLJ direction
   step (residual formed inside the line solve) along x/y/z on the finest
   level (needs a level that runs it: LSG_ADLJ_FUSED, or LSG_ADLJ_AUTO in
   FP32), 12/13 the y/z steps with the segment maps walked by each thread
   instead of composed by log-step scans, 14/15 the same for the y/z line
   solves of the reference schedule, 16/17 those line solves with 4-cell
   segments (the FP64 z-line solve's own form), 18/19 the first coarse
   level's residual with 8 / 16 z-planes per thread (for comparison).
   Returns the mean duration of one launch and the algorithmic HBM bytes one
   launch moves (compulsory traffic of its inputs and outputs).  Needs
   lsg_setup with the multigrid preconditioner. */
int lsg_profile_kernel(lsg_ctx* ctx, int which, int reps, double* ms_per_launch, double* bytes_per_launch);

/* Self-test of the bounded waits: runs the one-launch ILU(0) sweep of an
   ILU(0) context with one CTA leaving before its first barrier arrival, so
   the other CTAs' first wait runs out (after about one second) and the
   kernel returns with its error flag set.  Returns LSG_ERR_CUDA with
   lsg_last_error describing it (the expected result); the context stays
   usable.  Needs lsg_setup with LSG_PC_ILU0 on a grid whose sweep has two
   CTAs or more. */
int lsg_selftest_wait_limit(lsg_ctx* ctx);

/* Residual r = b - A x and its squared 2-norm for a 7-point operator given
   as seven coefficient planes (layout of lsg_set_matrix_stencil7), without
   allocating device memory.  No counterpart in the reference: it is for
   callers that cannot call cudaMalloc (a host application recording a CUDA
   graph, a solver embedded under a device-memory budget owned by its host
   program).  All pointers are device pointers owned by the caller; r may be
   NULL (norm only); *norm2 receives ||b - A x||^2 (FP64).  Work is queued on
   `stream` (a cudaStream_t, NULL = legacy default stream); read *norm2 after
   synchronising it.  The stream must belong to the calling thread's current
   device: the scratch address used is the current device's, and the
   pointers must be that device's memory.  Scratch is a file-scope device array of the library
   (4096 block partials + a counter, about 32 KiB per GPU, held until the
   process exits), which caps the grid at 16,777,216 cells; larger grids are
   rejected with LSG_ERR_ARG and a message on stderr.  The first call on a
   device looks up the array's device address (cudaGetSymbolAddress), so make
   that first call before any stream capture.  All calls share the array:
   calls that overlap on the GPU race and must be serialised by the caller. */
int lsg_residual_norm_noalloc(int N, int M, int K, const double* planes, const double* x, const double* b,
                              double* r, double* norm2, void* stream);

/* Change the absolute stopping tolerance of the next solves without a new
   set-up (the hierarchy, factors and graphs stay): what the reference's
   equations do when they set solver.eps before a solve
   (IterativeSolverInterface::eps, iterative_solver_interface.h:66), e.g. a
   tolerance relative to each right-hand side's norm. */
int lsg_set_tolerance(lsg_ctx* ctx, double eps);

/* Mesh build of the flow task on the device: the restatement, for a uniform
   grid, of BaseTaskDescription::buildMesh (base_task_description.h:330-371)
   for a flow past fixed bodies -- the level set (the task's buildLS, e.g.
   FlowSphereTaskDescription::calcLevelSetSphere,
   flow_sphere_task_description.h:57-74), the edge fractions alpha with the
   in-place oscillation fix (FlowTaskDescription::calcAlpha,
   flow_task_description.h:102-136; checkOscLS / BuildAlpha,
   ls_stag_uniform_mesh.h:2906-2963), face and cell types (calcTypeOfCells,
   flow_task_description.h:175-230; TypeOfSide / TypeOfCell,
   ls_stag_uniform_mesh.h:2969-2977, :3624-3675), face fractions theta
   (calcTheta; getThetaZ / BuildTheta / tbBuildTheta, :1652-1837), cell
   volumes (kernel v, :1838-2714) and their inverses
   (ls_stag_base_mesh_params.h:77-85), staggered cell types (cvu / cvv / cvw,
   :108-136), staggered volumes (mx / my / mz, :2804-2826) and their inverses,
   the immersed-boundary face areas (buildDelta_ib: calcDeltaIB, :186-1650)
   and inverse distances (buildInvBaseDelta_ib: calcInvBaseDeltaIb,
   :3395-3620).  Bit-identical to the reference's arrays.
     N, M, K    base grid; h[3] the uniform cell sizes (nodes at (i + 1/2) h);
     block[4]   the level-set block hs, hf, vs, vf of the task (the reference's
                hs_loc .. vf_loc, flow_task_description.h:388-398): cells
                [hs, hf) x [vs, vf) x [0, K) are built from the level set, all
                others are plain fluid / box-border cells;
                1 <= hs < hf <= N-1, 1 <= vs < vf <= M-1;
     bodies     n_bodies records of 17 doubles (kind 0 sphere / 1 ellipsoid,
                centre[3], radius, semi-axes[3], rotation[9] row major, body
                frame = R (x - c)), merged by max (phi > 0 inside); or
     phi        (host, N*M*K doubles, used when not NULL) the task's own level
                set at the upper cell corners; values outside the block are
                taken as 0, as the reference's walks find them;
     *ms        (may be NULL) device time of the build.
   The mesh stays on the device of the context. */
int lsg_mesh_build(lsg_ctx* ctx, int N, int M, int K, const double* h, const int* block, int n_bodies,
                   const double* bodies, const double* phi, double* ms);
/* Copy one array of the built mesh to host memory `out` (the reference's
   layouts: coord triples x, y, z per cell for alpha, theta, delta and the
   side types (east, north, top faces); staggered arrays on the x-grid
   (N-1)MK, y-grid N(M-1)K, z-grid NM(K-1)). */
#define LSG_MESH_PHI_LS 0     /* level set as evaluated (double n) */
#define LSG_MESH_PHI 1        /* after the oscillation fix (double n) */
#define LSG_MESH_ALPHA 2      /* double 3n */
#define LSG_MESH_SIDE_TYPE 3  /* int 3n (SideTypes codes) */
#define LSG_MESH_CELL_TYPE 4  /* int n (CellTypes codes) */
#define LSG_MESH_THETA 5      /* double 3n */
#define LSG_MESH_DELTA 6      /* double 3n */
#define LSG_MESH_VOF 7        /* double n */
#define LSG_MESH_INV_VOF 8    /* double n */
#define LSG_MESH_XTYPE 9      /* int, x-grid */
#define LSG_MESH_YTYPE 10     /* int, y-grid */
#define LSG_MESH_ZTYPE 11     /* int, z-grid */
#define LSG_MESH_VOF_X 12     /* double, x-grid */
#define LSG_MESH_VOF_Y 13
#define LSG_MESH_VOF_Z 14
#define LSG_MESH_INV_MX 15    /* double, x-grid: 1 / M_x */
#define LSG_MESH_INV_MY 16
#define LSG_MESH_INV_MZ 17
/* immersed-boundary face areas (calcDeltaIB, ls_stag_uniform_mesh.h:186-1650)
   and inverse distances (calcInvBaseDeltaIb, :3395-3620), double 3n each */
#define LSG_MESH_DIB_EN 18
#define LSG_MESH_DIB_WS 19
#define LSG_MESH_DIB_NB 20
#define LSG_MESH_DIB_ST 21
#define LSG_MESH_DIB_MAX 22
#define LSG_MESH_INV_DIB_NE 23
#define LSG_MESH_INV_DIB_TN 24
int lsg_mesh_get(lsg_ctx* ctx, int field, void* out);
/* Fixed-point sweeps the oscillation fix took in the last build (>= 1). */
int lsg_mesh_osc_sweeps(const lsg_ctx* ctx);
/* Set the context's operator to the Laplace operator assembled from the
   built mesh (lsg_set_matrix_geometry on the device-resident arrays, with
   the staggered types of lsg_set_staggered_types), pin0 / pin1 the pinned
   rows (N-1 and NM-1 for the flow task). */
int lsg_set_matrix_mesh(lsg_ctx* ctx, long long pin0, long long pin1);

/* Library build string (version, arch). */
/* ---- native fixed-body flow time step ------------------------------------
   TimeSteppingMethodInterface::step (time_stepping_method_interface.h:180-214)
   for a flow past bodies that do not move, over the contexts the caller set
   up: the pressure-equation context (geometry from lsg_set_matrix_geometry or
   lsg_set_matrix_mesh, staggered types from lsg_set_staggered_types: fluxes,
   convective operator, right-hand sides, projection), the pressure solver
   context (the same context, or one holding the same operator with its pins
   negated for the FP32 cycle), and the three momentum solver contexts
   (lsg_set_matrix_helmholtz + lsg_setup).  One step: pressure source term;
   per component the convective term, right-hand side with its
   Adams-Bashforth history and the ILU-FGMRES solve from the current velocity
   (the three solves concurrently, one host thread and context each);
   b = D u* + flux and the pressure solve from 0; the projection.  The state
   lives in device memory owned by the stepper.  The contexts must outlive
   it and are not used by anyone else during a step. */
typedef struct lsg_flow lsg_flow;
typedef struct lsg_flow_desc {
    int N, M, K;              /* base grid */
    int device;               /* CUDA device of the contexts */
    lsg_ctx* pres;            /* pressure equation (geometry, staggered types) */
    lsg_ctx* psolve;          /* pressure solver (may be pres) */
    lsg_ctx* mom[3];          /* momentum solvers x, y, z */
    /* copied at creation; host or device pointers */
    const int* side_type;     /* 3n, as for lsg_laplace_flux */
    const double* vib;        /* 3n */
    const double* u_w;        /* M*K inflow profile */
    const double* theta;      /* 3n */
    const double* delta;      /* 3n */
    const double* vof[3];     /* staggered volumes, x/y/z grids */
    const double* hflux[3];   /* Helmholtz source terms (lsg_helmholtz_flux) */
    double bc[18];            /* boundary velocities, as for lsg_helmholtz_flux */
    double bc_lap[5];         /* U_E, V_S, V_N, W_B, W_T */
    double coef, coef2, vbase;
    double p_rel_tol;         /* > 0: each pressure solve to p_rel_tol * ||b||; 0: the context's eps */
    int zconv_reference;      /* as for lsg_convective_apply */
    int reserved[7];
} lsg_flow_desc;
int lsg_flow_create(const lsg_flow_desc* desc, lsg_flow** out);
int lsg_flow_destroy(lsg_flow* flow);
const char* lsg_flow_last_error(const lsg_flow* flow);
/* The current and previous velocities and the pressure (host or device
   pointers); prev_aux = the three momentum histories, or null to form them
   from the state as HelmholtzDiscreteEquation::set does (flux2 + C(u) u). */
int lsg_flow_set_state(lsg_flow* flow, const double* const u[3], const double* const uprev[3], const double* p,
                       const double* const prev_aux[3]);
/* One time step; its[4] = iterations of the x, y, z momentum and pressure
   solves.  Returns LSG_OK, a solve's LSG_NOT_CONVERGED / LSG_BREAKDOWN
   (the step completes), or a negative error. */
int lsg_flow_step(lsg_flow* flow, int its[4]);
/* Copy the current velocities, pressure and previous velocities out (any
   pointer may be null; host or device). */
int lsg_flow_state(lsg_flow* flow, double* const u[3], double* p, double* const uprev[3]);

const char* lsg_version(void);

#ifdef __cplusplus
}
#endif

#endif /* LSSTAG_B200_H */
