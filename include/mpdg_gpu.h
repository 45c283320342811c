/*
 * mpdg_gpu.h -- C ABI of the B200 (sm_100a) matrix-free operator library.
 *
 * Drop-in boundary for MeltPoolDG's matrix-free hot path.  Each entry point replaces one member
 * of the reference interface (paths inside the MeltPoolDG source tree):
 *
 *   OperatorMatrixFree<dim,number>            include/meltpooldg/core/operator_base.hpp:189-283
 *     vmult(dst, src)                         :239-243   -> mpdg_op_vmult / _f32 / _host
 *     create_rhs(dst, src)                    :208-212   -> mpdg_op_create_rhs
 *     compute_inverse_diagonal_from_matrixfree(diag) :268-272 -> mpdg_op_compute_inverse_diagonal
 *   OperatorBase::reset_time_increment(dt)    :41-46     -> mpdg_op_reset_time_increment
 *   OperatorBase::reset_dof_index(idx)        :31-35     -> mpdg_op_reset_dof_index
 *   HeatDiffuseMultiPhaseOperator             source/heat/heat_diffuse_operator.cpp:38-80 (ctor)
 *   AdvectionDiffusionOperator                source/level_set/advection_diffusion_operator.cpp
 *   LinearSolver::solve                       include/meltpooldg/linear_algebra/linear_solver.hpp:26-134
 *                                                        -> mpdg_solve
 *   JacobiPreconditioner                      include/meltpooldg/linear_algebra/preconditioner_jacobi.hpp:25-89
 *                                                        -> MPDG_PRECOND_JACOBI in mpdg_solve
 *
 * Conventions
 *  - Vectors are in lexicographic lattice order (x fastest) over the (k m + 1)^3 Gauss-Lobatto
 *    support points of a structured box mesh of axis-aligned hexahedra.  deal.II's DoF numbering
 *    is mapped onto it once by the caller (one permutation of the DoF indices).
 *  - Pointers are DEVICE pointers unless the function name ends in _host.
 *  - vmult zeroes dst; Dirichlet-constrained entries of src are read as 0 and those of dst stay 0
 *    (deal.II MatrixFree semantics).  create_rhs accumulates into dst, reads its inputs plainly
 *    and skips constrained rows.  The inverse diagonal has 1 on constrained rows.
 *  - Every call is stream-ordered on the handle's stream; one host thread per handle.
 *  - Functions return MPDG_OK (0) or an error code; mpdg_last_error() describes the last error of
 *    the calling thread.
 */
#ifndef MPDG_GPU_H
#define MPDG_GPU_H

#include <stdint.h>

#if defined(__GNUC__)
#define MPDG_API __attribute__((visibility("default")))
#else
#define MPDG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum mpdg_status
{
  MPDG_OK                = 0,
  MPDG_ERR_ARG           = 1, /* invalid argument                                          */
  MPDG_ERR_CUDA          = 2, /* CUDA runtime error                                        */
  MPDG_ERR_NOT_CONVERGED = 3, /* SolverControl::NoConvergence (linear_solver.hpp:124-129)   */
  MPDG_ERR_ZERO_DT       = 4, /* ExcZeroTimeIncrement (include/meltpooldg/core/exceptions.hpp:6) */
  MPDG_ERR_TIMEOUT       = 5, /* a bounded device-side wait gave up                        */
  MPDG_ERR_UNSUPPORTED   = 6, /* configuration not provided by this library                */
  MPDG_ERR_NOMEM         = 7  /* device allocation failed                                  */
};

enum mpdg_op_kind
{
  MPDG_HEAT    = 0, /* (rho c_p/dt) M + div(k grad), source/heat/heat_diffuse_operator.cpp      */
  MPDG_ADVDIFF = 1, /* M/dt + theta (v.grad + eps K), source/level_set/advection_diffusion_operator.cpp */
  MPDG_REINIT  = 2  /* M/dt + div(D grad), D = eps_t I + (eps_n - eps_t) n n^T: conservative level-set
                       reinitialisation, source/level_set/olsson_CG_operator.cpp (FE_Q(1..3); set the
                       normal field with mpdg_op_set_reinit) */
};

enum mpdg_solver_kind
{
  MPDG_CG    = 0, /* dealii::SolverCG                          */
  MPDG_GMRES = 1  /* dealii::SolverGMRES, right preconditioning */
};

enum mpdg_precond_kind
{
  MPDG_PRECOND_IDENTITY = 0,
  MPDG_PRECOND_JACOBI   = 1
};

typedef struct mpdg_mesh_desc
{
  int32_t        degree;          /* FE_Q degree: heat 1..4, advection-diffusion 1..3, reinitialisation
                                     1..3 */
  int32_t        cells[3];        /* cells per direction                                */
  double         origin[3];       /* lower corner of the box                            */
  double         length[3];       /* box edge lengths                                   */
  uint32_t       dirichlet_faces; /* homogeneous Dirichlet on whole faces: bit 2d = low face of
                                     dim d, bit 2d+1 = high face                         */
  const uint8_t *dirichlet_mask;  /* optional HOST array of n_dofs flags (nonzero = constrained),
                                     added to the faces; NULL for none                   */
} mpdg_mesh_desc;

typedef struct mpdg_op_params
{
  int32_t       kind;               /* mpdg_op_kind                                            */
  int32_t       reserved;
  /* heat */
  double        rho_cp;             /* density * specific heat capacity                        */
  double        dt;                 /* time increment (must be > 0)                            */
  double        conductivity;       /* k when conductivity_cells == NULL                       */
  const double *conductivity_cells; /* optional HOST array of n_cells per-cell conductivities
                                       (lexicographic cells, x fastest)                      */
  /* advection-diffusion */
  double        theta;              /* one-step-theta: 1 implicit Euler, 0.5 Crank-Nicolson    */
  double        diffusivity;        /* eps                                                      */
  double        velocity[12];       /* affine velocity v(x) = velocity[0..2] + G x with
                                       G = velocity[3..11] row-major                          */
} mpdg_op_params;

typedef struct mpdg_solver_params
{
  int32_t solver;   /* mpdg_solver_kind                                           */
  int32_t precond;  /* mpdg_precond_kind                                          */
  int32_t max_it;   /* ReductionControl max_steps (LinearSolverData default 10000) */
  int32_t restart;  /* GMRES basis size (default 30)                               */
  double  abs_tol;  /* ReductionControl tolerance (default 1e-20)                  */
  double  rel_tol;  /* ReductionControl reduction (default 1e-12)                  */
} mpdg_solver_params;

typedef struct mpdg_solve_info
{
  int32_t iterations;       /* SolverControl::last_step()                               */
  int32_t status;           /* MPDG_OK or MPDG_ERR_NOT_CONVERGED                        */
  double  initial_residual; /* |b - A x0|                                                */
  double  final_residual;   /* last checked residual                                     */
  double *history;          /* optional HOST buffer for residuals 0..iterations (may be NULL) */
  int32_t history_capacity; /* entries available in history                              */
  int32_t inner_iterations; /* mixed precision: total inner FP32 iterations              */
} mpdg_solve_info;

typedef struct mpdg_mixed_params
{
  double  outer_rel_tol;   /* FP64 defect correction: |b - A x| <= outer_rel_tol |b|     */
  double  inner_rel_tol;   /* FP32 Jacobi-CG (or GMRES) reduction per outer step           */
  int32_t max_outer;
  int32_t max_inner;
  int32_t solver;          /* mpdg_solver_kind of the inner solver                         */
  int32_t restart;         /* inner GMRES basis size                                       */
  int32_t inexact_last;    /* 0: every inner solve reduces its residual by inner_rel_tol;
                              1: an inner solve needs no more than the outer tolerance asks
                              for: it stops at max(inner_rel_tol, 0.5 outer_tol / |r|)   */
  int32_t reserved;
} mpdg_mixed_params;

typedef struct mpdg_adjoint_params
{
  int32_t n_steps;          /* implicit-Euler steps                                      */
  int32_t checkpoint_every; /* forward states kept every checkpoint_every steps          */
  double  cg_rel_tol;       /* relative tolerance of every Jacobi-CG solve               */
  int32_t cg_max_it;
  int32_t reserved;
} mpdg_adjoint_params;

typedef struct mpdg_adjoint_result
{
  double  objective;      /* J = 1/2 sum_n |T_n - T*_n|^2 (Euclidean, free DoFs)          */
  double  grad_amplitude; /* dJ/dA                                                        */
  int32_t forward_solves; /* including the recomputation between checkpoints             */
  int32_t adjoint_solves;
  int64_t cg_iterations;
} mpdg_adjoint_result;

typedef struct mpdg_op mpdg_op;

/* Operator lifetime -- HeatDiffuseMultiPhaseOperator / AdvectionDiffusionOperator constructors */
MPDG_API int     mpdg_op_create(const mpdg_mesh_desc *mesh, const mpdg_op_params *params, mpdg_op **out);
MPDG_API int     mpdg_op_destroy(mpdg_op *op);
MPDG_API int64_t mpdg_op_n_dofs(const mpdg_op *op);
MPDG_API int64_t mpdg_op_n_cells(const mpdg_op *op);
MPDG_API int     mpdg_op_set_stream(mpdg_op *op, void *cuda_stream);

/* OperatorBase::reset_time_increment (operator_base.hpp:41-46); dt <= 0 -> MPDG_ERR_ZERO_DT */
MPDG_API int mpdg_op_reset_time_increment(mpdg_op *op, double dt);
/* OperatorBase::reset_dof_index (operator_base.hpp:31-35): 1 = with Dirichlet constraints
   (dof_idx, default), 0 = without (dof_no_bc_idx, used by the Dirichlet lifting of
   include/meltpooldg/linear_algebra/utilities_matrixfree.hpp:33-100) */
MPDG_API int mpdg_op_reset_dof_index(mpdg_op *op, int with_dirichlet);
/* replace the per-cell conductivity (heat); k_cells has n_cells entries (device pointer) */
MPDG_API int mpdg_op_set_conductivity(mpdg_op *op, const double *k_cells);

/* Boundary-face terms of the heat operator on whole box faces (bit 2d = low face of dimension d,
   bit 2d+1 = high face), HeatData's convection / radiation sections and the Neumann map of the
   reference (source/heat/heat_diffuse_operator.cpp: rhs_boundary_loop :719-781, tangent
   :1088-1129, both in vmult :239-264 and in the diagonal :297-357):
     vmult          += int_f (h + 4 eps sigma T^3) u phi            over convection / radiation faces
     create_rhs     -= int_f [eps sigma (T^4 - T_inf^4) + h (T - T_inf) + g.n] phi
     inverse diag   built from diag_i + int_f (h + 4 eps sigma T^3) phi_i^2
   sigma = 5.670374419e-8 (include/meltpooldg/utilities/physical_constants.hpp:6).  g.n is one
   constant normal flux per face (the reference evaluates a Function there).  A face may not carry
   both a Neumann flux and convection / radiation (the reference's AssertThrow, :744-748), nor be a
   Dirichlet face: MPDG_ERR_ARG.  The tangent and the diagonal read T with Dirichlet DoFs as 0, the
   rhs reads T plainly (FEFaceEvaluation gather_evaluate vs read_dof_values_plain). */
typedef struct mpdg_heat_bc
{
  uint32_t convection_faces;
  uint32_t radiation_faces;
  uint32_t neumann_faces;
  uint32_t reserved;
  double   convection_coefficient;          /* HeatData::convection.convection_coefficient */
  double   convection_temperature_infinity; /* HeatData::convection.temperature_infinity   */
  double   emissivity;                      /* HeatData::radiation.emissivity              */
  double   radiation_temperature_infinity;  /* HeatData::radiation.temperature_infinity    */
  double   neumann_flux[6];                 /* g . n on each Neumann face                  */
} mpdg_heat_bc;
MPDG_API int mpdg_op_set_heat_bc(mpdg_op *op, const mpdg_heat_bc *bc);
/* SUPG streamline stabilisation of the advection-diffusion operator (AdvectionDiffusionData::
   conv_stab, source/level_set/advection_diffusion_operator.cpp:455-533): vmult, create_rhs and the
   inverse diagonal add int tau_c (v.grad phi)(u/dt + theta v.grad u - theta eps lap u) (theta - 1 in
   create_rhs), tau_c = (coefficient < 0 ? 1 / max_q |v| (0 if below 1e-6) : coefficient) times the
   cell diameter / sqrt(3), with the affine velocity or the DoF-vector field of
   mpdg_op_set_velocity_field.  enabled = 0 switches it off (ConvectionStabilizationType::none). */
MPDG_API int mpdg_op_set_supg(mpdg_op *op, int enabled, double coefficient);
/* Reinitialisation operator (MPDG_REINIT; source/level_set/olsson_CG_operator.cpp, no wetting
   boundary faces, no interface penalty): normal and tangential diffusion lengths (the reference's
   normal_diffusion_length / tangential_diffusion_length, equal for all cells of a uniform mesh),
   the normalisation tolerance (normalize divides by |n| above it and by the tolerance below,
   include/meltpooldg/utilities/dealii_tensor.hpp:175-191) and the normal field: three DEVICE arrays
   of n_dofs entries on the operator's lattice, read plainly and kept by reference.  vmult applies
   dpsi/dt (mass) + eps_n (grad dpsi . n) n + eps_t (grad dpsi - (grad dpsi . n) n) (:438-470);
   create_rhs(dst, psi_old) OVERWRITES dst with int [(1 - psi_old^2)/2 n - D grad psi_old] . grad phi
   and zeroes the constrained rows (:197-260); the inverse diagonal uses the advection rule
   (:357-436). */
MPDG_API int mpdg_op_set_reinit(mpdg_op *op, double eps_normal, double eps_tangential, double normal_tolerance,
                                const double *nx, const double *ny, const double *nz);

/* Right-hand sides of the level set's projections, FE_Q(1..3), on the lattice and constraint set of
   op (any kind; the projection itself is M + damping K, a heat operator with rho_cp = dt = 1 and
   conductivity = the reference's cell-size-dependent damping, solved per component), no narrow band:
   - NormalVectorOperator::create_rhs (source/level_set/normal_vector_operator.cpp:160-240):
     n_d += int (grad psi)_d phi, or the gradient normalised (|.| > 1e-16, else divided by 1e-16) when
     normalized != 0; accumulating, psi read plainly;
   - CurvatureOperator::create_rhs (source/level_set/curvature_operator.cpp:190-255):
     dst = -int div(n) phi with n = normalize(n_i, normal_tolerance) applied to every DoF value of
     the normal field first; dst overwritten.
   Constrained rows are not written (stay 0 in the curvature rhs). */
MPDG_API int mpdg_level_set_normal_rhs(mpdg_op *op, const double *psi, int normalized, double *nx, double *ny,
                                       double *nz);
MPDG_API int mpdg_level_set_curvature_rhs(mpdg_op *op, const double *nx, const double *ny, const double *nz,
                                          double normal_tolerance, double *dst);
/* Narrow band of the normal-vector and curvature projections (NormalVectorData / CurvatureData
   ::narrow_band, include/meltpooldg/level_set/level_set_tools.hpp:357-368): on a heat handle used as
   the projection operator (rho_c_p = dt = 1, conductivity = the damping), every integrand is
   multiplied at each Gauss point by 1 where |level_set(x_q)| < threshold and 0 elsewhere -- the
   operator's mass and stiffness terms (vmult, inverse diagonal, normal_vector_operator.cpp:326-358,
   inverted with the relative rule of :318-321), the gradient in mpdg_level_set_normal_rhs (masked
   by |psi|, :184-191) and the divergence in mpdg_level_set_curvature_rhs (masked by |level_set|,
   curvature_operator.cpp:209-214).  level_set: DEVICE array of n_dofs the caller keeps alive
   (read plainly); NULL or threshold <= 0 removes the band.  Constant conductivity, Dirichlet faces
   only. */
MPDG_API int mpdg_op_set_narrow_band(mpdg_op *op, const double *level_set, double threshold);
/* Wetting boundary faces of the reinitialisation operator (OlssonOperator's boundary loops with
   wetting_bc_ids, source/level_set/olsson_CG_operator.cpp:550-716): on the box faces in `faces`
   (bit 2d low / 2d+1 high face of dim d) vmult adds int (D grad u . n_f) phi and create_rhs adds
   -int (-c(psi) n + D grad psi) . n_f phi, D = eps_n n n^T + eps_t (I - n n^T), c(psi) = (1 - psi^2)/2,
   n the unit interface normal, n_f the outward face normal; the inverse diagonal includes the
   faces' terms of the wetting faces (the reference's diagonal adds those of every boundary face
   when its face integrals are on, :377-405).  0 removes them. */
MPDG_API int mpdg_op_set_wetting(mpdg_op *op, uint32_t faces);
/* Advection velocity as a finite-element DoF vector (AdvectionDiffusionOperator with
   advection_velocity, source/level_set/advection_diffusion_operator.cpp:461-466, 475-479): three
   DEVICE arrays of n_dofs, the components of an FE_Q(k) field on the operator's lattice, kept by
   reference (the caller keeps them alive and current) and read plainly per cell; they replace the
   affine velocity of mpdg_op_params in vmult, create_rhs, the inverse diagonal and the inflow
   detection of mpdg_op_set_inflow_outflow, and in the SUPG terms of mpdg_op_set_supg (tau_c's
   max_q |v| included, :510-520).  All NULL returns to the affine velocity.  FE_Q degree 1..3.
   On a heat operator the field is its convection velocity (HeatDiffuseOperator with velocity,
   source/heat/heat_diffuse_operator.cpp:448-453, 499-500, 1038-1041): vmult adds
   int rho c_p (v . grad u) phi, create_rhs subtracts int rho c_p (v . grad T) phi, and the inverse
   diagonal includes the term (heat inversion rule); with a constant conductivity and material only
   (no per-cell k, no temperature-dependent material, no narrow band). */
MPDG_API int mpdg_op_set_velocity_field(mpdg_op *op, const double *vx, const double *vy, const double *vz);
/* Inflow/outflow condition of the advection-diffusion operator
   (AdvectionDiffusionOperation::create_inflow_outflow_constraints,
   source/level_set/advection_diffusion_operation.cpp:369-499, with the operator's set_inflow_outflow_bc
   and do_pre_vmult / do_post_vmult, source/level_set/advection_diffusion_operator.cpp:536-578).
   faces: 6-bit mask of the box faces that carry the condition (bit 2d low / 2d+1 high face of dim d,
   0 removes it).  Every support point of such a face where the outward normal n and the velocity v
   satisfy n . v <= 0 is an inflow DoF (Dirichlet DoFs excluded); values: DEVICE array of n_dofs
   holding the condition's function at the lattice points, read at the inflow DoFs during this call.
   With the condition set, vmult treats the inflow DoFs as identity rows (src reads 0 there, dst_i =
   src_i), the inverse diagonal is 1 there, and mpdg_op_create_rhs_and_apply_dirichlet lifts the
   inflow values as additional inhomogeneous constraints (its apply runs without the hooks) and
   zeroes those rows of the right-hand side.  mpdg_op_distribute_inflow writes the values into x
   (the solve's last step, advection_diffusion_operation.cpp:288-296); mpdg_op_n_inflow counts the
   inflow DoFs; mpdg_op_set_inflow_outflow_pre_post switches the vmult / diagonal hooks
   (set_apply_inflow_outflow_constraints_pre_post_matrix_free). */
MPDG_API int     mpdg_op_set_inflow_outflow(mpdg_op *op, uint32_t faces, const double *values);
MPDG_API int64_t mpdg_op_n_inflow(const mpdg_op *op);
MPDG_API int     mpdg_op_set_inflow_outflow_pre_post(mpdg_op *op, int enabled);
MPDG_API int     mpdg_op_distribute_inflow(mpdg_op *op, double *x);

/* The linearisation temperature of the radiation tangent and diagonal (the operator's const
   reference to the temperature vector, heat_diffuse_operator.hpp:121-135): a DEVICE array of
   n_dofs entries that the caller keeps alive and current; NULL detaches it.  vmult and the
   inverse diagonal of an operator with radiation faces and no temperature return MPDG_ERR_ARG. */
MPDG_API int mpdg_op_set_temperature(mpdg_op *op, const double *temperature);

/* Temperature-dependent material of the heat operator, MaterialTypes::liquid_solid without latent
   heat (include/meltpooldg/core/material.templates.hpp:296-360, :540-620, :748-765), FE_Q(1..3):
   solid fraction f_s = clamp((T_liquidus - T) / (T_liquidus - T_solidus), 0, 1) (mushy zone) or
   T < T_solidus (sharp); rho, c_p and k blend cubically, v_l + (v_s - v_l)(3 f_s^2 - 2 f_s^3).
   With it vmult applies the solidification tangent (source/heat/heat_diffuse_operator.cpp:1029-1050)
     (rho c_p(T) / dt + d(rho c_p)/dT (T - T_old) / dt) u,  k(T) grad u + dk/dT grad T u
   at the temperature of mpdg_op_set_temperature and the old temperature of
   mpdg_op_set_old_temperature (both read plainly); create_rhs(dst, T, T_old, q) adds
   M q - int rho c_p(T) (T - T_old) / dt phi - int k(T) grad T . grad phi (:485-527); the inverse
   diagonal is the tangent's.  rho_cp and the conductivity of mpdg_op_params are then unused.
   NULL switches it off. */
typedef struct mpdg_solid_liquid
{
  double  liquid_density, liquid_specific_heat, liquid_conductivity;
  double  solid_density, solid_specific_heat, solid_conductivity;
  double  liquidus_temperature, solidus_temperature;
  int32_t sharp; /* SolidLiquidPropertiesTransitionType: 0 mushy_zone, 1 sharp */
  int32_t reserved;
  /* latent heat of fusion per unit mass (MaterialData::latent_heat_of_fusion, material.hpp:654-655);
     > 0 adds the apparent capacity of the mushy zone to the specific heat
     (material.templates.hpp:561-614, source/heat/apparent_capacity.cpp:157-300) */
  double  latent_heat;
  int32_t capacity_type; /* 0 quadratic-linear-quadratic tent (the default), 1 quartic bell, 2 constant */
  int32_t reserved2;
} mpdg_solid_liquid;
MPDG_API int mpdg_op_set_solidification(mpdg_op *op, const mpdg_solid_liquid *material);
MPDG_API int mpdg_op_set_old_temperature(mpdg_op *op, const double *temperature_old);

/* OperatorMatrixFree::vmult (operator_base.hpp:239-243): dst = A src (FP64 / FP32) */
MPDG_API int mpdg_op_vmult(mpdg_op *op, double *dst, const double *src);
MPDG_API int mpdg_op_vmult_f32(mpdg_op *op, float *dst, const float *src);
/* vmult with host buffers: host->device copy, apply, device->host copy (end-to-end call) */
MPDG_API int mpdg_op_vmult_host(mpdg_op *op, double *dst_host, const double *src_host);
/* dst += scale A src (no zeroing) */
MPDG_API int mpdg_op_vmult_add(mpdg_op *op, double *dst, const double *src, double scale);
/* r = b - A x */
MPDG_API int mpdg_op_residual(mpdg_op *op, double *r, const double *b, const double *x);

/* OperatorMatrixFree::compute_inverse_diagonal_from_matrixfree (operator_base.hpp:268-272) */
MPDG_API int mpdg_op_compute_inverse_diagonal(mpdg_op *op, double *diag);
MPDG_API int mpdg_op_compute_inverse_diagonal_f32(mpdg_op *op, float *diag);

/* OperatorMatrixFree::create_rhs (operator_base.hpp:208-212), accumulating into dst.
   heat (heat_diffuse_operator.cpp:393-529, 783-806):
     dst += -[(rho c_p/dt)(T - T_old) - q] phi - k grad T . grad phi    (a = T, b = T_old, c = q)
   advection-diffusion (advection_diffusion_operator.cpp:274-358):
     dst += (u_old/dt - (1-theta) v.grad u_old) phi - (1-theta) eps grad u_old . grad phi (a = u_old) */
MPDG_API int mpdg_op_create_rhs(mpdg_op *op, double *dst, const double *a, const double *b, const double *c);

/* LinearSolver::solve (linear_solver.hpp:26-134) on the operator: FP64, device x (initial guess
   in, solution out) and b.  Returns MPDG_ERR_NOT_CONVERGED like SolverControl::NoConvergence. */
MPDG_API int mpdg_solve(mpdg_op *op, double *x, const double *b, const mpdg_solver_params *params, mpdg_solve_info *info);
/* The same solve entirely in FP32 (operator, vectors; dot products accumulated in FP64) */
MPDG_API int mpdg_solve_f32(mpdg_op *op, float *x, const float *b, const mpdg_solver_params *params, mpdg_solve_info *info);

/* FP32-inner / FP64-outer defect correction (no reference counterpart: the reference instantiates
   double only, heat_diffuse_operator.cpp:1214-1216).  Outer: r = b - A64 x in FP64, stop when
   |r| <= outer_rel_tol |b|; inner: FP32 operator and vectors with Jacobi preconditioning solve
   A32 e = r to inner_rel_tol; x += e in FP64. */
MPDG_API int mpdg_solve_mixed(mpdg_op *op, double *x, const double *b, const mpdg_mixed_params *params, mpdg_solve_info *info);

/* Transient heat problem on a heat operator (rho c_p and dt from the operator, conductivity
   k = exp(log_k) per cell, overwriting the operator's conductivity):
     (rho c_p M / dt + K(k)) T_n = rho c_p M T_{n-1} / dt + A M qhat_n,  n = 1..n_steps,  T_0 = 0,
   i.e. the implicit-Euler step of the heat equation with source A qhat_n read like the heat_source
   of source/heat/heat_diffuse_operator.cpp:445-447,493-495.  No reference counterpart (the reference
   has no adjoint).  Device arrays: log_k (n_cells), qhat (n_steps * n_dofs), T_target (n_steps *
   n_dofs), grad_log_k (n_cells).
   mpdg_adjoint_heat: J and its gradient by the discrete adjoint (A^T lam_n = (T_n - T*_n) + rho c_p
   M lam_{n+1} / dt, dJ/dz_c = -sum_n k_c lam_n^T K_c T_n, dJ/dA = sum_n lam_n^T M qhat_n), with the
   forward states checkpointed every checkpoint_every steps and recomputed between checkpoints.
   grad_log_k == NULL evaluates J only. */
MPDG_API int mpdg_adjoint_heat(mpdg_op *op, const double *log_k, const double *qhat, double amplitude,
                               const double *T_target, const mpdg_adjoint_params *params, double *grad_log_k,
                               mpdg_adjoint_result *result);
/* Forward states T_1..T_n_steps of the same problem into T_out (n_steps * n_dofs, device). */
MPDG_API int mpdg_heat_forward(mpdg_op *op, const double *log_k, const double *qhat, double amplitude,
                               const mpdg_adjoint_params *params, double *T_out);
/* Per-cell unit-conductivity stiffness form form_c = lam_c^T K_c T_c (device arrays). */
MPDG_API int mpdg_heat_cell_stiffness_form(mpdg_op *op, const double *lam, const double *T, double *form);

/* Allocation-free heat vmult.  No counterpart in the reference (the reference allocates through
   deal.II and never runs on a GPU).  Some callers must not allocate device memory at all: a host
   application that reserves its whole HBM budget up front in its own pool (where a cudaMalloc can
   fail or fragment that pool), and latency-bound time loops in which cudaMalloc / cudaFree would
   synchronise the device.  This entry point computes dst = A src exactly like mpdg_op_vmult on an
   operator built from the same mesh and parameters, without an operator handle and without any
   device allocation: the launch bookkeeping (brick ticket, per-brick flags, wait error word) lives
   in a fixed 256 KiB array in the library's device memory, held by every GPU that loads the
   library until the process exits.
     - mesh: Dirichlet faces only (dirichlet_mask must be NULL); FE_Q degree 1..4.
     - params: kind MPDG_HEAT; params->conductivity_cells must be NULL; a per-cell conductivity is
       passed as the DEVICE array k_cells_dev (n_cells entries) or NULL for params->conductivity.
     - dst, src: distinct device arrays of n_dofs entries; cuda_stream: a cudaStream_t of the
       current device (NULL = legacy default stream).
     - Meshes that need more than MPDG_NOALLOC_MAX_BRICKS brick flags are rejected with
       MPDG_ERR_UNSUPPORTED before any GPU work and before dst / src are looked at (the brick is
       32x4x16 cells at degree 1, 32x4x8 at degree 2, 32x2x4 at degrees 3 and 4; e.g. 160^3 cells
       of degree 4 still fit).
     - The first call on a device does the set-up: it looks up the scratch address on the current
       device and loads the interpolation tables; make that first call before any stream capture.
     - Every call clears the ticket and flags it uses (stream-ordered, before its kernel).  All calls
       on a device share the one array, so calls that overlap on the GPU (different streams or host
       threads without ordering) race and give wrong results: order them.
     - A bounded device wait that gives up records an error word in the scratch array; read it
       with mpdg_heat_vmult_noalloc_errors after the call (every call clears it first). */
#define MPDG_NOALLOC_SCRATCH_BYTES (256 * 1024)
#define MPDG_NOALLOC_MAX_BRICKS ((MPDG_NOALLOC_SCRATCH_BYTES - 256) / 4)
MPDG_API int mpdg_heat_vmult_noalloc(const mpdg_mesh_desc *mesh, const mpdg_op_params *params,
                                     const double *k_cells_dev, double *dst, const double *src, void *cuda_stream);
/* The error word of the allocation-free vmult on the current device, read after the work already
   enqueued on cuda_stream (the call synchronises that stream) and then cleared: 0 when every bounded
   wait of the last call ended normally, nonzero when one gave up (that call's dst is then not
   valid).  Copies from and to the fixed scratch array; allocates nothing. */
MPDG_API int mpdg_heat_vmult_noalloc_errors(void *cuda_stream, int *error_word);

/* create_rhs_and_apply_dirichlet_matrixfree (include/meltpooldg/linear_algebra/utilities_matrixfree.hpp:33-100):
   with the Dirichlet constraints switched off (the no-BC DoF set), temp = -A x_D + create_rhs(a, b, c)
   where x_D holds dirichlet_values on the constrained DoFs and 0 elsewhere (constraints.distribute on
   a zero vector); then rhs = temp (zero_out != 0) or rhs += temp, and the constrained rows of rhs are
   set to 0.  All arrays are device arrays of n_dofs entries; b, c may be NULL as in create_rhs. */
MPDG_API int mpdg_op_create_rhs_and_apply_dirichlet(mpdg_op *op, double *rhs, const double *a, const double *b,
                                                    const double *c, const double *dirichlet_values, int zero_out);

/* Vector operations on the handle's stream over n_dofs entries (device arrays), as used by the
   reference's Newton loop on distributed vectors (source/linear_algebra/newton_raphson_solver.cpp:
   rhs = 0 and solution_update = 0 at :163-164, solution += solution_update at :75, l2_norm in
   is_converged at :121-122).  mpdg_vec_axpby: y = a x + b y (x == NULL means 0).  mpdg_vec_norm:
   Euclidean norm, deterministic (fixed summation order), written to *out (host). */
MPDG_API int mpdg_vec_fill(mpdg_op *op, double *x, double value);
MPDG_API int mpdg_vec_axpby(mpdg_op *op, double *y, double a, const double *x, double b);
MPDG_API int mpdg_vec_norm(mpdg_op *op, const double *x, double *out);
/* x . y, deterministic, written to *out (host); the Gram-Schmidt dots of the least-squares
   projection predictor (include/meltpooldg/linear_algebra/predictor.hpp:37-66) */
MPDG_API int mpdg_vec_dot(mpdg_op *op, const double *x, const double *y, double *out);
/* AffineConstraints::distribute for Dirichlet values held in a vector: dst = values on the DoFs
   constrained by the operator's current constraint set, other entries untouched
   (source/heat/heat_diffuse_operation.cpp:249 after the predictor) */
MPDG_API int mpdg_op_distribute_constraints(mpdg_op *op, double *dst, const double *values);
/* A device vector of n_dofs doubles, zero-filled on the handle's stream, for host layers that do
   not link the CUDA runtime themselves (solution history, predictor work vectors). */
MPDG_API int mpdg_vec_alloc(mpdg_op *op, double **x);
MPDG_API int mpdg_vec_free(double *x);

/* The error code recorded by a bounded device wait that gave up (1) or by a stale brick ticket (2)
   since the last call, 0 when none; reading resets it. */
MPDG_API int mpdg_op_device_errors(mpdg_op *op);

/* Failure injection for tests; no counterpart in the reference (its MPI ranks have no device-side
   waits).  The apply kernels deal bricks out through a ticket counter and wait, bounded, for the
   per-brick flags of their lower neighbours; these hooks make such a wait run out on purpose
   without faulting or hanging the GPU.
   mpdg_op_test_set_wait_limit: sleeps (about 32 ns each) before a wait of this handle's kernels gives
   up and records its error word; 0 restores the default (2^22).
   mpdg_op_test_set_ticket: writes the brick ticket counter, stream-ordered and synchronised, as a
   counter left behind by an aborted launch would look.  A following apply deals out bricks from
   that value on: bricks below it are never processed, so their upper neighbours' waits give up, and
   tickets past the last brick are reported and skipped.  The last CTA of that launch resets the
   counter, so later launches are normal again.
   mpdg_op_n_bricks: bricks of the handle's FP64 apply (the range of useful ticket values). */
MPDG_API int mpdg_op_test_set_wait_limit(mpdg_op *op, unsigned spins);
/* Selects the implementation of the Jacobi-CG iteration behind mpdg_solve / mpdg_solve_f32 / the
   inner solves of mpdg_solve_mixed (LinearSolver::solve with SolverCG, linear_solver.hpp:106-110):
   fused != 0 (the default) runs one sweep per iteration where the operator allows it (heat, FE_Q(2),
   Dirichlet on whole faces only, no boundary-face terms, constant material): the vector updates, the
   preconditioner, the operator apply and the dot products of an iteration in one launch, with the
   next step lengths from a recurrence of the dot products.  fused == 0 runs the three-pass
   iteration (p update, apply with the fused p.Ap, x/r update).  Both follow SolverCG's iterates and
   ReductionControl's test. */
MPDG_API int mpdg_op_set_cg_variant(mpdg_op *op, int fused);
MPDG_API int mpdg_op_test_set_ticket(mpdg_op *op, unsigned value);
MPDG_API int mpdg_op_n_bricks(const mpdg_op *op);

/* Description of the last error on the calling thread. */
MPDG_API const char *mpdg_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* MPDG_GPU_H */
