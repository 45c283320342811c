// mpdg.hpp -- header-only C++17 host layer over the C ABI of libmpdg_b200 (include/mpdg_gpu.h).
//
// It mirrors the reference's host-side classes for the matrix-free hot path so that a C++ caller
// drives the B200 operators the way MeltPoolDG drives its deal.II operators:
//
//   OperatorMatrixFree          include/meltpooldg/core/operator_base.hpp:189-283
//   HeatDiffuseOperator         source/heat/heat_diffuse_operator.cpp (single phase)
//   AdvectionDiffusionOperator  source/level_set/advection_diffusion_operator.cpp
//   LinearSolverData            include/meltpooldg/linear_algebra/linear_solver_data.hpp:37-47
//   LinearSolver::solve         include/meltpooldg/linear_algebra/linear_solver.hpp:26-134
//   NonlinearSolverData         include/meltpooldg/linear_algebra/nonlinear_solver_data.hpp:11-25
//   NewtonRaphsonSolver         source/linear_algebra/newton_raphson_solver.cpp:22-165
//   HeatDiffuseOperation        source/heat/heat_diffuse_operation.cpp:86-102, 213-289 (the Newton
//                               time step of the heat equation, predictor "none")
//
// Vectors are device arrays of n_dofs() doubles in lexicographic lattice order, owned by the
// caller.  Errors become exceptions as in the reference: SolverControl::NoConvergence ->
// mpdg::NoConvergence, ExcZeroTimeIncrement -> mpdg::ZeroTimeIncrement, ExcNewtonDidNotConverge ->
// mpdg::NewtonDidNotConverge, everything else mpdg::Error with mpdg_last_error() as the message.
#pragma once

#include <cstdint>
#include <functional>
#include <stdexcept>
#include <string>
#include <utility>

#include "mpdg_gpu.h"

namespace mpdg
{
  class Error : public std::runtime_error
  {
  public:
    Error(int code, const std::string &msg)
      : std::runtime_error(msg)
      , code(code)
    {}
    int code;
  };

  class NoConvergence : public Error
  {
  public:
    NoConvergence(int iterations, double residual, const std::string &msg)
      : Error(MPDG_ERR_NOT_CONVERGED, msg)
      , last_step(iterations)
      , last_residual(residual)
    {}
    int    last_step;
    double last_residual;
  };

  class ZeroTimeIncrement : public Error
  {
  public:
    using Error::Error;
  };

  class NewtonDidNotConverge : public Error
  {
  public:
    using Error::Error;
  };

  inline void
  check(int rc)
  {
    if (rc == MPDG_OK)
      return;
    const std::string msg = mpdg_last_error();
    if (rc == MPDG_ERR_ZERO_DT)
      throw ZeroTimeIncrement(rc, msg);
    throw Error(rc, msg);
  }

  // ---- operators ---------------------------------------------------------------------------------
  class OperatorMatrixFree
  {
  public:
    OperatorMatrixFree(const mpdg_mesh_desc &mesh, const mpdg_op_params &params)
    {
      check(mpdg_op_create(&mesh, &params, &op_));
    }
    OperatorMatrixFree(const OperatorMatrixFree &) = delete;
    OperatorMatrixFree &operator=(const OperatorMatrixFree &) = delete;
    OperatorMatrixFree(OperatorMatrixFree &&o) noexcept
      : op_(std::exchange(o.op_, nullptr))
    {}
    virtual ~OperatorMatrixFree()
    {
      if (op_)
        mpdg_op_destroy(op_);
    }

    int64_t
    n_dofs() const
    {
      return mpdg_op_n_dofs(op_);
    }
    void
    set_stream(void *cuda_stream)
    {
      check(mpdg_op_set_stream(op_, cuda_stream));
    }
    // operator_base.hpp:41-46
    void
    reset_time_increment(double dt)
    {
      check(mpdg_op_reset_time_increment(op_, dt));
    }
    // operator_base.hpp:31-35 (true: Dirichlet constraints, false: the no-BC DoF set)
    void
    reset_dof_index(bool with_dirichlet)
    {
      check(mpdg_op_reset_dof_index(op_, with_dirichlet ? 1 : 0));
    }
    // operator_base.hpp:239-243
    void
    vmult(double *dst, const double *src) const
    {
      check(mpdg_op_vmult(op_, dst, src));
    }
    void
    vmult(float *dst, const float *src) const
    {
      check(mpdg_op_vmult_f32(op_, dst, src));
    }
    // dst += scale * A src
    void
    vmult_add(double *dst, const double *src, double scale = 1.0) const
    {
      check(mpdg_op_vmult_add(op_, dst, src, scale));
    }
    // r = b - A x
    void
    residual(double *r, const double *b, const double *x) const
    {
      check(mpdg_op_residual(op_, r, b, x));
    }
    // operator_base.hpp:208-212 (accumulating; heat: a = T, b = T_old, c = q; advection: a = u_old)
    void
    create_rhs(double *dst, const double *a, const double *b = nullptr, const double *c = nullptr) const
    {
      check(mpdg_op_create_rhs(op_, dst, a, b, c));
    }
    // utilities_matrixfree.hpp:33-100 (x_D = dirichlet_values on constrained DoFs)
    void
    create_rhs_and_apply_dirichlet(double *rhs, const double *a, const double *dirichlet_values,
                                   const double *b = nullptr, const double *c = nullptr, bool zero_out = true) const
    {
      check(mpdg_op_create_rhs_and_apply_dirichlet(op_, rhs, a, b, c, dirichlet_values, zero_out ? 1 : 0));
    }
    // operator_base.hpp:268-272
    void
    compute_inverse_diagonal_from_matrixfree(double *diag) const
    {
      check(mpdg_op_compute_inverse_diagonal(op_, diag));
    }
    // vector operations on the operator's stream (n_dofs entries)
    void
    fill(double *x, double value) const
    {
      check(mpdg_vec_fill(op_, x, value));
    }
    void
    axpby(double *y, double a, const double *x, double b) const
    {
      check(mpdg_vec_axpby(op_, y, a, x, b));
    }
    double
    l2_norm(const double *x) const
    {
      double n = 0.0;
      check(mpdg_vec_norm(op_, x, &n));
      return n;
    }
    mpdg_op *
    handle() const
    {
      return op_;
    }

  private:
    mpdg_op *op_ = nullptr;
  };

  class HeatDiffuseOperator : public OperatorMatrixFree
  {
  public:
    static mpdg_op_params
    params(double rho_cp, double dt, double conductivity, const double *conductivity_cells_host)
    {
      mpdg_op_params p{};
      p.kind               = MPDG_HEAT;
      p.rho_cp             = rho_cp;
      p.dt                 = dt;
      p.conductivity       = conductivity;
      p.conductivity_cells = conductivity_cells_host;
      return p;
    }
    HeatDiffuseOperator(const mpdg_mesh_desc &mesh, double rho_cp, double dt, double conductivity,
                        const double *conductivity_cells_host = nullptr)
      : OperatorMatrixFree(mesh, params(rho_cp, dt, conductivity, conductivity_cells_host))
    {}
    // per-cell conductivity (device array of n_cells entries)
    void
    set_conductivity(const double *k_cells)
    {
      check(mpdg_op_set_conductivity(handle(), k_cells));
    }
    // HeatData's convection / radiation sections and constant Neumann fluxes on box faces
    void
    set_boundary_conditions(const mpdg_heat_bc &bc)
    {
      check(mpdg_op_set_heat_bc(handle(), &bc));
    }
    // the temperature the radiation tangent is linearised at (device array, kept by reference)
    void
    set_temperature(const double *temperature)
    {
      check(mpdg_op_set_temperature(handle(), temperature));
    }
  };

  class AdvectionDiffusionOperator : public OperatorMatrixFree
  {
  public:
    static mpdg_op_params
    params(double dt, double theta, double diffusivity, const double velocity[12])
    {
      mpdg_op_params p{};
      p.kind        = MPDG_ADVDIFF;
      p.dt          = dt;
      p.theta       = theta;
      p.diffusivity = diffusivity;
      for (int i = 0; i < 12; ++i)
        p.velocity[i] = velocity[i];
      return p;
    }
    AdvectionDiffusionOperator(const mpdg_mesh_desc &mesh, double dt, double theta, double diffusivity,
                               const double velocity[12])
      : OperatorMatrixFree(mesh, params(dt, theta, diffusivity, velocity))
    {}
  };

  // ---- linear solver -----------------------------------------------------------------------------
  struct LinearSolverData
  {
    int    solver_type         = MPDG_GMRES; // the reference's default solver type
    int    preconditioner_type = MPDG_PRECOND_IDENTITY;
    int    max_iterations      = 10000;
    double rel_tolerance       = 1e-12;
    double abs_tolerance       = 1e-20;
    int    restart             = 30;
  };

  struct LinearSolver
  {
    // returns the number of iterations (last_step()); throws NoConvergence like linear_solver.hpp:124-129
    static int
    solve(const OperatorMatrixFree &op, double *solution, const double *rhs, const LinearSolverData &d)
    {
      mpdg_solver_params p{};
      p.solver  = d.solver_type;
      p.precond = d.preconditioner_type;
      p.max_it  = d.max_iterations;
      p.restart = d.restart;
      p.abs_tol = d.abs_tolerance;
      p.rel_tol = d.rel_tolerance;
      mpdg_solve_info info{};
      const int       rc = mpdg_solve(op.handle(), solution, rhs, &p, &info);
      if (rc == MPDG_ERR_NOT_CONVERGED)
        throw NoConvergence(info.iterations, info.final_residual, mpdg_last_error());
      check(rc);
      return info.iterations;
    }
  };

  // ---- Newton-Raphson ----------------------------------------------------------------------------
  struct NonlinearSolverData
  {
    int    max_nonlinear_iterations       = 10;
    double field_correction_tolerance     = 1e-10;
    double residual_tolerance             = 1e-9;
    int    max_nonlinear_iterations_alt   = 0;
    double field_correction_tolerance_alt = 1e-9;
    double residual_tolerance_alt         = 1e-8;
    bool   use_relative_tolerances        = false;
  };

  // newton_raphson_solver.cpp:22-165.  The caller provides the residual and Jacobian-solve rules and
  // two work vectors (rhs, solution update) of n_dofs() entries; vector operations run through op.
  class NewtonRaphsonSolver
  {
  public:
    NewtonRaphsonSolver(const NonlinearSolverData &data, const OperatorMatrixFree &op, double *rhs,
                        double *solution_update)
      : data_(data)
      , op_(op)
      , rhs_(rhs)
      , du_(solution_update)
    {}

    std::function<void(const double *evaluation_point, double *rhs)>    residual;
    std::function<int(const double *rhs, double *solution_update)>      solve_with_jacobian;
    std::function<void(double *solution)>                               distribute_constraints;

    void
    solve(double *solution)
    {
      if (!residual || !solve_with_jacobian)
        throw Error(MPDG_ERR_ARG, "NewtonRaphsonSolver: residual and solve_with_jacobian must be set");
      double    res_tol = data_.residual_tolerance, cor_tol = data_.field_correction_tolerance;
      const int max_it  = data_.max_nonlinear_iterations + data_.max_nonlinear_iterations_alt;
      double    r0      = 0.0;
      linear_iterations = 0;
      for (int i = 0; i < max_it; ++i)
        {
          if (i == data_.max_nonlinear_iterations)
            {
              res_tol = data_.residual_tolerance_alt;
              cor_tol = data_.field_correction_tolerance_alt;
            }
          // solve_increment (:160-165)
          op_.fill(rhs_, 0.0);
          op_.fill(du_, 0.0);
          residual(solution, rhs_);
          linear_iterations += solve_with_jacobian(rhs_, du_);
          // is_converged (:116-150)
          double res_norm = op_.l2_norm(rhs_), upd_norm = op_.l2_norm(du_);
          if (i == 0)
            r0 = res_norm;
          if (data_.use_relative_tolerances)
            {
              if (r0 > 0.0)
                res_norm /= r0;
              const double sol_norm = op_.l2_norm(solution);
              if (sol_norm > 0.0)
                upd_norm /= sol_norm;
            }
          last_residual = res_norm;
          if (res_norm < res_tol && upd_norm < cor_tol)
            {
              iterations = i;
              return;
            }
          op_.axpby(solution, 1.0, du_, 1.0); // solution += solution_update
          if (distribute_constraints)
            distribute_constraints(solution);
        }
      throw NewtonDidNotConverge(MPDG_ERR_NOT_CONVERGED, "Newton-Raphson solver did not converge");
    }

    int    iterations        = 0;
    int    linear_iterations = 0;
    double last_residual     = 0.0;

  private:
    NonlinearSolverData       data_;
    const OperatorMatrixFree &op_;
    double                   *rhs_, *du_;
  };

  // heat_diffuse_operation.cpp:86-102 (Newton rules) and :213-289 (time step), single phase, no
  // predictor (PredictorType::none keeps the current solution as the initial guess).  T, T_old and
  // the work vectors are device arrays of n_dofs() entries; q (heat source, may be null) is read
  // plainly like heat_source in create_rhs.  The operator is linearised at T (its temperature
  // reference, heat_diffuse_operator.hpp:121-135), so radiation faces get the tangent of the
  // current Newton iterate.
  class HeatDiffuseOperation
  {
  public:
    HeatDiffuseOperation(HeatDiffuseOperator &op, double *T, double *T_old, const double *q, double *rhs,
                         double *solution_update, double *zero, const LinearSolverData &linear,
                         const NonlinearSolverData &nonlinear)
      : op_(op)
      , T_(T)
      , T_old_(T_old)
      , q_(q)
      , zero_(zero)
      , linear_(linear)
      , newton_(nonlinear, op, rhs, solution_update)
    {
      op_.fill(zero_, 0.0);
      op_.set_temperature(T_);
      newton_.residual = [this](const double * /*evaluation_point*/, double *rhs) {
        op_.create_rhs(rhs, T_, T_old_, q_ ? q_ : zero_);
      };
      newton_.solve_with_jacobian = [this](const double *rhs, double *du) -> int {
        return LinearSolver::solve(op_, du, rhs, linear_);
      };
    }

    // init_time_advance: reset the time increment and commit the old solution
    void
    init_time_advance(double dt)
    {
      op_.reset_time_increment(dt);
      op_.axpby(T_old_, 1.0, T_, 0.0);
    }

    // solve: Newton on the current time step (ExcNewtonDidNotConverge -> HeatTransferNoConvergence)
    void
    solve()
    {
      newton_.solve(T_);
    }

    const NewtonRaphsonSolver &
    newton() const
    {
      return newton_;
    }

  private:
    HeatDiffuseOperator &op_;
    double              *T_, *T_old_;
    const double        *q_;
    double              *zero_;
    LinearSolverData     linear_;
    NewtonRaphsonSolver  newton_;
  };
} // namespace mpdg
