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

#include <algorithm>
#include <cstdint>
#include <functional>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

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
    double
    dot(const double *x, const double *y) const
    {
      double d = 0.0;
      check(mpdg_vec_dot(op_, x, y, &d));
      return d;
    }
    // constraints.distribute(dst) with the Dirichlet values held in values
    void
    distribute_constraints(double *dst, const double *values) const
    {
      check(mpdg_op_distribute_constraints(op_, dst, values));
    }
    // NormalVectorOperator::create_rhs (normal_vector_operator.cpp:160-240) on this lattice:
    // n_d += int (grad psi)_d phi, the gradient normalised when normalized is true
    void
    level_set_normal_rhs(const double *psi, double *nx, double *ny, double *nz, bool normalized = false) const
    {
      check(mpdg_level_set_normal_rhs(op_, psi, normalized ? 1 : 0, nx, ny, nz));
    }
    // CurvatureOperator::create_rhs (curvature_operator.cpp:190-255) on this lattice:
    // dst = -int div(n) phi with n normalised at every DoF (overwrites dst)
    void
    level_set_curvature_rhs(double *dst, const double *nx, const double *ny, const double *nz,
                            double normal_tolerance) const
    {
      check(mpdg_level_set_curvature_rhs(op_, nx, ny, nz, normal_tolerance, dst));
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
    // the temperature the radiation and solidification tangents are linearised at (device array,
    // kept by reference)
    void
    set_temperature(const double *temperature)
    {
      check(mpdg_op_set_temperature(handle(), temperature));
    }
    // temperature-dependent material (nullptr switches it off) and the old temperature it needs
    void
    set_solidification(const mpdg_solid_liquid *material)
    {
      check(mpdg_op_set_solidification(handle(), material));
    }
    void
    set_old_temperature(const double *temperature_old)
    {
      check(mpdg_op_set_old_temperature(handle(), temperature_old));
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
    // AdvectionDiffusionData::conv_stab (type SUPG or none, coefficient < 0: h_c / max |v|)
    void
    set_convection_stabilization(bool supg, double coefficient)
    {
      check(mpdg_op_set_supg(handle(), supg ? 1 : 0, coefficient));
    }
  };

  // OlssonOperator (source/level_set/olsson_CG_operator.cpp), default configuration: create_rhs
  // overwrites dst (create_rhs(dst, psi_old)); the normal field is three device arrays kept by
  // reference
  class OlssonOperator : public OperatorMatrixFree
  {
  public:
    static mpdg_op_params
    params(double dt)
    {
      mpdg_op_params p{};
      p.kind = MPDG_REINIT;
      p.dt   = dt;
      return p;
    }
    OlssonOperator(const mpdg_mesh_desc &mesh, double dt)
      : OperatorMatrixFree(mesh, params(dt))
    {}
    void
    set_normal(double eps_normal, double eps_tangential, double normal_tolerance, const double *nx, const double *ny,
               const double *nz)
    {
      check(mpdg_op_set_reinit(handle(), eps_normal, eps_tangential, normal_tolerance, nx, ny, nz));
    }
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

  // A device vector of n_dofs() doubles owned by the host layer (zero-filled).
  class DeviceVector
  {
  public:
    DeviceVector() = default;
    explicit DeviceVector(const OperatorMatrixFree &op)
    {
      check(mpdg_vec_alloc(op.handle(), &p_));
    }
    DeviceVector(DeviceVector &&o) noexcept
      : p_(std::exchange(o.p_, nullptr))
    {}
    DeviceVector &
    operator=(DeviceVector &&o) noexcept
    {
      std::swap(p_, o.p_);
      return *this;
    }
    DeviceVector(const DeviceVector &) = delete;
    DeviceVector &operator=(const DeviceVector &) = delete;
    ~DeviceVector()
    {
      if (p_)
        mpdg_vec_free(p_);
    }
    double *
    get() const
    {
      return p_;
    }

  private:
    double *p_ = nullptr;
  };

  // ---- predictors (include/meltpooldg/linear_algebra/predictor.hpp, predictor_data.hpp) ------------
  enum class PredictorType
  {
    none,
    zero,
    linear_extrapolation,
    least_squares_projection
  };

  struct PredictorData
  {
    PredictorType type                   = PredictorType::none;
    int           n_old_solution_vectors = 2; // least_squares_projection only
  };

  // LeastSquaresProjection::vmult (predictor.hpp:37-84): the combination sum_s c_s x_s of the old
  // solutions x_0 .. x_{n-1} that minimises |A sum_s c_s x_s - rhs|.  The images A x_s are
  // orthogonalised one after the other (Gram-Schmidt against the already orthogonalised ones, with
  // the coefficients P(j, s) / P(j, j)); an image whose remaining squared norm falls below 1e-16 of
  // the first one ends the basis.  The coefficients follow from the upper-triangular system P c = V^T rhs
  // by back substitution.  work holds at least n vectors.
  inline void
  least_squares_projection(const OperatorMatrixFree &A, double *solution, const double *rhs,
                           const std::vector<const double *> &old, const std::vector<double *> &work)
  {
    const int           n = (int)old.size();
    std::vector<double> P((size_t)n * n, 0.0);
    auto                at = [&](int i, int j) -> double & { return P[(size_t)i * n + j]; };
    int                 step = 0;
    for (; step < n; ++step)
      {
        double *v = work[step];
        A.vmult(v, old[step]);
        at(0, step) = A.dot(v, work[0]);
        for (int j = 0; j < step; ++j)
          {
            A.axpby(v, -at(j, step) / at(j, j), work[j], 1.0);
            at(j + 1, step) = A.dot(v, work[j + 1]);
          }
        if (at(step, step) < 1e-16 * at(0, 0))
          break;
      }
    std::vector<double> c(step);
    for (int s = 0; s < step; ++s)
      c[s] = A.dot(work[s], rhs);
    for (int s = step - 1; s >= 0; --s)
      {
        double sum = c[s];
        for (int j = s + 1; j < step; ++j)
          sum -= c[j] * at(s, j);
        c[s] = sum / at(s, s);
      }
    A.axpby(solution, step > 0 ? c[0] : 0.0, old[0], 0.0);
    for (int s = 1; s < step; ++s)
      A.axpby(solution, c[s], old[s], 1.0);
  }

  // heat_diffuse_operation.cpp:86-102 (Newton rules) and :213-289 (time step), single phase.  The
  // solution history holds max(n_old_solution_vectors, 2) vectors (:47-48): T (current), T_old and,
  // for a longer least-squares history, vectors of its own.  init_time_advance runs the predictor
  // (Predictor::vmult, predictor.hpp:118-160): none keeps the current solution, zero starts from 0,
  // linear_extrapolation extrapolates with the ratio of the current to the old time increment
  // (predictor_linear.hpp), least_squares_projection projects once n_old_solution_vectors calls have
  // filled the history (until then it keeps the current solution, as none does: the reference swaps
  // the current solution into the predictor buffer there before committing the history, which would
  // leave the recent old solution zero, and that is not followed).  Then the history is committed
  // (solution_history.hpp:70-77), the prediction becomes the current solution and the Dirichlet
  // values of the previous solution are distributed into it (:249).  T, T_old and
  // the work vectors are device arrays of n_dofs() entries; q (heat source, may be null) is read
  // plainly like heat_source in create_rhs.  The operator is linearised at T (its temperature
  // reference, heat_diffuse_operator.hpp:121-135), so radiation faces get the tangent of the
  // current Newton iterate.
  class HeatDiffuseOperation
  {
  public:
    HeatDiffuseOperation(HeatDiffuseOperator &op, double *T, double *T_old, const double *q, double *rhs,
                         double *solution_update, double *zero, const LinearSolverData &linear,
                         const NonlinearSolverData &nonlinear, const PredictorData &predictor = PredictorData())
      : op_(op)
      , T_(T)
      , T_old_(T_old)
      , q_(q)
      , zero_(zero)
      , linear_(linear)
      , predictor_(predictor)
      , newton_(nonlinear, op, rhs, solution_update)
    {
      op_.fill(zero_, 0.0);
      op_.set_temperature(T_);
      op_.set_old_temperature(T_old_);
      // solution history: every old slot starts as the initial solution (SolutionHistory::apply_old)
      const int n_hist = std::max(predictor_.n_old_solution_vectors, 2);
      history_         = {T_, T_old_};
      for (int i = 2; i < n_hist; ++i)
        {
          owned_.emplace_back(op_);
          history_.push_back(owned_.back().get());
        }
      for (size_t i = 1; i < history_.size(); ++i)
        op_.axpby(history_[i], 1.0, T_, 0.0);
      newton_.residual = [this](const double * /*evaluation_point*/, double *rhs) {
        op_.create_rhs(rhs, T_, T_old_, q_ ? q_ : zero_);
      };
      newton_.solve_with_jacobian = [this](const double *rhs, double *du) -> int {
        return LinearSolver::solve(op_, du, rhs, linear_);
      };
    }

    // init_time_advance (:213-250): reset the time increment, predict, commit the history
    void
    init_time_advance(double dt)
    {
      op_.reset_time_increment(dt);
      dt_old_ = n_calls_ == 0 ? dt : dt_cur_;
      dt_cur_ = dt;
      if (!buffer_.get())
        buffer_ = DeviceVector(op_);
      double *pred = buffer_.get();
      switch (predictor_.type)
        {
          case PredictorType::none:
            op_.axpby(pred, 1.0, T_, 0.0);
            break;
          case PredictorType::zero:
            op_.fill(pred, 0.0);
            break;
          case PredictorType::linear_extrapolation:
            {
              const double r = dt_cur_ / dt_old_;
              op_.axpby(pred, 1.0 + r, T_, 0.0);
              op_.axpby(pred, -r, history_[1], 1.0);
              break;
            }
          case PredictorType::least_squares_projection:
            {
              const int n_old = predictor_.n_old_solution_vectors;
              if (n_calls_ >= n_old)
                {
                  // rhs of the projection: create_rhs at T_old = T (:236-243)
                  if (!lsp_rhs_.get())
                    lsp_rhs_ = DeviceVector(op_);
                  while ((int)lsp_work_.size() < n_old)
                    lsp_work_.emplace_back(op_);
                  op_.fill(lsp_rhs_.get(), 0.0);
                  op_.create_rhs(lsp_rhs_.get(), T_, T_, q_ ? q_ : zero_);
                  std::vector<const double *> old(history_.begin(), history_.begin() + n_old);
                  std::vector<double *>       work;
                  for (auto &w : lsp_work_)
                    work.push_back(w.get());
                  least_squares_projection(op_, pred, lsp_rhs_.get(), old, work);
                }
              else
                op_.axpby(pred, 1.0, T_, 0.0);
              break;
            }
        }
      for (size_t i = history_.size() - 1; i >= 1; --i)
        op_.axpby(history_[i], 1.0, history_[i - 1], 0.0);
      op_.axpby(T_, 1.0, pred, 0.0);
      op_.distribute_constraints(T_, history_[1]);
      ++n_calls_;
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
    HeatDiffuseOperator      &op_;
    double                   *T_, *T_old_;
    const double             *q_;
    double                   *zero_;
    LinearSolverData          linear_;
    PredictorData             predictor_;
    NewtonRaphsonSolver       newton_;
    std::vector<double *>     history_;
    std::vector<DeviceVector> owned_, lsp_work_;
    DeviceVector              buffer_, lsp_rhs_;
    double                    dt_cur_ = 0.0, dt_old_ = 0.0;
    int                       n_calls_ = 0;
  };
} // namespace mpdg
