// The predictors of the heat time step through the C++ host layer (include/mpdg/mpdg.hpp):
// 8 x 8 x 8 FE_Q(2) cells on [0,1]^3, rho c_p = 1, k = 1, Dirichlet on the x = 0 face (T = 1000
// there), convection on the x = 1 face, radiation on the y and z faces, T0 = 1000 - 300 x; five
// implicit-Euler steps with time increments 1e-2, 1e-2, 2e-2, 1e-2, 1.5e-2, each solved by Newton
// with Jacobi-CG.  For each predictor type (none, zero, linear_extrapolation,
// least_squares_projection with 3 old solutions) writes, per step, the predicted temperature (after
// init_time_advance) and the solution (after solve) as n_dofs doubles each to <argv[1]>_<type>.bin.
#include <cuda_runtime.h>

#include <cstdio>
#include <string>
#include <vector>

#include "mpdg/mpdg.hpp"

int
main(int argc, char **argv)
{
  if (argc < 2)
    {
      std::fprintf(stderr, "usage: heat_predictor <output prefix>\n");
      return 2;
    }
  try
    {
      mpdg_mesh_desc mesh{};
      mesh.degree          = 2;
      mesh.cells[0]        = 8, mesh.cells[1] = 8, mesh.cells[2] = 8;
      mesh.length[0]       = 1.0, mesh.length[1] = 1.0, mesh.length[2] = 1.0;
      mesh.dirichlet_faces = 0b000001;
      mpdg::HeatDiffuseOperator op(mesh, 1.0, 1e-2, 1.0);
      mpdg_heat_bc              bc{};
      bc.convection_faces                = 0b000010;
      bc.convection_coefficient          = 10.0;
      bc.convection_temperature_infinity = 300.0;
      bc.radiation_faces                 = 0b111100;
      bc.emissivity                      = 0.6;
      bc.radiation_temperature_infinity  = 300.0;
      op.set_boundary_conditions(bc);
      const int64_t       n = op.n_dofs();
      std::vector<double> T0(n), host(n);
      for (int64_t i = 0; i < n; ++i)
        T0[i] = 1000.0 - 300.0 * (double)(i % 17) / 16.0; // x of the lattice point
      double *T = nullptr, *T_old = nullptr, *rhs = nullptr, *du = nullptr, *zero = nullptr;
      for (double **v : {&T, &T_old, &rhs, &du, &zero})
        if (cudaMalloc(v, sizeof(double) * n) != cudaSuccess)
          throw mpdg::Error(MPDG_ERR_NOMEM, "cudaMalloc");
      mpdg::LinearSolverData lin;
      lin.solver_type         = MPDG_CG;
      lin.preconditioner_type = MPDG_PRECOND_JACOBI;
      lin.rel_tolerance       = 1e-12;
      mpdg::NonlinearSolverData nl;
      nl.residual_tolerance         = 1e-8;
      nl.field_correction_tolerance = 1e-9;
      nl.max_nonlinear_iterations   = 30; // the zero predictor starts every step from 0 K
      const double dts[5] = {1e-2, 1e-2, 2e-2, 1e-2, 1.5e-2};
      const struct
      {
        const char         *name;
        mpdg::PredictorType type;
      } kinds[4] = {{"none", mpdg::PredictorType::none},
                    {"zero", mpdg::PredictorType::zero},
                    {"linear_extrapolation", mpdg::PredictorType::linear_extrapolation},
                    {"least_squares_projection", mpdg::PredictorType::least_squares_projection}};
      for (const auto &kind : kinds)
        {
          cudaMemcpy(T, T0.data(), sizeof(double) * n, cudaMemcpyHostToDevice);
          mpdg::PredictorData pd;
          pd.type                   = kind.type;
          pd.n_old_solution_vectors = 3;
          mpdg::HeatDiffuseOperation heat(op, T, T_old, nullptr, rhs, du, zero, lin, nl, pd);
          const std::string          path = std::string(argv[1]) + "_" + kind.name + ".bin";
          std::FILE                 *f    = std::fopen(path.c_str(), "wb");
          if (!f)
            throw mpdg::Error(MPDG_ERR_ARG, "cannot open the output file");
          int newton_total = 0;
          for (double dt : dts)
            {
              heat.init_time_advance(dt);
              cudaMemcpy(host.data(), T, sizeof(double) * n, cudaMemcpyDeviceToHost);
              std::fwrite(host.data(), sizeof(double), n, f);
              heat.solve();
              cudaMemcpy(host.data(), T, sizeof(double) * n, cudaMemcpyDeviceToHost);
              std::fwrite(host.data(), sizeof(double), n, f);
              newton_total += heat.newton().iterations;
            }
          std::fclose(f);
          std::printf("%s: %d Newton iterations\n", kind.name, newton_total);
        }
      for (double *v : {T, T_old, rhs, du, zero})
        cudaFree(v);
    }
  catch (const mpdg::Error &e)
    {
      std::fprintf(stderr, "error %d: %s\n", e.code, e.what());
      return 1;
    }
  return 0;
}
