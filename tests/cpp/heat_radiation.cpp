// Nonlinear heat time steps with radiation and convection faces through the C++ host layer
// (include/mpdg/mpdg.hpp): 8 x 8 x 8 FE_Q(2) cells on [0,1]^3, rho c_p = 1, k = 1, no Dirichlet
// face; convection h = 10, T_inf = 300 on the x faces; radiation emissivity 0.6, T_inf = 300 on
// the y and z faces; T0 = 1000 - 300 x; dt = 1e-2, 3 implicit-Euler steps, each solved by Newton
// (the radiation tangent linearised at the current iterate) with Jacobi-CG (relative 1e-12).
// Writes the temperature after every step (n_dofs doubles per step) to the file argv[1].
#include <cuda_runtime.h>

#include <cstdio>
#include <vector>

#include "mpdg/mpdg.hpp"

int
main(int argc, char **argv)
{
  if (argc < 2)
    {
      std::fprintf(stderr, "usage: heat_radiation <output file>\n");
      return 2;
    }
  try
    {
      mpdg_mesh_desc mesh{};
      mesh.degree   = 2;
      mesh.cells[0] = 8, mesh.cells[1] = 8, mesh.cells[2] = 8;
      mesh.length[0] = 1.0, mesh.length[1] = 1.0, mesh.length[2] = 1.0;
      mpdg::HeatDiffuseOperator op(mesh, 1.0, 1e-2, 1.0);
      mpdg_heat_bc              bc{};
      bc.convection_faces                = 0b000011;
      bc.convection_coefficient          = 10.0;
      bc.convection_temperature_infinity = 300.0;
      bc.radiation_faces                 = 0b111100;
      bc.emissivity                      = 0.6;
      bc.radiation_temperature_infinity  = 300.0;
      op.set_boundary_conditions(bc);
      const int64_t       n = op.n_dofs();
      std::vector<double> T0(n);
      for (int64_t i = 0; i < n; ++i)
        T0[i] = 1000.0 - 300.0 * (double)(i % 17) / 16.0; // x of the lattice point
      double *T = nullptr, *T_old = nullptr, *rhs = nullptr, *du = nullptr, *zero = nullptr;
      for (double **v : {&T, &T_old, &rhs, &du, &zero})
        if (cudaMalloc(v, sizeof(double) * n) != cudaSuccess)
          throw mpdg::Error(MPDG_ERR_NOMEM, "cudaMalloc");
      cudaMemcpy(T, T0.data(), sizeof(double) * n, cudaMemcpyHostToDevice);

      mpdg::LinearSolverData lin;
      lin.solver_type         = MPDG_CG;
      lin.preconditioner_type = MPDG_PRECOND_JACOBI;
      lin.rel_tolerance       = 1e-12;
      mpdg::NonlinearSolverData nl;
      nl.residual_tolerance         = 1e-8;
      nl.field_correction_tolerance = 1e-9;
      mpdg::HeatDiffuseOperation heat(op, T, T_old, nullptr, rhs, du, zero, lin, nl);

      std::FILE *f = std::fopen(argv[1], "wb");
      if (!f)
        throw mpdg::Error(MPDG_ERR_ARG, "cannot open the output file");
      std::vector<double> host(n);
      for (int step = 0; step < 3; ++step)
        {
          heat.init_time_advance(1e-2);
          heat.solve();
          cudaMemcpy(host.data(), T, sizeof(double) * n, cudaMemcpyDeviceToHost);
          std::fwrite(host.data(), sizeof(double), n, f);
          std::printf("step %d: %d Newton iterations, %d linear iterations\n", step + 1, heat.newton().iterations,
                      heat.newton().linear_iterations);
        }
      std::fclose(f);
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
