// The reference's unidirectional heat case driven through the C++ host layer (include/mpdg/mpdg.hpp):
// 32 x 32 x 1 FE_Q(1) cells on [0, 0.1]^2 x [0, 1] (the 2-D case of
// applications/mp-heat-transfer/cases/unidirectional_heat_transfer/tests/unidirectional_heat_transfer.json
// as a slab of depth 1), T0 = x, rho = c_p = k = 1, no boundary condition, dt = 1e-4, 5 implicit-Euler
// steps, each solved by Newton (residual tolerance 5e-9) with Jacobi-GMRES (relative 1e-12).
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
      std::fprintf(stderr, "usage: heat_newton <output file>\n");
      return 2;
    }
  try
    {
      mpdg_mesh_desc mesh{};
      mesh.degree = 1;
      mesh.cells[0] = 32, mesh.cells[1] = 32, mesh.cells[2] = 1;
      mesh.length[0] = 0.1, mesh.length[1] = 0.1, mesh.length[2] = 1.0;
      mpdg::HeatDiffuseOperator op(mesh, 1.0, 1e-4, 1.0);
      const int64_t             n = op.n_dofs();
      std::vector<double>       T0(n);
      for (int64_t i = 0; i < n; ++i)
        T0[i] = 0.1 * (double)(i % 33) / 32.0; // x of the lattice point
      double *T = nullptr, *T_old = nullptr, *rhs = nullptr, *du = nullptr, *zero = nullptr;
      for (double **v : {&T, &T_old, &rhs, &du, &zero})
        if (cudaMalloc(v, sizeof(double) * n) != cudaSuccess)
          throw mpdg::Error(MPDG_ERR_NOMEM, "cudaMalloc");
      cudaMemcpy(T, T0.data(), sizeof(double) * n, cudaMemcpyHostToDevice);

      mpdg::LinearSolverData lin;
      lin.solver_type         = MPDG_GMRES;
      lin.preconditioner_type = MPDG_PRECOND_JACOBI;
      lin.rel_tolerance       = 1e-12;
      mpdg::NonlinearSolverData nl;
      nl.residual_tolerance = 5e-9;
      mpdg::HeatDiffuseOperation heat(op, T, T_old, nullptr, rhs, du, zero, lin, nl);

      std::FILE *f = std::fopen(argv[1], "wb");
      if (!f)
        throw mpdg::Error(MPDG_ERR_ARG, "cannot open the output file");
      std::vector<double> host(n);
      for (int step = 0; step < 5; ++step)
        {
          heat.init_time_advance(1e-4);
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
