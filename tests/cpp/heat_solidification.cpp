// Nonlinear heat time steps with temperature-dependent material through the C++ host layer
// (include/mpdg/mpdg.hpp): 8 x 8 x 8 FE_Q(2) cells on [0,1]^3, liquid (7.4, 0.8, 30) and solid
// (7.9, 0.6, 20) density / specific heat / conductivity, liquidus 1700, solidus 1600 (mushy zone),
// Dirichlet T = 1500 on the x = 0 face, T0 = 1500 + 250 x; dt = 2e-3, 3 implicit-Euler steps, each
// solved by Newton (the solidification tangent at the current iterate) with Jacobi-GMRES.
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
      std::fprintf(stderr, "usage: heat_solidification <output file>\n");
      return 2;
    }
  try
    {
      mpdg_mesh_desc mesh{};
      mesh.degree          = 2;
      mesh.cells[0]        = 8, mesh.cells[1] = 8, mesh.cells[2] = 8;
      mesh.length[0]       = 1.0, mesh.length[1] = 1.0, mesh.length[2] = 1.0;
      mesh.dirichlet_faces = 0b000001;
      mpdg::HeatDiffuseOperator op(mesh, 1.0, 2e-3, 1.0);
      mpdg_solid_liquid         mat{};
      mat.liquid_density       = 7.4;
      mat.liquid_specific_heat = 0.8;
      mat.liquid_conductivity  = 30.0;
      mat.solid_density        = 7.9;
      mat.solid_specific_heat  = 0.6;
      mat.solid_conductivity   = 20.0;
      mat.liquidus_temperature = 1700.0;
      mat.solidus_temperature  = 1600.0;
      op.set_solidification(&mat);
      const int64_t       n = op.n_dofs();
      std::vector<double> T0(n), host(n);
      for (int64_t i = 0; i < n; ++i)
        T0[i] = 1500.0 + 250.0 * (double)(i % 17) / 16.0; // x of the lattice point
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
      nl.residual_tolerance         = 1e-8;
      nl.field_correction_tolerance = 1e-9;
      nl.max_nonlinear_iterations   = 30;
      mpdg::HeatDiffuseOperation heat(op, T, T_old, nullptr, rhs, du, zero, lin, nl);
      std::FILE *f = std::fopen(argv[1], "wb");
      if (!f)
        throw mpdg::Error(MPDG_ERR_ARG, "cannot open the output file");
      for (int step = 0; step < 3; ++step)
        {
          heat.init_time_advance(2e-3);
          heat.solve();
          cudaMemcpy(host.data(), T, sizeof(double) * n, cudaMemcpyDeviceToHost);
          std::fwrite(host.data(), sizeof(double), n, f);
          std::printf("step %d: %d Newton iterations\n", step + 1, heat.newton().iterations);
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
