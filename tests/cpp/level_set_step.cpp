// One level-set step through the C++ host layer (include/mpdg/mpdg.hpp), in the order of
// LevelSetOperation::solve (source/level_set/level_set_operation.cpp): advect the indicator with
// the SUPG-stabilised advection-diffusion operator (GMRES), project its normal vector and curvature
// (M + damping K, a heat operator with rho c_p = dt = 1, Jacobi-CG per component), and take
// conservative reinitialisation (Olsson) steps along the projected normal (Jacobi-CG).
// 12 x 12 x 12 FE_Q(2) cells on [0,1]^3, natural boundaries everywhere; psi0 = (1 - tanh((|x - c| -
// 0.25) / 0.04)) / 2 with c = (0.5, 0.6, 0.5); rigid rotation v = (-(y - 0.5), x - 0.5, 0).
// Writes psi after the advection, the three normal components, the curvature and psi after the
// reinitialisation (6 x n_dofs doubles) to the file argv[1].
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <vector>

#include "mpdg/mpdg.hpp"

int
main(int argc, char **argv)
{
  if (argc < 2)
    {
      std::fprintf(stderr, "usage: level_set_step <output file>\n");
      return 2;
    }
  try
    {
      const int      m = 12, k = 2, nl = k * m + 1;
      const double   h = 1.0 / m;
      mpdg_mesh_desc mesh{};
      mesh.degree   = k;
      mesh.cells[0] = m, mesh.cells[1] = m, mesh.cells[2] = m;
      mesh.length[0] = 1.0, mesh.length[1] = 1.0, mesh.length[2] = 1.0;

      const double velocity[12] = {0.5, -0.5, 0.0, 0.0, -1.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      mpdg::AdvectionDiffusionOperator adv(mesh, 5e-3, 1.0, 1e-3, velocity);
      adv.set_convection_stabilization(true, 0.1);
      const int64_t n = adv.n_dofs();

      // lattice coordinates of the FE_Q(2) support points: cell corners and midpoints
      std::vector<double> psi0(n);
      for (int64_t i = 0; i < n; ++i)
        {
          const double x = h / k * (double)(i % nl), y = h / k * (double)((i / nl) % nl),
                       z = h / k * (double)(i / ((int64_t)nl * nl));
          const double r = std::sqrt((x - 0.5) * (x - 0.5) + (y - 0.6) * (y - 0.6) + (z - 0.5) * (z - 0.5));
          psi0[i]        = 0.5 * (1.0 - std::tanh((r - 0.25) / 0.04));
        }
      mpdg::DeviceVector psi_old(adv), psi(adv), rhs(adv), nx(adv), ny(adv), nz(adv), kappa(adv), dpsi(adv);
      cudaMemcpy(psi_old.get(), psi0.data(), sizeof(double) * n, cudaMemcpyHostToDevice);

      // advection: (M/dt + A) psi = M psi_old / dt (create_rhs accumulates into a zero vector)
      mpdg::LinearSolverData gmres;
      gmres.solver_type         = MPDG_GMRES;
      gmres.preconditioner_type = MPDG_PRECOND_JACOBI;
      gmres.rel_tolerance       = 1e-12;
      adv.create_rhs(rhs.get(), psi_old.get());
      adv.axpby(psi.get(), 1.0, psi_old.get(), 0.0);
      const int it_adv = mpdg::LinearSolver::solve(adv, psi.get(), rhs.get(), gmres);

      // normal vector and curvature projections
      mpdg::HeatDiffuseOperator projection(mesh, 1.0, 1.0, h * h); // damping h^2
      mpdg::LinearSolverData    cg;
      cg.solver_type         = MPDG_CG;
      cg.preconditioner_type = MPDG_PRECOND_JACOBI;
      cg.rel_tolerance       = 1e-12;
      double *normal[3]      = {nx.get(), ny.get(), nz.get()};
      projection.level_set_normal_rhs(psi.get(), nx.get(), ny.get(), nz.get());
      int it_proj = 0;
      for (double *c : normal)
        {
          projection.axpby(rhs.get(), 1.0, c, 0.0);
          projection.fill(c, 0.0);
          it_proj += mpdg::LinearSolver::solve(projection, c, rhs.get(), cg);
        }
      const double tol = 1e-10;
      projection.level_set_curvature_rhs(rhs.get(), nx.get(), ny.get(), nz.get(), tol);
      it_proj += mpdg::LinearSolver::solve(projection, kappa.get(), rhs.get(), cg);

      std::FILE *f = std::fopen(argv[1], "wb");
      if (!f)
        throw mpdg::Error(MPDG_ERR_ARG, "cannot open the output file");
      std::vector<double> host(n);
      auto                dump = [&](const double *d) {
        cudaMemcpy(host.data(), d, sizeof(double) * n, cudaMemcpyDeviceToHost);
        std::fwrite(host.data(), sizeof(double), n, f);
      };
      for (const double *d : {(const double *)psi.get(), (const double *)nx.get(), (const double *)ny.get(),
                              (const double *)nz.get(), (const double *)kappa.get()})
        dump(d);

      // conservative reinitialisation: (M/dt + D) dpsi = rhs(psi), psi += dpsi, 3 pseudo-time steps
      mpdg::OlssonOperator reinit(mesh, 0.25 * h);
      reinit.set_normal(0.5 * h, 0.0, tol, nx.get(), ny.get(), nz.get());
      int it_reinit = 0;
      for (int step = 0; step < 3; ++step)
        {
          reinit.create_rhs(rhs.get(), psi.get()); // overwrites
          reinit.fill(dpsi.get(), 0.0);
          it_reinit += mpdg::LinearSolver::solve(reinit, dpsi.get(), rhs.get(), cg);
          reinit.axpby(psi.get(), 1.0, dpsi.get(), 1.0);
        }
      dump(psi.get());
      std::fclose(f);
      std::printf("{\"advection_iterations\": %d, \"projection_iterations\": %d, \"reinit_iterations\": %d}\n",
                  it_adv, it_proj, it_reinit);
      return 0;
    }
  catch (const mpdg::Error &e)
    {
      std::fprintf(stderr, "mpdg error %d: %s\n", e.code, e.what());
      return 1;
    }
}
