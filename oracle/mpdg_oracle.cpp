// CPU ORACLE — test infrastructure only.
//
// This file is the CPU restatement of MeltPoolDG's matrix-free operator hot path that the CUDA
// library is checked against.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
// leg may load it; the product library (meltpooldg_b200/libmpdg_b200.so) never links it.
//
// What it restates (reference paths are relative to the MeltPoolDG source tree):
//  * the heat tangent  (rho*cp/dt) u phi + k grad u . grad phi
//      source/heat/heat_diffuse_operator.cpp:1029-1079 (tangent_local_cell_operation)
//  * the heat right-hand side  -[(rho*cp/dt)(T - T_old) - q] phi - k grad T . grad phi
//      source/heat/heat_diffuse_operator.cpp:485-527 (rhs_cell_loop)
//  * the heat inverse diagonal with the |d| > 1e-10 rule
//      source/heat/heat_diffuse_operator.cpp:271-284
//  * the advection-diffusion tangent  u/dt phi + theta v.grad u phi + theta eps grad u . grad phi
//      source/level_set/advection_diffusion_operator.cpp:448-495
//  * its right-hand side  (u_old/dt - (1-theta) v.grad u_old) phi - (1-theta) eps grad u_old . grad phi
//      source/level_set/advection_diffusion_operator.cpp:274-358
//  * its inverse diagonal with the |d| > 1e-14 max(1,|d|_inf) rule
//      source/level_set/advection_diffusion_operator.cpp:399-446
//  * SolverCG / SolverGMRES(right preconditioned) driven by ReductionControl(max_it, abs, rel)
//      include/meltpooldg/linear_algebra/linear_solver.hpp:36-118
//  * the Jacobi preconditioner dst = inv_diag .* src
//      include/meltpooldg/linear_algebra/preconditioner_jacobi.hpp:51-69
//
// deal.II conventions restated (the arithmetic of FEEvaluation lives in deal.II, which is not
// vendored by the reference): FE_Q(k) with Gauss-Lobatto support points, QGauss(k+1) cell
// quadrature (include/meltpooldg/utilities/fe_util.hpp:30, source/utilities/fe_util.cpp:58),
// read_dof_values() reads Dirichlet-constrained DoFs as 0, distribute_local_to_global() skips
// constrained rows, compute_diagonal() puts 1 on constrained rows.
//
// The operator is evaluated the way FEEvaluation does it: interpolate to the Gauss points,
// evaluate gradients there, apply the point-wise physics, integrate back (sum factorisation over
// the tensor-product basis).  The CUDA library uses a different factorisation of the same
// bilinear form, so agreement between the two is a real check.
//
// Mesh: a structured box of m[0] x m[1] x m[2] axis-aligned hexahedra; DoFs live on the
// (k m + 1)^3 Gauss-Lobatto lattice and are numbered lexicographically, x fastest.
//
// Cells are processed in 8 colour classes (parity of the cell coordinates), so threads never
// write the same DoF concurrently and every result is bit-identical for any thread count.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

typedef struct orc_op
{
  int32_t        degree;  // FE_Q degree k (1..6)
  int32_t        m[3];    // cells per direction
  double         origin[3];
  double         length[3];
  const uint8_t *cmask;   // per-DoF Dirichlet flag (NULL: no constraints)
  int32_t        kind;    // 0: heat, 1: advection-diffusion
  int32_t        pad_;
  double         rho_cp;  // heat: rho * c_p
  double         dt;      // time increment
  double         k_const; // heat: conductivity when k_cell == NULL
  const double  *k_cell;  // heat: per-cell conductivity (NULL: k_const)
  double         theta;   // advection: one-step-theta weight
  double         eps;     // advection: diffusivity
  double         vel[12]; // advection: v(x) = vel[0..2] + G x, G = vel[3..11] row-major
  const uint8_t *imask;   // advection: inflow DoFs with identity rows (NULL: none), see apply_impl
} orc_op;

} // extern "C"

namespace
{
  constexpr int MAXN = 8;

  // ---- 1D polynomial machinery ---------------------------------------------------------------

  // Legendre P_n and P_n' at x in [-1,1].
  void
  legendre(int n, double x, double &p, double &dp)
  {
    double p0 = 1.0, p1 = x;
    if (n == 0)
      {
        p  = 1.0;
        dp = 0.0;
        return;
      }
    for (int k = 2; k <= n; ++k)
      {
        const double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
        p0              = p1;
        p1              = p2;
      }
    p  = p1;
    dp = (std::abs(x) < 1.0) ? n * (p0 - x * p1) / (1.0 - x * x) : 0.5 * n * (n + 1) * std::pow(x, n - 1);
  }

  // Gauss-Lobatto points of degree k on [0,1]: 0, 1 and the roots of P_k'.
  void
  gauss_lobatto(int k, double *pts)
  {
    pts[0] = 0.0;
    pts[k] = 1.0;
    for (int i = 1; i < k; ++i)
      {
        double x = -std::cos(M_PI * i / k);
        for (int it = 0; it < 100; ++it)
          {
            double p, dp;
            legendre(k, x, p, dp);
            // P'' from the Legendre equation (1-x^2) P'' = 2x P' - k(k+1) P
            const double ddp = (2.0 * x * dp - k * (k + 1.0) * p) / (1.0 - x * x);
            const double dx  = dp / ddp;
            x -= dx;
            if (std::abs(dx) < 1e-16)
              break;
          }
        pts[i] = 0.5 * (x + 1.0);
      }
    std::sort(pts, pts + k + 1);
  }

  // n-point Gauss-Legendre rule on [0,1].
  void
  gauss(int n, double *pts, double *wts)
  {
    for (int i = 0; i < n; ++i)
      {
        double x = -std::cos(M_PI * (i + 0.75) / (n + 0.5));
        double p = 0, dp = 1;
        for (int it = 0; it < 100; ++it)
          {
            legendre(n, x, p, dp);
            const double dx = p / dp;
            x -= dx;
            if (std::abs(dx) < 1e-16)
              break;
          }
        legendre(n, x, p, dp);
        pts[i] = 0.5 * (x + 1.0);
        wts[i] = 1.0 / ((1.0 - x * x) * dp * dp); // 2/((1-x^2)P'^2) mapped to [0,1]
      }
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j)
        if (pts[j] < pts[i])
          {
            std::swap(pts[i], pts[j]);
            std::swap(wts[i], wts[j]);
          }
  }

  // Lagrange basis on nodes x[0..n-1]: value and derivative of phi_i at t.
  void
  lagrange(int n, const double *x, int i, double t, double &val, double &der)
  {
    val = 1.0;
    for (int j = 0; j < n; ++j)
      if (j != i)
        val *= (t - x[j]) / (x[i] - x[j]);
    der = 0.0;
    for (int m = 0; m < n; ++m)
      {
        if (m == i)
          continue;
        double prod = 1.0 / (x[i] - x[m]);
        for (int j = 0; j < n; ++j)
          if (j != i && j != m)
            prod *= (t - x[j]) / (x[i] - x[j]);
        der += prod;
      }
  }

  struct Basis1D
  {
    int    n;              // nodes = quadrature points = k+1
    double nodes[MAXN];    // Gauss-Lobatto support points on [0,1]
    double qp[MAXN];       // Gauss points on [0,1]
    double qw[MAXN];       // Gauss weights on [0,1]
    double B[MAXN * MAXN]; // B[q*n+i] = phi_i(qp_q)
    double G[MAXN * MAXN]; // G[q*n+i] = phi_i'(qp_q)
  };

  Basis1D
  make_basis(int degree)
  {
    Basis1D b{};
    b.n = degree + 1;
    gauss_lobatto(degree, b.nodes);
    gauss(b.n, b.qp, b.qw);
    for (int q = 0; q < b.n; ++q)
      for (int i = 0; i < b.n; ++i)
        lagrange(b.n, b.nodes, i, b.qp[q], b.B[q * b.n + i], b.G[q * b.n + i]);
    return b;
  }

  // ---- geometry / lattice ---------------------------------------------------------------------

  struct Lattice
  {
    int64_t n[3]; // lattice points per direction
    int64_t ndofs;
    int64_t ncells;
    double  h[3];
  };

  Lattice
  lattice(const orc_op &op)
  {
    Lattice L;
    for (int d = 0; d < 3; ++d)
      {
        L.n[d] = (int64_t)op.degree * op.m[d] + 1;
        L.h[d] = op.length[d] / op.m[d];
      }
    L.ndofs  = L.n[0] * L.n[1] * L.n[2];
    L.ncells = (int64_t)op.m[0] * op.m[1] * op.m[2];
    return L;
  }

  // ---- tensor contractions on an N^3 cell array stored [z][y][x] -------------------------------

  template <int N, int AX, bool TR, bool ADD>
  inline void
  contract(const double *S, const double *in, double *out)
  {
    constexpr int st = AX == 0 ? 1 : (AX == 1 ? N : N * N);
    for (int k = 0; k < N; ++k)
      for (int j = 0; j < N; ++j)
        {
          const int base = AX == 0 ? k * N * N + j * N : (AX == 1 ? k * N * N + j : k * N + j);
          for (int a = 0; a < N; ++a)
            {
              double s = 0.0;
              for (int b = 0; b < N; ++b)
                s += (TR ? S[b * N + a] : S[a * N + b]) * in[base + b * st];
              if (ADD)
                out[base + a * st] += s;
              else
                out[base + a * st] = s;
            }
        }
  }

  // Values and reference-coordinate gradients at the Gauss points.
  template <int N>
  inline void
  evaluate(const Basis1D &b, const double *u, double *uq, double *dx, double *dy, double *dz)
  {
    double X0[N * N * N], X1[N * N * N], Y00[N * N * N], Y01[N * N * N], Y10[N * N * N];
    contract<N, 0, false, false>(b.B, u, X0);
    contract<N, 0, false, false>(b.G, u, X1);
    contract<N, 1, false, false>(b.B, X0, Y00);
    contract<N, 1, false, false>(b.G, X0, Y01);
    contract<N, 1, false, false>(b.B, X1, Y10);
    contract<N, 2, false, false>(b.B, Y00, uq);
    contract<N, 2, false, false>(b.G, Y00, dz);
    contract<N, 2, false, false>(b.B, Y01, dy);
    contract<N, 2, false, false>(b.B, Y10, dx);
  }

  // out_i = sum_q [ v_q phi_i + gx_q d_xi phi_i + gy_q d_eta phi_i + gz_q d_zeta phi_i ]
  template <int N>
  inline void
  integrate(const Basis1D &b, const double *v, const double *gx, const double *gy, const double *gz, double *out)
  {
    double Z0[N * N * N], Z1[N * N * N], Z2[N * N * N], Y0[N * N * N], Y2[N * N * N];
    contract<N, 2, true, false>(b.B, v, Z0);
    contract<N, 2, true, true>(b.G, gz, Z0);
    contract<N, 2, true, false>(b.B, gy, Z1);
    contract<N, 2, true, false>(b.B, gx, Z2);
    contract<N, 1, true, false>(b.B, Z0, Y0);
    contract<N, 1, true, true>(b.G, Z1, Y0);
    contract<N, 1, true, false>(b.B, Z2, Y2);
    contract<N, 0, true, false>(b.B, Y0, out);
    contract<N, 0, true, true>(b.G, Y2, out);
  }

  struct CellGeom
  {
    double origin[3];
    double h[3];
  };

  // Point-wise physics.  'mode' selects tangent (0) or right-hand side (1).  The inputs at q are
  // the values/physical gradients of up to three fields; outputs are already multiplied by JxW
  // and by the inverse Jacobian of the test-function gradient.
  template <int N>
  void
  local_operator(const orc_op &op, const Basis1D &b, const CellGeom &g, double kc, int mode,
                 const double *u0, const double *u1, const double *u2, double *out)
  {
    constexpr int NQ = N * N * N;
    double        q0[NQ], d0x[NQ], d0y[NQ], d0z[NQ];
    double        q1[NQ], q2[NQ], t1[NQ], t2[NQ], t3[NQ];
    double        V[NQ], GX[NQ], GY[NQ], GZ[NQ];
    evaluate<N>(b, u0, q0, d0x, d0y, d0z);
    const bool heat = op.kind == 0;
    if (heat && mode == 1)
      {
        evaluate<N>(b, u1, q1, t1, t2, t3); // T_old: values only
        evaluate<N>(b, u2, q2, t1, t2, t3); // q: values only
      }
    const double detJ = g.h[0] * g.h[1] * g.h[2];
    for (int qz = 0; qz < N; ++qz)
      for (int qy = 0; qy < N; ++qy)
        for (int qx = 0; qx < N; ++qx)
          {
            const int    q   = (qz * N + qy) * N + qx;
            const double JxW = b.qw[qx] * b.qw[qy] * b.qw[qz] * detJ;
            const double gx  = d0x[q] / g.h[0], gy = d0y[q] / g.h[1], gz = d0z[q] / g.h[2];
            double       val, fx, fy, fz;
            if (heat)
              {
                const double inv_dt = 1.0 / op.dt;
                if (mode == 0)
                  {
                    val = inv_dt * op.rho_cp * q0[q];
                    fx  = kc * gx;
                    fy  = kc * gy;
                    fz  = kc * gz;
                  }
                else
                  {
                    val = -(inv_dt * op.rho_cp * (q0[q] - q1[q]) - q2[q]);
                    fx  = -kc * gx;
                    fy  = -kc * gy;
                    fz  = -kc * gz;
                  }
              }
            else
              {
                const double x = g.origin[0] + g.h[0] * b.qp[qx];
                const double y = g.origin[1] + g.h[1] * b.qp[qy];
                const double z = g.origin[2] + g.h[2] * b.qp[qz];
                const double *v = op.vel;
                const double vx = v[0] + v[3] * x + v[4] * y + v[5] * z;
                const double vy = v[1] + v[6] * x + v[7] * y + v[8] * z;
                const double vz = v[2] + v[9] * x + v[10] * y + v[11] * z;
                const double vg = vx * gx + vy * gy + vz * gz;
                if (mode == 0)
                  {
                    val = q0[q] / op.dt + op.theta * vg;
                    fx  = op.theta * op.eps * gx;
                    fy  = op.theta * op.eps * gy;
                    fz  = op.theta * op.eps * gz;
                  }
                else
                  {
                    val = q0[q] / op.dt - (1.0 - op.theta) * vg;
                    fx  = -(1.0 - op.theta) * op.eps * gx;
                    fy  = -(1.0 - op.theta) * op.eps * gy;
                    fz  = -(1.0 - op.theta) * op.eps * gz;
                  }
              }
            V[q]  = val * JxW;
            GX[q] = fx * JxW / g.h[0];
            GY[q] = fy * JxW / g.h[1];
            GZ[q] = fz * JxW / g.h[2];
          }
    integrate<N>(b, V, GX, GY, GZ, out);
  }

  struct CellIndex
  {
    int64_t idx[MAXN * MAXN * MAXN];
  };

  inline void
  cell_dofs(const orc_op &op, const Lattice &L, int cx, int cy, int cz, int64_t *idx)
  {
    const int n = op.degree + 1;
    for (int l = 0; l < n; ++l)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
          {
            const int64_t I = (int64_t)op.degree * cx + i, J = (int64_t)op.degree * cy + j,
                          K = (int64_t)op.degree * cz + l;
            idx[(l * n + j) * n + i] = I + L.n[0] * (J + L.n[1] * K);
          }
  }

  inline CellGeom
  cell_geom(const orc_op &op, const Lattice &L, int cx, int cy, int cz)
  {
    CellGeom g;
    const int c[3] = {cx, cy, cz};
    for (int d = 0; d < 3; ++d)
      {
        g.h[d]      = L.h[d];
        g.origin[d] = op.origin[d] + c[d] * L.h[d];
      }
    return g;
  }

  inline double
  cell_k(const orc_op &op, int64_t cell)
  {
    return op.k_cell ? op.k_cell[cell] : op.k_const;
  }

  // Loop over cells in 8 colour classes; f(cx,cy,cz,cell_index).
  template <typename F>
  void
  colored_cell_loop(const orc_op &op, F &&f)
  {
    for (int color = 0; color < 8; ++color)
      {
        const int px = color & 1, py = (color >> 1) & 1, pz = (color >> 2) & 1;
        const int nx = (op.m[0] - px + 1) / 2, ny = (op.m[1] - py + 1) / 2, nz = (op.m[2] - pz + 1) / 2;
        const int64_t total = (int64_t)nx * ny * nz;
#pragma omp parallel for schedule(static)
        for (int64_t t = 0; t < total; ++t)
          {
            const int ix = (int)(t % nx), iy = (int)((t / nx) % ny), iz = (int)(t / ((int64_t)nx * ny));
            const int cx = 2 * ix + px, cy = 2 * iy + py, cz = 2 * iz + pz;
            f(cx, cy, cz, (int64_t)cx + (int64_t)op.m[0] * (cy + (int64_t)op.m[1] * cz));
          }
      }
  }

  // Inflow DoFs (imask) of the advection operator follow AdvectionDiffusionOperator::do_pre_vmult /
  // do_post_vmult (source/level_set/advection_diffusion_operator.cpp:543-578): src reads 0 there,
  // and the row is the identity (vmult: dst_i = src_i; the add form: dst_i += src_i).
  template <int N>
  void
  apply_impl(const orc_op &op, const double *src, double *dst, bool zero_dst)
  {
    const Lattice L = lattice(op);
    const Basis1D b = make_basis(op.degree);
    if (zero_dst)
      std::memset(dst, 0, sizeof(double) * L.ndofs);
    auto skip = [&](int64_t i) { return (op.cmask && op.cmask[i]) || (op.imask && op.imask[i]); };
    colored_cell_loop(op, [&](int cx, int cy, int cz, int64_t cell) {
      int64_t idx[N * N * N];
      double  u[N * N * N], out[N * N * N];
      cell_dofs(op, L, cx, cy, cz, idx);
      for (int i = 0; i < N * N * N; ++i)
        u[i] = skip(idx[i]) ? 0.0 : src[idx[i]];
      const CellGeom g = cell_geom(op, L, cx, cy, cz);
      local_operator<N>(op, b, g, cell_k(op, cell), 0, u, nullptr, nullptr, out);
      for (int i = 0; i < N * N * N; ++i)
        if (!skip(idx[i]))
          dst[idx[i]] += out[i];
    });
    if (op.imask)
      for (int64_t i = 0; i < L.ndofs; ++i)
        if (op.imask[i] && !(op.cmask && op.cmask[i]))
          dst[i] += src[i];
  }

  template <int N>
  void
  rhs_impl(const orc_op &op, const double *a, const double *b_, const double *c, double *dst)
  {
    const Lattice L = lattice(op);
    const Basis1D b = make_basis(op.degree);
    colored_cell_loop(op, [&](int cx, int cy, int cz, int64_t cell) {
      int64_t idx[N * N * N];
      double  u0[N * N * N], u1[N * N * N], u2[N * N * N], out[N * N * N];
      cell_dofs(op, L, cx, cy, cz, idx);
      for (int i = 0; i < N * N * N; ++i)
        {
          u0[i] = a[idx[i]]; // plain reads: read_dof_values_plain
          u1[i] = b_ ? b_[idx[i]] : 0.0;
          u2[i] = c ? c[idx[i]] : 0.0;
        }
      const CellGeom g = cell_geom(op, L, cx, cy, cz);
      local_operator<N>(op, b, g, cell_k(op, cell), 1, u0, u1, u2, out);
      for (int i = 0; i < N * N * N; ++i)
        if (!(op.cmask && op.cmask[idx[i]]))
          dst[idx[i]] += out[i];
    });
  }

  // Diagonal by one local apply per unit vector (MatrixFreeTools::compute_diagonal).
  template <int N>
  void
  diag_impl(const orc_op &op, double *diag)
  {
    const Lattice L = lattice(op);
    const Basis1D b = make_basis(op.degree);
    std::memset(diag, 0, sizeof(double) * L.ndofs);
    colored_cell_loop(op, [&](int cx, int cy, int cz, int64_t cell) {
      int64_t idx[N * N * N];
      double  u[N * N * N], out[N * N * N];
      cell_dofs(op, L, cx, cy, cz, idx);
      const CellGeom g  = cell_geom(op, L, cx, cy, cz);
      const double   kc = cell_k(op, cell);
      for (int i = 0; i < N * N * N; ++i)
        {
          if (op.cmask && op.cmask[idx[i]])
            continue;
          std::memset(u, 0, sizeof(u));
          u[i] = 1.0;
          local_operator<N>(op, b, g, kc, 0, u, nullptr, nullptr, out);
          diag[idx[i]] += out[i];
        }
    });
    if (op.cmask)
      for (int64_t i = 0; i < L.ndofs; ++i)
        if (op.cmask[i])
          diag[i] = 1.0;
  }

  // Cell-wise stiffness bilinear form  a_c = lam_c^T K_c T_c  with unit conductivity.
  template <int N>
  void
  cell_stiffness_form_impl(const orc_op &op, const double *lam, const double *T, double *form)
  {
    const Lattice L = lattice(op);
    const Basis1D b = make_basis(op.degree);
    orc_op        unit = op;
    unit.kind          = 0;
    unit.rho_cp        = 0.0;
    unit.dt            = 1.0;
    colored_cell_loop(op, [&](int cx, int cy, int cz, int64_t cell) {
      int64_t idx[N * N * N];
      double  u[N * N * N], out[N * N * N];
      cell_dofs(op, L, cx, cy, cz, idx);
      for (int i = 0; i < N * N * N; ++i)
        u[i] = (op.cmask && op.cmask[idx[i]]) ? 0.0 : T[idx[i]];
      const CellGeom g = cell_geom(op, L, cx, cy, cz);
      local_operator<N>(unit, b, g, 1.0, 0, u, nullptr, nullptr, out);
      double s = 0.0;
      for (int i = 0; i < N * N * N; ++i)
        if (!(op.cmask && op.cmask[idx[i]]))
          s += lam[idx[i]] * out[i];
      form[cell] = s;
    });
  }

  template <int N>
  double
  l2_norm_impl(const orc_op &op, const double *u)
  {
    const Lattice        L = lattice(op);
    const Basis1D        b = make_basis(op.degree);
    std::vector<double>  part(L.ncells);
#pragma omp parallel for schedule(static)
    for (int64_t cell = 0; cell < L.ncells; ++cell)
      {
        const int cx = (int)(cell % op.m[0]), cy = (int)((cell / op.m[0]) % op.m[1]),
                  cz = (int)(cell / ((int64_t)op.m[0] * op.m[1]));
        int64_t idx[N * N * N];
        double  uc[N * N * N], uq[N * N * N], X0[N * N * N], Y0[N * N * N];
        cell_dofs(op, L, cx, cy, cz, idx);
        for (int i = 0; i < N * N * N; ++i)
          uc[i] = u[idx[i]];
        contract<N, 0, false, false>(b.B, uc, X0);
        contract<N, 1, false, false>(b.B, X0, Y0);
        contract<N, 2, false, false>(b.B, Y0, uq);
        double s = 0.0;
        for (int qz = 0; qz < N; ++qz)
          for (int qy = 0; qy < N; ++qy)
            for (int qx = 0; qx < N; ++qx)
              {
                const double v = uq[(qz * N + qy) * N + qx];
                s += b.qw[qx] * b.qw[qy] * b.qw[qz] * v * v;
              }
        part[cell] = s * L.h[0] * L.h[1] * L.h[2];
      }
    double s = 0.0;
    for (double p : part)
      s += p;
    return std::sqrt(s);
  }

  // ---- batched heat apply for the timed CPU baseline ---------------------------------------------
  // The same heat tangent as apply_impl, evaluated the way deal.II's FEEvaluation does it on a CPU:
  // cells in batches of 8 (SIMD lanes, one cell per lane) within one colour class, values at the
  // Gauss points by three sweeps of B, gradients by the collocation derivative on the Gauss points
  // (exact for the degree-k interpolant), integration by the transposed sweeps.
  typedef double v8 __attribute__((vector_size(64)));

  template <int N, int AX, bool TR, bool ADD>
  inline void
  vcontract(const double *S, const v8 *in, v8 *out)
  {
    constexpr int st = AX == 0 ? 1 : (AX == 1 ? N : N * N);
    for (int k = 0; k < N; ++k)
      for (int j = 0; j < N; ++j)
        {
          const int base = AX == 0 ? k * N * N + j * N : (AX == 1 ? k * N * N + j : k * N + j);
          v8        in_l[N];
          for (int b = 0; b < N; ++b)
            in_l[b] = in[base + b * st];
          for (int a = 0; a < N; ++a)
            {
              v8 acc = ADD ? out[base + a * st] : v8{};
              for (int b = 0; b < N; ++b)
                acc += (TR ? S[b * N + a] : S[a * N + b]) * in_l[b];
              out[base + a * st] = acc;
            }
        }
  }

  template <int N>
  void
  apply_batched_impl(const orc_op &op, const double *src, double *dst)
  {
    constexpr int N3 = N * N * N, W = 8;
    const Lattice L = lattice(op);
    const Basis1D b = make_basis(op.degree);
    double        Dq[N * N]; // collocation derivative on the Gauss points: Dq[q*N+r] = l_r'(x_q)
    for (int q = 0; q < N; ++q)
      for (int r = 0; r < N; ++r)
        {
          double val, der;
          lagrange(N, b.qp, r, b.qp[q], val, der);
          Dq[q * N + r] = der;
        }
    double wq[N3];
    for (int qz = 0; qz < N; ++qz)
      for (int qy = 0; qy < N; ++qy)
        for (int qx = 0; qx < N; ++qx)
          wq[(qz * N + qy) * N + qx] = b.qw[qx] * b.qw[qy] * b.qw[qz] * L.h[0] * L.h[1] * L.h[2];
    const double mass = op.rho_cp / op.dt, ih2[3] = {1.0 / (L.h[0] * L.h[0]), 1.0 / (L.h[1] * L.h[1]),
                                                      1.0 / (L.h[2] * L.h[2])};
    int64_t off[N3];
    for (int l = 0; l < N; ++l)
      for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i)
          off[(l * N + j) * N + i] = i + L.n[0] * (j + L.n[1] * (int64_t)l);
    std::memset(dst, 0, sizeof(double) * L.ndofs);
    for (int color = 0; color < 8; ++color)
      {
        const int     px = color & 1, py = (color >> 1) & 1, pz = (color >> 2) & 1;
        const int     nx = (op.m[0] - px + 1) / 2, ny = (op.m[1] - py + 1) / 2, nz = (op.m[2] - pz + 1) / 2;
        const int     nb = (nx + W - 1) / W;
        const int64_t total = (int64_t)nb * ny * nz;
#pragma omp parallel for schedule(static)
        for (int64_t t = 0; t < total; ++t)
          {
            const int ib = (int)(t % nb), iy = (int)((t / nb) % ny), iz = (int)(t / ((int64_t)nb * ny));
            const int cy = 2 * iy + py, cz = 2 * iz + pz;
            int       cxl[W];
            bool      ok[W];
            v8        kv;
            for (int l = 0; l < W; ++l)
              {
                const int ix = ib * W + l;
                ok[l]        = ix < nx;
                cxl[l]       = ok[l] ? 2 * ix + px : px;
                kv[l] = ok[l] ? cell_k(op, (int64_t)cxl[l] + (int64_t)op.m[0] * (cy + (int64_t)op.m[1] * cz)) : 0.0;
              }
            v8 u[N3], uq[N3], gx[N3], gy[N3], gz[N3];
            // lane l's DoF q sits at base + 2 k l + off[q] (the batch's cells are 2 apart in x)
            const int64_t base = (int64_t)op.degree * cxl[0] + L.n[0] * ((int64_t)op.degree * cy +
                                                                         L.n[1] * (int64_t)op.degree * cz);
            const int64_t lstride = 2 * (int64_t)op.degree;
            for (int q = 0; q < N3; ++q)
              {
                const int64_t o = base + off[q];
                for (int l = 0; l < W; ++l)
                  {
                    const int64_t id = o + lstride * l;
                    u[q][l]          = (!ok[l] || (op.cmask && op.cmask[id])) ? 0.0 : src[id];
                  }
              }
            vcontract<N, 0, false, false>(b.B, u, gx);
            vcontract<N, 1, false, false>(b.B, gx, gy);
            vcontract<N, 2, false, false>(b.B, gy, uq);
            vcontract<N, 0, false, false>(Dq, uq, gx);
            vcontract<N, 1, false, false>(Dq, uq, gy);
            vcontract<N, 2, false, false>(Dq, uq, gz);
            for (int q = 0; q < N3; ++q)
              {
                const double w = wq[q];
                uq[q]          = (w * mass) * uq[q];
                gx[q]          = (w * ih2[0]) * kv * gx[q];
                gy[q]          = (w * ih2[1]) * kv * gy[q];
                gz[q]          = (w * ih2[2]) * kv * gz[q];
              }
            vcontract<N, 0, true, true>(Dq, gx, uq);
            vcontract<N, 1, true, true>(Dq, gy, uq);
            vcontract<N, 2, true, true>(Dq, gz, uq);
            vcontract<N, 2, true, false>(b.B, uq, gx);
            vcontract<N, 1, true, false>(b.B, gx, gy);
            vcontract<N, 0, true, false>(b.B, gy, u);
            for (int q = 0; q < N3; ++q)
              {
                const int64_t o = base + off[q];
                for (int l = 0; l < W; ++l)
                  {
                    const int64_t id = o + lstride * l;
                    if (ok[l] && !(op.cmask && op.cmask[id]))
                      dst[id] += u[q][l];
                  }
              }
          }
      }
  }

#define ORC_DISPATCH(deg, call)                                                                      \
  switch ((deg) + 1)                                                                                 \
    {                                                                                                \
      case 2: call(2); break;                                                                        \
      case 3: call(3); break;                                                                        \
      case 4: call(4); break;                                                                        \
      case 5: call(5); break;                                                                        \
      case 6: call(6); break;                                                                        \
      case 7: call(7); break;                                                                        \
      default: return -1;                                                                            \
    }

  // ---- deterministic vector reductions --------------------------------------------------------

  constexpr int64_t RBLOCK = 4096;

  double
  dot(const double *a, const double *b, int64_t n)
  {
    const int64_t       nb = (n + RBLOCK - 1) / RBLOCK;
    std::vector<double> part(nb);
#pragma omp parallel for schedule(static)
    for (int64_t blk = 0; blk < nb; ++blk)
      {
        double        s  = 0.0;
        const int64_t e  = std::min(n, (blk + 1) * RBLOCK);
        for (int64_t i = blk * RBLOCK; i < e; ++i)
          s += a[i] * b[i];
        part[blk] = s;
      }
    double s = 0.0;
    for (double p : part)
      s += p;
    return s;
  }

  // ReductionControl(max_it, abs_tol, rel_tol): 0 iterate, 1 success, 2 failure
  struct Control
  {
    int    max_it;
    double abs_tol, rel_tol;
    double reduced_tol = 0.0;
    int
    check(int step, double value)
    {
      if (step == 0)
        reduced_tol = value * rel_tol;
      if (value <= reduced_tol)
        return 1;
      if (value <= abs_tol)
        return 1;
      if (step >= max_it || std::isnan(value))
        return 2;
      return 0;
    }
  };
} // namespace

extern "C" {

int
orc_apply(const orc_op *op, const double *src, double *dst)
{
#define CALL(N) apply_impl<N>(*op, src, dst, true)
  ORC_DISPATCH(op->degree, CALL)
#undef CALL
  return 0;
}

// dst = A src of the heat operator, cell-batched sum factorisation (the timed CPU baseline)
int
orc_apply_batched(const orc_op *op, const double *src, double *dst)
{
  if (op->kind != 0)
    return -1;
#define CALL(N) apply_batched_impl<N>(*op, src, dst)
  ORC_DISPATCH(op->degree, CALL)
#undef CALL
  return 0;
}

// dst += A src (rows per the constraint mask)
int
orc_apply_add(const orc_op *op, const double *src, double *dst)
{
#define CALL(N) apply_impl<N>(*op, src, dst, false)
  ORC_DISPATCH(op->degree, CALL)
#undef CALL
  return 0;
}

// Heat: dst += -[(rho cp/dt)(T - T_old) - q] phi - k grad T . grad phi
// Advection: dst += (u_old/dt - (1-theta) v.grad u_old) phi - (1-theta) eps grad u_old . grad phi
//   (a = u_old, b and c unused)
int
orc_create_rhs(const orc_op *op, double *dst, const double *a, const double *b, const double *c)
{
#define CALL(N) rhs_impl<N>(*op, a, b, c, dst)
  ORC_DISPATCH(op->degree, CALL)
#undef CALL
  return 0;
}

int
orc_diagonal(const orc_op *op, double *diag)
{
#define CALL(N) diag_impl<N>(*op, diag)
  ORC_DISPATCH(op->degree, CALL)
#undef CALL
  return 0;
}

// compute_inverse_diagonal_from_matrixfree for either operator kind
int
orc_inverse_diagonal(const orc_op *op, double *diag)
{
  if (orc_diagonal(op, diag))
    return -1;
  const Lattice L = lattice(*op);
  if (op->kind == 0)
    {
      for (int64_t i = 0; i < L.ndofs; ++i)
        diag[i] = std::abs(diag[i]) > 1.0e-10 ? 1.0 / diag[i] : 1.0;
    }
  else
    {
      double linf = 0.0;
      for (int64_t i = 0; i < L.ndofs; ++i)
        linf = std::max(linf, std::abs(diag[i]));
      linf = std::max(1.0, linf);
      for (int64_t i = 0; i < L.ndofs; ++i)
        diag[i] = (std::abs(diag[i]) > 1.0e-14 * linf) ? 1.0 / diag[i] : 1.0;
      // inflow rows are identity rows (advection_diffusion_operator.cpp:444-445)
      if (op->imask)
        for (int64_t i = 0; i < L.ndofs; ++i)
          if (op->imask[i])
            diag[i] = 1.0;
    }
  return 0;
}

int
orc_cell_stiffness_form(const orc_op *op, const double *lam, const double *T, double *form)
{
#define CALL(N) cell_stiffness_form_impl<N>(*op, lam, T, form)
  ORC_DISPATCH(op->degree, CALL)
#undef CALL
  return 0;
}

double
orc_l2_norm(const orc_op *op, const double *u)
{
  double r = -1.0;
#define CALL(N) r = l2_norm_impl<N>(*op, u)
  switch (op->degree + 1)
    {
      case 2: CALL(2); break;
      case 3: CALL(3); break;
      case 4: CALL(4); break;
      case 5: CALL(5); break;
      case 6: CALL(6); break;
      case 7: CALL(7); break;
      default: break;
    }
#undef CALL
  return r;
}

double
orc_dot(const double *a, const double *b, int64_t n)
{
  return dot(a, b, n);
}

int64_t
orc_n_dofs(const orc_op *op)
{
  return lattice(*op).ndofs;
}

// Basis tables (for tests): nodes, Gauss points/weights, B and G (n*n each).
int
orc_basis(int degree, double *nodes, double *qp, double *qw, double *B, double *G)
{
  if (degree < 1 || degree + 1 > MAXN)
    return -1;
  const Basis1D b = make_basis(degree);
  const int     n = b.n;
  std::memcpy(nodes, b.nodes, sizeof(double) * n);
  std::memcpy(qp, b.qp, sizeof(double) * n);
  std::memcpy(qw, b.qw, sizeof(double) * n);
  std::memcpy(B, b.B, sizeof(double) * n * n);
  std::memcpy(G, b.G, sizeof(double) * n * n);
  return 0;
}

// SolverCG with a Jacobi preconditioner (inv_diag == NULL: identity) and ReductionControl.
// Returns 0 on convergence, 1 on failure (SolverControl::NoConvergence), -1 on bad input.
// *n_it = last_step(); hist[0..n_it] the residual norms if hist != NULL (size max_it+1).
int
orc_cg(const orc_op *op, const double *inv_diag, double *x, const double *b, int max_it,
       double abs_tol, double rel_tol, int *n_it, double *hist)
{
  const int64_t       n = orc_n_dofs(op);
  std::vector<double> r(n), z(n), p(n), v(n);
  Control             ctl{max_it, abs_tol, rel_tol};
  orc_apply(op, x, v.data());
#pragma omp parallel for
  for (int64_t i = 0; i < n; ++i)
    r[i] = b[i] - v[i];
  double res = std::sqrt(dot(r.data(), r.data(), n));
  if (hist)
    hist[0] = res;
  int state = ctl.check(0, res);
  int it    = 0;
  double rho_old = 0.0;
  while (state == 0)
    {
      ++it;
#pragma omp parallel for
      for (int64_t i = 0; i < n; ++i)
        z[i] = inv_diag ? inv_diag[i] * r[i] : r[i];
      const double rho = dot(r.data(), z.data(), n);
      if (it == 1)
        {
#pragma omp parallel for
          for (int64_t i = 0; i < n; ++i)
            p[i] = z[i];
        }
      else
        {
          const double beta = rho / rho_old;
#pragma omp parallel for
          for (int64_t i = 0; i < n; ++i)
            p[i] = z[i] + beta * p[i];
        }
      orc_apply(op, p.data(), v.data());
      const double alpha = rho / dot(p.data(), v.data(), n);
#pragma omp parallel for
      for (int64_t i = 0; i < n; ++i)
        {
          x[i] += alpha * p[i];
          r[i] -= alpha * v[i];
        }
      res = std::sqrt(dot(r.data(), r.data(), n));
      if (hist)
        hist[it] = res;
      rho_old = rho;
      state   = ctl.check(it, res);
    }
  if (n_it)
    *n_it = it;
  return state == 1 ? 0 : 1;
}

// Restarted GMRES(restart) with right preconditioning and modified Gram-Schmidt.
int
orc_gmres(const orc_op *op, const double *inv_diag, double *x, const double *b, int max_it,
          double abs_tol, double rel_tol, int restart, int *n_it, double *hist)
{
  const int64_t                    n = orc_n_dofs(op);
  const int                        m = restart;
  std::vector<std::vector<double>> V(m + 1, std::vector<double>(n));
  std::vector<double>              w(n), z(n);
  std::vector<double>              H((m + 1) * m), cs(m), sn(m), g(m + 1), y(m);
  Control                          ctl{max_it, abs_tol, rel_tol};
  int                              it    = 0;
  int                              state = 0;
  bool                             first = true;
  while (true)
    {
      orc_apply(op, x, w.data());
#pragma omp parallel for
      for (int64_t i = 0; i < n; ++i)
        V[0][i] = b[i] - w[i];
      const double beta = std::sqrt(dot(V[0].data(), V[0].data(), n));
      if (first)
        {
          if (hist)
            hist[0] = beta;
          first = false;
        }
      state = ctl.check(it, beta);
      if (state != 0)
        break;
#pragma omp parallel for
      for (int64_t i = 0; i < n; ++i)
        V[0][i] /= beta;
      std::fill(g.begin(), g.end(), 0.0);
      g[0]  = beta;
      int j = 0;
      for (; j < m; ++j)
        {
          ++it;
#pragma omp parallel for
          for (int64_t i = 0; i < n; ++i)
            z[i] = inv_diag ? inv_diag[i] * V[j][i] : V[j][i];
          orc_apply(op, z.data(), w.data());
          for (int i = 0; i <= j; ++i)
            {
              const double h = dot(w.data(), V[i].data(), n);
              H[i * m + j]   = h;
#pragma omp parallel for
              for (int64_t k = 0; k < n; ++k)
                w[k] -= h * V[i][k];
            }
          const double hn   = std::sqrt(dot(w.data(), w.data(), n));
          H[(j + 1) * m + j] = hn;
          if (hn > 0)
            {
#pragma omp parallel for
              for (int64_t k = 0; k < n; ++k)
                V[j + 1][k] = w[k] / hn;
            }
          for (int i = 0; i < j; ++i)
            {
              const double t0 = H[i * m + j], t1 = H[(i + 1) * m + j];
              H[i * m + j]       = cs[i] * t0 + sn[i] * t1;
              H[(i + 1) * m + j] = -sn[i] * t0 + cs[i] * t1;
            }
          const double a = H[j * m + j], c = H[(j + 1) * m + j];
          const double r = std::hypot(a, c);
          cs[j]          = a / r;
          sn[j]          = c / r;
          H[j * m + j]   = r;
          H[(j + 1) * m + j] = 0.0;
          g[j + 1]           = -sn[j] * g[j];
          g[j]               = cs[j] * g[j];
          const double res   = std::abs(g[j + 1]);
          if (hist)
            hist[it] = res;
          state = ctl.check(it, res);
          if (state != 0 || hn == 0.0)
            {
              ++j;
              break;
            }
        }
      // y = H^-1 g (upper triangular j x j), x += P V y
      for (int i = j - 1; i >= 0; --i)
        {
          double s = g[i];
          for (int k = i + 1; k < j; ++k)
            s -= H[i * m + k] * y[k];
          y[i] = s / H[i * m + i];
        }
      std::fill(z.begin(), z.end(), 0.0);
      for (int i = 0; i < j; ++i)
        {
#pragma omp parallel for
          for (int64_t k = 0; k < n; ++k)
            z[k] += y[i] * V[i][k];
        }
#pragma omp parallel for
      for (int64_t k = 0; k < n; ++k)
        x[k] += inv_diag ? inv_diag[k] * z[k] : z[k];
      if (state != 0)
        break;
    }
  if (n_it)
    *n_it = it;
  return state == 1 ? 0 : 1;
}

int
orc_num_threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

} // extern "C"
