// C ABI (include/mpdg_gpu.h) and the host-side solver loops.
//
// The solver loops restate the algorithms the reference calls through
// include/meltpooldg/linear_algebra/linear_solver.hpp:26-134:
//   * dealii::SolverCG with the Jacobi preconditioner (preconditioner_jacobi.hpp:51-69) and
//     ReductionControl(max_it, abs_tol, rel_tol): the scalar recurrences run on the device
//     (CGState, vec.cu) so the host enqueues batches of iterations and only polls the state;
//   * dealii::SolverGMRES with right preconditioning (linear_solver.hpp:112-118), classical
//     Gram-Schmidt with one fused dot pass and one fused update pass per iteration, Givens
//     rotations and the least-squares update on the host in FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <type_traits>
#include <vector>

#include "mpdg_gpu.h"
#include "cgfused.h"
#include "tables.h"
#include "kernels.h"

using namespace mpdg;

namespace
{
  thread_local std::string g_last_error = "no error";

  int
  fail(int code, const std::string &msg)
  {
    g_last_error = msg;
    return code;
  }

  int
  cuda_fail(cudaError_t e, const char *where)
  {
    return fail(MPDG_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
  }

#define MPDG_CUDA(...)                                                                                         \
  do                                                                                                           \
    {                                                                                                          \
      cudaError_t e__ = (__VA_ARGS__);                                                                         \
      if (e__ != cudaSuccess)                                                                                  \
        return cuda_fail(e__, #__VA_ARGS__);                                                                   \
    }                                                                                                          \
  while (0)

  // host-side ReductionControl (GMRES)
  struct Control
  {
    int    max_it;
    double abs_tol, rel_tol, reduced = 0.0;
    int
    check(int step, double v)
    {
      if (step == 0)
        reduced = v * rel_tol;
      if (v <= reduced)
        return 1;
      if (v <= abs_tol)
        return 1;
      if (step >= max_it || std::isnan(v))
        return 2;
      return 0;
    }
  };
} // namespace

struct mpdg_op
{
  int       kind   = MPDG_HEAT;
  int       degree = 2;
  int       m[3]{};
  double    origin[3]{}, length[3]{}, h[3]{};
  uint32_t  faces  = 0;
  uint8_t  *d_mask = nullptr;
  bool      with_bc = true;
  double    rho_cp = 1.0, dt = 1.0, k = 1.0;
  double   *d_k64 = nullptr;
  float    *d_k32 = nullptr;
  double    theta = 1.0, eps = 0.0, vel[12]{};
  HeatFaceBC    fbc{};            // boundary-face terms (heat)
  bool          solid = false;    // temperature-dependent material (heat, FE_Q(1, 2))
  SolidMaterial smat{};
  const double *d_temp_old = nullptr; // T_old of the solidification tangent (not owned)
  long long     sync_cap = 0;         // brick flags allocated in d_sync (after the 3 counters)
  int           supg = 0;         // SUPG stabilisation (advection-diffusion)
  // inflow/outflow condition (advection-diffusion): inflow DoFs are identity rows of vmult
  uint8_t      *d_mask_io  = nullptr; // Dirichlet mask | inflow flags: the apply's read / write mask
  long long    *d_in_idx   = nullptr; // inflow DoFs
  double       *d_in_val   = nullptr; // their prescribed values
  long long     n_inflow   = 0;
  bool          inflow_prepost = true; // set_apply_inflow_outflow_constraints_pre_post_matrix_free
  // narrow band of the normal-vector / curvature projections (heat handles): level set (not owned)
  const double *d_band_ls = nullptr;
  double        band      = 0.0;
  bool
  banded() const
  {
    return kind == MPDG_HEAT && d_band_ls != nullptr && band > 0.0;
  }
  double        eps_n = 0.0, eps_t = 0.0, ntol = 1e-16; // reinitialisation
  unsigned      wetting = 0;                           // reinitialisation: wetting boundary faces
  const double *d_normal[3]{};                           // reinitialisation normal field (not owned)
  const double *d_vfield[3]{};                           // advection velocity as a DoF vector (not owned)
  double        supg_coef = 0.0;
  const double *d_temp = nullptr; // linearisation temperature of the radiation tangent (not owned)
  int       brick[3]{}, nbr[3]{};
  int       nbr32[3]{};  // bricks per direction of the FP32 apply (its column segments may be longer)
  long long ndofs = 0, ncells = 0;
  unsigned *d_sync = nullptr; // [0] ticket, [1] done, [2] reducer counter, [3..] flags
  int      *d_err  = nullptr;
  unsigned  epoch  = 0;
  unsigned  spin_limit = SPIN_LIMIT; // bound of every spin wait of this handle's kernels
  bool      fused_cg   = true;       // one-sweep PCG iteration where the operator allows it
  double   *d_red  = nullptr; // reducer partials
  double   *d_part = nullptr; // one partial per brick for the fused CG dot product (heat)
  double   *d_scal = nullptr; // 64 scalars
  CGState  *d_cg   = nullptr;
  CGState  *h_cg   = nullptr; // pinned mirror
  double   *h_scal = nullptr; // pinned scalars
  cudaStream_t stream = nullptr;
  std::map<std::string, std::pair<void *, size_t>> ws;
  // copy streams and events of the slab-pipelined host-buffer apply (created on first use)
  cudaStream_t             s_h2d = nullptr, s_d2h = nullptr;
  std::vector<cudaEvent_t> ev;

  template <typename T = double>
  GridDesc
  grid() const
  {
    GridDesc g;
    for (int d = 0; d < 3; ++d)
      {
        g.m[d]   = m[d];
        g.nbr[d] = sizeof(T) == 4 ? nbr32[d] : nbr[d];
        g.n[d]   = degree * m[d] + 1;
      }
    g.faces = with_bc ? faces : 0u;
    g.cmask = with_bc ? d_mask : nullptr;
    return g;
  }
  SyncDesc
  sync()
  {
    if (++epoch == 0)
      ++epoch;
    SyncDesc s;
    s.ticket = d_sync;
    s.done   = d_sync + 1;
    s.flags  = d_sync + 3;
    s.epoch  = epoch;
    s.error  = d_err;
    s.spin_limit = spin_limit;
    return s;
  }
  bool
  tangent_faces() const
  {
    return kind == MPDG_HEAT && heat_faces_active(fbc, 0);
  }
  Reducer
  reducer() const
  {
    return Reducer{d_red, d_sync + 2};
  }
  template <typename T>
  T *
  vec(const std::string &name, size_t count = 0)
  {
    const size_t bytes = sizeof(T) * (count ? count : (size_t)ndofs);
    auto         it    = ws.find(name);
    if (it != ws.end() && it->second.second >= bytes)
      return static_cast<T *>(it->second.first);
    if (it != ws.end())
      {
        cudaFree(it->second.first);
        ws.erase(it);
      }
    void *p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess)
      return nullptr;
    ws[name] = {p, bytes};
    return static_cast<T *>(p);
  }
  template <typename T>
  const T *
  kcell() const;
};

template <>
const double *
mpdg_op::kcell<double>() const
{
  return d_k64;
}
template <>
const float *
mpdg_op::kcell<float>() const
{
  return d_k32;
}

namespace
{
  HeatGeom
  heat_geom(const mpdg_op *op, double mass_scale)
  {
    HeatGeom g;
    g.mass_coef = mass_scale * op->h[0] * op->h[1] * op->h[2];
    g.cx        = op->h[1] * op->h[2] / op->h[0];
    g.cy        = op->h[0] * op->h[2] / op->h[1];
    g.cz        = op->h[0] * op->h[1] / op->h[2];
    return g;
  }

  AdvParams
  adv_params(const mpdg_op *op, double theta_override, bool use_override)
  {
    AdvParams p;
    const double th = use_override ? theta_override : op->theta;
    p.inv_dt        = 1.0 / op->dt;
    p.theta_adv     = th;
    p.theta_dif     = th * op->eps;
    for (int i = 0; i < 12; ++i)
      p.vel[i] = op->vel[i];
    for (int d = 0; d < 3; ++d)
      {
        p.origin[d] = op->origin[d];
        p.h[d]      = op->h[d];
      }
    p.supg      = op->supg;
    p.supg_coef = op->supg_coef;
    for (int d = 0; d < 3; ++d)
      p.vfield[d] = op->d_vfield[d];
    return p;
  }

  // The heat tangent with a convection velocity (heat_diffuse_operator.cpp:1029-1044, velocity a DoF
  // vector): rho c_p / dt u + rho c_p v . grad u tested with phi plus k grad u . grad phi, i.e. the
  // advection-diffusion form with 1/dt -> rho c_p / dt, theta -> rho c_p, theta eps -> k (the
  // velocity term alone for create_rhs: adv = -rho c_p, no mass, no diffusion).
  // the lattice of a heat operator with the brick counts of the advection-form kernels
  template <typename T>
  GridDesc
  heat_velocity_grid(const mpdg_op *op)
  {
    GridDesc g = op->grid<T>();
    int      sh[3];
    adv_brick_shape<T>(op->degree, sh);
    for (int d = 0; d < 3; ++d)
      g.nbr[d] = (op->m[d] + sh[d] - 1) / sh[d];
    return g;
  }

  AdvParams
  heat_velocity_params(const mpdg_op *op, bool rhs_term)
  {
    AdvParams p = adv_params(op, 0.0, false);
    p.inv_dt    = rhs_term ? 0.0 : op->rho_cp / op->dt;
    p.theta_adv = rhs_term ? -op->rho_cp : op->rho_cp;
    p.theta_dif = rhs_term ? 0.0 : op->k;
    for (int i = 0; i < 12; ++i)
      p.vel[i] = 0.0;
    p.supg = 0;
    return p;
  }

  template <typename T>
  ReinitLaunch<T>
  reinit_launch(const mpdg_op *op, double scale, const T *src, T *dst, int mask_src)
  {
    ReinitLaunch<T> r;
    r.degree           = op->degree;
    r.scale            = scale;
    r.dt               = op->dt;
    r.eps_normal       = op->eps_n;
    r.eps_tangential   = op->eps_t;
    r.normal_tolerance = op->ntol;
    for (int d = 0; d < 3; ++d)
      {
        r.hlen[d]   = op->h[d];
        r.normal[d] = op->d_normal[d];
      }
    r.grid     = op->grid<T>();
    r.src      = src;
    r.dst      = dst;
    r.mask_src = mask_src;
    r.wetting  = op->wetting;
    return r;
  }

  // The heat operator rho c_p / dt M + k K as the isotropic point-wise kernel with the narrow band
  // of the handle ('which' as in apply: 1 mass only, 2 stiffness only)
  template <typename T>
  ReinitLaunch<T>
  band_launch(const mpdg_op *op, int which, double scale, const T *src, T *dst, int mask_src)
  {
    ReinitLaunch<T> r;
    r.degree           = op->degree;
    r.scale            = scale;
    r.dt               = which == 2 ? 1e300 : op->dt / op->rho_cp;
    r.eps_normal       = which == 1 ? 0.0 : op->k;
    r.eps_tangential   = r.eps_normal;
    r.normal_tolerance = 1.0;
    for (int d = 0; d < 3; ++d)
      {
        r.hlen[d]   = op->h[d];
        r.normal[d] = nullptr;
      }
    r.grid     = op->grid<T>();
    r.src      = src;
    r.dst      = dst;
    r.mask_src = mask_src;
    r.band_ls  = op->d_band_ls;
    r.band     = op->band;
    return r;
  }

  // Temperature-dependent material: the tangent (rhs = false) or the residual part of create_rhs
  // (rhs = true, dst +=, src unused) with the operator's temperature and old temperature.  FP32
  // applies read FP32 copies of both.
  template <typename T>
  int
  solid_apply(mpdg_op *op, int mode, double scale, T *dst, const T *src, const T *b, int mask_src, const int *skip,
              bool rhs, const double *temp = nullptr, const double *temp_old = nullptr)
  {
    const double *t64 = temp ? temp : op->d_temp, *to64 = temp_old ? temp_old : op->d_temp_old;
    if (!t64 || !to64)
      return fail(MPDG_ERR_ARG, "the solidification tangent needs the temperature and the old temperature "
                                "(mpdg_op_set_temperature, mpdg_op_set_old_temperature)");
    HeatSolidLaunch<T> h;
    h.degree = op->degree;
    h.mode   = mode;
    h.rhs    = rhs ? 1 : 0;
    h.scale  = scale;
    h.dt     = op->dt;
    for (int d = 0; d < 3; ++d)
      h.hlen[d] = op->h[d];
    h.mat  = op->smat;
    h.grid = op->grid<T>();
    int shape[3];
    heat_solid_brick_shape<T>(op->degree, shape);
    for (int d = 0; d < 3; ++d)
      h.grid.nbr[d] = (op->m[d] + shape[d] - 1) / shape[d];
    h.sync = op->sync();
    if constexpr (std::is_same<T, double>::value)
      {
        h.temp     = t64;
        h.temp_old = to64;
      }
    else
      {
        T *t32 = op->vec<T>("solid_t32"), *to32 = op->vec<T>("solid_to32");
        if (!t32 || !to32)
          return fail(MPDG_ERR_NOMEM, "FP32 temperature copies");
        MPDG_CUDA(vec_convert<T, double>(t32, t64, op->ndofs, op->stream));
        MPDG_CUDA(vec_convert<T, double>(to32, to64, op->ndofs, op->stream));
        h.temp     = t32;
        h.temp_old = to32;
      }
    h.src      = src;
    h.dst      = dst;
    h.b        = b;
    h.mask_src = mask_src;
    h.skip     = skip;
    MPDG_CUDA(heat_solid_apply<T>(h, op->stream));
    return MPDG_OK;
  }

  // Generic apply.  mode: OutMode; 'which' selects the physics variant:
  //   0 tangent, 1 mass only (heat, coefficient mass_scale), 2 stiffness only (heat, scale on k),
  //   3 advection with theta replaced by theta - 1 (create_rhs)
  template <typename T>
  int
  apply(mpdg_op *op, int mode, double scale, T *dst, const T *src, const T *b, int mask_src, int which = 0,
        const int *skip = nullptr, const DotSink *dot = nullptr)
  {
    if (op->banded())
      {
        // the projection operator M + damping K with a narrow band (normal_vector_operator.cpp:
        // 326-358, curvature_operator.cpp:337-369): the isotropic form of the point-wise kernel
        if (mode == (int)OutMode::Set)
          MPDG_CUDA(vec_fill<T>(dst, T(0), op->ndofs, op->stream));
        else if (mode == (int)OutMode::BPlus && dst != b)
          MPDG_CUDA(cudaMemcpyAsync(dst, b, sizeof(T) * op->ndofs, cudaMemcpyDeviceToDevice, op->stream));
        MPDG_CUDA(reinit_integrate<T>(band_launch<T>(op, which, scale, src, dst, mask_src), 0, op->stream));
        return MPDG_OK;
      }
    if (op->kind == MPDG_HEAT)
      {
        HeatLaunch<T> h;
        h.degree = op->degree;
        h.mode   = mode;
        h.scale  = scale;
        h.geo    = heat_geom(op, which == 2 ? 0.0 : (which == 1 ? 1.0 : op->rho_cp / op->dt));
        h.grid   = op->grid<T>();
        h.sync   = op->sync();
        h.kconst = which == 1 ? 0.0 : op->k;
        h.kcell  = which == 1 ? nullptr : op->kcell<T>();
        h.src    = src;
        h.dst    = dst;
        h.b      = b;
        h.mask_src = mask_src;
        h.skip     = skip;
        h.march    = op->d_mask == nullptr;
        if (dot)
          h.dot = *dot;
        if (which == 0 && op->tangent_faces() && op->fbc.radiation_faces && !op->d_temp)
          return fail(MPDG_ERR_ARG, "radiation faces need the linearisation temperature (mpdg_op_set_temperature)");
        if (which == 0 && op->solid)
          {
            if (int e = solid_apply<T>(op, mode, scale, dst, src, b, mask_src, skip, false))
              return e;
          }
        else if (which == 0 && op->d_vfield[0])
          {
            AdvLaunch<T> a;
            a.degree   = op->degree;
            a.mode     = mode;
            a.scale    = scale;
            a.p        = heat_velocity_params(op, false);
            a.grid     = heat_velocity_grid<T>(op);
            a.sync     = op->sync();
            a.src      = src;
            a.dst      = dst;
            a.b        = b;
            a.mask_src = mask_src;
            a.skip     = skip;
            MPDG_CUDA(adv_apply<T>(a, op->stream));
          }
        else
          MPDG_CUDA(heat_apply<T>(h, op->stream));
        if (which == 0 && op->tangent_faces())
          {
            HeatFaceLaunch<T> f;
            f.degree = op->degree;
            f.mode   = 0;
            f.scale  = scale;
            for (int d = 0; d < 3; ++d)
              f.hlen[d] = op->h[d];
            f.grid = h.grid;
            f.bc   = op->fbc;
            f.temp = op->d_temp;
            f.src  = src;
            f.dst  = dst;
            f.skip = skip;
            MPDG_CUDA(heat_faces<T>(f, op->stream));
          }
      }
    else if (op->kind == MPDG_REINIT)
      {
        if (!op->d_normal[0] || !op->d_normal[1] || !op->d_normal[2])
          return fail(MPDG_ERR_ARG, "the reinitialisation operator needs its normal field (mpdg_op_set_reinit)");
        // dst prepared for the atomics of the cell kernel: 0 (Set) or b (BPlus); Add adds in place
        if (mode == (int)OutMode::Set)
          MPDG_CUDA(vec_fill<T>(dst, T(0), op->ndofs, op->stream));
        else if (mode == (int)OutMode::BPlus && dst != b)
          MPDG_CUDA(cudaMemcpyAsync(dst, b, sizeof(T) * op->ndofs, cudaMemcpyDeviceToDevice, op->stream));
        MPDG_CUDA(reinit_integrate<T>(reinit_launch<T>(op, scale, src, dst, mask_src), 0, op->stream));
      }
    else
      {
        AdvLaunch<T> h;
        h.degree   = op->degree;
        h.mode     = mode;
        h.scale    = scale;
        h.p        = adv_params(op, op->theta - 1.0, which == 3);
        h.grid     = op->grid<T>();
        h.sync     = op->sync();
        h.src      = src;
        h.dst      = dst;
        h.b        = b;
        h.mask_src = mask_src;
        h.skip     = skip;
        // inflow rows (advection_diffusion_operator.cpp:543-578): src reads 0 there, the cell
        // terms skip those rows, and the row is the identity
        const bool hooks = which == 0 && op->n_inflow > 0 && op->with_bc && op->inflow_prepost;
        if (hooks)
          h.grid.cmask = op->d_mask_io;
        MPDG_CUDA(adv_apply<T>(h, op->stream));
        if (hooks)
          MPDG_CUDA(idx_add_scaled<T>(dst, src, op->d_in_idx, op->n_inflow, scale, op->stream));
      }
    return MPDG_OK;
  }

  // inverse diagonal: 1 on the inflow rows (advection_diffusion_operator.cpp:440-445)
  template <typename T>
  int
  inflow_unit_diagonal(mpdg_op *op, T *diag)
  {
    if (op->kind == MPDG_ADVDIFF && op->n_inflow > 0 && op->with_bc && op->inflow_prepost)
      MPDG_CUDA(idx_set<T>(diag, op->d_in_idx, nullptr, op->n_inflow, T(1), op->stream));
    return MPDG_OK;
  }

  template <typename T>
  int
  inverse_diagonal_cells(mpdg_op *op, T *diag);

  template <typename T>
  int
  inverse_diagonal(mpdg_op *op, T *diag)
  {
    if (int e = inverse_diagonal_cells<T>(op, diag))
      return e;
    return inflow_unit_diagonal<T>(op, diag);
  }

  template <typename T>
  int
  inverse_diagonal_cells(mpdg_op *op, T *diag)
  {
    const GridDesc g = op->grid();
    if (op->banded())
      {
        // diagonal of the banded projection, inverted with NormalVectorOperator's relative rule
        // (normal_vector_operator.cpp:318-321): |d| > 1e-14 max(1, |d|_inf) ? 1/d : 1
        double *d64 = std::is_same<T, double>::value ? reinterpret_cast<double *>(diag) : op->vec<double>("band_diag");
        if (!d64)
          return fail(MPDG_ERR_NOMEM, "diagonal work vector");
        MPDG_CUDA(vec_fill<double>(d64, 0.0, op->ndofs, op->stream));
        ReinitLaunch<double> r = band_launch<double>(op, 0, 1.0, nullptr, nullptr, 0);
        r.diag                 = d64;
        MPDG_CUDA(reinit_integrate<double>(r, 2, op->stream));
        MPDG_CUDA(vec_set_constrained<double>(d64, 1.0, g, op->stream));
        MPDG_CUDA(vec_absmax<double>(d64, op->ndofs, op->d_scal, op->reducer(), op->stream));
        MPDG_CUDA(vec_invert_rel<double>(d64, op->d_scal, op->ndofs, op->stream));
        if (!std::is_same<T, double>::value)
          MPDG_CUDA(vec_convert<T, double>(diag, d64, op->ndofs, op->stream));
        return MPDG_OK;
      }
    if (op->kind == MPDG_HEAT && (op->tangent_faces() || op->solid))
      {
        // cell and face parts summed in FP64, then inverted (|d| > 1e-10 ? 1/d : 1)
        if (op->fbc.radiation_faces && !op->d_temp)
          return fail(MPDG_ERR_ARG, "radiation faces need the linearisation temperature (mpdg_op_set_temperature)");
        if (op->solid && (!op->d_temp || !op->d_temp_old))
          return fail(MPDG_ERR_ARG, "the solidification tangent needs the temperature and the old temperature");
        double *d64 = std::is_same<T, double>::value ? reinterpret_cast<double *>(diag) : op->vec<double>("face_diag");
        if (!d64)
          return fail(MPDG_ERR_NOMEM, "diagonal work vector");
        if (op->solid)
          {
            MPDG_CUDA(vec_fill<double>(d64, 0.0, op->ndofs, op->stream));
            MPDG_CUDA(heat_solid_diagonal(g, op->degree, op->smat, op->dt, op->h, op->d_temp, op->d_temp_old, d64,
                                          op->stream));
            MPDG_CUDA(vec_set_constrained<double>(d64, 1.0, g, op->stream));
          }
        else
          MPDG_CUDA(heat_diagonal<double>(g, op->degree, heat_geom(op, op->rho_cp / op->dt), op->k,
                                          op->kcell<double>(), d64, false, 0.0, op->stream));
        HeatFaceLaunch<double> f;
        f.degree = op->degree;
        f.mode   = 2;
        for (int d = 0; d < 3; ++d)
          f.hlen[d] = op->h[d];
        f.grid = g;
        f.bc   = op->fbc;
        f.temp = op->d_temp;
        f.diag = d64;
        MPDG_CUDA(heat_faces<double>(f, op->stream));
        MPDG_CUDA(vec_invert<double>(d64, 1.0e-10, op->ndofs, op->stream));
        if (!std::is_same<T, double>::value)
          MPDG_CUDA(vec_convert<T, double>(diag, d64, op->ndofs, op->stream));
      }
    else if (op->kind == MPDG_HEAT && op->d_vfield[0])
      {
        // with a convection velocity: the per-cell diagonal of the whole tangent in FP64, then the
        // heat operator's inversion rule (|d| > 1e-10 ? 1/d : 1, constrained rows 1)
        double *f64 = std::is_same<T, double>::value ? reinterpret_cast<double *>(diag) : op->vec<double>("vf_diag");
        if (!f64)
          return fail(MPDG_ERR_NOMEM, "diagonal work vector");
        MPDG_CUDA(vec_fill<double>(f64, 0.0, op->ndofs, op->stream));
        MPDG_CUDA(adv_field_diagonal(g, op->degree, heat_velocity_params(op, false), f64, op->stream));
        MPDG_CUDA(vec_set_constrained<double>(f64, 1.0, g, op->stream));
        MPDG_CUDA(vec_invert<double>(f64, 1.0e-10, op->ndofs, op->stream));
        if (!std::is_same<T, double>::value)
          MPDG_CUDA(vec_convert<T, double>(diag, f64, op->ndofs, op->stream));
      }
    else if (op->kind == MPDG_HEAT)
      {
        MPDG_CUDA(heat_diagonal<T>(g, op->degree, heat_geom(op, op->rho_cp / op->dt), op->k, op->kcell<T>(), diag,
                                   true, 1.0e-10, op->stream));
      }
    else
      {
        if (op->kind == MPDG_REINIT)
          {
            if (!op->d_normal[0] || !op->d_normal[1] || !op->d_normal[2])
              return fail(MPDG_ERR_ARG, "the reinitialisation operator needs its normal field (mpdg_op_set_reinit)");
            double *r64 = std::is_same<T, double>::value ? reinterpret_cast<double *>(diag) : op->vec<double>("reinit_diag");
            if (!r64)
              return fail(MPDG_ERR_NOMEM, "diagonal work vector");
            MPDG_CUDA(vec_fill<double>(r64, 0.0, op->ndofs, op->stream));
            ReinitLaunch<double> r = reinit_launch<double>(op, 1.0, nullptr, nullptr, 0);
            r.diag                 = r64;
            MPDG_CUDA(reinit_integrate<double>(r, 2, op->stream));
            MPDG_CUDA(vec_set_constrained<double>(r64, 1.0, g, op->stream));
            MPDG_CUDA(vec_absmax<double>(r64, op->ndofs, op->d_scal, op->reducer(), op->stream));
            MPDG_CUDA(vec_invert_rel<double>(r64, op->d_scal, op->ndofs, op->stream));
            if (!std::is_same<T, double>::value)
              MPDG_CUDA(vec_convert<T, double>(diag, r64, op->ndofs, op->stream));
            return MPDG_OK;
          }
        if (op->d_vfield[0])
          {
            // DoF-vector velocity: the per-cell diagonal in FP64, inverted with the advection rule
            double *f64 = std::is_same<T, double>::value ? reinterpret_cast<double *>(diag) : op->vec<double>("vf_diag");
            if (!f64)
              return fail(MPDG_ERR_NOMEM, "diagonal work vector");
            MPDG_CUDA(vec_fill<double>(f64, 0.0, op->ndofs, op->stream));
            MPDG_CUDA(adv_field_diagonal(g, op->degree, adv_params(op, 0, false), f64, op->stream));
            MPDG_CUDA(adv_supg_diagonal<double>(g, op->degree, adv_params(op, 0, false), f64, op->stream));
            MPDG_CUDA(vec_set_constrained<double>(f64, 1.0, g, op->stream));
            MPDG_CUDA(vec_absmax<double>(f64, op->ndofs, op->d_scal, op->reducer(), op->stream));
            MPDG_CUDA(vec_invert_rel<double>(f64, op->d_scal, op->ndofs, op->stream));
            if (!std::is_same<T, double>::value)
              MPDG_CUDA(vec_convert<T, double>(diag, f64, op->ndofs, op->stream));
            return MPDG_OK;
          }
        // the SUPG part sums terms of both signs: an FP32 diagonal is computed in FP64 and rounded once
        double *d64 = std::is_same<T, double>::value ? reinterpret_cast<double *>(diag)
                                                     : (op->supg ? op->vec<double>("supg_diag") : nullptr);
        if (d64)
          {
            MPDG_CUDA(adv_diagonal<double>(g, op->degree, adv_params(op, 0, false), d64, op->stream));
            MPDG_CUDA(adv_supg_diagonal<double>(g, op->degree, adv_params(op, 0, false), d64, op->stream));
            MPDG_CUDA(vec_absmax<double>(d64, op->ndofs, op->d_scal, op->reducer(), op->stream));
            MPDG_CUDA(vec_invert_rel<double>(d64, op->d_scal, op->ndofs, op->stream));
            if (!std::is_same<T, double>::value)
              MPDG_CUDA(vec_convert<T, double>(diag, d64, op->ndofs, op->stream));
          }
        else if (op->supg)
          return fail(MPDG_ERR_NOMEM, "diagonal work vector");
        else
          {
            MPDG_CUDA(adv_diagonal<T>(g, op->degree, adv_params(op, 0, false), diag, op->stream));
            MPDG_CUDA(vec_absmax<T>(diag, op->ndofs, op->d_scal, op->reducer(), op->stream));
            MPDG_CUDA(vec_invert_rel<T>(diag, op->d_scal, op->ndofs, op->stream));
          }
      }
    return MPDG_OK;
  }

  int
  check_op(const mpdg_op *op)
  {
    if (!op)
      return fail(MPDG_ERR_ARG, "null operator handle");
    return MPDG_OK;
  }

  // Copies between the operator's device data and the host, ordered on the operator's stream (which
  // may be a non-blocking stream: a plain cudaMemcpy on the legacy stream would not wait for its work)
  int
  stream_copy(const mpdg_op *op, void *dst, const void *src, size_t bytes, cudaMemcpyKind kind)
  {
    MPDG_CUDA(cudaMemcpyAsync(dst, src, bytes, kind, op->stream));
    MPDG_CUDA(cudaStreamSynchronize(op->stream));
    return MPDG_OK;
  }

  // Iterations to enqueue before the next convergence check of the CG loop.  The residual reduction
  // rate of the previous batch, extrapolated to the tolerance, bounds it from above, so that few of
  // the enqueued iterations run after convergence (each costs its launches, which return at once);
  // otherwise the batch doubles up to 64.
  inline int
  next_cg_batch(int prev, int it, double res, double tol, int it_prev, double res_prev)
  {
    const int cap = std::min(2 * prev, 64);
    if (it > it_prev && res > 0.0 && res_prev > res && tol > 0.0 && tol < res)
      {
        const double need = std::log(tol / res) / (std::log(res / res_prev) / (it - it_prev));
        if (need < cap)
          return std::max(2, (int)std::ceil(need));
      }
    return cap;
  }

  // whether the one-sweep PCG iteration (cgfused.cu) covers this operator: heat, FE_Q(2), Dirichlet
  // on whole faces only, no boundary-face terms, constant material
  bool
  fused_cg_applies(const mpdg_op *op)
  {
    return op->fused_cg && op->kind == MPDG_HEAT && op->degree == 2 && op->d_mask == nullptr && op->with_bc &&
           !op->tangent_faces() && !op->solid && !op->banded() && !op->d_vfield[0];
  }

  // Preconditioned CG with one launch per iteration (cgfused.cu): the same iterates as cg_solve in
  // exact arithmetic, vectors in the padded layout of the sweep, x copied in and out once per solve.
  template <typename T>
  int
  cg_solve_fused(mpdg_op *op, T *x, const T *b, const T *invd, int max_it, double abs_tol, double rel_tol,
                 mpdg_solve_info *info, const char *tag, bool x_zero)
  {
    const std::string t(tag);
    FusedCG<T>        f;
    for (int d = 0; d < 3; ++d)
      {
        f.m[d] = op->m[d];
        f.n[d] = op->degree * op->m[d] + 1;
      }
    f.P0     = FusedCG<T>::padded_pitch(f.n[0]);
    f.faces  = op->faces;
    const HeatGeom geo = heat_geom(op, op->rho_cp / op->dt);
    f.mass_coef = geo.mass_coef;
    f.geo[0] = geo.cx;
    f.geo[1] = geo.cy;
    f.geo[2] = geo.cz;
    f.kconst = op->k;
    f.kcell  = op->kcell<T>();
    int dev = 0, sms = 148;
    MPDG_CUDA(cudaGetDevice(&dev));
    MPDG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    f.plan(sms);
    const long long plen = f.padded_len(), rows = (long long)f.n[1] * f.n[2];
    T *X = op->vec<T>(t + "fX", plen), *D = op->vec<T>(t + "fD", plen);
    T *R[2] = {op->vec<T>(t + "fR0", plen), op->vec<T>(t + "fR1", plen)};
    T *P[2] = {op->vec<T>(t + "fP0", plen), op->vec<T>(t + "fP1", plen)};
    T *V[2] = {op->vec<T>(t + "fV0", plen), op->vec<T>(t + "fV1", plen)};
    double    *part  = op->vec<double>(t + "fpart", (size_t)5 * f.ntiles);
    long long *range = op->vec<long long>(t + "frange", f.range.size());
    if (!range)
      return fail(MPDG_ERR_NOMEM, "fused CG ranges");
    MPDG_CUDA(cudaMemcpyAsync(range, f.range.data(), sizeof(long long) * f.range.size(), cudaMemcpyHostToDevice,
                              op->stream));
    f.d_range = range;
    double *hist = op->vec<double>(t + "hist", (size_t)max_it + 2);
    if (!X || !D || !R[0] || !R[1] || !P[0] || !P[1] || !V[0] || !V[1] || !part || !hist)
      return fail(MPDG_ERR_NOMEM, "fused CG work vectors");
    // r_0 = b - A x_0 (b itself for a zero initial guess), x_0 and the inverse diagonal, padded
    if (x_zero)
      MPDG_CUDA(pad_rows<T, T>(R[0], b, f.n[0], f.P0, rows, op->stream));
    else
      {
        T *r = op->vec<T>(t + "r");
        if (!r)
          return fail(MPDG_ERR_NOMEM, "CG work vector");
        if (int e = apply<T>(op, (int)OutMode::BPlus, -1.0, r, x, b, 1))
          return e;
        MPDG_CUDA(pad_rows<T, T>(R[0], r, f.n[0], f.P0, rows, op->stream));
      }
    if (x_zero)
      MPDG_CUDA(vec_fill<T>(X, T(0), plen, op->stream));
    else
      MPDG_CUDA(pad_rows<T, T>(X, x, f.n[0], f.P0, rows, op->stream));
    if (invd)
      MPDG_CUDA(pad_rows<T, T>(D, invd, f.n[0], f.P0, rows, op->stream));
    else
      MPDG_CUDA(vec_fill<T>(D, T(1), plen, op->stream));
    CUtensorMap mX, mD, mR[2], mP[2], mV[2];
    int         me = f.make_map(&mX, X) | f.make_map(&mD, D);
    for (int i = 0; i < 2; ++i)
      me |= f.make_map(&mR[i], R[i]) | f.make_map(&mP[i], P[i]) | f.make_map(&mV[i], V[i]);
    if (me)
      return fail(MPDG_ERR_CUDA, "cuTensorMapEncodeTiled failed for the fused CG vectors");
    CGState st{};
    st.abs_tol = abs_tol;
    st.rel_tol = rel_tol;
    st.max_it  = max_it;
    *op->h_cg  = st;
    MPDG_CUDA(cudaMemcpyAsync(op->d_cg, op->h_cg, sizeof(CGState), cudaMemcpyHostToDevice, op->stream));
    unsigned *counter = op->d_sync + 1;
    MPDG_CUDA(f.sweep(true, mR[0], mV[0], mP[0], mX, mD, X, R[1], P[0], V[0], op->d_cg, part, counter, hist,
                      op->d_err, op->spin_limit, op->stream));
    long long k = 1; // next sweep
    int       batch = 4, it_prev = 0;
    double    res_prev = -1.0;
    for (;;)
      {
        MPDG_CUDA(cudaMemcpyAsync(op->h_cg, op->d_cg, sizeof(CGState), cudaMemcpyDeviceToHost, op->stream));
        MPDG_CUDA(cudaStreamSynchronize(op->stream));
        const CGState &cur = *op->h_cg;
        if (cur.done)
          break;
        if (k > 1)
          {
            batch    = next_cg_batch(batch, cur.it, cur.res, cur.tol, it_prev, it_prev == 0 ? cur.res0 : res_prev);
            it_prev  = cur.it;
            res_prev = cur.res;
          }
        for (int j = 0; j < batch; ++j, ++k)
          {
            const int i = (int)((k - 1) & 1), o = (int)(k & 1);
            MPDG_CUDA(f.sweep(false, mR[i], mV[i], mP[i], mX, mD, X, R[o], P[o], V[o], op->d_cg, part, counter,
                              hist, op->d_err, op->spin_limit, op->stream));
          }
      }
    MPDG_CUDA(unpad_rows<T, T>(x, X, f.n[0], f.P0, rows, op->stream));
    const CGState &fin = *op->h_cg;
    if (info)
      {
        info->iterations       = fin.it;
        info->status           = fin.done == 1 ? MPDG_OK : MPDG_ERR_NOT_CONVERGED;
        info->initial_residual = fin.res0;
        info->final_residual   = fin.res;
        if (info->history && info->history_capacity > 0)
          {
            const int cnt = std::min(info->history_capacity, fin.it + 1);
            if (int e = stream_copy(op, info->history, hist, sizeof(double) * cnt, cudaMemcpyDeviceToHost))
              return e;
          }
      }
    MPDG_CUDA(cudaStreamSynchronize(op->stream));
    int dev_err = 0;
    if (int e = stream_copy(op, &dev_err, op->d_err, sizeof(int), cudaMemcpyDeviceToHost))
      return e;
    if (dev_err)
      return fail(MPDG_ERR_TIMEOUT, "a bounded device wait gave up during the CG solve");
    if (fin.done != 1)
      return fail(MPDG_ERR_NOT_CONVERGED, "CG did not converge in " + std::to_string(fin.it) + " iterations");
    return MPDG_OK;
  }

  // ---------------------------------------------------------------------------------------------
  // Preconditioned CG (dealii::SolverCG semantics), all scalars on the device.  x_zero: the caller
  // guarantees x == 0, so the initial residual is b itself and its apply is skipped; b_scratch (with
  // x_zero only): b is the caller's scratch and becomes the residual vector in place.
  template <typename T>
  int
  cg_solve(mpdg_op *op, T *x, const T *b, const T *invd, int max_it, double abs_tol, double rel_tol,
           mpdg_solve_info *info, const char *tag, bool x_zero = false, T *b_scratch = nullptr)
  {
    if (fused_cg_applies(op))
      return cg_solve_fused<T>(op, x, b, invd, max_it, abs_tol, rel_tol, info, tag, x_zero);
    const long long n = op->ndofs;
    const std::string t(tag);
    T *r = x_zero && b_scratch == b ? b_scratch : op->vec<T>(t + "r");
    T *p = op->vec<T>(t + "p"), *v = op->vec<T>(t + "v");
    if (!r || !p || !v)
      return fail(MPDG_ERR_NOMEM, "CG work vectors");
    double *hist = op->vec<double>(t + "hist", (size_t)max_it + 2);
    if (!hist)
      return fail(MPDG_ERR_NOMEM, "CG history");
    CGState st{};
    st.abs_tol = abs_tol;
    st.rel_tol = rel_tol;
    st.max_it  = max_it;
    *op->h_cg  = st;
    MPDG_CUDA(cudaMemcpyAsync(op->d_cg, op->h_cg, sizeof(CGState), cudaMemcpyHostToDevice, op->stream));
    // r = b - A x
    if (x_zero)
      {
        if (r != b)
          MPDG_CUDA(cudaMemcpyAsync(r, b, sizeof(T) * n, cudaMemcpyDeviceToDevice, op->stream));
      }
    else if (int e = apply<T>(op, (int)OutMode::BPlus, -1.0, r, x, b, 1))
      return e;
    MPDG_CUDA(cg_init<T>(r, invd, p, op->d_cg, hist, op->reducer(), n, op->stream));
    // heat operators without a per-DoF mask fuse p^T A p into the apply and set alpha on the device
    // (not the narrow-band projection, whose apply is the point-wise kernel)
    const bool fused = op->kind == MPDG_HEAT && op->d_part != nullptr && !op->tangent_faces() && !op->solid &&
                       !op->banded() && !op->d_vfield[0] && heat_apply_fuses_dot(op->degree, op->d_mask != nullptr, true);
    DotSink    sink;
    sink.part  = op->d_part;
    sink.alpha = &op->d_cg->alpha;
    sink.rho   = &op->d_cg->rho;
    int    batch = 4, it_prev = 0;
    double res_prev = -1.0;
    for (;;)
      {
        for (int k = 0; k < batch; ++k)
          {
            MPDG_CUDA(cg_update_p<T>(r, invd, p, op->d_cg, n, op->stream));
            if (int e = apply<T>(op, (int)OutMode::Set, 1.0, v, p, nullptr, 1, 0, &op->d_cg->done,
                                 fused ? &sink : nullptr))
              return e;
            if (!fused)
              MPDG_CUDA(cg_alpha<T>(p, v, op->d_cg, op->reducer(), n, op->stream));
            MPDG_CUDA(cg_update_xr<T>(x, r, p, v, invd, op->d_cg, hist, op->reducer(), n, op->stream));
          }
        MPDG_CUDA(cudaMemcpyAsync(op->h_cg, op->d_cg, sizeof(CGState), cudaMemcpyDeviceToHost, op->stream));
        MPDG_CUDA(cudaStreamSynchronize(op->stream));
        const CGState &cur = *op->h_cg;
        if (cur.done)
          break;
        batch    = next_cg_batch(batch, cur.it, cur.res, cur.tol, it_prev, it_prev == 0 ? cur.res0 : res_prev);
        it_prev  = cur.it;
        res_prev = cur.res;
      }
    const CGState &f = *op->h_cg;
    if (info)
      {
        info->iterations       = f.it;
        info->status           = f.done == 1 ? MPDG_OK : MPDG_ERR_NOT_CONVERGED;
        info->initial_residual = f.res0;
        info->final_residual   = f.res;
        if (info->history && info->history_capacity > 0)
          {
            const int cnt = std::min(info->history_capacity, f.it + 1);
            if (int e = stream_copy(op, info->history, hist, sizeof(double) * cnt, cudaMemcpyDeviceToHost))
              return e;
          }
      }
    int dev_err = 0;
    if (int e = stream_copy(op, &dev_err, op->d_err, sizeof(int), cudaMemcpyDeviceToHost))
      return e;
    if (dev_err)
      return fail(MPDG_ERR_TIMEOUT, "a bounded device wait gave up during the CG solve");
    if (f.done != 1)
      return fail(MPDG_ERR_NOT_CONVERGED, "CG did not converge in " + std::to_string(f.it) + " iterations");
    return MPDG_OK;
  }

  // ---------------------------------------------------------------------------------------------
  // Right-preconditioned restarted GMRES (dealii::SolverGMRES with right_preconditioning = true).
  template <typename T>
  int
  gmres_solve(mpdg_op *op, T *x, const T *b, const T *invd, int max_it, double abs_tol, double rel_tol, int restart,
              mpdg_solve_info *info, const char *tag)
  {
    const long long   n = op->ndofs;
    const std::string t(tag);
    const int         m = std::max(1, std::min(restart, 31));
    std::vector<T *>  V(m + 1);
    for (int i = 0; i <= m; ++i)
      {
        V[i] = op->vec<T>(t + "V" + std::to_string(i));
        if (!V[i])
          return fail(MPDG_ERR_NOMEM, "GMRES basis");
      }
    T *z = op->vec<T>(t + "z");
    if (!z)
      return fail(MPDG_ERR_NOMEM, "GMRES work vector");
    double             *d_h = op->d_scal; // [0..m+1]
    std::vector<double> H((m + 1) * m, 0.0), cs(m), sn(m), g(m + 1), y(m);
    std::vector<double> hist;
    Control             ctl{max_it, abs_tol, rel_tol};
    int                 it = 0, state = 0;
    double              res0 = 0.0, res = 0.0;
    bool                first = true;
    const Reducer       red   = op->reducer();
    auto fetch = [&](int cnt) -> int {
      MPDG_CUDA(cudaMemcpyAsync(op->h_scal, d_h, sizeof(double) * cnt, cudaMemcpyDeviceToHost, op->stream));
      MPDG_CUDA(cudaStreamSynchronize(op->stream));
      return MPDG_OK;
    };
    for (;;)
      {
        if (int e = apply<T>(op, (int)OutMode::BPlus, -1.0, V[0], x, b, 1))
          return e;
        const T *v0 = V[0];
        MPDG_CUDA(vec_multidot<T>(&v0, &v0, 1, n, d_h, red, op->stream));
        if (int e = fetch(1))
          return e;
        const double beta = std::sqrt(op->h_scal[0]);
        if (first)
          {
            res0  = beta;
            first = false;
            hist.push_back(beta);
          }
        res   = beta;
        state = ctl.check(it, beta);
        if (state != 0)
          break;
        MPDG_CUDA(vec_axpby<T>(V[0], 1.0 / beta, V[0], 0.0, nullptr, n, op->stream));
        std::fill(g.begin(), g.end(), 0.0);
        std::fill(H.begin(), H.end(), 0.0);
        g[0]  = beta;
        int j = 0;
        for (; j < m; ++j)
          {
            ++it;
            const T *zin = V[j];
            if (invd)
              {
                MPDG_CUDA(vec_scale<T>(z, V[j], invd, n, op->stream));
                zin = z;
              }
            if (int e = apply<T>(op, (int)OutMode::Set, 1.0, V[j + 1], zin, nullptr, 1))
              return e;
            std::vector<const T *> Vc(V.begin(), V.begin() + j + 1);
            MPDG_CUDA(vec_dots_against<T>(V[j + 1], Vc.data(), j + 1, n, d_h, red, op->stream));
            MPDG_CUDA(vec_orth_update<T>(V[j + 1], Vc.data(), d_h, j + 1, n, d_h + j + 1, red, op->stream));
            if (int e = fetch(j + 2))
              return e;
            const double hn = std::sqrt(std::max(0.0, op->h_scal[j + 1]));
            for (int i = 0; i <= j; ++i)
              H[i * m + j] = op->h_scal[i];
            H[(j + 1) * m + j] = hn;
            if (hn > 0.0)
              MPDG_CUDA(vec_axpby<T>(V[j + 1], 1.0 / hn, V[j + 1], 0.0, nullptr, n, op->stream));
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
            H[j * m + j]       = r;
            H[(j + 1) * m + j] = 0.0;
            g[j + 1]           = -sn[j] * g[j];
            g[j]               = cs[j] * g[j];
            res                = std::abs(g[j + 1]);
            hist.push_back(res);
            state = ctl.check(it, res);
            if (state != 0 || hn == 0.0)
              {
                ++j;
                break;
              }
          }
        for (int i = j - 1; i >= 0; --i)
          {
            double s = g[i];
            for (int kk = i + 1; kk < j; ++kk)
              s -= H[i * m + kk] * y[kk];
            y[i] = s / H[i * m + i];
          }
        std::memcpy(op->h_scal, y.data(), sizeof(double) * j);
        MPDG_CUDA(cudaMemcpyAsync(d_h, op->h_scal, sizeof(double) * j, cudaMemcpyHostToDevice, op->stream));
        MPDG_CUDA(vec_fill<T>(z, T(0), n, op->stream));
        std::vector<const T *> Vc(V.begin(), V.begin() + j);
        MPDG_CUDA(vec_multiaxpy<T>(z, Vc.data(), d_h, j, n, 1.0, op->stream));
        if (invd)
          MPDG_CUDA(vec_scale<T>(z, z, invd, n, op->stream));
        MPDG_CUDA(vec_axpby<T>(x, 1.0, x, 1.0, z, n, op->stream));
        MPDG_CUDA(cudaStreamSynchronize(op->stream));
        if (state != 0)
          break;
      }
    if (info)
      {
        info->iterations       = it;
        info->status           = state == 1 ? MPDG_OK : MPDG_ERR_NOT_CONVERGED;
        info->initial_residual = res0;
        info->final_residual   = res;
        if (info->history && info->history_capacity > 0)
          {
            const int cnt = std::min<int>(info->history_capacity, (int)hist.size());
            std::memcpy(info->history, hist.data(), sizeof(double) * cnt);
          }
      }
    if (state != 1)
      return fail(MPDG_ERR_NOT_CONVERGED, "GMRES did not converge in " + std::to_string(it) + " iterations");
    return MPDG_OK;
  }

  template <typename T>
  int
  solve_typed(mpdg_op *op, T *x, const T *b, const mpdg_solver_params *prm, mpdg_solve_info *info, const char *tag)
  {
    if (!prm || !x || !b)
      return fail(MPDG_ERR_ARG, "null argument to solve");
    T *invd = nullptr;
    if (prm->precond == MPDG_PRECOND_JACOBI)
      {
        invd = op->vec<T>(std::string(tag) + "invd");
        if (!invd)
          return fail(MPDG_ERR_NOMEM, "inverse diagonal");
        // JacobiPreconditioner::update (preconditioner_jacobi.hpp:65-69) once per solve
        if (int e = inverse_diagonal<T>(op, invd))
          return e;
      }
    const int max_it = prm->max_it > 0 ? prm->max_it : 10000;
    if (prm->solver == MPDG_CG)
      return cg_solve<T>(op, x, b, invd, max_it, prm->abs_tol, prm->rel_tol, info, tag);
    if (prm->solver == MPDG_GMRES)
      return gmres_solve<T>(op, x, b, invd, max_it, prm->abs_tol, prm->rel_tol, prm->restart > 0 ? prm->restart : 30,
                            info, tag);
    return fail(MPDG_ERR_ARG, "unknown solver kind");
  }
} // namespace

extern "C" {

const char *
mpdg_last_error(void)
{
  return g_last_error.c_str();
}

int
mpdg_op_create(const mpdg_mesh_desc *mesh, const mpdg_op_params *params, mpdg_op **out)
{
  if (!mesh || !params || !out)
    return fail(MPDG_ERR_ARG, "null argument to mpdg_op_create");
  *out = nullptr;
  if (params->kind != MPDG_HEAT && params->kind != MPDG_ADVDIFF && params->kind != MPDG_REINIT)
    return fail(MPDG_ERR_ARG, "unknown operator kind");
  if (params->kind == MPDG_REINIT && (mesh->degree < 1 || mesh->degree > 3))
    return fail(MPDG_ERR_UNSUPPORTED, "reinitialisation operator: FE_Q degree must be 1..3");
  if (params->kind == MPDG_HEAT && (mesh->degree < 1 || mesh->degree > 4))
    return fail(MPDG_ERR_UNSUPPORTED, "heat operator: FE_Q degree must be 1..4");
  if (params->kind == MPDG_ADVDIFF && (mesh->degree < 1 || mesh->degree > 3))
    return fail(MPDG_ERR_UNSUPPORTED, "advection-diffusion operator: FE_Q degree must be 1..3");
  for (int d = 0; d < 3; ++d)
    if (mesh->cells[d] < 1 || !(mesh->length[d] > 0.0))
      return fail(MPDG_ERR_ARG, "mesh cells and lengths must be positive");
  if (!(params->dt > 0.0))
    return fail(MPDG_ERR_ZERO_DT, "time increment must be positive (ExcZeroTimeIncrement)");
  const long long n0 = (long long)mesh->degree * mesh->cells[0] + 1, n1 = (long long)mesh->degree * mesh->cells[1] + 1,
                  n2 = (long long)mesh->degree * mesh->cells[2] + 1;
  // lattice indices are 32-bit in the kernels
  if (n0 * n1 * n2 >= (1LL << 31))
    return fail(MPDG_ERR_UNSUPPORTED, "an operator holds fewer than 2^31 DoFs");

  mpdg_op *op = new mpdg_op();
  op->kind    = params->kind;
  op->degree  = mesh->degree;
  for (int d = 0; d < 3; ++d)
    {
      op->m[d]      = mesh->cells[d];
      op->origin[d] = mesh->origin[d];
      op->length[d] = mesh->length[d];
      op->h[d]      = mesh->length[d] / mesh->cells[d];
    }
  op->faces  = mesh->dirichlet_faces & 63u;
  op->rho_cp = params->rho_cp;
  op->dt     = params->dt;
  op->k      = params->conductivity;
  op->theta  = params->theta;
  op->eps    = params->diffusivity;
  for (int i = 0; i < 12; ++i)
    op->vel[i] = params->velocity[i];
  int brick32[3];
  if (op->kind == MPDG_HEAT)
    {
      heat_brick_shape<double>(op->degree, op->brick, mesh->dirichlet_mask == nullptr);
      heat_brick_shape<float>(op->degree, brick32, mesh->dirichlet_mask == nullptr);
    }
  else
    {
      adv_brick_shape<double>(op->degree, op->brick);
      adv_brick_shape<float>(op->degree, brick32);
    }
  for (int d = 0; d < 3; ++d)
    {
      op->nbr[d]   = (op->m[d] + op->brick[d] - 1) / op->brick[d];
      op->nbr32[d] = (op->m[d] + brick32[d] - 1) / brick32[d];
    }
  op->ndofs             = n0 * n1 * n2;
  op->ncells            = (long long)op->m[0] * op->m[1] * op->m[2];
  // brick flags and fused-dot partials serve the FP64 and the FP32 apply (and, for a heat operator
  // at k <= 3, the advection-form kernels of its convection velocity, on their own bricks)
  long long nbrk = std::max((long long)op->nbr[0] * op->nbr[1] * op->nbr[2],
                            (long long)op->nbr32[0] * op->nbr32[1] * op->nbr32[2]);
  if (op->kind == MPDG_HEAT && op->degree <= 3)
    for (int prec = 0; prec < 2; ++prec)
      {
        int sh[3];
        if (prec == 0)
          adv_brick_shape<double>(op->degree, sh);
        else
          adv_brick_shape<float>(op->degree, sh);
        long long nb = 1;
        for (int d = 0; d < 3; ++d)
          nb *= (op->m[d] + sh[d] - 1) / sh[d];
        nbrk = std::max(nbrk, nb);
      }
  auto            clean = [&](int code, const std::string &msg) {
    mpdg_op_destroy(op);
    return fail(code, msg);
  };
  if (cudaMalloc(&op->d_sync, sizeof(unsigned) * (3 + nbrk)) != cudaSuccess ||
      cudaMalloc(&op->d_err, sizeof(int)) != cudaSuccess ||
      cudaMalloc(&op->d_red, sizeof(double) * RED_BLOCKS * 40) != cudaSuccess ||
      cudaMalloc(&op->d_scal, sizeof(double) * 64) != cudaSuccess ||
      cudaMalloc(&op->d_cg, sizeof(CGState)) != cudaSuccess ||
      cudaMallocHost(&op->h_cg, sizeof(CGState)) != cudaSuccess ||
      cudaMallocHost(&op->h_scal, sizeof(double) * 64) != cudaSuccess)
    return clean(MPDG_ERR_NOMEM, "device allocation in mpdg_op_create");
  if (op->kind == MPDG_HEAT && cudaMalloc(&op->d_part, sizeof(double) * nbrk) != cudaSuccess)
    return clean(MPDG_ERR_NOMEM, "fused dot partials");
  op->sync_cap = nbrk;
  if (cudaMemset(op->d_sync, 0, sizeof(unsigned) * (3 + nbrk)) != cudaSuccess ||
      cudaMemset(op->d_err, 0, sizeof(int)) != cudaSuccess)
    return clean(MPDG_ERR_CUDA, "cudaMemset in mpdg_op_create");
  if (mesh->dirichlet_mask)
    {
      if (cudaMalloc(&op->d_mask, op->ndofs) != cudaSuccess)
        return clean(MPDG_ERR_NOMEM, "Dirichlet mask");
      if (cudaMemcpy(op->d_mask, mesh->dirichlet_mask, op->ndofs, cudaMemcpyHostToDevice) != cudaSuccess)
        return clean(MPDG_ERR_CUDA, "Dirichlet mask copy");
    }
  if (op->kind == MPDG_HEAT && params->conductivity_cells)
    {
      std::vector<float> k32(op->ncells);
      for (long long c = 0; c < op->ncells; ++c)
        k32[c] = (float)params->conductivity_cells[c];
      if (cudaMalloc(&op->d_k64, sizeof(double) * op->ncells) != cudaSuccess ||
          cudaMalloc(&op->d_k32, sizeof(float) * op->ncells) != cudaSuccess)
        return clean(MPDG_ERR_NOMEM, "conductivity field");
      if (cudaMemcpy(op->d_k64, params->conductivity_cells, sizeof(double) * op->ncells, cudaMemcpyHostToDevice) !=
            cudaSuccess ||
          cudaMemcpy(op->d_k32, k32.data(), sizeof(float) * op->ncells, cudaMemcpyHostToDevice) != cudaSuccess)
        return clean(MPDG_ERR_CUDA, "conductivity copy");
    }
  (void)tables(op->degree); // build the 1-D tables once
  // the set-up above ran on the legacy stream; the operator's stream may not wait for it
  if (cudaDeviceSynchronize() != cudaSuccess)
    return clean(MPDG_ERR_CUDA, "set-up synchronisation in mpdg_op_create");
  *out = op;
  return MPDG_OK;
}

int
mpdg_op_destroy(mpdg_op *op)
{
  if (!op)
    return MPDG_OK;
  if (op->stream)
    cudaStreamSynchronize(op->stream);
  else
    cudaDeviceSynchronize();
  cudaFree(op->d_mask_io);
  cudaFree(op->d_in_idx);
  cudaFree(op->d_in_val);
  for (auto &kv : op->ws)
    cudaFree(kv.second.first);
  cudaFree(op->d_sync);
  cudaFree(op->d_err);
  cudaFree(op->d_red);
  cudaFree(op->d_part);
  for (cudaEvent_t e : op->ev)
    cudaEventDestroy(e);
  if (op->s_h2d)
    cudaStreamDestroy(op->s_h2d);
  if (op->s_d2h)
    cudaStreamDestroy(op->s_d2h);
  cudaFree(op->d_scal);
  cudaFree(op->d_cg);
  cudaFree(op->d_mask);
  cudaFree(op->d_k64);
  cudaFree(op->d_k32);
  if (op->h_cg)
    cudaFreeHost(op->h_cg);
  if (op->h_scal)
    cudaFreeHost(op->h_scal);
  delete op;
  return MPDG_OK;
}

int64_t
mpdg_op_n_dofs(const mpdg_op *op)
{
  return op ? op->ndofs : -1;
}

int64_t
mpdg_op_n_cells(const mpdg_op *op)
{
  return op ? op->ncells : -1;
}

int
mpdg_op_set_stream(mpdg_op *op, void *stream)
{
  if (int e = check_op(op))
    return e;
  op->stream = static_cast<cudaStream_t>(stream);
  return MPDG_OK;
}

int
mpdg_op_reset_time_increment(mpdg_op *op, double dt)
{
  if (int e = check_op(op))
    return e;
  if (!(dt > 0.0))
    return fail(MPDG_ERR_ZERO_DT, "time increment must be positive (ExcZeroTimeIncrement)");
  op->dt = dt;
  return MPDG_OK;
}

int
mpdg_op_reset_dof_index(mpdg_op *op, int with_dirichlet)
{
  if (int e = check_op(op))
    return e;
  op->with_bc = with_dirichlet != 0;
  return MPDG_OK;
}

int
mpdg_op_set_conductivity(mpdg_op *op, const double *k_cells)
{
  if (int e = check_op(op))
    return e;
  if (op->kind != MPDG_HEAT || !k_cells)
    return fail(MPDG_ERR_ARG, "conductivity applies to the heat operator");
  if (op->d_vfield[0])
    return fail(MPDG_ERR_UNSUPPORTED, "a per-cell conductivity with a convection velocity is not supported");
  if (!op->d_k64)
    {
      if (cudaMalloc(&op->d_k64, sizeof(double) * op->ncells) != cudaSuccess ||
          cudaMalloc(&op->d_k32, sizeof(float) * op->ncells) != cudaSuccess)
        return fail(MPDG_ERR_NOMEM, "conductivity field");
    }
  MPDG_CUDA(cudaMemcpyAsync(op->d_k64, k_cells, sizeof(double) * op->ncells, cudaMemcpyDeviceToDevice, op->stream));
  MPDG_CUDA(vec_convert<float, double>(op->d_k32, op->d_k64, op->ncells, op->stream));
  return MPDG_OK;
}

int
mpdg_op_set_heat_bc(mpdg_op *op, const mpdg_heat_bc *bc)
{
  if (int e = check_op(op))
    return e;
  if (op->kind != MPDG_HEAT || !bc)
    return fail(MPDG_ERR_ARG, "boundary-face terms apply to the heat operator");
  const uint32_t conv = bc->convection_faces, rad = bc->radiation_faces, neu = bc->neumann_faces;
  if ((conv | rad | neu) & ~63u)
    return fail(MPDG_ERR_ARG, "face masks have 6 bits");
  if (neu & (conv | rad))
    return fail(MPDG_ERR_ARG, "a face cannot carry both a Neumann flux and radiation / convection");
  if ((conv | rad | neu) & op->faces)
    return fail(MPDG_ERR_ARG, "a Dirichlet face cannot carry boundary-face terms");
  HeatFaceBC f;
  f.convection_faces                = conv;
  f.radiation_faces                 = rad;
  f.neumann_faces                   = neu;
  f.convection_coefficient          = bc->convection_coefficient;
  f.convection_temperature_infinity = bc->convection_temperature_infinity;
  f.emissivity_sigma                = bc->emissivity * 5.670374419e-8; // Stefan-Boltzmann, W/(m^2 K^4)
  f.radiation_temperature_infinity  = bc->radiation_temperature_infinity;
  for (int i = 0; i < 6; ++i)
    f.neumann_flux[i] = bc->neumann_flux[i];
  op->fbc = f;
  return MPDG_OK;
}

int
mpdg_op_set_solidification(mpdg_op *op, const mpdg_solid_liquid *mat)
{
  if (int e = check_op(op))
    return e;
  if (op->kind != MPDG_HEAT)
    return fail(MPDG_ERR_ARG, "temperature-dependent material applies to the heat operator");
  if (!mat)
    {
      op->solid = false;
      return MPDG_OK;
    }
  if (op->d_vfield[0])
    return fail(MPDG_ERR_UNSUPPORTED, "temperature-dependent material with a convection velocity is not supported");
  if (op->degree > 3)
    return fail(MPDG_ERR_UNSUPPORTED, "temperature-dependent material supports FE_Q degree 1..3");
  if (!(mat->liquid_density > 0 && mat->liquid_specific_heat > 0 && mat->liquid_conductivity > 0 &&
        mat->solid_density > 0 && mat->solid_specific_heat > 0 && mat->solid_conductivity > 0) ||
      (!mat->sharp && !(mat->liquidus_temperature > mat->solidus_temperature)) || !(mat->latent_heat >= 0.0) ||
      mat->capacity_type < 0 || mat->capacity_type > 2)
    return fail(MPDG_ERR_ARG, "material parameters must be positive and the liquidus above the solidus");
  // the solid-phase kernel's bricks may outnumber the flags allocated for the constant-material ones
  int shape[3];
  heat_solid_brick_shape<float>(op->degree, shape);
  long long nb = 1;
  for (int d = 0; d < 3; ++d)
    nb *= (op->m[d] + shape[d] - 1) / shape[d];
  if (nb > op->sync_cap)
    {
      unsigned *fresh = nullptr;
      MPDG_CUDA(cudaStreamSynchronize(op->stream));
      if (cudaMalloc(&fresh, sizeof(unsigned) * (3 + nb)) != cudaSuccess)
        return fail(MPDG_ERR_NOMEM, "brick flags");
      MPDG_CUDA(cudaMemsetAsync(fresh, 0, sizeof(unsigned) * (3 + nb), op->stream));
      MPDG_CUDA(cudaFree(op->d_sync));
      op->d_sync   = fresh;
      op->sync_cap = nb;
      op->epoch    = 0;
    }
  SolidMaterial m;
  m.rho_l      = mat->liquid_density;
  m.cp_l       = mat->liquid_specific_heat;
  m.k_l        = mat->liquid_conductivity;
  m.rho_s      = mat->solid_density;
  m.cp_s       = mat->solid_specific_heat;
  m.k_s        = mat->solid_conductivity;
  m.t_liquidus = mat->liquidus_temperature;
  m.t_solidus  = mat->solidus_temperature;
  m.sharp      = mat->sharp ? 1 : 0;
  m.latent_heat   = mat->latent_heat;
  m.capacity_type = mat->capacity_type;
  op->smat     = m;
  op->solid    = true;
  return MPDG_OK;
}

int
mpdg_op_set_old_temperature(mpdg_op *op, const double *temperature_old)
{
  if (int e = check_op(op))
    return e;
  if (op->kind != MPDG_HEAT)
    return fail(MPDG_ERR_ARG, "the old temperature belongs to the heat operator");
  op->d_temp_old = temperature_old;
  return MPDG_OK;
}

int
mpdg_op_set_reinit(mpdg_op *op, double eps_normal, double eps_tangential, double normal_tolerance, const double *nx,
                   const double *ny, const double *nz)
{
  if (int e = check_op(op))
    return e;
  if (op->kind != MPDG_REINIT)
    return fail(MPDG_ERR_ARG, "mpdg_op_set_reinit applies to the reinitialisation operator");
  if (!(eps_normal >= 0.0) || !(eps_tangential >= 0.0) || !(normal_tolerance > 0.0) || !nx || !ny || !nz)
    return fail(MPDG_ERR_ARG, "diffusion lengths >= 0, a positive tolerance and three normal components");
  op->eps_n       = eps_normal;
  op->eps_t       = eps_tangential;
  op->ntol        = normal_tolerance;
  op->d_normal[0] = nx;
  op->d_normal[1] = ny;
  op->d_normal[2] = nz;
  return MPDG_OK;
}

int
mpdg_level_set_normal_rhs(mpdg_op *op, const double *psi, int normalized, double *nx, double *ny, double *nz)
{
  if (int e = check_op(op))
    return e;
  if (!psi || !nx || !ny || !nz)
    return fail(MPDG_ERR_ARG, "null argument to mpdg_level_set_normal_rhs");
  if (op->degree > 3)
    return fail(MPDG_ERR_UNSUPPORTED, "the level-set right-hand sides support FE_Q degree 1..3");
  // the normal's narrow band masks with the level set psi itself (normal_vector_operator.cpp:184-189)
  MPDG_CUDA(level_set_rhs(op->grid(), op->degree, op->h, 0, normalized ? 1 : 0, 0.0, psi, nullptr, nullptr, nx, ny,
                          nz, op->stream, op->banded() ? psi : nullptr, op->band));
  return MPDG_OK;
}

int
mpdg_level_set_curvature_rhs(mpdg_op *op, const double *nx, const double *ny, const double *nz, double normal_tolerance,
                             double *dst)
{
  if (int e = check_op(op))
    return e;
  if (!nx || !ny || !nz || !dst || !(normal_tolerance > 0.0))
    return fail(MPDG_ERR_ARG, "invalid argument to mpdg_level_set_curvature_rhs");
  if (op->degree > 3)
    return fail(MPDG_ERR_UNSUPPORTED, "the level-set right-hand sides support FE_Q degree 1..3");
  MPDG_CUDA(vec_fill<double>(dst, 0.0, op->ndofs, op->stream));
  MPDG_CUDA(level_set_rhs(op->grid(), op->degree, op->h, 1, 0, normal_tolerance, nx, ny, nz, dst, nullptr, nullptr,
                          op->stream, op->banded() ? op->d_band_ls : nullptr, op->band));
  return MPDG_OK;
}

int
mpdg_op_set_velocity_field(mpdg_op *op, const double *vx, const double *vy, const double *vz)
{
  if (int e = check_op(op))
    return e;
  if (op->kind != MPDG_ADVDIFF && op->kind != MPDG_HEAT)
    return fail(MPDG_ERR_ARG, "a velocity field belongs to the advection-diffusion or the heat operator");
  if ((vx || vy || vz) && !(vx && vy && vz))
    return fail(MPDG_ERR_ARG, "a velocity field needs all three components");
  if (vx && op->kind == MPDG_HEAT && (op->d_k64 || op->solid || op->banded()))
    return fail(MPDG_ERR_UNSUPPORTED, "the heat operator's convection velocity takes a constant conductivity and "
                                      "material and no narrow band");
  if (vx && op->degree > 3)
    return fail(MPDG_ERR_UNSUPPORTED, "a DoF-vector velocity is supported for FE_Q degree 1..3");
  op->d_vfield[0] = vx;
  op->d_vfield[1] = vy;
  op->d_vfield[2] = vz;
  return MPDG_OK;
}

int
mpdg_op_set_wetting(mpdg_op *op, uint32_t faces)
{
  if (int e = check_op(op))
    return e;
  if (op->kind != MPDG_REINIT)
    return fail(MPDG_ERR_ARG, "wetting boundary faces belong to the reinitialisation operator");
  if (faces & ~63u)
    return fail(MPDG_ERR_ARG, "wetting faces: a 6-bit mask of box faces");
  op->wetting = faces;
  return MPDG_OK;
}

int
mpdg_op_set_narrow_band(mpdg_op *op, const double *level_set, double threshold)
{
  if (int e = check_op(op))
    return e;
  if (op->kind != MPDG_HEAT)
    return fail(MPDG_ERR_ARG, "the narrow band belongs to the projection (heat-form) operators");
  if (!level_set || !(threshold > 0.0))
    {
      op->d_band_ls = nullptr;
      op->band      = 0.0;
      return MPDG_OK;
    }
  if (op->degree > 3)
    return fail(MPDG_ERR_UNSUPPORTED, "the narrow band supports FE_Q degree 1..3");
  if (op->d_k64 || op->d_mask || op->solid || op->d_vfield[0] || heat_faces_active(op->fbc, 0) ||
      heat_faces_active(op->fbc, 1))
    return fail(MPDG_ERR_UNSUPPORTED, "the narrow band takes a constant damping, Dirichlet faces only and no "
                                      "boundary-face terms, convection velocity or temperature-dependent material");
  op->d_band_ls = level_set;
  op->band      = threshold;
  return MPDG_OK;
}

int
mpdg_op_set_supg(mpdg_op *op, int enabled, double coefficient)
{
  if (int e = check_op(op))
    return e;
  if (op->kind != MPDG_ADVDIFF)
    return fail(MPDG_ERR_ARG, "SUPG stabilisation applies to the advection-diffusion operator");
  op->supg      = enabled ? 1 : 0;
  op->supg_coef = coefficient;
  return MPDG_OK;
}

int
mpdg_op_set_inflow_outflow(mpdg_op *op, uint32_t faces, const double *values)
{
  if (int e = check_op(op))
    return e;
  if (op->kind != MPDG_ADVDIFF)
    return fail(MPDG_ERR_ARG, "inflow/outflow conditions belong to the advection-diffusion operator");
  if (faces & ~63u)
    return fail(MPDG_ERR_ARG, "inflow/outflow faces: a 6-bit mask of box faces");
  if (faces && !values)
    return fail(MPDG_ERR_ARG, "inflow/outflow conditions need their values on the lattice");
  cudaFree(op->d_mask_io);
  cudaFree(op->d_in_idx);
  cudaFree(op->d_in_val);
  op->d_mask_io = nullptr;
  op->d_in_idx  = nullptr;
  op->d_in_val  = nullptr;
  op->n_inflow  = 0;
  if (!faces)
    return MPDG_OK;
  // support points of the marked faces where the outward normal n and the (affine) velocity v
  // satisfy n . v <= 0 (advection_diffusion_operation.cpp:369-499), Dirichlet DoFs excluded; the
  // coordinates are origin + h (c + node_i), the last point origin + length
  const int       K = op->degree, n[3] = {K * op->m[0] + 1, K * op->m[1] + 1, K * op->m[2] + 1};
  const Tables1D &t = tables(K);
  std::vector<double> xs[3];
  for (int d = 0; d < 3; ++d)
    {
      xs[d].resize(n[d]);
      for (int I = 0; I < n[d]; ++I)
        {
          const int c = std::min(I / K, op->m[d] - 1), i = I - K * c;
          xs[d][I] = I == n[d] - 1 ? op->origin[d] + op->length[d] : op->origin[d] + op->h[d] * (c + t.nodes[i]);
        }
    }
  std::vector<uint8_t> dmask;
  if (op->d_mask)
    {
      dmask.resize(op->ndofs);
      if (int e = stream_copy(op, dmask.data(), op->d_mask, op->ndofs, cudaMemcpyDeviceToHost))
        return e;
    }
  // a DoF-vector velocity is evaluated at the support points: its nodal values there
  std::vector<double> vf[3];
  if (op->d_vfield[0])
    for (int d = 0; d < 3; ++d)
      {
        vf[d].resize(op->ndofs);
        if (int e = stream_copy(op, vf[d].data(), op->d_vfield[d], sizeof(double) * op->ndofs, cudaMemcpyDeviceToHost))
          return e;
      }
  std::vector<uint8_t>   flag(op->ndofs, 0);
  std::vector<long long> idx;
  for (int L = 0; L < n[2]; ++L)
    for (int J = 0; J < n[1]; ++J)
      for (int I = 0; I < n[0]; ++I)
        {
          const int  lat[3] = {I, J, L};
          const long long q = I + (long long)n[0] * (J + (long long)n[1] * L);
          bool       in     = false;
          for (int f = 0; f < 6 && !in; ++f)
            {
              const int d = f / 2, side = f % 2;
              if (!((faces >> f) & 1u) || lat[d] != (side ? n[d] - 1 : 0))
                continue;
              const double x = xs[0][I], y = xs[1][J], z = xs[2][L];
              const double v = vf[0].empty() ? op->vel[d] + op->vel[3 + 3 * d] * x + op->vel[4 + 3 * d] * y +
                                                 op->vel[5 + 3 * d] * z
                                             : vf[d][q];
              in             = (side ? v : -v) <= 0.0;
            }
          bool con = false;
          for (int f = 0; f < 6; ++f)
            if (((op->faces >> f) & 1u) && lat[f / 2] == (f % 2 ? n[f / 2] - 1 : 0))
              con = true;
          if (!dmask.empty() && dmask[q])
            con = true;
          if (in && !con)
            {
              flag[q] = 1;
              idx.push_back(q);
            }
          if (con || in)
            flag[q] = 1; // the apply's mask: Dirichlet and inflow DoFs
        }
  op->n_inflow = (long long)idx.size();
  if (cudaMalloc(&op->d_mask_io, op->ndofs) != cudaSuccess ||
      cudaMalloc(&op->d_in_idx, sizeof(long long) * std::max<size_t>(1, idx.size())) != cudaSuccess ||
      cudaMalloc(&op->d_in_val, sizeof(double) * std::max<size_t>(1, idx.size())) != cudaSuccess)
    return fail(MPDG_ERR_NOMEM, "inflow/outflow constraint storage");
  if (int e = stream_copy(op, op->d_mask_io, flag.data(), op->ndofs, cudaMemcpyHostToDevice))
    return e;
  if (!idx.empty())
    {
      if (int e = stream_copy(op, op->d_in_idx, idx.data(), sizeof(long long) * idx.size(), cudaMemcpyHostToDevice))
        return e;
      MPDG_CUDA(idx_gather(op->d_in_val, values, op->d_in_idx, op->n_inflow, op->stream));
      MPDG_CUDA(cudaStreamSynchronize(op->stream));
    }
  return MPDG_OK;
}

int64_t
mpdg_op_n_inflow(const mpdg_op *op)
{
  return op ? op->n_inflow : -1;
}

int
mpdg_op_set_inflow_outflow_pre_post(mpdg_op *op, int enabled)
{
  if (int e = check_op(op))
    return e;
  op->inflow_prepost = enabled != 0;
  return MPDG_OK;
}

int
mpdg_op_distribute_inflow(mpdg_op *op, double *x)
{
  if (int e = check_op(op))
    return e;
  if (!x)
    return fail(MPDG_ERR_ARG, "null vector passed to mpdg_op_distribute_inflow");
  MPDG_CUDA(idx_set<double>(x, op->d_in_idx, op->d_in_val, op->n_inflow, 0.0, op->stream));
  return MPDG_OK;
}

int
mpdg_op_set_temperature(mpdg_op *op, const double *temperature)
{
  if (int e = check_op(op))
    return e;
  if (op->kind != MPDG_HEAT)
    return fail(MPDG_ERR_ARG, "the linearisation temperature belongs to the heat operator");
  op->d_temp = temperature;
  return MPDG_OK;
}

int
mpdg_op_vmult(mpdg_op *op, double *dst, const double *src)
{
  if (int e = check_op(op))
    return e;
  if (!dst || !src || dst == src)
    return fail(MPDG_ERR_ARG, "vmult needs distinct non-null dst and src");
  return apply<double>(op, (int)OutMode::Set, 1.0, dst, src, nullptr, 1);
}

int
mpdg_op_vmult_f32(mpdg_op *op, float *dst, const float *src)
{
  if (int e = check_op(op))
    return e;
  if (!dst || !src || dst == src)
    return fail(MPDG_ERR_ARG, "vmult needs distinct non-null dst and src");
  return apply<float>(op, (int)OutMode::Set, 1.0, dst, src, nullptr, 1);
}

int
mpdg_op_vmult_add(mpdg_op *op, double *dst, const double *src, double scale)
{
  if (int e = check_op(op))
    return e;
  if (!dst || !src || dst == src)
    return fail(MPDG_ERR_ARG, "vmult_add needs distinct non-null dst and src");
  return apply<double>(op, (int)OutMode::Add, scale, dst, src, nullptr, 1);
}

int
mpdg_op_residual(mpdg_op *op, double *r, const double *b, const double *x)
{
  if (int e = check_op(op))
    return e;
  if (!r || !b || !x || r == x)
    return fail(MPDG_ERR_ARG, "residual needs non-null r, b, x with r != x");
  return apply<double>(op, (int)OutMode::BPlus, -1.0, r, x, b, 1);
}

#ifndef MPDG_HOST_SLABS
#define MPDG_HOST_SLABS 8
#endif

namespace
{
  // Host-buffer apply of a heat operator, pipelined over z-slabs of cells: slab s (cells
  // [c_s, c_s+1)) is applied as a mesh of its own as soon as its input planes [K c_s, K c_s+1] are on
  // the device; its low boundary plane accumulates onto the previous slab's values (acc_lo_z), and
  // the output planes [K c_s, K c_s+1) are final once slab s is done, so their device-to-host copy
  // overlaps the host-to-device copies of the later slabs (both PCIe directions at once).
  int
  vmult_host_slabs(mpdg_op *op, double *dst_host, const double *src_host, double *ds, double *dd)
  {
    constexpr int S = MPDG_HOST_SLABS;
    if (!op->s_h2d)
      {
        MPDG_CUDA(cudaStreamCreateWithFlags(&op->s_h2d, cudaStreamNonBlocking));
        MPDG_CUDA(cudaStreamCreateWithFlags(&op->s_d2h, cudaStreamNonBlocking));
      }
    while ((int)op->ev.size() < 2 * S + 1)
      {
        cudaEvent_t e;
        MPDG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        op->ev.push_back(e);
      }
    const int    K = op->degree, m2 = op->m[2];
    const size_t plane = (size_t)(K * op->m[0] + 1) * (size_t)(K * op->m[1] + 1);
    int          c[S + 1];
    for (int s = 0; s <= S; ++s)
      c[s] = (int)((long long)m2 * s / S);
    // the copies start after the work already on the operator's stream
    MPDG_CUDA(cudaEventRecord(op->ev[2 * S], op->stream));
    MPDG_CUDA(cudaStreamWaitEvent(op->s_h2d, op->ev[2 * S], 0));
    for (int s = 0; s < S; ++s)
      {
        const size_t p0 = (size_t)K * c[s], p1 = (size_t)K * c[s + 1]; // input planes [p0, p1]
        const size_t q0 = s == 0 ? 0 : (size_t)K * c[s] + 1;            // not copied before
        MPDG_CUDA(cudaMemcpyAsync(ds + q0 * plane, src_host + q0 * plane, sizeof(double) * (p1 + 1 - q0) * plane,
                                  cudaMemcpyHostToDevice, op->s_h2d));
        MPDG_CUDA(cudaEventRecord(op->ev[s], op->s_h2d));
        MPDG_CUDA(cudaStreamWaitEvent(op->stream, op->ev[s], 0));
        // slab s as a lattice of its own
        HeatLaunch<double> h;
        h.degree   = K;
        h.mode     = (int)OutMode::Set;
        h.scale    = 1.0;
        h.geo      = heat_geom(op, op->rho_cp / op->dt);
        h.grid     = op->grid();
        h.grid.m[2] = c[s + 1] - c[s];
        h.grid.n[2] = K * h.grid.m[2] + 1;
        h.grid.nbr[2] = (h.grid.m[2] + op->brick[2] - 1) / op->brick[2];
        if (s > 0)
          h.grid.faces &= ~16u; // the slab's low plane is not the domain's
        if (s + 1 < S)
          h.grid.faces &= ~32u;
        h.grid.acc_lo_z = s > 0 ? 1u : 0u;
        h.sync     = op->sync();
        h.kconst   = op->k;
        h.kcell    = op->d_k64 ? op->d_k64 + (size_t)c[s] * op->m[0] * op->m[1] : nullptr;
        h.src      = ds + p0 * plane;
        h.dst      = dd + p0 * plane;
        h.mask_src = 1;
        h.march    = true;
        MPDG_CUDA(heat_apply<double>(h, op->stream));
        MPDG_CUDA(cudaEventRecord(op->ev[S + s], op->stream));
        MPDG_CUDA(cudaStreamWaitEvent(op->s_d2h, op->ev[S + s], 0));
        const size_t o1 = s + 1 < S ? p1 : p1 + 1; // output planes [p0, o1)
        MPDG_CUDA(cudaMemcpyAsync(dst_host + p0 * plane, dd + p0 * plane, sizeof(double) * (o1 - p0) * plane,
                                  cudaMemcpyDeviceToHost, op->s_d2h));
      }
    MPDG_CUDA(cudaStreamSynchronize(op->s_d2h));
    MPDG_CUDA(cudaStreamSynchronize(op->stream));
    return MPDG_OK;
  }
} // namespace

int
mpdg_op_vmult_host(mpdg_op *op, double *dst_host, const double *src_host)
{
  if (int e = check_op(op))
    return e;
  if (!dst_host || !src_host)
    return fail(MPDG_ERR_ARG, "null host buffer");
  double *ds = op->vec<double>("host_src"), *dd = op->vec<double>("host_dst");
  if (!ds || !dd)
    return fail(MPDG_ERR_NOMEM, "staging vectors");
  const size_t bytes = sizeof(double) * op->ndofs;
  if (op->kind == MPDG_HEAT && op->d_mask == nullptr && !op->tangent_faces() && !op->solid && op->m[2] >= 16 &&
      op->ndofs >= (1 << 22))
    return vmult_host_slabs(op, dst_host, src_host, ds, dd);
  MPDG_CUDA(cudaMemcpyAsync(ds, src_host, bytes, cudaMemcpyHostToDevice, op->stream));
  if (int e = apply<double>(op, (int)OutMode::Set, 1.0, dd, ds, nullptr, 1))
    return e;
  MPDG_CUDA(cudaMemcpyAsync(dst_host, dd, bytes, cudaMemcpyDeviceToHost, op->stream));
  MPDG_CUDA(cudaStreamSynchronize(op->stream));
  return MPDG_OK;
}

int
mpdg_op_compute_inverse_diagonal(mpdg_op *op, double *diag)
{
  if (int e = check_op(op))
    return e;
  if (!diag)
    return fail(MPDG_ERR_ARG, "null diagonal");
  return inverse_diagonal<double>(op, diag);
}

int
mpdg_op_compute_inverse_diagonal_f32(mpdg_op *op, float *diag)
{
  if (int e = check_op(op))
    return e;
  if (!diag)
    return fail(MPDG_ERR_ARG, "null diagonal");
  return inverse_diagonal<float>(op, diag);
}

int
mpdg_op_create_rhs(mpdg_op *op, double *dst, const double *a, const double *b, const double *c)
{
  if (int e = check_op(op))
    return e;
  if (!(op->dt > 0.0))
    return fail(MPDG_ERR_ZERO_DT, "time increment must be positive (ExcZeroTimeIncrement)");
  if (!dst || !a)
    return fail(MPDG_ERR_ARG, "create_rhs needs dst and its first input");
  if (op->kind == MPDG_REINIT)
    {
      // olsson_CG_operator.cpp:197-260: dst is overwritten, constrained rows end at 0
      if (!op->d_normal[0] || !op->d_normal[1] || !op->d_normal[2])
        return fail(MPDG_ERR_ARG, "the reinitialisation operator needs its normal field (mpdg_op_set_reinit)");
      MPDG_CUDA(vec_fill<double>(dst, 0.0, op->ndofs, op->stream));
      MPDG_CUDA(reinit_integrate<double>(reinit_launch<double>(op, 1.0, a, dst, 0), 1, op->stream));
      return MPDG_OK;
    }
  if (op->kind == MPDG_HEAT && op->solid)
    {
      // dst += M q - int rho c_p(T) (T - T_old) / dt phi - int k(T) grad T . grad phi (+ faces)
      if (!b)
        return fail(MPDG_ERR_ARG, "create_rhs with temperature-dependent material needs T_old");
      if (c)
        if (int e = apply<double>(op, (int)OutMode::Add, 1.0, dst, c, nullptr, 0, 1))
          return e;
      if (int e = solid_apply<double>(op, (int)OutMode::Add, 1.0, dst, nullptr, nullptr, 0, nullptr, true, a, b))
        return e;
      if (heat_faces_active(op->fbc, 1))
        {
          HeatFaceLaunch<double> f;
          f.degree = op->degree;
          f.mode   = 1;
          for (int d = 0; d < 3; ++d)
            f.hlen[d] = op->h[d];
          f.grid = op->grid();
          f.bc   = op->fbc;
          f.temp = a;
          f.dst  = dst;
          MPDG_CUDA(heat_faces<double>(f, op->stream));
        }
      return MPDG_OK;
    }
  if (op->kind == MPDG_HEAT)
    {
      // v = (rho c_p/dt)(T_old - T) + q ; dst += M v - K_k T   (plain reads, free rows)
      double *v = op->vec<double>("rhs_tmp");
      if (!v)
        return fail(MPDG_ERR_NOMEM, "rhs work vector");
      const double s = op->rho_cp / op->dt;
      MPDG_CUDA(vec_axpby<double>(v, -s, a, b ? s : 0.0, b, op->ndofs, op->stream));
      if (c)
        MPDG_CUDA(vec_axpby<double>(v, 1.0, v, 1.0, c, op->ndofs, op->stream));
      if (int e = apply<double>(op, (int)OutMode::Add, 1.0, dst, v, nullptr, 0, 1))
        return e;
      if (int e = apply<double>(op, (int)OutMode::Add, -1.0, dst, a, nullptr, 0, 2))
        return e;
      if (op->d_vfield[0])
        {
          // dst -= int rho c_p (v . grad T) phi (heat_diffuse_operator.cpp:499-500), plain reads
          AdvLaunch<double> h;
          h.degree   = op->degree;
          h.mode     = (int)OutMode::Add;
          h.scale    = 1.0;
          h.p        = heat_velocity_params(op, true);
          h.grid     = heat_velocity_grid<double>(op);
          h.sync     = op->sync();
          h.src      = a;
          h.dst      = dst;
          h.b        = nullptr;
          h.mask_src = 0;
          h.skip     = nullptr;
          MPDG_CUDA(adv_apply<double>(h, op->stream));
        }
      if (heat_faces_active(op->fbc, 1))
        {
          HeatFaceLaunch<double> f;
          f.degree = op->degree;
          f.mode   = 1;
          for (int d = 0; d < 3; ++d)
            f.hlen[d] = op->h[d];
          f.grid = op->grid();
          f.bc   = op->fbc;
          f.temp = a;
          f.dst  = dst;
          MPDG_CUDA(heat_faces<double>(f, op->stream));
        }
      return MPDG_OK;
    }
  return apply<double>(op, (int)OutMode::Add, 1.0, dst, a, nullptr, 0, 3);
}

int
mpdg_solve(mpdg_op *op, double *x, const double *b, const mpdg_solver_params *params, mpdg_solve_info *info)
{
  if (int e = check_op(op))
    return e;
  return solve_typed<double>(op, x, b, params, info, "s64_");
}

int
mpdg_solve_f32(mpdg_op *op, float *x, const float *b, const mpdg_solver_params *params, mpdg_solve_info *info)
{
  if (int e = check_op(op))
    return e;
  return solve_typed<float>(op, x, b, params, info, "s32_");
}

int
mpdg_solve_mixed(mpdg_op *op, double *x, const double *b, const mpdg_mixed_params *prm, mpdg_solve_info *info)
{
  if (int e = check_op(op))
    return e;
  if (!x || !b || !prm)
    return fail(MPDG_ERR_ARG, "null argument to mpdg_solve_mixed");
  const long long n   = op->ndofs;
  double         *r64 = op->vec<double>("mx_r64");
  float          *r32 = op->vec<float>("mx_r32"), *e32 = op->vec<float>("mx_e32"), *invd32 = op->vec<float>("mx_invd32");
  double         *invd64 = op->vec<double>("mx_invd64");
  if (!r64 || !r32 || !e32 || !invd32 || !invd64)
    return fail(MPDG_ERR_NOMEM, "mixed-precision work vectors");
  // Jacobi diagonal computed in FP64 and rounded once
  if (int e = inverse_diagonal<double>(op, invd64))
    return e;
  MPDG_CUDA(vec_convert<float, double>(invd32, invd64, n, op->stream));
  const double *bb = b;
  MPDG_CUDA(vec_multidot<double>(&bb, &bb, 1, n, op->d_scal, op->reducer(), op->stream));
  // a zero initial guess (max |x| == 0) makes the first outer residual b itself
  MPDG_CUDA(vec_absmax<double>(x, n, op->d_scal + 1, op->reducer(), op->stream));
  if (int e = stream_copy(op, op->h_scal, op->d_scal, 2 * sizeof(double), cudaMemcpyDeviceToHost))
    return e;
  const double bnorm  = std::sqrt(op->h_scal[0]);
  const bool   x_zero = op->h_scal[1] == 0.0;
  const double tol   = prm->outer_rel_tol * bnorm;
  int          inner_total = 0, outer = 0, status = MPDG_ERR_NOT_CONVERGED;
  double       res = 0.0, res0 = -1.0;
  std::vector<double> hist;
  for (outer = 0; outer <= prm->max_outer; ++outer)
    {
      const bool    from_b = outer == 0 && x_zero;
      const double *r_cur  = from_b ? b : r64;
      if (from_b)
        res = bnorm;
      else
        {
          if (int e = apply<double>(op, (int)OutMode::BPlus, -1.0, r64, x, b, 1))
            return e;
          const double *rr = r64;
          MPDG_CUDA(vec_multidot<double>(&rr, &rr, 1, n, op->d_scal, op->reducer(), op->stream));
          MPDG_CUDA(cudaMemcpyAsync(op->h_scal, op->d_scal, sizeof(double), cudaMemcpyDeviceToHost, op->stream));
          MPDG_CUDA(cudaStreamSynchronize(op->stream));
          res = std::sqrt(op->h_scal[0]);
        }
      if (res0 < 0)
        res0 = res;
      hist.push_back(res);
      if (res <= tol)
        {
          status = MPDG_OK;
          break;
        }
      if (outer == prm->max_outer)
        break;
      MPDG_CUDA(vec_convert<float, double>(r32, r_cur, n, op->stream));
      MPDG_CUDA(vec_fill<float>(e32, 0.0f, n, op->stream));
      mpdg_solve_info in{};
      int             rc;
      // the correction of a residual already close to the outer tolerance needs only the reduction
      // that reaches it (with a factor 2 to spare), never more than inner_rel_tol asks for
      const double inner_tol =
        prm->inexact_last ? std::min(0.5, std::max(prm->inner_rel_tol, 0.5 * tol / res)) : prm->inner_rel_tol;
      if (prm->solver == MPDG_GMRES)
        rc = gmres_solve<float>(op, e32, r32, invd32, prm->max_inner, 0.0, inner_tol,
                                prm->restart > 0 ? prm->restart : 30, &in, "mi32_");
      else
        rc = cg_solve<float>(op, e32, r32, invd32, prm->max_inner, 0.0, inner_tol, &in, "mi32_", true, r32);
      if (rc != MPDG_OK && rc != MPDG_ERR_NOT_CONVERGED)
        return rc;
      inner_total += in.iterations;
      MPDG_CUDA(vec_add_f32_to_f64(x, e32, n, op->stream));
    }
  if (info)
    {
      info->iterations       = outer;
      info->inner_iterations = inner_total;
      info->status           = status;
      info->initial_residual = res0;
      info->final_residual   = res;
      if (info->history && info->history_capacity > 0)
        {
          const int cnt = std::min<int>(info->history_capacity, (int)hist.size());
          std::memcpy(info->history, hist.data(), sizeof(double) * cnt);
        }
    }
  if (status != MPDG_OK)
    return fail(MPDG_ERR_NOT_CONVERGED, "mixed-precision defect correction did not converge");
  return MPDG_OK;
}

namespace
{
  // Forward sweep of the transient heat problem; states n = first+1..last are written to out[]
  // (out may be null), the last state to Tlast.  J accumulated when target != null.
  int
  heat_forward_range(mpdg_op *op, const double *invd, const double *qhat, double amplitude, const double *T_first,
                     int first, int last, const double *target, double *J, double **out, double *Tlast,
                     const mpdg_adjoint_params *prm, long long *iters, int *solves)
  {
    const long long n   = op->ndofs;
    double         *v   = op->vec<double>("adj_v"), *rhs = op->vec<double>("adj_rhs");
    double         *Ta  = op->vec<double>("adj_Ta"), *Tb = op->vec<double>("adj_Tb");
    if (!v || !rhs || !Ta || !Tb)
      return fail(MPDG_ERR_NOMEM, "adjoint work vectors");
    MPDG_CUDA(cudaMemcpyAsync(Ta, T_first, sizeof(double) * n, cudaMemcpyDeviceToDevice, op->stream));
    for (int step = first + 1; step <= last; ++step)
      {
        // rhs = M (rho c_p T_{n-1} / dt + A qhat_n), plain reads, constrained rows 0
        MPDG_CUDA(vec_axpby<double>(v, op->rho_cp / op->dt, Ta, amplitude, qhat + (size_t)(step - 1) * n, n, op->stream));
        if (int e = apply<double>(op, (int)OutMode::Set, 1.0, rhs, v, nullptr, 0, 1))
          return e;
        MPDG_CUDA(cudaMemcpyAsync(Tb, Ta, sizeof(double) * n, cudaMemcpyDeviceToDevice, op->stream));
        mpdg_solve_info in{};
        if (int e = cg_solve<double>(op, Tb, rhs, invd, prm->cg_max_it > 0 ? prm->cg_max_it : 10000, 0.0,
                                     prm->cg_rel_tol, &in, "adjcg_"))
          return e;
        *iters += in.iterations;
        ++*solves;
        if (target)
          {
            MPDG_CUDA(vec_axpby<double>(v, 1.0, Tb, -1.0, target + (size_t)(step - 1) * n, n, op->stream));
            MPDG_CUDA(vec_set_constrained<double>(v, 0.0, op->grid(), op->stream));
            const double *vv = v;
            MPDG_CUDA(vec_multidot<double>(&vv, &vv, 1, n, op->d_scal, op->reducer(), op->stream));
            MPDG_CUDA(cudaMemcpyAsync(op->h_scal, op->d_scal, sizeof(double), cudaMemcpyDeviceToHost, op->stream));
            MPDG_CUDA(cudaStreamSynchronize(op->stream));
            *J += 0.5 * op->h_scal[0];
          }
        if (out && out[step - first - 1])
          MPDG_CUDA(cudaMemcpyAsync(out[step - first - 1], Tb, sizeof(double) * n, cudaMemcpyDeviceToDevice, op->stream));
        std::swap(Ta, Tb);
      }
    if (Tlast)
      MPDG_CUDA(cudaMemcpyAsync(Tlast, Ta, sizeof(double) * n, cudaMemcpyDeviceToDevice, op->stream));
    return MPDG_OK;
  }

  int
  adjoint_setup(mpdg_op *op, const double *log_k, double **invd)
  {
    if (op->kind != MPDG_HEAT)
      return fail(MPDG_ERR_ARG, "the adjoint needs a heat operator");
    if (op->degree > 2)
      return fail(MPDG_ERR_UNSUPPORTED, "the adjoint supports FE_Q degree 1..2");
    double *k = op->vec<double>("adj_k", (size_t)op->ncells);
    *invd     = op->vec<double>("adj_invd");
    if (!k || !*invd)
      return fail(MPDG_ERR_NOMEM, "adjoint coefficient vectors");
    MPDG_CUDA(vec_exp(k, log_k, op->ncells, op->stream));
    if (int e = mpdg_op_set_conductivity(op, k))
      return e;
    return inverse_diagonal<double>(op, *invd);
  }
} // namespace

int
mpdg_heat_forward(mpdg_op *op, const double *log_k, const double *qhat, double amplitude,
                  const mpdg_adjoint_params *prm, double *T_out)
{
  if (int e = check_op(op))
    return e;
  if (!log_k || !qhat || !prm || !T_out || prm->n_steps < 1)
    return fail(MPDG_ERR_ARG, "invalid argument to mpdg_heat_forward");
  double *invd = nullptr;
  if (int e = adjoint_setup(op, log_k, &invd))
    return e;
  const long long      n = op->ndofs;
  std::vector<double *> out(prm->n_steps);
  for (int i = 0; i < prm->n_steps; ++i)
    out[i] = T_out + (size_t)i * n;
  double *zero = op->vec<double>("adj_zero");
  if (!zero)
    return fail(MPDG_ERR_NOMEM, "adjoint work vector");
  MPDG_CUDA(vec_fill<double>(zero, 0.0, n, op->stream));
  long long it = 0;
  int       solves = 0;
  double    J      = 0.0;
  if (int e = heat_forward_range(op, invd, qhat, amplitude, zero, 0, prm->n_steps, nullptr, &J, out.data(), nullptr,
                                 prm, &it, &solves))
    return e;
  MPDG_CUDA(cudaStreamSynchronize(op->stream));
  return MPDG_OK;
}

int
mpdg_adjoint_heat(mpdg_op *op, const double *log_k, const double *qhat, double amplitude, const double *T_target,
                  const mpdg_adjoint_params *prm, double *grad, mpdg_adjoint_result *res)
{
  if (int e = check_op(op))
    return e;
  if (!log_k || !qhat || !T_target || !prm || prm->n_steps < 1)
    return fail(MPDG_ERR_ARG, "invalid argument to mpdg_adjoint_heat");
  if (heat_faces_active(op->fbc, 1) || op->solid)
    return fail(MPDG_ERR_UNSUPPORTED, "the adjoint covers operators without boundary-face terms or "
                                      "temperature-dependent material");
  double *invd = nullptr;
  if (int e = adjoint_setup(op, log_k, &invd))
    return e;
  const long long n  = op->ndofs;
  const int       S  = prm->n_steps;
  const int       ce = std::max(1, std::min(prm->checkpoint_every > 0 ? prm->checkpoint_every : 5, S));
  const int       ncp = (S + ce - 1) / ce; // checkpoints T_0, T_ce, ... (segment starts)
  std::vector<double *> cp(ncp), seg(ce);
  for (int i = 0; i < ncp; ++i)
    if (!(cp[i] = op->vec<double>("adj_cp" + std::to_string(i))))
      return fail(MPDG_ERR_NOMEM, "checkpoint storage");
  for (int i = 0; i < ce; ++i)
    if (!(seg[i] = op->vec<double>("adj_seg" + std::to_string(i))))
      return fail(MPDG_ERR_NOMEM, "segment storage");
  double *lam = op->vec<double>("adj_lam"), *lamn = op->vec<double>("adj_lamn"), *rhs = op->vec<double>("adj_arhs"),
         *v = op->vec<double>("adj_av"), *Mq = op->vec<double>("adj_Mq");
  if (!lam || !lamn || !rhs || !v || !Mq)
    return fail(MPDG_ERR_NOMEM, "adjoint vectors");
  long long it = 0;
  int       fsolves = 0, asolves = 0;
  double    J       = 0.0;
  // forward pass: J and the checkpoints T_{s ce}
  MPDG_CUDA(vec_fill<double>(cp[0], 0.0, n, op->stream));
  for (int s = 0; s < ncp; ++s)
    {
      const int a = s * ce, b = std::min(S, a + ce);
      if (int e = heat_forward_range(op, invd, qhat, amplitude, cp[s], a, b, T_target, &J, nullptr,
                                     s + 1 < ncp ? cp[s + 1] : nullptr, prm, &it, &fsolves))
        return e;
    }
  double gA = 0.0;
  if (grad)
    {
      MPDG_CUDA(vec_fill<double>(grad, 0.0, op->ncells, op->stream));
      MPDG_CUDA(vec_fill<double>(lamn, 0.0, n, op->stream));
      const HeatGeom geo = heat_geom(op, 0.0);
      for (int s = ncp - 1; s >= 0; --s)
        {
          const int a = s * ce, b = std::min(S, a + ce);
          // recompute T_{a+1..b} from the checkpoint T_a
          double dummy = 0.0;
          if (int e = heat_forward_range(op, invd, qhat, amplitude, cp[s], a, b, nullptr, &dummy, seg.data(), nullptr,
                                         prm, &it, &fsolves))
            return e;
          for (int step = b; step > a; --step)
            {
              const double *Tn = seg[step - a - 1];
              // rhs = rho c_p M lam_{n+1} / dt + (T_n - T*_n) on free rows
              if (int e = apply<double>(op, (int)OutMode::Set, op->rho_cp / op->dt, rhs, lamn, nullptr, 1, 1))
                return e;
              MPDG_CUDA(vec_axpby<double>(v, 1.0, Tn, -1.0, T_target + (size_t)(step - 1) * n, n, op->stream));
              MPDG_CUDA(vec_set_constrained<double>(v, 0.0, op->grid(), op->stream));
              MPDG_CUDA(vec_axpby<double>(rhs, 1.0, rhs, 1.0, v, n, op->stream));
              MPDG_CUDA(cudaMemcpyAsync(lam, lamn, sizeof(double) * n, cudaMemcpyDeviceToDevice, op->stream));
              mpdg_solve_info in{};
              if (int e = cg_solve<double>(op, lam, rhs, invd, prm->cg_max_it > 0 ? prm->cg_max_it : 10000, 0.0,
                                           prm->cg_rel_tol, &in, "adjcg_"))
                return e;
              it += in.iterations;
              ++asolves;
              // dJ/dz_c -= k_c lam^T K_c T_n   (fused per-cell reduction)
              MPDG_CUDA(heat_cell_form(op->grid(), op->degree, geo, -1.0, lam, Tn, op->d_k64, op->k, grad, true,
                                       op->stream));
              // dJ/dA += lam^T M qhat_n
              if (int e = apply<double>(op, (int)OutMode::Set, 1.0, Mq, qhat + (size_t)(step - 1) * n, nullptr, 0, 1))
                return e;
              const double *x0 = lam, *y0 = Mq;
              MPDG_CUDA(vec_multidot<double>(&x0, &y0, 1, n, op->d_scal, op->reducer(), op->stream));
              MPDG_CUDA(cudaMemcpyAsync(op->h_scal, op->d_scal, sizeof(double), cudaMemcpyDeviceToHost, op->stream));
              MPDG_CUDA(cudaStreamSynchronize(op->stream));
              gA += op->h_scal[0];
              std::swap(lam, lamn);
            }
        }
    }
  MPDG_CUDA(cudaStreamSynchronize(op->stream));
  if (res)
    {
      res->objective      = J;
      res->grad_amplitude = gA;
      res->forward_solves = fsolves;
      res->adjoint_solves = asolves;
      res->cg_iterations  = it;
    }
  return MPDG_OK;
}

int
mpdg_heat_cell_stiffness_form(mpdg_op *op, const double *lam, const double *T, double *form)
{
  if (int e = check_op(op))
    return e;
  if (!lam || !T || !form || op->kind != MPDG_HEAT)
    return fail(MPDG_ERR_ARG, "invalid argument to mpdg_heat_cell_stiffness_form");
  if (op->degree > 2)
    return fail(MPDG_ERR_UNSUPPORTED, "cell forms support FE_Q degree 1..2");
  MPDG_CUDA(heat_cell_form(op->grid(), op->degree, heat_geom(op, 0.0), 1.0, lam, T, nullptr, 1.0, form, false,
                           op->stream));
  return MPDG_OK;
}

int
mpdg_op_create_rhs_and_apply_dirichlet(mpdg_op *op, double *rhs, const double *a, const double *b, const double *c,
                                       const double *dirichlet_values, int zero_out)
{
  if (int e = check_op(op))
    return e;
  if (!rhs || !a || !dirichlet_values)
    return fail(MPDG_ERR_ARG, "null argument to mpdg_op_create_rhs_and_apply_dirichlet");
  double *bc = op->vec<double>("lift_bc"), *tmp = op->vec<double>("lift_tmp");
  if (!bc || !tmp)
    return fail(MPDG_ERR_NOMEM, "lifting work vectors");
  const GridDesc with_bc = op->grid(); // the constraint set of the operator (dof_idx)
  MPDG_CUDA(vec_copy_constrained<double>(bc, dirichlet_values, with_bc, op->stream));
  // inflow DoFs enter as additional inhomogeneous constraints (advection_diffusion_operation.cpp:
  // 262-270 with utilities_matrixfree.hpp:63-68); the apply below runs without the inflow hooks
  if (op->n_inflow > 0)
    MPDG_CUDA(idx_set<double>(bc, op->d_in_idx, op->d_in_val, op->n_inflow, 0.0, op->stream));
  const bool saved = op->with_bc;
  op->with_bc      = false; // reset_dof_index(dof_no_bc_idx)
  int rc           = apply<double>(op, (int)OutMode::Set, -1.0, tmp, bc, nullptr, 1);
  if (rc == MPDG_OK)
    rc = mpdg_op_create_rhs(op, tmp, a, b, c);
  op->with_bc = saved; // reset_dof_index(dof_idx)
  if (rc != MPDG_OK)
    return rc;
  MPDG_CUDA(vec_axpby<double>(rhs, 1.0, tmp, zero_out ? 0.0 : 1.0, zero_out ? nullptr : rhs, op->ndofs, op->stream));
  if (op->n_inflow > 0)
    MPDG_CUDA(idx_set<double>(rhs, op->d_in_idx, nullptr, op->n_inflow, 0.0, op->stream));
  MPDG_CUDA(vec_set_constrained<double>(rhs, 0.0, with_bc, op->stream));
  return MPDG_OK;
}

int
mpdg_vec_fill(mpdg_op *op, double *x, double value)
{
  if (int e = check_op(op))
    return e;
  if (!x)
    return fail(MPDG_ERR_ARG, "null vector passed to mpdg_vec_fill");
  MPDG_CUDA(vec_fill<double>(x, value, op->ndofs, op->stream));
  return MPDG_OK;
}

int
mpdg_vec_axpby(mpdg_op *op, double *y, double a, const double *x, double b)
{
  if (int e = check_op(op))
    return e;
  if (!y)
    return fail(MPDG_ERR_ARG, "null vector passed to mpdg_vec_axpby");
  MPDG_CUDA(vec_axpby<double>(y, a, x, b, y, op->ndofs, op->stream));
  return MPDG_OK;
}

int
mpdg_vec_norm(mpdg_op *op, const double *x, double *out)
{
  if (int e = check_op(op))
    return e;
  if (!x || !out)
    return fail(MPDG_ERR_ARG, "null argument to mpdg_vec_norm");
  MPDG_CUDA(vec_multidot<double>(&x, &x, 1, op->ndofs, op->d_scal, op->reducer(), op->stream));
  MPDG_CUDA(cudaMemcpyAsync(op->h_scal, op->d_scal, sizeof(double), cudaMemcpyDeviceToHost, op->stream));
  MPDG_CUDA(cudaStreamSynchronize(op->stream));
  *out = std::sqrt(op->h_scal[0]);
  return MPDG_OK;
}

int
mpdg_vec_dot(mpdg_op *op, const double *x, const double *y, double *out)
{
  if (int e = check_op(op))
    return e;
  if (!x || !y || !out)
    return fail(MPDG_ERR_ARG, "null argument to mpdg_vec_dot");
  MPDG_CUDA(vec_multidot<double>(&x, &y, 1, op->ndofs, op->d_scal, op->reducer(), op->stream));
  MPDG_CUDA(cudaMemcpyAsync(op->h_scal, op->d_scal, sizeof(double), cudaMemcpyDeviceToHost, op->stream));
  MPDG_CUDA(cudaStreamSynchronize(op->stream));
  *out = op->h_scal[0];
  return MPDG_OK;
}

int
mpdg_op_distribute_constraints(mpdg_op *op, double *dst, const double *values)
{
  if (int e = check_op(op))
    return e;
  if (!dst || !values)
    return fail(MPDG_ERR_ARG, "null argument to mpdg_op_distribute_constraints");
  MPDG_CUDA(vec_distribute_constrained<double>(dst, values, op->grid(), op->stream));
  return MPDG_OK;
}

int
mpdg_vec_alloc(mpdg_op *op, double **x)
{
  if (int e = check_op(op))
    return e;
  if (!x)
    return fail(MPDG_ERR_ARG, "null argument to mpdg_vec_alloc");
  *x = nullptr;
  if (cudaMalloc(x, sizeof(double) * op->ndofs) != cudaSuccess)
    return fail(MPDG_ERR_NOMEM, "mpdg_vec_alloc");
  MPDG_CUDA(cudaMemsetAsync(*x, 0, sizeof(double) * op->ndofs, op->stream));
  return MPDG_OK;
}

int
mpdg_vec_free(double *x)
{
  if (x && cudaFree(x) != cudaSuccess)
    return fail(MPDG_ERR_CUDA, "cudaFree in mpdg_vec_free");
  return MPDG_OK;
}

int
mpdg_op_test_set_wait_limit(mpdg_op *op, unsigned spins)
{
  if (int e = check_op(op))
    return e;
  op->spin_limit = spins ? spins : SPIN_LIMIT;
  return MPDG_OK;
}

int
mpdg_op_test_set_ticket(mpdg_op *op, unsigned value)
{
  if (int e = check_op(op))
    return e;
  // stream-ordered: the next launch on the handle's stream finds this counter
  MPDG_CUDA(cudaMemcpyAsync(op->d_sync, &value, sizeof(unsigned), cudaMemcpyHostToDevice, op->stream));
  MPDG_CUDA(cudaStreamSynchronize(op->stream));
  return MPDG_OK;
}

int
mpdg_op_set_cg_variant(mpdg_op *op, int fused)
{
  if (int e = check_op(op))
    return e;
  op->fused_cg = fused != 0;
  return MPDG_OK;
}

int
mpdg_op_n_bricks(const mpdg_op *op)
{
  if (!op)
    return -1;
  return op->nbr[0] * op->nbr[1] * op->nbr[2];
}

int
mpdg_op_device_errors(mpdg_op *op)
{
  if (!op)
    return -1;
  int v = 0;
  if (cudaMemcpyAsync(&v, op->d_err, sizeof(int), cudaMemcpyDeviceToHost, op->stream) != cudaSuccess ||
      cudaStreamSynchronize(op->stream) != cudaSuccess)
    return -1;
  cudaMemsetAsync(op->d_err, 0, sizeof(int), op->stream);
  return v;
}

} // extern "C"

namespace mpdg
{
  int
  record_failure(int code, const char *msg)
  {
    return fail(code, msg);
  }
} // namespace mpdg
