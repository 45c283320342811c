// Internal launch interfaces of the CUDA kernels (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "brick.cuh"
#include "tables.h"

namespace mpdg
{
  // Geometry factors of the uniform box mesh (hx, hy, hz per cell).
  struct HeatGeom
  {
    double mass_coef; // multiplies M(x)M(x)M (rho c_p / dt * hx hy hz for the tangent)
    double cx, cy, cz; // hy hz / hx, hx hz / hy, hx hy / hz
  };

  template <typename T>
  struct HeatLaunch
  {
    int         degree   = 2;
    int         mode     = 0;   // OutMode
    double      scale    = 1.0; // dst (+)= scale * A src
    HeatGeom    geo{};
    GridDesc    grid{};
    SyncDesc    sync{};
    double      kconst   = 1.0;
    const T    *kcell    = nullptr;
    const T    *src      = nullptr;
    T          *dst      = nullptr;
    const T    *b        = nullptr;
    int         mask_src = 1;
    const int  *skip     = nullptr; // device flag: return at once when nonzero
    bool        march    = true;    // column-marching / pencil kernels (operator without per-DoF mask)
    DotSink     dot{};              // fused src^T A src -> CG step length (Set mode, heat_apply_fuses_dot)
  };

  // whether the apply kernel chosen for these settings can fuse the CG dot product (DotSink)
  bool heat_apply_fuses_dot(int K, bool has_dof_mask, bool march);

  template <typename T>
  cudaError_t heat_apply(const HeatLaunch<T> &h, cudaStream_t s);

  template <typename T>
  cudaError_t heat_diagonal(const GridDesc &g, int K, const HeatGeom &geo, double kconst, const T *kcell,
                            T *diag, bool invert, double threshold, cudaStream_t s);

  template <typename T>
  void heat_brick_shape(int K, int shape[3], bool march);

  // ---- boundary-face terms of the heat operator (faces.cu); face f: bit 2d low / 2d+1 high of dim d
  struct HeatFaceBC
  {
    unsigned convection_faces = 0, radiation_faces = 0, neumann_faces = 0;
    double   convection_coefficient = 0.0, convection_temperature_infinity = 0.0;
    double   emissivity_sigma = 0.0, radiation_temperature_infinity = 0.0; // eps * Stefan-Boltzmann
    double   neumann_flux[6]{};                                              // g . n per face
  };

  template <typename T>
  struct HeatFaceLaunch
  {
    int           degree = 2;
    int           mode   = 0; // 0 tangent (dst += scale F src), 1 rhs (dst += face rhs of temp), 2 diagonal
    double        scale  = 1.0;
    double        hlen[3]{};
    GridDesc      grid{};
    HeatFaceBC    bc{};
    const double *temp = nullptr; // linearisation point / temperature of the rhs
    const T      *src  = nullptr;
    T            *dst  = nullptr;
    double       *diag = nullptr;
    const int    *skip = nullptr;
  };

  // ---- temperature-dependent material (solid / liquid phases, heat_solid.cu), FE_Q(1, 2)
  struct SolidMaterial
  {
    double rho_l = 1.0, cp_l = 1.0, k_l = 1.0; // liquid
    double rho_s = 1.0, cp_s = 1.0, k_s = 1.0; // solid
    double t_liquidus = 1.0, t_solidus = 0.0;
    int    sharp = 0;                          // 0 mushy zone, 1 sharp transition at t_solidus
    double latent_heat   = 0.0;                // > 0: apparent capacity over the mushy zone
    int    capacity_type = 0;                  // 0 quadratic-linear-quadratic, 1 quartic bell, 2 constant
  };

  template <typename T>
  struct HeatSolidLaunch
  {
    int           degree = 2;
    int           mode   = 0;     // OutMode of the tangent apply
    int           rhs    = 0;     // 1: dst += residual part of create_rhs (Add), src unused
    double        scale  = 1.0;   // tangent: dst (+)= scale * A src
    double        dt     = 1.0;
    double        hlen[3]{};
    SolidMaterial mat{};
    GridDesc      grid{};         // nbr from heat_solid_brick_shape
    SyncDesc      sync{};
    const T      *src      = nullptr;
    const T      *temp     = nullptr; // linearisation temperature (plain reads)
    const T      *temp_old = nullptr;
    T            *dst      = nullptr;
    const T      *b        = nullptr;
    int           mask_src = 1;
    const int    *skip     = nullptr;
  };

  template <typename T>
  void heat_solid_brick_shape(int K, int shape[3]);
  template <typename T>
  cudaError_t heat_solid_apply(const HeatSolidLaunch<T> &h, cudaStream_t s);
  // adds the tangent's diagonal on the free rows of diag (FP64)
  cudaError_t heat_solid_diagonal(const GridDesc &g, int K, const SolidMaterial &mat, double dt, const double hlen[3],
                                  const double *temp, const double *temp_old, double *diag, cudaStream_t s);

  // ---- conservative level-set reinitialisation (Olsson, reinit.cu), FE_Q(1, 2)
  template <typename T>
  struct ReinitLaunch
  {
    int           degree = 1;
    double        scale = 1.0, dt = 1.0, eps_normal = 0.0, eps_tangential = 0.0, normal_tolerance = 1e-16;
    double        hlen[3]{};
    GridDesc      grid{};
    const T      *src = nullptr;
    const double *normal[3]{};
    T            *dst  = nullptr;
    double       *diag = nullptr;
    int           mask_src = 1;
    const double *band_ls = nullptr; // narrow band: integrands masked where |level set| >= band
    double        band    = 0.0;
    unsigned      wetting = 0;       // wetting boundary faces (reinitialisation operator)
    bool          faces_only = false;
  };
  // mode 0: dst += scale * A src on free rows; 1: dst += the rhs integrand of psi_old = src (plain);
  // 2: diag += the tangent's diagonal on free rows
  template <typename T>
  cudaError_t reinit_integrate(const ReinitLaunch<T> &h, int mode, cudaStream_t s);
  // normal-vector (mode 0: out_d += int grad_d psi phi, normalised on request) and curvature (mode 1:
  // out0 += -int div(normalize(n_i, tol)) phi) right-hand sides, FE_Q(1, 2), free rows only
  // band_ls / band: optional narrow band (integrand masked where |band_ls(x_q)| >= band)
  cudaError_t level_set_rhs(const GridDesc &g, int K, const double hlen[3], int mode, int normalized, double tol,
                            const double *in0, const double *in1, const double *in2, double *out0, double *out1,
                            double *out2, cudaStream_t s, const double *band_ls = nullptr, double band = 0.0);

  // whether mode (0 tangent / 2 diagonal, 1 rhs) has any face to integrate
  bool heat_faces_active(const HeatFaceBC &bc, int mode);

  template <typename T>
  cudaError_t heat_faces(const HeatFaceLaunch<T> &h, cudaStream_t s);

  // ---- advection-diffusion (source/level_set/advection_diffusion_operator.cpp)
  struct AdvParams
  {
    double inv_dt;
    double theta_adv; // multiplies v . grad u
    double theta_dif; // multiplies eps grad u . grad phi (already times eps)
    double vel[12];   // v(x) = vel[0..2] + G x, G = vel[3..11] row-major
    double origin[3];
    double h[3];
    int    supg      = 0;   // SUPG streamline stabilisation (ConvectionStabilizationType::SUPG)
    double supg_coef = 0.0; // < 0: tau_c = h_c / max_q |v|, else tau_c = supg_coef h_c
    const double *vfield[3] = {nullptr, nullptr, nullptr}; // velocity as a DoF vector (else affine)
  };

  template <typename T>
  struct AdvLaunch
  {
    int       degree   = 2;
    int       mode     = 0;
    double    scale    = 1.0;
    AdvParams p{};
    GridDesc  grid{};
    SyncDesc  sync{};
    const T  *src      = nullptr;
    T        *dst      = nullptr;
    const T  *b        = nullptr;
    int       mask_src = 1;
    const int *skip    = nullptr;
  };

  template <typename T>
  cudaError_t adv_apply(const AdvLaunch<T> &h, cudaStream_t s);

  // per-cell diagonal entries gathered per DoF, then optionally inverted with the advection rule
  template <typename T>
  cudaError_t adv_diagonal(const GridDesc &g, int K, const AdvParams &p, T *diag, cudaStream_t s);
  // adds the SUPG part of the diagonal (p.supg) on the free rows
  template <typename T>
  cudaError_t adv_supg_diagonal(const GridDesc &g, int K, const AdvParams &p, T *diag, cudaStream_t s);
  // diagonal of the tangent with a DoF-vector velocity (p.vfield), added on the free rows (FP64)
  cudaError_t adv_field_diagonal(const GridDesc &g, int K, const AdvParams &p, double *diag, cudaStream_t s);

  template <typename T>
  void adv_brick_shape(int K, int shape[3]);

  // ---- vectors and reductions (double accumulation for every vector type)
  constexpr int RED_BLOCKS  = 592; // 4 x 148 SMs
  constexpr int RED_THREADS = 256;

  struct Reducer
  {
    double   *partials; // RED_BLOCKS * 8
    unsigned *counter;  // last-block ticket
  };

  // PCG state kept on the device (deal.II SolverCG + ReductionControl semantics)
  struct CGState
  {
    double rho;      // r . z of the current iteration
    double alpha;
    double beta;
    double res0;     // initial residual norm
    double tol;      // max(abs_tol, rel_tol * res0)
    double abs_tol;
    double rel_tol;
    double res;      // last residual norm
    int    it;       // completed iterations
    int    max_it;
    int    done;     // 0 iterate, 1 converged, 2 failed
    int    pad;
  };

  template <typename T>
  cudaError_t cg_init(const T *r, const T *invd, T *p, CGState *st, double *hist, Reducer red, long long n,
                      cudaStream_t s);
  template <typename T>
  cudaError_t cg_update_p(const T *r, const T *invd, T *p, const CGState *st, long long n, cudaStream_t s);
  template <typename T>
  cudaError_t cg_alpha(const T *p, const T *v, CGState *st, Reducer red, long long n, cudaStream_t s);
  template <typename T>
  cudaError_t cg_update_xr(T *x, T *r, const T *p, const T *v, const T *invd, CGState *st, double *hist,
                           Reducer red, long long n, cudaStream_t s);

  // generic helpers
  template <typename T>
  cudaError_t vec_fill(T *x, T v, long long n, cudaStream_t s);
  template <typename Tdst, typename Tsrc>
  cudaError_t vec_convert(Tdst *dst, const Tsrc *src, long long n, cudaStream_t s);
  // dst = a*x + b*y (elementwise, any of x / y may be null meaning 0)
  template <typename T>
  cudaError_t vec_axpby(T *dst, double a, const T *x, double b, const T *y, long long n, cudaStream_t s);
  // x64 += (double) e32
  cudaError_t vec_add_f32_to_f64(double *x, const float *e, long long n, cudaStream_t s);
  // out[k] = sum_i x_k[i] * y_k[i], k < m <= 8 (deterministic)
  template <typename T>
  cudaError_t vec_multidot(const T *const *x, const T *const *y, int m, long long n, double *out_dev, Reducer red,
                           cudaStream_t s);
  // h_k = w . v_k (k < m), out[m] = ||w||^2
  template <typename T>
  cudaError_t vec_dots_against(const T *w, const T *const *v, int m, long long n, double *out_dev, Reducer red,
                               cudaStream_t s);
  // dst = src * invd (Jacobi)
  template <typename T>
  cudaError_t vec_scale(T *dst, const T *src, const T *invd, long long n, cudaStream_t s);
  // x += sum_k c_k v_k (coefficients on the device), then optionally x *= invd first on the sum
  template <typename T>
  cudaError_t vec_multiaxpy(T *x, const T *const *v, const double *coef_dev, int m, long long n, double post_scale,
                            cudaStream_t s);
  // w -= sum_k h_k v_k and returns ||w||^2 into out_dev (coefficients on the device)
  template <typename T>
  cudaError_t vec_orth_update(T *w, const T *const *v, const double *h_dev, int m, long long n, double *out_dev,
                              Reducer red, cudaStream_t s);
  // inverse of a diagonal with the heat rule (|d| > thr ? 1/d : 1) in place
  template <typename T>
  cudaError_t vec_invert(T *d, double thr, long long n, cudaStream_t s);
  // max |d| (deterministic) into out_dev
  template <typename T>
  cudaError_t vec_absmax(const T *d, long long n, double *out_dev, Reducer red, cudaStream_t s);
  // d = |d| > 1e-14 max(1, *amax) ? 1/d : 1 (advection rule, amax on the device)
  template <typename T>
  cudaError_t vec_invert_rel(T *d, const double *amax_dev, long long n, cudaStream_t s);
  // records an error message for mpdg_last_error() and returns code (capi.cu)
  int record_failure(int code, const char *msg);
  // adjoint helpers (adjoint.cu): g_c (+)= scale k_c lam_c^T K_c T_c, and k = exp(z)
  cudaError_t heat_cell_form(const GridDesc &g, int K, const HeatGeom &geo, double scale, const double *lam,
                             const double *T, const double *k, double kconst, double *out, bool accumulate,
                             cudaStream_t s);
  cudaError_t vec_exp(double *k, const double *z, long long n, cudaStream_t s);
  // set constrained entries (face mask / per-DoF mask) of x to v
  template <typename T>
  cudaError_t vec_set_constrained(T *x, T v, const GridDesc &g, cudaStream_t s);
  // dst = src on constrained DoFs, 0 elsewhere
  template <typename T>
  cudaError_t vec_copy_constrained(T *dst, const T *src, const GridDesc &g, cudaStream_t s);
  // dst = src on constrained DoFs, other entries untouched
  template <typename T>
  cudaError_t vec_distribute_constrained(T *dst, const T *src, const GridDesc &g, cudaStream_t s);
  // dst[idx[k]] += scale src[idx[k]];  dst[idx[k]] = vals ? vals[k] : fill;  out[k] = src[idx[k]]
  template <typename T>
  cudaError_t idx_add_scaled(T *dst, const T *src, const long long *idx, long long n, double scale, cudaStream_t s);
  template <typename T>
  cudaError_t idx_set(T *dst, const long long *idx, const double *vals, long long n, T fill, cudaStream_t s);
  cudaError_t idx_gather(double *out, const double *src, const long long *idx, long long n, cudaStream_t s);
} // namespace mpdg
