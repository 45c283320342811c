// Advection-diffusion operator kernels.  Reference: source/level_set/advection_diffusion_operator.cpp
//   vmult :236-272 (cell_loop, zero dst), tangent_local_cell_operation :448-495
//     val = u/dt + theta v.grad u,  grad = theta eps grad u
//   create_rhs :274-358: val = u_old/dt - (1-theta) v.grad u_old, grad = -(1-theta) eps grad u_old
//     (the same kernel with theta replaced by theta - 1, plain reads)
//   compute_inverse_diagonal_from_matrixfree :399-446
// The velocity is an affine field v(x) = v0 + G x evaluated analytically at the Gauss points (the
// reference evaluates a dealii::Function there, :475-479); rigid rotations are affine.
//
// Per cell (one thread), FEEvaluation-style sum factorisation in registers:
//   u_q = (B(x)B(x)B) u;  for d: g = D_d u_q (collocation derivative on the Gauss points),
//   R += JxW theta v_d g / h_d,  R += D_d^T (JxW theta eps g / h_d^2);  out = (B(x)B(x)B)^T R,
// starting from R = JxW u_q / dt.  Peak register use is three cell arrays (u_q, R, g).
//
// SUPG (ConvectionStabilizationType::SUPG, :455-457, :486-490, stabilisation parameter :497-533):
// the strong residual s = u/dt + theta v.grad u - theta eps lap u at the Gauss points (the second
// derivative is the collocation derivative applied twice: exact for the degree-k interpolant), tested
// with tau_c v.grad phi; tau_c = (coefficient < 0 ? 1 / max_q |v| (0 below 1e-6) : coefficient) times
// the cell size diameter / sqrt(3) (source/core/scratch_data.cpp:262-277).  The rhs uses the same
// form with theta replaced by theta - 1 (:322-345).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <set>

#include "brick.cuh"
#include "kernels.h"
#include "sumfac.cuh"

namespace mpdg
{
  // Per degree (1..3) in constant memory, uploaded once per device:
  //   [B (n*n): phi_i(x_q) | D (n*n): collocation derivative on the Gauss points |
  //    qp (n): Gauss points | qw3 (n^3): tensor Gauss weights]
  constexpr int ADV_KMAX = 3;
  constexpr int ADV_TAB  = 2 * 16 + 4 + 64;
  __constant__ double c_adv_d[ADV_KMAX + 1][ADV_TAB];
  __constant__ float  c_adv_f[ADV_KMAX + 1][ADV_TAB];

  template <typename T>
  __device__ __forceinline__ const T *
  adv_table(int K)
  {
    if constexpr (sizeof(T) == 8)
      return c_adv_d[K];
    else
      return c_adv_f[K];
  }

  template <typename T, int N>
  struct AdvArgs
  {
    T            det;
    T            supg_coef, cell_size;
    GridDesc     g;
    SyncDesc     s;
    T            inv_dt, th_adv, th_dif; // already multiplied by scale
    T            vel[12];
    T            origin[3], h[3];
    const T     *src;
    T           *dst;
    const T     *b;
    int          mask_src;
    const int   *skip;
    const double *vfield[3]; // velocity as a DoF vector (three FE_Q(k) components), else affine
    // cell-independent factors per direction d and Gauss point q (N^3 <= 27 used):
    //   pa = th_adv det / h_d w_q,  pb = pa (G_d. (h (x) qp_q)),  pd = th_dif det / h_d^2 w_q;
    // pm = det inv_dt w_q.  The velocity term of a cell is (vd0 pa + pb) g, vd0 = v_d(cell origin).
    T pa[3][64], pb[3][64], pd[3][64], pm[64];
  };

  // out = M in along a line (in place), M[a*N+b], TR: transpose
  template <typename T, int N, int S, bool TR>
  __device__ __forceinline__ void
  line_mat(T *v, const int base, const T *M)
  {
    T in[N];
#pragma unroll
    for (int k = 0; k < N; ++k)
      in[k] = v[base + k * S];
#pragma unroll
    for (int a = 0; a < N; ++a)
      {
        T s = (TR ? M[a] : M[a * N]) * in[0];
#pragma unroll
        for (int k = 1; k < N; ++k)
          s = fma(TR ? M[k * N + a] : M[a * N + k], in[k], s);
        v[base + a * S] = s;
      }
  }

  // acc += M^T g along a line
  template <typename T, int N, int S>
  __device__ __forceinline__ void
  line_mat_tr_acc(T *acc, const T *g, const int base, const T *M)
  {
#pragma unroll
    for (int a = 0; a < N; ++a)
      {
        T s = acc[base + a * S];
#pragma unroll
        for (int k = 0; k < N; ++k)
          s = fma(M[k * N + a], g[base + k * S], s);
        acc[base + a * S] = s;
      }
  }

  template <typename T, int N, int D, bool TR>
  __device__ __forceinline__ void
  sweep(T *v, const T *M)
  {
    constexpr int S = D == 0 ? 1 : (D == 1 ? N : N * N);
#pragma unroll
    for (int a = 0; a < N; ++a)
#pragma unroll
      for (int c = 0; c < N; ++c)
        {
          const int base = D == 0 ? (a * N + c) * N : (D == 1 ? a * N * N + c : a * N + c);
          line_mat<T, N, S, TR>(v, base, M);
        }
  }

  template <typename T, int N, int D>
  __device__ __forceinline__ void
  sweep_tr_acc(T *acc, const T *g, const T *M)
  {
    constexpr int S = D == 0 ? 1 : (D == 1 ? N : N * N);
#pragma unroll
    for (int a = 0; a < N; ++a)
#pragma unroll
      for (int c = 0; c < N; ++c)
        {
          const int base = D == 0 ? (a * N + c) * N : (D == 1 ? a * N * N + c : a * N + c);
          line_mat_tr_acc<T, N, S>(acc, g, base, M);
        }
  }

  // One direction d of the advection and diffusion terms, line by line (a line along d at a time):
  //   g = D_d uq along the line;  R += theta_adv v_d JxW g / h_d;  R += D_d^T (theta_dif JxW g / h_d^2)
  // with the cell-independent factors of each point precomputed (AdvArgs::pa, pb, pd): the velocity
  // weight is vd0 pa_q + pb_q (affine field) or vq_q pa_q (DoF-vector field).  Only the k+1 values of
  // one line are live besides uq and R.
  template <typename T, int N, int D>
  __device__ __forceinline__ void
  adv_direction(const T *uq, T *R, const T *tD, const T *pa, const T *pb, const T *pd, T vd0, bool dif,
                const T *vq = nullptr)
  {
    constexpr int S = D == 0 ? 1 : (D == 1 ? N : N * N);
#pragma unroll
    for (int a = 0; a < N; ++a)
#pragma unroll
      for (int c = 0; c < N; ++c)
        {
          const int base = D == 0 ? (a * N + c) * N : (D == 1 ? a * N * N + c : a * N + c);
          T         g[N];
#pragma unroll
          for (int r = 0; r < N; ++r)
            {
              T s = tD[r * N] * uq[base];
#pragma unroll
              for (int k = 1; k < N; ++k)
                s = fma(tD[r * N + k], uq[base + k * S], s);
              g[r] = s;
            }
#pragma unroll
          for (int r = 0; r < N; ++r)
            {
              const int q = base + r * S;
              const T   w = vq ? vq[q] * pa[q] : fma(vd0, pa[q], pb[q]);
              R[q]        = fma(w, g[r], R[q]);
              g[r] *= pd[q];
            }
          if (dif)
#pragma unroll
            for (int r = 0; r < N; ++r)
              {
                T s = R[base + r * S];
#pragma unroll
                for (int k = 0; k < N; ++k)
                  s = fma(tD[k * N + r], g[k], s);
                R[base + r * S] = s;
              }
        }
  }

  // SUPG, direction D of the strong residual: s += theta_adv v_d (D_d u_q) / h_d - theta_dif (D_d D_d u_q) / h_d^2
  // (v_d from the affine field, or vq = v_d at the Gauss points of a DoF-vector field)
  template <typename T, int N, int D>
  __device__ __forceinline__ void
  supg_residual(const T *uq, T *sres, const T *tD, const T *tqp, T inv_h, T vd0, T gx, T gy, T gz, T th_adv,
                T th_dif, const T *vq = nullptr)
  {
    constexpr int S = D == 0 ? 1 : (D == 1 ? N : N * N);
#pragma unroll
    for (int a = 0; a < N; ++a)
#pragma unroll
      for (int c = 0; c < N; ++c)
        {
          const int base = D == 0 ? (a * N + c) * N : (D == 1 ? a * N * N + c : a * N + c);
          T         g[N];
#pragma unroll
          for (int r = 0; r < N; ++r)
            {
              T s = tD[r * N] * uq[base];
#pragma unroll
              for (int k = 1; k < N; ++k)
                s = fma(tD[r * N + k], uq[base + k * S], s);
              g[r] = s;
            }
#pragma unroll
          for (int r = 0; r < N; ++r)
            {
              T gg = tD[r * N] * g[0];
#pragma unroll
              for (int k = 1; k < N; ++k)
                gg = fma(tD[r * N + k], g[k], gg);
              const int q  = base + r * S;
              const int qx = q % N, qy = (q / N) % N, qz = q / (N * N);
              const T   vd = vq ? vq[q] : vd0 + gx * tqp[qx] + gy * tqp[qy] + gz * tqp[qz];
              sres[q] += th_adv * vd * g[r] * inv_h - th_dif * gg * inv_h * inv_h;
            }
        }
  }

  // SUPG, direction D of the test with tau v.grad phi: R += D_d^T (c_t w3 v_d s), c_t = tau det / h_d
  template <typename T, int N, int D>
  __device__ __forceinline__ void
  supg_test(const T *sres, T *R, const T *tD, const T *tqp, const T *tw3, T c_t, T vd0, T gx, T gy, T gz,
            const T *vq = nullptr)
  {
    constexpr int S = D == 0 ? 1 : (D == 1 ? N : N * N);
#pragma unroll
    for (int a = 0; a < N; ++a)
#pragma unroll
      for (int c = 0; c < N; ++c)
        {
          const int base = D == 0 ? (a * N + c) * N : (D == 1 ? a * N * N + c : a * N + c);
          T         t[N];
#pragma unroll
          for (int r = 0; r < N; ++r)
            {
              const int q  = base + r * S;
              const int qx = q % N, qy = (q / N) % N, qz = q / (N * N);
              const T   vd = vq ? vq[q] : vd0 + gx * tqp[qx] + gy * tqp[qy] + gz * tqp[qz];
              t[r]         = c_t * tw3[q] * vd * sres[q];
            }
#pragma unroll
          for (int r = 0; r < N; ++r)
            {
              T s = R[base + r * S];
#pragma unroll
              for (int k = 0; k < N; ++k)
                s = fma(tD[k * N + r], t[k], s);
              R[base + r * S] = s;
            }
        }
  }

  // tau_c of the cell with lower corner (x0, y0, z0)
  template <typename T, int N>
  __device__ __forceinline__ T
  supg_tau(const T *vel, const T *h, const T *tqp, T x0, T y0, T z0, T coef, T cell_size)
  {
    T tau = coef;
    if (coef < T(0))
      {
        T vmax = T(0);
#pragma unroll
        for (int qz = 0; qz < N; ++qz)
#pragma unroll
          for (int qy = 0; qy < N; ++qy)
#pragma unroll
            for (int qx = 0; qx < N; ++qx)
              {
                const T x = x0 + h[0] * tqp[qx], y = y0 + h[1] * tqp[qy], z = z0 + h[2] * tqp[qz];
                T       n2 = T(0);
#pragma unroll
                for (int d = 0; d < 3; ++d)
                  {
                    const T v = vel[d] + vel[3 + 3 * d] * x + vel[4 + 3 * d] * y + vel[5 + 3 * d] * z;
                    n2        = fma(v, v, n2);
                  }
                vmax = fmax(vmax, sqrt(n2));
              }
        tau = vmax >= T(1e-6) ? T(1) / vmax : T(0);
      }
    return tau * cell_size;
  }

#ifndef MPDG_ADV_MINB_F64
#define MPDG_ADV_MINB_F64 2
#endif
#ifndef MPDG_ADV_MINB_F32
#define MPDG_ADV_MINB_F32 4
#endif

  template <int K, typename T>
  struct AdvLayout
  {
    static constexpr int  N  = K + 1;
    static constexpr int  BX = 8, BY = 8, BZ = (K == 1 ? 8 : (K == 2 ? 4 : 2));
    static constexpr int  NT = BX * BY * BZ;
    using BR                 = Brick<K, BX, BY, BZ, NT>;
    static constexpr size_t bytes = sizeof(T) * 2 * (size_t)BR::NPTS; // staged input + accumulator
    // SUPG with a DoF-vector velocity at k <= 2: the velocity's three components staged as well
    static constexpr bool   STAGE_FIELD  = K <= 2;
    static constexpr size_t bytes_staged = bytes + sizeof(double) * 3 * (size_t)BR::NPTS;
    // CTAs per SM (k = 3: two CTAs of 128 threads, so that the two 64-value cell arrays fit registers)
    static constexpr int    MINB  = K == 3 ? 2 : (sizeof(T) == 8 ? MPDG_ADV_MINB_F64 : MPDG_ADV_MINB_F32);
  };

  // The SUPG form keeps a third cell array (the strong residual).  At k = 2 it is held to half the
  // CTAs per SM of the plain form (at least one); at k = 1 the arrays are small and the plain
  // occupancy wins despite some spilling (Q1 FP64: 658 against 988 us per 7.2 M DoFs).
  template <int K, typename T, bool SUPG>
  struct AdvMinBlocks
  {
    static constexpr int value =
      (SUPG && K == 2) ? (AdvLayout<K, T>::MINB > 1 ? AdvLayout<K, T>::MINB / 2 : 1) : AdvLayout<K, T>::MINB;
  };

  // Velocity component d of a DoF-vector field at the cell's Gauss points: the cell's nodal values
  // read plainly (advection_diffusion_operator.cpp:461-466), interpolated by three sweeps of B.
  template <typename T, int N>
  __device__ __forceinline__ void
  field_at_points(const double *f, const GridDesc &g, int cx, int cy, int cz, const T *tB, T *vq)
  {
    constexpr int K = N - 1;
#pragma unroll
    for (int l = 0; l < N; ++l)
#pragma unroll
      for (int j = 0; j < N; ++j)
#pragma unroll
        for (int i = 0; i < N; ++i)
          vq[(l * N + j) * N + i] =
            (T)f[(long long)(K * cx + i) + (long long)g.n[0] * ((long long)(K * cy + j) + (long long)g.n[1] * (K * cz + l))];
    sweep<T, N, 0, false>(vq, tB);
    sweep<T, N, 1, false>(vq, tB);
    sweep<T, N, 2, false>(vq, tB);
  }

  // The same from the brick's staged copy of the component (cell's first point at brick index base)
  template <typename T, int N, int PX, int PY>
  __device__ __forceinline__ void
  field_at_points_staged(const double *sf, int base, const T *tB, T *vq)
  {
#pragma unroll
    for (int l = 0; l < N; ++l)
#pragma unroll
      for (int j = 0; j < N; ++j)
#pragma unroll
        for (int i = 0; i < N; ++i)
          vq[(l * N + j) * N + i] = (T)sf[base + l * PY * PX + j * PX + i];
    sweep<T, N, 0, false>(vq, tB);
    sweep<T, N, 1, false>(vq, tB);
    sweep<T, N, 2, false>(vq, tB);
  }

  // SUPG = true: the stabilised form; VDOF = true: the velocity is a DoF vector (three cell arrays
  // live in both cases; the DoF-vector form keeps the plain form's occupancy and spills, measured
  // faster than half the CTAs per SM: 287 against 375 us FP64, 194 against 216 us FP32 on 96^3 k = 2)
  template <int K, typename T, OutMode MODE, bool SUPG, bool VDOF = false>
  __global__ void __launch_bounds__(AdvLayout<K, T>::BR::NT, AdvMinBlocks<K, T, SUPG>::value)
  adv_apply_kernel(const __grid_constant__ AdvArgs<T, K + 1> a)
  {
    using LAY             = AdvLayout<K, T>;
    using BR              = typename LAY::BR;
    constexpr int  N      = K + 1, NT = BR::NT, NP = BR::NPTS, PX = BR::PX, PY = BR::PY;
    constexpr int  BX     = BR::BX, BY = BR::BY;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *const s_src = reinterpret_cast<T *>(smem_raw);
    T *const s_dst = s_src + NP;
    __shared__ unsigned s_ticket;
    if (a.skip != nullptr && *a.skip != 0)
      return;

    BR br;
    if (!brick_begin<BR, T, MODE>(br, a.g, a.s, a.dst, a.b, &s_ticket))
      return;
    for (int p = threadIdx.x; p < NP; p += NT)
      s_dst[p] = T(0);
    // SUPG with a DoF-vector velocity reads each component three times per cell: staged per brick
    constexpr bool STAGE = SUPG && VDOF && LAY::STAGE_FIELD;
    double *const  s_f   = reinterpret_cast<double *>(s_dst + NP);
    if constexpr (STAGE)
#pragma unroll
      for (int d = 0; d < 3; ++d)
        brick_stage<BR, double, false>(br, a.vfield[d], false, s_f + d * NP);
    brick_stage(br, a.src, a.mask_src != 0, s_src);

    const int  tx = threadIdx.x % BX, ty = (threadIdx.x / BX) % BY, tz = threadIdx.x / (BX * BY);
    const int  cx = br.c0[0] + tx, cy = br.c0[1] + ty, cz = br.c0[2] + tz;
    const bool valid = cx < a.g.m[0] && cy < a.g.m[1] && cz < a.g.m[2];
    const int  base = (K * tz) * PY * PX + (K * ty) * PX + K * tx;

    const T *tb  = adv_table<T>(K);
    const T *tB  = tb, *tD = tb + N * N, *tqp = tb + 2 * N * N, *tw3 = tb + 2 * N * N + N;
    // velocity component d of a DoF-vector field at the cell's Gauss points
    auto field = [&](int d, T *vq) {
      if constexpr (STAGE)
        field_at_points_staged<T, N, PX, PY>(s_f + d * NP, base, tB, vq);
      else
        field_at_points<T, N>(a.vfield[d], a.g, cx, cy, cz, tB, vq);
    };
    T uq[N * N * N], R[N * N * N];
    if (valid)
      {
#pragma unroll
        for (int l = 0; l < N; ++l)
#pragma unroll
          for (int j = 0; j < N; ++j)
#pragma unroll
            for (int i = 0; i < N; ++i)
              uq[(l * N + j) * N + i] = s_src[base + l * PY * PX + j * PX + i];
        sweep<T, N, 0, false>(uq, tB);
        sweep<T, N, 1, false>(uq, tB);
        sweep<T, N, 2, false>(uq, tB);
        // cell origin and the velocity there
        const T x0 = a.origin[0] + a.h[0] * cx, y0 = a.origin[1] + a.h[1] * cy, z0 = a.origin[2] + a.h[2] * cz;
#pragma unroll
        for (int q = 0; q < N * N * N; ++q)
          R[q] = a.pm[q] * uq[q];
        {
          const T th_adv = a.th_adv, th_dif = a.th_dif;
#define MPDG_ADV_DIR(d)                                                                                         \
  {                                                                                                             \
    const T vd0 = a.vel[d] + a.vel[3 + 3 * d] * x0 + a.vel[4 + 3 * d] * y0 + a.vel[5 + 3 * d] * z0;            \
    if constexpr (VDOF)                                                                                         \
      {                                                                                                         \
        T vq[N * N * N];                                                                                        \
        field(d, vq);                                                                                           \
        adv_direction<T, N, d>(uq, R, tD, a.pa[d], a.pb[d], a.pd[d], vd0, th_dif != T(0), vq);                  \
      }                                                                                                         \
    else                                                                                                        \
      adv_direction<T, N, d>(uq, R, tD, a.pa[d], a.pb[d], a.pd[d], vd0, th_dif != T(0));                       \
  }
          if constexpr (SUPG && VDOF)
            {
              // SUPG with a DoF-vector velocity: one component at the Gauss points at a time (four
              // cell arrays live: u_q, R, the strong residual and the component).  Pass 1: the
              // advection terms and |v|^2 at the points (kept in the residual's array) for tau_c
              // (advection_diffusion_operator.cpp:510-520); pass 2: the strong residual; pass 3 its test
              // with tau_c v.grad phi.
              T sres[N * N * N], vq[N * N * N];
#pragma unroll
              for (int q = 0; q < N * N * N; ++q)
                sres[q] = T(0);
#pragma unroll
              for (int d = 0; d < 3; ++d)
                {
                  field(d, vq);
                  if (d == 0)
                    adv_direction<T, N, 0>(uq, R, tD, a.pa[0], a.pb[0], a.pd[0], T(0), th_dif != T(0), vq);
                  else if (d == 1)
                    adv_direction<T, N, 1>(uq, R, tD, a.pa[1], a.pb[1], a.pd[1], T(0), th_dif != T(0), vq);
                  else
                    adv_direction<T, N, 2>(uq, R, tD, a.pa[2], a.pb[2], a.pd[2], T(0), th_dif != T(0), vq);
#pragma unroll
                  for (int q = 0; q < N * N * N; ++q)
                    sres[q] = fma(vq[q], vq[q], sres[q]);
                }
              T tau = a.supg_coef;
              if (tau < T(0))
                {
                  T vmax = T(0);
#pragma unroll
                  for (int q = 0; q < N * N * N; ++q)
                    vmax = fmax(vmax, sqrt(sres[q]));
                  tau = vmax >= T(1e-6) ? T(1) / vmax : T(0);
                }
              tau *= a.cell_size;
#pragma unroll
              for (int q = 0; q < N * N * N; ++q)
                sres[q] = a.inv_dt * uq[q];
              const T ih[3] = {T(1) / a.h[0], T(1) / a.h[1], T(1) / a.h[2]};
              const T z     = T(0);
              field(0, vq);
              supg_residual<T, N, 0>(uq, sres, tD, tqp, ih[0], z, z, z, z, th_adv, th_dif, vq);
              field(1, vq);
              supg_residual<T, N, 1>(uq, sres, tD, tqp, ih[1], z, z, z, z, th_adv, th_dif, vq);
              field(2, vq);
              supg_residual<T, N, 2>(uq, sres, tD, tqp, ih[2], z, z, z, z, th_adv, th_dif, vq);
              const T td = tau * a.det;
              field(0, vq);
              supg_test<T, N, 0>(sres, R, tD, tqp, tw3, td * ih[0], z, z, z, z, vq);
              field(1, vq);
              supg_test<T, N, 1>(sres, R, tD, tqp, tw3, td * ih[1], z, z, z, z, vq);
              field(2, vq);
              supg_test<T, N, 2>(sres, R, tD, tqp, tw3, td * ih[2], z, z, z, z, vq);
            }
          else
            {
              MPDG_ADV_DIR(0)
              MPDG_ADV_DIR(1)
              MPDG_ADV_DIR(2)
            }
#undef MPDG_ADV_DIR
          if constexpr (SUPG && !VDOF)
            {
              const T tau = supg_tau<T, N>(a.vel, a.h, tqp, x0, y0, z0, a.supg_coef, a.cell_size);
              T       sres[N * N * N];
#pragma unroll
              for (int q = 0; q < N * N * N; ++q)
                sres[q] = a.inv_dt * uq[q];
              T vd0[3], gv[3][3], ih[3];
#pragma unroll
              for (int d = 0; d < 3; ++d)
                {
                  ih[d]  = T(1) / a.h[d];
                  vd0[d] = a.vel[d] + a.vel[3 + 3 * d] * x0 + a.vel[4 + 3 * d] * y0 + a.vel[5 + 3 * d] * z0;
#pragma unroll
                  for (int e = 0; e < 3; ++e)
                    gv[d][e] = a.vel[3 + 3 * d + e] * a.h[e];
                }
              supg_residual<T, N, 0>(uq, sres, tD, tqp, ih[0], vd0[0], gv[0][0], gv[0][1], gv[0][2], th_adv, th_dif);
              supg_residual<T, N, 1>(uq, sres, tD, tqp, ih[1], vd0[1], gv[1][0], gv[1][1], gv[1][2], th_adv, th_dif);
              supg_residual<T, N, 2>(uq, sres, tD, tqp, ih[2], vd0[2], gv[2][0], gv[2][1], gv[2][2], th_adv, th_dif);
              const T td = tau * a.det;
              supg_test<T, N, 0>(sres, R, tD, tqp, tw3, td * ih[0], vd0[0], gv[0][0], gv[0][1], gv[0][2]);
              supg_test<T, N, 1>(sres, R, tD, tqp, tw3, td * ih[1], vd0[1], gv[1][0], gv[1][1], gv[1][2]);
              supg_test<T, N, 2>(sres, R, tD, tqp, tw3, td * ih[2], vd0[2], gv[2][0], gv[2][1], gv[2][2]);
            }
        }
        sweep<T, N, 2, true>(R, tB);
        sweep<T, N, 1, true>(R, tB);
        sweep<T, N, 0, true>(R, tB);
        // cells sharing a lattice point add into the brick accumulator concurrently
#pragma unroll
        for (int l = 0; l < N; ++l)
#pragma unroll
          for (int j = 0; j < N; ++j)
#pragma unroll
            for (int i = 0; i < N; ++i)
              atomicAdd(s_dst + (base + l * PY * PX + j * PX + i), R[(l * N + j) * N + i]);
      }
    __syncthreads();
    brick_end<BR, T, MODE>(br, a.g, a.s, s_dst, a.dst, a.b);
  }

  // ------------------------------------------------------------------------------------------
  static cudaError_t
  upload_adv_tables()
  {
    static std::mutex           mtx;
    static std::set<int>        done;
    int                         dev = 0;
    cudaError_t                 e   = cudaGetDevice(&dev);
    if (e != cudaSuccess)
      return e;
    std::lock_guard<std::mutex> lock(mtx);
    if (done.count(dev))
      return cudaSuccess;
    double hd[ADV_KMAX + 1][ADV_TAB] = {};
    float  hf[ADV_KMAX + 1][ADV_TAB] = {};
    for (int K = 1; K <= ADV_KMAX; ++K)
      {
        const Tables1D &t = tables(K);
        const int       n = t.n;
        int             o = 0;
        for (int i = 0; i < n * n; ++i)
          hd[K][o++] = t.B[i];
        for (int i = 0; i < n * n; ++i)
          hd[K][o++] = t.Dq[i];
        for (int i = 0; i < n; ++i)
          hd[K][o++] = t.qp[i];
        for (int qz = 0; qz < n; ++qz)
          for (int qy = 0; qy < n; ++qy)
            for (int qx = 0; qx < n; ++qx)
              hd[K][o++] = t.qw[qx] * t.qw[qy] * t.qw[qz];
        for (int i = 0; i < o; ++i)
          hf[K][i] = (float)hd[K][i];
      }
    if ((e = cudaMemcpyToSymbol(c_adv_d, hd, sizeof(hd))) != cudaSuccess)
      return e;
    if ((e = cudaMemcpyToSymbol(c_adv_f, hf, sizeof(hf))) != cudaSuccess)
      return e;
    // the copies ran on the legacy stream: complete them before kernels on other streams read the tables
    if ((e = cudaStreamSynchronize(cudaStreamLegacy)) != cudaSuccess)
      return e;
    done.insert(dev);
    return cudaSuccess;
  }

  template <int K, typename T, OutMode MODE>
  static cudaError_t
  launch_adv(const AdvLaunch<T> &h, cudaStream_t stream)
  {
    constexpr int   N = K + 1;
    using LAY         = AdvLayout<K, T>;
    AdvArgs<T, N> a;
    cudaError_t   ue = upload_adv_tables();
    if (ue != cudaSuccess)
      return ue;
    a.det = (T)(h.p.h[0] * h.p.h[1] * h.p.h[2]);
    a.g      = h.grid;
    a.s      = h.sync;
    a.inv_dt = (T)(h.scale * h.p.inv_dt);
    a.th_adv = (T)(h.scale * h.p.theta_adv);
    a.th_dif = (T)(h.scale * h.p.theta_dif);
    for (int i = 0; i < 12; ++i)
      a.vel[i] = (T)h.p.vel[i];
    for (int d = 0; d < 3; ++d)
      {
        a.origin[d] = (T)h.p.origin[d];
        a.h[d]      = (T)h.p.h[d];
      }
    a.src      = h.src;
    a.dst      = h.dst;
    a.b        = h.b;
    a.mask_src = h.mask_src;
    a.skip     = h.skip;
    a.supg_coef = (T)h.p.supg_coef;
    a.cell_size = (T)(std::sqrt(h.p.h[0] * h.p.h[0] + h.p.h[1] * h.p.h[1] + h.p.h[2] * h.p.h[2]) / std::sqrt(3.0));
    for (int d = 0; d < 3; ++d)
      a.vfield[d] = h.p.vfield[d];
    {
      // cell-independent point factors (see AdvArgs), in double, rounded once
      const Tables1D &t   = tables(K);
      const double    det = h.p.h[0] * h.p.h[1] * h.p.h[2];
      const double    ta = h.scale * h.p.theta_adv, td = h.scale * h.p.theta_dif, ti = h.scale * h.p.inv_dt;
      for (int qz = 0; qz < N; ++qz)
        for (int qy = 0; qy < N; ++qy)
          for (int qx = 0; qx < N; ++qx)
            {
              const int    q  = (qz * N + qy) * N + qx;
              const double w3 = t.qw[qx] * t.qw[qy] * t.qw[qz];
              a.pm[q]         = (T)(det * ti * w3);
              for (int d = 0; d < 3; ++d)
                {
                  const double pa = ta * det / h.p.h[d] * w3;
                  const double gv = h.p.vel[3 + 3 * d] * h.p.h[0] * t.qp[qx] + h.p.vel[4 + 3 * d] * h.p.h[1] * t.qp[qy] +
                                    h.p.vel[5 + 3 * d] * h.p.h[2] * t.qp[qz];
                  a.pa[d][q] = (T)pa;
                  a.pb[d][q] = (T)(pa * gv);
                  a.pd[d][q] = (T)(td * det / (h.p.h[d] * h.p.h[d]) * w3);
                }
            }
    }
    const bool vdof = h.p.vfield[0] != nullptr;
    auto kern = h.p.supg ? (vdof ? adv_apply_kernel<K, T, MODE, true, true> : adv_apply_kernel<K, T, MODE, true>)
                         : (vdof ? adv_apply_kernel<K, T, MODE, false, true> : adv_apply_kernel<K, T, MODE, false>);
    static std::atomic<unsigned long long> devices{0}, devices_supg{0}, devices_vdof{0}, devices_sv{0};
    const size_t bytes = h.p.supg && vdof && LAY::STAGE_FIELD ? LAY::bytes_staged : LAY::bytes;
    if (cudaError_t e = ensure_smem(kern, bytes,
                                    h.p.supg ? (vdof ? devices_sv : devices_supg) : (vdof ? devices_vdof : devices));
        e != cudaSuccess)
      return e;
    const unsigned nbricks = (unsigned)h.grid.nbr[0] * h.grid.nbr[1] * h.grid.nbr[2];
    kern<<<nbricks, LAY::BR::NT, bytes, stream>>>(a);
    return cudaGetLastError();
  }

  template <int K, typename T>
  static cudaError_t
  adv_mode(const AdvLaunch<T> &h, cudaStream_t s)
  {
    switch (h.mode)
      {
        case 0: return launch_adv<K, T, OutMode::Set>(h, s);
        case 1: return launch_adv<K, T, OutMode::Add>(h, s);
        default: return launch_adv<K, T, OutMode::BPlus>(h, s);
      }
  }

  template <typename T>
  cudaError_t
  adv_apply(const AdvLaunch<T> &h, cudaStream_t s)
  {
    switch (h.degree)
      {
        case 1: return adv_mode<1, T>(h, s);
        case 2: return adv_mode<2, T>(h, s);
        case 3: return adv_mode<3, T>(h, s);
        default: return cudaErrorInvalidValue;
      }
  }

  template <typename T>
  void
  adv_brick_shape(int K, int shape[3])
  {
    if (K == 1)
      {
        shape[0] = AdvLayout<1, T>::BX;
        shape[1] = AdvLayout<1, T>::BY;
        shape[2] = AdvLayout<1, T>::BZ;
      }
    else if (K == 2)
      {
        shape[0] = AdvLayout<2, T>::BX;
        shape[1] = AdvLayout<2, T>::BY;
        shape[2] = AdvLayout<2, T>::BZ;
      }
    else
      {
        shape[0] = AdvLayout<3, T>::BX;
        shape[1] = AdvLayout<3, T>::BY;
        shape[2] = AdvLayout<3, T>::BZ;
      }
  }


  // ---- diagonal in closed form (MatrixFreeTools::compute_diagonal of the tangent).
  // With phi_i = phi_a(x) phi_b(y) phi_c(z) and an affine velocity, every term of
  //   A_ii = int phi_i^2 / dt + theta v . grad(phi_i) phi_i + theta eps |grad phi_i|^2
  // over a box cell is a sum of products of 1-D quadrature moments of the local indices (a, b, c):
  //   m   = h S[a],  mX = h (x0 S[a] + h S1[a])        (int phi^2,   int x phi^2)
  //   t   = T[a],    tX = x0 T[a] + h T1[a]            (int phi' phi, int x phi' phi)
  //   dd  = D[a] / h                                     (int phi'^2)
  // with S = sum w B^2, S1 = sum w q B^2, T = sum w G B, T1 = sum w q G B, D = sum w G^2 on the
  // reference Gauss rule.  One thread per DoF sums the (<= 8) cells sharing it; constrained -> 1.
  template <typename T>
  struct AdvDiagArgs
  {
    GridDesc g;
    T        S[MAX_N], S1[MAX_N], T0[MAX_N], T1[MAX_N], D[MAX_N];
    T        inv_dt, th_adv, th_dif;
    T        vel[12], origin[3], h[3];
    T       *diag;
  };

  template <int K, typename T>
  __global__ void
  adv_diag_kernel(const __grid_constant__ AdvDiagArgs<T> a)
  {
    const int       n0 = a.g.n[0], n1 = a.g.n[1];
    const long long rows = (long long)n1 * a.g.n[2];
    for (long long row = blockIdx.x; row < rows; row += gridDim.x)
      {
        const int             J = (int)(row % n1), L = (int)(row / n1);
        const Neighbours1D<K> ny(J, a.g.m[1]), nz(L, a.g.m[2]);
        for (int I = threadIdx.x; I < n0; I += blockDim.x)
          {
            const long long idx = (long long)I + (long long)n0 * row;
            if (is_constrained(a.g, I, J, L, idx))
              {
                a.diag[idx] = T(1);
                continue;
              }
            const Neighbours1D<K> nx(I, a.g.m[0]);
            const Neighbours1D<K> *nb[3] = {&nx, &ny, &nz};
            T                      d     = T(0);
#pragma unroll
            for (int z = 0; z < 2; ++z)
#pragma unroll
              for (int y = 0; y < 2; ++y)
#pragma unroll
                for (int x = 0; x < 2; ++x)
                  {
                    if (!(nx.v[x] && ny.v[y] && nz.v[z]))
                      continue;
                    const int sel[3] = {x, y, z};
                    T         m[3], mX[3], t[3], tX[3], dd[3];
#pragma unroll
                    for (int e = 0; e < 3; ++e)
                      {
                        const int li = nb[e]->l[sel[e]];
                        const T   h  = a.h[e], x0 = a.origin[e] + h * (T)nb[e]->c[sel[e]];
                        m[e]         = h * a.S[li];
                        mX[e]        = h * (x0 * a.S[li] + h * a.S1[li]);
                        t[e]         = a.T0[li];
                        tX[e]        = x0 * a.T0[li] + h * a.T1[li];
                        dd[e]        = a.D[li] / h;
                      }
                    T v = a.inv_dt * m[0] * m[1] * m[2] +
                          a.th_dif * (dd[0] * m[1] * m[2] + m[0] * dd[1] * m[2] + m[0] * m[1] * dd[2]);
                    T adv = T(0);
#pragma unroll
                    for (int dir = 0; dir < 3; ++dir)
                      {
                        const int e1 = (dir + 1) % 3, e2 = (dir + 2) % 3;
                        // int v_dir (d phi / d x_dir) phi, v_dir = vel[dir] + sum_e G[dir][e] x_e
                        T term = a.vel[dir] * t[dir] * m[e1] * m[e2];
                        term += a.vel[3 + 3 * dir + dir] * tX[dir] * m[e1] * m[e2];
                        term += a.vel[3 + 3 * dir + e1] * t[dir] * mX[e1] * m[e2];
                        term += a.vel[3 + 3 * dir + e2] * t[dir] * m[e1] * mX[e2];
                        adv += term;
                      }
                    d += v + a.th_adv * adv;
                  }
            a.diag[idx] = d;
          }
      }
  }

  template <typename T>
  cudaError_t
  adv_diagonal(const GridDesc &g, int K, const AdvParams &p, T *diag, cudaStream_t s)
  {
    if (K < 1 || K > ADV_KMAX)
      return cudaErrorInvalidValue;
    AdvDiagArgs<T>   a{};
    const Tables1D &t = tables(K);
    const int       n = t.n;
    for (int i = 0; i < n; ++i)
      {
        double S = 0, S1 = 0, T0 = 0, T1 = 0, D = 0;
        for (int q = 0; q < n; ++q)
          {
            const double w = t.qw[q], b = t.B[q * n + i], gq = t.G[q * n + i];
            S += w * b * b;
            S1 += w * t.qp[q] * b * b;
            T0 += w * gq * b;
            T1 += w * t.qp[q] * gq * b;
            D += w * gq * gq;
          }
        a.S[i] = (T)S, a.S1[i] = (T)S1, a.T0[i] = (T)T0, a.T1[i] = (T)T1, a.D[i] = (T)D;
      }
    a.g      = g;
    a.inv_dt = (T)p.inv_dt;
    a.th_adv = (T)p.theta_adv;
    a.th_dif = (T)p.theta_dif;
    for (int i = 0; i < 12; ++i)
      a.vel[i] = (T)p.vel[i];
    for (int d = 0; d < 3; ++d)
      {
        a.origin[d] = (T)p.origin[d];
        a.h[d]      = (T)p.h[d];
      }
    a.diag                  = diag;
    const long long rows    = (long long)g.n[1] * g.n[2];
    const int       blocks  = (int)std::min<long long>(rows, 148LL * 32);
    const int       threads = std::min(1024, std::max(32, (g.n[0] + 31) / 32 * 32));
    if (K == 1)
      adv_diag_kernel<1, T><<<blocks, threads, 0, s>>>(a);
    else if (K == 2)
      adv_diag_kernel<2, T><<<blocks, threads, 0, s>>>(a);
    else
      adv_diag_kernel<3, T><<<blocks, threads, 0, s>>>(a);
    return cudaGetLastError();
  }

  // ---- SUPG part of the diagonal: one thread per cell; for each free local DoF i
  //   tau_c sum_q JxW (v.grad phi_i)(phi_i / dt + theta v.grad phi_i - theta eps lap phi_i)
  // with the 1-D values B, derivatives G and second derivatives H of the basis at the Gauss points.
  template <typename T>
  struct AdvSupgDiagArgs
  {
    GridDesc g;
    T        B[MAX_N * MAX_N], G[MAX_N * MAX_N], H[MAX_N * MAX_N], qp[MAX_N], qw[MAX_N];
    T        inv_dt, th_adv, th_dif, coef, cell_size, det;
    T        vel[12], origin[3], h[3];
    const double *f[3]; // DoF-vector velocity (FIELD kernels)
    T       *diag;
  };

  // FIELD: the velocity is a DoF vector, evaluated at the cell's Gauss points from its nodal values
  template <int K, typename T, bool FIELD>
  __global__ void
  adv_supg_diag_kernel(const __grid_constant__ AdvSupgDiagArgs<T> a)
  {
    constexpr int   N     = K + 1, N3 = N * N * N;
    const int       m0    = a.g.m[0], m1 = a.g.m[1];
    const long long ncell = (long long)m0 * m1 * a.g.m[2];
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x)
      {
        const int cx = (int)(c % m0), cy = (int)((c / m0) % m1), cz = (int)(c / ((long long)m0 * m1));
        const T   x0 = a.origin[0] + a.h[0] * cx, y0 = a.origin[1] + a.h[1] * cy, z0 = a.origin[2] + a.h[2] * cz;
        T         vq[FIELD ? 3 : 1][FIELD ? N3 : 1];
        T         tau;
        if constexpr (FIELD)
          {
#pragma unroll
            for (int d = 0; d < 3; ++d)
              field_at_points<T, N>(a.f[d], a.g, cx, cy, cz, a.B, vq[d]);
            tau = a.coef;
            if (tau < T(0))
              {
                T vmax = T(0);
#pragma unroll
                for (int q = 0; q < N3; ++q)
                  vmax = fmax(vmax, sqrt(vq[0][q] * vq[0][q] + vq[1][q] * vq[1][q] + vq[2][q] * vq[2][q]));
                tau = vmax >= T(1e-6) ? T(1) / vmax : T(0);
              }
            tau *= a.cell_size;
          }
        else
          tau = supg_tau<T, N>(a.vel, a.h, a.qp, x0, y0, z0, a.coef, a.cell_size);
        if (tau == T(0))
          continue;
        const T ih[3] = {T(1) / a.h[0], T(1) / a.h[1], T(1) / a.h[2]};
        for (int l = 0; l < N; ++l)
          for (int j = 0; j < N; ++j)
            for (int i = 0; i < N; ++i)
              {
                const int       I = K * cx + i, J = K * cy + j, L = K * cz + l;
                const long long idx = (long long)I + (long long)a.g.n[0] * ((long long)J + (long long)a.g.n[1] * L);
                if (is_constrained(a.g, I, J, L, idx))
                  continue;
                T sum = T(0);
                for (int qz = 0; qz < N; ++qz)
                  for (int qy = 0; qy < N; ++qy)
#pragma unroll
                    for (int qx = 0; qx < N; ++qx)
                      {
                        const T bx = a.B[qx * N + i], by = a.B[qy * N + j], bz = a.B[qz * N + l];
                        const T gx = a.G[qx * N + i] * ih[0], gy = a.G[qy * N + j] * ih[1], gz = a.G[qz * N + l] * ih[2];
                        const T hx = a.H[qx * N + i] * ih[0] * ih[0], hy = a.H[qy * N + j] * ih[1] * ih[1],
                                hz = a.H[qz * N + l] * ih[2] * ih[2];
                        const T phi = bx * by * bz;
                        const T dp[3] = {gx * by * bz, bx * gy * bz, bx * by * gz};
                        const T lap   = hx * by * bz + bx * hy * bz + bx * by * hz;
                        const T x = x0 + a.h[0] * a.qp[qx], y = y0 + a.h[1] * a.qp[qy], z = z0 + a.h[2] * a.qp[qz];
                        T       vg = T(0);
#pragma unroll
                        for (int d = 0; d < 3; ++d)
                          {
                            T vd;
                            if constexpr (FIELD)
                              vd = vq[d][(qz * N + qy) * N + qx];
                            else
                              vd = a.vel[d] + a.vel[3 + 3 * d] * x + a.vel[4 + 3 * d] * y + a.vel[5 + 3 * d] * z;
                            vg += vd * dp[d];
                          }
                        sum += a.qw[qx] * a.qw[qy] * a.qw[qz] * vg * (a.inv_dt * phi + a.th_adv * vg - a.th_dif * lap);
                      }
                atomicAdd(a.diag + idx, tau * a.det * sum);
              }
      }
  }

  template <typename T>
  cudaError_t
  adv_supg_diagonal(const GridDesc &g, int K, const AdvParams &p, T *diag, cudaStream_t s)
  {
    if (!p.supg)
      return cudaSuccess;
    if (K < 1 || K > ADV_KMAX)
      return cudaErrorInvalidValue;
    AdvSupgDiagArgs<T> a{};
    const Tables1D    &t = tables(K);
    const int          n = t.n;
    for (int q = 0; q < n; ++q)
      {
        a.qp[q] = (T)t.qp[q];
        a.qw[q] = (T)t.qw[q];
        for (int i = 0; i < n; ++i)
          {
            double hsum = 0.0; // second derivative: collocation derivative of G on the Gauss points
            for (int r = 0; r < n; ++r)
              hsum += t.Dq[q * n + r] * t.G[r * n + i];
            a.B[q * n + i] = (T)t.B[q * n + i];
            a.G[q * n + i] = (T)t.G[q * n + i];
            a.H[q * n + i] = (T)hsum;
          }
      }
    a.g         = g;
    a.inv_dt    = (T)p.inv_dt;
    a.th_adv    = (T)p.theta_adv;
    a.th_dif    = (T)p.theta_dif;
    a.coef      = (T)p.supg_coef;
    a.cell_size = (T)(std::sqrt(p.h[0] * p.h[0] + p.h[1] * p.h[1] + p.h[2] * p.h[2]) / std::sqrt(3.0));
    a.det       = (T)(p.h[0] * p.h[1] * p.h[2]);
    for (int i = 0; i < 12; ++i)
      a.vel[i] = (T)p.vel[i];
    for (int d = 0; d < 3; ++d)
      {
        a.origin[d] = (T)p.origin[d];
        a.h[d]      = (T)p.h[d];
      }
    a.diag                 = diag;
    for (int d = 0; d < 3; ++d)
      a.f[d] = p.vfield[d];
    const bool      field  = p.vfield[0] != nullptr;
    const long long ncell  = (long long)g.m[0] * g.m[1] * g.m[2];
    const int       blocks = (int)std::max<long long>(1, std::min<long long>((ncell + 127) / 128, 148LL * 16));
    if (K == 1)
      (field ? adv_supg_diag_kernel<1, T, true> : adv_supg_diag_kernel<1, T, false>)<<<blocks, 128, 0, s>>>(a);
    else if (K == 2)
      (field ? adv_supg_diag_kernel<2, T, true> : adv_supg_diag_kernel<2, T, false>)<<<blocks, 128, 0, s>>>(a);
    else
      (field ? adv_supg_diag_kernel<3, T, true> : adv_supg_diag_kernel<3, T, false>)<<<blocks, 128, 0, s>>>(a);
    return cudaGetLastError();
  }

  // ---- diagonal with a DoF-vector velocity: one thread per cell; the velocity at the Gauss points
  // from the cell's nodal values, then for each free local DoF i
  //   sum_q JxW (phi_i^2 / dt + theta_adv (v.grad phi_i) phi_i + theta_dif |grad phi_i|^2)
  // (MatrixFreeTools::compute_diagonal of the tangent, advection_diffusion_operator.cpp:399-446)
  struct AdvFieldDiagArgs
  {
    GridDesc      g;
    double        B[MAX_N * MAX_N], G[MAX_N * MAX_N], qw[MAX_N];
    double        inv_dt, th_adv, th_dif, det, h[3];
    const double *f[3];
    double       *diag;
  };

  template <int K>
  __global__ void
  adv_field_diag_kernel(const __grid_constant__ AdvFieldDiagArgs a)
  {
    constexpr int   N = K + 1, N3 = N * N * N;
    const int       m0 = a.g.m[0], m1 = a.g.m[1];
    const long long ncell = (long long)m0 * m1 * a.g.m[2];
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x)
      {
        const int cx = (int)(c % m0), cy = (int)((c / m0) % m1), cz = (int)(c / ((long long)m0 * m1));
        double    vq[3][N3];
#pragma unroll
        for (int d = 0; d < 3; ++d)
          field_at_points<double, N>(a.f[d], a.g, cx, cy, cz, a.B, vq[d]);
        const double ih[3] = {1.0 / a.h[0], 1.0 / a.h[1], 1.0 / a.h[2]};
        for (int l = 0; l < N; ++l)
          for (int j = 0; j < N; ++j)
            for (int i = 0; i < N; ++i)
              {
                const int       I = K * cx + i, J = K * cy + j, L = K * cz + l;
                const long long idx = (long long)I + (long long)a.g.n[0] * ((long long)J + (long long)a.g.n[1] * L);
                if (is_constrained(a.g, I, J, L, idx))
                  continue;
                double sum = 0.0;
                for (int qz = 0; qz < N; ++qz)
                  for (int qy = 0; qy < N; ++qy)
#pragma unroll
                    for (int qx = 0; qx < N; ++qx)
                      {
                        const int    q  = (qz * N + qy) * N + qx;
                        const double bx = a.B[qx * N + i], by = a.B[qy * N + j], bz = a.B[qz * N + l];
                        const double dp[3] = {a.G[qx * N + i] * ih[0] * by * bz, bx * a.G[qy * N + j] * ih[1] * bz,
                                              bx * by * a.G[qz * N + l] * ih[2]};
                        const double phi = bx * by * bz;
                        const double vg  = vq[0][q] * dp[0] + vq[1][q] * dp[1] + vq[2][q] * dp[2];
                        const double pp  = dp[0] * dp[0] + dp[1] * dp[1] + dp[2] * dp[2];
                        sum += a.qw[qx] * a.qw[qy] * a.qw[qz] * (a.inv_dt * phi * phi + a.th_adv * vg * phi + a.th_dif * pp);
                      }
                atomicAdd(a.diag + idx, a.det * sum);
              }
      }
  }

  cudaError_t
  adv_field_diagonal(const GridDesc &g, int K, const AdvParams &p, double *diag, cudaStream_t s)
  {
    if (K < 1 || K > ADV_KMAX || !p.vfield[0] || !p.vfield[1] || !p.vfield[2])
      return cudaErrorInvalidValue;
    AdvFieldDiagArgs a{};
    const Tables1D  &t = tables(K);
    const int        n = t.n;
    for (int q = 0; q < n; ++q)
      {
        a.qw[q] = t.qw[q];
        for (int i = 0; i < n; ++i)
          {
            a.B[q * n + i] = t.B[q * n + i];
            a.G[q * n + i] = t.G[q * n + i];
          }
      }
    a.g      = g;
    a.inv_dt = p.inv_dt;
    a.th_adv = p.theta_adv;
    a.th_dif = p.theta_dif;
    a.det    = p.h[0] * p.h[1] * p.h[2];
    for (int d = 0; d < 3; ++d)
      {
        a.h[d] = p.h[d];
        a.f[d] = p.vfield[d];
      }
    a.diag                 = diag;
    const long long ncell  = (long long)g.m[0] * g.m[1] * g.m[2];
    const int       blocks = (int)std::max<long long>(1, std::min<long long>((ncell + 127) / 128, 148LL * 16));
    if (K == 1)
      adv_field_diag_kernel<1><<<blocks, 128, 0, s>>>(a);
    else if (K == 2)
      adv_field_diag_kernel<2><<<blocks, 128, 0, s>>>(a);
    else
      adv_field_diag_kernel<3><<<blocks, 128, 0, s>>>(a);
    return cudaGetLastError();
  }

  template cudaError_t adv_supg_diagonal<double>(const GridDesc &, int, const AdvParams &, double *, cudaStream_t);
  template cudaError_t adv_supg_diagonal<float>(const GridDesc &, int, const AdvParams &, float *, cudaStream_t);
  template cudaError_t adv_apply<double>(const AdvLaunch<double> &, cudaStream_t);
  template cudaError_t adv_apply<float>(const AdvLaunch<float> &, cudaStream_t);
  template cudaError_t adv_diagonal<double>(const GridDesc &, int, const AdvParams &, double *, cudaStream_t);
  template cudaError_t adv_diagonal<float>(const GridDesc &, int, const AdvParams &, float *, cudaStream_t);
  template void adv_brick_shape<double>(int, int[3]);
  template void adv_brick_shape<float>(int, int[3]);
} // namespace mpdg
