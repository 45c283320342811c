// Heat operator with temperature-dependent material (solid / liquid phases), FE_Q(1, 2).
//
// Reference: source/heat/heat_diffuse_operator.cpp, tangent_local_cell_operation :1029-1050 with
// do_solidification (material of Material::compute_parameters, MaterialTypes::liquid_solid,
// include/meltpooldg/core/material.templates.hpp:296-360, :540-620, :748-765):
//   tangent   val  = (rho c_p(T) / dt + d(rho c_p)/dT (T - T_old) / dt) u
//             grad = k(T) grad u + dk/dT grad T u
//   residual  (rhs_cell_loop :485-527)  val = rho c_p(T) (T - T_old) / dt,  grad = k(T) grad T,
//             submitted with a minus sign (the heat source enters through the mass apply)
// T and T_old are read plainly (read_dof_values_plain), u with constraints.  Solid fraction
// f_s = clamp((T_liquidus - T) / (T_liquidus - T_solidus), 0, 1) (mushy zone) or T < T_solidus
// (sharp); a property is the cubic blend v_l + (v_s - v_l)(3 f_s^2 - 2 f_s^3) (f_s = 0 / 1 give
// v_l / v_s), its temperature derivative -(v_s - v_l)(6 f_s - 6 f_s^2) / (T_liquidus - T_solidus)
// (0 at f_s = 0 or 1).  No latent heat (apparent capacity).
//
// Per cell (one thread), quadrature form in registers: the values of u, T and T_old at the Gauss
// points (three sweeps of the 1-D basis each), the mass-like term pointwise, then Gauss point by
// Gauss point the conductivity (once), the three gradients by the collocation derivative and the
// flux tested with its transpose, and the transposed basis sweeps back to the nodes; cells add into
// the brick accumulator in shared memory and the brick is written as in the other brick kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "brick.cuh"
#include "kernels.h"

#ifndef MPDG_SOLID_MINB_F64
#define MPDG_SOLID_MINB_F64 2
#endif
#ifndef MPDG_SOLID_MINB_F32
#define MPDG_SOLID_MINB_F32 4
#endif

namespace mpdg
{
  namespace
  {
    template <typename T>
    struct SolidMat
    {
      T   rho_l, cp_l, k_l, rho_s, cp_s, k_s, t_liquidus, t_solidus, inv_mushy;
      int sharp;
      T   latent;   // latent heat of fusion (0: none)
      int cap_type; // apparent capacity: 0 quadratic-linear-quadratic, 1 quartic bell, 2 constant
    };

    // Ramp from (x1, y1) to (x2, y2) with zero slope at both ends: quadratic on [x1, x1 + delta],
    // linear in between, quadratic on [x2 - delta, x2] (value and slope continuous).
    template <typename T>
    __device__ __forceinline__ void
    zero_slope_ramp(T x, T x1, T x2, T y1, T y2, T delta, T &val, T &der)
    {
      const T s = (y2 - y1) / (x2 - x1 - delta);
      if (x < x1 + delta)
        {
          val = y1 + T(0.5) * s * (x - x1) * (x - x1) / delta;
          der = s * (x - x1) / delta;
        }
      else if (x > x2 - delta)
        {
          val = y2 - T(0.5) * s * (x2 - x) * (x2 - x) / delta;
          der = s * (x2 - x) / delta;
        }
      else
        {
          val = y1 + s * (x - x1 - T(0.5) * delta);
          der = s;
        }
    }

    // Apparent specific heat of the latent heat and its temperature derivative at solid fraction fs
    // (include/meltpooldg/core/material.templates.hpp:561-614, source/heat/apparent_capacity.cpp:
    // 157-300): zero outside the mushy zone, each shape integrating to L over [T_solidus, T_liquidus]:
    // constant L / dT; quartic bell L (2 / dT) 15/16 (1 - x^2)^2 with x = 1 - 2 fs; the default tent of
    // peak 2 L / dT at the mid temperature with flat-ended flanks of width dT / 6, evaluated at
    // T = T_liquidus - fs dT.
    template <typename T>
    __device__ __forceinline__ void
    apparent_capacity(const SolidMat<T> &m, T fs, T &c, T &dc)
    {
      c = dc = T(0);
      if (!(m.latent > T(0)) || !(fs > T(0)) || !(fs < T(1)))
        return;
      const T L = m.latent, dT = m.t_liquidus - m.t_solidus;
      if (m.cap_type == 2)
        c = L / dT;
      else if (m.cap_type == 1)
        {
          const T r = T(2) / dT, x = T(1) - T(2) * fs;
          c         = L * r * T(15.0 / 16.0) * (T(1) - x * x) * (T(1) - x * x);
          dc        = L * r * r * T(15.0 / 4.0) * (x * x - T(1)) * x;
        }
      else
        {
          const T t = m.t_liquidus - fs * dT, tp = T(0.5) * (m.t_solidus + m.t_liquidus);
          const T peak = T(2) * L / dT, delta = dT / T(6);
          if (t <= tp)
            zero_slope_ramp(t, m.t_solidus, tp, T(0), peak, delta, c, dc);
          else
            zero_slope_ramp(t, tp, m.t_liquidus, peak, T(0), delta, c, dc);
        }
    }

    // solid fraction, cubic blend weight and its temperature derivative at temperature t
    template <typename T>
    __device__ __forceinline__ void
    solid_fraction(const SolidMat<T> &m, T t, T &fs, T &w, T &dw)
    {
      if (m.sharp)
        fs = t < m.t_solidus ? T(1) : T(0);
      else
        fs = fmin(fmax((m.t_liquidus - t) * m.inv_mushy, T(0)), T(1));
      w  = (T(3) - T(2) * fs) * fs * fs;
      dw = (fs == T(0) || fs == T(1)) ? T(0) : -m.inv_mushy * (T(6) * fs - T(6) * fs * fs);
    }
    template <typename T>
    __device__ __forceinline__ T
    solid_blend(T fs, T w, T vl, T vs)
    {
      return fs == T(0) ? vl : (fs == T(1) ? vs : vl + (vs - vl) * w);
    }
    // k and dk/dT at temperature t
    template <typename T>
    __device__ __forceinline__ void
    solid_conductivity(const SolidMat<T> &m, T t, T &k, T &dk)
    {
      T fs, w, dw;
      solid_fraction(m, t, fs, w, dw);
      k  = solid_blend(fs, w, m.k_l, m.k_s);
      dk = (m.k_s - m.k_l) * dw;
    }

    // rho c_p, k and their temperature derivatives at temperature t
    template <typename T>
    __device__ __forceinline__ void
    solid_material(const SolidMat<T> &m, T t, T &rc, T &k, T &drc, T &dk)
    {
      T fs;
      if (m.sharp)
        fs = t < m.t_solidus ? T(1) : T(0);
      else
        fs = fmin(fmax((m.t_liquidus - t) * m.inv_mushy, T(0)), T(1));
      const bool end = fs == T(0) || fs == T(1);
      const T    w   = (T(3) - T(2) * fs) * fs * fs, dw = -m.inv_mushy * (T(6) * fs - T(6) * fs * fs);
      auto       pr  = [&](T vl, T vs) { return fs == T(0) ? vl : (fs == T(1) ? vs : vl + (vs - vl) * w); };
      auto       dpr = [&](T vl, T vs) { return end ? T(0) : (vs - vl) * dw; };
      T          ca, dca;
      apparent_capacity(m, fs, ca, dca);
      const T rho = pr(m.rho_l, m.rho_s), cp = pr(m.cp_l, m.cp_s) + ca;
      rc          = rho * cp;
      k           = pr(m.k_l, m.k_s);
      drc         = dpr(m.rho_l, m.rho_s) * cp + rho * (dpr(m.cp_l, m.cp_s) + dca);
      dk          = dpr(m.k_l, m.k_s);
    }

    template <typename T, int N>
    struct SolidArgs
    {
      GridDesc    g;
      SyncDesc    s;
      SolidMat<T> m;
      T           det, inv_dt, h[3];
      T           B[N * N], D[N * N], w3[N * N * N];
      const T    *src;
      const T    *temp, *temp_old;
      T          *dst;
      const T    *b;
      int         mask_src, rhs;
      const int  *skip;
    };

    template <int K, typename T>
    struct SolidLayout
    {
      static constexpr int BX = 8, BY = 8, BZ = (K == 1 ? 8 : (K == 2 ? 4 : 2));
      static constexpr int NT = BX * BY * BZ;
      using BR                = Brick<K, BX, BY, BZ, NT>;
      static constexpr size_t bytes = sizeof(T) * 4 * (size_t)BR::NPTS; // u, T, T_old, accumulator
      // CTAs per SM (k = 3: 128-thread CTAs, 140 KB of staging in FP64, one per SM)
      static constexpr int    MINB  = K == 3 ? 1 : (sizeof(T) == 8 ? MPDG_SOLID_MINB_F64 : MPDG_SOLID_MINB_F32);
    };

    // v = M v along direction D of an N^3 array (TR: M^T)
    template <typename T, int N, int D, bool TR>
    __device__ __forceinline__ void
    solid_sweep(T *v, const T *M)
    {
      constexpr int S = D == 0 ? 1 : (D == 1 ? N : N * N);
#pragma unroll
      for (int a = 0; a < N; ++a)
#pragma unroll
        for (int c = 0; c < N; ++c)
          {
            const int base = D == 0 ? (a * N + c) * N : (D == 1 ? a * N * N + c : a * N + c);
            T         in[N];
#pragma unroll
            for (int k = 0; k < N; ++k)
              in[k] = v[base + k * S];
#pragma unroll
            for (int r = 0; r < N; ++r)
              {
                T s = T(0);
#pragma unroll
                for (int k = 0; k < N; ++k)
                  s = fma(TR ? M[k * N + r] : M[r * N + k], in[k], s);
                v[base + r * S] = s;
              }
          }
    }

    template <int K, typename T, OutMode MODE, bool RHS>
    __global__ void __launch_bounds__(SolidLayout<K, T>::NT, SolidLayout<K, T>::MINB)
    heat_solid_kernel(const __grid_constant__ SolidArgs<T, K + 1> a)
    {
      using LAY            = SolidLayout<K, T>;
      using BR             = typename LAY::BR;
      constexpr int N      = K + 1, NP = BR::NPTS, PX = BR::PX, PY = BR::PY;
      constexpr int BX     = BR::BX, BY = BR::BY;
      extern __shared__ __align__(16) unsigned char smem_raw[];
      T *const s_u   = reinterpret_cast<T *>(smem_raw);
      T *const s_t   = s_u + NP;
      T *const s_to  = s_t + NP;
      T *const s_dst = s_to + NP;
      __shared__ unsigned s_ticket;
      if (a.skip != nullptr && *a.skip != 0)
        return;
      BR br;
      if (!brick_begin<BR, T, MODE>(br, a.g, a.s, a.dst, a.b, &s_ticket))
        return;
      for (int p = threadIdx.x; p < NP; p += BR::NT)
        s_dst[p] = T(0);
      if constexpr (!RHS)
        brick_stage(br, a.src, a.mask_src != 0, s_u);
      brick_stage(br, a.temp, false, s_t);
      brick_stage(br, a.temp_old, false, s_to);

      const int  tx = threadIdx.x % BX, ty = (threadIdx.x / BX) % BY, tz = threadIdx.x / (BX * BY);
      const int  cx = br.c0[0] + tx, cy = br.c0[1] + ty, cz = br.c0[2] + tz;
      const bool valid = cx < a.g.m[0] && cy < a.g.m[1] && cz < a.g.m[2];
      const int  base  = (K * tz) * PY * PX + (K * ty) * PX + K * tx;
      if (valid)
        {
          T tq[N * N * N], R[N * N * N], uq[N * N * N];
#pragma unroll
          for (int l = 0; l < N; ++l)
#pragma unroll
            for (int j = 0; j < N; ++j)
#pragma unroll
              for (int i = 0; i < N; ++i)
                {
                  const int o = base + l * PY * PX + j * PX + i, q = (l * N + j) * N + i;
                  tq[q]       = s_t[o];
                  R[q]        = s_to[o];
                  if constexpr (!RHS)
                    uq[q] = s_u[o];
                }
          solid_sweep<T, N, 0, false>(tq, a.B);
          solid_sweep<T, N, 1, false>(tq, a.B);
          solid_sweep<T, N, 2, false>(tq, a.B);
          solid_sweep<T, N, 0, false>(R, a.B);
          solid_sweep<T, N, 1, false>(R, a.B);
          solid_sweep<T, N, 2, false>(R, a.B);
          if constexpr (!RHS)
            {
              solid_sweep<T, N, 0, false>(uq, a.B);
              solid_sweep<T, N, 1, false>(uq, a.B);
              solid_sweep<T, N, 2, false>(uq, a.B);
            }
          // mass-like term (R holds T_old at the Gauss points until here)
#pragma unroll
          for (int q = 0; q < N * N * N; ++q)
            {
              T rc, k, drc, dk;
              solid_material(a.m, tq[q], rc, k, drc, dk);
              const T jw = a.det * a.w3[q] * a.inv_dt;
              if constexpr (RHS)
                R[q] = -jw * rc * (tq[q] - R[q]);
              else
                R[q] = jw * (rc + drc * (tq[q] - R[q])) * uq[q];
            }
          // fluxes point by point: the conductivity once per Gauss point, the three gradients by
          // the collocation derivative along each direction, the test by its transpose
          const T ih2[3] = {T(1) / (a.h[0] * a.h[0]), T(1) / (a.h[1] * a.h[1]), T(1) / (a.h[2] * a.h[2])};
#pragma unroll
          for (int qz = 0; qz < N; ++qz)
#pragma unroll
            for (int qy = 0; qy < N; ++qy)
#pragma unroll
              for (int qx = 0; qx < N; ++qx)
                {
                  const int q = (qz * N + qy) * N + qx;
                  T         gt[3] = {T(0), T(0), T(0)}, gu[3] = {T(0), T(0), T(0)};
#pragma unroll
                  for (int k = 0; k < N; ++k)
                    {
                      const int qk[3] = {(qz * N + qy) * N + k, (qz * N + k) * N + qx, (k * N + qy) * N + qx};
                      const T   dd[3] = {a.D[qx * N + k], a.D[qy * N + k], a.D[qz * N + k]};
#pragma unroll
                      for (int d = 0; d < 3; ++d)
                        {
                          gt[d] = fma(dd[d], tq[qk[d]], gt[d]);
                          if constexpr (!RHS)
                            gu[d] = fma(dd[d], uq[qk[d]], gu[d]);
                        }
                    }
                  T k, dk;
                  solid_conductivity(a.m, tq[q], k, dk);
                  const T jw = a.det * a.w3[q];
                  T       f[3];
#pragma unroll
                  for (int d = 0; d < 3; ++d)
                    f[d] = RHS ? -jw * ih2[d] * k * gt[d] : jw * ih2[d] * (k * gu[d] + dk * gt[d] * uq[q]);
#pragma unroll
                  for (int k2 = 0; k2 < N; ++k2)
                    {
                      R[(qz * N + qy) * N + k2] = fma(a.D[qx * N + k2], f[0], R[(qz * N + qy) * N + k2]);
                      R[(qz * N + k2) * N + qx] = fma(a.D[qy * N + k2], f[1], R[(qz * N + k2) * N + qx]);
                      R[(k2 * N + qy) * N + qx] = fma(a.D[qz * N + k2], f[2], R[(k2 * N + qy) * N + qx]);
                    }
                }
          solid_sweep<T, N, 2, true>(R, a.B);
          solid_sweep<T, N, 1, true>(R, a.B);
          solid_sweep<T, N, 0, true>(R, a.B);
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

    // ---- diagonal of the tangent: one thread per cell; for each Gauss point the values of T,
    // grad T and T_old, then every free local DoF's entry
    //   sum_q JxW [(rho c_p / dt + d(rho c_p)/dT (T - T_old) / dt) phi_i^2 + k |grad phi_i|^2
    //              + dk/dT (grad T . grad phi_i) phi_i]
    template <typename T, int N>
    struct SolidDiagArgs
    {
      GridDesc      g;
      SolidMat<T>   m;
      T             det, inv_dt, h[3];
      T             B[N * N], G[N * N], w[N];
      const double *temp, *temp_old;
      double       *diag;
    };

    template <int K, typename T>
    __global__ void __launch_bounds__(128)
    heat_solid_diag_kernel(const __grid_constant__ SolidDiagArgs<T, K + 1> a)
    {
      constexpr int   N     = K + 1;
      const int       m0    = a.g.m[0], m1 = a.g.m[1];
      const long long ncell = (long long)m0 * m1 * a.g.m[2];
      for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x)
        {
          const int cx = (int)(c % m0), cy = (int)((c / m0) % m1), cz = (int)(c / ((long long)m0 * m1));
          T         tn[N * N * N], ton[N * N * N], d[N * N * N];
          long long idx[N * N * N];
#pragma unroll
          for (int l = 0; l < N; ++l)
#pragma unroll
            for (int j = 0; j < N; ++j)
#pragma unroll
              for (int i = 0; i < N; ++i)
                {
                  const int       q  = (l * N + j) * N + i;
                  const int       I = K * cx + i, J = K * cy + j, L = K * cz + l;
                  const long long id = (long long)I + (long long)a.g.n[0] * ((long long)J + (long long)a.g.n[1] * L);
                  idx[q]             = is_constrained(a.g, I, J, L, id) ? -1 : id;
                  tn[q]              = (T)a.temp[id];
                  ton[q]             = (T)a.temp_old[id];
                  d[q]               = T(0);
                }
          const T ih[3] = {T(1) / a.h[0], T(1) / a.h[1], T(1) / a.h[2]};
          for (int qz = 0; qz < N; ++qz)
            for (int qy = 0; qy < N; ++qy)
              for (int qx = 0; qx < N; ++qx)
                {
                  T tv = T(0), to = T(0), g0 = T(0), g1 = T(0), g2 = T(0);
#pragma unroll
                  for (int l = 0; l < N; ++l)
#pragma unroll
                    for (int j = 0; j < N; ++j)
#pragma unroll
                      for (int i = 0; i < N; ++i)
                        {
                          const int q   = (l * N + j) * N + i;
                          const T   bx = a.B[qx * N + i], by = a.B[qy * N + j], bz = a.B[qz * N + l];
                          const T   gx = a.G[qx * N + i], gy = a.G[qy * N + j], gz = a.G[qz * N + l];
                          tv += bx * by * bz * tn[q];
                          to += bx * by * bz * ton[q];
                          g0 += gx * by * bz * tn[q];
                          g1 += bx * gy * bz * tn[q];
                          g2 += bx * by * gz * tn[q];
                        }
                  g0 *= ih[0], g1 *= ih[1], g2 *= ih[2];
                  T rc, k, drc, dk;
                  solid_material(a.m, tv, rc, k, drc, dk);
                  const T jw = a.det * a.w[qx] * a.w[qy] * a.w[qz];
                  const T cm = (rc + drc * (tv - to)) * a.inv_dt;
#pragma unroll
                  for (int l = 0; l < N; ++l)
#pragma unroll
                    for (int j = 0; j < N; ++j)
#pragma unroll
                      for (int i = 0; i < N; ++i)
                        {
                          const T bx = a.B[qx * N + i], by = a.B[qy * N + j], bz = a.B[qz * N + l];
                          const T px = a.G[qx * N + i] * ih[0] * by * bz, py = bx * a.G[qy * N + j] * ih[1] * bz,
                                  pz  = bx * by * a.G[qz * N + l] * ih[2];
                          const T phi = bx * by * bz;
                          d[(l * N + j) * N + i] += jw * (cm * phi * phi + k * (px * px + py * py + pz * pz) +
                                                          dk * (g0 * px + g1 * py + g2 * pz) * phi);
                        }
                }
#pragma unroll
          for (int q = 0; q < N * N * N; ++q)
            if (idx[q] >= 0)
              atomicAdd(a.diag + idx[q], (double)d[q]);
        }
    }

    template <typename T>
    SolidMat<T>
    solid_mat(const SolidMaterial &m)
    {
      SolidMat<T> s;
      s.rho_l = (T)m.rho_l, s.cp_l = (T)m.cp_l, s.k_l = (T)m.k_l;
      s.rho_s = (T)m.rho_s, s.cp_s = (T)m.cp_s, s.k_s = (T)m.k_s;
      s.t_liquidus = (T)m.t_liquidus, s.t_solidus = (T)m.t_solidus;
      s.inv_mushy  = m.t_liquidus > m.t_solidus ? (T)(1.0 / (m.t_liquidus - m.t_solidus)) : T(0);
      s.sharp      = m.sharp;
      s.latent     = (T)m.latent_heat;
      s.cap_type   = m.capacity_type;
      return s;
    }

    template <int K, typename T, OutMode MODE, bool RHS>
    cudaError_t
    launch_solid(const HeatSolidLaunch<T> &h, cudaStream_t stream)
    {
      constexpr int    N = K + 1;
      using LAY          = SolidLayout<K, T>;
      SolidArgs<T, N> a{};
      a.g      = h.grid;
      a.s      = h.sync;
      a.m      = solid_mat<T>(h.mat);
      a.det    = (T)(h.scale * h.hlen[0] * h.hlen[1] * h.hlen[2]);
      a.inv_dt = (T)(1.0 / h.dt);
      for (int d = 0; d < 3; ++d)
        a.h[d] = (T)h.hlen[d];
      const Tables1D &t = tables(K);
      for (int i = 0; i < N * N; ++i)
        {
          a.B[i] = (T)t.B[i];
          a.D[i] = (T)t.Dq[i];
        }
      for (int qz = 0; qz < N; ++qz)
        for (int qy = 0; qy < N; ++qy)
          for (int qx = 0; qx < N; ++qx)
            a.w3[(qz * N + qy) * N + qx] = (T)(t.qw[qx] * t.qw[qy] * t.qw[qz]);
      a.src      = h.src;
      a.temp     = h.temp;
      a.temp_old = h.temp_old;
      a.dst      = h.dst;
      a.b        = h.b;
      a.mask_src = h.mask_src;
      a.rhs      = RHS ? 1 : 0;
      a.skip     = h.skip;
      auto                                   kern = heat_solid_kernel<K, T, MODE, RHS>;
      static std::atomic<unsigned long long> devices{0};
      if (cudaError_t e = ensure_smem(kern, LAY::bytes, devices); e != cudaSuccess)
        return e;
      const unsigned nbricks = (unsigned)h.grid.nbr[0] * h.grid.nbr[1] * h.grid.nbr[2];
      kern<<<nbricks, LAY::BR::NT, LAY::bytes, stream>>>(a);
      return cudaGetLastError();
    }

    template <int K, typename T>
    cudaError_t
    solid_mode(const HeatSolidLaunch<T> &h, cudaStream_t s)
    {
      if (h.rhs)
        return launch_solid<K, T, OutMode::Add, true>(h, s);
      switch (h.mode)
        {
          case 0: return launch_solid<K, T, OutMode::Set, false>(h, s);
          case 1: return launch_solid<K, T, OutMode::Add, false>(h, s);
          default: return launch_solid<K, T, OutMode::BPlus, false>(h, s);
        }
    }
  } // namespace

  template <typename T>
  void
  heat_solid_brick_shape(int K, int shape[3])
  {
    shape[0] = 8;
    shape[1] = 8;
    shape[2] = K == 1 ? SolidLayout<1, T>::BZ : (K == 2 ? SolidLayout<2, T>::BZ : SolidLayout<3, T>::BZ);
  }

  template <typename T>
  cudaError_t
  heat_solid_apply(const HeatSolidLaunch<T> &h, cudaStream_t s)
  {
    switch (h.degree)
      {
        case 1: return solid_mode<1, T>(h, s);
        case 2: return solid_mode<2, T>(h, s);
        case 3: return solid_mode<3, T>(h, s);
        default: return cudaErrorInvalidValue;
      }
  }

  cudaError_t
  heat_solid_diagonal(const GridDesc &g, int K, const SolidMaterial &mat, double dt, const double hlen[3],
                      const double *temp, const double *temp_old, double *diag, cudaStream_t s)
  {
    if (K < 1 || K > 3)
      return cudaErrorInvalidValue;
    const Tables1D &t      = tables(K);
    const long long ncell  = (long long)g.m[0] * g.m[1] * g.m[2];
    const int       blocks = (int)std::max<long long>(1, std::min<long long>((ncell + 127) / 128, 148LL * 16));
    auto            fill   = [&](auto &a, int n) {
      a.g      = g;
      a.m      = solid_mat<double>(mat);
      a.det    = hlen[0] * hlen[1] * hlen[2];
      a.inv_dt = 1.0 / dt;
      for (int d = 0; d < 3; ++d)
        a.h[d] = hlen[d];
      for (int i = 0; i < n * n; ++i)
        {
          a.B[i] = t.B[i];
          a.G[i] = t.G[i];
        }
      for (int q = 0; q < n; ++q)
        a.w[q] = t.qw[q];
      a.temp     = temp;
      a.temp_old = temp_old;
      a.diag     = diag;
    };
    if (K == 1)
      {
        SolidDiagArgs<double, 2> a{};
        fill(a, 2);
        heat_solid_diag_kernel<1, double><<<blocks, 128, 0, s>>>(a);
      }
    else if (K == 2)
      {
        SolidDiagArgs<double, 3> a{};
        fill(a, 3);
        heat_solid_diag_kernel<2, double><<<blocks, 128, 0, s>>>(a);
      }
    else
      {
        SolidDiagArgs<double, 4> a{};
        fill(a, 4);
        heat_solid_diag_kernel<3, double><<<blocks, 128, 0, s>>>(a);
      }
    return cudaGetLastError();
  }

  template cudaError_t heat_solid_apply<double>(const HeatSolidLaunch<double> &, cudaStream_t);
  template cudaError_t heat_solid_apply<float>(const HeatSolidLaunch<float> &, cudaStream_t);
  template void        heat_solid_brick_shape<double>(int, int[3]);
  template void        heat_solid_brick_shape<float>(int, int[3]);
} // namespace mpdg
