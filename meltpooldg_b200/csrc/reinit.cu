// Conservative level-set reinitialisation operator (Olsson), FE_Q(1..3).
//
// Reference: source/level_set/olsson_CG_operator.cpp, default configuration (no wetting boundary
// faces, no interface penalty):
//   tangent  (:438-470)  val = dpsi / dt,  grad = eps_n (grad dpsi . n) n + eps_t (grad dpsi - (grad dpsi . n) n)
//   rhs      (:197-260)  dst = int [c(psi) n - eps_n (grad psi . n) n - eps_t (grad psi - (grad psi . n) n)] . grad phi,
//                        c(psi) = (1 - psi^2) / 2 (:24-29), dst overwritten, constrained rows 0
// with the unit normal n = normalize(n_h(x_q), tol) of the normal field n_h (three FE_Q components
// on the same lattice, read plainly; normalize divides by |n_h| above tol and by tol otherwise,
// include/meltpooldg/utilities/dealii_tensor.hpp:175-191).  The reference caches n at the Gauss
// points while it assembles the rhs and reuses the cache in vmult; here it is evaluated from the
// normal field at every apply (the same as long as the field does not change in between).
//
// One thread per cell, point-wise quadrature: at each Gauss point the value and gradient of the
// input and the normal field come from the cell's nodal values (tensor products of the 1-D basis
// values and derivatives), and the integrand is tested against every nodal basis function; cells
// add into dst with atomics (dst is prepared by the host: zero, or b for b + A x).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "brick.cuh"
#include "kernels.h"

namespace mpdg
{
  namespace
  {
    template <typename T, int N>
    struct ReinitArgs
    {
      GridDesc      g;
      T             scale, inv_dt, eps_n, eps_t, tol, det, ih[3];
      T             B[N * N], G[N * N], w[N];
      const T      *src;
      const double *n[3];
      T            *dst;
      double       *diag;
      int           mode; // 0 tangent apply, 1 rhs (src = psi_old, plain), 2 diagonal
      int           mask_src;
      const double *band_ls; // narrow band (include/meltpooldg/level_set/level_set_tools.hpp:357-368)
      T             band;
      unsigned      wetting; // wetting boundary faces (bit 2d low / 2d+1 high face of dim d)
      T             Vend[2 * N], Dend[2 * N]; // basis values / derivatives at x = 0 and x = 1
    };

    template <int K, typename T>
    __global__ void __launch_bounds__(128)
    reinit_kernel(const __grid_constant__ ReinitArgs<T, K + 1> a)
    {
      constexpr int   N     = K + 1, N3 = N * N * N;
      const int       m0    = a.g.m[0], m1 = a.g.m[1];
      const long long ncell = (long long)m0 * m1 * a.g.m[2];
      for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x)
        {
          const int cx = (int)(c % m0), cy = (int)((c / m0) % m1), cz = (int)(c / ((long long)m0 * m1));
          long long idx[N3];
          bool      con[N3];
          T         u[N3], R[N3], ls[N3];
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
                  idx[q]             = id;
                  con[q]             = is_constrained(a.g, I, J, L, id);
                  u[q]               = (a.mode == 2 || (a.mask_src && con[q])) ? T(0) : a.src[id];
                  R[q]               = T(0);
                  ls[q]              = a.band_ls ? (T)a.band_ls[id] : T(0); // read plainly
                }
          for (int qz = 0; qz < N; ++qz)
            for (int qy = 0; qy < N; ++qy)
              for (int qx = 0; qx < N; ++qx)
                {
                  // value and gradient of u and the normal field at the Gauss point
                  // (the isotropic form, eps_n == eps_t, has no normal field: n == nullptr)
                  T uv = T(0), g[3] = {T(0), T(0), T(0)}, nv[3] = {T(0), T(0), T(0)}, lq = T(0);
                  const bool has_n = a.n[0] != nullptr;
#pragma unroll
                  for (int l = 0; l < N; ++l)
#pragma unroll
                    for (int j = 0; j < N; ++j)
#pragma unroll
                      for (int i = 0; i < N; ++i)
                        {
                          const int q   = (l * N + j) * N + i;
                          const T   bx = a.B[qx * N + i], by = a.B[qy * N + j], bz = a.B[qz * N + l];
                          const T   phi = bx * by * bz;
                          uv += phi * u[q];
                          lq += phi * ls[q];
                          g[0] += a.G[qx * N + i] * by * bz * u[q];
                          g[1] += bx * a.G[qy * N + j] * bz * u[q];
                          g[2] += bx * by * a.G[qz * N + l] * u[q];
                          if (has_n)
#pragma unroll
                            for (int d = 0; d < 3; ++d)
                              nv[d] += phi * (T)a.n[d][idx[q]];
                        }
#pragma unroll
                  for (int d = 0; d < 3; ++d)
                    g[d] *= a.ih[d];
                  if (has_n)
                    {
                      const T nn  = sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
                      const T inv = nn > a.tol ? T(1) / nn : T(1) / a.tol;
#pragma unroll
                      for (int d = 0; d < 3; ++d)
                        nv[d] *= inv;
                    }
                  // narrow band: the point contributes only where |level set| < band
                  const T jw = (a.band_ls && !(fabs(lq) < a.band)) ? T(0) : a.det * a.w[qx] * a.w[qy] * a.w[qz];
                  if (a.mode == 2)
                    {
                      // diagonal: int phi_i^2 / dt + grad phi_i . D grad phi_i
#pragma unroll
                      for (int l = 0; l < N; ++l)
#pragma unroll
                        for (int j = 0; j < N; ++j)
#pragma unroll
                          for (int i = 0; i < N; ++i)
                            {
                              const T bx = a.B[qx * N + i], by = a.B[qy * N + j], bz = a.B[qz * N + l];
                              const T p[3] = {a.G[qx * N + i] * a.ih[0] * by * bz, bx * a.G[qy * N + j] * a.ih[1] * bz,
                                              bx * by * a.G[qz * N + l] * a.ih[2]};
                              const T phi = bx * by * bz;
                              const T pn  = p[0] * nv[0] + p[1] * nv[1] + p[2] * nv[2];
                              const T pp  = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
                              R[(l * N + j) * N + i] += jw * (a.inv_dt * phi * phi + a.eps_t * pp + (a.eps_n - a.eps_t) * pn * pn);
                            }
                      continue;
                    }
                  // integrand: value part and gradient part (flux)
                  const T gn = g[0] * nv[0] + g[1] * nv[1] + g[2] * nv[2];
                  T       val, f[3];
                  if (a.mode == 0)
                    {
                      val = jw * a.inv_dt * uv;
#pragma unroll
                      for (int d = 0; d < 3; ++d)
                        f[d] = jw * (a.eps_t * g[d] + (a.eps_n - a.eps_t) * gn * nv[d]);
                    }
                  else
                    {
                      val            = T(0);
                      const T cflux = T(0.5) * (T(1) - uv * uv);
#pragma unroll
                      for (int d = 0; d < 3; ++d)
                        f[d] = jw * (cflux * nv[d] - a.eps_t * g[d] - (a.eps_n - a.eps_t) * gn * nv[d]);
                    }
#pragma unroll
                  for (int l = 0; l < N; ++l)
#pragma unroll
                    for (int j = 0; j < N; ++j)
#pragma unroll
                      for (int i = 0; i < N; ++i)
                        {
                          const T bx = a.B[qx * N + i], by = a.B[qy * N + j], bz = a.B[qz * N + l];
                          R[(l * N + j) * N + i] += val * bx * by * bz + f[0] * a.G[qx * N + i] * a.ih[0] * by * bz +
                                                    f[1] * bx * a.G[qy * N + j] * a.ih[1] * bz +
                                                    f[2] * bx * by * a.G[qz * N + l] * a.ih[2];
                        }
                }
#pragma unroll
          for (int q = 0; q < N3; ++q)
            if (!con[q])
              {
                if (a.mode == 2)
                  atomicAdd(a.diag + idx[q], (double)R[q]);
                else
                  atomicAdd(a.dst + idx[q], a.scale * R[q]);
              }
        }
    }

    // Wetting boundary faces of the reinitialisation operator (olsson_CG_operator.cpp:550-716), one
    // thread per boundary cell face: at the face's Gauss points the flux D grad u . n_f with
    // D = eps_n n n^T + eps_t (I - n n^T) (tangent, src read with constraints; diagonal: per basis
    // function), or -(-c(psi) n + D grad psi) . n_f with c(psi) = (1 - psi^2) / 2 (rhs, plain reads),
    // tested with the basis values on the face.
    template <int K, typename T>
    __global__ void __launch_bounds__(128)
    wetting_kernel(const __grid_constant__ ReinitArgs<T, K + 1> a)
    {
      constexpr int N = K + 1, N3 = N * N * N;
      const int     m[3] = {a.g.m[0], a.g.m[1], a.g.m[2]};
      long long     count[6], total = 0;
      for (int f = 0; f < 6; ++f)
        {
          const int d = f >> 1;
          count[f]    = ((a.wetting >> f) & 1u) ? (long long)m[(d + 1) % 3] * m[(d + 2) % 3] : 0;
          total += count[f];
        }
      const T hl[3] = {T(1) / a.ih[0], T(1) / a.ih[1], T(1) / a.ih[2]};
      for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x)
        {
          int       f = 0;
          long long r = t;
          while (r >= count[f])
            r -= count[f++];
          const int d = f >> 1, side = f & 1, ea = (d + 1) % 3, eb = (d + 2) % 3;
          int       c[3];
          c[d]  = side ? m[d] - 1 : 0;
          c[ea] = (int)(r % m[ea]);
          c[eb] = (int)(r / m[ea]);
          long long idx[N3];
          bool      con[N3];
          T         u[N3], R[N3], nn[3][N3];
#pragma unroll
          for (int l = 0; l < N; ++l)
#pragma unroll
            for (int j = 0; j < N; ++j)
#pragma unroll
              for (int i = 0; i < N; ++i)
                {
                  const int       q = (l * N + j) * N + i;
                  const int       I = K * c[0] + i, J = K * c[1] + j, L = K * c[2] + l;
                  const long long id = (long long)I + (long long)a.g.n[0] * ((long long)J + (long long)a.g.n[1] * L);
                  idx[q]            = id;
                  con[q]            = is_constrained(a.g, I, J, L, id);
                  u[q]              = (a.mode == 2 || (a.mode == 0 && a.mask_src && con[q])) ? T(0) : a.src[id];
                  R[q]              = T(0);
#pragma unroll
                  for (int e = 0; e < 3; ++e)
                    nn[e][q] = (T)a.n[e][id];
                }
          const T *Vd = a.Vend + side * N, *Dd = a.Dend + side * N;
          const T  W0 = hl[0] * hl[1] * hl[2] / hl[d], sgn = side ? T(1) : T(-1);
          for (int qb = 0; qb < N; ++qb)
            for (int qa = 0; qa < N; ++qa)
              {
                // per node: value and the three derivative factors at this face point
                auto factors = [&](int i, int j, int l, T &val, T gr[3]) {
                  const int ii[3] = {i, j, l};
                  T         v[3], dv[3];
#pragma unroll
                  for (int e = 0; e < 3; ++e)
                    {
                      if (e == d)
                        {
                          v[e]  = Vd[ii[e]];
                          dv[e] = Dd[ii[e]] * a.ih[e];
                        }
                      else
                        {
                          const int qe = e == ea ? qa : qb;
                          v[e]         = a.B[qe * N + ii[e]];
                          dv[e]        = a.G[qe * N + ii[e]] * a.ih[e];
                        }
                    }
                  val   = v[0] * v[1] * v[2];
                  gr[0] = dv[0] * v[1] * v[2];
                  gr[1] = v[0] * dv[1] * v[2];
                  gr[2] = v[0] * v[1] * dv[2];
                };
                T uv = T(0), g[3] = {T(0), T(0), T(0)}, nv[3] = {T(0), T(0), T(0)};
#pragma unroll
                for (int l = 0; l < N; ++l)
#pragma unroll
                  for (int j = 0; j < N; ++j)
#pragma unroll
                    for (int i = 0; i < N; ++i)
                      {
                        const int q = (l * N + j) * N + i;
                        T         val, gr[3];
                        factors(i, j, l, val, gr);
                        uv += val * u[q];
#pragma unroll
                        for (int e = 0; e < 3; ++e)
                          {
                            g[e] += gr[e] * u[q];
                            nv[e] += val * nn[e][q];
                          }
                      }
                const T nrm = sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
                const T inv = nrm > a.tol ? T(1) / nrm : T(1) / a.tol;
#pragma unroll
                for (int e = 0; e < 3; ++e)
                  nv[e] *= inv;
                const T W  = W0 * a.w[qa] * a.w[qb];
                const T gn = g[0] * nv[0] + g[1] * nv[1] + g[2] * nv[2];
                T       integrand;
                if (a.mode == 1)
                  integrand = -sgn * (-T(0.5) * (T(1) - uv * uv) * nv[d] + a.eps_t * g[d] + (a.eps_n - a.eps_t) * gn * nv[d]);
                else
                  integrand = sgn * (a.eps_t * g[d] + (a.eps_n - a.eps_t) * gn * nv[d]);
#pragma unroll
                for (int l = 0; l < N; ++l)
#pragma unroll
                  for (int j = 0; j < N; ++j)
#pragma unroll
                    for (int i = 0; i < N; ++i)
                      {
                        const int q = (l * N + j) * N + i;
                        T         val, gr[3];
                        factors(i, j, l, val, gr);
                        if (a.mode == 2)
                          {
                            const T pn = gr[0] * nv[0] + gr[1] * nv[1] + gr[2] * nv[2];
                            R[q] += W * sgn * (a.eps_t * gr[d] + (a.eps_n - a.eps_t) * pn * nv[d]) * val;
                          }
                        else
                          R[q] += W * integrand * val;
                      }
              }
#pragma unroll
          for (int q = 0; q < N3; ++q)
            if (!con[q])
              {
                if (a.mode == 2)
                  atomicAdd(a.diag + idx[q], (double)R[q]);
                else
                  atomicAdd(a.dst + idx[q], (a.mode == 0 ? a.scale : T(1)) * R[q]);
              }
        }
    }

    template <int K, typename T>
    cudaError_t
    launch_reinit(const ReinitLaunch<T> &h, int mode, cudaStream_t s)
    {
      constexpr int     N = K + 1;
      ReinitArgs<T, N> a{};
      a.g      = h.grid;
      a.scale  = (T)h.scale;
      a.inv_dt = (T)(1.0 / h.dt);
      a.eps_n  = (T)h.eps_normal;
      a.eps_t  = (T)h.eps_tangential;
      a.tol    = (T)h.normal_tolerance;
      a.det    = (T)(h.hlen[0] * h.hlen[1] * h.hlen[2]);
      for (int d = 0; d < 3; ++d)
        {
          a.ih[d] = (T)(1.0 / h.hlen[d]);
          a.n[d]  = h.normal[d];
        }
      const Tables1D &t = tables(K);
      for (int i = 0; i < N * N; ++i)
        {
          a.B[i] = (T)t.B[i];
          a.G[i] = (T)t.G[i];
        }
      for (int q = 0; q < N; ++q)
        a.w[q] = (T)t.qw[q];
      a.src      = h.src;
      a.dst      = h.dst;
      a.diag     = h.diag;
      a.mode     = mode;
      a.mask_src = h.mask_src;
      a.band_ls  = h.band > 0.0 ? h.band_ls : nullptr;
      a.band     = (T)h.band;
      a.wetting  = h.wetting;
      // basis values and derivatives at the end points of [0, 1] (Lagrange on the Gauss-Lobatto
      // nodes: the values are the unit rows of the first and last node; the derivatives are the rows
      // of the nodal differentiation matrix there, from the barycentric weights)
      for (int side = 0; side < 2; ++side)
        {
          const int jn = side ? N - 1 : 0;
          for (int i = 0; i < N; ++i)
            {
              a.Vend[side * N + i] = i == jn ? T(1) : T(0);
              double wi = 1.0, wj = 1.0;
              for (int k = 0; k < N; ++k)
                {
                  if (k != i)
                    wi /= (t.nodes[i] - t.nodes[k]);
                  if (k != jn)
                    wj /= (t.nodes[jn] - t.nodes[k]);
                }
              double dji = 0.0;
              if (i != jn)
                dji = wi / wj / (t.nodes[jn] - t.nodes[i]);
              else
                for (int k = 0; k < N; ++k)
                  if (k != jn)
                    {
                      double wk = 1.0;
                      for (int kk = 0; kk < N; ++kk)
                        if (kk != k)
                          wk /= (t.nodes[k] - t.nodes[kk]);
                      dji -= wk / wj / (t.nodes[jn] - t.nodes[k]);
                    }
              a.Dend[side * N + i] = (T)dji;
            }
        }
      const long long ncell  = (long long)h.grid.m[0] * h.grid.m[1] * h.grid.m[2];
      const int       blocks = (int)std::max<long long>(1, std::min<long long>((ncell + 127) / 128, 148LL * 16));
      if (!h.faces_only)
        reinit_kernel<K, T><<<blocks, 128, 0, s>>>(a);
      if (h.wetting && a.n[0] != nullptr)
        {
          cudaError_t e = cudaGetLastError();
          if (e != cudaSuccess)
            return e;
          wetting_kernel<K, T><<<148, 128, 0, s>>>(a);
        }
      return cudaGetLastError();
    }
  } // namespace

  namespace
  {
    // Right-hand sides of the normal-vector and curvature projections (one thread per cell):
    //   mode 0: dst_d += int g_d phi, g = grad psi, or normalize(grad psi, 1e-16) when normalized
    //           (normal_vector_operator.cpp:160-240, no narrow band)
    //   mode 1: dst   += -int div(n) phi with n = normalize(n_i, tol) at every DoF
    //           (curvature_operator.cpp:190-255, no narrow band)
    template <int K>
    __global__ void __launch_bounds__(128)
    level_set_rhs_kernel(const GridDesc g, const double *B, const double *G, const double *w, double det, double ihx,
                         double ihy, double ihz, int mode, int normalized, double tol, const double *in0,
                         const double *in1, const double *in2, double *out0, double *out1, double *out2,
                         const double *band_ls, double band)
    {
      constexpr int   N = K + 1, N3 = N * N * N;
      const double    ih[3] = {ihx, ihy, ihz};
      const int       m0 = g.m[0], m1 = g.m[1];
      const long long ncell = (long long)m0 * m1 * g.m[2];
      for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x)
        {
          const int cx = (int)(c % m0), cy = (int)((c / m0) % m1), cz = (int)(c / ((long long)m0 * m1));
          long long idx[N3];
          bool      con[N3];
          double    v[3][N3], R[3][N3], ls[N3];
#pragma unroll
          for (int l = 0; l < N; ++l)
#pragma unroll
            for (int j = 0; j < N; ++j)
#pragma unroll
              for (int i = 0; i < N; ++i)
                {
                  const int       q = (l * N + j) * N + i;
                  const int       I = K * cx + i, J = K * cy + j, L = K * cz + l;
                  const long long id = (long long)I + (long long)g.n[0] * ((long long)J + (long long)g.n[1] * L);
                  idx[q]            = id;
                  con[q]            = is_constrained(g, I, J, L, id);
                  ls[q]             = band_ls ? band_ls[id] : 0.0;
                  if (mode == 0)
                    v[0][q] = in0[id];
                  else
                    {
                      const double a = in0[id], b = in1[id], e = in2[id];
                      const double nn = sqrt(a * a + b * b + e * e), s = nn > tol ? 1.0 / nn : 1.0 / tol;
                      v[0][q] = a * s, v[1][q] = b * s, v[2][q] = e * s;
                    }
#pragma unroll
                  for (int d = 0; d < 3; ++d)
                    R[d][q] = 0.0;
                }
          for (int qz = 0; qz < N; ++qz)
            for (int qy = 0; qy < N; ++qy)
              for (int qx = 0; qx < N; ++qx)
                {
                  double gv[3] = {0.0, 0.0, 0.0}, div = 0.0, lq = 0.0;
#pragma unroll
                  for (int l = 0; l < N; ++l)
#pragma unroll
                    for (int j = 0; j < N; ++j)
#pragma unroll
                      for (int i = 0; i < N; ++i)
                        {
                          const int    q  = (l * N + j) * N + i;
                          const double bx = B[qx * N + i], by = B[qy * N + j], bz = B[qz * N + l];
                          const double p[3] = {G[qx * N + i] * ih[0] * by * bz, bx * G[qy * N + j] * ih[1] * bz,
                                               bx * by * G[qz * N + l] * ih[2]};
                          lq += bx * by * bz * ls[q];
                          if (mode == 0)
                            {
#pragma unroll
                              for (int d = 0; d < 3; ++d)
                                gv[d] += p[d] * v[0][q];
                            }
                          else
                            div += p[0] * v[0][q] + p[1] * v[1][q] + p[2] * v[2][q];
                        }
                  // narrow band (normal_vector_operator.cpp:184-191, curvature_operator.cpp:209-214):
                  // the gradient (before its normalisation) or the divergence is masked by
                  // |level set| < band at the point
                  if (band_ls && !(fabs(lq) < band))
                    {
                      gv[0] = gv[1] = gv[2] = 0.0;
                      div                   = 0.0;
                    }
                  if (mode == 0 && normalized)
                    {
                      const double nn = sqrt(gv[0] * gv[0] + gv[1] * gv[1] + gv[2] * gv[2]);
                      const double s  = nn > 1e-16 ? 1.0 / nn : 1e16;
#pragma unroll
                      for (int d = 0; d < 3; ++d)
                        gv[d] *= s;
                    }
                  const double jw = det * w[qx] * w[qy] * w[qz];
#pragma unroll
                  for (int l = 0; l < N; ++l)
#pragma unroll
                    for (int j = 0; j < N; ++j)
#pragma unroll
                      for (int i = 0; i < N; ++i)
                        {
                          const double phi = B[qx * N + i] * B[qy * N + j] * B[qz * N + l] * jw;
                          if (mode == 0)
                            {
#pragma unroll
                              for (int d = 0; d < 3; ++d)
                                R[d][(l * N + j) * N + i] += gv[d] * phi;
                            }
                          else
                            R[0][(l * N + j) * N + i] -= div * phi;
                        }
                }
#pragma unroll
          for (int q = 0; q < N3; ++q)
            if (!con[q])
              {
                atomicAdd(out0 + idx[q], R[0][q]);
                if (mode == 0)
                  {
                    atomicAdd(out1 + idx[q], R[1][q]);
                    atomicAdd(out2 + idx[q], R[2][q]);
                  }
              }
        }
    }

    // 1-D tables of degree K in device memory for the level-set rhs kernels (uploaded once per device)
    const double *
    level_set_tables(int K)
    {
      static std::mutex mtx;
      static double    *dev[64][3] = {}; // [device][degree]
      int               d          = 0;
      if (cudaGetDevice(&d) != cudaSuccess || d >= 64)
        return nullptr;
      std::lock_guard<std::mutex> lock(mtx);
      if (!dev[d][K])
        {
          const Tables1D &t = tables(K);
          const int       n = t.n;
          double          h[3 * MAX_N * MAX_N]{};
          for (int i = 0; i < n * n; ++i)
            {
              h[i]         = t.B[i];
              h[n * n + i] = t.G[i];
            }
          for (int q = 0; q < n; ++q)
            h[2 * n * n + q] = t.qw[q];
          double *p = nullptr;
          // a legacy-stream copy, completed before kernels on other streams read the table
          if (cudaMalloc(&p, sizeof(h)) != cudaSuccess || cudaMemcpy(p, h, sizeof(h), cudaMemcpyHostToDevice) != cudaSuccess ||
              cudaStreamSynchronize(cudaStreamLegacy) != cudaSuccess)
            return nullptr;
          dev[d][K] = p;
        }
      return dev[d][K];
    }
  } // namespace

  cudaError_t
  level_set_rhs(const GridDesc &g, int K, const double hlen[3], int mode, int normalized, double tol,
                const double *in0, const double *in1, const double *in2, double *out0, double *out1, double *out2,
                cudaStream_t s, const double *band_ls, double band)
  {
    if (!(band > 0.0))
      band_ls = nullptr;
    if (K < 1 || K > 3)
      return cudaErrorInvalidValue;
    const double *tab = level_set_tables(K);
    if (!tab)
      return cudaErrorMemoryAllocation;
    const int       n      = K + 1;
    const long long ncell  = (long long)g.m[0] * g.m[1] * g.m[2];
    const int       blocks = (int)std::max<long long>(1, std::min<long long>((ncell + 127) / 128, 148LL * 16));
    const double    det    = hlen[0] * hlen[1] * hlen[2];
    if (K == 1)
      level_set_rhs_kernel<1><<<blocks, 128, 0, s>>>(g, tab, tab + n * n, tab + 2 * n * n, det, 1.0 / hlen[0],
                                                      1.0 / hlen[1], 1.0 / hlen[2], mode, normalized, tol, in0, in1,
                                                      in2, out0, out1, out2, band_ls, band);
    else if (K == 2)
      level_set_rhs_kernel<2><<<blocks, 128, 0, s>>>(g, tab, tab + n * n, tab + 2 * n * n, det, 1.0 / hlen[0],
                                                      1.0 / hlen[1], 1.0 / hlen[2], mode, normalized, tol, in0, in1,
                                                      in2, out0, out1, out2, band_ls, band);
    else
      level_set_rhs_kernel<3><<<blocks, 128, 0, s>>>(g, tab, tab + n * n, tab + 2 * n * n, det, 1.0 / hlen[0],
                                                      1.0 / hlen[1], 1.0 / hlen[2], mode, normalized, tol, in0, in1,
                                                      in2, out0, out1, out2, band_ls, band);
    return cudaGetLastError();
  }

  template <typename T>
  cudaError_t
  reinit_integrate(const ReinitLaunch<T> &h, int mode, cudaStream_t s)
  {
    switch (h.degree)
      {
        case 1: return launch_reinit<1, T>(h, mode, s);
        case 2: return launch_reinit<2, T>(h, mode, s);
        case 3: return launch_reinit<3, T>(h, mode, s);
        default: return cudaErrorInvalidValue;
      }
  }

  template cudaError_t reinit_integrate<double>(const ReinitLaunch<double> &, int, cudaStream_t);
  template cudaError_t reinit_integrate<float>(const ReinitLaunch<float> &, int, cudaStream_t);
} // namespace mpdg
