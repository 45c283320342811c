// Conservative level-set reinitialisation operator (Olsson), FE_Q(1, 2).
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
          T         u[N3], R[N3];
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
                }
          for (int qz = 0; qz < N; ++qz)
            for (int qy = 0; qy < N; ++qy)
              for (int qx = 0; qx < N; ++qx)
                {
                  // value and gradient of u and the normal field at the Gauss point
                  T uv = T(0), g[3] = {T(0), T(0), T(0)}, nv[3] = {T(0), T(0), T(0)};
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
                          g[0] += a.G[qx * N + i] * by * bz * u[q];
                          g[1] += bx * a.G[qy * N + j] * bz * u[q];
                          g[2] += bx * by * a.G[qz * N + l] * u[q];
#pragma unroll
                          for (int d = 0; d < 3; ++d)
                            nv[d] += phi * (T)a.n[d][idx[q]];
                        }
#pragma unroll
                  for (int d = 0; d < 3; ++d)
                    g[d] *= a.ih[d];
                  const T nn  = sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
                  const T inv = nn > a.tol ? T(1) / nn : T(1) / a.tol;
#pragma unroll
                  for (int d = 0; d < 3; ++d)
                    nv[d] *= inv;
                  const T jw = a.det * a.w[qx] * a.w[qy] * a.w[qz];
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
      const long long ncell  = (long long)h.grid.m[0] * h.grid.m[1] * h.grid.m[2];
      const int       blocks = (int)std::max<long long>(1, std::min<long long>((ncell + 127) / 128, 148LL * 16));
      reinit_kernel<K, T><<<blocks, 128, 0, s>>>(a);
      return cudaGetLastError();
    }
  } // namespace

  template <typename T>
  cudaError_t
  reinit_integrate(const ReinitLaunch<T> &h, int mode, cudaStream_t s)
  {
    switch (h.degree)
      {
        case 1: return launch_reinit<1, T>(h, mode, s);
        case 2: return launch_reinit<2, T>(h, mode, s);
        default: return cudaErrorInvalidValue;
      }
  }

  template cudaError_t reinit_integrate<double>(const ReinitLaunch<double> &, int, cudaStream_t);
  template cudaError_t reinit_integrate<float>(const ReinitLaunch<float> &, int, cudaStream_t);
} // namespace mpdg
