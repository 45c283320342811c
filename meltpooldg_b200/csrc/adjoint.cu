// Kernels of the adjoint of the transient heat problem (no reference counterpart: the reference
// has no adjoint; the forward operator is HeatDiffuseMultiPhaseOperator's tangent,
// source/heat/heat_diffuse_operator.cpp:1029-1079).
//
//  * exp_kernel: k_c = exp(z_c) (per-cell log-conductivity -> conductivity)
//  * cell_form_kernel: the fused coefficient-gradient reduction
//        g_c += s * k_c * lam_c^T K_c T_c ,
//    K_c the unit-conductivity cell stiffness.  With the fast-diagonalisation basis of sumfac.cuh
//    K_c = W3^T (cx Lx + cy Ly + cz Lz) W3, so the form is the Lambda-weighted dot product of the two
//    transformed cells (two forward transforms, no inverse).  One thread per cell, deterministic
//    (no atomics: every cell owns its gradient entry).
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <set>

#include "brick.cuh"
#include "kernels.h"
#include "sumfac.cuh"

namespace mpdg
{
  __constant__ double c_adj_tab[3][32]; // per degree (1, 2): WE | WO | lambda

  struct FormArgs
  {
    GridDesc      g;
    int           K;
    double        cx, cy, cz;
    double        scale; // s
    const double *lam, *T, *k; // k: per-cell conductivity (may be null: kconst)
    double        kconst;
    double       *out;   // accumulated per cell
    int           accumulate;
  };

  template <int K>
  __global__ void
  cell_form_kernel(const __grid_constant__ FormArgs a)
  {
    constexpr int N = K + 1, NE = (N + 1) / 2, NO = N / 2;
    const long long ncells = (long long)a.g.m[0] * a.g.m[1] * a.g.m[2];
    const double   *we = c_adj_tab[K], *wo = we + NE * NE, *lam1 = we + NE * NE + NO * NO;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncells; c += (long long)gridDim.x * blockDim.x)
      {
        const int cx = (int)(c % a.g.m[0]), cy = (int)((c / a.g.m[0]) % a.g.m[1]),
                  cz = (int)(c / ((long long)a.g.m[0] * a.g.m[1]));
        double    u[N * N * N], v[N * N * N];
#pragma unroll
        for (int l = 0; l < N; ++l)
#pragma unroll
          for (int j = 0; j < N; ++j)
#pragma unroll
            for (int i = 0; i < N; ++i)
              {
                const int       I = K * cx + i, J = K * cy + j, L = K * cz + l;
                const long long idx = lattice_index(a.g, I, J, L);
                const bool      con = is_constrained(a.g, I, J, L, idx);
                u[(l * N + j) * N + i] = con ? 0.0 : a.lam[idx];
                v[(l * N + j) * N + i] = con ? 0.0 : a.T[idx];
              }
        xy_planes<double, N, N, true>(u, we, wo);
        xy_planes<double, N, N, true>(v, we, wo);
#pragma unroll
        for (int q = 0; q < N * N; ++q)
          {
            fwd_line<double, N, N * N>(u, q, we, wo);
            fwd_line<double, N, N * N>(v, q, we, wo);
          }
        double s = 0.0;
#pragma unroll
        for (int l = 0; l < N; ++l)
#pragma unroll
          for (int j = 0; j < N; ++j)
#pragma unroll
            for (int i = 0; i < N; ++i)
              {
                const double w = a.cx * lam1[i] + a.cy * lam1[j] + a.cz * lam1[l];
                s += w * u[(l * N + j) * N + i] * v[(l * N + j) * N + i];
              }
        const double kc = a.k ? a.k[c] : a.kconst;
        const double r  = a.scale * kc * s;
        a.out[c]        = a.accumulate ? a.out[c] + r : r;
      }
  }

  __global__ void
  exp_kernel(double *k, const double *z, long long n)
  {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      k[i] = exp(z[i]);
  }

  static cudaError_t
  upload_adj_tables()
  {
    static std::mutex    mtx;
    static std::set<int> done;
    int                  dev = 0;
    cudaError_t          e   = cudaGetDevice(&dev);
    if (e != cudaSuccess)
      return e;
    std::lock_guard<std::mutex> lock(mtx);
    if (done.count(dev))
      return cudaSuccess;
    double h[3][32] = {};
    for (int K = 1; K <= 2; ++K)
      {
        const Tables1D &t = tables(K);
        int             o = 0;
        for (int i = 0; i < t.ne * t.ne; ++i)
          h[K][o++] = t.WE[i];
        for (int i = 0; i < t.no * t.no; ++i)
          h[K][o++] = t.WO[i];
        for (int i = 0; i < t.n; ++i)
          h[K][o++] = t.lam[i];
      }
    if ((e = cudaMemcpyToSymbol(c_adj_tab, h, sizeof(h))) != cudaSuccess)
      return e;
    // the copy ran on the legacy stream: complete it before kernels on other streams read the table
    if ((e = cudaStreamSynchronize(cudaStreamLegacy)) != cudaSuccess)
      return e;
    done.insert(dev);
    return cudaSuccess;
  }

  cudaError_t
  heat_cell_form(const GridDesc &g, int K, const HeatGeom &geo, double scale, const double *lam, const double *T,
                 const double *k, double kconst, double *out, bool accumulate, cudaStream_t s)
  {
    if (K < 1 || K > 2)
      return cudaErrorInvalidValue;
    cudaError_t e = upload_adj_tables();
    if (e != cudaSuccess)
      return e;
    FormArgs a;
    a.g          = g;
    a.K          = K;
    a.cx         = geo.cx;
    a.cy         = geo.cy;
    a.cz         = geo.cz;
    a.scale      = scale;
    a.lam        = lam;
    a.T          = T;
    a.k          = k;
    a.kconst     = kconst;
    a.out        = out;
    a.accumulate = accumulate ? 1 : 0;
    const long long nc     = (long long)g.m[0] * g.m[1] * g.m[2];
    const int       blocks = (int)std::min<long long>((nc + 127) / 128, 148LL * 16);
    if (K == 1)
      cell_form_kernel<1><<<blocks, 128, 0, s>>>(a);
    else
      cell_form_kernel<2><<<blocks, 128, 0, s>>>(a);
    return cudaGetLastError();
  }

  cudaError_t
  vec_exp(double *k, const double *z, long long n, cudaStream_t s)
  {
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
    exp_kernel<<<blocks > 0 ? blocks : 1, 256, 0, s>>>(k, z, n);
    return cudaGetLastError();
  }
} // namespace mpdg
