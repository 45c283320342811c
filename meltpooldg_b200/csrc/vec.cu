// Vector kernels and deterministic reductions for the Krylov solvers.
//
// Every reduction runs on a fixed grid of RED_BLOCKS blocks with a grid-stride loop, reduces in
// registers/shared memory in a fixed order, writes one partial per block, and the last block to
// finish (threadfence + ticket) sums the partials in block order.  Results are therefore
// bit-reproducible run to run.  Sums are accumulated in double for every vector type, so the FP32
// inner solver keeps FP64 dot products and norms.
//
// The PCG kernels carry the scalar recurrences of dealii::SolverCG on the device (CGState): the
// host enqueues iterations without waiting for the scalars, and every kernel returns at once
// when the state says the solve has finished.  ReductionControl semantics
// (include/meltpooldg/linear_algebra/linear_solver.hpp:36): converged when the unpreconditioned
// residual norm is <= rel_tol * |r_0| or <= abs_tol; failed at max_it or on NaN.
#include <cuda_runtime.h>

#include <cmath>

#include "kernels.h"

namespace mpdg
{
  namespace
  {
    constexpr int NWARP = RED_THREADS / 32;

    __device__ __forceinline__ double
    warp_sum(double v)
    {
#pragma unroll
      for (int off = 16; off > 0; off >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, off);
      return v;
    }

    __device__ __forceinline__ double
    warp_max(double v)
    {
#pragma unroll
      for (int off = 16; off > 0; off >>= 1)
        v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
      return v;
    }

    // Block-reduce M values; the last block sums the per-block partials in order and calls fin()
    // on thread 0 with the totals.  MAX selects a max-reduction instead of a sum.
    template <int M, bool MAX = false, class Fin>
    __device__ __forceinline__ void
    reduce_finish(double (&v)[M], int m_active, Reducer red, Fin fin)
    {
      __shared__ double sh[M][NWARP];
      __shared__ double tot[M];
      __shared__ bool   last;
      const int         lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
      for (int k = 0; k < M; ++k)
        if (k < m_active)
          {
            const double w = MAX ? warp_max(v[k]) : warp_sum(v[k]);
            if (lane == 0)
              sh[k][warp] = w;
          }
      __syncthreads();
      if (warp == 0)
        {
#pragma unroll
          for (int k = 0; k < M; ++k)
            if (k < m_active)
              {
                double s = lane < NWARP ? sh[k][lane] : (MAX ? -INFINITY : 0.0);
                s        = MAX ? warp_max(s) : warp_sum(s);
                if (lane == 0)
                  red.partials[k * RED_BLOCKS + blockIdx.x] = s;
              }
        }
      if (threadIdx.x == 0)
        {
          __threadfence();
          last = (atomicAdd(red.counter, 1u) == gridDim.x - 1);
        }
      __syncthreads();
      if (!last)
        return;
      for (int k = 0; k < m_active; ++k)
        {
          double s = MAX ? -INFINITY : 0.0;
          for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
            {
              const double p = __ldcg(red.partials + k * RED_BLOCKS + b);
              s              = MAX ? fmax(s, p) : s + p;
            }
          s = MAX ? warp_max(s) : warp_sum(s);
          if (lane == 0)
            sh[0][warp] = s;
          __syncthreads();
          if (threadIdx.x == 0)
            {
              double t = sh[0][0];
              for (int w = 1; w < NWARP; ++w)
                t = MAX ? fmax(t, sh[0][w]) : t + sh[0][w];
              tot[k] = t;
            }
          __syncthreads();
        }
      if (threadIdx.x == 0)
        {
          fin(tot);
          *red.counter = 0u;
          __threadfence();
        }
    }

    __device__ __forceinline__ int
    control_check(const CGState &st, int step, double value)
    {
      if (value <= st.rel_tol * st.res0)
        return 1;
      if (value <= st.abs_tol)
        return 1;
      if (step >= st.max_it || isnan(value))
        return 2;
      return 0;
    }

    template <typename T>
    __global__ void
    cg_init_kernel(const T *__restrict__ r, const T *__restrict__ invd, CGState *st, double *hist, Reducer red,
                   long long n)
    {
      double v[2] = {0.0, 0.0};
      for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        {
          const double ri = (double)r[i];
          const double zi = invd ? (double)(T)(r[i] * invd[i]) : ri;
          v[0] += ri * ri;
          v[1] += ri * zi;
        }
      reduce_finish<2>(v, 2, red, [&](double *tot) {
        const double res = sqrt(tot[0]);
        st->res0         = res;
        st->res          = res;
        st->tol          = fmax(st->abs_tol, st->rel_tol * res);
        st->rho          = tot[1];
        st->beta         = 0.0;
        st->it           = 0;
        if (hist)
          hist[0] = res;
        st->done = control_check(*st, 0, res);
      });
    }

    // 16-byte packs for the streaming CG kernels (4 floats / 2 doubles per access)
    template <typename T>
    struct Pack;
    template <>
    struct Pack<float>
    {
      using V                  = float4;
      static constexpr int W   = 4;
      __device__ static float &at(V &v, int k) { return (&v.x)[k]; }
    };
    template <>
    struct Pack<double>
    {
      using V                  = double2;
      static constexpr int W   = 2;
      __device__ static double &at(V &v, int k) { return (&v.x)[k]; }
    };

    template <typename T>
    __global__ void
    cg_update_p_kernel(const T *__restrict__ r, const T *__restrict__ invd, T *__restrict__ p, const CGState *st,
                       long long n, int packed)
    {
      if (st->done)
        return;
      const T         beta  = (T)st->beta;
      const bool      first = st->it == 0;
      const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x, stride = (long long)gridDim.x * blockDim.x;
      using P               = Pack<T>;
      const long long nv    = packed ? n / P::W : 0;
      for (long long i = tid; i < nv; i += stride)
        {
          typename P::V rv = reinterpret_cast<const typename P::V *>(r)[i];
          typename P::V dv = invd ? reinterpret_cast<const typename P::V *>(invd)[i] : rv;
          typename P::V pv = first ? rv : reinterpret_cast<const typename P::V *>(p)[i];
#pragma unroll
          for (int k = 0; k < P::W; ++k)
            {
              const T z    = invd ? P::at(rv, k) * P::at(dv, k) : P::at(rv, k);
              P::at(pv, k) = first ? z : z + beta * P::at(pv, k);
            }
          reinterpret_cast<typename P::V *>(p)[i] = pv;
        }
      for (long long i = nv * P::W + tid; i < n; i += stride)
        {
          const T z = invd ? r[i] * invd[i] : r[i];
          p[i]      = first ? z : z + beta * p[i];
        }
    }

    template <typename T>
    __global__ void
    cg_alpha_kernel(const T *__restrict__ p, const T *__restrict__ v, CGState *st, Reducer red, long long n)
    {
      if (st->done)
        return;
      double a[1] = {0.0};
      for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        a[0] += (double)p[i] * (double)v[i];
      reduce_finish<1>(a, 1, red, [&](double *tot) { st->alpha = st->rho / tot[0]; });
    }

    // The x / r update walks the vectors from the high end down: the apply before it finishes at the
    // high end, so the first packs it reads of p and v are still in L2, and cg_update_p after it starts
    // at the low end, where this kernel has just left r, invd and p.
#ifndef MPDG_CG_XR_REVERSE
#define MPDG_CG_XR_REVERSE 1
#endif
    template <typename T>
    __global__ void
    cg_update_xr_kernel(T *__restrict__ x, T *__restrict__ r, const T *__restrict__ p, const T *__restrict__ v,
                        const T *__restrict__ invd, CGState *st, double *hist, Reducer red, long long n, int packed)
    {
      if (st->done)
        return;
      const T alpha = (T)st->alpha;
      double  a[2]  = {0.0, 0.0};
      const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x, stride = (long long)gridDim.x * blockDim.x;
      using P               = Pack<T>;
      const long long nv    = packed ? n / P::W : 0;
      for (long long i0 = tid; i0 < nv; i0 += stride)
        {
          const long long i = MPDG_CG_XR_REVERSE ? nv - 1 - i0 : i0;
          using V = typename P::V;
          V xv = reinterpret_cast<const V *>(x)[i], rv = reinterpret_cast<const V *>(r)[i];
          V pv = reinterpret_cast<const V *>(p)[i], vv = reinterpret_cast<const V *>(v)[i];
          V dv = rv;
          if (invd)
            dv = reinterpret_cast<const V *>(invd)[i];
#pragma unroll
          for (int k = 0; k < P::W; ++k)
            {
              P::at(xv, k) += alpha * P::at(pv, k);
              const T ri   = P::at(rv, k) - alpha * P::at(vv, k);
              P::at(rv, k) = ri;
              const T zi   = invd ? ri * P::at(dv, k) : ri;
              a[0] += (double)ri * (double)ri;
              a[1] += (double)ri * (double)zi;
            }
          reinterpret_cast<V *>(x)[i] = xv;
          reinterpret_cast<V *>(r)[i] = rv;
        }
      for (long long i = nv * P::W + tid; i < n; i += stride)
        {
          x[i] += alpha * p[i];
          const T ri = r[i] - alpha * v[i];
          r[i]       = ri;
          const T zi = invd ? ri * invd[i] : ri;
          a[0] += (double)ri * (double)ri;
          a[1] += (double)ri * (double)zi;
        }
      reduce_finish<2>(a, 2, red, [&](double *tot) {
        const int    it  = st->it + 1;
        const double res = sqrt(tot[0]);
        st->it           = it;
        st->res          = res;
        if (hist)
          hist[it] = res;
        st->done = control_check(*st, it, res);
        st->beta = tot[1] / st->rho;
        st->rho  = tot[1];
      });
    }

    template <typename T>
    __global__ void
    fill_kernel(T *x, T v, long long n)
    {
      for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] = v;
    }

    template <typename Td, typename Ts>
    __global__ void
    convert_kernel(Td *d, const Ts *s, long long n)
    {
      for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        d[i] = (Td)s[i];
    }

    template <typename T>
    __global__ void
    axpby_kernel(T *d, T a, const T *x, T b, const T *y, long long n)
    {
      for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        {
          T v = T(0);
          if (x)
            v = a * x[i];
          if (y)
            v = fma(b, y[i], v);
          d[i] = v;
        }
    }

    __global__ void
    add_f32_kernel(double *x, const float *e, long long n)
    {
      for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] += (double)e[i];
    }

    template <typename T>
    __global__ void
    scale_kernel(T *d, const T *s, const T *w, long long n)
    {
      for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        d[i] = w ? s[i] * w[i] : s[i];
    }

    constexpr int MAXV = 32;
    template <typename T>
    struct VecList
    {
      const T *v[MAXV];
    };

    template <typename T>
    struct PairList
    {
      const T *x[8];
      const T *y[8];
    };

    template <typename T>
    __global__ void
    multidot_kernel(const __grid_constant__ PairList<T> L, int m, long long n, double *out, Reducer red)
    {
      double a[8] = {};
      for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        {
#pragma unroll
          for (int k = 0; k < 8; ++k)
            if (k < m)
              a[k] += (double)L.x[k][i] * (double)L.y[k][i];
        }
      reduce_finish<8>(a, m, red, [&](double *tot) {
        for (int k = 0; k < m; ++k)
          out[k] = tot[k];
      });
    }

    // x += post * sum_k c_k v_k   (post = scalar); coefficients read from the device
    template <typename T>
    __global__ void
    multiaxpy_kernel(T *x, const __grid_constant__ VecList<T> L, const double *c, int m, long long n, double post)
    {
      __shared__ double cs[MAXV];
      if (threadIdx.x < MAXV)
        cs[threadIdx.x] = threadIdx.x < m ? c[threadIdx.x] : 0.0;
      __syncthreads();
      for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        {
          double s = 0.0;
          for (int k = 0; k < m; ++k)
            s += cs[k] * (double)L.v[k][i];
          x[i] += (T)(post * s);
        }
    }

    // h_k = w . v_k (k < m), plus ||w||^2 as entry m
    // h_k = w . v_k (k < m <= MB), out[m] = |w|^2; 16-byte packs when every vector is aligned
    template <typename T, int MB>
    __global__ void
    dots_against_kernel(const T *w, const __grid_constant__ VecList<T> L, int m, long long n, double *out, Reducer red,
                        int packed)
    {
      double          a[MB + 1] = {};
      const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x, stride = (long long)gridDim.x * blockDim.x;
      using P               = Pack<T>;
      using V               = typename P::V;
      const long long nv    = packed ? n / P::W : 0;
      for (long long i = tid; i < nv; i += stride)
        {
          V      wv = reinterpret_cast<const V *>(w)[i];
          double wd[P::W];
#pragma unroll
          for (int e = 0; e < P::W; ++e)
            {
              wd[e] = (double)P::at(wv, e);
              a[MB] += wd[e] * wd[e];
            }
#pragma unroll
          for (int k = 0; k < MB; ++k)
            if (k < m)
              {
                V vv = reinterpret_cast<const V *>(L.v[k])[i];
#pragma unroll
                for (int e = 0; e < P::W; ++e)
                  a[k] += wd[e] * (double)P::at(vv, e);
              }
        }
      for (long long i = nv * P::W + tid; i < n; i += stride)
        {
          const double wi = (double)w[i];
#pragma unroll
          for (int k = 0; k < MB; ++k)
            if (k < m)
              a[k] += wi * (double)L.v[k][i];
          a[MB] += wi * wi;
        }
      // move the norm entry next to the m dots
      double b[MB + 1];
#pragma unroll
      for (int k = 0; k <= MB; ++k)
        b[k] = (k < m) ? a[k] : (k == m ? a[MB] : 0.0);
      reduce_finish<MB + 1>(b, m + 1, red, [&](double *tot) {
        for (int k = 0; k <= m; ++k)
          out[k] = tot[k];
      });
    }

    // w -= sum_k h_k v_k (k < m <= MB); out[0] = ||w||^2
    template <typename T, int MB>
    __global__ void
    orth_update_kernel(T *w, const __grid_constant__ VecList<T> L, const double *h, int m, long long n, double *out,
                       Reducer red, int packed)
    {
      __shared__ double hs[MB];
      if (threadIdx.x < MB)
        hs[threadIdx.x] = threadIdx.x < m ? h[threadIdx.x] : 0.0;
      __syncthreads();
      double          a[1] = {0.0};
      const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x, stride = (long long)gridDim.x * blockDim.x;
      using P               = Pack<T>;
      using V               = typename P::V;
      const long long nv    = packed ? n / P::W : 0;
      for (long long i = tid; i < nv; i += stride)
        {
          V      wv = reinterpret_cast<const V *>(w)[i];
          double sd[P::W];
#pragma unroll
          for (int e = 0; e < P::W; ++e)
            sd[e] = (double)P::at(wv, e);
#pragma unroll
          for (int k = 0; k < MB; ++k)
            if (k < m)
              {
                V vv = reinterpret_cast<const V *>(L.v[k])[i];
#pragma unroll
                for (int e = 0; e < P::W; ++e)
                  sd[e] -= hs[k] * (double)P::at(vv, e);
              }
#pragma unroll
          for (int e = 0; e < P::W; ++e)
            {
              const T t     = (T)sd[e];
              P::at(wv, e) = t;
              a[0] += (double)t * (double)t;
            }
          reinterpret_cast<V *>(w)[i] = wv;
        }
      for (long long i = nv * P::W + tid; i < n; i += stride)
        {
          double s = (double)w[i];
          for (int k = 0; k < m; ++k)
            s -= hs[k] * (double)L.v[k][i];
          const T t = (T)s;
          w[i]      = t;
          a[0] += (double)t * (double)t;
        }
      reduce_finish<1>(a, 1, red, [&](double *tot) { out[0] = tot[0]; });
    }

    template <typename T>
    __global__ void
    invert_kernel(T *d, T thr, long long n)
    {
      for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        d[i] = (fabs(d[i]) > thr) ? T(1) / d[i] : T(1);
    }

    template <typename T>
    __global__ void
    absmax_kernel(const T *d, long long n, double *out, Reducer red)
    {
      double a[1] = {0.0};
      for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        a[0] = fmax(a[0], fabs((double)d[i]));
      reduce_finish<1, true>(a, 1, red, [&](double *tot) { out[0] = tot[0]; });
    }

    template <typename T>
    __global__ void
    invert_rel_kernel(T *d, const double *amax, long long n)
    {
      const double thr = 1.0e-14 * fmax(1.0, *amax);
      for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        d[i] = (fabs((double)d[i]) > thr) ? T(1) / d[i] : T(1);
    }

    template <typename T>
    __global__ void
    set_constrained_kernel(T *x, T v, const GridDesc g)
    {
      const long long n = (long long)g.n[0] * g.n[1] * g.n[2];
      for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        {
          const int I = (int)(i % g.n[0]), J = (int)((i / g.n[0]) % g.n[1]), L = (int)(i / ((long long)g.n[0] * g.n[1]));
          if (is_constrained(g, I, J, L, i))
            x[i] = v;
        }
    }

    // dst = src on constrained DoFs, 0 elsewhere
    template <typename T>
    __global__ void
    copy_constrained_kernel(T *dst, const T *src, const GridDesc g)
    {
      const long long n = (long long)g.n[0] * g.n[1] * g.n[2];
      for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        {
          const int I = (int)(i % g.n[0]), J = (int)((i / g.n[0]) % g.n[1]), L = (int)(i / ((long long)g.n[0] * g.n[1]));
          dst[i]      = is_constrained(g, I, J, L, i) ? src[i] : T(0);
        }
    }

    // dst = src on constrained DoFs, other entries untouched (AffineConstraints::distribute with
    // the Dirichlet values held in src)
    template <typename T>
    __global__ void
    distribute_constrained_kernel(T *dst, const T *src, const GridDesc g)
    {
      const long long n = (long long)g.n[0] * g.n[1] * g.n[2];
      for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        {
          const int I = (int)(i % g.n[0]), J = (int)((i / g.n[0]) % g.n[1]), L = (int)(i / ((long long)g.n[0] * g.n[1]));
          if (is_constrained(g, I, J, L, i))
            dst[i] = src[i];
        }
    }

    inline int
    aligned16(const void *p)
    {
      return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; // null counts as aligned (unused operand)
    }

    int
    stream_blocks(long long n)
    {
      const long long b = (n + 255) / 256;
      return (int)(b < 148LL * 16 ? (b > 0 ? b : 1) : 148LL * 16);
    }
  } // namespace

  template <typename T>
  cudaError_t
  cg_init(const T *r, const T *invd, T *p, CGState *st, double *hist, Reducer red, long long n, cudaStream_t s)
  {
    (void)p;
    cg_init_kernel<T><<<RED_BLOCKS, RED_THREADS, 0, s>>>(r, invd, st, hist, red, n);
    return cudaGetLastError();
  }
  template <typename T>
  cudaError_t
  cg_update_p(const T *r, const T *invd, T *p, const CGState *st, long long n, cudaStream_t s)
  {
    const int packed = aligned16(r) && aligned16(invd) && aligned16(p);
    cg_update_p_kernel<T><<<stream_blocks(packed ? (n + 3) / 4 : n), 256, 0, s>>>(r, invd, p, st, n, packed);
    return cudaGetLastError();
  }
  template <typename T>
  cudaError_t
  cg_alpha(const T *p, const T *v, CGState *st, Reducer red, long long n, cudaStream_t s)
  {
    cg_alpha_kernel<T><<<RED_BLOCKS, RED_THREADS, 0, s>>>(p, v, st, red, n);
    return cudaGetLastError();
  }
  template <typename T>
  cudaError_t
  cg_update_xr(T *x, T *r, const T *p, const T *v, const T *invd, CGState *st, double *hist, Reducer red,
               long long n, cudaStream_t s)
  {
    const int packed = aligned16(x) && aligned16(r) && aligned16(p) && aligned16(v) && aligned16(invd);
    cg_update_xr_kernel<T><<<RED_BLOCKS, RED_THREADS, 0, s>>>(x, r, p, v, invd, st, hist, red, n, packed);
    return cudaGetLastError();
  }

  template <typename T>
  cudaError_t
  vec_fill(T *x, T v, long long n, cudaStream_t s)
  {
    fill_kernel<T><<<stream_blocks(n), 256, 0, s>>>(x, v, n);
    return cudaGetLastError();
  }
  template <typename Td, typename Ts>
  cudaError_t
  vec_convert(Td *d, const Ts *src, long long n, cudaStream_t s)
  {
    convert_kernel<Td, Ts><<<stream_blocks(n), 256, 0, s>>>(d, src, n);
    return cudaGetLastError();
  }
  template <typename T>
  cudaError_t
  vec_axpby(T *d, double a, const T *x, double b, const T *y, long long n, cudaStream_t s)
  {
    axpby_kernel<T><<<stream_blocks(n), 256, 0, s>>>(d, (T)a, x, (T)b, y, n);
    return cudaGetLastError();
  }
  cudaError_t
  vec_add_f32_to_f64(double *x, const float *e, long long n, cudaStream_t s)
  {
    add_f32_kernel<<<stream_blocks(n), 256, 0, s>>>(x, e, n);
    return cudaGetLastError();
  }
  template <typename T>
  cudaError_t
  vec_multidot(const T *const *x, const T *const *y, int m, long long n, double *out, Reducer red, cudaStream_t s)
  {
    if (m < 1 || m > 8)
      return cudaErrorInvalidValue;
    PairList<T> L{};
    for (int k = 0; k < m; ++k)
      {
        L.x[k] = x[k];
        L.y[k] = y[k];
      }
    multidot_kernel<T><<<RED_BLOCKS, RED_THREADS, 0, s>>>(L, m, n, out, red);
    return cudaGetLastError();
  }
  template <typename T>
  cudaError_t
  vec_scale(T *d, const T *src, const T *w, long long n, cudaStream_t s)
  {
    scale_kernel<T><<<stream_blocks(n), 256, 0, s>>>(d, src, w, n);
    return cudaGetLastError();
  }
  template <typename T>
  cudaError_t
  vec_multiaxpy(T *x, const T *const *v, const double *c, int m, long long n, double post, cudaStream_t s)
  {
    if (m < 1 || m > MAXV)
      return cudaErrorInvalidValue;
    VecList<T> L{};
    for (int k = 0; k < m; ++k)
      L.v[k] = v[k];
    multiaxpy_kernel<T><<<stream_blocks(n), 256, 0, s>>>(x, L, c, m, n, post);
    return cudaGetLastError();
  }
  template <typename T>
  cudaError_t
  vec_dots_against(const T *w, const T *const *v, int m, long long n, double *out, Reducer red, cudaStream_t s)
  {
    if (m < 1 || m > MAXV)
      return cudaErrorInvalidValue;
    VecList<T> L{};
    int        packed = aligned16(w);
    for (int k = 0; k < m; ++k)
      {
        L.v[k] = v[k];
        packed = packed && aligned16(v[k]);
      }
    if (m <= 4)
      dots_against_kernel<T, 4><<<RED_BLOCKS, RED_THREADS, 0, s>>>(w, L, m, n, out, red, packed);
    else if (m <= 8)
      dots_against_kernel<T, 8><<<RED_BLOCKS, RED_THREADS, 0, s>>>(w, L, m, n, out, red, packed);
    else if (m <= 16)
      dots_against_kernel<T, 16><<<RED_BLOCKS, RED_THREADS, 0, s>>>(w, L, m, n, out, red, packed);
    else
      dots_against_kernel<T, MAXV><<<RED_BLOCKS, RED_THREADS, 0, s>>>(w, L, m, n, out, red, packed);
    return cudaGetLastError();
  }
  template <typename T>
  cudaError_t
  vec_orth_update(T *w, const T *const *v, const double *h, int m, long long n, double *out, Reducer red,
                  cudaStream_t s)
  {
    if (m < 1 || m > MAXV)
      return cudaErrorInvalidValue;
    VecList<T> L{};
    int        packed = aligned16(w);
    for (int k = 0; k < m; ++k)
      {
        L.v[k] = v[k];
        packed = packed && aligned16(v[k]);
      }
    if (m <= 4)
      orth_update_kernel<T, 4><<<RED_BLOCKS, RED_THREADS, 0, s>>>(w, L, h, m, n, out, red, packed);
    else if (m <= 8)
      orth_update_kernel<T, 8><<<RED_BLOCKS, RED_THREADS, 0, s>>>(w, L, h, m, n, out, red, packed);
    else if (m <= 16)
      orth_update_kernel<T, 16><<<RED_BLOCKS, RED_THREADS, 0, s>>>(w, L, h, m, n, out, red, packed);
    else
      orth_update_kernel<T, MAXV><<<RED_BLOCKS, RED_THREADS, 0, s>>>(w, L, h, m, n, out, red, packed);
    return cudaGetLastError();
  }
  template <typename T>
  cudaError_t
  vec_invert(T *d, double thr, long long n, cudaStream_t s)
  {
    invert_kernel<T><<<stream_blocks(n), 256, 0, s>>>(d, (T)thr, n);
    return cudaGetLastError();
  }
  template <typename T>
  cudaError_t
  vec_absmax(const T *d, long long n, double *out, Reducer red, cudaStream_t s)
  {
    absmax_kernel<T><<<RED_BLOCKS, RED_THREADS, 0, s>>>(d, n, out, red);
    return cudaGetLastError();
  }
  template <typename T>
  cudaError_t
  vec_invert_rel(T *d, const double *amax, long long n, cudaStream_t s)
  {
    invert_rel_kernel<T><<<stream_blocks(n), 256, 0, s>>>(d, amax, n);
    return cudaGetLastError();
  }
  template <typename T>
  cudaError_t
  vec_copy_constrained(T *dst, const T *src, const GridDesc &g, cudaStream_t s)
  {
    const long long n = (long long)g.n[0] * g.n[1] * g.n[2];
    copy_constrained_kernel<T><<<stream_blocks(n), 256, 0, s>>>(dst, src, g);
    return cudaGetLastError();
  }

  template <typename T>
  cudaError_t
  vec_distribute_constrained(T *dst, const T *src, const GridDesc &g, cudaStream_t s)
  {
    const long long n = (long long)g.n[0] * g.n[1] * g.n[2];
    distribute_constrained_kernel<T><<<stream_blocks(n), 256, 0, s>>>(dst, src, g);
    return cudaGetLastError();
  }

  template <typename T>
  cudaError_t
  vec_set_constrained(T *x, T v, const GridDesc &g, cudaStream_t s)
  {
    const long long n = (long long)g.n[0] * g.n[1] * g.n[2];
    set_constrained_kernel<T><<<stream_blocks(n), 256, 0, s>>>(x, v, g);
    return cudaGetLastError();
  }

  // ---- indexed operations over a DoF list (inflow rows of the advection operator)
  template <typename T>
  __global__ void
  idx_add_scaled_kernel(T *dst, const T *src, const long long *idx, long long n, T scale)
  {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
      {
        const long long i = idx[k];
        dst[i] += scale * src[i];
      }
  }
  template <typename T>
  __global__ void
  idx_set_kernel(T *dst, const long long *idx, const double *vals, long long n, T fill)
  {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
      dst[idx[k]] = vals ? (T)vals[k] : fill;
  }
  __global__ void
  idx_gather_kernel(double *out, const double *src, const long long *idx, long long n)
  {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
      out[k] = src[idx[k]];
  }

  template <typename T>
  cudaError_t
  idx_add_scaled(T *dst, const T *src, const long long *idx, long long n, double scale, cudaStream_t s)
  {
    if (n <= 0)
      return cudaSuccess;
    idx_add_scaled_kernel<T><<<stream_blocks(n), 256, 0, s>>>(dst, src, idx, n, (T)scale);
    return cudaGetLastError();
  }
  template <typename T>
  cudaError_t
  idx_set(T *dst, const long long *idx, const double *vals, long long n, T fill, cudaStream_t s)
  {
    if (n <= 0)
      return cudaSuccess;
    idx_set_kernel<T><<<stream_blocks(n), 256, 0, s>>>(dst, idx, vals, n, fill);
    return cudaGetLastError();
  }
  cudaError_t
  idx_gather(double *out, const double *src, const long long *idx, long long n, cudaStream_t s)
  {
    if (n <= 0)
      return cudaSuccess;
    idx_gather_kernel<<<stream_blocks(n), 256, 0, s>>>(out, src, idx, n);
    return cudaGetLastError();
  }

#define MPDG_INST(T)                                                                                         \
  template cudaError_t idx_add_scaled<T>(T *, const T *, const long long *, long long, double, cudaStream_t); \
  template cudaError_t idx_set<T>(T *, const long long *, const double *, long long, T, cudaStream_t);       \
  template cudaError_t cg_init<T>(const T *, const T *, T *, CGState *, double *, Reducer, long long, cudaStream_t); \
  template cudaError_t cg_update_p<T>(const T *, const T *, T *, const CGState *, long long, cudaStream_t);      \
  template cudaError_t cg_alpha<T>(const T *, const T *, CGState *, Reducer, long long, cudaStream_t);          \
  template cudaError_t cg_update_xr<T>(T *, T *, const T *, const T *, const T *, CGState *, double *, Reducer,  \
                                       long long, cudaStream_t);                                                \
  template cudaError_t vec_fill<T>(T *, T, long long, cudaStream_t);                                            \
  template cudaError_t vec_axpby<T>(T *, double, const T *, double, const T *, long long, cudaStream_t);        \
  template cudaError_t vec_multidot<T>(const T *const *, const T *const *, int, long long, double *, Reducer,    \
                                       cudaStream_t);                                                           \
  template cudaError_t vec_scale<T>(T *, const T *, const T *, long long, cudaStream_t);                        \
  template cudaError_t vec_multiaxpy<T>(T *, const T *const *, const double *, int, long long, double,          \
                                        cudaStream_t);                                                          \
  template cudaError_t vec_dots_against<T>(const T *, const T *const *, int, long long, double *, Reducer,       \
                                           cudaStream_t);                                                       \
  template cudaError_t vec_orth_update<T>(T *, const T *const *, const double *, int, long long, double *,      \
                                          Reducer, cudaStream_t);                                               \
  template cudaError_t vec_invert<T>(T *, double, long long, cudaStream_t);                                     \
  template cudaError_t vec_absmax<T>(const T *, long long, double *, Reducer, cudaStream_t);                    \
  template cudaError_t vec_invert_rel<T>(T *, const double *, long long, cudaStream_t);                         \
  template cudaError_t vec_set_constrained<T>(T *, T, const GridDesc &, cudaStream_t);                            \
  template cudaError_t vec_copy_constrained<T>(T *, const T *, const GridDesc &, cudaStream_t);             \
  template cudaError_t vec_distribute_constrained<T>(T *, const T *, const GridDesc &, cudaStream_t);
  MPDG_INST(double)
  MPDG_INST(float)
#undef MPDG_INST
  template cudaError_t vec_convert<float, double>(float *, const double *, long long, cudaStream_t);
  template cudaError_t vec_convert<double, float>(double *, const float *, long long, cudaStream_t);
} // namespace mpdg
