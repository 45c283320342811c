// Heat operator kernels: matrix-free apply (fast diagonalisation, see sumfac.cuh) and the
// DoF-parallel diagonal.  Reference: source/heat/heat_diffuse_operator.cpp
//   vmult                      :179-197  (MatrixFree::loop, zero_dst = true)
//   tangent_local_cell_operation :1029-1079 (val = rho c_p/dt u, grad = k grad u)
//   compute_inverse_diagonal_from_matrixfree :271-284 (|d| > 1e-10 ? 1/d : 1)
//
// Work decomposition: one CTA per brick of cells (brick.cuh).  For k <= 2 one thread holds a whole
// cell (n^3 <= 27 values) in registers.  For k >= 3 a cell is split over two threads in different
// warps by the reflection parity of its z-modes: the "odd" thread transforms the floor(n/2) odd
// z-planes (u_l - u_{n-1-l}), the "even" thread the ceil(n/2) even z-planes (u_l + u_{n-1-l},
// u_mid); each adds its part of the nodal output (out_l = E_l + O_l, out_{n-1-l} = E_l - O_l).
// Cells add their outputs into a shared-memory accumulator of the brick with shared-memory atomics
// (no ordering between cells that share lattice points is needed).
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>
#include <set>

#include "brick.cuh"
#include "kernels.h"
#include "march.cuh"
#include "pencil.cuh"
#include "sumfac.cuh"

namespace mpdg
{
  // 1-D fast-diagonalisation tables per degree in constant memory (uploaded once per device):
  // [WE (ne*ne) | WO (no*no) | lambda (n)]
  constexpr int FD_TAB = 32;
  __constant__ double c_fd_d[5][FD_TAB];
  __constant__ float  c_fd_f[5][FD_TAB];

  template <typename T>
  __device__ __forceinline__ const T *
  fd_table(int K)
  {
    if constexpr (sizeof(T) == 8)
      return c_fd_d[K];
    else
      return c_fd_f[K];
  }

  template <typename T, int N>
  struct HeatArgs
  {
    T          cx, cy, cz; // stiffness geometry factors (hy hz / hx, ...)
    GridDesc   g;
    SyncDesc   s;
    T          alpha;  // scale * rho c_p / dt * hx hy hz
    T          kscale; // scale (multiplies the conductivity)
    T          kconst; // conductivity when kcell == nullptr
    const T   *kcell;  // per-cell conductivity
    const T   *src;
    T         *dst;
    const T   *b;      // BPlus mode: dst = b + A src (may alias dst)
    int        mask_src;
    const int *skip;   // return at once when *skip != 0 (a solve has finished)
    DotSink    dot;    // fused src^T A src (CG step length), see brick.cuh
  };

  template <int K, typename T>
  struct HeatBrickShape;
  template <typename T>
  struct HeatBrickShape<1, T>
  {
    static constexpr int BX = 8, BY = 8, BZ = 4;
  };
  template <typename T>
  struct HeatBrickShape<2, T>
  {
    static constexpr int BX = 8, BY = 8, BZ = 4;
  };
  template <typename T>
  struct HeatBrickShape<3, T>
  {
    static constexpr int BX = 4, BY = 4, BZ = 4;
  };
  template <typename T>
  struct HeatBrickShape<4, T>
  {
    static constexpr int BX = 4, BY = 4, BZ = 4;
  };

  template <int K, typename T>
  struct HeatLayout
  {
    static constexpr int  N = K + 1, NE = (N + 1) / 2, NO = N / 2;
    using S                 = HeatBrickShape<K, T>;
    static constexpr bool TWO = (N >= 4);
    static constexpr int  NC  = S::BX * S::BY * S::BZ;
    static constexpr int  NT  = TWO ? 2 * NC : NC;
    using BR                  = Brick<K, S::BX, S::BY, S::BZ, NT>;
    static constexpr size_t bytes = sizeof(T) * 2 * (size_t)BR::NPTS; // staged input + accumulator
  };

  template <int K, typename T, OutMode MODE>
  __global__ void __launch_bounds__(HeatLayout<K, T>::NT)
  heat_apply_kernel(const __grid_constant__ HeatArgs<T, K + 1> a)
  {
    using L          = HeatLayout<K, T>;
    using BR         = typename L::BR;
    constexpr int N  = K + 1, NE = L::NE, NO = L::NO;
    constexpr int NC = L::NC, PX = BR::PX, PY = BR::PY;
    constexpr int BX = BR::BX, BY = BR::BY;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *const s_src = reinterpret_cast<T *>(smem_raw); // staged input brick
    T *const s_dst = s_src + BR::NPTS;                // brick accumulator
    __shared__ unsigned s_ticket;
    if (a.skip != nullptr && *a.skip != 0)
      return;

    BR br;
    if (!brick_begin<BR, T, MODE>(br, a.g, a.s, a.dst, a.b, &s_ticket))
      return;
    for (int p = threadIdx.x; p < BR::NPTS; p += BR::NT)
      s_dst[p] = T(0);
    brick_stage(br, a.src, a.mask_src != 0, s_src);

    const int  cell = threadIdx.x % NC;       // cell of the brick handled by this thread
    const int  role = threadIdx.x / NC;       // 0: whole cell / even z-modes, 1: odd z-modes
    const int  tx = cell % BX, ty = (cell / BX) % BY, tz = cell / (BX * BY);
    const int  cx = br.c0[0] + tx, cy = br.c0[1] + ty, cz = br.c0[2] + tz;
    const bool valid = cx < a.g.m[0] && cy < a.g.m[1] && cz < a.g.m[2];
    const int  base = (K * tz) * PY * PX + (K * ty) * PX + K * tx;
    T          kc   = T(0);
    if (valid)
      {
        const long long c = (long long)cx + (long long)a.g.m[0] * ((long long)cy + (long long)a.g.m[1] * cz);
        kc                = a.kscale * (a.kcell ? a.kcell[c] : a.kconst);
      }
    const T  alpha = a.alpha;
    const T *tb    = fd_table<T>(K);
    const T *we    = tb;
    const T *wo    = tb + NE * NE;
    const T *lam   = tb + NE * NE + NO * NO;
    const T  kcx = kc * a.cx, kcy = kc * a.cy, kcz = kc * a.cz;
    // multiply P modal planes (modal z index z0 + c) by alpha + k_c (cx lam_a + cy lam_b + cz lam_c)
    auto scale_planes = [&](T *v, const int P, const int z0) {
#pragma unroll
      for (int c = 0; c < N; ++c)
        if (c < P)
          {
            const T tz = fma(kcz, lam[z0 + c], alpha);
#pragma unroll
            for (int b = 0; b < N; ++b)
              {
                const T tyz = fma(kcy, lam[b], tz);
#pragma unroll
                for (int aa = 0; aa < N; ++aa)
                  v[(c * N + b) * N + aa] *= fma(kcx, lam[aa], tyz);
              }
          }
    };
    // cells sharing a lattice point add into the brick accumulator concurrently
    auto add_point = [&](const int i, const int j, const int l, const T v) {
      atomicAdd(s_dst + (base + l * PY * PX + j * PX + i), v);
    };

    if (valid)
      {
        if constexpr (!L::TWO)
          {
            T u[N * N * N];
#pragma unroll
            for (int l = 0; l < N; ++l)
#pragma unroll
              for (int j = 0; j < N; ++j)
#pragma unroll
                for (int i = 0; i < N; ++i)
                  u[(l * N + j) * N + i] = s_src[base + l * PY * PX + j * PX + i];
            xy_planes<T, N, N, true>(u, we, wo);
#pragma unroll
            for (int q = 0; q < N * N; ++q)
              fwd_line<T, N, N * N>(u, q, we, wo);
            scale_planes(u, N, 0);
#pragma unroll
            for (int q = 0; q < N * N; ++q)
              bwd_line<T, N, N * N>(u, q, we, wo);
            xy_planes<T, N, N, false>(u, we, wo);
#pragma unroll
            for (int l = 0; l < N; ++l)
#pragma unroll
              for (int j = 0; j < N; ++j)
#pragma unroll
                for (int i = 0; i < N; ++i)
                  add_point(i, j, l, u[(l * N + j) * N + i]);
          }
        else if (role == 1)
          {
            // odd z-modes: o_k = u_k - u_{N-1-k}; the result O_k adds +O_k to plane k and -O_k to
            // plane N-1-k of the nodal output
            T v[NO * N * N];
#pragma unroll
            for (int k = 0; k < NO; ++k)
#pragma unroll
              for (int j = 0; j < N; ++j)
#pragma unroll
                for (int i = 0; i < N; ++i)
                  v[(k * N + j) * N + i] = s_src[base + k * PY * PX + j * PX + i] -
                                           s_src[base + (N - 1 - k) * PY * PX + j * PX + i];
#pragma unroll
            for (int q = 0; q < N * N; ++q)
              {
                T t[NO];
#pragma unroll
                for (int m = 0; m < NO; ++m)
                  {
                    T s = wo[m * NO] * v[q];
#pragma unroll
                    for (int k = 1; k < NO; ++k)
                      s = fma(wo[m * NO + k], v[k * N * N + q], s);
                    t[m] = s;
                  }
#pragma unroll
                for (int m = 0; m < NO; ++m)
                  v[m * N * N + q] = t[m];
              }
            xy_planes<T, N, NO, true>(v, we, wo);
            scale_planes(v, NO, NE);
            xy_planes<T, N, NO, false>(v, we, wo);
#pragma unroll
            for (int q = 0; q < N * N; ++q)
              {
                T t[NO];
#pragma unroll
                for (int k = 0; k < NO; ++k)
                  {
                    T s = wo[k] * v[q];
#pragma unroll
                    for (int m = 1; m < NO; ++m)
                      s = fma(wo[m * NO + k], v[m * N * N + q], s);
                    t[k] = s;
                  }
#pragma unroll
                for (int k = 0; k < NO; ++k)
                  {
                    add_point(q % N, q / N, k, t[k]);
                    add_point(q % N, q / N, N - 1 - k, -t[k]);
                  }
              }
          }
        else
          {
            // even z-modes: e_k = u_k + u_{N-1-k}, e_mid = u_mid; E_k goes to planes k and N-1-k
            T e[NE * N * N];
#pragma unroll
            for (int k = 0; k < NE; ++k)
#pragma unroll
              for (int j = 0; j < N; ++j)
#pragma unroll
                for (int i = 0; i < N; ++i)
                  {
                    const T lo = s_src[base + k * PY * PX + j * PX + i];
                    e[(k * N + j) * N + i] =
                      (k < N / 2) ? lo + s_src[base + (N - 1 - k) * PY * PX + j * PX + i] : lo;
                  }
#pragma unroll
            for (int q = 0; q < N * N; ++q)
              {
                T t[NE];
#pragma unroll
                for (int m = 0; m < NE; ++m)
                  {
                    T s = we[m * NE] * e[q];
#pragma unroll
                    for (int k = 1; k < NE; ++k)
                      s = fma(we[m * NE + k], e[k * N * N + q], s);
                    t[m] = s;
                  }
#pragma unroll
                for (int m = 0; m < NE; ++m)
                  e[m * N * N + q] = t[m];
              }
            xy_planes<T, N, NE, true>(e, we, wo);
            scale_planes(e, NE, 0);
            xy_planes<T, N, NE, false>(e, we, wo);
#pragma unroll
            for (int q = 0; q < N * N; ++q)
              {
                T t[NE];
#pragma unroll
                for (int k = 0; k < NE; ++k)
                  {
                    T s = we[k] * e[q];
#pragma unroll
                    for (int m = 1; m < NE; ++m)
                      s = fma(we[m * NE + k], e[m * N * N + q], s);
                    t[k] = s;
                  }
#pragma unroll
                for (int k = 0; k < NE; ++k)
                  {
                    add_point(q % N, q / N, k, t[k]);
                    if (k < N / 2)
                      add_point(q % N, q / N, N - 1 - k, t[k]);
                  }
              }
          }
      }
    __syncthreads();
    brick_end<BR, T, MODE>(br, a.g, a.s, s_dst, a.dst, a.b);
  }

  // ---- k <= 2: column-marching apply (march.cuh) with the fast-diagonalisation cell operator
  template <int K, typename T>
  struct HeatCellOp
  {
    static constexpr int N = K + 1, NE = (N + 1) / 2, NO = N / 2;
    const HeatArgs<T, N> &a;
    template <bool DOT>
    __device__ __forceinline__ double
    apply(T *u, bool valid, int cx, int cy, int cz) const
    {
      T form = T(0);
      T kc = T(0);
      if (valid)
        {
          const long long c = (long long)cx + (long long)a.g.m[0] * ((long long)cy + (long long)a.g.m[1] * cz);
          kc                = a.kscale * (a.kcell ? a.kcell[c] : a.kconst);
        }
      const T *tb  = fd_table<T>(K);
      const T *we  = tb;
      const T *wo  = tb + NE * NE;
      const T *lam = tb + NE * NE + NO * NO;
      const T  kcx = kc * a.cx, kcy = kc * a.cy, kcz = kc * a.cz, alpha = a.alpha;
      xy_planes<T, N, N, true>(u, we, wo);
#pragma unroll
      for (int q = 0; q < N * N; ++q)
        fwd_line<T, N, N * N>(u, q, we, wo);
#pragma unroll
      for (int c = 0; c < N; ++c)
        {
          const T tz = fma(kcz, lam[c], alpha);
#pragma unroll
          for (int b = 0; b < N; ++b)
            {
              const T tyz = fma(kcy, lam[b], tz);
#pragma unroll
              for (int aa = 0; aa < N; ++aa)
                {
                  const T d = fma(kcx, lam[aa], tyz);
                  T      &v = u[(c * N + b) * N + aa];
                  if constexpr (DOT)
                    form = fma(d * v, v, form);
                  v *= d;
                }
            }
        }
#pragma unroll
      for (int q = 0; q < N * N; ++q)
        bwd_line<T, N, N * N>(u, q, we, wo);
      xy_planes<T, N, N, false>(u, we, wo);
      return (double)form;
    }
  };

#ifndef MPDG_MARCH_MINB_F64
#define MPDG_MARCH_MINB_F64 5
#endif
#ifndef MPDG_MARCH_MINB_F32
#define MPDG_MARCH_MINB_F32 8
#endif
  // CTAs per SM the register allocation of the column-marching kernel is held to
  template <typename T>
  struct MarchMinBlocks
  {
    static constexpr int value = sizeof(T) == 8 ? MPDG_MARCH_MINB_F64 : MPDG_MARCH_MINB_F32;
  };

  template <int K, typename T, OutMode MODE, bool DOT>
  __global__ void __launch_bounds__(MarchShape<K, T>::NT, MarchMinBlocks<T>::value)
  heat_march_kernel(const __grid_constant__ HeatArgs<T, K + 1> a)
  {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned s_ticket;
    __shared__ double   s_red[MarchShape<K, T>::NT / 32];
    if (a.skip != nullptr && *a.skip != 0)
      return;
    HeatCellOp<K, T> op{a};
    march_body<K, T, MODE, HeatCellOp<K, T>, DOT>(a.g, a.s, a.src, a.dst, a.b, a.mask_src != 0, op,
                                                  reinterpret_cast<T *>(smem_raw), &s_ticket, a.dot, s_red);
  }

  // ---- k >= 3: pencil-marching apply (pencil.cuh); the x lines are scaled by the diagonal of the
  // fast-diagonalisation basis, a + k_c (cx lam_a + cy lam_b + cz lam_c)
  template <int K, typename T>
  struct HeatPencilOp
  {
    static constexpr int N = K + 1, NE = (N + 1) / 2, NO = N / 2;
    const HeatArgs<T, N> &a;
    __device__ __forceinline__ const T *
    we() const
    {
      return fd_table<T>(K);
    }
    __device__ __forceinline__ const T *
    wo() const
    {
      return fd_table<T>(K) + NE * NE;
    }
    __device__ __forceinline__ const T *
    lam() const
    {
      return fd_table<T>(K) + NE * NE + NO * NO;
    }
    __device__ __forceinline__ T
    alpha() const
    {
      return a.alpha;
    }
    __device__ __forceinline__ T
    cxg() const
    {
      return a.cx;
    }
    __device__ __forceinline__ T
    cyg() const
    {
      return a.cy;
    }
    __device__ __forceinline__ T
    czg() const
    {
      return a.cz;
    }
    // scaled conductivity of cell (cx, cy, cz)
    __device__ __forceinline__ T
    kcell(int cx, int cy, int cz) const
    {
      const long long cell = (long long)cx + (long long)a.g.m[0] * ((long long)cy + (long long)a.g.m[1] * cz);
      return a.kscale * (a.kcell ? a.kcell[cell] : a.kconst);
    }
    // unscaled per-cell conductivity (nullptr: the constant kconst()) and the scale applied to it
    __device__ __forceinline__ const T *
    kcell_ptr(int cx, int cy, int cz) const
    {
      const long long cell = (long long)cx + (long long)a.g.m[0] * ((long long)cy + (long long)a.g.m[1] * cz);
      return a.kcell ? a.kcell + cell : nullptr;
    }
    __device__ __forceinline__ T
    kconst() const
    {
      return a.kconst;
    }
    __device__ __forceinline__ T
    kscale() const
    {
      return a.kscale;
    }
  };

  template <int K, typename T, OutMode MODE, bool DOT>
  __global__ void __launch_bounds__(PencilShape<K>::NT, PencilShape<K>::MINB)
  heat_pencil_kernel(const __grid_constant__ HeatArgs<T, K + 1> a)
  {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned s_ticket;
    __shared__ double   s_red[PencilShape<K>::NT / 32];
    if (a.skip != nullptr && *a.skip != 0)
      return;
    HeatPencilOp<K, T> op{a};
    pencil_body<K, T, MODE, HeatPencilOp<K, T>, DOT>(a.g, a.s, a.src, a.dst, a.b, a.mask_src != 0, op,
                                                     reinterpret_cast<T *>(smem_raw), &s_ticket, a.dot, s_red);
  }

  // ---- diagonal: closed-form per-cell entries gathered per DoF (deterministic, no atomics)
  template <typename T>
  struct DiagArgs
  {
    GridDesc g;
    int      K;
    T        alpha, cx, cy, cz; // mass coefficient and stiffness geometry factors
    T        kconst;
    const T *kcell;
    T        mdiag[8], kdiag[8]; // 1-D M_ii, K_ii
    T        threshold;          // |d| > threshold ? 1/d : 1
    T       *diag;
    int      invert;
  };

  // One CTA per lattice row (J, L) in a grid-stride loop, threads along x (coalesced stores); the
  // diagonal entry is the sum over the (up to 8) cells sharing the point of the tensor-product form
  // a Mx My Mz + k_c (cx Kx My Mz + cy Mx Ky Mz + cz Mx My Kz) at the point's local indices.
  template <int K, typename T>
  __global__ void
  heat_diag_kernel(const __grid_constant__ DiagArgs<T> a)
  {
    const int       n0 = a.g.n[0], n1 = a.g.n[1];
    const long long rows = (long long)n1 * a.g.n[2];
    for (long long row = blockIdx.x; row < rows; row += gridDim.x)
      {
        const int        J = (int)(row % n1), L = (int)(row / n1);
        const Neighbours1D<K> ny(J, a.g.m[1]), nz(L, a.g.m[2]);
        const bool rowcon = ((a.g.faces & 4u) && J == 0) || ((a.g.faces & 8u) && J == n1 - 1) ||
                            ((a.g.faces & 16u) && L == 0) || ((a.g.faces & 32u) && L == a.g.n[2] - 1);
        for (int I = threadIdx.x; I < n0; I += blockDim.x)
          {
            const long long idx = (long long)I + (long long)n0 * row;
            bool con = rowcon || ((a.g.faces & 1u) && I == 0) || ((a.g.faces & 2u) && I == n0 - 1);
            if (a.g.cmask != nullptr && a.g.cmask[idx] != 0)
              con = true;
            T d = T(0);
            if (!con)
              {
                const Neighbours1D<K> nx(I, a.g.m[0]);
#pragma unroll
                for (int z = 0; z < 2; ++z)
#pragma unroll
                  for (int y = 0; y < 2; ++y)
#pragma unroll
                    for (int x = 0; x < 2; ++x)
                      if (nx.v[x] && ny.v[y] && nz.v[z])
                        {
                          const long long cell = (long long)nx.c[x] +
                                                 (long long)a.g.m[0] * ((long long)ny.c[y] + (long long)a.g.m[1] * nz.c[z]);
                          const T kc = a.kcell ? a.kcell[cell] : a.kconst;
                          const T mx = a.mdiag[nx.l[x]], my = a.mdiag[ny.l[y]], mz = a.mdiag[nz.l[z]];
                          const T kx = a.kdiag[nx.l[x]], ky = a.kdiag[ny.l[y]], kz = a.kdiag[nz.l[z]];
                          d += a.alpha * mx * my * mz + kc * (a.cx * kx * my * mz + a.cy * mx * ky * mz + a.cz * mx * my * kz);
                        }
              }
            else
              d = T(1);
            if (a.invert && !con)
              d = (fabs(d) > a.threshold) ? T(1) / d : T(1);
            a.diag[idx] = d;
          }
      }
  }

  // ------------------------------------------------------------------------------------------
  // host launchers

  // Upload the 1-D tables of every degree once per device.
  static cudaError_t
  upload_fd_tables()
  {
    static std::mutex          mtx;
    static std::set<int>       done;
    int                        dev = 0;
    cudaError_t                e   = cudaGetDevice(&dev);
    if (e != cudaSuccess)
      return e;
    std::lock_guard<std::mutex> lock(mtx);
    if (done.count(dev))
      return cudaSuccess;
    double hd[5][FD_TAB] = {};
    float  hf[5][FD_TAB] = {};
    for (int K = 1; K <= 4; ++K)
      {
        const Tables1D &t = tables(K);
        int             o = 0;
        for (int i = 0; i < t.ne * t.ne; ++i)
          hd[K][o++] = t.WE[i];
        for (int i = 0; i < t.no * t.no; ++i)
          hd[K][o++] = t.WO[i];
        for (int i = 0; i < t.n; ++i)
          hd[K][o++] = t.lam[i];
        for (int i = 0; i < o; ++i)
          hf[K][i] = (float)hd[K][i];
      }
    if ((e = cudaMemcpyToSymbol(c_fd_d, hd, sizeof(hd))) != cudaSuccess)
      return e;
    if ((e = cudaMemcpyToSymbol(c_fd_f, hf, sizeof(hf))) != cudaSuccess)
      return e;
    // the copies ran on the legacy stream: complete them before kernels on other streams read the tables
    if ((e = cudaStreamSynchronize(cudaStreamLegacy)) != cudaSuccess)
      return e;
    done.insert(dev);
    return cudaSuccess;
  }

  template <int K, typename T, OutMode MODE>
  static cudaError_t
  launch_apply(const HeatLaunch<T> &h, cudaStream_t stream)
  {
    using L = HeatLayout<K, T>;
    HeatArgs<T, K + 1> a;
    cudaError_t        ue = upload_fd_tables();
    if (ue != cudaSuccess)
      return ue;
    a.cx       = (T)h.geo.cx;
    a.cy       = (T)h.geo.cy;
    a.cz       = (T)h.geo.cz;
    a.g        = h.grid;
    a.s        = h.sync;
    a.alpha    = (T)(h.scale * h.geo.mass_coef);
    a.kscale   = (T)h.scale;
    a.kconst   = (T)h.kconst;
    a.kcell    = h.kcell;
    a.src      = h.src;
    a.dst      = h.dst;
    a.b        = h.b;
    a.mask_src = h.mask_src;
    a.skip     = h.skip;
    a.dot      = h.dot;
    const unsigned nbricks = (unsigned)h.grid.nbr[0] * h.grid.nbr[1] * h.grid.nbr[2];
    if constexpr (K <= 2)
      if (h.grid.cmask == nullptr && h.march)
        {
          using ML = MarchLayout<K, T>;
          static std::atomic<unsigned long long> dev_plain{0}, dev_dot{0};
          if constexpr (MODE == OutMode::Set)
            if (h.dot.part != nullptr)
              {
                auto        kern = heat_march_kernel<K, T, MODE, true>;
                cudaError_t e    = ensure_smem(kern, ML::bytes, dev_dot);
                if (e != cudaSuccess)
                  return e;
                kern<<<nbricks, ML::S::NT, ML::bytes, stream>>>(a);
                return cudaGetLastError();
              }
          auto        kern = heat_march_kernel<K, T, MODE, false>;
          cudaError_t e    = ensure_smem(kern, ML::bytes, dev_plain);
          if (e != cudaSuccess)
            return e;
          kern<<<nbricks, ML::S::NT, ML::bytes, stream>>>(a);
          return cudaGetLastError();
        }
    if constexpr (K >= 3)
      if (h.grid.cmask == nullptr && h.march)
        {
          using PL = PencilLayout<K, T>;
          static std::atomic<unsigned long long> dev_plain{0}, dev_dot{0};
          if constexpr (MODE == OutMode::Set)
            if (h.dot.part != nullptr)
              {
                auto        kern = heat_pencil_kernel<K, T, MODE, true>;
                cudaError_t e    = ensure_smem(kern, PL::bytes, dev_dot);
                if (e != cudaSuccess)
                  return e;
                kern<<<nbricks, PL::S::NT, PL::bytes, stream>>>(a);
                return cudaGetLastError();
              }
          auto        kern = heat_pencil_kernel<K, T, MODE, false>;
          cudaError_t e    = ensure_smem(kern, PL::bytes, dev_plain);
          if (e != cudaSuccess)
            return e;
          kern<<<nbricks, PL::S::NT, PL::bytes, stream>>>(a);
          return cudaGetLastError();
        }
    if (h.dot.part != nullptr)
      return cudaErrorInvalidValue; // the brick kernel has no fused dot (heat_apply_fuses_dot is false)
    {
        auto                                   kern = heat_apply_kernel<K, T, MODE>;
        static std::atomic<unsigned long long> dev_brick{0};
        cudaError_t                            e = ensure_smem(kern, L::bytes, dev_brick);
        if (e != cudaSuccess)
          return e;
        kern<<<nbricks, L::BR::NT, L::bytes, stream>>>(a);
      }
    return cudaGetLastError();
  }

  template <typename T>
  static void
  brick_shape(int K, int &bx, int &by, int &bz)
  {
    switch (K)
      {
        case 1: bx = MarchShape<1, T>::BX; by = MarchShape<1, T>::BY; bz = MarchShape<1, T>::BZ; break;
        case 2: bx = MarchShape<2, T>::BX; by = MarchShape<2, T>::BY; bz = MarchShape<2, T>::BZ; break;
        case 3: bx = HeatBrickShape<3, T>::BX; by = HeatBrickShape<3, T>::BY; bz = HeatBrickShape<3, T>::BZ; break;
        default: bx = HeatBrickShape<4, T>::BX; by = HeatBrickShape<4, T>::BY; bz = HeatBrickShape<4, T>::BZ; break;
      }
  }

  template <typename T>
  void
  heat_brick_shape(int K, int shape[3], bool march)
  {
    brick_shape<T>(K, shape[0], shape[1], shape[2]);
    if (march && K >= 3)
      {
        shape[0] = PencilShape<3>::BX;
        shape[1] = PencilShape<3>::BY;
        shape[2] = PencilShape<3>::BZ;
        static_assert(PencilShape<3>::BX == PencilShape<4>::BX && PencilShape<3>::BY == PencilShape<4>::BY &&
                        PencilShape<3>::BZ == PencilShape<4>::BZ,
                      "one pencil brick shape for k = 3, 4");
      }
    if (!march && K <= 2)
      {
        shape[0] = K == 1 ? HeatBrickShape<1, T>::BX : HeatBrickShape<2, T>::BX;
        shape[1] = K == 1 ? HeatBrickShape<1, T>::BY : HeatBrickShape<2, T>::BY;
        shape[2] = K == 1 ? HeatBrickShape<1, T>::BZ : HeatBrickShape<2, T>::BZ;
      }
  }

  template <int K, typename T>
  static cudaError_t
  dispatch_mode(const HeatLaunch<T> &h, cudaStream_t s)
  {
    switch (h.mode)
      {
        case 0: return launch_apply<K, T, OutMode::Set>(h, s);
        case 1: return launch_apply<K, T, OutMode::Add>(h, s);
        default: return launch_apply<K, T, OutMode::BPlus>(h, s);
      }
  }

  bool
  heat_apply_fuses_dot(int K, bool has_dof_mask, bool march)
  {
    return K >= 1 && K <= 4 && !has_dof_mask && march;
  }

  template <typename T>
  cudaError_t
  heat_apply(const HeatLaunch<T> &h, cudaStream_t s)
  {
    switch (h.degree)
      {
        case 1: return dispatch_mode<1, T>(h, s);
        case 2: return dispatch_mode<2, T>(h, s);
        case 3: return dispatch_mode<3, T>(h, s);
        case 4: return dispatch_mode<4, T>(h, s);
        default: return cudaErrorInvalidValue;
      }
  }

  template <typename T>
  cudaError_t
  heat_diagonal(const GridDesc &g, int K, const HeatGeom &geo, double kconst, const T *kcell, T *diag,
                bool invert, double threshold, cudaStream_t s)
  {
    if (K < 1 || K > 7)
      return cudaErrorInvalidValue;
    DiagArgs<T>     a;
    const Tables1D &t = tables(K);
    a.g               = g;
    a.K               = K;
    a.alpha           = (T)geo.mass_coef;
    a.cx              = (T)geo.cx;
    a.cy              = (T)geo.cy;
    a.cz              = (T)geo.cz;
    a.kconst          = (T)kconst;
    a.kcell           = kcell;
    for (int i = 0; i < 8; ++i)
      {
        a.mdiag[i] = i <= K ? (T)t.M[i * t.n + i] : T(0);
        a.kdiag[i] = i <= K ? (T)t.K[i * t.n + i] : T(0);
      }
    a.threshold = (T)threshold;
    a.diag      = diag;
    a.invert    = invert ? 1 : 0;
    const long long rows    = (long long)g.n[1] * g.n[2];
    const int       blocks  = (int)std::min<long long>(rows, 148LL * 32);
    const int       threads = std::min(1024, std::max(32, (g.n[0] + 31) / 32 * 32));
    switch (K)
      {
        case 1: heat_diag_kernel<1, T><<<blocks, threads, 0, s>>>(a); break;
        case 2: heat_diag_kernel<2, T><<<blocks, threads, 0, s>>>(a); break;
        case 3: heat_diag_kernel<3, T><<<blocks, threads, 0, s>>>(a); break;
        case 4: heat_diag_kernel<4, T><<<blocks, threads, 0, s>>>(a); break;
        default: return cudaErrorInvalidValue;
      }
    return cudaGetLastError();
  }

  template cudaError_t heat_apply<double>(const HeatLaunch<double> &, cudaStream_t);
  template cudaError_t heat_apply<float>(const HeatLaunch<float> &, cudaStream_t);
  template cudaError_t heat_diagonal<double>(const GridDesc &, int, const HeatGeom &, double, const double *, double *,
                                             bool, double, cudaStream_t);
  template cudaError_t heat_diagonal<float>(const GridDesc &, int, const HeatGeom &, double, const float *, float *,
                                            bool, double, cudaStream_t);
  template void heat_brick_shape<double>(int, int[3], bool);
  template void heat_brick_shape<float>(int, int[3], bool);
} // namespace mpdg
