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
#include <cuda_runtime.h>

#include <mutex>
#include <set>

#include "brick.cuh"
#include "kernels.h"
#include "sumfac.cuh"

namespace mpdg
{
  // Per degree (1, 2) in constant memory, uploaded once per device:
  //   [B (n*n): phi_i(x_q) | D (n*n): collocation derivative on the Gauss points |
  //    qp (n): Gauss points | qw3 (n^3): tensor Gauss weights]
  constexpr int ADV_TAB = 48;
  __constant__ double c_adv_d[3][ADV_TAB];
  __constant__ float  c_adv_f[3][ADV_TAB];

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

  template <int K, typename T>
  struct AdvLayout
  {
    static constexpr int  N  = K + 1;
    static constexpr int  BX = 8, BY = 8, BZ = (K == 1 ? 8 : 4);
    static constexpr int  NT = BX * BY * BZ;
    using BR                 = Brick<K, BX, BY, BZ, NT>;
    static constexpr size_t bytes = sizeof(T) * 2 * (size_t)BR::NPTS; // staged input + accumulator
  };

  template <int K, typename T, OutMode MODE>
  __global__ void __launch_bounds__(AdvLayout<K, T>::BR::NT)
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
    brick_stage(br, a.src, a.mask_src != 0, s_src);

    const int  tx = threadIdx.x % BX, ty = (threadIdx.x / BX) % BY, tz = threadIdx.x / (BX * BY);
    const int  cx = br.c0[0] + tx, cy = br.c0[1] + ty, cz = br.c0[2] + tz;
    const bool valid = cx < a.g.m[0] && cy < a.g.m[1] && cz < a.g.m[2];
    const int  base = (K * tz) * PY * PX + (K * ty) * PX + K * tx;

    const T *tb  = adv_table<T>(K);
    const T *tB  = tb, *tD = tb + N * N, *tqp = tb + 2 * N * N, *tw3 = tb + 2 * N * N + N;
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
        const T c_mass = a.det * a.inv_dt;
#pragma unroll
        for (int q = 0; q < N * N * N; ++q)
          R[q] = (tw3[q] * c_mass) * uq[q];
#pragma unroll
        for (int d = 0; d < 3; ++d)
          {
            T g[N * N * N];
#pragma unroll
            for (int q = 0; q < N * N * N; ++q)
              g[q] = uq[q];
            if (d == 0)
              sweep<T, N, 0, false>(g, tD);
            else if (d == 1)
              sweep<T, N, 1, false>(g, tD);
            else
              sweep<T, N, 2, false>(g, tD);
            const T inv_h = T(1) / a.h[d];
            const T c_g   = a.det * inv_h;
            const T vd0   = a.vel[d] + a.vel[3 + 3 * d] * x0 + a.vel[4 + 3 * d] * y0 + a.vel[5 + 3 * d] * z0;
            const T gx = a.vel[3 + 3 * d] * a.h[0], gy = a.vel[4 + 3 * d] * a.h[1], gz = a.vel[5 + 3 * d] * a.h[2];
#pragma unroll
            for (int qz = 0; qz < N; ++qz)
#pragma unroll
              for (int qy = 0; qy < N; ++qy)
#pragma unroll
                for (int qx = 0; qx < N; ++qx)
                  {
                    const int q  = (qz * N + qy) * N + qx;
                    const T   vd = vd0 + gx * tqp[qx] + gy * tqp[qy] + gz * tqp[qz];
                    const T   gw = g[q] * (c_g * tw3[q]);
                    R[q]         = fma(a.th_adv * vd, gw, R[q]);
                    g[q]         = a.th_dif * gw * inv_h;
                  }
            if (a.th_dif != T(0))
              {
                if (d == 0)
                  sweep_tr_acc<T, N, 0>(R, g, tD);
                else if (d == 1)
                  sweep_tr_acc<T, N, 1>(R, g, tD);
                else
                  sweep_tr_acc<T, N, 2>(R, g, tD);
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

  // ---- local diagonal entries per cell: A_c[ii] by quadrature (MatrixFreeTools::compute_diagonal)
  template <typename T, int N>
  struct AdvDiagArgs
  {
    T        B[N * N], G[N * N], qp[N], qw[N];
    T        inv_dt, th_adv, th_dif;
    T        vel[12], origin[3], h[3];
    int      m[3];
    T       *cellbuf; // ncells * N^3
  };

  template <typename T, int N>
  __global__ void
  adv_cell_diag_kernel(const __grid_constant__ AdvDiagArgs<T, N> a)
  {
    const long long ncells = (long long)a.m[0] * a.m[1] * a.m[2];
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncells; c += (long long)gridDim.x * blockDim.x)
      {
        const int cx = (int)(c % a.m[0]), cy = (int)((c / a.m[0]) % a.m[1]), cz = (int)(c / ((long long)a.m[0] * a.m[1]));
        const T   x0 = a.origin[0] + a.h[0] * cx, y0 = a.origin[1] + a.h[1] * cy, z0 = a.origin[2] + a.h[2] * cz;
        const T   det = a.h[0] * a.h[1] * a.h[2];
        for (int l = 0; l < N; ++l)
          for (int j = 0; j < N; ++j)
            for (int i = 0; i < N; ++i)
              {
                T s = 0;
                for (int qz = 0; qz < N; ++qz)
                  for (int qy = 0; qy < N; ++qy)
                    for (int qx = 0; qx < N; ++qx)
                      {
                        const T bx = a.B[qx * N + i], by = a.B[qy * N + j], bz = a.B[qz * N + l];
                        const T phi = bx * by * bz;
                        const T gx = a.G[qx * N + i] * by * bz / a.h[0];
                        const T gy = bx * a.G[qy * N + j] * bz / a.h[1];
                        const T gz = bx * by * a.G[qz * N + l] / a.h[2];
                        const T x = x0 + a.h[0] * a.qp[qx], y = y0 + a.h[1] * a.qp[qy], z = z0 + a.h[2] * a.qp[qz];
                        const T vx = a.vel[0] + a.vel[3] * x + a.vel[4] * y + a.vel[5] * z;
                        const T vy = a.vel[1] + a.vel[6] * x + a.vel[7] * y + a.vel[8] * z;
                        const T vz = a.vel[2] + a.vel[9] * x + a.vel[10] * y + a.vel[11] * z;
                        const T JxW = a.qw[qx] * a.qw[qy] * a.qw[qz] * det;
                        s += JxW * (a.inv_dt * phi * phi + a.th_adv * phi * (vx * gx + vy * gy + vz * gz) +
                                    a.th_dif * (gx * gx + gy * gy + gz * gz));
                      }
                a.cellbuf[c * N * N * N + (l * N + j) * N + i] = s;
              }
      }
  }

  // diag[P] = sum over the (<= 8) cells containing P of their local entry; constrained -> 1
  template <typename T>
  __global__ void
  gather_cellbuf_kernel(const GridDesc g, int K, const T *cellbuf, T *diag)
  {
    const int       N     = K + 1;
    const long long ndofs = (long long)g.n[0] * g.n[1] * g.n[2];
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < ndofs;
         idx += (long long)gridDim.x * blockDim.x)
      {
        const int I = (int)(idx % g.n[0]), J = (int)((idx / g.n[0]) % g.n[1]), L = (int)(idx / ((long long)g.n[0] * g.n[1]));
        if (is_constrained(g, I, J, L, idx))
          {
            diag[idx] = T(1);
            continue;
          }
        int       cs[3][2], ls[3][2], nc[3];
        const int P[3] = {I, J, L};
        for (int d = 0; d < 3; ++d)
          {
            nc[d]       = 0;
            const int q = P[d] / K, r = P[d] % K;
            if (r == 0)
              {
                if (q - 1 >= 0)
                  {
                    cs[d][nc[d]] = q - 1;
                    ls[d][nc[d]] = K;
                    ++nc[d];
                  }
                if (q < g.m[d])
                  {
                    cs[d][nc[d]] = q;
                    ls[d][nc[d]] = 0;
                    ++nc[d];
                  }
              }
            else
              {
                cs[d][0] = q;
                ls[d][0] = r;
                nc[d]    = 1;
              }
          }
        T s = T(0);
        for (int z = 0; z < nc[2]; ++z)
          for (int y = 0; y < nc[1]; ++y)
            for (int x = 0; x < nc[0]; ++x)
              {
                const long long cell = (long long)cs[0][x] + (long long)g.m[0] * ((long long)cs[1][y] + (long long)g.m[1] * cs[2][z]);
                s += cellbuf[cell * N * N * N + (ls[2][z] * N + ls[1][y]) * N + ls[0][x]];
              }
        diag[idx] = s;
      }
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
    double hd[3][ADV_TAB] = {};
    float  hf[3][ADV_TAB] = {};
    for (int K = 1; K <= 2; ++K)
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
    auto kern  = adv_apply_kernel<K, T, MODE>;
    static thread_local bool attr_done = false;
    if (!attr_done)
      {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LAY::bytes);
        if (e != cudaSuccess)
          return e;
        attr_done = true;
      }
    const unsigned nbricks = (unsigned)h.grid.nbr[0] * h.grid.nbr[1] * h.grid.nbr[2];
    kern<<<nbricks, LAY::BR::NT, LAY::bytes, stream>>>(a);
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
    else
      {
        shape[0] = AdvLayout<2, T>::BX;
        shape[1] = AdvLayout<2, T>::BY;
        shape[2] = AdvLayout<2, T>::BZ;
      }
  }

  template <typename T, int N>
  static cudaError_t
  cell_diag(const GridDesc &g, const AdvParams &p, T *cellbuf, cudaStream_t s)
  {
    AdvDiagArgs<T, N> a;
    const Tables1D   &t = tables(N - 1);
    for (int i = 0; i < N * N; ++i)
      {
        a.B[i] = (T)t.B[i];
        a.G[i] = (T)t.G[i];
      }
    for (int q = 0; q < N; ++q)
      {
        a.qp[q] = (T)t.qp[q];
        a.qw[q] = (T)t.qw[q];
      }
    a.inv_dt = (T)p.inv_dt;
    a.th_adv = (T)p.theta_adv;
    a.th_dif = (T)p.theta_dif;
    for (int i = 0; i < 12; ++i)
      a.vel[i] = (T)p.vel[i];
    for (int d = 0; d < 3; ++d)
      {
        a.origin[d] = (T)p.origin[d];
        a.h[d]      = (T)p.h[d];
        a.m[d]      = g.m[d];
      }
    a.cellbuf             = cellbuf;
    const long long nc    = (long long)g.m[0] * g.m[1] * g.m[2];
    const int       blocks = (int)std::min<long long>((nc + 127) / 128, 148LL * 16);
    adv_cell_diag_kernel<T, N><<<blocks, 128, 0, s>>>(a);
    return cudaGetLastError();
  }

  template <typename T>
  cudaError_t
  adv_diagonal(const GridDesc &g, int K, const AdvParams &p, T *diag, T *cellbuf, cudaStream_t s)
  {
    cudaError_t e;
    if (K == 1)
      e = cell_diag<T, 2>(g, p, cellbuf, s);
    else if (K == 2)
      e = cell_diag<T, 3>(g, p, cellbuf, s);
    else
      return cudaErrorInvalidValue;
    if (e != cudaSuccess)
      return e;
    const long long n      = (long long)g.n[0] * g.n[1] * g.n[2];
    const int       blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
    gather_cellbuf_kernel<T><<<blocks, 256, 0, s>>>(g, K, cellbuf, diag);
    return cudaGetLastError();
  }

  template cudaError_t adv_apply<double>(const AdvLaunch<double> &, cudaStream_t);
  template cudaError_t adv_apply<float>(const AdvLaunch<float> &, cudaStream_t);
  template cudaError_t adv_diagonal<double>(const GridDesc &, int, const AdvParams &, double *, double *, cudaStream_t);
  template cudaError_t adv_diagonal<float>(const GridDesc &, int, const AdvParams &, float *, float *, cudaStream_t);
  template void adv_brick_shape<double>(int, int[3]);
  template void adv_brick_shape<float>(int, int[3]);
} // namespace mpdg
