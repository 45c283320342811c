// Register-resident 1-D contractions for one hexahedral cell (n = k+1 values per line).
//
// Heat operator, fast diagonalisation.  On an axis-aligned box cell of size hx x hy x hz the heat
// tangent of source/heat/heat_diffuse_operator.cpp:1029-1079 integrated with QGauss(k+1) is
//   A_c = a M(x)M(x)M + k_c (cx K(x)M(x)M + cy M(x)K(x)M + cz M(x)M(x)K),
//   a = rho c_p / dt * hx hy hz,  cx = hy hz / hx (and cyclic),
// with the 1-D reference mass M and stiffness K (QGauss(k+1) integrates both exactly).  With the
// generalised eigenbasis K v = lambda M v, v^T M v = 1, and W = V^T M:  M = W^T W, K = W^T Lambda W,
//   A_c = (W(x)W(x)W)^T diag(a + k_c (cx lam_a + cy lam_b + cz lam_c)) (W(x)W(x)W).
// Reflection symmetry of the Gauss-Lobatto nodes makes every eigenvector even or odd, so each 1-D
// transform folds a line into even/odd halves first (e_i = u_i + u_{n-1-i}, o_i = u_i - u_{n-1-i})
// and applies a ceil(n/2)^2 and a floor(n/2)^2 block instead of an n^2 matrix.
#pragma once

namespace mpdg
{
  template <typename T, int N>
  struct FDTab
  {
    static constexpr int NE = (N + 1) / 2, NO = N / 2;
    T                    we[NE * NE];                   // even block (rows: modes)
    T                    wo[NO > 0 ? NO * NO : 1];      // odd block
    T                    lam3[N * N * N];               // cx lam_a + cy lam_b + cz lam_c (modal order)
  };

  // nodal -> modal along one line v[b + k*S], k < N; modal order: even modes, then odd modes.
  // The values may be packed pairs (TT the scalar type of the tables, T the value type).
  template <typename T, int N, int S, typename TT = T>
  __device__ __forceinline__ void
  fwd_line(T *v, const int b, const TT *we, const TT *wo)
  {
    constexpr int NE = (N + 1) / 2, NO = N / 2;
    T             e[NE], o[NO > 0 ? NO : 1];
#pragma unroll
    for (int k = 0; k < N / 2; ++k)
      {
        const T a = v[b + k * S], c = v[b + (N - 1 - k) * S];
        e[k]      = a + c;
        o[k]      = a - c;
      }
    if constexpr (N % 2 == 1)
      e[N / 2] = v[b + (N / 2) * S];
#pragma unroll
    for (int m = 0; m < NE; ++m)
      {
        T s = we[m * NE] * e[0];
#pragma unroll
        for (int k = 1; k < NE; ++k)
          s = fma(we[m * NE + k], e[k], s);
        v[b + m * S] = s;
      }
#pragma unroll
    for (int m = 0; m < NO; ++m)
      {
        T s = wo[m * NO] * o[0];
#pragma unroll
        for (int k = 1; k < NO; ++k)
          s = fma(wo[m * NO + k], o[k], s);
        v[b + (NE + m) * S] = s;
      }
  }

  // modal -> nodal along one line (transpose of fwd_line)
  template <typename T, int N, int S, typename TT = T>
  __device__ __forceinline__ void
  bwd_line(T *v, const int b, const TT *we, const TT *wo)
  {
    constexpr int NE = (N + 1) / 2, NO = N / 2;
    T             ev[NE], od[NO > 0 ? NO : 1];
#pragma unroll
    for (int m = 0; m < NE; ++m)
      ev[m] = v[b + m * S];
#pragma unroll
    for (int m = 0; m < NO; ++m)
      od[m] = v[b + (NE + m) * S];
#pragma unroll
    for (int k = 0; k < N / 2; ++k)
      {
        T E = we[k] * ev[0];
#pragma unroll
        for (int m = 1; m < NE; ++m)
          E = fma(we[m * NE + k], ev[m], E);
        T O = wo[k] * od[0];
#pragma unroll
        for (int m = 1; m < NO; ++m)
          O = fma(wo[m * NO + k], od[m], O);
        v[b + k * S]           = E + O;
        v[b + (N - 1 - k) * S] = E - O;
      }
    if constexpr (N % 2 == 1)
      {
        T E = we[N / 2] * ev[0];
#pragma unroll
        for (int m = 1; m < NE; ++m)
          E = fma(we[m * NE + N / 2], ev[m], E);
        v[b + (N / 2) * S] = E;
      }
  }

  // Apply fwd/bwd in x and y to P planes of N x N values (plane stride N*N, x fastest).
  template <typename T, int N, int P, bool FWD, typename TT = T>
  __device__ __forceinline__ void
  xy_planes(T *v, const TT *we, const TT *wo)
  {
    if constexpr (FWD)
      {
#pragma unroll
        for (int p = 0; p < P; ++p)
          {
#pragma unroll
            for (int j = 0; j < N; ++j)
              fwd_line<T, N, 1, TT>(v, p * N * N + j * N, we, wo);
#pragma unroll
            for (int i = 0; i < N; ++i)
              fwd_line<T, N, N, TT>(v, p * N * N + i, we, wo);
          }
      }
    else
      {
#pragma unroll
        for (int p = 0; p < P; ++p)
          {
#pragma unroll
            for (int i = 0; i < N; ++i)
              bwd_line<T, N, N, TT>(v, p * N * N + i, we, wo);
#pragma unroll
            for (int j = 0; j < N; ++j)
              bwd_line<T, N, 1, TT>(v, p * N * N + j * N, we, wo);
          }
      }
  }

  // Compile-time index of a shell point (some local index 0) in the per-cell shell array.
  template <int N>
  __host__ __device__ constexpr int
  shell_index(int i, int j, int l)
  {
    constexpr int K = N - 1;
    return l == 0 ? j * N + i : (j == 0 ? N * N + (l - 1) * N + i : N * N + K * N + (l - 1) * K + (j - 1));
  }
} // namespace mpdg
