// 1-D tables of the FE_Q(k) element with QGauss(k+1): Gauss-Lobatto support points (deal.II's
// FE_Q default), Gauss quadrature, basis values/derivatives, and the generalised eigenbasis of
// the 1-D stiffness/mass pair used by the fast-diagonalisation apply of the heat operator.
#include "tables.h"

#include <algorithm>
#include <cmath>
#include <mutex>

namespace mpdg
{
  namespace
  {
    void
    legendre(int n, double x, double &p, double &dp)
    {
      double p0 = 1.0, p1 = x;
      if (n == 0)
        {
          p  = 1.0;
          dp = 0.0;
          return;
        }
      for (int k = 2; k <= n; ++k)
        {
          const double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
          p0              = p1;
          p1              = p2;
        }
      p  = p1;
      dp = n * (p0 - x * p1) / (1.0 - x * x);
    }

    // interior Gauss-Lobatto points: roots of P_k' by Newton, with P_k'' from Legendre's equation
    void
    lobatto(int k, double *x01)
    {
      x01[0] = 0.0;
      x01[k] = 1.0;
      for (int i = 1; i < k; ++i)
        {
          double x = -std::cos(M_PI * i / k);
          for (int it = 0; it < 200; ++it)
            {
              double p, dp;
              legendre(k, x, p, dp);
              const double ddp = (2.0 * x * dp - k * (k + 1.0) * p) / (1.0 - x * x);
              const double dx  = dp / ddp;
              x -= dx;
              if (std::abs(dx) < 1e-17)
                break;
            }
          x01[i] = 0.5 * (x + 1.0);
        }
      std::sort(x01, x01 + k + 1);
    }

    void
    gauss(int n, double *x01, double *w01)
    {
      for (int i = 0; i < n; ++i)
        {
          double x = -std::cos(M_PI * (i + 0.75) / (n + 0.5));
          double p = 0.0, dp = 1.0;
          for (int it = 0; it < 200; ++it)
            {
              legendre(n, x, p, dp);
              const double dx = p / dp;
              x -= dx;
              if (std::abs(dx) < 1e-17)
                break;
            }
          legendre(n, x, p, dp);
          x01[i] = 0.5 * (x + 1.0);
          w01[i] = 1.0 / ((1.0 - x * x) * dp * dp);
        }
      for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j)
          if (x01[j] < x01[i])
            {
              std::swap(x01[i], x01[j]);
              std::swap(w01[i], w01[j]);
            }
    }

    void
    lagrange(int n, const double *x, int i, double t, double &val, double &der)
    {
      val = 1.0;
      for (int j = 0; j < n; ++j)
        if (j != i)
          val *= (t - x[j]) / (x[i] - x[j]);
      der = 0.0;
      for (int m = 0; m < n; ++m)
        {
          if (m == i)
            continue;
          double prod = 1.0 / (x[i] - x[m]);
          for (int j = 0; j < n; ++j)
            if (j != i && j != m)
              prod *= (t - x[j]) / (x[i] - x[j]);
          der += prod;
        }
    }

    // cyclic Jacobi eigen-decomposition of a small symmetric matrix A (n x n, row-major);
    // on return A is diagonal (eigenvalues), V holds the eigenvectors in its columns
    void
    jacobi_eigen(int n, double *A, double *V)
    {
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
          V[i * n + j] = (i == j) ? 1.0 : 0.0;
      for (int sweep = 0; sweep < 100; ++sweep)
        {
          double off = 0.0;
          for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q)
              off += A[p * n + q] * A[p * n + q];
          if (off < 1e-32)
            break;
          for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q)
              {
                const double apq = A[p * n + q];
                if (std::abs(apq) < 1e-300)
                  continue;
                const double theta = (A[q * n + q] - A[p * n + p]) / (2.0 * apq);
                const double t     = (theta >= 0 ? 1.0 : -1.0) / (std::abs(theta) + std::sqrt(theta * theta + 1.0));
                const double c     = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; ++k)
                  {
                    const double akp = A[k * n + p], akq = A[k * n + q];
                    A[k * n + p]     = c * akp - s * akq;
                    A[k * n + q]     = s * akp + c * akq;
                  }
                for (int k = 0; k < n; ++k)
                  {
                    const double apk = A[p * n + k], aqk = A[q * n + k];
                    A[p * n + k]     = c * apk - s * aqk;
                    A[q * n + k]     = s * apk + c * aqk;
                  }
                for (int k = 0; k < n; ++k)
                  {
                    const double vkp = V[k * n + p], vkq = V[k * n + q];
                    V[k * n + p]     = c * vkp - s * vkq;
                    V[k * n + q]     = s * vkp + c * vkq;
                  }
              }
        }
    }

    // Solve Kp y = lambda Mp y on one parity subspace spanned by the columns of F (n x m).
    // Writes W rows (m x m, on folded coordinates) and eigenvalues (ascending).
    void
    parity_eigen(const Tables1D &t, int m, const double *F, double *W, double *lam)
    {
      const int n = t.n;
      double    Mp[MAX_N * MAX_N], Kp[MAX_N * MAX_N];
      for (int a = 0; a < m; ++a)
        for (int b = 0; b < m; ++b)
          {
            double sm = 0.0, sk = 0.0;
            for (int i = 0; i < n; ++i)
              for (int j = 0; j < n; ++j)
                {
                  sm += F[i * m + a] * t.M[i * n + j] * F[j * m + b];
                  sk += F[i * m + a] * t.K[i * n + j] * F[j * m + b];
                }
            Mp[a * m + b] = sm;
            Kp[a * m + b] = sk;
          }
      // Cholesky Mp = L L^T
      double L[MAX_N * MAX_N] = {};
      for (int i = 0; i < m; ++i)
        for (int j = 0; j <= i; ++j)
          {
            double s = Mp[i * m + j];
            for (int k = 0; k < j; ++k)
              s -= L[i * m + k] * L[j * m + k];
            L[i * m + j] = (i == j) ? std::sqrt(s) : s / L[j * m + j];
          }
      // Li = L^{-1}
      double Li[MAX_N * MAX_N] = {};
      for (int c = 0; c < m; ++c)
        for (int i = 0; i < m; ++i)
          {
            double s = (i == c) ? 1.0 : 0.0;
            for (int k = 0; k < i; ++k)
              s -= L[i * m + k] * Li[k * m + c];
            Li[i * m + c] = s / L[i * m + i];
          }
      // C = Li Kp Li^T
      double C[MAX_N * MAX_N], Q[MAX_N * MAX_N];
      for (int a = 0; a < m; ++a)
        for (int b = 0; b < m; ++b)
          {
            double s = 0.0;
            for (int i = 0; i < m; ++i)
              for (int j = 0; j < m; ++j)
                s += Li[a * m + i] * Kp[i * m + j] * Li[b * m + j];
            C[a * m + b] = s;
          }
      jacobi_eigen(m, C, Q);
      int order[MAX_N];
      for (int i = 0; i < m; ++i)
        order[i] = i;
      std::sort(order, order + m, [&](int a, int b) { return C[a * m + a] < C[b * m + b]; });
      for (int r = 0; r < m; ++r)
        {
          const int col = order[r];
          lam[r]        = C[col * m + col];
          // y = Li^T q (M-orthonormal in the folded space); nodal v = F y; w = v^T M (row)
          double y[MAX_N], v[MAX_N], w[MAX_N];
          for (int i = 0; i < m; ++i)
            {
              double s = 0.0;
              for (int k = 0; k < m; ++k)
                s += Li[k * m + i] * Q[k * m + col];
              y[i] = s;
            }
          for (int i = 0; i < n; ++i)
            {
              double s = 0.0;
              for (int k = 0; k < m; ++k)
                s += F[i * m + k] * y[k];
              v[i] = s;
            }
          for (int j = 0; j < n; ++j)
            {
              double s = 0.0;
              for (int i = 0; i < n; ++i)
                s += v[i] * t.M[i * n + j];
              w[j] = s;
            }
          // fix the sign so that the first folded coefficient is non-negative (deterministic tables)
          const double sgn = (w[0] < 0.0) ? -1.0 : 1.0;
          for (int k = 0; k < m; ++k)
            W[r * m + k] = sgn * w[k];
        }
    }

    Tables1D
    build(int degree)
    {
      Tables1D t;
      const int n = degree + 1;
      t.n         = n;
      t.ne        = (n + 1) / 2;
      t.no        = n / 2;
      lobatto(degree, t.nodes);
      gauss(n, t.qp, t.qw);
      for (int q = 0; q < n; ++q)
        for (int i = 0; i < n; ++i)
          lagrange(n, t.nodes, i, t.qp[q], t.B[q * n + i], t.G[q * n + i]);
      for (int q = 0; q < n; ++q)
        for (int r = 0; r < n; ++r)
          {
            double v, d;
            lagrange(n, t.qp, r, t.qp[q], v, d);
            t.Dq[q * n + r] = d;
          }
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
          {
            double sm = 0.0, sk = 0.0;
            for (int q = 0; q < n; ++q)
              {
                sm += t.qw[q] * t.B[q * n + i] * t.B[q * n + j];
                sk += t.qw[q] * t.G[q * n + i] * t.G[q * n + j];
              }
            t.M[i * n + j] = sm;
            t.K[i * n + j] = sk;
          }
      double Fe[MAX_N * MAX_N] = {}, Fo[MAX_N * MAX_N] = {};
      for (int k = 0; k < n / 2; ++k)
        {
          Fe[k * t.ne + k]           = 1.0;
          Fe[(n - 1 - k) * t.ne + k] = 1.0;
          Fo[k * t.no + k]           = 1.0;
          Fo[(n - 1 - k) * t.no + k] = -1.0;
        }
      if (n % 2)
        Fe[(n / 2) * t.ne + n / 2] = 1.0;
      parity_eigen(t, t.ne, Fe, t.WE, t.lam);
      if (t.no > 0)
        parity_eigen(t, t.no, Fo, t.WO, t.lam + t.ne);
      return t;
    }
  } // namespace

  const Tables1D &
  tables(int degree)
  {
    static std::once_flag once[MAX_N];
    static Tables1D       cache[MAX_N];
    if (degree < 1 || degree >= MAX_N)
      degree = 1;
    std::call_once(once[degree], [&] { cache[degree] = build(degree); });
    return cache[degree];
  }
} // namespace mpdg
