// Host-side 1-D tables of the FE_Q(k) / QGauss(k+1) reference element.
#pragma once

#include <vector>

namespace mpdg
{
  constexpr int MAX_N = 6; // nodes per direction supported by the tables (degree <= 5)

  struct Tables1D
  {
    int    n  = 0; // nodes = Gauss points = degree + 1
    int    ne = 0; // even modes  = ceil(n/2)
    int    no = 0; // odd modes   = floor(n/2)
    double nodes[MAX_N]{};        // Gauss-Lobatto support points on [0,1]
    double qp[MAX_N]{}, qw[MAX_N]{}; // Gauss points / weights on [0,1]
    double B[MAX_N * MAX_N]{};    // B[q*n+i] = phi_i(qp_q)
    double G[MAX_N * MAX_N]{};    // G[q*n+i] = phi_i'(qp_q)
    double Dq[MAX_N * MAX_N]{};   // collocation derivative on the Gauss points: Dq[q*n+r] = ell_r'(qp_q)
    double M[MAX_N * MAX_N]{};    // 1-D mass      M[i*n+j] = sum_q w phi_i phi_j
    double K[MAX_N * MAX_N]{};    // 1-D stiffness K[i*n+j] = sum_q w phi_i' phi_j'
    // Generalised eigenbasis K v = lambda M v, v^T M v = 1, split by reflection parity.
    // Forward (nodal -> modal) on folded coordinates:
    //   even modes: u_hat_e[m] = sum_k WE[m*ne+k] e_k, e_k = u_k + u_{n-1-k} (k < n/2), e_mid = u_mid
    //   odd  modes: u_hat_o[m] = sum_k WO[m*no+k] o_k, o_k = u_k - u_{n-1-k}
    double WE[MAX_N * MAX_N]{};
    double WO[MAX_N * MAX_N]{};
    double lam[MAX_N]{}; // eigenvalues in modal order: even modes first, then odd
  };

  // Builds and caches the tables of one degree (thread-safe after the first call per degree).
  const Tables1D &tables(int degree);
} // namespace mpdg
