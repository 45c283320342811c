// Boundary-face terms of the heat operator: convection h (T - T_inf), radiation
// eps sigma (T^4 - T_inf^4) and a constant normal heat flux, on whole faces of the box.
//
//   tangent   (source/heat/heat_diffuse_operator.cpp:1088-1129, vmult's boundary face loop
//              :239-264):  dst += scale * int_f (h + 4 eps sigma T^3) u phi
//   rhs       (:719-781):  dst -= int_f [eps sigma (T^4 - T_inf^4) + h (T - T_inf) + g.n] phi
//   diagonal  (:297-357, MatrixFreeTools::compute_diagonal's boundary operation):
//              diag_i += int_f (h + 4 eps sigma T^3) phi_i^2
//
// Face quadrature is QGauss(k+1) in both face directions, as the cell quadrature.  The tangent and
// the diagonal read u and T with constraints (Dirichlet DoFs as 0: FEFaceEvaluation::read_dof_values
// and gather_evaluate); the rhs reads T plain (read_dof_values_plain).  Constrained rows are never
// written.  One thread per boundary cell face: it gathers the (k+1)^2 face values, interpolates them
// to the Gauss points with two 1-D passes, forms the integrand and integrates back with the
// transposed passes, then adds into dst with atomics (DoFs on patch edges are shared by up to four
// face patches of one face and by the patches of an adjacent face).
#include "kernels.h"

namespace mpdg
{
  namespace
  {
    template <typename T>
    struct FaceArgs
    {
      GridDesc      g;
      int           K;
      int           mode; // 0 tangent, 1 rhs, 2 diagonal
      double        scale;
      double        hlen[3];
      HeatFaceBC    bc;
      int           off[7]; // first patch of face f (faces without a term have no patches)
      const double *temp;
      const T      *src;
      T            *dst;
      double       *diag;
      const int    *skip;
      double        B[MAX_N * MAX_N]; // B[q*n+i] = phi_i(qp_q)
      double        w[MAX_N];
    };

    template <int N, typename T>
    __device__ __forceinline__ void
    face_patch(const FaceArgs<T> &a, int p)
    {
      constexpr int K = N - 1;
      int           f = 0;
      while (f < 5 && p >= a.off[f + 1])
        ++f;
      const int d = f >> 1, side = f & 1;
      const int da = d == 0 ? 1 : 0, db = d == 2 ? 1 : 2; // tangential directions, da < db
      const int q  = p - a.off[f];
      const int ca = q % a.g.m[da], cb = q / a.g.m[da];
      const double area = a.hlen[da] * a.hlen[db];
      const unsigned bit = 1u << f;
      const bool conv = (a.bc.convection_faces & bit) != 0, rad = (a.bc.radiation_faces & bit) != 0;
      const bool neu  = (a.bc.neumann_faces & bit) != 0;

      long long idx[N * N];
      bool      con[N * N];
      double    u[N * N], t[N * N];
      int       c[3];
      c[d] = side ? a.g.n[d] - 1 : 0;
#pragma unroll
      for (int j = 0; j < N; ++j)
#pragma unroll
        for (int i = 0; i < N; ++i)
          {
            c[da] = K * ca + i;
            c[db] = K * cb + j;
            const long long id = (long long)c[0] + (long long)a.g.n[0] * ((long long)c[1] + (long long)a.g.n[1] * c[2]);
            const bool      cn = is_constrained(a.g, c[0], c[1], c[2], id);
            idx[j * N + i]     = id;
            con[j * N + i]     = cn;
            const bool need_t  = rad || (a.mode == 1 && conv);
            t[j * N + i]       = need_t && a.temp != nullptr && (a.mode == 1 || !cn) ? a.temp[id] : 0.0;
            u[j * N + i]       = a.mode == 0 && !cn ? (double)a.src[id] : 0.0;
          }
      // values at the Gauss points: first along a, then along b
      double uq[N * N], tq[N * N];
#pragma unroll
      for (int j = 0; j < N; ++j)
#pragma unroll
        for (int qa = 0; qa < N; ++qa)
          {
            double su = 0.0, st = 0.0;
#pragma unroll
            for (int i = 0; i < N; ++i)
              {
                su += a.B[qa * N + i] * u[j * N + i];
                st += a.B[qa * N + i] * t[j * N + i];
              }
            uq[j * N + qa] = su;
            tq[j * N + qa] = st;
          }
#pragma unroll
      for (int qa = 0; qa < N; ++qa)
        {
          double su[N], st[N];
#pragma unroll
          for (int qb = 0; qb < N; ++qb)
            {
              su[qb] = 0.0;
              st[qb] = 0.0;
#pragma unroll
              for (int j = 0; j < N; ++j)
                {
                  su[qb] += a.B[qb * N + j] * uq[j * N + qa];
                  st[qb] += a.B[qb * N + j] * tq[j * N + qa];
                }
            }
#pragma unroll
          for (int qb = 0; qb < N; ++qb)
            {
              uq[qb * N + qa] = su[qb];
              tq[qb * N + qa] = st[qb];
            }
        }
      // integrand times the quadrature weight
      double fq[N * N];
#pragma unroll
      for (int qb = 0; qb < N; ++qb)
#pragma unroll
        for (int qa = 0; qa < N; ++qa)
          {
            const double W  = a.w[qa] * a.w[qb] * area;
            const double Tq = tq[qb * N + qa];
            double       v;
            if (a.mode == 1)
              {
                v = 0.0;
                if (rad)
                  {
                    const double T2 = Tq * Tq, Ti = a.bc.radiation_temperature_infinity, Ti2 = Ti * Ti;
                    v -= a.bc.emissivity_sigma * (T2 * T2 - Ti2 * Ti2);
                  }
                if (conv)
                  v -= a.bc.convection_coefficient * (Tq - a.bc.convection_temperature_infinity);
                if (neu)
                  v -= a.bc.neumann_flux[f];
              }
            else
              {
                v = 0.0;
                if (conv)
                  v += a.bc.convection_coefficient;
                if (rad)
                  v += 4.0 * a.bc.emissivity_sigma * Tq * Tq * Tq;
                if (a.mode == 0)
                  v *= uq[qb * N + qa];
              }
            fq[qb * N + qa] = v * W;
          }
      if (a.mode == 2)
        {
          // diag_i += sum_q c_q W_q phi_i(q)^2
#pragma unroll
          for (int j = 0; j < N; ++j)
#pragma unroll
            for (int i = 0; i < N; ++i)
              if (!con[j * N + i])
                {
                  double s = 0.0;
#pragma unroll
                  for (int qb = 0; qb < N; ++qb)
#pragma unroll
                    for (int qa = 0; qa < N; ++qa)
                      {
                        const double ba = a.B[qa * N + i], bb = a.B[qb * N + j];
                        s += fq[qb * N + qa] * ba * ba * bb * bb;
                      }
                  atomicAdd(a.diag + idx[j * N + i], s);
                }
          return;
        }
      // integrate: transposed passes, b first
      double r1[N * N];
#pragma unroll
      for (int qa = 0; qa < N; ++qa)
#pragma unroll
        for (int j = 0; j < N; ++j)
          {
            double s = 0.0;
#pragma unroll
            for (int qb = 0; qb < N; ++qb)
              s += a.B[qb * N + j] * fq[qb * N + qa];
            r1[j * N + qa] = s;
          }
#pragma unroll
      for (int j = 0; j < N; ++j)
#pragma unroll
        for (int i = 0; i < N; ++i)
          if (!con[j * N + i])
            {
              double s = 0.0;
#pragma unroll
              for (int qa = 0; qa < N; ++qa)
                s += a.B[qa * N + i] * r1[j * N + qa];
              atomicAdd(a.dst + idx[j * N + i], (T)(a.mode == 0 ? a.scale * s : s));
            }
    }

    template <int N, typename T>
    __global__ void __launch_bounds__(128)
    heat_face_kernel(const __grid_constant__ FaceArgs<T> a)
    {
      if (a.skip != nullptr && *a.skip != 0)
        return;
      const int p = blockIdx.x * blockDim.x + threadIdx.x;
      if (p < a.off[6])
        face_patch<N, T>(a, p);
    }
  } // namespace

  bool
  heat_faces_active(const HeatFaceBC &bc, int mode)
  {
    const unsigned tangent = bc.convection_faces | bc.radiation_faces;
    return (mode == 1 ? (tangent | bc.neumann_faces) : tangent) != 0u;
  }

  template <typename T>
  cudaError_t
  heat_faces(const HeatFaceLaunch<T> &h, cudaStream_t s)
  {
    if (h.degree < 1 || h.degree > 4)
      return cudaErrorInvalidValue;
    FaceArgs<T> a{};
    a.g     = h.grid;
    a.K     = h.degree;
    a.mode  = h.mode;
    a.scale = h.scale;
    for (int d = 0; d < 3; ++d)
      a.hlen[d] = h.hlen[d];
    a.bc   = h.bc;
    a.temp = h.temp;
    a.src  = h.src;
    a.dst  = h.dst;
    a.diag = h.diag;
    a.skip = h.skip;
    const unsigned faces = h.mode == 1 ? (h.bc.convection_faces | h.bc.radiation_faces | h.bc.neumann_faces)
                                       : (h.bc.convection_faces | h.bc.radiation_faces);
    int total = 0;
    for (int f = 0; f < 6; ++f)
      {
        a.off[f]     = total;
        const int d  = f >> 1;
        const int da = d == 0 ? 1 : 0, db = d == 2 ? 1 : 2;
        if (faces & (1u << f))
          total += h.grid.m[da] * h.grid.m[db];
      }
    a.off[6] = total;
    if (total == 0)
      return cudaSuccess;
    const Tables1D &t = tables(h.degree);
    const int       N = h.degree + 1;
    for (int i = 0; i < N * N; ++i)
      a.B[i] = t.B[i];
    for (int q = 0; q < N; ++q)
      a.w[q] = t.qw[q];
    const int blocks = (total + 127) / 128;
    switch (N)
      {
        case 2: heat_face_kernel<2, T><<<blocks, 128, 0, s>>>(a); break;
        case 3: heat_face_kernel<3, T><<<blocks, 128, 0, s>>>(a); break;
        case 4: heat_face_kernel<4, T><<<blocks, 128, 0, s>>>(a); break;
        default: heat_face_kernel<5, T><<<blocks, 128, 0, s>>>(a); break;
      }
    return cudaGetLastError();
  }

  template cudaError_t heat_faces<double>(const HeatFaceLaunch<double> &, cudaStream_t);
  template cudaError_t heat_faces<float>(const HeatFaceLaunch<float> &, cudaStream_t);
} // namespace mpdg
