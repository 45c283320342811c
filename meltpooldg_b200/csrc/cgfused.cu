// One launch per Jacobi-PCG iteration of the FE_Q(2) heat operator (dealii::SolverCG semantics,
// include/meltpooldg/linear_algebra/linear_solver.hpp:106-110 with the Jacobi preconditioner of
// preconditioner_jacobi.hpp:51-56): the vector updates, the preconditioner, the operator apply
// (source/heat/heat_diffuse_operator.cpp:179-197, tangent :1029-1079) and every dot product of the
// iteration happen in one sweep over the lattice.
//
// Recurrence.  Sweep k reads x_{k-1}, r_{k-1}, p_{k-1}, v_{k-1} = A p_{k-1} and the inverse diagonal
// d, and with the step lengths a = alpha_{k-1}, b = beta_k of the previous sweep forms, per DoF,
//   r_k = r_{k-1} - a v_{k-1},  x_k = x_{k-1} + a p_{k-1},  z_k = d r_k,  p_k = z_k + b p_{k-1},
// then applies v_k = A p_k and sums
//   S0 = r_k.z_k (rho_k),  S6 = r_k.r_k,  S1 = p_k.v_k,  S2 = z_k.v_k,  S3 = v_k.(d v_k).
// The last CTA sets alpha_k = S0 / S1 and, since r_{k+1} = r_k - alpha_k v_k,
//   rho_{k+1} = S0 - 2 alpha_k S2 + alpha_k^2 S3,  beta_{k+1} = rho_{k+1} / S0,
// so the next sweep can form p_{k+1} without another pass.  |r_k| = sqrt(S6) is the residual that
// SolverCG checks after iteration k (ReductionControl: |r_k| <= max(abs_tol, rel_tol |r_0|)).  Sweep 0
// forms z_0, p_0 = z_0 and v_0 only.  Per iteration the sweep reads x, r, p, v, d and writes x, r,
// p, v: s (9 N + N_c) bytes, against s (13 N + N_c) for separate update / apply / update passes.
//
// Tiles.  The lattice is cut into columns of 32 x TY cells in x, y and into slabs of cell layers in
// z; the (column, layer) pairs, taken slab by slab and column by column within a slab, are dealt out
// in equal contiguous ranges to a grid of one CTA per resident slot, so every SM gets the same
// number of layers and the CTAs running side by side work on neighbouring columns at nearly the same
// layers (their halo planes are shared through L2).  A CTA's range is one or a few pieces (a segment
// of z layers of one column); it owns the lattice points of each piece and marches through it
// layer by layer.  It also computes the cells of one halo layer
// on its low side in x, y and z (a halo column warp, a halo row warp, a halo cell layer), so every
// owned point receives all of its cell contributions inside the CTA: no atomics, no inter-CTA
// waits, and each owned point's update and dot products are done by one thread.  The vectors use a
// padded layout (x rows of P0 >= n0 + 1 entries, P0 a multiple of 8), so that every lattice plane
// of a tile is one TMA box (cp.async.bulk.tensor.3d into shared memory, zero fill outside the
// lattice).  Per layer: the two new lattice planes are staged by TMA while the previous layer's
// cells compute; each point of a staged plane is updated (owned points also written out) and its
// p_k goes to a ring of three planes; every thread then applies the fast-diagonalisation cell
// operator (sumfac.cuh) to its cell's 27 values of p_k; x faces are combined by warp shuffles, y
// faces through shared memory, z faces carried in registers; owned points of the finished planes
// get v_k, S2 and S3.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include <type_traits>

#include "cgfused.h"
#include "pack2.cuh"
#include "sumfac.cuh"
#include "tables.h"

namespace mpdg
{
  namespace cgf
  {
    constexpr int K = 2, N = 3, NE = 2, NO = 1;
    constexpr int XOFF = 4;   // staged x index of lattice point 2 cx0
    constexpr int NV   = 5;   // staged vectors: r, v, p, x, d

    template <typename T, int TY>
    struct Shape
    {
      // cells per lane in x: two adjacent cells per thread in FP32, computed as packed pairs
      static constexpr int C     = sizeof(T) == 4 ? FUSED_C_F32 : 1;
      using LV                   = std::conditional_t<C == 2, F2, T>; // a lane's values of one point
      static constexpr int TX    = 32 * C;      // owned cells per tile in x
      static constexpr int SX    = 2 * TX + 8;  // staged x points per row: lattice x from 2 cx0 - 4 (TMA x alignment)
      static constexpr int OXW   = 2 * TX + 4;  // owned window in x: lattice x from 2 cx0 (2 TX + 2 used; rows of 16 bytes x k)
      static constexpr int RY    = 2 * TY + 3;  // staged rows: lattice y from 2 cy0 - 2
      static constexpr int PLANE = SX * RY;     // staged points per plane
      static constexpr int OYW   = 2 * TY + 1;  // owned window rows: lattice y from 2 cy0
      static constexpr int OPL   = OXW * OYW;   // owned window points per plane
      static constexpr int NW    = TY + 2;      // warps: TY main rows, halo row, halo column
      static constexpr int NT    = 32 * NW;
      // shared memory layout (bytes, 128-byte aligned sections)
      static constexpr size_t align(size_t b) { return (b + 127) / 128 * 128; }
      static constexpr size_t STAGE_B = align(sizeof(T) * PLANE);      // one vector, one plane
      static constexpr size_t O_STAGE = 0;                              // [2 slots][NV] planes
      static constexpr size_t O_PRING = O_STAGE + 2 * NV * STAGE_B;     // [3] planes of p_k
      static constexpr size_t O_ZS    = O_PRING + 3 * STAGE_B;          // [3] owned planes of z
      static constexpr size_t O_DS    = O_ZS + align(3 * sizeof(T) * OPL); // [3] owned planes of d
      static constexpr size_t O_YX    = O_DS + align(3 * sizeof(T) * OPL);
      static constexpr size_t O_HX    = O_YX + align(sizeof(LV) * (TY + 1) * 9 * 32);
      static constexpr size_t O_RED   = O_HX + align(sizeof(T) * (TY + 1) * 9);
      static constexpr size_t O_BAR   = O_RED + align(sizeof(double) * NW * 5);
      static constexpr size_t BYTES   = O_BAR + 128;
    };

    template <typename T>
    struct Sweep
    {
      int           m[3], n[3];
      int           P0;          // padded x pitch (elements)
      unsigned      faces;       // Dirichlet faces (bit 2d low, 2d+1 high of dim d)
      int           tiles_x, tiles_y, ty;
      long long     layers;      // columns x cell layers
      int           slab;        // layers of a slab: the sequence is slab by slab, column by column
      const long long *range;    // CTA b takes sequence positions [range[b], range[b + 1])
      T             alpha_m, cx, cy, cz; // mass coefficient, stiffness geometry factors
      T             kconst;
      const T      *kcell;
      T             we[NE * NE], wo[NO * NO], lam[N];
      T            *x;           // in place (owned points)
      T            *r_out, *p_out, *v_out;
      CGState      *st;
      double       *part;        // 5 partial sums per CTA
      unsigned     *counter;     // last-CTA ticket (0 between launches)
      double       *hist;
      int          *err;
      unsigned      spin_limit;
    };

    // ---- TMA / mbarrier primitives (sm_90+ PTX)
    __device__ __forceinline__ unsigned
    smem_u32(const void *p)
    {
      return (unsigned)__cvta_generic_to_shared(p);
    }
    __device__ __forceinline__ void
    mbar_init(unsigned long long *bar, unsigned count)
    {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    }
    __device__ __forceinline__ void
    mbar_expect_tx(unsigned long long *bar, unsigned bytes)
    {
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                   : "memory");
    }
    // bounded wait for the phase with the given parity; false when the limit ran out
    __device__ __forceinline__ bool
    mbar_wait(unsigned long long *bar, unsigned parity, unsigned limit)
    {
      const unsigned a = smem_u32(bar);
      for (unsigned it = 0; it < limit; ++it)
        {
          unsigned ok;
          asm volatile("{\n\t.reg .pred p;\n\t"
                       "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                       "selp.u32 %0, 1, 0, p;\n\t}"
                       : "=r"(ok)
                       : "r"(a), "r"(parity)
                       : "memory");
          if (ok)
            return true;
        }
      return false;
    }
    __device__ __forceinline__ void
    tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, unsigned long long *bar)
    {
      asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                   " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
                   "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
                   : "memory");
    }

    template <typename T>
    struct Pair;
    template <>
    struct Pair<double>
    {
      using V = double2;
    };
    template <>
    struct Pair<float>
    {
      using V = float2;
    };

    // W consecutive values of T as one aligned vector access (W * sizeof(T) = 16 bytes, or a pair)
    template <typename T, int W>
    struct Vec;
    template <>
    struct Vec<double, 2>
    {
      using V = double2;
    };
    template <>
    struct Vec<float, 2>
    {
      using V = float2;
    };
    template <>
    struct Vec<float, 4>
    {
      using V = float4;
    };
    template <typename T, int W>
    __device__ __forceinline__ void
    vload(T (&e)[W], const T *p)
    {
      *reinterpret_cast<typename Vec<T, W>::V *>(e) = *reinterpret_cast<const typename Vec<T, W>::V *>(p);
    }
    template <typename T, int W>
    __device__ __forceinline__ void
    vstore(T *p, const T (&e)[W])
    {
      *reinterpret_cast<typename Vec<T, W>::V *>(p) = *reinterpret_cast<const typename Vec<T, W>::V *>(e);
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

    template <typename T, int TY, bool FIRST>
    __global__ void __launch_bounds__(Shape<T, TY>::NT, Shape<T, TY>::BYTES <= 112 * 1024 ? 2 : 1)
    heat_cg_sweep_kernel(const __grid_constant__ Sweep<T> a, const __grid_constant__ CUtensorMap tm_r,
                         const __grid_constant__ CUtensorMap tm_v, const __grid_constant__ CUtensorMap tm_p,
                         const __grid_constant__ CUtensorMap tm_x, const __grid_constant__ CUtensorMap tm_d)
    {
      using S  = Shape<T, TY>;
      using PV = typename Pair<T>::V;
      using LV = typename S::LV;
      constexpr int C = S::C, TX = S::TX, SX = S::SX, OXW = S::OXW;
      extern __shared__ __align__(128) unsigned char smem[];
      T                  *stage = reinterpret_cast<T *>(smem + S::O_STAGE);
      T                  *pring = reinterpret_cast<T *>(smem + S::O_PRING);
      T                  *zs    = reinterpret_cast<T *>(smem + S::O_ZS);
      T                  *ds    = reinterpret_cast<T *>(smem + S::O_DS);
      LV                 *yx    = reinterpret_cast<LV *>(smem + S::O_YX);
      T                  *hx    = reinterpret_cast<T *>(smem + S::O_HX);
      double             *red   = reinterpret_cast<double *>(smem + S::O_RED);
      unsigned long long *bar   = reinterpret_cast<unsigned long long *>(smem + S::O_BAR);
      __shared__ unsigned s_last;

      if (a.st->done)
        return;
      const T   alpha = FIRST ? T(0) : (T)a.st->alpha;
      const T   beta  = FIRST ? T(0) : (T)a.st->beta;
      const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
      const int tile = blockIdx.x;
      const int n0 = a.n[0], n1 = a.n[1], n2 = a.n[2];
      const long long plane_stride = (long long)a.P0 * n1;

      // thread's cell: main rows (warp < TY), halo row (warp == TY), halo column (warp == TY + 1)
      const int  role = warp < TY ? 0 : (warp == TY ? 1 : 2);
      const int  cxl = role == 2 ? -1 : C * lane, cyl = role == 0 ? warp : (role == 1 ? -1 : lane - 1);
      const bool active = role != 2 || lane <= TY;
      const int  sxi = XOFF + 2 * cxl, syi = 2 + 2 * cyl; // staged index of the cell's first point

      // the thread's sums S0, S6, S1, S2, S3 in the working precision (a few hundred terms per thread
      // in FP32); the CTA and grid sums are in double
      T acc[5] = {T(0), T(0), T(0), T(0), T(0)};

      if (tid == 0)
        {
          mbar_init(&bar[0], 1);
          mbar_init(&bar[1], 1);
          asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
      __syncthreads();

      const unsigned box_bytes = (unsigned)(sizeof(T) * S::PLANE);
      unsigned       phase[2]  = {0u, 0u}; // mbarrier parities, carried across the pieces
      bool           failed    = false;

      // fast-diagonalisation tables (k = 2: even block 2 x 2, odd block 1 x 1), read in place from
      // the kernel parameters (constant bank operands, no registers)
      const T *we = a.we, *wo = a.wo, *lam = a.lam;

      // this CTA's range of the (column, cell layer) sequence, as pieces of single columns
      const long long g_end = a.range[tile + 1];
      for (long long gcur = a.range[tile]; gcur < g_end;)
        {
          // sequence position -> (slab, column, layer); only the last slab may be lower
          const long long ncol = (long long)a.tiles_x * a.tiles_y;
          const int       sl   = (int)(gcur / (ncol * a.slab));
          const int       hs   = min(a.slab, a.m[2] - sl * a.slab); // height of this slab
          const long long off  = gcur - (long long)sl * ncol * a.slab;
          const long long col  = off / hs;
          const int       cz0  = sl * a.slab + (int)(off - col * hs);
          const int       cz1  = (int)min((long long)(sl * a.slab + hs), (long long)cz0 + (g_end - gcur));
          gcur += cz1 - cz0;
          const int  txi = (int)(col % a.tiles_x), tyi = (int)(col / a.tiles_x);
          const int  cx0 = TX * txi, cy0 = TY * tyi;
          const int  lz_begin = cz0 > 0 ? cz0 - 1 : 0;
          const int  XB = 2 * cx0 - XOFF, Y0 = 2 * cy0 - 2;
          const int  cx = cx0 + cxl, cy = cy0 + cyl;
          const bool vxy    = active && cx >= 0 && cx < a.m[0] && cy >= 0 && cy < a.m[1];
          const bool last_x = cx == a.m[0] - 1, last_y = cy == a.m[1] - 1;
          // the second cell of the lane (two cells per lane; the halo column has one)
          const bool vx1 = C == 2 && role != 2 && vxy && cx + 1 < a.m[0];

          auto issue = [&](int slot, int L) {
            // one thread: the plane L of every staged vector into slot
            T *base = stage + (size_t)slot * NV * (S::STAGE_B / sizeof(T));
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect_tx(&bar[slot], (FIRST ? 2u : (unsigned)NV) * box_bytes);
            const size_t vs = S::STAGE_B / sizeof(T);
            tma_load_3d(base + 0 * vs, &tm_r, XB, Y0, L, &bar[slot]);
            if constexpr (!FIRST)
              {
                tma_load_3d(base + 1 * vs, &tm_v, XB, Y0, L, &bar[slot]);
                tma_load_3d(base + 2 * vs, &tm_p, XB, Y0, L, &bar[slot]);
                tma_load_3d(base + 3 * vs, &tm_x, XB, Y0, L, &bar[slot]);
              }
            tma_load_3d(base + 4 * vs, &tm_d, XB, Y0, L, &bar[slot]);
          };

          const int  Pfirst = 2 * lz_begin, Plast = 2 * cz1; // planes of the segment (with its halo)
          if (tid == 0)
            {
              issue(0, Pfirst);
              if (Pfirst + 1 <= Plast)
                issue(1, Pfirst + 1);
            }

          auto owned_z = [&](int L) { return L >= 2 * cz0 && L < n2 && (L < 2 * cz1 || L == n2 - 1); };
          auto constrained_xy = [&](int I, int J) {
            const unsigned f = a.faces;
            return ((f & 1u) && I == 0) || ((f & 2u) && I == n0 - 1) || ((f & 4u) && J == 0) ||
                   ((f & 8u) && J == n1 - 1);
          };

          // The update works on units of W consecutive staged points, one aligned vector per vector
          // and unit: pairs in FP64, quads (16 bytes) in FP32.  The thread's units of a staged plane
          // and their plane-independent parts (at most PR units) are packed into one word: the staged
          // index (12 bits) and the flags; the window index of z and d follows from the staged index,
          // (row - 2) OXW + (x - XOFF).
          constexpr int W  = sizeof(T) == 4 ? 4 : 2;
          constexpr int UR = W == 4 ? SX / 4 : SX / 2 - 2; // units per staged row (quads: all 72 x)
          constexpr int NU = UR * S::RY;
          constexpr int PR = (NU + S::NT - 1) / S::NT;
          constexpr unsigned F_VALID = 1u, F_JOWN = 2u, F_WIN = 4u, F_IN = 8u, F_CON = 8u << W, F_OWN = 8u << (2 * W);
          static_assert(S::PLANE < 4096 && 12 + 3 + 3 * W <= 32, "staged index and flags must fit one word");
          // a tile that takes a whole SM keeps the words in registers; at two CTAs per SM the
          // registers are short and the words are recomputed per plane
          constexpr bool KEEP = S::BYTES > 112 * 1024;
          auto unit_word = [&](int k) {
              const int q   = tid + k * S::NT;
              const int row = q / UR, uu = q - row * UR;
              const int xi  = W == 4 ? 4 * uu : 2 + 2 * uu; // staged x index of the unit's first point
              const int I   = XB + xi, J = Y0 + row;         // lattice coordinates of that point
              unsigned   f   = q < NU ? F_VALID : 0u;
              const bool Jin = J >= 0 && J < n1;
              if (J >= 2 * cy0 && J < n1 && (J < 2 * cy0 + 2 * TY || J == n1 - 1))
                f |= F_JOWN;
#pragma unroll
              for (int h = 0; h < W; ++h)
                {
                  const int Ih = I + h;
                  if (Jin && Ih >= 0 && Ih < n0)
                    f |= F_IN << h;
                  if (constrained_xy(Ih, J))
                    f |= F_CON << h;
                  // the lattice's last point belongs to the tile whose cells end there (a quad of the
                  // tile to its left may reach it too)
                  if (Ih >= 2 * cx0 && Ih < n0 && (Ih < 2 * cx0 + 2 * TX || (Ih == n0 - 1 && Ih == 2 * cx0 + 2 * TX)))
                    f |= F_OWN << h;
                }
              if (I - 2 * cx0 >= 0 && I - 2 * cx0 <= OXW - W && (f & F_JOWN))
                f |= F_WIN;
              return (f & F_VALID) ? (unsigned)(row * SX + xi) | (f << 12) : 0u;
          };
          unsigned pr_w[KEEP ? PR : 1];
          if constexpr (KEEP)
#pragma unroll
            for (int k = 0; k < PR; ++k)
              pr_w[k] = unit_word(k);

          // ---- U stage of plane L: vector updates on every staged point the cells read; owned points
          // are written back and summed
          auto update_plane = [&](int L) {
            const int slot = (L - Pfirst) & 1;
            if (!mbar_wait(&bar[slot], phase[slot], a.spin_limit))
              failed = true;
            phase[slot] ^= 1u;
            const T *sb   = stage + (size_t)slot * NV * (S::STAGE_B / sizeof(T));
            const size_t vs = S::STAGE_B / sizeof(T);
            const T *sr = sb, *sv = sb + vs, *sp = sb + 2 * vs, *sxv = sb + 3 * vs, *sd = sb + 4 * vs;
            T       *pr = pring + (size_t)(L % 3) * (S::STAGE_B / sizeof(T));
            T       *zr = zs + (size_t)(L % 3) * S::OPL, *dr = ds + (size_t)(L % 3) * S::OPL;
            const bool Lin = L >= 0 && L < n2, Lown = owned_z(L);
            const bool Lcon = ((a.faces & 16u) && L == 0) || ((a.faces & 32u) && L == n2 - 1);
            const long long gL = (long long)L * plane_stride;
#pragma unroll
            for (int k = 0; k < PR; ++k)
              {
                const unsigned w = KEEP ? pr_w[KEEP ? k : 0] : unit_word(k), f = w >> 12;
                if (!(f & F_VALID))
                  continue;
                const int si = (int)(w & 4095u);
                T         rv[W], dv[W], vv[W], pv[W], xv[W];
                vload<T, W>(rv, sr + si);
                vload<T, W>(dv, sd + si);
                if constexpr (!FIRST)
                  {
                    vload<T, W>(vv, sv + si);
                    vload<T, W>(pv, sp + si);
                    vload<T, W>(xv, sxv + si);
                  }
                T pn[W], rn[W], zn[W];
#pragma unroll
                for (int h = 0; h < W; ++h)
                  {
                    const bool free = Lin && (f & (F_IN << h)) && !Lcon && !(f & (F_CON << h));
                    const T    r    = FIRST ? rv[h] : rv[h] - alpha * vv[h];
                    const T    z    = dv[h] * r;
                    rn[h]           = r;
                    zn[h]           = free ? z : T(0);
                    pn[h]           = free ? (FIRST ? z : z + beta * pv[h]) : T(0);
                  }
                vstore<T, W>(pr + si, pn);
                if (Lown && (f & F_JOWN))
                  {
                    // I and P0 are multiples of W: the unit is one aligned vector in global memory
                    const int       row = si / SX, xi = si - row * SX;
                    const long long g   = gL + (long long)(Y0 + row) * a.P0 + (XB + xi);
                    const int       zi  = (row - 2) * OXW + (xi - XOFF);
                    constexpr unsigned ALL = ((1u << W) - 1u) * F_OWN;
                    T xn[W];
#pragma unroll
                    for (int h = 0; h < W; ++h)
                      xn[h] = xv[h] + alpha * pv[h];
                    if ((f & ALL) == ALL)
                      {
                        if constexpr (!FIRST)
                          {
                            vstore<T, W>(a.x + g, xn);
                            vstore<T, W>(a.r_out + g, rn);
                          }
                        vstore<T, W>(a.p_out + g, pn);
                      }
                    else
#pragma unroll
                      for (int h = 0; h < W; ++h)
                        if (f & (F_OWN << h))
                          {
                            if constexpr (!FIRST)
                              {
                                a.x[g + h]     = xn[h];
                                a.r_out[g + h] = rn[h];
                              }
                            a.p_out[g + h] = pn[h];
                          }
                    // z and d of the owned window (points outside it are never read)
                    if (f & F_WIN)
                      {
                        vstore<T, W>(zr + zi, zn);
                        vstore<T, W>(dr + zi, dv);
                      }
#pragma unroll
                    for (int h = 0; h < W; ++h)
                      if (f & (F_OWN << h))
                        {
                          acc[0] = fma(rn[h], zn[h], acc[0]);
                          acc[1] = fma(rn[h], rn[h], acc[1]);
                        }
                  }
              }
          };

          auto refill = [&](int L_done) {
            // the slot of plane L_done is free once every thread passed the barrier before this call
            const int Ln = L_done + 2;
            if (tid == 0 && Ln <= Plast)
              issue((L_done - Pfirst) & 1, Ln);
          };

          update_plane(Pfirst);
          __syncthreads();
          refill(Pfirst);

          // a scalar as the lane's value type, and one cell's component of a lane value
          auto bc = [](T x) -> LV {
            if constexpr (C == 2)
              return f2(x);
            else
              return x;
          };
          auto comp = [](const LV &v, int c) -> T {
            if constexpr (C == 2)
              return c ? v.v.y : v.v.x;
            else
              return v;
          };
          LV carry[N * N];
#pragma unroll
          for (int q = 0; q < N * N; ++q)
            carry[q] = bc(T(0));

          for (int lz = lz_begin; lz < cz1; ++lz)
            {
              const bool halo_layer = lz < cz0;
              // conductivity of the lane's cells
              auto kload = [&](int x, bool v) -> T {
                if (!v)
                  return T(0);
                return a.kcell ? a.kcell[(long long)x + (long long)a.m[0] * ((long long)cy + (long long)a.m[1] * lz)]
                               : a.kconst;
              };
              LV kc;
              if constexpr (C == 2)
                kc = f2(kload(cx, vxy), kload(cx + 1, vx1));
              else
                kc = kload(cx, vxy);
              // both planes of the layer, then one barrier before their slots are refilled and the
              // cells read the p ring
              update_plane(2 * lz + 1);
              update_plane(2 * lz + 2);
              __syncthreads();
              refill(2 * lz + 1);
              refill(2 * lz + 2);

              // ---- cell stage: u = A_c p_c for the lane's cells
              LV u[N * N * N];
#pragma unroll
              for (int l = 0; l < N; ++l)
                {
                  const T *pl = pring + (size_t)((2 * lz + l) % 3) * (S::STAGE_B / sizeof(T));
#pragma unroll
                  for (int j = 0; j < N; ++j)
                    {
                      const T *row = pl + (syi + j) * SX + sxi;
                      if constexpr (C == 2)
                        {
                          // the two cells' 5 points of the row: one aligned quad and one more (the
                          // halo column: its single cell, an aligned pair and one more)
                          T r[5] = {T(0), T(0), T(0), T(0), T(0)};
                          if (vxy)
                            {
                              if (role != 2)
                                {
                                  const float4 q4 = *reinterpret_cast<const float4 *>(row);
                                  r[0] = q4.x, r[1] = q4.y, r[2] = q4.z, r[3] = q4.w;
                                  r[4] = row[4];
                                }
                              else
                                {
                                  const PV q2 = *reinterpret_cast<const PV *>(row);
                                  r[0] = q2.x, r[1] = q2.y, r[2] = row[2];
                                }
                            }
#pragma unroll
                          for (int i = 0; i < N; ++i)
                            u[(l * N + j) * N + i] = f2(r[i], vx1 ? r[i + 2] : T(0));
                        }
                      else
                        {
                          // sxi and SX are even: points 0, 1 of the row are one aligned pair
                          const PV p01 = vxy ? *reinterpret_cast<const PV *>(row) : PV{T(0), T(0)};
                          u[(l * N + j) * N + 0] = p01.x;
                          u[(l * N + j) * N + 1] = p01.y;
                          u[(l * N + j) * N + 2] = vxy ? row[2] : T(0);
                        }
                    }
                }
              {
                const LV kcx = kc * bc(a.cx), kcy = kc * bc(a.cy), kcz = kc * bc(a.cz), am = bc(a.alpha_m);
                xy_planes<LV, N, N, true, T>(u, we, wo);
#pragma unroll
                for (int q = 0; q < N * N; ++q)
                  fwd_line<LV, N, N * N, T>(u, q, we, wo);
                LV form = bc(T(0));
#pragma unroll
                for (int c = 0; c < N; ++c)
                  {
                    const LV tz = fma(kcz, bc(lam[c]), am);
#pragma unroll
                    for (int b = 0; b < N; ++b)
                      {
                        const LV tyz = fma(kcy, bc(lam[b]), tz);
#pragma unroll
                        for (int aa = 0; aa < N; ++aa)
                          {
                            const LV d = fma(kcx, bc(lam[aa]), tyz);
                            LV      &v = u[(c * N + b) * N + aa];
                            form       = fma(d * v, v, form);
                            v *= d;
                          }
                      }
                  }
                if (role == 0 && !halo_layer)
                  {
                    if (vxy)
                      acc[2] += comp(form, 0);
                    if (C == 2 && vx1)
                      acc[2] += comp(form, 1);
                  }
#pragma unroll
                for (int q = 0; q < N * N; ++q)
                  bwd_line<LV, N, N * N, T>(u, q, we, wo);
                xy_planes<LV, N, N, false, T>(u, we, wo);
              }
              // ---- faces.  FP64 takes the y faces first: the main rows and the halo row hand their
              // cells' y = 2 faces to the next row through shared memory; the halo column, whose lanes
              // are consecutive rows, adds its lower neighbour's y = 2 face by a shuffle and hands its
              // x = 2 face to lane 0 of every row; after one barrier the main rows add the lower row's
              // faces and then the left neighbour's x = 2 faces (which by then hold their own lower
              // neighbours' parts).  FP32 takes the x faces first (halo column through shared memory,
              // barrier, shuffles) and then the y faces, one barrier more per layer but measured
              // faster there (206 against 223 us per iteration).  Either way every owned point ends up
              // with the contributions of all the cells that share it.
              constexpr bool YFIRST = sizeof(T) == 8;
              if (role == 2)
                {
                  if constexpr (YFIRST)
#pragma unroll
                    for (int l = 0; l < N; ++l)
#pragma unroll
                      for (int i = 0; i < N; ++i)
                        {
                          const LV &f = u[(l * N + K) * N + i];
                          LV        b;
                          if constexpr (C == 2)
                            b = f2(__shfl_up_sync(0xffffffffu, f.v.x, 1), __shfl_up_sync(0xffffffffu, f.v.y, 1));
                          else
                            b = __shfl_up_sync(0xffffffffu, f, 1);
                          if (lane > 0)
                            u[(l * N) * N + i] += b;
                        }
                  if (active)
#pragma unroll
                    for (int q = 0; q < N * N; ++q)
                      hx[lane * 9 + q] = comp(u[q * N + K], 0);
                }
              if constexpr (!YFIRST)
                {
                  __syncthreads();
                  if (role != 2)
                    {
                      const int hrow = role == 0 ? warp + 1 : 0; // halo column lane of this row
#pragma unroll
                      for (int q = 0; q < N * N; ++q)
                        {
                          if constexpr (C == 2)
                            {
                              // the lane's second cell takes its first cell's x = 2 face; the first cell
                              // takes the x = 2 face of the left lane's second cell
                              const T v = __shfl_up_sync(0xffffffffu, u[q * N + K].v.y, 1);
                              u[q * N].v.y += u[q * N + K].v.x;
                              u[q * N].v.x += lane > 0 ? v : hx[hrow * 9 + q];
                            }
                          else
                            {
                              const T v = __shfl_up_sync(0xffffffffu, u[q * N + K], 1);
                              u[q * N] += lane > 0 ? v : hx[hrow * 9 + q];
                            }
                        }
                    }
                }
              if (role != 2)
                {
                  const int slot = role == 0 ? warp : TY;
#pragma unroll
                  for (int l = 0; l < N; ++l)
#pragma unroll
                    for (int i = 0; i < N; ++i)
                      yx[((slot * N + l) * N + i) * 32 + lane] = u[(l * N + K) * N + i];
                }
              __syncthreads();
              if (role == 0)
                {
                  const int from = warp == 0 ? TY : warp - 1;
#pragma unroll
                  for (int l = 0; l < N; ++l)
#pragma unroll
                    for (int i = 0; i < N; ++i)
                      u[(l * N) * N + i] += yx[((from * N + l) * N + i) * 32 + lane];
                  if constexpr (YFIRST)
                    {
                      const int hrow = warp + 1; // halo column lane of this row
#pragma unroll
                      for (int q = 0; q < N * N; ++q)
                        {
                          if constexpr (C == 2)
                            {
                              // the lane's second cell takes its first cell's x = 2 face; the first cell
                              // takes the x = 2 face of the left lane's second cell
                              const T v = __shfl_up_sync(0xffffffffu, u[q * N + K].v.y, 1);
                              u[q * N].v.y += u[q * N + K].v.x;
                              u[q * N].v.x += lane > 0 ? v : hx[hrow * 9 + q];
                            }
                          else
                            {
                              const T v = __shfl_up_sync(0xffffffffu, u[q * N + K], 1);
                              u[q * N] += lane > 0 ? v : hx[hrow * 9 + q];
                            }
                        }
                    }
                  // z faces: add the carried face, carry this layer's z = 2 face
#pragma unroll
                  for (int q = 0; q < N * N; ++q)
                    {
                      u[q] += carry[q];
                      carry[q] = u[K * N * N + q];
                    }
                  // ---- owned points of the finished planes: v_k, S2, S3
                  if (!halo_layer && vxy)
                    {
                      const int nl = lz == a.m[2] - 1 ? 3 : 2;
                      for (int l = 0; l < nl; ++l)
                        {
                          const int  L    = 2 * lz + l;
                          const T   *zl   = zs + (size_t)(L % 3) * S::OPL, *dl = ds + (size_t)(L % 3) * S::OPL;
                          const bool Lcon = ((a.faces & 16u) && L == 0) || ((a.faces & 32u) && L == n2 - 1);
#pragma unroll
                          for (int j = 0; j < N; ++j)
                            {
                              if (j == K && !last_y)
                                continue;
                              const int  J    = 2 * cy + j;
                              T         *vrow = a.v_out + (long long)L * plane_stride + (long long)J * a.P0;
                              const bool Jcon = Lcon || ((a.faces & 4u) && J == 0) || ((a.faces & 8u) && J == n1 - 1);
#pragma unroll
                              for (int c = 0; c < C; ++c)
                                {
                                  if (c == 1 && !vx1)
                                    continue;
                                  const int  xc = cx + c;
                                  const bool lx = xc == a.m[0] - 1;
                                  const int  o0 = (J - 2 * cy0) * OXW + 2 * (xc - cx0); // even: aligned pairs
                                  const PV   z01 = *reinterpret_cast<const PV *>(zl + o0);
                                  const PV   d01 = *reinterpret_cast<const PV *>(dl + o0);
                                  const T    zz[N] = {z01.x, z01.y, lx ? zl[o0 + 2] : T(0)};
                                  const T    dd[N] = {d01.x, d01.y, lx ? dl[o0 + 2] : T(0)};
                                  T          vv[N];
                                  T          s2 = T(0), s3 = T(0);
#pragma unroll
                                  for (int i = 0; i < N; ++i)
                                    {
                                      const int  I   = 2 * xc + i;
                                      const bool con = Jcon || ((a.faces & 1u) && I == 0) || ((a.faces & 2u) && I == n0 - 1);
                                      vv[i]          = con ? T(0) : comp(u[(l * N + j) * N + i], c);
                                      if (i < K || lx)
                                        {
                                          s2 = fma(zz[i], vv[i], s2);
                                          s3 = fma(dd[i] * vv[i], vv[i], s3);
                                        }
                                    }
                                  acc[3] += s2;
                                  acc[4] += s3;
                                  *reinterpret_cast<PV *>(vrow + 2 * xc) = PV{vv[0], vv[1]};
                                  if (lx)
                                    vrow[2 * xc + 2] = vv[2];
                                }
                            }
                        }
                    }
                }
              __syncthreads();
            }
        }

      // ---- CTA sums in a fixed order, then the last CTA adds the tiles in order and steps the state
#pragma unroll
      for (int k = 0; k < 5; ++k)
        {
          double v = (double)acc[k];
#pragma unroll
          for (int off = 16; off > 0; off >>= 1)
            v += __shfl_down_sync(0xffffffffu, v, off);
          if (lane == 0)
            red[warp * 5 + k] = v;
        }
      __syncthreads();
      const int ntiles = gridDim.x;
      if (tid < 5)
        {
          double t = 0.0;
          for (int w = 0; w < S::NW; ++w)
            t += red[w * 5 + tid];
          a.part[(size_t)tid * ntiles + tile] = t;
        }
      if (failed)
        atomicExch(a.err, 3);
      __syncthreads();
      if (tid == 0)
        {
          __threadfence();
          s_last = atomicAdd(a.counter, 1u) == (unsigned)ntiles - 1 ? 1u : 0u;
        }
      __syncthreads();
      if (!s_last)
        return;
      __threadfence();
      for (int k = 0; k < 5; ++k)
        {
          double t = 0.0;
          for (int i = tid; i < ntiles; i += S::NT)
            t += __ldcg(a.part + (size_t)k * ntiles + i);
#pragma unroll
          for (int off = 16; off > 0; off >>= 1)
            t += __shfl_down_sync(0xffffffffu, t, off);
          if (lane == 0)
            red[warp * 5 + k] = t;
        }
      __syncthreads();
      if (tid == 0)
        {
          double s[5];
          for (int k = 0; k < 5; ++k)
            {
              s[k] = 0.0;
              for (int w = 0; w < S::NW; ++w)
                s[k] += red[w * 5 + k];
            }
          CGState    &st  = *a.st;
          const double res = sqrt(s[1]);
          int          it  = 0;
          if (FIRST)
            {
              st.res0 = res;
              st.tol  = fmax(st.abs_tol, st.rel_tol * res);
            }
          else
            it = st.it + 1;
          st.it  = it;
          st.res = res;
          if (a.hist)
            a.hist[it] = res;
          const double rho   = s[0];
          const double alph  = rho / s[2];
          const double rho_n = rho - 2.0 * alph * s[3] + alph * alph * s[4];
          st.rho             = rho;
          st.alpha           = alph;
          st.beta            = rho_n / rho;
          st.done            = control_check(st, it, res);
          *a.counter         = 0u;
          __threadfence();
        }
    }
  } // namespace cgf

  // ------------------------------------------------------------------------------------------
  // host side

  namespace
  {
    PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
    {
      static std::once_flag                    once;
      static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
      std::call_once(once, [] {
        void                          *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
          fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
      });
      return fn;
    }
  } // namespace

  template <typename T>
  int
  FusedCG<T>::make_map(CUtensorMap *map, const T *base) const
  {
    auto fn = encode_fn();
    if (!fn)
      return 1;
    const int       TY   = sizeof(T) == 8 ? FUSED_TY_F64 : FUSED_TY_F32;
    cuuint64_t      dims[3]    = {(cuuint64_t)n[0], (cuuint64_t)n[1], (cuuint64_t)n[2]};
    cuuint64_t      strides[2] = {(cuuint64_t)P0 * sizeof(T), (cuuint64_t)P0 * n[1] * sizeof(T)};
    cuuint32_t      box[3]     = {(cuuint32_t)cgf::Shape<T, sizeof(T) == 8 ? FUSED_TY_F64 : FUSED_TY_F32>::SX,
                                  (cuuint32_t)(2 * TY + 3), 1u};
    cuuint32_t      estr[3]    = {1u, 1u, 1u};
    const CUresult  r = fn(map, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                          const_cast<T *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : 2;
  }

  template <typename T>
  size_t
  FusedCG<T>::smem_bytes()
  {
    return sizeof(T) == 8 ? cgf::Shape<double, FUSED_TY_F64>::BYTES : cgf::Shape<float, FUSED_TY_F32>::BYTES;
  }

  template <typename T>
  int
  FusedCG<T>::threads()
  {
    return sizeof(T) == 8 ? cgf::Shape<double, FUSED_TY_F64>::NT : cgf::Shape<float, FUSED_TY_F32>::NT;
  }

  template <typename T>
  void
  FusedCG<T>::plan(int sm_count)
  {
    const int TY = sizeof(T) == 8 ? FUSED_TY_F64 : FUSED_TY_F32;
    constexpr int TXC = cgf::Shape<T, sizeof(T) == 8 ? FUSED_TY_F64 : FUSED_TY_F32>::TX;
    tiles_x      = (m[0] + TXC - 1) / TXC;
    tiles_y      = (m[1] + TY - 1) / TY;
    // CTAs resident per SM from the shared memory footprint (227 KB usable per CTA, 228 KB per SM)
    const int per_sm = std::max(1, (int)(233472 / (smem_bytes() + 1024)));
    // one CTA per resident slot, each with an equal share of the columns' layers; a share below
    // four layers would spend more on its halo layer than it saves, so small lattices use fewer CTAs
    // (at 48^3 a floor of 8 or 16 layers measured 1.5x / 2.5x slower: more CTAs win down to 4)
    layers = (long long)tiles_x * tiles_y * m[2];
    ntiles = (int)std::max(1LL, std::min((long long)sm_count * per_sm, layers / 4));
    // slabs about one share high, so that the CTAs working at the same time hold neighbouring
    // columns at about the same layers and read each other's halo planes from L2
    slab = (int)std::max(1LL, std::min((long long)m[2], (layers + ntiles / 2) / ntiles));
    // ranges of equal cost: a piece costs its layers plus about 1.5 (its halo layer and the
    // staging ramp), so CTAs whose range is cut into short pieces (the last, lower slab) take
    // fewer layers; the smallest cost bound that needs at most ntiles ranges, by bisection
    const long long ncol = (long long)tiles_x * tiles_y;
    auto greedy = [&](double bound, std::vector<long long> *out) {
      long long n = 0, pos = 0;
      double    cost = 0.0;
      bool      open = false;
      if (out)
        out->assign(1, 0);
      for (int z0 = 0; z0 < m[2]; z0 += slab)
        {
          const int hs = std::min(slab, m[2] - z0);
          for (long long c = 0; c < ncol; ++c)
            {
              long long left = hs;
              while (left > 0)
                {
                  long long take = (long long)std::floor(bound - cost - 1.5);
                  if (take <= 0)
                    {
                      if (!open) // a bound below one layer per piece: take one anyway
                        take = 1;
                      else
                        {
                          ++n;
                          if (out)
                            out->push_back(pos);
                          cost = 0.0;
                          open = false;
                          continue;
                        }
                    }
                  take = std::min(take, left);
                  cost += (double)take + 1.5;
                  open = true;
                  pos += take;
                  left -= take;
                }
            }
        }
      if (open)
        {
          ++n;
          if (out)
            out->push_back(pos);
        }
      return n;
    };
    double lo = (double)layers / ntiles, hi = lo + 3.0 * (1.5 + slab);
    for (int it = 0; it < 60; ++it)
      {
        const double mid = 0.5 * (lo + hi);
        if (greedy(mid, nullptr) <= ntiles)
          hi = mid;
        else
          lo = mid;
      }
    greedy(hi, &range);
    while ((long long)range.size() < ntiles + 1LL) // fewer ranges than CTAs: empty ranges at the end
      range.push_back(layers);
  }

  template <typename T>
  cudaError_t
  FusedCG<T>::sweep(bool first, const CUtensorMap &r_in, const CUtensorMap &v_in, const CUtensorMap &p_in,
                    const CUtensorMap &x, const CUtensorMap &d, T *x_ptr, T *r_out, T *p_out, T *v_out,
                    CGState *st, double *part, unsigned *counter, double *hist, int *err, unsigned spin_limit,
                    cudaStream_t s) const
  {
    constexpr int TY = sizeof(T) == 8 ? FUSED_TY_F64 : FUSED_TY_F32;
    cgf::Sweep<T> a{};
    for (int i = 0; i < 3; ++i)
      {
        a.m[i] = m[i];
        a.n[i] = n[i];
      }
    a.P0      = P0;
    a.faces   = faces;
    a.tiles_x = tiles_x;
    a.tiles_y = tiles_y;
    a.layers  = layers;
    a.slab    = slab;
    a.range   = d_range;
    a.ty      = TY;
    a.alpha_m = (T)mass_coef;
    a.cx      = (T)geo[0];
    a.cy      = (T)geo[1];
    a.cz      = (T)geo[2];
    a.kconst  = (T)kconst;
    a.kcell   = kcell;
    const Tables1D &t = tables(2);
    for (int i = 0; i < cgf::NE * cgf::NE; ++i)
      a.we[i] = (T)t.WE[i];
    a.wo[0] = (T)t.WO[0];
    for (int i = 0; i < cgf::N; ++i)
      a.lam[i] = (T)t.lam[i];
    a.x          = x_ptr;
    a.r_out      = r_out;
    a.p_out      = p_out;
    a.v_out      = v_out;
    a.st         = st;
    a.part       = part;
    a.counter    = counter;
    a.hist       = hist;
    a.err        = err;
    a.spin_limit = spin_limit;
    const size_t bytes = smem_bytes();
    if (first)
      {
        auto k = cgf::heat_cg_sweep_kernel<T, TY, true>;
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess)
          return e;
        k<<<ntiles, threads(), bytes, s>>>(a, r_in, v_in, p_in, x, d);
      }
    else
      {
        auto k = cgf::heat_cg_sweep_kernel<T, TY, false>;
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess)
          return e;
        k<<<ntiles, threads(), bytes, s>>>(a, r_in, v_in, p_in, x, d);
      }
    return cudaGetLastError();
  }

  // padded layout conversions: rows of n0 entries <-> rows of P0 entries (padding zero)
  template <typename Td, typename Ts>
  __global__ void
  pad_rows_kernel(Td *dst, const Ts *src, int n0, int P0, long long rows)
  {
    for (long long row = blockIdx.x; row < rows; row += gridDim.x)
      for (int i = threadIdx.x; i < P0; i += blockDim.x)
        dst[row * P0 + i] = i < n0 ? (Td)src[row * n0 + i] : Td(0);
  }
  template <typename Td, typename Ts>
  __global__ void
  unpad_rows_kernel(Td *dst, const Ts *src, int n0, int P0, long long rows)
  {
    for (long long row = blockIdx.x; row < rows; row += gridDim.x)
      for (int i = threadIdx.x; i < n0; i += blockDim.x)
        dst[row * n0 + i] = (Td)src[row * P0 + i];
  }

  template <typename Td, typename Ts>
  cudaError_t
  pad_rows(Td *dst, const Ts *src, int n0, int P0, long long rows, cudaStream_t s)
  {
    pad_rows_kernel<Td, Ts><<<(int)std::min<long long>(rows, 148LL * 16), 256, 0, s>>>(dst, src, n0, P0, rows);
    return cudaGetLastError();
  }
  template <typename Td, typename Ts>
  cudaError_t
  unpad_rows(Td *dst, const Ts *src, int n0, int P0, long long rows, cudaStream_t s)
  {
    unpad_rows_kernel<Td, Ts><<<(int)std::min<long long>(rows, 148LL * 16), 256, 0, s>>>(dst, src, n0, P0, rows);
    return cudaGetLastError();
  }

  template struct FusedCG<double>;
  template struct FusedCG<float>;
  template cudaError_t pad_rows<double, double>(double *, const double *, int, int, long long, cudaStream_t);
  template cudaError_t pad_rows<float, float>(float *, const float *, int, int, long long, cudaStream_t);
  template cudaError_t unpad_rows<double, double>(double *, const double *, int, int, long long, cudaStream_t);
  template cudaError_t unpad_rows<float, float>(float *, const float *, int, int, long long, cudaStream_t);
} // namespace mpdg
