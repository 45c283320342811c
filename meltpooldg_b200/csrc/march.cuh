// Column-marching apply for low degrees (k <= 2): one thread per cell, no shared-memory reduction.
//
// A CTA of 4 warps owns a column of 32 x 4 cells (x, y) and marches through a segment of BZ cell
// layers in z.  Lane = cell x-index, warp = cell y-index.  Per layer:
//   1. the (k+1) lattice planes of the layer are staged into shared memory with cp.async (double
//      buffered: the next layer is in flight while the current one is computed);
//   2. each thread applies the cell operator to its cell's (k+1)^3 values in registers;
//   3. x-neighbours combine their common face with warp shuffles (lane t adds lane t-1's x = k face
//      into its x = 0 face), y-neighbours through a small shared exchange buffer, z-neighbours by
//      carrying the z = k face in registers to the next layer of the same thread;
//   4. each thread then owns the points i, j, l in [0, k) of its cell (plus the column's high faces
//      for the last lane / warp / layer) and writes them to global memory with coalesced stores.
// Points on the faces shared with neighbouring columns / segments are combined with global atomics,
// initialised by their owner through the ticket / flag handshake of brick.cuh.
#pragma once

#include "brick.cuh"

namespace mpdg
{
#ifndef MPDG_MARCH_BZ2_F32
#define MPDG_MARCH_BZ2_F32 16
#endif
  // Cell layers per column segment: longer segments amortise the brick handshake and the staging
  // prologue; for k = 2 in FP64 the 8-layer segment gives more CTAs per wave and wins.
  template <int K, typename T>
  struct MarchShape
  {
    static constexpr int BX = 32, BY = 4, NT = 128;
    static constexpr int BZ = K == 1 ? 16 : (sizeof(T) == 4 ? MPDG_MARCH_BZ2_F32 : 8);
  };

  template <int K, typename T>
  struct MarchLayout
  {
    using S                 = MarchShape<K, T>;
    static constexpr int N  = K + 1;
    static constexpr int PX = K * S::BX + 1, PY = K * S::BY + 1, NPL = K + 1;
    static constexpr int LAYER = NPL * PY * PX;           // staged points per layer
    static constexpr int YX    = S::BY * N * N * 32;      // y-exchange buffer
    static constexpr size_t bytes = sizeof(T) * (2 * (size_t)LAYER + YX);
    using BR = Brick<K, S::BX, S::BY, S::BZ, S::NT>;      // geometry / handshake of the column segment
  };

  // Stage layer lz of the column into buf (cp.async; zeros outside the domain and, with mask, on
  // Dirichlet planes -- decided per row plus two compares per point).
  template <class LAY, class BR, typename T>
  __device__ __forceinline__ void
  march_stage(const BR &br, int lz, const T *src, bool mask, T *buf)
  {
    constexpr int K = LAY::N - 1;
    constexpr int PX = LAY::PX, PY = LAY::PY, NR = LAY::NPL * PY;
    const int     lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool    mx0 = mask && br.con_lo[0], mx1 = mask && br.con_hi[0];
    for (int r = warp; r < NR; r += LAY::S::NT / 32)
      {
        const int  l = r / PY, py = r % PY, pz = K * lz + l;
        const bool rowcon = mask && ((br.con_lo[1] && py == 0) || (br.con_hi[1] && py == br.nv[1] - 1) ||
                                     (br.con_lo[2] && pz == 0) || (br.con_hi[2] && pz == br.nv[2] - 1));
        const bool rowv    = py < br.nv[1] && pz < br.nv[2] && !rowcon;
        const int  rowbase = br.g0[0] + br.sy * (br.g0[1] + py) + br.sz * (br.g0[2] + pz);
#pragma unroll
        for (int c = 0; c < (PX + 31) / 32; ++c)
          {
            const int px = lane + 32 * c;
            if (px >= PX)
              break;
            const bool valid = rowv && px < br.nv[0] && !(mx0 && px == 0) && !(mx1 && px == br.nv[0] - 1);
            cp_async_elem(buf + r * PX + px, src + (valid ? rowbase + px : 0), valid);
          }
      }
    asm volatile("cp.async.commit_group;" ::: "memory");
  }

  // The marching body.  Cell operator: Op::apply(u, valid, cx, cy, cz) in place on (k+1)^3 values.
  // With DOT the cell operator returns the cell's form src_c^T A_c src_c and the sum over the brick
  // goes to the fused dot product (release_ticket_dot).
  template <int K, typename T, OutMode MODE, class Op, bool DOT = false>
  __device__ __forceinline__ void
  march_body(const GridDesc &g, const SyncDesc &s, const T *src, T *dst, const T *bvec, bool mask_src, const Op &op,
             T *smem, unsigned *s_ticket, const DotSink &dot = DotSink{}, double *s_red = nullptr)
  {
    double dsum = 0.0;
    using LAY       = MarchLayout<K, T>;
    using BR        = typename LAY::BR;
    constexpr int N = K + 1, PX = LAY::PX, PY = LAY::PY, BZ = LAY::S::BZ;
    T *buf0 = smem, *buf1 = smem + LAY::LAYER, *yx = smem + 2 * LAY::LAYER;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    BR        br;
    if (!brick_begin<BR, T, MODE>(br, g, s, dst, bvec, s_ticket))
      return;
    if constexpr (MODE != OutMode::Add)
      if (br.has_lower_neighbour())
        brick_wait_lower(br, g, s);
    const int  cx = br.c0[0] + lane, cy = br.c0[1] + warp;
    const bool vxy       = cx < g.m[0] && cy < g.m[1];
    const bool last_lane = cx == min(br.c0[0] + 32, g.m[0]) - 1;
    const bool last_warp = cy == min(br.c0[1] + 4, g.m[1]) - 1;
    const int  nlayers   = min(BZ, g.m[2] - br.c0[2]);
    const bool do_mask   = mask_src && br.any_con; // only bricks on a constrained face pay for masking
    // flags: x / y faces shared with the lower neighbour columns, Dirichlet planes through the cell
    const bool cI0 = br.con_lo[0] && cx == 0, cIK = br.con_hi[0] && K * cx + K == g.n[0] - 1;
    const bool cJ0 = br.con_lo[1] && cy == 0, cJK = br.con_hi[1] && K * cy + K == g.n[1] - 1;
    T carry[N * N];
#pragma unroll
    for (int q = 0; q < N * N; ++q)
      carry[q] = T(0);
    const int cbase0 = (br.g0[0] + K * lane) + br.sy * (br.g0[1] + K * warp) + br.sz * br.g0[2];
    march_stage<LAY>(br, 0, src, do_mask, buf0);
    for (int lz = 0; lz < nlayers; ++lz)
      {
        T *cur = (lz & 1) ? buf1 : buf0;
        if (lz + 1 < nlayers)
          {
            march_stage<LAY>(br, lz + 1, src, do_mask, (lz & 1) ? buf0 : buf1);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
          }
        else
          asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncthreads();
        const bool last_layer = lz == nlayers - 1;
        const int  cz         = br.c0[2] + lz;
        T          u[N * N * N];
#pragma unroll
        for (int l = 0; l < N; ++l)
#pragma unroll
          for (int j = 0; j < N; ++j)
#pragma unroll
            for (int i = 0; i < N; ++i)
              u[(l * N + j) * N + i] = vxy ? cur[(l * PY + K * warp + j) * PX + K * lane + i] : T(0);
        if constexpr (DOT)
          dsum += op.template apply<true>(u, vxy, cx, cy, cz);
        else
          op.template apply<false>(u, vxy, cx, cy, cz);
        // x: lane t adds lane t-1's x = K face; only the last lane keeps its own
#pragma unroll
        for (int q = 0; q < N * N; ++q)
          {
            const T v = __shfl_up_sync(0xffffffffu, u[q * N + K], 1);
            if (lane > 0)
              u[q * N] += v;
            if (!last_lane)
              u[q * N + K] = T(0);
          }
        // y: warp w adds warp w-1's y = K face; only the last warp keeps its own
#pragma unroll
        for (int l = 0; l < N; ++l)
#pragma unroll
          for (int i = 0; i < N; ++i)
            yx[((warp * N + l) * N + i) * 32 + lane] = u[(l * N + K) * N + i];
        __syncthreads();
        if (warp > 0)
#pragma unroll
          for (int l = 0; l < N; ++l)
#pragma unroll
            for (int i = 0; i < N; ++i)
              u[(l * N) * N + i] += yx[(((warp - 1) * N + l) * N + i) * 32 + lane];
        if (!last_warp)
#pragma unroll
          for (int l = 0; l < N; ++l)
#pragma unroll
            for (int i = 0; i < N; ++i)
              u[(l * N + K) * N + i] = T(0);
        // z: add the carried face, carry this layer's z = K face
#pragma unroll
        for (int q = 0; q < N * N; ++q)
          {
            u[q] += carry[q];
            carry[q] = u[K * N * N + q];
          }
        // ---- write-out.  Every brick-face point was initialised by its owner (brick_init_publish),
        // so a face point is an atomic add (skipped on constrained rows) and an interior point a
        // plain store; interior points are never constrained (Dirichlet planes are domain faces).
        if (vxy)
          {
            const int  cbase = cbase0 + br.sz * (K * lz);
            const bool f_x0 = lane == 0, f_y0 = warp == 0, f_z0 = lz == 0;
            const bool cL0 = br.con_lo[2] && cz == 0, cLK = br.con_hi[2] && K * cz + K == g.n[2] - 1;
#define MPDG_PUT(i, j, l)                                                                                      \
  {                                                                                                            \
    const int idx_ = cbase + (j) * br.sy + (l) * br.sz + (i);                                                  \
    const T   v_   = u[((l) * N + (j)) * N + (i)];                                                             \
    const bool face_ = ((i) == 0 && f_x0) || (i) == K || ((j) == 0 && f_y0) || (j) == K || ((l) == 0 && f_z0) || \
                       (l) == K;                                                                               \
    if (face_)                                                                                                 \
      {                                                                                                        \
        const bool cn_ = ((i) == 0 && cI0) || ((i) == K && cIK) || ((j) == 0 && cJ0) || ((j) == K && cJK) ||    \
                         ((l) == 0 && cL0) || ((l) == K && cLK);                                               \
        if (!cn_)                                                                                              \
          atomicAdd(dst + idx_, v_);                                                                           \
      }                                                                                                        \
    else if constexpr (MODE == OutMode::Set)                                                                   \
      dst[idx_] = v_;                                                                                          \
    else if constexpr (MODE == OutMode::Add)                                                                   \
      dst[idx_] += v_;                                                                                         \
    else                                                                                                       \
      dst[idx_] = bvec[idx_] + v_;                                                                             \
  }
#pragma unroll
            for (int l = 0; l < K; ++l)
#pragma unroll
              for (int j = 0; j < K; ++j)
#pragma unroll
                for (int i = 0; i < K; ++i)
                  MPDG_PUT(i, j, l)
            if (last_lane)
#pragma unroll
              for (int l = 0; l < K; ++l)
#pragma unroll
                for (int j = 0; j < K; ++j)
                  MPDG_PUT(K, j, l)
            if (last_warp)
#pragma unroll
              for (int l = 0; l < K; ++l)
#pragma unroll
                for (int i = 0; i < N; ++i)
                  if (i < K || last_lane)
                    MPDG_PUT(i, K, l)
            if (last_layer)
#pragma unroll
              for (int j = 0; j < N; ++j)
#pragma unroll
                for (int i = 0; i < N; ++i)
                  if ((i < K || last_lane) && (j < K || last_warp))
                    MPDG_PUT(i, j, K)
#undef MPDG_PUT
          }
        // no barrier here: the next layer's cp.async staging overwrites the buffer every thread
        // finished reading before this layer's y-exchange barrier, and the next y-exchange writes
        // come after the next layer's first barrier
      }
    if constexpr (DOT)
      release_ticket_dot<LAY::S::NT>(s, dot, br.id, dsum, s_red, s_ticket);
    else if constexpr (MODE != OutMode::Add)
      release_ticket(s);
  }
} // namespace mpdg
