// Pencil-marching apply for higher degrees (k = 3, 4): one thread per x lattice point.
//
// A CTA of K*32 threads owns a brick of 32 x BY x BZ cells.  Thread p holds the "pencil" of the
// current cell row at x lattice point p: the (k+1) x (k+1) values at the y and z lattice points of
// one cell (y row r, z layer lz).  The brick is visited row by row (y inner, z outer); per row step:
//   1. each thread loads its pencil from global memory (coalesced: consecutive threads read
//      consecutive x points) and applies the forward 1-D transforms in z and y in registers;
//   2. the transformed pencils go to shared memory (one column per x point, odd stride: no bank
//      conflicts); the x direction is done per cell and (y, z) mode: read the cell's k+1 values,
//      forward transform, diagonal scale, backward transform, write back -- interior x points in
//      place, the two face points of the cell into separate face buffers;
//   3. each thread reads its x point back (face points add the results of both adjacent cells,
//      so x faces inside the brick are combined without atomics), applies the backward y and z
//      transforms and holds the (k+1)^2 output values of its pencil;
//   4. y faces between the rows of the brick are carried in registers to the next row step, z faces
//      between layers in shared memory to the next layer (per thread, no synchronisation); points
//      owned by the pencil are written with coalesced plain stores; points on the brick's faces
//      are combined with global atomics, initialised by their owner through the ticket / flag
//      handshake of brick.cuh.
// The last x point of a full brick (x = 32 k) has no thread of its own: lanes 0..k of warp 0 process
// that pencil cooperatively (one z line and one y line each, exchanged through shared memory).
#pragma once

#include "brick.cuh"
#include "sumfac.cuh"

namespace mpdg
{
  template <int K>
  struct PencilShape
  {
    static constexpr int N = K + 1, M = N * N;
    static constexpr int BX = 32, BY = 2, BZ = 4;
    static constexpr int NT = K * BX;        // threads: x points 0 .. K*BX-1
    static constexpr int TP = K * BX + 1;    // x points of the transposition buffer (odd)
    static constexpr int MP = M | 1;         // face-buffer stride (odd)
  };

  template <int K, typename T>
  struct PencilLayout
  {
    using S                    = PencilShape<K>;
    static constexpr int TB    = S::M * S::TP;          // transposition buffer
    static constexpr int FB    = S::BX * S::MP;         // one face buffer
    static constexpr int ZC    = S::BY * K * S::NT;     // z carries
    static constexpr int XS    = S::M;                  // exchange of the cooperative pencil
    static constexpr size_t bytes = sizeof(T) * (size_t)(TB + 2 * FB + ZC + XS);
    using BR = Brick<K, S::BX, S::BY, S::BZ, S::NT>;
  };

  // Op supplies the per-cell diagonal: scale(kc, b, c) -> beta, and kcx; see heat.cu.
  template <int K, typename T, OutMode MODE, class Op>
  __device__ __forceinline__ void
  pencil_body(const GridDesc &g, const SyncDesc &s, const T *src, T *dst, const T *bvec, bool mask_src, const Op &op,
              T *smem, unsigned *s_ticket)
  {
    using LAY       = PencilLayout<K, T>;
    using SH        = typename LAY::S;
    using BR        = typename LAY::BR;
    constexpr int N = K + 1, M = SH::M, TP = SH::TP, MP = SH::MP, BX = SH::BX, NT = SH::NT;
    T *tb = smem, *e0 = smem + LAY::TB, *e4 = e0 + LAY::FB, *zc = e4 + LAY::FB, *xs = zc + LAY::ZC;
    const int p = threadIdx.x, lane = p & 31, warp = p >> 5;
    BR        br;
    if (!brick_begin<BR, T, MODE>(br, g, s, dst, bvec, s_ticket))
      return;
    if constexpr (MODE != OutMode::Add)
      if (br.has_lower_neighbour())
        brick_wait_lower(br, g, s);
    const T  *we = op.we(), *wo = op.wo();
    const int ncx = min(BX, g.m[0] - br.c0[0]), ncy = min(SH::BY, g.m[1] - br.c0[1]),
              ncz = min(SH::BZ, g.m[2] - br.c0[2]);
    const int  plast = K * ncx;               // brick's high x face (x point)
    const bool xin   = p <= plast;
    const bool extra = ncx == BX;             // x point K*BX exists and is done cooperatively
    const bool xface = p == 0 || p == plast;
    const bool xcon  = (br.con_lo[0] && p == 0) || (br.con_hi[0] && p == plast);
    const bool xcon_in = mask_src && xcon;
    const int  qx = p % K, cxp = p / K;       // x point = K cxp + qx
    const int  sy = br.sy, sz = br.sz;
    const int  xbase = br.g0[0] + p;
    const bool exl   = extra && warp == 0 && lane < N; // lanes of the cooperative pencil
    const int  xbE   = br.g0[0] + K * BX;
    const bool xconE = br.con_hi[0] && extra;

    T ycar[N];
#pragma unroll
    for (int l = 0; l < N; ++l)
      ycar[l] = T(0);

    for (int lz = 0; lz < ncz; ++lz)
      {
        const int  gz0 = br.g0[2] + K * lz;
        const bool llo = br.con_lo[2] && lz == 0, lhi = br.con_hi[2] && lz == ncz - 1;
        for (int r = 0; r < ncy; ++r)
          {
            const int  gy0 = br.g0[1] + K * r;
            const bool jlo = br.con_lo[1] && r == 0, jhi = br.con_hi[1] && r == ncy - 1;
            const int  base = gy0 * sy + gz0 * sz;
            // ---- 1. load and transform the pencil (z lines, then y lines)
            T u[M];
            {
              const bool ok = xin && !xcon_in;
              const T   *s0 = src + (xbase + base);
#pragma unroll
              for (int l = 0; l < N; ++l)
#pragma unroll
                for (int j = 0; j < N; ++j)
                  {
                    bool v = ok;
                    if (mask_src)
                      v = v && !((j == 0 && jlo) || (j == K && jhi) || (l == 0 && llo) || (l == K && lhi));
                    u[l * N + j] = v ? s0[j * sy + l * sz] : T(0);
                  }
            }
#pragma unroll
            for (int j = 0; j < N; ++j)
              fwd_line<T, N, N>(u, j, we, wo);
#pragma unroll
            for (int c = 0; c < N; ++c)
              fwd_line<T, N, 1>(u, c * N, we, wo);
#pragma unroll
            for (int m = 0; m < M; ++m)
              tb[m * TP + p] = u[m];
            if (exl)
              {
                // cooperative pencil at x point K*BX: lane j transforms the z line of y point j
                const int  j  = lane;
                const bool ok = !(mask_src && xconE) && !(mask_src && ((j == 0 && jlo) || (j == K && jhi)));
                T          v[N];
#pragma unroll
                for (int l = 0; l < N; ++l)
                  {
                    const bool okl = ok && !(mask_src && ((l == 0 && llo) || (l == K && lhi)));
                    v[l]           = okl ? src[xbE + base + j * sy + l * sz] : T(0);
                  }
                fwd_line<T, N, 1>(v, 0, we, wo);
#pragma unroll
                for (int c = 0; c < N; ++c)
                  xs[j * N + c] = v[c];
              }
            __syncwarp();
            if (exl)
              {
                const int c = lane; // lane c transforms the y line of z mode c
                T         v[N];
#pragma unroll
                for (int b = 0; b < N; ++b)
                  v[b] = xs[b * N + c];
                fwd_line<T, N, 1>(v, 0, we, wo);
#pragma unroll
                for (int b = 0; b < N; ++b)
                  tb[(c * N + b) * TP + K * BX] = v[b];
              }
            __syncthreads();
            // ---- 2. x lines: one (cell, mode) line per thread and round
            {
              const int cy = br.c0[1] + r, cz = br.c0[2] + lz;
              for (int L = p; L < ncx * M; L += NT)
                {
                  const int cx = L / M, m = L - cx * M, b = m % N, c = m / N;
                  T         x[N];
#pragma unroll
                  for (int i = 0; i < N; ++i)
                    x[i] = tb[m * TP + K * cx + i];
                  fwd_line<T, N, 1>(x, 0, we, wo);
                  op.scale_line(x, br.c0[0] + cx, cy, cz, b, c);
                  bwd_line<T, N, 1>(x, 0, we, wo);
#pragma unroll
                  for (int i = 1; i < K; ++i)
                    tb[m * TP + K * cx + i] = x[i];
                  e0[cx * MP + m] = x[0];
                  e4[cx * MP + m] = x[K];
                }
            }
            __syncthreads();
            // ---- 3. read back, backward y and z transforms
#pragma unroll
            for (int m = 0; m < M; ++m)
              {
                T v;
                if (qx != 0)
                  v = tb[m * TP + p];
                else
                  {
                    v = (cxp < ncx) ? e0[cxp * MP + m] : T(0);
                    if (cxp > 0)
                      v += e4[(cxp - 1) * MP + m];
                  }
                u[m] = v;
              }
#pragma unroll
            for (int c = 0; c < N; ++c)
              bwd_line<T, N, 1>(u, c * N, we, wo);
#pragma unroll
            for (int j = 0; j < N; ++j)
              bwd_line<T, N, N>(u, j, we, wo);
            if (exl)
              {
                const int c = lane;
                T         v[N];
#pragma unroll
                for (int b = 0; b < N; ++b)
                  v[b] = e4[(BX - 1) * MP + c * N + b];
                bwd_line<T, N, 1>(v, 0, we, wo);
#pragma unroll
                for (int j = 0; j < N; ++j)
                  xs[j * N + c] = v[j];
              }
            __syncwarp();
            if (exl)
              {
                const int j = lane;
                T         v[N];
#pragma unroll
                for (int c = 0; c < N; ++c)
                  v[c] = xs[j * N + c];
                bwd_line<T, N, 1>(v, 0, we, wo);
                const bool cj = (j == 0 && jlo) || (j == K && jhi);
#pragma unroll
                for (int l = 0; l < N; ++l)
                  {
                    const bool cn = xconE || cj || (l == 0 && llo) || (l == K && lhi);
                    if (!cn)
                      atomicAdd(dst + (xbE + base + j * sy + l * sz), v[l]);
                  }
              }
            // ---- 4. combine and write the pencil's points
            if (xin)
              {
                T *d0 = dst + (xbase + base);
                if (xface)
                  {
                    // brick x face: every point atomically
#pragma unroll
                    for (int l = 0; l < N; ++l)
#pragma unroll
                      for (int j = 0; j < N; ++j)
                        {
                          const bool cn = xcon || (j == 0 && jlo) || (j == K && jhi) || (l == 0 && llo) ||
                                          (l == K && lhi);
                          if (!cn)
                            atomicAdd(d0 + (j * sy + l * sz), u[l * N + j]);
                        }
                  }
                else
                  {
                    const bool ylast = r == ncy - 1, zlast = lz == ncz - 1;
                    T         *zcr   = zc + r * K * NT + p;
                    if (r > 0)
#pragma unroll
                      for (int l = 0; l < N; ++l)
                        u[l * N] += ycar[l];
                    if (lz > 0)
#pragma unroll
                      for (int j = 0; j < K; ++j)
                        u[j] += zcr[j * NT];
#pragma unroll
                    for (int l = 0; l < N; ++l)
                      ycar[l] = u[l * N + K];
                    if (!zlast)
#pragma unroll
                      for (int j = 0; j < K; ++j)
                        zcr[j * NT] = u[K * N + j];
                    // owned points j, l < K; brick faces (low y of row 0, low z of layer 0, high y of
                    // the last row, high z of the last layer) atomically
#pragma unroll
                    for (int l = 0; l < N; ++l)
#pragma unroll
                      for (int j = 0; j < N; ++j)
                        {
                          if (j == K && !ylast)
                            continue; // carried to the next row
                          if (l == K && !zlast && j < K)
                            continue; // carried to the next layer
                          const int  off  = j * sy + l * sz;
                          const T    v    = u[l * N + j];
                          const bool face = (j == 0 && r == 0) || (l == 0 && lz == 0) || j == K || l == K;
                          if (face)
                            {
                              const bool cn = (j == 0 && jlo) || (j == K && jhi) || (l == 0 && llo) || (l == K && lhi);
                              if (!cn)
                                atomicAdd(d0 + off, v);
                            }
                          else if constexpr (MODE == OutMode::Set)
                            d0[off] = v;
                          else if constexpr (MODE == OutMode::Add)
                            d0[off] += v;
                          else
                            d0[off] = bvec[xbase + base + off] + v;
                        }
                  }
              }
            __syncthreads();
          }
      }
    if constexpr (MODE != OutMode::Add)
      release_ticket(s);
  }
} // namespace mpdg
