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
//      transforms and holds the (k+1)^2 output values of its pencil; with MPDG_PENCIL_PREFETCH the
//      thread then starts the asynchronous copy (cp.async) of its pencil of the next row step into
//      its (now free) transposition-buffer column, with the next row's conductivities, so that the
//      loads of step 1 are in flight during this step's backward transforms and stores (on for
//      k = 3 and for FP32; at k = 4 in FP64 the plain loads measured faster);
//   4. y faces between the rows of the brick are carried in registers to the next row step, z faces
//      between layers in shared memory to the next layer (per thread, no synchronisation); points
//      owned by the pencil are written with coalesced plain stores; points on the brick's faces
//      are combined with global atomics, initialised by their owner through the ticket / flag
//      handshake of brick.cuh.
// The last x point of a full brick (x = 32 k) has no thread of its own: lanes 0..k of warp 1 process
// that pencil cooperatively (one z line and one y line each, exchanged through shared memory).
#pragma once

#include "brick.cuh"
#include "sumfac.cuh"

#ifndef MPDG_PENCIL_BY
#define MPDG_PENCIL_BY 2
#endif
#ifndef MPDG_PENCIL_BZ
#define MPDG_PENCIL_BZ 4
#endif
#ifndef MPDG_PENCIL_MINB3
#define MPDG_PENCIL_MINB3 5
#endif

#ifndef MPDG_PENCIL_MINB4
#define MPDG_PENCIL_MINB4 4
#endif
#ifndef MPDG_PENCIL_XPAIR
#define MPDG_PENCIL_XPAIR 0
#endif
#ifndef MPDG_PENCIL_PREFETCH
#define MPDG_PENCIL_PREFETCH -1 // -1: by degree and precision (measured); 0 off; 1 on
#endif

namespace mpdg
{
  template <int K>
  struct PencilShape
  {
    static constexpr int N = K + 1, M = N * N;
    static constexpr int BX = 32, BY = MPDG_PENCIL_BY, BZ = MPDG_PENCIL_BZ;
    // CTAs per SM the register allocation is held to (K = 4: 4 x 128 threads at <= 128 registers)
    static constexpr int MINB = K == 3 ? MPDG_PENCIL_MINB3 : MPDG_PENCIL_MINB4;
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
    static constexpr int KC    = S::BX;                 // conductivity of the row's cells
    static constexpr int MU    = S::M;                  // cy lam_b + cz lam_c per (y, z) mode
    static constexpr size_t bytes = sizeof(T) * (size_t)(TB + 2 * FB + ZC + XS + KC + MU);
    using BR = Brick<K, S::BX, S::BY, S::BZ, S::NT>;
  };

  // Op supplies the fast-diagonalisation tables and the per-cell scaling:
  //   we(), wo(), lam()  1-D tables;  alpha(), cxg(), cyg(), czg()  geometry;  kcell(cell)  k_c.
  // With DOT the x lines also add d_mode * (modal value)^2, i.e. the cells' forms src_c^T A_c src_c,
  // to the fused dot product (release_ticket_dot).
  template <int K, typename T, OutMode MODE, class Op, bool DOT = false>
  __device__ __forceinline__ void
  pencil_body(const GridDesc &g, const SyncDesc &s, const T *src, T *dst, const T *bvec, bool mask_src, const Op &op,
              T *smem, unsigned *s_ticket, const DotSink &dot = DotSink{}, double *s_red = nullptr)
  {
    double dsum = 0.0;
    using LAY       = PencilLayout<K, T>;
    using SH        = typename LAY::S;
    using BR        = typename LAY::BR;
    constexpr int N = K + 1, M = SH::M, TP = SH::TP, MP = SH::MP, BX = SH::BX, NT = SH::NT;
    T *tb = smem, *e0 = smem + LAY::TB, *e4 = e0 + LAY::FB, *zc = e4 + LAY::FB, *xs = zc + LAY::ZC;
    T *kcs = xs + LAY::XS, *mus = kcs + LAY::KC;
    const int p = threadIdx.x, lane = p & 31, warp = p >> 5;
    BR        br;
    constexpr bool PF = MPDG_PENCIL_PREFETCH < 0 ? (K == 3 || sizeof(T) == 4) : MPDG_PENCIL_PREFETCH != 0;
    if (!brick_begin<BR, T, MODE>(br, g, s, dst, bvec, s_ticket))
      return;
    const int ncx = min(BX, g.m[0] - br.c0[0]), ncy = min(SH::BY, g.m[1] - br.c0[1]),
              ncz = min(SH::BZ, g.m[2] - br.c0[2]);
    const int  plast = K * ncx;               // brick's high x face (x point)
    const bool xin   = p <= plast;
    const int  sy = br.sy, sz = br.sz;
    const int  xbase = br.g0[0] + (xin ? p : plast); // clamped: every load stays inside the lattice
    // asynchronous copy of row step (rr, ll): the thread's pencil into its own column of tb, the
    // row's (unscaled) conductivities into kcs
    auto prefetch = [&](int rr, int ll) {
      const T *s0 = src + (xbase + (br.g0[1] + K * rr) * sy + (br.g0[2] + K * ll) * sz);
#pragma unroll
      for (int l = 0; l < N; ++l)
#pragma unroll
        for (int j = 0; j < N; ++j)
          cp_async_elem(tb + (l * N + j) * TP + p, s0 + (j * sy + l * sz), true);
      if (p < ncx)
        {
          const T *kp = op.kcell_ptr(br.c0[0] + p, br.c0[1] + rr, br.c0[2] + ll);
          if (kp != nullptr)
            cp_async_elem(kcs + p, kp, true);
          else
            kcs[p] = op.kconst();
        }
    };
    if constexpr (PF)
      prefetch(0, 0);
    if constexpr (MODE != OutMode::Add)
      if (br.has_lower_neighbour())
        brick_wait_lower(br, g, s);
    const T *we = op.we(), *wo = op.wo(), *lam = op.lam();
    // with the prefetch kcs holds unscaled conductivities: the scale goes into the geometry factors
    const T kmul = PF ? op.kscale() : T(1);
    if (p < M)
      mus[p] = kmul * (op.cyg() * lam[p % N] + op.czg() * lam[p / N]);
    const T   alpha = op.alpha(), cxg = kmul * op.cxg();
    const bool extra = ncx == BX;             // x point K*BX exists and is done cooperatively
    const bool xface = p == 0 || p == plast;
    const bool xcon  = (br.con_lo[0] && p == 0) || (br.con_hi[0] && p == plast);
    const bool zero_pencil = !xin || (mask_src && xcon);
    const int  qx = p % K, cxp = p / K;       // x point = K cxp + qx
    // the cooperative pencil runs on warp 1, the extra round of x lines on the last warp and the x = 0
    // face atomics on warp 0, so that no warp carries two of these
    const bool exl   = extra && warp == 1 && lane < N; // lanes of the cooperative pencil
    const int  xbE   = br.g0[0] + K * BX;
    const bool xconE = br.con_hi[0] && extra;
    // first x line of this thread and the increments of (cell, mode) per round of NT lines
    constexpr int DCX = NT / M, DM = NT % M;
    const int     q_line   = (p + 32) % NT;   // the last warp starts at line 0
    const int     cx_first = q_line / M, m_first = q_line % M;

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
            const int  cy = br.c0[1] + r, cz = br.c0[2] + lz;
            // ---- 1. load and transform the pencil (z lines, then y lines)
            T u[M];
            if constexpr (PF)
              {
                cp_async_wait_all(); // this thread's copies; the barrier below publishes kcs
#pragma unroll
                for (int m = 0; m < M; ++m)
                  u[m] = tb[m * TP + p];
              }
            else
              {
                const T *s0 = src + (xbase + base);
#pragma unroll
                for (int l = 0; l < N; ++l)
#pragma unroll
                  for (int j = 0; j < N; ++j)
                    u[l * N + j] = s0[j * sy + l * sz];
                if (p < ncx)
                  kcs[p] = op.kcell(br.c0[0] + p, cy, cz);
              }
            if (zero_pencil)
#pragma unroll
              for (int q = 0; q < M; ++q)
                u[q] = T(0);
            if (mask_src)
              {
                if (jlo)
#pragma unroll
                  for (int l = 0; l < N; ++l)
                    u[l * N] = T(0);
                if (jhi)
#pragma unroll
                  for (int l = 0; l < N; ++l)
                    u[l * N + K] = T(0);
                if (llo)
#pragma unroll
                  for (int j = 0; j < N; ++j)
                    u[j] = T(0);
                if (lhi)
#pragma unroll
                  for (int j = 0; j < N; ++j)
                    u[K * N + j] = T(0);
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
                const bool ok = !(mask_src && (xconE || (j == 0 && jlo) || (j == K && jhi)));
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
            // ---- 2. x lines: (cell, mode) lines per thread and round
#if MPDG_PENCIL_XPAIR == 2
            // K consecutive threads share a cell and take its modes g, g + K, ... (g = thread % K),
            // two lines per round: the cell's conductivity is read once, the line offsets advance by
            // a constant, and a warp's 8 cells x K mode groups hit distinct banks
            {
              constexpr int G = NT / BX; // threads per cell (= K)
              const int     cxg_ = p / G, g = p % G;
              if (cxg_ < ncx)
                {
                  const T kc  = kcs[cxg_];
                  const T kcx = kc * cxg;
                  T      *tl  = tb + K * cxg_;
                  for (int m = g; m < M; m += 2 * G)
                    {
                      const int  mb = m + G;
                      const bool hb = mb < M;
                      const int  m2 = hb ? mb : m;
                      T          x[N], y[N];
#pragma unroll
                      for (int i = 0; i < N; ++i)
                        {
                          x[i] = tl[m * TP + i];
                          y[i] = tl[m2 * TP + i];
                        }
                      fwd_line<T, N, 1>(x, 0, we, wo);
                      fwd_line<T, N, 1>(y, 0, we, wo);
                      const T ba = fma(kc, mus[m], alpha), bb = fma(kc, mus[m2], alpha);
                      T       fa = T(0), fb = T(0);
#pragma unroll
                      for (int i = 0; i < N; ++i)
                        {
                          const T da = fma(kcx, lam[i], ba), db = fma(kcx, lam[i], bb);
                          if constexpr (DOT)
                            {
                              fa = fma(da * x[i], x[i], fa);
                              fb = fma(db * y[i], y[i], fb);
                            }
                          x[i] *= da;
                          y[i] *= db;
                        }
                      if constexpr (DOT)
                        dsum += hb ? (double)fa + (double)fb : (double)fa;
                      bwd_line<T, N, 1>(x, 0, we, wo);
                      bwd_line<T, N, 1>(y, 0, we, wo);
#pragma unroll
                      for (int i = 1; i < K; ++i)
                        tl[m * TP + i] = x[i];
                      e0[cxg_ * MP + m] = x[0];
                      e4[cxg_ * MP + m] = x[K];
                      if (hb)
                        {
#pragma unroll
                          for (int i = 1; i < K; ++i)
                            tl[mb * TP + i] = y[i];
                          e0[cxg_ * MP + mb] = y[0];
                          e4[cxg_ * MP + mb] = y[K];
                        }
                    }
                }
            }
#elif MPDG_PENCIL_XPAIR
            // two lines per round, interleaved: twice the independent work per round
            {
              auto next = [&](int &c, int &mm) {
                c += DCX;
                mm += DM;
                if (mm >= M)
                  {
                    mm -= M;
                    ++c;
                  }
              };
              int cx = cx_first, m = m_first;
              while (cx < ncx)
                {
                  int cb = cx, mb = m;
                  next(cb, mb);
                  const bool hb  = cb < ncx;
                  const int  cy2 = hb ? cb : cx, my2 = hb ? mb : m; // the second line, or the first again
                  T          x[N], y[N];
#pragma unroll
                  for (int i = 0; i < N; ++i)
                    {
                      x[i] = tb[m * TP + K * cx + i];
                      y[i] = tb[my2 * TP + K * cy2 + i];
                    }
                  fwd_line<T, N, 1>(x, 0, we, wo);
                  fwd_line<T, N, 1>(y, 0, we, wo);
                  const T kca = kcs[cx], kcb = kcs[cy2];
                  const T ba = fma(kca, mus[m], alpha), bb = fma(kcb, mus[my2], alpha);
                  const T kxa = kca * cxg, kxb = kcb * cxg;
                  T       fa = T(0), fb = T(0);
#pragma unroll
                  for (int i = 0; i < N; ++i)
                    {
                      const T da = fma(kxa, lam[i], ba), db = fma(kxb, lam[i], bb);
                      if constexpr (DOT)
                        {
                          fa = fma(da * x[i], x[i], fa);
                          fb = fma(db * y[i], y[i], fb);
                        }
                      x[i] *= da;
                      y[i] *= db;
                    }
                  if constexpr (DOT)
                    dsum += hb ? (double)fa + (double)fb : (double)fa;
                  bwd_line<T, N, 1>(x, 0, we, wo);
                  bwd_line<T, N, 1>(y, 0, we, wo);
#pragma unroll
                  for (int i = 1; i < K; ++i)
                    tb[m * TP + K * cx + i] = x[i];
                  e0[cx * MP + m] = x[0];
                  e4[cx * MP + m] = x[K];
                  if (hb)
                    {
#pragma unroll
                      for (int i = 1; i < K; ++i)
                        tb[mb * TP + K * cb + i] = y[i];
                      e0[cb * MP + mb] = y[0];
                      e4[cb * MP + mb] = y[K];
                    }
                  cx = cb;
                  m  = mb;
                  next(cx, m);
                }
            }
#else
            {
              int cx = cx_first, m = m_first;
              while (cx < ncx)
                {
                  T x[N];
#pragma unroll
                  for (int i = 0; i < N; ++i)
                    x[i] = tb[m * TP + K * cx + i];
                  fwd_line<T, N, 1>(x, 0, we, wo);
                  const T kc   = kcs[cx];
                  const T beta = fma(kc, mus[m], alpha);
                  const T kcx  = kc * cxg;
                  T form = T(0);
#pragma unroll
                  for (int i = 0; i < N; ++i)
                    {
                      const T d = fma(kcx, lam[i], beta);
                      if constexpr (DOT)
                        form = fma(d * x[i], x[i], form);
                      x[i] *= d;
                    }
                  if constexpr (DOT)
                    dsum += (double)form;
                  bwd_line<T, N, 1>(x, 0, we, wo);
#pragma unroll
                  for (int i = 1; i < K; ++i)
                    tb[m * TP + K * cx + i] = x[i];
                  e0[cx * MP + m] = x[0];
                  e4[cx * MP + m] = x[K];
                  cx += DCX;
                  m += DM;
                  if (m >= M)
                    {
                      m -= M;
                      ++cx;
                    }
                }
            }
#endif
            __syncthreads();
            // ---- 3. read back (face points: both adjacent cells), backward y and z transforms
#pragma unroll
            for (int m = 0; m < M; ++m)
              u[m] = tb[m * TP + p];
            if (qx == 0)
              {
                const T *f0 = e0 + cxp * MP, *f4 = e4 + (cxp - 1) * MP;
                const bool h0 = cxp < ncx, h4 = cxp > 0;
#pragma unroll
                for (int m = 0; m < M; ++m)
                  u[m] = (h0 ? f0[m] : T(0)) + (h4 ? f4[m] : T(0));
              }
            if constexpr (PF)
              {
                // the next row step's loads, in flight during the rest of this one
                const bool nl = r + 1 == ncy;
                if (!nl || lz + 1 < ncz)
                  prefetch(nl ? 0 : r + 1, nl ? lz + 1 : lz);
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
            T *d0 = dst + (xbase + base);
            if (xin && xface)
              {
                // brick x face: every point atomically
#pragma unroll
                for (int l = 0; l < N; ++l)
#pragma unroll
                  for (int j = 0; j < N; ++j)
                    {
                      const bool cn =
                        xcon || (j == 0 && jlo) || (j == K && jhi) || (l == 0 && llo) || (l == K && lhi);
                      if (!cn)
                        atomicAdd(d0 + (j * sy + l * sz), u[l * N + j]);
                    }
              }
            else if (xin)
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
                auto put = [&](int j, int l) {
                  const int off = j * sy + l * sz;
                  const T   v   = u[l * N + j];
                  if constexpr (MODE == OutMode::Set)
                    d0[off] = v;
                  else if constexpr (MODE == OutMode::Add)
                    d0[off] += v;
                  else
                    d0[off] = bvec[xbase + base + off] + v;
                };
                auto add = [&](int j, int l) { atomicAdd(d0 + (j * sy + l * sz), u[l * N + j]); };
                // interior of the pencil's owned block: plain stores
#pragma unroll
                for (int l = 1; l < K; ++l)
#pragma unroll
                  for (int j = 1; j < K; ++j)
                    put(j, l);
                // y = 0 row (l = 1..K-1): low y face of the brick in row 0
                if (r == 0)
                  {
                    if (!jlo)
#pragma unroll
                      for (int l = 1; l < K; ++l)
                        add(0, l);
                  }
                else
#pragma unroll
                  for (int l = 1; l < K; ++l)
                    put(0, l);
                // z = 0 plane (j = 1..K-1): low z face of the brick in layer 0
                if (lz == 0)
                  {
                    if (!llo)
#pragma unroll
                      for (int j = 1; j < K; ++j)
                        add(j, 0);
                  }
                else
#pragma unroll
                  for (int j = 1; j < K; ++j)
                    put(j, 0);
                // corner line (0, 0)
                if (r == 0 || lz == 0)
                  {
                    if (!jlo && !llo)
                      add(0, 0);
                  }
                else
                  put(0, 0);
                // y = K row of the last row: high y face (all l); otherwise carried
                if (ylast && !jhi)
                  {
#pragma unroll
                    for (int l = 1; l < K; ++l)
                      add(K, l);
                    if (!llo)
                      add(K, 0);
                    if (!lhi)
                      add(K, K);
                  }
                // z = K plane (j < K) of the last layer: high z face; otherwise carried
                if (zlast && !lhi)
                  {
#pragma unroll
                    for (int j = 1; j < K; ++j)
                      add(j, K);
                    if (!jlo)
                      add(0, K);
                  }
              }
            // no barrier here: the next row's first barrier (after its pencil transforms) already
            // orders every shared buffer it reuses -- tb columns are rewritten only by their own
            // thread before it, the face buffers only after it, and kcs (nobody reads it between the
            // x-line barrier of this row and the first barrier of the next) by its prefetch
          }
      }
    if constexpr (DOT)
      release_ticket_dot<NT>(s, dot, br.id, dsum, s_red, s_ticket);
    else if constexpr (MODE != OutMode::Add)
      release_ticket(s);
  }
} // namespace mpdg
