// Brick machinery shared by the matrix-free kernels.
//
// One CTA processes one brick of BX x BY x BZ cells.
//
//  * Staging: the brick's (K BX+1)(K BY+1)(K BZ+1) lattice points of the input are copied into
//    shared memory with cp.async (all copies in flight at once, zero-fill for points outside the
//    domain).  Dirichlet-constrained points read as 0 when the operator reads "with constraints"
//    (deal.II read_dof_values); plain reads otherwise (read_dof_values_plain).
//  * In-brick reduction: cells add their local outputs into a shared-memory accumulator of the
//    brick's lattice points (shared-memory atomics; contention is rare because cells only share
//    the points of common faces).
//  * Brick faces: a lattice point on the low face of a brick (that has a lower neighbour brick)
//    belongs to that lower brick; a point on the high face belongs to this brick but also gets
//    contributions from the upper brick.  Those points are combined with global atomics; all
//    other points are written with plain, coalesced stores.
//  * Initialisation of atomically combined points without a separate pass: bricks are dealt out
//    through a ticket counter in lexicographic order, so a brick's lower neighbours always took
//    their tickets earlier.  Right after taking its ticket a brick initialises the high-face
//    points it owns and publishes a per-brick flag (= launch epoch); before adding into a lower
//    neighbour's points a brick waits for that neighbour's flag.  A lower neighbour is resident
//    and sets its flag before any wait of its own, so every wait ends; each spin is bounded
//    anyway and records an error word instead of hanging.
//  * Per-point bookkeeping uses per-brick precomputed geometry (clipped extents, which faces are
//    shared or constrained), so a lattice point costs a few integer operations.
#pragma once

#include <atomic>
#include <cstdint>

#include <cuda_runtime.h>

namespace mpdg
{
  enum class OutMode : int
  {
    Set   = 0, // dst = A src           (constrained rows 0)
    Add   = 1, // dst += A src          (constrained rows untouched)
    BPlus = 2, // dst = b + A src       (constrained rows b)
  };

  struct GridDesc
  {
    int            m[3];   // cells per direction
    int            nbr[3]; // bricks per direction
    int            n[3];   // lattice points per direction (K m + 1)
    unsigned       faces;  // Dirichlet faces: bit 2d low face of dim d, bit 2d+1 high face
    const uint8_t *cmask;  // optional per-DoF Dirichlet flags (device), may be null
    unsigned       acc_lo_z = 0; // the lattice is a z-slab of a larger one: its low z plane already
                                 // holds the previous slab's contributions and is only added into
  };

  constexpr unsigned SPIN_LIMIT    = 1u << 22; // x 32 ns sleeps: ~0.1-0.2 s
  constexpr int      ERR_FLAG_WAIT = 1;
  constexpr int      ERR_TICKET    = 2;

  struct SyncDesc
  {
    unsigned *ticket;                  // brick ticket counter (0 between launches)
    unsigned *done;                    // finished-CTA counter (0 between launches)
    unsigned *flags;                   // per-brick init flags (== epoch when initialised)
    unsigned  epoch;                   // launch epoch (never 0)
    int      *error;                   // set to a nonzero code when a bounded wait gives up
    unsigned  spin_limit = SPIN_LIMIT; // sleeps before a wait gives up
  };

  // Optional fused dot product of an apply dst = A src: the kernel sums src^T A src cell by cell and
  // the last CTA sets *alpha = *rho / (sum) -- the step length of a CG iteration whose search
  // direction is src.  Disabled when part == nullptr.
  struct DotSink
  {
    double       *part  = nullptr; // one partial per brick
    double       *alpha = nullptr;
    const double *rho   = nullptr;
  };

  // Dynamic shared memory above 48 KB is opted into once per kernel and device.
  template <class F>
  inline cudaError_t
  ensure_smem(F kern, size_t bytes, std::atomic<unsigned long long> &devices)
  {
    int         dev = 0;
    cudaError_t e   = cudaGetDevice(&dev);
    if (e != cudaSuccess)
      return e;
    const unsigned long long bit = 1ull << (dev & 63);
    if (devices.load() & bit)
      return cudaSuccess;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess)
      devices.fetch_or(bit);
    return e;
  }

  __device__ __forceinline__ long long
  lattice_index(const GridDesc &g, int I, int J, int L)
  {
    return (long long)I + (long long)g.n[0] * ((long long)J + (long long)g.n[1] * L);
  }

  __device__ __forceinline__ bool
  is_constrained(const GridDesc &g, int I, int J, int L, long long idx)
  {
    const unsigned f = g.faces;
    if (f)
      {
        if (((f & 1u) && I == 0) || ((f & 2u) && I == g.n[0] - 1) || ((f & 4u) && J == 0) ||
            ((f & 8u) && J == g.n[1] - 1) || ((f & 16u) && L == 0) || ((f & 32u) && L == g.n[2] - 1))
          return true;
      }
    return g.cmask != nullptr && g.cmask[idx] != 0;
  }

  // The cells that share lattice index P along one direction (1 or 2) and P's local index in each.
  template <int K>
  struct Neighbours1D
  {
    int  c[2], l[2];
    bool v[2];
    __device__ __forceinline__
    Neighbours1D(int P, int m)
    {
      const int q = P / K, r = P - q * K;
      if (r == 0)
        {
          c[0] = q - 1, l[0] = K, v[0] = q - 1 >= 0;
          c[1] = q, l[1] = 0, v[1] = q < m;
        }
      else
        {
          c[0] = q, l[0] = r, v[0] = true;
          c[1] = q, l[1] = r, v[1] = false;
        }
    }
  };

  __device__ __forceinline__ unsigned
  ld_acquire(const unsigned *p)
  {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
  }

  __device__ __forceinline__ void
  st_release(unsigned *p, unsigned v)
  {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
  }

  // Asynchronous global->shared copy of one element (cp.async); src_size 0 writes zeros without
  // reading global memory.
  template <typename T>
  __device__ __forceinline__ void
  cp_async_elem(T *smem, const T *gmem, bool valid)
  {
    const unsigned saddr  = (unsigned)__cvta_generic_to_shared(smem);
    const int      nbytes = valid ? (int)sizeof(T) : 0;
    if constexpr (sizeof(T) == 8)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(saddr), "l"(gmem), "r"(nbytes) : "memory");
    else
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(saddr), "l"(gmem), "r"(nbytes) : "memory");
  }

  __device__ __forceinline__ void
  cp_async_wait_all()
  {
    asm volatile("cp.async.wait_all;" ::: "memory");
  }

  template <int K_, int BX_, int BY_, int BZ_, int NT_>
  struct Brick
  {
    static constexpr int K = K_, BX = BX_, BY = BY_, BZ = BZ_;
    static constexpr int PX = K * BX + 1, PY = K * BY + 1, PZ = K * BZ + 1;
    static constexpr int NPTS = PX * PY * PZ;
    static constexpr int NC   = BX * BY * BZ; // cells per brick
    static constexpr int NT   = NT_;          // threads per CTA
    // row walk: a thread keeps the x-column px = tid % PX and visits rows tid / PX + k * RSTEP
    static constexpr int ROWS   = PY * PZ;
    static constexpr int RSTEP  = NT / PX;
    static constexpr int RITER  = RSTEP > 0 ? (ROWS + RSTEP - 1) / RSTEP : 0;
    int            c0[3];                // first cell of the brick
    int            g0[3];                // first lattice point (K c0)
    int            nv[3];                // lattice points of the brick inside the domain
    int            lo_sh[3], hi_sh[3];   // low / high face shared with a neighbour brick
    int            con_lo[3], con_hi[3]; // Dirichlet on the brick's low / high plane
    int            any_con;              // some constrained point may lie in the brick
    int            sy, sz;               // lattice strides (operators hold < 2^31 DoFs)
    const uint8_t *cmask;
    unsigned       id;

    __device__ __forceinline__ void
    set(const GridDesc &g, unsigned t)
    {
      id    = t;
      c0[0] = (int)(t % (unsigned)g.nbr[0]) * BX;
      c0[1] = (int)((t / (unsigned)g.nbr[0]) % (unsigned)g.nbr[1]) * BY;
      c0[2] = (int)(t / (unsigned)(g.nbr[0] * g.nbr[1])) * BZ;
      const int B[3] = {BX, BY, BZ}, P[3] = {PX, PY, PZ};
      any_con        = g.cmask != nullptr;
#pragma unroll
      for (int d = 0; d < 3; ++d)
        {
          g0[d]     = K * c0[d];
          nv[d]     = min(P[d], g.n[d] - g0[d]);
          lo_sh[d]  = c0[d] > 0;
          hi_sh[d]  = c0[d] + B[d] < g.m[d];
          con_lo[d] = ((g.faces >> (2 * d)) & 1u) && g0[d] == 0;
          con_hi[d] = ((g.faces >> (2 * d + 1)) & 1u) && g0[d] + nv[d] == g.n[d];
          any_con |= con_lo[d] | con_hi[d];
        }
      sy    = g.n[0];
      sz    = g.n[0] * g.n[1];
      cmask = g.cmask;
    }
    __device__ __forceinline__ bool
    inside(int px, int py, int pz) const
    {
      return px < nv[0] && py < nv[1] && pz < nv[2];
    }
    __device__ __forceinline__ int
    index(int px, int py, int pz) const
    {
      return (g0[0] + px) + sy * (g0[1] + py) + sz * (g0[2] + pz);
    }
    __device__ __forceinline__ bool
    constrained(int px, int py, int pz, int idx) const
    {
      if (!any_con)
        return false;
      const bool f = (con_lo[0] && px == 0) || (con_hi[0] && px == nv[0] - 1) || (con_lo[1] && py == 0) ||
                     (con_hi[1] && py == nv[1] - 1) || (con_lo[2] && pz == 0) || (con_hi[2] && pz == nv[2] - 1);
      return f || (cmask != nullptr && cmask[idx] != 0);
    }
    __device__ __forceinline__ bool
    low_shared(int px, int py, int pz) const
    {
      return (px == 0 && lo_sh[0]) || (py == 0 && lo_sh[1]) || (pz == 0 && lo_sh[2]);
    }
    __device__ __forceinline__ bool
    high_shared(int px, int py, int pz) const
    {
      return (px == PX - 1 && hi_sh[0]) || (py == PY - 1 && hi_sh[1]) || (pz == PZ - 1 && hi_sh[2]);
    }
    __device__ __forceinline__ bool
    has_lower_neighbour() const
    {
      return lo_sh[0] || lo_sh[1] || lo_sh[2];
    }
  };

  // Take a ticket from the counter (bricks are dealt out in lexicographic order).
  __device__ __forceinline__ unsigned
  take_ticket(const SyncDesc &s, unsigned *s_ticket)
  {
    if (threadIdx.x == 0)
      *s_ticket = atomicAdd(s.ticket, 1u);
    __syncthreads();
    return *s_ticket;
  }

  // Last CTA resets the counters for the next launch on the stream.
  __device__ __forceinline__ void
  release_ticket(const SyncDesc &s)
  {
    if (threadIdx.x == 0)
      {
        __threadfence();
        if (atomicAdd(s.done, 1u) == gridDim.x - 1)
          {
            *s.ticket = 0u;
            *s.done   = 0u;
            __threadfence();
          }
      }
  }

  // Sum of one double per thread over the CTA in a fixed order (valid in thread 0); scratch holds
  // NT / 32 doubles and is reusable on return.
  template <int NT>
  __device__ __forceinline__ double
  cta_sum(double v, double *scratch)
  {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
      v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0)
      scratch[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
#pragma unroll
      for (int w = 0; w < NT / 32; ++w)
        t += scratch[w];
    __syncthreads();
    return t;
  }

  // release_ticket with the fused dot: every CTA stores the sum of its bricks' cell forms, the last
  // CTA to finish adds the partials in brick order (deterministic) and sets the step length.
  template <int NT>
  __device__ __forceinline__ void
  release_ticket_dot(const SyncDesc &s, const DotSink &d, unsigned id, double local, double *scratch,
                     unsigned *s_flag)
  {
    const double t = cta_sum<NT>(local, scratch);
    if (threadIdx.x == 0)
      {
        d.part[id] = t;
        __threadfence();
        *s_flag = atomicAdd(s.done, 1u) == gridDim.x - 1 ? 1u : 0u;
      }
    __syncthreads();
    if (*s_flag)
      {
        __threadfence();
        double acc = 0.0;
        for (unsigned i = threadIdx.x; i < gridDim.x; i += NT)
          acc += __ldcg(d.part + i);
        const double tot = cta_sum<NT>(acc, scratch);
        if (threadIdx.x == 0)
          {
            *d.alpha  = *d.rho / tot;
            *s.ticket = 0u;
            *s.done   = 0u;
            __threadfence();
          }
      }
  }

  // Initialise the face points the brick owns (Set: 0, BPlus: b) and publish the flag.  A brick owns
  // its high faces (also where they are the domain boundary) and, at the domain's low boundary, its
  // low faces; low faces shared with a lower brick belong to that brick.  Edge points are visited
  // up to three times with the same value.
  template <class BR, typename T, OutMode MODE>
  __device__ __forceinline__ void
  brick_init_publish(const BR &br, const SyncDesc &s, T *dst, const T *bvec, unsigned acc_lo_z = 0)
  {
    static_assert(MODE != OutMode::Add, "Add mode needs no initialisation");
    auto put = [&](int px, int py, int pz) {
      if (br.low_shared(px, py, pz))
        return;
      if (acc_lo_z && pz == 0 && br.g0[2] == 0)
        return; // accumulated onto the previous slab's values, never reset
      const int idx = br.index(px, py, pz);
      dst[idx]      = (MODE == OutMode::BPlus) ? bvec[idx] : T(0);
    };
    // face by face (side 0: low face, only at the domain boundary; side 1: high face), the faces
    // normal to y and z in rows along x so that consecutive threads store consecutive points
#pragma unroll
    for (int side = 0; side < 2; ++side)
      {
        if (side == 0 && br.lo_sh[0])
          continue;
        const int px = side ? br.nv[0] - 1 : 0;
        for (int e = threadIdx.x; e < BR::PY * BR::PZ; e += BR::NT)
          {
            const int py = e % BR::PY, pz = e / BR::PY;
            if (py < br.nv[1] && pz < br.nv[2])
              put(px, py, pz);
          }
      }
#pragma unroll
    for (int side = 0; side < 2; ++side)
      {
        if (side == 0 && br.lo_sh[1])
          continue;
        const int py = side ? br.nv[1] - 1 : 0;
        for (int e = threadIdx.x; e < BR::PX * BR::PZ; e += BR::NT)
          {
            const int px = e % BR::PX, pz = e / BR::PX;
            if (px < br.nv[0] && pz < br.nv[2])
              put(px, py, pz);
          }
      }
#pragma unroll
    for (int side = 0; side < 2; ++side)
      {
        if (side == 0 && br.lo_sh[2])
          continue;
        const int pz = side ? br.nv[2] - 1 : 0;
        for (int e = threadIdx.x; e < BR::PX * BR::PY; e += BR::NT)
          {
            const int px = e % BR::PX, py = e / BR::PX;
            if (px < br.nv[0] && py < br.nv[1])
              put(px, py, pz);
          }
      }
    __syncthreads();
    if (threadIdx.x == 0)
      {
        __threadfence();
        st_release(s.flags + br.id, s.epoch);
      }
  }

  // Stage the brick's lattice points of src into shared memory (row walk, cp.async).  WAIT = false
  // only issues the copies (a later staging call with WAIT waits for all of the thread's copies).
  template <class BR, typename T, bool WAIT = true>
  __device__ __forceinline__ void
  brick_stage(const BR &br, const T *src, bool mask_src, T *s_src)
  {
    static_assert(BR::RSTEP >= 1, "brick rows wider than the CTA");
    const int  px  = threadIdx.x % BR::PX;
    const int  r0  = threadIdx.x / BR::PX;
    const bool act = r0 < BR::RSTEP;
    const bool xin = px < br.nv[0];
    const bool chk = mask_src && br.any_con;
#pragma unroll 4
    for (int k = 0; k < BR::RITER; ++k)
      {
        const int row = r0 + k * BR::RSTEP;
        if (!act || row >= BR::ROWS)
          break;
        const int py = row % BR::PY, pz = row / BR::PY;
        bool      valid = xin && py < br.nv[1] && pz < br.nv[2];
        const int idx   = valid ? br.index(px, py, pz) : 0;
        if (chk && valid && br.constrained(px, py, pz, idx))
          valid = false;
        cp_async_elem(s_src + row * BR::PX + px, src + idx, valid);
      }
    if constexpr (WAIT)
      {
        cp_async_wait_all();
        __syncthreads();
      }
  }

  // Write the brick's accumulated values: plain stores for brick-interior points, atomics on points
  // shared with neighbour bricks, constrained rows per mode.  Row walk as in brick_stage; U rows per
  // round so that the loads of b / dst (BPlus / Add) are in flight together.
  template <class BR, typename T, OutMode MODE>
  __device__ __forceinline__ void
  brick_output(const BR &br, const T *s_dst, T *dst, const T *bvec)
  {
    static_assert(BR::RSTEP >= 1, "brick rows wider than the CTA");
    constexpr int U   = 4;
    const int     px  = threadIdx.x % BR::PX;
    const int     r0  = threadIdx.x / BR::PX;
    if (r0 >= BR::RSTEP || px >= br.nv[0])
      return;
    const bool xsh = (px == 0 && br.lo_sh[0]) || (px == BR::PX - 1 && br.hi_sh[0]);
    for (int k0 = 0; k0 < BR::RITER; k0 += U)
      {
        int  idx[U];
        int  kind[U]; // 0 skip, 1 atomic, 2 plain, 3 constrained plain
        T    bv[U];
#pragma unroll
        for (int u = 0; u < U; ++u)
          {
            const int row = r0 + (k0 + u) * BR::RSTEP;
            kind[u]       = 0;
            idx[u]        = 0;
            bv[u]         = T(0);
            if (row < BR::ROWS)
              {
                const int py = row % BR::PY, pz = row / BR::PY;
                if (py < br.nv[1] && pz < br.nv[2])
                  {
                    idx[u]            = br.index(px, py, pz);
                    const bool shared = xsh || (py == 0 && br.lo_sh[1]) || (pz == 0 && br.lo_sh[2]) ||
                                        (py == BR::PY - 1 && br.hi_sh[1]) || (pz == BR::PZ - 1 && br.hi_sh[2]);
                    const bool con    = br.constrained(px, py, pz, idx[u]);
                    kind[u]           = shared ? (con ? 0 : 1) : (con ? 3 : 2);
                    if constexpr (MODE == OutMode::BPlus)
                      {
                        if (kind[u] >= 2)
                          bv[u] = bvec[idx[u]];
                      }
                    else if constexpr (MODE == OutMode::Add)
                      {
                        if (kind[u] == 2)
                          bv[u] = dst[idx[u]];
                      }
                  }
              }
          }
#pragma unroll
        for (int u = 0; u < U; ++u)
          {
            const int row = r0 + (k0 + u) * BR::RSTEP;
            if (kind[u] == 0)
              continue;
            const T v = s_dst[row * BR::PX + px];
            if (kind[u] == 1)
              atomicAdd(dst + idx[u], v);
            else if (kind[u] == 2)
              dst[idx[u]] = (MODE == OutMode::Set) ? v : bv[u] + v;
            else
              {
                if constexpr (MODE == OutMode::Set)
                  dst[idx[u]] = T(0);
                else if constexpr (MODE == OutMode::BPlus)
                  dst[idx[u]] = bv[u];
              }
          }
      }
  }

  // Wait (bounded) until the lower neighbour bricks have initialised their high-face points.
  template <class BR>
  __device__ __forceinline__ void
  brick_wait_lower(const BR &br, const GridDesc &g, const SyncDesc &s)
  {
    if (threadIdx.x < 7)
      {
        const unsigned t  = threadIdx.x + 1; // offsets (ox,oy,oz) in {0,1}^3 minus (0,0,0)
        const int      ox = (t & 1u) ? 1 : 0, oy = (t & 2u) ? 1 : 0, oz = (t & 4u) ? 1 : 0;
        const int bx = br.c0[0] / BR::BX - ox, by = br.c0[1] / BR::BY - oy, bz = br.c0[2] / BR::BZ - oz;
        if (bx >= 0 && by >= 0 && bz >= 0)
          {
            const unsigned nb = (unsigned)bx + (unsigned)g.nbr[0] * ((unsigned)by + (unsigned)g.nbr[1] * (unsigned)bz);
            unsigned       it = 0;
            while (ld_acquire(s.flags + nb) != s.epoch)
              {
                if (++it > s.spin_limit)
                  {
                    atomicExch(s.error, ERR_FLAG_WAIT);
                    break;
                  }
                __nanosleep(32);
              }
          }
      }
    __syncthreads();
  }

  // Ticket / flag prologue shared by the apply kernels; returns false when the CTA has to quit.
  template <class BR, typename T, OutMode MODE>
  __device__ __forceinline__ bool
  brick_begin(BR &br, const GridDesc &g, const SyncDesc &s, T *dst, const T *bvec, unsigned *s_ticket)
  {
    if constexpr (MODE != OutMode::Add)
      {
        const unsigned t = take_ticket(s, s_ticket);
        if (t >= (unsigned)(g.nbr[0] * g.nbr[1] * g.nbr[2]))
          {
            // stale counter: never index past the flag array; report and keep the count
            if (threadIdx.x == 0)
              atomicExch(s.error, ERR_TICKET);
            release_ticket(s);
            return false;
          }
        br.set(g, t);
        brick_init_publish<BR, T, MODE>(br, s, dst, bvec, g.acc_lo_z);
      }
    else
      br.set(g, blockIdx.x);
    return true;
  }

  template <class BR, typename T, OutMode MODE>
  __device__ __forceinline__ void
  brick_end(const BR &br, const GridDesc &g, const SyncDesc &s, const T *s_dst, T *dst, const T *bvec)
  {
    if constexpr (MODE != OutMode::Add)
      if (br.has_lower_neighbour())
        brick_wait_lower(br, g, s);
    brick_output<BR, T, MODE>(br, s_dst, dst, bvec);
    if constexpr (MODE != OutMode::Add)
      release_ticket(s);
  }
} // namespace mpdg
