// Host interface of the one-launch-per-iteration Jacobi-PCG of the FE_Q(2) heat operator
// (cgfused.cu).  Internal to the library, not part of the C ABI.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "kernels.h"

namespace mpdg
{
#ifndef MPDG_FUSED_TY_F64
#define MPDG_FUSED_TY_F64 8
#endif
#ifndef MPDG_FUSED_C_F32
#define MPDG_FUSED_C_F32 1
#endif
#ifndef MPDG_FUSED_TY_F32
#define MPDG_FUSED_TY_F32 (MPDG_FUSED_C_F32 == 2 ? 8 : 16)
#endif
  constexpr int FUSED_TY_F64 = MPDG_FUSED_TY_F64; // owned cell rows per tile (FP64)
  // owned cell rows per tile (FP32): 16 rows take one SM each (200 KB of shared memory, 18 warps) and
  // halve the share of halo rows against two CTAs of 8 rows per SM (215 against 246 us per iteration
  // on 128^3)
  constexpr int FUSED_TY_F32 = MPDG_FUSED_TY_F32;
  // cells per lane in x (FP32): 2 computes two adjacent cells per thread as packed FP32 pairs
  // (tiles of 64 x 8 cells, one CTA per SM, 10 warps); it measured slower than one cell per lane
  // with 16-row tiles (215 against 206 us per iteration on 128^3: half the resident warps, and the
  // register cap of a 320-thread CTA spills), so 1 is the default and 2 stays selectable
  // (-DMPDG_FUSED_C_F32=2)
  constexpr int FUSED_C_F32 = MPDG_FUSED_C_F32;
  static_assert(FUSED_C_F32 == 1 || FUSED_C_F32 == 2, "one or two cells per lane");

  // Problem description and tiling of the fused sweep; vectors in the padded layout (x rows of P0
  // entries, P0 = n0 rounded up to a multiple of 8 and > n0).
  template <typename T>
  struct FusedCG
  {
    int      m[3]{}, n[3]{};
    int      P0 = 0;
    unsigned faces = 0;
    double   mass_coef = 0.0, geo[3]{}, kconst = 1.0;
    const T *kcell = nullptr;
    int       tiles_x = 0, tiles_y = 0, ntiles = 0; // ntiles: CTAs of the sweep (one partial sum each)
    long long layers  = 0;                          // columns x cell layers
    int       slab    = 1;                          // cell layers per slab of the CTA sequence
    std::vector<long long> range;                   // CTA b: sequence positions [range[b], range[b+1])
    const long long       *d_range = nullptr;       // the same on the device (uploaded by the caller)

    static int padded_pitch(int n0) { return (n0 + 8) / 8 * 8; }
    long long  padded_len() const { return (long long)P0 * n[1] * n[2]; }
    void       plan(int sm_count);
    int        make_map(CUtensorMap *map, const T *base) const;
    static size_t smem_bytes();
    static int    threads();
    cudaError_t   sweep(bool first, const CUtensorMap &r_in, const CUtensorMap &v_in, const CUtensorMap &p_in,
                        const CUtensorMap &x, const CUtensorMap &d, T *x_ptr, T *r_out, T *p_out, T *v_out,
                        CGState *st, double *part, unsigned *counter, double *hist, int *err, unsigned spin_limit,
                        cudaStream_t s) const;
  };

  template <typename Td, typename Ts>
  cudaError_t pad_rows(Td *dst, const Ts *src, int n0, int P0, long long rows, cudaStream_t s);
  template <typename Td, typename Ts>
  cudaError_t unpad_rows(Td *dst, const Ts *src, int n0, int P0, long long rows, cudaStream_t s);
} // namespace mpdg
