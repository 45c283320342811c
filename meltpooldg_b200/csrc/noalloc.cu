// Allocation-free heat vmult: the heat apply kernels with their launch bookkeeping (brick ticket,
// per-brick init flags, wait error word) in a fixed file-scope device array instead of memory from
// cudaMalloc.  Callers that must not allocate device memory -- hosts that reserve their whole HBM
// budget in their own pool, time loops in which cudaMalloc / cudaFree would synchronise the device --
// get dst = A src through mpdg_heat_vmult_noalloc without an operator handle.  Nothing here calls
// cudaMalloc, cudaFree or any routine that allocates device memory.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <string>

#include "kernels.h"
#include "mpdg_gpu.h"

// Scratch layout (32-bit words): [0] brick ticket, [1] done counter, [3] wait error word, then one
// init flag per brick from word 64 (byte 256) on.  Every GPU that loads the library holds these
// MPDG_NOALLOC_SCRATCH_BYTES until the process exits; all calls on a device share them.  In host
// code the name only stands for the array: kernels get its device address from
// cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char mpdg_noalloc_scratch[MPDG_NOALLOC_SCRATCH_BYTES];

namespace
{
  constexpr int kMaxDevices    = 64;
  constexpr int kFlagWordStart = 64; // byte 256

  std::mutex g_setup_mutex;
  unsigned  *g_scratch[kMaxDevices] = {};

  // Set-up, once per device, with that device current: the device address of the scratch array.
  cudaError_t
  scratch_of_current_device(unsigned **out)
  {
    int         dev = 0;
    cudaError_t e   = cudaGetDevice(&dev);
    if (e != cudaSuccess)
      return e;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (dev < kMaxDevices && g_scratch[dev])
      {
        *out = g_scratch[dev];
        return cudaSuccess;
      }
    unsigned *ptr = nullptr;
    e             = cudaGetSymbolAddress((void **)&ptr, mpdg_noalloc_scratch);
    if (e != cudaSuccess)
      return e;
    if (dev < kMaxDevices)
      g_scratch[dev] = ptr;
    *out = ptr;
    return cudaSuccess;
  }

  int
  reject(int code, const std::string &msg)
  {
    return mpdg::record_failure(code, msg.c_str());
  }
} // namespace

extern "C" MPDG_API int
mpdg_heat_vmult_noalloc(const mpdg_mesh_desc *mesh, const mpdg_op_params *params, const double *k_cells_dev,
                        double *dst, const double *src, void *cuda_stream)
{
  using namespace mpdg;
  if (!mesh || !params)
    return reject(MPDG_ERR_ARG, "null argument to mpdg_heat_vmult_noalloc");
  if (params->kind != MPDG_HEAT)
    return reject(MPDG_ERR_ARG, "mpdg_heat_vmult_noalloc applies the heat operator only");
  if (mesh->degree < 1 || mesh->degree > 4)
    return reject(MPDG_ERR_UNSUPPORTED, "heat operator: FE_Q degree must be 1..4");
  for (int d = 0; d < 3; ++d)
    if (mesh->cells[d] < 1 || !(mesh->length[d] > 0.0))
      return reject(MPDG_ERR_ARG, "mesh cells and lengths must be positive");
  if (!(params->dt > 0.0))
    return reject(MPDG_ERR_ZERO_DT, "time increment must be positive (ExcZeroTimeIncrement)");
  if (mesh->dirichlet_mask)
    return reject(MPDG_ERR_UNSUPPORTED,
                  "mpdg_heat_vmult_noalloc takes Dirichlet faces only (a per-DoF mask needs device memory)");
  if (params->conductivity_cells)
    return reject(MPDG_ERR_ARG, "mpdg_heat_vmult_noalloc takes a per-cell conductivity as the device array "
                                "k_cells_dev (params->conductivity_cells must be NULL)");
  long long n[3];
  for (int d = 0; d < 3; ++d)
    n[d] = (long long)mesh->degree * mesh->cells[d] + 1;
  if (n[0] * n[1] * n[2] >= (1LL << 31))
    return reject(MPDG_ERR_UNSUPPORTED, "an operator holds fewer than 2^31 DoFs");

  int brick[3];
  heat_brick_shape<double>(mesh->degree, brick, true);
  GridDesc g;
  for (int d = 0; d < 3; ++d)
    {
      g.m[d]   = mesh->cells[d];
      g.nbr[d] = (mesh->cells[d] + brick[d] - 1) / brick[d];
      g.n[d]   = (int)n[d];
    }
  g.faces              = mesh->dirichlet_faces & 63u;
  g.cmask              = nullptr;
  const long long nbrk = (long long)g.nbr[0] * g.nbr[1] * g.nbr[2];
  if (nbrk > (long long)MPDG_NOALLOC_MAX_BRICKS)
    {
      char msg[256];
      std::snprintf(msg, sizeof(msg),
                    "mpdg_heat_vmult_noalloc: the mesh needs %lld brick flags, the fixed scratch array holds at "
                    "most %d (%d bytes); use mpdg_op_vmult",
                    nbrk, (int)MPDG_NOALLOC_MAX_BRICKS, (int)MPDG_NOALLOC_SCRATCH_BYTES);
      return reject(MPDG_ERR_UNSUPPORTED, msg);
    }
  // the vectors are checked last, so a size that is too large is reported whatever they are
  if (!dst || !src)
    return reject(MPDG_ERR_ARG, "null vector passed to mpdg_heat_vmult_noalloc");
  if (dst == src)
    return reject(MPDG_ERR_ARG, "mpdg_heat_vmult_noalloc needs distinct dst and src");

  unsigned   *scratch = nullptr;
  cudaError_t e       = scratch_of_current_device(&scratch);
  if (e != cudaSuccess)
    return reject(MPDG_ERR_CUDA, std::string("cudaGetSymbolAddress of the scratch array: ") + cudaGetErrorString(e));
  cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
  // ticket, done, error word and this mesh's flags must start at zero (epoch 1 marks "initialised")
  e = cudaMemsetAsync(scratch, 0, sizeof(unsigned) * (kFlagWordStart + nbrk), stream);
  if (e != cudaSuccess)
    return reject(MPDG_ERR_CUDA, std::string("clearing the scratch array: ") + cudaGetErrorString(e));

  const double hx = mesh->length[0] / mesh->cells[0], hy = mesh->length[1] / mesh->cells[1],
               hz = mesh->length[2] / mesh->cells[2];
  HeatLaunch<double> h;
  h.degree        = mesh->degree;
  h.mode          = (int)OutMode::Set;
  h.scale         = 1.0;
  h.geo.mass_coef = params->rho_cp / params->dt * hx * hy * hz;
  h.geo.cx        = hy * hz / hx;
  h.geo.cy        = hx * hz / hy;
  h.geo.cz        = hx * hy / hz;
  h.grid          = g;
  h.sync.ticket   = scratch;
  h.sync.done     = scratch + 1;
  h.sync.flags    = scratch + kFlagWordStart;
  h.sync.epoch    = 1u;
  h.sync.error    = reinterpret_cast<int *>(scratch + 3);
  h.kconst        = params->conductivity;
  h.kcell         = k_cells_dev;
  h.src           = src;
  h.dst           = dst;
  h.b             = nullptr;
  h.mask_src      = 1;
  h.skip          = nullptr;
  h.march         = true;
  e               = heat_apply<double>(h, stream);
  if (e != cudaSuccess)
    return reject(MPDG_ERR_CUDA, std::string("heat apply launch: ") + cudaGetErrorString(e));
  return MPDG_OK;
}

extern "C" MPDG_API int
mpdg_heat_vmult_noalloc_errors(void *cuda_stream, int *error_word)
{
  // Reads the wait error word (scratch word 3) after the calls already enqueued on cuda_stream and
  // clears it.  Copies to and from the symbol: no device memory is allocated.
  if (!error_word)
    return reject(MPDG_ERR_ARG, "null argument to mpdg_heat_vmult_noalloc_errors");
  cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
  int          word   = 0;
  const int    zero   = 0;
  const size_t off    = 3 * sizeof(unsigned);
  cudaError_t  e = cudaMemcpyFromSymbolAsync(&word, mpdg_noalloc_scratch, sizeof(int), off, cudaMemcpyDeviceToHost,
                                             stream);
  if (e == cudaSuccess)
    e = cudaMemcpyToSymbolAsync(mpdg_noalloc_scratch, &zero, sizeof(int), off, cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess)
    return reject(MPDG_ERR_CUDA, std::string("reading the scratch error word: ") + cudaGetErrorString(e));
  *error_word = word;
  return MPDG_OK;
}
