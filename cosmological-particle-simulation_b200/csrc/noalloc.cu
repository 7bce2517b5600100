// noalloc.cu — a CIC deposit that allocates no device memory.
//
// cpm_mesh_deposit allocates its scratch (the 64-bit fixed-point mass mesh, staging and sort
// buffers) on first use. Some host programs cannot let a library do that: a program whose device
// memory is owned by its own allocator or pool (a caching allocator that has reserved the GPU's
// memory, an engine with a fixed memory budget), or a real-time loop in which a cudaMalloc — which
// may synchronise the device — would stall its other streams. For them, cpm_mesh_deposit_noalloc
// takes positions and the output mesh as device pointers and keeps its only scratch, the
// fixed-point mesh and a status word, in the file-scope arrays below: meshes up to
// NOALLOC_MAX_MESH^3 cells (64^3 = 262,144 cells, 2 MiB, held on every GPU that loads this library
// until the process exits).
//
// The arrays' addresses are looked up once per device with cudaGetSymbolAddress (the host-side
// name of a __device__ array is not a device address). The first call on each device does that
// lookup.
//
// Every call on a device shares the one array and leaves the last call's sums in it; each call
// clears the cells it uses and the status word before depositing. Calls whose work overlaps on the
// GPU (different streams) race on the arrays: order them on one stream.
//
// The call returns before the GPU has run, so it cannot report bad positions in its return code.
// A NaN or infinite coordinate instead sets every output cell to NaN, which the caller sees once
// its stream has synchronised (cpm_mesh_deposit returns CPM_E_NONFINITE for the same input).
#include <cmath>
#include <mutex>
#include <string>

#include "cpm_host.h"
#include "cpm_internal.cuh"

namespace {

constexpr int NOALLOC_MAX_MESH = 64;
constexpr size_t NOALLOC_MAX_CELLS = (size_t)NOALLOC_MAX_MESH * NOALLOC_MAX_MESH * NOALLOC_MAX_MESH;
constexpr int NOALLOC_MAX_DEVICES = 64;

__device__ __align__(256) unsigned long long g_noalloc_mesh[NOALLOC_MAX_CELLS];
__device__ __align__(256) cpm::DevStatus g_noalloc_status;

struct NoallocAddrs {
  unsigned long long* mesh = nullptr;
  cpm::DevStatus* status = nullptr;
};

std::mutex g_noalloc_mu;
NoallocAddrs g_noalloc_addr[NOALLOC_MAX_DEVICES];

// cells = (float)fx * 2^-shift, as launch_fixed_to_f32; every cell NaN when a position was not finite.
__global__ void k_noalloc_cells(const unsigned long long* __restrict__ fx, size_t m, float inv_scale,
                                const cpm::DevStatus* __restrict__ st, float* __restrict__ out) {
  const bool bad = st->code != cpm::DEV_OK;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x)
    out[i] = bad ? __int_as_float(0x7fc00000) : __fmul_rn(__ull2float_rn(fx[i]), inv_scale);
}

}  // namespace

using namespace cpm;

extern "C" int cpm_mesh_deposit_noalloc(const float* x3_dev, size_t n, int n_mesh, float box_size, float mass,
                                        float* cells_dev, void* stream) {
  if (!cells_dev || (!x3_dev && n))
    return set_error(nullptr, CPM_E_INVALID, "cpm_mesh_deposit_noalloc: null pointer");
  if (n_mesh < 1 || n_mesh > NOALLOC_MAX_MESH)
    return set_error(nullptr, CPM_E_CAPACITY,
                     "cpm_mesh_deposit_noalloc: n_mesh = " + std::to_string(n_mesh) + " exceeds the static scratch of " +
                         std::to_string(NOALLOC_MAX_MESH) + "^3 cells (use cpm_mesh_deposit for larger meshes)");
  if (!(box_size > 0.0f) || !std::isfinite(box_size) || !std::isfinite(mass) || mass < 0.0f)
    return set_error(nullptr, CPM_E_INVALID, "cpm_mesh_deposit_noalloc: box_size must be > 0 and mass finite, >= 0");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return set_error(nullptr, CPM_E_NO_DEVICE, std::string("cpm_mesh_deposit_noalloc: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES)
    return set_error(nullptr, CPM_E_INVALID, "cpm_mesh_deposit_noalloc: device index out of range");
  NoallocAddrs a;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev].mesh) {
      void* pm = nullptr;
      void* ps = nullptr;
      e = cudaGetSymbolAddress(&pm, g_noalloc_mesh);
      if (e == cudaSuccess) e = cudaGetSymbolAddress(&ps, g_noalloc_status);
      if (e != cudaSuccess || !pm || !ps)
        return set_error(nullptr, CPM_E_CUDA,
                         std::string("cpm_mesh_deposit_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_noalloc_addr[dev].mesh = static_cast<unsigned long long*>(pm);
      g_noalloc_addr[dev].status = static_cast<DevStatus*>(ps);
    }
    a = g_noalloc_addr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t m = (size_t)n_mesh * n_mesh * n_mesh;
  const int shift = fixed_point_shift((double)mass * (double)n + 1.0);
  e = cudaMemsetAsync(a.status, 0, sizeof(DevStatus), s);
  if (e != cudaSuccess)
    return set_error(nullptr, CPM_E_CUDA, std::string("cpm_mesh_deposit_noalloc: ") + cudaGetErrorString(e));
  launch_check_finite(x3_dev, n, a.status, s);
  // Zeroes the first m cells of the array, then deposits (sorted input takes the shared-memory tiles).
  launch_deposit_fixed(x3_dev, n, mass, n_mesh, box_size / (float)n_mesh, shift, a.mesh, s);
  count_launch();
  k_noalloc_cells<<<(unsigned)((m + 255) / 256), 256, 0, s>>>(a.mesh, m, std::ldexp(1.0f, -shift), a.status,
                                                               cells_dev);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_error(nullptr, CPM_E_CUDA, std::string("cpm_mesh_deposit_noalloc: ") + cudaGetErrorString(e));
  return CPM_OK;
}
