// noalloc.cu — a CIC deposit that allocates no device memory.
//
// cpm_mesh_deposit allocates its scratch (the 64-bit fixed-point mass mesh, staging and sort
// buffers) on first use. Some callers cannot allow that: code running while a CUDA stream is being
// captured into a graph, or a host program whose device memory is owned by its own allocator or
// pool, may not call cudaMalloc. For them, cpm_mesh_deposit_noalloc takes positions and the output
// mesh as device pointers and keeps its only scratch, the fixed-point mesh, in the file-scope array
// below: meshes up to NOALLOC_MAX_MESH^3 cells (64^3 = 262,144 cells, 2 MiB, held on every GPU that
// loads this library until the process exits).
//
// The array's address is looked up once per device with cudaGetSymbolAddress (the host-side name
// of a __device__ array is not a device address). The first call on each device does that lookup,
// so make that first call before any stream capture begins.
//
// Every call on a device shares the one array and leaves the last call's sums in it; each call
// clears it before depositing. Calls whose work overlaps on the GPU (different streams, or a
// stream and a graph replay) race on the array: order them on one stream.
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

std::mutex g_noalloc_mu;
unsigned long long* g_noalloc_addr[NOALLOC_MAX_DEVICES] = {};

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
  unsigned long long* mesh = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_mesh);
      if (e != cudaSuccess || !p)
        return set_error(nullptr, CPM_E_CUDA,
                         std::string("cpm_mesh_deposit_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_noalloc_addr[dev] = static_cast<unsigned long long*>(p);
    }
    mesh = g_noalloc_addr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t m = (size_t)n_mesh * n_mesh * n_mesh;
  const int shift = fixed_point_shift((double)mass * (double)n + 1.0);
  // Zeroes the first m cells of the array, then deposits; unsorted input takes the global-atomic path.
  launch_deposit_fixed(x3_dev, n, mass, n_mesh, box_size / (float)n_mesh, shift, mesh, s);
  launch_fixed_to_f32(mesh, m, shift, 0, 0.0f, cells_dev, s);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_error(nullptr, CPM_E_CUDA, std::string("cpm_mesh_deposit_noalloc: ") + cudaGetErrorString(e));
  return CPM_OK;
}
