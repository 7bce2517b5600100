// api.cu — the fine-grained C ABI (include/cpm.h): contexts and the per-function entry points
// that stand in for mesh.rs, fft.rs, poisson.rs and tree.rs.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "cpm_internal.cuh"
#include "cpm_host.h"

using namespace cpm;

namespace cpm {

thread_local std::string g_last_error;

int set_error(std::string* slot, int code, const std::string& msg) {
  if (slot) *slot = msg;
  g_last_error = msg;
  return code;
}

int check_device_once(std::string* err) {
  static int state = -1;  // -1 unknown, 0 ok, else error code
  if (state == 0) return CPM_OK;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_error(err, CPM_E_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, dev);
  if (e != cudaSuccess) return set_error(err, CPM_E_NO_DEVICE, cudaGetErrorString(e));
  if (prop.major != 10) {
    return set_error(err, CPM_E_NO_DEVICE,
                     "libcpm_cuda is built for sm_100a; device " + std::string(prop.name) + " is sm_" +
                         std::to_string(prop.major) + std::to_string(prop.minor));
  }
  state = 0;
  return CPM_OK;
}

}  // namespace cpm

struct cpm_ctx {
  int n_mesh = 0;
  float box = 0.0f;
  cudaStream_t stream = nullptr;
  std::string err;
  FftPlan plan;
  SortScratch sort;
  TreeNodes tree;
  DevBuf x, x_sorted, keys, vals, acc, acc_sorted, out;
  DevBuf mesh_fx, mesh_a, mesh_b, mesh_c, mesh_d, spec;
  DevBuf status, tree_counters, pk;
  uint64_t last_nodes = 0, last_pairs = 0, last_accepts = 0;
  uint32_t last_depth = 0;
};

#define CPM_CU(ctx, call)                                                                                    \
  do {                                                                                                       \
    cudaError_t e_ = (call);                                                                                 \
    if (e_ != cudaSuccess)                                                                                   \
      return set_error(&(ctx)->err, e_ == cudaErrorMemoryAllocation ? CPM_E_NOMEM : CPM_E_CUDA,                \
                       std::string(#call) + ": " + cudaGetErrorString(e_));                                  \
  } while (0)

static int sync_and_check(cpm_ctx* c) {
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(&c->err, CPM_E_CUDA, std::string("kernel: ") + cudaGetErrorString(e));
  DevStatus st{0, 0};
  e = cudaMemcpy(&st, c->status.p, sizeof(DevStatus), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return set_error(&c->err, CPM_E_CUDA, cudaGetErrorString(e));
  if (st.code != DEV_OK) {
    cudaMemsetAsync(c->status.p, 0, sizeof(DevStatus), c->stream);
    cudaStreamSynchronize(c->stream);
    if (st.code == DEV_NONFINITE)
      return set_error(&c->err, CPM_E_NONFINITE, "non-finite position at particle " + std::to_string(st.detail));
    return set_error(&c->err, CPM_E_DEVICE,
                     "device status " + std::to_string(st.code) + " detail " + std::to_string(st.detail));
  }
  return CPM_OK;
}

static int reset_status(cpm_ctx* c) {
  CPM_CU(c, ensure(c->status, sizeof(DevStatus)));
  CPM_CU(c, cudaMemsetAsync(c->status.p, 0, sizeof(DevStatus), c->stream));
  return CPM_OK;
}

extern "C" {

const char* cpm_version(void) { return "cpm 0.1.0 sm_100a"; }

const char* cpm_last_error(const cpm_ctx* ctx) { return ctx ? ctx->err.c_str() : g_last_error.c_str(); }

int cpm_ctx_create(int n_mesh, float box_size, size_t max_particles, uint32_t flags, cpm_ctx** out) {
  (void)flags;
  if (!out) return set_error(nullptr, CPM_E_INVALID, "cpm_ctx_create: out is NULL");
  *out = nullptr;
  if (n_mesh <= 0 || !(box_size > 0.0f) || !std::isfinite(box_size))
    return set_error(nullptr, CPM_E_INVALID, "cpm_ctx_create: n_mesh must be > 0 and box_size finite and > 0");
  int rc = check_device_once(nullptr);
  if (rc != CPM_OK) return rc;
  cpm_ctx* c = new cpm_ctx();
  c->n_mesh = n_mesh;
  c->box = box_size;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return set_error(nullptr, CPM_E_CUDA, "cudaStreamCreate failed");
  }
  if (reset_status(c) != CPM_OK) {
    cpm_ctx_destroy(c);
    return set_error(nullptr, CPM_E_NOMEM, "cpm_ctx_create: status word allocation failed");
  }
  if (max_particles) {
    if (ensure(c->x, 3 * max_particles * sizeof(float)) != cudaSuccess) {
      cpm_ctx_destroy(c);
      return set_error(nullptr, CPM_E_NOMEM, "cpm_ctx_create: particle buffer allocation failed");
    }
  }
  *out = c;
  return CPM_OK;
}

int cpm_ctx_destroy(cpm_ctx* c) {
  if (!c) return CPM_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  fft_plan_free(c->plan);
  for (DevBuf* b : {&c->sort.keys_alt, &c->sort.vals_alt, &c->sort.block_hist, &c->sort.scan_tmp, &c->tree.geo,
                    &c->tree.mass, &c->tree.link, &c->tree.counters, &c->tree.prefix, &c->tree.scan_tmp, &c->tree.x4, &c->x,
                    &c->x_sorted, &c->keys, &c->vals, &c->acc, &c->acc_sorted, &c->out, &c->mesh_fx, &c->mesh_a,
                    &c->mesh_b, &c->mesh_c, &c->mesh_d, &c->spec, &c->status, &c->tree_counters, &c->pk})
    release(*b);
  tree_walk_free(c->tree);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return CPM_OK;
}

static int upload_positions(cpm_ctx* c, const float* x3, size_t n) {
  CPM_CU(c, ensure(c->x, 3 * n * sizeof(float)));
  CPM_CU(c, cudaMemcpyAsync(c->x.p, x3, 3 * n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  launch_check_finite(as<float>(c->x), n, as<DevStatus>(c->status), c->stream);
  return CPM_OK;
}

static int mesh_cells(cpm_ctx* c, size_t* m) {
  const size_t n = (size_t)c->n_mesh;
  *m = n * n * n;
  return CPM_OK;
}

// Uploads x3, sorts it by octant key (so that each CTA's particles are compact and the deposit's
// shared-memory tile path is taken) and deposits `mass` per particle into c->mesh_fx.
static int deposit_fixed_ctx(cpm_ctx* c, const float* x3, size_t n, float mass, int* shift_out) {
  size_t m;
  mesh_cells(c, &m);
  int rc;
  CPM_CU(c, ensure(c->mesh_fx, m * sizeof(unsigned long long)));
  if (n) {
    if ((rc = upload_positions(c, x3, n))) return rc;
    CPM_CU(c, ensure(c->keys, n * sizeof(uint64_t)));
    CPM_CU(c, ensure(c->vals, n * sizeof(uint32_t)));
    CPM_CU(c, ensure(c->x_sorted, 3 * n * sizeof(float)));
    launch_octant_keys(as<float>(c->x), n, c->box, KEY_LEVELS, as<uint64_t>(c->keys), as<uint32_t>(c->vals),
                       as<DevStatus>(c->status), c->stream);
    CPM_CU(c, radix_sort_pairs(as<uint64_t>(c->keys), as<uint32_t>(c->vals), n, 3 * KEY_LEVELS, c->sort, c->stream));
    launch_permute3(as<float>(c->x), as<uint32_t>(c->vals), n, as<float>(c->x_sorted), c->stream);
  }
  const float h = c->box / (float)c->n_mesh;
  const int shift = fixed_point_shift((double)std::fabs(mass) * (double)n + 1.0);
  launch_deposit_fixed(as<float>(c->x_sorted), n, mass, c->n_mesh, h, shift, as<unsigned long long>(c->mesh_fx),
                       c->stream);
  *shift_out = shift;
  return CPM_OK;
}

static int deposit_common(cpm_ctx* c, const float* x3, size_t n, float mass, int to_delta, float* out) {
  if (!c) return set_error(nullptr, CPM_E_INVALID, "context is NULL");
  if ((!x3 && n) || !out) return set_error(&c->err, CPM_E_INVALID, "deposit: null pointer");
  if (!std::isfinite(mass)) return set_error(&c->err, CPM_E_INVALID, "deposit: mass must be finite");
  size_t m;
  mesh_cells(c, &m);
  int rc = reset_status(c);
  if (rc) return rc;
  CPM_CU(c, ensure(c->mesh_fx, m * sizeof(unsigned long long)));
  CPM_CU(c, ensure(c->mesh_a, m * sizeof(float)));
  if (n) {
    if ((rc = upload_positions(c, x3, n))) return rc;
    // Sorting by octant key keeps each CTA's particles compact, so the shared-memory tile path is taken.
    CPM_CU(c, ensure(c->keys, n * sizeof(uint64_t)));
    CPM_CU(c, ensure(c->vals, n * sizeof(uint32_t)));
    CPM_CU(c, ensure(c->x_sorted, 3 * n * sizeof(float)));
    launch_octant_keys(as<float>(c->x), n, c->box, KEY_LEVELS, as<uint64_t>(c->keys), as<uint32_t>(c->vals),
                       as<DevStatus>(c->status), c->stream);
    CPM_CU(c, radix_sort_pairs(as<uint64_t>(c->keys), as<uint32_t>(c->vals), n, 3 * KEY_LEVELS, c->sort, c->stream));
    launch_permute3(as<float>(c->x), as<uint32_t>(c->vals), n, as<float>(c->x_sorted), c->stream);
  }
  const float h = c->box / (float)c->n_mesh;
  const double total = (double)std::fabs(mass) * (double)n + 1.0;
  const int shift = fixed_point_shift(total);
  if (mass < 0.0f) return set_error(&c->err, CPM_E_INVALID, "deposit: mass must be >= 0");
  launch_deposit_fixed(as<float>(c->x_sorted), n, mass, c->n_mesh, h, shift, as<unsigned long long>(c->mesh_fx),
                       c->stream);
  const float mean = (float)n / (float)m;
  launch_fixed_to_f32(as<unsigned long long>(c->mesh_fx), m, shift, to_delta, mean, as<float>(c->mesh_a), c->stream);
  CPM_CU(c, cudaMemcpyAsync(out, c->mesh_a.p, m * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  return sync_and_check(c);
}

int cpm_fft_supported(int n) { return fft_supported(n) ? 1 : 0; }

int cpm_density_grid(cpm_ctx* c, const float* delta, int n, float* grid, int* grid_n) {
  if (!c) return set_error(nullptr, CPM_E_INVALID, "context is NULL");
  if (!delta || !grid) return set_error(&c->err, CPM_E_INVALID, "density_grid: null pointer");
  if (n != c->n_mesh) return set_error(&c->err, CPM_E_MESH_MISMATCH, "density_grid: n differs from the context's mesh");
  int rc = reset_status(c);
  if (rc) return rc;
  const size_t m3 = (size_t)n * n * n;
  const int gm = density_grid_side(n);
  const size_t gm3 = (size_t)gm * gm * gm;
  CPM_CU(c, ensure(c->mesh_a, m3 * sizeof(float)));
  CPM_CU(c, ensure(c->mesh_b, gm3 * sizeof(float)));
  CPM_CU(c, cudaMemcpyAsync(c->mesh_a.p, delta, m3 * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  launch_downsample_grid(as<float>(c->mesh_a), n, as<float>(c->mesh_b), c->stream);
  CPM_CU(c, cudaMemcpyAsync(grid, c->mesh_b.p, gm3 * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  if ((rc = sync_and_check(c))) return rc;
  if (grid_n) *grid_n = gm;
  return CPM_OK;
}

int cpm_power_spectrum(cpm_ctx* c, const float* x3, size_t n, int n_shells, double* k_mean, double* p_mean,
                       uint64_t* counts) {
  if (!c) return set_error(nullptr, CPM_E_INVALID, "context is NULL");
  if (!x3 || !k_mean || !p_mean || !counts) return set_error(&c->err, CPM_E_INVALID, "power_spectrum: null pointer");
  if (n == 0) return set_error(&c->err, CPM_E_INVALID, "power_spectrum: no particles");
  if (n_shells < 1 || n_shells > PK_MAX_SHELLS)
    return set_error(&c->err, CPM_E_INVALID, "power_spectrum: n_shells must be in [1, 2048]");
  if (!poisson_supported(c->n_mesh))
    return set_error(&c->err, CPM_E_UNSUPPORTED, std::string("power_spectrum: mesh size must be ") + fft_sizes_text());
  int rc = reset_status(c);
  if (rc) return rc;
  int shift = 0;
  if ((rc = deposit_fixed_ctx(c, x3, n, 1.0f, &shift))) return rc;
  CPM_CU(c, fft_plan_init(c->plan, c->n_mesh));
  CPM_CU(c, ensure(c->spec, half_spectrum_elems(c->n_mesh) * sizeof(float2)));
  CPM_CU(c, ensure(c->pk, sizeof(PkSums)));
  size_t m;
  mesh_cells(c, &m);
  launch_r2c3(c->plan, nullptr, as<unsigned long long>(c->mesh_fx), shift, (float)n / (float)m, as<float2>(c->spec),
              c->stream);
  launch_pk_bin(as<float2>(c->spec), c->n_mesh, n_shells, as<PkSums>(c->pk), c->stream);
  std::vector<PkSums> host(1);
  CPM_CU(c, cudaMemcpyAsync(host.data(), c->pk.p, sizeof(PkSums), cudaMemcpyDeviceToHost, c->stream));
  if ((rc = sync_and_check(c))) return rc;
  pk_finish(host[0], c->n_mesh, c->box, n_shells, k_mean, p_mean, counts);
  return CPM_OK;
}

int cpm_mesh_deposit(cpm_ctx* c, const float* x3, size_t n, float mass, float* cells_out) {
  return deposit_common(c, x3, n, mass, 0, cells_out);
}

int cpm_density_contrast(cpm_ctx* c, const float* x3, size_t n, float* delta_out) {
  return deposit_common(c, x3, n, 1.0f, 1, delta_out);
}

int cpm_mesh_interpolate(cpm_ctx* c, const float* cells, const float* x3, size_t n, float* out) {
  if (!c) return set_error(nullptr, CPM_E_INVALID, "context is NULL");
  if (!cells || (!x3 && n) || (!out && n)) return set_error(&c->err, CPM_E_INVALID, "interpolate: null pointer");
  if (n == 0) return CPM_OK;
  size_t m;
  mesh_cells(c, &m);
  int rc = reset_status(c);
  if (rc) return rc;
  CPM_CU(c, ensure(c->mesh_a, m * sizeof(float)));
  CPM_CU(c, cudaMemcpyAsync(c->mesh_a.p, cells, m * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  if ((rc = upload_positions(c, x3, n))) return rc;
  CPM_CU(c, ensure(c->out, n * sizeof(float)));
  launch_interpolate(as<float>(c->mesh_a), as<float>(c->x), n, c->n_mesh, c->box / (float)c->n_mesh, as<float>(c->out),
                     c->stream);
  CPM_CU(c, cudaMemcpyAsync(out, c->out.p, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  return sync_and_check(c);
}

int cpm_mesh_interpolate3(cpm_ctx* c, const float* gx, const float* gy, const float* gz, const float* x3, size_t n,
                          float* out3) {
  if (!c) return set_error(nullptr, CPM_E_INVALID, "context is NULL");
  if (!gx || !gy || !gz || (!x3 && n) || (!out3 && n))
    return set_error(&c->err, CPM_E_INVALID, "interpolate3: null pointer");
  if (n == 0) return CPM_OK;
  size_t m;
  mesh_cells(c, &m);
  int rc = reset_status(c);
  if (rc) return rc;
  CPM_CU(c, ensure(c->mesh_a, m * sizeof(float)));
  CPM_CU(c, ensure(c->mesh_b, m * sizeof(float)));
  CPM_CU(c, ensure(c->mesh_c, m * sizeof(float)));
  CPM_CU(c, cudaMemcpyAsync(c->mesh_a.p, gx, m * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  CPM_CU(c, cudaMemcpyAsync(c->mesh_b.p, gy, m * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  CPM_CU(c, cudaMemcpyAsync(c->mesh_c.p, gz, m * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  if ((rc = upload_positions(c, x3, n))) return rc;
  CPM_CU(c, ensure(c->acc, 3 * n * sizeof(float)));
  launch_interpolate3(as<float>(c->mesh_a), as<float>(c->mesh_b), as<float>(c->mesh_c), as<float>(c->x), n, c->n_mesh,
                      c->box / (float)c->n_mesh, as<float>(c->acc), c->stream);
  CPM_CU(c, cudaMemcpyAsync(out3, c->acc.p, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  return sync_and_check(c);
}

int cpm_fft3(cpm_ctx* c, cpm_cf32* data, int n, int inverse) {
  if (!c) return set_error(nullptr, CPM_E_INVALID, "context is NULL");
  if (!data) return set_error(&c->err, CPM_E_INVALID, "fft3: data is NULL");
  if (n != c->n_mesh) return set_error(&c->err, CPM_E_MESH_MISMATCH, "fft3: n differs from the context's mesh size");
  if (!fft_supported(n))
    return set_error(&c->err, CPM_E_UNSUPPORTED, "fft3: n = " + std::to_string(n) + " is not one of " + fft_sizes_text());
  int rc = reset_status(c);
  if (rc) return rc;
  CPM_CU(c, fft_plan_init(c->plan, n));
  const size_t m = (size_t)n * n * n;
  CPM_CU(c, ensure(c->spec, m * sizeof(float2)));
  CPM_CU(c, cudaMemcpyAsync(c->spec.p, data, m * sizeof(float2), cudaMemcpyHostToDevice, c->stream));
  launch_fft3_c2c(c->plan, as<float2>(c->spec), inverse ? 1 : 0, c->stream);
  CPM_CU(c, cudaMemcpyAsync(data, c->spec.p, m * sizeof(float2), cudaMemcpyDeviceToHost, c->stream));
  return sync_and_check(c);
}

float cpm_wavenumber(size_t i, size_t n, float box_size) {
  const float two_pi_over_l = 2.0f * (float)3.14159265358979323846 / box_size;
  if (n % 2 == 0 && i == n / 2) return 0.0f;
  if (i <= n / 2) return (float)i * two_pi_over_l;
  return ((float)i - (float)n) * two_pi_over_l;
}

int cpm_poisson_accel(cpm_ctx* c, const float* delta, int n, const cpm_cosmology* cosmo, float a, float r_split,
                      float* gx, float* gy, float* gz) {
  if (!c) return set_error(nullptr, CPM_E_INVALID, "context is NULL");
  if (!delta || !cosmo || !gx || !gy || !gz) return set_error(&c->err, CPM_E_INVALID, "poisson: null pointer");
  if (n != c->n_mesh) return set_error(&c->err, CPM_E_MESH_MISMATCH, "poisson: mesh size must match the solver");
  if (!poisson_supported(n))
    return set_error(&c->err, CPM_E_UNSUPPORTED, "poisson: n = " + std::to_string(n) + " is not one of " + fft_sizes_text());
  if (!(a > 0.0f)) return set_error(&c->err, CPM_E_INVALID, "poisson: a must be > 0");
  int rc = reset_status(c);
  if (rc) return rc;
  CPM_CU(c, fft_plan_init(c->plan, n));
  const size_t m = (size_t)n * n * n;
  const size_t half = half_spectrum_elems(n);
  CPM_CU(c, ensure(c->mesh_d, m * sizeof(float)));
  CPM_CU(c, ensure(c->mesh_a, m * sizeof(float)));
  CPM_CU(c, ensure(c->mesh_b, m * sizeof(float)));
  CPM_CU(c, ensure(c->mesh_c, m * sizeof(float)));
  CPM_CU(c, ensure(c->spec, 3 * half * sizeof(float2)));
  CPM_CU(c, cudaMemcpyAsync(c->mesh_d.p, delta, m * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  PoissonParams pp = make_poisson_params(n, c->box, cosmo->omega_m, a, r_split, 0);
  launch_poisson(c->plan, pp, as<float>(c->mesh_d), nullptr, 0, 0.0f, as<float2>(c->spec), as<float>(c->mesh_a),
                 as<float>(c->mesh_b), as<float>(c->mesh_c), c->stream);
  CPM_CU(c, cudaMemcpyAsync(gx, c->mesh_a.p, m * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  CPM_CU(c, cudaMemcpyAsync(gy, c->mesh_b.p, m * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  CPM_CU(c, cudaMemcpyAsync(gz, c->mesh_c.p, m * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  return sync_and_check(c);
}

cpm_force_split cpm_force_split_with(float box_size, size_t mesh_n, size_t pps, float softening_scale, float theta) {
  const float cell = box_size / (float)mesh_n;
  const float r_split = 1.25f * cell;
  const float spacing = box_size / (float)pps;
  cpm_force_split s;
  s.r_split = r_split;
  s.r_cut = 4.5f * r_split;
  s.softening = softening_scale * spacing;
  s.theta = theta;
  return s;
}

float cpm_short_range_factor(float r, float r_split) {
  const float u = r / (2.0f * r_split);
  return erfcf(u) + TWO_OVER_SQRT_PI * u * std::exp(-u * u);
}

int cpm_tree_accel(cpm_ctx* c, const float* x3, size_t n, float box_size, const cpm_force_split* split, float k,
                   float* acc3) {
  if (!c) return set_error(nullptr, CPM_E_INVALID, "context is NULL");
  if ((!x3 && n) || !split || (!acc3 && n)) return set_error(&c->err, CPM_E_INVALID, "tree_accel: null pointer");
  if (!(box_size > 0.0f)) return set_error(&c->err, CPM_E_INVALID, "tree_accel: box_size must be > 0");
  if (n == 0) return CPM_OK;
  if (n > 0x7FFFFFFFull) return set_error(&c->err, CPM_E_CAPACITY, "tree_accel: more than 2^31-1 particles");
  int rc = reset_status(c);
  if (rc) return rc;
  if ((rc = upload_positions(c, x3, n))) return rc;
  CPM_CU(c, ensure(c->keys, n * sizeof(uint64_t)));
  CPM_CU(c, ensure(c->vals, n * sizeof(uint32_t)));
  CPM_CU(c, ensure(c->x_sorted, 3 * n * sizeof(float)));
  CPM_CU(c, ensure(c->acc_sorted, 3 * n * sizeof(float)));
  CPM_CU(c, ensure(c->acc, 3 * n * sizeof(float)));
  CPM_CU(c, ensure(c->tree_counters, sizeof(TreeCounters)));
  CPM_CU(c, cudaMemsetAsync(c->tree_counters.p, 0, sizeof(TreeCounters), c->stream));
  launch_octant_keys(as<float>(c->x), n, box_size, KEY_LEVELS, as<uint64_t>(c->keys), as<uint32_t>(c->vals),
                     as<DevStatus>(c->status), c->stream);
  CPM_CU(c, radix_sort_pairs(as<uint64_t>(c->keys), as<uint32_t>(c->vals), n, 3 * KEY_LEVELS, c->sort, c->stream));
  launch_permute3(as<float>(c->x), as<uint32_t>(c->vals), n, as<float>(c->x_sorted), c->stream);
  CPM_CU(c, tree_build(c->tree, as<uint64_t>(c->keys), as<float>(c->x_sorted), n, box_size, as<DevStatus>(c->status),
                       c->stream));
  launch_tree_walk(c->tree, as<float>(c->x_sorted), n, box_size, *split, k, as<float>(c->acc_sorted), 0,
                   as<TreeCounters>(c->tree_counters), as<DevStatus>(c->status), c->stream);
  launch_scatter3(as<float>(c->acc_sorted), as<uint32_t>(c->vals), n, as<float>(c->acc), c->stream);
  CPM_CU(c, cudaMemcpyAsync(acc3, c->acc.p, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  rc = sync_and_check(c);
  if (rc) return rc;
  uint32_t cnt[64];
  CPM_CU(c, cudaMemcpy(cnt, c->tree.counters.p, sizeof(cnt), cudaMemcpyDeviceToHost));
  uint64_t nodes = 0;
  for (int d = 0; d <= KEY_LEVELS; ++d) nodes += cnt[d];
  unsigned long long tc[4];
  CPM_CU(c, cudaMemcpy(tc, c->tree_counters.p, sizeof(tc), cudaMemcpyDeviceToHost));
  c->last_nodes = nodes;
  c->last_pairs = tc[0];
  c->last_accepts = tc[1];
  c->last_depth = cnt[33];
  return CPM_OK;
}

int cpm_octant_keys(cpm_ctx* c, const float* x3, size_t n, float box_size, int levels, uint64_t* keys_out,
                    uint32_t* perm_out) {
  if (!c) return set_error(nullptr, CPM_E_INVALID, "context is NULL");
  if ((!x3 && n)) return set_error(&c->err, CPM_E_INVALID, "octant_keys: null pointer");
  if (levels < 1 || levels > KEY_LEVELS) return set_error(&c->err, CPM_E_INVALID, "octant_keys: levels must be 1..21");
  if (n == 0) return CPM_OK;
  int rc = reset_status(c);
  if (rc) return rc;
  if ((rc = upload_positions(c, x3, n))) return rc;
  CPM_CU(c, ensure(c->keys, n * sizeof(uint64_t)));
  CPM_CU(c, ensure(c->vals, n * sizeof(uint32_t)));
  launch_octant_keys(as<float>(c->x), n, box_size, levels, as<uint64_t>(c->keys), as<uint32_t>(c->vals),
                     as<DevStatus>(c->status), c->stream);
  if (keys_out)
    CPM_CU(c, cudaMemcpyAsync(keys_out, c->keys.p, n * sizeof(uint64_t), cudaMemcpyDeviceToHost, c->stream));
  if (perm_out) {
    CPM_CU(c, radix_sort_pairs(as<uint64_t>(c->keys), as<uint32_t>(c->vals), n, 3 * levels, c->sort, c->stream));
    CPM_CU(c, cudaMemcpyAsync(perm_out, c->vals.p, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
  }
  return sync_and_check(c);
}

int cpm_tree_stats(cpm_ctx* c, uint64_t* nodes, uint64_t* leaf_pairs, uint64_t* node_accepts, uint32_t* max_depth) {
  if (!c) return set_error(nullptr, CPM_E_INVALID, "context is NULL");
  if (nodes) *nodes = c->last_nodes;
  if (leaf_pairs) *leaf_pairs = c->last_pairs;
  if (node_accepts) *node_accepts = c->last_accepts;
  if (max_depth) *max_depth = c->last_depth;
  return CPM_OK;
}

}  // extern "C"
