// sim.cu — device-resident simulation (integrator.rs:34-186 `Simulation`).
//
// State lives in HBM in octant-key order: x, p, acc (AoS f32) and id (the caller's index of each
// particle). One KDK step is
//   kick(k1) + drift(d)            (integrator.rs:178-181; k1, d from the reference's f32 factors)
//   keys -> radix sort -> permute x, p, id into key order
//   CIC deposit (u64 fixed point)  -> FFT-Poisson (poisson.rs) -> gather (integrator.rs:144-148)
//   tree build + walk, added to the PM force (integrator.rs:149-159)
//   kick(k2)                       (integrator.rs:183-184)
// Particles are reordered every step; each particle's update is independent of its position in
// the arrays, so the order only changes f32 summation order inside tree leaves.
//
// CUDA graphs. The step's scalars (kick and drift factors, the Green's function prefactor, the
// tree coupling) live in a device block written by a one-thread kernel before each step, so the
// kernel sequence of a step is the same every time except for the sorted-buffer swap, which
// alternates. Each buffer parity gets one graph, captured from the first step of that parity
// that follows an uncaptured (allocating) one and replayed for every later step of that parity.
// CPM_SIM_NO_GRAPH launches every kernel directly, and so does CPM_SIM_TIMING, whose per-phase
// event records are made on the stream between the kernels.
//
// With a net attached (cpm_sim_set_learned), the gather phase also evaluates the learned
// short-range field on the mesh and adds it for particles whose density contrast is below the
// threshold; the tree walk then runs for the other particles only (learned_step.cu).
//
// CPM_SIM_FIXED_POINT keeps the master positions as uint32 fixed point q (x = q L / 2^32) in key
// order beside x: the drift adds round(p d 2^32 / L) to q, so the periodic wrap is exact and the
// resolution is L / 2^32 everywhere in the box; x (f32, what every force kernel reads) is
// rewritten from q after each drift. Positions given by the caller are rounded to the grid.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "cpm_host.h"
#include "cpm_internal.cuh"
#include "tune_cache.h"

using namespace cpm;

namespace {
constexpr int N_PHASES = 8;
}

struct cpm_sim {
  cpm_sim_params P{};
  cudaStream_t stream = nullptr;
  std::string err;
  size_t n = 0;
  float box = 0.0f, h = 0.0f, mean = 0.0f, a = 0.0f;
  int shift = 0;
  FftPlan plan;
  SortScratch sort;
  TreeNodes tree;
  DevBuf x, p, acc, id, x2, p2, id2, keys, vals, fx, gx, gy, gz, spec, status, counters, pk;
  // Per-step phase events, one set per buffer parity. The set of parity q is read back when the
  // next step of parity q is issued: the step in between is already queued, so the GPU does not
  // wait for the host.
  cudaEvent_t ev[2][N_PHASES] = {};
  bool ev_pending[2] = {false, false};
  int ev_set = -1;  // set the current step records into (-1: not inside a step)
  double phase_ms[N_PHASES] = {};
  uint64_t timed_steps = 0;
  uint32_t launches = 0;
  int parity = 0;                     // flips with every force evaluation (the sorted buffers swap)
  bool warm[2] = {false, false};      // an uncaptured step of this parity has run
  bool no_graph[2] = {false, false};  // capture failed for this parity: launch directly
  cudaGraphExec_t graph[2] = {};
  uint32_t graph_launches[2] = {0, 0};
  DevBuf stepv;     // StepScalars of the current step
  DevBuf q, q2;     // fixed-point positions (CPM_SIM_FIXED_POINT) and their sort scratch
  DevBuf snap;      // device outputs of cpm_sim_snapshot
  DevBuf host_tmp;  // caller-order staging of cpm_sim_step_host
  // cpm_sim_step_host copies the new positions out on a second stream while the forces are
  // computed: they are final once the step has sorted them.
  DevBuf host_tmp_x;
  cudaStream_t side = nullptr;
  cudaEvent_t ev_sorted = nullptr;
  float* x_out = nullptr;      // caller-order destination of this step's positions, or null
  bool direct_step = false;    // run the next step uncaptured
  // Learned short-range force (cpm_sim_set_learned): the net, the density-contrast threshold above
  // which particles keep the tree walk, the net's input scale, and the dense-particle list.
  cpm_net* net = nullptr;
  float net_threshold = 50.0f;
  float net_in_scale = 1.0f;
  DevBuf flag, offset, list, list_n, scan_tmp;
  // Octant keys of the particles (the sort is by Hilbert keys in `keys`): as computed, and in the
  // sorted order (the tree build reads each child's octant from them).
  DevBuf okeys, okeys_sorted;
  // A batch of nb boxes of n_box particles each (the ensemble): particles box by box, nb meshes one
  // after another, the box index above `levels` octant digits in the sort keys. nb = 1: one box.
  int nb = 1;
  size_t n_box = 0;
  int levels = KEY_LEVELS;
  // Autotuned launch choices (FFT plan in `plan`, walk warps in `tree`) and the timings.
  int dep_ppt = 4;
  float tune_ms[N_TUNE] = {};
  bool tuned = false;
};

#define SIM_CU(s, call)                                                                                      \
  do {                                                                                                       \
    cudaError_t e_ = (call);                                                                                 \
    if (e_ != cudaSuccess)                                                                                   \
      return set_error(&(s)->err, e_ == cudaErrorMemoryAllocation ? CPM_E_NOMEM : CPM_E_CUDA,                \
                       std::string(#call) + ": " + cudaGetErrorString(e_));                                  \
  } while (0)

static int sim_check(cpm_sim* s) {
  cudaError_t e = cudaStreamSynchronize(s->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(&s->err, CPM_E_CUDA, std::string("kernel: ") + cudaGetErrorString(e));
  DevStatus st{0, 0};
  e = cudaMemcpy(&st, s->status.p, sizeof(st), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return set_error(&s->err, CPM_E_CUDA, cudaGetErrorString(e));
  if (st.code != DEV_OK) {
    cudaMemset(s->status.p, 0, sizeof(DevStatus));
    if (st.code == DEV_NONFINITE)
      return set_error(&s->err, CPM_E_NONFINITE, "non-finite position at particle " + std::to_string(st.detail));
    return set_error(&s->err, CPM_E_DEVICE,
                     "device status " + std::to_string(st.code) + " detail " + std::to_string(st.detail));
  }
  if (s->net) {  // the net's kernels report a wait that ran out in their own status word
    int ns = 0;
    e = cudaMemcpy(&ns, net_status_word(s->net), sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return set_error(&s->err, CPM_E_CUDA, cudaGetErrorString(e));
    if (ns != 0) {
      cudaMemset(net_status_word(s->net), 0, sizeof(int));
      return set_error(&s->err, CPM_E_DEVICE, "learned short-range net: status " + std::to_string(ns));
    }
  }
  return CPM_OK;
}

static void mark(cpm_sim* s, int phase) {
  if ((s->P.flags & CPM_SIM_TIMING) && s->ev_set >= 0) cudaEventRecord(s->ev[s->ev_set][phase], s->stream);
}

// Folds the recorded step of event set q into phase_ms. Phases: 0 kick+drift, 1 keys+sort+reorder,
// 2 deposit, 3 FFT-Poisson, 4 gather, 5 tree build, 6 walk + second kick, 7 whole step.
static int flush_set(cpm_sim* s, int q) {
  if (!s->ev_pending[q]) return CPM_OK;
  SIM_CU(s, cudaEventSynchronize(s->ev[q][7]));
  float ms;
  for (int ph = 0; ph < 6; ++ph) {
    SIM_CU(s, cudaEventElapsedTime(&ms, s->ev[q][ph], s->ev[q][ph + 1]));
    s->phase_ms[ph] += ms;
  }
  SIM_CU(s, cudaEventElapsedTime(&ms, s->ev[q][6], s->ev[q][7]));
  s->phase_ms[6] += ms;
  SIM_CU(s, cudaEventElapsedTime(&ms, s->ev[q][0], s->ev[q][7]));
  s->phase_ms[7] += ms;
  s->timed_steps += 1;
  s->ev_pending[q] = false;
  return CPM_OK;
}

static int flush_timing(cpm_sim* s) {
  int rc = flush_set(s, s->parity ^ 1);
  if (!rc) rc = flush_set(s, s->parity);
  return rc;
}

// The swap of the sorted buffers that ends a key sort.
static void swap_sorted(cpm_sim* s) {
  std::swap(s->x, s->x2);
  std::swap(s->p, s->p2);
  std::swap(s->id, s->id2);
  std::swap(s->q, s->q2);
  s->parity ^= 1;
}

static bool fixed_point(const cpm_sim* s) { return (s->P.flags & CPM_SIM_FIXED_POINT) != 0; }

// Particles of one box (the N of the reference's formulas, integrator.rs:120, :152).
static size_t per_box(const cpm_sim* s) { return s->nb > 1 ? s->n_box : s->n; }
// Particles per box of a batch, 0 for a single box (the batched kernels' parameter).
static size_t batch_box(const cpm_sim* s) { return s->nb > 1 ? s->n_box : 0; }
static size_t mesh_cells(const cpm_sim* s) { return (size_t)s->P.mesh_n * s->P.mesh_n * s->P.mesh_n; }

// Output scale of the learned short-range field: the tree coupling K(a) (integrator.rs:150-152) times
// the mean particles per cell over the cell size, which makes the net's output dimensionless.
static float net_field_scale(const cpm_sim* s, float a) {
  const float m = (float)((double)s->P.mesh_n * s->P.mesh_n * s->P.mesh_n);
  return tree_coupling(s->P.cosmo.omega_m, s->box, a, per_box(s)) * ((float)per_box(s) / m) / s->h;
}

// Sort into key order, then the force: deposit, FFT-Poisson, gather, tree. Phases 1..6. With
// `dev`, the Poisson prefactor and the tree coupling are read from the device step block.
static int sim_accelerations(cpm_sim* s, float a, const StepScalars* dev = nullptr) {
  const size_t n = s->n;
  const int mn = s->P.mesh_n;
  mark(s, 1);
  // Hilbert order: sorting by the Hilbert keys of the octant cubes keeps every octree node's
  // particles contiguous (the tree is the same), and the walk's groups of 32 consecutive particles
  // are more compact than in octant order, so fewer sources lie in a group's reach but outside its
  // particles' own.
  launch_octant_keys(as<float>(s->x), n, s->box, s->levels, as<uint64_t>(s->okeys), as<uint32_t>(s->vals),
                     as<DevStatus>(s->status), s->stream, batch_box(s), as<uint64_t>(s->keys));
  SIM_CU(s, radix_sort_pairs(as<uint64_t>(s->keys), as<uint32_t>(s->vals), n, 63, s->sort, s->stream));
  launch_permute_u64(as<uint64_t>(s->okeys), as<uint32_t>(s->vals), n, as<uint64_t>(s->okeys_sorted), s->stream);
  launch_permute3(as<float>(s->x), as<uint32_t>(s->vals), n, as<float>(s->x2), s->stream);
  launch_permute3(as<float>(s->p), as<uint32_t>(s->vals), n, as<float>(s->p2), s->stream);
  launch_permute_u32(as<uint32_t>(s->id), as<uint32_t>(s->vals), n, as<uint32_t>(s->id2), s->stream);
  if (fixed_point(s))  // the 32-bit words of q move like those of x
    launch_permute3(as<float>(s->q), as<uint32_t>(s->vals), n, as<float>(s->q2), s->stream);
  swap_sorted(s);
  if (s->x_out) {
    SIM_CU(s, cudaEventRecord(s->ev_sorted, s->stream));
    SIM_CU(s, cudaStreamWaitEvent(s->side, s->ev_sorted, 0));
    launch_scatter3(as<float>(s->x), as<uint32_t>(s->id), n, as<float>(s->host_tmp_x), s->side);
    SIM_CU(s, cudaMemcpyAsync(s->x_out, s->host_tmp_x.p, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, s->side));
    s->x_out = nullptr;
  }
  mark(s, 2);
  launch_deposit_fixed(as<float>(s->x), n, 1.0f, mn, s->h, s->shift, as<unsigned long long>(s->fx), s->stream,
                       s->dep_ppt, batch_box(s));
  mark(s, 3);
  const float r_split = s->P.use_tree ? s->P.split.r_split : 0.0f;
  PoissonParams pp =
      make_poisson_params(mn, s->box, s->P.cosmo.omega_m, a, r_split, (s->P.flags & CPM_SIM_DECONVOLVE) ? 1 : 0);
  if (dev) pp.prefactor_dev = &dev->prefactor;
  pp.boxes = s->nb;
  launch_poisson(s->plan, pp, nullptr, as<unsigned long long>(s->fx), s->shift, s->mean, as<float2>(s->spec),
                 as<float>(s->gx), as<float>(s->gy), as<float>(s->gz), s->stream);
  mark(s, 4);
  const bool learned = s->net && s->P.use_tree;
  if (learned) {
    const float scale = net_field_scale(s, a);
    const float4* field = net_field_from_mesh(s->net, as<unsigned long long>(s->fx), s->shift, s->mean, s->net_in_scale,
                                              scale, dev ? &dev->net_scale : nullptr, s->stream);
    launch_learned_gather(as<float>(s->gx), as<float>(s->gy), as<float>(s->gz), as<unsigned long long>(s->fx),
                          s->shift, s->mean, field, as<float>(s->x), n, mn, s->h, s->net_threshold, as<float>(s->acc),
                          as<uint32_t>(s->flag), s->stream);
  } else {
    launch_interpolate3(as<float>(s->gx), as<float>(s->gy), as<float>(s->gz), as<float>(s->x), n, mn, s->h,
                        as<float>(s->acc), s->stream, batch_box(s));
  }
  mark(s, 5);
  if (s->P.use_tree) {
    if (learned)
      SIM_CU(s, launch_compact(as<uint32_t>(s->flag), as<uint32_t>(s->offset), n, as<uint32_t>(s->list),
                               as<uint32_t>(s->list_n), s->scan_tmp, s->stream));
    const uint32_t* walk_list = learned ? as<uint32_t>(s->list) : nullptr;
    const uint32_t* walk_n = learned ? as<uint32_t>(s->list_n) : nullptr;
    const float quad_half = (s->P.flags & CPM_SIM_QUADRUPOLE) ? quad_half_bound(s->P.split) : 0.0f;
    SIM_CU(s, tree_build(s->tree, as<uint64_t>(s->keys), as<float>(s->x), n, s->box, as<DevStatus>(s->status),
                         s->stream, quad_half, s->levels, batch_box(s), as<uint64_t>(s->okeys_sorted)));
    mark(s, 6);
    SIM_CU(s, cudaMemsetAsync(s->counters.p, 0, sizeof(TreeCounters), s->stream));
    const float k = tree_coupling(s->P.cosmo.omega_m, s->box, a, per_box(s));
    launch_tree_walk(s->tree, as<float>(s->x), n, s->box, s->P.split, k, as<float>(s->acc), 1,
                     as<TreeCounters>(s->counters), as<DevStatus>(s->status), s->stream,
                     dev ? &dev->tree_k : nullptr, walk_list, walk_n);
  } else {
    mark(s, 6);
  }
  return CPM_OK;
}

// ---------------------------------------------------------------------------------------------
// Autotuner. The compiled alternatives of three launch parameters are timed on the simulation's
// own first state (after its first force evaluation, so the mesh, the sorted particles and the tree
// are real), and the fastest is kept:
//   FFT plan of the Poisson passes        Stockham stages of largest radix 8 (512 = 8.8.8) or 4
//                                         (4.4.4.4.2) over the CTA, or (0) one warp per 256- or
//                                         512-point line with register stages (radix 8 elsewhere)
//   deposit tile                          256 x {2, 4, 8} sorted particles per CTA
//   walk group                            {2, 4, 8} warps of 32 particles per block
// Each candidate runs once untimed and twice timed with CUDA events on the simulation's stream;
// the work repeats what the force evaluation did (deposit, Poisson solve) or writes to scratch
// (walk), so the state is unchanged. Choices are cached per workload (particles, mesh, tree,
// quadrupoles) for the process, and in the file named by CPM_TUNE_CACHE when it is set (one line
// per workload: key, plan, tile, warps). CPM_SIM_NO_AUTOTUNE keeps 8, 4 and 4.
namespace {
std::mutex g_tune_mu;
std::map<std::string, TuneChoice> g_tune_cache;
bool g_tune_file_read = false;

std::string sim_tune_key(const cpm_sim* s) {
  return cpm::tune_key(per_box(s), s->P.mesh_n, s->nb, s->P.use_tree, (s->P.flags & CPM_SIM_QUADRUPOLE) ? 1 : 0);
}

template <typename F>
float time_ms(cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1, F&& f) {
  f();
  cudaEventRecord(e0, st);
  f();
  f();
  cudaEventRecord(e1, st);
  cudaEventSynchronize(e1);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, e0, e1);
  return 0.5f * ms;
}
}  // namespace

static void apply_tuning(cpm_sim* s, const TuneChoice& c) {
  s->plan.max_radix = c.radix;
  s->dep_ppt = c.ppt;
  s->tree.walk_warps = c.warps;
  for (int i = 0; i < N_TUNE; ++i) s->tune_ms[i] = c.ms[i];
  s->tuned = true;
}

// A workload tuned before (this process or the cache file) takes its choices before its first
// force evaluation, so that its arithmetic (the radix plan rounds differently) is that of the plan
// it keeps.
static void sim_apply_cached_tuning(cpm_sim* s) {
  if (s->P.flags & CPM_SIM_NO_AUTOTUNE) return;
  std::lock_guard<std::mutex> lock(g_tune_mu);
  if (!g_tune_file_read) {
    tune_file_load(std::getenv("CPM_TUNE_CACHE"), g_tune_cache);
    g_tune_file_read = true;
  }
  auto it = g_tune_cache.find(sim_tune_key(s));
  if (it != g_tune_cache.end()) apply_tuning(s, it->second);
}

static int sim_autotune(cpm_sim* s) {
  if ((s->P.flags & CPM_SIM_NO_AUTOTUNE) || s->tuned) return CPM_OK;
  const std::string key = sim_tune_key(s);
  const int radix_used = s->plan.max_radix;
  SIM_CU(s, cudaStreamSynchronize(s->stream));
  cudaEvent_t e0, e1;
  SIM_CU(s, cudaEventCreate(&e0));
  SIM_CU(s, cudaEventCreate(&e1));
  TuneChoice c;
  const int mn = s->P.mesh_n;
  const float r_split = s->P.use_tree ? s->P.split.r_split : 0.0f;
  PoissonParams pp =
      make_poisson_params(mn, s->box, s->P.cosmo.omega_m, s->a, r_split, (s->P.flags & CPM_SIM_DECONVOLVE) ? 1 : 0);
  pp.boxes = s->nb;
  for (int k = 0; k < 3; ++k) {
    s->plan.max_radix = TUNE_PLANS[k];
    c.ms[k] = time_ms(s->stream, e0, e1, [&] {
      launch_poisson(s->plan, pp, nullptr, as<unsigned long long>(s->fx), s->shift, s->mean, as<float2>(s->spec),
                     as<float>(s->gx), as<float>(s->gy), as<float>(s->gz), s->stream);
    });
  }
  for (int k = 0; k < 3; ++k) {
    c.ms[3 + k] = time_ms(s->stream, e0, e1, [&] {
      launch_deposit_fixed(as<float>(s->x), s->n, 1.0f, mn, s->h, s->shift, as<unsigned long long>(s->fx), s->stream,
                           TUNE_PPT[k], batch_box(s));
    });
  }
  if (s->P.use_tree && s->tree.geo.p && !(s->P.flags & CPM_SIM_QUADRUPOLE)) {
    int rc = ensure(s->host_tmp, 3 * s->n * sizeof(float)) == cudaSuccess ? CPM_OK : CPM_E_NOMEM;
    if (rc) return set_error(&s->err, rc, "autotune: scratch allocation failed");
    const float kk = tree_coupling(s->P.cosmo.omega_m, s->box, s->a, per_box(s));
    // the walk as the step runs it (a learned simulation's list from the first force evaluation)
    const bool learned = s->net != nullptr;
    const uint32_t* wl = learned ? as<uint32_t>(s->list) : nullptr;
    const uint32_t* wn = learned ? as<uint32_t>(s->list_n) : nullptr;
    for (int k = 0; k < 3; ++k) {
      s->tree.walk_warps = TUNE_WARPS[k];
      c.ms[6 + k] = time_ms(s->stream, e0, e1, [&] {
        launch_tree_walk(s->tree, as<float>(s->x), s->n, s->box, s->P.split, kk, as<float>(s->host_tmp), 0, nullptr,
                         as<DevStatus>(s->status), s->stream, nullptr, wl, wn);
      });
    }
  }
  tune_select(c);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  apply_tuning(s, c);
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_cache[key] = c;
    tune_file_append(std::getenv("CPM_TUNE_CACHE"), key, c);
  }
  int rc = sim_check(s);
  // the first force evaluation ran with another radix plan: repeat it with the one kept
  if (!rc && c.radix != radix_used && (rc = sim_accelerations(s, s->a, nullptr)) == CPM_OK) rc = sim_check(s);
  return rc;
}

// Validates the parameters and allocates every device buffer of a simulation.
static int sim_new(const cpm_sim_params* params, float a0, cpm_sim** out, int nb = 1) {
  const cpm_sim_params& P = *params;
  if (P.n_particles == 0 || P.n_particles * (size_t)(nb > 0 ? nb : 1) > 0x7FFFFFFFull)
    return set_error(nullptr, CPM_E_INVALID, "cpm_sim_create: n_particles must be in [1, 2^31)");
  if (nb < 1 || nb > 64 || (nb > 1 && (P.n_particles % 2048 != 0 || P.mesh_n > 512)))
    return set_error(nullptr, CPM_E_INVALID,
                     "batch: 1..64 boxes of a multiple of 2048 particles each, meshes up to 512");
  if (!(P.box_size > 0.0f) || !(a0 > 0.0f)) return set_error(nullptr, CPM_E_INVALID, "cpm_sim_create: box and a0 must be > 0");
  if (!poisson_supported(P.mesh_n))
    return set_error(nullptr, CPM_E_UNSUPPORTED,
                     "cpm_sim_create: mesh_n = " + std::to_string(P.mesh_n) + " is not one of " + fft_sizes_text());
  int rc = check_device_once(nullptr);
  if (rc) return rc;
  cpm_sim* s = new cpm_sim();
  s->P = P;
  s->nb = nb;
  s->n_box = P.n_particles;
  s->levels = nb > 1 ? KEY_LEVELS - 2 : KEY_LEVELS;  // 19 octant digits under 6 bits of box index
  s->tree.n_box = nb > 1 ? (uint32_t)P.n_particles : 0u;
  s->n = P.n_particles * (size_t)nb;
  s->box = P.box_size;
  s->h = P.box_size / (float)P.mesh_n;
  const size_t m = (size_t)P.mesh_n * P.mesh_n * P.mesh_n * (size_t)nb;
  s->mean = (float)P.n_particles / (float)((size_t)P.mesh_n * P.mesh_n * P.mesh_n);  // integrator.rs:120-121
  s->shift = fixed_point_shift((double)P.n_particles + 1.0);
  s->a = a0;
  auto fail = [&](int code) {
    g_last_error = s->err;
    cpm_sim_destroy(s);
    return code;
  };
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(CPM_E_CUDA);
  if (P.flags & CPM_SIM_TIMING)
    for (auto& row : s->ev)
      for (auto& e : row)
        if (cudaEventCreate(&e) != cudaSuccess) return fail(CPM_E_CUDA);
  const size_t n = s->n;
  const size_t half = half_spectrum_elems(P.mesh_n);
  bool ok = true;
  for (DevBuf* b : {&s->x, &s->p, &s->acc, &s->x2, &s->p2}) ok = ok && ensure(*b, 3 * n * sizeof(float)) == cudaSuccess;
  for (DevBuf* b : {&s->id, &s->id2, &s->vals}) ok = ok && ensure(*b, n * sizeof(uint32_t)) == cudaSuccess;
  ok = ok && ensure(s->keys, n * sizeof(uint64_t)) == cudaSuccess;
  ok = ok && ensure(s->okeys, n * sizeof(uint64_t)) == cudaSuccess;
  ok = ok && ensure(s->okeys_sorted, n * sizeof(uint64_t)) == cudaSuccess;
  ok = ok && ensure(s->fx, m * sizeof(unsigned long long)) == cudaSuccess;
  for (DevBuf* b : {&s->gx, &s->gy, &s->gz}) ok = ok && ensure(*b, m * sizeof(float)) == cudaSuccess;
  ok = ok && ensure(s->spec, 3 * half * (size_t)nb * sizeof(float2)) == cudaSuccess;
  ok = ok && ensure(s->status, sizeof(DevStatus)) == cudaSuccess;
  ok = ok && ensure(s->counters, sizeof(TreeCounters)) == cudaSuccess;
  ok = ok && ensure(s->stepv, sizeof(StepScalars)) == cudaSuccess;
  if (P.flags & CPM_SIM_FIXED_POINT)
    for (DevBuf* b : {&s->q, &s->q2}) ok = ok && ensure(*b, 3 * n * sizeof(uint32_t)) == cudaSuccess;
  ok = ok && fft_plan_init(s->plan, P.mesh_n) == cudaSuccess;
  if (!ok) {
    s->err = "cpm_sim_create: device allocation failed";
    return fail(CPM_E_NOMEM);
  }
  cudaMemsetAsync(s->status.p, 0, sizeof(DevStatus), s->stream);
  cudaMemsetAsync(s->counters.p, 0, sizeof(TreeCounters), s->stream);
  sim_apply_cached_tuning(s);
  *out = s;
  return CPM_OK;
}

extern "C" {

int cpm_sim_create(const cpm_sim_params* params, const float* x3, const float* p3, float a0, cpm_sim** out) {
  if (!out) return set_error(nullptr, CPM_E_INVALID, "cpm_sim_create: out is NULL");
  *out = nullptr;
  if (!params || !x3 || !p3) return set_error(nullptr, CPM_E_INVALID, "cpm_sim_create: null pointer");
  cpm_sim* s = nullptr;
  int rc = sim_new(params, a0, &s);
  if (rc) return rc;
  if ((rc = cpm_sim_set_state(s, x3, p3)) != CPM_OK || (rc = sim_autotune(s)) != CPM_OK) {
    g_last_error = s->err;
    cpm_sim_destroy(s);
    return rc;
  }
  *out = s;
  return CPM_OK;
}

int cpm_sim_create_zeldovich(const cpm_sim_params* params, int n_side, float n_s, float sigma8, float a0,
                             uint64_t seed, cpm_sim** out) {
  if (!out) return set_error(nullptr, CPM_E_INVALID, "cpm_sim_create_zeldovich: out is NULL");
  *out = nullptr;
  if (!params) return set_error(nullptr, CPM_E_INVALID, "cpm_sim_create_zeldovich: params is NULL");
  if (!fft_supported(n_side) || (size_t)n_side * n_side * n_side != params->n_particles)
    return set_error(nullptr, CPM_E_INVALID,
                     std::string("cpm_sim_create_zeldovich: n_side must be one of ") + fft_sizes_text() + " with n_side^3 == n_particles");
  if (!(sigma8 > 0.0f)) return set_error(nullptr, CPM_E_INVALID, "cpm_sim_create_zeldovich: sigma8 must be > 0");
  cpm_sim* s = nullptr;
  int rc = sim_new(params, a0, &s);
  if (rc) return rc;
  DevBuf modes, work;
  FftPlan plan;
  cudaError_t e = generate_zeldovich(n_side, s->box, s->P.cosmo, n_s, sigma8, a0, seed, as<float>(s->x),
                                     as<float>(s->p), modes, work, plan, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  release(modes);
  release(work);
  fft_plan_free(plan);
  if (e != cudaSuccess) {
    set_error(&s->err, e == cudaErrorMemoryAllocation ? CPM_E_NOMEM : CPM_E_CUDA,
              std::string("cpm_sim_create_zeldovich: ") + cudaGetErrorString(e));
    cpm_sim_destroy(s);
    return e == cudaErrorMemoryAllocation ? CPM_E_NOMEM : CPM_E_CUDA;
  }
  launch_iota(as<uint32_t>(s->id), s->n, s->stream);
  if (fixed_point(s)) launch_to_fixed(as<float>(s->x), as<uint32_t>(s->q), s->n, s->box, s->stream);
  rc = sim_accelerations(s, s->a);
  if (rc == CPM_OK) rc = sim_check(s);
  if (rc == CPM_OK) rc = sim_autotune(s);
  if (rc) {
    g_last_error = s->err;
    cpm_sim_destroy(s);
    return rc;
  }
  *out = s;
  return CPM_OK;
}

int cpm_sim_set_state(cpm_sim* s, const float* x3, const float* p3) {
  if (!s || !x3 || !p3) return set_error(s ? &s->err : nullptr, CPM_E_INVALID, "cpm_sim_set_state: null pointer");
  const size_t n = s->n;
  SIM_CU(s, cudaMemcpyAsync(s->x.p, x3, 3 * n * sizeof(float), cudaMemcpyHostToDevice, s->stream));
  SIM_CU(s, cudaMemcpyAsync(s->p.p, p3, 3 * n * sizeof(float), cudaMemcpyHostToDevice, s->stream));
  std::vector<uint32_t> iota(n);
  for (size_t i = 0; i < n; ++i) iota[i] = (uint32_t)i;
  SIM_CU(s, cudaMemcpyAsync(s->id.p, iota.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream));
  launch_check_finite(as<float>(s->x), n, as<DevStatus>(s->status), s->stream);
  if (fixed_point(s)) launch_to_fixed(as<float>(s->x), as<uint32_t>(s->q), n, s->box, s->stream);
  int rc = sim_accelerations(s, s->a);
  if (rc) return rc;
  return sim_check(s);
}

// One KDK step with the scalars in the device block: phases 0..7.
static int step_body(cpm_sim* s, float a1) {
  const StepScalars* dev = as<StepScalars>(s->stepv);
  mark(s, 0);
  if (fixed_point(s))
    launch_kick_drift_fixed(as<uint32_t>(s->q), as<float>(s->x), as<float>(s->p), as<float>(s->acc), s->n, s->box,
                            s->stream, dev);
  else
    launch_kick_kick_drift(as<float>(s->x), as<float>(s->p), as<float>(s->acc), s->n, 0.0f, 0, 0.0f, 0.0f, s->box,
                           s->stream, dev);
  int rc = sim_accelerations(s, a1, dev);
  if (rc) return rc;
  launch_kick(as<float>(s->p), as<float>(s->acc), s->n, 0.0f, s->stream, &dev->k2);
  mark(s, 7);
  return CPM_OK;
}

// Captures step_body into the graph of parity q and launches it. On a capture failure the
// host-side buffer swap is undone and the step runs uncaptured (and parity q stays uncaptured).
static int step_captured(cpm_sim* s, int q, float a1) {
  const unsigned long long l0 = launch_count();
  cudaError_t e = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
  int rc = e == cudaSuccess ? step_body(s, a1) : CPM_E_CUDA;
  cudaGraph_t g = nullptr;
  if (e == cudaSuccess) e = cudaStreamEndCapture(s->stream, &g);
  if (rc == CPM_OK && e == cudaSuccess && g) e = cudaGraphInstantiate(&s->graph[q], g, 0);
  if (g) cudaGraphDestroy(g);
  if (rc != CPM_OK || e != cudaSuccess || !s->graph[q]) {
    cudaGetLastError();
    if (s->graph[q]) cudaGraphExecDestroy(s->graph[q]);
    s->graph[q] = nullptr;
    s->no_graph[q] = true;
    if (s->parity != q) swap_sorted(s);
    return step_body(s, a1);
  }
  s->graph_launches[q] = (uint32_t)(launch_count() - l0);
  SIM_CU(s, cudaGraphLaunch(s->graph[q], s->stream));
  return CPM_OK;
}

// Writes the scalars of the step a -> a1 into the device step block, on stream `st`: the reference's
// f32 factors (integrator.rs:263-297) from the host, or in precision mode the FP64 device factors.
static void sim_write_step_scalars(cpm_sim* s, float a1, cudaStream_t st) {
  const cpm_cosmology& c = s->P.cosmo;
  const float a0 = s->a;
  if (fixed_point(s)) {
    const double m = (double)s->P.mesh_n * s->P.mesh_n * s->P.mesh_n;
    launch_step_factors64(as<StepScalars>(s->stepv), c, (double)a0, (double)a1, (double)s->box, (double)per_box(s),
                          ((double)per_box(s) / m) / (double)s->h, st);
    return;
  }
  const float am = midpoint(c, a0, a1);
  StepScalars sc;
  sc.k1 = kick_factor(c, a0, am);
  sc.d = drift_factor(c, a0, a1);
  sc.k2 = kick_factor(c, am, a1);
  sc.prefactor = make_poisson_params(s->P.mesh_n, s->box, c.omega_m, a1, 0.0f, 0).prefactor;
  sc.tree_k = tree_coupling(c.omega_m, s->box, a1, per_box(s));
  sc.net_scale = net_field_scale(s, a1);
  sc.pad_ = 0.0f;
  sc.d64 = (double)sc.d;
  launch_set_step_scalars(as<StepScalars>(s->stepv), sc, st);
}

int cpm_sim_step_to(cpm_sim* s, float a1) {
  if (!s) return set_error(nullptr, CPM_E_INVALID, "cpm_sim_step_to: sim is NULL");
  if (!(a1 > 0.0f) || !std::isfinite(a1)) return set_error(&s->err, CPM_E_INVALID, "cpm_sim_step_to: a1 must be > 0");
  const int q = s->parity;
  int rc;
  if ((s->P.flags & CPM_SIM_TIMING) && (rc = flush_set(s, q))) return rc;
  sim_write_step_scalars(s, a1, s->stream);
  const unsigned long long l0 = launch_count();
  s->ev_set = q;
  const bool graphs =
      !(s->P.flags & (CPM_SIM_NO_GRAPH | CPM_SIM_TIMING)) && !s->direct_step && s->warm[q] && !s->no_graph[q];
  if (graphs && s->graph[q]) {
    const cudaError_t e = cudaGraphLaunch(s->graph[q], s->stream);
    if (e == cudaSuccess) swap_sorted(s);  // the host side of the replayed sort
    rc = e == cudaSuccess ? CPM_OK
                          : set_error(&s->err, CPM_E_CUDA, std::string("cudaGraphLaunch: ") + cudaGetErrorString(e));
    s->launches = 1 + s->graph_launches[q];
  } else if (graphs) {
    rc = step_captured(s, q, a1);
    s->launches = 1 + (s->graph[q] ? s->graph_launches[q] : (uint32_t)(launch_count() - l0));
  } else {
    rc = step_body(s, a1);
    s->warm[q] = true;
    s->launches = 1 + (uint32_t)(launch_count() - l0);
  }
  s->ev_set = -1;
  if (rc) return rc;
  if (s->P.flags & CPM_SIM_TIMING) s->ev_pending[q] = true;
  s->a = a1;
  return CPM_OK;
}

// Scatter caller-order host data through the staging buffer into key order: dst[i] = src[id[i]].
static int upload_caller_order(cpm_sim* s, const float* host3, float* dst3) {
  const size_t n = s->n;
  SIM_CU(s, ensure(s->host_tmp, 3 * n * sizeof(float)));
  SIM_CU(s, cudaMemcpyAsync(s->host_tmp.p, host3, 3 * n * sizeof(float), cudaMemcpyHostToDevice, s->stream));
  launch_permute3(as<float>(s->host_tmp), as<uint32_t>(s->id), n, dst3, s->stream);
  return CPM_OK;
}

static int download_caller_order(cpm_sim* s, const float* src3, float* host3) {
  const size_t n = s->n;
  SIM_CU(s, ensure(s->host_tmp, 3 * n * sizeof(float)));
  launch_scatter3(src3, as<uint32_t>(s->id), n, as<float>(s->host_tmp), s->stream);
  SIM_CU(s, cudaMemcpyAsync(host3, s->host_tmp.p, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
  return CPM_OK;
}

// The step runs uncaptured so that the positions' copy to the host can start on the second
// stream right after the sort and overlap the force computation; the momenta follow at the end.
int cpm_sim_step_host(cpm_sim* s, float a1, float* x3, float* p3) {
  if (!s || !x3 || !p3) return set_error(s ? &s->err : nullptr, CPM_E_INVALID, "cpm_sim_step_host: null pointer");
  if (!s->side) {
    SIM_CU(s, cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking));
    SIM_CU(s, cudaEventCreateWithFlags(&s->ev_sorted, cudaEventDisableTiming));
  }
  SIM_CU(s, ensure(s->host_tmp_x, 3 * s->n * sizeof(float)));
  int rc = upload_caller_order(s, x3, as<float>(s->x));
  if (!rc && fixed_point(s)) launch_to_fixed(as<float>(s->x), as<uint32_t>(s->q), s->n, s->box, s->stream);
  if (!rc) rc = upload_caller_order(s, p3, as<float>(s->p));
  if (!rc) {
    s->x_out = x3;
    s->direct_step = true;
    rc = cpm_sim_step_to(s, a1);
    s->direct_step = false;
    if (s->x_out) {  // the step ended before its sort
      s->x_out = nullptr;
      if (!rc) rc = download_caller_order(s, as<float>(s->x), x3);
    }
  }
  if (!rc) rc = download_caller_order(s, as<float>(s->p), p3);
  const cudaError_t e = cudaStreamSynchronize(s->side);
  if (rc) return rc;
  if (e != cudaSuccess) return set_error(&s->err, CPM_E_CUDA, std::string("position copy: ") + cudaGetErrorString(e));
  return sim_check(s);
}

int cpm_sim_get_state(cpm_sim* s, float* x3, float* p3, float* acc3, float* delta, float* a) {
  if (!s) return set_error(nullptr, CPM_E_INVALID, "cpm_sim_get_state: sim is NULL");
  const size_t n = s->n;
  const float* srcs[3] = {as<float>(s->x), as<float>(s->p), as<float>(s->acc)};
  float* dsts[3] = {x3, p3, acc3};
  for (int q = 0; q < 3; ++q) {
    if (!dsts[q]) continue;
    launch_scatter3(srcs[q], as<uint32_t>(s->id), n, as<float>(s->x2), s->stream);
    SIM_CU(s, cudaMemcpyAsync(dsts[q], s->x2.p, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
  }
  if (delta) {
    const size_t m = mesh_cells(s) * (size_t)s->nb;
    launch_fixed_to_f32(as<unsigned long long>(s->fx), m, s->shift, 1, s->mean, as<float>(s->gx), s->stream);
    SIM_CU(s, cudaMemcpyAsync(delta, s->gx.p, m * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
  }
  if (a) *a = s->a;
  return sim_check(s);
}

int cpm_sim_power_spectrum(cpm_sim* s, int n_shells, double* k_mean, double* p_mean, uint64_t* counts) {
  if (!s) return set_error(nullptr, CPM_E_INVALID, "cpm_sim_power_spectrum: sim is NULL");
  if (!k_mean || !p_mean || !counts) return set_error(&s->err, CPM_E_INVALID, "cpm_sim_power_spectrum: null pointer");
  if (n_shells < 1 || n_shells > PK_MAX_SHELLS)
    return set_error(&s->err, CPM_E_INVALID, "cpm_sim_power_spectrum: n_shells must be in [1, 2048]");
  if (s->nb > 1) return set_error(&s->err, CPM_E_INVALID, "cpm_sim_power_spectrum: a batch (use the ensemble's)");
  const int mn = s->P.mesh_n;
  // The deposit of the current positions (the mesh of the last force evaluation may predate a
  // set_state); the next step deposits again before it uses the mesh.
  launch_deposit_fixed(as<float>(s->x), s->n, 1.0f, mn, s->h, s->shift, as<unsigned long long>(s->fx), s->stream);
  launch_r2c3(s->plan, nullptr, as<unsigned long long>(s->fx), s->shift, s->mean, as<float2>(s->spec), s->stream);
  SIM_CU(s, ensure(s->pk, sizeof(PkSums)));
  launch_pk_bin(as<float2>(s->spec), mn, n_shells, as<PkSums>(s->pk), s->stream);
  std::vector<PkSums> host(1);
  SIM_CU(s, cudaMemcpyAsync(host.data(), s->pk.p, sizeof(PkSums), cudaMemcpyDeviceToHost, s->stream));
  int rc = sim_check(s);
  if (rc) return rc;
  pk_finish(host[0], mn, s->box, n_shells, k_mean, p_mean, counts);
  return CPM_OK;
}

int cpm_sim_snapshot(cpm_sim* s, float* speeds, float* densities, float* rsd3, float* grid, int* grid_n,
                     float* max_speed) {
  if (!s) return set_error(nullptr, CPM_E_INVALID, "cpm_sim_snapshot: sim is NULL");
  if (s->nb > 1) return set_error(&s->err, CPM_E_INVALID, "cpm_sim_snapshot: not for a batch of boxes");
  const size_t n = s->n;
  const int mn = s->P.mesh_n;
  const size_t m3 = (size_t)mn * mn * mn;
  const int gm = density_grid_side(mn);
  const size_t gm3 = (size_t)gm * gm * gm;
  SIM_CU(s, ensure(s->snap, (5 * n + gm3 + 1) * sizeof(float)));
  float* base = as<float>(s->snap);
  float *d_speeds = base, *d_dens = base + n, *d_rsd = base + 2 * n, *d_grid = base + 5 * n;
  unsigned int* d_max = reinterpret_cast<unsigned int*>(base + 5 * n + gm3);
  if (densities || grid)  // delta of the last force evaluation (integrator.rs:117-126)
    launch_fixed_to_f32(as<unsigned long long>(s->fx), m3, s->shift, 1, s->mean, as<float>(s->gx), s->stream);
  if (densities) launch_interpolate(as<float>(s->gx), as<float>(s->x), n, mn, s->h, as<float>(s->x2), s->stream);
  SIM_CU(s, cudaMemsetAsync(d_max, 0, sizeof(unsigned int), s->stream));
  const float a = s->a;
  const float e = cosmo_e(s->P.cosmo, a);
  const float rsd_scale = 1.0f / (a * a * e);  // frame.rs:66
  launch_snapshot_particles(as<float>(s->p), densities ? as<float>(s->x2) : nullptr, as<uint32_t>(s->id), n, a,
                            rsd_scale, speeds ? d_speeds : nullptr, densities ? d_dens : nullptr,
                            rsd3 ? d_rsd : nullptr, d_max, s->stream);
  if (grid) launch_downsample_grid(as<float>(s->gx), mn, d_grid, s->stream);
  if (speeds) SIM_CU(s, cudaMemcpyAsync(speeds, d_speeds, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
  if (densities) SIM_CU(s, cudaMemcpyAsync(densities, d_dens, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
  if (rsd3) SIM_CU(s, cudaMemcpyAsync(rsd3, d_rsd, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
  if (grid) SIM_CU(s, cudaMemcpyAsync(grid, d_grid, gm3 * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
  unsigned int bits = 0;
  SIM_CU(s, cudaMemcpyAsync(&bits, d_max, sizeof(bits), cudaMemcpyDeviceToHost, s->stream));
  const int rc = sim_check(s);
  if (rc) return rc;
  if (grid_n) *grid_n = gm;
  if (max_speed) std::memcpy(max_speed, &bits, sizeof(float));
  return CPM_OK;
}

int cpm_sim_phase_times(cpm_sim* s, double* ms8, uint64_t* steps, int reset) {
  if (!s) return set_error(nullptr, CPM_E_INVALID, "cpm_sim_phase_times: sim is NULL");
  int rc = flush_timing(s);
  if (rc) return rc;
  if (ms8)
    for (int i = 0; i < N_PHASES; ++i) ms8[i] = s->timed_steps ? s->phase_ms[i] / (double)s->timed_steps : 0.0;
  if (steps) *steps = s->timed_steps;
  if (reset) {
    for (double& v : s->phase_ms) v = 0.0;
    s->timed_steps = 0;
  }
  return CPM_OK;
}

int cpm_sim_walk_candidates(cpm_sim* s, uint64_t* candidates) {
  if (!s || !candidates) return set_error(nullptr, CPM_E_INVALID, "cpm_sim_walk_candidates: null pointer");
  SIM_CU(s, cudaStreamSynchronize(s->stream));
  unsigned long long tc[4] = {0, 0, 0, 0};
  SIM_CU(s, cudaMemcpy(tc, s->counters.p, sizeof(tc), cudaMemcpyDeviceToHost));
  *candidates = tc[2];
  return CPM_OK;
}

int cpm_sim_counters(cpm_sim* s, uint64_t* nodes, uint64_t* leaf_pairs, uint64_t* node_accepts,
                     uint32_t* launches_per_step) {
  if (!s) return set_error(nullptr, CPM_E_INVALID, "cpm_sim_counters: sim is NULL");
  SIM_CU(s, cudaStreamSynchronize(s->stream));
  unsigned long long tc[4] = {0, 0, 0, 0};
  SIM_CU(s, cudaMemcpy(tc, s->counters.p, sizeof(tc), cudaMemcpyDeviceToHost));
  uint64_t nn = 0;
  if (s->tree.counters.p) {
    uint32_t cnt[64];
    SIM_CU(s, cudaMemcpy(cnt, s->tree.counters.p, sizeof(cnt), cudaMemcpyDeviceToHost));
    for (int d = 0; d <= KEY_LEVELS; ++d) nn += cnt[d];
  }
  if (nodes) *nodes = nn;
  if (leaf_pairs) *leaf_pairs = tc[0];
  if (node_accepts) *node_accepts = tc[1];
  if (launches_per_step) *launches_per_step = s->launches;
  return CPM_OK;
}

int cpm_sim_tree_depth(cpm_sim* s, uint32_t* max_depth, uint64_t* key_depth_leaves) {
  if (!s) return set_error(nullptr, CPM_E_INVALID, "cpm_sim_tree_depth: sim is NULL");
  SIM_CU(s, cudaStreamSynchronize(s->stream));
  uint32_t cnt[64] = {};
  if (s->tree.counters.p) SIM_CU(s, cudaMemcpy(cnt, s->tree.counters.p, sizeof(cnt), cudaMemcpyDeviceToHost));
  if (max_depth) *max_depth = cnt[33];         // deepest level that split
  if (key_depth_leaves) *key_depth_leaves = cnt[32];  // nodes kept as leaves at the key depth
  return CPM_OK;
}

// State file: a 128-byte little-endian header, then x[n][3] and p[n][3] (f32, caller order).
//   0  char[8]  "CPMSTATE"        8 u32 version (1)       12 u32 flags (CPM_SIM_*)
//  16  u64 n_particles            24 f32 a                28 f32 box_size
//  32  i32 mesh_n                 36 i32 use_tree         40 f32 omega_r, omega_m, omega_l, h0
//  56  f32 r_split, r_cut, softening, theta               72 u64 payload bytes (24 n)
//  80  u64 FNV-1a 64 hash of the payload                  88 .. 127 zero
namespace {
constexpr size_t STATE_HEADER = 128;

uint64_t fnv1a64(const unsigned char* p, size_t len, uint64_t h) {
  for (size_t i = 0; i < len; ++i) {
    h ^= p[i];
    h *= 0x100000001B3ull;
  }
  return h;
}
}  // namespace

int cpm_sim_save(cpm_sim* s, const char* path) {
  if (!s || !path) return set_error(s ? &s->err : nullptr, CPM_E_INVALID, "cpm_sim_save: null pointer");
  const size_t n = s->n;
  std::vector<float> xp(6 * n);
  float a = 0.0f;
  int rc = cpm_sim_get_state(s, xp.data(), xp.data() + 3 * n, nullptr, nullptr, &a);
  if (rc) return rc;
  unsigned char hdr[STATE_HEADER] = {};
  const uint32_t version = 1, flags = s->P.flags;
  const uint64_t nn = n, payload = 24 * (uint64_t)n;
  const int32_t mesh = s->P.mesh_n, use_tree = s->P.use_tree;
  const float cosmo[4] = {s->P.cosmo.omega_r, s->P.cosmo.omega_m, s->P.cosmo.omega_l, s->P.cosmo.h0};
  const float split[4] = {s->P.split.r_split, s->P.split.r_cut, s->P.split.softening, s->P.split.theta};
  const uint64_t hash = fnv1a64(reinterpret_cast<const unsigned char*>(xp.data()), payload, 0xCBF29CE484222325ull);
  std::memcpy(hdr, "CPMSTATE", 8);
  std::memcpy(hdr + 8, &version, 4);
  std::memcpy(hdr + 12, &flags, 4);
  std::memcpy(hdr + 16, &nn, 8);
  std::memcpy(hdr + 24, &a, 4);
  std::memcpy(hdr + 28, &s->P.box_size, 4);
  std::memcpy(hdr + 32, &mesh, 4);
  std::memcpy(hdr + 36, &use_tree, 4);
  std::memcpy(hdr + 40, cosmo, 16);
  std::memcpy(hdr + 56, split, 16);
  std::memcpy(hdr + 72, &payload, 8);
  std::memcpy(hdr + 80, &hash, 8);
  FILE* f = std::fopen(path, "wb");
  if (!f) return set_error(&s->err, CPM_E_INVALID, std::string("cpm_sim_save: cannot open ") + path);
  const bool ok = std::fwrite(hdr, 1, STATE_HEADER, f) == STATE_HEADER &&
                  std::fwrite(xp.data(), 1, payload, f) == payload;
  const bool closed = std::fclose(f) == 0;
  if (!ok || !closed) return set_error(&s->err, CPM_E_INVALID, std::string("cpm_sim_save: write failed: ") + path);
  return CPM_OK;
}

int cpm_sim_load(const char* path, uint32_t extra_flags, cpm_sim** out) {
  if (!path || !out) return set_error(nullptr, CPM_E_INVALID, "cpm_sim_load: null pointer");
  *out = nullptr;
  FILE* f = std::fopen(path, "rb");
  if (!f) return set_error(nullptr, CPM_E_INVALID, std::string("cpm_sim_load: cannot open ") + path);
  unsigned char hdr[STATE_HEADER];
  if (std::fread(hdr, 1, STATE_HEADER, f) != STATE_HEADER || std::memcmp(hdr, "CPMSTATE", 8) != 0) {
    std::fclose(f);
    return set_error(nullptr, CPM_E_INVALID, std::string("cpm_sim_load: not a state file: ") + path);
  }
  uint32_t version, flags;
  uint64_t nn, payload, hash;
  float a, box, cosmo[4], split[4];
  int32_t mesh, use_tree;
  std::memcpy(&version, hdr + 8, 4);
  std::memcpy(&flags, hdr + 12, 4);
  std::memcpy(&nn, hdr + 16, 8);
  std::memcpy(&a, hdr + 24, 4);
  std::memcpy(&box, hdr + 28, 4);
  std::memcpy(&mesh, hdr + 32, 4);
  std::memcpy(&use_tree, hdr + 36, 4);
  std::memcpy(cosmo, hdr + 40, 16);
  std::memcpy(split, hdr + 56, 16);
  std::memcpy(&payload, hdr + 72, 8);
  std::memcpy(&hash, hdr + 80, 8);
  if (version != 1 || nn == 0 || nn > 0x7FFFFFFFull || payload != 24 * nn) {
    std::fclose(f);
    return set_error(nullptr, CPM_E_INVALID, std::string("cpm_sim_load: unsupported or corrupt header: ") + path);
  }
  std::vector<float> xp(6 * nn);
  const bool ok = std::fread(xp.data(), 1, payload, f) == payload;
  std::fclose(f);
  if (!ok || fnv1a64(reinterpret_cast<const unsigned char*>(xp.data()), payload, 0xCBF29CE484222325ull) != hash)
    return set_error(nullptr, CPM_E_INVALID, std::string("cpm_sim_load: truncated or corrupt payload: ") + path);
  cpm_sim_params P{};
  P.cosmo = cpm_cosmology{cosmo[0], cosmo[1], cosmo[2], cosmo[3]};
  P.box_size = box;
  P.mesh_n = mesh;
  P.n_particles = nn;
  P.use_tree = use_tree;
  P.split = cpm_force_split{split[0], split[1], split[2], split[3]};
  P.flags = flags | extra_flags;
  return cpm_sim_create(&P, xp.data(), xp.data() + 3 * nn, a, out);
}

int cpm_step_factors(const cpm_cosmology* c, double a0, double a1, int fp64, double* k1, double* d, double* k2) {
  if (!c || !k1 || !d || !k2) return set_error(nullptr, CPM_E_INVALID, "cpm_step_factors: null pointer");
  if (!(a0 > 0.0) || !(a1 > 0.0)) return set_error(nullptr, CPM_E_INVALID, "cpm_step_factors: a0, a1 must be > 0");
  if (!fp64) {  // the reference's f32 arithmetic on the host
    const float fa0 = (float)a0, fa1 = (float)a1;
    const float am = midpoint(*c, fa0, fa1);
    *k1 = kick_factor(*c, fa0, am);
    *d = drift_factor(*c, fa0, fa1);
    *k2 = kick_factor(*c, am, fa1);
    return CPM_OK;
  }
  int rc = check_device_once(nullptr);
  if (rc) return rc;
  DevBuf b;
  cudaError_t e = ensure(b, sizeof(StepScalars));
  if (e == cudaSuccess) {
    launch_step_factors64(as<StepScalars>(b), *c, a0, a1, 1.0, 1.0, 1.0, nullptr);
    StepScalars v{};
    e = cudaMemcpy(&v, b.p, sizeof(v), cudaMemcpyDeviceToHost);
    *k1 = v.k1;
    *d = v.d64;
    *k2 = v.k2;
  }
  release(b);
  if (e != cudaSuccess) return set_error(nullptr, CPM_E_CUDA, std::string("cpm_step_factors: ") + cudaGetErrorString(e));
  return CPM_OK;
}

int cpm_sim_set_learned(cpm_sim* s, cpm_net* net, float delta_threshold, float in_scale) {
  if (!s) return set_error(nullptr, CPM_E_INVALID, "cpm_sim_set_learned: sim is NULL");
  if (net && net_mesh(net) != s->P.mesh_n)
    return set_error(&s->err, CPM_E_MESH_MISMATCH, "cpm_sim_set_learned: the net's mesh differs from the simulation's");
  if (net && !s->P.use_tree)
    return set_error(&s->err, CPM_E_INVALID, "cpm_sim_set_learned: a pure PM simulation has no short-range force");
  if (net && s->nb > 1) return set_error(&s->err, CPM_E_INVALID, "cpm_sim_set_learned: not for a batch of boxes");
  if (net && (!std::isfinite(delta_threshold) || !(in_scale > 0.0f) || !std::isfinite(in_scale)))
    return set_error(&s->err, CPM_E_INVALID, "cpm_sim_set_learned: threshold must be finite and in_scale > 0");
  if (net) {
    for (DevBuf* b : {&s->flag, &s->offset, &s->list}) SIM_CU(s, ensure(*b, s->n * sizeof(uint32_t)));
    SIM_CU(s, ensure(s->list_n, sizeof(uint32_t)));
    SIM_CU(s, cudaMemsetAsync(s->list_n.p, 0, sizeof(uint32_t), s->stream));
  }
  SIM_CU(s, cudaStreamSynchronize(s->stream));
  // the captured step graphs hold the previous force assembly: capture again
  for (int q = 0; q < 2; ++q) {
    if (s->graph[q]) cudaGraphExecDestroy(s->graph[q]);
    s->graph[q] = nullptr;
    s->warm[q] = false;
    s->no_graph[q] = false;
  }
  s->net = net;
  s->net_threshold = delta_threshold;
  s->net_in_scale = in_scale;
  return CPM_OK;
}

int cpm_sim_short_range(cpm_sim* s, float* sr3) {
  if (!s || !sr3) return set_error(s ? &s->err : nullptr, CPM_E_INVALID, "cpm_sim_short_range: null pointer");
  if (!s->P.use_tree || !s->tree.geo.p)
    return set_error(&s->err, CPM_E_INVALID, "cpm_sim_short_range: the simulation has no tree");
  const size_t n = s->n;
  SIM_CU(s, ensure(s->host_tmp, 3 * n * sizeof(float)));
  // the tree of the last force evaluation was built on the current positions (the kick that ends a
  // step changes the momenta only)
  const float k = tree_coupling(s->P.cosmo.omega_m, s->box, s->a, per_box(s));
  launch_tree_walk(s->tree, as<float>(s->x), n, s->box, s->P.split, k, as<float>(s->host_tmp), 0, nullptr,
                   as<DevStatus>(s->status), s->stream);
  launch_scatter3(as<float>(s->host_tmp), as<uint32_t>(s->id), n, as<float>(s->x2), s->stream);
  SIM_CU(s, cudaMemcpyAsync(sr3, s->x2.p, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
  return sim_check(s);
}

int cpm_sim_autotune_report(cpm_sim* s, int* fft_radix, int* deposit_tile, int* walk_warps, float* ms9) {
  if (!s) return set_error(nullptr, CPM_E_INVALID, "cpm_sim_autotune_report: sim is NULL");
  if (fft_radix) *fft_radix = s->plan.max_radix;
  if (deposit_tile) *deposit_tile = 256 * s->dep_ppt;
  if (walk_warps) *walk_warps = s->tree.walk_warps;
  if (ms9)
    for (int i = 0; i < N_TUNE; ++i) ms9[i] = s->tune_ms[i];
  return CPM_OK;
}

int cpm_sim_set_tuning(cpm_sim* s, int fft_radix, int deposit_tile, int walk_warps) {
  if (!s) return set_error(nullptr, CPM_E_INVALID, "cpm_sim_set_tuning: sim is NULL");
  if ((fft_radix != 0 && fft_radix != 4 && fft_radix != 8) ||
      (deposit_tile != 512 && deposit_tile != 1024 && deposit_tile != 2048) ||
      (walk_warps != 2 && walk_warps != 4 && walk_warps != 8))
    return set_error(&s->err, CPM_E_INVALID,
                     "cpm_sim_set_tuning: FFT plan 8, 4 or 0, tile 512, 1024 or 2048, warps 2, 4 or 8");
  SIM_CU(s, cudaStreamSynchronize(s->stream));
  s->plan.max_radix = fft_radix;
  s->dep_ppt = deposit_tile / 256;
  s->tree.walk_warps = walk_warps;
  s->tuned = true;
  for (int q = 0; q < 2; ++q) {  // the captured graphs hold the old launches
    if (s->graph[q]) cudaGraphExecDestroy(s->graph[q]);
    s->graph[q] = nullptr;
    s->warm[q] = false;
    s->no_graph[q] = false;
  }
  return CPM_OK;
}

int cpm_sim_learned_walked(cpm_sim* s, uint64_t* walked) {
  if (!s || !walked) return set_error(nullptr, CPM_E_INVALID, "cpm_sim_learned_walked: null pointer");
  SIM_CU(s, cudaStreamSynchronize(s->stream));
  uint32_t v = 0;
  if (s->net && s->list_n.p) SIM_CU(s, cudaMemcpy(&v, s->list_n.p, sizeof(v), cudaMemcpyDeviceToHost));
  *walked = s->net ? (uint64_t)v : (uint64_t)s->n;
  return CPM_OK;
}

void* cpm_sim_stream(cpm_sim* s) { return s ? (void*)s->stream : nullptr; }

int cpm_sim_graphs(cpm_sim* s) { return s ? (s->graph[0] ? 1 : 0) + (s->graph[1] ? 1 : 0) : 0; }

int cpm_sim_destroy(cpm_sim* s) {
  if (!s) return CPM_OK;
  if (s->stream) cudaStreamSynchronize(s->stream);
  if (s->side) cudaStreamSynchronize(s->side);
  fft_plan_free(s->plan);
  for (DevBuf* b : {&s->sort.keys_alt, &s->sort.vals_alt, &s->sort.block_hist, &s->sort.scan_tmp, &s->tree.geo,
                    &s->tree.mass, &s->tree.link, &s->tree.counters, &s->tree.prefix, &s->tree.scan_tmp, &s->tree.x4, &s->tree.quad, &s->x, &s->p,
                    &s->acc, &s->id, &s->x2, &s->p2, &s->id2, &s->keys, &s->vals, &s->fx, &s->gx, &s->gy, &s->gz,
                    &s->spec, &s->status, &s->counters, &s->pk, &s->q, &s->q2, &s->snap, &s->flag, &s->offset,
                    &s->list, &s->list_n, &s->scan_tmp, &s->okeys, &s->okeys_sorted})
    release(*b);
  tree_walk_free(s->tree);
  release(s->host_tmp);
  release(s->host_tmp_x);
  release(s->stepv);
  for (cudaGraphExec_t& g : s->graph)
    if (g) cudaGraphExecDestroy(g);
  for (auto& row : s->ev)
    for (auto& e : row)
      if (e) cudaEventDestroy(e);
  if (s->stream) cudaStreamDestroy(s->stream);
  if (s->side) cudaStreamDestroy(s->side);
  if (s->ev_sorted) cudaEventDestroy(s->ev_sorted);
  delete s;
  return CPM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Ensemble: many independent realisations of uneven sizes (no counterpart in the reference, which
// runs one realisation per run, runner.rs:228-260). Each size class is one batched simulation
// (its boxes share every launch: keys, sort, deposit, the batched FFT passes, gather, tree build
// with one root per box, walk), and a step of the whole ensemble is one CUDA graph: the classes
// run as parallel branches forked from the ensemble's stream and joined back.
// ---------------------------------------------------------------------------------------------
struct cpm_ensemble {
  std::vector<cpm_sim*> classes;
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t graph[2] = {};
  bool warm[2] = {false, false};
  bool no_graph[2] = {false, false};
  std::string err;
  float a = 0.0f;
};

namespace {

// Forks every class off the ensemble's stream, runs its step body on its own stream, joins back.
int ensemble_branches(cpm_ensemble* e, float a1) {
  cudaError_t ce = cudaEventRecord(e->fork, e->stream);
  for (size_t c = 0; c < e->classes.size() && ce == cudaSuccess; ++c) {
    cpm_sim* s = e->classes[c];
    ce = cudaStreamWaitEvent(s->stream, e->fork, 0);
    if (ce != cudaSuccess) break;
    const int rc = step_body(s, a1);
    if (rc) {
      e->err = s->err;
      return rc;
    }
    ce = cudaEventRecord(e->join[c], s->stream);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(e->stream, e->join[c], 0);
  }
  if (ce != cudaSuccess) return set_error(&e->err, CPM_E_CUDA, std::string("ensemble step: ") + cudaGetErrorString(ce));
  return CPM_OK;
}

}  // namespace

extern "C" {

int cpm_ensemble_destroy(cpm_ensemble* e) {
  if (!e) return CPM_OK;
  if (e->stream) cudaStreamSynchronize(e->stream);
  for (cudaGraphExec_t& g : e->graph)
    if (g) cudaGraphExecDestroy(g);
  for (cpm_sim* s : e->classes) cpm_sim_destroy(s);
  for (cudaEvent_t ev : e->join)
    if (ev) cudaEventDestroy(ev);
  if (e->fork) cudaEventDestroy(e->fork);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
  return CPM_OK;
}

int cpm_ensemble_create(const cpm_cosmology* cosmo, float box_size, float n_s, float sigma8, float a0, int n_classes,
                        const cpm_ensemble_class* classes, uint32_t flags, cpm_ensemble** out) {
  if (!out) return set_error(nullptr, CPM_E_INVALID, "cpm_ensemble_create: out is NULL");
  *out = nullptr;
  if (!cosmo || !classes || n_classes < 1 || n_classes > 16)
    return set_error(nullptr, CPM_E_INVALID, "cpm_ensemble_create: 1..16 classes and a cosmology are required");
  if (!(box_size > 0.0f) || !(a0 > 0.0f) || !(sigma8 > 0.0f))
    return set_error(nullptr, CPM_E_INVALID, "cpm_ensemble_create: box, a0 and sigma8 must be > 0");
  if (flags & (CPM_SIM_TIMING | CPM_SIM_QUADRUPOLE))
    return set_error(nullptr, CPM_E_INVALID, "cpm_ensemble_create: CPM_SIM_TIMING and CPM_SIM_QUADRUPOLE are per simulation");
  for (int c = 0; c < n_classes; ++c) {
    const cpm_ensemble_class& k = classes[c];
    const size_t nbox = (size_t)k.n_side * k.n_side * k.n_side;
    if (!fft_supported(k.n_side) || k.n_boxes < 1 || k.n_boxes > 64 || nbox % 2048 != 0 || k.mesh_n > 512 ||
        !poisson_supported(k.mesh_n))
      return set_error(nullptr, CPM_E_INVALID,
                       "cpm_ensemble_create: class " + std::to_string(c) +
                           ": 1..64 boxes, n_side a supported FFT length with n_side^3 a multiple of 2048, "
                           "mesh a supported length up to 512");
  }
  int rc = check_device_once(nullptr);
  if (rc) return rc;
  cpm_ensemble* e = new cpm_ensemble();
  e->a = a0;
  auto fail = [&](int code, const std::string& msg) {
    set_error(nullptr, code, msg);
    cpm_ensemble_destroy(e);
    return code;
  };
  if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) != cudaSuccess)
    return fail(CPM_E_CUDA, "cpm_ensemble_create: stream or event creation failed");
  e->join.assign((size_t)n_classes, nullptr);
  for (auto& ev : e->join)
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
      return fail(CPM_E_CUDA, "cpm_ensemble_create: event creation failed");
  for (int c = 0; c < n_classes; ++c) {
    const cpm_ensemble_class& k = classes[c];
    cpm_sim_params P{};
    P.cosmo = *cosmo;
    P.box_size = box_size;
    P.mesh_n = k.mesh_n;
    P.n_particles = (size_t)k.n_side * k.n_side * k.n_side;
    P.use_tree = 1;
    P.split = k.split;
    P.flags = flags;
    cpm_sim* s = nullptr;
    rc = sim_new(&P, a0, &s, k.n_boxes);
    if (rc) return fail(rc, g_last_error);
    e->classes.push_back(s);
    // ics.rs:119-182 for every box of the class, seeds first_seed + b, into the box's slice
    DevBuf modes, work;
    FftPlan plan;
    cudaError_t ce = cudaSuccess;
    for (int b = 0; b < k.n_boxes && ce == cudaSuccess; ++b)
      ce = generate_zeldovich(k.n_side, box_size, *cosmo, n_s, sigma8, a0, k.first_seed + (uint64_t)b,
                              as<float>(s->x) + 3 * P.n_particles * (size_t)b,
                              as<float>(s->p) + 3 * P.n_particles * (size_t)b, modes, work, plan, s->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s->stream);
    release(modes);
    release(work);
    fft_plan_free(plan);
    if (ce != cudaSuccess)
      return fail(ce == cudaErrorMemoryAllocation ? CPM_E_NOMEM : CPM_E_CUDA,
                  std::string("cpm_ensemble_create: initial conditions: ") + cudaGetErrorString(ce));
    launch_iota(as<uint32_t>(s->id), s->n, s->stream);
    if (fixed_point(s)) launch_to_fixed(as<float>(s->x), as<uint32_t>(s->q), s->n, s->box, s->stream);
    rc = sim_accelerations(s, s->a);
    if (rc == CPM_OK) rc = sim_check(s);
    if (rc == CPM_OK) rc = sim_autotune(s);
    if (rc) return fail(rc, s->err);
  }
  *out = e;
  return CPM_OK;
}

int cpm_ensemble_step_to(cpm_ensemble* e, float a1) {
  if (!e) return set_error(nullptr, CPM_E_INVALID, "cpm_ensemble_step_to: ensemble is NULL");
  if (!(a1 > 0.0f) || !std::isfinite(a1)) return set_error(&e->err, CPM_E_INVALID, "cpm_ensemble_step_to: a1 must be > 0");
  // every class's step scalars, on the ensemble's stream ahead of the branches
  for (cpm_sim* s : e->classes) sim_write_step_scalars(s, a1, e->stream);
  const int q = e->classes[0]->parity;  // the classes' sorted buffers alternate together
  const bool graphs = !(e->classes[0]->P.flags & CPM_SIM_NO_GRAPH) && e->warm[q] && !e->no_graph[q];
  int rc = CPM_OK;
  if (graphs && e->graph[q]) {
    const cudaError_t ce = cudaGraphLaunch(e->graph[q], e->stream);
    if (ce != cudaSuccess) return set_error(&e->err, CPM_E_CUDA, std::string("cudaGraphLaunch: ") + cudaGetErrorString(ce));
    for (cpm_sim* s : e->classes) swap_sorted(s);  // the host side of the replayed sorts
  } else if (graphs) {
    cudaError_t ce = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal);
    rc = ce == cudaSuccess ? ensemble_branches(e, a1) : CPM_E_CUDA;
    cudaGraph_t g = nullptr;
    if (ce == cudaSuccess) ce = cudaStreamEndCapture(e->stream, &g);
    if (rc == CPM_OK && ce == cudaSuccess && g) ce = cudaGraphInstantiate(&e->graph[q], g, 0);
    if (g) cudaGraphDestroy(g);
    if (rc != CPM_OK || ce != cudaSuccess || !e->graph[q]) {
      // capture failed: undo the host-side swaps of the captured step and run it directly
      cudaGetLastError();
      if (e->graph[q]) cudaGraphExecDestroy(e->graph[q]);
      e->graph[q] = nullptr;
      e->no_graph[q] = true;
      for (cpm_sim* s : e->classes)
        if (s->parity != q) swap_sorted(s);
      rc = ensemble_branches(e, a1);
    } else {
      ce = cudaGraphLaunch(e->graph[q], e->stream);
      if (ce != cudaSuccess)
        return set_error(&e->err, CPM_E_CUDA, std::string("cudaGraphLaunch: ") + cudaGetErrorString(ce));
    }
  } else {
    rc = ensemble_branches(e, a1);
    e->warm[q] = true;
  }
  if (rc) return rc;
  for (cpm_sim* s : e->classes) s->a = a1;
  e->a = a1;
  return CPM_OK;
}

int cpm_ensemble_get_state(cpm_ensemble* e, int cls, int box, float* x3, float* p3, float* acc3) {
  if (!e || cls < 0 || cls >= (int)e->classes.size())
    return set_error(e ? &e->err : nullptr, CPM_E_INVALID, "cpm_ensemble_get_state: bad ensemble or class");
  cpm_sim* s = e->classes[(size_t)cls];
  if (box < 0 || box >= s->nb) return set_error(&e->err, CPM_E_INVALID, "cpm_ensemble_get_state: bad box");
  SIM_CU(s, cudaStreamSynchronize(e->stream));
  const size_t nb = s->n_box, off = (size_t)box * nb;
  const float* srcs[3] = {as<float>(s->x), as<float>(s->p), as<float>(s->acc)};
  float* dsts[3] = {x3, p3, acc3};
  for (int k = 0; k < 3; ++k) {
    if (!dsts[k]) continue;
    launch_scatter3(srcs[k], as<uint32_t>(s->id), s->n, as<float>(s->x2), s->stream);
    SIM_CU(s, cudaMemcpyAsync(dsts[k], as<float>(s->x2) + 3 * off, 3 * nb * sizeof(float), cudaMemcpyDeviceToHost,
                              s->stream));
  }
  const int rc = sim_check(s);
  if (rc) e->err = s->err;
  return rc;
}

int cpm_ensemble_power_spectrum(cpm_ensemble* e, int cls, int box, int n_shells, double* k_mean, double* p_mean,
                                uint64_t* counts) {
  if (!e || cls < 0 || cls >= (int)e->classes.size() || !k_mean || !p_mean || !counts)
    return set_error(e ? &e->err : nullptr, CPM_E_INVALID, "cpm_ensemble_power_spectrum: bad arguments");
  cpm_sim* s = e->classes[(size_t)cls];
  if (box < 0 || box >= s->nb || n_shells < 1 || n_shells > PK_MAX_SHELLS)
    return set_error(&e->err, CPM_E_INVALID, "cpm_ensemble_power_spectrum: bad box or n_shells");
  SIM_CU(s, cudaStreamSynchronize(e->stream));
  const int mn = s->P.mesh_n;
  launch_deposit_fixed(as<float>(s->x), s->n, 1.0f, mn, s->h, s->shift, as<unsigned long long>(s->fx), s->stream,
                       s->dep_ppt, batch_box(s));
  launch_r2c3(s->plan, nullptr, as<unsigned long long>(s->fx) + mesh_cells(s) * (size_t)box, s->shift, s->mean,
              as<float2>(s->spec), s->stream);
  SIM_CU(s, ensure(s->pk, sizeof(PkSums)));
  launch_pk_bin(as<float2>(s->spec), mn, n_shells, as<PkSums>(s->pk), s->stream);
  std::vector<PkSums> host(1);
  SIM_CU(s, cudaMemcpyAsync(host.data(), s->pk.p, sizeof(PkSums), cudaMemcpyDeviceToHost, s->stream));
  const int rc = sim_check(s);
  if (rc) {
    e->err = s->err;
    return rc;
  }
  pk_finish(host[0], mn, s->box, n_shells, k_mean, p_mean, counts);
  return CPM_OK;
}

int cpm_ensemble_graphs(cpm_ensemble* e) { return e ? (e->graph[0] ? 1 : 0) + (e->graph[1] ? 1 : 0) : 0; }

void* cpm_ensemble_stream(cpm_ensemble* e) { return e ? (void*)e->stream : nullptr; }

const char* cpm_ensemble_last_error(const cpm_ensemble* e) { return e ? e->err.c_str() : g_last_error.c_str(); }

}  // extern "C"
