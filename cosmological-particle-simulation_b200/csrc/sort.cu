// sort.cu — octant keys of the tree descent, stable LSD radix sort of (u64 key, u32 value)
// pairs, and exclusive scans. HBM-bound integer work: coalesced tiles, per-warp ranking with
// ballots, no tensor cores.
#include <algorithm>
#include <atomic>
#include <mutex>
#include <vector>

#include "cpm_host.h"
#include "cpm_internal.cuh"

namespace cpm {

constexpr int HFSM_STATES = 24;  // orientations of a cube: an upper bound on the Hilbert curve's states

static std::atomic<unsigned long long> g_launches{0};
unsigned long long launch_count() { return g_launches.load(std::memory_order_relaxed); }
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

cudaError_t ensure(DevBuf& b, size_t bytes) {
  if (b.p != nullptr && b.bytes >= bytes) return cudaSuccess;
  release(b);
  const size_t want = bytes ? bytes : 16;
  cudaError_t e = cudaMalloc(&b.p, want);
  if (e != cudaSuccess) {
    b.p = nullptr;
    b.bytes = 0;
    return e;
  }
  b.bytes = want;
  return cudaSuccess;
}

void release(DevBuf& b) {
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
}

// ---------------------------------------------------------------------------------------------
// Octant keys: tree.rs:186-250 descent. At depth d the octant is (x>=cx)|(y>=cy)<<1|(z>=cz)<<2
// against the node centre; the child centre is centre +- half/2, in f32. The first digit is the
// most significant. Comparisons and additions only, so the digits are bit-exact.
// ---------------------------------------------------------------------------------------------
// With a batch of boxes (n_box > 0: particle i belongs to box i / n_box, boxes one after another),
// the box index goes above the octant digits (bit `box_shift` up), so sorting keeps every box's
// particles together and in box order.
//
// With hkeys, also the particle's Hilbert key over the same cubes: the octant digits are the bits of
// integer coordinates (digit d holds bit levels-1-d of each axis), which J. Skilling's transform
// of axes to the transposed Hilbert index ("Programming the Hilbert curve", AIP Conf. Proc. 707,
// 381, 2004) maps to a key whose first 3d bits name the same level-d cube as the octant key's:
// sorting by it keeps every octree node's particles contiguous and orders the nodes, and the
// particles, along a Hilbert curve.
template <int BITS>
__host__ __device__ __forceinline__ uint64_t hilbert_from_axes(uint32_t X0, uint32_t X1, uint32_t X2) {
  uint32_t X[3] = {X0, X1, X2};
#pragma unroll
  for (int b = BITS - 1; b >= 1; --b) {  // undo excess work, Q = 2^b
    const uint32_t Q = 1u << b, P = Q - 1;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const uint32_t t = (X[0] ^ X[i]) & P;
      const bool inv = (X[i] & Q) != 0u;
      X[0] ^= inv ? P : t;  // invert the low bits of X[0], or exchange them with X[i]'s
      if (i) X[i] ^= inv ? 0u : t;
    }
  }
  X[1] ^= X[0];  // Gray encode
  X[2] ^= X[1];
  uint32_t t = 0;
#pragma unroll
  for (int b = BITS - 1; b >= 1; --b)
    if (X[2] & (1u << b)) t ^= (1u << b) - 1u;
  X[0] ^= t;
  X[1] ^= t;
  X[2] ^= t;
  uint64_t key = 0;
#pragma unroll
  for (int j = BITS - 1; j >= 0; --j)
    key = (key << 3) | (uint64_t)((((X[0] >> j) & 1u) << 2) | (((X[1] >> j) & 1u) << 1) | ((X[2] >> j) & 1u));
  return key;
}

// The same keys digit by digit: because a key's first 3d bits depend only on the first d octant
// digits, digit d is a function of the octant at depth d and of a state (the orientation of the
// curve in the depth-d cube) that the previous digits determine. The state machine is derived on
// the host from hilbert_from_axes itself (states told apart by the order in which they visit the
// eight octants; each transition read off from a representative prefix) and used only after it
// reproduces the transform on every prefix of up to four digits and on 2^16 random coordinates.
// Entry [state * 8 + octant] = digit | next state << 3.
struct HilbertFsm {
  unsigned char t[HFSM_STATES * 8];
  int start = 0;
  int states = 0;
  int ok = 0;
};

static uint64_t hilbert_host(int bits, uint32_t a0, uint32_t a1, uint32_t a2) {
  return bits == KEY_LEVELS ? hilbert_from_axes<KEY_LEVELS>(a0, a1, a2)
                            : hilbert_from_axes<KEY_LEVELS - 2>(a0, a1, a2);
}

static uint64_t hilbert_fsm_host(const HilbertFsm& f, int bits, uint32_t a0, uint32_t a1, uint32_t a2) {
  uint32_t st = (uint32_t)f.start;
  uint64_t key = 0;
  for (int d = 0; d < bits; ++d) {
    const int j = bits - 1 - d;
    const uint32_t o = ((a0 >> j) & 1u) | (((a1 >> j) & 1u) << 1) | (((a2 >> j) & 1u) << 2);
    const uint32_t e = f.t[st * 8 + o];
    key = (key << 3) | (e & 7u);
    st = e >> 3;
  }
  return key;
}

static HilbertFsm derive_hilbert_fsm(int bits) {
  HilbertFsm f;
  // key of the point whose first digits are `pre` (octants, most significant first), zeros after
  auto key_of = [&](const std::vector<uint32_t>& pre) {
    uint32_t a0 = 0, a1 = 0, a2 = 0;
    for (int d = 0; d < bits; ++d) {
      const uint32_t o = d < (int)pre.size() ? pre[d] : 0u;
      a0 = (a0 << 1) | (o & 1u);
      a1 = (a1 << 1) | ((o >> 1) & 1u);
      a2 = (a2 << 1) | ((o >> 2) & 1u);
    }
    return hilbert_host(bits, a0, a1, a2);
  };
  // the digits of the eight octants below prefix `pre`: the state's signature
  auto order_of = [&](std::vector<uint32_t> pre) {
    const int d = (int)pre.size();
    uint32_t sig = 0;
    pre.push_back(0);
    for (uint32_t o = 0; o < 8; ++o) {
      pre.back() = o;
      sig |= (uint32_t)((key_of(pre) >> (3 * (bits - 1 - d))) & 7u) << (3 * o);
    }
    return sig;
  };
  std::vector<uint32_t> sigs;
  std::vector<std::vector<uint32_t>> reps;
  sigs.push_back(order_of({}));
  reps.push_back({});
  for (size_t q = 0; q < sigs.size(); ++q) {
    if ((int)reps[q].size() + 2 > bits || sigs.size() > (size_t)HFSM_STATES) return f;
    for (uint32_t o = 0; o < 8; ++o) {
      std::vector<uint32_t> child = reps[q];
      child.push_back(o);
      const uint32_t sig = order_of(child);
      size_t id = std::find(sigs.begin(), sigs.end(), sig) - sigs.begin();
      if (id == sigs.size()) {
        if (sigs.size() == (size_t)HFSM_STATES) return f;
        sigs.push_back(sig);
        reps.push_back(child);
      }
      f.t[q * 8 + o] = (unsigned char)(((sigs[q] >> (3 * o)) & 7u) | (id << 3));
    }
  }
  f.states = (int)sigs.size();
  // every prefix of up to four digits (the rest zero), then random coordinates
  for (uint32_t p = 0; p < 4096u; ++p)
    for (int len = 1; len <= 4; ++len) {
      std::vector<uint32_t> pre;
      for (int d = 0; d < len; ++d) pre.push_back((p >> (3 * d)) & 7u);
      uint32_t a0 = 0, a1 = 0, a2 = 0;
      for (int d = 0; d < bits; ++d) {
        const uint32_t o = d < len ? pre[d] : 0u;
        a0 = (a0 << 1) | (o & 1u);
        a1 = (a1 << 1) | ((o >> 1) & 1u);
        a2 = (a2 << 1) | ((o >> 2) & 1u);
      }
      if (hilbert_fsm_host(f, bits, a0, a1, a2) != hilbert_host(bits, a0, a1, a2)) return f;
    }
  uint64_t r = 0x9E3779B97F4A7C15ull;
  const uint32_t mask = (1u << bits) - 1u;
  for (int k = 0; k < (1 << 16); ++k) {
    r ^= r << 13;
    r ^= r >> 7;
    r ^= r << 17;
    const uint32_t a0 = (uint32_t)r & mask, a1 = (uint32_t)(r >> 21) & mask, a2 = (uint32_t)(r >> 42) & mask;
    if (hilbert_fsm_host(f, bits, a0, a1, a2) != hilbert_host(bits, a0, a1, a2)) return f;
  }
  f.ok = 1;
  return f;
}

// The state machines of the two key depths in use (21 digits; 19 under a batch of boxes), derived once.
static const HilbertFsm& hilbert_fsm(int bits) {
  static std::once_flag once;
  static HilbertFsm f21, f19;
  std::call_once(once, [] {
    f21 = derive_hilbert_fsm(KEY_LEVELS);
    f19 = derive_hilbert_fsm(KEY_LEVELS - 2);
  });
  return bits == KEY_LEVELS ? f21 : f19;
}

__global__ void k_octant_keys(const float* __restrict__ x3, size_t n, float half0, int levels,
                              uint64_t* __restrict__ keys, uint32_t* __restrict__ vals, DevStatus* st,
                              size_t n_box, int box_shift, uint64_t* __restrict__ hkeys, HilbertFsm fsm) {
  __shared__ unsigned char table[HFSM_STATES * 8];
  const bool use_fsm = hkeys && fsm.ok;
  if (use_fsm) {
    for (int j = threadIdx.x; j < HFSM_STATES * 8; j += blockDim.x) table[j] = fsm.t[j];
    __syncthreads();
  }
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float p0 = x3[3 * i], p1 = x3[3 * i + 1], p2 = x3[3 * i + 2];
  if (!(isfinite(p0) && isfinite(p1) && isfinite(p2))) dev_fail(st, DEV_NONFINITE, (int)i);
  float half = half0, c0 = half0, c1 = half0, c2 = half0;
  uint64_t key = 0, hkey = 0;
  uint32_t a0 = 0, a1 = 0, a2 = 0;  // the digits' bits per axis
  uint32_t state = (uint32_t)fsm.start;
  for (int d = 0; d < levels; ++d) {
    const uint32_t o = (uint32_t)(p0 >= c0) | ((uint32_t)(p1 >= c1) << 1) | ((uint32_t)(p2 >= c2) << 2);
    key = (key << 3) | o;
    if (use_fsm) {
      const uint32_t e = table[state * 8 + o];
      hkey = (hkey << 3) | (e & 7u);
      state = e >> 3;
    } else {
      a0 = (a0 << 1) | (o & 1u);
      a1 = (a1 << 1) | ((o >> 1) & 1u);
      a2 = (a2 << 1) | ((o >> 2) & 1u);
    }
    const float q = half * 0.5f;  // == half / 2.0 exactly
    c0 = __fadd_rn(c0, (o & 1u) ? q : -q);
    c1 = __fadd_rn(c1, (o & 2u) ? q : -q);
    c2 = __fadd_rn(c2, (o & 4u) ? q : -q);
    half = q;
  }
  const uint64_t boxbits = n_box ? (uint64_t)(i / n_box) << box_shift : 0ull;
  keys[i] = key | boxbits;
  if (hkeys) {
    const uint64_t h = use_fsm ? hkey
                               : (levels == KEY_LEVELS ? hilbert_from_axes<KEY_LEVELS>(a0, a1, a2)
                                                       : hilbert_from_axes<KEY_LEVELS - 2>(a0, a1, a2));
    hkeys[i] = h | boxbits;
  }
  if (vals) vals[i] = (uint32_t)i;
}

void launch_octant_keys(const float* x3, size_t n, float box, int levels, uint64_t* keys, uint32_t* vals,
                        DevStatus* st, cudaStream_t s, size_t n_box, uint64_t* hkeys) {
  if (n == 0) return;
  const int T = 256;
  count_launch();
  HilbertFsm fsm;  // ok = 0: the direct transform
  if (hkeys && (levels == KEY_LEVELS || levels == KEY_LEVELS - 2)) fsm = hilbert_fsm(levels);
  k_octant_keys<<<(unsigned)((n + T - 1) / T), T, 0, s>>>(x3, n, box / 2.0f, levels, keys, vals, st, n_box,
                                                          3 * levels, hkeys, fsm);
}

__global__ void k_permute_u64(const uint64_t* __restrict__ in, const uint32_t* __restrict__ perm, size_t n,
                              uint64_t* __restrict__ out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = in[perm[i]];
}

void launch_permute_u64(const uint64_t* in, const uint32_t* perm, size_t n, uint64_t* out, cudaStream_t s) {
  if (n == 0) return;
  count_launch();
  const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16);
  k_permute_u64<<<blocks, 256, 0, s>>>(in, perm, n, out);
}

// ---------------------------------------------------------------------------------------------
// Exclusive scan of u32: tiles of 2048 (256 threads x 8 items), multi-level for large n.
// ---------------------------------------------------------------------------------------------
constexpr int SC_THREADS = 256;
constexpr int SC_ITEMS = 8;
constexpr int SC_TILE = SC_THREADS * SC_ITEMS;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total, uint32_t* warp_sums) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < (SC_THREADS / 32) ? warp_sums[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < (SC_THREADS / 32)) warp_sums[lane] = w;
  }
  __syncthreads();
  const uint32_t warp_prefix = warp ? warp_sums[warp - 1] : 0u;
  *total = warp_sums[SC_THREADS / 32 - 1];
  return warp_prefix + x - v;
}

__global__ void __launch_bounds__(SC_THREADS) k_scan_reduce(const uint32_t* __restrict__ in, size_t n,
                                                            uint32_t* __restrict__ partial) {
  __shared__ uint32_t ws[SC_THREADS / 32];
  const size_t base = (size_t)blockIdx.x * SC_TILE;
  uint32_t sum = 0;
#pragma unroll
  for (int j = 0; j < SC_ITEMS; ++j) {
    const size_t i = base + (size_t)j * SC_THREADS + threadIdx.x;
    if (i < n) sum += in[i];
  }
  uint32_t total;
  block_exclusive_scan(sum, &total, ws);
  if (threadIdx.x == 0) partial[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SC_THREADS) k_scan_tile(const uint32_t* __restrict__ in, uint32_t* out, size_t n,
                                                          const uint32_t* __restrict__ block_offsets) {
  __shared__ uint32_t ws[SC_THREADS / 32];
  const size_t base = (size_t)blockIdx.x * SC_TILE + (size_t)threadIdx.x * SC_ITEMS;
  uint32_t v[SC_ITEMS];
  uint32_t sum = 0;
#pragma unroll
  for (int j = 0; j < SC_ITEMS; ++j) {
    const size_t i = base + j;
    v[j] = i < n ? in[i] : 0u;
    sum += v[j];
  }
  uint32_t total;
  uint32_t run = block_exclusive_scan(sum, &total, ws);
  if (block_offsets) run += block_offsets[blockIdx.x];
#pragma unroll
  for (int j = 0; j < SC_ITEMS; ++j) {
    const size_t i = base + j;
    if (i < n) out[i] = run;
    run += v[j];
  }
}

static size_t scan_tmp_words(size_t n) {
  size_t total = 0;
  while (n > (size_t)SC_TILE) {
    n = (n + SC_TILE - 1) / SC_TILE;
    total += n + 64;
  }
  return total + 64;
}

static void scan_rec(const uint32_t* in, uint32_t* out, size_t n, uint32_t* tmp, cudaStream_t s) {
  if (n == 0) return;
  if (n <= (size_t)SC_TILE) {
    count_launch();
    k_scan_tile<<<1, SC_THREADS, 0, s>>>(in, out, n, nullptr);
    return;
  }
  const size_t nb = (n + SC_TILE - 1) / SC_TILE;
  uint32_t* partial = tmp;
  count_launch();
  k_scan_reduce<<<(unsigned)nb, SC_THREADS, 0, s>>>(in, n, partial);
  scan_rec(partial, partial, nb, tmp + nb + 64, s);
  count_launch();
  k_scan_tile<<<(unsigned)nb, SC_THREADS, 0, s>>>(in, out, n, partial);
}

cudaError_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, size_t n, DevBuf& tmp, cudaStream_t s) {
  cudaError_t e = ensure(tmp, scan_tmp_words(n) * sizeof(uint32_t));
  if (e != cudaSuccess) return e;
  scan_rec(in, out, n, as<uint32_t>(tmp), s);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// LSD radix sort, 8-bit digits. Per pass: block histograms (digit-major), exclusive scan of the
// histograms, then a stable scatter. Within a block each warp ranks a contiguous sub-tile in
// warp-striped rounds (lanes with equal digits found by ballots), so equal digits keep their
// input order.
// ---------------------------------------------------------------------------------------------
constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_BINS = 256;

// The lanes whose 9-bit value d equals this lane's (a digit, or 0x100 | lane for a lane without
// an element): one ballot per bit, the same mask as __match_any_sync.
__device__ __forceinline__ uint32_t match_digit(uint32_t d) {
  uint32_t peers = 0xffffffffu;
#pragma unroll
  for (int b = 0; b < 9; ++b) {
    const uint32_t bal = __ballot_sync(0xffffffffu, (d >> b) & 1u);
    peers &= ((d >> b) & 1u) ? bal : ~bal;
  }
  return peers;
}

__global__ void __launch_bounds__(RS_THREADS) k_radix_hist(const uint64_t* __restrict__ keys, size_t n, int shift,
                                                           uint32_t* __restrict__ block_hist, int nblocks) {
  __shared__ uint32_t h[RS_BINS];
  for (int t = threadIdx.x; t < RS_BINS; t += RS_THREADS) h[t] = 0;
  __syncthreads();
  const size_t base = (size_t)blockIdx.x * RS_TILE;
  const int lane = threadIdx.x & 31;
#pragma unroll 4
  for (int j = 0; j < RS_ITEMS; ++j) {
    const size_t i = base + (size_t)j * RS_THREADS + threadIdx.x;
    const bool valid = i < n;
    const uint32_t d = valid ? (uint32_t)((keys[i] >> shift) & (RS_BINS - 1)) : (0x100u | (uint32_t)lane);
    const uint32_t peers = match_digit(d);
    if (valid && (__ffs(peers) - 1) == lane) atomicAdd(&h[d], (uint32_t)__popc(peers));
  }
  __syncthreads();
  for (int t = threadIdx.x; t < RS_BINS; t += RS_THREADS) block_hist[(size_t)t * nblocks + blockIdx.x] = h[t];
}

// Dynamic shared memory of k_radix_scatter: per-warp digit counts, the block's digit starts and
// global bases, and the tile reordered by digit.
constexpr size_t RS_SCATTER_SMEM =
    sizeof(uint32_t) * (RS_WARPS * RS_BINS + 2 * RS_BINS) + (sizeof(uint64_t) + sizeof(uint32_t)) * RS_TILE;

// One stable pass: the tile is ranked by digit (per warp with match_digit, warps in order),
// reordered in shared memory, and each digit's run is written out contiguously, so consecutive
// threads store consecutive addresses.
__global__ void __launch_bounds__(RS_THREADS) k_radix_scatter(const uint64_t* __restrict__ kin,
                                                              const uint32_t* __restrict__ vin,
                                                              uint64_t* __restrict__ kout,
                                                              uint32_t* __restrict__ vout, size_t n, int shift,
                                                              const uint32_t* __restrict__ offsets, int nblocks) {
  extern __shared__ __align__(16) unsigned char rs_smem[];
  uint64_t* sk = reinterpret_cast<uint64_t*>(rs_smem);                       // [RS_TILE]
  uint32_t* sv = reinterpret_cast<uint32_t*>(sk + RS_TILE);                  // [RS_TILE]
  uint32_t(*wc)[RS_BINS] = reinterpret_cast<uint32_t(*)[RS_BINS]>(sv + RS_TILE);  // [RS_WARPS][RS_BINS]
  uint32_t* dstart = &wc[RS_WARPS][0];                                       // [RS_BINS]
  uint32_t* gbase = dstart + RS_BINS;                                        // [RS_BINS]
  __shared__ uint32_t warp_tot[RS_WARPS];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int t = threadIdx.x; t < RS_WARPS * RS_BINS; t += RS_THREADS) (&wc[0][0])[t] = 0;
  __syncthreads();
  const unsigned lt_mask = (1u << lane) - 1u;
  const size_t tile0 = (size_t)blockIdx.x * RS_TILE;
  const size_t wbase = tile0 + (size_t)warp * 32 * RS_ITEMS;
  uint64_t k[RS_ITEMS];
  uint32_t v[RS_ITEMS];
  uint32_t rank[RS_ITEMS];
#pragma unroll
  for (int j = 0; j < RS_ITEMS; ++j) {
    const size_t i = wbase + (size_t)j * 32 + lane;
    const bool valid = i < n;
    k[j] = valid ? kin[i] : 0ull;
    v[j] = valid ? vin[i] : 0u;
    const uint32_t d = valid ? (uint32_t)((k[j] >> shift) & (RS_BINS - 1)) : (0x100u | (uint32_t)lane);
    const uint32_t peers = match_digit(d);
    uint32_t prev = 0;
    if (valid) prev = wc[warp][d];
    __syncwarp();
    if (valid) {
      rank[j] = prev + (uint32_t)__popc(peers & lt_mask);
      if ((__ffs(peers) - 1) == lane) wc[warp][d] = prev + (uint32_t)__popc(peers);
    }
    __syncwarp();
  }
  __syncthreads();
  // Thread t = digit t: its block total, then the exclusive scan over digits (block-local starts).
  static_assert(RS_THREADS == RS_BINS, "one thread per digit");
  const int t = threadIdx.x;
  uint32_t tot = 0;
#pragma unroll
  for (int w = 0; w < RS_WARPS; ++w) tot += wc[w][t];
  uint32_t incl = tot;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  uint32_t before = 0;
  for (int w = 0; w < warp; ++w) before += warp_tot[w];
  const uint32_t start = before + incl - tot;
  dstart[t] = start;
  gbase[t] = offsets[(size_t)t * nblocks + blockIdx.x] - start;
  uint32_t run = start;
#pragma unroll
  for (int w = 0; w < RS_WARPS; ++w) {
    const uint32_t c = wc[w][t];
    wc[w][t] = run;
    run += c;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < RS_ITEMS; ++j) {
    const size_t i = wbase + (size_t)j * 32 + lane;
    if (i < n) {
      const uint32_t d = (uint32_t)((k[j] >> shift) & (RS_BINS - 1));
      const uint32_t lp = wc[warp][d] + rank[j];
      sk[lp] = k[j];
      sv[lp] = v[j];
    }
  }
  __syncthreads();
  const uint32_t count = (uint32_t)min((size_t)RS_TILE, n - tile0);
  for (uint32_t q = threadIdx.x; q < count; q += RS_THREADS) {
    const uint64_t key = sk[q];
    const uint32_t pos = gbase[(uint32_t)((key >> shift) & (RS_BINS - 1))] + q;
    kout[pos] = key;
    vout[pos] = sv[q];
  }
}

cudaError_t radix_sort_pairs(uint64_t* keys, uint32_t* vals, size_t n, int bits, SortScratch& sc, cudaStream_t s) {
  if (n <= 1 || bits <= 0) return cudaSuccess;
  if (n > 0xFFFFFFFFull) return cudaErrorInvalidValue;
  const int nblocks = (int)((n + RS_TILE - 1) / RS_TILE);
  cudaError_t e;
  if ((e = ensure(sc.keys_alt, n * sizeof(uint64_t))) != cudaSuccess) return e;
  if ((e = ensure(sc.vals_alt, n * sizeof(uint32_t))) != cudaSuccess) return e;
  if ((e = ensure(sc.block_hist, (size_t)RS_BINS * nblocks * sizeof(uint32_t))) != cudaSuccess) return e;
  uint64_t* ka = keys;
  uint32_t* va = vals;
  uint64_t* kb = as<uint64_t>(sc.keys_alt);
  uint32_t* vb = as<uint32_t>(sc.vals_alt);
  uint32_t* hist = as<uint32_t>(sc.block_hist);
  const int passes = (bits + 7) / 8;
  // The attribute belongs to the current device, so it is set on every call (a cheap host call).
  if ((e = cudaFuncSetAttribute(k_radix_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)RS_SCATTER_SMEM)) != cudaSuccess)
    return e;
  for (int p = 0; p < passes; ++p) {
    const int shift = 8 * p;
    count_launch();
    k_radix_hist<<<nblocks, RS_THREADS, 0, s>>>(ka, n, shift, hist, nblocks);
    if ((e = exclusive_scan_u32(hist, hist, (size_t)RS_BINS * nblocks, sc.scan_tmp, s)) != cudaSuccess) return e;
    count_launch();
    k_radix_scatter<<<nblocks, RS_THREADS, RS_SCATTER_SMEM, s>>>(ka, va, kb, vb, n, shift, hist, nblocks);
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  if (ka != keys) {
    if ((e = cudaMemcpyAsync(keys, ka, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(vals, va, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

}  // namespace cpm

// Self-check of the table-driven Hilbert keys (host only): `samples` random integer coordinates
// (xorshift from `seed`) keyed by the state machine and by the transform; mismatches counted.
extern "C" int cpm_hilbert_fsm_check(int levels, uint64_t samples, uint64_t seed, uint64_t* mismatches, int* states) {
  using namespace cpm;
  if ((levels != KEY_LEVELS && levels != KEY_LEVELS - 2) || !mismatches || !states)
    return set_error(nullptr, CPM_E_INVALID, "cpm_hilbert_fsm_check: levels must be 21 or 19, outputs non-null");
  const HilbertFsm& f = hilbert_fsm(levels);
  *states = f.ok ? f.states : 0;
  uint64_t bad = 0, r = seed | 1ull;
  const uint32_t mask = (1u << levels) - 1u;
  for (uint64_t k = 0; k < samples; ++k) {
    r ^= r << 13;
    r ^= r >> 7;
    r ^= r << 17;
    const uint32_t a0 = (uint32_t)r & mask, a1 = (uint32_t)(r >> 21) & mask, a2 = (uint32_t)(r >> 42) & mask;
    if (!f.ok || hilbert_fsm_host(f, levels, a0, a1, a2) != hilbert_host(levels, a0, a1, a2)) ++bad;
  }
  *mismatches = bad;
  return CPM_OK;
}
