// tree.cu — octree build from sorted octant keys (tree.rs:171-250). The walk is in walk.cu.
//
// Build. Particles are sorted by their 63-bit octant key (21 digits of the reference's descent,
// tree.rs:186-250), or by the Hilbert key of the same cubes (the simulation's order), so every
// node of the reference's tree is a contiguous range of the sorted array: the particles whose
// first d digits equal the node's prefix. One kernel per level splits each node of that level
// that holds more than LEAF_SIZE particles: the 8 sub-ranges are found on digit d+1 (sorted
// within the node: a thread per node on wide levels, a warp per node on levels with few nodes),
// and the non-empty ones become children, allocated contiguously in digit order; a child's octant
// (its centre, and the node's octant mask that the walk's children[0] rule reads) is the octant
// digit of its first particle. Node centres are built with the reference's
// f32 arithmetic (centre +- half/2), so they are bit-identical. A node deeper than the 21 key
// digits that still holds more than LEAF_SIZE particles stays a leaf (the reference would keep
// splitting to depth 40); such nodes are counted.
//
// Centres of mass come from an FP64 exclusive prefix sum of the sorted positions: the sum over a
// node is P[end] - P[start], divided by the count and rounded once to f32. (The reference sums
// in f32 sequentially in input order; the difference is f32 round-off of that sum.)
#include <algorithm>
#include <vector>

#include "cpm_internal.cuh"

namespace cpm {

constexpr int BUILD_THREADS = 256;
constexpr int BUILD_BLOCKS = 148 * 4;

// counters layout (u32): [0..KEY_LEVELS+1] per-level node counts (level 0 = root),
// [32] nodes that hit the key-depth limit with > LEAF_SIZE particles, [33] max depth.
constexpr int CNT_DEPTH_LIMIT = 32;
constexpr int CNT_MAX_DEPTH = 33;
constexpr int CNT_WORDS = 64;

__device__ __forceinline__ uint32_t digit_at(uint64_t key, int shift) { return (uint32_t)(key >> shift) & 7u; }

// First index in [lo, hi) whose digit at `shift` is >= o, or hi if none (digits non-decreasing in
// the range), found by the whole warp: each round probes 32 evenly spaced keys and keeps the
// interval between the last probe below o and the first at or above it, so a range of c keys
// takes about log32(c) rounds of one load per lane.
__device__ __forceinline__ uint32_t warp_lower_bound(const uint64_t* __restrict__ keys, uint32_t lo, uint32_t hi,
                                                     uint32_t o, int shift, int lane) {
  const unsigned FULL = 0xffffffffu;
  while (hi - lo >= 32u) {
    const uint32_t p = lo + (uint32_t)(((uint64_t)(hi - lo) * (uint32_t)lane) >> 5);  // p_0 = lo
    const uint32_t ge = __ballot_sync(FULL, digit_at(__ldg(keys + p), shift) >= o);
    if (ge & 1u) return lo;
    const int j = ge ? __ffs(ge) - 1 : 32;  // first probe at or above o (32: none)
    const uint32_t plo = __shfl_sync(FULL, p, j - 1);
    const uint32_t phi = j < 32 ? __shfl_sync(FULL, p, j & 31) : hi;
    lo = plo + 1u;
    hi = phi;
  }
  const uint32_t p = lo + (uint32_t)lane;
  const uint32_t ge = __ballot_sync(FULL, p >= hi || digit_at(__ldg(keys + p), shift) >= o);
  return lo + (uint32_t)(__ffs(ge) - 1);  // lane hi - lo (< 32) always votes
}

// The root of every box (one box, or a batch of `roots` boxes of n_box particles each, sorted box by
// box): node b covers the particles of box b, the cube [0, L]^3 of its own box.
__global__ void k_tree_root(uint4* link, float4* geo, uint32_t* counters, uint32_t n, float half0, uint32_t roots,
                            uint32_t n_box) {
  for (uint32_t b = threadIdx.x; b < roots; b += blockDim.x) {
    const uint32_t s0 = roots > 1 ? b * n_box : 0u, e0 = roots > 1 ? min(n, (b + 1) * n_box) : n;
    link[b] = make_uint4(s0, e0, 0u, 0u);
    geo[b] = make_float4(half0, half0, half0, half0);
  }
  if (threadIdx.x < CNT_WORDS) counters[threadIdx.x] = threadIdx.x == 0 ? roots : 0u;
}

// first index in [lo, hi) whose digit is >= o (digits non-decreasing in the range)
__device__ __forceinline__ uint32_t lower_bound_digit(const uint64_t* __restrict__ keys, uint32_t lo, uint32_t hi,
                                                      uint32_t o, int shift) {
  while (lo < hi) {
    const uint32_t mid = lo + ((hi - lo) >> 1);
    if (digit_at(__ldg(keys + mid), shift) < o)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// Splits the nodes of level d. A level with more nodes than the grid has warps takes one node
// per thread: the 8 octant sub-ranges by counting the digits d+1 of a small node's keys, or by
// binary search on them in a larger one. A smaller level (the top
// levels, and the sparse deep levels of clustered states), where a thread's searches would be
// a long chain of dependent loads with little else in flight, takes one node per warp: nodes of
// up to SMALL_NODE particles count the digits of all their keys (coalesced loads, a ballot per
// octant), larger ones search the 7 boundaries with warp_lower_bound.
constexpr uint32_t SMALL_NODE = 256;
constexpr uint32_t SCAN_NODE = 64;  // thread path: nodes up to this size count their digits

// keys: the sort keys (octant or Hilbert digits split the node); okeys: the particles' octant keys
// (a child's octant is the digit of its first particle; the same array as keys for octant order).
__global__ void __launch_bounds__(BUILD_THREADS) k_tree_level(int d, int levels, const uint64_t* __restrict__ keys,
                                                              const uint64_t* __restrict__ okeys, uint4* link,
                                                              float4* geo, uint32_t* counters, uint32_t capacity,
                                                              DevStatus* st) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  uint32_t lb = 0;
  for (int j = 0; j < d; ++j) lb += counters[j];
  const uint32_t cnt = counters[d];
  const uint32_t next_base = lb + cnt;
  // After a capacity failure the counters overshoot; never touch nodes past the arrays.
  const uint32_t level_end = min(next_base, capacity);
  const int shift = 3 * (levels - 1 - d);
  const uint32_t warps = gridDim.x * (BUILD_THREADS / 32);
  if (cnt > warps) {
    // Thread per node; each warp allocates the children of its 32 nodes with one atomic (an
    // atomic per node on the level's single counter serialises wide levels).
    for (uint32_t base = lb + blockIdx.x * BUILD_THREADS + (threadIdx.x & ~31u); base < level_end;
         base += gridDim.x * BUILD_THREADS) {
      const uint32_t node = base + (uint32_t)lane;
      const bool valid = node < level_end;
      const uint4 L = valid ? link[node] : make_uint4(0u, 0u, 0u, 0u);
      const uint32_t s = L.x, e = L.y, c = e - s;
      bool split = false;
      if (valid) {
        if (c <= (uint32_t)LEAF_SIZE || d >= MAX_DEPTH) {
          link[node] = make_uint4(s, e, 0u, (uint32_t)d << 8);
        } else if (d >= levels) {
          atomicAdd(&counters[CNT_DEPTH_LIMIT], 1u);
          link[node] = make_uint4(s, e, 0u, (uint32_t)d << 8);
        } else {
          split = true;
        }
      }
      uint32_t b[9];
      b[0] = s;
      b[8] = e;
      uint32_t mask = 0;
      if (split) {
        if (c <= SCAN_NODE) {
          // Small node: read its keys in order and count each digit (eight 8-bit counters in
          // one word); a few sectors instead of the scattered probes of seven binary searches.
          unsigned long long counts = 0ull;
          for (uint32_t i = s; i < e; ++i) counts += 1ull << (8u * digit_at(__ldg(keys + i), shift));
#pragma unroll
          for (int o = 1; o < 8; ++o) b[o] = b[o - 1] + (uint32_t)((counts >> (8 * (o - 1))) & 0xFFull);
        } else {
          uint32_t lo = s;
#pragma unroll
          for (uint32_t o = 1; o < 8; ++o) {
            lo = lower_bound_digit(keys, lo, e, o, shift);
            b[o] = lo;
          }
        }
#pragma unroll
        for (int o = 0; o < 8; ++o)
          if (b[o + 1] > b[o]) mask |= 1u << o;
      }
      // octant of each non-empty sub-range (its first particle's octant digit)
      uint32_t octmask = 0, octs = 0;
      if (split) {
#pragma unroll
        for (int o = 0; o < 8; ++o)
          if (mask & (1u << o)) {
            const uint32_t oc = okeys == keys ? (uint32_t)o : digit_at(__ldg(okeys + b[o]), shift);
            octmask |= 1u << oc;
            octs |= oc << (3 * o);
          }
      }
      // Children of the warp's nodes: an inclusive scan of their counts, one atomic by lane 31.
      const uint32_t nch = (uint32_t)__popc(mask);
      uint32_t incl = nch;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += y;
      }
      uint32_t wbase = 0;
      if (lane == 31 && incl > 0u) wbase = atomicAdd(&counters[d + 1], incl);
      wbase = __shfl_sync(FULL, wbase, 31);
      const uint32_t any_split = __ballot_sync(FULL, split);
      if (lane == 0 && any_split != 0u) atomicMax(&counters[CNT_MAX_DEPTH], (uint32_t)(d + 1));
      if (!split) continue;
      const uint32_t first = next_base + wbase + incl - nch;
      if (first + nch > capacity) {
        dev_fail(st, DEV_NODE_CAPACITY, (int)(first + nch));
        link[node] = make_uint4(s, e, 0u, (uint32_t)d << 8);
        continue;
      }
      const float4 G = geo[node];
      const float q = G.w * 0.5f;  // half / 2.0
      uint32_t r = 0;
#pragma unroll
      for (int o = 0; o < 8; ++o) {
        if (!(mask & (1u << o))) continue;
        const uint32_t child = first + r++;
        const uint32_t oc = (octs >> (3 * o)) & 7u;
        link[child] = make_uint4(b[o], b[o + 1], 0u, 0u);
        geo[child] = make_float4(__fadd_rn(G.x, (oc & 1) ? q : -q), __fadd_rn(G.y, (oc & 2) ? q : -q),
                                 __fadd_rn(G.z, (oc & 4) ? q : -q), q);
      }
      link[node] = make_uint4(s, e, first, octmask | ((uint32_t)d << 8));
    }
    return;
  }
  for (uint32_t node = lb + blockIdx.x * (BUILD_THREADS / 32) + (threadIdx.x >> 5); node < level_end;
       node += warps) {
    const uint4 L = link[node];
    const uint32_t s = L.x, e = L.y, c = e - s;
    if (c <= (uint32_t)LEAF_SIZE || d >= MAX_DEPTH) {
      if (lane == 0) link[node] = make_uint4(s, e, 0u, (uint32_t)d << 8);
      continue;
    }
    if (d >= levels) {
      if (lane == 0) {
        atomicAdd(&counters[CNT_DEPTH_LIMIT], 1u);
        link[node] = make_uint4(s, e, 0u, (uint32_t)d << 8);
      }
      continue;
    }
    uint32_t bo = s;  // lane o (1..7): first index whose digit is >= o
    if (c <= SMALL_NODE) {
      uint32_t below = 0;  // lane o: keys with digit < o
      for (uint32_t i0 = s; i0 < e; i0 += 32) {
        const uint32_t i = i0 + (uint32_t)lane;
        const uint32_t dg = i < e ? digit_at(__ldg(keys + i), shift) : 8u;
#pragma unroll
        for (uint32_t o = 1; o < 8; ++o) {
          const uint32_t bal = __ballot_sync(FULL, dg < o);
          if ((uint32_t)lane == o) below += (uint32_t)__popc(bal);
        }
      }
      bo = s + below;
    } else {
      uint32_t lo = s;
      for (uint32_t o = 1; o < 8; ++o) {
        lo = warp_lower_bound(keys, lo, e, o, shift, lane);
        if ((uint32_t)lane == o) bo = lo;
      }
    }
    // Lane o < 8: octant o's range [olo, ohi) (b[0] = s, b[8] = e).
    const uint32_t nb = __shfl_sync(FULL, bo, (lane + 1) & 31);
    const uint32_t olo = lane == 0 ? s : bo, ohi = lane == 7 ? e : nb;
    const uint32_t mask = __ballot_sync(FULL, lane < 8 && ohi > olo);
    const uint32_t nch = (uint32_t)__popc(mask);
    uint32_t first = 0;
    if (lane == 0) first = next_base + atomicAdd(&counters[d + 1], nch);
    first = __shfl_sync(FULL, first, 0);
    if (first + nch > capacity) {
      if (lane == 0) {
        dev_fail(st, DEV_NODE_CAPACITY, (int)(first + nch));
        link[node] = make_uint4(s, e, 0u, (uint32_t)d << 8);
      }
      continue;
    }
    // lane o: the octant of sub-range o (its first particle's octant digit)
    const bool live = lane < 8 && ((mask >> lane) & 1u);
    const uint32_t oc = !live ? 0u : (okeys == keys ? (uint32_t)lane : digit_at(__ldg(okeys + olo), shift));
    const uint32_t octmask = __reduce_or_sync(FULL, live ? 1u << oc : 0u);
    if (live) {
      const float4 G = geo[node];
      const float q = G.w * 0.5f;  // half / 2.0
      const uint32_t child = first + (uint32_t)__popc(mask & ((1u << lane) - 1u));
      link[child] = make_uint4(olo, ohi, 0u, 0u);
      geo[child] = make_float4(__fadd_rn(G.x, (oc & 1) ? q : -q), __fadd_rn(G.y, (oc & 2) ? q : -q),
                               __fadd_rn(G.z, (oc & 4) ? q : -q), q);
    }
    if (lane == 0) {
      link[node] = make_uint4(s, e, first, octmask | ((uint32_t)d << 8));
      atomicMax(&counters[CNT_MAX_DEPTH], (uint32_t)(d + 1));
    }
  }
}

// ---------------------------------------------------------------------------------------------
// FP64 exclusive prefix sums of sorted positions: P[i] = sum_{j<i} x_j, P[n] = total.
// ---------------------------------------------------------------------------------------------
constexpr int PS_THREADS = 256;
constexpr int PS_ITEMS = 8;
constexpr int PS_TILE = PS_THREADS * PS_ITEMS;

struct D3 {
  double x, y, z;
};
__device__ __forceinline__ D3 d3add(D3 a, D3 b) { return D3{a.x + b.x, a.y + b.y, a.z + b.z}; }

__device__ __forceinline__ D3 shfl_up_d3(D3 v, int o) {
  return D3{__shfl_up_sync(0xffffffffu, v.x, o), __shfl_up_sync(0xffffffffu, v.y, o),
            __shfl_up_sync(0xffffffffu, v.z, o)};
}

// Block-wide exclusive scan of D3 (per-thread partial), returns the thread's prefix and the total.
__device__ __forceinline__ D3 block_scan_d3(D3 v, D3* total, D3* ws) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  D3 x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const D3 y = shfl_up_d3(x, o);
    if (lane >= o) x = d3add(x, y);
  }
  if (lane == 31) ws[warp] = x;
  __syncthreads();
  if (warp == 0) {
    D3 w = lane < PS_THREADS / 32 ? ws[lane] : D3{0.0, 0.0, 0.0};
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const D3 y = shfl_up_d3(w, o);
      if (lane >= o) w = d3add(w, y);
    }
    if (lane < PS_THREADS / 32) ws[lane] = w;
  }
  __syncthreads();
  const D3 wp = warp ? ws[warp - 1] : D3{0.0, 0.0, 0.0};
  *total = ws[PS_THREADS / 32 - 1];
  return D3{wp.x + x.x - v.x, wp.y + x.y - v.y, wp.z + x.z - v.z};
}

__global__ void __launch_bounds__(PS_THREADS) k_pos_reduce(const float* __restrict__ x3, size_t n, D3* partial) {
  __shared__ D3 ws[PS_THREADS / 32];
  const size_t base = (size_t)blockIdx.x * PS_TILE + (size_t)threadIdx.x * PS_ITEMS;
  D3 s{0.0, 0.0, 0.0};
#pragma unroll
  for (int j = 0; j < PS_ITEMS; ++j) {
    const size_t i = base + j;
    if (i < n) s = d3add(s, D3{(double)x3[3 * i], (double)x3[3 * i + 1], (double)x3[3 * i + 2]});
  }
  D3 total;
  block_scan_d3(s, &total, ws);
  if (threadIdx.x == 0) partial[blockIdx.x] = total;
}

// Exclusive scan of the block partials in one block (sequential chunks of PS_THREADS).
__global__ void __launch_bounds__(PS_THREADS) k_partial_scan(D3* partial, size_t nb) {
  __shared__ D3 ws[PS_THREADS / 32];
  D3 carry{0.0, 0.0, 0.0};
  for (size_t c0 = 0; c0 < nb; c0 += PS_THREADS) {
    const size_t i = c0 + threadIdx.x;
    const D3 v = i < nb ? partial[i] : D3{0.0, 0.0, 0.0};
    D3 total;
    const D3 ex = block_scan_d3(v, &total, ws);
    if (i < nb) partial[i] = d3add(carry, ex);
    carry = d3add(carry, total);
    __syncthreads();
  }
}

__global__ void __launch_bounds__(PS_THREADS) k_pos_prefix(const float* __restrict__ x3, size_t n,
                                                           const D3* __restrict__ partial, double* P) {
  __shared__ D3 ws[PS_THREADS / 32];
  const size_t base = (size_t)blockIdx.x * PS_TILE + (size_t)threadIdx.x * PS_ITEMS;
  D3 v[PS_ITEMS];
  D3 s{0.0, 0.0, 0.0};
#pragma unroll
  for (int j = 0; j < PS_ITEMS; ++j) {
    const size_t i = base + j;
    v[j] = i < n ? D3{(double)x3[3 * i], (double)x3[3 * i + 1], (double)x3[3 * i + 2]} : D3{0.0, 0.0, 0.0};
    s = d3add(s, v[j]);
  }
  D3 total;
  D3 run = d3add(block_scan_d3(s, &total, ws), partial[blockIdx.x]);
#pragma unroll
  for (int j = 0; j < PS_ITEMS; ++j) {
    const size_t i = base + j;
    if (i <= n) {
      P[3 * i] = run.x;
      P[3 * i + 1] = run.y;
      P[3 * i + 2] = run.z;
    }
    run = d3add(run, v[j]);
  }
}

__global__ void k_tree_com(const uint4* __restrict__ link, const double* __restrict__ P, float4* mass,
                           const uint32_t* __restrict__ counters, uint32_t capacity) {
  uint32_t total = 0;
  for (int j = 0; j <= KEY_LEVELS; ++j) total += counters[j];
  total = min(total, capacity);
  for (uint32_t node = blockIdx.x * blockDim.x + threadIdx.x; node < total; node += gridDim.x * blockDim.x) {
    const uint4 L = link[node];
    const double c = (double)(L.y - L.x);
    const double sx = P[3 * (size_t)L.y] - P[3 * (size_t)L.x];
    const double sy = P[3 * (size_t)L.y + 1] - P[3 * (size_t)L.x + 1];
    const double sz = P[3 * (size_t)L.y + 2] - P[3 * (size_t)L.x + 2];
    mass[node] = make_float4((float)(sx / c), (float)(sy / c), (float)(sz / c), (float)(L.y - L.x));
  }
}

// Second moments about the centre of mass, T = sum_j (x_j - com)(x_j - com)^T over the node's
// particles (unit masses), one warp per node with FP64 sums; stored as (Txx, Tyy, Tzz, Txy),
// (Txz, Tyz, 0, 0). Nodes with half >= half_max are never accepted by the walk and get zeros.
// No counterpart in the reference, whose tree carries monopoles only (tree.rs:68-80).
__global__ void k_tree_quad(const uint4* __restrict__ link, const float4* __restrict__ geo,
                            const float4* __restrict__ mass, const float* __restrict__ x3, float4* __restrict__ quad,
                            const uint32_t* __restrict__ counters, uint32_t capacity, float half_max) {
  uint32_t total = 0;
  for (int j = 0; j <= KEY_LEVELS; ++j) total += counters[j];
  total = min(total, capacity);
  const int lane = threadIdx.x & 31;
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t node = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); node < total; node += warps) {
    double t[6] = {0, 0, 0, 0, 0, 0};
    if (geo[node].w < half_max) {
      const uint4 L = link[node];
      const float4 M = mass[node];
      for (uint32_t i = L.x + lane; i < L.y; i += 32) {
        const double dx = (double)x3[3 * (size_t)i] - M.x, dy = (double)x3[3 * (size_t)i + 1] - M.y,
                     dz = (double)x3[3 * (size_t)i + 2] - M.z;
        t[0] += dx * dx;
        t[1] += dy * dy;
        t[2] += dz * dz;
        t[3] += dx * dy;
        t[4] += dx * dz;
        t[5] += dy * dz;
      }
#pragma unroll
      for (int k = 0; k < 6; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t[k] += __shfl_xor_sync(0xffffffffu, t[k], o);
    }
    if (lane == 0) {
      quad[2 * (size_t)node] = make_float4((float)t[0], (float)t[1], (float)t[2], (float)t[3]);
      quad[2 * (size_t)node + 1] = make_float4((float)t[4], (float)t[5], 0.0f, 0.0f);
    }
  }
}

cudaError_t tree_build(TreeNodes& t, const uint64_t* sorted_keys, const float* sorted_x3, size_t n, float box,
                       DevStatus* st, cudaStream_t s, float quad_half_max, int levels, size_t n_box,
                       const uint64_t* octant_keys) {
  if (n == 0) return cudaSuccess;
  const size_t cap = 2 * n + 64;
  cudaError_t e;
  if (t.capacity < cap || !t.link.p) {
    if ((e = ensure(t.geo, cap * sizeof(float4))) != cudaSuccess) return e;
    if ((e = ensure(t.mass, cap * sizeof(float4))) != cudaSuccess) return e;
    if ((e = ensure(t.link, cap * sizeof(uint4))) != cudaSuccess) return e;
    t.capacity = cap;
  }
  if ((e = ensure(t.counters, CNT_WORDS * sizeof(uint32_t))) != cudaSuccess) return e;
  if ((e = ensure(t.prefix, 3 * (n + 1) * sizeof(double))) != cudaSuccess) return e;
  const size_t nb = (n + 1 + PS_TILE - 1) / PS_TILE;
  if ((e = ensure(t.scan_tmp, (nb + 1) * sizeof(D3))) != cudaSuccess) return e;

  uint4* link = as<uint4>(t.link);
  float4* geo = as<float4>(t.geo);
  uint32_t* counters = as<uint32_t>(t.counters);
  count_launch();
  const uint32_t roots = n_box ? (uint32_t)((n + n_box - 1) / n_box) : 1u;
  k_tree_root<<<1, 256, 0, s>>>(link, geo, counters, (uint32_t)n, box / 2.0f, roots, (uint32_t)n_box);
  for (int d = 0; d <= levels; ++d) {
    count_launch();
    k_tree_level<<<BUILD_BLOCKS, BUILD_THREADS, 0, s>>>(d, levels, sorted_keys,
                                                        octant_keys ? octant_keys : sorted_keys, link, geo,
                                                        counters, (uint32_t)t.capacity, st);
  }

  D3* partial = as<D3>(t.scan_tmp);
  double* P = as<double>(t.prefix);
  count_launch();
  k_pos_reduce<<<(unsigned)nb, PS_THREADS, 0, s>>>(sorted_x3, n, partial);
  count_launch();
  k_partial_scan<<<1, PS_THREADS, 0, s>>>(partial, nb);
  count_launch();
  k_pos_prefix<<<(unsigned)nb, PS_THREADS, 0, s>>>(sorted_x3, n, partial, P);
  count_launch();
  k_tree_com<<<BUILD_BLOCKS, BUILD_THREADS, 0, s>>>(link, P, as<float4>(t.mass), counters, (uint32_t)t.capacity);
  t.has_quad = quad_half_max > 0.0f;
  if (t.has_quad) {
    if ((e = ensure(t.quad, 2 * t.capacity * sizeof(float4))) != cudaSuccess) return e;
    count_launch();
    k_tree_quad<<<BUILD_BLOCKS, BUILD_THREADS, 0, s>>>(link, geo, as<float4>(t.mass), sorted_x3, as<float4>(t.quad),
                                                       counters, (uint32_t)t.capacity, quad_half_max);
  }
  return cudaGetLastError();
}

}  // namespace cpm
