// tune_cache.h — the autotuner's record of a workload's launch choices: the selection rule over the
// timed candidates, the workload key, and the one-line text form of the cache file named by
// CPM_TUNE_CACHE. Host-only C++ (no CUDA), shared by sim.cu and the CPU tests.
//
// Cache file: one line per workload, "<key>|<fft plan> <deposit ppt> <walk warps>", appended as
// workloads are tuned; when a key appears more than once the last line wins. A line whose values are
// not among the compiled alternatives (FFT plan 0, 4 or 8; 2, 4 or 8 particles per thread; 2, 4 or
// 8 warps) is ignored, so a damaged file can only cost a fresh tuning, never an invalid launch.
#pragma once

#include <cstddef>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>

namespace cpm {

constexpr int N_TUNE = 9;  // timed candidates: 3 FFT plans, 3 deposit tiles, 3 walk groups

struct TuneChoice {
  int radix = 8, ppt = 4, warps = 4;
  float ms[N_TUNE] = {};  // plan 8, 4, 0; tile 512, 1024, 2048; warps 2, 4, 8 (0 = not timed)
};

constexpr int TUNE_PLANS[3] = {8, 4, 0};
constexpr int TUNE_PPT[3] = {2, 4, 8};
constexpr int TUNE_WARPS[3] = {2, 4, 8};

// The candidate with the smallest measured time among ms[0..count-1] (ties: the earlier one);
// candidates with no time (<= 0, not timed) are skipped; -1 when none was timed.
inline int tune_argmin(const float* ms, int count) {
  int best = -1;
  for (int k = 0; k < count; ++k)
    if (ms[k] > 0.0f && (best < 0 || ms[k] < ms[best])) best = k;
  return best;
}

// Applies the selection rule to c.ms: each parameter takes its fastest timed candidate and keeps its
// current value when none of its candidates was timed.
inline void tune_select(TuneChoice& c) {
  int k = tune_argmin(c.ms, 3);
  if (k >= 0) c.radix = TUNE_PLANS[k];
  k = tune_argmin(c.ms + 3, 3);
  if (k >= 0) c.ppt = TUNE_PPT[k];
  k = tune_argmin(c.ms + 6, 3);
  if (k >= 0) c.warps = TUNE_WARPS[k];
}

inline bool tune_valid(const TuneChoice& c) {
  auto in = [](int v, const int (&set)[3]) { return v == set[0] || v == set[1] || v == set[2]; };
  return in(c.radix, TUNE_PLANS) && in(c.ppt, TUNE_PPT) && in(c.warps, TUNE_WARPS);
}

inline std::string tune_key(size_t particles_per_box, int mesh, int boxes, int tree, int quad) {
  char buf[160];
  std::snprintf(buf, sizeof(buf), "n=%zu mesh=%d boxes=%d tree=%d quad=%d", particles_per_box, mesh, boxes, tree, quad);
  return buf;
}

inline std::string tune_format_line(const std::string& key, const TuneChoice& c) {
  char buf[64];
  std::snprintf(buf, sizeof(buf), "|%d %d %d\n", c.radix, c.ppt, c.warps);
  return key + buf;
}

// Parses one line; false (and nothing set) when it is not a valid record.
inline bool tune_parse_line(const char* line, std::string& key, TuneChoice& c) {
  const char* bar = std::strchr(line, '|');
  if (!bar || bar == line) return false;
  TuneChoice t;
  if (std::sscanf(bar + 1, "%d %d %d", &t.radix, &t.ppt, &t.warps) != 3 || !tune_valid(t)) return false;
  key.assign(line, (size_t)(bar - line));
  c = t;
  return true;
}

inline void tune_file_load(const char* path, std::map<std::string, TuneChoice>& cache) {
  if (!path) return;
  FILE* f = std::fopen(path, "r");
  if (!f) return;
  char line[256];
  while (std::fgets(line, sizeof(line), f)) {
    std::string key;
    TuneChoice c;
    if (tune_parse_line(line, key, c)) cache[key] = c;
  }
  std::fclose(f);
}

inline bool tune_file_append(const char* path, const std::string& key, const TuneChoice& c) {
  if (!path) return false;
  FILE* f = std::fopen(path, "a");
  if (!f) return false;
  const std::string ln = tune_format_line(key, c);
  const bool ok = std::fputs(ln.c_str(), f) >= 0;
  std::fclose(f);
  return ok;
}

}  // namespace cpm
