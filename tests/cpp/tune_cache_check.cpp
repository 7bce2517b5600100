// CPU check of the autotuner's selection rule and cache file (csrc/tune_cache.h): prints one line
// per check and exits non-zero on the first failure.
#include <cstdio>
#include <cstdlib>
#include <map>
#include <string>

#include "tune_cache.h"

using namespace cpm;

static int failures = 0;
#define CHECK(cond)                                                   \
  do {                                                                \
    if (!(cond)) {                                                    \
      std::printf("FAIL %s:%d %s\n", __FILE__, __LINE__, #cond);     \
      ++failures;                                                     \
    }                                                                 \
  } while (0)

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  const std::string path = argv[1];

  // selection: the fastest timed candidate of each parameter, ties to the earlier one
  {
    TuneChoice c;
    const float ms[N_TUNE] = {4.11f, 4.57f, 4.62f, 1.10f, 1.098f, 1.20f, 56.3f, 54.9f, 59.4f};
    for (int i = 0; i < N_TUNE; ++i) c.ms[i] = ms[i];
    tune_select(c);
    CHECK(c.radix == 8 && c.ppt == 4 && c.warps == 4);
    const float ms2[N_TUNE] = {3.0f, 3.0f, 2.0f, 0.4f, 0.5f, 0.5f, 0.0f, 0.0f, 0.0f};
    TuneChoice d;
    d.warps = 4;
    for (int i = 0; i < N_TUNE; ++i) d.ms[i] = ms2[i];
    tune_select(d);
    CHECK(d.radix == 0 && d.ppt == 2 && d.warps == 4);  // walk not timed: default kept
    const float tie[3] = {1.0f, 1.0f, 1.0f};
    CHECK(tune_argmin(tie, 3) == 0);
    const float none[3] = {0.0f, 0.0f, 0.0f};
    CHECK(tune_argmin(none, 3) == -1);
    std::printf("selection ok\n");
  }

  // key and line round trip
  {
    const std::string key = tune_key(16777216, 512, 1, 1, 0);
    CHECK(key == "n=16777216 mesh=512 boxes=1 tree=1 quad=0");
    TuneChoice c;
    c.radix = 4;
    c.ppt = 8;
    c.warps = 2;
    const std::string ln = tune_format_line(key, c);
    CHECK(ln == key + "|4 8 2\n");
    std::string k2;
    TuneChoice c2;
    CHECK(tune_parse_line(ln.c_str(), k2, c2) && k2 == key && c2.radix == 4 && c2.ppt == 8 && c2.warps == 2);
    std::printf("line ok\n");
  }

  // invalid records are rejected and leave the output untouched
  {
    std::string k = "unchanged";
    TuneChoice c;
    const char* bad[] = {"no separator 8 4 4\n", "|8 4 4\n", "key|8 4\n", "key|3 4 4\n", "key|8 5 4\n",
                         "key|8 4 16\n", "key|x y z\n"};
    for (const char* b : bad) CHECK(!tune_parse_line(b, k, c) && k == "unchanged" && c.radix == 8);
    std::printf("rejection ok\n");
  }

  // file: appended records, the last record of a key wins, damaged lines are skipped
  {
    std::remove(path.c_str());
    TuneChoice a, b, z;
    a.radix = 8, a.ppt = 4, a.warps = 4;
    b.radix = 0, b.ppt = 2, b.warps = 8;
    z.radix = 4, z.ppt = 8, z.warps = 2;
    CHECK(tune_file_append(path.c_str(), "w1", a));
    CHECK(tune_file_append(path.c_str(), "w2", z));
    FILE* f = std::fopen(path.c_str(), "a");
    CHECK(f != nullptr);
    if (f) {
      std::fputs("w1|7 7 7\ngarbage\n", f);
      std::fclose(f);
    }
    CHECK(tune_file_append(path.c_str(), "w1", b));
    std::map<std::string, TuneChoice> cache;
    tune_file_load(path.c_str(), cache);
    CHECK(cache.size() == 2);
    CHECK(cache["w1"].radix == 0 && cache["w1"].ppt == 2 && cache["w1"].warps == 8);
    CHECK(cache["w2"].radix == 4 && cache["w2"].ppt == 8 && cache["w2"].warps == 2);
    std::map<std::string, TuneChoice> empty;
    tune_file_load((path + ".missing").c_str(), empty);
    tune_file_load(nullptr, empty);
    CHECK(empty.empty());
    std::printf("file ok\n");
  }
  return failures ? 1 : 0;
}
