// CPU check of the autotuner's key and choice cache (macau_b200/csrc/tune.h): histogram keys,
// the per-process map, and the file cache named by MACAU_B200_TUNE_CACHE (written by one
// process, read back by the next).  Usage: tune_cache_check write|read <path>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "tune.h"

static int fail(const char* what) {
  std::printf("FAIL %s\n", what);
  return 1;
}

int main(int argc, char** argv) {
  if (argc != 3) return fail("usage");
  setenv("MACAU_B200_TUNE_CACHE", argv[2], 1);
  // rows of lengths 0, 1, 2, 3, 4, 1000: log2 buckets 0: {0, 1}, 1: {2, 3}, 2: {4}, 9: {1000}
  const std::vector<long long> ptr = {0, 0, 1, 3, 6, 10, 1010};
  const std::string key = mg::tune_key("tc", 32, 148, ptr);
  if (key != "tc:K32:sm148:n6:e1010:h2,2,1,0,0,0,0,0,0,1") return fail(key.c_str());
  const std::string other = mg::tune_key("fp64", 32, 148, ptr);
  if (other == key) return fail("kinds share a key");
  mg::TuneCache& c = mg::TuneCache::get();
  mg::TuneChoice got;
  if (std::strcmp(argv[1], "write") == 0) {
    if (c.find(key, &got)) return fail("fresh cache has the key");
    mg::TuneChoice a;
    a.thr = 1024;
    a.groups = 2;
    a.ms = 0.5;
    a.ms_default = 0.75;
    a.candidates = 10;
    c.put(key, a);
    if (!c.find(key, &got) || got.thr != 1024 || got.groups != 2) return fail("in-process");
    a.thr = 2048;  // a later choice for the same key wins
    c.put(key, a);
    if (!c.find(key, &got) || got.thr != 2048) return fail("overwrite");
    c.clear();
    if (c.find(key, &got)) return fail("clear");
  } else {
    if (!c.find(key, &got)) return fail("file cache not read");
    if (got.thr != 2048 || got.groups != 2 || got.candidates != 10 || got.ms != 0.5 ||
        got.ms_default != 0.75)
      return fail("file cache values");
    if (c.find(other, &got)) return fail("unknown key found");
  }
  std::printf("OK\n");
  return 0;
}
