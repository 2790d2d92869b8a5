// Autotuner of the row samplers' work split and CTA shape.
//
// A sampler launch pulls tasks (whole rows, or parts of rows longer than a split threshold)
// from a queue in descending length order, so the threshold sets the bucket shape of the
// power-law row lengths: a low one evens out the tail of the launch at the cost of more partial
// Grams to reduce, a high one the reverse.  The CUDA-core sampler also has a CTA shape (row groups
// per CTA).  The best pair depends on the row-length histogram, K and the SM count, so the
// context times every candidate on its own data and keeps the fastest.
//
// Choices are cached per process by (sampler kind, K, SM count, rows, entries, log2 histogram of
// the row lengths), and, when the environment variable MACAU_B200_TUNE_CACHE names a file, in
// that file too (one "key value" line per choice), so later contexts on the same data skip the
// timing.
#pragma once

#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

namespace mg {

struct TuneChoice {
  long long thr = 0;   // split threshold (entries)
  int groups = 0;      // row groups per CTA of the CUDA-core sampler (0: not applicable)
  double ms = 0.0;     // measured half-sweep time of the choice
  double ms_default = 0.0;  // measured half-sweep time of the default choice
  int candidates = 0;  // candidates timed
};

// Key of a tuning problem: sampler kind, K, SM count, rows, entries and the exact log2 histogram
// of the row lengths (bucket b counts rows with 2^b <= len < 2^(b+1); empty rows in bucket 0).
inline std::string tune_key(const char* kind, int K, int sms, const std::vector<long long>& ptr) {
  long long hist[40] = {0};
  const long long n = (long long)ptr.size() - 1;
  for (long long r = 0; r < n; r++) {
    const long long len = ptr[r + 1] - ptr[r];
    int b = 0;
    while (b < 39 && (2LL << b) <= len) b++;
    hist[b]++;
  }
  std::ostringstream os;
  os << kind << ":K" << K << ":sm" << sms << ":n" << n << ":e" << (n > 0 ? ptr[n] : 0) << ":h";
  int last = 39;
  while (last > 0 && hist[last] == 0) last--;
  for (int b = 0; b <= last; b++) os << (b ? "," : "") << hist[b];
  return os.str();
}

class TuneCache {
 public:
  static TuneCache& get() {
    static TuneCache c;
    return c;
  }
  bool find(const std::string& key, TuneChoice* out) {
    std::lock_guard<std::mutex> g(mu_);
    load();
    auto it = map_.find(key);
    if (it == map_.end()) return false;
    *out = it->second;
    return true;
  }
  void put(const std::string& key, const TuneChoice& c) {
    std::lock_guard<std::mutex> g(mu_);
    load();
    map_[key] = c;
    const char* path = std::getenv("MACAU_B200_TUNE_CACHE");
    if (path && *path) {
      if (FILE* f = std::fopen(path, "a")) {
        std::fprintf(f, "%s %lld %d %.6f %.6f %d\n", key.c_str(), c.thr, c.groups, c.ms,
                     c.ms_default, c.candidates);
        std::fclose(f);
      }
    }
  }
  void clear() {
    std::lock_guard<std::mutex> g(mu_);
    map_.clear();
    loaded_ = true;  // a cleared cache does not re-read the file
  }

 private:
  void load() {
    if (loaded_) return;
    loaded_ = true;
    const char* path = std::getenv("MACAU_B200_TUNE_CACHE");
    if (!path || !*path) return;
    FILE* f = std::fopen(path, "r");
    if (!f) return;
    char key[4096];
    TuneChoice c;
    while (std::fscanf(f, "%4095s %lld %d %lf %lf %d", key, &c.thr, &c.groups, &c.ms,
                       &c.ms_default, &c.candidates) == 6)
      map_[key] = c;  // later lines win
    std::fclose(f);
  }
  std::mutex mu_;
  std::map<std::string, TuneChoice> map_;
  bool loaded_ = false;
};

}  // namespace mg
