// Host-side helpers shared by the library's contexts: a device buffer owning one cudaMalloc,
// and the work split of CSR rows into sampler tasks.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <list>
#include <vector>

#include "common.cuh"

namespace mg {

// Host<->device byte counters of the current process (defined in context.cu).
extern long long g_h2d_bytes;
extern long long g_d2h_bytes;

template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { reset(); }
  void reset() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    reset();
    if (count == 0) count = 1;
    MG_CUDA(cudaMalloc(&p, count * sizeof(T)));
    n = count;
  }
  void alloc_zero(size_t count, cudaStream_t s) {
    alloc(count);
    MG_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
  }
  void upload(const T* h, size_t count, cudaStream_t s) {
    alloc(count);
    if (count) MG_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    g_h2d_bytes += (long long)(count * sizeof(T));
  }
};

// Device copies of buffers, taken on a stream and written back when the object goes out of
// scope, also while an exception unwinds (a failed write-back there is ignored; it surfaces at
// the next checked call).  The autotuner keeps the state its timing runs overwrite in one.
class DeviceBackup {
 public:
  explicit DeviceBackup(cudaStream_t s) : s_(s) {}
  DeviceBackup(const DeviceBackup&) = delete;
  DeviceBackup& operator=(const DeviceBackup&) = delete;
  void save(void* p, size_t bytes) {
    if (!p || bytes == 0) return;
    items_.emplace_back();
    Item& it = items_.back();
    it.dst = p;
    it.bytes = bytes;
    it.copy.alloc(bytes);
    MG_CUDA(cudaMemcpyAsync(it.copy.p, p, bytes, cudaMemcpyDeviceToDevice, s_));
    it.ok = true;
  }
  ~DeviceBackup() {
    for (Item& it : items_)
      if (it.ok) cudaMemcpyAsync(it.dst, it.copy.p, it.bytes, cudaMemcpyDeviceToDevice, s_);
    cudaStreamSynchronize(s_);
  }

 private:
  struct Item {
    void* dst = nullptr;
    size_t bytes = 0;
    bool ok = false;
    DBuf<unsigned char> copy;
  };
  cudaStream_t s_;
  std::list<Item> items_;  // DBuf does not move: list nodes stay in place
};

// Task list over rows lo .. hi - 1 (all rows when hi < 0) with lengths len(r) = ptr[r+1] - ptr[r]
// (positions ptr[r]): rows longer than `thr` are cut into near-equal parts whose boundaries are
// multiples of `align` entries (relative to the row start); tasks sorted by descending length
// (stable).
inline std::vector<RowTask> make_tasks(const std::vector<long long>& ptr, long long thr,
                                       int align, int& nsplit, int& nslots, long long lo = 0,
                                       long long hi = -1) {
  const long long n = (long long)ptr.size() - 1;
  if (hi < 0 || hi > n) hi = n;
  if (lo < 0) lo = 0;
  std::vector<RowTask> tasks;
  tasks.reserve((size_t)std::max(0LL, hi - lo) + 16);
  nsplit = 0;
  nslots = 0;
  for (long long r = lo; r < hi; r++) {
    const long long len = ptr[r + 1] - ptr[r];
    if (len <= thr) {
      tasks.push_back(RowTask{ptr[r], (int)r, (int)len, 0, 1, 0, 0});
      continue;
    }
    const long long units = (len + align - 1) / align;
    const int parts = (int)((len + thr - 1) / thr);
    for (int q = 0; q < parts; q++) {
      const long long b = std::min(len, align * (units * q / parts));
      const long long e = std::min(len, align * (units * (q + 1) / parts));
      tasks.push_back(RowTask{ptr[r] + b, (int)r, (int)(e - b), q, parts, nslots, nsplit});
    }
    nslots += parts;
    nsplit++;
  }
  // stable sort by descending length: a counting sort over the lengths (each at most thr + align)
  int maxlen = 0;
  for (const RowTask& t : tasks) maxlen = std::max(maxlen, t.len);
  std::vector<size_t> start((size_t)maxlen + 2, 0);
  for (const RowTask& t : tasks) start[(size_t)(maxlen - t.len) + 1]++;
  for (size_t b = 1; b < start.size(); b++) start[b] += start[b - 1];
  std::vector<RowTask> out(tasks.size());
  for (const RowTask& t : tasks) out[start[(size_t)(maxlen - t.len)]++] = t;
  return out;
}

// Reorders a task list sorted by descending length in groups of four consecutive tasks (the
// tensor-core sampler's work unit) so that long and short groups alternate: a group costs its
// k-blocks (longest task / 16) in the gather pipeline and `row_cost` k-blocks' worth of time per
// unsplit row in the in-kernel finish, and the next group is the longest remaining one while
// the finish work so far exceeds the gather work, else the shortest remaining one.  Each CTA
// then meets a mix of both instead of a run of long groups (gather-bound, finishers idle)
// followed by a run of short ones (finish-bound, gather pipeline idle).
inline void interleave_groups(std::vector<RowTask>& tasks, double row_cost) {
  const size_t n = tasks.size(), ng = (n + 3) / 4;
  if (ng < 3) return;
  auto gather = [&](size_t g) { return (double)(tasks[4 * g].len / 16); };
  auto finish = [&](size_t g) {
    double f = 0.0;
    for (size_t t = 4 * g; t < std::min(n, 4 * g + 4); t++) f += tasks[t].nparts == 1 ? row_cost : 0.0;
    return f;
  };
  std::vector<RowTask> out;
  out.reserve(n);
  size_t lo = 0, hi = ng - 1;
  double balance = 0.0;  // gather minus finish work of the groups placed so far
  // the last group may be partial: it stays last
  const bool partial = n % 4 != 0;
  if (partial) hi--;
  while (lo <= hi && hi < ng) {
    const size_t g = balance <= 0.0 ? lo++ : hi--;
    balance += gather(g) - finish(g);
    for (size_t t = 4 * g; t < 4 * g + 4; t++) out.push_back(tasks[t]);
    if (hi == (size_t)-1) break;
  }
  if (partial)
    for (size_t t = 4 * (ng - 1); t < n; t++) out.push_back(tasks[t]);
  tasks.swap(out);
}

}  // namespace mg
