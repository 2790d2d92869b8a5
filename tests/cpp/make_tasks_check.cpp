// CPU check of the row samplers' work split (make_tasks in macau_b200/csrc/host_util.h), the
// knob the autotuner varies: for power-law row lengths and every split threshold it may pick,
// each row's entries are covered exactly once by its parts, part boundaries sit on the alignment
// grid relative to the row start, no part is longer than the threshold rounded up to the
// alignment, split rows get distinct counters and consecutive scratch slots, and the list is
// sorted by descending length, stably.  Then interleave_groups (the tensor-core sampler's group
// order): the same groups of four, each once and intact, the partial last group last, the
// longest group first, and both ends of the sorted list used before the middle.
// Prints OK or the first failure.
#include <cmath>
#include <cstdio>
#include <map>
#include <random>
#include <vector>

#include "host_util.h"

namespace mg {
long long g_h2d_bytes = 0;
long long g_d2h_bytes = 0;
}  // namespace mg

static int fail(const char* what, long long a, long long b) {
  std::printf("FAIL %s %lld %lld\n", what, a, b);
  return 1;
}

static int check(const std::vector<long long>& ptr, long long thr, int align) {
  int nsplit = 0, nslots = 0;
  const std::vector<mg::RowTask> t = mg::make_tasks(ptr, thr, align, nsplit, nslots);
  const long long n = (long long)ptr.size() - 1;
  std::vector<long long> covered(n, 0);
  std::vector<int> seen_split(nsplit, 0), seen_slot(nslots, 0);
  const long long cap = (thr + align - 1) / align * align;
  for (size_t i = 0; i < t.size(); i++) {
    const mg::RowTask& k = t[i];
    if (k.row < 0 || k.row >= n) return fail("row", k.row, n);
    const long long len = ptr[k.row + 1] - ptr[k.row];
    const long long off = k.begin - ptr[k.row];
    if (off < 0 || off + k.len > len) return fail("range", k.row, off);
    if (off % align) return fail("alignment", k.row, off);
    if (k.nparts > 1 && k.len > cap) return fail("part length", k.len, cap);
    if (k.nparts == 1 && (k.len != len || off != 0)) return fail("whole row", k.row, k.len);
    if (k.nparts > 1) {
      if (k.part < 0 || k.part >= k.nparts) return fail("part index", k.part, k.nparts);
      if (k.split < 0 || k.split >= nsplit) return fail("split counter", k.split, nsplit);
      if (k.slot < 0 || k.slot + k.nparts > nslots) return fail("slots", k.slot, nslots);
      seen_slot[k.slot + k.part]++;
      if (k.part == 0) seen_split[k.split]++;
    }
    covered[k.row] += k.len;
    if (i > 0 && t[i - 1].len < k.len) return fail("descending", t[i - 1].len, k.len);
    if (i > 0 && t[i - 1].len == k.len &&
        (t[i - 1].row > k.row || (t[i - 1].row == k.row && t[i - 1].part > k.part)))
      return fail("stable", t[i - 1].row, k.row);
  }
  for (long long r = 0; r < n; r++)
    if (covered[r] != ptr[r + 1] - ptr[r]) return fail("coverage", r, covered[r]);
  for (int v : seen_split)
    if (v != 1) return fail("split counters", v, nsplit);
  for (int v : seen_slot)
    if (v != 1) return fail("slot use", v, nslots);
  return 0;
}

static int check_interleave(const std::vector<long long>& ptr, long long thr, double row_cost) {
  int nsplit = 0, nslots = 0;
  const std::vector<mg::RowTask> sorted = mg::make_tasks(ptr, thr, 16, nsplit, nslots);
  std::vector<mg::RowTask> t = sorted;
  mg::interleave_groups(t, row_cost);
  if (t.size() != sorted.size()) return fail("interleave size", (long long)t.size(), (long long)sorted.size());
  const size_t ng = (sorted.size() + 3) / 4;
  if (ng < 3) return 0;
  // map each output group to its input group by its first task
  std::map<std::pair<int, int>, size_t> first;
  for (size_t h = 0; h < ng; h++) first[{sorted[4 * h].row, sorted[4 * h].part}] = h;
  std::vector<int> used(ng, 0);
  std::vector<size_t> order;
  for (size_t g = 0; g < ng; g++) {
    const auto it = first.find({t[4 * g].row, t[4 * g].part});
    if (it == first.end()) return fail("interleave unknown group", (long long)g, 0);
    const size_t src = it->second;
    if (used[src]++) return fail("interleave repeated group", (long long)src, 0);
    for (size_t k = 4 * g; k < std::min(t.size(), 4 * g + 4); k++)
      if (t[k].row != sorted[4 * src + (k - 4 * g)].row ||
          t[k].part != sorted[4 * src + (k - 4 * g)].part)
        return fail("interleave group contents", (long long)g, (long long)k);
    if (sorted.size() % 4 && src == ng - 1 && g != ng - 1)
      return fail("partial group not last", (long long)g, 0);
    order.push_back(src);
  }
  if (order[0] != 0) return fail("interleave first group", (long long)order[0], 0);
  // the first half of the output draws on both the first and the last quarter of the input
  size_t head = 0, tail = 0;
  for (size_t g = 0; g < ng / 2; g++) {
    head += order[g] < ng / 4;
    tail += order[g] >= ng - ng / 4 - 1;
  }
  if (head == 0 || tail == 0) return fail("interleave ends", (long long)head, (long long)tail);
  return 0;
}

int main() {
  std::mt19937_64 rng(7);
  // power-law row lengths in [0, 20000] (p(k) ~ 1/k), plus the edge lengths
  std::vector<long long> lens = {0, 1, 15, 16, 17, 255, 256, 257, 4095, 4096, 4097, 20000};
  std::uniform_real_distribution<double> u(0.0, 1.0);
  for (int i = 0; i < 20000; i++) lens.push_back((long long)std::exp(u(rng) * std::log(20001.0)) - 1);
  for (int align : {1, 16}) {
    std::vector<long long> ptr(1, 0);
    for (long long l : lens) ptr.push_back(ptr.back() + (align == 16 ? (l + 15) / 16 * 16 : l));
    for (long long thr : {256LL, 454LL, 909LL, 1819LL, 3638LL, 7277LL, 16384LL}) {
      const long long t = align == 16 ? (thr + 15) / 16 * 16 : thr;
      if (check(ptr, t, align)) return 1;
      if (align == 16)
        for (double rc : {4.0, 16.0})
          if (check_interleave(ptr, t, rc)) return 1;
    }
  }
  std::printf("OK\n");
  return 0;
}
