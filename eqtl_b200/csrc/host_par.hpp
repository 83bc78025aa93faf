// Host-side helpers for the scan epilogue work that stays on the CPU (the
// candidate lists of a scan are O(1e5) entries): a thread-parallel loop and
// an LSD radix sort of 64-bit keys.
#pragma once
#include <stdint.h>

#include <algorithm>
#include <thread>
#include <vector>

namespace eqtl {

// f(i) for i in [0, n), split into contiguous ranges over the host threads;
// small n runs inline.
template <class F>
void parallel_for(size_t n, F&& f, size_t min_per_thread = 4096) {
  const size_t hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t nt = std::min(hw, (n + min_per_thread - 1) / std::max<size_t>(min_per_thread, 1));
  if (nt <= 1) {
    for (size_t i = 0; i < n; ++i) f(i);
    return;
  }
  std::vector<std::thread> th;
  th.reserve(nt);
  const size_t step = (n + nt - 1) / nt;
  for (size_t t = 0; t < nt; ++t) {
    const size_t lo = t * step, hi = std::min(n, lo + step);
    if (lo >= hi) break;
    th.emplace_back([&f, lo, hi] {
      for (size_t i = lo; i < hi; ++i) f(i);
    });
  }
  for (auto& x : th) x.join();
}

// Sorts keys ascending (stable, LSD, 16-bit digits) and applies the same
// permutation to idx when it is given. Digits above the largest key are
// skipped.
inline void radix_sort_u64(std::vector<uint64_t>& keys, std::vector<uint32_t>* idx = nullptr) {
  const size_t n = keys.size();
  if (n < 2) return;
  uint64_t mx = 0;
  for (uint64_t k : keys) mx |= k;
  std::vector<uint64_t> kt(n);
  std::vector<uint32_t> it(idx ? n : 0);
  std::vector<uint32_t> cnt(1 << 16);
  for (int shift = 0; shift < 64 && (mx >> shift) != 0; shift += 16) {
    std::fill(cnt.begin(), cnt.end(), 0u);
    for (uint64_t k : keys) ++cnt[(k >> shift) & 0xFFFF];
    uint32_t s = 0;
    for (uint32_t& c : cnt) {
      const uint32_t v = c;
      c = s;
      s += v;
    }
    for (size_t i = 0; i < n; ++i) {
      const uint32_t d = cnt[(keys[i] >> shift) & 0xFFFF]++;
      kt[d] = keys[i];
      if (idx) it[d] = (*idx)[i];
    }
    keys.swap(kt);
    if (idx) idx->swap(it);
  }
}

}  // namespace eqtl
