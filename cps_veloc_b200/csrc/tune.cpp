#include "tune.h"

#include <mutex>
#include <vector>

namespace cpsgpu {

namespace {
std::mutex g_mu;
struct Entry {
  TuneKey key;
  dim3 block;
  int order;
};
std::vector<Entry> g_table;
}  // namespace

dim3 hop_block(const TuneKey &k, bool mix) {
  {
    std::lock_guard<std::mutex> lk(g_mu);
    for (auto &e : g_table)
      if (e.key == k) return e.block;
  }
  if (mix) {
    // a block holds every slice of its sites
    int bx = 256 / (k.ls > 0 ? k.ls : 1);
    int p = 1;
    while (p * 2 <= bx) p *= 2;
    return dim3(p < 1 ? 1 : p, k.ls);
  }
  if (k.ls <= 1) return dim3(128, 1);
  // 32 consecutive sites per warp; several slices per block share links in L1
  int bs = (k.ls % 4 == 0) ? 4 : (k.ls % 2 == 0 ? 2 : 1);
  return dim3(32, bs);
}

int hop_order(const TuneKey &k) {
  std::lock_guard<std::mutex> lk(g_mu);
  for (auto &e : g_table)
    if (e.key == k) return e.order;
  return ORDER_SLICES;
}

void tune_set(const TuneKey &k, dim3 block, int order) {
  std::lock_guard<std::mutex> lk(g_mu);
  for (auto &e : g_table)
    if (e.key == k) {
      e.block = block;
      e.order = order;
      return;
    }
  g_table.push_back({k, block, order});
}

void tune_clear() {
  std::lock_guard<std::mutex> lk(g_mu);
  g_table.clear();
}

int tune_count() {
  std::lock_guard<std::mutex> lk(g_mu);
  return (int)g_table.size();
}

}  // namespace cpsgpu
