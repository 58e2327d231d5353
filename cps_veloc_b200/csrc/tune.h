// Launch-shape table for the hop kernels.  Defaults come from the block
// shapes below; the autotuner (autotune.cu, exposed as cpsgpu_autotune)
// times candidate shapes on the live lattice and records the fastest per
// key.  A shape is (sites per block, slices per block, slices per thread):
// z = 2 selects the DWF slice-pair kernel where Ls allows it; with it goes
// the order in which the grid's blocks traverse the (site block, slice
// group) pairs (HopOrder).
#pragma once
#include <cuda_runtime.h>

namespace cpsgpu {

struct TuneKey {
  int prec, recon, ep, kind, ls;
  bool operator==(const TuneKey &o) const {
    return prec == o.prec && recon == o.recon && ep == o.ep && kind == o.kind && ls == o.ls;
  }
};

// block traversal orders of a hop launch: consecutive blocks take
//   ORDER_SLICES: the slice groups of one site block (its links stay in L1);
//   ORDER_SITES:  the site blocks of one slice group, in lexicographic order
//                 (the slice groups on the grid's y dimension)
enum HopOrder { ORDER_SLICES = 0, ORDER_SITES = 1, ORDER_COUNT = 2 };

dim3 hop_block(const TuneKey &k, bool mix);
int hop_order(const TuneKey &k);
void tune_set(const TuneKey &k, dim3 block, int order = ORDER_SLICES);
void tune_clear();
int tune_count();

}  // namespace cpsgpu
