// Launch-shape table for the hop kernels.  Defaults come from the block
// shapes below; the autotuner (autotune.cu, exposed as cpsgpu_autotune)
// times candidate shapes on the live lattice and records the fastest per
// key.  A shape is (sites per block, slices per block, slices per thread):
// z = 2 selects the DWF slice-pair kernel where Ls allows it.
#pragma once
#include <cuda_runtime.h>

namespace cpsgpu {

struct TuneKey {
  int prec, recon, ep, kind, ls;
  bool operator==(const TuneKey &o) const {
    return prec == o.prec && recon == o.recon && ep == o.ep && kind == o.kind && ls == o.ls;
  }
};

dim3 hop_block(const TuneKey &k, bool mix);
void tune_set(const TuneKey &k, dim3 block);
void tune_clear();
int tune_count();

}  // namespace cpsgpu
