// The recursive parity tree of the fractal KRFFT plans (plan layer, host only).
#pragma once

#include <vector>

#include "cfft_internal.h"

namespace cfft {

// A leaf of the fractal KRFFT's recursive parity tree: its grid, and the stride and
// offset at which it samples the full grid, with its depth below the root.
struct TreeLeaf {
  int n[3], scale[3], offset[3], depth;
};

// build_recursive_tree + collect_leaves (src/fractal_krfft.jl:300-636).  flags bit 0:
// child translations from the half-grid-shifted operations; bit 1: no centring split.
void fractal_tree(const std::vector<SymOp>& ops, const int* N, int dim, int flags, std::vector<TreeLeaf>* leaves,
                  int* n_inner);

}  // namespace cfft
