// Tile planning shared by the scalar-kernel launchers.
#pragma once

#include <vector>

#include "kernels_common.cuh"

namespace kfb {

// Same-label tiles of (tm rows of bucket set a) x (tn rows of bucket set b).
// Symmetric problems (a and b the same buckets, tm == tn) keep the tiles with
// b-block >= a-block; the ones on the diagonal get diag = 1.
std::vector<PairTile> make_pair_tiles(const Buckets &a, const Buckets &b, bool symmetric, int tm,
                                      int tn);

}  // namespace kfb
