// Tile planning shared by the scalar-kernel launchers.
#pragma once

#include <vector>

#include "kernels_common.cuh"

namespace kfb {

// Same-label tiles of (tm rows of bucket set a) x (tn rows of bucket set b).
// Symmetric problems (a and b the same buckets, tm == tn) keep the tiles with
// b-block >= a-block; the ones on the diagonal get diag = 1.
// Tile pairs (tm rows of a, tn rows of b) of every shared label.  With
// row_bytes > 0 (bytes of one packed row) the list is ordered in square
// super-blocks of tiles whose packed rows fit in half of the L2 cache, so the
// CTAs working on neighbouring tiles at the same time reuse operand tiles from
// L2 instead of streaming a whole label bucket from DRAM per tile row;
// row_bytes = 0 keeps the plain row-major order.
std::vector<PairTile> make_pair_tiles(const Buckets &a, const Buckets &b, bool symmetric, int tm,
                                      int tn, size_t row_bytes = 0);

}  // namespace kfb
