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
// merge > 1: `merge` consecutive column tiles of a super-block row form one
// tile (wider MMA tiles); diag then marks a tile whose first column tile is
// the diagonal one, and b_end stops at the tile's own columns.
std::vector<PairTile> make_pair_tiles(const Buckets &a, const Buckets &b, bool symmetric, int tm,
                                      int tn, size_t row_bytes = 0, int merge = 1);

// The same tiles in the same order, described by their L2 super-blocks (a
// few hundred entries instead of one entry per tile) and expanded into the
// tile list by a device kernel: the host plans O(super-blocks) work and
// uploads a few KB instead of building and copying ~10 MB per call.
struct SuperBlock {
    int sa, ea, sb, eb;  // bucket row ranges of the label
    int bi, bj, g;       // first tile row / column, tiles per side
    int nti, ntj;        // tiles of the label
    int symmetric;
    long long offset;    // index of the super-block's first tile in the list
};
std::vector<SuperBlock> make_super_blocks(const Buckets &a, const Buckets &b, bool symmetric,
                                          int tm, int tn, size_t row_bytes, long long &ntiles);
kfb_status expand_tiles(const std::vector<SuperBlock> &sbs, long long ntiles, int tm, int tn,
                        DevBuf &tiles, cudaStream_t s, int merge = 1);
// Rewrite the offsets of sbs for tiles of `merge` column tiles; returns the
// number of merged tiles.
long long merge_offsets(std::vector<SuperBlock> &sbs, int merge);

}  // namespace kfb
