// Host side of the hot phases' tiling: cutting a CSR matrix into tiles of
// rows, estimating each tile's cost, and dealing the tiles to the blocks of
// a team.  Plain C++ with no CUDA types, so that the host tests can build
// these functions alone.
#pragma once

#include <cstdint>
#include <vector>

namespace prima {

// A tile table entry: (first row, first nonzero) of a tile; the table ends
// with (rows, nnz).  Laid out as a CUDA int2, which the device reads.
struct TileEdge {
  int32_t row, nnz;
};

// Tiles of at most max_rows rows, starting at multiples of 4, grown 4 rows at
// a time while their nonzeros (rounded out to 16-byte granules of 4 entries)
// fit cap; a group of 4 rows that alone does not fit is a tile of its own.
std::vector<TileEdge> tile_table(const int32_t *rp, int64_t rows, int64_t cap, int64_t max_rows);

// Estimated time of one tile from its rows, its nonzeros and the distinct
// 32-byte sectors of the gathered vector that it touches.
float tile_cost(int64_t rows, int64_t nnz, int64_t sectors);

// tile_cost of every tile of t, over a matrix with row pointers rp and column
// indices ci gathering a vector of cols words of word (4 or 8) bytes.
std::vector<float> tile_costs(const std::vector<TileEdge> &t, const int32_t *rp, const int32_t *ci, int64_t cols,
                              int word);

// The tiles of t handed to a team of nb blocks as (start, end) pairs, slot
// rank + k*nb holding block rank's k-th tile (see prima_tiles.cpp).
std::vector<TileEdge> deal_tiles(const std::vector<TileEdge> &t, const std::vector<float> &cost, int nb);

}  // namespace prima
