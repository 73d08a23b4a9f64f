// Host side of the hot phases' tiling (see prima_tiles.h).
#include "prima_tiles.h"

#include <algorithm>
#include <functional>
#include <queue>
#include <utility>

// Weights of the tiles' cost estimate (tile_cost): the distinct sectors a
// tile gathers.  All-zero weights but the first deal the tiles round-robin.
#ifndef PRIMA_TILE_COST_SECTOR
#define PRIMA_TILE_COST_TILE 0.0f
#define PRIMA_TILE_COST_ROW 0.0f
#define PRIMA_TILE_COST_NNZ 0.0f
#define PRIMA_TILE_COST_SECTOR 1.0f
#endif

namespace prima {

std::vector<TileEdge> tile_table(const int32_t *rp, int64_t rows, int64_t cap, int64_t max_rows) {
  std::vector<TileEdge> table;
  table.reserve((size_t)(rows / 16 + 2));
  int64_t r = 0;
  while (r < rows) {
    table.push_back(TileEdge{(int32_t)r, rp[r]});
    int64_t e = r;
    while (e < rows && e - r < max_rows) {
      const int64_t e2 = std::min<int64_t>(rows, e + 4);
      if (e > r && (((int64_t)rp[e2] + 3) & ~3) - (rp[r] & ~3) > cap) break;
      e = e2;
    }
    r = e;
  }
  table.push_back(TileEdge{(int32_t)rows, rp[rows]});
  return table;
}

// Only the weights' ratios matter.  On the 1.34M-column DC-LOPF, dealing by
// sectors took the slowest block's mean work per phase from 22.6 to 21.2 us
// (K') and 18.7 to 17.7 us (K), against dealing round-robin.
float tile_cost(int64_t rows, int64_t nnz, int64_t sectors) {
  constexpr float kTile = PRIMA_TILE_COST_TILE, kRow = PRIMA_TILE_COST_ROW, kNnz = PRIMA_TILE_COST_NNZ,
                  kSector = PRIMA_TILE_COST_SECTOR;
  return kTile + kRow * (float)rows + kNnz * (float)nnz + kSector * (float)sectors;
}

// A marker per sector, stamped with the tile's number, counts each sector
// once per tile.
std::vector<float> tile_costs(const std::vector<TileEdge> &t, const int32_t *rp, const int32_t *ci, int64_t cols,
                              int word) {
  const int shift = word == 8 ? 2 : 3;  // words per 32-byte sector: 4 or 8
  const int64_t nt = (int64_t)t.size() - 1;
  std::vector<int32_t> mark((size_t)((cols >> shift) + 1), -1);
  std::vector<float> cost((size_t)std::max<int64_t>(nt, 0));
  for (int64_t j = 0; j < nt; j++) {
    int64_t sectors = 0;
    for (int64_t k = rp[t[j].row]; k < rp[t[j + 1].row]; k++) {
      int32_t &mk = mark[(size_t)(ci[k] >> shift)];
      if (mk != (int32_t)j) mk = (int32_t)j, sectors++;
    }
    cost[j] = tile_cost(t[j + 1].row - t[j].row, (int64_t)rp[t[j + 1].row] - rp[t[j].row], sectors);
  }
  return cost;
}

// Every block keeps the tile count of a round-robin deal (the first ntiles
// mod nb blocks one more), and the tiles go out heaviest first (ties in
// table order), each to the least-loaded block that still has room (ties to
// the lower block); a block then runs its tiles in table order.  The deal
// depends only on the table, the costs and nb, so a problem's sums group the
// same way on every run.  With nb <= 1, or no more tiles than blocks, slot j
// holds tile j.
std::vector<TileEdge> deal_tiles(const std::vector<TileEdge> &t, const std::vector<float> &cost, int nb) {
  const int64_t nt = std::max<int64_t>((int64_t)t.size() - 1, 0);
  std::vector<TileEdge> pairs((size_t)(2 * nt));
  std::vector<int64_t> slot_tile((size_t)nt);
  if (nb <= 1 || nt <= nb) {
    for (int64_t j = 0; j < nt; j++) slot_tile[j] = j;
  } else {
    std::vector<int64_t> order((size_t)nt);
    for (int64_t j = 0; j < nt; j++) order[j] = j;
    std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) { return cost[x] > cost[y]; });
    std::vector<int64_t> room((size_t)nb);
    for (int b = 0; b < nb; b++) room[b] = nt / nb + (b < nt % nb ? 1 : 0);
    using Load = std::pair<double, int>;
    std::priority_queue<Load, std::vector<Load>, std::greater<Load>> heap;
    for (int b = 0; b < nb; b++) heap.push({0.0, b});
    std::vector<std::vector<int64_t>> mine((size_t)nb);
    for (int64_t j : order) {
      const Load top = heap.top();
      heap.pop();
      mine[top.second].push_back(j);
      if (--room[top.second] > 0) heap.push({top.first + (double)cost[j], top.second});
    }
    for (int b = 0; b < nb; b++) {
      std::sort(mine[b].begin(), mine[b].end());
      for (size_t k = 0; k < mine[b].size(); k++) slot_tile[(size_t)b + k * (size_t)nb] = mine[b][k];
    }
  }
  for (int64_t s = 0; s < nt; s++) {
    pairs[2 * s] = t[slot_tile[s]];
    pairs[2 * s + 1] = t[slot_tile[s] + 1];
  }
  return pairs;
}

}  // namespace prima
