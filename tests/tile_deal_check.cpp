// Test driver for the hot phases' host-side tiling (prima_tiles.cpp), built
// and run by tests/test_tile_deal.py with the host compiler alone.
//
// stdin (binary, little-endian): int64 rows, cols, cap, max_rows, word, nb;
// int32 rp[rows + 1]; int32 ci[rp[rows]].
// stdout (binary): int64 ntiles; int32 table[2 * (ntiles + 1)];
// float cost[ntiles]; int32 pairs[4 * ntiles].
#include <cstdio>
#include <vector>

#include "prima_tiles.h"

template <typename V>
static bool read_into(V *p, size_t n) {
  return std::fread(p, sizeof(V), n, stdin) == n;
}

int main() {
  int64_t hdr[6];
  if (!read_into(hdr, 6)) return 2;
  const int64_t rows = hdr[0], cols = hdr[1], cap = hdr[2], max_rows = hdr[3];
  const int word = (int)hdr[4], nb = (int)hdr[5];
  std::vector<int32_t> rp((size_t)rows + 1);
  if (!read_into(rp.data(), rp.size())) return 2;
  std::vector<int32_t> ci((size_t)rp[(size_t)rows]);
  if (!ci.empty() && !read_into(ci.data(), ci.size())) return 2;

  const std::vector<prima::TileEdge> t = prima::tile_table(rp.data(), rows, cap, max_rows);
  const std::vector<float> cost = prima::tile_costs(t, rp.data(), ci.data(), cols, word);
  const std::vector<prima::TileEdge> pairs = prima::deal_tiles(t, cost, nb);

  const int64_t nt = (int64_t)t.size() - 1;
  std::fwrite(&nt, sizeof(nt), 1, stdout);
  std::fwrite(t.data(), sizeof(prima::TileEdge), t.size(), stdout);
  std::fwrite(cost.data(), sizeof(float), cost.size(), stdout);
  std::fwrite(pairs.data(), sizeof(prima::TileEdge), pairs.size(), stdout);
  return 0;
}
