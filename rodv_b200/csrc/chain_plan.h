// chain_plan.h -- how the packer turns a region's single-pass reads into
// chain items (host only, no device calls): which reads pair up, which pairs
// share an item's lanes, and which work class each item runs in.
#pragma once
#include <cstdint>
#include <vector>

#include "engine.h"

namespace rodv {

// A uniform-gap class's chain kernel as packed: an item holds `lanes` lanes
// of `rows` rows each (two items of 16 lanes with 2R rows per warp for the
// lane-grouped variants); `cost` is the relative time of one item.
struct ChainGeom {
  int cls;
  uint32_t lanes, rows;
  double cost;
};

// One chain item: its class and read pairs, reads[first, first + 2 * pairs)
// of the region's RegionChains (x, then y or kNoPair).
struct ChainPairs {
  int cls;
  uint32_t first, pairs;
};

// The chain items of one region, its leftover read (kNoPair: none) and the
// planner's scratch (reused across regions by one thread).
struct RegionChains {
  std::vector<uint32_t> reads;
  std::vector<ChainPairs> items;
  uint32_t leftover = kNoPair;
  std::vector<uint32_t> pair_item, item_free, item_fill, item_lens;
  std::vector<int> item_cls;
  std::vector<uint32_t> bucket[kWarp + 1];
};

// geom[R] for R = 1..8 from the chain items per warp of each uniform class's
// packed kernel variant (1, or 2 for the lane-grouped ones).
void chain_geometry(const int (&items_per_warp)[kMaxRowsPerLane + 1],
                    ChainGeom (&geom)[kMaxRowsPerLane + 1]);

// Lanes of `rows` rows that a uniform-gap read pair takes whose longer read
// has len bases: its rows, a pass-through row and the sum row.
inline uint32_t pair_lanes(uint32_t len, uint32_t rows) { return (len + 1) / rows + 1; }

// The single-pass reads read_start .. read_start + num_reads - 1 (read_class[r]
// of each, multi-pass ones left out), in increasing (uniform gaps, length).
void sort_single_pass(const uint32_t* read_lengths, const uint8_t* read_class,
                      uint32_t read_start, uint32_t num_reads, std::vector<uint32_t>& out);

// The chain items of a region's sorted single-pass reads sr (sort_single_pass).
// Reads with per-row gap priors pair neighbour by neighbour, one pair per
// item, in the class of the pair's longer read (an odd last one pairs with
// the shortest uniform read, in a per-row class).  Uniform-gap reads either
// do the same or, where the cost table finds it cheaper (stack_uniform),
// pair neighbours in decreasing length (the shortest of an odd count is the
// leftover), go by best fit into items of the R = 8 class and then each
// item into the cheapest uniform class that holds its pairs.  Depends on the
// region's reads only.
void plan_region_chains(const uint32_t* read_lengths, const uint8_t* read_class,
                        const ChainGeom (&geom)[kMaxRowsPerLane + 1], bool stack_uniform,
                        const std::vector<uint32_t>& sr, RegionChains& rc);

}  // namespace rodv
