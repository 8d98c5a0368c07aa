// chain_plan.cpp -- the packer's placement of a region's single-pass reads in
// chain items (chain_plan.h).  Replaces the reference's SIMD grouping
// (greedy_grouping, src/core/pairhmm_schedule.cpp:46-105) for the warp
// wavefront's geometry.
#include "chain_plan.h"

#include <algorithm>

namespace rodv {

namespace {

// Time per computed cell (lane rows x columns, padding included) of the
// uniform-gap chain kernels by rows per lane R, relative to R = 8: the
// autotuner's per-class batches (reads of 32R - 5 bases, one read pair per
// item) on B200 with each class's fastest variant, measured with a running
// sum per step (with the sum row they agree within 3%, R = 4 excepted at
// 1.089).  R <= 4 run as two 16-lane items per warp with 2R rows per lane,
// hence their closeness to R = 8.
constexpr double kChainCellCost[kMaxRowsPerLane + 1] = {0.0,   1.53,  1.20,  1.09, 1.024,
                                                        1.093, 1.047, 1.031, 1.0};

}  // namespace

void chain_geometry(const int (&items_per_warp)[kMaxRowsPerLane + 1],
                    ChainGeom (&geom)[kMaxRowsPerLane + 1]) {
  geom[0] = ChainGeom{};
  for (int R = 1; R <= kMaxRowsPerLane; ++R) {
    const int ipw = items_per_warp[R] > 1 ? items_per_warp[R] : 1;
    geom[R] = ChainGeom{single_pass_class(R, true), (uint32_t)(kWarp / ipw), (uint32_t)(R * ipw),
                        R * kChainCellCost[R]};
  }
}

void sort_single_pass(const uint32_t* read_lengths, const uint8_t* read_class,
                      uint32_t read_start, uint32_t num_reads, std::vector<uint32_t>& out) {
  out.clear();
  for (uint32_t r = 0; r < num_reads; ++r) {
    const uint32_t read = read_start + r;
    if (!class_multi(read_class[read])) out.push_back(read);
  }
  std::stable_sort(out.begin(), out.end(), [&](uint32_t x, uint32_t y) {
    const uint32_t kx = ((read_class[x] & 1u) << 20) | read_lengths[x];
    const uint32_t ky = ((read_class[y] & 1u) << 20) | read_lengths[y];
    return kx < ky;
  });
}

void plan_region_chains(const uint32_t* read_lengths, const uint8_t* read_class,
                        const ChainGeom (&geom)[kMaxRowsPerLane + 1], bool stack_uniform,
                        const std::vector<uint32_t>& sr, RegionChains& rc) {
  const ChainGeom& stack_geom = geom[kMaxRowsPerLane];
  // the cheapest uniform class whose items hold pairs with longer reads of
  // lengths lens
  auto cheapest = [&](const uint32_t* lens, size_t n) -> const ChainGeom& {
    const ChainGeom* best = &stack_geom;
    for (int R = 1; R < kMaxRowsPerLane; ++R) {
      uint32_t lanes = 0;
      for (size_t i = 0; i < n; ++i) lanes += pair_lanes(lens[i], geom[R].rows);
      if (lanes <= geom[R].lanes && geom[R].cost < best->cost) best = &geom[R];
    }
    return *best;
  };
  auto pair_class = [&](uint32_t x, uint32_t y) {
    const uint32_t len = std::max(read_lengths[x], read_lengths[y]);
    return class_of(len, (read_class[x] & 1) && (read_class[y] & 1));
  };
  rc.reads.clear();
  rc.items.clear();
  rc.leftover = kNoPair;
  size_t nu = 0;  // reads with per-row gap priors come first
  while (nu < sr.size() && !(read_class[sr[nu]] & 1)) ++nu;
  auto add_pair = [&](uint32_t x, uint32_t y) {
    rc.items.push_back(ChainPairs{pair_class(x, y), (uint32_t)rc.reads.size(), 1});
    rc.reads.push_back(x);
    rc.reads.push_back(y);
  };
  const size_t m = ((nu & 1) && nu < sr.size()) ? nu + 1 : nu;
  size_t k = 0;
  for (; k + 1 < m; k += 2) add_pair(sr[k], sr[k + 1]);
  if (k < m) {  // odd per-row reads and no uniform one
    rc.leftover = sr[k];
    return;
  }
  const size_t nU = sr.size() - m;  // uniform reads sr[m..), increasing length
  if (nU == 0) return;
  // cost of the one-pair item of a pair whose longer read has `len` bases
  // (a leftover: half of one)
  auto pair_cost = [&](uint32_t len) { return cheapest(&len, 1).cost; };
  double classic = 0.0;
  for (size_t i = m; i + 1 < sr.size(); i += 2) classic += pair_cost(read_lengths[sr[i + 1]]);
  if (nU & 1) classic += 0.5 * pair_cost(read_lengths[sr.back()]);
  // Stacked: neighbours in decreasing length pair up (the shortest read of an
  // odd count is the leftover), the pairs go by best fit in that order into
  // items of the R = 8 class (a pair takes the item with the fewest free
  // lanes that still holds its pair_lanes), and each item then goes to the
  // cheapest uniform class that holds its pairs.
  const size_t np = nU / 2;
  bool stacked = false;
  double cost = 0.0;
  if (stack_uniform && np >= 2) {
    rc.pair_item.assign(np, 0);
    rc.item_free.clear();
    for (auto& v : rc.bucket) v.clear();
    for (size_t q = 0; q < np; ++q) {
      const uint32_t x = sr[sr.size() - 1 - 2 * q];
      const uint32_t lanes = pair_lanes(read_lengths[x], stack_geom.rows);
      uint32_t it = kNoPair;
      for (uint32_t f = lanes; f <= stack_geom.lanes && it == kNoPair; ++f)
        if (!rc.bucket[f].empty()) {
          it = rc.bucket[f].back();
          rc.bucket[f].pop_back();
        }
      if (it == kNoPair) {
        it = (uint32_t)rc.item_free.size();
        rc.item_free.push_back(stack_geom.lanes);
      }
      rc.item_free[it] -= lanes;
      rc.bucket[rc.item_free[it]].push_back(it);
      rc.pair_item[q] = it;
    }
    // the items' pairs, item after item, each item's in placement order
    const uint32_t nit = (uint32_t)rc.item_free.size();
    rc.item_fill.assign(nit + 1, 0);
    for (uint32_t it : rc.pair_item) rc.item_fill[it + 1] += 2;
    for (uint32_t it = 0; it < nit; ++it) rc.item_fill[it + 1] += rc.item_fill[it];
    rc.item_lens.resize(np);
    rc.item_cls.resize(nit);
    {
      std::vector<uint32_t>& at = rc.item_free;  // reused: next pair slot per item
      for (uint32_t it = 0; it < nit; ++it) at[it] = rc.item_fill[it] / 2;
      for (size_t q = 0; q < np; ++q)
        rc.item_lens[at[rc.pair_item[q]]++] = read_lengths[sr[sr.size() - 1 - 2 * q]];
    }
    for (uint32_t it = 0; it < nit; ++it) {
      const uint32_t p0 = rc.item_fill[it] / 2, p1 = rc.item_fill[it + 1] / 2;
      const ChainGeom& g = cheapest(rc.item_lens.data() + p0, p1 - p0);
      rc.item_cls[it] = g.cls;
      cost += g.cost;
    }
    if (nU & 1) cost += 0.5 * pair_cost(read_lengths[sr[m]]);
    stacked = cost < classic;
  }
  if (!stacked) {
    size_t i = m;
    for (; i + 1 < sr.size(); i += 2) add_pair(sr[i], sr[i + 1]);
    if (i < sr.size()) rc.leftover = sr[i];
    return;
  }
  const uint32_t nit = (uint32_t)rc.item_cls.size();
  const uint32_t base = (uint32_t)rc.reads.size();
  rc.reads.resize(base + 2 * np);
  for (uint32_t it = 0; it < nit; ++it)
    rc.items.push_back(ChainPairs{rc.item_cls[it], base + rc.item_fill[it],
                                  (rc.item_fill[it + 1] - rc.item_fill[it]) / 2});
  for (size_t q = 0; q < np; ++q) {
    uint32_t& at = rc.item_fill[rc.pair_item[q]];
    rc.reads[base + at] = sr[sr.size() - 1 - 2 * q];
    rc.reads[base + at + 1] = sr[sr.size() - 2 - 2 * q];
    at += 2;
  }
  if (nU & 1) rc.leftover = sr[m];
}

}  // namespace rodv
