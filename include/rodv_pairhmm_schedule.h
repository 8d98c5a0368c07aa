// rodv_pairhmm_schedule.h -- C++ drop-in for roDV's batch-compute call.
//
// Declares pairhmm::schedule::schedule_pairhmm with the signature of
// src/core/pairhmm_schedule.h:14-25 (roDV), so code written against roDV's
// scheduler links against librodv_pairhmm.so unchanged.  The definition
// (rodv_b200/csrc/schedule_shim.cpp) sends the region to the B200 engine.
//
// Semantics kept from the reference:
//   * returns false when there are no haplotypes or no reads
//     (pairhmm_schedule.cpp:130-132);
//   * result is resized to [M][N], hap-major, log10 likelihoods;
//   * use_double = true computes every pair in FP64.
// Differences:
//   * max_idle_ratio_float / max_idle_ratio_double are accepted and have no
//     effect (they tune the reference's CPU SIMD grouping);
//   * verbose prints the engine's statistics instead of per-group logs, and
//     nothing is printed otherwise;
//   * inputs the reference would read out of bounds (quality arrays shorter
//     than the read, bases other than A/C/G/T/N, empty sequences) make the
//     call return false instead.
#ifndef RODV_PAIRHMM_SCHEDULE_H_
#define RODV_PAIRHMM_SCHEDULE_H_

#include <cstdint>
#include <vector>

namespace pairhmm {
namespace schedule {

bool schedule_pairhmm(const std::vector<std::vector<uint8_t>>& haplotypes,
                      const std::vector<std::vector<uint8_t>>& reads,
                      std::vector<std::vector<double>>& result,
                      const std::vector<std::vector<uint8_t>>& quality,
                      const std::vector<std::vector<uint8_t>>& insertion_qualities,
                      const std::vector<std::vector<uint8_t>>& deletion_qualities,
                      const std::vector<std::vector<uint8_t>>& gap_contiguous_qualities,
                      bool use_double = false, double max_idle_ratio_float = 0.1,
                      double max_idle_ratio_double = 0.1, bool verbose = false);

}  // namespace schedule
}  // namespace pairhmm

#endif  // RODV_PAIRHMM_SCHEDULE_H_
