// tables.h -- PairHMM prior tables, built on the host once per process.
//
// These follow roDV's Context<float> / Context<double>
// (src/core/pairhmm/common/context.h:22-166), which themselves follow Intel
// GKL: ph2pr[q] = 10^(-q/10); a Jacobian log10(1 + 10^-x) table with step
// 1e-4 up to 8; matchToMatch[(max*(max+1))/2 + min] =
// 1 - 10^approxLog10Sum(-0.1*max, -0.1*min).  The float tables are built the
// way Context<float> builds them (Jacobian sum evaluated in float, then the
// pow/log1p in double) so that FP32 priors equal the reference's bit for bit.
// The kernels only ever index quals masked with &127, so the tables cover
// q in [0, 127].
#pragma once
#include <vector>

#include "layout.h"

namespace rodv {

struct HostPriorTables {
  std::vector<float> ph2pr_f, mm_f;     // 128, kMmTableSize
  std::vector<double> ph2pr_d, mm_d;
};

// Built on first use; thread-safe.
const HostPriorTables& host_prior_tables();

}  // namespace rodv
