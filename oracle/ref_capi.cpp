// ref_capi.cpp -- C entry points over the reference's own PairHMM API.
//
// TEST AND BASELINE INFRASTRUCTURE ONLY.  Compiled together with the
// reference's src/core sources (read in place, never copied) into
// oracle/_ref/libref_pairhmm.so by oracle/Makefile.  Tests use it to pin the
// oracle against the reference; bench.py times it as the CPU baseline.
//
// Entry points wrap, without changing them:
//   pairhmm::schedule::schedule_pairhmm   src/core/pairhmm_schedule.h:14-25
//   pairhmm::intra::computeLikelihoods*   src/core/pairhmm/intra/pairhmm_api.h:17-20
//   pairhmm::common::init_native (FTZ)    src/core/pairhmm/common/common.h:58-62
#include "pairhmm_schedule.h"
#include "pairhmm/common/common.h"
#include "pairhmm/common/cpu_features.h"
#include "pairhmm/intra/pairhmm_api.h"

#include <fcntl.h>
#include <cstdio>
#include <unistd.h>

#include <atomic>
#include <cstdint>
#include <thread>
#include <vector>

namespace {

struct RegionDesc {
  uint32_t hap_start, num_haps, read_start, num_reads;
};

struct Flat {
  const RegionDesc* regions;
  const uint8_t* hap_bases;
  const uint64_t* hap_off;
  const uint32_t* hap_len;
  const uint8_t *read_bases, *q, *ins, *del, *gcp;
  const uint64_t* read_off;
  const uint32_t* read_len;
};

using VV = std::vector<std::vector<uint8_t>>;

// Builds the reference's vector-of-vectors inputs for region g and runs
// schedule_pairhmm on them; results go hap-major to out.
bool run_region(const Flat& f, uint32_t g, double* out, bool use_double, double rf,
                double rd) {
  const RegionDesc& rg = f.regions[g];
  VV haps(rg.num_haps), reads(rg.num_reads), q(rg.num_reads), ins(rg.num_reads),
      del(rg.num_reads), gcp(rg.num_reads);
  for (uint32_t h = 0; h < rg.num_haps; ++h) {
    const uint8_t* p = f.hap_bases + f.hap_off[rg.hap_start + h];
    haps[h].assign(p, p + f.hap_len[rg.hap_start + h]);
  }
  for (uint32_t r = 0; r < rg.num_reads; ++r) {
    const uint64_t o = f.read_off[rg.read_start + r];
    const uint32_t n = f.read_len[rg.read_start + r];
    reads[r].assign(f.read_bases + o, f.read_bases + o + n);
    q[r].assign(f.q + o, f.q + o + n);
    ins[r].assign(f.ins + o, f.ins + o + n);
    del[r].assign(f.del + o, f.del + o + n);
    gcp[r].assign(f.gcp + o, f.gcp + o + n);
  }
  std::vector<std::vector<double>> result;
  bool ok = pairhmm::schedule::schedule_pairhmm(haps, reads, result, q, ins, del, gcp,
                                                use_double, rf, rd, false);
  if (!ok) return false;
  for (uint32_t h = 0; h < rg.num_haps; ++h)
    for (uint32_t r = 0; r < rg.num_reads; ++r)
      out[(uint64_t)h * rg.num_reads + r] = result[h][r];
  return true;
}

// schedule_pairhmm prints two lines to stderr on every call
// (pairhmm_schedule.cpp:336-337); batches silence fd 2 while they run.
struct QuietStderr {
  int saved = -1;
  explicit QuietStderr(bool on) {
    if (!on) return;
    fflush(stderr);
    saved = dup(2);
    int devnull = open("/dev/null", O_WRONLY);
    if (devnull >= 0) {
      dup2(devnull, 2);
      close(devnull);
    }
  }
  ~QuietStderr() {
    if (saved >= 0) {
      fflush(stderr);
      dup2(saved, 2);
      close(saved);
    }
  }
};

}  // namespace

extern "C" {

// 2 = AVX-512 path, 1 = AVX2 path, 0 = neither (reference computes nothing).
int ref_isa() {
  if (pairhmm::common::CpuFeatures::hasAVX512Support()) return 2;
  if (pairhmm::common::CpuFeatures::hasAVX2Support()) return 1;
  return 0;
}

// One pair through the reference's intra kernel (FP32, FP64 below 1e-28).
double ref_intra_pair(const uint8_t* hap, uint32_t hap_len, const uint8_t* read,
                      const uint8_t* q, const uint8_t* ins, const uint8_t* del,
                      const uint8_t* gcp, uint32_t read_len, int use_double) {
  pairhmm::common::init_native();
  pairhmm::common::TestCase tc;
  tc.rslen = read_len;
  tc.haplen = hap_len;
  tc.hap = hap;
  tc.rs = read;
  tc.q = q;
  tc.i = ins;
  tc.d = del;
  tc.c = gcp;
  const int isa = ref_isa();
#if defined(REF_HAVE_AVX512)
  if (isa == 2) return pairhmm::intra::computeLikelihoodsAVX512(tc, use_double != 0);
#endif
  if (isa >= 1) return pairhmm::intra::computeLikelihoodsAVX2(tc, use_double != 0);
  return 0.0;
}

// Runs schedule_pairhmm over every region on `threads` worker threads, one
// region per task; results hap-major at out + out_off[g].  A single-threaded
// warm-up call runs first because the reference initialises its static
// tables lazily without synchronisation (context.h:94-106).  Returns the
// number of regions for which schedule_pairhmm returned false.
int ref_schedule_batch(const RegionDesc* regions, uint32_t num_regions,
                       const uint8_t* hap_bases, const uint64_t* hap_off,
                       const uint32_t* hap_len, const uint8_t* read_bases, const uint8_t* q,
                       const uint8_t* ins, const uint8_t* del, const uint8_t* gcp,
                       const uint64_t* read_off, const uint32_t* read_len,
                       const uint64_t* out_off, double* out, int use_double,
                       double ratio_f, double ratio_d, int threads, int quiet) {
  if (num_regions == 0) return 0;
  Flat f{regions, hap_bases, hap_off, hap_len, read_bases, q, ins, del, gcp, read_off,
         read_len};
  QuietStderr qs(quiet != 0);
  pairhmm::common::init_native();
  std::atomic<int> failures{0};
  if (!run_region(f, 0, out + out_off[0], use_double != 0, ratio_f, ratio_d)) failures++;
  std::atomic<uint32_t> next{1};
  auto worker = [&]() {
    pairhmm::common::init_native();
    for (;;) {
      uint32_t g = next.fetch_add(1);
      if (g >= num_regions) break;
      if (!run_region(f, g, out + out_off[g], use_double != 0, ratio_f, ratio_d))
        failures++;
    }
  };
  if (threads < 1) threads = 1;
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
  for (auto& th : pool) th.join();
  return failures.load();
}

}  // extern "C"
