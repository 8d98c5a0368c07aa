/*
 * pairhmm_oracle.c -- CPU oracle for the PairHMM forward likelihood.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA engine in
 * rodv_b200/ is compared against.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load it.  The product path never calls it:
 * the engine has no CPU fallback.
 *
 * It restates, in plain scalar C, the algorithm of roDV's src/core PairHMM
 * (itself a re-templating of Intel GKL's PairHMM):
 *
 *   tables      Context<T> in src/core/pairhmm/common/context.h:22-166
 *               ph2pr[q] = 10^(-q/10)              (context.h:109-111 double,
 *                                                    context.h:149-151 float)
 *               Jacobian log10(1+10^-x) table, step 1e-4, tolerance 8
 *                                                   (context.h:44-48)
 *               matchToMatchProb[max(max+1)/2+min]  (context.h:50-60)
 *               approximateLog10SumLog10            (context.h:66-82)
 *               set_mm_prob(ins, del)               (context.h:115-126, :155-166)
 *               INITIAL_CONSTANT 2^1020 / 2^120     (context.h:101, :141)
 *   priors      per read row, quals masked with &127
 *               (pairhmm/intra/pairhmm_impl.cpp:88-115,
 *                pairhmm/inter/pairhmm_inter.cpp:80-98)
 *               match = 1 - ph2pr[q], mismatch = ph2pr[q] / 3
 *               (pairhmm_impl.cpp:156-158)
 *   recurrence  compute_mxy, pairhmm_impl.cpp:245-290:
 *               M = ((M_d*mm + I_d*gapm) + D_d*gapm) * e
 *               I = M_u*mi + I_u*ii
 *               D = M_l*md + D_l*dd
 *   boundary    row 0: M = I = 0, D = INITIAL_CONSTANT / haplen in every column
 *               (pairhmm_impl.cpp:62-69); column 0 rows >= 1: M = I = D = 0
 *   result      sum over columns of (M + I) in the last read row
 *               (pairhmm_impl.cpp:397-438, pairhmm_inter.cpp:220-234)
 *   N bases     'N' on either side matches every base
 *               (common.h:42-56, pairhmm_impl.cpp:26-42)
 *   precision   FP32 first; a result below 1e-28 is recomputed in FP64
 *               (intra/pairhmm_api.cpp:4-23, pairhmm_schedule.cpp:21,229-248)
 *   log10       FP32: log10(x) - 36.1236000061 (float constant);
 *               FP64: log10(x) - 307.050595577260822
 *               (intra/pairhmm_api.cpp:9-10, inter/pairhmm_inter_api.h:8-15)
 *
 * Besides the reference semantics it offers an FP64 mode with per-row
 * power-of-two renormalisation ("scaled"), which gives the true log10
 * likelihood for pairs whose value is below the FP64 range of the 2^1020
 * scaling (log10 < about -615), where the reference itself returns -inf.
 *
 * Pinning: tests/test_oracle.py checks this file against the 104 golden
 * lines of the reference's resouces/pairhmm-testdata.txt (committed as
 * tests/golden/gkl_testdata.tsv), the two hand-computed values of
 * src/core/test/pairhmm_unittest.cpp:103-137, and, where it is built, the
 * reference itself (oracle/_ref).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#if defined(__x86_64__)
#include <xmmintrin.h>
#endif

#define MAX_QUAL 254
#define JAC_TOL 8.0
#define JAC_STEP 0.0001
#define JAC_SIZE ((int)(JAC_TOL / JAC_STEP) + 1)
#define MM_SIZE (((MAX_QUAL + 1) * (MAX_QUAL + 2)) >> 1)

/* log10 offsets of the two initial constants, exactly as the reference
 * spells them (the FP32 one is a float literal, not 120*log10(2)). */
static const float LOG10_INIT_F = 36.1236000061f;
static const double LOG10_INIT_D = 307.050595577260822;
static const float MIN_ACCEPTED_F = 1e-28f;

static double ph2pr_d[128];
static float ph2pr_f[128];
static double jac_d[JAC_SIZE];
static float jac_f[JAC_SIZE];
static double mm_d[MM_SIZE];
static float mm_f[MM_SIZE];
static pthread_once_t tables_once = PTHREAD_ONCE_INIT;

static int fast_round_d(double v) { return v > 0.0 ? (int)(v + 0.5) : (int)(v - 0.5); }
static int fast_round_f(float v) { return v > 0.0f ? (int)(v + 0.5f) : (int)(v - 0.5f); }

/* approximateLog10SumLog10 evaluated in double (context.h:66-82). */
static double approx_sum_d(double small, double big) {
  if (small > big) { double t = big; big = small; small = t; }
  if (isinf(small) || isinf(big)) return big;
  double diff = big - small;
  if (diff >= JAC_TOL) return big;
  int ind = fast_round_d(diff * (1.0 / JAC_STEP));
  return big + jac_d[ind];
}

/* The same function evaluated in float, as Context<float> does. */
static float approx_sum_f(float small, float big) {
  if (small > big) { float t = big; big = small; small = t; }
  if (isinf(small) || isinf(big)) return big;
  float diff = big - small;
  if (diff >= (float)JAC_TOL) return big;
  int ind = fast_round_f(diff * (float)(1.0 / JAC_STEP));
  return big + jac_f[ind];
}

static void init_tables(void) {
  for (int k = 0; k < JAC_SIZE; k++) {
    double v = log10(1.0 + pow(10.0, -((double)k) * JAC_STEP));
    jac_d[k] = v;
    jac_f[k] = (float)v;
  }
  const double inv_ln10 = 1.0 / log(10.0);
  for (int i = 0, off = 0; i <= MAX_QUAL; off += ++i) {
    for (int j = 0; j <= i; j++) {
      double s_d = approx_sum_d(-0.1 * i, -0.1 * j);
      double l_d = log1p(-fmin(1.0, pow(10.0, s_d))) * inv_ln10;
      mm_d[off + j] = pow(10.0, l_d);
      float s_f = approx_sum_f((float)(-0.1 * i), (float)(-0.1 * j));
      double l_f = log1p(-fmin(1.0, pow(10.0, (double)s_f))) * inv_ln10;
      mm_f[off + j] = (float)pow(10.0, l_f);
    }
  }
  for (int x = 0; x < 128; x++) {
    ph2pr_d[x] = pow(10.0, -((double)x) / 10.0);
    ph2pr_f[x] = powf(10.f, -((float)x) / 10.f);
  }
}

static void ensure_tables(void) { pthread_once(&tables_once, init_tables); }

static double mm_prob_d(unsigned a, unsigned b) {
  unsigned lo = a <= b ? a : b, hi = a <= b ? b : a;
  return mm_d[((hi * (hi + 1)) >> 1) + lo];
}
static float mm_prob_f(unsigned a, unsigned b) {
  unsigned lo = a <= b ? a : b, hi = a <= b ? b : a;
  return mm_f[((hi * (hi + 1)) >> 1) + lo];
}

/* Base code: A0 C1 G2 T3 N4, anything else -1. */
static int base_code(uint8_t b) {
  switch (b) {
    case 'A': return 0;
    case 'C': return 1;
    case 'G': return 2;
    case 'T': return 3;
    case 'N': return 4;
    default: return -1;
  }
}
static int bases_match(uint8_t r, uint8_t h) {
  int rc = base_code(r), hc = base_code(h);
  return rc == 4 || hc == 4 || rc == hc;
}

typedef struct {
  const uint8_t *hap, *read, *q, *ins, *del, *gcp;
  uint32_t hap_len, read_len;
} pair_view;

/* ---- FP32 forward, reference order of operations ---------------------- */
static float forward_f32(const pair_view *p) {
  const uint32_t H = p->hap_len, R = p->read_len;
  float *mprev = calloc(H + 1, sizeof(float)), *iprev = calloc(H + 1, sizeof(float));
  float *dprev = malloc((H + 1) * sizeof(float));
  float *mcur = calloc(H + 1, sizeof(float)), *icur = calloc(H + 1, sizeof(float));
  float *dcur = calloc(H + 1, sizeof(float));
  const float init_d = ldexpf(1.f, 120) / (float)H;
  for (uint32_t j = 0; j <= H; j++) dprev[j] = init_d;
  float sum_m = 0.f, sum_i = 0.f;
  for (uint32_t i = 1; i <= R; i++) {
    unsigned qi = p->q[i - 1] & 127, ii_ = p->ins[i - 1] & 127;
    unsigned di = p->del[i - 1] & 127, ci = p->gcp[i - 1] & 127;
    float dist = ph2pr_f[qi];
    float match = 1.0f - dist, mismatch = dist / 3.0f;
    float mm = mm_prob_f(ii_, di), gapm = 1.0f - ph2pr_f[ci];
    float mi = ph2pr_f[ii_], ii = ph2pr_f[ci], md = ph2pr_f[di], dd = ph2pr_f[ci];
    mcur[0] = icur[0] = dcur[0] = 0.f;
    for (uint32_t j = 1; j <= H; j++) {
      float e = bases_match(p->read[i - 1], p->hap[j - 1]) ? match : mismatch;
      float m = ((mprev[j - 1] * mm + iprev[j - 1] * gapm) + dprev[j - 1] * gapm) * e;
      float x = mprev[j] * mi + iprev[j] * ii;
      float y = mcur[j - 1] * md + dcur[j - 1] * dd;
      mcur[j] = m; icur[j] = x; dcur[j] = y;
    }
    float *t;
    t = mprev; mprev = mcur; mcur = t;
    t = iprev; iprev = icur; icur = t;
    t = dprev; dprev = dcur; dcur = t;
  }
  for (uint32_t j = 1; j <= H; j++) { sum_m += mprev[j]; sum_i += iprev[j]; }
  free(mprev); free(iprev); free(dprev); free(mcur); free(icur); free(dcur);
  return sum_m + sum_i;
}

/* ---- FP64 forward; scaled = per-row power-of-two renormalisation -------- */
static double forward_f64(const pair_view *p, int scaled, long *exp_out) {
  const uint32_t H = p->hap_len, R = p->read_len;
  double *mprev = calloc(H + 1, sizeof(double)), *iprev = calloc(H + 1, sizeof(double));
  double *dprev = malloc((H + 1) * sizeof(double));
  double *mcur = calloc(H + 1, sizeof(double)), *icur = calloc(H + 1, sizeof(double));
  double *dcur = calloc(H + 1, sizeof(double));
  const double init_d = (scaled ? 1.0 : ldexp(1.0, 1020)) / (double)H;
  long expo = 0;
  for (uint32_t j = 0; j <= H; j++) dprev[j] = init_d;
  for (uint32_t i = 1; i <= R; i++) {
    unsigned qi = p->q[i - 1] & 127, ii_ = p->ins[i - 1] & 127;
    unsigned di = p->del[i - 1] & 127, ci = p->gcp[i - 1] & 127;
    double dist = ph2pr_d[qi];
    double match = 1.0 - dist, mismatch = dist / 3.0;
    double mm = mm_prob_d(ii_, di), gapm = 1.0 - ph2pr_d[ci];
    double mi = ph2pr_d[ii_], ii = ph2pr_d[ci], md = ph2pr_d[di], dd = ph2pr_d[ci];
    mcur[0] = icur[0] = dcur[0] = 0.0;
    double rowmax = 0.0;
    for (uint32_t j = 1; j <= H; j++) {
      double e = bases_match(p->read[i - 1], p->hap[j - 1]) ? match : mismatch;
      double m = ((mprev[j - 1] * mm + iprev[j - 1] * gapm) + dprev[j - 1] * gapm) * e;
      double x = mprev[j] * mi + iprev[j] * ii;
      double y = mcur[j - 1] * md + dcur[j - 1] * dd;
      mcur[j] = m; icur[j] = x; dcur[j] = y;
      if (scaled) {
        double a = m > x ? m : x;
        a = a > y ? a : y;
        rowmax = a > rowmax ? a : rowmax;
      }
    }
    if (scaled && rowmax > 0.0) {
      int e2;
      frexp(rowmax, &e2);
      for (uint32_t j = 1; j <= H; j++) {
        mcur[j] = ldexp(mcur[j], -e2);
        icur[j] = ldexp(icur[j], -e2);
        dcur[j] = ldexp(dcur[j], -e2);
      }
      expo += e2;
    }
    double *t;
    t = mprev; mprev = mcur; mcur = t;
    t = iprev; iprev = icur; icur = t;
    t = dprev; dprev = dcur; dcur = t;
  }
  double sum_m = 0.0, sum_i = 0.0;
  for (uint32_t j = 1; j <= H; j++) { sum_m += mprev[j]; sum_i += iprev[j]; }
  free(mprev); free(iprev); free(dprev); free(mcur); free(icur); free(dcur);
  if (exp_out) *exp_out = expo;
  return sum_m + sum_i;
}

/* Modes of oracle_pair_log10. */
enum {
  ORACLE_REFERENCE = 0, /* FP32, FP64 rescue below 1e-28: the reference's answer */
  ORACLE_FP64 = 1,      /* FP64 with 2^1020 scaling for every pair */
  ORACLE_SCALED = 2,    /* FP64 with per-row renormalisation: the true value */
  ORACLE_FP32_RAW = 3,  /* raw scaled FP32 sum (no log10), for threshold checks */
};

/* Returns 1 when every base is one of A C G T N (the engine's input domain). */
int oracle_valid_bases(const uint8_t *s, uint32_t n) {
  for (uint32_t k = 0; k < n; k++)
    if (base_code(s[k]) < 0) return 0;
  return 1;
}

double oracle_pair_log10(const uint8_t *hap, uint32_t hap_len, const uint8_t *read,
                         const uint8_t *q, const uint8_t *ins, const uint8_t *del,
                         const uint8_t *gcp, uint32_t read_len, int mode) {
  ensure_tables();
#if defined(__x86_64__)
  /* The reference enables FTZ before computing (common.h:58-62). */
  unsigned int csr = _mm_getcsr();
  _MM_SET_FLUSH_ZERO_MODE(_MM_FLUSH_ZERO_ON);
#endif
  pair_view p = {hap, read, q, ins, del, gcp, hap_len, read_len};
  double out;
  if (mode == ORACLE_REFERENCE || mode == ORACLE_FP32_RAW) {
    float f = forward_f32(&p);
    if (mode == ORACLE_FP32_RAW) {
      out = (double)f;
    } else if ((double)f < (double)MIN_ACCEPTED_F) {
      out = log10(forward_f64(&p, 0, NULL)) - LOG10_INIT_D;
    } else {
      out = log10((double)f) - (double)LOG10_INIT_F;
    }
  } else if (mode == ORACLE_FP64) {
    out = log10(forward_f64(&p, 0, NULL)) - LOG10_INIT_D;
  } else {
    long e2 = 0;
    double v = forward_f64(&p, 1, &e2);
    out = log10(v) + (double)e2 * log10(2.0);
  }
#if defined(__x86_64__)
  _mm_setcsr(csr);
#endif
  return out;
}

/* ---- region batches (the reference's schedule_pairhmm shape) ------------ */
/* Region g holds haps [hap_start, hap_start+num_haps) and reads
 * [read_start, read_start+num_reads); its results are written hap-major at
 * out + out_offset[g], like result[h][r] of schedule_pairhmm. */
typedef struct {
  uint32_t hap_start, num_haps, read_start, num_reads;
} oracle_region;

typedef struct {
  const oracle_region *regions;
  uint32_t num_regions;
  const uint8_t *hap_bases;
  const uint64_t *hap_off;
  const uint32_t *hap_len;
  const uint8_t *read_bases, *q, *ins, *del, *gcp;
  const uint64_t *read_off;
  const uint32_t *read_len;
  double *out;
  const uint64_t *out_off;
  int mode;
  uint64_t total_pairs;
  uint64_t next; /* atomic work counter over pairs */
} batch_job;

static void *batch_worker(void *arg) {
  batch_job *job = (batch_job *)arg;
  for (;;) {
    uint64_t k = __atomic_fetch_add(&job->next, 64, __ATOMIC_RELAXED);
    if (k >= job->total_pairs) break;
    uint64_t end = k + 64 < job->total_pairs ? k + 64 : job->total_pairs;
    /* locate region of pair k by binary search over out_off */
    uint32_t lo = 0, hi = job->num_regions;
    while (hi - lo > 1) {
      uint32_t mid = (lo + hi) / 2;
      if (job->out_off[mid] <= k) lo = mid; else hi = mid;
    }
    uint32_t g = lo;
    for (uint64_t t = k; t < end; t++) {
      while (g + 1 < job->num_regions && job->out_off[g + 1] <= t) g++;
      const oracle_region *rg = &job->regions[g];
      uint64_t local = t - job->out_off[g];
      uint32_t h = rg->hap_start + (uint32_t)(local / rg->num_reads);
      uint32_t r = rg->read_start + (uint32_t)(local % rg->num_reads);
      uint64_t ro = job->read_off[r];
      job->out[t] = oracle_pair_log10(job->hap_bases + job->hap_off[h], job->hap_len[h],
                                      job->read_bases + ro, job->q + ro, job->ins + ro,
                                      job->del + ro, job->gcp + ro, job->read_len[r],
                                      job->mode);
    }
  }
  return NULL;
}

/* Computes every (hap, read) pair of every region with `threads` threads.
 * out_off must hold num_regions+1 prefix offsets of num_haps*num_reads. */
int oracle_batch(const oracle_region *regions, uint32_t num_regions,
                 const uint8_t *hap_bases, const uint64_t *hap_off, const uint32_t *hap_len,
                 const uint8_t *read_bases, const uint8_t *q, const uint8_t *ins,
                 const uint8_t *del, const uint8_t *gcp, const uint64_t *read_off,
                 const uint32_t *read_len, const uint64_t *out_off, double *out, int mode,
                 int threads) {
  ensure_tables();
  if (num_regions == 0) return 0;
  batch_job job = {regions, num_regions, hap_bases, hap_off, hap_len, read_bases, q, ins,
                   del, gcp, read_off, read_len, out, out_off, mode,
                   out_off[num_regions], 0};
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  pthread_t tids[256];
  for (int t = 0; t < threads; t++) pthread_create(&tids[t], NULL, batch_worker, &job);
  for (int t = 0; t < threads; t++) pthread_join(tids[t], NULL);
  return 0;
}

/* Exposes the prior tables so host-side packing code can be checked. */
double oracle_ph2pr(int q) { ensure_tables(); return ph2pr_d[q & 127]; }
float oracle_ph2pr_f(int q) { ensure_tables(); return ph2pr_f[q & 127]; }
double oracle_mm_prob(int ins, int del) { ensure_tables(); return mm_prob_d(ins & 127, del & 127); }
float oracle_mm_prob_f(int ins, int del) { ensure_tables(); return mm_prob_f(ins & 127, del & 127); }
