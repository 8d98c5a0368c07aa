// pairhmm_fwd.cuh -- the PairHMM forward recurrence as a warp wavefront.
//
// Recurrence (roDV compute_mxy, src/core/pairhmm/intra/pairhmm_impl.cpp:245-290;
// the same body as process_matrix_cell, pairhmm/inter/pairhmm_inter.cpp:276-287),
// i = read row, j = haplotype column:
//   M[i][j] = e(i,j) * (mm_i*M[i-1][j-1] + gapm_i*(I[i-1][j-1] + D[i-1][j-1]))
//   I[i][j] = mi_i*M[i-1][j] + ii_i*I[i-1][j]
//   D[i][j] = md_i*M[i][j-1] + dd_i*D[i][j-1]          (dd_i == ii_i == ph2pr[gcp_i])
// Row 0: M = I = 0, D = INITIAL_CONSTANT/haplen for every column
// (pairhmm_impl.cpp:62-69); column 0, rows >= 1: zero.  Result:
// sum over columns of M + I in the last read row (pairhmm_impl.cpp:413-438).
//
// Mapping.  One warp owns a work item.  Lane t holds R consecutive read rows
// of the current pass in registers and sweeps the haplotype columns; lane t
// runs one column behind lane t-1, so at step s lane t is at column
// j = s - t + 1.  The only cross-lane dependency, the row above the lane's
// first row, arrives by one __shfl_up_sync per state value per step: lane t-1
// computed exactly that cell (same column) one step earlier, and the diagonal
// cell is the previous step's value.  Lane 0's row above is the row-0
// boundary on the first pass and, on later passes of a long read, the last
// row of the previous pass, which lane 31 stored to a per-warp scratch buffer.
//
// Rows past the end of the read are "pass-through" rows: emission 0, so
// M = 0, and mi = ii = 1 (I = M_above + I_above), md = 0 (D stays 0).  The
// value M + I of the read's last row therefore travels unchanged to lane 31's
// last row, whose running column sum is the result; no lane needs to know
// which register holds the last row.
//
// Emission.  e(i,j) depends on the read base of row i and the haplotype base
// of column j.  Each lane keeps, in shared memory, a table E[code][k] of its
// rows' emissions for each of the five haplotype codes, laid out so that the
// per-step load of R values is a conflict-free 16-byte vector load per lane.
//
// Precision policies.  F32x2 packs two independent pairs into the two halves
// of the sm_100 f32x2 instructions (__ffma2_rn / __fadd2_rn / __fmul2_rn), so
// one warp instruction advances two DP cells.  F64 runs one pair per warp in
// double precision: it is the rescue pass for pairs whose FP32 result is below
// the reference's acceptance threshold (MIN_ACCEPTED 1e-28,
// pairhmm/intra/pairhmm_api.cpp:4-23, pairhmm_schedule.cpp:229-248).
//
// Uniform-gap form.  When a read's ins/del/gcp quals are constant (GATK data,
// and every benchmark config), the kernel stores M~ = M/gapm instead of M:
//   M~ = e*(mm*M~_d + I_d + D_d),  I = (mi*gapm)*M~_u + ii*I_u,
//   D = (md*gapm)*M~_l + dd*D_l
// which is 7 arithmetic instructions per cell instead of 8.  The result is
// gapm*sum(M~) + sum(I).
#pragma once
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "layout.h"

namespace rodv {

constexpr unsigned kFullMask = 0xffffffffu;
constexpr float kMinAcceptedF = 1e-28f;
// log10 offsets of the two scaling constants, spelled as the reference
// spells them (pairhmm/inter/pairhmm_inter_api.h:8-15): the FP32 one is a float
// literal, promoted to double for the FP64 log10 conversion.
constexpr double kLog10InitF = (double)36.1236000061f;
constexpr double kLog10InitD = 307.050595577260822;
constexpr double kDblMin = 2.2250738585072014e-308;  // smallest normal double

struct F32x2 {
  using V = float2;
  using S = float;
  static constexpr int kSlots = 2;
  static constexpr int kVec = 4;  // table entries per 16-byte load
  __device__ __forceinline__ static V add(V a, V b) { return __fadd2_rn(a, b); }
  __device__ __forceinline__ static V mul(V a, V b) { return __fmul2_rn(a, b); }
  __device__ __forceinline__ static V fma(V a, V b, V c) { return __ffma2_rn(a, b, c); }
  __device__ __forceinline__ static V zero() { return make_float2(0.f, 0.f); }
  __device__ __forceinline__ static V make(S x, S y) { return make_float2(x, y); }
  __device__ __forceinline__ static V shfl_up(V v) {
    return make_float2(__shfl_up_sync(kFullMask, v.x, 1), __shfl_up_sync(kFullMask, v.y, 1));
  }
  __device__ __forceinline__ static S sx(V v) { return v.x; }
  __device__ __forceinline__ static S sy(V v) { return v.y; }
  // 2^120, Context<float>::INITIAL_CONSTANT (context.h:141)
  __device__ __forceinline__ static S init_const() { return __int_as_float(0x7b800000); }
};

struct F64 {
  using V = double;
  using S = double;
  static constexpr int kSlots = 1;
  static constexpr int kVec = 2;
  __device__ __forceinline__ static V add(V a, V b) { return a + b; }
  __device__ __forceinline__ static V mul(V a, V b) { return a * b; }
  __device__ __forceinline__ static V fma(V a, V b, V c) { return __fma_rn(a, b, c); }
  __device__ __forceinline__ static V zero() { return 0.0; }
  __device__ __forceinline__ static V make(S x, S) { return x; }
  __device__ __forceinline__ static V shfl_up(V v) { return __shfl_up_sync(kFullMask, v, 1); }
  __device__ __forceinline__ static S sx(V v) { return v; }
  __device__ __forceinline__ static S sy(V v) { return v; }
  // 2^1020, Context<double>::INITIAL_CONSTANT (context.h:101)
  __device__ __forceinline__ static S init_const() { return __longlong_as_double(0x7fb0000000000000ll); }
};

template <class S>
struct Tables;
template <>
struct Tables<float> {
  __device__ __forceinline__ static const float* ph2pr(const PriorTables& t) { return t.ph2pr_f; }
  __device__ __forceinline__ static const float* mm(const PriorTables& t) { return t.mm_f; }
};
template <>
struct Tables<double> {
  __device__ __forceinline__ static const double* ph2pr(const PriorTables& t) { return t.ph2pr_d; }
  __device__ __forceinline__ static const double* mm(const PriorTables& t) { return t.mm_d; }
};

// Priors of one read row (pairhmm_impl.cpp:88-115, pairhmm_inter.cpp:83-98).
template <class S>
struct RowPriors {
  S mm, gapm, mi, ii, md, match, mismatch;
};

template <class S>
__device__ __forceinline__ RowPriors<S> row_priors(uint32_t w, const PriorTables& t) {
  const S* ph2pr = Tables<S>::ph2pr(t);
  const uint32_t q = rw_q(w), ins = rw_ins(w), del = rw_del(w), gcp = rw_gcp(w);
  RowPriors<S> p;
  const S dist = __ldg(ph2pr + q);
  p.match = S(1) - dist;
  p.mismatch = dist / S(3);
  const uint32_t lo = ins <= del ? ins : del, hi = ins <= del ? del : ins;
  p.mm = __ldg(Tables<S>::mm(t) + ((hi * (hi + 1)) >> 1) + lo);
  p.gapm = S(1) - __ldg(ph2pr + gcp);
  p.mi = __ldg(ph2pr + ins);
  p.ii = __ldg(ph2pr + gcp);
  p.md = __ldg(ph2pr + del);
  return p;
}

// Shared-memory bytes of one warp's emission tables for R rows per lane.
template <class P, int R>
struct TableShape {
  static constexpr int kRq = (R + P::kVec - 1) / P::kVec * P::kVec;   // rows, padded
  static constexpr int kNv = kRq / P::kVec;                          // 16-byte loads per slot
  static constexpr int kBytesPerWarp = P::kSlots * 5 * kRq * kWarp * (int)sizeof(typename P::S);
};

// Per-slot state of the pair being computed.
struct SlotInfo {
  const uint8_t* hap;   // first base code of the haplotype
  uint32_t H, L;
  uint64_t row_off;
  uint64_t out;
  uint32_t pair;
  bool valid;
};

template <class P, int R, bool UNIFORM, bool MULTI>
struct Forward {
  using V = typename P::V;
  using S = typename P::S;
  using Shape = TableShape<P, R>;
  static constexpr int kWarpsPerBlock = 4;

  // Boundary row written by lane 31 of one pass and read by lane 0 of the next.
  struct BoundaryCell {
    V m, i, d;
  };

  __device__ static void run_item(const BatchView& b, const ClassLaunch& c, uint32_t item,
                                  int lane, int gwarp, uint4* table) {
    SlotInfo sl[2];
    uint32_t pair_ids[2];
    if (P::kSlots == 2) {
      pair_ids[0] = c.work[2 * item];
      pair_ids[1] = c.work[2 * item + 1];
    } else {
      pair_ids[0] = c.work[item];
      pair_ids[1] = kNoPair;
    }
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const uint32_t pid = (s == 1 && pair_ids[1] == kNoPair) ? pair_ids[0] : pair_ids[s];
      const PairDesc pd = b.pairs[pid];
      const HapDesc hd = b.haps[pd.hap];
      const ReadDesc rd = b.reads[pd.read];
      sl[s].hap = b.hap_codes + hd.code_off;
      sl[s].H = hd.len;
      sl[s].L = rd.len;
      sl[s].row_off = rd.row_off;
      sl[s].out = pd.out;
      sl[s].pair = pid;
      sl[s].valid = (s == 0) || (pair_ids[1] != kNoPair);
    }
    const uint32_t Lmax = sl[0].L > sl[1].L ? sl[0].L : sl[1].L;
    const uint32_t passes = MULTI ? (Lmax + kWarp * R - 1) / (kWarp * R) : 1;
    if (sl[0].H == 0 || sl[1].H == 0 || sl[0].L == 0 || sl[1].L == 0 ||
        (!MULTI && Lmax > (uint32_t)(kWarp * R)) ||
        (MULTI && (uint64_t)sl[0].H + 40 > c.scratch_cols)) {
      if (lane == 0) atomicOr(c.error_flags, kErrBadLength);
      return;
    }
    const int nsteps = (int)sl[0].H + kWarp - 1;    // slot x has the longer haplotype
    const int nfreeze = (int)sl[1].H + kWarp - 1;   // slot y's last accumulated step + 1
    const V init = P::make(P::init_const() / (S)sl[0].H, P::init_const() / (S)sl[1].H);

    // Uniform-gap priors come from the read's first row.
    RowPriors<S> u0 = row_priors<S>(b.read_rows[sl[0].row_off], b.tab);
    RowPriors<S> u1 = row_priors<S>(b.read_rows[sl[1].row_off], b.tab);
    const V gapmU = P::make(u0.gapm, u1.gapm);
    const V mmU = P::make(u0.mm, u1.mm);
    const V mdU = P::make(u0.md * u0.gapm, u1.md * u1.gapm);
    const V ddU = P::make(u0.ii, u1.ii);

    BoundaryCell* buf = nullptr;
    if (MULTI) buf = reinterpret_cast<BoundaryCell*>(c.scratch) + (size_t)gwarp * c.scratch_cols;

    V acc_m = P::zero(), acc_i = P::zero();
    S frozen_m = 0, frozen_i = 0;

    for (uint32_t pass = 0; pass < passes; ++pass) {
      const bool last = (pass + 1 == passes);
      // ---- per-row priors and emission tables for this lane's R rows ----
      V pmm[UNIFORM ? 1 : R], pgapm[UNIFORM ? 1 : R], pmd[UNIFORM ? 1 : R];
      V pmi[R], pii[R];
      S* tab = reinterpret_cast<S*>(table);
#pragma unroll
      for (int k = 0; k < R; ++k) {
        const uint32_t row = pass * (kWarp * R) + lane * R + k;  // 0-based read row
        S mmv[2], gv[2], miv[2], iiv[2], mdv[2];
#pragma unroll
        for (int s = 0; s < P::kSlots; ++s) {
          const bool real = row < sl[s].L;
          const uint32_t w = real ? b.read_rows[sl[s].row_off + row] : 0u;
          const RowPriors<S> rp = row_priors<S>(w, b.tab);
          const uint32_t rc = rw_code(w);
#pragma unroll
          for (int code = 0; code < 5; ++code) {
            const bool hit = (rc == (uint32_t)code) || rc == kN || code == kN;
            const S e = real ? (hit ? rp.match : rp.mismatch) : S(0);
            // element (slot, code, k) of this lane's table
            const int idx = (((s * 5 + code) * Shape::kNv + k / P::kVec) * kWarp + lane) * P::kVec +
                            (k % P::kVec);
            tab[idx] = e;
          }
          if (UNIFORM) {
            const RowPriors<S>& up = (s == 0) ? u0 : u1;
            miv[s] = real ? up.mi * up.gapm : up.gapm;
            iiv[s] = real ? up.ii : S(1);
          } else {
            mmv[s] = real ? rp.mm : S(0);
            gv[s] = real ? rp.gapm : S(0);
            miv[s] = real ? rp.mi : S(1);
            iiv[s] = real ? rp.ii : S(1);
            mdv[s] = real ? rp.md : S(0);
          }
        }
        if (P::kSlots == 1) {
          miv[1] = miv[0]; iiv[1] = iiv[0];
          mmv[1] = mmv[0]; gv[1] = gv[0]; mdv[1] = mdv[0];
        }
        pmi[k] = P::make(miv[0], miv[1]);
        pii[k] = P::make(iiv[0], iiv[1]);
        if (!UNIFORM) {
          pmm[UNIFORM ? 0 : k] = P::make(mmv[0], mmv[1]);
          pgapm[UNIFORM ? 0 : k] = P::make(gv[0], gv[1]);
          pmd[UNIFORM ? 0 : k] = P::make(mdv[0], mdv[1]);
        }
      }

      // ---- sweep ----
      V M[R], I[R], D[R];
#pragma unroll
      for (int k = 0; k < R; ++k) M[k] = I[k] = D[k] = P::zero();
      V dg_m = P::zero(), dg_i = P::zero(), dg_d = P::zero();
      if (lane == 0 && pass == 0) dg_d = init;
      const V top_const_d = init;
      const uint4* tab_x = table + lane;
      const uint4* tab_y = table + 5 * Shape::kNv * kWarp + lane;
      const uint8_t* hx = sl[0].hap - lane;
      const uint8_t* hy = sl[1].hap - lane;

#pragma unroll 2
      for (int s = 0; s < nsteps; ++s) {
        V up_m = P::shfl_up(M[R - 1]);
        V up_i = P::shfl_up(I[R - 1]);
        V up_d = P::shfl_up(D[R - 1]);
        if (lane == 0) {
          if (MULTI && pass > 0) {
            const BoundaryCell cell = buf[s + 1];
            up_m = cell.m; up_i = cell.i; up_d = cell.d;
          } else {
            up_m = P::zero(); up_i = P::zero(); up_d = top_const_d;
          }
        }
        // emission values of this lane's rows for its current column
        S ex[Shape::kRq], ey[Shape::kRq];
        {
          const uint32_t cx = hx[s];
          const uint4* px = tab_x + cx * (Shape::kNv * kWarp);
#pragma unroll
          for (int v = 0; v < Shape::kNv; ++v) {
            const uint4 raw = px[v * kWarp];
            const S* f = reinterpret_cast<const S*>(&raw);
#pragma unroll
            for (int e = 0; e < P::kVec; ++e) ex[v * P::kVec + e] = f[e];
          }
          if (P::kSlots == 2) {
            const uint32_t cy = hy[s];
            const uint4* py = tab_y + cy * (Shape::kNv * kWarp);
#pragma unroll
            for (int v = 0; v < Shape::kNv; ++v) {
              const uint4 raw = py[v * kWarp];
              const S* f = reinterpret_cast<const S*>(&raw);
#pragma unroll
              for (int e = 0; e < P::kVec; ++e) ey[v * P::kVec + e] = f[e];
            }
          }
        }
        V dm = dg_m, di = dg_i, dd = dg_d, um = up_m, ui = up_i;
#pragma unroll
        for (int k = 0; k < R; ++k) {
          const V oM = M[k], oI = I[k], oD = D[k];
          V t = P::add(di, dd);
          if (UNIFORM) {
            t = P::fma(mmU, dm, t);
          } else {
            t = P::mul(pgapm[k], t);
            t = P::fma(pmm[k], dm, t);
          }
          if (P::kSlots == 2) {
            M[k] = P::make(P::sx(t) * ex[k], P::sy(t) * ey[k]);
          } else {
            M[k] = P::mul(t, P::make(ex[k], ex[k]));
          }
          I[k] = P::fma(pii[k], ui, P::mul(pmi[k], um));
          if (UNIFORM) {
            D[k] = P::fma(ddU, oD, P::mul(mdU, oM));
          } else {
            D[k] = P::fma(pii[k], oD, P::mul(pmd[k], oM));
          }
          dm = oM; di = oI; dd = oD;
          um = M[k]; ui = I[k];
        }
        dg_m = up_m; dg_i = up_i; dg_d = up_d;
        if (MULTI && !last && lane == kWarp - 1) {
          const int col = s - (kWarp - 1) + 1;
          if (col >= 1 && col <= (int)sl[0].H) {
            BoundaryCell cell;
            cell.m = M[R - 1]; cell.i = I[R - 1]; cell.d = D[R - 1];
            buf[col] = cell;
          }
        }
        if (last) {
          acc_m = P::add(acc_m, M[R - 1]);
          acc_i = P::add(acc_i, I[R - 1]);
          if (P::kSlots == 2 && s == nfreeze - 1) {
            frozen_m = P::sy(acc_m);
            frozen_i = P::sy(acc_i);
          }
        }
      }
      if (MULTI) __syncwarp();
    }

    if (lane != kWarp - 1) return;
    S res[2];
    res[0] = UNIFORM ? P::sx(gapmU) * P::sx(acc_m) + P::sx(acc_i) : P::sx(acc_m) + P::sx(acc_i);
    if (P::kSlots == 2)
      res[1] = UNIFORM ? P::sy(gapmU) * frozen_m + frozen_i : frozen_m + frozen_i;
#pragma unroll
    for (int s = 0; s < P::kSlots; ++s) {
      if (!sl[s].valid) continue;
      finish(b, c, sl[s], res[s]);
    }
  }

  __device__ static void finish(const BatchView& b, const ClassLaunch& c, const SlotInfo& sl,
                                S raw);
};

// FP32 result: accept at >= 1e-28 with an FP64 log10, else queue for FP64.
template <class P, int R, bool UNIFORM, bool MULTI>
__device__ void Forward<P, R, UNIFORM, MULTI>::finish(const BatchView& b, const ClassLaunch& c,
                                                      const SlotInfo& sl, S raw) {
  if (P::kSlots == 2) {
    if (raw >= kMinAcceptedF) {
      b.out[sl.out] = log10((double)raw) - kLog10InitF;
    } else {
      const uint32_t k = atomicAdd(c.rescue_count, 1u);
      c.rescue_list[k] = sl.pair;
    }
  } else {
    // The reference computes with flush-to-zero on (common.h:58-62), which on
    // x86 also flushes FP64 denormals: a likelihood below the normal FP64
    // range of the 2^1020 scaling becomes 0 and its log10 is -inf.  The GPU's
    // FP64 keeps denormals, so such a result is mapped to -inf here.
    b.out[sl.out] = (raw >= kDblMin) ? log10((double)raw) - kLog10InitD : -CUDART_INF;
  }
}

template <class P, int R, bool UNIFORM, bool MULTI>
__global__ void __launch_bounds__(Forward<P, R, UNIFORM, MULTI>::kWarpsPerBlock * kWarp)
    forward_kernel(BatchView b, ClassLaunch c) {
  using F = Forward<P, R, UNIFORM, MULTI>;
  extern __shared__ uint4 smem[];
  const int lane = threadIdx.x & (kWarp - 1);
  const int warp = threadIdx.x / kWarp;
  uint4* table = smem + warp * (TableShape<P, R>::kBytesPerWarp / 16);
  const int gwarp = blockIdx.x * F::kWarpsPerBlock + warp;
  const uint32_t n = c.work_count ? *c.work_count : c.static_count;
  for (;;) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(c.counter, 1u);
    item = __shfl_sync(kFullMask, item, 0);
    if (item >= n) break;
    F::run_item(b, c, item, lane, gwarp, table);
  }
}

}  // namespace rodv
