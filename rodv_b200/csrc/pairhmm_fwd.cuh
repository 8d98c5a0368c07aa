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
// value M + I of the read's last row therefore travels unchanged down to the
// last lane's last row, whose column sum is the result; no lane needs to know
// which register holds the last row.  Chain sweeps (run_chain) stack several
// read pairs down the lanes, each with its own first lane (row 0's boundary)
// and last lane; in the scaled form a pair's last row is a sum row whose D
// keeps that column sum.
//
// Emission.  e(i,j) depends on the read base of row i and the haplotype base
// of column j.  Each lane keeps, in shared memory, a table E[code][k] of its
// rows' emissions for each of the six haplotype codes (A, C, G, T, N and the
// separator between a chain's haplotypes), laid out so that the per-step
// loads are conflict-free 16-byte vector loads.
//
// Precision policies.  F32x2 packs two independent pairs into the two halves
// of the sm_100 f32x2 instructions (fma / add / mul .rn.f32x2), so
// one warp instruction advances two DP cells.  F64 runs one pair per warp in
// double precision: it is the rescue pass for pairs whose FP32 result is below
// the reference's acceptance threshold (MIN_ACCEPTED 1e-28,
// pairhmm/intra/pairhmm_api.cpp:4-23, pairhmm_schedule.cpp:229-248).
//
// Item shapes (F32x2).  SAME: both pairs share the haplotype (two reads of
// one region against one haplotype): one code load per step, the two slots'
// emissions interleaved in the table so that every row's pair of emissions is
// one f32x2 operand, and every FP32 instruction of the step is an f32x2
// instruction (a scalar FP32 instruction holds one half of the FMA pipe and
// stalls the next f32x2 one).  DIFF: any two pairs (the leftovers of SAME
// pairing); separate per-slot tables, scalar emission multiplies, and the
// shorter haplotype's running sum frozen when its last column has passed.
//
// Uniform-gap form.  When a read's ins/del/gcp quals are constant, ins == del
// and mi*gapm >= 1e-6 (GATK data, and every benchmark config), the kernels run
// the scaled 5-operation form (load_rows): M~ = M/gapm, I^ = I/c, D^ = D/c
// with c = mi*gapm folded into the emission table, 5 arithmetic instructions
// per cell instead of 8.
//
// MINB is the launch-bounds occupancy target (blocks per SM); it caps the
// registers per thread and is chosen per work class by the autotuner.
#pragma once
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "layout.h"

namespace rodv {

constexpr unsigned kFullMask = 0xffffffffu;
constexpr int kStepBlock = 8;  // chain sweeps: steps per block (unrolled)
constexpr float kMinAcceptedF = 1e-28f;
// log10 offsets of the two scaling constants, spelled as the reference
// spells them (pairhmm/inter/pairhmm_inter_api.h:8-15): the FP32 one is a float
// literal, promoted to double for the FP64 log10 conversion.
constexpr double kLog10InitF = (double)36.1236000061f;
constexpr double kLog10InitD = 307.050595577260822;
constexpr double kDblMin = 2.2250738585072014e-308;  // smallest normal double

// f32x2 arithmetic as PTX with an explicit .rn rounding modifier.  Results
// must not depend on the step at which a haplotype starts in a sweep (a chain
// item starts haplotypes at arbitrary steps of a 2-way unrolled loop), so the
// one product that is summed -- the last row's M into its running sum -- is
// accumulated with an explicit FMA on every step (acc = fma(t, e, acc)): a
// multiply followed by an add there was observed to be fused on only one of
// the two unrolled steps.
__device__ __forceinline__ unsigned long long f2_bits(float2 v) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(v.x), "f"(v.y));
  return r;
}
__device__ __forceinline__ float2 f2_value(unsigned long long r) {
  float2 v;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
  return v;
}

// cp.async of 8 bytes global -> shared (through L1), and its group controls.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned dst = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

struct F32x2 {
  using V = float2;
  using S = float;
  static constexpr int kSlots = 2;
  __device__ __forceinline__ static V add(V a, V b) {
    unsigned long long r;
    asm("add.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_bits(a)), "l"(f2_bits(b)));
    return f2_value(r);
  }
  __device__ __forceinline__ static V mul(V a, V b) {
    unsigned long long r;
    asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_bits(a)), "l"(f2_bits(b)));
    return f2_value(r);
  }
  __device__ __forceinline__ static V fma(V a, V b, V c) {
    unsigned long long r;
    asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;"
        : "=l"(r)
        : "l"(f2_bits(a)), "l"(f2_bits(b)), "l"(f2_bits(c)));
    return f2_value(r);
  }
  __device__ __forceinline__ static V zero() { return make_float2(0.f, 0.f); }
  __device__ __forceinline__ static V make(S x, S y) { return make_float2(x, y); }
  __device__ __forceinline__ static V shfl_up(V v) {
    // one 64-bit shuffle of the register pair (no moves to assemble the pair)
    return f2_value(__shfl_up_sync(kFullMask, f2_bits(v), 1));
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
  __device__ __forceinline__ static V add(V a, V b) { return a + b; }
  __device__ __forceinline__ static V mul(V a, V b) { return a * b; }
  __device__ __forceinline__ static V fma(V a, V b, V c) { return __fma_rn(a, b, c); }
  __device__ __forceinline__ static V zero() { return 0.0; }
  __device__ __forceinline__ static V make(S x, S) { return x; }
  __device__ __forceinline__ static V shfl_up(V v) { return __shfl_up_sync(kFullMask, v, 1); }
  __device__ __forceinline__ static S sx(V v) { return v; }
  __device__ __forceinline__ static S sy(V v) { return v; }
  // 2^1020, Context<double>::INITIAL_CONSTANT (context.h:101)
  __device__ __forceinline__ static S init_const() {
    return __longlong_as_double(0x7fb0000000000000ll);
  }
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

// Shared-memory shape of one warp's emission tables for R rows per lane
// (kNumCodes codes; the separator code's entries are all 0).
//   SAME layout (F64 always, F32x2 same-haplotype items): element (code, k)
//     is one 8-byte V.  Per code, R/2 blocks of 16-byte vectors holding rows
//     k, k+1 of each lane (vec index (code * kCodeVecs + k/2) * 32 + lane, in
//     16-byte units), then, for odd R, one block of 8-byte entries holding the
//     last row (byte offset code * kCodeBytes + (R/2) * 512 + lane * 8).  A
//     step loads R/2 16-byte vectors and, for odd R, one 8-byte entry: R * 8
//     bytes per lane, no padding row.  Both kinds of load are free of bank
//     conflicts whatever code each lane reads (kCodeBytes is a multiple of 128).
//   DIFF layout (F32x2 two-haplotype items): per slot, element (slot, code, k)
//     is one float; a 16-byte vector holds rows k..k+3 of the lane:
//     vec index (((slot * kNumCodes + code) * kNv + k/4) * 32 + lane).
template <class P, int R, bool SAME>
struct TableShape {
  static constexpr bool kSameLayout = SAME || P::kSlots == 1;
  static constexpr int kRowsPerVec = kSameLayout ? 2 : 4;
  static constexpr int kRq = (R + kRowsPerVec - 1) / kRowsPerVec * kRowsPerVec;
  static constexpr int kNv = kRq / kRowsPerVec;  // 16-byte loads per code (DIFF, per slot)
  static constexpr int kTables = kSameLayout ? 1 : 2;
  // SAME layout: paired-row vectors and the odd last row per code
  static constexpr int kPairVecs = R / 2;
  static constexpr bool kOddRow = (R % 2) != 0;
  static constexpr int kCodeBytes = kPairVecs * kWarp * 16 + (kOddRow ? kWarp * 8 : 0);
  static constexpr int kBytesPerWarp =
      kSameLayout ? kNumCodes * kCodeBytes : kTables * kNumCodes * kNv * kWarp * 16;
  static_assert(!kSameLayout || kCodeBytes % 128 == 0, "code blocks must start on bank 0");
};

// Per-slot state of the pair being computed.
struct SlotInfo {
  const uint8_t* hap;   // first base code of the haplotype
  uint32_t H, L;
  uint64_t row_off;
};

// Per-group shared memory of a chain sweep beyond the emission table: the
// column of the separator after each haplotype (the last one is the virtual
// separator just past the chain's end) and the region's read count (the
// stride of a read's results).  After the groups' ChainMeta a chain warp
// keeps 32 words: where each lane parks its pair's sums (run_chain).
struct ChainMeta {
  uint32_t sep[kChainHaps + 3];  // kChainHaps + 1 used
  uint32_t stride;
};

// GROUP: lanes per wavefront.  32 (the whole warp) for every kernel but the
// chain kernels of short reads, which split the warp into two 16-lane groups
// with twice the rows per lane, each sweeping its own chain item.
template <class P, int R, bool UNIFORM, bool MULTI, bool SAME, int MINB, int GROUP = 32>
struct Forward {
  using V = typename P::V;
  using S = typename P::S;
  using Shape = TableShape<P, R, SAME>;
  static constexpr bool kSameHap = Shape::kSameLayout;
  // Single-pass same-haplotype FP32 kernels take chain items.
  static constexpr bool kChain = SAME && !MULTI && P::kSlots == 2;
  static constexpr int kGroup = GROUP;
  static constexpr int kGroups = kWarp / GROUP;       // chain items per warp
  static constexpr int kGroupHaps = kChainHaps / kGroups;  // haplotypes per chain item
  static_assert(GROUP == 32 || kChain, "lane groups are for chain kernels only");
  // Kernels of the uniform-gap classes use the scaled 5-operation form
  // (reads of these classes have equal insertion and deletion quality), FP64
  // ones too.  The form keeps I and D at the reference's magnitude and M
  // mi times smaller (mi*gapm >= 1e-6 in these classes), so it reaches the
  // FP64 denormal range only for pairs whose likelihood is within that factor
  // of the 2^1020 scaling's underflow limit (log10 about -615, below which
  // the reference returns -inf); there M keeps at least 32 of its 52
  // mantissa bits (37 at ins = del = 45, gcp = 10), 1e-10 relative or better.
  static constexpr bool kScaled = UNIFORM;
  static constexpr int kWarpsPerBlock = 4;
  // Multi-pass kernels also keep a ring of 2 x 32 boundary cells per warp
  // (the next 32 columns of the previous pass's last row, see run_item).
  static constexpr int kRingCells = 2 * kWarp;
  static constexpr int kSmemPerWarp =
      Shape::kBytesPerWarp + (kChain ? kGroups * (int)sizeof(ChainMeta) + kWarp * 4 : 0) +
      (MULTI ? kRingCells * 3 * (int)sizeof(V) : 0);

  // Shuffles within a lane group (the row above comes from the previous lane
  // of the same group).
  __device__ __forceinline__ static V group_shfl_up(V v) {
    if constexpr (P::kSlots == 2) {
      return f2_value(__shfl_up_sync(kFullMask, f2_bits(v), 1, GROUP));
    } else {
      return P::shfl_up(v);
    }
  }

  // Boundary row written by lane 31 of one pass and read by lane 0 of the next.
  struct BoundaryCell {
    V m, i, d;
  };

  // Transition priors of this lane's R rows (per row, or the read's uniform
  // values), both slots packed.
  struct Priors {
    V mm[UNIFORM ? 1 : R], gapm[UNIFORM ? 1 : R], md[UNIFORM ? 1 : R];
    V mi[R], ii[R];
    V mmU, mdU, ddU;
    V iiN;  // kScaled: ii of the next lane's first row (the row below this lane's last)
  };

  // Writes emission e of (slot, code, row k) into this lane's table.
  __device__ __forceinline__ static void put_emission(S* tab, int slot, int code, int k, int lane,
                                                      S e) {
    if (kSameHap) {
      static_assert(sizeof(V) == 8, "SAME layout entries are 8 bytes");
      // V = S[kSlots]; a 16-byte vector holds 2 rows of V, an odd last row
      // sits in the code's 8-byte block
      const int byte = (k < 2 * Shape::kPairVecs)
                           ? code * Shape::kCodeBytes + ((k / 2) * kWarp + lane) * 16 + (k % 2) * 8
                           : code * Shape::kCodeBytes + Shape::kPairVecs * kWarp * 16 + lane * 8;
      tab[byte / (int)sizeof(S) + slot] = e;
    } else {
      const int vec = ((slot * kNumCodes + code) * Shape::kNv + k / 4) * kWarp + lane;
      tab[vec * 4 + (k % 4)] = e;
    }
  }

  // Emission tables and priors of this lane (table slot `lane`) for read rows
  // first_row[s] + [0, R) of the two slots s (reads of L[s] rows starting at
  // row word row_off[s]).
  // Rows past a read's end are pass-through rows: emission 0, mi = ii = 1,
  // md = 0 (in the uniform form mi*gapm = gapm, since M~ = M/gapm).
  //
  // Scaled form (kScaled; uniform gaps with mi == md).  With c = mi*gapm the
  // sweep keeps M~ = M/gapm, I^ = I/c, D^ = D/c of a DP whose row 0 holds
  // D = c*init, so that
  //   M~ = (e*c) * ((mm/c)*M~_d + I^_d + D^_d)
  //   I^ = ii*I^_u + M~_u
  //   D^ = dd*D^_l + M~_l
  // (5 operations per cell) and row 0 is D^ = init.  The first pass-through
  // row below the read's last row L takes ii = mi instead of 1, so it holds
  // mi*I^_L + M~_L = (M_L + I_L)/gapm, and the rows below it copy that value
  // down.  The likelihood term of a DP with row 0 = init is (M_L + I_L)/c, so
  // the result is (sum of that row)/mi when lane 31's last register is a
  // pass-through row, and sum(M~_L)/mi + sum(I^_L) when it is row L itself.
  // (Scaling row L by 1/mi instead would make the next row's (mm/c)*M~
  // overflow for likely pairs on short haplotypes.)
  // sum_lane (scaled form, chain sweeps): this lane's last row is a pair's
  // sum row, a pass-through row with emission 1 for every code (run_chain).
  __device__ __forceinline__ static void load_rows(const BatchView& b, const uint32_t (&L)[2],
                                                   const uint64_t (&row_off)[2],
                                                   const uint32_t (&first_row)[2], int lane,
                                                   uint4* table, Priors& p,
                                                   bool sum_lane = false) {
    RowPriors<S> u[2];
    S cs[2] = {S(1), S(1)};  // emission scale of rows before the last (kScaled)
    if (UNIFORM) {  // uniform-gap priors come from the read's first row
      u[0] = row_priors<S>(b.read_rows[row_off[0]], b.tab);
      u[1] = row_priors<S>(b.read_rows[row_off[1]], b.tab);
      if (kScaled) {
        cs[0] = u[0].mi * u[0].gapm;
        cs[1] = u[1].mi * u[1].gapm;
        p.mmU = P::make(u[0].mm / cs[0], u[1].mm / cs[1]);
      } else {
        p.mmU = P::make(u[0].mm, u[1].mm);
        p.mdU = P::make(u[0].md * u[0].gapm, u[1].md * u[1].gapm);
      }
      p.ddU = P::make(u[0].ii, u[1].ii);
    }
    S* tab = reinterpret_cast<S*>(table);
#pragma unroll
    for (int k = 0; k < R; ++k) {
      S mmv[2], gv[2], miv[2], iiv[2], mdv[2];
#pragma unroll
      for (int s = 0; s < P::kSlots; ++s) {
        const uint32_t row = first_row[s] + k;  // 0-based read row
        const bool real = row < L[s];
        const uint32_t w = real ? b.read_rows[row_off[s] + row] : 0u;
        const RowPriors<S> rp = row_priors<S>(w, b.tab);
        const uint32_t rc = rw_code(w);
        const S scale = kScaled ? cs[s] : S(1);
#pragma unroll
        for (int code = 0; code < kN + 1; ++code) {
          const bool hit = (rc == (uint32_t)code) || rc == kN || code == kN;
          const S e = hit ? rp.match : rp.mismatch;
          put_emission(tab, s, code, k, lane, real ? (kScaled ? e * scale : e) : S(0));
        }
        put_emission(tab, s, kSep, k, lane, S(0));
        if (kScaled) {
          iiv[s] = real ? u[s].ii : (row == L[s] ? u[s].mi : S(1));
        } else if (UNIFORM) {
          miv[s] = real ? u[s].mi * u[s].gapm : u[s].gapm;
          iiv[s] = real ? u[s].ii : S(1);
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
      p.mi[k] = P::make(miv[0], miv[1]);
      p.ii[k] = P::make(iiv[0], iiv[1]);
      if (!UNIFORM) {
        p.mm[UNIFORM ? 0 : k] = P::make(mmv[0], mmv[1]);
        p.gapm[UNIFORM ? 0 : k] = P::make(gv[0], gv[1]);
        p.md[UNIFORM ? 0 : k] = P::make(mdv[0], mdv[1]);
      }
    }
    if (kScaled && sum_lane) {
#pragma unroll
      for (int s = 0; s < P::kSlots; ++s)
#pragma unroll
        for (int code = 0; code < kNumCodes; ++code) put_emission(tab, s, code, R - 1, lane, S(1));
    }
    if (kScaled) {
      S iin[2];
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const uint32_t row = first_row[s] + R;
        iin[s] = row < L[s] ? u[s].ii : (row == L[s] ? u[s].mi : S(1));
      }
      p.iiN = P::make(iin[0], iin[1]);
    }
  }

  // Emission values of this lane's rows for haplotype codes cx (slot x) and
  // cy (slot y; used by the DIFF layout only).
  __device__ __forceinline__ static void load_emission(const uint4* table, int lane, uint32_t cx,
                                                       uint32_t cy, V (&e)[R]) {
    if (kSameHap) {
      const uint8_t* base = reinterpret_cast<const uint8_t*>(table) + cx * Shape::kCodeBytes;
      const uint4* px = reinterpret_cast<const uint4*>(base) + lane;
#pragma unroll
      for (int v = 0; v < Shape::kPairVecs; ++v) {
        const uint4 raw = px[v * kWarp];
        const V* f = reinterpret_cast<const V*>(&raw);
        e[2 * v] = f[0];
        e[2 * v + 1] = f[1];
      }
      if constexpr (Shape::kOddRow) {
        const uint2 raw =
            reinterpret_cast<const uint2*>(base + Shape::kPairVecs * kWarp * 16)[lane];
        e[R - 1] = *reinterpret_cast<const V*>(&raw);
      }
    } else {
      S ex[Shape::kRq], ey[Shape::kRq];
      const uint4* px = table + lane + cx * (Shape::kNv * kWarp);
      const uint4* py = table + kNumCodes * Shape::kNv * kWarp + lane + cy * (Shape::kNv * kWarp);
#pragma unroll
      for (int v = 0; v < Shape::kNv; ++v) {
        const uint4 rx = px[v * kWarp], ry = py[v * kWarp];
        const S* fx = reinterpret_cast<const S*>(&rx);
        const S* fy = reinterpret_cast<const S*>(&ry);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          ex[v * 4 + q] = fx[q];
          ey[v * 4 + q] = fy[q];
        }
      }
#pragma unroll
      for (int k = 0; k < R; ++k) e[k] = P::make(ex[k], ey[k]);
    }
  }

  // One column of this lane's R rows.  (M, I, D)[k] hold the previous
  // column on entry (the left neighbours) and this column on exit; dg is the
  // row above the lane's first row at the previous column, up the same row
  // at this column.  t_last: the last row's M before the emission multiply
  // (M[R-1] = t_last * e[R-1]), for the running sum of the last row.
  __device__ __forceinline__ static void cells(const V (&e)[R], V up_m, V up_i, V up_d, V& dg_m,
                                               V& dg_i, V& dg_d, V (&M)[R], V (&I)[R], V (&D)[R],
                                               const Priors& p, V& t_last) {
    V dm = dg_m, di = dg_i, dd = dg_d, um = up_m, ui = up_i;
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const V oM = M[k], oI = I[k], oD = D[k];
      V t = P::add(di, dd);
      if (UNIFORM) {
        t = P::fma(p.mmU, dm, t);
      } else {
        t = P::mul(p.gapm[k], t);
        t = P::fma(p.mm[k], dm, t);
      }
      if (kSameHap) {
        M[k] = P::mul(t, e[k]);
      } else {
        M[k] = P::make(P::sx(t) * P::sx(e[k]), P::sy(t) * P::sy(e[k]));
      }
      if (k == R - 1) t_last = t;
      if (kScaled) {
        I[k] = P::fma(p.ii[k], ui, um);
        D[k] = P::fma(p.ddU, oD, oM);
      } else {
        I[k] = P::fma(p.ii[k], ui, P::mul(p.mi[k], um));
        if (UNIFORM) {
          D[k] = P::fma(p.ddU, oD, P::mul(p.mdU, oM));
        } else {
          D[k] = P::fma(p.ii[k], oD, P::mul(p.md[k], oM));
        }
      }
      dm = oM; di = oI; dd = oD;
      um = M[k]; ui = I[k];
    }
    dg_m = up_m; dg_i = up_i; dg_d = up_d;
  }

  // cells() of the scaled form with the row above the lane's first row
  // folded by the lane above (run_chain): t0 is the first row's M term
  // (mm/c)*M~_d + I^_d + D^_d and i0 its I^, both computed by the lane above
  // with the same operations cells() would apply here, so the results are
  // bitwise the same while the lanes exchange two values a step instead of
  // three.  D takes each row's ii: the read's dd on its rows (uniform gaps:
  // ii == dd, the value cells() uses), and 1 on pass-through rows below row
  // L, where M is 0 and D stays 0 -- except on a chain sweep's sum row, whose
  // emission 1 makes its M the pass-through value one column back and its D
  // the exact running sum of the earlier ones (run_chain).
  __device__ __forceinline__ static void cells_scaled(const V (&e)[R], V t0, V i0, V (&M)[R],
                                                      V (&I)[R], V (&D)[R], const Priors& p,
                                                      V& t_last) {
    V dm = P::zero(), di = P::zero(), dd = P::zero(), um = P::zero(), ui = P::zero();
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const V oM = M[k], oI = I[k], oD = D[k];
      const V t = k == 0 ? t0 : P::fma(p.mmU, dm, P::add(di, dd));
      M[k] = P::mul(t, e[k]);
      if (k == R - 1) t_last = t;
      I[k] = k == 0 ? i0 : P::fma(p.ii[k], ui, um);
      D[k] = P::fma(p.ii[k], oD, oM);
      dm = oM; di = oI; dd = oD;
      um = M[k]; ui = I[k];
    }
  }

  // The two pairs of work item `item` (the second one's read is kNoPair when
  // the item holds one pair).
  __device__ __forceinline__ static void load_refs(const ClassLaunch& c, uint32_t item,
                                                   PairRef refs[2]) {
    if (P::kSlots == 1) {
      refs[0] = static_cast<const PairRef*>(c.work)[item];
      refs[1] = refs[0];
      refs[1].read = kNoPair;
    } else if (SAME) {
      const SameItem it = static_cast<const SameItem*>(c.work)[item];
      refs[0] = PairRef{it.hap, it.read_x, it.out_x};
      refs[1] = PairRef{it.hap, it.read_y, it.out_x + (it.read_y - it.read_x)};
    } else {
      const DiffItem it = static_cast<const DiffItem*>(c.work)[item];
      refs[0] = it.x;
      refs[1] = it.y;
    }
  }

  // gapm of a uniform-gap read (every row has the same gcp quality).
  __device__ __forceinline__ static S uniform_gapm(const BatchView& b, uint32_t read) {
    const uint32_t w = b.read_rows[b.reads[read].row_off];
    return S(1) - __ldg(Tables<S>::ph2pr(b.tab) + rw_gcp(w));
  }

  // The scaled form's likelihood from the last register's column sums of
  // M~ (acc_m) and I^ (acc_i); rows: the rows the sweep held for the read.
  // accept_min: the FP32 acceptance bound for it.  The scaled sweep keeps M
  // about c = mi*gapm times smaller than the reference's FP32 sweep, so its
  // bound is 1e-28/c: an accepted result keeps the reference's headroom above
  // the FP32 denormal range (below the bound, the pair goes to FP64).
  __device__ __forceinline__ static double scaled_result(const BatchView& b, uint32_t read,
                                                         uint32_t len, uint32_t rows, S acc_m,
                                                         S acc_i, double* accept_min) {
    const uint32_t w = b.read_rows[b.reads[read].row_off];
    const double mi = (double)__ldg(Tables<S>::ph2pr(b.tab) + rw_ins(w));
    const double gapm = 1.0 - (double)__ldg(Tables<S>::ph2pr(b.tab) + rw_gcp(w));
    *accept_min = (double)kMinAcceptedF / (mi * gapm);
    return len < rows ? (double)acc_i / mi : (double)acc_m / mi + (double)acc_i;
  }

  // Early end of an FP32 multi-pass sweep.  Every alignment emits read row r
  // from M or I at some column, and the transition and emission factors of
  // the rest of a path are <= 1, so a pair's likelihood is at most
  // sum_j (M + I)[r][j] for any row r.  After each pass but the last, the
  // warp sums the boundary row (the pass's last row, kept for the next pass)
  // and decides per slot whether that bound is below the FP32 acceptance
  // bound, with a 1e-6 margin for the rounding of the remaining rows.  Such a
  // pair is rejected at the end of the sweep whatever the remaining passes
  // compute, so when both slots are decided the sweep stops and queues them
  // for FP64 now: the same pairs reach FP64 and every result is unchanged.
  // `row`: 0-based read row of the boundary; H: the slots' haplotype lengths.
  __device__ static bool sweep_rejected(const BatchView& b, const ClassLaunch& c,
                                        const BoundaryCell* buf, const uint32_t (&H)[2],
                                        const uint32_t (&L)[2], uint32_t row, int lane,
                                        uint32_t item) {
    const bool rejected = row_bound_rejects(b, c, buf, H, L, row, lane, item);
    if (rejected && lane == 0) {
      PairRef refs[2];
      load_refs(c, item, refs);
      finish(b, c, refs[0], 0.0);
      if (refs[1].read != kNoPair) finish(b, c, refs[1], 0.0);
    }
    return rejected;
  }

  // The decision of sweep_rejected, taken by the whole warp (the same value
  // in every lane); nothing is written.
  __device__ static bool row_bound_rejects(const BatchView& b, const ClassLaunch& c,
                                           const BoundaryCell* buf, const uint32_t (&H)[2],
                                           const uint32_t (&L)[2], uint32_t row, int lane,
                                           uint32_t item) {
    V sm = P::zero(), si = P::zero();
    for (uint32_t col = 1 + (uint32_t)lane; col <= H[0]; col += kWarp) {
      const BoundaryCell cell = buf[col];
      const bool y_in = col <= H[1];
      sm = P::add(sm, P::make(P::sx(cell.m), y_in ? P::sy(cell.m) : S(0)));
      si = P::add(si, P::make(P::sx(cell.i), y_in ? P::sy(cell.i) : S(0)));
    }
    double sum_m[2] = {(double)P::sx(sm), (double)P::sy(sm)};
    double sum_i[2] = {(double)P::sx(si), (double)P::sy(si)};
#pragma unroll
    for (int d = 16; d >= 1; d /= 2) {
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        sum_m[s] += __shfl_xor_sync(kFullMask, sum_m[s], d);
        sum_i[s] += __shfl_xor_sync(kFullMask, sum_i[s], d);
      }
    }
    PairRef refs[2];
    load_refs(c, item, refs);
    bool rejected = true;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      if (s == 1 && refs[1].read == kNoPair) continue;
      const uint32_t w = b.read_rows[b.reads[refs[s].read].row_off];
      const double mi = (double)__ldg(Tables<S>::ph2pr(b.tab) + rw_ins(w));
      const double gapm = 1.0 - (double)__ldg(Tables<S>::ph2pr(b.tab) + rw_gcp(w));
      double bound, amin = (double)kMinAcceptedF;
      if (kScaled) {
        // M~ = mi * M and I^ = I; a pass-through row holds mi * (M_L + I_L) in I^
        bound = row < L[s] ? sum_m[s] / mi + sum_i[s] : sum_i[s] / mi;
        amin /= mi * gapm;
      } else if (UNIFORM) {
        bound = gapm * sum_m[s] + sum_i[s];  // M is kept divided by gapm
      } else {
        bound = sum_m[s] + sum_i[s];
      }
      rejected = rejected && bound >= 0.0 && bound < amin * 1e-6;
    }
    return rejected;
  }

  // One pair per slot (SameItem, DiffItem or, for F64, PairRef), swept in one
  // or (MULTI) several passes of 32R rows.
  __device__ static void run_item(const BatchView& b, const ClassLaunch& c, uint32_t item,
                                  int lane, int gwarp, uint4* table) {
    PairRef refs[2];
    load_refs(c, item, refs);
    SlotInfo sl[2];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const bool valid = (s == 0) || refs[1].read != kNoPair;
      const PairRef r = valid ? refs[s] : refs[0];
      const HapDesc hd = b.haps[r.hap];
      const ReadDesc rd = b.reads[r.read];
      sl[s].hap = b.hap_codes + hd.code_off;
      sl[s].H = hd.len;
      sl[s].L = rd.len;
      sl[s].row_off = rd.row_off;
    }
    const uint32_t Lmax = sl[0].L > sl[1].L ? sl[0].L : sl[1].L;
    // (pipe_passes: the last pass ends in pass-through rows, as in the
    // pipelined sweep, so both give the same results)
    const uint32_t passes = MULTI ? pipe_passes(Lmax, R) : 1;
    if (sl[0].H == 0 || sl[1].H == 0 || sl[0].L == 0 || sl[1].L == 0 ||
        (kSameHap && sl[0].hap != sl[1].hap) || (!MULTI && Lmax > (uint32_t)(kWarp * R)) ||
        (MULTI && (uint64_t)sl[0].H + 40 > c.scratch_cols)) {
      if (lane == 0) atomicOr(c.error_flags, kErrBadLength);
      return;
    }
    const int nsteps = (int)sl[0].H + kWarp - 1;    // slot x has the longer haplotype
    const int nfreeze = (int)sl[1].H + kWarp - 1;   // slot y's last accumulated step + 1
    const V init = P::make(P::init_const() / (S)sl[0].H, P::init_const() / (S)sl[1].H);
    const uint32_t L[2] = {sl[0].L, sl[1].L};
    const uint64_t row_off[2] = {sl[0].row_off, sl[1].row_off};

    BoundaryCell* buf = nullptr;
    if (MULTI) buf = reinterpret_cast<BoundaryCell*>(c.scratch) + (size_t)gwarp * c.scratch_cols;
    // Lane 0 of a pass after the first takes the row above from the previous
    // pass's boundary row in scratch, one cell per step.  Read from global
    // memory at each step, that load's latency sat on every step's critical
    // path; instead the warp copies the cells of the next 32 steps into a
    // shared-memory ring with cp.async (one cell per lane, coalesced) while it
    // computes the current 32, and lane 0 reads the ring.  Copies stop at the
    // warp's scratch_cols (cells past the last step's are never read).
    BoundaryCell* ring = reinterpret_cast<BoundaryCell*>(table + Shape::kBytesPerWarp / 16);
    auto fetch_chunk = [&](int chunk) {  // cells of steps [32 chunk, 32 chunk + 32)
      const uint32_t idx = (uint32_t)chunk * kWarp + 1u + (uint32_t)lane;
      if (idx < c.scratch_cols) {
        BoundaryCell* dst = ring + (chunk & 1) * kWarp + lane;
        const BoundaryCell* src = buf + idx;
        cp_async8(&dst->m, &src->m);
        cp_async8(&dst->i, &src->i);
        cp_async8(&dst->d, &src->d);
      }
      cp_async_commit();
    };

    V acc_m = P::zero(), acc_i = P::zero();
    S frozen_m = 0, frozen_i = 0;

    for (uint32_t pass = 0; pass < passes; ++pass) {
      const bool last = (pass + 1 == passes);
      Priors pr;
      const uint32_t fr = pass * (kWarp * R) + lane * R;
      load_rows(b, L, row_off, {fr, fr}, lane, table, pr);

      V M[R], I[R], D[R];
#pragma unroll
      for (int k = 0; k < R; ++k) M[k] = I[k] = D[k] = P::zero();
      V dg_m = P::zero(), dg_i = P::zero(), dg_d = P::zero();
      if (lane == 0 && pass == 0) dg_d = init;
      const uint8_t* hx = sl[0].hap - lane;
      const uint8_t* hy = sl[1].hap - lane;
      const bool from_ring = MULTI && pass > 0;
      if (from_ring) fetch_chunk(0);
      // codes of the next step loaded one step ahead (the emission loads wait
      // on them); the last step's read lands one byte further into the code
      // array's tail padding
      uint32_t cx_next = hx[0], cy_next = kSameHap ? 0u : (uint32_t)hy[0];

#pragma unroll 4
      for (int s = 0; s < nsteps; ++s) {
        const uint32_t cx = cx_next, cy = cy_next;
        cx_next = hx[s + 1];
        if (!kSameHap) cy_next = hy[s + 1];
        if (from_ring && (s & (kWarp - 1)) == 0) {
          cp_async_wait_all();  // this chunk's cells
          __syncwarp();
          fetch_chunk(s / kWarp + 1);
        }
        V up_m = P::shfl_up(M[R - 1]);
        V up_i = P::shfl_up(I[R - 1]);
        V up_d = P::shfl_up(D[R - 1]);
        if (lane == 0) {
          if (from_ring) {
            const BoundaryCell cell = ring[((s / kWarp) & 1) * kWarp + (s & (kWarp - 1))];
            up_m = cell.m; up_i = cell.i; up_d = cell.d;
          } else {
            up_m = P::zero(); up_i = P::zero(); up_d = init;
          }
        }
        V e[R], t_last;
        load_emission(table, lane, cx, cy, e);
        cells(e, up_m, up_i, up_d, dg_m, dg_i, dg_d, M, I, D, pr, t_last);
        if (MULTI && !last && lane == kWarp - 1) {
          const int col = s - (kWarp - 1) + 1;
          if (col >= 1 && col <= (int)sl[0].H) {
            BoundaryCell cell;
            cell.m = M[R - 1]; cell.i = I[R - 1]; cell.d = D[R - 1];
            buf[col] = cell;
          }
        }
        if (last) {
          acc_m = P::fma(t_last, e[R - 1], acc_m);  // += M[R-1], one rounding
          acc_i = P::add(acc_i, I[R - 1]);
          if (P::kSlots == 2 && !kSameHap && s == nfreeze - 1) {
            frozen_m = P::sy(acc_m);
            frozen_i = P::sy(acc_i);
          }
        }
      }
      if (MULTI) {
        cp_async_wait_all();  // the prefetch past the last step lands before the ring is reused
        __syncwarp();
      }
      if constexpr (MULTI && P::kSlots == 2) {
        const uint32_t H[2] = {sl[0].H, sl[1].H};
        if (!last && sweep_rejected(b, c, buf, H, L, (pass + 1) * (kWarp * R) - 1, lane, item))
          return;
      }
    }

    if (lane != kWarp - 1) return;
    if (P::kSlots == 2 && kSameHap) {  // both slots ran exactly their own columns
      frozen_m = P::sy(acc_m);
      frozen_i = P::sy(acc_i);
    }
    // Values needed only now are re-read rather than kept live in registers
    // through the sweep.
    PairRef fr[2];
    load_refs(c, item, fr);
    const bool valid_y = P::kSlots == 2 && fr[1].read != kNoPair;
    double res[2] = {0.0, 0.0};
    double amin[2] = {(double)kMinAcceptedF, (double)kMinAcceptedF};
    if (kScaled) {
      const uint32_t rows = passes * kWarp * R;
      res[0] = scaled_result(b, fr[0].read, L[0], rows, P::sx(acc_m), P::sx(acc_i), &amin[0]);
      if (valid_y)
        res[1] = scaled_result(b, fr[1].read, L[1], rows, frozen_m, frozen_i, &amin[1]);
    } else if (UNIFORM) {
      res[0] = uniform_gapm(b, fr[0].read) * P::sx(acc_m) + P::sx(acc_i);
      if (valid_y) res[1] = uniform_gapm(b, fr[1].read) * frozen_m + frozen_i;
    } else {
      res[0] = P::sx(acc_m) + P::sx(acc_i);
      res[1] = frozen_m + frozen_i;
    }
    finish(b, c, fr[0], res[0], amin[0]);
    if (valid_y) finish(b, c, fr[1], res[1], amin[1]);
  }

  // A chain item: reads x and y against haplotypes hap_start .. +num_haps-1,
  // swept as one column sequence h0 sep h1 sep ... (the packed layout of
  // consecutive haplotypes).  Each lane crosses a separator one step after
  // its left neighbour; the separator column is the next haplotype's
  // column 0:
  //   M = 0 there (its emission is 0 for every row),
  //   I = 0 there (the column above it is 0 down from row 0),
  //   D is set to 0 by the lane after it computes the separator column.
  // So every haplotype sees the reference's column-0 boundary, and the
  // wavefront fills and drains once per chain instead of once per pair.  A
  // virtual separator just past the chain's last haplotype (the packed layout
  // has a separator code after every haplotype) ends the last haplotype's
  // sums the same way, so the two lane groups of a short-read warp can sweep
  // chains of different lengths in the same loop.
  // Row 0 uses one scaling constant for the whole chain, 2^120/norm_len
  // (norm_len: the region's longest haplotype, so no value exceeds the
  // reference's); the DP is linear in it, so haplotype i's result is
  // rescaled by (2^120/H_i)/(2^120/norm_len) in FP64 before the acceptance
  // test and log10.
  // `first`: the first chain item of this warp's lane groups (group g takes
  // item first + g); `count`: how many items exist (a group without one
  // repeats the first and writes nothing).
  //
  // Read pairs: lane e of a group fetches pair e, a scan of the pairs' lane
  // counts gives each pair's first lane, and every lane then takes the pair
  // covering it (lanes past the last pair extend its pass-through rows).  A
  // lane's lag, its distance from its pair's first lane, is the step at which
  // it reaches the chain's first column: a pair's first lane takes row 0's
  // boundary from step 0, as lane 0 of a one-pair item does, and its last
  // lane, whose last row is a pass-through row, parks the pair's sums.
  __device__ static void run_chain(const BatchView& b, const ClassLaunch& c, uint32_t first,
                                   uint32_t count, int lane, uint4* table) {
    const int grp = lane / GROUP;            // lane group
    const int gl = lane & (GROUP - 1);       // lane within its group
    const bool active = first + (uint32_t)grp < count;
    ChainMeta* const metas = reinterpret_cast<ChainMeta*>(table + Shape::kBytesPerWarp / 16);
    ChainMeta* meta = metas + grp;
    // per lane of the warp: the out index of (the item's first haplotype,
    // the x read) where the lane parks its pair's sums, else kNoStore
    uint32_t* park = reinterpret_cast<uint32_t*>(metas + kGroups);
    constexpr uint32_t kNoStore = 0xffffffffu;
    const ChainItem* item_ptr =
        static_cast<const ChainItem*>(c.work) + first + (active ? (uint32_t)grp : 0u);
    const ChainItem it = *item_ptr;
    const uint32_t n = it.num_haps;
    // lane gl of a group holds haplotype gl's length and code offset
    uint32_t hl = 0;
    uint64_t co = 0;
    if ((uint32_t)gl < n && n <= (uint32_t)kGroupHaps) {
      const HapDesc hd = b.haps[it.hap_start + gl];
      hl = hd.len;
      co = hd.code_off;
    }
    const uint64_t co_next = __shfl_down_sync(kFullMask, co, 1, GROUP);
    const bool bad_counts = n == 0 || n > (uint32_t)kGroupHaps || it.pairs == 0 ||
                            it.pairs > (uint32_t)GROUP;
    bool bad = bad_counts || ((uint32_t)gl < n && (hl == 0 || hl > it.norm_len ||
                                                   ((uint32_t)gl + 1 < n && co_next != co + hl + 1)));
    // pair e at lane e: its reads and lanes
    const bool holder = !bad_counts && (uint32_t)gl < it.pairs;
    const uint32_t hrx = holder ? c.stack[it.stack + 2u * gl] : 0u;
    const uint32_t hry = holder ? c.stack[it.stack + 2u * gl + 1u] : kNoPair;
    const uint32_t lx = holder ? b.reads[hrx].len : 0u;
    const uint32_t ly = (holder && hry != kNoPair) ? b.reads[hry].len : 0u;
    bad = bad || (holder && (lx == 0 || (hry != kNoPair && ly == 0)));
    // rows of a pair: its longer read's, a pass-through row and, in the
    // scaled form, the sum row
    const uint32_t hlanes = holder ? (max(lx, ly) + (kScaled ? 1u : 0u)) / R + 1 : 0u;
    uint32_t end = hlanes;  // lanes of pairs 0..gl
#pragma unroll
    for (int d = 1; d < GROUP; d *= 2) {
      const uint32_t v = __shfl_up_sync(kFullMask, end, d, GROUP);
      if (gl >= d) end += v;
    }
    const uint32_t hstart = end - hlanes;
    bad = bad || __shfl_sync(kFullMask, end, GROUP - 1, GROUP) > (uint32_t)GROUP;
    if (__any_sync(kFullMask, bad)) {
      if (lane == 0) atomicOr(c.error_flags, kErrChain);
      return;
    }
    // the pair covering this lane
    const uint32_t starts =
        __reduce_or_sync(kFullMask, holder ? 1u << (hstart + (uint32_t)(grp * GROUP)) : 0u) >>
        (grp * GROUP);
    const int e = __popc(starts & ((2u << gl) - 1u)) - 1;
    const uint32_t rx = __shfl_sync(kFullMask, hrx, e, GROUP);
    const uint32_t ry0 = __shfl_sync(kFullMask, hry, e, GROUP);
    const uint32_t st = __shfl_sync(kFullMask, hstart, e, GROUP);
    const uint32_t nl = __shfl_sync(kFullMask, hlanes, e, GROUP);
    const int lag = gl - (int)st;
    // steps past the longer chain's last column for every pair's last lane
    // to reach its virtual end separator
    const uint32_t maxnl = __reduce_max_sync(kFullMask, hlanes);
    const uint32_t ry = ry0 != kNoPair ? ry0 : rx;  // no y read: x again, not stored
    const bool parks = active && (uint32_t)lag == nl - 1;
    park[lane] = parks ? it.out0 + (rx - it.read_base) : kNoStore;
    if (gl == 0) meta->stride = it.stride;
    const ReadDesc dx = b.reads[rx], dy = b.reads[ry];
    const uint32_t L[2] = {dx.len, dy.len};
    const uint64_t row_off[2] = {dx.row_off, dy.row_off};
    // end column (exclusive) + 1 of haplotype gl in the chain's columns
    uint32_t endc = (uint32_t)gl < n ? hl + 1 : 0;
#pragma unroll
    for (int d = 1; d < GROUP; d *= 2) {
      const uint32_t v = __shfl_up_sync(kFullMask, endc, d, GROUP);
      if (gl >= d) endc += v;
    }
    constexpr uint32_t kNever = 0x40000000u;  // beyond every chain's last step
    // separator after haplotype gl (the last one: the virtual end separator)
    meta->sep[gl] = ((uint32_t)gl < n) ? endc - 1 : kNever;  // kGroupHaps == GROUP
    if (gl == 0) meta->sep[kGroupHaps] = kNever;
    const uint32_t ncols = __shfl_sync(kFullMask, endc, (int)n - 1, GROUP) - 1;  // sum H + n - 1
    uint32_t span = ncols;  // columns of the longer chain of the warp
    if (kGroups > 1) span = max(span, __shfl_xor_sync(kFullMask, span, GROUP));
    const uint64_t co0 = __shfl_sync(kFullMask, co, 0, GROUP);
    const S init_s = P::init_const() / (S)it.norm_len;
    const V init = P::make(init_s, init_s);
    Priors pr;
    const uint32_t fr = (uint32_t)lag * R;  // this lane's first row in its pair's reads
    load_rows(b, L, row_off, {fr, fr}, lane, table, pr, (uint32_t)lag == nl - 1);
    __syncwarp();

    const bool top = lag == 0;  // a pair's first lane
    V M[R], I[R], D[R];
#pragma unroll
    for (int k = 0; k < R; ++k) M[k] = I[k] = D[k] = P::zero();
    V dg_m = P::zero(), dg_i = P::zero(), dg_d = P::zero();
    if (top) dg_d = init;
    // scaled form: the first row's M term of the previous column (row 0 of
    // the DP, D^ = init, for a pair's first lane)
    V dg_t = top ? init : P::zero();
    // column s - lag at step s
    const uint8_t* hx = b.hap_codes + co0 - lag;
    uint32_t hi = 0;                          // this lane's haplotype in the chain
    int nxt = (int)meta->sep[0] + lag;        // step at which this lane is at the next separator
    // A pair's lanes hold its reads' rows and at least one pass-through row
    // below each: the first (row L) holds the value whose sum over a
    // haplotype's columns gives the result, and the rows below copy it down.
    // Scaled form: the last lane's last row (the sum row) has emission 1, so
    // its M is that value one column back and its D (dd = 1) the exact
    // running sum of the earlier columns: D + M at a separator column is the
    // sum, with no add per step.  Per-row form: a running sum of I of the last
    // row (acc_i).
    V acc_i = P::zero();
    // through the virtual end separator of the longer chain, for every
    // pair's last lane
    const int nsteps = (int)span + (int)maxnl;
    // A lane of the shorter chain of a two-group warp keeps stepping past its
    // virtual end separator (column ncols) with nothing left to compute; its
    // code index stays clamped there so it reads no byte past its chain.
    const int last_s = (int)ncols + lag;

    // the haplotype code of the next step is loaded one step ahead (the
    // emission loads wait on it); the sweep runs in blocks of kStepBlock
    // steps, up to kStepBlock - 1 steps past the last one, whose columns
    // (past every lane's last separator) change no stored sum, and whose code
    // reads stay inside the code array's tail padding
    uint32_t code_next = hx[0];
    // one step of the sweep
    auto step = [&](int s) {
      V e[R], t_last;
      const uint32_t code = code_next;
      code_next = hx[kGroups > 1 ? min(s + 1, last_s) : s + 1];
      if constexpr (kScaled) {
        // the lane above hands over the M term (used one column later) and
        // the I^ of this lane's first row
        V in_t = group_shfl_up(P::fma(pr.mmU, M[R - 1], P::add(I[R - 1], D[R - 1])));
        V in_i = group_shfl_up(P::fma(pr.iiN, I[R - 1], M[R - 1]));
        if (top) {
          in_t = init; in_i = P::zero();
        }
        load_emission(table, lane, code, 0u, e);
        cells_scaled(e, dg_t, in_i, M, I, D, pr, t_last);
        dg_t = in_t;
      } else {
        V up_m = group_shfl_up(M[R - 1]);
        V up_i = group_shfl_up(I[R - 1]);
        V up_d = group_shfl_up(D[R - 1]);
        if (top) {
          up_m = P::zero(); up_i = P::zero(); up_d = init;
        }
        load_emission(table, lane, code, 0u, e);
        cells(e, up_m, up_i, up_d, dg_m, dg_i, dg_d, M, I, D, pr, t_last);
      }
      (void)t_last;
      if constexpr (!kScaled) acc_i = P::add(acc_i, I[R - 1]);
      if (s == nxt) {  // this lane just computed a separator column
        const V sum = kScaled ? P::add(D[R - 1], M[R - 1]) : acc_i;
#pragma unroll
        for (int k = 0; k < R; ++k) D[k] = P::zero();
        if constexpr (kScaled)
          M[R - 1] = P::zero();  // the sum row's value of the last column
        else
          acc_i = P::zero();
        // a pair's sums over haplotype hi (x and y halves), parked in the x
        // read's result slot until the sweep ends
        const uint32_t px = park[lane];
        if (px != kNoStore)
          reinterpret_cast<float2*>(b.out)[px + hi * meta->stride] =
              make_float2(P::sx(sum), P::sy(sum));
        ++hi;
        nxt = (int)meta->sep[hi] + lag;
      }
    };
    // Blocks of kStepBlock fully unrolled steps: the compiler overlaps
    // neighbouring steps' independent work (measured on the uneven batch at
    // 0.3 scale: 2 steps per loop iteration 3,875 GCUPS, 4 steps 3,976, 8
    // steps 4,028; with one running sum, 4,113 -- while a warp-uniform branch
    // that skipped the per-step separator test in blocks holding no lane's
    // separator made it slower, 4,020).
    const int nblocks = (nsteps + kStepBlock - 1) / kStepBlock;
#pragma unroll 1
    for (int s0 = 0; s0 < nblocks * kStepBlock; s0 += kStepBlock) {
#pragma unroll
      for (int i = 0; i < kStepBlock; ++i) step(s0 + i);
    }
    // the parked sums (written by other lanes of the warp) to results; the
    // item is read again rather than kept in registers through the sweep
    __syncwarp();
    if (active) {
      const ChainItem ci = *item_ptr;
      const uint32_t nh = ci.num_haps;
      const uint32_t ne = ci.pairs * nh;
      for (uint32_t p = (uint32_t)gl; p < ne; p += GROUP) {
        const uint32_t q = p / nh, h = p - q * nh;  // pair q of the item, haplotype h
        const uint32_t base = ci.out0 + h * ci.stride - ci.read_base;
        const uint32_t read[2] = {c.stack[ci.stack + 2 * q], c.stack[ci.stack + 2 * q + 1]};
        const float2 a = reinterpret_cast<const float2*>(b.out)[base + read[0]];
        const double ratio =
            (double)(P::init_const() / (S)b.haps[ci.hap_start + h].len) / (double)init_s;
#pragma unroll
        for (int s = 0; s < 2; ++s) {
          if (read[s] == kNoPair) continue;
          const S sum = s == 0 ? a.x : a.y;
          double res, amin = (double)kMinAcceptedF;
          if (kScaled) {  // the pass-through row holds (M_L + I_L)/gapm: the sum / mi
            const uint32_t len = b.reads[read[s]].len;
            res = scaled_result(b, read[s], len, len + 1, S(0), sum, &amin);
          } else {        // the pass-through row holds M_L + I_L (its M is 0)
            res = sum;
          }
          finish(b, c, PairRef{ci.hap_start + h, read[s], base + read[s]}, res * ratio, amin);
        }
      }
    }
    __syncwarp();
  }

  // The final log10 of one pair from its scaled likelihood `raw` (an FP32
  // result, possibly rescaled in FP64, or an FP64 result).
  // FP32: accepted at >= accept_min (1e-28, the reference's bound, or the
  // scaled form's bound) with an FP64 log10, else queued for FP64.
  // pos: the pair's list position under kLaunchRescueByItem.
  __device__ static void finish(const BatchView& b, const ClassLaunch& c, const PairRef& ref,
                                double raw, double accept_min = (double)kMinAcceptedF,
                                uint32_t pos = 0) {
    // A likelihood is finite and >= 0; anything else is an arithmetic fault,
    // reported rather than passed on (it would fail the acceptance test and
    // end up as a wrong FP64 value or -inf).
    if (!(raw >= 0.0) || isinf(raw)) {
      atomicOr(c.error_flags, kErrNonFinite);
      b.out[ref.out] = CUDART_NAN;
      return;
    }
    if (P::kSlots == 2) {
      if (raw >= accept_min) {
        if (b.raw_prec) {
          b.out[ref.out] = raw;
          b.raw_prec[ref.out] = 0;
        } else {
          b.out[ref.out] = log10(raw) - kLog10InitF;
        }
      } else {
        const uint32_t k = atomicAdd(c.rescue_count, 1u);
        c.rescue_list[(c.flags & kLaunchRescueByItem) ? pos : k] = ref;
      }
    } else {
      // The reference computes with flush-to-zero on (common.h:58-62), which on
      // x86 also flushes FP64 denormals: a likelihood below the normal FP64
      // range of the 2^1020 scaling becomes 0 and its log10 is -inf.  The GPU's
      // FP64 keeps denormals, so such a result is mapped to 0 (-inf) here.
      if (b.raw_prec) {
        b.out[ref.out] = raw >= kDblMin ? raw : 0.0;
        b.raw_prec[ref.out] = 1;
      } else {
        b.out[ref.out] = (raw >= kDblMin) ? log10(raw) - kLog10InitD : -CUDART_INF;
      }
    }
  }
};

template <class P, int R, bool UNIFORM, bool MULTI, bool SAME, int MINB, int GROUP = 32>
__global__ void __launch_bounds__(
    Forward<P, R, UNIFORM, MULTI, SAME, MINB, GROUP>::kWarpsPerBlock * kWarp, MINB)
    forward_kernel(BatchView b, ClassLaunch c) {
  using F = Forward<P, R, UNIFORM, MULTI, SAME, MINB, GROUP>;
  extern __shared__ uint4 smem[];
  const int lane = threadIdx.x & (kWarp - 1);
  const int warp = threadIdx.x / kWarp;
  uint4* table = smem + warp * (F::kSmemPerWarp / 16);
  const int gwarp = blockIdx.x * F::kWarpsPerBlock + warp;
  const uint32_t n = c.work_count ? *c.work_count : c.static_count;
  for (;;) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(c.counter, (uint32_t)F::kGroups);
    item = __shfl_sync(kFullMask, item, 0);
    if (item >= n) break;
    if constexpr (F::kChain)
      F::run_chain(b, c, item, n, lane, table);
    else
      F::run_item(b, c, item, lane, gwarp, table);
  }
}

}  // namespace rodv
