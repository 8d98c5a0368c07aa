// pairhmm_pipe.cuh -- multi-pass sweeps of long reads with the passes of one
// work item running concurrently on the warps of a block.
//
// A read longer than one pass (32 lanes x R rows) is swept in passes of 32R
// rows; pass p needs the last row of pass p-1 (its boundary row) column by
// column.  Swept one pass after the other by one warp, a pair of a 2,000-base
// read and a 5,000-base haplotype takes 8 x 5,031 steps in sequence, and the
// longest pairs of a batch set the length of the whole launch.  Here the W
// warps of a block take one work item together: warp w sweeps passes w, w+W,
// w+2W, ...  Lane 31 of the warp on pass p writes the pass's last row into a
// boundary row in global memory and publishes, after every 32 steps, how far
// it has come; lane 0 of the warp on pass p+1 reads that row through a
// shared-memory ring (cp.async, 32 columns ahead), waiting for the
// publication before each chunk.  Pass p+1 thus trails pass p by about 100
// steps instead of a whole pass, and the item's sweep takes about ceil(P/W)
// passes plus (W-1) x 100 steps.
//
// What crosses a pass boundary is what the lanes of a warp hand each other.
// In the scaled form (uniform gaps) that is two values per column: the M term
// of the row below, t = (mm/c) M~ + I^ + D^ (used one column later), and the
// row below's I^ = ii' I^ + M~ (ii' of the row below), both computed by the
// lane above with the operations the lane below would apply, so the results
// are bitwise those of a three-value hand-over of (M~, I^, D^).  Other forms
// hand over (M, I, D).  A boundary cell is 16 or 24 bytes.
//
// Boundary rows.  A block owns W+1 rows; pass p writes row p mod (W+1) and
// reads row (p-1) mod (W+1).  The next pass to write a row, p+W+1, runs on
// the same warp as p+1, the row's only reader, after p+1 has finished, so a
// producer never waits for a consumer.  Every wait is a consumer (pass p)
// waiting for its producer (pass p-1): waits point to strictly earlier
// passes, so they cannot form a cycle.  Each wait also gives up after a
// bounded number of polls, sets kErrWaitTimeout and stops the item, so a
// kernel always ends.  A row starts with kPad cells before its column 0:
// lane 31 stores its hand-over every step, the first 31 of which are columns
// <= 0 (zeros, never read), so no store needs a column test.
//
// Progress words live in shared memory: (pass << 17) | column, written with a
// CTA-scope release by the producing lane after its row stores (and a block
// fence), read with a CTA-scope acquire by every lane of the consumer before
// it copies the chunk.  The warps are in one block, so they share the SM's
// L1 and the CTA scope suffices.
//
// FP32 items stop early as in the single-warp sweep: after each pass but the
// last, the warp that swept it bounds the likelihood by the sum over the row
// it wrote (rejects(), the bound of Forward::row_bound_rejects restated for
// the hand-over cells); once both slots are below the acceptance bound the
// item stops on every warp and both pairs go to FP64.  The bound is exact, so
// the rescued pairs and every result are those of the full sweep.  (Holding
// pass 1 back until pass 0's verdict, so that a rejected item costs one pass
// instead of the passes in flight, made no difference on 2,000 pairs of
// 1,000-2,000-base reads and 2,000-5,000-base haplotypes that all go to FP64
// (2.92 ms FP32 pass either way, since the warps of these latency-bound
// sweeps leave issue slots free); at a quarter of the pairs it was slower,
// 1.34 against 1.19 ms.)
//
// Results are committed after a block barrier at the end of the item: by the
// warp that swept the last pass, or, for a rejected item, as FP64 rescues.
// The per-cell arithmetic is the single-warp sweep's (Forward::cells), and the
// pass count (pipe_passes, layout.h) leaves at least one pass-through row at
// the end, so a result is always the column sum of the I of a pass-through
// row (its M is 0): it depends neither on W nor on the strip height R nor on
// the item's other read.
#pragma once
#include <type_traits>

#include "pairhmm_fwd.cuh"

namespace rodv {

__device__ __forceinline__ uint32_t ld_acquire_cta(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.cta.shared.u32 %0, [%1];"
               : "=r"(v)
               : "r"((unsigned)__cvta_generic_to_shared(p))
               : "memory");
  return v;
}
__device__ __forceinline__ void st_release_cta(uint32_t* p, uint32_t v) {
  asm volatile("st.release.cta.shared.u32 [%0], %1;" ::"r"(
                   (unsigned)__cvta_generic_to_shared(p)),
               "r"(v)
               : "memory");
}
// cp.async of 16 bytes global -> shared (L2 only); both addresses 16-byte aligned
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned dst = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(gmem) : "memory");
}

template <class P, int R, bool UNIFORM, bool SAME, int MINB, int W>
struct PipeForward {
  using F = Forward<P, R, UNIFORM, true, SAME, MINB>;
  using V = typename P::V;
  using S = typename P::S;
  static constexpr bool kTwo = F::kScaled;  // two-value hand-over (t, i)
  struct HandCell {
    V t, i;
  };
  using Cell = typename std::conditional<kTwo, HandCell, typename F::BoundaryCell>::type;
  static_assert(sizeof(Cell) <= 24, "the engine sizes boundary rows at 24 bytes a cell");
  static constexpr int kRows = W + 1;                   // boundary rows per block
  static constexpr int kPad = kWarp;                    // cells before column 0 of a row
  // Steps per loop iteration, measured on the 2,000 long pairs above.  FP32:
  // four (FP32 pass 2.78 ms, 3.09 at two).  FP64: two, 166 registers at R = 8,
  // so three warps a sub-partition (FP64 pass 7.19 ms; 7.33 at four, 173
  // registers and two warps; 8.25 at one; 9.76 at one capped to 128
  // registers and four warps).
  static constexpr int kUnroll = P::kSlots == 1 ? 2 : 4;
  static constexpr int kSmemPerWarp = F::kSmemPerWarp;  // emission table + cell ring
  // polls of a progress word (about 100 ns each) before a wait gives up
  static constexpr uint32_t kWaitPolls = 1u << 24;
  static constexpr uint32_t kStopRejected = 1u, kStopFailed = 2u;

  struct Ctl {
    uint32_t item;
    uint32_t stop;         // 0, kStopRejected or kStopFailed
    uint32_t prog[kRows];  // per boundary row: (pass << 17) | last column published
  };

  __device__ __forceinline__ static uint32_t enc(uint32_t pass, uint32_t col) {
    return (pass << 17) | col;
  }

  __device__ __forceinline__ static bool stopped(Ctl& ctl) {
    return __any_sync(kFullMask, *reinterpret_cast<volatile uint32_t*>(&ctl.stop) != 0u);
  }

  // The whole warp waits until *word >= want; false (in every lane) when the
  // item stopped meanwhile or the wait expired (which stops the item).
  __device__ static bool wait_word(Ctl& ctl, const uint32_t* word, uint32_t want, uint32_t* err,
                                   uint32_t polls) {
    for (uint32_t k = 0;; ++k) {
      if (__all_sync(kFullMask, ld_acquire_cta(word) >= want)) return true;
      if (stopped(ctl)) return false;
      if (k >= polls) {
        if ((threadIdx.x & (kWarp - 1)) == 0) {
          atomicOr(err, kErrWaitTimeout);
          atomicExch(&ctl.stop, kStopFailed);
        }
        __syncwarp();
        return false;
      }
      __nanosleep(64);
    }
  }

  // The FP32 early-rejection decision after a pass (the same value in every
  // lane), from the hand-over cells of the pass's last row r.  With c = mi
  // gapm, t = (mm/gapm) M~/mi + I^ + D^ >= min(1, mm/gapm) (M~/mi + I^), so
  // max(1, gapm/mm) sum_j t bounds the sum Forward::row_bound_rejects bounds
  // the likelihood by (sum M~/mi + sum I^, rows r < L); a pass-through row
  // (r >= L) has M~ = D^ = 0 and t = I^, and its bound is sum t / mi.  The
  // acceptance test and its 1e-6 margin are the same.
  __device__ static bool rejects(const BatchView& b, const ClassLaunch& c, const Cell* row0,
                                 const uint32_t (&H)[2], const uint32_t (&L)[2], uint32_t row,
                                 int lane, uint32_t item) {
    if constexpr (!kTwo) {
      return F::row_bound_rejects(b, c, row0, H, L, row, lane, item);
    } else {
      V st = P::zero();
      for (uint32_t col = 1 + (uint32_t)lane; col <= H[0]; col += kWarp) {
        const V t = row0[col].t;
        st = P::add(st, P::make(P::sx(t), col <= H[1] ? P::sy(t) : S(0)));
      }
      double sum[2] = {(double)P::sx(st), (double)P::sy(st)};
#pragma unroll
      for (int d = 16; d >= 1; d /= 2) {
        sum[0] += __shfl_xor_sync(kFullMask, sum[0], d);
        sum[1] += __shfl_xor_sync(kFullMask, sum[1], d);
      }
      PairRef refs[2];
      F::load_refs(c, item, refs);
      bool rejected = true;
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (s == 1 && refs[1].read == kNoPair) continue;
        const uint32_t w = b.read_rows[b.reads[refs[s].read].row_off];
        const S* ph2pr = Tables<S>::ph2pr(b.tab);
        const double mi = (double)__ldg(ph2pr + rw_ins(w));
        const double gapm = 1.0 - (double)__ldg(ph2pr + rw_gcp(w));
        const double mm = (double)row_priors<S>(w, b.tab).mm;
        const double bound = row < L[s] ? (gapm > mm ? gapm / mm : 1.0) * sum[s] : sum[s] / mi;
        const double amin = (double)kMinAcceptedF / (mi * gapm);  // as scaled_result's
        rejected = rejected && mm > 0.0 && bound >= 0.0 && bound < amin * 1e-6;
      }
      return rejected;
    }
  }

  // What the warp of the item's last pass keeps for the commit.
  struct Sums {
    V acc;          // column sum of the I of the last row (a pass-through row)
    S frozen;       // slot y's sum at its own last column (two-haplotype items)
    uint32_t passes;
    bool ok;        // the item's descriptors were valid
  };

  // This warp's passes of work item `item`.
  __device__ static Sums run(const BatchView& b, const ClassLaunch& c, uint32_t item, int warp,
                             int lane, uint4* table, Ctl& ctl, Cell* rows) {
    Sums out;
    out.acc = P::zero();
    out.frozen = 0;
    out.passes = 0;
    out.ok = false;
    PairRef refs[2];
    F::load_refs(c, item, refs);
    // an FP64 list position that no rescue filled (kLaunchRescueByItem lists)
    if (P::kSlots == 1 && refs[0].read == kNoPair) return out;
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
    if (sl[0].H == 0 || sl[1].H == 0 || sl[0].L == 0 || sl[1].L == 0 ||
        (F::kSameHap && sl[0].hap != sl[1].hap) || sl[1].H > sl[0].H ||
        (uint64_t)sl[0].H + 40 > c.scratch_cols) {
      if (warp == 0 && lane == 0) atomicOr(c.error_flags, kErrBadLength);
      return out;
    }
    out.ok = true;
    const uint32_t passes = pipe_passes(Lmax, R);
    out.passes = passes;
    const uint32_t H = sl[0].H;
    const int nsteps = (int)H + kWarp - 1;         // slot x has the longer haplotype
    const int nfreeze = (int)sl[1].H + kWarp - 1;  // slot y's last accumulated step + 1
    const V init = P::make(P::init_const() / (S)sl[0].H, P::init_const() / (S)sl[1].H);
    const uint32_t L[2] = {sl[0].L, sl[1].L};
    const uint64_t row_off[2] = {sl[0].row_off, sl[1].row_off};
    Cell* ring = reinterpret_cast<Cell*>(table + F::Shape::kBytesPerWarp / 16);
    const uint32_t polls = c.wait_polls ? c.wait_polls : kWaitPolls;
    const bool publish = (c.flags & kLaunchNoPublish) == 0;

    for (uint32_t p = (uint32_t)warp; p < passes; p += W) {
      if (stopped(ctl)) break;
      const bool last = p + 1 == passes;
      const bool store = !last && lane == kWarp - 1;
      const int out_row = (int)(p % kRows);
      const int in_row = (int)((p + kRows - 1) % kRows);
      Cell* const out_cells = rows + (size_t)out_row * c.scratch_cols + kPad;  // column 0
      // lane 31's step s holds column s - 30 after the step
      Cell* const dst = out_cells - (kWarp - 2);
      const Cell* const src = rows + (size_t)in_row * c.scratch_cols + kPad;
      // cells of steps [32 k, 32 k + 32) from the previous pass's row
      // (columns 32 k + 1 .. 32 k + 32), copied once they are published
      auto fetch_chunk = [&](int k) -> bool {
        const uint32_t first = (uint32_t)k * kWarp + 1u;
        if (first <= H) {
          const uint32_t upto = first + kWarp - 1 < H ? first + kWarp - 1 : H;
          if (!wait_word(ctl, &ctl.prog[in_row], enc(p - 1, upto), c.error_flags, polls))
            return false;
        }
        const uint32_t idx = first + (uint32_t)lane;
        if (idx + kPad < c.scratch_cols) {
          Cell* d = ring + (k & 1) * kWarp + lane;
          const Cell* s = src + idx;
          if constexpr (kTwo) {
            cp_async16(d, s);
          } else {
            cp_async8(&d->m, &s->m);
            cp_async8(&d->i, &s->i);
            cp_async8(&d->d, &s->d);
          }
        }
        cp_async_commit();
        return true;
      };

      typename F::Priors pr;
      const uint32_t fr = p * (kWarp * R) + lane * R;
      F::load_rows(b, L, row_off, {fr, fr}, lane, table, pr);
      V M[R], I[R], D[R];
#pragma unroll
      for (int k = 0; k < R; ++k) M[k] = I[k] = D[k] = P::zero();
      const bool from_ring = p > 0;
      bool alive = true;
      if (from_ring) {
        alive = fetch_chunk(0);
      } else {
        // pass 0: lane 0's row above is row 0 of the DP at every column
        Cell top;
        if constexpr (kTwo) {
          top.t = init; top.i = P::zero();
        } else {
          top.m = P::zero(); top.i = P::zero(); top.d = init;
        }
        ring[lane] = top;
        ring[kWarp + lane] = top;
      }
      __syncwarp();
      uint32_t cx_next = sl[0].hap[-lane];
      uint32_t cy_next = F::kSameHap ? 0u : (uint32_t)sl[1].hap[-lane];
      const uint8_t* hx = sl[0].hap - lane + 1;  // code of the step after s: hx[s]
      const uint8_t* hy = sl[1].hap - lane + 1;
      V acc = P::zero();
      S frozen = 0;
      // two-value form: this lane's hand-over for the lane below, and the M
      // term of its first row carried to the next column
      V h_t = P::zero(), h_i = P::zero();
      V dg_t = (lane == 0 && p == 0) ? init : P::zero();
      // three-value form: the row above at the previous column
      V dg_m = P::zero(), dg_i = P::zero(), dg_d = (lane == 0 && p == 0) ? init : P::zero();

      const int nchunks = (nsteps + kWarp - 1) / kWarp;
      for (int k = 0; k < nchunks; ++k) {
        if (from_ring) {
          cp_async_wait_all();  // this chunk's cells
          __syncwarp();
          if (!fetch_chunk(k + 1)) {
            alive = false;
            break;
          }
        } else if (stopped(ctl)) {
          alive = false;
          break;
        }
        const Cell* rc = ring + (k & 1) * kWarp;
        const int s0 = k * kWarp;
        const int cnt = nsteps - s0 < kWarp ? nsteps - s0 : kWarp;
#pragma unroll kUnroll
        for (int i = 0; i < cnt; ++i) {
          const int s = s0 + i;
          const uint32_t cx = cx_next, cy = cy_next;
          cx_next = hx[s];
          if (!F::kSameHap) cy_next = hy[s];
          V e[R], t_last;
          if constexpr (kTwo) {
            V in_t = P::shfl_up(h_t), in_i = P::shfl_up(h_i);
            if (lane == 0) {
              const Cell cl = rc[i];
              in_t = cl.t; in_i = cl.i;
            }
            F::load_emission(table, lane, cx, cy, e);
            F::cells_scaled(e, dg_t, in_i, M, I, D, pr, t_last);
            dg_t = in_t;
            h_t = P::fma(pr.mmU, M[R - 1], P::add(I[R - 1], D[R - 1]));
            h_i = P::fma(pr.iiN, I[R - 1], M[R - 1]);
            if (store) dst[s] = Cell{h_t, h_i};
          } else {
            V up_m = P::shfl_up(M[R - 1]);
            V up_i = P::shfl_up(I[R - 1]);
            V up_d = P::shfl_up(D[R - 1]);
            if (lane == 0) {
              const Cell cl = rc[i];
              up_m = cl.m; up_i = cl.i; up_d = cl.d;
            }
            F::load_emission(table, lane, cx, cy, e);
            F::cells(e, up_m, up_i, up_d, dg_m, dg_i, dg_d, M, I, D, pr, t_last);
            if (store) {
              Cell cl;
              cl.m = M[R - 1]; cl.i = I[R - 1]; cl.d = D[R - 1];
              dst[s] = cl;
            }
          }
          (void)t_last;
          if (last) {
            acc = P::add(acc, I[R - 1]);
            if (P::kSlots == 2 && !F::kSameHap && s == nfreeze - 1) frozen = P::sy(acc);
          }
        }
        if (store && publish) {
          // columns up to (the chunk's last step) - 30 are stored
          const int col = s0 + cnt - 1 - (kWarp - 2);
          if (col >= 1) {
            __threadfence_block();
            st_release_cta(&ctl.prog[out_row], enc(p, (uint32_t)col));
          }
        }
      }
      if (from_ring) {
        cp_async_wait_all();  // the prefetch past the last step lands before the ring is reused
        __syncwarp();
      }
      if (!alive) break;
      if (last) {
        out.acc = acc;
        out.frozen = frozen;
      } else if constexpr (P::kSlots == 2) {
        __syncwarp();  // lane 31's row stores are visible to the whole warp
        const uint32_t Hs[2] = {sl[0].H, sl[1].H};
        if (rejects(b, c, out_cells, Hs, L, (p + 1) * (kWarp * R) - 1, lane, item)) {
          if (lane == 0) atomicCAS(&ctl.stop, 0u, kStopRejected);
          break;
        }
      }
    }
    return out;
  }

  // After the block barrier that ends the item: the results, or the FP64
  // rescue of a rejected item.
  __device__ static void commit(const BatchView& b, const ClassLaunch& c, uint32_t item,
                                int warp, int lane, const Ctl& ctl, const Sums& sm) {
    if (!sm.ok) return;
    const uint32_t stop = ctl.stop;
    if (stop == kStopFailed) return;  // the error flag is set
    PairRef fr[2];
    F::load_refs(c, item, fr);
    const bool valid_y = P::kSlots == 2 && fr[1].read != kNoPair;
    const uint32_t pos = c.rescue_base + 2u * item;  // kLaunchRescueByItem positions
    if (stop == kStopRejected) {
      if (warp == 0 && lane == 0) {
        F::finish(b, c, fr[0], 0.0, (double)kMinAcceptedF, pos);
        if (valid_y) F::finish(b, c, fr[1], 0.0, (double)kMinAcceptedF, pos + 1);
      }
      return;
    }
    if (warp != (int)((sm.passes - 1) % W) || lane != kWarp - 1) return;
    // both slots of a same-haplotype item ran exactly their own columns
    const S fy = (P::kSlots == 2 && F::kSameHap) ? P::sy(sm.acc) : sm.frozen;
    const uint32_t Lx = b.reads[fr[0].read].len;
    const uint32_t Ly = valid_y ? b.reads[fr[1].read].len : 0u;
    const uint32_t rows = sm.passes * kWarp * R;
    double res[2] = {0.0, 0.0};
    double amin[2] = {(double)kMinAcceptedF, (double)kMinAcceptedF};
    if (F::kScaled) {
      res[0] = F::scaled_result(b, fr[0].read, Lx, rows, S(0), P::sx(sm.acc), &amin[0]);
      if (valid_y) res[1] = F::scaled_result(b, fr[1].read, Ly, rows, S(0), fy, &amin[1]);
    } else {
      // the pass-through row holds M_L + I_L in its I (non-uniform form)
      res[0] = P::sx(sm.acc);
      res[1] = fy;
    }
    F::finish(b, c, fr[0], res[0], amin[0], pos);
    if (valid_y) F::finish(b, c, fr[1], res[1], amin[1], pos + 1);
  }
};

// One work item per block at a time; c.scratch holds kRows boundary rows of
// c.scratch_cols cells for every block of the grid.
template <class P, int R, bool UNIFORM, bool SAME, int MINB, int W>
__global__ void __launch_bounds__(W * kWarp, MINB)
    forward_pipe_kernel(BatchView b, ClassLaunch c) {
  using F = PipeForward<P, R, UNIFORM, SAME, MINB, W>;
  extern __shared__ uint4 smem[];
  __shared__ typename F::Ctl ctl;
  const int lane = threadIdx.x & (kWarp - 1);
  const int warp = threadIdx.x / kWarp;
  uint4* table = smem + warp * (F::kSmemPerWarp / 16);
  typename F::Cell* rows = reinterpret_cast<typename F::Cell*>(c.scratch) +
                           (size_t)blockIdx.x * F::kRows * c.scratch_cols;
  const uint32_t n = c.work_count ? *c.work_count : c.static_count;
  for (;;) {
    if (threadIdx.x == 0) {
      ctl.item = atomicAdd(c.counter, 1u);
      ctl.stop = 0;
#pragma unroll
      for (int k = 0; k < F::kRows; ++k) ctl.prog[k] = 0;
    }
    __syncthreads();
    const uint32_t item = ctl.item;
    if (item >= n) break;
    const typename F::Sums sm = F::run(b, c, item, warp, lane, table, ctl, rows);
    __syncthreads();
    F::commit(b, c, item, warp, lane, ctl, sm);
    __syncthreads();  // ctl is reset for the next item
  }
}

}  // namespace rodv
