// CUDA kernels of the B200 range solver (sm_100a).
//
// Work decomposition: one CTA owns one game ("spot") at a time and walks its
// level-ordered tree program (ps_device.hpp): forward steps propagate the
// opponent's reach top-down, backward steps evaluate terminals and combine
// children bottom-up with the DCFR regret / strategy update fused in.  The ops
// of one step are independent, so each warp takes whole ops (a node's update,
// or a run of terminals that read the same reach): hand vectors are streamed
// by the warp four hands per lane (128-bit loads and stores of regrets,
// strategy sums and the per-node reach / value vectors), different warps
// overlap different nodes' memory latency, and a step ends with one
// __syncthreads.  A whole solve of a spot - all iterations plus the
// exploitability checks - runs inside one persistent launch that pulls spots
// from a device work queue.
//
// Terminal evaluation restates crates/range-solver/src/game/evaluation.rs
// without its sequential merge: the opponent reach is gathered into
// hand-strength order and into per-card groups (both precomputed per board by
// k_setup), the warp scans that list segment by segment into its shared-memory
// buffer, and every hand reads its win / lose / blocked sums at precomputed
// positions - O(n) work per terminal, no CTA-wide barrier.
#include <cuda/atomic>
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <vector>

#include "ps_device.hpp"
#include "ps_handeval.hpp"
#include "ps_launch.hpp"

namespace ps {

enum Mode { M_DCFR = 0, M_BR = 1, M_AVG = 2, M_AVG_SAVE = 3 };

// Error bits reported through the error word of every launch.
constexpr int ERR_SCRATCH = 1;  // a spot needed more scratch than its CTA owns
constexpr int ERR_SETUP = 2;    // setup tables exceeded their bounds
constexpr int ERR_WAIT = 4;     // a grid barrier gave up waiting for the other CTAs

constexpr uint32_t THR_INVALID = 0xFFFFFFFFu;

// Optional per-phase cycle counters (build with -DPS_PHASE_TIMERS): lane 0 of
// every warp adds the clock64 cycles it spent in each phase, so the totals
// split the warps' time between terminal scans and lookups, node ops and
// barrier waits.  Read and cleared by ps_debug_phase_cycles in such builds.
enum Phase { PH_SCAN = 0, PH_LOOKUP, PH_FWD_OPP, PH_FWD_CHANCE, PH_BWD_TRAV, PH_BWD_OPP, PH_BWD_CHANCE, PH_BARRIER,
             PH_ROOT, PH_COUNT };
#ifdef PS_PHASE_TIMERS
__device__ unsigned long long g_phase[16];
#define PHASE_T0(v) const long long v = clock64()
#define PHASE_ADD(k, v)                                                                           \
  do {                                                                                            \
    if ((threadIdx.x & 31) == 0) atomicAdd(&g_phase[k], (unsigned long long)(clock64() - (v))); \
  } while (0)
#else
#define PHASE_T0(v) \
  do {              \
  } while (0)
#define PHASE_ADD(k, v) \
  do {                  \
  } while (0)
#endif

// A pointer into the dynamic shared memory, re-derived from the shared array
// itself: the compiler then knows its address space, and accesses through it
// are 32-bit shared loads and stores instead of generic ones.
__device__ __forceinline__ float* shared_view(float* p) {
  extern __shared__ float4 smem4[];
  float* base = reinterpret_cast<float*>(smem4);
  return base + (p - base);
}

struct Tables {  // board tables of one board, in shared or global memory
  const uint16_t* gidx[2];   // opponent-indexed gather lists
  const uint32_t* heads[2];  // opponent-indexed segment-start bitmaps
  const uint4* thr[2];       // player-indexed lookup records
  int nvalid[2];
};

struct Ctx {
  const SpotDev* sp;
  float* slots;
  int vstride;
  const float* root_reach;
  int grid;      // 1: every CTA of the launch works on this one spot (steps end in a grid barrier);
                 // 2: the same on the CTAs of one cluster (steps end in the cluster barrier)
  unsigned* bar; // grid mode: barrier counter and generation
  double* gred;  // grid mode: root reductions shared by all CTAs
  int* err;
  float* buf;    // smem: this warp's scan buffer [scan_buf_floats(vstride)] (null for warps >= bufs)
  int bufs;      // warps 0 .. bufs-1 own a scan buffer
  int owner;     // >= 0: adjoint pass, terminal values are player owner's payoffs (see warp_terms)
  int signed_reach;  // reach may be negative: terminal scans take segment starts from the bitmap
  float* bgrad;  // boundary gradient buffer [num_boundary][2][vstride], or null
  float* breach; // boundary reach buffer [num_boundary][2][vstride] (reach of each player), or null
  double* red;   // smem: reduction scratch       [32]
  Tables t0;     // board-0 tables (shared memory when staged, else global)
  int split;     // 1: node ops may be split over idle warps (few items per step)
  int part, parts;  // split node op: this item's column block and the number of blocks
  long long wait_ns;  // grid mode: how long a grid barrier waits for the other CTAs
  int sg;        // strategy cache of DCFR passes (SG_WRITE / SG_READ bits, 0 = none)
};

// Regret matching gives a player's strategy twice per DCFR iteration from the
// same regrets: in the opponent's pass (forward op, the player is the
// opponent) and in the player's own pass (backward op), which then updates
// them; no pass between the two changes the regrets.  With a strategy cache
// (SpotDev::SG, laid out like R) the forward op stores what it computes
// (SG_WRITE) and the backward op of the next pass reads it (SG_READ) instead
// of repeating the denominator sweep and the divisions.  The values are the
// same bits either way.
constexpr int SG_WRITE = 1, SG_READ = 2;

__device__ __forceinline__ const float* slot_in(const Ctx& c, uint16_t id) {
  return id == SLOT_ROOT_REACH ? c.root_reach : c.slots + (size_t)id * c.vstride;
}
__device__ __forceinline__ float* slot_at(const Ctx& c, uint16_t id) {
  return c.slots + (size_t)id * c.vstride;
}

// max(x, y) of the reference (sliceop.rs:5-12): no NaN propagation.
__device__ __forceinline__ float fmax_ref(float x, float y) { return x > y ? x : y; }

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }

__device__ __forceinline__ float4 max0(float4 a) {
  return make_float4(fmax_ref(a.x, 0.f), fmax_ref(a.y, 0.f), fmax_ref(a.z, 0.f), fmax_ref(a.w, 0.f));
}
__device__ __forceinline__ float4 add4(float4 a, float4 b) {
  return make_float4(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z), __fadd_rn(a.w, b.w));
}
__device__ __forceinline__ float4 mul4(float4 a, float4 b) {
  return make_float4(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y), __fmul_rn(a.z, b.z), __fmul_rn(a.w, b.w));
}
__device__ __forceinline__ float div_def(float m, float d, float def) { return d == 0.0f ? def : __fdiv_rn(m, d); }
__device__ __forceinline__ float4 sigma4(float4 m, float4 d, float def) {
  return make_float4(div_def(m.x, d.x, def), div_def(m.y, d.y, def), div_def(m.z, d.z, def), div_def(m.w, d.w, def));
}
__device__ __forceinline__ float4 max4(float4 a, float4 b) {
  return make_float4(fmax_ref(a.x, b.x), fmax_ref(a.y, b.y), fmax_ref(a.z, b.z), fmax_ref(a.w, b.w));
}
// DCFR regret update of one element (solver.rs:570-589): R * (R >= +0 ? alpha : beta) + cfv - result
__device__ __forceinline__ float regret_upd(float r, float cv, float res, float alpha, float beta) {
  return __fsub_rn(__fadd_rn(__fmul_rn(r, signbit(r) ? beta : alpha), cv), res);
}

__device__ __forceinline__ float warp_incl_scan(float x, int lane) {
#pragma unroll
  for (int s = 1; s < 32; s <<= 1) {
    float y = __shfl_up_sync(0xffffffffu, x, s);
    if (lane >= s) x += y;
  }
  return x;
}

// Asks L2 for the n floats at p, one 128-byte line per lane at a time, without
// waiting: an op issues this for every row it will stream before its first
// load, so its dependent loop iterations find the rows in L2 instead of each
// paying a DRAM round trip.
#ifndef PS_PREFETCH
#define PS_PREFETCH 1
#endif
__device__ __forceinline__ void prefetch_l2_bytes(const void* p, int bytes) {
#if PS_PREFETCH
  const char* b = static_cast<const char*>(p);
  for (int i = (threadIdx.x & 31) * 128; i < bytes; i += 32 * 128)
    asm volatile("prefetch.global.L2 [%0];" ::"l"(__cvta_generic_to_global(b + i)));
#endif
}
__device__ __forceinline__ void prefetch_l2(const float* p, int n) { prefetch_l2_bytes(p, 4 * n); }

// ---------------------------------------------------------------------------
// Forward ops
// ---------------------------------------------------------------------------

// Opponent decision node (solver.rs:418-445; utility.rs:227-250 for BR / AVG):
// sigma from regret matching (DCFR) or from the normalised cumulative strategy,
// then children's reach = sigma_a * reach.  Two sweeps over the actions: the
// first forms the denominator, the second (L1 hits) the children.
// finalize only (M_AVG_SAVE): IP cfvalues of the node for four hands, out of line
__device__ __noinline__ void save_ip_cfv(const SpotDev& sp, const NodeDev& nd, int h, float4 res) {
  const float v[4] = {res.x, res.y, res.z, res.w};
  for (int k = 0; k < 4; ++k)
    if (h + k < sp.H[1]) sp.ipcfv[nd.ip_off + h + k] = v[k];
}

template <bool SPLIT>
__device__ __forceinline__ void op_fwd_opp_t(const Ctx& c, const Op& op, int o, int mode) {
  // SPLIT: this item is column block c.part of c.parts (interleaved 32-column blocks)
  const int part = SPLIT ? c.part : 0, parts = SPLIT ? c.parts : 1;
  const SpotDev& sp = *c.sp;
  const int hso = sp.hs[o], na = op.na, q4 = hso >> 2;
  const float* base = (mode == M_DCFR ? sp.R : sp.S) + sp.nodes[op.node].rs_off;
  const float* src = slot_in(c, op.src);
  float* dst = slot_at(c, op.blk);
  float* sgw = mode == M_DCFR && (c.sg & SG_WRITE) ? sp.SG + sp.nodes[op.node].rs_off : nullptr;
  const float def = 1.0f / (float)na;
  if (part == 0) prefetch_l2(base, na * hso);
  for (int q = part * 32 + (threadIdx.x & 31); q < q4; q += 32 * parts) {
    const int h = q << 2;
    float4 d = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int a = 0; a < na; ++a) {
      float4 x = ld4(base + a * hso + h);
      if (mode == M_DCFR) x = max0(x);
      d = a == 0 ? x : add4(d, x);
    }
    const float4 r = ld4(src + h);
    for (int a = 0; a < na; ++a) {
      float4 x = ld4(base + a * hso + h);
      if (mode == M_DCFR) x = max0(x);
      const float4 s = sigma4(x, d, def);
      if (sgw) st4(sgw + a * hso + h, s);
      st4(dst + (size_t)a * c.vstride + h, mul4(s, r));
    }
  }
}
__device__ __forceinline__ void op_fwd_opp(const Ctx& c, const Op& op, int o, int mode) {
  op_fwd_opp_t<false>(c, op, o, mode);
}

// Chance node (solver.rs:264-276): one scaled reach shared by all children.
template <bool SPLIT>
__device__ __forceinline__ void op_fwd_chance_t(const Ctx& c, const Op& op, int o) {
  // SPLIT: this item is column block c.part of c.parts (interleaved 32-column blocks)
  const int part = SPLIT ? c.part : 0, parts = SPLIT ? c.parts : 1;
  const SpotDev& sp = *c.sp;
  const int q4 = sp.hs[o] >> 2;
  const float f = __fdiv_rn(1.0f, (float)sp.nodes[op.node].chance_factor);
  const float4 f4 = make_float4(f, f, f, f);
  const float* src = slot_in(c, op.src);
  float* dst = slot_at(c, op.blk);
  for (int q = part * 32 + (threadIdx.x & 31); q < q4; q += 32 * parts)
    st4(dst + (q << 2), mul4(ld4(src + (q << 2)), f4));
}
__device__ __forceinline__ void op_fwd_chance(const Ctx& c, const Op& op, int o) { op_fwd_chance_t<false>(c, op, o); }

// ---------------------------------------------------------------------------
// Backward ops
// ---------------------------------------------------------------------------

// Traverser decision node.
//   DCFR (solver.rs:333-416, :556-589): sigma = regret match(R); cfv = sum sigma_a cfv_a;
//        S = S * gamma + sigma; R = R * (R >= +0 ? alpha : beta) + cfv_a - cfv.
//   BR   (utility.rs:953-966): cfv = max_a cfv_a.
//   AVG  (utility.rs:689-727): sigma = S / sum S; cfv = sum sigma_a cfv_a; SAVE stores cfv_a.
// Three sweeps over the actions (denominator, result + S, regrets) keep the
// per-thread state to a few float4 registers; repeated loads hit L1.
template <bool SPLIT>
__device__ __forceinline__ void op_bwd_trav_t(const Ctx& c, const Op& op, int p, const Discount dc, int mode) {
  // SPLIT: this item is column block c.part of c.parts (interleaved 32-column blocks)
  const int part = SPLIT ? c.part : 0, parts = SPLIT ? c.parts : 1;
  const SpotDev& sp = *c.sp;
  const int hsp = sp.hs[p], na = op.na, q4 = hsp >> 2;
  const NodeDev& nd = sp.nodes[op.node];
  float* R = sp.R + nd.rs_off;
  float* S = sp.S + nd.rs_off;
  const float* cb = slot_at(c, op.blk);
  float* dst = slot_at(c, op.dst);
  const float* sgr = mode == M_DCFR && (c.sg & SG_READ) ? sp.SG + nd.rs_off : nullptr;
  const float def = 1.0f / (float)na;
  if (part == 0) {
    if (mode != M_BR) {
      prefetch_l2(mode == M_DCFR ? R : S, na * hsp);
      if (mode == M_DCFR) prefetch_l2(S, na * hsp);
      if (sgr) prefetch_l2(sgr, na * hsp);
    }
    for (int a = 0; a < na; ++a) prefetch_l2(cb + (size_t)a * c.vstride, hsp);
  }
  for (int q = part * 32 + (threadIdx.x & 31); q < q4; q += 32 * parts) {
    const int h = q << 2;
    float4 res = make_float4(0.f, 0.f, 0.f, 0.f);
    if (mode == M_BR) {
      res = ld4(cb + h);
      for (int a = 1; a < na; ++a) res = max4(res, ld4(cb + (size_t)a * c.vstride + h));
    } else {
      const float* W = mode == M_DCFR ? R : S;
      float4 d = make_float4(0.f, 0.f, 0.f, 0.f);
      if (!sgr)
        for (int a = 0; a < na; ++a) {
          float4 x = ld4(W + a * hsp + h);
          if (mode == M_DCFR) x = max0(x);
          d = a == 0 ? x : add4(d, x);
        }
      for (int a = 0; a < na; ++a) {
        float4 s;
        if (sgr) {
          s = ld4(sgr + a * hsp + h);
        } else {
          float4 x = ld4(W + a * hsp + h);
          if (mode == M_DCFR) x = max0(x);
          s = sigma4(x, d, def);
        }
        const float4 cv = ld4(cb + (size_t)a * c.vstride + h);
        const float4 t = mul4(s, cv);
        res = a == 0 ? t : add4(res, t);
        if (mode == M_DCFR) {
          const float4 g = make_float4(dc.gamma, dc.gamma, dc.gamma, dc.gamma);
          st4(S + a * hsp + h, add4(mul4(ld4(S + a * hsp + h), g), s));
        } else if (mode == M_AVG_SAVE) {
          st4(R + a * hsp + h, cv);
        }
      }
      if (mode == M_DCFR) {
        for (int a = 0; a < na; ++a) {
          const float4 r = ld4(R + a * hsp + h);
          const float4 cv = ld4(cb + (size_t)a * c.vstride + h);
          st4(R + a * hsp + h, make_float4(regret_upd(r.x, cv.x, res.x, dc.alpha, dc.beta),
                                           regret_upd(r.y, cv.y, res.y, dc.alpha, dc.beta),
                                           regret_upd(r.z, cv.z, res.z, dc.alpha, dc.beta),
                                           regret_upd(r.w, cv.w, res.w, dc.alpha, dc.beta)));
        }
      }
    }
    st4(dst + h, res);
    if (mode == M_AVG_SAVE && p == 1 && nd.ip_off != 0xFFFFFFFFu) save_ip_cfv(sp, nd, h, res);
  }
}
__device__ __forceinline__ void op_bwd_trav(const Ctx& c, const Op& op, int p, const Discount dc, int mode) {
  op_bwd_trav_t<false>(c, op, p, dc, mode);
}

// Opponent decision node: cfv = sum_a cfv_a (solver.rs:471).
template <bool SPLIT>
__device__ __forceinline__ void op_bwd_opp_t(const Ctx& c, const Op& op, int p, int mode) {
  // SPLIT: this item is column block c.part of c.parts (interleaved 32-column blocks)
  const int part = SPLIT ? c.part : 0, parts = SPLIT ? c.parts : 1;
  const SpotDev& sp = *c.sp;
  const int q4 = sp.hs[p] >> 2, na = op.na;
  const NodeDev& nd = sp.nodes[op.node];
  const float* cb = slot_at(c, op.blk);
  float* dst = slot_at(c, op.dst);
  if (part == 0)
    for (int a = 0; a < na; ++a) prefetch_l2(cb + (size_t)a * c.vstride, sp.hs[p]);
  for (int q = part * 32 + (threadIdx.x & 31); q < q4; q += 32 * parts) {
    const int h = q << 2;
    float4 res = ld4(cb + h);
    for (int a = 1; a < na; ++a) res = add4(res, ld4(cb + (size_t)a * c.vstride + h));
    st4(dst + h, res);
    if (mode == M_AVG_SAVE && p == 1 && nd.ip_off != 0xFFFFFFFFu) save_ip_cfv(sp, nd, h, res);
  }
}
__device__ __forceinline__ void op_bwd_opp(const Ctx& c, const Op& op, int p, int mode) {
  op_bwd_opp_t<false>(c, op, p, mode);
}

// Chance node: cfv = sum over dealt cards, plus the suit-swapped rows of the
// isomorphic cards that were not dealt (solver.rs:291-325).
template <bool SPLIT>
__device__ __forceinline__ void op_bwd_chance_t(const Ctx& c, const Op& op, int p, int mode) {
  // SPLIT: this item is column block c.part of c.parts (interleaved 32-column blocks)
  const int part = SPLIT ? c.part : 0, parts = SPLIT ? c.parts : 1;
  const SpotDev& sp = *c.sp;
  const int hsp = sp.hs[p], na = op.na;
  const NodeDev& nd = sp.nodes[op.node];
  const float* cb = slot_at(c, op.blk);
  float* dst = slot_at(c, op.dst);
  int i0 = 0, i1 = 0;
  if (op.board != 0xFFFF) {
    i0 = sp.iso_off[op.board];
    i1 = sp.iso_off[op.board + 1];
  }
  for (int h = part * 32 + (threadIdx.x & 31); h < hsp; h += 32 * parts) {
    float res = cb[h];
    for (int a = 1; a < na; ++a) res = __fadd_rn(res, cb[(size_t)a * c.vstride + h]);
    for (int i = i0; i < i1; ++i) {
      const int ref = sp.iso_ent[2 * i], perm = sp.iso_ent[2 * i + 1];
      const int hh = sp.iso_perm[p][(size_t)perm * hsp + h];
      res = __fadd_rn(res, cb[(size_t)ref * c.vstride + hh]);
    }
    dst[h] = res;
    if (mode == M_AVG_SAVE && nd.ch_player == p && h < sp.H[p]) sp.chcfv[nd.ch_off + h] = res;
  }
}
__device__ __forceinline__ void op_bwd_chance(const Ctx& c, const Op& op, int p, int mode) {
  op_bwd_chance_t<false>(c, op, p, mode);
}

// ---------------------------------------------------------------------------
// Terminal evaluation (game/evaluation.rs:57-634)
// ---------------------------------------------------------------------------
//
// Per board and opponent o the gather list holds the V valid opponent hands in
// (strength, index) order followed by, for every card c, the valid opponent
// hands holding c in the same order (segment [coff[c], coff[c+1])).  After the
// scans, for a hand h with thresholds
//   lt = #opp weaker, le = #opp weaker-or-tied, ltc / lec = the same counts
//   inside each of its two card segments,
// the reference's sums are prefix lookups:
//   win  = P(lt) - Q_c1(ltc1) - Q_c2(ltc2)       (strictly weaker, not blocked)
//   lose = (T - P(le)) - (M_c1 - Q_c1(lec1)) - (M_c2 - Q_c2(lec2))
//   fold = T + r_same - M_c1 - M_c2               (inclusion-exclusion)
// The scan buffer holds entry j of the list at kScanBase + j above four zeros,
// so every prefix is one load at a position k_setup precomputes (an empty
// prefix points at a zero): the hand's 16-byte record is eight u16 positions,
//   x = P(lt) | P(le) << 16, y = Q_c1(ltc1) | Q_c1(lec1) << 16,
//   z = M_c1 | Q_c2(ltc2) << 16, w = Q_c2(lec2) | M_c2 << 16,
// and T is the prefix of all V entries.
__device__ __forceinline__ void board_tables(const Ctx& c, int b, Tables& t) {
  if (b == 0) {
    t = c.t0;
    return;
  }
  const SpotDev& sp = *c.sp;
  for (int q = 0; q < 2; ++q) {
    t.gidx[q] = sp.gidx[q] + (size_t)b * 3 * sp.hs[q];
    t.heads[q] = sp.heads[q] + (size_t)b * head_words(sp.hs[q]);
    t.thr[q] = reinterpret_cast<const uint4*>(sp.thr[q]) + (size_t)b * sp.hs[q];
    t.nvalid[q] = sp.nvalid[q][b];
  }
}

// Evaluates a run of n terminals that read the same reach on the same board,
// for traverser p, with the calling warp alone, in three phases whose memory
// accesses are issued as independent batches:
//  1. gather: every lane reads four gather indices at a time (16 entries per
//     batch) and the opponent reach at those indices; a segment start is
//     stored as -x (reach values are >= +0, so the sign bit flags a start even
//     for a zero);
//  2. scan: each lane scans a contiguous chunk of the 3V-entry list of odd
//     length (the lanes' strided shared-memory accesses then fall in distinct
//     banks), a segmented warp scan of the chunk totals gives each chunk its
//     carry-in, and the chunk's entries before its first segment start add it;
//  3. lookups: per terminal, every hand reads its 16-byte record and its
//     win / lose / blocked sums at the recorded positions of the scan.
// GEN = false is the copy the solve passes use (non-negative reach, the
// traverser's own payoffs, no boundary gradients); GEN = true adds what the
// average-strategy passes of root_cfvalues_with_reach and the adjoint need.
// SPLIT (solve passes of launches whose CTAs hold a lone spot): the run is
// part c.part of c.parts warps; each gathers and scans the whole list in its
// own buffer and evaluates the hands of its interleaved 32-hand blocks.
// CTA (grid mode, every warp holding a buffer): the whole CTA evaluates the
// run in warp 0's buffer.  All warps gather, warp 0 alone scans (the same
// chunks, so the same sums), and warp w evaluates hand blocks w, w + W, ...;
// every thread of the CTA calls it for the same runs.
// Raked showdown value of one hand (evaluation.rs:429-537), out of line: the
// solve loop of unraked trees never takes it, and the per-hand loop stays small.
__device__ __noinline__ float raked_showdown_value(float cw, float cl, float ctie, float win, float Ple, float Q1le,
                                                   float Q2le, float Tsum, float M1, float M2, const float* rch,
                                                   uint32_t si) {
  const float rs = si != 0xFFFF ? rch[si] : 0.f;
  const float tie = Ple - Q1le - Q2le;
  const float tot = Tsum - M1 - M2;
  return cw * win + ctie * (tie - win + rs) + cl * (tot - tie);
}


#ifndef PS_GATHER_U
#define PS_GATHER_U 2  // groups of four entries each lane gathers per round (2 measured best of 1-4)
#endif
template <bool GEN, bool SPLIT = false, bool CTA = false>
__device__ __forceinline__ void warp_terms_inl(const Ctx& c, const Op* ops, int n, int p) {
  static_assert(!CTA || (SPLIT && !GEN), "CTA runs are solve-pass runs of lone spots");
  PHASE_T0(t_scan);
  const SpotDev& sp = *c.sp;
  const int o = p ^ 1;
  const int Hp = sp.H[p], hsp = sp.hs[p];
  const int lane = threadIdx.x & 31;
  Tables T;
  board_tables(c, ops[0].board, T);
  const int V = T.nvalid[o], n3 = 3 * V;
  const uint16_t* g = T.gidx[o];
  const uint32_t* hd = T.heads[o];
  const float* rch = slot_in(c, ops[0].src);
  prefetch_l2_bytes(T.thr[p], 16 * Hp);
  const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  // the scan buffer (in CTA mode warp 0's: buffers are scan_buf_floats apart,
  // one spot a launch); entry j of the gathered list lives at e[j]
  float* buf = shared_view(CTA ? c.buf - (size_t)warp * scan_buf_floats(c.vstride) : c.buf);
  float* e = buf + kScanBase;
  if (lane == 0 && (!CTA || warp == 0)) st4(buf, make_float4(0.f, 0.f, 0.f, 0.f));  // what empty prefixes read
  // adjoint pass at a depth boundary: the reach is weighted by the payoff
  // owner's boundary values.  Where the gathered values may be negative
  // (caller-given reach, boundary weights) segment starts come from the
  // bitmap; solve passes mark them in the sign bit of the non-negative reach.
  const bool adjm = GEN && c.owner >= 0;
  const NodeDev& nd0 = sp.nodes[ops[0].node];
  const float* bw = adjm && ops[0].term == TERM_BOUNDARY
                        ? sp.bcfv + ((size_t)nd0.boundary * 2 + c.owner) * c.vstride
                        : nullptr;
  const bool bits = GEN && (bw != nullptr || c.signed_reach != 0);
  {  // 1. gather
    const int n4 = (n3 + 3) >> 2;  // groups of four entries
    constexpr int kU = PS_GATHER_U;
    for (int w0 = (CTA ? warp * 32 * kU : 0) + lane; w0 < n4; w0 += 32 * kU * (CTA ? nwarps : 1)) {
      uint2 ix[kU];
      uint32_t hb[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int w = w0 + 32 * u;
        ix[u] = w < n4 ? *reinterpret_cast<const uint2*>(g + 4 * w) : make_uint2(0u, 0u);
        hb[u] = w < n4 ? hd[w >> 3] >> ((4 * w) & 31) : 0u;
      }
      float x[kU][4];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int k = 4 * (w0 + 32 * u);
        const uint32_t id[4] = {ix[u].x & 0xFFFFu, ix[u].x >> 16, ix[u].y & 0xFFFFu, ix[u].y >> 16};
#pragma unroll
        for (int e = 0; e < 4; ++e) x[u][e] = k + e < n3 ? (GEN && bw ? rch[id[e]] * bw[id[e]] : rch[id[e]]) : 0.f;
      }
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int k = 4 * (w0 + 32 * u);
        if (k >= n3) continue;
        const uint32_t m = bits ? 0u : hb[u];
        float4 v;
        v.x = (m & 1u) ? -x[u][0] : x[u][0];
        v.y = (m & 2u) ? -x[u][1] : x[u][1];
        v.z = (m & 4u) ? -x[u][2] : x[u][2];
        v.w = (m & 8u) ? -x[u][3] : x[u][3];
        st4(e + k, v);  // entries past n3 are never read
      }
    }
  }
  if (CTA)
    __syncthreads();
  else
    __syncwarp();
  if (!CTA || warp == 0) {  // 2. chunked segmented scan
    const int C = ((n3 + 31) >> 5) | 1;
    const int lo = min(lane * C, n3), hi = min(lo + C, n3);
    float run = 0.f;
    int first = hi;
    if (bits) {
      for (int j = lo; j < hi; ++j) {
        const float x = e[j];
        if ((hd[j >> 5] >> (j & 31)) & 1u) {
          run = x;
          first = min(first, j);
        } else {
          run = __fadd_rn(run, x);
        }
        e[j] = run;
      }
    } else {
      // a segment start carries the sign bit of its non-negative value
#pragma unroll 2
      for (int j = lo; j < hi; ++j) {
        const float x = e[j], y = fabsf(x);
        run = signbit(x) ? y : __fadd_rn(run, y);
        e[j] = run;
      }
      // the chunk's first segment start, from the bitmap the signs came from
      for (int w = lo >> 5; lo < hi && w <= (hi - 1) >> 5; ++w) {
        const uint32_t m = hd[w] & (w == lo >> 5 ? ~0u << (lo & 31) : ~0u);
        if (m) {
          first = min(hi, (w << 5) + __ffs(m) - 1);
          break;
        }
      }
    }
    float v = run;
    bool f = first < hi;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const float vv = __shfl_up_sync(0xffffffffu, v, d);
      const bool ff = __shfl_up_sync(0xffffffffu, (int)f, d) != 0;
      if (lane >= d) {
        if (!f) v = __fadd_rn(v, vv);
        f = f || ff;
      }
    }
    float in = __shfl_up_sync(0xffffffffu, v, 1);
    if (lane == 0) in = 0.f;
    for (int j = lo; j < first; ++j) e[j] = __fadd_rn(e[j], in);
  }
  if (CTA)
    __syncthreads();
  else
    __syncwarp();
  PHASE_ADD(PH_SCAN, t_scan);
  PHASE_T0(t_look);
  if (GEN && c.breach && ops[0].term == TERM_BOUNDARY && !adjm) {  // the opponent's reach at this boundary
    float* row = c.breach + ((size_t)nd0.boundary * 2 + o) * c.vstride;
    for (int h = lane; h < sp.H[o]; h += 32) row[h] = rch[h];
  }
  // 3. lookups: every prefix is one load at a position of the hand's record
  const uint4* thr = T.thr[p];
  const uint16_t* same = sp.same[p];
  const float Tsum = buf[kScanBase - 1 + V];  // all V entries (0 when V = 0)
  const int pay = adjm ? c.owner : p;  // whose payoffs the values are
  const int part = CTA ? warp : SPLIT ? c.part : 0, parts = CTA ? nwarps : SPLIT ? c.parts : 1;
  const int h0 = part * 32 + lane, hstep = 32 * parts;
  for (int j = 0; j < n; ++j) {
    const Op& op = ops[j];
    const NodeDev& nd = sp.nodes[op.node];
    float* dst = slot_at(c, op.dst);
    const float aw = nd.amount_win, al = nd.amount_lose;
    // showdown coefficients of the traverser's win / loss (swapped when the
    // values are the opponent's payoffs)
    const float cw = adjm ? al : aw, cl = adjm ? aw : al;
    float* grow = GEN && c.bgrad && op.term == TERM_BOUNDARY && !adjm
                      ? c.bgrad + ((size_t)nd.boundary * 2 + p) * c.vstride
                      : nullptr;
    // the next hand's record is requested before this hand's value is stored:
    // the store may alias it, so the compiler would not issue it earlier
    uint4 tn = h0 < Hp ? thr[h0] : make_uint4(THR_INVALID, 0, 0, 0);
    if (!GEN && op.term == TERM_BOUNDARY) {
      // depth-boundary values in a loop of their own, which keeps the fold /
      // showdown loop of full trees small (evaluation.rs:544-605)
      const float* brow = sp.bcfv + ((size_t)nd.boundary * 2 + p) * c.vstride;
      for (int h = h0; h < hsp; h += hstep) {
        float v = 0.f;
        const uint4 t = tn;
        tn = h + hstep < Hp ? thr[h + hstep] : make_uint4(THR_INVALID, 0, 0, 0);
        if (t.x != THR_INVALID) {
          const float M1 = buf[t.z & 0xFFFF], M2 = buf[t.w >> 16];
          const uint32_t si = same[h];
          const float rs = si != 0xFFFF ? rch[si] : 0.f;
          const float adj = Tsum + rs - M1 - M2;
          v = __fmul_rn(__fmul_rn(brow[h], nd.payoff_scale), adj);
        }
        dst[h] = v;
      }
      continue;
    }
    // whole-warp runs (no split copies: those of the lone-spot grid ran slower so)
    if (!GEN && !SPLIT && op.term == TERM_SHOWDOWN && !sp.raked) {  // unraked showdowns in a loop of their own
#pragma unroll 2
      for (int h = h0; h < hsp; h += hstep) {
        float v = 0.f;
        const uint4 t = tn;
        tn = h + hstep < Hp ? thr[h + hstep] : make_uint4(THR_INVALID, 0, 0, 0);
        if (t.x != THR_INVALID) {
          const float M1 = buf[t.z & 0xFFFF], M2 = buf[t.w >> 16];
          const float Plt = buf[t.x & 0xFFFF], Ple = buf[t.x >> 16];
          const float Q1lt = buf[t.y & 0xFFFF], Q1le = buf[t.y >> 16];
          const float Q2lt = buf[t.z >> 16], Q2le = buf[t.w & 0xFFFF];
          const float win = Plt - Q1lt - Q2lt;
          const float lose = (Tsum - Ple) - (M1 - Q1le) - (M2 - Q2le);
          v = __fadd_rn(__fmul_rn(cw, win), __fmul_rn(cl, lose));
        }
        dst[h] = v;
      }
      continue;
    }
    if (!GEN && !SPLIT && op.term == TERM_FOLD) {  // folds in a loop of their own
      const float cf = op.fold_pl != pay ? aw : al;
#pragma unroll 2
      for (int h = h0; h < hsp; h += hstep) {
        float v = 0.f;
        const uint4 t = tn;
        tn = h + hstep < Hp ? thr[h + hstep] : make_uint4(THR_INVALID, 0, 0, 0);
        if (t.x != THR_INVALID) {
          const float M1 = buf[t.z & 0xFFFF], M2 = buf[t.w >> 16];
          const uint32_t si = same[h];
          const float rs = si != 0xFFFF ? rch[si] : 0.f;
          const float adj = Tsum + rs - M1 - M2;
          v = __fmul_rn(cf, adj);
        }
        dst[h] = v;
      }
      continue;
    }
    for (int h = h0; h < hsp; h += hstep) {
      float v = 0.f;
      const uint4 t = tn;
      tn = h + hstep < Hp ? thr[h + hstep] : make_uint4(THR_INVALID, 0, 0, 0);
      if (t.x != THR_INVALID) {
        const float M1 = buf[t.z & 0xFFFF], M2 = buf[t.w >> 16];
        if (op.term == TERM_SHOWDOWN) {
          const float Plt = buf[t.x & 0xFFFF], Ple = buf[t.x >> 16];
          const float Q1lt = buf[t.y & 0xFFFF], Q1le = buf[t.y >> 16];
          const float Q2lt = buf[t.z >> 16], Q2le = buf[t.w & 0xFFFF];
          const float win = Plt - Q1lt - Q2lt;
          if (!sp.raked) {
            const float lose = (Tsum - Ple) - (M1 - Q1le) - (M2 - Q2le);
            v = __fadd_rn(__fmul_rn(cw, win), __fmul_rn(cl, lose));
          } else {
            v = raked_showdown_value(cw, cl, nd.amount_tie, win, Ple, Q1le, Q2le, Tsum, M1, M2, rch, same[h]);
          }
        } else {
          const uint32_t si = same[h];
          const float rs = si != 0xFFFF ? (GEN && bw ? rch[si] * bw[si] : rch[si]) : 0.f;
          const float adj = Tsum + rs - M1 - M2;
          if (op.term == TERM_FOLD) {
            v = __fmul_rn(op.fold_pl != pay ? aw : al, adj);
          } else if (GEN && adjm) {
            v = __fmul_rn(nd.payoff_scale, adj);
          } else if (GEN) {  // boundary values of the general passes (solve passes loop above)
            const float bv = sp.bcfv[((size_t)nd.boundary * 2 + p) * c.vstride + h];
            v = __fmul_rn(__fmul_rn(bv, nd.payoff_scale), adj);
            if (grow) grow[h] = __fmul_rn(nd.payoff_scale, adj);
          }
        }
      }
      if (GEN && grow && t.x == THR_INVALID) grow[h] = 0.f;
      dst[h] = v;
    }
  }
  if (GEN && bw && c.bgrad) {  // dV/dB = (scale * blocked opponent reach) * own adjoint reach / chance path
    float* grow = c.bgrad + ((size_t)nd0.boundary * 2 + c.owner) * c.vstride;
    const float inv = __fdiv_rn(1.0f, nd0.path_scale);
    for (int h = lane; h < sp.H[c.owner]; h += 32) grow[h] = __fmul_rn(__fmul_rn(grow[h], rch[h]), inv);
  }
  if (CTA)
    __syncthreads();  // the buffer is free for the CTA's next run
  else
    __syncwarp();  // the buffer is free for this warp's next run
  PHASE_ADD(PH_LOOKUP, t_look);
}
// The out-of-line copies the step-synchronous and grid passes call.  The
// dataflow kernel inlines its two copies at their call sites instead: its
// items then keep the context in registers rather than passing it through
// local memory (6770 against 5786 spots/s on the datagen batch), while the
// grid kernel, which calls several copies, ran slower with them inlined.
template <bool GEN, bool SPLIT = false, bool CTA = false>
__device__ __noinline__ void warp_terms(const Ctx& c, const Op* ops, int n, int p) {
  warp_terms_inl<GEN, SPLIT, CTA>(c, ops, n, p);
}

// ---------------------------------------------------------------------------
// Pass driver and root reductions
// ---------------------------------------------------------------------------
// Grid barrier of a cooperative launch (all CTAs resident): a counter, a
// generation word and an abort word in global memory (bar[0..2]), device-scope
// release / acquire.  A wait gives up after c.wait_ns nanoseconds of the
// global timer (or, as a backstop should the timer stall, after wait_ns / 16
// polls), reports ERR_WAIT and sets the abort word.  From then on every
// barrier of every CTA returns false at once - also one that was already
// waiting - and the pass and iteration loops end, so a failed launch ends with
// an error status instead of a hung GPU.  The result is the same on every
// thread of the CTA (s_grid_ok, written by thread 0 between two barriers).
constexpr long long kGridWaitNs = 1000000000LL;  // 1 s: a grid step takes microseconds
__shared__ int s_grid_ok;  // grid mode: 0 once the launch is aborted

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ bool grid_barrier(const Ctx& c) {
  if (c.grid == 2) {
    // one cluster: the hardware barrier over every thread of its CTAs, with
    // cluster-scope release / acquire (the spot's global-memory vectors and
    // root values are written and read by those CTAs only).  Every CTA runs
    // the same steps, so every thread arrives; nothing spins.
    asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
    return true;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    cuda::atomic_ref<unsigned, cuda::thread_scope_device> count(c.bar[0]), gen(c.bar[1]), abort_(c.bar[2]);
    int ok = abort_.load(cuda::memory_order_relaxed) == 0u;
    if (ok) {
      const unsigned g = gen.load(cuda::memory_order_acquire);
      if (count.fetch_add(1u, cuda::memory_order_acq_rel) == gridDim.x - 1) {
        count.store(0u, cuda::memory_order_relaxed);
        gen.store(g + 1u, cuda::memory_order_release);
      } else {
        const unsigned long long t0 = global_ns();
        const unsigned long long max_polls = (unsigned long long)(c.wait_ns / 16) + 65536ull;
        for (unsigned long long n = 0; gen.load(cuda::memory_order_acquire) == g; ++n) {
          if (abort_.load(cuda::memory_order_relaxed) != 0u) {
            ok = 0;
            break;
          }
          if (n >= max_polls || ((n & 31) == 31 && (long long)(global_ns() - t0) > c.wait_ns)) {
            atomicOr(c.err, ERR_WAIT);
            abort_.store(1u, cuda::memory_order_relaxed);
            ok = 0;
            break;
          }
          __nanosleep(32);
        }
      }
    }
    s_grid_ok = ok;
  }
  __syncthreads();
  return s_grid_ok != 0;
}

// false once a grid-mode launch has been aborted (uniform over the CTA: read
// only after a barrier); always true outside grid mode
__device__ __forceinline__ bool grid_live(const Ctx& c) { return !c.grid || s_grid_ok != 0; }

__device__ __forceinline__ bool step_barrier(const Ctx& c) {
  if (c.grid) return grid_barrier(c);
  __syncthreads();
  return true;
}

// One pass for traverser p over the K spots cs[0..K) in lockstep (spots of
// one tree shape share the step structure; only the spots in `active` take
// part).  A step's items of all spots are interleaved over the warps, so one
// barrier per step serves K spots.
constexpr int kMaxInst = 4;  // spots per CTA at most

__device__ __noinline__ void run_pass_multi(Ctx* cs, int K, unsigned active, int p, const Discount dc, int mode) {
  int first = 0;
  while (first < K && !(active >> first & 1u)) ++first;
  if (first == K) return;
  const Ctx& c = cs[first];
  const SpotDev& sp = *c.sp;
  const Step* steps = sp.steps[p];
  const int o = p ^ 1;
  const int warp = threadIdx.x >> 5, nw0 = blockDim.x >> 5;
  // in grid mode the items of a step are spread over the warps of all CTAs
  const int nw = c.grid ? gridDim.x * nw0 : nw0;
  const int gw = c.grid ? blockIdx.x * nw0 + warp : warp;
  const int nb = c.grid ? gridDim.x * c.bufs : c.bufs;
  const int gb = c.grid ? blockIdx.x * c.bufs + warp : warp;
  const bool gen = c.owner >= 0 || c.signed_reach || c.bgrad || c.breach;
  for (int s = 0; s < sp.nsteps[p]; ++s) {
    const Step st = steps[s];
    // terminal runs go round robin to the warps that own a scan buffer; node
    // ops go round robin to all warps, starting at the first warp without a
    // run.  Item j belongs to spot j % K.
    const int ng = K * st.n_groups, ne = K * st.n_elem;
    if (warp < c.bufs)
      for (int j = gb; j < ng; j += nb) {
        const int k = j % K;
        if (!(active >> k & 1u)) continue;
        const Ctx& ck = cs[k];
        const Op* lead = ck.sp->ops[p] + st.begin + st.n_elem + ck.sp->groups[p][st.gbegin + j / K];
        if (gen)
          warp_terms<true>(ck, lead, lead->na, p);
        else
          warp_terms<false>(ck, lead, lead->na, p);
      }
    const int start = min(ng, nb) % nw;
    for (int i = (gw - start + nw) % nw; i < ne; i += nw) {
      const int k = i % K;
      if (!(active >> k & 1u)) continue;
      const Ctx& ck = cs[k];
      const Op op = ck.sp->ops[p][st.begin + i / K];
      PHASE_T0(t_op);
      switch (op.type) {
        case OP_FWD_OPP: op_fwd_opp(ck, op, o, mode); break;
        case OP_FWD_CHANCE: op_fwd_chance(ck, op, o); break;
        case OP_BWD_TRAV: op_bwd_trav(ck, op, p, dc, mode); break;
        case OP_BWD_OPP: op_bwd_opp(ck, op, p, mode); break;
        case OP_BWD_CHANCE: op_bwd_chance(ck, op, p, mode); break;
        default: break;
      }
      PHASE_ADD(op.type == OP_FWD_OPP      ? PH_FWD_OPP
                : op.type == OP_FWD_CHANCE ? PH_FWD_CHANCE
                : op.type == OP_BWD_TRAV   ? PH_BWD_TRAV
                : op.type == OP_BWD_OPP    ? PH_BWD_OPP
                                           : PH_BWD_CHANCE,
                t_op);
    }
    PHASE_T0(t_bar);
    const bool live = step_barrier(c);
    PHASE_ADD(PH_BARRIER, t_bar);
    if (!live) return;
  }
}

// One pass of one spot whose CTA (or grid) has few items per step: node ops
// and terminal runs are split over the warps a step leaves idle, in
// interleaved 32-column (32-hand) blocks, and in grid mode a step with few
// runs gives each a whole CTA.  Each hand's arithmetic is that of
// run_pass_multi; only the warp that runs it differs.
__device__ __noinline__ void run_pass_split(const Ctx& c, int p, const Discount dc, int mode) {
  const SpotDev& sp = *c.sp;
  const Step* steps = sp.steps[p];
  const int o = p ^ 1;
  const int warp = threadIdx.x >> 5, nw0 = blockDim.x >> 5;
  const int nw = c.grid ? gridDim.x * nw0 : nw0;
  const int gw = c.grid ? blockIdx.x * nw0 + warp : warp;
  const int nb = c.grid ? gridDim.x * c.bufs : c.bufs;
  const int gb = c.grid ? blockIdx.x * c.bufs + warp : warp;
  const bool gen = c.owner >= 0 || c.signed_reach || c.bgrad || c.breach;
  for (int s = 0; s < sp.nsteps[p]; ++s) {
    const Step st = steps[s];
    const int ng = st.n_groups, ne = st.n_elem;
    // terminal runs of the solve passes: in grid mode with few runs, a CTA a
    // run (CTAs 0 .. ng-1); otherwise split over the buffer warps a step
    // leaves idle (at most 8 parts a run, and at most half the warps when the
    // step has node ops to split as well)
    // (a cluster has few CTAs: there a step without node ops gives a CTA to
    // each of up to gridDim.x runs)
    const bool cta_runs = c.grid && !gen && ng > 0 && c.bufs == nw0 &&
                          (2 * ng <= (int)gridDim.x || (c.grid == 2 && ne == 0 && ng <= (int)gridDim.x));
    const int TP = gen || ng == 0 ? 1 : max(1, min(8, min(nb, ne > 0 ? nw / 2 : nw) / ng));
    if (cta_runs) {
      for (int j = blockIdx.x; j < ng; j += gridDim.x) {
        const Op* lead = sp.ops[p] + st.begin + st.n_elem + sp.groups[p][st.gbegin + j];
        warp_terms<false, true, true>(c, lead, lead->na, p);
      }
    } else if (warp < c.bufs) {
      if (TP == 1) {
        for (int j = gb; j < ng; j += nb) {
          const Op* lead = sp.ops[p] + st.begin + st.n_elem + sp.groups[p][st.gbegin + j];
          if (gen)
            warp_terms<true>(c, lead, lead->na, p);
          else
            warp_terms<false>(c, lead, lead->na, p);
        }
      } else {
        Ctx cr = c;
        cr.parts = TP;
        for (int i = gb; i < ng * TP; i += nb) {
          const Op* lead = sp.ops[p] + st.begin + st.n_elem + sp.groups[p][st.gbegin + i / TP];
          cr.part = i % TP;
          warp_terms<false, true>(cr, lead, lead->na, p);
        }
      }
    }
    const int busy = cta_runs ? ng * nw0 : min(ng * TP, nb);
    // node ops in up to 16 parts: a 1128-hand row is 282 float4 columns, so 9
    // parts cover it in one round
    const int P = ne > 0 ? max(1, min(16, (nw - busy) / ne)) : 1;
    const int start = busy % nw;
    Ctx cw = c;
    cw.parts = P;
    for (int i = (gw - start + nw) % nw; i < ne * P; i += nw) {
      const Op op = sp.ops[p][st.begin + i / P];
      cw.part = i % P;
      switch (op.type) {
        case OP_FWD_OPP: op_fwd_opp_t<true>(cw, op, o, mode); break;
        case OP_FWD_CHANCE: op_fwd_chance_t<true>(cw, op, o); break;
        case OP_BWD_TRAV: op_bwd_trav_t<true>(cw, op, p, dc, mode); break;
        case OP_BWD_OPP: op_bwd_opp_t<true>(cw, op, p, mode); break;
        case OP_BWD_CHANCE: op_bwd_chance_t<true>(cw, op, p, mode); break;
        default: break;
      }
    }
    if (!step_barrier(c)) return;
  }
}

__device__ void run_pass(const Ctx& c, int p, const Discount dc, int mode) {
  if (c.split)
    run_pass_split(c, p, dc, mode);
  else
    run_pass_multi(const_cast<Ctx*>(&c), 1, 1u, p, dc, mode);
}

// run_pass_multi; in the SPLIT instantiation of k_solve (launches whose CTAs
// each hold a lone spot), run_pass_split for K == 1.  Batches run the plain
// instantiation, whose code never reaches the split functions.
template <bool SPLIT>
__device__ __forceinline__ void pass_multi(Ctx* cs, int K, unsigned active, int p, const Discount dc, int mode) {
  if (SPLIT && K == 1) {
    if (active & 1u) run_pass_split(cs[0], p, dc, mode);
  } else {
    run_pass_multi(cs, K, active, p, dc, mode);
  }
}

// sum_h w[h] * v[h] accumulated in f64 (utility.rs:118-122) in one fixed
// order, whatever the caller's thread count: 256 strided partial sums
// (h = j, j + 256, ...), the 32 partials of each group j / 32 combined by a
// shuffle tree, the 8 group sums added in order.  One warp computes it
// (result on all its lanes), so a CTA of any size and a single warp of the
// dataflow solve produce the same bits.
__device__ double warp_dot_f64(const float* w, const float* v, int n) {
  const int lane = threadIdx.x & 31;
  double tot = 0.0;
  for (int k = 0; k < 8; ++k) {
    double acc = 0.0;
    for (int h = 32 * k + lane; h < n; h += 256) acc += (double)w[h] * (double)v[h];
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, s);
    tot += __shfl_sync(0xffffffffu, acc, 0);
  }
  return tot;
}

// warp_dot_f64 for a whole CTA: warp 0 computes it, every thread gets it.
__device__ double block_dot_f64(const Ctx& c, const float* w, const float* v, int n) {
  __syncthreads();
  if (threadIdx.x < 32) {
    const double d = warp_dot_f64(w, v, n);
    if (threadIdx.x == 0) c.red[0] = d;
  }
  __syncthreads();
  const double tot = c.red[0];
  __syncthreads();
  return tot;
}

// Exploitability (utility.rs:380-392, :450-543): best-response passes for both
// players, root values weighted by the initial ranges in f64.
// Root value sum_h w[h] v[h] in f64 on every thread; in grid mode CTA 0
// reduces and publishes it to the others through a grid barrier.
__device__ double root_dot(const Ctx& c, const float* w, const float* v, int n, int slot) {
  if (!c.grid) return block_dot_f64(c, w, v, n);
  if (blockIdx.x == 0) {
    const double d = block_dot_f64(c, w, v, n);
    if (threadIdx.x == 0) c.gred[slot] = d;
  }
  grid_barrier(c);
  return *reinterpret_cast<volatile double*>(c.gred + slot);
}

// Exploitability of the active spots of cs (same as spot_exploitability,
// passes shared by the K spots); results in out[k].
template <bool SPLIT>
__device__ void exploitability_multi(Ctx* cs, int K, unsigned active, float* out) {
  const Discount dz{0.f, 0.f, 0.f, 0.f};
  float mes[kMaxInst][2], cur[kMaxInst][2];
  const bool raked = cs[0].sp->raked != 0;  // an instance holds spots of one rake setting
  for (int p = 0; p < 2; ++p) {
    for (int k = 0; k < K; ++k) cs[k].root_reach = cs[k].sp->w[p ^ 1];
    pass_multi<SPLIT>(cs, K, active, p, dz, M_BR);
    for (int k = 0; k < K; ++k)
      if (active >> k & 1u) {
        const SpotDev& sp = *cs[k].sp;
        mes[k][p] = (float)block_dot_f64(cs[k], sp.w[p], slot_at(cs[k], sp.root_slot[p]), sp.H[p]);
      }
  }
  if (raked)
    for (int p = 0; p < 2; ++p) {
      for (int k = 0; k < K; ++k) cs[k].root_reach = cs[k].sp->w[p ^ 1];
      pass_multi<SPLIT>(cs, K, active, p, dz, M_AVG);
      for (int k = 0; k < K; ++k)
        if (active >> k & 1u) {
          const SpotDev& sp = *cs[k].sp;
          cur[k][p] = (float)block_dot_f64(cs[k], sp.w[p], slot_at(cs[k], sp.root_slot[p]), sp.H[p]);
        }
    }
  for (int k = 0; k < K; ++k)
    if (active >> k & 1u)
      out[k] = raked ? ((mes[k][0] - cur[k][0]) + (mes[k][1] - cur[k][1])) * 0.5f : (mes[k][0] + mes[k][1]) * 0.5f;
}

// The strategy-cache bits of DCFR pass p: player 0's strategy is cached by
// pass 1 of the previous iteration, so pass 0 of a launch's first iteration
// computes it.
__device__ __forceinline__ int sg_bits(const SpotDev& sp, int p, bool first) {
  return sp.SG == nullptr ? 0 : SG_WRITE | (p == 1 || !first ? SG_READ : 0);
}

template <bool SPLIT>
__device__ void dcfr_iteration_multi(Ctx* cs, int K, unsigned active, const Discount dc, bool first) {
  for (int p = 0; p < 2; ++p) {  // alternating updates (solver.rs:144-155)
    for (int k = 0; k < K; ++k) {
      cs[k].root_reach = cs[k].sp->w[p ^ 1];
      cs[k].sg = sg_bits(*cs[k].sp, p, first);
    }
    pass_multi<SPLIT>(cs, K, active, p, dc, M_DCFR);
  }
}

__device__ float spot_exploitability(Ctx& c) {
  const SpotDev& sp = *c.sp;
  const Discount dz{0.f, 0.f, 0.f, 0.f};
  float mes[2] = {0.f, 0.f};
  for (int p = 0; p < 2 && grid_live(c); ++p) {
    c.root_reach = sp.w[p ^ 1];
    run_pass(c, p, dz, M_BR);
    mes[p] = (float)root_dot(c, sp.w[p], slot_at(c, sp.root_slot[p]), sp.H[p], p);
  }
  if (!sp.raked) return (mes[0] + mes[1]) * 0.5f;
  float cur[2] = {0.f, 0.f};
  for (int p = 0; p < 2 && grid_live(c); ++p) {
    c.root_reach = sp.w[p ^ 1];
    run_pass(c, p, dz, M_AVG);
    cur[p] = (float)root_dot(c, sp.w[p], slot_at(c, sp.root_slot[p]), sp.H[p], 2 + p);
  }
  return ((mes[0] - cur[0]) + (mes[1] - cur[1])) * 0.5f;
}

__device__ void dcfr_iteration(Ctx& c, const Discount dc, bool first) {
  const SpotDev& sp = *c.sp;
  for (int p = 0; p < 2 && grid_live(c); ++p) {  // alternating updates (solver.rs:144-155)
    c.root_reach = sp.w[p ^ 1];
    c.sg = sg_bits(sp, p, first);
    run_pass(c, p, dc, M_DCFR);
  }
}

// Binds a CTA to a spot: scratch slots, shared-memory regions and the board-0
// tables, copied into shared memory when the plan reserves room for them.
__device__ bool bind_ctx(Ctx& c, const SpotDev* sp, float* scratch, size_t scratch_floats, char* smem,
                         const SmemPlan plan, int* err) {
  c.sp = sp;
  c.vstride = sp->vstride;
  c.owner = -1;
  c.signed_reach = 0;
  c.bgrad = nullptr;
  c.breach = nullptr;
  c.grid = 0;
  c.bar = nullptr;
  c.gred = nullptr;
  c.wait_ns = kGridWaitNs;
  c.sg = 0;
  c.err = err;
  c.slots = scratch;
  char* p = smem;
  const int tb = table_bytes_for(sp->hs[0], sp->hs[1]);
  const bool staged = sp->num_boards == 1 && tb <= plan.tables;
  char* tables = p;
  p += plan.tables;
  const int warp_id = threadIdx.x >> 5;
  c.buf = warp_id < plan.bufs ? reinterpret_cast<float*>(p) + (size_t)warp_id * scan_buf_floats(plan.vstride) : nullptr;
  c.bufs = plan.bufs;
  c.split = plan.split;
  c.part = 0;
  c.parts = 1;
  p += (size_t)plan.bufs * scan_buf_floats(plan.vstride) * 4;
  c.red = reinterpret_cast<double*>(p);
  if ((size_t)sp->num_slots * sp->vstride > scratch_floats || sp->vstride > plan.vstride) {
    if (threadIdx.x == 0) atomicOr(err, ERR_SCRATCH);
    return false;
  }
  for (int q = 0; q < 2; ++q) {
    c.t0.gidx[q] = sp->gidx[q];
    c.t0.heads[q] = sp->heads[q];
    c.t0.thr[q] = reinterpret_cast<const uint4*>(sp->thr[q]);
    c.t0.nvalid[q] = sp->nvalid[q][0];
  }
  if (staged) {
    __syncthreads();  // the previous spot's users of the staged tables are done
    uint4* thr_s = reinterpret_cast<uint4*>(tables);
    uint32_t* hd_s = reinterpret_cast<uint32_t*>(tables + 16 * (sp->hs[0] + sp->hs[1]));
    uint16_t* g_s = reinterpret_cast<uint16_t*>(hd_s + head_words16(sp->hs[0]) + head_words16(sp->hs[1]));
    for (int q = 0; q < 2; ++q) {
      const int hs = sp->hs[q];
      uint4* ts = thr_s + (q ? sp->hs[0] : 0);
      const uint4* tg = reinterpret_cast<const uint4*>(sp->thr[q]);
      for (int i = threadIdx.x; i < hs; i += blockDim.x) ts[i] = tg[i];
      uint32_t* hs_ = hd_s + (q ? head_words16(sp->hs[0]) : 0);
      for (int i = threadIdx.x; i < head_words(hs); i += blockDim.x) hs_[i] = sp->heads[q][i];
      uint16_t* gs = g_s + (q ? 3 * sp->hs[0] : 0);
      for (int i = threadIdx.x; i < 3 * hs; i += blockDim.x) gs[i] = sp->gidx[q][i];
      c.t0.thr[q] = ts;
      c.t0.heads[q] = hs_;
      c.t0.gidx[q] = gs;
    }
    __syncthreads();
  }
  return true;
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
#ifndef PS_LB_MIN
#define PS_LB_MIN 4  // CTAs of kMaxSolveBlock threads per SM the register budget is sized for (64 registers)
#endif
#define PS_SOLVE_BOUNDS __launch_bounds__(kMaxSolveBlock, PS_LB_MIN)

// Batched persistent solve: CTAs pull instances (up to K spots of one tree
// shape) from `counter` and run job's work on them (SolveJob): the full
// reference solve loop (solver.rs:108-176) per spot, or a fixed iteration
// range, then the optional average-strategy epilogue.
template <bool SPLIT>
__global__ void PS_SOLVE_BOUNDS k_solve(const SpotDev* __restrict__ spots, int ninst, int K,
                                        const int* __restrict__ inst, int* counter, const Discount* __restrict__ disc,
                                        SolveJob job, const float* __restrict__ target, float* scratch,
                                        size_t scratch_floats, float* out_expl, int* out_iters, SmemPlan plan,
                                        int* err) {
  extern __shared__ float4 smem4[];
  char* smem = reinterpret_cast<char*>(smem4);
  __shared__ int s_inst;
  float* my_scratch = scratch + (size_t)blockIdx.x * K * scratch_floats;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_inst = atomicAdd(counter, 1);
    __syncthreads();
    const int q = s_inst;
    if (q >= ninst) return;
    // an instance: up to K spots of one tree shape, solved in lockstep
    Ctx cs[kMaxInst];
    int ids[kMaxInst];
    float tgt[kMaxInst], expl[kMaxInst];
    int iters[kMaxInst];
    unsigned active = 0;
    for (int k = 0; k < K; ++k) {
      ids[k] = inst[(size_t)q * K + k];
      if (ids[k] >= 0 && bind_ctx(cs[k], &spots[ids[k]], my_scratch + (size_t)k * scratch_floats, scratch_floats,
                                  smem, plan, err))
        active |= 1u << k;
      else
        cs[k] = cs[0];  // placeholder; never active
      tgt[k] = ids[k] >= 0 ? target[ids[k]] : 0.f;
      expl[k] = 0.f;
      iters[k] = 0;
    }
    if (!active) continue;
    if (job.adjoint) {
      // the fixed-strategy evaluation and its adjoint for every spot, as
      // ps_eval_fixed_strategy_adjoint runs them for one game: forward passes
      // from the spots' weights (values, boundary-gradient factors), then the
      // transposed passes from the cotangents with the payoffs of the other
      // player (owner)
      const Discount dz{0.f, 0.f, 0.f, 0.f};
      for (int k = 0; k < K; ++k) {
        cs[k].signed_reach = 1;
        cs[k].bgrad = cs[k].sp->bgrad;
      }
      for (int pass = 0; pass < 4; ++pass) {
        const int p = pass < 2 ? pass : 3 - pass;  // traversers 0, 1, then 1, 0
        for (int k = 0; k < K; ++k) {
          cs[k].root_reach = pass < 2 ? cs[k].sp->w[p ^ 1] : cs[k].sp->adj_g[p ^ 1];
          cs[k].owner = pass < 2 ? -1 : (p ^ 1);
        }
        pass_multi<SPLIT>(cs, K, active, p, dz, M_AVG);
        for (int k = 0; k < K; ++k) {
          if (!(active >> k & 1u)) continue;
          const SpotDev& sp = *cs[k].sp;
          float* dst = pass < 2 ? sp.root_out[p] : sp.adj_dw[p];
          const float* r = slot_at(cs[k], sp.root_slot[p]);
          for (int h = threadIdx.x; h < sp.H[p]; h += blockDim.x) dst[h] = r[h];
        }
        __syncthreads();
      }
      continue;
    }
    int t = job.t0;
    if (job.checks) {
      // the reference loop per spot (solver.rs:108-176): expl = exploitability;
      // for t < max_iter { if expl <= target break; iterate(t); if (t+1) % 5 == 0
      // || t+1 == max_iter: expl = exploitability }; a spot leaves the lockstep
      // set at the first check that meets its target
      const int max_iter = job.t1;
      exploitability_multi<SPLIT>(cs, K, active, expl);
      unsigned live = 0;
      for (int k = 0; k < K; ++k)
        if ((active >> k & 1u) && !(expl[k] <= tgt[k])) live |= 1u << k;
      for (t = 0; t < max_iter && live; ++t) {
        dcfr_iteration_multi<SPLIT>(cs, K, live, disc[t], t == 0);
        if ((t + 1) % 5 == 0 || t + 1 == max_iter) {
          exploitability_multi<SPLIT>(cs, K, live, expl);
          for (int k = 0; k < K; ++k)
            if ((live >> k & 1u) && expl[k] <= tgt[k]) {
              iters[k] = t + 1;
              live &= ~(1u << k);
            }
        }
      }
      for (int k = 0; k < K; ++k)
        if (live >> k & 1u) iters[k] = t;
    } else {
      // a fixed iteration range (batch.rs:414-535 run_iterations)
      for (; t < job.t1; ++t) dcfr_iteration_multi<SPLIT>(cs, K, active, disc[t], t == job.t0);
      for (int k = 0; k < K; ++k) iters[k] = t;
      if (job.epilogue & EPI_EXPL) exploitability_multi<SPLIT>(cs, K, active, expl);
    }
    if (threadIdx.x == 0 && (job.checks || (job.epilogue & EPI_EXPL)))
      for (int k = 0; k < K; ++k)
        if (active >> k & 1u) {
          out_expl[ids[k]] = expl[k];
          out_iters[ids[k]] = iters[k];
        }
    if (!(job.epilogue & EPI_ROOT)) continue;
    // root cfvalues of both players under the average strategy: the
    // per-hand values a datagen record needs (the reference computes them on
    // the host from the strategy sums); the same passes record the reach at
    // the depth boundaries (batch.rs:765-790 compute_reach_at_nodes)
    const Discount dz{0.f, 0.f, 0.f, 0.f};
    for (int k = 0; k < K; ++k) cs[k].breach = cs[k].sp->breach;
    for (int p = 0; p < 2; ++p) {
      for (int k = 0; k < K; ++k) cs[k].root_reach = cs[k].sp->w[p ^ 1];
      pass_multi<SPLIT>(cs, K, active, p, dz, M_AVG);
      for (int k = 0; k < K; ++k) {
        if (!(active >> k & 1u)) continue;
        const SpotDev& sp = *cs[k].sp;
        if (!sp.root_out[p]) continue;
        const float* r = slot_at(cs[k], sp.root_slot[p]);
        for (int h = threadIdx.x; h < sp.hs[p]; h += blockDim.x) sp.root_out[p][h] = r[h];
      }
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------
// Dataflow batched solve: per-spot steps claimed from a work queue
// ---------------------------------------------------------------------------
// k_flow holds up to kMaxLanes spots per CTA at once ("lanes").  Each lane is
// at its own point of its spot's solve - a pass and a step of that pass - and
// the step's items (terminal runs, and node ops cut into `parts` interleaved
// column blocks) are claimed by warps from two counters per lane: terminal
// runs by the warps that own a scan buffer, node ops by any warp.  The warp
// that finishes a step's last item moves the lane on: to the next step, or at
// the end of a pass to the pass's root work (the exploitability dot products
// and the stop decision of the reference loop, solver.rs:108-176; the root
// values of the epilogue) and the next pass, or - when the spot is solved - to
// the next spot of the batch queue.  So no warp waits at a CTA barrier for the
// slowest item of a step: it takes an item of another lane.  Every item runs
// the same arithmetic as in k_solve, so results are the same bits.
//
// Claims: a 64-bit word per lane and item kind holds (count << 20 | next) of
// the current step.  A claim is an atomicAdd of 1; it is valid when the old
// next < count.  Only the finisher of a step rewrites the words (after the new
// step's fields), and a step cannot end while one of its items is claimed but
// unfinished, so a valid claim always refers to the step whose fields the
// claimer then reads.  Ordering: an item's writes (global and shared) are
// fenced at CTA scope before its completion is counted; the finisher fences
// after the count and before publishing the next step; a claimer fences after
// its claim.
constexpr int kMaxLanes = 8;
constexpr int kMaxFlowBlock = 1024;
enum LanePhase : int { LP_BR0 = 0, LP_BR1, LP_AVG0, LP_AVG1, LP_DCFR0, LP_DCFR1, LP_EPI0, LP_EPI1, LP_RETIRED };

struct Lane {
  unsigned long long wt, wn;  // claims of terminal runs / node-op parts: count << 20 | next
  int done, total;            // finished items of the current step, and its item count
  int begin, n_elem, gbegin, parts;  // the current step (node ops are cut into `parts` column blocks)
  int spot, phase, step, t;   // spot id, pass (LanePhase), step of the pass, iterations done
  float expl, target, mes0, mes1, cur0;
  int iters;
  float* slots;               // the lane's scratch slots
};

__device__ __forceinline__ int lane_player(int phase) { return (phase - LP_BR0) & 1; }
__device__ __forceinline__ int lane_mode(int phase) {
  return phase <= LP_BR1 ? M_BR : phase <= LP_AVG1 ? M_AVG : phase <= LP_DCFR1 ? M_DCFR : M_AVG;
}

__device__ __forceinline__ unsigned long long claim_word(int count) {
  return (unsigned long long)count << 20;
}
// one claim from w (lane 0 of the warp); -1 if none is left
__device__ __forceinline__ int try_claim(unsigned long long* w) {
  const unsigned long long v = *reinterpret_cast<volatile unsigned long long*>(w);
  if ((v & 0xFFFFFull) >= ((v >> 20) & 0xFFFFFull)) return -1;
  const unsigned long long old = atomicAdd(w, 1ull);
  const unsigned nxt = (unsigned)(old & 0xFFFFFull), cnt = (unsigned)((old >> 20) & 0xFFFFFull);
  return nxt < cnt ? (int)nxt : -1;
}

struct FlowArgs {
  const SpotDev* spots;
  int ninst;
  const int* inst;
  int* counter;
  const Discount* disc;
  SolveJob job;
  const float* target;
  float* scratch;
  size_t scratch_floats;
  float* out_expl;
  int* out_iters;
  int* err;
  int lanes;       // lanes per CTA
  int node_parts;  // column blocks per node op (1 = whole ops)
};

// Publications of the CTA's lanes so far.  Items appear only when a step is
// published, so a warp that found none at epoch e scans the claim words again
// only once the epoch has moved: an idle poll is one shared load.
__shared__ unsigned s_flow_epoch;

// Publishes step L.step of the lane's current pass (finisher / binder only).
// A thin step (few terminal runs and node ops) cuts its node ops into more
// column blocks, so that the step offers about PS_FLOW_ADAPT items per warp
// of the CTA's share for this lane (at most one block per 128 hands of the
// wider player); the batch's node_parts is the floor.  Each hand's arithmetic
// is unchanged.  Measured on the 4096 datagen spots at 1024 threads, 3 spots
// and 3 parts per CTA, two runs each on one box: 0 (off) 6976-6977 spots/s,
// 1: 7004-7010, 2: 7068-7085, 3: 7039-7044, 4: 7012-7015.
#ifndef PS_FLOW_ADAPT
#define PS_FLOW_ADAPT 2
#endif
__device__ void lane_publish_step(Lane& L, const SpotDev& sp, int node_parts, int lanes) {
  const int p = lane_player(L.phase);
  const Step st = sp.steps[p][L.step];
  L.begin = st.begin;
  L.n_elem = st.n_elem;
  L.gbegin = st.gbegin;
#if PS_FLOW_ADAPT
  if (st.n_elem > 0) {
    // thin steps: more column blocks, up to one per 32 columns of the wider player
    const int target = (PS_FLOW_ADAPT * (int)(blockDim.x >> 5) + lanes - 1) / lanes;
    const int cap = max(1, (max(sp.hs[0], sp.hs[1]) + 127) >> 7);
    const int want = (target - st.n_groups + st.n_elem - 1) / st.n_elem;
    node_parts = max(node_parts, min(cap, want));
  }
#endif
  L.parts = node_parts;
  L.total = st.n_groups + st.n_elem * node_parts;
  L.done = 0;
  __threadfence_block();
  // The step can end once every item is claimed and done, after which its
  // finisher publishes the next step.  So an empty kind's word (count 0, no
  // claims) goes first and the other last: no exchange of this step can land
  // after a later step's.  With both kinds present, the step cannot end before
  // the second word is out.
  const unsigned long long t = claim_word(st.n_groups), n = claim_word(st.n_elem * node_parts);
  if (st.n_groups == 0) {
    atomicExch(&L.wt, t);
    atomicExch(&L.wn, n);
  } else {
    atomicExch(&L.wn, n);
    atomicExch(&L.wt, t);
  }
  __threadfence_block();  // the claim words before the epoch that announces them
  atomicAdd(&s_flow_epoch, 1u);
}

// The reference loop's decision after a completed exploitability check
// (solver.rs:137-159): stop at the target or at the iteration limit; a
// fixed-range job's closing check ends the spot.  -1 = the spot is finished.
__device__ int lane_after_check(const Lane& L, const FlowArgs& A) {
  if (A.job.checks && !(L.expl <= L.target) && L.t < A.job.t1) return LP_DCFR0;
  return -1;
}

// After an iteration's second pass: a check every 5 iterations and after the
// last one (solve loop), or the next iteration of a fixed range.
__device__ int lane_after_iterations(const Lane& L, const FlowArgs& A) {
  const SolveJob& j = A.job;
  if (j.checks) return (L.t % 5 == 0 || L.t >= j.t1) ? LP_BR0 : LP_DCFR0;
  if (L.t < j.t1) return LP_DCFR0;
  return (j.epilogue & EPI_EXPL) ? LP_BR0 : -1;
}

// Binds the lane to the next spot of the queue (lane 0 of the calling warp);
// false when the queue is empty and the lane retires.  The lane starts before
// the first step of its first pass (step -1).
__device__ bool lane_bind(Lane& L, const FlowArgs& A, float* my_scratch, const SmemPlan& plan) {
  for (;;) {
    const int q = atomicAdd(A.counter, 1);
    if (q >= A.ninst) {
      L.phase = LP_RETIRED;
      return false;
    }
    const int id = A.inst[q];
    if (id < 0) continue;
    const SpotDev& sp = A.spots[id];
    if ((size_t)sp.num_slots * sp.vstride > A.scratch_floats || sp.vstride > plan.vstride) {
      atomicOr(A.err, ERR_SCRATCH);
      continue;
    }
    const SolveJob& j = A.job;
    int phase;
    if (j.checks) {
      L.t = 0;
      phase = LP_BR0;  // the exploitability before the first iteration
    } else {
      L.t = j.t0;
      phase = L.t < j.t1 ? LP_DCFR0 : (j.epilogue & EPI_EXPL) ? LP_BR0 : (j.epilogue & EPI_ROOT) ? LP_EPI0 : -1;
      if (phase < 0) continue;  // nothing to run for this spot
    }
    L.spot = id;
    L.slots = my_scratch;
    L.target = A.target[id];
    L.expl = 0.f;
    L.mes0 = L.mes1 = L.cur0 = 0.f;
    L.iters = 0;
    L.phase = phase;
    L.step = -1;
    return true;
  }
}

// The root work of the pass that just finished and the lane's next phase
// (whole warp; lane 0 owns the scalar state).  -1 = the spot is finished.
__device__ int lane_pass_end(Lane& L, const FlowArgs& A) {
  const SpotDev& sp = A.spots[L.spot];
  const int lane = threadIdx.x & 31;
  const int p = lane_player(L.phase);
  const float* root = L.slots + (size_t)sp.root_slot[p] * sp.vstride;
  int next = -1;
  if (L.phase <= LP_AVG1) {  // a pass of an exploitability check (utility.rs:380-392)
    const float v = (float)warp_dot_f64(sp.w[p], root, sp.H[p]);
    if (lane == 0) {
      bool complete = false;
      if (L.phase == LP_BR0) {
        L.mes0 = v;
        next = LP_BR1;
      } else if (L.phase == LP_BR1) {
        L.mes1 = v;
        if (sp.raked) {
          next = LP_AVG0;
        } else {
          L.expl = (L.mes0 + L.mes1) * 0.5f;
          complete = true;
        }
      } else if (L.phase == LP_AVG0) {
        L.cur0 = v;
        next = LP_AVG1;
      } else {
        L.expl = ((L.mes0 - L.cur0) + (L.mes1 - v)) * 0.5f;
        complete = true;
      }
      if (complete) {
        next = lane_after_check(L, A);
        if (next < 0) L.iters = L.t;
      }
    }
    next = __shfl_sync(0xffffffffu, next, 0);
  } else if (L.phase == LP_DCFR0) {
    next = LP_DCFR1;
  } else if (L.phase == LP_DCFR1) {
    if (lane == 0) {
      L.t += 1;
      next = lane_after_iterations(L, A);
      if (next < 0) L.iters = L.t;
    }
    next = __shfl_sync(0xffffffffu, next, 0);
  } else {  // LP_EPI0 / LP_EPI1: root values under the average strategy
    if (sp.root_out[p])
      for (int h = lane; h < sp.hs[p]; h += 32) sp.root_out[p][h] = root[h];
    return L.phase == LP_EPI0 ? LP_EPI1 : -1;
  }
  if (next < 0 && (A.job.epilogue & EPI_ROOT)) next = LP_EPI0;
  return next;
}

// The finisher's move (whole warp): from the step that just ended (L.step;
// -1 = before a pass) to the next step with items, through the root work of
// any pass that ends and to the next spot when this one is finished.  Leaves
// the lane published (false) or retired (true).  Once a step is published
// other warps own the lane again, so nothing of it is read afterwards.
#ifndef PS_FLOW_MOVE_OUTLINE
#define PS_FLOW_MOVE_OUTLINE 0
#endif
#if PS_FLOW_MOVE_OUTLINE
__device__ __noinline__ bool lane_move(Lane& L, const FlowArgs& A, const SmemPlan& plan) {
#else
__device__ bool lane_move(Lane& L, const FlowArgs& A, const SmemPlan& plan) {
#endif
  const int lane = threadIdx.x & 31;
  for (;;) {
    __syncwarp();
    const SpotDev& sp = A.spots[L.spot];
    const int p = lane_player(L.phase);
    if (L.step + 1 < sp.nsteps[p]) {
      __syncwarp();  // every lane has read the fields above before lane 0 publishes
      if (lane == 0) {
        L.step += 1;
        lane_publish_step(L, sp, A.node_parts, A.lanes);
      }
      return false;
    }
    const int next = lane_pass_end(L, A);
    __syncwarp();
    if (next < 0) {  // the spot is finished: its results, then the next spot
      int bound = 0;
      if (lane == 0) {
        if (A.job.checks || (A.job.epilogue & EPI_EXPL)) {
          A.out_expl[L.spot] = L.expl;
          A.out_iters[L.spot] = L.iters;
        }
        bound = lane_bind(L, A, L.slots, plan);
      }
      if (!__shfl_sync(0xffffffffu, bound, 0)) return true;
      continue;
    }
    if (lane == 0) {
      L.phase = next;
      L.step = -1;
    }
  }
}

// Runs item `idx` of the lane's current step: a terminal run (term) or a
// node-op column block.
__device__ void lane_item(const Lane& L, const FlowArgs& A, int term, int idx, float* buf, int bufs) {
  const SpotDev& sp = A.spots[L.spot];
  const int p = lane_player(L.phase), o = p ^ 1, mode = lane_mode(L.phase);
  Ctx c;
  c.sp = &sp;
  c.slots = L.slots;
  c.vstride = sp.vstride;
  c.root_reach = sp.w[o];
  c.grid = 0;
  c.bar = nullptr;
  c.gred = nullptr;
  c.wait_ns = 0;
  c.err = A.err;
  c.buf = buf;
  c.bufs = bufs;
  c.owner = -1;
  c.signed_reach = 0;
  c.bgrad = nullptr;
  c.breach = L.phase >= LP_EPI0 ? sp.breach : nullptr;
  c.red = nullptr;
  c.split = 0;
  c.part = 0;
  c.parts = 1;
  // the strategy cache: player 0's strategy is cached by pass 1 of the
  // previous iteration, so pass 0 of the spot's first iteration in this
  // launch computes it
  c.sg = 0;
  if (mode == M_DCFR && sp.SG != nullptr)
    c.sg = SG_WRITE | (p == 1 || L.t > (A.job.checks ? 0 : A.job.t0) ? SG_READ : 0);
  for (int q = 0; q < 2; ++q) {
    c.t0.gidx[q] = sp.gidx[q];
    c.t0.heads[q] = sp.heads[q];
    c.t0.thr[q] = reinterpret_cast<const uint4*>(sp.thr[q]);
    c.t0.nvalid[q] = sp.nvalid[q][0];
  }
  const Discount dc = mode == M_DCFR ? A.disc[L.t] : Discount{0.f, 0.f, 0.f, 0.f};
  if (term) {
    const Op* lead = sp.ops[p] + L.begin + L.n_elem + sp.groups[p][L.gbegin + idx];
    if (c.breach)
      warp_terms_inl<true>(c, lead, lead->na, p);
    else
      warp_terms_inl<false>(c, lead, lead->na, p);
    return;
  }
  const int P = L.parts;
  const Op op = sp.ops[p][L.begin + idx / P];
  if (P == 1) {
    switch (op.type) {
      case OP_FWD_OPP: op_fwd_opp(c, op, o, mode); break;
      case OP_FWD_CHANCE: op_fwd_chance(c, op, o); break;
      case OP_BWD_TRAV: op_bwd_trav(c, op, p, dc, mode); break;
      case OP_BWD_OPP: op_bwd_opp(c, op, p, mode); break;
      case OP_BWD_CHANCE: op_bwd_chance(c, op, p, mode); break;
      default: break;
    }
  } else {
    c.part = idx % P;
    c.parts = P;
    switch (op.type) {
      case OP_FWD_OPP: op_fwd_opp_t<true>(c, op, o, mode); break;
      case OP_FWD_CHANCE: op_fwd_chance_t<true>(c, op, o); break;
      case OP_BWD_TRAV: op_bwd_trav_t<true>(c, op, p, dc, mode); break;
      case OP_BWD_OPP: op_bwd_opp_t<true>(c, op, p, mode); break;
      case OP_BWD_CHANCE: op_bwd_chance_t<true>(c, op, p, mode); break;
      default: break;
    }
  }
}

constexpr long long kFlowIdleNs = 2000000000LL;  // 2 s without any finished step in the CTA: give up
#ifndef PS_FLOW_SLEEP_MIN
#define PS_FLOW_SLEEP_MIN 32
#endif
#ifndef PS_FLOW_SLEEP_MAX
#define PS_FLOW_SLEEP_MAX 2048
#endif
constexpr unsigned kFlowSleepMinNs = PS_FLOW_SLEEP_MIN, kFlowSleepMaxNs = PS_FLOW_SLEEP_MAX;  // idle back-off

__global__ void __launch_bounds__(kMaxFlowBlock, 1) k_flow(FlowArgs A, SmemPlan plan) {
  extern __shared__ float4 smem4[];
  char* smem = reinterpret_cast<char*>(smem4);
  __shared__ Lane lanes[kMaxLanes];
  __shared__ int s_retired;
  __shared__ unsigned s_progress;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int K = A.lanes;
  float* buf = warp < plan.bufs
                   ? reinterpret_cast<float*>(smem + plan.tables) + (size_t)warp * scan_buf_floats(plan.vstride)
                   : nullptr;
  // bind every lane to its first spot (warp k binds lane k)
  if (threadIdx.x == 0) {
    s_retired = 0;
    s_progress = 0;
    s_flow_epoch = 0;
  }
  __syncthreads();
  if (warp < K) {
    Lane& L = lanes[warp];
    int bound = 0;
    if (lane == 0) {
      L.wt = L.wn = 0ull;
      L.done = L.total = 0;
      bound = lane_bind(L, A, A.scratch + ((size_t)blockIdx.x * K + warp) * A.scratch_floats, plan);
      if (!bound) atomicAdd(&s_retired, 1);
    }
    if (__shfl_sync(0xffffffffu, bound, 0) && lane_move(L, A, plan) && lane == 0) atomicAdd(&s_retired, 1);
  }
  __syncthreads();
  unsigned seen = 0;
  unsigned long long idle_since = global_ns();
  unsigned backoff = kFlowSleepMinNs, polls = 0;
  unsigned empty_epoch = ~0u;  // lane 0: the epoch of this warp's last scan that found nothing
  int start = warp % K;
  for (;;) {
    int k = -1, idx = -1, term = 0;
    if (lane == 0) {
      const unsigned ep = *reinterpret_cast<volatile unsigned*>(&s_flow_epoch);
      if (ep != empty_epoch) {
        __threadfence_block();  // the claim words published up to epoch ep
        for (int r = 0; r < K && idx < 0; ++r) {
          k = start + r < K ? start + r : start + r - K;
          Lane& L = lanes[k];
          if (buf) {
            idx = try_claim(&L.wt);
            term = idx >= 0;
          }
          if (idx < 0) idx = try_claim(&L.wn);
        }
        if (idx < 0) empty_epoch = ep;
        __threadfence_block();  // acquire: the claimed step's fields and inputs
      }
    }
    idx = __shfl_sync(0xffffffffu, idx, 0);
    if (idx >= 0) {
      k = __shfl_sync(0xffffffffu, k, 0);
      term = __shfl_sync(0xffffffffu, term, 0);
      __syncwarp();
      Lane& L = lanes[k];
      lane_item(L, A, term, idx, buf, plan.bufs);
      __threadfence_block();  // every lane's writes of the item before its count
      __syncwarp();
      int last = 0;
      if (lane == 0) {
        // the step's item count is read before this item is counted: until then
        // the step cannot end, so it is this step's (read after the count, it
        // could be the next step's, published by the real finisher meanwhile)
        const int total = L.total;
        const int d = atomicAdd(&L.done, 1);
        last = d + 1 == total;
        if (last) __threadfence_block();  // acquire: every item of the step
      }
      if (__shfl_sync(0xffffffffu, last, 0)) {
        const bool retired = lane_move(L, A, plan);
        if (lane == 0) {
          if (retired) atomicAdd(&s_retired, 1);
          atomicAdd(&s_progress, 1u);
        }
      }
      start = k;  // stay with this lane while it has work (its rows are warm)
      backoff = kFlowSleepMinNs;
      polls = 0;
      continue;
    }
    // nothing to claim: finished, or wait for a step to end.  Idle warps back
    // off (32 ns doubling to 2048 ns) so their polls take few issue slots from
    // the working ones; the wait bound is checked every 16 polls.
    int stop = 0;
    if (lane == 0) {
      if (*reinterpret_cast<volatile int*>(&s_retired) >= K) {
        stop = 1;
      } else if ((++polls & 15) == 0) {
        const unsigned pr = *reinterpret_cast<volatile unsigned*>(&s_progress);
        const unsigned long long now = global_ns();
        if (pr != seen) {
          seen = pr;
          idle_since = now;
        } else if ((long long)(now - idle_since) > kFlowIdleNs) {
          atomicOr(A.err, ERR_WAIT);
          stop = 1;
        }
      }
    }
    if (__shfl_sync(0xffffffffu, stop, 0)) return;
    __nanosleep(backoff);
    backoff = min(2 * backoff, kFlowSleepMaxNs);
  }
}

// One spot on every CTA of a cooperative launch (large trees).  All CTAs run
// the same loop and take the same decisions: the exploitability reaches them
// through root_dot.  job.kind:
//   GRID_SOLVE    the solve loop of k_solve to job.t1 iterations or job.target
//   GRID_ITERATE  iterations [job.t0, job.t1), no checks
//   GRID_EXPL     exploitability only
//   GRID_FINALIZE the average-strategy passes that store the query values
//   GRID_AVERAGE  one average pass of job.player (k_average with save == 0)
__global__ void PS_SOLVE_BOUNDS k_grid(const SpotDev* __restrict__ spot, const Discount* __restrict__ disc,
                                       float* scratch, size_t scratch_floats, float* out_expl, int* out_iters,
                                       unsigned* bar, double* gred, GridJob job, SmemPlan plan, int* err) {
  extern __shared__ float4 smem4[];
  char* smem = reinterpret_cast<char*>(smem4);
  Ctx c;
  const bool ok = bind_ctx(c, spot, scratch, scratch_floats, smem, plan, err);
  if (!ok) return;  // the check is the same on every CTA
  c.grid = job.cluster ? 2 : 1;
  c.bar = bar;
  c.gred = gred;
  c.wait_ns = job.wait_ns;
  if (threadIdx.x == 0) s_grid_ok = 1;
  __syncthreads();
  const SpotDev& sp = *spot;
  const Discount dz{0.f, 0.f, 0.f, 0.f};
  switch (job.kind) {
    case GRID_ITERATE:
      for (int t = job.t0; t < job.t1 && grid_live(c); ++t) dcfr_iteration(c, disc[t], t == job.t0);
      return;
    case GRID_FINALIZE:
      for (int p = 0; p < 2 && grid_live(c); ++p) {
        c.root_reach = sp.w[p ^ 1];
        run_pass(c, p, dz, M_AVG_SAVE);
      }
      return;
    case GRID_AVERAGE: {
      c.root_reach = job.root_reach ? job.root_reach : sp.w[job.player ^ 1];
      c.signed_reach = job.root_reach != nullptr;
      c.owner = job.owner;
      c.bgrad = job.bgrad;
      c.breach = job.breach;
      run_pass(c, job.player, dz, M_AVG);
      if (blockIdx.x == 0) {
        const float* r = slot_at(c, sp.root_slot[job.player]);
        for (int h = threadIdx.x; h < sp.H[job.player]; h += blockDim.x) job.out[h] = r[h];
      }
      return;
    }
    default:
      break;
  }
  float expl = spot_exploitability(c);
  int t = 0;
  if (job.kind == GRID_SOLVE)
    for (; t < job.t1 && grid_live(c); ++t) {
      if (expl <= job.target) break;
      dcfr_iteration(c, disc[t], t == 0);
      if ((t + 1) % 5 == 0 || t + 1 == job.t1) expl = spot_exploitability(c);
    }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *out_expl = expl;
    if (out_iters) *out_iters = t;
  }
}

// Fixed iteration range [t0, t1) for every spot (CTA-strided), no checks.
__global__ void PS_SOLVE_BOUNDS k_iterate(const SpotDev* __restrict__ spots, int nspots,
                                          const Discount* __restrict__ disc, int t0, int t1, float* scratch,
                                          size_t scratch_floats, SmemPlan plan, int* err) {
  extern __shared__ float4 smem4[];
  char* smem = reinterpret_cast<char*>(smem4);
  float* my_scratch = scratch + (size_t)blockIdx.x * scratch_floats;
  for (int si = blockIdx.x; si < nspots; si += gridDim.x) {
    Ctx c;
    if (!bind_ctx(c, &spots[si], my_scratch, scratch_floats, smem, plan, err)) continue;
    for (int t = t0; t < t1; ++t) dcfr_iteration(c, disc[t], t == t0);
    __syncthreads();
  }
}

__global__ void PS_SOLVE_BOUNDS k_exploitability(const SpotDev* __restrict__ spots, int nspots, float* scratch,
                                                 size_t scratch_floats, float* out, SmemPlan plan, int* err) {
  extern __shared__ float4 smem4[];
  char* smem = reinterpret_cast<char*>(smem4);
  float* my_scratch = scratch + (size_t)blockIdx.x * scratch_floats;
  for (int si = blockIdx.x; si < nspots; si += gridDim.x) {
    Ctx c;
    if (!bind_ctx(c, &spots[si], my_scratch, scratch_floats, smem, plan, err)) continue;
    float e = spot_exploitability(c);
    if (threadIdx.x == 0) out[si] = e;
    __syncthreads();
  }
}

// Average-strategy values (utility.rs:552-795).  save != 0: finalize (stores
// the per-node cfvalues for queries) for both players.  Otherwise one pass for
// `player` from `root_reach` (root_cfvalues_with_reach), root values to out.
//
// owner >= 0 (with save == 0): the adjoint pass of fixed-strategy evaluation.
// The pass runs player's tree program with the average strategy from
// root_reach, but every terminal returns the payoffs of `owner` (the other
// player): out is then the vector-Jacobian product of owner's root cfvalues
// (cotangent root_reach) with respect to player's initial weights.  bgrad
// (when not null) collects the boundary-value gradients: a plain pass stores
// scale * blocked opponent reach at each boundary leaf, the adjoint pass for
// the other player multiplies it by that player's adjoint reach.
__global__ void PS_SOLVE_BOUNDS k_average(const SpotDev* __restrict__ spots, int nspots, int save, int player,
                                          const float* root_reach, float* scratch, size_t scratch_floats, float* out,
                                          int owner, float* bgrad, float* breach, SmemPlan plan, int* err) {
  extern __shared__ float4 smem4[];
  char* smem = reinterpret_cast<char*>(smem4);
  float* my_scratch = scratch + (size_t)blockIdx.x * scratch_floats;
  const Discount dz{0.f, 0.f, 0.f, 0.f};
  for (int si = blockIdx.x; si < nspots; si += gridDim.x) {
    Ctx c;
    if (!bind_ctx(c, &spots[si], my_scratch, scratch_floats, smem, plan, err)) continue;
    const SpotDev& sp = spots[si];
    if (save) {
      for (int p = 0; p < 2; ++p) {
        c.root_reach = sp.w[p ^ 1];
        run_pass(c, p, dz, M_AVG_SAVE);
      }
    } else {
      c.root_reach = root_reach ? root_reach : sp.w[player ^ 1];
      c.signed_reach = root_reach != nullptr;
      c.owner = owner;
      c.bgrad = bgrad;
      c.breach = breach;
      run_pass(c, player, dz, M_AVG);
      const float* r = slot_at(c, sp.root_slot[player]);
      for (int h = threadIdx.x; h < sp.H[player]; h += blockDim.x) out[(size_t)si * sp.hs[player] + h] = r[h];
    }
    __syncthreads();
  }
}

// Single-terminal evaluation for host queries (query.rs:699-712 evaluates a
// terminal with the current weights): reach in slot 0, values out in slot 1.
__global__ void k_eval_terminal(const SpotDev* __restrict__ spots, Op op, int player, float* scratch,
                                size_t scratch_floats, SmemPlan plan, int* err) {
  extern __shared__ float4 smem4[];
  char* smem = reinterpret_cast<char*>(smem4);
  Ctx c;
  if (!bind_ctx(c, &spots[0], scratch, scratch_floats, smem, plan, err)) return;
  c.root_reach = nullptr;
  op.na = 1;
  if (threadIdx.x < 32) warp_terms<false>(c, &op, 1, player);
}

// ---------------------------------------------------------------------------
// Board setup: strengths, orders, card groups and thresholds (card.rs:163-226,
// card.rs:81-156).  One CTA per (spot, board).
// ---------------------------------------------------------------------------
constexpr int kSetupMaxH = 1344;  // >= 1326
constexpr int kSortN = 2048;      // next power of two >= max hands
constexpr int kSortN2 = 4096;     // >= 2 * max valid hands

__device__ void bitonic_sort_u32(uint32_t* a, int n) {  // n power of two, ascending
  for (int k = 2; k <= n; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        int ixj = i ^ j;
        if (ixj > i) {
          uint32_t x = a[i], y = a[ixj];
          bool up = (i & k) == 0;
          if ((x > y) == up) {
            a[i] = y;
            a[ixj] = x;
          }
        }
      }
      __syncthreads();
    }
  }
}

__device__ int lower_bound_u16(const uint16_t* a, int n, uint16_t v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int m = (lo + hi) >> 1;
    if (a[m] < v) lo = m + 1;
    else hi = m;
  }
  return lo;
}
__device__ int upper_bound_u16(const uint16_t* a, int n, uint16_t v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int m = (lo + hi) >> 1;
    if (a[m] <= v) lo = m + 1;
    else hi = m;
  }
  return lo;
}

struct SetupSmem {
  uint32_t keys[kSortN2];
  uint16_t sord[2][kSortN];   // strengths in order, per player
  uint16_t ord[2][kSortN];    // hand index in order
  uint16_t istr[2][kSortN2];  // strength of each card-group entry
  uint16_t coff[2][56];
  uint16_t strength[2][kSetupMaxH];
  int nvalid[2];
};

__global__ void k_setup(const SpotDev* __restrict__ spots, const int2* __restrict__ work, int nwork,
                        const int32_t* __restrict__ table, int* err) {
  extern __shared__ float4 smem4[];
  SetupSmem& S = *reinterpret_cast<SetupSmem*>(smem4);
  for (int wi = blockIdx.x; wi < nwork; wi += gridDim.x) {
    const int2 wk = work[wi];
    const SpotDev& sp = spots[wk.x];
    const int b = wk.y;
    const uint8_t* bc = sp.board_cards + 5 * b;
    const bool full = bc[4] != 255;
    uint64_t bmask = 0;
    for (int k = 0; k < 5; ++k)
      if (bc[k] != 255) bmask |= 1ull << bc[k];
    if (sp.H[0] > kSetupMaxH || sp.H[1] > kSetupMaxH) {
      if (threadIdx.x == 0) atomicOr(err, ERR_SETUP);
      continue;
    }
    for (int q = 0; q < 2; ++q) {
      const int H = sp.H[q];
      const uint8_t* cards = sp.cards[q];
      for (int i = threadIdx.x; i < kSortN; i += blockDim.x) {
        uint32_t key = 0xFFFFFFFFu;
        if (i < H) {
          const int c1 = cards[2 * i], c2 = cards[2 * i + 1];
          const bool ok = !((bmask >> c1) & 1) && !((bmask >> c2) & 1);
          uint16_t st = 0;
          if (ok && full) {
            int c7[7] = {bc[0], bc[1], bc[2], bc[3], bc[4], c1, c2};
            st = (uint16_t)(table_index(table, kHandTableSize, hand_value7(c7)) + 1);
          }
          S.strength[q][i] = st;
          if (ok) key = ((uint32_t)st << 16) | (uint32_t)i;
        }
        S.keys[i] = key;
      }
      __syncthreads();
      bitonic_sort_u32(S.keys, kSortN);
      if (threadIdx.x == 0) S.nvalid[q] = 0;
      __syncthreads();
      for (int i = threadIdx.x; i < kSortN; i += blockDim.x) {
        const uint32_t key = S.keys[i];
        if (key != 0xFFFFFFFFu) {
          S.ord[q][i] = (uint16_t)(key & 0xFFFF);
          S.sord[q][i] = (uint16_t)(key >> 16);
          if (i + 1 == kSortN || S.keys[i + 1] == 0xFFFFFFFFu) S.nvalid[q] = i + 1;
        }
      }
      __syncthreads();
      const int V = S.nvalid[q];
      // card groups: keys (card << 16 | position in strength order)
      for (int i = threadIdx.x; i < kSortN2; i += blockDim.x) {
        uint32_t key = 0xFFFFFFFFu;
        if (i < 2 * V) {
          const int k = i >> 1;
          const int h = S.ord[q][k];
          const int card = cards[2 * h + (i & 1)];
          key = ((uint32_t)card << 16) | (uint32_t)k;
        }
        S.keys[i] = key;
      }
      __syncthreads();
      bitonic_sort_u32(S.keys, kSortN2);
      uint16_t* gidx = sp.gidx[q] + (size_t)b * 3 * sp.hs[q];
      for (int i = threadIdx.x; i < V; i += blockDim.x) gidx[i] = S.ord[q][i];
      for (int i = threadIdx.x; i < 2 * V; i += blockDim.x) {
        const uint32_t key = S.keys[i];
        const int k = key & 0xFFFF;
        gidx[V + i] = S.ord[q][k];
        S.istr[q][i] = S.sord[q][k];
        const int card = key >> 16;
        const int prev = i == 0 ? -1 : (int)(S.keys[i - 1] >> 16);
        for (int cc = prev + 1; cc <= card; ++cc) S.coff[q][cc] = (uint16_t)i;
        if (i == 2 * V - 1)
          for (int cc = card + 1; cc <= 52; ++cc) S.coff[q][cc] = (uint16_t)(2 * V);
      }
      if (V == 0 && threadIdx.x < 53) S.coff[q][threadIdx.x] = 0;
      __syncthreads();
      uint16_t* co = sp.coff[q] + (size_t)b * 56;
      if (threadIdx.x < 56) co[threadIdx.x] = threadIdx.x <= 52 ? S.coff[q][threadIdx.x] : 0;
      if (threadIdx.x == 0) sp.nvalid[q][b] = V;
      // segment starts of the gather list: 0 (strength order) and every non-empty card group
      uint32_t* hd = sp.heads[q] + (size_t)b * head_words(sp.hs[q]);
      for (int i = threadIdx.x; i < head_words(sp.hs[q]); i += blockDim.x) {
        uint32_t wv = 0;
        for (int bit = 0; bit < 32; ++bit) {
          const int k = 32 * i + bit;
          bool h = k == 0 && V > 0;
          if (k >= V && k < 3 * V) {
            const int r = k - V;
            // r starts a group if it equals coff[c] for a non-empty group c
            int lo = 0, hi = 52;
            while (lo < hi) {
              const int m = (lo + hi) >> 1;
              if (S.coff[q][m + 1] <= r) lo = m + 1;
              else hi = m;
            }
            h = S.coff[q][lo] == r;
          }
          if (h) wv |= 1u << bit;
        }
        hd[i] = wv;
      }
      __syncthreads();
    }
    // lookup records of player p's hands against opponent o = p ^ 1, 16 bytes per
    // hand: the scan-buffer positions of the hand's eight prefixes (see the
    // terminal evaluation above); x = ~0 if the hand is blocked on this board.
    // With lt / le the opponent hands strictly weaker / weaker-or-tied and l / e
    // the same counts inside card group c (starting at a_c, n_c entries):
    //   P(k)    = kScanBase - 1 + k           (k = 0 reads the zero below the list)
    //   Q_c(k)  = k ? kScanBase - 1 + V + a_c + k : 0
    //   x = P(lt) | P(le) << 16, y = Q_c1(l1) | Q_c1(e1) << 16,
    //   z = Q_c1(n_c1) | Q_c2(l2) << 16, w = Q_c2(e2) | Q_c2(n_c2) << 16
    for (int p = 0; p < 2; ++p) {
      const int o = p ^ 1;
      const int Hp = sp.H[p], hsp = sp.hs[p], Vo = S.nvalid[o];
      uint4* thr = reinterpret_cast<uint4*>(sp.thr[p]) + (size_t)b * hsp;
      for (int h = threadIdx.x; h < hsp; h += blockDim.x) {
        uint4 v = make_uint4(THR_INVALID, 0, 0, 0);
        if (h < Hp) {
          const int c1 = sp.cards[p][2 * h], c2 = sp.cards[p][2 * h + 1];
          const bool ok = !((bmask >> c1) & 1) && !((bmask >> c2) & 1);
          if (ok) {
            const uint16_t s = S.strength[p][h];
            const uint32_t lt = lower_bound_u16(S.sord[o], Vo, s), le = upper_bound_u16(S.sord[o], Vo, s);
            const int a1 = S.coff[o][c1], n1 = S.coff[o][c1 + 1] - a1;
            const int a2 = S.coff[o][c2], n2 = S.coff[o][c2 + 1] - a2;
            const uint32_t l1 = lower_bound_u16(S.istr[o] + a1, n1, s), e1 = upper_bound_u16(S.istr[o] + a1, n1, s);
            const uint32_t l2 = lower_bound_u16(S.istr[o] + a2, n2, s), e2 = upper_bound_u16(S.istr[o] + a2, n2, s);
            const uint32_t pb = kScanBase - 1, cb = kScanBase - 1 + Vo;
            auto Q = [&](int a, uint32_t k) { return k ? cb + (uint32_t)a + k : 0u; };
            v.x = (pb + lt) | ((pb + le) << 16);
            v.y = Q(a1, l1) | (Q(a1, e1) << 16);
            v.z = Q(a1, (uint32_t)n1) | (Q(a2, l2) << 16);
            v.w = Q(a2, e2) | (Q(a2, (uint32_t)n2) << 16);
          }
        }
        thr[h] = v;
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Host-side launch wrappers
// ---------------------------------------------------------------------------
// The dynamic shared memory a kernel may use is set only when it differs from
// the value set last (per device and context).  Setting it while the kernel
// runs for another batch waits for that launch to end (measured: 440 ms of a
// 600 ms solve, when a datagen job builds its next batch), and back-to-back
// batches of one shape ask for the same value.  It is set exactly, not only
// raised: a larger limit than the launch needs cost the one-game-at-a-time
// path 14% (45.8 -> 39.4 spots/s), as games of different sizes then ran with
// less L1.  The calling thread's last error is cleared on every return, so
// the launch after it reports its own error; a failure is still returned.
struct SmemLimit {
  const void* fn;
  int dev;
  unsigned long long ctx;
  size_t bytes;
};
static std::mutex g_smem_mu;
static std::vector<SmemLimit> g_smem_limits;

static cudaError_t set_smem(const void* fn, size_t bytes) {
  int dev = 0;
  unsigned long long ctx = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = current_context_id(&ctx);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return e;
  }
  std::lock_guard<std::mutex> lk(g_smem_mu);
  SmemLimit* l = nullptr;
  for (auto& x : g_smem_limits)
    if (x.fn == fn && x.dev == dev && x.ctx == ctx) l = &x;
  if (!l || l->bytes != bytes) {
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) {
      if (l)
        l->bytes = bytes;
      else
        g_smem_limits.push_back(SmemLimit{fn, dev, ctx, bytes});
    }
  }
  cudaGetLastError();
  return e;
}

size_t setup_smem_bytes() { return sizeof(SetupSmem); }

cudaError_t launch_setup(const SpotDev* spots, const int2* work, int nwork, const int32_t* table, int* err,
                         int grid, cudaStream_t s) {
  size_t sm = sizeof(SetupSmem);
  cudaError_t e = set_smem((const void*)k_setup, sm);
  if (e != cudaSuccess) return e;
  k_setup<<<grid, 512, sm, s>>>(spots, work, nwork, table, err);
  return cudaGetLastError();
}

cudaError_t launch_solve(const SpotDev* spots, int ninst, int K, const int* inst, int* counter,
                         const Discount* disc, const SolveJob& job, const float* target, float* scratch,
                         size_t scratch_floats, float* out_expl, int* out_iters, int* err, int grid, int block,
                         const SmemPlan& plan, cudaStream_t s) {
  if (K < 1 || K > kMaxInst || job.t0 < 0 || job.t1 < job.t0 || (job.checks && job.t0 != 0) ||
      (job.adjoint && (job.checks || job.t1 != job.t0)))
    return cudaErrorInvalidValue;
  size_t smem = plan.total();
  const void* fn = plan.split ? (const void*)k_solve<true> : (const void*)k_solve<false>;
  cudaError_t e = set_smem(fn, smem);
  if (e != cudaSuccess) return e;
  if (plan.split)
    k_solve<true><<<grid, block, smem, s>>>(spots, ninst, K, inst, counter, disc, job, target, scratch, scratch_floats,
                                     out_expl, out_iters, plan, err);
  else
    k_solve<false><<<grid, block, smem, s>>>(spots, ninst, K, inst, counter, disc, job, target, scratch, scratch_floats,
                                     out_expl, out_iters, plan, err);
  return cudaGetLastError();
}

cudaError_t launch_flow(const SpotDev* spots, int ninst, const int* inst, int* counter, const Discount* disc,
                        const SolveJob& job, const float* target, float* scratch, size_t scratch_floats,
                        float* out_expl, int* out_iters, int* err, int grid, int block, int lanes, int node_parts,
                        const SmemPlan& plan, cudaStream_t s) {
  if (block < 64 || block > kMaxFlowBlock || block % 32 || lanes < 1 || lanes > kMaxLanes || lanes > block / 32 ||
      node_parts < 1 || node_parts > 16 || plan.bufs < 1 || plan.bufs > block / 32 || job.adjoint || job.t0 < 0 ||
      job.t1 < job.t0 || (job.checks && job.t0 != 0))
    return cudaErrorInvalidValue;
  size_t smem = plan.total();
  cudaError_t e = set_smem((const void*)k_flow, smem);
  if (e != cudaSuccess) return e;
  FlowArgs A{spots, ninst, inst, counter, disc, job, target, scratch, scratch_floats, out_expl, out_iters, err,
             lanes, node_parts};
  k_flow<<<grid, block, smem, s>>>(A, plan);
  return cudaGetLastError();
}

int flow_occupancy(int block, const SmemPlan& plan) {
  int n = 0;
  size_t smem = plan.total();
  if (set_smem((const void*)k_flow, smem) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_flow, block, smem) != cudaSuccess) return 0;
  return n;
}

int grid_ctas(int block, const SmemPlan& plan) {
  int dev = 0, nsm = 0, per_sm = 0;
  size_t smem = plan.total();
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  if (set_smem((const void*)k_grid, smem) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_grid, block, smem) != cudaSuccess) return 0;
  return nsm * per_sm;
}

static cudaError_t grid_cluster_attrs() {
  cudaError_t e = cudaFuncSetAttribute((const void*)k_grid, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  return e;
}

int grid_cluster_fits(int ctas, int block, const SmemPlan& plan) {
  if (ctas < 2 || ctas > 16) return 0;
  const size_t smem = plan.total();
  if (set_smem((const void*)k_grid, smem) != cudaSuccess || grid_cluster_attrs() != cudaSuccess) return 0;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = ctas;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(ctas);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, (const void*)k_grid, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n > 0 ? ctas : 0;
}

cudaError_t launch_grid(const SpotDev* spot, const GridJob& job, const Discount* disc, float* scratch,
                        size_t scratch_floats, float* out_expl, int* out_iters, unsigned* bar, double* gred,
                        int* err, int grid, int block, const SmemPlan& plan, cudaStream_t s, int cluster) {
  size_t smem = plan.total();
  cudaError_t e = set_smem((const void*)k_grid, smem);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(bar, 0, 4 * sizeof(unsigned), s);  // count, generation, abort word
  if (e != cudaSuccess) return e;
  GridJob j = job;
  j.cluster = cluster ? 1 : 0;
  SmemPlan pl = plan;
  void* args[] = {(void*)&spot, (void*)&disc, (void*)&scratch, (void*)&scratch_floats, (void*)&out_expl,
                  (void*)&out_iters, (void*)&bar, (void*)&gred, (void*)&j, (void*)&pl, (void*)&err};
  if (!cluster) return cudaLaunchCooperativeKernel((const void*)k_grid, dim3(grid), dim3(block), args, smem, s);
  if (grid < 2 || grid > 16) return cudaErrorInvalidValue;
  if ((e = grid_cluster_attrs()) != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = grid;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelExC(&cfg, (const void*)k_grid, args);
}

cudaError_t launch_iterate(const SpotDev* spots, int nspots, const Discount* disc, int t0, int t1, float* scratch,
                           size_t scratch_floats, int* err, int grid, int block, const SmemPlan& plan,
                           cudaStream_t s) {
  size_t smem = plan.total();
  cudaError_t e = set_smem((const void*)k_iterate, smem);
  if (e != cudaSuccess) return e;
  k_iterate<<<grid, block, smem, s>>>(spots, nspots, disc, t0, t1, scratch, scratch_floats, plan, err);
  return cudaGetLastError();
}

cudaError_t launch_exploitability(const SpotDev* spots, int nspots, float* scratch, size_t scratch_floats,
                                  float* out, int* err, int grid, int block, const SmemPlan& plan, cudaStream_t s) {
  size_t smem = plan.total();
  cudaError_t e = set_smem((const void*)k_exploitability, smem);
  if (e != cudaSuccess) return e;
  k_exploitability<<<grid, block, smem, s>>>(spots, nspots, scratch, scratch_floats, out, plan, err);
  return cudaGetLastError();
}

cudaError_t launch_average(const SpotDev* spots, int nspots, int save, int player, const float* root_reach,
                           float* scratch, size_t scratch_floats, float* out, int* err, int grid, int block,
                           const SmemPlan& plan, cudaStream_t s, int owner, float* bgrad, float* breach) {
  size_t smem = plan.total();
  cudaError_t e = set_smem((const void*)k_average, smem);
  if (e != cudaSuccess) return e;
  k_average<<<grid, block, smem, s>>>(spots, nspots, save, player, root_reach, scratch, scratch_floats, out, owner,
                                       bgrad, breach, plan,
                                       err);
  return cudaGetLastError();
}

cudaError_t launch_eval_terminal(const SpotDev* spots, Op op, int player, float* scratch, size_t scratch_floats,
                                 int* err, int block, const SmemPlan& plan, cudaStream_t s) {
  size_t smem = plan.total();
  cudaError_t e = set_smem((const void*)k_eval_terminal, smem);
  if (e != cudaSuccess) return e;
  k_eval_terminal<<<1, block, smem, s>>>(spots, op, player, scratch, scratch_floats, plan, err);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Exploitability without allocation
// ---------------------------------------------------------------------------
// Some hosts cannot allocate device memory at the moment they evaluate a game:
// an engine that reserves the GPU's memory for its own pool at start-up and
// lets plug-ins use only what they were given, or a caller on a latency-bound
// thread where cudaMalloc's implicit device synchronisation is not allowed.
// For them the working slots of the exploitability kernel live in this fixed
// array, sized once at build time: a 256-byte header (word 0 the result, word
// 1 the kernel's error flag) followed by kFixedScratchFloats floats of slots.
static __device__ __align__(256) float g_fixed_scratch[kFixedScratchHeader + kFixedScratchFloats];

static std::mutex g_fixed_mu;
struct FixedBase {
  unsigned long long ctx = 0;  // id of the context the address belongs to (0 = none yet)
  float* p = nullptr;
};
static FixedBase g_fixed_base[64];  // per device ordinal

// The driver's context functions, reached through the runtime (no link to libcuda).
using CtxGetCurrentFn = int (*)(void**);
using CtxGetIdFn = int (*)(void*, unsigned long long*);
static CtxGetCurrentFn g_ctx_get_current = nullptr;
static CtxGetIdFn g_ctx_get_id = nullptr;
static std::once_flag g_ctx_once;

cudaError_t current_context_id(unsigned long long* id) {
  std::call_once(g_ctx_once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(f);
  });
  if (!g_ctx_get_current || !g_ctx_get_id) return cudaErrorNotSupported;
  // cudaSetDevice makes the device's primary context current, creating it
  // first when there is none: on a new thread, or after a cudaDeviceReset,
  // which leaves the destroyed context current until the runtime's next call
  // that needs one
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = cudaSetDevice(dev);
  if (e != cudaSuccess) return e;
  void* ctx = nullptr;
  if (g_ctx_get_current(&ctx) != 0 || !ctx) return cudaErrorDeviceUninitialized;
  return g_ctx_get_id(ctx, id) == 0 ? cudaSuccess : cudaErrorDeviceUninitialized;
}

// The array's address in the current context, looked up on the first call in
// each context (a device reset ends the context that the old address belonged to).
static cudaError_t fixed_scratch_base(float** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  unsigned long long ctx = 0;
  e = current_context_id(&ctx);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_fixed_mu);
  FixedBase& fb = g_fixed_base[dev];
  if (fb.ctx != ctx || !fb.p) {
    float* p = nullptr;
    e = cudaGetSymbolAddress((void**)&p, g_fixed_scratch);
    if (e != cudaSuccess) return e;
    fb.p = p;
    fb.ctx = ctx;
  }
  *out = fb.p;
  return cudaSuccess;
}

cudaError_t launch_exploitability_fixed(const SpotDev* spot, size_t slot_floats, int block, const SmemPlan& plan,
                                        cudaStream_t s, float* host_out, int* host_err) {
  if (slot_floats > kFixedScratchFloats) return cudaErrorInvalidValue;
  float* base = nullptr;
  cudaError_t e = fixed_scratch_base(&base);
  if (e != cudaSuccess) return e;
  // the header keeps the previous call's result and flag: clear it; the
  // slots need no clearing, every pass writes a slot before reading it
  e = cudaMemsetAsync(base, 0, kFixedScratchHeader * sizeof(float), s);
  if (e != cudaSuccess) return e;
  size_t smem = plan.total();
  e = set_smem((const void*)k_exploitability, smem);
  if (e != cudaSuccess) return e;
  k_exploitability<<<1, block, smem, s>>>(spot, 1, base + kFixedScratchHeader, slot_floats, base, plan,
                                          reinterpret_cast<int*>(base + 1));
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  float head[2];
  e = cudaMemcpyAsync(head, base, sizeof(head), cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return e;
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  *host_out = head[0];
  __builtin_memcpy(host_err, &head[1], sizeof(int));
  return cudaSuccess;
}

// Test hook of the bounded grid barrier (launch_debug_barrier_timeout): CTA 0
// enters `rounds` grid barriers that the other CTAs never join - or, with
// all_join, that every CTA joins (the cost of a grid barrier).
__global__ void k_debug_barrier_timeout(unsigned* bar, int* err, int* passed, int rounds, long long wait_ns,
                                        int all_join) {
  Ctx c{};
  c.grid = 1;
  c.bar = bar;
  c.err = err;
  c.wait_ns = wait_ns;
  if (threadIdx.x == 0) s_grid_ok = 1;
  __syncthreads();
  if (blockIdx.x != 0 && !all_join) return;
  int n = 0;
  for (int r = 0; r < rounds; ++r)
    if (grid_barrier(c)) ++n;
  if (threadIdx.x == 0 && blockIdx.x == 0) *passed = n;
}

cudaError_t launch_debug_barrier_timeout(int ctas, int rounds, long long wait_ns, int all_join, unsigned* bar,
                                         int* err, int* passed, cudaStream_t s) {
  int dev = 0, nsm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  // at most one 64-thread CTA per SM: every CTA of the cooperative launch is resident
  if (ctas < 2 || ctas > nsm || rounds < 1 || wait_ns < 0 || wait_ns > kGridWaitNs) return cudaErrorInvalidValue;
  e = cudaMemsetAsync(bar, 0, 4 * sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  void* args[] = {(void*)&bar, (void*)&err, (void*)&passed, (void*)&rounds, (void*)&wait_ns, (void*)&all_join};
  return cudaLaunchCooperativeKernel((const void*)k_debug_barrier_timeout, dim3(ctas), dim3(64), args, 0, s);
}

#ifdef PS_PHASE_TIMERS
extern "C" int ps_debug_phase_cycles(unsigned long long* out, int n) {
  unsigned long long z[16] = {};
  if (n > 16) n = 16;
  if (cudaMemcpyFromSymbol(out, g_phase, sizeof(unsigned long long) * n) != cudaSuccess) return -3;
  if (cudaMemcpyToSymbol(g_phase, z, sizeof(z)) != cudaSuccess) return -3;
  return n;
}
#endif

int solve_occupancy(int block, const SmemPlan& plan) {
  int n = 0;
  size_t smem = plan.total();
  set_smem((const void*)k_solve<false>, smem);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_solve<false>, block, smem) != cudaSuccess) return 1;
  return n < 1 ? 1 : n;
}

}  // namespace ps
