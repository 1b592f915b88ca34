// CUDA kernels of the B200 range solver (sm_100a).
//
// Work decomposition: one CTA owns one game ("spot") at a time and walks its
// level-ordered tree program (ps_device.hpp): forward steps propagate the
// opponent's reach top-down, backward steps evaluate terminals and combine
// children bottom-up with the DCFR regret / strategy update fused in.  Every
// hand vector is processed by all threads of the CTA (one hand per thread per
// sweep of the loop); steps are separated by __syncthreads only, so a whole
// solve of a spot - all iterations plus the exploitability checks - runs
// inside one persistent launch that pulls spots from a device work queue.
//
// Terminal evaluation restates crates/range-solver/src/game/evaluation.rs
// without its sequential merge: the opponent reach is gathered into
// hand-strength order and into per-card groups (both precomputed per board by
// k_setup), scanned with warp shuffles, and every hand reads its win / lose /
// blocked sums at precomputed thresholds - O(n) work per terminal.
#include <cuda_runtime.h>
#include <stdint.h>

#include "ps_device.hpp"
#include "ps_handeval.hpp"

namespace ps {

enum Mode { M_DCFR = 0, M_BR = 1, M_AVG = 2, M_AVG_SAVE = 3 };

// Error bits reported through the error word of every launch.
constexpr int ERR_SCRATCH = 1;  // a spot needed more scratch than its CTA owns
constexpr int ERR_SETUP = 2;    // setup tables exceeded their bounds

struct Ctx {
  const SpotDev* sp;
  float* slots;
  int vstride;
  const float* root_reach;
  float* rch;    // smem: staged opponent reach  [vstride]
  float* buf;    // smem: scan results           [3 * vstride]
  float* carry;  // smem: per-warp chunk totals  [32]
  double* red;   // smem: reduction scratch      [32]
};

__device__ __forceinline__ const float* slot_in(const Ctx& c, uint16_t id) {
  return id == SLOT_ROOT_REACH ? c.root_reach : c.slots + (size_t)id * c.vstride;
}
__device__ __forceinline__ float* slot_at(const Ctx& c, uint16_t id) {
  return c.slots + (size_t)id * c.vstride;
}

// max(x, y) of the reference (sliceop.rs:5-12): no NaN propagation.
__device__ __forceinline__ float fmax_ref(float x, float y) { return x > y ? x : y; }

__device__ __forceinline__ float warp_incl_scan(float x, int lane) {
#pragma unroll
  for (int s = 1; s < 32; s <<= 1) {
    float y = __shfl_up_sync(0xffffffffu, x, s);
    if (lane >= s) x += y;
  }
  return x;
}

// ---------------------------------------------------------------------------
// Forward ops
// ---------------------------------------------------------------------------

// Opponent decision node (solver.rs:418-445; utility.rs:227-250 for BR / AVG):
// sigma from regret matching (DCFR) or from the normalised cumulative strategy,
// then children's reach = sigma_a * reach.
template <int MODE>
__device__ void op_fwd_opp(const Ctx& c, const Op& op, int o) {
  const SpotDev& sp = *c.sp;
  const int hso = sp.hs[o], na = op.na;
  const float* base = (MODE == M_DCFR ? sp.R : sp.S) + sp.nodes[op.node].rs_off;
  const float* src = slot_in(c, op.src);
  float* dst = slot_at(c, op.blk);
  const float def = 1.0f / (float)na;
  for (int h = threadIdx.x; h < hso; h += blockDim.x) {
    float v[kMaxActions];
    float d = 0.f;
#pragma unroll
    for (int a = 0; a < kMaxActions; ++a) {
      if (a < na) {
        float x = base[a * hso + h];
        v[a] = MODE == M_DCFR ? fmax_ref(x, 0.0f) : x;
        d = a == 0 ? v[a] : __fadd_rn(d, v[a]);
      }
    }
    const float r = src[h];
#pragma unroll
    for (int a = 0; a < kMaxActions; ++a)
      if (a < na) dst[(size_t)a * c.vstride + h] = __fmul_rn(d == 0.0f ? def : __fdiv_rn(v[a], d), r);
  }
}

// Chance node (solver.rs:264-276): one scaled reach shared by all children.
__device__ void op_fwd_chance(const Ctx& c, const Op& op, int o) {
  const SpotDev& sp = *c.sp;
  const int hso = sp.hs[o];
  const float f = __fdiv_rn(1.0f, (float)sp.nodes[op.node].chance_factor);
  const float* src = slot_in(c, op.src);
  float* dst = slot_at(c, op.blk);
  for (int h = threadIdx.x; h < hso; h += blockDim.x) dst[h] = __fmul_rn(src[h], f);
}

// ---------------------------------------------------------------------------
// Backward ops
// ---------------------------------------------------------------------------

// Traverser decision node.
//   DCFR (solver.rs:333-416, :556-589): sigma = regret match(R); cfv = sum sigma_a cfv_a;
//        S = S * gamma + sigma; R = R * (R >= +0 ? alpha : beta) + cfv_a - cfv.
//   BR   (utility.rs:953-966): cfv = max_a cfv_a.
//   AVG  (utility.rs:689-727): sigma = S / sum S; cfv = sum sigma_a cfv_a; SAVE stores cfv_a.
template <int MODE>
__device__ void op_bwd_trav(const Ctx& c, const Op& op, int p, const Discount dc) {
  const SpotDev& sp = *c.sp;
  const int hsp = sp.hs[p], na = op.na;
  const NodeDev nd = sp.nodes[op.node];
  float* R = sp.R + nd.rs_off;
  float* S = sp.S + nd.rs_off;
  const float* cb = slot_at(c, op.blk);
  float* dst = slot_at(c, op.dst);
  const float def = 1.0f / (float)na;
  for (int h = threadIdx.x; h < hsp; h += blockDim.x) {
    float cv[kMaxActions];
#pragma unroll
    for (int a = 0; a < kMaxActions; ++a)
      if (a < na) cv[a] = cb[(size_t)a * c.vstride + h];
    float res = 0.f;
    if (MODE == M_BR) {
      res = cv[0];
#pragma unroll
      for (int a = 1; a < kMaxActions; ++a)
        if (a < na) res = fmax_ref(res, cv[a]);
    } else if (MODE == M_DCFR) {
      float r[kMaxActions], m[kMaxActions];
      float d = 0.f;
#pragma unroll
      for (int a = 0; a < kMaxActions; ++a) {
        if (a < na) {
          r[a] = R[a * hsp + h];
          m[a] = fmax_ref(r[a], 0.0f);
          d = a == 0 ? m[a] : __fadd_rn(d, m[a]);
        }
      }
#pragma unroll
      for (int a = 0; a < kMaxActions; ++a) {
        if (a < na) {
          m[a] = d == 0.0f ? def : __fdiv_rn(m[a], d);
          float t = __fmul_rn(m[a], cv[a]);
          res = a == 0 ? t : __fadd_rn(res, t);
          S[a * hsp + h] = __fadd_rn(__fmul_rn(S[a * hsp + h], dc.gamma), m[a]);
        }
      }
#pragma unroll
      for (int a = 0; a < kMaxActions; ++a) {
        if (a < na) {
          float coef = signbit(r[a]) ? dc.beta : dc.alpha;
          R[a * hsp + h] = __fsub_rn(__fadd_rn(__fmul_rn(r[a], coef), cv[a]), res);
        }
      }
    } else {
      float s[kMaxActions];
      float d = 0.f;
#pragma unroll
      for (int a = 0; a < kMaxActions; ++a) {
        if (a < na) {
          s[a] = S[a * hsp + h];
          d = a == 0 ? s[a] : __fadd_rn(d, s[a]);
        }
      }
#pragma unroll
      for (int a = 0; a < kMaxActions; ++a) {
        if (a < na) {
          float t = __fmul_rn(d == 0.0f ? def : __fdiv_rn(s[a], d), cv[a]);
          res = a == 0 ? t : __fadd_rn(res, t);
          if (MODE == M_AVG_SAVE) R[a * hsp + h] = cv[a];
        }
      }
    }
    dst[h] = res;
    if (MODE == M_AVG_SAVE && p == 1 && nd.ip_off != 0xFFFFFFFFu && h < sp.H[1]) sp.ipcfv[nd.ip_off + h] = res;
  }
}

// Opponent decision node: cfv = sum_a cfv_a (solver.rs:471).
template <int MODE>
__device__ void op_bwd_opp(const Ctx& c, const Op& op, int p) {
  const SpotDev& sp = *c.sp;
  const int hsp = sp.hs[p], na = op.na;
  const NodeDev nd = sp.nodes[op.node];
  const float* cb = slot_at(c, op.blk);
  float* dst = slot_at(c, op.dst);
  for (int h = threadIdx.x; h < hsp; h += blockDim.x) {
    float res = cb[h];
    for (int a = 1; a < na; ++a) res = __fadd_rn(res, cb[(size_t)a * c.vstride + h]);
    dst[h] = res;
    if (MODE == M_AVG_SAVE && p == 1 && nd.ip_off != 0xFFFFFFFFu && h < sp.H[1]) sp.ipcfv[nd.ip_off + h] = res;
  }
}

// Chance node: cfv = sum over dealt cards, plus the suit-swapped rows of the
// isomorphic cards that were not dealt (solver.rs:291-325).
template <int MODE>
__device__ void op_bwd_chance(const Ctx& c, const Op& op, int p) {
  const SpotDev& sp = *c.sp;
  const int hsp = sp.hs[p], na = op.na;
  const NodeDev nd = sp.nodes[op.node];
  const float* cb = slot_at(c, op.blk);
  float* dst = slot_at(c, op.dst);
  int i0 = 0, i1 = 0;
  if (op.board != 0xFFFF) {
    i0 = sp.iso_off[op.board];
    i1 = sp.iso_off[op.board + 1];
  }
  for (int h = threadIdx.x; h < hsp; h += blockDim.x) {
    float res = cb[h];
    for (int a = 1; a < na; ++a) res = __fadd_rn(res, cb[(size_t)a * c.vstride + h]);
    for (int i = i0; i < i1; ++i) {
      const int ref = sp.iso_ent[2 * i], perm = sp.iso_ent[2 * i + 1];
      const int hh = sp.iso_perm[p][(size_t)perm * hsp + h];
      res = __fadd_rn(res, cb[(size_t)ref * c.vstride + hh]);
    }
    dst[h] = res;
    if (MODE == M_AVG_SAVE && nd.ch_player == p && h < sp.H[p]) sp.chcfv[nd.ch_off + h] = res;
  }
}

// ---------------------------------------------------------------------------
// Terminal evaluation (game/evaluation.rs:57-634)
// ---------------------------------------------------------------------------
//
// Per board b and opponent o the gather list holds the V valid opponent hands
// in (strength, index) order followed by, for every card c, the valid
// opponent hands holding c in the same order (segment [coff[c], coff[c+1])).
// After the scans, for a hand h with thresholds
//   lt = #opp weaker, le = #opp weaker-or-tied, ltc / lec = the same counts
//   inside each of its two card segments,
// the reference's sums are prefix lookups:
//   win  = P(lt) - Q_c1(ltc1) - Q_c2(ltc2)       (strictly weaker, not blocked)
//   lose = (T - P(le)) - (M_c1 - Q_c1(lec1)) - (M_c2 - Q_c2(lec2))
//   fold = T + r_same - M_c1 - M_c2               (inclusion-exclusion)
__device__ void op_term(const Ctx& c, const Op& op, int p) {
  const SpotDev& sp = *c.sp;
  const int o = p ^ 1;
  const int Ho = sp.H[o], Hp = sp.H[p], hso = sp.hs[o], hsp = sp.hs[p];
  const int b = op.board;
  const int V = sp.nvalid[o][b];
  const uint16_t* g = sp.gidx[o] + (size_t)b * 3 * hso;
  const uint16_t* co = sp.coff[o] + (size_t)b * 56;
  const float* src = slot_in(c, op.src);
  float* dst = slot_at(c, op.dst);
  float* rch = c.rch;
  float* buf = c.buf;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;

  __syncthreads();  // the previous terminal's lookups are done with rch / buf
  for (int i = tid; i < Ho; i += nt) rch[i] = src[i];
  __syncthreads();

  const int ntile = (V + 31) >> 5;
  const int cpw = (ntile + nw - 1) / nw;
  {  // strength-ordered segment: each warp scans a contiguous chunk of tiles
    float run = 0.f;
    const int t0 = warp * cpw, t1 = min(ntile, t0 + cpw);
    for (int t = t0; t < t1; ++t) {
      const int k = t * 32 + lane;
      float x = k < V ? rch[g[k]] : 0.f;
      x = warp_incl_scan(x, lane) + run;
      if (k < V) buf[k] = x;
      run = __shfl_sync(0xffffffffu, x, 31);
    }
    if (lane == 0) c.carry[warp] = run;
  }
  for (int cc = warp; cc < 52; cc += nw) {  // per-card segments
    const int s0 = co[cc], s1 = co[cc + 1];
    float run = 0.f;
    for (int k0 = s0; k0 < s1; k0 += 32) {
      const int k = k0 + lane;
      float x = k < s1 ? rch[g[V + k]] : 0.f;
      x = warp_incl_scan(x, lane) + run;
      if (k < s1) buf[V + k] = x;
      run = __shfl_sync(0xffffffffu, x, 31);
    }
  }
  __syncthreads();

  // exclusive prefix of the chunk totals, one per lane
  float cpre = lane < nw ? c.carry[lane] : 0.f;
  {
    float incl = warp_incl_scan(cpre, lane);
    cpre = incl - cpre;
  }
  const NodeDev nd = sp.nodes[op.node];
  const uint16_t* thr = sp.thr[p] + (size_t)b * hsp * kThrWords;
  const uint8_t* pc = sp.cards[p];
  const uint16_t* same = sp.same[p];
  // T = sum of all valid opponent reach
  float T;
  {
    int j = V - 1;
    int w = j >= 0 ? (j >> 5) / cpw : 0;
    float base = j >= 0 ? buf[j] : 0.f;
    float add = __shfl_sync(0xffffffffu, cpre, w & 31);
    T = j >= 0 ? base + add : 0.f;
  }
  for (int h0 = 0; h0 < hsp; h0 += nt) {  // uniform trip count: shuffles below
    const int h = h0 + tid;
    float v = 0.f;
    uint4 t = make_uint4(0, 0, 0, 0);
    if (h < Hp) t = *reinterpret_cast<const uint4*>(thr + (size_t)h * kThrWords);
    const int lt = t.x & 0xFFFF, le = t.x >> 16;
    // prefix sums over the strength-ordered part need the chunk carry
    const int jl = lt - 1, je = le - 1;
    const int wl = jl >= 0 ? (jl >> 5) / cpw : 0, we = je >= 0 ? (je >> 5) / cpw : 0;
    const float cl = __shfl_sync(0xffffffffu, cpre, wl & 31);
    const float ce = __shfl_sync(0xffffffffu, cpre, we & 31);
    const bool valid = h < Hp && (t.w & 0xFFFF) != 0 && V > 0;
    if (valid) {
      const int c1 = pc[2 * h], c2 = pc[2 * h + 1];
      const int s1a = co[c1], s1b = co[c1 + 1], s2a = co[c2], s2b = co[c2 + 1];
      const float* q1 = buf + V + s1a;
      const float* q2 = buf + V + s2a;
      const float M1 = s1b > s1a ? q1[s1b - s1a - 1] : 0.f;
      const float M2 = s2b > s2a ? q2[s2b - s2a - 1] : 0.f;
      if (op.term == TERM_SHOWDOWN) {
        const int ltc1 = t.y & 0xFFFF, lec1 = t.y >> 16, ltc2 = t.z & 0xFFFF, lec2 = t.z >> 16;
        const float Plt = jl >= 0 ? buf[jl] + cl : 0.f;
        const float Ple = je >= 0 ? buf[je] + ce : 0.f;
        const float Q1lt = ltc1 > 0 ? q1[ltc1 - 1] : 0.f, Q1le = lec1 > 0 ? q1[lec1 - 1] : 0.f;
        const float Q2lt = ltc2 > 0 ? q2[ltc2 - 1] : 0.f, Q2le = lec2 > 0 ? q2[lec2 - 1] : 0.f;
        const float win = Plt - Q1lt - Q2lt;
        if (!sp.raked) {
          const float lose = (T - Ple) - (M1 - Q1le) - (M2 - Q2le);
          v = __fadd_rn(__fmul_rn(nd.amount_win, win), __fmul_rn(nd.amount_lose, lose));
        } else {
          const uint16_t si = same[h];
          const float rs = si != 0xFFFF ? rch[si] : 0.f;
          const float tie = Ple - Q1le - Q2le;
          const float tot = T - M1 - M2;
          v = nd.amount_win * win + nd.amount_tie * (tie - win + rs) + nd.amount_lose * (tot - tie);
        }
      } else {
        const uint16_t si = same[h];
        const float rs = si != 0xFFFF ? rch[si] : 0.f;
        const float adj = T + rs - M1 - M2;
        if (op.term == TERM_FOLD) {
          v = __fmul_rn(op.fold_pl != p ? nd.amount_win : nd.amount_lose, adj);
        } else {
          const float bv = sp.bcfv[((size_t)nd.boundary * 2 + p) * c.vstride + h];
          v = __fmul_rn(__fmul_rn(bv, nd.payoff_scale), adj);
        }
      }
    }
    if (h < hsp) dst[h] = v;
  }
}

// ---------------------------------------------------------------------------
// Pass driver and root reductions
// ---------------------------------------------------------------------------
template <int MODE>
__device__ void run_pass(const Ctx& c, int p, const Discount dc) {
  const SpotDev& sp = *c.sp;
  const Step* steps = sp.steps[p];
  const Op* ops = sp.ops[p];
  const int o = p ^ 1;
  for (int s = 0; s < sp.nsteps[p]; ++s) {
    const Step st = steps[s];
    for (int i = 0; i < st.n_elem; ++i) {
      const Op op = ops[st.begin + i];
      switch (op.type) {
        case OP_FWD_OPP: op_fwd_opp<MODE>(c, op, o); break;
        case OP_FWD_CHANCE: op_fwd_chance(c, op, o); break;
        case OP_BWD_TRAV: op_bwd_trav<MODE>(c, op, p, dc); break;
        case OP_BWD_OPP: op_bwd_opp<MODE>(c, op, p); break;
        case OP_BWD_CHANCE: op_bwd_chance<MODE>(c, op, p); break;
        default: break;
      }
    }
    for (int i = 0; i < st.n_term; ++i) op_term(c, ops[st.begin + st.n_elem + i], p);
    __syncthreads();
  }
}

// sum_h w[h] * v[h] accumulated in f64 (utility.rs:118-122), result on all threads.
__device__ double block_dot_f64(const Ctx& c, const float* w, const float* v, int n) {
  double acc = 0.0;
  for (int h = threadIdx.x; h < n; h += blockDim.x) acc += (double)w[h] * (double)v[h];
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, s);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) c.red[warp] = acc;
  __syncthreads();
  double tot = 0.0;
  for (int i = 0; i < nw; ++i) tot += c.red[i];
  __syncthreads();
  return tot;
}

// Exploitability (utility.rs:380-392, :450-543): best-response passes for both
// players, root values weighted by the initial ranges in f64.
__device__ float spot_exploitability(Ctx& c) {
  const SpotDev& sp = *c.sp;
  const Discount dz{0.f, 0.f, 0.f, 0.f};
  float mes[2];
  for (int p = 0; p < 2; ++p) {
    c.root_reach = sp.w[p ^ 1];
    run_pass<M_BR>(c, p, dz);
    mes[p] = (float)block_dot_f64(c, sp.w[p], slot_at(c, sp.root_slot[p]), sp.H[p]);
  }
  if (!sp.raked) return (mes[0] + mes[1]) * 0.5f;
  float cur[2];
  for (int p = 0; p < 2; ++p) {
    c.root_reach = sp.w[p ^ 1];
    run_pass<M_AVG>(c, p, dz);
    cur[p] = (float)block_dot_f64(c, sp.w[p], slot_at(c, sp.root_slot[p]), sp.H[p]);
  }
  return ((mes[0] - cur[0]) + (mes[1] - cur[1])) * 0.5f;
}

__device__ void dcfr_iteration(Ctx& c, const Discount dc) {
  const SpotDev& sp = *c.sp;
  for (int p = 0; p < 2; ++p) {  // alternating updates (solver.rs:144-155)
    c.root_reach = sp.w[p ^ 1];
    run_pass<M_DCFR>(c, p, dc);
  }
}

__device__ bool bind_ctx(Ctx& c, const SpotDev* sp, float* scratch, size_t scratch_floats, float* smem,
                         int* err) {
  c.sp = sp;
  c.vstride = sp->vstride;
  c.slots = scratch;
  c.rch = smem;
  c.buf = smem + sp->vstride;
  c.carry = smem + 4 * sp->vstride;
  c.red = reinterpret_cast<double*>(smem + 4 * sp->vstride + 32);
  if ((size_t)sp->num_slots * sp->vstride > scratch_floats) {
    if (threadIdx.x == 0) atomicOr(err, ERR_SCRATCH);
    return false;
  }
  return true;
}

// Dynamic shared memory needed for a given max vstride.
__host__ __device__ inline size_t smem_bytes(int vstride) { return (size_t)(4 * vstride + 32) * 4 + 32 * 8; }

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------

// Batched persistent solve: CTAs pull spots from `counter` (in `order`), and
// run the full reference solve loop (solver.rs:108-176) per spot:
//   expl = exploitability; for t < max_iter { if expl <= target break;
//   iterate(t); if (t+1) % 5 == 0 || t+1 == max_iter: expl = exploitability }.
__global__ void k_solve(const SpotDev* __restrict__ spots, int nspots, const int* __restrict__ order,
                        int* counter, const Discount* __restrict__ disc, int max_iter,
                        const float* __restrict__ target, float* scratch, size_t scratch_floats,
                        float* out_expl, int* out_iters, int* err) {
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  __shared__ int s_spot;
  float* my_scratch = scratch + (size_t)blockIdx.x * scratch_floats;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_spot = atomicAdd(counter, 1);
    __syncthreads();
    const int k = s_spot;
    if (k >= nspots) return;
    const int si = order ? order[k] : k;
    Ctx c;
    if (!bind_ctx(c, &spots[si], my_scratch, scratch_floats, smem, err)) continue;
    const float tgt = target[si];
    float expl = spot_exploitability(c);
    int t = 0;
    for (; t < max_iter; ++t) {
      if (expl <= tgt) break;
      dcfr_iteration(c, disc[t]);
      if ((t + 1) % 5 == 0 || t + 1 == max_iter) expl = spot_exploitability(c);
    }
    if (threadIdx.x == 0) {
      out_expl[si] = expl;
      out_iters[si] = t;
    }
  }
}

// Fixed iteration range [t0, t1) for every spot (CTA-strided), no checks.
__global__ void k_iterate(const SpotDev* __restrict__ spots, int nspots, const Discount* __restrict__ disc,
                          int t0, int t1, float* scratch, size_t scratch_floats, int* err) {
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  float* my_scratch = scratch + (size_t)blockIdx.x * scratch_floats;
  for (int si = blockIdx.x; si < nspots; si += gridDim.x) {
    Ctx c;
    if (!bind_ctx(c, &spots[si], my_scratch, scratch_floats, smem, err)) continue;
    for (int t = t0; t < t1; ++t) dcfr_iteration(c, disc[t]);
    __syncthreads();
  }
}

__global__ void k_exploitability(const SpotDev* __restrict__ spots, int nspots, float* scratch,
                                 size_t scratch_floats, float* out, int* err) {
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  float* my_scratch = scratch + (size_t)blockIdx.x * scratch_floats;
  for (int si = blockIdx.x; si < nspots; si += gridDim.x) {
    Ctx c;
    if (!bind_ctx(c, &spots[si], my_scratch, scratch_floats, smem, err)) continue;
    float e = spot_exploitability(c);
    if (threadIdx.x == 0) out[si] = e;
    __syncthreads();
  }
}

// Average-strategy values (utility.rs:552-795).  save != 0: finalize (stores
// the per-node cfvalues for queries) for both players.  Otherwise one pass for
// `player` from `root_reach` (root_cfvalues_with_reach), root values to out.
__global__ void k_average(const SpotDev* __restrict__ spots, int nspots, int save, int player,
                          const float* root_reach, float* scratch, size_t scratch_floats, float* out,
                          int* err) {
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  float* my_scratch = scratch + (size_t)blockIdx.x * scratch_floats;
  const Discount dz{0.f, 0.f, 0.f, 0.f};
  for (int si = blockIdx.x; si < nspots; si += gridDim.x) {
    Ctx c;
    if (!bind_ctx(c, &spots[si], my_scratch, scratch_floats, smem, err)) continue;
    const SpotDev& sp = spots[si];
    if (save) {
      for (int p = 0; p < 2; ++p) {
        c.root_reach = sp.w[p ^ 1];
        run_pass<M_AVG_SAVE>(c, p, dz);
      }
    } else {
      c.root_reach = root_reach ? root_reach : sp.w[player ^ 1];
      run_pass<M_AVG>(c, player, dz);
      const float* r = slot_at(c, sp.root_slot[player]);
      for (int h = threadIdx.x; h < sp.H[player]; h += blockDim.x) out[(size_t)si * sp.hs[player] + h] = r[h];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Board setup: strengths, orders, card groups and thresholds (card.rs:163-226,
// card.rs:81-156).  One CTA per (spot, board).
// ---------------------------------------------------------------------------
constexpr int kSetupMaxH = 1344;  // >= 1326 rounded for sorting headroom
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
  uint16_t istr[2][kSortN2 / 2 * 2];  // strength of each card-group entry
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
      __syncthreads();
    }
    // thresholds of player p's hands against opponent o = p ^ 1
    for (int p = 0; p < 2; ++p) {
      const int o = p ^ 1;
      const int Hp = sp.H[p], hsp = sp.hs[p], Vo = S.nvalid[o];
      uint16_t* thr = sp.thr[p] + (size_t)b * hsp * kThrWords;
      for (int h = threadIdx.x; h < hsp; h += blockDim.x) {
        uint16_t r[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (h < Hp) {
          const int c1 = sp.cards[p][2 * h], c2 = sp.cards[p][2 * h + 1];
          const bool ok = !((bmask >> c1) & 1) && !((bmask >> c2) & 1);
          if (ok) {
            const uint16_t s = S.strength[p][h];
            r[0] = (uint16_t)lower_bound_u16(S.sord[o], Vo, s);
            r[1] = (uint16_t)upper_bound_u16(S.sord[o], Vo, s);
            const int a1 = S.coff[o][c1], n1 = S.coff[o][c1 + 1] - a1;
            const int a2 = S.coff[o][c2], n2 = S.coff[o][c2 + 1] - a2;
            r[2] = (uint16_t)lower_bound_u16(S.istr[o] + a1, n1, s);
            r[3] = (uint16_t)upper_bound_u16(S.istr[o] + a1, n1, s);
            r[4] = (uint16_t)lower_bound_u16(S.istr[o] + a2, n2, s);
            r[5] = (uint16_t)upper_bound_u16(S.istr[o] + a2, n2, s);
            r[6] = 1;
          }
        }
        uint4 v;
        v.x = r[0] | ((uint32_t)r[1] << 16);
        v.y = r[2] | ((uint32_t)r[3] << 16);
        v.z = r[4] | ((uint32_t)r[5] << 16);
        v.w = r[6] | ((uint32_t)r[7] << 16);
        *reinterpret_cast<uint4*>(thr + (size_t)h * kThrWords) = v;
      }
    }
    __syncthreads();
  }
}

size_t setup_smem_bytes() { return sizeof(SetupSmem); }

}  // namespace ps

// ---------------------------------------------------------------------------
// Single-terminal evaluation for host queries (query.rs:699-712 evaluates a
// terminal with the current weights): reach in slot 0, values out in slot 1.
// ---------------------------------------------------------------------------
namespace ps {
__global__ void k_eval_terminal(const SpotDev* __restrict__ spots, Op op, int player, float* scratch,
                                size_t scratch_floats, int* err) {
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  Ctx c;
  if (!bind_ctx(c, &spots[0], scratch, scratch_floats, smem, err)) return;
  c.root_reach = nullptr;
  op_term(c, op, player);
}

// ---------------------------------------------------------------------------
// Host-side launch wrappers
// ---------------------------------------------------------------------------
static cudaError_t set_smem(const void* fn, size_t bytes) {
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

size_t solve_smem(int vstride) { return smem_bytes(vstride); }

cudaError_t launch_setup(const SpotDev* spots, const int2* work, int nwork, const int32_t* table, int* err,
                         int grid, cudaStream_t s) {
  size_t sm = sizeof(SetupSmem);
  cudaError_t e = set_smem((const void*)k_setup, sm);
  if (e != cudaSuccess) return e;
  k_setup<<<grid, 512, sm, s>>>(spots, work, nwork, table, err);
  return cudaGetLastError();
}

cudaError_t launch_solve(const SpotDev* spots, int nspots, const int* order, int* counter, const Discount* disc,
                         int max_iter, const float* target, float* scratch, size_t scratch_floats, float* out_expl,
                         int* out_iters, int* err, int grid, int block, size_t smem, cudaStream_t s) {
  cudaError_t e = set_smem((const void*)k_solve, smem);
  if (e != cudaSuccess) return e;
  k_solve<<<grid, block, smem, s>>>(spots, nspots, order, counter, disc, max_iter, target, scratch,
                                     scratch_floats, out_expl, out_iters, err);
  return cudaGetLastError();
}

cudaError_t launch_iterate(const SpotDev* spots, int nspots, const Discount* disc, int t0, int t1,
                           float* scratch, size_t scratch_floats, int* err, int grid, int block, size_t smem,
                           cudaStream_t s) {
  cudaError_t e = set_smem((const void*)k_iterate, smem);
  if (e != cudaSuccess) return e;
  k_iterate<<<grid, block, smem, s>>>(spots, nspots, disc, t0, t1, scratch, scratch_floats, err);
  return cudaGetLastError();
}

cudaError_t launch_exploitability(const SpotDev* spots, int nspots, float* scratch, size_t scratch_floats,
                                  float* out, int* err, int grid, int block, size_t smem, cudaStream_t s) {
  cudaError_t e = set_smem((const void*)k_exploitability, smem);
  if (e != cudaSuccess) return e;
  k_exploitability<<<grid, block, smem, s>>>(spots, nspots, scratch, scratch_floats, out, err);
  return cudaGetLastError();
}

cudaError_t launch_average(const SpotDev* spots, int nspots, int save, int player, const float* root_reach,
                           float* scratch, size_t scratch_floats, float* out, int* err, int grid, int block,
                           size_t smem, cudaStream_t s) {
  cudaError_t e = set_smem((const void*)k_average, smem);
  if (e != cudaSuccess) return e;
  k_average<<<grid, block, smem, s>>>(spots, nspots, save, player, root_reach, scratch, scratch_floats, out, err);
  return cudaGetLastError();
}

cudaError_t launch_eval_terminal(const SpotDev* spots, Op op, int player, float* scratch, size_t scratch_floats,
                                 int* err, int block, size_t smem, cudaStream_t s) {
  cudaError_t e = set_smem((const void*)k_eval_terminal, smem);
  if (e != cudaSuccess) return e;
  k_eval_terminal<<<1, block, smem, s>>>(spots, op, player, scratch, scratch_floats, err);
  return cudaGetLastError();
}

int solve_occupancy(int block, size_t smem) {
  int n = 0;
  set_smem((const void*)k_solve, smem);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_solve, block, smem) != cudaSuccess) return 1;
  return n < 1 ? 1 : n;
}
}  // namespace ps
