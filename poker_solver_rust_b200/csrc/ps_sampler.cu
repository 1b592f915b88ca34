// Situation sampling on the device: boards, pot / stack and two R(S,p) ranges
// per situation (cfvnet datagen/sampler.rs:30-60, :142-205 and
// datagen/range_gen.rs:18-167), one block per situation.
//
// Random numbers: a counter-based SplitMix64 stream (Vigna's published
// generator), key(i) = mix(seed + (i + 1) * G), draw(i, c) = mix(key(i) +
// (c + 1) * G), so that every draw of every situation is addressable and the
// R(S,p) recursion runs in parallel.  The reference draws from rand's ChaCha8
// in recursion order; the distribution is the same, the stream is not.
// Counters: board cards from 0, pot / stack from 1 << 16, range r's split at
// the node covering sorted positions [lo, hi) at ((r + 1) << 32) | lo << 12 | hi.
#include <cuda_runtime.h>
#include <stdint.h>

#include "ps_launch.hpp"

namespace ps {

namespace {

constexpr int kCombosS = 1326;
constexpr uint64_t kGolden = 0x9E3779B97F4A7C15ull;

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ uint64_t draw(uint64_t key, uint64_t ctr) { return mix64(key + (ctr + 1) * kGolden); }

// uniform integer in [0, n) from the top 32 bits (multiply-shift)
__device__ __forceinline__ int draw_int(uint64_t key, uint64_t ctr, uint32_t n) {
  return (int)(((draw(key, ctr) >> 32) * (uint64_t)n) >> 32);
}

// uniform double in [0, 1) with 53 random bits
__device__ __forceinline__ double draw_unit(uint64_t key, uint64_t ctr) {
  return (double)(draw(key, ctr) >> 11) * 0x1.0p-53;
}

__device__ __forceinline__ int top_bits(int x, int n) {  // the n highest set bits of x
  int r = 0;
  for (int k = 0; k < n && x; ++k) {
    const int b = 1 << (31 - __clz(x));
    r |= b;
    x ^= b;
  }
  return r;
}

__device__ __forceinline__ int straight_top(int ranks) {  // top-rank bit of a 5-rank run (wheel: the five)
  const int run = ranks & (ranks << 1) & (ranks << 2) & (ranks << 3) & (ranks << 4);
  if (run) return top_bits(run, 1);
  return (ranks & 0x100F) == 0x100F ? 1 << 3 : 0;
}

// 7-card value with the encoding of range_gen.rs:184-268: category << 26,
// then the ranks that decide within the category (primary set << 13 | kickers).
__device__ int eval7(const int* cards) {
  int all = 0, suited[4] = {0, 0, 0, 0}, cnt[13];
  for (int r = 0; r < 13; ++r) cnt[r] = 0;
  for (int k = 0; k < 7; ++k) {
    const int r = cards[k] >> 2;
    all |= 1 << r;
    suited[cards[k] & 3] |= 1 << r;
    ++cnt[r];
  }
  int by_count[5] = {0, 0, 0, 0, 0};
  for (int r = 0; r < 13; ++r) by_count[cnt[r]] |= 1 << r;
  int flush = -1;
  for (int s = 0; s < 4; ++s)
    if (__popc(suited[s]) >= 5) flush = s;
  if (flush >= 0) {
    const int sf = straight_top(suited[flush]);
    return sf ? (8 << 26) | sf : (5 << 26) | top_bits(suited[flush], 5);
  }
  if (by_count[4]) return (7 << 26) | (by_count[4] << 13) | top_bits(all ^ by_count[4], 1);
  if (__popc(by_count[3]) == 2) {
    const int t = top_bits(by_count[3], 1);
    return (6 << 26) | (t << 13) | (by_count[3] ^ t);
  }
  if (by_count[3] && by_count[2]) return (6 << 26) | (by_count[3] << 13) | top_bits(by_count[2], 1);
  const int st = straight_top(all);
  if (st) return (4 << 26) | st;
  if (by_count[3]) return (3 << 26) | (by_count[3] << 13) | top_bits(by_count[1], 2);
  if (__popc(by_count[2]) >= 2) {
    const int two = top_bits(by_count[2], 2);
    return (2 << 26) | (two << 13) | top_bits(all ^ two, 1);
  }
  if (by_count[2]) return (1 << 26) | (by_count[2] << 13) | top_bits(by_count[1], 3);
  return top_bits(all, 5);
}

__device__ __forceinline__ void combo_pair(int idx, int& c1, int& c2) {
  int a = 0;
  while (a + 1 < 51 && (a + 1) * (101 - (a + 1)) / 2 + (a + 1) <= idx) ++a;
  c1 = a;
  c2 = idx - a * (101 - a) / 2 + 1;
}

}  // namespace

__global__ void k_sample_situations(SamplerParams P, uint8_t* __restrict__ boards, int32_t* __restrict__ pots,
                                    int32_t* __restrict__ stacks, float* __restrict__ ranges, int* err) {
  const int64_t idx = P.first + blockIdx.x;
  const uint64_t key = mix64(P.seed + (uint64_t)(idx + 1) * kGolden);
  __shared__ double s_val[kCombosS];
  __shared__ uint16_t s_pos[kCombosS];
  __shared__ int s_board[5], s_pot, s_stack, s_nvalid, s_bad;
  const int bs = P.board_size;
  if (threadIdx.x == 0) {
    // sampler.rs:142-160: cards by rejection until bs distinct ones
    uint64_t used = 0, ctr = 0;
    int bad = 0;
    for (int k = 0; k < bs; ++k) {
      int c;
      do {
        c = draw_int(key, ctr++, 52);
      } while ((used >> c & 1) && ctr < 4096);
      if (used >> c & 1) bad = 1;
      used |= 1ull << c;
      s_board[k] = c;
    }
    for (int k = bs; k < 5; ++k) s_board[k] = 0;
    // pot and stack (sampler.rs:42-51, :165-205)
    uint64_t pc = 1u << 16;
    int pot = 0, stack = 0;
    if (P.nspr == 0) {
      const int iv = draw_int(key, pc++, (uint32_t)P.npot);
      const int lo = P.pot[iv][0], hi = P.pot[iv][1];
      pot = lo + draw_int(key, pc++, (uint32_t)(hi - lo));
      const int max_stack = P.initial_stack - pot / 2;
      stack = max_stack < 5 ? 5 : 5 + draw_int(key, pc++, (uint32_t)(max_stack - 5 + 1));
    } else {
      const double sf = (double)P.initial_stack;
      bool found = false;
      for (int attempt = 0; attempt < 10000 && !found; ++attempt) {
        const int si = draw_int(key, pc++, (uint32_t)P.nspr);
        const double slo = P.spr[si][0], shi = P.spr[si][1];
        const double spr = slo + draw_unit(key, pc++) * (shi - slo);
        const double pmin = spr > 0.0 ? ceil(5.0 / spr) : ceil(2.0 * (sf - 5.0));
        const double pmax = sf / (spr + 0.5);
        const int flo = (int)fmin(fmax(pmin, 1.0), 1.0e9), fhi = (int)pmax;
        if (flo > fhi) continue;
        int blo[kMaxSamplerIntervals], bhi[kMaxSamplerIntervals], nb = 0;
        for (int k = 0; k < P.npot; ++k) {
          const int lo = max(P.pot[k][0], flo), hi = min(P.pot[k][1], fhi + 1);
          if (lo < hi) {
            blo[nb] = lo;
            bhi[nb] = hi;
            ++nb;
          }
        }
        if (nb == 0) continue;
        const int b = draw_int(key, pc++, (uint32_t)nb);
        const int p = blo[b] + draw_int(key, pc++, (uint32_t)(bhi[b] - blo[b]));
        const int max_stack = P.initial_stack - p / 2;
        if (max_stack < 5) continue;
        const int s = min(max((int)fmin(round(spr * (double)p), 2.0e9), 5), max_stack);
        const double actual = (double)s / (double)p;
        if (actual >= slo && actual < shi) {
          pot = p;
          stack = s;
          found = true;
        }
      }
      if (!found) bad = 1;
    }
    s_pot = pot;
    s_stack = stack;
    s_bad = bad;
  }
  __syncthreads();
  if (s_bad) {
    if (threadIdx.x == 0) atomicExch(err, 1);
    return;
  }
  uint64_t bmask = 0;
  for (int k = 0; k < bs; ++k) bmask |= 1ull << s_board[k];
  // hand strengths (range_gen.rs:18-56): the 7-card value on a 5-card board,
  // its average over the 46 river cards on a 4-card board; 0 = blocked
  for (int c = threadIdx.x; c < kCombosS; c += blockDim.x) {
    int c1, c2;
    combo_pair(c, c1, c2);
    const uint64_t hm = (1ull << c1) | (1ull << c2);
    double v = 0.0;
    if (!(hm & bmask)) {
      int cards[7] = {c1, c2, s_board[0], s_board[1], s_board[2], s_board[3], s_board[4]};
      if (bs == 5) {
        v = (double)eval7(cards);
      } else {
        long long sum = 0;
        int n = 0;
        for (int r = 0; r < 52; ++r) {
          if ((bmask | hm) >> r & 1) continue;
          cards[6] = r;
          sum += eval7(cards);
          ++n;
        }
        v = (double)sum / (double)n;
      }
    }
    s_val[c] = v;
  }
  __syncthreads();
  // position of each valid combo in the stable ascending order (ties by index)
  int nv = 0;
  for (int c = threadIdx.x; c < kCombosS; c += blockDim.x) {
    const double v = s_val[c];
    if (v <= 0.0) continue;
    int pos = 0;
    for (int d = 0; d < kCombosS; ++d) {
      const double w = s_val[d];
      pos += (w > 0.0) && (w < v || (w == v && d < c));
    }
    s_pos[c] = (uint16_t)pos;
    ++nv;
  }
  nv = __reduce_add_sync(0xffffffffu, nv);
  if (threadIdx.x == 0) s_nvalid = 0;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) atomicAdd(&s_nvalid, nv);
  __syncthreads();
  const int n = s_nvalid;
  // R(S,p) (range_gen.rs:120-167): each node of the recursion over sorted
  // positions [lo, hi) splits its mass p at a uniform point; the larger part
  // goes to the stronger half [lo + len/2, hi).  A combo's mass is the product
  // along its root-to-leaf path, in the recursion's f64 arithmetic.
  const size_t out0 = (size_t)blockIdx.x * 2 * kCombosS;
  for (int r = 0; r < 2; ++r)
    for (int c = threadIdx.x; c < kCombosS; c += blockDim.x) {
      float m = 0.f;
      if (s_val[c] > 0.0) {
        const int k = s_pos[c];
        int lo = 0, hi = n;
        double p = 1.0;
        while (hi - lo > 1 && p > 0.0) {
          const double u = draw_unit(key, ((uint64_t)(r + 1) << 32) | ((uint64_t)lo << 12) | (uint64_t)hi);
          const double d = u * p, rem = p - d;
          const int mid = lo + (hi - lo) / 2;
          if (k >= mid) {
            p = fmax(d, rem);
            lo = mid;
          } else {
            p = fmin(d, rem);
            hi = mid;
          }
        }
        m = p > 0.0 ? (float)p : 0.f;
      }
      ranges[out0 + (size_t)r * kCombosS + c] = m;
    }
  if (threadIdx.x == 0) {
    for (int k = 0; k < 5; ++k) boards[(size_t)blockIdx.x * 5 + k] = (uint8_t)s_board[k];
    pots[blockIdx.x] = s_pot;
    stacks[blockIdx.x] = s_stack;
  }
}

cudaError_t launch_sample_situations(const SamplerParams& P, int n, uint8_t* boards, int32_t* pots, int32_t* stacks,
                                     float* ranges, int* err, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_sample_situations<<<n, 256, 0, s>>>(P, boards, pots, stacks, ranges, err);
  return cudaGetLastError();
}

}  // namespace ps
