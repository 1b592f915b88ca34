// Device side of the turn-datagen boundary pipeline: the reach-weighted
// average of boundary-value-network outputs over the 48 river cards, with card
// blocking (cfvnet/src/datagen/gpu_boundary_eval.rs:207-269 does it on the
// host in f64, and it is that pipeline's measured bottleneck).
//
// For boundary item i, player p (opponent o), river r of the 48 cards not on
// the item's 4-card board and combo c:
//   w_o[r]  = sum over combos c' without card r of reach_o[c']          (f64)
//   cfv_p[h] = (pot + stack) * sum_{r not in hand h} w_o[r] * net[i][p][r][c(h)]
//                              / sum_{r not in hand h} w_o[r]            (0 if the sum is 0)
// Player 0 is weighted by IP reach, player 1 by OOP reach, as in the reference.
#include <cuda_runtime.h>
#include <stdint.h>

namespace ps {

constexpr int kRivers = 48;
constexpr int kCombos = 1326;

// (c1, c2), c1 < c2, of a combo index (inverse of card.rs:50-55): c1 is the
// last card whose first combo, c1 * (101 - c1) / 2 + c1, is at most idx
__device__ __forceinline__ void combo_cards(int idx, int& c1, int& c2) {
  int a = 0;
  while (a + 1 < 51 && (a + 1) * (101 - (a + 1)) / 2 + (a + 1) <= idx) ++a;
  c1 = a;
  c2 = idx - a * (101 - a) / 2 + 1;
}

__global__ void k_boundary_river_reduce(int n, const uint8_t* __restrict__ boards, const float* __restrict__ denorm,
                                        const float* __restrict__ net, const float* __restrict__ reach,
                                        const int32_t* __restrict__ hands, int H, float* __restrict__ out) {
  const int item = blockIdx.x >> 1, p = blockIdx.x & 1, o = p ^ 1;
  if (item >= n) return;
  __shared__ double s_w[kRivers];
  __shared__ double s_red[32];
  __shared__ uint8_t s_river[kRivers];
  const uint8_t* bd = boards + 4 * item;
  if (threadIdx.x == 0) {
    int k = 0;
    for (int c = 0; c < 52; ++c)
      if (c != bd[0] && c != bd[1] && c != bd[2] && c != bd[3]) s_river[k++] = (uint8_t)c;
  }
  // total opponent reach
  const float* ro = reach + ((size_t)item * 2 + o) * kCombos;
  double t = 0.0;
  for (int c = threadIdx.x; c < kCombos; c += blockDim.x) t += (double)ro[c];
  for (int s = 16; s > 0; s >>= 1) t += __shfl_down_sync(0xffffffffu, t, s);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += s_red[w];
    s_red[0] = tot;
  }
  __syncthreads();
  const double total = s_red[0];
  // per river: total minus the reach of the 51 combos holding the river card
  for (int ri = threadIdx.x; ri < kRivers; ri += blockDim.x) {
    const int r = s_river[ri];
    double blocked = 0.0;
    for (int x = 0; x < 52; ++x) {
      if (x == r) continue;
      const int a = x < r ? x : r, b = x < r ? r : x;
      blocked += (double)ro[a * (101 - a) / 2 + b - 1];
    }
    s_w[ri] = total - blocked;
  }
  __syncthreads();
  const float* np_ = net + ((size_t)item * 2 + p) * kRivers * kCombos;
  const double scale = (double)denorm[item];
  for (int h = threadIdx.x; h < H; h += blockDim.x) {
    const int combo = hands[h];
    if (combo < 0 || combo >= kCombos) {  // not a combo: no value
      out[((size_t)item * 2 + p) * H + h] = 0.0f;
      continue;
    }
    int c1, c2;
    combo_cards(combo, c1, c2);
    double num = 0.0, den = 0.0;
    for (int ri = 0; ri < kRivers; ++ri) {
      const int r = s_river[ri];
      if (r == c1 || r == c2) continue;
      num += s_w[ri] * (double)np_[(size_t)ri * kCombos + combo];
      den += s_w[ri];
    }
    out[((size_t)item * 2 + p) * H + h] = den > 0.0 ? (float)(num / den * scale) : 0.0f;
  }
}

cudaError_t launch_boundary_river_reduce(int n, const uint8_t* boards, const float* denorm, const float* net,
                                         const float* reach, const int32_t* hands, int H, float* out,
                                         cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_boundary_river_reduce<<<2 * n, 256, 0, s>>>(n, boards, denorm, net, reach, hands, H, out);
  return cudaGetLastError();
}

}  // namespace ps
