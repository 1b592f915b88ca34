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
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "ps_launch.hpp"

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

__device__ __forceinline__ double net_value(const float* p, size_t i) { return (double)p[i]; }
__device__ __forceinline__ double net_value(const __nv_bfloat16* p, size_t i) { return (double)__bfloat162float(p[i]); }

template <typename T>
__global__ void k_boundary_river_reduce(int n, const uint8_t* __restrict__ boards, const float* __restrict__ denorm,
                                        const T* __restrict__ net, const float* __restrict__ reach,
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
  const T* np_ = net + ((size_t)item * 2 + p) * kRivers * kCombos;
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
      num += s_w[ri] * net_value(np_, (size_t)ri * kCombos + combo);
      den += s_w[ri];
    }
    out[((size_t)item * 2 + p) * H + h] = den > 0.0 ? (float)(num / den * scale) : 0.0f;
  }
}

// combo index of two distinct cards (card.rs:50-55)
__device__ __forceinline__ int combo_index(int a, int b) {
  const int lo = a < b ? a : b, hi = a < b ? b : a;
  return lo * (101 - lo) / 2 + hi - 1;
}

// One block per boundary item (spot, ordinal), both players: between the
// spot's hand-order rows (stride vstride) and the item's 1326-combo rows.
__global__ void k_boundary_combo(const SpotDev* __restrict__ spots, const int2* __restrict__ items, int which,
                                 const float* __restrict__ in, float* __restrict__ out) {
  const int2 it = items[blockIdx.x];
  const SpotDev& sp = spots[it.x];
  for (int p = 0; p < 2; ++p) {
    const uint8_t* cards = sp.cards[p];
    const size_t hrow = ((size_t)it.y * 2 + p) * sp.vstride;
    const size_t crow = ((size_t)blockIdx.x * 2 + p) * kCombos;
    if (which == BC_SET_VALUES) {
      float* dst = const_cast<float*>(sp.bcfv) + hrow;
      const float* src = in + crow;
      for (int h = threadIdx.x; h < sp.vstride; h += blockDim.x)
        dst[h] = h < sp.H[p] ? src[combo_index(cards[2 * h], cards[2 * h + 1])] : 0.f;
    } else {
      const float* from = which == BC_REACH ? sp.breach : sp.bgrad;
      float* dst = out + crow;
      for (int c = threadIdx.x; c < kCombos; c += blockDim.x) dst[c] = 0.f;
      __syncthreads();
      if (from)
        for (int h = threadIdx.x; h < sp.H[p]; h += blockDim.x)
          dst[combo_index(cards[2 * h], cards[2 * h + 1])] = from[hrow + h];
      __syncthreads();
    }
  }
}

cudaError_t launch_boundary_combo(const SpotDev* spots, const int2* items, int nitems, int which,
                                  const float* in, float* out, cudaStream_t s) {
  if (nitems <= 0) return cudaSuccess;
  k_boundary_combo<<<nitems, 256, 0, s>>>(spots, items, which, in, out);
  return cudaGetLastError();
}

// One block per spot, both players: between the spot's hand-order vectors and
// its 1326-combo rows.
__global__ void k_spot_combo(const SpotDev* __restrict__ spots, int which, const float* __restrict__ in,
                             float* __restrict__ out) {
  const SpotDev& sp = spots[blockIdx.x];
  for (int p = 0; p < 2; ++p) {
    const uint8_t* cards = sp.cards[p];
    const size_t crow = ((size_t)blockIdx.x * 2 + p) * kCombos;
    if (which == SC_COT) {
      float* dst = sp.adj_g[p];
      for (int h = threadIdx.x; h < sp.hs[p]; h += blockDim.x)
        dst[h] = h < sp.H[p] ? in[crow + combo_index(cards[2 * h], cards[2 * h + 1])] : 0.f;
    } else {
      const float* from = which == SC_ROOT ? sp.root_out[p] : sp.adj_dw[p];
      float* dst = out + crow;
      for (int c = threadIdx.x; c < kCombos; c += blockDim.x) dst[c] = 0.f;
      __syncthreads();
      if (from)
        for (int h = threadIdx.x; h < sp.H[p]; h += blockDim.x)
          dst[combo_index(cards[2 * h], cards[2 * h + 1])] = from[h];
      __syncthreads();
    }
  }
}

cudaError_t launch_spot_combo(const SpotDev* spots, int n, int which, const float* in, float* out,
                              cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_spot_combo<<<n, 256, 0, s>>>(spots, which, in, out);
  return cudaGetLastError();
}

// Input rows of the boundary network, one block per (item, player): the
// item's two reach rows are staged in shared memory and written out once per
// river card with the hands holding that card zeroed.  Pure store bandwidth:
// 2720 values per row, written as 16-byte (f32) or 8-byte (bf16) vectors.
template <bool BF16>
__global__ void k_boundary_encode(const uint8_t* __restrict__ boards, const float* __restrict__ pots,
                                  const float* __restrict__ stacks, const float* __restrict__ reach,
                                  void* __restrict__ out) {
  const int item = blockIdx.x >> 1, player = blockIdx.x & 1;
  __shared__ float s_r[2 * kCombos];
  __shared__ uint16_t s_pair[kCombos];  // c1 | c2 << 8
  __shared__ uint8_t s_river[kRivers];
  const uint8_t* bd = boards + 4 * item;
  const uint64_t bmask = (1ull << bd[0]) | (1ull << bd[1]) | (1ull << bd[2]) | (1ull << bd[3]);
  if (threadIdx.x == 0) {
    int k = 0;
    for (int c = 0; c < 52; ++c)
      if (!(bmask >> c & 1)) s_river[k++] = (uint8_t)c;
  }
  for (int c1 = threadIdx.x; c1 < 51; c1 += blockDim.x)
    for (int c2 = c1 + 1; c2 < 52; ++c2) s_pair[combo_index(c1, c2)] = (uint16_t)(c1 | c2 << 8);
  const float* r = reach + (size_t)item * 2 * kCombos;
  for (int c = threadIdx.x; c < 2 * kCombos; c += blockDim.x) s_r[c] = r[c];
  // boundary_evaluator.rs:35-36, :54-56 in f32
  const float pot = pots[item], stack = stacks[item];
  const float total = __fadd_rn(pot, stack);
  const float norm = total > 0.f ? total : 1.f;
  const float fpot = __fdiv_rn(pot, norm), fstack = __fdiv_rn(stack, norm), fpl = (float)player;
  const unsigned ranks4 = (1u << (bd[0] >> 2)) | (1u << (bd[1] >> 2)) | (1u << (bd[2] >> 2)) | (1u << (bd[3] >> 2));
  __syncthreads();
  constexpr int kVec = kBoundaryInput / 4;
  for (int ri = 0; ri < kRivers; ++ri) {
    const int river = s_river[ri];
    const uint64_t b5 = bmask | (1ull << river);
    const unsigned ranks = ranks4 | (1u << (river >> 2));
    const size_t row = ((size_t)blockIdx.x * kRivers + ri) * kBoundaryInput;
    for (int q = threadIdx.x; q < kVec; q += blockDim.x) {
      float v[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int f = 4 * q + e;
        float x;
        if (f < 2 * kCombos) {
          const int c = f < kCombos ? f : f - kCombos;
          const unsigned pr = s_pair[c];
          x = ((pr & 0xFF) == (unsigned)river || (pr >> 8) == (unsigned)river) ? 0.f : s_r[f];
        } else if (f < 2 * kCombos + 52) {
          x = (b5 >> (f - 2 * kCombos) & 1) ? 1.f : 0.f;
        } else if (f < 2 * kCombos + 65) {
          x = (ranks >> (f - 2 * kCombos - 52) & 1) ? 1.f : 0.f;
        } else {
          x = f == kBoundaryInput - 3 ? fpot : f == kBoundaryInput - 2 ? fstack : fpl;
        }
        v[e] = x;
      }
      if (BF16) {
        __nv_bfloat162 a = __floats2bfloat162_rn(v[0], v[1]), b = __floats2bfloat162_rn(v[2], v[3]);
        uint2 w;
        w.x = *reinterpret_cast<unsigned*>(&a);
        w.y = *reinterpret_cast<unsigned*>(&b);
        reinterpret_cast<uint2*>(static_cast<__nv_bfloat16*>(out) + row)[q] = w;
      } else {
        reinterpret_cast<float4*>(static_cast<float*>(out) + row)[q] = make_float4(v[0], v[1], v[2], v[3]);
      }
    }
  }
}

cudaError_t launch_boundary_encode(int n, const uint8_t* boards, const float* pots, const float* stacks,
                                   const float* reach, void* out, int bf16, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  if (bf16)
    k_boundary_encode<true><<<2 * n, 256, 0, s>>>(boards, pots, stacks, reach, out);
  else
    k_boundary_encode<false><<<2 * n, 256, 0, s>>>(boards, pots, stacks, reach, out);
  return cudaGetLastError();
}

// Training records (cfvnet datagen/storage.rs:5-57), one block per (spot,
// player), packed byte by byte (the format is unaligned):
//   [board_size u8][board][pot f32][stack f32][player u8][game_value f32]
//   [oop_range f32 x1326][ip_range f32 x1326][cfvs f32 x1326][valid_mask u8 x1326]
// with the values of the GPU river datagen (datagen/domain/pipeline.rs:353-411):
// cfvs[c] = (f64(f32(rootcfv[h] * num_combinations)) - pot/2) / (pot/2) for the
// hands of the player's list, 0 elsewhere; valid_mask marks the hands of
// either player's list (one mask for both records);
// game_value = sum over combos of range * cfv, in f32, in combo order.
__device__ __forceinline__ void put_bytes(uint8_t* dst, const void* src, int n) {
  const uint8_t* s = static_cast<const uint8_t*>(src);
  for (int i = 0; i < n; ++i) dst[i] = s[i];
}

__global__ void k_pack_records(const SpotDev* __restrict__ spots, const float* __restrict__ ranges,
                               const RecordMeta* __restrict__ meta, uint8_t* __restrict__ out) {
  const int spot = blockIdx.x >> 1, player = blockIdx.x & 1;
  const SpotDev& sp = spots[spot];
  const RecordMeta m = meta[spot];
  const int bs = m.board_size;
  const size_t rsize = 1 + bs + 4 + 4 + 1 + 4 + 3 * 4 * kCombos + kCombos;
  uint8_t* rec = out + (size_t)blockIdx.x * rsize;
  __shared__ float s_cfv[kCombos];
  __shared__ uint8_t s_valid[kCombos];
  for (int c = threadIdx.x; c < kCombos; c += blockDim.x) {
    s_cfv[c] = 0.f;
    s_valid[c] = 0;
  }
  __syncthreads();
  const double half = 0.5 * (double)m.pot;
  const double norm = half > 0.0 ? half : 1.0;
  const float comb = (float)sp.num_combinations;
  const uint8_t* cards = sp.cards[player];
  for (int h = threadIdx.x; h < sp.H[player]; h += blockDim.x) {
    const int c = combo_index(cards[2 * h], cards[2 * h + 1]);
    const float ev = __fmul_rn(sp.root_out[player][h], comb);
    s_cfv[c] = (float)(((double)ev - half) / norm);
  }
  // one mask for both records: the hands of either player (pipeline.rs:366-377)
  for (int q = 0; q < 2; ++q)
    for (int h = threadIdx.x; h < sp.H[q]; h += blockDim.x)
      s_valid[combo_index(sp.cards[q][2 * h], sp.cards[q][2 * h + 1])] = 1;
  __syncthreads();
  const float* rg = ranges + (size_t)spot * 2 * kCombos;
  uint8_t* body = rec + 1 + bs + 13;
  for (int i = threadIdx.x; i < 3 * kCombos; i += blockDim.x) {
    const float v = i < 2 * kCombos ? rg[i] : s_cfv[i - 2 * kCombos];
    put_bytes(body + 4 * i, &v, 4);
  }
  for (int c = threadIdx.x; c < kCombos; c += blockDim.x) body[12 * kCombos + c] = s_valid[c];
  if (threadIdx.x == 0) {
    const float* own = rg + (size_t)player * kCombos;
    float gv = 0.f;
    for (int c = 0; c < kCombos; ++c) gv = __fadd_rn(gv, __fmul_rn(own[c], s_cfv[c]));
    rec[0] = (uint8_t)bs;
    for (int k = 0; k < bs; ++k) rec[1 + k] = m.board[k];
    put_bytes(rec + 1 + bs, &m.pot, 4);
    put_bytes(rec + 5 + bs, &m.stack, 4);
    rec[9 + bs] = (uint8_t)player;
    put_bytes(rec + 10 + bs, &gv, 4);
  }
}

cudaError_t launch_pack_records(const SpotDev* spots, int n, const float* ranges, const RecordMeta* meta,
                                uint8_t* out, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_pack_records<<<2 * n, 256, 0, s>>>(spots, ranges, meta, out);
  return cudaGetLastError();
}

cudaError_t launch_boundary_river_reduce(int n, const uint8_t* boards, const float* denorm, const void* net,
                                         int net_bf16, const float* reach, const int32_t* hands, int H, float* out,
                                         cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  if (net_bf16)
    k_boundary_river_reduce<__nv_bfloat16><<<2 * n, 256, 0, s>>>(
        n, boards, denorm, static_cast<const __nv_bfloat16*>(net), reach, hands, H, out);
  else
    k_boundary_river_reduce<float><<<2 * n, 256, 0, s>>>(n, boards, denorm, static_cast<const float*>(net), reach,
                                                         hands, H, out);
  return cudaGetLastError();
}

// First layer of a boundary network (a Linear over the 2720 input values)
// for every input row of boundary_encode, without writing the rows: for item
// i, player p and river card r,
//   W x = W_reach [oop|ip] - sum over combos holding r of W_reach[., c] reach[c]
//         + board / rank one-hot columns + pot, stack, player columns (+ bias)
// base[i] = W_reach [oop|ip] and percard[i][k] (the sum over the combos
// holding card k) come from the caller's GEMMs.  One block per item: the
// river-independent part of the row goes to shared memory, then every
// (river, column) element is independent and coalesced along the columns;
// both players' rows come from one read of percard (they differ by the player
// column).  out [n][2][48][h].
template <bool BF16>
__global__ void k_boundary_first_layer(const uint8_t* __restrict__ boards, const float* __restrict__ pots,
                                       const float* __restrict__ stacks, const float* __restrict__ base,
                                       const float* __restrict__ percard, const float* __restrict__ wcols,
                                       const float* __restrict__ bias, int h, void* __restrict__ out) {
  extern __shared__ float s_c[];  // [h]
  __shared__ uint8_t s_river[kRivers];
  const int item = blockIdx.x;
  const uint8_t* bd = boards + 4 * item;
  const uint64_t bmask = (1ull << bd[0]) | (1ull << bd[1]) | (1ull << bd[2]) | (1ull << bd[3]);
  const unsigned ranks4 = (1u << (bd[0] >> 2)) | (1u << (bd[1] >> 2)) | (1u << (bd[2] >> 2)) | (1u << (bd[3] >> 2));
  if (threadIdx.x == 0) {
    int k = 0;
    for (int c = 0; c < 52; ++c)
      if (!(bmask >> c & 1)) s_river[k++] = (uint8_t)c;
  }
  const float pot = pots[item], stack = stacks[item];
  const float total = __fadd_rn(pot, stack);
  const float norm = total > 0.f ? total : 1.f;
  const float fpot = __fdiv_rn(pot, norm), fstack = __fdiv_rn(stack, norm);
  const float* wpot = wcols + (size_t)(52 + 13) * h;
  const float* wstack = wpot + h;
  const float* wplayer = wstack + h;
  for (int j = threadIdx.x; j < h; j += blockDim.x) {
    float c = base[(size_t)item * h + j];
    for (int k = 0; k < 4; ++k) c += wcols[(size_t)bd[k] * h + j];
    for (int q = 0; q < 13; ++q)
      if (ranks4 >> q & 1) c += wcols[(size_t)(52 + q) * h + j];
    s_c[j] = c + fpot * wpot[j] + fstack * wstack[j] + (bias ? bias[j] : 0.f);
  }
  __syncthreads();
  const float* pc = percard + (size_t)item * 52 * h;
  const size_t o0 = (size_t)item * 2 * kRivers * h, o1 = o0 + (size_t)kRivers * h;
  for (int e = threadIdx.x; e < kRivers * h; e += blockDim.x) {
    const int ri = e / h, j = e - ri * h;
    const int r = s_river[ri];
    float v = s_c[j] - pc[(size_t)r * h + j] + wcols[(size_t)r * h + j];
    if (!(ranks4 >> (r >> 2) & 1)) v += wcols[(size_t)(52 + (r >> 2)) * h + j];
    const float v1 = v + wplayer[j];
    if (BF16) {
      static_cast<__nv_bfloat16*>(out)[o0 + e] = __float2bfloat16_rn(v);
      static_cast<__nv_bfloat16*>(out)[o1 + e] = __float2bfloat16_rn(v1);
    } else {
      static_cast<float*>(out)[o0 + e] = v;
      static_cast<float*>(out)[o1 + e] = v1;
    }
  }
}

cudaError_t launch_boundary_first_layer(int n, const uint8_t* boards, const float* pots, const float* stacks,
                                        const float* base, const float* percard, const float* wcols,
                                        const float* bias, int h, void* out, int bf16, cudaStream_t s) {
  if (n <= 0 || h <= 0) return cudaSuccess;
  if (h > kMaxFirstLayerWidth) return cudaErrorInvalidValue;
  const size_t smem = sizeof(float) * (size_t)h;
  if (bf16)
    k_boundary_first_layer<true><<<n, 256, smem, s>>>(boards, pots, stacks, base, percard, wcols, bias, h, out);
  else
    k_boundary_first_layer<false><<<n, 256, smem, s>>>(boards, pots, stacks, base, percard, wcols, bias, h, out);
  return cudaGetLastError();
}

}  // namespace ps
