// 7-card hand evaluation shared by host and device code.
//
// The rank value follows the reference's `Hand::evaluate_internal`
// (crates/range-solver/src/hand.rs:77-146): category in bits 26+, then the
// deciding rank sets; the strength index is the position of that value in the
// sorted table of all distinct values (hand.rs:68-75, hand_table.rs).
//
// The table itself is built here without enumerating all C(52,7) hands: a
// hand's value depends only on its rank multiset and on the rank set of a
// flush suit when one exists, so the table is the union of
//   (a) the non-flush value of every 7-card rank multiset with counts <= 4
//       (each such multiset can be dealt with no five cards of one suit), and
//   (b) the flush value of every rank set of 5..7 distinct ranks (with at most
//       two other cards, a flush hand can never also hold quads or a full
//       house, so the flush branch always decides).
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define PS_HD __host__ __device__ __forceinline__
#else
#define PS_HD inline
#endif

namespace ps {

constexpr int kHandTableSize = 4824;

PS_HD int ps_popc(uint32_t x) {
#ifdef __CUDA_ARCH__
  return __popc(x);
#else
  return __builtin_popcount(x);
#endif
}

PS_HD int ps_msb(uint32_t x) {  // index of the highest set bit, x != 0
#ifdef __CUDA_ARCH__
  return 31 - __clz(x);
#else
  return 31 - __builtin_clz(x);
#endif
}

PS_HD uint32_t top_bits(uint32_t x, int n) {  // keep the n highest set bits
  uint32_t r = 0;
  for (int i = 0; i < n; ++i) {
    uint32_t b = 1u << ps_msb(x);
    x ^= b;
    r |= b;
  }
  return r;
}

PS_HD uint32_t straight_top(uint32_t rs) {  // highest straight in a rank set
  uint32_t s = rs & (rs << 1) & (rs << 2) & (rs << 3) & (rs << 4);
  if (s) return 1u << ps_msb(s);
  return (rs & 0x100Fu) == 0x100Fu ? (1u << 3) : 0u;
}

// Non-flush value from per-rank counts (the branches after the flush test).
PS_HD int32_t value_from_counts(const int cnt[13]) {
  uint32_t rankset = 0, by_count[5] = {0, 0, 0, 0, 0};
  for (int r = 0; r < 13; ++r) {
    if (cnt[r]) rankset |= 1u << r;
    by_count[cnt[r]] |= 1u << r;
  }
  if (by_count[4]) return (int32_t)((7u << 26) | (by_count[4] << 13) | top_bits(rankset ^ by_count[4], 1));
  if (ps_popc(by_count[3]) == 2) {
    uint32_t t = top_bits(by_count[3], 1);
    return (int32_t)((6u << 26) | (t << 13) | (by_count[3] ^ t));
  }
  if (by_count[3] && by_count[2])
    return (int32_t)((6u << 26) | (by_count[3] << 13) | top_bits(by_count[2], 1));
  uint32_t st = straight_top(rankset);
  if (st) return (int32_t)((4u << 26) | st);
  if (by_count[3]) return (int32_t)((3u << 26) | (by_count[3] << 13) | top_bits(by_count[1], 2));
  if (ps_popc(by_count[2]) >= 2) {
    uint32_t p = top_bits(by_count[2], 2);
    return (int32_t)((2u << 26) | (p << 13) | top_bits(rankset ^ p, 1));
  }
  if (by_count[2]) return (int32_t)((1u << 26) | (by_count[2] << 13) | top_bits(by_count[1], 3));
  return (int32_t)top_bits(rankset, 5);
}

// Flush value of a suit rank set with >= 5 ranks.
PS_HD int32_t value_of_flush(uint32_t suit_ranks) {
  uint32_t sf = straight_top(suit_ranks);
  if (sf) return (int32_t)((8u << 26) | sf);
  return (int32_t)((5u << 26) | top_bits(suit_ranks, 5));
}

// Value of 7 cards (card = 4 * rank + suit).
PS_HD int32_t hand_value7(const int c[7]) {
  int cnt[13] = {0};
  uint32_t suit_ranks[4] = {0, 0, 0, 0};
  for (int k = 0; k < 7; ++k) {
    cnt[c[k] >> 2] += 1;
    suit_ranks[c[k] & 3] |= 1u << (c[k] >> 2);
  }
  // The last suit with five or more cards decides (only one can have five of seven).
  for (int s = 3; s >= 0; --s)
    if (ps_popc(suit_ranks[s]) >= 5) return value_of_flush(suit_ranks[s]);
  return value_from_counts(cnt);
}

// Position of `v` in the sorted table (binary search; table in any memory space).
PS_HD int table_index(const int32_t* table, int n, int32_t v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (table[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Builds the sorted distinct-value table on the host.  Returns its length.
int build_hand_table(int32_t* out, int cap);

}  // namespace ps
