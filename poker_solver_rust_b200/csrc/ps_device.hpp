// Plain-data structures shared by the host tree compiler and the CUDA
// kernels: the per-spot device descriptor and the level-ordered tree program.
#pragma once
#include <cstdint>

namespace ps {

// Opcodes of the tree program (one op = one node's work for one traverser pass).
enum OpType : uint8_t {
  OP_FWD_OPP = 1,    // opponent decision node: children's reach = reach * sigma_a
  OP_FWD_CHANCE = 2, // chance node: children's reach = reach / chance_factor
  OP_TERM = 3,       // terminal: fold / showdown / depth-boundary evaluation
  OP_BWD_TRAV = 4,   // traverser decision node: cfv = combine(children), regret/strategy update
  OP_BWD_OPP = 5,    // opponent decision node: cfv = sum of children
  OP_BWD_CHANCE = 6, // chance node: cfv = sum of children (+ isomorphic swaps)
};

enum TermKind : uint8_t { TERM_FOLD = 0, TERM_SHOWDOWN = 1, TERM_BOUNDARY = 2 };

constexpr uint16_t SLOT_ROOT_REACH = 0xFFFF;  // the opponent's initial weights
constexpr int kMaxActions = 16;
constexpr int kThrWords = 8;  // per-hand lookup record (u16 x 8 = 16 bytes)

// 16-byte op record.
struct Op {
  uint8_t type;
  uint8_t na;        // number of children (decision / chance nodes)
  uint8_t term;      // TermKind (OP_TERM)
  uint8_t fold_pl;   // folded player (TERM_FOLD)
  uint32_t node;     // arena index
  uint16_t src;      // reach slot read by this op
  uint16_t dst;      // cfv slot written by BWD / TERM ops
  uint16_t blk;      // children block: reach block (FWD) / cfv block (BWD)
  uint16_t board;    // board id (OP_TERM) / isomorphism list id (OP_BWD_CHANCE)
};
static_assert(sizeof(Op) == 16, "Op must stay 16 bytes");

// Program step: ops[begin, begin + n_elem) are node ops, the next n_term ops
// are terminals grouped in runs that read the same reach on the same board
// (group g starts at begin + n_elem + groups[gbegin + g]; the leader's `na`
// holds the run length).  All of a step's ops are independent.
struct Step {
  int32_t begin;
  int16_t n_elem, n_term, n_groups, pad;
  int32_t gbegin;
};

// Per-node tables indexed by arena index.
struct NodeDev {
  int32_t amount;        // chips each player has put in
  uint32_t rs_off;       // R/S element offset (decision nodes)
  uint32_t ip_off;       // IP cfvalue storage offset (or 0xFFFFFFFF)
  uint32_t ch_off;       // chance cfvalue storage offset (or 0xFFFFFFFF)
  int32_t chance_factor; // 45 (turn deal) / 44 (river deal) for chance nodes
  int32_t ch_player;     // player whose cfvalues a chance node stores (or -1)
  int32_t boundary;      // depth-boundary ordinal (or -1)
  float amount_win;      // terminal payoffs per unit of reach, rounded from f64
  float amount_lose;     //   (game/evaluation.rs:64-68, :430)
  float amount_tie;
  float payoff_scale;    // half_pot / num_combinations (depth boundary)
  float path_scale;      // product of 1 / chance_factor over the chance nodes above
};
static_assert(sizeof(NodeDev) == 48, "NodeDev layout");

// One game on the device.  All pointers are device pointers.
struct SpotDev {
  int32_t H[2];        // private hands per player
  int32_t hs[2];       // row stride of each player's vectors (H rounded up to 4)
  int32_t vstride;     // slot stride in floats
  int32_t num_slots;
  int32_t num_boards;
  int32_t starting_pot;
  int32_t nsteps[2];
  int32_t root_slot[2];
  int32_t raked;
  int32_t num_boundary;
  double num_combinations;
  double rake_rate, rake_cap;
  const uint8_t* cards[2];   // [H][2]
  const float* w[2];         // [hs] initial weights (zero padded)
  const uint16_t* same[2];   // [hs] same-hand index in the opponent list
  const Op* ops[2];
  const Step* steps[2];
  const uint16_t* groups[2];  // terminal-group leader offsets of every step
  const NodeDev* nodes;
  const uint8_t* board_cards; // [num_boards][5], 255 = none
  uint16_t* gidx[2];   // opponent o: [num_boards][3 * hs[o]] gather order (ord, then by card)
  uint16_t* coff[2];   // opponent o: [num_boards][56] card segment starts within the card part
  uint16_t* thr[2];    // player p: [num_boards][hs[p]] 16-byte lookup records vs the opponent
  uint32_t* heads[2];  // opponent o: [num_boards][(3 * hs[o] + 31) / 32] segment-start bits of the gather list
  int32_t* nvalid[2];  // player: [num_boards] valid hand count
  const float* bcfv;   // boundary cfvs [num_boundary][2][vstride] (pot-normalised)
  const uint16_t* iso_perm[2]; // player: [perm id][hs] index of the suit-swapped hand
  const int32_t* iso_off;      // iso list id -> [begin, end) in iso_ent
  const int32_t* iso_ent;      // pairs (reference child index, perm id)
  float* R;            // regrets / saved cfvalues
  float* S;            // cumulative strategy
  float* SG;           // strategy cache of the DCFR passes, laid out like R, or null
  float* ipcfv;        // IP cfvalues at root / chance children (finalize)
  float* chcfv;        // chance-node cfvalues (finalize)
  float* slots;        // [num_slots][vstride] scratch vectors
  float* root_out[2];  // [hs] root cfv per player (exploitability / root_cfvalues)
  float* breach;       // [num_boundary][2][vstride] each player's reach at each boundary under the
                       // average strategy (written by the batched solve's epilogue), or null
  // batched adjoint of the fixed-strategy evaluation (null until first used):
  float* adj_g[2];     // [hs] cotangent of player p's root cfvalues
  float* adj_dw[2];    // [hs] gradient with respect to player p's initial weights
  float* bgrad;        // [num_boundary][2][vstride] gradient with respect to the boundary values, or null
};

// One DCFR iteration's discount factors (computed on the host in f64, solver.rs:26-44).
struct Discount {
  float alpha, beta, gamma, pad;
};

}  // namespace ps
