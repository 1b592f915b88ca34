// Host side of the B200 range solver: bet-size menus, the abstract action
// tree, the game arena (same node order as the reference's PostFlopGame, so
// node indices returned by queries match), per-hand setup and the compiler
// that turns a game into the level-ordered GPU tree program.
#pragma once
#include <array>
#include <cstdint>
#include <string>
#include <vector>

#include "ps_device.hpp"

namespace ps {

constexpr uint8_t NOT_DEALT = 255;
constexpr uint8_t PL_OOP = 0, PL_IP = 1, PL_CHANCE = 2, PL_MASK = 3, PL_CHANCE_FLAG = 4,
                  PL_TERMINAL_FLAG = 8, PL_FOLD_FLAG = 24, PL_BOUNDARY_FLAG = 40;

inline int pair_index(int c1, int c2) {  // crates/range-solver/src/card.rs:50-55
  if (c1 > c2) { int t = c1; c1 = c2; c2 = t; }
  return c1 * (101 - c1) / 2 + c2 - 1;
}

// ---- bet sizes (crates/range-solver/src/bet_size.rs) ----
struct BetSize {
  enum Kind { Pot = 0, PrevBet = 1, Add = 2, Geo = 3, AllIn = 4 } kind;
  double ratio;  // Pot / PrevBet ratio, Geo max ratio
  int n;         // Add amount, Geo streets
  int cap;       // Add raise cap
};
struct BetMenu {
  std::vector<BetSize> bet, raise;
};
bool parse_menu(const std::string& s, bool raise, std::vector<BetSize>& out, std::string& err);

// ---- action tree (crates/range-solver/src/action_tree.rs) ----
enum ActKind : int32_t { ACT_NONE = 0, ACT_FOLD, ACT_CHECK, ACT_CALL, ACT_BET, ACT_RAISE, ACT_ALLIN, ACT_CHANCE };
struct Act {
  int32_t kind = ACT_NONE, amount = 0;
  bool operator<(const Act& o) const { return kind != o.kind ? kind < o.kind : amount < o.amount; }
  bool operator==(const Act& o) const { return kind == o.kind && amount == o.amount; }
};

struct TreeCfg {
  int initial_state = 2;  // 0 flop, 1 turn, 2 river
  int32_t starting_pot = 0, effective_stack = 0;
  double rake_rate = 0, rake_cap = 0;
  BetMenu menu[3][2];
  bool has_donk[2] = {false, false};  // turn, river
  std::vector<BetSize> donk[2];
  double add_allin_threshold = 0, force_allin_threshold = 0, merging_threshold = 0;
  int depth_limit = -1;
  int max_bets = 0;  // extension: >0 caps bets+raises per street (0 = no cap, the reference)
};

// Flat abstract tree: children of node i are kids[first .. first+n).
struct ATree {
  struct N {
    uint8_t player;
    uint8_t street;
    int32_t amount;
    int32_t first, n;
    Act act;  // action leading to this node
  };
  std::vector<N> nodes;
  TreeCfg cfg;
  static bool build(const TreeCfg& cfg, ATree& out, std::string& err);
  bool has_invalid_terminal() const;
};

// ---- the game ----
struct ArenaNode {
  Act prev;
  uint8_t player = PL_OOP;
  uint8_t turn = NOT_DEALT, river = NOT_DEALT;
  int32_t amount = 0;
  uint32_t child_off = 0;
  uint16_t nch = 0;
  uint32_t rs_off = 0xFFFFFFFFu, ip_off = 0xFFFFFFFFu, ch_off = 0xFFFFFFFFu;
  bool terminal() const { return (player & PL_TERMINAL_FLAG) != 0; }
  bool chance() const { return (player & PL_CHANCE_FLAG) != 0; }
  bool boundary() const { return (player & PL_BOUNDARY_FLAG) == PL_BOUNDARY_FLAG; }
  bool fold() const { return (player & PL_FOLD_FLAG) == PL_FOLD_FLAG; }
};

struct Program {
  std::vector<Op> ops;
  std::vector<Step> steps;
  std::vector<uint16_t> groups;
  int root_slot = -1;
  int num_slots = 0;
  bool verified = false;  // the slot replay of compile found every read intact
};

struct IsoEntry {
  int32_t child;  // index of the reference child within the chance node
  int32_t perm;   // swap permutation id
};

struct Game {
  // configuration
  TreeCfg cfg;
  float range[2][1326];
  uint8_t flop[3], turn, river;
  // hands (crates/range-solver/src/range.rs:256-275, interpreter.rs:645-662)
  std::vector<std::array<uint8_t, 2>> cards[2];
  std::vector<float> w[2];
  std::vector<uint16_t> same[2];
  double num_combinations = 0;
  int H[2] = {0, 0}, hs[2] = {0, 0}, vstride = 0;
  // arena
  std::vector<ArenaNode> arena;
  uint64_t num_storage = 0, num_storage_ip = 0, num_storage_chance = 0;
  std::vector<int32_t> bnd_ordinal;  // arena -> ordinal or -1
  int num_boundary = 0;
  // boards: id -> 5 board cards (255 = not dealt); board 0 is the root board
  std::vector<std::array<uint8_t, 5>> boards;
  std::vector<int32_t> node_board;  // arena -> board id
  // isomorphism (crates/range-solver/src/isomorphism.rs)
  std::vector<uint8_t> iso_ref_turn;
  std::vector<uint8_t> iso_card_turn;
  std::vector<std::vector<uint8_t>> iso_ref_river;  // [52]
  std::vector<uint8_t> iso_card_river[4];
  std::vector<std::array<uint8_t, 2>> iso_swaps;     // perm id -> (suit1, suit2)
  std::vector<std::vector<uint16_t>> iso_perm[2];    // perm id -> per-player permutation
  int iso_perm_turn[4] = {-1, -1, -1, -1};           // suit -> perm id
  int iso_perm_river[4][4];                          // [turn suit][suit] -> perm id
  std::vector<int32_t> iso_list_off;                 // per chance node -> begin in iso_list
  std::vector<IsoEntry> iso_list;
  std::vector<int32_t> chance_iso_id;                // arena -> iso list id (or -1)
  // programs per traverser
  Program prog[2];
  int num_slots = 0;

  bool terminals_first = false;  // the programs evaluate every terminal of a pass in one step
  int program_choice = -1;       // -1: terminals-first when the game runs in grid mode; 0 / 1: as chosen

  bool init(const float* r0, const float* r1, const uint8_t board[5], const TreeCfg& cfg,
            std::string& err);
  int chance_factor(const ArenaNode& n) const { return n.turn == NOT_DEALT ? 45 : 44; }
  // recompiles both traversers' programs (terminals_first: see compile)
  bool recompile(bool terminals_first, std::string& err);

 private:
  bool check_cards(std::string& err);
  void init_isomorphism();
  void build_arena(const ATree& t);
  void compile(int p, bool terminals_first = false);
};

// f64 discount schedule of DCFR (crates/range-solver/src/solver.rs:26-44)
Discount discount_params(uint32_t t);

}  // namespace ps
