// ORACLE — test infrastructure only. A CPU restatement of the reference's
// `crates/range-solver` (tjennings/poker_solver_rust), used as the checker for
// the CUDA path and as the timed CPU baseline.  Nothing in the product links,
// imports or executes this code.
//
// Parity pins: the hand table and its category counts are checked against the
// reference's HAND_TABLE (crates/range-solver/src/hand_table.rs, by digest) and
// its exhaustive test (hand.rs:407-449); discount parameters against
// solver.rs:688-722; action lists against examples/basic.rs:101-116.  No golden
// strategy / CFV values exist in the reference and the Rust reference cannot
// be built here, so the solve's floating-point results are parity unpinned:
// they rest on this line-by-line restatement of the cited code.
//
// The scalar type F is float for the parity build (same rounding sequence as
// the reference's f32 vectors with f64 accumulators) and double for the FP64
// error-reference build.
#pragma once
#include <array>
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace oracle {

using Card = uint8_t;
constexpr Card NOT_DEALT = 255;

// card.rs:50-55
inline int card_pair_to_index(int c1, int c2) {
  if (c1 > c2) { int t = c1; c1 = c2; c2 = t; }
  return c1 * (101 - c1) / 2 + c2 - 1;
}
// card.rs:61-65
std::pair<int, int> index_to_card_pair(int index);

// hand.rs:68-146 and hand_table.rs
int32_t hand_evaluate_internal(const int cards[7]);
const std::vector<int32_t>& hand_table();
void set_hand_table_path(const char* path);
// threads for the chance children of solve passes (1 = sequential)
void set_chance_threads(int n);
uint16_t hand_evaluate(const int cards[7]);
// Exhaustive enumeration over all C(52,7) hands (hand.rs:407-449): fills
// the sorted distinct value table and the 9 category counts.
void hand_table_exhaustive(std::vector<int32_t>& table, uint64_t counts[9]);

// bet_size.rs:55-80
enum BetKind { PotRelative = 0, PrevBetRelative = 1, Additive = 2, Geometric = 3, AllIn = 4 };
struct BetSize {
  BetKind kind;
  double f;  // ratio (PotRelative, PrevBetRelative), max ratio (Geometric)
  int i;     // adder (Additive), num_streets (Geometric)
  int cap;   // raise cap (Additive)
};
struct BetSizeOptions {
  std::vector<BetSize> bet, raise;
};
bool parse_bet_size_options(const std::string& bet, const std::string& raise, BetSizeOptions& out,
                            std::string& err);
bool parse_donk_size_options(const std::string& donk, std::vector<BetSize>& out, std::string& err);

// action_tree.rs:11-18
constexpr uint8_t PLAYER_OOP = 0, PLAYER_IP = 1, PLAYER_CHANCE = 2, PLAYER_MASK = 3,
                  PLAYER_CHANCE_FLAG = 4, PLAYER_TERMINAL_FLAG = 8, PLAYER_FOLD_FLAG = 24,
                  PLAYER_DEPTH_BOUNDARY_FLAG = 40;

// action_tree.rs:26-51 (derived Ord: variant, then payload)
enum ActionKind { A_None = 0, A_Fold, A_Check, A_Call, A_Bet, A_Raise, A_AllIn, A_Chance };
struct Action {
  ActionKind kind = A_None;
  int32_t amount = 0;  // card for A_Chance
  bool operator<(const Action& o) const {
    return kind != o.kind ? kind < o.kind : amount < o.amount;
  }
  bool operator==(const Action& o) const { return kind == o.kind && amount == o.amount; }
};

enum BoardState { Flop = 0, Turn = 1, River = 2 };

// action_tree.rs:130-192
struct TreeConfig {
  BoardState initial_state = Flop;
  int32_t starting_pot = 0, effective_stack = 0;
  double rake_rate = 0, rake_cap = 0;
  BetSizeOptions flop_bet_sizes[2], turn_bet_sizes[2], river_bet_sizes[2];
  bool has_turn_donk = false, has_river_donk = false;
  std::vector<BetSize> turn_donk_sizes, river_donk_sizes;
  double add_allin_threshold = 0, force_allin_threshold = 0, merging_threshold = 0;
  int depth_limit = -1;  // -1 = None
};

struct ActionTreeNode {
  uint8_t player = 0;
  BoardState board_state = Flop;
  int32_t amount = 0;
  std::vector<Action> actions;
  std::vector<std::unique_ptr<ActionTreeNode>> children;
  bool is_terminal() const { return (player & PLAYER_TERMINAL_FLAG) != 0; }
  bool is_chance() const { return (player & PLAYER_CHANCE_FLAG) != 0; }
};

struct ActionTree {
  TreeConfig config;
  std::unique_ptr<ActionTreeNode> root;
  static bool create(const TreeConfig& cfg, ActionTree& out, std::string& err);
  std::vector<std::vector<Action>> invalid_terminals() const;
};

// range.rs:215-275 over raw 1326-weight data
struct Range {
  float data[1326] = {0};
  void get_hands_weights(uint64_t dead_mask, std::vector<std::pair<Card, Card>>& hands,
                         std::vector<float>& weights) const;
  bool is_suit_isomorphic(int s1, int s2) const;
  bool is_empty() const;
  bool is_valid() const;
};

struct CardConfig {
  Range range[2];
  Card flop[3] = {NOT_DEALT, NOT_DEALT, NOT_DEALT};
  Card turn = NOT_DEALT, river = NOT_DEALT;
};

// game/mod.rs:90-93
struct StrengthItem {
  uint16_t strength, index;
  bool operator<(const StrengthItem& o) const {
    return strength != o.strength ? strength < o.strength : index < o.index;
  }
};

using SwapList = std::array<std::vector<std::pair<uint16_t, uint16_t>>, 2>;
using Indices = std::array<std::vector<uint16_t>, 2>;

enum class State { ConfigError = 0, Uninitialized = 1, TreeBuilt = 2, MemoryAllocated = 3, Solved = 4 };

// game/mod.rs:135-152 (storage pointers as offsets)
struct Node {
  Action prev_action;
  uint8_t player = PLAYER_OOP;
  Card turn = NOT_DEALT, river = NOT_DEALT;
  bool is_locked = false;
  int32_t amount = 0;
  uint32_t children_offset = 0;
  uint16_t num_children = 0;
  uint16_t num_elements_ip = 0;
  uint32_t num_elements = 0;
  size_t s1 = 0, s2 = 0, s3 = 0;
  bool is_terminal() const { return (player & PLAYER_TERMINAL_FLAG) != 0; }
  bool is_chance() const { return (player & PLAYER_CHANCE_FLAG) != 0; }
  bool is_depth_boundary() const {
    return (player & PLAYER_DEPTH_BOUNDARY_FLAG) == PLAYER_DEPTH_BOUNDARY_FLAG;
  }
  int cfvalue_storage_player() const {  // node.rs (GameNode impl)
    int prev = player & PLAYER_MASK;
    return prev == 0 ? 1 : prev == 1 ? 0 : -1;
  }
};

struct DiscountParams {  // solver.rs:20-44
  float alpha_t, beta_t, gamma_t;
  explicit DiscountParams(uint32_t t);
};

template <class F>
struct Game {
  State state = State::Uninitialized;
  CardConfig card_config;
  TreeConfig tree_config;
  std::unique_ptr<ActionTreeNode> action_root;

  double num_combinations = 0;
  std::vector<F> initial_weights[2];
  std::vector<std::pair<Card, Card>> private_cards[2];
  std::vector<uint16_t> same_hand_index[2];
  Indices valid_indices_flop;
  std::vector<Indices> valid_indices_turn, valid_indices_river;
  std::vector<std::array<std::vector<StrengthItem>, 2>> hand_strength;

  std::vector<uint8_t> isomorphism_ref_turn;
  std::vector<Card> isomorphism_card_turn;
  std::array<SwapList, 4> isomorphism_swap_turn;
  std::vector<std::vector<uint8_t>> isomorphism_ref_river;
  std::array<std::vector<Card>, 4> isomorphism_card_river;
  std::array<std::array<SwapList, 4>, 4> isomorphism_swap_river;

  uint64_t num_nodes_street[3] = {0, 0, 0};
  uint64_t num_storage = 0, num_storage_ip = 0, num_storage_chance = 0;
  std::vector<Node> arena;
  std::vector<F> storage1, storage2, storage_ip, storage_chance;
  std::map<size_t, std::vector<F>> locking_strategy;

  // depth boundary (single continuation)
  std::vector<uint32_t> node_to_boundary;
  std::vector<std::vector<F>> boundary_cfvs;   // [ordinal*2 + player]
  std::vector<std::vector<F>> boundary_reach;  // [ordinal*2 + player]

  // interpreter state (query.rs)
  std::vector<size_t> action_history, node_history;
  bool is_normalized_weight_cached = false;
  Card turn = NOT_DEALT, river = NOT_DEALT;
  int turn_swapped_suit[2] = {-1, -1};
  int turn_swap = -1;
  int river_swap[2] = {-1, -1};
  int32_t total_bet_amount[2] = {0, 0};
  std::vector<F> weights[2], normalized_weights[2], cfvalues_cache[2];

  // -------- construction (interpreter.rs) --------
  bool with_config(const CardConfig& cc, ActionTree&& tree, std::string& err);
  void allocate_memory();
  size_t num_private_hands(int p) const { return private_cards[p].size(); }
  size_t node_index(const Node* n) const { return (size_t)(n - arena.data()); }
  Node* child(Node* n, int a) { return n + n->children_offset + a; }
  int chance_factor(const Node& n) const { return n.turn == NOT_DEALT ? 45 : 44; }
  bool is_ready() const { return state == State::MemoryAllocated; }
  bool is_solved() const { return state == State::Solved; }
  bool is_raked() const { return tree_config.rake_rate > 0.0 && tree_config.rake_cap > 0.0; }
  size_t num_boundary_nodes() const { return boundary_cfvs.size() / 2; }
  const std::vector<uint8_t>& isomorphic_chances(const Node& n) const;
  const SwapList& isomorphic_swap(const Node& n, size_t i) const;
  const std::vector<F>* locking(const Node& n) const;

  // -------- evaluation (evaluation.rs) --------
  void evaluate(F* result, const Node& node, int player, const F* cfreach);

  // -------- solver (solver.rs, utility.rs) --------
  void solve_recursive(F* result, Node* node, int player, const F* cfreach, const DiscountParams& p);
  void solve_step(uint32_t t);
  void solve_pass(uint32_t t, int player);  // one traverser pass of solve_step
  float solve(uint32_t max_iter, float target, bool print, uint32_t* iters_run = nullptr);
  void compute_cfvalue_recursive(F* result, Node* node, int player, const F* cfreach, bool save);
  void compute_best_cfv_recursive(F* result, Node* node, int player, const F* cfreach);
  std::array<float, 2> compute_mes_ev();
  std::array<float, 2> compute_current_ev();
  float compute_exploitability();
  void finalize();
  std::vector<F> root_cfvalues_with_reach(int player, const F* opp_reach);

  // -------- queries (query.rs) --------
  Node* cur_node() { return &arena[node_history.empty() ? 0 : node_history.back()]; }
  void back_to_root();
  bool is_terminal_node();
  bool is_chance_node();
  std::vector<Action> available_actions();
  uint64_t possible_cards();
  int current_player() { return cur_node()->player; }
  void play(size_t action);
  std::vector<F> strategy();
  std::vector<F> strategy_at_index(size_t idx);
  void cache_normalized_weights();
  std::vector<F> expected_values_detail(int player);
  std::vector<F> expected_values(int player);
  void apply_swap(F* slice, int player, bool reverse);
  void assign_zero_weights();
  void lock_current_strategy(const F* strategy);

 private:
  bool check_card_config(std::string& err);
  void init_card_fields();
  void compute_isomorphism();
  bool init_root(std::string& err);
  void count_num_nodes(uint64_t out[3]);
  void build_tree_recursive(size_t node_index, const ActionTreeNode& an, uint64_t info[3]);
  void push_chances(size_t node_index, uint64_t info[3]);
  void push_actions(size_t node_index, const ActionTreeNode& an, uint64_t info[3]);
  void allocate_memory_nodes();
  void evaluate_boundary_single(F* result, const Node& node, int player, const F* cfreach,
                                const std::vector<F>& bcfvs, double half_pot);
  const Indices& valid_indices_for(const Node& node) const;
};

}  // namespace oracle
