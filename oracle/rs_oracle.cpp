// ORACLE — test infrastructure only (see rs_oracle.hpp).  CPU restatement of
// crates/range-solver.  Every function cites the reference file:line it
// follows; paths are relative to crates/range-solver/src/.
#include "rs_oracle.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <condition_variable>
#include <cstring>
#include <atomic>
#include <functional>
#include <mutex>
#include <stdexcept>
#include <thread>

namespace oracle {

// ---------------------------------------------------------------------------
// card.rs
// ---------------------------------------------------------------------------

// card.rs:61-65
std::pair<int, int> index_to_card_pair(int index) {
  int c1 = (103 - (int)std::ceil(std::sqrt(103.0 * 103.0 - 8.0 * (double)index))) / 2;
  int c2 = index - c1 * (101 - c1) / 2 + 1;
  return {c1, c2};
}

// ---------------------------------------------------------------------------
// hand.rs
// ---------------------------------------------------------------------------

static inline int32_t keep_n_msb(int32_t x, int n) {  // hand.rs:18-27
  int32_t ret = 0;
  for (int i = 0; i < n; ++i) {
    int32_t bit = (int32_t)(1u << (31 - __builtin_clz((uint32_t)x)));
    x ^= bit;
    ret |= bit;
  }
  return ret;
}

static inline int32_t find_straight(int32_t rs) {  // hand.rs:31-42
  const int32_t WHEEL = 0x100F;
  int32_t s = rs & (rs << 1) & (rs << 2) & (rs << 3) & (rs << 4);
  if (s != 0) return keep_n_msb(s, 1);
  if ((rs & WHEEL) == WHEEL) return 1 << 3;
  return 0;
}

// hand.rs:77-146
int32_t hand_evaluate_internal(const int cards[7]) {
  int32_t rankset = 0, rankset_suit[4] = {0, 0, 0, 0}, rankset_of_count[5] = {0, 0, 0, 0, 0};
  int rank_count[13] = {0};
  for (int k = 0; k < 7; ++k) {
    int rank = cards[k] / 4, suit = cards[k] % 4;
    rankset |= 1 << rank;
    rankset_suit[suit] |= 1 << rank;
    rank_count[rank] += 1;
  }
  for (int r = 0; r < 13; ++r) rankset_of_count[rank_count[r]] |= 1 << r;
  int flush_suit = -1;
  for (int s = 0; s < 4; ++s)
    if (__builtin_popcount((uint32_t)rankset_suit[s]) >= 5) flush_suit = s;
  int32_t is_straight = find_straight(rankset);
  if (flush_suit >= 0) {
    int32_t sf = find_straight(rankset_suit[flush_suit]);
    if (sf != 0) return (8 << 26) | sf;
    return (5 << 26) | keep_n_msb(rankset_suit[flush_suit], 5);
  } else if (rankset_of_count[4] != 0) {
    int32_t remaining = keep_n_msb(rankset ^ rankset_of_count[4], 1);
    return (7 << 26) | (rankset_of_count[4] << 13) | remaining;
  } else if (__builtin_popcount((uint32_t)rankset_of_count[3]) == 2) {
    int32_t trips = keep_n_msb(rankset_of_count[3], 1);
    int32_t pair = rankset_of_count[3] ^ trips;
    return (6 << 26) | (trips << 13) | pair;
  } else if (rankset_of_count[3] != 0 && rankset_of_count[2] != 0) {
    int32_t pair = keep_n_msb(rankset_of_count[2], 1);
    return (6 << 26) | (rankset_of_count[3] << 13) | pair;
  } else if (is_straight != 0) {
    return (4 << 26) | is_straight;
  } else if (rankset_of_count[3] != 0) {
    int32_t remaining = keep_n_msb(rankset_of_count[1], 2);
    return (3 << 26) | (rankset_of_count[3] << 13) | remaining;
  } else if (__builtin_popcount((uint32_t)rankset_of_count[2]) >= 2) {
    int32_t pairs = keep_n_msb(rankset_of_count[2], 2);
    int32_t remaining = keep_n_msb(rankset ^ pairs, 1);
    return (2 << 26) | (pairs << 13) | remaining;
  } else if (rankset_of_count[2] != 0) {
    int32_t remaining = keep_n_msb(rankset_of_count[1], 3);
    return (1 << 26) | (rankset_of_count[2] << 13) | remaining;
  }
  return keep_n_msb(rankset, 5);
}

// The reference's test_all_hands_exhaustive (hand.rs:407-449): every 7-card
// set evaluated, the set of distinct values is the table, counts by category.
void hand_table_exhaustive(std::vector<int32_t>& table, uint64_t counts[9]) {
  const int T = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
  std::vector<std::vector<int32_t>> vals(T);
  std::vector<std::array<uint64_t, 9>> cnt(T);
  std::vector<std::thread> th;
  for (int t = 0; t < T; ++t) {
    th.emplace_back([&, t]() {
      std::vector<int32_t> local;
      std::array<uint64_t, 9> c{};
      int cards[7];
      for (int i = t; i < 52; i += T) {
        cards[0] = i;
        for (int j = i + 1; j < 52; ++j) {
          cards[1] = j;
          for (int k = j + 1; k < 52; ++k) {
            cards[2] = k;
            for (int m = k + 1; m < 52; ++m) {
              cards[3] = m;
              for (int n = m + 1; n < 52; ++n) {
                cards[4] = n;
                for (int p = n + 1; p < 52; ++p) {
                  cards[5] = p;
                  for (int q = p + 1; q < 52; ++q) {
                    cards[6] = q;
                    int32_t raw = hand_evaluate_internal(cards);
                    auto it = std::lower_bound(local.begin(), local.end(), raw);
                    if (it == local.end() || *it != raw) local.insert(it, raw);
                    c[raw >> 26] += 1;
                  }
                }
              }
            }
          }
        }
      }
      vals[t] = std::move(local);
      cnt[t] = c;
    });
  }
  for (auto& x : th) x.join();
  table.clear();
  for (int i = 0; i < 9; ++i) counts[i] = 0;
  for (int t = 0; t < T; ++t) {
    table.insert(table.end(), vals[t].begin(), vals[t].end());
    for (int i = 0; i < 9; ++i) counts[i] += cnt[t][i];
  }
  std::sort(table.begin(), table.end());
  table.erase(std::unique(table.begin(), table.end()), table.end());
}

// The evaluation table: loaded from the file the oracle build generates with
// hand_table_exhaustive (oracle/_build/hand_table.bin), else enumerated here.
static std::vector<int32_t> g_table;
static std::once_flag g_table_once;
static std::string g_table_path;

void set_hand_table_path(const char* p) { g_table_path = p ? p : ""; }

const std::vector<int32_t>& hand_table() {
  std::call_once(g_table_once, []() {
    if (!g_table_path.empty()) {
      FILE* f = fopen(g_table_path.c_str(), "rb");
      if (f) {
        std::vector<int32_t> t(4824);
        size_t n = fread(t.data(), 4, t.size(), f);
        fclose(f);
        if (n == t.size()) {
          g_table = std::move(t);
          return;
        }
      }
    }
    uint64_t c[9];
    hand_table_exhaustive(g_table, c);
  });
  return g_table;
}

// hand.rs:68-75: strength index = position in the sorted table.
uint16_t hand_evaluate(const int cards[7]) {
  const auto& t = hand_table();
  int32_t v = hand_evaluate_internal(cards);
  auto it = std::lower_bound(t.begin(), t.end(), v);
  if (it == t.end() || *it != v) throw std::runtime_error("hand value missing from table");
  return (uint16_t)(it - t.begin());
}

// ---------------------------------------------------------------------------
// bet_size.rs
// ---------------------------------------------------------------------------

static std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && isspace((unsigned char)s[a])) ++a;
  while (b > a && isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

static std::vector<std::string> split(const std::string& s, char c) {
  std::vector<std::string> out;
  size_t st = 0;
  for (size_t i = 0; i <= s.size(); ++i) {
    if (i == s.size() || s[i] == c) {
      out.push_back(s.substr(st, i - st));
      st = i + 1;
    }
  }
  return out;
}

// bet_size.rs:149-155
static bool parse_float(const std::string& s, double& out) {
  for (char ch : s)
    if (ch == '+' || ch == '-' || isalpha((unsigned char)ch)) return false;
  if (s.empty()) return false;
  char* end = nullptr;
  out = strtod(s.c_str(), &end);
  return end && *end == '\0';
}

static bool strip_suffix(const std::string& s, char c, std::string& out) {
  if (!s.empty() && s.back() == c) {
    out = s.substr(0, s.size() - 1);
    return true;
  }
  return false;
}

// bet_size.rs:157-260
static bool bet_size_from_str(const std::string& s, bool is_raise, BetSize& out, std::string& err) {
  std::string sl = s;
  for (auto& ch : sl) ch = (char)tolower((unsigned char)ch);
  err = "Invalid bet size: " + s;
  std::string pre;
  double fl;
  if (strip_suffix(sl, 'x', pre)) {
    if (!is_raise) {
      err = "Relative size to the previous bet is not allowed: " + s;
      return false;
    }
    if (!parse_float(pre, fl)) return false;
    if (fl <= 1.0) {
      err = "Multiplier must be greater than 1.0: " + s;
      return false;
    }
    out = {PrevBetRelative, fl, 0, 0};
    return true;
  } else if (sl.find('c') != std::string::npos) {
    auto parts = split(sl, 'c');
    if (parts.size() < 2) return false;
    double add;
    if (!parse_float(parts[0], add)) return false;
    if (std::trunc(add) != add) {
      err = "Additional size must be an integer: " + s;
      return false;
    }
    if (add > 2147483647.0) {
      err = "Additional size must be less than 2^31: " + s;
      return false;
    }
    int cap = 0;
    if (!parts[1].empty()) {
      if (!is_raise) {
        err = "Raise cap is not allowed: " + s;
        return false;
      }
      std::string fs;
      if (!strip_suffix(parts[1], 'r', fs)) return false;
      if (!parse_float(fs, fl)) return false;
      if (std::trunc(fl) != fl || fl == 0.0) {
        err = "Raise cap must be a positive integer: " + s;
        return false;
      } else if (fl > 100.0) {
        err = "Raise cap must be less than or equal to 100: " + s;
        return false;
      }
      cap = (int)fl;
    }
    if (parts.size() > 2) return false;
    out = {Additive, 0.0, (int)add, cap};
    return true;
  } else if (sl.find('e') != std::string::npos) {
    auto parts = split(sl, 'e');
    if (parts.size() < 2) return false;
    int ns = 0;
    if (!parts[0].empty()) {
      if (!parse_float(parts[0], fl)) return false;
      if (std::trunc(fl) != fl || fl == 0.0) {
        err = "Number of streets must be a positive integer: " + s;
        return false;
      } else if (fl > 100.0) {
        err = "Number of streets must be less than or equal to 100: " + s;
        return false;
      }
      ns = (int)fl;
    }
    double mx = INFINITY;
    if (!parts[1].empty()) {
      std::string ps;
      if (!strip_suffix(parts[1], '%', ps)) return false;
      if (!parse_float(ps, fl)) return false;
      mx = fl / 100.0;
    }
    if (parts.size() > 2) return false;
    out = {Geometric, mx, ns, 0};
    return true;
  } else if (strip_suffix(sl, '%', pre)) {
    if (!parse_float(pre, fl)) return false;
    out = {PotRelative, fl / 100.0, 0, 0};
    return true;
  } else if (sl == "a") {
    out = {AllIn, 0.0, 0, 0};
    return true;
  }
  return false;
}

// Derived PartialOrd of the BetSize enum (variant, then fields in order).
static bool bet_less(const BetSize& l, const BetSize& r) {
  if (l.kind != r.kind) return l.kind < r.kind;
  switch (l.kind) {
    case PotRelative:
    case PrevBetRelative: return l.f < r.f;
    case Additive: return l.i != r.i ? l.i < r.i : l.cap < r.cap;
    case Geometric: return l.i != r.i ? l.i < r.i : l.f < r.f;
    default: return false;
  }
}

static bool parse_list(const std::string& str, bool is_raise, std::vector<BetSize>& out,
                       std::string& err) {
  auto parts = split(str, ',');
  for (auto& p : parts) p = trim(p);
  if (parts.back().empty()) parts.pop_back();
  out.clear();
  for (auto& p : parts) {
    BetSize b;
    if (!bet_size_from_str(p, is_raise, b, err)) return false;
    out.push_back(b);
  }
  std::sort(out.begin(), out.end(), bet_less);
  return true;
}

// bet_size.rs:82-112
bool parse_bet_size_options(const std::string& bet, const std::string& raise, BetSizeOptions& out,
                            std::string& err) {
  return parse_list(bet, false, out.bet, err) && parse_list(raise, true, out.raise, err);
}

// bet_size.rs:114-137
bool parse_donk_size_options(const std::string& donk, std::vector<BetSize>& out, std::string& err) {
  return parse_list(donk, false, out, err);
}

// ---------------------------------------------------------------------------
// action_tree.rs
// ---------------------------------------------------------------------------

namespace {
struct BuildTreeInfo {  // action_tree.rs:226-293
  Action prev_action;
  int32_t num_bets = 0;
  bool allin_flag = false, oop_call_flag = false;
  int32_t stack[2] = {0, 0};
  int32_t prev_amount = 0;
  int street_transitions = 0;

  static BuildTreeInfo make(int32_t stack) {
    BuildTreeInfo b;
    b.stack[0] = b.stack[1] = stack;
    return b;
  }
  BuildTreeInfo create_next(uint8_t player, Action action) const {
    BuildTreeInfo n = *this;
    switch (action.kind) {
      case A_Check: n.oop_call_flag = false; break;
      case A_Call:
        n.num_bets = 0;
        n.oop_call_flag = player == PLAYER_OOP;
        n.stack[player] = n.stack[player ^ 1];
        n.prev_amount = 0;
        break;
      case A_Bet:
      case A_Raise:
      case A_AllIn: {
        int32_t to_call = n.stack[player] - n.stack[player ^ 1];
        n.num_bets += 1;
        n.allin_flag = action.kind == A_AllIn;
        n.stack[player] -= action.amount - n.prev_amount + to_call;
        n.prev_amount = action.amount;
        break;
      }
      case A_Chance: n.street_transitions += 1; break;
      default: break;
    }
    n.prev_action = action;
    return n;
  }
};

inline int32_t rround(double x) { return (int32_t)std::round(x); }

// action_tree.rs:1200-1229
std::vector<Action> merge_bet_actions(const std::vector<Action>& actions, int32_t pot,
                                      int32_t offset, double param) {
  const double EPS = 1e-12;
  auto get_amount = [](const Action& a) {
    return (a.kind == A_Bet || a.kind == A_Raise || a.kind == A_AllIn) ? a.amount : -1;
  };
  int32_t cur_amount = 2147483647;
  std::vector<Action> ret;
  for (auto it = actions.rbegin(); it != actions.rend(); ++it) {
    int32_t amount = get_amount(*it);
    if (amount > 0) {
      double ratio = (double)(amount - offset) / (double)pot;
      double cur_ratio = (double)(cur_amount - offset) / (double)pot;
      double threshold_ratio = (cur_ratio - param) / (1.0 + param);
      if (ratio < threshold_ratio * (1.0 - EPS)) {
        ret.push_back(*it);
        cur_amount = amount;
      }
    } else {
      ret.push_back(*it);
    }
  }
  std::reverse(ret.begin(), ret.end());
  return ret;
}

// action_tree.rs:705-925
void push_actions(const TreeConfig& cfg, ActionTreeNode& node, const BuildTreeInfo& info) {
  uint8_t player = node.player, opponent = node.player ^ 1;
  int32_t player_stack = info.stack[player], opponent_stack = info.stack[opponent];
  int32_t prev_amount = info.prev_amount;
  int32_t to_call = player_stack - opponent_stack;
  int32_t pot = cfg.starting_pot + 2 * (node.amount + to_call);
  int32_t max_amount = opponent_stack + prev_amount;
  int32_t min_amount = std::min(std::max(prev_amount + to_call, 1), max_amount);
  double spr_after_call = (double)opponent_stack / (double)pot;
  auto compute_geometric = [&](int num_streets, double max_ratio) {
    double ratio = (std::pow(2.0 * spr_after_call + 1.0, 1.0 / (double)num_streets) - 1.0) / 2.0;
    return rround((double)pot * std::min(ratio, max_ratio));
  };
  const BetSizeOptions* bet_options;
  const std::vector<BetSize>* donk_options = nullptr;
  int num_remaining_streets;
  switch (node.board_state) {
    case Flop: bet_options = cfg.flop_bet_sizes; num_remaining_streets = 3; break;
    case Turn:
      bet_options = cfg.turn_bet_sizes;
      if (cfg.has_turn_donk) donk_options = &cfg.turn_donk_sizes;
      num_remaining_streets = 2;
      break;
    default:
      bet_options = cfg.river_bet_sizes;
      if (cfg.has_river_donk) donk_options = &cfg.river_donk_sizes;
      num_remaining_streets = 1;
      break;
  }
  std::vector<Action> actions;
  auto push_bet_list = [&](const std::vector<BetSize>& list) {
    for (const auto& b : list) {
      switch (b.kind) {
        case PotRelative: actions.push_back({A_Bet, rround((double)pot * b.f)}); break;
        case PrevBetRelative: throw std::runtime_error("Unexpected `PrevBetRelative`");
        case Additive: actions.push_back({A_Bet, b.i}); break;
        case Geometric: {
          int ns = b.i == 0 ? num_remaining_streets : b.i;
          actions.push_back({A_Bet, compute_geometric(ns, b.f)});
          break;
        }
        case AllIn: actions.push_back({A_AllIn, max_amount}); break;
      }
    }
    if (max_amount <= rround((double)pot * cfg.add_allin_threshold))
      actions.push_back({A_AllIn, max_amount});
  };
  if (donk_options && info.prev_action.kind == A_Chance && info.oop_call_flag) {
    actions.push_back({A_Check, 0});
    push_bet_list(*donk_options);
  } else if (info.prev_action.kind == A_None || info.prev_action.kind == A_Check ||
             info.prev_action.kind == A_Chance) {
    actions.push_back({A_Check, 0});
    push_bet_list(bet_options[player].bet);
  } else {
    actions.push_back({A_Fold, 0});
    actions.push_back({A_Call, 0});
    if (!info.allin_flag) {
      for (const auto& b : bet_options[player].raise) {
        switch (b.kind) {
          case PotRelative:
            actions.push_back({A_Raise, prev_amount + rround((double)pot * b.f)});
            break;
          case PrevBetRelative:
            actions.push_back({A_Raise, rround((double)prev_amount * b.f)});
            break;
          case Additive:
            if (b.cap == 0 || info.num_bets <= b.cap)
              actions.push_back({A_Raise, prev_amount + b.i});
            break;
          case Geometric: {
            int ns = b.i == 0 ? std::max(num_remaining_streets - info.num_bets + 1, 1)
                              : std::max(b.i - info.num_bets + 1, 1);
            actions.push_back({A_Raise, prev_amount + compute_geometric(ns, b.f)});
            break;
          }
          case AllIn: actions.push_back({A_AllIn, max_amount}); break;
        }
      }
      double allin_threshold = (double)pot * cfg.add_allin_threshold;
      if (max_amount <= prev_amount + rround(allin_threshold))
        actions.push_back({A_AllIn, max_amount});
    }
  }
  auto is_above_threshold = [&](int32_t amount) {
    int32_t new_amount_diff = amount - prev_amount;
    int32_t new_pot = pot + 2 * new_amount_diff;
    int32_t threshold = rround((double)new_pot * cfg.force_allin_threshold);
    return max_amount <= amount + threshold;
  };
  for (auto& a : actions) {
    if (a.kind == A_Bet || a.kind == A_Raise) {
      int32_t clamped = std::min(std::max(a.amount, min_amount), max_amount);
      if (is_above_threshold(clamped))
        a = {A_AllIn, max_amount};
      else if (clamped != a.amount)
        a.amount = clamped;
    }
  }
  std::sort(actions.begin(), actions.end());
  actions.erase(std::unique(actions.begin(), actions.end()), actions.end());
  actions = merge_bet_actions(actions, pot, prev_amount, cfg.merging_threshold);

  bool depth_limit_reached = cfg.depth_limit >= 0 && info.street_transitions >= cfg.depth_limit;
  uint8_t player_after_call = node.board_state == River ? PLAYER_TERMINAL_FLAG
                              : depth_limit_reached     ? PLAYER_DEPTH_BOUNDARY_FLAG
                                                        : (uint8_t)(PLAYER_CHANCE_FLAG | player);
  uint8_t player_after_check = player == PLAYER_OOP ? opponent : player_after_call;
  for (const auto& a : actions) {
    int32_t amount = node.amount;
    uint8_t next_player;
    switch (a.kind) {
      case A_Fold: next_player = PLAYER_FOLD_FLAG | player; break;
      case A_Check: next_player = player_after_check; break;
      case A_Call:
        amount += to_call;
        next_player = player_after_call;
        break;
      case A_Bet:
      case A_Raise:
      case A_AllIn:
        amount += to_call;
        next_player = opponent;
        break;
      default: throw std::runtime_error("Unexpected action");
    }
    node.actions.push_back(a);
    auto c = std::make_unique<ActionTreeNode>();
    c->player = next_player;
    c->board_state = node.board_state;
    c->amount = amount;
    node.children.push_back(std::move(c));
  }
}

// action_tree.rs:646-702
void build_tree_recursive(const TreeConfig& cfg, ActionTreeNode& node, const BuildTreeInfo& info) {
  if (node.is_terminal()) return;
  if (node.is_chance()) {
    if (cfg.depth_limit >= 0 && info.street_transitions >= cfg.depth_limit) {
      node.player = PLAYER_DEPTH_BOUNDARY_FLAG;
      node.actions.clear();
      node.children.clear();
      return;
    }
    BoardState next_state = node.board_state == Flop ? Turn : River;
    bool second_blocked = cfg.depth_limit >= 0 && info.street_transitions + 1 >= cfg.depth_limit;
    uint8_t next_player;
    if (!info.allin_flag)
      next_player = PLAYER_OOP;
    else if (node.board_state == Flop)
      next_player = second_blocked ? PLAYER_DEPTH_BOUNDARY_FLAG
                                   : (uint8_t)(PLAYER_CHANCE_FLAG | PLAYER_CHANCE);
    else
      next_player = PLAYER_TERMINAL_FLAG;
    node.actions.push_back({A_Chance, 0});
    auto c = std::make_unique<ActionTreeNode>();
    c->player = next_player;
    c->board_state = next_state;
    c->amount = node.amount;
    node.children.push_back(std::move(c));
    build_tree_recursive(cfg, *node.children[0], info.create_next(0, {A_Chance, 0}));
  } else {
    push_actions(cfg, node, info);
    for (size_t i = 0; i < node.children.size(); ++i)
      build_tree_recursive(cfg, *node.children[i], info.create_next(node.player, node.actions[i]));
  }
}

void invalid_terminals_recursive(const ActionTreeNode& node, std::vector<std::vector<Action>>& out,
                                 std::vector<Action>& line) {  // action_tree.rs:928-945
  if (node.is_terminal()) return;
  if (node.children.empty()) {
    out.push_back(line);
  } else if (node.is_chance()) {
    invalid_terminals_recursive(*node.children[0], out, line);
  } else {
    for (size_t i = 0; i < node.children.size(); ++i) {
      line.push_back(node.actions[i]);
      invalid_terminals_recursive(*node.children[i], out, line);
      line.pop_back();
    }
  }
}

// action_tree.rs:1177-1198
void count_num_action_nodes_recursive(const ActionTreeNode& node, int street, uint64_t count[3]) {
  count[street] += 1;
  if (node.is_terminal()) return;
  if (node.is_chance()) {
    count_num_action_nodes_recursive(*node.children[0], street + 1, count);
  } else {
    for (const auto& c : node.children) count_num_action_nodes_recursive(*c, street, count);
  }
}
}  // namespace

// action_tree.rs:326-334 + check_config :560-628 + build_tree :631-636
bool ActionTree::create(const TreeConfig& cfg, ActionTree& out, std::string& err) {
  char buf[160];
  if (cfg.starting_pot <= 0) {
    snprintf(buf, sizeof buf, "Starting pot must be positive: %d", cfg.starting_pot);
    err = buf;
    return false;
  }
  if (cfg.effective_stack <= 0) {
    snprintf(buf, sizeof buf, "Effective stack must be positive: %d", cfg.effective_stack);
    err = buf;
    return false;
  }
  if (cfg.rake_rate < 0.0) { err = "Rake rate must be non-negative"; return false; }
  if (cfg.rake_rate > 1.0) { err = "Rake rate must be less than or equal to 1.0"; return false; }
  if (cfg.rake_cap < 0.0) { err = "Rake cap must be non-negative"; return false; }
  if (cfg.add_allin_threshold < 0.0) { err = "Add all-in threshold must be non-negative"; return false; }
  if (cfg.force_allin_threshold < 0.0) { err = "Force all-in threshold must be non-negative"; return false; }
  if (cfg.merging_threshold < 0.0) { err = "Merging threshold must be non-negative"; return false; }
  out.config = cfg;
  out.root = std::make_unique<ActionTreeNode>();
  out.root->board_state = cfg.initial_state;
  try {
    build_tree_recursive(out.config, *out.root, BuildTreeInfo::make(cfg.effective_stack));
  } catch (const std::exception& e) {
    err = e.what();
    return false;
  }
  return true;
}

std::vector<std::vector<Action>> ActionTree::invalid_terminals() const {
  std::vector<std::vector<Action>> out;
  std::vector<Action> line;
  invalid_terminals_recursive(*root, out, line);
  return out;
}

// ---------------------------------------------------------------------------
// range.rs
// ---------------------------------------------------------------------------

// range.rs:256-275
void Range::get_hands_weights(uint64_t dead, std::vector<std::pair<Card, Card>>& hands,
                              std::vector<float>& weights) const {
  hands.clear();
  weights.clear();
  for (int c1 = 0; c1 < 52; ++c1)
    for (int c2 = c1 + 1; c2 < 52; ++c2) {
      uint64_t m = (1ull << c1) | (1ull << c2);
      float w = data[card_pair_to_index(c1, c2)];
      if (w > 0.0f && (m & dead) == 0) {
        hands.push_back({(Card)c1, (Card)c2});
        weights.push_back(w);
      }
    }
}

// range.rs:426-450
bool Range::is_suit_isomorphic(int s1, int s2) const {
  auto rep = [&](int s) { return s == s1 ? s2 : s == s2 ? s1 : s; };
  for (int c1 = 0; c1 < 52; ++c1)
    for (int c2 = c1 + 1; c2 < 52; ++c2) {
      int r1 = (c1 & ~3) | rep(c1 & 3), r2 = (c2 & ~3) | rep(c2 & 3);
      if (data[card_pair_to_index(c1, c2)] != data[card_pair_to_index(r1, r2)]) return false;
    }
  return true;
}

bool Range::is_empty() const {
  for (float w : data)
    if (w != 0.0f) return false;
  return true;
}
bool Range::is_valid() const {
  for (float w : data)
    if (!(w >= 0.0f && w <= 1.0f)) return false;
  return true;
}

// ---------------------------------------------------------------------------
// solver.rs:26-44
// ---------------------------------------------------------------------------

DiscountParams::DiscountParams(uint32_t t) {
  uint32_t nearest_lower_power_of_4 = t == 0 ? 0 : 1u << ((31 - __builtin_clz(t)) & ~1);
  double t_alpha = (double)std::max((int32_t)t - 1, 0);
  double t_gamma = (double)(t - nearest_lower_power_of_4);
  double pow_alpha = t_alpha * std::sqrt(t_alpha);
  double g = t_gamma / (t_gamma + 1.0);
  double pow_gamma = (g * g) * g;
  alpha_t = (float)(pow_alpha / (pow_alpha + 1.0));
  beta_t = 0.5f;
  gamma_t = (float)pow_gamma;
}

// ---------------------------------------------------------------------------
// Game: construction (game/interpreter.rs, card.rs, isomorphism.rs)
// ---------------------------------------------------------------------------

template <class F>
bool Game<F>::with_config(const CardConfig& cc, ActionTree&& tree, std::string& err) {
  // interpreter.rs:128-166
  state = State::ConfigError;
  if (!tree.invalid_terminals().empty()) {
    err = "Invalid terminal found in action tree";
    return false;
  }
  card_config = cc;
  tree_config = tree.config;
  action_root = std::move(tree.root);
  if (!check_card_config(err)) return false;
  init_card_fields();
  if (!init_root(err)) return false;
  state = State::TreeBuilt;
  for (int p = 0; p < 2; ++p) {  // init_interpreter, interpreter.rs:1010-1019
    weights[p].assign(num_private_hands(p), (F)0);
    normalized_weights[p].assign(num_private_hands(p), (F)0);
    cfvalues_cache[p].assign(num_private_hands(p), (F)0);
  }
  return true;
}

// interpreter.rs:542-642
template <class F>
bool Game<F>::check_card_config(std::string& err) {
  const auto& c = card_config;
  char buf[200];
  for (int i = 0; i < 3; ++i)
    if (c.flop[i] == NOT_DEALT) { err = "Flop cards not initialized"; return false; }
  for (int i = 0; i < 3; ++i)
    if (c.flop[i] >= 52) { err = "Flop cards must be in [0, 52)"; return false; }
  if (c.flop[0] == c.flop[1] || c.flop[0] == c.flop[2] || c.flop[1] == c.flop[2]) {
    err = "Flop cards must be unique";
    return false;
  }
  auto in_flop = [&](Card x) { return x == c.flop[0] || x == c.flop[1] || x == c.flop[2]; };
  if (c.turn != NOT_DEALT) {
    if (c.turn >= 52) { snprintf(buf, sizeof buf, "Turn card must be in [0, 52): turn = %d", c.turn); err = buf; return false; }
    if (in_flop(c.turn)) { snprintf(buf, sizeof buf, "Turn card must be different from flop cards: turn = %d", c.turn); err = buf; return false; }
  }
  if (c.river != NOT_DEALT) {
    if (c.river >= 52) { snprintf(buf, sizeof buf, "River card must be in [0, 52): river = %d", c.river); err = buf; return false; }
    if (in_flop(c.river)) { snprintf(buf, sizeof buf, "River card must be different from flop cards: river = %d", c.river); err = buf; return false; }
    if (c.turn == c.river) { snprintf(buf, sizeof buf, "River card must be different from turn card: river = %d", c.river); err = buf; return false; }
    if (c.turn == NOT_DEALT) { snprintf(buf, sizeof buf, "River card specified without turn card: river = %d", c.river); err = buf; return false; }
  }
  BoardState expected = c.turn == NOT_DEALT ? Flop : c.river == NOT_DEALT ? Turn : River;
  if (tree_config.initial_state != expected) {
    err = "Invalid initial state of `tree_config`";
    return false;
  }
  if (c.range[0].is_empty()) { err = "OOP range is empty"; return false; }
  if (c.range[1].is_empty()) { err = "IP range is empty"; return false; }
  if (!c.range[0].is_valid()) { err = "OOP range is invalid (loaded broken data?)"; return false; }
  if (!c.range[1].is_valid()) { err = "IP range is invalid (loaded broken data?)"; return false; }

  // init_hands, interpreter.rs:645-662
  uint64_t board_mask = (1ull << c.flop[0]) | (1ull << c.flop[1]) | (1ull << c.flop[2]);
  if (c.turn != NOT_DEALT) board_mask |= 1ull << c.turn;
  if (c.river != NOT_DEALT) board_mask |= 1ull << c.river;
  for (int p = 0; p < 2; ++p) {
    std::vector<float> w;
    c.range[p].get_hands_weights(board_mask, private_cards[p], w);
    initial_weights[p].assign(w.begin(), w.end());
  }
  num_combinations = 0.0;
  for (size_t i = 0; i < private_cards[0].size(); ++i) {
    auto [c1, c2] = private_cards[0][i];
    uint64_t om = (1ull << c1) | (1ull << c2);
    double w1 = (double)(float)initial_weights[0][i];
    for (size_t j = 0; j < private_cards[1].size(); ++j) {
      auto [c3, c4] = private_cards[1][j];
      uint64_t im = (1ull << c3) | (1ull << c4);
      if ((om & im) == 0) num_combinations += w1 * (double)(float)initial_weights[1][j];
    }
  }
  if (num_combinations == 0.0) {
    err = "Valid card assignment does not exist";
    return false;
  }
  return true;
}

// card.rs:127-156
static Indices valid_indices_internal(const std::vector<std::pair<Card, Card>> pc[2], int b1, int b2) {
  Indices ret;
  uint64_t bm = 0;
  if (b1 != NOT_DEALT) bm |= 1ull << b1;
  if (b2 != NOT_DEALT) bm |= 1ull << b2;
  for (int p = 0; p < 2; ++p)
    for (size_t i = 0; i < pc[p].size(); ++i) {
      uint64_t hm = (1ull << pc[p][i].first) | (1ull << pc[p][i].second);
      if ((hm & bm) == 0) ret[p].push_back((uint16_t)i);
    }
  return ret;
}

// interpreter.rs:671-704 (same_hand_index), card.rs:81-226, isomorphism.rs
template <class F>
void Game<F>::init_card_fields() {
  for (int p = 0; p < 2; ++p) {
    same_hand_index[p].clear();
    const auto& opp = private_cards[p ^ 1];
    for (const auto& h : private_cards[p]) {
      auto it = std::lower_bound(opp.begin(), opp.end(), h);
      same_hand_index[p].push_back(it != opp.end() && *it == h ? (uint16_t)(it - opp.begin())
                                                               : (uint16_t)0xFFFF);
    }
  }
  const auto& c = card_config;
  auto in_flop = [&](int x) { return x == c.flop[0] || x == c.flop[1] || x == c.flop[2]; };
  // card.rs:81-122
  valid_indices_flop = Indices();
  if (c.turn == NOT_DEALT)
    for (int p = 0; p < 2; ++p)
      for (size_t i = 0; i < private_cards[p].size(); ++i) valid_indices_flop[p].push_back((uint16_t)i);
  valid_indices_turn.assign(52, Indices());
  for (int b = 0; b < 52; ++b)
    if (!in_flop(b) && (c.turn == NOT_DEALT || c.turn == b) && c.river == NOT_DEALT)
      valid_indices_turn[b] = valid_indices_internal(private_cards, b, NOT_DEALT);
  valid_indices_river.assign(1326, Indices());
  hand_strength.assign(1326, {});
  for (int b1 = 0; b1 < 52; ++b1)
    for (int b2 = b1 + 1; b2 < 52; ++b2) {
      if (in_flop(b1) || in_flop(b2)) continue;
      if (!(c.turn == NOT_DEALT || b1 == c.turn || b2 == c.turn)) continue;
      if (!(c.river == NOT_DEALT || b1 == c.river || b2 == c.river)) continue;
      int idx = card_pair_to_index(b1, b2);
      valid_indices_river[idx] = valid_indices_internal(private_cards, b1, b2);
      // card.rs:163-226
      int cards[7] = {c.flop[0], c.flop[1], c.flop[2], b1, b2, 0, 0};
      for (int p = 0; p < 2; ++p) {
        auto& v = hand_strength[idx][p];
        v.push_back({0, 0});
        v.push_back({0xFFFF, 0xFFFF});
        for (size_t i = 0; i < private_cards[p].size(); ++i) {
          int h1 = private_cards[p][i].first, h2 = private_cards[p][i].second;
          bool blocked = false;
          for (int k = 0; k < 5; ++k)
            if (cards[k] == h1 || cards[k] == h2) blocked = true;
          if (blocked) continue;
          cards[5] = h1;
          cards[6] = h2;
          v.push_back({(uint16_t)(hand_evaluate(cards) + 1), (uint16_t)i});
        }
        std::sort(v.begin(), v.end());
      }
    }
  compute_isomorphism();
}

// isomorphism.rs:160-202
static void isomorphism_swap_internal(std::array<SwapList, 4>& swap_list, std::vector<size_t>& rev,
                                      int suit1, int suit2,
                                      const std::vector<std::pair<Card, Card>> pc[2]) {
  auto& sl = swap_list[suit1];
  auto replacer = [&](int card) {
    if ((card & 3) == suit1) return card - suit1 + suit2;
    if ((card & 3) == suit2) return card + suit1 - suit2;
    return card;
  };
  for (int p = 0; p < 2; ++p) {
    if (!sl[p].empty()) continue;
    std::fill(rev.begin(), rev.end(), (size_t)-1);
    for (size_t i = 0; i < pc[p].size(); ++i) rev[card_pair_to_index(pc[p][i].first, pc[p][i].second)] = i;
    for (size_t i = 0; i < pc[p].size(); ++i) {
      int c1 = replacer(pc[p][i].first), c2 = replacer(pc[p][i].second);
      size_t index = rev[card_pair_to_index(c1, c2)];
      if (index != (size_t)-1 && i < index) sl[p].push_back({(uint16_t)i, (uint16_t)index});
    }
  }
}

// isomorphism.rs:209-234
static void isomorphism_internal(std::vector<uint8_t>& iref, std::vector<Card>& icard, uint64_t mask,
                                 const int isomorphic_suit[4]) {
  bool push_card = icard.empty();
  uint8_t counter = 0;
  uint8_t indices[52] = {0};
  for (int card = 0; card < 52; ++card) {
    if ((1ull << card) & mask) continue;
    int suit = card & 3;
    if (isomorphic_suit[suit] >= 0) {
      int replace_card = card - suit + isomorphic_suit[suit];
      iref.push_back(indices[replace_card]);
      if (push_card) icard.push_back((Card)card);
    } else {
      indices[card] = counter++;
    }
  }
}

// isomorphism.rs:33-154
template <class F>
void Game<F>::compute_isomorphism() {
  const auto& c = card_config;
  int suit_iso[4] = {0, 0, 0, 0};
  int next_index = 1;
  for (int s2 = 1; s2 < 4; ++s2) {
    bool found = false;
    for (int s1 = 0; s1 < s2; ++s1) {
      if (c.range[0].is_suit_isomorphic(s1, s2) && c.range[1].is_suit_isomorphic(s1, s2)) {
        suit_iso[s2] = suit_iso[s1];
        found = true;
        break;
      }
    }
    if (!found) suit_iso[s2] = next_index++;
  }
  uint64_t flop_mask = (1ull << c.flop[0]) | (1ull << c.flop[1]) | (1ull << c.flop[2]);
  uint16_t flop_rankset[4] = {0, 0, 0, 0};
  for (int k = 0; k < 3; ++k) flop_rankset[c.flop[k] & 3] |= (uint16_t)(1 << (c.flop[k] >> 2));
  int iso_suit[4] = {-1, -1, -1, -1};
  std::vector<size_t> rev(1326, (size_t)-1);
  isomorphism_ref_turn.clear();
  isomorphism_card_turn.clear();
  isomorphism_swap_turn = {};
  if (c.turn == NOT_DEALT) {
    for (int s1 = 1; s1 < 4; ++s1)
      for (int s2 = 0; s2 < s1; ++s2)
        if (flop_rankset[s1] == flop_rankset[s2] && suit_iso[s1] == suit_iso[s2]) {
          iso_suit[s1] = s2;
          isomorphism_swap_internal(isomorphism_swap_turn, rev, s1, s2, private_cards);
          break;
        }
    isomorphism_internal(isomorphism_ref_turn, isomorphism_card_turn, flop_mask, iso_suit);
  }
  isomorphism_ref_river.assign(52, {});
  isomorphism_card_river = {};
  isomorphism_swap_river = {};
  if (c.river == NOT_DEALT) {
    for (int t = 0; t < 52; ++t) {
      if (((1ull << t) & flop_mask) || (c.turn != NOT_DEALT && c.turn != t)) continue;
      uint64_t turn_mask = flop_mask | (1ull << t);
      uint16_t turn_rankset[4] = {flop_rankset[0], flop_rankset[1], flop_rankset[2], flop_rankset[3]};
      turn_rankset[t & 3] |= (uint16_t)(1 << (t >> 2));
      for (int k = 0; k < 4; ++k) iso_suit[k] = -1;
      for (int s1 = 1; s1 < 4; ++s1)
        for (int s2 = 0; s2 < s1; ++s2)
          if ((flop_rankset[s1] == flop_rankset[s2] || c.turn != NOT_DEALT) &&
              turn_rankset[s1] == turn_rankset[s2] && suit_iso[s1] == suit_iso[s2]) {
            iso_suit[s1] = s2;
            isomorphism_swap_internal(isomorphism_swap_river[t & 3], rev, s1, s2, private_cards);
            break;
          }
      isomorphism_internal(isomorphism_ref_river[t], isomorphism_card_river[t & 3], turn_mask, iso_suit);
    }
  }
}

// interpreter.rs:708-743
template <class F>
void Game<F>::count_num_nodes(uint64_t out[3]) {
  uint64_t turn_coef, river_coef;
  const auto& c = card_config;
  if (c.turn == NOT_DEALT) {
    river_coef = 0;
    uint64_t flop_mask = (1ull << c.flop[0]) | (1ull << c.flop[1]) | (1ull << c.flop[2]);
    uint64_t skip = 0;
    for (Card x : isomorphism_card_turn) skip += 1ull << x;
    for (int t = 0; t < 52; ++t)
      if (((1ull << t) & (flop_mask | skip)) == 0) river_coef += 48 - isomorphism_card_river[t & 3].size();
    turn_coef = 49 - isomorphism_card_turn.size();
  } else if (c.river == NOT_DEALT) {
    turn_coef = 1;
    river_coef = 48 - isomorphism_card_river[c.turn & 3].size();
  } else {
    turn_coef = 0;
    river_coef = 1;
  }
  uint64_t cnt[3] = {0, 0, 0};
  count_num_action_nodes_recursive(*action_root, (int)tree_config.initial_state, cnt);
  out[0] = cnt[0];
  out[1] = cnt[1] * turn_coef;
  out[2] = cnt[2] * river_coef;
}

// interpreter.rs:746-806
template <class F>
bool Game<F>::init_root(std::string& err) {
  count_num_nodes(num_nodes_street);
  uint64_t total = num_nodes_street[0] + num_nodes_street[1] + num_nodes_street[2];
  if (total > 0xFFFFFFFFull) {
    err = "Too many nodes";
    return false;
  }
  arena.assign(total, Node());
  uint64_t info[3] = {0, num_nodes_street[0], num_nodes_street[0] + num_nodes_street[1]};
  info[(int)tree_config.initial_state] += 1;
  arena[0].turn = card_config.turn;
  arena[0].river = card_config.river;
  num_storage = num_storage_ip = num_storage_chance = 0;
  build_tree_recursive(0, *action_root, info);
  node_to_boundary.assign(total, 0xFFFFFFFFu);
  uint32_t bc = 0;
  for (size_t i = 0; i < arena.size(); ++i)
    if (arena[i].is_depth_boundary()) node_to_boundary[i] = bc++;
  boundary_cfvs.assign((size_t)bc * 2, {});
  boundary_reach.assign((size_t)bc * 2, {});
  return true;
}

// interpreter.rs:809-853
template <class F>
void Game<F>::build_tree_recursive(size_t ni, const ActionTreeNode& an, uint64_t info[3]) {
  arena[ni].player = an.player;
  arena[ni].amount = an.amount;
  if (arena[ni].is_terminal()) return;
  if (arena[ni].is_chance()) {
    push_chances(ni, info);
    size_t n = arena[ni].num_children, off = arena[ni].children_offset;
    for (size_t a = 0; a < n; ++a) build_tree_recursive(ni + off + a, *an.children[0], info);
  } else {
    push_actions(ni, an, info);
    size_t n = arena[ni].num_children, off = arena[ni].children_offset;
    for (size_t a = 0; a < n; ++a) build_tree_recursive(ni + off + a, *an.children[a], info);
  }
}

// interpreter.rs:856-905
template <class F>
void Game<F>::push_chances(size_t ni, uint64_t info[3]) {
  Node& node = arena[ni];
  const auto& c = card_config;
  uint64_t flop_mask = (1ull << c.flop[0]) | (1ull << c.flop[1]) | (1ull << c.flop[2]);
  if (node.turn == NOT_DEALT) {
    uint64_t skip = 0;
    for (Card x : isomorphism_card_turn) skip += 1ull << x;
    node.children_offset = (uint32_t)(info[1] - ni);
    for (int card = 0; card < 52; ++card)
      if (((1ull << card) & (flop_mask | skip)) == 0) {
        node.num_children += 1;
        Node& ch = arena[ni + node.children_offset + node.num_children - 1];
        ch.prev_action = {A_Chance, card};
        ch.turn = (Card)card;
      }
    info[1] += node.num_children;
  } else {
    uint64_t turn_mask = flop_mask | (1ull << node.turn);
    uint64_t skip = 0;
    for (Card x : isomorphism_card_river[node.turn & 3]) skip += 1ull << x;
    node.children_offset = (uint32_t)(info[2] - ni);
    for (int card = 0; card < 52; ++card)
      if (((1ull << card) & (turn_mask | skip)) == 0) {
        node.num_children += 1;
        Node& ch = arena[ni + node.children_offset + node.num_children - 1];
        ch.prev_action = {A_Chance, card};
        ch.turn = node.turn;
        ch.river = (Card)card;
      }
    info[2] += node.num_children;
  }
  int sp = node.cfvalue_storage_player();
  node.num_elements = sp < 0 ? 0 : (uint32_t)num_private_hands(sp);
  num_storage_chance += node.num_elements;
}

// interpreter.rs:908-947
template <class F>
void Game<F>::push_actions(size_t ni, const ActionTreeNode& an, uint64_t info[3]) {
  Node& node = arena[ni];
  int street = node.turn == NOT_DEALT ? 0 : node.river == NOT_DEALT ? 1 : 2;
  node.children_offset = (uint32_t)(info[street] - ni);
  node.num_children = (uint16_t)an.children.size();
  info[street] += node.num_children;
  for (size_t a = 0; a < an.children.size(); ++a) {
    Node& ch = arena[ni + node.children_offset + a];
    ch.prev_action = an.actions[a];
    ch.turn = node.turn;
    ch.river = node.river;
  }
  node.num_elements = (uint32_t)(node.num_children * num_private_hands(node.player));
  node.num_elements_ip = (node.prev_action.kind == A_None || node.prev_action.kind == A_Chance)
                             ? (uint16_t)num_private_hands(PLAYER_IP)
                             : 0;
  num_storage += node.num_elements;
  num_storage_ip += node.num_elements_ip;
}

// interpreter.rs:212-249 (uncompressed storage only)
template <class F>
void Game<F>::allocate_memory() {
  if (state <= State::Uninitialized) throw std::runtime_error("Game is not successfully initialized");
  state = State::MemoryAllocated;
  storage1.assign(num_storage, (F)0);
  storage2.assign(num_storage, (F)0);
  storage_ip.assign(num_storage_ip, (F)0);
  storage_chance.assign(num_storage_chance, (F)0);
  allocate_memory_nodes();
}

// interpreter.rs:971-1007
template <class F>
void Game<F>::allocate_memory_nodes() {
  size_t ac = 0, ic = 0, cc = 0;
  for (auto& n : arena) {
    if (n.is_terminal()) continue;
    if (n.is_chance()) {
      n.s1 = cc;
      cc += n.num_elements;
    } else {
      n.s1 = n.s2 = ac;
      n.s3 = ic;
      ac += n.num_elements;
      ic += n.num_elements_ip;
    }
  }
}

// interpreter.rs:84-102
template <class F>
const std::vector<uint8_t>& Game<F>::isomorphic_chances(const Node& n) const {
  return n.turn == NOT_DEALT ? isomorphism_ref_turn : isomorphism_ref_river[n.turn];
}
template <class F>
const SwapList& Game<F>::isomorphic_swap(const Node& n, size_t i) const {
  if (n.turn == NOT_DEALT) return isomorphism_swap_turn[isomorphism_card_turn[i] & 3];
  return isomorphism_swap_river[n.turn & 3][isomorphism_card_river[n.turn & 3][i] & 3];
}
template <class F>
const std::vector<F>* Game<F>::locking(const Node& n) const {
  if (!n.is_locked) return nullptr;
  return &locking_strategy.at(node_index(&n));
}

// ---------------------------------------------------------------------------
// game/evaluation.rs
// ---------------------------------------------------------------------------

template <class F>
const Indices& Game<F>::valid_indices_for(const Node& node) const {
  if (node.river != NOT_DEALT) return valid_indices_river[card_pair_to_index(node.turn, node.river)];
  if (node.turn != NOT_DEALT) return valid_indices_turn[node.turn];
  return valid_indices_flop;
}

static inline double min_f64(double x, double y) { return x < y ? x : y; }

// evaluation.rs:57-538 (boundary single-continuation, fold, unraked/raked showdown)
template <class F>
void Game<F>::evaluate(F* result, const Node& node, int player, const F* cfreach) {
  double pot = (double)(tree_config.starting_pot + 2 * node.amount);
  double half_pot = 0.5 * pot;
  double rake = min_f64(pot * tree_config.rake_rate, tree_config.rake_cap);
  double amount_win = (half_pot - rake) / num_combinations;
  double amount_lose = -half_pot / num_combinations;
  const auto& pcards = private_cards[player];
  const auto& ocards = private_cards[player ^ 1];
  size_t nh = num_private_hands(player), no = num_private_hands(player ^ 1);
  double cfreach_sum = 0.0;
  double cfreach_minus[52];
  for (int k = 0; k < 52; ++k) cfreach_minus[k] = 0.0;
  for (size_t i = 0; i < nh; ++i) result[i] = (F)0;

  if (node.is_depth_boundary()) {  // evaluation.rs:87-179 (K <= 1)
    size_t ordinal = node_to_boundary[node_index(&node)];
    int opp = player ^ 1;
    boundary_reach[ordinal * 2 + opp].assign(cfreach, cfreach + no);
    const auto& b = boundary_cfvs[ordinal * 2 + player];
    if (b.empty()) throw std::runtime_error("boundary_cfvs empty with no evaluator set");
    evaluate_boundary_single(result, node, player, cfreach, b, half_pot);
    return;
  }

  if ((node.player & PLAYER_FOLD_FLAG) == PLAYER_FOLD_FLAG) {  // evaluation.rs:293-353
    int folded = node.player & PLAYER_MASK;
    double payoff = folded != player ? amount_win : amount_lose;
    const auto& vi = valid_indices_for(node);
    for (uint16_t i : vi[player ^ 1]) {
      F r = cfreach[i];
      if (r != (F)0) {
        double rd = (double)r;
        cfreach_sum += rd;
        cfreach_minus[ocards[i].first] += rd;
        cfreach_minus[ocards[i].second] += rd;
      }
    }
    if (cfreach_sum == 0.0) return;
    const auto& same = same_hand_index[player];
    for (uint16_t i : vi[player]) {
      double cs = same[i] == 0xFFFF ? 0.0 : (double)cfreach[same[i]];
      double cr = cfreach_sum + cs - cfreach_minus[pcards[i].first] - cfreach_minus[pcards[i].second];
      result[i] = (F)(payoff * cr);
    }
  } else if (rake == 0.0) {  // evaluation.rs:357-425
    const auto& hs = hand_strength[card_pair_to_index(node.turn, node.river)];
    const auto& ps = hs[player];
    const auto& os = hs[player ^ 1];
    size_t i = 1;
    for (size_t k = 1; k + 1 < ps.size(); ++k) {
      uint16_t strength = ps[k].strength, index = ps[k].index;
      while (os[i].strength < strength) {
        size_t oi = os[i].index;
        F r = cfreach[oi];
        if (r != (F)0) {
          double rd = (double)r;
          cfreach_sum += rd;
          cfreach_minus[ocards[oi].first] += rd;
          cfreach_minus[ocards[oi].second] += rd;
        }
        ++i;
      }
      double cr = cfreach_sum - cfreach_minus[pcards[index].first] - cfreach_minus[pcards[index].second];
      result[index] = (F)(amount_win * cr);
    }
    cfreach_sum = 0.0;
    for (int c = 0; c < 52; ++c) cfreach_minus[c] = 0.0;
    i = os.size() - 2;
    for (size_t k = ps.size() - 2; k >= 1; --k) {
      uint16_t strength = ps[k].strength, index = ps[k].index;
      while (os[i].strength > strength) {
        size_t oi = os[i].index;
        F r = cfreach[oi];
        if (r != (F)0) {
          double rd = (double)r;
          cfreach_sum += rd;
          cfreach_minus[ocards[oi].first] += rd;
          cfreach_minus[ocards[oi].second] += rd;
        }
        --i;
      }
      double cr = cfreach_sum - cfreach_minus[pcards[index].first] - cfreach_minus[pcards[index].second];
      result[index] += (F)(amount_lose * cr);
    }
  } else {  // evaluation.rs:429-537
    double amount_tie = -0.5 * rake / num_combinations;
    const auto& same = same_hand_index[player];
    const auto& hs = hand_strength[card_pair_to_index(node.turn, node.river)];
    const auto& ps = hs[player];
    const auto& os = hs[player ^ 1];
    for (size_t k = 1; k + 1 < os.size(); ++k) {
      size_t idx = os[k].index;
      F r = cfreach[idx];
      if (r != (F)0) {
        double rd = (double)r;
        cfreach_sum += rd;
        cfreach_minus[ocards[idx].first] += rd;
        cfreach_minus[ocards[idx].second] += rd;
      }
    }
    if (cfreach_sum == 0.0) return;
    double sum_win = 0.0, sum_tie = 0.0, minus_win[52], minus_tie[52];
    for (int c = 0; c < 52; ++c) minus_win[c] = minus_tie[c] = 0.0;
    size_t i = 1, j = 1;
    uint16_t prev_strength = 0;
    for (size_t k = 1; k + 1 < ps.size(); ++k) {
      uint16_t strength = ps[k].strength, index = ps[k].index;
      if (strength > prev_strength) {
        prev_strength = strength;
        if (i < j) {
          sum_win = sum_tie;
          std::memcpy(minus_win, minus_tie, sizeof minus_win);
          i = j;
        }
        while (os[i].strength < strength) {
          size_t oi = os[i].index;
          double r = (double)cfreach[oi];
          sum_win += r;
          minus_win[ocards[oi].first] += r;
          minus_win[ocards[oi].second] += r;
          ++i;
        }
        if (j < i) {
          sum_tie = sum_win;
          std::memcpy(minus_tie, minus_win, sizeof minus_tie);
          j = i;
        }
        while (os[j].strength == strength) {
          size_t oi = os[j].index;
          double r = (double)cfreach[oi];
          sum_tie += r;
          minus_tie[ocards[oi].first] += r;
          minus_tie[ocards[oi].second] += r;
          ++j;
        }
      }
      int c1 = pcards[index].first, c2 = pcards[index].second;
      double total = cfreach_sum - cfreach_minus[c1] - cfreach_minus[c2];
      double win = sum_win - minus_win[c1] - minus_win[c2];
      double tie = sum_tie - minus_tie[c1] - minus_tie[c2];
      double cs = same[index] == 0xFFFF ? 0.0 : (double)cfreach[same[index]];
      double v = amount_win * win + amount_tie * (tie - win + cs) + amount_lose * (total - tie);
      result[index] = (F)v;
    }
  }
}

// evaluation.rs:544-605
template <class F>
void Game<F>::evaluate_boundary_single(F* result, const Node& node, int player, const F* cfreach,
                                       const std::vector<F>& bcfvs, double half_pot) {
  double payoff_scale = half_pot / num_combinations;
  const auto& vi = valid_indices_for(node);
  const auto& pcards = private_cards[player];
  const auto& ocards = private_cards[player ^ 1];
  double sum = 0.0, minus[52];
  for (int c = 0; c < 52; ++c) minus[c] = 0.0;
  for (uint16_t i : vi[player ^ 1]) {
    F r = cfreach[i];
    if (r != (F)0) {
      double rd = (double)r;
      sum += rd;
      minus[ocards[i].first] += rd;
      minus[ocards[i].second] += rd;
    }
  }
  if (sum == 0.0) return;
  const auto& same = same_hand_index[player];
  for (uint16_t i : vi[player]) {
    double cs = same[i] == 0xFFFF ? 0.0 : (double)cfreach[same[i]];
    double adj = sum + cs - minus[pcards[i].first] - minus[pcards[i].second];
    double b = (double)bcfvs[i];
    result[i] = (F)(b * payoff_scale * adj);
  }
}

// ---------------------------------------------------------------------------
// solver.rs / sliceop.rs / utility.rs
// ---------------------------------------------------------------------------

template <class F>
static inline F fmax_ref(F x, F y) {  // sliceop.rs:5-12
  return x > y ? x : y;
}

template <class F>
static inline bool sign_positive(F x) {
  return !std::signbit(x);
}

// solver.rs:600-626 with div_slice (sliceop.rs:35-39)
template <class F>
static void regret_matching(const F* regret, size_t na, size_t nh, std::vector<F>& strategy) {
  strategy.resize(na * nh);
  for (size_t k = 0; k < na * nh; ++k) strategy[k] = fmax_ref<F>(regret[k], (F)0);
  std::vector<F> denom(strategy.begin(), strategy.begin() + nh);
  for (size_t a = 1; a < na; ++a)
    for (size_t h = 0; h < nh; ++h) denom[h] += strategy[a * nh + h];
  F def = (F)1 / (F)na;
  for (size_t a = 0; a < na; ++a)
    for (size_t h = 0; h < nh; ++h) {
      F& s = strategy[a * nh + h];
      s = denom[h] == (F)0 ? def : s / denom[h];
    }
}

// utility.rs:227-250
template <class F>
static void normalized_strategy(const F* s, size_t na, size_t nh, std::vector<F>& out) {
  out.resize(na * nh);
  std::vector<F> denom(s, s + nh);
  for (size_t a = 1; a < na; ++a)
    for (size_t h = 0; h < nh; ++h) denom[h] += s[a * nh + h];
  F def = (F)1 / (F)na;
  for (size_t a = 0; a < na; ++a)
    for (size_t h = 0; h < nh; ++h) out[a * nh + h] = denom[h] == (F)0 ? def : s[a * nh + h] / denom[h];
}

// utility.rs:334-343
template <class F>
static void apply_locking_strategy(std::vector<F>& dst, const std::vector<F>* locking) {
  if (!locking) return;
  for (size_t k = 0; k < dst.size(); ++k)
    if (sign_positive((*locking)[k])) dst[k] = (*locking)[k];
}

template <class F>
static void apply_swap_list(F* v, const std::vector<std::pair<uint16_t, uint16_t>>& sl) {
  for (auto [i, j] : sl) std::swap(v[i], v[j]);
}

// Chance children evaluated in parallel on a persistent pool, as the
// reference's solve_recursive does with rayon (solver.rs:264-326 over
// for_each_child): children write disjoint slices and are summed in child
// order afterwards, so the results do not depend on the thread count.
// Nested calls from a worker run inline.
namespace {
struct ChancePool {
  std::mutex m, run_mu;
  std::condition_variable cv, done;
  std::vector<std::thread> workers;
  const std::function<void(size_t)>* job = nullptr;
  size_t count = 0;
  std::atomic<size_t> next{0};
  size_t finished = 0;  // workers that have checked in for the current job
  uint64_t gen = 0;
  bool stop = false;
  static thread_local bool in_worker;

  void resize(int n) {
    shutdown();
    stop = false;
    for (int i = 0; i + 1 < n; ++i) workers.emplace_back([this] { loop(); });
  }
  void shutdown() {
    {
      std::lock_guard<std::mutex> lk(m);
      stop = true;
    }
    cv.notify_all();
    for (auto& t : workers) t.join();
    workers.clear();
  }
  // every worker takes part in every job and checks in when done, so no
  // worker can still hold a job when the next one starts
  void loop() {
    in_worker = true;
    uint64_t seen = 0;
    for (;;) {
      const std::function<void(size_t)>* f;
      size_t n;
      {
        std::unique_lock<std::mutex> lk(m);
        cv.wait(lk, [&] { return stop || gen != seen; });
        if (stop) return;
        seen = gen;
        f = job;
        n = count;
      }
      for (size_t i; (i = next.fetch_add(1)) < n;) (*f)(i);
      {
        std::lock_guard<std::mutex> lk(m);
        ++finished;
      }
      done.notify_all();
    }
  }
  void parallel_for(size_t n, const std::function<void(size_t)>& f) {
    if (workers.empty() || in_worker || n < 2) {
      for (size_t i = 0; i < n; ++i) f(i);
      return;
    }
    std::lock_guard<std::mutex> outer(run_mu);
    {
      std::lock_guard<std::mutex> lk(m);
      job = &f;
      count = n;
      next = 0;
      finished = 0;
      ++gen;
    }
    cv.notify_all();
    in_worker = true;
    for (size_t i; (i = next.fetch_add(1)) < n;) f(i);
    in_worker = false;
    std::unique_lock<std::mutex> lk(m);
    done.wait(lk, [&] { return finished == workers.size(); });
  }
  ~ChancePool() { shutdown(); }
};
thread_local bool ChancePool::in_worker = false;
ChancePool g_chance_pool;
}  // namespace

void set_chance_threads(int n) { g_chance_pool.resize(n < 1 ? 1 : n); }

// solver.rs:221-479
template <class F>
void Game<F>::solve_recursive(F* result, Node* node, int player, const F* cfreach,
                              const DiscountParams& params) {
  if (node->is_terminal()) {
    evaluate(result, *node, player, cfreach);
    return;
  }
  size_t na = node->num_children;
  size_t nh = num_private_hands(player);
  if (na == 1 && !node->is_chance()) {
    solve_recursive(result, child(node, 0), player, cfreach, params);
    return;
  }
  std::vector<F> cfv(na * nh);
  if (node->is_chance()) {  // solver.rs:264-326
    size_t no = num_private_hands(player ^ 1);
    std::vector<F> upd(no);
    F scalar = (F)1 / (F)chance_factor(*node);
    for (size_t i = 0; i < no; ++i) upd[i] = cfreach[i] * scalar;
    const std::function<void(size_t)> one = [&](size_t a) {
      solve_recursive(&cfv[a * nh], child(node, a), player, upd.data(), params);
    };
    g_chance_pool.parallel_for(na, one);
    std::vector<double> acc(nh);
    for (size_t h = 0; h < nh; ++h) acc[h] = (double)cfv[h];
    for (size_t a = 1; a < na; ++a)
      for (size_t h = 0; h < nh; ++h) acc[h] += (double)cfv[a * nh + h];
    const auto& iso = isomorphic_chances(*node);
    for (size_t i = 0; i < iso.size(); ++i) {
      const auto& sl = isomorphic_swap(*node, i)[player];
      F* tmp = &cfv[iso[i] * nh];
      apply_swap_list(tmp, sl);
      for (size_t h = 0; h < nh; ++h) acc[h] += (double)tmp[h];
      apply_swap_list(tmp, sl);
    }
    for (size_t h = 0; h < nh; ++h) result[h] = (F)acc[h];
  } else if (node->player == player) {  // solver.rs:333-416
    for (size_t a = 0; a < na; ++a) solve_recursive(&cfv[a * nh], child(node, a), player, cfreach, params);
    std::vector<F> strategy;
    F* R = &storage2[node->s2];
    F* S = &storage1[node->s1];
    regret_matching(R, na, nh, strategy);
    apply_locking_strategy(strategy, locking(*node));
    for (size_t h = 0; h < nh; ++h) result[h] = strategy[h] * cfv[h];
    for (size_t a = 1; a < na; ++a)
      for (size_t h = 0; h < nh; ++h) result[h] += strategy[a * nh + h] * cfv[a * nh + h];
    // solver.rs:556-567
    for (size_t k = 0; k < na * nh; ++k) S[k] = S[k] * params.gamma_t + strategy[k];
    // solver.rs:570-589
    for (size_t k = 0; k < na * nh; ++k) {
      F coef = sign_positive(R[k]) ? (F)params.alpha_t : (F)params.beta_t;
      R[k] = R[k] * coef + cfv[k];
    }
    for (size_t a = 0; a < na; ++a)
      for (size_t h = 0; h < nh; ++h) R[a * nh + h] -= result[h];
  } else {  // solver.rs:418-478
    size_t no = num_private_hands(player ^ 1);
    std::vector<F> strategy;
    regret_matching(&storage2[node->s2], na, no, strategy);
    apply_locking_strategy(strategy, locking(*node));
    for (size_t a = 0; a < na; ++a)
      for (size_t i = 0; i < no; ++i) strategy[a * no + i] *= cfreach[i];
    for (size_t a = 0; a < na; ++a)
      solve_recursive(&cfv[a * nh], child(node, a), player, &strategy[a * no], params);
    for (size_t h = 0; h < nh; ++h) result[h] = cfv[h];
    for (size_t a = 1; a < na; ++a)
      for (size_t h = 0; h < nh; ++h) result[h] += cfv[a * nh + h];
  }
}

// solver.rs:184-209
template <class F>
void Game<F>::solve_step(uint32_t t) {
  if (is_solved()) throw std::runtime_error("Game is already solved");
  if (!is_ready()) throw std::runtime_error("Game is not ready");
  DiscountParams params(t);
  for (int p = 0; p < 2; ++p) {
    std::vector<F> result(num_private_hands(p));
    solve_recursive(result.data(), &arena[0], p, initial_weights[p ^ 1].data(), params);
  }
}

// one player's traversal of solve_step (solver.rs:197-208), for per-pass checks
template <class F>
void Game<F>::solve_pass(uint32_t t, int p) {
  if (!is_ready()) throw std::runtime_error("Game is not ready");
  DiscountParams params(t);
  std::vector<F> result(num_private_hands(p));
  solve_recursive(result.data(), &arena[0], p, initial_weights[p ^ 1].data(), params);
}

// solver.rs:108-176
template <class F>
float Game<F>::solve(uint32_t max_iter, float target, bool print, uint32_t* iters_run) {
  if (is_solved()) throw std::runtime_error("Game is already solved");
  if (!is_ready()) throw std::runtime_error("Game is not ready");
  float expl = compute_exploitability();
  if (print) printf("iteration: 0 / %u (exploitability = %.4e)", max_iter, expl);
  uint32_t t = 0;
  for (; t < max_iter; ++t) {
    if (expl <= target) break;
    DiscountParams params(t);
    for (int p = 0; p < 2; ++p) {
      std::vector<F> result(num_private_hands(p));
      solve_recursive(result.data(), &arena[0], p, initial_weights[p ^ 1].data(), params);
    }
    if ((t + 1) % 5 == 0 || t + 1 == max_iter) expl = compute_exploitability();
    if (print) printf("\riteration: %u / %u (exploitability = %.4e)", t + 1, max_iter, expl);
  }
  if (print) printf("\n");
  if (iters_run) *iters_run = t;
  finalize();
  return expl;
}

// utility.rs:552-795
template <class F>
void Game<F>::compute_cfvalue_recursive(F* result, Node* node, int player, const F* cfreach, bool save) {
  if (node->is_terminal()) {
    evaluate(result, *node, player, cfreach);
    return;
  }
  size_t na = node->num_children;
  size_t nh = num_private_hands(player);
  if (!node->is_chance() && node->player != player && na == 1) {
    compute_cfvalue_recursive(result, child(node, 0), player, cfreach, save);
    return;
  }
  std::vector<F> cfv(na * nh);
  if (node->is_chance()) {
    size_t no = num_private_hands(player ^ 1);
    std::vector<F> upd(no);
    F scalar = (F)1 / (F)chance_factor(*node);
    for (size_t i = 0; i < no; ++i) upd[i] = cfreach[i] * scalar;
    // chance children in parallel (utility.rs:682 for_each_child), summed in child order below
    const std::function<void(size_t)> one = [&](size_t a) {
      compute_cfvalue_recursive(&cfv[a * nh], child(node, a), player, upd.data(), save);
    };
    g_chance_pool.parallel_for(na, one);
    std::vector<double> acc(nh);
    for (size_t h = 0; h < nh; ++h) acc[h] = (double)cfv[h];
    for (size_t a = 1; a < na; ++a)
      for (size_t h = 0; h < nh; ++h) acc[h] += (double)cfv[a * nh + h];
    const auto& iso = isomorphic_chances(*node);
    for (size_t i = 0; i < iso.size(); ++i) {
      const auto& sl = isomorphic_swap(*node, i)[player];
      F* tmp = &cfv[iso[i] * nh];
      apply_swap_list(tmp, sl);
      for (size_t h = 0; h < nh; ++h) acc[h] += (double)tmp[h];
      apply_swap_list(tmp, sl);
    }
    for (size_t h = 0; h < nh; ++h) result[h] = (F)acc[h];
    if (save && node->cfvalue_storage_player() == player)
      std::copy(result, result + nh, &storage_chance[node->s1]);
  } else if (node->player == player) {
    for (size_t a = 0; a < na; ++a) compute_cfvalue_recursive(&cfv[a * nh], child(node, a), player, cfreach, save);
    std::vector<F> strategy;
    normalized_strategy(&storage1[node->s1], na, nh, strategy);
    apply_locking_strategy(strategy, locking(*node));
    for (size_t h = 0; h < nh; ++h) result[h] = strategy[h] * cfv[h];
    for (size_t a = 1; a < na; ++a)
      for (size_t h = 0; h < nh; ++h) result[h] += strategy[a * nh + h] * cfv[a * nh + h];
    if (save) std::copy(cfv.begin(), cfv.end(), &storage2[node->s2]);
  } else {
    size_t no = num_private_hands(player ^ 1);
    std::vector<F> strategy;
    normalized_strategy(&storage1[node->s1], na, no, strategy);
    apply_locking_strategy(strategy, locking(*node));
    for (size_t a = 0; a < na; ++a)
      for (size_t i = 0; i < no; ++i) strategy[a * no + i] *= cfreach[i];
    for (size_t a = 0; a < na; ++a)
      compute_cfvalue_recursive(&cfv[a * nh], child(node, a), player, &strategy[a * no], save);
    for (size_t h = 0; h < nh; ++h) result[h] = cfv[h];
    for (size_t a = 1; a < na; ++a)
      for (size_t h = 0; h < nh; ++h) result[h] += cfv[a * nh + h];
  }
  if (save && node->num_elements_ip != 0 && player == 1)
    std::copy(result, result + nh, &storage_ip[node->s3]);
}

// utility.rs:804-988
template <class F>
void Game<F>::compute_best_cfv_recursive(F* result, Node* node, int player, const F* cfreach) {
  if (node->is_terminal()) {
    evaluate(result, *node, player, cfreach);
    return;
  }
  size_t na = node->num_children;
  size_t nh = num_private_hands(player);
  if (na == 1 && !node->is_chance()) {
    compute_best_cfv_recursive(result, child(node, 0), player, cfreach);
    return;
  }
  std::vector<F> cfv(na * nh);
  if (node->is_chance()) {
    size_t no = num_private_hands(player ^ 1);
    std::vector<F> upd(no);
    F scalar = (F)1 / (F)chance_factor(*node);
    for (size_t i = 0; i < no; ++i) upd[i] = cfreach[i] * scalar;
    // chance children in parallel (utility.rs:852 for_each_child), summed in child order below
    const std::function<void(size_t)> one = [&](size_t a) {
      compute_best_cfv_recursive(&cfv[a * nh], child(node, a), player, upd.data());
    };
    g_chance_pool.parallel_for(na, one);
    std::vector<double> acc(nh);
    for (size_t h = 0; h < nh; ++h) acc[h] = (double)cfv[h];
    for (size_t a = 1; a < na; ++a)
      for (size_t h = 0; h < nh; ++h) acc[h] += (double)cfv[a * nh + h];
    const auto& iso = isomorphic_chances(*node);
    for (size_t i = 0; i < iso.size(); ++i) {
      const auto& sl = isomorphic_swap(*node, i)[player];
      F* tmp = &cfv[iso[i] * nh];
      apply_swap_list(tmp, sl);
      for (size_t h = 0; h < nh; ++h) acc[h] += (double)tmp[h];
      apply_swap_list(tmp, sl);
    }
    for (size_t h = 0; h < nh; ++h) result[h] = (F)acc[h];
  } else if (node->player == player) {
    for (size_t a = 0; a < na; ++a) compute_best_cfv_recursive(&cfv[a * nh], child(node, a), player, cfreach);
    const auto* lk = locking(*node);
    if (!lk) {  // sliceop.rs:128-145
      for (size_t h = 0; h < nh; ++h) result[h] = cfv[h];
      for (size_t a = 1; a < na; ++a)
        for (size_t h = 0; h < nh; ++h) result[h] = fmax_ref<F>(result[h], cfv[a * nh + h]);
    } else {  // sliceop.rs:147-180
      const auto& L = *lk;
      for (size_t h = 0; h < nh; ++h) result[h] = sign_positive(L[h]) ? cfv[h] * L[h] : cfv[h];
      for (size_t a = 1; a < na; ++a)
        for (size_t h = 0; h < nh; ++h) {
          F s2 = L[a * nh + h], s1 = cfv[a * nh + h];
          if (sign_positive(s2)) result[h] += s1 * s2;
          else result[h] = fmax_ref<F>(result[h], s1);
        }
    }
  } else {
    size_t no = num_private_hands(player ^ 1);
    std::vector<F> strategy;
    normalized_strategy(&storage1[node->s1], na, no, strategy);
    apply_locking_strategy(strategy, locking(*node));
    for (size_t a = 0; a < na; ++a)
      for (size_t i = 0; i < no; ++i) strategy[a * no + i] *= cfreach[i];
    for (size_t a = 0; a < na; ++a)
      compute_best_cfv_recursive(&cfv[a * nh], child(node, a), player, &strategy[a * no]);
    for (size_t h = 0; h < nh; ++h) result[h] = cfv[h];
    for (size_t a = 1; a < na; ++a)
      for (size_t h = 0; h < nh; ++h) result[h] += cfv[a * nh + h];
  }
}

// utility.rs:118-122
template <class F>
static float weighted_sum(const std::vector<F>& v, const std::vector<F>& w) {
  double s = 0.0;
  for (size_t i = 0; i < v.size(); ++i) s = s + (double)v[i] * (double)w[i];
  return (float)s;
}

// utility.rs:501-543
template <class F>
std::array<float, 2> Game<F>::compute_mes_ev() {
  std::array<float, 2> ev;
  for (int p = 0; p < 2; ++p) {
    std::vector<F> cfv(num_private_hands(p));
    compute_best_cfv_recursive(cfv.data(), &arena[0], p, initial_weights[p ^ 1].data());
    ev[p] = weighted_sum(cfv, initial_weights[p]);
  }
  return ev;
}

// utility.rs:450-495
template <class F>
std::array<float, 2> Game<F>::compute_current_ev() {
  std::array<float, 2> ev;
  for (int p = 0; p < 2; ++p) {
    std::vector<F> cfv(num_private_hands(p));
    compute_cfvalue_recursive(cfv.data(), &arena[0], p, initial_weights[p ^ 1].data(), false);
    ev[p] = weighted_sum(cfv, initial_weights[p]);
  }
  return ev;
}

// utility.rs:380-392
template <class F>
float Game<F>::compute_exploitability() {
  if (!is_ready() && !is_solved()) throw std::runtime_error("Game is not ready");
  auto mes = compute_mes_ev();
  if (!is_raked()) return (mes[0] + mes[1]) * 0.5f;
  auto cur = compute_current_ev();
  return ((mes[0] - cur[0]) + (mes[1] - cur[1])) * 0.5f;
}

// utility.rs:348-372
template <class F>
void Game<F>::finalize() {
  if (is_solved()) throw std::runtime_error("Game is already solved");
  if (!is_ready()) throw std::runtime_error("Game is not ready");
  for (int p = 0; p < 2; ++p) {
    std::vector<F> cfv(num_private_hands(p));
    compute_cfvalue_recursive(cfv.data(), &arena[0], p, initial_weights[p ^ 1].data(), true);
  }
  state = State::Solved;  // interpreter.rs:67-71 (set_solved re-applies the history)
  auto h = action_history;
  back_to_root();
  for (size_t a : h) play(a);
}

// utility.rs:422-443
template <class F>
std::vector<F> Game<F>::root_cfvalues_with_reach(int player, const F* opp_reach) {
  if (!is_ready() && !is_solved()) throw std::runtime_error("Game is not ready");
  std::vector<F> out(num_private_hands(player));
  compute_cfvalue_recursive(out.data(), &arena[0], player, opp_reach, false);
  return out;
}

// ---------------------------------------------------------------------------
// game/query.rs
// ---------------------------------------------------------------------------

template <class F>
void Game<F>::back_to_root() {  // query.rs:24-42
  action_history.clear();
  node_history.clear();
  is_normalized_weight_cached = false;
  turn = card_config.turn;
  river = card_config.river;
  turn_swapped_suit[0] = turn_swapped_suit[1] = -1;
  turn_swap = -1;
  river_swap[0] = river_swap[1] = -1;
  total_bet_amount[0] = total_bet_amount[1] = 0;
  for (int p = 0; p < 2; ++p) weights[p] = initial_weights[p];
  assign_zero_weights();
}

template <class F>
bool Game<F>::is_terminal_node() {  // query.rs:67-73
  Node* n = cur_node();
  return n->is_terminal() || n->amount == tree_config.effective_stack;
}

template <class F>
bool Game<F>::is_chance_node() {
  return cur_node()->is_chance() && !is_terminal_node();
}

template <class F>
std::vector<Action> Game<F>::available_actions() {  // query.rs:85-98
  std::vector<Action> out;
  if (is_terminal_node()) return out;
  Node* n = cur_node();
  for (int a = 0; a < n->num_children; ++a) out.push_back(child(n, a)->prev_action);
  return out;
}

template <class F>
uint64_t Game<F>::possible_cards() {  // query.rs:100-136
  if (!is_chance_node()) return 0;
  const auto& c = card_config;
  uint64_t board = (1ull << c.flop[0]) | (1ull << c.flop[1]) | (1ull << c.flop[2]);
  uint64_t dead = 0;
  if (turn != NOT_DEALT) board |= 1ull << turn;
  for (int card = 0; card < 52; ++card) {
    uint64_t bit = 1ull << card;
    uint64_t nb = board | bit;
    bool alive = false;
    if (nb != board) {
      for (const auto& o : private_cards[0]) {
        uint64_t om = (1ull << o.first) | (1ull << o.second);
        if (om & nb) continue;
        uint64_t cm = om | nb;
        for (const auto& i : private_cards[1]) {
          uint64_t im = (1ull << i.first) | (1ull << i.second);
          if ((im & cm) == 0) { alive = true; break; }
        }
        if (alive) break;
      }
    }
    if (!alive) dead |= bit;
  }
  return ((1ull << 52) - 1) ^ dead;
}

template <class F>
void Game<F>::apply_swap(F* slice, int player, bool reverse) {  // query.rs:863-883
  const std::vector<std::pair<uint16_t, uint16_t>>* ts =
      turn_swap >= 0 ? &isomorphism_swap_turn[turn_swap][player] : nullptr;
  const std::vector<std::pair<uint16_t, uint16_t>>* rs =
      river_swap[0] >= 0 ? &isomorphism_swap_river[river_swap[0]][river_swap[1]][player] : nullptr;
  const std::vector<std::pair<uint16_t, uint16_t>>* order[2] = {ts, rs};
  if (reverse) std::swap(order[0], order[1]);
  for (auto* s : order)
    if (s) apply_swap_list(slice, *s);
}

template <class F>
void Game<F>::assign_zero_weights() {  // query.rs:886-920
  uint64_t board = 0;
  if (turn != NOT_DEALT) board |= 1ull << turn;
  if (river != NOT_DEALT) board |= 1ull << river;
  for (int p = 0; p < 2; ++p) {
    uint64_t dead = (1ull << 52) - 1;
    for (const auto& o : private_cards[p ^ 1]) {
      uint64_t m = (1ull << o.first) | (1ull << o.second);
      if ((m & board) == 0) dead &= m;
      if (dead == 0) break;
    }
    dead |= board;
    for (size_t i = 0; i < private_cards[p].size(); ++i) {
      uint64_t m = (1ull << private_cards[p][i].first) | (1ull << private_cards[p][i].second);
      if (m & dead) weights[p][i] = (F)0;
    }
  }
}

template <class F>
void Game<F>::play(size_t action) {  // query.rs:186-335
  if (state < State::MemoryAllocated) throw std::runtime_error("Memory is not allocated");
  if (is_terminal_node()) throw std::runtime_error("Terminal node is not allowed");
  if (is_chance_node()) {
    bool is_turn = turn == NOT_DEALT;
    int actual = action == (size_t)-1 ? __builtin_ctzll(possible_cards()) : (int)action;
    int action_card = actual;
    if (turn_swapped_suit[0] >= 0) {
      int s1 = turn_swapped_suit[0], s2 = turn_swapped_suit[1];
      if ((actual & 3) == s1) action_card = actual - s1 + s2;
      else if ((actual & 3) == s2) action_card = actual + s1 - s2;
    }
    auto acts = available_actions();
    size_t ai = (size_t)-1;
    for (size_t i = 0; i < acts.size(); ++i)
      if (acts[i].kind == A_Chance && acts[i].amount == action_card) { ai = i; break; }
    if (ai == (size_t)-1) {
      Node* n = cur_node();
      const auto& iso = isomorphic_chances(*n);
      const auto& icards = n->turn == NOT_DEALT ? isomorphism_card_turn : isomorphism_card_river[n->turn & 3];
      for (size_t i = 0; i < iso.size(); ++i)
        if (action_card == icards[i]) {
          ai = iso[i];
          if (is_turn) {
            turn_swapped_suit[0] = action_card & 3;
            turn_swapped_suit[1] = acts[ai].amount & 3;
            turn_swap = action_card & 3;
          } else {
            river_swap[0] = turn & 3;
            river_swap[1] = isomorphism_card_river[turn & 3][i] & 3;
          }
          break;
        }
    }
    if (ai == (size_t)-1) throw std::runtime_error("Invalid action");
    Node* n = cur_node();
    node_history.push_back(node_index(child(n, ai)));
    if (is_turn) turn = (Card)actual;
    else river = (Card)actual;
    assign_zero_weights();
  } else {
    Node* n = cur_node();
    if (action >= n->num_children) throw std::runtime_error("Invalid action");
    int player = n->player;
    size_t nh = num_private_hands(player);
    if (n->num_children > 1) {
      auto st = strategy();
      for (size_t h = 0; h < nh; ++h) weights[player][h] *= st[action * nh + h];
    }
    for (size_t h = 0; h < nh; ++h) cfvalues_cache[player][h] = storage2[n->s2 + action * nh + h];
    Action pa = child(n, action)->prev_action;
    if (pa.kind == A_Call) {
      total_bet_amount[player] = total_bet_amount[player ^ 1];
    } else if (pa.kind == A_Bet || pa.kind == A_Raise || pa.kind == A_AllIn) {
      int32_t prev_bet = (n->prev_action.kind == A_Bet || n->prev_action.kind == A_Raise ||
                          n->prev_action.kind == A_AllIn)
                             ? n->prev_action.amount
                             : 0;
      int32_t to_call = total_bet_amount[player ^ 1] - total_bet_amount[player];
      total_bet_amount[player] += pa.amount - prev_bet + to_call;
    }
    node_history.push_back(node_index(child(n, action)));
  }
  action_history.push_back(action);
  is_normalized_weight_cached = false;
}

template <class F>
std::vector<F> Game<F>::strategy() {  // query.rs:346-378
  Node* n = cur_node();
  int player = n->player;
  size_t na = n->num_children, nh = num_private_hands(player);
  std::vector<F> ret;
  normalized_strategy(&storage1[n->s1], na, nh, ret);
  apply_locking_strategy(ret, locking(*n));
  for (size_t a = 0; a < na; ++a) apply_swap(&ret[a * nh], player, false);
  return ret;
}

template <class F>
std::vector<F> Game<F>::strategy_at_index(size_t idx) {  // query.rs:386-402
  Node* n = &arena[idx];
  if (n->is_terminal() || n->is_chance()) throw std::runtime_error("strategy_at_index requires a decision node");
  std::vector<F> ret;
  normalized_strategy(&storage1[n->s1], n->num_children, num_private_hands(n->player), ret);
  return ret;
}

template <class F>
void Game<F>::cache_normalized_weights() {  // query.rs:498-567
  if (is_normalized_weight_cached) return;
  uint64_t board = 0;
  if (turn != NOT_DEALT) board |= 1ull << turn;
  if (river != NOT_DEALT) board |= 1ull << river;
  double ws[2] = {0, 0}, wsm[2][52];
  for (int p = 0; p < 2; ++p) {
    for (int c = 0; c < 52; ++c) wsm[p][c] = 0.0;
    for (size_t i = 0; i < private_cards[p].size(); ++i) {
      auto [c1, c2] = private_cards[p][i];
      uint64_t m = (1ull << c1) | (1ull << c2);
      if ((m & board) == 0) {
        double w = (double)weights[p][i];
        ws[p] += w;
        wsm[p][c1] += w;
        wsm[p][c2] += w;
      }
    }
  }
  for (int p = 0; p < 2; ++p) {
    for (size_t i = 0; i < private_cards[p].size(); ++i) {
      auto [c1, c2] = private_cards[p][i];
      uint64_t m = (1ull << c1) | (1ull << c2);
      if ((m & board) == 0) {
        uint16_t si = same_hand_index[p][i];
        double ows = si == 0xFFFF ? 0.0 : (double)weights[p ^ 1][si];
        double ow = ws[p ^ 1] + ows - wsm[p ^ 1][c1] - wsm[p ^ 1][c2];
        normalized_weights[p][i] = weights[p][i] * (F)ow;
      } else {
        normalized_weights[p][i] = (F)0;
      }
    }
  }
  is_normalized_weight_cached = true;
}

template <class F>
std::vector<F> Game<F>::expected_values_detail(int player) {  // query.rs:699-760
  if (state != State::Solved) throw std::runtime_error("Game is not solved");
  if (!is_normalized_weight_cached) throw std::runtime_error("Normalized weights are not cached");
  Node* node = cur_node();
  size_t nh = num_private_hands(player);
  size_t cf = 1;
  if (card_config.turn == NOT_DEALT && turn != NOT_DEALT) cf *= 45;
  if (card_config.river == NOT_DEALT && river != NOT_DEALT) cf *= 44;
  bool have_actions = false;
  F normalizer = (F)(num_combinations * (double)cf);
  std::vector<F> ret;
  if (node->is_terminal()) {
    normalizer = (F)num_combinations;
    ret.assign(nh, (F)0);
    std::vector<F> cr = weights[player ^ 1];
    evaluate(ret.data(), *node, player, cr.data());
  } else if (node->is_chance() && node->cfvalue_storage_player() == player) {
    ret.assign(&storage_chance[node->s1], &storage_chance[node->s1] + node->num_elements);
  } else if (node->num_elements_ip != 0 && player == PLAYER_IP) {
    ret.assign(&storage_ip[node->s3], &storage_ip[node->s3] + node->num_elements_ip);
  } else if (player == current_player()) {
    have_actions = true;
    ret.assign(&storage2[node->s2], &storage2[node->s2] + node->num_elements);
  } else {
    ret = cfvalues_cache[player];
  }
  int32_t bias = std::max(total_bet_amount[player] - total_bet_amount[player ^ 1], 0);
  for (size_t a = 0; a * nh < ret.size(); ++a) {
    bool is_fold = have_actions && child(node, (int)a)->prev_action.kind == A_Fold;
    apply_swap(&ret[a * nh], player, false);
    for (size_t h = 0; h < nh; ++h) {
      F& v = ret[a * nh + h];
      F wr = weights[player][h], wn = normalized_weights[player][h];
      if (is_fold || wn == (F)0) {
        v = (F)0;
      } else {
        v *= normalizer * (wr / wn);
        v += (F)tree_config.starting_pot * (F)0.5 + (F)(node->amount + bias);
      }
    }
  }
  return ret;
}

template <class F>
std::vector<F> Game<F>::expected_values(int player) {  // query.rs:639-681
  auto detail = expected_values_detail(player);
  if (is_terminal_node() || is_chance_node() || current_player() != player) return detail;
  Node* n = cur_node();
  size_t na = n->num_children, nh = num_private_hands(player);
  auto st = strategy();
  std::vector<F> ret(nh);
  for (size_t i = 0; i < nh; ++i) {
    F ev = (F)0;
    for (size_t j = 0; j < na; ++j) ev += detail[i + j * nh] * st[i + j * nh];
    ret[i] = ev;
  }
  return ret;
}

template <class F>
void Game<F>::lock_current_strategy(const F* strategy_in) {  // query.rs:772-822
  Node* n = cur_node();
  int player = n->player;
  size_t na = n->num_children, nh = num_private_hands(player);
  std::vector<F> lk(na * nh, (F)-1);
  for (size_t h = 0; h < nh; ++h) {
    double sum = 0.0;
    bool lock = false;
    for (size_t a = 0; a < na; ++a) {
      F f = strategy_in[a * nh + h];
      if (f > (F)0) {
        sum += (double)f;
        lock = true;
      }
    }
    if (lock)
      for (size_t a = 0; a < na; ++a) {
        double f = (double)std::max(strategy_in[a * nh + h], (F)0);
        lk[a * nh + h] = (F)(f / sum);
      }
  }
  for (size_t a = 0; a < na; ++a) apply_swap(&lk[a * nh], player, true);
  n->is_locked = true;
  locking_strategy[node_index(n)] = lk;
}

template struct Game<float>;
template struct Game<double>;

}  // namespace oracle
