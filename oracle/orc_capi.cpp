// ORACLE — test infrastructure only.  extern "C" surface of the CPU
// restatement so pytest (ctypes) can drive it as the checker and bench.py can
// time it as the CPU baseline.  Every array crossing this boundary is float32
// in, float64 out (the FP64 oracle build writes its native precision).
#include <cstring>
#include <stdexcept>
#include <string>

#include "rs_oracle.hpp"

using namespace oracle;

namespace {
thread_local std::string g_err;

struct OrcGame {
  int fp64 = 0;
  Game<float>* g32 = nullptr;
  Game<double>* g64 = nullptr;
};

#define ORC_TRY(body)          \
  try {                        \
    body                       \
  } catch (const std::exception& e) { \
    g_err = e.what();          \
    return -1;                 \
  }

template <class Fn>
auto with(OrcGame* h, Fn&& fn) {
  if (h->fp64) return fn(*h->g64);
  return fn(*h->g32);
}

template <class V>
void to_f64(const V& v, double* out) {
  for (size_t i = 0; i < v.size(); ++i) out[i] = (double)v[i];
}
}  // namespace

extern "C" {

struct OrcTreeConfig {
  int32_t initial_state, starting_pot, effective_stack, depth_limit;
  double rake_rate, rake_cap, add_allin_threshold, force_allin_threshold, merging_threshold;
  const char* sizes[12];  // [street(flop,turn,river)][player][bet,raise]
  const char* donk[2];    // turn, river; NULL = None
};

const char* orc_last_error() { return g_err.c_str(); }

void orc_set_hand_table_path(const char* p) { set_hand_table_path(p); }
void orc_set_chance_threads(int n) { set_chance_threads(n); }

int orc_hand_table_exhaustive(int32_t* table_out, int cap, uint64_t* counts9) {
  std::vector<int32_t> t;
  hand_table_exhaustive(t, counts9);
  for (size_t i = 0; i < t.size() && (int)i < cap; ++i) table_out[i] = t[i];
  return (int)t.size();
}

int orc_hand_table(int32_t* out, int cap) {
  const auto& t = hand_table();
  for (size_t i = 0; i < t.size() && (int)i < cap; ++i) out[i] = t[i];
  return (int)t.size();
}

int32_t orc_hand_evaluate_internal(const int32_t* cards7) { return hand_evaluate_internal(cards7); }
int32_t orc_hand_evaluate(const int32_t* cards7) { return hand_evaluate(cards7); }

void orc_discount_params(uint32_t t, float* out3) {
  DiscountParams p(t);
  out3[0] = p.alpha_t;
  out3[1] = p.beta_t;
  out3[2] = p.gamma_t;
}

static bool build_tree_config(const OrcTreeConfig* c, TreeConfig& tc, std::string& err) {
  tc.initial_state = (BoardState)c->initial_state;
  tc.starting_pot = c->starting_pot;
  tc.effective_stack = c->effective_stack;
  tc.rake_rate = c->rake_rate;
  tc.rake_cap = c->rake_cap;
  tc.add_allin_threshold = c->add_allin_threshold;
  tc.force_allin_threshold = c->force_allin_threshold;
  tc.merging_threshold = c->merging_threshold;
  tc.depth_limit = c->depth_limit;
  BetSizeOptions* streets[3] = {tc.flop_bet_sizes, tc.turn_bet_sizes, tc.river_bet_sizes};
  for (int s = 0; s < 3; ++s)
    for (int p = 0; p < 2; ++p) {
      const char* b = c->sizes[s * 4 + p * 2 + 0];
      const char* r = c->sizes[s * 4 + p * 2 + 1];
      if (!parse_bet_size_options(b ? b : "", r ? r : "", streets[s][p], err)) return false;
    }
  if (c->donk[0]) {
    tc.has_turn_donk = true;
    if (!parse_donk_size_options(c->donk[0], tc.turn_donk_sizes, err)) return false;
  }
  if (c->donk[1]) {
    tc.has_river_donk = true;
    if (!parse_donk_size_options(c->donk[1], tc.river_donk_sizes, err)) return false;
  }
  return true;
}

// Parses one bet-size list (bet_size.rs:82-112); kinds / f / i / cap per entry.
int orc_parse_bet_sizes(const char* s, int is_raise, int32_t* kinds, double* f, int32_t* i, int32_t* cap, int n) {
  BetSizeOptions o;
  std::string err;
  if (!parse_bet_size_options(is_raise ? "" : s, is_raise ? s : "", o, err)) {
    g_err = err;
    return -1;
  }
  const auto& v = is_raise ? o.raise : o.bet;
  for (size_t k = 0; k < v.size() && (int)k < n; ++k) {
    kinds[k] = v[k].kind;
    f[k] = v[k].f;
    i[k] = v[k].i;
    cap[k] = v[k].cap;
  }
  return (int)v.size();
}

// Returns the root actions of the abstract action tree (kinds, amounts).
int orc_action_tree_root(const OrcTreeConfig* c, int32_t* kinds, int32_t* amounts, int cap) {
  TreeConfig tc;
  std::string err;
  if (!build_tree_config(c, tc, err)) {
    g_err = err;
    return -1;
  }
  ActionTree t;
  if (!ActionTree::create(tc, t, err)) {
    g_err = err;
    return -1;
  }
  int n = (int)t.root->actions.size();
  for (int i = 0; i < n && i < cap; ++i) {
    kinds[i] = t.root->actions[i].kind;
    amounts[i] = t.root->actions[i].amount;
  }
  return n;
}

void* orc_game_new(const float* range_oop, const float* range_ip, const uint8_t* board5,
                   const OrcTreeConfig* c, int fp64) {
  try {
    TreeConfig tc;
    std::string err;
    if (!build_tree_config(c, tc, err)) {
      g_err = err;
      return nullptr;
    }
    ActionTree tree;
    if (!ActionTree::create(tc, tree, err)) {
      g_err = err;
      return nullptr;
    }
    CardConfig cc;
    std::memcpy(cc.range[0].data, range_oop, sizeof(float) * 1326);
    std::memcpy(cc.range[1].data, range_ip, sizeof(float) * 1326);
    for (int i = 0; i < 3; ++i) cc.flop[i] = board5[i];
    cc.turn = board5[3];
    cc.river = board5[4];
    auto* h = new OrcGame();
    h->fp64 = fp64;
    bool ok;
    if (fp64) {
      h->g64 = new Game<double>();
      ok = h->g64->with_config(cc, std::move(tree), err);
    } else {
      h->g32 = new Game<float>();
      ok = h->g32->with_config(cc, std::move(tree), err);
    }
    if (!ok) {
      g_err = err;
      delete h->g32;
      delete h->g64;
      delete h;
      return nullptr;
    }
    return h;
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}

void orc_game_free(void* p) {
  auto* h = (OrcGame*)p;
  if (!h) return;
  delete h->g32;
  delete h->g64;
  delete h;
}

int orc_allocate_memory(void* p) {
  ORC_TRY(return with((OrcGame*)p, [](auto& g) { g.allocate_memory(); return 0; });)
}

int64_t orc_num_private_hands(void* p, int pl) {
  return with((OrcGame*)p, [&](auto& g) { return (int64_t)g.num_private_hands(pl); });
}

int orc_private_cards(void* p, int pl, uint8_t* out) {
  return with((OrcGame*)p, [&](auto& g) {
    for (size_t i = 0; i < g.private_cards[pl].size(); ++i) {
      out[2 * i] = g.private_cards[pl][i].first;
      out[2 * i + 1] = g.private_cards[pl][i].second;
    }
    return 0;
  });
}

int orc_initial_weights(void* p, int pl, double* out) {
  return with((OrcGame*)p, [&](auto& g) { to_f64(g.initial_weights[pl], out); return 0; });
}

double orc_num_combinations(void* p) {
  return with((OrcGame*)p, [](auto& g) { return g.num_combinations; });
}

int64_t orc_num_nodes(void* p) {
  return with((OrcGame*)p, [](auto& g) { return (int64_t)g.arena.size(); });
}

// out: player, amount, turn, river, num_children, children_offset, prev_kind, prev_amount
int orc_node_info(void* p, int64_t idx, int32_t* out) {
  return with((OrcGame*)p, [&](auto& g) {
    const Node& n = g.arena[idx];
    out[0] = n.player;
    out[1] = n.amount;
    out[2] = n.turn;
    out[3] = n.river;
    out[4] = n.num_children;
    out[5] = (int32_t)n.children_offset;
    out[6] = n.prev_action.kind;
    out[7] = n.prev_action.amount;
    return 0;
  });
}

int orc_same_hand_index(void* p, int pl, uint16_t* out) {
  return with((OrcGame*)p, [&](auto& g) {
    std::memcpy(out, g.same_hand_index[pl].data(), 2 * g.same_hand_index[pl].size());
    return 0;
  });
}

// kind 0 = flop, 1 = turn (key = turn card), 2 = river (key = pair index)
int orc_valid_indices(void* p, int kind, int key, int pl, uint16_t* out) {
  return with((OrcGame*)p, [&](auto& g) {
    const Indices& ix = kind == 0 ? g.valid_indices_flop
                        : kind == 1 ? g.valid_indices_turn[key]
                                    : g.valid_indices_river[key];
    std::memcpy(out, ix[pl].data(), 2 * ix[pl].size());
    return (int)ix[pl].size();
  });
}

int orc_hand_strength(void* p, int pair_index, int pl, uint16_t* strength, uint16_t* index) {
  return with((OrcGame*)p, [&](auto& g) {
    const auto& v = g.hand_strength[pair_index][pl];
    for (size_t i = 0; i < v.size(); ++i) {
      strength[i] = v[i].strength;
      index[i] = v[i].index;
    }
    return (int)v.size();
  });
}

// Sizes of the isomorphism tables: ref_turn, card_turn, ref_river[turn].
int orc_isomorphism_counts(void* p, int turn, int32_t* out3) {
  return with((OrcGame*)p, [&](auto& g) {
    out3[0] = (int32_t)g.isomorphism_ref_turn.size();
    out3[1] = (int32_t)g.isomorphism_card_turn.size();
    out3[2] = turn < 52 ? (int32_t)g.isomorphism_ref_river[turn].size() : 0;
    return 0;
  });
}

float orc_solve(void* p, uint32_t max_iter, float target, int print, uint32_t* iters) {
  try {
    return with((OrcGame*)p, [&](auto& g) { return g.solve(max_iter, target, print != 0, iters); });
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1.0f;
  }
}

int orc_solve_step(void* p, uint32_t t) {
  ORC_TRY(return with((OrcGame*)p, [&](auto& g) { g.solve_step(t); return 0; });)
}

int orc_solve_pass(void* p, uint32_t t, int player) {
  ORC_TRY(return with((OrcGame*)p, [&](auto& g) { g.solve_pass(t, player); return 0; });)
}

// Overwrites one decision node's storage (1 strategy sums, 2 regrets) from float32 rows.
int orc_seed_node_storage(void* p, int64_t idx, int which, const float* v, int64_t n) {
  return with((OrcGame*)p, [&](auto& g) {
    const Node& nd = g.arena[idx];
    if (nd.is_terminal() || nd.is_chance() || (int64_t)nd.num_elements != n) return -1;
    auto& st = which == 1 ? g.storage1 : g.storage2;
    for (int64_t i = 0; i < n; ++i) st[nd.s1 + i] = v[i];
    return 0;
  });
}

float orc_exploitability(void* p) {
  try {
    return with((OrcGame*)p, [](auto& g) { return g.compute_exploitability(); });
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1.0f;
  }
}

int orc_mes_ev(void* p, float* out2) {
  ORC_TRY(return with((OrcGame*)p, [&](auto& g) { auto e = g.compute_mes_ev(); out2[0] = e[0]; out2[1] = e[1]; return 0; });)
}

int orc_current_ev(void* p, float* out2) {
  ORC_TRY(return with((OrcGame*)p, [&](auto& g) { auto e = g.compute_current_ev(); out2[0] = e[0]; out2[1] = e[1]; return 0; });)
}

int orc_finalize(void* p) {
  ORC_TRY(return with((OrcGame*)p, [](auto& g) { g.finalize(); return 0; });)
}

int orc_root_cfvalues_with_reach(void* p, int pl, const float* reach, double* out) {
  ORC_TRY(return with((OrcGame*)p, [&](auto& g) {
    using F = typename std::remove_reference_t<decltype(g.initial_weights[0])>::value_type;
    std::vector<F> r(reach, reach + g.num_private_hands(pl ^ 1));
    auto v = g.root_cfvalues_with_reach(pl, r.data());
    to_f64(v, out);
    return 0;
  });)
}

// which: 1 = strategy sum (storage1), 2 = regrets / cfvalues (storage2),
// 3 = IP cfvalues, 4 = chance cfvalues
int64_t orc_node_storage(void* p, int64_t idx, int which, double* out) {
  return with((OrcGame*)p, [&](auto& g) -> int64_t {
    const Node& n = g.arena[idx];
    if (n.is_terminal()) return 0;
    if (which == 4) {
      if (!n.is_chance()) return 0;
      for (size_t i = 0; i < n.num_elements; ++i) out[i] = (double)g.storage_chance[n.s1 + i];
      return n.num_elements;
    }
    if (n.is_chance()) return 0;
    if (which == 3) {
      for (size_t i = 0; i < n.num_elements_ip; ++i) out[i] = (double)g.storage_ip[n.s3 + i];
      return n.num_elements_ip;
    }
    const auto& st = which == 1 ? g.storage1 : g.storage2;
    for (size_t i = 0; i < n.num_elements; ++i) out[i] = (double)st[n.s1 + i];
    return n.num_elements;
  });
}

int64_t orc_strategy_at_index(void* p, int64_t idx, double* out) {
  try {
    return with((OrcGame*)p, [&](auto& g) -> int64_t {
      auto v = g.strategy_at_index(idx);
      to_f64(v, out);
      return (int64_t)v.size();
    });
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

int64_t orc_num_boundary_nodes(void* p) {
  return with((OrcGame*)p, [](auto& g) { return (int64_t)g.num_boundary_nodes(); });
}

int orc_boundary_node_indices(void* p, int64_t* out) {
  return with((OrcGame*)p, [&](auto& g) {
    for (size_t i = 0; i < g.node_to_boundary.size(); ++i)
      if (g.node_to_boundary[i] != 0xFFFFFFFFu) out[g.node_to_boundary[i]] = (int64_t)i;
    return 0;
  });
}

int orc_set_boundary_cfvs(void* p, int64_t ordinal, int pl, const float* v, int64_t n) {
  return with((OrcGame*)p, [&](auto& g) {
    size_t idx = ordinal * 2 + pl;
    if (idx < g.boundary_cfvs.size()) g.boundary_cfvs[idx].assign(v, v + n);
    return 0;
  });
}

// Central differences of L = g0 . cfv0 + g1 . cfv1, where cfv_p are the root
// cfvalues of player p under the game's current average strategy with the
// opponent's reach w_{1-p} (root_cfvalues_with_reach, utility.rs:422-443), at n
// coordinates: kind 0 = weight w_p[hand], kind 1 = boundary value of player p
// at boundary `ord`, hand `hand` (set_boundary_cfvs, interpreter.rs:343).
// L is linear in every coordinate, so a central difference is exact up to
// rounding.  Each perturbed input is rounded to f32, as the device reads it,
// and the step actually taken divides the difference.  Only the term that the
// coordinate reaches is re-evaluated: a weight of p moves cfv_{1-p}, a
// boundary value of p moves cfv_p.  Test infrastructure: FP64 games only.
int orc_fd_central(void* p, const float* w0, const float* w1, const float* g0, const float* g1, int n,
                   const int32_t* kind, const int32_t* ord, const int32_t* pl, const int32_t* hand, double h,
                   double* out) {
  auto* hd = (OrcGame*)p;
  if (!hd || !hd->fp64) {
    g_err = "orc_fd_central needs an FP64 game";
    return -1;
  }
  try {
    Game<double>& g = *hd->g64;
    const float* w[2] = {w0, w1};
    const float* gv[2] = {g0, g1};
    std::vector<double> wd[2];
    for (int q = 0; q < 2; ++q) wd[q].assign(w[q], w[q] + g.num_private_hands(q));
    // value of g_q . cfv_q with opponent reach r
    auto term = [&](int q, const std::vector<double>& r) {
      std::vector<double> v = g.root_cfvalues_with_reach(q, r.data());
      double acc = 0.0;
      for (size_t i = 0; i < v.size(); ++i) acc += (double)gv[q][i] * v[i];
      return acc;
    };
    for (int i = 0; i < n; ++i) {
      const int q = pl[i], j = hand[i];
      if (q < 0 || q > 1 || j < 0 || (size_t)j >= g.num_private_hands(q)) throw std::runtime_error("bad coordinate");
      if (kind[i] == 0) {
        std::vector<double> r = wd[q];
        const double xp = (double)(float)(r[j] + h), xm = (double)(float)(r[j] - h);
        r[j] = xp;
        const double lp = term(q ^ 1, r);
        r[j] = xm;
        const double lm = term(q ^ 1, r);
        out[i] = (lp - lm) / (xp - xm);
      } else {
        const size_t k = (size_t)ord[i] * 2 + q;
        if (k >= g.boundary_cfvs.size() || (size_t)j >= g.boundary_cfvs[k].size())
          throw std::runtime_error("bad boundary coordinate");
        const double x0 = g.boundary_cfvs[k][j];
        const double xp = (double)(float)(x0 + h), xm = (double)(float)(x0 - h);
        g.boundary_cfvs[k][j] = xp;
        const double lp = term(q, wd[q ^ 1]);
        g.boundary_cfvs[k][j] = xm;
        const double lm = term(q, wd[q ^ 1]);
        g.boundary_cfvs[k][j] = x0;
        out[i] = (lp - lm) / (xp - xm);
      }
    }
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

int orc_boundary_reach(void* p, int64_t ordinal, int pl, double* out) {
  return with((OrcGame*)p, [&](auto& g) {
    const auto& r = g.boundary_reach[ordinal * 2 + pl];
    to_f64(r, out);
    return (int)r.size();
  });
}

int orc_evaluate_node(void* p, int64_t idx, int pl, const float* cfreach, double* out) {
  ORC_TRY(return with((OrcGame*)p, [&](auto& g) {
    using F = typename std::remove_reference_t<decltype(g.initial_weights[0])>::value_type;
    std::vector<F> r(cfreach, cfreach + g.num_private_hands(pl ^ 1));
    std::vector<F> res(g.num_private_hands(pl));
    g.evaluate(res.data(), g.arena[idx], pl, r.data());
    to_f64(res, out);
    return 0;
  });)
}

// -------- navigation / queries (query.rs) --------
int orc_back_to_root(void* p) {
  ORC_TRY(return with((OrcGame*)p, [](auto& g) { g.back_to_root(); return 0; });)
}

int orc_play(void* p, int64_t action) {
  ORC_TRY(return with((OrcGame*)p, [&](auto& g) { g.play(action < 0 ? (size_t)-1 : (size_t)action); return 0; });)
}

int orc_available_actions(void* p, int32_t* kinds, int32_t* amounts, int cap) {
  return with((OrcGame*)p, [&](auto& g) {
    auto a = g.available_actions();
    for (size_t i = 0; i < a.size() && (int)i < cap; ++i) {
      kinds[i] = a[i].kind;
      amounts[i] = a[i].amount;
    }
    return (int)a.size();
  });
}

int orc_is_terminal_node(void* p) { return with((OrcGame*)p, [](auto& g) { return (int)g.is_terminal_node(); }); }
int orc_is_chance_node(void* p) { return with((OrcGame*)p, [](auto& g) { return (int)g.is_chance_node(); }); }
int orc_current_player(void* p) { return with((OrcGame*)p, [](auto& g) { return g.current_player(); }); }
uint64_t orc_possible_cards(void* p) { return with((OrcGame*)p, [](auto& g) { return g.possible_cards(); }); }
int64_t orc_current_node_index(void* p) {
  return with((OrcGame*)p, [](auto& g) { return (int64_t)g.node_index(g.cur_node()); });
}

int64_t orc_strategy(void* p, double* out) {
  try {
    return with((OrcGame*)p, [&](auto& g) -> int64_t { auto v = g.strategy(); to_f64(v, out); return (int64_t)v.size(); });
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

int orc_cache_normalized_weights(void* p) {
  ORC_TRY(return with((OrcGame*)p, [](auto& g) { g.cache_normalized_weights(); return 0; });)
}

int orc_weights(void* p, int pl, int normalized, double* out) {
  return with((OrcGame*)p, [&](auto& g) {
    to_f64(normalized ? g.normalized_weights[pl] : g.weights[pl], out);
    return 0;
  });
}

int64_t orc_expected_values(void* p, int pl, int detail, double* out) {
  try {
    return with((OrcGame*)p, [&](auto& g) -> int64_t {
      auto v = detail ? g.expected_values_detail(pl) : g.expected_values(pl);
      to_f64(v, out);
      return (int64_t)v.size();
    });
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

int orc_total_bet_amount(void* p, int32_t* out2) {
  return with((OrcGame*)p, [&](auto& g) { out2[0] = g.total_bet_amount[0]; out2[1] = g.total_bet_amount[1]; return 0; });
}

int orc_lock_current_strategy(void* p, const float* strategy) {
  ORC_TRY(return with((OrcGame*)p, [&](auto& g) {
    using F = typename std::remove_reference_t<decltype(g.initial_weights[0])>::value_type;
    auto* n = g.cur_node();
    size_t cnt = (size_t)n->num_children * g.num_private_hands(n->player);
    std::vector<F> s(strategy, strategy + cnt);
    g.lock_current_strategy(s.data());
    return 0;
  });)
}

}  // extern "C"
