// Host side of the B200 range solver (see ps_host.hpp).  Reference citations
// are paths inside crates/range-solver/src of tjennings/poker_solver_rust.
#include "ps_host.hpp"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <functional>

#include "ps_handeval.hpp"

namespace ps {

// ---------------------------------------------------------------------------
// Hand table by rank-multiset enumeration (see ps_handeval.hpp)
// ---------------------------------------------------------------------------
int build_hand_table(int32_t* out, int cap) {
  std::vector<int32_t> v;
  v.reserve(60000);
  int cnt[13];
  std::function<void(int, int)> rec = [&](int r, int left) {
    if (r == 13) {
      if (left == 0) v.push_back(value_from_counts(cnt));
      return;
    }
    for (int k = 0; k <= 4 && k <= left; ++k) {
      cnt[r] = k;
      rec(r + 1, left - k);
    }
    cnt[r] = 0;
  };
  rec(0, 7);
  for (uint32_t m = 0; m < (1u << 13); ++m) {
    int pc = ps_popc(m);
    if (pc >= 5 && pc <= 7) v.push_back(value_of_flush(m));
  }
  std::sort(v.begin(), v.end());
  v.erase(std::unique(v.begin(), v.end()), v.end());
  for (size_t i = 0; i < v.size() && (int)i < cap; ++i) out[i] = v[i];
  return (int)v.size();
}

// ---------------------------------------------------------------------------
// Bet-size menus (bet_size.rs:82-260)
// ---------------------------------------------------------------------------
static bool num_ok(const std::string& s, double& out) {  // bet_size.rs:149-155
  if (s.empty()) return false;
  for (char c : s)
    if (c == '+' || c == '-' || isalpha((unsigned char)c)) return false;
  char* e = nullptr;
  out = strtod(s.c_str(), &e);
  return *e == 0;
}

static bool parse_one(std::string s, bool raise, BetSize& b, std::string& err) {
  std::string orig = s;
  for (auto& c : s) c = (char)tolower((unsigned char)c);
  err = "Invalid bet size: " + orig;
  double x;
  auto pos_int = [&](const std::string& t, double lim, int& o) {
    double f;
    if (!num_ok(t, f) || std::trunc(f) != f || f == 0.0 || f > lim) return false;
    o = (int)f;
    return true;
  };
  if (!s.empty() && s.back() == 'x') {
    if (!raise) { err = "Relative size to the previous bet is not allowed: " + orig; return false; }
    if (!num_ok(s.substr(0, s.size() - 1), x)) return false;
    if (x <= 1.0) { err = "Multiplier must be greater than 1.0: " + orig; return false; }
    b = {BetSize::PrevBet, x, 0, 0};
    return true;
  }
  size_t cpos = s.find('c');
  if (cpos != std::string::npos) {
    std::string a = s.substr(0, cpos), rest = s.substr(cpos + 1);
    if (rest.find('c') != std::string::npos) return false;
    if (!num_ok(a, x)) return false;
    if (std::trunc(x) != x) { err = "Additional size must be an integer: " + orig; return false; }
    if (x > 2147483647.0) { err = "Additional size must be less than 2^31: " + orig; return false; }
    int cap = 0;
    if (!rest.empty()) {
      if (!raise) { err = "Raise cap is not allowed: " + orig; return false; }
      if (rest.back() != 'r') return false;
      if (!pos_int(rest.substr(0, rest.size() - 1), 100.0, cap)) {
        err = "Raise cap must be a positive integer <= 100: " + orig;
        return false;
      }
    }
    b = {BetSize::Add, 0.0, (int)x, cap};
    return true;
  }
  size_t epos = s.find('e');
  if (epos != std::string::npos) {
    std::string a = s.substr(0, epos), rest = s.substr(epos + 1);
    if (rest.find('e') != std::string::npos) return false;
    int n = 0;
    if (!a.empty() && !pos_int(a, 100.0, n)) {
      err = "Number of streets must be a positive integer <= 100: " + orig;
      return false;
    }
    double mx = INFINITY;
    if (!rest.empty()) {
      if (rest.back() != '%' || !num_ok(rest.substr(0, rest.size() - 1), x)) return false;
      mx = x / 100.0;
    }
    b = {BetSize::Geo, mx, n, 0};
    return true;
  }
  if (!s.empty() && s.back() == '%') {
    if (!num_ok(s.substr(0, s.size() - 1), x)) return false;
    b = {BetSize::Pot, x / 100.0, 0, 0};
    return true;
  }
  if (s == "a") {
    b = {BetSize::AllIn, 0.0, 0, 0};
    return true;
  }
  return false;
}

bool parse_menu(const std::string& str, bool raise, std::vector<BetSize>& out, std::string& err) {
  std::vector<std::string> items;
  size_t st = 0;
  for (size_t i = 0; i <= str.size(); ++i)
    if (i == str.size() || str[i] == ',') {
      std::string t = str.substr(st, i - st);
      size_t a = t.find_first_not_of(" \t\r\n"), z = t.find_last_not_of(" \t\r\n");
      items.push_back(a == std::string::npos ? "" : t.substr(a, z - a + 1));
      st = i + 1;
    }
  if (items.back().empty()) items.pop_back();
  out.clear();
  for (auto& it : items) {
    BetSize b;
    if (!parse_one(it, raise, b, err)) return false;
    out.push_back(b);
  }
  std::sort(out.begin(), out.end(), [](const BetSize& l, const BetSize& r) {
    if (l.kind != r.kind) return l.kind < r.kind;
    if (l.kind == BetSize::Pot || l.kind == BetSize::PrevBet) return l.ratio < r.ratio;
    if (l.kind == BetSize::Add) return l.n != r.n ? l.n < r.n : l.cap < r.cap;
    if (l.kind == BetSize::Geo) return l.n != r.n ? l.n < r.n : l.ratio < r.ratio;
    return false;
  });
  return true;
}

// ---------------------------------------------------------------------------
// Action tree (action_tree.rs:226-293, :646-925, :1200-1229)
// ---------------------------------------------------------------------------
namespace {
struct Line {  // betting state along a line of play
  Act prev;
  int32_t bets = 0;
  bool allin = false, oop_called = false;
  int32_t stack[2];
  int32_t prev_amount = 0;
  int transitions = 0;
  int street_bets = 0;  // extension counter for TreeCfg::max_bets

  Line next(uint8_t pl, Act a) const {
    Line n = *this;
    if (a.kind == ACT_CHECK) {
      n.oop_called = false;
    } else if (a.kind == ACT_CALL) {
      n.bets = 0;
      n.oop_called = pl == PL_OOP;
      n.stack[pl] = n.stack[pl ^ 1];
      n.prev_amount = 0;
    } else if (a.kind == ACT_BET || a.kind == ACT_RAISE || a.kind == ACT_ALLIN) {
      int32_t to_call = n.stack[pl] - n.stack[pl ^ 1];
      n.bets += 1;
      n.street_bets += 1;
      n.allin = a.kind == ACT_ALLIN;
      n.stack[pl] -= a.amount - n.prev_amount + to_call;
      n.prev_amount = a.amount;
    } else if (a.kind == ACT_CHANCE) {
      n.transitions += 1;
      n.street_bets = 0;
    }
    n.prev = a;
    return n;
  }
};

inline int32_t iround(double x) { return (int32_t)std::round(x); }

struct Builder {
  const TreeCfg& c;
  std::vector<ATree::N>& nodes;

  std::vector<Act> actions_for(const ATree::N& nd, const Line& L) {
    uint8_t pl = nd.player, op = pl ^ 1;
    int32_t to_call = L.stack[pl] - L.stack[op];
    int32_t pot = c.starting_pot + 2 * (nd.amount + to_call);
    int32_t max_amount = L.stack[op] + L.prev_amount;
    int32_t min_amount = std::min(std::max(L.prev_amount + to_call, 1), max_amount);
    double spr = (double)L.stack[op] / (double)pot;
    auto geo = [&](int ns, double mx) {
      double ratio = (std::pow(2.0 * spr + 1.0, 1.0 / (double)ns) - 1.0) / 2.0;
      return iround((double)pot * std::min(ratio, mx));
    };
    int street = nd.street, remaining = 3 - street;
    const std::vector<BetSize>* donk = street >= 1 && c.has_donk[street - 1] ? &c.donk[street - 1] : nullptr;
    std::vector<Act> acts;
    auto opening = [&](const std::vector<BetSize>& menu) {
      acts.push_back({ACT_CHECK, 0});
      for (const auto& b : menu) {
        if (b.kind == BetSize::Pot) acts.push_back({ACT_BET, iround((double)pot * b.ratio)});
        else if (b.kind == BetSize::Add) acts.push_back({ACT_BET, b.n});
        else if (b.kind == BetSize::Geo) acts.push_back({ACT_BET, geo(b.n == 0 ? remaining : b.n, b.ratio)});
        else if (b.kind == BetSize::AllIn) acts.push_back({ACT_ALLIN, max_amount});
      }
      if (max_amount <= iround((double)pot * c.add_allin_threshold)) acts.push_back({ACT_ALLIN, max_amount});
    };
    bool capped = c.max_bets > 0 && L.street_bets >= c.max_bets;
    if (donk && L.prev.kind == ACT_CHANCE && L.oop_called) {
      opening(*donk);
    } else if (L.prev.kind == ACT_NONE || L.prev.kind == ACT_CHECK || L.prev.kind == ACT_CHANCE) {
      opening(c.menu[street][pl].bet);
    } else {
      acts.push_back({ACT_FOLD, 0});
      acts.push_back({ACT_CALL, 0});
      if (!L.allin && !capped) {
        for (const auto& b : c.menu[street][pl].raise) {
          if (b.kind == BetSize::Pot) acts.push_back({ACT_RAISE, L.prev_amount + iround((double)pot * b.ratio)});
          else if (b.kind == BetSize::PrevBet) acts.push_back({ACT_RAISE, iround((double)L.prev_amount * b.ratio)});
          else if (b.kind == BetSize::Add) {
            if (b.cap == 0 || L.bets <= b.cap) acts.push_back({ACT_RAISE, L.prev_amount + b.n});
          } else if (b.kind == BetSize::Geo) {
            int ns = b.n == 0 ? std::max(remaining - L.bets + 1, 1) : std::max(b.n - L.bets + 1, 1);
            acts.push_back({ACT_RAISE, L.prev_amount + geo(ns, b.ratio)});
          } else {
            acts.push_back({ACT_ALLIN, max_amount});
          }
        }
        if (max_amount <= L.prev_amount + iround((double)pot * c.add_allin_threshold))
          acts.push_back({ACT_ALLIN, max_amount});
      }
    }
    auto above = [&](int32_t amount) {
      int32_t new_pot = pot + 2 * (amount - L.prev_amount);
      return max_amount <= amount + iround((double)new_pot * c.force_allin_threshold);
    };
    for (auto& a : acts)
      if (a.kind == ACT_BET || a.kind == ACT_RAISE) {
        int32_t cl = std::min(std::max(a.amount, min_amount), max_amount);
        if (above(cl)) a = {ACT_ALLIN, max_amount};
        else a.amount = cl;
      }
    std::sort(acts.begin(), acts.end());
    acts.erase(std::unique(acts.begin(), acts.end()), acts.end());
    // merge close bet sizes (action_tree.rs:1200-1229)
    std::vector<Act> kept;
    int32_t cur = 2147483647;
    for (auto it = acts.rbegin(); it != acts.rend(); ++it) {
      bool sized = it->kind == ACT_BET || it->kind == ACT_RAISE || it->kind == ACT_ALLIN;
      int32_t amt = sized ? it->amount : -1;
      if (amt > 0) {
        double ratio = (double)(amt - L.prev_amount) / (double)pot;
        double cur_ratio = (double)(cur - L.prev_amount) / (double)pot;
        double thr = (cur_ratio - c.merging_threshold) / (1.0 + c.merging_threshold);
        if (ratio < thr * (1.0 - 1e-12)) {
          kept.push_back(*it);
          cur = amt;
        }
      } else {
        kept.push_back(*it);
      }
    }
    std::reverse(kept.begin(), kept.end());
    return kept;
  }

  void expand(int idx, const Line& L) {
    ATree::N nd = nodes[idx];
    if (nd.player & PL_TERMINAL_FLAG) return;
    if (nd.player & PL_CHANCE_FLAG) {
      if (c.depth_limit >= 0 && L.transitions >= c.depth_limit) {
        nodes[idx].player = PL_BOUNDARY_FLAG;
        return;
      }
      bool second_blocked = c.depth_limit >= 0 && L.transitions + 1 >= c.depth_limit;
      uint8_t np = !L.allin ? PL_OOP
                   : nd.street == 0 ? (second_blocked ? PL_BOUNDARY_FLAG : (uint8_t)(PL_CHANCE_FLAG | PL_CHANCE))
                                    : PL_TERMINAL_FLAG;
      int first = (int)nodes.size();
      nodes[idx].first = first;
      nodes[idx].n = 1;
      nodes.push_back({np, (uint8_t)(nd.street + 1), nd.amount, -1, 0, {ACT_CHANCE, 0}});
      expand(first, L.next(0, {ACT_CHANCE, 0}));
      return;
    }
    auto acts = actions_for(nd, L);
    uint8_t pl = nd.player, op = pl ^ 1;
    int32_t to_call = L.stack[pl] - L.stack[op];
    bool dl = c.depth_limit >= 0 && L.transitions >= c.depth_limit;
    uint8_t after_call = nd.street == 2 ? PL_TERMINAL_FLAG : dl ? PL_BOUNDARY_FLAG : (uint8_t)(PL_CHANCE_FLAG | pl);
    uint8_t after_check = pl == PL_OOP ? op : after_call;
    int first = (int)nodes.size();
    nodes[idx].first = first;
    nodes[idx].n = (int)acts.size();
    for (const auto& a : acts) {
      int32_t amount = nd.amount;
      uint8_t np;
      if (a.kind == ACT_FOLD) np = PL_FOLD_FLAG | pl;
      else if (a.kind == ACT_CHECK) np = after_check;
      else if (a.kind == ACT_CALL) { amount += to_call; np = after_call; }
      else { amount += to_call; np = op; }
      nodes.push_back({np, nd.street, amount, -1, 0, a});
    }
    for (size_t k = 0; k < acts.size(); ++k) expand(first + (int)k, L.next(pl, acts[k]));
  }
};
}  // namespace

bool ATree::build(const TreeCfg& cfg, ATree& out, std::string& err) {
  if (cfg.starting_pot <= 0) { err = "Starting pot must be positive: " + std::to_string(cfg.starting_pot); return false; }
  if (cfg.effective_stack <= 0) { err = "Effective stack must be positive: " + std::to_string(cfg.effective_stack); return false; }
  if (cfg.rake_rate < 0.0) { err = "Rake rate must be non-negative"; return false; }
  if (cfg.rake_rate > 1.0) { err = "Rake rate must be less than or equal to 1.0"; return false; }
  if (cfg.rake_cap < 0.0) { err = "Rake cap must be non-negative"; return false; }
  if (cfg.add_allin_threshold < 0.0 || cfg.force_allin_threshold < 0.0 || cfg.merging_threshold < 0.0) {
    err = "Thresholds must be non-negative";
    return false;
  }
  for (int s = 0; s < 3; ++s)
    for (int p = 0; p < 2; ++p)
      for (const auto& b : cfg.menu[s][p].bet)
        if (b.kind == BetSize::PrevBet) { err = "Unexpected `PrevBetRelative`"; return false; }
  out.cfg = cfg;
  out.nodes.clear();
  out.nodes.push_back({PL_OOP, (uint8_t)cfg.initial_state, 0, -1, 0, {ACT_NONE, 0}});
  Line L;
  L.stack[0] = L.stack[1] = cfg.effective_stack;
  Builder b{out.cfg, out.nodes};
  b.expand(0, L);
  return true;
}

bool ATree::has_invalid_terminal() const {  // action_tree.rs:928-945
  for (const auto& n : nodes)
    if (!(n.player & PL_TERMINAL_FLAG) && n.n == 0) return true;
  return false;
}

// ---------------------------------------------------------------------------
// Game construction
// ---------------------------------------------------------------------------
Discount discount_params(uint32_t t) {  // solver.rs:26-44
  uint32_t p4 = t == 0 ? 0 : 1u << ((31 - __builtin_clz(t)) & ~1);
  double ta = (double)std::max((int32_t)t - 1, 0);
  double tg = (double)(t - p4);
  double pa = ta * std::sqrt(ta);
  double g = tg / (tg + 1.0);
  Discount d;
  d.alpha = (float)(pa / (pa + 1.0));
  d.beta = 0.5f;
  d.gamma = (float)((g * g) * g);
  d.pad = 0.f;
  return d;
}

bool Game::check_cards(std::string& err) {  // interpreter.rs:542-662
  auto bad = [](int c) { return c >= 52; };
  if (flop[0] == NOT_DEALT || flop[1] == NOT_DEALT || flop[2] == NOT_DEALT) { err = "Flop cards not initialized"; return false; }
  if (bad(flop[0]) || bad(flop[1]) || bad(flop[2])) { err = "Flop cards must be in [0, 52)"; return false; }
  if (flop[0] == flop[1] || flop[0] == flop[2] || flop[1] == flop[2]) { err = "Flop cards must be unique"; return false; }
  auto in_flop = [&](int x) { return x == flop[0] || x == flop[1] || x == flop[2]; };
  if (turn != NOT_DEALT && (bad(turn) || in_flop(turn))) { err = "Invalid turn card: " + std::to_string(turn); return false; }
  if (river != NOT_DEALT) {
    if (bad(river) || in_flop(river) || river == turn) { err = "Invalid river card: " + std::to_string(river); return false; }
    if (turn == NOT_DEALT) { err = "River card specified without turn card"; return false; }
  }
  int expected = turn == NOT_DEALT ? 0 : river == NOT_DEALT ? 1 : 2;
  if (cfg.initial_state != expected) { err = "Invalid initial state of `tree_config`"; return false; }
  for (int p = 0; p < 2; ++p) {
    bool any = false, valid = true;
    for (int i = 0; i < 1326; ++i) {  // bitwise, no branches: the compiler vectorises it
      any |= range[p][i] != 0.0f;
      valid &= (range[p][i] >= 0.0f) & (range[p][i] <= 1.0f);
    }
    if (!any) { err = p == 0 ? "OOP range is empty" : "IP range is empty"; return false; }
    if (!valid) { err = p == 0 ? "OOP range is invalid" : "IP range is invalid"; return false; }
  }
  uint64_t dead = (1ull << flop[0]) | (1ull << flop[1]) | (1ull << flop[2]);
  if (turn != NOT_DEALT) dead |= 1ull << turn;
  if (river != NOT_DEALT) dead |= 1ull << river;
  // the hand lists are written without branches (every combo is stored at
  // the running count, which advances only for a kept hand): a range's zero
  // weights follow no pattern the branch predictor could learn
  int pos[2][1326];
  for (int p = 0; p < 2; ++p) {
    cards[p].resize(1326);
    w[p].resize(1326);
    std::array<uint8_t, 2>* cp = cards[p].data();
    float* wp = w[p].data();
    int k = 0, m = 0;  // k = pair_index(c1, c2) in this loop order, m = hands kept
    for (int c1 = 0; c1 < 52; ++c1)
      for (int c2 = c1 + 1; c2 < 52; ++c2, ++k) {
        const float x = range[p][k];
        const int keep = (x > 0.0f) & ((dead & ((1ull << c1) | (1ull << c2))) == 0);
        cp[m] = {(uint8_t)c1, (uint8_t)c2};
        wp[m] = x;
        pos[p][k] = keep ? m : -1;
        m += keep;
      }
    cards[p].resize(m);
    w[p].resize(m);
    H[p] = m;
    hs[p] = (H[p] + 3) & ~3;
  }
  vstride = (std::max(hs[0], hs[1]) + 31) & ~31;
  for (int p = 0; p < 2; ++p) {
    same[p].resize(H[p]);
    for (int i = 0; i < H[p]; ++i) {
      const int q = pos[p ^ 1][pair_index(cards[p][i][0], cards[p][i][1])];
      same[p][i] = q >= 0 ? (uint16_t)q : (uint16_t)0xFFFF;
    }
  }
  // C = sum over compatible (oop, ip) pairs of w_oop * w_ip (interpreter.rs:619-635),
  // by inclusion-exclusion: all pairs - pairs sharing a card + identical pairs.
  double W[2] = {0, 0}, M[2][52];
  for (int p = 0; p < 2; ++p) {
    for (int c = 0; c < 52; ++c) M[p][c] = 0;
    for (int i = 0; i < H[p]; ++i) {
      double x = (double)w[p][i];
      W[p] += x;
      M[p][cards[p][i][0]] += x;
      M[p][cards[p][i][1]] += x;
    }
  }
  double shared = 0, ident = 0;
  for (int c = 0; c < 52; ++c) shared += M[0][c] * M[1][c];
  for (int i = 0; i < H[0]; ++i)
    if (same[0][i] != 0xFFFF) ident += (double)w[0][i] * (double)w[1][same[0][i]];
  num_combinations = W[0] * W[1] - shared + ident;
  if (!(num_combinations > 0.0)) { err = "Valid card assignment does not exist"; return false; }
  return true;
}

static bool suit_iso(const float* r, int s1, int s2) {  // range.rs:426-450
  auto rep = [&](int s) { return s == s1 ? s2 : s == s2 ? s1 : s; };
  for (int c1 = 0; c1 < 52; ++c1)
    for (int c2 = c1 + 1; c2 < 52; ++c2)
      if (r[pair_index(c1, c2)] != r[pair_index((c1 & ~3) | rep(c1 & 3), (c2 & ~3) | rep(c2 & 3))]) return false;
  return true;
}

// isomorphism.rs:33-234
void Game::init_isomorphism() {
  int cls[4] = {0, 0, 0, 0}, next = 1;
  for (int s2 = 1; s2 < 4; ++s2) {
    int found = -1;
    for (int s1 = 0; s1 < s2 && found < 0; ++s1)
      if (suit_iso(range[0], s1, s2) && suit_iso(range[1], s1, s2)) found = s1;
    cls[s2] = found >= 0 ? cls[found] : next++;
  }
  uint64_t fmask = (1ull << flop[0]) | (1ull << flop[1]) | (1ull << flop[2]);
  uint16_t frs[4] = {0, 0, 0, 0};
  for (int k = 0; k < 3; ++k) frs[flop[k] & 3] |= (uint16_t)(1 << (flop[k] >> 2));
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) iso_perm_river[a][b] = -1;
  auto perm_for = [&](int s1, int s2) {
    for (size_t i = 0; i < iso_swaps.size(); ++i)
      if (iso_swaps[i][0] == s1 && iso_swaps[i][1] == s2) return (int)i;
    iso_swaps.push_back({(uint8_t)s1, (uint8_t)s2});
    for (int p = 0; p < 2; ++p) {
      std::vector<int> rev(1326, -1);
      for (int i = 0; i < H[p]; ++i) rev[pair_index(cards[p][i][0], cards[p][i][1])] = i;
      std::vector<uint16_t> perm(hs[p]);
      for (int i = 0; i < hs[p]; ++i) perm[i] = (uint16_t)i;
      auto repl = [&](int c) { return (c & 3) == s1 ? c - s1 + s2 : (c & 3) == s2 ? c + s1 - s2 : c; };
      for (int i = 0; i < H[p]; ++i) {
        int j = rev[pair_index(repl(cards[p][i][0]), repl(cards[p][i][1]))];
        if (j >= 0) perm[i] = (uint16_t)j;
      }
      iso_perm[p].push_back(perm);
    }
    return (int)iso_swaps.size() - 1;
  };
  auto internal = [&](std::vector<uint8_t>& iref, std::vector<uint8_t>& icard, uint64_t mask, const int iso_suit[4]) {
    bool push = icard.empty();
    uint8_t counter = 0, idx[52] = {0};
    for (int c = 0; c < 52; ++c) {
      if ((1ull << c) & mask) continue;
      int s = c & 3;
      if (iso_suit[s] >= 0) {
        iref.push_back(idx[c - s + iso_suit[s]]);
        if (push) icard.push_back((uint8_t)c);
      } else {
        idx[c] = counter++;
      }
    }
  };
  iso_ref_turn.clear();
  iso_card_turn.clear();
  if (turn == NOT_DEALT) {
    int isu[4] = {-1, -1, -1, -1};
    for (int s1 = 1; s1 < 4; ++s1)
      for (int s2 = 0; s2 < s1; ++s2)
        if (frs[s1] == frs[s2] && cls[s1] == cls[s2]) {
          isu[s1] = s2;
          iso_perm_turn[s1] = perm_for(s1, s2);
          break;
        }
    internal(iso_ref_turn, iso_card_turn, fmask, isu);
  }
  iso_ref_river.assign(52, {});
  for (auto& v : iso_card_river) v.clear();
  if (river == NOT_DEALT) {
    for (int t = 0; t < 52; ++t) {
      if (((1ull << t) & fmask) || (turn != NOT_DEALT && turn != t)) continue;
      uint16_t trs[4] = {frs[0], frs[1], frs[2], frs[3]};
      trs[t & 3] |= (uint16_t)(1 << (t >> 2));
      int isu[4] = {-1, -1, -1, -1};
      for (int s1 = 1; s1 < 4; ++s1)
        for (int s2 = 0; s2 < s1; ++s2)
          if ((frs[s1] == frs[s2] || turn != NOT_DEALT) && trs[s1] == trs[s2] && cls[s1] == cls[s2]) {
            isu[s1] = s2;
            iso_perm_river[t & 3][s1] = perm_for(s1, s2);
            break;
          }
      internal(iso_ref_river[t], iso_card_river[t & 3], fmask | (1ull << t), isu);
    }
  }
}

void Game::build_arena(const ATree& t) {  // interpreter.rs:708-947
  uint64_t cnt[3] = {0, 0, 0};
  std::function<void(int, int)> count = [&](int i, int street) {
    cnt[street] += 1;
    const auto& n = t.nodes[i];
    if (n.player & PL_TERMINAL_FLAG) return;
    if (n.player & PL_CHANCE_FLAG) count(n.first, street + 1);
    else
      for (int k = 0; k < n.n; ++k) count(n.first + k, street);
  };
  count(0, cfg.initial_state);
  uint64_t fmask = (1ull << flop[0]) | (1ull << flop[1]) | (1ull << flop[2]);
  uint64_t turn_coef, river_coef;
  if (turn == NOT_DEALT) {
    uint64_t skip = 0;
    for (auto c : iso_card_turn) skip |= 1ull << c;
    river_coef = 0;
    for (int x = 0; x < 52; ++x)
      if (!((1ull << x) & (fmask | skip))) river_coef += 48 - iso_card_river[x & 3].size();
    turn_coef = 49 - iso_card_turn.size();
  } else if (river == NOT_DEALT) {
    turn_coef = 1;
    river_coef = 48 - iso_card_river[turn & 3].size();
  } else {
    turn_coef = 0;
    river_coef = 1;
  }
  uint64_t nn[3] = {cnt[0], cnt[1] * turn_coef, cnt[2] * river_coef};
  arena.assign(nn[0] + nn[1] + nn[2], ArenaNode());
  uint64_t base[3] = {0, nn[0], nn[0] + nn[1]};
  base[cfg.initial_state] += 1;
  arena[0].turn = turn;
  arena[0].river = river;
  std::function<void(size_t, int)> build = [&](size_t ni, int ai) {
    const auto& an = t.nodes[ai];
    ArenaNode& n = arena[ni];
    n.player = an.player;
    n.amount = an.amount;
    if (n.terminal()) return;
    if (n.chance()) {
      uint64_t mask, skip = 0;
      int street;
      if (n.turn == NOT_DEALT) {
        mask = fmask;
        for (auto c : iso_card_turn) skip |= 1ull << c;
        street = 1;
      } else {
        mask = fmask | (1ull << n.turn);
        for (auto c : iso_card_river[n.turn & 3]) skip |= 1ull << c;
        street = 2;
      }
      n.child_off = (uint32_t)(base[street] - ni);
      for (int c = 0; c < 52; ++c)
        if (!((1ull << c) & (mask | skip))) {
          ArenaNode& ch = arena[ni + n.child_off + n.nch];
          n.nch += 1;
          ch.prev = {ACT_CHANCE, c};
          if (street == 1) ch.turn = (uint8_t)c;
          else { ch.turn = n.turn; ch.river = (uint8_t)c; }
        }
      base[street] += n.nch;
      size_t off = n.child_off, nch = n.nch;
      for (size_t a = 0; a < nch; ++a) build(ni + off + a, an.first);
    } else {
      int street = n.turn == NOT_DEALT ? 0 : n.river == NOT_DEALT ? 1 : 2;
      n.child_off = (uint32_t)(base[street] - ni);
      n.nch = (uint16_t)an.n;
      base[street] += an.n;
      for (int a = 0; a < an.n; ++a) {
        ArenaNode& ch = arena[ni + n.child_off + a];
        ch.prev = t.nodes[an.first + a].act;
        ch.turn = n.turn;
        ch.river = n.river;
      }
      size_t off = n.child_off;
      for (int a = 0; a < an.n; ++a) build(ni + off + a, an.first + a);
    }
  };
  build(0, 0);
  // storage offsets in arena order (interpreter.rs:971-1007); R/S rows padded to hs
  num_storage = num_storage_ip = num_storage_chance = 0;
  bnd_ordinal.assign(arena.size(), -1);
  num_boundary = 0;
  for (size_t i = 0; i < arena.size(); ++i) {
    ArenaNode& n = arena[i];
    if (n.terminal()) {
      if (n.boundary()) bnd_ordinal[i] = num_boundary++;
      continue;
    }
    if (n.chance()) {
      int sp = n.player & PL_MASK;
      if (sp == 0 || sp == 1) {
        n.ch_off = (uint32_t)num_storage_chance;
        num_storage_chance += H[sp ^ 1];
      }
    } else {
      n.rs_off = (uint32_t)num_storage;
      num_storage += (uint64_t)n.nch * hs[n.player];
      if (n.prev.kind == ACT_NONE || n.prev.kind == ACT_CHANCE) {
        n.ip_off = (uint32_t)num_storage_ip;
        num_storage_ip += H[PL_IP];
      }
    }
  }
  // boards and isomorphism lists per chance node
  boards.clear();
  boards.push_back({flop[0], flop[1], flop[2], turn, river});
  node_board.assign(arena.size(), 0);
  chance_iso_id.assign(arena.size(), -1);
  iso_list_off.assign(1, 0);
  iso_list.clear();
  std::vector<int> board_of(1326 + 53, -1);
  for (size_t i = 0; i < arena.size(); ++i) {
    const ArenaNode& n = arena[i];
    if (n.turn != turn || n.river != river) {
      int key = n.river != NOT_DEALT ? pair_index(n.turn, n.river) : 1326 + n.turn;
      if (board_of[key] < 0) {
        board_of[key] = (int)boards.size();
        boards.push_back({flop[0], flop[1], flop[2], n.turn, n.river});
      }
      node_board[i] = board_of[key];
    }
    if (n.chance() && !n.terminal()) {
      const auto& iref = n.turn == NOT_DEALT ? iso_ref_turn : iso_ref_river[n.turn];
      const auto& icard = n.turn == NOT_DEALT ? iso_card_turn : iso_card_river[n.turn & 3];
      if (!iref.empty()) {
        chance_iso_id[i] = (int)iso_list_off.size() - 1;
        for (size_t k = 0; k < iref.size(); ++k) {
          int perm = n.turn == NOT_DEALT ? iso_perm_turn[icard[k] & 3] : iso_perm_river[n.turn & 3][icard[k] & 3];
          iso_list.push_back({(int32_t)iref[k], perm});
        }
        iso_list_off.push_back((int32_t)iso_list.size());
      }
    }
  }
}

// Level-ordered program for traverser p (see ps_device.hpp for the op set).
// terminals_first: every terminal of the pass is evaluated in one step right
// after the forward sweep (a terminal reads only reach vectors the forward
// sweep wrote), so the backward steps hold node ops alone.  A pass then has
// one step of terminal runs - the long items - instead of one per depth,
// which shortens a lone game's chain of grid barriers; the price is that
// every cfv block with a terminal child lives from that step on.  Each op's
// arithmetic is the same either way.
void Game::compile(int p, bool terminals_first) {
  Program& P = prog[p];
  P.ops.clear();
  P.steps.clear();
  P.groups.clear();
  auto eff = [&](size_t c) {
    while (!arena[c].terminal() && !arena[c].chance() && arena[c].nch == 1) c += arena[c].child_off;
    return c;
  };
  const size_t N = arena.size();
  std::vector<int> depth(N, -1);
  std::vector<size_t> order;
  size_t root = eff(0);
  depth[root] = 0;
  order.push_back(root);
  for (size_t k = 0; k < order.size(); ++k) {
    size_t n = order[k];
    const ArenaNode& a = arena[n];
    if (a.terminal()) continue;
    for (int c = 0; c < a.nch; ++c) {
      size_t e = eff(n + a.child_off + c);
      depth[e] = depth[n] + 1;
      order.push_back(e);
    }
  }
  int D = 0;
  for (size_t n : order) D = std::max(D, depth[n]);
  const int T = D + 1;  // terminals_first: the step of every terminal
  auto tf = [&](int d) { return d; };
  auto tb = [&](int d) { return (terminals_first ? D + 2 : D + 1) + (D - d); };
  // slot blocks
  struct Blk { int size, birth, death, base; };
  std::vector<Blk> blks;
  std::vector<int> reach_blk(N, -1), reach_idx(N, 0), rb(N, -1), cb(N, -1);
  std::vector<int> cfv_blk(N, -1), cfv_idx(N, 0);
  for (size_t n : order) {
    const ArenaNode& a = arena[n];
    if (a.terminal()) continue;
    bool chance = a.chance();
    bool opp = !chance && a.player != p;
    if (chance || opp) {
      rb[n] = (int)blks.size();
      blks.push_back({chance ? 1 : (int)a.nch, tf(depth[n]), -1, -1});
    }
    cb[n] = (int)blks.size();
    bool term_child = false;
    for (int c = 0; c < a.nch && terminals_first; ++c) term_child |= arena[eff(n + a.child_off + c)].terminal();
    blks.push_back({(int)a.nch, term_child ? T : tb(depth[n] + 1), tb(depth[n]), -1});
    for (int c = 0; c < a.nch; ++c) {
      size_t e = eff(n + a.child_off + c);
      if (chance) { reach_blk[e] = rb[n]; reach_idx[e] = 0; }
      else if (opp) { reach_blk[e] = rb[n]; reach_idx[e] = c; }
      else { reach_blk[e] = reach_blk[n]; reach_idx[e] = reach_idx[n]; }
      cfv_blk[e] = cb[n];
      cfv_idx[e] = c;
    }
  }
  int out_blk = (int)blks.size();
  blks.push_back({1, tb(0), tb(0) + 1, -1});
  cfv_blk[root] = out_blk;
  cfv_idx[root] = 0;
  for (size_t n : order) {  // reach lifetimes
    int b = reach_blk[n];
    if (b < 0) continue;
    const ArenaNode& a = arena[n];
    int use = a.terminal() ? (terminals_first ? T : tb(depth[n])) : (a.chance() || a.player != p) ? tf(depth[n]) : -1;
    blks[b].death = std::max(blks[b].death, use);
  }
  for (auto& b : blks)
    if (b.death < b.birth) b.death = b.birth;  // produced but unused
  // first-fit contiguous allocation in birth order
  std::vector<int> idx(blks.size());
  for (size_t i = 0; i < idx.size(); ++i) idx[i] = (int)i;
  std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return blks[x].birth < blks[y].birth; });
  std::vector<int> busy_until;
  for (int i : idx) {
    Blk& b = blks[i];
    int s = 0;
    for (;; ++s) {
      bool ok = true;
      for (int k = 0; k < b.size && ok; ++k)
        if (s + k < (int)busy_until.size() && busy_until[s + k] >= b.birth) ok = false;
      if (ok) break;
    }
    if ((int)busy_until.size() < s + b.size) busy_until.resize(s + b.size, -1);
    for (int k = 0; k < b.size; ++k) busy_until[s + k] = b.death;
    b.base = s;
  }
  P.num_slots = (int)busy_until.size();
  P.root_slot = blks[out_blk].base;
  auto reach_slot = [&](size_t n) -> uint16_t {
    return reach_blk[n] < 0 ? SLOT_ROOT_REACH : (uint16_t)(blks[reach_blk[n]].base + reach_idx[n]);
  };
  auto cfv_slot = [&](size_t n) { return (uint16_t)(blks[cfv_blk[n]].base + cfv_idx[n]); };
  // semantic keys of slot contents, for the verification below: reach vector
  // (block, index) or cfv vector (block, index); -1 = the opponent's weights
  auto reach_key = [&](size_t n) -> int64_t {
    return reach_blk[n] < 0 ? -1 : ((int64_t)reach_blk[n] << 17) | ((int64_t)reach_idx[n] << 1);
  };
  auto cfv_key = [&](int blk, int idx) -> int64_t { return ((int64_t)blk << 17) | ((int64_t)idx << 1) | 1; };
  // emit
  std::vector<std::vector<size_t>> at(D + 1);
  for (size_t n : order) at[depth[n]].push_back(n);
  auto push_step = [&](int begin, int ne, int nt) {
    if (ne + nt == 0) return;
    Step st{};
    st.begin = begin;
    st.n_elem = (int16_t)ne;
    st.n_term = (int16_t)nt;
    st.gbegin = (int32_t)P.groups.size();
    // runs of terminals with the same (board, reach): the leader carries the run length
    for (int i = 0; i < nt;) {
      int j = i + 1;
      Op& lead = P.ops[begin + ne + i];
      // a depth-boundary terminal always forms a run of its own: the adjoint
      // pass weights its reach by that node's boundary values
      while (j < nt && j - i < 255 && lead.term != TERM_BOUNDARY && P.ops[begin + ne + j].term != TERM_BOUNDARY &&
             P.ops[begin + ne + j].board == lead.board && P.ops[begin + ne + j].src == lead.src)
        ++j;
      lead.na = (uint8_t)(j - i);
      P.groups.push_back((uint16_t)i);
      i = j;
    }
    st.n_groups = (int16_t)(P.groups.size() - st.gbegin);
    P.steps.push_back(st);
  };
  for (int d = 0; d <= D; ++d) {
    int begin = (int)P.ops.size();
    for (size_t n : at[d]) {
      const ArenaNode& a = arena[n];
      if (a.terminal()) continue;
      Op o{};
      o.node = (uint32_t)n;
      o.na = (uint8_t)a.nch;
      o.src = reach_slot(n);
      o.dst = 0;
      if (a.chance()) {
        o.type = OP_FWD_CHANCE;
        o.blk = (uint16_t)blks[rb[n]].base;
        P.ops.push_back(o);
      } else if (a.player != p) {
        o.type = OP_FWD_OPP;
        o.blk = (uint16_t)blks[rb[n]].base;
        P.ops.push_back(o);
      }
    }
    push_step(begin, (int)P.ops.size() - begin, 0);
  }
  // terminals of the step `range` (all depths when terminals_first), runs of
  // the same (board, reach) adjacent, so a batch scans that reach once
  auto emit_terminals = [&](const std::vector<size_t>& terms_in) {
    std::vector<size_t> terms = terms_in;
    std::stable_sort(terms.begin(), terms.end(), [&](size_t x, size_t y) {
      int bx = node_board[x], by = node_board[y];
      if (bx != by) return bx < by;
      return reach_slot(x) < reach_slot(y);
    });
    for (size_t n : terms) {
      const ArenaNode& a = arena[n];
      Op o{};
      o.type = OP_TERM;
      o.node = (uint32_t)n;
      o.src = reach_slot(n);
      o.dst = cfv_slot(n);
      o.board = (uint16_t)node_board[n];
      if (a.boundary()) o.term = TERM_BOUNDARY;
      else if (a.fold()) { o.term = TERM_FOLD; o.fold_pl = a.player & PL_MASK; }
      else o.term = TERM_SHOWDOWN;
      P.ops.push_back(o);
    }
  };
  if (terminals_first) {
    std::vector<size_t> all;
    for (int d = D; d >= 0; --d)
      for (size_t n : at[d])
        if (arena[n].terminal()) all.push_back(n);
    int begin = (int)P.ops.size();
    emit_terminals(all);
    push_step(begin, 0, (int)P.ops.size() - begin);
  }
  for (int d = D; d >= 0; --d) {
    int begin = (int)P.ops.size();
    for (size_t n : at[d]) {
      const ArenaNode& a = arena[n];
      if (a.terminal()) continue;
      Op o{};
      o.node = (uint32_t)n;
      o.na = (uint8_t)a.nch;
      o.blk = (uint16_t)blks[cb[n]].base;
      o.dst = cfv_slot(n);
      o.src = reach_slot(n);
      if (a.chance()) {
        o.type = OP_BWD_CHANCE;
        o.board = (uint16_t)(chance_iso_id[n] < 0 ? 0xFFFF : chance_iso_id[n]);
      } else {
        o.type = a.player == p ? OP_BWD_TRAV : OP_BWD_OPP;
      }
      P.ops.push_back(o);
    }
    int ne = (int)P.ops.size() - begin;
    if (!terminals_first) {
      std::vector<size_t> terms;
      for (size_t n : at[d])
        if (arena[n].terminal()) terms.push_back(n);
      emit_terminals(terms);
    }
    push_step(begin, ne, (int)P.ops.size() - begin - ne);
  }
  // Verification: replay the pass step by step with the meaning of every
  // slot.  Each read must find the vector the op expects; within a step no
  // two ops write one slot and no op reads a slot another op of the step
  // writes (the ops of a step run concurrently).
  {
    std::vector<int64_t> content(P.num_slots, INT64_MIN);
    std::vector<int> wstep(P.num_slots, -1);
    P.verified = true;
    for (size_t si = 0; si < P.steps.size() && P.verified; ++si) {
      const Step& st = P.steps[si];
      std::vector<std::pair<int, int64_t>> writes;
      std::vector<std::pair<int, int64_t>> reads;
      for (int k = st.begin; k < st.begin + st.n_elem + st.n_term; ++k) {
        const Op& o = P.ops[k];
        const size_t n = o.node;
        const ArenaNode& a = arena[n];
        if (o.type == OP_FWD_OPP || o.type == OP_FWD_CHANCE || o.type == OP_TERM)
          if (o.src != SLOT_ROOT_REACH) reads.push_back({o.src, reach_key(n)});
        if (o.type == OP_FWD_OPP)
          for (int c = 0; c < a.nch; ++c) writes.push_back({o.blk + c, ((int64_t)rb[n] << 17) | ((int64_t)c << 1)});
        else if (o.type == OP_FWD_CHANCE)
          writes.push_back({o.blk, (int64_t)rb[n] << 17});
        else if (o.type == OP_TERM)
          writes.push_back({o.dst, cfv_key(cfv_blk[n], cfv_idx[n])});
        else {  // backward node ops read every child's cfv
          for (int c = 0; c < a.nch; ++c) reads.push_back({o.blk + c, cfv_key(cb[n], c)});
          writes.push_back({o.dst, cfv_key(cfv_blk[n], cfv_idx[n])});
        }
      }
      for (auto [slot, key] : reads)
        if (slot >= P.num_slots || content[slot] != key) P.verified = false;
      for (auto [slot, key] : writes) {
        if (slot >= P.num_slots || wstep[slot] == (int)si) P.verified = false;
        else wstep[slot] = (int)si;
      }
      for (auto [slot, key] : reads)
        if (slot < P.num_slots && wstep[slot] == (int)si) P.verified = false;
      for (auto [slot, key] : writes)
        if (slot < P.num_slots) content[slot] = key;
    }
    const int root_key_ok = P.root_slot >= 0 && P.root_slot < P.num_slots &&
                            content[P.root_slot] == cfv_key(out_blk, 0);
    if (!root_key_ok) P.verified = false;
  }
}

// Recompiles both traversers' programs (terminals_first: see compile).
bool Game::recompile(bool tf, std::string& err) {
  terminals_first = tf;
  compile(0, tf);
  compile(1, tf);
  if (!prog[0].verified || !prog[1].verified) { err = "tree program failed its slot verification"; return false; }
  num_slots = std::max(prog[0].num_slots, prog[1].num_slots);
  if (num_slots >= 0xFFF0) { err = "Tree too wide for the slot allocator"; return false; }
  for (int p = 0; p < 2; ++p)
    for (const auto& st : prog[p].steps)
      if (st.n_elem > 32000 || st.n_term > 32000) { err = "Tree level too wide"; return false; }
  return true;
}

bool Game::init(const float* r0, const float* r1, const uint8_t b[5], const TreeCfg& c, std::string& err) {
  cfg = c;
  std::memcpy(range[0], r0, sizeof(range[0]));
  std::memcpy(range[1], r1, sizeof(range[1]));
  flop[0] = b[0];
  flop[1] = b[1];
  flop[2] = b[2];
  turn = b[3];
  river = b[4];
  ATree t;
  if (!ATree::build(cfg, t, err)) return false;
  if (t.has_invalid_terminal()) { err = "Invalid terminal found in action tree"; return false; }
  if (!check_cards(err)) return false;
  init_isomorphism();
  build_arena(t);
  for (const auto& n : arena)
    if (!n.terminal() && !n.chance() && n.nch > kMaxActions) {
      err = "Too many actions at one node (max " + std::to_string(kMaxActions) + ")";
      return false;
    }
  return recompile(false, err);
}

}  // namespace ps
