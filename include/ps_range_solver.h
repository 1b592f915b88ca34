/*
 * ps_range_solver.h - C ABI of the B200 range solver (drop-in for the game /
 * solve path of tjennings/poker_solver_rust `crates/range-solver`).
 *
 * Every entry point replaces one reference function; the comment beside it
 * names the reference item (paths relative to crates/range-solver/src).
 * Conventions: plain pointers and sizes, host memory unless a name says
 * "device"; every function returns PS_OK (0) or a negative PS_ERR_* code and
 * never aborts the caller - the reference's panics ("Game is already solved",
 * "Game is not ready") become PS_ERR_STATE; the message of the last error on
 * the calling thread is ps_last_error().  A game owns one CUDA stream; calls
 * on one game must not overlap, different games may be used from different
 * threads.  The library requires an sm_100 GPU; there is no CPU fallback.
 */
#ifndef PS_RANGE_SOLVER_H
#define PS_RANGE_SOLVER_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PS_OK 0
#define PS_ERR_INVALID (-1)     /* invalid configuration or argument */
#define PS_ERR_STATE (-2)       /* call not allowed in the game's state */
#define PS_ERR_CUDA (-3)        /* CUDA runtime error or no usable GPU */
#define PS_ERR_UNSUPPORTED (-4) /* feature the library does not support */
#define PS_ERR_DEVICE (-5)      /* a kernel reported an error flag */

/* action_tree.rs:130-192 TreeConfig; bet sizes are the reference's strings
 * (bet_size.rs:82-112, e.g. "50%, 100%, a" / "2.5x" / "20c3r" / "2e"). */
typedef struct ps_tree_config {
  int32_t initial_state; /* BoardState: 0 flop, 1 turn, 2 river */
  int32_t starting_pot;
  int32_t effective_stack;
  int32_t depth_limit; /* -1 = None */
  double rake_rate;
  double rake_cap;
  double add_allin_threshold;
  double force_allin_threshold;
  double merging_threshold;
  const char* bet_sizes[3][2][2]; /* [flop, turn, river][oop, ip][bet, raise]; NULL = "" */
  const char* donk_sizes[2];      /* turn, river; NULL = None */
  int32_t max_bets;               /* extension, not in the reference: cap on bets + raises
                                     per street (0 = no cap, the reference behaviour) */
  int32_t reserved;
} ps_tree_config;

/* card.rs:19-32 CardConfig; ranges as range.rs:38-39 raw data (1326 weights in
 * card_pair_to_index order, each in [0, 1]); 255 = card not dealt.  The
 * weights are read during ps_game_new / ps_batch_new only and may be freed
 * when the call returns. */
typedef struct ps_card_config {
  const float* range[2];
  uint8_t flop[3];
  uint8_t turn;
  uint8_t river;
  uint8_t reserved[3];
} ps_card_config;

typedef struct ps_game ps_game;

/* ---- game lifecycle (game/interpreter.rs) ---- */
/* ActionTree::new + PostFlopGame::with_config (action_tree.rs:326, interpreter.rs:128) */
int ps_game_new(const ps_card_config* cards, const ps_tree_config* tree, ps_game** out);
void ps_game_free(ps_game* g);
/* PostFlopGame::memory_usage (interpreter.rs:188): bytes of f32 state on the device */
int ps_game_memory_usage(ps_game* g, uint64_t* bytes);
/* No counterpart in the reference.  The shape of the game's compiled tree
 * program, host-side only (no GPU needed), for sizing device memory and
 * launches: out[0] working slots, out[1] slot stride (floats), out[2..3]
 * steps of traverser 0 / 1, out[4..5] node ops of traverser 0 / 1, out[6..7]
 * terminal ops, out[8..9] terminal runs (terminals sharing one reach scan),
 * out[10] S = sum over decision edges of the acting player's hands (the
 * per-iteration state stream is 20 * S bytes), out[11] boards. */
int ps_game_program_info(ps_game* g, int64_t out[12]);
/* No counterpart in the reference.  Chooses the game's tree program before
 * allocate_memory (host-side only): 1 evaluates every terminal of a pass in
 * one step after the forward sweep, 0 the terminals of each depth in that
 * depth's backward step.  Results are the same bits either way; the first
 * has fewer long steps (one per pass) and keeps more vectors alive at once.
 * Without a choice, a game that runs in grid mode (one game of at least 16
 * nodes) takes 1 and every other game 0.  The compiler replays each program
 * against its slot assignment and rejects one that fails (PS_ERR_INVALID). */
int ps_game_set_terminals_first(ps_game* g, int enable);
/* PostFlopGame::allocate_memory (interpreter.rs:212); compression -> PS_ERR_UNSUPPORTED */
int ps_game_allocate_memory(ps_game* g, int enable_compression);

/* ---- solver (solver.rs, utility.rs) ---- */
/* solve (solver.rs:108): DCFR until max_iter or exploitability <= target (chips) */
int ps_solve(ps_game* g, uint32_t max_iter, float target, int print_progress, float* out_exploitability);
/* number of iterations the last ps_solve ran */
int ps_last_iterations(ps_game* g, uint32_t* out);
/* solve_step (solver.rs:184) */
int ps_solve_step(ps_game* g, uint32_t current_iteration);
/* compute_exploitability (utility.rs:380), chips */
int ps_compute_exploitability(ps_game* g, float* out);
/* No counterpart in the reference.  The same value as
 * ps_compute_exploitability, for callers that cannot allocate device memory
 * when they call it (an engine that hands plug-ins a fixed share of GPU memory
 * reserved at start-up, or a latency-bound thread that must not take
 * cudaMalloc's implicit device synchronisation): it allocates nothing and uses
 * a fixed 16 MiB device array of the library for its working slots.  Games
 * whose slots need more than that (4 Mi floats = num_slots x slot stride) get
 * PS_ERR_INVALID: river trees fit with room to spare, turn trees usually do
 * not (every river subtree is live at once; 100bb turn trees with one or two
 * sizes need 10-15 Mi floats) and stay on ps_compute_exploitability.  The
 * array is part of the library's device code: every device that loads the
 * library reserves its 16 MiB until the process exits, whether or not this
 * function is called.  The first call in a CUDA context looks the array up,
 * so make it before any stream capture on that device; after a device reset
 * (a new context) the next call looks it up again.  Each call waits for its
 * kernel and reads the result back before it returns.  All calls share the
 * one array: calls whose kernels overlap on the GPU (different games on
 * different streams or threads) race and must be serialised by the caller. */
int ps_compute_exploitability_noalloc(ps_game* g, float* out);
/* finalize (utility.rs:348) */
int ps_finalize(ps_game* g);
/* root_cfvalues_with_reach (utility.rs:422); opp_reach NULL = initial weights (root_cfvalues, :407) */
int ps_root_cfvalues_with_reach(ps_game* g, int player, const float* opp_reach, float* out);

/* ---- fixed-strategy evaluation and its adjoint ----
 * No counterpart in the reference, which has no gradients.  With the average
 * strategy held fixed, cfv_p (root cfvalues of player p, the values of
 * root_cfvalues_with_reach, utility.rs:422) is linear in the opponent's
 * initial weights and in p's boundary values.  These entry points take the
 * weights as arguments (solver hand order, H_p values each) instead of the
 * game's; games with isomorphic chance pruning get PS_ERR_UNSUPPORTED. */
/* forward: cfv0 = cfv_0(w1, B), cfv1 = cfv_1(w0, B) */
int ps_eval_fixed_strategy(ps_game* g, const float* w0, const float* w1, float* cfv0, float* cfv1);
/* vector-Jacobian product for cotangents g0, g1 on cfv0, cfv1 (NULL = zero):
 * dw0 = g1 . dcfv1/dw0, dw1 = g0 . dcfv0/dw1 (cfv_p does not depend on w_p), and
 * dbcfv = d(g0 . cfv0 + g1 . cfv1)/dB laid out per boundary ordinal k as
 * [H0 values for player 0][H1 values for player 1] (NULL = not wanted) */
int ps_eval_fixed_strategy_adjoint(ps_game* g, const float* w0, const float* w1, const float* g0, const float* g1,
                                   float* dw0, float* dw1, float* dbcfv);
/* The same two calls with every array in device memory of the game's device
 * when on_device = 1 (host memory when 0): a trainer keeps its tensors on the
 * GPU, and nothing passes through the host.  The call does not wait for
 * other streams: the work that writes the inputs must be finished before it;
 * the results are complete when it returns. */
int ps_eval_fixed_strategy_ex(ps_game* g, const float* w0, const float* w1, float* cfv0, float* cfv1,
                              int32_t on_device);
int ps_eval_fixed_strategy_adjoint_ex(ps_game* g, const float* w0, const float* w1, const float* g0,
                                      const float* g1, float* dw0, float* dw1, float* dbcfv, int32_t on_device);
/* Every boundary value of the game in one call (set_boundary_cfvs,
 * interpreter.rs:343, for each ordinal and player): values [n_boundary][H0 +
 * H1], per ordinal player 0's H0 values then player 1's; device memory when
 * on_device = 1. */
int ps_set_boundary_cfvs_all(ps_game* g, const float* values, int32_t on_device);

/* ---- game data (game/mod.rs, interpreter.rs) ---- */
int ps_num_private_hands(ps_game* g, int player);
int ps_private_cards(ps_game* g, int player, uint8_t* out_pairs);  /* private_cards(): [H][2] */
int ps_initial_weights(ps_game* g, int player, float* out);
double ps_num_combinations(ps_game* g);
int64_t ps_num_nodes(ps_game* g);
/* node fields: player, amount, turn, river, num_children, children_offset, prev kind, prev amount */
int ps_node_info(ps_game* g, int64_t node, int32_t out[8]);
int ps_child_indices(ps_game* g, int64_t node, int64_t* out, int cap); /* query.rs:475 */
int ps_strategy_at_index(ps_game* g, int64_t node, float* out);     /* query.rs:386 */
/* raw per-node storage: 1 cumulative strategy, 2 regrets (cfvalues after finalize),
 * 3 IP cfvalues, 4 chance cfvalues; returns the element count */
int64_t ps_node_storage(ps_game* g, int64_t node, int which, float* out);
/* writes one node's storage (which = 1 cumulative strategy, 2 regrets), rows of
 * H_actor values per action - the general form of seed_strategy (query.rs:438-469) */
int ps_seed_node_storage(ps_game* g, int64_t node, int which, const float* values, int64_t n);
int ps_same_hand_index(ps_game* g, int player, uint16_t* out);      /* game/mod.rs:288 */
/* hand strength order for board (turn, river) as computed on the device:
 * ascending (strength, index) items incl. the (0,0) / (65535,65535) sentinels
 * (card.rs:163-226); returns the item count */
int ps_hand_strength(ps_game* g, int turn, int river, int player, uint16_t* strength, uint16_t* index);
/* valid_indices for a board (card.rs:81-156); returns the count */
int ps_valid_indices(ps_game* g, int turn, int river, int player, uint16_t* out);

/* ---- depth boundary (interpreter.rs:307-534) ---- */
int64_t ps_num_boundary_nodes(ps_game* g);
int ps_boundary_node_indices(ps_game* g, int64_t* out);
int ps_set_boundary_cfvs(ps_game* g, int64_t ordinal, int player, const float* cfvs, int64_t n);
/* reach of each player at every boundary under the average strategy from the
 * initial weights (compute_reach_at_nodes, gpu-range-solver batch.rs:765-790;
 * the range solver's boundary_reach, evaluation.rs:97, holds the same vector
 * after an average-strategy pass); laid out per ordinal k as [H0 values of
 * player 0][H1 values of player 1] */
int ps_boundary_reach(ps_game* g, float* out);

/* ---- turn datagen: boundary values from network outputs ----
 * The reach-weighted average over the 48 river cards with card blocking of
 * cfvnet/src/datagen/gpu_boundary_eval.rs:207-269, on the device.  n boundary
 * items (a request's boundaries, flattened), each with its 4-card board
 * (host [n][4]), pot and effective stack (host [n]).  Device arrays:
 *   net   [n][2][48][1326]  network outputs per player, river (the 48 cards not on
 *                           the board, ascending) and combo (card_pair_to_index order);
 *                           f32, or bf16 when net_bf16
 *   reach [n][2][1326]      OOP and IP reach at the boundary, combo order
 *   hands [H]               combo index of each output hand
 *   out   [n][2][H]         player 0 averaged with IP-reach weights, player 1 with OOP
 * stream: a cudaStream_t (NULL = the default stream); returns after the work is done. */
int ps_boundary_river_reduce(int32_t n, const uint8_t* boards, const float* pots, const float* stacks,
                             const void* net, int32_t net_bf16, const float* reach, const int32_t* hands, int32_t H,
                             float* out, void* stream);
/* The first Linear layer (h outputs over the 2720 inputs) of a boundary
 * network for every input row that ps_boundary_encode would write, without
 * writing those rows (no reference counterpart; the reference runs the layer
 * on the materialised rows, gpu_boundary_eval.rs:164-197).  A river card's row
 * differs from the unmasked reach only in the 51 combos holding that card, so
 *   row(i, p, r) = base[i] - percard[i][r] + the board, rank, pot, stack and
 *                  player columns + bias,
 * with base [n][h] = W[:, :2652] [oop | ip] and percard [n][52][h] = the same
 * product over the combos holding each card (both from the caller's GEMMs),
 * wcols [68][h] = W[:, 2652:] transposed, bias [h] or null; h <= 8192.
 * boards, pots, stacks: host; the rest device; out [n][2][48][h], f32 or bf16. */
int ps_boundary_first_layer(int32_t n, const uint8_t* boards, const float* pots, const float* stacks,
                            const float* base, const float* percard, const float* wcols, const float* bias, int32_t h,
                            void* out, int32_t out_bf16, void* stream);

/* ---- navigation and queries (game/query.rs) ---- */
int ps_back_to_root(ps_game* g);
int ps_play(ps_game* g, int64_t action); /* action = -1: first possible card */
int ps_available_actions(ps_game* g, int32_t* kinds, int32_t* amounts, int cap);
int ps_is_terminal_node(ps_game* g);
int ps_is_chance_node(ps_game* g);
int ps_current_player(ps_game* g);
int64_t ps_current_node_index(ps_game* g);
uint64_t ps_possible_cards(ps_game* g);
int ps_strategy(ps_game* g, float* out); /* returns the element count */
int ps_cache_normalized_weights(ps_game* g);
int ps_weights(ps_game* g, int player, int normalized, float* out);
int ps_expected_values(ps_game* g, int player, int detail, float* out); /* returns count */
int ps_total_bet_amount(ps_game* g, int32_t out[2]);

/* ---- checkpoint (storage_buffers / set_storage_buffers, interpreter.rs:265-300) ---- */
int ps_state_export(ps_game* g, void* buf, uint64_t cap, uint64_t* needed);
int ps_state_import(ps_game* g, const void* buf, uint64_t size);

/* ---- batched solve (replaces per-spot GpuBatchSolver launches,
 *      crates/gpu-range-solver/src/batch.rs:79-610) ---- */
typedef struct ps_batch ps_batch;
typedef struct ps_batch_opts {
  int32_t block_threads;  /* threads per CTA, a multiple of 32 up to 256 (0 = default 256,
                             -1 = autotune: time each shape on a sample of the batch) */
  int32_t ctas_per_sm;    /* 0 = as many as fit */
  int32_t sort_by_cost;   /* 1 = hand out the largest spots first */
  int32_t stage_tables;   /* 1 = copy a spot's board tables to shared memory, 0 = read them
                             from global memory, -1 = default (0) */
  int32_t scan_buffers;   /* warps per CTA that evaluate terminal runs, each with a shared-memory
                             scan buffer of 12 bytes per hand (0 = half the warps; the
                             autotuner then also tries all of them) */
  int32_t instances_per_cta; /* spots of one tree shape a CTA solves in lockstep, 1..4
                                (0 = 1); they share each step's barrier */
  int32_t scheduler;      /* PS_SCHED_DEFAULT (0): dataflow for batches of more spots than SMs,
                             step-synchronous otherwise; PS_SCHED_STEP (1): every CTA walks
                             its spot's steps with one barrier per step (k_solve);
                             PS_SCHED_FLOW (2): each CTA holds several spots at once and its
                             warps take the ready items of any of them (k_flow).  Results
                             are the same bits either way. */
  int32_t flow_threads;   /* dataflow: threads per CTA, a multiple of 32 from 128 to 1024
                             (0 = 1024; with block_threads = -1 the autotuner chooses) */
  int32_t flow_spots_per_cta; /* dataflow: spots a CTA holds at once, 1..8 (0 = 3, or autotuned) */
  int32_t node_parts;     /* dataflow: column blocks each node op is cut into, 1..16
                             (0 = 3, or autotuned) */
} ps_batch_opts;
#define PS_SCHED_DEFAULT 0
#define PS_SCHED_STEP 1
#define PS_SCHED_FLOW 2
int ps_batch_new(const ps_card_config* cards, const ps_tree_config* trees, int32_t n,
                 const ps_batch_opts* opts, ps_batch** out);
void ps_batch_free(ps_batch* b);
/* one persistent launch: every spot runs solve() to max_iter or target[i] chips */
int ps_batch_solve(ps_batch* b, uint32_t max_iter, const float* target_chips);
int ps_batch_results(ps_batch* b, float* exploitability, int32_t* iterations);
int ps_batch_root_strategy(ps_batch* b, int32_t spot, float* out); /* returns count */
/* per-spot state after a solve (replaces extract_results, batch.rs:587-609,
 * which downloads the strategy sums): nodes in the arena order of
 * ps_num_nodes / ps_node_info for the same spot; ps_batch_node_storage gives a
 * decision node's [A][H_actor] rows, which = 1 strategy sums, 2 regrets, as
 * ps_node_storage does for a single game; returns the count (0 for terminal
 * and chance nodes) */
int64_t ps_batch_num_nodes(ps_batch* b, int32_t spot);
int64_t ps_batch_node_storage(ps_batch* b, int32_t spot, int64_t node, int which, float* out);
/* root cfvalues of `player` under the average strategy after the last
 * ps_batch_solve, computed on the device at the end of each spot's solve
 * (replaces compute_evs_from_strategy_sum, gpu-range-solver batch.rs:799-933);
 * H_player values, returns the count */
int ps_batch_root_cfvalues(ps_batch* b, int32_t spot, int player, float* out);
/* device time in ms of the last ps_batch_solve (setup excluded / included) */
int ps_batch_last_timing(ps_batch* b, float* solve_ms, float* setup_ms);
/* algorithmic bytes of one DCFR iteration of spot i: 20 * sum_edges H_actor */
double ps_batch_iteration_bytes(ps_batch* b, int32_t spot);
int ps_batch_config(ps_batch* b, int32_t* block_threads, int32_t* grid, int32_t* ctas_per_sm);
/* the trials of the last autotune (block_threads = -1): CTA size, scan-buffer warps
 * and device ms of the fixed trial work each; returns the count (0 when the choice
 * came from the cache or was given) */
int ps_batch_autotune_log(ps_batch* b, int32_t* block_threads, int32_t* scan_buffers, float* trial_ms, int cap);
/* scan-buffer warps per CTA the batch runs with */
int ps_batch_scan_buffers(ps_batch* b);
/* the launch shape of the batch's solves: out[0] scheduler (PS_SCHED_STEP or
 * PS_SCHED_FLOW), [1] threads per CTA, [2] CTAs, [3] CTAs per SM, [4]
 * scan-buffer warps per CTA, [5] spots per CTA, [6] node-op parts, [7] 1 when
 * a single spot runs in grid mode (every SM on it), 2 when it runs on the CTAs
 * of one thread-block cluster */
int ps_batch_schedule(ps_batch* b, int32_t out[8]);
/* No counterpart in the reference.  The launch shape of a single game's
 * solves, as ps_batch_schedule; in grid mode out[2] is the CTAs of the grid
 * (or of the cluster).  PS_ERR_STATE before allocate_memory. */
int ps_game_schedule(ps_game* g, int32_t out[8]);
/* the trials of the last autotune: per trial 4 values (threads per CTA,
 * scan-buffer warps, spots per CTA, node-op parts; the last two 0 for a
 * step-synchronous trial) and its device ms; returns the count.  A dataflow
 * autotune lists its sweep (every shape, 6 iterations on one wave of sample
 * spots) and, once the batch's first fresh ps_batch_solve has run, the refine
 * runs of the shapes within 6% of the sweep's best (that solve's targets and
 * iteration limit on four waves of spots); a shape's second entry is its
 * refine run, and the fastest refine run is the choice. */
int ps_batch_autotune_trials(ps_batch* b, int32_t* shape, float* trial_ms, int cap);
/* bytes copied host->device by ps_batch_new and device->host by ps_batch_results */
int ps_batch_io_bytes(ps_batch* b, uint64_t* h2d, uint64_t* d2h);

/* ---- batched depth-limited solving (turn datagen with boundary values:
 *      gpu-range-solver batch.rs:279-585 set_leaf_injection / run_iterations /
 *      download_reach / update_leaf_cfvs, driven by cfvnet
 *      datagen/domain/pipeline.rs:648-700) ----
 * A boundary item is one depth boundary of one spot: items are listed spot by
 * spot, ordinals ascending.  Per-item arrays use the 1326-combo layout
 * (card_pair_to_index, card.rs:50-55), [items][2][1326], row p = player p. */
#define PS_EPI_ROOT 1 /* root cfvalues + boundary reach under the average strategy */
#define PS_EPI_EXPL 2 /* exploitability of every spot (ps_batch_results) */
/* DCFR iterations [t0, t1) of every spot from the current state, no
 * exploitability checks (batch.rs:414 run_iterations), in one launch; then the
 * epilogue bits.  The first call after ps_batch_new or ps_batch_reset starts
 * from zero regrets and strategy sums. */
int ps_batch_run_iterations(ps_batch* b, uint32_t t0, uint32_t t1, int32_t epilogue);
/* the next ps_batch_run_iterations starts from zero state (boundary values stay) */
int ps_batch_reset(ps_batch* b);
int64_t ps_batch_num_boundary_items(ps_batch* b);
/* per item: spot, ordinal, the spot's 4-card board, the boundary node's pot
 * (starting_pot + 2 * amount) and the stack behind it (effective_stack - amount);
 * any pointer may be null */
int ps_batch_boundary_items(ps_batch* b, int32_t* spot, int32_t* ordinal, uint8_t* boards, float* pots,
                            float* stacks);
/* boundary values of every item, [items][2][1326]; each spot takes the entries
 * of its own hands (replaces update_leaf_cfvs, batch.rs:557-585, with the
 * semantics of set_boundary_cfvs, interpreter.rs:343).  on_device = 1: a
 * device pointer whose values are ready; the call returns once they are
 * consumed.  Values are zero until set. */
int ps_batch_set_boundary_cfvs(ps_batch* b, const float* values, int32_t on_device);
/* each player's reach at every boundary under the average strategy as of the
 * last PS_EPI_ROOT epilogue (or ps_batch_solve), [items][2][1326], 0 outside
 * the spot's hands (replaces download_reach + compute_reach_at_nodes,
 * batch.rs:537-555, :765-790) */
int ps_batch_boundary_reach(ps_batch* b, float* out, int32_t on_device);
/* both players' root cfvalues of every spot under the average strategy as of
 * the last PS_EPI_ROOT epilogue, ps_batch_solve or ps_batch_adjoint, [n][2][1326]
 * (0 outside the spot's hands) */
int ps_batch_root_cfvalues_all(ps_batch* b, float* out, int32_t on_device);
/* batched fixed-strategy evaluation and its adjoint: ps_eval_fixed_strategy_adjoint
 * (no reference counterpart; the adjoint of utility.rs:422-443) for every spot at
 * once, with each spot's initial weights and its average strategy held fixed.
 * cot [n][2][1326]: dL/d(root cfvalues of player p).  Refreshes the root
 * cfvalues; dw [n][2][1326]: dL/d(initial weights of player p); dB
 * [items][2][1326]: dL/d(boundary values).  dw or dB may be null.  Spots with
 * isomorphic chance pruning: PS_ERR_UNSUPPORTED. */
int ps_batch_adjoint(ps_batch* b, const float* cot, float* dw, float* dB, int32_t on_device);
/* training records of every spot (cfvnet datagen/storage.rs:5-57 format, two
 * per spot: player 0 then 1) from the root cfvalues of the last ps_batch_solve
 * or PS_EPI_ROOT epilogue, with the values of the GPU river datagen
 * (datagen/domain/pipeline.rs:353-411): cfvs = (root cfvalue * num_combinations
 * - pot/2) / (pot/2) on the player's hands, valid_mask = either player's hands,
 * game_value = sum(range * cfvs) in f32; replaces compute_evs_from_strategy_sum
 * + the record assembly.  All spots need the same board size.
 * ps_batch_record_bytes: the size of the packed records. */
int64_t ps_batch_record_bytes(ps_batch* b);
int ps_batch_records(ps_batch* b, uint8_t* out, int32_t on_device);
/* ---- situation sampling (cfvnet datagen/sampler.rs:30-60, :142-205 and
 *      range_gen.rs:18-167) ---- */
typedef struct ps_sampler_config {
  int32_t board_size;          /* 4 (turn) or 5 (river) */
  int32_t initial_stack;       /* chips (config.rs:72, default 200) */
  int32_t num_pot_intervals;   /* 1..16 */
  const int32_t* pot_intervals; /* [k][2], [lo, hi) (config.rs:151, default [[4,20],[20,80],[80,200],[200,400]]) */
  int32_t num_spr_intervals;   /* 0..16; 0 = pot, then stack uniform in [5, initial_stack - pot/2] */
  const double* spr_intervals; /* [k][2], [lo, hi): SPR bucket first, then a feasible pot bucket */
  uint64_t seed;
} ps_sampler_config;
/* situations first .. first + n - 1 of the seed's stream, on the device: a
 * board of board_size distinct cards (boards [n][5], unused slots 0), pot and
 * effective stack (pots, stacks [n]), and the OOP and IP ranges [n][2][1326]
 * drawn by the R(S,p) procedure over the combos ordered by hand strength (each
 * sums to 1, board-blocked combos 0).  The draws come from a counter-based
 * SplitMix64 stream instead of the reference's ChaCha8: same distributions,
 * different numbers.  Output pointers are device memory; stream: a
 * cudaStream_t or null. */
int ps_sample_situations(const ps_sampler_config* cfg, int64_t first, int32_t n, uint8_t* boards, int32_t* pots,
                         int32_t* stacks, float* ranges, void* stream);
/* boundary-network input rows (cfvnet eval/boundary_evaluator.rs:27-60, rows
 * ordered as gpu_boundary_eval.rs:164-185): for each of n items, player and
 * river card not on the board, 2720 values: oop reach | ip reach (zeroed where
 * a hand holds the river) | 52 board one-hot | 13 rank presence |
 * pot/(pot+stack) | stack/(pot+stack) | player.  boards [n][4], pots, stacks:
 * host; reach [n][2][1326] and out [n][2][48][2720]: device (f32, or bf16 when
 * out_bf16).  stream: a cudaStream_t or null */
int ps_boundary_encode(int32_t n, const uint8_t* boards, const float* pots, const float* stacks, const float* reach,
                       void* out, int32_t out_bf16, void* stream);

/* ---- misc ---- */
/* BetSizeOptions::try_from one list (bet_size.rs:82-112): per entry the kind
 * (0 PotRelative, 1 PrevBetRelative, 2 Additive, 3 Geometric, 4 AllIn), its
 * float (ratio / max ratio), int (adder / streets) and raise cap; returns the
 * count */
int ps_parse_bet_sizes(const char* sizes, int is_raise, int32_t* kinds, double* values, int32_t* ints,
                       int32_t* caps, int cap);
const char* ps_last_error(void);
int ps_hand_table(int32_t* out, int cap); /* hand_table.rs values as built here */
int ps_discount_params(uint32_t t, float out[3]); /* solver.rs:26-44 */

/* ---- test hooks (no reference counterpart) ---- */
/* The bounded grid barrier of single-game grid mode: a cooperative launch of
 * `ctas` CTAs (2 to the SM count) in which CTA 0 enters `rounds` grid barriers
 * that no other CTA joins.  The first wait gives up after wait_ns nanoseconds
 * (at most 1 s) and sets the launch's error word to 4 (a barrier gave up) and
 * its abort word; every later barrier then returns at once.  With all_join = 1
 * every CTA enters the barriers instead, so none runs out and the kernel time
 * divided by rounds is the cost of one grid barrier.  Out: the error word, the
 * number of barriers CTA 0 got through and the kernel's time in ms.  No
 * kernel of this call waits without a bound. */
int ps_debug_grid_barrier_timeout(int32_t ctas, int32_t rounds, int64_t wait_ns, int32_t all_join, int32_t* err,
                                  int32_t* passed, float* ms);

#ifdef __cplusplus
}
#endif
#endif
