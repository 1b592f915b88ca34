// Host-callable launchers of the kernels in ps_kernels.cu and the shared
// memory plan they share with the host.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>

#include "ps_device.hpp"

namespace ps {

__host__ __device__ inline int head_words(int hs) { return (3 * hs + 31) / 32; }
// bitmap words rounded up to 16 bytes, so staged gather lists stay 16-byte aligned
__host__ __device__ inline int head_words16(int hs) { return (head_words(hs) + 3) & ~3; }

// Board tables of one board staged in shared memory: lookup records (16 bytes
// per hand), segment-start bitmaps and gather lists (u16, 3 * hs per player).
__host__ __device__ inline int table_bytes_for(int hs0, int hs1) {
  int b = 16 * (hs0 + hs1) + 4 * (head_words16(hs0) + head_words16(hs1)) + 2 * (3 * hs0 + 3 * hs1);
  return (b + 15) & ~15;
}

// A terminal scan buffer: four zero floats (what an empty prefix reads), then
// the 3V entries of the gathered list, rounded up to whole float4s.
constexpr int kScanBase = 4;
__host__ __device__ inline int scan_buf_floats(int vstride) { return 3 * vstride + 2 * kScanBase; }

// Shared-memory plan of one solve CTA (computed on the host per launch): one
// terminal scan buffer (scan_buf_floats(vstride) floats) per scan warp,
// optional staged board tables, and a small reduction area.
struct SmemPlan {
  int vstride;  // max slot stride of the launch (floats)
  int hs_max;   // max padded hand count
  int warps;    // warps per CTA
  int bufs;     // warps 0 .. bufs-1 own a terminal scan buffer and evaluate the terminal runs
  int tables;   // bytes reserved for staged board tables (0 = tables stay in global memory)
  int split = 0; // 1: a lone spot's node ops may be split over idle warps (launches with fewer spots
                 // than SMs and grid mode, where latency is not hidden by other CTAs; same results)
  __host__ __device__ size_t total() const {
    return (size_t)tables + (size_t)bufs * scan_buf_floats(vstride) * 4 + 32 * 8;
  }
};

constexpr int kMaxSolveBlock = 256;  // threads per CTA the solve kernels are compiled for (launch bounds)
size_t setup_smem_bytes();
int solve_occupancy(int block, const SmemPlan& plan);
// Grid mode for one large spot: the work of one cooperative launch of k_grid
// (every CTA on the same spot), the number of CTAs that can be co-resident for
// it, and the launch.  bar: 4 unsigned (barrier count, generation, abort
// word), gred: 4 double, both device memory.
enum GridKind { GRID_SOLVE = 0, GRID_ITERATE = 1, GRID_EXPL = 2, GRID_FINALIZE = 3, GRID_AVERAGE = 4 };
struct GridJob {
  int kind;
  int t0, t1;              // iteration range (GRID_ITERATE) / max iterations (GRID_SOLVE)
  float target;            // GRID_SOLVE: stop once exploitability <= target
  int player, owner;       // GRID_AVERAGE: traverser and payoff owner (-1 = the traverser)
  const float* root_reach; // GRID_AVERAGE: opponent reach at the root (null = initial weights)
  float* bgrad;            // GRID_AVERAGE: boundary gradient buffer or null
  float* out;              // GRID_AVERAGE: root values [H_player]
  float* breach = nullptr; // GRID_AVERAGE: boundary reach buffer or null
  long long wait_ns = 1000000000LL;  // a grid barrier's wait limit before the launch aborts with ERR_WAIT
  int cluster = 0;                   // set by launch_grid: the CTAs form one cluster (hardware barrier)
};
int grid_ctas(int block, const SmemPlan& plan);
// Reach-weighted 48-river average of boundary-network outputs (ps_datagen.cu):
// boards [n][4], denorm [n] (pot + stack), net [n][2][48][1326] (f32, or bf16
// when net_bf16), reach [n][2][1326], hands [H] combo indices, out [n][2][H];
// all device pointers.
cudaError_t launch_boundary_river_reduce(int n, const uint8_t* boards, const float* denorm, const void* net,
                                         int net_bf16, const float* reach, const int32_t* hands, int H, float* out,
                                         cudaStream_t s);
// First layer of a boundary network over every input row of
// launch_boundary_encode without the rows: base [n][h] (weights times the
// reach rows), percard [n][52][h] (weights times the reach of the combos
// holding each card), wcols [68][h] (the board, rank, pot, stack and player
// columns), bias [h] or null; out [n][2][48][h], f32 or bf16; h at most
// kMaxFirstLayerWidth (its row part stays in shared memory).
constexpr int kMaxFirstLayerWidth = 8192;
cudaError_t launch_boundary_first_layer(int n, const uint8_t* boards, const float* pots, const float* stacks,
                                        const float* base, const float* percard, const float* wcols,
                                        const float* bias, int h, void* out, int bf16, cudaStream_t s);
// Boundary items of a batch (item = (spot, boundary ordinal)) in the 1326-combo
// layout (card.rs:50-55 index), [items][2][1326], against each spot's hand-order
// buffers.  which: BC_SET_VALUES gathers `in` into sp.bcfv; BC_REACH / BC_GRAD
// scatter sp.breach / sp.bgrad into `out` (combos outside the spot's hand list
// read 0).
enum { BC_SET_VALUES = 0, BC_REACH = 1, BC_GRAD = 2 };
cudaError_t launch_boundary_combo(const SpotDev* spots, const int2* items, int nitems, int which,
                                  const float* in, float* out, cudaStream_t s);
// Per-spot vectors of a batch in the combo layout, [n][2][1326]: SC_ROOT and
// SC_DW scatter sp.root_out / sp.adj_dw into `out`; SC_COT gathers `in` into
// sp.adj_g.
enum { SC_ROOT = 0, SC_COT = 1, SC_DW = 2 };
cudaError_t launch_spot_combo(const SpotDev* spots, int n, int which, const float* in, float* out,
                              cudaStream_t s);
// Boundary-network input rows (cfvnet eval/boundary_evaluator.rs:27-60) for
// every item, player and river card not on the item's board: [n][2][48][2720],
// oop reach | ip reach (1326 each, zeroed where a hand holds the river card) |
// 52 board one-hot | 13 rank presence | pot/(pot+stack) | stack/(pot+stack) | player.
// boards [n][4], pots [n], stacks [n], reach [n][2][1326]; device pointers;
// out is f32, or bf16 (round to nearest even) when bf16 != 0.
constexpr int kBoundaryInput = 2720;
cudaError_t launch_boundary_encode(int n, const uint8_t* boards, const float* pots, const float* stacks,
                                   const float* reach, void* out, int bf16, cudaStream_t s);
// Per-spot fields of a training record that the device descriptor lacks.
struct RecordMeta {
  float pot, stack;   // starting pot and effective stack
  uint8_t board[5];
  uint8_t board_size; // 3, 4 or 5
  uint8_t pad[2];
};
// Packed training records (cfvnet datagen/storage.rs) of every spot from its
// root cfvalues (sp.root_out): 2n records, spot by spot, player 0 then 1.
// ranges [n][2][1326] are the spots' input ranges; all device pointers.
cudaError_t launch_pack_records(const SpotDev* spots, int n, const float* ranges, const RecordMeta* meta,
                                uint8_t* out, cudaStream_t s);
// Situation sampler (ps_sampler.cu): the datagen configuration of
// cfvnet config.rs:150-160 (pot intervals [lo, hi), optional SPR intervals,
// initial stack) for situations first .. first + n - 1 of the seed's stream.
constexpr int kMaxSamplerIntervals = 16;
struct SamplerParams {
  int board_size, initial_stack, npot, nspr;
  int pot[kMaxSamplerIntervals][2];
  double spr[kMaxSamplerIntervals][2];
  uint64_t seed;
  int64_t first;
};
// boards [n][5] (unused slots 0), pots [n], stacks [n], ranges [n][2][1326]
// (OOP, IP); err is set to 1 when a situation cannot be drawn (the SPR
// rejection exhausted); all device pointers.
cudaError_t launch_sample_situations(const SamplerParams& P, int n, uint8_t* boards, int32_t* pots, int32_t* stacks,
                                     float* ranges, int* err, cudaStream_t s);
// cluster = 0: a cooperative launch of `grid` CTAs whose steps end in the
// software grid barrier; cluster = 1: one thread-block cluster of `grid` CTAs
// (at most 16) whose steps end in the hardware cluster barrier.
cudaError_t launch_grid(const SpotDev* spot, const GridJob& job, const Discount* disc, float* scratch,
                        size_t scratch_floats, float* out_expl, int* out_iters, unsigned* bar, double* gred,
                        int* err, int grid, int block, const SmemPlan& plan, cudaStream_t s, int cluster = 0);
// CTAs of one cluster launch of k_grid that fit the device at once (0 = none)
int grid_cluster_fits(int ctas, int block, const SmemPlan& plan);
cudaError_t launch_setup(const SpotDev* spots, const int2* work, int nwork, const int32_t* table, int* err,
                         int grid, cudaStream_t s);
// Work of one persistent batched-solve launch.
//   checks = 1: the reference's solve loop over iterations [0, t1): exploitability
//     before the first iteration, after every fifth and after the last one; a
//     spot stops at the first check that meets its target (t0 must be 0).
//   checks = 0: iterations [t0, t1) for every spot, no checks (the reference
//     GPU batch's run_iterations); EPI_EXPL adds one exploitability at the end.
//   EPI_ROOT: afterwards, both players' root cfvalues under the average
//     strategy into sp.root_out; spots with a boundary-reach buffer (sp.breach)
//     also record each player's reach at every depth boundary in the same passes.
//   adjoint = 1 (no iterations): the fixed-strategy evaluation under the
//     average strategy from the spots' weights (sp.root_out) and its adjoint
//     from the cotangents sp.adj_g (sp.adj_dw, sp.bgrad zeroed beforehand).
enum { EPI_ROOT = 1, EPI_EXPL = 2 };
struct SolveJob {
  int t0, t1;
  int checks;
  int epilogue;
  int adjoint = 0;
};
// Persistent batched solve over `ninst` instances of K spots (inst: [ninst][K]
// spot ids, -1 = empty); scratch holds K * scratch_floats floats per CTA.
cudaError_t launch_solve(const SpotDev* spots, int ninst, int K, const int* inst, int* counter,
                         const Discount* disc, const SolveJob& job, const float* target, float* scratch,
                         size_t scratch_floats, float* out_expl, int* out_iters, int* err, int grid, int block,
                         const SmemPlan& plan, cudaStream_t s);
// Dataflow batched solve (k_flow): each CTA holds `lanes` spots at once, each
// at its own step; warps claim the steps' items (terminal runs; node ops cut
// into node_parts column blocks) instead of waiting at per-step barriers.
// The same jobs as launch_solve except the adjoint; inst: [ninst] spot ids in
// the order they are handed out; scratch holds lanes * scratch_floats floats
// per CTA.  Results equal launch_solve's bit for bit.
constexpr int kMaxFlowThreads = 1024;
constexpr int kMaxFlowLanes = 8;
cudaError_t launch_flow(const SpotDev* spots, int ninst, const int* inst, int* counter, const Discount* disc,
                        const SolveJob& job, const float* target, float* scratch, size_t scratch_floats,
                        float* out_expl, int* out_iters, int* err, int grid, int block, int lanes, int node_parts,
                        const SmemPlan& plan, cudaStream_t s);
int flow_occupancy(int block, const SmemPlan& plan);  // CTAs per SM (0 = does not fit)
cudaError_t launch_iterate(const SpotDev* spots, int nspots, const Discount* disc, int t0, int t1,
                           float* scratch, size_t scratch_floats, int* err, int grid, int block,
                           const SmemPlan& plan, cudaStream_t s);
cudaError_t launch_exploitability(const SpotDev* spots, int nspots, float* scratch, size_t scratch_floats,
                                  float* out, int* err, int grid, int block, const SmemPlan& plan, cudaStream_t s);
cudaError_t launch_average(const SpotDev* spots, int nspots, int save, int player, const float* root_reach,
                           float* scratch, size_t scratch_floats, float* out, int* err, int grid, int block,
                           const SmemPlan& plan, cudaStream_t s, int owner = -1,
                           float* bgrad = nullptr, float* breach = nullptr);
cudaError_t launch_eval_terminal(const SpotDev* spots, Op op, int player, float* scratch, size_t scratch_floats,
                                 int* err, int block, const SmemPlan& plan, cudaStream_t s);

// Exploitability of one game with its working slots in a fixed, statically
// sized device array instead of allocated memory.  The array holds a 256-byte
// header (result and error flag) and kFixedScratchFloats floats of slots
// (16 MiB); a game needs num_slots * vstride of them.  The first call in a
// CUDA context looks up the array's address (cudaGetSymbolAddress) with that
// context's device current; a device reset ends the context, and the next
// call looks the address up again in the new one.  Every call uses the same
// array: calls whose kernels overlap on the GPU overwrite each other's slots.
constexpr size_t kFixedScratchHeader = 64;
constexpr size_t kFixedScratchFloats = (size_t)4 << 20;
cudaError_t launch_exploitability_fixed(const SpotDev* spot, size_t slot_floats, int block, const SmemPlan& plan,
                                        cudaStream_t s, float* host_out, int* host_err);

// Unique id of the CUDA context current on the calling thread (the driver's
// cuCtxGetId, which never repeats within a process, unlike a context handle
// whose address a new context may reuse).  Initialises the current device's
// primary context when none is current.  Caches of device pointers are keyed
// on it: a cudaDeviceReset destroys the context they were made in.
cudaError_t current_context_id(unsigned long long* id);

// Test hook for the bounded grid barrier: a cooperative launch of `ctas` CTAs
// (at most one per SM) in which CTA 0 enters `rounds` grid barriers that no
// other CTA joins.  The first wait gives up after wait_ns nanoseconds and
// reports ERR_WAIT (4) in *err; every later barrier must return at once.
// *passed counts the barriers CTA 0 got through (0 when the abort works).
// With all_join every CTA enters the barriers (no wait runs out; the kernel
// time / rounds is the cost of one grid barrier).  bar: 4 unsigned of device
// memory.
cudaError_t launch_debug_barrier_timeout(int ctas, int rounds, long long wait_ns, int all_join, unsigned* bar,
                                         int* err, int* passed, cudaStream_t s);
}  // namespace ps
