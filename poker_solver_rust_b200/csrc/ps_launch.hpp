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

// Shared-memory plan of one solve CTA (computed on the host per launch): one
// terminal scan buffer (3 * vstride floats) per warp, optional staged board
// tables, and a small reduction area.
struct SmemPlan {
  int vstride;  // max slot stride of the launch (floats)
  int hs_max;   // max padded hand count
  int warps;    // warps per CTA
  int bufs;     // warps 0 .. bufs-1 own a terminal scan buffer and evaluate the terminal runs
  int tables;   // bytes reserved for staged board tables (0 = tables stay in global memory)
  __host__ __device__ size_t total() const {
    return (size_t)tables + (size_t)bufs * 3 * vstride * 4 + 32 * 8;
  }
};

constexpr int kMaxSolveBlock = 256;  // threads per CTA the solve kernels are compiled for (launch bounds)
size_t setup_smem_bytes();
int solve_occupancy(int block, const SmemPlan& plan);
// Grid mode for one large spot: the work of one cooperative launch of k_grid
// (every CTA on the same spot), the number of CTAs that can be co-resident for
// it, and the launch.  bar: 2 unsigned, gred: 4 double, both device memory.
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
};
int grid_ctas(int block, const SmemPlan& plan);
// Reach-weighted 48-river average of boundary-network outputs (ps_datagen.cu):
// boards [n][4], denorm [n] (pot + stack), net [n][2][48][1326], reach
// [n][2][1326], hands [H] combo indices, out [n][2][H]; all device pointers.
cudaError_t launch_boundary_river_reduce(int n, const uint8_t* boards, const float* denorm, const float* net,
                                         const float* reach, const int32_t* hands, int H, float* out,
                                         cudaStream_t s);
cudaError_t launch_grid(const SpotDev* spot, const GridJob& job, const Discount* disc, float* scratch,
                        size_t scratch_floats, float* out_expl, int* out_iters, unsigned* bar, double* gred,
                        int* err, int grid, int block, const SmemPlan& plan, cudaStream_t s);
cudaError_t launch_setup(const SpotDev* spots, const int2* work, int nwork, const int32_t* table, int* err,
                         int grid, cudaStream_t s);
// Persistent batched solve over `ninst` instances of K spots (inst: [ninst][K]
// spot ids, -1 = empty); scratch holds K * scratch_floats floats per CTA.
cudaError_t launch_solve(const SpotDev* spots, int ninst, int K, const int* inst, int* counter,
                         const Discount* disc, int max_iter, const float* target, float* scratch,
                         size_t scratch_floats, float* out_expl, int* out_iters, int* err, int grid, int block,
                         const SmemPlan& plan, cudaStream_t s);
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
// (16 MiB); a game needs num_slots * vstride of them.  The first call on a
// device looks up the array's address (cudaGetSymbolAddress) with that device
// current.  Every call uses the same array: calls whose kernels overlap on
// the GPU overwrite each other's slots.
constexpr size_t kFixedScratchHeader = 64;
constexpr size_t kFixedScratchFloats = (size_t)4 << 20;
cudaError_t launch_exploitability_fixed(const SpotDev* spot, size_t slot_floats, int block, const SmemPlan& plan,
                                        cudaStream_t s, float* host_out, int* host_err);
}  // namespace ps
