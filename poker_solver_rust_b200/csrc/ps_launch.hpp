// Host-callable launchers of the kernels in ps_kernels.cu.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>

#include "ps_device.hpp"

namespace ps {
size_t solve_smem(int vstride);
size_t setup_smem_bytes();
int solve_occupancy(int block, size_t smem);
cudaError_t launch_setup(const SpotDev* spots, const int2* work, int nwork, const int32_t* table, int* err,
                         int grid, cudaStream_t s);
cudaError_t launch_solve(const SpotDev* spots, int nspots, const int* order, int* counter, const Discount* disc,
                         int max_iter, const float* target, float* scratch, size_t scratch_floats, float* out_expl,
                         int* out_iters, int* err, int grid, int block, size_t smem, cudaStream_t s);
cudaError_t launch_iterate(const SpotDev* spots, int nspots, const Discount* disc, int t0, int t1,
                           float* scratch, size_t scratch_floats, int* err, int grid, int block, size_t smem,
                           cudaStream_t s);
cudaError_t launch_exploitability(const SpotDev* spots, int nspots, float* scratch, size_t scratch_floats,
                                  float* out, int* err, int grid, int block, size_t smem, cudaStream_t s);
cudaError_t launch_average(const SpotDev* spots, int nspots, int save, int player, const float* root_reach,
                           float* scratch, size_t scratch_floats, float* out, int* err, int grid, int block,
                           size_t smem, cudaStream_t s);
cudaError_t launch_eval_terminal(const SpotDev* spots, Op op, int player, float* scratch, size_t scratch_floats,
                                 int* err, int block, size_t smem, cudaStream_t s);
}  // namespace ps
