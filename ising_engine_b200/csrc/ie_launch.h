// Host-side launch wrappers of the kernels in ie_kernels.cu.
#pragma once
#include <cuda_runtime.h>

#include "ie_kernels.cuh"
#include "ie_level.cuh"

namespace ie {
cudaError_t set_smem_limits(size_t pt_bytes);
size_t batch_smem(int tpl, uint32_t spin_cap, bool serve);
int batch_occupancy(uint32_t mode, int tpl, uint32_t spin_cap, bool serve);
cudaError_t launch_batch(const DevArrays& A, const RunArgs& R, uint32_t mode, int tpl, uint32_t spin_cap, int grid,
                         cudaStream_t st);
int window_occupancy(uint32_t mode, uint32_t spin_cap);
cudaError_t launch_window(const DevArrays& A, const RunArgs& R, uint32_t mode, uint32_t spin_cap, int grid,
                          cudaStream_t st);
int chain_occupancy(uint32_t mode, uint32_t spin_cap);
cudaError_t launch_chain(const DevArrays& A, const RunArgs& R, uint32_t mode, uint32_t spin_cap, int grid,
                         cudaStream_t st);
cudaError_t launch_exchange(const DevArrays& A, const RunArgs& R, uint32_t ninst, uint32_t mode, uint32_t steps,
                            bool exchange, cudaStream_t st);
cudaError_t launch_swap(const DevArrays& A, uint32_t inst, uint32_t n_words, int sm_count, cudaStream_t st);
cudaError_t launch_icm(const DevArrays& A, uint32_t inst, uint32_t mode, uint32_t cells, uint32_t* count,
                       uint32_t* rank, uint8_t* flags, uint32_t* stack, uint32_t slots, cudaStream_t st);
cudaError_t launch_resample(const DevArrays& A, uint32_t inst, uint32_t mode, uint32_t n_words, uint32_t pop_len,
                            const uint32_t* parents, const uint64_t* old_spins, const int32_t* old_ei,
                            const double* old_ef, int sm_count, cudaStream_t st);
cudaError_t launch_pt(const DevArrays& A, const RunArgs& R, uint32_t inst0, uint32_t ninst, uint32_t mode,
                      int block, int tab_stride, size_t smem, cudaStream_t st);
cudaError_t launch_init(const DevArrays& A, uint32_t inst0, uint32_t ninst, const uint32_t* draw_idx,
                        const uint32_t* unclamped, cudaStream_t st);
cudaError_t launch_energy(const DevArrays& A, uint32_t inst0, uint32_t ninst, cudaStream_t st);
cudaError_t launch_energy_check(const DevArrays& A, uint32_t inst0, uint32_t ninst, double* out, cudaStream_t st);
cudaError_t launch_model_energy(const DevArrays& A, uint32_t inst, uint32_t nt, double offset, double* out,
                                cudaStream_t st);
cudaError_t launch_incumbent(const DevArrays& A, uint32_t inst, double offset, double* inc_e, uint64_t* inc_state,
                             uint32_t n_words, cudaStream_t st);
cudaError_t launch_best_extract(const DevArrays& A, uint32_t inst, const double* es, uint32_t count, int8_t* state,
                                double* best, int32_t* found, cudaStream_t st);
cudaError_t launch_one_opt(const DevArrays& A, uint32_t inst, int8_t* state, const uint8_t* clamped, double* gains,
                           double* improvement, uint64_t* flips, uint64_t max_flips, cudaStream_t st);
size_t level_smem(uint32_t mode, uint32_t ntab, uint32_t spin_cap, bool ov = false);
int level_occupancy(uint32_t mode, bool gsp, int threads, size_t smem);
// resident clusters of `split` CTAs of the split (cluster) form, GPU-wide
int level_clusters(uint32_t mode, int threads, size_t smem, uint32_t split);
cudaError_t launch_level(const DevArrays& A, const RunArgs& R, const LvlArgs& L, uint32_t mode, bool gsp, int threads,
                         int grid, cudaStream_t st, uint32_t split = 1);
void set_last_error(const char* msg);
cudaError_t probe_peaks(int sm_count, double* int_ops_per_s, double* xoshiro_per_s);
}  // namespace ie
