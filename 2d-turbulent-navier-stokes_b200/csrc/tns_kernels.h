// tns_kernels.h -- launchers of the FP64 kernels (tns_kernels.cu) used by the runtime.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "tns_device.cuh"
#include "tns_batch.cuh"

namespace tns {

cudaError_t configure_kernels();
size_t stage_smem_bytes();
size_t visc_smem_bytes();
size_t diss_smem_bytes();
int dtmin_blocks(const Mesh& M);

void launch_dissipation(const Params& P, const Mesh& M, const double* q, double* d, double* dt,
                        const double* dtmin, cudaStream_t s);
void launch_viscous(const Params& P, const Mesh& M, const double* q, double* vis, cudaStream_t s);
// error: bit 1 is set when a tile's static-block copy did not complete (must not be null)
void launch_stage(const Params& P, const Mesh& M, const double* qin, const double* qold,
                  double* qout, const double* d, const double* vis, const double* dt,
                  const double* dtmin, double alpha, unsigned long long* cdiff,
                  unsigned int* status, unsigned int* error, cudaStream_t s);
void launch_dtmin(const Params& P, const Mesh& M, const double* q, double* partial,
                  unsigned int* counter, double* dtmin, cudaStream_t s);
void launch_time_step_scratch(const Params& P, const double* q, const double* cfldl,
                              long long ncell, double* dt, double* partial,
                              unsigned int* counter, double* dtmin, int nblocks,
                              cudaStream_t s);
void launch_gport(const Params& P, const Mesh& M, const double* q, const int* ghosts, int nport,
                  double* gport, cudaStream_t s);
void launch_prim_out(const Params& P, const Mesh& M, const double* q, double* out,
                     cudaStream_t s);

void launch_node_average(const Mesh& M, const double* prim, double* out, cudaStream_t s);
// mode 0: force / mass flow / area sums (out[4]); mode 1: total-pressure sums (out[2])
void launch_boundary_sums(const Params& P, const Mesh& M, const double* prim, int type, int side,
                          int mode, double* out, cudaStream_t s);
void launch_face_states(const Params& P, const Mesh& M, const double* prim, double* out, cudaStream_t s);

// accuracy check of the FP64 helpers (fn 0 = pow06, 1 = tanh_ratio)
void launch_debug_math(int fn, long long n, const double* a, const double* b, double* out, cudaStream_t s);

// batched multi-case kernels: kernel 0 dissipation, 1 viscous, 2 stage
void launch_batch_f64(const BatchCase* cases, const int4* tiles, const int* active, int ntiles,
                      int kernel, int stage, int monitor, cudaStream_t s);
void launch_batch_mx(const BatchCase* cases, const int4* tiles, const int* active, int ntiles,
                     int kernel, int parity, int stage, int monitor, cudaStream_t s);

// persistent batched iterations (schedule 3): dynamic shared memory, the resident grid
// (blocks per SM x SMs, 0 if unknown) and the cooperative launch of `iters` unmonitored
// iterations; bar = arrival counter and generation (zero before the launch), error bit 2
// = a grid barrier gave up
size_t persistent_smem_bytes(bool mixed);
int persistent_grid(bool mixed);
cudaError_t launch_persistent(bool mixed, const BatchCase* cases, const int4* tiles, const int* active,
                              int ntiles, int iters, int parity, int grid, unsigned int* bar,
                              unsigned int* error, cudaStream_t s);
const void* persistent_kernel_mx();
cudaError_t launch_persistent_mx(const BatchCase* cases, const int4* tiles, const int* active, int ntiles,
                                 int iters, int parity, int grid, unsigned int* bar, unsigned int* error,
                                 cudaStream_t s);
size_t stage_mx_smem_bytes();
size_t visc_mx_smem_bytes();
size_t diss_mx_smem_bytes();

// mixed FP32/FP64 path (tns_kernels_mx.cu)
cudaError_t configure_kernels_mx();
void launch_dissipation_mx(const Params& P, const Mesh& M, const double* q, float* d, float* dt,
                           const double* dtmin, cudaStream_t s);
void launch_dissipation_mx2(const Params& P, const Mesh& M, const double* q, float* d, float* dt,
                            const double* dtmin, cudaStream_t s);
void launch_viscous_mx(const Params& P, const Mesh& M, const double* q, float* vis, cudaStream_t s);
void launch_stage_mx(const Params& P, const Mesh& M, const double* cold, const float* dqin,
                     float* dqout, double* qout, const float* d, const float* vis, const float* dt,
                     const double* dtmin, double alpha, unsigned long long* cdiff,
                     unsigned int* status, unsigned int* error, cudaStream_t s);
void launch_gport_mx(const Params& P, const Mesh& M, const double* cold, const float* dq,
                     const int* ghosts, int nport, double* gport, cudaStream_t s);
void launch_prim_out_mx(const Params& P, const Mesh& M, const double* cold, const float* dq,
                        double* out, cudaStream_t s);

}  // namespace tns
