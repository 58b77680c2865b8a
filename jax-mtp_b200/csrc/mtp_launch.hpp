// mtp_launch.hpp - host launchers of the device kernels (mtp_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "mtp_device.cuh"

namespace mtp {

constexpr int kReduceBlocks = 256;   // fixed: the reduction order never depends on the GPU

// Dynamic shared memory of the evaluation kernel for A atoms per block
// (vglobal: value space in global memory, io.vscratch holding
// blocks * A * v_size values).
size_t eval_smem_bytes(const DevModel& md, int n_pad, int threads, bool fp64, bool vglobal, int A);
bool eval_variant_exists(bool fp64, bool vglobal, int A);
// Blocks per SM that fit for the evaluation kernel (0 if it does not fit).
int eval_blocks_per_sm(const DevModel& md, int n_pad, int threads, bool fp64, bool vglobal, int A);
cudaError_t launch_eval(const DevModel& md, const DevIO& io, int threads, int blocks, bool fp64, bool vglobal, int A,
                        cudaStream_t st);

// Incoming-slot lists: for every atom k, the slots (i, s) whose neighbour is k,
// sorted by slot id.  in_ptr [natoms + 1].
cudaError_t launch_incoming(int natoms, int stride, const int* js, const int* jtypes, const int* counts,
                            int* in_cnt, int* in_ptr, int* in_cursor, int* in_slot, int* block_tmp,
                            cudaStream_t st);

// forces[i] = own slot gradients - incoming slot gradients; wown [natoms][6]
// = -sym(sum_s r_is (x) g_is) (LAMMPS order xx,yy,zz,xy,xz,yz); when vatom
// is non-null it receives the half/half split of every pair's virial.
cudaError_t launch_force_gather(int natoms, int stride, const double* rijs, const int* counts,
                                const double* pair_grad, const int* in_ptr, const int* in_slot,
                                double* forces, double* wown, double* vatom, cudaStream_t st);

// out[0] = sum site_energy[0..natoms), out[1..6] = sum wown; fixed order.
cudaError_t launch_totals(int natoms, const double* site_energy, const double* wown, double* partials,
                          double* out, cudaStream_t st);

// Per-configuration energy [nconfig] and reference-convention stress [nconfig][6].
cudaError_t launch_config_totals(int natoms, int nconfig, const int* cfg_ptr, const double* site_energy,
                                 const double* wown, const double* volumes, double* energy, double* stress,
                                 cudaStream_t st);
// cfg_ptr [nconfig + 1] from a non-decreasing cfg_of_atom; flags bad input in err.
cudaError_t launch_config_ptr(int natoms, int nconfig, const int* cfg_of_atom, int* cfg_ptr, int* err,
                              cudaStream_t st);

// Rows [nlocal][stride] (r_ij, owner index, species, count) from positions
// x [nall][3] and candidate lists neigh [nlocal][list_stride]: candidates
// closer than cutoff, in list order; more than stride sets kErrCapacity.
cudaError_t launch_rows_from_positions(int nlocal, int nall, const double* x, const int* species, const int* owner,
                                       int list_stride, const int* neigh, const int* numneigh, double cutoff,
                                       int stride, double* rijs, int* js, int* jtypes, int* counts, int* err,
                                       cudaStream_t st);

// FMA-chain peak probe.
cudaError_t measure_fma_peak(double* fp64_tflops, double* fp32_tflops);

}  // namespace mtp
