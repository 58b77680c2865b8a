// mtp_train.hpp - the coefficient adjoint of the batched evaluation (training).
//
// For a loss L(E_c, F_k, sigma_c) with upstream gradients gE, gF, gS the
// gradient with respect to every coefficient p is
//
//     dL/dp = sum_i d/dp [ a_i E_i + sum_s dr_is . dE_i/dr_is ],
//     a_i   = gE[c(i)],
//     dr_is = gF_i - gF_{j_is} (when j_is is a real atom) + C_c r_is,
//
// with C_c the symmetric matrix that maps the reference's stress
// sym(sum r (x) g)/V (jax_backend.py:355-360) onto gS.  The bracket is a
// directional derivative of the site energy, so the kernel carries dual
// numbers (value, tangent along dr) through the radial functions, the basic
// moments and the contraction tree, and runs the reverse programs on the
// duals: that yields the mixed second derivatives the force and stress terms
// of the loss need (what jax.grad of training/motep_jax_train_function.py:67-87
// differentiates through), in one pass per atom, deterministically.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "mtp_device.cuh"

namespace mtp {

struct TrainIO {
  int natoms, nbr_stride, nconfig;
  const int* itypes;
  const double* rijs;
  const int* js;
  const int* jtypes;
  const int* counts;
  const int* cfg;         // [natoms] configuration of each atom
  const double* volumes;  // [nconfig]
  const double* gE;       // [nconfig]
  const double* gF;       // [natoms][3]
  const double* gS;       // [nconfig][6] (xx, yy, zz, yz, xz, xy)
  int* err;
};

struct TrainWorkspace {
  double* partials = nullptr;   // [grid][Sa + S + S*S*R*K]
  size_t partials_cap = 0;
  void* vscratch = nullptr;     // [grid][2 * v_size] when the value space is global
  size_t vscratch_cap = 0;
};

void train_free(TrainWorkspace& w);

// Whether the adjoint's value space (value and tangent of every slot) fits in
// shared memory for `threads` lanes; otherwise it lives in global memory.
bool adjoint_fits_shared(const DevModel& md, int n_pad, int threads);

// Runs the adjoint kernel (FP64) and the fixed-order reduction into the outputs.
cudaError_t launch_adjoint(const DevModel& md, const TrainIO& io, int threads, int sm_count, TrainWorkspace& ws,
                           double* gspecies, double* gmoment, double* gradial, cudaStream_t st, std::string& err);

}  // namespace mtp
