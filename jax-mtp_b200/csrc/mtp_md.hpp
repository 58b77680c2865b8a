// mtp_md.hpp - device neighbour lists, r_ij packing and velocity Verlet.
#pragma once

#include <cuda_runtime.h>

namespace mtp {

constexpr int kMaxMdSpecies = 16;

struct Box {
  double h[3][3];     // rows are the lattice vectors
  double hinv[3][3];  // fractional = cartesian . hinv
  int nc[3];          // cells along each lattice vector (cell width >= cutoff)
};

struct CellScratch {
  int* cell = nullptr;    // [n]
  int* img = nullptr;     // [n][3] periodic image of each atom
  int* cnt = nullptr;     // [ncell]
  int* ptr = nullptr;     // [ncell + 1]
  int* cursor = nullptr;  // [ncell]
  int* atoms = nullptr;   // [n]
  int* blk = nullptr;     // scan scratch
  int n_cap = 0, cell_cap = 0;
};

struct VerletParams {
  double dt;                        // ps
  double ftm2v;                     // (eV/A)/amu -> A/ps^2
  double inv_mass[kMaxMdSpecies];   // 1/amu per species
};

bool make_box(const double* cell9, double cutoff, Box& b);
cudaError_t scan_exclusive(int n, const int* in, int* out, int* blk, cudaStream_t st);
cudaError_t launch_neighbors(int n, const double* x, const Box& b, const int* types, double cutoff, int stride,
                             int* js, int* shifts, int* jtypes, int* counts, CellScratch& cs, int* err,
                             cudaStream_t st);
cudaError_t launch_pack_rij(int n, int stride, const double* x, const Box& b, const int* js, const int* shifts,
                            const int* counts, double* rij, cudaStream_t st);
// stage 1: half kick + drift; stage 2: half kick
cudaError_t launch_verlet(int n, double* x, double* v, const double* f, const int* types, const VerletParams& p,
                          int stage, cudaStream_t st);

}  // namespace mtp
