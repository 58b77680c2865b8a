// mtp_md.cu - device neighbour lists and velocity-Verlet integration.
//
// The reference builds its padded neighbour rows on the host every MD step
// from LAMMPS's full neighbour list (pair_style_files/pair_jax_mtp.cpp:110-167)
// and copies them across PCIe (zero_overhead.cpp:61-117).  Here the rows are
// built on the device with a cell list, keep (owner index, periodic image)
// per slot, and are re-packed into r_ij = x_j - x_i + image . H every step
// while the list is reused (a skin distance covers the motion in between).
//
// Determinism: atoms are binned by a counting sort whose cells are then
// sorted by atom id; neighbour cells are visited in a fixed order, so every
// row has the same slot order on every run.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "mtp_md.hpp"

namespace mtp {

namespace {

__device__ __forceinline__ void frac_of(const double* x, const Box& b, double* f) {
  for (int a = 0; a < 3; ++a) f[a] = x[0] * b.hinv[0][a] + x[1] * b.hinv[1][a] + x[2] * b.hinv[2][a];
}

__device__ __forceinline__ int pack_image(int a, int b, int c) {
  return ((a + 512) & 1023) | (((b + 512) & 1023) << 10) | (((c + 512) & 1023) << 20);
}

__device__ __forceinline__ void unpack_image(int s, int& a, int& b, int& c) {
  a = (s & 1023) - 512;
  b = ((s >> 10) & 1023) - 512;
  c = ((s >> 20) & 1023) - 512;
}

}  // namespace

__global__ void k_cell_assign(int n, const double* __restrict__ x, Box b, int* __restrict__ cell,
                              int* __restrict__ img, int* __restrict__ cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double f[3];
  frac_of(x + 3 * i, b, f);
  int c[3];
  for (int a = 0; a < 3; ++a) {
    const double fl = floor(f[a]);
    img[3 * i + a] = static_cast<int>(fl);
    const double w = f[a] - fl;
    c[a] = min(b.nc[a] - 1, max(0, static_cast<int>(w * b.nc[a])));
  }
  const int id = (c[0] * b.nc[1] + c[1]) * b.nc[2] + c[2];
  cell[i] = id;
  atomicAdd(cnt + id, 1);
}

__global__ void k_cell_fill(int n, const int* __restrict__ cell, const int* __restrict__ ptr,
                            int* __restrict__ cursor, int* __restrict__ atoms) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = cell[i];
  const int pos = atomicAdd(cursor + c, 1);
  atoms[ptr[c] + pos] = i;
}

__global__ void k_cell_sort(int ncell, const int* __restrict__ ptr, int* __restrict__ atoms) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  const int b = ptr[c], e = ptr[c + 1];
  for (int x = b + 1; x < e; ++x) {
    const int v = atoms[x];
    int y = x - 1;
    while (y >= b && atoms[y] > v) {
      atoms[y + 1] = atoms[y];
      --y;
    }
    atoms[y + 1] = v;
  }
}

// One thread per centre atom: visit the 27 cells around its own in a fixed order.
__global__ void k_build_rows(int n, const double* __restrict__ x, Box b, const int* __restrict__ cell,
                             const int* __restrict__ img, const int* __restrict__ ptr,
                             const int* __restrict__ atoms, const int* __restrict__ types, double rc2, int stride,
                             int* __restrict__ js, int* __restrict__ shifts, int* __restrict__ jtypes,
                             int* __restrict__ counts, int* __restrict__ err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int ci = cell[i];
  const int c0 = ci / (b.nc[1] * b.nc[2]), c1 = (ci / b.nc[2]) % b.nc[1], c2 = ci % b.nc[2];
  const int ki0 = img[3 * i], ki1 = img[3 * i + 1], ki2 = img[3 * i + 2];
  // wrapped position of i
  double wi[3];
  for (int a = 0; a < 3; ++a)
    wi[a] = x[3 * i + a] - (ki0 * b.h[0][a] + ki1 * b.h[1][a] + ki2 * b.h[2][a]);
  int m = 0;
  const size_t row = static_cast<size_t>(i) * stride;
  for (int d0 = -1; d0 <= 1; ++d0) {
    int n0 = c0 + d0, s0 = 0;
    if (n0 < 0) { n0 += b.nc[0]; s0 = -1; } else if (n0 >= b.nc[0]) { n0 -= b.nc[0]; s0 = 1; }
    for (int d1 = -1; d1 <= 1; ++d1) {
      int n1 = c1 + d1, s1 = 0;
      if (n1 < 0) { n1 += b.nc[1]; s1 = -1; } else if (n1 >= b.nc[1]) { n1 -= b.nc[1]; s1 = 1; }
      for (int d2 = -1; d2 <= 1; ++d2) {
        int n2 = c2 + d2, s2 = 0;
        if (n2 < 0) { n2 += b.nc[2]; s2 = -1; } else if (n2 >= b.nc[2]) { n2 -= b.nc[2]; s2 = 1; }
        const int cj = (n0 * b.nc[1] + n1) * b.nc[2] + n2;
        const double sh[3] = {s0 * b.h[0][0] + s1 * b.h[1][0] + s2 * b.h[2][0],
                              s0 * b.h[0][1] + s1 * b.h[1][1] + s2 * b.h[2][1],
                              s0 * b.h[0][2] + s1 * b.h[1][2] + s2 * b.h[2][2]};
        for (int p = ptr[cj]; p < ptr[cj + 1]; ++p) {
          const int j = atoms[p];
          if (j == i && s0 == 0 && s1 == 0 && s2 == 0) continue;
          const int kj0 = img[3 * j], kj1 = img[3 * j + 1], kj2 = img[3 * j + 2];
          double r[3], r2 = 0.0;
          for (int a = 0; a < 3; ++a) {
            const double wj = x[3 * j + a] - (kj0 * b.h[0][a] + kj1 * b.h[1][a] + kj2 * b.h[2][a]);
            r[a] = wj + sh[a] - wi[a];
            r2 += r[a] * r[a];
          }
          if (r2 >= rc2) continue;
          if (m < stride) {
            js[row + m] = j;
            shifts[row + m] = pack_image(s0 - kj0 + ki0, s1 - kj1 + ki1, s2 - kj2 + ki2);
            jtypes[row + m] = types[j];
          }
          ++m;
        }
      }
    }
  }
  if (m > stride) {
    atomicOr(err, 4);   // capacity: a row needs more than `stride` slots
    m = stride;
  }
  counts[i] = m;
  for (int s = m; s < stride; ++s) {
    js[row + s] = -1;
    shifts[row + s] = pack_image(0, 0, 0);
    jtypes[row + s] = -1;
  }
}

__global__ void k_pack_rij(int n, int stride, const double* __restrict__ x, Box b, const int* __restrict__ js,
                           const int* __restrict__ shifts, const int* __restrict__ counts, double* __restrict__ rij) {
  const size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
  if (t >= static_cast<size_t>(n) * stride) return;
  const int i = static_cast<int>(t / stride), s = static_cast<int>(t % stride);
  double* r = rij + 3 * t;
  if (s >= counts[i]) {
    r[0] = r[1] = r[2] = 0.0;
    return;
  }
  const int j = js[t];
  int a, bb, c;
  unpack_image(shifts[t], a, bb, c);
  for (int k = 0; k < 3; ++k)
    r[k] = x[3 * j + k] - x[3 * i + k] + a * b.h[0][k] + bb * b.h[1][k] + c * b.h[2][k];
}

__global__ void k_verlet(int n, double* __restrict__ x, double* __restrict__ v, const double* __restrict__ f,
                         const int* __restrict__ types, VerletParams p, int stage) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int t = types[i];
  t = t < 0 ? 0 : (t >= kMaxMdSpecies ? kMaxMdSpecies - 1 : t);
  const double a = 0.5 * p.dt * p.ftm2v * p.inv_mass[t];
  for (int k = 0; k < 3; ++k) {
    double vk = v[3 * i + k] + a * f[3 * i + k];
    v[3 * i + k] = vk;
    if (stage == 1) x[3 * i + k] += p.dt * vk;
  }
}

bool make_box(const double* cell9, double cutoff, Box& b) {
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) b.h[r][c] = cell9[3 * r + c];
  const double (*h)[3] = b.h;
  const double det = h[0][0] * (h[1][1] * h[2][2] - h[1][2] * h[2][1]) -
                     h[0][1] * (h[1][0] * h[2][2] - h[1][2] * h[2][0]) +
                     h[0][2] * (h[1][0] * h[2][1] - h[1][1] * h[2][0]);
  if (!(std::fabs(det) > 0.0)) return false;
  // inverse (x_frac = x_cart . hinv)
  b.hinv[0][0] = (h[1][1] * h[2][2] - h[1][2] * h[2][1]) / det;
  b.hinv[0][1] = (h[0][2] * h[2][1] - h[0][1] * h[2][2]) / det;
  b.hinv[0][2] = (h[0][1] * h[1][2] - h[0][2] * h[1][1]) / det;
  b.hinv[1][0] = (h[1][2] * h[2][0] - h[1][0] * h[2][2]) / det;
  b.hinv[1][1] = (h[0][0] * h[2][2] - h[0][2] * h[2][0]) / det;
  b.hinv[1][2] = (h[0][2] * h[1][0] - h[0][0] * h[1][2]) / det;
  b.hinv[2][0] = (h[1][0] * h[2][1] - h[1][1] * h[2][0]) / det;
  b.hinv[2][1] = (h[0][1] * h[2][0] - h[0][0] * h[2][1]) / det;
  b.hinv[2][2] = (h[0][0] * h[1][1] - h[0][1] * h[1][0]) / det;
  // plane spacing along each lattice vector = |det| / |a_b x a_c|
  for (int a = 0; a < 3; ++a) {
    const int p = (a + 1) % 3, q = (a + 2) % 3;
    const double cx = h[p][1] * h[q][2] - h[p][2] * h[q][1];
    const double cy = h[p][2] * h[q][0] - h[p][0] * h[q][2];
    const double cz = h[p][0] * h[q][1] - h[p][1] * h[q][0];
    const double spacing = std::fabs(det) / std::sqrt(cx * cx + cy * cy + cz * cz);
    b.nc[a] = static_cast<int>(std::floor(spacing / cutoff));
  }
  return true;
}

cudaError_t launch_neighbors(int n, const double* x, const Box& b, const int* types, double cutoff, int stride,
                             int* js, int* shifts, int* jtypes, int* counts, CellScratch& cs, int* err,
                             cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int ncell = b.nc[0] * b.nc[1] * b.nc[2];
  cudaMemsetAsync(cs.cnt, 0, sizeof(int) * ncell, st);
  cudaMemsetAsync(cs.cursor, 0, sizeof(int) * ncell, st);
  k_cell_assign<<<(n + 255) / 256, 256, 0, st>>>(n, x, b, cs.cell, cs.img, cs.cnt);
  cudaError_t e = scan_exclusive(ncell, cs.cnt, cs.ptr, cs.blk, st);
  if (e != cudaSuccess) return e;
  k_cell_fill<<<(n + 255) / 256, 256, 0, st>>>(n, cs.cell, cs.ptr, cs.cursor, cs.atoms);
  k_cell_sort<<<(ncell + 127) / 128, 128, 0, st>>>(ncell, cs.ptr, cs.atoms);
  k_build_rows<<<(n + 127) / 128, 128, 0, st>>>(n, x, b, cs.cell, cs.img, cs.ptr, cs.atoms, types, cutoff * cutoff,
                                               stride, js, shifts, jtypes, counts, err);
  return cudaGetLastError();
}

cudaError_t launch_pack_rij(int n, int stride, const double* x, const Box& b, const int* js, const int* shifts,
                            const int* counts, double* rij, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const size_t tot = static_cast<size_t>(n) * stride;
  k_pack_rij<<<static_cast<unsigned>((tot + 255) / 256), 256, 0, st>>>(n, stride, x, b, js, shifts, counts, rij);
  return cudaGetLastError();
}

cudaError_t launch_verlet(int n, double* x, double* v, const double* f, const int* types, const VerletParams& p,
                          int stage, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_verlet<<<(n + 255) / 256, 256, 0, st>>>(n, x, v, f, types, p, stage);
  return cudaGetLastError();
}

}  // namespace mtp
