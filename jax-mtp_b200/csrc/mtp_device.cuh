// mtp_device.cuh - sm_100a kernels of the MTP evaluator.
//
// One persistent thread block evaluates A centre atoms at a time (a
// grid-stride loop over groups of A atoms):
//
//   N1  neighbour staging: the slots of the atoms' padded rows are read with
//       coalesced loads in one sweep, tested (t_j >= 0, |r| < max_dist),
//       compacted with warp ballots, and each kept neighbour gets its unit
//       vector, distance, radial functions f_mu(d), f'_mu(d) (Chebyshev basis
//       times the smooth cutoff, jax_backend.py:83-95, 108-160) and the powers
//       of its unit vector components, all in shared memory;
//   N2  basic moments m[(mu, a, b, c)] = sum_j f_mu(d_j) u_x^a u_y^b u_z^c
//       (conversion.py:66-81), one thread per (atom, monomial), only the
//       radial functions that have a moment at the monomial's degree;
//   T   contraction tree (conversion.py:95-102) by the lane programs of the
//       schedule, then E_i = xi[t_i] + theta . m[mapping] (jax_backend.py:101-106);
//   R   reverse programs: dE_i/dm for every moment, gathered per source, so
//       no two threads ever add into the same value;
//   N3  per neighbour: dE_i/dr_ij from dE_i/dm of the basic moments by nested
//       Horner over the monomial simplex (the analytic form of
//       jax.value_and_grad at jax_backend.py:56), two neighbours per thread
//       in FP32 and one in FP64,
//       written to the per-slot gradient array.
//
// The A atoms of a block share every lane-program entry: their values are
// interleaved [slot][atom] so one vector access serves all of them.
//
// Forces then come from a per-atom gather (k_force_gather): the atom's own
// slot gradients minus the gradients of the slots that point at it, in a
// fixed order, so results are bitwise reproducible without atomics
// (jax_backend.py:263-303 uses an atomic segment_sum instead).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "mtp_model.hpp"

namespace mtp {

enum ErrBits : int { kErrNonFinite = 1, kErrSpecies = 2, kErrCapacity = 4 };

struct DevPass {
  int offset;
  int steps;
};

// Everything the evaluation kernel needs about the potential (device pointers).
struct DevModel {
  const uint2* entries;
  DevPass fwd[kMaxPasses];
  DevPass rev[kMaxPasses];
  int nfwd, nrev;
  // steps each warp runs in each pass, [nfwd + nrev][lanes / 32]: a warp
  // stops after its longest lane's program (Pass::wsteps)
  const int* warp_steps;
  const double* radial;     // [S][S][R][K]
  const double* species;    // [S]
  const double* theta;      // [Sa]
  const int* mapping;       // [Sa]
  const int* seed_idx;      // [nseed]
  const double* seed_val;   // [nseed]
  const int* zero_list;     // [nzero]
  const int* mono_abc;      // [P][4]
  const int* mono_k;        // [P][kMaxR]
  const int* dense_k;       // [Q][kMaxR] basic moment of dense slot and mu, or -1
  int nseed, nzero;
  int S, R, K, M, B, P, D, Sa;
  int Q, npairs;
  int tri;                  // Schedule::tri: step k of a force-phase chain has k / 2 + 1 radial functions,
                            // and the basic moments' adjoints are in chain order (dm_pos)
  const int* dm_pos;        // [M] adjoint position of each moment (Schedule::dm_pos)
  const int* n3_pairs;      // Schedule::n3_pairs / n3_off (level-structured bases)
  const int* n3_off;
  const int* n3_pairs_half;  // Schedule::n3_pairs_half / n3_off_half (the FP64 kernel)
  const int* n3_off_half;
  int nmu[kMaxDegree + 1];  // radial functions with a basic moment of each degree
  int v_m, v_dm, v_zero, v_one, v_size;
  double scaling, rmin, rmax;
};

struct DevIO {
  int natoms;
  int nbr_stride;
  int n_pad;                // staging rows (>= max count, <= nbr_stride rounded)
  const int* itypes;        // [natoms]
  const double* rijs;       // [natoms][nbr_stride][3]
  const int* jtypes;        // [natoms][nbr_stride]
  const int* counts;        // [natoms] or null
  double* site_energy;      // [natoms]
  double* pair_grad;        // [natoms][nbr_stride][3]
  int* err;                 // error bits
  void* vscratch;           // [grid][v_size] value space when it lives in global memory
};

// Shared-memory carve of the evaluation kernel.
// Lane-program entries requested ahead of use (registers), per thread.
constexpr int kPrefetch = kStepAlign;

// Radial-function values the basic-moment phase reads with one load: four
// in FP32 (16 bytes; rows padded to match), one in FP64 (vector loads were
// measured slower there).
template <typename T>
constexpr int kRadVec = sizeof(T) == 4 ? 4 : 1;

// Shared-memory carve of the evaluation kernel for A atoms per block: the
// value space is interleaved [slot][atom] so one vector access serves all A
// atoms; neighbour staging is kept per atom.  The dense dE/dm table of the
// force phase reuses the moment half of the value space (dead once the
// reverse passes are done) when it fits there (Q R <= M); with the value
// space in global memory, or when it does not fit, it gets its own region.
struct SmemLayout {
  int pws;        // stride of a power row (3 (D+1), rounded up to odd)
  int rs;         // stride of a radial-function row (R rounded up to kRadVec)
  bool dmt_in_v;  // dense table in the moment half of the value space
  bool n3p_in_v;  // force-phase partial sums in the moment half of the value space
  size_t v, rad, u, f, fp, pw, slot, dmt, n3p, red, cnt, total;
};

// Values of the force phase's partial-sum buffer on level-structured bases:
// (G_x, G_y, G_z, S) of 32 neighbours from each warp.
__host__ __device__ inline int n3_partials(int threads) { return 4 * threads; }

template <typename T>
__host__ __device__ inline SmemLayout smem_layout(int v_size, int M, int S, int R, int K, int D, int n_pad,
                                                  int threads, int A, bool tri) {
  SmemLayout L;
  L.pws = 3 * (D + 1);
  if ((L.pws & 1) == 0) L.pws += 1;
  const int Q = (D + 1) * (D + 2) * (D + 3) / 6;
  // level-structured bases need no dense table; their partial sums use the
  // moment half of the value space (dead after the reverse passes) when it
  // holds them
  L.dmt_in_v = tri || (v_size > 0 && Q * R <= M);
  L.n3p_in_v = tri && v_size > 0 && n3_partials(threads) <= M * A;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    size_t at = (o + 31) & ~size_t(31);
    o = at + bytes;
    return at;
  };
  L.v = take(sizeof(T) * v_size * A);
  L.rad = take(sizeof(T) * S * S * R * K);
  L.u = take(sizeof(T) * 4 * n_pad * A);
  L.rs = (R + kRadVec<T> - 1) / kRadVec<T> * kRadVec<T>;
  L.f = take(sizeof(T) * L.rs * n_pad * A);
  L.fp = take(sizeof(T) * L.rs * n_pad * A);
  L.pw = take(sizeof(T) * L.pws * n_pad * A);
  L.slot = take(sizeof(int) * n_pad * A);
  L.dmt = L.dmt_in_v ? L.v : take(sizeof(T) * R * Q * A);
  L.n3p = !tri || L.n3p_in_v ? L.v : take(sizeof(T) * n3_partials(threads));
  L.red = take(sizeof(double) * (threads / 32) * A);
  L.cnt = take(sizeof(int) * (threads / 32 + 8));   // per-warp counts, then per-atom totals
  L.total = (o + 31) & ~size_t(31);
  return L;
}

__device__ __forceinline__ double dev_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float dev_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double dev_fma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float dev_fma(float a, float b, float c) { return fmaf(a, b, c); }

// A values of one value-space slot, loaded/stored as one vector access.
template <typename T, int A>
struct __align__(sizeof(T) * A) Pack {
  T v[A];
};

// Integer multiplicity of an entry (y & kMultMask < 2^14) as T without an
// int-to-float conversion instruction: OR-ing m into the mantissa of 2^23
// (2^52) gives the float (double) 2^23 + m exactly, and subtracting 2^23
// (2^52) leaves m exactly.
template <typename T>
__device__ __forceinline__ T entry_mult(uint32_t y);
template <>
__device__ __forceinline__ float entry_mult<float>(uint32_t y) {
  return __int_as_float(static_cast<int>((y & kMultMask) | 0x4B000000u)) - 8388608.0f;
}
template <>
__device__ __forceinline__ double entry_mult<double>(uint32_t y) {
  return __hiloint2double(0x43300000, static_cast<int>(y & kMultMask)) - 4503599627370496.0;
}

// Stream one lane program pass: every thread walks its column of the
// [steps][LANES] entry array with PF entries in flight (registers), so the L2
// latency of the program overlaps the arithmetic.  LANES is a template
// argument so every request is one load at a constant offset; PF divides
// kStepAlign, so steps is a multiple of PF and the program holds PF rows after
// any pass: nothing is bounds-tested.  Each entry feeds A atoms:
// acc[a] += c * V[x][a] * V[y][a]; STORE/ADD flush into V[d][a].
// Operands are read through Vr and flushes go through V: a pass never reads a
// slot that it writes, so the two views do not alias.  kEarly: the operand
// gathers of all PF entries in flight are issued before any of their flushes
// (allowed for the same reason); with the value space in global memory this
// overlaps PF gathers' latencies (level-28 FP64 forward 54.1 -> 38.4 ms at
// 32,000 atoms), in shared memory it gains 0.1-0.6 % at the tuned shapes
// (2.5 % at 256 lanes x 1 atom in FP64).  Both use it.
template <typename T, int A, int LANES, int PF, bool kEarly>
__device__ __forceinline__ void run_pass(const uint2* __restrict__ ent, int steps, int tid, T* __restrict__ V,
                                         const T* __restrict__ Vr) {
  static_assert(PF >= 1 && kStepAlign % PF == 0, "prefetch depth must divide the pass step alignment");
  const uint2* p = ent + tid;
  uint2 buf[PF];
#pragma unroll
  for (int k = 0; k < PF; ++k) buf[k] = __ldg(p + k * LANES);
  T acc[A];
#pragma unroll
  for (int a = 0; a < A; ++a) acc[a] = T(0);
  for (int s0 = 0; s0 < steps; s0 += PF) {
    p += PF * LANES;
    uint2 ek[PF];
    Pack<T, A> va[PF], vb[PF];
#pragma unroll
    for (int k = 0; k < PF; ++k) {
      ek[k] = buf[k];
      if (kEarly) {
        va[k] = *reinterpret_cast<const Pack<T, A>*>(Vr + (ek[k].x & 0xFFFFu) * A);
        vb[k] = *reinterpret_cast<const Pack<T, A>*>(Vr + (ek[k].x >> 16) * A);
      }
      buf[k] = __ldg(p + k * LANES);
    }
#pragma unroll
    for (int k = 0; k < PF; ++k) {
      const uint2 e = ek[k];
      const T c = entry_mult<T>(e.y);
      if (!kEarly) {
        va[k] = *reinterpret_cast<const Pack<T, A>*>(Vr + (e.x & 0xFFFFu) * A);
        vb[k] = *reinterpret_cast<const Pack<T, A>*>(Vr + (e.x >> 16) * A);
      }
#pragma unroll
      for (int a = 0; a < A; ++a) acc[a] = dev_fma(c * va[k].v[a], vb[k].v[a], acc[a]);
      if (e.y & (3u << kOpShift)) {
        Pack<T, A>* dst = reinterpret_cast<Pack<T, A>*>(V + (e.y >> kDstShift) * A);
        Pack<T, A> out;
        if (e.y & (kOpStore << kOpShift)) {
#pragma unroll
          for (int a = 0; a < A; ++a) out.v[a] = acc[a];
        } else {
          out = *dst;
#pragma unroll
          for (int a = 0; a < A; ++a) out.v[a] += acc[a];
        }
        *dst = out;
#pragma unroll
        for (int a = 0; a < A; ++a) acc[a] = T(0);
      }
    }
  }
}

// Lane p of every warp gets its warp's step count of pass p (forward passes,
// then reverse ones; at most 32 passes), so a pass reads its count with a
// shuffle instead of a load.
__device__ __forceinline__ int warp_steps_of_lane(const DevModel& md, int tid, int NT) {
  const int p = tid & 31;
  return p < md.nfwd + md.nrev ? __ldg(md.warp_steps + p * (NT >> 5) + (tid >> 5)) : 0;
}

// run_pass for the block's lane count (128, 256 or 512 threads).
template <typename T, int A, bool kEarly, int PF = kPrefetch>
__device__ __forceinline__ void run_pass_n(const uint2* __restrict__ ent, int steps, int lanes, int tid,
                                           T* __restrict__ V) {
  if (lanes == 512) run_pass<T, A, 512, PF, kEarly>(ent, steps, tid, V, V);
  else if (lanes == 256) run_pass<T, A, 256, PF, kEarly>(ent, steps, tid, V, V);
  else run_pass<T, A, 128, PF, kEarly>(ent, steps, tid, V, V);
}

// Generic lane-program streamer (used by the dual-number kernels): every thread
// walks its column of the [steps][LANES] entries with PF in flight.  PF divides
// kStepAlign, so steps is a multiple of PF and the rows after a pass exist;
// LANES is fixed so every request is one load at a constant offset.  A Body
// has load(e) (the entry's operand gathers) and apply(e, operands) (the
// arithmetic and the flush); with kEarly the gathers of all PF entries are
// issued before the first apply, which a pass allows because it never reads a
// slot that it writes.
template <int LANES, int PF, bool kEarly, typename Body>
__device__ __forceinline__ void stream_entries_t(const uint2* __restrict__ ent, int steps, int tid, Body& body) {
  static_assert(PF >= 1 && kStepAlign % PF == 0, "prefetch depth must divide the pass step alignment");
  const uint2* p = ent + tid;
  uint2 buf[PF];
#pragma unroll
  for (int k = 0; k < PF; ++k) buf[k] = __ldg(p + k * LANES);
  for (int s0 = 0; s0 < steps; s0 += PF) {
    p += PF * LANES;
    uint2 ek[PF];
    typename Body::Operands op[PF];
#pragma unroll
    for (int k = 0; k < PF; ++k) {
      ek[k] = buf[k];
      if (kEarly) op[k] = body.load(ek[k]);
      buf[k] = __ldg(p + k * LANES);
    }
#pragma unroll
    for (int k = 0; k < PF; ++k) {
      if (!kEarly) op[k] = body.load(ek[k]);
      body.apply(ek[k], op[k]);
    }
  }
}

template <int PF, bool kEarly, typename Body>
__device__ __forceinline__ void stream_entries_n(const uint2* __restrict__ ent, int steps, int lanes, int tid,
                                                 Body& body) {
  if (lanes == 512) stream_entries_t<512, PF, kEarly>(ent, steps, tid, body);
  else if (lanes == 256) stream_entries_t<256, PF, kEarly>(ent, steps, tid, body);
  else stream_entries_t<128, PF, kEarly>(ent, steps, tid, body);
}

// Force-phase sums of one or (kTwo) two neighbours over this thread's share
// of the monomial simplex.  With W_s = sum_mu Dm[s][mu] f_mu(d), W'_s the same with
// f'_mu, and Q(u) = sum_s W_s u_x^a u_y^b u_z^c over slots s = (a, b, c):
//   G = grad_u Q = (Gx, Gy, Gz),   S = sum_s W'_s u_x^a u_y^b u_z^c.
// Each (a, b) pair is a Horner chain in u_z over c = D-a-b .. 0 (value and
// z-derivative), scaled by the stored powers of u_x and u_y.  The dE/dm rows
// are per atom, so two neighbours share every row load and their chains run
// side by side.  The tpn threads of a neighbour pair take the (a, b)
// pairs in snake order (sl, 2 tpn-1-sl, 2 tpn+sl, ...) of the pair order
// (a + b ascending), so their shares differ by one pair at most.  dmt is the
// dense table [slot][R] in pair order (bases without the level structure;
// level-structured ones use n3_transposed).
template <typename T, int R, bool kTwo>
__device__ __forceinline__ void n3_sums(const T* __restrict__ dmt, int D,
                                        int npairs, int D1, const T* __restrict__ fq0, const T* __restrict__ fpq0,
                                        const T* __restrict__ fq1, const T* __restrict__ fpq1, bool two,
                                        const T* __restrict__ pw0, const T* __restrict__ pw1, T uz0, T uz1, int sl,
                                        int tpn, T (&S)[2], T (&Gx)[2], T (&Gy)[2], T (&Gz)[2]) {
  T f0[R], fp0[R], f1[R], fp1[R];
#pragma unroll
  for (int mu = 0; mu < R; ++mu) {
    f0[mu] = fq0[mu];
    fp0[mu] = fpq0[mu];
    f1[mu] = kTwo && two ? fq1[mu] : T(0);
    fp1[mu] = kTwo && two ? fpq1[mu] : T(0);
  }
  // diagonal s = a + b of the current pair, its first pair index, and the
  // first dense slot of the diagonal (pair order: each pair of diagonal s
  // owns D - s + 1 slots, so slot bases follow without a table lookup)
  int s = 0, sb = 0, slot_sb = 0;
  for (int k = 0;; ++k) {
    const int i = (k >> 1) * 2 * tpn + ((k & 1) ? 2 * tpn - 1 - sl : sl);
    if (i >= npairs) break;
    while (i >= sb + s + 1) {
      sb += s + 1;
      slot_sb += (s + 1) * (D - s + 1);
      ++s;
    }
    const int ea = i - sb, eb = s - ea, top = D - s;
    const T* drow = dmt + (slot_sb + ea * (D - s + 1) + top) * R;
    T h0 = T(0), hz0 = T(0), hs0 = T(0), h1 = T(0), hz1 = T(0), hs1 = T(0);
    // one Horner step over the table row
    auto step = [&](const T* row) {
      T w0 = T(0), wp0 = T(0), w1 = T(0), wp1 = T(0);
#pragma unroll
      for (int mu = 0; mu < R; ++mu) {
        const T g = row[mu];
        w0 = dev_fma(g, f0[mu], w0);
        wp0 = dev_fma(g, fp0[mu], wp0);
        if (kTwo) {
          w1 = dev_fma(g, f1[mu], w1);
          wp1 = dev_fma(g, fp1[mu], wp1);
        }
      }
      hz0 = dev_fma(hz0, uz0, h0);
      h0 = dev_fma(h0, uz0, w0);
      hs0 = dev_fma(hs0, uz0, wp0);
      if (kTwo) {
        hz1 = dev_fma(hz1, uz1, h1);
        h1 = dev_fma(h1, uz1, w1);
        hs1 = dev_fma(hs1, uz1, wp1);
      }
    };
#pragma unroll 1
    for (int c = top; c >= 0; --c, drow -= R) step(drow);
    {
      const T xa = pw0[ea], yb = pw0[D1 + eb];
      const T dxa = ea > 0 ? static_cast<T>(ea) * pw0[ea - 1] : T(0);
      const T dyb = eb > 0 ? static_cast<T>(eb) * pw0[D1 + eb - 1] : T(0);
      const T xy = xa * yb;
      Gx[0] = dev_fma(dxa * yb, h0, Gx[0]);
      Gy[0] = dev_fma(xa * dyb, h0, Gy[0]);
      Gz[0] = dev_fma(xy, hz0, Gz[0]);
      S[0] = dev_fma(xy, hs0, S[0]);
    }
    if (kTwo) {
      const T xa = pw1[ea], yb = pw1[D1 + eb];
      const T dxa = ea > 0 ? static_cast<T>(ea) * pw1[ea - 1] : T(0);
      const T dyb = eb > 0 ? static_cast<T>(eb) * pw1[D1 + eb - 1] : T(0);
      const T xy = xa * yb;
      Gx[1] = dev_fma(dxa * yb, h1, Gx[1]);
      Gy[1] = dev_fma(xa * dyb, h1, Gy[1]);
      Gz[1] = dev_fma(xy, hz1, Gz[1]);
      S[1] = dev_fma(xy, hs1, S[1]);
    }
  }
}

// Force phase on level-structured bases.  The warps form groups of GW =
// min(warps, kN3GroupWarps); group g takes the chunks of 32 kept neighbours
// c = g, g + groups, ... (item j = 32 c + lane over the A atoms' lists in
// turn), and the warps of a group take disjoint sets of monomial pairs
// (Schedule::n3_pairs, at most 32 per warp; each lane holds one pair word and
// the warp shuffles it out), so all lanes of a warp read the same adjoint row
// at every step (one shared-memory wavefront per gather; the A atoms' values
// of a slot are adjacent) and no lane reduces with its neighbours.  Per item
// and pair: the Horner chain in u_z over steps k = 0 .. top with the radial
// functions mu <= k / 2, then the powers of u_x and u_y; the group's partial
// sums (G, S) meet in P ([4][warps][32]) and its first warp adds them in warp
// order (deterministic) and writes the slot gradients.
template <typename T, int A, int R>
__device__ __forceinline__ void n3_transposed(const DevModel& md, const DevIO& io, const SmemLayout& L,
                                              unsigned char* smem, const T* __restrict__ V,
                                              const int (&nv_a)[A], int base, int tid, int NT, T* __restrict__ P) {
  const int w = tid >> 5, lane = tid & 31, NW = NT >> 5;
  // FP64 runs groups of half the width (fewer, shorter rounds for its fewer
  // atoms per block; measured faster there, slower in FP32)
  constexpr bool kHalf = sizeof(T) == 8;
  const int* n3_off = kHalf ? md.n3_off_half : md.n3_off;
  const int* n3_pairs = kHalf ? md.n3_pairs_half : md.n3_pairs;
  const int GW = min(NW, kHalf ? kN3GroupWarps / 2 : kN3GroupWarps), g = w / GW, wg = w - g * GW, NG = NW / GW;
  const int D1 = md.D + 1, pws = L.pws, n_pad = io.n_pad;
  const int p0 = __ldg(n3_off + wg), np = __ldg(n3_off + wg + 1) - p0;
  const int myword = lane < np ? __ldg(n3_pairs + p0 + lane) : 0;
  int J = 0;
#pragma unroll
  for (int a = 0; a < A; ++a) J += nv_a[a];
  // every group runs the same number of rounds (the block barriers match)
  for (int c0 = 0; c0 < J; c0 += 32 * NG) {
    const int j = c0 + 32 * g + lane;
    const bool act = j < J;
    int a = 0, q = act ? j : 0;
#pragma unroll
    for (int aa = 0; aa + 1 < A; ++aa)
      if (a == aa && q >= nv_a[aa]) {
        q -= nv_a[aa];
        a = aa + 1;
      }
    const T* sF = reinterpret_cast<const T*>(smem + L.f) + (static_cast<size_t>(a) * n_pad + q) * L.rs;
    const T* sFp = reinterpret_cast<const T*>(smem + L.fp) + (static_cast<size_t>(a) * n_pad + q) * L.rs;
    const T* sU = reinterpret_cast<const T*>(smem + L.u) + (static_cast<size_t>(a) * n_pad + q) * 4;
    const T* pw = reinterpret_cast<const T*>(smem + L.pw) + (static_cast<size_t>(a) * n_pad + q) * pws;
    T f[R], fp[R];
#pragma unroll
    for (int mu = 0; mu < R; ++mu) {
      f[mu] = sF[mu];
      fp[mu] = sFp[mu];
    }
    const T uz = sU[2];
    const T* dmv = V + static_cast<size_t>(md.v_dm) * A + a;
    T Gx = T(0), Gy = T(0), Gz = T(0), Ss = T(0);
    for (int pi = 0; pi < np; ++pi) {
      const int word = __shfl_sync(0xffffffffu, myword, pi);
      if (act) {
        const int ea = word & 15, eb = (word >> 4) & 15, top = (word >> 8) & 15;
        const T* drow = dmv + static_cast<size_t>(word >> 12) * A;
        T h = T(0), hz = T(0), hs = T(0);
#pragma unroll
        for (int k = 0; k <= kMaxDegree; ++k) {
          if (k > top) break;
          const T* row = drow + (((k + 1) * (k + 1)) >> 2) * A;
          T wv = T(0), wp = T(0);
#pragma unroll
          for (int mu = 0; mu < R; ++mu) {
            if (mu <= k / 2) {
              const T g = row[mu * A];
              wv = dev_fma(g, f[mu], wv);
              wp = dev_fma(g, fp[mu], wp);
            }
          }
          hz = dev_fma(hz, uz, h);
          h = dev_fma(h, uz, wv);
          hs = dev_fma(hs, uz, wp);
        }
        const T xa = pw[ea], yb = pw[D1 + eb];
        const T dxa = ea > 0 ? static_cast<T>(ea) * pw[ea - 1] : T(0);
        const T dyb = eb > 0 ? static_cast<T>(eb) * pw[D1 + eb - 1] : T(0);
        const T xy = xa * yb;
        Gx = dev_fma(dxa * yb, h, Gx);
        Gy = dev_fma(xa * dyb, h, Gy);
        Gz = dev_fma(xy, hz, Gz);
        Ss = dev_fma(xy, hs, Ss);
      }
    }
    P[(0 * NW + w) * 32 + lane] = Gx;
    P[(1 * NW + w) * 32 + lane] = Gy;
    P[(2 * NW + w) * 32 + lane] = Gz;
    P[(3 * NW + w) * 32 + lane] = Ss;
    __syncthreads();
    if (wg == 0 && act) {
      T gx_ = T(0), gy_ = T(0), gz_ = T(0), s_ = T(0);
      for (int ww = w; ww < w + GW; ++ww) {
        gx_ += P[(0 * NW + ww) * 32 + lane];
        gy_ += P[(1 * NW + ww) * 32 + lane];
        gz_ += P[(2 * NW + ww) * 32 + lane];
        s_ += P[(3 * NW + ww) * 32 + lane];
      }
      const T ux = sU[0], uy = sU[1], d = sU[3];
      const T ug = ux * gx_ + uy * gy_ + uz * gz_;
      const T inv_d = T(1) / d;
      const T gx = ux * s_ + (gx_ - ux * ug) * inv_d;
      const T gy = uy * s_ + (gy_ - uy * ug) * inv_d;
      const T gz = uz * s_ + (gz_ - uz * ug) * inv_d;
      const int atom = base + a;
      const int slot = reinterpret_cast<const int*>(smem + L.slot)[a * n_pad + q];
      double* grow = io.pair_grad + (static_cast<size_t>(atom) * io.nbr_stride + slot) * 3;
      grow[0] = static_cast<double>(gx);
      grow[1] = static_cast<double>(gy);
      grow[2] = static_cast<double>(gz);
      if (!(isfinite(static_cast<double>(gx)) && isfinite(static_cast<double>(gy)) &&
            isfinite(static_cast<double>(gz))))
        atomicOr(io.err, kErrNonFinite);
    }
    __syncthreads();
  }
}

// Basic moments of one (atom, monomial) task for NM radial functions:
// acc[mu] = sum_q f_mu(d_q) u_x^a u_y^b u_z^c over the kept neighbours.  The
// radial rows (stride rs) are read kRadVec values per load.
template <typename T, int NM>
__device__ __forceinline__ void moment_task(const T* __restrict__ sF, const T* __restrict__ sPw, int rs, int pws, int D1,
                                            int nv, int ea, int eb, int ec, T (&acc)[kMaxR]) {
  constexpr int VW = kRadVec<T>, NV = (NM + VW - 1) / VW;
  using V4 = typename std::conditional<sizeof(T) == 4, float4, double>::type;
#pragma unroll 4
  for (int q = 0; q < nv; ++q) {
    const T* pw = sPw + q * pws;
    const T mono = pw[ea] * pw[D1 + eb] * pw[2 * D1 + ec];
    T f[NV * VW];
#pragma unroll
    for (int v = 0; v < NV; ++v) *reinterpret_cast<V4*>(f + v * VW) = reinterpret_cast<const V4*>(sF + q * rs)[v];
#pragma unroll
    for (int mu = 0; mu < NM; ++mu) acc[mu] = dev_fma(f[mu], mono, acc[mu]);
  }
}

// Per-warp sums of A doubles per thread: lane 0 of warp w writes atom a's
// sum to red[a * warps + w] (summed later in warp order: deterministic).
template <int A>
__device__ __forceinline__ void warp_partials(double (&v)[A], double* red) {
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
#pragma unroll
  for (int a = 0; a < A; ++a) {
    for (int o = 16; o > 0; o >>= 1) v[a] += __shfl_xor_sync(0xffffffffu, v[a], o);
    if (l == 0) red[a * nw + w] = v[a];
  }
}

// ---------------------------------------------------------------------------
// evaluation kernel
// ---------------------------------------------------------------------------
// A atoms per block share every lane-program entry.  kVGlobal: the value
// space (moments, adjoints, partials) is a private slice of global memory
// (L1/L2-resident) instead of shared memory; used when it does not fit in
// shared memory (level 28 in FP64).
// Register budget per thread: the FP32 one-atom variant runs three 256-thread
// blocks per SM (80 registers fit 768 threads); the others run one block of
// up to 512 threads.
template <typename T, bool kVGlobal, int A>
struct EvalRegs {
  static constexpr int value = (sizeof(T) == 4 && !kVGlobal && A == 1) ? 64 : 128;
};

template <typename T, bool kVGlobal, int A>
__global__ void __maxnreg__((EvalRegs<T, kVGlobal, A>::value)) k_mtp_eval(DevModel md, DevIO io) {
  extern __shared__ __align__(32) unsigned char smem[];
  const int NT = blockDim.x;
  const int tid = threadIdx.x;
  // this warp's step count of pass p (forward passes, then reverse ones) is
  // held by lane p and shuffled out at the pass: no load before a pass
  const int my_wsteps = warp_steps_of_lane(md, tid, NT);
  const SmemLayout L = smem_layout<T>(kVGlobal ? 0 : md.v_size, md.M, md.S, md.R, md.K, md.D, io.n_pad, NT, A,
                                     md.tri != 0);
  T* V = kVGlobal ? reinterpret_cast<T*>(io.vscratch) + static_cast<size_t>(blockIdx.x) * md.v_size * A
                  : reinterpret_cast<T*>(smem + L.v);
  T* sRad = reinterpret_cast<T*>(smem + L.rad);
  double* sRed = reinterpret_cast<double*>(smem + L.red);
  int* sCnt = reinterpret_cast<int*>(smem + L.cnt);
  const int n_pad = io.n_pad;

  const int S = md.S, R = md.R, K = md.K, P = md.P, D1 = md.D + 1, pws = L.pws;
  // per-block constants
  for (int x = tid; x < S * S * R * K; x += NT) sRad[x] = static_cast<T>(md.radial[x]);
  for (int a = tid; a < A; a += NT) {
    V[md.v_zero * A + a] = T(0);
    V[md.v_one * A + a] = T(1);
  }
  const T rmax = static_cast<T>(md.rmax);
  const T inv_range = static_cast<T>(1.0 / (md.rmax - md.rmin));
  const T rsum = static_cast<T>(md.rmin + md.rmax);
  const T scal = static_cast<T>(md.scaling);
  __syncthreads();

  for (int base = blockIdx.x * A; base < io.natoms; base += gridDim.x * A) {
    // ask L2 for the rows of this block's next atoms now, so their staging
    // loads find them there instead of in DRAM (a hint; nothing waits on it)
    {
      const int next = base + gridDim.x * A;
      if (next < io.natoms) {
        const int na = min(A, io.natoms - next);
        const char* r0 = reinterpret_cast<const char*>(io.rijs + static_cast<size_t>(next) * io.nbr_stride * 3);
        const char* t0 = reinterpret_cast<const char*>(io.jtypes + static_cast<size_t>(next) * io.nbr_stride);
        const int rl = (na * io.nbr_stride * 24 + 127) >> 7, tl = (na * io.nbr_stride * 4 + 127) >> 7;
        for (int x = tid; x < rl + tl; x += NT) {
          const char* a = x < rl ? r0 + 128 * static_cast<size_t>(x) : t0 + 128 * static_cast<size_t>(x - rl);
          asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
        }
      }
    }
    // moments that are read but never written (the force phase of the
    // previous atom may have reused their slots for its dense table)
    for (int x = tid; x < md.nzero * A; x += NT) V[(md.v_m + md.zero_list[x / A]) * A + x % A] = T(0);
    int it_a[A], nv_a[A], cnt_a[A];
    // ---- N1: staging of every atom of the block ---------------------------
#pragma unroll
    for (int a = 0; a < A; ++a) {
      const int atom = base + a;
      const bool real = atom < io.natoms;
      int it = real ? __ldg(io.itypes + atom) : 0;
      if (it < 0 || it >= S) {
        if (tid == 0) atomicOr(io.err, kErrSpecies);
        it = 0;
      }
      it_a[a] = it;
      int cnt = real ? (io.counts ? __ldg(io.counts + atom) : io.nbr_stride) : 0;
      if (cnt > n_pad || cnt < 0) {
        if (tid == 0) atomicOr(io.err, kErrCapacity);
        cnt = cnt < 0 ? 0 : n_pad;
      }
      cnt_a[a] = cnt;
      nv_a[a] = 0;
    }
    // tasks (atom, slot) with each atom's slots padded to whole warps, so a
    // warp's ballot covers one atom.  In FP64, when the block has twice as
    // many threads as tasks, every task has two threads (role 0: tid < NV,
    // role 1: the thread NV above it): both load and test the slot (the same
    // ballot), role 0 stores the direction and the radial functions, role 1
    // the powers (measured faster in FP64, not in FP32)
    const int S32 = (io.nbr_stride + 31) & ~31;
    const int NV = A * S32;
    const bool split = sizeof(T) == 8 && 2 * NV <= NT;
    const int span = split ? NV : NT;   // tasks per sweep
    const int role = split ? (tid < NV ? 0 : tid < 2 * NV ? 1 : 2) : 0;
    for (int v0 = 0; v0 < NV; v0 += span) {
      const int v = v0 + (split ? tid - role * NV : tid);
      const int a = (role < 2 && v < NV) ? v / S32 : A;
      const int s = v - a * S32;
      int it = 0, cnt = 0;
#pragma unroll
      for (int aa = 0; aa < A; ++aa)
        if (aa == a) {
          it = it_a[aa];
          cnt = cnt_a[aa];
        }
      const int atom = base + a;
      const bool real = a < A && atom < io.natoms;
      const size_t arow = static_cast<size_t>(real ? atom : 0) * io.nbr_stride;
      const double* rrow = io.rijs + arow * 3;
      const int* trow = io.jtypes + arow;
      double* grow = io.pair_grad + arow * 3;
      bool valid = false;
      T rx = T(0), ry = T(0), rz = T(0), d = T(0);
      int jt = -1;
      if (real && s < io.nbr_stride) {
        if (s < cnt) {
          jt = __ldg(trow + s);
          rx = static_cast<T>(__ldg(rrow + 3 * s));
          ry = static_cast<T>(__ldg(rrow + 3 * s + 1));
          rz = static_cast<T>(__ldg(rrow + 3 * s + 2));
          if (jt >= S) {
            atomicOr(io.err, kErrSpecies);
            jt = -1;
          }
          const T r2 = rx * rx + ry * ry + rz * rz;
          d = dev_sqrt(r2);
          valid = (jt >= 0) && (r2 > T(0)) && (d < rmax);
        }
        if (!valid && role == 0) {
          grow[3 * s] = 0.0;
          grow[3 * s + 1] = 0.0;
          grow[3 * s + 2] = 0.0;
        }
      }
      const unsigned bal = __ballot_sync(0xffffffffu, valid);
      const int w = tid >> 5, l = tid & 31, nw = NT >> 5;
      const int wt = w - role * (NV >> 5);   // the role-0 warp of these tasks
      if (l == 0 && role == 0) sCnt[w] = __popc(bal);
      __syncthreads();
      if (tid == 0) {
        // exclusive offsets of each warp within its atom's kept slots of this
        // sweep; per-atom totals after the warp counts
        int accn = 0, cur = -1;
        for (int i = 0; i < (span >> 5); ++i) {
          const int ai = (v0 + 32 * i) / S32;
          if (ai != cur) {
            if (cur >= 0 && cur < A) sCnt[nw + cur] = accn;
            cur = ai;
            accn = 0;
          }
          const int c = sCnt[i];
          sCnt[i] = accn;
          accn += c;
        }
        if (cur >= 0 && cur < A) sCnt[nw + cur] = accn;
      }
      __syncthreads();
      if (valid) {
        int nv = 0;
#pragma unroll
        for (int aa = 0; aa < A; ++aa)
          if (aa == a) nv = nv_a[aa];
        const int q = nv + sCnt[wt] + __popc(bal & ((1u << l) - 1u));
        T* sU = reinterpret_cast<T*>(smem + L.u) + static_cast<size_t>(a) * 4 * n_pad;
        T* sF = reinterpret_cast<T*>(smem + L.f) + static_cast<size_t>(a) * L.rs * n_pad;
        T* sFp = reinterpret_cast<T*>(smem + L.fp) + static_cast<size_t>(a) * L.rs * n_pad;
        T* sPw = reinterpret_cast<T*>(smem + L.pw) + static_cast<size_t>(a) * pws * n_pad;
        int* sSlot = reinterpret_cast<int*>(smem + L.slot) + a * n_pad;
        const T inv_d = T(1) / d;
        const T ux = rx * inv_d, uy = ry * inv_d, uz = rz * inv_d;
        if (role == 0) {
          sU[4 * q] = ux;
          sU[4 * q + 1] = uy;
          sU[4 * q + 2] = uz;
          sU[4 * q + 3] = d;
          sSlot[q] = s;
          // Chebyshev T_n(x) and dT_n/dx by their recurrences, folded into
          // sum_n c[t_i, t_j, mu, n] T_n for every mu as the terms appear
          const T x = (T(2) * d - rsum) * inv_range;
          const T dxdd = T(2) * inv_range;
          const T* c = sRad + (static_cast<size_t>(it) * S + jt) * R * K;
          T bas[kMaxR], dbas[kMaxR];
#pragma unroll
          for (int mu = 0; mu < kMaxR; ++mu) {
            bas[mu] = mu < R ? c[mu * K] : T(0);   // T_0 = 1, T_0' = 0
            dbas[mu] = T(0);
          }
          T t_prev = T(1), t_cur = x, dt_prev = T(0), dt_cur = T(1);
          for (int n = 1; n < K; ++n) {
#pragma unroll
            for (int mu = 0; mu < kMaxR; ++mu) {
              if (mu < R) {
                bas[mu] = dev_fma(c[mu * K + n], t_cur, bas[mu]);
                dbas[mu] = dev_fma(c[mu * K + n], dt_cur, dbas[mu]);
              }
            }
            const T t_next = T(2) * x * t_cur - t_prev;
            const T dt_next = T(2) * t_cur + T(2) * x * dt_cur - dt_prev;
            t_prev = t_cur;
            t_cur = t_next;
            dt_prev = dt_cur;
            dt_cur = dt_next;
          }
          const T gap = rmax - d;
          const T smooth = gap * gap;
#pragma unroll
          for (int mu = 0; mu < kMaxR; ++mu) {
            if (mu < R) {
              sF[q * L.rs + mu] = scal * smooth * bas[mu];
              sFp[q * L.rs + mu] = scal * (T(-2) * gap * bas[mu] + smooth * dbas[mu] * dxdd);
            }
          }
        }
        if (role == 1 || !split) {
          T* pw = sPw + q * pws;
          T px = T(1), py = T(1), pz = T(1);
          for (int e = 0; e < D1; ++e) {
            pw[e] = px;
            pw[D1 + e] = py;
            pw[2 * D1 + e] = pz;
            px *= ux;
            py *= uy;
            pz *= uz;
          }
        }
      }
      // atoms touched by this sweep add its kept count
#pragma unroll
      for (int aa = 0; aa < A; ++aa) {
        const int first = v0 / S32, last = (v0 + span - 1) / S32;
        if (aa >= first && aa <= last) nv_a[aa] += sCnt[nw + aa];
      }
      __syncthreads();
    }
    // ---- N2: basic moments m[(mu, a, b, c)] of every atom of the block ------
    // tasks (atom, monomial), most radial functions first: monomials are
    // sorted by degree (descending), so monomial P-1-j has the j-th most.  A
    // warp takes 32 consecutive monomials of one atom (one radial-function
    // count and one neighbour list per warp; the warp's largest count is
    // used), warp slots go round-robin over the atoms, and odd rounds run the
    // slots in reverse (snake), so each thread's rounds add up to about the
    // same cost and the last, partial round gets the cheapest monomials.
    const int P32 = (P + 31) & ~31;
    for (int t0 = 0; t0 < A * P32; t0 += NT) {
      const int pos = t0 + (((t0 / NT) & 1) ? NT - 1 - tid : tid);
      const int blk = pos >> 5, j = (blk / A) * 32 + (pos & 31);
      const bool act = pos < A * P32 && j < P;
      const int a = act ? blk % A : 0, p = act ? P - 1 - j : 0;
      const int4 abc = __ldg(reinterpret_cast<const int4*>(md.mono_abc) + p);
      int nv = 0;
#pragma unroll
      for (int aa = 0; aa < A; ++aa)
        if (act && aa == a) nv = nv_a[aa];
      const int nm = __reduce_max_sync(0xffffffffu, act ? md.nmu[abc.w] : 0);
      const T* sF = reinterpret_cast<const T*>(smem + L.f) + static_cast<size_t>(a) * L.rs * n_pad;
      const T* sPw = reinterpret_cast<const T*>(smem + L.pw) + static_cast<size_t>(a) * pws * n_pad;
      T acc[kMaxR];
#pragma unroll
      for (int mu = 0; mu < kMaxR; ++mu) acc[mu] = T(0);
      switch (nm) {
        case 0: break;
        case 1: moment_task<T, 1>(sF, sPw, L.rs, pws, D1, nv, abc.x, abc.y, abc.z, acc); break;
        case 2: moment_task<T, 2>(sF, sPw, L.rs, pws, D1, nv, abc.x, abc.y, abc.z, acc); break;
        case 3: moment_task<T, 3>(sF, sPw, L.rs, pws, D1, nv, abc.x, abc.y, abc.z, acc); break;
        case 4: moment_task<T, 4>(sF, sPw, L.rs, pws, D1, nv, abc.x, abc.y, abc.z, acc); break;
        case 5: moment_task<T, 5>(sF, sPw, L.rs, pws, D1, nv, abc.x, abc.y, abc.z, acc); break;
        case 6: moment_task<T, 6>(sF, sPw, L.rs, pws, D1, nv, abc.x, abc.y, abc.z, acc); break;
        case 7: moment_task<T, 7>(sF, sPw, L.rs, pws, D1, nv, abc.x, abc.y, abc.z, acc); break;
        default: moment_task<T, 8>(sF, sPw, L.rs, pws, D1, nv, abc.x, abc.y, abc.z, acc); break;
      }
      if (act) {
#pragma unroll
        for (int mu = 0; mu < kMaxR; ++mu) {
          if (mu < nm) {
            const int k = __ldg(md.mono_k + kMaxR * p + mu);
            if (k >= 0) V[(md.v_m + k) * A + a] = acc[mu];
          }
        }
      }
    }
    // adjoint seeds
    for (int x = tid; x < md.M * A; x += NT) V[md.v_dm * A + x] = T(0);
    __syncthreads();
    for (int x = tid; x < md.nseed * A; x += NT)
      V[(md.v_dm + md.seed_idx[x / A]) * A + x % A] = static_cast<T>(md.seed_val[x / A]);

    // ---- T: forward contraction passes ----------------------------------
    for (int ps = 0; ps < md.nfwd; ++ps) {
      run_pass_n<T, A, true>(md.entries + md.fwd[ps].offset, __shfl_sync(0xFFFFFFFFu, my_wsteps, ps), NT, tid,
                                 V);
      __syncthreads();
    }
    // energy: E_i = xi[t_i] + sum_alpha theta_alpha m[map_alpha] in FP64
    {
      double ep[A];
#pragma unroll
      for (int a = 0; a < A; ++a) ep[a] = 0.0;
      for (int al = tid; al < md.Sa; al += NT) {
        const double th = __ldg(md.theta + al);
        const int k = md.v_m + __ldg(md.mapping + al);
#pragma unroll
        for (int a = 0; a < A; ++a) ep[a] = fma(th, static_cast<double>(V[k * A + a]), ep[a]);
      }
      // warp sums now; the block sum waits for the reverse passes' barriers
      // (no barrier of its own on the critical path)
      warp_partials<A>(ep, sRed);
    }

    // ---- R: reverse passes (dE/dm) ---------------------------------------
    for (int ps = 0; ps < md.nrev; ++ps) {
      run_pass_n<T, A, true>(md.entries + md.rev[ps].offset,
                                 __shfl_sync(0xFFFFFFFFu, my_wsteps, md.nfwd + ps), NT, tid, V);
      __syncthreads();
    }

    // site energies: thread a adds atom a's warp sums in warp order
    if (md.nrev == 0) __syncthreads();
#pragma unroll
    for (int a = 0; a < A; ++a) {
      if (tid == a && base + a < io.natoms) {
        double ep = 0.0;
        for (int i = 0; i < (NT >> 5); ++i) ep += sRed[a * (NT >> 5) + i];
        const double e = __ldg(md.species + it_a[a]) + ep;
        io.site_energy[base + a] = e;
        if (!isfinite(e)) atomicOr(io.err, kErrNonFinite);
      }
    }

    // ---- N3: dE_i/dr_ij per kept neighbour -------------------------------
    // level-structured bases read the basic moments' adjoints in place (chain
    // order); otherwise a dense table Dm[a][slot][mu] = dE/dm of basic moment
    // (mu, slot) over the full monomial simplex in pair order (0 where the
    // basis has no moment) is filled first
    if (md.tri) {
      T* P = L.n3p_in_v ? V + static_cast<size_t>(md.v_m) * A : reinterpret_cast<T*>(smem + L.n3p);
      switch (R) {
#define MTP_N3T_CASE(RR) \
  case RR: n3_transposed<T, A, RR>(md, io, L, smem, V, nv_a, base, tid, NT, P); break;
        MTP_N3T_CASE(1) MTP_N3T_CASE(2) MTP_N3T_CASE(3) MTP_N3T_CASE(4)
        MTP_N3T_CASE(5) MTP_N3T_CASE(6) MTP_N3T_CASE(7) MTP_N3T_CASE(8)
#undef MTP_N3T_CASE
        default: break;
      }
      __syncthreads();
      continue;
    }
    T* sDm = L.dmt_in_v ? V + md.v_m * A : reinterpret_cast<T*>(smem + L.dmt);
    const int QR = md.Q * R;
    for (int x = tid; x < QR * A; x += NT) {
      const int a = x / QR, r = x - a * QR;
      const int k = __ldg(md.dense_k + (r / R) * kMaxR + r % R);
      sDm[x] = k >= 0 ? V[(md.v_dm + __ldg(md.dm_pos + k)) * A + a] : T(0);
    }
    __syncthreads();
#pragma unroll
    for (int a = 0; a < A; ++a) {
      const int atom = base + a;
      const int nv = nv_a[a];
      const T* sU = reinterpret_cast<T*>(smem + L.u) + static_cast<size_t>(a) * 4 * n_pad;
      const T* sF = reinterpret_cast<T*>(smem + L.f) + static_cast<size_t>(a) * L.rs * n_pad;
      const T* sFp = reinterpret_cast<T*>(smem + L.fp) + static_cast<size_t>(a) * L.rs * n_pad;
      const T* sPw = reinterpret_cast<T*>(smem + L.pw) + static_cast<size_t>(a) * pws * n_pad;
      const int* sSlot = reinterpret_cast<int*>(smem + L.slot) + a * n_pad;
      double* grow = io.pair_grad + static_cast<size_t>(atom < io.natoms ? atom : 0) * io.nbr_stride * 3;
      // FP32: threads take pairs of neighbours (q, q + nt), which share every
      // table-row load; FP64: one neighbour per thread (the second
      // neighbour's registers would spill at the 128-register budget)
      constexpr bool kTwoN = sizeof(T) == 4;
      const int nt = kTwoN ? (nv + 1) >> 1 : nv;
      int tpn = 32;
      while (tpn > 1 && tpn * nt > NT) tpn >>= 1;
      const int total = nt * tpn;
      for (int b0 = 0; b0 < total; b0 += NT) {
        const int idx = b0 + tid;
        const bool active = idx < total;
        const int q0 = active ? idx / tpn : 0;
        const int q1 = q0 + nt;
        const bool two = kTwoN && active && q1 < nv;
        const int sl = idx & (tpn - 1);
        T Ssum[2] = {T(0), T(0)}, Gx[2] = {T(0), T(0)}, Gy[2] = {T(0), T(0)}, Gz[2] = {T(0), T(0)};
        if (active) {
          const T* dmt = sDm + static_cast<size_t>(a) * QR;
          const int qb = two ? q1 : q0;
          switch (R) {
#define MTP_N3_CASE(RR)                                                                                        \
  case RR:                                                                                                     \
    n3_sums<T, RR, kTwoN>(dmt, md.D, md.npairs, D1, sF + q0 * L.rs, sFp + q0 * L.rs, sF + qb * L.rs, \
                                   sFp + qb * L.rs, two, sPw + q0 * pws, sPw + qb * pws, sU[4 * q0 + 2],         \
                                   sU[4 * qb + 2], sl, tpn, Ssum, Gx, Gy, Gz);                                \
    break;
            MTP_N3_CASE(1) MTP_N3_CASE(2) MTP_N3_CASE(3) MTP_N3_CASE(4)
            MTP_N3_CASE(5) MTP_N3_CASE(6) MTP_N3_CASE(7) MTP_N3_CASE(8)
#undef MTP_N3_CASE
            default: break;
          }
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          for (int o = tpn >> 1; o > 0; o >>= 1) {
            Ssum[j] += __shfl_xor_sync(0xffffffffu, Ssum[j], o);
            Gx[j] += __shfl_xor_sync(0xffffffffu, Gx[j], o);
            Gy[j] += __shfl_xor_sync(0xffffffffu, Gy[j], o);
            Gz[j] += __shfl_xor_sync(0xffffffffu, Gz[j], o);
          }
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int q = j ? q1 : q0;
          if (active && sl == 0 && (j == 0 || two)) {
            const T ux = sU[4 * q], uy = sU[4 * q + 1], uz = sU[4 * q + 2], d = sU[4 * q + 3];
            const T ug = ux * Gx[j] + uy * Gy[j] + uz * Gz[j];
            const T inv_d = T(1) / d;
            const T gx = ux * Ssum[j] + (Gx[j] - ux * ug) * inv_d;
            const T gy = uy * Ssum[j] + (Gy[j] - uy * ug) * inv_d;
            const T gz = uz * Ssum[j] + (Gz[j] - uz * ug) * inv_d;
            const int s = sSlot[q];
            grow[3 * s] = static_cast<double>(gx);
            grow[3 * s + 1] = static_cast<double>(gy);
            grow[3 * s + 2] = static_cast<double>(gz);
            if (!(isfinite(static_cast<double>(gx)) && isfinite(static_cast<double>(gy)) &&
                  isfinite(static_cast<double>(gz))))
              atomicOr(io.err, kErrNonFinite);
          }
        }
      }
    }
    __syncthreads();
  }
}

}  // namespace mtp
