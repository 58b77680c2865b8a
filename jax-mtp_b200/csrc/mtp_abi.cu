// mtp_abi.cu - the C ABI (include/mtp_b200.h): handles, device buffers, calls.
//
// Replaces the reference bridge pair_style_files/zero_overhead.cpp: instead
// of refilling NumPy buffers with sentinels and calling a deserialised JAX
// executable through CPython every step (zero_overhead.cpp:61-117, 171-272),
// a handle owns device buffers sized by the pair style's capacities and
// launches the sm_100a kernels directly.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mtp_b200.h"
#include "mtp_launch.hpp"
#include "mtp_md.hpp"
#include "mtp_model.hpp"
#include "mtp_train.hpp"

using namespace mtp;

namespace {

std::string g_create_error;

struct DeviceSchedule {
  Schedule sched;
  uint2* d_entries = nullptr;
  int* d_n3_pairs = nullptr;   // Schedule::n3_pairs / n3_off (level-structured bases)
  int* d_n3_off = nullptr;
  int* d_n3_pairs_half = nullptr;   // the same for the FP64 kernel's half-width groups
  int* d_n3_off_half = nullptr;
  int* d_warp_steps = nullptr;  // [forward passes, reverse passes][lanes / 32] (Pass::wsteps)
};

// Arguments of a host-buffer call that a cached CUDA graph replays.  The graph
// holds the host and device addresses, the sizes and the launch shapes, so it
// is valid for exactly these and for one generation of the handle's device
// state (bumped whenever coefficients, launch settings or scratch change).
struct HostCallKey {
  int kind = -1;   // 0: mtp_compute, 1: mtp_compute_positions
  int natoms = -1, stride = 0, flags = 0, extra = 0;
  long long gen = -1;
  const void* p[8] = {};
  bool operator==(const HostCallKey& o) const {
    if (kind != o.kind || natoms != o.natoms || stride != o.stride || flags != o.flags || extra != o.extra ||
        gen != o.gen)
      return false;
    for (int k = 0; k < 8; ++k)
      if (p[k] != o.p[k]) return false;
    return true;
  }
};

template <typename T>
cudaError_t dalloc(T** p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  return cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T));
}

}  // namespace

struct mtp_handle {
  Potential pot;
  int max_atoms = 0, max_nbr = 0, debug = 0, precision = 0;
  double cutoff = 0.0;
  int device = 0, sm_count = 0;
  cudaStream_t own_stream = nullptr, stream = nullptr;
  int threads = 256, blocks_per_sm = 0;
  int last_threads = 0, last_blocks = 0, last_bps = 0;
  bool last_vglobal = false;
  void* d_vscratch = nullptr;
  size_t vscratch_bytes = 0;
  size_t last_smem = 0;
  std::map<int, DeviceSchedule> scheds;
  // potential tables on the device
  double *d_radial = nullptr, *d_species = nullptr, *d_theta = nullptr, *d_seed_val = nullptr;
  int *d_mapping = nullptr, *d_seed_idx = nullptr, *d_zero = nullptr, *d_abc = nullptr, *d_mk = nullptr;
  int* d_dense_k = nullptr;
  int* d_dm_pos = nullptr;   // Schedule::dm_pos (the same for every schedule of the potential)
  int nseed = 0;
  // input / output / scratch buffers sized by the capacities
  int *d_itypes = nullptr, *d_js = nullptr, *d_jtypes = nullptr, *d_counts = nullptr;
  double* d_rijs = nullptr;
  double *d_G = nullptr, *d_E = nullptr, *d_F = nullptr, *d_wown = nullptr, *d_vatom = nullptr;
  int *d_in_cnt = nullptr, *d_in_ptr = nullptr, *d_in_cursor = nullptr, *d_in_slot = nullptr, *d_blk = nullptr;
  double *d_partials = nullptr, *d_tot = nullptr;
  int* d_err = nullptr;
  int* d_cfg_ptr = nullptr;
  int cfg_cap = 0;
  double* h_tot = nullptr;   // pinned [7]
  int* h_err = nullptr;      // pinned [1]
  TrainWorkspace train;
  CellScratch cells;
  // launch decisions by (requested lanes, stride, precision): no occupancy
  // queries after the first call, so later calls can be graph-captured
  struct LaunchChoice { int lanes, bps; bool vglobal; size_t smem; int A; };
  int apb = 0;          // requested atoms per block (0: chosen by occupancy)
  int last_apb = 1;
  std::map<long long, LaunchChoice> launch_cache;
  // profiling of the evaluation kernel
  bool profiling = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_events;
  // host-buffer calls (mtp_compute) on large systems copy the inputs in atom
  // chunks on copy_stream while the evaluation kernel runs on earlier chunks
  cudaStream_t copy_stream = nullptr;
  std::vector<cudaEvent_t> chunk_events;
  int prof_used = 0;
  // mtp_execute_potential: page-locked staging of the per-atom rows
  // (allocated on first use, max_atoms x max_nbr)
  double *hp_rij = nullptr, *hp_F = nullptr;
  int *hp_js = nullptr, *hp_jt = nullptr, *hp_cnt = nullptr, *hp_types = nullptr;
  // mtp_compute below kPipelineMinAtoms with page-locked buffers: the call's
  // copies, kernels and read-backs become one CUDA graph, captured on the
  // second consecutive call with the same arguments and replayed while they
  // repeat (a pair style calls with the same buffers every step)
  long long gen = 0;
  HostCallKey graph_key, seen_key;
  cudaGraphExec_t graph_exec = nullptr;
  bool seen_uncapturable = false;
  long long graph_captures = 0, graph_replays = 0;
  // mtp_compute_positions: positions, species and owners of local and ghost
  // atoms [all_cap], candidate lists [neigh_cap], list lengths [max_atoms]
  double* d_xall = nullptr;
  int *d_spall = nullptr, *d_owner = nullptr, *d_neigh = nullptr, *d_numneigh = nullptr;
  size_t all_cap = 0, neigh_cap = 0;
  // statistics
  long long calls = 0;
  double total_ms = 0.0;
  std::string err;
};

namespace {

int fail(mtp_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  else g_create_error = msg;
  return code;
}

// A CUDA call failed: record it, and let work already queued on the handle's
// streams (copies from or to the caller's host buffers among it) finish
// before the error returns, so the caller may reuse or free those buffers.
int cuda_fail(mtp_handle* h, cudaError_t e, const char* what) {
  const int st = fail(h, MTP_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  if (h) {
    cudaStreamSynchronize(h->stream);
    if (h->copy_stream) cudaStreamSynchronize(h->copy_stream);
    cudaGetLastError();
  }
  return st;
}

#define MTP_CUDA(h, call)                                  \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) return cuda_fail((h), e_, #call); \
  } while (0)

DevModel make_model(mtp_handle* h, const DeviceSchedule& ds) {
  DevModel md{};
  const Schedule& s = ds.sched;
  md.entries = ds.d_entries;
  md.nfwd = static_cast<int>(s.fwd.size());
  md.nrev = static_cast<int>(s.rev.size());
  for (int i = 0; i < md.nfwd; ++i) md.fwd[i] = DevPass{s.fwd[i].offset, s.fwd[i].steps};
  for (int i = 0; i < md.nrev; ++i) md.rev[i] = DevPass{s.rev[i].offset, s.rev[i].steps};
  md.radial = h->d_radial;
  md.species = h->d_species;
  md.theta = h->d_theta;
  md.mapping = h->d_mapping;
  md.seed_idx = h->d_seed_idx;
  md.seed_val = h->d_seed_val;
  md.nseed = h->nseed;
  md.zero_list = h->d_zero;
  md.nzero = static_cast<int>(s.zero_list.size());
  md.mono_abc = h->d_abc;
  md.mono_k = h->d_mk;
  md.dense_k = h->d_dense_k;
  md.dm_pos = h->d_dm_pos;
  md.n3_pairs = ds.d_n3_pairs;
  md.n3_off = ds.d_n3_off;
  md.n3_pairs_half = ds.d_n3_pairs_half;
  md.n3_off_half = ds.d_n3_off_half;
  md.warp_steps = ds.d_warp_steps;
  md.Q = s.Q;
  md.npairs = s.npairs;
  md.tri = s.tri ? 1 : 0;
  for (int v = 0; v <= s.D; ++v) md.nmu[v] = s.nmu[v];
  md.S = h->pot.S;
  md.R = h->pot.R;
  md.K = h->pot.K;
  md.M = h->pot.M;
  md.B = h->pot.B;
  md.P = s.P;
  md.D = s.D;
  md.Sa = h->pot.Sa;
  md.v_m = s.v_m;
  md.v_dm = s.v_dm;
  md.v_zero = s.v_zero;
  md.v_one = s.v_one;
  md.v_size = s.v_size;
  md.scaling = h->pot.scaling;
  md.rmin = h->pot.min_dist;
  md.rmax = h->pot.max_dist;
  return md;
}

// Bytes of one operand access of the evaluation kernel (sets the bank model
// the schedule's entry order is tuned for).
inline int access_width(bool fp64, int atoms_per_block) { return (fp64 ? 8 : 4) * atoms_per_block; }

// Dynamic shared memory one block of this part can opt in to.
constexpr size_t kMaxSmemPerBlock = 227 * 1024;

// Schedule for `lanes` threads and `width`-byte operand accesses, built on
// first use.  With `upload` (every call that launches with it) its programs
// also go to the device on first use, after refine_schedule where the value
// space can sit in shared memory (bank order matters only there); a schedule
// that is only sized (launch-shape candidates) is neither refined nor
// uploaded, and no launch ever sees an unrefined copy of a refined one.
int get_schedule(mtp_handle* h, int lanes, int width, DeviceSchedule** out, bool upload = true) {
  const int key = lanes * 64 + width;
  auto it = h->scheds.find(key);
  if (it == h->scheds.end()) {
    DeviceSchedule ds;
    std::string err;
    if (!build_schedule(h->pot, lanes, ds.sched, err, width)) return fail(h, MTP_E_FORMAT, err);
    if (h->d_abc == nullptr) {
      MTP_CUDA(h, dalloc(&h->d_abc, ds.sched.mono_abc.size()));
      MTP_CUDA(h, cudaMemcpy(h->d_abc, ds.sched.mono_abc.data(), ds.sched.mono_abc.size() * sizeof(int),
                             cudaMemcpyHostToDevice));
      MTP_CUDA(h, dalloc(&h->d_mk, ds.sched.mono_k.size()));
      MTP_CUDA(h, cudaMemcpy(h->d_mk, ds.sched.mono_k.data(), ds.sched.mono_k.size() * sizeof(int),
                             cudaMemcpyHostToDevice));
      MTP_CUDA(h, dalloc(&h->d_dense_k, ds.sched.dense_k.size()));
      MTP_CUDA(h, cudaMemcpy(h->d_dense_k, ds.sched.dense_k.data(), ds.sched.dense_k.size() * sizeof(int),
                             cudaMemcpyHostToDevice));
      MTP_CUDA(h, dalloc(&h->d_dm_pos, ds.sched.dm_pos.size()));
      MTP_CUDA(h, cudaMemcpy(h->d_dm_pos, ds.sched.dm_pos.data(), ds.sched.dm_pos.size() * sizeof(int),
                             cudaMemcpyHostToDevice));
      MTP_CUDA(h, dalloc(&h->d_zero, ds.sched.zero_list.size()));
      if (!ds.sched.zero_list.empty())
        MTP_CUDA(h, cudaMemcpy(h->d_zero, ds.sched.zero_list.data(), ds.sched.zero_list.size() * sizeof(int),
                               cudaMemcpyHostToDevice));
    }
    it = h->scheds.emplace(key, ds).first;
  }
  DeviceSchedule& ds = it->second;
  if (upload && ds.d_entries == nullptr) {
    if (static_cast<size_t>(ds.sched.v_size) * width <= kMaxSmemPerBlock) refine_schedule(ds.sched);
    const auto& ent = ds.sched.entries;
    MTP_CUDA(h, dalloc(&ds.d_entries, ent.size() / 2));
    MTP_CUDA(h, cudaMemcpy(ds.d_entries, ent.data(), ent.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    std::vector<int> ws;
    for (const Pass& p : ds.sched.fwd) ws.insert(ws.end(), p.wsteps.begin(), p.wsteps.end());
    for (const Pass& p : ds.sched.rev) ws.insert(ws.end(), p.wsteps.begin(), p.wsteps.end());
    MTP_CUDA(h, dalloc(&ds.d_warp_steps, ws.size()));
    MTP_CUDA(h, cudaMemcpy(ds.d_warp_steps, ws.data(), ws.size() * sizeof(int), cudaMemcpyHostToDevice));
    if (ds.sched.tri) {
      const auto& np = ds.sched.n3_pairs;
      const auto& no = ds.sched.n3_off;
      MTP_CUDA(h, dalloc(&ds.d_n3_pairs, np.size()));
      MTP_CUDA(h, cudaMemcpy(ds.d_n3_pairs, np.data(), np.size() * sizeof(int), cudaMemcpyHostToDevice));
      MTP_CUDA(h, dalloc(&ds.d_n3_off, no.size()));
      MTP_CUDA(h, cudaMemcpy(ds.d_n3_off, no.data(), no.size() * sizeof(int), cudaMemcpyHostToDevice));
      const auto& nph = ds.sched.n3_pairs_half;
      const auto& noh = ds.sched.n3_off_half;
      MTP_CUDA(h, dalloc(&ds.d_n3_pairs_half, nph.size()));
      MTP_CUDA(h, cudaMemcpy(ds.d_n3_pairs_half, nph.data(), nph.size() * sizeof(int), cudaMemcpyHostToDevice));
      MTP_CUDA(h, dalloc(&ds.d_n3_off_half, noh.size()));
      MTP_CUDA(h, cudaMemcpy(ds.d_n3_off_half, noh.data(), noh.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
  }
  *out = &ds;
  return MTP_OK;
}

int upload_coeffs(mtp_handle* h) {
  const Potential& p = h->pot;
  MTP_CUDA(h, cudaMemcpy(h->d_radial, p.radial.data(), p.radial.size() * sizeof(double), cudaMemcpyHostToDevice));
  MTP_CUDA(h, cudaMemcpy(h->d_species, p.species.data(), p.species.size() * sizeof(double), cudaMemcpyHostToDevice));
  MTP_CUDA(h, cudaMemcpy(h->d_theta, p.moment.data(), p.moment.size() * sizeof(double), cudaMemcpyHostToDevice));
  std::vector<int> si;
  std::vector<double> sv;
  seed_list(p, si, sv);
  // seeds go to the adjoint positions of their moments
  std::vector<int> dm_pos;
  adjoint_layout(p, dm_pos);
  for (int& k : si) k = dm_pos[k];
  h->nseed = static_cast<int>(si.size());
  MTP_CUDA(h, cudaMemcpy(h->d_seed_idx, si.data(), si.size() * sizeof(int), cudaMemcpyHostToDevice));
  MTP_CUDA(h, cudaMemcpy(h->d_seed_val, sv.data(), sv.size() * sizeof(double), cudaMemcpyHostToDevice));
  return MTP_OK;
}

void free_handle(mtp_handle* h) {
  if (!h) return;
  auto F = [](void* p) { if (p) cudaFree(p); };
  for (auto& kv : h->scheds) {
    F(kv.second.d_entries);
    F(kv.second.d_n3_pairs);
    F(kv.second.d_n3_off);
    F(kv.second.d_n3_pairs_half);
    F(kv.second.d_n3_off_half);
    F(kv.second.d_warp_steps);
  }
  F(h->d_radial); F(h->d_species); F(h->d_theta); F(h->d_seed_val);
  F(h->d_mapping); F(h->d_seed_idx); F(h->d_zero); F(h->d_abc); F(h->d_mk); F(h->d_dense_k); F(h->d_dm_pos);
  F(h->d_itypes); F(h->d_js); F(h->d_jtypes); F(h->d_counts); F(h->d_rijs);
  F(h->d_G); F(h->d_E); F(h->d_F); F(h->d_wown); F(h->d_vatom);
  F(h->d_in_cnt); F(h->d_in_ptr); F(h->d_in_cursor); F(h->d_in_slot); F(h->d_blk);
  F(h->d_partials); F(h->d_tot); F(h->d_err); F(h->d_cfg_ptr); F(h->d_vscratch);
  F(h->d_xall); F(h->d_spall); F(h->d_owner); F(h->d_neigh); F(h->d_numneigh);
  train_free(h->train);
  F(h->cells.cell); F(h->cells.img); F(h->cells.cnt); F(h->cells.ptr); F(h->cells.cursor); F(h->cells.atoms);
  F(h->cells.blk);
  for (auto& ev : h->prof_events) {
    cudaEventDestroy(ev.first);
    cudaEventDestroy(ev.second);
  }
  if (h->h_tot) cudaFreeHost(h->h_tot);
  if (h->h_err) cudaFreeHost(h->h_err);
  for (auto ev : h->chunk_events) cudaEventDestroy(ev);
  if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
  if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
  for (void* q : {static_cast<void*>(h->hp_rij), static_cast<void*>(h->hp_F), static_cast<void*>(h->hp_js),
                  static_cast<void*>(h->hp_jt), static_cast<void*>(h->hp_cnt), static_cast<void*>(h->hp_types)})
    if (q) cudaFreeHost(q);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
}

// Launch shape for the evaluation kernel.  Candidates are (lanes, atoms per
// block) with the value space in shared memory; the one with the most atoms
// in flight per SM (A x blocks/SM) wins, ties going to more warps.  When none
// fits, the value space moves to global memory (A = 1).  Decisions are cached
// per (request, stride, precision), so later calls make no occupancy queries.
int pick_launch(mtp_handle* h, int natoms, int stride, DeviceSchedule** ds_out, int* blocks_out, bool fp64,
                bool* vglobal_out) {
  const long long key = (static_cast<long long>(h->threads) << 40) | (static_cast<long long>(h->apb) << 36) |
                        (static_cast<long long>(h->blocks_per_sm) << 28) | (static_cast<long long>(stride) << 2) |
                        (fp64 ? 1 : 0);
  auto hit = h->launch_cache.find(key);
  mtp_handle::LaunchChoice c{};
  if (hit != h->launch_cache.end()) {
    c = hit->second;
  } else {
    std::vector<int> lanes_c = {h->threads};
    for (int alt : {256, 128})
      if (alt < h->threads) lanes_c.push_back(alt);
    std::vector<int> a_c;
    if (h->apb > 0) a_c = {h->apb};
    else if (fp64) a_c = {2, 1};
    else a_c = {4, 2, 1};
    int best = -1;
    for (int lanes : lanes_c) {
      for (int A : a_c) {
        if (!eval_variant_exists(fp64, false, A)) continue;
        DeviceSchedule* ds = nullptr;
        int st = get_schedule(h, lanes, access_width(fp64, A), &ds, false);
        if (st != MTP_OK) return st;
        const DevModel md = make_model(h, *ds);
        int bps = eval_blocks_per_sm(md, stride, lanes, fp64, false, A);
        if (h->blocks_per_sm > 0) bps = std::min(bps, h->blocks_per_sm);
        if (bps <= 0) continue;
        const int score = (A * bps) * 1024 + bps * lanes / 32;
        if (score > best) {
          best = score;
          c = mtp_handle::LaunchChoice{lanes, bps, false, 0, A};
        }
      }
    }
    if (best < 0) {
      // value space in global memory: 512 lanes give an SM 16 warps with one
      // block, so the blocks' value spaces stay within L2
      const int lanes = 512;
      DeviceSchedule* ds = nullptr;
      int st = get_schedule(h, lanes, access_width(fp64, 1), &ds, false);
      if (st != MTP_OK) return st;
      int bps = eval_blocks_per_sm(make_model(h, *ds), stride, lanes, fp64, true, 1);
      if (h->blocks_per_sm > 0) bps = std::min(bps, h->blocks_per_sm);
      if (bps <= 0)
        return fail(h, MTP_E_CAPACITY, "the evaluation block does not fit in shared memory for this basis and max_nbr");
      c = mtp_handle::LaunchChoice{lanes, std::min(bps, 1), true, 0, 1};
    }
    DeviceSchedule* ds = nullptr;
    int st = get_schedule(h, c.lanes, access_width(fp64, c.A), &ds);
    if (st != MTP_OK) return st;
    c.smem = eval_smem_bytes(make_model(h, *ds), stride, c.lanes, fp64, c.vglobal, c.A);
    h->launch_cache[key] = c;
  }
  DeviceSchedule* ds = nullptr;
  int st = get_schedule(h, c.lanes, access_width(fp64, c.A), &ds);
  if (st != MTP_OK) return st;
  const long long groups = (static_cast<long long>(natoms) + c.A - 1) / c.A;
  const long long blocks = std::max(1LL, std::min<long long>(static_cast<long long>(c.bps) * h->sm_count, groups));
  if (c.vglobal) {
    const size_t need = static_cast<size_t>(blocks) * ds->sched.v_size * c.A * (fp64 ? sizeof(double) : sizeof(float));
    if (need > h->vscratch_bytes) {
      if (h->d_vscratch) cudaFree(h->d_vscratch);
      h->d_vscratch = nullptr;
      h->vscratch_bytes = 0;
      MTP_CUDA(h, cudaMalloc(&h->d_vscratch, need));
      h->vscratch_bytes = need;
      ++h->gen;
    }
  }
  *ds_out = ds;
  *blocks_out = static_cast<int>(blocks);
  *vglobal_out = c.vglobal;
  h->last_threads = c.lanes;
  h->last_blocks = static_cast<int>(blocks);
  h->last_bps = c.bps;
  h->last_vglobal = c.vglobal;
  h->last_smem = c.smem;
  h->last_apb = c.A;
  return MTP_OK;
}

// Evaluation kernel on atoms [lo, lo + n) of device rows (site energies and
// per-slot gradients of those atoms).
int eval_range(mtp_handle* h, int lo, int n, int stride, const int* itypes, const double* rijs, const int* jtypes,
               const int* counts) {
  const bool fp64 = h->precision == MTP_PRECISION_FP64;
  DeviceSchedule* ds = nullptr;
  int blocks = 0;
  bool vglobal = false;
  int st = pick_launch(h, n, stride, &ds, &blocks, fp64, &vglobal);
  if (st != MTP_OK) return st;
  DevModel md = make_model(h, *ds);
  const size_t rows = static_cast<size_t>(lo) * stride;
  DevIO io{};
  io.natoms = n;
  io.nbr_stride = stride;
  io.n_pad = stride;
  io.itypes = itypes + lo;
  io.rijs = rijs + 3 * rows;
  io.jtypes = jtypes + rows;
  io.counts = counts ? counts + lo : nullptr;
  io.site_energy = h->d_E + lo;
  io.pair_grad = h->d_G + 3 * rows;
  io.err = h->d_err;
  io.vscratch = h->d_vscratch;
  MTP_CUDA(h, launch_eval(md, io, h->last_threads, blocks, fp64, vglobal, h->last_apb, h->stream));
  return MTP_OK;
}

// Profiling events around the evaluation launches of one call (mtp_profile).
int prof_begin(mtp_handle* h, cudaEvent_t* e1) {
  *e1 = nullptr;
  if (!h->profiling) return MTP_OK;
  if (h->prof_used == static_cast<int>(h->prof_events.size())) {
    cudaEvent_t a, b;
    MTP_CUDA(h, cudaEventCreate(&a));
    MTP_CUDA(h, cudaEventCreate(&b));
    h->prof_events.push_back({a, b});
  }
  const cudaEvent_t e0 = h->prof_events[h->prof_used].first;
  *e1 = h->prof_events[h->prof_used].second;
  ++h->prof_used;
  MTP_CUDA(h, cudaEventRecord(e0, h->stream));
  return MTP_OK;
}

// Evaluate site energies and per-slot gradients, then forces and virials.
int run_device(mtp_handle* h, int natoms, int stride, const int* itypes, const double* rijs, const int* js,
               const int* jtypes, const int* counts, bool rebuild_incoming, double* forces, double* vatom) {
  if (rebuild_incoming) {
    MTP_CUDA(h, launch_incoming(natoms, stride, js, jtypes, counts, h->d_in_cnt, h->d_in_ptr, h->d_in_cursor,
                                h->d_in_slot, h->d_blk, h->stream));
  }
  cudaEvent_t e1 = nullptr;
  int st = prof_begin(h, &e1);
  if (st != MTP_OK) return st;
  st = eval_range(h, 0, natoms, stride, itypes, rijs, jtypes, counts);
  if (st != MTP_OK) return st;
  if (e1) MTP_CUDA(h, cudaEventRecord(e1, h->stream));
  MTP_CUDA(h, launch_force_gather(natoms, stride, rijs, counts, h->d_G, h->d_in_ptr, h->d_in_slot, forces,
                                  h->d_wown, vatom, h->stream));
  return MTP_OK;
}

// Systems from this size on are copied in chunks that overlap the evaluation.
constexpr int kPipelineMinAtoms = 65536;
constexpr int kPipelineChunks = 16;

// run_device for host input buffers: the inputs of chunk k go up on the copy
// stream while the evaluation kernel works on chunk k-1 (events order each
// chunk's kernel after its copies); the incoming lists and the force gather
// need every row and follow the last chunk.  With pinned host buffers the
// copies overlap the kernels; pageable ones are still correct.
int run_host_pipelined_body(mtp_handle* h, int natoms, int stride, const int* itypes, const double* rijs,
                            const int* js, const int* jtypes, const int* counts, double* vatom) {
  const cudaStream_t s = h->stream;
  if (!h->copy_stream) MTP_CUDA(h, cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
  const int nch = std::max(1, std::min(kPipelineChunks, natoms / (kPipelineMinAtoms / 2)));
  while (static_cast<int>(h->chunk_events.size()) < nch + 1) {
    cudaEvent_t ev;
    MTP_CUDA(h, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    h->chunk_events.push_back(ev);
  }
  // the copies may only overwrite the device rows once earlier work on the
  // compute stream is done with them
  MTP_CUDA(h, cudaEventRecord(h->chunk_events[nch], s));
  MTP_CUDA(h, cudaStreamWaitEvent(h->copy_stream, h->chunk_events[nch], 0));
  for (int k = 0; k < nch; ++k) {
    const size_t lo = static_cast<size_t>(natoms) * k / nch, hi = static_cast<size_t>(natoms) * (k + 1) / nch;
    const size_t n = hi - lo, r0 = lo * stride, nr = n * stride;
    const cudaStream_t c = h->copy_stream;
    MTP_CUDA(h, cudaMemcpyAsync(h->d_itypes + lo, itypes + lo, n * sizeof(int), cudaMemcpyHostToDevice, c));
    MTP_CUDA(h, cudaMemcpyAsync(h->d_rijs + 3 * r0, rijs + 3 * r0, 3 * nr * sizeof(double), cudaMemcpyHostToDevice, c));
    MTP_CUDA(h, cudaMemcpyAsync(h->d_js + r0, js + r0, nr * sizeof(int), cudaMemcpyHostToDevice, c));
    MTP_CUDA(h, cudaMemcpyAsync(h->d_jtypes + r0, jtypes + r0, nr * sizeof(int), cudaMemcpyHostToDevice, c));
    if (counts) MTP_CUDA(h, cudaMemcpyAsync(h->d_counts + lo, counts + lo, n * sizeof(int), cudaMemcpyHostToDevice, c));
    MTP_CUDA(h, cudaEventRecord(h->chunk_events[k], c));
  }
  cudaEvent_t e1 = nullptr;
  for (int k = 0; k < nch; ++k) {
    const int lo = static_cast<int>(static_cast<size_t>(natoms) * k / nch);
    const int hi = static_cast<int>(static_cast<size_t>(natoms) * (k + 1) / nch);
    MTP_CUDA(h, cudaStreamWaitEvent(s, h->chunk_events[k], 0));
    if (k == 0) {
      int st = prof_begin(h, &e1);
      if (st != MTP_OK) return st;
    }
    int st = eval_range(h, lo, hi - lo, stride, h->d_itypes, h->d_rijs, h->d_jtypes, counts ? h->d_counts : nullptr);
    if (st != MTP_OK) return st;
  }
  if (e1) MTP_CUDA(h, cudaEventRecord(e1, s));
  MTP_CUDA(h, launch_incoming(natoms, stride, h->d_js, h->d_jtypes, counts ? h->d_counts : nullptr, h->d_in_cnt,
                              h->d_in_ptr, h->d_in_cursor, h->d_in_slot, h->d_blk, s));
  MTP_CUDA(h, launch_force_gather(natoms, stride, h->d_rijs, counts ? h->d_counts : nullptr, h->d_G, h->d_in_ptr,
                                  h->d_in_slot, h->d_F, h->d_wown, vatom, s));
  return MTP_OK;
}

// A failure part-way leaves copies from the caller's host buffers in flight:
// they finish before the call returns, so the caller may free the buffers.
int run_host_pipelined(mtp_handle* h, int natoms, int stride, const int* itypes, const double* rijs, const int* js,
                       const int* jtypes, const int* counts, double* vatom) {
  const int st = run_host_pipelined_body(h, natoms, stride, itypes, rijs, js, jtypes, counts, vatom);
  if (st != MTP_OK && h->copy_stream) cudaStreamSynchronize(h->copy_stream);
  return st;
}

// Status from the device error flags already copied to h_err by finished work
// (the flags are cleared on the device when set).
int take_err_flags(mtp_handle* h) {
  const int f = *h->h_err;
  if (f) MTP_CUDA(h, cudaMemsetAsync(h->d_err, 0, sizeof(int), h->stream));
  if (f & kErrSpecies) return fail(h, MTP_E_SPECIES, "a species index is outside [0, species_count)");
  if (f & kErrCapacity) return fail(h, MTP_E_CAPACITY, "a neighbour count exceeds the row length");
  if (f & kErrNonFinite) return fail(h, MTP_E_NONFINITE, "non-finite energy or force produced on the device");
  return MTP_OK;
}

int read_err_flags(mtp_handle* h) {
  MTP_CUDA(h, cudaMemcpyAsync(h->h_err, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  MTP_CUDA(h, cudaStreamSynchronize(h->stream));
  return take_err_flags(h);
}

// True when [p, p + bytes) is page-locked host memory (cudaHostAlloc or
// cudaHostRegister): its first and last byte are checked on every call, so a
// buffer freed and replaced by pageable memory at the same address is seen.
bool host_pinned(const void* p, size_t bytes) {
  if (!p || bytes == 0) return true;
  const char* c = static_cast<const char*>(p);
  for (const char* q : {c, c + bytes - 1}) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, q) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    if (a.type != cudaMemoryTypeHost) return false;
  }
  return true;
}

// Enqueue one host-buffer call below kPipelineMinAtoms on the handle's stream:
// input copies, evaluation, totals, and the copies of the results and of the
// device error flags back to the host.  Nothing here synchronises or
// allocates, so it can be captured into a graph.
int enqueue_small_call(mtp_handle* h, int natoms, int stride, const int* itypes, const double* rijs, const int* js,
                       const int* jtypes, const int* counts, int flags, double* forces, double* eatom,
                       double* vatom) {
  const cudaStream_t s = h->stream;
  const size_t N = natoms, NS = N * stride;
  if (natoms > 0) {
    MTP_CUDA(h, cudaMemcpyAsync(h->d_itypes, itypes, N * sizeof(int), cudaMemcpyHostToDevice, s));
    MTP_CUDA(h, cudaMemcpyAsync(h->d_rijs, rijs, 3 * NS * sizeof(double), cudaMemcpyHostToDevice, s));
    MTP_CUDA(h, cudaMemcpyAsync(h->d_js, js, NS * sizeof(int), cudaMemcpyHostToDevice, s));
    MTP_CUDA(h, cudaMemcpyAsync(h->d_jtypes, jtypes, NS * sizeof(int), cudaMemcpyHostToDevice, s));
    if (counts) MTP_CUDA(h, cudaMemcpyAsync(h->d_counts, counts, N * sizeof(int), cudaMemcpyHostToDevice, s));
  }
  int st = run_device(h, natoms, stride, h->d_itypes, h->d_rijs, h->d_js, h->d_jtypes, counts ? h->d_counts : nullptr,
                      true, h->d_F, (flags & MTP_VATOM) ? h->d_vatom : nullptr);
  if (st != MTP_OK) return st;
  MTP_CUDA(h, launch_totals(natoms, h->d_E, h->d_wown, h->d_partials, h->d_tot, s));
  if (natoms > 0) {
    MTP_CUDA(h, cudaMemcpyAsync(forces, h->d_F, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (flags & MTP_EATOM) MTP_CUDA(h, cudaMemcpyAsync(eatom, h->d_E, N * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (flags & MTP_VATOM)
      MTP_CUDA(h, cudaMemcpyAsync(vatom, h->d_vatom, 6 * N * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  MTP_CUDA(h, cudaMemcpyAsync(h->h_tot, h->d_tot, 7 * sizeof(double), cudaMemcpyDeviceToHost, s));
  MTP_CUDA(h, cudaMemcpyAsync(h->h_err, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
  return MTP_OK;
}

// Run one synchronous host-buffer call.  With every host buffer page-locked
// (pinned), the second consecutive call with the same key is captured into a
// graph and later ones replay it (one launch instead of about twenty copies
// and kernels); otherwise enqueue() runs directly.  The results are the same
// either way: the graph holds the same operations.
template <typename Enqueue>
int run_graphable(mtp_handle* h, const HostCallKey& key, bool pinned, Enqueue&& enqueue) {
  const cudaStream_t s = h->stream;
  bool launched = false;
  if (pinned && h->graph_exec && key == h->graph_key) {
    MTP_CUDA(h, cudaGraphLaunch(h->graph_exec, s));
    launched = true;
    ++h->graph_replays;
  } else if (pinned && key == h->seen_key && !h->seen_uncapturable) {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ex = nullptr;
    bool ok = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
      const int cst = enqueue();
      const cudaError_t ce = cudaStreamEndCapture(s, &g);
      ok = cst == MTP_OK && ce == cudaSuccess && g != nullptr;
    }
    if (ok) ok = cudaGraphInstantiate(&ex, g, 0) == cudaSuccess;
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    if (ok) {
      if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
      h->graph_exec = ex;
      h->graph_key = key;
      MTP_CUDA(h, cudaGraphLaunch(ex, s));
      launched = true;
      ++h->graph_captures;
    } else {
      h->seen_uncapturable = true;
    }
  } else if (pinned) {
    h->seen_key = key;
    h->seen_uncapturable = false;
  }
  if (!launched) {
    const int st = enqueue();
    if (st != MTP_OK) {
      cudaStreamSynchronize(s);   // copies from the caller's buffers complete before the error returns
      return st;
    }
  }
  MTP_CUDA(h, cudaStreamSynchronize(s));
  return take_err_flags(h);
}

// One host-buffer call of mtp_compute below kPipelineMinAtoms (run_graphable).
int run_small_call(mtp_handle* h, int natoms, int stride, const int* itypes, const double* rijs, const int* js,
                   const int* jtypes, const int* counts, int flags, double* forces, double* eatom, double* vatom) {
  const size_t N = natoms, NS = N * stride;
  HostCallKey key;
  key.kind = 0;
  key.natoms = natoms;
  key.stride = stride;
  key.flags = flags & (MTP_EATOM | MTP_VATOM);
  key.gen = h->gen;
  const void* ptrs[8] = {itypes, rijs, js, jtypes, counts, forces,
                         (flags & MTP_EATOM) ? eatom : nullptr, (flags & MTP_VATOM) ? vatom : nullptr};
  for (int k = 0; k < 8; ++k) key.p[k] = ptrs[k];
  const bool pinned = natoms > 0 && !h->profiling && host_pinned(itypes, N * sizeof(int)) &&
                      host_pinned(rijs, 3 * NS * sizeof(double)) && host_pinned(js, NS * sizeof(int)) &&
                      host_pinned(jtypes, NS * sizeof(int)) && host_pinned(counts, counts ? N * sizeof(int) : 0) &&
                      host_pinned(forces, 3 * N * sizeof(double)) &&
                      host_pinned(key.p[6], (flags & MTP_EATOM) ? N * sizeof(double) : 0) &&
                      host_pinned(key.p[7], (flags & MTP_VATOM) ? 6 * N * sizeof(double) : 0);
  return run_graphable(h, key, pinned, [&]() {
    return enqueue_small_call(h, natoms, stride, itypes, rijs, js, jtypes, counts, flags, forces, eatom, vatom);
  });
}

bool ends_with(const std::string& s, const std::string& suf) {
  return s.size() >= suf.size() && s.compare(s.size() - suf.size(), suf.size(), suf) == 0;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int mtp_abi_version(void) { return MTP_B200_ABI_VERSION; }

int mtp_parse_info(const char* path, int* out8, char* errbuf, int err_len) {
  if (!path || !out8) return MTP_E_INVALID;
  Potential pot;
  std::string err;
  if (!parse_mtp_file(path, pot, err)) {
    if (errbuf && err_len > 0) std::snprintf(errbuf, err_len, "%s", err.c_str());
    return MTP_E_FORMAT;
  }
  int D = 0;
  for (int k = 0; k < pot.B; ++k) D = std::max(D, pot.basic[4 * k + 1] + pot.basic[4 * k + 2] + pot.basic[4 * k + 3]);
  const int v[8] = {pot.S, pot.R, pot.K, pot.M, pot.B, pot.T, pot.Sa, D};
  std::memcpy(out8, v, sizeof(v));
  return MTP_OK;
}

int mtp_schedule_emulate(const char* path, int lanes, int width, const double* basic, double* moments,
                         double* dmoments, double* energy_part) {
  if (!path || !basic || !moments || !dmoments) return MTP_E_INVALID;
  if (width != 4 && width != 8 && width != 16) return MTP_E_INVALID;
  Potential pot;
  std::string err;
  if (!parse_mtp_file(path, pot, err)) return MTP_E_FORMAT;
  Schedule s;
  if (!build_schedule(pot, lanes, s, err, width)) return MTP_E_FORMAT;
  refine_schedule(s);
  std::vector<double> V(s.v_size, 0.0);
  for (int k = 0; k < pot.B; ++k) V[s.v_m + k] = basic[k];
  double e = emulate_schedule(pot, s, V);
  for (int k = 0; k < pot.M; ++k) {
    moments[k] = V[s.v_m + k];
    dmoments[k] = V[s.v_dm + s.dm_pos[k]];
  }
  if (energy_part) *energy_part = e;
  return MTP_OK;
}

int mtp_create(const char* mtp_path, int max_atoms, int max_nbr, double cutoff, int debug_level, int precision,
               mtp_handle** out) {
  if (!out) return fail(nullptr, MTP_E_INVALID, "out is null");
  *out = nullptr;
  if (!mtp_path) return fail(nullptr, MTP_E_INVALID, "mtp_path is null");
  if (max_atoms <= 0 || max_nbr <= 0 || !(cutoff > 0.0))
    return fail(nullptr, MTP_E_INVALID, "max_atoms, max_nbr and cutoff must be positive");
  if (precision != MTP_PRECISION_FP64 && precision != MTP_PRECISION_MIXED)
    return fail(nullptr, MTP_E_INVALID, "precision must be MTP_PRECISION_FP64 or MTP_PRECISION_MIXED");
  if (max_nbr > 1024) return fail(nullptr, MTP_E_CAPACITY, "max_nbr above the supported 1024");
  if (static_cast<long long>(max_atoms) * max_nbr >= (1LL << 31))
    return fail(nullptr, MTP_E_CAPACITY, "max_atoms * max_nbr must stay below 2^31");
  std::string path(mtp_path);
  if (ends_with(path, ".bin"))
    return fail(nullptr, MTP_E_FORMAT,
                "'" + path + "' looks like a jax.export .bin; this engine reads the .mtp potential file itself");
  auto* h = new mtp_handle();
  h->max_atoms = max_atoms;
  h->max_nbr = max_nbr;
  h->cutoff = cutoff;
  h->debug = debug_level;
  h->precision = precision;
  std::string err;
  if (!parse_mtp_file(path, h->pot, err)) {
    delete h;
    return fail(nullptr, MTP_E_FORMAT, err);
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    delete h;
    return fail(nullptr, MTP_E_NODEVICE, "no CUDA device");
  }
  auto bail = [&](int code) {
    g_create_error = h->err;
    free_handle(h);
    return code;
  };
  if (cudaGetDevice(&h->device) != cudaSuccess) return bail(cuda_fail(h, cudaGetLastError(), "cudaGetDevice"));
  cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, h->device);
  if (cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(cuda_fail(h, cudaGetLastError(), "cudaStreamCreate"));
  h->stream = h->own_stream;
  const Potential& p = h->pot;
  const size_t N = static_cast<size_t>(max_atoms), NS = N * max_nbr;
  bool ok = dalloc(&h->d_radial, p.radial.size()) == cudaSuccess && dalloc(&h->d_species, p.S) == cudaSuccess &&
            dalloc(&h->d_theta, p.Sa) == cudaSuccess && dalloc(&h->d_mapping, p.Sa) == cudaSuccess &&
            dalloc(&h->d_seed_idx, p.Sa) == cudaSuccess && dalloc(&h->d_seed_val, p.Sa) == cudaSuccess &&
            dalloc(&h->d_itypes, N) == cudaSuccess && dalloc(&h->d_js, NS) == cudaSuccess &&
            dalloc(&h->d_jtypes, NS) == cudaSuccess && dalloc(&h->d_counts, N) == cudaSuccess &&
            dalloc(&h->d_rijs, 3 * NS) == cudaSuccess && dalloc(&h->d_G, 3 * NS) == cudaSuccess &&
            dalloc(&h->d_E, N) == cudaSuccess && dalloc(&h->d_F, 3 * N) == cudaSuccess &&
            dalloc(&h->d_wown, 6 * N) == cudaSuccess && dalloc(&h->d_vatom, 6 * N) == cudaSuccess &&
            dalloc(&h->d_in_cnt, N) == cudaSuccess && dalloc(&h->d_in_ptr, N + 1) == cudaSuccess &&
            dalloc(&h->d_in_cursor, N) == cudaSuccess && dalloc(&h->d_in_slot, NS) == cudaSuccess &&
            dalloc(&h->d_blk, (N + 1023) / 1024 + 1) == cudaSuccess &&
            dalloc(&h->d_partials, 7 * kReduceBlocks) == cudaSuccess && dalloc(&h->d_tot, 8) == cudaSuccess &&
            dalloc(&h->d_err, 1) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    h->err = "device allocation failed for the requested capacities";
    return bail(MTP_E_OOM);
  }
  if (cudaMallocHost(&h->h_tot, 8 * sizeof(double)) != cudaSuccess ||
      cudaMallocHost(&h->h_err, sizeof(int)) != cudaSuccess) {
    h->err = "pinned host allocation failed";
    return bail(MTP_E_OOM);
  }
  cudaMemset(h->d_err, 0, sizeof(int));
  if (cudaMemcpy(h->d_mapping, p.mapping.data(), p.Sa * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(cuda_fail(h, cudaGetLastError(), "upload mapping"));
  int st = upload_coeffs(h);
  if (st != MTP_OK) return bail(st);
  DeviceSchedule* ds = nullptr;
  st = get_schedule(h, h->threads, access_width(precision == MTP_PRECISION_FP64, 1), &ds, false);
  if (st != MTP_OK) return bail(st);
  if (h->debug >= 1) {
    std::fprintf(stderr, "[mtp_b200] %s: S=%d R=%d K=%d M=%d B=%d T=%d Sa=%d; %d fwd + %d rev passes, %d value slots\n",
                 path.c_str(), p.S, p.R, p.K, p.M, p.B, p.T, p.Sa, static_cast<int>(ds->sched.fwd.size()),
                 static_cast<int>(ds->sched.rev.size()), ds->sched.v_size);
  }
  *out = h;
  return MTP_OK;
}

void mtp_destroy(mtp_handle* h) {
  if (!h) return;
  if (h->debug >= 1 && h->calls > 0)
    std::fprintf(stderr, "[mtp_b200] %lld calls, %.3f ms total, %.3f ms/call\n", h->calls, h->total_ms,
                 h->total_ms / h->calls);
  if (h->stream) cudaStreamSynchronize(h->stream);
  free_handle(h);
}

const char* mtp_last_error(const mtp_handle* h) { return h ? h->err.c_str() : g_create_error.c_str(); }

int mtp_set_stream(mtp_handle* h, void* s) {
  if (!h) return MTP_E_INVALID;
  h->stream = static_cast<cudaStream_t>(s);
  return MTP_OK;
}

int mtp_use_own_stream(mtp_handle* h) {
  if (!h) return MTP_E_INVALID;
  h->stream = h->own_stream;
  return MTP_OK;
}

int mtp_get_info(const mtp_handle* h, int* out8) {
  if (!h || !out8) return MTP_E_INVALID;
  const Potential& p = h->pot;
  int D = 0;
  for (int k = 0; k < p.B; ++k) D = std::max(D, p.basic[4 * k + 1] + p.basic[4 * k + 2] + p.basic[4 * k + 3]);
  const int v[8] = {p.S, p.R, p.K, p.M, p.B, p.T, p.Sa, D};
  std::memcpy(out8, v, sizeof(v));
  return MTP_OK;
}

int mtp_get_stats(const mtp_handle* h, double* out4) {
  if (!h || !out4) return MTP_E_INVALID;
  out4[0] = static_cast<double>(h->calls);
  out4[1] = h->total_ms;
  out4[2] = static_cast<double>(h->graph_captures);
  out4[3] = static_cast<double>(h->graph_replays);
  return MTP_OK;
}

int mtp_set_coeffs(mtp_handle* h, const double* species, const double* moment, const double* radial) {
  if (!h) return MTP_E_INVALID;
  Potential& p = h->pot;
  if (species) std::copy(species, species + p.S, p.species.begin());
  if (moment) std::copy(moment, moment + p.Sa, p.moment.begin());
  if (radial) std::copy(radial, radial + p.radial.size(), p.radial.begin());
  MTP_CUDA(h, cudaStreamSynchronize(h->stream));
  ++h->gen;
  return upload_coeffs(h);
}

int mtp_set_launch(mtp_handle* h, int threads, int bps, int apb) {
  if (!h) return MTP_E_INVALID;
  if (threads != 128 && threads != 256 && threads != 512)
    return fail(h, MTP_E_INVALID, "threads_per_block must be 128, 256 or 512");
  if (apb != 0 && apb != 1 && apb != 2 && apb != 4)
    return fail(h, MTP_E_INVALID, "atoms_per_block must be 0 (automatic), 1, 2 or 4");
  h->threads = threads;
  h->blocks_per_sm = std::max(0, bps);
  h->apb = apb;
  ++h->gen;
  return MTP_OK;
}

int mtp_get_launch(const mtp_handle* h, int* out5) {
  if (!h || !out5) return MTP_E_INVALID;
  out5[0] = h->last_threads;
  out5[1] = h->last_blocks;
  out5[2] = static_cast<int>(h->last_smem);
  out5[3] = h->last_bps;
  out5[4] = h->last_apb;
  return MTP_OK;
}

int mtp_sync_status(mtp_handle* h) {
  if (!h) return MTP_E_INVALID;
  return read_err_flags(h);
}

int mtp_compute_device(mtp_handle* h, int natoms, int stride, const int* d_itypes, const double* d_rijs,
                       const int* d_js, const int* d_jtypes, const int* d_counts, int flags, double* d_energy,
                       double* d_forces, double* d_virial, double* d_eatom, double* d_vatom) {
  if (!h) return MTP_E_INVALID;
  if (natoms < 0 || stride <= 0) return fail(h, MTP_E_INVALID, "natoms must be >= 0 and nbr_stride > 0");
  if (natoms > h->max_atoms) return fail(h, MTP_E_CAPACITY, "natoms exceeds max_atoms");
  if (stride > h->max_nbr) return fail(h, MTP_E_CAPACITY, "nbr_stride exceeds max_nbr");
  if (natoms > 0 && (!d_itypes || !d_rijs || !d_js || !d_jtypes || !d_forces))
    return fail(h, MTP_E_INVALID, "null input or forces pointer");
  if ((flags & MTP_EFLAG) && !d_energy) return fail(h, MTP_E_INVALID, "MTP_EFLAG without an energy pointer");
  if ((flags & MTP_VFLAG) && !d_virial) return fail(h, MTP_E_INVALID, "MTP_VFLAG without a virial pointer");
  if ((flags & MTP_EATOM) && !d_eatom) return fail(h, MTP_E_INVALID, "MTP_EATOM without an eatom pointer");
  if ((flags & MTP_VATOM) && !d_vatom) return fail(h, MTP_E_INVALID, "MTP_VATOM without a vatom pointer");
  const bool rebuild = !(flags & MTP_REUSE_NEIGHBORS);
  int st = run_device(h, natoms, stride, d_itypes, d_rijs, d_js, d_jtypes, d_counts, rebuild, d_forces,
                      (flags & MTP_VATOM) ? d_vatom : nullptr);
  if (st != MTP_OK) return st;
  if (flags & (MTP_EFLAG | MTP_VFLAG)) {
    MTP_CUDA(h, launch_totals(natoms, h->d_E, h->d_wown, h->d_partials, h->d_tot, h->stream));
    if (flags & MTP_EFLAG)
      MTP_CUDA(h, cudaMemcpyAsync(d_energy, h->d_tot, sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    if (flags & MTP_VFLAG)
      MTP_CUDA(h, cudaMemcpyAsync(d_virial, h->d_tot + 1, 6 * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  }
  if ((flags & MTP_EATOM) && natoms > 0)
    MTP_CUDA(h, cudaMemcpyAsync(d_eatom, h->d_E, natoms * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  h->calls++;
  return MTP_OK;
}

int mtp_compute_positions_device(mtp_handle* h, int nlocal, int nall, const double* d_x, const int* d_species,
                                 const int* d_owner, int list_stride, const int* d_neigh, const int* d_numneigh,
                                 int flags, double* d_energy, double* d_forces, double* d_virial, double* d_eatom,
                                 double* d_vatom) {
  if (!h) return MTP_E_INVALID;
  if (nlocal < 0 || nall < nlocal || list_stride < 0)
    return fail(h, MTP_E_INVALID, "need 0 <= nlocal <= nall and list_stride >= 0");
  if (nlocal > h->max_atoms) return fail(h, MTP_E_CAPACITY, "nlocal exceeds max_atoms");
  if (nlocal > 0 && (list_stride == 0 || !d_x || !d_species || !d_owner || !d_neigh || !d_numneigh || !d_forces))
    return fail(h, MTP_E_INVALID, "null input or forces pointer, or list_stride 0 with atoms");
  if ((flags & MTP_EFLAG) && !d_energy) return fail(h, MTP_E_INVALID, "MTP_EFLAG without an energy pointer");
  if ((flags & MTP_VFLAG) && !d_virial) return fail(h, MTP_E_INVALID, "MTP_VFLAG without a virial pointer");
  if ((flags & MTP_EATOM) && !d_eatom) return fail(h, MTP_E_INVALID, "MTP_EATOM without an eatom pointer");
  if ((flags & MTP_VATOM) && !d_vatom) return fail(h, MTP_E_INVALID, "MTP_VATOM without a vatom pointer");
  const int stride = h->max_nbr;
  if (nlocal > 0)
    MTP_CUDA(h, launch_rows_from_positions(nlocal, nall, d_x, d_species, d_owner, list_stride, d_neigh, d_numneigh,
                                           h->cutoff, stride, h->d_rijs, h->d_js, h->d_jtypes, h->d_counts,
                                           h->d_err, h->stream));
  int st = run_device(h, nlocal, stride, nlocal > 0 ? d_species : h->d_itypes, h->d_rijs, h->d_js, h->d_jtypes,
                      h->d_counts, true, d_forces, (flags & MTP_VATOM) ? d_vatom : nullptr);
  if (st != MTP_OK) return st;
  if (flags & (MTP_EFLAG | MTP_VFLAG)) {
    MTP_CUDA(h, launch_totals(nlocal, h->d_E, h->d_wown, h->d_partials, h->d_tot, h->stream));
    if (flags & MTP_EFLAG)
      MTP_CUDA(h, cudaMemcpyAsync(d_energy, h->d_tot, sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    if (flags & MTP_VFLAG)
      MTP_CUDA(h, cudaMemcpyAsync(d_virial, h->d_tot + 1, 6 * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  }
  if ((flags & MTP_EATOM) && nlocal > 0)
    MTP_CUDA(h, cudaMemcpyAsync(d_eatom, h->d_E, nlocal * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  h->calls++;
  return MTP_OK;
}

int mtp_compute(mtp_handle* h, int natoms, int stride, const int* itypes, const double* rijs, const int* js,
                const int* jtypes, const int* counts, int flags, double* energy, double* forces, double* virial,
                double* eatom, double* vatom) {
  if (!h) return MTP_E_INVALID;
  if (natoms < 0 || stride <= 0) return fail(h, MTP_E_INVALID, "natoms must be >= 0 and nbr_stride > 0");
  if (natoms > h->max_atoms)
    return fail(h, MTP_E_CAPACITY, "natoms " + std::to_string(natoms) + " exceeds max_atoms " +
                                        std::to_string(h->max_atoms));
  if (stride > h->max_nbr) return fail(h, MTP_E_CAPACITY, "nbr_stride exceeds max_nbr");
  if (natoms > 0 && (!itypes || !rijs || !js || !jtypes || !forces))
    return fail(h, MTP_E_INVALID, "null input or forces pointer");
  if ((flags & MTP_EFLAG) && !energy) return fail(h, MTP_E_INVALID, "MTP_EFLAG without an energy pointer");
  if ((flags & MTP_VFLAG) && !virial) return fail(h, MTP_E_INVALID, "MTP_VFLAG without a virial pointer");
  if ((flags & MTP_EATOM) && !eatom) return fail(h, MTP_E_INVALID, "MTP_EATOM without an eatom pointer");
  if ((flags & MTP_VATOM) && !vatom) return fail(h, MTP_E_INVALID, "MTP_VATOM without a vatom pointer");
  if (counts) {
    for (int i = 0; i < natoms; ++i)
      if (counts[i] < 0 || counts[i] > stride)
        return fail(h, MTP_E_CAPACITY, "atom " + std::to_string(i) + " has " + std::to_string(counts[i]) +
                                            " neighbours, more than the row length " + std::to_string(stride));
  }
  auto t0 = std::chrono::steady_clock::now();
  const size_t N = natoms;
  cudaStream_t s = h->stream;
  int st;
  if (natoms >= kPipelineMinAtoms) {
    st = run_host_pipelined(h, natoms, stride, itypes, rijs, js, jtypes, counts,
                            (flags & MTP_VATOM) ? h->d_vatom : nullptr);
    if (st != MTP_OK) {
      cudaStreamSynchronize(s);   // copies from the caller's buffers complete before the error returns
      return st;
    }
    MTP_CUDA(h, launch_totals(natoms, h->d_E, h->d_wown, h->d_partials, h->d_tot, s));
    MTP_CUDA(h, cudaMemcpyAsync(forces, h->d_F, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (flags & MTP_EATOM) MTP_CUDA(h, cudaMemcpyAsync(eatom, h->d_E, N * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (flags & MTP_VATOM)
      MTP_CUDA(h, cudaMemcpyAsync(vatom, h->d_vatom, 6 * N * sizeof(double), cudaMemcpyDeviceToHost, s));
    MTP_CUDA(h, cudaMemcpyAsync(h->h_tot, h->d_tot, 7 * sizeof(double), cudaMemcpyDeviceToHost, s));
    st = read_err_flags(h);   // synchronises the stream
  } else {
    st = run_small_call(h, natoms, stride, itypes, rijs, js, jtypes, counts, flags, forces, eatom, vatom);
  }
  if (st != MTP_OK) return st;
  if (flags & MTP_EFLAG) *energy = h->h_tot[0];
  if (flags & MTP_VFLAG)
    for (int c = 0; c < 6; ++c) virial[c] = h->h_tot[1 + c];
  h->calls++;
  double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  h->total_ms += ms;
  if (h->debug >= 2) std::fprintf(stderr, "[mtp_b200] call %lld: natoms=%d %.3f ms\n", h->calls, natoms, ms);
  return MTP_OK;
}

int mtp_compute_positions(mtp_handle* h, int nlocal, int nall, const double* x, const int* species, const int* owner,
                          int list_stride, const int* neigh, const int* numneigh, int flags, double* energy,
                          double* forces, double* virial, double* eatom, double* vatom) {
  if (!h) return MTP_E_INVALID;
  if (nlocal < 0 || nall < nlocal || list_stride < 0)
    return fail(h, MTP_E_INVALID, "need 0 <= nlocal <= nall and list_stride >= 0");
  if (nlocal > h->max_atoms)
    return fail(h, MTP_E_CAPACITY, "nlocal " + std::to_string(nlocal) + " exceeds max_atoms " +
                                        std::to_string(h->max_atoms));
  if (nlocal > 0 && (list_stride == 0 || !x || !species || !owner || !neigh || !numneigh || !forces))
    return fail(h, MTP_E_INVALID, "null input or forces pointer, or list_stride 0 with atoms");
  if ((flags & MTP_EFLAG) && !energy) return fail(h, MTP_E_INVALID, "MTP_EFLAG without an energy pointer");
  if ((flags & MTP_VFLAG) && !virial) return fail(h, MTP_E_INVALID, "MTP_VFLAG without a virial pointer");
  if ((flags & MTP_EATOM) && !eatom) return fail(h, MTP_E_INVALID, "MTP_EATOM without an eatom pointer");
  if ((flags & MTP_VATOM) && !vatom) return fail(h, MTP_E_INVALID, "MTP_VATOM without a vatom pointer");
  auto t0 = std::chrono::steady_clock::now();
  const cudaStream_t s = h->stream;
  const size_t N = nlocal, NA = nall, NN = N * list_stride;
  if (NA > h->all_cap) {
    MTP_CUDA(h, cudaStreamSynchronize(s));
    cudaFree(h->d_xall);
    cudaFree(h->d_spall);
    cudaFree(h->d_owner);
    h->d_xall = nullptr;
    h->d_spall = h->d_owner = nullptr;
    h->all_cap = 0;
    ++h->gen;
    MTP_CUDA(h, dalloc(&h->d_xall, 3 * NA));
    MTP_CUDA(h, dalloc(&h->d_spall, NA));
    MTP_CUDA(h, dalloc(&h->d_owner, NA));
    h->all_cap = NA;
  }
  if (NN > h->neigh_cap) {
    MTP_CUDA(h, cudaStreamSynchronize(s));
    cudaFree(h->d_neigh);
    h->d_neigh = nullptr;
    h->neigh_cap = 0;
    ++h->gen;
    MTP_CUDA(h, dalloc(&h->d_neigh, NN));
    h->neigh_cap = NN;
  }
  if (!h->d_numneigh) MTP_CUDA(h, dalloc(&h->d_numneigh, static_cast<size_t>(h->max_atoms)));
  const int stride = h->max_nbr;
  // copies, rows, evaluation, totals and read-backs; nothing here
  // synchronises or allocates, so run_graphable may capture it
  auto enqueue = [&]() -> int {
    if (nlocal > 0) {
      MTP_CUDA(h, cudaMemcpyAsync(h->d_xall, x, 3 * NA * sizeof(double), cudaMemcpyHostToDevice, s));
      MTP_CUDA(h, cudaMemcpyAsync(h->d_spall, species, NA * sizeof(int), cudaMemcpyHostToDevice, s));
      MTP_CUDA(h, cudaMemcpyAsync(h->d_owner, owner, NA * sizeof(int), cudaMemcpyHostToDevice, s));
      MTP_CUDA(h, cudaMemcpyAsync(h->d_neigh, neigh, NN * sizeof(int), cudaMemcpyHostToDevice, s));
      MTP_CUDA(h, cudaMemcpyAsync(h->d_numneigh, numneigh, N * sizeof(int), cudaMemcpyHostToDevice, s));
      MTP_CUDA(h, launch_rows_from_positions(nlocal, nall, h->d_xall, h->d_spall, h->d_owner, list_stride,
                                             h->d_neigh, h->d_numneigh, h->cutoff, stride, h->d_rijs, h->d_js,
                                             h->d_jtypes, h->d_counts, h->d_err, s));
    }
    int st = run_device(h, nlocal, stride, nlocal > 0 ? h->d_spall : h->d_itypes, h->d_rijs, h->d_js, h->d_jtypes,
                        h->d_counts, true, h->d_F, (flags & MTP_VATOM) ? h->d_vatom : nullptr);
    if (st != MTP_OK) return st;
    MTP_CUDA(h, launch_totals(nlocal, h->d_E, h->d_wown, h->d_partials, h->d_tot, s));
    if (nlocal > 0) {
      MTP_CUDA(h, cudaMemcpyAsync(forces, h->d_F, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, s));
      if (flags & MTP_EATOM)
        MTP_CUDA(h, cudaMemcpyAsync(eatom, h->d_E, N * sizeof(double), cudaMemcpyDeviceToHost, s));
      if (flags & MTP_VATOM)
        MTP_CUDA(h, cudaMemcpyAsync(vatom, h->d_vatom, 6 * N * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    MTP_CUDA(h, cudaMemcpyAsync(h->h_tot, h->d_tot, 7 * sizeof(double), cudaMemcpyDeviceToHost, s));
    MTP_CUDA(h, cudaMemcpyAsync(h->h_err, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    return MTP_OK;
  };
  HostCallKey key;
  key.kind = 1;
  key.natoms = nlocal;
  key.stride = list_stride;
  key.extra = nall;
  key.flags = flags & (MTP_EATOM | MTP_VATOM);
  key.gen = h->gen;
  const void* ptrs[8] = {x, species, owner, neigh, numneigh, forces,
                         (flags & MTP_EATOM) ? eatom : nullptr, (flags & MTP_VATOM) ? vatom : nullptr};
  for (int k = 0; k < 8; ++k) key.p[k] = ptrs[k];
  const bool pinned = nlocal > 0 && !h->profiling && host_pinned(x, 3 * NA * sizeof(double)) &&
                      host_pinned(species, NA * sizeof(int)) && host_pinned(owner, NA * sizeof(int)) &&
                      host_pinned(neigh, NN * sizeof(int)) && host_pinned(numneigh, N * sizeof(int)) &&
                      host_pinned(forces, 3 * N * sizeof(double)) &&
                      host_pinned(key.p[6], (flags & MTP_EATOM) ? N * sizeof(double) : 0) &&
                      host_pinned(key.p[7], (flags & MTP_VATOM) ? 6 * N * sizeof(double) : 0);
  const int st = run_graphable(h, key, pinned, enqueue);
  if (st != MTP_OK) return st;
  if (flags & MTP_EFLAG) *energy = h->h_tot[0];
  if (flags & MTP_VFLAG)
    for (int c = 0; c < 6; ++c) virial[c] = h->h_tot[1 + c];
  h->calls++;
  h->total_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return MTP_OK;
}

int mtp_execute_potential(mtp_handle* h, int natoms, int nneigh_total, const double* const* atom_positions,
                          const int* atom_types, const int* const* neighbor_lists, const int* neighbor_counts,
                          const int* const* neighbor_types_lists, double volume, double* energy, double** forces,
                          double* stress) {
  (void)nneigh_total;
  if (!h) return MTP_E_INVALID;
  if (natoms < 0) return fail(h, MTP_E_INVALID, "natoms must be >= 0");
  if (natoms > h->max_atoms) return fail(h, MTP_E_CAPACITY, "natoms exceeds max_atoms");
  if (natoms > 0 && (!atom_positions || !atom_types || !neighbor_lists || !neighbor_counts || !neighbor_types_lists ||
                     !forces || !energy || !stress))
    return fail(h, MTP_E_INVALID, "null argument");
  const int stride = h->max_nbr;
  for (int i = 0; i < natoms; ++i) {
    const int c = neighbor_counts[i];
    if (c < 0 || c > stride)
      return fail(h, MTP_E_CAPACITY, "atom " + std::to_string(i) + " has " + std::to_string(c) +
                                          " neighbours, more than MAX_ATOMS_PER_NEIGHBOR");
  }
  // persistent page-locked staging (the reference bridge refilled persistent
  // NumPy buffers, zero_overhead.cpp:61-117): no allocation per step, and the
  // rows reach the GPU by DMA
  if (!h->hp_rij) {
    const size_t rows = static_cast<size_t>(h->max_atoms), slots = rows * stride;
    void *a = nullptr, *b = nullptr, *c = nullptr, *d = nullptr, *e = nullptr, *f = nullptr;
    const bool ok = cudaHostAlloc(&a, 3 * slots * sizeof(double), cudaHostAllocDefault) == cudaSuccess &&
                    cudaHostAlloc(&b, slots * sizeof(int), cudaHostAllocDefault) == cudaSuccess &&
                    cudaHostAlloc(&c, slots * sizeof(int), cudaHostAllocDefault) == cudaSuccess &&
                    cudaHostAlloc(&d, std::max<size_t>(rows, 1) * sizeof(int), cudaHostAllocDefault) == cudaSuccess &&
                    cudaHostAlloc(&e, std::max<size_t>(rows, 1) * sizeof(int), cudaHostAllocDefault) == cudaSuccess &&
                    cudaHostAlloc(&f, 3 * std::max<size_t>(rows, 1) * sizeof(double), cudaHostAllocDefault) ==
                        cudaSuccess;
    if (!ok) {
      for (void* q : {a, b, c, d, e, f})
        if (q) cudaFreeHost(q);
      cudaGetLastError();
      return fail(h, MTP_E_OOM, "mtp_execute_potential: page-locked staging allocation failed");
    }
    h->hp_rij = static_cast<double*>(a);
    h->hp_js = static_cast<int*>(b);
    h->hp_jt = static_cast<int*>(c);
    h->hp_cnt = static_cast<int*>(d);
    h->hp_types = static_cast<int*>(e);
    h->hp_F = static_cast<double*>(f);
  }
  // pack the counted slots of each row into the flat layout (what the
  // reference bridge copies into its NumPy buffers, zero_overhead.cpp:94-116);
  // slots past a row's count are never read
  for (int i = 0; i < natoms; ++i) {
    const int c = neighbor_counts[i];
    h->hp_cnt[i] = c;
    h->hp_types[i] = atom_types[i];
    if (c == 0) continue;
    std::memcpy(h->hp_rij + static_cast<size_t>(i) * stride * 3, atom_positions[i], 3 * c * sizeof(double));
    std::memcpy(h->hp_js + static_cast<size_t>(i) * stride, neighbor_lists[i], c * sizeof(int));
    std::memcpy(h->hp_jt + static_cast<size_t>(i) * stride, neighbor_types_lists[i], c * sizeof(int));
  }
  double vir[6] = {0, 0, 0, 0, 0, 0}, e = 0.0;
  int st = mtp_compute(h, natoms, stride, h->hp_types, h->hp_rij, h->hp_js, h->hp_jt, h->hp_cnt,
                       MTP_EFLAG | MTP_VFLAG, &e, h->hp_F, vir, nullptr, nullptr);
  if (st != MTP_OK) return st;
  *energy = e;
  for (int i = 0; i < natoms; ++i)
    for (int c = 0; c < 3; ++c) forces[i][c] = h->hp_F[3 * static_cast<size_t>(i) + c];
  // reference stress: +sym(sum r g)/V, order xx,yy,zz,yz,xz,xy (jax_backend.py:355-360)
  const double iv = 1.0 / volume;
  stress[0] = -vir[0] * iv;
  stress[1] = -vir[1] * iv;
  stress[2] = -vir[2] * iv;
  stress[3] = -vir[5] * iv;
  stress[4] = -vir[4] * iv;
  stress[5] = -vir[3] * iv;
  return MTP_OK;
}

int mtp_compute_batch_device(mtp_handle* h, int natoms, int stride, int nconfig, const int* d_itypes,
                             const double* d_rijs, const int* d_js, const int* d_jtypes, const int* d_counts,
                             const int* d_cfg, const double* d_volumes, double* d_energy, double* d_forces,
                             double* d_stress) {
  if (!h) return MTP_E_INVALID;
  if (natoms < 0 || stride <= 0 || nconfig < 0) return fail(h, MTP_E_INVALID, "bad sizes");
  if (natoms > h->max_atoms) return fail(h, MTP_E_CAPACITY, "natoms exceeds max_atoms");
  if (stride > h->max_nbr) return fail(h, MTP_E_CAPACITY, "nbr_stride exceeds max_nbr");
  if (natoms > 0 && (!d_itypes || !d_rijs || !d_js || !d_jtypes || !d_cfg || !d_volumes || !d_energy ||
                     !d_forces || !d_stress))
    return fail(h, MTP_E_INVALID, "null pointer");
  if (nconfig + 1 > h->cfg_cap) {
    if (h->d_cfg_ptr) cudaFree(h->d_cfg_ptr);
    h->d_cfg_ptr = nullptr;
    MTP_CUDA(h, dalloc(&h->d_cfg_ptr, nconfig + 1));
    h->cfg_cap = nconfig + 1;
  }
  MTP_CUDA(h, launch_config_ptr(natoms, nconfig, d_cfg, h->d_cfg_ptr, h->d_err, h->stream));
  int st = run_device(h, natoms, stride, d_itypes, d_rijs, d_js, d_jtypes, d_counts, true, d_forces, nullptr);
  if (st != MTP_OK) return st;
  MTP_CUDA(h, launch_config_totals(natoms, nconfig, h->d_cfg_ptr, h->d_E, h->d_wown, d_volumes, d_energy, d_stress,
                                   h->stream));
  h->calls++;
  return MTP_OK;
}

int mtp_adjoint_batch_device(mtp_handle* h, int natoms, int stride, int nconfig, const int* d_itypes,
                             const double* d_rijs, const int* d_js, const int* d_jtypes, const int* d_counts,
                             const int* d_cfg, const double* d_volumes, const double* d_gE, const double* d_gF,
                             const double* d_gS, double* d_gspecies, double* d_gmoment, double* d_gradial) {
  if (!h) return MTP_E_INVALID;
  if (natoms < 0 || stride <= 0 || nconfig < 0) return fail(h, MTP_E_INVALID, "bad sizes");
  if (natoms > h->max_atoms) return fail(h, MTP_E_CAPACITY, "natoms exceeds max_atoms");
  if (stride > h->max_nbr) return fail(h, MTP_E_CAPACITY, "nbr_stride exceeds max_nbr");
  if (!d_gspecies || !d_gmoment || !d_gradial) return fail(h, MTP_E_INVALID, "null gradient pointer");
  if (natoms > 0 && (!d_itypes || !d_rijs || !d_js || !d_jtypes || !d_cfg || !d_volumes || !d_gE || !d_gF || !d_gS))
    return fail(h, MTP_E_INVALID, "null pointer");
  // with the value space in global memory, 512 lanes give the SM twice the
  // warps for the same L2 footprint
  int lanes = h->threads;
  DeviceSchedule* ds = nullptr;
  int st = get_schedule(h, lanes, access_width(true, 1), &ds, false);
  if (st != MTP_OK) return st;
  if (lanes < 512 && !adjoint_fits_shared(make_model(h, *ds), stride, lanes)) lanes = 512;
  st = get_schedule(h, lanes, access_width(true, 1), &ds);
  if (st != MTP_OK) return st;
  DevModel md = make_model(h, *ds);
  TrainIO tio{};
  tio.natoms = natoms;
  tio.nbr_stride = stride;
  tio.nconfig = nconfig;
  tio.itypes = d_itypes;
  tio.rijs = d_rijs;
  tio.js = d_js;
  tio.jtypes = d_jtypes;
  tio.counts = d_counts;
  tio.cfg = d_cfg;
  tio.volumes = d_volumes;
  tio.gE = d_gE;
  tio.gF = d_gF;
  tio.gS = d_gS;
  tio.err = h->d_err;
  std::string err;
  cudaError_t ce = launch_adjoint(md, tio, lanes, h->sm_count, h->train, d_gspecies, d_gmoment, d_gradial,
                                  h->stream, err);
  if (!err.empty()) return fail(h, MTP_E_CAPACITY, err);
  if (ce != cudaSuccess) return cuda_fail(h, ce, "adjoint");
  h->calls++;
  return MTP_OK;
}

namespace {
int ensure_cells(mtp_handle* h, int n, int ncell) {
  CellScratch& c = h->cells;
  if (n > c.n_cap) {
    if (c.cell) cudaFree(c.cell);
    if (c.img) cudaFree(c.img);
    if (c.atoms) cudaFree(c.atoms);
    c.cell = c.img = c.atoms = nullptr;
    c.n_cap = 0;
    MTP_CUDA(h, dalloc(&c.cell, n));
    MTP_CUDA(h, dalloc(&c.img, 3 * static_cast<size_t>(n)));
    MTP_CUDA(h, dalloc(&c.atoms, n));
    c.n_cap = n;
  }
  if (ncell > c.cell_cap) {
    if (c.cnt) cudaFree(c.cnt);
    if (c.ptr) cudaFree(c.ptr);
    if (c.cursor) cudaFree(c.cursor);
    if (c.blk) cudaFree(c.blk);
    c.cnt = c.ptr = c.cursor = c.blk = nullptr;
    c.cell_cap = 0;
    MTP_CUDA(h, dalloc(&c.cnt, ncell));
    MTP_CUDA(h, dalloc(&c.ptr, ncell + 1));
    MTP_CUDA(h, dalloc(&c.cursor, ncell));
    MTP_CUDA(h, dalloc(&c.blk, ncell / 1024 + 2));
    c.cell_cap = ncell;
  }
  return MTP_OK;
}
}  // namespace

int mtp_neighbors_device(mtp_handle* h, int natoms, const double* d_pos, const double* cell9, const int* d_types,
                         double cutoff, int stride, int* d_js, int* d_image, int* d_jtypes, int* d_counts) {
  if (!h) return MTP_E_INVALID;
  if (natoms < 0 || stride <= 0 || !(cutoff > 0.0) || !cell9) return fail(h, MTP_E_INVALID, "bad arguments");
  if (natoms > 0 && (!d_pos || !d_types || !d_js || !d_image || !d_jtypes || !d_counts))
    return fail(h, MTP_E_INVALID, "null pointer");
  Box b;
  if (!make_box(cell9, cutoff, b)) return fail(h, MTP_E_INVALID, "singular cell");
  if (b.nc[0] < 1 || b.nc[1] < 1 || b.nc[2] < 1)
    return fail(h, MTP_E_INVALID, "cell thinner than the cutoff: build these rows on the host");
  const long long ncell = static_cast<long long>(b.nc[0]) * b.nc[1] * b.nc[2];
  if (ncell > (1LL << 28)) return fail(h, MTP_E_CAPACITY, "too many cells");
  int st = ensure_cells(h, natoms, static_cast<int>(ncell));
  if (st != MTP_OK) return st;
  MTP_CUDA(h, launch_neighbors(natoms, d_pos, b, d_types, cutoff, stride, d_js, d_image, d_jtypes, d_counts,
                               h->cells, h->d_err, h->stream));
  return MTP_OK;
}

int mtp_pack_rij_device(mtp_handle* h, int natoms, int stride, const double* d_pos, const double* cell9,
                        const int* d_js, const int* d_image, const int* d_counts, double* d_rijs) {
  if (!h) return MTP_E_INVALID;
  if (natoms < 0 || stride <= 0 || !cell9) return fail(h, MTP_E_INVALID, "bad arguments");
  if (natoms > 0 && (!d_pos || !d_js || !d_image || !d_counts || !d_rijs)) return fail(h, MTP_E_INVALID, "null pointer");
  Box b;
  if (!make_box(cell9, 1.0, b)) return fail(h, MTP_E_INVALID, "singular cell");
  MTP_CUDA(h, launch_pack_rij(natoms, stride, d_pos, b, d_js, d_image, d_counts, d_rijs, h->stream));
  return MTP_OK;
}

int mtp_verlet_device(mtp_handle* h, int natoms, double* d_x, double* d_v, const double* d_f, const int* d_types,
                      const double* masses, int nmasses, double dt, int stage) {
  if (!h) return MTP_E_INVALID;
  if (natoms < 0 || !masses || nmasses <= 0 || nmasses > kMaxMdSpecies || (stage != 1 && stage != 2))
    return fail(h, MTP_E_INVALID, "bad arguments");
  VerletParams p{};
  p.dt = dt;
  p.ftm2v = 1.0 / 1.0364269e-4;   // LAMMPS 'metal' force->ftm2v
  for (int t = 0; t < kMaxMdSpecies; ++t) p.inv_mass[t] = 1.0 / masses[std::min(t, nmasses - 1)];
  MTP_CUDA(h, launch_verlet(natoms, d_x, d_v, d_f, d_types, p, stage, h->stream));
  return MTP_OK;
}

int mtp_profile(mtp_handle* h, int enable) {
  if (!h) return MTP_E_INVALID;
  h->profiling = enable != 0;
  h->prof_used = 0;
  return MTP_OK;
}

int mtp_profile_read(mtp_handle* h, double* ms, int* launches) {
  if (!h || !ms || !launches) return MTP_E_INVALID;
  MTP_CUDA(h, cudaStreamSynchronize(h->stream));
  double tot = 0.0;
  for (int i = 0; i < h->prof_used; ++i) {
    float x = 0.f;
    MTP_CUDA(h, cudaEventElapsedTime(&x, h->prof_events[i].first, h->prof_events[i].second));
    tot += x;
  }
  *ms = tot;
  *launches = h->prof_used;
  return MTP_OK;
}

int mtp_measure_fma_peak(double* fp64, double* fp32) {
  if (!fp64 || !fp32) return MTP_E_INVALID;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return MTP_E_NODEVICE;
  }
  return measure_fma_peak(fp64, fp32) == cudaSuccess ? MTP_OK : MTP_E_CUDA;
}

int mtp_host_alloc(size_t bytes, void** out) {
  if (!out) return fail(nullptr, MTP_E_INVALID, "mtp_host_alloc: null output pointer");
  *out = nullptr;
  if (bytes == 0) return MTP_OK;
  const cudaError_t e = cudaHostAlloc(out, bytes, cudaHostAllocDefault);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *out = nullptr;
    return fail(nullptr, e == cudaErrorMemoryAllocation ? MTP_E_OOM : MTP_E_CUDA,
                std::string("mtp_host_alloc: ") + cudaGetErrorString(e));
  }
  return MTP_OK;
}

int mtp_host_free(void* p) {
  if (!p) return MTP_OK;
  const cudaError_t e = cudaFreeHost(p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(nullptr, MTP_E_CUDA, std::string("mtp_host_free: ") + cudaGetErrorString(e));
  }
  return MTP_OK;
}

}  // extern "C"

// ===========================================================================
// Allocation-free evaluation (mtp_compute_device_noalloc)
// ===========================================================================
// Some callers cannot let a library call cudaMalloc: code that runs while a
// CUDA stream is being captured into a graph (allocation is illegal there),
// code that must not synchronise the device (cudaMalloc/cudaFree may), and
// hosts whose memory pool owns the whole device.  This variant of
// mtp_compute_device keeps every piece of its scratch memory in one
// file-scope device array of fixed size instead of handle buffers, and uses
// only the contraction schedules the handle already uploaded.
namespace {

constexpr size_t al256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

struct NoAllocLayout {
  size_t grad, energy, wown, in_cnt, in_ptr, in_cursor, in_slot, blk, partials, tot, total;
};

constexpr NoAllocLayout noalloc_layout() {
  NoAllocLayout L{};
  const size_t atoms = MTP_NOALLOC_MAX_ATOMS, slots = MTP_NOALLOC_MAX_SLOTS;
  size_t o = 0;
  L.grad = o;      o = al256(o + slots * 3 * sizeof(double));
  L.energy = o;    o = al256(o + atoms * sizeof(double));
  L.wown = o;      o = al256(o + atoms * 6 * sizeof(double));
  L.in_cnt = o;    o = al256(o + atoms * sizeof(int));
  L.in_ptr = o;    o = al256(o + (atoms + 1) * sizeof(int));
  L.in_cursor = o; o = al256(o + atoms * sizeof(int));
  L.in_slot = o;   o = al256(o + slots * sizeof(int));
  L.blk = o;       o = al256(o + (atoms / 1024 + 2) * sizeof(int));
  L.partials = o;  o = al256(o + 7 * kReduceBlocks * sizeof(double));
  L.tot = o;       o = al256(o + 8 * sizeof(double));
  L.total = o;
  return L;
}

constexpr NoAllocLayout kNoAlloc = noalloc_layout();

// The scratch (about 8.5 MB).  Every GPU that loads this library holds it
// until the process exits; all calls on a device share it.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAlloc.total];

// Device address of g_noalloc_scratch on the current device.  In host code
// the symbol is only a host-side stand-in, so the address is asked for once
// per device (with that device current) and cached for the life of the
// process; a reset of the device's primary context (cudaDeviceReset) makes the
// cached address stale, which the header states as a limit of this path.
int noalloc_base(mtp_handle* h, unsigned char** out) {
  static std::mutex mu;
  static unsigned char* base[64] = {};
  int dev = -1;
  MTP_CUDA(h, cudaGetDevice(&dev));
  if (dev != h->device) return fail(h, MTP_E_INVALID, "the current CUDA device is not the handle's device");
  if (dev < 0 || dev >= 64) return fail(h, MTP_E_INVALID, "device ordinal above 63");
  std::lock_guard<std::mutex> lock(mu);
  if (!base[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return cuda_fail(h, e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    base[dev] = static_cast<unsigned char*>(p);
  }
  *out = base[dev];
  return MTP_OK;
}

}  // namespace

extern "C" {

int mtp_compute_device_noalloc(mtp_handle* h, int natoms, int stride, const int* d_itypes, const double* d_rijs,
                               const int* d_js, const int* d_jtypes, const int* d_counts, double* d_energy,
                               double* d_forces, double* d_virial) {
  if (!h) return MTP_E_INVALID;
  if (natoms < 0 || stride <= 0) return fail(h, MTP_E_INVALID, "natoms must be >= 0 and nbr_stride > 0");
  if (natoms > MTP_NOALLOC_MAX_ATOMS)
    return fail(h, MTP_E_CAPACITY, "natoms " + std::to_string(natoms) + " exceeds the allocation-free limit of " +
                                        std::to_string(MTP_NOALLOC_MAX_ATOMS) + " atoms");
  if (static_cast<long long>(natoms) * stride > MTP_NOALLOC_MAX_SLOTS)
    return fail(h, MTP_E_CAPACITY, "natoms * nbr_stride exceeds the allocation-free limit of " +
                                        std::to_string(MTP_NOALLOC_MAX_SLOTS) + " neighbour slots");
  if (stride > h->max_nbr) return fail(h, MTP_E_CAPACITY, "nbr_stride exceeds max_nbr");
  if (natoms > 0 && (!d_itypes || !d_rijs || !d_js || !d_jtypes || !d_forces || !d_energy || !d_virial))
    return fail(h, MTP_E_INVALID, "null pointer");
  unsigned char* base = nullptr;
  int st = noalloc_base(h, &base);
  if (st != MTP_OK) return st;
  const bool fp64 = h->precision == MTP_PRECISION_FP64;

  // launch shape from the schedules already on the device, each paired only
  // with the atoms per block whose operand width its entry order was tuned
  // for, within the handle's launch limits (mtp_set_launch); the value space
  // must fit in shared memory (its global-memory form would need an allocation)
  const DeviceSchedule* ds = nullptr;
  int lanes = 0, A = 1, bps = 0, best = -1;
  for (const auto& kv : h->scheds) {
    const DevModel md = make_model(h, kv.second);
    const int sl = kv.second.sched.lanes;
    if (sl > h->threads) continue;
    for (int a : {4, 2, 1}) {
      if (!eval_variant_exists(fp64, false, a)) continue;
      if (h->apb > 0 && a != h->apb) continue;
      if (kv.second.sched.width != access_width(fp64, a)) continue;
      int b = eval_blocks_per_sm(md, stride, sl, fp64, false, a);
      if (h->blocks_per_sm > 0) b = std::min(b, h->blocks_per_sm);
      if (b <= 0) continue;
      const int score = (a * b) * 1024 + b * sl / 32;
      if (score > best) {
        best = score;
        ds = &kv.second;
        lanes = sl;
        A = a;
        bps = b;
      }
    }
  }
  if (!ds)
    return fail(h, MTP_E_CAPACITY,
                "no uploaded schedule gives a shared-memory launch within the handle's launch limits (either the "
                "value space of this basis does not fit in shared memory, which the allocation-free path cannot "
                "replace by global memory, or no allocating call has uploaded a schedule for these limits yet)");

  double* grad = reinterpret_cast<double*>(base + kNoAlloc.grad);
  double* energy = reinterpret_cast<double*>(base + kNoAlloc.energy);
  double* wown = reinterpret_cast<double*>(base + kNoAlloc.wown);
  int* in_cnt = reinterpret_cast<int*>(base + kNoAlloc.in_cnt);
  int* in_ptr = reinterpret_cast<int*>(base + kNoAlloc.in_ptr);
  int* in_cursor = reinterpret_cast<int*>(base + kNoAlloc.in_cursor);
  int* in_slot = reinterpret_cast<int*>(base + kNoAlloc.in_slot);
  int* blk = reinterpret_cast<int*>(base + kNoAlloc.blk);
  double* partials = reinterpret_cast<double*>(base + kNoAlloc.partials);
  double* tot = reinterpret_cast<double*>(base + kNoAlloc.tot);

  // The array keeps the previous call's contents.  The incoming-slot counters
  // must start at zero (launch_incoming clears in_cnt and in_cursor first);
  // every other piece is fully rewritten before it is read: each slot's
  // gradient (zero for skipped slots), each site energy and per-atom virial,
  // the scan blocks, the partials and the totals.
  DevModel md = make_model(h, *ds);
  DevIO io{};
  io.natoms = natoms;
  io.nbr_stride = stride;
  io.n_pad = stride;
  io.itypes = d_itypes;
  io.rijs = d_rijs;
  io.jtypes = d_jtypes;
  io.counts = d_counts;
  io.site_energy = energy;
  io.pair_grad = grad;
  io.err = h->d_err;
  io.vscratch = nullptr;
  const long long groups = (static_cast<long long>(natoms) + A - 1) / A;
  const int blocks = static_cast<int>(std::max(1LL, std::min<long long>(static_cast<long long>(bps) * h->sm_count,
                                                                         groups)));
  MTP_CUDA(h, launch_incoming(natoms, stride, d_js, d_jtypes, d_counts, in_cnt, in_ptr, in_cursor, in_slot, blk,
                              h->stream));
  MTP_CUDA(h, launch_eval(md, io, lanes, blocks, fp64, false, A, h->stream));
  MTP_CUDA(h, launch_force_gather(natoms, stride, d_rijs, d_counts, grad, in_ptr, in_slot, d_forces, wown, nullptr,
                                  h->stream));
  MTP_CUDA(h, launch_totals(natoms, energy, wown, partials, tot, h->stream));
  MTP_CUDA(h, cudaMemcpyAsync(d_energy, tot, sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  MTP_CUDA(h, cudaMemcpyAsync(d_virial, tot + 1, 6 * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  h->calls++;
  return MTP_OK;
}

}  // extern "C"
