// mtp_model.hpp - host-side potential tables and the contraction schedule.
//
// The potential is the MLIP .mtp file the reference reads with read_mtp
// (motep_original_files/mtp.py:31-70).  The schedule turns its
// alpha_index_times list (m[i3] += mult * m[i1] * m[i2], conversion.py:95-102)
// into lane programs a CUDA block executes without atomics:
//
//   * forward: one pass per tree depth; each lane owns whole target moments
//     and accumulates their products in a register;
//   * reverse (dE/dm): the adjoint of every product is gathered per source
//     moment (dm[s] += mult * dm[t] * m[other]); long source lists are split
//     into chunks that write partial slots, summed in a fixed order by a
//     following combine pass.
//
// Every pass is a dense [steps][lanes] array of 8-byte entries so a warp
// reads its entries with one coalesced 256-byte load per step:
//
//   x = a | b << 16                     operand slots of the product
//   y = mult | op << 14 | dst << 16     integer multiplicity (< 2^14), flush
//                                       op (none/store/add), flush slot
//
// Steps are padded to a multiple of kStepAlign with no-op entries (operands
// the constant-zero slot, y = 0), and kStepAlign no-op rows follow the last
// pass, so a lane may request the kStepAlign rows after any step without a
// bounds test.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace mtp {

constexpr int kMaxR = 8;       // radial functions supported by the kernels
constexpr int kMaxK = 16;      // Chebyshev terms supported by the kernels
constexpr int kMaxDegree = 12; // monomial degree supported by the kernels
constexpr int kMaxPasses = 16;
constexpr int kStepAlign = 4;
constexpr int kN3GroupWarps = 8;  // warps that share one neighbour chunk in the FP32 force phase (half in FP64)   // pass steps are a multiple of this; as many no-op rows end the program

struct Potential {
  std::string version, potential_name, potential_tag, radial_basis_type;
  double scaling = 1.0, min_dist = 0.0, max_dist = 0.0;
  int S = 0, R = 0, K = 0, M = 0, B = 0, T = 0, Sa = 0;
  std::vector<double> radial;   // [S][S][R][K]
  std::vector<int> basic;       // [B][4] (mu, a, b, c)
  std::vector<int> times;       // [T][4] (i1, i2, mult, i3)
  std::vector<int> mapping;     // [Sa]
  std::vector<double> species;  // [S]
  std::vector<double> moment;   // [Sa]
};

// Parse .mtp text; returns false and sets err on malformed input.
bool parse_mtp_text(const std::string& text, Potential& out, std::string& err);
bool parse_mtp_file(const std::string& path, Potential& out, std::string& err);

// Program entry ops.
enum : uint32_t { kOpNone = 0, kOpStore = 1, kOpAdd = 2 };
// Fields of the second entry word.
constexpr uint32_t kMultMask = 0x3FFFu;
constexpr int kOpShift = 14;
constexpr int kDstShift = 16;

struct Pass {
  int offset = 0;   // first entry (index into Schedule::entries)
  int steps = 0;    // entries per lane (a multiple of kStepAlign)
  // steps each warp of the block runs: its longest lane's program rounded up
  // to kStepAlign (the rows after that are no-ops for all of its lanes)
  std::vector<int> wsteps;
};

struct Schedule {
  int lanes = 0;          // threads per block the programs were built for
  int width = 4;          // bytes per operand access the entry order was tuned for
  // Value-space layout (indices into the per-atom value array V):
  int v_m = 0;            // moments m[0..M)
  int v_dm = 0;           // adjoints dE/dm[0..M)
  int v_part = 0;         // partial sums of split lists
  int n_part = 0;
  int v_zero = 0;         // constant 0
  int v_one = 0;          // constant 1
  int v_size = 0;
  // monomials of the basic moments
  int D = 0;              // max degree
  int P = 0;              // distinct monomials
  std::vector<int> mono_abc;    // [P][4] (a, b, c, degree), degree descending
  std::vector<int> nmu;         // [D + 1] radial functions with a basic moment of each degree
  std::vector<int> mono_k;      // [P][kMaxR] basic-moment index for each mu or -1
  // The full monomial simplex a + b + c <= D in "pair order": pairs (a, b)
  // by s = a + b ascending, then a ascending; each pair owns the run of
  // slots c = 0 .. D - s.  Used by the force phase (nested Horner in z, y).
  int Q = 0;                    // (D+1)(D+2)(D+3)/6 slots
  int npairs = 0;               // (D+1)(D+2)/2 pairs
  std::vector<int> dense_k;     // [Q][kMaxR] basic-moment index of slot and mu, or -1
  // Level-structured basis (adjoint_layout): radial function mu meets exactly
  // the monomials of degree <= D - 2 mu.  Then a force-phase Horner step
  // k = D - degree has the radial functions mu <= k / 2, and the adjoints of
  // the basic moments are laid out in that chain order (dm_pos), so the force
  // phase reads them in place.
  bool tri = false;
  // dE/dm of moment k lives at v_dm + dm_pos[k] (a permutation of [0, M))
  std::vector<int> dm_pos;
  // Force phase on level-structured bases: the block's warps form groups of
  // min(lanes / 32, kN3GroupWarps) (FP32 kernel; n3_*_half: of half that,
  // FP64 kernel) that take neighbour chunks in turn, and warp w of a group
  // takes the monomial pairs n3_pairs[n3_off[w] .. n3_off[w + 1]) (at most
  // 32, balanced by chain cost), each one word a | b << 4 | top << 8 |
  // chain base << 12 (top = D - a - b; chain base = the pair's first
  // adjoint position).
  std::vector<int> n3_pairs, n3_off, n3_pairs_half, n3_off_half;
  std::vector<int> zero_list;   // non-basic moments never written (must read as 0)
  std::vector<Pass> fwd, rev;   // passes in execution order
  std::vector<uint32_t> entries;  // pairs (x, y) per entry: 2 words; kStepAlign no-op rows at the end
  int max_depth = 0;
};

// Build the schedule for `lanes` threads per block whose operand accesses are
// `width` bytes (sizeof(real) x atoms per block; it sets the bank model the
// entry order is tuned for).  Fails (false, err) if the table does not have a
// write-before-read order, or exceeds index limits.
bool build_schedule(const Potential& pot, int lanes, Schedule& out, std::string& err, int width = 4);

// Local search over a built schedule against shared-memory bank conflicts:
// an entry whose bank key sets a gather's wavefront count trades steps with
// another entry of the same job (the flush stays at the job's last step), or
// in a forward pass its two operands trade places, whenever that lowers the
// wavefronts of both steps (bank model of build_schedule's `width`).  The
// sums are unchanged up to their order; candidates come from a fixed-seed
// generator, so the result is a pure function of the schedule.
void refine_schedule(Schedule& s);

// Execute the schedule for one atom on the host (bit-for-bit the device
// arithmetic order, in double): V must have v_size entries with basic moments
// in V[v_m .. v_m + B) set.  Fills moments, adjoints (seeded with moment
// coefficients), and returns sum_alpha theta_alpha m[map_alpha].
double emulate_schedule(const Potential& pot, const Schedule& s, std::vector<double>& V);

// Position of every moment's adjoint within the adjoint region (dm_pos, a
// permutation of [0, M)); returns whether the basis is level-structured:
// every basic moment (mu, a, b, c) has 2 mu <= D - (a + b + c) and every such
// (mu, monomial) is a basic moment.  Then the basic moments' adjoints take
// positions [0, B) in force-phase chain order: monomial pairs (a, b) by
// a + b, then a; within a pair k = D - a - b - c = 0 .. D - a - b, and within
// a step mu = 0 .. k / 2, so step k of a pair starts floor((k + 1)^2 / 4)
// after the pair's first position and a pair of s = a + b holds
// floor((D - s + 2)^2 / 4).  Otherwise (and for every non-basic moment)
// dm_pos[k] = k.
bool adjoint_layout(const Potential& pot, std::vector<int>& dm_pos);

// Seeds of the reverse pass: unique moments of the mapping with summed theta.
void seed_list(const Potential& pot, std::vector<int>& idx, std::vector<double>& val);

}  // namespace mtp
