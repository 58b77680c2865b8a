/* ----------------------------------------------------------------------
   pair_style jax/mtp on the B200 MTP engine (C ABI include/mtp_b200.h)

   Keeps the reference pair style's surface (pair_style_files/pair_jax_mtp.h,
   pair_jax_mtp.cpp:228-282):

     pair_style jax/mtp <potential.mtp> MAX_ATOMS MAX_ATOMS_PER_NEIGHBOR MTP_CUTOFF [DEBUG_LEVEL] [fp64|mixed]
                        [rows device|host]
     pair_coeff * *

   The first argument is the .mtp potential itself (the reference took a
   jax.export .bin compiled from it; a .bin is rejected with a clear error).
   Needs atom IDs, a full neighbour list, and one MPI rank (as the reference).
   rows device (the default) sends positions and the neighbour list and lets
   the GPU build the rows (mtp_compute_positions); rows host packs r_ij on
   the host as the reference did (mtp_compute).  Both give the same results.
------------------------------------------------------------------------- */

#ifdef PAIR_CLASS
// clang-format off
PairStyle(jax/mtp,PairMTPB200);
// clang-format on
#else

#ifndef LMP_PAIR_MTP_B200_H
#define LMP_PAIR_MTP_B200_H

#include <cstddef>
#include <vector>

#include "mtp_b200.h"
#include "pair.h"

namespace LAMMPS_NS {

// Page-locked host array from mtp_host_alloc: the rows the pair style packs
// here reach the GPU by DMA, without the driver's staging copy of pageable
// memory.  Reallocates only when the size changes.
template <typename T> class PinnedArray {
 public:
  PinnedArray() = default;
  ~PinnedArray() { mtp_host_free(p_); }
  PinnedArray(const PinnedArray &) = delete;
  PinnedArray &operator=(const PinnedArray &) = delete;
  // n elements, each set to v; false if the allocation failed
  bool assign(size_t n, T v)
  {
    if (n != n_) {
      mtp_host_free(p_);
      p_ = nullptr;
      n_ = 0;
      void *q = nullptr;
      if (mtp_host_alloc(n * sizeof(T), &q) != MTP_OK) return false;
      p_ = static_cast<T *>(q);
      n_ = n;
    }
    for (size_t i = 0; i < n_; ++i) p_[i] = v;
    return true;
  }
  // at least n elements (contents kept only when nothing is reallocated)
  bool ensure(size_t n)
  {
    if (n <= n_) return true;
    mtp_host_free(p_);
    p_ = nullptr;
    n_ = 0;
    void *q = nullptr;
    if (mtp_host_alloc(n * sizeof(T), &q) != MTP_OK) return false;
    p_ = static_cast<T *>(q);
    n_ = n;
    return true;
  }
  size_t size() const { return n_; }
  T *data() { return p_; }
  T &operator[](size_t i) { return p_[i]; }

 private:
  T *p_ = nullptr;
  size_t n_ = 0;
};

class PairMTPB200 : public Pair {
 public:
  PairMTPB200(class LAMMPS *);
  ~PairMTPB200() override;

  void compute(int, int) override;
  void settings(int, char **) override;
  void coeff(int, char **) override;
  double init_one(int, int) override;
  void init_style() override;

  // statistics, for a driver's summary
  long long calls() const { return total_calls; }

 protected:
  void allocate();
  void grow_buffers();

  char *mtp_path;
  double cutoff;
  int max_atoms, max_nbr, debug_level, precision;
  int rows_on_device;
  mtp_handle *handle;
  long long total_calls;

  // persistent flat buffers [max_atoms][max_nbr] in page-locked memory (no
  // per-step allocation)
  PinnedArray<double> rij;
  PinnedArray<int> js, jtypes, counts, itypes;
  PinnedArray<double> fbuf, ebuf, vbuf;
  std::vector<int> tag_to_local;
  // rows device: positions, species and owners of local + ghost atoms, and
  // the neighbour list [nlocal][list stride], page-locked
  PinnedArray<double> xall;
  PinnedArray<int> spall, owner, neigh, nneigh;
};

}    // namespace LAMMPS_NS

#endif
#endif
