// lammps_shim.h - the few LAMMPS classes pair_mtp_b200.cpp uses, for building
// and running the pair style without a LAMMPS tree (mini_lammps.cpp drives it).
// Names and signatures follow the LAMMPS API; behaviour is the minimum needed.
#pragma once

#include <cstdint>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#define FLERR __FILE__, __LINE__
#define NEIGHMASK 0x1FFFFFFF

namespace LAMMPS_NS {

typedef int tagint;
class LAMMPS;
class Pair;

namespace NeighConst {
enum { REQ_DEFAULT = 0, REQ_FULL = 1 };
}

class Error {
 public:
  [[noreturn]] void all(const std::string &file, int line, const std::string &msg) {
    throw std::runtime_error(msg + " (" + file + ":" + std::to_string(line) + ")");
  }
  [[noreturn]] void one(const std::string &file, int line, const std::string &msg) { all(file, line, msg); }
};

class Memory {
 public:
  template <typename T>
  T **create(T **&a, int n1, int n2, const char *) {
    T *data = static_cast<T *>(std::calloc(static_cast<size_t>(n1) * n2 + 1, sizeof(T)));
    a = static_cast<T **>(std::malloc(sizeof(T *) * (n1 > 0 ? n1 : 1)));
    for (int i = 0; i < n1; ++i) a[i] = data + static_cast<size_t>(i) * n2;
    return a;
  }
  template <typename T>
  void destroy(T **&a) {
    if (a) {
      std::free(a[0]);
      std::free(a);
    }
    a = nullptr;
  }
};

class Atom {
 public:
  int nlocal = 0, nghost = 0, ntypes = 0, tag_enable = 1;
  double **x = nullptr, **f = nullptr;
  int *type = nullptr;
  tagint *tag = nullptr;
};

class NeighList {
 public:
  int inum = 0;
  int *ilist = nullptr, *numneigh = nullptr;
  int **firstneigh = nullptr;
};

class Neighbor {
 public:
  int requested_full = 0;
  void add_request(Pair *, int flags) { requested_full = (flags & NeighConst::REQ_FULL) ? 1 : 0; }
};

class Comm {
 public:
  int me = 0, nprocs = 1;
};

class Force {
 public:
  int newton_pair = 1;
};

class LAMMPS {
 public:
  Atom *atom = nullptr;
  Neighbor *neighbor = nullptr;
  Error *error = nullptr;
  Memory *memory = nullptr;
  Comm *comm = nullptr;
  Force *force = nullptr;
};

class Pointers {
 public:
  explicit Pointers(LAMMPS *ptr)
      : lmp(ptr), atom(ptr->atom), neighbor(ptr->neighbor), error(ptr->error), memory(ptr->memory),
        comm(ptr->comm), force(ptr->force) {}
  virtual ~Pointers() = default;

 protected:
  LAMMPS *lmp;
  Atom *&atom;
  Neighbor *&neighbor;
  Error *&error;
  Memory *&memory;
  Comm *&comm;
  Force *&force;
};

namespace utils {
inline int inumeric(const char *, int, const char *s, bool, LAMMPS *) { return std::atoi(s); }
inline double numeric(const char *, int, const char *s, bool, LAMMPS *) { return std::atof(s); }
}  // namespace utils

class Pair : public Pointers {
 public:
  explicit Pair(LAMMPS *l) : Pointers(l) {}
  ~Pair() override {
    memory->destroy(vatom);
    std::free(eatom);
  }
  virtual void compute(int, int) = 0;
  virtual void settings(int, char **) = 0;
  virtual void coeff(int, char **) = 0;
  virtual double init_one(int, int) = 0;
  virtual void init_style() = 0;

  // energy/virial accumulators as in LAMMPS Pair::ev_init
  void ev_init(int eflag, int vflag) {
    eflag_global = eflag & 1;
    eflag_atom = (eflag & 2) ? 1 : 0;
    vflag_global = (vflag & 3) ? 1 : 0;
    vflag_atom = (vflag & 4) ? 1 : 0;
    eng_vdwl = 0.0;
    for (double &v : virial) v = 0.0;
    const int n = atom->nlocal;
    if (eflag_atom) {
      if (n > maxeatom) {
        std::free(eatom);
        eatom = static_cast<double *>(std::calloc(n, sizeof(double)));
        maxeatom = n;
      }
      for (int i = 0; i < n; ++i) eatom[i] = 0.0;
    }
    if (vflag_atom) {
      if (n > maxvatom) {
        memory->destroy(vatom);
        memory->create(vatom, n, 6, "pair:vatom");
        maxvatom = n;
      }
      for (int i = 0; i < n; ++i)
        for (int k = 0; k < 6; ++k) vatom[i][k] = 0.0;
    }
  }

  NeighList *list = nullptr;
  double eng_vdwl = 0.0, virial[6] = {0, 0, 0, 0, 0, 0};
  double *eatom = nullptr;
  double **vatom = nullptr;
  int maxeatom = 0, maxvatom = 0;
  int eflag_global = 0, eflag_atom = 0, vflag_global = 0, vflag_atom = 0;
  int allocated = 0, single_enable = 1, restartinfo = 1, one_coeff = 0, manybody_flag = 0;
  int no_virial_fdotr_compute = 0;
  int **setflag = nullptr;
  double **cutsq = nullptr;
};

}  // namespace LAMMPS_NS
