/* ----------------------------------------------------------------------
   pair_style jax/mtp on the B200 MTP engine.

   Per step (compare PairJaxMTP::compute, pair_jax_mtp.cpp:69-207):
     - for every local atom i of the full list, neighbours j with
       |x_j - x_i| < MTP_CUTOFF form row i: r_ij = x_j - x_i (the ghost
       coordinates already hold the periodic image), the owner's local
       index, the owner's species (type - 1); a ghost without a local owner
       gets species -1 and is skipped by the evaluator, as in the reference
       (pair_jax_mtp.cpp:137-151).  With rows device (the default) the GPU
       builds the rows from positions and the list (mtp_compute_positions);
       with rows host they are packed here into persistent page-locked
       buffers (mtp_compute);
     - one call (energy, forces with the reaction terms folded onto owners,
       virial, optional per-atom energy/virial);
     - f[i] += F_i, eng_vdwl += E, virial += W (LAMMPS convention).
   Differences from the reference, each a fix: a row longer than
   MAX_ATOMS_PER_NEIGHBOR and nlocal > MAX_ATOMS are errors instead of silent
   truncation/overflow (pair_jax_mtp.cpp:90-98, 132); the virial is the LAMMPS
   virial instead of the stress divided by the volume in the wrong order and
   sign (pair_jax_mtp.cpp:203-205); no minimum-image folding of ghost vectors
   (pair_jax_mtp.cpp:128), which only matters for boxes under twice the cutoff.
------------------------------------------------------------------------- */

#include "pair_mtp_b200.h"

#include <cstring>
#include <string>

#include "atom.h"
#include "comm.h"
#include "error.h"
#include "force.h"
#include "memory.h"
#include "mtp_b200.h"
#include "neigh_list.h"
#include "neighbor.h"

using namespace LAMMPS_NS;

PairMTPB200::PairMTPB200(LAMMPS *lmp) : Pair(lmp)
{
  single_enable = 0;
  restartinfo = 0;
  one_coeff = 1;
  manybody_flag = 1;
  no_virial_fdotr_compute = 1;
  mtp_path = nullptr;
  cutoff = 0.0;
  max_atoms = max_nbr = 0;
  debug_level = 0;
  precision = MTP_PRECISION_FP64;
  rows_on_device = 1;
  handle = nullptr;
  total_calls = 0;
}

PairMTPB200::~PairMTPB200()
{
  if (handle) mtp_destroy(handle);
  delete[] mtp_path;
  if (allocated) {
    memory->destroy(setflag);
    memory->destroy(cutsq);
  }
}

void PairMTPB200::grow_buffers()
{
  const size_t rows = static_cast<size_t>(max_atoms);
  const size_t slots = rows * max_nbr;
  if (rij.size() != 3 * slots) {
    const bool ok = rij.assign(3 * slots, 0.0) && js.assign(slots, -1) && jtypes.assign(slots, -1) &&
        counts.assign(rows, 0) && itypes.assign(rows, 0) && fbuf.assign(3 * rows, 0.0) &&
        ebuf.assign(rows, 0.0) && vbuf.assign(6 * rows, 0.0);
    if (!ok) error->one(FLERR, std::string("pair jax/mtp: page-locked buffers: ") + mtp_last_error(nullptr));
  }
}

void PairMTPB200::compute(int eflag, int vflag)
{
  ev_init(eflag, vflag);
  double **x = atom->x;
  double **f = atom->f;
  int *type = atom->type;
  tagint *tag = atom->tag;
  const int nlocal = atom->nlocal;
  const int nall = nlocal + atom->nghost;

  if (nlocal > max_atoms)
    error->one(FLERR, "pair jax/mtp: " + std::to_string(nlocal) + " local atoms exceed MAX_ATOMS " +
                          std::to_string(max_atoms));
  grow_buffers();

  // owner of every ghost: local index of the atom with the same tag
  tagint maxtag = 0;
  for (int i = 0; i < nlocal; ++i) maxtag = tag[i] > maxtag ? tag[i] : maxtag;
  tag_to_local.assign(static_cast<size_t>(maxtag) + 1, -1);
  for (int i = 0; i < nlocal; ++i) tag_to_local[tag[i]] = i;
  auto owner_of = [&](int j) {
    if (j < nlocal) return j;
    return (tag[j] >= 0 && tag[j] <= maxtag) ? tag_to_local[tag[j]] : -1;
  };

  const int inum = list->inum;
  const int *ilist = list->ilist;
  const int *numneigh = list->numneigh;
  int **firstneigh = list->firstneigh;

  int flags = MTP_EFLAG | MTP_VFLAG;
  if (eflag_atom) flags |= MTP_EATOM;
  if (vflag_atom) flags |= MTP_VATOM;
  double energy = 0.0, w[6] = {0, 0, 0, 0, 0, 0};
  int status;
  if (rows_on_device) {
    // positions, species and owners of every atom, and the neighbour list as
    // it is (skin included): the GPU keeps the candidates inside the cutoff
    // (mtp_compute_positions)
    int lstride = 1;
    for (int ii = 0; ii < inum; ++ii) lstride = numneigh[ilist[ii]] > lstride ? numneigh[ilist[ii]] : lstride;
    const size_t na = static_cast<size_t>(nall);
    if (!(xall.ensure(3 * na) && spall.ensure(na) && owner.ensure(na) &&
          neigh.ensure(static_cast<size_t>(nlocal) * lstride) && nneigh.ensure(static_cast<size_t>(nlocal) + 1)))
      error->one(FLERR, std::string("pair jax/mtp: page-locked buffers: ") + mtp_last_error(nullptr));
    for (int j = 0; j < nall; ++j) {
      xall[3 * j] = x[j][0];
      xall[3 * j + 1] = x[j][1];
      xall[3 * j + 2] = x[j][2];
      spall[j] = type[j] - 1;
      owner[j] = owner_of(j);
    }
    std::memset(nneigh.data(), 0, sizeof(int) * nlocal);
    for (int ii = 0; ii < inum; ++ii) {
      const int i = ilist[ii];
      const int *jlist = firstneigh[i];
      int *row = neigh.data() + static_cast<size_t>(i) * lstride;
      for (int jj = 0; jj < numneigh[i]; ++jj) row[jj] = jlist[jj] & NEIGHMASK;
      nneigh[i] = numneigh[i];
    }
    status = mtp_compute_positions(handle, nlocal, nall, xall.data(), spall.data(), owner.data(), lstride,
                                   neigh.data(), nneigh.data(), flags, &energy, fbuf.data(), w,
                                   eflag_atom ? ebuf.data() : nullptr, vflag_atom ? vbuf.data() : nullptr);
  } else {
    // rows packed on the host, as the reference pair style does
    const double rc2 = cutoff * cutoff;
    std::memset(counts.data(), 0, sizeof(int) * nlocal);
    for (int i = 0; i < nlocal; ++i) itypes[i] = type[i] - 1;
    for (int ii = 0; ii < inum; ++ii) {
      const int i = ilist[ii];
      const double xi = x[i][0], yi = x[i][1], zi = x[i][2];
      const int *jlist = firstneigh[i];
      const size_t row = static_cast<size_t>(i) * max_nbr;
      int n = 0;
      for (int jj = 0; jj < numneigh[i]; ++jj) {
        const int j = jlist[jj] & NEIGHMASK;
        if (j == i || j >= nall) continue;
        const double dx = x[j][0] - xi, dy = x[j][1] - yi, dz = x[j][2] - zi;
        if (dx * dx + dy * dy + dz * dz >= rc2) continue;
        if (n == max_nbr)
          error->one(FLERR, "pair jax/mtp: atom " + std::to_string(tag[i]) +
                                " has more neighbours than MAX_ATOMS_PER_NEIGHBOR " + std::to_string(max_nbr));
        const int own = owner_of(j);
        double *r = &rij[3 * (row + n)];
        r[0] = dx;
        r[1] = dy;
        r[2] = dz;
        js[row + n] = own;
        jtypes[row + n] = own >= 0 ? type[j] - 1 : -1;
        ++n;
      }
      counts[i] = n;
    }
    status = mtp_compute(handle, nlocal, max_nbr, itypes.data(), rij.data(), js.data(), jtypes.data(), counts.data(),
                         flags, &energy, fbuf.data(), w, eflag_atom ? ebuf.data() : nullptr,
                         vflag_atom ? vbuf.data() : nullptr);
  }
  if (status != MTP_OK) error->one(FLERR, std::string("pair jax/mtp: ") + mtp_last_error(handle));

  for (int i = 0; i < nlocal; ++i) {
    f[i][0] += fbuf[3 * i];
    f[i][1] += fbuf[3 * i + 1];
    f[i][2] += fbuf[3 * i + 2];
  }
  if (eflag_global) eng_vdwl += energy;
  if (vflag_global)
    for (int k = 0; k < 6; ++k) virial[k] += w[k];
  if (eflag_atom)
    for (int i = 0; i < nlocal; ++i) eatom[i] += ebuf[i];
  if (vflag_atom)
    for (int i = 0; i < nlocal; ++i)
      for (int k = 0; k < 6; ++k) vatom[i][k] += vbuf[6 * i + k];
  ++total_calls;
}

void PairMTPB200::settings(int narg, char **arg)
{
  // trailing "rows device|host" keyword
  if (narg >= 6 && strcmp(arg[narg - 2], "rows") == 0) {
    if (strcmp(arg[narg - 1], "device") == 0) rows_on_device = 1;
    else if (strcmp(arg[narg - 1], "host") == 0) rows_on_device = 0;
    else error->all(FLERR, "pair jax/mtp: rows must be device or host");
    narg -= 2;
  }
  if (narg < 4 || narg > 6)
    error->all(FLERR, "Illegal pair_style command: pair_style jax/mtp <potential.mtp> <max_atoms> "
                      "<max_neighbors> <cutoff> [debug_level] [fp64|mixed] [rows device|host]");
  delete[] mtp_path;
  mtp_path = new char[strlen(arg[0]) + 1];
  strcpy(mtp_path, arg[0]);
  max_atoms = utils::inumeric(FLERR, arg[1], false, lmp);
  max_nbr = utils::inumeric(FLERR, arg[2], false, lmp);
  cutoff = utils::numeric(FLERR, arg[3], false, lmp);
  if (narg >= 5) debug_level = utils::inumeric(FLERR, arg[4], false, lmp);
  if (narg >= 6) {
    if (strcmp(arg[5], "fp64") == 0) precision = MTP_PRECISION_FP64;
    else if (strcmp(arg[5], "mixed") == 0) precision = MTP_PRECISION_MIXED;
    else error->all(FLERR, "pair jax/mtp: precision must be fp64 or mixed");
  }
  if (max_atoms <= 0 || max_nbr <= 0 || cutoff <= 0.0)
    error->all(FLERR, "max_atoms, max_neighbors, and cutoff must be positive");
}

void PairMTPB200::allocate()
{
  allocated = 1;
  const int n = atom->ntypes;
  memory->create(setflag, n + 1, n + 1, "pair:setflag");
  memory->create(cutsq, n + 1, n + 1, "pair:cutsq");
}

void PairMTPB200::coeff(int narg, char **arg)
{
  if (narg != 2 || strcmp(arg[0], "*") != 0 || strcmp(arg[1], "*") != 0)
    error->all(FLERR, "Incorrect args for pair coefficients: pair_coeff * *");
  if (!allocated) allocate();
  for (int i = 1; i <= atom->ntypes; i++)
    for (int j = 1; j <= atom->ntypes; j++) {
      setflag[i][j] = 1;
      cutsq[i][j] = cutoff * cutoff;
    }
}

double PairMTPB200::init_one(int i, int j)
{
  if (setflag[i][j] == 0) error->all(FLERR, "All pair coeffs are not set");
  return cutoff;
}

void PairMTPB200::init_style()
{
  if (atom->tag_enable == 0) error->all(FLERR, "Pair style jax/mtp requires atom IDs");
  if (comm->nprocs != 1) error->all(FLERR, "Pair style jax/mtp runs on one MPI rank");
  neighbor->add_request(this, NeighConst::REQ_FULL);
  if (!handle) {
    const int status = mtp_create(mtp_path, max_atoms, max_nbr, cutoff, debug_level, precision, &handle);
    if (status != MTP_OK) {
      handle = nullptr;
      error->all(FLERR, std::string("pair jax/mtp: ") + mtp_last_error(nullptr));
    }
    int info[8];
    mtp_get_info(handle, info);
    if (info[0] < atom->ntypes)
      error->all(FLERR, "pair jax/mtp: the potential has fewer species than atom types");
  }
}
