// mini_lammps.cpp - a small LAMMPS-like host MD driver for pair_style jax/mtp.
//
// Drives PairMTPB200 exactly as LAMMPS would with `units metal`, `atom_style
// atomic`, one MPI rank, `fix nve`, and a full neighbour list with ghost
// atoms: it owns local + ghost coordinates, builds the full list with bins
// every `every` steps (skin distance), refreshes ghost coordinates every step,
// and calls Pair::compute(eflag, vflag).  It is the host-side call path of the
// reference's config (pair_style_files/pair_jax_mtp.cpp:69-207) with the
// engine behind the C ABI, used to test and time the pair style without a
// LAMMPS installation.
//
// usage: mini_lammps <data.txt> <potential.mtp> <max_atoms> <max_nbr> <cutoff> <mass_amu>
//                    <dt_ps> <steps> <every> <skin> [fp64|mixed] [thermo_every]
//                    [device|host rows] [nve|boxrelax] [ftol_eV_per_A] [ptol_bar] [out.txt]
// data.txt: "natoms ntypes" / "Lx Ly Lz" / natoms lines "tag type x y z vx vy vz"
// (orthorhombic box [0, L)).  Prints thermo lines and a final JSON summary.
//
// Mode nve (default): velocity Verlet for <steps> steps (LAMMPS `fix nve`).
// Mode boxrelax: the energy minimisation of the reference's own input,
// `fix box/relax iso 0.0` + `minimize` (test_lammps.in:27-28), driven by the
// pair style's virial: atoms relax by FIRE at fixed box until max |F| <
// ftol, then the box is rescaled isotropically (atoms affinely) by a secant
// step on the pressure P = (W_xx + W_yy + W_zz) / (3 V) towards zero, for at
// most <steps> box updates or until |P| < ptol with the atoms relaxed.
// Prints one "relax" line per box update and a final JSON summary with the
// box, the energy and the pressure; with out.txt, the final box and local
// atoms are written there in the data-file format (zero velocities).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "pair_mtp_b200.h"

using namespace LAMMPS_NS;

namespace {

constexpr double kMvv2e = 1.0364269e-4;   // amu A^2/ps^2 -> eV
constexpr double kBoltz = 8.617343e-5;    // eV/K (LAMMPS metal)

struct Sim {
  int nlocal = 0, nghost = 0, ntypes = 0;
  double L[3] = {0, 0, 0};
  std::vector<double> xbuf, fbuf, v;
  std::vector<double*> x, f;
  std::vector<int> type, tag;
  std::vector<int> ghost_owner;
  std::vector<double> ghost_shift;
  // full neighbour list
  std::vector<int> ilist, numneigh, pages;
  std::vector<int*> firstneigh;
};

void set_ptrs(Sim& s) {
  const int n = s.nlocal + s.nghost;
  s.x.resize(n);
  s.f.resize(n);
  for (int i = 0; i < n; ++i) {
    s.x[i] = &s.xbuf[3 * i];
    s.f[i] = &s.fbuf[3 * i];
  }
}

// periodic images of local atoms within `rcut` of the box faces
void build_ghosts(Sim& s, double rcut) {
  s.ghost_owner.clear();
  s.ghost_shift.clear();
  for (int i = 0; i < s.nlocal; ++i)
    for (int a = 0; a < 3; ++a) {
      s.xbuf[3 * i + a] -= std::floor(s.xbuf[3 * i + a] / s.L[a]) * s.L[a];
    }
  for (int sx = -1; sx <= 1; ++sx)
    for (int sy = -1; sy <= 1; ++sy)
      for (int sz = -1; sz <= 1; ++sz) {
        if (!sx && !sy && !sz) continue;
        const int sh[3] = {sx, sy, sz};
        for (int i = 0; i < s.nlocal; ++i) {
          bool keep = true;
          for (int a = 0; a < 3 && keep; ++a) {
            const double y = s.xbuf[3 * i + a] + sh[a] * s.L[a];
            keep = y >= -rcut && y < s.L[a] + rcut;
          }
          if (!keep) continue;
          s.ghost_owner.push_back(i);
          for (int a = 0; a < 3; ++a) s.ghost_shift.push_back(sh[a] * s.L[a]);
        }
      }
  s.nghost = static_cast<int>(s.ghost_owner.size());
  const int n = s.nlocal + s.nghost;
  s.xbuf.resize(3 * n);
  s.fbuf.assign(3 * n, 0.0);
  s.type.resize(n);
  s.tag.resize(n);
  for (int g = 0; g < s.nghost; ++g) {
    const int o = s.ghost_owner[g], k = s.nlocal + g;
    s.type[k] = s.type[o];
    s.tag[k] = s.tag[o];
    for (int a = 0; a < 3; ++a) s.xbuf[3 * k + a] = s.xbuf[3 * o + a] + s.ghost_shift[3 * g + a];
  }
  set_ptrs(s);
}

void update_ghosts(Sim& s) {
  for (int g = 0; g < s.nghost; ++g) {
    const int o = s.ghost_owner[g], k = s.nlocal + g;
    for (int a = 0; a < 3; ++a) s.xbuf[3 * k + a] = s.xbuf[3 * o + a] + s.ghost_shift[3 * g + a];
  }
}

// full list of every local atom over local + ghost atoms, binned
void build_list(Sim& s, double rcut) {
  const int n = s.nlocal + s.nghost;
  int nb[3];
  double lo[3], bw[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = -rcut;
    nb[a] = std::max(1, static_cast<int>(std::floor((s.L[a] + 2 * rcut) / rcut)));
    bw[a] = (s.L[a] + 2 * rcut) / nb[a];
  }
  const int nbins = nb[0] * nb[1] * nb[2];
  std::vector<int> head(nbins, -1), next(n, -1), bin_of(n);
  for (int i = n - 1; i >= 0; --i) {
    int c[3];
    for (int a = 0; a < 3; ++a) c[a] = std::min(nb[a] - 1, std::max(0, static_cast<int>((s.xbuf[3 * i + a] - lo[a]) / bw[a])));
    const int b = (c[0] * nb[1] + c[1]) * nb[2] + c[2];
    bin_of[i] = b;
    next[i] = head[b];
    head[b] = i;
  }
  const double rc2 = rcut * rcut;
  s.ilist.resize(s.nlocal);
  s.numneigh.assign(s.nlocal, 0);
  s.pages.clear();
  std::vector<size_t> start(s.nlocal);
  for (int i = 0; i < s.nlocal; ++i) {
    s.ilist[i] = i;
    start[i] = s.pages.size();
    const int b = bin_of[i];
    const int c0 = b / (nb[1] * nb[2]), c1 = (b / nb[2]) % nb[1], c2 = b % nb[2];
    for (int d0 = -1; d0 <= 1; ++d0)
      for (int d1 = -1; d1 <= 1; ++d1)
        for (int d2 = -1; d2 <= 1; ++d2) {
          const int e0 = c0 + d0, e1 = c1 + d1, e2 = c2 + d2;
          if (e0 < 0 || e1 < 0 || e2 < 0 || e0 >= nb[0] || e1 >= nb[1] || e2 >= nb[2]) continue;
          for (int j = head[(e0 * nb[1] + e1) * nb[2] + e2]; j >= 0; j = next[j]) {
            if (j == i) continue;
            double r2 = 0.0;
            for (int a = 0; a < 3; ++a) {
              const double d = s.xbuf[3 * j + a] - s.xbuf[3 * i + a];
              r2 += d * d;
            }
            if (r2 < rc2) s.pages.push_back(j);
          }
        }
    s.numneigh[i] = static_cast<int>(s.pages.size() - start[i]);
  }
  s.firstneigh.resize(s.nlocal);
  for (int i = 0; i < s.nlocal; ++i) s.firstneigh[i] = s.pages.data() + start[i];
}

constexpr double kNktv2p = 1.6021765e6;   // eV/A^3 -> bar (LAMMPS metal)

// Total force on the local atoms after the ghost forces went to their owners.
double max_force(const Sim& s) {
  double m = 0.0;
  for (int i = 0; i < s.nlocal; ++i)
    for (int a = 0; a < 3; ++a) m = std::max(m, std::fabs(s.fbuf[3 * i + a]));
  return m;
}

void fold_ghost_forces(Sim& s) {
  for (int g = 0; g < s.nghost; ++g)
    for (int a = 0; a < 3; ++a) s.fbuf[3 * s.ghost_owner[g] + a] += s.fbuf[3 * (s.nlocal + g) + a];
}

// fix box/relax iso 0.0 + minimize, as alternating FIRE atom relaxation at
// fixed box and secant steps of the isotropic box length on the pressure.
template <typename Pair, typename Rebuild, typename Bind, typename Force>
int box_relax(Sim& s, Pair& pair, Rebuild rebuild, Bind bind, Force force_call, double mass, double dt,
              int max_box_steps, double ftol, double ptol_bar) {
  auto evaluate = [&](double* pe, double* press) {
    rebuild();
    bind();
    force_call(1, 1);
    fold_ghost_forces(s);
    const double vol = s.L[0] * s.L[1] * s.L[2];
    *pe = pair.eng_vdwl;
    *press = (pair.virial[0] + pair.virial[1] + pair.virial[2]) / (3.0 * vol);   // eV/A^3, T = 0
  };
  // FIRE (Bitzek et al., PRL 97, 170201 (2006)) on the atoms at fixed box
  auto relax_atoms = [&](double* pe, double* press) {
    const int n = s.nlocal;
    std::vector<double> vel(3 * n, 0.0);
    double dtf = dt, alpha = 0.1;
    int npos = 0, it = 0;
    evaluate(pe, press);
    for (; it < 20000 && max_force(s) >= ftol; ++it) {
      double P = 0.0, vn = 0.0, fn = 0.0;
      for (int k = 0; k < 3 * n; ++k) {
        P += s.fbuf[k] * vel[k];
        vn += vel[k] * vel[k];
        fn += s.fbuf[k] * s.fbuf[k];
      }
      vn = std::sqrt(vn);
      fn = std::sqrt(fn);
      if (P > 0.0) {
        for (int k = 0; k < 3 * n; ++k) vel[k] = (1.0 - alpha) * vel[k] + alpha * s.fbuf[k] / fn * vn;
        if (++npos > 5) {
          dtf = std::min(dtf * 1.1, 10.0 * dt);
          alpha *= 0.99;
        }
      } else {
        std::fill(vel.begin(), vel.end(), 0.0);
        dtf *= 0.5;
        alpha = 0.1;
        npos = 0;
      }
      const double im = 1.0 / (mass * kMvv2e);
      for (int k = 0; k < 3 * n; ++k) {
        vel[k] += dtf * s.fbuf[k] * im;
        s.xbuf[k] += dtf * vel[k];
      }
      evaluate(pe, press);
    }
    return it;
  };
  double pe = 0.0, press = 0.0;
  int atom_iters = relax_atoms(&pe, &press);
  double Lprev = 0.0, Pprev = 0.0;
  int k = 0;
  bool converged = false;
  for (; k < max_box_steps; ++k) {
    std::printf("relax %d L %.12f %.12f %.12f pe %.12f press_bar %.6f fmax %.3e atom_iters %d\n", k, s.L[0],
                s.L[1], s.L[2], pe, press * kNktv2p, max_force(s), atom_iters);
    if (std::fabs(press * kNktv2p) < ptol_bar && max_force(s) < ftol) {
      converged = true;
      break;
    }
    const double L = s.L[0];
    double Lnew;
    if (k == 0) {
      // first step: a 0.1 % trial strain in the direction of the pressure
      Lnew = L * (press > 0.0 ? 1.001 : 0.999);
    } else {
      Lnew = L - press * (L - Lprev) / (press - Pprev);
    }
    Lnew = std::min(std::max(Lnew, 0.98 * L), 1.02 * L);
    Lprev = L;
    Pprev = press;
    const double f = Lnew / L;
    for (int a = 0; a < 3; ++a) s.L[a] *= f;
    for (int i = 0; i < s.nlocal; ++i)
      for (int a = 0; a < 3; ++a) s.xbuf[3 * i + a] *= f;
    atom_iters = relax_atoms(&pe, &press);
  }
  std::printf("{\"mode\": \"boxrelax\", \"atoms\": %d, \"box\": [%.15g, %.15g, %.15g], \"pe\": %.15g, "
              "\"press_bar\": %.9g, \"fmax\": %.6g, \"box_steps\": %d, \"converged\": %s, "
              "\"pair_calls\": %lld}\n",
              s.nlocal, s.L[0], s.L[1], s.L[2], pe, press * kNktv2p, max_force(s), k, converged ? "true" : "false",
              pair.calls());
  return converged ? 0 : 3;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 11) {
    std::fprintf(stderr, "usage: %s data.txt potential.mtp max_atoms max_nbr cutoff mass dt steps every skin "
                         "[fp64|mixed] [thermo_every] [device|host rows] [nve|boxrelax] [ftol] [ptol_bar]\n",
                 argv[0]);
    return 2;
  }
  const std::string data = argv[1], pot = argv[2];
  const int max_atoms = std::atoi(argv[3]), max_nbr = std::atoi(argv[4]);
  const double cutoff = std::atof(argv[5]), mass = std::atof(argv[6]), dt = std::atof(argv[7]);
  const int steps = std::atoi(argv[8]), every = std::atoi(argv[9]);
  const double skin = std::atof(argv[10]);
  const std::string prec = argc > 11 ? argv[11] : "fp64";
  const int thermo = argc > 12 ? std::atoi(argv[12]) : 100;
  const std::string rows = argc > 13 ? argv[13] : "device";
  const std::string mode = argc > 14 ? argv[14] : "nve";
  const double ftol = argc > 15 ? std::atof(argv[15]) : 1e-6;
  const double ptol_bar = argc > 16 ? std::atof(argv[16]) : 0.1;
  const std::string out_path = argc > 17 ? argv[17] : "";
  if (mode != "nve" && mode != "boxrelax") {
    std::fprintf(stderr, "unknown mode '%s' (nve or boxrelax)\n", mode.c_str());
    return 2;
  }

  Sim s;
  {
    std::ifstream in(data);
    if (!in) { std::fprintf(stderr, "cannot open %s\n", data.c_str()); return 2; }
    in >> s.nlocal >> s.ntypes >> s.L[0] >> s.L[1] >> s.L[2];
    s.xbuf.resize(3 * s.nlocal);
    s.v.resize(3 * s.nlocal);
    s.type.resize(s.nlocal);
    s.tag.resize(s.nlocal);
    for (int i = 0; i < s.nlocal; ++i)
      in >> s.tag[i] >> s.type[i] >> s.xbuf[3 * i] >> s.xbuf[3 * i + 1] >> s.xbuf[3 * i + 2] >> s.v[3 * i] >>
          s.v[3 * i + 1] >> s.v[3 * i + 2];
    if (!in) { std::fprintf(stderr, "bad data file\n"); return 2; }
  }

  Atom atom;
  Neighbor neighbor;
  Error error;
  Memory memory;
  Comm comm;
  Force force;
  LAMMPS lmp;
  lmp.atom = &atom;
  lmp.neighbor = &neighbor;
  lmp.error = &error;
  lmp.memory = &memory;
  lmp.comm = &comm;
  lmp.force = &force;
  atom.ntypes = s.ntypes;

  NeighList list;
  int rc = 0;
  try {
    PairMTPB200 pair(&lmp);
    std::string a1 = pot, a2 = std::to_string(max_atoms), a3 = std::to_string(max_nbr), a4 = argv[5], a5 = "0";
    std::string a7 = "rows", a8 = rows;
    char* sargs[] = {&a1[0], &a2[0], &a3[0], &a4[0], &a5[0], const_cast<char*>(prec.c_str()), &a7[0], &a8[0]};
    pair.settings(8, sargs);
    char star[] = "*";
    char* cargs[] = {star, star};
    pair.coeff(2, cargs);
    pair.init_style();
    pair.list = &list;

    const double rlist = cutoff + skin;
    auto rebuild = [&]() {
      build_ghosts(s, rlist);
      build_list(s, rlist);
      list.inum = s.nlocal;
      list.ilist = s.ilist.data();
      list.numneigh = s.numneigh.data();
      list.firstneigh = s.firstneigh.data();
    };
    auto bind = [&]() {
      atom.nlocal = s.nlocal;
      atom.nghost = s.nghost;
      atom.x = s.x.data();
      atom.f = s.f.data();
      atom.type = s.type.data();
      atom.tag = s.tag.data();
    };
    double pair_ms = 0.0;
    auto force_call = [&](int eflag, int vflag) {
      std::fill(s.fbuf.begin(), s.fbuf.end(), 0.0);
      auto t0 = std::chrono::steady_clock::now();
      pair.compute(eflag, vflag);
      pair_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    };
    const double vol = s.L[0] * s.L[1] * s.L[2];
    auto thermo_line = [&](int step) {
      double ke = 0.0;
      for (int i = 0; i < s.nlocal; ++i)
        for (int a = 0; a < 3; ++a) ke += 0.5 * mass * s.v[3 * i + a] * s.v[3 * i + a] * kMvv2e;
      const double pe = pair.eng_vdwl;
      const double T = 2.0 * ke / (3.0 * s.nlocal * kBoltz);
      // pressure in bar (LAMMPS metal nktv2p = 1.6021765e6)
      const double press = (2.0 * ke / 3.0 + (pair.virial[0] + pair.virial[1] + pair.virial[2]) / 3.0) / vol * 1.6021765e6;
      std::printf("step %d pe %.10f ke %.10f etotal %.10f temp %.3f press %.6f\n", step, pe, ke, pe + ke, T, press);
      return pe + ke;
    };

    if (mode == "boxrelax") {
      rc = box_relax(s, pair, rebuild, bind, force_call, mass, dt, steps, ftol, ptol_bar);
      if (!out_path.empty()) {
        std::FILE* fo = std::fopen(out_path.c_str(), "w");
        if (!fo) {
          std::fprintf(stderr, "cannot write %s\n", out_path.c_str());
          return 2;
        }
        std::fprintf(fo, "%d %d\n%.17g %.17g %.17g\n", s.nlocal, s.ntypes, s.L[0], s.L[1], s.L[2]);
        for (int i = 0; i < s.nlocal; ++i)
          std::fprintf(fo, "%d %d %.17g %.17g %.17g 0 0 0\n", s.tag[i], s.type[i], s.xbuf[3 * i], s.xbuf[3 * i + 1],
                       s.xbuf[3 * i + 2]);
        std::fclose(fo);
      }
      return rc;
    }
    rebuild();
    bind();
    force_call(1, 1);
    const double e_start = thermo_line(0);
    double e_last = e_start;
    const double dtf = 0.5 * dt / (mass * kMvv2e);
    auto t_start = std::chrono::steady_clock::now();
    pair_ms = 0.0;
    for (int step = 1; step <= steps; ++step) {
      for (int i = 0; i < s.nlocal; ++i)
        for (int a = 0; a < 3; ++a) {
          s.v[3 * i + a] += dtf * s.f[i][a];
          s.xbuf[3 * i + a] += dt * s.v[3 * i + a];
        }
      if (step % every == 0) {
        rebuild();
      } else {
        update_ghosts(s);
      }
      bind();
      const bool th = (step % thermo == 0) || step == steps;
      force_call(th ? 1 : 0, th ? 1 : 0);
      // reverse communication of ghost forces to their owners
      for (int g = 0; g < s.nghost; ++g)
        for (int a = 0; a < 3; ++a) s.f[s.ghost_owner[g]][a] += s.f[s.nlocal + g][a];
      for (int i = 0; i < s.nlocal; ++i)
        for (int a = 0; a < 3; ++a) s.v[3 * i + a] += dtf * s.f[i][a];
      if (th) e_last = thermo_line(step);
    }
    const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    std::printf("{\"atoms\": %d, \"steps\": %d, \"wall_s\": %.6f, \"atom_steps_per_s\": %.3f, "
                "\"pair_ms_per_step\": %.6f, \"energy_drift_eV_per_atom\": %.3e, \"pair_calls\": %lld}\n",
                s.nlocal, steps, wall, s.nlocal * static_cast<double>(steps) / wall, pair_ms / steps,
                (e_last - e_start) / s.nlocal, pair.calls());
  } catch (const std::exception& e) {
    std::fprintf(stderr, "ERROR: %s\n", e.what());
    rc = 1;
  }
  return rc;
}
