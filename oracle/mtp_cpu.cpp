// mtp_cpu.cpp - FP64 CPU restatement of the MTP energy/force/stress path.
//
// TEST INFRASTRUCTURE ONLY: the checker and the timed CPU baseline.  Only
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it;
// the product never does.
//
// Follows the reference's algorithm literally, with OpenMP over atoms:
//   * radial functions: Chebyshev T_n of x = (2d - (rmin + rmax)) / (rmax - rmin),
//     times scaling * (rmax - d)^2, contracted with c[t_i, t_j, mu, :]
//     (jax_backend.py:83-95, 108-160); a slot counts when t_j >= 0 and
//     d < rmax (jax_backend.py:86-88);
//   * basic moments m_k = sum_j f_{mu_k}(d_j) u_x^a u_y^b u_z^c and the
//     contraction list applied in table order, m[i3] += mult m[i1] m[i2]
//     (motep_original_files/jax_engine/conversion.py:59-102);
//   * E_i = xi[t_i] + sum_a theta_a m[map_a] (jax_backend.py:101-106);
//   * dE_i/dr_ij by the reverse of that program (what jax.value_and_grad
//     computes at jax_backend.py:56);
//   * forces with the reference's Newton-3rd accumulation and masks
//     (jax_backend.py:263-303), serially in atom/slot order;
//   * LAMMPS virial W = -sym(sum r (x) g) (the reference's stress is -W/V in
//     order xx,yy,zz,yz,xz,xy, jax_backend.py:355-360).
#include <omp.h>

#include <cmath>
#include <cstring>
#include <vector>

namespace {

struct CpuModel {
  int S, R, K, M, B, T, Sa, maxdeg;
  double scaling, rmin, rmax;
  std::vector<double> radial, species, moment;
  std::vector<int> basic, times, mapping;
};

}  // namespace

extern "C" {

void* mtpcpu_create(int S, int R, int K, int M, int B, int T, int Sa, double scaling, double rmin, double rmax,
                    const double* radial, const int* basic, const int* times, const int* mapping,
                    const double* species, const double* moment) {
  auto* m = new CpuModel();
  m->S = S; m->R = R; m->K = K; m->M = M; m->B = B; m->T = T; m->Sa = Sa;
  m->scaling = scaling; m->rmin = rmin; m->rmax = rmax;
  m->radial.assign(radial, radial + static_cast<size_t>(S) * S * R * K);
  m->basic.assign(basic, basic + 4 * B);
  m->times.assign(times, times + 4 * T);
  m->mapping.assign(mapping, mapping + Sa);
  m->species.assign(species, species + S);
  m->moment.assign(moment, moment + Sa);
  m->maxdeg = 0;
  for (int k = 0; k < B; ++k) {
    int dgr = basic[4 * k + 1] + basic[4 * k + 2] + basic[4 * k + 3];
    if (dgr > m->maxdeg) m->maxdeg = dgr;
  }
  return m;
}

void mtpcpu_destroy(void* h) { delete static_cast<CpuModel*>(h); }

// Per-atom energies and per-slot gradients g [N][stride][3] (nthreads <= 0: all).
int mtpcpu_site(void* hp, int natoms, int stride, const int* itypes, const double* rijs, const int* jtypes,
                const int* counts, int nthreads, double* site_energy, double* grads) {
  const CpuModel& md = *static_cast<CpuModel*>(hp);
  if (nthreads > 0) omp_set_num_threads(nthreads);
  int bad = 0;
#pragma omp parallel reduction(| : bad)
  {
    const int R = md.R, K = md.K, M = md.M, B = md.B, D1 = md.maxdeg + 1;
    std::vector<double> m(M), dm(M), f, fp, pw, u;
    std::vector<int> slot;
#pragma omp for schedule(dynamic, 16)
    for (int i = 0; i < natoms; ++i) {
      const int it = itypes[i];
      if (it < 0 || it >= md.S) {
        bad = 1;
        continue;
      }
      const int cnt = counts ? counts[i] : stride;
      f.assign(static_cast<size_t>(cnt) * R, 0.0);
      fp.assign(static_cast<size_t>(cnt) * R, 0.0);
      pw.assign(static_cast<size_t>(cnt) * 3 * D1, 0.0);
      u.assign(static_cast<size_t>(cnt) * 4, 0.0);
      slot.clear();
      double* g = grads + static_cast<size_t>(i) * stride * 3;
      std::memset(g, 0, sizeof(double) * stride * 3);
      int nv = 0;
      for (int s = 0; s < cnt; ++s) {
        const int jt = jtypes[static_cast<size_t>(i) * stride + s];
        if (jt < 0) continue;
        if (jt >= md.S) { bad = 1; continue; }
        const double* r = rijs + 3 * (static_cast<size_t>(i) * stride + s);
        const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        const double d = std::sqrt(r2);
        if (!(r2 > 0.0) || !(d < md.rmax)) continue;
        const double inv_range = 1.0 / (md.rmax - md.rmin);
        const double x = (2.0 * d - (md.rmin + md.rmax)) * inv_range;
        std::vector<double> Tn(K), dTn(K);
        Tn[0] = 1.0; dTn[0] = 0.0;
        if (K > 1) { Tn[1] = x; dTn[1] = 1.0; }
        for (int n = 2; n < K; ++n) {
          Tn[n] = 2.0 * x * Tn[n - 1] - Tn[n - 2];
          dTn[n] = 2.0 * Tn[n - 1] + 2.0 * x * dTn[n - 1] - dTn[n - 2];
        }
        const double gap = md.rmax - d, smooth = gap * gap;
        const double* c = &md.radial[(static_cast<size_t>(it) * md.S + jt) * R * K];
        for (int mu = 0; mu < R; ++mu) {
          double b = 0.0, db = 0.0;
          for (int n = 0; n < K; ++n) {
            b += c[mu * K + n] * Tn[n];
            db += c[mu * K + n] * dTn[n];
          }
          f[nv * R + mu] = md.scaling * smooth * b;
          fp[nv * R + mu] = md.scaling * (-2.0 * gap * b + smooth * db * 2.0 * inv_range);
        }
        const double ux = r[0] / d, uy = r[1] / d, uz = r[2] / d;
        u[4 * nv] = ux; u[4 * nv + 1] = uy; u[4 * nv + 2] = uz; u[4 * nv + 3] = d;
        double* p = &pw[static_cast<size_t>(nv) * 3 * D1];
        p[0] = p[D1] = p[2 * D1] = 1.0;
        for (int e = 1; e < D1; ++e) {
          p[e] = p[e - 1] * ux;
          p[D1 + e] = p[D1 + e - 1] * uy;
          p[2 * D1 + e] = p[2 * D1 + e - 1] * uz;
        }
        slot.push_back(s);
        ++nv;
      }
      // basic moments, then the contraction list in table order
      for (int k = 0; k < M; ++k) m[k] = 0.0;
      for (int k = 0; k < B; ++k) {
        const int mu = md.basic[4 * k], a = md.basic[4 * k + 1], b = md.basic[4 * k + 2], cc = md.basic[4 * k + 3];
        double acc = 0.0;
        for (int q = 0; q < nv; ++q) {
          const double* p = &pw[static_cast<size_t>(q) * 3 * D1];
          acc += f[q * R + mu] * p[a] * p[D1 + b] * p[2 * D1 + cc];
        }
        m[k] = acc;
      }
      for (int e = 0; e < md.T; ++e) {
        const int* t = &md.times[4 * e];
        m[t[3]] += t[2] * m[t[0]] * m[t[1]];
      }
      double E = md.species[it];
      for (int a = 0; a < md.Sa; ++a) E += md.moment[a] * m[md.mapping[a]];
      site_energy[i] = E;
      // reverse of the program
      for (int k = 0; k < M; ++k) dm[k] = 0.0;
      for (int a = 0; a < md.Sa; ++a) dm[md.mapping[a]] += md.moment[a];
      for (int e = md.T - 1; e >= 0; --e) {
        const int* t = &md.times[4 * e];
        const double w = t[2] * dm[t[3]];
        dm[t[0]] += w * m[t[1]];
        dm[t[1]] += w * m[t[0]];
      }
      // dE/dr per kept neighbour
      for (int q = 0; q < nv; ++q) {
        const double* p = &pw[static_cast<size_t>(q) * 3 * D1];
        double Ssum = 0.0, Gx = 0.0, Gy = 0.0, Gz = 0.0;
        for (int k = 0; k < B; ++k) {
          const int mu = md.basic[4 * k], a = md.basic[4 * k + 1], b = md.basic[4 * k + 2], cc = md.basic[4 * k + 3];
          const double wv = dm[k] * f[q * R + mu], wp = dm[k] * fp[q * R + mu];
          const double px = p[a], py = p[D1 + b], pz = p[2 * D1 + cc];
          Ssum += wp * px * py * pz;
          if (a) Gx += wv * a * p[a - 1] * py * pz;
          if (b) Gy += wv * b * px * p[D1 + b - 1] * pz;
          if (cc) Gz += wv * cc * px * py * p[2 * D1 + cc - 1];
        }
        const double ux = u[4 * q], uy = u[4 * q + 1], uz = u[4 * q + 2], d = u[4 * q + 3];
        const double ug = ux * Gx + uy * Gy + uz * Gz;
        double* gs = g + 3 * slot[q];
        gs[0] = ux * Ssum + (Gx - ux * ug) / d;
        gs[1] = uy * Ssum + (Gy - uy * ug) / d;
        gs[2] = uz * Ssum + (Gz - uz * ug) / d;
      }
    }
  }
  return bad;
}

// Full evaluation: total energy, site energies, forces [N][3], LAMMPS virial [6].
int mtpcpu_compute(void* hp, int natoms, int stride, const int* itypes, const double* rijs, const int* js,
                   const int* jtypes, const int* counts, int nthreads, double* energy, double* site_energy,
                   double* forces, double* virial, double* grads) {
  int bad = mtpcpu_site(hp, natoms, stride, itypes, rijs, jtypes, counts, nthreads, site_energy, grads);
  double E = 0.0, W[6] = {0, 0, 0, 0, 0, 0};
  std::memset(forces, 0, sizeof(double) * 3 * natoms);
  for (int i = 0; i < natoms; ++i) {
    E += site_energy[i];
    const int cnt = counts ? counts[i] : stride;
    for (int s = 0; s < cnt; ++s) {
      const size_t x = static_cast<size_t>(i) * stride + s;
      const double* g = grads + 3 * x;
      const double* r = rijs + 3 * x;
      forces[3 * i] += g[0];
      forces[3 * i + 1] += g[1];
      forces[3 * i + 2] += g[2];
      const int j = js[x];
      if (jtypes[x] >= 0 && j >= 0 && j < natoms) {
        forces[3 * j] -= g[0];
        forces[3 * j + 1] -= g[1];
        forces[3 * j + 2] -= g[2];
      }
      W[0] -= r[0] * g[0];
      W[1] -= r[1] * g[1];
      W[2] -= r[2] * g[2];
      W[3] -= 0.5 * (r[0] * g[1] + r[1] * g[0]);
      W[4] -= 0.5 * (r[0] * g[2] + r[2] * g[0]);
      W[5] -= 0.5 * (r[1] * g[2] + r[2] * g[1]);
    }
  }
  *energy = E;
  std::memcpy(virial, W, sizeof(W));
  return bad;
}

}  // extern "C"
