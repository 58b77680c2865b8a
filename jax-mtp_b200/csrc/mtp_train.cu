// mtp_train.cu - dual-number adjoint kernel for the coefficient gradient.
#include <algorithm>

#include "mtp_train.hpp"

namespace mtp {

struct TrainSmem {
  int pws;
  size_t v, rad, u, du, f, fp, phi, phip, pw, A, Bv, jt, gxi, grad, red, cnt, total;
};

template <typename T>
__host__ __device__ inline TrainSmem train_layout(int v_size, int S, int R, int K, int P, int D, int Sa, int n_pad,
                                                  int threads) {
  TrainSmem L;
  L.pws = 3 * (D + 1);
  if ((L.pws & 1) == 0) L.pws += 1;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    size_t at = (o + 15) & ~size_t(15);
    o = at + bytes;
    return at;
  };
  L.v = take(sizeof(T) * 2 * v_size);
  L.rad = take(sizeof(T) * S * S * R * K);
  L.u = take(sizeof(T) * 4 * n_pad);
  L.du = take(sizeof(T) * 4 * n_pad);
  L.f = take(sizeof(T) * R * n_pad);
  L.fp = take(sizeof(T) * R * n_pad);
  L.phi = take(sizeof(T) * K * n_pad);
  L.phip = take(sizeof(T) * K * n_pad);
  L.pw = take(sizeof(T) * L.pws * n_pad);
  L.A = take(sizeof(T) * R * n_pad);
  L.Bv = take(sizeof(T) * R * n_pad);
  L.jt = take(sizeof(int) * n_pad);
  L.gxi = take(sizeof(double) * S);
  L.grad = take(sizeof(double) * S * S * R * K);
  L.red = take(sizeof(double) * (threads / 32));
  L.cnt = take(sizeof(int) * (threads / 32 + 1));
  L.total = (o + 15) & ~size_t(15);
  return L;
}

// A value and its tangent side by side, so one 16-byte access serves both.
template <typename T>
struct Dual2;
template <>
struct Dual2<double> {
  using type = double2;
  static __device__ __forceinline__ double2 make(double v, double t) { return make_double2(v, t); }
};
template <>
struct Dual2<float> {
  using type = float2;
  static __device__ __forceinline__ float2 make(float v, float t) { return make_float2(v, t); }
};

// Forward pass on duals: (m3, dm3) += c * (m1 m2, dm1 m2 + m1 dm2).
// Operands are read through Vr and flushes go through V: a pass never reads
// a slot that it writes, so the two views do not alias (which lets the loads
// of later entries move ahead of earlier flushes).
template <typename T>
struct DualOperands {
  typename Dual2<T>::type a, b;
};

template <typename T>
struct DualFwdBody {
  using Operands = DualOperands<T>;
  typename Dual2<T>::type* __restrict__ V;
  const typename Dual2<T>::type* __restrict__ Vr;
  T acc, tac;
  __device__ __forceinline__ Operands load(const uint2 e) const { return {Vr[e.x & 0xFFFFu], Vr[e.x >> 16]}; }
  __device__ __forceinline__ void apply(const uint2 e, const Operands& o) {
    const T c = entry_mult<T>(e.y);
    const auto A = o.a, B = o.b;
    acc = dev_fma(c * A.x, B.x, acc);
    tac = dev_fma(c, dev_fma(A.y, B.x, A.x * B.y), tac);
    const uint32_t op = (e.y >> kOpShift) & 3u;
    if (op) {
      const uint32_t d = e.y >> kDstShift;
      if (op == kOpStore) {
        V[d] = Dual2<T>::make(acc, tac);
      } else {
        const auto o = V[d];
        V[d] = Dual2<T>::make(o.x + acc, o.y + tac);
      }
      acc = T(0);
      tac = T(0);
    }
  }
};

// Reverse pass on duals (entries dst = adj[s], a = adj[t], b = m[o]):
//   lambda_s += c (lambda_t m_o + tau_t dm_o),  tau_s += c tau_t m_o.
template <typename T>
struct DualRevBody {
  using Operands = DualOperands<T>;
  typename Dual2<T>::type* __restrict__ V;
  const typename Dual2<T>::type* __restrict__ Vr;
  T acc, tac;
  __device__ __forceinline__ Operands load(const uint2 e) const { return {Vr[e.x & 0xFFFFu], Vr[e.x >> 16]}; }
  __device__ __forceinline__ void apply(const uint2 e, const Operands& o) {
    const T c = entry_mult<T>(e.y);
    const auto A = o.a, B = o.b;   // (lambda_t, tau_t), (m_o, dm_o)
    acc = dev_fma(c, dev_fma(A.x, B.x, A.y * B.y), acc);
    tac = dev_fma(c * A.y, B.x, tac);
    const uint32_t op = (e.y >> kOpShift) & 3u;
    if (op) {
      const uint32_t d = e.y >> kDstShift;
      if (op == kOpStore) {
        V[d] = Dual2<T>::make(acc, tac);
      } else {
        const auto o = V[d];
        V[d] = Dual2<T>::make(o.x + acc, o.y + tac);
      }
      acc = T(0);
      tac = T(0);
    }
  }
};

template <typename T, bool kVGlobal>
__global__ void __launch_bounds__(512) k_mtp_adjoint(DevModel md, TrainIO io, int n_pad, void* vscratch,
                                                     double* partials) {
  extern __shared__ __align__(32) unsigned char smem[];
  const int NT = blockDim.x, tid = threadIdx.x;
  const int my_wsteps = warp_steps_of_lane(md, tid, NT);
  const int S = md.S, R = md.R, K = md.K, P = md.P, D1 = md.D + 1;
  const TrainSmem L = train_layout<T>(kVGlobal ? 0 : md.v_size, S, R, K, P, md.D, md.Sa, n_pad, NT);
  using T2 = typename Dual2<T>::type;
  // program entries in flight per thread; with the value space in global
  // memory their operand gathers are issued before any of their flushes
  // (level 28, 32 configurations: 26.1 ms with two entries in flight and
  // gathers at use -> 19.0 ms)
  constexpr int kStreamDepth = kPrefetch;
  T2* V = kVGlobal ? reinterpret_cast<T2*>(vscratch) + static_cast<size_t>(blockIdx.x) * md.v_size
                   : reinterpret_cast<T2*>(smem + L.v);
  T* sRad = reinterpret_cast<T*>(smem + L.rad);
  T* sU = reinterpret_cast<T*>(smem + L.u);
  T* sDu = reinterpret_cast<T*>(smem + L.du);
  T* sF = reinterpret_cast<T*>(smem + L.f);
  T* sFp = reinterpret_cast<T*>(smem + L.fp);
  T* sPhi = reinterpret_cast<T*>(smem + L.phi);
  T* sPhip = reinterpret_cast<T*>(smem + L.phip);
  T* sPw = reinterpret_cast<T*>(smem + L.pw);
  T* sA = reinterpret_cast<T*>(smem + L.A);
  T* sB = reinterpret_cast<T*>(smem + L.Bv);
  int* sJt = reinterpret_cast<int*>(smem + L.jt);
  double* gXi = reinterpret_cast<double*>(smem + L.gxi);
  double* gRad = reinterpret_cast<double*>(smem + L.grad);
  int* sCnt = reinterpret_cast<int*>(smem + L.cnt);
  const int pws = L.pws;
  const int nrad = S * S * R * K;
  // this block's partial gradients [Sa | S | S*S*R*K]; the moment part is
  // accumulated here directly (each thread owns the same coefficients for
  // every atom), species and radial parts in shared memory
  double* out = partials + static_cast<size_t>(blockIdx.x) * (md.Sa + S + nrad);
  const int4* mono_abc = reinterpret_cast<const int4*>(md.mono_abc);

  for (int x = tid; x < nrad; x += NT) {
    sRad[x] = static_cast<T>(md.radial[x]);
    gRad[x] = 0.0;
  }
  for (int x = tid; x < md.Sa; x += NT) out[x] = 0.0;
  for (int x = tid; x < S; x += NT) gXi[x] = 0.0;
  for (int x = tid; x < md.nzero; x += NT) V[md.v_m + md.zero_list[x]] = Dual2<T>::make(T(0), T(0));
  if (tid == 0) {
    V[md.v_zero] = Dual2<T>::make(T(0), T(0));
    V[md.v_one] = Dual2<T>::make(T(1), T(0));
  }
  const T rmax = static_cast<T>(md.rmax);
  const T inv_range = static_cast<T>(1.0 / (md.rmax - md.rmin));
  const T rsum = static_cast<T>(md.rmin + md.rmax);
  const T scal = static_cast<T>(md.scaling);
  __syncthreads();

  for (int atom = blockIdx.x; atom < io.natoms; atom += gridDim.x) {
    int it = __ldg(io.itypes + atom);
    if (it < 0 || it >= S) {
      if (tid == 0) atomicOr(io.err, kErrSpecies);
      it = 0;
    }
    int cfg = __ldg(io.cfg + atom);
    if (cfg < 0 || cfg >= io.nconfig) {
      if (tid == 0) atomicOr(io.err, kErrCapacity);
      cfg = 0;
    }
    const T a_i = static_cast<T>(__ldg(io.gE + cfg));
    // C maps r onto the stress-loss direction: sum_v gS_v sigma_v = sum_s (C r_s) . g_s
    const double iv = 1.0 / __ldg(io.volumes + cfg);
    const double* gs = io.gS + 6 * cfg;
    const T c00 = static_cast<T>(gs[0] * iv), c11 = static_cast<T>(gs[1] * iv), c22 = static_cast<T>(gs[2] * iv);
    const T c12 = static_cast<T>(0.5 * gs[3] * iv), c02 = static_cast<T>(0.5 * gs[4] * iv);
    const T c01 = static_cast<T>(0.5 * gs[5] * iv);
    const T gfx = static_cast<T>(__ldg(io.gF + 3 * atom)), gfy = static_cast<T>(__ldg(io.gF + 3 * atom + 1)),
            gfz = static_cast<T>(__ldg(io.gF + 3 * atom + 2));
    int cnt = io.counts ? __ldg(io.counts + atom) : io.nbr_stride;
    if (cnt > n_pad || cnt < 0) {
      if (tid == 0) atomicOr(io.err, kErrCapacity);
      cnt = cnt < 0 ? 0 : n_pad;
    }
    const size_t row = static_cast<size_t>(atom) * io.nbr_stride;

    // ---- N1: stage neighbours with their tangents -------------------------
    int nv = 0;
    for (int s0 = 0; s0 < io.nbr_stride; s0 += NT) {
      const int s = s0 + tid;
      bool valid = false;
      T rx = T(0), ry = T(0), rz = T(0), d = T(0);
      int jt = -1, j = -1;
      if (s < cnt) {
        jt = __ldg(io.jtypes + row + s);
        j = __ldg(io.js + row + s);
        rx = static_cast<T>(__ldg(io.rijs + 3 * (row + s)));
        ry = static_cast<T>(__ldg(io.rijs + 3 * (row + s) + 1));
        rz = static_cast<T>(__ldg(io.rijs + 3 * (row + s) + 2));
        if (jt >= S) {
          atomicOr(io.err, kErrSpecies);
          jt = -1;
        }
        const T r2 = rx * rx + ry * ry + rz * rz;
        d = dev_sqrt(r2);
        valid = (jt >= 0) && (r2 > T(0)) && (d < rmax);
      }
      const unsigned bal = __ballot_sync(0xffffffffu, valid);
      const int w = tid >> 5, l = tid & 31;
      if (l == 0) sCnt[w] = __popc(bal);
      __syncthreads();
      if (tid == 0) {
        int acc = 0;
        for (int i = 0; i < (NT >> 5); ++i) {
          int c = sCnt[i];
          sCnt[i] = acc;
          acc += c;
        }
        sCnt[NT >> 5] = acc;
      }
      __syncthreads();
      if (valid) {
        const int q = nv + sCnt[w] + __popc(bal & ((1u << l) - 1u));
        const T inv_d = T(1) / d;
        const T ux = rx * inv_d, uy = ry * inv_d, uz = rz * inv_d;
        // direction of the neighbour vector: force part + stress part
        T drx = gfx, dry = gfy, drz = gfz;
        if (j >= 0 && j < io.natoms) {
          drx -= static_cast<T>(__ldg(io.gF + 3 * j));
          dry -= static_cast<T>(__ldg(io.gF + 3 * j + 1));
          drz -= static_cast<T>(__ldg(io.gF + 3 * j + 2));
        }
        drx += c00 * rx + c01 * ry + c02 * rz;
        dry += c01 * rx + c11 * ry + c12 * rz;
        drz += c02 * rx + c12 * ry + c22 * rz;
        const T dd = ux * drx + uy * dry + uz * drz;
        sU[4 * q] = ux;
        sU[4 * q + 1] = uy;
        sU[4 * q + 2] = uz;
        sU[4 * q + 3] = d;
        sDu[4 * q] = (drx - ux * dd) * inv_d;
        sDu[4 * q + 1] = (dry - uy * dd) * inv_d;
        sDu[4 * q + 2] = (drz - uz * dd) * inv_d;
        sDu[4 * q + 3] = dd;
        sJt[q] = jt;
        const T x = (T(2) * d - rsum) * inv_range;
        const T dxdd = T(2) * inv_range;
        const T gap = rmax - d;
        const T smooth = gap * gap;
        const T* c = sRad + (static_cast<size_t>(it) * S + jt) * R * K;
        T base[kMaxR], dbase[kMaxR];
#pragma unroll
        for (int mu = 0; mu < kMaxR; ++mu) {
          base[mu] = T(0);
          dbase[mu] = T(0);
        }
        T t_prev = T(0), t_cur = T(1), dt_prev = T(0), dt_cur = T(0);
        for (int n = 0; n < K; ++n) {
          sPhi[q * K + n] = scal * smooth * t_cur;
          sPhip[q * K + n] = scal * (T(-2) * gap * t_cur + smooth * dt_cur * dxdd);
#pragma unroll
          for (int mu = 0; mu < kMaxR; ++mu) {
            if (mu < R) {
              base[mu] = dev_fma(c[mu * K + n], t_cur, base[mu]);
              dbase[mu] = dev_fma(c[mu * K + n], dt_cur, dbase[mu]);
            }
          }
          T t_next, dt_next;
          if (n == 0) {
            t_next = x;
            dt_next = T(1);
          } else {
            t_next = T(2) * x * t_cur - t_prev;
            dt_next = T(2) * t_cur + T(2) * x * dt_cur - dt_prev;
          }
          t_prev = t_cur;
          t_cur = t_next;
          dt_prev = dt_cur;
          dt_cur = dt_next;
        }
#pragma unroll
        for (int mu = 0; mu < kMaxR; ++mu) {
          if (mu < R) {
            sF[q * R + mu] = scal * smooth * base[mu];
            sFp[q * R + mu] = scal * (T(-2) * gap * base[mu] + smooth * dbase[mu] * dxdd);
          }
        }
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
      nv += sCnt[NT >> 5];
      __syncthreads();
    }

    // ---- N2: basic moments and their tangents ------------------------------
    for (int p = tid; p < P; p += NT) {
      const int4 abc = __ldg(mono_abc + p);
      const int a = abc.x, b = abc.y, cc = abc.z;
      const T am = static_cast<T>(a), bm = static_cast<T>(b), cm = static_cast<T>(cc);
      T acc[kMaxR], tac[kMaxR];
#pragma unroll
      for (int mu = 0; mu < kMaxR; ++mu) {
        acc[mu] = T(0);
        tac[mu] = T(0);
      }
      for (int q = 0; q < nv; ++q) {
        const T* pw = sPw + q * pws;
        const T px = pw[a], py = pw[D1 + b], pz = pw[2 * D1 + cc];
        const T mono = px * py * pz;
        const T* du = sDu + 4 * q;
        const T dmono = am * pw[a > 0 ? a - 1 : 0] * py * pz * du[0] +
                        bm * px * pw[D1 + (b > 0 ? b - 1 : 0)] * pz * du[1] +
                        cm * px * py * pw[2 * D1 + (cc > 0 ? cc - 1 : 0)] * du[2];
        const T dmd = du[3] * mono;
#pragma unroll
        for (int mu = 0; mu < kMaxR; ++mu) {
          if (mu < R) {
            const T f = sF[q * R + mu];
            acc[mu] = dev_fma(f, mono, acc[mu]);
            tac[mu] = dev_fma(sFp[q * R + mu], dmd, dev_fma(f, dmono, tac[mu]));
          }
        }
      }
#pragma unroll
      for (int mu = 0; mu < kMaxR; ++mu) {
        if (mu < R) {
          const int k = __ldg(md.mono_k + kMaxR * p + mu);
          if (k >= 0) V[md.v_m + k] = Dual2<T>::make(acc[mu], tac[mu]);
        }
      }
    }
    for (int x = tid; x < md.M; x += NT) V[md.v_dm + x] = Dual2<T>::make(T(0), T(0));
    __syncthreads();
    for (int x = tid; x < md.nseed; x += NT) {
      const T sv = static_cast<T>(md.seed_val[x]);
      V[md.v_dm + md.seed_idx[x]] = Dual2<T>::make(a_i * sv, sv);
    }

    // ---- dual forward tree --------------------------------------------------
    for (int ps = 0; ps < md.nfwd; ++ps) {
      DualFwdBody<T> body{V, V, T(0), T(0)};
      stream_entries_n<kStreamDepth, kVGlobal>(md.entries + md.fwd[ps].offset,
                                               __shfl_sync(0xFFFFFFFFu, my_wsteps, ps), NT, tid, body);
      __syncthreads();
    }
    for (int a = tid; a < md.Sa; a += NT) {
      const T2 v = V[md.v_m + __ldg(md.mapping + a)];
      out[a] += static_cast<double>(a_i) * static_cast<double>(v.x) + static_cast<double>(v.y);
    }
    if (tid == 0) gXi[it] += static_cast<double>(a_i);

    // ---- dual reverse tree ---------------------------------------------------
    for (int ps = 0; ps < md.nrev; ++ps) {
      DualRevBody<T> body{V, V, T(0), T(0)};
      stream_entries_n<kStreamDepth, kVGlobal>(md.entries + md.rev[ps].offset,
                                               __shfl_sync(0xFFFFFFFFu, my_wsteps, md.nfwd + ps), NT, tid, body);
      __syncthreads();
    }

    // ---- N3: per-neighbour radial sensitivities ------------------------------
    {
      int tpn = 32;
      while (tpn > 1 && tpn * nv > NT) tpn >>= 1;
      const int total = nv * tpn;
      for (int base = 0; base < total; base += NT) {
        const int idx = base + tid;
        const bool active = idx < total;
        const int q = active ? idx / tpn : 0;
        const int sl = idx & (tpn - 1);
        T GA[kMaxR], GB[kMaxR];
#pragma unroll
        for (int mu = 0; mu < kMaxR; ++mu) {
          GA[mu] = T(0);
          GB[mu] = T(0);
        }
        if (active) {
          const T* pw = sPw + q * pws;
          const T* du = sDu + 4 * q;
          for (int p = sl; p < P; p += tpn) {
            const int4 abc = __ldg(mono_abc + p);
            const int a = abc.x, b = abc.y, cc = abc.z;
            const T px = pw[a], py = pw[D1 + b], pz = pw[2 * D1 + cc];
            const T mono = px * py * pz;
            const T dmono = static_cast<T>(a) * pw[a > 0 ? a - 1 : 0] * py * pz * du[0] +
                            static_cast<T>(b) * px * pw[D1 + (b > 0 ? b - 1 : 0)] * pz * du[1] +
                            static_cast<T>(cc) * px * py * pw[2 * D1 + (cc > 0 ? cc - 1 : 0)] * du[2];
#pragma unroll
            for (int mu = 0; mu < kMaxR; ++mu) {
              if (mu < R) {
                const int k = __ldg(md.mono_k + kMaxR * p + mu);
                if (k >= 0) {
                  const T2 lt = V[md.v_dm + __ldg(md.dm_pos + k)];   // (lambda, tau)
                  GA[mu] = dev_fma(lt.x, mono, dev_fma(lt.y, dmono, GA[mu]));
                  GB[mu] = dev_fma(lt.y, mono, GB[mu]);
                }
              }
            }
          }
        }
        for (int o = tpn >> 1; o > 0; o >>= 1) {
#pragma unroll
          for (int mu = 0; mu < kMaxR; ++mu) {
            GA[mu] += __shfl_xor_sync(0xffffffffu, GA[mu], o);
            GB[mu] += __shfl_xor_sync(0xffffffffu, GB[mu], o);
          }
        }
        if (active && sl == 0) {
          const T dd = sDu[4 * q + 3];
#pragma unroll
          for (int mu = 0; mu < kMaxR; ++mu) {
            if (mu < R) {
              sA[q * R + mu] = GA[mu];
              sB[q * R + mu] = dd * GB[mu];
            }
          }
        }
      }
    }
    __syncthreads();
    // ---- N4: radial coefficient gradient, one thread per (mu, n) -------------
    for (int x = tid; x < R * K; x += NT) {
      const int mu = x / K, n = x % K;
      for (int q = 0; q < nv; ++q) {
        const double g = static_cast<double>(sA[q * R + mu]) * static_cast<double>(sPhi[q * K + n]) +
                         static_cast<double>(sB[q * R + mu]) * static_cast<double>(sPhip[q * K + n]);
        gRad[((it * S + sJt[q]) * R + mu) * K + n] += g;
      }
    }
    __syncthreads();
  }
  // per-block partials: [Sa | S | S*S*R*K] (the moment part is already there)
  for (int x = tid; x < S; x += NT) out[md.Sa + x] = gXi[x];
  for (int x = tid; x < nrad; x += NT) out[md.Sa + S + x] = gRad[x];
}

__global__ void k_adjoint_reduce(int nblocks, int Sa, int S, int nrad, const double* __restrict__ partials,
                                 double* __restrict__ gmoment, double* __restrict__ gspecies,
                                 double* __restrict__ gradial) {
  const int np = Sa + S + nrad;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= np) return;
  double s = 0.0;
  for (int b = 0; b < nblocks; ++b) s += partials[static_cast<size_t>(b) * np + x];
  if (x < Sa) gmoment[x] = s;
  else if (x < Sa + S) gspecies[x - Sa] = s;
  else gradial[x - Sa - S] = s;
}

void train_free(TrainWorkspace& w) {
  if (w.partials) cudaFree(w.partials);
  if (w.vscratch) cudaFree(w.vscratch);
  w = TrainWorkspace();
}

template <bool G>
static cudaError_t adjoint_smem_limit(size_t bytes) {
  static size_t granted = 0;
  if (bytes <= granted) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(k_mtp_adjoint<double, G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(bytes));
  if (e == cudaSuccess) granted = bytes;
  return e;
}

template <bool G>
static int adjoint_occupancy(size_t bytes, int threads) {
  if (bytes > 227 * 1024) return 0;
  int nb = 0;
  if (adjoint_smem_limit<G>(bytes) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_mtp_adjoint<double, G>, threads, bytes) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return nb;
}

bool adjoint_fits_shared(const DevModel& md, int n_pad, int threads) {
  const TrainSmem L = train_layout<double>(md.v_size, md.S, md.R, md.K, md.P, md.D, md.Sa, n_pad, threads);
  return adjoint_occupancy<false>(L.total, threads) > 0;
}

cudaError_t launch_adjoint(const DevModel& md, const TrainIO& io, int threads, int sm_count, TrainWorkspace& ws,
                           double* gspecies, double* gmoment, double* gradial, cudaStream_t st, std::string& err) {
  const int n_pad = io.nbr_stride;
  const int nrad = md.S * md.S * md.R * md.K;
  const int np = md.Sa + md.S + nrad;
  bool vglobal = false;
  TrainSmem L = train_layout<double>(md.v_size, md.S, md.R, md.K, md.P, md.D, md.Sa, n_pad, threads);
  int bps = adjoint_occupancy<false>(L.total, threads);
  if (bps <= 0) {
    vglobal = true;
    L = train_layout<double>(0, md.S, md.R, md.K, md.P, md.D, md.Sa, n_pad, threads);
    bps = adjoint_occupancy<true>(L.total, threads);
  }
  if (bps <= 0) {
    err = "the adjoint block does not fit in shared memory for this basis and nbr_stride";
    return cudaSuccess;
  }
  int blocks = std::max(1, std::min(io.natoms, bps * sm_count));
  if (vglobal) {
    // the blocks' global value spaces should stay resident in L2: cap their
    // total at 5/8 of it (but keep one block per SM)
    int dev = 0, l2 = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev);
    const size_t per = static_cast<size_t>(2) * md.v_size * sizeof(double);
    const int cap = static_cast<int>(std::max<size_t>(sm_count, (static_cast<size_t>(l2) * 5 / 8) / per));
    blocks = std::max(1, std::min(blocks, cap));
  }
  const size_t need_p = static_cast<size_t>(blocks) * np;
  if (need_p > ws.partials_cap) {
    if (ws.partials) cudaFree(ws.partials);
    ws.partials = nullptr;
    cudaError_t e = cudaMalloc(&ws.partials, need_p * sizeof(double));
    if (e != cudaSuccess) return e;
    ws.partials_cap = need_p;
  }
  if (vglobal) {
    const size_t need_v = static_cast<size_t>(blocks) * 2 * md.v_size * sizeof(double);
    if (need_v > ws.vscratch_cap) {
      if (ws.vscratch) cudaFree(ws.vscratch);
      ws.vscratch = nullptr;
      cudaError_t e = cudaMalloc(&ws.vscratch, need_v);
      if (e != cudaSuccess) return e;
      ws.vscratch_cap = need_v;
    }
  }
  if (io.natoms > 0) {
    if (vglobal)
      k_mtp_adjoint<double, true><<<blocks, threads, L.total, st>>>(md, io, n_pad, ws.vscratch, ws.partials);
    else
      k_mtp_adjoint<double, false><<<blocks, threads, L.total, st>>>(md, io, n_pad, ws.vscratch, ws.partials);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_adjoint_reduce<<<(np + 255) / 256, 256, 0, st>>>(blocks, md.Sa, md.S, nrad, ws.partials, gmoment, gspecies,
                                                      gradial);
  } else {
    cudaMemsetAsync(gmoment, 0, md.Sa * sizeof(double), st);
    cudaMemsetAsync(gspecies, 0, md.S * sizeof(double), st);
    cudaMemsetAsync(gradial, 0, nrad * sizeof(double), st);
  }
  return cudaGetLastError();
}

}  // namespace mtp
