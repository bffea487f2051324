// ctc_esp.cu -- molecular electrostatic potential from Hermite pair densities.
//
// The reference builds all M(M+1)/2 point-charge integrals V_{mu nu}(C) per
// point with the McMurchie-Davidson E and R recursions (Helgaker 9.5.6-7,
// 9.9.18-20; include/integral_coeffs.cuh:17-238, src/evaluate_electrostatic.cu:
// 16-10158) and then contracts them with D in a serial host loop of cublasDtpttr,
// cublasDsymm, a Hadamard product and thrust::reduce per point
// (src/evaluate_electrostatic.cu:10319-10344).  Since
//     sum_{mu nu} D_{mu nu} V_{mu nu}(C)
//        = sum_{pairs ab} (2 pi / p) sum_{tuv} h^{ab}_{tuv} R_{tuv}(p, P - C),
//     h^{ab}_{tuv} = sum_{mu in a, nu in b} D_{mu nu} c_mu c_nu E^x_t E^y_u E^z_v
// depends on the point only through R, the Hermite densities h are built once
// per molecule (host, all cores) and each point costs one Boys evaluation and
// one R recursion per significant primitive pair -- no integral matrix.
// Pairs are grouped by L = l_a + l_b; each class runs as its own kernel
// (registers sized for its L), over a 2-D grid of 128-point blocks x slices
// of the class's pairs.
//
// Boys function F_n(T) (FP64): beyond a per-L threshold (T >= 38 + 3L, where
// the neglected e^{-T} terms are below 2e-17 relative) the asymptotic forms
// hold -- a far pair is a point multipole and costs one rsqrt and no
// exponential; 99% of (point, pair) evaluations on molecular surfaces are of
// this kind.  Below it, a 7-term Taylor expansion about the nearest point of
// a 0.05-spaced table gives F_L, and F_{n-1} = (2T F_n + e^{-T})/(2n-1)
// (downward recursion, stable) gives the rest.  The table is built at set-up
// from the series F_m(T) = e^{-T} sum_i (2T)^i / ((2m+1)(2m+3)...(2m+2i+1)).
// (The reference uses forward recursion from erf, include/boys_functions.cuh:13-31,
// which loses digits at small T and divides by zero at T = 0.)
//
// V(C) = sum_A Z_A / |C - R_A| - electronic part (src/evaluate_electrostatic.cu:10357-10369).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "ctc_internal.h"

#define CTC_TERMS_HOST
#include "ctc_terms.inc"
#undef CTC_TERMS_HOST

namespace ctc {

namespace {

constexpr int kLmax = 8;                 // g x g
constexpr int kTaylor = 7;               // terms of the Taylor expansion
constexpr int kNF = kLmax + kTaylor;     // orders stored per table point
constexpr double kTstep = 0.05;
constexpr double kTmax = 64.0;           // table range: above every far_T(L <= 8)
constexpr int kNT = (int)(kTmax / kTstep) + 2;
constexpr double kPi = 3.14159265358979323846;

__host__ __device__ constexpr int ntuv(int L) { return (L + 1) * (L + 2) * (L + 3) / 6; }
// index of (t,u,v): totals ascending; within a total s, t descending then u descending
__host__ __device__ constexpr int tuv_index(int t, int u, int v) {
  int s = t + u + v;
  int base = s * (s + 1) * (s + 2) / 6;
  int before = 0;
  for (int tt = s; tt > t; --tt) before += s - tt + 1;
  return base + before + (s - t - u);
}

struct EspPair {
  double Px, Py, Pz, p;
  double f0c;  // sqrt(pi / p) / 2: F_0 = f0c / |P - C| in the far field
  double pad;
};
struct EspBatch {
  int32_t b0, b1;   // pairs [b0, b1)
  int32_t h0;       // first Hermite coefficient
  int32_t L;
};

double boys_series(int m, double T) {
  double term = 1.0 / (2 * m + 1), sum = term;
  for (int i = 1; i < 1000; ++i) {
    term *= 2.0 * T / (2 * m + 2 * i + 1);
    sum += term;
    if (term < 1e-18 * sum) break;
  }
  return std::exp(-T) * sum;
}

}  // namespace

// pairs per batch of class L: up to 256, with the batch's Hermite
// coefficients within 32 KB (one barrier pair per batch in the class kernels)
constexpr int kBatchPairs = 256;
constexpr int kBatchH = 4096;
__host__ __device__ constexpr int batch_pairs(int L) {
  return kBatchPairs < kBatchH / ntuv(L) ? kBatchPairs : kBatchH / ntuv(L);
}

struct EspTables {
  double* d_boys = nullptr;
  EspPair* d_pairs = nullptr;
  double* d_h = nullptr;
  EspBatch* d_batches = nullptr;
  double* d_atoms = nullptr;  // x y z Z per atom
  int npairs = 0, nbatch = 0, natom = 0;
  int lb0[kLmax + 2] = {};  // batches of class L: [lb0[L], lb0[L + 1])
  size_t nh = 0;
  // algorithmic FP64 work per point: sum over the kept pairs of
  // 2 n_tuv(L) (contraction) + 2 n_R(L) (R recursion) + 10 (L + 1) (Boys)
  double flops_per_point = 0.0;
  double mean_L = 0.0;
};

namespace {

// ------------------------------------------------------------------ device side
// First T from which the asymptotic forms F_0 = sqrt(pi/T)/2, F_n =
// (2n-1)/(2T) F_{n-1} agree with F_n(T) to 2e-17 relative for every n <= L
// (the neglected terms are e^{-T} and erfc(sqrt T); thresholds checked against
// the incomplete-gamma form of F_n in 40-digit arithmetic: 37, 41, 44, 47, 50,
// 53, 55, 58, 60 for L = 0..8).
__host__ __device__ constexpr double far_T(int L) { return 38.0 + 3.0 * L; }

// G_n = R^n_000 = (-2p)^n F_n(T), n = 0..L, at T = p r2.
//  far field (T >= far_T(L)): the p dependence cancels except in F_0,
//    G_0 = (sqrt(pi/p)/2) / r,  G_n = -(2n-1) G_{n-1} / r2  -- no exponential;
//  otherwise: F_L from the 7-term Taylor table about the nearest 0.05 step,
//    F_{n-1} = (2T F_n + e^{-T}) / (2n-1) downwards (stable for every T).
template <int L>
__device__ __forceinline__ void boys_g(double p, double f0c, double r2, const double* __restrict__ tab,
                                       double* G) {
  const double T = p * r2;
  if (T >= far_T(L)) {
    const double ri = rsqrt(r2);
    const double ri2 = ri * ri;
    G[0] = f0c * ri;
#pragma unroll
    for (int n = 1; n <= L; ++n) G[n] = -(double)(2 * n - 1) * ri2 * G[n - 1];
  } else {
    const double e = exp(-T);
    const int i = __double2int_rn(T * (1.0 / kTstep));
    const double d = i * kTstep - T;  // -(T - T_i)
    const double* row = tab + i * kNF + L;
    double F[L + 1];
    double fl = row[kTaylor - 1];
#pragma unroll
    for (int k = kTaylor - 2; k >= 0; --k) fl = row[k] + fl * d * (1.0 / (double)(k + 1));
    F[L] = fl;
#pragma unroll
    for (int n = L; n > 0; --n) F[n - 1] = (2.0 * T * F[n] + e) * (1.0 / (double)(2 * n - 1));
    double m = 1.0;
#pragma unroll
    for (int n = 0; n <= L; ++n) {
      G[n] = m * F[n];
      m *= -2.0 * p;
    }
  }
}

// R^0_{tuv}(p, X, Y, Z) for t+u+v <= L, in place from level L down to 0,
// from G_n = R^n_000.
template <int L>
__device__ __forceinline__ void hermite_r(double X, double Y, double Z, const double* G, double* R) {
  R[0] = G[L];
#pragma unroll
  for (int n = L - 1; n >= 0; --n) {
    // level n: totals L-n down to 1 from level n+1, then total 0
#pragma unroll
    for (int s = L - n; s >= 1; --s) {
#pragma unroll
      for (int t = s; t >= 0; --t) {
#pragma unroll
        for (int u = s - t; u >= 0; --u) {
          const int v = s - t - u;
          double r;
          if (t > 0) {
            r = X * R[tuv_index(t - 1, u, v)];
            if (t > 1) r += (t - 1) * R[tuv_index(t - 2, u, v)];
          } else if (u > 0) {
            r = Y * R[tuv_index(t, u - 1, v)];
            if (u > 1) r += (u - 1) * R[tuv_index(t, u - 2, v)];
          } else {
            r = Z * R[tuv_index(t, u, v - 1)];
            if (v > 1) r += (v - 1) * R[tuv_index(t, u, v - 2)];
          }
          R[tuv_index(t, u, v)] = r;
        }
      }
    }
    R[0] = G[n];
  }
}

constexpr int kEspThreads = 128;

// Electronic ESP of the pairs of one angular class L: block (x, y) takes 128
// points and slice y of the class's batches and writes its partial sum
// sum_pairs sum_tuv h_tuv R_tuv (h already carries 2 pi / p) to row y of
// part.  Rows are summed in a fixed order by esp_finish_kernel, so results do
// not depend on the launch shape's timing.
template <int L>
__global__ void __launch_bounds__(kEspThreads)
    esp_class_kernel(const EspPair* __restrict__ pairs, const double* __restrict__ hbuf,
                     const EspBatch* __restrict__ batches, int b0, int nb, const double* __restrict__ tab,
                     const double* __restrict__ pts, int64_t n, double* __restrict__ part) {
  constexpr int NT = ntuv(L);
  constexpr int BP = batch_pairs(L);
  constexpr bool PAIRS2 = L <= 4;  // registers stay below ~170 up to L = 4
  __shared__ EspPair sp[BP];
  __shared__ double sh[BP * NT];
  const int slices = gridDim.y, y = blockIdx.y;
  const int bb = b0 + (int)((int64_t)nb * y / slices), be = b0 + (int)((int64_t)nb * (y + 1) / slices);
  const int64_t ip = (int64_t)blockIdx.x * kEspThreads + threadIdx.x;
  const bool live = ip < n;
  double cx = 0, cy = 0, cz = 0;
  if (live) {
    cx = pts[3 * ip];
    cy = pts[3 * ip + 1];
    cz = pts[3 * ip + 2];
  }
  double acc = 0.0;
  for (int b = bb; b < be; ++b) {
    const EspBatch bt = batches[b];
    const int np = bt.b1 - bt.b0;
    __syncthreads();
    for (int i = threadIdx.x; i < np; i += kEspThreads) sp[i] = pairs[bt.b0 + i];
    for (int i = threadIdx.x; i < np * NT; i += kEspThreads) sh[i] = hbuf[bt.h0 + i];
    __syncthreads();
    if (!live) continue;
    auto pair_sum = [&](int i) -> double {
      const EspPair q = sp[i];
      const double X = q.Px - cx, Y = q.Py - cy, Z = q.Pz - cz;
      double G[L + 1];
      boys_g<L>(q.p, q.f0c, X * X + Y * Y + Z * Z, tab, G);
      double R[NT];
      hermite_r<L>(X, Y, Z, G, R);
      const double* h = sh + i * NT;
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < NT; ++k) s += h[k] * R[k];
      return s;
    };
    int i = 0;
    if (PAIRS2) {
      // two pairs per iteration: two independent dependency chains (Boys, R
      // recursion, dot product) for the FP64 pipe; added in pair order
      for (; i + 1 < np; i += 2) {
        const double s0 = pair_sum(i), s1 = pair_sum(i + 1);
        acc += s0;
        acc += s1;
      }
    }
    for (; i < np; ++i) acc += pair_sum(i);
  }
  if (live) part[(int64_t)y * n + ip] = acc;
}

// V = sum_A Z_A / |C - R_A| - (sum of the rows of part, in row order).
__global__ void __launch_bounds__(256)
    esp_finish_kernel(const double* __restrict__ part, int rows, const double* __restrict__ atoms, int natom,
                      const double* __restrict__ pts, int64_t n, double* __restrict__ out) {
  const int64_t ip = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ip >= n) return;
  const double cx = pts[3 * ip], cy = pts[3 * ip + 1], cz = pts[3 * ip + 2];
  double elec = 0.0;
  for (int r = 0; r < rows; ++r) elec += part[(int64_t)r * n + ip];
  double nuc = 0.0;
  for (int a = 0; a < natom; ++a) {
    const double dx = cx - atoms[4 * a], dy = cy - atoms[4 * a + 1], dz = cz - atoms[4 * a + 2];
    nuc += atoms[4 * a + 3] / sqrt(dx * dx + dy * dy + dz * dz);
  }
  out[ip] = nuc - elec;
}

// ------------------------------------------------------------------ host side
void hermite_e(int la, int lb, double a, double b, double XAB, std::vector<double>& E) {
  const int L = la + lb;
  const double p = a + b, mu = a * b / p;
  const double XPA = -(b / p) * XAB, XPB = (a / p) * XAB;
  E.assign((size_t)(la + 1) * (lb + 1) * (L + 1), 0.0);
  auto at = [&](int i, int j, int t) -> double& { return E[((size_t)i * (lb + 1) + j) * (L + 1) + t]; };
  at(0, 0, 0) = std::exp(-mu * XAB * XAB);
  for (int i = 0; i <= la; ++i)
    for (int j = 0; j <= lb; ++j) {
      if (i == 0 && j == 0) continue;
      for (int t = 0; t <= i + j; ++t) {
        if (j == 0) {
          double em = t >= 1 ? at(i - 1, 0, t - 1) : 0.0;
          double e0 = t <= i - 1 ? at(i - 1, 0, t) : 0.0;
          double ep = t + 1 <= i - 1 ? at(i - 1, 0, t + 1) : 0.0;
          at(i, j, t) = em / (2 * p) + XPA * e0 + (t + 1) * ep;
        } else {
          double em = t >= 1 ? at(i, j - 1, t - 1) : 0.0;
          double e0 = t <= i + j - 1 ? at(i, j - 1, t) : 0.0;
          double ep = t + 1 <= i + j - 1 ? at(i, j - 1, t + 1) : 0.0;
          at(i, j, t) = em / (2 * p) + XPB * e0 + (t + 1) * ep;
        }
      }
    }
}

struct Mono { int a, b, c; };

// Cartesian monomials of degree l and the component -> monomial coefficient matrix.
void seg_monomials(int type, std::vector<Mono>& monos, std::vector<double>& Tm /*ncomp x nmono*/) {
  const int l = l_of_type(type), nc = ncomp_of_type(type);
  monos.clear();
  for (int a = l; a >= 0; --a)
    for (int b = l - a; b >= 0; --b) monos.push_back({a, b, l - a - b});
  Tm.assign((size_t)nc * monos.size(), 0.0);
  for (int j = 0; j < nc; ++j)
    for (int t = h_comp_off[type][j]; t < h_comp_off[type][j + 1]; ++t) {
      const Term& T = h_terms[t];
      for (size_t m = 0; m < monos.size(); ++m)
        if (monos[m].a == T.a && monos[m].b == T.b && monos[m].c == T.z) Tm[j * monos.size() + m] += T.c;
    }
}

struct PairOut {
  int L;
  double bound;  // upper bound of |pair contribution| at any point
  EspPair pr;
  std::vector<double> h;
};

// Upper bound of |R^0_tuv(p, X)| over all points for t + u + v = s, used to
// bound a pair's contribution: (2p)^(s/2) times a generous constant in s.
inline double r_bound(double p, int s) { return std::pow(2.0 * p + 1.0, 0.5 * s) * std::pow(3.0, s); }

}  // namespace

void destroy_esp(ctc_molecule* mol) {
  if (!mol->esp) return;
  cudaFree(mol->esp->d_boys);
  cudaFree(mol->esp->d_pairs);
  cudaFree(mol->esp->d_h);
  cudaFree(mol->esp->d_batches);
  cudaFree(mol->esp->d_atoms);
  delete mol->esp;
  mol->esp = nullptr;
  mol->esp_valid = false;
}

static int build_esp(ctc_molecule* mol) {
  destroy_esp(mol);
  if (int rc = refresh_host_density(mol); rc != CTC_OK) return rc;
  for (const DevSeg& s : mol->segs)
    if (s.l > 4) return fail(CTC_ERR_UNSUPPORTED, "ESP: angular momentum above g");
  const int nseg = mol->nseg, M = mol->M;
  // per-segment monomial data
  std::vector<std::vector<Mono>> monos(nseg);
  std::vector<std::vector<double>> Tm(nseg);
  for (int s = 0; s < nseg; ++s) seg_monomials(mol->segs[s].type, monos[s], Tm[s]);
  const double eps = 1e-22;            // pre-filter before the Hermite densities are formed
  const double budget = 1e-11;         // total |ESP| error allowed for the pairs dropped below
  unsigned nthr = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
  std::vector<std::vector<PairOut>> outs(nthr);
  auto worker = [&](unsigned tid) {
    std::vector<double> Ex, Ey, Ez, Dc;
    for (int I = (int)tid; I < nseg; I += (int)nthr) {
      const DevSeg& A = mol->segs[I];
      const int nA = ncomp_of_type(A.type), mA = (int)monos[I].size();
      for (int J = I; J < nseg; ++J) {
        const DevSeg& B = mol->segs[J];
        const int nB = ncomp_of_type(B.type), mB = (int)monos[J].size();
        const double fac = (I == J) ? 1.0 : 2.0;
        // Cartesian-monomial density Dc = Tm_A^T D_AB Tm_B
        Dc.assign((size_t)mA * mB, 0.0);
        double dmax = 0.0;
        for (int i = 0; i < nA; ++i)
          for (int j = 0; j < nB; ++j) {
            const double d = mol->D[(size_t)(A.ao0 + i) * M + (B.ao0 + j)];
            if (d == 0.0) continue;
            for (int ma = 0; ma < mA; ++ma) {
              const double ta = Tm[I][(size_t)i * mA + ma];
              if (ta == 0.0) continue;
              for (int mb = 0; mb < mB; ++mb) Dc[(size_t)ma * mB + mb] += d * ta * Tm[J][(size_t)j * mB + mb];
            }
          }
        for (double v : Dc) dmax = std::max(dmax, std::fabs(v));
        if (dmax == 0.0) continue;
        const int L = A.l + B.l, NT = ntuv(L);
        const double XAB = A.cx - B.cx, YAB = A.cy - B.cy, ZAB = A.cz - B.cz;
        const double R2 = XAB * XAB + YAB * YAB + ZAB * ZAB;
        for (int ka = 0; ka < A.nprim; ++ka) {
          const double a = mol->alpha[A.prim0 + ka], ca = mol->coef[A.prim0 + ka];
          for (int kb = 0; kb < B.nprim; ++kb) {
            const double b = mol->alpha[B.prim0 + kb], cb = mol->coef[B.prim0 + kb];
            const double p = a + b, mu = a * b / p;
            const double K = std::exp(-mu * R2);
            const double pref = 2.0 * kPi / p;
            const double scale = fac * ca * cb;
            // bound on |h| * |R| (|R_tuv| <= (2p)^(s/2) * s!! F-like factors)
            const double bound = std::fabs(scale) * K * dmax * pref * mA * mB *
                                 std::pow(1.0 + 2.0 * p, 0.5 * L) * std::pow(2.0, L);
            if (bound < eps) continue;
            hermite_e(A.l, B.l, a, b, XAB, Ex);
            hermite_e(A.l, B.l, a, b, YAB, Ey);
            hermite_e(A.l, B.l, a, b, ZAB, Ez);
            PairOut po;
            po.L = L;
            po.pr = {(a * A.cx + b * B.cx) / p, (a * A.cy + b * B.cy) / p, (a * A.cz + b * B.cz) / p, p,
                     0.5 * std::sqrt(kPi / p), 0.0};
            po.h.assign(NT, 0.0);
            const int LB1 = B.l + 1, L1 = L + 1;
            for (int ma = 0; ma < mA; ++ma) {
              const Mono& u = monos[I][ma];
              for (int mb = 0; mb < mB; ++mb) {
                const double dc = Dc[(size_t)ma * mB + mb] * scale;
                if (dc == 0.0) continue;
                const Mono& w = monos[J][mb];
                for (int t = 0; t <= u.a + w.a; ++t) {
                  const double ex = Ex[((size_t)u.a * LB1 + w.a) * L1 + t] * dc;
                  for (int uu = 0; uu <= u.b + w.b; ++uu) {
                    const double exy = ex * Ey[((size_t)u.b * LB1 + w.b) * L1 + uu];
                    for (int v = 0; v <= u.c + w.c; ++v)
                      po.h[tuv_index(t, uu, v)] += exy * Ez[((size_t)u.c * LB1 + w.c) * L1 + v];
                  }
                }
              }
            }
            double bnd = 0.0;
            for (int tt = 0; tt <= L; ++tt)
              for (int uu = 0; uu <= L - tt; ++uu)
                for (int vv = 0; vv <= L - tt - uu; ++vv)
                  bnd += std::fabs(po.h[tuv_index(tt, uu, vv)]) * r_bound(p, tt + uu + vv);
            po.bound = bnd * pref;
            if (po.bound < eps) continue;
            for (double& v : po.h) v *= pref;  // the kernels sum h_tuv R_tuv with 2 pi / p folded in
            outs[tid].push_back(std::move(po));
          }
        }
      }
    }
  };
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nthr; ++t) th.emplace_back(worker, t);
  for (auto& t : th) t.join();
  // drop the weakest pairs while their summed bound stays within the budget:
  // pairs are ranked by (bound, thread, position) and exactly the accumulated
  // prefix is dropped, so ties at the cut never drop more than the budget
  {
    struct Ranked { double bound; uint32_t list, pos; };
    std::vector<Ranked> rk;
    for (uint32_t l = 0; l < outs.size(); ++l)
      for (uint32_t i = 0; i < outs[l].size(); ++i) rk.push_back({outs[l][i].bound, l, i});
    std::sort(rk.begin(), rk.end(), [](const Ranked& a, const Ranked& b) {
      return a.bound != b.bound ? a.bound < b.bound : (a.list != b.list ? a.list < b.list : a.pos < b.pos);
    });
    std::vector<std::vector<char>> drop(outs.size());
    for (size_t l = 0; l < outs.size(); ++l) drop[l].assign(outs[l].size(), 0);
    double acc = 0.0;
    for (const Ranked& r : rk) {
      if (acc + r.bound > budget) break;
      acc += r.bound;
      drop[r.list][r.pos] = 1;
    }
    for (size_t l = 0; l < outs.size(); ++l) {
      size_t w = 0;
      for (size_t i = 0; i < outs[l].size(); ++i) {
        if (drop[l][i]) continue;
        if (w != i) outs[l][w] = std::move(outs[l][i]);  // a self-move would empty h
        ++w;
      }
      outs[l].resize(w);
    }
  }
  // gather, sorted by L, into batches of equal L
  std::vector<EspPair> pairs;
  std::vector<double> hv;
  std::vector<EspBatch> batches;
  int lb0[kLmax + 2] = {};
  for (int L = 0; L <= kLmax; ++L) {
    const int per = batch_pairs(L);
    lb0[L] = (int)batches.size();
    int in_batch = 0;
    for (auto& o : outs)
      for (auto& po : o) {
        if (po.L != L) continue;
        if (in_batch == 0) batches.push_back({(int32_t)pairs.size(), (int32_t)pairs.size(), (int32_t)hv.size(), L});
        pairs.push_back(po.pr);
        hv.insert(hv.end(), po.h.begin(), po.h.end());
        batches.back().b1 = (int32_t)pairs.size();
        if (++in_batch == per) in_batch = 0;
      }
  }
  lb0[kLmax + 1] = (int)batches.size();
  if (hv.size() > (size_t)INT32_MAX) return fail(CTC_ERR_UNSUPPORTED, "ESP: too many pair coefficients");
  // Boys table
  std::vector<double> tab((size_t)kNT * kNF);
  for (int i = 0; i < kNT; ++i)
    for (int m = 0; m < kNF; ++m) tab[(size_t)i * kNF + m] = boys_series(m, i * kTstep);
  std::vector<double> atoms(4 * (size_t)std::max(mol->natom, 1));
  for (int a = 0; a < mol->natom; ++a) {
    atoms[4 * a] = mol->atom_xyz[3 * a];
    atoms[4 * a + 1] = mol->atom_xyz[3 * a + 1];
    atoms[4 * a + 2] = mol->atom_xyz[3 * a + 2];
    atoms[4 * a + 3] = mol->charges[a];
  }
  EspTables* e = new EspTables();
  mol->esp = e;
  for (const EspBatch& bt : batches) {
    int nR = 0;
    for (int j = 0; j <= bt.L; ++j) nR += ntuv(j);
    const int np = bt.b1 - bt.b0;
    e->flops_per_point += (double)np * (2.0 * ntuv(bt.L) + 2.0 * nR + 10.0 * (bt.L + 1));
    e->mean_L += (double)np * bt.L;
  }
  if (!pairs.empty()) e->mean_L /= (double)pairs.size();
  std::copy(lb0, lb0 + kLmax + 2, e->lb0);
  e->npairs = (int)pairs.size();
  e->nbatch = (int)batches.size();
  e->natom = mol->natom;
  e->nh = hv.size();
  auto up = [&](void** dst, const void* src, size_t bytes) -> int {
    if (bytes == 0) bytes = 8;
    CTC_CUDA_TRY(cudaMalloc(dst, bytes));
    if (src) CTC_CUDA_TRY(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
    return CTC_OK;
  };
  int rc;
  if ((rc = up((void**)&e->d_boys, tab.data(), tab.size() * sizeof(double))) ||
      (rc = up((void**)&e->d_pairs, pairs.empty() ? nullptr : pairs.data(), pairs.size() * sizeof(EspPair))) ||
      (rc = up((void**)&e->d_h, hv.empty() ? nullptr : hv.data(), hv.size() * sizeof(double))) ||
      (rc = up((void**)&e->d_batches, batches.empty() ? nullptr : batches.data(), batches.size() * sizeof(EspBatch))) ||
      (rc = up((void**)&e->d_atoms, atoms.data(), atoms.size() * sizeof(double)))) {
    destroy_esp(mol);
    return rc;
  }
  mol->esp_valid = true;
  if (std::getenv("CTC_LOG"))
    std::fprintf(stderr, "[ctc] esp tables: %d primitive pairs, %d batches, %zu Hermite coefficients\n",
                 e->npairs, e->nbatch, e->nh);
  return CTC_OK;
}

int esp_info(ctc_molecule* mol, double* info) {
  if (!mol->esp_valid) {
    int rc = build_esp(mol);
    if (rc != CTC_OK) return rc;
  }
  info[0] = mol->esp->npairs;
  info[1] = mol->esp->flops_per_point;
  info[2] = (double)mol->esp->nh;
  info[3] = mol->esp->mean_L;
  return CTC_OK;
}

int eval_esp(ctc_molecule* mol, const double* d_points, int64_t n, double* d_out, cudaStream_t st) {
  if (n < 0) return fail(CTC_ERR_INVALID, "eval_esp: negative point count");
  if (n == 0) return CTC_OK;
  if (!mol->esp_valid) {
    int rc = build_esp(mol);
    if (rc != CTC_OK) return rc;
  }
  const EspTables* e = mol->esp;
  int nsm = 148;
  if (int rc = device_sm_count(&nsm); rc != CTC_OK) return rc;
  // points per pass: bounds the partial-sum rows (rows x points x 8 B)
  constexpr int64_t kChunk = (int64_t)1 << 22;
  for (int64_t p0 = 0; p0 < n; p0 += kChunk) {
    const int64_t m = std::min(kChunk, n - p0);
    const int64_t gx = (m + kEspThreads - 1) / kEspThreads;
    // slices of each class's batches: about 8 blocks per SM in every class kernel
    int sl[kLmax + 1], rows = 0;
    for (int L = 0; L <= kLmax; ++L) {
      const int nb = e->lb0[L + 1] - e->lb0[L];
      const int64_t want = (8 * (int64_t)nsm + gx - 1) / gx;
      sl[L] = nb == 0 ? 0 : (int)std::max<int64_t>(1, std::min<int64_t>({want, (int64_t)nb, 65535}));
      rows += sl[L];
    }
    if (int rc = mol->ws_esp.ensure(sizeof(double) * std::max<int64_t>(1, (int64_t)rows * m), st); rc != CTC_OK)
      return rc;
    double* part = (double*)mol->ws_esp.p;
    const double* pts = d_points + 3 * p0;
    int r = 0;
    for (int L = 0; L <= kLmax; ++L) {
      if (!sl[L]) continue;
      const dim3 grid((unsigned)gx, (unsigned)sl[L]);
      const int b0 = e->lb0[L], nb = e->lb0[L + 1] - e->lb0[L];
      double* pr = part + (int64_t)r * m;
#define CTC_ESP_CLASS(LL)                                                                                   \
  case LL:                                                                                                  \
    esp_class_kernel<LL><<<grid, kEspThreads, 0, st>>>(e->d_pairs, e->d_h, e->d_batches, b0, nb, e->d_boys, \
                                                      pts, m, pr);                                         \
    break;
      switch (L) {
        CTC_ESP_CLASS(0)
        CTC_ESP_CLASS(1)
        CTC_ESP_CLASS(2)
        CTC_ESP_CLASS(3)
        CTC_ESP_CLASS(4)
        CTC_ESP_CLASS(5)
        CTC_ESP_CLASS(6)
        CTC_ESP_CLASS(7)
        CTC_ESP_CLASS(8)
      }
#undef CTC_ESP_CLASS
      CTC_CUDA_TRY(cudaGetLastError());
      r += sl[L];
    }
    esp_finish_kernel<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(part, rows, e->d_atoms, e->natom, pts, m,
                                                                   d_out + p0);
    CTC_CUDA_TRY(cudaGetLastError());
  }
  return CTC_OK;
}

}  // namespace ctc
