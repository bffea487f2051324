// ctc_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A plain FP64 CPU restatement of the reference's grid-evaluation algorithms,
// used by tests/, the smoke check and bench.py's CPU-baseline leg as the
// checker.  Nothing in the product links, imports or calls this file.
//
// Parity pin: the outputs of this file are checked against golden vectors that
// the reference's own CUDA drivers produced (tests/golden/, made by
// tests/golden/make_golden.py through oracle/ref_harness.cpp).
//
// What it restates (reference file:line):
//   * shell sizes / fchk angular-momentum codes     include/contracted_shell.h:10-37
//   * AO component order (Cartesian and pure)        src/evaluate_density.cu:80,114,143,196,235-236,314
//   * primitive normalisation, pure norms            src/cuda_basis_utils.cu:7-109
//   * real solid harmonics d, f, g                   src/cuda_basis_utils.cu:111-224
//   * AO values / 1st / 2nd derivatives              src/evaluate_density.cu:25-393,
//                                                    src/evaluate_gradient.cu:18-1127,
//                                                    src/evaluate_hessian.cu:17-1835
//   * rho = sum (Phi D) o Phi                         src/evaluate_density.cu:663-840
//   * grad rho = 2 sum (dk Phi D) o Phi               src/evaluate_gradient.cu:1197-1422
//   * Hessian = 2[(di Phi D) o dj Phi + (Phi D) o di dj Phi]   src/evaluate_hessian.cu:1906-2307
//   * Laplacian, tau_PD, tau_alpha                   src/evaluate_laplacian.cu:479-841,
//                                                    src/evaluate_kinetic_dens.cu:12-214
//   * RDG (masked divide at 1e-20), Shannon, W, TF, GGE, general(ish) KED
//                                                    src/evaluate_densbased.cu:44-222,
//                                                    src/cuda_utils.cu:71-84
//   * ESP: McMurchie-Davidson E (Helgaker 9.5.6/7) and R (9.9.18-20)
//          recursions, V = sum Z/|r-R| - sum D o V    include/integral_coeffs.cuh:17-238,
//                                                    src/evaluate_electrostatic.cu:10161-10370
//     The Boys function here is evaluated accurately (series + downward
//     recursion); the reference's forward recursion (include/boys_functions.cuh:13-31)
//     loses digits at small T and is NaN at T = 0.
//
// Build: oracle/Makefile (g++ -O3 -march=native -fopenmp -shared).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <omp.h>

namespace {

constexpr double kPi = 3.14159265358979323846264338327950288;

struct Term { double c; int a, b, z; };
using Comp = std::vector<Term>;

double dfact(int n) { double r = 1.0; while (n > 1) { r *= n; n -= 2; } return r; }

// Cartesian component order of the reference for each l.
const int kCart[5][15][3] = {
  {{0,0,0}},
  {{1,0,0},{0,1,0},{0,0,1}},
  {{2,0,0},{0,2,0},{0,0,2},{1,1,0},{1,0,1},{0,1,1}},
  {{3,0,0},{0,3,0},{0,0,3},{1,2,0},{2,1,0},{2,0,1},{1,0,2},{0,1,2},{0,2,1},{1,1,1}},
  {{0,0,4},{0,1,3},{0,2,2},{0,3,1},{0,4,0},{1,0,3},{1,1,2},{1,2,1},{1,3,0},{2,0,2},
   {2,1,1},{2,2,0},{3,0,1},{3,1,0},{4,0,0}}};

// Component list of one segment: polynomial terms including the angular part
// of the normalisation (the radial part N_l(alpha) = (2a/pi)^(3/4) (4a)^(l/2)
// is folded into the primitive coefficients).
std::vector<Comp> components(int angmom) {
  std::vector<Comp> out;
  int l = std::abs(angmom);
  if (angmom >= 0) {
    int n = (l + 1) * (l + 2) / 2;
    for (int i = 0; i < n; ++i) {
      int a = kCart[l][i][0], b = kCart[l][i][1], c = kCart[l][i][2];
      double nrm = 1.0 / std::sqrt(dfact(2 * a - 1) * dfact(2 * b - 1) * dfact(2 * c - 1));
      out.push_back({{nrm, a, b, c}});
    }
    return out;
  }
  const double s3 = std::sqrt(3.0), s15 = std::sqrt(15.0), s1p5 = std::sqrt(1.5),
               s2p5 = std::sqrt(2.5), s5 = std::sqrt(5.0), s35 = std::sqrt(35.0),
               s17p5 = std::sqrt(17.5);
  if (l == 2) {
    // order m = 0, 1, -1, 2, -2
    out.push_back({{1.0, 0, 0, 2}, {-0.5, 2, 0, 0}, {-0.5, 0, 2, 0}});
    out.push_back({{s3, 1, 0, 1}});
    out.push_back({{s3, 0, 1, 1}});
    out.push_back({{0.5 * s3, 2, 0, 0}, {-0.5 * s3, 0, 2, 0}});
    out.push_back({{s3, 1, 1, 0}});
  } else if (l == 3) {
    // order m = 0, 1, -1, 2, -2, 3, -3
    out.push_back({{1.0, 0, 0, 3}, {-1.5, 2, 0, 1}, {-1.5, 0, 2, 1}});
    out.push_back({{2 * s1p5, 1, 0, 2}, {-0.5 * s1p5, 3, 0, 0}, {-0.5 * s1p5, 1, 2, 0}});
    out.push_back({{2 * s1p5, 0, 1, 2}, {-0.5 * s1p5, 2, 1, 0}, {-0.5 * s1p5, 0, 3, 0}});
    out.push_back({{0.5 * s15, 2, 0, 1}, {-0.5 * s15, 0, 2, 1}});
    out.push_back({{s15, 1, 1, 1}});
    out.push_back({{0.5 * s2p5, 3, 0, 0}, {-1.5 * s2p5, 1, 2, 0}});
    out.push_back({{1.5 * s2p5, 2, 1, 0}, {-0.5 * s2p5, 0, 3, 0}});
  } else if (l == 4) {
    // order m = 0, 1, -1, 2, -2, 3, -3, 4, -4
    out.push_back({{1.0, 0, 0, 4}, {0.375, 4, 0, 0}, {0.375, 0, 4, 0}, {0.75, 2, 2, 0},
                   {-3.0, 2, 0, 2}, {-3.0, 0, 2, 2}});
    out.push_back({{2 * s2p5, 1, 0, 3}, {-1.5 * s2p5, 3, 0, 1}, {-1.5 * s2p5, 1, 2, 1}});
    out.push_back({{2 * s2p5, 0, 1, 3}, {-1.5 * s2p5, 2, 1, 1}, {-1.5 * s2p5, 0, 3, 1}});
    out.push_back({{1.5 * s5, 2, 0, 2}, {-1.5 * s5, 0, 2, 2}, {-0.25 * s5, 4, 0, 0},
                   {0.25 * s5, 0, 4, 0}});
    out.push_back({{3 * s5, 1, 1, 2}, {-0.5 * s5, 3, 1, 0}, {-0.5 * s5, 1, 3, 0}});
    out.push_back({{0.5 * s17p5, 3, 0, 1}, {-1.5 * s17p5, 1, 2, 1}});
    out.push_back({{1.5 * s17p5, 2, 1, 1}, {-0.5 * s17p5, 0, 3, 1}});
    out.push_back({{s35 / 8, 4, 0, 0}, {-6 * s35 / 8, 2, 2, 0}, {s35 / 8, 0, 4, 0}});
    out.push_back({{0.5 * s35, 3, 1, 0}, {-0.5 * s35, 1, 3, 0}});
  }
  double nrm = 1.0 / std::sqrt(dfact(2 * l - 1));
  for (auto& c : out) for (auto& t : c) t.c *= nrm;
  return out;
}

int nfunc(int angmom) {
  switch (angmom) {
    case 0: return 1; case 1: return 3; case 2: return 6; case -2: return 5;
    case 3: return 10; case -3: return 7; case 4: return 15; case -4: return 9;
  }
  return -1;
}

struct Seg {
  double c[3];
  int l;
  int atom;
  int ao;                       // first AO index
  std::vector<double> alpha;    // exponents
  std::vector<double> coef;     // coefficient * N_l(alpha)
  std::vector<Comp> comps;
};

}  // namespace

extern "C" {

// Flat basis: the same layout as the product's C ABI (generalised shells).
struct ctco_basis {
  int32_t nshell;
  const double* centers;      // [nshell][3]
  const int32_t* shell_atom;  // [nshell] or null
  const int32_t* nprim;       // [nshell]
  const int32_t* nseg;        // [nshell]
  const int32_t* angmoms;     // [sum nseg]
  const double* exps;         // [sum nprim]
  const double* coeffs;       // [sum nseg*nprim]
};

}  // extern "C"

namespace {

int expand(const ctco_basis* b, std::vector<Seg>& segs) {
  segs.clear();
  int ao = 0, ia = 0, ip = 0, ic = 0;
  for (int s = 0; s < b->nshell; ++s) {
    int K = b->nprim[s], S = b->nseg[s];
    for (int g = 0; g < S; ++g) {
      Seg sg;
      int am = b->angmoms[ia + g];
      if (nfunc(am) < 0) return -1;
      sg.l = std::abs(am);
      for (int d = 0; d < 3; ++d) sg.c[d] = b->centers[3 * s + d];
      sg.atom = b->shell_atom ? b->shell_atom[s] : -1;
      sg.ao = ao;
      for (int k = 0; k < K; ++k) {
        double a = b->exps[ip + k];
        double n = std::pow(2.0 * a / kPi, 0.75) * std::pow(4.0 * a, 0.5 * sg.l);
        sg.alpha.push_back(a);
        sg.coef.push_back(b->coeffs[ic + g * K + k] * n);
      }
      sg.comps = components(am);
      ao += nfunc(am);
      segs.push_back(std::move(sg));
    }
    ia += S; ip += K; ic += S * K;
  }
  return ao;
}

inline double pw(double x, int n) {
  if (n < 0) return 0.0;
  double r = 1.0;
  for (int i = 0; i < n; ++i) r *= x;
  return r;
}

// Values (deriv=0), + gradient (deriv=1), + 6 second derivatives (deriv=2,
// order xx xy xz yy yz zz) of every AO of one segment at one point.
// out[q][j] for q in [0, nq), j over the segment's components.
void eval_seg(const Seg& s, const double* p, int deriv, double* out, int stride) {
  double x = p[0] - s.c[0], y = p[1] - s.c[1], z = p[2] - s.c[2];
  double r2 = x * x + y * y + z * z;
  double R0 = 0, R1 = 0, R2 = 0;
  for (size_t k = 0; k < s.alpha.size(); ++k) {
    double e = s.coef[k] * std::exp(-s.alpha[k] * r2);
    R0 += e;
    R1 += s.alpha[k] * e;
    R2 += s.alpha[k] * s.alpha[k] * e;
  }
  int nq = deriv == 0 ? 1 : (deriv == 1 ? 4 : 10);
  for (size_t j = 0; j < s.comps.size(); ++j) {
    double q[10] = {0};
    for (const Term& t : s.comps[j]) {
      int a = t.a, b = t.b, c = t.z;
      double X0 = pw(x, a), Y0 = pw(y, b), Z0 = pw(z, c);
      q[0] += t.c * X0 * Y0 * Z0 * R0;
      if (deriv >= 1) {
        // d/dx [x^a e] = a x^(a-1) e - 2 alpha x^(a+1) e
        double Xa = a * pw(x, a - 1), Xb = pw(x, a + 1);
        double Ya = b * pw(y, b - 1), Yb = pw(y, b + 1);
        double Za = c * pw(z, c - 1), Zb = pw(z, c + 1);
        q[1] += t.c * (Xa * Y0 * Z0 * R0 - 2 * Xb * Y0 * Z0 * R1);
        q[2] += t.c * (X0 * Ya * Z0 * R0 - 2 * X0 * Yb * Z0 * R1);
        q[3] += t.c * (X0 * Y0 * Za * R0 - 2 * X0 * Y0 * Zb * R1);
        if (deriv >= 2) {
          // d2/dx2 [x^a e] = a(a-1) x^(a-2) - 2 alpha (2a+1) x^a + 4 alpha^2 x^(a+2)
          double Xaa = a * (a - 1) * pw(x, a - 2), Xc = (2 * a + 1) * X0, Xd = pw(x, a + 2);
          double Yaa = b * (b - 1) * pw(y, b - 2), Yc = (2 * b + 1) * Y0, Yd = pw(y, b + 2);
          double Zaa = c * (c - 1) * pw(z, c - 2), Zc = (2 * c + 1) * Z0, Zd = pw(z, c + 2);
          q[4] += t.c * ((Xaa * R0 - 2 * Xc * R1 + 4 * Xd * R2) * Y0 * Z0);
          q[5] += t.c * ((Xa * Ya * R0 - 2 * (Xa * Yb + Xb * Ya) * R1 + 4 * Xb * Yb * R2) * Z0);
          q[6] += t.c * ((Xa * Za * R0 - 2 * (Xa * Zb + Xb * Za) * R1 + 4 * Xb * Zb * R2) * Y0);
          q[7] += t.c * ((Yaa * R0 - 2 * Yc * R1 + 4 * Yd * R2) * X0 * Z0);
          q[8] += t.c * ((Ya * Za * R0 - 2 * (Ya * Zb + Yb * Za) * R1 + 4 * Yb * Zb * R2) * X0);
          q[9] += t.c * ((Zaa * R0 - 2 * Zc * R1 + 4 * Zd * R2) * X0 * Y0);
        }
      }
    }
    for (int k = 0; k < nq; ++k) out[k * stride + j] = q[k];
  }
}

// AO block for points [p0, p0+nb): buf[q][b][M]
void ao_block(const std::vector<Seg>& segs, int M, const double* pts, int nb, int deriv,
              double* buf) {
  int nq = deriv == 0 ? 1 : (deriv == 1 ? 4 : 10);
  std::vector<double> tmp(10 * 16);
  for (int b = 0; b < nb; ++b) {
    for (const Seg& s : segs) {
      eval_seg(s, pts + 3 * b, deriv, tmp.data(), 16);
      int n = (int)s.comps.size();
      for (int q = 0; q < nq; ++q)
        for (int j = 0; j < n; ++j) buf[((size_t)q * nb + b) * M + s.ao + j] = tmp[q * 16 + j];
    }
  }
}

// G[b][nu] = sum_mu A[b][mu] D[mu][nu]
void gemm_rows(const double* A, const double* D, int nb, int M, double* G) {
  std::fill(G, G + (size_t)nb * M, 0.0);
  for (int b = 0; b < nb; ++b) {
    const double* a = A + (size_t)b * M;
    double* g = G + (size_t)b * M;
    for (int mu = 0; mu < M; ++mu) {
      double am = a[mu];
      if (am == 0.0) continue;
      const double* d = D + (size_t)mu * M;
      for (int nu = 0; nu < M; ++nu) g[nu] += am * d[nu];
    }
  }
}

inline double dot(const double* a, const double* b, int n) {
  double s = 0;
  for (int i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

// ---------------------------------------------------------------- Boys / MD
void boys(int nmax, double T, double* F) {
  if (T < 1e-14) {
    for (int n = 0; n <= nmax; ++n) F[n] = 1.0 / (2 * n + 1) - T / (2 * n + 3);
    return;
  }
  double e = std::exp(-T);
  if (T > 45.0) {
    F[0] = 0.5 * std::sqrt(kPi / T);
    for (int n = 1; n <= nmax; ++n) F[n] = ((2 * n - 1) * F[n - 1] - e) / (2 * T);
    return;
  }
  // F_m(T) = e^{-T} sum_i (2T)^i / ((2m+1)(2m+3)...(2m+2i+1))
  double term = 1.0 / (2 * nmax + 1), sum = term;
  for (int i = 1; i < 400; ++i) {
    term *= 2 * T / (2 * nmax + 2 * i + 1);
    sum += term;
    if (term < 1e-18 * sum) break;
  }
  F[nmax] = e * sum;
  for (int n = nmax; n > 0; --n) F[n - 1] = (2 * T * F[n] + e) / (2 * n - 1);
}

// Hermite expansion coefficients E^{ij}_t for one Cartesian direction,
// i <= li, j <= lj, t <= i + j.  E[(i*(lj+1)+j)*(L+1)+t]
void hermite_E(int li, int lj, double a, double b, double XAB, std::vector<double>& E) {
  int L = li + lj;
  double p = a + b, mu = a * b / p;
  double XPA = -(b / p) * XAB, XPB = (a / p) * XAB;
  E.assign((li + 1) * (lj + 1) * (L + 1), 0.0);
  auto at = [&](int i, int j, int t) -> double& { return E[(i * (lj + 1) + j) * (L + 1) + t]; };
  at(0, 0, 0) = std::exp(-mu * XAB * XAB);
  for (int i = 0; i <= li; ++i) {
    for (int j = 0; j <= lj; ++j) {
      if (i == 0 && j == 0) continue;
      for (int t = 0; t <= i + j; ++t) {
        double v;
        if (j == 0) {
          double em = t >= 1 ? at(i - 1, 0, t - 1) : 0.0;
          double e0 = t <= i - 1 ? at(i - 1, 0, t) : 0.0;
          double ep = t + 1 <= i - 1 ? at(i - 1, 0, t + 1) : 0.0;
          v = em / (2 * p) + XPA * e0 + (t + 1) * ep;
        } else {
          double em = t >= 1 ? at(i, j - 1, t - 1) : 0.0;
          double e0 = t <= i + j - 1 ? at(i, j - 1, t) : 0.0;
          double ep = t + 1 <= i + j - 1 ? at(i, j - 1, t + 1) : 0.0;
          v = em / (2 * p) + XPB * e0 + (t + 1) * ep;
        }
        at(i, j, t) = v;
      }
    }
  }
}

// R^0_{tuv} for t+u+v <= L.  Rout[(t*(L+1)+u)*(L+1)+v]
void hermite_R(int L, double p, double X, double Y, double Z, std::vector<double>& Rout) {
  double T = p * (X * X + Y * Y + Z * Z);
  std::vector<double> F(L + 1);
  boys(L, T, F.data());
  int S = L + 1;
  // R[n][t][u][v]
  std::vector<double> R((size_t)S * S * S * S, 0.0);
  auto at = [&](int n, int t, int u, int v) -> double& {
    return R[(((size_t)n * S + t) * S + u) * S + v];
  };
  double m2p = 1.0;
  for (int n = 0; n <= L; ++n) { at(n, 0, 0, 0) = m2p * F[n]; m2p *= -2 * p; }
  for (int tot = 1; tot <= L; ++tot) {
    for (int n = 0; n <= L - tot; ++n) {
      for (int t = 0; t <= tot; ++t) {
        for (int u = 0; u <= tot - t; ++u) {
          int v = tot - t - u;
          double r;
          if (t > 0) {
            r = X * at(n + 1, t - 1, u, v) + (t > 1 ? (t - 1) * at(n + 1, t - 2, u, v) : 0.0);
          } else if (u > 0) {
            r = Y * at(n + 1, t, u - 1, v) + (u > 1 ? (u - 1) * at(n + 1, t, u - 2, v) : 0.0);
          } else {
            r = Z * at(n + 1, t, u, v - 1) + (v > 1 ? (v - 1) * at(n + 1, t, u, v - 2) : 0.0);
          }
          at(n, t, u, v) = r;
        }
      }
    }
  }
  Rout.assign((size_t)S * S * S, 0.0);
  for (int t = 0; t <= L; ++t)
    for (int u = 0; u <= L - t; ++u)
      for (int v = 0; v <= L - t - u; ++v) Rout[((size_t)t * S + u) * S + v] = at(0, t, u, v);
}

// Electronic part sum_{mu,nu} D_{mu nu} V_{mu nu}(C) at one point.
double esp_electronic(const std::vector<Seg>& segs, const double* D, int M, const double* C) {
  double total = 0.0;
  std::vector<double> Ex, Ey, Ez, R;
  std::vector<double> V;  // [ni][nj] AO block
  for (size_t I = 0; I < segs.size(); ++I) {
    const Seg& A = segs[I];
    for (size_t J = I; J < segs.size(); ++J) {
      const Seg& B = segs[J];
      int la = A.l, lb = B.l, L = la + lb, S = L + 1;
      int na = (int)A.comps.size(), nb = (int)B.comps.size();
      V.assign((size_t)na * nb, 0.0);
      for (size_t ka = 0; ka < A.alpha.size(); ++ka) {
        for (size_t kb = 0; kb < B.alpha.size(); ++kb) {
          double a = A.alpha[ka], b = B.alpha[kb], p = a + b;
          double P[3];
          for (int d = 0; d < 3; ++d) P[d] = (a * A.c[d] + b * B.c[d]) / p;
          hermite_E(la, lb, a, b, A.c[0] - B.c[0], Ex);
          hermite_E(la, lb, a, b, A.c[1] - B.c[1], Ey);
          hermite_E(la, lb, a, b, A.c[2] - B.c[2], Ez);
          hermite_R(L, p, P[0] - C[0], P[1] - C[1], P[2] - C[2], R);
          double pref = A.coef[ka] * B.coef[kb] * 2.0 * kPi / p;
          auto E = [&](const std::vector<double>& e, int i, int j, int t) {
            return e[(i * (lb + 1) + j) * (L + 1) + t];
          };
          for (int ia = 0; ia < na; ++ia) {
            for (const Term& ta : A.comps[ia]) {
              for (int ib = 0; ib < nb; ++ib) {
                for (const Term& tb : B.comps[ib]) {
                  double s = 0.0;
                  for (int t = 0; t <= ta.a + tb.a; ++t) {
                    double ex = E(Ex, ta.a, tb.a, t);
                    for (int u = 0; u <= ta.b + tb.b; ++u) {
                      double exy = ex * E(Ey, ta.b, tb.b, u);
                      for (int v = 0; v <= ta.z + tb.z; ++v)
                        s += exy * E(Ez, ta.z, tb.z, v) * R[((size_t)t * S + u) * S + v];
                    }
                  }
                  V[(size_t)ia * nb + ib] += pref * ta.c * tb.c * s;
                }
              }
            }
          }
        }
      }
      double fac = (I == J) ? 1.0 : 2.0;
      for (int ia = 0; ia < na; ++ia)
        for (int ib = 0; ib < nb; ++ib)
          total += fac * D[(size_t)(A.ao + ia) * M + (B.ao + ib)] * V[(size_t)ia * nb + ib];
    }
  }
  return total;
}

}  // namespace

extern "C" {

// Number of AO functions of a basis, or -1 on an unknown angular momentum.
int ctco_nbasis(const ctco_basis* b) {
  std::vector<Seg> segs;
  return expand(b, segs);
}

// AO values and derivatives: out[q][n][M], q in [0,1|4|10) as deriv = 0|1|2
// (order: value, x, y, z, xx, xy, xz, yy, yz, zz).
int ctco_eval_ao(const ctco_basis* b, const double* pts, int64_t n, int deriv, double* out,
                 int nthreads) {
  std::vector<Seg> segs;
  int M = expand(b, segs);
  if (M < 0) return -1;
  int nq = deriv == 0 ? 1 : (deriv == 1 ? 4 : 10);
  if (nthreads > 0) omp_set_num_threads(nthreads);
  const int BLK = 16;
#pragma omp parallel
  {
    std::vector<double> buf((size_t)nq * BLK * M);
#pragma omp for schedule(dynamic)
    for (int64_t p0 = 0; p0 < n; p0 += BLK) {
      int nb = (int)std::min<int64_t>(BLK, n - p0);
      ao_block(segs, M, pts + 3 * p0, nb, deriv, buf.data());
      for (int q = 0; q < nq; ++q)
        for (int bb = 0; bb < nb; ++bb)
          std::memcpy(out + ((size_t)q * n + p0 + bb) * M, buf.data() + ((size_t)q * nb + bb) * M,
                      sizeof(double) * M);
    }
  }
  return M;
}

// Local descriptors.  Any output pointer may be null.
//   rho (n)  grad (n,3)  hess (n,3,3)  lap (n)  tau_pd (n)  tau_a (n) = tau_pd + alpha*lap
//   rdg (n)  shannon (n)
int ctco_eval_local(const ctco_basis* b, const double* D, int M, const double* pts, int64_t n,
                    double alpha, double* rho, double* grad, double* hess, double* lap,
                    double* tau_pd, double* tau_a, double* rdg, double* shannon, int nthreads) {
  std::vector<Seg> segs;
  if (expand(b, segs) != M) return -1;
  bool need_g = hess || lap || tau_pd || tau_a;
  bool need_d1 = grad || need_g || rdg;
  bool need_d2 = hess || lap || tau_a;
  int deriv = need_d2 ? 2 : (need_d1 ? 1 : 0);
  int nq = deriv == 0 ? 1 : (deriv == 1 ? 4 : 10);
  if (nthreads > 0) omp_set_num_threads(nthreads);
  const int BLK = 16;
  const double rdg_pref = 0.5 / std::pow(3.0 * kPi * kPi, 1.0 / 3.0);
#pragma omp parallel
  {
    std::vector<double> buf((size_t)nq * BLK * M);
    std::vector<double> G((size_t)4 * BLK * M);
#pragma omp for schedule(dynamic)
    for (int64_t p0 = 0; p0 < n; p0 += BLK) {
      int nb = (int)std::min<int64_t>(BLK, n - p0);
      ao_block(segs, M, pts + 3 * p0, nb, deriv, buf.data());
      auto A = [&](int q, int bb) { return buf.data() + ((size_t)q * nb + bb) * M; };
      auto Gq = [&](int q, int bb) { return G.data() + ((size_t)q * nb + bb) * M; };
      gemm_rows(A(0, 0), D, nb, M, Gq(0, 0));
      if (need_g)
        for (int k = 1; k <= 3; ++k) gemm_rows(A(k, 0), D, nb, M, Gq(k, 0));
      for (int bb = 0; bb < nb; ++bb) {
        int64_t p = p0 + bb;
        double r = dot(Gq(0, bb), A(0, bb), M);
        double g[3] = {0, 0, 0};
        if (need_d1)
          for (int k = 0; k < 3; ++k) g[k] = 2.0 * dot(Gq(0, bb), A(1 + k, bb), M);
        double H[3][3] = {{0}};
        double tpd = 0.0;
        if (need_g) {
          for (int k = 0; k < 3; ++k) tpd += dot(Gq(1 + k, bb), A(1 + k, bb), M);
          tpd *= 0.5;
        }
        if (need_d2) {
          // second-derivative rows 4..9 = xx xy xz yy yz zz
          const int idx[3][3] = {{4, 5, 6}, {5, 7, 8}, {6, 8, 9}};
          for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
              H[i][j] = 2.0 * (dot(Gq(1 + i, bb), A(1 + j, bb), M) +
                               dot(Gq(0, bb), A(idx[i][j], bb), M));
        }
        double lp = H[0][0] + H[1][1] + H[2][2];
        if (rho) rho[p] = r;
        if (grad) for (int k = 0; k < 3; ++k) grad[3 * p + k] = g[k];
        if (hess) for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) hess[9 * p + 3 * i + j] = H[i][j];
        if (lap) lap[p] = lp;
        if (tau_pd) tau_pd[p] = tpd;
        if (tau_a) tau_a[p] = tpd + alpha * lp;
        if (rdg) {
          double nrm = std::sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
          double d43 = std::pow(r, 4.0 / 3.0);
          double q = d43 > 1e-20 ? nrm / d43 : 1e-20;
          rdg[p] = rdg_pref * q;
        }
        if (shannon) shannon[p] = r * std::log(r);
      }
    }
  }
  return 0;
}

// Electrostatic potential V(C) = sum_A Z_A/|C - R_A| - sum_{mu nu} D_{mu nu} V_{mu nu}(C).
int ctco_eval_esp(const ctco_basis* b, const double* D, int M, int natom, const double* atoms,
                  const double* charges, const double* pts, int64_t n, double* out,
                  int nthreads) {
  std::vector<Seg> segs;
  if (expand(b, segs) != M) return -1;
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic)
  for (int64_t p = 0; p < n; ++p) {
    const double* C = pts + 3 * p;
    double v = -esp_electronic(segs, D, M, C);
    for (int a = 0; a < natom; ++a) {
      double dx = C[0] - atoms[3 * a], dy = C[1] - atoms[3 * a + 1], dz = C[2] - atoms[3 * a + 2];
      v += charges[a] / std::sqrt(dx * dx + dy * dy + dz * dz);
    }
    out[p] = v;
  }
  return 0;
}

// Adjoint of (rho, grad rho) for a grid functional.  v_rho (n) and v_grad
// (n,3, may be null) are dL/drho_g and dL/d(grad rho)_g (weights included).
//   dLdD[mu][nu] = sum_g v_rho phi_mu phi_nu + v_grad.(grad phi_mu phi_nu + phi_mu grad phi_nu)
//   dLdR[A][j]   = sum_g sum_{mu on A} -2 v_rho dj phi_mu G0_mu
//                  - 2 sum_k v_k (dj dk phi_mu G0_mu + dj phi_mu Gk_mu)
// with G0 = Phi D and Gk = dk Phi D.  Points and weights are held fixed.
int ctco_adjoint(const ctco_basis* b, const double* D, int M, int natom, const double* pts,
                 int64_t n, const double* v_rho, const double* v_grad, double* dLdD,
                 double* dLdR, int nthreads) {
  std::vector<Seg> segs;
  if (expand(b, segs) != M) return -1;
  std::vector<int> ao_atom(M, -1);
  for (const Seg& s : segs)
    for (size_t j = 0; j < s.comps.size(); ++j) ao_atom[s.ao + j] = s.atom;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  int deriv = v_grad ? 2 : 1;
  int nq = deriv == 1 ? 4 : 10;
  int nthr = omp_get_max_threads();
  std::vector<std::vector<double>> accD(nthr, std::vector<double>(dLdD ? (size_t)M * M : 0, 0.0));
  std::vector<std::vector<double>> accR(nthr, std::vector<double>((size_t)natom * 3, 0.0));
  const int BLK = 16;
#pragma omp parallel
  {
    int tid = omp_get_thread_num();
    std::vector<double> buf((size_t)nq * BLK * M);
    std::vector<double> G((size_t)4 * BLK * M);
    std::vector<double> W((size_t)BLK * M);
    double* aD = accD[tid].data();
    double* aR = accR[tid].data();
#pragma omp for schedule(dynamic)
    for (int64_t p0 = 0; p0 < n; p0 += BLK) {
      int nb = (int)std::min<int64_t>(BLK, n - p0);
      ao_block(segs, M, pts + 3 * p0, nb, deriv, buf.data());
      auto A = [&](int q, int bb) { return buf.data() + ((size_t)q * nb + bb) * M; };
      auto Gq = [&](int q, int bb) { return G.data() + ((size_t)q * nb + bb) * M; };
      if (dLdD) {
        // W_mu = v_rho phi_mu + 2 sum_k v_k dk phi_mu ; dLdD += sym(W phi^T)
        for (int bb = 0; bb < nb; ++bb) {
          int64_t p = p0 + bb;
          const double* ph = A(0, bb);
          double* w = W.data() + (size_t)bb * M;
          // v_rho phi phi^T + sum_k v_k (dk phi phi^T + phi dk phi^T)
          // = 0.5*(w phi^T + phi w^T) with w = v_rho phi + 2 sum_k v_k dk phi
          for (int mu = 0; mu < M; ++mu) w[mu] = v_rho[p] * ph[mu];
          if (v_grad)
            for (int k = 0; k < 3; ++k) {
              const double* dk = A(1 + k, bb);
              double vk = 2.0 * v_grad[3 * p + k];
              for (int mu = 0; mu < M; ++mu) w[mu] += vk * dk[mu];
            }
          for (int mu = 0; mu < M; ++mu) {
            double wm = w[mu], pm = ph[mu];
            double* row = aD + (size_t)mu * M;
            for (int nu = 0; nu < M; ++nu) row[nu] += 0.5 * (wm * ph[nu] + pm * w[nu]);
          }
        }
      }
      if (dLdR) {
        gemm_rows(A(0, 0), D, nb, M, Gq(0, 0));
        if (v_grad)
          for (int k = 1; k <= 3; ++k) gemm_rows(A(k, 0), D, nb, M, Gq(k, 0));
        const int idx[3][3] = {{4, 5, 6}, {5, 7, 8}, {6, 8, 9}};
        for (int bb = 0; bb < nb; ++bb) {
          int64_t p = p0 + bb;
          for (int mu = 0; mu < M; ++mu) {
            int at = ao_atom[mu];
            if (at < 0) continue;
            double g0 = Gq(0, bb)[mu];
            for (int j = 0; j < 3; ++j) {
              double dj = A(1 + j, bb)[mu];
              double acc = -2.0 * v_rho[p] * dj * g0;
              if (v_grad)
                for (int k = 0; k < 3; ++k) {
                  double vk = v_grad[3 * p + k];
                  acc -= 2.0 * vk * (A(idx[j][k], bb)[mu] * g0 + dj * Gq(1 + k, bb)[mu]);
                }
              aR[3 * at + j] += acc;
            }
          }
        }
      }
    }
  }
  if (dLdD) {
    std::fill(dLdD, dLdD + (size_t)M * M, 0.0);
    for (int t = 0; t < nthr; ++t)
      for (size_t i = 0; i < (size_t)M * M; ++i) dLdD[i] += accD[t][i];
  }
  if (dLdR) {
    std::fill(dLdR, dLdR + (size_t)natom * 3, 0.0);
    for (int t = 0; t < nthr; ++t)
      for (int i = 0; i < natom * 3; ++i) dLdR[i] += accR[t][i];
  }
  return 0;
}

}  // extern "C"
