// ctc_wfn.cpp -- native reader of AIM wavefunction files (.wfn, .wfx).
//
// The reference's Molecule(str) (src/pymolecule.cu:18-23) loads its file
// through the Python iodata package (src/iodata.cpp:15-211), which also reads
// these formats.  Both describe the orbitals over individual primitive
// Gaussians: every primitive has a centre, a Cartesian type x^a y^b z^c and an
// exponent, and every orbital a coefficient per primitive that multiplies the
// UNnormalised primitive x^a y^b z^c exp(-alpha r^2).
//
// The reader turns every distinct (centre, l, exponent) into a Cartesian shell
// of one primitive with contraction coefficient 1, whose component (a, b, c)
// is, in the library's convention, N_l(alpha) / sqrt((2a-1)!! (2b-1)!! (2c-1)!!)
// x^a y^b z^c exp(-alpha r^2) with N_l(alpha) = (2 alpha/pi)^(3/4) (4 alpha)^(l/2);
// an orbital's coefficient on that function is its file coefficient divided
// by that factor.  The density matrix is sum_i occ_i c_i c_i^T over the
// orbitals with their occupations (the MO one-particle density matrix,
// src/iodata.cpp:157-160).  The basis is larger than the contracted basis the
// orbitals came from (one function per primitive component), the density it
// describes is the same.
//
// Primitive types 1..20 (s, p, d, f) follow the AIMPAC numbering:
//   1 s; 2-4 x y z; 5-10 xx yy zz xy xz yz;
//   11-20 xxx yyy zzz xxy xxz yyz xyy xzz yzz xyz.
// g primitives (types 21..35) are refused: their order differs between the
// programs that write these files.
//
// .wfn: fixed-format text (title; "GAUSSIAN nmo MOL ORBITALS nprim
// PRIMITIVES natom NUCLEI"; one line per nucleus with its coordinates and
// "CHARGE ="; CENTRE ASSIGNMENTS and TYPE ASSIGNMENTS in 20I3 after a 20-column
// label; EXPONENTS; per orbital an "MO ... OCC NO = ... ORB. ENERGY = ..." line
// and its nprim coefficients).
// .wfx: tagged text; the sections read are Number of Nuclei, Number of
// Primitives, Atomic Numbers, Nuclear Charges, Nuclear Cartesian Coordinates,
// Primitive Centers, Primitive Types, Primitive Exponents, Molecular Orbital
// Occupation Numbers, Molecular Orbital Spin Types (optional) and Molecular
// Orbital Primitive Coefficients (blocks after each <MO Number>).
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "ctc_internal.h"
#include "ctc_wfnfile.h"

using namespace ctc;

namespace {

struct Prim {
  int center;
  int type;
  double alpha;
};

struct Orbital {
  double occ = 0.0;
  bool beta = false;
  std::vector<double> coef;
};

struct Raw {
  std::vector<int> numbers;
  std::vector<double> charges, coords;
  std::vector<Prim> prims;
  std::vector<Orbital> mos;
  bool have_spin = false;
};

double to_double(std::string tok) {
  for (char& c : tok)
    if (c == 'D' || c == 'd') c = 'E';
  char* end = nullptr;
  const double v = std::strtod(tok.c_str(), &end);
  return (end && *end == '\0' && !tok.empty()) ? v : NAN;
}

std::vector<std::string> split(const std::string& s) {
  std::istringstream ss(s);
  std::vector<std::string> t;
  std::string w;
  while (ss >> w) t.push_back(w);
  return t;
}

std::string upper(std::string s) {
  for (char& c : s) c = (char)std::toupper((unsigned char)c);
  return s;
}

// exponents (a, b, c) of AIMPAC primitive types 1..20
bool type_powers(int t, int& a, int& b, int& c) {
  static const int P[20][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0},
                               {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1},
                               {3, 0, 0}, {0, 3, 0}, {0, 0, 3}, {2, 1, 0}, {2, 0, 1},
                               {0, 2, 1}, {1, 2, 0}, {1, 0, 2}, {0, 1, 2}, {1, 1, 1}};
  if (t < 1 || t > 20) return false;
  a = P[t - 1][0];
  b = P[t - 1][1];
  c = P[t - 1][2];
  return true;
}

// the library's Cartesian component order of shell l
int cart_index(int l, int a, int b, int c) {
  static const int C[4][10][3] = {
      {{0, 0, 0}},
      {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}},
      {{2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}},
      {{3, 0, 0}, {0, 3, 0}, {0, 0, 3}, {1, 2, 0}, {2, 1, 0}, {2, 0, 1}, {1, 0, 2}, {0, 1, 2},
       {0, 2, 1}, {1, 1, 1}}};
  const int n = (l + 1) * (l + 2) / 2;
  for (int j = 0; j < n; ++j)
    if (C[l][j][0] == a && C[l][j][1] == b && C[l][j][2] == c) return j;
  return -1;
}

double dfact(int n) {
  double r = 1.0;
  for (; n > 1; n -= 2) r *= n;
  return r;
}

int read_wfn(std::istream& in, Raw& r) {
  auto bad = [](const std::string& m) { return fail(CTC_ERR_INVALID, "wfn: " + m); };
  std::string line;
  if (!std::getline(in, line)) return bad("empty file");  // title
  if (!std::getline(in, line)) return bad("no header line");
  const std::vector<std::string> h = split(line);
  int nmo = -1, nprim = -1, natom = -1;
  for (size_t i = 1; i < h.size(); ++i) {
    const std::string u = upper(h[i]);
    if (u == "MOL") nmo = std::atoi(h[i - 1].c_str());
    if (u == "PRIMITIVES") nprim = std::atoi(h[i - 1].c_str());
    if (u == "NUCLEI") natom = std::atoi(h[i - 1].c_str());
  }
  if (nmo <= 0 || nprim <= 0 || natom <= 0)
    return bad("header must give 'n MOL ORBITALS n PRIMITIVES n NUCLEI'");
  for (int a = 0; a < natom; ++a) {
    if (!std::getline(in, line)) return bad("file ends in the nuclei");
    const size_t close = line.find(')');
    const size_t q = upper(line).find("CHARGE");
    if (close == std::string::npos || q == std::string::npos) return bad("nucleus line without '(CENTRE n)' and 'CHARGE ='");
    const std::vector<std::string> xyz = split(line.substr(close + 1, q - close - 1));
    if (xyz.size() < 3) return bad("nucleus line without three coordinates");
    for (int d = 0; d < 3; ++d) r.coords.push_back(to_double(xyz[d]));
    const size_t eq = line.find('=', q);
    const double z = eq == std::string::npos ? NAN : to_double(split(line.substr(eq + 1)).empty() ? "" : split(line.substr(eq + 1))[0]);
    if (std::isnan(z) || std::isnan(r.coords.back())) return bad("bad nucleus line");
    r.charges.push_back(z);
    r.numbers.push_back((int)std::lround(z));
  }
  std::vector<int> centers, types;
  std::vector<double> exps;
  auto fixed_ints = [&](const std::string& l, std::vector<int>& out) {
    for (size_t p = 20; p < l.size(); p += 3) {
      const std::string f = l.substr(p, 3);
      if (f.find_first_not_of(' ') == std::string::npos) continue;
      out.push_back(std::atoi(f.c_str()));
    }
  };
  while ((int)centers.size() < nprim && std::getline(in, line)) {
    if (upper(line).rfind("CENTRE ASSIGNMENTS", 0) != 0) return bad("expected CENTRE ASSIGNMENTS");
    fixed_ints(line, centers);
  }
  while ((int)types.size() < nprim && std::getline(in, line)) {
    if (upper(line).rfind("TYPE ASSIGNMENTS", 0) != 0) return bad("expected TYPE ASSIGNMENTS");
    fixed_ints(line, types);
  }
  while ((int)exps.size() < nprim && std::getline(in, line)) {
    if (upper(line).rfind("EXPONENTS", 0) != 0) return bad("expected EXPONENTS");
    for (const std::string& t : split(line.substr(9))) exps.push_back(to_double(t));
  }
  if ((int)centers.size() != nprim || (int)types.size() != nprim || (int)exps.size() != nprim)
    return bad("primitive sections do not hold " + std::to_string(nprim) + " entries");
  for (int p = 0; p < nprim; ++p) r.prims.push_back({centers[p] - 1, types[p], exps[p]});
  for (int i = 0; i < nmo; ++i) {
    if (!std::getline(in, line)) return bad("file ends before orbital " + std::to_string(i + 1));
    const std::string u = upper(line);
    const size_t o = u.find("OCC NO");
    if (u.rfind("MO", 0) != 0 || o == std::string::npos) return bad("expected an 'MO ... OCC NO =' line");
    Orbital mo;
    const size_t eq = line.find('=', o);
    const std::vector<std::string> v = split(line.substr(eq + 1));
    mo.occ = v.empty() ? NAN : to_double(v[0]);
    if (std::isnan(mo.occ)) return bad("bad occupation");
    while ((int)mo.coef.size() < nprim && std::getline(in, line))
      for (const std::string& t : split(line)) mo.coef.push_back(to_double(t));
    if ((int)mo.coef.size() != nprim) return bad("orbital " + std::to_string(i + 1) + " has too few coefficients");
    r.mos.push_back(std::move(mo));
  }
  return CTC_OK;
}

int read_wfx(const std::string& text, Raw& r) {
  auto bad = [](const std::string& m) { return fail(CTC_ERR_INVALID, "wfx: " + m); };
  auto section = [&](const std::string& tag, std::string& out) -> bool {
    const std::string open = "<" + tag + ">", close = "</" + tag + ">";
    const size_t a = text.find(open);
    if (a == std::string::npos) return false;
    const size_t b = text.find(close, a);
    if (b == std::string::npos) return false;
    out = text.substr(a + open.size(), b - a - open.size());
    return true;
  };
  std::string s;
  auto ints = [&](const std::string& tag, std::vector<int>& v) -> bool {
    if (!section(tag, s)) return false;
    for (const std::string& t : split(s)) v.push_back(std::atoi(t.c_str()));
    return true;
  };
  auto reals = [&](const std::string& tag, std::vector<double>& v) -> bool {
    if (!section(tag, s)) return false;
    for (const std::string& t : split(s)) v.push_back(to_double(t));
    return true;
  };
  if (section("Keywords", s) && upper(s).find("GTO") == std::string::npos)
    return bad("only GTO wavefunctions are supported");
  std::vector<int> n, centers, types;
  if (!ints("Number of Nuclei", n) || n.size() != 1) return bad("missing <Number of Nuclei>");
  const int natom = n[0];
  n.clear();
  if (!ints("Number of Primitives", n) || n.size() != 1) return bad("missing <Number of Primitives>");
  const int nprim = n[0];
  std::vector<double> exps, occ;
  if (!ints("Atomic Numbers", r.numbers) || (int)r.numbers.size() != natom) return bad("missing or short <Atomic Numbers>");
  if (!reals("Nuclear Charges", r.charges)) r.charges.assign(r.numbers.begin(), r.numbers.end());
  if (!reals("Nuclear Cartesian Coordinates", r.coords) || (int)r.coords.size() != 3 * natom)
    return bad("missing or short <Nuclear Cartesian Coordinates>");
  if (!ints("Primitive Centers", centers) || !ints("Primitive Types", types) || !reals("Primitive Exponents", exps) ||
      (int)centers.size() != nprim || (int)types.size() != nprim || (int)exps.size() != nprim)
    return bad("primitive sections missing or not of <Number of Primitives> entries");
  for (int p = 0; p < nprim; ++p) r.prims.push_back({centers[p] - 1, types[p], exps[p]});
  if (!reals("Molecular Orbital Occupation Numbers", occ)) return bad("missing <Molecular Orbital Occupation Numbers>");
  std::vector<bool> beta(occ.size(), false);
  if (section("Molecular Orbital Spin Types", s)) {
    // one entry per orbital: "Alpha", "Beta" or "Alpha and Beta"
    std::istringstream ss(s);
    std::string l;
    size_t i = 0;
    while (std::getline(ss, l) && i < occ.size()) {
      const std::string u = upper(l);
      if (u.find_first_not_of(" \t\r") == std::string::npos) continue;
      r.have_spin = true;
      beta[i++] = u.find("BETA") != std::string::npos && u.find("ALPHA") == std::string::npos;
    }
  }
  if (!section("Molecular Orbital Primitive Coefficients", s)) return bad("missing <Molecular Orbital Primitive Coefficients>");
  const std::string tag = "</MO Number>";
  size_t pos = 0;
  for (size_t i = 0; i < occ.size(); ++i) {
    const size_t a = s.find(tag, pos);
    if (a == std::string::npos) return bad("fewer coefficient blocks than occupation numbers");
    size_t b = s.find("<MO Number>", a);
    if (b == std::string::npos) b = s.size();
    Orbital mo;
    mo.occ = occ[i];
    mo.beta = beta[i];
    for (const std::string& t : split(s.substr(a + tag.size(), b - a - tag.size()))) mo.coef.push_back(to_double(t));
    if ((int)mo.coef.size() != nprim) return bad("orbital " + std::to_string(i + 1) + " does not have <Number of Primitives> coefficients");
    r.mos.push_back(std::move(mo));
    pos = b;
  }
  return CTC_OK;
}

}  // namespace

extern "C" {

int ctc_wfn_load(const char* path, ctc_fchk** out) {
  if (!path || !out) return fail(CTC_ERR_INVALID, "ctc_wfn_load: null argument");
  *out = nullptr;
  std::ifstream in(path);
  if (!in) return fail(CTC_ERR_INVALID, "wfn: cannot open '" + std::string(path) + "'");
  std::stringstream buf;
  buf << in.rdbuf();
  const std::string text = buf.str();
  Raw r;
  int rc;
  if (text.find("<Number of Primitives>") != std::string::npos) {
    rc = read_wfx(text, r);
  } else {
    std::istringstream ss(text);
    rc = read_wfn(ss, r);
  }
  if (rc != CTC_OK) return rc;
  auto bad = [](const std::string& m) { return fail(CTC_ERR_INVALID, "wfn: " + m); };
  for (double v : r.coords)
    if (std::isnan(v)) return bad("bad nuclear coordinate");
  const int natom = (int)r.numbers.size();
  auto* f = new ctc_fchk();
  f->path = path;
  f->natom = natom;
  f->numbers = r.numbers;
  f->charges = r.charges;
  f->coords = r.coords;
  // one single-primitive Cartesian shell per distinct (centre, l, exponent)
  std::map<std::tuple<int, int, double>, int> shell_of;  // -> first function of the shell
  std::vector<int> func(r.prims.size());
  std::vector<double> scale(r.prims.size());
  int nfun = 0;
  for (size_t p = 0; p < r.prims.size(); ++p) {
    const Prim& q = r.prims[p];
    int a, b, c;
    if (q.type >= 21 && q.type <= 35) {
      delete f;
      return bad("g primitives (types 21-35) are not supported");
    }
    if (!type_powers(q.type, a, b, c)) {
      delete f;
      return bad("primitive type " + std::to_string(q.type) + " is not supported");
    }
    if (q.center < 0 || q.center >= natom || !(q.alpha > 0.0)) {
      delete f;
      return bad("primitive " + std::to_string(p + 1) + " has a bad centre or exponent");
    }
    const int l = a + b + c;
    const auto key = std::make_tuple(q.center, l, q.alpha);
    auto it = shell_of.find(key);
    if (it == shell_of.end()) {
      it = shell_of.emplace(key, nfun).first;
      for (int d = 0; d < 3; ++d) f->centers.push_back(f->coords[3 * q.center + d]);
      f->shell_atom.push_back(q.center);
      f->nprim.push_back(1);
      f->nseg.push_back(1);
      f->angmoms.push_back(l);
      f->exps.push_back(q.alpha);
      f->coeffs.push_back(1.0);
      nfun += (l + 1) * (l + 2) / 2;
    }
    func[p] = it->second + cart_index(l, a, b, c);
    const double nrm = std::pow(2.0 * q.alpha / M_PI, 0.75) * std::pow(4.0 * q.alpha, 0.5 * l) /
                       std::sqrt(dfact(2 * a - 1) * dfact(2 * b - 1) * dfact(2 * c - 1));
    scale[p] = 1.0 / nrm;
  }
  const int M = nfun;
  f->nbasis = M;
  f->D.assign((size_t)M * M, 0.0);
  std::vector<double> cv(M);
  double na = 0.0, nb = 0.0, ne = 0.0;
  for (const Orbital& mo : r.mos) {
    ne += mo.occ;
    if (r.have_spin) (mo.beta ? nb : na) += mo.occ;
    if (mo.occ == 0.0) continue;
    std::fill(cv.begin(), cv.end(), 0.0);
    for (size_t p = 0; p < r.prims.size(); ++p) {
      if (std::isnan(mo.coef[p])) {
        delete f;
        return bad("bad orbital coefficient");
      }
      cv[func[p]] += mo.coef[p] * scale[p];
    }
    for (int i = 0; i < M; ++i) {
      const double ci = mo.occ * cv[i];
      if (ci == 0.0) continue;
      double* row = f->D.data() + (size_t)i * M;
      for (int j = 0; j < M; ++j) row[j] += ci * cv[j];
    }
  }
  if (!r.have_spin || na + nb == 0.0) {
    na = std::ceil(ne / 2.0 - 1e-9);
    nb = ne - na;
  }
  f->nalpha = (int32_t)std::lround(na);
  f->nbeta = (int32_t)std::lround(nb);
  *out = f;
  return CTC_OK;
}

}  // extern "C"
