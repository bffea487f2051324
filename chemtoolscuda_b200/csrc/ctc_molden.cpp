// ctc_molden.cpp -- native reader of Molden files (.molden).
//
// The reference's Molecule(str) (src/pymolecule.cu:18-23) loads its file
// through the Python iodata package (src/iodata.cpp:15-211), which also reads
// Molden files; this reader gives the same molecule without Python.  The file
// holds the atoms, the contracted Gaussian basis per atom and the molecular
// orbitals with their occupations; the result is the same host object as the
// fchk reader's (ctc_wfnfile.h), so ctc_fchk_view_get and ctc_molecule_create
// take it from there.
//
// Conventions of the format as this reader applies them:
//   * [Atoms] AU or Angs: "symbol index Z x y z"; shells sit on their atoms;
//   * [GTO]: per atom "index 0", then shells "label nprim [scale]" followed by
//     nprim lines "exponent coefficient" (sp: "exponent s-coefficient
//     p-coefficient"); labels s, p, sp, d, f, g; a scale factor other than 1
//     is refused; coefficients multiply normalised primitives, as in fchk;
//   * spherical flags: [5D] (pure d and f), [5D10F] (pure d), [7F] (pure f),
//     [5D7F] (pure d and f), [9G] (pure g); without a flag shells are
//     Cartesian;
//   * basis functions within a shell in Molden's order: Cartesian d and f and
//     every pure shell in the order the library uses; Cartesian g in Molden's
//     order xxxx yyyy zzzz xxxy xxxz yyyx yyyz zzzx zzzy xxyy xxzz yyzz xxyz
//     yyxz zzxy, permuted here into the library's (zzzz yzzz ... xxxx);
//   * [MO]: per orbital "Sym=", "Ene=", "Spin=", "Occup=" lines, then
//     "index coefficient" lines (zero coefficients may be left out).
// The density matrix is sum_i occ_i c_i c_i^T over the orbitals with their
// occupations as written (2 for a doubly occupied restricted orbital, 1 for an
// occupied spin orbital), the MO one-particle density matrix the reference
// forms from the same orbitals (src/iodata.cpp:157-160).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "ctc_internal.h"
#include "ctc_wfnfile.h"

using namespace ctc;

namespace {

constexpr double kBohrPerAngstrom = 1.0 / 0.529177210903;  // CODATA 2018 Bohr radius

std::string lower(std::string s) {
  for (char& c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

double to_double(std::string tok) {
  for (char& c : tok)
    if (c == 'D' || c == 'd') c = 'E';  // Fortran exponents
  char* end = nullptr;
  const double v = std::strtod(tok.c_str(), &end);
  return (end && *end == '\0') ? v : NAN;
}

bool is_int(const std::string& tok) {
  if (tok.empty()) return false;
  size_t i = (tok[0] == '-' || tok[0] == '+') ? 1 : 0;
  if (i == tok.size()) return false;
  for (; i < tok.size(); ++i)
    if (!std::isdigit((unsigned char)tok[i])) return false;
  return true;
}

std::vector<std::string> split(const std::string& line) {
  std::istringstream ss(line);
  std::vector<std::string> t;
  std::string w;
  while (ss >> w) t.push_back(w);
  return t;
}

struct RawShell {
  int atom = 0;
  int l = 0;       // 0..4, or -1 for sp
  std::vector<double> exps, c0, c1;
};

struct RawMO {
  bool beta = false;
  double occ = 0.0;
  std::vector<std::pair<int, double>> coef;  // (1-based index, value)
};

// position in the library's Cartesian g order of each component in Molden's
int g_cart_position(int molden_index) {
  static const int mol[15][3] = {{4, 0, 0}, {0, 4, 0}, {0, 0, 4}, {3, 1, 0}, {3, 0, 1},
                                 {1, 3, 0}, {0, 3, 1}, {1, 0, 3}, {0, 1, 3}, {2, 2, 0},
                                 {2, 0, 2}, {0, 2, 2}, {2, 1, 1}, {1, 2, 1}, {1, 1, 2}};
  static const int lib[15][3] = {{0, 0, 4}, {0, 1, 3}, {0, 2, 2}, {0, 3, 1}, {0, 4, 0},
                                 {1, 0, 3}, {1, 1, 2}, {1, 2, 1}, {1, 3, 0}, {2, 0, 2},
                                 {2, 1, 1}, {2, 2, 0}, {3, 0, 1}, {3, 1, 0}, {4, 0, 0}};
  for (int j = 0; j < 15; ++j)
    if (lib[j][0] == mol[molden_index][0] && lib[j][1] == mol[molden_index][1] &&
        lib[j][2] == mol[molden_index][2])
      return j;
  return -1;
}

int ncomp(int t) {
  const int l = t < 0 ? -t : t;
  return t < 0 ? 2 * l + 1 : (l + 1) * (l + 2) / 2;
}

}  // namespace

extern "C" {

int ctc_molden_load(const char* path, ctc_fchk** out) {
  if (!path || !out) return fail(CTC_ERR_INVALID, "ctc_molden_load: null argument");
  *out = nullptr;
  std::ifstream in(path);
  if (!in) return fail(CTC_ERR_INVALID, "molden: cannot open '" + std::string(path) + "'");
  auto bad = [&](const std::string& msg) { return fail(CTC_ERR_INVALID, "molden: " + msg); };

  std::vector<int> numbers;
  std::vector<double> coords;
  std::vector<RawShell> shells;
  std::vector<RawMO> mos;
  bool pure_d = false, pure_f = false, pure_g = false, have_gto = false, have_atoms = false;
  double unit = 1.0;
  std::string section;
  int cur_atom = -1;
  bool mo_in_coefs = false;
  std::string line;
  int lineno = 0;
  while (std::getline(in, line)) {
    ++lineno;
    const std::vector<std::string> t = split(line);
    const std::string where = " (line " + std::to_string(lineno) + ")";
    if (!t.empty() && t[0][0] == '[') {
      const size_t close = line.find(']');
      const std::string name = lower(line.substr(line.find('[') + 1, close == std::string::npos ? std::string::npos : close - line.find('[') - 1));
      const std::string rest = close == std::string::npos ? "" : lower(line.substr(close + 1));
      if (name == "5d") pure_d = pure_f = true;
      else if (name == "5d10f") pure_d = true;
      else if (name == "7f") pure_f = true;
      else if (name == "5d7f") pure_d = pure_f = true;
      else if (name == "9g") pure_g = true;
      else if (name == "sto") return bad("Slater-type orbitals ([STO]) are not supported");
      if (name == "atoms") {
        have_atoms = true;
        unit = rest.find("angs") != std::string::npos ? kBohrPerAngstrom : 1.0;
      }
      if (name == "gto") have_gto = true;
      section = name;
      cur_atom = -1;
      mo_in_coefs = false;
      continue;
    }
    if (section == "atoms") {
      if (t.empty()) continue;
      if (t.size() < 6) return bad("atom line needs 'symbol index Z x y z'" + where);
      numbers.push_back(std::atoi(t[2].c_str()));
      for (int d = 0; d < 3; ++d) {
        const double v = to_double(t[3 + d]);
        if (std::isnan(v)) return bad("bad coordinate" + where);
        coords.push_back(v * unit);
      }
    } else if (section == "gto") {
      if (t.empty()) {
        cur_atom = -1;
        continue;
      }
      if (is_int(t[0])) {  // "atom_index 0" starts an atom's shells
        cur_atom = std::atoi(t[0].c_str()) - 1;
        continue;
      }
      if (cur_atom < 0) return bad("shell outside an atom block" + where);
      const std::string lab = lower(t[0]);
      RawShell sh;
      sh.atom = cur_atom;
      if (lab == "s") sh.l = 0;
      else if (lab == "p") sh.l = 1;
      else if (lab == "sp") sh.l = -1;
      else if (lab == "d") sh.l = 2;
      else if (lab == "f") sh.l = 3;
      else if (lab == "g") sh.l = 4;
      else return bad("shell label '" + t[0] + "' is not supported (s, p, sp, d, f, g)" + where);
      if (t.size() < 2 || !is_int(t[1])) return bad("shell line needs a primitive count" + where);
      const int K = std::atoi(t[1].c_str());
      if (K <= 0) return bad("non-positive primitive count" + where);
      if (t.size() >= 3) {
        const double scale = to_double(t[2]);
        if (std::isnan(scale) || std::fabs(scale - 1.0) > 1e-12)
          return bad("shell scale factors other than 1 are not supported" + where);
      }
      for (int k = 0; k < K; ++k) {
        if (!std::getline(in, line)) return bad("file ends inside a shell" + where);
        ++lineno;
        const std::vector<std::string> p = split(line);
        const size_t need = sh.l == -1 ? 3 : 2;
        if (p.size() < need) return bad("primitive line needs " + std::to_string(need) + " numbers (line " + std::to_string(lineno) + ")");
        const double e = to_double(p[0]), a = to_double(p[1]), b = sh.l == -1 ? to_double(p[2]) : 0.0;
        if (std::isnan(e) || std::isnan(a) || std::isnan(b) || !(e > 0.0))
          return bad("bad primitive (line " + std::to_string(lineno) + ")");
        sh.exps.push_back(e);
        sh.c0.push_back(a);
        if (sh.l == -1) sh.c1.push_back(b);
      }
      shells.push_back(std::move(sh));
    } else if (section == "mo") {
      if (t.empty()) continue;
      const std::string k = lower(t[0]);
      const size_t eq = line.find('=');
      if (eq != std::string::npos) {
        // a key line: a new orbital starts at the first key after coefficients
        if (mo_in_coefs || mos.empty()) mos.emplace_back();
        mo_in_coefs = false;
        const std::string key = lower(line.substr(0, eq));
        const std::string val = line.substr(eq + 1);
        if (key.find("spin") != std::string::npos) mos.back().beta = lower(val).find("beta") != std::string::npos;
        if (key.find("occup") != std::string::npos) {
          const std::vector<std::string> v = split(val);
          const double o = v.empty() ? NAN : to_double(v[0]);
          if (std::isnan(o)) return bad("bad occupation" + where);
          mos.back().occ = o;
        }
        continue;
      }
      if (mos.empty()) return bad("coefficients before the first orbital header" + where);
      if (t.size() < 2 || !is_int(t[0])) return bad("coefficient line needs 'index value'" + where);
      const double v = to_double(t[1]);
      if (std::isnan(v)) return bad("bad coefficient" + where);
      mos.back().coef.emplace_back(std::atoi(t[0].c_str()), v);
      mo_in_coefs = true;
    }
  }
  if (!have_atoms || numbers.empty()) return bad("no [Atoms] section");
  if (!have_gto || shells.empty()) return bad("no [GTO] section");
  if (mos.empty()) return bad("no [MO] section");

  auto* f = new ctc_fchk();
  f->path = path;
  f->natom = (int32_t)numbers.size();
  f->numbers = numbers;
  f->charges.assign(numbers.begin(), numbers.end());
  f->coords = coords;
  // basis, and for every function its column in the library's order
  std::vector<int> where_of;  // Molden function index -> library index
  int nfun = 0;
  for (const RawShell& sh : shells) {
    if (sh.atom < 0 || sh.atom >= f->natom) {
      delete f;
      return bad("shell on atom " + std::to_string(sh.atom + 1) + " of " + std::to_string(f->natom));
    }
    for (int d = 0; d < 3; ++d) f->centers.push_back(f->coords[3 * sh.atom + d]);
    f->shell_atom.push_back(sh.atom);
    f->nprim.push_back((int32_t)sh.exps.size());
    f->exps.insert(f->exps.end(), sh.exps.begin(), sh.exps.end());
    if (sh.l == -1) {
      f->nseg.push_back(2);
      f->angmoms.push_back(0);
      f->angmoms.push_back(1);
      f->coeffs.insert(f->coeffs.end(), sh.c0.begin(), sh.c0.end());
      f->coeffs.insert(f->coeffs.end(), sh.c1.begin(), sh.c1.end());
      for (int j = 0; j < 4; ++j) where_of.push_back(nfun + j);
      nfun += 4;
      continue;
    }
    const bool pure = (sh.l == 2 && pure_d) || (sh.l == 3 && pure_f) || (sh.l == 4 && pure_g);
    const int type = pure ? -sh.l : sh.l;
    f->nseg.push_back(1);
    f->angmoms.push_back(type);
    f->coeffs.insert(f->coeffs.end(), sh.c0.begin(), sh.c0.end());
    const int nc = ncomp(type);
    for (int j = 0; j < nc; ++j) where_of.push_back(nfun + (type == 4 ? g_cart_position(j) : j));
    nfun += nc;
  }
  f->nbasis = nfun;
  const int M = nfun;
  f->D.assign((size_t)M * M, 0.0);
  std::vector<double> c(M);
  double na = 0.0, nb = 0.0;
  bool any_beta = false;
  for (const RawMO& mo : mos) any_beta |= mo.beta;
  for (const RawMO& mo : mos)
    for (const auto& ic : mo.coef)
      if (ic.first < 1 || ic.first > M) {
        delete f;
        return bad("orbital coefficient index " + std::to_string(ic.first) + " outside 1.." + std::to_string(M));
      }
  for (const RawMO& mo : mos) {
    if (any_beta) (mo.beta ? nb : na) += mo.occ;
    else {
      na += std::min(mo.occ, 1.0);
      nb += std::max(mo.occ - 1.0, 0.0);
    }
    if (mo.occ == 0.0) continue;
    std::fill(c.begin(), c.end(), 0.0);
    for (const auto& ic : mo.coef) c[where_of[ic.first - 1]] = ic.second;
    for (int a = 0; a < M; ++a) {
      const double ca = mo.occ * c[a];
      if (ca == 0.0) continue;
      double* row = f->D.data() + (size_t)a * M;
      for (int b = 0; b < M; ++b) row[b] += ca * c[b];
    }
  }
  f->nalpha = (int32_t)std::lround(na);
  f->nbeta = (int32_t)std::lround(nb);
  *out = f;
  return CTC_OK;
}

int ctc_molecule_create_from_file(const char* path, ctc_molecule** out) {
  if (!path || !out) return fail(CTC_ERR_INVALID, "ctc_molecule_create_from_file: null argument");
  *out = nullptr;
  const std::string p = lower(path);
  auto ends = [&](const std::string& s) { return p.size() >= s.size() && p.compare(p.size() - s.size(), s.size(), s) == 0; };
  const bool molden = ends(".molden") || ends(".molden.input") || ends(".mold");
  const bool wfn = ends(".wfn") || ends(".wfx");
  ctc_fchk* f = nullptr;
  int rc = molden ? ctc_molden_load(path, &f) : wfn ? ctc_wfn_load(path, &f) : ctc_fchk_load(path, &f);
  if (rc != CTC_OK) return rc;
  ctc_fchk_view v;
  ctc_fchk_view_get(f, &v);
  rc = ctc_molecule_create(&v.basis, v.natom, v.atom_xyz, v.atom_charges, v.density, v.nbasis, out);
  ctc_fchk_destroy(f);
  return rc;
}

}  // extern "C"
