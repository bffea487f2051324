// ctc_fchk.cpp -- native reader of Gaussian formatted checkpoint (.fchk) files.
//
// Replaces the reference's route through the Python iodata package
// (src/iodata.cpp:15-211, chemtools::get_molecular_basis_from_fchk, used by
// Molecule(str) at src/pymolecule.cu:18-23): the basis, the atoms and the
// one-particle density matrix are read directly from the text sections of the
// file, with no Python in the loop.
//
// Conventions taken from the file as Gaussian writes it:
//   * "Shell types": 0 s, 1 p, -1 sp (one shell, an s and a p contraction with
//     shared exponents; the p coefficients are "P(S=P) Contraction
//     coefficients"), +-2 d, +-3 f, +-4 g with negative = pure (spherical);
//     the same codes as ctc_basis.angmoms;
//   * basis functions within a shell in Gaussian's order, which is the order
//     of the reference's AO kernels (src/evaluate_density.cu:80-314);
//   * contraction coefficients multiply normalised primitives;
//   * "Alpha/Beta MO coefficients": MO-major, nbasis coefficients per orbital.
// The density matrix is the MO one-particle density matrix, as the reference
// builds it from iodata (src/iodata.cpp:157-160, (C occ) C^T): restricted
// files (no beta orbitals) occupy the first n_beta orbitals twice and the next
// n_alpha - n_beta once; unrestricted files sum the alpha and beta
// projectors over their occupied orbitals.
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "ctc_internal.h"
#include "ctc_wfnfile.h"

using namespace ctc;


namespace {

struct Section {
  char type = 0;  // 'I', 'R', 'C', 'L'
  bool array = false;
  std::vector<double> real;
  std::vector<long long> ints;
};

// Reads every section of the file; scalar sections keep one value.
int parse(const std::string& path, std::map<std::string, Section>& out) {
  std::ifstream in(path);
  if (!in) return fail(CTC_ERR_INVALID, "fchk: cannot open '" + path + "'");
  std::string line;
  int lineno = 0;
  // the first two lines are the title and the job/method/basis line
  for (int i = 0; i < 2 && std::getline(in, line); ++i) ++lineno;
  while (std::getline(in, line)) {
    ++lineno;
    if (line.size() < 45 || std::isspace((unsigned char)line[0])) continue;
    std::string label = line.substr(0, 43);
    while (!label.empty() && label.back() == ' ') label.pop_back();
    const char type = line[43];
    if (type != 'I' && type != 'R' && type != 'C' && type != 'L') continue;
    Section sec;
    sec.type = type;
    const std::string rest = line.substr(44);
    const size_t npos = rest.find("N=");
    if (npos == std::string::npos) {
      std::istringstream ss(rest);
      if (type == 'R') {
        double v;
        if (ss >> v) sec.real.push_back(v);
      } else if (type == 'I') {
        long long v;
        if (ss >> v) sec.ints.push_back(v);
      }
      out[label] = std::move(sec);
      continue;
    }
    sec.array = true;
    const long long count = std::atoll(rest.c_str() + npos + 2);
    if (count < 0) return fail(CTC_ERR_INVALID, "fchk: bad count at line " + std::to_string(lineno));
    if (type == 'C' || type == 'L') continue;  // not needed; their data lines start with blanks
    long long got = 0;
    while (got < count && std::getline(in, line)) {
      ++lineno;
      std::istringstream ss(line);
      if (type == 'R') {
        std::string tok;
        while (got < count && ss >> tok) {
          // Fortran may write exponents as D; strtod expects E
          for (char& c : tok)
            if (c == 'D' || c == 'd') c = 'E';
          sec.real.push_back(std::strtod(tok.c_str(), nullptr));
          ++got;
        }
      } else {
        long long v;
        while (got < count && ss >> v) {
          sec.ints.push_back(v);
          ++got;
        }
      }
    }
    if (got != count)
      return fail(CTC_ERR_INVALID, "fchk: section '" + label + "' ends early (" + std::to_string(got) +
                                       " of " + std::to_string(count) + " values)");
    out[label] = std::move(sec);
  }
  return CTC_OK;
}

int ncomp(int t) {
  const int l = t < 0 ? -t : t;
  return t < 0 ? 2 * l + 1 : (l + 1) * (l + 2) / 2;
}

}  // namespace

extern "C" {

int ctc_fchk_load(const char* path, ctc_fchk** out) {
  if (!path || !out) return fail(CTC_ERR_INVALID, "ctc_fchk_load: null argument");
  *out = nullptr;
  std::map<std::string, Section> s;
  int rc = parse(path, s);
  if (rc != CTC_OK) return rc;
  auto need = [&](const char* name, char type, bool array) -> const Section* {
    auto it = s.find(name);
    if (it == s.end() || it->second.type != type || it->second.array != array) return nullptr;
    return &it->second;
  };
  const char* required[] = {"Number of atoms", "Number of basis functions", "Number of alpha electrons",
                            "Number of beta electrons"};
  for (const char* r : required)
    if (!need(r, 'I', false) || need(r, 'I', false)->ints.empty())
      return fail(CTC_ERR_INVALID, std::string("fchk: missing '") + r + "'");
  auto* f = new ctc_fchk();
  f->path = path;
  f->natom = (int32_t)need("Number of atoms", 'I', false)->ints[0];
  f->nbasis = (int32_t)need("Number of basis functions", 'I', false)->ints[0];
  f->nalpha = (int32_t)need("Number of alpha electrons", 'I', false)->ints[0];
  f->nbeta = (int32_t)need("Number of beta electrons", 'I', false)->ints[0];
  auto bad = [&](const std::string& msg) {
    delete f;
    return fail(CTC_ERR_INVALID, "fchk: " + msg);
  };
  const Section* an = need("Atomic numbers", 'I', true);
  const Section* nc = need("Nuclear charges", 'R', true);
  const Section* xyz = need("Current cartesian coordinates", 'R', true);
  const Section* st = need("Shell types", 'I', true);
  const Section* np = need("Number of primitives per shell", 'I', true);
  const Section* sa = need("Shell to atom map", 'I', true);
  const Section* pe = need("Primitive exponents", 'R', true);
  const Section* cc = need("Contraction coefficients", 'R', true);
  const Section* sp = need("P(S=P) Contraction coefficients", 'R', true);
  const Section* sc = need("Coordinates of each shell", 'R', true);
  const Section* ca = need("Alpha MO coefficients", 'R', true);
  const Section* cb = need("Beta MO coefficients", 'R', true);
  if (!an || !xyz || !st || !np || !sa || !pe || !cc || !sc || !ca)
    return bad("a basis, atom or orbital section is missing");
  if ((int)an->ints.size() != f->natom || (int)xyz->real.size() != 3 * f->natom)
    return bad("atom sections do not match 'Number of atoms'");
  const size_t nshell = st->ints.size();
  if (np->ints.size() != nshell || sa->ints.size() != nshell || sc->real.size() != 3 * nshell)
    return bad("shell sections differ in length");
  f->numbers.assign(an->ints.begin(), an->ints.end());
  f->charges = nc ? nc->real : std::vector<double>(f->numbers.begin(), f->numbers.end());
  f->coords = xyz->real;
  size_t ip = 0;
  int nfun = 0;
  for (size_t i = 0; i < nshell; ++i) {
    const int t = (int)st->ints[i];
    const int K = (int)np->ints[i];
    if (K <= 0 || ip + K > pe->real.size() || ip + K > cc->real.size()) return bad("primitive counts exceed the data");
    if (t < -4 || t > 4) return bad("shell type " + std::to_string(t) + " is not supported (s..g)");
    const int atom = (int)sa->ints[i] - 1;
    if (atom < 0 || atom >= f->natom) return bad("shell to atom map out of range");
    for (int d = 0; d < 3; ++d) f->centers.push_back(sc->real[3 * i + d]);
    f->shell_atom.push_back(atom);
    f->nprim.push_back(K);
    f->exps.insert(f->exps.end(), pe->real.begin() + ip, pe->real.begin() + ip + K);
    if (t == -1) {
      if (!sp || ip + K > sp->real.size()) return bad("sp shell without P(S=P) coefficients");
      f->nseg.push_back(2);
      f->angmoms.push_back(0);
      f->angmoms.push_back(1);
      f->coeffs.insert(f->coeffs.end(), cc->real.begin() + ip, cc->real.begin() + ip + K);
      f->coeffs.insert(f->coeffs.end(), sp->real.begin() + ip, sp->real.begin() + ip + K);
      nfun += 4;
    } else {
      f->nseg.push_back(1);
      f->angmoms.push_back(t);
      f->coeffs.insert(f->coeffs.end(), cc->real.begin() + ip, cc->real.begin() + ip + K);
      nfun += ncomp(t);
    }
    ip += K;
  }
  if (nfun != f->nbasis)
    return bad("shells give " + std::to_string(nfun) + " functions, the file declares " +
               std::to_string(f->nbasis));
  // MO one-particle density matrix
  const int M = f->nbasis;
  if (ca->real.size() % M != 0) return bad("alpha MO coefficients are not a multiple of the basis size");
  const int nmo = (int)(ca->real.size() / M);
  f->D.assign((size_t)M * M, 0.0);
  auto add = [&](const std::vector<double>& C, int nocc, double occ) {
    if (nocc > nmo) nocc = nmo;
    for (int i = 0; i < nocc; ++i) {
      const double* c = C.data() + (size_t)i * M;
      for (int a = 0; a < M; ++a) {
        const double ca_ = occ * c[a];
        if (ca_ == 0.0) continue;
        double* row = f->D.data() + (size_t)a * M;
        for (int b = 0; b < M; ++b) row[b] += ca_ * c[b];
      }
    }
  };
  if (cb) {
    if (cb->real.size() != ca->real.size()) return bad("alpha and beta MO coefficients differ in size");
    add(ca->real, f->nalpha, 1.0);
    add(cb->real, f->nbeta, 1.0);
  } else {
    const int nd = f->nbeta < f->nalpha ? f->nbeta : f->nalpha;
    add(ca->real, nd, 2.0);
    // singly occupied orbitals of a restricted open-shell wavefunction
    std::vector<double> rest(ca->real.begin() + (size_t)nd * M, ca->real.end());
    const int ns = (f->nalpha > f->nbeta ? f->nalpha - f->nbeta : f->nbeta - f->nalpha);
    add(rest, ns, 1.0);
  }
  *out = f;
  return CTC_OK;
}

int ctc_fchk_view_get(const ctc_fchk* f, ctc_fchk_view* v) {
  if (!f || !v) return fail(CTC_ERR_INVALID, "ctc_fchk_view_get: null argument");
  v->basis.nshell = (int32_t)f->nprim.size();
  v->basis.centers = f->centers.data();
  v->basis.shell_atom = f->shell_atom.data();
  v->basis.nprim = f->nprim.data();
  v->basis.nseg = f->nseg.data();
  v->basis.angmoms = f->angmoms.data();
  v->basis.exps = f->exps.data();
  v->basis.coeffs = f->coeffs.data();
  v->natom = f->natom;
  v->atom_xyz = f->coords.data();
  v->atom_charges = f->charges.data();
  v->atomic_numbers = f->numbers.data();
  v->nbasis = f->nbasis;
  v->nalpha = f->nalpha;
  v->nbeta = f->nbeta;
  v->density = f->D.data();
  return CTC_OK;
}

void ctc_fchk_destroy(ctc_fchk* f) { delete f; }

int ctc_molecule_create_from_fchk(const char* path, ctc_molecule** out) {
  if (!out) return fail(CTC_ERR_INVALID, "ctc_molecule_create_from_fchk: null argument");
  *out = nullptr;
  ctc_fchk* f = nullptr;
  int rc = ctc_fchk_load(path, &f);
  if (rc != CTC_OK) return rc;
  ctc_fchk_view v;
  ctc_fchk_view_get(f, &v);
  rc = ctc_molecule_create(&v.basis, v.natom, v.atom_xyz, v.atom_charges, v.density, v.nbasis, out);
  ctc_fchk_destroy(f);
  return rc;
}

}  // extern "C"
