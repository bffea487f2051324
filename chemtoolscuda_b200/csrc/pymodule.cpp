// pymodule.cpp -- pybind11 module `_chemtools_cuda`: the chemtools_cuda.Molecule API.
//
// Mirrors the reference's Python surface (src/pybind.cpp:9-305): every bound
// method name is kept, plus the names the reference's README and tests use
// (compute_electron_density, ..._gradient, ..._hessian,
// compute_laplacian_electron_density, compute_electron_density_on_cubic_grid)
// and basis_set_to_constant_memory.  Points are numpy (N, 3) float64 arrays;
// results come back as fresh numpy arrays of the reference's shapes.  All work
// goes through the C ABI of include/chemtools_cuda.h with the GIL released.
#include <cctype>
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cstdint>
#include <initializer_list>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/chemtools_cuda.h"

namespace py = pybind11;
using arr = py::array_t<double, py::array::c_style | py::array::forcecast>;
using iarr = py::array_t<int32_t, py::array::c_style | py::array::forcecast>;

namespace {

void check(int rc, const char* what) {
  if (rc == CTC_OK) return;
  std::string msg = std::string(what) + ": " + ctc_last_error();
  if (rc == CTC_ERR_INVALID) throw py::value_error(msg);
  if (rc == CTC_ERR_UNSUPPORTED) throw std::runtime_error(msg);
  throw std::runtime_error(msg);
}

int parse_precision(const std::string& p) {
  if (p == "fp64" || p == "FP64" || p == "double") return CTC_PREC_FP64;
  if (p == "tc" || p == "TC" || p == "tc_split" || p == "split") return CTC_PREC_TC_SPLIT;
  throw py::value_error("precision must be 'fp64' or 'tc' (got '" + p + "')");
}

arr points_arg(const arr& pts) {
  if (pts.ndim() != 2 || pts.shape(1) != 3) throw py::value_error("points must have shape (N, 3)");
  return pts;
}

const char* kKeys[12] = {"rho", "grad", "hess", "lap", "tau_pd", "tau_alpha",
                         "rdg", "shannon", "weizsacker", "thomas_fermi", "gge", "general_ked"};

double** slot(ctc_outputs& o, int i) {
  double** s[12] = {&o.rho, &o.grad, &o.hess, &o.lap, &o.tau_pd, &o.tau_alpha,
                    &o.rdg, &o.shannon, &o.weizsacker, &o.thomas_fermi, &o.gge, &o.general_ked};
  return s[i];
}

int key_index(const std::string& k) {
  for (int i = 0; i < 12; ++i)
    if (k == kKeys[i]) return i;
  throw py::value_error("unknown descriptor '" + k + "'");
}

class Molecule {
 public:
  Molecule(ctc_molecule* h, arr coords, iarr numbers, std::string path)
      : h_(h), coords_(std::move(coords)), numbers_(std::move(numbers)), path_(std::move(path)) {}
  ~Molecule() {
    if (h_) ctc_molecule_destroy(h_);
  }
  Molecule(const Molecule&) = delete;
  Molecule& operator=(const Molecule&) = delete;

  static std::unique_ptr<Molecule> from_arrays(arr centers, py::object shell_atom, iarr nprim,
                                               iarr nseg, iarr angmoms, arr exps, arr coeffs,
                                               arr coords, arr charges, arr D, py::object numbers,
                                               std::string path) {
    if (D.ndim() != 2 || D.shape(0) != D.shape(1)) throw py::value_error("D must be square");
    if (coords.ndim() != 2 || coords.shape(1) != 3) throw py::value_error("coords must be (natom, 3)");
    int natom = (int)coords.shape(0);
    if (charges.size() != natom) throw py::value_error("charges must have one entry per atom");
    if (centers.ndim() != 2 || centers.shape(1) != 3) throw py::value_error("centers must be (nshell, 3)");
    int nshell = (int)centers.shape(0);
    if (nprim.size() != nshell || nseg.size() != nshell)
      throw py::value_error("nprim and nseg need one entry per shell");
    iarr sa;
    const int32_t* sa_ptr = nullptr;
    if (!shell_atom.is_none()) {
      sa = shell_atom.cast<iarr>();
      if (sa.size() != nshell) throw py::value_error("shell_atom needs one entry per shell");
      sa_ptr = sa.data();
    }
    ctc_basis b{nshell, centers.data(), sa_ptr, nprim.data(), nseg.data(), angmoms.data(),
                exps.data(), coeffs.data()};
    ctc_molecule* h = nullptr;
    {
      py::gil_scoped_release rel;
      check(ctc_molecule_create(&b, natom, coords.data(), charges.data(), D.data(),
                                (int32_t)D.shape(0), &h),
            "Molecule");
    }
    iarr nums;
    if (numbers.is_none()) {
      nums = iarr(natom);
      for (int a = 0; a < natom; ++a) nums.mutable_data()[a] = (int32_t)charges.data()[a];
    } else {
      nums = numbers.cast<iarr>();
    }
    return std::make_unique<Molecule>(h, arr(coords), nums, path);
  }

  // Molecule(path): a Gaussian formatted checkpoint file, a Molden file
  // (.molden, .molden.input, .mold) or an AIM wavefunction file (.wfn, .wfx),
  // read by the library's native readers (the reference's Molecule(str),
  // src/pybind.cpp:15, loads them through the Python iodata package).
  static bool has_ext(std::string p, std::initializer_list<const char*> exts) {
    for (char& c : p) c = (char)std::tolower((unsigned char)c);
    for (const char* e : exts) {
      const std::string s(e);
      if (p.size() >= s.size() && p.compare(p.size() - s.size(), s.size(), s) == 0) return true;
    }
    return false;
  }
  static std::unique_ptr<Molecule> from_fchk(const std::string& path) {
    ctc_fchk* f = nullptr;
    check(has_ext(path, {".molden", ".molden.input", ".mold"}) ? ctc_molden_load(path.c_str(), &f)
          : has_ext(path, {".wfn", ".wfx"})                     ? ctc_wfn_load(path.c_str(), &f)
                                                                : ctc_fchk_load(path.c_str(), &f),
          "Molecule");
    ctc_fchk_view v;
    ctc_fchk_view_get(f, &v);
    ctc_molecule* h = nullptr;
    int rc;
    {
      py::gil_scoped_release rel;
      rc = ctc_molecule_create(&v.basis, v.natom, v.atom_xyz, v.atom_charges, v.density, v.nbasis, &h);
    }
    arr coords({(py::ssize_t)v.natom, (py::ssize_t)3});
    iarr nums((py::ssize_t)v.natom);
    for (int a = 0; a < v.natom; ++a) {
      for (int d = 0; d < 3; ++d) coords.mutable_data()[3 * a + d] = v.atom_xyz[3 * a + d];
      nums.mutable_data()[a] = v.atomic_numbers[a];
    }
    ctc_fchk_destroy(f);
    check(rc, "Molecule");
    return std::make_unique<Molecule>(h, coords, nums, path);
  }

  // ---- generic evaluation (host arrays) ----
  py::dict local(const arr& pts_in, const std::vector<std::string>& keys, const std::string& prec,
                 double alpha, double gge_a, double gge_b, double ked_a) {
    arr pts = points_arg(pts_in);
    const py::ssize_t n = pts.shape(0);
    ctc_outputs o{};
    py::dict res;
    std::vector<arr> keep;
    for (const std::string& k : keys) {
      int i = key_index(k);
      arr a;
      if (i == 1) a = arr({n, (py::ssize_t)3});
      else if (i == 2) a = arr({n, (py::ssize_t)3, (py::ssize_t)3});
      else a = arr({n});
      *slot(o, i) = a.mutable_data();
      res[py::str(k)] = a;
      keep.push_back(a);
    }
    ctc_params p{alpha, gge_a, gge_b, ked_a};
    int pr = parse_precision(prec);
    {
      py::gil_scoped_release rel;
      check(ctc_eval_local_host(h_, pts.data(), n, pr, &p, &o), "compute_local_descriptors");
    }
    return res;
  }

  arr one(const arr& pts, const char* key, const std::string& prec, double alpha = 0.0,
          double gge_a = 0.0, double gge_b = 0.0, double ked_a = 1.0) {
    py::dict d = local(pts, {key}, prec, alpha, gge_a, gge_b, ked_a);
    return d[key].cast<arr>();
  }

  arr esp(const arr& pts_in) {
    arr pts = points_arg(pts_in);
    const py::ssize_t n = pts.shape(0);
    arr out({n});
    {
      py::gil_scoped_release rel;
      check(ctc_eval_esp_host(h_, pts.data(), n, out.mutable_data()), "compute_electrostatic_potential");
    }
    return out;
  }

  arr cubic(const arr& origin, const arr& axes, const iarr& shape, bool disp, const std::string& prec) {
    (void)disp;
    if (origin.size() != 3 || axes.size() != 9 || shape.size() != 3)
      throw py::value_error("origin (3,), axes (3,3) and shape (3,) expected");
    const int32_t* s = shape.data();
    const int64_t n = (int64_t)s[0] * s[1] * s[2];
    arr out({(py::ssize_t)s[0], (py::ssize_t)s[1], (py::ssize_t)s[2]});
    if (n == 0) return out;
    double* d = nullptr;
    {
      py::gil_scoped_release rel;
      if (cudaMallocWrap(&d, n) != 0) throw std::runtime_error("cubic grid: device allocation failed");
      ctc_outputs o{};
      o.rho = d;
      int rc = ctc_eval_cubic(h_, origin.data(), axes.data(), s, parse_precision(prec), nullptr, &o, nullptr);
      int rc2 = rc == CTC_OK ? copyBack(out.mutable_data(), d, n) : 0;
      cudaFreeWrap(d);
      check(rc, "compute_electron_density_on_cubic_grid");
      if (rc2 != 0) throw std::runtime_error("cubic grid: copy back failed");
    }
    return out;
  }

  arr norm(const arr& v) {
    if (v.ndim() != 2 || v.shape(1) != 3) throw py::value_error("array must have shape (N, 3)");
    const py::ssize_t n = v.shape(0);
    arr out({n});
    const double* a = v.data();
    double* o = out.mutable_data();
    for (py::ssize_t i = 0; i < n; ++i)
      o[i] = std::sqrt(a[3 * i] * a[3 * i] + a[3 * i + 1] * a[3 * i + 1] + a[3 * i + 2] * a[3 * i + 2]);
    return out;
  }

  void prepare(bool do_segmented_basis, const std::string& prec) {
    (void)do_segmented_basis;
    py::gil_scoped_release rel;
    check(ctc_molecule_prepare(h_, parse_precision(prec)), "basis_set_to_constant_memory");
  }

  // ---- device pointers (used by the torch layer and the benchmark) ----
  void local_device(uintptr_t pts, int64_t n, const std::string& prec, py::dict ptrs, double alpha,
                    double gge_a, double gge_b, double ked_a, uintptr_t stream) {
    ctc_outputs o{};
    for (auto item : ptrs) *slot(o, key_index(item.first.cast<std::string>())) = (double*)item.second.cast<uintptr_t>();
    ctc_params p{alpha, gge_a, gge_b, ked_a};
    int pr = parse_precision(prec);
    py::gil_scoped_release rel;
    check(ctc_eval_local(h_, (const double*)pts, n, pr, &p, &o, (void*)stream), "eval_local_device");
  }
  void cubic_device(const arr& origin, const arr& axes, const iarr& shape, const std::string& prec,
                    py::dict ptrs, double alpha, double gge_a, double gge_b, double ked_a,
                    uintptr_t stream) {
    if (origin.size() != 3 || axes.size() != 9 || shape.size() != 3)
      throw py::value_error("origin (3), axes (3, 3) and shape (3) expected");
    ctc_outputs o{};
    for (auto item : ptrs) *slot(o, key_index(item.first.cast<std::string>())) = (double*)item.second.cast<uintptr_t>();
    ctc_params p{alpha, gge_a, gge_b, ked_a};
    int pr = parse_precision(prec);
    py::gil_scoped_release rel;
    check(ctc_eval_cubic(h_, origin.data(), axes.data(), shape.data(), pr, &p, &o, (void*)stream),
          "eval_cubic_device");
  }
  void esp_device(uintptr_t pts, int64_t n, uintptr_t out, uintptr_t stream) {
    py::gil_scoped_release rel;
    check(ctc_eval_esp(h_, (const double*)pts, n, (double*)out, (void*)stream), "eval_esp_device");
  }
  void ao_device(uintptr_t pts, int64_t n, int deriv, uintptr_t out, uintptr_t stream) {
    py::gil_scoped_release rel;
    check(ctc_eval_ao(h_, (const double*)pts, n, deriv, (double*)out, (void*)stream), "eval_ao_device");
  }
  void adjoint_device(uintptr_t pts, int64_t n, uintptr_t v_rho, uintptr_t v_grad, uintptr_t dLdD,
                      uintptr_t dLdR, uintptr_t stream) {
    py::gil_scoped_release rel;
    check(ctc_adjoint(h_, (const double*)pts, n, (const double*)v_rho, (const double*)v_grad,
                      (double*)dLdD, (double*)dLdR, (void*)stream),
          "adjoint_device");
  }
  void set_density_matrix_device(uintptr_t D, uintptr_t stream) {
    py::gil_scoped_release rel;
    check(ctc_molecule_set_density_matrix(h_, (const double*)D, (void*)stream), "set_density_matrix");
  }
  void set_coordinates(const arr& xyz) {
    if (xyz.ndim() != 2 || xyz.shape(1) != 3 || xyz.shape(0) != coords_.shape(0))
      throw py::value_error("coordinates must be (natom, 3)");
    check(ctc_molecule_set_coordinates(h_, xyz.data()), "set_coordinates");
    arr c({xyz.shape(0), (py::ssize_t)3});
    std::copy(xyz.data(), xyz.data() + xyz.size(), c.mutable_data());
    coords_ = c;
  }

  arr coordinates() const { return coords_; }
  iarr numbers() const { return numbers_; }
  int nbasis() const { return ctc_molecule_nbasis(h_); }
  int natom() const { return ctc_molecule_natom(h_); }
  const std::string& path() const { return path_; }
  uintptr_t handle() const { return (uintptr_t)h_; }

 private:
  static int cudaMallocWrap(double** p, int64_t n);
  static void cudaFreeWrap(double* p);
  static int copyBack(double* h, const double* d, int64_t n);
  ctc_molecule* h_ = nullptr;
  arr coords_;
  iarr numbers_;
  std::string path_;
};

}  // namespace

// small CUDA runtime helpers (kept out of the class body to keep cuda headers local)
#include <cuda_runtime.h>
int Molecule::cudaMallocWrap(double** p, int64_t n) {
  return cudaMalloc((void**)p, sizeof(double) * n) == cudaSuccess ? 0 : -1;
}
void Molecule::cudaFreeWrap(double* p) { cudaFree(p); }
int Molecule::copyBack(double* h, const double* d, int64_t n) {
  return cudaMemcpy(h, d, sizeof(double) * n, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -1;
}

PYBIND11_MODULE(_chemtools_cuda, m) {
  m.doc() = "B200-native grid evaluation of Gaussian-basis density descriptors (chemtools_cuda API).";
  m.attr("CTC_PREC_FP64") = CTC_PREC_FP64;
  m.attr("CTC_PREC_TC_SPLIT") = CTC_PREC_TC_SPLIT;
  m.def("version", []() { return std::string(ctc_version()); });
  m.def("last_error", []() { return std::string(ctc_last_error()); });

  py::class_<Molecule>(m, "Molecule")
      .def(py::init(&Molecule::from_fchk), py::arg("file_path"),
           "Molecule from a Gaussian formatted checkpoint (.fchk), Molden (.molden) or AIM (.wfn, .wfx) file.")
      .def_static("from_fchk", &Molecule::from_fchk, py::arg("file_path"))
      .def_static("from_arrays", &Molecule::from_arrays, py::arg("centers"), py::arg("shell_atom"),
                  py::arg("nprim"), py::arg("nseg"), py::arg("angmoms"), py::arg("exps"),
                  py::arg("coeffs"), py::arg("coords"), py::arg("charges"), py::arg("D"),
                  py::arg("numbers") = py::none(), py::arg("path") = std::string())
      .def("compute_local_descriptors", &Molecule::local, py::arg("points"), py::arg("keys"),
           py::arg("precision") = "fp64", py::arg("alpha") = 0.0, py::arg("gge_a") = 1.0 / 9.0,
           py::arg("gge_b") = 1.0 / 6.0, py::arg("ked_a") = 1.0,
           "All requested local descriptors from one fused pass: dict key -> array.")
      .def("compute_density", [](Molecule& s, const arr& p, const std::string& pr) { return s.one(p, "rho", pr); },
           py::arg("points"), py::arg("precision") = "fp64", "Electron density rho (N,).")
      .def("compute_electron_density", [](Molecule& s, const arr& p, const std::string& pr) { return s.one(p, "rho", pr); },
           py::arg("points"), py::arg("precision") = "fp64")
      .def("compute_gradient", [](Molecule& s, const arr& p, const std::string& pr) { return s.one(p, "grad", pr); },
           py::arg("points"), py::arg("precision") = "fp64", "Gradient of rho (N, 3).")
      .def("compute_electron_density_gradient", [](Molecule& s, const arr& p, const std::string& pr) { return s.one(p, "grad", pr); },
           py::arg("points"), py::arg("precision") = "fp64")
      .def("compute_hessian", [](Molecule& s, const arr& p, const std::string& pr) { return s.one(p, "hess", pr); },
           py::arg("points"), py::arg("precision") = "fp64", "Hessian of rho (N, 3, 3).")
      .def("compute_electron_density_hessian", [](Molecule& s, const arr& p, const std::string& pr) { return s.one(p, "hess", pr); },
           py::arg("points"), py::arg("precision") = "fp64")
      .def("compute_laplacian", [](Molecule& s, const arr& p, const std::string& pr) { return s.one(p, "lap", pr); },
           py::arg("points"), py::arg("precision") = "fp64", "Laplacian of rho (N,).")
      .def("compute_laplacian_electron_density", [](Molecule& s, const arr& p, const std::string& pr) { return s.one(p, "lap", pr); },
           py::arg("points"), py::arg("precision") = "fp64")
      .def("compute_positive_definite_kinetic_energy_density",
           [](Molecule& s, const arr& p, const std::string& pr) { return s.one(p, "tau_pd", pr); },
           py::arg("points"), py::arg("precision") = "fp64")
      .def("compute_general_kinetic_energy_density",
           [](Molecule& s, const arr& p, double alpha, const std::string& pr) { return s.one(p, "tau_alpha", pr, alpha); },
           py::arg("points"), py::arg("alpha"), py::arg("precision") = "fp64",
           "tau_alpha = tau_PD + alpha * lap (the documented definition).")
      .def("compute_norm_of_vector", &Molecule::norm, py::arg("array"))
      .def("compute_reduced_density_gradient",
           [](Molecule& s, const arr& p, const std::string& pr) { return s.one(p, "rdg", pr); },
           py::arg("points"), py::arg("precision") = "fp64")
      .def("compute_weizsacker_ked", [](Molecule& s, const arr& p, const std::string& pr) { return s.one(p, "weizsacker", pr); },
           py::arg("points"), py::arg("precision") = "fp64")
      .def("compute_thomas_fermi_ked", [](Molecule& s, const arr& p, const std::string& pr) { return s.one(p, "thomas_fermi", pr); },
           py::arg("points"), py::arg("precision") = "fp64")
      .def("compute_general_gradient_expansion_ked",
           [](Molecule& s, const arr& p, double a, double b, const std::string& pr) { return s.one(p, "gge", pr, 0.0, a, b); },
           py::arg("points"), py::arg("a"), py::arg("b"), py::arg("precision") = "fp64")
      .def("compute_gradient_expansion_ked",
           [](Molecule& s, const arr& p, const std::string& pr) { return s.one(p, "gge", pr, 0.0, 1.0 / 9.0, 1.0 / 6.0); },
           py::arg("points"), py::arg("precision") = "fp64")
      .def("compute_empirical_gradient_expansion_ked",
           [](Molecule& s, const arr& p, const std::string& pr) { return s.one(p, "gge", pr, 0.0, 1.0 / 5.0, 1.0 / 6.0); },
           py::arg("points"), py::arg("precision") = "fp64")
      .def("compute_general_ked",
           [](Molecule& s, const arr& p, double a, const std::string& pr) { return s.one(p, "general_ked", pr, 0.0, 0.0, 0.0, a); },
           py::arg("points"), py::arg("a"), py::arg("precision") = "fp64",
           "tau_PD + (a - 1)/4 * lap.")
      .def("compute_schrodinger_ked",
           [](Molecule& s, const arr& p, const std::string& pr) { return s.one(p, "general_ked", pr, 0.0, 0.0, 0.0, 0.0); },
           py::arg("points"), py::arg("precision") = "fp64")
      .def("compute_shannon_information_density",
           [](Molecule& s, const arr& p, const std::string& pr) { return s.one(p, "shannon", pr); },
           py::arg("points"), py::arg("precision") = "fp64")
      .def("compute_electrostatic_potential", &Molecule::esp, py::arg("points"))
      .def("compute_electron_density_on_cubic_grid", &Molecule::cubic, py::arg("origin"),
           py::arg("axes"), py::arg("shape"), py::arg("disp") = false, py::arg("precision") = "fp64")
      .def("compute_electron_density_cubic", &Molecule::cubic, py::arg("origin"), py::arg("axes"),
           py::arg("shape"), py::arg("disp") = false, py::arg("precision") = "fp64")
      .def("basis_set_to_constant_memory", &Molecule::prepare, py::arg("do_segmented_basis") = false,
           py::arg("precision") = "fp64",
           "Make the device tables resident (idempotent; the argument is accepted and ignored).")
      .def("eval_local_device", &Molecule::local_device, py::arg("points_ptr"), py::arg("n"),
           py::arg("precision"), py::arg("ptrs"), py::arg("alpha") = 0.0, py::arg("gge_a") = 1.0 / 9.0,
           py::arg("gge_b") = 1.0 / 6.0, py::arg("ked_a") = 1.0, py::arg("stream") = 0)
      .def("eval_cubic_device", &Molecule::cubic_device, py::arg("origin"), py::arg("axes"),
           py::arg("shape"), py::arg("precision"), py::arg("ptrs"), py::arg("alpha") = 0.0,
           py::arg("gge_a") = 1.0 / 9.0, py::arg("gge_b") = 1.0 / 6.0, py::arg("ked_a") = 1.0,
           py::arg("stream") = 0)
      .def("eval_esp_device", &Molecule::esp_device, py::arg("points_ptr"), py::arg("n"),
           py::arg("out_ptr"), py::arg("stream") = 0)
      .def("eval_ao_device", &Molecule::ao_device, py::arg("points_ptr"), py::arg("n"),
           py::arg("deriv"), py::arg("out_ptr"), py::arg("stream") = 0)
      .def("adjoint_device", &Molecule::adjoint_device, py::arg("points_ptr"), py::arg("n"),
           py::arg("v_rho_ptr"), py::arg("v_grad_ptr"), py::arg("dLdD_ptr"), py::arg("dLdR_ptr"),
           py::arg("stream") = 0)
      .def("set_density_matrix_device", &Molecule::set_density_matrix_device, py::arg("D_ptr"),
           py::arg("stream") = 0)
      .def("set_coordinates", &Molecule::set_coordinates, py::arg("coords"))
      .def_property_readonly("coordinates", &Molecule::coordinates)
      .def_property_readonly("numbers", &Molecule::numbers)
      .def_property_readonly("nbasis", &Molecule::nbasis)
      .def_property_readonly("natom", &Molecule::natom)
      .def_property_readonly("handle", &Molecule::handle)
      .def("get_file_path", &Molecule::path);
}
