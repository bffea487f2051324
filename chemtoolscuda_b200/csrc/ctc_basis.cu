// ctc_basis.cu -- molecule handle: basis tables, density matrix, scratch, errors.
//
// The reference packs its basis into a 60 KB __constant__ array before every
// kernel launch, one constant-memory-sized chunk of shells at a time
// (src/basis_to_gpu.cu:13-220).  Here a molecule handle owns its tables in
// global memory, built once: one 56-byte record per segmented shell (centre,
// screening radius, type, primitive range, first AO), primitive exponents and
// coefficients with the radial normalisation N_l(a) = (2a/pi)^(3/4) (4a)^(l/2)
// folded in (src/cuda_basis_utils.cu:7-109), and the AO -> atom map used by
// the adjoint.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <tuple>

#include "ctc_internal.h"

namespace ctc {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

// Kernel attributes are per device: a kernel launched on a second GPU needs its
// own cudaFuncSetAttribute.  One entry per (device, kernel, bytes) that has
// been configured, under a mutex so that host threads may call in together.
namespace {
std::mutex g_attr_mu;
std::vector<std::tuple<int, const void*, int>> g_attr_done;
std::mutex g_sm_mu;
std::vector<std::pair<int, int>> g_sm_count;  // (device, SM count)
}  // namespace

// d_D (Mpad x Mpad, internal AO order, zero padded) from a caller's D
// (M x M, caller's order): d_D[i][j] = D[perm[i]][perm[j]].
__global__ void permute_density_kernel(const double* __restrict__ D, int M, int Mpad,
                                       const int32_t* __restrict__ perm, double* __restrict__ out) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)Mpad * Mpad) return;
  const int i = (int)(e / Mpad), j = (int)(e % Mpad);
  out[e] = (i < M && j < M) ? D[(int64_t)perm[i] * M + perm[j]] : 0.0;
}

int refresh_host_density(ctc_molecule* m) {
  if (!m->host_D_stale) return CTC_OK;
  const int M = m->M, Mp = m->Mpad;
  std::vector<double> pad((size_t)Mp * Mp);
  CTC_CUDA_TRY(cudaDeviceSynchronize());
  CTC_CUDA_TRY(cudaMemcpy(pad.data(), m->d_D, sizeof(double) * pad.size(), cudaMemcpyDeviceToHost));
  for (int i = 0; i < M; ++i)
    std::memcpy(&m->D[(size_t)i * M], &pad[(size_t)i * Mp], sizeof(double) * M);
  m->host_D_stale = false;
  return CTC_OK;
}

int ensure_smem_attr(const void* kernel, int bytes) {
  int dev = 0;
  CTC_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(g_attr_mu);
  const auto key = std::make_tuple(dev, kernel, bytes);
  if (std::find(g_attr_done.begin(), g_attr_done.end(), key) != g_attr_done.end()) return CTC_OK;
  CTC_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  g_attr_done.push_back(key);
  return CTC_OK;
}

int device_sm_count(int* out) {
  int dev = 0;
  CTC_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(g_sm_mu);
  for (const auto& e : g_sm_count)
    if (e.first == dev) {
      *out = e.second;
      return CTC_OK;
    }
  int n = 0;
  CTC_CUDA_TRY(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
  g_sm_count.push_back({dev, n});
  *out = n;
  return CTC_OK;
}

int type_of_angmom(int am) {
  switch (am) {
    case 0: return 0;
    case 1: return 1;
    case 2: return 2;
    case -2: return 3;
    case 3: return 4;
    case -3: return 5;
    case 4: return 6;
    case -4: return 7;
  }
  return -1;
}

int ncomp_of_type(int t) {
  static const int n[kNumTypes] = {1, 3, 6, 5, 10, 7, 15, 9};
  return (t >= 0 && t < kNumTypes) ? n[t] : -1;
}

int l_of_type(int t) {
  static const int l[kNumTypes] = {0, 1, 2, 2, 3, 3, 4, 4};
  return (t >= 0 && t < kNumTypes) ? l[t] : -1;
}

// CTC_SCRATCH_LIMIT_BYTES caps every scratch allocation of a molecule: a
// larger request fails with CTC_ERR_NOMEM as if the device were out of
// memory (a bound for a process sharing the GPU, and the way the tests make
// the out-of-memory path run).
static size_t scratch_limit() {
  const char* e = std::getenv("CTC_SCRATCH_LIMIT_BYTES");
  if (!e) return 0;
  const long long v = std::atoll(e);
  return v > 0 ? (size_t)v : 0;
}

int Scratch::ensure(size_t need, cudaStream_t st) {
  if (need <= bytes) return CTC_OK;
  const size_t lim = scratch_limit();
  if (lim && need > lim)
    return fail(CTC_ERR_NOMEM, "scratch allocation of " + std::to_string(need) +
                                   " bytes exceeds CTC_SCRATCH_LIMIT_BYTES = " + std::to_string(lim));
  if (p) {
    cudaError_t e = cudaFreeAsync(p, st);
    if (e != cudaSuccess) return fail(CTC_ERR_CUDA, std::string("cudaFreeAsync: ") + cudaGetErrorString(e));
    p = nullptr;
    bytes = 0;
  }
  size_t alloc = std::max(need, (size_t)1 << 20);
  cudaError_t e = cudaMallocAsync(&p, alloc, st);
  if (e != cudaSuccess) {
    p = nullptr;
    return fail(CTC_ERR_NOMEM, std::string("scratch allocation of ") + std::to_string(alloc) +
                                   " bytes failed: " + cudaGetErrorString(e));
  }
  bytes = alloc;
  return CTC_OK;
}

void Scratch::release() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}

int64_t chunk_points(const ctc_molecule* mol, int nq_ao) {
  // AO buffer (nq * Mpad doubles per point) plus int8 planes; keep a chunk
  // around 2 GB so that the working set stays bounded for any basis size.
  size_t per_pt = (size_t)mol->Mpad * (8 * (size_t)nq_ao + 16);
  int64_t n = (int64_t)((size_t)2 << 30) / (int64_t)per_pt;
  n = std::max<int64_t>(n, 128);
  n = std::min<int64_t>(n, 1 << 20);
  return (n / 128) * 128;
}

// The status word.  Kernels that can fail on the device (bounded waits of the
// tensor-core pipeline) set the molecule's device word with atomicExch; it
// stays set until it is reported.  After such kernels post_status enqueues a
// copy of it into pinned host memory and records an event, so the call
// itself never waits.  poll_status (at the start of the next call) reports a
// copy that has landed; check_status waits for the stream first.
static std::string status_message(int32_t code) {
  if (code == 0x7101)
    return "a bounded wait of the tensor-core contraction ran out (status 0x7101); "
           "the call's outputs are incomplete";
  if (code == 0x7201)
    return "a tile's significant functions exceeded the workspace capacity (status 0x7201); "
           "the call's outputs are incomplete";
  return "kernel status " + std::to_string(code);
}

static int report_status(ctc_molecule* mol, cudaStream_t st, const char* what) {
  const int32_t h = *mol->h_status;
  if (h == 0) return CTC_OK;
  *mol->h_status = 0;
  mol->status_pending = false;
  CTC_CUDA_TRY(cudaMemsetAsync(mol->d_status, 0, sizeof(int32_t), st));
  return fail(CTC_ERR_DEVICE, std::string(what) + ": " + status_message(h));
}

int post_status(ctc_molecule* mol, cudaStream_t st) {
  CTC_CUDA_TRY(cudaMemcpyAsync(mol->h_status, mol->d_status, sizeof(int32_t),
                               cudaMemcpyDeviceToHost, st));
  CTC_CUDA_TRY(cudaEventRecord(mol->status_ev, st));
  mol->status_pending = true;
  return CTC_OK;
}

int poll_status(ctc_molecule* mol, cudaStream_t st) {
  if (!mol->status_pending) return CTC_OK;
  const cudaError_t q = cudaEventQuery(mol->status_ev);
  if (q == cudaErrorNotReady) return CTC_OK;
  CTC_CUDA_TRY(q);
  mol->status_pending = *mol->h_status != 0;
  return report_status(mol, st, "an earlier call on this molecule");
}

int check_status(ctc_molecule* mol, cudaStream_t st, const char* what) {
  CTC_CUDA_TRY(cudaStreamSynchronize(st));
  if (mol->status_pending) CTC_CUDA_TRY(cudaEventSynchronize(mol->status_ev));
  int32_t h = 0;
  CTC_CUDA_TRY(cudaMemcpy(&h, mol->d_status, sizeof(int32_t), cudaMemcpyDeviceToHost));
  if (h != 0 && *mol->h_status == 0) *mol->h_status = h;
  mol->status_pending = false;
  return report_status(mol, st, what);
}

// Radius beyond which |AO|, |grad AO| and |hess AO| of a segment stay below
// eps for every component: a conservative bound using the largest polynomial
// coefficient of the segment's type.
static double screening_radius2(const std::vector<double>& a, const std::vector<double>& c, int l) {
  const double eps = 1e-18;
  const double tmax = 4.0;  // bound on |angular coefficients| (pure g peaks at ~3.4)
  double rlast = 0.0;
  for (double r = 0.05; r < 200.0; r += 0.05) {
    double f = 0.0;
    for (size_t k = 0; k < a.size(); ++k) {
      double ar = a[k] * r;
      double poly = std::pow(r, l) * (1.0 + l / std::max(r, 1e-3) + 2 * ar) *
                    (1.0 + (l * l + l) / std::max(r * r, 1e-6) + 4 * ar * r + 4 * ar * ar + 2 * a[k]);
      f += std::fabs(c[k]) * tmax * poly * std::exp(-a[k] * r * r);
    }
    if (f > eps) rlast = r;
  }
  double rc = rlast + 0.1;
  return rc * rc;
}

}  // namespace ctc

using namespace ctc;

static void clear_prof(ctc_molecule* m) {
  for (int k = 0; k < 2; ++k) {
    for (auto& pr : m->prof_ev[k]) {
      cudaEventDestroy(pr.first);
      cudaEventDestroy(pr.second);
    }
    m->prof_ev[k].clear();
  }
}

extern "C" {

const char* ctc_last_error(void) { return g_last_error.c_str(); }

const char* ctc_version(void) { return "chemtoolscuda_b200 0.1 (sm_100a)"; }

int ctc_molecule_create(const ctc_basis* b, int32_t natom, const double* atom_xyz,
                        const double* atom_charges, const double* D, int32_t nbasis,
                        ctc_molecule** out) {
  if (!b || !out || !D || (natom > 0 && (!atom_xyz || !atom_charges)))
    return fail(CTC_ERR_INVALID, "ctc_molecule_create: null argument");
  if (b->nshell <= 0 || !b->centers || !b->nprim || !b->nseg || !b->angmoms || !b->exps ||
      !b->coeffs)
    return fail(CTC_ERR_INVALID, "ctc_molecule_create: empty or incomplete basis");
  *out = nullptr;
  ctc_molecule* m = new ctc_molecule();
  CTC_CUDA_TRY(cudaGetDevice(&m->device));
  m->natom = natom;
  m->atom_xyz.assign(atom_xyz, atom_xyz + 3 * (size_t)natom);
  m->charges.assign(atom_charges, atom_charges + natom);
  int ao = 0, ia = 0, ip = 0, ic = 0;
  for (int s = 0; s < b->nshell; ++s) {
    int K = b->nprim[s], S = b->nseg[s];
    if (K <= 0 || S <= 0) {
      delete m;
      return fail(CTC_ERR_INVALID, "shell " + std::to_string(s) + ": nprim and nseg must be > 0");
    }
    int atom = b->shell_atom ? b->shell_atom[s] : -1;
    if (!b->shell_atom) {
      for (int a = 0; a < natom; ++a) {
        double dx = b->centers[3 * s] - atom_xyz[3 * a], dy = b->centers[3 * s + 1] - atom_xyz[3 * a + 1],
               dz = b->centers[3 * s + 2] - atom_xyz[3 * a + 2];
        if (dx * dx + dy * dy + dz * dz < 1e-12) { atom = a; break; }
      }
    }
    if (atom >= natom) {
      delete m;
      return fail(CTC_ERR_INVALID, "shell " + std::to_string(s) + ": atom index out of range");
    }
    for (int g = 0; g < S; ++g) {
      int am = b->angmoms[ia + g];
      int t = type_of_angmom(am);
      if (t < 0) {
        delete m;
        return fail(CTC_ERR_INVALID, "shell " + std::to_string(s) + ": unsupported angular momentum " +
                                         std::to_string(am) + " (supported: 0,1,+-2,+-3,+-4)");
      }
      DevSeg sg;
      sg.cx = b->centers[3 * s];
      sg.cy = b->centers[3 * s + 1];
      sg.cz = b->centers[3 * s + 2];
      sg.type = t;
      sg.l = l_of_type(t);
      sg.nprim = K;
      sg.prim0 = (int)m->alpha.size();
      sg.ao0 = ao;
      sg.orig_ao0 = ao;
      sg.pad = 0;
      sg.atom = atom;
      std::vector<double> aa, cc;
      for (int k = 0; k < K; ++k) {
        double a = b->exps[ip + k];
        if (!(a > 0.0)) {
          delete m;
          return fail(CTC_ERR_INVALID, "shell " + std::to_string(s) + ": exponents must be > 0");
        }
        double nrm = std::pow(2.0 * a / M_PI, 0.75) * std::pow(4.0 * a, 0.5 * sg.l);
        aa.push_back(a);
        cc.push_back(b->coeffs[ic + g * K + k] * nrm);
      }
      sg.rcut2 = screening_radius2(aa, cc, sg.l);
      m->alpha.insert(m->alpha.end(), aa.begin(), aa.end());
      m->coef.insert(m->coef.end(), cc.begin(), cc.end());
      m->segs.push_back(sg);
      ao += ncomp_of_type(t);
    }
    ia += S;
    ip += K;
    ic += S * K;
  }
  if (ao != nbasis) {
    delete m;
    return fail(CTC_ERR_INVALID, "basis has " + std::to_string(ao) + " functions but D is " +
                                     std::to_string(nbasis) + " x " + std::to_string(nbasis));
  }
  m->M = ao;
  m->Mpad = (ao + 127) / 128 * 128;
  m->nseg = (int)m->segs.size();
  // Internal AO order: segments grouped by atom, atoms in Morton order of
  // their positions, so that the AOs significant on a compact point tile form
  // few contiguous runs (gathers of D rows/columns then touch whole sectors).
  {
    std::vector<uint64_t> key(natom, 0);
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int a = 0; a < natom; ++a)
      for (int d = 0; d < 3; ++d) {
        lo[d] = std::min(lo[d], atom_xyz[3 * a + d]);
        hi[d] = std::max(hi[d], atom_xyz[3 * a + d]);
      }
    auto spread = [](uint64_t v) {
      uint64_t r = 0;
      for (int b = 0; b < 21; ++b) r |= ((v >> b) & 1ull) << (3 * b);
      return r;
    };
    for (int a = 0; a < natom; ++a) {
      uint64_t q[3];
      for (int d = 0; d < 3; ++d) {
        const double ext = std::max(hi[d] - lo[d], 1e-9);
        q[d] = (uint64_t)std::min(2097151.0, std::max(0.0, (atom_xyz[3 * a + d] - lo[d]) / ext * 2097151.0));
      }
      key[a] = spread(q[0]) | (spread(q[1]) << 1) | (spread(q[2]) << 2);
    }
    std::vector<int> rank_of(natom);
    {
      std::vector<int> order(natom);
      for (int a = 0; a < natom; ++a) order[a] = a;
      std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return key[x] < key[y]; });
      for (int r = 0; r < natom; ++r) rank_of[order[r]] = r;
    }
    std::vector<int> so(m->nseg);
    for (int i = 0; i < m->nseg; ++i) so[i] = i;
    std::stable_sort(so.begin(), so.end(), [&](int x, int y) {
      const int ax = m->segs[x].atom, ay = m->segs[y].atom;
      const int rx = ax < 0 ? natom : rank_of[ax], ry = ay < 0 ? natom : rank_of[ay];
      return rx < ry;
    });
    std::vector<DevSeg> ns;
    m->ao_perm.assign(ao, 0);
    std::vector<int32_t> new_atom;
    int k = 0;
    for (int i : so) {
      DevSeg sg = m->segs[i];
      sg.orig_ao0 = sg.ao0;
      sg.ao0 = k;
      const int nc = ncomp_of_type(sg.type);
      for (int j = 0; j < nc; ++j) {
        m->ao_perm[k + j] = sg.orig_ao0 + j;
        new_atom.push_back(sg.atom);
      }
      k += nc;
      ns.push_back(sg);
    }
    m->segs.swap(ns);
    m->ao_atom.swap(new_atom);
  }
  m->seg_order.resize(m->nseg);
  for (int i = 0; i < m->nseg; ++i) m->seg_order[i] = i;
  std::stable_sort(m->seg_order.begin(), m->seg_order.end(), [&](int x, int y) {
    if (m->segs[x].type != m->segs[y].type) return m->segs[x].type < m->segs[y].type;
    return m->segs[x].nprim < m->segs[y].nprim;
  });
  m->D.resize((size_t)ao * ao);
  for (int i = 0; i < ao; ++i) {
    const double* src = D + (size_t)m->ao_perm[i] * ao;
    for (int j = 0; j < ao; ++j) m->D[(size_t)i * ao + j] = src[m->ao_perm[j]];
  }
  m->ao_atom.resize(m->Mpad, -1);
  std::vector<int32_t> iperm(ao);
  for (int i = 0; i < ao; ++i) iperm[m->ao_perm[i]] = i;

  size_t MM = (size_t)m->Mpad * m->Mpad;
  std::vector<double> Dpad(MM, 0.0);
  for (int i = 0; i < ao; ++i)
    std::memcpy(&Dpad[(size_t)i * m->Mpad], &m->D[(size_t)i * ao], sizeof(double) * ao);
#define ALLOC_COPY(dst, src, count)                                                          \
  do {                                                                                       \
    cudaError_t _e = cudaMalloc((void**)&(dst), sizeof(*(dst)) * (count));                   \
    if (_e == cudaSuccess)                                                                   \
      _e = cudaMemcpy((dst), (src), sizeof(*(dst)) * (count), cudaMemcpyHostToDevice);       \
    if (_e != cudaSuccess) {                                                                 \
      ctc_molecule_destroy(m);                                                               \
      return fail(CTC_ERR_NOMEM, std::string("device table upload: ") + cudaGetErrorString(_e)); \
    }                                                                                        \
  } while (0)
  ALLOC_COPY(m->d_segs, m->segs.data(), m->segs.size());
  ALLOC_COPY(m->d_alpha, m->alpha.data(), m->alpha.size());
  ALLOC_COPY(m->d_coef, m->coef.data(), m->coef.size());
  ALLOC_COPY(m->d_order, m->seg_order.data(), m->seg_order.size());
  ALLOC_COPY(m->d_ao_atom, m->ao_atom.data(), m->ao_atom.size());
  ALLOC_COPY(m->d_D, Dpad.data(), MM);
  ALLOC_COPY(m->d_ao_iperm, iperm.data(), iperm.size());
  ALLOC_COPY(m->d_ao_perm, m->ao_perm.data(), m->ao_perm.size());
#undef ALLOC_COPY
  if (cudaMalloc((void**)&m->d_status, sizeof(int32_t)) != cudaSuccess ||
      cudaMemset(m->d_status, 0, sizeof(int32_t)) != cudaSuccess ||
      cudaMallocHost((void**)&m->h_status, 4 * sizeof(int32_t)) != cudaSuccess ||
      cudaEventCreateWithFlags(&m->status_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaMalloc((void**)&m->d_stats, sizeof(double) * 8) != cudaSuccess ||
      cudaMemset(m->d_stats, 0, sizeof(double) * 8) != cudaSuccess) {
    ctc_molecule_destroy(m);
    return fail(CTC_ERR_NOMEM, "status word allocation failed");
  }
  *out = m;
  return CTC_OK;
}

int ctc_molecule_destroy(ctc_molecule* m) {
  if (!m) return CTC_OK;
  cudaDeviceSynchronize();
  clear_prof(m);
  destroy_esp(m);
  cudaFree(m->d_segs);
  cudaFree(m->d_alpha);
  cudaFree(m->d_coef);
  cudaFree(m->d_order);
  cudaFree(m->d_ao_atom);
  cudaFree(m->d_D);
  cudaFree(m->d_ao_iperm);
  cudaFree(m->d_ao_perm);
  cudaFree(m->d_Dsl);
  cudaFree(m->d_Dscale);
  cudaFree(m->d_nzpair);
  cudaFree(m->d_status);
  if (m->h_status) cudaFreeHost(m->h_status);
  if (m->status_ev) cudaEventDestroy(m->status_ev);
  cudaFree(m->d_stats);
  m->ws_ao.release();
  m->ws_sl.release();
  m->ws_part.release();
  m->ws_misc.release();
  m->ws_cap.release();
  m->ws_esp.release();
  m->ws_adj.release();
  if (m->hostpipe) {
    m->hostpipe->release();
    delete m->hostpipe;
  }
  delete m;
  return CTC_OK;
}

int ctc_molecule_nbasis(const ctc_molecule* m) { return m ? m->M : fail(CTC_ERR_INVALID, "null molecule"); }
int ctc_molecule_natom(const ctc_molecule* m) { return m ? m->natom : fail(CTC_ERR_INVALID, "null molecule"); }

int ctc_molecule_set_density_matrix(ctc_molecule* m, const double* d_D, void* stream) {
  if (!m || !d_D) return fail(CTC_ERR_INVALID, "set_density_matrix: null argument");
  cudaStream_t st = (cudaStream_t)stream;
  const int M = m->M, Mp = m->Mpad;
  const int64_t total = (int64_t)Mp * Mp;
  ctc::permute_density_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(d_D, M, Mp, m->d_ao_perm,
                                                                               m->d_D);
  CTC_CUDA_TRY(cudaGetLastError());
  // the host copy (used only to build the ESP tables) is fetched again when needed
  m->host_D_stale = true;
  m->dsl_valid = false;
  m->esp_valid = false;
  return CTC_OK;
}

int ctc_molecule_set_coordinates(ctc_molecule* m, const double* xyz) {
  if (!m || !xyz) return fail(CTC_ERR_INVALID, "set_coordinates: null argument");
  for (auto& s : m->segs) {
    if (s.atom < 0) continue;
    s.cx = xyz[3 * s.atom];
    s.cy = xyz[3 * s.atom + 1];
    s.cz = xyz[3 * s.atom + 2];
  }
  m->atom_xyz.assign(xyz, xyz + 3 * (size_t)m->natom);
  CTC_CUDA_TRY(cudaMemcpy(m->d_segs, m->segs.data(), sizeof(DevSeg) * m->segs.size(),
                          cudaMemcpyHostToDevice));
  m->esp_valid = false;
  return CTC_OK;
}

int ctc_molecule_get_stats(ctc_molecule* m, double* stats) {
  if (!m || !stats) return fail(CTC_ERR_INVALID, "get_stats: null argument");
  double d[8] = {0};
  CTC_CUDA_TRY(cudaDeviceSynchronize());
  CTC_CUDA_TRY(cudaMemcpy(d, m->d_stats, sizeof(double) * 8, cudaMemcpyDeviceToHost));
  for (int i = 0; i < 8; ++i) stats[i] = 0.0;
  stats[0] = d[0];
  stats[1] = d[1];
  stats[2] = d[2];
  stats[3] = d[3];
  stats[4] = m->host_launches;
  stats[5] = m->host_chunks;
  for (int k = 0; k < 2; ++k) {
    double ms_total = 0.0;
    for (auto& pr : m->prof_ev[k]) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, pr.first, pr.second) == cudaSuccess) ms_total += ms;
    }
    stats[6 + k] = ms_total;
  }
  return CTC_OK;
}

int ctc_molecule_set_profiling(ctc_molecule* m, int32_t on) {
  if (!m) return fail(CTC_ERR_INVALID, "set_profiling: null molecule");
  m->prof = on != 0;
  return CTC_OK;
}

int ctc_molecule_sync_status(ctc_molecule* m, void* stream) {
  if (!m) return fail(CTC_ERR_INVALID, "sync_status: null molecule");
  return check_status(m, (cudaStream_t)stream, "device status");
}

int ctc_molecule_set_wait_limit(ctc_molecule* m, int64_t cycles) {
  if (!m) return fail(CTC_ERR_INVALID, "set_wait_limit: null molecule");
  if (cycles < 0) return fail(CTC_ERR_INVALID, "set_wait_limit: negative cycle count");
  m->wait_cycles = cycles;
  return CTC_OK;
}

int ctc_molecule_reset_stats(ctc_molecule* m) {
  if (!m) return fail(CTC_ERR_INVALID, "reset_stats: null molecule");
  CTC_CUDA_TRY(cudaDeviceSynchronize());
  CTC_CUDA_TRY(cudaMemset(m->d_stats, 0, sizeof(double) * 8));
  m->host_launches = 0;
  m->host_chunks = 0;
  clear_prof(m);
  return CTC_OK;
}

int ctc_molecule_prepare(ctc_molecule* m, int32_t precision) {
  if (!m) return fail(CTC_ERR_INVALID, "prepare: null molecule");
  if (precision == CTC_PREC_TC_SPLIT) return prepare_tc(m, 0);
  if (precision != CTC_PREC_FP64) return fail(CTC_ERR_INVALID, "prepare: unknown precision");
  return CTC_OK;
}

}  // extern "C"
