// ctc_api.cu -- extern "C" entry points of include/chemtools_cuda.h.
//
// Device-pointer calls are stream-ordered and validate their arguments on the
// host.  Host-pointer calls (the reference's own calling convention: host
// arrays in, host vector out, e.g. src/evaluate_density.cu:663-673) stage
// points and results through pinned buffers in slabs, so the copies of one
// slab overlap the kernels of the next on two streams.
#include <algorithm>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "ctc_internal.h"

using namespace ctc;

namespace {

bool any_output(const ctc_outputs* o) {
  return o->rho || o->grad || o->hess || o->lap || o->tau_pd || o->tau_alpha || o->rdg ||
         o->shannon || o->weizsacker || o->thomas_fermi || o->gge || o->general_ked;
}

ctc_params default_params(const ctc_params* p) {
  if (p) return *p;
  ctc_params d;
  d.alpha = 0.0;
  d.gge_a = 1.0 / 9.0;
  d.gge_b = 1.0 / 6.0;
  d.ked_a = 1.0;
  return d;
}

// scalar widths of the output slots in doubles per point
const int kWidth[12] = {1, 3, 9, 1, 1, 1, 1, 1, 1, 1, 1, 1};

double** slot(ctc_outputs* o, int i) {
  double** s[12] = {&o->rho, &o->grad, &o->hess, &o->lap, &o->tau_pd, &o->tau_alpha,
                    &o->rdg, &o->shannon, &o->weizsacker, &o->thomas_fermi, &o->gge,
                    &o->general_ked};
  return s[i];
}

// memcpy of large host buffers on several threads: one thread moves ~4-10
// GB/s, and the host side of the host-buffer pipeline moves ~160 B per point.
// One copy job -- a list of (dst, src, bytes) segments, e.g. all outputs of a
// slab -- is cut at equal byte offsets over up to 16 threads, so small and
// large outputs share the threads (one output at a time left the 8 MB
// outputs of a 2^20-point slab on one thread each).
struct CopySeg {
  void* dst;
  const void* src;
  size_t bytes;
};
void par_copy_segs(const std::vector<CopySeg>& segs) {
  size_t total = 0;
  for (const CopySeg& g : segs) total += g.bytes;
  constexpr size_t kSlice = (size_t)2 << 20;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t nt = std::max<size_t>(1, std::min<size_t>({(size_t)16, (size_t)hw, total / kSlice}));
  auto run = [&](size_t lo, size_t hi) {  // bytes [lo, hi) of the concatenated segments
    size_t base = 0;
    for (const CopySeg& g : segs) {
      const size_t a = std::max(lo, base), b = std::min(hi, base + g.bytes);
      if (a < b) std::memcpy((char*)g.dst + (a - base), (const char*)g.src + (a - base), b - a);
      base += g.bytes;
    }
  };
  if (nt <= 1) {
    run(0, total);
    return;
  }
  const size_t part = (total + nt - 1) / nt;
  std::vector<std::thread> th;
  for (size_t t = 1; t < nt; ++t) {
    const size_t lo = t * part, hi = std::min(total, lo + part);
    if (lo < hi) th.emplace_back(run, lo, hi);
  }
  run(0, std::min(total, part));
  for (auto& x : th) x.join();
}

void par_copy(void* dst, const void* src, size_t bytes) { par_copy_segs({{dst, src, bytes}}); }

}  // namespace

namespace ctc {

int HostPipe::ensure(size_t slab_bytes) {
  if (!cs) {
    CTC_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    CTC_CUDA_TRY(cudaStreamCreateWithFlags(&h2d, cudaStreamNonBlocking));
    CTC_CUDA_TRY(cudaStreamCreateWithFlags(&d2h, cudaStreamNonBlocking));
    for (int b = 0; b < 2; ++b) {
      CTC_CUDA_TRY(cudaEventCreateWithFlags(&ev_in[b], cudaEventDisableTiming));
      CTC_CUDA_TRY(cudaEventCreateWithFlags(&ev_comp[b], cudaEventDisableTiming));
      CTC_CUDA_TRY(cudaEventCreateWithFlags(&ev_out[b], cudaEventDisableTiming));
    }
  }
  if (slab_bytes <= bytes) return CTC_OK;
  for (int b = 0; b < 2; ++b) {
    if (pin[b]) cudaFreeHost(pin[b]);
    if (dbuf[b]) cudaFree(dbuf[b]);
    pin[b] = nullptr;
    dbuf[b] = nullptr;
  }
  bytes = 0;
  for (int b = 0; b < 2; ++b) {
    if (cudaMallocHost(&pin[b], slab_bytes) != cudaSuccess) {
      cudaGetLastError();
      return fail(CTC_ERR_NOMEM, "ctc_eval_local_host: pinned host staging allocation failed");
    }
    if (cudaMalloc((void**)&dbuf[b], slab_bytes) != cudaSuccess) {
      cudaGetLastError();
      return fail(CTC_ERR_NOMEM, "ctc_eval_local_host: device staging allocation failed");
    }
  }
  bytes = slab_bytes;
  return CTC_OK;
}

void HostPipe::release() {
  for (int b = 0; b < 2; ++b) {
    if (pin[b]) cudaFreeHost(pin[b]);
    if (dbuf[b]) cudaFree(dbuf[b]);
    if (ev_in[b]) cudaEventDestroy(ev_in[b]);
    if (ev_comp[b]) cudaEventDestroy(ev_comp[b]);
    if (ev_out[b]) cudaEventDestroy(ev_out[b]);
  }
  if (cs) cudaStreamDestroy(cs);
  if (h2d) cudaStreamDestroy(h2d);
  if (d2h) cudaStreamDestroy(d2h);
  *this = HostPipe();
}

}  // namespace ctc

extern "C" {

int ctc_eval_local(ctc_molecule* mol, const double* d_points, int64_t n, int32_t precision,
                   const ctc_params* params, const ctc_outputs* d_out, void* stream) {
  if (!mol || !d_out) return fail(CTC_ERR_INVALID, "ctc_eval_local: null argument");
  if (n < 0) return fail(CTC_ERR_INVALID, "ctc_eval_local: negative point count");
  if (n > 0 && !d_points) return fail(CTC_ERR_INVALID, "ctc_eval_local: null points");
  if (!any_output(d_out)) return CTC_OK;
  PointSrc src{};
  src.pts = d_points;
  ctc_params prm = default_params(params);
  return eval_local(mol, src, n, precision, &prm, d_out, (cudaStream_t)stream);
}

int ctc_eval_cubic(ctc_molecule* mol, const double* origin, const double* axes,
                   const int32_t* shape, int32_t precision, const ctc_params* params,
                   const ctc_outputs* d_out, void* stream) {
  if (!mol || !origin || !axes || !shape || !d_out)
    return fail(CTC_ERR_INVALID, "ctc_eval_cubic: null argument");
  if (shape[0] < 0 || shape[1] < 0 || shape[2] < 0)
    return fail(CTC_ERR_INVALID, "ctc_eval_cubic: negative shape");
  if (!any_output(d_out)) return CTC_OK;
  PointSrc src{};
  src.cubic = 1;
  for (int i = 0; i < 3; ++i) src.o[i] = origin[i];
  for (int i = 0; i < 9; ++i) src.ax[i] = axes[i];
  src.ny = shape[1];
  src.nz = shape[2];
  int64_t n = (int64_t)shape[0] * shape[1] * shape[2];
  if (n == 0) return CTC_OK;
  ctc_params prm = default_params(params);
  return eval_local(mol, src, n, precision, &prm, d_out, (cudaStream_t)stream);
}

int ctc_eval_ao(ctc_molecule* mol, const double* d_points, int64_t n, int32_t deriv,
                double* d_out, void* stream) {
  if (!mol || !d_out || (n > 0 && !d_points)) return fail(CTC_ERR_INVALID, "ctc_eval_ao: null argument");
  if (deriv < 0 || deriv > 2) return fail(CTC_ERR_INVALID, "ctc_eval_ao: deriv must be 0, 1 or 2");
  if (n <= 0) return n < 0 ? fail(CTC_ERR_INVALID, "ctc_eval_ao: negative point count") : CTC_OK;
  PointSrc src{};
  src.pts = d_points;
  return launch_ao_public(mol, src, n, deriv, d_out, (cudaStream_t)stream);
}

int ctc_eval_esp(ctc_molecule* mol, const double* d_points, int64_t n, double* d_out, void* stream) {
  if (!mol || !d_out || (n > 0 && !d_points)) return fail(CTC_ERR_INVALID, "ctc_eval_esp: null argument");
  return eval_esp(mol, d_points, n, d_out, (cudaStream_t)stream);
}

int ctc_molecule_esp_info(ctc_molecule* mol, double* info) {
  if (!mol || !info) return fail(CTC_ERR_INVALID, "ctc_molecule_esp_info: null argument");
  return esp_info(mol, info);
}

int ctc_adjoint(ctc_molecule* mol, const double* d_points, int64_t n, const double* d_v_rho,
                const double* d_v_grad, double* d_dLdD, double* d_dLdR, void* stream) {
  if (!mol || (n > 0 && (!d_points || !d_v_rho)))
    return fail(CTC_ERR_INVALID, "ctc_adjoint: null argument");
  if (n < 0) return fail(CTC_ERR_INVALID, "ctc_adjoint: negative point count");
  if (n == 0 || (!d_dLdD && !d_dLdR)) return CTC_OK;
  return eval_adjoint(mol, d_points, n, d_v_rho, d_v_grad, d_dLdD, d_dLdR, (cudaStream_t)stream);
}

// Host-buffer variants: slabs of points go host -> device, through the
// device path and back.  Kernels run on the molecule's compute stream (its
// scratch is not shared across streams); the host->device copy of slab k+1
// and the device->host copy of slab k-1 run on two copy streams while slab k
// computes, ordered by events, and the host thread moves slab k-1's results
// out of pinned memory (several threads) meanwhile.  Streams, events and
// staging belong to the molecule (HostPipe): created on the first call.
int ctc_eval_local_host(ctc_molecule* mol, const double* h_points, int64_t n, int32_t precision,
                        const ctc_params* params, const ctc_outputs* h_out) {
  if (!mol || !h_out || (n > 0 && !h_points)) return fail(CTC_ERR_INVALID, "ctc_eval_local_host: null argument");
  if (n < 0) return fail(CTC_ERR_INVALID, "ctc_eval_local_host: negative point count");
  if (n == 0 || !any_output(h_out)) return CTC_OK;
  ctc_params prm = default_params(params);
  int width = 3;
  for (int i = 0; i < 12; ++i)
    if (*slot(const_cast<ctc_outputs*>(h_out), i)) width += kWidth[i];
  // slabs of up to 2^20 points: large enough that the device pipeline's
  // per-call costs (point sort, chunk tails) stay small, small enough that
  // the two staging slabs stay a few hundred MB
  const int64_t slab = std::min<int64_t>(n, (int64_t)1 << 20);
  const size_t slab_bytes = sizeof(double) * (size_t)slab * width;
  if (!mol->hostpipe) mol->hostpipe = new HostPipe();
  HostPipe& hp = *mol->hostpipe;
  int rc = hp.ensure(slab_bytes);
  if (rc != CTC_OK) return rc;
  cudaStream_t cs = hp.cs, h2d = hp.h2d, d2h = hp.d2h;
  auto cuda_ok = [&](cudaError_t e, const char* what) {
    if (e != cudaSuccess && rc == CTC_OK) rc = fail(CTC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return rc == CTC_OK;
  };
  int64_t pending_off[2] = {-1, -1}, pending_n[2] = {0, 0};
  auto drain = [&](int b) {
    if (pending_off[b] < 0 || rc != CTC_OK) return;
    if (!cuda_ok(cudaEventSynchronize(hp.ev_out[b]), "ctc_eval_local_host: wait")) return;
    const double* hb = (const double*)hp.pin[b] + 3 * (size_t)pending_n[b];
    std::vector<CopySeg> segs;
    for (int i = 0; i < 12; ++i) {
      double* dst = *slot(const_cast<ctc_outputs*>(h_out), i);
      if (!dst) continue;
      segs.push_back({dst + kWidth[i] * pending_off[b], hb, sizeof(double) * kWidth[i] * pending_n[b]});
      hb += kWidth[i] * pending_n[b];
    }
    par_copy_segs(segs);
    pending_off[b] = -1;
  };
  int b = 0;
  for (int64_t off = 0; off < n && rc == CTC_OK; off += slab, b ^= 1) {
    const int64_t m = std::min(slab, n - off);
    drain(b);
    if (rc != CTC_OK) break;
    double* hpin = (double*)hp.pin[b];
    double* dp = hp.dbuf[b];
    par_copy(hpin, h_points + 3 * off, sizeof(double) * 3 * m);
    if (!cuda_ok(cudaMemcpyAsync(dp, hpin, sizeof(double) * 3 * m, cudaMemcpyHostToDevice, h2d), "H2D") ||
        !cuda_ok(cudaEventRecord(hp.ev_in[b], h2d), "event") ||
        !cuda_ok(cudaStreamWaitEvent(cs, hp.ev_in[b], 0), "event"))
      break;
    ctc_outputs d{};
    double* cur = dp + 3 * m;
    for (int i = 0; i < 12; ++i) {
      if (!*slot(const_cast<ctc_outputs*>(h_out), i)) continue;
      *slot(&d, i) = cur;
      cur += kWidth[i] * m;
    }
    PointSrc src{};
    src.pts = dp;
    rc = eval_local(mol, src, m, precision, &prm, &d, cs);
    if (rc != CTC_OK) break;
    if (!cuda_ok(cudaEventRecord(hp.ev_comp[b], cs), "event") ||
        !cuda_ok(cudaStreamWaitEvent(d2h, hp.ev_comp[b], 0), "event") ||
        !cuda_ok(cudaMemcpyAsync(hpin + 3 * m, dp + 3 * m, sizeof(double) * (width - 3) * m,
                                 cudaMemcpyDeviceToHost, d2h), "D2H") ||
        !cuda_ok(cudaEventRecord(hp.ev_out[b], d2h), "event"))
      break;
    pending_off[b] = off;
    pending_n[b] = m;
  }
  drain(b);
  drain(b ^ 1);
  // a device-side failure of the tensor-core kernels of this call
  if (rc == CTC_OK) rc = check_status(mol, cs, "ctc_eval_local_host");
  // leave nothing of this call in flight (also after an error)
  cudaStreamSynchronize(cs);
  cudaStreamSynchronize(h2d);
  cudaStreamSynchronize(d2h);
  return rc;
}

int ctc_eval_esp_host(ctc_molecule* mol, const double* h_points, int64_t n, double* h_out) {
  if (!mol || !h_out || (n > 0 && !h_points)) return fail(CTC_ERR_INVALID, "ctc_eval_esp_host: null argument");
  if (n < 0) return fail(CTC_ERR_INVALID, "ctc_eval_esp_host: negative point count");
  if (n == 0) return CTC_OK;
  double* d = nullptr;
  if (cudaMalloc((void**)&d, sizeof(double) * 4 * (size_t)n) != cudaSuccess)
    return fail(CTC_ERR_NOMEM, "ctc_eval_esp_host: device allocation failed");
  int rc = CTC_OK;
  if (cudaMemcpy(d, h_points, sizeof(double) * 3 * n, cudaMemcpyHostToDevice) != cudaSuccess)
    rc = fail(CTC_ERR_CUDA, "ctc_eval_esp_host: H2D copy failed");
  if (rc == CTC_OK) rc = eval_esp(mol, d, n, d + 3 * n, 0);
  if (rc == CTC_OK && cudaMemcpy(h_out, d + 3 * n, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = fail(CTC_ERR_CUDA, "ctc_eval_esp_host: D2H copy failed");
  cudaFree(d);
  return rc;
}

}  // extern "C"
