// ctc_internal.h -- shared declarations of the B200 grid-evaluation library.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/chemtools_cuda.h"

namespace ctc {

// --------------------------------------------------------------------------- error handling
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);

// Sets a kernel's dynamic shared-memory limit once per (device, kernel, size):
// the attribute is per device, so every device a kernel runs on needs it.
// Thread-safe.  kernel is the __global__ function's address.
int ensure_smem_attr(const void* kernel, int bytes);
// Streaming multiprocessors of the current device (cached per device).
int device_sm_count(int* out);
__global__ void permute_density_kernel(const double* __restrict__ D, int M, int Mpad,
                                       const int32_t* __restrict__ perm, double* __restrict__ out);

#define CTC_CUDA_TRY(expr)                                                               \
  do {                                                                                   \
    cudaError_t _e = (expr);                                                             \
    if (_e != cudaSuccess)                                                               \
      return ::ctc::fail(CTC_ERR_CUDA, std::string(#expr " -> ") + cudaGetErrorString(_e)); \
  } while (0)

// --------------------------------------------------------------------------- basis tables
// Segment types: fchk angular-momentum code -> table index.
//   0 s, 1 p, 2 d (6), -2 d (5), 3 f (10), -3 f (7), 4 g (15), -4 g (9)
constexpr int kNumTypes = 8;
int type_of_angmom(int angmom);          // -1 when unknown
int ncomp_of_type(int type);
int l_of_type(int type);

// One segmented shell as the kernels see it (64 bytes).
struct DevSeg {
  double cx, cy, cz;
  double rcut2;     // squared radius beyond which every AO (and derivative) is < 1e-18
  int32_t type;     // 0..7
  int32_t l;
  int32_t nprim;
  int32_t prim0;    // first primitive in the primitive arrays
  int32_t ao0;      // first AO index (internal, spatially sorted order)
  int32_t atom;     // owning atom or -1
  int32_t orig_ao0; // first AO index in the caller's order
  int32_t pad;
};
static_assert(sizeof(DevSeg) == 64, "DevSeg layout");

// Polynomial term of one AO component: coef * x^a y^b z^c (angular normalisation folded in).
struct Term {
  double c;
  int8_t a, b, z, pad;
};

// Where the point coordinates of a launch come from.
struct PointSrc {
  const double* pts;   // row-major (N,3) when not cubic
  double o[3];         // cubic origin
  double ax[9];        // cubic axes, row i = axis i
  int32_t ny, nz;      // cubic shape (x extent implied)
  int32_t cubic;
  int64_t offset;      // global index of the first point of this launch
};

__host__ __device__ inline void point_of(const PointSrc& s, int64_t i, double& x, double& y,
                                         double& z) {
  int64_t g = s.offset + i;
  if (s.cubic) {
    int64_t k = g % s.nz;
    int64_t j = (g / s.nz) % s.ny;
    int64_t ii = g / ((int64_t)s.nz * s.ny);
    double fi = (double)ii, fj = (double)j, fk = (double)k;
    x = s.o[0] + fi * s.ax[0] + fj * s.ax[3] + fk * s.ax[6];
    y = s.o[1] + fi * s.ax[1] + fj * s.ax[4] + fk * s.ax[7];
    z = s.o[2] + fi * s.ax[2] + fj * s.ax[5] + fk * s.ax[8];
  } else {
    x = s.pts[3 * g];
    y = s.pts[3 * g + 1];
    z = s.pts[3 * g + 2];
  }
}

// Device scratch owned by a molecule; grows on demand, released stream-ordered.
struct Scratch {
  void* p = nullptr;
  size_t bytes = 0;
  int ensure(size_t need, cudaStream_t st);
  void release();
};

// ESP pair data built once per molecule (see ctc_esp.cu).
struct EspTables;

// Host-buffer pipeline of a molecule (ctc_eval_local_host): a compute stream,
// two copy streams, their events, and two slabs of device and pinned host
// staging.  Created on the first host-buffer call and kept with the handle,
// so later calls create and allocate nothing.
struct HostPipe {
  cudaStream_t cs = nullptr, h2d = nullptr, d2h = nullptr;
  cudaEvent_t ev_in[2] = {nullptr, nullptr}, ev_comp[2] = {nullptr, nullptr},
              ev_out[2] = {nullptr, nullptr};
  void* pin[2] = {nullptr, nullptr};
  double* dbuf[2] = {nullptr, nullptr};
  size_t bytes = 0;  // of each staging buffer
  int ensure(size_t slab_bytes);
  void release();
};

// One chunk of point tiles of the screened local pipeline (device pointers).
// A tile holds TP points; its significant segments, compacted, define the
// tile's own K dimension (kt, padded to a multiple of 64).
struct TileBatch {
  int C = 0;          // tiles in this chunk
  int TP = 0;         // points per tile (32 or 128)
  int Kcap = 0;       // capacity of the compact K dimension (>= Mpad)
  int nq = 0;         // AO quantities per point (1, 4, 10)
  double* xyz = nullptr;    // [C][TP][3]
  int64_t* out = nullptr;   // [C][TP] output index, -1 for padding
  int32_t* nsig = nullptr;  // [C] significant segments
  int32_t* ktrue = nullptr; // [C] compact AOs before padding
  int32_t* kt = nullptr;    // [C] compact AOs padded to 64
  int32_t* segs = nullptr;  // [C][nseg] significant segment ids
  int32_t* k0 = nullptr;    // [C][nseg] compact offset of each significant segment
  int32_t* aomap = nullptr; // [C][Kcap] compact -> AO index, -1 for padding
  double* ao = nullptr;     // [C][nq][TP][Kcap] AO values and derivatives
};
constexpr int kKtAlign = 64;

}  // namespace ctc

struct ctc_molecule {
  int device = 0;
  int natom = 0, M = 0, Mpad = 0, nseg = 0;
  std::vector<ctc::DevSeg> segs;             // host copy
  std::vector<double> alpha, coef;           // host copies (coef includes N_l(alpha))
  std::vector<int32_t> seg_order;            // segments sorted by type, nprim
  std::vector<double> atom_xyz, charges;
  std::vector<double> D;                     // host copy, M x M
  std::vector<int32_t> ao_atom;              // AO -> atom (internal order)
  std::vector<int32_t> ao_perm;              // internal AO -> caller's AO
  int32_t* d_ao_iperm = nullptr;             // caller's AO -> internal AO
  int32_t* d_ao_perm = nullptr;              // internal AO -> caller's AO
  bool host_D_stale = false;                 // D replaced on the device since the host copy was made
  // device tables
  ctc::DevSeg* d_segs = nullptr;
  double* d_alpha = nullptr;
  double* d_coef = nullptr;
  int32_t* d_order = nullptr;
  int32_t* d_ao_atom = nullptr;
  double* d_D = nullptr;                     // Mpad x Mpad, zero padded
  // split-precision copy of D (4 int8 byte planes, row scales)
  int8_t* d_Dsl = nullptr;
  double* d_Dscale = nullptr;
  bool dsl_valid = false;
  // atom pairs with a non-zero block of D (natom x natom bytes), built with
  // the split copy when some atom-pair block of D is zero (a cut-off density
  // matrix); the tensor-core kernel then skips the K stages of tiles whose
  // D block is entirely zero.  nullptr: every block is taken.
  uint8_t* d_nzpair = nullptr;
  // status word written by kernels (sticky until reported), its pinned host
  // copy ([0]; [1] receives the capacity pre-pass's count), and the event
  // recorded after the copy was enqueued
  int32_t* d_status = nullptr;
  int32_t* h_status = nullptr;
  cudaEvent_t status_ev = nullptr;
  bool status_pending = false;
  // limit of the tensor-core pipeline's waits in SM cycles (0: the default)
  int64_t wait_cycles = 0;
  // work counters: [0] tiles [1] points [2] sum kt_true [3] sum rows*kt^2 (device, doubles)
  double* d_stats = nullptr;
  double host_launches = 0, host_chunks = 0;
  // optional kernel timing: event pairs of contraction (0) and AO (1) kernels
  bool prof = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_ev[2];
  // scratch
  ctc::Scratch ws_ao, ws_sl, ws_part, ws_misc, ws_cap, ws_esp, ws_adj;
  ctc::EspTables* esp = nullptr;
  bool esp_valid = false;
  ctc::HostPipe* hostpipe = nullptr;
};

namespace ctc {

// ---- kernels / launchers (ctc_ao.cu) ----
// AO block of every tile of a batch on its significant segments only.
int launch_ao_tiles(const ctc_molecule* mol, const TileBatch& tb, int deriv, cudaStream_t st);
// Same, and in the same kernel the int8 digit planes of the tile rows
// (nqa = 4: 32 points x {phi, d phi}; nqa = 1: 128 points x phi) with one
// exponent per row, for the tensor-core split path: planes [C][5][128][Kcap],
// eexp [C][128].
// order (optional) lists the tiles in the order the CTAs take them.
int launch_ao_tiles_sliced(const ctc_molecule* mol, const TileBatch& tb, int deriv, int nqa,
                           int8_t* planes, int32_t* eexp, const int32_t* order, cudaStream_t st);
int launch_ao(const ctc_molecule* mol, const PointSrc& src, int64_t n, int deriv, double* out,
              int nq_out, int ld, cudaStream_t st);
// AO output in (nq, n, M) layout for ctc_eval_ao.
int launch_ao_public(const ctc_molecule* mol, const PointSrc& src, int64_t n, int deriv,
                     double* out, cudaStream_t st);

// ---- local descriptors (ctc_local.cu) ----
struct LocalPlan {
  int nq_ao;    // AO quantities produced per point (1, 4, 10)
  int nqa;      // GEMM row quantities (1: Phi only, 4: Phi and grad Phi)
  int deriv;    // AO derivative order
};
LocalPlan plan_local(const ctc_outputs* o);
int eval_local(ctc_molecule* mol, const PointSrc& src, int64_t n, int precision,
               const ctc_params* prm, const ctc_outputs* out, cudaStream_t st);

// ---- tensor-core split path (ctc_tc.cu) ----
int prepare_tc(ctc_molecule* mol, cudaStream_t st);
// Workspace of the digit planes and row exponents of a chunk of tiles, and
// the chunk's tile order (largest compact K first), computed here from tb.kt;
// tc_local_tiles on the same batch uses all three.
int tc_slice_workspace(ctc_molecule* mol, const TileBatch& tb, int nqa, cudaStream_t st,
                       int8_t** planes, int32_t** eexp, const int32_t** order);
int tc_local_tiles(ctc_molecule* mol, const LocalPlan& plan, const TileBatch& tb,
                   const ctc_params* prm, const ctc_outputs* out, cudaStream_t st);

// ---- FP64 path (ctc_local.cu) ----
int fp64_local_tiles(ctc_molecule* mol, const LocalPlan& plan, const TileBatch& tb,
                     const ctc_params* prm, const ctc_outputs* out, cudaStream_t st);

// per-point finalisation shared by the contraction kernels (ctc_local.cu)
struct LocalSums;

// Host copy of D (internal order) brought up to date after a device-side
// replacement (ctc_molecule_set_density_matrix); synchronises the device.
int refresh_host_density(ctc_molecule* mol);

// ---- ESP (ctc_esp.cu) ----
int eval_esp(ctc_molecule* mol, const double* d_points, int64_t n, double* d_out, cudaStream_t st);
// [0] kept primitive pairs, [1] FP64 flops per point, [2] Hermite coefficients, [3] mean L
int esp_info(ctc_molecule* mol, double* info);
void destroy_esp(ctc_molecule* mol);

// ---- adjoint (ctc_adjoint.cu) ----
int eval_adjoint(ctc_molecule* mol, const double* d_points, int64_t n, const double* v_rho,
                 const double* v_grad, double* dLdD, double* dLdR, cudaStream_t st);

// chunk size (points) for a given AO footprint
int64_t chunk_points(const ctc_molecule* mol, int nq_ao);

// status word helpers: post_status enqueues the copy of the word after the
// kernels just launched (no wait), poll_status reports a landed copy without
// waiting, check_status synchronises the stream and reports
int post_status(ctc_molecule* mol, cudaStream_t st);
int poll_status(ctc_molecule* mol, cudaStream_t st);
int check_status(ctc_molecule* mol, cudaStream_t st, const char* what);

// Records a start/stop event pair around a launch when profiling is on.
struct ProfScope {
  ctc_molecule* mol;
  int kind;
  cudaStream_t st;
  cudaEvent_t b = nullptr, e = nullptr;
  ProfScope(ctc_molecule* m, int k, cudaStream_t s) : mol(m), kind(k), st(s) {
    if (mol->prof && cudaEventCreate(&b) == cudaSuccess && cudaEventCreate(&e) == cudaSuccess)
      cudaEventRecord(b, st);
  }
  ~ProfScope() {
    if (b && e) {
      cudaEventRecord(e, st);
      mol->prof_ev[kind].push_back({b, e});
    }
  }
};

}  // namespace ctc
