// ctc_noalloc.cu -- local descriptors in the FP64 form without any device
// allocation inside the call.
//
// Who needs this.  ctc_eval_local sizes its chunk workspace to the request and
// takes it from the stream-ordered allocator (cudaMallocAsync) on first use.
// Some callers cannot let a library allocate device memory during a call:
//   * applications that reserve nearly all of HBM up front for their own
//     caching allocator or memory arena (a serving process, a large simulation
//     code) -- a later cudaMalloc from a library fails or fragments their pool;
//   * pipelines that allocate only at start-up by policy, so that a long run
//     can never fail with out-of-memory halfway through;
//   * processes that share a GPU under a fixed device-memory quota (for
//     example an MPS client with a pinned memory limit), where a library's own
//     allocation counts against the caller's quota and can fail mid-run.
// For them ctc_eval_local_noalloc runs the same screened tile pipeline and the
// same kernels (point tiling, screening, AO block, FP64 contraction and
// descriptor epilogue) with all of its scratch carved out of one fixed array
// compiled into this library.
//
// The fixed array.  g_noalloc_scratch is a file-scope __device__ array of
// kNoAllocScratchBytes (64 MiB).  Every GPU on which the library is loaded
// holds those 64 MiB until the process exits, whether or not this entry point
// is used.  In host code the name g_noalloc_scratch is only a host-side
// stand-in for the device symbol, never a device address: the device address
// is looked up once per device with cudaGetSymbolAddress, while that device
// is current, on the first call made on that device, and cached.  Make that
// first call on each device before any stream capture begins.
//
// Limits.  At most kNoAllocMaxPoints (1,048,576) points per call; more points
// are rejected with CTC_ERR_INVALID and a message naming the limit (split the
// request).  The part of the array left after the point sort holds whole
// chunks of point tiles; a basis too large for even one 32-point tile (AO
// block of 10 x 32 x Mpad doubles, about Mpad > 20,000 functions) is
// rejected the same way.  Only the FP64 form is offered: the tensor-core
// form needs per-molecule sliced operands that are allocated at set-up.
//
// Sharing.  All calls on a device share the one array and it keeps the last
// call's contents.  Nothing in it has to start at zero: every region (Morton
// keys, the sorted permutation, tile points, tile lists, AO block with its
// padding) is written by this call before it is read.  Two calls whose work
// overlaps on the GPU race on the array -- calls on different streams, from
// different host threads, or on different molecules alike -- so issue them
// on one stream, or order the streams with events.
#include <mutex>

#include "ctc_tiles.cuh"

namespace ctc {
namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)64 << 20;
constexpr int64_t kNoAllocMaxPoints = (int64_t)1 << 20;
constexpr int kNoAllocMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (looked up once
// per device, then cached).
int noalloc_scratch(void** out) {
  int dev = 0;
  CTC_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices)
    return fail(CTC_ERR_UNSUPPORTED, "ctc_eval_local_noalloc: device ordinal " + std::to_string(dev) +
                                         " beyond the supported " + std::to_string(kNoAllocMaxDevices));
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(CTC_ERR_CUDA, std::string("ctc_eval_local_noalloc: cudaGetSymbolAddress: ") +
                                    cudaGetErrorString(e));
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return CTC_OK;
}

int eval_local_noalloc(ctc_molecule* mol, const double* d_points, int64_t n, const ctc_params* prm,
                       const ctc_outputs* out, cudaStream_t st) {
  int dev = 0;
  CTC_CUDA_TRY(cudaGetDevice(&dev));
  if (dev != mol->device)
    return fail(CTC_ERR_INVALID, "ctc_eval_local_noalloc: the molecule lives on device " +
                                     std::to_string(mol->device) + ", the current device is " +
                                     std::to_string(dev));
  void* base = nullptr;
  int rc = noalloc_scratch(&base);
  if (rc != CTC_OK) return rc;

  const LocalPlan plan = plan_local(out);
  const int TP = 128 / plan.nqa;
  const int64_t ntiles = (n + TP - 1) / TP;

  // Morton order of the points over the molecule's box padded by 12 bohr,
  // the same ordering ctc_eval_local uses.
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int a = 0; a < mol->natom; ++a)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], mol->atom_xyz[3 * a + d]);
      hi[d] = std::max(hi[d], mol->atom_xyz[3 * a + d]);
    }
  if (mol->natom == 0)
    for (int d = 0; d < 3; ++d) { lo[d] = -1; hi[d] = 1; }
  double ext = 0;
  for (int d = 0; d < 3; ++d) {
    lo[d] -= 12.0;
    hi[d] += 12.0;
    ext = std::max(ext, hi[d] - lo[d]);
  }
  size_t sort_tmp = 0;
  CTC_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, sort_tmp, (uint32_t*)nullptr,
                                               (uint32_t*)nullptr, (int32_t*)nullptr,
                                               (int32_t*)nullptr, (int)n, 0, kMortonSortBits,
                                               st));
  Carve cv{(char*)base};
  uint32_t* k_in = cv.take<uint32_t>(n);
  uint32_t* k_out = cv.take<uint32_t>(n);
  int32_t* v_in = cv.take<int32_t>(n);
  int32_t* perm = cv.take<int32_t>(n);
  void* tmp = cv.take<char>(sort_tmp);
  const size_t sort_end = (cv.off + 255) / 256 * 256;
  if (sort_end > kNoAllocScratchBytes)
    return fail(CTC_ERR_INVALID, "ctc_eval_local_noalloc: sorting " + std::to_string(n) +
                                     " points needs " + std::to_string(sort_end) +
                                     " bytes of the fixed 64 MiB scratch");

  // Chunk of tiles: the largest C whose tile lists and AO block fit in what
  // the sort left.
  const size_t ao_per_tile = sizeof(double) * (size_t)plan.nq_ao * TP * mol->Mpad;
  const size_t avail = kNoAllocScratchBytes - sort_end;
  auto chunk_bytes = [&](int64_t c) {
    return tile_bytes(mol, (int)c, TP, mol->Mpad) + 256 + ao_per_tile * (size_t)c;
  };
  int64_t C = std::min<int64_t>(ntiles, (int64_t)(avail / (ao_per_tile + 1)));
  while (C > 0 && chunk_bytes(C) > avail) --C;
  if (C < 1)
    return fail(CTC_ERR_INVALID, "ctc_eval_local_noalloc: one tile of this basis (" +
                                     std::to_string(mol->M) + " functions) needs " +
                                     std::to_string(chunk_bytes(1)) + " bytes, " +
                                     std::to_string(avail) +
                                     " are left in the fixed 64 MiB scratch; use ctc_eval_local");

  TileBatch tb;
  tb.TP = TP;
  tb.Kcap = mol->Mpad;
  tb.nq = plan.nq_ao;
  {
    Carve tc{(char*)base + sort_end};
    tb.xyz = tc.take<double>((size_t)C * TP * 3);
    tb.out = tc.take<int64_t>((size_t)C * TP);
    tb.nsig = tc.take<int32_t>(C);
    tb.ktrue = tc.take<int32_t>(C);
    tb.kt = tc.take<int32_t>(C);
    tb.segs = tc.take<int32_t>((size_t)C * mol->nseg);
    tb.k0 = tc.take<int32_t>((size_t)C * mol->nseg);
    tb.aomap = tc.take<int32_t>((size_t)C * tb.Kcap);
    tb.ao = tc.take<double>(ao_per_tile / sizeof(double) * (size_t)C);
    if (sort_end + tc.off > kNoAllocScratchBytes)
      return fail(CTC_ERR_INVALID, "ctc_eval_local_noalloc: internal scratch layout overflow");
  }

  morton_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_points, n, lo[0], lo[1], lo[2],
                                                              1024.0 / ext, k_in, v_in);
  CTC_CUDA_TRY(cudaGetLastError());
  CTC_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, sort_tmp, k_in, k_out, v_in, perm, (int)n, 0,
                                               kMortonSortBits, st));
  mol->host_launches += 2;
  for (int64_t t0 = 0; t0 < ntiles; t0 += C) {
    tb.C = (int)std::min<int64_t>(C, ntiles - t0);
    const unsigned g = (unsigned)(((int64_t)tb.C * TP + 255) / 256);
    tile_gather_kernel<<<g, 256, 0, st>>>(d_points, perm, n, t0, tb);
    CTC_CUDA_TRY(cudaGetLastError());
    screen_kernel<<<tb.C, kTileThreads, 0, st>>>(mol->d_segs, mol->nseg, tb, 128, mol->d_stats,
                                                 mol->d_status);
    CTC_CUDA_TRY(cudaGetLastError());
    if ((rc = launch_ao_tiles(mol, tb, plan.deriv, st)) != CTC_OK) return rc;
    if ((rc = fp64_local_tiles(mol, plan, tb, prm, out, st)) != CTC_OK) return rc;
    mol->host_launches += 4;
    mol->host_chunks += 1;
  }
  return CTC_OK;
}

}  // namespace
}  // namespace ctc

using namespace ctc;

extern "C" int ctc_eval_local_noalloc(ctc_molecule* mol, const double* d_points, int64_t n,
                                      const ctc_params* params, const ctc_outputs* d_out,
                                      void* stream) {
  if (!mol || !d_out) return fail(CTC_ERR_INVALID, "ctc_eval_local_noalloc: null argument");
  if (n < 0) return fail(CTC_ERR_INVALID, "ctc_eval_local_noalloc: negative point count");
  if (n > kNoAllocMaxPoints)
    return fail(CTC_ERR_INVALID, "ctc_eval_local_noalloc: " + std::to_string(n) +
                                     " points exceed the maximum of " +
                                     std::to_string(kNoAllocMaxPoints) +
                                     " per call (fixed 64 MiB scratch); split the request");
  if (n > 0 && !d_points) return fail(CTC_ERR_INVALID, "ctc_eval_local_noalloc: null points");
  const ctc_outputs* o = d_out;
  if (!(o->rho || o->grad || o->hess || o->lap || o->tau_pd || o->tau_alpha || o->rdg ||
        o->shannon || o->weizsacker || o->thomas_fermi || o->gge || o->general_ked) ||
      n == 0)
    return CTC_OK;
  ctc_params prm;
  if (params) {
    prm = *params;
  } else {
    prm.alpha = 0.0;
    prm.gge_a = 1.0 / 9.0;
    prm.gge_b = 1.0 / 6.0;
    prm.ked_a = 1.0;
  }
  return eval_local_noalloc(mol, d_points, n, &prm, d_out, (cudaStream_t)stream);
}
