// noalloc.cu -- an HLLC step for callers that cannot allocate device memory.
//
// rb_hllc_step takes its scratch (the stage-1 state U1, the per-tile loss ledger,
// reduction slots) from a workspace the caller allocates. Some callers cannot do
// that: a host that owns every device allocation through its own allocator (a
// game or visualisation engine embedding the solver, a plugin host that forbids
// new allocations after start-up), a framework whose allocator is frozen while it
// records a CUDA graph, or a stepping loop that cannot afford the implicit device
// synchronisation of cudaMalloc/cudaFree. rb_hllc_step_noalloc serves them: its
// scratch is the file-scope array below, which a GPU reserves when the library's
// device code is loaded on it (with lazy module loading, at the first call) and
// holds until the process exits.
//
// Limits and sharing:
//  * at most kMaxCells cells (1,048,576, e.g. 1024 x 1024) per call; larger grids
//    are rejected with RB_ERR_ARG;
//  * every call uses the same array and leaves its contents behind; the loss
//    ledger, which must start at zero, is cleared at the start of each call, so
//    calls that overlap on the GPU (different streams, or threads racing on one
//    device) corrupt each other's scratch;
//  * the error word in the array is sticky: a step that produces a non-finite
//    state sets RB_DEVERR_NONFINITE there, and it stays set until
//    rb_hllc_noalloc_read_error reads and clears it;
//  * the first call on each device looks up the array's device address with
//    cudaGetSymbolAddress (with that device current); under CUDA's lazy module
//    loading (the default since CUDA 12.2) that lookup is also when the device
//    reserves the array. Make that first call at start-up, before any stream
//    capture on the device and before the host's allocator is frozen.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "rb_common.cuh"
#include "rb_kernels.h"

namespace {

constexpr int64_t kMaxCells = int64_t(1) << 20;
constexpr int64_t kMaxTiles = int64_t(1) << 17;  // ledger slots; any shape within kMaxCells needs fewer
constexpr size_t kPlane = (size_t)kMaxCells * sizeof(float);
constexpr size_t kLedgerOff = rb::WS_LEDGER;
constexpr size_t kU1Off = kLedgerOff + (size_t)kMaxTiles * 2 * sizeof(double);
constexpr size_t kScratchBytes = kU1Off + 3 * kPlane;  // ~14.1 MiB

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_addr[kMaxDevices] = {nullptr};

int fail(int code, const char* msg) {
  rb::set_last_error(msg);  // read back with rb_last_error
  return code;
}

// The device address of the scratch array on the current device (looked up once).
int scratch_address(unsigned char** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return fail(RB_ERR_CUDA, "rb_hllc_step_noalloc: no usable current CUDA device");
  std::lock_guard<std::mutex> lock(g_mu);
  if (g_addr[dev] == nullptr) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      return fail(RB_ERR_CUDA, "rb_hllc_step_noalloc: cudaGetSymbolAddress of the static scratch failed");
    g_addr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_addr[dev];
  return RB_OK;
}

}  // namespace

extern "C" int rb_hllc_step_noalloc(const rb_hllc_fields* f, int32_t cur, const rb_step_args* a, double* loss_out,
                                    void* stream) {
  static const char* who = "rb_hllc_step_noalloc";
  if (f == nullptr || a == nullptr) return fail(RB_ERR_ARG, "rb_hllc_step_noalloc: null argument");
  int rc = rb::check_grid(f->ny, f->nx, f->dx, who);
  if (rc) return rc;
  if ((int64_t)f->ny * (int64_t)f->nx > kMaxCells)
    return fail(RB_ERR_ARG,
                "rb_hllc_step_noalloc: grid exceeds the 1048576-cell static scratch (use rb_hllc_step with a "
                "workspace)");
  // one read of the kernel variant serves the tile count, the launches and the ledger sum
  const int variant = rb::hllc_current_variant();
  const int64_t tiles = (int64_t)rb::hllc_tiles_of(variant, f->ny, f->nx);
  if (tiles > kMaxTiles)
    return fail(RB_ERR_ARG, "rb_hllc_step_noalloc: grid shape needs more ledger slots than the static scratch has");
  if (cur != 0 && cur != 1) return fail(RB_ERR_ARG, "rb_hllc_step_noalloc: cur must be 0 or 1");
  if ((rc = rb::check_dt(a->dt, who))) return rc;
  if ((rc = rb::check_bc(f->bc, true, who))) return rc;
  if (!f->h[0] || !f->h[1] || !f->hu[0] || !f->hu[1] || !f->hv[0] || !f->hv[1] || !f->z || !f->n)
    return fail(RB_ERR_ARG, "rb_hllc_step_noalloc: missing state buffer");

  unsigned char* base = nullptr;
  if ((rc = scratch_address(&base))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t nslots = (size_t)tiles;
  // The ledger must start at zero; U1 and the sum partials are overwritten before
  // they are read, and the error word accumulates until it is read.
  if (cudaMemsetAsync(base + kLedgerOff, 0, nslots * 2 * sizeof(double), s) != cudaSuccess)
    return fail(RB_ERR_CUDA, "rb_hllc_step_noalloc: clearing the static scratch failed");

  const bool banks = f->infil != nullptr || f->bc[0] == RB_BC_OPEN || f->bc[1] == RB_BC_OPEN ||
                     f->bc[2] == RB_BC_OPEN || f->bc[3] == RB_BC_OPEN || f->bc[0] == RB_BC_STAGE ||
                     f->bc[1] == RB_BC_STAGE || f->bc[2] == RB_BC_STAGE || f->bc[3] == RB_BC_STAGE;
  rb::HllcParams p{};
  p.ny = f->ny;
  p.nx = f->nx;
  p.dx32 = (float)f->dx;
  p.dt32 = (float)a->dt;
  p.cur = cur;
  p.z = f->z;
  p.n = f->n;
  for (int b = 0; b < 2; b++) {
    p.hb[b] = f->h[b];
    p.hub[b] = f->hu[b];
    p.hvb[b] = f->hv[b];
  }
  p.h1 = (float*)(base + kU1Off);
  p.hu1 = (float*)(base + kU1Off + kPlane);
  p.hv1 = (float*)(base + kU1Off + 2 * kPlane);
  p.h_comp = f->h_comp;
  p.rain_field = f->rain_field;
  p.infil = f->infil;
  p.rain32 = (float)a->rain;
  p.scale32 = (float)a->rain_scale;
  p.rain_mode = (f->h_comp != nullptr && f->rain_field == nullptr) ? 1 : (a->rain != 0.0 ? 2 : 0);
  for (int e = 0; e < 4; e++) {
    p.bc[e] = f->bc[e];
    p.stage[e] = (float)a->stage[e];
  }
  p.wt = 0.5 * a->dt / f->dx;
  p.ledger = banks ? (double*)(base + kLedgerOff) : nullptr;
  p.err = &reinterpret_cast<rb::WsHeader*>(base)->err;
  p.clk = nullptr;
  p.smax_key = nullptr;
  if (rb::hllc_stage_launch_variant(p, 1, variant, s) != cudaSuccess ||
      rb::hllc_stage_launch_variant(p, 2, variant, s) != cudaSuccess)
    return fail(RB_ERR_CUDA, "rb_hllc_step_noalloc: kernel launch failed");
  if (loss_out != nullptr &&
      rb::sum_ledger((const double*)(base + kLedgerOff), nslots, (double*)(base + rb::WS_PARTIALS), loss_out, s) !=
          cudaSuccess)
    return fail(RB_ERR_CUDA, "rb_hllc_step_noalloc: ledger sum launch failed");
  return RB_OK;
}

extern "C" int rb_hllc_noalloc_read_error(uint32_t* err_out, void* stream) {
  if (err_out == nullptr) return fail(RB_ERR_ARG, "rb_hllc_noalloc_read_error: null argument");
  unsigned char* base = nullptr;
  int rc = scratch_address(&base);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  unsigned int* word = &reinterpret_cast<rb::WsHeader*>(base)->err;
  unsigned int host = 0;
  if (cudaMemcpyAsync(&host, word, sizeof host, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemsetAsync(word, 0, sizeof(unsigned int), s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
    return fail(RB_ERR_CUDA, "rb_hllc_noalloc_read_error: reading the static scratch's error word failed");
  *err_out = host;
  return RB_OK;
}
