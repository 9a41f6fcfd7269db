// snap_sweep_noalloc: the FP64 sweep of all octants and groups for callers
// that cannot allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is not available or not
// allowed -- inside a host callback or another library's allocator-free
// section, in a process whose memory pool is owned by someone else, or in a
// tight real-time loop that must not touch the allocator.  snap_create()
// cannot be used there because it allocates the sweep scratch.
//
// How: the scratch (coefficient tables, work-item tables, tile-boundary faces,
// progress flags, error word) lives in one file-scope __device__ array of
// SNAP_NOALLOC_SCRATCH_BYTES bytes.  The octants are swept one launch at a
// time and accumulated straight into the caller's flux, so no per-octant flux
// slots are needed.  The host side calls no allocating CUDA or library
// routine.
//
// Caveats for callers:
//  - CUDA loads a library's code lazily by default (one module per .cu file
//    here), so the array and the kernels' code are placed on a device when
//    they are first used there: by the set-up call (all three array arguments
//    NULL), or else by the first sweep.  From then on the device holds them
//    until the process exits.  Make that set-up call, with the device
//    current, outside any section that must not allocate.
//  - All calls share the one array and it keeps the contents of the last
//    call; everything that must start at zero is cleared by each call.  Calls
//    that overlap on the GPU (other streams, other host threads) race on it.
//  - The first call on a device looks the array's device address up with
//    cudaGetSymbolAddress (host code cannot use the symbol itself: it is a
//    host-side stand-in, not a device address) and keeps it for that device.
//    Make that first call before any stream capture on that device.  A
//    cudaDeviceReset invalidates the kept address; calls after a reset of
//    the device are not supported.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <string>

#include "device_util.cuh"
#include "internal.h"
#include "snap_b200.h"

using namespace snapb200;

namespace {

__device__ __align__(256) unsigned char g_noalloc_scratch[SNAP_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
void *g_addr[kMaxDevices] = {};

// The device address of the scratch array on the current device (looked up
// once per device).
cudaError_t scratch_address(int device, void **out) {
  std::lock_guard<std::mutex> lk(g_addr_mu);
  if (!g_addr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_addr[device] = p;
  }
  *out = g_addr[device];
  return cudaSuccess;
}

// Coefficient and MMA fragment tables from the quadrature (same content and
// lane order as the tables snap_create builds on the host).
__global__ void noalloc_tables_kernel(const double *mu, const double *eta, const double *xi,
                                      const double *w, const double *ec, double hi, double hj,
                                      double hk, int A, int M, int NT, int MK, int MN,
                                      double *coef, double *bt1, double *bt2) {
  const int AP = 8 * NT, B1 = MK * NT * 32, B2 = 2 * NT * MN * 32;
  const int total = 4 * AP + 8 * B1 + 8 * B2;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    if (i < 4 * AP) {
      const int r = i / AP, a = i % AP;
      double v = 0.0;
      if (a < A) v = r == 0 ? hi * mu[a] : r == 1 ? hj * eta[a] : r == 2 ? hk * xi[a] : w[a];
      coef[i] = v;
    } else if (i < 4 * AP + 8 * B1) {
      const int j = i - 4 * AP, o = j / B1, rem = j % B1;
      const int kt = rem / (NT * 32), nt = (rem / 32) % NT, l = rem % 32;
      const int m = (l & 3) * MK + kt, a = 8 * nt + (l >> 2);
      bt1[(size_t)o * B1 + b1_slot(kt, nt, l, NT, MK, true)] =
          (m < M && a < A) ? ec[((size_t)o * M + m) * A + a] : 0.0;
    } else {
      const int j = i - 4 * AP - 8 * B1, o = j / B2, rem = j % B2;
      const int t = rem / (MN * 32), mt = (rem / 32) % MN, l = rem % 32;
      const int a = 8 * (t >> 1) + 2 * (l & 3) + (t & 1);
      const int r = l >> 2;
      const int m = (r >> 1) * 2 * MN + 2 * mt + (r & 1);
      bt2[(size_t)o * B2 + b2_slot(t, mt, l, MN, true)] =
          (m < M && a < A) ? ec[((size_t)o * M + m) * A + a] * w[a] : 0.0;
    }
  }
}

// Work items of one octant: ordered by tile diagonal, then group, then tile,
// so every item's upstream neighbours precede it.
__global__ void noalloc_items_kernel(int G, int tx_n, int ty_n, int *table, int *index) {
  const int n = G * tx_n * ty_n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int g = i / (tx_n * ty_n), tx = (i / ty_n) % tx_n, ty = i % ty_n;
    const int d = tx + ty;
    int before = 0;   // items on earlier diagonals
    for (int dd = 0; dd < d; ++dd)
      before += min(dd, tx_n - 1) - max(0, dd - (ty_n - 1)) + 1;
    const int on_d = min(d, tx_n - 1) - max(0, d - (ty_n - 1)) + 1;
    const int item = G * before + g * on_d + (tx - max(0, d - (ty_n - 1)));
    table[item] = (g << 16) | (tx << 8) | ty;
    index[(g * tx_n + tx) * ty_n + ty] = item;
  }
}

int fail(int code, const std::string &msg) { return set_last_error(code, msg); }

// Device-side wait limit: SNAP_B200_TIMEOUT_MS as for snap_create, else 2 s.
long long timeout_ns() {
  long long ns = 2000000000LL;
  if (const char *t = getenv("SNAP_B200_TIMEOUT_MS")) ns = atoll(t) * 1000000LL;
  return ns;
}

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace

extern "C" int snap_sweep_noalloc(const snap_config *cfg, const double *qtot, const double *t_xs,
                                  double *flux, void *stream) {
  if (!cfg) return fail(SNAP_ERR_BAD_ARG, "null configuration");
  // all three arrays NULL: set-up only (load the code, look the array up)
  const bool setup_only = !qtot && !t_xs && !flux;
  if (!setup_only && (!qtot || !t_xs || !flux)) return fail(SNAP_ERR_BAD_ARG, "null argument");
  if (cfg->precision != SNAP_FP64) return fail(SNAP_ERR_UNSUPPORTED, "FP64 contexts only");
  if (cfg->nx < 8 || cfg->ny < 8 || cfg->nz < 1 || cfg->nx % 8 || cfg->ny % 8 || cfg->nang < 1 ||
      cfg->nang > 64 || cfg->ng < 1 || cfg->nmom < 1 || cfg->nmom > 4 || !cfg->mu || !cfg->eta ||
      !cfg->xi || !cfg->w || !cfg->ec)
    return fail(SNAP_ERR_BAD_ARG, "invalid configuration (nx, ny multiples of 8; 1..64 angles)");
  if (cfg->nx / 8 > 255 || cfg->ny / 8 > 255 || cfg->ng >= 32768)
    return fail(SNAP_ERR_UNSUPPORTED, "grid or group count beyond the sweep's item encoding");
  cudaStream_t st = (cudaStream_t)stream;
  SweepShape sh{};
  const int A = cfg->nang, M = cfg->nmom * cfg->nmom, G = cfg->ng;
  sh.NT = (A + 7) / 8;
  sh.MK = M == 1 ? 0 : (M + 3) / 4;
  sh.MN = sh.MK == 0 ? 0 : (sh.MK + 1) / 2;
  sh.TY = 8;
  const int AP = 8 * sh.NT, B1 = sh.MK * sh.NT * 32, B2 = 2 * sh.NT * sh.MN * 32;
  const int tiles_x = cfg->nx / 8, tiles_y = cfg->ny / 8;
  const long long n_items = (long long)G * tiles_x * tiles_y;

  // carve the static array
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off = align256(off + bytes);
    return at;
  };
  const size_t o_quad = take(sizeof(double) * (4 * (size_t)A + (size_t)8 * M * A));
  const size_t o_coef = take(sizeof(double) * 4 * AP);
  const size_t o_bt1 = take(sizeof(double) * 8 * (size_t)B1);
  const size_t o_bt2 = take(sizeof(double) * 8 * (size_t)B2);
  const size_t o_bx = take(sizeof(double) * (size_t)n_items * cfg->nz * sh.TY * AP);
  const size_t o_by = take(sizeof(double) * (size_t)n_items * cfg->nz * 8 * AP);
  const size_t o_tab = take(sizeof(int) * (size_t)n_items);
  const size_t o_idx = take(sizeof(int) * (size_t)n_items);
  const size_t n_prog = (size_t)n_items * sh.TY;   // completed steps per (item, warp)
  const size_t o_ctl = take(sizeof(int) * (n_prog + 2));   // progress, counter, error
  if (off > SNAP_NOALLOC_SCRATCH_BYTES)
    return fail(SNAP_ERR_UNSUPPORTED,
                "problem needs " + std::to_string(off) + " bytes of sweep scratch; the static limit "
                "of snap_sweep_noalloc is " + std::to_string((size_t)SNAP_NOALLOC_SCRATCH_BYTES) +
                " bytes (use snap_create/snap_sweep for larger problems)");

  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess || device < 0 || device >= kMaxDevices)
    return fail(SNAP_ERR_CUDA, "no usable current device");
  void *base_v = nullptr;
  e = scratch_address(device, &base_v);
  if (e != cudaSuccess)
    return fail(SNAP_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  char *base = (char *)base_v;
  double *quad = (double *)(base + o_quad);
  int *ctl = (int *)(base + o_ctl);

  if (!sweep_fp64_supported(sh))
    return fail(SNAP_ERR_UNSUPPORTED, "no compiled sweep kernel for this shape");
  int blocks = 0, sms = 0;
  size_t smem = 0;
  e = sweep_fp64_occupancy(sh, &blocks, &smem);
  if (e != cudaSuccess)
    return fail(SNAP_ERR_CUDA, std::string("sweep occupancy query: ") + cudaGetErrorString(e));
  if (blocks < 1) return fail(SNAP_ERR_UNSUPPORTED, "sweep kernel does not fit on the device");
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess || sms < 1)
    return fail(SNAP_ERR_CUDA, std::string("multiprocessor count: ") + cudaGetErrorString(e));
  const int grid = (int)std::min<long long>((long long)blocks * sms, n_items);
  if (setup_only) {
    // the table kernels live in this file's module (loaded by the symbol
    // lookup above); querying them makes sure their code is resident too
    cudaFuncAttributes fa;
    e = cudaFuncGetAttributes(&fa, noalloc_tables_kernel);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, noalloc_items_kernel);
    if (e != cudaSuccess)
      return fail(SNAP_ERR_CUDA, std::string("loading the table kernels: ") + cudaGetErrorString(e));
    return SNAP_OK;
  }

#define NA_CUDA(x)                                                              \
  do {                                                                          \
    cudaError_t e_ = (x);                                                       \
    if (e_ != cudaSuccess) return fail(SNAP_ERR_CUDA, std::string(#x ": ") +    \
                                               cudaGetErrorString(e_));         \
  } while (0)
  NA_CUDA(cudaMemcpyAsync(quad, cfg->mu, sizeof(double) * A, cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(quad + A, cfg->eta, sizeof(double) * A, cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(quad + 2 * A, cfg->xi, sizeof(double) * A, cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(quad + 3 * A, cfg->w, sizeof(double) * A, cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(quad + 4 * A, cfg->ec, sizeof(double) * 8 * M * A,
                          cudaMemcpyHostToDevice, st));
  noalloc_tables_kernel<<<64, 256, 0, st>>>(quad, quad + A, quad + 2 * A, quad + 3 * A,
                                            quad + 4 * A, cfg->hi, cfg->hj, cfg->hk, A, M, sh.NT,
                                            sh.MK, sh.MN, (double *)(base + o_coef),
                                            (double *)(base + o_bt1), (double *)(base + o_bt2));
  NA_CUDA(cudaGetLastError());
  noalloc_items_kernel<<<64, 256, 0, st>>>(G, tiles_x, tiles_y, (int *)(base + o_tab),
                                           (int *)(base + o_idx));
  NA_CUDA(cudaGetLastError());

  SweepParams p{};
  p.nx = cfg->nx;
  p.ny = cfg->ny;
  p.nz = cfg->nz;
  p.M = M;
  p.A = A;
  p.G = G;
  p.tiles_x = tiles_x;
  p.tiles_y = tiles_y;
  p.n_items = (int)n_items;
  p.fixup = cfg->fixup;
  p.timeout_ns = timeout_ns();
  p.item_table = (const int *)(base + o_tab);
  p.item_index = (const int *)(base + o_idx);
  p.qtot = qtot;
  p.t_xs = t_xs;
  p.phi_slots = flux;   // one octant per launch, accumulated into the caller's flux
  p.bx = base + o_bx;
  p.by = base + o_by;
  p.progress = ctl;
  p.counter = ctl + n_prog;
  p.error = ctl + n_prog + 1;
  p.bt1 = base + o_bt1;
  p.bt2 = base + o_bt2;
  p.coef = base + o_coef;
  NA_CUDA(cudaMemsetAsync(p.error, 0, sizeof(int), st));
  for (int oct = 0; oct < 8; ++oct) {
    p.o_base = oct;
    p.accumulate = oct > 0;
    NA_CUDA(cudaMemsetAsync(ctl, 0, sizeof(int) * (n_prog + 1), st));
    NA_CUDA(launch_sweep_fp64(sh, p, grid, st));
  }
  int err = 0;
  NA_CUDA(cudaMemcpyAsync(&err, p.error, sizeof(int), cudaMemcpyDeviceToHost, st));
  NA_CUDA(cudaStreamSynchronize(st));
#undef NA_CUDA
  if (err == DEV_ERR_TIMEOUT)
    return fail(SNAP_ERR_DEVICE_TIMEOUT, "a sweep tile waited past its limit for an upstream tile");
  if (err != 0) return fail(SNAP_ERR_CUDA, "device error word set");
  return SNAP_OK;
}
