// C ABI of snap_b200: context creation, task-level entry points and the host
// driver of the steady-state solve loop (a sequential restatement of the
// reference's predicated loop, snap.cc:409-541).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"
#include "snap_b200.h"

using namespace snapb200;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char *what) {
  return fail(SNAP_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define SNAP_CUDA(call)                                  \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);  \
  } while (0)

}  // namespace

int snapb200::set_last_error(int code, const std::string &msg) { return fail(code, msg); }

struct snap_ctx {
  snap_config cfg{};
  std::vector<double> mu, eta, xi, w, ec;
  int device = 0;
  int fp32 = 0;
  int M = 1, A = 1;
  SweepShape shape{};
  int AP = 8;
  int P = 8;            // octants per sweep launch (= flux slots)
  int tiles_x = 1, tiles_y = 1, n_items = 0;
  int grid = 0;
  long long C = 0;
  long long timeout_ns = 2000000000LL;
  size_t wsize = 8;     // bytes per sweep-side word
  // device buffers
  void *d_coef = nullptr, *d_bt1 = nullptr, *d_bt2 = nullptr;
  void *d_bt1w = nullptr, *d_bt2n = nullptr;   // adjoint tables: ec*w (expansion), ec (accumulation)
  void *d_pc_store = nullptr;                   // forward state for the adjoint
  uint8_t *d_flag_store = nullptr;
  void *d_sbar_slots = nullptr;                 // adjoint of t_xs per octant slot
  bool state_recorded = false;
  int *d_item_table = nullptr, *d_item_index = nullptr;
  // the inner iteration's sweep: work items of gchain groups each (their z
  // columns walked as one), so a warp's pipeline fills and drains once per
  // chain instead of once per group
  int gchain = 1, n_chain_items = 0, grid_chain = 0;
  int *d_chain_table = nullptr, *d_chain_index = nullptr;
  // FP32 contexts: the split-TF32 tensor-core sweep over group pairs
  int tc32 = 0;
  int n_pair_items = 0, grid_tc = 0;
  int grid_td = 0;   // CTAs of the time-dependent tiled sweep (0: not yet sized)
  int *d_pair_table = nullptr, *d_pair_index = nullptr;
  void *d_tc1 = nullptr, *d_tc2 = nullptr;
  uint32_t *d_scat_tc = nullptr;   // BF16 scattering fragments of the tensor-core outer source
  double *d_odm_tab = nullptr;     // FP64 scattering fragments of the outer source
  size_t odm_tab_words = 0;
  double *d_old0 = nullptr;        // [G][C] scalar flux before the current inner sweep
  bool atomic_octants = true;      // inner iterations add octants straight into the flux
  void *d_slots = nullptr, *d_bx = nullptr, *d_by = nullptr;
  size_t slots_bytes = 0;   // octant slots of every group (inner iterations need none)
  size_t slots_alloc = 0;   // bytes of octant slots allocated (first use, sized to its groups)
  size_t sbar_alloc = 0;    // bytes of sigma_t adjoint slots allocated
  int *d_ctrl = nullptr;   // [n_items * TY progress][counter][error][violations]
  int *h_ctrl = nullptr;   // pinned: error, violations, largest change (float bits)
  float prev_inner_df = 0.0f;   // FP32 contexts: largest change of the previous inner iteration
  int withhold_item1 = 0;       // snap_inject_stall: work item + 1 of the next sweep launch
  // general sweep (sweep_wide.cu): shapes the tiled kernel does not cover
  // (ragged meshes, more than 64 angles) and every time-dependent sweep
  bool wide_only = false;       // the tiled kernel cannot run this shape
  double *d_wquad = nullptr;    // [mu, eta, xi, w: 4*A][ec: 8*M*A]
  double *d_wscratch = nullptr; // general sweep: y pencils and z planes of 8*G blocks, or
                                // the x, y and z face planes of the wavefront form
  bool wave = false;            // the general sweep runs in its wavefront form
  double *d_vdelt0 = nullptr;   // [G] zeros: steady-state vdelt
  double *d_vdelt = nullptr;    // [G] vdelt of the current time-dependent solve
  std::vector<double> h_vdelt;
  // adjoint with group batches: the forward state of `state_groups` groups at
  // a time, recorded again for every batch of every adjoint iteration; work
  // items of a batch of g groups in batch_tables[g]
  int state_groups = 0;
  struct BatchTables {
    int n_items = 0;
    int P = 1;   // octants per launch of a batch (more than the context's when the faces allow)
    int *table = nullptr, *index = nullptr;
  };
  std::vector<BatchTables> batch_tables;
  // solve arrays, kept between snap_transport_solve calls (first call allocates)
  void *d_solve = nullptr;
  double *s_txs64 = nullptr, *s_sxs = nullptr, *s_q2 = nullptr, *s_fpo = nullptr;
  void *s_qtot = nullptr, *s_txsw = nullptr;
  size_t scratch_bytes = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;   // whole-solve timing
  cudaEvent_t sw0 = nullptr, sw1 = nullptr;   // sweep timing
  double sweep_ms = 0.0;
  long long sweep_calls = 0, launches = 0;

  int *progress() { return d_ctrl; }
  size_t n_progress() const { return (size_t)std::max(n_items, n_pair_items) * shape.TY; }
  int *counter() { return d_ctrl + n_progress(); }
  int *error() { return d_ctrl + n_progress() + 1; }
  int *violations() { return d_ctrl + n_progress() + 2; }
  unsigned *maxdf() { return (unsigned *)(d_ctrl + n_progress() + 3); }
};

namespace {

void free_ctx(snap_ctx *c) {
  if (!c) return;
  cudaFree(c->d_coef);
  cudaFree(c->d_bt1);
  cudaFree(c->d_bt2);
  cudaFree(c->d_bt1w);
  cudaFree(c->d_bt2n);
  cudaFree(c->d_pc_store);
  cudaFree(c->d_flag_store);
  cudaFree(c->d_sbar_slots);
  cudaFree(c->d_item_table);
  cudaFree(c->d_item_index);
  cudaFree(c->d_chain_table);
  cudaFree(c->d_chain_index);
  cudaFree(c->d_pair_table);
  cudaFree(c->d_pair_index);
  cudaFree(c->d_tc1);
  cudaFree(c->d_tc2);
  cudaFree(c->d_scat_tc);
  cudaFree(c->d_odm_tab);
  cudaFree(c->d_old0);
  cudaFree(c->d_slots);
  cudaFree(c->d_bx);
  cudaFree(c->d_by);
  cudaFree(c->d_ctrl);
  cudaFree(c->d_wquad);
  cudaFree(c->d_wscratch);
  cudaFree(c->d_vdelt0);
  cudaFree(c->d_vdelt);
  cudaFree(c->d_solve);
  for (auto &b : c->batch_tables) {
    cudaFree(b.table);
    cudaFree(b.index);
  }
  if (c->h_ctrl) cudaFreeHost(c->h_ctrl);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->sw0) cudaEventDestroy(c->sw0);
  if (c->sw1) cudaEventDestroy(c->sw1);
  delete c;
}

template <typename T>
int upload(void **dst, const std::vector<T> &v) {
  SNAP_CUDA(cudaMalloc(dst, std::max<size_t>(v.size(), 1) * sizeof(T)));
  SNAP_CUDA(cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return SNAP_OK;
}

// Per-octant MMA operand tables in the lane order of the m8n8k4 fragments
// (always double: both precisions contract on the FP64 tensor cores) and the
// per-angle coefficients in the sweep precision T.
template <typename T>
void build_tables(const snap_ctx *c, std::vector<T> &coef, std::vector<double> &bt1,
                  std::vector<double> &bt2) {
  const int AP = c->AP, NT = c->shape.NT, MK = c->shape.MK, MN = c->shape.MN, M = c->M,
            A = c->A;
  coef.assign(4 * AP, T(0));
  for (int a = 0; a < A; ++a) {
    coef[a] = (T)(c->cfg.hi * c->mu[a]);
    coef[AP + a] = (T)(c->cfg.hj * c->eta[a]);
    coef[2 * AP + a] = (T)(c->cfg.hk * c->xi[a]);
    coef[3 * AP + a] = (T)c->w[a];
  }
  auto ec = [&](int o, int m, int a) { return c->ec[((size_t)o * M + m) * A + a]; };
  const int B1 = MK * NT * 32, B2 = 2 * NT * MN * 32;
  bt1.assign((size_t)8 * B1, 0.0);
  bt2.assign((size_t)8 * B2, 0.0);
  for (int o = 0; o < 8; ++o) {
    for (int kt = 0; kt < MK; ++kt)
      for (int nt = 0; nt < NT; ++nt)
        for (int l = 0; l < 32; ++l) {
          const int m = (l & 3) * MK + kt, a = 8 * nt + (l >> 2);
          bt1[(size_t)o * B1 + b1_slot(kt, nt, l, NT, MK, sizeof(T) == 8)] =
              (m < M && a < A) ? ec(o, m, a) : 0.0;
        }
    for (int t = 0; t < 2 * NT; ++t)
      for (int mt = 0; mt < MN; ++mt)
        for (int l = 0; l < 32; ++l) {
          const int nt = t >> 1, h = t & 1;
          const int a = 8 * nt + 2 * (l & 3) + h;
          const int r = l >> 2;
          const int m = (r >> 1) * 2 * MN + 2 * mt + (r & 1);
          bt2[(size_t)o * B2 + b2_slot(t, mt, l, MN, sizeof(T) == 8)] =
              (m < M && a < A) ? ec(o, m, a) * c->w[a] : 0.0;
        }
  }
}

// x rounded to TF32 (10 explicit mantissa bits), to nearest with ties away
// from zero: add half of the dropped 13-bit field to the magnitude, truncate.
uint32_t tf32_bits(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return u;   // inf / nan unchanged
  return (u + 0x1000u) & 0xffffe000u;
}
float from_bits(uint32_t u) {
  float x;
  std::memcpy(&x, &u, 4);
  return x;
}
// {hi(b0), hi(b1), lo(b0), lo(b1)}: each value split into two TF32 parts
void put_split(uint32_t *dst, double b0, double b1) {
  const float f0 = (float)b0, f1 = (float)b1;
  const uint32_t h0 = tf32_bits(f0), h1 = tf32_bits(f1);
  dst[0] = h0;
  dst[1] = h1;
  dst[2] = tf32_bits(f0 - from_bits(h0));
  dst[3] = tf32_bits(f1 - from_bits(h1));
}

// Fragment tables of the split-TF32 FP32 sweep (m16n8k8 B operands, lane
// l = 4g + t, uint4 per lane):
//   source  [8][KT][NT][32]: ec[m][a] at k = moments 8kt + 2t, 8kt + 2t + 1
//           and n = angle 8nt + g;
//   moments [8][NT][KT][32]: ec[m][a] w[a] at k = angles 8nt + 2t, 8nt + 2t + 1
//           and n = moment 8mt + g.
void build_tc_tables(const snap_ctx *c, std::vector<uint32_t> &tc1, std::vector<uint32_t> &tc2) {
  const int NT = c->shape.NT, KT = c->shape.KT, M = c->M, A = c->A;
  auto ec = [&](int o, int m, int a) {
    return (m < M && a < A) ? c->ec[((size_t)o * M + m) * A + a] : 0.0;
  };
  auto ecw = [&](int o, int m, int a) { return (m < M && a < A) ? ec(o, m, a) * c->w[a] : 0.0; };
  const size_t F = (size_t)KT * NT * 32 * 4;
  tc1.assign(8 * F, 0u);
  tc2.assign(8 * F, 0u);
  for (int o = 0; o < 8; ++o)
    for (int kt = 0; kt < KT; ++kt)
      for (int nt = 0; nt < NT; ++nt)
        for (int l = 0; l < 32; ++l) {
          const int g = l >> 2, t = l & 3;
          put_split(&tc1[o * F + (((size_t)kt * NT + nt) * 32 + l) * 4],
                    ec(o, 8 * kt + 2 * t, 8 * nt + g), ec(o, 8 * kt + 2 * t + 1, 8 * nt + g));
          put_split(&tc2[o * F + (((size_t)nt * KT + kt) * 32 + l) * 4],
                    ecw(o, 8 * kt + g, 8 * nt + 2 * t), ecw(o, 8 * kt + g, 8 * nt + 2 * t + 1));
        }
}

// Adjoint tables: ec*w in the source-expansion layout and ec in the
// accumulation layout (the roles of the forward tables swapped).
void build_adjoint_tables(const snap_ctx *c, std::vector<double> &bt1w, std::vector<double> &bt2n) {
  const int NT = c->shape.NT, MK = c->shape.MK, MN = c->shape.MN, M = c->M, A = c->A;
  auto ec = [&](int o, int m, int a) { return c->ec[((size_t)o * M + m) * A + a]; };
  const int B1 = MK * NT * 32, B2 = 2 * NT * MN * 32;
  bt1w.assign((size_t)8 * B1, 0.0);
  bt2n.assign((size_t)8 * B2, 0.0);
  for (int o = 0; o < 8; ++o) {
    for (int kt = 0; kt < MK; ++kt)
      for (int nt = 0; nt < NT; ++nt)
        for (int l = 0; l < 32; ++l) {
          const int m = (l & 3) * MK + kt, a = 8 * nt + (l >> 2);
          bt1w[(size_t)o * B1 + (kt * NT + nt) * 32 + l] =
              (m < M && a < A) ? ec(o, m, a) * c->w[a] : 0.0;
        }
    for (int t = 0; t < 2 * NT; ++t)
      for (int mt = 0; mt < MN; ++mt)
        for (int l = 0; l < 32; ++l) {
          const int a = 8 * (t >> 1) + 2 * (l & 3) + (t & 1);
          const int r = l >> 2;
          const int m = (r >> 1) * 2 * MN + 2 * mt + (r & 1);
          bt2n[(size_t)o * B2 + (t * MN + mt) * 32 + l] = (m < M && a < A) ? ec(o, m, a) : 0.0;
        }
  }
}

// Work items of one launch, ordered by tile diagonal, then sweep, then tile:
// every item's upstream x and y neighbours precede it.
void build_items(int P, int G, int tx_n, int ty_n, std::vector<int> &table,
                 std::vector<int> &index) {
  const int S = P * G;
  table.clear();
  index.assign((size_t)S * tx_n * ty_n, -1);
  for (int d = 0; d <= tx_n + ty_n - 2; ++d)
    for (int sw = 0; sw < S; ++sw)
      for (int tx = std::max(0, d - (ty_n - 1)); tx <= std::min(d, tx_n - 1); ++tx) {
        const int ty = d - tx;
        index[((size_t)sw * tx_n + tx) * ty_n + ty] = (int)table.size();
        table.push_back((sw << 16) | (tx << 8) | ty);
      }
}

// Time-dependent terms of one inner iteration's sweep.
struct TdArgs {
  const double *vdelt;   // [G]
  const double *tf_in;   // [8][G][C][A]
  double *tf_out;        // [8][G][C][A]
  const double *qim;     // [8][G][C][A] or null
};

// Whether the time-dependent sweep runs on the tiled kernel: FP64 contexts
// with one flux moment whose shape the tiled kernel takes (at most 64
// angles); SNAP_B200_TD_GENERAL=1 sends it to the general kernel.
bool td_tiled(const snap_ctx *c) {
  if (const char *e = getenv("SNAP_B200_TD_GENERAL"))
    if (atoi(e) != 0) return false;
  return !c->wide_only && !c->fp32 && !c->tc32 && c->shape.MK == 0;
}

// mode 0: forward sweep; 1: forward sweep recording the state for the
// adjoint; 2: adjoint sweep (sigma_t adjoint when sbar != null).
// With atomic_flux (forward mode only), every octant adds its moments into
// that FP64 flux [G][C][cmom] instead of writing its slot.
int sweep_launches(snap_ctx *c, const void *qtot, const void *t_xs, cudaStream_t st,
                   int mode = 0, void *sbar = nullptr, double *atomic_flux = nullptr,
                   int g0 = 0, int gn = 0, const TdArgs *td = nullptr) {
  // gn > 0: only groups g0 .. g0+gn-1 (qtot and t_xs hold every group; the
  // slots, the recorded state and sbar hold the batch)
  const bool batch = gn > 0 && gn < c->cfg.ng;
  if (batch && ((int)c->batch_tables.size() <= gn || !c->batch_tables[gn].table))
    return fail(SNAP_ERR_BAD_ARG, "no work items for this group batch");
  SweepParams p{};
  p.nx = c->cfg.nx;
  p.ny = c->cfg.ny;
  p.nz = c->cfg.nz;
  p.M = c->M;
  p.A = c->A;
  p.G = batch ? gn : c->cfg.ng;
  p.tiles_x = c->tiles_x;
  p.tiles_y = c->tiles_y;
  p.n_items = batch ? c->batch_tables[gn].n_items : c->n_items;
  p.fixup = c->cfg.fixup;
  p.timeout_ns = c->timeout_ns;
  p.withhold_item1 = mode == 2 ? 0 : c->withhold_item1;
  c->withhold_item1 = 0;   // one launch only
  p.item_table = batch ? c->batch_tables[gn].table : c->d_item_table;
  p.item_index = batch ? c->batch_tables[gn].index : c->d_item_index;
  p.qtot = (const char *)qtot + (size_t)g0 * c->C * c->M * c->wsize;
  p.t_xs = (const char *)t_xs + (size_t)g0 * c->C * c->wsize;
  const int P = batch ? c->batch_tables[gn].P : c->P;   // octants per launch
  if (!atomic_flux) {
    // octant slots for the groups of this launch (first use allocates)
    const size_t need = (size_t)P * p.G * c->C * c->M * c->wsize;
    if (!c->d_slots || c->slots_alloc < need) {
      cudaFree(c->d_slots);
      c->scratch_bytes -= c->slots_alloc;
      c->slots_alloc = 0;
      if (cudaMalloc(&c->d_slots, need) != cudaSuccess) {
        cudaGetLastError();
        c->d_slots = nullptr;
        return fail(SNAP_ERR_OOM, "cannot allocate the octant flux slots");
      }
      c->slots_alloc = need;
      c->scratch_bytes += need;
    }
  }
  p.phi_slots = atomic_flux ? (void *)atomic_flux : c->d_slots;
  p.atomic_flux = atomic_flux ? 1 : 0;
  p.bx = c->d_bx;
  p.by = c->d_by;
  p.progress = c->progress();
  p.counter = c->counter();
  p.error = c->error();
  p.bt1 = mode == 2 ? c->d_bt1w : c->d_bt1;
  p.bt2 = mode == 2 ? c->d_bt2n : c->d_bt2;
  p.coef = c->d_coef;
  p.pc_store = mode >= 1 ? c->d_pc_store : nullptr;
  p.flag_store = mode >= 1 ? c->d_flag_store : nullptr;
  p.sigt_bar_slots = mode == 2 ? sbar : nullptr;
  int grid = c->grid;
  if (td) {   // the time-dependent form: every octant adds into the FP64 flux
    if (!atomic_flux || mode != 0 || batch) return fail(SNAP_ERR_BAD_ARG, "time-dependent sweep");
    p.vdelt = td->vdelt;
    p.tf_in = td->tf_in;
    p.tf_out = td->tf_out;
    p.qim = td->qim;
    if (c->grid_td == 0) {
      int blocks = 0, sms = 0;
      size_t smem = 0;
      if (sweep_fp64_td_occupancy(c->shape, &blocks, &smem) != cudaSuccess || blocks < 1)
        return fail(SNAP_ERR_UNSUPPORTED, "time-dependent tiled sweep does not fit on the device");
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
      c->grid_td = std::min(blocks * sms, c->n_items);
    }
    grid = c->grid_td;
  }
  const bool tc = c->tc32 && mode != 2;
  if (c->gchain > 1 && mode == 0 && atomic_flux && !td && !batch && !tc) {
    p.gchain = c->gchain;
    p.n_items = c->n_chain_items;
    p.item_table = c->d_chain_table;
    p.item_index = c->d_chain_index;
    grid = c->grid_chain;
  }
  if (tc) {
    p.n_items = c->n_pair_items;
    p.item_table = c->d_pair_table;
    p.item_index = c->d_pair_index;
    p.bt1 = c->d_tc1;
    p.bt2 = c->d_tc2;
    grid = c->grid_tc;
  }
  if (mode == 2) {
    int blocks = 0, sms = 0;
    size_t smem = 0;
    if (adjoint_dispatch(c->fp32, c->shape, 1, nullptr, 0, nullptr, &blocks, &smem) != cudaSuccess ||
        blocks < 1)
      return fail(SNAP_ERR_UNSUPPORTED, "no adjoint kernel for this shape (8x4 tiles only)");
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    grid = std::min(blocks * sms, p.n_items);
  }
  if (batch) grid = std::min(grid, p.n_items);
  for (int L = 0; L < 8 / P; ++L) {
    p.o_base = L * P;
    p.accumulate = L > 0;
    SNAP_CUDA(cudaMemsetAsync(c->d_ctrl, 0, sizeof(int) * (c->n_progress() + 1), st));
    cudaError_t e;
    if (td)
      e = launch_sweep_fp64_td(c->shape, p, grid, st);
    else if (mode == 2)
      e = adjoint_dispatch(c->fp32, c->shape, 0, &p, grid, st, nullptr, nullptr);
    else if (tc)
      e = launch_sweep_tc32(c->shape, p, grid, st);
    else
      e = c->fp32 ? launch_sweep_fp32(c->shape, p, grid, st)
                  : launch_sweep_fp64(c->shape, p, grid, st);
    if (e != cudaSuccess) return cuda_fail(e, "sweep launch");
    ++c->launches;
  }
  return SNAP_OK;
}

// Sweep plus the octant-slot reduction into `flux` (with the inner test when
// test != 0), bracketed by the context's sweep events.
int timed_sweep(snap_ctx *c, const void *qtot, const void *t_xs, void *flux, int flux_fp32,
                double *flux64, int test, double epsi, cudaStream_t st) {
  SNAP_CUDA(cudaEventRecord(c->sw0, st));
  int rc = sweep_launches(c, qtot, t_xs, st);
  if (rc) return rc;
  SNAP_CUDA(cudaEventRecord(c->sw1, st));
  SNAP_CUDA(k_reduce_slots(c->d_slots, c->P, c->fp32, flux, flux_fp32, flux64, c->cfg.ng, c->M,
                           c->C, test, epsi, c->violations(), st, test ? c->maxdf() : nullptr));
  ++c->launches;
  return SNAP_OK;
}

void account_sweep(snap_ctx *c) {
  float ms = 0.0f;
  if (cudaEventElapsedTime(&ms, c->sw0, c->sw1) == cudaSuccess) {
    c->sweep_ms += ms;
    ++c->sweep_calls;
  }
}

// Reads the device error word and the violation counter (synchronises).
int read_ctrl(snap_ctx *c, cudaStream_t st, int *violations) {
  SNAP_CUDA(cudaMemcpyAsync(c->h_ctrl, c->error(), 3 * sizeof(int), cudaMemcpyDeviceToHost, st));
  SNAP_CUDA(cudaStreamSynchronize(st));
  if (c->h_ctrl[0] == DEV_ERR_TIMEOUT)
    return fail(SNAP_ERR_DEVICE_TIMEOUT, "a sweep tile waited past its limit for an upstream tile");
  if (c->h_ctrl[0] != 0) return fail(SNAP_ERR_CUDA, "device error word set");
  if (violations) *violations = c->h_ctrl[1];
  return SNAP_OK;
}

int inner_iteration_impl(snap_ctx *c, const double *s_xs, const double *q2grp, const void *t_xs,
                         double *flux, void *qtot, double epsi, int *converged, cudaStream_t st,
                         const TdArgs *td);
int solve_impl(snap_ctx *c, const int32_t *mat, const double *qi, const double *sigt,
               const double *slgg, const double *sigt_scale, double *flux, snap_solve_info *info,
               cudaStream_t st, const snap_time_config *tc);

// Device quadrature tables and face scratch of the general sweep (allocated
// on first use).
int ensure_wide(snap_ctx *c) {
  if (c->d_wscratch) return SNAP_OK;
  const int A = c->A, M = c->M, G = c->cfg.ng;
  // the wavefront form where it takes the shape and its face planes fit in
  // a quarter of the free memory (SNAP_B200_WAVE=0: the cell-by-cell form)
  bool wave = wave_supported(A, M);
  if (const char *e = getenv("SNAP_B200_WAVE"))
    if (atoi(e) == 0) wave = false;
  const size_t wave_bytes =
      sizeof(double) * wave_scratch_doubles(c->cfg.nx, c->cfg.ny, c->cfg.nz, A, 8 * G);
  if (wave) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess || wave_bytes > free_b / 4) wave = false;
  }
  if (!wave && !wide_supported(A, c->cfg.nx, M))
    return fail(SNAP_ERR_UNSUPPORTED, "no general sweep for this shape");
  std::vector<double> q((size_t)4 * A + (size_t)8 * M * A);
  for (int a = 0; a < A; ++a) {
    q[a] = c->mu[a];
    q[A + a] = c->eta[a];
    q[2 * A + a] = c->xi[a];
    q[3 * A + a] = c->w[a];
  }
  std::copy(c->ec.begin(), c->ec.end(), q.begin() + 4 * A);
  int rc = upload((void **)&c->d_wquad, q);
  if (rc) return rc;
  const size_t per_block = (size_t)c->cfg.nx * (1 + c->cfg.ny) * A;
  const size_t bytes = wave ? wave_bytes : sizeof(double) * per_block * 8 * G;
  if (cudaMalloc((void **)&c->d_wscratch, bytes) != cudaSuccess ||
      cudaMalloc((void **)&c->d_vdelt0, sizeof(double) * G) != cudaSuccess ||
      cudaMemset(c->d_vdelt0, 0, sizeof(double) * G) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(c->d_wscratch);
    c->d_wscratch = nullptr;
    return fail(SNAP_ERR_OOM, "cannot allocate the general sweep's face scratch");
  }
  c->scratch_bytes += bytes + sizeof(double) * G;
  c->wave = wave;
  return SNAP_OK;
}

// One general sweep of all 8 octants and groups, adding every octant's
// moments into `flux` (double).  td != 0: time-dependent terms with vdelt
// [G], tf_in/tf_out [8][G][C][A]; qim: per-angle source or null.
int wide_sweep(snap_ctx *c, const double *qtot, const double *t_xs, double *flux,
               const double *vdelt, const double *tf_in, double *tf_out, const double *qim,
               cudaStream_t st) {
  int rc = ensure_wide(c);
  if (rc) return rc;
  const int A = c->A, M = c->M, G = c->cfg.ng;
  WideParams p{};
  p.nx = c->cfg.nx;
  p.ny = c->cfg.ny;
  p.nz = c->cfg.nz;
  p.A = A;
  p.M = M;
  p.G = G;
  p.o_base = 0;
  p.fixup = c->cfg.fixup;
  p.td = (vdelt && tf_in && tf_out) ? 1 : 0;
  p.hi = c->cfg.hi;
  p.hj = c->cfg.hj;
  p.hk = c->cfg.hk;
  p.mu = c->d_wquad;
  p.eta = c->d_wquad + A;
  p.xi = c->d_wquad + 2 * A;
  p.w = c->d_wquad + 3 * A;
  p.ec = c->d_wquad + 4 * A;
  p.qtot = qtot;
  p.t_xs = t_xs;
  p.vdelt = p.td ? vdelt : c->d_vdelt0;
  p.tf_in = tf_in;
  p.tf_out = tf_out;
  p.qim = qim;
  p.flux = flux;
  if (c->wave) {
    const size_t blocks = (size_t)8 * G;
    p.wx = c->d_wscratch;
    p.wy = p.wx + (size_t)c->cfg.ny * c->cfg.nz * A * blocks;
    p.wz = p.wy + (size_t)c->cfg.nx * c->cfg.nz * A * blocks;
    SNAP_CUDA(launch_sweep_wave(p, 8 * G, st));
  } else {
    p.ypen = c->d_wscratch;
    p.zpl = c->d_wscratch + (size_t)c->cfg.nx * A * 8 * G;
    SNAP_CUDA(launch_sweep_wide(p, 8 * G, st));
  }
  ++c->launches;
  return SNAP_OK;
}

}  // namespace

extern "C" {

const char *snap_last_error(void) { return g_last_error.c_str(); }

// The outer source of output groups g_lo .. g_lo+g_n-1 from the flux of G
// groups (kernels.cu: FP64 tensor-core form with its fragment table in
// d_odm_tab, grown on demand; the SIMT form when the table cannot be had).
cudaError_t outer_source(snap_ctx *c, const double *qi, const double *slgg, const int32_t *mat,
                         const double *flux, double *q2, int G, int g_lo, int g_n,
                         cudaStream_t st) {
  const size_t words = outer_dmma_table_words(G, g_n, c->cfg.nmat, c->cfg.nmom);
  if (words > c->odm_tab_words) {
    cudaFree(c->d_odm_tab);
    c->d_odm_tab = nullptr;
    c->odm_tab_words = 0;
    if (cudaMalloc((void **)&c->d_odm_tab, sizeof(double) * words) == cudaSuccess)
      c->odm_tab_words = words;
    else
      cudaGetLastError();   // fall back to the SIMT form
  }
  int launches = 0;
  const cudaError_t e = k_outer_source_groups(qi, slgg, mat, flux, q2, c->d_odm_tab, G,
                                              c->cfg.nmat, c->cfg.nmom, c->M, c->C, g_lo, g_n,
                                              &launches, st);
  c->launches += launches;
  return e;
}

int snap_create(const snap_config *cfg, int device, snap_ctx **out) {
  if (!cfg || !out) return fail(SNAP_ERR_BAD_ARG, "null argument");
  *out = nullptr;
  if (cfg->nx < 1 || cfg->ny < 1 || cfg->nz < 1 || cfg->nang < 1 || cfg->ng < 1 || cfg->nmom < 1 ||
      cfg->nmom > 4 || cfg->nmat < 1 || !cfg->mu || !cfg->eta || !cfg->xi || !cfg->w || !cfg->ec)
    return fail(SNAP_ERR_BAD_ARG, "invalid configuration");
  if (cfg->precision != SNAP_FP64 && cfg->precision != SNAP_FP32)
    return fail(SNAP_ERR_BAD_ARG, "unknown precision");
  int tile_y = cfg->ny % 4 == 0 ? 4 : 8;
  if (const char *te = getenv("SNAP_B200_TILE_Y")) tile_y = atoi(te) == 8 ? 8 : 4;
  // the tiled kernel: 8 x tile_y column tiles, at most 64 angles in registers;
  // other shapes run the general sweep (FP64 only, forward sweeps only)
  const bool tiled_ok = cfg->nx % 8 == 0 && cfg->ny % tile_y == 0 && cfg->nang <= 64 &&
                        cfg->nx / 8 <= 255 && cfg->ny / 8 <= 255 &&
                        (long long)8 * cfg->ng < 32768 &&
                        (long long)cfg->nx * cfg->ny * cfg->nz * cfg->nmom * cfg->nmom < (1LL << 31);
  if (!tiled_ok) {
    if (cfg->precision != SNAP_FP64)
      return fail(SNAP_ERR_UNSUPPORTED,
                  "FP32 sweeps need nx % 8 == 0, ny % 4 == 0 and at most 64 angles per octant");
    if (!wide_supported(cfg->nang, cfg->nx, cfg->nmom * cfg->nmom))
      return fail(SNAP_ERR_UNSUPPORTED, "at most 2048 angles per octant");
  }

  snap_ctx *c = new snap_ctx();
  c->cfg = *cfg;
  c->device = device;
  c->fp32 = cfg->precision == SNAP_FP32;
  c->A = cfg->nang;
  c->M = cfg->nmom * cfg->nmom;
  c->C = (long long)cfg->nx * cfg->ny * cfg->nz;
  c->mu.assign(cfg->mu, cfg->mu + cfg->nang);
  c->eta.assign(cfg->eta, cfg->eta + cfg->nang);
  c->xi.assign(cfg->xi, cfg->xi + cfg->nang);
  c->w.assign(cfg->w, cfg->w + cfg->nang);
  c->ec.assign(cfg->ec, cfg->ec + (size_t)8 * c->M * cfg->nang);
  c->cfg.mu = c->mu.data();
  c->cfg.eta = c->eta.data();
  c->cfg.xi = c->xi.data();
  c->cfg.w = c->w.data();
  c->cfg.ec = c->ec.data();
  if (const char *t = getenv("SNAP_B200_TIMEOUT_MS")) c->timeout_ns = atoll(t) * 1000000LL;

  c->shape.NT = (c->A + 7) / 8;
  c->shape.MK = c->M == 1 ? 0 : (c->M + 3) / 4;
  c->shape.MN = c->shape.MK == 0 ? 0 : (c->shape.MK + 1) / 2;
  c->shape.TY = tile_y;
  c->shape.KT = c->M == 1 ? 0 : (c->M + 7) / 8;
  c->AP = 8 * c->shape.NT;
  c->wsize = c->fp32 ? sizeof(float) : sizeof(double);
  const bool ok = c->fp32 ? sweep_fp32_supported(c->shape) : sweep_fp64_supported(c->shape);
  if (!tiled_ok || !ok) {
    if (c->fp32 || !wide_supported(c->A, cfg->nx, c->M)) {
      free_ctx(c);
      return fail(SNAP_ERR_UNSUPPORTED, "no compiled sweep kernel for this shape");
    }
    // general sweep only: no tiled tables or tile scratch
    c->wide_only = true;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
      free_ctx(c);
      return cuda_fail(e, "cudaSetDevice");
    }
    c->P = 8;
    c->n_items = 0;
    if (cudaMalloc((void **)&c->d_ctrl, sizeof(int) * 4) != cudaSuccess ||
        cudaMalloc((void **)&c->d_old0, sizeof(double) * (size_t)cfg->ng * c->C) != cudaSuccess ||
        cudaMemset(c->d_ctrl, 0, sizeof(int) * 4) != cudaSuccess ||
        cudaMallocHost((void **)&c->h_ctrl, 4 * sizeof(int)) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
        cudaEventCreate(&c->sw0) != cudaSuccess || cudaEventCreate(&c->sw1) != cudaSuccess) {
      cudaGetLastError();
      free_ctx(c);
      return fail(SNAP_ERR_OOM, "cannot allocate context buffers");
    }
    c->scratch_bytes = sizeof(int) * 4 + sizeof(double) * (size_t)cfg->ng * c->C;
    int rc = ensure_wide(c);
    if (rc) {
      free_ctx(c);
      return rc;
    }
    *out = c;
    return SNAP_OK;
  }
  c->tiles_x = cfg->nx / 8;
  c->tiles_y = cfg->ny / c->shape.TY;
  // FP32 contexts can sweep with the contractions on the TF32 tensor cores
  // (group pairs); measured slower than the FP64-tensor-core contractions on
  // the 64^3 deck, so it is opt-in
  c->tc32 = c->fp32 && sweep_tc32_supported(c->shape) && getenv("SNAP_B200_FP32_TC") &&
            atoi(getenv("SNAP_B200_FP32_TC")) != 0;

  int rc;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) {
    free_ctx(c);
    return cuda_fail(e, "cudaSetDevice");
  }
  // tables
  if (c->fp32) {
    std::vector<float> coef;
    std::vector<double> bt1, bt2;
    build_tables<float>(c, coef, bt1, bt2);
    if ((rc = upload(&c->d_coef, coef)) || (rc = upload(&c->d_bt1, bt1)) ||
        (rc = upload(&c->d_bt2, bt2))) {
      free_ctx(c);
      return rc;
    }
    if (c->tc32) {
      std::vector<uint32_t> tc1, tc2;
      build_tc_tables(c, tc1, tc2);
      if ((rc = upload(&c->d_tc1, tc1)) || (rc = upload(&c->d_tc2, tc2))) {
        free_ctx(c);
        return rc;
      }
    }
  } else {
    std::vector<double> coef, bt1, bt2;
    build_tables<double>(c, coef, bt1, bt2);
    if ((rc = upload(&c->d_coef, coef)) || (rc = upload(&c->d_bt1, bt1)) ||
        (rc = upload(&c->d_bt2, bt2))) {
      free_ctx(c);
      return rc;
    }
  }
  {
    std::vector<double> bt1w, bt2n;
    build_adjoint_tables(c, bt1w, bt2n);
    if ((rc = upload(&c->d_bt1w, bt1w)) || (rc = upload(&c->d_bt2n, bt2n))) {
      free_ctx(c);
      return rc;
    }
  }
  // flux slots and tile faces: as many octants per launch as memory allows
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  const size_t budget = (size_t)(0.55 * (double)free_b);
  const int G = cfg->ng;
  const int G_faces = c->tc32 ? 2 * ((G + 1) / 2) : G;   // group pairs carry a phantom member
  auto scratch_for = [&](int P) {
    const size_t items = (size_t)P * G_faces * c->tiles_x * c->tiles_y;
    return (size_t)P * G * c->C * c->M * c->wsize +
           items * (size_t)cfg->nz * (c->shape.TY + 8) * c->AP * c->wsize;
  };
  int P = 8;
  if (const char *pe = getenv("SNAP_B200_OCTANTS_PER_LAUNCH")) P = atoi(pe);
  if (P != 1 && P != 2 && P != 4 && P != 8) P = 8;
  while (P > 1 && scratch_for(P) > budget) P /= 2;
  c->P = P;
  std::vector<int> table, index;
  build_items(P, G, c->tiles_x, c->tiles_y, table, index);
  c->n_items = (int)table.size();
  if ((rc = upload((void **)&c->d_item_table, table)) ||
      (rc = upload((void **)&c->d_item_index, index))) {
    free_ctx(c);
    return rc;
  }
  if (c->tc32) {
    build_items(P, (G + 1) / 2, c->tiles_x, c->tiles_y, table, index);
    c->n_pair_items = (int)table.size();
    if ((rc = upload((void **)&c->d_pair_table, table)) ||
        (rc = upload((void **)&c->d_pair_index, index))) {
      free_ctx(c);
      return rc;
    }
  }
  const size_t slots_b = (size_t)P * G * c->C * c->M * c->wsize;
  // tile-edge faces: per item of one group, or of one group pair (two groups)
  const size_t face_items = std::max((size_t)c->n_items, (size_t)2 * c->n_pair_items);
  const size_t bx_b = face_items * cfg->nz * c->shape.TY * c->AP * c->wsize;
  const size_t by_b = face_items * cfg->nz * 8 * c->AP * c->wsize;
  c->slots_bytes = slots_b;
  if (cudaMalloc(&c->d_bx, bx_b) != cudaSuccess ||
      cudaMalloc(&c->d_by, by_b) != cudaSuccess ||
      cudaMalloc((void **)&c->d_ctrl, sizeof(int) * (c->n_progress() + 4)) != cudaSuccess ||
      cudaMalloc((void **)&c->d_old0, sizeof(double) * (size_t)G * c->C) != cudaSuccess) {
    cudaGetLastError();
    free_ctx(c);
    return fail(SNAP_ERR_OOM, "cannot allocate sweep scratch");
  }
  c->scratch_bytes = bx_b + by_b + sizeof(int) * (c->n_progress() + 4) +
                     sizeof(double) * (size_t)G * c->C;
  if (const char *os = getenv("SNAP_B200_OCTANT_SLOTS")) c->atomic_octants = atoi(os) == 0;
  if (cudaMemset(c->d_ctrl, 0, sizeof(int) * (c->n_progress() + 4)) != cudaSuccess ||
      cudaMallocHost((void **)&c->h_ctrl, 4 * sizeof(int)) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
      cudaEventCreate(&c->sw0) != cudaSuccess || cudaEventCreate(&c->sw1) != cudaSuccess) {
    free_ctx(c);
    return fail(SNAP_ERR_CUDA, "context setup failed");
  }
  int blocks = 0, sms = 0;
  size_t smem = 0;
  e = c->fp32 ? sweep_fp32_occupancy(c->shape, &blocks, &smem)
              : sweep_fp64_occupancy(c->shape, &blocks, &smem);
  if (e != cudaSuccess || blocks < 1) {
    free_ctx(c);
    return fail(SNAP_ERR_UNSUPPORTED, "sweep kernel does not fit on the device");
  }
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  c->grid = std::min(blocks * sms, c->n_items);
  if (const char *ge = getenv("SNAP_B200_GRID")) c->grid = std::max(1, std::min(atoi(ge), c->grid));
  // group chains: the smallest divisor of G whose chained column has at
  // least 1024 planes (the pipeline's fill and drain then cost under 1 %), or
  // a shorter one where that would leave fewer than 12 work items per
  // resident CTA (load balance over the queue).  Deck 2 (64 planes, 32
  // groups, FP64 sweep ms): chains of 1 / 2 / 4 / 8 / 16 groups 18.8 / 17.8 /
  // 17.4 / 17.7 / 18.7; FP32 with 2 / 4 / 8: 12.33 / 12.20 / 12.60; 128^3 /
  // 64 groups (FP64, from a zero flux): 1 / 2 / 8 / 32: 362 / 350 / 346 / 365.
  // SNAP_B200_GROUP_CHAIN sets it (a divisor of G; 1: none).  A divisor
  // keeps every item's face buffers inside the ones allocated above.
  {
    int gc = 0;
    if (const char *ce = getenv("SNAP_B200_GROUP_CHAIN")) gc = atoi(ce);
    if (gc < 1 || gc > G || G % gc != 0) {
      gc = G;
      for (int d = G; d >= 1; --d)
        if (G % d == 0 && (long long)d * cfg->nz >= 1024) gc = d;
      while (gc > 1 && (long long)c->n_items / gc < 12LL * c->grid) {
        int d = gc - 1;
        while (G % d != 0) --d;
        gc = d;
      }
    }
    if (gc > 1 && !c->wide_only && !c->tc32) {
      build_items(P, G / gc, c->tiles_x, c->tiles_y, table, index);
      if ((rc = upload((void **)&c->d_chain_table, table)) ||
          (rc = upload((void **)&c->d_chain_index, index))) {
        free_ctx(c);
        return rc;
      }
      c->gchain = gc;
      c->n_chain_items = (int)table.size();
      c->grid_chain = std::min(c->grid, c->n_chain_items);
    }
  }
  if (c->tc32) {
    e = sweep_tc32_occupancy(c->shape, &blocks, &smem);
    if (e != cudaSuccess || blocks < 1) {
      free_ctx(c);
      return fail(SNAP_ERR_UNSUPPORTED, "FP32 tensor-core sweep kernel does not fit on the device");
    }
    c->grid_tc = std::min(blocks * sms, c->n_pair_items);
  }
  // the outer source's fragment table, so that solves allocate nothing for it
  {
    const size_t words = outer_dmma_table_words(G, G, c->cfg.nmat, c->cfg.nmom);
    if (cudaMalloc((void **)&c->d_odm_tab, sizeof(double) * words) == cudaSuccess)
      c->odm_tab_words = words;
    else
      cudaGetLastError();
  }
  *out = c;
  return SNAP_OK;
}

int snap_destroy(snap_ctx *ctx) {
  free_ctx(ctx);
  return SNAP_OK;
}

size_t snap_scratch_bytes(const snap_ctx *ctx) { return ctx ? ctx->scratch_bytes : 0; }

int snap_inject_stall(snap_ctx *c, int item) {
  if (!c) return fail(SNAP_ERR_BAD_ARG, "null context");
  if (c->tc32 || c->wide_only)
    return fail(SNAP_ERR_UNSUPPORTED, "not available with the TF32 or the general sweep kernel");
  if (item < 0 || item >= c->n_items) return fail(SNAP_ERR_BAD_ARG, "work item out of range");
  c->withhold_item1 = item + 1;
  return SNAP_OK;
}

int snap_expand_xs(snap_ctx *c, const double *sig, const int32_t *mat, double *xs, void *stream) {
  if (!c || !sig || !mat || !xs) return fail(SNAP_ERR_BAD_ARG, "null argument");
  SNAP_CUDA(k_expand_xs(sig, mat, xs, c->cfg.ng, c->cfg.nmat, c->C, (cudaStream_t)stream));
  ++c->launches;
  return SNAP_OK;
}

int snap_expand_scattering_xs(snap_ctx *c, const double *slgg, const int32_t *mat, double *s_xs,
                              void *stream) {
  if (!c || !slgg || !mat || !s_xs) return fail(SNAP_ERR_BAD_ARG, "null argument");
  SNAP_CUDA(k_expand_scat(slgg, mat, s_xs, c->cfg.ng, c->cfg.nmat, c->cfg.nmom, c->C,
                          (cudaStream_t)stream));
  ++c->launches;
  return SNAP_OK;
}

int snap_calc_outer_source(snap_ctx *c, const double *qi, const double *slgg, const int32_t *mat,
                           const double *flux, double *q2grp, void *stream) {
  if (!c || !qi || !slgg || !mat || !flux || !q2grp) return fail(SNAP_ERR_BAD_ARG, "null argument");
  SNAP_CUDA(outer_source(c, qi, slgg, mat, flux, q2grp, c->cfg.ng, 0, c->cfg.ng,
                         (cudaStream_t)stream));
  return SNAP_OK;
}

int snap_calc_outer_source_tc(snap_ctx *c, const double *qi, const double *slgg,
                              const int32_t *mat, const double *flux, double *q2grp, void *stream) {
  if (!c || !qi || !slgg || !mat || !flux || !q2grp) return fail(SNAP_ERR_BAD_ARG, "null argument");
  if (!outer_tc_supported(c->cfg.ng, c->cfg.nmat, c->cfg.nmom))
    return fail(SNAP_ERR_UNSUPPORTED, "too many groups or materials for the tensor-core outer source");
  if (!c->d_scat_tc) {
    const size_t words = outer_tc_table_words(c->cfg.ng, c->cfg.nmat, c->cfg.nmom);
    if (cudaMalloc((void **)&c->d_scat_tc, sizeof(uint32_t) * words) != cudaSuccess) {
      cudaGetLastError();
      c->d_scat_tc = nullptr;
      return fail(SNAP_ERR_OOM, "cannot allocate the tensor-core scattering table");
    }
  }
  SNAP_CUDA(k_outer_source_tc(qi, slgg, mat, flux, q2grp, c->d_scat_tc, c->cfg.ng, c->cfg.nmat,
                              c->cfg.nmom, c->M, c->C, c->error(), c->timeout_ns,
                              (cudaStream_t)stream));
  c->launches += 2;
  return SNAP_OK;
}

int snap_calc_outer_source_groups(snap_ctx *c, int g_lo, int ng_total, const double *qi,
                                  const double *slgg, const int32_t *mat, const double *flux_all,
                                  double *q2grp, void *stream) {
  if (!c || !qi || !slgg || !mat || !flux_all || !q2grp) return fail(SNAP_ERR_BAD_ARG, "null argument");
  if (g_lo < 0 || ng_total < 1 || g_lo + c->cfg.ng > ng_total)
    return fail(SNAP_ERR_BAD_ARG, "group range outside the table");
  SNAP_CUDA(outer_source(c, qi, slgg, mat, flux_all, q2grp, ng_total, g_lo, c->cfg.ng,
                         (cudaStream_t)stream));
  return SNAP_OK;
}

int snap_calc_inner_source(snap_ctx *c, const double *s_xs, const double *q2grp,
                           const double *flux, void *qtot, void *stream) {
  if (!c || !s_xs || !q2grp || !flux || !qtot) return fail(SNAP_ERR_BAD_ARG, "null argument");
  SNAP_CUDA(k_inner_source(s_xs, q2grp, flux, qtot, c->fp32, c->cfg.ng, c->cfg.nmom, c->M, c->C,
                           (cudaStream_t)stream));
  ++c->launches;
  return SNAP_OK;
}

int snap_sweep(snap_ctx *c, const void *qtot, const void *t_xs, void *flux, void *stream) {
  if (!c || !qtot || !t_xs || !flux) return fail(SNAP_ERR_BAD_ARG, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  SNAP_CUDA(cudaMemsetAsync(c->error(), 0, 2 * sizeof(int), st));
  if (c->wide_only) {
    SNAP_CUDA(cudaMemsetAsync(flux, 0, sizeof(double) * c->cfg.ng * c->C * c->M, st));
    SNAP_CUDA(cudaEventRecord(c->sw0, st));
    int rc = wide_sweep(c, (const double *)qtot, (const double *)t_xs, (double *)flux, nullptr,
                        nullptr, nullptr, nullptr, st);
    if (rc) return rc;
    SNAP_CUDA(cudaEventRecord(c->sw1, st));
    rc = read_ctrl(c, st, nullptr);
    if (rc == SNAP_OK) account_sweep(c);
    return rc;
  }
  int rc = timed_sweep(c, qtot, t_xs, flux, c->fp32, nullptr, 0, 0.0, st);
  if (rc) return rc;
  rc = read_ctrl(c, st, nullptr);
  if (rc == SNAP_OK) account_sweep(c);
  return rc;
}

int snap_sweep_td(snap_ctx *c, const double *qtot, const double *t_xs, const double *vdelt,
                  const double *psi_t_in, double *psi_t_out, const double *qim, double *flux,
                  void *stream) {
  if (!c || !qtot || !t_xs || !flux || !vdelt || !psi_t_in || !psi_t_out)
    return fail(SNAP_ERR_BAD_ARG, "null argument");
  if (c->fp32) return fail(SNAP_ERR_UNSUPPORTED, "time-dependent sweeps run in FP64 contexts");
  cudaStream_t st = (cudaStream_t)stream;
  SNAP_CUDA(cudaMemsetAsync(c->error(), 0, 2 * sizeof(int), st));
  SNAP_CUDA(cudaMemsetAsync(flux, 0, sizeof(double) * c->cfg.ng * c->C * c->M, st));
  SNAP_CUDA(cudaEventRecord(c->sw0, st));
  const TdArgs td{vdelt, psi_t_in, psi_t_out, qim};
  int rc = td_tiled(c) ? sweep_launches(c, qtot, t_xs, st, 0, nullptr, flux, 0, 0, &td)
                       : wide_sweep(c, qtot, t_xs, flux, vdelt, psi_t_in, psi_t_out, qim, st);
  if (rc) return rc;
  SNAP_CUDA(cudaEventRecord(c->sw1, st));
  rc = read_ctrl(c, st, nullptr);
  if (rc == SNAP_OK) account_sweep(c);
  return rc;
}

int snap_inner_iteration(snap_ctx *c, const double *s_xs, const double *q2grp, const void *t_xs,
                         double *flux, void *qtot, double epsi, int *converged, void *stream) {
  if (!c || !s_xs || !q2grp || !t_xs || !flux || !qtot || !converged)
    return fail(SNAP_ERR_BAD_ARG, "null argument");
  return inner_iteration_impl(c, s_xs, q2grp, t_xs, flux, qtot, epsi, converged,
                              (cudaStream_t)stream, nullptr);
}

}  // extern "C"

namespace {

// The inner-loop body (snap.cc:487-503).  td != null: the time-dependent
// sweep (vdelt, the time-edge angular flux, the manufactured source) on the
// tiled kernel where td_tiled() allows, else on the general kernel.
int inner_iteration_impl(snap_ctx *c, const double *s_xs, const double *q2grp, const void *t_xs,
                         double *flux, void *qtot, double epsi, int *converged, cudaStream_t st,
                         const TdArgs *td) {
  SNAP_CUDA(cudaMemsetAsync(c->error(), 0, 3 * sizeof(int), st));
  // FP32 contexts: the sweep's rounding leaves a per-inner change of about
  // 1e-6 (max over cells) that no iteration removes, so the inner test
  // cannot usefully be tighter than 32 FP32 units (1.9e-6)
  constexpr double kFp32InnerFloor = 32.0 / 16777216.0;
  const double eps_in = c->fp32 ? std::max(epsi, kFp32InnerFloor) : epsi;
  int rc = SNAP_OK;
  if (td && td_tiled(c)) {
    // the time-dependent form of the tiled kernel, octants added into the flux
    SNAP_CUDA(k_inner_source_save(s_xs, q2grp, flux, qtot, 0, c->d_old0, c->cfg.ng, c->cfg.nmom,
                                  c->M, c->C, st));
    SNAP_CUDA(cudaEventRecord(c->sw0, st));
    rc = sweep_launches(c, qtot, t_xs, st, 0, nullptr, flux, 0, 0, td);
    if (rc) return rc;
    SNAP_CUDA(cudaEventRecord(c->sw1, st));
    SNAP_CUDA(k_test_change(flux, c->d_old0, c->M, (long long)c->cfg.ng * c->C, eps_in,
                            c->violations(), c->maxdf(), st));
    c->launches += 2;
  } else if (c->wide_only || td) {
    SNAP_CUDA(k_inner_source_save(s_xs, q2grp, flux, qtot, 0, c->d_old0, c->cfg.ng, c->cfg.nmom,
                                  c->M, c->C, st));
    SNAP_CUDA(cudaEventRecord(c->sw0, st));
    rc = wide_sweep(c, (const double *)qtot, (const double *)t_xs, flux,
                    td ? td->vdelt : nullptr, td ? td->tf_in : nullptr,
                    td ? td->tf_out : nullptr, td ? td->qim : nullptr, st);
    if (rc) return rc;
    SNAP_CUDA(cudaEventRecord(c->sw1, st));
    SNAP_CUDA(k_test_change(flux, c->d_old0, c->M, (long long)c->cfg.ng * c->C, eps_in,
                            c->violations(), c->maxdf(), st));
    c->launches += 2;
  } else if (c->atomic_octants && !c->tc32) {
    // inner source, old scalar flux saved and flux cleared in one pass; the
    // sweep adds every octant into the flux; the inner test reads it back
    SNAP_CUDA(k_inner_source_save(s_xs, q2grp, flux, qtot, c->fp32, c->d_old0, c->cfg.ng,
                                  c->cfg.nmom, c->M, c->C, st));
    SNAP_CUDA(cudaEventRecord(c->sw0, st));
    rc = sweep_launches(c, qtot, t_xs, st, 0, nullptr, flux);
    if (rc) return rc;
    SNAP_CUDA(cudaEventRecord(c->sw1, st));
    SNAP_CUDA(k_test_change(flux, c->d_old0, c->M, (long long)c->cfg.ng * c->C, eps_in,
                            c->violations(), c->maxdf(), st));
    c->launches += 2;
  } else {
    SNAP_CUDA(k_inner_source(s_xs, q2grp, flux, qtot, c->fp32, c->cfg.ng, c->cfg.nmom, c->M,
                             c->C, st));
    ++c->launches;
    rc = timed_sweep(c, qtot, t_xs, flux, 0, flux, 1, eps_in, st);
    if (rc) return rc;
  }
  int v = 0;
  rc = read_ctrl(c, st, &v);
  if (rc) return rc;
  account_sweep(c);
  *converged = v == 0;
  if (c->fp32) {
    // FP32 contexts also stop an inner loop that has stagnated at the FP32
    // rounding level: the largest change stopped falling (at least halving
    // per inner away from it) while below 2^-15 relative
    float df = 0.0f;
    std::memcpy(&df, &c->h_ctrl[2], sizeof(float));
    if (c->prev_inner_df > 0.0f && df <= 0x1p-15f && df >= 0.5f * c->prev_inner_df)
      *converged = 1;
    c->prev_inner_df = df;
  }
  return SNAP_OK;
}

// Solve arrays kept by the context between solves (allocated on the first).
int ensure_solve_arrays(snap_ctx *c) {
  if (c->d_solve) return SNAP_OK;
  const long long n = (long long)c->cfg.ng * c->C;
  const size_t t64 = sizeof(double) * n, sxs = sizeof(double) * n * c->cfg.nmom,
               q2 = sizeof(double) * n * c->M, fpo = sizeof(double) * n,
               qt = c->wsize * n * c->M, tsw = c->fp32 ? sizeof(float) * n : 0;
  const size_t bytes = t64 + sxs + q2 + fpo + qt + tsw + 5 * 256;
  if (cudaMalloc((void **)&c->d_solve, bytes) != cudaSuccess) {
    cudaGetLastError();
    c->d_solve = nullptr;
    return fail(SNAP_ERR_OOM, "cannot allocate solve arrays");
  }
  c->scratch_bytes += bytes;
  char *b = (char *)c->d_solve;
  auto take = [&](size_t sz) {
    char *at = b;
    b += (sz + 255) & ~(size_t)255;
    return at;
  };
  c->s_txs64 = (double *)take(t64);
  c->s_sxs = (double *)take(sxs);
  c->s_q2 = (double *)take(q2);
  c->s_fpo = (double *)take(fpo);
  c->s_qtot = take(qt);
  c->s_txsw = c->fp32 ? (void *)take(tsw) : (void *)c->s_txs64;
  return SNAP_OK;
}

// The solve loop: the reference's predicated loop (snap.cc:409-541) resolved
// sequentially, for one time step (tc == null: steady state, vdelt = 0) or
// tc->nsteps time steps with the time-edge angular flux passed from one step
// to the next (snap.cc:288-298, 401-407, 497-498).
int solve_impl(snap_ctx *c, const int32_t *mat, const double *qi, const double *sigt,
               const double *slgg, const double *sigt_scale, double *flux, snap_solve_info *info,
               cudaStream_t st, const snap_time_config *tc) {
  if (!c || !mat || !qi || !sigt || !slgg || !flux || !info)
    return fail(SNAP_ERR_BAD_ARG, "null argument");
  if (info->iitm < 1 || info->oitm < 1 || !(info->epsi > 0.0))
    return fail(SNAP_ERR_BAD_ARG, "iitm, oitm and epsi must be positive");
  const int G = c->cfg.ng, M = c->M, nmom = c->cfg.nmom;
  const long long C = c->C, n = (long long)G * C;
  int rc = ensure_solve_arrays(c);
  if (rc) return rc;
  double *t_xs64 = c->s_txs64, *s_xs = c->s_sxs, *q2grp = c->s_q2, *fpo = c->s_fpo;
  void *qtot = c->s_qtot, *t_xs_sw = c->s_txsw;
  // time-dependent state: vdelt per group and the two time-edge halves
  double *tf = nullptr, *tf_own = nullptr, *vdelt = nullptr;
  const size_t tf_half = (size_t)8 * n * c->A;
  if (tc) {
    if ((rc = ensure_wide(c))) return rc;
    if (!c->d_vdelt) {
      if (cudaMalloc((void **)&c->d_vdelt, sizeof(double) * G) != cudaSuccess) {
        cudaGetLastError();
        return fail(SNAP_ERR_OOM, "cannot allocate vdelt");
      }
    }
    vdelt = c->d_vdelt;
    if (tc->vdelt) {
      SNAP_CUDA(cudaMemcpyAsync(vdelt, tc->vdelt, sizeof(double) * G, cudaMemcpyDeviceToDevice, st));
    } else {
      // Snap::initialize_velocity (snap.cc:717-739): v_g = G - g, vdelt = 2/(dt v)
      c->h_vdelt.assign(G, 0.0);
      for (int g = 0; g < G; ++g) c->h_vdelt[g] = 2.0 / (tc->dt * double(G - g));
      SNAP_CUDA(cudaMemcpyAsync(vdelt, c->h_vdelt.data(), sizeof(double) * G,
                                cudaMemcpyHostToDevice, st));
    }
    tf = tc->psi_t;
    if (!tf) {
      if (cudaMalloc((void **)&tf_own, sizeof(double) * 2 * tf_half) != cudaSuccess) {
        cudaGetLastError();
        return fail(SNAP_ERR_OOM, "cannot allocate the time-edge angular flux");
      }
      tf = tf_own;
    }
    if (!tc->psi_t_initialised) SNAP_CUDA(cudaMemsetAsync(tf, 0, sizeof(double) * 2 * tf_half, st));
  }
#define STEP(x)                 \
  do {                          \
    cudaError_t e_ = (x);       \
    if (e_ != cudaSuccess) {    \
      rc = cuda_fail(e_, #x);   \
      goto done;                \
    }                           \
  } while (0)
  {
    info->inner_total = info->outer_total = info->converged = info->outers_lowp = 0;
    info->sweep_ms = info->total_ms = 0.0;
    info->records_len = 0;
    const double sweep_ms0 = c->sweep_ms;
    float ms = 0.0f;
    int rec = 0;   // entries of inners_per_outer
    auto now_us = []() {
      return std::chrono::duration<double, std::micro>(
                 std::chrono::steady_clock::now().time_since_epoch())
          .count();
    };
    auto log = [&](int kind, int step, int outer, int inner, int conv, double us) {
      if (info->records && info->records_len < info->records_cap)
        info->records[info->records_len++] = snap_iter_record{kind, step, outer, inner, conv, us};
    };
    STEP(cudaMemsetAsync(c->error(), 0, 2 * sizeof(int), st));
    STEP(cudaEventRecord(c->ev0, st));
    // per time step expansion (snap.cc:419-450); the tables do not change
    // between time steps, so the expansion runs once
    STEP(k_expand_xs(sigt, mat, t_xs64, G, c->cfg.nmat, C, st));
    if (sigt_scale) STEP(k_scale_xs(t_xs64, sigt_scale, G, C, st));
    STEP(k_expand_scat(slgg, mat, s_xs, G, c->cfg.nmat, nmom, C, st));
    c->launches += sigt_scale ? 3 : 2;
    if (c->fp32) {
      STEP(k_to_f32(t_xs64, (float *)t_xs_sw, n, st));
      ++c->launches;
    }
    STEP(cudaMemsetAsync(flux, 0, sizeof(double) * n * M, st));   // snap.cc:313-316
    // precision form: split-BF16 tcgen05 outer source while far from
    // convergence, where its plan batches 4 moments (else the FP64
    // tensor-core source is the faster one)
    const bool lowp = c->fp32 && !(getenv("SNAP_B200_FP32_EXACT_OUTER") &&
                                   atoi(getenv("SNAP_B200_FP32_EXACT_OUTER")) != 0) &&
                      outer_tc_preferred(G, c->cfg.nmat, nmom);
    // outer change above which the low-precision source is used: ten times
    // the outer convergence tolerance, so the outer iterations that can
    // converge run on the FP64 source
    const double kFar = 1000.0 * info->epsi;
    const int nsteps = tc ? tc->nsteps : 1;
    bool even = false;
    for (int cy = 0; cy < nsteps; ++cy) {
      TdArgs td{};
      if (tc) {
        even = !even;   // snap.cc:411: in = even ? even half : odd half
        td.vdelt = vdelt;
        td.tf_in = even ? tf : tf + tf_half;
        td.tf_out = even ? tf + tf_half : tf;
        td.qim = tc->qim;
        if (tc->qim && tc->qim_time_scaled) {
          // MMSScale (snap.cc:451-466): source at the middle of the step
          const double f = cy == 0 ? tc->dt * 0.5 : double(2 * cy + 1) / double(2 * cy - 1);
          STEP(k_scale(tc->qim, f, tf_half, st));
          ++c->launches;
        }
      }
      bool far = true;
      info->converged = 0;
      for (int o = 0; o < info->oitm; ++o) {
        const double t_outer = now_us();
        const bool use_tc = lowp && far && o > 0;   // outer 0 has zero flux: q2 = qi exactly
        c->prev_inner_df = 0.0f;                     // no stagnation test on an outer's first inner
        if (use_tc) {
          rc = snap_calc_outer_source_tc(c, qi, slgg, mat, flux, q2grp, st);
          if (rc) goto done;
          ++info->outers_lowp;
        } else {
          STEP(outer_source(c, qi, slgg, mat, flux, q2grp, G, 0, G, st));
        }
        STEP(k_moment0(flux, fpo, M, n, st));                        // save_fluxes -> flux0po
        ++c->launches;
        bool inner_conv = false;
        int inners = 0;
        double t_inner = now_us();
        for (int i = 0; i < info->iitm; ++i) {
          int conv = 0;
          rc = inner_iteration_impl(c, s_xs, q2grp, t_xs_sw, flux, qtot, info->epsi, &conv, st,
                                    tc ? &td : nullptr);
          if (rc) goto done;
          const double t_now = now_us();
          log(0, cy, o, i, conv, t_now - t_inner);
          t_inner = t_now;
          ++inners;
          ++info->inner_total;
          inner_conv = conv != 0;
          if (inner_conv) break;
        }
        if (rec < 1024) info->inners_per_outer[rec++] = inners;
        ++info->outer_total;
        if (o == 0) continue;                                        // snap.cc:521-522
        if (lowp && far) {
          // FP64 outer residual: every scalar flux within kFar of the last outer?
          STEP(cudaMemsetAsync(c->violations(), 0, sizeof(int), st));
          STEP(k_test_change(flux, fpo, M, n, kFar, c->violations(), c->maxdf(), st));
          ++c->launches;
          int v = 0;
          rc = read_ctrl(c, st, &v);
          if (rc) goto done;
          if (v == 0) far = false;
        }
        // convergence only on an outer iteration with the FP64 source
        if (inner_conv && !use_tc) {
          STEP(cudaMemsetAsync(c->violations(), 0, sizeof(int), st));
          STEP(k_test_change(flux, fpo, M, n, 100.0 * info->epsi, c->violations(), c->maxdf(), st));
          ++c->launches;
          int v = 0;
          rc = read_ctrl(c, st, &v);
          if (rc) goto done;
          log(1, cy, o, 0, v == 0, now_us() - t_outer);
          if (v == 0) {
            info->converged = 1;
            break;
          }
        } else {
          log(1, cy, o, 0, 0, now_us() - t_outer);   // the outer test fails without inner convergence
        }
      }
    }
    STEP(cudaEventRecord(c->ev1, st));
    STEP(cudaEventSynchronize(c->ev1));
    STEP(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    info->total_ms = ms;
    info->sweep_ms = c->sweep_ms - sweep_ms0;
  }
done:
  if (tf_own) {
    cudaStreamSynchronize(st);
    cudaFree(tf_own);
  }
#undef STEP
  return rc;
}

}  // namespace

extern "C" {

int snap_mms_init(snap_ctx *c, const int32_t *mat, const double *sigt, const double *slgg,
                  double lx, double ly, double lz, const int *chunk_cells, int timedep,
                  double tf, double dt, double *ref_flux, double *qim, double *qi,
                  void *stream) {
  if (!c || !mat || !sigt || !slgg || !ref_flux || !qim || (timedep && !qi))
    return fail(SNAP_ERR_BAD_ARG, "null argument");
  if (c->cfg.nmom != 1)
    return fail(SNAP_ERR_UNSUPPORTED, "the manufactured solution has no flux moments (nmom = 1)");
  if (!(lx > 0.0 && ly > 0.0 && lz > 0.0) || (timedep && !(dt > 0.0)))
    return fail(SNAP_ERR_BAD_ARG, "lengths and dt must be positive");
  cudaStream_t st = (cudaStream_t)stream;
  MmsGeometry geo{};
  geo.nx = c->cfg.nx;
  geo.ny = c->cfg.ny;
  geo.nz = c->cfg.nz;
  geo.A = c->A;
  geo.G = c->cfg.ng;
  geo.nmat = c->cfg.nmat;
  geo.lx = lx;
  geo.ly = ly;
  geo.lz = lz;
  geo.timedep = timedep;
  geo.tf = tf;
  geo.dt = dt;
  geo.quad[0] = c->mu.data();
  geo.quad[1] = c->eta.data();
  geo.quad[2] = c->xi.data();
  const int dims[3] = {geo.nx, geo.ny, geo.nz};
  for (int d = 0; d < 3; ++d) {
    geo.chunk[d] = chunk_cells ? chunk_cells[d] : dims[d];
    if (geo.chunk[d] < 1 || dims[d] % geo.chunk[d])
      return fail(SNAP_ERR_BAD_ARG, "chunk_cells must divide the mesh");
  }
  double *scratch = nullptr;
  const size_t words = mms_scratch_words(geo.nx, geo.ny, geo.nz, geo.A);
  SNAP_CUDA(cudaMalloc((void **)&scratch, sizeof(double) * words));
  cudaError_t e = mms_init(geo, mat, sigt, slgg, ref_flux, qim, qi, scratch, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(scratch);
  if (e != cudaSuccess) return cuda_fail(e, "manufactured solution");
  c->launches += timedep ? 3 : 2;
  return SNAP_OK;
}

int snap_mms_compare(snap_ctx *c, const double *flux, const double *ref_flux, double *out,
                     void *stream) {
  if (!c || !flux || !ref_flux || !out) return fail(SNAP_ERR_BAD_ARG, "null argument");
  void *scratch = nullptr;
  SNAP_CUDA(cudaMalloc(&scratch, 3 * sizeof(double)));
  cudaError_t e = mms_compare(flux, c->M, ref_flux, (long long)c->cfg.ng * c->C, scratch, out,
                              (cudaStream_t)stream);
  cudaFree(scratch);
  if (e != cudaSuccess) return cuda_fail(e, "manufactured-solution comparison");
  ++c->launches;
  return SNAP_OK;
}

int snap_get_timing(snap_ctx *c, snap_timing *out, int reset) {
  if (!c || !out) return fail(SNAP_ERR_BAD_ARG, "null argument");
  out->sweep_ms = c->sweep_ms;
  out->sweep_calls = c->sweep_calls;
  out->kernel_launches = c->launches;
  if (reset) {
    c->sweep_ms = 0.0;
    c->sweep_calls = 0;
    c->launches = 0;
  }
  return SNAP_OK;
}

int snap_test_convergence(snap_ctx *c, int kind, const double *flux, const double *prev,
                          double epsi, int *converged, void *stream) {
  if (!c || !flux || !prev || !converged || (kind != 0 && kind != 1))
    return fail(SNAP_ERR_BAD_ARG, "bad argument");
  cudaStream_t st = (cudaStream_t)stream;
  SNAP_CUDA(cudaMemsetAsync(c->error(), 0, 2 * sizeof(int), st));
  SNAP_CUDA(k_count_violations(flux, prev, c->M, (long long)c->cfg.ng * c->C, epsi,
                               c->violations(), st));
  ++c->launches;
  int v = 0;
  int rc = read_ctrl(c, st, &v);
  if (rc) return rc;
  *converged = v == 0;
  return SNAP_OK;
}

int snap_transport_solve(snap_ctx *c, const int32_t *mat, const double *qi, const double *sigt,
                         const double *slgg, const double *sigt_scale, double *flux,
                         snap_solve_info *info, void *stream) {
  return solve_impl(c, mat, qi, sigt, slgg, sigt_scale, flux, info, (cudaStream_t)stream, nullptr);
}

int snap_transport_solve_td(snap_ctx *c, const int32_t *mat, const double *qi, const double *sigt,
                            const double *slgg, const double *sigt_scale,
                            const snap_time_config *tc, double *flux, snap_solve_info *info,
                            void *stream) {
  if (!c || !tc) return fail(SNAP_ERR_BAD_ARG, "null argument");
  if (tc->nsteps < 1 || !(tc->dt > 0.0)) return fail(SNAP_ERR_BAD_ARG, "nsteps and dt must be positive");
  if (c->fp32) return fail(SNAP_ERR_UNSUPPORTED, "time-dependent solves run in FP64 contexts");
  return solve_impl(c, mat, qi, sigt, slgg, sigt_scale, flux, info, (cudaStream_t)stream, tc);
}

}  // extern "C"

namespace {

// Work items of a batch of gn groups (same order rules as build_items).
int ensure_batch_tables(snap_ctx *c, int gn) {
  if ((int)c->batch_tables.size() <= gn) c->batch_tables.resize(gn + 1);
  auto &b = c->batch_tables[gn];
  if (b.table) return SNAP_OK;
  // as many octants per launch as the tile-face scratch (sized for the
  // context's P octants of every group) holds for gn groups
  int P = 8;
  while (P > c->P && (size_t)P * gn > (size_t)c->P * c->cfg.ng) P /= 2;
  b.P = P;
  std::vector<int> table, index;
  build_items(P, gn, c->tiles_x, c->tiles_y, table, index);
  int rc;
  if ((rc = upload((void **)&b.table, table)) || (rc = upload((void **)&b.index, index))) return rc;
  b.n_items = (int)table.size();
  return SNAP_OK;
}

// Forward state for the adjoint of `groups` groups at a time.
int ensure_state(snap_ctx *c, int groups = 0) {
  if (groups <= 0) groups = c->cfg.ng;
  if (c->d_pc_store && c->state_groups >= groups) return SNAP_OK;
  if (c->d_pc_store) {
    cudaFree(c->d_pc_store);
    cudaFree(c->d_flag_store);
    c->scratch_bytes -= (size_t)8 * c->state_groups * c->C * c->AP * (c->wsize + 1);
    c->d_pc_store = nullptr;
    c->d_flag_store = nullptr;
    c->state_groups = 0;
  }
  const size_t n = (size_t)8 * groups * c->C * c->AP;
  if (cudaMalloc(&c->d_pc_store, n * c->wsize) != cudaSuccess ||
      cudaMalloc((void **)&c->d_flag_store, n) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(c->d_pc_store);
    c->d_pc_store = nullptr;
    return fail(SNAP_ERR_OOM, "cannot allocate the forward-state store for the adjoint");
  }
  c->scratch_bytes += n * (c->wsize + 1);
  c->state_groups = groups;
  return SNAP_OK;
}

int ensure_sbar(snap_ctx *c, int groups, int P) {
  const size_t need = (size_t)P * groups * c->C * c->wsize;
  if (c->d_sbar_slots && c->sbar_alloc >= need) return SNAP_OK;
  cudaFree(c->d_sbar_slots);
  c->scratch_bytes -= c->sbar_alloc;
  c->sbar_alloc = 0;
  if (cudaMalloc(&c->d_sbar_slots, need) != cudaSuccess) {
    cudaGetLastError();
    c->d_sbar_slots = nullptr;
    return fail(SNAP_ERR_OOM, "cannot allocate the sigma_t adjoint slots");
  }
  c->sbar_alloc = need;
  c->scratch_bytes += need;
  return SNAP_OK;
}

// qtot_bar: double [G][C][M], or float when qbar_fp32 (FP32 contexts' lean
// adjoint solve)
int adjoint_sweep_impl(snap_ctx *c, const void *phi_bar, const void *t_xs, void *qtot_bar,
                       double *sigt_bar, cudaStream_t st, int g0 = 0, int gn = 0,
                       int qbar_fp32 = 0) {
  const int groups = gn > 0 ? gn : c->cfg.ng;
  if ((sigt_bar || c->cfg.fixup) && (!c->state_recorded || c->state_groups < groups))
    return fail(SNAP_ERR_BAD_ARG, "record the forward state (snap_record_forward) first");
  const int P = (gn > 0 && gn < c->cfg.ng) ? c->batch_tables[gn].P : c->P;
  int rc;
  if (sigt_bar && (rc = ensure_sbar(c, groups, P))) return rc;
  SNAP_CUDA(cudaEventRecord(c->sw0, st));
  rc = sweep_launches(c, phi_bar, t_xs, st, 2, sigt_bar ? c->d_sbar_slots : nullptr, nullptr, g0,
                      gn);
  if (rc) return rc;
  SNAP_CUDA(cudaEventRecord(c->sw1, st));
  void *qb = (char *)qtot_bar + (size_t)g0 * c->C * c->M * (qbar_fp32 ? sizeof(float) : sizeof(double));
  SNAP_CUDA(k_reduce_slots(c->d_slots, P, c->fp32, qb, qbar_fp32, nullptr, groups, c->M, c->C,
                           0, 0.0, nullptr, st));
  ++c->launches;
  if (sigt_bar) {
    SNAP_CUDA(k_reduce_slots(c->d_sbar_slots, P, c->fp32, sigt_bar + (size_t)g0 * c->C, 0,
                             nullptr, groups, 1, c->C, 0, 0.0, nullptr, st));
    ++c->launches;
  }
  return SNAP_OK;
}

// One application of M^T L^-T D^T to every group (qtot_bar from phi_bar),
// with the forward state recorded from `qtot` batch by batch when the
// context holds the state of fewer groups than it sweeps.
int adjoint_apply(snap_ctx *c, const void *phi_bar, const void *t_xs, const void *qtot,
                  void *qtot_bar, double *sigt_bar, cudaStream_t st, int batch, int qbar_fp32) {
  const int G = c->cfg.ng;
  if (batch >= G)
    return adjoint_sweep_impl(c, phi_bar, t_xs, qtot_bar, sigt_bar, st, 0, 0, qbar_fp32);
  for (int g0 = 0; g0 < G; g0 += batch) {
    const int gn = std::min(batch, G - g0);
    int rc = sweep_launches(c, qtot, t_xs, st, 1, nullptr, nullptr, g0, gn);
    if (rc) return rc;
    rc = adjoint_sweep_impl(c, phi_bar, t_xs, qtot_bar, sigt_bar, st, g0, gn, qbar_fp32);
    if (rc) return rc;
  }
  return SNAP_OK;
}

}  // namespace

extern "C" {

int snap_record_forward(snap_ctx *c, const void *qtot, const void *t_xs, void *flux,
                        void *stream) {
  if (!c || !qtot || !t_xs || !flux) return fail(SNAP_ERR_BAD_ARG, "null argument");
  if (c->wide_only) return fail(SNAP_ERR_UNSUPPORTED, "the adjoint needs the tiled sweep's shapes");
  cudaStream_t st = (cudaStream_t)stream;
  int rc = ensure_state(c);
  if (rc) return rc;
  SNAP_CUDA(cudaMemsetAsync(c->error(), 0, 2 * sizeof(int), st));
  rc = sweep_launches(c, qtot, t_xs, st, 1);
  if (rc) return rc;
  SNAP_CUDA(k_reduce_slots(c->d_slots, c->P, c->fp32, flux, c->fp32, nullptr, c->cfg.ng, c->M, c->C,
                           0, 0.0, nullptr, st));
  ++c->launches;
  rc = read_ctrl(c, st, nullptr);
  if (rc == SNAP_OK) c->state_recorded = true;
  return rc;
}

int snap_adjoint_sweep(snap_ctx *c, const void *phi_bar, const void *t_xs, double *qtot_bar,
                       double *sigt_bar, void *stream) {
  if (!c || !phi_bar || !t_xs || !qtot_bar) return fail(SNAP_ERR_BAD_ARG, "null argument");
  if (c->wide_only) return fail(SNAP_ERR_UNSUPPORTED, "the adjoint needs the tiled sweep's shapes");
  cudaStream_t st = (cudaStream_t)stream;
  SNAP_CUDA(cudaMemsetAsync(c->error(), 0, 2 * sizeof(int), st));
  int rc = adjoint_sweep_impl(c, phi_bar, t_xs, qtot_bar, sigt_bar, st);
  if (rc) return rc;
  rc = read_ctrl(c, st, nullptr);
  if (rc == SNAP_OK) account_sweep(c);
  return rc;
}

int snap_adjoint_solve(snap_ctx *c, const int32_t *mat, const double *qi, const double *t_xs,
                       const double *slgg, const double *flux, const double *response,
                       double *grad_sigt, double *grad_qi, double *grad_sxs, snap_solve_info *info,
                       void *stream) {
  if (!c || !mat || !qi || !t_xs || !slgg || !flux || !response || !grad_sigt || !grad_qi || !info)
    return fail(SNAP_ERR_BAD_ARG, "null argument");
  if (info->iitm < 1 || info->oitm < 1 || !(info->epsi > 0.0))
    return fail(SNAP_ERR_BAD_ARG, "iitm, oitm and epsi must be positive");
  if (c->wide_only) return fail(SNAP_ERR_UNSUPPORTED, "the adjoint needs the tiled sweep's shapes");
  cudaStream_t st = (cudaStream_t)stream;
  const int G = c->cfg.ng, M = c->M, nmom = c->cfg.nmom;
  const long long C = c->C, n = (long long)G * C;
  const int f32 = c->fp32;
  // Work arrays: the context's solve arrays (total source, in-group
  // scattering, sweep-precision t_xs), and the adjoint vectors phi_bar and
  // qtot_bar in the sweep precision.  In FP32 contexts both fit in the space
  // of the FP64 outer-source array, which is free once the total source is
  // formed; FP64 contexts add one array for qtot_bar.
  int rc = ensure_solve_arrays(c);
  if (rc) return rc;
  double *qbar64 = nullptr;
  unsigned long long *d_norm = nullptr;
  if ((!f32 && cudaMalloc((void **)&qbar64, sizeof(double) * n * M) != cudaSuccess) ||
      cudaMalloc((void **)&d_norm, 2 * sizeof(unsigned long long)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(qbar64);
    return fail(SNAP_ERR_OOM, "cannot allocate adjoint solve arrays");
  }
  auto cleanup = [&]() {
    cudaFree(qbar64);
    cudaFree(d_norm);
  };
  void *pb = c->s_q2;                                        // phi_bar [G][C][M]
  void *qbar = f32 ? (void *)((float *)c->s_q2 + n * M) : (void *)qbar64;
  const void *t_sw = f32 ? c->s_txsw : (const void *)t_xs;
  void *qtot = c->s_qtot;
  // forward state of `batch` groups at a time: all groups when it fits in
  // 70 % of the free memory (recorded once), else batches recorded again
  // from the converged flux moments for every adjoint iteration
  int batch = G;
  {
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const size_t per_group = (size_t)8 * C * c->AP * (c->wsize + 1) +     // recorded state
                             (size_t)c->P * C * (M + 1) * c->wsize;         // octant slots
    const size_t held = c->d_pc_store ? (size_t)c->state_groups * per_group : 0;
    const size_t avail = (size_t)(0.7 * (double)(free_b + held));
    batch = (int)std::max<size_t>(1, std::min<size_t>((size_t)G, avail / per_group));
    if (const char *e = getenv("SNAP_B200_ADJOINT_GROUPS")) batch = std::max(1, std::min(G, atoi(e)));
  }
  rc = ensure_state(c, batch);
  if (!rc && batch < G) {
    rc = ensure_batch_tables(c, batch);
    if (!rc && G % batch) rc = ensure_batch_tables(c, G % batch);
  }
  if (rc) {
    cleanup();
    return rc;
  }
#define ASTEP(x)                \
  do {                          \
    cudaError_t e_ = (x);       \
    if (e_ != cudaSuccess) {    \
      rc = cuda_fail(e_, #x);   \
      goto adone;               \
    }                           \
  } while (0)
  {
    info->inner_total = info->outer_total = info->converged = info->outers_lowp = 0;
    const double sweep_ms0 = c->sweep_ms;
    float ms = 0.0f;
    const int maxit = info->iitm * info->oitm;
    ASTEP(cudaMemsetAsync(c->error(), 0, 2 * sizeof(int), st));
    ASTEP(cudaEventRecord(c->ev0, st));
    // the forward operator at the converged flux: total source
    ASTEP(k_expand_scat(slgg, mat, c->s_sxs, G, c->cfg.nmat, nmom, C, st));
    if (f32) ASTEP(k_to_f32(t_xs, (float *)c->s_txsw, n, st));
    ASTEP(outer_source(c, qi, slgg, mat, flux, c->s_q2, G, 0, G, st));
    ASTEP(k_inner_source(c->s_sxs, c->s_q2, flux, qtot, f32, G, nmom, M, C, st));
    c->launches += f32 ? 3 : 2;
    // forward sweep recording the cell-average fluxes and fixup flags (with
    // batches: recorded inside every adjoint application)
    if (batch >= G) {
      rc = sweep_launches(c, qtot, t_sw, st, 1);
      if (rc) goto adone;
    }
    c->state_recorded = true;
    // adjoint source iteration: phi_bar = r + S^T M^T L^-T D^T phi_bar,
    // converged when max|change| <= epsi * max|phi_bar| (the adjoint spans
    // many decades, so the forward test's per-cell form does not apply);
    // phi_bar starts at r (qtot_bar = 0)
    ASTEP(cudaMemsetAsync(qbar, 0, (f32 ? sizeof(float) : sizeof(double)) * n * M, st));
    ASTEP(cudaMemsetAsync(pb, 0, (f32 ? sizeof(float) : sizeof(double)) * n * M, st));
    ASTEP(cudaMemsetAsync(d_norm, 0, 2 * sizeof(unsigned long long), st));
    ASTEP(k_adjoint_update(response, slgg, mat, qbar, pb, f32, d_norm, G, c->cfg.nmat, nmom, M, C,
                           st));
    ++c->launches;
    for (int it = 0; it < maxit; ++it) {
      rc = adjoint_apply(c, pb, t_sw, qtot, qbar, nullptr, st, batch, f32);
      if (rc) goto adone;
      ASTEP(cudaMemsetAsync(d_norm, 0, 2 * sizeof(unsigned long long), st));
      ASTEP(k_adjoint_update(response, slgg, mat, qbar, pb, f32, d_norm, G, c->cfg.nmat, nmom, M,
                             C, st));
      ++c->launches;
      unsigned long long hn[2] = {0, 0};
      ASTEP(cudaMemcpyAsync(hn, d_norm, sizeof(hn), cudaMemcpyDeviceToHost, st));
      rc = read_ctrl(c, st, nullptr);
      if (rc) goto adone;
      account_sweep(c);
      ++info->inner_total;
      double dmax, amax;
      memcpy(&dmax, &hn[0], sizeof(double));
      memcpy(&amax, &hn[1], sizeof(double));
      if (dmax <= info->epsi * amax) {
        info->converged = 1;
        break;
      }
    }
    info->outer_total = 1;
    // gradients from the converged adjoint
    rc = adjoint_apply(c, pb, t_sw, qtot, qbar, grad_sigt, st, batch, f32);
    if (rc) goto adone;
    ASTEP(k_moment0_any(qbar, f32, grad_qi, M, n, st));
    if (grad_sxs) ASTEP(k_grad_sxs_any(qbar, f32, flux, grad_sxs, G, nmom, M, C, st));
    c->launches += grad_sxs ? 2 : 1;
    rc = read_ctrl(c, st, nullptr);
    if (rc) goto adone;
    account_sweep(c);
    ASTEP(cudaEventRecord(c->ev1, st));
    ASTEP(cudaEventSynchronize(c->ev1));
    ASTEP(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    info->total_ms = ms;
    info->sweep_ms = c->sweep_ms - sweep_ms0;
  }
adone:
  cleanup();
#undef ASTEP
  return rc;
}

}  // extern "C"
