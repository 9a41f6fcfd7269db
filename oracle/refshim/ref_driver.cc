/*
 * Sequential driver for the reference's own CPU task bodies (TEST
 * INFRASTRUCTURE ONLY).  Built with the unmodified reference sources
 * sweep.cc, outer.cc, inner.cc, expxs.cc, init.cc (compiled where they lie,
 * see oracle/Makefile) and the shim legion.h into oracle/_ref/libsnapref.so.
 *
 * What it restates (everything else is the reference's code):
 *  - Snap's static configuration (snap.cc:1032-1168) and the 3-D quadrature of
 *    compute_derived_globals (snap.cc:1171-1342, including its ec stride);
 *  - the region/field-space setup of Snap::setup (snap.cc:42-222) for a single
 *    spatial chunk;
 *  - the predicated solve loop of Snap::transport_solve (snap.cc:225-568)
 *    resolved sequentially, with the reference's own task constructors
 *    building every launcher and this file executing them;
 *  - the relaxed-coherence reductions (snap.cc:1832-1926) as CAS loops.
 * The cross sections come from the caller (the steady-state benchmark rule
 * replaces Snap::initialize_scattering).
 */
#include "snap.h"
#include "sweep.h"
#include "outer.h"
#include "inner.h"
#include "expxs.h"
#include "init.h"
#include "mms.h"

#include <atomic>
#include <chrono>
#include <cstdlib>
#include <mutex>
#include <thread>

using Legion::FieldLayout;

Legion::Logger log_snap("snap");
const Legion::Predicate Legion::Predicate::TRUE_PRED = Legion::Predicate();

/* ---- Snap statics (declared in snap.h, defined by snap.cc upstream) ---- */
int Snap::num_dims = 3;
int Snap::nx_chunks = 1, Snap::ny_chunks = 1, Snap::nz_chunks = 1;
int Snap::nx = 4, Snap::ny = 4, Snap::nz = 4;
double Snap::lx = 1.0, Snap::ly = 1.0, Snap::lz = 1.0;
int Snap::num_moments = 1, Snap::num_angles = 1, Snap::num_groups = 1;
double Snap::convergence_eps = 1e-4;
int Snap::max_inner_iters = 5, Snap::max_outer_iters = 100;
bool Snap::time_dependent = false;
double Snap::total_sim_time = 0.0;
int Snap::num_steps = 1;
Snap::MaterialLayout Snap::material_layout = Snap::CENTER_LAYOUT;
Snap::SourceLayout Snap::source_layout = Snap::CENTER_SOURCE;
bool Snap::dump_scatter = false, Snap::dump_iteration = false;
int Snap::dump_flux = 0;
bool Snap::flux_fixup = true, Snap::dump_solution = false;
int Snap::dump_kplane = 0, Snap::dump_population = 0;
bool Snap::minikba_sweep = true, Snap::single_angle_copy = false;
int Snap::num_corners = 8;
int Snap::nx_per_chunk = 4, Snap::ny_per_chunk = 4, Snap::nz_per_chunk = 4;
double Snap::dt = 0.0;
int Snap::cmom = 1, Snap::num_octants = 8;
double Snap::hi = 0.0, Snap::hj = 0.0, Snap::hk = 0.0;
double *Snap::mu = nullptr, *Snap::w = nullptr, *Snap::wmu = nullptr;
double *Snap::eta = nullptr, *Snap::weta = nullptr;
double *Snap::xi = nullptr, *Snap::wxi = nullptr;
double *Snap::ec = nullptr, *Snap::dinv = nullptr;
int Snap::lma[4] = {0, 0, 0, 0};
const char *Snap::task_names[LAST_TASK_ID] = {SNAP_TASK_NAMES};
LayoutConstraintID Snap::get_soa_layout(void) { return 1; }
LayoutConstraintID Snap::get_reduction_layout(void) { return 2; }

/* ---- reductions under relaxed coherence: lock-free add on a double ---- */
static inline void cas_add(double &target, double v) {
  std::atomic_ref<double> ref(target);
  double old = ref.load(std::memory_order_relaxed);
  while (!ref.compare_exchange_weak(old, old + v, std::memory_order_relaxed)) {
  }
}
const double SumReduction::identity = 0.0;
template <> void SumReduction::apply<true>(LHS &lhs, RHS rhs) { lhs += rhs; }
template <> void SumReduction::apply<false>(LHS &lhs, RHS rhs) { cas_add(lhs, rhs); }
template <> void SumReduction::fold<true>(RHS &a, RHS b) { a += b; }
template <> void SumReduction::fold<false>(RHS &a, RHS b) { cas_add(a, b); }
const MomentTriple TripleReduction::identity = MomentTriple();
template <> void TripleReduction::apply<true>(LHS &lhs, RHS rhs) {
  for (int i = 0; i < 3; i++) lhs[i] += rhs[i];
}
template <> void TripleReduction::apply<false>(LHS &lhs, RHS rhs) {
  for (int i = 0; i < 3; i++) cas_add(lhs[i], rhs[i]);
}
template <> void TripleReduction::fold<true>(RHS &a, RHS b) {
  for (int i = 0; i < 3; i++) a[i] += b[i];
}
template <> void TripleReduction::fold<false>(RHS &a, RHS b) {
  for (int i = 0; i < 3; i++) cas_add(a[i], b[i]);
}

/* ---- storage behind the shim's logical regions ---- */
namespace {
struct Store {
  Legion::IndexSpace is;
  std::vector<FieldID> fields;
  size_t field_size = 0;
  size_t volume = 0;
  char *mem = nullptr;  /* nullptr: region never touched (time flux, qim) */
  bool phantom = false;
  std::map<FieldID, size_t> index;
  char *field_base(FieldID f) const { return mem + index.at(f) * volume * field_size; }
};
std::vector<Store> g_stores;
bool g_phantom_next = false;

int register_store(const Legion::IndexSpace &is, const FieldSpace &fs) {
  Store s;
  s.is = is;
  s.fields = fs.fields;
  s.field_size = fs.field_size;
  s.volume = 1;
  for (int i = 0; i < is.dim; i++) s.volume *= (size_t)(is.hi[i] - is.lo[i] + 1);
  for (size_t i = 0; i < s.fields.size(); i++) s.index[s.fields[i]] = i;
  s.phantom = g_phantom_next;
  if (!s.phantom) {
    const size_t bytes = s.volume * s.field_size * s.fields.size();
    void *p = nullptr;
    if (posix_memalign(&p, 64, bytes ? bytes : 64)) abort();
    memset(p, 0, bytes);
    s.mem = (char *)p;
  }
  g_stores.push_back(s);
  return (int)g_stores.size() - 1;
}
}  // namespace

template <int DIM>
SnapArray<DIM>::SnapArray(IndexSpace<DIM> is, IndexPartition<DIM>, FieldSpace fs, Context c,
                          Runtime *rt, const char *)
    : ctx(c), runtime(rt) {
  const int h = register_store(is, fs);
  lr.handle = h;
  lr.is = is;
  lp.handle = h;
  lp.is = is;
  all_fields.insert(fs.fields.begin(), fs.fields.end());
  fill_buffer = nullptr;
  field_size = fs.field_size;
}
template <int DIM> SnapArray<DIM>::~SnapArray(void) {
  Store &s = g_stores[lr.handle];
  free(s.mem);
  s.mem = nullptr;
}
template class SnapArray<1>;
template class SnapArray<2>;
template class SnapArray<3>;

namespace {

Store &store_of(const SnapArray<3> &a) { return g_stores[a.get_region().handle]; }
Store &store_of(const SnapArray<2> &a) { return g_stores[a.get_region().handle]; }
Store &store_of(const SnapArray<1> &a) { return g_stores[a.get_region().handle]; }

PhysicalRegion map_store(const Store &s) {
  PhysicalRegion pr;
  pr.dim = s.is.dim;
  for (FieldID f : s.fields) {
    FieldLayout l;
    l.field_size = s.field_size;
    long long stride = (long long)s.field_size, off = 0;
    for (int i = 0; i < s.is.dim; i++) {
      l.strides[i] = stride;
      off += s.is.lo[i] * stride;
      stride *= (s.is.hi[i] - s.is.lo[i] + 1);
    }
    /* phantom stores are never dereferenced; give them a harmless base */
    char *base = s.phantom ? (char *)(uintptr_t)0x100000 : s.field_base(f);
    l.zero = base - off;
    pr.fields[f] = l;
  }
  return pr;
}

Runtime g_runtime;

/* Executes one point of an index launch built by a reference task ctor.
 * chunk: the point's spatial chunk (the sub-box its 3-D region requirements
 * project to, snap.cc:56-62); NULL for the whole space.  2-D (face) and 1-D
 * requirements see their whole space, which the task indexes with global
 * points (sweep.cc:217-239). */
template <typename RET>
RET execute(const IndexTaskLauncher &launcher,
            RET (*impl)(const Task *, const std::vector<PhysicalRegion> &, Context, Runtime *),
            const Legion::IndexSpace *chunk = nullptr) {
  Task task;
  task.args = launcher.global_arg.args;
  task.arglen = launcher.global_arg.arglen;
  task.futures = launcher.futures;
  std::vector<PhysicalRegion> regions;
  for (const RegionRequirement &rr : launcher.region_requirements) {
    RegionRequirement r = rr;
    const Store &s = g_stores[rr.region.handle];
    r.region.is = (chunk && s.is.dim == 3) ? *chunk : s.is;
    task.regions.push_back(r);
    regions.push_back(map_store(s));
  }
  return impl(&task, regions, nullptr, &g_runtime);
}

void fill_zero(const Store &s) {
  if (s.mem) memset(s.mem, 0, s.volume * s.field_size * s.fields.size());
}
void copy_store(const Store &src, const Store &dst) {
  memcpy(dst.mem, src.mem, src.volume * src.field_size * src.fields.size());
}

/* snap.cc:1171-1342, 3-D branch, including the reference's ec indexing
 * (ec[oct*num_angles*num_moments + moment*num_angles + idx]). */
void derive_globals() {
  Snap::cmom = Snap::num_moments * Snap::num_moments;
  Snap::num_octants = 8;
  Snap::hi = 2.0 / (Snap::lx / double(Snap::nx));
  Snap::hj = 2.0 / (Snap::ly / double(Snap::ny));
  Snap::hk = 2.0 / (Snap::lz / double(Snap::nz));
  const int A = Snap::num_angles, nm = Snap::num_moments;
  free(Snap::mu); free(Snap::w); free(Snap::wmu); free(Snap::eta);
  free(Snap::weta); free(Snap::xi); free(Snap::wxi); free(Snap::ec);
  Snap::mu = (double *)calloc(A, sizeof(double));
  Snap::w = (double *)calloc(A, sizeof(double));
  Snap::wmu = (double *)calloc(A, sizeof(double));
  Snap::eta = (double *)calloc(A, sizeof(double));
  Snap::weta = (double *)calloc(A, sizeof(double));
  Snap::xi = (double *)calloc(A, sizeof(double));
  Snap::wxi = (double *)calloc(A, sizeof(double));
  const double dm = 1.0 / double(A);
  Snap::mu[0] = 0.5 * dm;
  for (int i = 1; i < A; i++) Snap::mu[i] = Snap::mu[i - 1] + dm;
  Snap::eta[0] = 1.0 - 0.5 * dm;
  for (int i = 1; i < A; i++) Snap::eta[i] = Snap::eta[i - 1] - dm;
  for (int i = 0; i < A; i++)
    Snap::xi[i] = sqrt(1.0 - (Snap::mu[i] * Snap::mu[i] + Snap::eta[i] * Snap::eta[i]));
  for (int i = 0; i < A; i++) Snap::w[i] = 0.125 / double(A);
  for (int i = 0; i < A; i++) {
    Snap::wmu[i] = Snap::w[i] * Snap::mu[i];
    Snap::weta[i] = Snap::w[i] * Snap::eta[i];
    Snap::wxi[i] = Snap::w[i] * Snap::xi[i];
  }
  Snap::ec = (double *)calloc((size_t)A * Snap::cmom * 8, sizeof(double));
  for (int l = 0; l < nm; l++) Snap::lma[l] = 2 * (l + 1) - 1;
  for (int oct = 0; oct < 8; oct++) {
    const double is = (oct & 1) ? 1.0 : -1.0, js = (oct & 2) ? 1.0 : -1.0,
                 ks = (oct & 4) ? 1.0 : -1.0;
    for (int idx = 0; idx < A; idx++) Snap::ec[oct * A * nm + idx] = 1.0;
    int moment = 1;
    for (int l = 1; l < nm; l++)
      for (int m = 0; m < 2 * (l + 1) - 1; m++) {
        for (int idx = 0; idx < A; idx++)
          Snap::ec[oct * A * nm + moment * A + idx] =
              pow(is * Snap::mu[idx], 2 * (l + 1) - 3) * pow(ks * Snap::xi[idx] * js * Snap::eta[idx], m);
        moment++;
      }
  }
}

struct Problem {
  Snap *snap = nullptr;
  FieldSpace group_fs, moment_fs, flux_moment_fs, mat_fs, angle_fs, flux_fs;
  IndexSpace<3> sim_is;
  IndexSpace<1> material_is, point_is;
  IndexSpace<2> slgg_is, xy_is, yz_is, xz_is;
};

FieldSpace make_fs(const std::vector<FieldID> &f, size_t sz) {
  FieldSpace fs;
  fs.fields = f;
  fs.field_size = sz;
  return fs;
}
template <int D> IndexSpace<D> make_is(const long long *lo, const long long *hi) {
  IndexSpace<D> is;
  for (int i = 0; i < D; i++) { is.lo[i] = lo[i]; is.hi[i] = hi[i]; }
  return is;
}

void build_problem(Problem &p) {
  const int G = Snap::num_groups, A = Snap::num_angles;
  std::vector<FieldID> gf(G), ff;
  for (int g = 0; g < G; g++) gf[g] = SNAP_ENERGY_GROUP_FIELD(g);
  for (int g = 0; g < G; g++)
    for (int c = 0; c < 8; c++) ff.push_back(SNAP_FLUX_GROUP_FIELD(g, c));
  p.group_fs = make_fs(gf, sizeof(double));
  p.moment_fs = make_fs(gf, sizeof(MomentQuad));
  p.flux_moment_fs = make_fs(gf, sizeof(MomentTriple));
  p.mat_fs = make_fs({Snap::FID_SINGLE}, sizeof(int));
  p.angle_fs = make_fs(gf, sizeof(double) * A);
  p.flux_fs = make_fs(ff, sizeof(double) * A);
  const long long z3[3] = {0, 0, 0};
  const long long u3[3] = {Snap::nx - 1, Snap::ny - 1, Snap::nz - 1};
  p.sim_is = make_is<3>(z3, u3);
  const long long m_lo[1] = {1}, m_hi[1] = {Snap::material_layout == Snap::HOMOGENEOUS_LAYOUT ? 1 : 2};
  p.material_is = make_is<1>(m_lo, m_hi);
  const long long s_lo[2] = {1, 0}, s_hi[2] = {m_hi[0], G - 1};
  p.slgg_is = make_is<2>(s_lo, s_hi);
  p.point_is = make_is<1>(z3, z3);
  const long long xy_hi[2] = {Snap::nx - 1, Snap::ny - 1}, yz_hi[2] = {Snap::ny - 1, Snap::nz - 1},
                  xz_hi[2] = {Snap::nx - 1, Snap::nz - 1};
  p.xy_is = make_is<2>(z3, xy_hi);
  p.yz_is = make_is<2>(z3, yz_hi);
  p.xz_is = make_is<2>(z3, xz_hi);
}

/* Runs tasks from a list on nthreads host threads. */
template <typename F> void parallel_for(int n, int nthreads, F f) {
  if (nthreads <= 1 || n <= 1) {
    for (int i = 0; i < n; i++) f(i);
    return;
  }
  std::atomic<int> next(0);
  std::vector<std::thread> th;
  for (int t = 0; t < nthreads; t++)
    th.emplace_back([&]() {
      for (int i = next++; i < n; i = next++) f(i);
    });
  for (auto &t : th) t.join();
}

/* The spatial chunk boxes (snap.cc:56-62 blockify): calls f(box) for every
 * chunk, x fastest, or f(nullptr) once when the mesh is one chunk. */
template <typename F> void for_each_chunk(F f) {
  const int nc[3] = {Snap::nx_chunks, Snap::ny_chunks, Snap::nz_chunks};
  if (nc[0] * nc[1] * nc[2] == 1) {
    f((const Legion::IndexSpace *)nullptr);
    return;
  }
  const int per[3] = {Snap::nx_per_chunk, Snap::ny_per_chunk, Snap::nz_per_chunk};
  for (int kz = 0; kz < nc[2]; kz++)
    for (int ky = 0; ky < nc[1]; ky++)
      for (int kx = 0; kx < nc[0]; kx++) {
        const int ck[3] = {kx, ky, kz};
        Legion::IndexSpace box;
        box.dim = 3;
        for (int d = 0; d < 3; d++) {
          box.lo[d] = (long long)ck[d] * per[d];
          box.hi[d] = (long long)(ck[d] + 1) * per[d] - 1;
        }
        f((const Legion::IndexSpace *)&box);
      }
}

typedef void (*SweepImpl)(const Task *, const std::vector<PhysicalRegion> &, Context, Runtime *);

SweepImpl pick_sweep(int variant) {
  switch (variant) {
    case 0: return &MiniKBATask::cpu_implementation;
    case 1: return &MiniKBATask::sse_implementation;
#ifdef __AVX__
    case 2: return &MiniKBATask::avx_implementation;
#endif
    default: return nullptr;
  }
}

}  // namespace

extern "C" {

/* Sets the deck parameters (snap.cc:1032-1168 fields, single chunk). */
int snapref_configure(int nx, int ny, int nz, int nang, int ng, int nmom, int two_materials,
                      double epsi, int iitm, int oitm, int fixup) {
  if (nmom != 1) return -1; /* the reference's nmom > 1 CPU path is unsound */
  Snap::num_dims = 3;
  Snap::nx = Snap::nx_per_chunk = nx;
  Snap::ny = Snap::ny_per_chunk = ny;
  Snap::nz = Snap::nz_per_chunk = nz;
  Snap::nx_chunks = Snap::ny_chunks = Snap::nz_chunks = 1;
  Snap::lx = Snap::ly = Snap::lz = 1.0;
  Snap::num_angles = nang;
  Snap::num_groups = ng;
  Snap::num_moments = nmom;
  Snap::convergence_eps = epsi;
  Snap::max_inner_iters = iitm;
  Snap::max_outer_iters = oitm;
  Snap::flux_fixup = fixup != 0;
  Snap::time_dependent = false;
  Snap::total_sim_time = 0.0;
  Snap::num_steps = 1;
  Snap::dt = 0.0;
  Snap::material_layout = two_materials ? Snap::CENTER_LAYOUT : Snap::HOMOGENEOUS_LAYOUT;
  Snap::source_layout = Snap::CENTER_SOURCE;
  Snap::num_corners = 8;
  derive_globals();
  return 0;
}

/* Sets every deck parameter the solve path reads (the fields parse_arguments
 * fills, snap.cc:1032-1168), single spatial chunk.  mat_opt: 0 homogeneous,
 * 1 center, 2 corner; src_opt: 0 everywhere, 1 center, 2 corner. */
int snapref_configure_deck(int nx, int ny, int nz, double lx, double ly, double lz, int nang,
                           int ng, int nmom, double epsi, int iitm, int oitm, int fixup,
                           int timedep, double tf, int nsteps, int mat_opt, int src_opt,
                           int ichunk, int npey, int npez) {
  if (nmom != 1) return -1;
  if (mat_opt < 0 || mat_opt > 2 || src_opt < 0 || src_opt > 3 || nsteps < 1) return -2;
  if (ichunk < 1 || npey < 1 || npez < 1 || nx % ichunk || ny % npey || nz % npez) return -4;
  Snap::num_dims = 3;
  Snap::nx = nx;
  Snap::ny = ny;
  Snap::nz = nz;
  Snap::nx_chunks = ichunk;   /* snap.cc:1044-1046, 1161-1163 */
  Snap::ny_chunks = npey;
  Snap::nz_chunks = npez;
  Snap::nx_per_chunk = nx / ichunk;
  Snap::ny_per_chunk = ny / npey;
  Snap::nz_per_chunk = nz / npez;
  Snap::lx = lx;
  Snap::ly = ly;
  Snap::lz = lz;
  Snap::num_angles = nang;
  Snap::num_groups = ng;
  Snap::num_moments = nmom;
  Snap::convergence_eps = epsi;
  Snap::max_inner_iters = iitm;
  Snap::max_outer_iters = oitm;
  Snap::flux_fixup = fixup != 0;
  Snap::time_dependent = timedep != 0;
  Snap::total_sim_time = tf;
  Snap::num_steps = nsteps;
  static const Snap::MaterialLayout ml[3] = {Snap::HOMOGENEOUS_LAYOUT, Snap::CENTER_LAYOUT,
                                             Snap::CORNER_LAYOUT};
  static const Snap::SourceLayout sl[4] = {Snap::EVERYWHERE_SOURCE, Snap::CENTER_SOURCE,
                                           Snap::CORNER_SOURCE, Snap::MMS_SOURCE};
  Snap::material_layout = ml[mat_opt];
  Snap::source_layout = sl[src_opt];
  Snap::num_corners = 8;
  Snap::dt = tf / double(nsteps);   /* snap.cc:1174 */
  derive_globals();
  return 0;
}

/* Quadrature as the reference computes it (for cross-checks). */
void snapref_quadrature(double *mu, double *eta, double *xi, double *w) {
  for (int i = 0; i < Snap::num_angles; i++) {
    mu[i] = Snap::mu[i]; eta[i] = Snap::eta[i]; xi[i] = Snap::xi[i]; w[i] = Snap::w[i];
  }
}

/* Runs the reference's InitMaterial / InitSource tasks (center layouts,
 * init.cc:49-191) and returns mat [C] and qi [G][C]. */
int snapref_init_layout(int32_t *mat_out, double *qi_out) {
  Problem p;
  build_problem(p);
  Snap snap(nullptr, &g_runtime);
  IndexPartition<3> ip3;
  SnapArray<3> mat(p.sim_is, ip3, p.mat_fs, nullptr, &g_runtime, "mat");
  SnapArray<3> qi(p.sim_is, ip3, p.group_fs, nullptr, &g_runtime, "qi");
  int *m = (int *)store_of(mat).mem;
  for (size_t c = 0; c < store_of(mat).volume; c++) m[c] = 1; /* snap.cc:325 */
  /* snap.cc:345-349: InitMaterial runs for the non-homogeneous layouts only */
  if (Snap::material_layout != Snap::HOMOGENEOUS_LAYOUT) {
    InitMaterial im(snap, mat);
    execute<void>(im, &InitMaterial::cpu_implementation);
  }
  InitSource is(snap, qi);
  execute<void>(is, &InitSource::cpu_implementation);
  const size_t C = store_of(mat).volume;
  memcpy(mat_out, store_of(mat).mem, C * sizeof(int));
  memcpy(qi_out, store_of(qi).mem, C * Snap::num_groups * sizeof(double));
  return 0;
}

/*
 * Steady-state solve with the reference's task bodies.
 *   mat [C] (1-based), qi [G][C], sigt [G][nmat], slgg [G_to][nmat][G_from][nmom]
 *   variant: 0 scalar, 1 SSE, 2 AVX sweep body
 *   flux_out [G][C]; info[0] inner total, info[1] outer total, info[2]
 *   converged (last time step), info[3+r] inner iterations of the r-th
 *   outer iteration over all time steps (r < oitm * nsteps)
 *   max_inners_total > 0 stops after that many inner iterations (timing).
 * Returns seconds spent, or a negative error.
 */
double snapref_solve(const int32_t *mat_in, const double *qi_in, const double *sigt_in,
                     const double *slgg_in, int nmat, int variant, int nthreads,
                     int max_inners_total, double *flux_out, int *info,
                     double *sweep_seconds, double *mms_out, double *ref_flux_out) {
  SweepImpl sweep_impl = pick_sweep(variant);
  if (!sweep_impl) return -1.0;
  /* info holds 3 + oitm * nsteps entries: outer iterations of every step */
  const int max_records = Snap::max_outer_iters * Snap::num_steps;
  if (variant == 1 && Snap::num_angles % 2) return -2.0;
  if (variant == 2 && Snap::num_angles % 4) return -2.0;
  const int G = Snap::num_groups;
  Problem p;
  build_problem(p);
  Snap snap(nullptr, &g_runtime);
  IndexPartition<3> ip3;
  IndexPartition<2> ip2;
  IndexPartition<1> ip1;
  SnapArray<3> flux0(p.sim_is, ip3, p.group_fs, nullptr, &g_runtime, "flux0");
  SnapArray<3> flux0po(p.sim_is, ip3, p.group_fs, nullptr, &g_runtime, "flux0po");
  SnapArray<3> flux0pi(p.sim_is, ip3, p.group_fs, nullptr, &g_runtime, "flux0pi");
  SnapArray<3> fluxm(p.sim_is, ip3, p.flux_moment_fs, nullptr, &g_runtime, "fluxm");
  SnapArray<2> flux_xy(p.xy_is, ip2, p.flux_fs, nullptr, &g_runtime, "fluxXY");
  SnapArray<2> flux_yz(p.yz_is, ip2, p.flux_fs, nullptr, &g_runtime, "fluxYZ");
  SnapArray<2> flux_xz(p.xz_is, ip2, p.flux_fs, nullptr, &g_runtime, "fluxXZ");
  SnapArray<3> qi(p.sim_is, ip3, p.group_fs, nullptr, &g_runtime, "qi");
  SnapArray<3> q2grp0(p.sim_is, ip3, p.group_fs, nullptr, &g_runtime, "q2grp0");
  SnapArray<3> q2grpm(p.sim_is, ip3, p.flux_moment_fs, nullptr, &g_runtime, "q2grpm");
  SnapArray<3> qtot(p.sim_is, ip3, p.moment_fs, nullptr, &g_runtime, "qtot");
  SnapArray<3> mat(p.sim_is, ip3, p.mat_fs, nullptr, &g_runtime, "mat");
  SnapArray<1> sigt(p.material_is, ip1, p.group_fs, nullptr, &g_runtime, "sigt");
  SnapArray<1> siga(p.material_is, ip1, p.group_fs, nullptr, &g_runtime, "siga");
  SnapArray<2> slgg(p.slgg_is, ip2, p.moment_fs, nullptr, &g_runtime, "slgg");
  SnapArray<3> t_xs(p.sim_is, ip3, p.group_fs, nullptr, &g_runtime, "t_xs");
  SnapArray<3> a_xs(p.sim_is, ip3, p.group_fs, nullptr, &g_runtime, "a_xs");
  SnapArray<3> s_xs(p.sim_is, ip3, p.moment_fs, nullptr, &g_runtime, "s_xs");
  SnapArray<1> vdelt(p.point_is, ip1, p.group_fs, nullptr, &g_runtime, "vdelt");
  SnapArray<3> dinv(p.sim_is, ip3, p.angle_fs, nullptr, &g_runtime, "dinv");
  /* the MMS region is named by the sweep's region requirements but never
   * dereferenced outside MMS decks (sweep.cc:369); the time-edge angular
   * flux is real storage in time-dependent decks only (sweep.cc:413) */
  const bool td = Snap::time_dependent;
  const bool mms = Snap::source_layout == Snap::MMS_SOURCE;
  g_phantom_next = !mms;
  std::vector<SnapArray<3> *> qim(8);
  for (int i = 0; i < 8; i++)
    qim[i] = new SnapArray<3>(p.sim_is, ip3, p.angle_fs, nullptr, &g_runtime, "qim");
  SnapArray<3> ref_flux(p.sim_is, ip3, p.group_fs, nullptr, &g_runtime, "ref_flux");
  SnapArray<3> ref_fluxm(p.sim_is, ip3, p.flux_moment_fs, nullptr, &g_runtime, "ref_fluxm");
  SnapArray<1> vel(p.point_is, ip1, p.group_fs, nullptr, &g_runtime, "vel");
  g_phantom_next = !td;
  std::vector<SnapArray<3> *> tf_even(8), tf_odd(8);
  for (int i = 0; i < 8; i++) {
    tf_even[i] = new SnapArray<3>(p.sim_is, ip3, p.angle_fs, nullptr, &g_runtime, "tf even");
    tf_odd[i] = new SnapArray<3>(p.sim_is, ip3, p.angle_fs, nullptr, &g_runtime, "tf odd");
  }
  g_phantom_next = false;
  struct TfFree {
    std::vector<SnapArray<3> *> &a, &b;
    ~TfFree() {
      for (auto *x : a) delete x;
      for (auto *x : b) delete x;
    }
  } tf_free{tf_even, tf_odd};
  struct QimFree {
    std::vector<SnapArray<3> *> &a;
    ~QimFree() {
      for (auto *x : a) delete x;
    }
  } qim_free{qim};
  /* Snap::initialize_velocity (snap.cc:717-739): v_g = G - g,
   * vdelt = 2 / (dt v_g) when time dependent, else 0 */
  for (int g = 0; g < G; g++) {
    const double v = double(G - g);
    ((double *)store_of(vdelt).field_base(g))[0] = td ? 2.0 / (Snap::dt * v) : 0.0;
    if (mms) ((double *)store_of(vel).field_base(g))[0] = v;
  }

  const size_t C = store_of(flux0).volume;
  if (nmat != (int)store_of(sigt).volume) return -3.0;
  memcpy(store_of(mat).mem, mat_in, C * sizeof(int));
  memcpy(store_of(qi).mem, qi_in, C * G * sizeof(double));
  /* sigt field g, point m (1-based) */
  for (int g = 0; g < G; g++)
    for (int m = 0; m < nmat; m++) {
      ((double *)store_of(sigt).field_base(g))[m] = sigt_in[g * nmat + m];
      ((double *)store_of(siga).field_base(g))[m] = 0.5 * sigt_in[g * nmat + m];
    }
  /* slgg field g_to, point (m, g_from), MomentQuad */
  const int nmom = Snap::num_moments;
  for (int gt = 0; gt < G; gt++)
    for (int m = 0; m < nmat; m++)
      for (int gf = 0; gf < G; gf++) {
        MomentQuad *q = (MomentQuad *)store_of(slgg).field_base(gt);
        MomentQuad v;
        for (int l = 0; l < nmom && l < 4; l++) v[l] = slgg_in[(((size_t)gt * nmat + m) * G + gf) * nmom + l];
        q[m + (size_t)nmat * gf] = v;
      }

  /* per time step cross-section expansion (snap.cc:419-450), chunk = 1 group */
  for (int g = 0; g < G; g++) {
    ExpandCrossSection ea(snap, siga, mat, a_xs, g, g);
    execute<void>(ea, &ExpandCrossSection::cpu_implementation);
    ExpandCrossSection et(snap, sigt, mat, t_xs, g, g);
    execute<void>(et, &ExpandCrossSection::cpu_implementation);
    ExpandScatteringCrossSection es(snap, slgg, mat, s_xs, g, g);
    execute<void>(es, &ExpandScatteringCrossSection::cpu_implementation);
    CalculateGeometryParam gp(snap, t_xs, vdelt, dinv, g, g);
    execute<void>(gp, &CalculateGeometryParam::cpu_implementation);
  }

  /* the manufactured solution (snap.cc:373-388): reference flux, the
   * per-corner angular source and, time dependent, qi = flux / v with the
   * reference flux scaled to the middle of the last step */
  if (mms) {
    /* index launches over the chunks: each task sees its own sub-box */
    MMSInitFlux mf(snap, ref_flux, ref_fluxm);
    for_each_chunk([&](const Legion::IndexSpace *b) {
      execute<void>(mf, &MMSInitFlux::cpu_implementation, b);
    });
    for (int i = 0; i < 8; i++) {
      MMSInitSource ms(snap, ref_flux, ref_fluxm, mat, sigt, slgg, *qim[i], i);
      for_each_chunk([&](const Legion::IndexSpace *b) {
        execute<void>(ms, &MMSInitSource::cpu_implementation, b);
      });
    }
    if (td) {
      MMSInitTimeDependent mt(snap, vel, ref_flux, qi);
      for_each_chunk([&](const Legion::IndexSpace *b) {
        execute<void>(mt, &MMSInitTimeDependent::cpu_implementation, b);
      });
    }
  }

  Predicate pred;
  const Future true_future = Future::from_value<bool>(nullptr, true);
  int inner_total = 0, outer_total = 0, converged = 0, records = 0;
  double t_sweep = 0.0;
  const auto t0 = std::chrono::steady_clock::now();
  bool stop = false;
  bool even_time_step = false;
  for (int cy = 0; cy < Snap::num_steps && !stop; ++cy) {
  even_time_step = !even_time_step;   /* snap.cc:411 */
  if (mms) { /* snap.cc:451-466 */
    const double f = cy == 0 ? Snap::dt * 0.5 : double(2 * cy + 1) / double(2 * cy - 1);
    for (int i = 0; i < 8; i++) {
      MMSScale sc(snap, *qim[i], f);
      for_each_chunk([&](const Legion::IndexSpace *b) {
        execute<void>(sc, &MMSScale::cpu_implementation, b);
      });
    }
  }
  std::vector<SnapArray<3> *> &tf_in = even_time_step ? tf_even : tf_odd;
  std::vector<SnapArray<3> *> &tf_out = even_time_step ? tf_odd : tf_even;
  converged = 0;
  for (int otno = 0; otno < Snap::max_outer_iters && !stop; ++otno) {
    CalcOuterSource os(snap, pred, qi, slgg, mat, q2grp0, q2grpm, flux0, fluxm);
    execute<void>(os, &CalcOuterSource::cpu_implementation);
    copy_store(store_of(flux0), store_of(flux0po)); /* save_fluxes */
    bool inner_conv = false;
    int inners = 0;
    for (int inno = 0; inno < Snap::max_inner_iters; ++inno) {
      for (int g = 0; g < G; g++) {
        CalcInnerSource is(snap, pred, s_xs, flux0, fluxm, q2grp0, q2grpm, qtot, g, g);
        execute<void>(is, &CalcInnerSource::cpu_implementation);
      }
      copy_store(store_of(flux0), store_of(flux0pi));
      fill_zero(store_of(flux0));
      /* perform_sweeps (snap.cc:849-887): zero the faces, then every
       * (corner, group) task; they only share flux0 (CAS adds) */
      fill_zero(store_of(flux_xy));
      fill_zero(store_of(flux_yz));
      fill_zero(store_of(flux_xz));
      const auto ts = std::chrono::steady_clock::now();
      parallel_for(8 * G, nthreads, [&](int t) {
        const int corner = t / G, g = t % G;
        int ghost_offsets[3] = {0, 0, 0};
        for (int i = 0; i < 3; i++) ghost_offsets[i] = (corner & (1 << i)) >> i;
        MiniKBATask k(snap, pred, flux0, fluxm, qtot, vdelt, dinv, t_xs, *tf_in[corner],
                      *tf_out[corner], *qim[corner], flux_xy, flux_yz, flux_xz, g, g, corner,
                      ghost_offsets);
        if (Snap::nx_chunks * Snap::ny_chunks * Snap::nz_chunks == 1) {
          execute<void>(k, sweep_impl);
          return;
        }
        /* one task per spatial chunk (snap.cc:56-62 blockify), upstream
         * chunks first; chunks pass faces through the shared face arrays */
        const int nc[3] = {Snap::nx_chunks, Snap::ny_chunks, Snap::nz_chunks};
        const int per[3] = {Snap::nx_per_chunk, Snap::ny_per_chunk, Snap::nz_per_chunk};
        for (int kz = 0; kz < nc[2]; kz++)
          for (int ky = 0; ky < nc[1]; ky++)
            for (int kx = 0; kx < nc[0]; kx++) {
              const int ck[3] = {kx, ky, kz};
              Legion::IndexSpace box;
              box.dim = 3;
              for (int d = 0; d < 3; d++) {
                const int cc = (corner >> d) & 1 ? ck[d] : nc[d] - 1 - ck[d];
                box.lo[d] = (long long)cc * per[d];
                box.hi[d] = (long long)(cc + 1) * per[d] - 1;
              }
              execute<void>(k, sweep_impl, &box);
            }
      });
      t_sweep += std::chrono::duration<double>(std::chrono::steady_clock::now() - ts).count();
      inners++;
      inner_total++;
      bool conv = true;
      for (int g = 0; g < G && conv; g++) {
        TestInnerConvergence tc(snap, pred, flux0, flux0pi, true_future, g, g);
        conv = execute<bool>(tc, &TestInnerConvergence::cpu_implementation);
      }
      inner_conv = conv;
      if (max_inners_total > 0 && inner_total >= max_inners_total) { stop = true; break; }
      if (inner_conv) break;
    }
    if (info && records < max_records) info[3 + records] = inners;
    records++;
    outer_total++;
    if (stop) break;
    if (otno == 0) continue;
    const Future inner_future = Future::from_value<bool>(nullptr, inner_conv);
    bool conv = true;
    for (int g = 0; g < G && conv; g++) {
      TestOuterConvergence tc(snap, pred, flux0, flux0po, inner_future, true_future, g, g);
      conv = execute<bool>(tc, &TestOuterConvergence::cpu_implementation);
    }
    if (conv) { converged = 1; break; }
  }
  }
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (flux_out) memcpy(flux_out, store_of(flux0).mem, C * G * sizeof(double));
  if (mms) { /* snap.cc:542-560 */
    /* one result per chunk, folded as MMSReduction does (mms.cc:549-600):
     * max, min, sum */
    MMSCompare cmp(snap, flux0, ref_flux);
    double red[3] = {0.0, 0.0, 0.0};
    bool first = true;
    for_each_chunk([&](const Legion::IndexSpace *b) {
      const MomentTriple r = execute<MomentTriple>(cmp, &MMSCompare::cpu_implementation, b);
      if (first) {
        for (int i = 0; i < 3; i++) red[i] = r[i];
        first = false;
      } else {
        red[0] = std::max(red[0], r[0]);
        red[1] = std::min(red[1], r[1]);
        red[2] += r[2];
      }
    });
    if (mms_out) for (int i = 0; i < 3; i++) mms_out[i] = red[i];
    if (ref_flux_out) memcpy(ref_flux_out, store_of(ref_flux).mem, C * G * sizeof(double));
  }
  if (info) { info[0] = inner_total; info[1] = outer_total; info[2] = converged; }
  if (sweep_seconds) *sweep_seconds = t_sweep;
  return secs;
}

/*
 * Times `steps` inner iterations of the steady-state solve exactly as one
 * step of the GPU benchmark runs them: the inner source of every group
 * (snap.cc:487-491), the save of the scalar flux, the sweep of every corner
 * and group (snap.cc:494-499) and the inner test of every group
 * (snap.cc:500-503), each as a set of independent group (or corner x group)
 * tasks on nthreads host threads, the way the reference's index launches run
 * them.  One outer source (snap.cc:477) precedes the timed region.
 * Returns the seconds of the timed iterations (sweep seconds in *sweep_s).
 */
double snapref_time_inner(const int32_t *mat_in, const double *qi_in, const double *sigt_in,
                          const double *slgg_in, int nmat, int variant, int nthreads, int steps,
                          double *sweep_s) {
  SweepImpl sweep_impl = pick_sweep(variant);
  if (!sweep_impl || steps < 1) return -1.0;
  const int G = Snap::num_groups;
  Problem p;
  build_problem(p);
  Snap snap(nullptr, &g_runtime);
  IndexPartition<3> ip3;
  IndexPartition<2> ip2;
  IndexPartition<1> ip1;
  SnapArray<3> flux0(p.sim_is, ip3, p.group_fs, nullptr, &g_runtime, "flux0");
  SnapArray<3> flux0pi(p.sim_is, ip3, p.group_fs, nullptr, &g_runtime, "flux0pi");
  SnapArray<3> fluxm(p.sim_is, ip3, p.flux_moment_fs, nullptr, &g_runtime, "fluxm");
  SnapArray<2> flux_xy(p.xy_is, ip2, p.flux_fs, nullptr, &g_runtime, "fluxXY");
  SnapArray<2> flux_yz(p.yz_is, ip2, p.flux_fs, nullptr, &g_runtime, "fluxYZ");
  SnapArray<2> flux_xz(p.xz_is, ip2, p.flux_fs, nullptr, &g_runtime, "fluxXZ");
  SnapArray<3> qi(p.sim_is, ip3, p.group_fs, nullptr, &g_runtime, "qi");
  SnapArray<3> q2grp0(p.sim_is, ip3, p.group_fs, nullptr, &g_runtime, "q2grp0");
  SnapArray<3> q2grpm(p.sim_is, ip3, p.flux_moment_fs, nullptr, &g_runtime, "q2grpm");
  SnapArray<3> qtot(p.sim_is, ip3, p.moment_fs, nullptr, &g_runtime, "qtot");
  SnapArray<3> mat(p.sim_is, ip3, p.mat_fs, nullptr, &g_runtime, "mat");
  SnapArray<1> sigt(p.material_is, ip1, p.group_fs, nullptr, &g_runtime, "sigt");
  SnapArray<2> slgg(p.slgg_is, ip2, p.moment_fs, nullptr, &g_runtime, "slgg");
  SnapArray<3> t_xs(p.sim_is, ip3, p.group_fs, nullptr, &g_runtime, "t_xs");
  SnapArray<3> s_xs(p.sim_is, ip3, p.moment_fs, nullptr, &g_runtime, "s_xs");
  SnapArray<1> vdelt(p.point_is, ip1, p.group_fs, nullptr, &g_runtime, "vdelt");
  SnapArray<3> dinv(p.sim_is, ip3, p.angle_fs, nullptr, &g_runtime, "dinv");
  g_phantom_next = true;
  SnapArray<3> tf(p.sim_is, ip3, p.angle_fs, nullptr, &g_runtime, "time flux");
  SnapArray<3> qim(p.sim_is, ip3, p.angle_fs, nullptr, &g_runtime, "qim");
  g_phantom_next = false;
  const size_t C = store_of(flux0).volume;
  if (nmat != (int)store_of(sigt).volume) return -3.0;
  memcpy(store_of(mat).mem, mat_in, C * sizeof(int));
  memcpy(store_of(qi).mem, qi_in, C * G * sizeof(double));
  for (int g = 0; g < G; g++)
    for (int m = 0; m < nmat; m++) ((double *)store_of(sigt).field_base(g))[m] = sigt_in[g * nmat + m];
  for (int gt = 0; gt < G; gt++)
    for (int m = 0; m < nmat; m++)
      for (int gf = 0; gf < G; gf++) {
        MomentQuad v;
        v[0] = slgg_in[((size_t)gt * nmat + m) * G + gf];   /* nmom = 1 */
        ((MomentQuad *)store_of(slgg).field_base(gt))[m + (size_t)nmat * gf] = v;
      }
  parallel_for(G, nthreads, [&](int g) {
    ExpandCrossSection et(snap, sigt, mat, t_xs, g, g);
    execute<void>(et, &ExpandCrossSection::cpu_implementation);
    ExpandScatteringCrossSection es(snap, slgg, mat, s_xs, g, g);
    execute<void>(es, &ExpandScatteringCrossSection::cpu_implementation);
    CalculateGeometryParam gp(snap, t_xs, vdelt, dinv, g, g);
    execute<void>(gp, &CalculateGeometryParam::cpu_implementation);
  });
  Predicate pred;
  const Future true_future = Future::from_value<bool>(nullptr, true);
  CalcOuterSource os(snap, pred, qi, slgg, mat, q2grp0, q2grpm, flux0, fluxm);
  execute<void>(os, &CalcOuterSource::cpu_implementation);
  double t_sweep = 0.0;
  const auto t0 = std::chrono::steady_clock::now();
  for (int it = 0; it < steps; ++it) {
    parallel_for(G, nthreads, [&](int g) {
      CalcInnerSource is(snap, pred, s_xs, flux0, fluxm, q2grp0, q2grpm, qtot, g, g);
      execute<void>(is, &CalcInnerSource::cpu_implementation);
    });
    copy_store(store_of(flux0), store_of(flux0pi));
    fill_zero(store_of(flux0));
    fill_zero(store_of(flux_xy));
    fill_zero(store_of(flux_yz));
    fill_zero(store_of(flux_xz));
    const auto ts = std::chrono::steady_clock::now();
    parallel_for(8 * G, nthreads, [&](int t) {
      const int corner = t / G, g = t % G;
      int ghost_offsets[3] = {0, 0, 0};
      for (int i = 0; i < 3; i++) ghost_offsets[i] = (corner & (1 << i)) >> i;
      MiniKBATask k(snap, pred, flux0, fluxm, qtot, vdelt, dinv, t_xs, tf, tf, qim, flux_xy,
                    flux_yz, flux_xz, g, g, corner, ghost_offsets);
      execute<void>(k, sweep_impl);
    });
    t_sweep += std::chrono::duration<double>(std::chrono::steady_clock::now() - ts).count();
    std::atomic<int> conv_all(1);
    parallel_for(G, nthreads, [&](int g) {
      TestInnerConvergence tc(snap, pred, flux0, flux0pi, true_future, g, g);
      if (!execute<bool>(tc, &TestInnerConvergence::cpu_implementation)) conv_all = 0;
    });
  }
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (sweep_s) *sweep_s = t_sweep;
  return secs;
}

}  // extern "C"
