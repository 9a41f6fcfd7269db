/*
 * Minimal, from-scratch stand-in for the subset of the Legion C++ API that the
 * reference's CPU task bodies use (TEST INFRASTRUCTURE ONLY).
 *
 * The reference application needs the Legion runtime, which is not vendored
 * with it and not installed here.  Its CPU task variants (sweep.cc, outer.cc,
 * inner.cc, expxs.cc, init.cc) only touch a small surface: affine field
 * accessors, points/rects and their iterators, the Task descriptor, a few
 * launcher/registration types that the task constructors and
 * preregister_* functions name.  This header provides exactly that surface,
 * with sequential single-address-space semantics, so the unmodified reference
 * sources compile into the oracle's reference build (oracle/Makefile).
 * Nothing here schedules tasks: ref_driver.cc executes the launchers that the
 * reference's own task constructors build.
 */
#ifndef SNAP_REFSHIM_LEGION_H
#define SNAP_REFSHIM_LEGION_H

#include <cassert>
#include <cstddef>
#include <cstdarg>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <type_traits>
#include <map>
#include <set>
#include <string>
#include <vector>

/* ---- global enums that Legion exports unqualified (legion_config.h) ---- */
enum PrivilegeMode { NO_ACCESS = 0, READ_ONLY = 1, READ_WRITE = 2, WRITE_DISCARD = 3, REDUCE = 4 };
enum CoherenceProperty { EXCLUSIVE = 0, ATOMIC = 1, SIMULTANEOUS = 2, RELAXED = 3 };
enum ISAKind : unsigned long long {
  X86_ISA = 1ull << 0, SSE_ISA = 1ull << 1, AVX_ISA = 1ull << 2, CUDA_ISA = 1ull << 3,
  SM_30_ISA = 1ull << 4, AVX2_ISA = 1ull << 5
};
enum ResourceKind { L1_CACHE_SIZE, L1_CACHE_ASSOCIATIVITY, SHARED_MEMORY_SIZE, REGISTER_FILE_SIZE };
enum EqualityKind { GE_EK, LE_EK, EQ_EK };
enum LaunchKind { LEGION_CTAS_PER_SM, LEGION_THREADS_PER_CTA };
#define IDFMT "%llx"

namespace Realm {
template <typename FT, int N, typename T> struct AffineAccessor {};
}

namespace Legion {

typedef unsigned FieldID;
typedef unsigned ProjectionID;
typedef unsigned ReductionOpID;
typedef unsigned long LayoutConstraintID;
typedef unsigned VariantID;
typedef unsigned AddressSpace;
typedef unsigned TaskID;
typedef ::PrivilegeMode PrivilegeMode;
typedef int DimensionKind;

template <int DIM, typename T = long long> struct Point {
  T coords[DIM];
  Point() { for (int i = 0; i < DIM; i++) coords[i] = 0; }
  explicit Point(T a) { for (int i = 0; i < DIM; i++) coords[i] = a; }
  Point(T a, T b) { coords[0] = a; coords[1] = b; }
  Point(T a, T b, T c) { coords[0] = a; coords[1] = b; coords[2] = c; }
  explicit Point(const T *v) { for (int i = 0; i < DIM; i++) coords[i] = v[i]; }
  T &operator[](int i) { return coords[i]; }
  const T &operator[](int i) const { return coords[i]; }
  bool operator<(const Point &o) const {
    for (int i = 0; i < DIM; i++) if (coords[i] != o.coords[i]) return coords[i] < o.coords[i];
    return false;
  }
  bool operator==(const Point &o) const {
    for (int i = 0; i < DIM; i++) if (coords[i] != o.coords[i]) return false;
    return true;
  }
};

template <int DIM, typename T = long long> struct Rect {
  Point<DIM, T> lo, hi;
  Rect() {}
  Rect(const Point<DIM, T> &l, const Point<DIM, T> &h) : lo(l), hi(h) {}
  size_t volume() const {
    size_t v = 1;
    for (int i = 0; i < DIM; i++) {
      if (hi[i] < lo[i]) return 0;
      v *= (size_t)(hi[i] - lo[i] + 1);
    }
    return v;
  }
  bool empty() const { return volume() == 0; }
  Rect intersection(const Rect &o) const {
    Rect r;
    for (int i = 0; i < DIM; i++) {
      r.lo[i] = lo[i] > o.lo[i] ? lo[i] : o.lo[i];
      r.hi[i] = hi[i] < o.hi[i] ? hi[i] : o.hi[i];
    }
    return r;
  }
};

template <int D1, int D2, typename T = long long> struct Transform {};

/* An index space is a dense rectangle of up to three dimensions. */
struct IndexSpace {
  int dim = 0;
  long long lo[3] = {0, 0, 0}, hi[3] = {-1, -1, -1};
  bool operator==(const IndexSpace &o) const {
    if (dim != o.dim) return false;
    for (int i = 0; i < dim; i++) if (lo[i] != o.lo[i] || hi[i] != o.hi[i]) return false;
    return true;
  }
};
template <int DIM, typename T = long long> struct IndexSpaceT : public IndexSpace {
  IndexSpaceT() { dim = DIM; }
  explicit IndexSpaceT(const IndexSpace &is) : IndexSpace(is) {}
  explicit IndexSpaceT(const Rect<DIM, T> &r) {
    dim = DIM;
    for (int i = 0; i < DIM; i++) { lo[i] = r.lo[i]; hi[i] = r.hi[i]; }
  }
  Rect<DIM, T> bounds() const {
    Rect<DIM, T> r;
    for (int i = 0; i < DIM; i++) { r.lo[i] = lo[i]; r.hi[i] = hi[i]; }
    return r;
  }
};
struct IndexPartition { int id = 0; };
template <int DIM, typename T = long long> struct IndexPartitionT : public IndexPartition {};

struct FieldSpace {
  int id = 0;
  std::vector<FieldID> fields;
  size_t field_size = 0;
};

struct LogicalRegion {
  int handle = -1;
  IndexSpace is;
  IndexSpace get_index_space() const { return is; }
  bool operator<(const LogicalRegion &o) const { return handle < o.handle; }
  bool operator==(const LogicalRegion &o) const { return handle == o.handle; }
};
template <int DIM, typename T = long long> struct LogicalRegionT : public LogicalRegion {};
struct LogicalPartition {
  int handle = -1;
  IndexSpace is;
};
template <int DIM, typename T = long long> struct LogicalPartitionT : public LogicalPartition {};

template <int DIM, typename T = long long> struct DomainT {
  Rect<DIM, T> bounds;
};
struct DomainPoint {};
struct Domain {};

template <int DIM, typename T = long long> struct PointInRectIterator {
  Rect<DIM, T> rect;
  Point<DIM, T> p;
  bool valid;
  explicit PointInRectIterator(const Rect<DIM, T> &r) : rect(r), p(r.lo), valid(!r.empty()) {}
  bool operator()() const { return valid; }
  Point<DIM, T> operator*() const { return p; }
  void step() {
    /* dimension 0 varies fastest (Fortran order) */
    for (int i = 0; i < DIM; i++) {
      if (p[i] < rect.hi[i]) { p[i]++; return; }
      p[i] = rect.lo[i];
    }
    valid = false;
  }
  PointInRectIterator &operator++() { step(); return *this; }
  PointInRectIterator operator++(int) { PointInRectIterator t = *this; step(); return t; }
};
template <int DIM, typename T = long long> struct PointInDomainIterator
    : public PointInRectIterator<DIM, T> {
  explicit PointInDomainIterator(const DomainT<DIM, T> &d) : PointInRectIterator<DIM, T>(d.bounds) {}
};

/* A physical region maps each field to (address of point zero, byte
 * strides).  Storage belongs to ref_driver.cc. */
struct FieldLayout {
  char *zero = nullptr;
  long long strides[3] = {0, 0, 0};
  size_t field_size = 0;
};
struct PhysicalRegion {
  int dim = 0;
  std::map<FieldID, FieldLayout> fields;
  void wait_until_valid(bool = false) {}
  const FieldLayout &layout(FieldID fid) const {
    auto it = fields.find(fid);
    assert(it != fields.end());
    return it->second;
  }
};

template <typename FT, int REM, typename T> struct AccessorProxy {
  char *addr;
  const long long *strides;
  AccessorProxy<FT, REM - 1, T> operator[](T i) const {
    return AccessorProxy<FT, REM - 1, T>{addr + i * strides[0], strides + 1};
  }
};
template <typename FT, typename T> struct AccessorProxy<FT, 1, T> {
  char *addr;
  const long long *strides;
  FT &operator[](T i) const { return *reinterpret_cast<FT *>(addr + i * strides[0]); }
};

template <PrivilegeMode PRIV, typename FT, int N, typename T = long long,
          typename A = Realm::AffineAccessor<FT, N, T>, bool CB = false>
class FieldAccessor {
 public:
  FieldAccessor() {}
  FieldAccessor(const PhysicalRegion &region, FieldID fid, size_t actual_field_size = sizeof(FT)) {
    const FieldLayout &l = region.layout(fid);
    assert(actual_field_size <= l.field_size);
    zero = l.zero;
    for (int i = 0; i < 3; i++) strides[i] = l.strides[i];
  }
  FT *ptr(const Point<N, T> &p) const {
    char *a = zero;
    for (int i = 0; i < N; i++) a += p[i] * strides[i];
    return reinterpret_cast<FT *>(a);
  }
  FT &operator[](const Point<N, T> &p) const { return *ptr(p); }
  template <int M = N>
  typename std::enable_if<(M > 1), AccessorProxy<FT, N - 1, T>>::type operator[](T i) const {
    return AccessorProxy<FT, N - 1, T>{zero + i * strides[0], strides + 1};
  }
  template <int M = N>
  typename std::enable_if<(M == 1), FT &>::type operator[](T i) const {
    return *reinterpret_cast<FT *>(zero + i * strides[0]);
  }

 private:
  char *zero = nullptr;
  long long strides[3] = {0, 0, 0};
};

template <typename T> struct DeferredValue {
  T value;
  explicit DeferredValue(T v) : value(v) {}
  void write(T v) { value = v; }
};
template <typename T, int DIM, typename COORD_T = long long, bool CHECK_BOUNDS = false>
struct DeferredBuffer {};

struct Future {
  bool has_value = false;
  std::vector<char> data;
  template <typename T> static Future from_value(void *, const T &v) {
    Future f;
    f.has_value = true;
    f.data.resize(sizeof(T));
    memcpy(f.data.data(), &v, sizeof(T));
    return f;
  }
  template <typename T> T get_result(bool = false) const {
    assert(has_value && data.size() == sizeof(T));
    T v;
    memcpy(&v, data.data(), sizeof(T));
    return v;
  }
  void get_void_result(bool = false) const {}
};
struct FutureMap {
  void wait_all_results(bool = false) const {}
};
struct Predicate {
  static const Predicate TRUE_PRED;
  bool value = true;
};
struct TaskArgument {
  const void *args = nullptr;
  size_t arglen = 0;
  TaskArgument() {}
  TaskArgument(const void *a, size_t l) : args(a), arglen(l) {}
};
struct ArgumentMap {};

struct RegionRequirement {
  LogicalRegion region, parent;
  LogicalPartition partition;
  bool is_projection = false;
  ProjectionID projection = 0;
  PrivilegeMode privilege = NO_ACCESS;
  CoherenceProperty prop = EXCLUSIVE;
  ReductionOpID redop = 0;
  std::set<FieldID> privilege_fields;
  std::vector<FieldID> instance_fields;
  RegionRequirement() {}
  RegionRequirement(LogicalRegion h, PrivilegeMode p, CoherenceProperty c, LogicalRegion par)
      : region(h), parent(par), privilege(p), prop(c) {}
  RegionRequirement(LogicalPartition lp, ProjectionID proj, PrivilegeMode p,
                    CoherenceProperty c, LogicalRegion par)
      : region(par), parent(par), partition(lp), is_projection(true), projection(proj),
        privilege(p), prop(c) {}
  RegionRequirement(LogicalPartition lp, ProjectionID proj, ReductionOpID op,
                    CoherenceProperty c, LogicalRegion par)
      : region(par), parent(par), partition(lp), is_projection(true), projection(proj),
        privilege(REDUCE), prop(c), redop(op) {}
};

struct Processor {
  enum Kind { NO_KIND, LOC_PROC, TOC_PROC, UTIL_PROC, IO_PROC };
  unsigned long long id = 0;
};
struct Memory { unsigned long long id = 0; };
struct Machine {};

struct Mappable {};
struct Task : public Mappable {
  const void *args = nullptr;
  size_t arglen = 0;
  std::vector<RegionRequirement> regions;
  std::vector<Future> futures;
  const char *get_task_name() const { return "shim task"; }
  long long get_unique_id() const { return 0; }
};
struct Copy : public Mappable {};

namespace Internal { struct TaskContextShim; }
typedef Internal::TaskContextShim *Context;

struct TaskLauncher {};
struct CopyLauncher {};
struct FillLauncher {};
struct InlineLauncher {};
struct IndexCopyLauncher {};
struct IndexFillLauncher {};
struct PredicateLauncher {};
struct FieldAllocator {};
struct LayoutConstraintRegistrar {};
struct SpecializedConstraint {};
struct OrderingConstraint {};
struct FieldConstraint {};
struct LayoutConstraintSet {};
struct MemoryConstraint {};

struct IndexTaskLauncher {
  TaskID task_id = 0;
  TaskArgument global_arg;
  std::vector<RegionRequirement> region_requirements;
  std::vector<Future> futures;
  Future predicate_false_future;
  Predicate predicate;
  IndexTaskLauncher() {}
  template <typename D>
  IndexTaskLauncher(TaskID tid, const D &, const TaskArgument &arg, const ArgumentMap &,
                    const Predicate &pred = Predicate::TRUE_PRED)
      : task_id(tid), global_arg(arg), predicate(pred) {}
  unsigned add_region_requirement(const RegionRequirement &req) {
    region_requirements.push_back(req);
    return region_requirements.size() - 1;
  }
  void add_future(const Future &f) { futures.push_back(f); }
};

struct ISAConstraint {
  unsigned long long isa;
  ISAConstraint(unsigned long long k) : isa(k) {}
};
struct ResourceConstraint {
  ResourceConstraint(ResourceKind, EqualityKind, size_t) {}
};
struct LaunchConstraint {
  LaunchConstraint(LaunchKind, size_t) {}
};
struct ProcessorConstraint {
  ProcessorConstraint(Processor::Kind) {}
};
struct ExecutionConstraintSet {
  template <typename C> ExecutionConstraintSet &add_constraint(const C &) { return *this; }
};
struct TaskLayoutConstraintSet {
  TaskLayoutConstraintSet &add_layout_constraint(unsigned, LayoutConstraintID) { return *this; }
};
struct TaskVariantRegistrar {
  ExecutionConstraintSet execution_constraints;
  TaskLayoutConstraintSet layout_constraints;
  bool leaf_variant = false, inner_variant = false;
  TaskVariantRegistrar(TaskID, bool, const char * = nullptr) {}
  TaskVariantRegistrar(TaskID, const char * = nullptr) {}
  template <typename C> TaskVariantRegistrar &add_constraint(const C &) { return *this; }
};

struct ProjectionFunctor {
  virtual ~ProjectionFunctor() {}
};

struct Logger {
  explicit Logger(const char *) {}
  void info(const char *, ...) {}
  void debug(const char *, ...) {}
  void spew(const char *, ...) {}
  void print(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vfprintf(stderr, fmt, ap);
    va_end(ap);
    fputc('\n', stderr);
  }
  void warning(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vfprintf(stderr, fmt, ap);
    va_end(ap);
    fputc('\n', stderr);
  }
  void error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vfprintf(stderr, fmt, ap);
    va_end(ap);
    fputc('\n', stderr);
  }
};

class Runtime {
 public:
  template <int DIM, typename T>
  DomainT<DIM, T> get_index_space_domain(Context, const IndexSpaceT<DIM, T> &is) {
    DomainT<DIM, T> d;
    d.bounds = is.bounds();
    return d;
  }
  Processor get_executing_processor(Context) { return Processor(); }
  void attach_name(TaskID, const char *, bool = false) {}
  template <typename L> FutureMap execute_index_space(Context, const L &) { return FutureMap(); }
  template <typename L> Future execute_index_space(Context, const L &, ReductionOpID) { return Future(); }
  template <void (*TASK_PTR)(const Task *, const std::vector<PhysicalRegion> &, Context, Runtime *)>
  static VariantID preregister_task_variant(const TaskVariantRegistrar &, const char * = nullptr) {
    return 0;
  }
  template <typename RET, RET (*TASK_PTR)(const Task *, const std::vector<PhysicalRegion> &, Context, Runtime *)>
  static VariantID preregister_task_variant(const TaskVariantRegistrar &, const char * = nullptr) {
    return 0;
  }
};

}  // namespace Legion

#endif
