/*
 * Stand-in for Legion's default_mapper.h (TEST INFRASTRUCTURE ONLY): the
 * reference's snap.h declares a DefaultMapper subclass, so the base class and
 * the nested type names it mentions must exist.  No mapping happens.
 */
#ifndef SNAP_REFSHIM_DEFAULT_MAPPER_H
#define SNAP_REFSHIM_DEFAULT_MAPPER_H

#include "legion.h"

namespace Legion {
namespace Mapping {

struct MapperRuntime {};
struct MapperContextShim;
typedef MapperContextShim *MapperContext;
struct PhysicalInstance {
  bool operator<(const PhysicalInstance &) const { return false; }
};

class DefaultMapper {
 public:
  enum DefaultTunables {
    DEFAULT_TUNABLE_NODE_COUNT = 0,
    DEFAULT_TUNABLE_LOCAL_CPUS = 1,
    DEFAULT_TUNABLE_LOCAL_GPUS = 2,
    DEFAULT_TUNABLE_LOCAL_IOS = 3,
    DEFAULT_TUNABLE_LOCAL_OMPS = 4,
    DEFAULT_TUNABLE_LOCAL_PYS = 5,
    DEFAULT_TUNABLE_GLOBAL_CPUS = 6,
    DEFAULT_TUNABLE_GLOBAL_GPUS = 7,
    DEFAULT_TUNABLE_GLOBAL_IOS = 8,
    DEFAULT_TUNABLE_GLOBAL_OMPS = 9,
    DEFAULT_TUNABLE_GLOBAL_PYS = 10,
    DEFAULT_TUNABLE_LAST = 11,
  };
  struct SelectTunableInput {};
  struct SelectTunableOutput {};
  struct SpeculativeOutput {};
  struct MapCopyInput {};
  struct MapCopyOutput {};
  struct TaskOptions {};
  struct SliceTaskInput {};
  struct SliceTaskOutput {};
  struct MapTaskInput {};
  struct MapTaskOutput {};
  DefaultMapper(MapperRuntime *, Machine, Processor, const char *) {}
  virtual ~DefaultMapper() {}
};

}  // namespace Mapping
}  // namespace Legion

#endif
