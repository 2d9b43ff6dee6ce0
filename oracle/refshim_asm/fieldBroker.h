// Oracle (test infrastructure only): minimal stand-ins for the STK mesh and the
// reference's fieldBroker / mesh / domain / zone classes, with exactly the
// members that src/assemble/assembler.h names, so that the reference's own
// assembler<N>::applyCoeff_ compiles and runs on a plain CSR graph here. A node
// entity is its local id; every row is owned.
#pragma once
#include <cstddef>
#include <vector>

#include "types.h"

namespace stk {
namespace topology {
enum rank_t { NODE_RANK = 0, ELEMENT_RANK = 3 };
}
namespace mesh {
struct Entity {
  unsigned id = 0;
};
struct Part {};
using PartVector = std::vector<Part*>;
struct Selector {
  Selector operator&(const Selector&) const { return *this; }
  Selector operator!() const { return *this; }
};
inline Selector selectUnion(const PartVector&) { return {}; }
struct Bucket {
  using size_type = std::size_t;
  std::vector<Entity> e;
  size_type size() const { return e.size(); }
  Entity operator[](size_type i) const { return e[i]; }
};
using BucketVector = std::vector<Bucket*>;
struct MetaData {
  Selector locally_owned_part() const { return {}; }
  Selector universal_part() const { return {}; }
};
struct BulkData {
  BucketVector buckets;
  const BucketVector& get_buckets(topology::rank_t, const Selector&) const { return buckets; }
  label local_id(Entity e) const { return static_cast<label>(e.id); }
  label global_id(Entity e) const { return static_cast<label>(e.id); }
};
}  // namespace mesh
}  // namespace stk

namespace accel {
class zone {
 public:
  const stk::mesh::PartVector& interiorParts() const { return parts_; }

 private:
  stk::mesh::PartVector parts_;
};
class domain {
 public:
  const zone* zonePtr() const { return &zone_; }

 private:
  zone zone_;
};
class mesh {
 public:
  explicit mesh(label n) : n_(n) {}
  const stk::mesh::MetaData& metaDataRef() const { return meta_; }
  const stk::mesh::BulkData& bulkDataRef() const { return bulk_; }
  label nNodes() const { return n_; }

 private:
  label n_;
  stk::mesh::MetaData meta_;
  stk::mesh::BulkData bulk_;
};
class fieldBroker {
 public:
  explicit fieldBroker(label n) : mesh_(n) {}
  const mesh& meshRef() const { return mesh_; }

 private:
  mesh mesh_;
};
}  // namespace accel
