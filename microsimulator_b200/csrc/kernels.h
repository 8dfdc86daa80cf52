// Launchers of the device kernels, callable from the C++ host engine.
//
// Everything here takes device pointers and a stream and returns without
// synchronizing.  Layouts in HBM (by cell slot unless stated):
//   pos_len  float4  centre x, y, z and cylinder length
//   dir_rad  float4  unit axis x, y, z and radius
//   ids      u64     stable cell identifiers
// A contact ("touch") is a 64-byte record shared by the pair and wall paths.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace msb {

constexpr std::uint32_t kInvalidSlot = 0xFFFFFFFFu;
constexpr int kSmCount = 148;

// Device status word: the first failure wins.
enum DeviceStatus : std::uint32_t {
  kStatusOk = 0,
  kStatusIndex = 1,      // an identifier or index was invalid; the access was skipped
  kStatusCapacity = 2,   // more items than the buffer sized for them
  kStatusGeometry = 3,   // a geometry value was invalid (non-finite, negative, unnormalized)
  kStatusIterations = 4  // a bounded device loop reached its cap
};

// Grid sizes: a multiple of the SM count, at most `per_sm` blocks per SM.
inline int grid_for(std::uint64_t items, int threads, int per_sm = 8) {
  const std::uint64_t blocks = (items + threads - 1) / threads;
  const std::uint64_t cap = std::uint64_t(kSmCount) * per_sm;
  return int(blocks < 1 ? 1 : (blocks > cap ? cap : blocks));
}

void count_launch(int launches = 1);

struct GeometryView {
  const float4* pos_len;
  const float4* dir_rad;
  const std::uint64_t* ids;
  std::uint32_t count;
  // For a batch of independent colonies, the colony of each slot: the grid
  // gives every colony its own range of z boxes, so that no two colonies'
  // cells are ever candidates of one another.  Null for one system.
  const std::uint32_t* colony = nullptr;
  // Colonies still searched in a batch's refinement round (null: all).
  const std::uint32_t* colony_active = nullptr;
};

// One contact of a cell with a cell (s2 valid) or with a constraint (s2 =
// kInvalidSlot).  `partner` is the second slot or the constraint id; `tag`
// is the ordinal of a pair contact or the rod location of a wall contact;
// `kind` is the constraint kind of a wall contact.
struct alignas(16) Touch {
  std::uint32_t s1;
  std::uint32_t s2;
  std::uint64_t partner;
  float point[3];
  float normal[3];
  float sep;
  float weight;
  std::uint32_t tag;
  std::uint32_t kind;
  std::uint32_t pad[2];
};
static_assert(sizeof(Touch) == 64, "touch record is 64 bytes");

// A constraint on the device, sorted by id (layout of msb_constraint).
struct DeviceConstraint {
  std::uint64_t id;
  std::uint32_t kind;
  std::uint32_t region;
  float a[3];
  float b[3];
  float radius;
  float half_height;
  float coefficient;
  std::uint32_t reserved;
};

// The uniform grid of one contact search, written on the device.
struct GridParams {
  double low[3];
  double inv_width[3];
  std::uint64_t dims[3];
  std::uint32_t hashed;   // 0: dense boxes (x * dy + y) * dz + z; 1: hashed table
  std::uint32_t buckets;  // buckets in use
  std::uint32_t status;
  std::uint32_t colony_stride;  // z boxes per colony of a batch (0: one system)
};

// ---- primitives.cu
std::uint64_t scan_temp_words(std::uint64_t n);
void exclusive_scan(const std::uint32_t* in, std::uint32_t* out, std::uint64_t n, std::uint32_t* temp,
                    cudaStream_t stream);
std::uint64_t sort_temp_words(std::uint64_t n);
void radix_sort_pairs(std::uint32_t* keys, std::uint32_t* values, std::uint64_t n, int key_bits,
                      std::uint32_t* temp, cudaStream_t stream);
void iota(std::uint32_t* out, std::uint64_t n, cudaStream_t stream);

// ---- contacts.cu: cell list, broad and narrow phase, wall contacts
struct ContactSearchParams {
  float margin;
  float sine_threshold;
  float epsilon;
  // >= 0: the narrow phase first keeps only the pairs whose padded boxes
  // at this margin overlap (candidates taken from a wider or earlier search).
  float box_margin = -1.0f;
};

// Buckets to allocate for `cells` cells (dense limit or hashed table) + 1.
std::uint64_t grid_bucket_capacity(std::uint32_t cells);
std::uint32_t bound_partials(std::uint32_t cells);

// Padded FP64 boxes (6 doubles per cell) and the grid over them.
void launch_cell_bounds(GeometryView g, float margin, double* bounds, double* partials,
                        cudaStream_t stream);
// Boxes are box_scale (>= 1) times the widest padded capsule: any scale finds
// the same pairs, and the best one depends on the density.
void launch_grid_setup(const double* partials, std::uint32_t partial_count, std::uint32_t cells,
                       std::uint64_t bucket_capacity, GridParams* grid, cudaStream_t stream, float box_scale = 1.0f,
                       std::uint32_t colonies = 0);
void launch_bin_cells(GeometryView g, const double* bounds, const GridParams* grid,
                      std::uint32_t* cell_bucket, std::int64_t* cell_coords, std::uint32_t* bucket_counts,
                      cudaStream_t stream);
// Cells in bucket order: FP32 outward-rounded boxes (slot in lo.w) and ids.
void launch_scatter_cells(GeometryView g, const double* bounds, const std::uint32_t* cell_bucket,
                          const std::uint32_t* bucket_starts, std::uint32_t* bucket_fill, float4* sorted_lo,
                          float4* sorted_hi, std::uint64_t* sorted_id, cudaStream_t stream);
// Candidate pairs: per cell, partners of higher id whose boxes overlap.
// Counts go to counts[rank[cell]]; fill writes (first, second) slot pairs in
// (first id, second id) order at offsets[rank[cell]].
void launch_broad_phase(GeometryView g, const double* bounds, const GridParams* grid,
                        const std::uint32_t* bucket_starts, const float4* sorted_lo, const float4* sorted_hi,
                        const std::uint64_t* sorted_id, const std::int64_t* cell_coords,
                        const std::uint32_t* rank, std::uint32_t* counts, const std::uint32_t* offsets,
                        uint2* pairs, std::uint32_t* status, cudaStream_t stream, std::uint32_t* slab = nullptr);
// Partners a cell's slab row holds at most; the broad phase's single-pass
// form keeps them there (slab: cells x kSlabPartners words, by id rank).
constexpr std::uint32_t kSlabPartners = 32;
// Copies the slab rows of cells with at most kSlabPartners partners into
// the pair list (counts and offsets by id rank; order: slots by id rank).
void launch_compact_slab(std::uint32_t n, const std::uint32_t* counts, const std::uint32_t* offsets,
                         const std::uint32_t* order, const std::uint32_t* slab, uint2* pairs, cudaStream_t stream);
// Partial re-search of an overlap re-check (contacts.cu): the cells that
// moved further than the kept candidates allow (`allowance` = the kept
// padding margin less 1e-6: fast when 2 * moved > allowance), listed in
// `list` with *count (zeroed by the caller); the fast cells' partners on the
// current geometry's grid that the kept list lacks (its pairs by first cell
// at kept_offsets[rank[cell]]; count pass with pairs null, over `cap` list
// places, then fill); and the kept list merged with
// them in (first id, second id) order into `merged`.
void launch_fast_cells(GeometryView from, GeometryView to, double allowance, std::uint32_t* fast, std::uint32_t* list,
                       std::uint32_t* count, cudaStream_t stream);
void launch_fast_partners(GeometryView g, const double* bounds, const GridParams* grid,
                          const std::uint32_t* bucket_starts, const float4* sorted_lo, const float4* sorted_hi,
                          const std::uint64_t* sorted_id, const std::int64_t* cell_coords, const std::uint32_t* fast,
                          const std::uint32_t* list, const std::uint32_t* fast_count, std::uint32_t cap,
                          const uint2* kept, const std::uint32_t* kept_offsets, const std::uint32_t* rank,
                          std::uint32_t* counts, const std::uint32_t* offsets, uint2* pairs, cudaStream_t stream);
void launch_merge_fast_pairs(const uint2* fast_pairs, std::uint32_t fast_pair_count, uint2* sorted_fast,
                             const uint2* kept, std::uint32_t kept_count, const std::uint64_t* ids,
                             std::uint32_t* shift, std::uint32_t* shift_scan, std::uint32_t* temp, uint2* merged,
                             cudaStream_t stream);
// Narrow phase: per candidate, the number of contacts below the margin
// (count pass, `touches` null) or the contacts themselves at offsets[pair].
void launch_narrow_phase(GeometryView g, const uint2* pairs, std::uint64_t pair_count,
                         ContactSearchParams p, std::uint32_t* counts, const std::uint32_t* offsets,
                         Touch* touches, cudaStream_t stream, std::uint32_t* status = nullptr);
// Wall contacts of every cell: counts[rank[cell]] (count pass) or the
// contacts at touch_base + offsets[rank[cell]] (fill pass).  every_face
// selects find_external_contact_faces over find_external_contacts.
void launch_wall_contacts(GeometryView g, const DeviceConstraint* constraints,
                          std::uint32_t constraint_count, float margin, float epsilon,
                          std::uint32_t every_face, const std::uint32_t* rank, std::uint32_t* counts,
                          const std::uint32_t* offsets, Touch* touches, cudaStream_t stream);
// Touch records to the API's contact records.
void launch_touches_to_cell_contacts(const Touch* touches, std::uint64_t count,
                                     const std::uint64_t* ids, void* out, cudaStream_t stream);
void launch_touches_to_external_contacts(const Touch* touches, std::uint64_t count,
                                         const std::uint64_t* ids, void* out, cudaStream_t stream);

// Id order: `order` receives the slots sorted by id, `rank` the inverse.
// `keys_scratch` holds `cells` words.
void launch_id_low_words(const std::uint64_t* ids, std::uint32_t cells, int shift, const std::uint32_t* order,
                         std::uint32_t* keys, cudaStream_t stream);
void launch_invert_permutation(const std::uint32_t* order, std::uint32_t cells, std::uint32_t* rank,
                               cudaStream_t stream);
void launch_check_unique_ids(const std::uint64_t* ids, const std::uint32_t* order, std::uint32_t cells,
                             std::uint32_t* status, cudaStream_t stream);
void launch_max_u64(const std::uint64_t* values, std::uint32_t count, std::uint64_t* result,
                    cudaStream_t stream);

}  // namespace msb
