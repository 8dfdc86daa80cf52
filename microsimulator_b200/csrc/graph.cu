// The index of a contact graph on the device: what the ContactGraph
// constructor (cpp/core/contact_graph.cpp:302-349) and the
// ExternalContactGraph constructor (cpp/core/constraints.cpp:288-307) build
// on the host from a contact list.
//
//  * Validation: every contact is checked as validate_contact does
//    (contact_graph.cpp:217-237, constraints.cpp:126-145), in its order of
//    checks; the lowest failing contact is reported.
//  * Incidence: one entry per (contact, slot it touches), sorted by slot with
//    a stable radix sort, so each slot lists its contacts in contact order,
//    as the constructor's cursor fill does.
//  * Neighbours: the same entries carrying the partner's id, sorted by
//    (slot, partner id) with a chain of stable radix sorts (id words, then
//    slot), then packed by a scan of "first of its (slot, id) run" flags:
//    each slot's distinct partner ids in ascending order, as the
//    constructor's per-slot sort and unique.
//
// Everything is integer work, so the result is the reference's exactly.
#include "graph.h"

#include <bit>
#include <cstdint>

#include "device.cuh"
#include "kernels.h"
#include "../../include/msb200.h"

namespace msb {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ bool finite_vec(msb_vec3 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }

__device__ __forceinline__ bool unit_normal(msb_vec3 n) {
  return fabsf(norm(F3{n.x, n.y, n.z}) - 1.0f) <= 1.0e-4f;
}

// validate_contact(const CellContact&) (contact_graph.cpp:217-237).
__device__ std::uint32_t cell_contact_reason(const msb_cell_contact& c, std::uint64_t cell_count) {
  if (c.first_id == 0 || c.second_id == 0 || c.first_id >= c.second_id) return 1;
  if (c.first_slot >= cell_count || c.second_slot >= cell_count || c.first_slot == c.second_slot) return 2;
  if (c.ordinal > 1) return 3;
  if (!finite_vec(c.point_on_first) || !finite_vec(c.normal) || !isfinite(c.signed_separation) ||
      !isfinite(c.weight) || c.weight <= 0.0f) {
    return 4;
  }
  if (!unit_normal(c.normal)) return 5;
  return 0;
}

// validate_contact(const ExternalContact&) (constraints.cpp:126-145).
__device__ std::uint32_t external_contact_reason(const msb_external_contact& c, std::uint64_t cell_count) {
  if (c.cell_id == 0 || c.constraint_id == 0) return 1;
  if (c.cell_slot >= cell_count) return 2;
  if (c.constraint_kind > MSB_CONSTRAINT_CYLINDER || c.location > MSB_ROD_INTERIOR) return 3;
  if (!finite_vec(c.point_on_cell) || !finite_vec(c.normal) || !isfinite(c.signed_separation) ||
      !isfinite(c.weight) || c.weight <= 0.0f) {
    return 4;
  }
  if (!unit_normal(c.normal)) return 5;
  return 0;
}

template <bool External>
__global__ void validate_kernel(const void* __restrict__ records, std::uint64_t count, std::uint64_t cell_count,
                                unsigned long long* words) {
  unsigned long long largest = 0;
  for (std::uint64_t i = blockIdx.x * std::uint64_t(blockDim.x) + threadIdx.x; i < count;
       i += std::uint64_t(gridDim.x) * blockDim.x) {
    std::uint32_t reason;
    if constexpr (External) {
      reason = external_contact_reason(static_cast<const msb_external_contact*>(records)[i], cell_count);
    } else {
      const msb_cell_contact& c = static_cast<const msb_cell_contact*>(records)[i];
      reason = cell_contact_reason(c, cell_count);
      largest = smax<unsigned long long>(largest, c.second_id);
    }
    if (reason != 0) atomicMin(&words[0], (static_cast<unsigned long long>(i) << 8) | reason);
  }
  if constexpr (!External) {
    for (int o = 16; o > 0; o >>= 1) largest = smax(largest, __shfl_down_sync(0xFFFFFFFFu, largest, o));
    if ((threadIdx.x & 31) == 0 && largest != 0) atomicMax(&words[1], largest);
  }
}

// Entry e of a cell contact list: contact e / 2, its first slot (e even,
// partner = second id) or second slot (e odd, partner = first id).
__device__ __forceinline__ std::uint32_t entry_slot(const msb_cell_contact* c, std::uint32_t e) {
  const msb_cell_contact& r = c[e >> 1];
  return (e & 1u) != 0 ? r.second_slot : r.first_slot;
}
__device__ __forceinline__ std::uint64_t entry_partner(const msb_cell_contact* c, std::uint32_t e) {
  const msb_cell_contact& r = c[e >> 1];
  return (e & 1u) != 0 ? r.first_id : r.second_id;
}

template <bool External>
__global__ void slot_keys_kernel(const void* __restrict__ records, std::uint32_t entries,
                                 std::uint32_t* __restrict__ keys, std::uint32_t* __restrict__ values) {
  for (std::uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < entries; e += gridDim.x * blockDim.x) {
    if constexpr (External) {
      keys[e] = static_cast<const msb_external_contact*>(records)[e].cell_slot;
    } else {
      keys[e] = entry_slot(static_cast<const msb_cell_contact*>(records), e);
    }
    values[e] = e;
  }
}

template <bool External>
__global__ void incidence_indices_kernel(const std::uint32_t* __restrict__ values, std::uint32_t entries,
                                         std::uint64_t* __restrict__ indices) {
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < entries; i += gridDim.x * blockDim.x) {
    indices[i] = External ? values[i] : (values[i] >> 1);
  }
}

// offsets[s] = the first sorted entry whose slot is at least s.
__global__ void offsets_kernel(const std::uint32_t* __restrict__ keys, std::uint32_t entries,
                               std::uint64_t cell_count, std::uint64_t* __restrict__ offsets) {
  for (std::uint64_t s = blockIdx.x * std::uint64_t(blockDim.x) + threadIdx.x; s <= cell_count;
       s += std::uint64_t(gridDim.x) * blockDim.x) {
    std::uint32_t low = 0, high = entries;
    while (low < high) {
      const std::uint32_t mid = low + ((high - low) >> 1);
      if (std::uint64_t(keys[mid]) < s) {
        low = mid + 1;
      } else {
        high = mid;
      }
    }
    offsets[s] = low;
  }
}

// keys[i] = one 32-bit word of entry values[i]'s sort key: 0 = partner id low
// word, 1 = partner id high word, 2 = slot.  values = identity when `fresh`.
__global__ void neighbor_keys_kernel(const msb_cell_contact* __restrict__ contacts, std::uint32_t entries, int word,
                                     bool fresh, std::uint32_t* __restrict__ keys,
                                     std::uint32_t* __restrict__ values) {
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < entries; i += gridDim.x * blockDim.x) {
    if (fresh) values[i] = i;
    const std::uint32_t e = values[i];
    if (word == 2) {
      keys[i] = entry_slot(contacts, e);
    } else {
      const std::uint64_t id = entry_partner(contacts, e);
      keys[i] = word == 0 ? std::uint32_t(id) : std::uint32_t(id >> 32);
    }
  }
}

// flags[i] = 1 where entry i starts a run of equal (slot, partner id).
__global__ void run_flags_kernel(const msb_cell_contact* __restrict__ contacts, const std::uint32_t* __restrict__ keys,
                                 const std::uint32_t* __restrict__ values, std::uint32_t entries,
                                 std::uint32_t* __restrict__ flags) {
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < entries; i += gridDim.x * blockDim.x) {
    std::uint32_t flag = 1;
    if (i > 0 && keys[i] == keys[i - 1] &&
        entry_partner(contacts, values[i]) == entry_partner(contacts, values[i - 1])) {
      flag = 0;
    }
    flags[i] = flag;
  }
}

__global__ void pack_neighbors_kernel(const msb_cell_contact* __restrict__ contacts,
                                      const std::uint32_t* __restrict__ values, const std::uint32_t* __restrict__ flags,
                                      const std::uint32_t* __restrict__ positions, std::uint32_t entries,
                                      std::uint64_t capacity, std::uint64_t* __restrict__ ids) {
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < entries; i += gridDim.x * blockDim.x) {
    if (flags[i] != 0 && positions[i] < capacity) ids[positions[i]] = entry_partner(contacts, values[i]);
  }
}

// Neighbour offsets: the packed position of each slot's first incidence
// entry (both orders group the entries by slot alike); the total at the end.
__global__ void neighbor_offsets_kernel(const std::uint64_t* __restrict__ incidence_offsets,
                                        const std::uint32_t* __restrict__ flags,
                                        const std::uint32_t* __restrict__ positions, std::uint32_t entries,
                                        std::uint64_t cell_count, std::uint64_t* __restrict__ offsets,
                                        unsigned long long* total) {
  const std::uint64_t packed = entries == 0 ? 0 : std::uint64_t(positions[entries - 1]) + flags[entries - 1];
  for (std::uint64_t s = blockIdx.x * std::uint64_t(blockDim.x) + threadIdx.x; s <= cell_count;
       s += std::uint64_t(gridDim.x) * blockDim.x) {
    const std::uint64_t at = incidence_offsets[s];
    offsets[s] = at < entries ? positions[at] : packed;
    if (s == 0) *total = packed;
  }
}

int bits_for(std::uint64_t largest) { return largest == 0 ? 0 : int(std::bit_width(largest)); }

}  // namespace

std::uint64_t graph_scratch_words(std::uint64_t entries) {
  return 4 * entries + sort_temp_words(entries) + scan_temp_words(entries) + 64;
}

void launch_validate_contacts(const void* contacts, std::uint64_t count, std::uint64_t cell_count, bool external,
                              unsigned long long* words, cudaStream_t stream) {
  cudaMemsetAsync(words, 0xFF, sizeof(unsigned long long), stream);
  cudaMemsetAsync(words + 1, 0, sizeof(unsigned long long), stream);
  if (count == 0) return;
  if (external) {
    validate_kernel<true><<<grid_for(count, kThreads), kThreads, 0, stream>>>(contacts, count, cell_count, words);
  } else {
    validate_kernel<false><<<grid_for(count, kThreads), kThreads, 0, stream>>>(contacts, count, cell_count, words);
  }
  count_launch();
}

void build_incidence(const void* contacts, std::uint64_t count, std::uint64_t cell_count, bool external,
                     std::uint64_t* offsets, std::uint64_t* indices, std::uint32_t* scratch, cudaStream_t stream) {
  const std::uint32_t entries = std::uint32_t(external ? count : 2 * count);
  std::uint32_t* keys = scratch;
  std::uint32_t* values = scratch + entries;
  std::uint32_t* temp = scratch + 4ull * entries;
  if (entries > 0) {
    const int grid = grid_for(entries, kThreads);
    if (external) {
      slot_keys_kernel<true><<<grid, kThreads, 0, stream>>>(contacts, entries, keys, values);
    } else {
      slot_keys_kernel<false><<<grid, kThreads, 0, stream>>>(contacts, entries, keys, values);
    }
    count_launch();
    radix_sort_pairs(keys, values, entries, bits_for(cell_count - 1), temp, stream);
    if (external) {
      incidence_indices_kernel<true><<<grid, kThreads, 0, stream>>>(values, entries, indices);
    } else {
      incidence_indices_kernel<false><<<grid, kThreads, 0, stream>>>(values, entries, indices);
    }
    count_launch();
  }
  offsets_kernel<<<grid_for(cell_count + 1, kThreads), kThreads, 0, stream>>>(keys, entries, cell_count, offsets);
  count_launch();
}

void build_neighbors(const void* contacts, std::uint64_t count, std::uint64_t cell_count, std::uint64_t max_id,
                     const std::uint64_t* incidence_offsets, std::uint64_t* offsets, std::uint64_t* ids,
                     std::uint64_t capacity, std::uint32_t* scratch, unsigned long long* total,
                     cudaStream_t stream) {
  const auto* records = static_cast<const msb_cell_contact*>(contacts);
  const std::uint32_t entries = std::uint32_t(2 * count);
  std::uint32_t* keys = scratch;
  std::uint32_t* values = scratch + entries;
  std::uint32_t* flags = scratch + 2ull * entries;
  std::uint32_t* positions = scratch + 3ull * entries;
  std::uint32_t* temp = scratch + 4ull * entries;
  if (entries > 0) {
    const int grid = grid_for(entries, kThreads);
    const int id_bits = bits_for(max_id);
    // Least significant key first: partner id low word, high word, slot.
    neighbor_keys_kernel<<<grid, kThreads, 0, stream>>>(records, entries, 0, true, keys, values);
    count_launch();
    radix_sort_pairs(keys, values, entries, id_bits < 32 ? id_bits : 32, temp, stream);
    if (id_bits > 32) {
      neighbor_keys_kernel<<<grid, kThreads, 0, stream>>>(records, entries, 1, false, keys, values);
      count_launch();
      radix_sort_pairs(keys, values, entries, id_bits - 32, temp, stream);
    }
    neighbor_keys_kernel<<<grid, kThreads, 0, stream>>>(records, entries, 2, false, keys, values);
    count_launch();
    radix_sort_pairs(keys, values, entries, bits_for(cell_count - 1), temp, stream);
    run_flags_kernel<<<grid, kThreads, 0, stream>>>(records, keys, values, entries, flags);
    count_launch();
    exclusive_scan(flags, positions, entries, temp, stream);
    pack_neighbors_kernel<<<grid, kThreads, 0, stream>>>(records, values, flags, positions, entries, capacity, ids);
    count_launch();
  }
  neighbor_offsets_kernel<<<grid_for(cell_count + 1, kThreads), kThreads, 0, stream>>>(
      incidence_offsets, flags, positions, entries, cell_count, offsets, total);
  count_launch();
}

}  // namespace msb
