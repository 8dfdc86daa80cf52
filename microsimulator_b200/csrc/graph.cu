// The index of a contact graph on the device: what the ContactGraph
// constructor (cpp/core/contact_graph.cpp:302-349) and the
// ExternalContactGraph constructor (cpp/core/constraints.cpp:288-307) build
// on the host from a contact list.
//
//  * Validation: every contact is checked as validate_contact does
//    (contact_graph.cpp:217-237, constraints.cpp:126-145), in its order of
//    checks; the lowest failing contact is reported.
//  * Segments: one entry per (contact, slot it touches).  The validation
//    pass counts each slot's entries; a scan gives the slots' offsets.
//  * Short segments (every slot with at most kSegmentLimit entries, the case
//    of capsule colonies): the entries are scattered to their slot's range
//    in any order, then one thread per slot sorts its range by contact index
//    (the constructor's cursor fill lists a slot's contacts in contact
//    order), gathers the partners' ids, sorts them and drops repeats (the
//    constructor's per-slot sort and unique); a scan of the distinct counts
//    places each slot's ids.
//  * Any segment longer: the entries are sorted by slot with a stable radix
//    sort (incidence), and by (slot, partner id) with a chain of stable
//    radix sorts (id words, then slot), packed by a scan of "first of its
//    (slot, id) run" flags.
//
// Everything is integer work, so either way the result is the reference's
// exactly.
#include "graph.h"

#include <bit>
#include <cstdint>

#include "device.cuh"
#include "kernels.h"
#include "../../include/msb200.h"

namespace msb {
namespace {

constexpr int kThreads = 256;
// The longest segment the per-slot sort takes; longer ones take the radix path.
constexpr std::uint32_t kSegmentLimit = 64;

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

// Checks each contact and counts the entries of each slot (valid contacts
// only, so that every counted slot is in range).
template <bool External>
__global__ void validate_kernel(const void* __restrict__ records, std::uint64_t count, std::uint64_t cell_count,
                                unsigned long long* words, std::uint32_t* __restrict__ counts) {
  unsigned long long largest = 0;
  for (std::uint64_t i = blockIdx.x * std::uint64_t(blockDim.x) + threadIdx.x; i < count;
       i += std::uint64_t(gridDim.x) * blockDim.x) {
    std::uint32_t reason;
    if constexpr (External) {
      const msb_external_contact& c = static_cast<const msb_external_contact*>(records)[i];
      reason = external_contact_reason(c, cell_count);
      if (reason == 0) atomicAdd(&counts[c.cell_slot], 1u);
    } else {
      const msb_cell_contact& c = static_cast<const msb_cell_contact*>(records)[i];
      reason = cell_contact_reason(c, cell_count);
      largest = smax<unsigned long long>(largest, c.second_id);
      if (reason == 0) {
        atomicAdd(&counts[c.first_slot], 1u);
        atomicAdd(&counts[c.second_slot], 1u);
      }
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

// ---- short segments

// The largest segment (atomic max into *largest).
__global__ void largest_count_kernel(const std::uint32_t* __restrict__ counts, std::uint64_t cell_count,
                                     unsigned long long* largest) {
  std::uint32_t m = 0;
  for (std::uint64_t s = blockIdx.x * std::uint64_t(blockDim.x) + threadIdx.x; s < cell_count;
       s += std::uint64_t(gridDim.x) * blockDim.x) {
    m = smax(m, counts[s]);
  }
  for (int o = 16; o > 0; o >>= 1) m = smax(m, __shfl_down_sync(0xFFFFFFFFu, m, o));
  if ((threadIdx.x & 31) == 0 && m != 0) atomicMax(largest, static_cast<unsigned long long>(m));
}

// Each entry to a free place in its slot's range (counts run back to zero):
// its contact index and, for a neighbour index, the partner's id beside it
// (read here from the same 32-byte sector as the slots).
template <bool External, bool Neighbors>
__global__ void scatter_entries_kernel(const void* __restrict__ records, std::uint64_t count,
                                       const std::uint32_t* __restrict__ starts, std::uint32_t* __restrict__ counts,
                                       std::uint32_t* __restrict__ entries, std::uint64_t* __restrict__ partners) {
  for (std::uint64_t i = blockIdx.x * std::uint64_t(blockDim.x) + threadIdx.x; i < count;
       i += std::uint64_t(gridDim.x) * blockDim.x) {
    if constexpr (External) {
      const std::uint32_t slot = static_cast<const msb_external_contact*>(records)[i].cell_slot;
      entries[starts[slot] + atomicSub(&counts[slot], 1u) - 1u] = std::uint32_t(i);
    } else {
      const msb_cell_contact& c = static_cast<const msb_cell_contact*>(records)[i];
      const std::uint32_t a = starts[c.first_slot] + atomicSub(&counts[c.first_slot], 1u) - 1u;
      const std::uint32_t b = starts[c.second_slot] + atomicSub(&counts[c.second_slot], 1u) - 1u;
      entries[a] = std::uint32_t(i);
      entries[b] = std::uint32_t(i);
      if constexpr (Neighbors) {
        partners[a] = c.second_id;
        partners[b] = c.first_id;
      }
    }
  }
}

template <typename T>
__device__ __forceinline__ void insertion_sort(T* v, std::uint32_t n) {
  for (std::uint32_t i = 1; i < n; ++i) {
    const T x = v[i];
    std::uint32_t j = i;
    while (j > 0 && v[j - 1] > x) {
      v[j] = v[j - 1];
      --j;
    }
    v[j] = x;
  }
}

// Bitonic sorting network over N registers (indices fixed at compile time,
// so the array stays in registers).
template <int N, typename T>
__device__ __forceinline__ void bitonic_sort(T (&v)[N]) {
#pragma unroll
  for (int k = 2; k <= N; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
#pragma unroll
      for (int i = 0; i < N; ++i) {
        const int l = i ^ j;
        if (l > i) {
          const T a = v[i], b = v[l];
          const bool swap = (i & k) == 0 ? (a > b) : (a < b);
          v[i] = swap ? b : a;
          v[l] = swap ? a : b;
        }
      }
    }
  }
}

constexpr int kRegisterSegment = 16;

// One slot's segment [begin, begin + k): its contact indices sorted into
// `incidence`; with neighbours, its partner ids sorted, made distinct and
// written at the front of the same range of `distinct`.  Returns the
// distinct count.
template <bool Neighbors>
__device__ __forceinline__ std::uint32_t register_segment(const std::uint32_t* __restrict__ entries,
                                                          const std::uint64_t* __restrict__ partners,
                                                          std::uint32_t begin, std::uint32_t k,
                                                          std::uint64_t* __restrict__ incidence,
                                                          std::uint64_t* __restrict__ distinct) {
  std::uint32_t e[kRegisterSegment];
#pragma unroll
  for (int j = 0; j < kRegisterSegment; ++j) e[j] = std::uint32_t(j) < k ? entries[begin + j] : 0xFFFFFFFFu;
  bitonic_sort(e);
#pragma unroll
  for (int j = 0; j < kRegisterSegment; ++j) {
    if (std::uint32_t(j) < k) incidence[begin + j] = e[j];
  }
  if constexpr (!Neighbors) {
    return 0;
  } else {
    std::uint64_t p[kRegisterSegment];
#pragma unroll
    for (int j = 0; j < kRegisterSegment; ++j) p[j] = std::uint32_t(j) < k ? partners[begin + j] : ~0ull;
    bitonic_sort(p);
    std::uint32_t u = 0;
#pragma unroll
    for (int j = 0; j < kRegisterSegment; ++j) {
      if (std::uint32_t(j) < k && (j == 0 || p[j] != p[j - 1])) distinct[begin + u++] = p[j];
    }
    return u;
  }
}

// The same for segments of up to kSegmentLimit entries, in local memory.
template <bool Neighbors>
__device__ __noinline__ std::uint32_t local_segment(const std::uint32_t* __restrict__ entries,
                                                    const std::uint64_t* __restrict__ partners, std::uint32_t begin,
                                                    std::uint32_t k, std::uint64_t* __restrict__ incidence,
                                                    std::uint64_t* __restrict__ distinct) {
  std::uint32_t e[kSegmentLimit];
  for (std::uint32_t j = 0; j < k; ++j) e[j] = entries[begin + j];
  insertion_sort(e, k);
  for (std::uint32_t j = 0; j < k; ++j) incidence[begin + j] = e[j];
  if constexpr (!Neighbors) {
    return 0;
  } else {
    std::uint64_t p[kSegmentLimit];
    for (std::uint32_t j = 0; j < k; ++j) p[j] = partners[begin + j];
    insertion_sort(p, k);
    std::uint32_t u = 0;
    for (std::uint32_t j = 0; j < k; ++j) {
      if (j == 0 || p[j] != p[j - 1]) distinct[begin + u++] = p[j];
    }
    return u;
  }
}

// One thread per slot: its contacts in contact order (the incidence) and,
// with neighbours, its distinct partner ids with their count.
template <bool Neighbors>
__global__ void __launch_bounds__(kThreads) segment_kernel(
    const std::uint32_t* __restrict__ starts, const std::uint32_t* __restrict__ entries,
    const std::uint64_t* __restrict__ partners, std::uint64_t cell_count,
    std::uint64_t* __restrict__ incidence_offsets, std::uint64_t* __restrict__ incidence,
    std::uint64_t* __restrict__ distinct, std::uint32_t* __restrict__ distinct_counts) {
  for (std::uint64_t s = blockIdx.x * std::uint64_t(blockDim.x) + threadIdx.x; s <= cell_count;
       s += std::uint64_t(gridDim.x) * blockDim.x) {
    const std::uint32_t begin = starts[s];
    incidence_offsets[s] = begin;
    if (s == cell_count) {
      if constexpr (Neighbors) distinct_counts[s] = 0;
      continue;
    }
    const std::uint32_t k = starts[s + 1] - begin;
    const std::uint32_t u = k <= std::uint32_t(kRegisterSegment)
                                ? register_segment<Neighbors>(entries, partners, begin, k, incidence, distinct)
                                : local_segment<Neighbors>(entries, partners, begin, k, incidence, distinct);
    if constexpr (Neighbors) distinct_counts[s] = u;
  }
}

// Neighbour offsets and ids from each slot's distinct ids and their places.
__global__ void compact_neighbors_kernel(const std::uint32_t* __restrict__ starts,
                                         const std::uint32_t* __restrict__ distinct_counts,
                                         const std::uint32_t* __restrict__ places,
                                         const std::uint64_t* __restrict__ distinct, std::uint64_t cell_count,
                                         std::uint64_t capacity, std::uint64_t* __restrict__ offsets,
                                         std::uint64_t* __restrict__ ids, unsigned long long* total) {
  for (std::uint64_t s = blockIdx.x * std::uint64_t(blockDim.x) + threadIdx.x; s <= cell_count;
       s += std::uint64_t(gridDim.x) * blockDim.x) {
    const std::uint64_t place = places[s];
    offsets[s] = place;
    if (s == cell_count) {
      *total = place;
      continue;
    }
    const std::uint32_t from = starts[s];
    for (std::uint32_t j = 0; j < distinct_counts[s]; ++j) {
      if (place + j < capacity) ids[place + j] = distinct[from + j];
    }
  }
}

}  // namespace

namespace {

// Scratch layout (32-bit words): counts (cells + 1) first, then either path.
struct Layout {
  std::uint64_t slots;    // cells + 1
  std::uint64_t entries;  // incidence entries
  std::uint64_t short_words() const {
    // distinct ids and partners (u64 each), starts, distinct counts, places
    // (slots each), entries, the scan's temporary
    return 4 * entries + 3 * slots + entries + scan_temp_words(slots) + 8;
  }
  std::uint64_t radix_words() const { return 4 * entries + sort_temp_words(entries) + scan_temp_words(entries); }
};

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

}  // namespace

std::uint64_t graph_scratch_words(std::uint64_t entries, std::uint64_t cell_count) {
  const Layout l{cell_count + 1, entries};
  const std::uint64_t rest = l.short_words() > l.radix_words() ? l.short_words() : l.radix_words();
  return ((l.slots + 1) & ~1ull) + rest + 64;
}

void launch_validate_contacts(const void* contacts, std::uint64_t count, std::uint64_t cell_count, bool external,
                              unsigned long long* words, std::uint32_t* scratch, cudaStream_t stream) {
  cudaMemsetAsync(words, 0xFF, sizeof(unsigned long long), stream);
  cudaMemsetAsync(words + 1, 0, 3 * sizeof(unsigned long long), stream);
  cudaMemsetAsync(scratch, 0, (cell_count + 1) * sizeof(std::uint32_t), stream);
  if (count == 0) return;
  if (external) {
    validate_kernel<true><<<grid_for(count, kThreads), kThreads, 0, stream>>>(contacts, count, cell_count, words,
                                                                             scratch);
  } else {
    validate_kernel<false><<<grid_for(count, kThreads), kThreads, 0, stream>>>(contacts, count, cell_count, words,
                                                                              scratch);
  }
  count_launch();
  largest_count_kernel<<<grid_for(cell_count, kThreads), kThreads, 0, stream>>>(scratch, cell_count, words + 3);
  count_launch();
}

void build_graph_index(const void* contacts, std::uint64_t count, std::uint64_t cell_count, bool external,
                       std::uint64_t max_id, std::uint64_t largest_segment, const GraphIndexArrays& out,
                       std::uint32_t* scratch, unsigned long long* words, cudaStream_t stream) {
  const Layout l{cell_count + 1, external ? count : 2 * count};
  std::uint32_t* counts = scratch;
  std::uint32_t* rest = scratch + ((l.slots + 1) & ~1ull);
  const bool neighbors = !external && out.neighbor_offsets != nullptr;
  if (largest_segment > kSegmentLimit) {
    build_incidence(contacts, count, cell_count, external, out.incidence_offsets, out.incidence, rest, stream);
    if (neighbors) {
      build_neighbors(contacts, count, cell_count, max_id, out.incidence_offsets, out.neighbor_offsets,
                      out.neighbors, out.neighbor_capacity, rest, words + 2, stream);
    }
    return;
  }
  // Short segments.  rest: distinct ids and partners (u64, first for
  // alignment), starts, distinct counts, places, entries, scan temporary.
  auto* distinct = reinterpret_cast<std::uint64_t*>(rest);
  std::uint64_t* partners = distinct + l.entries;
  std::uint32_t* starts = rest + 4 * l.entries;
  std::uint32_t* distinct_counts = starts + l.slots;
  std::uint32_t* places = distinct_counts + l.slots;
  std::uint32_t* entries = places + l.slots;
  std::uint32_t* temp = entries + l.entries;
  exclusive_scan(counts, starts, l.slots, temp, stream);
  const int grid = grid_for(count, kThreads);
  if (count > 0) {
    if (external) {
      scatter_entries_kernel<true, false><<<grid, kThreads, 0, stream>>>(contacts, count, starts, counts, entries,
                                                                        nullptr);
    } else if (neighbors) {
      scatter_entries_kernel<false, true><<<grid, kThreads, 0, stream>>>(contacts, count, starts, counts, entries,
                                                                        partners);
    } else {
      scatter_entries_kernel<false, false><<<grid, kThreads, 0, stream>>>(contacts, count, starts, counts, entries,
                                                                         nullptr);
    }
    count_launch();
  }
  const int slot_grid = grid_for(l.slots, kThreads);
  if (neighbors) {
    segment_kernel<true><<<slot_grid, kThreads, 0, stream>>>(starts, entries, partners, cell_count,
                                                             out.incidence_offsets, out.incidence, distinct,
                                                             distinct_counts);
    count_launch();
    exclusive_scan(distinct_counts, places, l.slots, temp, stream);
    compact_neighbors_kernel<<<slot_grid, kThreads, 0, stream>>>(starts, distinct_counts, places, distinct,
                                                                 cell_count, out.neighbor_capacity,
                                                                 out.neighbor_offsets, out.neighbors, words + 2);
    count_launch();
  } else {
    segment_kernel<false><<<slot_grid, kThreads, 0, stream>>>(starts, entries, nullptr, cell_count,
                                                              out.incidence_offsets, out.incidence, nullptr,
                                                              nullptr);
    count_launch();
  }
}

}  // namespace msb
