// The index arrays of a contact graph built on the device (graph.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace msb {

// Index arrays in device memory.
struct GraphIndexArrays {
  std::uint64_t* incidence_offsets;  // cells + 1
  std::uint64_t* incidence;          // one per entry
  std::uint64_t* neighbor_offsets;   // cells + 1; null: no neighbour index
  std::uint64_t* neighbors;
  std::uint64_t neighbor_capacity;
};

// Scratch of a graph build, in 32-bit words, for `entries` incidence entries
// (two per cell contact, one per external contact) over `cell_count` slots.
std::uint64_t graph_scratch_words(std::uint64_t entries, std::uint64_t cell_count);

// Checks every contact as the reference's graph constructors do and counts
// each slot's entries into the scratch.  words (4, device): [0] a key
// (index << 8 | reason) of the lowest contact that fails, or ~0 if none;
// [1] the largest partner id (the cell contacts' second ids); [3] the most
// entries of any slot.  `external` selects msb_external_contact records
// instead of msb_cell_contact.
void launch_validate_contacts(const void* contacts, std::uint64_t count, std::uint64_t cell_count, bool external,
                              unsigned long long* words, std::uint32_t* scratch, cudaStream_t stream);

// After a validation that found no invalid contact (same scratch): per slot,
// its contacts in contact order, and (cell contacts, when
// out.neighbor_offsets is set) its distinct partner ids ascending, with the
// packed id count in words[2].  At most neighbor_capacity ids are written.
void build_graph_index(const void* contacts, std::uint64_t count, std::uint64_t cell_count, bool external,
                       std::uint64_t max_id, std::uint64_t largest_segment, const GraphIndexArrays& out,
                       std::uint32_t* scratch, unsigned long long* words, cudaStream_t stream);

}  // namespace msb
