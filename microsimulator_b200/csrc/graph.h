// The index arrays of a contact graph built on the device (graph.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace msb {

// Scratch of a graph build, in 32-bit words, for `entries` incidence entries
// (two per cell contact, one per external contact).
std::uint64_t graph_scratch_words(std::uint64_t entries);

// Checks every contact as the reference's graph constructors do.  words[0]
// receives a key (index << 8 | reason) of the lowest contact that fails, or
// ~0 if none; words[1] the largest partner id (the cell contacts' second ids).
// `external` selects msb_external_contact records instead of msb_cell_contact.
void launch_validate_contacts(const void* contacts, std::uint64_t count, std::uint64_t cell_count, bool external,
                              unsigned long long* words, cudaStream_t stream);

// Per slot, the contacts that touch it in contact order: offsets
// (cell_count + 1) and the packed contact indices (64-bit outputs, device
// memory).  `scratch` holds graph_scratch_words(entries) words, and leaves
// the (slot, entry) pairs sorted by slot in its first 2 * entries words.
void build_incidence(const void* contacts, std::uint64_t count, std::uint64_t cell_count, bool external,
                     std::uint64_t* offsets, std::uint64_t* indices, std::uint32_t* scratch, cudaStream_t stream);

// Per slot, the distinct partner ids of its contacts in ascending order:
// offsets (cell_count + 1) and up to `capacity` packed ids.  Needs the
// incidence offsets of build_incidence.  Returns the packed count through
// `total` (device word).
void build_neighbors(const void* contacts, std::uint64_t count, std::uint64_t cell_count, std::uint64_t max_id,
                     const std::uint64_t* incidence_offsets, std::uint64_t* offsets, std::uint64_t* ids,
                     std::uint64_t capacity, std::uint32_t* scratch, unsigned long long* total,
                     cudaStream_t stream);

}  // namespace msb
