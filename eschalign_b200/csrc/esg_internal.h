// esg_internal.h -- library-internal calls between the translation units of
// libeschalign_b200.so (not part of the C ABI; hidden from the symbol table).
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/eschalign_b200.h"

#define ESG_HIDDEN __attribute__((visibility("hidden")))

// What the traceback needs of a scorer: the int32 kernel's panel copy
// (1 B codes, references longest first: slot k is reference ridx[k]), the
// host map reference -> slot, the scheme, and where to run.
struct esg_internal_panel {
  const uint8_t* rcodes;
  const uint32_t* roff;
  const uint32_t* rlen;
  const uint32_t* slot_of;  // host array, n_refs entries
  const uint32_t* len_of;   // host array: reference lengths, panel order
  const uint8_t* h_codes;   // host array: the panel's codes (0-4), panel order
  const uint64_t* h_off;    // host array: reference r at h_codes[h_off[r]]
  uint32_t n_refs;
  uint32_t max_ref_len;
  int device;
  int sm_count;
  int mode;
  esg_scoring scoring;
  cudaStream_t stream;
  cudaMemPool_t pool;
};
ESG_HIDDEN void esg_internal_panel_of(esg_scorer* sc, esg_internal_panel* out);

// A submitted batch's reads on the device (NULL codes if not submitted).
ESG_HIDDEN void esg_internal_batch_reads(const esg_batch* b, const uint8_t** codes,
                                         const uint64_t** off, const uint32_t** len,
                                         uint32_t* n_reads, const uint32_t** host_len);

// esg_prepare with read k at reads[k] (reads gathered from several requests,
// no staging copy of their own).
ESG_HIDDEN esg_status esg_internal_prepare_ptrs(esg_scorer* sc, const uint8_t* const* reads,
                                                const uint32_t* len, uint32_t n_reads,
                                                uint32_t flags, esg_batch** out);

// Device bytes the scorer's batch pool holds but no batch uses (reusable
// without a new mapping).
ESG_HIDDEN size_t esg_internal_pool_spare(esg_scorer* sc);

// The scorer's device ordinal and tie capacity.
ESG_HIDDEN int esg_internal_device(const esg_scorer* sc);
ESG_HIDDEN uint32_t esg_internal_tie_capacity(const esg_scorer* sc);
// Bases of the scorer's panel (DP cells per read base and strand).
ESG_HIDDEN uint64_t esg_internal_panel_bases(const esg_scorer* sc);

// esg_align_batch with the CIGAR words into a vector sized to fit, on
// `stream` (NULL: the scorer's stream; the batch must be finished).
ESG_HIDDEN esg_status esg_internal_align_batch(esg_scorer* sc, esg_batch* b,
                                               const esg_align_job* jobs, uint32_t n_jobs,
                                               esg_alignment* out, std::vector<uint32_t>* ops,
                                               cudaStream_t stream = nullptr);

