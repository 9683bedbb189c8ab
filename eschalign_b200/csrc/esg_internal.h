// esg_internal.h -- library-internal calls between the translation units of
// libeschalign_b200.so (not part of the C ABI; hidden from the symbol table).
#pragma once
#include <cstddef>
#include <cstdint>

#include "../../include/eschalign_b200.h"

#define ESG_HIDDEN __attribute__((visibility("hidden")))

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
