// Host side of the global array queue: the sorted-array maintenance shared by the PHOLD
// engine (kind GPQ_QUEUE_GAQ) and the GAQ queue object.
#pragma once

#include <cuda_runtime.h>

#include <utility>
#include <vector>

#include "gpq.h"

struct PholdDev;

namespace gpq {

// Stable sort of n items by timestamp bits with the project's LSD radix sort.
// Keys must lie in [kmin, kmax]; only ceil(log2(kmax - kmin + 1) / 8) passes run.  The
// items start in `a`; `b` is a second buffer of n items; `hist` holds
// radix_hist_words(n) words.  *sorted receives a or b, whichever holds the result.  A tile
// whose TMA staging did not complete records GPQ_ERR_TIMEOUT in the device word *err.
gpq_status radix_sort_by_ts(gpq_item* a, gpq_item* b, uint32_t n, uint32_t kmin, uint32_t kmax, uint32_t* hist,
                            gpq_item** sorted, uint32_t* err, cudaStream_t st);
size_t radix_hist_words(uint32_t n);

// Exclusive scan of n words from `in` into `out` (in == out allowed) over the whole GPU;
// `scratch` holds scan_scratch_words(n) words.
gpq_status scan_exclusive(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* scratch, cudaStream_t st);
size_t scan_scratch_words(uint64_t n);

// Merge two arrays sorted by timestamp bits into `out` (A first on equal timestamps):
// merge-path splits in one pass (into `split`, merge_split_words(na + nb) words), then one
// CTA per output tile with its inputs staged by TMA; errors as for radix_sort_by_ts.
gpq_status merge_by_ts(const gpq_item* A, uint32_t na, const gpq_item* B, uint32_t nb, gpq_item* out, uint32_t* split,
                       uint32_t* err, cudaStream_t st);
size_t merge_split_words(uint32_t total);

struct GaqEngine;
gpq_status gaq_engine_create(const gpq_phold_config& c, GaqEngine** out);
void gaq_engine_destroy(GaqEngine* g);
gpq_status gaq_engine_populate(GaqEngine* g, const PholdDev& d, const gpq_item* dev_src, cudaStream_t st);
// Runs up to nsteps windows (0 = until done); *done = 1 when the minimum reached the end
// time; *windows += windows executed.  Returns the device error, if any.
gpq_status gaq_engine_run(GaqEngine* g, const PholdDev& d, uint32_t nsteps, int* done, uint64_t* windows,
                          cudaStream_t st);
// committed, pending, pending_csum, digest, pending_min (as float bits)
gpq_status gaq_engine_finalize(GaqEngine* g, const PholdDev& d, uint64_t out[4], uint32_t* pmin, cudaStream_t st);
uint32_t gaq_engine_launches_per_window();
// The engine's state for snapshots: its device buffers and host words (pointer, bytes).
void gaq_engine_state(GaqEngine* g, std::vector<std::pair<void*, size_t>>* dev,
                      std::vector<std::pair<void*, size_t>>* host);

}  // namespace gpq
