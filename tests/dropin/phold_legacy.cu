// TEST INFRASTRUCTURE: the drop-in PHOLD model driven through the reference's host queue
// names (include/gpq/legacy.h: queue_init, queue_post_init, queue_get_min_ts, queue_pre,
// queue_post, get_dequeue_count, queue_finish), in the order of the reference's des_run
// loop (src/des.cu:179-214) and model_init (src/phold.cu:124-163).
#include <cuda_runtime.h>

#include <vector>

#include "gpq.h"
#include "gpq/legacy.h"

#include "phold_handler.cuh"

extern "C" int dropin_phold_run_legacy(const gpq_phold_config* cfg, uint32_t* count, unsigned long long* csum,
                                       unsigned long long* ohash, unsigned long long* steps_out,
                                       unsigned long long* committed_out) {
  const uint32_t L = cfg->num_lps;
  gpq_queue_config qc = {};
  qc.kind = cfg->queue_kind;
  qc.num_lps = L;
  qc.capacity = cfg->capacity ? cfg->capacity : 256;
  qc.insert_capacity = cfg->insert_capacity ? cfg->insert_capacity : 64;
  int st = gpq_legacy_configure(&qc, cfg->lookahead, cfg->end_time);
  if (st) return st;
  queue_init();
  if ((st = gpq_legacy_status()) != GPQ_OK) return st;
  // model_init: the initial events in chunks of one event per LP, each followed by queue_post_init
  std::vector<gpq_item> all((size_t)L * cfg->events_per_lp), chunk(L);
  st = gpq_phold_initial_events(cfg, all.data(), all.size());
  for (uint32_t k = 0; !st && k < cfg->events_per_lp; ++k) {
    queue_pre();
    for (uint32_t lp = 0; lp < L; ++lp) chunk[lp] = all[(size_t)lp * cfg->events_per_lp + k];
    st = gpq_queue_insert(gpq_legacy_queue(), chunk.data(), L, 0, NULL);
    queue_post_init();
  }
  uint32_t* d_count = NULL;
  unsigned long long *d_csum = NULL, *d_ohash = NULL;
  cudaMalloc(&d_count, L * sizeof(uint32_t));
  cudaMalloc(&d_csum, L * sizeof(unsigned long long));
  cudaMalloc(&d_ohash, L * sizeof(unsigned long long));
  cudaMemset(d_count, 0, L * sizeof(uint32_t));
  cudaMemset(d_csum, 0, L * sizeof(unsigned long long));
  cudaMemset(d_ohash, 0, L * sizeof(unsigned long long));
  const gpq_phold_params p = dropin_params(cfg);
  unsigned long long steps = 0;
  while (!st && gpq_legacy_status() == GPQ_OK) {
    const float current_ts = queue_get_min_ts();
    if (!(current_ts < cfg->end_time)) break;
    queue_pre();
    handle_next_event<<<(L + 255) / 256, 256>>>(p, L, d_count, d_csum, d_ohash);
    if (cudaDeviceSynchronize() != cudaSuccess) { st = GPQ_ERR_CUDA; break; }
    queue_post();
    ++steps;
  }
  if (!st) st = gpq_legacy_status();
  cudaMemcpy(count, d_count, L * sizeof(uint32_t), cudaMemcpyDeviceToHost);
  cudaMemcpy(csum, d_csum, L * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
  cudaMemcpy(ohash, d_ohash, L * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
  *steps_out = steps;
  *committed_out = (unsigned long long)get_dequeue_count();
  queue_finish();
  cudaFree(d_count);
  cudaFree(d_csum);
  cudaFree(d_ohash);
  return st;
}
