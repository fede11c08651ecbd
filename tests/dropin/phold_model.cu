// TEST INFRASTRUCTURE: a PHOLD model written the way the reference writes its models --
// a handler kernel that peeks one event per LP, counts it, sets it done and inserts its
// child (src/phold.cu:81-117), driven by a host loop of get-min / window / handler /
// post steps (src/des.cu:154-214) -- compiled against include/gpq/queue.cuh and linked
// with libgpq.so.  It shows that a reference-style model drops onto the library's
// queues; the test compares its per-LP results with the CPU oracle.
#include <cuda_runtime.h>

#include <cstdio>
#include <vector>

#include "gpq.h"
#include "gpq/queue.cuh"

#include "phold_handler.cuh"

// Runs the model; per-LP outputs to host arrays of cfg->num_lps.  Returns 0 or a
// gpq_status.
extern "C" int dropin_phold_run(const gpq_phold_config* cfg, uint32_t* count, unsigned long long* csum,
                                unsigned long long* ohash, unsigned long long* steps_out,
                                unsigned long long* committed_out) {
  const uint32_t L = cfg->num_lps;
  gpq_queue_config qc = {};
  qc.kind = cfg->queue_kind;  // any queue kind
  qc.num_lps = L;
  qc.capacity = cfg->capacity ? cfg->capacity : 256;
  qc.insert_capacity = cfg->insert_capacity ? cfg->insert_capacity : 64;
  gpq_queue* q = NULL;
  int st = gpq_queue_create(&qc, &q);
  if (st) return st;
  std::vector<gpq_item> init((size_t)L * cfg->events_per_lp);
  st = gpq_phold_initial_events(cfg, init.data(), init.size());
  if (!st) st = gpq_queue_insert(q, init.data(), init.size(), 0, NULL);
  if (!st) st = gpq_queue_post_init(q, NULL);
  if (!st) st = gpq_queue_bind(q);
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
  while (!st) {
    float m = 0.f;
    st = gpq_queue_get_min(q, &m, NULL);                    // queue_get_min_ts
    if (st || !(m < cfg->end_time)) break;
    float bound = m + cfg->lookahead;                       // global_min + LOOKAHEAD
    if (cfg->end_time < bound) bound = cfg->end_time;       // and ts < end time
    st = gpq_queue_set_bound(q, bound, NULL);
    if (st) break;
    handle_next_event<<<(L + 255) / 256, 256, 0, (cudaStream_t)0>>>(p, L, d_count, d_csum, d_ohash);
    if (cudaDeviceSynchronize() != cudaSuccess) { st = GPQ_ERR_CUDA; break; }
    st = gpq_queue_post(q, NULL);                           // queue_post
    ++steps;
  }
  cudaMemcpy(count, d_count, L * sizeof(uint32_t), cudaMemcpyDeviceToHost);
  cudaMemcpy(csum, d_csum, L * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
  cudaMemcpy(ohash, d_ohash, L * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
  unsigned long long enq = 0, deq = 0;
  gpq_queue_counts(q, (uint64_t*)&enq, (uint64_t*)&deq, NULL);
  *steps_out = steps;
  *committed_out = deq;
  cudaFree(d_count);
  cudaFree(d_csum);
  cudaFree(d_ohash);
  gpq_queue_destroy(q);
  return st;
}
