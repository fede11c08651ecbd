// TEST INFRASTRUCTURE ONLY -- results of a run of the reference's queues under the
// adapter model (oracle/ref_adapter/phold_adapter.cu).
#pragma once
#include <stdint.h>

typedef struct gpq_ref_results {
  uint64_t num_lps;
  uint64_t committed;
  uint64_t windows;       // handler calls that committed an event (windows with minimum < end time)
  uint64_t pending;       // events left in the queues
  unsigned long long pending_csum;
  uint64_t error;         // 1 an insert refused by the queue, 2 the adapter's capacity guard
} gpq_ref_results;

int adapter_results(gpq_ref_results* out, uint32_t* count, unsigned long long* csum, unsigned long long* ohash);
