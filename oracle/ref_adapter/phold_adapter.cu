// TEST INFRASTRUCTURE ONLY -- the PHOLD model that drives the reference's own queues.
//
// oracle/build_ref.py compiles this file together with the reference's unmodified
// src/des.cu (the safe-window loop, src/des.cu:154-214) and ONE of its per-LP queues
// (src/local_array_queue.cu + src/sort.cu, src/local_heap_queue.cu or
// src/local_splay_queue.cu) into a binary under oracle/_ref/.  It implements the
// reference's model interface (src/model.h:9-18: model_init, model_handle_next,
// model_get_events, model_finish) the way src/phold.cu:81-163 does -- a handler kernel
// that peeks ONE event per LP, counts it, sets it done and inserts its child -- with
// this project's event semantics (include/gpq/model.h: counter-based draws, own
// logarithm, float32 timestamps) instead of curand, so that its per-LP results can be
// compared bit for bit with the CPU oracle and with the CUDA engine.
//
// Key packing.  The reference's item is `struct event { long ts; int node; }` ordered by
// `ts` (src/queue_item.h:13-26).  An event (ts, lp, id) is stored as
// ts = (bits(ts) << 32) | id, node = lp, so the reference's `<` orders an LP's events by
// (ts bits, id) -- the order (ts bits, lp, id) restricted to one LP.  The window test
// `ts < global_min + LOOKAHEAD` of the queues is made a float32 test by the generated
// config.h (LOOKAHEAD expands to gpq_ref_window_offset(global_min)).
//
// Nothing here may fault: every queue is sized from the generated config.h far above
// the workload's per-LP occupancy, and the adapter keeps its own per-LP count of queued
// events and refuses (error word, no write) an insert that would pass the queue's
// capacity -- the local heap and splay queues write inserts without a bound check.
#include <stdint.h>
#include <stdio.h>

#include "config.h"
#include "queue.h"
#include "queue.cuh"
#include "model.h"
#include "util.cuh"
#include "gpq/model.h"

#include "ref_adapter.h"

// declared by src/des.cu for its optional monotonicity check (src/phold.cu:38-47)
__device__ long lp_last_ts[NUM_LPS];
__device__ long lp_current_ts[NUM_LPS];

// capacity of one LP's queue, from the queue's own sizing macros
#if defined(_LOCAL_ARRAY_QUEUE)
#define GPQ_REF_LP_CAPACITY ((long)FEL_SIZE - 2)              // ring of FEL_SIZE slots
#elif defined(_LOCAL_HEAP_QUEUE)
#define GPQ_REF_LP_CAPACITY ((long)FEL_SIZE - 2)              // heap array of FEL_SIZE items
#elif defined(_LOCAL_SPLAY_QUEUE)
#define GPQ_REF_LP_CAPACITY ((long)(FEL_SIZE < (long)MALLOC_BUF_SIZE ? FEL_SIZE : (long)MALLOC_BUF_SIZE) - 2)
#else
#error "the adapter drives the local array, local heap or local splay queue"
#endif

static __device__ uint32_t a_count[NUM_LPS];
static __device__ unsigned long long a_csum[NUM_LPS];
static __device__ unsigned long long a_ohash[NUM_LPS];
static __device__ int a_queued[NUM_LPS];                 // events held by the LP's queue
static __device__ unsigned long long a_queued_csum;      // sum of ev_hash over queued events
static __device__ unsigned int a_error;                  // 1 insert refused by the queue, 2 capacity guard
static __device__ unsigned int a_committed_this_window;

static gpq_phold_params params() {
  gpq_phold_params p;
  p.seed = GPQ_REF_SEED;
  p.num_lps = NUM_LPS;
  p.dest_mode = GPQ_REF_DEST_MODE;
  p.ring_width = GPQ_REF_RING_WIDTH;
  p.ring_threshold = GPQ_REF_RING_THRESHOLD;
  p.lookahead = GPQ_REF_LOOKAHEAD;
  p.end_time = GPQ_REF_END_TIME;
  return p;
}

static __device__ __forceinline__ queue_item pack(const gpq_item e) {
  queue_item q;
  q.ts = (long)(((unsigned long long)gpq_f2u(e.ts) << 32) | (unsigned long long)e.id);
  q.node = (int)e.lp;
  return q;
}

static __device__ __forceinline__ gpq_item unpack(const queue_item q) {
  gpq_item e;
  e.ts = gpq_u2f((uint32_t)((unsigned long long)q.ts >> 32));
  e.id = (uint32_t)((unsigned long long)q.ts & 0xffffffffull);
  e.lp = (uint32_t)q.node;
  e.aux = 0;
  return e;
}

// Inserts through the reference's queue_insert, within the LP's capacity.
static __device__ void adapter_insert(const gpq_item e) {
  if (atomicAdd(&a_queued[e.lp], 1) >= GPQ_REF_LP_CAPACITY) {
    atomicSub(&a_queued[e.lp], 1);
    atomicOr(&a_error, 2u);
    return;
  }
  if (!queue_insert(pack(e))) {
    atomicSub(&a_queued[e.lp], 1);
    atomicOr(&a_error, 1u);
    return;
  }
  atomicAdd(&a_queued_csum, (unsigned long long)gpq_ev_hash(e.id, gpq_f2u(e.ts)));
}

// src/phold.cu:63-79 populates random nodes; here LP l receives its events l*P + k,
// the chunk `k` inserting event k of every LP.
static __global__ void adapter_populate(gpq_phold_params p, uint32_t k) {
  for (uint32_t lp = threadIdx.x + blockDim.x * blockIdx.x; lp < NUM_LPS; lp += blockDim.x * gridDim.x)
    adapter_insert(gpq_phold_initial(p, lp, k, GPQ_REF_EVENTS_PER_LP));
}

// src/phold.cu:81-117 with this project's event function; an event at or beyond the
// end time is never committed (it stays queued).
static __global__ void adapter_handle_next_event(gpq_phold_params p) {
  for (int idx = threadIdx.x + blockDim.x * blockIdx.x; idx < NUM_LPS; idx += blockDim.x * gridDim.x) {
    queue_item* ev = NULL;
    const int event_index = queue_peek(&ev, idx);
    if (event_index == -1) continue;
    const gpq_item e = unpack(*ev);
    if (!(e.ts < p.end_time)) continue;
    const uint32_t lp = e.lp;
    lp_last_ts[lp] = lp_current_ts[lp];
    lp_current_ts[lp] = ev->ts;
    const uint64_t h = gpq_ev_hash(e.id, gpq_f2u(e.ts));
    const uint32_t seq = a_count[lp];
    a_count[lp] = seq + 1;
    a_csum[lp] += h;
    a_ohash[lp] += gpq_seq_hash(h, seq);
    const gpq_item child = gpq_phold_child(p, e);
    queue_set_done(event_index);
    atomicSub(&a_queued[lp], 1);
    atomicAdd(&a_queued_csum, (unsigned long long)(0ull - h));
    adapter_insert(child);
    a_committed_this_window = 1u;
  }
}

static int g_threads = 0, g_blocks = 0;
static unsigned long long g_windows = 0, g_calls = 0;

void model_init() {
  g_threads = NUM_LPS < MAX_THREADS__PHOLD ? NUM_LPS : MAX_THREADS__PHOLD;
  g_blocks = (NUM_LPS + g_threads - 1) / g_threads;
  const gpq_phold_params p = params();
  for (uint32_t k = 0; k < GPQ_REF_EVENTS_PER_LP; ++k) {  // chunks of POPULATE_STEPS = NUM_LPS events
    queue_pre();
    adapter_populate<<<g_blocks, g_threads>>>(p, k);
    CudaCheckError();
    CudaSafeCall(cudaDeviceSynchronize());
    queue_post_init();
    CudaCheckError();
  }
}

void model_handle_next() {
  const unsigned int zero = 0;
  CudaSafeCall(cudaMemcpyToSymbol(a_committed_this_window, &zero, sizeof(zero)));
  adapter_handle_next_event<<<g_blocks, g_threads>>>(params());
  CudaSafeCall(cudaDeviceSynchronize());
  CudaCheckError();
  unsigned int any = 0;
  CudaSafeCall(cudaMemcpyFromSymbol(&any, a_committed_this_window, sizeof(any)));
  g_windows += any;  // a window whose minimum is below the end time commits at least that event
  // des_run ends on simulated time only; a minimum that stopped advancing (e.g. a failed
  // reduction) would loop forever, so the number of handler calls is capped
  if (++g_calls > GPQ_REF_MAX_CALLS) {
    fprintf(stderr, "adapter: more than %llu handler calls, stopping\n", (unsigned long long)GPQ_REF_MAX_CALLS);
    exit(3);
  }
}

long model_get_events() {
  static uint32_t c[NUM_LPS];
  CudaSafeCall(cudaMemcpyFromSymbol(c, a_count, sizeof(c)));
  long s = 0;
  for (int i = 0; i < NUM_LPS; ++i) s += c[i];
  return s;
}

void model_finish() {}

int adapter_results(gpq_ref_results* out, uint32_t* count, unsigned long long* csum, unsigned long long* ohash) {
  static int queued[NUM_LPS];
  CudaSafeCall(cudaMemcpyFromSymbol(count, a_count, sizeof(uint32_t) * NUM_LPS));
  CudaSafeCall(cudaMemcpyFromSymbol(csum, a_csum, sizeof(unsigned long long) * NUM_LPS));
  CudaSafeCall(cudaMemcpyFromSymbol(ohash, a_ohash, sizeof(unsigned long long) * NUM_LPS));
  CudaSafeCall(cudaMemcpyFromSymbol(queued, a_queued, sizeof(queued)));
  CudaSafeCall(cudaMemcpyFromSymbol(&out->pending_csum, a_queued_csum, sizeof(out->pending_csum)));
  unsigned int err = 0;
  CudaSafeCall(cudaMemcpyFromSymbol(&err, a_error, sizeof(err)));
  out->num_lps = NUM_LPS;
  out->error = err;
  out->windows = g_windows;
  out->committed = 0;
  out->pending = 0;
  for (int i = 0; i < NUM_LPS; ++i) {
    out->committed += count[i];
    out->pending += (unsigned long long)queued[i];
  }
  return 0;
}
