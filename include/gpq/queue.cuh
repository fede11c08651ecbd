/*
 * gpq/queue.cuh -- the reference's device queue functions for model kernels, over any
 * gpupq_b200 queue kind.
 *
 * The reference binds queue_insert / queue_peek / queue_set_done / queue_is_empty /
 * queue_length / queue_clear / queue_insert_or_update / queue_print to one queue
 * implementation by macro (src/queue.cuh:7-70) and model kernels call them per LP (PHOLD:
 * src/phold.cu:81-117).  Including this header in a CUDA translation unit gives those
 * names as inline __device__ functions (queue_print as a __global__) over the device view
 * of a gpq_queue, so a handler written like the reference's compiles against the library:
 *
 *     gpq_item* ev = NULL;
 *     int index = queue_peek(&ev, lp);          // lp's earliest item if ts < the window bound
 *     if (index != -1) {
 *       gpq_item child = ...;                  // the model's event function
 *       queue_set_done(index);
 *       bool ok = queue_insert(child);         // visible after the next gpq_queue_post
 *     }
 *
 * Views by kind:
 *   local array queue  the head of the LP's sorted run (src/local_array_queue.cu:760-779);
 *   local heap queue   the root of the LP's 4-ary heap (src/local_heap_queue.cu:430-447);
 *   global array, heap and local splay queues: the LP's head staged by
 *                      gpq_queue_set_bound (the reference's one item per LP per step,
 *                      src/global_array_queue.cu:147-179); queue_length, queue_is_empty
 *                      and queue_clear are host calls for these kinds (on the device
 *                      they set GPQ_ERR_UNSUPPORTED, which the next gpq_queue_post returns).
 *
 * The host binds a queue once (gpq_queue_bind, below: it copies the view into this
 * translation unit's __device__ variable), then per step sets the window
 * (gpq_queue_set_bound), launches the model kernel, and merges the inserted items
 * (gpq_queue_post) -- the reference's des_run loop (src/des.cu:154-214).
 *
 * Differences from the reference: items are gpq_item (the reference's `event.node` is
 * `lp`); queue_insert reports a full insert buffer by returning false and by the error
 * word that the next gpq_queue_post returns, instead of an assert; queue_insert_or_update
 * inserts (the reference's default build, without LOCAL_ARRAY_QUEUE_UPDATE_ELEMENTS).
 */
#ifndef GPQ_QUEUE_CUH
#define GPQ_QUEUE_CUH

#include <cuda_runtime.h>
#include <stdio.h>

#include "gpq.h"

typedef gpq_item queue_item;

/* The queue the device functions of this translation unit work on. */
static __device__ gpq_device_queue gpq_bound_queue;

/* Bind q for the device functions of this translation unit (host; blocks on nothing but
 * the symbol copy). */
static inline gpq_status gpq_queue_bind(gpq_queue* q) {
  gpq_device_queue v;
  const gpq_status s = gpq_queue_device_view(q, &v);
  if (s != GPQ_OK) return s;
  return cudaMemcpyToSymbol(gpq_bound_queue, &v, sizeof(v)) == cudaSuccess ? GPQ_OK : GPQ_ERR_CUDA;
}

/* queue_insert (src/queue.cuh:46-47): reserve a slot in the item's LP buffer. */
static __device__ __forceinline__ bool queue_insert(queue_item item) {
  const gpq_device_queue& q = gpq_bound_queue;
  const uint32_t pos = atomicAdd(&q.icnt[item.lp], 1u);
  if (pos >= q.ibc) {
    atomicCAS(q.err, 0u, (uint32_t)GPQ_ERR_INSERT_FULL);
    return false;
  }
  q.ibuf[(size_t)item.lp * q.ibc + pos] = item;
  atomicAdd(q.enqueued, 1ull);
  return true;
}

/* Removes the root of a 4-ary heap of n > 0 items (one thread): the last item sifts
 * down from the root past every child with a smaller (ts bits, id) key. */
static __device__ __forceinline__ void gpq_heap4_pop(queue_item* h, uint32_t n) {
  const uint32_t last = n - 1;
  if (last == 0) return;
  const queue_item x = h[last];
  const uint64_t kx = gpq_lp_key(x);
  uint32_t pos = 0;
  for (;;) {
    const uint32_t fc = pos * 4u + 1u;
    if (fc >= last) break;
    uint32_t b = fc;
    uint64_t kb = gpq_lp_key(h[fc]);
    for (uint32_t c = fc + 1u; c < fc + 4u && c < last; ++c) {
      const uint64_t kc = gpq_lp_key(h[c]);
      if (kc < kb) { kb = kc; b = c; }
    }
    if (kb >= kx) break;
    h[pos] = h[b];
    pos = b;
  }
  h[pos] = x;
}

/* queue_peek (src/queue.cuh:49-51): the index of lp's earliest item if it lies inside
 * the window (ts < bound), else -1; *item points at it until queue_set_done/post. */
static __device__ __forceinline__ int queue_peek(queue_item** item, int lp) {
  const gpq_device_queue& q = gpq_bound_queue;
  if (q.staged) {
    queue_item* it = q.head + lp;
    if (q.taken[lp] || !(it->ts < *q.bound)) return -1;
    *item = it;
    return lp;
  }
  if (q.kind == GPQ_QUEUE_LHQ) {
    if (q.size[lp] == 0u) return -1;
    queue_item* it = q.ring + ((size_t)lp << q.cap_log2);
    if (!(it->ts < *q.bound)) return -1;
    *item = it;
    return (int)((uint32_t)lp << q.cap_log2);
  }
  const uint32_t rd = q.rd[lp];
  if (rd == q.wr[lp]) return -1;
  const uint32_t slot = rd & ((1u << q.cap_log2) - 1u);
  queue_item* it = q.ring + ((size_t)lp << q.cap_log2) + slot;
  if (!(it->ts < *q.bound)) return -1;
  *item = it;
  return (int)(((uint32_t)lp << q.cap_log2) | slot);
}

/* queue_set_done (src/queue.cuh:53-54): the peeked item leaves lp's run. */
static __device__ __forceinline__ void queue_set_done(int index) {
  const gpq_device_queue& q = gpq_bound_queue;
  if (q.staged) {
    q.taken[index] = 1u;
    return;
  }
  const uint32_t lp = (uint32_t)index >> q.cap_log2;
  if (q.kind == GPQ_QUEUE_LHQ) {
    const uint32_t n = q.size[lp];
    gpq_heap4_pop(q.ring + ((size_t)lp << q.cap_log2), n);
    q.size[lp] = n - 1u;
  } else {
    q.rd[lp] += 1u;
  }
  atomicAdd(q.dequeued, 1ull);
}

/* queue_is_empty (src/queue.cuh:59-60): nothing queued and nothing inserted since the
 * last post (src/local_array_queue.cu:807-810). */
static __device__ __forceinline__ bool gpq_device_call_unsupported(const gpq_device_queue& q) {
  if (!q.staged) return false;
  atomicCAS(q.err, 0u, (uint32_t)GPQ_ERR_UNSUPPORTED);
  return true;
}

static __device__ __forceinline__ bool queue_is_empty(int lp) {
  const gpq_device_queue& q = gpq_bound_queue;
  if (gpq_device_call_unsupported(q)) return false;
  const bool none = q.kind == GPQ_QUEUE_LHQ ? q.size[lp] == 0u : q.rd[lp] == q.wr[lp];
  return none && q.icnt[lp] == 0u;
}

/* queue_length (src/queue.cuh:62-63): items in lp's run or heap. */
static __device__ __forceinline__ int queue_length(int lp) {
  const gpq_device_queue& q = gpq_bound_queue;
  if (gpq_device_call_unsupported(q)) return -1;
  return q.kind == GPQ_QUEUE_LHQ ? (int)q.size[lp] : (int)(q.wr[lp] - q.rd[lp]);
}

/* queue_clear (src/queue.cuh:65-66): drop lp's run. */
static __device__ __forceinline__ void queue_clear(int lp) {
  const gpq_device_queue& q = gpq_bound_queue;
  if (gpq_device_call_unsupported(q)) return;
  uint32_t n;
  if (q.kind == GPQ_QUEUE_LHQ) {
    n = q.size[lp];
    q.size[lp] = 0u;
  } else {
    n = q.wr[lp] - q.rd[lp];
    q.rd[lp] = q.wr[lp];
  }
  atomicAdd(q.dequeued, (unsigned long long)n);
}

/* queue_insert_or_update (src/queue.cuh:68-69). */
static __device__ __forceinline__ void queue_insert_or_update(queue_item item, int lp) {
  item.lp = (uint32_t)lp;
  queue_insert(item);
}

/* queue_print (src/queue.cuh:56-57, a __global__ as in the reference): prints lp's items
 * in key order (local array queue: its run; local heap queue: its heap in array order;
 * staged kinds: the staged head -- gpq_queue_dump lists every item of any kind). */
static __global__ void queue_print(int lp) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const gpq_device_queue& q = gpq_bound_queue;
  printf("[queue %d] lp %d:", (int)q.kind, lp);
  if (q.staged) {
    const queue_item h = q.head[lp];
    if (gpq_f2u(h.ts) != 0x7f800000u && !q.taken[lp]) printf(" (%.6f, id %u)", h.ts, h.id);
  } else if (q.kind == GPQ_QUEUE_LHQ) {
    const queue_item* it = q.ring + ((size_t)lp << q.cap_log2);
    for (uint32_t i = 0; i < q.size[lp]; ++i) printf(" (%.6f, id %u)", it[i].ts, it[i].id);
  } else {
    const uint32_t m = (1u << q.cap_log2) - 1u;
    const queue_item* it = q.ring + ((size_t)lp << q.cap_log2);
    for (uint32_t c = q.rd[lp]; c != q.wr[lp]; ++c) printf(" (%.6f, id %u)", it[c & m].ts, it[c & m].id);
  }
  printf("\n");
}

#endif /* GPQ_QUEUE_CUH */
