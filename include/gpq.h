/*
 * gpq.h -- C ABI of gpupq_b200 (libgpq.so), a B200-native rebuild of GPUPQ's
 * data-parallel priority-queue hot path.
 *
 * Plain C types only: pointers, sizes, and an opaque stream handle (`void*`,
 * a cudaStream_t; NULL = the library's own stream).  Every function returns a
 * gpq_status; nothing calls exit().  The reference's host functions abort the
 * process on errors (src/util.cuh:36-39, src/des.cu:37-40,57-61).
 *
 * Three groups of entry points:
 *   1. queue objects (gpq_queue_*): the reference's host queue API,
 *      src/queue.h:86-115, for one of the five queue kinds;
 *   2. the PHOLD engine (gpq_phold_*): the reference's DES driver + PHOLD model,
 *      src/des.cu:74-214 and src/phold.cu:124-192, run as a plain host-driven step
 *      loop (one launch per safe window, like des_run) or as one persistent launch;
 *   3. utilities (gpq_status_string, gpq_version).
 */
#ifndef GPQ_H
#define GPQ_H

#include <stddef.h>
#include <stdint.h>

#include "gpq/model.h" /* gpq_item, gpq_phold_params */
#include "gpq/astar.h" /* gpq_astar_grid */

#if defined(__GNUC__)
#define GPQ_API __attribute__((visibility("default")))
#else
#define GPQ_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum gpq_status {
  GPQ_OK = 0,
  GPQ_ERR_INVALID = 1,         /* bad argument or configuration */
  GPQ_ERR_CUDA = 2,            /* a CUDA runtime call failed */
  GPQ_ERR_QUEUE_FULL = 3,      /* a per-LP queue overflowed (reference: insert returns false,
                                  src/local_array_queue.cu:492-498) */
  GPQ_ERR_INSERT_FULL = 4,     /* a per-step insert buffer overflowed */
  GPQ_ERR_TIMEOUT = 5,         /* a device-side wait gave up (bounded spin) */
  GPQ_ERR_NOMEM = 6,           /* device allocation failed or budget exceeded */
  GPQ_ERR_UNSUPPORTED = 7,     /* option not available for this queue kind */
  GPQ_ERR_NOT_READY = 8        /* handle not populated / result not available */
} gpq_status;

/* The five queue kinds of the reference (src/config.h:8-13, src/queue.h:33-84). */
typedef enum gpq_queue_kind {
  GPQ_QUEUE_LAQ = 0, /* local array queue: per-LP sorted ring (src/local_array_queue.cu) */
  GPQ_QUEUE_GAQ = 1, /* global array queue: one globally sorted array (src/global_array_queue.cu) */
  GPQ_QUEUE_HQ = 2,  /* parallel heap of sorted r-item nodes (src/heap_queue.cu) */
  GPQ_QUEUE_LHQ = 3, /* local heap queue: per-LP array heap (src/local_heap_queue.cu) */
  GPQ_QUEUE_LSQ = 4  /* local splay queue: per-LP splay tree (src/local_splay_queue.cu) */
} gpq_queue_kind;

/* How the PHOLD engine drives its safe-window steps. */
typedef enum gpq_loop_mode {
  GPQ_LOOP_PLAIN = 0,      /* host loop: one launch per window + a D2H read of the minimum
                              (the reference's des_run, src/des.cu:154-214) */
  GPQ_LOOP_PERSISTENT = 1  /* one cooperative launch; windows separated by a bounded grid barrier */
} gpq_loop_mode;

/* ---------------------------------------------------------------------------------- */
/* 1. Queue objects                                                                   */
/* ---------------------------------------------------------------------------------- */

typedef struct gpq_queue gpq_queue;

typedef struct gpq_queue_config {
  uint32_t kind;            /* gpq_queue_kind */
  uint32_t num_lps;         /* number of logical processes (NUM_LPS, src/config.h:67) */
  uint32_t capacity;        /* per-LP capacity (LAQ/LHQ/LSQ); total capacity / num_lps (GAQ, HQ) */
  uint32_t insert_capacity; /* per-LP inserts accepted between two posts (LAQ/LHQ/LSQ);
                               total per post = insert_capacity * num_lps (GAQ, HQ) */
  uint32_t node_size;       /* HQ node size r (HQ_NODE_SIZE, src/config.h:88); 0 = default */
  uint32_t reserved[3];
} gpq_queue_config;

/* queue_init (src/queue.h:86-87). */
GPQ_API gpq_status gpq_queue_create(const gpq_queue_config* cfg, gpq_queue** out);
GPQ_API gpq_status gpq_queue_destroy(gpq_queue* q);

/* queue_insert for a batch of items (src/queue.cuh:46-47); items are HOST pointers
 * unless `items_on_device` is non-zero.  Takes effect at the next gpq_queue_post. */
GPQ_API gpq_status gpq_queue_insert(gpq_queue* q, const gpq_item* items, uint64_t n, int items_on_device, void* stream);

/* queue_pre / queue_post / queue_post_init (src/queue.h:89-98). */
GPQ_API gpq_status gpq_queue_pre(gpq_queue* q, void* stream);
GPQ_API gpq_status gpq_queue_post(gpq_queue* q, void* stream);
GPQ_API gpq_status gpq_queue_post_init(gpq_queue* q, void* stream);

/* queue_get_min_ts (src/queue.h:100-103): smallest timestamp over all queued items
 * (+inf when empty).  Blocks on the stream. */
GPQ_API gpq_status gpq_queue_get_min(gpq_queue* q, float* min_ts, void* stream);

/* queue_peek + queue_set_done for every LP at once (src/queue.cuh:49-54): removes, per
 * LP, up to `max_per_lp` items with ts < bound, in key order (0 = no limit; the
 * reference dequeues one per LP per step, src/phold.cu:84-94).  The removed items are
 * written to `out` (host array of `out_capacity` items) grouped by LP in ascending LP
 * order and key order inside an LP; `*n_out` receives their number. */
GPQ_API gpq_status gpq_queue_dequeue(gpq_queue* q, float bound, uint32_t max_per_lp, gpq_item* out,
                             uint64_t out_capacity, uint64_t* n_out, void* stream);

/* queue_length / queue_is_empty / queue_clear (src/queue.cuh:62-69) for one LP. */
GPQ_API gpq_status gpq_queue_length(gpq_queue* q, uint32_t lp, uint32_t* length, void* stream);
GPQ_API gpq_status gpq_queue_clear(gpq_queue* q, uint32_t lp, void* stream);

/* queue_print (src/queue.cuh:56-57) as data: the items of one LP in key order (for GAQ
 * and HQ the items of that LP in the global structure).  `*n_out` = item count. */
GPQ_API gpq_status gpq_queue_dump(gpq_queue* q, uint32_t lp, gpq_item* out, uint64_t out_capacity, uint64_t* n_out,
                          void* stream);

/* get_enqueue_count / get_dequeue_count (src/queue.h:110-113): items inserted and
 * removed since creation. */
GPQ_API gpq_status gpq_queue_counts(gpq_queue* q, uint64_t* enqueued, uint64_t* dequeued, void* stream);

/* Device-side access to a queue for model kernels: the reference's device queue
 * functions (queue_insert, queue_peek, queue_set_done, queue_is_empty, queue_length,
 * queue_clear, queue_insert_or_update, queue_print; src/queue.cuh:7-70) are provided as
 * inline __device__ functions over this view by include/gpq/queue.cuh.
 *   local array / local heap queue: the view is the queue's own per-LP arrays;
 *   global array / heap / local splay queue: `staged` is 1 -- gpq_queue_set_bound moves
 *     each LP's earliest item below the bound into head[lp] (the reference's one item per
 *     LP per step, src/global_array_queue.cu:147-179); queue_peek returns it,
 *     queue_set_done marks it taken, and gpq_queue_post gives back the untaken heads
 *     together with the inserted items.  queue_length, queue_is_empty and queue_clear are
 *     not offered on the device for these kinds (the call sets GPQ_ERR_UNSUPPORTED, which
 *     the next gpq_queue_post returns; the host functions gpq_queue_length/clear work). */
typedef struct gpq_device_queue {
  gpq_item* ring;               /* [num_lps << cap_log2] per-LP sorted runs (LAQ) or 4-ary heaps (LHQ) */
  uint32_t* rd;                 /* LAQ: per-LP read counter (fel_read); slot = counter & (cap - 1) */
  uint32_t* wr;                 /* LAQ: per-LP write counter (fel_write) */
  gpq_item* ibuf;               /* [num_lps][ibc] items inserted since the last post */
  uint32_t* icnt;               /* [num_lps] */
  const float* bound;           /* queue_peek returns the head iff its ts < *bound */
  unsigned long long* enqueued; /* get_enqueue_count */
  unsigned long long* dequeued; /* get_dequeue_count */
  uint32_t* err;                /* sticky error word read by the next gpq_queue_post */
  uint32_t num_lps, cap_log2, ibc;
  uint32_t kind;                /* gpq_queue_kind */
  uint32_t* size;               /* LHQ: per-LP heap size (root at slot 0, children of i at 4i+1..4i+4) */
  gpq_item* head;               /* staged kinds: [num_lps] earliest item below the bound (ts +inf: none) */
  uint32_t* taken;              /* staged kinds: [num_lps] set by queue_set_done */
  uint32_t staged;              /* 1 for the global array, heap and local splay queues */
} gpq_device_queue;

/* Fills *out with the device pointers of the queue's device view (allocated at the first
 * call for the staged kinds).  The view stays valid until gpq_queue_destroy. */
GPQ_API gpq_status gpq_queue_device_view(gpq_queue* q, gpq_device_queue* out);

/* Sets the window bound queue_peek tests against (the reference's global_min + LOOKAHEAD,
 * src/local_array_queue.cu:760-779); +inf at creation.  Stream-ordered for the local
 * array and local heap queues; for the staged kinds it also stages the heads and blocks
 * on the stream. */
GPQ_API gpq_status gpq_queue_set_bound(gpq_queue* q, float bound, void* stream);

/* The reference's host queue API over one library-owned queue (src/queue.h:86-115:
 * queue_init, queue_pre, queue_post, queue_post_init, queue_get_min_ts, queue_finish,
 * get_enqueue_count, get_dequeue_count).  include/gpq/legacy.h gives these the
 * reference's names; gpq_legacy_configure sets what the reference's config.h fixes at
 * compile time (the queue's kind and sizes, LOOKAHEAD, and an end time that caps the
 * window bound; 0 = none).  Errors are kept: gpq_legacy_status returns the first. */
GPQ_API gpq_status gpq_legacy_configure(const gpq_queue_config* cfg, float lookahead, float end_time);
GPQ_API gpq_status gpq_legacy_init(gpq_queue** out);      /* queue_init: (re)creates the queue */
GPQ_API gpq_queue* gpq_legacy_queue(void);                /* the queue (NULL before queue_init) */
GPQ_API gpq_status gpq_legacy_pre(void);                  /* queue_pre: bound = min + lookahead */
GPQ_API gpq_status gpq_legacy_post(void);                 /* queue_post / queue_post_init */
GPQ_API float gpq_legacy_get_min_ts(void);                /* queue_get_min_ts (cached until post) */
GPQ_API gpq_status gpq_legacy_counts(uint64_t* enqueued, uint64_t* dequeued);
GPQ_API gpq_status gpq_legacy_finish(void);               /* queue_finish */
GPQ_API gpq_status gpq_legacy_status(void);               /* first error since queue_init */

/* ---------------------------------------------------------------------------------- */
/* 2. PHOLD engine                                                                    */
/* ---------------------------------------------------------------------------------- */

typedef struct gpq_phold gpq_phold;

typedef struct gpq_phold_config {
  uint64_t seed;
  uint32_t num_lps;
  uint32_t events_per_lp;   /* initial events per LP (ids lp*events_per_lp + k) */
  float lookahead;          /* LOOKAHEAD (src/config.h:65) as float32 */
  float end_time;           /* events with ts >= end_time are never committed */
  uint32_t dest_mode;       /* GPQ_DEST_UNIFORM / GPQ_DEST_RING (gpq/model.h) */
  uint32_t ring_width;      /* ring neighbourhood +-ring_width (self excluded) */
  uint32_t ring_threshold;  /* ring with probability ring_threshold / 2^32 */
  uint32_t queue_kind;      /* gpq_queue_kind */
  uint32_t capacity;        /* per-LP queue capacity (power of two for LAQ) */
  uint32_t insert_capacity; /* per-LP insert-buffer slots per window */
  uint32_t loop_mode;       /* gpq_loop_mode */
  uint32_t block_threads;   /* CTA size (multiple of 32); 0 = tuned default */
  uint32_t ctas_per_sm;     /* persistent grid: CTAs per SM; 0 = occupancy maximum */
  uint32_t max_steps;       /* safety cap on windows; 0 = none */
  uint32_t lanes_per_lp;    /* LAQ: lanes that work on one LP (4, 8, 16 or 32); 0 = tuned default */
  uint32_t node_size;       /* HQ: items per heap node r, a power of two in [2, 2^22]: one CTA
                             * works a heap of nodes up to 1,024 items, the whole GPU (one
                             * cooperative launch) larger ones; 0 = the reference's 256 K
                             * (HQ_NODE_SIZE, src/config.h:88), lowered to the population
                             * rounded up to a power of two (at least 2,048) */
  uint32_t laq_mode;        /* LAQ: 0 = sorted runs, children merged each window; 1 = unordered
                               arrays, each window's safe events selected and ranked; 2 = time
                               buckets of 8-byte keys per LP, each window's buckets ranked
                               (bucket geometry from lookahead and events_per_lp; capacity and
                               insert_capacity unused) */
  uint32_t gaq_engine;      /* GAQ: 0 = one sorted array worked by the whole GPU in one
                             * cooperative launch when the population fits 4 M items (the heap
                             * kernel with a single node), else the kernel sequence below;
                             * 1 = the kernel sequence per window (radix sort, merge) replayed
                             * as a CUDA graph */
} gpq_phold_config;

typedef struct gpq_phold_result {
  uint64_t committed;     /* events committed (ts < end_time) */
  uint64_t steps;         /* safe windows executed */
  uint64_t pending;       /* events left queued at the end (all with ts >= end_time) */
  uint64_t pending_csum;  /* sum of ev_hash over the pending events */
  uint64_t digest;        /* order-sensitive digest over (lp, count, csum, ohash) */
  float final_min;        /* smallest pending timestamp at the end */
  float elapsed_ms;       /* device time of the last gpq_phold_run (CUDA events) */
  int32_t status;         /* device error word (gpq_status) */
  uint32_t reserved[3];
} gpq_phold_result;

GPQ_API gpq_status gpq_phold_create(const gpq_phold_config* cfg, gpq_phold** out);
GPQ_API gpq_status gpq_phold_destroy(gpq_phold* h);

/* model_init (src/phold.cu:124-163): resets all state and inserts the initial events.
 * `initial` = NULL generates them on the device from the seed; otherwise it is a HOST
 * array of n = num_lps * events_per_lp items (e.g. from gpq_phold_initial_events). */
GPQ_API gpq_status gpq_phold_populate(gpq_phold* h, const gpq_item* initial, uint64_t n, void* stream);

/* des_run (src/des.cu:134-221): run safe windows until the minimum reaches end_time.
 * Stream-ordered; the device time between start and end is recorded with CUDA events
 * on `stream` and reported in gpq_phold_result.elapsed_ms. */
GPQ_API gpq_status gpq_phold_run(gpq_phold* h, void* stream);

/* Run at most `nsteps` further windows (plain loop); *done = 1 once finished. */
GPQ_API gpq_status gpq_phold_step(gpq_phold* h, uint32_t nsteps, int* done, void* stream);

/* des_finish (src/des.cu:89-132) as data.  Blocks on the stream. */
GPQ_API gpq_status gpq_phold_result_get(gpq_phold* h, gpq_phold_result* out, void* stream);

/* model_get_events (src/phold.cu:169-182) per LP: committed count, order-insensitive
 * checksum and order-sensitive hash (HOST arrays of num_lps entries; any may be NULL). */
GPQ_API gpq_status gpq_phold_lp_stats(gpq_phold* h, uint32_t* count, uint64_t* csum, uint64_t* ohash, void* stream);

/* The initial events the engine would generate, written to a HOST array of
 * num_lps * events_per_lp items (host computation, bit-identical to the device). */
GPQ_API gpq_status gpq_phold_initial_events(const gpq_phold_config* cfg, gpq_item* out, uint64_t n);

/* Children of `n` events under `cfg` (the model's event function), computed on the
 * device; `events` and `children` are HOST arrays. */
GPQ_API gpq_status gpq_phold_children(const gpq_phold_config* cfg, const gpq_item* events, gpq_item* children,
                              uint64_t n);

/* Snapshot of a run's whole state between windows (its queues, per-LP outputs, window
 * slots and window count) into a HOST buffer, and its restore into a handle created with
 * the same configuration; the restored run continues exactly as the original would.  The
 * reference has no checkpoint; this lets a caller stop a long run and resume it later, or
 * run one prefix and branch several continuations from it.  With buf == NULL,
 * gpq_phold_snapshot only reports the size.  Both block on the stream. */
GPQ_API gpq_status gpq_phold_snapshot(gpq_phold* h, void* buf, uint64_t capacity, uint64_t* size, void* stream);
GPQ_API gpq_status gpq_phold_restore(gpq_phold* h, const void* buf, uint64_t size, void* stream);

/* Sharded PHOLD: one handle per shard (rank) of a run over cfg->num_lps LPs; shard r
 * holds LPs [r*P, min((r+1)*P, num_lps)), P = ceil(num_lps / world), and processes
 * their events.  The reference runs one GPU; this splits the LP space across GPUs with
 * one exchange per window, driven by the host (gpupq_b200.shard drives it over
 * torch.distributed):
 *   populate -> local minimum; the global minimum is the minimum over shards;
 *   window(global minimum) -> the shard's safe events run; children for other shards'
 *     LPs wait in the outbox ([world][capacity] device items, counts per destination);
 *     local minimum (pending events and all children, handed over or not);
 *   inject(the items other shards handed to this one) -> merged in the next window (the
 *     bucketed local array queue files them at once, as if pushed in the window run);
 *   repeat while the global minimum is below end_time.
 * A child is never safe in its parent's window, so handing children over between windows
 * changes no result: the shards' committed counts, pending events and digests add up
 * (final minimum: the minimum) to those of the unsharded run.  Per-LP queue kinds only
 * (LAQ in every form, LHQ, LSQ).  outbox_capacity 0 = the shard's LPs times
 * insert_capacity (bucketed form: events_per_lp) per destination.  gpq_phold_result_get
 * gives the shard's part. */
GPQ_API gpq_status gpq_phold_shard_create(const gpq_phold_config* cfg, uint32_t rank, uint32_t world,
                                          uint32_t outbox_capacity, gpq_phold** out);
GPQ_API gpq_status gpq_phold_shard_range(gpq_phold* h, uint32_t* lp_begin, uint32_t* lp_end, uint32_t* outbox_capacity);
GPQ_API gpq_status gpq_phold_shard_populate(gpq_phold* h, float* local_min, void* stream);
GPQ_API gpq_status gpq_phold_shard_window(gpq_phold* h, float global_min, float* local_min, uint32_t* out_counts,
                                          void* stream);
GPQ_API gpq_status gpq_phold_shard_outbox(gpq_phold* h, gpq_item** items, uint32_t* capacity);
GPQ_API gpq_status gpq_phold_shard_inject(gpq_phold* h, const gpq_item* items, uint64_t n, int on_device,
                                          void* stream);
/* Direct hand-over for the bucketed local array queue's shards (laq_mode 2) of one
 * process: shards[r] is shard r of the same run (same configuration), on this GPU or on a
 * GPU this one has peer access to (enabled here).  Afterwards the shard's windows file a
 * child of another shard's LP straight into that shard's time buckets (stores into its
 * memory; the same append rule as a local child), so no outbox, exchange or inject is
 * needed between windows -- only the minimum over the shards' local minima.  Call it for
 * every shard, after all of them are created and before the first window. */
GPQ_API gpq_status gpq_phold_shard_connect(gpq_phold* h, gpq_phold* const* shards, uint32_t world);

/* Launch geometry of the last gpq_phold_run: persistent grid (CTAs), CTA size, and the
 * number of kernel launches the run made (1 for the persistent loop, one per window
 * for the plain loop). */
GPQ_API gpq_status gpq_phold_launch_info(gpq_phold* h, uint32_t* grid, uint32_t* block, uint32_t* launches_per_run);

/* Allocation-free PHOLD run.  No counterpart in the reference (it allocates its queues
 * with cudaMalloc in queue_init, src/local_array_queue.cu:429-433).
 *
 * For callers that cannot allocate device memory at run time: an application whose
 * device memory is already owned by another allocator or fixed plan (a cudaMalloc would
 * fail or break the plan), or a latency-bound caller that cannot pay for cudaMalloc and
 * cudaFree, which may synchronize the device.  One call populates, runs every window
 * with the persistent loop, and reduces the results -- like gpq_phold_create + populate +
 * run + result_get + destroy, with the same results -- but allocates nothing: all queue
 * state lives in one fixed array of GPQ_STATIC_SCRATCH_BYTES (16 MiB) of device memory
 * that every GPU loading this library holds until the process exits.
 *
 *   d_initial  DEVICE array of num_lps * events_per_lp items grouped by LP (as from
 *              gpq_phold_initial_events), or NULL to generate them from the seed;
 *   d_count, d_csum, d_ohash  DEVICE arrays of num_lps entries, overwritten with the
 *              per-LP results (as gpq_phold_lp_stats);
 *   out        HOST result; elapsed_ms is not measured here (0).
 * Sorted local array queue only (queue_kind LAQ, laq_mode 0; anything else returns
 * GPQ_ERR_UNSUPPORTED).  A configuration whose queues need more than the fixed array
 * (about 1024 LPs at capacity 256 and insert capacity 64 use 6.3 MiB) is rejected with
 * GPQ_ERR_INVALID and a message naming the size.  The first call on a device (with that
 * device current) looks up the array's device address and caches it; make that first
 * call before any stream capture, and do not call this entry point on a device after a
 * cudaDeviceReset of it (the cached address would be stale).  All calls share the array and each call re-initializes what it needs:
 * calls that overlap on the GPU race with each other -- serialize them.  Blocks on
 * `stream` (NULL = the legacy default stream). */
#define GPQ_STATIC_SCRATCH_BYTES (16u * 1024u * 1024u)
GPQ_API gpq_status gpq_phold_run_static(const gpq_phold_config* cfg, const gpq_item* d_initial, uint32_t* d_count,
                                        uint64_t* d_csum, uint64_t* d_ohash, gpq_phold_result* out, void* stream);

/* ---------------------------------------------------------------------------------- */
/* 2b. A* grid search (the a_star model, src/a_star.cu:269-593, over sharded queues)   */
/* ---------------------------------------------------------------------------------- */

/* Engine knobs.  The open list of an instance is sharded by square tiles of the grid
 * (`tile` x `tile` cells per shard); each round expands, per instance, every open item
 * with f <= bound, where the window [min f, min f + window] moves when it is drained. */
typedef struct gpq_astar_config {
  uint32_t tile;              /* tile side, a power of two in [8, 128]; 0 = 64 */
  uint32_t window;            /* window width on f; 0 = 4 move costs */
  uint32_t inbox_capacity;    /* items one tile receives per round; 0 = 8 * tile */
  uint32_t open_capacity;     /* items one tile keeps above the window; 0 = tile * tile */
  uint32_t frontier_capacity; /* shared-memory frontier items (two buffers); 0 = 2048 (256 per warp) */
  uint32_t block_threads;     /* 64, 128 or 256; 0 = 256 */
  uint32_t ctas_per_sm;       /* 0 = one per SM for every SM's worth of tiles expected active at a
                                 once (sqrt(tiles) per instance), at most as many as fit */
  uint32_t max_rounds;        /* 0 = 2^20; reaching it is GPQ_ERR_TIMEOUT */
  uint32_t tile_worker;       /* who processes one tile visit: 0 = a CTA, 1 = a warp */
  uint32_t reserved[3];
} gpq_astar_config;

typedef struct gpq_astar_result {
  uint32_t cost;      /* C*; GPQ_ASTAR_INF (0xFFFFFFFF) when the goal is unreachable */
  uint32_t path_len;  /* cells on the canonical path, start and goal included */
  uint64_t expanded;  /* cells with g + h <= C* (every reached cell when unreachable) */
  uint64_t gsum;      /* sum of gpq_astar_cell_hash over the expanded cells */
  uint64_t path_hash; /* sum of gpq_astar_path_hash over the path, goal = position 0 */
  uint64_t pops;      /* expansions performed, re-expansions included */
  uint32_t windows;   /* window moves */
  int32_t status;     /* gpq_status of this instance */
} gpq_astar_result;

typedef struct gpq_astar gpq_astar;

GPQ_API gpq_status gpq_astar_create(const gpq_astar_config* cfg, gpq_astar** out);
GPQ_API gpq_status gpq_astar_destroy(gpq_astar* a);

/* Solve n instances (HOST array of grids) in one persistent launch; results to a HOST
 * array of n.  Device buffers grow as needed and are kept for the next call.  When an
 * instance overflows its tile buffers the batch runs again with four times the inbox
 * and open capacities (at most twice; the larger capacities stay); an instance that
 * still overflows reports GPQ_ERR_INSERT_FULL / GPQ_ERR_QUEUE_FULL in its status (its
 * other fields are then not meaningful).  Blocks on the stream. */
GPQ_API gpq_status gpq_astar_solve(gpq_astar* a, const gpq_astar_grid* grids, uint32_t n,
                                   gpq_astar_result* results, void* stream);

/* Device time of the last solve: the whole call (grid generation, search, results) and
 * the search launch alone; the number of rounds and of tile visits; the launch geometry.
 * Any pointer may be NULL. */
GPQ_API gpq_status gpq_astar_last_stats(gpq_astar* a, float* total_ms, float* search_ms, uint32_t* rounds,
                                        uint64_t* tile_visits, uint32_t* grid, uint32_t* block);

/* The canonical path of instance `index` of the last solve, goal first (HOST array). */
GPQ_API gpq_status gpq_astar_path(gpq_astar* a, uint32_t index, uint32_t* cells, uint32_t capacity,
                                  uint32_t* length, void* stream);

/* The g values of instance `index` of the last solve (HOST array of width * height). */
GPQ_API gpq_status gpq_astar_gcost(gpq_astar* a, uint32_t index, uint32_t* g, uint64_t capacity, void* stream);

/* Headless image of instance `index` of the last solve (the reference's path image,
 * dumpResult in src/a_star.cu:596-690, without its GL or agent map): a binary PPM file
 * (P6), one pixel per cell, row 0 at the top, colours: free unreached black, blocked grey
 * (90,90,90), reached but above the optimal cost dark blue (0,0,110), expanded
 * (g + h <= C*) light blue (60,140,255), canonical path red (255,40,40), start green
 * (0,220,0), goal yellow (255,230,0).  Grids up to 2^28 cells.  Blocks on the stream. */
GPQ_API gpq_status gpq_astar_write_ppm(gpq_astar* a, uint32_t index, const char* filename, void* stream);

/* Resident A* instances for serving.  No counterpart in the reference, whose agents run
 * to completion inside one a_star launch (src/a_star.cu:269-593).  A session reserves a
 * cell space (max_cells: g values, predecessor moves and blocked bits, 5.125 bytes a cell) and a tile space
 * (max_tiles tile records with their inboxes and open arrays) once; admitted instances
 * take free ranges of both, all running instances advance together, a bounded number of
 * rounds per step (one persistent launch), and finished ones are collected and give
 * their ranges back.  Between steps everything stays in device memory. */
typedef struct gpq_astar_session gpq_astar_session;

GPQ_API gpq_status gpq_astar_session_create(const gpq_astar_config* cfg, uint64_t max_cells, uint32_t max_tiles,
                                            uint32_t max_instances, gpq_astar_session** out);
GPQ_API gpq_status gpq_astar_session_destroy(gpq_astar_session* s);

/* Admit one instance; *slot names it until it is collected.  GPQ_ERR_NOMEM (and nothing
 * changes) when its cells or tiles do not fit in the free ranges now. */
GPQ_API gpq_status gpq_astar_session_admit(gpq_astar_session* s, const gpq_astar_grid* grid, uint32_t* slot);

/* Initialize the instances admitted since the last step, then advance every running
 * instance by at most `rounds` rounds (0 = until all are done).  *running = instances
 * admitted and not yet collected.  Blocks on the stream. */
GPQ_API gpq_status gpq_astar_session_step(gpq_astar_session* s, uint32_t rounds, uint32_t* running, void* stream);

/* Results of up to `capacity` finished instances (HOST arrays), which leave the session.
 * *n = how many. */
GPQ_API gpq_status gpq_astar_session_collect(gpq_astar_session* s, uint32_t* slots, gpq_astar_result* results,
                                             uint32_t capacity, uint32_t* n, void* stream);

/* Cells and tiles held by admitted instances, and their number. */
GPQ_API gpq_status gpq_astar_session_usage(gpq_astar_session* s, uint64_t* cells_used, uint64_t* tiles_used,
                                           uint32_t* instances);

/* Device bytes a session of these sizes reserves. */
GPQ_API uint64_t gpq_astar_session_bytes(const gpq_astar_config* cfg, uint64_t max_cells, uint32_t max_tiles,
                                         uint32_t max_instances);

/* Grid of query `index` of a batch: side log-uniform in [side_lo, side_hi], obstacle
 * density uniform in [dens_lo, dens_hi], start and goal distinct and uniform over the
 * free cells, all drawn from seed base_seed + index (host computation). */
GPQ_API gpq_status gpq_astar_query(uint64_t base_seed, uint32_t index, uint32_t conn, uint32_t side_lo,
                                   uint32_t side_hi, double dens_lo, double dens_hi, gpq_astar_grid* out);

/* Resident PHOLD instances: many runs of different sizes in one persistent launch
 * (batched runs, and the PHOLD side of serving).  No counterpart in the reference, which
 * runs one model per process (src/des.cu:74-214).  A session reserves an LP space of
 * max_lps local array queues (capacity items each, insert_capacity children per window)
 * once; an admitted run takes a free LP range, and all running instances advance
 * together one window per grid barrier, each inside its own safe window
 * [min_i, min_i + lookahead_i), so each run commits exactly what it commits alone (same
 * committed count, steps, digest, pending events).  Finished runs are collected and give
 * their LPs back. */
typedef struct gpq_phold_session gpq_phold_session;

GPQ_API gpq_status gpq_phold_session_create(uint32_t max_lps, uint32_t capacity, uint32_t insert_capacity,
                                            uint32_t max_instances, uint32_t lanes_per_lp,
                                            gpq_phold_session** out);
/* A session whose LP space holds time buckets instead of sorted rings (the bucketed local
 * array queue, gpq_phold_config.laq_mode 2): `buckets` buckets of `bucket_slots` keys per
 * LP (powers of two; 0 = 32 and 16) and spill lists of max(64, bucket_slots) keys.  An
 * admitted run gets a bucket width from its lookahead and events_per_lp; a run whose
 * lookahead needs more buckets is refused (GPQ_ERR_INVALID).  Same results as the sorted
 * form. */
GPQ_API gpq_status gpq_phold_session_create_bucketed(uint32_t max_lps, uint32_t buckets, uint32_t bucket_slots,
                                                     uint32_t max_instances, gpq_phold_session** out);
GPQ_API gpq_status gpq_phold_session_destroy(gpq_phold_session* s);

/* Admit one run (its queue_kind, capacity, insert_capacity and loop fields are ignored:
 * the session's local array queues are used); GPQ_ERR_NOMEM when its LPs do not fit now. */
GPQ_API gpq_status gpq_phold_session_admit(gpq_phold_session* s, const gpq_phold_config* cfg, uint32_t* slot);

/* Populate the runs admitted since the last step, then advance every running instance by
 * at most `windows` windows (0 = until all are done).  Blocks on the stream. */
GPQ_API gpq_status gpq_phold_session_step(gpq_phold_session* s, uint32_t windows, uint32_t* running, void* stream);

/* Results of up to `capacity` finished runs (HOST arrays; elapsed_ms is 0), which leave
 * the session. */
GPQ_API gpq_status gpq_phold_session_collect(gpq_phold_session* s, uint32_t* slots, gpq_phold_result* results,
                                             uint32_t capacity, uint32_t* n, void* stream);
GPQ_API gpq_status gpq_phold_session_usage(gpq_phold_session* s, uint64_t* lps_used, uint32_t* instances);
/* Whole-session state between steps: every resident run (queues, per-LP checksums, window
 * counters, slots, the LP-range allocator), so a serving process can stop and resume, or
 * branch several continuations from one point.  Admissions not yet started are started
 * first, at the session's next window, as the next step would start them.  Per-LP arrays
 * are saved up to the highest LP in use.  A snapshot restores into a session created with
 * the same parameters, whatever that session holds; it then steps and collects exactly as
 * the original would have.  With buf == NULL the snapshot only reports its size.  Both
 * block on the stream. */
GPQ_API gpq_status gpq_phold_session_snapshot(gpq_phold_session* s, void* buf, uint64_t capacity, uint64_t* size,
                                              void* stream);
GPQ_API gpq_status gpq_phold_session_restore(gpq_phold_session* s, const void* buf, uint64_t size, void* stream);
GPQ_API uint64_t gpq_phold_session_bytes(uint32_t max_lps, uint32_t capacity, uint32_t insert_capacity,
                                         uint32_t max_instances);
GPQ_API uint64_t gpq_phold_session_bytes_bucketed(uint32_t max_lps, uint32_t buckets, uint32_t bucket_slots,
                                                  uint32_t max_instances);

/* ---------------------------------------------------------------------------------- */
/* 2c. Serving: a stream of A* queries and PHOLD runs                                  */
/* ---------------------------------------------------------------------------------- */

#define GPQ_REQ_ASTAR 0u
#define GPQ_REQ_PHOLD 1u
#define GPQ_SERVE_BATCHED 0u /* continuous batching over the resident sessions */
#define GPQ_SERVE_PLAIN 1u   /* one request per launch, in arrival order */

typedef struct gpq_serve_request {
  double arrival;  /* seconds after the stream starts */
  uint32_t kind;   /* GPQ_REQ_ASTAR or GPQ_REQ_PHOLD */
  uint32_t reserved;
  gpq_astar_grid astar;
  gpq_phold_config phold;
} gpq_serve_request;

typedef struct gpq_serve_response {
  double admitted; /* seconds after the start when the request got its resources */
  double finished; /* seconds after the start when its result was on the host */
  int32_t status;  /* gpq_status of the request */
  uint32_t reserved;
  gpq_astar_result astar;
  gpq_phold_result phold; /* elapsed_ms is 0 in batched mode */
} gpq_serve_response;

typedef struct gpq_serve_config {
  uint64_t hbm_budget;            /* device bytes for resident request state; 0 = 120 GiB */
  uint32_t mode;                  /* GPQ_SERVE_BATCHED or GPQ_SERVE_PLAIN */
  uint32_t realtime;              /* 1: admit no request before its arrival (host clock);
                                     0: every request has arrived at the start */
  uint32_t astar_rounds;          /* A* rounds per step; 0 = 32 */
  uint32_t phold_windows;         /* PHOLD windows per step; 0 = 32 */
  double astar_share;             /* part of the budget for A* state; 0 = 0.75 */
  gpq_astar_config astar;
  uint32_t phold_capacity;        /* per-LP queue capacity; 0 = 256 */
  uint32_t phold_insert_capacity; /* per-LP children per window; 0 = 64 */
  uint32_t phold_lanes_per_lp;    /* sorted form: lanes per LP; 0 = 8 */
  uint32_t phold_form;            /* 0 = sorted rings, 1 = time buckets (gpq_phold_session_create_bucketed) */
  uint32_t reserved[4];
} gpq_serve_config;

typedef struct gpq_serve_stats {
  double makespan;   /* seconds from the start to the last result */
  double throughput; /* requests per second of makespan */
  double p50, p99, p999; /* latency (finished - arrival) percentiles in seconds */
  uint64_t steps;    /* engine steps (batched) or launches (plain) */
  uint32_t max_resident;
  uint32_t reserved;
} gpq_serve_stats;

/* Serve n requests (HOST arrays).  Batched: requests are admitted in arrival order as
 * long as their state fits the budget (A* cells and tiles, PHOLD LPs), stay resident,
 * and advance together step by step; each result equals the request's result alone.
 * Plain: each request runs alone with its own launch (gpq_astar_solve, gpq_phold_run),
 * one after another.  A request that can never fit reports GPQ_ERR_NOMEM. */
GPQ_API gpq_status gpq_serve_run(const gpq_serve_config* cfg, const gpq_serve_request* reqs, uint32_t n,
                                 gpq_serve_response* out, gpq_serve_stats* stats);

/* The mixed request stream: Poisson arrivals at `rate` per second for `duration`
 * seconds; a request is an A* query with probability astar_fraction (4-connected, unit
 * costs, side log-uniform in [128, 4096], obstacle density 0.2, gpq_astar_query with
 * base seed `seed`), else a PHOLD run (LPs log-uniform in [256, 65536], 32 events per
 * LP, lookahead 0.5, end time 200, uniform destinations, seed + index).  Writes up to
 * `capacity` requests; with out == NULL only counts them. */
GPQ_API gpq_status gpq_serve_stream(uint64_t seed, double rate, double duration, double astar_fraction,
                                    gpq_serve_request* out, uint32_t capacity, uint32_t* n);

/* Page-locked host memory for the end-to-end path (host <-> device copies). */
GPQ_API gpq_status gpq_host_alloc(uint64_t bytes, void** out);
GPQ_API gpq_status gpq_host_free(void* p);

/* Device-side timeout of bounded waits (grid barrier spins), in spin iterations. */
GPQ_API gpq_status gpq_set_spin_limit(uint64_t iterations);

/* ---------------------------------------------------------------------------------- */
/* 2c. Reference-semantics A* (the reference's agent model, src/a_star.cu:124-593)     */
/* ---------------------------------------------------------------------------------- */

/* Semantics in include/gpq/astar_ref.h: half-precision f, eight pops per round, 3 x 3
 * exploration with clamped coordinates, de-duplication and the f_ol filter, stop when
 * the goal is popped, a pool of agents handed to concurrent slots (get_new_agent); ties
 * of (f, h) go by cell id, so results are deterministic.  Agents are independent, so
 * each slot (one warp) runs its agents to completion inside one persistent launch --
 * the reference launches one kernel per round for all agents. */
typedef struct gpq_astar_ref gpq_astar_ref;

typedef struct gpq_astar_ref_config {
  uint32_t width, height;   /* map size (A_STAR_GRID_X, A_STAR_GRID_Y) */
  uint32_t slots;           /* concurrent agents (NUM_CONCURRENT_AGENTS); 0 = 2048 */
  uint32_t open_capacity;   /* open-list items per slot; 0 = 4 * width * height */
  uint32_t reserved[4];
} gpq_astar_ref_config;

typedef struct gpq_astar_ref_agent {
  uint32_t start, goal;     /* cells (y * width + x) */
} gpq_astar_ref_agent;

typedef struct gpq_astar_ref_result {
  uint32_t found;           /* the goal was popped */
  float cost;               /* its f (half precision, as a float) when popped */
  uint32_t pops;            /* vertices popped, duplicates included */
  uint32_t rounds;          /* rounds of at most eight pops */
  uint32_t status;          /* gpq_status; GPQ_ERR_QUEUE_FULL: open_capacity too small */
  uint32_t reserved;
} gpq_astar_ref_result;

GPQ_API gpq_status gpq_astar_ref_create(const gpq_astar_ref_config* cfg, gpq_astar_ref** out);
GPQ_API gpq_status gpq_astar_ref_destroy(gpq_astar_ref* h);
/* Runs the n agents (HOST arrays) on the map (HOST, width * height bytes, non-zero =
 * wall); results in agent order.  Blocks on the stream. */
GPQ_API gpq_status gpq_astar_ref_solve(gpq_astar_ref* h, const uint8_t* map, const gpq_astar_ref_agent* agents,
                                       uint32_t n, gpq_astar_ref_result* results, void* stream);
/* Device time of the last solve's search kernel (CUDA events). */
GPQ_API gpq_status gpq_astar_ref_last_ms(gpq_astar_ref* h, float* ms);
/* The reference's random map (src/a_star.cu:747-765): obstacle_frac * width * height
 * squares at uniform positions, side max(1, (int)(size_mean * Exp(1))), drawn from seed. */
GPQ_API gpq_status gpq_astar_ref_map(uint32_t width, uint32_t height, float obstacle_frac, float size_mean,
                                     uint64_t seed, uint8_t* map);
/* n agents with uniformly random free start and goal cells (src/a_star.cu:768-789). */
GPQ_API gpq_status gpq_astar_ref_agents(const uint8_t* map, uint32_t width, uint32_t height, uint32_t n,
                                        uint64_t seed, gpq_astar_ref_agent* out);

/* ---------------------------------------------------------------------------------- */
/* 3. Utilities                                                                       */
/* ---------------------------------------------------------------------------------- */

GPQ_API const char* gpq_status_string(gpq_status s);
GPQ_API const char* gpq_version(void);
/* Human-readable text of the last error seen on this thread (static storage). */
GPQ_API const char* gpq_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* GPQ_H */
