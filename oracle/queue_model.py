"""Queue-level semantic model of the reference's five queues (test infrastructure only).

A pure-Python restatement, for small cases, of what the reference's queue plugin
contract (src/queue.h:86-115, src/queue.cuh:46-70) guarantees at its boundary,
independent of each queue's internal layout:

  * queue_insert(item) puts the item into its LP's queue (src/local_array_queue.cu:486-513,
    src/global_array_queue.cu:347-365, src/heap_queue.cu:1809-1826, src/local_heap_queue.cu:398-419,
    src/local_splay_queue.cu:275-292); it becomes visible after queue_post;
  * queue_get_min_ts returns the smallest timestamp of all queued items
    (src/local_array_queue.cu:460-478, src/heap_queue.cu:1783-1806);
  * a step dequeues, per LP, the earliest items whose timestamp lies below the window
    bound (min + LOOKAHEAD), at most `max_per_lp` of them (the reference takes one per LP:
    src/phold.cu:84-94, src/global_array_queue.cu:147-179, src/heap_queue.cu:478-547);
  * items are ordered by timestamp; the rebuild breaks ties by (ts bits, LP, id);
  * the heap queue takes its candidates from the root only: the reference stops its scan
    of the merged buffer at the root's maximum (src/heap_queue.cu:1588-1592, "the next
    event for an LP is not in the root but in a child node"), and the root of a heap in
    order holds the `root_size` globally smallest items (`root_size` = node size).

Used to check the reference's own known-answer vectors (tests/golden/reference_kats.json)
and, on the GPU, the rebuilt queues against the same semantics.
"""
import struct


def ts_bits(ts: float) -> int:
    return struct.unpack("<I", struct.pack("<f", ts))[0]


def key(item):
    """item = (ts, lp, id)"""
    ts, lp, iid = item[0], item[1], item[2]
    return (ts_bits(ts), lp, iid)


class QueueModel:
    def __init__(self, num_lps: int, root_size: int = 0):
        self.num_lps = num_lps
        self.root_size = root_size  # 0: every queued item is a candidate
        self.lps = [[] for _ in range(num_lps)]
        self.pending = []
        self.enqueued = 0
        self.dequeued = 0

    def insert(self, ts: float, lp: int, iid: int):
        self.pending.append((float(ts), int(lp), int(iid)))
        self.enqueued += 1

    def post(self):
        for it in self.pending:
            self.lps[it[1]].append(it)
        self.pending = []
        for q in self.lps:
            q.sort(key=key)

    def get_min(self) -> float:
        heads = [q[0][0] for q in self.lps if q]
        return min(heads) if heads else float("inf")

    def dequeue(self, bound: float, max_per_lp: int = 0):
        limit = [len(q) for q in self.lps]
        if self.root_size:
            limit = [0] * self.num_lps
            for it in self.global_items()[: self.root_size]:
                limit[it[1]] += 1
        out = []
        for lp, q in enumerate(self.lps):
            n = 0
            while q and n < limit[lp] and q[0][0] < bound and (max_per_lp == 0 or n < max_per_lp):
                out.append(q.pop(0))
                n += 1
        self.dequeued += len(out)
        return out

    def lp_items(self, lp: int):
        return list(self.lps[lp])

    def global_items(self):
        allit = [it for q in self.lps for it in q]
        return sorted(allit, key=key)

    def length(self, lp: int) -> int:
        return len(self.lps[lp])

    def clear(self, lp: int):
        self.dequeued += len(self.lps[lp])
        self.lps[lp] = []
