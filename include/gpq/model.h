/*
 * gpq/model.h -- event semantics shared by the host and device code of gpupq_b200.
 *
 * Everything here is a pure function of its arguments and is evaluated with
 * single IEEE-754 float operations (no FMA contraction: device code uses the
 * explicit __f*_rn intrinsics, host code is compiled with -ffp-contract=off),
 * so the host and the GPU produce the same bits.
 *
 * Item layout.  The reference's PHOLD item is `struct event { long ts; int node; }`
 * (src/queue_item.h:13-16), 16 bytes with padding, ordered by `ts` only
 * (src/queue_item.h:20-26).  Here an item is 16 bytes packed as
 * (float ts, uint32 lp, uint32 id, uint32 aux) so that a lane moves one item with
 * one 16-byte vector load; the order is the strict total order
 * (ts bits, lp, id), which equals the reference's `<` wherever the reference's
 * order is defined and breaks its ties deterministically.
 *
 * PHOLD event function.  The reference draws the child's node and time from a
 * per-LP curand state (src/phold.cu:81-117).  Here the child is a pure function
 * of the parent event (seed, id, ts bits): its random draws come from a
 * counter-based generator built on the SplitMix64 finaliser (Steele, Lea and
 * Flood, "Fast splittable pseudorandom number generators", OOPSLA 2014), and
 * Exp(1) is -ln(u) with the logarithm computed by the atanh series
 * ln(m) = 2*atanh((m-1)/(m+1)) after range reduction to m in [sqrt(1/2), sqrt(2)).
 * The child keeps its parent's id (the population is conserved, one child per
 * event as in src/phold.cu:103-114), so an event's result does not depend on
 * the order in which a step processes the events.
 */
#ifndef GPQ_MODEL_H
#define GPQ_MODEL_H

#include <stdint.h>
#if !defined(__CUDACC__)
#include <string.h>
#endif

#if defined(__CUDACC__)
#define GPQ_HD __host__ __device__ __forceinline__
#else
#define GPQ_HD static inline
#endif

#if defined(__CUDA_ARCH__)
#define GPQ_FADD(a, b) __fadd_rn((a), (b))
#define GPQ_FSUB(a, b) __fsub_rn((a), (b))
#define GPQ_FMUL(a, b) __fmul_rn((a), (b))
#define GPQ_FDIV(a, b) __fdiv_rn((a), (b))
#else
#define GPQ_FADD(a, b) ((a) + (b))
#define GPQ_FSUB(a, b) ((a) - (b))
#define GPQ_FMUL(a, b) ((a) * (b))
#define GPQ_FDIV(a, b) ((a) / (b))
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* One queue item: 16 bytes, 16-byte aligned. */
typedef struct
#if defined(__CUDACC__)
__align__(16)
#endif
gpq_item {
  float ts;      /* timestamp (PHOLD) */
  uint32_t lp;   /* owning logical process (the queue it lives in) */
  uint32_t id;   /* event id: unique among live events of one run */
  uint32_t aux;  /* payload: the LP that created the event (PHOLD) */
} gpq_item;

#ifdef __cplusplus
}
#endif

#define GPQ_GOLDEN64 0x9E3779B97F4A7C15ULL
#define GPQ_TS_INIT_DOMAIN 0xFFFFFFFFu /* ts bits used to key the initial draws (a NaN pattern, never a real ts) */

GPQ_HD uint32_t gpq_f2u(float x) {
#if defined(__CUDA_ARCH__)
  return __float_as_uint(x);
#else
  uint32_t u; memcpy(&u, &x, 4); return u;
#endif
}

GPQ_HD float gpq_u2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float x; memcpy(&x, &u, 4); return x;
#endif
}

/* Strict total order on items: (ts bits, lp, id).  Timestamps are finite and
 * non-negative, so comparing their bit patterns as unsigned integers is the
 * same as comparing them as floats. */
GPQ_HD int gpq_item_less(const gpq_item a, const gpq_item b) {
  uint32_t ta = gpq_f2u(a.ts), tb = gpq_f2u(b.ts);
  if (ta != tb) return ta < tb;
  if (a.lp != b.lp) return a.lp < b.lp;
  return a.id < b.id;
}

/* 64-bit key that orders the items of ONE LP's queue exactly like gpq_item_less
 * (lp is constant inside a per-LP queue). */
GPQ_HD uint64_t gpq_lp_key(const gpq_item a) {
  return ((uint64_t)gpq_f2u(a.ts) << 32) | (uint64_t)a.id;
}

/* SplitMix64 finaliser (bijective 64-bit mixer). */
GPQ_HD uint64_t gpq_mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

/* Counter-based draw #`draw` for the event (seed, id, ts_bits). */
GPQ_HD uint64_t gpq_draw(uint64_t seed, uint32_t id, uint32_t ts_bits, uint32_t draw) {
  uint64_t k = gpq_mix64(seed ^ ((uint64_t)id * GPQ_GOLDEN64));
  return gpq_mix64(k ^ (((uint64_t)ts_bits << 8) | (uint64_t)(draw & 0xffu)));
}

/* Uniform in (0, 1]: the top 24 bits of a draw, plus one, times 2^-24 (exact). */
GPQ_HD float gpq_unit_open0(uint64_t r) {
  uint32_t u24 = (uint32_t)(r >> 40);
  return GPQ_FMUL((float)(u24 + 1u), 5.9604644775390625e-8f);
}

/* Natural logarithm of a positive normal float, own implementation:
 * x = 2^e * m with m in [sqrt(1/2), sqrt(2)), s = (m-1)/(m+1),
 * ln(m) = 2*(s + s^3/3 + s^5/5 + s^7/7 + s^9/9) (atanh series), evaluated in
 * Horner form with one rounding per operation. */
GPQ_HD float gpq_logf(float x) {
  uint32_t b = gpq_f2u(x);
  int e = (int)((b >> 23) & 0xffu) - 127;
  float m = gpq_u2f((b & 0x007fffffu) | 0x3f800000u);
  if (m > 1.41421354f) {
    m = GPQ_FMUL(m, 0.5f);
    e += 1;
  }
  float s = GPQ_FDIV(GPQ_FSUB(m, 1.0f), GPQ_FADD(m, 1.0f));
  float z = GPQ_FMUL(s, s);
  float p = 0.222222224f;                      /* 2/9 */
  p = GPQ_FADD(GPQ_FMUL(p, z), 0.285714298f);  /* 2/7 */
  p = GPQ_FADD(GPQ_FMUL(p, z), 0.400000006f);  /* 2/5 */
  p = GPQ_FADD(GPQ_FMUL(p, z), 0.666666687f);  /* 2/3 */
  p = GPQ_FADD(GPQ_FMUL(p, z), 2.0f);
  float lm = GPQ_FMUL(s, p);
  return GPQ_FADD(GPQ_FMUL((float)e, 0.693147182f), lm);
}

/* Exp(1) sample from a draw: 0 - ln(u), u in (0, 1]; result in [+0, 16.64]
 * (written as a subtraction so that u == 1 gives +0, never -0). */
GPQ_HD float gpq_exp1(uint64_t r) {
  return GPQ_FSUB(0.0f, gpq_logf(gpq_unit_open0(r)));
}

/* Uniform integer in [0, n) by multiply-shift of the high 32 bits. */
GPQ_HD uint32_t gpq_uniform_below(uint64_t r, uint32_t n) {
  return (uint32_t)(((r >> 32) * (uint64_t)n) >> 32);
}

/* Destination rules. */
#define GPQ_DEST_UNIFORM 0u /* uniform over all LPs */
#define GPQ_DEST_RING 1u    /* with probability ring_threshold/2^32 a neighbour within
                               +-ring_width on the ring (self excluded), else uniform */

typedef struct gpq_phold_params {
  uint64_t seed;
  uint32_t num_lps;
  uint32_t dest_mode;
  uint32_t ring_width;
  uint32_t ring_threshold;
  float lookahead;
  float end_time;
} gpq_phold_params;

GPQ_HD uint32_t gpq_phold_dest(const gpq_phold_params p, uint32_t lp, uint64_t r) {
  if (p.dest_mode == GPQ_DEST_RING && (uint32_t)r < p.ring_threshold) {
    uint32_t w = p.ring_width;
    uint32_t k = gpq_uniform_below(r, 2u * w);            /* [0, 2w) */
    int32_t off = (k < w) ? (int32_t)k - (int32_t)w : (int32_t)k - (int32_t)w + 1;
    /* (lp + off) mod num_lps; 2w < num_lps, so one correction step is exact */
    int64_t d = (int64_t)lp + off;
    if (d < 0) d += p.num_lps;
    else if (d >= (int64_t)p.num_lps) d -= p.num_lps;
    return (uint32_t)d;
  }
  return gpq_uniform_below(r, p.num_lps);
}

/* The child of event `ev` (the reference's handle_next_event body, src/phold.cu:95-114):
 * ts' = ts + (lookahead + Exp(1)), lp' from the destination rule, id' = id. */
GPQ_HD gpq_item gpq_phold_child(const gpq_phold_params p, const gpq_item ev) {
  uint32_t tb = gpq_f2u(ev.ts);
  uint64_t r0 = gpq_draw(p.seed, ev.id, tb, 0);
  uint64_t r1 = gpq_draw(p.seed, ev.id, tb, 1);
  float delta = GPQ_FADD(p.lookahead, gpq_exp1(r1));
  gpq_item c;
  c.ts = GPQ_FADD(ev.ts, delta);
  c.lp = gpq_phold_dest(p, ev.lp, r0);
  c.id = ev.id;
  c.aux = ev.lp;
  return c;
}

/* Initial event k of LP `lp` (fixed count per LP): id = lp*per_lp + k, ts = Exp(1). */
GPQ_HD gpq_item gpq_phold_initial(const gpq_phold_params p, uint32_t lp, uint32_t k, uint32_t per_lp) {
  gpq_item e;
  e.id = lp * per_lp + k;
  e.lp = lp;
  e.aux = lp;
  e.ts = gpq_exp1(gpq_draw(p.seed, e.id, GPQ_TS_INIT_DOMAIN, 0));
  return e;
}

/* Per-event hashes for the LP outputs.
 * csum  (order-insensitive): sum over committed events of ev_hash.
 * ohash (order-sensitive):   sum over committed events of mix64(ev_hash + seq*golden),
 *                            seq = the event's 0-based position in its LP's sequence. */
GPQ_HD uint64_t gpq_ev_hash(uint32_t id, uint32_t ts_bits) {
  return gpq_mix64(((uint64_t)id << 32) | (uint64_t)ts_bits);
}

GPQ_HD uint64_t gpq_seq_hash(uint64_t ev_hash, uint64_t seq) {
  return gpq_mix64(ev_hash + seq * GPQ_GOLDEN64);
}

#endif /* GPQ_MODEL_H */
