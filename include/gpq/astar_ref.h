/*
 * gpq/astar_ref.h -- the reference's own A* semantics (src/a_star.cu:124-593), for the
 * reference-semantics A* mode (gpq_astar_ref_*), shared by the host and device code.
 *
 * Unlike the exact A* of gpq/astar.h, this mode reproduces what the reference's agents
 * compute, step for step:
 *   map      one W x H obstacle map shared by all agents (src/a_star.cu:747-765 draws
 *            random squares; gpq_astar_ref_map draws them with this project's RNG);
 *   agents   a pool of agents (start, goal) handed to concurrent slots as slots free up
 *            (get_new_agent, src/a_star.cu:150-164);
 *   h        octile distance in float: sqrt(2) * min(dx, dy) + max - min, evaluated in
 *            double and rounded to float (src/a_star.cu:124-135);
 *   f        half precision: a neighbour's g = f(cur) - h(cur, goal) + h(cur, nb) in float,
 *            f(nb) = half(g + h(nb, goal)) (src/a_star.cu:487-496);
 *   round    pop min(open-list length, 8) vertices (A_STAR_MAX_PARALLEL_OL_ENTRIES) and
 *            close them; if one of them is the goal, the agent ends (found); else every
 *            popped vertex explores the 8 cells of its 3 x 3 square, coordinates clamped
 *            to the map (src/a_star.cu:384-399), keeping cells that are neither closed nor
 *            walls; duplicates within the round keep the smallest f (src/a_star.cu:
 *            508-530); a cell enters the open list only if its f beats the best f it was
 *            ever inserted with (f_ol, src/a_star.cu:537-560); an agent whose open list
 *            is empty after a round ends without a path;
 *   order    the open list pops by f, then by h(cell, goal) (src/queue_item.h:56-73); the
 *            reference leaves equal (f, h) in insertion order, which depends on its
 *            thread schedule -- here such ties go by cell id, so every result is a
 *            function of the map and the agent.
 * Outputs per agent: found, the goal's f when popped (the path cost estimate), popped
 * vertices (duplicates included) and rounds.
 */
#ifndef GPQ_ASTAR_REF_H
#define GPQ_ASTAR_REF_H

#include "gpq/model.h"

#define GPQ_ASTAR_REF_POPS 8u  /* A_STAR_MAX_PARALLEL_OL_ENTRIES (src/config.h) */

#if defined(__CUDA_ARCH__)
#define GPQ_DMUL(a, b) __dmul_rn((a), (b))
#define GPQ_DADD(a, b) __dadd_rn((a), (b))
#define GPQ_DSUB(a, b) __dsub_rn((a), (b))
#else
#define GPQ_DMUL(a, b) ((a) * (b))
#define GPQ_DADD(a, b) ((a) + (b))
#define GPQ_DSUB(a, b) ((a) - (b))
#endif

/* h (src/a_star.cu:124-135): sqrt(2) * min + max - min in double, rounded to float. */
GPQ_HD float gpq_astar_ref_h(int x0, int y0, int x1, int y1) {
  const int dx = x0 > x1 ? x0 - x1 : x1 - x0, dy = y0 > y1 ? y0 - y1 : y1 - y0;
  const int mn = dx < dy ? dx : dy, mx = dx < dy ? dy : dx;
  double t = GPQ_DMUL(1.4142135623730951, (double)mn);
  t = GPQ_DADD(t, (double)mx);
  t = GPQ_DSUB(t, (double)mn);
  return (float)t;
}

/* IEEE 754 binary16 <-> binary32 for non-negative finite values, round to nearest even
 * (the conversion __float2half performs); written from the format definition. */
GPQ_HD uint32_t gpq_f32_to_f16_bits(float f) {
  const uint32_t u = gpq_f2u(f);
  const uint32_t sign = (u >> 16) & 0x8000u;
  const int e = (int)((u >> 23) & 0xffu) - 127;
  uint32_t m = u & 0x7fffffu;
  if (e > 15) return sign | 0x7c00u;                 /* overflow (and inf/nan) -> inf */
  if (e >= -14) {                                    /* normal half */
    uint32_t h = sign | ((uint32_t)(e + 15) << 10) | (m >> 13);
    const uint32_t rem = m & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h += 1u;  /* carries into the exponent */
    return h;
  }
  if (e < -25) return sign;                          /* below half the smallest subnormal */
  m |= 0x800000u;                                    /* subnormal half: value = m * 2^(e-23) */
  const int shift = -e - 1;                          /* (m >> shift) counts units of 2^-24 */
  uint32_t h = sign | (m >> shift);
  const uint32_t rem = m & ((1u << shift) - 1u), half = 1u << (shift - 1);
  if (rem > half || (rem == half && (h & 1u))) h += 1u;
  return h;
}

GPQ_HD float gpq_f16_bits_to_f32(uint32_t h) {
  const uint32_t sign = (h & 0x8000u) << 16;
  const uint32_t e = (h >> 10) & 0x1fu, m = h & 0x3ffu;
  if (e == 0x1fu) return gpq_u2f(sign | 0x7f800000u | (m << 13));
  if (e != 0) return gpq_u2f(sign | ((e + 112u) << 23) | (m << 13));
  if (m == 0) return gpq_u2f(sign);
  /* subnormal: m * 2^-24 */
  return GPQ_FMUL((float)m, 5.9604644775390625e-8f) * (sign ? -1.0f : 1.0f);
}

/* Open-list key of a vertex: (f half bits, h float bits, cell), compared as unsigned
 * integers (f and h are >= +0, so bit order is value order). */
GPQ_HD uint64_t gpq_astar_ref_key(uint32_t f_half, float h) {
  return ((uint64_t)f_half << 32) | (uint64_t)gpq_f2u(h);
}

#endif /* GPQ_ASTAR_REF_H */
