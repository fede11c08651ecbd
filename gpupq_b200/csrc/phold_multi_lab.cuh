// Many PHOLD runs in one persistent launch over the bucketed local array queue (batched
// and served PHOLD; the single-run form is lab.cuh).
//
// The runs share one LP space as in phold_multi.cuh (run i owns LPs [lp0_i, lp0_i + L_i),
// every LP knows its run, each run advances inside its own window), and every LP holds
// the time buckets of lab.cuh.  The LP space is split evenly over all warps of the grid;
// a warp walks its share in chunks of LPs of one run (lab_chunk_lps of the run, at most
// kLabWarpLps) and processes each
// chunk with the single-run warp window (lab_warp_window) under that run's window: its
// minimum, bound, end time, bucket width (runs may differ) and bucket history.  A chunk
// folds its minimum into its run's slot with one atomic.
//
// Per run: the bucket width in PmInstDev::aux, the top bucket of its last four windows
// (wj), and the minimum at its first inactive window (fin), which the finalisation uses
// to tell its pending keys from the dead ones after other runs have moved the window
// slots on.
#pragma once

#include "lab.cuh"
#include "phold_multi.cuh"

struct PmbDev {
  LabDev q;       // buckets, counts and spill lists of the LP space (q.wj, q.inv_w unused)
  uint32_t* wj;   // [max_inst * 4] top bucket of run i's window s in wj[4 i + (s & 3)]
  uint32_t* fin;  // [max_inst] run i's minimum at its first inactive window (~0u: not reached yet)
};

__device__ __forceinline__ float pmb_inv_w(const PmInstDev& I) { return __uint_as_float(I.aux); }

// Windows s0, s0 + 1, ... while some run is active, at most step_windows of them (0 = no
// limit).  Dynamic shared memory: lab_cta_smem_bytes(blockDim.x).
static __global__ void __launch_bounds__(1024, 1) pmb_persistent_kernel(PmDev d, PmbDev b, uint32_t s0,
                                                                        uint32_t step_windows) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_any;
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u, nw = blockDim.x >> 5;
  const LabWarpSmem sm = lab_warp_smem(smem_raw + (size_t)warp * lab_warp_smem_bytes());
  const uint32_t gw = blockIdx.x * nw + warp, ngw = gridDim.x * nw;
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
  unsigned long long target = 0;
  uint32_t s = s0;
  for (;; ++s) {
    // every block takes the same decision from the same slots
    if (threadIdx.x == 0) s_any = 0;
    __syncthreads();
    int any = 0;
    for (uint32_t i = threadIdx.x; i < d.n_inst && !any; i += blockDim.x) any = pm_active(d, i, s);
    if (any) s_any = 1;
    __syncthreads();
    if (!s_any || ld_relaxed_u32(&d.ctl->err) != 0u || (step_windows && s - s0 >= step_windows)) break;
    for (uint32_t i = tid; i < d.n_inst; i += nthreads) {
      if (pm_active(d, i, s)) {
        PmInstDev& I = d.inst[i];
        I.windows += 1u;
        const float m = gpq_u2f(ld_relaxed_u32(&d.mins[3 * i + s % 3u]));
        b.wj[4 * i + (s & 3u)] = lab_bucket(gpq_f2u(GPQ_FADD(m, I.p.lookahead)), pmb_inv_w(I));
      } else if (d.on[i] && d.inst[i].w0 + d.inst[i].windows == s) {
        b.fin[i] = ld_relaxed_u32(&d.mins[3 * i + s % 3u]);  // first inactive window
      }
      d.mins[3 * i + (s + 2u) % 3u] = kInfBits;  // slots of window s + 2, last read in window s - 1
      d.errs[3 * i + (s + 2u) % 3u] = 0u;
    }
    // this warp's share of the LP space, in chunks of one run
    const uint32_t pw = (d.n_lps + ngw - 1u) / ngw;
    const uint32_t lo = min(d.n_lps, gw * pw), hi = min(d.n_lps, lo + pw);
    for (uint32_t pos = lo; pos < hi;) {
      uint32_t span = min(hi - pos, kLabWarpLps);
      const uint32_t own = (lane < span) ? d.lp_inst[pos + lane] : 0u;
      const uint32_t i0 = __shfl_sync(GPQ_FULL_MASK, own, 0);
      if (i0 != ~0u) {
        const PmInstDev& I = d.inst[i0];
        span = min(span, lab_chunk_lps(I.p.lookahead, pmb_inv_w(I), I.per_lp));
      }
      const uint32_t diff = __ballot_sync(GPQ_FULL_MASK, lane < span && own != i0);
      const uint32_t n = diff ? (uint32_t)__ffs(diff) - 1u : span;
      if (i0 != ~0u && pm_active(d, i0, s)) {
        const PmInstDev& I = d.inst[i0];
        const float m = gpq_u2f(ld_relaxed_u32(&d.mins[3 * i0 + s % 3u]));
        const LabWin w = lab_window_of(I.p, pmb_inv_w(I), s, m, ld_relaxed_u32(&b.wj[4 * i0 + ((s + 3u) & 3u)]));
        const LabCtx x{I.p, d.max_lps, I.lp0, &d.inst[i0].err, &d.errs[3 * i0 + (s + 1u) % 3u]};
        lab_state_load(d.count, d.csum, d.ohash, sm, pos, n);
        const uint32_t mn = warp_min_u32(lab_warp_window(x, b.q, w, pos, n, sm));
        lab_state_store(d.count, d.csum, d.ohash, sm, pos, n);
        if (lane == 0 && mn != kInfBits) atomicMin(&d.mins[3 * i0 + (s + 1u) % 3u], mn);
      }
      pos += n;
    }
    target += gridDim.x;
    if (!grid_barrier(&d.ctl->bar, target, d.spin_limit, &d.ctl->err)) {
      s += 1u;
      break;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) d.ctl->phase = s;
}

// Initial events of the runs in list[0, n) (blockIdx.y = position in the list), one warp
// per LP: the LP's buckets, counts and spill lists reset, its initial events (ids
// l * per_lp + k over local LPs l) filed into buckets [0, NB) or the spill list read by
// window s, per-LP outputs zeroed, the run's first minimum into its slot for window s.
static __global__ void pmb_populate_kernel(PmDev d, PmbDev b, const uint32_t* list, uint32_t s) {
  const uint32_t inst = list[blockIdx.y];
  const PmInstDev I = d.inst[inst];
  const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const uint32_t P = I.per_lp, NB = 1u << b.q.nb_log2, C = 1u << b.q.c_log2;
  const float inv_w = pmb_inv_w(I);
  const uint32_t pb = (s + 1u) & 1u;  // the spill list window s reads
  if (blockIdx.x == 0 && threadIdx.x < 4) b.wj[4 * inst + threadIdx.x] = 0u;
  if (blockIdx.x == 0 && threadIdx.x == 0) b.fin[inst] = ~0u;
  for (uint32_t l = blockIdx.x * wpb + wib; l < I.p.num_lps; l += gridDim.x * wpb) {
    const uint32_t lp = I.lp0 + l;
    const size_t lpb = (size_t)lp << b.q.nb_log2;
    for (uint32_t j = lane; j < NB; j += 32) b.q.cnt[lpb + j] = 0u;
    for (uint32_t j = lane; j < (NB << b.q.c_log2); j += 32) b.q.keys[(lpb << b.q.c_log2) + j] = ~0ull;
    if (lane < 2) b.q.scnt[(size_t)lane * d.max_lps + lp] = 0u;
    __syncwarp();
    uint32_t mn = kInfBits;
    for (uint32_t j = lane; j < P; j += 32) {
      const gpq_item e = gpq_phold_initial(I.p, l, j, P);
      const uint32_t tb = gpq_f2u(e.ts);
      const unsigned long long key = lab_key(tb, e.id);
      const uint32_t jb = lab_bucket(tb, inv_w);
      bool placed = false;
      if (jb < NB) {
        const uint32_t pos = atomicAdd(&b.q.cnt[lpb + jb], 1u);
        if (pos < C) {
          b.q.keys[((lpb + jb) << b.q.c_log2) + pos] = key;
          placed = true;
        }
      }
      if (!placed) {
        const size_t sl = (size_t)pb * d.max_lps + lp;
        const uint32_t pos = atomicAdd(&b.q.scnt[sl], 1u);
        if (pos < b.q.F) b.q.spill[sl * b.q.F + pos] = key;
        else gpq_set_error(&d.inst[inst].err, GPQ_ERR_QUEUE_FULL);
      }
      mn = min(mn, tb);
    }
    mn = warp_min_u32(mn);
    if (lane == 0) {
      d.count[lp] = 0;
      d.csum[lp] = 0;
      d.ohash[lp] = 0;
      d.lp_inst[lp] = inst;
      if (mn != kInfBits) atomicMin(&d.mins[3 * inst + s % 3u], mn);
    }
  }
}

// Results of the finished runs in list[0, n) (blockIdx.y = position in the list):
// committed count, pending events (the live keys of the buckets and the spill list of the
// run's last window), the digest over local LP numbers, the pending minimum.
static __global__ void pmb_finalize_kernel(PmDev d, PmbDev b, const uint32_t* list, PmAcc* acc) {
  const uint32_t j = blockIdx.y, inst = list[j];
  const PmInstDev I = d.inst[inst];
  const uint32_t lane = threadIdx.x & 31u, wpb = blockDim.x >> 5;
  const uint32_t s = I.w0 + I.windows;  // the run's first inactive window
  const uint32_t prevb = (s + 1u) & 1u;
  const uint32_t f = b.fin[inst];
  const uint32_t mb = (f != ~0u) ? f : d.mins[3 * inst + s % 3u];  // pending keys are >= it
  const uint32_t NB = 1u << b.q.nb_log2, C = 1u << b.q.c_log2;
  uint64_t pend = 0, pcs = 0, dig = 0, com = 0;
  uint32_t pmin = kInfBits;
  for (uint32_t l = blockIdx.x * wpb + (threadIdx.x >> 5); l < I.p.num_lps; l += gridDim.x * wpb) {
    const uint32_t lp = I.lp0 + l;
    const size_t lpb = (size_t)lp << b.q.nb_log2;
    for (uint32_t b0 = 0; b0 < NB; b0 += 32) {
      const uint32_t c = (b0 + lane < NB) ? min(b.q.cnt[lpb + b0 + lane], C) : 0u;
      uint32_t nz = __ballot_sync(GPQ_FULL_MASK, c > 0);
      while (nz) {
        const uint32_t l2 = (uint32_t)__ffs(nz) - 1u;
        nz &= nz - 1u;
        const uint32_t cl = __shfl_sync(GPQ_FULL_MASK, c, l2);
        const unsigned long long* bk = b.q.keys + ((lpb + b0 + l2) << b.q.c_log2);
        for (uint32_t q2 = lane; q2 < cl; q2 += 32) {
          const unsigned long long k = bk[q2];
          const uint32_t t = (uint32_t)(k >> 32);
          if (t < mb || t > kInfBits) continue;  // dead: consumed in an earlier window
          pcs += gpq_ev_hash((uint32_t)k, t);
          pend += 1;
          pmin = min(pmin, t);
        }
      }
    }
    const size_t sl = (size_t)prevb * d.max_lps + lp;
    const uint32_t sc = min(b.q.scnt[sl], b.q.F);
    for (uint32_t q2 = lane; q2 < sc; q2 += 32) {
      const unsigned long long k = b.q.spill[sl * b.q.F + q2];
      const uint32_t t = (uint32_t)(k >> 32);
      pcs += gpq_ev_hash((uint32_t)k, t);
      pend += 1;
      pmin = min(pmin, t);
    }
    if (lane == 0) {
      const uint32_t c = d.count[lp];
      com += c;
      dig += gpq_mix64(gpq_mix64(gpq_mix64(((uint64_t)l << 32) | c) ^ d.csum[lp]) + d.ohash[lp]);
    }
  }
  pend = warp_sum_u64(pend);
  pcs = warp_sum_u64(pcs);
  dig = warp_sum_u64(dig);
  com = warp_sum_u64(com);
  pmin = warp_min_u32(pmin);
  if (lane == 0) {
    atomicAdd(&acc[j].pending, (unsigned long long)pend);
    atomicAdd(&acc[j].pending_csum, (unsigned long long)pcs);
    atomicAdd(&acc[j].digest, (unsigned long long)dig);
    atomicAdd(&acc[j].committed, (unsigned long long)com);
    atomicMin(&acc[j].pending_min, pmin);
  }
}
