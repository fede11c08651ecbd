// TEST INFRASTRUCTURE: an A* model written the way the reference writes its agents
// (src/a_star.cu:269-593): one open list per agent, i.e. per LP of a gpupq_b200 queue,
// driven through the device queue functions of include/gpq/queue.cuh -- queue_peek and
// queue_set_done to pop, queue_insert_or_update for improved neighbours, queue_is_empty
// to detect an exhausted search and queue_clear when the goal is reached.  One thread per
// agent pops one item per round (the reference pops up to eight per round, which makes
// its result depend on the schedule; one pop per round is plain A*, so the cost found is
// the optimal cost C* the oracle computes).  Open-list items: ts = f, lp = agent,
// id = cell, aux = g (include/gpq/astar.h).
#include <cuda_runtime.h>

#include <vector>

#include "gpq.h"
#include "gpq/astar.h"
#include "gpq/queue.cuh"

namespace {

constexpr uint32_t kMaxCells = 64 * 64;

struct AgentArrays {
  const gpq_astar_grid* grid;  // [agents]
  uint32_t* g;                 // [agents][kMaxCells]
  unsigned char* closed;       // [agents][kMaxCells]
  uint32_t* cost;              // [agents]
  uint32_t* done;              // [agents]
  unsigned long long* pops;
  unsigned int* n_done;
};

__global__ void astar_agent_start(AgentArrays a, uint32_t agents) {
  for (uint32_t ag = blockIdx.x * blockDim.x + threadIdx.x; ag < agents; ag += gridDim.x * blockDim.x) {
    const gpq_astar_grid gr = a.grid[ag];
    const uint32_t h = gpq_astar_h(4, gr.start, gr.goal, gr.width);
    a.g[(size_t)ag * kMaxCells + gr.start] = 0;
    gpq_item it;
    it.ts = (float)h;
    it.lp = ag;
    it.id = gr.start;
    it.aux = 0;
    queue_insert_or_update(it, (int)ag);
  }
}

__global__ void astar_agent_round(AgentArrays a, uint32_t agents) {
  for (uint32_t ag = blockIdx.x * blockDim.x + threadIdx.x; ag < agents; ag += gridDim.x * blockDim.x) {
    if (a.done[ag]) continue;
    const gpq_astar_grid gr = a.grid[ag];
    uint32_t* g = a.g + (size_t)ag * kMaxCells;
    unsigned char* closed = a.closed + (size_t)ag * kMaxCells;
    queue_item* top = NULL;
    const int index = queue_peek(&top, (int)ag);
    if (index == -1) {
      if (queue_is_empty((int)ag)) {  // open list exhausted: the goal is unreachable
        a.cost[ag] = GPQ_ASTAR_INF;
        a.done[ag] = 1;
        atomicAdd(a.n_done, 1u);
      }
      continue;
    }
    const gpq_item it = *top;
    queue_set_done(index);
    atomicAdd(a.pops, 1ull);
    const uint32_t cell = it.id, gc = it.aux;
    if (closed[cell] || gc > g[cell]) continue;  // a stale entry of an improved cell
    closed[cell] = 1;
    if (cell == gr.goal) {
      a.cost[ag] = gc;
      a.done[ag] = 1;
      atomicAdd(a.n_done, 1u);
      queue_clear((int)ag);
      continue;
    }
#define AGENT_BLOCKED(c) gpq_astar_blocked(&gr, (c))
    for (int k = 0; k < 4; ++k) {
      uint32_t nb;
      GPQ_ASTAR_NEIGHBOUR(nb, gr, cell, k, AGENT_BLOCKED);
      if (nb == GPQ_ASTAR_INF || closed[nb]) continue;
      const uint32_t ng = gc + 1u;
      if (ng >= g[nb]) continue;
      g[nb] = ng;
      gpq_item c;
      c.ts = (float)(ng + gpq_astar_h(4, nb, gr.goal, gr.width));
      c.lp = ag;
      c.id = nb;
      c.aux = ng;
      queue_insert_or_update(c, (int)ag);
    }
#undef AGENT_BLOCKED
  }
}

}  // namespace

// Solves `agents` 4-connected grids of at most 64 x 64 cells, one agent per LP of a queue
// of kind `kind`; cost_out[i] = C* (GPQ_ASTAR_INF when unreachable).  Returns 0 or a
// gpq_status.
extern "C" int dropin_astar_run(const gpq_astar_grid* grids, uint32_t agents, uint32_t kind, uint32_t* cost_out,
                                unsigned long long* pops_out, unsigned long long* rounds_out) {
  for (uint32_t i = 0; i < agents; ++i)
    if (grids[i].width * grids[i].height > kMaxCells || grids[i].conn != 4) return GPQ_ERR_INVALID;
  gpq_queue_config qc = {};
  qc.kind = kind;
  qc.num_lps = agents;
  qc.capacity = 8192;
  qc.insert_capacity = 8;
  gpq_queue* q = NULL;
  int st = gpq_queue_create(&qc, &q);
  if (st) return st;
  if ((st = gpq_queue_bind(q)) != GPQ_OK) return st;
  AgentArrays a = {};
  gpq_astar_grid* d_grid = NULL;
  cudaMalloc(&d_grid, agents * sizeof(gpq_astar_grid));
  cudaMemcpy(d_grid, grids, agents * sizeof(gpq_astar_grid), cudaMemcpyHostToDevice);
  a.grid = d_grid;
  cudaMalloc(&a.g, (size_t)agents * kMaxCells * sizeof(uint32_t));
  cudaMemset(a.g, 0xff, (size_t)agents * kMaxCells * sizeof(uint32_t));
  cudaMalloc(&a.closed, (size_t)agents * kMaxCells);
  cudaMemset(a.closed, 0, (size_t)agents * kMaxCells);
  cudaMalloc(&a.cost, agents * sizeof(uint32_t));
  cudaMalloc(&a.done, agents * sizeof(uint32_t));
  cudaMemset(a.done, 0, agents * sizeof(uint32_t));
  cudaMalloc(&a.pops, sizeof(unsigned long long));
  cudaMemset(a.pops, 0, sizeof(unsigned long long));
  cudaMalloc(&a.n_done, sizeof(unsigned int));
  cudaMemset(a.n_done, 0, sizeof(unsigned int));
  const uint32_t blocks = (agents + 127) / 128;
  astar_agent_start<<<blocks, 128>>>(a, agents);
  if (cudaDeviceSynchronize() != cudaSuccess) st = GPQ_ERR_CUDA;  // the queue posts on its own stream
  if (!st) st = gpq_queue_post(q, NULL);
  unsigned long long rounds = 0;
  unsigned int n_done = 0;
  const float inf = __builtin_inff();
  while (!st && n_done < agents && rounds < 4u * kMaxCells + 16u) {
    st = gpq_queue_set_bound(q, inf, NULL);  // A*: no window, every open item may be popped
    if (st) break;
    astar_agent_round<<<blocks, 128>>>(a, agents);
    if (cudaDeviceSynchronize() != cudaSuccess) { st = GPQ_ERR_CUDA; break; }
    st = gpq_queue_post(q, NULL);
    ++rounds;
    if (cudaMemcpy(&n_done, a.n_done, sizeof(n_done), cudaMemcpyDeviceToHost) != cudaSuccess) st = GPQ_ERR_CUDA;
  }
  if (!st && n_done < agents) st = GPQ_ERR_TIMEOUT;
  cudaMemcpy(cost_out, a.cost, agents * sizeof(uint32_t), cudaMemcpyDeviceToHost);
  cudaMemcpy(pops_out, a.pops, sizeof(unsigned long long), cudaMemcpyDeviceToHost);
  *rounds_out = rounds;
  cudaFree(d_grid);
  cudaFree(a.g);
  cudaFree(a.closed);
  cudaFree(a.cost);
  cudaFree(a.done);
  cudaFree(a.pops);
  cudaFree(a.n_done);
  gpq_queue_destroy(q);
  return st;
}
