// Serving form: many resident Newton-step solves advanced together.
//
// Each attached solve ("slot") owns its FP64/FP32 blocks, its MAS hierarchy
// and numeric inverses, its right-hand side and PCG vectors.  One launch runs
// `passes` pipeline passes over every attached slot; a pass is
//   serve_spmv      : ITER   q = A32 p, p^T q -> alpha
//   serve_residual  : INIT   x = 0, r = g            -> ||r||, ||g||
//                     REFINE r = g - A64 x (FP64)    -> ||r||, ||g||
//                     (done when ||r|| <= tol ||g||, else START)
//   serve_update    : ITER   d += alpha p, r -= alpha q;  START  d = 0
//                     (both write the FP32 level-0 residual)
//   serve_restrict  : MAS restriction of the large levels (one launch each,
//                     a warp per node)
//   serve_tail      : MAS restriction of the small levels (one CTA a slot)
//   serve_gemv      : MAS domain inverses (one CTA a domain)
//   serve_collect   : z = M^-1 r, r^T z, r^T r -> beta; inner stop -> REFINE
//   serve_direction : ITER   p = z + beta p;  REFINE  x += d
// so every pass moves each live slot by one PCG iteration (a refinement
// costs one pass too: its FP64 residual and the restart share the pass).
// This is the precision form of the single-solve path: FP32 blocks and MAS
// inside, FP64 vectors, reductions and refinement residuals.
//
// CTAs are mapped to (slot, local block) by per-kernel tables, so a slot's
// arithmetic (its block partition and its fixed-order reductions) does not
// depend on which other slots share the launch: a solve gives bit-identical
// results alone and in any mix.  Converged slots retire on the device (their
// CTAs return at once) until the host detaches them; the host attaches new
// solves between launches (continuous batching).  The tables have fixed
// capacities per size bucket, so one CUDA graph per bucket is replayed.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "ys_mas_dev.cuh"
#include "ys_pcg.cuh"

namespace ys {

enum ServePhase : int {
  kServeEmpty = YS_SERVE_EMPTY,
  kServeInit = YS_SERVE_INIT,
  kServeRefine = YS_SERVE_REFINE,
  kServeStart = YS_SERVE_START,
  kServeIter = YS_SERVE_ITER,
  kServeDone = YS_SERVE_DONE,
  kServeFailed = YS_SERVE_FAILED
};

struct ServeSlot {
  MasDev M;
  SpmvSet A;
  uint32_t nv;
  uint32_t first_tail;    // first MAS level restricted by the tail kernel
  uint32_t row_blocks;    // CTAs of the row kernels
  uint32_t spmv_blocks;   // CTAs of the SpMV (kRowLanes threads a row)
  const double* g;
  double* x;
  double* d;
  double* r;
  double* p;
  float4* p32;            // FP32 copy of p (x, y, z, 0) for the FP32 SpMV
  double* q;
  double* z;
  double* partials;       // [2 * spmv_blocks]
  unsigned* tickets;      // [2]
  double target2;         // tol^2 of the true relative residual
  double refine_tol;
  uint32_t max_it;
};

struct SlotState {
  int phase;
  int fresh;              // p = z on the next direction update
  uint32_t iterations;
  uint32_t refinements;
  double delta_new;
  double delta_old;
  double alpha;
  double beta;
  double tol_inner;       // absolute threshold on the inner r^T r
  double rr;              // last FP64 residual ||g - A64 x||^2
  double gg;
};

struct ServeDev {
  ServeSlot* slots;
  SlotState* state;
  const uint32_t* map_rows;
  const uint32_t* map_spmv;
  const uint32_t* map_gemv;
  const uint32_t* map_tail;
  const uint32_t* map_restrict[kMaxLevels];
  uint32_t n_rows, n_spmv, n_gemv, n_tail;
  uint32_t n_restrict[kMaxLevels];
};

constexpr uint32_t kLocalBits = 24;
constexpr uint32_t kLocalMask = (1u << kLocalBits) - 1;
constexpr uint32_t kServeMaxSlots = 256;

__device__ __forceinline__ bool map_entry(const uint32_t* __restrict__ map, uint32_t count, uint32_t& slot,
                                          uint32_t& local) {
  if (blockIdx.x >= count) return false;
  const uint32_t e = map[blockIdx.x];
  slot = e >> kLocalBits;
  local = e & kLocalMask;
  return true;
}

// grid_reduce_last over the `nblk` CTAs of one slot (local index `local`).
template <int NV>
__device__ __forceinline__ bool slot_reduce_last(double (&v)[NV], double* __restrict__ partials,
                                                 unsigned* __restrict__ ticket, uint32_t local, uint32_t nblk) {
  __shared__ double red[kPcgBlock / 32];
  __shared__ bool last;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    const double s = block_sum<kPcgBlock>(v[k], red);
    if (threadIdx.x == 0) partials[(uint64_t)k * nblk + local] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == nblk - 1;
  __syncthreads();
  if (!last) return false;
  __threadfence();
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    v[k] = block_sum<kPcgBlock>(thread_partial_sum(partials + (uint64_t)k * nblk, nblk), red);
  }
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

// ITER: q = A32 p (FP32 blocks, float4 copy of p), p^T q -> alpha.  Kept
// apart from the FP64 residual kernel so it runs at the FP32 gather's
// register count (occupancy).
__global__ void __launch_bounds__(kPcgBlock) serve_spmv(const ServeDev* __restrict__ S) {
  uint32_t s, b;
  if (!map_entry(S->map_spmv, S->n_spmv, s, b)) return;
  const ServeSlot& T = S->slots[s];
  SlotState& st = S->state[s];
  if (st.phase != kServeIter) return;
  const uint32_t t = b * blockDim.x + threadIdx.x;
  const uint32_t i = t / kRowLanes;
  const int lane = (int)(t % kRowLanes);
  const bool valid = i < T.nv;
  double v[1] = {0.0};
  double q0, q1, q2;
  spmv3_group_x32(&T.A, 1, i, valid, lane, T.p32, q0, q1, q2);
  if (valid && lane == 0) {
    T.q[3ull * i] = q0; T.q[3ull * i + 1] = q1; T.q[3ull * i + 2] = q2;
    v[0] = T.p[3ull * i] * q0 + T.p[3ull * i + 1] * q1 + T.p[3ull * i + 2] * q2;
  }
  if (!slot_reduce_last<1>(v, T.partials, T.tickets, b, T.spmv_blocks)) return;
  if (threadIdx.x != 0) return;
  const double curv = v[0];
  st.delta_old = st.delta_new;
  if (!isfinite(curv) || curv <= 0.0) {
    st.alpha = 0.0;
    st.phase = kServeFailed;
  } else {
    st.alpha = st.delta_new / curv;
  }
}

// INIT: x = 0, r = g; REFINE: r = g - A64 x (FP64 blocks); both -> ||r||,
// ||g||, then DONE when ||r|| <= tol ||g||, else START with the next inner
// tolerance.
__global__ void __launch_bounds__(kPcgBlock) serve_residual(const ServeDev* __restrict__ S) {
  uint32_t s, b;
  if (!map_entry(S->map_spmv, S->n_spmv, s, b)) return;
  const ServeSlot& T = S->slots[s];
  SlotState& st = S->state[s];
  const int phase = st.phase;
  if (phase != kServeInit && phase != kServeRefine) return;
  const uint32_t t = b * blockDim.x + threadIdx.x;
  const uint32_t i = t / kRowLanes;
  const int lane = (int)(t % kRowLanes);
  const bool valid = i < T.nv;
  double v[2] = {0.0, 0.0};
  if (phase == kServeRefine) {
    double h[3];
    spmv3_group(&T.A, 1, false, i, valid, lane, T.x, h[0], h[1], h[2]);
    if (valid && lane == 0) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double g = T.g[3ull * i + k], r = g - h[k];
        T.r[3ull * i + k] = r;
        v[0] += r * r;
        v[1] += g * g;
      }
    }
  } else if (valid && lane == 0) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double g = T.g[3ull * i + k];
      T.x[3ull * i + k] = 0.0;
      T.r[3ull * i + k] = g;
      v[0] += g * g;
    }
    v[1] = v[0];
  }
  if (!slot_reduce_last<2>(v, T.partials, T.tickets, b, T.spmv_blocks)) return;
  if (threadIdx.x != 0) return;
  const double rr = v[0], gg = v[1];
  if (phase == kServeRefine) st.refinements += 1;
  st.rr = rr;
  st.gg = gg;
  if (!(isfinite(rr) && isfinite(gg))) {
    st.phase = kServeFailed;
  } else if (rr <= T.target2 * gg) {
    st.phase = kServeDone;
  } else if (st.iterations >= T.max_it) {
    st.phase = kServeFailed;
  } else {
    // inner relative tolerance: the same rule as the single-solve refinement
    const double tau = fmin(fmax(T.refine_tol, 0.5 * sqrt(T.target2 * gg / rr)), 0.5);
    st.tol_inner = tau * tau * rr;
    st.phase = kServeStart;
  }
}

__global__ void __launch_bounds__(kPcgBlock) serve_update(const ServeDev* __restrict__ S) {
  uint32_t s, b;
  if (!map_entry(S->map_rows, S->n_rows, s, b)) return;
  const ServeSlot& T = S->slots[s];
  const int phase = S->state[s].phase;
  if (phase != kServeStart && phase != kServeIter) return;
  const uint32_t i = b * blockDim.x + threadIdx.x;
  if (i >= T.nv) return;
  float* rl = T.M.rl;
  if (phase == kServeIter) {
    const double alpha = S->state[s].alpha;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      T.d[3ull * i + k] = T.d[3ull * i + k] + T.p[3ull * i + k] * alpha;
      const double r = T.r[3ull * i + k] - T.q[3ull * i + k] * alpha;
      T.r[3ull * i + k] = r;
      rl[3ull * i + k] = (float)r;
    }
  } else {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      T.d[3ull * i + k] = 0.0;
      rl[3ull * i + k] = (float)T.r[3ull * i + k];
    }
  }
}

__device__ __forceinline__ bool mas_live(const ServeDev* __restrict__ S, uint32_t s) {
  const int phase = S->state[s].phase;
  return phase == kServeStart || phase == kServeIter;
}

__global__ void __launch_bounds__(kPcgBlock) serve_restrict(const ServeDev* __restrict__ S, uint32_t level) {
  uint32_t s, b;
  if (!map_entry(S->map_restrict[level], S->n_restrict[level], s, b) || !mas_live(S, s)) return;
  const ServeSlot& T = S->slots[s];
  const uint32_t p = T.M.level_node_offset[level] + ((b * blockDim.x + threadIdx.x) >> 5);
  if (p < T.M.level_node_offset[level + 1]) restrict_node_warp(T.M, T.r, level, p, (int)(threadIdx.x & 31));
}

__global__ void __launch_bounds__(1024) serve_tail(const ServeDev* __restrict__ S) {
  uint32_t s, b;
  if (!map_entry(S->map_tail, S->n_tail, s, b) || !mas_live(S, s)) return;
  const ServeSlot& T = S->slots[s];
  restrict_tail_levels(T.M, T.r, T.first_tail);
}

__global__ void __launch_bounds__(kGemvThreads) serve_gemv(const ServeDev* __restrict__ S) {
  extern __shared__ float4 serve_smem[];
  uint32_t s, d;
  if (!map_entry(S->map_gemv, S->n_gemv, s, d) || !mas_live(S, s)) return;
  gemv_domain(S->slots[s].M, d, serve_smem);
}

__global__ void __launch_bounds__(kPcgBlock) serve_collect(const ServeDev* __restrict__ S) {
  uint32_t s, b;
  if (!map_entry(S->map_rows, S->n_rows, s, b)) return;
  const ServeSlot& T = S->slots[s];
  SlotState& st = S->state[s];
  const int phase = st.phase;
  if (phase != kServeStart && phase != kServeIter) return;
  const uint32_t i = b * blockDim.x + threadIdx.x;
  double v[2] = {0.0, 0.0};
  if (i < T.nv) {
    double z[3];
    collect_levels(T.M, T.nv, i, z);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double r = T.r[3ull * i + k];
      T.z[3ull * i + k] = z[k];
      v[0] += r * z[k];
      v[1] += r * r;
    }
  }
  if (!slot_reduce_last<2>(v, T.partials, T.tickets + 1, b, T.row_blocks)) return;
  if (threadIdx.x != 0) return;
  const double next = v[0];
  if (phase == kServeStart) {
    st.delta_new = next;
    st.beta = 0.0;
    st.fresh = 1;
    st.phase = isfinite(next) && next > 0.0 ? kServeIter : kServeFailed;
    return;
  }
  const double prev = st.delta_old;
  const uint32_t it = st.iterations + 1;
  st.iterations = it;
  st.delta_new = next;
  st.fresh = 0;
  if (!isfinite(next) || next < 0.0 || !isfinite(prev) || prev <= 0.0) {
    st.beta = 0.0;
    st.phase = kServeFailed;
  } else {
    st.beta = next / prev;
    // inner solve done (or out of budget): fold d into x and take the FP64
    // residual in the next pass
    if (v[1] <= st.tol_inner || next == 0.0 || it >= T.max_it) st.phase = kServeRefine;
  }
}

__global__ void __launch_bounds__(kPcgBlock) serve_direction(const ServeDev* __restrict__ S) {
  uint32_t s, b;
  if (!map_entry(S->map_rows, S->n_rows, s, b)) return;
  const ServeSlot& T = S->slots[s];
  const SlotState& st = S->state[s];
  const int phase = st.phase;
  const uint32_t i = b * blockDim.x + threadIdx.x;
  if (i >= T.nv) return;
  if (phase == kServeIter) {
    double p[3];
    if (st.fresh) {
#pragma unroll
      for (int k = 0; k < 3; ++k) p[k] = T.z[3ull * i + k];
    } else {
      const double beta = st.beta;
#pragma unroll
      for (int k = 0; k < 3; ++k) p[k] = T.z[3ull * i + k] + T.p[3ull * i + k] * beta;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) T.p[3ull * i + k] = p[k];
    T.p32[i] = make_float4((float)p[0], (float)p[1], (float)p[2], 0.0f);
  } else if (phase == kServeRefine) {
#pragma unroll
    for (int k = 0; k < 3; ++k) T.x[3ull * i + k] += T.d[3ull * i + k];
  }
}

// ---- host side ---------------------------------------------------------------

struct Bucket {
  uint32_t rows, spmv, gemv, tail, smem, levels;
  uint32_t restrict_cap[kMaxLevels];
  bool operator<(const Bucket& o) const { return std::memcmp(this, &o, sizeof(Bucket)) < 0; }
};

struct ServeHandle {
  uint32_t max_slots = 0;
  uint32_t passes = 0;
  ServeSlot* d_slots = nullptr;
  SlotState* d_state = nullptr;
  ServeDev* d_dev = nullptr;
  uint32_t* d_maps = nullptr;
  size_t map_capacity = 0;        // uint32 entries
  uint32_t* h_maps = nullptr;     // pinned staging
  size_t h_map_capacity = 0;
  ServeDev* h_dev = nullptr;      // pinned
  ServeSlot* h_slots = nullptr;   // pinned
  SlotState* h_state = nullptr;   // pinned initial states of attached slots
  SlotState* h_status = nullptr;  // pinned status reads
  cudaEvent_t staged = nullptr;   // staging copies done
  std::vector<uint8_t> attached;
  std::vector<uint8_t> fresh;     // attached since the last launch
  bool dirty = true;
  Bucket bucket{};
  std::map<Bucket, cudaGraphExec_t> graphs;
};

static uint32_t round_cap(uint32_t n) {
  uint32_t c = 64;
  while (c < n) c <<= 1;
  return c;
}

static cudaError_t add_node(cudaGraph_t g, cudaGraphNode_t* node, cudaGraphNode_t* prev, const void* fn,
                            unsigned grid, unsigned block, size_t smem, void** args) {
  cudaKernelNodeParams kp{};
  kp.func = const_cast<void*>(fn);
  kp.gridDim = dim3(grid);
  kp.blockDim = dim3(block);
  kp.sharedMemBytes = (unsigned)smem;
  kp.kernelParams = args;
  const cudaError_t e = cudaGraphAddKernelNode(node, g, *prev ? prev : nullptr, *prev ? 1 : 0, &kp);
  if (e == cudaSuccess) *prev = *node;
  return e;
}

static cudaError_t build_graph(ServeHandle* h, const Bucket& k, cudaGraphExec_t* exec) {
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaGraphCreate(&g, 0);
  if (e != cudaSuccess) return e;
  const ServeDev* dev = h->d_dev;
  void* a[] = {&dev};
  uint32_t lv[kMaxLevels];
  void* al[kMaxLevels][2];
  for (uint32_t l = 0; l < kMaxLevels; ++l) {
    lv[l] = l;
    al[l][0] = &dev;
    al[l][1] = &lv[l];
  }
  cudaGraphNode_t prev = nullptr, n = nullptr;
  for (uint32_t pass = 0; pass < h->passes && e == cudaSuccess; ++pass) {
    e = add_node(g, &n, &prev, (const void*)serve_spmv, k.spmv, kPcgBlock, 0, a);
    if (e == cudaSuccess) e = add_node(g, &n, &prev, (const void*)serve_residual, k.spmv, kPcgBlock, 0, a);
    if (e == cudaSuccess) e = add_node(g, &n, &prev, (const void*)serve_update, k.rows, kPcgBlock, 0, a);
    for (uint32_t l = 1; l < k.levels && e == cudaSuccess; ++l)
      if (k.restrict_cap[l])
        e = add_node(g, &n, &prev, (const void*)serve_restrict, k.restrict_cap[l], kPcgBlock, 0, al[l]);
    if (e == cudaSuccess) e = add_node(g, &n, &prev, (const void*)serve_tail, k.tail, 1024, 0, a);
    if (e == cudaSuccess) e = add_node(g, &n, &prev, (const void*)serve_gemv, k.gemv, kGemvThreads, k.smem, a);
    if (e == cudaSuccess) e = add_node(g, &n, &prev, (const void*)serve_collect, k.rows, kPcgBlock, 0, a);
    if (e == cudaSuccess) e = add_node(g, &n, &prev, (const void*)serve_direction, k.rows, kPcgBlock, 0, a);
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(exec, g, 0);
  cudaGraphDestroy(g);
  return e;
}

// Rebuild the CTA tables of the attached slots into pinned staging, grow the
// device table buffer if needed and pick the bucket.
static int32_t stage_maps(ServeHandle* h, cudaStream_t s) {
  std::vector<uint32_t> rows, spmv, gemv, tail, res[kMaxLevels];
  uint32_t smem_dofs = 3;
  for (uint32_t k = 0; k < h->max_slots; ++k) {
    if (!h->attached[k]) continue;
    const ServeSlot& T = h->h_slots[k];
    const uint32_t tag = k << kLocalBits;
    for (uint32_t b = 0; b < T.row_blocks; ++b) rows.push_back(tag | b);
    for (uint32_t b = 0; b < T.spmv_blocks; ++b) spmv.push_back(tag | b);
    for (uint32_t d = 0; d < T.M.num_domains; ++d) gemv.push_back(tag | d);
    tail.push_back(tag);
    for (uint32_t l = 1; l < T.first_tail; ++l) {
      const uint32_t cnt = T.M.level_node_offset[l + 1] - T.M.level_node_offset[l];
      // a warp per node
      for (uint32_t b = 0; b < (32 * cnt + kPcgBlock - 1) / kPcgBlock; ++b) res[l].push_back(tag | b);
    }
    smem_dofs = std::max(smem_dofs, T.M.max_dofs);
  }
  Bucket k{};
  k.rows = round_cap((uint32_t)rows.size());
  k.spmv = round_cap((uint32_t)spmv.size());
  k.gemv = round_cap((uint32_t)gemv.size());
  k.tail = round_cap((uint32_t)tail.size());
  k.smem = (uint32_t)gemv_smem_bytes(smem_dofs);
  k.levels = 1;
  for (uint32_t l = 1; l < kMaxLevels; ++l) {
    k.restrict_cap[l] = res[l].empty() ? 0u : round_cap((uint32_t)res[l].size());
    if (!res[l].empty()) k.levels = l + 1;
  }
  size_t total = (size_t)k.rows + k.spmv + k.gemv + k.tail;
  for (uint32_t l = 1; l < kMaxLevels; ++l) total += k.restrict_cap[l];
  // staging is rewritten only after the previous staging copies finished
  YS_CUDA_TRY(cudaEventSynchronize(h->staged));
  if (total > h->h_map_capacity) {
    if (h->h_maps) cudaFreeHost(h->h_maps);
    h->h_maps = nullptr;
    h->h_map_capacity = 0;
    YS_CUDA_TRY(cudaMallocHost(&h->h_maps, sizeof(uint32_t) * total));
    h->h_map_capacity = total;
  }
  if (total > h->map_capacity) {
    // the old tables may still be read by a launch in flight
    YS_CUDA_TRY(cudaStreamSynchronize(s));
    if (h->d_maps) cudaFree(h->d_maps);
    h->d_maps = nullptr;
    h->map_capacity = 0;
    YS_CUDA_TRY(cudaMalloc(&h->d_maps, sizeof(uint32_t) * total));
    h->map_capacity = total;
  }
  ServeDev& D = *h->h_dev;
  D.slots = h->d_slots;
  D.state = h->d_state;
  size_t off = 0;
  auto place = [&](const std::vector<uint32_t>& v, uint32_t cap, const uint32_t** dst, uint32_t* count) {
    if (!v.empty()) std::memcpy(h->h_maps + off, v.data(), sizeof(uint32_t) * v.size());
    *dst = h->d_maps + off;
    *count = (uint32_t)v.size();
    off += cap;
  };
  place(rows, k.rows, &D.map_rows, &D.n_rows);
  place(spmv, k.spmv, &D.map_spmv, &D.n_spmv);
  place(gemv, k.gemv, &D.map_gemv, &D.n_gemv);
  place(tail, k.tail, &D.map_tail, &D.n_tail);
  for (uint32_t l = 0; l < kMaxLevels; ++l) {
    D.map_restrict[l] = nullptr;
    D.n_restrict[l] = 0;
    if (l >= 1 && k.restrict_cap[l]) place(res[l], k.restrict_cap[l], &D.map_restrict[l], &D.n_restrict[l]);
  }
  YS_CUDA_TRY(cudaMemcpyAsync(h->d_maps, h->h_maps, sizeof(uint32_t) * off, cudaMemcpyHostToDevice, s));
  YS_CUDA_TRY(cudaMemcpyAsync(h->d_dev, h->h_dev, sizeof(ServeDev), cudaMemcpyHostToDevice, s));
  h->bucket = k;
  return YS_OK;
}

}  // namespace ys

extern "C" {

uint64_t ys_serve_workspace_doubles(uint32_t num_vars) {
  const uint64_t spmv_blocks = ((uint64_t)num_vars * ys::kRowLanes + ys::kPcgBlock - 1) / ys::kPcgBlock;
  // FP32 copy of p (4 floats a variable, first: 16-byte aligned) + d, r, p,
  // q, z + partials + tickets
  return 2ull * num_vars + 15ull * num_vars + 2 * spmv_blocks + 2;
}

int32_t ys_serve_create(uint32_t max_slots, uint32_t passes_per_launch, void** handle) {
  YS_REQUIRE(handle, YS_ERR_INVALID, "null handle");
  YS_REQUIRE(max_slots >= 1 && max_slots <= ys::kServeMaxSlots, YS_ERR_INVALID, "max_slots must be 1..256");
  YS_REQUIRE(passes_per_launch >= 1 && passes_per_launch <= 64, YS_ERR_INVALID, "passes_per_launch must be 1..64");
  auto* h = new ys::ServeHandle();
  h->max_slots = max_slots;
  h->passes = passes_per_launch;
  h->attached.assign(max_slots, 0);
  h->fresh.assign(max_slots, 0);
  cudaError_t e = cudaMalloc(&h->d_slots, sizeof(ys::ServeSlot) * max_slots);
  if (e == cudaSuccess) e = cudaMalloc(&h->d_state, sizeof(ys::SlotState) * max_slots);
  if (e == cudaSuccess) e = cudaMalloc(&h->d_dev, sizeof(ys::ServeDev));
  if (e == cudaSuccess) e = cudaMallocHost(&h->h_dev, sizeof(ys::ServeDev));
  if (e == cudaSuccess) e = cudaMallocHost(&h->h_slots, sizeof(ys::ServeSlot) * max_slots);
  if (e == cudaSuccess) e = cudaMallocHost(&h->h_state, sizeof(ys::SlotState) * max_slots);
  if (e == cudaSuccess) e = cudaMallocHost(&h->h_status, sizeof(ys::SlotState) * max_slots);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->staged, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMemset(h->d_state, 0, sizeof(ys::SlotState) * max_slots);
  if (e == cudaSuccess) {
    std::memset(h->h_dev, 0, sizeof(ys::ServeDev));
    std::memset(h->h_slots, 0, sizeof(ys::ServeSlot) * max_slots);
    std::memset(h->h_state, 0, sizeof(ys::SlotState) * max_slots);
    e = cudaEventRecord(h->staged, 0);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ys::serve_gemv, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)ys::gemv_smem_bytes(128));
  if (e != cudaSuccess) {
    ys_set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
    ys_serve_destroy(h);
    return YS_ERR_CUDA;
  }
  *handle = h;
  return YS_OK;
}

int32_t ys_serve_attach(void* handle, uint32_t slot, const ys_serve_slot_desc* d) {
  YS_REQUIRE(handle && d, YS_ERR_INVALID, "null argument");
  auto* h = static_cast<ys::ServeHandle*>(handle);
  YS_REQUIRE(slot < h->max_slots, YS_ERR_INVALID, "slot index out of range");
  YS_REQUIRE(!h->attached[slot], YS_ERR_INVALID, "slot already attached");
  const ys::MasDev* M = ys::mas_device_state(d->mas);
  YS_REQUIRE(M, YS_ERR_INVALID, "missing MAS handle");
  YS_REQUIRE(d->matrix.num_sets == 1, YS_ERR_INVALID, "one 3x3 block set per slot");
  YS_REQUIRE(d->matrix.values[0] && d->matrix.values32[0], YS_ERR_INVALID, "FP64 and FP32 block values required");
  YS_REQUIRE(d->matrix.num_vars == M->nv && M->nv > 0, YS_ERR_INVALID, "matrix and MAS sizes differ");
  YS_REQUIRE(M->nv <= (ys::kLocalMask / ys::kRowLanes) * (uint32_t)ys::kPcgBlock && M->num_domains <= ys::kLocalMask,
             YS_ERR_CAPACITY, "slot too large for the CTA tables");
  YS_REQUIRE(d->rhs && d->solution && d->workspace, YS_ERR_INVALID, "null vector");
  YS_REQUIRE((reinterpret_cast<uintptr_t>(d->workspace) & 15) == 0, YS_ERR_INVALID,
             "workspace must be 16-byte aligned");
  YS_REQUIRE(d->tolerance > 0.0 && d->max_iterations >= 1, YS_ERR_INVALID, "bad tolerance / iteration budget");
  // the staging entry of this slot may still be the source of a pending copy
  YS_CUDA_TRY(cudaEventSynchronize(h->staged));
  ys::ServeSlot& T = h->h_slots[slot];
  std::memset(&T, 0, sizeof(T));
  T.M = *M;
  T.A = ys::SpmvSet{d->matrix.values[0], d->matrix.values32[0], d->matrix.row_ptr[0], d->matrix.entry_block[0],
                    d->matrix.entry_col[0]};
  T.nv = M->nv;
  T.first_tail = ys::restrict_tail_first(*M);
  T.row_blocks = (T.nv + ys::kPcgBlock - 1) / ys::kPcgBlock;
  T.spmv_blocks = (uint32_t)(((uint64_t)T.nv * ys::kRowLanes + ys::kPcgBlock - 1) / ys::kPcgBlock);
  T.g = d->rhs;
  T.x = d->solution;
  const uint64_t n = 3ull * T.nv;
  double* w = d->workspace;
  T.p32 = reinterpret_cast<float4*>(w); w += 2ull * T.nv;
  T.d = w; w += n;
  T.r = w; w += n;
  T.p = w; w += n;
  T.q = w; w += n;
  T.z = w; w += n;
  T.partials = w; w += 2ull * T.spmv_blocks;
  T.tickets = reinterpret_cast<unsigned*>(w);
  T.target2 = d->tolerance * d->tolerance;
  T.refine_tol = d->refinement_tolerance;
  T.max_it = d->max_iterations;
  ys::SlotState& st = h->h_state[slot];
  std::memset(&st, 0, sizeof(st));
  st.phase = ys::kServeInit;
  h->attached[slot] = 1;
  h->fresh[slot] = 1;
  h->dirty = true;
  return YS_OK;
}

int32_t ys_serve_detach(void* handle, uint32_t slot) {
  YS_REQUIRE(handle, YS_ERR_INVALID, "null handle");
  auto* h = static_cast<ys::ServeHandle*>(handle);
  YS_REQUIRE(slot < h->max_slots && h->attached[slot], YS_ERR_INVALID, "slot not attached");
  h->attached[slot] = 0;
  h->fresh[slot] = 0;
  h->dirty = true;
  return YS_OK;
}

int32_t ys_serve_launch(void* handle, void* stream) {
  YS_REQUIRE(handle, YS_ERR_INVALID, "null handle");
  auto* h = static_cast<ys::ServeHandle*>(handle);
  cudaStream_t s = (cudaStream_t)stream;
  bool any = false;
  for (uint32_t k = 0; k < h->max_slots; ++k) any = any || h->attached[k];
  if (!any) return YS_OK;
  if (h->dirty) {
    const int32_t rc = ys::stage_maps(h, s);
    if (rc != YS_OK) return rc;
    for (uint32_t k = 0; k < h->max_slots; ++k) {
      if (!h->fresh[k]) continue;
      const ys::ServeSlot& T = h->h_slots[k];
      YS_CUDA_TRY(cudaMemcpyAsync(h->d_slots + k, h->h_slots + k, sizeof(ys::ServeSlot), cudaMemcpyHostToDevice, s));
      YS_CUDA_TRY(cudaMemcpyAsync(h->d_state + k, h->h_state + k, sizeof(ys::SlotState), cudaMemcpyHostToDevice, s));
      YS_CUDA_TRY(cudaMemsetAsync(T.tickets, 0, 2 * sizeof(unsigned), s));
      h->fresh[k] = 0;
    }
    YS_CUDA_TRY(cudaEventRecord(h->staged, s));
    h->dirty = false;
  }
  auto it = h->graphs.find(h->bucket);
  if (it == h->graphs.end()) {
    cudaGraphExec_t exec = nullptr;
    YS_CUDA_TRY(ys::build_graph(h, h->bucket, &exec));
    it = h->graphs.emplace(h->bucket, exec).first;
  }
  YS_CUDA_TRY(cudaGraphLaunch(it->second, s));
  return YS_OK;
}

int32_t ys_serve_status(void* handle, void* stream, ys_serve_slot_status* out) {
  YS_REQUIRE(handle && out, YS_ERR_INVALID, "null argument");
  auto* h = static_cast<ys::ServeHandle*>(handle);
  cudaStream_t s = (cudaStream_t)stream;
  YS_CUDA_TRY(cudaEventSynchronize(h->staged));
  YS_CUDA_TRY(
      cudaMemcpyAsync(h->h_status, h->d_state, sizeof(ys::SlotState) * h->max_slots, cudaMemcpyDeviceToHost, s));
  YS_CUDA_TRY(cudaStreamSynchronize(s));
  for (uint32_t k = 0; k < h->max_slots; ++k) {
    const ys::SlotState& st = h->h_status[k];
    ys_serve_slot_status& o = out[k];
    if (!h->attached[k]) {
      o = ys_serve_slot_status{YS_SERVE_EMPTY, 0, 0, 0.0};
      continue;
    }
    o.phase = h->fresh[k] ? YS_SERVE_INIT : st.phase;
    o.iterations = h->fresh[k] ? 0u : st.iterations;
    o.refinements = h->fresh[k] ? 0u : st.refinements;
    o.relative_residual = (!h->fresh[k] && st.gg > 0.0) ? std::sqrt(st.rr / st.gg) : 0.0;
  }
  return YS_OK;
}

int32_t ys_serve_destroy(void* handle) {
  if (!handle) return YS_OK;
  auto* h = static_cast<ys::ServeHandle*>(handle);
  for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second);
  if (h->staged) {
    cudaEventSynchronize(h->staged);
    cudaEventDestroy(h->staged);
  }
  cudaFree(h->d_slots);
  cudaFree(h->d_state);
  cudaFree(h->d_dev);
  cudaFree(h->d_maps);
  if (h->h_maps) cudaFreeHost(h->h_maps);
  if (h->h_dev) cudaFreeHost(h->h_dev);
  if (h->h_slots) cudaFreeHost(h->h_slots);
  if (h->h_state) cudaFreeHost(h->h_state);
  if (h->h_status) cudaFreeHost(h->h_status);
  delete h;
  return YS_OK;
}

}  // extern "C"
