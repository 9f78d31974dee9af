// MAS preconditioner hooks used by the PCG graph builder.
#pragma once

#include "ys_pcg.cuh"

namespace ys {

struct MasPcgHooks {
  void* params = nullptr;  // owned by the MAS handle
  bool fused_direction = false;  // the loop body's last MAS node also updates p
};

// Nodes computing r = g - H x (or r = g), z = M^-1 r, p = z and the initial
// reductions / stop threshold; sets the loop condition.  `*last` receives the
// final node.
cudaError_t mas_add_init_nodes(void* mas, cudaGraph_t g, const cudaGraphNode_t* deps, size_t ndeps,
                               cudaGraphNode_t* last, uint32_t nv, const double* rhs, double* x, double* r, double* p,
                               float4* p32, double* q, double* z, double* st, double* partials, unsigned* tickets, const SpmvSet* sets,
                               int nsets, int fp32, int stop_rule, int zero_guess, double tolerance, uint32_t max_it,
                               cudaGraphConditionalHandle cond, MasPcgHooks* hooks);

// Nodes of the loop body after spmv_dot: x/r update, z = M^-1 r, r^T z,
// beta and the stop test.
cudaError_t mas_add_update_nodes(void* mas, cudaGraph_t body, const cudaGraphNode_t* deps, size_t ndeps,
                                 cudaGraphNode_t* last, MasPcgHooks* hooks);

}  // namespace ys
