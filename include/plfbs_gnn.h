/* plfbs_gnn.h — learned warm start for plfbs: a mesh graph network over the
 * solver's own face connectivity that predicts a near-converged field from
 * geometry and Reynolds number, trained on solves this library generates.
 * No counterpart in the reference (its solver always starts from the
 * initial-condition field); the network's output enters the solver through
 * plfbs_warm_start (plfbs.h).
 *
 * Network (hidden width 64, ReLU, BF16 tensor-core matrix products with FP32
 * accumulation, FP32 activations and master weights):
 *   h0 = MLP_n(node features),  e0 = MLP_e(edge features)
 *   for l = 1..L:  e_l = e_{l-1} + MLP_el([e_{l-1}, h_{l-1}[src], h_{l-1}[dst]])
 *                  h_l = h_{l-1} + MLP_nl([h_{l-1}, sum of e_l over edges into the node])
 *   y = MLP_d(h_L)
 * Every MLP is Linear(k, 64) -> ReLU -> Linear(64, m). Parameters are one
 * flat FP32 array, MLP by MLP in the order n, e, (e1, n1), ..., (eL, nL), d;
 * each as W1 [k][64] row-major, b1 [64], W2 [64][m], b2 [m].
 * All entry points return 0 or a negative PLFBS_ERR_* code (plfbs.h);
 * messages through plfbs_gnn_last_error (per thread for a NULL network).
 */
#ifndef PLFBS_GNN_H
#define PLFBS_GNN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct plfbs_gnn plfbs_gnn;

typedef struct {
  int32_t n_nodes;        /* graph nodes (the mesh's interior cells) */
  int32_t n_edges;        /* directed edges (two per internal face) */
  int32_t node_features;  /* 1..16 */
  int32_t edge_features;  /* 1..16 */
  int32_t layers;         /* message-passing layers, 1..16 */
  int32_t outputs;        /* 1..16 */
} plfbs_gnn_shape;

/* Builds the graph (src/dst [n_edges], 0-based node ids; edge_features
 * [n_edges][edge_features], fixed for the graph) on `device` and allocates
 * the activations needed for training. Parameters start at zero. */
int plfbs_gnn_create(const plfbs_gnn_shape* shape, const int32_t* src, const int32_t* dst,
                     const float* edge_features, int32_t device, plfbs_gnn** out);

/* Number of parameters of the flat array described above. */
int plfbs_gnn_param_count(plfbs_gnn* g, int64_t* n);
int plfbs_gnn_set_params(plfbs_gnn* g, const float* params, int64_t n);
int plfbs_gnn_get_params(plfbs_gnn* g, float* params, int64_t n);

/* y [n_nodes][outputs] from node_features [n_nodes][node_features] (host). */
int plfbs_gnn_forward(plfbs_gnn* g, const float* node_features, float* y);

/* Mean squared error against target [n_nodes][outputs] and its gradient with
 * respect to every parameter (grad [param_count], host). */
int plfbs_gnn_gradients(plfbs_gnn* g, const float* node_features, const float* target,
                        double* loss, float* grad);

/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8, bias-corrected) on the mean
 * squared error of one graph; *loss is the loss before the step. */
int plfbs_gnn_train_step(plfbs_gnn* g, const float* node_features, const float* target,
                         float learning_rate, double* loss);

/* Which tensor-core instructions the MLPs use, forward and backward: 1 =
 * tcgen05 (accumulators in tensor memory, one thread issuing the MMAs; the
 * backward's weight gradients accumulated in tensor memory over a block's
 * tiles; the default), 0 = warp-level mma.sync. */
int plfbs_gnn_set_tensor_cores(plfbs_gnn* g, int32_t kind);

const char* plfbs_gnn_last_error(const plfbs_gnn* g);
void plfbs_gnn_destroy(plfbs_gnn* g);

#ifdef __cplusplus
}
#endif
#endif /* PLFBS_GNN_H */
