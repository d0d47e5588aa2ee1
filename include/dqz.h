/*
 * dqz.h -- C ABI of libdqz.so, the B200 (sm_100a) kernels behind the
 * graph-tensor-network hot path of LuchnikovI/dequantizer.
 *
 * Conventions
 *  - Complex numbers are interleaved (re, im) pairs: complex128 = 2 doubles,
 *    complex64 = 2 floats, the memory layout of numpy / torch complex dtypes.
 *  - Every pointer argument except `const dqz_graph_t *` is a DEVICE pointer.
 *    The graph descriptor itself is a host struct whose members are device
 *    pointers; it is read on the host at launch time.
 *  - Every entry point enqueues work on `stream` and returns without
 *    synchronising. The return value is a dqz_status_t: DQZ_OK, or an
 *    argument / launch error detected on the host.
 *  - Node tensors are row-major over (a_0, ..., a_{k-1}, s): bonds in the
 *    node's neighbour order, physical index last
 *    (dequantizer/src/graph/tensor_graph.py:188). A message between a node and
 *    an edge of bond dimension chi is a chi x chi row-major matrix m[b][a]
 *    contracted over its second index (dequantizer/src/tensor_ops.py:45).
 *  - Half-edge h = node_half[v] + slot is bond `slot` of node v. Per half-edge
 *    the state holds n2e[h] (node -> edge message) and e2n[h]
 *    (edge -> node message).
 */
#ifndef DQZ_H
#define DQZ_H

#include <stdint.h>
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  DQZ_OK = 0,
  DQZ_ERR_ARG = 1,          /* bad pointer / size / shape argument        */
  DQZ_ERR_UNSUPPORTED = 2,  /* shape outside the kernels' supported range */
  DQZ_ERR_CUDA = 3,         /* a CUDA launch or runtime call failed       */
  DQZ_ERR_NOT_CONVERGED = 4,
  DQZ_ERR_NONFINITE = 5
} dqz_status_t;

/* Supported ranges of the kernels (checked on the host before launch). */
#define DQZ_MAX_DEGREE 8
#define DQZ_MAX_CHI 64
#define DQZ_MAX_PHYS 8

/* Device-resident description of a packed tensor graph (all members are
 * device pointers except the counts). Built by dequantizer_b200.layout. */
typedef struct {
  int32_t n_nodes;
  int32_t n_edges;
  int32_t n_halves;            /* half-edges = sum of node degrees; equals
                                  2 * n_edges when every edge has both ends
                                  in the layout                              */
  const int32_t *node_degree;  /* [n_nodes]                                */
  const int32_t *node_phys;    /* [n_nodes] physical dimension              */
  const int32_t *node_half;    /* [n_nodes] first half-edge of the node      */
  const int64_t *node_off;     /* [n_nodes] tensor offset (complex elements) */
  const int32_t *half_node;    /* [2E]                                       */
  const int32_t *half_edge;    /* [2E]                                       */
  const int32_t *half_twin;    /* [2E] the other end's half-edge             */
  const int64_t *half_msg_off; /* [2E] message offset (complex elements)     */
  const int32_t *edge_half;    /* [2E] (half of neighbours[0], of neighbours[1]) */
  const int64_t *edge_lam_off; /* [E] lambda offset (real elements)          */
  int32_t *edge_chi;           /* [E] current bond dimension                 */
} dqz_graph_t;

/* Library / device information. */
int dqz_version(void);
int dqz_device_supported(int device); /* 1 when the device is sm_100 */

/* ---- Launch-shape knobs (no reference counterpart) -------------------------
 * Read by the host side of the entry points at every launch; 0 means the
 * built-in rule. Set by the autotuner (dequantizer_b200/autotune.py), which
 * times the candidates on the caller's shapes. Process-wide, not thread-safe
 * against concurrent launches from other host threads. */
#define DQZ_TUNE_GAUGE_EDGE_WARPS 0 /* warps per CTA of the one-warp vidal_edges kernel (1..8)   */
#define DQZ_TUNE_GAUGE_DIST_WARPS 1 /* warps per CTA of the one-warp vidal_distance kernel (1..8) */
#define DQZ_TUNE_GAUGE_PATH 2       /* 1: one-warp gauge kernels where they apply, 2: one CTA per item */
#define DQZ_TUNE_SU_GRID 3          /* CTAs of simple_update (>= 1), jobs loop over the grid     */
#define DQZ_TUNE_SU_ONCHIP 4        /* simple update: 1 = one-CTA global-scratch kernel only,
                                       2 = cluster forms at any batch size, 3 = no global-workspace
                                       cluster form, 4 = the global-workspace cluster form (256
                                       threads) for every job with 256+ rows                      */
#define DQZ_TUNE_SWEEP_ONECTA 5     /* asynchronous one-launch sweep in one CTA: 1 = never,
                                       2 = wherever its warps' buffers fit                     */
#define DQZ_TUNE_COUNT 6
int dqz_set_tuning(int32_t knob, int32_t value); /* DQZ_ERR_ARG for an unknown knob or value < 0 */
int32_t dqz_get_tuning(int32_t knob);            /* -1 for an unknown knob */

/* ---- Belief propagation (dequantizer/src/mappings/belief_propagation.py:24-64,
 *      dequantizer/src/tensor_ops.py:36-76) ---------------------------------- */

/* Source of the incoming edge->node message for each half-edge. */
#define DQZ_SRC_E2N_OLD 0  /* e2n_old[h]                                   */
#define DQZ_SRC_N2E_OLD 1  /* n2e_old[twin(h)]  (edge already passed, twin node not yet) */
#define DQZ_SRC_N2E_NEW 2  /* n2e_new[twin(h)]  (twin node updated earlier this sweep)   */

/* Node update: for every half-edge listed in `halves` (n_halves of them),
 * n2e_new[h] = pass_through_node output for bond h, with the k-1 incoming
 * messages taken per `src_sel`. Replaces tensor_ops.py:36-60.
 * `scratch` may be NULL when dqz_bp_node_scratch_bytes returns 0. */
int dqz_bp_node_update(const dqz_graph_t *g, const void *tensors /*c128*/,
                       const void *n2e_old, const void *e2n_old, void *n2e_new,
                       const uint8_t *src_sel, const int32_t *halves, int32_t n_halves,
                       int32_t max_slice, int32_t max_chi, void *scratch, cudaStream_t stream);
size_t dqz_bp_node_scratch_bytes(int32_t n_halves, int32_t max_slice, int32_t max_chi);

/* Node update specialised for degree-3 nodes whose three bonds all have
 * dimension `chi` (8 or 16) and physical dimension 2, e.g. random 3-regular
 * graphs. Same result as dqz_bp_node_update (tensor_ops.py:36-60).
 * precision 64: tensors and messages complex128; precision 32: complex64
 * with FP32 arithmetic. A node of any other shape is skipped and sets
 * *error_flag (device int) to 1. Needs no scratch. */
int dqz_bp_node_update_k3(const dqz_graph_t *g, int32_t chi, int32_t precision, const void *tensors,
                          const void *n2e_old, const void *e2n_old, void *n2e_new,
                          const uint8_t *src_sel, const int32_t *halves, int32_t n_halves,
                          int32_t *error_flag, cudaStream_t stream);

/* Mixed-precision node update on tensor cores for the same shapes with
 * chi = 16: BF16 products, FP32 accumulation, complex64 messages. One CTA per
 * node (all three outgoing messages); `nodes` lists the nodes to update.
 * `tensors_bf16` holds every node tensor as BF16 planes, node v at
 * v * 16384 elements, [s][re|im][a][b][c], built by dqz_pack_bf16_planes. */
int dqz_bp_node_update_k3_tc(const dqz_graph_t *g, const void *tensors_bf16, const void *n2e_old,
                             const void *e2n_old, void *n2e_new, const uint8_t *src_sel,
                             const int32_t *nodes, int32_t n_nodes, int32_t *error_flag,
                             cudaStream_t stream);
/* complex64 node tensors (node_off layout) -> BF16 planes for the kernel above. */
int dqz_pack_bf16_planes(const dqz_graph_t *g, const void *tensors_c64, void *tensors_bf16,
                         cudaStream_t stream);

/* The same node update with the mode products on the 5th-generation tensor
 * cores (tcgen05.mma, accumulators in tensor memory; the three final 16 x 16
 * contractions as warp-level MMAs). `tensors_bf16` holds every node tensor as
 * dqz_bf16_umma_elems_per_node() BF16 elements at v * that count, 16-byte
 * aligned, built by dqz_pack_bf16_umma. A node of any other shape sets
 * *error_flag to 1; a wait that runs out (no progress for seconds) sets it to 2. */
int dqz_bp_node_update_k3_umma(const dqz_graph_t *g, const void *tensors_bf16, const void *n2e_old,
                               const void *e2n_old, void *n2e_new, const uint8_t *src_sel,
                               const int32_t *nodes, int32_t n_nodes, int32_t *error_flag,
                               cudaStream_t stream);
size_t dqz_bf16_umma_elems_per_node(void);
/* complex64 node tensors (node_off layout) -> the BF16 core layouts above. */
int dqz_pack_bf16_umma(const dqz_graph_t *g, const void *tensors_c64, void *tensors_bf16,
                       cudaStream_t stream);
/* The same for nodes first .. first + count - 1 only (a pipelined load packs
 * each chunk of nodes as soon as its tensors have arrived). */
int dqz_pack_bf16_umma_nodes(const dqz_graph_t *g, const void *tensors_c64, void *tensors_bf16,
                             int32_t first, int32_t count, cudaStream_t stream);

/* A whole sweep (tensor_ops.py:36-76, mappings/belief_propagation.py:24-64) in
 * one launch: the node levels of a schedule in order, then the edge pass, with
 * a grid-wide barrier between levels (a cooperative launch; the grid is sized
 * so that every CTA is resident). halves[level_off[l] .. level_off[l+1]) are
 * the half-edges of level l; max_level bounds the half-edges of one level,
 * max_slice the node-tensor slice (node size / bond dimension), max_chi the
 * bonds. The results equal one dqz_bp_node_update launch per level followed by
 * dqz_bp_edge_pass, bit for bit. sync: two device words of scratch (zeroed by
 * the call). A barrier wait that runs out (seconds) sets *error_flag to 3 and
 * ends the launch. DQZ_ERR_UNSUPPORTED when a slice does not fit in shared
 * memory (use the per-level launches then). Small nodes (slices up to 256
 * elements) with narrow levels run in one CTA instead: a warp per half-edge,
 * a CTA barrier between levels, the same results (knob
 * DQZ_TUNE_SWEEP_ONECTA). */
int dqz_bp_sweep_levels(const dqz_graph_t *g, const void *tensors, const void *n2e_old, const void *e2n_old,
                        void *n2e_new, void *e2n_new, const uint8_t *src_sel, const uint8_t *edge_new,
                        const int32_t *halves, const int32_t *level_off, int32_t n_levels, int32_t max_level,
                        int32_t max_slice, int32_t max_chi, uint32_t *sync, int32_t *error_flag,
                        cudaStream_t stream);

/* The one-CTA form of dqz_bp_sweep_levels driven by a host-built plan, one
 * entry of DQZ_PLAN_WORDS int64 words per item in the order of the level
 * table (level l: items level_off[l] .. level_off[l+1]): node tensor offset,
 * degree k, physical dimension d, slot e of the outgoing bond, outgoing
 * message offset (half_msg_off of the item's half-edge), the bond dimensions
 * (DQZ_MAX_DEGREE words, the first k used), then for every other bond in bond
 * order its incoming message as offset * 4 + source (DQZ_SRC_*: the offset
 * into e2n_old, n2e_old or n2e_new). A warp per item, a CTA barrier between
 * levels, then the edge pass; the same results as dqz_bp_sweep_levels, bit
 * for bit. DQZ_ERR_UNSUPPORTED when a warp's buffers (two bond slices, the
 * node tensor, its messages) do not fit in shared memory eight times. */
#define DQZ_PLAN_WORDS (5 + DQZ_MAX_DEGREE + DQZ_MAX_DEGREE - 1)
int dqz_bp_sweep_planned(const dqz_graph_t *g, const void *tensors, const void *n2e_old, const void *e2n_old,
                         void *n2e_new, void *e2n_new, const uint8_t *edge_new, const int64_t *plan,
                         const int32_t *level_off, int32_t n_levels, int32_t max_level, int32_t max_slice,
                         int32_t max_chi, cudaStream_t stream);

/* The same sweep for large bonds: the work items of level l are
 * (item_half[i], item_slice[i]) for i in item_off[l] .. item_off[l+1] (every
 * slice of the bond of every half-edge of the level), spread over the grid;
 * each writes one column of its unnormalised message, then a second barrier
 * pass divides each message of the level by its trace. Bit-identical to the
 * per-level launches; max_items bounds the items of one level. */
int dqz_bp_sweep_sliced(const dqz_graph_t *g, const void *tensors, const void *n2e_old, const void *e2n_old,
                        void *n2e_new, void *e2n_new, const uint8_t *src_sel, const uint8_t *edge_new,
                        const int32_t *halves, const int32_t *level_off, const int32_t *item_half,
                        const int32_t *item_slice, const int32_t *item_off, int32_t n_levels, int32_t max_items,
                        int32_t max_slice, int32_t max_chi, uint32_t *sync, int32_t *error_flag,
                        cudaStream_t stream);

/* Edge pass on complex64 messages (see dqz_bp_edge_pass). */
int dqz_bp_edge_pass_c64(const dqz_graph_t *g, const void *n2e_old, const void *n2e_new,
                         const uint8_t *edge_new, void *e2n_new, cudaStream_t stream);

/* Edge pass (tensor_ops.py:70-76): e2n_new[h] = (edge_new[h] ? n2e_new : n2e_old)[twin(h)]
 * for every half-edge. */
int dqz_bp_edge_pass(const dqz_graph_t *g, const void *n2e_old, const void *n2e_new,
                     const uint8_t *edge_new, void *e2n_new, int32_t max_chi, cudaStream_t stream);

/* Mean Frobenius distance over all 4E messages (mappings/messages_distance.py:14-22):
 * out[0] = (sum_h |n2e_a[h]-n2e_b[h]| + |e2n_a[h]-e2n_b[h]|) / (4E).
 * `partial` is device scratch of 2*(2E) doubles. */
int dqz_messages_distance(const dqz_graph_t *g, const void *n2e_a, const void *n2e_b,
                          const void *e2n_a, const void *e2n_b, double *partial, double *out,
                          int32_t max_chi, cudaStream_t stream);

/* partial[h] = |n2e_a[h] - n2e_b[h]|_F for every half-edge, complex64 arenas
 * (the per-message terms of mappings/messages_distance.py:14-22 over the
 * node->edge messages; the batched annealer sums them per instance). */
int dqz_message_changes_c64(const dqz_graph_t *g, const void *n2e_a, const void *n2e_b, double *partial,
                            cudaStream_t stream);

/* out[0] = scale * sum(partial[0..n)), deterministic single-CTA reduction. */
int dqz_reduce_sum(const double *partial, int32_t n, double scale, double *out, cudaStream_t stream);

/* out[0] = mean over i < n of |a[seg_off[i]:seg_off[i+1]] - b[...]|_F (complex128
 * segments; messages_distance.py:14-22 over messages packed in one order).
 * partial: n doubles of scratch. */
int dqz_segment_distance(const void *a, const void *b, const int64_t *seg_off, int32_t n,
                         double *partial, double *out, cudaStream_t stream);

/* *count += number of non-finite (NaN or +-Inf) words among the n real words
 * at data (elem_bytes 8: doubles, 4: floats; a complex array of m entries is
 * 2m words). The caller zeroes *count. The reference has no such check: its
 * arithmetic carries NaN through silently; this backs the DQZ_ERR_NONFINITE
 * status of the host-side loops. */
int dqz_count_nonfinite(const void *data, int64_t n, int32_t elem_bytes, int32_t *count, cudaStream_t stream);

/* Copies n segments: dst[dst_off[i] .. + count[i]) = src[src_off[i] .. + count[i]),
 * offsets and counts in elements of elem_bytes (8 or 16). Used to move node
 * tensors / lambdas into a layout with larger capacities. */
int dqz_repack(const void *src, void *dst, const int64_t *src_off, const int64_t *dst_off,
               const int64_t *count, int32_t n, int32_t elem_bytes, cudaStream_t stream);

/* ---- Adjoint of the node update (reverse of tensor_ops.py:36-60) ----------
 * Transposed message sweep for implicit differentiation at a BP fixed point.
 * For each listed node v and each bond e, with n2e_cot[(v,e)] the cotangent
 * of the outgoing message N_{v,e}(T_v, {e2n[(v,f)]}_{f != e}):
 *   e2n_cot[(v,f)] = sum_{e != f} (dN_{v,e} / d e2n[(v,f)])^* n2e_cot[(v,e)]
 *   t_cot[v]      += sum_e (dN_{v,e} / dT_v)^* n2e_cot[(v,e)]   (t_cot may be NULL)
 * Cotangents are grad z = dL/dRe z + i dL/dIm z. e2n_cot entries of the listed
 * nodes are overwritten; max_size / max_chi bound the node sizes and bonds. */
int dqz_bp_node_vjp(const dqz_graph_t *g, const void *tensors, const void *e2n, const void *n2e_cot,
                    void *e2n_cot, void *t_cot, const int32_t *nodes, int32_t n_nodes, int32_t max_size,
                    int32_t max_chi, void *scratch, cudaStream_t stream);
size_t dqz_bp_node_vjp_scratch_bytes(int32_t n_nodes, int32_t max_size);

/* ---- Batched reduced QR (the QR of tensor_ops.py:288, LAPACK conventions) --
 * For each of `batch` row-major m x k complex128 matrices A_b: A_b = Q_b R_b with
 * Q_b (m x min(m,k), orthonormal columns, row-major) and R_b (min(m,k) x k,
 * upper trapezoidal, row-major). Householder reflectors as zgeqr2, Q formed
 * as zung2r. Used by the differentiable two-site decomposition. */
int dqz_qr_batched(const void *a, int64_t batch, int32_t m, int32_t k, void *q, void *r, void *scratch,
                   cudaStream_t stream);
size_t dqz_qr_batched_scratch_bytes(int64_t batch, int32_t m, int32_t k);

/* ---- Dense state vector (quantum_emulator/exact_quantum_emulator.py:11-147) --
 * complex128 state of 2^n amplitudes in device memory; the qubit at position p
 * (traversal order of the nodes) is bit n-1-p of the amplitude index.
 * Gates are HOST arrays of complex128 (re, im interleaved): 2x2 g[o][i] for
 * apply1, 2x2x2x2 g[o1][o2][i1][i2] for apply2 (first qubit = pos1). */
#define DQZ_SV_MAX_QUBITS 34
int dqz_sv_set_basis(void *state, int32_t n, int64_t index, cudaStream_t stream);
int dqz_sv_apply1(void *state, int32_t n, int32_t pos, const double *gate, cudaStream_t stream);
int dqz_sv_apply2(void *state, int32_t n, int32_t pos1, int32_t pos2, const double *gate, cudaStream_t stream);
/* rho (device, 2x2 complex128) = one-qubit reduced density matrix of position pos. */
int dqz_sv_density1(const void *state, int32_t n, int32_t pos, void *rho, void *scratch, cudaStream_t stream);
size_t dqz_sv_density_scratch_bytes(int32_t n);
/* Projects position pos onto |result> and multiplies the state by scale. */
int dqz_sv_project(void *state, int32_t n, int32_t pos, int32_t result, double scale, cudaStream_t stream);

/* ---- Vidal gauge (mappings/vidal_gauge.py:21-63, tensor_ops.py:88-130) ---- */

/* Per edge: eigendecompose both node->edge messages, build sqrt / safe inverse
 * sqrt, SVD of sqrt(m_f) sqrt(m_b)^T; write lambdas and the two
 * orthogonalisers orth[h] (chi x chi, complex128, at half_msg_off[h]).
 * edges: the n_sel edges to process, or NULL for all; the outputs of the
 * other edges are left as they are. */
int dqz_vidal_edges(const dqz_graph_t *g, const void *n2e, double eps, void *orth,
                    double *lambdas, int32_t max_chi, const int32_t *edges, int32_t n_sel,
                    void *scratch, cudaStream_t stream);
size_t dqz_vidal_edges_scratch_bytes(int32_t n_edges, int32_t max_chi);
/* Per node: T_out = T x_e orth[h_e] over every bond (bond index contracted
 * with the row index), normalised. nodes: the n_sel nodes, or NULL for all. */
int dqz_absorb(const dqz_graph_t *g, const void *tensors_in, const void *orth, void *tensors_out,
               int32_t max_size, const int32_t *nodes, int32_t n_sel, void *scratch, cudaStream_t stream);
size_t dqz_absorb_scratch_bytes(int32_t n_nodes, int32_t max_size);
/* The same for nodes too large for shared memory, spread over one CTA per
 * (node, output index of the node's first bond); every element is computed
 * as dqz_absorb computes it, only the normalisation's sum runs in another
 * order. max_slice bounds node size / first bond dimension (e.g. the largest
 * bond slice); tensors_out must not be tensors_in; scratch holds
 * dqz_absorb_split_scratch_bytes(n) bytes. DQZ_ERR_UNSUPPORTED when two
 * slices do not fit in shared memory. Two launches. */
int dqz_absorb_split(const dqz_graph_t *g, const void *tensors_in, const void *orth, void *tensors_out,
                     int64_t max_slice, const int32_t *nodes, int32_t n_sel, void *scratch, cudaStream_t stream);
size_t dqz_absorb_split_scratch_bytes(int32_t n_nodes);
/* The same for degree-3 nodes with physical dimension 2 and every bond of
 * dimension chi (8 or 16), one CTA per node with the tensor held in shared
 * memory; needs no scratch. A node of any other shape is skipped and sets
 * *error_flag (device int) to 1. */
int dqz_absorb_k3(const dqz_graph_t *g, int32_t chi, const void *tensors_in, const void *orth,
                  void *tensors_out, const int32_t *nodes, int32_t n_sel, int32_t *error_flag,
                  cudaStream_t stream);

/* ---- Vidal distance (mappings/vidal_distance.py:17-42, tensor_ops.py:143-175)
 * partial[h] = trace norm for half-edge h; out (optional, NULL to skip) =
 * sum over all half-edges / (2E). max_slice bounds node size / bond
 * dimension over the processed half-edges. halves: the n_sel half-edges to
 * recompute, or NULL for all (the other partial entries are kept). */
int dqz_vidal_distance(const dqz_graph_t *g, const void *tensors, const double *lambdas,
                       double eps, double *partial /*[2E]*/, double *out,
                       int32_t max_chi, int32_t max_slice, const int32_t *halves, int32_t n_sel,
                       cudaStream_t stream);

/* ---- Symmetric gauge (mappings/symmetric_gauge.py:17-61, tensor_ops.py:189-199) */
int dqz_symmetric_gauge(const dqz_graph_t *g, const void *tensors_in, const double *lambdas,
                        double eps, void *tensors_out, cudaStream_t stream);
int dqz_lambdas_to_messages(const dqz_graph_t *g, const double *lambdas, void *n2e, void *e2n,
                            int32_t max_chi, cudaStream_t stream);

/* ---- One-site density matrices (mappings/density_matrix.py:16-37) ---------- */
/* rho[v] (d x d, complex128, at v * DQZ_MAX_PHYS^2) for every node in `nodes`. */
int dqz_density_matrices(const dqz_graph_t *g, const void *tensors, const void *e2n,
                         const int32_t *nodes, int32_t n_nodes, void *rho,
                         int32_t max_size, void *scratch, cudaStream_t stream);
size_t dqz_density_scratch_bytes(int32_t n_nodes, int32_t max_size);

/* ---- Gates (tensor_graph.py:268-446, tensor_ops.py:202-389) --------------- */

/* apply1 (tensor_graph.py:268-275) on n distinct nodes: T[..., o] = sum_i T[..., i] G[o, i],
 * normalised, in place. gates: n x d x d complex128. */
int dqz_apply1(const dqz_graph_t *g, void *tensors, const int32_t *nodes, const void *gates,
               int32_t n, cudaStream_t stream);

/* apply2 halves (tensor_ops.py:221-262): out tensor with bond `slot` grown by r.
 * One launch handles n (node, slot, half) jobs; in/out offsets per job. */
int dqz_apply_half_gates(const void *tensors_in, void *tensors_out, const int64_t *in_off,
                         const int64_t *out_off, const int32_t *shape /*n x (DQZ_MAX_DEGREE+2)*/,
                         const void *halves /*n x 4 x d x d*/, int32_t n, cudaStream_t stream);

/* Simple update (tensor_ops.py:265-389) for n node-disjoint edges in parallel.
 * For job j: edge edges[j], controlling node = endpoint `first_is_ctrl[j] ? 0 : 1`,
 * halves = halves[j] (2 x 4 x d x d: controlling then controlled, rank[j] rows used).
 * Writes Gamma tensors in place (capacity layout), lambdas, edge_chi, and
 * err/entropy per job. max_rows / max_cols bound the rows (d x the other
 * bonds) and columns (bond x gate rank) of the jobs' matrices.
 * Jobs with a 256-row matrix or more run on a cluster form (two CTAs per job,
 * one per side, a two-step QR): in batches of at most one job per SM with
 * their matrices in shared memory where they fit, else in a global workspace
 * inside `scratch`; in larger batches all in the global workspace (256
 * threads a CTA); the others on a one-CTA kernel with its matrices in
 * `scratch`. The scratch (dqz_simple_update_scratch_bytes) also
 * holds one byte per job recording which form did it. Knob
 * DQZ_TUNE_SU_ONCHIP: 1 sends every job to the one-CTA kernel, 2 uses the
 * cluster forms at any batch size, 3 keeps the global-workspace cluster form
 * off. Results agree to rounding and singular-vector phases. */
int dqz_simple_update(const dqz_graph_t *g, void *tensors, double *lambdas,
                      const int32_t *edges, const uint8_t *ctrl_is_first, const void *halves,
                      const int32_t *ranks, int32_t n, double eps, int32_t max_rank,
                      int32_t max_rows, int32_t max_cols, double *err, double *entropy,
                      void *scratch, cudaStream_t stream);
size_t dqz_simple_update_scratch_bytes(int32_t n, int32_t max_rows, int32_t max_cols);

/* Size of the library-owned scratch array behind dqz_simple_update_noalloc. */
#define DQZ_NOALLOC_SCRATCH_BYTES (32u << 20) /* 32 MiB */

/* dqz_simple_update without a scratch argument and without any device
 * allocation. No counterpart in the reference: it exists for callers that
 * cannot allocate device memory themselves -- for example a host program that
 * hands this library only its input and output buffers from a pool it manages
 * under a fixed memory budget, or a latency-bound loop that cannot afford the
 * implicit device synchronisation of cudaMalloc / cudaFree.
 *  - The scratch is a DQZ_NOALLOC_SCRATCH_BYTES (32 MiB) array compiled into
 *    the library; every GPU that loads the library holds it until the process
 *    exits. One job needs 64 * max_rows * max_cols bytes; a call whose job
 *    needs more returns DQZ_ERR_UNSUPPORTED. Jobs beyond the number of slices
 *    that fit run one after another inside the launch.
 *  - The first call on each device looks up the array's device address
 *    (cudaGetSymbolAddress with that device current); make that first call
 *    before any stream capture. The address is kept for the life of the
 *    process: calls after a cudaDeviceReset of that device are not supported.
 *  - The DQZ_TUNE_SU_GRID knob applies as for dqz_simple_update, capped at
 *    the number of job slices that fit in the array.
 *  - Every call uses the same array and it keeps whatever the last call left
 *    there (the kernel writes every scratch word before reading it). Calls
 *    whose kernels overlap on the GPU -- on different streams, or from
 *    different host threads -- race on the array; serialise them.
 * Arguments and results are those of dqz_simple_update. */
int dqz_simple_update_noalloc(const dqz_graph_t *g, void *tensors, double *lambdas,
                              const int32_t *edges, const uint8_t *ctrl_is_first, const void *halves,
                              const int32_t *ranks, int32_t n, double eps, int32_t max_rank,
                              int32_t max_rows, int32_t max_cols, double *err, double *entropy,
                              cudaStream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* DQZ_H */
