/*
 * dlp.h - C ABI of libdlp.so, the sm_100a kernels behind the dynlp-compatible Python API.
 *
 * Conventions (shared by every entry point):
 *   - All pointers are device pointers owned by the caller; no entry point allocates device
 *     memory. Scratch comes from a caller-provided workspace whose size a *_workspace_bytes
 *     query returns.
 *   - Every function returns an int status (DLP_OK = 0). Launches are asynchronous on the
 *     given stream (a cudaStream_t; NULL = legacy default stream) unless documented otherwise.
 *   - Rows of a sparse matrix are given as [rbeg[r], rend[r]) ranges into col/w. Plain CSR
 *     passes rbeg = indptr, rend = indptr + 1. Row ranges with slack capacity (the resident
 *     edge-updatable graph) pass separate begin/end arrays. Stored entries with weight 0 are
 *     "inert" (deleted edges or edges leaving the solved set), as in the reference
 *     (dynlp/kernels.py:323, dynlp/stream.py:202-204).
 *   - Dense n x C score/residual matrices are row-major with a leading dimension ld >= C
 *     (in elements). Index arrays are int32, as in the reference (dynlp/stream.py:161).
 *   - Precision codes: DLP_F32, DLP_F64, DLP_BF16. Supported (weights, X, Y) combinations for
 *     the row kernels: (f32,f32,f32), (f64,f64,f64), (f32,f64,f64) [fp64 residual over fp32-
 *     stored weights], (bf16,bf16,f32) and (bf16,bf16,bf16) [fp32 accumulation]. The dense
 *     vectors a/diag/rhs use the Y precision (fp32 when Y is bf16).
 */
#ifndef DLP_H
#define DLP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  DLP_OK = 0,
  DLP_ERR_INVALID = 1,   /* bad pointer, size, shape or leading dimension */
  DLP_ERR_DTYPE = 2,     /* unsupported precision combination */
  DLP_ERR_CUDA = 3,      /* a CUDA runtime call failed; dlp_last_cuda_error() on the calling thread has the code */
  DLP_ERR_CAP = 4,       /* iteration cap reached before convergence */
  DLP_ERR_CANCELLED = 5, /* the host cancel flag was set */
  DLP_ERR_WORKSPACE = 6, /* workspace missing or too small */
  DLP_ERR_OVERFLOW = 7,  /* a row of the resident graph ran out of slack; rebuild needed */
  DLP_ERR_DEVICE = 8,    /* a device-side check failed (bad index or bounded wait ran out) */
  DLP_ERR_SCRATCH_LIMIT = 9 /* size beyond the fixed scratch of an allocation-free entry point */
};

enum { DLP_F32 = 0, DLP_F64 = 1, DLP_BF16 = 2 };

typedef struct CUstream_st *dlp_stream_t;

/* ---- library ---------------------------------------------------------------------------- */
int dlp_version(void);
const char *dlp_status_string(int status);
int dlp_last_cuda_error(void);
/* number of SMs of the current device (used for persistent grid sizes) */
int dlp_sm_count(void);
/* kernels this library has launched in the process so far (graph replays count their kernels) */
unsigned long long dlp_launch_count(void);

/* Cancellation of the device-side loops (no reference counterpart: the reference has no way to stop
 * a solve). `word` points at an int32 the device can read: device memory, or pinned host memory
 * (cudaHostAlloc / cudaMallocHost, usable on the device under unified addressing). While it holds a
 * non-zero value, dlp_pcg stops at its next stop decision (once per iteration) and dlp_fused_push
 * at its next round, each returning DLP_ERR_CANCELLED with consistent outputs (the iterate and its
 * residual, or Z and R with no residual taken but not pushed). NULL unregisters. One word per
 * process; calls already running keep the word they started with. */
int dlp_set_cancel_word(const int32_t *word);

/* ---- (a) row-major SpMM with fused axpy / residual epilogue -------------------------------
 * Replaces kernels.spmm_axpy (dynlp/kernels.py:140-166, :240-266, launcher :377-393),
 * solvers.apply_A (dynlp/solvers.py:46-49) and the changed-row residual refresh of
 * IncrementalLP.solve (dynlp/solvers.py:404-407).
 *   for each output row i (rows == NULL: i = r = 0..n_rows-1; else r = rows[i]):
 *     acc       = sum_{j in [rbeg[r], rend[r])} w[j] * X[col[j], :]
 *     Y[o, c]   = cr * RHS[r, c] + alpha * a[r] * X[r, c] + b * acc[c]
 *   with o = i when compact_out != 0, else o = r. a == NULL drops the a-term, RHS == NULL the
 *   RHS-term. group = edge lanes per row (power of two <= 32; <= 0 picks from the mean degree
 *   avg_deg, like kernels.auto_group, dynlp/kernels.py:365-370). */
int dlp_spmm(const int32_t *rbeg, const int32_t *rend, const int32_t *col, const void *w, int w_dtype,
             int32_t n_rows, const int32_t *rows, int32_t C, const void *X, int64_t ldx, int x_dtype,
             const void *a, double alpha, double b, const void *RHS, int64_t ldr, double cr, void *Y,
             int64_t ldy, int y_dtype, int compact_out, int32_t group, double avg_deg, dlp_stream_t stream);

/* Mixed-precision SpMM in the apply_A form: Y = alpha * a[r] * X_own[r, :] + b * sum_j w_lo[j] *
 * X_lo[col_j, :], with bf16 weights and gathered rows, fp32 accumulation, the own-row term from the
 * fp32 X_own (NULL: from X_lo) and fp32 a / Y (config: SpMM on BF16 weights/scores). */
int dlp_spmm_lowp(const int32_t *rbeg, const int32_t *rend, const int32_t *col, const void *w_lo, int32_t n_rows,
                  int32_t C, const void *X_lo, int64_t ld_lo, const void *X_own, int64_t ld_own, const void *a,
                  double alpha, double b, void *Y, int64_t ldy, int32_t group, double avg_deg, dlp_stream_t stream);

/* ---- (b) frontier Jacobi ------------------------------------------------------------------
 * Replaces the frontier_jacobi kernels (dynlp/kernels.py:31-103, :186-220; FrontierOps.jacobi
 * :464-474): for g < nf, r = frontier[g]:
 *   Y[g, c] = (rhs[r, c] + sum_j w_j X[col_j, c]) / diag[r];  changed[g] = any_c |Y[g,c]-X[r,c]| > delta
 * changed may be NULL. When out_list != NULL the rows with changed[g] are appended to out_list
 * (unordered, warp-aggregated atomics) and *out_count (device int, caller-zeroed) counts them.
 * X, rhs, diag, Y share one precision (f32 or f64); w is f32 or matches it. */
int dlp_frontier_jacobi(const int32_t *rbeg, const int32_t *rend, const int32_t *col, const void *w,
                        int w_dtype, const int32_t *frontier, int32_t nf, int32_t C, const void *X,
                        int64_t ldx, const void *rhs, int64_t ldr, const void *diag, double delta, void *Y,
                        int64_t ldy, int dtype, uint8_t *changed, int32_t *out_list, int32_t *out_count,
                        int32_t group, double avg_deg, dlp_stream_t stream);

/* ---- (b) residual push scatter and neighbour marking --------------------------------------
 * Replaces push_scatter (dynlp/kernels.py:105-126, :222-238; FrontierOps.push :476-486):
 *   R[col_j, :] += w_j * D[g, :] for every stored entry j of row frontier[g]; mark[col_j] = 1.
 * mark may be NULL. R and D share one precision (f32 or f64). */
int dlp_push_scatter(const int32_t *rbeg, const int32_t *rend, const int32_t *col, const void *w, int w_dtype,
                     const int32_t *frontier, int32_t nf, int32_t C, const void *D, int64_t ldd, void *R,
                     int64_t ldr, int dtype, uint8_t *mark, int32_t group, double avg_deg,
                     dlp_stream_t stream);

/* Replaces mark_neighbors (dynlp/kernels.py:128-138): mark[col_j] = 1 for entries of rows[0..nr). */
int dlp_mark_neighbors(const int32_t *rbeg, const int32_t *rend, const int32_t *col, const int32_t *rows,
                       int32_t nr, uint8_t *mark, dlp_stream_t stream);

/* ---- synchronous push round helpers (solvers.push, dynlp/solvers.py:100-125) -------------
 * take: for g < nc, r = cand[g]: D[g,:] = R[r,:] / diag[r]; Z[r,:] += D[g,:]; R[r,:] = 0; mark[r] = 1. */
int dlp_push_take(const int32_t *cand, int32_t nc, int32_t C, void *Z, int64_t ldz, void *R, int64_t ldr,
                  const void *diag, void *D, int64_t ldd, int dtype, uint8_t *mark, dlp_stream_t stream);

/* Violating filter of a vertex list: keep[g] = any_c |R[r,c]| > eps[c] * diag[r] for r = idx[g]
 * (idx == NULL: r = g, g < n). eps is fp64. Optionally clears mark[r]. Output is a uint8 flag per g. */
int dlp_violating(const int32_t *idx, int32_t n, int32_t C, const void *R, int64_t ldr, const void *diag,
                  int dtype, const double *eps, uint8_t *flag, uint8_t *clear_mark, dlp_stream_t stream);

/* ---- ordered stream compaction ------------------------------------------------------------
 * out[0..*count) = the g < n with flag[g] != 0, ascending (numpy flatnonzero); idx != NULL maps
 * g -> idx[g]. *count is a device int32. Needs dlp_compact_workspace_bytes(n) of workspace. */
size_t dlp_compact_workspace_bytes(int32_t n);
int dlp_compact(const uint8_t *flag, const int32_t *idx, int32_t n, int32_t *out, int32_t *count, void *ws,
                size_t ws_bytes, dlp_stream_t stream);

/* ---- column reductions (fp64 results) -----------------------------------------------------
 * kind 0: out[c] = max_r |X[r,c]| / diag[r]            (rho_cols, dynlp/solvers.py:52-54)
 * kind 1: out[c] = sum_r X[r,c] * Y[r,c]                (PCG dots, dynlp/solvers.py:76,79,94)
 * kind 2: out[c] = sum_r X[r,c]^2                       (2-norms for the relative residual)
 * kind 3: out[c] = max_r |X[r,c]|
 * diag/Y may be NULL when unused. out is a device double[C]; rows restricted by mask when
 * mask != NULL (mask[r] != 0). Partial sums per block over a fixed grid, then an ordered final
 * pass: the result does not depend on scheduling. Workspace: dlp_colreduce_workspace_bytes(C). */
size_t dlp_colreduce_workspace_bytes(int32_t C);

/* Allocation-free variant of dlp_colreduce (no counterpart in the reference): same kinds, inputs,
 * output and results, but it takes no workspace. It is for callers that cannot allocate device
 * memory when they need the reduction (a server that reserved all of HBM for its own pool, a host
 * runtime bridged through an FFI with no device allocator, code that must avoid the implicit
 * synchronisation of an allocation). Its partial sums live in a fixed array inside the library,
 * sized for C <= 64 columns (151,552 bytes, held on every GPU that loads the library until exit);
 * wider inputs return DLP_ERR_SCRATCH_LIMIT. The first call on each device looks the array's
 * device address up (cudaGetSymbolAddress), so make that first call before any stream capture.
 * All calls on a device share the array: calls that overlap on the GPU race and must be
 * serialised by the caller. It allocates nothing and calls no allocating routine. The looked-up
 * address is kept for the life of the process: after a cudaDeviceReset of a device, do not call it
 * on that device again in the same process. */
int dlp_colreduce_noalloc(int kind, int32_t n, int32_t C, const void *X, int64_t ldx, const void *Y, int64_t ldy,
                          const void *diag, int dtype, const uint8_t *mask, double *out, dlp_stream_t stream);
int dlp_colreduce(int kind, int32_t n, int32_t C, const void *X, int64_t ldx, const void *Y, int64_t ldy,
                  const void *diag, int dtype, const uint8_t *mask, double *out, void *ws, size_t ws_bytes,
                  dlp_stream_t stream);

/* ---- (f) connected components ---------------------------------------------------------------
 * Replaces cc.connected_components (dynlp/cc.py:8-23). parent[0..n) receives, for every vertex,
 * the smallest vertex id of its component (hook-larger-under-smaller union-find with path
 * halving, then full compression). Edges: m entries (rows[i], cols[i]); endpoints outside
 * [0, n) are rejected with DLP_ERR_DEVICE via *err (device int, caller-zeroed; may be NULL). */
int dlp_cc_edges(int32_t n, const int32_t *rows, const int32_t *cols, int64_t m, int32_t *parent, int32_t *err,
                 dlp_stream_t stream);

/* Graph form used by the grounding checks (dynlp/stream.py:150-159, :275-280): vertices 0..n-1
 * plus a sink vertex n. An entry (u, v) of the row ranges joins u and v when vmask[u] and
 * w != 0 (w may be NULL: all entries live) and vmask[v]; it joins u and the sink when vmask[u]
 * and sink[v]. parent has n + 1 entries. vmask/sink may be NULL (all 1 / all 0). The row ranges
 * must be symmetric (entry (u, v) live iff (v, u) is). With a workspace of
 * dlp_cc_graph_workspace_bytes() the edges go in the sampling-then-skip order (the rows of the
 * dominant component are not hooked twice); ws = NULL hooks every entry. Same result either way. */
size_t dlp_cc_graph_workspace_bytes(void);
int dlp_cc_graph(int32_t n, const int32_t *rbeg, const int32_t *rend, const int32_t *col, const void *w,
                 int w_dtype, const uint8_t *vmask, const uint8_t *sink, int32_t *parent, int32_t *err, void *ws,
                 size_t ws_bytes, dlp_stream_t stream);

/* dlp_cc_graph without a sink, for a graph that changes by small batches between calls (the
 * per-batch components of the resident stream; no reference counterpart beyond dynlp/cc.py:8-23 run
 * per batch in dynlp/stream.py:150-153). Same parent (n + 1 entries; minimum vertex id of every
 * component of the vmask-induced subgraph over live entries, parent[n] = n) as dlp_cc_graph with
 * sink = NULL. The workspace carries state between calls: zero it before the first call; each call
 * starts a breadth-first search from the root of the previous call's most frequent component and
 * leaves the rows it did not reach to the union-find. Asynchronous (no host read).
 * Workspace: dlp_cc_graph_warm_workspace_bytes(n). */
size_t dlp_cc_graph_warm_workspace_bytes(int32_t n);
int dlp_cc_graph_warm(int32_t n, const int32_t *rbeg, const int32_t *rend, const int32_t *col, const void *w,
                      int w_dtype, const uint8_t *vmask, int32_t *parent, int32_t *err, void *ws, size_t ws_bytes,
                      dlp_stream_t stream);

/* The grounded set (dynlp/stream.py:150-159, :275-280) without a full labelling: on entry umask
 * holds the previous grounded set; on exit umask[u] = 1 iff vmask[u] and u's component in the
 * graph form of dlp_cc_graph (same arguments, same symmetric row ranges) reaches the sink, i.e.
 * exactly the vertices with parent[u] == parent[n] there; in_t[u] = 1 where membership changed;
 * *count (device int, caller-zeroed) += number of changes. Bottom-up reachability sweeps, checked
 * on the host every few sweeps; when they have not settled after 32, dlp_cc_graph finishes the
 * job (same result). *sweeps_out (host, may be NULL) = sweeps run, negated if the fallback ran.
 * Workspace: dlp_ground_reach_workspace_bytes(n). Synchronises the stream. */
size_t dlp_ground_reach_workspace_bytes(int32_t n);
int dlp_ground_reach(int32_t n, const int32_t *rbeg, const int32_t *rend, const int32_t *col, const void *w,
                     int w_dtype, const uint8_t *vmask, const uint8_t *sink, uint8_t *umask, uint8_t *in_t,
                     int32_t *count, int32_t *err, int32_t *sweeps_out, void *ws, size_t ws_bytes,
                     dlp_stream_t stream);

/* The reference's component labels of the masked vertices: connected_components over the
 * subgraph that vmask induces, numbered as dynlp/stream.py:150-153 with dynlp/cc.py:22 number them
 * (local ids = the masked vertices in ascending order; a component's label = the rank of its smallest
 * local id among the components'). Input: parent of dlp_cc_graph with the same vmask (fully
 * compressed; roots are minimum vertex ids). Output: label[i] for the i-th masked vertex, *n_comp =
 * components, *n_masked = masked vertices (device ints). Workspace: dlp_cc_mask_labels_workspace_bytes. */
size_t dlp_cc_mask_labels_workspace_bytes(int32_t n);
int dlp_cc_mask_labels(int32_t n, const int32_t *parent, const uint8_t *vmask, int32_t *label, int32_t *n_comp,
                       int32_t *n_masked, void *ws, size_t ws_bytes, dlp_stream_t stream);

/* Canonical relabel: label[i] = rank of parent[i] among the roots (parent[r] == r; parent must be
 * fully compressed, as dlp_cc_edges/dlp_cc_graph leave it), i.e. the
 * labels numpy.unique(parent, return_inverse=True) gives (dynlp/cc.py:22-23); *n_comp = number
 * of roots (device int). Needs dlp_compact_workspace_bytes(n). */
int dlp_cc_relabel(int32_t n, const int32_t *parent, int32_t *label, int32_t *n_comp, void *ws, size_t ws_bytes,
                   dlp_stream_t stream);


/* One pass of the certification check (dynlp/solvers.py:295-301, :322-337) over an n x C residual
 * R (the last column the h column's): out[c] = max_u |R_uc| / diag_u (rho_cols), out[C + c] =
 * sum_u R_uc^2, out[2C + c] = sum_u rhs_uc^2 (skipped when rhs is NULL), out[3C] = max_u |H_u| (H: one
 * column, stride ldh; skipped when NULL). All in fp64 with a fixed reduction order. dtype of R, rhs,
 * H and diag: f32/f64. Workspace: dlp_residual_stats_workspace_bytes(C); out: device double[3C+1]. */
size_t dlp_residual_stats_workspace_bytes(int32_t C);
int dlp_residual_stats(int32_t n, int32_t C, const void *R, int64_t ldr, const void *rhs, int64_t ldrhs,
                       const void *diag, const void *H, int64_t ldh, int dtype, double *out, void *ws,
                       size_t ws_bytes, dlp_stream_t stream);

/* ---- (d) fused block PCG, Jacobi preconditioner --------------------------------------------
 * Replaces solvers.pcg with jacobi_M (dynlp/solvers.py:62-97): one CG per column of
 * (diag - W) Z = rhs, starting from the Z given. Per iteration three kernels (SpMM + pAp, residual
 * update + rz/norms/violation, direction update); inner products and norms summed in fp64 (for fp32
 * rows of 9-12 columns, each lane's pAp partial over its dozen or so rows is fp32), reduced in a
 * fixed order. Stop rule `mode`: bit 0 = the reference's max_uc |R_uc|/(eps_c diag_u) <= 1,
 * bit 1 = max_c ||R_c||_2 / rhs_norm[c] <= target_relres (both bits: both must hold); bit 2 = a zero
 * start: Z is set to 0 (its incoming values are ignored) and the initial residual is rhs itself (no
 * SpMM; R is written in the first sweep); bit 3 = always the three-kernel iteration; bit 4 = no
 * recheck: a proposed stop is final (status 5) without the true-residual confirmation below, for a
 * caller that confirms on its own residual (R then holds the recurrence residual). Without bit 3,
 * fp32 solves whose rows take a whole-row gather (9-12 columns with ldp == ldap >= 12 and P, AP on
 * 16-byte boundaries; or 5-8 columns with ldp == ldap a multiple of 8 and P, AP on 32-byte boundaries; no
 * bf16 mirror) run two kernels per iteration: the SpMM also sums
 * q_c = sum AP^2/diag and predicts beta = alpha^2 q / rz - 1 (exact for A-conjugate successive
 * directions), and one sweep updates R, Z and the next direction; P and AP trade places every
 * iteration (on return either may hold the last direction), and rz of the stored residual stays
 * exact for the next alpha. A proposed
 * stop is confirmed on the true residual rhs - A Z (solvers.py:85-89), and a failed confirmation
 * resumes with the reference's beta (rz of the true residual over rz of the iteration);
 * `patience` iterations without a 10% improvement stop the solve as the reference's stall rule
 * does (:90-92).
 * eps and rhs_norm are HOST arrays of C doubles (rhs_norm may be NULL when bit 1 is unused).
 * R, P, AP are caller-provided n x C scratch matrices (R holds the final residual; for fp32 rows of
 * 9-12 columns with ldap >= 12 on 16-byte boundaries AP is written whole, its padding columns
 * included). With
 * use_graph != 0 the iteration loop runs on the device as one CUDA graph with a conditional WHILE
 * node (cached per problem; the host reads the control block once per loop and once per recheck);
 * where conditional nodes are unavailable, chunks of check_every iterations are replayed as graphs.
 * use_graph == 0 launches the kernels directly and reads the control block every check_every
 * iterations.
 * Synchronous: returns after the solve; *status_out = 5 converged, 2 stalled, 3 iteration cap
 * (the call returns DLP_ERR_CAP), 4 breakdown (a non-finite residual entry), 6 cancelled (returns
 * DLP_ERR_CANCELLED); the outputs are filled in every case. eps may be NULL when bit 0 is unused.
 * (dtype, w_dtype) in {(f32,f32), (f64,f64), (f64,f32)}. Workspace: dlp_pcg_workspace_bytes(C).
 * The control block and per-column constants go up in one copy from a pinned host buffer of a few
 * KB kept per host thread and device (allocated on the first call); the control block comes back
 * through pinned memory.
 * Mixed precision (fp32 only): with w_lo (bf16 copy of w) and P_lo (a bf16 n x C buffer, ld_lo) the
 * SpMM gathers the bf16 mirror of P that the direction update keeps (fp32 accumulation), while the
 * diagonal term, pAp and every vector update stay fp32; NULL for both = full-precision gathers. */
size_t dlp_pcg_workspace_bytes(int32_t C);
int dlp_pcg(const int32_t *rbeg, const int32_t *rend, const int32_t *col, const void *w, int w_dtype, int32_t n,
            int32_t C, const void *diag, const void *rhs, int64_t ldrhs, void *Z, int64_t ldz, void *R, int64_t ldr,
            void *P, int64_t ldp, void *AP, int64_t ldap, int dtype, const double *eps, const double *rhs_norm,
            double target_relres, int32_t mode, int32_t max_iter, int32_t patience, int32_t check_every,
            int32_t use_graph, double avg_deg, void *ws, size_t ws_bytes, int32_t *iters_out, double *viol_out,
            double *relres_out, int32_t *status_out, dlp_stream_t stream, const void *w_lo, void *P_lo,
            int64_t ld_lo);


/* ---- (c) resident graph: edge-batch patch of the grounded system ---------------------------
 * No reference counterpart for edge updates (the reference streams vertices); closest are
 * IncrementalStream._toggle / _label_update (dynlp/stream.py:206-235). Row r owns slots
 * [rbeg[r], rcap[r]) of col/aw/w, of which [rbeg[r], rend[r]) are stored entries. aw = graph edge
 * weights (0 = deleted: a tombstone, revived by a later insertion of the edge unless its row was
 * squeezed); w = the solver
 * operator W_UU (aw masked to 0 unless both ends are in U = umask). Each applied change updates
 * rowsum[u] = sum_v w(u,v) and B[u, y_l] = sum of aw(u,l) over labelled l (both fp64, B n x K)
 * and flags changed[u] for every solved row whose equation changed. Deletions (du, dv) and
 * insertions (iu, iv, iw; iw == NULL: weight 1) are undirected; self-loops and absent deletions
 * are ignored, an insertion of a present edge sets its weight, and among repeated insertions of
 * one edge the largest batch index wins. *err (device int, caller-zeroed) reports endpoints out of
 * range; *overflow = 1 when a row ran out of slack (the edges that did not fit are not applied
 * and the graph stays consistent: rebuild with more slack and run the insertions again).
 * *n_applied (device int, may be NULL) counts applied updates. With squeeze (n bytes, zero on
 * entry and on return; may be NULL) the rows that lost entries drop them (survivors keep their order,
 * rend shrinks), so their slots serve later insertions instead of staying as tombstones. */
int dlp_graph_delete(int32_t n, const int32_t *rbeg, int32_t *rend, int32_t *col, float *aw, float *w,
                     const int32_t *du, const int32_t *dv, int32_t nd, const uint8_t *umask, const uint8_t *labeled,
                     const int32_t *y, int32_t K, double *rowsum, double *B, uint8_t *changed, int32_t *n_applied,
                     int32_t *err, uint8_t *squeeze, dlp_stream_t stream);
size_t dlp_graph_insert_workspace_bytes(int32_t ni);
int dlp_graph_insert(int32_t n, const int32_t *rbeg, int32_t *rend, const int32_t *rcap, int32_t *col, float *aw,
                     float *w, const int32_t *iu, const int32_t *iv, const float *iw, int32_t ni,
                     const uint8_t *umask, const uint8_t *labeled, const int32_t *y, int32_t K, double *rowsum,
                     double *B, uint8_t *changed, int32_t *overflow, int32_t *n_applied, int32_t *err, void *ws,
                     size_t ws_bytes, dlp_stream_t stream);

/* Membership change of the vertices T[0..nt) (in_t[v] = 1 marks them; umask already holds the new
 * U): solver weights of their entries and mirror entries follow umask, neighbours' row sums move
 * by the difference and are flagged changed, and the row sums of T are recomputed
 * (IncrementalStream._toggle, dynlp/stream.py:206-228). T == NULL: the rows u < nt with in_t[u] != 0
 * (pass nt = n; no list and no host count needed). */
int dlp_graph_toggle(const int32_t *rbeg, const int32_t *rend, const int32_t *col, const float *aw, float *w,
                     const int32_t *T, int32_t nt, const uint8_t *in_t, const uint8_t *umask, double *rowsum,
                     uint8_t *changed, dlp_stream_t stream);

/* Compact CSR of the solver operator: indptr[0..n] and the entries with w != 0 of every row, in
 * stored order (col_out/w_out must hold the number of such entries; the total slot count is a safe
 * capacity). The solver iterates on this copy, so no slack slot or inert entry is streamed. */
size_t dlp_graph_to_csr_workspace_bytes(int32_t n);
int dlp_graph_to_csr(int32_t n, const int32_t *rbeg, const int32_t *rend, const int32_t *col, const float *w,
                     int32_t *indptr, int32_t *col_out, float *w_out, void *ws, size_t ws_bytes, dlp_stream_t stream);

/* rowsum[r] = sum of w over the stored entries of r, for r = rows[g] (rows == NULL: all nr rows). */
int dlp_graph_rowsum(const int32_t *rbeg, const int32_t *rend, const float *w, const int32_t *rows, int32_t nr,
                     double *rowsum, dlp_stream_t stream);

/* The equations of the listed rows (rows == NULL: rows 0..nr-1) in the resident global-index form
 * (dynlp/stream.py:329-331): solved rows (umask) get s = sum_c B[u,c] + eta, diag = s + rowsum[u],
 * rhs[u, 0..C) = B[u, col0 .. col0+C) + eta * prior[0..C) (col0 = 1, C = 1 for the binary case,
 * stream.py:331) and, with with_h, rhs[u, C] = diag (the h column, solvers.py:312-313); inert rows
 * get diag = 1, rhs = 0 (rhs[u, C] = 1). prior is a device double[C]. fp32 copies optional. */
int dlp_system_rows(const int32_t *rows, int32_t nr, const uint8_t *umask, const double *B, int32_t K,
                    const double *rowsum, double eta, const double *prior, int32_t C, int32_t col0, int32_t with_h,
                    double *diag64, double *rhs64, int64_t ldr64, float *diag32, float *rhs32, int64_t ldr32,
                    dlp_stream_t stream);

/* Scores of rows whose membership changed: solved rows start at (prior, h0); inert rows get their
 * exact values F = 0, h = 1 (IncrementalLP._park, dynlp/solvers.py:365-368); R rows are zeroed. */
int dlp_park_rows(const int32_t *rows, int32_t nr, const uint8_t *umask, int32_t C, int32_t with_h,
                  const double *prior, double h0, double *Z, int64_t ldz, double *R, int64_t ldr,
                  dlp_stream_t stream);


/* ---- vector helpers of the refinement loop (dynlp/solvers.py:333-337) and grounding ---------
 * op 0: Y = X / scale[c] (the scaled residual, cast to Y's precision); op 1: Y += X * scale[c]
 * (Z64 += D * scale); op 2: Y = X * scale[c]; op 3: Y = X + Y * scale[c] (P = Y + beta P).
 * scale is a device double[C]. Precisions: f32/f64. */
int dlp_cols_scale(int32_t n, int32_t C, const void *X, int64_t ldx, int x_dtype, const double *scale, int32_t op,
                   void *Y, int64_t ldy, int y_dtype, dlp_stream_t stream);

/* Class-sum elimination for the refinement's corrections (no reference counterpart: the reference
 * solves every class column). On a grounded row the class right-hand sides sum to the grounding
 * (dynlp/stream.py:163-165: s = sum_c B_c + eta, rhs = B + eta * prior, sum_c prior_c = 1), so the
 * scores sum to one and the last of the K class columns follows from the others.
 * dlp_class_sum_rhs: E[:, j] = R[:, j] / scale[j] for j < K - 1 and E[:, K - 1] = R[:, K] / scale[K]
 * (R: fp64 n x (K + 1), the K classes and h; E: fp32 n x K, the classes but the last, and h).
 * dlp_class_sum_update: Z[:, j] += D[:, j] scale[j] for j < K - 1, Z[:, K] += D[:, K - 1] scale[K],
 * then Z[:, K - 1] = 1 - sum_{j < K - 1} Z[:, j] on the rows with solved[r] != 0 (every row when
 * solved is NULL) and 0 elsewhere (Z: fp64 n x (K + 1); D: fp32 n x K). 2 <= K <= 256. Asynchronous. */
int dlp_class_sum_rhs(int32_t n, int32_t K, const double *R, int64_t ldr, const double *scale, float *E,
                      int64_t lde, dlp_stream_t stream);
int dlp_class_sum_update(int32_t n, int32_t K, const float *D, int64_t ldd, const double *scale, double *Z,
                         int64_t ldz, const uint8_t *solved, dlp_stream_t stream);

/* Labels of the rows (solvers.predict, dynlp/solvers.py:166-167): binary != 0 (the K == 2 column):
 * label = F[r,0] > 0.5; otherwise the first column of the row's maximum over C columns (numpy
 * argmax). Rows with mask[r] == 0 get -1 (mask NULL: every row). labels[0..n) holds the previous
 * labels on entry and the new ones on exit; the rows whose label changed are listed in ascending
 * order in changed[0..*n_changed) (device int), and, with changed_label != NULL, their new labels in
 * changed_label[]. dtype of F: f32/f64. Workspace: dlp_predict_workspace_bytes(n). */
size_t dlp_predict_workspace_bytes(int32_t n);
int dlp_predict(int32_t n, int32_t C, const void *F, int64_t ldf, int dtype, int32_t binary, const uint8_t *mask,
                int32_t *labels, int32_t *changed, int32_t *changed_label, int32_t *n_changed, void *ws,
                size_t ws_bytes, dlp_stream_t stream);

/* Labelled vertices L entering (sign = +1) or leaving (sign = -1) the active set
 * (IncrementalStream._label_update, dynlp/stream.py:230-235): B[v, y[l]] += sign * aw(l, v) for every
 * live entry (l, v); changed[v] = 1 where umask[v] (changed may be NULL). */
int dlp_label_update(const int32_t *L, int32_t nl, double sign, const int32_t *rbeg, const int32_t *rend,
                     const int32_t *col, const float *aw, const int32_t *y, int32_t K, double *B, const uint8_t *umask,
                     uint8_t *changed, dlp_stream_t stream);

/* DynLP step 1's per-vertex scale for the m new vertices rows[0..m) (new_components,
 * dynlp/stream.py:72-76): s[i] = fp32 row-order sum over live entries (w > 0) of fp32(1 - w/wmax),
 * divided by max(count, 1), plus 1e-6. w: f32 or f64 (the term is formed in that precision). */
int dlp_new_dissim(const int32_t *rows, int32_t m, const int32_t *rbeg, const int32_t *rend, const void *w,
                   int w_dtype, double wmax, float *s, dlp_stream_t stream);

/* After dlp_cc_graph with the labelled vertices as sink: umask[v] = vmask[v] && parent[v] ==
 * parent[n] (the grounded vertices, dynlp/stream.py:150-159, :275-280); in_t[v] = 1 where membership
 * changed; *count (device int, caller-zeroed) += number of changes. */
int dlp_ground_update(int32_t n, const int32_t *parent, const uint8_t *vmask, uint8_t *umask, uint8_t *in_t,
                      int32_t *count, dlp_stream_t stream);


/* ---- (b) residual push with device-resident frontiers ------------------------------------------
 * Replaces FusedPush.run (dynlp/kernels.py:396-433; its kernels push_round + compact_frontier,
 * :269-350) with the round semantics of the synchronous push (dynlp/solvers.py:100-125): starting
 * from the candidate rows cand[0..ncand) (device, distinct), every round takes the residual of all
 * its frontier rows first,
 *   d = R[u,:] / diag[u]; Z[u,:] += d; R[u,:] = 0,
 * then pushes R[v,:] += w_uv d over their live entries, and the touched rows with
 * any_c |R[v,c]| > eps[c] * diag[v] (compared in the working precision) form the next frontier,
 * until the frontier is empty or max_rounds rounds ran. The frontiers are those of the synchronous
 * push up to the order of the floating-point atomic sums. With use_graph != 0 the rounds run as a
 * device-side loop (a CUDA graph with a conditional WHILE node; check_every unused); otherwise the
 * host reads the control block every check_every rounds. eps is a HOST array of C doubles. C <= 33.
 * (dtype, w_dtype) in {(f32,f32), (f64,f32), (f64,f64)}. Workspace: dlp_fused_push_workspace_bytes.
 * Synchronous: *rounds_out, *converged_out (1 = no row violates), *edges_out (stored entries of the
 * frontier rows, the reference's edge visits). Returns DLP_ERR_CAP when rows still violate after
 * max_rounds rounds and DLP_ERR_CANCELLED when the cancel word stopped it; in both cases the outputs
 * are filled and R is the residual of Z (every taken residual was pushed). */
size_t dlp_fused_push_workspace_bytes(int32_t n, int32_t C);
int dlp_fused_push(const int32_t *rbeg, const int32_t *rend, const int32_t *col, const void *w, int w_dtype,
                   int32_t n, int32_t C, const void *diag, void *Z, int64_t ldz, void *R, int64_t ldr, int dtype,
                   const double *eps, const int32_t *cand, int32_t ncand, int32_t max_rounds, int32_t check_every,
                   int32_t use_graph, void *ws, size_t ws_bytes, int32_t *rounds_out, int32_t *converged_out,
                   unsigned long long *edges_out, dlp_stream_t stream);
/* Totals of the last dlp_fused_push run on the workspace `ws`: out[0] = rounds, out[1] = frontier
 * rows summed over the rounds, out[2] = touched rows, out[3] = stored entries streamed (the byte
 * model of the push kernels is per frontier row, per entry and per touched row). Synchronous. */
int dlp_fused_push_counts(const void *ws, unsigned long long *out, dlp_stream_t stream);


/* ---- (e) aggregation AMG: setup and V-cycle (dynlp/amg.py) ---------------------------------
 * Heavy-edge handshake matching (amg.py:32-64) on a plain CSR (indptr/col/w fp32): `rounds`
 * rounds of mutual heaviest-admissible-neighbour choices (ties: smallest id), then unmatched
 * vertices join their heaviest matched neighbour, the rest stay single; agg[u] = rank of the
 * aggregate's representative (numpy.unique's inverse); *n_agg (device int) = number of aggregates. */
size_t dlp_amg_match_workspace_bytes(int32_t n);
int dlp_amg_match(int32_t n, const int32_t *indptr, const int32_t *col, const float *w, int32_t rounds, int32_t *agg,
                  int32_t *n_agg, void *ws, size_t ws_bytes, dlp_stream_t stream);
/* Members of each aggregate in ascending fine id: off[0..nc] and members[0..n). */
size_t dlp_amg_members_workspace_bytes(int32_t nc);
int dlp_amg_members(int32_t n, int32_t nc, const int32_t *agg, int32_t *off, int32_t *members, void *ws,
                    size_t ws_bytes, dlp_stream_t stream);
/* Galerkin coarse operator of the piecewise-constant prolongation (amg.py:67-74), in two steps:
 * plan (per-coarse-row table offsets toff[0..nc], toff[nc] = slots to provide), then coarsen:
 * W_c[a, b] = sum of w(u, v) over u in a, v in b, a != b (sorted rows, fp64 sums in a fixed order,
 * stored fp32), s_c[a] = sum of s over a (s_fine may be NULL). tkey/tval: toff[nc] slots each.
 * Both take dlp_amg_members_workspace_bytes(nc) of workspace. */
int dlp_amg_coarse_plan(int32_t nc, const int32_t *off, const int32_t *members, const int32_t *indptr, int32_t *toff,
                        void *ws, size_t ws_bytes, dlp_stream_t stream);
int dlp_amg_coarsen(int32_t nc, const int32_t *off, const int32_t *members, const int32_t *indptr, const int32_t *col,
                    const float *w, const int32_t *agg, const int32_t *toff, int32_t *tkey, double *tval,
                    int64_t total_slots, const double *s_fine, double *s_coarse, int32_t *indptr_c, int32_t *col_c,
                    float *w_c, void *ws, size_t ws_bytes, dlp_stream_t stream);
/* Sort-based Galerkin coarsening (the coalesce of dynlp/amg.py:67-74), in two calls around a stable
 * sort by key the caller runs: dlp_amg_coarse_keys writes, for each of the fine operator's stored
 * entries j (rows u < n), key[j] = agg[u] * nc + agg[col[j]] and val[j] = w[j], or key[j] = INT64_MAX
 * when both ends share an aggregate; after the stable sort (keys with their values),
 * dlp_amg_coarse_reduce sums each run of equal keys front to back in fp64 (the fine CSR order) into
 * the sorted coarse CSR (indptr_c[nc+1], col_c, w_c in fp32, *nnz_c device int), and with s_coarse,
 * s_c[a] = the fine grounding summed over the members of a in member order. m < 2^31 entries.
 * Workspace: dlp_amg_coarse_reduce_workspace_bytes(m, nc). */
int dlp_amg_coarse_keys(int32_t n, const int32_t *indptr, const int32_t *col, const float *w, const int32_t *agg,
                        int32_t nc, int64_t *key, double *val, dlp_stream_t stream);
size_t dlp_amg_coarse_reduce_workspace_bytes(int64_t m, int32_t nc);
int dlp_amg_coarse_reduce(int64_t m, const int64_t *key, const double *val, int32_t nc, const int32_t *off,
                          const int32_t *members, const double *s_fine, double *s_coarse, int32_t *indptr_c,
                          int32_t *col_c, float *w_c, int32_t *nnz_c, void *ws, size_t ws_bytes,
                          dlp_stream_t stream);

/* Stable ascending sort of m (key, value) pairs in place, keys above max_key ordered as max_key (the
 * coarsening's "no entry" marker, INT64_MAX, sorts last): LSD radix, 8 bits per pass over the bits
 * of max_key. keys_tmp / vals_tmp: m spare entries each. m < 2^30. (The sort of the reference's
 * coalesce, dynlp/graphs.py:36-44 as used by dynlp/amg.py:67-74.)
 * Workspace: dlp_sort_pairs_workspace_bytes(m). */
size_t dlp_sort_pairs_workspace_bytes(int64_t m);
int dlp_sort_pairs(int64_t m, int64_t max_key, int64_t *keys, double *vals, int64_t *keys_tmp, double *vals_tmp,
                   void *ws, size_t ws_bytes, dlp_stream_t stream);

/* V-cycle pieces (amg.py:28-31 Level.apply, :114-131 _smooth / _cycle):
 * restrict Rc[a,:] = sum over members of R (ordered); prolong X[u,:] += Xc[agg[u],:];
 * scale_rows X = omega R / diag; jacobi_sweep Y = X + omega ((RHS + W X) / diag - X);
 * dense_apply Y = M X with M a row-major fp64 nc x nc matrix (the coarsest-level inverse). */
int dlp_amg_restrict(int32_t nc, int32_t C, const int32_t *off, const int32_t *members, const void *R, int64_t ldr,
                     void *Rc, int64_t ldc, int dtype, dlp_stream_t stream);
int dlp_amg_prolong_add(int32_t n, int32_t C, const int32_t *agg, const void *Xc, int64_t ldc, void *X, int64_t ldx,
                        int dtype, dlp_stream_t stream);
int dlp_amg_scale_rows(int32_t n, int32_t C, double omega, const void *R, int64_t ldr, const void *diag, void *X,
                       int64_t ldx, int dtype, dlp_stream_t stream);
int dlp_amg_jacobi_sweep(int32_t n, int32_t C, const int32_t *indptr, const int32_t *col, const float *w,
                         const void *X, int64_t ldx, const void *RHS, int64_t ldr, const void *diag, double omega,
                         void *Y, int64_t ldy, int dtype, dlp_stream_t stream);
int dlp_dense_apply(int32_t nc, int32_t C, const double *M, const void *X, int64_t ldx, void *Y, int64_t ldy,
                    int dtype, dlp_stream_t stream);


/* ---- (e) the V-cycle and the AMG-preconditioned PCG on the device ------------------------------
 * A hierarchy is described level by level (level 0 = the operator of the solve): the level's
 * operator W as plain CSR with fp32 weights, its diagonal s + rowsum(W) in the working precision,
 * and the aggregation to the next level (agg: level row -> next-level row; off/members: the rows of
 * each next-level aggregate in ascending order). The coarsest level has no aggregation. */
typedef struct {
  int32_t n;                    /* rows of the level */
  int64_t nnz;                  /* stored entries of its W */
  const int32_t *indptr, *col;  /* W (plain CSR) */
  const float *w;
  const void *diag;             /* s + rowsum(W), working precision */
  const int32_t *agg;           /* level -> next level (NULL on the coarsest) */
  const int32_t *off, *members; /* next-level aggregates (NULL on the coarsest) */
} dlp_amg_level;

/* One V-cycle Y = M(R) (dynlp/amg.py:114-134 _smooth / _cycle): on each level X = omega R / diag,
 * nu - 1 damped Jacobi sweeps, the residual restricted to the next level, the cycle there, its result
 * prolonged and added, nu sweeps; on the coarsest level the dense fp64 inverse coarse_inv (row-major
 * n x n) when given, else coarse_sweeps sweeps. nu >= 1. dtype f32/f64 (R, Y, every diag). All
 * intermediate vectors live in the workspace: dlp_amg_vcycle_workspace_bytes(levels, nlev, C, dtype). */
size_t dlp_amg_vcycle_workspace_bytes(const dlp_amg_level *levels, int32_t nlev, int32_t C, int dtype);
int dlp_amg_vcycle(const dlp_amg_level *levels, int32_t nlev, const double *coarse_inv, int32_t nu, double omega,
                   int32_t coarse_sweeps, int32_t C, int dtype, const void *R, int64_t ldr, void *Y, int64_t ldy,
                   void *ws, size_t ws_bytes, dlp_stream_t stream);

/* Replaces solvers.pcg with the AMG preconditioner (dynlp/solvers.py:66-97, M = amg.AMG): one CG per
 * column of (diag - W) Z = rhs from the Z given, with M(R) = dlp_amg_vcycle over `levels` (level 0
 * is the operator rbeg/rend/col/w of the solve). Per iteration: AP = A P, pAp, alpha, Z += alpha P,
 * R -= alpha AP, the stop metric (mode bit 0: max_uc |R_uc| / (eps_c diag_u) <= 1; bit 1:
 * max_c ||R_c|| / rhs_norm[c] <= target_relres), Y = M(R), rz = R.Y, beta, P = Y + beta P; inner
 * products in fp64 with a fixed reduction order. With use_graph != 0 the iterations run on the device
 * as one CUDA graph with a conditional WHILE node (cached per problem), stopping at a proposed stop,
 * the patience rule (no 10% improvement in `patience` iterations), the cap or the cancel word; a
 * proposed stop is confirmed on the true residual as the reference does (solvers.py:85-89), and a
 * failed confirmation resumes from the true residual. Y is an n x C scratch like R, P and AP.
 * eps and rhs_norm are HOST arrays of C doubles. Synchronous: *status_out = 5 converged, 2 stalled,
 * 3 cap (returns DLP_ERR_CAP), 4 breakdown, 6 cancelled (returns DLP_ERR_CANCELLED).
 * Mixed precision (fp32 only), as in dlp_pcg: with w_lo (bf16 copy of w) and P_lo (bf16 n x C, ld_lo)
 * the apply gathers the bf16 mirror of P that the direction update keeps (fp32 accumulation).
 * Workspace: dlp_pcg_amg_workspace_bytes(levels, nlev, C, dtype). */
size_t dlp_pcg_amg_workspace_bytes(const dlp_amg_level *levels, int32_t nlev, int32_t C, int dtype);
int dlp_pcg_amg(const int32_t *rbeg, const int32_t *rend, const int32_t *col, const float *w, int32_t n, int32_t C,
                const void *diag, const void *rhs, int64_t ldrhs, void *Z, int64_t ldz, void *R, int64_t ldr, void *P,
                int64_t ldp, void *AP, int64_t ldap, void *Y, int64_t ldy, int dtype, const double *eps,
                const double *rhs_norm, double target_relres, int32_t mode, int32_t max_iter, int32_t patience,
                int32_t use_graph, double avg_deg, const dlp_amg_level *levels, int32_t nlev,
                const double *coarse_inv, int32_t nu, double omega, int32_t coarse_sweeps, void *ws,
                size_t ws_bytes, int32_t *iters_out, double *relres_out, int32_t *status_out,
                dlp_stream_t stream, const void *w_lo, void *P_lo, int64_t ld_lo);


/* The inverse of a dense symmetric positive definite fp64 matrix A (n x n, row-major), in place:
 * Gauss-Jordan elimination without pivoting, two launches per pivot (the coarsest AMG level's solve,
 * dynlp/amg.py:105-108 inverts it with the library's LU). Asynchronous.
 * Workspace: dlp_dense_spd_inverse_workspace_bytes(n). */
size_t dlp_dense_spd_inverse_workspace_bytes(int32_t n);
int dlp_dense_spd_inverse(int32_t n, double *A, void *ws, size_t ws_bytes, dlp_stream_t stream);


/* ---- batched independent solves (config: many instances in one launch sequence) -------------
 * No reference counterpart (the reference solves one system at a time). Block PCG with the Jacobi
 * preconditioner over a concatenated block-diagonal CSR (indptr/col/w fp32, N rows, C <= 64
 * columns) holding `ninst` independent systems. Rows are cut into `ntiles` tiles that never
 * straddle two instances: tile t covers rows [tile_beg[t], tile_end[t]) of instance tile_inst[t],
 * and instance i owns tiles [inst_tiles[i], inst_tiles[i+1]) (inst_tiles has ninst + 1 entries).
 * Every instance runs its own CG (its own alpha, beta and stop state; reductions per instance in
 * a fixed tile order, so an instance gets the iterates it would get alone) until the stop rule
 * `mode` (as in dlp_pcg; eps_dev and rhs_norm_dev are DEVICE arrays of ninst x C doubles) holds,
 * confirmed on its true residual. Synchronous: per-instance iterations, status (5 converged,
 * 2 stalled, 3 cap, 4 breakdown) and relative residuals are written to HOST arrays of ninst. */
size_t dlp_pcg_batched_workspace_bytes(int32_t ninst, int32_t ntiles, int32_t C);
int dlp_pcg_batched(const int32_t *indptr, const int32_t *col, const float *w, int32_t N, int32_t C, const void *diag,
                    const void *rhs, int64_t ldrhs, void *Z, int64_t ldz, void *R, int64_t ldr, void *P, int64_t ldp,
                    void *AP, int64_t ldap, int dtype, int32_t ninst, int32_t ntiles, const int32_t *tile_inst,
                    const int32_t *tile_beg, const int32_t *tile_end, const int32_t *inst_tiles,
                    const double *eps_dev, const double *rhs_norm_dev, double target_relres, int32_t mode,
                    int32_t max_iter, int32_t patience, int32_t check_every, int32_t use_graph, int32_t group,
                    double avg_deg, void *ws, size_t ws_bytes, int32_t *iters_out, int32_t *status_out,
                    double *relres_out, dlp_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* DLP_H */
