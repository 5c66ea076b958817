// Residual push with device-resident frontiers: the work behind FusedPush.run (dynlp/kernels.py:396-433)
// with the round semantics of the synchronous push (dynlp/solvers.py:100-125).
//
// A round moves the residual of every frontier row u into its score and onto its neighbours:
//   d_u = R[u,:] / diag[u];  Z[u,:] += d_u;  R[u,:] = 0;  R[v,:] += w_uv d_u for every live entry (u, v)
// and the next frontier is the set of rows the round touched that still violate
// |R[v,c]| > eps[c] * diag[v] for some column c.
//
// Rounds are synchronous: every frontier row's residual is taken before any push of the round
// lands, so the sequence of frontiers is the one the synchronous push defines (up to the order of
// the floating-point atomic sums), not a schedule-dependent relaxation. Each round is two launches:
//   k_push_scatter  one group of G lanes per frontier row streams the row's entries, adds w * d
//                   into the neighbours' residual rows (16-byte vector atomics where the rows allow),
//                   and records first touches in a bitmap; the touched rows go to a list through
//                   warp-aggregated appends (one atomic per warp);
//   k_push_sift     one thread per touched row clears its bit, tests the row and, when it violates,
//                   takes its residual for the next round at a slot reserved by a warp-aggregated
//                   append: the next frontier's scaled residuals d are stored compactly (D), so the
//                   scatter reads them as rows and no take races a push.
// Counters live in a control block on the device with two copies of the frontier and touched
// counts; the round of one parity resets the copies the other parity fills next, so the rounds chain
// without the host. The loop itself runs on the device: a CUDA graph with a WHILE conditional node
// around two rounds; the scatter that finds the frontier empty (or the run stopped) clears the loop
// flag. The round cap and the host's cancel word are checked where a round would take residuals,
// so a stopped run never leaves a taken residual unpushed: R stays the residual of Z.
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "common.cuh"

namespace dlp {

constexpr int kPushThreads = 256;
constexpr int kPushBody = 2;  // rounds per pass of the device-side loop (an even count: parities alternate)
// Lanes per frontier row. Eight: the graphs of the workloads have mean degrees of 8 to 32, and a
// row's entries are streamed in ceil(degree / 8) warp-uniform steps.
constexpr int kPushGroup = 8;

enum { kRunning = 0, kConverged = 1, kCapped = 2, kCancelled = 3 };

struct PushCtl {
  int32_t rounds;      // rounds whose scatter ran
  int32_t max_rounds;
  int32_t status;      // kRunning, kConverged, kCapped, kCancelled
  int32_t pad;
  int32_t fcnt[2];     // frontier size for the round of each parity
  int32_t tcnt[2];     // touched rows of the round of each parity
  unsigned long long edges;          // stored entries streamed (the reference's edge visits)
  unsigned long long frontier_rows;  // sum of the frontier sizes of the rounds run
  unsigned long long touched_rows;   // sum of the touched-list sizes
};

template <typename T>
struct PushArgs {
  const int32_t *rbeg, *rend, *col;
  const void *w;
  const T *diag;
  T *Z;
  int64_t ldz;
  T *R;
  int64_t ldr;
  int32_t C;
  const double *eps;
  int32_t *front;    // frontier rows (n)
  T *D;              // their scaled residuals, C per row (n x C)
  int32_t *touched;  // touched rows (n)
  uint32_t *bits;    // first-touch bitmap (ceil(n / 32) words; zero between rounds)
  PushCtl *ctl;
  const int32_t *cancel;
  cudaGraphConditionalHandle cond;
  int has_cond;
};

// R[v, 0..C) += s * d[0..C): 16-byte vector atomics over whole groups of four (the row must start on
// a 16-byte boundary), then the remaining columns one by one. Only the C columns are written.
template <typename T, int CMAX, bool VEC4>
__device__ __forceinline__ void push_row(T *r, const T (&d)[CMAX], T s, int C) {
  int c0 = 0;
  if constexpr (VEC4 && sizeof(T) == 4) {
#pragma unroll
    for (int c = 0; c + 4 <= CMAX; c += 4) {
      if (c + 4 <= C) {
        atomicAdd(reinterpret_cast<float4 *>(r + c), make_float4(s * d[c], s * d[c + 1], s * d[c + 2], s * d[c + 3]));
        c0 = c + 4;
      }
    }
  }
#pragma unroll
  for (int c = 0; c < CMAX; ++c)
    if (c >= c0 && c < C) atomic_add(r + c, s * d[c]);
}

template <typename TW, typename T, int CMAX, int G, bool VEC4>
__global__ void __launch_bounds__(kPushThreads) k_push_scatter(PushArgs<T> a, int p) {
  PushCtl *ctl = a.ctl;
  const int q = p ^ 1;
  const int nf = ctl->fcnt[p];
  const int status = ctl->status;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ctl->fcnt[q] = 0;  // this round's sift fills the next frontier
    ctl->tcnt[q] = 0;  // and the next round's scatter the next touched list
    if (status != kRunning || nf == 0) {
      if (status == kRunning) ctl->status = kConverged;
      if (a.has_cond) cudaGraphSetConditional(a.cond, 0u);
    } else {
      ctl->rounds += 1;
      ctl->frontier_rows += (unsigned long long)nf;
    }
  }
  if (status != kRunning || nf == 0) return;
  const TW *__restrict__ w = (const TW *)a.w;
  const int lane = lane_id();
  const int gl = lane % G;  // lane within the row's group
  constexpr int kGroups = 32 / G;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long stride = (((long long)gridDim.x * blockDim.x) >> 5) * kGroups;
  unsigned long long my_edges = 0;
  for (long long base = warp * kGroups; base < nf; base += stride) {  // warp-uniform bounds
    const long long g = base + lane / G;
    const bool valid = g < nf;
    int beg = 0, end = 0;
    T d[CMAX];
#pragma unroll
    for (int c = 0; c < CMAX; ++c) d[c] = T(0);
    if (valid) {
      const int u = a.front[g];
      beg = a.rbeg[u];
      end = a.rend[u];
      const T *dr = a.D + g * a.C;
#pragma unroll
      for (int c = 0; c < CMAX; ++c)
        if (c < a.C) d[c] = dr[c];
      if (gl == 0) my_edges += (unsigned long long)(end - beg);
    }
    int trips = valid ? (end - beg + G - 1) / G : 0;
    trips = __reduce_max_sync(0xffffffffu, trips);
    for (int t = 0; t < trips; ++t) {
      const int j = beg + gl + t * G;
      bool first = false;
      int32_t v = 0;
      if (j < end) {
        const T wv = cvt<T>(w[j]);
        if (wv != T(0)) {  // inert entries (deleted edges, edges leaving the solved set) carry nothing
          v = a.col[j];
          push_row<T, CMAX, VEC4>(a.R + (long long)v * a.ldr, d, wv, a.C);
          const uint32_t bit = 1u << (v & 31);
          first = (atomicOr(a.bits + (v >> 5), bit) & bit) == 0u;
        }
      }
      warp_append(first, v, a.touched, &ctl->tcnt[p]);
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) my_edges += __shfl_xor_sync(0xffffffffu, my_edges, off);
  if (lane == 0 && my_edges) atomicAdd(&ctl->edges, my_edges);
}

// The take of one row: d = R[v,:] / diag[v] stored at D[slot,:]; Z[v,:] += d; R[v,:] = 0.
template <typename T>
__device__ __forceinline__ void take_row(const PushArgs<T> &a, int32_t v, int slot, T dv) {
  T *r = a.R + (long long)v * a.ldr;
  T *z = a.Z + (long long)v * a.ldz;
  T *dd = a.D + (long long)slot * a.C;
  for (int c = 0; c < a.C; ++c) {
    const T x = r[c] / dv;
    dd[c] = x;
    z[c] += x;
    r[c] = T(0);
  }
}

template <typename T>
__global__ void __launch_bounds__(kPushThreads) k_push_sift(PushArgs<T> a, int p) {
  PushCtl *ctl = a.ctl;
  const int q = p ^ 1;
  const int nt = ctl->tcnt[p];
  __shared__ int s_allow;
  if (threadIdx.x == 0) {
    const int cancelled = read_cancel(a.cancel);
    s_allow = cancelled ? -kCancelled : (ctl->rounds < ctl->max_rounds ? 1 : -kCapped);
    if (blockIdx.x == 0) ctl->touched_rows += (unsigned long long)nt;
  }
  __syncthreads();
  const int allow = s_allow;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long b = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); b < nt; b += stride) {
    const long long i = b + (threadIdx.x & 31);
    bool viol = false;
    int32_t v = 0;
    T dv = T(1);
    if (i < nt) {
      v = a.touched[i];
      atomicAnd(a.bits + (v >> 5), ~(1u << (v & 31)));
      dv = a.diag[v];
      const T *r = a.R + (long long)v * a.ldr;
      // in the working precision, as the synchronous push compares (dynlp/solvers.py:105-106)
      for (int c = 0; c < a.C; ++c) viol |= fabs(r[c]) > (T)a.eps[c] * dv;
    }
    if (allow < 0) {
      if (viol) ctl->status = -allow;  // a violating row is left for a round that will not run
      continue;
    }
    const int slot = warp_reserve(viol, &ctl->fcnt[q]);
    if (viol) {
      a.front[slot] = v;
      take_row(a, v, slot, dv);
    }
  }
}

// The first round's take: the candidate rows cand[0..nc) become the frontier of parity 0.
template <typename T>
__global__ void __launch_bounds__(kPushThreads) k_push_seed(PushArgs<T> a, const int32_t *__restrict__ cand, int nc) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nc) return;
  const int32_t u = cand[g];
  a.front[g] = u;
  take_row(a, u, (int)g, a.diag[u]);
}

// ---- host side ----------------------------------------------------------------------------------
static size_t al256(size_t x) { return (x + 255) / 256 * 256; }

struct PushWs {
  PushCtl *ctl;
  double *eps;
  int32_t *front, *touched;
  uint32_t *bits;
  void *D;
};

static size_t push_ws_bytes(int32_t n, int32_t C, size_t elem) {
  const size_t nn = (size_t)(n > 0 ? n : 1), cc = (size_t)(C > 0 ? C : 1);
  return al256(sizeof(PushCtl)) + al256(sizeof(double) * cc) + 2 * al256(sizeof(int32_t) * nn) +
         al256(sizeof(uint32_t) * ((nn + 31) / 32)) + al256(elem * nn * cc);
}

static PushWs carve_push(void *ws, int32_t n, int32_t C) {
  const size_t nn = (size_t)(n > 0 ? n : 1), cc = (size_t)(C > 0 ? C : 1);
  char *p = (char *)ws;
  PushWs W;
  W.ctl = (PushCtl *)p;
  p += al256(sizeof(PushCtl));
  W.eps = (double *)p;
  p += al256(sizeof(double) * cc);
  W.front = (int32_t *)p;
  p += al256(sizeof(int32_t) * nn);
  W.touched = (int32_t *)p;
  p += al256(sizeof(int32_t) * nn);
  W.bits = (uint32_t *)p;
  p += al256(sizeof(uint32_t) * ((nn + 31) / 32));
  W.D = p;
  return W;
}

struct PushProblem {
  const int32_t *rbeg, *rend, *col;
  const void *w;
  int w_dtype;
  int32_t n, C;
  const void *diag;
  void *Z;
  int64_t ldz;
  void *R;
  int64_t ldr;
  int dtype;
};

template <typename T>
static PushArgs<T> push_args(const PushProblem &q, const PushWs &W, const int32_t *cancel,
                             cudaGraphConditionalHandle cond, int has_cond) {
  PushArgs<T> a;
  a.rbeg = q.rbeg;
  a.rend = q.rend;
  a.col = q.col;
  a.w = q.w;
  a.diag = (const T *)q.diag;
  a.Z = (T *)q.Z;
  a.ldz = q.ldz;
  a.R = (T *)q.R;
  a.ldr = q.ldr;
  a.C = q.C;
  a.eps = W.eps;
  a.front = W.front;
  a.D = (T *)W.D;
  a.touched = W.touched;
  a.bits = W.bits;
  a.ctl = W.ctl;
  a.cancel = cancel;
  a.cond = cond;
  a.has_cond = has_cond;
  return a;
}

static bool vec4_ok(const PushProblem &q) {
  return q.dtype == DLP_F32 && q.ldr % 4 == 0 && ((uintptr_t)q.R & 15u) == 0;
}

template <typename TW, typename T, int CMAX, int G, bool VEC4>
static void launch_round_t(const PushArgs<T> &a, int p, int grid, cudaStream_t s) {
  k_push_scatter<TW, T, CMAX, G, VEC4><<<grid, kPushThreads, 0, s>>>(a, p);
  k_push_sift<T><<<grid, kPushThreads, 0, s>>>(a, p);
}

template <typename TW, typename T, int CMAX>
static void launch_round_g(const PushProblem &q, const PushArgs<T> &a, int p, int grid, cudaStream_t s) {
  if (vec4_ok(q)) launch_round_t<TW, T, CMAX, kPushGroup, true>(a, p, grid, s);
  else launch_round_t<TW, T, CMAX, kPushGroup, false>(a, p, grid, s);
}

template <typename TW, typename T>
static int launch_round_c(const PushProblem &q, const PushArgs<T> &a, int p, int grid, cudaStream_t s) {
  if (q.C <= 4) launch_round_g<TW, T, 4>(q, a, p, grid, s);
  else if (q.C <= 12) launch_round_g<TW, T, 12>(q, a, p, grid, s);
  else if (q.C <= 20) launch_round_g<TW, T, 20>(q, a, p, grid, s);
  else if (q.C <= 33) launch_round_g<TW, T, 33>(q, a, p, grid, s);
  else return DLP_ERR_INVALID;
  return check_launch(2);
}

// One round of parity p (scatter + sift).
static int launch_round(const PushProblem &q, const PushWs &W, const int32_t *cancel, cudaGraphConditionalHandle cond,
                        int has_cond, int p, int grid, cudaStream_t s) {
  if (q.dtype == DLP_F32 && q.w_dtype == DLP_F32)
    return launch_round_c<float, float>(q, push_args<float>(q, W, cancel, cond, has_cond), p, grid, s);
  if (q.dtype == DLP_F64 && q.w_dtype == DLP_F32)
    return launch_round_c<float, double>(q, push_args<double>(q, W, cancel, cond, has_cond), p, grid, s);
  if (q.dtype == DLP_F64 && q.w_dtype == DLP_F64)
    return launch_round_c<double, double>(q, push_args<double>(q, W, cancel, cond, has_cond), p, grid, s);
  return DLP_ERR_DTYPE;
}

static int launch_seed(const PushProblem &q, const PushWs &W, const int32_t *cand, int nc, cudaStream_t s) {
  const int grid = ceil_div_i(nc, kPushThreads);
  if (q.dtype == DLP_F32)
    k_push_seed<float><<<grid, kPushThreads, 0, s>>>(push_args<float>(q, W, nullptr, 0, 0), cand, nc);
  else
    k_push_seed<double><<<grid, kPushThreads, 0, s>>>(push_args<double>(q, W, nullptr, 0, 0), cand, nc);
  return check_launch();
}

// Cache of instantiated loop graphs, one per problem signature. Entries are shared references: an
// eviction drops the cache's reference only, and a graph another thread is replaying stays alive
// until that thread lets go of its own reference.
struct PushKey {
  std::vector<uintptr_t> v;
  bool operator==(const PushKey &o) const { return v == o.v; }
};
struct PushKeyHash {
  size_t operator()(const PushKey &k) const {
    size_t h = 1469598103934665603ull;
    for (auto x : k.v) h = (h ^ x) * 1099511628211ull;
    return h;
  }
};

static std::mutex g_push_mu;
static std::unordered_map<PushKey, GraphRef, PushKeyHash> g_push_graphs;
static cudaStream_t g_push_capture[64];

static int push_loop_graph(const PushProblem &q, const PushWs &W, const int32_t *cancel, int grid, GraphRef *out) {
  int dev = 0;
  DLP_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return DLP_ERR_INVALID;
  PushKey key{{(uintptr_t)dev, (uintptr_t)q.rbeg, (uintptr_t)q.rend, (uintptr_t)q.col, (uintptr_t)q.w,
               (uintptr_t)q.w_dtype, (uintptr_t)q.n, (uintptr_t)q.C, (uintptr_t)q.diag, (uintptr_t)q.Z,
               (uintptr_t)q.ldz, (uintptr_t)q.R, (uintptr_t)q.ldr, (uintptr_t)q.dtype, (uintptr_t)W.ctl,
               (uintptr_t)cancel, (uintptr_t)grid}};
  std::lock_guard<std::mutex> lk(g_push_mu);
  auto it = g_push_graphs.find(key);
  if (it != g_push_graphs.end()) {
    *out = it->second;
    return DLP_OK;
  }
  if (!g_push_capture[dev]) DLP_CUDA(cudaStreamCreateWithFlags(&g_push_capture[dev], cudaStreamNonBlocking));
  cudaStream_t cs = g_push_capture[dev];
  cudaGraph_t g = nullptr;
  DLP_CUDA(cudaGraphCreate(&g, 0));
  auto fail = [&](cudaError_t e) {
    cudaGraphDestroy(g);
    set_cuda_error(e);
    return DLP_ERR_CUDA;
  };
  cudaGraphConditionalHandle h = 0;
  cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 1u, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) return fail(e);
  cudaGraphNodeParams np{};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node = nullptr;
  e = cudaGraphAddNode(&node, g, nullptr, 0, &np);
  if (e != cudaSuccess) return fail(e);
  e = cudaStreamBeginCaptureToGraph(cs, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                    cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return fail(e);
  int st = DLP_OK;
  for (int r = 0; r < kPushBody && st == DLP_OK; ++r) st = launch_round(q, W, cancel, h, 1, r & 1, grid, cs);
  cudaGraph_t captured = nullptr;
  e = cudaStreamEndCapture(cs, &captured);
  if (st != DLP_OK) {
    cudaGraphDestroy(g);
    return st;
  }
  if (e != cudaSuccess) return fail(e);
  cudaGraphExec_t ex = nullptr;
  e = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    set_cuda_error(e);
    return DLP_ERR_CUDA;
  }
  auto ref = std::make_shared<GraphExec>();
  ref->ex = ex;
  if (g_push_graphs.size() >= 32) g_push_graphs.clear();  // holders keep their own references
  g_push_graphs.emplace(key, ref);
  *out = ref;
  return DLP_OK;
}

}  // namespace dlp

using namespace dlp;

extern "C" {

size_t dlp_fused_push_workspace_bytes(int32_t n, int32_t C) { return push_ws_bytes(n, C, sizeof(double)); }

int dlp_fused_push(const int32_t *rbeg, const int32_t *rend, const int32_t *col, const void *w, int w_dtype,
                   int32_t n, int32_t C, const void *diag, void *Z, int64_t ldz, void *R, int64_t ldr, int dtype,
                   const double *eps, const int32_t *cand, int32_t ncand, int32_t max_rounds, int32_t check_every,
                   int32_t use_graph, void *ws, size_t ws_bytes, int32_t *rounds_out, int32_t *converged_out,
                   unsigned long long *edges_out, dlp_stream_t stream) {
  if (n < 0 || C <= 0 || C > 33 || ldz < C || ldr < C || ncand < 0 || ncand > n || !eps) return DLP_ERR_INVALID;
  if (!(dtype == DLP_F32 && w_dtype == DLP_F32) && !(dtype == DLP_F64 && (w_dtype == DLP_F32 || w_dtype == DLP_F64)))
    return DLP_ERR_DTYPE;
  if (!ws || ws_bytes < push_ws_bytes(n, C, sizeof(double))) return DLP_ERR_WORKSPACE;
  if (rounds_out) *rounds_out = 0;
  if (converged_out) *converged_out = 1;
  if (edges_out) *edges_out = 0;
  if (ncand == 0) return DLP_OK;
  if (!rbeg || !rend || !col || !w || !diag || !Z || !R || !cand) return DLP_ERR_INVALID;
  if (converged_out) *converged_out = 0;
  if (max_rounds <= 0) return DLP_ERR_CAP;
  cudaStream_t s = (cudaStream_t)stream;
  PushProblem q{rbeg, rend, col, w, w_dtype, n, C, diag, Z, ldz, R, ldr, dtype};
  PushWs W = carve_push(ws, n, C);
  const int32_t *cancel = cancel_word();
  PushCtl h{};
  h.max_rounds = max_rounds;
  h.fcnt[0] = ncand;
  DLP_CUDA(cudaMemcpyAsync(W.ctl, &h, sizeof(h), cudaMemcpyHostToDevice, s));
  DLP_CUDA(cudaMemcpyAsync(W.eps, eps, sizeof(double) * (size_t)C, cudaMemcpyHostToDevice, s));
  DLP_CUDA(cudaMemsetAsync(W.bits, 0, sizeof(uint32_t) * (((size_t)n + 31) / 32), s));
  DLP_TRY(launch_seed(q, W, cand, ncand, s));
  const int grid = sm_count() * 8;
  GraphRef loop;
  if (use_graph) DLP_TRY(push_loop_graph(q, W, cancel, grid, &loop));
  PushCtl out{};
  if (loop) {
    // the loop stops itself: every pass either runs rounds or ends the run, and a run ends at the
    // round cap at the latest
    DLP_CUDA(cudaGraphLaunch(loop->ex, s));
    note_launches(2ull * kPushBody);
  } else {
    const int every = check_every > 0 ? check_every : 8;
    for (long long r = 0; r <= (long long)max_rounds + 1; r += 2 * ((every + 1) / 2)) {
      for (int i = 0; i < (every + 1) / 2; ++i) {
        DLP_TRY(launch_round(q, W, cancel, 0, 0, 0, grid, s));
        DLP_TRY(launch_round(q, W, cancel, 0, 0, 1, grid, s));
      }
      DLP_CUDA(cudaMemcpyAsync(&out, W.ctl, sizeof(out), cudaMemcpyDeviceToHost, s));
      DLP_CUDA(cudaStreamSynchronize(s));
      if (out.status != kRunning) break;
    }
  }
  DLP_CUDA(cudaMemcpyAsync(&out, W.ctl, sizeof(out), cudaMemcpyDeviceToHost, s));
  DLP_CUDA(cudaStreamSynchronize(s));
  if (rounds_out) *rounds_out = out.rounds;
  if (converged_out) *converged_out = out.status == kConverged ? 1 : 0;
  if (edges_out) *edges_out = out.edges;
  if (out.status == kCapped) return DLP_ERR_CAP;
  if (out.status == kCancelled) return DLP_ERR_CANCELLED;
  if (out.status != kConverged) return DLP_ERR_DEVICE;  // the loop ended without a decision
  return DLP_OK;
}

int dlp_fused_push_counts(const void *ws, unsigned long long *out, dlp_stream_t stream) {
  if (!ws || !out) return DLP_ERR_INVALID;
  PushCtl c{};
  cudaStream_t s = (cudaStream_t)stream;
  DLP_CUDA(cudaMemcpyAsync(&c, ws, sizeof(c), cudaMemcpyDeviceToHost, s));
  DLP_CUDA(cudaStreamSynchronize(s));
  out[0] = (unsigned long long)c.rounds;
  out[1] = c.frontier_rows;
  out[2] = c.touched_rows;
  out[3] = c.edges;
  return DLP_OK;
}

}  // extern "C"
