// Asynchronous residual push with device-resident frontiers (FusedPush, dynlp/kernels.py:269-350,
// :396-433). Each round takes the residual of every frontier vertex (atomicExch, so pushes landing
// during the round are kept for the next one), adds r/diag to its score and scatters w*r/diag to
// its neighbours with atomics; the first touch of a neighbour appends it to the touched list. A
// compaction then keeps the touched vertices that still violate |r_c| > eps_c * diag. Appends are
// warp-aggregated (one atomic per warp). Frontier and touched counters are double-buffered and each
// kernel resets the counter the other one fills next, so rounds chain without host work; a chunk of
// rounds is replayed as a CUDA graph and the host reads one counter per chunk.
// The relaxation is chaotic (schedule-dependent), like the reference's; the residual stays exact up
// to rounding, which is what the stop test reads.
#include <cstdio>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "common.cuh"

namespace dlp {

constexpr int kPushThreads = 256;
constexpr int kPushGroup = 8;  // lanes per frontier vertex

template <typename TW, typename T, int CMAX>
__global__ void __launch_bounds__(kPushThreads)
    k_push_round(const int32_t *__restrict__ rbeg, const int32_t *__restrict__ rend, const int32_t *__restrict__ col,
                 const TW *__restrict__ w, const T *__restrict__ diag, const int32_t *__restrict__ frontier,
                 const int32_t *fcount, int32_t *fcount_next, T *Z, int64_t ldz, T *R, int64_t ldr, int32_t C,
                 int32_t *mark, int32_t *touched, int32_t *tcount, unsigned long long *edges) {
  const int nf = *fcount;
  if (blockIdx.x == 0 && threadIdx.x == 0) *fcount_next = 0;
  const int lane_w = threadIdx.x & 31;
  const int lane = lane_w % kPushGroup;
  const int gbase = lane_w - lane;
  constexpr int gpw = 32 / kPushGroup;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long stride = (((long long)gridDim.x * blockDim.x) >> 5) * gpw;
  unsigned long long my_edges = 0;
  for (long long g0 = warp * gpw; g0 < nf; g0 += stride) {  // warp-uniform
    const long long g = g0 + lane_w / kPushGroup;
    const bool valid = g < nf;
    const int u = valid ? frontier[g] : 0;
    T d[CMAX];
#pragma unroll
    for (int c = 0; c < CMAX; ++c) d[c] = T(0);
    if (valid && lane == 0) {
      const T dv = diag[u];
#pragma unroll
      for (int c = 0; c < CMAX; ++c) {
        if (c < C) {
          T r;
          if constexpr (sizeof(T) == 8)
            r = __longlong_as_double((long long)atomicExch((unsigned long long *)&R[(long long)u * ldr + c], 0ull));
          else
            r = atomicExch(&R[(long long)u * ldr + c], 0.0f);
          d[c] = r / dv;
          Z[(long long)u * ldz + c] += d[c];
        }
      }
    }
#pragma unroll
    for (int c = 0; c < CMAX; ++c)
      if (c < C) d[c] = __shfl_sync(0xffffffffu, d[c], gbase);
    if (valid) {
      const int beg = rbeg[u], end = rend[u];
      if (lane == 0) my_edges += (unsigned long long)(end - beg);
      for (int j = beg + lane; j < end; j += kPushGroup) {
        const T wv = cvt<T>(w[j]);
        if (wv == T(0)) continue;  // inert entries (outside U, deleted edges)
        const long long v = col[j];
#pragma unroll
        for (int c = 0; c < CMAX; ++c)
          if (c < C) atomic_add(&R[v * ldr + c], wv * d[c]);
        const bool first = atomicExch(&mark[v], 1) == 0;
        if (first) touched[atomicAdd(tcount, 1)] = (int32_t)v;
      }
    }
  }
  // one edge-counter atomic per warp
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) my_edges += __shfl_xor_sync(0xffffffffu, my_edges, off);
  if (lane_w == 0 && my_edges) atomicAdd(edges, my_edges);
}

template <typename T>
__global__ void __launch_bounds__(kPushThreads)
    k_push_compact(const int32_t *__restrict__ touched, const int32_t *tcount, int32_t *tcount_next, int32_t *mark,
                   const T *R, int64_t ldr, int32_t C, const T *__restrict__ diag, const double *__restrict__ eps,
                   int32_t *out, int32_t *fcount_out) {
  const int nt = *tcount;
  if (blockIdx.x == 0 && threadIdx.x == 0) *tcount_next = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  // warp-uniform trip count so the aggregated append sees whole warps
  const long long base0 = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31);
  for (long long b = base0; b < nt; b += stride) {
    const long long i = b + (threadIdx.x & 31);
    bool viol = false;
    int32_t v = 0;
    if (i < nt) {
      v = touched[i];
      mark[v] = 0;
      const T dv = diag[v];
      for (int c = 0; c < C; ++c) viol |= fabs(R[(long long)v * ldr + c]) > (T)eps[c] * dv;
    }
    warp_append(viol, v, out, fcount_out);
  }
}

struct PushWs {
  int32_t *front0, *front1, *touched, *mark, *cnt;  // cnt: fcnt[2], tcnt[2]
  unsigned long long *edges;
  double *eps;
};

static size_t al256(size_t x) { return (x + 255) / 256 * 256; }

static size_t push_ws_bytes(int32_t n, int32_t C) {
  return 4 * al256(sizeof(int32_t) * (size_t)(n > 0 ? n : 1)) + al256(sizeof(int32_t) * 4) +
         al256(sizeof(unsigned long long)) + al256(sizeof(double) * (size_t)(C > 0 ? C : 1));
}

static PushWs carve_push(void *ws, int32_t n, int32_t C) {
  char *p = (char *)ws;
  PushWs W;
  const size_t vn = al256(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  W.front0 = (int32_t *)p;
  p += vn;
  W.front1 = (int32_t *)p;
  p += vn;
  W.touched = (int32_t *)p;
  p += vn;
  W.mark = (int32_t *)p;
  p += vn;
  W.cnt = (int32_t *)p;
  p += al256(sizeof(int32_t) * 4);
  W.edges = (unsigned long long *)p;
  p += al256(sizeof(unsigned long long));
  W.eps = (double *)p;
  (void)C;
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

template <typename TW, typename T, int CMAX>
static void launch_round_t(const PushProblem &q, const PushWs &W, int p, int grid, cudaStream_t s) {
  int32_t *front[2] = {W.front0, W.front1};
  const int qq = 1 - p;
  k_push_round<TW, T, CMAX><<<grid, kPushThreads, 0, s>>>(
      q.rbeg, q.rend, q.col, (const TW *)q.w, (const T *)q.diag, front[p], W.cnt + p, W.cnt + qq, (T *)q.Z, q.ldz,
      (T *)q.R, q.ldr, q.C, W.mark, W.touched, W.cnt + 2 + p, W.edges);
  k_push_compact<T><<<grid, kPushThreads, 0, s>>>(W.touched, W.cnt + 2 + p, W.cnt + 2 + qq, W.mark, (const T *)q.R,
                                                   q.ldr, q.C, (const T *)q.diag, W.eps, front[qq], W.cnt + qq);
}

template <typename TW, typename T>
static int launch_round_c(const PushProblem &q, const PushWs &W, int p, int grid, cudaStream_t s) {
  if (q.C <= 4) launch_round_t<TW, T, 4>(q, W, p, grid, s);
  else if (q.C <= 9) launch_round_t<TW, T, 9>(q, W, p, grid, s);
  else if (q.C <= 17) launch_round_t<TW, T, 17>(q, W, p, grid, s);
  else if (q.C <= 33) launch_round_t<TW, T, 33>(q, W, p, grid, s);
  else return DLP_ERR_INVALID;
  return check_launch(2);
}

static int launch_round(const PushProblem &q, const PushWs &W, int p, int grid, cudaStream_t s) {
  if (q.dtype == DLP_F32 && q.w_dtype == DLP_F32) return launch_round_c<float, float>(q, W, p, grid, s);
  if (q.dtype == DLP_F64 && q.w_dtype == DLP_F32) return launch_round_c<float, double>(q, W, p, grid, s);
  if (q.dtype == DLP_F64 && q.w_dtype == DLP_F64) return launch_round_c<double, double>(q, W, p, grid, s);
  return DLP_ERR_DTYPE;
}

static std::mutex g_push_mu;
static std::unordered_map<std::string, cudaGraphExec_t> g_push_graphs;
static cudaStream_t g_push_capture[64];

static int push_chunk_graph(const PushProblem &q, const PushWs &W, int pairs, int grid, cudaGraphExec_t *out) {
  int dev = 0;
  DLP_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return DLP_ERR_INVALID;
  char key[512];
  snprintf(key, sizeof(key), "%d|%p|%p|%p|%p|%d|%d|%d|%p|%p|%lld|%p|%lld|%d|%p|%d|%d", dev, (const void *)q.rbeg,
           (const void *)q.rend, (const void *)q.col, q.w, q.w_dtype, q.n, q.C, q.diag, q.Z, (long long)q.ldz, q.R,
           (long long)q.ldr, q.dtype, (void *)W.front0, pairs, grid);
  std::lock_guard<std::mutex> lk(g_push_mu);
  auto it = g_push_graphs.find(key);
  if (it != g_push_graphs.end()) {
    *out = it->second;
    return DLP_OK;
  }
  if (!g_push_capture[dev]) DLP_CUDA(cudaStreamCreateWithFlags(&g_push_capture[dev], cudaStreamNonBlocking));
  cudaStream_t cs = g_push_capture[dev];
  DLP_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  int st = DLP_OK;
  for (int i = 0; i < pairs && st == DLP_OK; ++i) {
    st = launch_round(q, W, 0, grid, cs);
    if (st == DLP_OK) st = launch_round(q, W, 1, grid, cs);
  }
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(cs, &g);
  if (st != DLP_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  if (e != cudaSuccess) {
    set_cuda_error(e);
    return DLP_ERR_CUDA;
  }
  cudaGraphExec_t ex = nullptr;
  const cudaError_t e2 = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (e2 != cudaSuccess) {
    set_cuda_error(e2);
    return DLP_ERR_CUDA;
  }
  if (g_push_graphs.size() >= 32) {
    for (auto &kv : g_push_graphs) cudaGraphExecDestroy(kv.second);
    g_push_graphs.clear();
  }
  g_push_graphs.emplace(key, ex);
  *out = ex;
  return DLP_OK;
}

}  // namespace dlp

using namespace dlp;

extern "C" {

size_t dlp_fused_push_workspace_bytes(int32_t n, int32_t C) { return push_ws_bytes(n, C); }

int dlp_fused_push(const int32_t *rbeg, const int32_t *rend, const int32_t *col, const void *w, int w_dtype,
                   int32_t n, int32_t C, const void *diag, void *Z, int64_t ldz, void *R, int64_t ldr, int dtype,
                   const double *eps, const int32_t *cand, int32_t ncand, int32_t max_rounds, int32_t check_every,
                   int32_t use_graph, void *ws, size_t ws_bytes, int32_t *rounds_out, int32_t *converged_out,
                   unsigned long long *edges_out, dlp_stream_t stream) {
  if (n < 0 || C <= 0 || C > 33 || ldz < C || ldr < C || ncand < 0 || ncand > n || !eps) return DLP_ERR_INVALID;
  if (!ws || ws_bytes < push_ws_bytes(n, C)) return DLP_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  PushProblem q{rbeg, rend, col, w, w_dtype, n, C, diag, Z, ldz, R, ldr, dtype};
  PushWs W = carve_push(ws, n, C);
  if (rounds_out) *rounds_out = 0;
  if (converged_out) *converged_out = 1;
  if (edges_out) *edges_out = 0;
  if (ncand == 0) return DLP_OK;
  if (!rbeg || !rend || !col || !w || !diag || !Z || !R || !cand) return DLP_ERR_INVALID;
  DLP_CUDA(cudaMemsetAsync(W.mark, 0, sizeof(int32_t) * (size_t)n, s));
  DLP_CUDA(cudaMemsetAsync(W.cnt, 0, sizeof(int32_t) * 4, s));
  DLP_CUDA(cudaMemsetAsync(W.edges, 0, sizeof(unsigned long long), s));
  DLP_CUDA(cudaMemcpyAsync(W.front0, cand, sizeof(int32_t) * (size_t)ncand, cudaMemcpyDeviceToDevice, s));
  DLP_CUDA(cudaMemcpyAsync(W.cnt, &ncand, sizeof(int32_t), cudaMemcpyHostToDevice, s));
  DLP_CUDA(cudaMemcpyAsync(W.eps, eps, sizeof(double) * (size_t)C, cudaMemcpyHostToDevice, s));
  const int grid = sm_count() * 8;
  const int pairs = std::max(1, (check_every > 0 ? check_every : 8) / 2);
  cudaGraphExec_t ex = nullptr;
  if (use_graph) DLP_TRY(push_chunk_graph(q, W, pairs, grid, &ex));
  int rounds = 0;
  int32_t f0 = ncand;
  while (rounds < max_rounds) {
    if (ex) {
      DLP_CUDA(cudaGraphLaunch(ex, s));
      note_launches(4ull * pairs);
    } else {
      for (int i = 0; i < pairs; ++i) {
        DLP_TRY(launch_round(q, W, 0, grid, s));
        DLP_TRY(launch_round(q, W, 1, grid, s));
      }
    }
    rounds += 2 * pairs;
    DLP_CUDA(cudaMemcpyAsync(&f0, W.cnt, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    DLP_CUDA(cudaStreamSynchronize(s));
    if (f0 == 0) break;
  }
  unsigned long long e = 0;
  DLP_CUDA(cudaMemcpyAsync(&e, W.edges, sizeof(e), cudaMemcpyDeviceToHost, s));
  DLP_CUDA(cudaStreamSynchronize(s));
  if (rounds_out) *rounds_out = rounds;
  if (converged_out) *converged_out = f0 == 0 ? 1 : 0;
  if (edges_out) *edges_out = e;
  return DLP_OK;
}

}  // extern "C"
