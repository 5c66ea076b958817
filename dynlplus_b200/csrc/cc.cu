// Connected components (dynlp/cc.py:8-23) as a lock-free union-find: every edge hooks the larger
// of its two roots under the smaller one with atomicCAS, finds use path halving, and a final pass
// compresses every vertex to its root. Because a root is only ever hooked under a smaller id, the
// root of each component is its minimum vertex id, whatever the schedule: the result is the
// reference's canonical labelling before its rank relabel (cc.py:22), bit-exact.
#include <algorithm>

#include "common.cuh"

namespace dlp {

int compact_roots(const int32_t *parent, int32_t n, int32_t *pos, int32_t *count, void *ws, size_t ws_bytes,
                  cudaStream_t s);
int compact_masked_roots(const int32_t *parent, const uint8_t *mask, int32_t n, int32_t *pos, int32_t *count,
                         void *ws, size_t ws_bytes, cudaStream_t s);
int compact_positions(const uint8_t *flag, int32_t n, int32_t *pos, int32_t *count, void *ws, size_t ws_bytes,
                      cudaStream_t s);
size_t compact_ws_bytes(int32_t n);

constexpr int kCcThreads = 256;
constexpr int kMaxSteps = 1 << 26;  // bound on any chase / retry loop (far above any path length)

__global__ void k_cc_init(int32_t *parent, int32_t n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) parent[i] = (int32_t)i;
}

// Root of x with path halving. parent[] only ever decreases, so stale reads are safe.
__device__ __forceinline__ int32_t find_root(volatile int32_t *parent, int32_t x, int32_t *err) {
  int32_t cur = parent[x];
  if (cur == x) return x;
  int32_t prev = x;
  int steps = 0;
  int32_t next;
  while (cur > (next = parent[cur])) {
    parent[prev] = next;
    prev = cur;
    cur = next;
    if (++steps > kMaxSteps) {
      if (err) atomicExch(err, DLP_ERR_DEVICE);
      break;
    }
  }
  return cur;
}

__device__ __forceinline__ void unite(int32_t *parent_, int32_t a, int32_t b, int32_t *err) {
  volatile int32_t *parent = parent_;
  int32_t ra = find_root(parent, a, err), rb = find_root(parent, b, err);
  int steps = 0;
  while (ra != rb) {
    if (ra < rb) {
      const int32_t t = ra;
      ra = rb;
      rb = t;
    }
    // hook ra (larger) under rb (smaller)
    const int32_t ret = atomicCAS(parent_ + ra, ra, rb);
    if (ret == ra) break;
    ra = ret;  // ra was hooked meanwhile: climb from its new parent
    if (++steps > kMaxSteps) {
      if (err) atomicExch(err, DLP_ERR_DEVICE);
      break;
    }
  }
}

__global__ void __launch_bounds__(kCcThreads)
    k_cc_edges(int32_t n, const int32_t *__restrict__ rows, const int32_t *__restrict__ cols, int64_t m,
               int32_t *parent, int32_t *err) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m;
       i += (long long)gridDim.x * blockDim.x) {
    const int32_t a = rows[i], b = cols[i];
    if ((unsigned)a >= (unsigned)n || (unsigned)b >= (unsigned)n) {
      if (err) atomicExch(err, DLP_ERR_DEVICE);
      continue;
    }
    if (a != b) unite(parent, a, b, err);
  }
}

// Graph form, in the sampling-then-skip order of Afforest (Sutton, Ben-Nun, Barak, IPDPS 2018):
//   1. kCcSample rounds: every vertex hooks its k-th live in-mask neighbour, then compress;
//   2. the most frequent root L among a fixed sample of vertices is taken as the big component;
//   3. the rows of every vertex outside L are hooked in full (both directions, so an edge whose
//      other end lies in L is still seen); rows of L are skipped, except for their sink entries
//      until L is joined to the sink.
// Any edge skipped in 3 has both ends in L, so the partition is the full one; and since every hook
// puts a larger root under a smaller one, each root is still its component's minimum vertex id.
constexpr int kCcSample = 2;
constexpr int kCcModeSample = 1024;

template <typename TW>
__device__ __forceinline__ bool live(const TW *w, int j) {
  return !w || cvt<float>(w[j]) != 0.0f;
}

// Sampling round k: every vertex of the mask hooks its k-th live in-mask neighbour (CSR order).
// One neighbour per round with a compression in between keeps every find one or two hops long.
template <typename TW>
__global__ void __launch_bounds__(kCcThreads)
    k_cc_sample(int32_t n, int k, const int32_t *__restrict__ rbeg, const int32_t *__restrict__ rend,
                const int32_t *__restrict__ col, const TW *__restrict__ w, const uint8_t *__restrict__ vmask,
                int32_t *parent, int32_t *err) {
  for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < n;
       u += (long long)gridDim.x * blockDim.x) {
    if (vmask && !vmask[u]) continue;
    const int end = rend[u];
    int seen = 0;
    for (int j = rbeg[u]; j < end; ++j) {
      if (!live(w, j)) continue;
      const int32_t v = col[j];
      if ((unsigned)v >= (unsigned)n) {
        if (err) atomicExch(err, DLP_ERR_DEVICE);
        continue;
      }
      if (vmask && !vmask[v]) continue;
      if (seen++ == k) {
        unite(parent, (int32_t)u, v, err);
        break;
      }
    }
  }
}

// One block: the most frequent root among kCcModeSample in-mask vertices spread over [0, n)
// (ties: the smaller root); -1 when no sampled vertex is in the mask. scratch[1] = 0 (L not yet
// joined to the sink).
__global__ void __launch_bounds__(kCcModeSample) k_cc_big(int32_t n, const uint8_t *__restrict__ vmask,
                                                          const int32_t *__restrict__ parent, int32_t *scratch) {
  __shared__ int32_t root[kCcModeSample];
  __shared__ unsigned long long best;
  const int k = threadIdx.x;
  const int S = n < kCcModeSample ? n : kCcModeSample;
  int32_t r = -1;
  if (k < S) {
    const int32_t i = (int32_t)(((long long)k * n) / S);
    if (!vmask || vmask[i]) r = parent[i];
  }
  root[k] = r;
  if (k == 0) best = 0ull;
  __syncthreads();
  if (r >= 0) {
    unsigned cnt = 0;
    for (int j = 0; j < S; ++j) cnt += root[j] == r;
    // larger count first, then smaller root
    const unsigned long long key = ((unsigned long long)cnt << 32) | (0xffffffffu - (unsigned)r);
    atomicMax(&best, key);
  }
  __syncthreads();
  if (k == 0) {
    scratch[0] = best ? (int32_t)(0xffffffffu - (unsigned)(best & 0xffffffffu)) : -1;
    scratch[1] = 0;
  }
}

// 8 lanes per row; sink vertex id = n. With scratch == NULL every row is hooked in full (entry
// (u, v) once, from the smaller end).
template <typename TW>
__global__ void __launch_bounds__(kCcThreads)
    k_cc_graph(int32_t n, const int32_t *__restrict__ rbeg, const int32_t *__restrict__ rend,
               const int32_t *__restrict__ col, const TW *__restrict__ w, const uint8_t *__restrict__ vmask,
               const uint8_t *__restrict__ sink, int32_t *parent, int32_t *err, int32_t *scratch) {
  const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const int32_t big = scratch ? scratch[0] : -1;
  volatile int32_t *grounded = scratch ? scratch + 1 : nullptr;
  for (long long t = t0; t < (long long)n * 8; t += stride) {
    const int32_t u = (int32_t)(t >> 3);
    const int l = (int)(t & 7);
    if (vmask && !vmask[u]) continue;
    const bool inL = big >= 0 && ((volatile int32_t *)parent)[u] == big;
    if (inL && (!sink || *grounded)) continue;
    const int beg = rbeg[u], end = rend[u];
    for (int j = beg + l; j < end; j += 8) {
      if (!live(w, j)) continue;
      const int32_t v = col[j];
      if ((unsigned)v >= (unsigned)n) {
        if (err) atomicExch(err, DLP_ERR_DEVICE);
        continue;
      }
      if (!vmask || vmask[v]) {
        // skipped rows (L) are covered from the other end; without a sample pass the mirror
        // entry (v, u) covers the pair once
        if (!inL && (scratch || u < v)) unite(parent, u, v, err);
      } else if (sink && sink[v]) {
        unite(parent, u, n, err);
        if (inL) *grounded = 1;
      }
    }
  }
}

__global__ void k_cc_compress(int32_t *parent_, int32_t n, int32_t *err) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  volatile int32_t *parent = parent_;
  int32_t x = parent[i];
  int steps = 0;
  while (true) {
    const int32_t p = parent[x];
    if (p == x) break;
    x = p;
    if (++steps > kMaxSteps) {
      if (err) atomicExch(err, DLP_ERR_DEVICE);
      break;
    }
  }
  parent[i] = x;
}

__global__ void k_cc_gather_rank(const int32_t *__restrict__ parent, int32_t n, int32_t *label) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t p = parent[i];
  if (p != (int32_t)i) label[i] = label[p];
}

// ------------------------------------------------------------------------------------------------
// Grounded set by reachability: the vertices of the mask whose component (live in-mask entries)
// holds an entry to a sink vertex outside the mask -- the set {u : parent[u] == parent[n]} of the
// graph form above, found by bottom-up sweeps instead of a full union-find: an unreached vertex of
// the mask joins as soon as one of its live entries leads to a sink vertex or to a reached vertex.
// Marks are read and written in place, so one sweep carries a mark along many hops; a sweep that
// marks nothing ends it (the reached set is then closed under adjacency, i.e. whole components).
// ------------------------------------------------------------------------------------------------
template <typename TW>
__global__ void __launch_bounds__(kCcThreads)
    k_reach_sweep(int32_t n, const int32_t *__restrict__ rbeg, const int32_t *__restrict__ rend,
                  const int32_t *__restrict__ col, const TW *__restrict__ w, const uint8_t *__restrict__ vmask,
                  const uint8_t *__restrict__ sink, uint8_t *reached_, int32_t *flag, int32_t *err) {
  volatile uint8_t *reached = reached_;
  bool any = false;
  for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < n;
       u += (long long)gridDim.x * blockDim.x) {
    if ((vmask && !vmask[u]) || reached[u]) continue;
    const int end = rend[u];
    for (int j = rbeg[u]; j < end; ++j) {
      if (!live(w, j)) continue;
      const int32_t v = col[j];
      if ((unsigned)v >= (unsigned)n) {
        if (err) atomicExch(err, DLP_ERR_DEVICE);
        continue;
      }
      const bool inm = !vmask || vmask[v];
      if (inm ? reached[v] != 0 : (sink && sink[v])) {
        reached[u] = 1;
        any = true;
        break;
      }
    }
  }
  if (__any_sync(0xffffffffu, any) && lane_id() == 0) atomicAdd(flag, 1);
}

// umask[v] = reached[v] (or root(v) == root(sink) when parent is given); in_t[v] = membership
// changed; *count += |changed|
__global__ void k_ground_apply(int32_t n, const uint8_t *__restrict__ reached, const int32_t *__restrict__ parent,
                               const uint8_t *__restrict__ vmask, uint8_t *umask, uint8_t *in_t, int32_t *count) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  bool ch = false;
  if (v < n) {
    const bool nu = parent ? ((!vmask || vmask[v]) && parent[v] == parent[n]) : reached[v] != 0;
    const bool ou = umask[v] != 0;
    ch = nu != ou;
    umask[v] = nu ? 1 : 0;
    in_t[v] = ch ? 1 : 0;
  }
  const unsigned b = __ballot_sync(0xffffffffu, ch);
  if ((threadIdx.x & 31) == 0 && b) atomicAdd(count, __popc(b));
}

// label[lpos[v]] = rank[parent[v]] for every masked v: the rank of its component's minimum id,
// written at the vertex's place among the masked vertices.
__global__ void k_cc_mask_gather(int32_t n, const int32_t *__restrict__ parent, const uint8_t *__restrict__ vmask,
                                 const int32_t *__restrict__ rank, const int32_t *__restrict__ lpos, int32_t *label) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n && vmask[v]) label[lpos[v]] = rank[parent[v]];
}

// ------------------------------------------------------------------------------------------------
// Components of a graph that changes by small batches between calls (warm start). The masked
// subgraph of the workloads is one giant component plus a few tiny ones, so instead of Afforest's
// sampling rounds the giant component is found by a breadth-first search from the root the previous
// call found for its most frequent component: top-down levels (8 lanes per frontier vertex,
// first-touch bits, warp-aggregated appends) while the frontier is small, then bottom-up sweeps over
// the bitmap. Every reached vertex is connected to the seed, so the reached set R is one connected
// set whatever the seed; its vertices start under R's minimum id, and the union-find then hooks the
// rows outside R in full (k_cc_graph with R as the skipped component). The result is the exact
// minimum-id labelling of dlp_cc_graph; a poor seed (a vertex cut off by the batch) only leaves more
// rows to the union-find. No host read: the schedule of levels is fixed and levels past the end of
// the search return at once.
// ------------------------------------------------------------------------------------------------
constexpr int kWarmDown = 7;  // top-down levels at most
constexpr int kWarmUp = 4;    // bottom-up sweeps at most
// control words: [0] seed, then R's root (k_cc_graph's skipped root), [1] sink flag of k_cc_graph
// (unused: no sink), [2] bottom-up switch, [3] minimum reached id, [4 + l] frontier size of level l
enum { kWSeed = 0, kWUp = 2, kWMin = 3, kWCnt = 4 };

__global__ void k_warm_seed(int32_t n, const uint8_t *__restrict__ vmask, uint32_t *bits, int32_t *front0,
                            int32_t *ctl) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int32_t sd = ctl[kWSeed];
  ctl[1] = 0;
  ctl[kWUp] = 0;
  ctl[kWMin] = 0x7fffffff;
  for (int l = 0; l <= kWarmDown; ++l) ctl[kWCnt + l] = 0;
  if (sd >= 0 && sd < n && (!vmask || vmask[sd])) {
    bits[sd >> 5] |= 1u << (sd & 31);
    front0[0] = sd;
    ctl[kWCnt] = 1;
  }
}

template <typename TW>
__global__ void __launch_bounds__(kCcThreads)
    k_bfs_down(int32_t n, const int32_t *__restrict__ rbeg, const int32_t *__restrict__ rend,
               const int32_t *__restrict__ col, const TW *__restrict__ w, const uint8_t *__restrict__ vmask,
               uint32_t *bits, const int32_t *__restrict__ front_in, int32_t *front_out, int32_t *ctl, int level,
               int cap) {
  constexpr int G = 8, kGroups = 32 / G;
  const int nf = ctl[kWCnt + level];
  if (nf == 0) return;
  if (nf > cap) {  // a large frontier: the bottom-up sweeps take over from the bitmap
    if (blockIdx.x == 0 && threadIdx.x == 0) ctl[kWUp] = 1;
    return;
  }
  const int lane = lane_id(), gl = lane % G;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long stride = (((long long)gridDim.x * blockDim.x) >> 5) * kGroups;
  for (long long base = warp * kGroups; base < nf; base += stride) {  // warp-uniform bounds
    const long long g = base + lane / G;
    int beg = 0, end = 0;
    if (g < nf) {
      const int32_t u = front_in[g];
      beg = rbeg[u];
      end = rend[u];
    }
    const int trips = __reduce_max_sync(0xffffffffu, (end - beg + G - 1) / G);
    for (int t = 0; t < trips; ++t) {
      const int j = beg + gl + t * G;
      bool fresh = false;
      int32_t v = 0;
      if (j < end && live(w, j)) {
        v = col[j];
        if ((unsigned)v < (unsigned)n && (!vmask || vmask[v])) {
          const uint32_t bit = 1u << (v & 31);
          fresh = (atomicOr(bits + (v >> 5), bit) & bit) == 0u;
        }
      }
      warp_append(fresh, v, front_out, ctl + kWCnt + level + 1);
    }
  }
}

// Bottom-up sweep: an unreached vertex of the mask joins when one of its live in-mask entries
// leads to a reached vertex (bits read and written in place, so a sweep carries marks many hops).
template <typename TW>
__global__ void __launch_bounds__(kCcThreads)
    k_bfs_up(int32_t n, const int32_t *__restrict__ rbeg, const int32_t *__restrict__ rend,
             const int32_t *__restrict__ col, const TW *__restrict__ w, const uint8_t *__restrict__ vmask,
             uint32_t *bits_, const int32_t *ctl) {
  if (!ctl[kWUp] && !ctl[kWCnt + kWarmDown]) return;  // the top-down levels finished the search
  volatile uint32_t *bits = bits_;
  for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < n;
       u += (long long)gridDim.x * blockDim.x) {
    if (vmask && !vmask[u]) continue;
    const uint32_t ub = 1u << (u & 31);
    if (bits[u >> 5] & ub) continue;
    const int end = rend[u];
    for (int j = rbeg[u]; j < end; ++j) {
      if (!live(w, j)) continue;
      const int32_t v = col[j];
      if ((unsigned)v >= (unsigned)n || (vmask && !vmask[v])) continue;
      if (bits[v >> 5] & (1u << (v & 31))) {
        atomicOr(bits_ + (u >> 5), ub);
        break;
      }
    }
  }
}

// Smallest reached id: the first set bit of each word, then a minimum.
__global__ void k_warm_min(int32_t n, const uint32_t *__restrict__ bits, int32_t *ctl) {
  const long long wd = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int32_t m = 0x7fffffff;
  if (wd < ((long long)n + 31) / 32 && bits[wd]) m = (int32_t)(wd * 32 + __ffs(bits[wd]) - 1);
  m = __reduce_min_sync(0xffffffffu, m);
  if (lane_id() == 0 && m != 0x7fffffff) atomicMin(ctl + kWMin, m);
}

// parent[v] = R's minimum id for the reached vertices, v otherwise (parent[n] = n, the unused sink);
// control word 0 becomes R's root for k_cc_graph (-1 when nothing was reached).
__global__ void k_warm_parent(int32_t n, const uint32_t *__restrict__ bits, int32_t *parent, int32_t *ctl) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int32_t m = ctl[kWMin];
  if (v < n) parent[v] = (bits[v >> 5] >> (v & 31)) & 1u ? m : (int32_t)v;
  else if (v == n) parent[v] = (int32_t)n;
  if (v == 0) ctl[kWSeed] = m == 0x7fffffff ? -1 : m;
}

static int grid_persist(long long work) {
  long long blocks = (work + kCcThreads - 1) / kCcThreads;
  const long long cap = (long long)sm_count() * 8;
  if (blocks > cap) blocks = cap;
  return (int)(blocks < 1 ? 1 : blocks);
}

}  // namespace dlp

using namespace dlp;

extern "C" {

int dlp_cc_edges(int32_t n, const int32_t *rows, const int32_t *cols, int64_t m, int32_t *parent, int32_t *err,
                 dlp_stream_t stream) {
  if (n < 0 || m < 0 || (n > 0 && !parent) || (m > 0 && (!rows || !cols))) return DLP_ERR_INVALID;
  if (n == 0) return DLP_OK;
  cudaStream_t s = (cudaStream_t)stream;
  k_cc_init<<<ceil_div_i(n, kCcThreads), kCcThreads, 0, s>>>(parent, n);
  if (m > 0) k_cc_edges<<<grid_persist(m), kCcThreads, 0, s>>>(n, rows, cols, m, parent, err);
  k_cc_compress<<<ceil_div_i(n, kCcThreads), kCcThreads, 0, s>>>(parent, n, err);
  return check_launch(m > 0 ? 3 : 2);
}

size_t dlp_cc_graph_workspace_bytes(void) { return 256; }

int dlp_cc_graph(int32_t n, const int32_t *rbeg, const int32_t *rend, const int32_t *col, const void *w,
                 int w_dtype, const uint8_t *vmask, const uint8_t *sink, int32_t *parent, int32_t *err, void *ws,
                 size_t ws_bytes, dlp_stream_t stream) {
  if (n < 0 || !parent) return DLP_ERR_INVALID;
  if (ws && ws_bytes < dlp_cc_graph_workspace_bytes()) return DLP_ERR_WORKSPACE;
  if (n > 0 && (!rbeg || !rend || !col)) return DLP_ERR_INVALID;
  if (w && w_dtype != DLP_F32 && w_dtype != DLP_F64 && w_dtype != DLP_BF16) return DLP_ERR_DTYPE;
  cudaStream_t s = (cudaStream_t)stream;
  int32_t *scratch = (int32_t *)ws;
  int launches = 2;
  k_cc_init<<<ceil_div_i((long long)n + 1, kCcThreads), kCcThreads, 0, s>>>(parent, n + 1);
  if (n > 0) {
    const int grid = grid_persist((long long)n * 8);
    const int grid1 = grid_persist(n);
#define DLP_CC_PASSES(TW)                                                                                      \
  if (scratch) {                                                                                               \
    for (int k = 0; k < kCcSample; ++k) {                                                                     \
      k_cc_sample<TW><<<grid1, kCcThreads, 0, s>>>(n, k, rbeg, rend, col, (const TW *)w, vmask, parent, err);   \
      k_cc_compress<<<ceil_div_i(n, kCcThreads), kCcThreads, 0, s>>>(parent, n, err);                         \
    }                                                                                                          \
    k_cc_big<<<1, kCcModeSample, 0, s>>>(n, vmask, parent, scratch);                                           \
    launches += 2 * kCcSample + 1;                                                                             \
  }                                                                                                            \
  k_cc_graph<TW><<<grid, kCcThreads, 0, s>>>(n, rbeg, rend, col, (const TW *)w, vmask, sink, parent, err, scratch); \
  launches += 1;
    if (!w || w_dtype == DLP_F32) {
      DLP_CC_PASSES(float)
    } else if (w_dtype == DLP_F64) {
      DLP_CC_PASSES(double)
    } else {
      DLP_CC_PASSES(bf16)
    }
#undef DLP_CC_PASSES
  }
  k_cc_compress<<<ceil_div_i((long long)n + 1, kCcThreads), kCcThreads, 0, s>>>(parent, n + 1, err);
  return check_launch(launches);
}

static size_t warm_ws_layout(int32_t n, size_t *off_bits, size_t *off_f0, size_t *off_f1) {
  const size_t nn = (size_t)(n > 0 ? n : 1);
  size_t b = 256;  // control words
  *off_bits = b;
  b += ((nn + 31) / 32 * 4 + 255) / 256 * 256;
  *off_f0 = b;
  b += (nn * 4 + 255) / 256 * 256;
  *off_f1 = b;
  return b + (nn * 4 + 255) / 256 * 256;
}

constexpr int kReachBatch = 4;      // sweeps between host checks
constexpr int kReachMaxSweeps = 32; // then the union-find finishes the job

static size_t reach_ws_layout(int32_t n, size_t *off_flags, size_t *off_parent, size_t *off_cc) {
  size_t b = ((size_t)n + 255) / 256 * 256;  // reached
  *off_flags = b;
  b += 256;                                  // one flag per sweep (kReachMaxSweeps ints)
  *off_parent = b;
  b += ((size_t)n + 1 + 63) / 64 * 256;      // parent of the fallback (n + 1 ints)
  *off_cc = b;
  return b + 256;                            // dlp_cc_graph workspace
}

size_t dlp_cc_graph_warm_workspace_bytes(int32_t n) {
  size_t a, b, c;
  return warm_ws_layout(n, &a, &b, &c);
}

int dlp_cc_graph_warm(int32_t n, const int32_t *rbeg, const int32_t *rend, const int32_t *col, const void *w,
                      int w_dtype, const uint8_t *vmask, int32_t *parent, int32_t *err, void *ws, size_t ws_bytes,
                      dlp_stream_t stream) {
  if (n < 0 || !parent) return DLP_ERR_INVALID;
  if (n > 0 && (!rbeg || !rend || !col)) return DLP_ERR_INVALID;
  if (w && w_dtype != DLP_F32 && w_dtype != DLP_F64 && w_dtype != DLP_BF16) return DLP_ERR_DTYPE;
  size_t off_bits, off_f0, off_f1;
  if (!ws || ws_bytes < warm_ws_layout(n, &off_bits, &off_f0, &off_f1)) return DLP_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 0) {
    k_cc_init<<<1, kCcThreads, 0, s>>>(parent, 1);
    return check_launch();
  }
  char *base = (char *)ws;
  int32_t *ctl = (int32_t *)base;
  uint32_t *bits = (uint32_t *)(base + off_bits);
  int32_t *front[2] = {(int32_t *)(base + off_f0), (int32_t *)(base + off_f1)};
  DLP_CUDA(cudaMemsetAsync(bits, 0, ((size_t)n + 31) / 32 * 4, s));
  k_warm_seed<<<1, 32, 0, s>>>(n, vmask, bits, front[0], ctl);
  const int cap = std::max(n / 16, 1024);
  const int grid = grid_persist((long long)n * 8);
  const int grid1 = grid_persist(n);
#define DLP_WARM_PASSES(TW)                                                                                       \
  for (int l = 0; l < kWarmDown; ++l)                                                                            \
    k_bfs_down<TW><<<grid, kCcThreads, 0, s>>>(n, rbeg, rend, col, (const TW *)w, vmask, bits, front[l & 1],      \
                                               front[(l + 1) & 1], ctl, l, cap);                                  \
  for (int u = 0; u < kWarmUp; ++u)                                                                              \
    k_bfs_up<TW><<<grid1, kCcThreads, 0, s>>>(n, rbeg, rend, col, (const TW *)w, vmask, bits, ctl);               \
  k_warm_min<<<ceil_div_i(((long long)n + 31) / 32, kCcThreads), kCcThreads, 0, s>>>(n, bits, ctl);              \
  k_warm_parent<<<ceil_div_i((long long)n + 1, kCcThreads), kCcThreads, 0, s>>>(n, bits, parent, ctl);           \
  k_cc_graph<TW><<<grid, kCcThreads, 0, s>>>(n, rbeg, rend, col, (const TW *)w, vmask, nullptr, parent, err, ctl);
  if (!w || w_dtype == DLP_F32) {
    DLP_WARM_PASSES(float)
  } else if (w_dtype == DLP_F64) {
    DLP_WARM_PASSES(double)
  } else {
    DLP_WARM_PASSES(bf16)
  }
#undef DLP_WARM_PASSES
  k_cc_compress<<<ceil_div_i((long long)n + 1, kCcThreads), kCcThreads, 0, s>>>(parent, n + 1, err);
  k_cc_big<<<1, kCcModeSample, 0, s>>>(n, vmask, parent, ctl);  // the next call's seed
  return check_launch(kWarmDown + kWarmUp + 6);
}

size_t dlp_ground_reach_workspace_bytes(int32_t n) {
  size_t a, b, c;
  return reach_ws_layout(n < 0 ? 0 : n, &a, &b, &c);
}

int dlp_ground_reach(int32_t n, const int32_t *rbeg, const int32_t *rend, const int32_t *col, const void *w,
                     int w_dtype, const uint8_t *vmask, const uint8_t *sink, uint8_t *umask, uint8_t *in_t,
                     int32_t *count, int32_t *err, int32_t *sweeps_out, void *ws, size_t ws_bytes,
                     dlp_stream_t stream) {
  if (n < 0 || (n > 0 && (!rbeg || !rend || !col || !umask || !in_t || !count))) return DLP_ERR_INVALID;
  if (w && w_dtype != DLP_F32 && w_dtype != DLP_F64 && w_dtype != DLP_BF16) return DLP_ERR_DTYPE;
  size_t off_flags, off_parent, off_cc;
  if (!ws || ws_bytes < reach_ws_layout(n, &off_flags, &off_parent, &off_cc)) return DLP_ERR_WORKSPACE;
  if (sweeps_out) *sweeps_out = 0;
  if (n == 0) return DLP_OK;
  cudaStream_t s = (cudaStream_t)stream;
  char *base = (char *)ws;
  uint8_t *reached = (uint8_t *)base;
  int32_t *flags = (int32_t *)(base + off_flags);
  DLP_CUDA(cudaMemsetAsync(reached, 0, (size_t)n, s));
  DLP_CUDA(cudaMemsetAsync(flags, 0, sizeof(int32_t) * kReachMaxSweeps, s));
  const int grid = grid_persist(n);
  int done = 0;
  bool converged = false;
  while (!converged && done < kReachMaxSweeps) {
    for (int k = 0; k < kReachBatch; ++k, ++done) {
      if (!w || w_dtype == DLP_F32)
        k_reach_sweep<float><<<grid, kCcThreads, 0, s>>>(n, rbeg, rend, col, (const float *)w, vmask, sink, reached,
                                                          flags + done, err);
      else if (w_dtype == DLP_F64)
        k_reach_sweep<double><<<grid, kCcThreads, 0, s>>>(n, rbeg, rend, col, (const double *)w, vmask, sink,
                                                           reached, flags + done, err);
      else
        k_reach_sweep<bf16><<<grid, kCcThreads, 0, s>>>(n, rbeg, rend, col, (const bf16 *)w, vmask, sink, reached,
                                                         flags + done, err);
    }
    DLP_TRY(check_launch(kReachBatch));
    int32_t h[kReachBatch];
    DLP_CUDA(cudaMemcpyAsync(h, flags + done - kReachBatch, sizeof(h), cudaMemcpyDeviceToHost, s));
    DLP_CUDA(cudaStreamSynchronize(s));
    for (int k = 0; k < kReachBatch; ++k) {
      if (h[k] == 0) {
        converged = true;
        if (sweeps_out) *sweeps_out = done - kReachBatch + k + 1;
        break;
      }
    }
  }
  const int32_t *parent = nullptr;
  if (!converged) {  // long chains: the union-find settles the rest exactly
    int32_t *par = (int32_t *)(base + off_parent);
    DLP_TRY(dlp_cc_graph(n, rbeg, rend, col, w, w_dtype, vmask, sink, par, err, base + off_cc, 256, stream));
    parent = par;
    if (sweeps_out) *sweeps_out = -done;
  }
  k_ground_apply<<<ceil_div_i(n, 256), 256, 0, s>>>(n, reached, parent, vmask, umask, in_t, count);
  return check_launch();
}

size_t dlp_cc_mask_labels_workspace_bytes(int32_t n) {
  const size_t v = ((size_t)(n > 0 ? n : 1) * sizeof(int32_t) + 255) / 256 * 256;
  return 2 * v + compact_ws_bytes(n);
}

int dlp_cc_mask_labels(int32_t n, const int32_t *parent, const uint8_t *vmask, int32_t *label, int32_t *n_comp,
                       int32_t *n_masked, void *ws, size_t ws_bytes, dlp_stream_t stream) {
  if (n < 0 || !n_comp || !n_masked || (n > 0 && (!parent || !vmask || !label))) return DLP_ERR_INVALID;
  if (!ws || ws_bytes < dlp_cc_mask_labels_workspace_bytes(n)) return DLP_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t v = ((size_t)(n > 0 ? n : 1) * sizeof(int32_t) + 255) / 256 * 256;
  int32_t *rank = (int32_t *)ws;
  int32_t *lpos = (int32_t *)((char *)ws + v);
  void *cws = (char *)ws + 2 * v;
  const size_t cbytes = ws_bytes - 2 * v;
  DLP_TRY(compact_masked_roots(parent, vmask, n, rank, n_comp, cws, cbytes, s));
  DLP_TRY(compact_positions(vmask, n, lpos, n_masked, cws, cbytes, s));
  if (n > 0) k_cc_mask_gather<<<ceil_div_i(n, kCcThreads), kCcThreads, 0, s>>>(n, parent, vmask, rank, lpos, label);
  return check_launch(n > 0 ? 1 : 0);
}

int dlp_cc_relabel(int32_t n, const int32_t *parent, int32_t *label, int32_t *n_comp, void *ws, size_t ws_bytes,
                   dlp_stream_t stream) {
  if (n < 0 || (n > 0 && (!parent || !label)) || !n_comp) return DLP_ERR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  // label[root] = rank of the root among roots; then every vertex copies its root's rank.
  DLP_TRY(compact_roots(parent, n, label, n_comp, ws, ws_bytes, s));
  if (n > 0) k_cc_gather_rank<<<ceil_div_i(n, kCcThreads), kCcThreads, 0, s>>>(parent, n, label);
  return check_launch(n > 0 ? 1 : 0);
}

}  // extern "C"
