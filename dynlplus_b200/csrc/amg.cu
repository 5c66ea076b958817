// Aggregation AMG for grounded graph Laplacians (dynlp/amg.py), setup and V-cycle, on the device.
//
// Setup (per level): heavy-edge handshake matching (amg.py:32-64) with one thread per vertex
// scanning its row (max weight among admissible neighbours, smallest id among ties: the
// reference's scatter_max / scatter_min pair), mutual choices pair up, unmatched vertices join
// their heaviest matched neighbour, the rest stay single; aggregates are numbered by the rank of
// their representative (numpy.unique's inverse). The Galerkin coarse operator of the piecewise-
// constant prolongation, W_c = sum of inter-aggregate weights, s_c = sum of grounding
// (amg.py:67-74), is built per coarse row by one thread accumulating its members' rows in a
// private open-addressing table, in a fixed member order with fp64 sums: deterministic.
// Cycle (amg.py:119-134): damped Jacobi sweeps, restriction as ordered segment sums over the
// aggregates, prolongation by gather, and the dense fp64 inverse at the coarsest level.
#include <algorithm>
#include <climits>

#include "common.cuh"

namespace dlp {

int exclusive_scan_i32(const int32_t *in, int32_t n, int32_t *out, void *ws, size_t ws_bytes, cudaStream_t s);
size_t compact_ws_bytes(int32_t n);

constexpr int kAT = 256;
static int g1(long long w) { return ceil_div_i(w > 0 ? w : 1, kAT); }

// mode 0: u unmatched, neighbours unmatched; mode 1: u unmatched, neighbours matched.
__global__ void k_best_choice(int32_t n, const int32_t *__restrict__ indptr, const int32_t *__restrict__ col,
                              const float *__restrict__ w, const uint8_t *__restrict__ matched, int mode,
                              int32_t *choice) {
  const long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) return;
  int32_t pick = n;
  if (!matched[u]) {
    float best = -INFINITY;
    for (int j = indptr[u]; j < indptr[u + 1]; ++j) {
      const int32_t v = col[j];
      const bool ok = mode == 0 ? !matched[v] : matched[v];
      if (!ok) continue;
      const float x = w[j];
      if (x > best || (x == best && v < pick)) {
        best = x;
        pick = v;
      }
    }
  }
  choice[u] = pick;
}

__global__ void k_mutual(int32_t n, const int32_t *__restrict__ choice, uint8_t *matched, int32_t *agg) {
  const long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) return;
  const int32_t c = choice[u];
  if (c < n && choice[c] == (int32_t)u) {
    matched[u] = 1;
    agg[u] = c < u ? c : (int32_t)u;
  }
}

__global__ void k_join(int32_t n, const int32_t *__restrict__ choice, int32_t *agg) {
  const long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) return;
  const int32_t c = choice[u];
  if (c < n) agg[u] = agg[c];  // c is matched: its agg was final before this kernel
}

__global__ void k_self_and_flag(int32_t n, int32_t *agg, int32_t *flag) {
  const long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) return;
  if (agg[u] < 0) agg[u] = (int32_t)u;
  flag[agg[u]] = 1;  // benign race: all writers store 1
}

__global__ void k_rank_gather(int32_t n, const int32_t *__restrict__ rank, int32_t *agg) {
  const long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) return;
  agg[u] = rank[agg[u]];
}

// members of each aggregate, ascending fine ids: count, scan, fill (positions by atomics), sort.
__global__ void k_count_members(int32_t n, const int32_t *__restrict__ agg, int32_t *cnt) {
  const long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (u < n) atomicAdd(cnt + agg[u], 1);
}

__global__ void k_fill_members(int32_t n, const int32_t *__restrict__ agg, const int32_t *__restrict__ off,
                               int32_t *cursor, int32_t *members) {
  const long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (u < n) {
    const int32_t a = agg[u];
    members[off[a] + atomicAdd(cursor + a, 1)] = (int32_t)u;
  }
}

__global__ void k_sort_members(int32_t nc, const int32_t *__restrict__ off, int32_t *members) {
  const long long a = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= nc) return;
  const int b = off[a], e = off[a + 1];
  for (int i = b + 1; i < e; ++i) {  // aggregates are small: insertion sort
    const int32_t x = members[i];
    int j = i - 1;
    while (j >= b && members[j] > x) {
      members[j + 1] = members[j];
      --j;
    }
    members[j + 1] = x;
  }
}

// upper bound of coarse row lengths (sum of member degrees) and the table capacity per row
__global__ void k_coarse_bound(int32_t nc, const int32_t *__restrict__ off, const int32_t *__restrict__ members,
                               const int32_t *__restrict__ indptr, int32_t *cap) {
  const long long a = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= nc) return;
  int ub = 0;
  for (int i = off[a]; i < off[a + 1]; ++i) {
    const int32_t u = members[i];
    ub += indptr[u + 1] - indptr[u];
  }
  int c = 4;
  while (c < 2 * ub) c <<= 1;
  cap[a] = ub ? c : 0;
}

__global__ void k_coarse_accumulate(int32_t nc, const int32_t *__restrict__ off, const int32_t *__restrict__ members,
                                    const int32_t *__restrict__ indptr, const int32_t *__restrict__ col,
                                    const float *__restrict__ w, const int32_t *__restrict__ agg,
                                    const int32_t *__restrict__ toff, int32_t *tkey, double *tval,
                                    const double *__restrict__ s, double *sc, int32_t *rowcnt) {
  const long long a = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= nc) return;
  const int t0 = toff[a], cap = toff[a + 1] - toff[a];
  double sa = 0.0;
  int cnt = 0;
  for (int i = off[a]; i < off[a + 1]; ++i) {
    const int32_t u = members[i];
    if (s) sa += s[u];
    for (int j = indptr[u]; j < indptr[u + 1]; ++j) {
      const int32_t b = agg[col[j]];
      if (b == (int32_t)a) continue;
      unsigned h = ((unsigned)b * 2654435761u) & (unsigned)(cap - 1);
      while (true) {
        const int32_t k = tkey[t0 + h];
        if (k == b) {
          tval[t0 + h] += (double)w[j];
          break;
        }
        if (k < 0) {
          tkey[t0 + h] = b;
          tval[t0 + h] = (double)w[j];
          ++cnt;
          break;
        }
        h = (h + 1) & (unsigned)(cap - 1);  // cap >= 2 * entries: terminates
      }
    }
  }
  if (sc) sc[a] = sa;
  rowcnt[a] = cnt;
}

__global__ void k_coarse_emit(int32_t nc, const int32_t *__restrict__ toff, const int32_t *__restrict__ tkey,
                              const double *__restrict__ tval, const int32_t *__restrict__ indptr_c, int32_t *col_c,
                              float *w_c) {
  const long long a = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= nc) return;
  const int b = indptr_c[a];
  int o = b;
  for (int h = toff[a]; h < toff[a + 1]; ++h) {
    const int32_t k = tkey[h];
    if (k < 0) continue;
    // insertion into the row's sorted position (rows are short)
    const float x = (float)tval[h];
    int j = o - 1;
    while (j >= b && col_c[j] > k) {
      col_c[j + 1] = col_c[j];
      w_c[j + 1] = w_c[j];
      --j;
    }
    col_c[j + 1] = k;
    w_c[j + 1] = x;
    ++o;
  }
}

// ---- sort-based Galerkin coarsening ------------------------------------------------------------
// keys: entry j of row u -> agg[u] * nc + agg[col[j]] (a sentinel when both ends share an aggregate);
// after a stable sort by key, each key's entries sit together in their CSR order, so summing a run
// front to back reproduces the per-row accumulation order of the reference's coalesce.
constexpr long long kNoKey = 0x7fffffffffffffffll;

__global__ void k_coarse_keys(int32_t n, const int32_t *__restrict__ indptr, const int32_t *__restrict__ col,
                              const float *__restrict__ w, const int32_t *__restrict__ agg, int32_t nc, long long *key,
                              double *val) {
  // 8 lanes per row
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long u = t >> 3;
  if (u >= n) return;
  const long long a = agg[u];
  for (int j = indptr[u] + (int)(t & 7); j < indptr[u + 1]; j += 8) {
    const long long b = agg[col[j]];
    key[j] = a == b ? kNoKey : a * nc + b;
    val[j] = (double)w[j];
  }
}

// flag[i] = 1 where a run of equal (kept) keys starts
__global__ void k_run_starts(long long m, const long long *__restrict__ key, int32_t *flag) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const long long k = key[i];
  flag[i] = (k != kNoKey && (i == 0 || key[i - 1] != k)) ? 1 : 0;
}

// one thread per run: the run's sum (front to back) becomes coarse entry pos[i]; rows counted
__global__ void k_run_emit(long long m, const long long *__restrict__ key, const double *__restrict__ val,
                           const int32_t *__restrict__ flag, const int32_t *__restrict__ pos, int32_t nc,
                           int32_t *col_c, float *w_c, int32_t *rowcnt) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m || !flag[i]) return;
  const long long k = key[i];
  double acc = val[i];
  for (long long j = i + 1; j < m && key[j] == k; ++j) acc += val[j];
  const int32_t a = (int32_t)(k / nc);
  col_c[pos[i]] = (int32_t)(k - (long long)a * nc);
  w_c[pos[i]] = (float)acc;
  atomicAdd(rowcnt + a, 1);
}

// s_c[a] = sum of s over the members of aggregate a, in member order
__global__ void k_member_sum(int32_t nc, const int32_t *__restrict__ off, const int32_t *__restrict__ members,
                             const double *__restrict__ s, double *sc) {
  const long long a = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= nc) return;
  double acc = 0.0;
  for (int i = off[a]; i < off[a + 1]; ++i) acc += s[members[i]];
  sc[a] = acc;
}

// ---- cycle kernels ------------------------------------------------------------------------------
template <typename T>
__global__ void k_restrict(int32_t nc, int32_t C, const int32_t *__restrict__ off, const int32_t *__restrict__ members,
                           const T *__restrict__ R, int64_t ldr, T *Rc, int64_t ldc) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nc * C) return;
  const long long a = t / C;
  const int c = (int)(t % C);
  T s = T(0);
  for (int i = off[a]; i < off[a + 1]; ++i) s += R[(long long)members[i] * ldr + c];
  Rc[a * ldc + c] = s;
}

template <typename T>
__global__ void k_prolong_add(int32_t n, int32_t C, const int32_t *__restrict__ agg, const T *__restrict__ Xc,
                              int64_t ldc, T *X, int64_t ldx) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * C) return;
  const long long u = t / C;
  const int c = (int)(t % C);
  X[u * ldx + c] += Xc[(long long)agg[u] * ldc + c];
}

// X = omega * R / diag (the first smoothing sweep from X = 0)
template <typename T>
__global__ void k_scale_rows(int32_t n, int32_t C, double omega, const T *__restrict__ R, int64_t ldr,
                             const T *__restrict__ diag, T *X, int64_t ldx) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * C) return;
  const long long u = t / C;
  const int c = (int)(t % C);
  X[u * ldx + c] = (T)omega * R[u * ldr + c] / diag[u];
}

// Y[i, c] = sum_j M[i, j] * X[j, c] for a dense row-major fp64 M (nc x nc); X, Y in T.
template <typename T>
__global__ void k_dense_apply(int32_t nc, int32_t C, const double *__restrict__ M, const T *__restrict__ X, int64_t ldx,
                              T *Y, int64_t ldy) {
  // one warp per output row: lanes stride over j, shuffle-reduce per column (C <= 64)
  const long long row = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= nc) return;
  for (int c0 = 0; c0 < C; c0 += 8) {
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int j = lane; j < nc; j += 32) {
      const double m = M[row * nc + j];
#pragma unroll
      for (int k = 0; k < 8; ++k)
        if (c0 + k < C) acc[k] = fma(m, (double)X[(long long)j * ldx + c0 + k], acc[k]);
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
      if (lane == 0 && c0 + k < C) Y[row * ldy + c0 + k] = (T)acc[k];
    }
  }
}

// damped Jacobi sweep over all rows: Y = X + omega * ((RHS + W X) / diag - X)
template <typename T>
__global__ void k_jacobi_sweep(int32_t n, int32_t C, const int32_t *__restrict__ indptr, const int32_t *__restrict__ col,
                               const float *__restrict__ w, const T *__restrict__ X, int64_t ldx,
                               const T *__restrict__ RHS, int64_t ldr, const T *__restrict__ diag, double omega, T *Y,
                               int64_t ldy) {
  // 4 lanes per row, columns looped (coarse levels are narrow in rows, not in columns)
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long r = t >> 2;
  const int l = (int)(t & 3);
  const bool valid = r < n;
  const int beg = valid ? indptr[r] : 0, end = valid ? indptr[r + 1] : 0;
  for (int c0 = 0; c0 < C; c0 += 8) {
    T acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int j = beg + l; j < end; j += 4) {
      const long long v = col[j];
      const T x = (T)w[j];
#pragma unroll
      for (int k = 0; k < 8; ++k)
        if (c0 + k < C) acc[k] += x * X[v * ldx + c0 + k];
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], 1);
      acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], 2);
    }
    if (valid && l == 0) {
      const T d = diag[r];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int c = c0 + k;
        if (c < C) {
          const T xo = X[r * ldx + c];
          Y[r * ldy + c] = xo + (T)omega * ((RHS[r * ldr + c] + acc[k]) / d - xo);
        }
      }
    }
  }
}

}  // namespace dlp

using namespace dlp;

extern "C" {

size_t dlp_amg_match_workspace_bytes(int32_t n) { return 3 * (((size_t)(n > 0 ? n : 1) * 4 + 4 + 255) / 256 * 256) + compact_ws_bytes(n); }

int dlp_amg_match(int32_t n, const int32_t *indptr, const int32_t *col, const float *w, int32_t rounds, int32_t *agg,
                  int32_t *n_agg, void *ws, size_t ws_bytes, dlp_stream_t stream) {
  if (n < 0 || rounds < 0 || !agg || !n_agg) return DLP_ERR_INVALID;
  if (!ws || ws_bytes < dlp_amg_match_workspace_bytes(n)) return DLP_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 0) {
    DLP_CUDA(cudaMemsetAsync(n_agg, 0, sizeof(int32_t), s));
    return DLP_OK;
  }
  if (!indptr || !col || !w) return DLP_ERR_INVALID;
  const size_t vb = ((size_t)n * 4 + 4 + 255) / 256 * 256;  // n + 1 ints: the scan writes its total
  char *p = (char *)ws;
  int32_t *choice = (int32_t *)p;
  uint8_t *matched = (uint8_t *)(p + vb);
  int32_t *flag = (int32_t *)(p + 2 * vb);
  void *cws = p + 3 * vb;
  const size_t cbytes = ws_bytes - 3 * vb;
  DLP_CUDA(cudaMemsetAsync(matched, 0, (size_t)n, s));
  DLP_CUDA(cudaMemsetAsync(agg, 0xff, sizeof(int32_t) * (size_t)n, s));
  int launches = 0;
  for (int r = 0; r < rounds; ++r) {
    k_best_choice<<<g1(n), kAT, 0, s>>>(n, indptr, col, w, matched, 0, choice);
    k_mutual<<<g1(n), kAT, 0, s>>>(n, choice, matched, agg);
    launches += 2;
  }
  k_best_choice<<<g1(n), kAT, 0, s>>>(n, indptr, col, w, matched, 1, choice);
  k_join<<<g1(n), kAT, 0, s>>>(n, choice, agg);
  DLP_CUDA(cudaMemsetAsync(flag, 0, sizeof(int32_t) * (size_t)n, s));
  k_self_and_flag<<<g1(n), kAT, 0, s>>>(n, agg, flag);
  // rank of each representative: exclusive scan of the flags, then every vertex maps through it
  DLP_TRY(exclusive_scan_i32(flag, n, choice, cws, cbytes, s));
  k_rank_gather<<<g1(n), kAT, 0, s>>>(n, choice, agg);
  DLP_CUDA(cudaMemcpyAsync(n_agg, choice + n, sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
  return check_launch(launches + 4);
}

size_t dlp_amg_members_workspace_bytes(int32_t nc) { return (((size_t)(nc > 0 ? nc : 1) * 4 + 255) / 256 * 256) + compact_ws_bytes(nc); }

int dlp_amg_members(int32_t n, int32_t nc, const int32_t *agg, int32_t *off, int32_t *members, void *ws,
                    size_t ws_bytes, dlp_stream_t stream) {
  if (n < 0 || nc < 0 || !off || (n > 0 && (!agg || !members))) return DLP_ERR_INVALID;
  if (!ws || ws_bytes < dlp_amg_members_workspace_bytes(nc)) return DLP_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t vb = ((size_t)(nc > 0 ? nc : 1) * 4 + 255) / 256 * 256;
  int32_t *cnt = (int32_t *)ws;
  DLP_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (size_t)(nc > 0 ? nc : 1), s));
  k_count_members<<<g1(n), kAT, 0, s>>>(n, agg, cnt);
  DLP_TRY(exclusive_scan_i32(cnt, nc, off, (char *)ws + vb, ws_bytes - vb, s));
  DLP_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (size_t)(nc > 0 ? nc : 1), s));
  k_fill_members<<<g1(n), kAT, 0, s>>>(n, agg, off, cnt, members);
  k_sort_members<<<g1(nc), kAT, 0, s>>>(nc, off, members);
  return check_launch(3);
}

// Table capacity (slots) for the coarse operator: toff[0..nc] is written; returns the total in
// *total_slots (device int). Call with a workspace of dlp_amg_members_workspace_bytes(nc).
int dlp_amg_coarse_plan(int32_t nc, const int32_t *off, const int32_t *members, const int32_t *indptr, int32_t *toff,
                        void *ws, size_t ws_bytes, dlp_stream_t stream) {
  if (nc < 0 || !toff) return DLP_ERR_INVALID;
  if (!ws || ws_bytes < dlp_amg_members_workspace_bytes(nc)) return DLP_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t vb = ((size_t)(nc > 0 ? nc : 1) * 4 + 255) / 256 * 256;
  int32_t *cap = (int32_t *)ws;
  if (nc > 0) k_coarse_bound<<<g1(nc), kAT, 0, s>>>(nc, off, members, indptr, cap);
  DLP_TRY(exclusive_scan_i32(cap, nc, toff, (char *)ws + vb, ws_bytes - vb, s));
  return check_launch(nc > 0 ? 1 : 0);
}

int dlp_amg_coarsen(int32_t nc, const int32_t *off, const int32_t *members, const int32_t *indptr, const int32_t *col,
                    const float *w, const int32_t *agg, const int32_t *toff, int32_t *tkey, double *tval,
                    int64_t total_slots, const double *s_fine, double *s_coarse, int32_t *indptr_c, int32_t *col_c,
                    float *w_c, void *ws, size_t ws_bytes, dlp_stream_t stream) {
  if (nc < 0 || total_slots < 0 || !indptr_c) return DLP_ERR_INVALID;
  if (!ws || ws_bytes < dlp_amg_members_workspace_bytes(nc)) return DLP_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t vb = ((size_t)(nc > 0 ? nc : 1) * 4 + 255) / 256 * 256;
  int32_t *rowcnt = (int32_t *)ws;
  if (total_slots > 0) DLP_CUDA(cudaMemsetAsync(tkey, 0xff, sizeof(int32_t) * (size_t)total_slots, s));
  if (nc > 0)
    k_coarse_accumulate<<<g1(nc), kAT, 0, s>>>(nc, off, members, indptr, col, w, agg, toff, tkey, tval, s_fine,
                                                s_coarse, rowcnt);
  DLP_TRY(exclusive_scan_i32(rowcnt, nc, indptr_c, (char *)ws + vb, ws_bytes - vb, s));
  if (nc > 0) k_coarse_emit<<<g1(nc), kAT, 0, s>>>(nc, toff, tkey, tval, indptr_c, col_c, w_c);
  return check_launch(nc > 0 ? 2 : 0);
}

int dlp_amg_restrict(int32_t nc, int32_t C, const int32_t *off, const int32_t *members, const void *R, int64_t ldr,
                     void *Rc, int64_t ldc, int dtype, dlp_stream_t stream) {
  if (nc < 0 || C <= 0 || ldr < C || ldc < C) return DLP_ERR_INVALID;
  if (nc == 0) return DLP_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const long long t = (long long)nc * C;
  if (dtype == DLP_F32)
    k_restrict<float><<<g1(t), kAT, 0, s>>>(nc, C, off, members, (const float *)R, ldr, (float *)Rc, ldc);
  else if (dtype == DLP_F64)
    k_restrict<double><<<g1(t), kAT, 0, s>>>(nc, C, off, members, (const double *)R, ldr, (double *)Rc, ldc);
  else
    return DLP_ERR_DTYPE;
  return check_launch();
}

int dlp_amg_prolong_add(int32_t n, int32_t C, const int32_t *agg, const void *Xc, int64_t ldc, void *X, int64_t ldx,
                        int dtype, dlp_stream_t stream) {
  if (n < 0 || C <= 0 || ldx < C || ldc < C) return DLP_ERR_INVALID;
  if (n == 0) return DLP_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const long long t = (long long)n * C;
  if (dtype == DLP_F32)
    k_prolong_add<float><<<g1(t), kAT, 0, s>>>(n, C, agg, (const float *)Xc, ldc, (float *)X, ldx);
  else if (dtype == DLP_F64)
    k_prolong_add<double><<<g1(t), kAT, 0, s>>>(n, C, agg, (const double *)Xc, ldc, (double *)X, ldx);
  else
    return DLP_ERR_DTYPE;
  return check_launch();
}

int dlp_amg_scale_rows(int32_t n, int32_t C, double omega, const void *R, int64_t ldr, const void *diag, void *X,
                       int64_t ldx, int dtype, dlp_stream_t stream) {
  if (n < 0 || C <= 0 || ldr < C || ldx < C) return DLP_ERR_INVALID;
  if (n == 0) return DLP_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const long long t = (long long)n * C;
  if (dtype == DLP_F32)
    k_scale_rows<float><<<g1(t), kAT, 0, s>>>(n, C, omega, (const float *)R, ldr, (const float *)diag, (float *)X, ldx);
  else if (dtype == DLP_F64)
    k_scale_rows<double><<<g1(t), kAT, 0, s>>>(n, C, omega, (const double *)R, ldr, (const double *)diag, (double *)X,
                                               ldx);
  else
    return DLP_ERR_DTYPE;
  return check_launch();
}

int dlp_amg_jacobi_sweep(int32_t n, int32_t C, const int32_t *indptr, const int32_t *col, const float *w,
                         const void *X, int64_t ldx, const void *RHS, int64_t ldr, const void *diag, double omega,
                         void *Y, int64_t ldy, int dtype, dlp_stream_t stream) {
  if (n < 0 || C <= 0 || ldx < C || ldr < C || ldy < C) return DLP_ERR_INVALID;
  if (n == 0) return DLP_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const long long t = (long long)n * 4;
  if (dtype == DLP_F32)
    k_jacobi_sweep<float><<<g1(t), kAT, 0, s>>>(n, C, indptr, col, w, (const float *)X, ldx, (const float *)RHS, ldr,
                                                (const float *)diag, omega, (float *)Y, ldy);
  else if (dtype == DLP_F64)
    k_jacobi_sweep<double><<<g1(t), kAT, 0, s>>>(n, C, indptr, col, w, (const double *)X, ldx, (const double *)RHS,
                                                 ldr, (const double *)diag, omega, (double *)Y, ldy);
  else
    return DLP_ERR_DTYPE;
  return check_launch();
}

int dlp_dense_apply(int32_t nc, int32_t C, const double *M, const void *X, int64_t ldx, void *Y, int64_t ldy,
                    int dtype, dlp_stream_t stream) {
  if (nc < 0 || C <= 0 || ldx < C || ldy < C) return DLP_ERR_INVALID;
  if (nc == 0) return DLP_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const long long t = (long long)nc * 32;
  if (dtype == DLP_F32)
    k_dense_apply<float><<<g1(t), kAT, 0, s>>>(nc, C, M, (const float *)X, ldx, (float *)Y, ldy);
  else if (dtype == DLP_F64)
    k_dense_apply<double><<<g1(t), kAT, 0, s>>>(nc, C, M, (const double *)X, ldx, (double *)Y, ldy);
  else
    return DLP_ERR_DTYPE;
  return check_launch();
}

int dlp_amg_coarse_keys(int32_t n, const int32_t *indptr, const int32_t *col, const float *w, const int32_t *agg,
                        int32_t nc, int64_t *key, double *val, dlp_stream_t stream) {
  if (n < 0 || nc < 0 || (n > 0 && (!indptr || !col || !w || !agg || !key || !val))) return DLP_ERR_INVALID;
  if (n == 0) return DLP_OK;
  k_coarse_keys<<<g1((long long)n * 8), kAT, 0, (cudaStream_t)stream>>>(n, indptr, col, w, agg, nc,
                                                                        (long long *)key, val);
  return check_launch();
}

size_t dlp_amg_coarse_reduce_workspace_bytes(int64_t m, int32_t nc) {
  const size_t a = (((size_t)(m > 0 ? m : 1) * 4 + 4 + 255) / 256 * 256) * 2;  // flags, positions (m + 1)
  const size_t b = (((size_t)(nc > 0 ? nc : 1) * 4 + 255) / 256 * 256);          // row counts
  return a + b + compact_ws_bytes((int32_t)std::min<int64_t>(std::max<int64_t>(m, nc), INT32_MAX - 1));
}

int dlp_amg_coarse_reduce(int64_t m, const int64_t *key, const double *val, int32_t nc, const int32_t *off,
                          const int32_t *members, const double *s_fine, double *s_coarse, int32_t *indptr_c,
                          int32_t *col_c, float *w_c, int32_t *nnz_c, void *ws, size_t ws_bytes,
                          dlp_stream_t stream) {
  if (m < 0 || m >= INT32_MAX || nc < 0 || !indptr_c || !nnz_c || (m > 0 && (!key || !val || !col_c || !w_c)))
    return DLP_ERR_INVALID;
  if (s_coarse && (!s_fine || !off || !members)) return DLP_ERR_INVALID;
  if (!ws || ws_bytes < dlp_amg_coarse_reduce_workspace_bytes(m, nc)) return DLP_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  char *p = (char *)ws;
  const size_t fb = ((size_t)(m > 0 ? m : 1) * 4 + 4 + 255) / 256 * 256;  // m + 1 ints: the scan writes pos[m]
  int32_t *flag = (int32_t *)p;
  int32_t *pos = (int32_t *)(p + fb);
  int32_t *rowcnt = (int32_t *)(p + 2 * fb);
  void *scan_ws = p + 2 * fb + (((size_t)(nc > 0 ? nc : 1) * 4 + 255) / 256 * 256);
  const size_t scan_bytes = ws_bytes - (size_t)((char *)scan_ws - p);
  if (nc > 0) DLP_CUDA(cudaMemsetAsync(rowcnt, 0, sizeof(int32_t) * (size_t)nc, s));
  int launches = 0;
  if (m > 0) {
    k_run_starts<<<g1(m), kAT, 0, s>>>(m, (const long long *)key, flag);
    launches += 1;
  }
  // pos = exclusive scan of the run starts; pos[m] = number of coarse entries
  DLP_TRY(exclusive_scan_i32(flag, (int32_t)m, pos, scan_ws, scan_bytes, s));
  if (m > 0) {
    k_run_emit<<<g1(m), kAT, 0, s>>>(m, (const long long *)key, val, flag, pos, nc, col_c, w_c, rowcnt);
    launches += 1;
  }
  DLP_TRY(exclusive_scan_i32(rowcnt, nc, indptr_c, scan_ws, scan_bytes, s));
  DLP_CUDA(cudaMemcpyAsync(nnz_c, indptr_c + nc, sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
  if (s_coarse && nc > 0) {
    k_member_sum<<<g1(nc), kAT, 0, s>>>(nc, off, members, s_fine, s_coarse);
    launches += 1;
  }
  return check_launch(launches);
}

}  // extern "C"
