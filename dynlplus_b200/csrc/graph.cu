// The resident, edge-updatable graph and the per-batch patch of the grounded system.
//
// Layout: row r owns slots [rbeg[r], rcap[r]) of col/aw/w; [rbeg[r], rend[r]) are stored entries.
// aw holds the graph's edge weights (0 = a deleted edge: a tombstone that a later insertion of the
// same edge revives, unless the deletion squeezed its row); w holds the solver's operator W_UU (aw masked to 0 unless both endpoints are
// in the solved set U), the in-place masking of dynlp/stream.py:202-228. The patch keeps, for the
// grounded system (dynlp/stream.py:142-177 in its resident form :300-346):
//   rowsum[u] = sum_v w(u, v)                        (fp64)
//   B[u, c]   = sum of aw(u, l) over labelled l with class c   (fp64, n x K)
// and flags every row whose equation changed in `changed`.
//
// Edge batches: deletions first, then insertions; an insertion of a present edge sets its weight;
// repeated insertions of one edge in a batch keep the one with the largest batch index. The
// reference has no edge-level update; these are the semantics of the oracle's apply_edges.
#include "common.cuh"

namespace dlp {

int exclusive_scan_i32(const int32_t *in, int32_t n, int32_t *out, void *ws, size_t ws_bytes, cudaStream_t s);
size_t compact_ws_bytes(int32_t n);

constexpr int kGThreads = 256;
constexpr unsigned long long kEmpty = ~0ull;

__device__ __forceinline__ int find_entry(const int32_t *__restrict__ col, int beg, int end, int32_t v) {
  for (int j = beg; j < end; ++j)
    if (col[j] == v) return j;
  return -1;
}

// Effect of a weight change d on edge {a, b} on the grounded system.
__device__ __forceinline__ void account(int32_t a, int32_t b, int ja, int jb, float wnew, float d, float *w,
                                        const uint8_t *umask, const uint8_t *labeled, const int32_t *y, int32_t K,
                                        double *rowsum, double *B, uint8_t *changed) {
  const bool ua = umask[a], ub = umask[b];
  if (ua && ub) {
    if (ja >= 0) w[ja] = wnew;
    if (jb >= 0) w[jb] = wnew;
    atomicAdd(rowsum + a, (double)d);
    atomicAdd(rowsum + b, (double)d);
    changed[a] = 1;
    changed[b] = 1;
  } else {
    if (ja >= 0) w[ja] = 0.0f;
    if (jb >= 0) w[jb] = 0.0f;
  }
  if (labeled[b] && !labeled[a]) {
    atomicAdd(B + (long long)a * K + y[b], (double)d);
    if (ua) changed[a] = 1;
  }
  if (labeled[a] && !labeled[b]) {
    atomicAdd(B + (long long)b * K + y[a], (double)d);
    if (ub) changed[b] = 1;
  }
}

__global__ void __launch_bounds__(kGThreads)
    k_graph_delete(int32_t n, const int32_t *__restrict__ rbeg, const int32_t *rend, const int32_t *__restrict__ col,
                   float *aw, float *w, const int32_t *__restrict__ du, const int32_t *__restrict__ dv, int32_t nd,
                   const uint8_t *__restrict__ umask, const uint8_t *__restrict__ labeled,
                   const int32_t *__restrict__ y, int32_t K, double *rowsum, double *B, uint8_t *changed,
                   int32_t *n_applied, int32_t *err, uint8_t *squeeze) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nd) return;
  int32_t a = du[i], b = dv[i];
  if ((unsigned)a >= (unsigned)n || (unsigned)b >= (unsigned)n) {
    atomicExch(err, DLP_ERR_INVALID);
    return;
  }
  if (a == b) return;
  if (a > b) {
    const int32_t t = a;
    a = b;
    b = t;
  }
  const int ja = find_entry(col, rbeg[a], rend[a], b);
  if (ja < 0) return;
  // the canonical (min, max) entry decides which duplicate owns the deletion
  const float old = atomicExch(aw + ja, 0.0f);
  if (old == 0.0f) return;
  const int jb = find_entry(col, rbeg[b], rend[b], a);
  if (jb >= 0) aw[jb] = 0.0f;
  else atomicExch(err, DLP_ERR_DEVICE);  // asymmetric graph
  account(a, b, ja, jb, 0.0f, -old, w, umask, labeled, y, K, rowsum, B, changed);
  if (squeeze) {
    squeeze[a] = 1;
    squeeze[b] = 1;
  }
  if (n_applied) atomicAdd(n_applied, 1);
}

// Rows flagged in squeeze drop their deleted entries (aw == 0): the survivors move down in order
// (col, aw, w together) and rend shrinks, so the slots are free for later insertions instead of
// accumulating as tombstones until the row overflows. One thread per row; clears the flag.
__global__ void __launch_bounds__(kGThreads)
    k_graph_squeeze(int32_t n, const int32_t *__restrict__ rbeg, int32_t *rend, int32_t *col, float *aw, float *w,
                    uint8_t *squeeze) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n || !squeeze[r]) return;
  squeeze[r] = 0;
  const int end = rend[r];
  int k = rbeg[r];
  for (int j = k; j < end; ++j) {
    const float a = aw[j];
    if (a == 0.0f) continue;
    if (j != k) {
      col[k] = col[j];
      aw[k] = a;
      w[k] = w[j];
    }
    ++k;
  }
  rend[r] = k;
}

// Dedupe table: key (a << 32 | b) with the largest batch index that inserts it.
__global__ void k_dedupe(const int32_t *__restrict__ iu, const int32_t *__restrict__ iv, int32_t ni,
                         unsigned long long *keys, int32_t *best, uint32_t mask, int32_t n, int32_t *err) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ni) return;
  int32_t a = iu[i], b = iv[i];
  if ((unsigned)a >= (unsigned)n || (unsigned)b >= (unsigned)n) {
    atomicExch(err, DLP_ERR_INVALID);
    return;
  }
  if (a == b) return;
  if (a > b) {
    const int32_t t = a;
    a = b;
    b = t;
  }
  const unsigned long long key = ((unsigned long long)(uint32_t)a << 32) | (uint32_t)b;
  uint32_t h = (uint32_t)((key * 0x9E3779B97F4A7C15ull) >> 32) & mask;
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    const unsigned long long prev = atomicCAS(keys + h, kEmpty, key);
    if (prev == kEmpty || prev == key) {
      atomicMax(best + h, (int32_t)i);
      return;
    }
    h = (h + 1) & mask;
  }
  atomicExch(err, DLP_ERR_DEVICE);  // table full: cannot happen with 2x capacity
}

// Insertions run in two launches so that no row is searched while another thread appends to it.
// k_insert_find looks up both directed entries of every owned insertion in the rows as they stand
// before the batch's appends (stale column ids beyond rend are never read), and k_insert_apply then
// appends the missing ones and sets the weights. Each undirected pair has one owner (the dedupe), so
// the entries a pass touches are its own.
__global__ void __launch_bounds__(kGThreads)
    k_insert_find(int32_t n, const int32_t *__restrict__ rbeg, const int32_t *__restrict__ rend,
                  const int32_t *__restrict__ col, const int32_t *__restrict__ iu, const int32_t *__restrict__ iv,
                  int32_t ni, const unsigned long long *__restrict__ keys, const int32_t *__restrict__ best,
                  uint32_t mask, int32_t *__restrict__ slot_a, int32_t *__restrict__ slot_b) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ni) return;
  int32_t a = iu[i], b = iv[i];
  slot_a[i] = -2;  // -2: not this insertion's edge (invalid, a self-loop or a later duplicate owns it)
  if ((unsigned)a >= (unsigned)n || (unsigned)b >= (unsigned)n || a == b) return;
  if (a > b) {
    const int32_t t = a;
    a = b;
    b = t;
  }
  const unsigned long long key = ((unsigned long long)(uint32_t)a << 32) | (uint32_t)b;
  uint32_t h = (uint32_t)((key * 0x9E3779B97F4A7C15ull) >> 32) & mask;
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    if (keys[h] == key) break;
    h = (h + 1) & mask;
  }
  if (keys[h] != key || best[h] != (int32_t)i) return;
  slot_a[i] = find_entry(col, rbeg[a], rend[a], b);
  slot_b[i] = find_entry(col, rbeg[b], rend[b], a);
}

__global__ void __launch_bounds__(kGThreads)
    k_insert_apply(int32_t n, int32_t *rend, const int32_t *__restrict__ rcap, int32_t *col, float *aw, float *w,
                   const int32_t *__restrict__ iu, const int32_t *__restrict__ iv, const float *__restrict__ iw,
                   int32_t ni, const int32_t *__restrict__ slot_a, const int32_t *__restrict__ slot_b,
                   const uint8_t *__restrict__ umask, const uint8_t *__restrict__ labeled,
                   const int32_t *__restrict__ y, int32_t K, double *rowsum, double *B, uint8_t *changed,
                   int32_t *overflow, int32_t *n_applied) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ni) return;
  int ja = slot_a[i];
  if (ja == -2) return;
  int jb = slot_b[i];
  int32_t a = iu[i], b = iv[i];
  if (a > b) {
    const int32_t t = a;
    a = b;
    b = t;
  }
  const float wn = iw ? iw[i] : 1.0f;
  const float old = ja >= 0 ? aw[ja] : 0.0f;
  if (ja < 0) {
    ja = atomicAdd(rend + a, 1);
    if (ja >= rcap[a]) {
      atomicExch(overflow, 1);
      return;
    }
    col[ja] = b;
    aw[ja] = 0.0f;  // a tombstone until the mirror entry is in place too
    w[ja] = 0.0f;
  }
  if (jb < 0) {
    jb = atomicAdd(rend + b, 1);
    if (jb >= rcap[b]) {
      // row a keeps its entry at the old weight (a tombstone when new): the retry after the
      // rebuild finds it and completes the insertion
      atomicExch(overflow, 1);
      return;
    }
    col[jb] = a;
    w[jb] = 0.0f;
  }
  aw[ja] = wn;
  aw[jb] = wn;
  if (wn != old) account(a, b, ja, jb, wn, wn - old, w, umask, labeled, y, K, rowsum, B, changed);
  if (n_applied) atomicAdd(n_applied, 1);
}

__global__ void k_clamp_rend(int32_t n, int32_t *rend, const int32_t *__restrict__ rcap) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n && rend[r] > rcap[r]) rend[r] = rcap[r];
}

// Membership change of the vertices T (in_t[v] = 1 for v in T): solver weights of their entries
// and of the mirror entries follow umask; neighbours' row sums move by the difference
// (dynlp/stream.py:206-228). Rows of T get their sums recomputed by k_rowsum afterwards.
__global__ void __launch_bounds__(kGThreads)
    k_graph_toggle(const int32_t *__restrict__ rbeg, const int32_t *__restrict__ rend,
                   const int32_t *__restrict__ col, const float *__restrict__ aw, float *w,
                   const int32_t *__restrict__ T, int32_t nt, const uint8_t *__restrict__ in_t,
                   const uint8_t *__restrict__ umask, double *rowsum, uint8_t *changed) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long g = t >> 3;
  const int l = (int)(t & 7);
  if (g >= nt) return;
  const int32_t u = T ? T[g] : (int32_t)g;  // no list: every row flagged in in_t
  if (!T && !in_t[u]) return;
  const bool uu = umask[u];
  for (int j = rbeg[u] + l; j < rend[u]; j += 8) {
    const int32_t x = col[j];
    const float nw = (uu && umask[x]) ? aw[j] : 0.0f;
    const float ow = w[j];
    w[j] = nw;
    if (!in_t[x] && nw != ow) {
      const int jx = find_entry(col, rbeg[x], rend[x], u);
      if (jx >= 0) w[jx] = nw;
      if (umask[x]) {
        atomicAdd(rowsum + x, (double)(nw - ow));
        changed[x] = 1;
      }
    }
  }
  if (l == 0) changed[u] = 1;
}

// rowsum[r] for the rows flagged in flag (the toggled rows when they come without a list).
__global__ void k_rowsum_flagged(const int32_t *__restrict__ rbeg, const int32_t *__restrict__ rend,
                                 const float *__restrict__ w, const uint8_t *__restrict__ flag, int32_t nr,
                                 double *rowsum) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nr || !flag[r]) return;
  double s = 0.0;
  for (int j = rbeg[r]; j < rend[r]; ++j) s += (double)w[j];
  rowsum[r] = s;
}

__global__ void k_rowsum(const int32_t *__restrict__ rbeg, const int32_t *__restrict__ rend,
                         const float *__restrict__ w, const int32_t *__restrict__ rows, int32_t nr, double *rowsum) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nr) return;
  const int32_t r = rows ? rows[g] : (int32_t)g;
  double s = 0.0;
  for (int j = rbeg[r]; j < rend[r]; ++j) s += (double)w[j];
  rowsum[r] = s;
}

// The equations of the rows listed (dynlp/stream.py:329-331): solved rows get
//   s = sum_c B[u, c] + eta, diag = s + rowsum, rhs = B[u, cols] + eta * prior, rhs_h = diag,
// inert rows diag = 1, rhs = 0 (and the h column's rhs = 1). Writes fp64 and optional fp32 copies.
__global__ void k_system_rows(const int32_t *__restrict__ rows, int32_t nr, const uint8_t *__restrict__ umask,
                              const double *__restrict__ B, int32_t K, const double *__restrict__ rowsum, double eta,
                              const double *__restrict__ prior, int32_t C, int32_t col0, int32_t with_h,
                              double *diag64, double *rhs64, int64_t ldr64, float *diag32, float *rhs32,
                              int64_t ldr32) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nr) return;
  const long long u = rows ? rows[g] : g;
  const bool on = umask[u];
  double s = eta;
  for (int c = 0; c < K; ++c) s += B[u * K + c];
  const double d = on ? s + rowsum[u] : 1.0;
  diag64[u] = d;
  if (diag32) diag32[u] = (float)d;
  for (int c = 0; c < C; ++c) {
    const double v = on ? B[u * K + col0 + c] + eta * prior[c] : 0.0;
    rhs64[u * ldr64 + c] = v;
    if (rhs32) rhs32[u * ldr32 + c] = (float)v;
  }
  if (with_h) {
    rhs64[u * ldr64 + C] = d;
    if (rhs32) rhs32[u * ldr32 + C] = (float)d;
  }
}

// Inert rows leaving U: Z = (0, ..., 0, 1) (F = 0, h = 1: their exact solution), R = 0.
// Rows entering U: Z = (prior, h0).
__global__ void k_park(const int32_t *__restrict__ rows, int32_t nr, const uint8_t *__restrict__ umask, int32_t C,
                       int32_t with_h, const double *__restrict__ prior, double h0, double *Z, int64_t ldz,
                       double *R, int64_t ldr) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nr) return;
  const long long u = rows[g];
  const bool on = umask[u];
  for (int c = 0; c < C; ++c) {
    Z[u * ldz + c] = on ? prior[c] : 0.0;
    if (R) R[u * ldr + c] = 0.0;
  }
  if (with_h) {
    Z[u * ldz + C] = on ? h0 : 1.0;
    if (R) R[u * ldr + C] = 0.0;
  }
}

// Compact CSR of the solver operator: the entries with w != 0 of every row, in stored order.
// Solver CSR from the slots. The count keeps one thread per row (its serial scan is cheaper than a
// group of lanes per row, measured: 22 vs 50 us at n = 1M); the copy uses a group of kLiveGroup
// lanes per row reading the row's slots kLiveGroup at a time (consecutive: coalesced), ballot +
// popcount giving each live entry its place, so the compact row keeps the slot order (measured: 73
// vs 104 us with one thread per row).
constexpr int kLiveGroup = 8;

__global__ void k_live_count(int32_t n, const int32_t *__restrict__ rbeg, const int32_t *__restrict__ rend,
                             const float *__restrict__ w, int32_t *cnt) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  int c = 0;
  for (int j = rbeg[r]; j < rend[r]; ++j) c += w[j] != 0.0f;
  cnt[r] = c;
}

__global__ void k_live_copy(int32_t n, const int32_t *__restrict__ rbeg, const int32_t *__restrict__ rend,
                            const int32_t *__restrict__ col, const float *__restrict__ w,
                            const int32_t *__restrict__ indptr, int32_t *col_out, float *w_out) {
  constexpr int G = kLiveGroup;
  const int lane = threadIdx.x & 31, gl = lane & (G - 1), gshift = lane & ~(G - 1);
  const long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / G;
  const bool valid = r < n;
  const int b = valid ? rbeg[r] : 0, e = valid ? rend[r] : 0;
  int o = valid ? indptr[r] : 0;
  for (int base = b; __any_sync(0xffffffffu, base < e); base += G) {
    const int j = base + gl;
    const float x = j < e ? w[j] : 0.0f;
    const bool lv = x != 0.0f;
    const unsigned m = (__ballot_sync(0xffffffffu, lv) >> gshift) & ((1u << G) - 1);
    if (lv) {
      const int p = o + __popc(m & ((1u << gl) - 1));
      col_out[p] = col[j];
      w_out[p] = x;
    }
    o += __popc(m);
  }
}

static int grid1(long long work) { return ceil_div_i(work > 0 ? work : 1, kGThreads); }

static uint32_t table_size(int32_t ni) {
  uint32_t s = 16;
  while (s < (uint32_t)ni * 2u) s <<= 1;
  return s;
}

// Labelled vertices entering (sign +1) or leaving (sign -1) the active set: every live neighbour v of
// l gets B[v, y[l]] += sign * aw(l, v), and is flagged changed when it is solved
// (dynlp/stream.py:230-235). One group of 8 lanes per labelled vertex.
__global__ void __launch_bounds__(kGThreads)
    k_label_update(const int32_t *__restrict__ L, int32_t nl, double sign, const int32_t *__restrict__ rbeg,
                   const int32_t *__restrict__ rend, const int32_t *__restrict__ col, const float *__restrict__ aw,
                   const int32_t *__restrict__ y, int32_t K, double *B, const uint8_t *__restrict__ umask,
                   uint8_t *changed) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long g = t >> 3;
  const int l8 = (int)(t & 7);
  if (g >= nl) return;
  const int32_t l = L[g];
  const int32_t c = y[l];
  for (int j = rbeg[l] + l8; j < rend[l]; j += 8) {
    const float a = aw[j];
    if (a == 0.0f) continue;
    const int32_t v = col[j];
    atomicAdd(B + (long long)v * K + c, sign * (double)a);
    if (changed && umask[v]) changed[v] = 1;
  }
}

// Per new vertex (DynLP step 1, dynlp/stream.py:72-76): its mean dissimilarity over its live
// entries, s = (sum over w > 0 of (1 - w / wmax), each term rounded to fp32, summed in fp32 in
// row order) / max(count, 1) + 1e-6. The terms are formed in the weights' precision first, as
// the reference's vectorised expression does; one thread per row keeps the row order.
template <typename TW>
__global__ void k_new_dissim(const int32_t *__restrict__ rows, int32_t m, const int32_t *__restrict__ rbeg,
                             const int32_t *__restrict__ rend, const TW *__restrict__ w, double wmax, float *s) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int32_t r = rows[i];
  const TW wm = (TW)wmax;
  float acc = 0.0f, cnt = 0.0f;
  for (int j = rbeg[r]; j < rend[r]; ++j) {
    const TW x = w[j];
    if (!(x > (TW)0)) continue;
    acc = __fadd_rn(acc, (float)((TW)1 - x / wm));
    cnt = __fadd_rn(cnt, 1.0f);
  }
  s[i] = __fadd_rn(__fdiv_rn(acc, fmaxf(cnt, 1.0f)), 1e-6f);
}

}  // namespace dlp

using namespace dlp;

extern "C" {

int dlp_graph_delete(int32_t n, const int32_t *rbeg, int32_t *rend, int32_t *col, float *aw, float *w,
                     const int32_t *du, const int32_t *dv, int32_t nd, const uint8_t *umask, const uint8_t *labeled,
                     const int32_t *y, int32_t K, double *rowsum, double *B, uint8_t *changed, int32_t *n_applied,
                     int32_t *err, uint8_t *squeeze, dlp_stream_t stream) {
  if (n < 0 || nd < 0 || K <= 0) return DLP_ERR_INVALID;
  if (nd == 0) return DLP_OK;
  if (!rbeg || !rend || !col || !aw || !w || !du || !dv || !umask || !labeled || !y || !rowsum || !B || !changed ||
      !err)
    return DLP_ERR_INVALID;
  k_graph_delete<<<grid1(nd), kGThreads, 0, (cudaStream_t)stream>>>(n, rbeg, rend, col, aw, w, du, dv, nd, umask,
                                                                     labeled, y, K, rowsum, B, changed, n_applied,
                                                                     err, squeeze);
  if (squeeze) k_graph_squeeze<<<grid1(n), kGThreads, 0, (cudaStream_t)stream>>>(n, rbeg, rend, col, aw, w, squeeze);
  return check_launch(squeeze ? 2 : 1);
}

size_t dlp_graph_insert_workspace_bytes(int32_t ni) {
  const size_t ts = table_size(ni > 0 ? ni : 1);
  const size_t m = (size_t)(ni > 0 ? ni : 1);
  return ts * sizeof(unsigned long long) + ts * sizeof(int32_t) + 2 * m * sizeof(int32_t) + 256;
}

int dlp_graph_insert(int32_t n, const int32_t *rbeg, int32_t *rend, const int32_t *rcap, int32_t *col, float *aw,
                     float *w, const int32_t *iu, const int32_t *iv, const float *iw, int32_t ni,
                     const uint8_t *umask, const uint8_t *labeled, const int32_t *y, int32_t K, double *rowsum,
                     double *B, uint8_t *changed, int32_t *overflow, int32_t *n_applied, int32_t *err, void *ws,
                     size_t ws_bytes, dlp_stream_t stream) {
  if (n < 0 || ni < 0 || K <= 0) return DLP_ERR_INVALID;
  if (ni == 0) return DLP_OK;
  if (!rbeg || !rend || !rcap || !col || !aw || !w || !iu || !iv || !umask || !labeled || !y || !rowsum || !B ||
      !changed || !overflow || !err)
    return DLP_ERR_INVALID;
  if (!ws || ws_bytes < dlp_graph_insert_workspace_bytes(ni)) return DLP_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  const uint32_t ts = table_size(ni);
  unsigned long long *keys = (unsigned long long *)ws;
  int32_t *best = (int32_t *)(keys + ts);
  int32_t *slot_a = best + ts;
  int32_t *slot_b = slot_a + ni;
  DLP_CUDA(cudaMemsetAsync(keys, 0xff, ts * sizeof(unsigned long long), s));
  DLP_CUDA(cudaMemsetAsync(best, 0xff, ts * sizeof(int32_t), s));
  k_dedupe<<<grid1(ni), kGThreads, 0, s>>>(iu, iv, ni, keys, best, ts - 1, n, err);
  k_insert_find<<<grid1(ni), kGThreads, 0, s>>>(n, rbeg, rend, col, iu, iv, ni, keys, best, ts - 1, slot_a, slot_b);
  k_insert_apply<<<grid1(ni), kGThreads, 0, s>>>(n, rend, rcap, col, aw, w, iu, iv, iw, ni, slot_a, slot_b, umask,
                                                  labeled, y, K, rowsum, B, changed, overflow, n_applied);
  k_clamp_rend<<<grid1(n), kGThreads, 0, s>>>(n, rend, rcap);
  return check_launch(4);
}

int dlp_graph_toggle(const int32_t *rbeg, const int32_t *rend, const int32_t *col, const float *aw, float *w,
                     const int32_t *T, int32_t nt, const uint8_t *in_t, const uint8_t *umask, double *rowsum,
                     uint8_t *changed, dlp_stream_t stream) {
  if (nt < 0) return DLP_ERR_INVALID;
  if (nt == 0) return DLP_OK;
  if (!rbeg || !rend || !col || !aw || !w || !in_t || !umask || !rowsum || !changed) return DLP_ERR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  k_graph_toggle<<<grid1((long long)nt * 8), kGThreads, 0, s>>>(rbeg, rend, col, aw, w, T, nt, in_t, umask, rowsum,
                                                                 changed);
  if (T)
    k_rowsum<<<grid1(nt), kGThreads, 0, s>>>(rbeg, rend, w, T, nt, rowsum);
  else
    k_rowsum_flagged<<<grid1(nt), kGThreads, 0, s>>>(rbeg, rend, w, in_t, nt, rowsum);
  return check_launch(2);
}

size_t dlp_graph_to_csr_workspace_bytes(int32_t n) { return compact_ws_bytes(n) + sizeof(int32_t) * (size_t)(n > 0 ? n : 1) + 256; }

int dlp_graph_to_csr(int32_t n, const int32_t *rbeg, const int32_t *rend, const int32_t *col, const float *w,
                     int32_t *indptr, int32_t *col_out, float *w_out, void *ws, size_t ws_bytes, dlp_stream_t stream) {
  if (n < 0 || !indptr) return DLP_ERR_INVALID;
  if (n > 0 && (!rbeg || !rend || !col || !w || !col_out || !w_out)) return DLP_ERR_INVALID;
  if (!ws || ws_bytes < dlp_graph_to_csr_workspace_bytes(n)) return DLP_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  int32_t *cnt = (int32_t *)ws;
  void *scan_ws = (char *)ws + ((sizeof(int32_t) * (size_t)(n > 0 ? n : 1) + 255) / 256 * 256);
  const size_t scan_bytes = ws_bytes - ((sizeof(int32_t) * (size_t)(n > 0 ? n : 1) + 255) / 256 * 256);
  if (n > 0) k_live_count<<<grid1(n), kGThreads, 0, s>>>(n, rbeg, rend, w, cnt);
  DLP_TRY(exclusive_scan_i32(cnt, n, indptr, scan_ws, scan_bytes, s));
  if (n > 0)
    k_live_copy<<<grid1((long long)n * kLiveGroup), kGThreads, 0, s>>>(n, rbeg, rend, col, w, indptr, col_out, w_out);
  return check_launch(n > 0 ? 2 : 0);
}

int dlp_graph_rowsum(const int32_t *rbeg, const int32_t *rend, const float *w, const int32_t *rows, int32_t nr,
                     double *rowsum, dlp_stream_t stream) {
  if (nr < 0 || (nr > 0 && (!rbeg || !rend || !w || !rowsum))) return DLP_ERR_INVALID;
  if (nr == 0) return DLP_OK;
  k_rowsum<<<grid1(nr), kGThreads, 0, (cudaStream_t)stream>>>(rbeg, rend, w, rows, nr, rowsum);
  return check_launch();
}

int dlp_system_rows(const int32_t *rows, int32_t nr, const uint8_t *umask, const double *B, int32_t K,
                    const double *rowsum, double eta, const double *prior, int32_t C, int32_t col0, int32_t with_h,
                    double *diag64, double *rhs64, int64_t ldr64, float *diag32, float *rhs32, int64_t ldr32,
                    dlp_stream_t stream) {
  if (nr < 0 || K <= 0 || C <= 0 || col0 < 0 || col0 + C > K || ldr64 < C + (with_h ? 1 : 0)) return DLP_ERR_INVALID;
  if (rhs32 && ldr32 < C + (with_h ? 1 : 0)) return DLP_ERR_INVALID;
  if (nr == 0) return DLP_OK;
  if (!umask || !B || !rowsum || !prior || !diag64 || !rhs64) return DLP_ERR_INVALID;
  k_system_rows<<<grid1(nr), kGThreads, 0, (cudaStream_t)stream>>>(rows, nr, umask, B, K, rowsum, eta, prior, C, col0,
                                                                    with_h, diag64, rhs64, ldr64, diag32, rhs32,
                                                                    ldr32);
  return check_launch();
}

int dlp_park_rows(const int32_t *rows, int32_t nr, const uint8_t *umask, int32_t C, int32_t with_h,
                  const double *prior, double h0, double *Z, int64_t ldz, double *R, int64_t ldr,
                  dlp_stream_t stream) {
  if (nr < 0 || C <= 0) return DLP_ERR_INVALID;
  if (nr == 0) return DLP_OK;
  if (!rows || !umask || !prior || !Z) return DLP_ERR_INVALID;
  k_park<<<grid1(nr), kGThreads, 0, (cudaStream_t)stream>>>(rows, nr, umask, C, with_h, prior, h0, Z, ldz, R, ldr);
  return check_launch();
}

int dlp_label_update(const int32_t *L, int32_t nl, double sign, const int32_t *rbeg, const int32_t *rend,
                     const int32_t *col, const float *aw, const int32_t *y, int32_t K, double *B, const uint8_t *umask,
                     uint8_t *changed, dlp_stream_t stream) {
  if (nl < 0 || K <= 0) return DLP_ERR_INVALID;
  if (nl == 0) return DLP_OK;
  if (!L || !rbeg || !rend || !col || !aw || !y || !B || (changed && !umask)) return DLP_ERR_INVALID;
  k_label_update<<<grid1((long long)nl * 8), kGThreads, 0, (cudaStream_t)stream>>>(L, nl, sign, rbeg, rend, col, aw,
                                                                                   y, K, B, umask, changed);
  return check_launch();
}

int dlp_new_dissim(const int32_t *rows, int32_t m, const int32_t *rbeg, const int32_t *rend, const void *w,
                   int w_dtype, double wmax, float *s, dlp_stream_t stream) {
  if (m < 0 || !(wmax > 0.0)) return DLP_ERR_INVALID;
  if (m == 0) return DLP_OK;
  if (!rows || !rbeg || !rend || !w || !s) return DLP_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  if (w_dtype == DLP_F32)
    k_new_dissim<float><<<grid1(m), kGThreads, 0, st>>>(rows, m, rbeg, rend, (const float *)w, wmax, s);
  else if (w_dtype == DLP_F64)
    k_new_dissim<double><<<grid1(m), kGThreads, 0, st>>>(rows, m, rbeg, rend, (const double *)w, wmax, s);
  else
    return DLP_ERR_DTYPE;
  return check_launch();
}

}  // extern "C"
