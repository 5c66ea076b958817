// Ordered stream compaction (numpy.flatnonzero semantics) and deterministic column reductions.
#include <algorithm>
#include <mutex>

#include "common.cuh"

namespace dlp {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kTile = kScanThreads * kScanItems;

static inline int n_tiles(int32_t n) { return (int)((n + kTile - 1) / kTile); }

// Block-wide exclusive scan of one int per thread (256 threads). Returns the block total.
__device__ __forceinline__ int block_exclusive_scan(int v, int &excl) {
  __shared__ int warp_tot[kScanThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int inc = v;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, inc, off);
    if (lane >= off) inc += t;
  }
  if (lane == 31) warp_tot[wid] = inc;
  __syncthreads();
  int wpre = 0, total = 0;
#pragma unroll
  for (int w = 0; w < kScanThreads / 32; ++w) {
    const int t = warp_tot[w];
    if (w < wid) wpre += t;
    total += t;
  }
  excl = wpre + inc - v;
  __syncthreads();
  return total;
}

template <typename Pred>
__global__ void __launch_bounds__(kScanThreads) k_tile_count(Pred pred, int32_t n, int32_t *tile_cnt) {
  const long long base = (long long)blockIdx.x * kTile + (long long)threadIdx.x * kScanItems;
  int c = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const long long g = base + i;
    if (g < n && pred(g)) ++c;
  }
  int excl;
  const int tot = block_exclusive_scan(c, excl);
  if (threadIdx.x == 0) tile_cnt[blockIdx.x] = tot;
}

// Single-block exclusive scan of tile counts in place; total to *count (and *count2 if given).
__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(int32_t *tile, int nt, int32_t *count) {
  int carry = 0;
  for (int base = 0; base < nt; base += kScanThreads) {
    const int i = base + threadIdx.x;
    const int v = i < nt ? tile[i] : 0;
    int excl;
    const int tot = block_exclusive_scan(v, excl);
    if (i < nt) tile[i] = carry + excl;
    carry += tot;
  }
  if (threadIdx.x == 0 && count) *count = carry;
}

template <typename Pred>
__global__ void __launch_bounds__(kScanThreads)
    k_tile_write(Pred pred, int32_t n, const int32_t *__restrict__ tile_off, const int32_t *__restrict__ idx,
                 int32_t *out, int32_t *pos) {
  const long long base = (long long)blockIdx.x * kTile + (long long)threadIdx.x * kScanItems;
  bool f[kScanItems];
  int c = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const long long g = base + i;
    f[i] = g < n && pred(g);
    c += f[i];
  }
  int excl;
  block_exclusive_scan(c, excl);
  int o = tile_off[blockIdx.x] + excl;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (f[i]) {
      const long long g = base + i;
      if (out) out[o] = idx ? idx[g] : (int32_t)g;
      if (pos) pos[g] = o;
      ++o;
    }
  }
}

struct FlagPred {
  const uint8_t *flag;
  __device__ bool operator()(long long g) const { return flag[g] != 0; }
};
struct RootPred {
  const int32_t *parent;
  __device__ bool operator()(long long g) const { return parent[g] == (int32_t)g; }
};

struct MaskedRootPred {
  const int32_t *parent;
  const uint8_t *mask;
  __device__ bool operator()(long long g) const { return mask[g] != 0 && parent[g] == (int32_t)g; }
};

template <typename Pred>
static int compact_impl(Pred pred, const int32_t *idx, int32_t n, int32_t *out, int32_t *pos, int32_t *count,
                        void *ws, size_t ws_bytes, cudaStream_t s) {
  const int nt = n_tiles(n);
  if (n == 0) {
    if (count) DLP_CUDA(cudaMemsetAsync(count, 0, sizeof(int32_t), s));
    return DLP_OK;
  }
  if (!ws || ws_bytes < (size_t)nt * sizeof(int32_t)) return DLP_ERR_WORKSPACE;
  int32_t *tile = (int32_t *)ws;
  k_tile_count<<<nt, kScanThreads, 0, s>>>(pred, n, tile);
  k_scan_tiles<<<1, kScanThreads, 0, s>>>(tile, nt, count);
  k_tile_write<<<nt, kScanThreads, 0, s>>>(pred, n, tile, idx, out, pos);
  return check_launch(3);
}

// Exclusive scan of int32 counts: out[0] = 0, out[i+1] = sum_{j<=i} in[j] (out has n + 1 entries).
__global__ void __launch_bounds__(kScanThreads) k_tile_sum_i32(const int32_t *__restrict__ in, int32_t n,
                                                               int32_t *tile_sum) {
  const long long base = (long long)blockIdx.x * kTile + (long long)threadIdx.x * kScanItems;
  int c = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i)
    if (base + i < n) c += in[base + i];
  int excl;
  const int tot = block_exclusive_scan(c, excl);
  if (threadIdx.x == 0) tile_sum[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kScanThreads) k_tile_scan_i32(const int32_t *__restrict__ in, int32_t n,
                                                                const int32_t *__restrict__ tile_off, int32_t *out) {
  const long long base = (long long)blockIdx.x * kTile + (long long)threadIdx.x * kScanItems;
  int v[kScanItems];
  int c = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    v[i] = base + i < n ? in[base + i] : 0;
    c += v[i];
  }
  int excl;
  block_exclusive_scan(c, excl);
  int o = tile_off[blockIdx.x] + excl;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (base + i < n) out[base + i] = o;
    o += v[i];
  }
  if (base + kScanItems >= n && base < n) out[n] = o;  // the thread holding the last element
}

int exclusive_scan_i32(const int32_t *in, int32_t n, int32_t *out, void *ws, size_t ws_bytes, cudaStream_t s) {
  const int nt = n_tiles(n);
  if (n == 0) {
    DLP_CUDA(cudaMemsetAsync(out, 0, sizeof(int32_t), s));
    return DLP_OK;
  }
  if (!ws || ws_bytes < (size_t)nt * sizeof(int32_t)) return DLP_ERR_WORKSPACE;
  int32_t *tile = (int32_t *)ws;
  k_tile_sum_i32<<<nt, kScanThreads, 0, s>>>(in, n, tile);
  k_scan_tiles<<<1, kScanThreads, 0, s>>>(tile, nt, nullptr);
  k_tile_scan_i32<<<nt, kScanThreads, 0, s>>>(in, n, tile, out);
  return check_launch(3);
}

// ------------------------------------------------------------------------------------------------
// Stable LSD radix sort of (int64 key, fp64 value) pairs, 8 bits per pass (the AMG coarsening's
// sort by coarse entry). Keys above max_key order as max_key (the "no entry" marker sorts last).
// Per pass: tile histograms stored digit-major, one exclusive scan of them (each (digit, tile) gets
// its first output slot), then a stable scatter: a tile is taken in chunks of 256 elements in input
// order; inside a chunk equal digits are ranked by __match_any_sync per warp and per-warp counts in
// shared memory, and a running count per digit carries over to the next chunk.
// ------------------------------------------------------------------------------------------------
constexpr int kRsItems = 8;
constexpr int kRsTile = kScanThreads * kRsItems;

__device__ __forceinline__ int rs_digit(long long k, long long maxk, int shift) {
  k = k > maxk ? maxk : k;
  return (int)((k >> shift) & 255);
}

__global__ void __launch_bounds__(kScanThreads) k_rs_hist(long long m, const long long *__restrict__ keys,
                                                          long long maxk, int shift, int32_t *hist, int ntiles) {
  __shared__ int32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const long long base = (long long)blockIdx.x * kRsTile;
#pragma unroll
  for (int i = 0; i < kRsItems; ++i) {
    const long long e = base + (long long)i * kScanThreads + threadIdx.x;
    if (e < m) atomicAdd(&h[rs_digit(keys[e], maxk, shift)], 1);
  }
  __syncthreads();
  hist[(long long)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(kScanThreads)
    k_rs_scatter(long long m, const long long *__restrict__ keys, const double *__restrict__ vals, long long maxk,
                 int shift, const int32_t *__restrict__ offs, int ntiles, long long *keys_out, double *vals_out) {
  __shared__ int32_t s_base[256];
  __shared__ int32_t s_cnt[kScanThreads / 32][256];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  s_base[tid] = offs[(long long)tid * ntiles + blockIdx.x];
#pragma unroll
  for (int w = 0; w < kScanThreads / 32; ++w) s_cnt[w][tid] = 0;
  __syncthreads();
  const long long base = (long long)blockIdx.x * kRsTile;
  for (int i = 0; i < kRsItems; ++i) {
    const long long e = base + (long long)i * kScanThreads + tid;
    const bool valid = e < m;
    long long k = 0;
    double v = 0.0;
    int d = 256;  // no digit: past the end
    if (valid) {
      k = keys[e];
      v = vals[e];
      d = rs_digit(k, maxk, shift);
    }
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int wrank = __popc(peers & ((1u << lane) - 1u));
    if (valid && wrank == 0) s_cnt[wid][d] = __popc(peers);
    __syncthreads();
    if (valid) {
      int pre = 0;
      for (int w = 0; w < wid; ++w) pre += s_cnt[w][d];
      const int dest = s_base[d] + pre + wrank;
      keys_out[dest] = k;
      vals_out[dest] = v;
    }
    __syncthreads();
    int tot = 0;
#pragma unroll
    for (int w = 0; w < kScanThreads / 32; ++w) {
      tot += s_cnt[w][tid];
      s_cnt[w][tid] = 0;
    }
    s_base[tid] += tot;
    __syncthreads();
  }
}

size_t compact_ws_bytes(int32_t n) { return ((size_t)n_tiles(n) * sizeof(int32_t) + 255) / 256 * 256 + 256; }

int compact_roots(const int32_t *parent, int32_t n, int32_t *pos, int32_t *count, void *ws, size_t ws_bytes,
                  cudaStream_t s) {
  return compact_impl(RootPred{parent}, nullptr, n, nullptr, pos, count, ws, ws_bytes, s);
}

// pos[root] = rank of each masked root (mask[g] && parent[g] == g) among them; *count = their number.
int compact_masked_roots(const int32_t *parent, const uint8_t *mask, int32_t n, int32_t *pos, int32_t *count,
                         void *ws, size_t ws_bytes, cudaStream_t s) {
  return compact_impl(MaskedRootPred{parent, mask}, nullptr, n, nullptr, pos, count, ws, ws_bytes, s);
}

// out[0..*count) = the flagged g in ascending order (numpy.flatnonzero).
int compact_flags(const uint8_t *flag, int32_t n, int32_t *out, int32_t *count, void *ws, size_t ws_bytes,
                  cudaStream_t s) {
  return compact_impl(FlagPred{flag}, nullptr, n, out, nullptr, count, ws, ws_bytes, s);
}

// pos[g] = rank of g among the flagged entries (flag[g] != 0); *count = their number.
int compact_positions(const uint8_t *flag, int32_t n, int32_t *pos, int32_t *count, void *ws, size_t ws_bytes,
                      cudaStream_t s) {
  return compact_impl(FlagPred{flag}, nullptr, n, nullptr, pos, count, ws, ws_bytes, s);
}

// ------------------------------------------------------------------------------------------------
// column reductions: per-block partials over a fixed grid, then an ordered final pass
// ------------------------------------------------------------------------------------------------
constexpr int kRedBlocks = 296;
constexpr int kRedCols = 8;

template <typename T>
__global__ void __launch_bounds__(256)
    k_colreduce_partial(int kind, int32_t n, int32_t C, const T *__restrict__ X, int64_t ldx,
                        const T *__restrict__ Y, int64_t ldy, const T *__restrict__ diag,
                        const uint8_t *__restrict__ mask, double *partial) {
  __shared__ double sm[8][kRedCols];
  const long long chunk = ((long long)n + gridDim.x - 1) / gridDim.x;
  const long long r0 = (long long)blockIdx.x * chunk;
  const long long r1 = r0 + chunk < n ? r0 + chunk : n;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const bool is_max = kind == 0 || kind == 3;
  for (int c0 = 0; c0 < C; c0 += kRedCols) {
    double acc[kRedCols];
#pragma unroll
    for (int i = 0; i < kRedCols; ++i) acc[i] = 0.0;
    for (long long r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
      if (mask && !mask[r]) continue;
      double dinv = 1.0;
      if (kind == 0) dinv = 1.0 / (double)diag[r];
#pragma unroll
      for (int i = 0; i < kRedCols; ++i) {
        const int c = c0 + i;
        if (c < C) {
          const double x = (double)X[r * ldx + c];
          if (kind == 0) acc[i] = fmax(acc[i], fabs(x) * dinv);
          else if (kind == 1) acc[i] = fma(x, (double)Y[r * ldy + c], acc[i]);
          else if (kind == 2) acc[i] = fma(x, x, acc[i]);
          else acc[i] = fmax(acc[i], fabs(x));
        }
      }
    }
#pragma unroll
    for (int i = 0; i < kRedCols; ++i) {
      double v = acc[i];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double t = __shfl_xor_sync(0xffffffffu, v, off);
        v = is_max ? fmax(v, t) : v + t;
      }
      if (lane == 0) sm[wid][i] = v;
    }
    __syncthreads();
    if (threadIdx.x < kRedCols && c0 + threadIdx.x < C) {
      double v = sm[0][threadIdx.x];
      for (int w = 1; w < (int)(blockDim.x >> 5); ++w) v = is_max ? fmax(v, sm[w][threadIdx.x]) : v + sm[w][threadIdx.x];
      partial[(long long)blockIdx.x * C + c0 + threadIdx.x] = v;
    }
    __syncthreads();
  }
}

// One warp per column (lane-strided partials, fixed-order tree): deterministic.
__global__ void k_colreduce_final(int kind, int32_t C, int nb, const double *__restrict__ partial, double *out) {
  const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (c >= C) return;
  const double v = warp_strided_reduce(partial + c, C, nb, kind == 0 || kind == 3);
  if ((threadIdx.x & 31) == 0) out[c] = v;
}

// ------------------------------------------------------------------------------------------------
// Allocation-free column reduction. Some callers cannot allocate device memory at the point where
// they need a reduction: a serving process that reserved all of HBM for its own pool up front, a
// host runtime reached through a foreign-function bridge that has no device allocator wired in,
// or code that must not trigger the implicit synchronisation an allocation can cause. For them
// the per-block partial sums live in this fixed file-scope array instead of a caller workspace.
// Every GPU that loads the library holds it (kRedBlocks x kStaticMaxCols doubles = 151,552 bytes)
// until the process exits. All calls on a device share it, so calls that overlap on the GPU (on
// different streams, or from different host threads) race and must be serialised by the caller.
// Nothing in it has to start at zero: each call writes every partial it later reads.
// ------------------------------------------------------------------------------------------------
constexpr int kStaticMaxCols = 64;
static __device__ __align__(256) double g_colreduce_scratch[kRedBlocks * kStaticMaxCols];

constexpr int kMaxDevices = 64;
static std::mutex g_scratch_mu;
static double *g_scratch_addr[kMaxDevices];

// Device address of the array on the current device, looked up once per device. The name
// g_colreduce_scratch on the host is only a stand-in for the symbol, not a device address.
static int scratch_address(double **out) {
  int dev = 0;
  DLP_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return DLP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_colreduce_scratch);
    if (e != cudaSuccess) {
      set_cuda_error(e);
      return DLP_ERR_CUDA;
    }
    g_scratch_addr[dev] = (double *)p;
  }
  *out = g_scratch_addr[dev];
  return DLP_OK;
}

}  // namespace dlp

using namespace dlp;

extern "C" {

int dlp_colreduce_noalloc(int kind, int32_t n, int32_t C, const void *X, int64_t ldx, const void *Y, int64_t ldy,
                          const void *diag, int dtype, const uint8_t *mask, double *out, dlp_stream_t stream) {
  if (kind < 0 || kind > 3 || n < 0 || C <= 0 || ldx < C || !out) return DLP_ERR_INVALID;
  if (C > kStaticMaxCols) return DLP_ERR_SCRATCH_LIMIT;
  if (n > 0 && !X) return DLP_ERR_INVALID;
  if (kind == 0 && n > 0 && !diag) return DLP_ERR_INVALID;
  if (kind == 1 && n > 0 && (!Y || ldy < C)) return DLP_ERR_INVALID;
  double *partial = nullptr;
  DLP_TRY(scratch_address(&partial));
  cudaStream_t s = (cudaStream_t)stream;
  const int nb = n > 0 ? (n < kRedBlocks ? (n + 255) / 256 : kRedBlocks) : 0;
  if (nb > 0) {
    if (dtype == DLP_F32)
      k_colreduce_partial<float><<<nb, 256, 0, s>>>(kind, n, C, (const float *)X, ldx, (const float *)Y, ldy,
                                                    (const float *)diag, mask, partial);
    else if (dtype == DLP_F64)
      k_colreduce_partial<double><<<nb, 256, 0, s>>>(kind, n, C, (const double *)X, ldx, (const double *)Y, ldy,
                                                     (const double *)diag, mask, partial);
    else
      return DLP_ERR_DTYPE;
  }
  k_colreduce_final<<<(C + 7) / 8, 256, 0, s>>>(kind, C, nb, partial, out);
  return check_launch(nb > 0 ? 2 : 1);
}

size_t dlp_compact_workspace_bytes(int32_t n) { return compact_ws_bytes(n < 0 ? 0 : n); }

int dlp_compact(const uint8_t *flag, const int32_t *idx, int32_t n, int32_t *out, int32_t *count, void *ws,
                size_t ws_bytes, dlp_stream_t stream) {
  if (n < 0 || (n > 0 && (!flag || !out || !count))) return DLP_ERR_INVALID;
  return compact_impl(FlagPred{flag}, idx, n, out, nullptr, count, ws, ws_bytes, (cudaStream_t)stream);
}

size_t dlp_colreduce_workspace_bytes(int32_t C) { return (size_t)kRedBlocks * (C > 0 ? C : 1) * sizeof(double); }

int dlp_colreduce(int kind, int32_t n, int32_t C, const void *X, int64_t ldx, const void *Y, int64_t ldy,
                  const void *diag, int dtype, const uint8_t *mask, double *out, void *ws, size_t ws_bytes,
                  dlp_stream_t stream) {
  if (kind < 0 || kind > 3 || n < 0 || C <= 0 || ldx < C || !out) return DLP_ERR_INVALID;
  if (n > 0 && !X) return DLP_ERR_INVALID;
  if (kind == 0 && n > 0 && !diag) return DLP_ERR_INVALID;
  if (kind == 1 && n > 0 && (!Y || ldy < C)) return DLP_ERR_INVALID;
  if (!ws || ws_bytes < dlp_colreduce_workspace_bytes(C)) return DLP_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  double *partial = (double *)ws;
  const int nb = n > 0 ? (n < kRedBlocks ? (n + 255) / 256 : kRedBlocks) : 0;
  if (nb > 0) {
    if (dtype == DLP_F32)
      k_colreduce_partial<float><<<nb, 256, 0, s>>>(kind, n, C, (const float *)X, ldx, (const float *)Y, ldy,
                                                    (const float *)diag, mask, partial);
    else if (dtype == DLP_F64)
      k_colreduce_partial<double><<<nb, 256, 0, s>>>(kind, n, C, (const double *)X, ldx, (const double *)Y, ldy,
                                                     (const double *)diag, mask, partial);
    else
      return DLP_ERR_DTYPE;
  }
  k_colreduce_final<<<(C + 7) / 8, 256, 0, s>>>(kind, C, nb, partial, out);
  return check_launch(nb > 0 ? 2 : 1);
}


size_t dlp_sort_pairs_workspace_bytes(int64_t m) {
  const long long nt = (m + kRsTile - 1) / kRsTile;
  const long long h = 256 * (nt > 0 ? nt : 1);
  return (((size_t)h * 4 + 255) / 256 * 256) + (((size_t)(h + 1) * 4 + 255) / 256 * 256) +
         compact_ws_bytes((int32_t)std::min<long long>(h, INT32_MAX - 1));
}

int dlp_sort_pairs(int64_t m, int64_t max_key, int64_t *keys, double *vals, int64_t *keys_tmp, double *vals_tmp,
                   void *ws, size_t ws_bytes, dlp_stream_t stream) {
  if (m < 0 || max_key < 0 || (m > 0 && (!keys || !vals || !keys_tmp || !vals_tmp))) return DLP_ERR_INVALID;
  if (m >= ((long long)INT32_MAX / 2)) return DLP_ERR_INVALID;
  if (!ws || ws_bytes < dlp_sort_pairs_workspace_bytes(m)) return DLP_ERR_WORKSPACE;
  if (m <= 1) return DLP_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const int ntiles = (int)((m + kRsTile - 1) / kRsTile);
  const long long h = 256LL * ntiles;
  char *p = (char *)ws;
  int32_t *hist = (int32_t *)p;
  p += ((size_t)h * 4 + 255) / 256 * 256;
  int32_t *offs = (int32_t *)p;
  p += ((size_t)(h + 1) * 4 + 255) / 256 * 256;
  const size_t scan_bytes = ws_bytes - (size_t)(p - (char *)ws);
  int bits = 0;
  for (unsigned long long x = (unsigned long long)max_key; x; x >>= 1) ++bits;
  const int passes = bits > 0 ? (bits + 7) / 8 : 1;
  long long *kin = (long long *)keys, *kout = (long long *)keys_tmp;
  double *vin = vals, *vout = vals_tmp;
  int launches = 0;
  for (int pass = 0; pass < passes; ++pass) {
    const int shift = 8 * pass;
    k_rs_hist<<<ntiles, kScanThreads, 0, s>>>(m, kin, max_key, shift, hist, ntiles);
    DLP_TRY(exclusive_scan_i32(hist, (int32_t)h, offs, p, scan_bytes, s));
    k_rs_scatter<<<ntiles, kScanThreads, 0, s>>>(m, kin, vin, max_key, shift, offs, ntiles, kout, vout);
    launches += 2;
    std::swap(kin, kout);
    std::swap(vin, vout);
  }
  if (kin != (long long *)keys) {  // an odd number of passes: the result is in the spare arrays
    DLP_CUDA(cudaMemcpyAsync(keys, kin, sizeof(long long) * (size_t)m, cudaMemcpyDeviceToDevice, s));
    DLP_CUDA(cudaMemcpyAsync(vals, vin, sizeof(double) * (size_t)m, cudaMemcpyDeviceToDevice, s));
  }
  return check_launch(launches);
}

}  // extern "C"
