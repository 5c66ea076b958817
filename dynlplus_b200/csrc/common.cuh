// Shared device helpers for libdlp (sm_100a only).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <memory>

#include "dlp.h"

namespace dlp {

using bf16 = __nv_bfloat16;

// ---- status plumbing --------------------------------------------------------------------------
void set_cuda_error(cudaError_t e);
int check_launch(int kernels = 1);  // cudaGetLastError -> status; counts `kernels` launches
int sm_count();
void note_launches(unsigned long long k);  // kernels launched outside check_launch (graph replays)
// The word dlp_set_cancel_word registered (NULL: none). Device loops read it with volatile loads.
const int32_t *cancel_word();

// One thread's read of the cancel word (host-mapped or device memory; NULL reads as 0).
__device__ __forceinline__ int read_cancel(const int32_t *word) {
  return word ? *(const volatile int32_t *)word : 0;
}

#define DLP_TRY(expr)                 \
  do {                                \
    int _st = (expr);                 \
    if (_st != DLP_OK) return _st;    \
  } while (0)

#define DLP_CUDA(expr)                         \
  do {                                         \
    cudaError_t _e = (expr);                   \
    if (_e != cudaSuccess) {                   \
      ::dlp::set_cuda_error(_e);               \
      return DLP_ERR_CUDA;                     \
    }                                          \
  } while (0)

// An instantiated CUDA graph shared between a cache and the solves replaying it: the cache may
// drop its reference (eviction) while another thread's solve still replays the graph; the graph is
// destroyed when the last holder lets go.
struct GraphExec {
  cudaGraphExec_t ex = nullptr;
  GraphExec() = default;
  GraphExec(const GraphExec &) = delete;
  GraphExec &operator=(const GraphExec &) = delete;
  ~GraphExec() {
    if (ex) cudaGraphExecDestroy(ex);
  }
};
using GraphRef = std::shared_ptr<GraphExec>;

inline size_t dtype_size(int dt) { return dt == DLP_F64 ? 8 : dt == DLP_F32 ? 4 : dt == DLP_BF16 ? 2 : 0; }

// ---- conversions ------------------------------------------------------------------------------
template <typename TA, typename T>
__device__ __forceinline__ TA cvt(T x) { return static_cast<TA>(x); }
template <>
__device__ __forceinline__ float cvt<float, bf16>(bf16 x) { return __bfloat162float(x); }
template <>
__device__ __forceinline__ double cvt<double, bf16>(bf16 x) { return (double)__bfloat162float(x); }
template <>
__device__ __forceinline__ bf16 cvt<bf16, float>(float x) { return __float2bfloat16_rn(x); }
template <>
__device__ __forceinline__ bf16 cvt<bf16, double>(double x) { return __double2bfloat16(x); }

template <typename T>
__device__ __forceinline__ T ld_stream(const T *p) { return __ldcs(p); }
template <>
__device__ __forceinline__ bf16 ld_stream<bf16>(const bf16 *p) {
  unsigned short u = __ldcs(reinterpret_cast<const unsigned short *>(p));
  return __ushort_as_bfloat16(u);
}

// Load VW consecutive elements of T (16-byte vector when VW*sizeof(T) == 16), converted to TA.
template <typename T, int VW, typename TA>
__device__ __forceinline__ void load_vec(const T *__restrict__ p, TA (&out)[VW]) {
  if constexpr (VW * sizeof(T) == 16) {
    const uint4 raw = __ldg(reinterpret_cast<const uint4 *>(p));
    const T *e = reinterpret_cast<const T *>(&raw);
#pragma unroll
    for (int i = 0; i < VW; ++i) out[i] = cvt<TA>(e[i]);
  } else {
#pragma unroll
    for (int i = 0; i < VW; ++i) out[i] = cvt<TA>(p[i]);
  }
}

// Same, through the coherent path (data written earlier in the same kernel or by atomics).
template <typename T, int VW, typename TA>
__device__ __forceinline__ void load_vec_coherent(const T *p, TA (&out)[VW]) {
  if constexpr (VW * sizeof(T) == 16) {
    const uint4 raw = __ldcg(reinterpret_cast<const uint4 *>(p));
    const T *e = reinterpret_cast<const T *>(&raw);
#pragma unroll
    for (int i = 0; i < VW; ++i) out[i] = cvt<TA>(e[i]);
  } else {
#pragma unroll
    for (int i = 0; i < VW; ++i) out[i] = cvt<TA>(__ldcg(p + i));
  }
}

__device__ __forceinline__ void atomic_add(float *p, float v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_add(double *p, double v) { atomicAdd(p, v); }

// Hardware lane id (correct for 1-D and multi-dimensional blocks alike).
__device__ __forceinline__ int lane_id() {
  unsigned l;
  asm volatile("mov.u32 %0, %%laneid;" : "=r"(l));
  return (int)l;
}

// Warp-aggregated append: every lane with pred=true gets a unique slot in out (order within a
// warp follows lane order; across warps it is unordered).
__device__ __forceinline__ void warp_append(bool pred, int32_t value, int32_t *out, int32_t *count) {
  const unsigned mask = __activemask();
  const unsigned ballot = __ballot_sync(mask, pred);
  if (!ballot) return;
  const int lane = lane_id();
  const int leader = __ffs(ballot) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(count, __popc(ballot));
  base = __shfl_sync(mask, base, leader);
  if (pred) out[base + __popc(ballot & ((1u << lane) - 1u))] = value;
}

// Warp-aggregated slot reservation: the lanes with pred=true get consecutive slots of `count`
// (lane order within the warp, one atomic per warp); returns the lane's slot, or -1 without pred.
__device__ __forceinline__ int warp_reserve(bool pred, int32_t *count) {
  const unsigned mask = __activemask();
  const unsigned ballot = __ballot_sync(mask, pred);
  if (!ballot) return -1;
  const int lane = lane_id();
  const int leader = __ffs(ballot) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(count, __popc(ballot));
  base = __shfl_sync(mask, base, leader);
  return pred ? base + __popc(ballot & ((1u << lane) - 1u)) : -1;
}

// Deterministic warp-wide sum (or max) of base[b * stride] over b < nb: lane l takes b = l, l+32,
// ... in groups of 8 independent loads (8 accumulators, so 8 loads are in flight per lane), the
// accumulators are combined in a fixed tree, then a fixed xor tree across lanes. All lanes get the
// result; the order depends only on nb.
__device__ __forceinline__ double warp_strided_reduce(const double *base, long long stride, int nb, bool is_max) {
  const int lane = lane_id();
  double a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = 0.0;
  int b = lane;
  for (; b + 7 * 32 < nb; b += 8 * 32) {
    double x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = base[(long long)(b + 32 * k) * stride];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = is_max ? fmax(a[k], x[k]) : a[k] + x[k];
  }
#pragma unroll
  for (int k = 0; k < 7; ++k) {  // the tail: fewer than 8 loads left per lane
    if (b + 32 * k < nb) {
      const double x = base[(long long)(b + 32 * k) * stride];
      a[k] = is_max ? fmax(a[k], x) : a[k] + x;
    }
  }
#pragma unroll
  for (int w = 4; w > 0; w >>= 1)
#pragma unroll
    for (int k = 0; k < w; ++k) a[k] = is_max ? fmax(a[k], a[k + w]) : a[k] + a[k + w];
  double v = a[0];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const double t = __shfl_xor_sync(0xffffffffu, v, off);
    v = is_max ? fmax(v, t) : v + t;
  }
  return v;
}

inline int ceil_div_i(long long a, long long b) { return (int)((a + b - 1) / b); }

inline int next_pow2(int x) {
  int p = 1;
  while (p < x) p <<= 1;
  return p;
}

// kernels.auto_group (dynlp/kernels.py:365-370): power-of-two lanes near the mean degree, in [2, 32].
inline int auto_group(double avg_deg) {
  int g = 2;
  double d = avg_deg > 1.0 ? avg_deg : 1.0;
  while (g < 32 && g * 2 <= d) g *= 2;
  return g;
}

}  // namespace dlp
