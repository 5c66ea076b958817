// Column-scaled vector updates of the refinement loop and the grounding update.
#include "common.cuh"

namespace dlp {

// op 0: Y = X / scale[c]   op 1: Y += X * scale[c]   op 2: Y = X * scale[c]   op 3: Y = X + Y * scale[c]
// Thread t of the grid owns column c = t mod C of rows t/C, t/C + RS, ... (RS = threads / C): no
// integer division per element, consecutive threads on consecutive columns of a row, and
// kColsUnroll rows loaded before any is stored.
constexpr int kColsUnroll = 4;
constexpr int kColsThreads = 256;

template <typename TX, typename TY>
__global__ void __launch_bounds__(kColsThreads) k_cols_scale(int32_t n, int32_t C, const TX *__restrict__ X,
                                                             int64_t ldx, const double *__restrict__ scale, int op,
                                                             TY *Y, int64_t ldy) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long RS = (long long)gridDim.x * blockDim.x / C;
  const long long r0 = t / C;
  const int c = (int)(t - r0 * C);
  if (r0 >= RS) return;
  const double s = scale[c];
  const bool rd = sizeof(TY) != 2 && (op == 1 || op == 3);  // the op reads Y
  const long long sx = RS * ldx, sy = RS * ldy;
  long long ox = r0 * ldx + c, oy = r0 * ldy + c;
  for (long long r = r0; r < n; r += kColsUnroll * RS) {
    double x[kColsUnroll], y[kColsUnroll];
#pragma unroll
    for (int u = 0; u < kColsUnroll; ++u) {
      const bool ok = r + u * RS < n;
      x[u] = ok ? (double)X[ox + u * sx] : 0.0;
      if constexpr (sizeof(TY) != 2) y[u] = (ok && rd) ? (double)Y[oy + u * sy] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kColsUnroll; ++u) {
      if (r + u * RS >= n) continue;
      TY *yp = Y + oy + u * sy;
      if constexpr (sizeof(TY) == 2) {
        *yp = cvt<TY>(x[u] * s);  // the bf16 mirror: op 2 only
      } else {
        if (op == 0) *yp = (TY)(x[u] / s);
        else if (op == 1) *yp = (TY)(y[u] + x[u] * s);
        else if (op == 2) *yp = (TY)(x[u] * s);
        else *yp = (TY)(x[u] + y[u] * s);
      }
    }
    ox += kColsUnroll * sx;
    oy += kColsUnroll * sy;
  }
}

// umask[v] = vmask[v] && root(v) == root(sink); in_t[v] = membership changed; counts[0] += |changed|
__global__ void k_ground_update(int32_t n, const int32_t *__restrict__ parent, const uint8_t *__restrict__ vmask,
                                uint8_t *umask, uint8_t *in_t, int32_t *counts) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  bool ch = false;
  if (v < n) {
    const bool nu = vmask[v] && parent[v] == parent[n];
    const bool ou = umask[v] != 0;
    ch = nu != ou;
    umask[v] = nu ? 1 : 0;
    in_t[v] = ch ? 1 : 0;
  }
  const unsigned b = __ballot_sync(0xffffffffu, ch);
  if ((threadIdx.x & 31) == 0 && b) atomicAdd(counts, __popc(b));
}

}  // namespace dlp

using namespace dlp;

extern "C" {

int dlp_cols_scale(int32_t n, int32_t C, const void *X, int64_t ldx, int x_dtype, const double *scale, int32_t op,
                   void *Y, int64_t ldy, int y_dtype, dlp_stream_t stream) {
  if (n < 0 || C <= 0 || ldx < C || ldy < C || op < 0 || op > 3) return DLP_ERR_INVALID;
  if (n == 0) return DLP_OK;
  if (!X || !Y || !scale) return DLP_ERR_INVALID;
  // enough threads for a row pass (>= C) and for the elements, at most 8 resident blocks per SM
  long long blocks = ceil_div_i((long long)n * C, (long long)kColsThreads * kColsUnroll);
  blocks = std::min(blocks, (long long)sm_count() * 8);
  blocks = std::max(blocks, (long long)ceil_div_i((long long)C, kColsThreads));
  const int grid = (int)blocks;
  cudaStream_t s = (cudaStream_t)stream;
  if (x_dtype == DLP_F64 && y_dtype == DLP_F32)
    k_cols_scale<double, float><<<grid, kColsThreads, 0, s>>>(n, C, (const double *)X, ldx, scale, op, (float *)Y, ldy);
  else if (x_dtype == DLP_F32 && y_dtype == DLP_F64)
    k_cols_scale<float, double><<<grid, kColsThreads, 0, s>>>(n, C, (const float *)X, ldx, scale, op, (double *)Y, ldy);
  else if (x_dtype == DLP_F64 && y_dtype == DLP_F64)
    k_cols_scale<double, double><<<grid, kColsThreads, 0, s>>>(n, C, (const double *)X, ldx, scale, op, (double *)Y, ldy);
  else if (x_dtype == DLP_F32 && y_dtype == DLP_F32)
    k_cols_scale<float, float><<<grid, kColsThreads, 0, s>>>(n, C, (const float *)X, ldx, scale, op, (float *)Y, ldy);
  else if (x_dtype == DLP_F32 && y_dtype == DLP_BF16 && op == 2)
    k_cols_scale<float, bf16><<<grid, kColsThreads, 0, s>>>(n, C, (const float *)X, ldx, scale, op, (bf16 *)Y, ldy);
  else
    return DLP_ERR_DTYPE;
  return check_launch();
}

int dlp_ground_update(int32_t n, const int32_t *parent, const uint8_t *vmask, uint8_t *umask, uint8_t *in_t,
                      int32_t *count, dlp_stream_t stream) {
  if (n < 0 || !parent || !vmask || !umask || !in_t || !count) return DLP_ERR_INVALID;
  if (n == 0) return DLP_OK;
  k_ground_update<<<ceil_div_i(n, 256), 256, 0, (cudaStream_t)stream>>>(n, parent, vmask, umask, in_t, count);
  return check_launch();
}

}  // extern "C"
