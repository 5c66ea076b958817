// Column-scaled vector updates of the refinement loop and the grounding update.
#include "common.cuh"
#include "gather.cuh"

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

// Labels (solvers.predict, dynlp/solvers.py:166-167): binary: F[r,0] > 0.5; otherwise the first
// column holding the row's maximum (numpy argmax). Rows outside the mask get -1. flag[r] = the label
// differs from the one labels[r] held on entry; labels[r] takes the new one.
template <typename T>
__global__ void k_predict(int32_t n, int32_t C, const T *__restrict__ F, int64_t ldf, int32_t binary,
                          const uint8_t *__restrict__ mask, int32_t *labels, uint8_t *flag) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  int32_t lab = -1;
  if (!mask || mask[r]) {
    const T *f = F + r * ldf;
    if (binary) {
      lab = f[0] > T(0.5) ? 1 : 0;
    } else {
      T best = f[0];
      lab = 0;
      for (int c = 1; c < C; ++c) {
        const T x = f[c];
        if (x > best) {
          best = x;
          lab = c;
        }
      }
    }
  }
  flag[r] = labels[r] != lab ? 1 : 0;
  labels[r] = lab;
}

// out_label[i] = labels[rows[i]] for i < *count.
__global__ void k_gather_labels(const int32_t *__restrict__ rows, const int32_t *__restrict__ count,
                                const int32_t *__restrict__ labels, int32_t *out_label, int32_t cap) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < cap && i < *count) out_label[i] = labels[rows[i]];
}

int compact_flags(const uint8_t *flag, int32_t n, int32_t *out, int32_t *count, void *ws, size_t ws_bytes,
                  cudaStream_t s);
size_t compact_ws_bytes(int32_t n);

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

extern "C++" {
// Class-sum elimination: the right-hand side of a correction without its last class column, and the
// update that adds the correction and sets the last class to one minus the others. One thread per row
// (K + 1 <= 16 values), sums in ascending column order in fp64.
// WHOLE (K = 8 with the rows aligned: R rows of 9 doubles at 16-byte boundaries with ld >= 10 even,
// E / D rows of 8 floats at 32-byte boundaries): each row in whole-row vector loads and stores.
template <bool WHOLE>
__global__ void k_class_sum_rhs(int32_t n, int32_t K, const double *__restrict__ R, int64_t ldr,
                                const double *__restrict__ scale, float *__restrict__ E, int64_t lde) {
  if constexpr (WHOLE) {
    double sc[9];
#pragma unroll
    for (int j = 0; j < 9; ++j) sc[j] = scale[j];
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
      double raw[5][2];
      const bool hi = load_row10d(R + r * ldr, raw);
      float e[2][4];
#pragma unroll
      for (int j = 0; j < 7; ++j) e[j / 4][j % 4] = (float)(row10_col(raw, hi, j) / sc[j]);
      e[1][3] = (float)(row10_col(raw, hi, 8) / sc[8]);
      store_row8(E + r * lde, e);
    }
    return;
  }
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
    const double *rr = R + r * ldr;
    float *er = E + r * lde;
    for (int j = 0; j < K - 1; ++j) er[j] = (float)(rr[j] / scale[j]);
    er[K - 1] = (float)(rr[K] / scale[K]);
  }
}

template <bool WHOLE>
__global__ void k_class_sum_update(int32_t n, int32_t K, const float *__restrict__ D, int64_t ldd,
                                   const double *__restrict__ scale, double *__restrict__ Z, int64_t ldz,
                                   const uint8_t *__restrict__ solved) {
  if constexpr (WHOLE) {
    double sc[9];
#pragma unroll
    for (int j = 0; j < 9; ++j) sc[j] = scale[j];
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
      double raw[5][2];
      const bool hi = load_row10d(Z + r * ldz, raw);
      float d[2][4];
      load_row8(D + r * ldd, d);
      double z[10];
      double sum = 0.0;
#pragma unroll
      for (int j = 0; j < 7; ++j) {
        z[j] = row10_col(raw, hi, j) + (double)d[j / 4][j % 4] * sc[j];
        sum += z[j];
      }
      z[8] = row10_col(raw, hi, 8) + (double)d[1][3] * sc[8];
      z[7] = (!solved || solved[r]) ? 1.0 - sum : 0.0;
      z[9] = 0.0;
      store_row10d<false>(Z + r * ldz, z);  // exactly the 9 values: the tenth slot is padding
    }
    return;
  }
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
    const float *dr = D + r * ldd;
    double *zr = Z + r * ldz;
    double sum = 0.0;
    for (int j = 0; j < K - 1; ++j) {
      const double z = zr[j] + (double)dr[j] * scale[j];
      zr[j] = z;
      sum += z;
    }
    zr[K] = zr[K] + (double)dr[K - 1] * scale[K];
    zr[K - 1] = (!solved || solved[r]) ? 1.0 - sum : 0.0;
  }
}

}  // extern "C++"

size_t dlp_predict_workspace_bytes(int32_t n) {
  return ((size_t)(n > 0 ? n : 1) + 255) / 256 * 256 + compact_ws_bytes(n);
}

int dlp_predict(int32_t n, int32_t C, const void *F, int64_t ldf, int dtype, int32_t binary, const uint8_t *mask,
                int32_t *labels, int32_t *changed, int32_t *changed_label, int32_t *n_changed, void *ws,
                size_t ws_bytes, dlp_stream_t stream) {
  if (n < 0 || C <= 0 || ldf < C || !n_changed || (n > 0 && (!F || !labels || !changed))) return DLP_ERR_INVALID;
  if (!ws || ws_bytes < dlp_predict_workspace_bytes(n)) return DLP_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 0) {
    DLP_CUDA(cudaMemsetAsync(n_changed, 0, sizeof(int32_t), s));
    return DLP_OK;
  }
  uint8_t *flag = (uint8_t *)ws;
  const size_t fb = ((size_t)n + 255) / 256 * 256;
  const int grid = ceil_div_i(n, 256);
  if (dtype == DLP_F64)
    k_predict<double><<<grid, 256, 0, s>>>(n, C, (const double *)F, ldf, binary, mask, labels, flag);
  else if (dtype == DLP_F32)
    k_predict<float><<<grid, 256, 0, s>>>(n, C, (const float *)F, ldf, binary, mask, labels, flag);
  else
    return DLP_ERR_DTYPE;
  DLP_TRY(check_launch());
  DLP_TRY(compact_flags(flag, n, changed, n_changed, (char *)ws + fb, ws_bytes - fb, s));
  if (changed_label) {
    k_gather_labels<<<grid, 256, 0, s>>>(changed, n_changed, labels, changed_label, n);
    DLP_TRY(check_launch());
  }
  return DLP_OK;
}

int dlp_ground_update(int32_t n, const int32_t *parent, const uint8_t *vmask, uint8_t *umask, uint8_t *in_t,
                      int32_t *count, dlp_stream_t stream) {
  if (n < 0 || !parent || !vmask || !umask || !in_t || !count) return DLP_ERR_INVALID;
  if (n == 0) return DLP_OK;
  k_ground_update<<<ceil_div_i(n, 256), 256, 0, (cudaStream_t)stream>>>(n, parent, vmask, umask, in_t, count);
  return check_launch();
}

int dlp_class_sum_rhs(int32_t n, int32_t K, const double *R, int64_t ldr, const double *scale, float *E,
                      int64_t lde, dlp_stream_t stream) {
  if (n < 0 || K < 2 || K > 256 || ldr < K + 1 || lde < K) return DLP_ERR_INVALID;
  if (n == 0) return DLP_OK;
  if (!R || !scale || !E) return DLP_ERR_INVALID;
  const int grid = (int)std::min<long long>(ceil_div_i((long long)n, 256LL), (long long)sm_count() * 8);
  const bool whole = K == 8 && (uintptr_t)R % 16 == 0 && ldr % 2 == 0 && ldr >= 10 && (uintptr_t)E % 32 == 0 &&
                     lde % 8 == 0;
  if (whole) k_class_sum_rhs<true><<<grid, 256, 0, (cudaStream_t)stream>>>(n, K, R, ldr, scale, E, lde);
  else k_class_sum_rhs<false><<<grid, 256, 0, (cudaStream_t)stream>>>(n, K, R, ldr, scale, E, lde);
  return check_launch();
}

int dlp_class_sum_update(int32_t n, int32_t K, const float *D, int64_t ldd, const double *scale, double *Z,
                         int64_t ldz, const uint8_t *solved, dlp_stream_t stream) {
  if (n < 0 || K < 2 || K > 256 || ldd < K || ldz < K + 1) return DLP_ERR_INVALID;
  if (n == 0) return DLP_OK;
  if (!D || !scale || !Z) return DLP_ERR_INVALID;
  const int grid = (int)std::min<long long>(ceil_div_i((long long)n, 256LL), (long long)sm_count() * 8);
  const bool whole = K == 8 && (uintptr_t)Z % 16 == 0 && ldz % 2 == 0 && ldz >= 10 && (uintptr_t)D % 32 == 0 &&
                     ldd % 8 == 0;
  if (whole) k_class_sum_update<true><<<grid, 256, 0, (cudaStream_t)stream>>>(n, K, D, ldd, scale, Z, ldz, solved);
  else k_class_sum_update<false><<<grid, 256, 0, (cudaStream_t)stream>>>(n, K, D, ldd, scale, Z, ldz, solved);
  return check_launch();
}

}  // extern "C"
