// Row kernels over the sparse operator: SpMM with fused epilogues, frontier Jacobi, push
// scatter, neighbour marking and the synchronous-push helpers.
//
// Lane layout (shared by the gather kernels). A group of G lanes (power of two <= 32) owns one
// output row. Inside the group, LV "vector lanes" split the k-wide row into 16-byte vectors
// (VW elements each, NV vectors per row; lane cl holds vectors cl, cl+LV, ...; VPL per lane) and
// ES = G/LV "edge slots" stride over the row's stored entries. LV = 1 is the reference's row map
// (dynlp/kernels.py:141-166), LV > 1 its class-parallel map (:240-266), here with 16-byte
// vector gathers of X when the leading dimension allows it.
#include <algorithm>
#include <atomic>

#include "gather.cuh"

namespace dlp {

namespace {
// per calling thread, as cudaGetLastError: a thread reads the code of its own failed call even while
// other threads (the serving loop's workers) call the library
thread_local cudaError_t g_last_cuda = cudaSuccess;
std::atomic<unsigned long long> g_launches{0};
std::atomic<const int32_t *> g_cancel{nullptr};
}

const int32_t *cancel_word() { return g_cancel.load(std::memory_order_acquire); }

void set_cuda_error(cudaError_t e) { g_last_cuda = e; }

void note_launches(unsigned long long k) { g_launches.fetch_add(k, std::memory_order_relaxed); }

int check_launch(int kernels) {
  g_launches.fetch_add((unsigned long long)kernels, std::memory_order_relaxed);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_cuda_error(e);
    return DLP_ERR_CUDA;
  }
  return DLP_OK;
}

int sm_count() {
  static const int cached = [] {  // initialised once, thread-safe
    int dev = 0, c = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev);
    return c > 0 ? c : 148;
  }();
  return cached;
}

// ------------------------------------------------------------------------------------------------
// SpMM + fused epilogue
// ------------------------------------------------------------------------------------------------
template <class T>
struct SpmmArgs {
  const int32_t *rbeg, *rend, *col;
  const typename T::TW *w;
  int32_t n_rows;
  const int32_t *rows;
  int32_t C;
  const typename T::TX *X;
  int64_t ldx;
  const typename T::TV *a;
  double alpha, b;
  const typename T::TV *rhs;
  int64_t ldr;
  double cr;
  typename T::TY *Y;
  int64_t ldy;
  int compact;
  int G, LV, NV;
  const typename T::TV *Xo;  // own-row values for the a-term (NULL: X itself)
  int64_t ldxo;
  // kRow10D epilogue: the own row and the RHS row are read whole (three loads) and the Y row is
  // written in three or four vector stores (exactly its C values) when their rows are 16-byte
  // aligned and hold 10 values
  int own10, rhs10, y10;
  // kRow12F epilogue: the own row is read whole (two loads) when its rows are 16-byte aligned and
  // hold 12 values, and the Y row is written in two or three vector stores (exactly its C values)
  // when its rows start on 16-byte boundaries
  int own12, y12;
};

// ROW as in gather_row. kRow12F runs with two rows in flight per lane (measured on B200 at n = 1M,
// degree 10, C = 9: 133 us against 137 us for per-vector loads with four in flight and 157 us for the
// two-load path with four).
template <class T, int VW, int VPL, int ROW = kRowVec>
__global__ void __launch_bounds__(kThreads) k_spmm(SpmmArgs<T> p) {
  using TA = typename T::TA;
  using TX = typename T::TX;
  const int lane = threadIdx.x & 31;
  const int G = p.G, LV = p.LV, NV = p.NV;
  const int gl = lane & (G - 1);
  const int cl = gl & (LV - 1);
  const int es = gl / LV;
  const int ES = G / LV;
  const int gpw = 32 / G;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long g0 = warp * gpw; g0 < p.n_rows; g0 += nwarps * gpw) {
    const long long gi = g0 + lane / G;
    const bool valid = gi < p.n_rows;
    const int r = valid ? (p.rows ? p.rows[gi] : (int)gi) : 0;
    const int beg = valid ? p.rbeg[r] : 0;
    const int end = valid ? p.rend[r] : 0;
    TA acc[VPL][VW];
    // gathered rows in flight per lane by row layout (measured at n = 1M, degree 10): four 10-double
    // rows (the fp64 residual 278 -> 267 us against two), two 12-float rows (three: 121 -> 133 us)
    gather_row<typename T::TW, TX, TA, VW, VPL,
               (ROW == kRow12F ? 2 : ROW == kRow16H ? 4 : ROW == kRow10D ? 4 : gather_batch_wide<TA, VW, VPL>()),
               ROW>(
        p.col, p.w, p.X, p.ldx, beg, end, es, ES, cl, LV, NV, G, acc);
    if constexpr (ROW == kRow10D) {
      if (valid && es == 0) {  // same arithmetic, in the same order, as the per-column epilogue below
        const long long orow = p.compact ? gi : (long long)r;
        const double av = p.a ? (double)p.alpha * (double)p.a[r] : 0.0;
        double yv[10];  // terms added one row at a time: each row read just before its use
#pragma unroll
        for (int c = 0; c < 10; ++c) yv[c] = (double)p.b * acc[c / 2][c % 2];
        if (p.a) {
          if (p.own10) {
            double xo[5][2];
            const bool hx = load_row10d(p.Xo ? p.Xo + (long long)r * p.ldxo : p.X + (long long)r * p.ldx, xo);
#pragma unroll
            for (int c = 0; c < 10; ++c) yv[c] = fmaa(av, row10_col(xo, hx, c), yv[c]);
          } else {
#pragma unroll
            for (int c = 0; c < 10; ++c)
              if (c < p.C)
                yv[c] = fmaa(av, p.Xo ? p.Xo[(long long)r * p.ldxo + c] : p.X[(long long)r * p.ldx + c], yv[c]);
          }
        }
        if (p.rhs) {
          if (p.rhs10) {
            double rh[5][2];
            const bool hr = load_row10d(p.rhs + (long long)r * p.ldr, rh);
#pragma unroll
            for (int c = 0; c < 10; ++c) yv[c] += (double)p.cr * row10_col(rh, hr, c);
          } else {
#pragma unroll
            for (int c = 0; c < 10; ++c)
              if (c < p.C) yv[c] += (double)p.cr * p.rhs[(long long)r * p.ldr + c];
          }
        }
        if (p.y10) {  // exactly the C = 9 or 10 columns: the caller's other columns stay untouched
          if (p.C == 10) store_row10d<true>(p.Y + orow * p.ldy, yv);
          else store_row10d<false>(p.Y + orow * p.ldy, yv);
        } else {
#pragma unroll
          for (int c = 0; c < 10; ++c)
            if (c < p.C) p.Y[orow * p.ldy + c] = yv[c];
        }
      }
      continue;
    }
    if constexpr (ROW == kRow8F) {
      if (valid && es == 0 && (p.own12 || p.y12)) {  // the per-column arithmetic below, 8-float rows
        const long long orow = p.compact ? gi : (long long)r;
        const float av = p.a ? (float)p.alpha * (float)p.a[r] : 0.f;
        float yv[2][4];
#pragma unroll
        for (int c = 0; c < 8; ++c) yv[c / 4][c % 4] = (float)p.b * acc[c / 4][c % 4];
        if (p.a) {
          if (p.own12) {
            float xo[2][4];
            load_row8(p.Xo ? (const float *)p.Xo + (long long)r * p.ldxo : (const float *)p.X + (long long)r * p.ldx,
                      xo);
#pragma unroll
            for (int c = 0; c < 8; ++c) yv[c / 4][c % 4] = fmaa(av, xo[c / 4][c % 4], yv[c / 4][c % 4]);
          } else {
#pragma unroll
            for (int c = 0; c < 8; ++c)
              if (c < p.C)
                yv[c / 4][c % 4] = fmaa(av, p.Xo ? (float)p.Xo[(long long)r * p.ldxo + c]
                                                 : (float)p.X[(long long)r * p.ldx + c], yv[c / 4][c % 4]);
          }
        }
        if (p.rhs) {
#pragma unroll
          for (int c = 0; c < 8; ++c)
            if (c < p.C) yv[c / 4][c % 4] += (float)p.cr * (float)p.rhs[(long long)r * p.ldr + c];
        }
        if (p.y12) {
          store_row8((float *)(p.Y + orow * p.ldy), yv);
        } else {
#pragma unroll
          for (int c = 0; c < 8; ++c)
            if (c < p.C) p.Y[orow * p.ldy + c] = yv[c / 4][c % 4];
        }
        continue;
      }
    }
    if constexpr (ROW == kRow12F || ROW == kRow16H) {
      if (valid && es == 0 && (p.own12 || p.y12)) {  // the per-column arithmetic below, whole rows
        const long long orow = p.compact ? gi : (long long)r;
        const float av = p.a ? (float)p.alpha * (float)p.a[r] : 0.f;
        float yv[12];
#pragma unroll
        for (int c = 0; c < 12; ++c) yv[c] = (float)p.b * acc[c / VW][c % VW];
        if (p.a) {
          if (p.own12) {
            float xo[3][4];
            const float *orow_x;  // the fp32 own row (the bf16 form reads it from Xo)
            if constexpr (ROW == kRow16H) orow_x = (const float *)p.Xo + (long long)r * p.ldxo;
            else orow_x = p.Xo ? (const float *)p.Xo + (long long)r * p.ldxo : (const float *)p.X + (long long)r * p.ldx;
            const bool hx = load_row12(orow_x, xo);
#pragma unroll
            for (int c = 0; c < 12; ++c) yv[c] = fmaa(av, row12_col(xo, hx, c), yv[c]);
          } else {
#pragma unroll
            for (int c = 0; c < 12; ++c)
              if (c < p.C)
                yv[c] = fmaa(av, p.Xo ? (float)p.Xo[(long long)r * p.ldxo + c] : cvt<float>(p.X[(long long)r * p.ldx + c]),
                             yv[c]);
          }
        }
        if (p.rhs) {
#pragma unroll
          for (int c = 0; c < 12; ++c)
            if (c < p.C) yv[c] += (float)p.cr * (float)p.rhs[(long long)r * p.ldr + c];
        }
        if (p.y12) {
          store_row_exact12((float *)(p.Y + orow * p.ldy), yv, p.C);
        } else {
#pragma unroll
          for (int c = 0; c < 12; ++c)
            if (c < p.C) p.Y[orow * p.ldy + c] = yv[c];
        }
        continue;
      }
    }
    if (valid && es == 0) {
      const long long orow = p.compact ? gi : (long long)r;
      const TA av = p.a ? (TA)p.alpha * cvt<TA>(p.a[r]) : TA(0);
#pragma unroll
      for (int k = 0; k < VPL; ++k) {
        const int vi = cl + k * LV;
        if (vi < NV) {
#pragma unroll
          for (int i = 0; i < VW; ++i) {
            const int c = vi * VW + i;
            if (c < p.C) {
              TA y = (TA)p.b * acc[k][i];
              if (p.a)
                y = fmaa(av, p.Xo ? cvt<TA>(p.Xo[(long long)r * p.ldxo + c]) : cvt<TA>(p.X[(long long)r * p.ldx + c]),
                         y);
              if (p.rhs) y += (TA)p.cr * cvt<TA>(p.rhs[(long long)r * p.ldr + c]);
              p.Y[orow * p.ldy + c] = cvt<typename T::TY>(y);
            }
          }
        }
      }
    }
  }
}

template <class T, int VW>
static int launch_spmm_vw(const SpmmArgs<T> &a, int VPL, dlp_stream_t s) {
  const int grid = grid_for(a.n_rows, a.G);
  constexpr bool kRow12 =
      VW == 4 && std::is_same<typename T::TX, float>::value && std::is_same<typename T::TA, float>::value;
  constexpr bool kRow10 =
      VW == 2 && std::is_same<typename T::TX, double>::value && std::is_same<typename T::TA, double>::value;
  constexpr bool kRow16 =
      VW == 8 && std::is_same<typename T::TX, bf16>::value && std::is_same<typename T::TA, float>::value;
  switch (VPL) {
    case 1: k_spmm<T, VW, 1><<<grid, kThreads, 0, (cudaStream_t)s>>>(a); break;
    case 2:
      // bf16 rows of 16 values held whole by one lane: one 256-bit load per gathered row
      if (kRow16 && a.LV == 1 && (uintptr_t)a.X % 32 == 0 && (a.ldx * 2) % 32 == 0) {
        k_spmm<T, VW, 2, (kRow16 ? kRow16H : kRowVec)><<<grid, kThreads, 0, (cudaStream_t)s>>>(a);
      } else if (kRow12 && a.LV == 1 && (uintptr_t)a.X % 32 == 0 && a.ldx % 8 == 0) {
        // fp32 rows of 8 values held whole by one lane: one 256-bit load per gathered row
        k_spmm<T, VW, 2, (kRow12 ? kRow8F : kRowVec)><<<grid, kThreads, 0, (cudaStream_t)s>>>(a);
      } else {
        k_spmm<T, VW, 2><<<grid, kThreads, 0, (cudaStream_t)s>>>(a);
      }
      break;
    case 3:
      if (kRow12 && a.LV == 1) {  // fp32 12-float rows held whole by one lane: two loads per row
        k_spmm<T, VW, 3, (kRow12 ? kRow12F : kRowVec)><<<grid, kThreads, 0, (cudaStream_t)s>>>(a);
      } else {
        k_spmm<T, VW, 3><<<grid, kThreads, 0, (cudaStream_t)s>>>(a);
      }
      break;
    case 4: k_spmm<T, VW, 4><<<grid, kThreads, 0, (cudaStream_t)s>>>(a); break;
    case 8: k_spmm<T, VW, 8><<<grid, kThreads, 0, (cudaStream_t)s>>>(a); break;
    case 5:  // fp64 10-double rows held whole by one lane (run_spmm): three loads per row
      if constexpr (kRow10) {
        k_spmm<T, VW, 5, kRow10D><<<grid, kThreads, 0, (cudaStream_t)s>>>(a);
        break;
      }
      return DLP_ERR_INVALID;
    default: return DLP_ERR_INVALID;
  }
  return check_launch();
}

template <class T>
static int run_spmm(const int32_t *rbeg, const int32_t *rend, const int32_t *col, const void *w, int32_t n_rows,
                    const int32_t *rows, int32_t C, const void *X, int64_t ldx, const void *a, double alpha,
                    double b, const void *RHS, int64_t ldr, double cr, void *Y, int64_t ldy, int compact,
                    int32_t group, double avg_deg, dlp_stream_t s, const void *Xo = nullptr, int64_t ldxo = 0) {
  Layout L;
  DLP_TRY(choose_layout(C, sizeof(typename T::TX), X, ldx, group, avg_deg, &L));
  if (std::is_same<typename T::TX, double>::value && std::is_same<typename T::TA, double>::value && L.VW == 2 &&
      L.NV == 5) {
    // fp64 rows of five 16-byte vectors (9-10 columns): one lane holds the whole row and reads it in
    // three loads (load_row10d); the edge slots per row stay as chosen
    L.G /= L.LV;
    L.LV = 1;
    L.VPL = 5;
  }
  SpmmArgs<T> p{rbeg, rend, col, (const typename T::TW *)w, n_rows, rows, C, (const typename T::TX *)X, ldx,
                (const typename T::TV *)a, alpha, b, (const typename T::TV *)RHS, ldr, cr,
                (typename T::TY *)Y, ldy, compact, L.G, L.LV, L.NV, (const typename T::TV *)Xo, ldxo, 0, 0, 0,
                0, 0};
  const bool f32_12 = std::is_same<typename T::TX, float>::value && std::is_same<typename T::TA, float>::value &&
                      L.VW == 4 && L.VPL == 3 && L.LV == 1 && C >= 9;
  const bool bf16_16 = std::is_same<typename T::TX, bf16>::value && std::is_same<typename T::TA, float>::value &&
                       L.VW == 8 && L.VPL == 2 && L.LV == 1 && C >= 9 && C <= 12;
  const bool f32_8 = std::is_same<typename T::TX, float>::value && std::is_same<typename T::TA, float>::value &&
                     std::is_same<typename T::TY, float>::value && std::is_same<typename T::TV, float>::value &&
                     L.VW == 4 && L.VPL == 2 && L.LV == 1 && (uintptr_t)X % 32 == 0 && ldx % 8 == 0;
  if (f32_8) {  // the kRow8F layout (launch_spmm_vw): whole-row epilogue where the rows allow it
    auto rows8 = [](const void *q, int64_t ldq) { return q && (uintptr_t)q % 32 == 0 && ldq % 8 == 0; };
    p.own12 = Xo ? rows8(Xo, ldxo) : 1;
    p.y12 = C == 8 && rows8(Y, ldy);
  }
  if (std::is_same<typename T::TY, float>::value && std::is_same<typename T::TV, float>::value && (f32_12 || bf16_16)) {
    // the kRow12F / kRow16H layouts (launch_spmm_vw): whole-row epilogue (fp32 own row and output)
    // where the rows allow it
    auto rows12 = [](const void *q, int64_t ldq) { return q && (uintptr_t)q % 16 == 0 && ldq % 4 == 0 && ldq >= 12; };
    p.own12 = Xo ? rows12(Xo, ldxo) : (f32_12 && rows12(X, ldx));
    p.y12 = Y && (uintptr_t)Y % 16 == 0 && ldy % 4 == 0;
  }
  if (L.VPL == 5 && L.LV == 1) {  // the kRow10D layout chosen above: whole-row epilogue where aligned
    auto rows10 = [](const void *q, int64_t ldq) { return q && (uintptr_t)q % 16 == 0 && ldq % 2 == 0 && ldq >= 10; };
    p.own10 = Xo ? rows10(Xo, ldxo) : 1;
    p.rhs10 = rows10(RHS, ldr);
    p.y10 = rows10(Y, ldy);
  }
  constexpr int VWV = 16 / sizeof(typename T::TX);
  if (L.VW == 1) return launch_spmm_vw<T, 1>(p, L.VPL, s);
  return launch_spmm_vw<T, VWV>(p, L.VPL, s);
}

// ------------------------------------------------------------------------------------------------
// Frontier Jacobi (dynlp/kernels.py:31-103, :186-220)
// ------------------------------------------------------------------------------------------------
template <class T>
struct JacArgs {
  const int32_t *rbeg, *rend, *col;
  const typename T::TW *w;
  const int32_t *frontier;
  int32_t nf, C;
  const typename T::TX *X;
  int64_t ldx;
  const typename T::TX *rhs;
  int64_t ldr;
  const typename T::TX *diag;
  double delta;
  typename T::TX *Y;
  int64_t ldy;
  uint8_t *changed;
  int32_t *out_list, *out_count;
  int G, LV, NV;
};

template <class T, int VW, int VPL>
__global__ void __launch_bounds__(kThreads) k_jacobi(JacArgs<T> p) {
  using TA = typename T::TA;
  using TX = typename T::TX;
  const int lane = threadIdx.x & 31;
  const int G = p.G, LV = p.LV, NV = p.NV;
  const int gl = lane & (G - 1);
  const int cl = gl & (LV - 1);
  const int es = gl / LV;
  const int ES = G / LV;
  const int gpw = 32 / G;
  const int gbase = lane & ~(G - 1);
  const unsigned gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << gbase);
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long g0 = warp * gpw; g0 < p.nf; g0 += nwarps * gpw) {
    const long long gi = g0 + lane / G;
    const bool valid = gi < p.nf;
    const int r = valid ? p.frontier[gi] : 0;
    const int beg = valid ? p.rbeg[r] : 0;
    const int end = valid ? p.rend[r] : 0;
    TA acc[VPL][VW];
    gather_row<typename T::TW, TX, TA, VW, VPL>(p.col, p.w, p.X, p.ldx, beg, end, es, ES, cl, LV, NV, G, acc);
    bool ch = false;
    if (valid && es == 0) {
      const TA inv = TA(1) / cvt<TA>(p.diag[r]);
#pragma unroll
      for (int k = 0; k < VPL; ++k) {
        const int vi = cl + k * LV;
        if (vi < NV) {
#pragma unroll
          for (int i = 0; i < VW; ++i) {
            const int c = vi * VW + i;
            if (c < p.C) {
              const TA yv = (cvt<TA>(p.rhs[(long long)r * p.ldr + c]) + acc[k][i]) * inv;
              p.Y[gi * p.ldy + c] = cvt<TX>(yv);
              ch |= fabs(yv - cvt<TA>(p.X[(long long)r * p.ldx + c])) > (TA)p.delta;
            }
          }
        }
      }
    }
    const unsigned bal = __ballot_sync(0xffffffffu, ch);
    const bool any = (bal & gmask) != 0;
    if (valid && gl == 0 && p.changed) p.changed[gi] = any ? 1 : 0;
    if (p.out_list) warp_append(valid && gl == 0 && any, r, p.out_list, p.out_count);
  }
}

template <class T, int VW>
static int launch_jac_vw(const JacArgs<T> &a, int VPL, dlp_stream_t s) {
  const int grid = grid_for(a.nf, a.G);
  switch (VPL) {
    case 1: k_jacobi<T, VW, 1><<<grid, kThreads, 0, (cudaStream_t)s>>>(a); break;
    case 2: k_jacobi<T, VW, 2><<<grid, kThreads, 0, (cudaStream_t)s>>>(a); break;
    case 3: k_jacobi<T, VW, 3><<<grid, kThreads, 0, (cudaStream_t)s>>>(a); break;
    case 4: k_jacobi<T, VW, 4><<<grid, kThreads, 0, (cudaStream_t)s>>>(a); break;
    case 8: k_jacobi<T, VW, 8><<<grid, kThreads, 0, (cudaStream_t)s>>>(a); break;
    default: return DLP_ERR_INVALID;
  }
  return check_launch();
}

template <class T>
static int run_jacobi(const int32_t *rbeg, const int32_t *rend, const int32_t *col, const void *w,
                      const int32_t *frontier, int32_t nf, int32_t C, const void *X, int64_t ldx, const void *rhs,
                      int64_t ldr, const void *diag, double delta, void *Y, int64_t ldy, uint8_t *changed,
                      int32_t *out_list, int32_t *out_count, int32_t group, double avg_deg, dlp_stream_t s) {
  Layout L;
  DLP_TRY(choose_layout(C, sizeof(typename T::TX), X, ldx, group, avg_deg, &L));
  JacArgs<T> p{rbeg, rend, col, (const typename T::TW *)w, frontier, nf, C, (const typename T::TX *)X, ldx,
               (const typename T::TX *)rhs, ldr, (const typename T::TX *)diag, delta, (typename T::TX *)Y, ldy,
               changed, out_list, out_count, L.G, L.LV, L.NV};
  constexpr int VWV = 16 / sizeof(typename T::TX);
  if (L.VW == 1) return launch_jac_vw<T, 1>(p, L.VPL, s);
  return launch_jac_vw<T, VWV>(p, L.VPL, s);
}

// ------------------------------------------------------------------------------------------------
// Push scatter (dynlp/kernels.py:105-126, :222-238)
// ------------------------------------------------------------------------------------------------
template <typename TW, typename TR>
__global__ void __launch_bounds__(kThreads)
    k_push_scatter(const int32_t *__restrict__ rbeg, const int32_t *__restrict__ rend,
                   const int32_t *__restrict__ col, const TW *__restrict__ w, const int32_t *__restrict__ frontier,
                   int32_t nf, int32_t C, const TR *__restrict__ D, int64_t ldd, TR *R, int64_t ldr,
                   uint8_t *mark, int G, int LV) {
  const int lane = threadIdx.x & 31;
  const int gl = lane & (G - 1);
  const int cl = gl & (LV - 1);
  const int es = gl / LV;
  const int ES = G / LV;
  const int gpw = 32 / G;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long g0 = warp * gpw; g0 < nf; g0 += nwarps * gpw) {
    const long long gi = g0 + lane / G;
    if (gi >= nf) continue;
    const int r = frontier[gi];
    const int beg = rbeg[r], end = rend[r];
    for (int j = beg + es; j < end; j += ES) {
      const long long v = col[j];
      const TR wv = cvt<TR>(w[j]);
      for (int c = cl; c < C; c += LV) atomic_add(&R[v * ldr + c], wv * D[gi * ldd + c]);
      if (cl == 0 && mark) mark[v] = 1;
    }
  }
}

__global__ void k_mark_neighbors(const int32_t *__restrict__ rbeg, const int32_t *__restrict__ rend,
                                 const int32_t *__restrict__ col, const int32_t *__restrict__ rows, int32_t nr,
                                 uint8_t *mark) {
  // 8 lanes per row
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long g = t >> 3;
  const int l = (int)(t & 7);
  if (g >= nr) return;
  const int r = rows[g];
  for (int j = rbeg[r] + l; j < rend[r]; j += 8) mark[col[j]] = 1;
}

// ------------------------------------------------------------------------------------------------
// synchronous push helpers (dynlp/solvers.py:100-125)
// ------------------------------------------------------------------------------------------------
template <typename T>
__global__ void k_push_take(const int32_t *__restrict__ cand, int32_t nc, int32_t C, T *Z, int64_t ldz, T *R,
                            int64_t ldr, const T *__restrict__ diag, T *D, int64_t ldd, uint8_t *mark) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nc * C) return;
  const long long g = t / C;
  const int c = (int)(t % C);
  const long long r = cand[g];
  const T d = R[r * ldr + c] / diag[r];
  D[g * ldd + c] = d;
  Z[r * ldz + c] += d;
  R[r * ldr + c] = T(0);
  if (c == 0 && mark) mark[r] = 1;
}

template <typename T>
__global__ void k_violating(const int32_t *__restrict__ idx, int32_t n, int32_t C, const T *__restrict__ R,
                            int64_t ldr, const T *__restrict__ diag, const double *__restrict__ eps, uint8_t *flag,
                            uint8_t *clear_mark) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  const long long r = idx ? idx[g] : g;
  const T dv = diag[r];
  bool viol = false;
  for (int c = 0; c < C; ++c) viol |= fabs(R[r * ldr + c]) > (T)eps[c] * dv;
  flag[g] = viol ? 1 : 0;
  if (clear_mark) clear_mark[r] = 0;
}

}  // namespace dlp

using namespace dlp;

extern "C" {

int dlp_version(void) { return 1; }

const char *dlp_status_string(int st) {
  switch (st) {
    case DLP_OK: return "ok";
    case DLP_ERR_INVALID: return "invalid argument";
    case DLP_ERR_DTYPE: return "unsupported precision combination";
    case DLP_ERR_CUDA: return "CUDA runtime error";
    case DLP_ERR_CAP: return "iteration cap reached";
    case DLP_ERR_CANCELLED: return "cancelled";
    case DLP_ERR_WORKSPACE: return "workspace too small";
    case DLP_ERR_OVERFLOW: return "row capacity exceeded";
    case DLP_ERR_DEVICE: return "device-side check failed";
    case DLP_ERR_SCRATCH_LIMIT: return "size exceeds the fixed scratch of an allocation-free entry point";
    default: return "unknown status";
  }
}

int dlp_last_cuda_error(void) { return (int)g_last_cuda; }

unsigned long long dlp_launch_count(void) { return g_launches.load(); }

int dlp_sm_count(void) { return sm_count(); }

int dlp_set_cancel_word(const int32_t *word) {
  g_cancel.store(word, std::memory_order_release);
  return DLP_OK;
}

int dlp_spmm(const int32_t *rbeg, const int32_t *rend, const int32_t *col, const void *w, int w_dtype,
             int32_t n_rows, const int32_t *rows, int32_t C, const void *X, int64_t ldx, int x_dtype,
             const void *a, double alpha, double b, const void *RHS, int64_t ldr, double cr, void *Y,
             int64_t ldy, int y_dtype, int compact_out, int32_t group, double avg_deg, dlp_stream_t stream) {
  if (n_rows < 0 || C <= 0 || ldx < C || ldy < C || (RHS && ldr < C)) return DLP_ERR_INVALID;
  if (n_rows == 0) return DLP_OK;
  if (!rbeg || !rend || !X || !Y || !w || !col) return DLP_ERR_INVALID;
#define DLP_SPMM_ARGS rbeg, rend, col, w, n_rows, rows, C, X, ldx, a, alpha, b, RHS, ldr, cr, Y, ldy, compact_out, \
                      group, avg_deg, stream
  if (w_dtype == DLP_F32 && x_dtype == DLP_F32 && y_dtype == DLP_F32) return run_spmm<T_F32>(DLP_SPMM_ARGS);
  if (w_dtype == DLP_F64 && x_dtype == DLP_F64 && y_dtype == DLP_F64) return run_spmm<T_F64>(DLP_SPMM_ARGS);
  if (w_dtype == DLP_F32 && x_dtype == DLP_F64 && y_dtype == DLP_F64) return run_spmm<T_W32X64>(DLP_SPMM_ARGS);
  if (w_dtype == DLP_BF16 && x_dtype == DLP_BF16 && y_dtype == DLP_F32) return run_spmm<T_BF16F>(DLP_SPMM_ARGS);
  if (w_dtype == DLP_BF16 && x_dtype == DLP_BF16 && y_dtype == DLP_BF16) return run_spmm<T_BF16B>(DLP_SPMM_ARGS);
#undef DLP_SPMM_ARGS
  return DLP_ERR_DTYPE;
}

int dlp_spmm_lowp(const int32_t *rbeg, const int32_t *rend, const int32_t *col, const void *w_lo, int32_t n_rows,
                  int32_t C, const void *X_lo, int64_t ld_lo, const void *X_own, int64_t ld_own, const void *a,
                  double alpha, double b, void *Y, int64_t ldy, int32_t group, double avg_deg, dlp_stream_t stream) {
  if (n_rows < 0 || C <= 0 || ld_lo < C || ldy < C || (X_own && ld_own < C)) return DLP_ERR_INVALID;
  if (n_rows == 0) return DLP_OK;
  if (!rbeg || !rend || !col || !w_lo || !X_lo || !Y) return DLP_ERR_INVALID;
  return run_spmm<T_BF16F>(rbeg, rend, col, w_lo, n_rows, nullptr, C, X_lo, ld_lo, a, alpha, b, nullptr, C, 0.0, Y,
                           ldy, 0, group, avg_deg, stream, X_own, ld_own);
}

int dlp_frontier_jacobi(const int32_t *rbeg, const int32_t *rend, const int32_t *col, const void *w,
                        int w_dtype, const int32_t *frontier, int32_t nf, int32_t C, const void *X,
                        int64_t ldx, const void *rhs, int64_t ldr, const void *diag, double delta, void *Y,
                        int64_t ldy, int dtype, uint8_t *changed, int32_t *out_list, int32_t *out_count,
                        int32_t group, double avg_deg, dlp_stream_t stream) {
  if (nf < 0 || C <= 0 || ldx < C || ldy < C || ldr < C) return DLP_ERR_INVALID;
  if (nf == 0) return DLP_OK;
  if (!rbeg || !rend || !col || !w || !frontier || !X || !rhs || !diag || !Y) return DLP_ERR_INVALID;
  if (out_list && !out_count) return DLP_ERR_INVALID;
#define DLP_JAC_ARGS rbeg, rend, col, w, frontier, nf, C, X, ldx, rhs, ldr, diag, delta, Y, ldy, changed, out_list, \
                     out_count, group, avg_deg, stream
  if (w_dtype == DLP_F32 && dtype == DLP_F32) return run_jacobi<T_F32>(DLP_JAC_ARGS);
  if (w_dtype == DLP_F64 && dtype == DLP_F64) return run_jacobi<T_F64>(DLP_JAC_ARGS);
  if (w_dtype == DLP_F32 && dtype == DLP_F64) return run_jacobi<T_W32X64>(DLP_JAC_ARGS);
#undef DLP_JAC_ARGS
  return DLP_ERR_DTYPE;
}

int dlp_push_scatter(const int32_t *rbeg, const int32_t *rend, const int32_t *col, const void *w, int w_dtype,
                     const int32_t *frontier, int32_t nf, int32_t C, const void *D, int64_t ldd, void *R,
                     int64_t ldr, int dtype, uint8_t *mark, int32_t group, double avg_deg,
                     dlp_stream_t stream) {
  if (nf < 0 || C <= 0 || ldd < C || ldr < C) return DLP_ERR_INVALID;
  if (nf == 0) return DLP_OK;
  if (!rbeg || !rend || !col || !w || !frontier || !D || !R) return DLP_ERR_INVALID;
  int LV = C <= 4 ? 1 : std::min(32, next_pow2((C + 3) / 4));
  int es = group > 0 ? std::min(group, 32) : auto_group(avg_deg);
  int p = 1;
  while (p * 2 <= es) p *= 2;
  es = std::max(1, std::min(p, 32 / LV));
  const int G = LV * es;
  const int grid = grid_for(nf, G);
  cudaStream_t s = (cudaStream_t)stream;
  if (w_dtype == DLP_F32 && dtype == DLP_F32)
    k_push_scatter<float, float><<<grid, kThreads, 0, s>>>(rbeg, rend, col, (const float *)w, frontier, nf, C,
                                                           (const float *)D, ldd, (float *)R, ldr, mark, G, LV);
  else if (w_dtype == DLP_F64 && dtype == DLP_F64)
    k_push_scatter<double, double><<<grid, kThreads, 0, s>>>(rbeg, rend, col, (const double *)w, frontier, nf, C,
                                                             (const double *)D, ldd, (double *)R, ldr, mark, G, LV);
  else if (w_dtype == DLP_F32 && dtype == DLP_F64)
    k_push_scatter<float, double><<<grid, kThreads, 0, s>>>(rbeg, rend, col, (const float *)w, frontier, nf, C,
                                                            (const double *)D, ldd, (double *)R, ldr, mark, G, LV);
  else
    return DLP_ERR_DTYPE;
  return check_launch();
}

int dlp_mark_neighbors(const int32_t *rbeg, const int32_t *rend, const int32_t *col, const int32_t *rows,
                       int32_t nr, uint8_t *mark, dlp_stream_t stream) {
  if (nr < 0) return DLP_ERR_INVALID;
  if (nr == 0) return DLP_OK;
  if (!rbeg || !rend || !col || !rows || !mark) return DLP_ERR_INVALID;
  const long long threads = (long long)nr * 8;
  k_mark_neighbors<<<ceil_div_i(threads, kThreads), kThreads, 0, (cudaStream_t)stream>>>(rbeg, rend, col, rows, nr,
                                                                                          mark);
  return check_launch();
}

int dlp_push_take(const int32_t *cand, int32_t nc, int32_t C, void *Z, int64_t ldz, void *R, int64_t ldr,
                  const void *diag, void *D, int64_t ldd, int dtype, uint8_t *mark, dlp_stream_t stream) {
  if (nc < 0 || C <= 0 || ldz < C || ldr < C || ldd < C) return DLP_ERR_INVALID;
  if (nc == 0) return DLP_OK;
  if (!cand || !Z || !R || !diag || !D) return DLP_ERR_INVALID;
  const long long t = (long long)nc * C;
  const int grid = ceil_div_i(t, kThreads);
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == DLP_F32)
    k_push_take<float><<<grid, kThreads, 0, s>>>(cand, nc, C, (float *)Z, ldz, (float *)R, ldr, (const float *)diag,
                                                 (float *)D, ldd, mark);
  else if (dtype == DLP_F64)
    k_push_take<double><<<grid, kThreads, 0, s>>>(cand, nc, C, (double *)Z, ldz, (double *)R, ldr,
                                                  (const double *)diag, (double *)D, ldd, mark);
  else
    return DLP_ERR_DTYPE;
  return check_launch();
}

int dlp_violating(const int32_t *idx, int32_t n, int32_t C, const void *R, int64_t ldr, const void *diag,
                  int dtype, const double *eps, uint8_t *flag, uint8_t *clear_mark, dlp_stream_t stream) {
  if (n < 0 || C <= 0 || ldr < C) return DLP_ERR_INVALID;
  if (n == 0) return DLP_OK;
  if (!R || !diag || !eps || !flag) return DLP_ERR_INVALID;
  const int grid = ceil_div_i(n, kThreads);
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == DLP_F32)
    k_violating<float><<<grid, kThreads, 0, s>>>(idx, n, C, (const float *)R, ldr, (const float *)diag, eps, flag,
                                                 clear_mark);
  else if (dtype == DLP_F64)
    k_violating<double><<<grid, kThreads, 0, s>>>(idx, n, C, (const double *)R, ldr, (const double *)diag, eps,
                                                  flag, clear_mark);
  else
    return DLP_ERR_DTYPE;
  return check_launch();
}

}  // extern "C"
