// Row-gather machinery shared by the SpMM-shaped kernels (rowops.cu, pcg.cu).
#pragma once

#include <algorithm>
#include <type_traits>

#include "common.cuh"

namespace dlp {

template <typename TW_, typename TX_, typename TY_, typename TV_, typename TA_>
struct Types {
  using TW = TW_;
  using TX = TX_;
  using TY = TY_;
  using TV = TV_;
  using TA = TA_;
};
using T_F32 = Types<float, float, float, float, float>;
using T_F64 = Types<double, double, double, double, double>;
using T_W32X64 = Types<float, double, double, double, double>;
using T_BF16F = Types<bf16, bf16, float, float, float>;
using T_BF16B = Types<bf16, bf16, bf16, float, float>;

__device__ __forceinline__ float fmaa(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fmaa(double a, double b, double c) { return fma(a, b, c); }

struct Layout {
  int G, LV, NV, VW, VPL;
};

constexpr int kThreads = 256;

// Host: pick the lane layout for a k-wide gather of `elem`-byte values at X with leading dim ld.
static inline int choose_layout(int C, size_t elem, const void *X, int64_t ld, int group, double avg_deg, Layout *L) {
  const int vwv = (int)(16 / elem);
  const bool vec = C > 1 && ((uintptr_t)X % 16 == 0) && ((ld * (int64_t)elem) % 16 == 0) &&
                   ld >= (int64_t)((C + vwv - 1) / vwv) * vwv;
  L->VW = vec ? vwv : 1;
  L->NV = (C + L->VW - 1) / L->VW;
  L->LV = L->NV <= 4 ? 1 : std::min(32, next_pow2((L->NV + 3) / 4));
  int vpl = (L->NV + L->LV - 1) / L->LV;
  if (vpl > 4) vpl = vpl <= 8 ? 8 : -1;
  if (vpl < 0) return DLP_ERR_INVALID;
  L->VPL = vpl;
  // edge slots: about a quarter of the mean degree (measured best on B200 for deg 10..32: each lane
  // keeps several independent gathers in flight instead of idling on short rows)
  int es = group > 0 ? std::min(group, 32) : std::max(1, (int)(avg_deg / 4.0));
  int p = 1;
  while (p * 2 <= es) p *= 2;  // power of two
  es = std::min(p, 32 / L->LV);
  if (es < 1) es = 1;
  L->G = L->LV * es;
  return DLP_OK;
}

static inline int grid_for(long long groups, int G) {
  long long threads = groups * G;
  long long blocks = (threads + kThreads - 1) / kThreads;
  long long cap = (long long)sm_count() * 8;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return (int)blocks;
}


// Entries per batch of a gather_row lane on the per-vector path, by the registers the batch holds
// (VPL x VW values of TA per entry). Measured on B200 (ER n = 1M, degree 10, 9 fp32 columns): the
// plain SpMM is fastest with four gathers in flight (about 48 registers of batch, one resident
// block fewer per SM); the PCG apply, capped at 64 registers for a fourth resident block, with two.
// The whole-row paths (kRow12F, kRow10D below) pass their own batch: two rows in flight for the
// fp32 SpMM and PCG apply, the wide batch for fp64.
template <typename TA, int VW, int VPL>
constexpr int gather_batch_wide() {
  return VPL * VW * (int)(sizeof(TA) / 4) <= 12 ? 4 : VPL * VW * (int)(sizeof(TA) / 4) <= 24 ? 2 : 1;
}
template <typename TA, int VW, int VPL>
constexpr int gather_batch_lean() {
  return VPL * VW * (int)(sizeof(TA) / 4) <= 8 ? 4 : VPL * VW * (int)(sizeof(TA) / 4) <= 16 ? 2 : 1;
}

// One 12-float row (three 16-byte vectors) at a 16-byte aligned address, in two loads: the row's
// 32-byte aligned half goes through one 256-bit load (sm_100 ld.global.v8) and the other 16 bytes
// through one 128-bit load. Same 48 bytes and the same two 32-byte sectors as three 128-bit loads,
// with one load instruction fewer per gathered row. The values stay in load order: raw[0..1] hold
// the 256-bit half and raw[2] the 128-bit part; with hi (the row starts 16 bytes into a 32-byte
// sector) columns 0-3 are raw[2], 4-11 raw[0..1], else columns 0-7 are raw[0..1], 8-11 raw[2].
// Both loads carry an L2 evict-last policy: the gathered block (P in the PCG) is then the last thing
// the streamed CSR (evict-first loads) pushes out of L2. Measured on B200 (n = 1M, degree 10, C = 9,
// kernel harness): the direction sweep that reads P next drops from 41.1 to 37.0 us, the apply is
// unchanged, and every iterate is bit-identical (a cache policy changes no value).
__device__ __forceinline__ uint64_t l2_evict_last() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
// The whole-row loads of the gathers (one lane reads a neighbour's entire row) bypass L1 allocation
// (L1::no_allocate): such a row is rarely read again from L1 (random neighbours), and not allocating
// them left L1 to the accesses that reuse it: the 8-column SpMM at n = 1M, degree 10 went from 86.7
// to 80.2 us, the PCG iteration on it from 132 to 124 us. The 16-byte vector gathers of wide rows
// (several lanes per row) keep allocating: without it the k = 32 serving stream measured slower
// (622.6 k against 637.1 k edge-updates/s, update p50 215 against 188 ms).
__device__ __forceinline__ bool load_row12(const float *__restrict__ xr, float (&raw)[3][4]) {
  const bool hi = ((uintptr_t)xr & 16u) != 0;
  const float *p8 = xr + (hi ? 4 : 0);
  const float *p4 = xr + (hi ? 0 : 8);
  const uint64_t pol = l2_evict_last();
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8], %9;"
      : "=f"(raw[0][0]), "=f"(raw[0][1]), "=f"(raw[0][2]), "=f"(raw[0][3]), "=f"(raw[1][0]), "=f"(raw[1][1]),
        "=f"(raw[1][2]), "=f"(raw[1][3])
      : "l"(p8), "l"(pol));
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
      : "=f"(raw[2][0]), "=f"(raw[2][1]), "=f"(raw[2][2]), "=f"(raw[2][3])
      : "l"(p4), "l"(pol));
  return hi;
}

// fp64 counterpart: one 10-double row (five 16-byte vectors) at a 16-byte aligned address in three
// loads (two 256-bit, one 128-bit) instead of five 128-bit ones; the same 80 bytes and sectors. raw in
// load order (flat f = 2 k + i): f 0-3 and 4-7 the two 256-bit loads, f 8-9 the 128-bit one. Without
// hi the row's columns are f 0-9 in order; with hi (the row starts 16 bytes into a 32-byte sector)
// columns 0-1 are f 8-9 and columns 2-9 are f 0-7.
__device__ __forceinline__ bool load_row10d(const double *__restrict__ xr, double (&raw)[5][2]) {
  const bool hi = ((uintptr_t)xr & 16u) != 0;
  const double *pa = xr + (hi ? 2 : 0);
  const double *pb = xr + (hi ? 6 : 4);
  const double *pg = xr + (hi ? 0 : 8);
  asm("ld.global.nc.L1::no_allocate.v4.f64 {%0, %1, %2, %3}, [%4];"
      : "=d"(raw[0][0]), "=d"(raw[0][1]), "=d"(raw[1][0]), "=d"(raw[1][1])
      : "l"(pa));
  asm("ld.global.nc.L1::no_allocate.v4.f64 {%0, %1, %2, %3}, [%4];"
      : "=d"(raw[2][0]), "=d"(raw[2][1]), "=d"(raw[3][0]), "=d"(raw[3][1])
      : "l"(pb));
  asm("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(raw[4][0]), "=d"(raw[4][1]) : "l"(pg));
  return hi;
}

// An fp32 row of 8 values at a 32-byte aligned address in one 256-bit load (L2 evict-last as in
// load_row12), and its store counterpart.
__device__ __forceinline__ void load_row8(const float *__restrict__ xr, float (&raw)[2][4]) {
  const uint64_t pol = l2_evict_last();
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8], %9;"
      : "=f"(raw[0][0]), "=f"(raw[0][1]), "=f"(raw[0][2]), "=f"(raw[0][3]), "=f"(raw[1][0]), "=f"(raw[1][1]),
        "=f"(raw[1][2]), "=f"(raw[1][3])
      : "l"(xr), "l"(pol));
}
__device__ __forceinline__ void store_row8(float *yr, const float (&v)[2][4]) {
  asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(yr), "f"(v[0][0]), "f"(v[0][1]),
               "f"(v[0][2]), "f"(v[0][3]), "f"(v[1][0]), "f"(v[1][1]), "f"(v[1][2]), "f"(v[1][3])
               : "memory");
}

// A bf16 row of 16 values (32 bytes, 32-byte aligned) in one 256-bit load, kept packed: word j
// holds columns 2j (low half) and 2j + 1 (high half). L2 evict-last as in load_row12.
__device__ __forceinline__ void load_row16h(const void *__restrict__ xr, uint32_t (&q)[8]) {
  const uint64_t pol = l2_evict_last();
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8], %9;"
      : "=r"(q[0]), "=r"(q[1]), "=r"(q[2]), "=r"(q[3]), "=r"(q[4]), "=r"(q[5]), "=r"(q[6]), "=r"(q[7])
      : "l"(xr), "l"(pol));
}

// Column c (0-9) of a row read by load_row10d.
__device__ __forceinline__ double row10_col(const double (&raw)[5][2], bool hi, int c) {
  const int fh = c < 2 ? 8 + c : c - 2;  // c is a compile-time index at every (unrolled) call
  return hi ? raw[fh / 2][fh % 2] : raw[c / 2][c % 2];
}

// Store counterpart of load_row10d: the values v of a row of 16-byte aligned address yr, exactly its
// first 10 (FULL) or 9 doubles, nothing beyond. 10: two 256-bit stores and one 128-bit store. 9
// (where the tenth slot may belong to the caller): one 256-bit, two 128-bit and one 64-bit store.
template <bool FULL>
__device__ __forceinline__ void store_row10d(double *yr, const double (&v)[10]) {
  const bool hi = ((uintptr_t)yr & 16u) != 0;
  double A[4];  // selects between fixed indices keep v in registers
#pragma unroll
  for (int k = 0; k < 4; ++k) A[k] = hi ? v[2 + k] : v[k];
  double *pa = yr + (hi ? 2 : 0);
  asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(pa), "d"(A[0]), "d"(A[1]), "d"(A[2]), "d"(A[3])
               : "memory");
  if constexpr (FULL) {  // hi: 0-1, 2-5, 6-9   else: 0-3, 4-7, 8-9
    double B[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) B[k] = hi ? v[6 + k] : v[4 + k];
    double *pb = yr + (hi ? 6 : 4);
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(pb), "d"(B[0]), "d"(B[1]), "d"(B[2]), "d"(B[3])
                 : "memory");
    *reinterpret_cast<double2 *>(yr + (hi ? 0 : 8)) = make_double2(hi ? v[0] : v[8], hi ? v[1] : v[9]);
  } else {  // hi: 2-5, 6-7, 0-1, 8   else: 0-3, 4-5, 6-7, 8
    *reinterpret_cast<double2 *>(yr + (hi ? 6 : 4)) = make_double2(hi ? v[6] : v[4], hi ? v[7] : v[5]);
    *reinterpret_cast<double2 *>(yr + (hi ? 0 : 6)) = make_double2(hi ? v[0] : v[6], hi ? v[1] : v[7]);
    yr[8] = v[8];
  }
}

// Store counterpart of load_row12: the 12 values v (columns 0-11) of a row at a 16-byte aligned
// address in one 256-bit store (the 32-byte aligned half) and one 128-bit store.
// Column c (0-11) of a row read by load_row12.
__device__ __forceinline__ float row12_col(const float (&raw)[3][4], bool hi, int c) {
  const int k = c / 4, i = c % 4;
  return hi ? (k == 0 ? raw[2][i] : k == 1 ? raw[0][i] : raw[1][i]) : (k == 0 ? raw[0][i] : k == 1 ? raw[1][i] : raw[2][i]);
}

// The first C (9-12) values v of an fp32 row at a 16-byte aligned address, and nothing past them:
// a 32-byte aligned run of 8 in one 256-bit store, 16-byte runs in 128-bit stores, the rest
// scalar (C = 9: two stores when the row starts on a 32-byte boundary, three otherwise).
__device__ __forceinline__ void store_row_exact12(float *yr, const float (&v)[12], int C) {
  const bool hi = ((uintptr_t)yr & 16u) != 0;
  if (!hi) {
    asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(yr), "f"(v[0]), "f"(v[1]),
                 "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7])
                 : "memory");
    if (C == 12) {
      *reinterpret_cast<float4 *>(yr + 8) = make_float4(v[8], v[9], v[10], v[11]);
    } else {
#pragma unroll
      for (int c = 8; c < 11; ++c)
        if (c < C) yr[c] = v[c];
    }
  } else {
    *reinterpret_cast<float4 *>(yr) = make_float4(v[0], v[1], v[2], v[3]);
    if (C == 12) {
      asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(yr + 4), "f"(v[4]), "f"(v[5]),
                   "f"(v[6]), "f"(v[7]), "f"(v[8]), "f"(v[9]), "f"(v[10]), "f"(v[11])
                   : "memory");
    } else {
      *reinterpret_cast<float4 *>(yr + 4) = make_float4(v[4], v[5], v[6], v[7]);
#pragma unroll
      for (int c = 8; c < 11; ++c)
        if (c < C) yr[c] = v[c];
    }
  }
}

__device__ __forceinline__ void store_row12(float *yr, const float (&v)[3][4]) {
  const bool hi = ((uintptr_t)yr & 16u) != 0;
  float *p8 = yr + (hi ? 4 : 0);
  float *p4 = yr + (hi ? 0 : 8);
  float e[8], g[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    e[i] = hi ? v[1][i] : v[0][i];
    e[4 + i] = hi ? v[2][i] : v[1][i];
    g[i] = hi ? v[0][i] : v[2][i];
  }
  asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p8), "f"(e[0]), "f"(e[1]), "f"(e[2]),
               "f"(e[3]), "f"(e[4]), "f"(e[5]), "f"(e[6]), "f"(e[7])
               : "memory");
  *reinterpret_cast<float4 *>(p4) = make_float4(g[0], g[1], g[2], g[3]);
}

// Sum over the stored entries of one row of w_j * X[col_j, :] for the lane's vectors, reduced
// over the group's edge slots (every lane of the warp must call this: it shuffles). Each lane
// takes its entries in batches of U: the U column indices and weights are loaded first, then the
// U neighbour rows, then the U multiply-adds, so U row gathers are in flight per lane instead of
// one. The per-lane accumulation order (entries beg+es, beg+es+ES, ...) is that of a plain loop.
// How a lane reads a gathered row: kRowVec one 16-byte vector at a time (VPL per lane, LV lanes per
// row); kRow12F the two loads of load_row12 (fp32 rows of three 16-byte vectors: VW 4, VPL 3) and
// kRow10D the three loads of load_row10d (fp64 rows of five: VW 2, VPL 5), each with the whole row
// held by one lane (the caller guarantees LV == 1).
// kRow16H reads a bf16 row of 16 values (two 16-byte vectors: VW 8, VPL 2) in one 256-bit load from a
// 32-byte aligned address and widens it to fp32 at the multiply-adds.
// kRow8F reads an fp32 row of 8 values (VW 4, VPL 2) in one 256-bit load from a 32-byte aligned
// address.
enum RowPath : int { kRowVec = 0, kRow12F = 1, kRow10D = 2, kRow16H = 3, kRow8F = 4 };

template <typename TW, typename TX, typename TA, int VW, int VPL, int U = gather_batch_wide<TA, VW, VPL>(),
          int ROW = kRowVec>
__device__ __forceinline__ void gather_row(const int32_t *__restrict__ col, const TW *__restrict__ w,
                                           const TX *__restrict__ X, int64_t ldx, int beg, int end, int es,
                                           int ES, int cl, int LV, int NV, int G, TA (&acc)[VPL][VW]) {
  static_assert(ROW != kRow12F ||
                    (std::is_same<TX, float>::value && std::is_same<TA, float>::value && VW == 4 && VPL == 3),
                "the two-load path gathers fp32 rows of three 16-byte vectors");
  static_assert(ROW != kRow10D ||
                    (std::is_same<TX, double>::value && std::is_same<TA, double>::value && VW == 2 && VPL == 5),
                "the three-load path gathers fp64 rows of five 16-byte vectors");
  static_assert(ROW != kRow8F ||
                    (std::is_same<TX, float>::value && std::is_same<TA, float>::value && VW == 4 && VPL == 2),
                "the one-load path gathers fp32 rows of two 16-byte vectors");
  static_assert(ROW != kRow16H ||
                    (std::is_same<TX, bf16>::value && std::is_same<TA, float>::value && VW == 8 && VPL == 2),
                "the one-load path gathers bf16 rows of two 16-byte vectors");
#pragma unroll
  for (int k = 0; k < VPL; ++k)
#pragma unroll
    for (int i = 0; i < VW; ++i) acc[k][i] = TA(0);
  for (int j0 = beg + es; j0 < end; j0 += U * ES) {
    int v[U];
    TA wv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int j = j0 + u * ES;
      v[u] = j < end ? ld_stream(col + j) : -1;
      wv[u] = j < end ? cvt<TA>(ld_stream(w + j)) : TA(0);
    }
    if constexpr (ROW == kRow16H) {
      uint32_t q[U][8];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (v[u] >= 0) {
          load_row16h(X + (long long)v[u] * ldx, q[u]);
        } else {
#pragma unroll
          for (int k = 0; k < 8; ++k) q[u][k] = 0u;
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u)
#pragma unroll
        for (int k = 0; k < 8; ++k) {  // bf16 -> fp32 widening is a 16-bit shift of the bit pattern
          const int c = 2 * k;
          acc[c / 8][c % 8] = fmaa(wv[u], __uint_as_float(q[u][k] << 16), acc[c / 8][c % 8]);
          acc[(c + 1) / 8][(c + 1) % 8] = fmaa(wv[u], __uint_as_float(q[u][k] & 0xffff0000u),
                                               acc[(c + 1) / 8][(c + 1) % 8]);
        }
      continue;
    }
    TA t[U][VPL][VW];
    bool hi[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const TX *xr = X + (long long)(v[u] < 0 ? 0 : v[u]) * ldx;
      hi[u] = false;
      if constexpr (ROW != kRowVec) {
        if (v[u] >= 0) {
          if constexpr (ROW == kRow12F) hi[u] = load_row12(xr, t[u]);
          else if constexpr (ROW == kRow10D) hi[u] = load_row10d(xr, t[u]);
          else if constexpr (ROW == kRow8F) load_row8(xr, t[u]);
        } else {
#pragma unroll
          for (int k = 0; k < VPL; ++k)
#pragma unroll
            for (int i = 0; i < VW; ++i) t[u][k][i] = TA(0);
        }
      } else {
#pragma unroll
        for (int k = 0; k < VPL; ++k) {
          const int vi = cl + k * LV;
          if (v[u] >= 0 && vi < NV) {
            load_vec<TX, VW, TA>(xr + (long long)vi * VW, t[u][k]);
          } else {
#pragma unroll
            for (int i = 0; i < VW; ++i) t[u][k][i] = TA(0);
          }
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if constexpr (ROW == kRow12F) {  // columns from the load order of load_row12
#pragma unroll
        for (int i = 0; i < VW; ++i) {
          acc[0][i] = fmaa(wv[u], hi[u] ? t[u][2][i] : t[u][0][i], acc[0][i]);
          acc[1][i] = fmaa(wv[u], hi[u] ? t[u][0][i] : t[u][1][i], acc[1][i]);
          acc[2][i] = fmaa(wv[u], hi[u] ? t[u][1][i] : t[u][2][i], acc[2][i]);
        }
      } else if constexpr (ROW == kRow10D) {  // columns from the load order of load_row10d
#pragma unroll
        for (int c = 0; c < 10; ++c) {
          const int fh = c < 2 ? 8 + c : c - 2;
          acc[c / 2][c % 2] = fmaa(wv[u], hi[u] ? t[u][fh / 2][fh % 2] : t[u][c / 2][c % 2], acc[c / 2][c % 2]);
        }
      } else {
#pragma unroll
        for (int k = 0; k < VPL; ++k)
#pragma unroll
          for (int i = 0; i < VW; ++i) acc[k][i] = fmaa(wv[u], t[u][k][i], acc[k][i]);
      }
    }
  }
  for (int off = LV; off < G; off <<= 1) {
#pragma unroll
    for (int k = 0; k < VPL; ++k)
#pragma unroll
      for (int i = 0; i < VW; ++i) acc[k][i] += __shfl_xor_sync(0xffffffffu, acc[k][i], off);
  }
}

}  // namespace dlp
