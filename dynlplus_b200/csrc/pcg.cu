// Block PCG with the Jacobi preconditioner, one CG per column (dynlp/solvers.py:66-97), fused for
// B200: three kernels per iteration, inner products summed in fp64 (fp32 only in the per-lane pAp
// partials of the fp32 whole-row apply, about a dozen rows each), convergence decided on the
// device, and the iteration loop itself on the device (a CUDA graph WHILE node whose flag K2
// sets), so the host waits once per solve instead of once per chunk of iterations.
//
//   K1 apply  : AP = diag*P - W P (row gather), pAp_c partials; last block: alpha_c = rz_c / pAp_c
//   K2 update : R -= alpha AP; rz_c = sum R^2/diag, ss_c = sum R^2, viol = max |R|/(eps_c diag);
//               last block: beta_c, stop decision (violation <= 1 and/or max_c ||R_c||/||rhs_c|| <=
//               target), patience, iteration cap
//   K3 dir    : Z += alpha P; P = R/diag + beta P   (P update skipped once a stop is proposed)
//
// A proposed stop is confirmed on the host against the true residual rhs - A Z, as the reference
// does (solvers.py:85-89); a failed recheck resumes the iteration from the true residual.
// Sums over rows go through per-block partials over a fixed grid and an ordered final pass, so
// the iterates do not depend on scheduling.
#include <cstddef>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "gather.cuh"

namespace dlp {

constexpr int kGroup = 32;      // blocks per first-level group of the grid reductions
constexpr int kMaxGroups = 64;  // groups per grid (grids of up to 2048 blocks)

struct PcgCtl {
  int32_t iters;
  int32_t done;   // 0 running, 1 stop proposed, 2 stalled, 3 iteration cap, 5 converged (confirmed),
                  // 6 cancelled (the host's cancel word was set)
  int32_t stall;
  int32_t go;     // set by K1 for the iteration in flight
  uint32_t cnt1, cnt2;
  int32_t mode, patience;
  int32_t max_iter, bad;  // bad: non-finite residual entries seen (breakdown)
  int32_t par, pad;       // two-kernel iteration: which of P / AP holds the current direction
  double best, viol, relres, target;
  // first-level counters of the grid reductions (last_block_grouped), one per group of blocks;
  // zero between launches. The host reads only the fields above them (kCtlHead).
  uint32_t gcnt1[kMaxGroups], gcnt2[kMaxGroups];
};
constexpr size_t kCtlHead = offsetof(PcgCtl, gcnt1);

// Per-block partials are stored output-major: output o of block b at part[o * nbmax + b].
struct PcgBufs {
  PcgCtl *ctl;
  // rzprev: rz of the iteration in flight, kept for the beta of a resume after a failed recheck
  double *alpha, *beta, *rz, *eps, *rhsn, *epsinv, *rzprev, *part1, *part2;
  double *gpart1, *gpart2;  // per-group partials: output o of group g at gpart[o * kMaxGroups + g]
  int nbmax;
  // set only in the kernels of the device-side loop graph: K2 writes the loop's continue flag
  int has_cond;
  cudaGraphConditionalHandle cond;
  const int32_t *cancel;  // the registered cancel word (NULL: none), read at every stop decision
};

constexpr int kUpdBlocksPerSM = 8;

static int upd_blocks() { return sm_count() * kUpdBlocksPerSM; }
static int apply_blocks() { return sm_count() * 8; }

static size_t align256(size_t x) { return (x + 255) / 256 * 256; }

static size_t pcg_ws_bytes(int C) {
  const size_t nb = (size_t)std::max(upd_blocks(), apply_blocks());
  size_t b = align256(sizeof(PcgCtl));
  b += 7 * align256(sizeof(double) * C);
  b += align256(sizeof(double) * nb * 2 * C);        // part1 (pAp; q of the two-kernel iteration)
  b += align256(sizeof(double) * nb * (2 * C + 1));  // part2 (rz, ss, violation)
  b += align256(sizeof(double) * kMaxGroups * 2 * C);        // gpart1
  b += align256(sizeof(double) * kMaxGroups * (2 * C + 1));  // gpart2
  return b;
}

// Bytes of the workspace's head: the control block and the seven per-column vectors (carve order).
static size_t head_bytes(int C) { return align256(sizeof(PcgCtl)) + 7 * align256(sizeof(double) * C); }

// Pinned host staging, one per host thread and device: the image of the workspace's head that a
// solve uploads in one copy, and the control block's read-backs. Before the image is rewritten the
// thread waits for the event recorded after its last upload, so a copy still in flight never sees
// the next solve's values. Kept for the thread's lifetime.
struct HostStage {
  char *img = nullptr;
  size_t cap = 0;
  PcgCtl *rd = nullptr;
  cudaEvent_t up = nullptr;
};
static thread_local HostStage t_stage[64];

static int stage_get(int dev, size_t bytes, HostStage **out) {
  if (dev < 0 || dev >= 64) return DLP_ERR_INVALID;
  HostStage &g = t_stage[dev];
  if (!g.up) DLP_CUDA(cudaEventCreateWithFlags(&g.up, cudaEventDisableTiming));
  DLP_CUDA(cudaEventSynchronize(g.up));
  if (g.cap < bytes) {
    if (g.img) DLP_CUDA(cudaFreeHost(g.img));
    g.img = nullptr;
    g.cap = 0;
    DLP_CUDA(cudaHostAlloc((void **)&g.img, bytes, cudaHostAllocPortable));
    g.cap = bytes;
  }
  if (!g.rd) DLP_CUDA(cudaHostAlloc((void **)&g.rd, sizeof(PcgCtl), cudaHostAllocPortable));
  *out = &g;
  return DLP_OK;
}

// The control block's head, read through the thread's pinned buffer (a blocking read).
static int read_ctl(const PcgBufs &B, HostStage *hs, cudaStream_t s, PcgCtl *cur) {
  DLP_CUDA(cudaMemcpyAsync(hs->rd, B.ctl, kCtlHead, cudaMemcpyDeviceToHost, s));
  DLP_CUDA(cudaStreamSynchronize(s));
  std::memcpy((void *)cur, hs->rd, kCtlHead);
  return DLP_OK;
}

static PcgBufs carve(void *ws, int C) {
  const size_t nb = (size_t)std::max(upd_blocks(), apply_blocks());
  char *p = (char *)ws;
  PcgBufs B;
  B.ctl = (PcgCtl *)p;
  p += align256(sizeof(PcgCtl));
  double **vecs[7] = {&B.alpha, &B.beta, &B.rz, &B.eps, &B.rhsn, &B.epsinv, &B.rzprev};
  for (auto v : vecs) {
    *v = (double *)p;
    p += align256(sizeof(double) * C);
  }
  B.part1 = (double *)p;
  p += align256(sizeof(double) * nb * 2 * C);
  B.part2 = (double *)p;
  p += align256(sizeof(double) * nb * (2 * C + 1));
  B.gpart1 = (double *)p;
  p += align256(sizeof(double) * kMaxGroups * 2 * C);
  B.gpart2 = (double *)p;
  B.nbmax = (int)nb;
  B.has_cond = 0;
  B.cond = 0;
  B.cancel = nullptr;
  return B;
}

// Last of `count` blocks to arrive at the counter gets true (after a device-wide fence).
__device__ __forceinline__ bool last_of(uint32_t *counter, uint32_t count) {
  __shared__ bool is_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    const uint32_t t = atomicAdd(counter, 1u);
    is_last = (t == count - 1);
  }
  __syncthreads();
  if (is_last) __threadfence();
  return is_last;
}

__device__ __forceinline__ int grid_groups() { return ((int)gridDim.x + kGroup - 1) / kGroup; }

// Deterministic reduction of at most 64 partials per output by the calling block: output o < NO is
// the sum (o < nsum) or the max (of non-negative values) of part[o * stride + b] over b < nb.
// Warp w takes outputs w*4 .. w*4+3, then w*4 + 4 NW, ...; lane l the partials l and l + 32; every
// load of a warp's pass is issued before its first sum, then a fixed xor tree; emit(o, v) runs on
// lane 0. The order depends only on nb. Ends with a block barrier.
template <int NT, class Emit>
__device__ __forceinline__ void small_partials_reduce(const double *part, long long stride, int nb, int NO, int nsum,
                                                      Emit emit) {
  constexpr int NW = NT / 32, kPer = 4;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int o0 = wid * kPer; o0 < NO; o0 += NW * kPer) {
    double x[kPer][2];
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const int o = o0 + k;
      const double *po = part + (long long)o * stride;
      x[k][0] = (o < NO && lane < nb) ? __ldcg(po + lane) : 0.0;
      x[k][1] = (o < NO && lane + 32 < nb) ? __ldcg(po + lane + 32) : 0.0;
    }
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const int o = o0 + k;
      const bool sum = o < nsum;
      double v = sum ? x[k][0] + x[k][1] : fmax(x[k][0], x[k][1]);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double y = __shfl_xor_sync(0xffffffffu, v, off);
        v = sum ? v + y : fmax(v, y);
      }
      if (lane == 0 && o < NO) emit(o, v);
    }
  }
  __syncthreads();
}

// Two-level last block of a grid reduction over per-block partials part[o * stride + b] (every
// block calls it after writing its own): the last block to finish in each group of kGroup
// consecutive blocks folds the group's partials into gpart[o * kMaxGroups + group] and resets the
// group's counter; the last of those returns true, and then reduces gpart over grid_groups()
// groups (small_partials_reduce). Two short reductions instead of one over the whole grid on the
// path after the slowest block.
template <int NT>
__device__ __forceinline__ bool last_block_grouped(const double *part, long long stride, int NO, int nsum,
                                                   uint32_t *gcnt, uint32_t *top, double *gpart) {
  const int g = (int)blockIdx.x / kGroup;
  const int gsize = min(kGroup, (int)gridDim.x - g * kGroup);
  if (!last_of(&gcnt[g], (uint32_t)gsize)) return false;
  small_partials_reduce<NT>(part + (long long)g * kGroup, stride, gsize, NO, nsum,
                            [&](int o, double v) { gpart[(long long)o * kMaxGroups + g] = v; });
  if (threadIdx.x == 0) gcnt[g] = 0;
  return last_of(top, (uint32_t)grid_groups());
}

// ------------------------------------------------------------------------------------------------
// K1: AP = diag*P - W P and pAp partials
// ------------------------------------------------------------------------------------------------
template <class T>
struct ApplyArgs {
  const int32_t *rbeg, *rend, *col;
  const typename T::TW *w;
  int32_t n, C;
  const typename T::TX *P;
  int64_t ldp;
  const typename T::TV *diag;
  typename T::TY *AP;
  int64_t ldap;
  PcgBufs B;
  int G, LV, NV;
  const typename T::TV *Pown;  // own-row P for the diagonal term and pAp (NULL: P itself)
  int64_t ldpo;
  int ap_row12;  // AP rows are 16-byte aligned and >= 12 wide: whole-row vector stores (two-load path)
};

// Small fp32 rows fit in 64 registers (4 blocks of 256 threads per SM); the wider or fp64 ones keep
// the compiler's choice rather than spill.
template <class T, int VW, int VPL>
constexpr int apply_min_blocks() {
  return (sizeof(typename T::TA) == 4 && VPL * VW <= 12 && VPL <= 4) ? 4 : 1;
}

// ROW12 as in gather_row: fp32 12-float rows held whole by one lane, two loads per row. Its lanes
// keep their pAp partials (about a dozen rows each) in fp32 and the rest of the sum runs in fp64,
// which frees the registers for two rows in flight per lane within the 64-register cap (measured on
// B200 at n = 1M, degree 10, C = 9: 123 us; fp64 lane partials allow one row in flight, 127 us; two
// spill, 166 us; per-vector loads 160 us).
//
// FUSE (fp32 whole rows only): the apply of the two-kernel iteration. P and AP trade places every
// iteration (ctl->par says which buffer holds the direction), and the lanes also sum
// q_c = sum AP^2 / diag, from which the last block predicts the iteration's beta before the residual
// update: with alpha = rz / pAp and the A-conjugacy of successive directions ((P_prev, A P) = 0, so
// (R / diag) . AP = pAp), rz_next = sum (R - alpha AP)^2 / diag = alpha^2 q - rz, and
// beta = rz_next / rz = alpha^2 q / rz - 1. The exact rz_next of the stored residual, summed by the
// fused sweep, is the one the next alpha uses.
// Reduce-scatter of 12 per-lane column values (padded to 16 slots) over the warp: lanes 2c and
// 2c + 1 return column c's sum over the 32 lanes (slot c = lane bits 4..1), lanes of slots >= 12 zero.
__device__ __forceinline__ float warp_scatter12(const float (&v)[12], int lane) {
  float v8[8], v4[4], v2[2];
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4, b1 = lane & 2;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const float lo = v[j], hi = j + 8 < 12 ? v[j + 8] : 0.f;
    v8[j] = (b4 ? hi : lo) + __shfl_xor_sync(0xffffffffu, b4 ? lo : hi, 16);
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) v4[j] = (b3 ? v8[j + 4] : v8[j]) + __shfl_xor_sync(0xffffffffu, b3 ? v8[j] : v8[j + 4], 8);
#pragma unroll
  for (int j = 0; j < 2; ++j) v2[j] = (b2 ? v4[j + 2] : v4[j]) + __shfl_xor_sync(0xffffffffu, b2 ? v4[j] : v4[j + 2], 4);
  const float v1 = (b1 ? v2[1] : v2[0]) + __shfl_xor_sync(0xffffffffu, b1 ? v2[0] : v2[1], 2);
  return v1 + __shfl_xor_sync(0xffffffffu, v1, 1);
}

template <class T, int VW, int VPL, int ROWP = kRowVec, bool FUSE = false>
__global__ void __launch_bounds__(kThreads, (apply_min_blocks<T, VW, VPL>())) k_pcg_apply(ApplyArgs<T> p) {
  using TA = typename T::TA;
  PcgCtl *ctl = p.B.ctl;
  if (ctl->done != 0) {
    if (blockIdx.x == 0 && threadIdx.x == 0) ctl->go = 0;
    return;
  }
  if (FUSE && ctl->par) {  // this iteration's direction is in the AP buffer; AP goes to the P buffer
    const typename T::TX *tp = p.P;
    p.P = (const typename T::TX *)p.AP;
    p.AP = (typename T::TY *)tp;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl->go = 1;
  __shared__ double sm[kThreads / 32][256];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int G = p.G, LV = p.LV, NV = p.NV;
  const int gl = lane & (G - 1);
  const int cl = gl & (LV - 1);
  const int es = gl / LV;
  const int ES = G / LV;
  const int gpw = 32 / G;
  constexpr bool WHOLE = ROWP == kRow12F || ROWP == kRow8F;  // one lane holds a whole fp32 row
  constexpr int NR = ROWP == kRow8F ? 2 : 3;                  // its 16-byte vectors
  using TD = typename std::conditional<WHOLE, float, double>::type;  // a lane's pAp partials
  TD dot[VPL][VW];
#pragma unroll
  for (int k = 0; k < VPL; ++k)
#pragma unroll
    for (int i = 0; i < VW; ++i) dot[k][i] = TD(0);
  // FUSE: pAp and q are summed over the warp's 32 rows after each batch (warp_scatter12), so a lane
  // keeps one running partial of each instead of a row's worth: the registers go to a second row in
  // flight. fp32 sums over 32 rows, accumulated in fp64.
  double pacc = 0.0, qacc = 0.0;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long g0 = warp * gpw; g0 < p.n; g0 += nwarps * gpw) {
    const long long r = g0 + lane / G;
    const bool valid = r < p.n;
    const int beg = valid ? p.rbeg[r] : 0;
    const int end = valid ? p.rend[r] : 0;
    TA acc[VPL][VW];
    // gathered rows in flight per lane: four 8-float rows (64 registers, no spill: 121.2 -> 119.1 us
    // per iteration at n = 1M against two), two 12-float rows
    gather_row<typename T::TW, typename T::TX, TA, VW, VPL,
               (ROWP == kRow8F ? 4 : WHOLE ? 2 : gather_batch_lean<TA, VW, VPL>()),
               (WHOLE ? ROWP : kRowVec)>(
        p.col, p.w, p.P, p.ldp, beg, end, es, ES, cl, LV, NV, G, acc);
    // FUSE: this row's P . AP and AP^2 / diag per column (0 past C and on invalid lanes)
    float pv_[FUSE ? 12 : 1], qv[FUSE ? 12 : 1];
    if constexpr (FUSE) {
#pragma unroll
      for (int c = 0; c < 12; ++c) pv_[c] = qv[c] = 0.f;
    }
    if (valid && es == 0) {
      const TA d = cvt<TA>(p.diag[r]);
      if constexpr (WHOLE) {
        // the own row whole too (two loads for 12 floats at a 16-byte boundary, one for 8 at 32)
        float pw[NR][4];
        bool hi = false;
        if constexpr (ROWP == kRow8F) load_row8(p.P + r * p.ldp, pw);
        else hi = load_row12(p.P + r * p.ldp, pw);
        float apv[NR][4];
#pragma unroll
        for (int k = 0; k < NR; ++k)
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int c = k * 4 + i;
            float pv;
            if constexpr (ROWP == kRow8F) pv = pw[k][i];
            else pv = k == 0 ? (hi ? pw[2][i] : pw[0][i]) : k == 1 ? (hi ? pw[0][i] : pw[1][i])
                                                          : (hi ? pw[1][i] : pw[2][i]);
            // padding columns too when the whole row is stored; zeros there when AP becomes the next
            // direction (FUSE), so the gathered padding stays zero
            apv[k][i] = (FUSE && c >= p.C) ? 0.f : d * pv - acc[k][i];
            if (c < p.C) {
              if (!p.ap_row12) p.AP[r * p.ldap + c] = apv[k][i];
              if constexpr (FUSE) pv_[c] = pv * apv[k][i];
              else dot[k][i] += (TD)pv * (TD)apv[k][i];
            }
          }
        if (p.ap_row12) {
          if constexpr (ROWP == kRow8F) store_row8(p.AP + r * p.ldap, apv);
          else store_row12(p.AP + r * p.ldap, apv);
        }
        if constexpr (FUSE) {
          const float rinv = __frcp_rn((float)d);
#pragma unroll
          for (int k = 0; k < NR; ++k)
#pragma unroll
            for (int i = 0; i < 4; ++i)
              if (k * 4 + i < p.C) qv[k * 4 + i] = apv[k][i] * apv[k][i] * rinv;
        }
      } else {
#pragma unroll
        for (int k = 0; k < VPL; ++k) {
          const int vi = cl + k * LV;
          if (vi < NV) {
#pragma unroll
            for (int i = 0; i < VW; ++i) {
              const int c = vi * VW + i;
              if (c < p.C) {
                const TA pv = p.Pown ? cvt<TA>(p.Pown[r * p.ldpo + c]) : cvt<TA>(p.P[r * p.ldp + c]);
                const TA ap = d * pv - acc[k][i];
                p.AP[r * p.ldap + c] = cvt<typename T::TY>(ap);
                dot[k][i] += (double)pv * (double)ap;
              }
            }
          }
        }
      }
    }
    if constexpr (FUSE) {
      pacc += (double)warp_scatter12(pv_, lane);
      qacc += (double)warp_scatter12(qv, lane);
    }
  }
  // lanes sharing a vector lane (same cl) hold the same columns: reduce over the other bits, in fp64
  constexpr int NQ = FUSE ? 2 : 1;  // pAp, and q when fused
  if constexpr (!FUSE) {
    double dsum[VPL][VW];
#pragma unroll
    for (int k = 0; k < VPL; ++k)
#pragma unroll
      for (int i = 0; i < VW; ++i) {
        double x = (double)dot[k][i];
        for (int off = LV; off < 32; off <<= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
        dsum[k][i] = x;
      }
    if (lane < LV) {
#pragma unroll
      for (int k = 0; k < VPL; ++k) {
        const int vi = lane + k * LV;
        if (vi < NV) {
#pragma unroll
          for (int i = 0; i < VW; ++i) {
            const int c = vi * VW + i;
            if (c < p.C) sm[wid][c] = dsum[k][i];
          }
        }
      }
    }
  }
  if constexpr (FUSE) {  // lanes 2c hold the warp's pAp and q of column c (slot of lane bits 4..1)
    const int slot = ((lane >> 4) & 1) * 8 + ((lane >> 3) & 1) * 4 + ((lane >> 2) & 1) * 2 + ((lane >> 1) & 1);
    if ((lane & 1) == 0 && slot < p.C) {
      sm[wid][slot] = pacc;
      sm[wid][p.C + slot] = qacc;
    }
  }
  __syncthreads();
  for (int c = threadIdx.x; c < NQ * p.C; c += blockDim.x) {
    double s = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) s += sm[w][c];
    p.B.part1[(long long)c * p.B.nbmax + blockIdx.x] = s;
  }
  if (last_block_grouped<kThreads>(p.B.part1, p.B.nbmax, NQ * p.C, NQ * p.C, ctl->gcnt1, &ctl->cnt1,
                                   p.B.gpart1)) {
    const PcgBufs &B = p.B;
    if constexpr (FUSE) {
      __shared__ double s_pq[2 * 12];
      small_partials_reduce<kThreads>(B.gpart1, kMaxGroups, grid_groups(), 2 * p.C, 2 * p.C,
                                      [&](int o, double s) { s_pq[o] = s; });
      for (int c = threadIdx.x; c < p.C; c += blockDim.x) {
        const double pap = s_pq[c], q = s_pq[p.C + c], rz = B.rz[c];
        double al = pap > 0.0 ? rz / pap : 0.0;
        al = isfinite(al) && fabs(al) < 1e30 ? al : 0.0;
        B.alpha[c] = al;
        const double be = rz > 0.0 ? al * al * q / rz - 1.0 : 0.0;
        B.beta[c] = isfinite(be) && be > 0.0 && be < 1e30 ? be : 0.0;
      }
    } else {
      small_partials_reduce<kThreads>(B.gpart1, kMaxGroups, grid_groups(), p.C, p.C, [&](int c, double s) {
        const double al = s > 0.0 ? B.rz[c] / s : 0.0;
        B.alpha[c] = isfinite(al) && fabs(al) < 1e30 ? al : 0.0;
      });
    }
    if (threadIdx.x == 0) ctl->cnt1 = 0;
  }
}

// ------------------------------------------------------------------------------------------------
// Element sweeps (K2, K3). Thread t of the grid owns column c = t mod ld of the rows t/ld,
// t/ld + RS, t/ld + 2 RS, ... with RS = (threads in the grid) / ld: its column never changes, so its
// per-column sums are scalars, and consecutive threads touch consecutive addresses of the
// row-major n x ld block. kSweepUnroll rows per batch are loaded before any is used.
// ------------------------------------------------------------------------------------------------
constexpr int kSweepUnroll = 4;
constexpr int kSweepThreads = 256;

// fp32 sweeps fit in 64 registers without spilling (4 resident blocks per SM); fp64 ones keep the
// compiler's choice.
template <typename T>
constexpr int sweep_min_blocks() {
  return sizeof(T) == 4 ? 4 : 1;
}

struct SweepIdx {
  long long r0, RS;
  int c;
  bool on;  // thread owns a column < C
};

__device__ __forceinline__ SweepIdx sweep_index(int64_t ld, int32_t C) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)gridDim.x * blockDim.x;
  SweepIdx s;
  s.RS = total / ld;
  s.r0 = t / ld;
  s.c = (int)(t - s.r0 * ld);
  s.on = s.r0 < s.RS && s.c < C;
  return s;
}

// Deterministic per-column block sums of the per-thread values v[tid] (thread tid of this block
// owns column (blockIdx.x * blockDim.x + tid) mod ld): warp w handles columns w, w+8, ...; the
// lanes take the column's threads in a fixed strided order, then a fixed xor tree.
__device__ __forceinline__ double block_column_sum(const double *v, int c, int64_t ld) {
  const long long base = (long long)blockIdx.x * blockDim.x;
  const int first = (int)(((c - base % ld) % ld + ld) % ld);
  const int lane = lane_id();
  double s = 0.0;
  for (long long tid = first + (long long)lane * ld; tid < blockDim.x; tid += 32 * ld) s += v[tid];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  return s;
}

// The last block of a residual sweep (K2, or the fused sweep of the two-kernel iteration): reduces
// the partials (rz_c, ss_c, violation), keeps rz for the next alpha and the one it replaces
// (rzprev: the beta of a resume after a failed recheck, rz_true / rz of the iteration, as the
// reference's loop has it), sets K3's beta (three-kernel phases 0 and 1), and takes the stop
// decision: violation <= 1 and/or max_c ||R_c||/||rhs_c|| <= target, patience, iteration cap,
// cancel word; the fused sweep flips which buffer holds the direction.
__device__ void finish_sweep(int phase, int32_t C, const PcgBufs &B, bool fused) {
  PcgCtl *ctl = B.ctl;
  const int tid = threadIdx.x;
  // outputs: rz_c (c < C), ss_c (C + c), violation (2C)
  __shared__ double s_out[2 * 256 + 1];
  small_partials_reduce<kSweepThreads>(B.gpart2, kMaxGroups, grid_groups(), 2 * C + 1, 2 * C,
                                       [&](int o, double v) { s_out[o] = v; });
  __shared__ double s_rel;
  if (tid == 0) s_rel = 0.0;
  __syncthreads();
  for (int c = tid; c < C; c += kSweepThreads) {
    const double a = s_out[c], b = s_out[C + c];
    const double rzo = B.rz[c];
    if (phase == 0) B.rzprev[c] = rzo;
    if (!fused) {
      const double den = phase == 1 ? B.rzprev[c] : rzo;
      const double be = (phase < 2 && den > 0.0) ? a / den : 0.0;
      B.beta[c] = isfinite(be) && fabs(be) < 1e30 ? be : 0.0;
    }
    B.rz[c] = a;
    const double rel = B.rhsn[c] > 0.0 ? sqrt(b) / B.rhsn[c] : sqrt(b);
    // fmax over non-negative doubles: the int64 view is monotone
    atomicMax((unsigned long long *)&s_rel, __double_as_longlong(rel));
  }
  __syncthreads();
  if (tid == 0) {
    const double v = s_out[2 * C];
    const double rel = s_rel;
    ctl->viol = v;
    ctl->relres = rel;
    double m = 0.0;
    if (ctl->mode & 1) m = fmax(m, v);
    if (ctl->mode & 2) m = fmax(m, ctl->target > 0.0 ? rel / ctl->target : rel);
    const bool conv = m <= 1.0 && !ctl->bad;
    if (phase == 0) ctl->iters += 1;
    if (phase == 0 && fused) ctl->par ^= 1;  // the next direction went into the other buffer
    if (phase >= 2) {  // the initial residual
      ctl->best = m;
      ctl->stall = 0;
      ctl->done = conv ? 5 : 0;
    } else if (phase == 0 && conv) {
      ctl->done = 1;  // proposed: confirmed against the true residual by the host
    } else if (phase == 1 && conv) {
      ctl->done = 5;
    } else {
      if (m < 0.9 * ctl->best) {
        ctl->best = m;
        ctl->stall = 0;
      } else {
        ctl->stall += 1;
      }
      if (ctl->stall >= ctl->patience) ctl->done = 2;
      else if (phase == 1) ctl->done = 0;
    }
    if (ctl->done == 0 && ctl->iters >= ctl->max_iter) ctl->done = 3;
    if (ctl->done == 0 && read_cancel(B.cancel)) ctl->done = 6;
    if (ctl->bad) ctl->done = 4;
    ctl->cnt2 = 0;
    // the device-side loop runs another iteration only while the solve is running
    if (B.has_cond) cudaGraphSetConditional(B.cond, ctl->done == 0 ? 1u : 0u);
  }
}

// K2: residual update + reductions + stop decision
//   phase 0: iteration (R -= alpha AP)      phase 1: recheck of a true residual
//   phase 2: initial residual (sets best, rz)
//   phase 3: as phase 2, the initial residual copied into R from the array passed as AP (the rhs of
//            a zero start) in the same sweep
// A non-finite residual entry stops the solve with status 4 (breakdown) instead of letting the
// max-reductions (which skip NaN) read it as convergence.
template <typename T>
__global__ void __launch_bounds__(kSweepThreads, (sweep_min_blocks<T>())) k_pcg_update(int phase, int32_t n, int32_t C, T *__restrict__ R,
                                                              int64_t ldr, const T *__restrict__ AP, int64_t ldap,
                                                              const T *__restrict__ diag, PcgBufs B) {
  PcgCtl *ctl = B.ctl;
  if (phase == 0 && !ctl->go) {
    if (B.has_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(B.cond, 0u);  // loop ends
    return;
  }
  // the loop flag starts cleared; the last block (ordered after this by its fence) sets it, so the
  // loop cannot run on without a decision
  if (B.has_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(B.cond, 0u);
  __shared__ double s_rz[kSweepThreads], s_ss[kSweepThreads], s_v[kSweepThreads / 32];
  const SweepIdx ix = sweep_index(ldr, C);
  double rz = 0.0, ss = 0.0, vmax = 0.0;
  bool bad = false;
  if (ix.on) {
    const int c = ix.c;
    const T al = phase == 0 ? (T)B.alpha[c] : T(0);
    // element offsets advance by addition (no 64-bit multiply per element)
    const long long rstep = ix.RS * ldr, astep = ix.RS * ldap;
    long long offr = ix.r0 * ldr + c, offa = ix.r0 * ldap + c;
    double rmax = 0.0;  // max |R| / diag; the column's 1/eps scales it once at the end
    auto element = [&](T rv, T ap, T dv, long long o) {
      if (phase == 0) {
        rv = rv - al * ap;
        R[o] = rv;
      } else if (phase == 3) {
        R[o] = rv;
      }
      const double r64 = (double)rv;
      const double dinv = __drcp_rn((double)dv);  // correctly rounded: the value of 1.0 / d
      const double r2 = r64 * r64;
      rz += r2 * dinv;
      ss += r2;
      rmax = fmax(rmax, fabs(r64) * dinv);
    };
    long long r = ix.r0;
    // full batches: kSweepUnroll rows in range, every load issued before any is used
    for (; r + (kSweepUnroll - 1) * ix.RS < n; r += kSweepUnroll * ix.RS) {
      T rv[kSweepUnroll], ap[kSweepUnroll], dv[kSweepUnroll];
#pragma unroll
      for (int u = 0; u < kSweepUnroll; ++u) {
        rv[u] = phase == 3 ? AP[offa + u * astep] : R[offr + u * rstep];
        dv[u] = diag[r + u * ix.RS];
        ap[u] = phase == 0 ? AP[offa + u * astep] : T(0);
      }
#pragma unroll
      for (int u = 0; u < kSweepUnroll; ++u) element(rv[u], ap[u], dv[u], offr + u * rstep);
      offr += kSweepUnroll * rstep;
      offa += kSweepUnroll * astep;
    }
    for (; r < n; r += ix.RS) {  // the last rows, one at a time
      element(phase == 3 ? AP[offa] : R[offr], phase == 0 ? AP[offa] : T(0), diag[r], offr);
      offr += rstep;
      offa += astep;
    }
    // a non-finite entry makes the fp64 sum of squares non-finite (fp32 squares cannot overflow it)
    bad = !isfinite(ss);
    // rounding is monotone, so scaling the max equals the max of the scaled ratios
    vmax = rmax * B.epsinv[c];
  }
  if (bad) ctl->bad = 1;
  const int tid = threadIdx.x, lane = lane_id(), wid = tid >> 5;
  s_rz[tid] = rz;
  s_ss[tid] = ss;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, off));
  if (lane == 0) s_v[wid] = vmax;
  __syncthreads();
  for (int c = wid; c < C; c += kSweepThreads / 32) {
    const double a = block_column_sum(s_rz, c, ldr);
    const double b = block_column_sum(s_ss, c, ldr);
    if (lane == 0) {
      B.part2[(long long)c * B.nbmax + blockIdx.x] = a;
      B.part2[(long long)(C + c) * B.nbmax + blockIdx.x] = b;
    }
  }
  if (tid == 0) {
    double v = 0.0;
    for (int w = 0; w < kSweepThreads / 32; ++w) v = fmax(v, s_v[w]);
    B.part2[(long long)(2 * C) * B.nbmax + blockIdx.x] = v;
  }
  if (last_block_grouped<kSweepThreads>(B.part2, B.nbmax, 2 * C + 1, 2 * C, ctl->gcnt2, &ctl->cnt2, B.gpart2))
    finish_sweep(phase, C, B, false);
}

// K2 of the two-kernel iteration: the residual update, the solution update and the next direction
// in one sweep, with the beta the apply predicted (k_pcg_apply, FUSE):
//   R -= alpha AP; Z += alpha P; P_next = R / diag + beta P; rz_c, ss_c, violation of the new R
// P_next is written over AP (the same element is read first), so the current direction stays intact
// for a resume after a failed recheck; the last block takes the stop decision as K2 does and
// flips ctl->par. buf0 / buf1 are the P and AP buffers (same leading dimension ld).
template <typename T>
__global__ void __launch_bounds__(kSweepThreads, (sweep_min_blocks<T>()))
    k_pcg_fused(int32_t n, int32_t C, T *__restrict__ R, int64_t ldr, T *__restrict__ Z, int64_t ldz, T *buf0,
                T *buf1, int64_t ld, const T *__restrict__ diag, PcgBufs B) {
  PcgCtl *ctl = B.ctl;
  if (!ctl->go) {
    if (B.has_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(B.cond, 0u);  // loop ends
    return;
  }
  if (B.has_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(B.cond, 0u);
  __shared__ double s_rz[kSweepThreads], s_ss[kSweepThreads], s_v[kSweepThreads / 32];
  const bool par = ctl->par != 0;
  const T *P = par ? buf1 : buf0;
  T *AP = par ? buf0 : buf1;  // AP in, the next direction out
  const SweepIdx ix = sweep_index(ldr, C);
  double rz = 0.0, ss = 0.0, vmax = 0.0;
  bool bad = false;
  if (ix.on) {
    const int c = ix.c;
    const T al = (T)B.alpha[c], be = (T)B.beta[c];
    const long long rstep = ix.RS * ldr, zstep = ix.RS * ldz, pstep = ix.RS * ld;
    long long offr = ix.r0 * ldr + c, offz = ix.r0 * ldz + c, offp = ix.r0 * ld + c;
    double rmax = 0.0;
    for (long long r = ix.r0; r < n; r += kSweepUnroll * ix.RS) {
      // every load of the batch is issued before any store
      T rv[kSweepUnroll], av[kSweepUnroll], pv[kSweepUnroll], zv[kSweepUnroll], dv[kSweepUnroll];
#pragma unroll
      for (int u = 0; u < kSweepUnroll; ++u) {
        const long long rr = r + u * ix.RS;
        const bool ok = rr < n;
        rv[u] = ok ? R[offr + u * rstep] : T(0);
        av[u] = ok ? AP[offp + u * pstep] : T(0);
        pv[u] = ok ? P[offp + u * pstep] : T(0);
        zv[u] = ok ? Z[offz + u * zstep] : T(0);
        dv[u] = ok ? diag[rr] : T(1);
      }
#pragma unroll
      for (int u = 0; u < kSweepUnroll; ++u) {
        const long long rr = r + u * ix.RS;
        if (rr < n) {
          const T rn = rv[u] - al * av[u];
          R[offr + u * rstep] = rn;
          Z[offz + u * zstep] = zv[u] + al * pv[u];
          const double r64 = (double)rn;
          const double dinv = __drcp_rn((double)dv[u]);  // correctly rounded: the value of 1.0 / d
          // R / diag rounded to T: for fp32 operands the fp64 product with the correctly rounded
          // reciprocal rounds to the same value as the fp32 quotient (the quotient is never within
          // 2^-49 relative of an fp32 rounding midpoint; the product is within 2^-52 of it)
          AP[offp + u * pstep] = (T)(r64 * dinv) + be * pv[u];
          const double r2 = r64 * r64;
          rz += r2 * dinv;
          ss += r2;
          rmax = fmax(rmax, fabs(r64) * dinv);
        }
      }
      offr += kSweepUnroll * rstep;
      offz += kSweepUnroll * zstep;
      offp += kSweepUnroll * pstep;
    }
    bad = !isfinite(ss);
    vmax = rmax * B.epsinv[c];
  }
  if (bad) ctl->bad = 1;
  const int tid = threadIdx.x, lane = lane_id(), wid = tid >> 5;
  s_rz[tid] = rz;
  s_ss[tid] = ss;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, off));
  if (lane == 0) s_v[wid] = vmax;
  __syncthreads();
  for (int c = wid; c < C; c += kSweepThreads / 32) {
    const double a = block_column_sum(s_rz, c, ldr);
    const double b = block_column_sum(s_ss, c, ldr);
    if (lane == 0) {
      B.part2[(long long)c * B.nbmax + blockIdx.x] = a;
      B.part2[(long long)(C + c) * B.nbmax + blockIdx.x] = b;
    }
  }
  if (tid == 0) {
    double v = 0.0;
    for (int w = 0; w < kSweepThreads / 32; ++w) v = fmax(v, s_v[w]);
    B.part2[(long long)(2 * C) * B.nbmax + blockIdx.x] = v;
  }
  if (last_block_grouped<kSweepThreads>(B.part2, B.nbmax, 2 * C + 1, 2 * C, ctl->gcnt2, &ctl->cnt2, B.gpart2))
    finish_sweep(0, C, B, true);
}

// Coherent 256-bit row access for the row sweep (rows it reads and then writes in the same launch),
// with an L2 eviction policy: R, Z, AP and the current direction are streamed through (evict-first)
// and the next direction, which the next apply gathers about ten times per row, is kept (evict-last).
// Measured on the 8-column iteration at n = 1M, degree 10: 124.4 -> 121.5 us.
__device__ __forceinline__ uint64_t l2_evict_first_pol() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ void ld_row8(const float *xr, float (&v)[8], uint64_t pol) {
  asm volatile("ld.global.L2::cache_hint.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8], %9;"
               : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
               : "l"(xr), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void st_row8(float *yr, const float (&v)[8], uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8}, %9;" ::"l"(yr), "f"(v[0]), "f"(v[1]),
               "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7]), "l"(pol)
               : "memory");
}

// Reduce-scatter of 16 per-lane values over the warp: lanes 2s and 2s + 1 return value s's sum over
// the 32 lanes (s = lane bits 4..1). Fixed order: it depends on nothing but the lane.
__device__ __forceinline__ double warp_scatter16(const double (&v)[16], int lane) {
  double v8[8], v4[4], v2[2];
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4, b1 = lane & 2;
#pragma unroll
  for (int j = 0; j < 8; ++j) v8[j] = (b4 ? v[j + 8] : v[j]) + __shfl_xor_sync(0xffffffffu, b4 ? v[j] : v[j + 8], 16);
#pragma unroll
  for (int j = 0; j < 4; ++j) v4[j] = (b3 ? v8[j + 4] : v8[j]) + __shfl_xor_sync(0xffffffffu, b3 ? v8[j] : v8[j + 4], 8);
#pragma unroll
  for (int j = 0; j < 2; ++j) v2[j] = (b2 ? v4[j + 2] : v4[j]) + __shfl_xor_sync(0xffffffffu, b2 ? v4[j] : v4[j + 2], 4);
  const double v1 = (b1 ? v2[1] : v2[0]) + __shfl_xor_sync(0xffffffffu, b1 ? v2[0] : v2[1], 2);
  return v1 + __shfl_xor_sync(0xffffffffu, v1, 1);
}

constexpr int kRowSweepBlocks = 2;  // resident blocks per SM of the row sweep (register-bound)

// The fused sweep (k_pcg_fused) for fp32 rows of at most 8 values on a 32-byte pitch (R, Z and both
// direction buffers): one thread per row, each row read and written in one 256-bit access per array,
// the reciprocal of the diagonal taken once per row. Same arithmetic per element as k_pcg_fused; the
// per-column sums rz, ss are kept per thread in fp64 and summed over the warp by a reduce-scatter,
// then over the block's warps in order. Padding columns (c >= C) of R and Z are written back as read,
// those of the next direction as zeros (the apply gathers whole rows of it).
__global__ void __launch_bounds__(kSweepThreads, kRowSweepBlocks)
    k_pcg_fused_rows8(int32_t n, int32_t C, float *R, int64_t ldr, float *Z, int64_t ldz, float *buf0,
                      float *buf1, int64_t ld, const float *__restrict__ diag, PcgBufs B) {
  PcgCtl *ctl = B.ctl;
  if (!ctl->go) {
    if (B.has_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(B.cond, 0u);  // loop ends
    return;
  }
  if (B.has_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(B.cond, 0u);
  __shared__ double s_w[kSweepThreads / 32][16];
  __shared__ double s_v[kSweepThreads / 32];
  const bool par = ctl->par != 0;
  const float *P = par ? buf1 : buf0;
  float *AP = par ? buf0 : buf1;  // AP in, the next direction out
  float al[8], be[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    al[c] = c < C ? (float)B.alpha[c] : 0.f;
    be[c] = c < C ? (float)B.beta[c] : 0.f;
  }
  double rz[8], ss[8], rmax[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) rz[c] = ss[c] = rmax[c] = 0.0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const uint64_t pf = l2_evict_first_pol(), pl = l2_evict_last();
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride) {
    float rv[8], av[8], pv[8], zv[8];
    ld_row8(R + r * ldr, rv, pf);
    ld_row8(AP + r * ld, av, pf);
    ld_row8(P + r * ld, pv, pf);
    ld_row8(Z + r * ldz, zv, pf);
    const double dinv = __drcp_rn((double)diag[r]);  // correctly rounded: the value of 1.0 / d
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      if (c < C) {
        const float rn = rv[c] - al[c] * av[c];
        zv[c] = zv[c] + al[c] * pv[c];
        const double r64 = (double)rn;
        // R / diag rounded to fp32 (as in k_pcg_fused)
        av[c] = (float)(r64 * dinv) + be[c] * pv[c];
        rv[c] = rn;
        const double r2 = r64 * r64;
        rz[c] += r2 * dinv;
        ss[c] += r2;
        rmax[c] = fmax(rmax[c], fabs(r64) * dinv);
      } else {
        av[c] = 0.f;
      }
    }
    st_row8(R + r * ldr, rv, pf);
    st_row8(Z + r * ldz, zv, pf);
    st_row8(AP + r * ld, av, pl);
  }
  // fp64 rounding is monotone: max over rows of (|r| / d) times eps^-1 is the max of the products
  double vmax = 0.0;
  bool bad = false;
#pragma unroll
  for (int c = 0; c < 8; ++c)
    if (c < C) {
      vmax = fmax(vmax, rmax[c] * B.epsinv[c]);
      bad = bad || !isfinite(ss[c]);
    }
  if (bad) ctl->bad = 1;
  const int tid = threadIdx.x, lane = lane_id(), wid = tid >> 5;
  double v16[16];
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    v16[c] = rz[c];
    v16[8 + c] = ss[c];
  }
  const double mine = warp_scatter16(v16, lane);
  if ((lane & 1) == 0) s_w[wid][lane >> 1] = mine;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, off));
  if (lane == 0) s_v[wid] = vmax;
  __syncthreads();
  if (tid < 16) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kSweepThreads / 32; ++w) s += s_w[w][tid];
    const int c = tid & 7;
    if (c < C) B.part2[(long long)((tid < 8 ? 0 : C) + c) * B.nbmax + blockIdx.x] = s;
  } else if (tid == 32) {
    double v = 0.0;
    for (int w = 0; w < kSweepThreads / 32; ++w) v = fmax(v, s_v[w]);
    B.part2[(long long)(2 * C) * B.nbmax + blockIdx.x] = v;
  }
  if (last_block_grouped<kSweepThreads>(B.part2, B.nbmax, 2 * C + 1, 2 * C, ctl->gcnt2, &ctl->cnt2, B.gpart2))
    finish_sweep(0, C, B, true);
}

// The zero start of the two-kernel iteration on rows of at most 8 floats on a 32-byte pitch
// (k_pcg_update phase 3 and k_pcg_dir mode 4 in one sweep): R = rhs, Z = 0, P = R / diag, and rz,
// ||R||^2 and the violation of R with the first stop decision (finish_sweep phase 3). One thread per
// row, whole-row accesses; the padding columns of R and Z are written back as read (read only when
// there are any), those of P as zeros. Same arithmetic per element as the two kernels it replaces.
__global__ void __launch_bounds__(kSweepThreads, kRowSweepBlocks)
    k_pcg_start_rows8(int32_t n, int32_t C, const float *__restrict__ rhs, int64_t ldrhs, float *R, int64_t ldr,
                      float *Z, int64_t ldz, float *P, int64_t ldp, const float *__restrict__ diag, PcgBufs B) {
  PcgCtl *ctl = B.ctl;
  __shared__ double s_w[kSweepThreads / 32][16];
  __shared__ double s_v[kSweepThreads / 32];
  double rz[8], ss[8], rmax[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) rz[c] = ss[c] = rmax[c] = 0.0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const uint64_t pf = l2_evict_first_pol(), pl = l2_evict_last();
  const bool pad = C < 8;
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride) {
    float bv[8], rv[8], zv[8], pv[8];
    ld_row8(rhs + r * ldrhs, bv, pf);
    if (pad) {
      ld_row8(R + r * ldr, rv, pf);
      ld_row8(Z + r * ldz, zv, pf);
    }
    const double dinv = __drcp_rn((double)diag[r]);  // correctly rounded: the value of 1.0 / d
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      if (c < C) {
        rv[c] = bv[c];
        zv[c] = 0.f;
        const double r64 = (double)bv[c];
        pv[c] = (float)(r64 * dinv);  // the fp32 quotient R / diag (as in k_pcg_fused)
        const double r2 = r64 * r64;
        rz[c] += r2 * dinv;
        ss[c] += r2;
        rmax[c] = fmax(rmax[c], fabs(r64) * dinv);
      } else {
        pv[c] = 0.f;
      }
    }
    st_row8(R + r * ldr, rv, pf);
    st_row8(Z + r * ldz, zv, pf);
    st_row8(P + r * ldp, pv, pl);
  }
  double vmax = 0.0;
  bool bad = false;
#pragma unroll
  for (int c = 0; c < 8; ++c)
    if (c < C) {
      vmax = fmax(vmax, rmax[c] * B.epsinv[c]);
      bad = bad || !isfinite(ss[c]);
    }
  if (bad) ctl->bad = 1;
  const int tid = threadIdx.x, lane = lane_id(), wid = tid >> 5;
  double v16[16];
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    v16[c] = rz[c];
    v16[8 + c] = ss[c];
  }
  const double mine = warp_scatter16(v16, lane);
  if ((lane & 1) == 0) s_w[wid][lane >> 1] = mine;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, off));
  if (lane == 0) s_v[wid] = vmax;
  __syncthreads();
  if (tid < 16) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < kSweepThreads / 32; ++w) t += s_w[w][tid];
    const int c = tid & 7;
    if (c < C) B.part2[(long long)((tid < 8 ? 0 : C) + c) * B.nbmax + blockIdx.x] = t;
  } else if (tid == 32) {
    double v = 0.0;
    for (int w = 0; w < kSweepThreads / 32; ++w) v = fmax(v, s_v[w]);
    B.part2[(long long)(2 * C) * B.nbmax + blockIdx.x] = v;
  }
  if (last_block_grouped<kSweepThreads>(B.part2, B.nbmax, 2 * C + 1, 2 * C, ctl->gcnt2, &ctl->cnt2, B.gpart2))
    finish_sweep(3, C, B, false);
}

// K3: Z += alpha P; P = R/diag + beta P
//   mode 0: both (skipping the P update when a stop was proposed)   mode 1: P update only
//   mode 2: P = R/diag      mode 4: P = R/diag and Z = 0 (a zero start)
template <typename T>
__global__ void __launch_bounds__(kSweepThreads, (sweep_min_blocks<T>())) k_pcg_dir(int mode, int32_t n, int32_t C, T *__restrict__ Z,
                                                           int64_t ldz, T *P, int64_t ldp,
                                                           const T *__restrict__ R, int64_t ldr,
                                                           const T *__restrict__ diag, PcgBufs B, bf16 *P_lo,
                                                           int64_t ld_lo, T *P2) {
  PcgCtl *ctl = B.ctl;
  if (mode == 0 && !ctl->go) return;
  // two-kernel iteration (P2 = its AP buffer): the new direction goes to the buffer ctl->par names,
  // from the old one in the other (a resume after a failed recheck keeps the reference's beta)
  T *Pin = P, *Pout = P;
  if (P2 && mode == 1) {
    if (ctl->par) Pout = P2;  // direction of the iteration in buf0 = P, the resumed one to buf1
    else Pin = P2;
  }
  const bool upd_p = mode != 0 || ctl->done == 0;
  const SweepIdx ix = sweep_index(ldr, C);
  if (!ix.on) return;
  const int c = ix.c;
  const T al = mode == 0 ? (T)B.alpha[c] : T(0);
  const bool init = mode == 2 || mode == 4;  // P = R/diag: the old P is not read
  const T be = init ? T(0) : (T)B.beta[c];
  const long long zstep = ix.RS * ldz, pstep = ix.RS * ldp, rstep = ix.RS * ldr;
  long long offz = ix.r0 * ldz + c, offp = ix.r0 * ldp + c, offr = ix.r0 * ldr + c;
  for (long long r = ix.r0; r < n; r += kSweepUnroll * ix.RS) {
    // every load of the batch is issued before any store (Z included)
    T pv[kSweepUnroll], rv[kSweepUnroll], dv[kSweepUnroll], zv[kSweepUnroll];
#pragma unroll
    for (int u = 0; u < kSweepUnroll; ++u) {
      const long long rr = r + u * ix.RS;
      const bool ok = rr < n;
      pv[u] = (ok && !init) ? Pin[offp + u * pstep] : T(0);
      zv[u] = (ok && mode == 0) ? Z[offz + u * zstep] : T(0);
      rv[u] = (ok && upd_p) ? R[offr + u * rstep] : T(0);
      dv[u] = (ok && upd_p) ? diag[rr] : T(1);
    }
#pragma unroll
    for (int u = 0; u < kSweepUnroll; ++u) {
      const long long rr = r + u * ix.RS;
      if (rr < n) {
        if (mode == 0) Z[offz + u * zstep] = zv[u] + al * pv[u];
        if (mode == 4) Z[offz + u * zstep] = T(0);
        if (upd_p) {
          const T y = rv[u] / dv[u];
          const T pn = init ? y : y + be * pv[u];
          Pout[offp + u * pstep] = pn;
          if (P_lo) P_lo[rr * ld_lo + c] = cvt<bf16>(pn);
        }
      }
    }
    offz += kSweepUnroll * zstep;
    offp += kSweepUnroll * pstep;
    offr += kSweepUnroll * rstep;
  }
}

// Blocks per SM of a grid-stride kernel that are resident at once: its grid is that many blocks per
// SM (one wave), since a second, partial wave leaves most SMs idle while it drains. Computed once
// per kernel instantiation from the occupancy calculator (first called before any stream capture),
// capped at the kUpdBlocksPerSM blocks per SM the partial-sum buffers hold.
template <class K>
static int resident_per_sm(K *kernel, int threads) {
  int per = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, 0) != cudaSuccess || per < 1) {
    (void)cudaGetLastError();
    per = 1;
  }
  return std::min(per, kUpdBlocksPerSM);
}

// The sweeps need ld <= threads in the grid (at least one row per pass): with one block per SM at
// least, dlp_pcg's check ld <= sm_count() * kSweepThreads covers every grid below.
template <typename TS>
static int update_grid() {
  static const int per = resident_per_sm(k_pcg_update<TS>, kSweepThreads);
  return sm_count() * per;
}
template <typename TS>
static int dir_grid() {
  static const int per = resident_per_sm(k_pcg_dir<TS>, kSweepThreads);
  return sm_count() * per;
}

// ------------------------------------------------------------------------------------------------
// Certification statistics in one sweep: per column max |R|/diag and sum R^2 (and sum rhs^2), plus
// max |H|. Per-thread column as in the PCG sweeps; per-block partials, then one warp per output.
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ double block_column_max(const double *v, int c, int64_t ld) {
  const long long base = (long long)blockIdx.x * blockDim.x;
  const int first = (int)(((c - base % ld) % ld + ld) % ld);
  const int lane = lane_id();
  double s = 0.0;
  for (long long tid = first + (long long)lane * ld; tid < blockDim.x; tid += 32 * ld) s = fmax(s, v[tid]);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) s = fmax(s, __shfl_xor_sync(0xffffffffu, s, off));
  return s;
}

template <typename T>
__global__ void __launch_bounds__(kSweepThreads)
    k_resid_stats(int32_t n, int32_t C, const T *__restrict__ R, int64_t ldr, const T *__restrict__ rhs,
                  int64_t ldrhs, const T *__restrict__ diag, const T *__restrict__ H, int64_t ldh, double *part) {
  __shared__ double s_m[kSweepThreads], s_r[kSweepThreads], s_b[kSweepThreads], s_h[kSweepThreads / 32];
  const SweepIdx ix = sweep_index(ldr, C);
  double mx = 0.0, rr = 0.0, bb = 0.0, hm = 0.0;
  if (ix.on) {
    const int c = ix.c;
    for (long long r = ix.r0; r < n; r += kSweepUnroll * ix.RS) {
      double x[kSweepUnroll], d[kSweepUnroll], b[kSweepUnroll], h[kSweepUnroll];
#pragma unroll
      for (int u = 0; u < kSweepUnroll; ++u) {
        const long long q = r + u * ix.RS;
        const bool ok = q < n;
        x[u] = ok ? (double)R[q * ldr + c] : 0.0;
        d[u] = ok ? (double)diag[q] : 1.0;
        b[u] = (ok && rhs) ? (double)rhs[q * ldrhs + c] : 0.0;
        h[u] = (ok && H && c == 0) ? (double)H[q * ldh] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < kSweepUnroll; ++u) {
        mx = fmax(mx, fabs(x[u]) / d[u]);
        rr = fma(x[u], x[u], rr);
        bb = fma(b[u], b[u], bb);
        hm = fmax(hm, fabs(h[u]));
      }
    }
  }
  const int tid = threadIdx.x, lane = lane_id(), wid = tid >> 5;
  s_m[tid] = mx;
  s_r[tid] = rr;
  s_b[tid] = bb;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) hm = fmax(hm, __shfl_xor_sync(0xffffffffu, hm, off));
  if (lane == 0) s_h[wid] = hm;
  __syncthreads();
  const int NO = 3 * C + 1;
  for (int c = wid; c < C; c += kSweepThreads / 32) {
    const double a = block_column_max(s_m, c, ldr);
    const double b = block_column_sum(s_r, c, ldr);
    const double e = block_column_sum(s_b, c, ldr);
    if (lane == 0) {
      part[(long long)blockIdx.x * NO + c] = a;
      part[(long long)blockIdx.x * NO + C + c] = b;
      part[(long long)blockIdx.x * NO + 2 * C + c] = e;
    }
  }
  if (tid == 0) {
    double v = 0.0;
    for (int w = 0; w < kSweepThreads / 32; ++w) v = fmax(v, s_h[w]);
    part[(long long)blockIdx.x * NO + 3 * C] = v;
  }
}

// The same statistics for fp64 residuals of at most 10 columns whose rows are whole 16-byte aligned
// runs of 10 doubles (ld >= 10): one thread per row, the row read in three loads (load_row10d) and
// the diagonal's reciprocal taken once per row (|R| times the correctly rounded reciprocal is
// within 2 ulp of the quotient); rhs per column (its whole rows cost the kernel a spill).
// Per-thread column sums in order, then a fixed xor tree over the warp and the warps in order,
// written in k_resid_stats's partials layout for k_resid_stats_final.
__global__ void __launch_bounds__(kSweepThreads, 2)
    k_resid_stats_rows10(int32_t n, int32_t C, const double *__restrict__ R, int64_t ldr,
                         const double *__restrict__ rhs, int64_t ldrhs, const double *__restrict__ diag,
                         const double *__restrict__ H, int64_t ldh, double *part) {
  double mx[10], rr[10], bb[10];
#pragma unroll
  for (int c = 0; c < 10; ++c) mx[c] = rr[c] = bb[c] = 0.0;
  double hm = 0.0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride) {
    double raw[5][2];
    const bool hi = load_row10d(R + r * ldr, raw);
    const double dinv = __drcp_rn(diag[r]);
#pragma unroll
    for (int c = 0; c < 10; ++c) {
      if (c < C) {
        const double x = row10_col(raw, hi, c);
        mx[c] = fmax(mx[c], fabs(x) * dinv);
        rr[c] = fma(x, x, rr[c]);
      }
    }
    if (rhs) {
#pragma unroll
      for (int c = 0; c < 10; ++c)
        if (c < C) {
          const double b = rhs[r * ldrhs + c];
          bb[c] = fma(b, b, bb[c]);
        }
    }
    if (H) hm = fmax(hm, fabs(H[r * ldh]));
  }
  __shared__ double s_w[kSweepThreads / 32][31];
  const int tid = threadIdx.x, lane = lane_id(), wid = tid >> 5;
  const int NO = 3 * C + 1;
#pragma unroll
  for (int c = 0; c < 10; ++c) {
    double a = mx[c], b = rr[c], e = bb[c];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      a = fmax(a, __shfl_xor_sync(0xffffffffu, a, off));
      b += __shfl_xor_sync(0xffffffffu, b, off);
      e += __shfl_xor_sync(0xffffffffu, e, off);
    }
    if (lane == 0 && c < C) {
      s_w[wid][c] = a;
      s_w[wid][C + c] = b;
      s_w[wid][2 * C + c] = e;
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) hm = fmax(hm, __shfl_xor_sync(0xffffffffu, hm, off));
  if (lane == 0) s_w[wid][3 * C] = hm;
  __syncthreads();
  for (int o = tid; o < NO; o += blockDim.x) {
    const bool is_max = o < C || o == 3 * C;
    double v = 0.0;
#pragma unroll
    for (int w = 0; w < kSweepThreads / 32; ++w) v = is_max ? fmax(v, s_w[w][o]) : v + s_w[w][o];
    part[(long long)blockIdx.x * NO + o] = v;
  }
}

__global__ void k_resid_stats_final(int32_t C, int nb, const double *__restrict__ part, double *out) {
  const int o = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int NO = 3 * C + 1;
  if (o >= NO) return;
  const bool is_max = o < C || o == 3 * C;
  const double v = warp_strided_reduce(part + o, NO, nb, is_max);
  if ((threadIdx.x & 31) == 0) out[o] = v;
}

// ------------------------------------------------------------------------------------------------
// host driver
// ------------------------------------------------------------------------------------------------
struct PcgProblem {
  const int32_t *rbeg, *rend, *col;
  const void *w;
  int w_dtype;
  int32_t n, C;
  const void *diag, *rhs;
  int64_t ldrhs;
  void *Z;
  int64_t ldz;
  void *R;
  int64_t ldr;
  void *P;
  int64_t ldp;
  void *AP;
  int64_t ldap;
  int dtype;
  double avg_deg;
  const void *w_lo;  // bf16 weights and the bf16 mirror of P (NULL: full precision gathers)
  void *P_lo;
  int64_t ld_lo;
  bool fused;  // the two-kernel iteration (fp32 whole rows, P and AP trade places)
  bool rows8;  // its sweep one row per thread (rows of at most 8 floats on a 32-byte pitch)
};

template <class T, bool FUSE = false>
static int launch_apply(const PcgProblem &q, const PcgBufs &B, cudaStream_t s, bool launch = true) {
  Layout L;
  const bool lo = sizeof(typename T::TX) == 2;
  const void *X = lo ? q.P_lo : q.P;
  const int64_t ldx = lo ? q.ld_lo : q.ldp;
  DLP_TRY(choose_layout(q.C, sizeof(typename T::TX), X, ldx, 0, q.avg_deg, &L));
  ApplyArgs<T> a{q.rbeg, q.rend, q.col, (const typename T::TW *)(lo ? q.w_lo : q.w), q.n, q.C,
                 (const typename T::TX *)X, ldx, (const typename T::TV *)q.diag, (typename T::TY *)q.AP, q.ldap, B,
                 L.G, L.LV, L.NV, lo ? (const typename T::TV *)q.P : nullptr, q.ldp,
                 (int)(q.ldap >= 12 && q.ldap % 4 == 0 && (uintptr_t)q.AP % 16 == 0)};
  constexpr int VWV = 16 / sizeof(typename T::TX);
  // launch == false only fills the one-wave grid cache (outside stream capture)
#define DLP_APPLY_ONE(VW_, VPL_)                                                        \
  case VPL_: {                                                                          \
    static const int per = resident_per_sm(k_pcg_apply<T, VW_, VPL_>, kThreads);       \
    if (launch) k_pcg_apply<T, VW_, VPL_><<<sm_count() * per, kThreads, 0, s>>>(a);     \
    break;                                                                              \
  }
#define DLP_APPLY_CASE(VW_)                                                             \
  switch (L.VPL) {                                                                      \
    DLP_APPLY_ONE(VW_, 1)                                                               \
    DLP_APPLY_ONE(VW_, 2)                                                               \
    DLP_APPLY_ONE(VW_, 3)                                                               \
    DLP_APPLY_ONE(VW_, 4)                                                               \
    DLP_APPLY_ONE(VW_, 8)                                                               \
    default: return DLP_ERR_INVALID;                                                    \
  }
  constexpr bool f32 = std::is_same<typename T::TX, float>::value && std::is_same<typename T::TA, float>::value;
  // whole fp32 rows held by one lane: 12 floats in two loads (load_row12) or 8 in one (load_row8)
  const bool w12 = f32 && L.VW == 4 && L.VPL == 3 && L.LV == 1;
  const bool w8 = f32 && L.VW == 4 && L.VPL == 2 && L.LV == 1 && (uintptr_t)X % 32 == 0 && ldx % 8 == 0 &&
                  (uintptr_t)q.AP % 32 == 0 && q.ldap % 8 == 0;
  if (w8) a.ap_row12 = 1;  // the 8-float AP row in one 256-bit store
  if constexpr (f32) {
    if constexpr (FUSE) {
      if (!(w12 || w8) || q.ldp != q.ldap) return DLP_ERR_INVALID;
      if (w8) {
        static const int per = resident_per_sm(k_pcg_apply<T, VWV, 2, kRow8F, true>, kThreads);
        if (launch) k_pcg_apply<T, VWV, 2, kRow8F, true><<<sm_count() * per, kThreads, 0, s>>>(a);
      } else {
        static const int per = resident_per_sm(k_pcg_apply<T, VWV, 3, kRow12F, true>, kThreads);
        if (launch) k_pcg_apply<T, VWV, 3, kRow12F, true><<<sm_count() * per, kThreads, 0, s>>>(a);
      }
      return launch ? check_launch() : DLP_OK;
    }
    if (w12) {
      static const int per = resident_per_sm(k_pcg_apply<T, VWV, 3, kRow12F>, kThreads);
      if (launch) k_pcg_apply<T, VWV, 3, kRow12F><<<sm_count() * per, kThreads, 0, s>>>(a);
      return launch ? check_launch() : DLP_OK;
    }
    if (w8) {
      static const int per = resident_per_sm(k_pcg_apply<T, VWV, 2, kRow8F>, kThreads);
      if (launch) k_pcg_apply<T, VWV, 2, kRow8F><<<sm_count() * per, kThreads, 0, s>>>(a);
      return launch ? check_launch() : DLP_OK;
    }
  } else if constexpr (FUSE) {
    return DLP_ERR_INVALID;
  }
  if (L.VW == 1) {
    DLP_APPLY_CASE(1)
  } else {
    DLP_APPLY_CASE(VWV)
  }
#undef DLP_APPLY_CASE
#undef DLP_APPLY_ONE
  return launch ? check_launch() : DLP_OK;
}

// src (phase 3 only): the array the initial residual is copied from, in place of AP
template <typename TS>
static int launch_update(int phase, const PcgProblem &q, const PcgBufs &B, cudaStream_t s,
                         const void *src = nullptr, int64_t ldsrc = 0) {
  const TS *ap = phase == 3 ? (const TS *)src : (const TS *)q.AP;
  const int64_t ldap = phase == 3 ? ldsrc : q.ldap;
  k_pcg_update<TS><<<update_grid<TS>(), kSweepThreads, 0, s>>>(phase, q.n, q.C, (TS *)q.R, q.ldr, ap, ldap,
                                                            (const TS *)q.diag, B);
  return check_launch();
}

template <typename TS>
static int launch_dir(int mode, const PcgProblem &q, const PcgBufs &B, cudaStream_t s) {
  k_pcg_dir<TS><<<dir_grid<TS>(), kSweepThreads, 0, s>>>(mode, q.n, q.C, (TS *)q.Z, q.ldz, (TS *)q.P, q.ldp,
                                                         (const TS *)q.R, q.ldr, (const TS *)q.diag, B,
                                                         (bf16 *)q.P_lo, q.ld_lo, q.fused ? (TS *)q.AP : nullptr);
  return check_launch();
}

static int fused_grid(bool rows8) {
  static const int per = resident_per_sm(k_pcg_fused<float>, kSweepThreads);
  static const int per_rows = resident_per_sm(k_pcg_fused_rows8, kSweepThreads);
  return sm_count() * (rows8 ? per_rows : per);
}

static int launch_fused(const PcgProblem &q, const PcgBufs &B, cudaStream_t s) {
  if (q.rows8) {
    k_pcg_fused_rows8<<<fused_grid(true), kSweepThreads, 0, s>>>(q.n, q.C, (float *)q.R, q.ldr, (float *)q.Z,
                                                                 q.ldz, (float *)q.P, (float *)q.AP, q.ldp,
                                                                 (const float *)q.diag, B);
  } else {
    k_pcg_fused<float><<<fused_grid(false), kSweepThreads, 0, s>>>(q.n, q.C, (float *)q.R, q.ldr, (float *)q.Z,
                                                                   q.ldz, (float *)q.P, (float *)q.AP, q.ldp,
                                                                   (const float *)q.diag, B);
  }
  return check_launch();
}

static int iteration(const PcgProblem &q, const PcgBufs &B, cudaStream_t s) {
  if (q.fused) {
    DLP_TRY((launch_apply<T_F32, true>(q, B, s)));
    return launch_fused(q, B, s);
  }
  if (q.dtype == DLP_F32) {
    if (q.w_lo) DLP_TRY(launch_apply<T_BF16F>(q, B, s));
    else DLP_TRY(launch_apply<T_F32>(q, B, s));
    DLP_TRY(launch_update<float>(0, q, B, s));
    return launch_dir<float>(0, q, B, s);
  }
  if (q.w_dtype == DLP_F64) DLP_TRY(launch_apply<T_F64>(q, B, s));
  else DLP_TRY(launch_apply<T_W32X64>(q, B, s));
  DLP_TRY(launch_update<double>(0, q, B, s));
  return launch_dir<double>(0, q, B, s);
}

// Fills the one-wave grid caches of the kernels iteration() launches, without launching.
static int prime_grids(const PcgProblem &q, const PcgBufs &B, cudaStream_t s) {
  if (q.fused) {
    (void)fused_grid(q.rows8);
    return launch_apply<T_F32, true>(q, B, s, false);
  }
  if (q.dtype == DLP_F32) {
    (void)update_grid<float>();
    (void)dir_grid<float>();
    return q.w_lo ? launch_apply<T_BF16F>(q, B, s, false) : launch_apply<T_F32>(q, B, s, false);
  }
  (void)update_grid<double>();
  (void)dir_grid<double>();
  return q.w_dtype == DLP_F64 ? launch_apply<T_F64>(q, B, s, false) : launch_apply<T_W32X64>(q, B, s, false);
}

static int true_residual(const PcgProblem &q, cudaStream_t s) {
  // R = rhs - diag*Z + W Z
  return dlp_spmm(q.rbeg, q.rend, q.col, q.w, q.w_dtype, q.n, nullptr, q.C, q.Z, q.ldz, q.dtype, q.diag, -1.0,
                  1.0, q.rhs, q.ldrhs, 1.0, q.R, q.ldr, q.dtype, 0, 0, q.avg_deg, (dlp_stream_t)s);
}

static int update_phase(int phase, const PcgProblem &q, const PcgBufs &B, cudaStream_t s) {
  return q.dtype == DLP_F32 ? launch_update<float>(phase, q, B, s) : launch_update<double>(phase, q, B, s);
}

// the initial phase of a zero start: R = rhs in the same sweep as the initial reductions
static int update_from_rhs(const PcgProblem &q, const PcgBufs &B, cudaStream_t s) {
  return q.dtype == DLP_F32 ? launch_update<float>(3, q, B, s, q.rhs, q.ldrhs)
                            : launch_update<double>(3, q, B, s, q.rhs, q.ldrhs);
}

static int dir_phase(int mode, const PcgProblem &q, const PcgBufs &B, cudaStream_t s) {
  return q.dtype == DLP_F32 ? launch_dir<float>(mode, q, B, s) : launch_dir<double>(mode, q, B, s);
}

// The zero start: R = rhs with its reductions and the first decision, then Z = 0 and P = R / diag;
// one row sweep where the rows allow it (k_pcg_start_rows8), else the two element sweeps.
static int zero_start(const PcgProblem &q, const PcgBufs &B, cudaStream_t s) {
  if (q.rows8 && (uintptr_t)q.rhs % 32 == 0 && q.ldrhs % 8 == 0) {
    static const int per = resident_per_sm(k_pcg_start_rows8, kSweepThreads);
    k_pcg_start_rows8<<<sm_count() * per, kSweepThreads, 0, s>>>(q.n, q.C, (const float *)q.rhs, q.ldrhs,
                                                                 (float *)q.R, q.ldr, (float *)q.Z, q.ldz,
                                                                 (float *)q.P, q.ldp, (const float *)q.diag, B);
    return check_launch();
  }
  DLP_TRY(update_from_rhs(q, B, s));
  return dir_phase(4, q, B, s);
}

// Graph cache: one instantiated chunk of `k` iterations per problem signature.
struct GraphKey {
  std::vector<uintptr_t> v;
  bool operator==(const GraphKey &o) const { return v == o.v; }
};
struct GraphKeyHash {
  size_t operator()(const GraphKey &k) const {
    size_t h = 1469598103934665603ull;
    for (auto x : k.v) h = (h ^ x) * 1099511628211ull;
    return h;
  }
};

static std::mutex g_graph_mu;
static std::unordered_map<GraphKey, GraphRef, GraphKeyHash> g_graphs;
static cudaStream_t g_capture_stream[64];

static int graph_key(const PcgProblem &q, const PcgBufs &B, int k, GraphKey *key) {
  int dev = 0;
  DLP_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return DLP_ERR_INVALID;
  // the mean degree enters the kernels only through the gather layout it selects: key on that, so
  // a graph whose entry count drifts from batch to batch keeps its instantiated chunk
  Layout L;
  {
    const bool lo = q.w_lo != nullptr;
    const size_t xs = lo ? 2 : (q.dtype == DLP_F32 ? 4 : 8);
    DLP_TRY(choose_layout(q.C, xs, lo ? q.P_lo : q.P, lo ? q.ld_lo : q.ldp, 0, q.avg_deg, &L));
  }
  *key = GraphKey{{(uintptr_t)dev, (uintptr_t)q.rbeg, (uintptr_t)q.rend, (uintptr_t)q.col, (uintptr_t)q.w,
                   (uintptr_t)q.w_dtype, (uintptr_t)q.n, (uintptr_t)q.C, (uintptr_t)q.diag, (uintptr_t)q.Z,
                   (uintptr_t)q.ldz, (uintptr_t)q.R, (uintptr_t)q.ldr, (uintptr_t)q.P, (uintptr_t)q.ldp,
                   (uintptr_t)q.AP, (uintptr_t)q.ldap, (uintptr_t)q.dtype, (uintptr_t)B.ctl, (uintptr_t)k,
                   (uintptr_t)q.w_lo, (uintptr_t)q.P_lo, (uintptr_t)q.ld_lo, (uintptr_t)L.G, (uintptr_t)L.LV,
                   (uintptr_t)L.VW, (uintptr_t)L.VPL, (uintptr_t)B.cancel, (uintptr_t)q.fused}};
  return DLP_OK;
}

static cudaStream_t capture_stream(int dev, int *st) {
  *st = DLP_OK;
  if (!g_capture_stream[dev]) {
    const cudaError_t e = cudaStreamCreateWithFlags(&g_capture_stream[dev], cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      set_cuda_error(e);
      *st = DLP_ERR_CUDA;
    }
  }
  return g_capture_stream[dev];
}

static int get_chunk_graph(const PcgProblem &q, const PcgBufs &B, int k, GraphRef *out) {
  GraphKey key;
  DLP_TRY(graph_key(q, B, k, &key));
  const int dev = (int)key.v[0];
  std::lock_guard<std::mutex> lk(g_graph_mu);
  auto it = g_graphs.find(key);
  if (it != g_graphs.end()) {
    *out = it->second;
    return DLP_OK;
  }
  int st = DLP_OK;
  cudaStream_t cs = capture_stream(dev, &st);
  DLP_TRY(st);
  DLP_TRY(prime_grids(q, B, cs));  // occupancy queries stay out of the capture
  DLP_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  for (int i = 0; i < k && st == DLP_OK; ++i) st = iteration(q, B, cs);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(cs, &g);
  if (st != DLP_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  if (e != cudaSuccess) {
    set_cuda_error(e);
    return DLP_ERR_CUDA;
  }
  cudaGraphExec_t ex = nullptr;
  e = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    set_cuda_error(e);
    return DLP_ERR_CUDA;
  }
  auto ref = std::make_shared<GraphExec>();
  ref->ex = ex;
  if (g_graphs.size() >= 32) g_graphs.clear();  // bounded cache; holders keep their graphs alive
  g_graphs.emplace(key, ref);
  *out = ref;
  return DLP_OK;
}

// The whole iteration loop as one graph: a WHILE conditional node whose body is kLoopBody
// iterations (K1, K2, K3 each); every K2 clears the loop flag and its last block sets it again while
// the solve runs, and a K2 that finds the stop already decided returns with the flag cleared, so the
// body repeats at most until the iteration cap. One launch and one read of the control block replace
// the chunk launches and their round trips; at most kLoopBody - 1 iterations run past the stop (as
// no-op launches). Measured on B200 (n = 1M, degree 10, C = 9, 17-18 iterations per solve): with two
// iterations per body the median batch latency is about 2% below that of 8-iteration chunk graphs,
// and one iteration per body is slower than both (each pass of the WHILE node costs a few us).
constexpr int kLoopBody = 2;

static int get_loop_graph(const PcgProblem &q, const PcgBufs &B, GraphRef *out) {
  GraphKey key;
  DLP_TRY(graph_key(q, B, -1, &key));
  const int dev = (int)key.v[0];
  std::lock_guard<std::mutex> lk(g_graph_mu);
  auto it = g_graphs.find(key);
  if (it != g_graphs.end()) {
    *out = it->second;
    return DLP_OK;
  }
  int st = DLP_OK;
  cudaStream_t cs = capture_stream(dev, &st);
  DLP_TRY(st);
  DLP_TRY(prime_grids(q, B, cs));  // occupancy queries stay out of the capture
  cudaGraph_t g = nullptr;
  DLP_CUDA(cudaGraphCreate(&g, 0));
  auto fail = [&](cudaError_t e) {
    cudaGraphDestroy(g);
    set_cuda_error(e);
    return DLP_ERR_CUDA;
  };
  cudaGraphConditionalHandle h = 0;
  cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 1u, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) return fail(e);
  cudaGraphNodeParams np{};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node = nullptr;
  e = cudaGraphAddNode(&node, g, nullptr, 0, &np);
  if (e != cudaSuccess) return fail(e);
  cudaGraph_t body = np.conditional.phGraph_out[0];
  PcgBufs Bc = B;
  Bc.has_cond = 1;
  Bc.cond = h;
  e = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return fail(e);
  for (int i = 0; i < kLoopBody && st == DLP_OK; ++i) st = iteration(q, Bc, cs);
  cudaGraph_t captured = nullptr;
  e = cudaStreamEndCapture(cs, &captured);
  if (st != DLP_OK) {
    cudaGraphDestroy(g);
    return st;
  }
  if (e != cudaSuccess) return fail(e);
  cudaGraphExec_t ex = nullptr;
  e = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    set_cuda_error(e);
    return DLP_ERR_CUDA;
  }
  auto ref = std::make_shared<GraphExec>();
  ref->ex = ex;
  if (g_graphs.size() >= 32) g_graphs.clear();  // bounded cache; holders keep their graphs alive
  g_graphs.emplace(key, ref);
  *out = ref;
  return DLP_OK;
}

}  // namespace dlp

using namespace dlp;

extern "C" {

size_t dlp_pcg_workspace_bytes(int32_t C) { return pcg_ws_bytes(C > 0 ? C : 1); }

int dlp_pcg(const int32_t *rbeg, const int32_t *rend, const int32_t *col, const void *w, int w_dtype, int32_t n,
            int32_t C, const void *diag, const void *rhs, int64_t ldrhs, void *Z, int64_t ldz, void *R, int64_t ldr,
            void *P, int64_t ldp, void *AP, int64_t ldap, int dtype, const double *eps, const double *rhs_norm,
            double target_relres, int32_t mode, int32_t max_iter, int32_t patience, int32_t check_every,
            int32_t use_graph, double avg_deg, void *ws, size_t ws_bytes, int32_t *iters_out, double *viol_out,
            double *relres_out, int32_t *status_out, dlp_stream_t stream, const void *w_lo, void *P_lo,
            int64_t ld_lo) {
  if (n < 0 || C <= 0 || C > 256 || ldz < C || ldr < C || ldp < C || ldap < C || ldrhs < C) return DLP_ERR_INVALID;
  if (ldr > (int64_t)sm_count() * kSweepThreads) return DLP_ERR_INVALID;
  if ((w_lo || P_lo) && (!w_lo || !P_lo || ld_lo < C || dtype != DLP_F32)) return DLP_ERR_INVALID;
  if ((mode & 3) == 0 || mode > 31 || ((mode & 1) && !eps) || ((mode & 2) && !rhs_norm)) return DLP_ERR_INVALID;
  if (!(dtype == DLP_F32 && w_dtype == DLP_F32) && !(dtype == DLP_F64 && (w_dtype == DLP_F64 || w_dtype == DLP_F32)))
    return DLP_ERR_DTYPE;
  if (!ws || ws_bytes < pcg_ws_bytes(C)) return DLP_ERR_WORKSPACE;
  // the grid reductions' group counters cover grids of up to kGroup * kMaxGroups blocks
  if (std::max(upd_blocks(), apply_blocks()) > kGroup * kMaxGroups) return DLP_ERR_INVALID;
  if (n == 0) {
    if (iters_out) *iters_out = 0;
    if (status_out) *status_out = 5;
    return DLP_OK;
  }
  cudaStream_t s = (cudaStream_t)stream;
  PcgProblem q{rbeg, rend, col, w, w_dtype, n, C, diag, rhs, ldrhs, Z, ldz, R, ldr, P, ldp, AP, ldap, dtype, avg_deg,
               w_lo, P_lo, ld_lo, false, false};
  if (dtype == DLP_F32 && w_dtype == DLP_F32 && !w_lo && !(mode & 8) && ldp == ldap &&
      (uintptr_t)AP % 16 == 0) {
    // the two-kernel iteration where the apply takes the fp32 whole-row path for P and for AP
    Layout L;
    DLP_TRY(choose_layout(C, sizeof(float), P, ldp, 0, avg_deg, &L));
    q.fused = (L.VW == 4 && L.VPL == 3 && L.LV == 1 && ldap >= 12 && ldap % 4 == 0) ||
              (L.VW == 4 && L.VPL == 2 && L.LV == 1 && ldp % 8 == 0 && (uintptr_t)P % 32 == 0 &&
               (uintptr_t)AP % 32 == 0);
    auto rows8 = [](const void *a, int64_t lda) { return (uintptr_t)a % 32 == 0 && lda % 8 == 0; };
    q.rows8 = q.fused && L.VPL == 2 && C <= 8 && rows8(P, ldp) && rows8(AP, ldap) && rows8(R, ldr) && rows8(Z, ldz);
  }
  PcgBufs B = carve(ws, C);
  B.cancel = cancel_word();
  int dev = 0;
  DLP_CUDA(cudaGetDevice(&dev));
  HostStage *hs = nullptr;
  DLP_TRY(stage_get(dev, head_bytes(C), &hs));
  {
    // the head in one upload: control block; alpha, beta, rz, rzprev zero; eps, its inverse and the
    // rhs norms (zero without them)
    char *img = hs->img;
    std::memset(img, 0, head_bytes(C));
    PcgCtl h{};
    h.mode = mode & 3;
    h.patience = patience > 0 ? patience : 400;
    h.max_iter = max_iter;
    h.target = target_relres;
    std::memcpy(img, &h, sizeof(h));
    auto vec = [&](int i) { return (double *)(img + align256(sizeof(PcgCtl)) + i * align256(sizeof(double) * C)); };
    double *e = vec(3), *rn = vec(4), *ei = vec(5);
    for (int c = 0; c < C; ++c) {
      e[c] = eps ? eps[c] : 1e300;
      ei[c] = 1.0 / e[c];
      rn[c] = rhs_norm ? rhs_norm[c] : 0.0;
    }
    DLP_CUDA(cudaMemcpyAsync(B.ctl, img, head_bytes(C), cudaMemcpyHostToDevice, s));
    DLP_CUDA(cudaEventRecord(hs->up, s));
  }
  // R = rhs - A Z, best = violation, rz = R.(R/diag), P = R/diag; a zero start takes R = rhs in the
  // update sweep itself and sets Z = 0 in the direction sweep (no SpMM, no separate copy)
  if (mode & 4) {
    DLP_TRY(zero_start(q, B, s));
  } else {
    DLP_TRY(true_residual(q, s));
    DLP_TRY(update_phase(2, q, B, s));
    DLP_TRY(dir_phase(2, q, B, s));
  }
  const int k = check_every > 0 ? check_every : 8;
  // graphs: the device-side loop, else (a driver without conditional nodes) chunks of k iterations
  GraphRef lref, gref;
  if (use_graph && get_loop_graph(q, B, &lref) != DLP_OK) {
    (void)cudaGetLastError();
    lref.reset();
  }
  if (use_graph && !lref) DLP_TRY(get_chunk_graph(q, B, k, &gref));
  cudaGraphExec_t lex = lref ? lref->ex : nullptr;
  cudaGraphExec_t ex = gref ? gref->ex : nullptr;
  PcgCtl cur{};
  if (max_iter <= 0) {
    DLP_TRY(read_ctl(B, hs, s, &cur));
    if (cur.done == 0) cur.done = 3;
  }
  // otherwise the first chunk goes out without a round trip: when the start already meets the
  // stop rule, its kernels see ctl->done and return at once
  while ((cur.done == 0 || cur.done == 1) && !cur.bad) {
    const int it0 = cur.iters;
    bool looped = false;
    if (cur.done == 0) {
      if (lex) {
        DLP_CUDA(cudaGraphLaunch(lex, s));
        looped = true;
      } else if (ex) {
        DLP_CUDA(cudaGraphLaunch(ex, s));
        note_launches(3ull * k);
      } else {
        for (int i = 0; i < k; ++i) DLP_TRY(iteration(q, B, s));
      }
    } else if (mode & 16) {
      cur.done = 5;  // the caller confirms the stop on a residual of its own (no recheck here)
      break;
    } else {
      // a stop was proposed: recheck on the true residual (dynlp/solvers.py:85-89)
      DLP_TRY(true_residual(q, s));
      DLP_TRY(update_phase(1, q, B, s));
      DLP_TRY(read_ctl(B, hs, s, &cur));
      if (cur.done != 0) break;
      DLP_TRY(dir_phase(1, q, B, s));  // resume from the true residual
    }
    DLP_TRY(read_ctl(B, hs, s, &cur));
    if (looped) {
      const int passes = std::max((cur.iters - it0 + kLoopBody - 1) / kLoopBody, 1);  // loop bodies run
      note_launches(3ull * kLoopBody * (unsigned long long)passes);
      if (cur.done == 0 && cur.iters == it0) return DLP_ERR_DEVICE;  // the loop stopped without a decision
    }
  }
  if (iters_out) *iters_out = cur.iters;
  if (viol_out) *viol_out = cur.viol;
  if (relres_out) *relres_out = cur.relres;
  if (status_out) *status_out = cur.done;
  if (cur.done == 3) return DLP_ERR_CAP;
  if (cur.done == 6) return DLP_ERR_CANCELLED;
  return DLP_OK;
}

size_t dlp_residual_stats_workspace_bytes(int32_t C) {
  return (size_t)upd_blocks() * (size_t)(3 * (C > 0 ? C : 1) + 1) * sizeof(double);
}

int dlp_residual_stats(int32_t n, int32_t C, const void *R, int64_t ldr, const void *rhs, int64_t ldrhs,
                       const void *diag, const void *H, int64_t ldh, int dtype, double *out, void *ws,
                       size_t ws_bytes, dlp_stream_t stream) {
  if (n < 0 || C <= 0 || ldr < C || (rhs && ldrhs < C) || !out || (n > 0 && (!R || !diag))) return DLP_ERR_INVALID;
  if (ldr > (int64_t)sm_count() * kSweepThreads) return DLP_ERR_INVALID;
  if (dtype != DLP_F32 && dtype != DLP_F64) return DLP_ERR_DTYPE;
  if (!ws || ws_bytes < dlp_residual_stats_workspace_bytes(C)) return DLP_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  static const int per32 = resident_per_sm(k_resid_stats<float>, kSweepThreads);
  static const int per64 = resident_per_sm(k_resid_stats<double>, kSweepThreads);
  const int nb = sm_count() * (dtype == DLP_F32 ? per32 : per64);  // one wave, <= upd_blocks()
  double *part = (double *)ws;
  auto rows10 = [](const void *a, int64_t lda) { return (uintptr_t)a % 16 == 0 && lda >= 10 && lda % 2 == 0; };
  int nbu = nb;
  if (dtype == DLP_F64 && C <= 10 && rows10(R, ldr)) {
    // whole fp64 rows, one per thread (the decision rests on R alone, so calls with and without rhs
    // sum R in the same order)
    static const int per_rows = resident_per_sm(k_resid_stats_rows10, kSweepThreads);
    nbu = std::min(sm_count() * per_rows, nb);
    k_resid_stats_rows10<<<nbu, kSweepThreads, 0, s>>>(n, C, (const double *)R, ldr, (const double *)rhs, ldrhs,
                                                        (const double *)diag, (const double *)H, ldh, part);
  } else if (dtype == DLP_F32) {
    k_resid_stats<float><<<nb, kSweepThreads, 0, s>>>(n, C, (const float *)R, ldr, (const float *)rhs, ldrhs,
                                                       (const float *)diag, (const float *)H, ldh, part);
  } else {
    k_resid_stats<double><<<nb, kSweepThreads, 0, s>>>(n, C, (const double *)R, ldr, (const double *)rhs, ldrhs,
                                                        (const double *)diag, (const double *)H, ldh, part);
  }
  const int NO = 3 * C + 1;
  k_resid_stats_final<<<(NO + 7) / 8, 256, 0, s>>>(C, nbu, part, out);
  return check_launch(2);
}

}  // extern "C"
