// Many independent harmonic solves in one launch sequence: block PCG over a concatenated
// (block-diagonal) CSR where every instance keeps its own CG scalars and stop state, so each
// instance follows the iterates it would follow alone.
//
// Rows are cut into tiles that never straddle two instances. Every kernel walks the tile list;
// reductions go tile -> instance in a fixed order (tile partials, then one block per instance),
// so an instance's sums do not depend on what else is in the batch. Instances stop independently
// (relative residual and/or the reference's violation rule, a true-residual recheck, patience,
// iteration cap) and stopped instances are skipped by the next iterations. Per iteration: select,
// apply (SpMM + pAp), instance reduce (alpha), update (R, rz, norms), instance reduce (beta, stop),
// direction (Z, P); a chunk of iterations is replayed as a CUDA graph.
#include <cstdio>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "gather.cuh"

namespace dlp {

struct BCtl {
  int32_t *done, *iters, *stall, *stopped, *sel;  // per instance
  double *best, *viol, *relres;                    // per instance
  double *alpha, *beta, *rz, *eps, *epsinv, *rhsn;  // per instance x C
  double *tp1, *tp2, *tpv;                          // tile partials
  int32_t *counts;                                  // [running, proposed]
};

struct BTiles {
  const int32_t *tinst, *tbeg, *tend;  // per tile
  const int32_t *toff;                 // tiles of instance i: [toff[i], toff[i+1])
  int32_t ntiles, ninst;
};

struct BParams {
  int32_t mode, patience, max_iter;
  double target;
};

static size_t a256(size_t x) { return (x + 255) / 256 * 256; }

static size_t bctl_bytes(int32_t B, int32_t T, int32_t C) {
  return 5 * a256(4 * (size_t)B) + 3 * a256(8 * (size_t)B) + 6 * a256(8 * (size_t)B * C) + a256(8 * (size_t)T * C) +
         a256(16 * (size_t)T * C) + a256(8 * (size_t)T) + a256(8);
}

static BCtl carve_b(void *ws, int32_t B, int32_t T, int32_t C) {
  char *p = (char *)ws;
  BCtl c;
  int32_t **ip[5] = {&c.done, &c.iters, &c.stall, &c.stopped, &c.sel};
  for (auto q : ip) {
    *q = (int32_t *)p;
    p += a256(4 * (size_t)B);
  }
  double **dp[3] = {&c.best, &c.viol, &c.relres};
  for (auto q : dp) {
    *q = (double *)p;
    p += a256(8 * (size_t)B);
  }
  double **cp[6] = {&c.alpha, &c.beta, &c.rz, &c.eps, &c.epsinv, &c.rhsn};
  for (auto q : cp) {
    *q = (double *)p;
    p += a256(8 * (size_t)B * C);
  }
  c.tp1 = (double *)p;
  p += a256(8 * (size_t)T * C);
  c.tp2 = (double *)p;
  p += a256(16 * (size_t)T * C);
  c.tpv = (double *)p;
  p += a256(8 * (size_t)T);
  c.counts = (int32_t *)p;
  return c;
}

// phase 0: running instances; phase 1: proposed stops; phase 2: all (initial residual)
__global__ void k_b_select(int32_t B, int phase, BCtl c) {
  __shared__ int s_run, s_prop;
  if (threadIdx.x == 0) s_run = s_prop = 0;
  __syncthreads();
  int run = 0, prop = 0;
  for (int i = threadIdx.x; i < B; i += blockDim.x) {
    const int d = c.done[i];
    run += d == 0;
    prop += d == 1;
    c.sel[i] = phase == 2 ? 1 : phase == 1 ? (d == 1) : (d == 0);
  }
  atomicAdd(&s_run, run);
  atomicAdd(&s_prop, prop);
  __syncthreads();
  if (threadIdx.x == 0) {
    c.counts[0] = s_run;
    c.counts[1] = s_prop;
  }
}

template <class T>
struct BApply {
  const int32_t *indptr, *col;
  const typename T::TW *w;
  int32_t C;
  const typename T::TX *P;
  int64_t ldp;
  const typename T::TV *diag;
  typename T::TY *AP;
  int64_t ldap;
  BTiles tl;
  BCtl c;
  int G, LV, NV;
};

template <class T, int VW, int VPL>
__global__ void __launch_bounds__(kThreads) k_b_apply(BApply<T> p) {
  using TA = typename T::TA;
  __shared__ double sm[kThreads / 32][64];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int G = p.G, LV = p.LV, NV = p.NV;
  const int gl = lane & (G - 1);
  const int cl = gl & (LV - 1);
  const int es = gl / LV;
  const int ES = G / LV;
  const int rpb = kThreads / G;  // rows per block pass
  for (int t = blockIdx.x; t < p.tl.ntiles; t += gridDim.x) {
    const int inst = p.tl.tinst[t];
    if (!p.c.sel[inst]) continue;  // uniform over the block
    double dot[VPL][VW];
#pragma unroll
    for (int k = 0; k < VPL; ++k)
#pragma unroll
      for (int i = 0; i < VW; ++i) dot[k][i] = 0.0;
    const int tb = p.tl.tbeg[t], te = p.tl.tend[t];
    for (int r0 = tb; r0 < te; r0 += rpb) {
      const int r = r0 + (int)(threadIdx.x / G);
      const bool valid = r < te;
      const int beg = valid ? p.indptr[r] : 0, end = valid ? p.indptr[r + 1] : 0;
      TA acc[VPL][VW];
      gather_row<typename T::TW, typename T::TX, TA, VW, VPL>(p.col, p.w, p.P, p.ldp, beg, end, es, ES, cl, LV, NV, G,
                                                                acc);
      if (valid && es == 0) {
        const TA d = cvt<TA>(p.diag[r]);
#pragma unroll
        for (int k = 0; k < VPL; ++k) {
          const int vi = cl + k * LV;
          if (vi < NV) {
#pragma unroll
            for (int i = 0; i < VW; ++i) {
              const int cc = vi * VW + i;
              if (cc < p.C) {
                const TA pv = cvt<TA>(p.P[(long long)r * p.ldp + cc]);
                const TA ap = d * pv - acc[k][i];
                p.AP[(long long)r * p.ldap + cc] = cvt<typename T::TY>(ap);
                dot[k][i] += (double)pv * (double)ap;
              }
            }
          }
        }
      }
    }
#pragma unroll
    for (int k = 0; k < VPL; ++k)
#pragma unroll
      for (int i = 0; i < VW; ++i)
        for (int off = LV; off < 32; off <<= 1) dot[k][i] += __shfl_xor_sync(0xffffffffu, dot[k][i], off);
    if (lane < LV) {
#pragma unroll
      for (int k = 0; k < VPL; ++k) {
        const int vi = lane + k * LV;
        if (vi < NV) {
#pragma unroll
          for (int i = 0; i < VW; ++i) {
            const int cc = vi * VW + i;
            if (cc < p.C) sm[wid][cc] = dot[k][i];
          }
        }
      }
    }
    __syncthreads();
    for (int cc = threadIdx.x; cc < p.C; cc += blockDim.x) {
      double s = 0.0;
      for (int w = 0; w < kThreads / 32; ++w) s += sm[w][cc];
      p.c.tp1[(long long)t * p.C + cc] = s;
    }
    __syncthreads();
  }
}

// one block per instance, one warp per column: alpha = rz / pAp
__global__ void k_b_alpha(int32_t C, BTiles tl, BCtl c) {
  const int inst = blockIdx.x;
  if (threadIdx.x == 0) c.stopped[inst] = 0;
  if (!c.sel[inst]) return;
  const int t0 = tl.toff[inst], nt = tl.toff[inst + 1] - t0;
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int cc = wid; cc < C; cc += blockDim.x >> 5) {
    const double s = warp_strided_reduce(c.tp1 + (long long)t0 * C + cc, C, nt, false);
    if (lane == 0) {
      const double al = s > 0.0 ? c.rz[(long long)inst * C + cc] / s : 0.0;
      c.alpha[(long long)inst * C + cc] = isfinite(al) && fabs(al) < 1e30 ? al : 0.0;
    }
  }
}

constexpr int kBCols = 8;  // column chunks of 32 lanes: C <= 256

template <typename TS>
__global__ void __launch_bounds__(256) k_b_update(int phase, int32_t C, TS *R, int64_t ldr, const TS *__restrict__ AP,
                                                  int64_t ldap, const TS *__restrict__ diag, BTiles tl, BCtl c) {
  const int CX = blockDim.x, RY = blockDim.y, tx = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * CX + tx;
  const int nch = (C + CX - 1) / CX;
  __shared__ double s_a[256], s_b[256], s_v[256];
  for (int t = blockIdx.x; t < tl.ntiles; t += gridDim.x) {
    const int inst = tl.tinst[t];
    if (!c.sel[inst]) continue;
    double rz[kBCols], ss[kBCols];
#pragma unroll
    for (int m = 0; m < kBCols; ++m) rz[m] = ss[m] = 0.0;
    double vmax = 0.0;
    const double *al = c.alpha + (long long)inst * C;
    const double *ei = c.epsinv + (long long)inst * C;
    for (int r = tl.tbeg[t] + ty; r < tl.tend[t]; r += RY) {
      const double dinv = 1.0 / (double)diag[r];
#pragma unroll
      for (int m = 0; m < kBCols; ++m) {
        const int cc = tx + m * CX;
        if (m < nch && cc < C) {
          TS rv = R[(long long)r * ldr + cc];
          if (phase == 0) {
            rv = rv - (TS)al[cc] * AP[(long long)r * ldap + cc];
            R[(long long)r * ldr + cc] = rv;
          }
          const double r64 = (double)rv;
          rz[m] += r64 * r64 * dinv;
          ss[m] += r64 * r64;
          vmax = fmax(vmax, isfinite(r64) ? fabs(r64) * dinv * ei[cc] : INFINITY);
        }
      }
    }
    s_v[tid] = vmax;
#pragma unroll
    for (int m = 0; m < kBCols; ++m) {
      if (m < nch) {
        s_a[tid] = rz[m];
        s_b[tid] = ss[m];
        __syncthreads();
        if (ty == 0) {
          double a = 0.0, b = 0.0;
          for (int y = 0; y < RY; ++y) {
            a += s_a[y * CX + tx];
            b += s_b[y * CX + tx];
          }
          const int cc = tx + m * CX;
          if (cc < C) {
            c.tp2[((long long)t * C + cc) * 2 + 0] = a;
            c.tp2[((long long)t * C + cc) * 2 + 1] = b;
          }
        }
        __syncthreads();
      }
    }
    if (tid == 0) {
      double v = 0.0;
      for (int q = 0; q < CX * RY; ++q) v = fmax(v, s_v[q]);
      c.tpv[t] = v;
    }
    __syncthreads();
  }
}

// one block per instance: beta, norms, stop decision
__global__ void k_b_beta(int phase, int32_t C, BTiles tl, BCtl c, BParams bp) {
  const int inst = blockIdx.x;
  if (!c.sel[inst]) return;
  const int t0 = tl.toff[inst], nt = tl.toff[inst + 1] - t0;
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __shared__ double s_rel, s_v;
  if (threadIdx.x == 0) s_rel = 0.0;
  __syncthreads();
  for (int cc = wid; cc < C; cc += blockDim.x >> 5) {
    const double a = warp_strided_reduce(c.tp2 + ((long long)t0 * C + cc) * 2 + 0, (long long)C * 2, nt, false);
    const double b = warp_strided_reduce(c.tp2 + ((long long)t0 * C + cc) * 2 + 1, (long long)C * 2, nt, false);
    if (lane == 0) {
      const long long k = (long long)inst * C + cc;
      const double rzo = c.rz[k];
      const double be = (phase != 2 && rzo > 0.0) ? a / rzo : 0.0;
      c.beta[k] = isfinite(be) && fabs(be) < 1e30 ? be : 0.0;
      c.rz[k] = a;
      const double rel = c.rhsn[k] > 0.0 ? sqrt(b) / c.rhsn[k] : sqrt(b);
      atomicMax((unsigned long long *)&s_rel, __double_as_longlong(isfinite(rel) ? rel : INFINITY));
    }
  }
  if (wid == 0) {
    const double v = warp_strided_reduce(c.tpv + t0, 1, nt, true);
    if (lane == 0) s_v = v;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  const double v = s_v, rel = s_rel;
  c.viol[inst] = v;
  c.relres[inst] = rel;
  double m = 0.0;
  if (bp.mode & 1) m = fmax(m, v);
  if (bp.mode & 2) m = fmax(m, bp.target > 0.0 ? rel / bp.target : rel);
  const bool bad = !isfinite(m);
  const bool conv = m <= 1.0;
  int d = c.done[inst];
  if (phase == 0) c.iters[inst] += 1;
  if (bad) {
    d = 4;
  } else if (phase == 2) {
    c.best[inst] = m;
    c.stall[inst] = 0;
    d = conv ? 5 : 0;
  } else if (phase == 0 && conv) {
    d = 1;
  } else if (phase == 1 && conv) {
    d = 5;
  } else {
    if (m < 0.9 * c.best[inst]) {
      c.best[inst] = m;
      c.stall[inst] = 0;
    } else {
      c.stall[inst] += 1;
    }
    if (c.stall[inst] >= bp.patience) d = 2;
    else if (phase == 1) d = 0;
  }
  if (d == 0 && c.iters[inst] >= bp.max_iter) d = 3;
  if (phase == 0 && d != 0) c.stopped[inst] = 1;
  if (phase == 1 && d == 0) c.stopped[inst] = 2;  // resumed: direction from the true residual
  c.done[inst] = d;
}

// mode 0: Z += alpha P, P = R/diag + beta P (P only while running); mode 1: P update for resumed
// instances; mode 2: P = R/diag for all selected
template <typename TS>
__global__ void __launch_bounds__(256) k_b_dir(int mode, int32_t C, TS *Z, int64_t ldz, TS *P, int64_t ldp,
                                               const TS *__restrict__ R, int64_t ldr, const TS *__restrict__ diag,
                                               BTiles tl, BCtl c) {
  const int CX = blockDim.x, RY = blockDim.y;
  const int nch = (C + CX - 1) / CX;
  for (int t = blockIdx.x; t < tl.ntiles; t += gridDim.x) {
    const int inst = tl.tinst[t];
    bool act, upd_p;
    if (mode == 0) {
      act = c.sel[inst];
      upd_p = c.done[inst] == 0;
    } else if (mode == 1) {
      act = c.stopped[inst] == 2;
      upd_p = act;
    } else {
      act = c.sel[inst];
      upd_p = act;
    }
    if (!act) continue;
    const double *al = c.alpha + (long long)inst * C;
    const double *be = c.beta + (long long)inst * C;
    for (int r = tl.tbeg[t] + threadIdx.y; r < tl.tend[t]; r += RY) {
      const TS dv = diag[r];
      for (int m = 0; m < nch; ++m) {
        const int cc = threadIdx.x + m * CX;
        if (cc >= C) break;
        const TS pv = P[(long long)r * ldp + cc];
        if (mode == 0) Z[(long long)r * ldz + cc] += (TS)al[cc] * pv;
        if (upd_p) {
          const TS y = R[(long long)r * ldr + cc] / dv;
          P[(long long)r * ldp + cc] = mode == 2 ? y : y + (TS)be[cc] * pv;
        }
      }
    }
  }
}

// R = rhs - diag Z + W Z on the rows of selected instances only
template <typename TS>
__global__ void k_b_true_residual(int32_t C, const int32_t *__restrict__ indptr, const int32_t *__restrict__ col,
                                  const float *__restrict__ w, const TS *__restrict__ Z, int64_t ldz,
                                  const TS *__restrict__ rhs, int64_t ldrhs, const TS *__restrict__ diag, TS *R,
                                  int64_t ldr, BTiles tl, BCtl c) {
  for (int t = blockIdx.x; t < tl.ntiles; t += gridDim.x) {
    if (!c.sel[tl.tinst[t]]) continue;
    for (int r = tl.tbeg[t] + (int)threadIdx.x; r < tl.tend[t]; r += blockDim.x) {
      for (int cc = 0; cc < C; ++cc) {
        double acc = 0.0;
        for (int j = indptr[r]; j < indptr[r + 1]; ++j) acc += (double)w[j] * (double)Z[(long long)col[j] * ldz + cc];
        R[(long long)r * ldr + cc] =
            (TS)((double)rhs[(long long)r * ldrhs + cc] - (double)diag[r] * (double)Z[(long long)r * ldz + cc] + acc);
      }
    }
  }
}

static dim3 b_upd_block(int C) {
  const int cx = std::min(32, next_pow2(std::max(C, 1)));
  return dim3(cx, 256 / cx);
}

struct BProblem {
  const int32_t *indptr, *col;
  const float *w;
  int32_t N, C;
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
  int group;
};

template <class T>
static int b_launch_apply(const BProblem &q, const BTiles &tl, const BCtl &c, cudaStream_t s) {
  Layout L;
  DLP_TRY(choose_layout(q.C, sizeof(typename T::TX), q.P, q.ldp, q.group, q.avg_deg, &L));
  BApply<T> a{q.indptr, q.col, (const typename T::TW *)q.w, q.C, (const typename T::TX *)q.P, q.ldp,
              (const typename T::TV *)q.diag, (typename T::TY *)q.AP, q.ldap, tl, c, L.G, L.LV, L.NV};
  const int grid = std::min(tl.ntiles, sm_count() * 8);
  constexpr int VWV = 16 / sizeof(typename T::TX);
#define DLP_BAPPLY(VW_)                                                       \
  switch (L.VPL) {                                                            \
    case 1: k_b_apply<T, VW_, 1><<<grid, kThreads, 0, s>>>(a); break;        \
    case 2: k_b_apply<T, VW_, 2><<<grid, kThreads, 0, s>>>(a); break;        \
    case 3: k_b_apply<T, VW_, 3><<<grid, kThreads, 0, s>>>(a); break;        \
    case 4: k_b_apply<T, VW_, 4><<<grid, kThreads, 0, s>>>(a); break;        \
    default: return DLP_ERR_INVALID;                                          \
  }
  if (L.VW == 1) {
    DLP_BAPPLY(1)
  } else {
    DLP_BAPPLY(VWV)
  }
#undef DLP_BAPPLY
  return check_launch();
}

template <typename TS>
static int b_iteration(const BProblem &q, const BTiles &tl, const BCtl &c, const BParams &bp, cudaStream_t s) {
  const int gridt = std::min(tl.ntiles, sm_count() * 8);
  k_b_select<<<1, 1024, 0, s>>>(tl.ninst, 0, c);
  if (q.dtype == DLP_F32) DLP_TRY(b_launch_apply<T_F32>(q, tl, c, s));
  else DLP_TRY(b_launch_apply<T_W32X64>(q, tl, c, s));
  k_b_alpha<<<tl.ninst, 256, 0, s>>>(q.C, tl, c);
  k_b_update<TS><<<gridt, b_upd_block(q.C), 0, s>>>(0, q.C, (TS *)q.R, q.ldr, (const TS *)q.AP, q.ldap,
                                                     (const TS *)q.diag, tl, c);
  k_b_beta<<<tl.ninst, 256, 0, s>>>(0, q.C, tl, c, bp);
  k_b_dir<TS><<<gridt, b_upd_block(q.C), 0, s>>>(0, q.C, (TS *)q.Z, q.ldz, (TS *)q.P, q.ldp, (const TS *)q.R, q.ldr,
                                                  (const TS *)q.diag, tl, c);
  return check_launch(5);
}

template <typename TS>
static int b_phase(int phase, const BProblem &q, const BTiles &tl, const BCtl &c, const BParams &bp, cudaStream_t s) {
  const int gridt = std::min(tl.ntiles, sm_count() * 8);
  k_b_select<<<1, 1024, 0, s>>>(tl.ninst, phase, c);
  k_b_true_residual<TS><<<gridt, 256, 0, s>>>(q.C, q.indptr, q.col, q.w, (const TS *)q.Z, q.ldz, (const TS *)q.rhs,
                                              q.ldrhs, (const TS *)q.diag, (TS *)q.R, q.ldr, tl, c);
  k_b_update<TS><<<gridt, b_upd_block(q.C), 0, s>>>(phase, q.C, (TS *)q.R, q.ldr, (const TS *)q.AP, q.ldap,
                                                     (const TS *)q.diag, tl, c);
  k_b_beta<<<tl.ninst, 256, 0, s>>>(phase, q.C, tl, c, bp);
  k_b_dir<TS><<<gridt, b_upd_block(q.C), 0, s>>>(phase == 2 ? 2 : 1, q.C, (TS *)q.Z, q.ldz, (TS *)q.P, q.ldp,
                                                  (const TS *)q.R, q.ldr, (const TS *)q.diag, tl, c);
  return check_launch(5);
}

static std::mutex g_b_mu;
static std::unordered_map<std::string, GraphRef> g_b_graphs;
static cudaStream_t g_b_capture[64];

template <typename TS>
static int b_chunk_graph(const BProblem &q, const BTiles &tl, const BCtl &c, const BParams &bp, int k,
                         GraphRef *out) {
  int dev = 0;
  DLP_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return DLP_ERR_INVALID;
  char key[640];
  // every field a captured kernel receives as an argument, exactly (the target to 17 digits)
  snprintf(key, sizeof(key), "%d|%p|%p|%p|%d|%d|%p|%p|%p|%lld|%p|%lld|%p|%lld|%p|%lld|%d|%p|%p|%d|%d|%p|%d|%d|%d|%.17g|%d|%d",
           dev, (const void *)q.indptr, (const void *)q.col, (const void *)q.w, q.N, q.C, q.diag, q.rhs, q.Z,
           (long long)q.ldz, q.R, (long long)q.ldr, q.P, (long long)q.ldp, q.AP, (long long)q.ldap, q.dtype,
           (const void *)tl.tinst, (void *)c.done, tl.ntiles, tl.ninst, (void *)c.tp1, bp.mode, bp.patience,
           bp.max_iter, bp.target, k, q.group);
  std::lock_guard<std::mutex> lk(g_b_mu);
  auto it = g_b_graphs.find(key);
  if (it != g_b_graphs.end()) {
    *out = it->second;
    return DLP_OK;
  }
  if (!g_b_capture[dev]) DLP_CUDA(cudaStreamCreateWithFlags(&g_b_capture[dev], cudaStreamNonBlocking));
  cudaStream_t cs = g_b_capture[dev];
  DLP_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  int st = DLP_OK;
  for (int i = 0; i < k && st == DLP_OK; ++i) st = b_iteration<TS>(q, tl, c, bp, cs);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(cs, &g);
  if (st != DLP_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  if (e != cudaSuccess) {
    set_cuda_error(e);
    return DLP_ERR_CUDA;
  }
  cudaGraphExec_t ex = nullptr;
  const cudaError_t e2 = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (e2 != cudaSuccess) {
    set_cuda_error(e2);
    return DLP_ERR_CUDA;
  }
  auto ref = std::make_shared<GraphExec>();
  ref->ex = ex;
  if (g_b_graphs.size() >= 16) g_b_graphs.clear();  // bounded cache; holders keep their graphs alive
  g_b_graphs.emplace(key, ref);
  *out = ref;
  return DLP_OK;
}

template <typename TS>
static int b_solve(const BProblem &q, const BTiles &tl, const BCtl &c, const BParams &bp, int k, int use_graph,
                   cudaStream_t s) {
  DLP_TRY(b_phase<TS>(2, q, tl, c, bp, s));
  GraphRef gref;
  if (use_graph) DLP_TRY(b_chunk_graph<TS>(q, tl, c, bp, k, &gref));
  cudaGraphExec_t ex = gref ? gref->ex : nullptr;
  int32_t counts[2] = {0, 0};
  for (int guard = 0; guard < (1 << 30); ++guard) {
    k_b_select<<<1, 1024, 0, s>>>(tl.ninst, 0, c);
    DLP_TRY(check_launch());
    DLP_CUDA(cudaMemcpyAsync(counts, c.counts, sizeof(counts), cudaMemcpyDeviceToHost, s));
    DLP_CUDA(cudaStreamSynchronize(s));
    if (counts[1] > 0) {  // proposed stops: confirm on the true residual, resume the others
      DLP_TRY(b_phase<TS>(1, q, tl, c, bp, s));
      continue;
    }
    if (counts[0] == 0) break;
    if (ex) {
      DLP_CUDA(cudaGraphLaunch(ex, s));
      note_launches(6ull * k);
    } else {
      for (int i = 0; i < k; ++i) DLP_TRY(b_iteration<TS>(q, tl, c, bp, s));
    }
  }
  return DLP_OK;
}

}  // namespace dlp

using namespace dlp;

extern "C" {

size_t dlp_pcg_batched_workspace_bytes(int32_t ninst, int32_t ntiles, int32_t C) {
  return bctl_bytes(ninst > 0 ? ninst : 1, ntiles > 0 ? ntiles : 1, C > 0 ? C : 1);
}

int dlp_pcg_batched(const int32_t *indptr, const int32_t *col, const float *w, int32_t N, int32_t C, const void *diag,
                    const void *rhs, int64_t ldrhs, void *Z, int64_t ldz, void *R, int64_t ldr, void *P, int64_t ldp,
                    void *AP, int64_t ldap, int dtype, int32_t ninst, int32_t ntiles, const int32_t *tile_inst,
                    const int32_t *tile_beg, const int32_t *tile_end, const int32_t *inst_tiles,
                    const double *eps_dev, const double *rhs_norm_dev, double target_relres, int32_t mode,
                    int32_t max_iter, int32_t patience, int32_t check_every, int32_t use_graph, int32_t group,
                    double avg_deg, void *ws, size_t ws_bytes, int32_t *iters_out, int32_t *status_out,
                    double *relres_out, dlp_stream_t stream) {
  if (N < 0 || C <= 0 || C > 64 || ninst <= 0 || ntiles <= 0 || ldz < C || ldr < C || ldp < C || ldap < C ||
      ldrhs < C)
    return DLP_ERR_INVALID;
  if (mode < 1 || mode > 3 || !eps_dev || !rhs_norm_dev || !tile_inst || !tile_beg || !tile_end || !inst_tiles)
    return DLP_ERR_INVALID;
  if (!(dtype == DLP_F32 || dtype == DLP_F64)) return DLP_ERR_DTYPE;
  if (!ws || ws_bytes < dlp_pcg_batched_workspace_bytes(ninst, ntiles, C)) return DLP_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  BCtl c = carve_b(ws, ninst, ntiles, C);
  BTiles tl{tile_inst, tile_beg, tile_end, inst_tiles, ntiles, ninst};
  BParams bp{mode, patience > 0 ? patience : 400, max_iter, target_relres};
  BProblem q{indptr, col, w, N, C, diag, rhs, ldrhs, Z, ldz, R, ldr, P, ldp, AP, ldap, dtype, avg_deg, group};
  const size_t iB = 4 * (size_t)ninst;
  DLP_CUDA(cudaMemsetAsync(c.done, 0, iB, s));
  DLP_CUDA(cudaMemsetAsync(c.iters, 0, iB, s));
  DLP_CUDA(cudaMemsetAsync(c.stall, 0, iB, s));
  DLP_CUDA(cudaMemsetAsync(c.stopped, 0, iB, s));
  DLP_CUDA(cudaMemsetAsync(c.rz, 0, 8 * (size_t)ninst * C, s));
  DLP_CUDA(cudaMemcpyAsync(c.eps, eps_dev, 8 * (size_t)ninst * C, cudaMemcpyDeviceToDevice, s));
  DLP_CUDA(cudaMemcpyAsync(c.rhsn, rhs_norm_dev, 8 * (size_t)ninst * C, cudaMemcpyDeviceToDevice, s));
  {
    // epsinv = 1 / eps on the host side of a small copy (ninst * C values)
    std::vector<double> e((size_t)ninst * C);
    DLP_CUDA(cudaMemcpyAsync(e.data(), eps_dev, 8 * e.size(), cudaMemcpyDeviceToHost, s));
    DLP_CUDA(cudaStreamSynchronize(s));
    for (auto &x : e) x = 1.0 / x;
    DLP_CUDA(cudaMemcpy(c.epsinv, e.data(), 8 * e.size(), cudaMemcpyHostToDevice));
  }
  const int k = check_every > 0 ? check_every : 8;
  if (dtype == DLP_F32) DLP_TRY(b_solve<float>(q, tl, c, bp, k, use_graph, s));
  else DLP_TRY(b_solve<double>(q, tl, c, bp, k, use_graph, s));
  if (iters_out) DLP_CUDA(cudaMemcpyAsync(iters_out, c.iters, iB, cudaMemcpyDeviceToHost, s));
  if (status_out) DLP_CUDA(cudaMemcpyAsync(status_out, c.done, iB, cudaMemcpyDeviceToHost, s));
  if (relres_out) DLP_CUDA(cudaMemcpyAsync(relres_out, c.relres, 8 * (size_t)ninst, cudaMemcpyDeviceToHost, s));
  DLP_CUDA(cudaStreamSynchronize(s));
  return DLP_OK;
}

}  // extern "C"
