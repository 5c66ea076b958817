// The AMG V-cycle as one library call and the AMG-preconditioned PCG with its iteration loop on the
// device (dynlp/amg.py:77-134 as the preconditioner of dynlp/solvers.py:66-97).
//
// The V-cycle launches the level kernels of amg.cu (scale, damped Jacobi sweeps, restriction,
// prolongation, the dense coarse solve) and the SpMM of rowops.cu for the level residuals, with every
// intermediate vector in one caller workspace, so a whole cycle is a fixed launch sequence that a
// CUDA graph can hold. The PCG iteration is
//   AP = A P; pAp = P.AP; alpha = rz / pAp; Z += alpha P; R -= alpha AP;
//   stop metric of R (decided on the device); Y = M(R); rz' = R.Y; beta = rz' / rz; P = Y + beta P
// with the fp64 column reductions of reduce.cu (fixed order). The loop runs as a CUDA graph whose
// WHILE node repeats the iteration while the decision kernel keeps its flag set; once a stop is
// proposed the rest of that pass leaves P and rz alone, so a failed confirmation on the true
// residual resumes exactly as the reference's loop does.
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "common.cuh"

namespace dlp {

static size_t al256a(size_t x) { return (x + 255) / 256 * 256; }

// ---- the V-cycle ------------------------------------------------------------------------------
struct VcPlan {
  // per level: two smoothing buffers, the level residual, and for levels >= 1 the restricted input
  // and the cycle's output there; rows padded to 16 bytes (ld) so the level SpMMs gather vectors
  std::vector<char *> A, B, Rr, Rin, Xout;
  int64_t ld = 0;
  size_t bytes = 0;
};

static size_t vc_plan(const dlp_amg_level *lv, int nlev, int C, size_t es, char *base, VcPlan *p) {
  size_t off = 0;
  const int per16 = (int)(16 / es);
  p->ld = (C + per16 - 1) / per16 * per16;
  auto take = [&](int n) {
    char *q = base ? base + off : nullptr;
    off += al256a((size_t)(n > 0 ? n : 1) * (size_t)p->ld * es);
    return q;
  };
  p->A.assign(nlev, nullptr);
  p->B.assign(nlev, nullptr);
  p->Rr.assign(nlev, nullptr);
  p->Rin.assign(nlev, nullptr);
  p->Xout.assign(nlev, nullptr);
  for (int l = 0; l < nlev; ++l) {
    p->A[l] = take(lv[l].n);
    p->B[l] = take(lv[l].n);
    p->Rr[l] = take(lv[l].n);
    if (l > 0) {
      p->Rin[l] = take(lv[l].n);
      p->Xout[l] = take(lv[l].n);
    }
  }
  p->bytes = off;
  return off;
}

struct VcArgs {
  const dlp_amg_level *lv;
  int nlev;
  const double *inv;
  int nu, coarse_sweeps, C, dtype;
  double omega;
  const VcPlan *plan;
  cudaStream_t s;
};

// Y = X + omega * res / diag, res = the level residual RHS - A X (damped Jacobi from the residual).
template <typename T>
__global__ void k_jacobi_update(int32_t n, int32_t C, const T *__restrict__ X, int64_t ldx, const T *__restrict__ res,
                                int64_t ldres, const T *__restrict__ diag, double omega, T *Y, int64_t ldy) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * C) return;
  const long long u = t / C;
  const int c = (int)(t - u * C);
  Y[u * ldy + c] = X[u * ldx + c] + (T)omega * res[u * ldres + c] / diag[u];
}

// One damped Jacobi sweep on level l, Y = X + omega (R - A X) / diag: the level residual by the
// row-gather SpMM into the level's residual buffer, then the update (X in the plan's ld, Y in ldy).
static int vc_sweep(const VcArgs &a, int l, const void *X, const void *R, int64_t ldr, void *Y, int64_t ldy) {
  const dlp_amg_level &L = a.lv[l];
  const int64_t ld = a.plan->ld;
  char *res = a.plan->Rr[l];
  DLP_TRY(dlp_spmm(L.indptr, L.indptr + 1, L.col, L.w, DLP_F32, L.n, nullptr, a.C, X, ld, a.dtype, L.diag, -1.0, 1.0,
                   R, ldr, 1.0, res, ld, a.dtype, 0, 0, L.n > 0 ? (double)L.nnz / L.n : 1.0, (dlp_stream_t)a.s));
  if (L.n == 0) return DLP_OK;
  const long long t = (long long)L.n * a.C;
  if (a.dtype == DLP_F32)
    k_jacobi_update<float><<<ceil_div_i(t, 256), 256, 0, a.s>>>(L.n, a.C, (const float *)X, ld, (const float *)res, ld,
                                                                (const float *)L.diag, a.omega, (float *)Y, ldy);
  else
    k_jacobi_update<double><<<ceil_div_i(t, 256), 256, 0, a.s>>>(L.n, a.C, (const double *)X, ld, (const double *)res,
                                                                 ld, (const double *)L.diag, a.omega, (double *)Y,
                                                                 ldy);
  return check_launch();
}

// Y (ld ldy) = the cycle's correction for R (ld ldr) on level l.
static int vc_cycle(const VcArgs &a, int l, const void *R, int64_t ldr, void *Y, int64_t ldy) {
  const dlp_amg_level &L = a.lv[l];
  const int C = a.C;
  const int64_t ld = a.plan->ld;
  const dlp_stream_t st = (dlp_stream_t)a.s;
  char *bufA = a.plan->A[l], *bufB = a.plan->B[l];
  if (l == a.nlev - 1) {  // the coarsest level
    if (a.inv) return dlp_dense_apply(L.n, C, a.inv, R, ldr, Y, ldy, a.dtype, st);
    if (a.coarse_sweeps <= 1) return dlp_amg_scale_rows(L.n, C, a.omega, R, ldr, L.diag, Y, ldy, a.dtype, st);
    DLP_TRY(dlp_amg_scale_rows(L.n, C, a.omega, R, ldr, L.diag, bufA, ld, a.dtype, st));
    char *cur = bufA;
    for (int i = 0; i < a.coarse_sweeps - 1; ++i) {
      if (i == a.coarse_sweeps - 2) {
        DLP_TRY(vc_sweep(a, l, cur, R, ldr, Y, ldy));
      } else {
        char *tgt = cur == bufA ? bufB : bufA;
        DLP_TRY(vc_sweep(a, l, cur, R, ldr, tgt, ld));
        cur = tgt;
      }
    }
    return DLP_OK;
  }
  // pre-smoothing: X = omega R / diag, then nu - 1 sweeps
  DLP_TRY(dlp_amg_scale_rows(L.n, C, a.omega, R, ldr, L.diag, bufA, ld, a.dtype, st));
  char *cur = bufA;
  for (int i = 0; i < a.nu - 1; ++i) {
    char *tgt = cur == bufA ? bufB : bufA;
    DLP_TRY(vc_sweep(a, l, cur, R, ldr, tgt, ld));
    cur = tgt;
  }
  // restriction of R - A X: Rr = R - diag X + W X
  char *Rr = a.plan->Rr[l];
  DLP_TRY(dlp_spmm(L.indptr, L.indptr + 1, L.col, L.w, DLP_F32, L.n, nullptr, C, cur, ld, a.dtype, L.diag, -1.0, 1.0,
                   R, ldr, 1.0, Rr, ld, a.dtype, 0, 0, L.n > 0 ? (double)L.nnz / L.n : 1.0, st));
  const dlp_amg_level &N = a.lv[l + 1];
  DLP_TRY(dlp_amg_restrict(N.n, C, L.off, L.members, Rr, ld, a.plan->Rin[l + 1], ld, a.dtype, st));
  DLP_TRY(vc_cycle(a, l + 1, a.plan->Rin[l + 1], ld, a.plan->Xout[l + 1], ld));
  DLP_TRY(dlp_amg_prolong_add(L.n, C, L.agg, a.plan->Xout[l + 1], ld, cur, ld, a.dtype, st));
  // post-smoothing: nu sweeps, the last one into Y
  for (int i = 0; i < a.nu; ++i) {
    if (i == a.nu - 1) {
      DLP_TRY(vc_sweep(a, l, cur, R, ldr, Y, ldy));
    } else {
      char *tgt = cur == bufA ? bufB : bufA;
      DLP_TRY(vc_sweep(a, l, cur, R, ldr, tgt, ld));
      cur = tgt;
    }
  }
  return DLP_OK;
}

static int vc_check(const dlp_amg_level *lv, int32_t nlev, int32_t C, int dtype) {
  if (!lv || nlev <= 0 || C <= 0) return DLP_ERR_INVALID;
  if (dtype != DLP_F32 && dtype != DLP_F64) return DLP_ERR_DTYPE;
  for (int l = 0; l < nlev; ++l) {
    const dlp_amg_level &L = lv[l];
    if (L.n < 0 || L.nnz < 0 || (L.n > 0 && (!L.indptr || !L.col || !L.w || !L.diag))) return DLP_ERR_INVALID;
    if (l + 1 < nlev && L.n > 0 && (!L.agg || !L.off || !L.members)) return DLP_ERR_INVALID;
  }
  return DLP_OK;
}

}  // namespace dlp

namespace dlp {

// ---- the AMG-preconditioned PCG ------------------------------------------------------------------
struct GCtl {
  int32_t iters;
  int32_t done;  // 0 running, 1 stop proposed, 2 stalled, 3 cap, 4 breakdown, 5 converged, 6 cancelled
  int32_t stall, patience, max_iter, mode;
  double best, metric, relres, target;
};

struct GBufs {
  GCtl *ctl;
  double *pAp, *rzA, *rzB, *viol, *ss, *eps, *rhsn;  // C doubles each
  void *red_ws;                                       // the column reductions' partials
  size_t red_bytes;
  char *vc;                                           // the V-cycle's vectors
  const int32_t *cancel;
  int has_cond;
  cudaGraphConditionalHandle cond;
};

constexpr int kGThreads = 256;
constexpr int kGUnroll = 4;

// Thread t owns column t mod C of rows t/C, t/C + RS, ... (RS = threads / C), as the PCG sweeps.
struct GIdx {
  long long r0, RS;
  int c;
  bool on;
};
__device__ __forceinline__ GIdx g_index(int32_t C) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long RS = (long long)gridDim.x * blockDim.x / C;
  GIdx g;
  g.RS = RS;
  g.r0 = t / C;
  g.c = (int)(t - g.r0 * C);
  g.on = g.r0 < RS;
  return g;
}

__device__ __forceinline__ double safe_ratio(double a, double b) {
  const double x = b > 0.0 ? a / b : 0.0;
  return isfinite(x) && fabs(x) < 1e30 ? x : 0.0;
}

// alpha = rz / pAp; Z += alpha P; R -= alpha AP. Block 0 keeps rz for the next beta (rzA = rzB).
// Nothing once a stop is decided.
template <typename T>
__global__ void __launch_bounds__(kGThreads)
    k_gpcg_step(int32_t n, int32_t C, T *Z, int64_t ldz, T *R, int64_t ldr, const T *__restrict__ P, int64_t ldp,
                const T *__restrict__ AP, int64_t ldap, GBufs B) {
  if (B.ctl->done != 0) return;
  if (blockIdx.x == 0)
    for (int c = threadIdx.x; c < C; c += blockDim.x) B.rzA[c] = B.rzB[c];
  const GIdx g = g_index(C);
  if (!g.on) return;
  const int c = g.c;
  const T al = (T)safe_ratio(B.rzB[c], B.pAp[c]);
  for (long long r = g.r0; r < n; r += kGUnroll * g.RS) {
    T pv[kGUnroll], av[kGUnroll], zv[kGUnroll], rv[kGUnroll];
#pragma unroll
    for (int u = 0; u < kGUnroll; ++u) {
      const long long rr = r + u * g.RS;
      const bool ok = rr < n;
      pv[u] = ok ? P[rr * ldp + c] : T(0);
      av[u] = ok ? AP[rr * ldap + c] : T(0);
      zv[u] = ok ? Z[rr * ldz + c] : T(0);
      rv[u] = ok ? R[rr * ldr + c] : T(0);
    }
#pragma unroll
    for (int u = 0; u < kGUnroll; ++u) {
      const long long rr = r + u * g.RS;
      if (rr < n) {
        Z[rr * ldz + c] = zv[u] + al * pv[u];
        R[rr * ldr + c] = rv[u] - al * av[u];
      }
    }
  }
}

// P = Y + beta P with beta = rzB / rzA (init: P = Y). Nothing once a stop is decided (the pass of the
// loop that proposed it keeps P for a resume after a failed confirmation).
template <typename T>
__global__ void __launch_bounds__(kGThreads)
    k_gpcg_dir(int init, int32_t n, int32_t C, T *P, int64_t ldp, const T *__restrict__ Y, int64_t ldy, GBufs B,
               bf16 *P_lo, int64_t ld_lo) {
  if (!init && B.ctl->done != 0) return;
  const GIdx g = g_index(C);
  if (!g.on) return;
  const int c = g.c;
  const T be = init ? T(0) : (T)safe_ratio(B.rzB[c], B.rzA[c]);
  for (long long r = g.r0; r < n; r += kGUnroll * g.RS) {
    T yv[kGUnroll], pv[kGUnroll];
#pragma unroll
    for (int u = 0; u < kGUnroll; ++u) {
      const long long rr = r + u * g.RS;
      const bool ok = rr < n;
      yv[u] = ok ? Y[rr * ldy + c] : T(0);
      pv[u] = (ok && !init) ? P[rr * ldp + c] : T(0);
    }
#pragma unroll
    for (int u = 0; u < kGUnroll; ++u) {
      const long long rr = r + u * g.RS;
      if (rr < n) {
        const T pn = yv[u] + be * pv[u];
        P[rr * ldp + c] = pn;
        if (P_lo) P_lo[rr * ld_lo + c] = cvt<bf16>(pn);  // the mirror the bf16 apply gathers
      }
    }
  }
}

// The stop decision (one thread), from viol[c] = max_u |R_uc| / diag_u and ss[c] = sum_u R_uc^2:
//   phase 0 (an iteration): stop proposed when the metric is <= 1, else the patience rule and the
//   cap; phase 1 (a true residual after a proposal): converged when <= 1, else the run goes on;
//   phase 2 (the initial residual). Sets the device loop's flag while the solve runs.
__global__ void k_gpcg_decide(int phase, int32_t C, GBufs B) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  GCtl *ctl = B.ctl;
  if (phase == 0 && ctl->done != 0) {
    if (B.has_cond) cudaGraphSetConditional(B.cond, 0u);
    return;
  }
  double mv = 0.0, rel = 0.0;
  bool bad = false;
  for (int c = 0; c < C; ++c) {
    if (!isfinite(B.ss[c]) || !isfinite(B.viol[c])) bad = true;
    mv = fmax(mv, B.viol[c] / B.eps[c]);
    rel = fmax(rel, B.rhsn[c] > 0.0 ? sqrt(B.ss[c]) / B.rhsn[c] : sqrt(B.ss[c]));
  }
  double m = 0.0;
  if (ctl->mode & 1) m = fmax(m, mv);
  if (ctl->mode & 2) m = fmax(m, ctl->target > 0.0 ? rel / ctl->target : rel);
  ctl->metric = m;
  ctl->relres = rel;
  const bool conv = m <= 1.0 && !bad;
  if (phase == 0) ctl->iters += 1;
  if (bad) {
    ctl->done = 4;
  } else if (phase == 2) {
    ctl->best = m;
    ctl->stall = 0;
    ctl->done = conv ? 5 : 0;
  } else if (conv) {
    ctl->done = phase == 0 ? 1 : 5;
  } else {
    if (m < 0.9 * ctl->best) {
      ctl->best = m;
      ctl->stall = 0;
    } else {
      ctl->stall += 1;
    }
    ctl->done = ctl->stall >= ctl->patience ? 2 : 0;
  }
  if (ctl->done == 0 && ctl->iters >= ctl->max_iter) ctl->done = 3;
  if (ctl->done == 0 && read_cancel(B.cancel)) ctl->done = 6;
  if (phase == 0 && B.has_cond) cudaGraphSetConditional(B.cond, ctl->done == 0 ? 1u : 0u);
}

}  // namespace dlp

namespace dlp {

struct GProblem {
  const int32_t *rbeg, *rend, *col;
  const float *w;
  int32_t n, C;
  const void *diag, *rhs;
  int64_t ldrhs;
  void *Z, *R, *P, *AP, *Y;
  int64_t ldz, ldr, ldp, ldap, ldy;
  int dtype;
  double avg_deg;
  VcArgs vc;
  const void *w_lo;  // bf16 weights and the bf16 mirror of P for the apply (NULL: full precision)
  void *P_lo;
  int64_t ld_lo;
};

static int g_grid(int32_t n, int32_t C) {
  long long blocks = ceil_div_i((long long)n * C, (long long)kGThreads * kGUnroll);
  blocks = std::min(blocks, (long long)sm_count() * 8);
  blocks = std::max(blocks, (long long)ceil_div_i((long long)C, kGThreads));
  return (int)std::max(blocks, 1LL);
}

// viol[c] = max_u |R_uc| / diag_u, ss[c] = sum_u R_uc^2 (fp64, fixed order)
static int g_stats(const GProblem &q, const GBufs &B, cudaStream_t s) {
  DLP_TRY(dlp_colreduce(0, q.n, q.C, q.R, q.ldr, nullptr, q.C, q.diag, q.dtype, nullptr, B.viol, B.red_ws,
                        B.red_bytes, (dlp_stream_t)s));
  return dlp_colreduce(2, q.n, q.C, q.R, q.ldr, nullptr, q.C, nullptr, q.dtype, nullptr, B.ss, B.red_ws, B.red_bytes,
                       (dlp_stream_t)s);
}

// R = rhs - A Z (the true residual)
static int g_residual(const GProblem &q, cudaStream_t s) {
  return dlp_spmm(q.rbeg, q.rend, q.col, q.w, DLP_F32, q.n, nullptr, q.C, q.Z, q.ldz, q.dtype, q.diag, -1.0, 1.0,
                  q.rhs, q.ldrhs, 1.0, q.R, q.ldr, q.dtype, 0, 0, q.avg_deg, (dlp_stream_t)s);
}

// Y = M(R); rzB = R.Y
static int g_precond(const GProblem &q, const GBufs &B, cudaStream_t s) {
  VcArgs a = q.vc;
  a.s = s;
  DLP_TRY(vc_cycle(a, 0, q.R, q.ldr, q.Y, q.ldy));
  return dlp_colreduce(1, q.n, q.C, q.R, q.ldr, q.Y, q.ldy, nullptr, q.dtype, nullptr, B.rzB, B.red_ws, B.red_bytes,
                       (dlp_stream_t)s);
}

template <typename T>
static int g_dir(int init, const GProblem &q, const GBufs &B, cudaStream_t s) {
  k_gpcg_dir<T><<<g_grid(q.n, q.C), kGThreads, 0, s>>>(init, q.n, q.C, (T *)q.P, q.ldp, (const T *)q.Y, q.ldy, B,
                                                       (bf16 *)q.P_lo, q.ld_lo);
  return check_launch();
}

static int g_dir_any(int init, const GProblem &q, const GBufs &B, cudaStream_t s) {
  return q.dtype == DLP_F32 ? g_dir<float>(init, q, B, s) : g_dir<double>(init, q, B, s);
}

static int g_decide(int phase, const GProblem &q, const GBufs &B, cudaStream_t s) {
  k_gpcg_decide<<<1, 32, 0, s>>>(phase, q.C, B);
  return check_launch();
}

// One iteration: AP = A P; pAp; alpha, Z, R; the stop decision; Y = M(R); rz; beta, P.
template <typename T>
static int g_iteration(const GProblem &q, const GBufs &B, cudaStream_t s) {
  const dlp_stream_t st = (dlp_stream_t)s;
  if (q.w_lo) {  // bf16 weights and gathered rows, fp32 accumulation; the own-row term from fp32 P
    DLP_TRY(dlp_spmm_lowp(q.rbeg, q.rend, q.col, q.w_lo, q.n, q.C, q.P_lo, q.ld_lo, q.P, q.ldp, q.diag, 1.0, -1.0,
                          q.AP, q.ldap, 0, q.avg_deg, st));
  } else {
    DLP_TRY(dlp_spmm(q.rbeg, q.rend, q.col, q.w, DLP_F32, q.n, nullptr, q.C, q.P, q.ldp, q.dtype, q.diag, 1.0, -1.0,
                     nullptr, q.C, 0.0, q.AP, q.ldap, q.dtype, 0, 0, q.avg_deg, st));
  }
  DLP_TRY(dlp_colreduce(1, q.n, q.C, q.P, q.ldp, q.AP, q.ldap, nullptr, q.dtype, nullptr, B.pAp, B.red_ws,
                        B.red_bytes, st));
  k_gpcg_step<T><<<g_grid(q.n, q.C), kGThreads, 0, s>>>(q.n, q.C, (T *)q.Z, q.ldz, (T *)q.R, q.ldr, (const T *)q.P,
                                                        q.ldp, (const T *)q.AP, q.ldap, B);
  DLP_TRY(check_launch());
  DLP_TRY(g_stats(q, B, s));
  DLP_TRY(g_decide(0, q, B, s));
  DLP_TRY(g_precond(q, B, s));
  return g_dir<T>(0, q, B, s);
}

static int g_iteration_any(const GProblem &q, const GBufs &B, cudaStream_t s) {
  return q.dtype == DLP_F32 ? g_iteration<float>(q, B, s) : g_iteration<double>(q, B, s);
}

// Cache of the loop graphs, one per problem signature (the level descriptors included).
struct GKey {
  std::vector<uintptr_t> v;
  bool operator==(const GKey &o) const { return v == o.v; }
};
struct GKeyHash {
  size_t operator()(const GKey &k) const {
    size_t h = 1469598103934665603ull;
    for (auto x : k.v) h = (h ^ x) * 1099511628211ull;
    return h;
  }
};
static std::mutex g_gmu;
static std::unordered_map<GKey, GraphRef, GKeyHash> g_ggraphs;
static cudaStream_t g_gcapture[64];

static int g_key(const GProblem &q, const GBufs &B, GKey *key) {
  int dev = 0;
  DLP_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return DLP_ERR_INVALID;
  std::vector<uintptr_t> v = {(uintptr_t)dev, (uintptr_t)q.rbeg, (uintptr_t)q.rend, (uintptr_t)q.col,
                              (uintptr_t)q.w, (uintptr_t)q.n, (uintptr_t)q.C, (uintptr_t)q.diag, (uintptr_t)q.Z,
                              (uintptr_t)q.ldz, (uintptr_t)q.R, (uintptr_t)q.ldr, (uintptr_t)q.P, (uintptr_t)q.ldp,
                              (uintptr_t)q.AP, (uintptr_t)q.ldap, (uintptr_t)q.Y, (uintptr_t)q.ldy,
                              (uintptr_t)q.dtype, (uintptr_t)B.ctl, (uintptr_t)B.cancel, (uintptr_t)q.vc.inv,
                              (uintptr_t)q.vc.nu, (uintptr_t)q.vc.coarse_sweeps, (uintptr_t)q.vc.nlev,
                              (uintptr_t)q.w_lo, (uintptr_t)q.P_lo, (uintptr_t)q.ld_lo};
  uint64_t om;
  std::memcpy(&om, &q.vc.omega, sizeof(om));
  v.push_back((uintptr_t)om);
  v.push_back((uintptr_t)(int64_t)(q.avg_deg * 1024.0));
  for (int l = 0; l < q.vc.nlev; ++l) {
    const dlp_amg_level &L = q.vc.lv[l];
    for (uintptr_t x : {(uintptr_t)L.n, (uintptr_t)L.nnz, (uintptr_t)L.indptr, (uintptr_t)L.col, (uintptr_t)L.w,
                        (uintptr_t)L.diag, (uintptr_t)L.agg, (uintptr_t)L.off, (uintptr_t)L.members})
      v.push_back(x);
  }
  key->v = std::move(v);
  return DLP_OK;
}

static int g_loop_graph(const GProblem &q, const GBufs &B0, GraphRef *out) {
  GKey key;
  DLP_TRY(g_key(q, B0, &key));
  const int dev = (int)key.v[0];
  std::lock_guard<std::mutex> lk(g_gmu);
  auto it = g_ggraphs.find(key);
  if (it != g_ggraphs.end()) {
    *out = it->second;
    return DLP_OK;
  }
  if (!g_gcapture[dev]) DLP_CUDA(cudaStreamCreateWithFlags(&g_gcapture[dev], cudaStreamNonBlocking));
  cudaStream_t cs = g_gcapture[dev];
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
  GBufs B = B0;
  B.has_cond = 1;
  B.cond = h;
  e = cudaStreamBeginCaptureToGraph(cs, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                    cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return fail(e);
  const int st = g_iteration_any(q, B, cs);
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
  if (g_ggraphs.size() >= 16) g_ggraphs.clear();  // holders keep their own references
  g_ggraphs.emplace(key, ref);
  *out = ref;
  return DLP_OK;
}

static size_t g_ws_layout(const dlp_amg_level *lv, int32_t nlev, int32_t C, int dtype, size_t *off_red,
                          size_t *red_bytes, size_t *off_vc) {
  const size_t cc = (size_t)(C > 0 ? C : 1);
  size_t b = al256a(sizeof(GCtl)) + 7 * al256a(sizeof(double) * cc);
  *off_red = b;
  *red_bytes = al256a(dlp_colreduce_workspace_bytes(C));
  b += *red_bytes;
  *off_vc = b;
  VcPlan p;
  b += vc_plan(lv, nlev, C, dtype == DLP_F64 ? 8 : 4, nullptr, &p);
  return b;
}

}  // namespace dlp

using namespace dlp;

extern "C" {

size_t dlp_amg_vcycle_workspace_bytes(const dlp_amg_level *levels, int32_t nlev, int32_t C, int dtype) {
  if (vc_check(levels, nlev, C, dtype) != DLP_OK) return 0;
  VcPlan p;
  return vc_plan(levels, nlev, C, dtype == DLP_F64 ? 8 : 4, nullptr, &p);
}

int dlp_amg_vcycle(const dlp_amg_level *levels, int32_t nlev, const double *coarse_inv, int32_t nu, double omega,
                   int32_t coarse_sweeps, int32_t C, int dtype, const void *R, int64_t ldr, void *Y, int64_t ldy,
                   void *ws, size_t ws_bytes, dlp_stream_t stream) {
  DLP_TRY(vc_check(levels, nlev, C, dtype));
  if (nu < 1 || ldr < C || ldy < C || (levels[0].n > 0 && (!R || !Y))) return DLP_ERR_INVALID;
  VcPlan p;
  if (!ws || ws_bytes < vc_plan(levels, nlev, C, dtype == DLP_F64 ? 8 : 4, nullptr, &p)) return DLP_ERR_WORKSPACE;
  vc_plan(levels, nlev, C, dtype == DLP_F64 ? 8 : 4, (char *)ws, &p);
  VcArgs a{levels, nlev, coarse_inv, nu, coarse_sweeps, C, dtype, omega, &p, (cudaStream_t)stream};
  if (levels[0].n == 0) return DLP_OK;
  return vc_cycle(a, 0, R, ldr, Y, ldy);
}

size_t dlp_pcg_amg_workspace_bytes(const dlp_amg_level *levels, int32_t nlev, int32_t C, int dtype) {
  if (vc_check(levels, nlev, C, dtype) != DLP_OK) return 0;
  size_t a, b, c;
  return g_ws_layout(levels, nlev, C, dtype, &a, &b, &c);
}

int dlp_pcg_amg(const int32_t *rbeg, const int32_t *rend, const int32_t *col, const float *w, int32_t n, int32_t C,
                const void *diag, const void *rhs, int64_t ldrhs, void *Z, int64_t ldz, void *R, int64_t ldr, void *P,
                int64_t ldp, void *AP, int64_t ldap, void *Y, int64_t ldy, int dtype, const double *eps,
                const double *rhs_norm, double target_relres, int32_t mode, int32_t max_iter, int32_t patience,
                int32_t use_graph, double avg_deg, const dlp_amg_level *levels, int32_t nlev,
                const double *coarse_inv, int32_t nu, double omega, int32_t coarse_sweeps, void *ws,
                size_t ws_bytes, int32_t *iters_out, double *relres_out, int32_t *status_out,
                dlp_stream_t stream, const void *w_lo, void *P_lo, int64_t ld_lo) {
  DLP_TRY(vc_check(levels, nlev, C, dtype));
  if ((w_lo || P_lo) && (!w_lo || !P_lo || ld_lo < C || dtype != DLP_F32)) return DLP_ERR_INVALID;
  if (n < 0 || levels[0].n != n || nu < 1) return DLP_ERR_INVALID;
  if (ldz < C || ldr < C || ldp < C || ldap < C || ldy < C || ldrhs < C) return DLP_ERR_INVALID;
  if ((mode & 3) == 0 || mode > 3 || ((mode & 1) && !eps) || ((mode & 2) && !rhs_norm)) return DLP_ERR_INVALID;
  size_t off_red, red_bytes, off_vc;
  if (!ws || ws_bytes < g_ws_layout(levels, nlev, C, dtype, &off_red, &red_bytes, &off_vc)) return DLP_ERR_WORKSPACE;
  if (iters_out) *iters_out = 0;
  if (n == 0) {
    if (status_out) *status_out = 5;
    return DLP_OK;
  }
  if (!rbeg || !rend || !col || !w || !diag || !rhs || !Z || !R || !P || !AP || !Y) return DLP_ERR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  char *base = (char *)ws;
  GBufs B{};
  B.ctl = (GCtl *)base;
  size_t o = al256a(sizeof(GCtl));
  double **vecs[7] = {&B.pAp, &B.rzA, &B.rzB, &B.viol, &B.ss, &B.eps, &B.rhsn};
  for (auto v : vecs) {
    *v = (double *)(base + o);
    o += al256a(sizeof(double) * (size_t)C);
  }
  B.red_ws = base + off_red;
  B.red_bytes = red_bytes;
  B.vc = base + off_vc;
  B.cancel = cancel_word();
  VcPlan plan;
  vc_plan(levels, nlev, C, dtype == DLP_F64 ? 8 : 4, B.vc, &plan);
  GProblem q{rbeg, rend, col, w, n, C, diag, rhs, ldrhs, Z, R, P, AP, Y, ldz, ldr, ldp, ldap, ldy, dtype,
             avg_deg > 0 ? avg_deg : 1.0,
             VcArgs{levels, nlev, coarse_inv, nu, coarse_sweeps, C, dtype, omega, &plan, s}, w_lo, P_lo, ld_lo};
  GCtl h{};
  h.patience = patience > 0 ? patience : 400;
  h.max_iter = max_iter;
  h.mode = mode;
  h.target = target_relres;
  DLP_CUDA(cudaMemcpyAsync(B.ctl, &h, sizeof(h), cudaMemcpyHostToDevice, s));
  {
    std::vector<double> e((size_t)C * 2);
    for (int c = 0; c < C; ++c) {
      e[c] = eps ? eps[c] : 1e300;
      e[C + c] = rhs_norm ? rhs_norm[c] : 0.0;
    }
    DLP_CUDA(cudaMemcpyAsync(B.eps, e.data(), sizeof(double) * C, cudaMemcpyHostToDevice, s));
    DLP_CUDA(cudaMemcpyAsync(B.rhsn, e.data() + C, sizeof(double) * C, cudaMemcpyHostToDevice, s));
  }
  GCtl cur{};
  auto read = [&]() -> int {
    DLP_CUDA(cudaMemcpyAsync(&cur, B.ctl, sizeof(cur), cudaMemcpyDeviceToHost, s));
    DLP_CUDA(cudaStreamSynchronize(s));
    return DLP_OK;
  };
  // the initial residual and its decision
  DLP_TRY(g_residual(q, s));
  DLP_TRY(g_stats(q, B, s));
  DLP_TRY(g_decide(2, q, B, s));
  DLP_TRY(read());
  if (cur.done == 0 && max_iter <= 0) cur.done = 3;
  if (cur.done == 0) {
    DLP_TRY(g_precond(q, B, s));  // Y = M(R), rz = R.Y
    DLP_TRY(g_dir_any(1, q, B, s));  // P = Y
  }
  GraphRef loop;
  if (use_graph && cur.done == 0) DLP_TRY(g_loop_graph(q, B, &loop));
  long long guard = 0;
  while (cur.done == 0 && guard++ < (long long)max_iter + 8) {
    const int it0 = cur.iters;
    if (loop) {
      DLP_CUDA(cudaGraphLaunch(loop->ex, s));
    } else {
      for (int k = 0; k < 4; ++k) DLP_TRY(g_iteration_any(q, B, s));
    }
    DLP_TRY(read());
    if (loop) note_launches(16ull * (unsigned long long)std::max(cur.iters - it0, 1));
    if (cur.done == 1) {  // a proposed stop: confirmed on the true residual (dynlp/solvers.py:85-89)
      DLP_TRY(g_residual(q, s));
      DLP_TRY(g_stats(q, B, s));
      DLP_TRY(g_decide(1, q, B, s));
      DLP_TRY(read());
      if (cur.done == 0) {  // not confirmed: resume from the true residual
        DLP_TRY(g_precond(q, B, s));
        DLP_TRY(g_dir_any(0, q, B, s));
      }
    } else if (cur.done == 0 && cur.iters == it0) {
      return DLP_ERR_DEVICE;  // a pass ended without a decision
    }
  }
  if (iters_out) *iters_out = cur.iters;
  if (relres_out) *relres_out = cur.relres;
  if (status_out) *status_out = cur.done;
  if (cur.done == 3) return DLP_ERR_CAP;
  if (cur.done == 6) return DLP_ERR_CANCELLED;
  return DLP_OK;
}

}  // extern "C"

// ---- the coarse operator's inverse (setup) ---------------------------------------------------------
// Gauss-Jordan elimination in place on a symmetric positive definite matrix (no pivoting needed):
// for each pivot k, the scaled pivot row and the pivot column are saved first (k_gj_save), then
// every element takes its update from the saved vectors (k_gj_update), so no thread reads what
// another thread of the same launch writes. After the last pivot A holds its inverse.
namespace dlp {

__global__ void k_gj_save(int32_t n, int32_t k, const double *__restrict__ A, double *fcol, double *rowk) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double piv = A[(long long)k * n + k];
  fcol[t] = A[t * n + k];
  rowk[t] = (t == k ? 1.0 : A[(long long)k * n + t]) / piv;
}

__global__ void k_gj_update(int32_t n, int32_t k, double *A, const double *__restrict__ fcol,
                            const double *__restrict__ rowk) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const long long i = t / n;
  const int j = (int)(t - i * n);
  if (i == k) {
    A[t] = rowk[j];
  } else {
    const double a = j == k ? 0.0 : A[t];
    A[t] = a - fcol[i] * rowk[j];
  }
}

}  // namespace dlp

extern "C" {

size_t dlp_dense_spd_inverse_workspace_bytes(int32_t n) { return 2 * al256a(sizeof(double) * (size_t)(n > 0 ? n : 1)); }

int dlp_dense_spd_inverse(int32_t n, double *A, void *ws, size_t ws_bytes, dlp_stream_t stream) {
  if (n < 0 || (n > 0 && !A)) return DLP_ERR_INVALID;
  if (n > 46340) return DLP_ERR_INVALID;  // n * n elements index an int64 but the grid is int
  if (!ws || ws_bytes < dlp_dense_spd_inverse_workspace_bytes(n)) return DLP_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  double *fcol = (double *)ws;
  double *rowk = (double *)((char *)ws + al256a(sizeof(double) * (size_t)(n > 0 ? n : 1)));
  const int g1 = ceil_div_i(n, 256);
  const int g2 = ceil_div_i((long long)n * n, 256);
  for (int k = 0; k < n; ++k) {
    k_gj_save<<<g1, 256, 0, s>>>(n, k, A, fcol, rowk);
    k_gj_update<<<g2, 256, 0, s>>>(n, k, A, fcol, rowk);
  }
  return check_launch(2 * n);
}

}  // extern "C"
