// hq_kernels.cu -- sm_100a kernels of the batched DQMC sweep (FP64).
//
//  k_interval  : one CTA per chain, G(tau,tau) resident in shared memory for a whole
//                stabilisation interval: wrap (src/dqmc_core.cpp:142-161), Metropolis
//                flips with delayed rank-k updates flushed by DMMA
//                (src/dqmc_core.cpp:102-119, src/hubbard.cpp:123-139), fused equal-time
//                estimators (include/observable_methods.hpp:39-151) and optional snapshots.
//  k_bchain    : B-matrix chain of one interval applied to U_top*D_top
//                (src/dqmc_core.cpp:190, :251 + the (M*U)*S product of svd_stack.hpp:144).
//  k_udt       : column-pivoted Householder UDV factorisation X P = Q R, X = Q D T
//                (the stack push of include/utils/svd_stack.hpp:107-175).
//  k_invert    : in-place Gauss-Jordan inverse with partial pivoting (the inverse() of
//                include/utils/stable_numerics.hpp:235).
//  k_gemm      : batched FP64 DMMA GEMM with the scalings of the G builders
//                (include/utils/stable_numerics.hpp:186-324) and the wrap-error epilogue
//                (:37-48, signed maximum).
//  k_measure   : equal-time estimators + snapshot of a freshly built G.
//  k_dyn_*     : time-displaced propagation and estimators (src/dqmc_core.cpp:291-390,
//                include/observable_methods.hpp:84-195).
#include <cuda_runtime.h>
#include <stdint.h>
#include <climits>
#include "hq_device.cuh"
#include "hq_kernels.h"

namespace hq {

// shared-memory leading dimension of an N x N matrix: odd, so that threads walking
// consecutive columns hit distinct banks
__host__ __device__ inline int smem_ld(int N) { return (N % 2 == 0) ? N + 1 : N; }

// leading dimension of the delayed-update panels: = 4 (mod 16) doubles, so that the DMMA
// fragment loads of the flush are free of bank conflicts
__host__ __device__ inline int panel_ld(int N) { return N + ((4 - N % 16) + 16) % 16; }

// bytes of dynamic shared memory of k_interval / k_bchain for a chain of size N with
// delay depth kmax (matrix in smem when `resident`)
__host__ __device__ inline size_t interval_smem_doubles(int N, int kmax, bool resident) {
  const size_t mat = resident ? (size_t)N * smem_ld(N) : 0;
  const size_t panels = (size_t)panel_ld(N) * kmax * 2;
  const size_t stage = (size_t)8 * (((N + 15) & ~15) + 4);
  const size_t work = panels > stage ? panels : stage;
  return mat + work + 3 * (size_t)N + (size_t)(N + 7) / 4 + 64;
}

struct SliceView {
  const int8_t* s;  // fields of the slice (shared memory)
};

// ---------------------------------------------------------------------------------
//  Equal-time estimators of one slice (include/observable_methods.hpp:39-74, 131-151)
//  filling = 2 - 2 trG/N ; docc = sum_i (1-G_ii)^2 / N ;
//  swave   = sum_ij [(1-G)_ji^2 + G_ij^2] / N = (2 sum G^2 - 2 trG + N) / N
// ---------------------------------------------------------------------------------
__device__ void measure_slice(const double* G, int ld, int N, double* acc, double* red) {
  double tr = 0.0, dd = 0.0, sq = 0.0;
  HQ_FOR_EACH_ELEM(N, i, j) {
    const double v = G[i + (size_t)j * ld];
    sq = fma(v, v, sq);
    if (i == j) { tr += v; dd += (1.0 - v) * (1.0 - v); }
  }
  block_sum3(tr, dd, sq, red);
  if (threadIdx.x == 0) {
    acc[HQ_ACC_FILLING] += 2.0 - 2.0 * tr / N;
    acc[HQ_ACC_DOCC] += dd / N;
    acc[HQ_ACC_SWAVE] += (2.0 * sq - 2.0 * tr + N) / N;
    acc[HQ_ACC_NSLICE] += 1.0;
  }
}

__device__ void copy_mat(double* dst, int ldd, const double* src, int lds, int N) {
  HQ_FOR_EACH_ELEM(N, i, j) dst[i + (size_t)j * ldd] = src[i + (size_t)j * lds];
}

// ---------------------------------------------------------------------------------
//  Metropolis sweep over the N sites of one slice with delayed rank-k updates.
//
//  The reference visits i = 0..N-1 in order, draws one uniform per site, and on
//  acceptance applies G -= gamma G[:,i] (e_i^T - G[i,:]), gamma = Delta/(1+(1-G_ii)Delta)
//  (src/hubbard.cpp:123-139). A rejected site leaves G unchanged, so the ratio of every
//  later site only depends on the current diagonal: all remaining sites are tested in
//  parallel and the first acceptance is taken, then the search resumes after it. The
//  accepted updates are kept as G = G0 + X Y (X: N x k, Y: k x N) and flushed into G0
//  with DMMA when k reaches kmax and at the end of the slice.
// ---------------------------------------------------------------------------------
// G[0:M, 0:Nc] += X[0:M, 0:k] Y[0:k, 0:Nc]  (X column-major ldx, Y row-major ldy), by 16 x 32
// strips of four 16 x 8 DMMA tiles that share the A fragments
__device__ void rank_update(double* G, int ld, int M, int Nc, const double* X, int ldx, const double* Y, int ldy,
                            int k) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int mt = (M + 15) / 16, ns = (Nc + 31) / 32;
  const int strips = mt * ns;
  for (int st = warp; st < strips; st += nwarps) {
    const int r0 = (st % mt) * 16, c0 = (st / mt) * 32;
    const int r = r0 + g;
    double acc[4][4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int c = c0 + t * 8 + 2 * q;
      acc[t][0] = (r < M && c < Nc) ? G[r + (size_t)c * ld] : 0.0;
      acc[t][1] = (r < M && c + 1 < Nc) ? G[r + (size_t)(c + 1) * ld] : 0.0;
      acc[t][2] = (r + 8 < M && c < Nc) ? G[r + 8 + (size_t)c * ld] : 0.0;
      acc[t][3] = (r + 8 < M && c + 1 < Nc) ? G[r + 8 + (size_t)(c + 1) * ld] : 0.0;
    }
    for (int m0 = 0; m0 < k; m0 += 4) {
      const int m = m0 + q;
      const bool mk = m < k;
      const double a0 = (r < M && mk) ? X[r + m * ldx] : 0.0;
      const double a1 = (r + 8 < M && mk) ? X[r + 8 + m * ldx] : 0.0;
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int cb = c0 + t * 8 + g;
        const double b0 = (cb < Nc && mk) ? Y[m * ldy + cb] : 0.0;
        dmma_16x8x4(acc[t], a0, a1, b0);
      }
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int c = c0 + t * 8 + 2 * q;
      if (r < M && c < Nc) G[r + (size_t)c * ld] = acc[t][0];
      if (r < M && c + 1 < Nc) G[r + (size_t)(c + 1) * ld] = acc[t][1];
      if (r + 8 < M && c < Nc) G[r + 8 + (size_t)c * ld] = acc[t][2];
      if (r + 8 < M && c + 1 < Nc) G[r + 8 + (size_t)(c + 1) * ld] = acc[t][3];
    }
  }
}

// G += X Y on the full N x N matrix (the flush of the delayed Metropolis panels)
__device__ void flush_panels(double* G, int ld, int N, const double* X, int ldx, const double* Y, int ldy, int k) {
  rank_update(G, ld, N, N, X, ldx, Y, ldy, k);
}

// barrier of the decision team (warps 0-3 of the interval kernel)
__device__ __forceinline__ void team_sync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

struct MetroShared {
  double* d;      // current diagonal [N]
  double* u;      // uniforms [N]
  double* rr;     // last ratio of each site [N] (ratio log)
  int8_t* s;      // fields of the slice [N]
  int8_t* flip;   // accepted flags [N]
  double* X;      // N x kmax
  double* Y;      // kmax x N (row-major)
  int* ired;      // >= 32 ints
  int* qj;        // accepted site of each panel column [kmax]
  double* qg;     // gamma of each panel column [kmax]
  double* gam;    // speculative gamma of the sites of a search round [128]
  volatile int* qn;    // panel columns published by the decision warp
  volatile int* qdone; // decision phase of this panel finished
};

__device__ void metropolis_slice(const HqChain& ch, double* G, int ld, const MetroShared& sh, uint32_t& rng,
                                 double& n_acc, int flags, long long log_base) {
  const int N = ch.N, kmax = ch.kmax;
  const int ldp = panel_ld(N);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool log = (flags & HQ_F_LOG_RATIOS) && ch.ratios;
  // uniforms of this slice: site i consumes engine draws 2i+1, 2i+2 after the current state
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const uint32_t x1 = minstd_mulmod(minstd_pow(2ull * i + 1), rng);
    const uint32_t x2 = minstd_mulmod(kMinstdA, x1);
    sh.u[i] = canonical_from_pair(x1, x2);
    sh.d[i] = G[i + (size_t)i * ld];
    sh.flip[i] = 0;
  }
  rng = minstd_mulmod(minstd_pow(2ull * N), rng);
  __syncthreads();
  int k = 0, start = 0;
  const int tid = threadIdx.x;
  constexpr int kTeam = 128;  // warps 0-3 walk the decision chain, warps 4-7 fill panels
  while (true) {
    // The decision team walks the chain of flips of this panel. For each accepted site j it
    // computes the entries p > j of G's current column / row j (all that later decisions of
    // this slice read) and the diagonal; the helper warps fill the entries p <= j of the
    // same panel columns from a shared-memory queue, off the critical path.
    if (tid == 0) { *sh.qn = 0; *sh.qdone = 0; }
    __syncthreads();
    if (tid < kTeam) {
      int kk = 0, round = 0;
      while (start < N && kk < kmax) {
        // first accepted site >= start: 128 sites per round. accept iff u < min(1, |r|),
        // r = a^2 / (1 + Delta), 1 + Delta = e^{-2 alpha s} > 0: u (1 + Delta) < a^2.
        // gamma = Delta / a is formed speculatively by every accepting thread.
        int j = -1;
        for (int base = start; base < N; base += kTeam) {
          const int i = base + tid;
          bool acc = false;
          if (i < N) {
            const double delta = sh.s[i] > 0 ? ch.delta_p : ch.delta_m;
            const double a = 1.0 + (1.0 - sh.d[i]) * delta;
            if (log) sh.rr[i] = (a * a) / (1.0 + delta);
            acc = sh.u[i] * (1.0 + delta) < a * a;
            if (acc) sh.gam[tid] = delta / a;
          }
          const unsigned bal = __ballot_sync(0xffffffffu, acc);
          int* wb = sh.ired + 8 + (round & 1) * 4;
          if ((tid & 31) == 0) wb[tid >> 5] = bal ? (tid & ~31) + __ffs(bal) - 1 : kTeam;
          team_sync();
          ++round;
          int first = kTeam;
#pragma unroll
          for (int w = 0; w < 4; ++w) first = min(first, wb[w]);
          if (first < kTeam) { j = base + first; break; }
        }
        if (j < 0) { start = N; break; }
        const double gamma = sh.gam[(j - start) % kTeam];  // written by the accepting thread of the round
        for (int p = j + 1 + tid; p < N; p += kTeam) {
          double c0 = G[p + (size_t)j * ld], c1 = 0.0, r0 = G[j + (size_t)p * ld], r1 = 0.0;
          int m = 0;
          for (; m + 1 < kk; m += 2) {
            c0 = fma(sh.X[p + m * ldp], sh.Y[m * ldp + j], c0);
            r0 = fma(sh.X[j + m * ldp], sh.Y[m * ldp + p], r0);
            c1 = fma(sh.X[p + (m + 1) * ldp], sh.Y[(m + 1) * ldp + j], c1);
            r1 = fma(sh.X[j + (m + 1) * ldp], sh.Y[(m + 1) * ldp + p], r1);
          }
          if (m < kk) {
            c0 = fma(sh.X[p + m * ldp], sh.Y[m * ldp + j], c0);
            r0 = fma(sh.X[j + m * ldp], sh.Y[m * ldp + p], r0);
          }
          const double xv = gamma * (c0 + c1);
          const double yv = r0 + r1;
          sh.X[p + kk * ldp] = xv;
          sh.Y[kk * ldp + p] = yv;
          sh.d[p] = fma(xv, yv, sh.d[p]);
        }
        if (tid == 0) {
          sh.flip[j] = 1;
          sh.qj[kk] = j;
          sh.qg[kk] = gamma;
        }
        __threadfence_block();
        team_sync();
        if (tid == 0) *sh.qn = kk + 1;  // entries p > j of column kk are visible to everyone
        n_acc += (tid == 0) ? 1.0 : 0.0;
        ++kk;
        start = j + 1;
      }
      if (tid == 0) {
        sh.ired[0] = kk;
        sh.ired[1] = start;
        __threadfence_block();
        *sh.qdone = 1;
      }
    } else {
      // helpers: rows p <= j of every published panel column, in publication order
      const int hid = tid - kTeam, nh = blockDim.x - kTeam;
      int next = 0;
      long long spins = 0;
      while (true) {
        int avail = *sh.qn;
        if (next >= avail) {
          if (*sh.qdone) {
            __threadfence_block();
            avail = *sh.qn;
            if (next >= avail) break;
          } else {
            if (++spins > (1ll << 24)) { ch.acc[HQ_ACC_STATUS] = 2.0; break; }  // bounded wait
            __nanosleep(64);
            continue;
          }
        }
        __threadfence_block();
        const int j = sh.qj[next];
        const double gamma = sh.qg[next];
        for (int p = hid; p <= j; p += nh) {
          double c0 = G[p + (size_t)j * ld], c1 = 0.0, r0 = G[j + (size_t)p * ld], r1 = 0.0;
          int m = 0;
          for (; m + 1 < next; m += 2) {
            c0 = fma(sh.X[p + m * ldp], sh.Y[m * ldp + j], c0);
            r0 = fma(sh.X[j + m * ldp], sh.Y[m * ldp + p], r0);
            c1 = fma(sh.X[p + (m + 1) * ldp], sh.Y[(m + 1) * ldp + j], c1);
            r1 = fma(sh.X[j + (m + 1) * ldp], sh.Y[(m + 1) * ldp + p], r1);
          }
          if (m < next) {
            c0 = fma(sh.X[p + m * ldp], sh.Y[m * ldp + j], c0);
            r0 = fma(sh.X[j + m * ldp], sh.Y[m * ldp + p], r0);
          }
          sh.X[p + next * ldp] = gamma * (c0 + c1);
          sh.Y[next * ldp + p] = (r0 + r1) - (p == j ? 1.0 : 0.0);
        }
        ++next;
      }
    }
    __syncthreads();
    k = sh.ired[0];
    start = sh.ired[1];
    if (k > 0 && (k == kmax || start >= N)) {
      flush_panels(G, ld, N, sh.X, ldp, sh.Y, ldp, k);
      k = 0;
    }
    __syncthreads();
    if (start >= N) break;
  }
  // apply the flips of this slice and optionally log the visit-time ratios
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    if (sh.flip[i]) sh.s[i] = -sh.s[i];
    if (log && log_base + i < ch.ratio_cap) ch.ratios[log_base + i] = sh.rr[i];
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------------
//  Register-panel Metropolis sweep of one slice (N <= blockDim.x, one site per thread).
//
//  Thread p owns site p: its uniform, field, current diagonal G_pp and its row of the
//  delayed-update panels (X[p, :], Y[:, p]) live in registers. Sites of a slice are
//  accepted in increasing order j_0 < j_1 < ..., so for a new flip j only the entries
//  p > j of G's current column / row j can influence later decisions of the slice:
//      col_p = G0[p, j] + sum_m X[p, m] Y[m, j],  row_p = G0[j, p] + sum_m X[j, m] Y[m, p]
//  with Y[m, j] and X[j, m] (j > j_m) published by thread j in shared memory. The entries
//  p <= j_m are filled just before the panel is flushed into G0 with DMMA.
// ---------------------------------------------------------------------------------
template <int KMAX>
__device__ void metropolis_slice_reg(const HqChain& ch, double* G, int ld, const MetroShared& sh, uint32_t& rng,
                                     double& n_acc, int flags, long long log_base) {
  const int N = ch.N;
  const int kmax = ch.kmax < KMAX ? ch.kmax : KMAX;
  const int ldp = panel_ld(N);
  const int p = threadIdx.x;
  const int lane = p & 31, warp = p >> 5, nwarps = blockDim.x >> 5;
  const bool owner = p < N;
  const bool log = (flags & HQ_F_LOG_RATIOS) && ch.ratios;
  double u = 0.0, d = 0.0, dlt = 0.0, rr = 0.0;
  bool flipped = false;
  if (owner) {
    const uint32_t x1 = minstd_mulmod(minstd_pow(2ull * p + 1), rng);
    const uint32_t x2 = minstd_mulmod(kMinstdA, x1);
    u = canonical_from_pair(x1, x2);
    d = G[p + (size_t)p * ld];
    dlt = sh.s[p] > 0 ? ch.delta_p : ch.delta_m;
  }
  rng = minstd_mulmod(minstd_pow(2ull * N), rng);
  double Xr[KMAX], Yr[KMAX];
#pragma unroll
  for (int m = 0; m < KMAX; ++m) { Xr[m] = 0.0; Yr[m] = 0.0; }
  int k = 0, start = 0, parity = 0;
  while (true) {
    // ---- first accepted site >= start: accept iff u (1 + Delta) < a^2 (u < min(1, |r|)) ----
    int cand = INT_MAX;
    if (owner && p >= start) {
      const double a = 1.0 + (1.0 - d) * dlt;
      if (log) rr = (a * a) / (1.0 + dlt);
      if (u * (1.0 + dlt) < a * a) {
        cand = p;
        sh.gam[p] = dlt / a;  // gamma of this site, used only if it is the first
      }
    }
    cand = __reduce_min_sync(0xffffffffu, cand);
    int* wb = sh.ired + 8 + parity * 16;
    parity ^= 1;
    if (lane == 0) wb[warp] = cand;
    __syncthreads();
    int j = INT_MAX;
    for (int w = 0; w < nwarps; ++w) j = min(j, wb[w]);
    if (j == INT_MAX) break;
    const double gamma = sh.gam[j];
    // ---- append column k: entries p > j (later decisions read only those) ----
    if (owner && p > j) {
      double c0 = G[p + (size_t)j * ld], c1 = 0.0, r0 = G[j + (size_t)p * ld], r1 = 0.0;
#pragma unroll
      for (int m = 0; m < KMAX; m += 2) {
        if (m < k) {
          c0 = fma(Xr[m], sh.Y[m * ldp + j], c0);
          r0 = fma(sh.X[j + m * ldp], Yr[m], r0);
        }
        if (m + 1 < k) {
          c1 = fma(Xr[m + 1], sh.Y[(m + 1) * ldp + j], c1);
          r1 = fma(sh.X[j + (m + 1) * ldp], Yr[m + 1], r1);
        }
      }
      const double xv = gamma * (c0 + c1), yv = r0 + r1;
#pragma unroll
      for (int m = 0; m < KMAX; ++m)
        if (m == k) { Xr[m] = xv; Yr[m] = yv; }
      sh.X[p + k * ldp] = xv;
      sh.Y[k * ldp + p] = yv;
      d = fma(xv, yv, d);
    }
    if (p == j) flipped = true;
    if (p == 0) { sh.qj[k] = j; sh.qg[k] = gamma; }
    n_acc += (p == 0) ? 1.0 : 0.0;
    ++k;
    start = j + 1;
    __syncthreads();
    if (k == kmax || start >= N) {
      // ---- fill the entries p <= j_m of the panel, then flush G0 += X Y ----
      if (owner) {
#pragma unroll
        for (int m = 0; m < KMAX; ++m) {
          if (m < k) {
            const int jm = sh.qj[m];
            if (p <= jm) {
              double c = G[p + (size_t)jm * ld], r = G[jm + (size_t)p * ld];
#pragma unroll
              for (int m2 = 0; m2 < KMAX; ++m2)
                if (m2 < m) {
                  c = fma(Xr[m2], sh.Y[m2 * ldp + jm], c);
                  r = fma(sh.X[jm + m2 * ldp], Yr[m2], r);
                }
              Xr[m] = sh.qg[m] * c;
              Yr[m] = r - (p == jm ? 1.0 : 0.0);
              sh.X[p + m * ldp] = Xr[m];
              sh.Y[m * ldp + p] = Yr[m];
            }
          }
        }
      }
      __syncthreads();
      flush_panels(G, ld, N, sh.X, ldp, sh.Y, ldp, k);
      k = 0;
      __syncthreads();
      if (owner) d = G[p + (size_t)p * ld];
      if (start >= N) break;
    }
  }
  if (k > 0) {
    // a slice that ended on a round without acceptance: fill and flush the open panel
    if (owner) {
#pragma unroll
      for (int m = 0; m < KMAX; ++m) {
        if (m < k) {
          const int jm = sh.qj[m];
          if (p <= jm) {
            double c = G[p + (size_t)jm * ld], r = G[jm + (size_t)p * ld];
#pragma unroll
            for (int m2 = 0; m2 < KMAX; ++m2)
              if (m2 < m) {
                c = fma(Xr[m2], sh.Y[m2 * ldp + jm], c);
                r = fma(sh.X[jm + m2 * ldp], Yr[m2], r);
              }
            Xr[m] = sh.qg[m] * c;
            Yr[m] = r - (p == jm ? 1.0 : 0.0);
            sh.X[p + m * ldp] = Xr[m];
            sh.Y[m * ldp + p] = Yr[m];
          }
        }
      }
    }
    __syncthreads();
    flush_panels(G, ld, N, sh.X, ldp, sh.Y, ldp, k);
    __syncthreads();
  }
  if (owner) {
    if (flipped) sh.s[p] = -sh.s[p];
    if (log && log_base + p < ch.ratio_cap) ch.ratios[log_base + p] = rr;
  }
  __syncthreads();
}

// picks the register-panel sweep when every site has its own thread
__device__ void metropolis_dispatch(const HqChain& ch, double* G, int ld, const MetroShared& sh, uint32_t& rng,
                                    double& n_acc, int flags, long long log_base) {
  if (ch.N <= (int)blockDim.x) {
    if (ch.kmax <= 8) metropolis_slice_reg<8>(ch, G, ld, sh, rng, n_acc, flags, log_base);
    else metropolis_slice_reg<16>(ch, G, ld, sh, rng, n_acc, flags, log_base);
  } else {
    metropolis_slice(ch, G, ld, sh, rng, n_acc, flags, log_base);
  }
}

// ---------------------------------------------------------------------------------
//  wrap of G by B(l) (src/dqmc_core.cpp:142-161, src/hubbard.cpp:293-331)
//   up  : G <- e^{V_l} E G E^{-1} e^{-V_l}
//   down: G <- E^{-1} e^{-V_l} G e^{V_l} E
// ---------------------------------------------------------------------------------
__device__ void wrap_slice(const HqChain& ch, double* G, int ld, const int8_t* s, int dir, double* stage) {
  const int N = ch.N;
  if (dir == HQ_UP) {
    apply_expk(ch, G, ld, 0, false, stage);
    apply_expk(ch, G, ld, 1, true, stage);
    HQ_FOR_EACH_ELEM(N, i, j) {
      const double fi = s[i] > 0 ? ch.ev_p : ch.ev_m;
      const double fj = s[j] > 0 ? ch.ev_m : ch.ev_p;
      G[i + (size_t)j * ld] *= fi * fj;
    }
    __syncthreads();
  } else {
    HQ_FOR_EACH_ELEM(N, i, j) {
      const double fi = s[i] > 0 ? ch.ev_m : ch.ev_p;
      const double fj = s[j] > 0 ? ch.ev_p : ch.ev_m;
      G[i + (size_t)j * ld] *= fi * fj;
    }
    __syncthreads();
    apply_expk(ch, G, ld, 0, true, stage);
    apply_expk(ch, G, ld, 1, false, stage);
  }
}

// slice range of interval b: up-sweep intervals are [b*pace+1, min((b+1)*pace, nt)];
// the down sweep visits the same intervals from the top (b counts from tau = beta)
__device__ __host__ inline void interval_range(int nt, int pace, int n_stab, int dir, int b, int& t_lo, int& t_hi) {
  const int bu = (dir == HQ_DOWN) ? (n_stab - 1 - b) : b;
  t_lo = bu * pace + 1;
  t_hi = min((bu + 1) * pace, nt);
}

// ---------------------------------------------------------------------------------
//  k_interval: the update (or no-update) slices of one stabilisation interval.
// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(HQ_INT_THREADS, 1)
k_interval(const HqChain* __restrict__ chains, int nchains, int dir, int b, int flags, int resident) {
  extern __shared__ __align__(16) double smem[];
  __shared__ HqChain ch;
  __shared__ double red[96];
  __shared__ int ired[64];
  const int c = blockIdx.x;
  if (c >= nchains) return;
  if (threadIdx.x == 0) ch = chains[c];
  __syncthreads();
  if (!ch.active || b >= ch.n_stab) return;
  const int N = ch.N;
  int t_lo, t_hi;
  interval_range(ch.nt, ch.pace, ch.n_stab, dir, b, t_lo, t_hi);

  // shared-memory carve-up
  double* p = smem;
  double* G;
  int ld;
  if (resident) {
    G = p;
    ld = smem_ld(N);
    p += (size_t)N * ld;
    copy_mat(G, ld, ch.G, N, N);
  } else {
    G = ch.G;
    ld = N;
  }
  const size_t panels = (size_t)panel_ld(N) * ch.kmax * 2;
  const size_t stage_n = (size_t)8 * (((N + 15) & ~15) + 4);
  double* work = p;
  p += panels > stage_n ? panels : stage_n;
  MetroShared sh;
  sh.X = work;
  sh.Y = work + (size_t)panel_ld(N) * ch.kmax;
  sh.d = p; p += N;
  sh.u = p; p += N;
  sh.rr = p; p += N;
  sh.s = reinterpret_cast<int8_t*>(p);
  sh.flip = sh.s + N;
  sh.ired = ired;
  __shared__ int qj_s[64];
  __shared__ double qg_s[64];
  __shared__ double gam_s[HQ_INT_THREADS];
  sh.gam = gam_s;
  __shared__ int qn_s, qdone_s;
  sh.qj = qj_s;
  sh.qg = qg_s;
  sh.qn = &qn_s;
  sh.qdone = &qdone_s;
  uint32_t rng = *ch.rng;
  double n_acc = 0.0, n_prop = 0.0;
  long long log_base = (flags & HQ_F_LOG_RATIOS) && ch.ratio_count ? *ch.ratio_count : 0;
  __syncthreads();

  const int nsl = t_hi - t_lo + 1;
  for (int step = 0; step < nsl; ++step) {
    const int t = (dir == HQ_DOWN) ? (t_hi - step) : (t_lo + step);
    const int l = t % ch.nt;
    for (int i = threadIdx.x; i < N; i += blockDim.x) sh.s[i] = ch.fields[(size_t)l * N + i];
    __syncthreads();
    if (dir == HQ_UP) {
      wrap_slice(ch, G, ld, sh.s, HQ_UP, work);
      metropolis_dispatch(ch, G, ld, sh, rng, n_acc, flags, log_base);
      n_prop += N;
      log_base += N;
    } else if (dir == HQ_DOWN) {
      metropolis_dispatch(ch, G, ld, sh, rng, n_acc, flags, log_base);
      n_prop += N;
      log_base += N;
      wrap_slice(ch, G, ld, sh.s, HQ_DOWN, work);
    } else {
      wrap_slice(ch, G, ld, sh.s, HQ_UP, work);
    }
    for (int i = threadIdx.x; i < N; i += blockDim.x) ch.fields[(size_t)l * N + i] = sh.s[i];
    // the last slice of the interval is measured after stabilisation
    if (step < nsl - 1) {
      const int lm = (dir == HQ_DOWN) ? ((t - 1) % ch.nt) : l;
      if (flags & HQ_F_MEASURE) measure_slice(G, ld, N, ch.acc, red);
      if ((flags & HQ_F_SNAPSHOT) && ch.snap_tt) copy_mat(ch.snap_tt + (size_t)lm * N * N, N, G, ld, N);
    }
    __syncthreads();
  }
  if (resident) copy_mat(ch.G, N, G, ld, N);
  if (threadIdx.x == 0) {
    *ch.rng = rng;
    ch.acc[HQ_ACC_PROPOSED] += n_prop;
    ch.acc[HQ_ACC_ACCEPTED] += n_acc;
    if ((flags & HQ_F_LOG_RATIOS) && ch.ratio_count) *ch.ratio_count = log_base;
  }
}

// ---------------------------------------------------------------------------------
//  k_bchain: X <- (U_top diag(D_top) or 1), then the B products of interval b:
//   up  : X <- B(t) X = e^{V_t} E X, t ascending            (src/dqmc_core.cpp:190)
//   down: X <- B(t)^T X = E e^{V_t} X, t descending           (src/dqmc_core.cpp:251)
//  dir UP pushes onto the left stack, DOWN onto the right stack; that stack holds b
//  entries before the push (top entry b-1, none when b = 0).
//  init: the right stack at initialisation (src/dqmc_core.cpp:67-87) is the down
//  direction without updates.
// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(HQ_INT_THREADS, 1)
k_bchain(const HqChain* __restrict__ chains, int nchains, int dir, int b, int resident) {
  extern __shared__ __align__(16) double smem[];
  __shared__ HqChain ch;
  __shared__ int8_t s[HQ_MAX_N];
  const int c = blockIdx.x;
  if (c >= nchains) return;
  if (threadIdx.x == 0) ch = chains[c];
  __syncthreads();
  if (!ch.active || b >= ch.n_stab) return;
  const int N = ch.N;
  int t_lo, t_hi;
  interval_range(ch.nt, ch.pace, ch.n_stab, dir, b, t_lo, t_hi);
  const int side = (dir == HQ_DOWN) ? 1 : 0;
  const int top = b - 1;  // the pushing stack holds b entries before this push
  double* X;
  int ld;
  double* p = smem;
  if (resident) { X = p; ld = smem_ld(N); p += (size_t)N * ld; } else { X = ch.X; ld = N; }
  double* stage = p;
  const size_t NN = (size_t)N * N;
  const double* U = top >= 0 ? ch.stackU + ((size_t)side * ch.n_stab + top) * NN : nullptr;
  const double* D = top >= 0 ? ch.stackD + ((size_t)side * ch.n_stab + top) * N : nullptr;
  HQ_FOR_EACH_ELEM(N, i, j) X[i + (size_t)j * ld] = U ? U[i + (size_t)j * N] * D[j] : (i == j ? 1.0 : 0.0);
  __syncthreads();
  const int nsl = t_hi - t_lo + 1;
  for (int step = 0; step < nsl; ++step) {
    const int t = (dir == HQ_DOWN) ? (t_hi - step) : (t_lo + step);
    const int l = t % ch.nt;
    for (int i = threadIdx.x; i < N; i += blockDim.x) s[i] = ch.fields[(size_t)l * N + i];
    __syncthreads();
    if (dir == HQ_DOWN) {
      scale_rows(X, ld, N, s, ch.ev_p, ch.ev_m);
      __syncthreads();
      apply_expk(ch, X, ld, 0, false, stage);
    } else {
      apply_expk(ch, X, ld, 0, false, stage);
      scale_rows(X, ld, N, s, ch.ev_p, ch.ev_m);
      __syncthreads();
    }
  }
  if (resident) copy_mat(ch.X, N, X, ld, N);
}

// ---------------------------------------------------------------------------------
//  k_udt: UDV factorisation X P = Q R of the stack push, X = Q D T with D = |diag R| and
//  T = D^-1 R P^T (the role of dgesvd in include/utils/svd_stack.hpp:107-175).
//  P sorts the columns of X by decreasing norm once ("pre-pivoting", C. Bauer, Fast and
//  stable determinant quantum Monte Carlo, SciPost Phys. Core 2, 011 (2020)); the QR of
//  the sorted matrix is blocked Householder in panels of kQB columns with compact-WY
//  trailing updates A <- (I - V T^T V^T) A, whose two products run on DMMA; Q is formed
//  in place by the same blocks backwards (Q = B_0 B_1 ..., B_p = I - V_p T_p V_p^T).
//  Output: U (= Q) and D into stack entry b of the pushing stack, T into W0.
// ---------------------------------------------------------------------------------
constexpr int kQB = 16;

// unblocked Householder QR of the panel columns [p0, p1) (rows p0..N-1), dlarfg convention
__device__ void qr_panel(double* A, int ld, int N, int p0, int p1, double* tau) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c = p0; c < p1; ++c) {
    if (warp == 0) {
      double xs = 0.0;
      for (int r = c + 1 + lane; r < N; r += 32) { const double v = A[r + (size_t)c * ld]; xs = fma(v, v, xs); }
      xs = warp_sum(xs);
      const double alpha = A[c + (size_t)c * ld];
      double ti = 0.0, beta = alpha;
      if (xs > 0.0) {
        beta = -copysign(hypot(alpha, sqrt(xs)), alpha);
        ti = (beta - alpha) / beta;
        const double sc = 1.0 / (alpha - beta);
        for (int r = c + 1 + lane; r < N; r += 32) A[r + (size_t)c * ld] *= sc;
      }
      __syncwarp();
      if (lane == 0) { A[c + (size_t)c * ld] = beta; tau[c] = ti; }
    }
    __syncthreads();
    // apply H_c to the remaining panel columns, one warp per column
    const double ti = tau[c];
    const int j = c + 1 + warp;
    if (ti != 0.0 && j < p1) {
      double w = (lane == 0) ? A[c + (size_t)j * ld] : 0.0;
      for (int r = c + 1 + lane; r < N; r += 32) w = fma(A[r + (size_t)c * ld], A[r + (size_t)j * ld], w);
      w = warp_sum(w) * ti;
      if (lane == 0) A[c + (size_t)j * ld] -= w;
      for (int r = c + 1 + lane; r < N; r += 32) A[r + (size_t)j * ld] = fma(-w, A[r + (size_t)c * ld], A[r + (size_t)j * ld]);
    }
    __syncthreads();
  }
}

// V of the panel [p0, p0+m) with explicit unit diagonal and zeros above (columns >= m
// zero), and the triangular factor T of H_p0 ... H_p0+m-1 = I - V T V^T
__device__ void wy_factor(const double* A, int ld, int N, int p0, int m, const double* tau, double* Vb, int ldv,
                          double* T, double* S) {
  for (int q = threadIdx.x >> 5; q < kQB; q += blockDim.x >> 5)
    for (int r = p0 + (threadIdx.x & 31); r < N; r += 32) {
      const int c = p0 + q;
      Vb[r + q * ldv] = (q >= m || r < c) ? 0.0 : (r == c ? 1.0 : A[r + (size_t)c * ld]);
    }
  __syncthreads();
  // S = V^T V (upper triangle), rows >= p0 + b are the only nonzero overlap
  for (int t = threadIdx.x; t < kQB * kQB; t += blockDim.x) {
    const int a = t / kQB, bb = t % kQB;
    double acc = 0.0;
    if (a <= bb && bb < m)
      for (int r = p0 + bb; r < N; ++r) acc = fma(Vb[r + a * ldv], Vb[r + bb * ldv], acc);
    S[t] = acc;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int i = threadIdx.x;
    for (int j = 0; j < kQB; ++j) {
      if (i < kQB) {
        double v = 0.0;
        if (j < m) {
          if (i == j) v = tau[p0 + j];
          else if (i < j) {
            double acc = 0.0;
            for (int l = i; l < j; ++l) acc = fma(T[i * kQB + l], S[l * kQB + j], acc);
            v = -tau[p0 + j] * acc;
          }
        }
        T[i * kQB + j] = v;
      }
    }
  }
  __syncthreads();
}

// A[p0:, col0:col0+nc] <- (I - V op(T) V^T) A[p0:, col0:col0+nc]; op(T) = T^T if trans
__device__ void wy_apply(double* A, int ld, int N, int p0, const double* Vb, int ldv, const double* T, bool trans,
                         double* W, int ldw, int col0, int nc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  // W = V^T A_sub (kQB x nc) with DMMA: m16 = the panel columns, k = rows p0..N-1
  const int nt8 = (nc + 7) / 8;
  for (int t = warp; t < nt8; t += nwarps) {
    const int cb = t * 8 + g;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int r0 = p0; r0 < N; r0 += 4) {
      const int r = r0 + q;
      const double a0 = (r < N) ? Vb[r + g * ldv] : 0.0;
      const double a1 = (r < N) ? Vb[r + (g + 8) * ldv] : 0.0;
      const double b0 = (r < N && cb < nc) ? A[r + (size_t)(col0 + cb) * ld] : 0.0;
      dmma_16x8x4(acc, a0, a1, b0);
    }
    const int c = t * 8 + 2 * q;
    if (c < nc) { W[g * ldw + c] = acc[0]; W[(g + 8) * ldw + c] = acc[2]; }
    if (c + 1 < nc) { W[g * ldw + c + 1] = acc[1]; W[(g + 8) * ldw + c + 1] = acc[3]; }
  }
  __syncthreads();
  // W <- -op(T) W, one thread per column
  for (int c = threadIdx.x; c < nc; c += blockDim.x) {
    double w[kQB];
#pragma unroll
    for (int l = 0; l < kQB; ++l) w[l] = W[l * ldw + c];
#pragma unroll
    for (int i = 0; i < kQB; ++i) {
      double acc = 0.0;
#pragma unroll
      for (int l = 0; l < kQB; ++l) acc = fma(trans ? T[l * kQB + i] : T[i * kQB + l], w[l], acc);
      W[i * ldw + c] = -acc;
    }
  }
  __syncthreads();
  // A_sub += V (-op(T) W)
  rank_update(A + p0 + (size_t)col0 * ld, ld, N - p0, nc, Vb + p0, ldv, W, ldw, kQB);
  __syncthreads();
}

__global__ void __launch_bounds__(HQ_THREADS, 1)
k_udt(const HqChain* __restrict__ chains, int nchains, int side, int unused, int b, int resident) {
  extern __shared__ __align__(16) double smem[];
  __shared__ HqChain ch;
  const int c = blockIdx.x;
  if (c >= nchains) return;
  if (threadIdx.x == 0) ch = chains[c];
  __syncthreads();
  if (!ch.active || b >= ch.n_stab) return;
  const int N = ch.N;
  const int entry = b;  // push position: the pushing stack holds b entries
  const int ldp = panel_ld(N);
  double* A;
  int ld;
  double* p = smem;
  if (resident) { A = p; ld = smem_ld(N); p += (size_t)N * ld; }
  else { A = ch.W3; ld = N; }  // W3 is free during a push
  double* Vb = p; p += (size_t)ldp * kQB;
  double* W = p; p += (size_t)kQB * ldp;
  double* T = p; p += kQB * kQB;
  double* S = p; p += kQB * kQB;
  double* tau = p; p += N;
  double* nrm = p; p += N;
  int* order = reinterpret_cast<int*>(p);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const double* X = ch.X;
  // ---- pre-pivoting: columns by decreasing norm (ties by index) ----
  for (int j = warp; j < N; j += nwarps) {
    double s2 = 0.0;
    for (int i = lane; i < N; i += 32) { const double v = X[i + (size_t)j * N]; s2 = fma(v, v, s2); }
    s2 = warp_sum(s2);
    if (lane == 0) nrm[j] = s2;
  }
  __syncthreads();
  for (int j = threadIdx.x; j < N; j += blockDim.x) {
    const double nj = nrm[j];
    int rank = 0;
    for (int i = 0; i < N; ++i) {
      const double ni = nrm[i];
      rank += (ni > nj || (ni == nj && i < j)) ? 1 : 0;
    }
    order[rank] = j;
  }
  __syncthreads();
  HQ_FOR_EACH_ELEM(N, i, j) A[i + (size_t)j * ld] = X[i + (size_t)order[j] * N];
  __syncthreads();
  // ---- blocked Householder QR ----
  for (int p0 = 0; p0 < N; p0 += kQB) {
    const int p1 = min(p0 + kQB, N);
    qr_panel(A, ld, N, p0, p1, tau);
    if (p1 < N) {
      wy_factor(A, ld, N, p0, p1 - p0, tau, Vb, ldp, T, S);
      wy_apply(A, ld, N, p0, Vb, ldp, T, true, W, ldp, p1, N - p1);
    }
  }
  // ---- D = |diag R|, T = D^-1 R P^T (T[:, order[c]] = row-scaled R[:, c]) ----
  const size_t NN = (size_t)N * N;
  double* Dout = ch.stackD + ((size_t)side * ch.n_stab + entry) * N;
  double* Tout = ch.W0;
  for (int r = threadIdx.x; r < N; r += blockDim.x) {
    const double dr = fabs(A[r + (size_t)r * ld]);
    Dout[r] = dr;
    nrm[r] = dr;
  }
  __syncthreads();
  HQ_FOR_EACH_ELEM(N, r, cc) {
    const double v = (r <= cc) ? A[r + (size_t)cc * ld] / nrm[r] : 0.0;
    Tout[r + (size_t)order[cc] * N] = (nrm[r] != 0.0) ? v : (r == cc ? 1.0 : 0.0);
  }
  __syncthreads();
  // ---- form Q in place, panels backwards ----
  for (int p0 = ((N - 1) / kQB) * kQB; p0 >= 0; p0 -= kQB) {
    const int p1 = min(p0 + kQB, N);
    if (p1 < N) {
      wy_factor(A, ld, N, p0, p1 - p0, tau, Vb, ldp, T, S);
      wy_apply(A, ld, N, p0, Vb, ldp, T, false, W, ldp, p1, N - p1);
    }
    // unblocked formation of the panel's own columns (dorg2r restricted to the panel)
    for (int i = p1 - 1; i >= p0; --i) {
      const double ti = tau[i];
      const int j = i + 1 + warp;
      if (ti != 0.0 && j < p1) {
        double w = (lane == 0) ? A[i + (size_t)j * ld] : 0.0;
        for (int r = i + 1 + lane; r < N; r += 32) w = fma(A[r + (size_t)i * ld], A[r + (size_t)j * ld], w);
        w = warp_sum(w) * ti;
        if (lane == 0) A[i + (size_t)j * ld] -= w;
        for (int r = i + 1 + lane; r < N; r += 32) A[r + (size_t)j * ld] = fma(-w, A[r + (size_t)i * ld], A[r + (size_t)j * ld]);
      }
      __syncthreads();
      for (int r = i + 1 + threadIdx.x; r < N; r += blockDim.x) A[r + (size_t)i * ld] *= -ti;
      if (threadIdx.x == 0) A[i + (size_t)i * ld] = 1.0 - ti;
      for (int r = threadIdx.x; r < i; r += blockDim.x) A[r + (size_t)i * ld] = 0.0;
      __syncthreads();
    }
  }
  double* Uout = ch.stackU + ((size_t)side * ch.n_stab + entry) * NN;
  copy_mat(Uout, N, A, ld, N);
}

// ---------------------------------------------------------------------------------
//  k_invert: in-place Gauss-Jordan inverse with partial (row) pivoting of the N x N
//  matrix at `which` (0: W1, 1: W2, 2: W3, 3: W5), blocked by panels of kGJ pivots.
//
//  Unblocked Gauss-Jordan reads and writes the whole matrix at every pivot, which in
//  shared memory costs ~N^3/8 cycles. Here the pivots of a panel are applied to the
//  panel's own columns only (one thread per row); their composition acts on every other
//  column j as  A[:, j] += (P - E_K) A[K, j]  (P: the panel columns afterwards, K: the
//  panel's pivot rows, E_K: their identity columns), a rank-kGJ update done with the DMMA
//  flush of the Metropolis panels. The row interchanges of a panel are applied to the
//  other columns before that update; the column interchanges that undo them are a
//  gather on the way out. Failure (zero pivot / non-finite) sets acc[STATUS].
// ---------------------------------------------------------------------------------
constexpr int kGJ = 16;

__global__ void __launch_bounds__(HQ_THREADS, 1)
k_invert(const HqChain* __restrict__ chains, int nchains, int b, int which, int resident) {
  extern __shared__ __align__(16) double smem[];
  __shared__ HqChain ch;
  const int c = blockIdx.x;
  if (c >= nchains) return;
  if (threadIdx.x == 0) ch = chains[c];
  __syncthreads();
  if (!ch.active || b >= ch.n_stab) return;
  const int N = ch.N;
  double* src = which == 0 ? ch.W1 : (which == 1 ? ch.W2 : (which == 2 ? ch.W3 : ch.W5));
  double* A;
  int ld;
  double* p = smem;
  if (resident) { A = p; ld = smem_ld(N); p += (size_t)N * ld; copy_mat(A, ld, src, N, N); }
  else { A = src; ld = N; }
  const int ldp = panel_ld(N);
  double* Wp = p; p += (size_t)ldp * kGJ;   // N x kGJ, column-major
  double* Bf = p; p += (size_t)ldp * kGJ;   // kGJ x N, row-major
  int* perm = reinterpret_cast<int*>(p);
  int* gidx = perm + N;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  for (int p0 = 0; p0 < N; p0 += kGJ) {
    const int nb = min(kGJ, N - p0);
    for (int q = 0; q < nb; ++q) {
      const int k = p0 + q;
      if (warp == 0) {
        // pivot search in column k over rows k..N-1, swap within the panel, scale the pivot row
        double best = -1.0;
        int bi = k;
        for (int r = k + lane; r < N; r += 32) {
          const double v = fabs(A[r + (size_t)k * ld]);
          if (v > best) { best = v; bi = r; }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const double ob = __shfl_xor_sync(0xffffffffu, best, o);
          const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
          if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
        }
        const bool ok = (best > 0.0) && isfinite(best);
        if (lane < nb && bi != k) {
          const int j = p0 + lane;
          const double t0 = A[k + (size_t)j * ld];
          A[k + (size_t)j * ld] = A[bi + (size_t)j * ld];
          A[bi + (size_t)j * ld] = t0;
        }
        __syncwarp();
        const double pv = A[k + (size_t)k * ld];
        const double pinv = ok ? 1.0 / pv : 0.0;
        __syncwarp();
        if (lane < nb) {
          const int j = p0 + lane;
          const double v = (j == k) ? 1.0 : A[k + (size_t)j * ld];
          A[k + (size_t)j * ld] = v * pinv;
        }
        if (lane == 0) {
          perm[k] = bi;
          if (!ok) ch.acc[HQ_ACC_STATUS] = 1.0;
        }
      }
      __syncthreads();
      // eliminate column k from every other row of the panel (one thread per row)
      for (int r = threadIdx.x; r < N; r += blockDim.x) {
        if (r == k) continue;
        const double f = A[r + (size_t)k * ld];
#pragma unroll 4
        for (int jj = 0; jj < nb; ++jj) {
          const int j = p0 + jj;
          const double base = (j == k) ? 0.0 : A[r + (size_t)j * ld];
          A[r + (size_t)j * ld] = fma(-f, A[k + (size_t)j * ld], base);
        }
      }
      __syncthreads();
    }
    // rows interchanges of this panel on every other column, then the pivot rows into Bf
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
      const bool in_panel = (j >= p0 && j < p0 + nb);
      if (!in_panel) {
        for (int q = 0; q < nb; ++q) {
          const int k = p0 + q, pr = perm[k];
          if (pr != k) {
            const double t0 = A[k + (size_t)j * ld];
            A[k + (size_t)j * ld] = A[pr + (size_t)j * ld];
            A[pr + (size_t)j * ld] = t0;
          }
        }
      }
      for (int q = 0; q < nb; ++q) Bf[q * ldp + j] = in_panel ? 0.0 : A[p0 + q + (size_t)j * ld];
    }
    for (int r = threadIdx.x; r < N; r += blockDim.x)
      for (int q = 0; q < nb; ++q) Wp[r + q * ldp] = A[r + (size_t)(p0 + q) * ld] - (r == p0 + q ? 1.0 : 0.0);
    __syncthreads();
    // A[:, j] += Wp Bf[:, j] for every column outside the panel (Bf is zero on the panel)
    flush_panels(A, ld, N, Wp, ldp, Bf, ldp, nb);
    __syncthreads();
  }
  // undo the row interchanges as column interchanges in reverse order: column j of the
  // inverse is column gidx[j] of A
  if (threadIdx.x == 0) {
    for (int j = 0; j < N; ++j) gidx[j] = j;
    for (int k = N - 1; k >= 0; --k) {
      const int t0 = gidx[k]; gidx[k] = gidx[perm[k]]; gidx[perm[k]] = t0;
    }
  }
  __syncthreads();
  if (resident) {
    HQ_FOR_EACH_ELEM(N, i, j) src[i + (size_t)j * N] = A[i + (size_t)gidx[j] * ld];
  } else {
    for (int k = N - 1; k >= 0; --k) {
      const int q = perm[k];
      if (q != k)
        for (int r = threadIdx.x; r < N; r += blockDim.x) {
          const double t0 = A[r + (size_t)k * ld];
          A[r + (size_t)k * ld] = A[r + (size_t)q * ld];
          A[r + (size_t)q * ld] = t0;
        }
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------------
//  k_gemm: batched C = alpha * op(A) diag(f(ks)) op(B) * rowscale * colscale + beta C.
//  64 x 64 output tile per CTA, 4 warps (each 32 x 32 = 2 x 4 DMMA m16n8k4 tiles),
//  k-chunks of 16 staged in shared memory.
// ---------------------------------------------------------------------------------
__device__ __forceinline__ double vscale(const double* v, int mode, int i) {
  if (!v || mode == 0) return 1.0;
  const double x = v[i];
  if (mode == 1) return x;
  if (mode == 2) return 1.0 / fmax(x, 1.0);
  return fmin(x, 1.0);
}

constexpr int GBM = 64, GBN = 64, GBK = 16, GLD = 68;

// 8-byte asynchronous global -> shared copy; zero-fills (reads 0 bytes of `src`, which
// the callers keep pointing at the operand's base) when `valid` is false
__device__ __forceinline__ void cp_async_8(double* dst, const double* src, bool valid) {
  const unsigned saddr = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  const int nbytes = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(saddr), "l"(src), "r"(nbytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int NPEND>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(NPEND)); }

__device__ __forceinline__ void gemm_load_chunk(const HqGemmJob& J, int m0, int n0, int k0, double* sA, double* sB) {
  // op(A) tile rows m0..m0+63, cols k0..k0+15 -> sA[k][m]; op(B) rows k0..k0+15, cols n0..n0+63 -> sB[k][n]
  for (int idx = threadIdx.x; idx < GBM * GBK; idx += blockDim.x) {
    int m, k;
    if (!J.ta) { m = idx % GBM; k = idx / GBM; } else { k = idx % GBK; m = idx / GBK; }
    const int gm = m0 + m, gk = k0 + k;
    const bool ok = gm < J.M && gk < J.K;
    const double* src = ok ? (!J.ta ? J.A + gm + (size_t)gk * J.lda : J.A + gk + (size_t)gm * J.lda) : J.A;
    cp_async_8(sA + k * GLD + m, src, ok);
  }
  for (int idx = threadIdx.x; idx < GBK * GBN; idx += blockDim.x) {
    int k, n;
    if (!J.tb) { k = idx % GBK; n = idx / GBK; } else { n = idx % GBN; k = idx / GBN; }
    const int gk = k0 + k, gn = n0 + n;
    const bool ok = gk < J.K && gn < J.Nc;
    const double* src = ok ? (!J.tb ? J.B + gk + (size_t)gn * J.ldb : J.B + gn + (size_t)gk * J.ldb) : J.B;
    cp_async_8(sB + k * GLD + n, src, ok);
  }
}

__global__ void __launch_bounds__(128)
k_gemm(const HqGemmJob* __restrict__ jobs, int njobs, int tiles_n) {
  __shared__ __align__(16) double sA[2][GBK * GLD];
  __shared__ __align__(16) double sB[2][GBK * GLD];
  __shared__ double sK[2][GBK];
  __shared__ double red[32];
  const int jb = blockIdx.y;
  if (jb >= njobs) return;
  const HqGemmJob J = jobs[jb];
  if (!J.active) return;
  const int tm = blockIdx.x / tiles_n, tn = blockIdx.x % tiles_n;
  const int m0 = tm * GBM, n0 = tn * GBN;
  if (m0 >= J.M || n0 >= J.Nc) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
  double acc[2][4][4];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = acc[a][b][2] = acc[a][b][3] = 0.0;
  const int nchunks = (J.K + GBK - 1) / GBK;
  gemm_load_chunk(J, m0, n0, 0, sA[0], sB[0]);
  if (threadIdx.x < GBK) sK[0][threadIdx.x] = (threadIdx.x < J.K) ? vscale(J.ks, J.ks_mode, threadIdx.x) : 0.0;
  cp_async_commit();
  for (int c = 0; c < nchunks; ++c) {
    const int cur = c & 1;
    if (c + 1 < nchunks) {
      const int k1 = (c + 1) * GBK;
      gemm_load_chunk(J, m0, n0, k1, sA[cur ^ 1], sB[cur ^ 1]);
      if (threadIdx.x < GBK) sK[cur ^ 1][threadIdx.x] = (k1 + threadIdx.x < J.K) ? vscale(J.ks, J.ks_mode, k1 + threadIdx.x) : 0.0;
    }
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const double* A_ = sA[cur];
    const double* B_ = sB[cur];
#pragma unroll
    for (int kk = 0; kk < GBK; kk += 4) {
      double a[2][2], bb[4];
      const double kscale = sK[cur][kk + q];
#pragma unroll
      for (int a_ = 0; a_ < 2; ++a_) {
        a[a_][0] = A_[(kk + q) * GLD + wm + a_ * 16 + g] * kscale;
        a[a_][1] = A_[(kk + q) * GLD + wm + a_ * 16 + g + 8] * kscale;
      }
#pragma unroll
      for (int b_ = 0; b_ < 4; ++b_) bb[b_] = B_[(kk + q) * GLD + wn + b_ * 8 + g];
#pragma unroll
      for (int a_ = 0; a_ < 2; ++a_)
#pragma unroll
        for (int b_ = 0; b_ < 4; ++b_) dmma_16x8x4(acc[a_][b_], a[a_][0], a[a_][1], bb[b_]);
    }
    __syncthreads();
  }
  cp_async_wait<0>();
  // epilogue
  double emax = -INFINITY;
#pragma unroll
  for (int a_ = 0; a_ < 2; ++a_)
#pragma unroll
    for (int b_ = 0; b_ < 4; ++b_)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int gm = m0 + wm + a_ * 16 + g + ((e & 2) ? 8 : 0);
        const int gn = n0 + wn + b_ * 8 + 2 * q + (e & 1);
        if (gm < J.M && gn < J.Nc) {
          double v = J.alpha * acc[a_][b_][e] * vscale(J.rs, J.rs_mode, gm) * vscale(J.cs, J.cs_mode, gn);
          double* cp = J.C + gm + (size_t)gn * J.ldc;
          const double old = (J.beta != 0.0 || J.epi == 1) ? *cp : 0.0;
          if (J.beta != 0.0) v = fma(J.beta, old, v);
          if (J.epi == 1) emax = fmax(emax, v - old);
          *cp = v;
        }
      }
  if (J.epi == 1 && J.err_out) {
    emax = block_max(emax, red);
    if (threadIdx.x == 0) atomic_max_double(J.err_out, emax);
  }
}

// ---------------------------------------------------------------------------------
//  k_measure: estimators + snapshot of G after a stabilisation (slice `lslice`
//  computed from the interval), the last slice of every interval.
// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(HQ_THREADS)
k_measure(const HqChain* __restrict__ chains, int nchains, int dir, int b, int flags) {
  __shared__ HqChain ch;
  __shared__ double red[96];
  const int c = blockIdx.x;
  if (c >= nchains) return;
  if (threadIdx.x == 0) ch = chains[c];
  __syncthreads();
  if (!ch.active || b >= ch.n_stab) return;
  const int N = ch.N;
  int t_lo, t_hi;
  interval_range(ch.nt, ch.pace, ch.n_stab, dir, b, t_lo, t_hi);
  // up / dynamic: the last slice is t_hi, stored at t_hi % nt; down: t_lo, stored at t_lo - 1
  const int lm = (dir == HQ_DOWN) ? ((t_lo - 1) % ch.nt) : (t_hi % ch.nt);
  if (flags & HQ_F_MEASURE) measure_slice(ch.G, N, N, ch.acc, red);
  if ((flags & HQ_F_SNAPSHOT) && ch.snap_tt) copy_mat(ch.snap_tt + (size_t)lm * N * N, N, ch.G, N, N);
}

// ---------------------------------------------------------------------------------
//  Dynamic (time-displaced) sweep, src/dqmc_core.cpp:291-390. Per slice t:
//    G(t,t) <- B G B^-1 ; G(t,0) <- B G(t,0) ; G(0,t) <- G(0,t) B^-1
//  k_dyn_slices applies this for the interval's slices to one of the three matrices per
//  CTA (blockIdx.y = 0: G(t,t), 1: G(t,0), 2: G(0,t)), except for the last slice which
//  is rebuilt by the boundary step, and stores the per-slice results.
// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(HQ_INT_THREADS, 1)
k_dyn_slices(const HqChain* __restrict__ chains, int nchains, int b, int flags, int resident) {
  extern __shared__ __align__(16) double smem[];
  __shared__ HqChain ch;
  __shared__ int8_t s[HQ_MAX_N];
  const int c = blockIdx.x, which = blockIdx.y;
  if (c >= nchains) return;
  if (threadIdx.x == 0) ch = chains[c];
  __syncthreads();
  if (!ch.active || b >= ch.n_stab) return;
  const int N = ch.N;
  int t_lo, t_hi;
  interval_range(ch.nt, ch.pace, ch.n_stab, HQ_UP, b, t_lo, t_hi);
  double* src = which == 0 ? ch.G : (which == 1 ? ch.Gt0 : ch.G0t);
  double* snap = which == 0 ? ch.snap_tt : (which == 1 ? ch.snap_t0 : ch.snap_0t);
  double* M;
  int ld;
  double* p = smem;
  if (resident) { M = p; ld = smem_ld(N); p += (size_t)N * ld; copy_mat(M, ld, src, N, N); }
  else { M = src; ld = N; }
  double* stage = p;
  __syncthreads();
  const int nsl = t_hi - t_lo + 1;
  for (int step = 0; step < nsl; ++step) {
    const int t = t_lo + step;
    const int l = t % ch.nt;
    for (int i = threadIdx.x; i < N; i += blockDim.x) s[i] = ch.fields[(size_t)l * N + i];
    __syncthreads();
    if (which != 2) {  // left multiplication by B(l) = e^V E
      apply_expk(ch, M, ld, 0, false, stage);
      scale_rows(M, ld, N, s, ch.ev_p, ch.ev_m);
      __syncthreads();
    }
    if (which != 1) {  // right multiplication by B(l)^-1 = E^-1 e^-V
      apply_expk(ch, M, ld, 1, true, stage);
      scale_cols(M, ld, N, s, ch.ev_m, ch.ev_p);
      __syncthreads();
    }
    if (step < nsl - 1 && snap) copy_mat(snap + (size_t)l * N * N, N, M, ld, N);
    __syncthreads();
  }
  if (resident) copy_mat(src, N, M, ld, N);
}

// G(t,0) <- G(t,t) and G(0,t) <- G(t,t) - 1 at the start of a dynamic sweep
// (src/dqmc_core.cpp:302-303)
__global__ void k_dyn_start(const HqChain* __restrict__ chains, int nchains) {
  const int c = blockIdx.x;
  if (c >= nchains) return;
  const HqChain& ch = chains[c];
  if (!ch.active) return;
  const int N = ch.N;
  for (int idx = threadIdx.x; idx < N * N; idx += blockDim.x) {
    const int i = idx % N, j = idx / N;
    const double v = ch.G[idx];
    ch.Gt0[idx] = v;
    ch.G0t[idx] = v - (i == j ? 1.0 : 0.0);
  }
}

// dynamic estimators of one slice l from G(t,0), G(0,t) (include/observable_methods.hpp:
// 110-120, 178-195) and the displacement-summed g(d) = sum_i G(t,0)[i+d, i] for G(k,t)
// (:84-103). dyn_acc layout: [0][nt] spin, [1][nt] ldos, [2 + d][nt] g(d) for d < N.
__device__ void dyn_measure(const HqChain& ch, const double* Gt0, const double* G0t, int l, double* red) {
  const int N = ch.N, L = ch.L;
  double sp = 0.0, ld = 0.0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const double a = Gt0[i + (size_t)i * N], b = G0t[i + (size_t)i * N];
    sp -= 2.0 * a * b;
    ld += a;
  }
  sp = block_sum(sp, red);
  ld = block_sum(ld, red);
  if (threadIdx.x == 0) {
    ch.dyn_acc[0 * ch.nt + l] += sp / (2.0 * N);
    ch.dyn_acc[1 * ch.nt + l] += ld / N;
  }
  // g(d): d = dx + L dy, sum over i of G[(xi+dx, yi+dy), i]
  for (int d = threadIdx.x; d < N; d += blockDim.x) {
    const int dx = d % L, dy = d / L;
    double acc = 0.0;
    for (int i = 0; i < N; ++i) {
      const int xi = i % L, yi = i / L;
      const int j = (xi + dx) % L + L * ((yi + dy) % L);
      acc += Gt0[j + (size_t)i * N];
    }
    ch.dyn_acc[(size_t)(2 + d) * ch.nt + l] += acc;
  }
}

// measure the dynamic estimators of every slice of interval b from the snapshots
// (slices of the interval other than the last) or from the fresh G's (the last one).
__global__ void __launch_bounds__(HQ_THREADS)
k_dyn_measure(const HqChain* __restrict__ chains, int nchains, int b, int last_only) {
  __shared__ HqChain ch;
  __shared__ double red[32];
  const int c = blockIdx.x;
  if (c >= nchains) return;
  if (threadIdx.x == 0) ch = chains[c];
  __syncthreads();
  if (!ch.active || b >= ch.n_stab) return;
  const int N = ch.N;
  int t_lo, t_hi;
  interval_range(ch.nt, ch.pace, ch.n_stab, HQ_UP, b, t_lo, t_hi);
  const size_t NN = (size_t)N * N;
  for (int t = last_only ? t_hi : t_lo; t <= t_hi; ++t) {
    const int l = t % ch.nt;
    const double* gt0;
    const double* g0t;
    if (t == t_hi) { gt0 = ch.Gt0; g0t = ch.G0t; }
    else { gt0 = ch.snap_t0 + l * NN; g0t = ch.snap_0t + l * NN; }
    dyn_measure(ch, gt0, g0t, l, red);
    __syncthreads();
  }
}

// at a dynamic boundary: copy the fresh G's into the snapshots of the boundary slice
// with the tau = 0 convention (src/dqmc_core.cpp:379-387)
__global__ void k_dyn_store(const HqChain* __restrict__ chains, int nchains, int b) {
  const int c = blockIdx.x;
  if (c >= nchains) return;
  const HqChain& ch = chains[c];
  if (!ch.active || b >= ch.n_stab) return;
  const int N = ch.N;
  int t_lo, t_hi;
  interval_range(ch.nt, ch.pace, ch.n_stab, HQ_UP, b, t_lo, t_hi);
  const int l = t_hi % ch.nt;
  const size_t NN = (size_t)N * N;
  for (int idx = threadIdx.x; idx < N * N; idx += blockDim.x) {
    const int i = idx % N, j = idx / N;
    const double gtt = ch.G[idx];
    if (ch.snap_tt) ch.snap_tt[l * NN + idx] = gtt;
    if (l == 0) {
      // at tau = beta the stored pair is G(0,0), G(0,0) - 1; the propagated matrices
      // are replaced likewise
      ch.Gt0[idx] = gtt;
      ch.G0t[idx] = gtt - (i == j ? 1.0 : 0.0);
    }
    if (ch.snap_t0) ch.snap_t0[l * NN + idx] = ch.Gt0[idx];
    if (ch.snap_0t) ch.snap_0t[l * NN + idx] = ch.G0t[idx];
  }
}

// commit the freshly built G(t,t), G(t,0), G(0,t) (in W3, W0, W5) after recording the
// signed wrap errors (src/dqmc_core.cpp:334-344)
__global__ void __launch_bounds__(HQ_THREADS) k_dyn_commit(const HqChain* __restrict__ chains, int nchains, int b) {
  __shared__ double red[32];
  const int c = blockIdx.x;
  if (c >= nchains) return;
  const HqChain& ch = chains[c];
  if (!ch.active || b >= ch.n_stab) return;
  const int NN = ch.N * ch.N;
  double ett = -INFINITY, edyn = -INFINITY;
  for (int idx = threadIdx.x; idx < NN; idx += blockDim.x) {
    const double ftt = ch.W3[idx], ft0 = ch.W0[idx], f0t = ch.W4[idx];
    ett = fmax(ett, ftt - ch.G[idx]);
    edyn = fmax(edyn, fmax(ft0 - ch.Gt0[idx], f0t - ch.G0t[idx]));
    ch.G[idx] = ftt;
    ch.Gt0[idx] = ft0;
    ch.G0t[idx] = f0t;
  }
  ett = block_max(ett, red);
  edyn = block_max(edyn, red);
  if (threadIdx.x == 0) {
    ch.acc[HQ_ACC_WRAP_TT] = fmax(ch.acc[HQ_ACC_WRAP_TT], ett);
    ch.acc[HQ_ACC_WRAP_DYN] = fmax(ch.acc[HQ_ACC_WRAP_DYN], edyn);
  }
}

// ---------------------------------------------------------------------------------
//  Adjoint of log|det(1 + B(nt-1)...B(0))| (no counterpart in the reference).
//  With G_l = (1 + B_l..B_1 B_nt..B_{l+1})^-1 the G of the up sweep after slice l:
//    d/dmu    = dt sum_l tr(1 - G_l)
//    d/dalpha = sum_l sum_i s_li (1 - G_l)_ii
//    d/dE     : tr(dE E^-1 D),  D = sum_l e^{-V_l} (1 - G_l) e^{V_l}
//  A no-update up pass wraps G slice by slice and is rebuilt from the stacks every
//  `pace` slices (the checkpoints), so no slice is stored. D accumulates in W4.
// ---------------------------------------------------------------------------------
__device__ void adj_accum(const HqChain& ch, const double* G, int ld, const int8_t* s, double* red) {
  const int N = ch.N;
  double tr = 0.0, sa = 0.0;
  for (int idx = threadIdx.x; idx < N * N; idx += blockDim.x) {
    const int i = idx % N, j = idx / N;
    const double one_m = (i == j ? 1.0 : 0.0) - G[i + (size_t)j * ld];
    const double f = (s[i] > 0 ? ch.ev_m : ch.ev_p) * (s[j] > 0 ? ch.ev_p : ch.ev_m);
    ch.W4[idx] += one_m * f;
    if (i == j) { tr += one_m; sa += (s[i] > 0 ? one_m : -one_m); }
  }
  tr = block_sum(tr, red);
  sa = block_sum(sa, red);
  if (threadIdx.x == 0) {
    ch.acc[HQ_ACC_DMU] += ch.dt * tr;
    ch.acc[HQ_ACC_DALPHA] += sa;
  }
}

__global__ void __launch_bounds__(HQ_INT_THREADS, 1)
k_adj_interval(const HqChain* __restrict__ chains, int nchains, int b, int resident) {
  extern __shared__ __align__(16) double smem[];
  __shared__ HqChain ch;
  __shared__ double red[32];
  __shared__ int8_t s[HQ_MAX_N];
  const int c = blockIdx.x;
  if (c >= nchains) return;
  if (threadIdx.x == 0) ch = chains[c];
  __syncthreads();
  if (!ch.active || b >= ch.n_stab) return;
  const int N = ch.N;
  int t_lo, t_hi;
  interval_range(ch.nt, ch.pace, ch.n_stab, HQ_UP, b, t_lo, t_hi);
  double* G;
  int ld;
  double* p = smem;
  if (resident) { G = p; ld = smem_ld(N); p += (size_t)N * ld; copy_mat(G, ld, ch.G, N, N); }
  else { G = ch.G; ld = N; }
  double* stage = p;
  __syncthreads();
  const int nsl = t_hi - t_lo + 1;
  for (int step = 0; step < nsl; ++step) {
    const int t = t_lo + step;
    const int l = t % ch.nt;
    for (int i = threadIdx.x; i < N; i += blockDim.x) s[i] = ch.fields[(size_t)l * N + i];
    __syncthreads();
    wrap_slice(ch, G, ld, s, HQ_UP, stage);
    if (step < nsl - 1) adj_accum(ch, G, ld, s, red);
    __syncthreads();
  }
  if (resident) copy_mat(ch.G, N, G, ld, N);
}

// the last slice of interval b, after the boundary rebuilt G
__global__ void __launch_bounds__(HQ_THREADS) k_adj_last(const HqChain* __restrict__ chains, int nchains, int b) {
  __shared__ HqChain ch;
  __shared__ double red[32];
  __shared__ int8_t s[HQ_MAX_N];
  const int c = blockIdx.x;
  if (c >= nchains) return;
  if (threadIdx.x == 0) ch = chains[c];
  __syncthreads();
  if (!ch.active || b >= ch.n_stab) return;
  const int N = ch.N;
  int t_lo, t_hi;
  interval_range(ch.nt, ch.pace, ch.n_stab, HQ_UP, b, t_lo, t_hi);
  const int l = t_hi % ch.nt;
  for (int i = threadIdx.x; i < N; i += blockDim.x) s[i] = ch.fields[(size_t)l * N + i];
  __syncthreads();
  adj_accum(ch, ch.G, N, s, red);
}

}  // namespace hq

// =====================================================================================
//  launch wrappers (host)
// =====================================================================================
namespace hq {

size_t smem_interval_bytes(int Nmax, int kmax, bool resident) {
  return interval_smem_doubles(Nmax, kmax, resident) * sizeof(double);
}
size_t smem_udt_bytes(int Nmax, bool resident) {
  return smem_matrix_bytes(Nmax, resident, 2 * kQB * panel_ld(Nmax) + 2 * kQB * kQB + 3 * Nmax + 64);
}
size_t smem_invert_bytes(int Nmax, bool resident) {
  return smem_matrix_bytes(Nmax, resident, 2 * kGJ * panel_ld(Nmax) + Nmax + 64);
}
size_t smem_matrix_bytes(int Nmax, bool resident, int extra_doubles) {
  const size_t mat = resident ? (size_t)Nmax * smem_ld(Nmax) : 0;
  return (mat + (size_t)extra_doubles) * sizeof(double);
}

// The dynamic shared-memory limit of a kernel is a per-device property of the function
// shared by every context of the process: it is only ever raised, so that preparing a
// context of small chains never lowers the limit an existing context of larger chains
// launches with.
constexpr int kMaxTrackedDevices = 64;
constexpr int kTrackedKernels = 6;
static size_t g_smem_set[kMaxTrackedDevices][kTrackedKernels];

static cudaError_t raise_smem(int slot, const void* fn, size_t bytes) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 0 && dev < kMaxTrackedDevices && g_smem_set[dev][slot] >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess && dev >= 0 && dev < kMaxTrackedDevices) g_smem_set[dev][slot] = bytes;
  return e;
}

// sets the dynamic shared-memory limits of every per-chain kernel (outside any stream
// capture) so that chains of up to Nmax sites can be launched
cudaError_t prepare_kernels(int Nmax, int kmax, bool resident) {
  const size_t mat_stage = smem_matrix_bytes(Nmax, resident, 8 * (((Nmax + 15) & ~15) + 4) + 64);
  cudaError_t e;
  if ((e = raise_smem(0, (const void*)k_interval, smem_interval_bytes(Nmax, kmax, resident))) != cudaSuccess) return e;
  if ((e = raise_smem(1, (const void*)k_bchain, mat_stage)) != cudaSuccess) return e;
  if ((e = raise_smem(2, (const void*)k_udt, smem_udt_bytes(Nmax, resident))) != cudaSuccess) return e;
  if ((e = raise_smem(3, (const void*)k_invert, smem_invert_bytes(Nmax, resident))) != cudaSuccess) return e;
  if ((e = raise_smem(4, (const void*)k_dyn_slices, mat_stage)) != cudaSuccess) return e;
  if ((e = raise_smem(5, (const void*)k_adj_interval, mat_stage)) != cudaSuccess) return e;
  return cudaSuccess;
}

cudaError_t launch_interval(const HqChain* chains, int n, int dir, int b, int flags, int Nmax, int kmax, bool resident,
                            cudaStream_t st) {
  const size_t bytes = smem_interval_bytes(Nmax, kmax, resident);
  k_interval<<<n, HQ_INT_THREADS, bytes, st>>>(chains, n, dir, b, flags, resident ? 1 : 0);
  return cudaGetLastError();
}
cudaError_t launch_bchain(const HqChain* chains, int n, int dir, int b, int Nmax, bool resident, cudaStream_t st) {
  const size_t bytes = smem_matrix_bytes(Nmax, resident, 8 * (((Nmax + 15) & ~15) + 4) + 64);
  k_bchain<<<n, HQ_INT_THREADS, bytes, st>>>(chains, n, dir, b, resident ? 1 : 0);
  return cudaGetLastError();
}
cudaError_t launch_udt(const HqChain* chains, int n, int side, int b, int Nmax, bool resident, cudaStream_t st) {
  const size_t bytes = smem_udt_bytes(Nmax, resident);
  k_udt<<<n, HQ_THREADS, bytes, st>>>(chains, n, side, 0, b, resident ? 1 : 0);
  return cudaGetLastError();
}
cudaError_t launch_invert(const HqChain* chains, int n, int b, int which, int Nmax, bool resident, cudaStream_t st) {
  const size_t bytes = smem_invert_bytes(Nmax, resident);
  k_invert<<<n, HQ_THREADS, bytes, st>>>(chains, n, b, which, resident ? 1 : 0);
  return cudaGetLastError();
}
cudaError_t launch_gemm(const HqGemmJob* jobs, int njobs, int Mmax, int Nmax, cudaStream_t st) {
  if (njobs <= 0) return cudaSuccess;
  const int tm = (Mmax + GBM - 1) / GBM, tn = (Nmax + GBN - 1) / GBN;
  dim3 grid(tm * tn, njobs);
  k_gemm<<<grid, 128, 0, st>>>(jobs, njobs, tn);
  return cudaGetLastError();
}
cudaError_t launch_measure(const HqChain* chains, int n, int dir, int b, int flags, cudaStream_t st) {
  k_measure<<<n, HQ_THREADS, 0, st>>>(chains, n, dir, b, flags);
  return cudaGetLastError();
}
cudaError_t launch_dyn_start(const HqChain* chains, int n, cudaStream_t st) {
  k_dyn_start<<<n, 256, 0, st>>>(chains, n);
  return cudaGetLastError();
}
cudaError_t launch_dyn_slices(const HqChain* chains, int n, int b, int flags, int Nmax, bool resident, cudaStream_t st) {
  const size_t bytes = smem_matrix_bytes(Nmax, resident, 8 * (((Nmax + 15) & ~15) + 4) + 64);
  dim3 grid(n, 3);
  k_dyn_slices<<<grid, HQ_INT_THREADS, bytes, st>>>(chains, n, b, flags, resident ? 1 : 0);
  return cudaGetLastError();
}
cudaError_t launch_dyn_measure(const HqChain* chains, int n, int b, int last_only, cudaStream_t st) {
  k_dyn_measure<<<n, HQ_THREADS, 0, st>>>(chains, n, b, last_only);
  return cudaGetLastError();
}
cudaError_t launch_dyn_store(const HqChain* chains, int n, int b, cudaStream_t st) {
  k_dyn_store<<<n, 256, 0, st>>>(chains, n, b);
  return cudaGetLastError();
}
cudaError_t launch_adj_interval(const HqChain* chains, int n, int b, int Nmax, bool resident, cudaStream_t st) {
  const size_t bytes = smem_matrix_bytes(Nmax, resident, 8 * (((Nmax + 15) & ~15) + 4) + 64);
  k_adj_interval<<<n, HQ_INT_THREADS, bytes, st>>>(chains, n, b, resident ? 1 : 0);
  return cudaGetLastError();
}
cudaError_t launch_adj_last(const HqChain* chains, int n, int b, cudaStream_t st) {
  k_adj_last<<<n, HQ_THREADS, 0, st>>>(chains, n, b);
  return cudaGetLastError();
}
cudaError_t launch_dyn_commit(const HqChain* chains, int n, int b, cudaStream_t st) {
  k_dyn_commit<<<n, HQ_THREADS, 0, st>>>(chains, n, b);
  return cudaGetLastError();
}

}  // namespace hq
