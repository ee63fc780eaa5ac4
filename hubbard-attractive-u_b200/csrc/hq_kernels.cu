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

// leading dimension of the resident G of k_interval: = 2 (mod 8) doubles, so that the DMMA
// accumulator tiles of the rank updates (lane 4g+q at row g, columns 2q, 2q+1) are free of
// bank conflicts
__host__ __device__ inline int interval_ld(int N) { return N + ((2 - N % 8) + 8) % 8; }

// bytes of dynamic shared memory of k_interval for a chain of size N with delay depth kmax
// (matrix in smem when `resident`)
__host__ __device__ inline size_t interval_smem_doubles(int N, int kmax, bool resident) {
  const size_t mat = resident ? (size_t)N * interval_ld(N) : 0;
  const size_t panels = (size_t)panel_ld(N) * kmax * 2;
  const size_t stage = (size_t)8 * (((N + 15) & ~15) + 4);
  const size_t work = panels > stage ? panels : stage;
  return mat + work + 3 * (size_t)N + (size_t)(N + 7) / 4 + (size_t)(N + 1) / 2 + 64;
}

struct SliceView {
  const int8_t* s;  // fields of the slice (shared memory)
};

// ---------------------------------------------------------------------------------
//  Equal-time estimators of one slice (include/observable_methods.hpp:39-74, 131-151)
//  filling = 2 - 2 trG/N ; docc = sum_i (1-G_ii)^2 / N ;
//  swave   = sum_ij [(1-G)_ji^2 + G_ij^2] / N = (2 sum G^2 - 2 trG + N) / N
// ---------------------------------------------------------------------------------
__device__ __forceinline__ void measure_slice(const double* G, int ld, int N, double* acc, double* red) {
  double tr = 0.0, dd = 0.0, sq = 0.0;
  HQ_FOR_EACH_ELEM(N, i, j) {
    const double v = G[i + (size_t)j * ld];
    sq = fma(v, v, sq);
    if (i == j) { tr += v; dd += (1.0 - v) * (1.0 - v); }
  }
  measure_commit(tr, dd, sq, N, acc, red);
}

__device__ __forceinline__ void copy_mat(double* dst, int ldd, const double* src, int lds, int N) {
  HQ_FOR_EACH_ELEM(N, i, j) dst[i + (size_t)j * ldd] = src[i + (size_t)j * lds];
}

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

// global -> shared copy of an N x N column-major matrix (shared ld `ldd`): every element is
// an asynchronous copy, all issued before one wait, so that the copy costs about one memory
// latency rather than one per loop trip. On return this thread's copies have landed; the
// caller's barrier makes all of them visible.
__device__ __forceinline__ void load_mat_async(double* dst, int ldd, const double* src, int lds, int N) {
  HQ_FOR_EACH_ELEM(N, i, j) cp_async_8(dst + i + (size_t)j * ldd, src + i + (size_t)j * lds, true);
  cp_async_commit();
  cp_async_wait<0>();
}

// ---------------------------------------------------------------------------------
//  Metropolis sweep over the N sites of one slice: submatrix (block-delayed) updates.
//
//  The reference visits i = 0..N-1 in order, draws one uniform per site, and on
//  acceptance applies G -= gamma G[:,i] (e_i^T - G[i,:]), gamma = Delta/(1+(1-G_ii)Delta)
//  (src/hubbard.cpp:123-139). Here the sites are taken in blocks J of NB consecutive
//  sites (E. Gull, P. Staar, S. Fuchs et al., Submatrix updates for the continuous-time
//  auxiliary-field algorithm, Phys. Rev. B 83, 075122 (2011), applied to the Ising HS
//  field):
//   1. the walk: one warp holds g = G[J, J] in registers and visits the NB sites in order
//      with the reference's acceptance test and rank-1 updates of g alone (every later
//      decision of the block reads only g's diagonal). For the a accepted flips
//      j_0 < j_1 < ... it records gamma_m, X[J, m] = gamma_m g[:, j_m] and
//      Y[m, J] = g[j_m, :] - e_{j_m}^T (g before flip m);
//   2. the a flips become the panels of G_new = G + X Y,
//        X[:, m] = gamma_m (G[:, j_m] + sum_{m'<m} X[:, m'] Y[m', j_m])
//        Y[m, :] = G[j_m, :] - e_{j_m}^T + sum_{m'<m} X[j_m, m'] Y[m', :]
//      one row of X and one column of Y per thread, with the coefficients X[J, :] and
//      Y[:, J] from the walk's records;
//   3. G += X Y by DMMA (rank a <= NB) over all warps.
//  The result equals the reference's sequence of rank-1 updates up to rounding.
// ---------------------------------------------------------------------------------
// G[0:M, 0:Nc] += X[0:M, 0:k] Y[0:k, 0:Nc]  (X column-major ldx, Y row-major ldy, k <= 16),
// by 16 x 32 strips of four 16 x 8 DMMA tiles that share the A fragments; the fragments of
// all k-steps are loaded before the strip's G tiles so that their latencies overlap
__device__ void rank_update(double* G, int ld, int M, int Nc, const double* X, int ldx, const double* Y, int ldy,
                            int k) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int mt = (M + 15) / 16, ns = (Nc + 31) / 32;
  const int strips = mt * ns;
  const int ksteps = (k + 3) >> 2;  // <= 4
  for (int st = warp; st < strips; st += nw) {
    const int r0 = (st % mt) * 16, c0 = (st / mt) * 32;
    const int r = r0 + g;
    double fa0[4], fa1[4], fb[4][4];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int m = 4 * s + q;
      const bool mk = s < ksteps && m < k;
      fa0[s] = (r < M && mk) ? X[r + m * ldx] : 0.0;
      fa1[s] = (r + 8 < M && mk) ? X[r + 8 + m * ldx] : 0.0;
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int cb = c0 + t * 8 + g;
        fb[s][t] = (cb < Nc && mk) ? Y[m * ldy + cb] : 0.0;
      }
    }
    double acc[4][4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int c = c0 + t * 8 + 2 * q;
      acc[t][0] = (r < M && c < Nc) ? G[r + (size_t)c * ld] : 0.0;
      acc[t][1] = (r < M && c + 1 < Nc) ? G[r + (size_t)(c + 1) * ld] : 0.0;
      acc[t][2] = (r + 8 < M && c < Nc) ? G[r + 8 + (size_t)c * ld] : 0.0;
      acc[t][3] = (r + 8 < M && c + 1 < Nc) ? G[r + 8 + (size_t)(c + 1) * ld] : 0.0;
    }
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      if (s < ksteps) {
#pragma unroll
        for (int t = 0; t < 4; ++t) dmma_16x8x4(acc[t], fa0[s], fa1[s], fb[s][t]);
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

struct MetroShared {
  double* dl;     // Delta of each site [N]
  double* u;      // uniforms [N]
  double* rr;     // visit-time ratio of each site [N] (ratio log)
  int8_t* s;      // fields of the slice [N]
  int8_t* flip;   // accepted flags [N]
  double* X;      // N x 16 panel (column-major, ld panel_ld(N))
  double* Y;      // 16 x N panel (row-major, ld panel_ld(N))
  double* xt;     // X[J_s, m] of the block at xt[s * NB + m] (16-byte aligned)
  double* yt;     // Y[m, J_s] of the block at yt[s * NB + m] (16-byte aligned)
  int* ired;      // >= 8 ints
  uint32_t* pw;   // a^(2i+1) mod m of each site [N]: the jump-ahead to site i's first draw
  int* qj;        // accepted site of each panel column [16]
  double* qg;     // gamma of each panel column [16]
};

// the walk of the block [b0, b0 + nb) by one warp (see above); writes the records, the
// accepted count into ired[slot] and the two triangular factors
template <int NB>
__device__ __forceinline__ void walk_block(const HqChain& ch, const double* G, int ld, const MetroShared& sh, int b0, int nb,
                           bool log, int slot, double& acc_count) {
  constexpr int R = (NB * NB >= 32) ? NB * NB / 32 : 1;  // rows of g held by one lane
  constexpr int H = NB / R;                              // lane groups (rows h*R .. h*R+R-1)
  const int lane = threadIdx.x & 31;
  // lane layout of g: lane le = h * NB + c holds g[h*R + i][c], i < R (lanes >= NB*H mirror)
  const int le = lane % (NB * H), c = le % NB, h = le / NB;
  const bool writer = lane < NB * H;
  double r[R];
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int row = h * R + i;
    r[i] = (row < nb && c < nb) ? G[b0 + row + (size_t)(b0 + c) * ld] : 0.0;
  }
  // per-site constants of the block, loaded before the walk (the walk's shared-memory
  // stores would otherwise order every later load behind them)
  double dls[NB], thr[NB];
#pragma unroll
  for (int s = 0; s < NB; ++s) {
    dls[s] = s < nb ? sh.dl[b0 + s] : 0.0;
    thr[s] = s < nb ? sh.u[b0 + s] * (1.0 + dls[s]) : 0.0;
  }
  // per-site records stay in registers during the walk (shared-memory stores would queue
  // with the shuffles on the same pipe): xk[s] = X[J_row, s] for the row this lane writes,
  // yk[s] = Y[s, J_c], the acceptance mask and, in lane s, gamma_s and the visit ratio
  double xk[NB], yk[NB], myg = 0.0, myr = 0.0;
  unsigned mask = 0u;
#pragma unroll
  for (int s = 0; s < NB; ++s) {
    xk[s] = 0.0;
    yk[s] = 0.0;
    if (s < nb) {
      const int ss = s / R, si = s % R;  // g[s][*] is held by group ss at register si
      // column s, row s and the diagonal entry of the current g; gamma is formed before
      // the decision so that its division overlaps the test
      const double dg = __shfl_sync(0xffffffffu, r[si], ss * NB + s);
      double colr[R];
#pragma unroll
      for (int i = 0; i < R; ++i) colr[i] = __shfl_sync(0xffffffffu, r[i], h * NB + s);
      const double yv = __shfl_sync(0xffffffffu, r[si], ss * NB + c) - (c == s ? 1.0 : 0.0);
      const double dl = dls[s];
      const double av = 1.0 + (1.0 - dg) * dl;
      const double gam = dl / av;
      if (log && lane == s) myr = (av * av) / (1.0 + dl);
      // accept iff u < min(1, |r|), r = a^2 / (1 + Delta), 1 + Delta = e^{-2 alpha s} > 0
      const bool acc = thr[s] < av * av;
      const double ge = acc ? gam : 0.0;
      double xs = colr[0];
#pragma unroll
      for (int i = 1; i < R; ++i) xs = (c == i) ? colr[i] : xs;
      xk[s] = ge * xs;
      yk[s] = yv;
      if (lane == s) myg = gam;
#pragma unroll
      for (int i = 0; i < R; ++i) r[i] = fma(ge * colr[i], yv, r[i]);
      mask |= acc ? (1u << s) : 0u;
    }
  }
  // the records of the accepted flips, in acceptance order
  const int a = __popc(mask);
#pragma unroll
  for (int s = 0; s < NB; ++s) {
    if (mask & (1u << s)) {
      const int m = __popc(mask & ((1u << s) - 1u));
      if (writer && c < R) sh.xt[(h * R + c) * NB + m] = xk[s];
      if (writer && h == 0) sh.yt[c * NB + m] = yk[s];
    }
  }
  if (lane < nb) {
    const bool acc = (mask >> lane) & 1u;
    if (acc) {
      const int m = __popc(mask & ((1u << lane) - 1u));
      sh.qj[m] = b0 + lane;
      sh.qg[m] = myg;
    }
    sh.flip[b0 + lane] = acc ? 1 : 0;
    if (log) sh.rr[b0 + lane] = myr;
  }
  if (lane == 0) sh.ired[slot] = a;
  acc_count += (lane == 0) ? (double)a : 0.0;
}

// the walk of a 16-site block with g tiled 4 rows x 2 columns per lane: lane 8 rg + cg holds
// g[4 rg + a][2 cg + b] (a < 4, b < 2). A step needs column s for the lane's four rows, row s
// for its two columns and the diagonal entry: 7 shuffles instead of the 10 of an 8 x 1 tile.
// Every entry is updated with the same expression as in walk_block, so the two walks agree
// bitwise. Records: lanes with cg < 4 write X[J_(4 rg + cg), m], lanes with rg < 2 write
// Y[m, J_(2 cg + rg)].
__device__ __forceinline__ void walk_block16(const HqChain& ch, const double* G, int ld, const MetroShared& sh, int b0,
                                             int nb, bool log, int slot, double& acc_count) {
  constexpr int NB = 16;
  const int lane = threadIdx.x & 31;
  const int rg = lane >> 3, cg = lane & 7;
  double r[4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const int row = 4 * rg + a, col = 2 * cg + b;
      r[a][b] = (row < nb && col < nb) ? G[b0 + row + (size_t)(b0 + col) * ld] : 0.0;
    }
  double dls[NB], thr[NB];
#pragma unroll
  for (int s = 0; s < NB; ++s) {
    dls[s] = s < nb ? sh.dl[b0 + s] : 0.0;
    thr[s] = s < nb ? sh.u[b0 + s] * (1.0 + dls[s]) : 0.0;
  }
  double xk[NB], yk[NB], myg = 0.0, myr = 0.0;
  unsigned mask = 0u;
#pragma unroll
  for (int s = 0; s < NB; ++s) {
    xk[s] = 0.0;
    yk[s] = 0.0;
    if (s < nb) {
      // g[s][s]; column s at the lane's rows (held by lane 8 rg + s/2, column slot s&1);
      // row s at the lane's columns (held by lane 8 (s/4) + cg, row slot s&3)
      const double dg = __shfl_sync(0xffffffffu, r[s & 3][s & 1], 8 * (s >> 2) + (s >> 1));
      double colr[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) colr[a] = __shfl_sync(0xffffffffu, r[a][s & 1], 8 * rg + (s >> 1));
      double rowv[2];
#pragma unroll
      for (int b = 0; b < 2; ++b)
        rowv[b] = __shfl_sync(0xffffffffu, r[s & 3][b], 8 * (s >> 2) + cg) - (2 * cg + b == s ? 1.0 : 0.0);
      const double dl = dls[s];
      const double av = 1.0 + (1.0 - dg) * dl;
      const double gam = dl / av;
      if (log && lane == s) myr = (av * av) / (1.0 + dl);
      const bool acc = thr[s] < av * av;
      const double ge = acc ? gam : 0.0;
      // the record row of this lane is 4 rg + cg (cg < 4), its record column 2 cg + rg (rg < 2)
      double xs = colr[0];
      xs = (cg == 1) ? colr[1] : xs;
      xs = (cg == 2) ? colr[2] : xs;
      xs = (cg == 3) ? colr[3] : xs;
      xk[s] = ge * xs;
      yk[s] = (rg & 1) ? rowv[1] : rowv[0];
      if (lane == s) myg = gam;
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const double f = ge * colr[a];
#pragma unroll
        for (int b = 0; b < 2; ++b) r[a][b] = fma(f, rowv[b], r[a][b]);
      }
      mask |= acc ? (1u << s) : 0u;
    }
  }
  const int a = __popc(mask);
#pragma unroll
  for (int s = 0; s < NB; ++s) {
    if (mask & (1u << s)) {
      const int m = __popc(mask & ((1u << s) - 1u));
      if (cg < 4) sh.xt[(4 * rg + cg) * NB + m] = xk[s];
      if (rg < 2) sh.yt[(2 * cg + rg) * NB + m] = yk[s];
    }
  }
  if (lane < nb) {
    const bool acc = (mask >> lane) & 1u;
    if (acc) {
      const int m = __popc(mask & ((1u << lane) - 1u));
      sh.qj[m] = b0 + lane;
      sh.qg[m] = myg;
    }
    sh.flip[b0 + lane] = acc ? 1 : 0;
    if (log) sh.rr[b0 + lane] = myr;
  }
  if (lane == 0) sh.ired[slot] = a;
  acc_count += (lane == 0) ? (double)a : 0.0;
}

// panels of the a flips of block [b0, b0 + NB): the two triangular recurrences, one row of X
// and one column of Y per thread; the coefficients of flip m are contiguous in the records
// (xt / yt at row j_m - b0) and are read in 16-byte pairs
template <int NB>
__device__ __forceinline__ void build_panels(const double* G, int ld, int N, const MetroShared& sh, int ldp, int a, int b0) {
  for (int p = threadIdx.x; p < N; p += blockDim.x) {
    double x[NB], y[NB];
#pragma unroll
    for (int m = 0; m < NB; ++m) {
      x[m] = 0.0;
      y[m] = 0.0;
      if (m < a) {
        const int jm = sh.qj[m], sj = jm - b0;
        const double* cy = sh.yt + sj * NB;  // Y[m2, j_m]
        const double* cx = sh.xt + sj * NB;  // X[j_m, m2]
        double cx0 = G[p + (size_t)jm * ld], cx1 = 0.0;
        double cy0 = G[jm + (size_t)p * ld] - (p == jm ? 1.0 : 0.0), cy1 = 0.0;
#pragma unroll
        for (int m2 = 0; m2 + 1 < m; m2 += 2) {
          const double2 vy = *reinterpret_cast<const double2*>(cy + m2);
          const double2 vx = *reinterpret_cast<const double2*>(cx + m2);
          cx0 = fma(x[m2], vy.x, cx0);
          cx1 = fma(x[m2 + 1], vy.y, cx1);
          cy0 = fma(vx.x, y[m2], cy0);
          cy1 = fma(vx.y, y[m2 + 1], cy1);
        }
        if (m & 1) {
          cx0 = fma(x[m - 1], cy[m - 1], cx0);
          cy0 = fma(cx[m - 1], y[m - 1], cy0);
        }
        x[m] = sh.qg[m] * (cx0 + cx1);
        y[m] = cy0 + cy1;
      }
    }
    // stores after the recurrence: the loads above are free to run ahead of them
#pragma unroll
    for (int m = 0; m < NB; ++m) {
      if (m < a) {
        sh.X[p + m * ldp] = x[m];
        sh.Y[m * ldp + p] = y[m];
      }
    }
  }
}

// G[0:M, 0:Nc] += X[:, 0:k] Y[0:k, :] (k <= 16): 48 x 32 warp tiles (3 x 4 DMMA tiles sharing
// their fragments; 144 = 3 x 48), all warps
__device__ __forceinline__ void rank_update48(double* G, int ld, int M, int Nc, const double* X, int ldx, const double* Y, int ldy,
                              int k) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int mt = (M + 47) / 48, ns = (Nc + 31) / 32;
  const int ksteps = (k + 3) >> 2;
  for (int st = warp; st < mt * ns; st += nw) {
    const int r0 = (st % mt) * 48, c0 = (st / mt) * 32;
    double acc[3][4][4];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int r = r0 + 16 * i + g, c = c0 + t * 8 + 2 * q;
        acc[i][t][0] = (r < M && c < Nc) ? G[r + (size_t)c * ld] : 0.0;
        acc[i][t][1] = (r < M && c + 1 < Nc) ? G[r + (size_t)(c + 1) * ld] : 0.0;
        acc[i][t][2] = (r + 8 < M && c < Nc) ? G[r + 8 + (size_t)c * ld] : 0.0;
        acc[i][t][3] = (r + 8 < M && c + 1 < Nc) ? G[r + 8 + (size_t)(c + 1) * ld] : 0.0;
      }
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      if (s < ksteps) {
        const int m = 4 * s + q;
        const bool mk = m < k;
        double fa[3][2], fb[4];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const int r = r0 + 16 * i + g;
          fa[i][0] = (r < M && mk) ? X[r + m * ldx] : 0.0;
          fa[i][1] = (r + 8 < M && mk) ? X[r + 8 + m * ldx] : 0.0;
        }
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          const int cb = c0 + t * 8 + g;
          fb[t] = (cb < Nc && mk) ? Y[m * ldy + cb] : 0.0;
        }
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int t = 0; t < 4; ++t) dmma_16x8x4(acc[i][t], fa[i][0], fa[i][1], fb[t]);
      }
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int r = r0 + 16 * i + g, c = c0 + t * 8 + 2 * q;
        if (r < M && c < Nc) G[r + (size_t)c * ld] = acc[i][t][0];
        if (r < M && c + 1 < Nc) G[r + (size_t)(c + 1) * ld] = acc[i][t][1];
        if (r + 8 < M && c < Nc) G[r + 8 + (size_t)c * ld] = acc[i][t][2];
        if (r + 8 < M && c + 1 < Nc) G[r + 8 + (size_t)(c + 1) * ld] = acc[i][t][3];
      }
  }
}

// the flush of one block's flips, G[0:N, 0:N] += X[:, 0:k] Y[0:k, :]
__device__ __forceinline__ void flush_block(double* G, int ld, int N, const double* X, int ldx, const double* Y, int ldy, int k) {
  rank_update48(G, ld, N, N, X, ldx, Y, ldy, k);
}

template <int NB>
__device__ __forceinline__ void metropolis_slice_blk(const HqChain& ch, double* G, int ld, const MetroShared& sh, uint32_t& rng,
                                     double& n_acc, int flags, long long log_base) {
  const int N = ch.N;
  const int ldp = panel_ld(N);
  const int tid = threadIdx.x, warp = tid >> 5;
  const bool log = (flags & HQ_F_LOG_RATIOS) && ch.ratios;
  // uniforms of this slice: site i consumes engine draws 2i+1, 2i+2 after the current state
  for (int i = tid; i < N; i += blockDim.x) {
    const uint32_t x1 = minstd_mulmod(sh.pw[i], rng);
    const uint32_t x2 = minstd_mulmod(kMinstdA, x1);
    sh.u[i] = canonical_from_pair(x1, x2);
    sh.dl[i] = sh.s[i] > 0 ? ch.delta_p : ch.delta_m;
    sh.flip[i] = 0;
  }
  rng = minstd_mulmod(minstd_pow(2ull * N), rng);
  __syncthreads();
  double acc_count = 0.0;
  for (int b0 = 0, bi = 0; b0 < N; b0 += NB, ++bi) {
    if (warp == 0) {
      if constexpr (NB == 16) walk_block16(ch, G, ld, sh, b0, min(NB, N - b0), log, bi & 1, acc_count);
      else walk_block<NB>(ch, G, ld, sh, b0, min(NB, N - b0), log, bi & 1, acc_count);
    }
    __syncthreads();
    // the count alternates between two words: with no flush (a == 0) no barrier follows,
    // and warp 0 writes the next block's count while other warps may still read this one
    const int a = sh.ired[bi & 1];
    if (a == 0) continue;
    build_panels<NB>(G, ld, N, sh, ldp, a, b0);
    __syncthreads();
    flush_block(G, ld, N, sh.X, ldp, sh.Y, ldp, a);
    __syncthreads();
  }
  __syncthreads();
  n_acc += acc_count;
  // apply the flips of this slice and optionally log the visit-time ratios
  for (int i = tid; i < N; i += blockDim.x) {
    if (sh.flip[i]) sh.s[i] = -sh.s[i];
    if (log && log_base + i < ch.ratio_cap) ch.ratios[log_base + i] = sh.rr[i];
  }
  __syncthreads();
}

// block size NB of the submatrix updates: the chain's delay depth (4, 8 or 16)
__device__ __forceinline__ void metropolis_dispatch(const HqChain& ch, double* G, int ld, const MetroShared& sh, uint32_t& rng,
                                    double& n_acc, int flags, long long log_base) {
  if (ch.kmax >= 16) metropolis_slice_blk<16>(ch, G, ld, sh, rng, n_acc, flags, log_base);
  else if (ch.kmax >= 8) metropolis_slice_blk<8>(ch, G, ld, sh, rng, n_acc, flags, log_base);
  else metropolis_slice_blk<4>(ch, G, ld, sh, rng, n_acc, flags, log_base);
}

// ---------------------------------------------------------------------------------
//  wrap of G by B(l) (src/dqmc_core.cpp:142-161, src/hubbard.cpp:293-331)
//   up  : G <- e^{V_l} E G E^{-1} e^{-V_l}
//   down: G <- E^{-1} e^{-V_l} G e^{V_l} E
// ---------------------------------------------------------------------------------
// With acc_meas (separable mode only) the equal-time estimators ride on the wrap: up, on the
// first pass's loads (the G before this wrap); down, on the last pass's stores (the G after it).
__device__ __forceinline__ void wrap_slice(const HqChain& ch, double* G, int ld, const int8_t* s, int dir, double* stage,
                                           double* acc_meas = nullptr, double* red = nullptr) {
  const int N = ch.N;
  if (ch.expk_mode == HQK_EXPK_SEPARABLE) {
    // the e^{+-V} scalings ride on the last pass (up) or on the first pass (down)
    if (dir == HQ_UP) {
      if (acc_meas)
        sep_apply_any<0, 0, 1, 0>(G, ld, N, ch.L, ch.sep_a, ch.sep_c, 0, nullptr, 1.0, 1.0, 1.0, 1.0, acc_meas, red);
      else
        sep_apply_any(G, ld, N, ch.L, ch.sep_a, ch.sep_c, 0);
      sep_apply_any<0, 2>(G, ld, N, ch.L, ch.sep_ai, ch.sep_ci, 1, s, ch.ev_p, ch.ev_m, ch.ev_m, ch.ev_p);
    } else {
      sep_apply_any<1, 0>(G, ld, N, ch.L, ch.sep_ai, ch.sep_ci, 0, s, ch.ev_m, ch.ev_p, ch.ev_p, ch.ev_m);
      if (acc_meas)
        sep_apply_any<0, 0, 0, 2>(G, ld, N, ch.L, ch.sep_a, ch.sep_c, 1, nullptr, 1.0, 1.0, 1.0, 1.0, acc_meas, red);
      else
        sep_apply_any(G, ld, N, ch.L, ch.sep_a, ch.sep_c, 1);
    }
    return;
  }
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
    ld = interval_ld(N);
    p += (size_t)N * ld;
    load_mat_async(G, ld, ch.G, N, N);
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
  sh.dl = p; p += N;
  sh.u = p; p += N;
  sh.rr = p; p += N;
  sh.s = reinterpret_cast<int8_t*>(p);
  sh.flip = sh.s + N;
  sh.pw = reinterpret_cast<uint32_t*>(p + (N + 7) / 4);
  for (int i = threadIdx.x; i < N; i += blockDim.x) sh.pw[i] = minstd_pow(2ull * i + 1);
  sh.ired = ired;
  __shared__ int qj_s[16];
  __shared__ double qg_s[16];
  __shared__ __align__(16) double xt_s[16 * 16];
  __shared__ __align__(16) double yt_s[16 * 16];
  sh.qj = qj_s;
  sh.qg = qg_s;
  sh.xt = xt_s;
  sh.yt = yt_s;
  uint32_t rng = *ch.rng;
  double n_acc = 0.0, n_prop = 0.0;
  long long log_base = (flags & HQ_F_LOG_RATIOS) && ch.ratio_count ? *ch.ratio_count : 0;
  __syncthreads();

  const int nsl = t_hi - t_lo + 1;
  // up / down sweeps in separable mode measure inside the wrap (up: slice t's G in the wrap of
  // slice t+1; down: in the wrap of slice t itself); the last slice of the interval is
  // measured after stabilisation
  const bool fused = (flags & HQ_F_MEASURE) && ch.expk_mode == HQK_EXPK_SEPARABLE &&
                     (dir == HQ_UP || dir == HQ_DOWN);
  for (int step = 0; step < nsl; ++step) {
    const int t = (dir == HQ_DOWN) ? (t_hi - step) : (t_lo + step);
    const int l = t % ch.nt;
    for (int i = threadIdx.x; i < N; i += blockDim.x) sh.s[i] = ch.fields[(size_t)l * N + i];
    __syncthreads();
    if (dir == HQ_UP) {
      wrap_slice(ch, G, ld, sh.s, HQ_UP, work, (fused && step > 0) ? ch.acc : nullptr, red);
      metropolis_dispatch(ch, G, ld, sh, rng, n_acc, flags, log_base);
      n_prop += N;
      log_base += N;
    } else if (dir == HQ_DOWN) {
      metropolis_dispatch(ch, G, ld, sh, rng, n_acc, flags, log_base);
      n_prop += N;
      log_base += N;
      wrap_slice(ch, G, ld, sh.s, HQ_DOWN, work, (fused && step < nsl - 1) ? ch.acc : nullptr, red);
    } else {
      wrap_slice(ch, G, ld, sh.s, HQ_UP, work);
    }
    for (int i = threadIdx.x; i < N; i += blockDim.x) ch.fields[(size_t)l * N + i] = sh.s[i];
    if (step < nsl - 1) {
      const int lm = (dir == HQ_DOWN) ? ((t - 1) % ch.nt) : l;
      if ((flags & HQ_F_MEASURE) && !fused) measure_slice(G, ld, N, ch.acc, red);
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
  if (U && resident) {
    // U and D land in shared memory by asynchronous copies (D in the stage area), then
    // the columns are scaled in place
    for (int j = threadIdx.x; j < N; j += blockDim.x) cp_async_8(stage + j, D + j, true);
    load_mat_async(X, ld, U, N, N);
    __syncthreads();
    HQ_FOR_EACH_ELEM(N, i, j) X[i + (size_t)j * ld] *= stage[j];
  } else if (U) {
    HQ_FOR_EACH_ELEM(N, i, j) X[i + (size_t)j * ld] = U[i + (size_t)j * N] * D[j];
  } else {
    HQ_FOR_EACH_ELEM(N, i, j) X[i + (size_t)j * ld] = (i == j ? 1.0 : 0.0);
  }
  __syncthreads();
  const int nsl = t_hi - t_lo + 1;
  for (int step = 0; step < nsl; ++step) {
    const int t = (dir == HQ_DOWN) ? (t_hi - step) : (t_lo + step);
    const int l = t % ch.nt;
    for (int i = threadIdx.x; i < N; i += blockDim.x) s[i] = ch.fields[(size_t)l * N + i];
    __syncthreads();
    if (ch.expk_mode == HQK_EXPK_SEPARABLE) {
      // e^{V} rides on the first pass (down: before expK) or the last pass (up: after it)
      if (dir == HQ_DOWN) sep_apply_any<1, 0>(X, ld, N, ch.L, ch.sep_a, ch.sep_c, 0, s, ch.ev_p, ch.ev_m, 1.0, 1.0);
      else sep_apply_any<0, 2>(X, ld, N, ch.L, ch.sep_a, ch.sep_c, 0, s, ch.ev_p, ch.ev_m, 1.0, 1.0);
    } else if (dir == HQ_DOWN) {
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

// reflector of column c (dlarfg convention) by the warp that holds the column in registers
// (x[t] = A[lane + 32 t, c]); writes the column (R entries, beta, v) and tau[c]
template <int RPL>
__device__ __forceinline__ void reflector_reg(double* A, int ld, int N, int c, double (&x)[RPL], double* tau) {
  const int lane = threadIdx.x & 31;
  double xs = 0.0, alpha = 0.0;
#pragma unroll
  for (int t = 0; t < RPL; ++t) {
    const int r = lane + 32 * t;
    if (r > c && r < N) xs = fma(x[t], x[t], xs);
    if (r == c) alpha = x[t];
  }
  xs = warp_sum(xs);
  alpha = __shfl_sync(0xffffffffu, alpha, c & 31);
  double ti = 0.0, beta = alpha;
  if (xs > 0.0) {
    // xs is an unscaled sum of squares already, so the norm needs no hypot
    beta = -copysign(sqrt(fma(alpha, alpha, xs)), alpha);
    ti = (beta - alpha) / beta;
    const double sc = 1.0 / (alpha - beta);
#pragma unroll
    for (int t = 0; t < RPL; ++t) {
      const int r = lane + 32 * t;
      if (r > c && r < N) x[t] *= sc;
    }
  }
#pragma unroll
  for (int t = 0; t < RPL; ++t) {
    const int r = lane + 32 * t;
    if (r == c) x[t] = beta;
    if (r < N) A[r + (size_t)c * ld] = x[t];
  }
  if (lane == 0) tau[c] = ti;
}

// Householder QR of the panel columns [p0, p1) for N <= 32 RPL: warp j holds column p0 + j in
// registers; the owner of column c+1 forms reflector c+1 right after applying reflector c,
// so one block barrier separates consecutive reflectors
template <int RPL>
__device__ void qr_panel_reg(double* A, int ld, int N, int p0, int p1, double* tau) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int col = p0 + warp;
  const bool own = col < p1;
  double x[RPL];
#pragma unroll
  for (int t = 0; t < RPL; ++t) {
    const int r = lane + 32 * t;
    x[t] = (own && r < N) ? A[r + (size_t)col * ld] : 0.0;
  }
  if (warp == 0) reflector_reg<RPL>(A, ld, N, p0, x, tau);
  __syncthreads();
  for (int c = p0; c + 1 < p1; ++c) {
    if (own && col > c) {
      const double ti = tau[c];
      if (ti != 0.0) {
        double v[RPL];
        double w = 0.0;
#pragma unroll
        for (int t = 0; t < RPL; ++t) {
          const int r = lane + 32 * t;
          v[t] = (r > c && r < N) ? A[r + (size_t)c * ld] : 0.0;
          w = (r == c) ? w + x[t] : fma(v[t], x[t], w);
        }
        w = warp_sum(w) * ti;
#pragma unroll
        for (int t = 0; t < RPL; ++t) {
          const int r = lane + 32 * t;
          if (r == c) x[t] -= w;
          else x[t] = fma(-w, v[t], x[t]);
        }
      }
      if (col == c + 1) reflector_reg<RPL>(A, ld, N, c + 1, x, tau);
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
  // S = V^T V on DMMA: warps 0 / 1 take output columns 0-7 / 8-15, four accumulator chains
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  if (warp < 2) {
    const int n0 = warp * 8;
    double acc[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u) acc[u][0] = acc[u][1] = acc[u][2] = acc[u][3] = 0.0;
    for (int r0 = p0; r0 < N; r0 += 16) {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int r = r0 + 4 * u + q;
        const bool ok = r < N;
        const double a0 = ok ? Vb[r + g * ldv] : 0.0;
        const double a1 = ok ? Vb[r + (g + 8) * ldv] : 0.0;
        const double b0 = ok ? Vb[r + (n0 + g) * ldv] : 0.0;
        dmma_16x8x4(acc[u], a0, a1, b0);
      }
    }
    const int cc = n0 + 2 * q;
    S[g * kQB + cc] = (acc[0][0] + acc[1][0]) + (acc[2][0] + acc[3][0]);
    S[g * kQB + cc + 1] = (acc[0][1] + acc[1][1]) + (acc[2][1] + acc[3][1]);
    S[(g + 8) * kQB + cc] = (acc[0][2] + acc[1][2]) + (acc[2][2] + acc[3][2]);
    S[(g + 8) * kQB + cc + 1] = (acc[0][3] + acc[1][3]) + (acc[2][3] + acc[3][3]);
  }
  __syncthreads();
  // T[i][j] = -tau_j sum_{i <= l < j} T[i][l] S[l][j] (T[i][i] = tau_i): lane i keeps row i
  if (warp == 0 && lane < kQB) {
    const int i = lane;
    double t[kQB];
#pragma unroll
    for (int j = 0; j < kQB; ++j) {
      double v = 0.0;
      if (j < m) {
        if (i == j) {
          v = tau[p0 + j];
        } else if (i < j) {
          double acc0 = 0.0, acc1 = 0.0;  // t[l] = 0 for l < i; two chains
#pragma unroll
          for (int l = 0; l < j; l += 2) {
            acc0 = fma(t[l], S[l * kQB + j], acc0);
            if (l + 1 < j) acc1 = fma(t[l + 1], S[(l + 1) * kQB + j], acc1);
          }
          v = -tau[p0 + j] * (acc0 + acc1);
        }
      }
      t[j] = v;
    }
#pragma unroll
    for (int j = 0; j < kQB; ++j) T[i * kQB + j] = t[j];
  }
  __syncthreads();
}

// A[p0:, col0:col0+nc] <- (I - V op(T) V^T) A[p0:, col0:col0+nc]; op(T) = T^T if trans
__device__ void wy_apply(double* A, int ld, int N, int p0, const double* Vb, int ldv, const double* T, bool trans,
                         double* W, int ldw, int col0, int nc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  // W = V^T A_sub (kQB x nc) with DMMA: m16 = the panel columns, k = rows p0..N-1, four
  // accumulator chains per 8-column tile
  const int nt8 = (nc + 7) / 8;
  for (int t = warp; t < nt8; t += nwarps) {
    const int cb = t * 8 + g;
    double acc[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u) acc[u][0] = acc[u][1] = acc[u][2] = acc[u][3] = 0.0;
    for (int r0 = p0; r0 < N; r0 += 16) {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int r = r0 + 4 * u + q;
        const double a0 = (r < N) ? Vb[r + g * ldv] : 0.0;
        const double a1 = (r < N) ? Vb[r + (g + 8) * ldv] : 0.0;
        const double b0 = (r < N && cb < nc) ? A[r + (size_t)(col0 + cb) * ld] : 0.0;
        dmma_16x8x4(acc[u], a0, a1, b0);
      }
    }
    const int c = t * 8 + 2 * q;
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[0][e] = (acc[0][e] + acc[1][e]) + (acc[2][e] + acc[3][e]);
    if (c < nc) { W[g * ldw + c] = acc[0][0]; W[(g + 8) * ldw + c] = acc[0][2]; }
    if (c + 1 < nc) { W[g * ldw + c + 1] = acc[0][1]; W[(g + 8) * ldw + c + 1] = acc[0][3]; }
  }
  __syncthreads();
  // W <- -op(T) W by DMMA, in place per 8-column tile (a tile's loads precede its stores)
  for (int t = warp; t < nt8; t += nwarps) {
    const int n = t * 8 + g;
    double bw[4];
#pragma unroll
    for (int s4 = 0; s4 < 4; ++s4) bw[s4] = (n < nc) ? W[(4 * s4 + q) * ldw + n] : 0.0;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int s4 = 0; s4 < 4; ++s4) {
      const int l = 4 * s4 + q;
      const double a0 = trans ? T[l * kQB + g] : T[g * kQB + l];
      const double a1 = trans ? T[l * kQB + g + 8] : T[(g + 8) * kQB + l];
      dmma_16x8x4(acc, a0, a1, bw[s4]);
    }
    const int c = t * 8 + 2 * q;
    if (c < nc) { W[g * ldw + c] = -acc[0]; W[(g + 8) * ldw + c] = -acc[2]; }
    if (c + 1 < nc) { W[g * ldw + c + 1] = -acc[1]; W[(g + 8) * ldw + c + 1] = -acc[3]; }
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
  if (resident) {
    HQ_FOR_EACH_ELEM(N, i, j) cp_async_8(A + i + (size_t)j * ld, X + i + (size_t)order[j] * N, true);
    cp_async_commit();
    cp_async_wait<0>();
  } else {
    HQ_FOR_EACH_ELEM(N, i, j) A[i + (size_t)j * ld] = X[i + (size_t)order[j] * N];
  }
  __syncthreads();
  // ---- blocked Householder QR ----
  for (int p0 = 0; p0 < N; p0 += kQB) {
    const int p1 = min(p0 + kQB, N);
    if (N <= 160) qr_panel_reg<5>(A, ld, N, p0, p1, tau);
    else qr_panel(A, ld, N, p0, p1, tau);
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
  // ---- form Q in place, panels backwards: the trailing columns get the panel's WY
  // transformation, the panel's own columns (identity columns until now) are in closed form
  //   Q[:, p0:p1] = E - V T V[p0:p1, :]^T ----
  for (int p0 = ((N - 1) / kQB) * kQB; p0 >= 0; p0 -= kQB) {
    const int p1 = min(p0 + kQB, N), m = p1 - p0;
    wy_factor(A, ld, N, p0, m, tau, Vb, ldp, T, S);
    if (p1 < N) wy_apply(A, ld, N, p0, Vb, ldp, T, false, W, ldp, p1, N - p1);
    for (int t = threadIdx.x; t < kQB * kQB; t += blockDim.x) {
      const int l = t / kQB, j = t % kQB;
      double acc = 0.0;
      if (j < m)
        for (int l2 = 0; l2 < kQB; ++l2) acc = fma(T[l * kQB + l2], Vb[(p0 + j) + l2 * ldp], acc);
      W[l * ldp + j] = -acc;
    }
    for (int idx = threadIdx.x; idx < N * m; idx += blockDim.x) {
      const int r = idx % N, j = idx / N;
      A[r + (size_t)(p0 + j) * ld] = (r == p0 + j) ? 1.0 : 0.0;
    }
    __syncthreads();
    rank_update(A + p0 + (size_t)p0 * ld, ld, N - p0, m, Vb + p0, ldp, W, ldp, kQB);
    __syncthreads();
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

// x[r / 32] (r warp-uniform) without an indexed access: written as a C++ select chain the
// compiler folds it back into x[r / 32], which moves x to local memory; selp keeps it in
// registers
template <int RPL>
__device__ __forceinline__ double slot_at(const double (&x)[RPL], int r) {
  const int t = r >> 5;
  double v = 0.0;
#pragma unroll
  for (int i = 0; i < RPL; ++i)
    asm("{\n\t.reg .pred p;\n\tsetp.eq.s32 p, %2, %3;\n\tselp.f64 %0, %1, %0, p;\n\t}" : "+d"(v) : "d"(x[i]), "r"(t), "r"(i));
  return v;
}

// pivot k of a register-resident Gauss-Jordan panel, by the warp that holds column k:
// partial pivoting (largest |A[r][k]|, r >= k, smallest index among equals), row swap in
// this column, the multipliers into fcol, the inverse's column k into x, and perm / pinv
template <int RPL>
__device__ __forceinline__ void gj_pivot_reg(double (&x)[RPL], int k, int N, double* fcol, double* pinv_out,
                                             int* perm, double* status) {
  const int lane = threadIdx.x & 31;
  double best = -1.0;
  int bi = N;
#pragma unroll
  for (int t = 0; t < RPL; ++t) {
    const int r = lane + 32 * t;
    if (r >= k && r < N) {
      const double v = fabs(x[t]);
      if (v > best || (v == best && r < bi)) { best = v; bi = r; }
    }
  }
  // warp argmax with three redux steps on the bit pattern of |x| (monotonic for non-negative
  // doubles; NaNs were skipped by the lane-local search): the high word, then the low word
  // among the lanes holding the maximum, then the smallest row among those
  {
    const unsigned long long bb = best < 0.0 ? 0ull : (unsigned long long)__double_as_longlong(best);
    const unsigned hi = (unsigned)(bb >> 32), lo = (unsigned)bb;
    const unsigned mh = __reduce_max_sync(0xffffffffu, hi);
    const unsigned ml = __reduce_max_sync(0xffffffffu, hi == mh ? lo : 0u);
    bi = (int)__reduce_min_sync(0xffffffffu, (hi == mh && lo == ml) ? (unsigned)bi : 0xffffffffu);
    best = __longlong_as_double((long long)(((unsigned long long)mh << 32) | ml));
  }
  const double vk = __shfl_sync(0xffffffffu, slot_at<RPL>(x, k), k & 31);
  const double vb = __shfl_sync(0xffffffffu, slot_at<RPL>(x, bi), bi & 31);
  const bool ok = (best > 0.0) && isfinite(best);
  const double pinv = ok ? 1.0 / vb : 0.0;
#pragma unroll
  for (int t = 0; t < RPL; ++t) {
    const int r = lane + 32 * t;
    double v = (r == k) ? vb : ((r == bi) ? vk : x[t]);
    if (r < N) fcol[r] = v;
    x[t] = (r == k) ? pinv : -v * pinv;
  }
  if (lane == 0) {
    perm[k] = bi;
    *pinv_out = pinv;
    if (!ok) *status = 1.0;
  }
}

// Gauss-Jordan on the panel columns [p0, p0 + nb) of A (all rows), N <= 32 RPL: warp j holds
// column p0 + j in registers; the owner of column k+1 takes pivot k+1 right after its own
// elimination step for pivot k, so one block barrier separates pivots. Multipliers and the
// reciprocal pivot are double-buffered by pivot parity (fcol: 2N doubles, pv: 2).
template <int RPL>
__device__ void gj_panel_reg(double* A, int ld, int N, int p0, int nb, int* perm, double* fcol, double* pv,
                             double* status) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool own = warp < nb;
  const int col = p0 + warp;
  double x[RPL];
#pragma unroll
  for (int t = 0; t < RPL; ++t) {
    const int r = lane + 32 * t;
    x[t] = (own && r < N) ? A[r + (size_t)col * ld] : 0.0;
  }
  if (warp == 0) gj_pivot_reg<RPL>(x, p0, N, fcol, pv, perm, status);
  __syncthreads();
  for (int q = 0; q < nb; ++q) {
    const int k = p0 + q, par = q & 1;
    if (own && warp != q) {
      const int bi = perm[k];
      const double pinv = pv[par];
      const double* f = fcol + par * N;
      // row swap k <-> bi in this column, then row k scaled by the pivot's reciprocal
      const double vk = __shfl_sync(0xffffffffu, slot_at<RPL>(x, k), k & 31);
      const double vb = __shfl_sync(0xffffffffu, slot_at<RPL>(x, bi), bi & 31);
      const double u = vb * pinv;
#pragma unroll
      for (int t = 0; t < RPL; ++t) {
        const int r = lane + 32 * t;
        const double v = (r == bi) ? vk : x[t];
        x[t] = (r == k) ? u : ((r < N) ? fma(-f[r < N ? r : 0], u, v) : v);
      }
      if (warp == q + 1 && q + 1 < nb) gj_pivot_reg<RPL>(x, k + 1, N, fcol + (par ^ 1) * N, pv + (par ^ 1), perm, status);
    }
    __syncthreads();
  }
#pragma unroll
  for (int t = 0; t < RPL; ++t) {
    const int r = lane + 32 * t;
    if (own && r < N) A[r + (size_t)col * ld] = x[t];
  }
  __syncthreads();
}

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
  if (resident) { A = p; ld = smem_ld(N); p += (size_t)N * ld; load_mat_async(A, ld, src, N, N); }
  else { A = src; ld = N; }
  const int ldp = panel_ld(N);
  double* Wp = p; p += (size_t)ldp * kGJ;   // N x kGJ, column-major
  double* Bf = p; p += (size_t)ldp * kGJ;   // kGJ x N, row-major
  int* perm = reinterpret_cast<int*>(p);
  int* gidx = perm + N;
  double* fcol = reinterpret_cast<double*>(gidx + N);  // 2 N multipliers (register panel)
  __shared__ double pv[2];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  for (int p0 = 0; p0 < N; p0 += kGJ) {
    const int nb = min(kGJ, N - p0);
    if (N <= 160) gj_panel_reg<5>(A, ld, N, p0, nb, perm, fcol, pv, ch.acc + HQ_ACC_STATUS);
    else for (int q = 0; q < nb; ++q) {
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

// scaling of index i: 1 (mode 0 or no vector), v[i] (1), 1 / max(v[i], 1) (2), min(v[i], 1) (3)
__device__ __forceinline__ double vscale(const double* v, int mode, int i) {
  if (!v || mode == 0) return 1.0;
  const double x = v[i];
  if (mode == 1) return x;
  if (mode == 2) return 1.0 / fmax(x, 1.0);
  return fmin(x, 1.0);
}


// ---------------------------------------------------------------------------------
//  k_gemm: batched C = alpha op(A) diag(ks) op(B) (row / column scalings, beta, wrap-error
//  epilogue), one CTA per 48 x 48 tile of one job (144 = 3 x 48: no padding for the 12 x 12
//  lattice). Six warps own 16 x 24 blocks (3 DMMA tiles each); K streams through shared
//  memory in chunks of 16 with cp.async double buffering. Shared layouts keep the fragment
//  loads free of bank conflicts for either transpose:
//    op(A) = A   : sA[k * kGLdm + m]     op(A) = A^T : sA[m * kGLdk + k]
//    op(B) = B   : sB[n * kGLdk + k]     op(B) = B^T : sB[k * kGLdm + n]
// ---------------------------------------------------------------------------------
constexpr int kGT = 48, kGKc = 16, kGLdm = 52, kGLdk = 20, kGWarps = 6;
constexpr int kGStage = (kGLdm * kGKc > kGT * kGLdk) ? kGLdm * kGKc : kGT * kGLdk;  // doubles

// copies 2 doubles (16 B) with zero fill of the invalid part; both addresses 16-byte aligned
__device__ __forceinline__ void cp_async_16(double* dst, const double* src, int nvalid) {
  const unsigned saddr = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  const int nbytes = nvalid <= 0 ? 0 : (nvalid >= 2 ? 16 : 8);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(saddr), "l"(src), "r"(nbytes));
}

// stages the chunk [k0, k0 + 16) x [r0, r0 + 48) of op(X) (r = m for A, n for B; R rows).
// kmaj: op(X) is contiguous along k in memory (A^T or B) -> layout [r][k]; otherwise
// contiguous along r -> layout [k][r]. `pair` selects 16-byte copies (even ld, aligned base).
__device__ __forceinline__ void g_stage(const double* X, int ldx, bool kmaj, int R, int K, int r0, int k0,
                                        double* sX, bool pair) {
  if (pair) {
    if (kmaj) {
      for (int idx = threadIdx.x; idx < kGT * (kGKc / 2); idx += blockDim.x) {
        const int r = idx / (kGKc / 2), k = 2 * (idx % (kGKc / 2));
        const int nv = (r0 + r < R) ? min(2, K - (k0 + k)) : 0;
        cp_async_16(sX + r * kGLdk + k, nv > 0 ? X + (k0 + k) + (size_t)(r0 + r) * ldx : X, nv);
      }
    } else {
      for (int idx = threadIdx.x; idx < (kGT / 2) * kGKc; idx += blockDim.x) {
        const int r = 2 * (idx % (kGT / 2)), k = idx / (kGT / 2);
        const int nv = (k0 + k < K) ? min(2, R - (r0 + r)) : 0;
        cp_async_16(sX + k * kGLdm + r, nv > 0 ? X + (r0 + r) + (size_t)(k0 + k) * ldx : X, nv);
      }
    }
  } else {
    for (int idx = threadIdx.x; idx < kGT * kGKc; idx += blockDim.x) {
      int r, k;
      if (kmaj) { r = idx / kGKc; k = idx % kGKc; } else { r = idx % kGT; k = idx / kGT; }
      const bool ok = k0 + k < K && r0 + r < R;
      const double* src = ok ? (kmaj ? X + (k0 + k) + (size_t)(r0 + r) * ldx : X + (r0 + r) + (size_t)(k0 + k) * ldx) : X;
      cp_async_8(kmaj ? sX + r * kGLdk + k : sX + k * kGLdm + r, src, ok);
    }
  }
}

__global__ void __launch_bounds__(kGWarps * 32, 4)
k_gemm(const HqGemmJob* __restrict__ jobs, int njobs, int tiles_n) {
  __shared__ __align__(16) double sA[2][kGStage];
  __shared__ __align__(16) double sB[2][kGStage];
  __shared__ double sK[2][kGKc];
  __shared__ double red[32];
  const int jb = blockIdx.y;
  if (jb >= njobs) return;
  const HqGemmJob J = jobs[jb];
  if (!J.active) return;
  const int m0 = (blockIdx.x / tiles_n) * kGT, n0 = (blockIdx.x % tiles_n) * kGT;
  if (m0 >= J.M || n0 >= J.Nc) return;
  const bool amaj = J.ta != 0;  // op(A) = A^T is contiguous along k
  const bool bmaj = J.tb == 0;  // op(B) = B is contiguous along k
  const bool pa = (J.lda % 2 == 0) && ((reinterpret_cast<uintptr_t>(J.A) & 15) == 0);
  const bool pb = (J.ldb % 2 == 0) && ((reinterpret_cast<uintptr_t>(J.B) & 15) == 0);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int wm = (warp % 3) * 16, wn = (warp / 3) * 24;
  double acc[3][4];
#pragma unroll
  for (int j = 0; j < 3; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0;
  const int nchunks = (J.K + kGKc - 1) / kGKc;
  g_stage(J.A, J.lda, amaj, J.M, J.K, m0, 0, sA[0], pa);
  g_stage(J.B, J.ldb, bmaj, J.Nc, J.K, n0, 0, sB[0], pb);
  if (threadIdx.x < kGKc) sK[0][threadIdx.x] = (threadIdx.x < J.K) ? vscale(J.ks, J.ks_mode, threadIdx.x) : 0.0;
  cp_async_commit();
  for (int c = 0; c < nchunks; ++c) {
    const int cur = c & 1;
    if (c + 1 < nchunks) {
      const int k1 = (c + 1) * kGKc;
      g_stage(J.A, J.lda, amaj, J.M, J.K, m0, k1, sA[cur ^ 1], pa);
      g_stage(J.B, J.ldb, bmaj, J.Nc, J.K, n0, k1, sB[cur ^ 1], pb);
      if (threadIdx.x < kGKc)
        sK[cur ^ 1][threadIdx.x] = (k1 + threadIdx.x < J.K) ? vscale(J.ks, J.ks_mode, k1 + threadIdx.x) : 0.0;
    }
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const double* A_ = sA[cur];
    const double* B_ = sB[cur];
#pragma unroll
    for (int kk = 0; kk < kGKc; kk += 4) {
      const int k = kk + q;
      const double ksc = sK[cur][k];
      const int m = wm + g;
      const double a0 = (amaj ? A_[m * kGLdk + k] : A_[k * kGLdm + m]) * ksc;
      const double a1 = (amaj ? A_[(m + 8) * kGLdk + k] : A_[k * kGLdm + m + 8]) * ksc;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const int n = wn + j * 8 + g;
        const double b0 = bmaj ? B_[n * kGLdk + k] : B_[k * kGLdm + n];
        dmma_16x8x4(acc[j], a0, a1, b0);
      }
    }
    __syncthreads();
  }
  cp_async_wait<0>();
  // epilogue: alpha, row / column scalings, beta, wrap-error maximum
  double emax = -INFINITY;
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int gm = m0 + wm + g + ((e & 2) ? 8 : 0);
      const int gn = n0 + wn + j * 8 + 2 * q + (e & 1);
      if (gm < J.M && gn < J.Nc) {
        double v = J.alpha * acc[j][e] * vscale(J.rs, J.rs_mode, gm) * vscale(J.cs, J.cs_mode, gn);
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
  if (resident) { M = p; ld = smem_ld(N); p += (size_t)N * ld; load_mat_async(M, ld, src, N, N); }
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
  if (resident) { G = p; ld = smem_ld(N); p += (size_t)N * ld; load_mat_async(G, ld, ch.G, N, N); }
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
  return smem_matrix_bytes(Nmax, resident, 2 * kGJ * panel_ld(Nmax) + 3 * Nmax + 64);
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
size_t max_static_smem() {
  const void* fns[] = {(const void*)k_interval, (const void*)k_bchain, (const void*)k_udt,
                       (const void*)k_invert, (const void*)k_dyn_slices, (const void*)k_adj_interval};
  size_t m = 0;
  for (const void* f : fns) {
    cudaFuncAttributes a;
    if (cudaFuncGetAttributes(&a, f) != cudaSuccess) return 16384;  // conservative
    m = a.sharedSizeBytes > m ? a.sharedSizeBytes : m;
  }
  return m;
}

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
  const int tm = (Mmax + kGT - 1) / kGT, tn = (Nmax + kGT - 1) / kGT;
  dim3 grid(tm * tn, njobs);
  k_gemm<<<grid, kGWarps * 32, 0, st>>>(jobs, njobs, tn);
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

// Copies every chain's accumulator block into one chain-major buffer, so that a single
// device-to-host copy reads the estimators of all chains.
__global__ void k_gather_acc(const HqChain* chains, int n, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * HQ_ACC_COUNT) return;
  const int c = i / HQ_ACC_COUNT;
  out[i] = chains[c].acc[i - c * HQ_ACC_COUNT];
}
cudaError_t launch_gather_acc(const HqChain* chains, int n, double* out, cudaStream_t st) {
  const int total = n * HQ_ACC_COUNT;
  k_gather_acc<<<(total + 255) / 256, 256, 0, st>>>(chains, n, out);
  return cudaGetLastError();
}

}  // namespace hq
