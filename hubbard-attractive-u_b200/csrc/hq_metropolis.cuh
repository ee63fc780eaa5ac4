// hq_metropolis.cuh -- building blocks of the submatrix Metropolis update shared by the
// interval kernels (one CTA per chain, and the thread-block-cluster variant for chains whose G
// spans several SMs): the acceptance test, the warp walks of a site block, the panel
// recurrences and the DMMA flush.
#pragma once
#include "hq_common.cuh"

namespace hq {

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

// The acceptance ratio exactly as the reference evaluates it (src/hubbard.cpp:123-130):
// r = (1 + (1 - G_ii) Delta)^2 / (1 + Delta), each operation rounded on its own (no FMA
// contraction), the square as one product.
__device__ __forceinline__ double reference_ratio(double gii, double dl) {
  const double a = __dadd_rn(1.0, __dmul_rn(__dadd_rn(1.0, -gii), dl));
  return __ddiv_rn(__dmul_rn(a, a), __dadd_rn(1.0, dl));
}

// The Metropolis decision of src/dqmc_core.cpp:110: accept iff u < min(1, |r|). The fast walk
// tests u (1 + Delta) < a^2 (thr = u (1 + Delta), 1 + Delta > 0), which needs no division on
// its dependency chain and equals the reference's test except when the two sides lie within
// a few rounding errors of each other. It only records whether that happened (thr and a are
// the same in every lane, so the flag is warp-uniform; it is set with probability ~1e-12 per
// proposal); the block is then walked again from its unchanged G with the reference's own
// form, u < min(1, |r|) with r as the reference evaluates it, for every decision.
template <bool EXACT>
__device__ __forceinline__ bool accept_flip(double thr, double av, double gii, double dl, const double* u, bool& near) {
  if (EXACT) return *u < fmin(1.0, fabs(reference_ratio(gii, dl)));
  const double a2 = av * av;
  near = near || fabs(thr - a2) <= 1e-12 * a2;
  return thr < a2;
}

// the walk of the block [b0, b0 + nb) by one warp (see above); writes the records and the
// accepted count into ired[slot]; returns the near-tie flag of the fast walk. LOGT false
// compiles the ratio log out (log is then ignored).
template <int NB, bool EXACT, bool LOGT = true>
__device__ __forceinline__ bool walk_block(const HqChain& ch, const double* G, int ld, const MetroShared& sh, int b0, int nb,
                           bool log, int slot) {
  log = LOGT && log;
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
  bool near = false;  // a decision came within rounding of the other side (fast walk only)
#pragma unroll
  for (int s = 0; s < NB; ++s) {
    xk[s] = 0.0;
    yk[s] = 0.0;
    if (s < nb) {
      const int ss = s / R, si = s % R;  // g[s][*] is held by group ss at register si
      // column s, row s and the diagonal entry of the current g. On the step's dependency
      // chain (g_ss -> a -> 1/a -> the rank-1 update -> the next g_ss): a as one FMA on
      // 1 + Delta, the correctly rounded reciprocal of a (formed before the decision so that
      // it overlaps the test), and one product with the column, which was scaled by Delta
      // beside the chain
      const double dg = __shfl_sync(0xffffffffu, r[si], ss * NB + s);
      double colr[R];
#pragma unroll
      for (int i = 0; i < R; ++i) colr[i] = __shfl_sync(0xffffffffu, r[i], h * NB + s);
      const double yv = __shfl_sync(0xffffffffu, r[si], ss * NB + c) - (c == s ? 1.0 : 0.0);
      const double dl = dls[s];
      const double av = fma(-dg, dl, 1.0 + dl);  // 1 + (1 - g_ss) Delta
      const double rc = __drcp_rn(av);
      const double gam = dl * rc;                // Delta / a
      if (LOGT && log && lane == s) myr = reference_ratio(dg, dl);
      // accept iff u < min(1, |r|), r = a^2 / (1 + Delta), 1 + Delta = e^{-2 alpha s} > 0
      const bool acc = accept_flip<EXACT>(thr[s], av, dg, dl, sh.u + b0 + s, near);
      const double ge = acc ? gam : 0.0;
      const double gr = acc ? rc : 0.0;
      double xs = colr[0];
#pragma unroll
      for (int i = 1; i < R; ++i) xs = (c == i) ? colr[i] : xs;
      xk[s] = ge * xs;
      yk[s] = yv;
      if (lane == s) myg = gam;
#pragma unroll
      for (int i = 0; i < R; ++i) r[i] = fma(gr * (dl * colr[i]), yv, r[i]);
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
  return near;
}

// the walk of a 16-site block with g tiled 4 rows x 2 columns per lane: lane 8 rg + cg holds
// g[4 rg + a][2 cg + b] (a < 4, b < 2). A step needs column s for the lane's four rows, row s
// for its two columns and the diagonal entry: 7 shuffles instead of the 10 of an 8 x 1 tile.
// Every entry is updated with the same expression as in walk_block, so the two walks agree
// bitwise. Records: lanes with cg < 4 write X[J_(4 rg + cg), m], lanes with rg < 2 write
// Y[m, J_(2 cg + rg)].
template <bool EXACT, bool LOGT = true>
__device__ __forceinline__ bool walk_block16(const HqChain& ch, const double* G, int ld, const MetroShared& sh, int b0,
                                             int nb, bool log, int slot) {
  constexpr int NB = 16;
  log = LOGT && log;
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
  bool near = false;  // a decision came within rounding of the other side (fast walk only)
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
      const double av = fma(-dg, dl, 1.0 + dl);  // 1 + (1 - g_ss) Delta (as in walk_block)
      const double rc = __drcp_rn(av);
      const double gam = dl * rc;                // Delta / a
      if (LOGT && log && lane == s) myr = reference_ratio(dg, dl);
      const bool acc = accept_flip<EXACT>(thr[s], av, dg, dl, sh.u + b0 + s, near);
      const double ge = acc ? gam : 0.0;
      const double gr = acc ? rc : 0.0;
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
        const double f = gr * (dl * colr[a]);
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
  return near;
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

}  // namespace hq
