// hq_udt.cuh -- the UDV factorisation of a stack push (blocked Householder QR with panel-wise
// column pivoting, in place of the dgesvd of include/utils/svd_stack.hpp:107-175), used by
// k_udt (one launch per push) and by the persistent sweep kernel.
#pragma once
#include "hq_common.cuh"

namespace hq {

// ---------------------------------------------------------------------------------
//  k_udt: UDV factorisation X P = Q R of the stack push, X = Q D T with D = |diag R| and
//  T = D^-1 R P^T (the role of dgesvd in include/utils/svd_stack.hpp:107-175).
//  P first sorts the columns of X by decreasing norm ("pre-pivoting", C. Bauer, Fast and
//  stable determinant quantum Monte Carlo, SciPost Phys. Core 2, 011 (2020)); the QR is
//  blocked Householder in panels of kQB columns with compact-WY trailing updates
//  A <- (I - V T^T V^T) A, whose two products run on DMMA. Before every later panel, the
//  kQB trailing columns of largest current norm (rows p0..N-1 of the updated matrix) are
//  swapped into the panel in decreasing order: the panel-wise form of column pivoting. A
//  single sort is not enough in the middle of a large-beta sweep: when the stacks on both
//  sides are long, pre-pivoting alone left the stabilised G up to ~5e-10 x max|G| from a
//  G stabilised at every slice (12 x 12, beta = 10), the re-selection keeps it below ~4e-11,
//  as column-pivoted QR does. Q is formed in place by the same blocks backwards
//  (Q = B_0 B_1 ..., B_p = I - V_p T_p V_p^T), with the T factors kept from the
//  factorisation.
//  Output: U (= Q) and D into stack entry b of the pushing stack, T into W0.
// ---------------------------------------------------------------------------------

// unblocked Householder QR of the panel columns [p0, p1) (rows p0..N-1), dlarfg convention
static __device__ void qr_panel(double* A, int ld, int N, int p0, int p1, double* tau) {
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
    // apply H_c to the remaining panel columns, one warp per column at a time
    const double ti = tau[c];
    for (int j = c + 1 + warp; ti != 0.0 && j < p1; j += blockDim.x >> 5) {
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
  // two partial sums: the lane's part of the reflector's dependency chain is half as long
  double xs0 = 0.0, xs1 = 0.0, alpha = 0.0;
#pragma unroll
  for (int t = 0; t < RPL; ++t) {
    const int r = lane + 32 * t;
    if (r > c && r < N) {
      if (t & 1) xs1 = fma(x[t], x[t], xs1);
      else xs0 = fma(x[t], x[t], xs0);
    }
    if (r == c) alpha = x[t];
  }
  const double xs = warp_sum(xs0 + xs1);
  alpha = __shfl_sync(0xffffffffu, alpha, c & 31);
  double ti = 0.0, beta = alpha;
  if (xs > 0.0) {
    // xs is an unscaled sum of squares already, so the norm needs no hypot
    beta = -copysign(sqrt(fma(alpha, alpha, xs)), alpha);
    ti = (beta - alpha) * __drcp_rn(beta);  // (beta - alpha) / beta
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

// Householder QR of the panel columns [p0, p1) for N <= 32 RPL: the panel's kQB columns are held
// in registers, CPW per warp by kQB / CPW warps (warp w holds columns p0 + w + i kQB / CPW);
// the owner of column c+1 forms reflector c+1 right after applying reflector c, so one block
// barrier separates consecutive reflectors
template <int RPL, int CPW>
__device__ void qr_panel_reg(double* A, int ld, int N, int p0, int p1, double* tau) {
  constexpr int NWP = kQB / CPW;  // warps that hold panel columns
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int col[CPW];
  bool own[CPW];
  double x[CPW][RPL];
#pragma unroll
  for (int i = 0; i < CPW; ++i) {
    col[i] = p0 + warp + i * NWP;
    own[i] = warp < NWP && col[i] < p1;
#pragma unroll
    for (int t = 0; t < RPL; ++t) {
      const int r = lane + 32 * t;
      x[i][t] = (own[i] && r < N) ? A[r + (size_t)col[i] * ld] : 0.0;
    }
  }
  if (warp == 0) reflector_reg<RPL>(A, ld, N, p0, x[0], tau);
  __syncthreads();
  for (int c = p0; c + 1 < p1; ++c) {
#pragma unroll
    for (int i = 0; i < CPW; ++i) {
      if (own[i] && col[i] > c) {
        const double ti = tau[c];
        if (ti != 0.0) {
          double v[RPL];
          double w0 = 0.0, w1 = 0.0;  // two partial sums (a shorter chain per lane)
#pragma unroll
          for (int t = 0; t < RPL; ++t) {
            const int r = lane + 32 * t;
            v[t] = (r > c && r < N) ? A[r + (size_t)c * ld] : 0.0;
            if (t & 1) w1 = (r == c) ? w1 + x[i][t] : fma(v[t], x[i][t], w1);
            else w0 = (r == c) ? w0 + x[i][t] : fma(v[t], x[i][t], w0);
          }
          const double w = warp_sum(w0 + w1) * ti;
#pragma unroll
          for (int t = 0; t < RPL; ++t) {
            const int r = lane + 32 * t;
            if (r == c) x[i][t] -= w;
            else x[i][t] = fma(-w, v[t], x[i][t]);
          }
        }
        if (col[i] == c + 1) reflector_reg<RPL>(A, ld, N, c + 1, x[i], tau);
      }
    }
    __syncthreads();
  }
}

// V of the panel [p0, p0+m) with explicit unit diagonal and zeros above (columns >= m zero)
static __device__ void wy_vfill(const double* A, int ld, int N, int p0, int m, double* Vb, int ldv) {
  for (int q = threadIdx.x >> 5; q < kQB; q += blockDim.x >> 5)
    for (int r = p0 + (threadIdx.x & 31); r < N; r += 32) {
      const int c = p0 + q;
      Vb[r + q * ldv] = (q >= m || r < c) ? 0.0 : (r == c ? 1.0 : A[r + (size_t)c * ld]);
    }
  __syncthreads();
}

// S = V^T V (kQB x kQB) on DMMA, by warps 0 and 1 only (output columns 0-7 / 8-15), four
// accumulator chains
__device__ __forceinline__ void wy_gram(int N, int p0, const double* Vb, int ldv, double* S) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, q = lane & 3;
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

// T[i][j] = -tau_j sum_{i <= l < j} T[i][l] S[l][j], T[i][i] = tau_i (columns j >= m zero), by
// warp 0 only: lane i keeps row i. Every lane runs the same instructions (t[l] = 0 for l < i,
// entries off the upper triangle selected to zero), so the loads of S and tau issue ahead of
// the recurrence.
__device__ __forceinline__ void wy_tfactor(int p0, int m, const double* tau, const double* S, double* T) {
  const int i = threadIdx.x & 31;
  double t[kQB];
#pragma unroll
  for (int j = 0; j < kQB; ++j) {
    const double tj = (j < m) ? tau[p0 + j] : 0.0;
    double acc0 = 0.0, acc1 = 0.0;  // two chains
#pragma unroll
    for (int l = 0; l < j; l += 2) {
      acc0 = fma(t[l], S[l * kQB + j], acc0);
      if (l + 1 < j) acc1 = fma(t[l + 1], S[(l + 1) * kQB + j], acc1);
    }
    const double v = -tj * (acc0 + acc1);
    t[j] = (j >= m) ? 0.0 : (i == j ? tj : (i < j ? v : 0.0));
  }
  if (i < kQB) {
#pragma unroll
    for (int j = 0; j < kQB; ++j) T[i * kQB + j] = t[j];
  }
}

// V of the panel [p0, p0+m) (wy_vfill) and the triangular factor T of
// H_p0 ... H_p0+m-1 = I - V T V^T
static __device__ void wy_factor(const double* A, int ld, int N, int p0, int m, const double* tau, double* Vb, int ldv,
                          double* T, double* S) {
  wy_vfill(A, ld, N, p0, m, Vb, ldv);
  if ((threadIdx.x >> 5) < 2) wy_gram(N, p0, Vb, ldv, S);
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) wy_tfactor(p0, m, tau, S, T);
  __syncthreads();
}

// W = V^T A_sub (kQB x nc, A_sub = A[p0:, col0:col0+nc]) with DMMA: m16 = the panel columns,
// k = rows p0..N-1, four accumulator chains per 8-column tile; tiles over warps w0, w0 + ws, ...
__device__ __forceinline__ void wy_vta(const double* A, int ld, int N, int p0, const double* Vb, int ldv, double* W,
                                       int ldw, int col0, int nc, int w0, int ws) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int nt8 = (nc + 7) / 8;
  for (int t = warp - w0; t < nt8; t += ws) {
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
}

// W <- -op(T) W (op(T) = T^T if trans) by DMMA, in place per 8-column tile (a tile's loads
// precede its stores), then A_sub += V W; W = V^T A_sub on entry, after a block barrier
static __device__ void wy_tw_rank(double* A, int ld, int N, int p0, const double* Vb, int ldv, const double* T, bool trans,
                           double* W, int ldw, int col0, int nc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int nt8 = (nc + 7) / 8;
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
  rank_update(A + p0 + (size_t)col0 * ld, ld, N - p0, nc, Vb + p0, ldv, W, ldw, kQB);
  __syncthreads();
}

// A[p0:, col0:col0+nc] <- (I - V op(T) V^T) A[p0:, col0:col0+nc]; op(T) = T^T if trans
static __device__ void wy_apply(double* A, int ld, int N, int p0, const double* Vb, int ldv, const double* T, bool trans,
                         double* W, int ldw, int col0, int nc) {
  wy_vta(A, ld, N, p0, Vb, ldv, W, ldw, col0, nc, 0, blockDim.x >> 5);
  __syncthreads();
  wy_tw_rank(A, ld, N, p0, Vb, ldv, T, trans, W, ldw, col0, nc);
}

// The trailing update of the factorisation, A_sub <- (I - V T^T V^T) A_sub with the panel's
// T formed on the way: warps 0 and 1 form S = V^T V and warp 0 then T (two-warp named
// barrier between them), while the other warps form W = V^T A_sub, which does not need T.
static __device__ void wy_forward(double* A, int ld, int N, int p0, int m, const double* tau, double* Vb, int ldv, double* T,
                           double* S, double* W, int ldw, int col0, int nc) {
  const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  wy_vfill(A, ld, N, p0, m, Vb, ldv);
  if (warp < 2) {
    wy_gram(N, p0, Vb, ldv, S);
    asm volatile("bar.sync 1, 64;" ::: "memory");
    if (warp == 0) wy_tfactor(p0, m, tau, S, T);
  } else {
    wy_vta(A, ld, N, p0, Vb, ldv, W, ldw, col0, nc, 2, nwarps - 2);
  }
  __syncthreads();
  wy_tw_rank(A, ld, N, p0, Vb, ldv, T, true, W, ldw, col0, nc);
}

// rk[j] = the rank of column j among the columns [lo, N) in decreasing nrm, ties by position,
// and who[r] = the column of rank r for r < m. Four threads per column, each counting over one
// residue of positions mod 4. The norms are compared as the integer patterns of their bits,
// which order non-negative doubles as numbers and make the ranks a permutation of
// 0 .. N-lo-1 whatever the values (NaN included).
static __device__ void column_ranks(const double* nrm, int lo, int N, int* rk, int m, int* who) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int nc = N - lo;
  for (int base = warp * 32; base < 4 * nc; base += nwarps * 32) {
    const int t = base + lane;
    int cnt = 0;
    if (t < 4 * nc) {
      const int j = lo + (t >> 2);
      const long long kj = __double_as_longlong(nrm[j]);
      int i = lo + (t & 3);
#pragma unroll 4
      for (; i < j; i += 4) cnt += __double_as_longlong(nrm[i]) >= kj ? 1 : 0;  // ahead of j: ties count
#pragma unroll 4
      for (; i < N; i += 4) cnt += __double_as_longlong(nrm[i]) > kj ? 1 : 0;   // j itself and behind
    }
    cnt += __shfl_xor_sync(0xffffffffu, cnt, 1);
    cnt += __shfl_xor_sync(0xffffffffu, cnt, 2);
    if (t < 4 * nc && (t & 3) == 0) {
      rk[lo + (t >> 2)] = cnt;
      if (cnt < m) who[cnt] = lo + (t >> 2);
    }
  }
}

// Column moves of one panel pivoting step (shared memory of k_udt): who[r] = the column of
// rank r; per tmp slot the new position of the column saved there (-1: the slot is unused),
// its norm and its original index.
struct PivotMoves {
  int who[kQB];
  int dst[2 * kQB], ord[2 * kQB];
  double nrm[2 * kQB];
};

// Panel-wise column pivoting before the panel [p0, p1), m = p1 - p0 columns:
//  1. the squared norms of the trailing columns over rows p0..N-1 (the matrix as updated by
//     the earlier panels); a warp takes four columns at a time, so that their loads and warp
//     reductions overlap (all RPL rows per lane unrolled when RPL > 0, N <= 32 RPL);
//  2. the rank of every trailing column in decreasing norm, ties by position (column_ranks);
//  3. the column of rank r < m goes to position p0 + r. A panel column of rank >= m goes to a
//     position vacated by a selected column outside the panel: the end of its chain w, the
//     column that moves to w, the column that moves to that one's position, ..., which
//     leaves the panel within m steps. The moving columns (at most 2m) are saved in tmp
//     (2 kQB columns of leading dimension ldt; slot r for rank r, slot m + w - p0 for panel
//     position w) and then written to their new positions with their norms and original
//     indices.
// The selected set and its order are those of m successive selections of the largest
// remaining norm (up to the order among equal norms).
template <int RPL>
__device__ void panel_pivot(double* A, int ld, int N, int p0, int p1, double* nrm, int* order, int* rk,
                            double* tmp, int ldt, PivotMoves& mv) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int m = p1 - p0;
  // warp w takes columns p0 + w, p0 + w + nwarps, ..., four at a time
  for (int j0 = p0 + warp; j0 < N; j0 += 4 * nwarps) {
    double s2[4] = {0.0, 0.0, 0.0, 0.0};
    if (RPL > 0) {
#pragma unroll
      for (int t = 0; t < (RPL > 0 ? RPL : 1); ++t) {
        const int r = p0 + lane + 32 * t;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int j = j0 + u * nwarps;
          if (r < N && j < N) {
            const double v = A[r + (size_t)j * ld];
            s2[u] = fma(v, v, s2[u]);
          }
        }
      }
    } else {
      for (int r = p0 + lane; r < N; r += 32) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int j = j0 + u * nwarps;
          if (j < N) {
            const double v = A[r + (size_t)j * ld];
            s2[u] = fma(v, v, s2[u]);
          }
        }
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) s2[u] = warp_sum(s2[u]);
    if (lane == 0) {
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (j0 + u * nwarps < N) nrm[j0 + u * nwarps] = s2[u];
    }
  }
  __syncthreads();
  column_ranks(nrm, p0, N, rk, m, mv.who);
  __syncthreads();
  for (int j = p0 + warp; j < N; j += nwarps) {  // uniform per warp
    const int r = rk[j];
    int slot = -1, np = j;
    if (r < m) {
      slot = r;
      np = p0 + r;
    } else if (j < p1) {
      slot = m + (j - p0);
      int x = mv.who[j - p0];
      for (int it = 0; it < kQB && x >= p0 && x < p1; ++it) x = mv.who[x - p0];
      np = x;
    }
    if (slot >= 0 && np != j) {
      const double* src = A + (size_t)j * ld;
      for (int rr = lane; rr < N; rr += 32) tmp[rr + (size_t)slot * ldt] = src[rr];
    }
    if (lane == 0) {
      if (slot >= 0) {
        mv.dst[slot] = np != j ? np : -1;
        mv.nrm[slot] = nrm[j];
        mv.ord[slot] = order[j];
      }
      if (j < p1 && slot < m) mv.dst[m + (j - p0)] = -1;  // a selected panel column: its slot is free
    }
  }
  __syncthreads();
  for (int sl = warp; sl < 2 * m; sl += nwarps) {
    const int d = mv.dst[sl];
    if (d >= 0) {
      double* dc = A + (size_t)d * ld;
      for (int rr = lane; rr < N; rr += 32) dc[rr] = tmp[rr + (size_t)sl * ldt];
      if (lane == 0) {
        nrm[d] = mv.nrm[sl];
        order[d] = mv.ord[sl];
      }
    }
  }
  __syncthreads();
}

// The factorisation of the push of interval b onto stack `side` of chain `ch` (X = ch.X; U, D
// into the stack entry b, T into W0). `smem` is the dynamic region (smem_udt_bytes); `mv` the
// pivot moves (shared); x_in_smem (resident only): X is already at the start of `smem` with
// leading dimension smem_ld(N), left there by bchain_body. CPW = panel columns per warp: 1 with 16 warps, 2 with 8. Phases
// (phase hook): 0 load, 1 panel pivoting, 2 panel QR, 3 trailing update, 4 D and T out, 5 Q: trailing
// blocks, 6 Q: panel columns, 7 U out. Every thread of the block calls it; the chain is active and
// b < n_stab.
template <int CPW, class Phase = NoPhase>
__device__ __forceinline__ void udt_body(const HqChain& ch, int side, int b, bool resident, double* smem, PivotMoves& mv,
                                         bool x_in_smem = false, Phase phase = Phase()) {
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
  int* rk = order + N;
  p += N;
  // T factors of the panels that have trailing columns, kept from the factorisation for the
  // formation of Q (panel i at Tc + i kQB^2)
  double* Tc = p;
  const double* X = ch.X;
  if (resident && x_in_smem) {
    // X is in place already: the B chain of the same block left it at the start of smem
  } else if (resident) {
    HQ_FOR_EACH_ELEM(N, i, j) cp_async_8(A + i + (size_t)j * ld, X + i + (size_t)j * N, true);
    cp_async_commit();
  } else {
    HQ_FOR_EACH_ELEM(N, i, j) A[i + (size_t)j * ld] = X[i + (size_t)j * N];
  }
  for (int j = threadIdx.x; j < N; j += blockDim.x) order[j] = j;
  if (resident && !x_in_smem) cp_async_wait<0>();
  __syncthreads();
  phase(0);
  // ---- blocked Householder QR; the pivoting of the first panel is the pre-pivoting (its 16
  // columns are the first 16 of the columns sorted by decreasing norm; the order of the
  // others does not matter, as every later panel selects by norm again) ----
  for (int p0 = 0; p0 < N; p0 += kQB) {
    const int p1 = min(p0 + kQB, N);
    if (N <= 160) {
      panel_pivot<5>(A, ld, N, p0, p1, nrm, order, rk, Vb, ldp, mv);
      phase(1);
      qr_panel_reg<5, CPW>(A, ld, N, p0, p1, tau);
    } else {
      panel_pivot<0>(A, ld, N, p0, p1, nrm, order, rk, Vb, ldp, mv);
      phase(1);
      qr_panel(A, ld, N, p0, p1, tau);
    }
    phase(2);
    if (p1 < N) {
      double* Tp = Tc + (size_t)(p0 / kQB) * kQB * kQB;
      wy_forward(A, ld, N, p0, p1 - p0, tau, Vb, ldp, Tp, S, W, ldp, p1, N - p1);
    }
    phase(3);
  }
  // ---- D = |diag R|, T = D^-1 R P^T (T[:, order[c]] = row-scaled R[:, c]) ----
  const size_t NN = (size_t)N * N;
  double* Dout = ch.stackD + ((size_t)side * ch.n_stab + entry) * N;
  double* Tout = ch.W0;
  for (int r = threadIdx.x; r < N; r += blockDim.x) {
    const double dr = fabs(A[r + (size_t)r * ld]);
    Dout[r] = dr;
    nrm[r] = dr != 0.0 ? 1.0 / dr : 0.0;  // row scale of T; 0 marks a zero row of R
  }
  __syncthreads();
  HQ_FOR_EACH_ELEM(N, r, cc) {
    const double ir = nrm[r];
    const double v = (r <= cc) ? A[r + (size_t)cc * ld] * ir : 0.0;
    Tout[r + (size_t)order[cc] * N] = (ir != 0.0) ? v : (r == cc ? 1.0 : 0.0);
  }
  __syncthreads();
  phase(4);
  // ---- form Q in place, panels backwards: the trailing columns get the panel's WY
  // transformation, the panel's own columns (identity columns until now) are in closed form
  //   Q[:, p0:p1] = E - V T V[p0:p1, :]^T ----
  for (int p0 = ((N - 1) / kQB) * kQB; p0 >= 0; p0 -= kQB) {
    const int p1 = min(p0 + kQB, N), m = p1 - p0;
    const double* Tp = T;
    if (p1 < N) {
      Tp = Tc + (size_t)(p0 / kQB) * kQB * kQB;
      wy_vfill(A, ld, N, p0, m, Vb, ldp);
      wy_apply(A, ld, N, p0, Vb, ldp, Tp, false, W, ldp, p1, N - p1);
    } else {
      wy_factor(A, ld, N, p0, m, tau, Vb, ldp, T, S);
    }
    phase(5);
    for (int t = threadIdx.x; t < kQB * kQB; t += blockDim.x) {
      const int l = t / kQB, j = t % kQB;
      double acc = 0.0;
      if (j < m)
        for (int l2 = 0; l2 < kQB; ++l2) acc = fma(Tp[l * kQB + l2], Vb[(p0 + j) + l2 * ldp], acc);
      W[l * ldp + j] = -acc;
    }
    for (int idx = threadIdx.x; idx < N * m; idx += blockDim.x) {
      const int r = idx % N, j = idx / N;
      A[r + (size_t)(p0 + j) * ld] = (r == p0 + j) ? 1.0 : 0.0;
    }
    __syncthreads();
    rank_update(A + p0 + (size_t)p0 * ld, ld, N - p0, m, Vb + p0, ldp, W, ldp, kQB);
    __syncthreads();
    phase(6);
  }
  double* Uout = ch.stackU + ((size_t)side * ch.n_stab + entry) * NN;
  copy_mat(Uout, N, A, ld, N);
  phase(7);
}

}  // namespace hq
