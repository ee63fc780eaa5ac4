// hq_udt.cu -- k_udt, the UDV factorisation of a stack push (blocked Householder QR with
// panel-wise column pivoting, in place of the dgesvd of include/utils/svd_stack.hpp:107-175).
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

// V of the panel [p0, p0+m) with explicit unit diagonal and zeros above (columns >= m zero)
__device__ void wy_vfill(const double* A, int ld, int N, int p0, int m, double* Vb, int ldv) {
  for (int q = threadIdx.x >> 5; q < kQB; q += blockDim.x >> 5)
    for (int r = p0 + (threadIdx.x & 31); r < N; r += 32) {
      const int c = p0 + q;
      Vb[r + q * ldv] = (q >= m || r < c) ? 0.0 : (r == c ? 1.0 : A[r + (size_t)c * ld]);
    }
  __syncthreads();
}

// V of the panel [p0, p0+m) (wy_vfill) and the triangular factor T of
// H_p0 ... H_p0+m-1 = I - V T V^T
__device__ void wy_factor(const double* A, int ld, int N, int p0, int m, const double* tau, double* Vb, int ldv,
                          double* T, double* S) {
  wy_vfill(A, ld, N, p0, m, Vb, ldv);
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

// rk[j] = the rank of column j among the columns [lo, N) in decreasing nrm, ties by position.
// Four threads per column, each counting over one residue of positions mod 4. The norms are
// compared as the integer patterns of their bits, which order non-negative doubles as numbers
// and make the ranks a permutation of 0 .. N-lo-1 whatever the values (NaN included).
__device__ void column_ranks(const double* nrm, int lo, int N, int* rk) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int nc = N - lo;
  for (int base = warp * 32; base < 4 * nc; base += nwarps * 32) {
    const int t = base + lane;
    int cnt = 0;
    if (t < 4 * nc) {
      const int j = lo + (t >> 2);
      const long long kj = __double_as_longlong(nrm[j]);
      for (int i = lo + (t & 3); i < N; i += 4) {
        const long long ki = __double_as_longlong(nrm[i]);
        cnt += (ki > kj || (ki == kj && i < j)) ? 1 : 0;
      }
    }
    cnt += __shfl_xor_sync(0xffffffffu, cnt, 1);
    cnt += __shfl_xor_sync(0xffffffffu, cnt, 2);
    if (t < 4 * nc && (t & 3) == 0) rk[lo + (t >> 2)] = cnt;
  }
}

// Column moves of one panel pivoting step (shared memory of k_udt).
struct PivotMoves {
  int src[2 * kQB], dst[2 * kQB], ord[2 * kQB];
  double nrm[2 * kQB];
  int vac[kQB];
  int count;
};

// Panel-wise column pivoting before the panel [p0, p1), m = p1 - p0 columns:
//  1. the squared norms of the trailing columns over rows p0..N-1 (the matrix as updated by
//     the earlier panels);
//  2. the rank of every trailing column in decreasing norm, ties by position, all ranks at
//     once (column_ranks);
//  3. the columns of rank < m go to positions p0 + rank; the panel's other columns take the
//     positions so vacated, both in position order (warp 0, by ballots). At most 2m columns
//     move: they are gathered (all rows) into tmp (2 kQB columns of leading dimension ldt)
//     and scattered to their new positions, with their norms and original indices.
// The selected set and its order are those of m successive selections of the largest
// remaining norm (up to the order among equal norms).
__device__ void panel_pivot(double* A, int ld, int N, int p0, int p1, double* nrm, int* order, int* rk,
                            double* tmp, int ldt, PivotMoves& mv) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int m = p1 - p0;
  for (int j = p0 + warp; j < N; j += nwarps) {
    double s2 = 0.0;
    for (int r = p0 + lane; r < N; r += 32) {
      const double v = A[r + (size_t)j * ld];
      s2 = fma(v, v, s2);
    }
    s2 = warp_sum(s2);
    if (lane == 0) nrm[j] = s2;
  }
  __syncthreads();
  column_ranks(nrm, p0, N, rk);
  __syncthreads();
  if (warp == 0) {
    const unsigned below = (1u << lane) - 1u;
    int nvac = 0;
    for (int base = p1; base < N; base += 32) {
      const int j = base + lane;
      const bool v = j < N && rk[j] < m;
      const unsigned b = __ballot_sync(0xffffffffu, v);
      const int s = nvac + __popc(b & below);
      if (v && s < kQB) mv.vac[s] = j;
      nvac += __popc(b);
    }
    __syncwarp();
    int ndisp = 0, nmv = 0;
    for (int base = p0; base < N; base += 32) {
      const int j = base + lane;
      int np = j;
      bool disp = false;
      if (j < N) {
        const int r = rk[j];
        if (r < m) np = p0 + r;
        else if (j < p1) disp = true;
      }
      const unsigned bd = __ballot_sync(0xffffffffu, disp);
      if (disp) {
        const int s = ndisp + __popc(bd & below);
        np = (s < nvac && s < kQB) ? mv.vac[s] : j;
      }
      ndisp += __popc(bd);
      const bool moves = j < N && np != j;
      const unsigned bm = __ballot_sync(0xffffffffu, moves);
      const int s = nmv + __popc(bm & below);
      if (moves && s < 2 * kQB) {
        mv.src[s] = j;
        mv.dst[s] = np;
        mv.nrm[s] = nrm[j];
        mv.ord[s] = order[j];
      }
      nmv += __popc(bm);
    }
    if (lane == 0) mv.count = min(nmv, 2 * kQB);
  }
  __syncthreads();
  const int nmv = mv.count;
  for (int t = warp; t < nmv; t += nwarps) {
    const double* s = A + (size_t)mv.src[t] * ld;
    for (int r = lane; r < N; r += 32) tmp[r + (size_t)t * ldt] = s[r];
  }
  __syncthreads();
  for (int t = warp; t < nmv; t += nwarps) {
    double* d = A + (size_t)mv.dst[t] * ld;
    for (int r = lane; r < N; r += 32) d[r] = tmp[r + (size_t)t * ldt];
    if (lane == 0) {
      nrm[mv.dst[t]] = mv.nrm[t];
      order[mv.dst[t]] = mv.ord[t];
    }
  }
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
  int* rk = order + N;
  p += N;
  // T factors of the panels that have trailing columns, kept from the factorisation for the
  // formation of Q (panel i at Tc + i kQB^2)
  double* Tc = p;
  __shared__ PivotMoves mv;
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
  column_ranks(nrm, 0, N, rk);
  __syncthreads();
  for (int j = threadIdx.x; j < N; j += blockDim.x) order[rk[j]] = j;
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
    if (p0 > 0) panel_pivot(A, ld, N, p0, p1, nrm, order, rk, Vb, ldp, mv);
    if (N <= 160) qr_panel_reg<5>(A, ld, N, p0, p1, tau);
    else qr_panel(A, ld, N, p0, p1, tau);
    if (p1 < N) {
      double* Tp = Tc + (size_t)(p0 / kQB) * kQB * kQB;
      wy_factor(A, ld, N, p0, p1 - p0, tau, Vb, ldp, Tp, S);
      wy_apply(A, ld, N, p0, Vb, ldp, Tp, true, W, ldp, p1, N - p1);
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
    const double* Tp = T;
    if (p1 < N) {
      Tp = Tc + (size_t)(p0 / kQB) * kQB * kQB;
      wy_vfill(A, ld, N, p0, m, Vb, ldp);
      wy_apply(A, ld, N, p0, Vb, ldp, Tp, false, W, ldp, p1, N - p1);
    } else {
      wy_factor(A, ld, N, p0, m, tau, Vb, ldp, T, S);
    }
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
  }
  double* Uout = ch.stackU + ((size_t)side * ch.n_stab + entry) * NN;
  copy_mat(Uout, N, A, ld, N);
}

cudaError_t launch_udt(const HqChain* chains, int n, int side, int b, int Nmax, bool resident, cudaStream_t st) {
  const size_t bytes = smem_udt_bytes(Nmax, resident);
  k_udt<<<n, HQ_THREADS, bytes, st>>>(chains, n, side, 0, b, resident ? 1 : 0);
  return cudaGetLastError();
}
const void* fn_udt() { return (const void*)k_udt; }

}  // namespace hq
