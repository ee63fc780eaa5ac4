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
//  (Q = B_0 B_1 ..., B_p = I - V_p T_p V_p^T).
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

// Panel-wise column pivoting before the panel [p0, p1): the norms of the trailing columns over
// rows p0..N-1 (the matrix as updated by the earlier panels); warp 0 then makes the p1 - p0
// selections one after the other, each moving the remaining column of largest norm (smallest
// index among equal norms) into the next panel position (norms and original indices swap with
// it), and records the swaps; finally every thread applies the recorded swaps, in order, to
// the rows it owns. piv holds kQB ints.
__device__ void panel_pivot(double* A, int ld, int N, int p0, int p1, double* nrm, int* order, int* piv) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
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
  if (warp == 0) {
    for (int q = p0; q < p1; ++q) {
      double best = -1.0;
      int bj = N;
      for (int j = q + lane; j < N; j += 32) {
        const double v = nrm[j];
        if (v > best) { best = v; bj = j; }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oj = __shfl_xor_sync(0xffffffffu, bj, o);
        if (ob > best || (ob == best && oj < bj)) { best = ob; bj = oj; }
      }
      if (bj >= N) bj = q;
      if (lane == 0) {
        piv[q - p0] = bj;
        if (bj != q) {
          const double tn = nrm[q]; nrm[q] = nrm[bj]; nrm[bj] = tn;
          const int to = order[q]; order[q] = order[bj]; order[bj] = to;
        }
      }
      __syncwarp();
    }
  }
  __syncthreads();
  for (int r = threadIdx.x; r < N; r += blockDim.x)
    for (int q = p0; q < p1; ++q) {
      const int jp = piv[q - p0];
      if (jp != q) {
        const double t0 = A[r + (size_t)q * ld];
        A[r + (size_t)q * ld] = A[r + (size_t)jp * ld];
        A[r + (size_t)jp * ld] = t0;
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
  __shared__ int piv[kQB];
  for (int p0 = 0; p0 < N; p0 += kQB) {
    const int p1 = min(p0 + kQB, N);
    if (p0 > 0) panel_pivot(A, ld, N, p0, p1, nrm, order, piv);
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

cudaError_t launch_udt(const HqChain* chains, int n, int side, int b, int Nmax, bool resident, cudaStream_t st) {
  const size_t bytes = smem_udt_bytes(Nmax, resident);
  k_udt<<<n, HQ_THREADS, bytes, st>>>(chains, n, side, 0, b, resident ? 1 : 0);
  return cudaGetLastError();
}
const void* fn_udt() { return (const void*)k_udt; }

}  // namespace hq
