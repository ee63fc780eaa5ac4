// hq_invert.cuh -- the blocked Gauss-Jordan inverse of the G builders (the inverse() of
// include/utils/stable_numerics.hpp:235), used by k_invert (one launch per builder) and by the
// persistent sweep kernel.
#pragma once
#include "hq_common.cuh"

namespace hq {

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

// the same for five slots as a tree of depth 3 (bits 0, 1 and 2 of r / 32)
template <>
__device__ __forceinline__ double slot_at<5>(const double (&x)[5], int r) {
  const int t = r >> 5;
  double a, b, c, v;
  asm("{\n\t.reg .pred p;\n\tsetp.ne.s32 p, %3, 0;\n\tselp.f64 %0, %2, %1, p;\n\t}" : "=d"(a) : "d"(x[0]), "d"(x[1]), "r"(t & 1));
  asm("{\n\t.reg .pred p;\n\tsetp.ne.s32 p, %3, 0;\n\tselp.f64 %0, %2, %1, p;\n\t}" : "=d"(b) : "d"(x[2]), "d"(x[3]), "r"(t & 1));
  asm("{\n\t.reg .pred p;\n\tsetp.ne.s32 p, %3, 0;\n\tselp.f64 %0, %2, %1, p;\n\t}" : "=d"(c) : "d"(a), "d"(b), "r"(t & 2));
  asm("{\n\t.reg .pred p;\n\tsetp.ne.s32 p, %3, 0;\n\tselp.f64 %0, %2, %1, p;\n\t}" : "=d"(v) : "d"(c), "d"(x[4]), "r"(t & 4));
  return v;
}

// pivot k of a register-resident Gauss-Jordan panel, by the warp that holds column k:
// partial pivoting (largest |A[r][k]|, r >= k, smallest index among equals), row swap in
// this column, the multipliers into fcol, the inverse's column k into x, and perm / pinv
template <int RPL>
__device__ __forceinline__ void gj_pivot_reg(double (&x)[RPL], int k, int N, double* fcol, double* pinv_out,
                                             int* perm, double* status) {
  const int lane = threadIdx.x & 31;
  // the lane's candidate: the largest |x[t]| over its rows r >= k, the smallest such row among
  // equals; rows out of range and NaNs are (-1, N) and never win. A pairwise tree over the slots
  // (depth 3 for five) gives the same pair as a scan in row order.
  double cv[RPL];
  int cr[RPL];
#pragma unroll
  for (int t = 0; t < RPL; ++t) {
    const int r = lane + 32 * t;
    const double v = fabs(x[t]);
    const bool ok = r >= k && r < N && v == v;
    cv[t] = ok ? v : -1.0;
    cr[t] = ok ? r : N;
  }
#pragma unroll
  for (int w = 1; w < RPL; w *= 2)
#pragma unroll
    for (int t = 0; t + w < RPL; t += 2 * w) {
      const bool tb = cv[t + w] > cv[t] || (cv[t + w] == cv[t] && cr[t + w] < cr[t]);
      cv[t] = tb ? cv[t + w] : cv[t];
      cr[t] = tb ? cr[t + w] : cr[t];
    }
  double best = cv[0];
  int bi = cr[0];
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
  const double pinv = ok ? __drcp_rn(vb) : 0.0;  // = 1 / vb, correctly rounded
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

// Gauss-Jordan on the panel columns [p0, p0 + nb) of A (all rows), N <= 32 RPL: the panel's
// columns are held in registers, CPW per warp by kGJ / CPW warps (warp w holds columns
// p0 + w + i kGJ / CPW); the owner of column k+1 takes pivot k+1 right after its own elimination
// step for pivot k, so one block barrier separates pivots. Multipliers and the reciprocal pivot
// are double-buffered by pivot parity (fcol: 2N doubles, pv: 2).
template <int RPL, int CPW>
__device__ void gj_panel_reg(double* A, int ld, int N, int p0, int nb, int* perm, double* fcol, double* pv,
                             double* status) {
  constexpr int NWP = kGJ / CPW;  // warps that hold panel columns
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int col[CPW];
  bool own[CPW];
  double x[CPW][RPL];
#pragma unroll
  for (int i = 0; i < CPW; ++i) {
    col[i] = p0 + warp + i * NWP;
    own[i] = warp < NWP && warp + i * NWP < nb;
#pragma unroll
    for (int t = 0; t < RPL; ++t) {
      const int r = lane + 32 * t;
      x[i][t] = (own[i] && r < N) ? A[r + (size_t)col[i] * ld] : 0.0;
    }
  }
  if (warp == 0) gj_pivot_reg<RPL>(x[0], p0, N, fcol, pv, perm, status);
  __syncthreads();
  for (int q = 0; q < nb; ++q) {
    const int k = p0 + q, par = q & 1;
#pragma unroll
    for (int i = 0; i < CPW; ++i) {
      if (own[i] && col[i] != k) {
        const int bi = perm[k];
        const double pinv = pv[par];
        const double* f = fcol + par * N;
        // row swap k <-> bi in this column, then row k scaled by the pivot's reciprocal
        const double vk = __shfl_sync(0xffffffffu, slot_at<RPL>(x[i], k), k & 31);
        const double vb = __shfl_sync(0xffffffffu, slot_at<RPL>(x[i], bi), bi & 31);
        const double u = vb * pinv;
#pragma unroll
        for (int t = 0; t < RPL; ++t) {
          const int r = lane + 32 * t;
          const double v = (r == bi) ? vk : x[i][t];
          x[i][t] = (r == k) ? u : ((r < N) ? fma(-f[r < N ? r : 0], u, v) : v);
        }
        if (col[i] == k + 1 && q + 1 < nb)
          gj_pivot_reg<RPL>(x[i], k + 1, N, fcol + (par ^ 1) * N, pv + (par ^ 1), perm, status);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < CPW; ++i)
#pragma unroll
    for (int t = 0; t < RPL; ++t) {
      const int r = lane + 32 * t;
      if (own[i] && r < N) A[r + (size_t)col[i] * ld] = x[i][t];
    }
  __syncthreads();
}

// The in-place inverse of the builder matrix `which` (0: W1, 1: W2, 2: W3, 3: W5) of chain `ch`.
// `smem` is the dynamic region (smem_invert_bytes); pv two shared doubles. CPW = panel columns
// per warp: 1 with 16 warps, 2 with 8. Phases (phase hook): 1 panel pivots, 2 row interchanges and
// panel staging, 3 rank update, 4 column order, 5 write-back. Every thread of the block calls it;
// the chain is active and b < n_stab.
template <int CPW, class Phase = NoPhase>
__device__ __forceinline__ void invert_body(const HqChain& ch, int which, bool resident, double* smem, double* pv,
                                            Phase phase = Phase()) {
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
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  for (int p0 = 0; p0 < N; p0 += kGJ) {
    const int nb = min(kGJ, N - p0);
    if (N <= 160) gj_panel_reg<5, CPW>(A, ld, N, p0, nb, perm, fcol, pv, ch.acc + HQ_ACC_STATUS);
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
    phase(1);
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
    phase(2);
    // A[:, j] += Wp Bf[:, j] for every column outside the panel (Bf is zero on the panel)
    flush_panels(A, ld, N, Wp, ldp, Bf, ldp, nb);
    __syncthreads();
    phase(3);
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
  phase(4);
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
  phase(5);
}

}  // namespace hq
