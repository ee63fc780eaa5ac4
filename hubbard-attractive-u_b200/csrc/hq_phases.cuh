// hq_phases.cuh -- per-chain phase bodies shared by the one-launch-per-phase kernels of
// hq_kernels.cu and the persistent sweep kernel: the B chain of a stack push, the estimators of a
// freshly built G and a one-CTA FP64 DMMA GEMM of the G builders.
#pragma once
#include "hq_common.cuh"

namespace hq {

// ---------------------------------------------------------------------------------
//  B chain: X <- (U_top diag(D_top) or 1), then the B products of interval b:
//   up  : X <- B(t) X = e^{V_t} E X, t ascending            (src/dqmc_core.cpp:190)
//   down: X <- B(t)^T X = E e^{V_t} X, t descending           (src/dqmc_core.cpp:251)
//  dir UP pushes onto the left stack, DOWN onto the right stack; that stack holds b
//  entries before the push (top entry b-1, none when b = 0).
//  init: the right stack at initialisation (src/dqmc_core.cpp:67-87) is the down
//  direction without updates.
// ---------------------------------------------------------------------------------
// The B products of interval b applied to the top of the pushing stack (X = U_top D_top, or 1),
// into ch.X. `smem` is the dynamic region (N x smem_ld(N) when resident, then the stage); s holds
// N fields (shared). keep_x (resident only): X stays at the start of `smem` (leading dimension
// smem_ld(N)) for the factorisation that follows in the same block, instead of going to ch.X.
// Every thread of the block calls it; the chain is active and b < n_stab.
__device__ __forceinline__ void bchain_body(const HqChain& ch, int dir, int b, bool resident, double* smem, int8_t* s,
                                            bool keep_x = false) {
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
  if (resident && !keep_x) copy_mat(ch.X, N, X, ld, N);
}

// ---------------------------------------------------------------------------------
//  Estimators + snapshot of G after a stabilisation (slice `lslice` computed from the
//  interval), the last slice of every interval.
// ---------------------------------------------------------------------------------
// The estimators and the snapshot of the freshly built G at the end of interval b (the
// interval's last slice). red: 96 shared doubles.
__device__ __forceinline__ void measure_body(const HqChain& ch, int dir, int b, int flags, double* red) {
  const int N = ch.N;
  int t_lo, t_hi;
  interval_range(ch.nt, ch.pace, ch.n_stab, dir, b, t_lo, t_hi);
  // up / dynamic: the last slice is t_hi, stored at t_hi % nt; down: t_lo, stored at t_lo - 1
  const int lm = (dir == HQ_DOWN) ? ((t_lo - 1) % ch.nt) : (t_hi % ch.nt);
  if (flags & HQ_F_MEASURE) measure_slice(ch.G, N, N, ch.acc, red);
  if ((flags & HQ_F_SNAPSHOT) && ch.snap_tt) copy_mat(ch.snap_tt + (size_t)lm * N * N, N, ch.G, N, N);
}

}  // namespace hq
