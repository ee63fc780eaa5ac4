// hq_common.cuh -- device helpers shared by the sm_100a kernel files: shared-memory layouts,
// asynchronous matrix loads, the DMMA rank update of panels, slice ranges of the stabilisation
// intervals and the wrap of G by one B matrix.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <climits>
#include "hq_device.cuh"
#include "hq_kernels.h"

namespace hq {

constexpr int kQB = 16;  // column panel of the blocked Householder UDV factorisation
constexpr int kGJ = 16;  // pivot panel of the blocked Gauss-Jordan inverse

// Phase hook of the factorisation bodies (invert_body, udt_body): called by every thread of the
// block at the end of each phase with the phase's number. The kernels use this no-op; a phase
// timer passes a hook that synchronises the block and reads the clock.
struct NoPhase {
  __device__ __forceinline__ void operator()(int) const {}
};

// shared-memory leading dimension of an N x N matrix: odd, so that threads walking
// consecutive columns hit distinct banks
__host__ __device__ constexpr inline int smem_ld(int N) { return (N % 2 == 0) ? N + 1 : N; }

// leading dimension of the delayed-update panels: = 4 (mod 16) doubles, so that the DMMA
// fragment loads of the flush are free of bank conflicts
__host__ __device__ constexpr inline int panel_ld(int N) { return N + ((4 - N % 16) + 16) % 16; }

// leading dimension of the resident G of k_interval: = 2 (mod 8) doubles, so that the DMMA
// accumulator tiles of the rank updates (lane 4g+q at row g, columns 2q, 2q+1) are free of
// bank conflicts
__host__ __device__ constexpr inline int interval_ld(int N) { return N + ((2 - N % 8) + 8) % 8; }

// bytes of dynamic shared memory of k_interval for a chain of size N with delay depth kmax
// (matrix in smem when `resident`)
__host__ __device__ inline size_t interval_smem_doubles(int N, int kmax, bool resident) {
  const size_t mat = resident ? (size_t)N * interval_ld(N) : 0;
  const size_t panels = (size_t)panel_ld(N) * kmax * 2;
  const size_t stage = (size_t)8 * (((N + 15) & ~15) + 4);
  const size_t work = panels > stage ? panels : stage;
  return mat + work + 3 * (size_t)N + (size_t)(N + 7) / 4 + (size_t)(N + 1) / 2 + 64;
}

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
// ---------------------------------------------------------------------------------
//  Bulk copies through the tensor-memory-access engine (cp.async.bulk, non-tensor form):
//  whole matrix columns between global and shared memory, completed on an mbarrier (loads)
//  or a bulk group (stores). Both addresses and the size must be multiples of 16 bytes:
//  columns of an even N with an even shared leading dimension.
// ---------------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void* p) { return static_cast<unsigned>(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// waits for phase `parity` of the mbarrier with an iteration limit (each try_wait suspends for
// a bounded time); false if the limit ran out
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
  for (int it = 0; it < (1 << 22); ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, unsigned bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(dst), "r"(smem_u32(src)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
// makes this thread's generic-proxy shared-memory writes visible to bulk copies issued later
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// whether the columns of an N x N matrix can move by bulk copies between global memory (leading
// dimension N, 16-byte aligned base) and shared memory (leading dimension ldd, aligned base)
__device__ __forceinline__ bool bulk_columns_ok(const double* gsrc, int N, int ldd) {
  return (N % 2 == 0) && (ldd % 2 == 0) && ((reinterpret_cast<uintptr_t>(gsrc) & 15) == 0);
}

// Loads an N x N column-major matrix into shared memory (leading dimension ldd) by one bulk copy
// per column, issued by warp 0 and completed on `bar` (initialised for one arrival, phase 0).
// Every thread waits for phase `parity` of the barrier (its uses so far, mod 2); on a wait that
// runs out the chain's status word is set. The caller has checked bulk_columns_ok. A barrier
// must separate mbar_init from this call.
__device__ __forceinline__ void load_mat_bulk(double* dst, int ldd, const double* src, int N, uint64_t* bar,
                                              double* status, unsigned parity = 0) {
  const unsigned col = static_cast<unsigned>(N) * sizeof(double);
  if (threadIdx.x == 0) mbar_arrive_expect_tx(bar, col * static_cast<unsigned>(N));
  __syncwarp();
  if (threadIdx.x < 32)
    for (int j = threadIdx.x; j < N; j += 32) bulk_g2s(dst + (size_t)j * ldd, src + (size_t)j * N, col, bar);
  if (!mbar_wait_bounded(bar, parity)) {
    if (threadIdx.x == 0) *status = 1.0;
    mbar_wait_bounded(bar, parity);  // the copies in flight still land in this CTA's shared memory
  }
}

// Stores an N x N matrix from shared memory (leading dimension lds) to global memory (leading
// dimension N) by one bulk copy per column from warp 0, and waits for the copies to complete.
// Every thread calls it after its last write of the matrix.
__device__ __forceinline__ void store_mat_bulk(double* dst, const double* src, int lds, int N) {
  fence_proxy_async_smem();
  __syncthreads();
  if (threadIdx.x < 32) {
    const unsigned col = static_cast<unsigned>(N) * sizeof(double);
    for (int j = threadIdx.x; j < N; j += 32) bulk_s2g(dst + (size_t)j * N, src + (size_t)j * lds, col);
    bulk_commit();
    bulk_wait_all();
  }
}

// G[0:M, 0:Nc] += X[0:M, 0:k] Y[0:k, 0:Nc]  (X column-major ldx, Y row-major ldy, k <= 16),
// by 16 x 32 strips of four 16 x 8 DMMA tiles that share the A fragments; the fragments of
// all k-steps are loaded before the strip's G tiles so that their latencies overlap
static __device__ void rank_update(double* G, int ld, int M, int Nc, const double* X, int ldx, const double* Y, int ldy,
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
static __device__ void flush_panels(double* G, int ld, int N, const double* X, int ldx, const double* Y, int ldy, int k) {
  rank_update(G, ld, N, N, X, ldx, Y, ldy, k);
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

// scaling of index i: 1 (mode 0 or no vector), v[i] (1), 1 / max(v[i], 1) (2), min(v[i], 1) (3)
__device__ __forceinline__ double vscale(const double* v, int mode, int i) {
  if (!v || mode == 0) return 1.0;
  const double x = v[i];
  if (mode == 1) return x;
  if (mode == 2) return 1.0 / fmax(x, 1.0);
  return fmin(x, 1.0);
}

}  // namespace hq
