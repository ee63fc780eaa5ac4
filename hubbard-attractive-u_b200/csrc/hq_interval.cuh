// hq_interval.cuh -- the body of one stabilisation interval of one chain: G(tau,tau) resident in
// shared memory while the slices of the interval are wrapped (src/dqmc_core.cpp:142-161) and
// updated by Metropolis flips with delayed rank-k updates flushed by DMMA
// (src/dqmc_core.cpp:102-119, src/hubbard.cpp:123-139); fused equal-time estimators
// (include/observable_methods.hpp:39-151) and optional per-slice snapshots. Used by k_interval
// (one launch per interval) and by the persistent sweep kernel.
#pragma once
#include "hq_metropolis.cuh"

namespace hq {

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
      const int nb = min(NB, N - b0);
      // the fast walk without the ratio log unless it is on; near a tie the exact walk again
      if constexpr (NB == 16) {
        const bool near = log ? walk_block16<false, true>(ch, G, ld, sh, b0, nb, true, bi & 1)
                              : walk_block16<false, false>(ch, G, ld, sh, b0, nb, false, bi & 1);
        if (near) walk_block16<true>(ch, G, ld, sh, b0, nb, log, bi & 1);
      } else {
        const bool near = log ? walk_block<NB, false, true>(ch, G, ld, sh, b0, nb, true, bi & 1)
                              : walk_block<NB, false, false>(ch, G, ld, sh, b0, nb, false, bi & 1);
        if (near) walk_block<NB, true>(ch, G, ld, sh, b0, nb, log, bi & 1);
      }
    }
    __syncthreads();
    // the count alternates between two words: with no flush (a == 0) no barrier follows,
    // and warp 0 writes the next block's count while other warps may still read this one
    const int a = sh.ired[bi & 1];
    if (tid == 0) acc_count += a;
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

// Shared-memory words of the interval body besides its dynamic region (interval_smem_doubles):
// reductions, block counts, the barrier of the bulk load of G and the walk records.
struct IntervalScratch {
  double* red;     // 96 doubles
  int* ired;       // 64 ints
  uint64_t* gbar;  // mbarrier of the bulk load of G (initialised for one arrival)
  int* qj;         // 16 ints
  double* qg;      // 16 doubles
  double* xt;      // 16 x 16 doubles, 16-byte aligned
  double* yt;      // 16 x 16 doubles, 16-byte aligned
};
constexpr int kIntervalScratchBytes = (96 + 16 + 512) * 8 + (64 + 16) * 4 + 16;

// Places the interval scratch at `p` (16-byte aligned, kIntervalScratchBytes long).
__device__ __forceinline__ IntervalScratch interval_scratch_at(void* p) {
  IntervalScratch sc;
  double* d = reinterpret_cast<double*>(p);
  sc.xt = d; d += 256;
  sc.yt = d; d += 256;
  sc.red = d; d += 96;
  sc.qg = d; d += 16;
  sc.gbar = reinterpret_cast<uint64_t*>(d); d += 2;
  sc.ired = reinterpret_cast<int*>(d);
  sc.qj = sc.ired + 64;
  return sc;
}

// The update (or no-update) slices of stabilisation interval b of chain `ch` in direction dir.
// `smem` is the dynamic region (interval_smem_doubles(N, kmax, resident) doubles); gpar is the
// phase parity of sc.gbar for this interval's bulk load of G. Every thread of the block calls
// it; the chain is active and b < n_stab.
__device__ __forceinline__ void interval_body(const HqChain& ch, int dir, int b, int flags, bool resident, double* smem,
                                              const IntervalScratch& sc, unsigned gpar) {
  const int N = ch.N;
  int t_lo, t_hi;
  interval_range(ch.nt, ch.pace, ch.n_stab, dir, b, t_lo, t_hi);

  // shared-memory carve-up; the resident G moves in and out by bulk copies of its columns
  // (cp.async per element where the columns are not 16-byte multiples)
  double* p = smem;
  double* G;
  int ld;
  bool bulk = false;
  if (resident) {
    G = p;
    ld = interval_ld(N);
    p += (size_t)N * ld;
    bulk = bulk_columns_ok(ch.G, N, ld);
    if (bulk) load_mat_bulk(G, ld, ch.G, N, sc.gbar, ch.acc + HQ_ACC_STATUS, gpar);
    else load_mat_async(G, ld, ch.G, N, N);
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
  sh.ired = sc.ired;
  sh.qj = sc.qj;
  sh.qg = sc.qg;
  sh.xt = sc.xt;
  sh.yt = sc.yt;
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
      wrap_slice(ch, G, ld, sh.s, HQ_UP, work, (fused && step > 0) ? ch.acc : nullptr, sc.red);
      metropolis_dispatch(ch, G, ld, sh, rng, n_acc, flags, log_base);
      n_prop += N;
      log_base += N;
    } else if (dir == HQ_DOWN) {
      metropolis_dispatch(ch, G, ld, sh, rng, n_acc, flags, log_base);
      n_prop += N;
      log_base += N;
      wrap_slice(ch, G, ld, sh.s, HQ_DOWN, work, (fused && step < nsl - 1) ? ch.acc : nullptr, sc.red);
    } else {
      wrap_slice(ch, G, ld, sh.s, HQ_UP, work);
    }
    for (int i = threadIdx.x; i < N; i += blockDim.x) ch.fields[(size_t)l * N + i] = sh.s[i];
    if (step < nsl - 1) {
      const int lm = (dir == HQ_DOWN) ? ((t - 1) % ch.nt) : l;
      if ((flags & HQ_F_MEASURE) && !fused) measure_slice(G, ld, N, ch.acc, sc.red);
      if ((flags & HQ_F_SNAPSHOT) && ch.snap_tt) copy_mat(ch.snap_tt + (size_t)lm * N * N, N, G, ld, N);
    }
    __syncthreads();
  }
  if (resident) {
    if (bulk) store_mat_bulk(ch.G, G, ld, N);
    else copy_mat(ch.G, N, G, ld, N);
  }
  if (threadIdx.x == 0) {
    *ch.rng = rng;
    ch.acc[HQ_ACC_PROPOSED] += n_prop;
    ch.acc[HQ_ACC_ACCEPTED] += n_acc;
    if ((flags & HQ_F_LOG_RATIOS) && ch.ratio_count) *ch.ratio_count = log_base;
  }
}

}  // namespace hq
