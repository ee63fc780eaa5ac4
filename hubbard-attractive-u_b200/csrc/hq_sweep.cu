// hq_sweep.cu -- k_sweep, the persistent kernel of one directional update sweep
// (src/dqmc_core.cpp:167-284) of every chain of a context: ONE launch per sweep.
//
// The grid holds one CTA of 8 warps per SM. Each CTA repeatedly takes a work item, the next
// stabilisation interval of one chain, and runs all of it in the order of the launch sequence
// it replaces:
//   interval_body (wrap + Metropolis of the interval's slices, G resident in shared memory)
//   bchain_body   (B products of the interval applied to the top of the pushing stack)
//   udt_body      (UDV factorisation of the push)
//   gemm_cta      (cumulative V^T of the push)
//   gemm_cta x 2, invert_body, gemm_cta x 2 (the equal-time G builder, wrap error)
//   measure_body  (estimators / snapshot of the fresh G)
// The items of a chain follow each other through per-chain progress words: the CTA that
// completes an interval publishes it with a release, and the CTA that claims the chain's next
// interval has acquired it. A CTA only claims an interval whose predecessor has completed, so it
// never waits on a running item: the kernel cannot deadlock, and when no chain is ready the
// waits end as running items complete. Every look at the queue is counted; when the limit runs
// out the context's abort word is raised (every CTA stops) and the chains' status words are set.
//
// Every phase performs the same floating-point operations as the kernel of the launch sequence
// it replaces (k_interval, k_bchain, k_udt, k_gemm, k_invert; the panel columns of the
// factorisations are held two per warp instead of one), so both paths give the same G and the
// same field trajectories; only the estimator sums are reduced over 8 warps instead of 16.
#include <algorithm>

#include "hq_cta_gemm.cuh"
#include "hq_interval.cuh"
#include "hq_invert.cuh"
#include "hq_phases.cuh"
#include "hq_udt.cuh"

namespace hq {

// ---------------------------------------------------------------------------------
//  Scheduling: an item is the next interval of one chain. Per chain, two words (zeroed before
//  every launch): progress (intervals completed in this sweep) and next (intervals claimed). A
//  chain is ready when progress == next < n_stab: its previous interval has completed and its
//  next one is unclaimed. A free CTA claims (compare-and-swap on next) the ready chain with the
//  longest remaining work, (n_stab - next) x its cost per interval (list scheduling by the
//  longest remaining path: chains of many or dear intervals go first, and chains of equal work
//  advance in step, so the sweep ends with all chains at once). When no chain is ready it sleeps
//  briefly and looks again; it never waits on one chain while another is ready.
//   ctl[0]            items claimed      ctl[1]  abort: a wait ran out
//   ctl[3 + c]        progress of chain c
//   ctl[3 + n + c]    next interval of chain c to claim
// ---------------------------------------------------------------------------------
constexpr int kSweepWaitLimit = 1 << 22;  // looks while nothing is ready (each sleeps ~0.25 us)

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_relaxed(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_proxy_async_all() { asm volatile("fence.proxy.async;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

// Warp 0 claims the next item (see above): {chain, interval}; {-1, 0} when every item is claimed,
// {-2, 0} when the abort word is raised or the wait limit ran out (the abort word is then raised).
// The lane that wins the claim has acquired the chain's progress word. cinfo[c] = {n_stab, cost}.
__device__ int2 take_item(const int2* __restrict__ cinfo, int nchains, int nitems, int* ctl) {
  const int lane = threadIdx.x & 31;
  const int* progress = ctl + 3;
  int* next = ctl + 3 + nchains;
  for (int look = 0; look < kSweepWaitLimit; ++look) {
    if (ld_relaxed(ctl + 1) != 0) return make_int2(-2, 0);
    if (ld_relaxed(ctl) >= nitems) return make_int2(-1, 0);
    // this lane's ready chain of the largest remaining work; among equals each CTA prefers the
    // chains from its own offset on (rank (c - rot) mod n), so that CTAs looking at the same time
    // claim different chains of equal work instead of contending for one
    const int rot = (int)(((long long)blockIdx.x * nchains) / gridDim.x);
    long long key = -1;
    int bc = -1, bb = 0, br = 0;
    for (int c = lane; c < nchains; c += 32) {
      const int2 ci = cinfo[c];
      const int nb = ld_relaxed(next + c);
      if (nb < ci.x && ld_acquire(progress + c) == nb) {
        const long long k = (long long)(ci.x - nb) * ci.y;
        const int r = c >= rot ? c - rot : c - rot + nchains;
        if (k > key || (k == key && r < br)) { key = k; bc = c; bb = nb; br = r; }
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const long long ok = __shfl_xor_sync(0xffffffffu, key, o);
      const int oc = __shfl_xor_sync(0xffffffffu, bc, o);
      const int ob = __shfl_xor_sync(0xffffffffu, bb, o);
      const int orr = __shfl_xor_sync(0xffffffffu, br, o);
      if (ok > key || (ok == key && oc >= 0 && (bc < 0 || orr < br))) { key = ok; bc = oc; bb = ob; br = orr; }
    }
    if (bc < 0) {
      __nanosleep(256);
      continue;
    }
    // every lane holds the winner; the lane that examined it (bc mod 32) claims it
    int got = 0;
    if (lane == (bc & 31)) {
      got = atomicCAS(next + bc, bb, bb + 1) == bb;
      if (got) atomicAdd(ctl, 1);
    }
    if (__shfl_sync(0xffffffffu, got, bc & 31)) return make_int2(bc, bb);
  }
  if (lane == 0) atomicExch(ctl + 1, 1);
  return make_int2(-2, 0);
}

// doubles of the B-chain region (matrix + stage), after which its fields of one slice sit
__host__ __device__ inline size_t bchain_doubles(int N) {
  return (size_t)N * smem_ld(N) + 8 * (((N + 15) & ~15) + 4) + 64;
}

__global__ void __launch_bounds__(HQ_INT_THREADS, 1)
k_sweep(const HqChain* __restrict__ chains, int nchains, const int2* __restrict__ cinfo, int nitems,
        const HqGemmJob* const* __restrict__ lists, int nstab_max, int dir, int flags, int* ctl,
        unsigned long long* clk) {
  extern __shared__ __align__(16) double smem[];
  __shared__ HqChain ch;
  __shared__ PivotMoves mv;
  __shared__ double red[96];
  __shared__ double pv[2];
  __shared__ int2 s_item;
  __shared__ HqGemmJob job;
  const int side = (dir == HQ_DOWN) ? 1 : 0;
  // phase cycles (HQ_F_PHASE_CLOCKS), taken by thread 0 after the barrier that ends a phase
  const bool clocks = (flags & HQ_F_PHASE_CLOCKS) && clk;
  long long t_mark = 0;
  auto mark = [&](int slot) {
    if (clocks && threadIdx.x == 0) {
      const long long t = clock64();
      atomicAdd(clk + slot, (unsigned long long)(t - t_mark));
      t_mark = t;
    }
  };
  for (;;) {
    if (threadIdx.x < 32) {
      if (threadIdx.x == 0) t_mark = clock64();
      const int2 it = take_item(cinfo, nchains, nitems, ctl);
      if (threadIdx.x == 0) {
        if (it.x >= 0) {
          ch = chains[it.x];
          mark(0);
          if (clocks) atomicAdd(clk + 9, 1ull);
        } else if (it.x == -2) {
          // a wait ran out: mark every chain's status (the sweep is incomplete)
          for (int c2 = 0; c2 < nchains; ++c2) chains[c2].acc[HQ_ACC_STATUS] = 2.0;
        }
        s_item = it;
      }
    }
    __syncthreads();
    if (s_item.x < 0) break;
    const int c = s_item.x, b = s_item.y, N = ch.N;
    // the previous interval of this chain may have run on another SM: thread 0 acquired its
    // release; every thread orders its loads (and, through the proxy fence, this CTA's bulk
    // copies) after it
    __threadfence();
    fence_proxy_async_all();
    // ---- wrap + Metropolis of the interval (G resident in shared memory) ----
    {
      const size_t off = (interval_smem_doubles(N, ch.kmax, true) + 1) & ~size_t(1);
      const IntervalScratch sc = interval_scratch_at(smem + off);
      if (threadIdx.x == 0) mbar_init(sc.gbar, 1);
      __syncthreads();
      interval_body(ch, dir, b, flags, true, smem, sc, 0u);
      // the bulk store of G has completed (warp 0 waited for it): order it before the generic
      // accesses of the phases below
      if (threadIdx.x < 32) fence_proxy_async_all();
      __syncthreads();
      if (threadIdx.x == 0) mbar_inval(sc.gbar);
      __syncthreads();
    }
    mark(1);
    // ---- stack push: B chain, UDV factorisation, cumulative V^T ----
    // X = B ... B U_top D_top stays in shared memory for the factorisation
    bchain_body(ch, dir, b, true, smem, reinterpret_cast<int8_t*>(smem + bchain_doubles(N)), true);
    __syncthreads();
    mark(2);
    udt_body<2>(ch, side, b, true, smem, mv, true);
    __syncthreads();
    mark(3);
    const HqGemmJob* const* L = lists + ((size_t)dir * nstab_max + b) * 5;
    // the push product and the equal-time G builder (src/dqmc_core.cpp:204-215 / :265-276):
    // products PH_PUSH, B1, B2, the inverse, products B3, B4; each product's job is staged in
    // shared memory (one call site of the GEMM)
    for (int ph = 0; ph < 5; ++ph) {
      if (ph == 3) {
        invert_body<2>(ch, 0, true, smem, pv);
        __syncthreads();
        mark(6);
      }
      if (threadIdx.x == 0) job = L[ph][c];
      __syncthreads();
      gemm_cta(job, smem, red);
      if (ph == 0) mark(4);
      if (ph == 2) mark(5);
    }
    mark(7);
    if (flags & (HQ_F_MEASURE | HQ_F_SNAPSHOT)) measure_body(ch, dir, b, flags, red);
    // ---- publish: interval b of chain c is complete ----
    __syncthreads();
    mark(8);
    if (threadIdx.x == 0) {
      __threadfence();
      st_release(ctl + 3 + c, b + 1);
    }
  }
}

size_t sweep_ctl_ints(int nchains) { return 3 + 2 * (size_t)nchains; }

// dynamic shared memory of k_sweep for chains of up to Nmax sites and delay depth kmax
size_t smem_sweep_bytes(int Nmax, int kmax) {
  size_t d = ((interval_smem_doubles(Nmax, kmax, true) + 1) & ~size_t(1)) * sizeof(double) + kIntervalScratchBytes;
  d = std::max(d, bchain_doubles(Nmax) * sizeof(double) + HQ_MAX_N);
  d = std::max(d, smem_udt_bytes(Nmax, true));
  d = std::max(d, smem_invert_bytes(Nmax, true));
  d = std::max(d, cta_gemm_doubles(Nmax, Nmax) * sizeof(double));
  return d;
}

// whether k_sweep can run chains of up to Nmax sites with delay depth kmax on this device
// (per-block opt-in shared memory optin) and whether its CTA can take one item of each such chain
bool sweep_fits(int Nmax, int kmax, size_t optin) {
  cudaFuncAttributes a;
  if (cudaFuncGetAttributes(&a, (const void*)k_sweep) != cudaSuccess) return false;
  return Nmax <= 160 && a.sharedSizeBytes + smem_sweep_bytes(Nmax, kmax) <= optin;
}

cudaError_t prepare_sweep(int Nmax, int kmax) {
  return cudaFuncSetAttribute((const void*)k_sweep, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smem_sweep_bytes(Nmax, kmax));
}

cudaError_t launch_sweep(const HqChain* chains, int nchains, const int2* cinfo, int nitems,
                         const HqGemmJob* const* lists, int nstab_max, int dir, int flags, int* ctl,
                         unsigned long long* clk, int grid, int Nmax, int kmax, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(ctl, 0, sweep_ctl_ints(nchains) * sizeof(int), st);
  if (e != cudaSuccess) return e;
  if (nitems <= 0) return cudaSuccess;
  k_sweep<<<std::min(grid, nitems), HQ_INT_THREADS, smem_sweep_bytes(Nmax, kmax), st>>>(
      chains, nchains, cinfo, nitems, lists, nstab_max, dir, flags, ctl, clk);
  return cudaGetLastError();
}
const void* fn_sweep() { return (const void*)k_sweep; }

}  // namespace hq
