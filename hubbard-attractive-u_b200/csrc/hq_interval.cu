// hq_interval.cu -- k_interval, the per-chain kernel of one stabilisation interval (the body is
// interval_body of hq_interval.cuh): one CTA per chain, G resident in shared memory.
#include "hq_interval.cuh"

namespace hq {

// ---------------------------------------------------------------------------------
//  k_interval: the update (or no-update) slices of one stabilisation interval.
// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(HQ_INT_THREADS, 1)
k_interval(const HqChain* __restrict__ chains, int nchains, int dir, int b, int flags, int resident) {
  extern __shared__ __align__(16) double smem[];
  __shared__ HqChain ch;
  __shared__ __align__(16) unsigned char scratch[kIntervalScratchBytes];
  const IntervalScratch sc = interval_scratch_at(scratch);
  const int c = blockIdx.x;
  if (c >= nchains) return;
  if (threadIdx.x == 0) {
    ch = chains[c];
    mbar_init(sc.gbar, 1);
  }
  __syncthreads();
  if (!ch.active || b >= ch.n_stab) return;
  interval_body(ch, dir, b, flags, resident != 0, smem, sc, 0u);
}

cudaError_t launch_interval(const HqChain* chains, int n, int dir, int b, int flags, int Nmax, int kmax, bool resident,
                            cudaStream_t st) {
  const size_t bytes = smem_interval_bytes(Nmax, kmax, resident);
  k_interval<<<n, HQ_INT_THREADS, bytes, st>>>(chains, n, dir, b, flags, resident ? 1 : 0);
  return cudaGetLastError();
}
const void* fn_interval() { return (const void*)k_interval; }

}  // namespace hq
