// hq_invert.cu -- k_invert, the blocked Gauss-Jordan inverse of the G builders, one CTA of 16
// warps per chain (the body is invert_body of hq_invert.cuh).
#include "hq_invert.cuh"

namespace hq {

__global__ void __launch_bounds__(HQ_THREADS, 1)
k_invert(const HqChain* __restrict__ chains, int nchains, int b, int which, int resident) {
  extern __shared__ __align__(16) double smem[];
  __shared__ HqChain ch;
  __shared__ double pv[2];
  const int c = blockIdx.x;
  if (c >= nchains) return;
  if (threadIdx.x == 0) ch = chains[c];
  __syncthreads();
  if (!ch.active || b >= ch.n_stab) return;
  invert_body<1>(ch, which, resident != 0, smem, pv);
}

cudaError_t launch_invert(const HqChain* chains, int n, int b, int which, int Nmax, bool resident, cudaStream_t st) {
  const size_t bytes = smem_invert_bytes(Nmax, resident);
  k_invert<<<n, HQ_THREADS, bytes, st>>>(chains, n, b, which, resident ? 1 : 0);
  return cudaGetLastError();
}
const void* fn_invert() { return (const void*)k_invert; }

}  // namespace hq
