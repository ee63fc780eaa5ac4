// hq_udt.cu -- k_udt, the UDV factorisation of a stack push, one CTA of 16 warps per chain (the
// body is udt_body of hq_udt.cuh).
#include "hq_udt.cuh"

namespace hq {

__global__ void __launch_bounds__(HQ_THREADS, 1)
k_udt(const HqChain* __restrict__ chains, int nchains, int side, int unused, int b, int resident) {
  extern __shared__ __align__(16) double smem[];
  __shared__ HqChain ch;
  __shared__ PivotMoves mv;
  const int c = blockIdx.x;
  if (c >= nchains) return;
  if (threadIdx.x == 0) ch = chains[c];
  __syncthreads();
  if (!ch.active || b >= ch.n_stab) return;
  udt_body<1>(ch, side, b, resident != 0, smem, mv);
}

cudaError_t launch_udt(const HqChain* chains, int n, int side, int b, int Nmax, bool resident, cudaStream_t st) {
  const size_t bytes = smem_udt_bytes(Nmax, resident);
  k_udt<<<n, HQ_THREADS, bytes, st>>>(chains, n, side, 0, b, resident ? 1 : 0);
  return cudaGetLastError();
}
const void* fn_udt() { return (const void*)k_udt; }

}  // namespace hq
