// hq_gemm.cu -- k_gemm, the batched FP64 DMMA GEMM of the G builders
// (include/utils/stable_numerics.hpp:186-324) with the wrap-error epilogue (:37-48).
#include "hq_common.cuh"

namespace hq {

// ---------------------------------------------------------------------------------
//  k_gemm: batched C = alpha op(A) diag(ks) op(B) (row / column scalings, beta, wrap-error
//  epilogue), one CTA per 48 x 48 tile of one job (144 = 3 x 48: no padding for the 12 x 12
//  lattice). Six warps own 16 x 24 blocks (3 DMMA tiles each); K streams through shared
//  memory in chunks of 16 with cp.async double buffering. Shared layouts keep the fragment
//  loads free of bank conflicts for either transpose:
//    op(A) = A   : sA[k * kGLdm + m]     op(A) = A^T : sA[m * kGLdk + k]
//    op(B) = B   : sB[n * kGLdk + k]     op(B) = B^T : sB[k * kGLdm + n]
// ---------------------------------------------------------------------------------
constexpr int kGT = 48, kGKc = 16, kGLdm = 52, kGLdk = 20, kGWarps = 6;
constexpr int kGStage = (kGLdm * kGKc > kGT * kGLdk) ? kGLdm * kGKc : kGT * kGLdk;  // doubles

// copies 2 doubles (16 B) with zero fill of the invalid part; both addresses 16-byte aligned
__device__ __forceinline__ void cp_async_16(double* dst, const double* src, int nvalid) {
  const unsigned saddr = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  const int nbytes = nvalid <= 0 ? 0 : (nvalid >= 2 ? 16 : 8);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(saddr), "l"(src), "r"(nbytes));
}

// stages the chunk [k0, k0 + 16) x [r0, r0 + 48) of op(X) (r = m for A, n for B; R rows).
// kmaj: op(X) is contiguous along k in memory (A^T or B) -> layout [r][k]; otherwise
// contiguous along r -> layout [k][r]. `pair` selects 16-byte copies (even ld, aligned base).
__device__ __forceinline__ void g_stage(const double* X, int ldx, bool kmaj, int R, int K, int r0, int k0,
                                        double* sX, bool pair) {
  if (pair) {
    if (kmaj) {
      for (int idx = threadIdx.x; idx < kGT * (kGKc / 2); idx += blockDim.x) {
        const int r = idx / (kGKc / 2), k = 2 * (idx % (kGKc / 2));
        const int nv = (r0 + r < R) ? min(2, K - (k0 + k)) : 0;
        cp_async_16(sX + r * kGLdk + k, nv > 0 ? X + (k0 + k) + (size_t)(r0 + r) * ldx : X, nv);
      }
    } else {
      for (int idx = threadIdx.x; idx < (kGT / 2) * kGKc; idx += blockDim.x) {
        const int r = 2 * (idx % (kGT / 2)), k = idx / (kGT / 2);
        const int nv = (k0 + k < K) ? min(2, R - (r0 + r)) : 0;
        cp_async_16(sX + k * kGLdm + r, nv > 0 ? X + (r0 + r) + (size_t)(k0 + k) * ldx : X, nv);
      }
    }
  } else {
    for (int idx = threadIdx.x; idx < kGT * kGKc; idx += blockDim.x) {
      int r, k;
      if (kmaj) { r = idx / kGKc; k = idx % kGKc; } else { r = idx % kGT; k = idx / kGT; }
      const bool ok = k0 + k < K && r0 + r < R;
      const double* src = ok ? (kmaj ? X + (k0 + k) + (size_t)(r0 + r) * ldx : X + (r0 + r) + (size_t)(k0 + k) * ldx) : X;
      cp_async_8(kmaj ? sX + r * kGLdk + k : sX + k * kGLdm + r, src, ok);
    }
  }
}

__global__ void __launch_bounds__(kGWarps * 32, 4)
k_gemm(const HqGemmJob* __restrict__ jobs, int njobs, int tiles_n) {
  __shared__ __align__(16) double sA[2][kGStage];
  __shared__ __align__(16) double sB[2][kGStage];
  __shared__ double sK[2][kGKc];
  __shared__ double red[32];
  const int jb = blockIdx.y;
  if (jb >= njobs) return;
  const HqGemmJob J = jobs[jb];
  if (!J.active) return;
  const int m0 = (blockIdx.x / tiles_n) * kGT, n0 = (blockIdx.x % tiles_n) * kGT;
  if (m0 >= J.M || n0 >= J.Nc) return;
  const bool amaj = J.ta != 0;  // op(A) = A^T is contiguous along k
  const bool bmaj = J.tb == 0;  // op(B) = B is contiguous along k
  const bool pa = (J.lda % 2 == 0) && ((reinterpret_cast<uintptr_t>(J.A) & 15) == 0);
  const bool pb = (J.ldb % 2 == 0) && ((reinterpret_cast<uintptr_t>(J.B) & 15) == 0);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int wm = (warp % 3) * 16, wn = (warp / 3) * 24;
  double acc[3][4];
#pragma unroll
  for (int j = 0; j < 3; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0;
  const int nchunks = (J.K + kGKc - 1) / kGKc;
  g_stage(J.A, J.lda, amaj, J.M, J.K, m0, 0, sA[0], pa);
  g_stage(J.B, J.ldb, bmaj, J.Nc, J.K, n0, 0, sB[0], pb);
  if (threadIdx.x < kGKc) sK[0][threadIdx.x] = (threadIdx.x < J.K) ? vscale(J.ks, J.ks_mode, threadIdx.x) : 0.0;
  cp_async_commit();
  for (int c = 0; c < nchunks; ++c) {
    const int cur = c & 1;
    if (c + 1 < nchunks) {
      const int k1 = (c + 1) * kGKc;
      g_stage(J.A, J.lda, amaj, J.M, J.K, m0, k1, sA[cur ^ 1], pa);
      g_stage(J.B, J.ldb, bmaj, J.Nc, J.K, n0, k1, sB[cur ^ 1], pb);
      if (threadIdx.x < kGKc)
        sK[cur ^ 1][threadIdx.x] = (k1 + threadIdx.x < J.K) ? vscale(J.ks, J.ks_mode, k1 + threadIdx.x) : 0.0;
    }
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const double* A_ = sA[cur];
    const double* B_ = sB[cur];
#pragma unroll
    for (int kk = 0; kk < kGKc; kk += 4) {
      const int k = kk + q;
      const double ksc = sK[cur][k];
      const int m = wm + g;
      const double a0 = (amaj ? A_[m * kGLdk + k] : A_[k * kGLdm + m]) * ksc;
      const double a1 = (amaj ? A_[(m + 8) * kGLdk + k] : A_[k * kGLdm + m + 8]) * ksc;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const int n = wn + j * 8 + g;
        const double b0 = bmaj ? B_[n * kGLdk + k] : B_[k * kGLdm + n];
        dmma_16x8x4(acc[j], a0, a1, b0);
      }
    }
    __syncthreads();
  }
  cp_async_wait<0>();
  // epilogue: alpha, row / column scalings, beta, wrap-error maximum
  double emax = -INFINITY;
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int gm = m0 + wm + g + ((e & 2) ? 8 : 0);
      const int gn = n0 + wn + j * 8 + 2 * q + (e & 1);
      if (gm < J.M && gn < J.Nc) {
        double v = J.alpha * acc[j][e] * vscale(J.rs, J.rs_mode, gm) * vscale(J.cs, J.cs_mode, gn);
        double* cp = J.C + gm + (size_t)gn * J.ldc;
        const double old = (J.beta != 0.0 || J.epi == 1) ? *cp : 0.0;
        if (J.beta != 0.0) v = fma(J.beta, old, v);
        if (J.epi == 1) emax = fmax(emax, v - old);
        *cp = v;
      }
    }
  if (J.epi == 1 && J.err_out) {
    emax = block_max(emax, red);
    if (threadIdx.x == 0) atomic_max_double(J.err_out, emax);
  }
}

cudaError_t launch_gemm(const HqGemmJob* jobs, int njobs, int Mmax, int Nmax, cudaStream_t st) {
  if (njobs <= 0) return cudaSuccess;
  const int tm = (Mmax + kGT - 1) / kGT, tn = (Nmax + kGT - 1) / kGT;
  dim3 grid(tm * tn, njobs);
  k_gemm<<<grid, kGWarps * 32, 0, st>>>(jobs, njobs, tn);
  return cudaGetLastError();
}

}  // namespace hq
