// hq_cta_gemm.cuh -- the one-CTA FP64 DMMA GEMM of the persistent sweep kernel: one builder or
// push product of one chain (the semantics of k_gemm) computed by the block that owns the chain.
#pragma once
#include "hq_common.cuh"

namespace hq {

// ---------------------------------------------------------------------------------
//  One-CTA GEMM of a builder job (the semantics of k_gemm: C = alpha op(A) diag(ks) op(B)
//  with row / column scalings, beta and the wrap-error epilogue). The output is cut into
//  16 x 24 blocks (three 16 x 8 DMMA tiles); warp w accumulates blocks w, w + 8, ... over
//  all of K, which streams through shared memory in chunks of 16 (cp.async, kCtaStages
//  buffers). Each output element sees the DMMA steps in increasing k, as in k_gemm, so the
//  two agree bitwise. Shared layouts (conflict-free fragment loads):
//    op(X) contiguous along k : sX[r * 20 + k]      otherwise : sX[k * ldr + r], ldr = 4 (mod 16)
// ---------------------------------------------------------------------------------
constexpr int kCtaKc = 16, kCtaLdk = 20, kCtaMaxB = 7;
#ifndef HQ_CTA_KK_UNROLL
#define HQ_CTA_KK_UNROLL 4
#endif
constexpr int kCtaKkUnroll = HQ_CTA_KK_UNROLL;

__host__ __device__ constexpr inline int cta_pad16(int x) { return (x + 15) & ~15; }
__host__ __device__ constexpr inline int cta_pad24(int x) { return ((x + 23) / 24) * 24; }
__host__ __device__ constexpr inline int cta_stage_doubles(int R) {
  return (kCtaKc * panel_ld(R) > R * kCtaLdk) ? kCtaKc * panel_ld(R) : R * kCtaLdk;
}
// chunks of K in flight: three stages hide the latency of operands that come from HBM
constexpr int kCtaStages = 3;
// doubles of shared memory of gemm_cta for M x Nc outputs: the stages of both operands, the
// k-scalings of as many chunks and the row / column scalings of the output
__host__ __device__ constexpr inline size_t cta_gemm_doubles(int M, int Nc) {
  return kCtaStages * ((size_t)cta_stage_doubles(cta_pad16(M)) + (size_t)cta_stage_doubles(cta_pad24(Nc)) + kCtaKc) +
         cta_pad16(M) + cta_pad24(Nc);
}

__device__ __forceinline__ void cta_cp16(double* dst, const double* src, int nvalid) {
  const unsigned saddr = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  const int nbytes = nvalid <= 0 ? 0 : (nvalid >= 2 ? 16 : 8);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(saddr), "l"(src), "r"(nbytes));
}

// stages rows [0, Rp) x k in [k0, k0 + 16) of op(X) by 16-byte copies (R valid rows, K valid k;
// zero fill). Copy idx moves elements (r, k), (r, k + 1) [op(X) contiguous along k: r = idx / 8]
// or (r, k), (r + 1, k) [otherwise: k = idx / (Rp / 2), by a float product with the reciprocal
// inv_half = 1 / (Rp / 2): (idx + 1/2) / (Rp / 2) lies at least 1 / Rp from an integer, far
// beyond the float's error for idx < 2^12]
template <bool KMAJ>
__device__ __forceinline__ void cta_stage16(const double* X, int ldx, int R, int Rp, int K, int k0, double* sX, int ldr,
                                            float inv_half) {
  const int half = Rp >> 1;
  const int total = KMAJ ? Rp * (kCtaKc / 2) : half * kCtaKc;
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    int r, k;
    if (KMAJ) {
      r = idx >> 3;
      k = 2 * (idx & 7);
    } else {
      k = __float2int_rz(((float)idx + 0.5f) * inv_half);
      r = 2 * (idx - k * half);
    }
    const int kk = k0 + k;
    const int nv = KMAJ ? (r < R ? min(2, K - kk) : 0) : (kk < K ? min(2, R - r) : 0);
    const size_t go = KMAJ ? kk + (size_t)r * ldx : r + (size_t)kk * ldx;
    cta_cp16(sX + (KMAJ ? r * kCtaLdk + k : k * ldr + r), nv > 0 ? X + go : X, nv);
  }
}

// stages rows [0, Rp) x k in [k0, k0 + 16) of op(X) by 8-byte copies (R valid rows, K valid k;
// zero fill): operands whose columns are not 16-byte aligned
__device__ __forceinline__ void cta_stage8(const double* X, int ldx, bool kmaj, int R, int Rp, int K, int k0, double* sX,
                                           int ldr) {
  for (int idx = threadIdx.x; idx < Rp * kCtaKc; idx += blockDim.x) {
    int r, k;
    if (kmaj) { r = idx / kCtaKc; k = idx % kCtaKc; } else { r = idx % Rp; k = idx / Rp; }
    const bool ok = k0 + k < K && r < R;
    const double* src = ok ? (kmaj ? X + (k0 + k) + (size_t)r * ldx : X + r + (size_t)(k0 + k) * ldx) : X;
    cp_async_8(kmaj ? sX + r * kCtaLdk + k : sX + k * ldr + r, src, ok);
  }
}

// C of job `job` for one transpose case (AMAJ: op(A) = A^T, contiguous along k; BMAJ: op(B) = B,
// contiguous along k; KS: k-scalings). Inlined by default (HQ_CTA_NOINLINE=1 makes it a call):
// measured 5-15% faster per product. `smem` holds cta_gemm_doubles(M, Nc) doubles, red >= 32
// doubles. Every thread calls it.
#ifndef HQ_CTA_NOINLINE
#define HQ_CTA_NOINLINE 0
#endif
#if HQ_CTA_NOINLINE
#define HQ_CTA_FN_ATTR __noinline__
#else
#define HQ_CTA_FN_ATTR __forceinline__
#endif
template <bool AMAJ, bool BMAJ, bool KS>
__device__ HQ_CTA_FN_ATTR void gemm_cta_t(const HqGemmJob& job, double* smem, double* red) {
  const double* __restrict__ Ag = job.A;
  const double* __restrict__ Bg = job.B;
  double* Cg = job.C;
  const double* ks = job.ks;
  const double* rs = job.rs;
  const double* cs = job.cs;
  const int M = job.M, Nc = job.Nc, K = job.K, lda = job.lda, ldb = job.ldb, ldc = job.ldc;
  const int ks_mode = job.ks_mode, rs_mode = job.rs_mode, cs_mode = job.cs_mode, epi = job.epi;
  const double alpha = job.alpha, beta = job.beta;
  double* err_out = job.err_out;
  const int Mp = cta_pad16(M), Np = cta_pad24(Nc);
  const int ldA = panel_ld(Mp), ldB = panel_ld(Np);
  const int SA = cta_stage_doubles(Mp), SB = cta_stage_doubles(Np);
  double* sA0 = smem;
  double* sB0 = smem + kCtaStages * (size_t)SA;
  double* sK0 = sB0 + kCtaStages * (size_t)SB;
  double* sR = sK0 + kCtaStages * kCtaKc;  // row scalings of the output
  double* sC = sR + Mp;           // column scalings
  const bool pa = (lda % 2 == 0) && ((reinterpret_cast<uintptr_t>(Ag) & 15) == 0);
  const bool pb = (ldb % 2 == 0) && ((reinterpret_cast<uintptr_t>(Bg) & 15) == 0);
  const float ihA = 2.0f / (float)Mp, ihB = 2.0f / (float)Np;
  auto stage = [&](int k0, int buf) {
    if (pa) cta_stage16<AMAJ>(Ag, lda, M, Mp, K, k0, sA0 + buf * (size_t)SA, ldA, ihA);
    else cta_stage8(Ag, lda, AMAJ, M, Mp, K, k0, sA0 + buf * (size_t)SA, ldA);
    if (pb) cta_stage16<BMAJ>(Bg, ldb, Nc, Np, K, k0, sB0 + buf * (size_t)SB, ldB, ihB);
    else cta_stage8(Bg, ldb, BMAJ, Nc, Np, K, k0, sB0 + buf * (size_t)SB, ldB);
  };
  for (int i = threadIdx.x; i < Mp; i += blockDim.x) sR[i] = i < M ? vscale(rs, rs_mode, i) : 0.0;
  for (int i = threadIdx.x; i < Np; i += blockDim.x) sC[i] = i < Nc ? vscale(cs, cs_mode, i) : 0.0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int mb = Mp / 16, nblk = mb * (Np / 24);
  const int nchunks = (K + kCtaKc - 1) / kCtaKc;
  const bool load_old = (beta != 0.0 || epi == 1);
  double emax = -INFINITY;
  for (int base = 0; base < nblk; base += nw * kCtaMaxB) {
    // the warp's blocks: first row (+ g) and first column of each (rows of blocks >= nblk are -1)
    int mrow[kCtaMaxB], ncol[kCtaMaxB];
#pragma unroll
    for (int i = 0; i < kCtaMaxB; ++i) {
      const int blk = base + warp + i * nw;
      mrow[i] = blk < nblk ? (blk % mb) * 16 + g : -1;
      ncol[i] = blk < nblk ? (blk / mb) * 24 : 0;
    }
    double acc[kCtaMaxB][3][4];
#pragma unroll
    for (int i = 0; i < kCtaMaxB; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) acc[i][j][0] = acc[i][j][1] = acc[i][j][2] = acc[i][j][3] = 0.0;
    __syncthreads();  // the stage buffers are free
    // chunk c lives in stage c mod kCtaStages; chunks c + 1 .. c + kCtaStages - 1 are in flight
    // while chunk c is multiplied
    auto stage_chunk = [&](int cc) {
      if (cc < nchunks) {
        const int k1 = cc * kCtaKc, buf = cc % kCtaStages;
        stage(k1, buf);
        if (threadIdx.x < kCtaKc)
          sK0[buf * kCtaKc + threadIdx.x] = (k1 + (int)threadIdx.x < K) ? vscale(ks, ks_mode, k1 + threadIdx.x) : 0.0;
      }
      cp_async_commit();
    };
#pragma unroll
    for (int cc = 0; cc < kCtaStages - 1; ++cc) stage_chunk(cc);
    for (int c = 0; c < nchunks; ++c) {
      const int cur = c % kCtaStages;
      stage_chunk(c + kCtaStages - 1);
      cp_async_wait<kCtaStages - 1>();
      __syncthreads();
      const double* A_ = sA0 + cur * (size_t)SA;
      const double* B_ = sB0 + cur * (size_t)SB;
      const double* K_ = sK0 + cur * kCtaKc;
#pragma unroll kCtaKkUnroll
      for (int kk = 0; kk < kCtaKc; kk += 4) {
        const int k = kk + q;
        const double ksc = KS ? K_[k] : 1.0;
#pragma unroll
        for (int i = 0; i < kCtaMaxB; ++i) {
          if (mrow[i] >= 0) {
            const int m = mrow[i];
            // without k-scalings (KS false) the factor is 1: the product is the value itself
            const double a0v = AMAJ ? A_[m * kCtaLdk + k] : A_[k * ldA + m];
            const double a1v = AMAJ ? A_[(m + 8) * kCtaLdk + k] : A_[k * ldA + m + 8];
            const double a0 = KS ? a0v * ksc : a0v;
            const double a1 = KS ? a1v * ksc : a1v;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
              const int n = ncol[i] + j * 8 + g;
              const double b0 = BMAJ ? B_[n * kCtaLdk + k] : B_[k * ldB + n];
              dmma_16x8x4(acc[i][j], a0, a1, b0);
            }
          }
        }
      }
      __syncthreads();
    }
    cp_async_wait<0>();
    // epilogue: alpha, row / column scalings, beta, wrap-error maximum (as k_gemm); per block the
    // old values are loaded before any of its stores, so that their latencies overlap
#pragma unroll
    for (int i = 0; i < kCtaMaxB; ++i) {
      if (mrow[i] >= 0) {
        const int m0 = mrow[i] - g, n0 = ncol[i];
        double old[3][4];
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int gm = m0 + g + ((e & 2) ? 8 : 0);
            const int gn = n0 + j * 8 + 2 * q + (e & 1);
            old[j][e] = (load_old && gm < M && gn < Nc) ? Cg[gm + (size_t)gn * ldc] : 0.0;
          }
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int gm = m0 + g + ((e & 2) ? 8 : 0);
            const int gn = n0 + j * 8 + 2 * q + (e & 1);
            if (gm < M && gn < Nc) {
              double v = alpha * acc[i][j][e] * sR[gm] * sC[gn];
              if (beta != 0.0) v = fma(beta, old[j][e], v);
              if (epi == 1) emax = fmax(emax, v - old[j][e]);
              Cg[gm + (size_t)gn * ldc] = v;
            }
          }
      }
    }
  }
  if (epi == 1 && err_out) {
    emax = block_max(emax, red);
    if (threadIdx.x == 0) atomic_max_double(err_out, emax);
  }
  __syncthreads();
}

// C of job `job` by the whole block (the transpose cases of the builders and the push, with or
// without k-scalings)
template <bool AMAJ, bool BMAJ>
__device__ __forceinline__ void gemm_cta_ks(const HqGemmJob& job, double* smem, double* red) {
  if (job.ks_mode != 0) gemm_cta_t<AMAJ, BMAJ, true>(job, smem, red);
  else gemm_cta_t<AMAJ, BMAJ, false>(job, smem, red);
}
__device__ __forceinline__ void gemm_cta(const HqGemmJob& job, double* smem, double* red) {
  if (!job.active) return;
  if (job.ta) {
    if (job.tb == 0) gemm_cta_ks<true, true>(job, smem, red);
    else gemm_cta_ks<true, false>(job, smem, red);
  } else {
    if (job.tb == 0) gemm_cta_ks<false, true>(job, smem, red);
    else gemm_cta_ks<false, false>(job, smem, red);
  }
}

}  // namespace hq
