// hq_device.cuh -- device helpers of the sm_100a DQMC kernels:
//   * the reference's random stream (std::default_random_engine = minstd_rand0 and
//     std::bernoulli_distribution / generate_canonical<double,53> of libstdc++),
//     replayed exactly with jump-ahead so every site of a slice gets its uniform at once;
//   * FP64 tensor-core (DMMA, mma.sync m16n8k4 .f64) fragment helpers;
//   * exp(-dt K) application: dense (DMMA) and separable (A (x) A circulant) forms;
//   * block reductions.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "hq_types.h"

namespace hq {

// ------------------------------------------------------------------------------------
//  minstd_rand0: x <- 16807 x mod (2^31 - 1)   (libstdc++ default_random_engine,
//  src/random.cpp:14). generate_canonical<double, 53> draws two values:
//     sum = (x1 - 1) + (x2 - 1) * R ;  ret = sum / round(R*R) ;  R = 2147483646
//  with plain IEEE double operations (no contraction), clamped below 1.
// ------------------------------------------------------------------------------------
constexpr uint32_t kMinstdA = 16807u;
constexpr uint32_t kMinstdM = 2147483647u;

// a * x mod m for a, x < m = 2^31 - 1, exactly, without a division: with t = a x =
// hi 2^31 + lo and 2^31 = 1 (mod m), t = lo + hi (mod m); two folds leave a value <= m + 1
__host__ __device__ inline uint32_t minstd_mulmod(uint64_t a, uint64_t x) {
  const uint64_t t = a * x;
  uint64_t r = (t & kMinstdM) + (t >> 31);
  r = (r & kMinstdM) + (r >> 31);
  return static_cast<uint32_t>(r >= kMinstdM ? r - kMinstdM : r);
}
// a^k mod m
__host__ __device__ inline uint32_t minstd_pow(uint64_t k) {
  uint64_t result = 1, base = kMinstdA;
  while (k) {
    if (k & 1) result = minstd_mulmod(result, base);
    base = minstd_mulmod(base, base);
    k >>= 1;
  }
  return static_cast<uint32_t>(result);
}

__device__ inline double canonical_from_pair(uint32_t x1, uint32_t x2) {
  const double R = 2147483646.0;
  const double RR = __dmul_rn(R, R);
  const double sum = __dadd_rn((double)(x1 - 1u), __dmul_rn((double)(x2 - 1u), R));
  double r = __ddiv_rn(sum, RR);
  if (r >= 1.0) r = 0.99999999999999988898;  // nextafter(1.0, 0.0)
  return r;
}

// ------------------------------------------------------------------------------------
//  DMMA m16n8k4 (FP64). Fragment ownership (lane = 4*g + q):
//    A (16x4, row): a0 = A[g][q], a1 = A[g+8][q]
//    B (4x8,  col): b0 = B[q][g]
//    C (16x8)     : c0 = C[g][2q], c1 = C[g][2q+1], c2 = C[g+8][2q], c3 = C[g+8][2q+1]
// ------------------------------------------------------------------------------------
__device__ __forceinline__ void dmma_16x8x4(double (&c)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

// ------------------------------------------------------------------------------------
//  Reductions
// ------------------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
// block-wide sum; red must hold >= 32 doubles; result valid in all threads
__device__ inline double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = (lane < nw) ? red[lane] : 0.0;
  t = warp_sum(t);
  return t;
}
__device__ inline double block_max(double v, double* red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = (lane < nw) ? red[lane] : -INFINITY;
  t = warp_max(t);
  return t;
}

// three block-wide sums in one reduction round (2 barriers)
__device__ inline void block_sum3(double& a, double& b, double& c, double* red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  a = warp_sum(a); b = warp_sum(b); c = warp_sum(c);
  __syncthreads();
  if (lane == 0) { red[w] = a; red[32 + w] = b; red[64 + w] = c; }
  __syncthreads();
  a = warp_sum(lane < nw ? red[lane] : 0.0);
  b = warp_sum(lane < nw ? red[32 + lane] : 0.0);
  c = warp_sum(lane < nw ? red[64 + lane] : 0.0);
}

// adds one slice's equal-time estimators to acc from this thread's partial sums of
// tr = sum_i G_ii, dd = sum_i (1 - G_ii)^2 and sq = sum_ij G_ij^2 (include/observable_methods.hpp:39-83)
__device__ inline void measure_commit(double tr, double dd, double sq, int N, double* acc, double* red) {
  block_sum3(tr, dd, sq, red);
  if (threadIdx.x == 0) {
    acc[HQ_ACC_FILLING] += 2.0 - 2.0 * tr / N;
    acc[HQ_ACC_DOCC] += dd / N;
    acc[HQ_ACC_SWAVE] += (2.0 * sq - 2.0 * tr + N) / N;
    acc[HQ_ACC_NSLICE] += 1.0;
  }
}

// Element loops over an N x N column-major matrix without integer division: warps walk
// the columns, lanes the rows (consecutive lanes touch consecutive addresses).
#define HQ_FOR_EACH_ELEM(N, i, j)                                                      \
  for (int j = (int)(threadIdx.x >> 5); j < (N); j += (int)(blockDim.x >> 5))          \
    for (int i = (int)(threadIdx.x & 31); i < (N); i += 32)

// atomic max on doubles (ordered-int trick; values may be negative)
__device__ inline void atomic_max_double(double* addr, double val) {
  unsigned long long* p = reinterpret_cast<unsigned long long*>(addr);
  unsigned long long old = *p, assumed;
  do {
    assumed = old;
    if (__longlong_as_double(assumed) >= val) return;
    old = atomicCAS(p, assumed, __double_as_longlong(val));
  } while (old != assumed);
}

// ------------------------------------------------------------------------------------
//  Separable exp(-dt K): for the uniform NN hopping on the L x L torus,
//    exp(-dt K) = exp(dt mu) * A (x) A,   A = exp(dt t H_1d) circulant, A[x][x'] = a[(x-x') mod L],
//  with site index i = x + L y (src/square_lattice.cpp:30-61). Applied to a matrix M with
//  leading dimension ld in two in-place passes of length-L circular convolutions.
//  side 0: M <- c (A(x)A) M  (rows);  side 1: M <- c M (A(x)A)  (columns).
//  rows/cols outside [0, N) are untouched. All threads of the block participate.
// ------------------------------------------------------------------------------------
// SC selects an optional diagonal scaling fused into the pass: element (i, j) is multiplied by
// (s[i] > 0 ? rp : rm) * (s[j] > 0 ? cp : cm), on load (SC = 1, before the convolution) or
// on store (SC = 2); SC = 0 leaves the pass unscaled
// MEAS = 1 / 2 also accumulates the equal-time estimator sums of the matrix as loaded /
// as stored (mtr, mdd, msq; see measure_commit)
template <int L, int SC, int MEAS = 0>
__device__ __forceinline__ void sep_pass(double* M, int ld, int N, const double* __restrict__ coef, double c, int side,
                                int pass, const int8_t* sf, double rp, double rm, double cp, double cm,
                                double& mtr, double& mdd, double& msq) {
  // circulant coefficients in registers (compile-time indices after unrolling)
  double a[L];
#pragma unroll
  for (int d = 0; d < L; ++d) a[d] = coef[d];
  const int nfib = N * L;  // N lines (columns for side 0, rows for side 1) x L fibers each
  for (int f = threadIdx.x; f < nfib; f += blockDim.x) {
    const int line = f % N;   // column j (side 0) or row i (side 1)
    const int o = f / N;      // the fixed lattice coordinate of the fiber
    // pass 0 runs over x with y = o (sites L*o + e); pass 1 over y with x = o (sites o + L*e)
    const int base_site = (pass == 0) ? (L * o) : o;
    const int step_site = (pass == 0) ? 1 : L;
    double* base = (side == 0) ? (M + base_site + (size_t)line * ld) : (M + line + (size_t)base_site * ld);
    const size_t stride = (side == 0) ? (size_t)step_site : (size_t)step_site * ld;
    // the factor of element e is (row factor) * (column factor); side 0: the line is column
    // j and the site row i; side 1: the line is row i and the site column j
    double lf = 1.0, sp = 1.0, sm = 1.0;
    if (SC) {
      const bool lpos = sf[line] > 0;
      lf = (side == 0) ? (lpos ? cp : cm) : (lpos ? rp : rm);
      sp = (side == 0) ? rp : cp;
      sm = (side == 0) ? rm : cm;
    }
    double v[L];
#pragma unroll
    for (int e = 0; e < L; ++e) {
      v[e] = base[e * stride];
      if (MEAS == 1) {
        msq = fma(v[e], v[e], msq);
        if (base_site + e * step_site == line) { mtr += v[e]; mdd += (1.0 - v[e]) * (1.0 - v[e]); }
      }
      if (SC == 1) {
        const double sfac = sf[base_site + e * step_site] > 0 ? sp : sm;
        v[e] *= (side == 0) ? sfac * lf : lf * sfac;
      }
    }
    // L independent accumulators, each summed over e2 in ascending order
    double acc[L];
#pragma unroll
    for (int e = 0; e < L; ++e) acc[e] = 0.0;
#pragma unroll
    for (int e2 = 0; e2 < L; ++e2) {
#pragma unroll
      for (int e = 0; e < L; ++e) acc[e] = fma(a[(e - e2 + L) % L], v[e2], acc[e]);
    }
#pragma unroll
    for (int e = 0; e < L; ++e) {
      double out = (pass == 1) ? acc[e] * c : acc[e];
      if (SC == 2) {
        const double sfac = sf[base_site + e * step_site] > 0 ? sp : sm;
        out *= (side == 0) ? sfac * lf : lf * sfac;
      }
      if (MEAS == 2) {
        msq = fma(out, out, msq);
        if (base_site + e * step_site == line) { mtr += out; mdd += (1.0 - out) * (1.0 - out); }
      }
      base[e * stride] = out;
    }
  }
}

// both passes of one side; SC0 / SC1 select the fused scaling of pass 0 / pass 1, M0 / M1
// the fused estimators of pass 0 / pass 1 (added to acc_meas)
template <int L, int SC0 = 0, int SC1 = 0, int M0 = 0, int M1 = 0>
__device__ __forceinline__ void sep_apply(double* M, int ld, int N, const double* a, double c, int side,
                                 const int8_t* sf = nullptr, double rp = 1.0, double rm = 1.0, double cp = 1.0,
                                 double cm = 1.0, double* acc_meas = nullptr, double* red = nullptr) {
  double mtr = 0.0, mdd = 0.0, msq = 0.0;
  sep_pass<L, SC0, M0>(M, ld, N, a, c, side, 0, sf, rp, rm, cp, cm, mtr, mdd, msq);
  __syncthreads();
  sep_pass<L, SC1, M1>(M, ld, N, a, c, side, 1, sf, rp, rm, cp, cm, mtr, mdd, msq);
  __syncthreads();
  if (M0 || M1) measure_commit(mtr, mdd, msq, N, acc_meas, red);
}

// dispatch on the lattice size to an exact compile-time fiber length (L <= HQ_MAX_L)
template <int SC0 = 0, int SC1 = 0, int M0 = 0, int M1 = 0>
__device__ __forceinline__ void sep_apply_any(double* M, int ld, int N, int L, const double* a, double c, int side,
                                     const int8_t* sf = nullptr, double rp = 1.0, double rm = 1.0,
                                     double cp = 1.0, double cm = 1.0, double* acc_meas = nullptr,
                                     double* red = nullptr) {
  switch (L) {
#define HQ_SEP_CASE(n) \
  case n: sep_apply<n, SC0, SC1, M0, M1>(M, ld, N, a, c, side, sf, rp, rm, cp, cm, acc_meas, red); break;
    HQ_SEP_CASE(1) HQ_SEP_CASE(2) HQ_SEP_CASE(3) HQ_SEP_CASE(4) HQ_SEP_CASE(5) HQ_SEP_CASE(6)
    HQ_SEP_CASE(7) HQ_SEP_CASE(8) HQ_SEP_CASE(9) HQ_SEP_CASE(10) HQ_SEP_CASE(11) HQ_SEP_CASE(12)
    HQ_SEP_CASE(13) HQ_SEP_CASE(14) HQ_SEP_CASE(15)
#undef HQ_SEP_CASE
    default: sep_apply<16, SC0, SC1, M0, M1>(M, ld, N, a, c, side, sf, rp, rm, cp, cm, acc_meas, red); break;
  }
}

// ------------------------------------------------------------------------------------
//  Dense exp(-dt K) application with DMMA, M in shared (or global) memory, E in global
//  (L2-resident: shared by every chain of the same parameters).
//  dense_apply:       M <- E M, by column blocks (E M[:, blk] needs only blk)
//  dense_apply_right: M <- M E, by row blocks    (M[blk, :] E needs only blk)
//  E is symmetric here (K real symmetric), so op(E) = E in both cases.
//  stage: shared scratch of >= 2 * (N16 * 8) doubles used to stage k-chunks of E.
//  The output of a block is accumulated in registers (<= kMaxFrag fragments per warp).
// ------------------------------------------------------------------------------------
constexpr int kMaxFrag = 8;

__device__ inline void dense_apply(double* M, int ld, int N, const double* __restrict__ E, double* stage) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int N16 = (N + 15) & ~15;       // padded row count
  const int mt = N16 / 16;              // 16-row tiles
  const int max_tiles = kMaxFrag * nwarps;
  int cb8 = max_tiles / mt;             // 8-wide column tiles per block
  if (cb8 < 1) cb8 = 1;
  const int nt8 = (N + 7) / 8;
  if (cb8 > nt8) cb8 = nt8;
  const int CB = cb8 * 8;
  const int lds = N16 + 4;              // stage leading dimension
  for (int c0 = 0; c0 < N; c0 += CB) {
    const int tiles = mt * cb8;
    double acc[kMaxFrag][4];
#pragma unroll
    for (int f = 0; f < kMaxFrag; ++f) acc[f][0] = acc[f][1] = acc[f][2] = acc[f][3] = 0.0;
    for (int k0 = 0; k0 < N; k0 += 8) {
      // stage[kk * lds + r] = E[r, k0 + kk]
      __syncthreads();
      for (int kk = threadIdx.x >> 5; kk < 8; kk += blockDim.x >> 5)
        for (int r = threadIdx.x & 31; r < N16; r += 32) {
          const int k = k0 + kk;
          stage[kk * lds + r] = (r < N && k < N) ? E[r + (size_t)k * N] : 0.0;
        }
      __syncthreads();
#pragma unroll
      for (int f = 0; f < kMaxFrag; ++f) {
        const int tile = warp + f * nwarps;
        if (tile < tiles) {
          const int tm = tile % mt, tn = tile / mt;
          const int r = tm * 16 + g;
          const int cc = c0 + tn * 8 + g;
#pragma unroll
          for (int ks = 0; ks < 8; ks += 4) {
            const int k = k0 + ks + q;
            const double a0 = stage[(ks + q) * lds + r];
            const double a1 = stage[(ks + q) * lds + r + 8];
            const double b0 = (k < N && cc < N) ? M[k + (size_t)cc * ld] : 0.0;
            dmma_16x8x4(acc[f], a0, a1, b0);
          }
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int f = 0; f < kMaxFrag; ++f) {
      const int tile = warp + f * nwarps;
      if (tile < tiles) {
        const int tm = tile % mt, tn = tile / mt;
        const int r = tm * 16 + g, c = c0 + tn * 8 + 2 * q;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int rr = r + ((e & 2) ? 8 : 0), cc = c + (e & 1);
          if (rr < N && cc < N && cc < c0 + CB) M[rr + (size_t)cc * ld] = acc[f][e];
        }
      }
    }
    __syncthreads();
  }
}

// side-1 dense application uses row blocks of height CB where the tiles enumerate
// (8-col tiles over all N) x (16-row tiles inside the block); keep the block height a
// multiple of 16 and the tile count within kMaxFrag * nwarps.
__device__ inline void dense_apply_right(double* M, int ld, int N, const double* __restrict__ E, double* stage) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int N8 = (N + 7) & ~7;
  const int nt8 = N8 / 8;                // 8-col tiles over all columns
  const int max_tiles = kMaxFrag * nwarps;
  int rb16 = max_tiles / nt8;            // 16-row tiles per block
  if (rb16 < 1) rb16 = 1;
  const int mt16 = (N + 15) / 16;
  if (rb16 > mt16) rb16 = mt16;
  const int RB = rb16 * 16;
  const int lds = N8 + 4;
  for (int r0 = 0; r0 < N; r0 += RB) {
    const int tiles = nt8 * rb16;
    double acc[kMaxFrag][4];
#pragma unroll
    for (int f = 0; f < kMaxFrag; ++f) acc[f][0] = acc[f][1] = acc[f][2] = acc[f][3] = 0.0;
    for (int k0 = 0; k0 < N; k0 += 8) {
      __syncthreads();
      // stage[kk * lds + c] = E[k0+kk, c]
      for (int kk = threadIdx.x >> 5; kk < 8; kk += blockDim.x >> 5)
        for (int c = threadIdx.x & 31; c < N8; c += 32) {
          const int k = k0 + kk;
          stage[kk * lds + c] = (c < N && k < N) ? E[k + (size_t)c * N] : 0.0;
        }
      __syncthreads();
#pragma unroll
      for (int f = 0; f < kMaxFrag; ++f) {
        const int tile = warp + f * nwarps;
        if (tile < tiles) {
          const int tc = tile % nt8, tr = tile / nt8;
#pragma unroll
          for (int ks = 0; ks < 8; ks += 4) {
            const int k = k0 + ks + q;
            const int r = r0 + tr * 16 + g;
            const double a0 = (r < N && k < N) ? M[r + (size_t)k * ld] : 0.0;
            const double a1 = (r + 8 < N && k < N) ? M[r + 8 + (size_t)k * ld] : 0.0;
            const double b0 = stage[(ks + q) * lds + tc * 8 + g];
            dmma_16x8x4(acc[f], a0, a1, b0);
          }
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int f = 0; f < kMaxFrag; ++f) {
      const int tile = warp + f * nwarps;
      if (tile < tiles) {
        const int tc = tile % nt8, tr = tile / nt8;
        const int r = r0 + tr * 16 + g, c = tc * 8 + 2 * q;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int rr = r + ((e & 2) ? 8 : 0), cc = c + (e & 1);
          if (rr < N && cc < N && rr < r0 + RB) M[rr + (size_t)cc * ld] = acc[f][e];
        }
      }
    }
    __syncthreads();
  }
}

// M <- diag(v) M (rows) with v_i = (s_i > 0 ? vp : vm) ; fields is the slice's int8 row
__device__ inline void scale_rows(double* M, int ld, int N, const int8_t* s, double vp, double vm) {
  HQ_FOR_EACH_ELEM(N, i, j) M[i + (size_t)j * ld] *= (s[i] > 0 ? vp : vm);
}
// M <- M diag(v) (columns)
__device__ inline void scale_cols(double* M, int ld, int N, const int8_t* s, double vp, double vm) {
  HQ_FOR_EACH_ELEM(N, i, j) M[i + (size_t)j * ld] *= (s[j] > 0 ? vp : vm);
}

// M <- expK M   (side 0)  /  M <- M expK (side 1); inv selects inv_expK
__device__ inline void apply_expk(const HqChain& ch, double* M, int ld, int side, bool inv, double* stage) {
  if (ch.expk_mode == HQK_EXPK_SEPARABLE) {
#ifndef HQ_TEST_NO_SEP
    sep_apply_any(M, ld, ch.N, ch.L, inv ? ch.sep_ai : ch.sep_a, inv ? ch.sep_ci : ch.sep_c, side);
#endif
  } else {
#ifndef HQ_TEST_NO_DENSE
    const double* E = inv ? ch.inv_expK : ch.expK;
    if (side == 0) dense_apply(M, ld, ch.N, E, stage);
    else dense_apply_right(M, ld, ch.N, E, stage);
#endif
  }
}

}  // namespace hq
