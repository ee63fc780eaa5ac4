// phase_timer.cu -- clock64 phase timings of the per-chain kernel bodies on one B200, for N = 144
// (the 12 x 12 lattice): the Gauss-Jordan inverse (invert_body) and the UDV push factorisation
// (udt_body), run through the library's own bodies with a phase hook that synchronises the block
// and reads the clock; the delayed-update flush of the interval kernel (flush_block) at ranks
// 4..16; the one-CTA builder products of the persistent sweep (gemm_cta) for each job case.
// One CTA per matrix, 128 (factorisations) or 148 (flush, products) CTAs, synthetic operands.
// Build: make -C hubbard-attractive-u_b200/microbench; run: ./phase_timer (one GPU).
#include <cmath>
#include <cstdio>
#include <vector>

#include "../csrc/hq_cta_gemm.cuh"
#include "../csrc/hq_invert.cuh"
#include "../csrc/hq_metropolis.cuh"
#include "../csrc/hq_udt.cuh"

using namespace hq;

constexpr int kN = 144;
constexpr int kSlots = 8;

// phase hook: cycles since the previous mark, per phase slot (kept by thread 0)
struct ClockPhase {
  long long* t;
  long long* acc;
  __device__ void operator()(int s) const {
    __syncthreads();
    if (threadIdx.x == 0) {
      const long long now = clock64();
      acc[s] += now - *t;
      *t = now;
    }
  }
};

__device__ void flush_clocks(const long long* acc, unsigned long long* clk) {
  if (threadIdx.x == 0)
    for (int s = 0; s < kSlots; ++s) atomicAdd(clk + s, (unsigned long long)acc[s]);
}

template <int CPW, int NT>
__global__ void __launch_bounds__(NT, 1) k_invert_phases(double* mats, double* accs, unsigned long long* clk) {
  extern __shared__ __align__(16) double smem[];
  __shared__ double pv[2];
  __shared__ long long t, acc[kSlots];
  HqChain ch{};
  ch.N = kN;
  ch.W1 = mats + (size_t)blockIdx.x * kN * kN;
  ch.acc = accs + (size_t)blockIdx.x * HQ_ACC_COUNT;
  if (threadIdx.x < kSlots) acc[threadIdx.x] = 0;
  if (threadIdx.x == 0) t = clock64();
  __syncthreads();
  invert_body<CPW>(ch, 0, true, smem, pv, ClockPhase{&t, acc});
  flush_clocks(acc, clk);
}

template <int CPW, int NT>
__global__ void __launch_bounds__(NT, 1) k_udt_phases(const double* X, double* U, double* D, double* T,
                                                     unsigned long long* clk) {
  extern __shared__ __align__(16) double smem[];
  __shared__ PivotMoves mv;
  __shared__ long long t, acc[kSlots];
  const size_t NN = (size_t)kN * kN;
  HqChain ch{};
  ch.N = kN;
  ch.n_stab = 1;
  ch.X = const_cast<double*>(X) + blockIdx.x * NN;
  ch.stackU = U + blockIdx.x * NN;
  ch.stackD = D + blockIdx.x * kN;
  ch.W0 = T + blockIdx.x * NN;
  if (threadIdx.x < kSlots) acc[threadIdx.x] = 0;
  if (threadIdx.x == 0) t = clock64();
  __syncthreads();
  udt_body<CPW>(ch, 0, 0, true, smem, mv, false, ClockPhase{&t, acc});
  flush_clocks(acc, clk);
}

__global__ void __launch_bounds__(HQ_INT_THREADS, 1) k_flush(unsigned long long* clk, int k, int reps) {
  extern __shared__ __align__(16) double smem[];
  const int ld = interval_ld(kN), ldp = panel_ld(kN);
  double* G = smem;
  double* X = G + kN * ld;
  double* Y = X + ldp * 16;
  for (int i = threadIdx.x; i < kN * ld; i += blockDim.x) G[i] = 1e-3 * ((i * 37 + blockIdx.x) % 101);
  for (int i = threadIdx.x; i < ldp * 16; i += blockDim.x) {
    X[i] = 1e-3 * ((i * 13) % 17 - 8);
    Y[i] = 1e-3 * ((i * 7) % 19 - 9);
  }
  __syncthreads();
  const long long t0 = clock64();
  for (int r = 0; r < reps; ++r) {
    flush_block(G, ld, kN, X, ldp, Y, ldp, k);
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(clk, (unsigned long long)(clock64() - t0));
}

// one builder product per CTA and repetition; operands rotate over nsets sets (beyond L2)
__global__ void __launch_bounds__(HQ_INT_THREADS, 1) k_products(const double* A, const double* B, double* C, const double* dv,
                                                              int nsets, HqGemmJob tmpl, int reps,
                                                              unsigned long long* clk) {
  extern __shared__ __align__(16) double smem[];
  __shared__ double red[32];
  const size_t NN = (size_t)kN * kN;
  long long tot = 0;
  for (int r = 0; r < reps; ++r) {
    const int s = (blockIdx.x + r * gridDim.x) % nsets;
    HqGemmJob j = tmpl;
    j.A = A + s * NN;
    j.B = B + s * NN;
    j.C = C + s * NN;
    j.ks = j.rs = dv + s * kN;
    j.cs = dv + ((s + 1) % nsets) * kN;
    j.err_out = C + (size_t)nsets * NN + blockIdx.x;
    __syncthreads();
    const long long t0 = clock64();
    gemm_cta(j, smem, red);
    __syncthreads();
    tot += clock64() - t0;
  }
  if (threadIdx.x == 0) atomicAdd(clk, (unsigned long long)tot);
}

static std::vector<double> random_matrices(int n, unsigned seed) {
  std::vector<double> h((size_t)n * kN * kN);
  for (auto& v : h) {
    seed = seed * 1664525u + 1013904223u;
    v = ((seed >> 8) * (1.0 / 16777216.0)) * 2.0 - 1.0;
  }
  return h;
}

static void print_phases(const char* what, const unsigned long long* c, int nb, const char* const* names, int n) {
  double tot = 0;
  for (int i = 0; i < n; ++i) tot += (double)c[i];
  std::printf("%s: %.0f cycles per matrix\n", what, tot / nb);
  for (int i = 0; i < n; ++i)
    if (names[i]) std::printf("  %-26s %9.0f  (%4.1f%%)\n", names[i], (double)c[i] / nb, 100.0 * c[i] / tot);
}

template <int CPW, int NT>
static void time_invert(const std::vector<double>& h, double* d, double* accs, unsigned long long* clk, int nb) {
  const size_t NN = (size_t)kN * kN;
  cudaMemcpy(d, h.data(), nb * NN * 8, cudaMemcpyHostToDevice);
  cudaMemset(accs, 0, (size_t)nb * HQ_ACC_COUNT * 8);
  cudaMemset(clk, 0, kSlots * 8);
  // the dynamic shared memory of k_invert (smem_invert_bytes, resident)
  const size_t smem = ((size_t)kN * smem_ld(kN) + 2 * kGJ * panel_ld(kN) + 3 * kN + 64) * 8;
  cudaFuncSetAttribute(k_invert_phases<CPW, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_invert_phases<CPW, NT><<<nb, NT, smem>>>(d, accs, clk);
  const cudaError_t e = cudaDeviceSynchronize();
  std::vector<double> inv(NN);
  unsigned long long c[kSlots];
  cudaMemcpy(inv.data(), d, NN * 8, cudaMemcpyDeviceToHost);
  cudaMemcpy(c, clk, sizeof c, cudaMemcpyDeviceToHost);
  double res = 0.0;  // max |A A^-1 - I| of the first matrix
  for (int i = 0; i < kN; ++i)
    for (int j = 0; j < kN; ++j) {
      double s = 0.0;
      for (int k = 0; k < kN; ++k) s += h[i + (size_t)k * kN] * inv[k + (size_t)j * kN];
      res = std::fmax(res, std::fabs(s - (i == j ? 1.0 : 0.0)));
    }
  char what[160];
  std::snprintf(what, sizeof what, "inverse, %d threads, %d panel column(s) per warp (%s, max|A A^-1 - I| %.1e)", NT, CPW,
                cudaGetErrorString(e), res);
  const char* names[kSlots] = {nullptr, "panel pivots", "row interchanges, staging", "rank-16 updates",
                               "column order", "write-back", nullptr, nullptr};
  print_phases(what, c, nb, names, kSlots);
}

template <int CPW, int NT>
static void time_udt(const std::vector<double>& h, double* X, double* U, double* D, double* T, unsigned long long* clk,
                     int nb) {
  const size_t NN = (size_t)kN * kN;
  cudaMemset(clk, 0, kSlots * 8);
  // the dynamic shared memory of k_udt (smem_udt_bytes, resident)
  const size_t smem = ((size_t)kN * smem_ld(kN) + 2 * kQB * panel_ld(kN) + 2 * kQB * kQB + 3 * kN + 64 +
                       ((kN - 1) / kQB) * kQB * kQB) * 8;
  cudaFuncSetAttribute(k_udt_phases<CPW, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_udt_phases<CPW, NT><<<nb, NT, smem>>>(X, U, D, T, clk);
  const cudaError_t e = cudaDeviceSynchronize();
  std::vector<double> hu(NN), hd(kN), ht(NN);
  unsigned long long c[kSlots];
  cudaMemcpy(hu.data(), U, NN * 8, cudaMemcpyDeviceToHost);
  cudaMemcpy(hd.data(), D, kN * 8, cudaMemcpyDeviceToHost);
  cudaMemcpy(ht.data(), T, NN * 8, cudaMemcpyDeviceToHost);
  cudaMemcpy(c, clk, sizeof c, cudaMemcpyDeviceToHost);
  double res = 0.0;  // max |U D T - X| of the first matrix
  for (int i = 0; i < kN; ++i)
    for (int j = 0; j < kN; ++j) {
      double s = 0.0;
      for (int k = 0; k < kN; ++k) s += hu[i + (size_t)k * kN] * hd[k] * ht[k + (size_t)j * kN];
      res = std::fmax(res, std::fabs(s - h[i + (size_t)j * kN]));
    }
  char what[160];
  std::snprintf(what, sizeof what, "UDV push, %d threads, %d panel column(s) per warp (%s, max|U D T - X| %.1e)", NT, CPW,
                cudaGetErrorString(e), res);
  const char* names[kSlots] = {"load", "panel pivoting", "panel QR (reflectors)", "trailing WY update", "D and T out",
                               "Q: trailing WY blocks", "Q: panel columns", "U out"};
  print_phases(what, c, nb, names, kSlots);
}

int main() {
  const int nb = 128;
  const size_t NN = (size_t)kN * kN;
  const std::vector<double> hm = random_matrices(nb, 12345u);
  double *d, *accs, *X, *U, *D, *T;
  unsigned long long* clk;
  cudaMalloc(&d, nb * NN * 8);
  cudaMalloc(&accs, (size_t)nb * HQ_ACC_COUNT * 8);
  cudaMalloc(&X, nb * NN * 8);
  cudaMalloc(&U, nb * NN * 8);
  cudaMalloc(&D, nb * kN * 8);
  cudaMalloc(&T, nb * NN * 8);
  cudaMalloc(&clk, kSlots * 8);
  // the configurations of the kernels: k_invert / k_udt (16 warps), the persistent sweep (8 warps)
  time_invert<1, HQ_THREADS>(hm, d, accs, clk, nb);
  time_invert<2, HQ_INT_THREADS>(hm, d, accs, clk, nb);
  cudaMemcpy(X, hm.data(), nb * NN * 8, cudaMemcpyHostToDevice);
  time_udt<1, HQ_THREADS>(hm, X, U, D, T, clk, nb);
  time_udt<2, HQ_INT_THREADS>(hm, X, U, D, T, clk, nb);

  // the flush of one 16-site block of delayed updates at rank k
  {
    const size_t smem = ((size_t)kN * interval_ld(kN) + 2 * panel_ld(kN) * 16) * 8;
    cudaFuncSetAttribute(k_flush, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    std::printf("flush_block (G += X Y, G 144 x 144 in shared memory, 8 warps):\n");
    for (int k : {4, 8, 10, 12, 16}) {
      const int reps = 200;
      cudaMemset(clk, 0, 8);
      k_flush<<<148, HQ_INT_THREADS, smem>>>(clk, k, reps);
      const cudaError_t e = cudaDeviceSynchronize();
      unsigned long long c;
      cudaMemcpy(&c, clk, 8, cudaMemcpyDeviceToHost);
      std::printf("  rank %2d: %7.0f cycles per flush (%s)\n", k, (double)c / (148.0 * reps), cudaGetErrorString(e));
    }
  }

  // the builder and push products of the persistent sweep, one CTA each
  {
    const int nsets = 1024;  // 3 x 1024 x 166 KB: operands come from HBM, as in the sweep
    double *A, *B, *C, *dv;
    cudaMalloc(&A, nsets * NN * 8);
    cudaMalloc(&B, nsets * NN * 8);
    cudaMalloc(&C, (nsets * NN + 148) * 8);
    cudaMalloc(&dv, (size_t)nsets * kN * 8);
    const std::vector<double> ho = random_matrices(64, 99u);
    for (int s = 0; s < nsets; s += 64) {
      cudaMemcpy(A + s * NN, ho.data(), 64 * NN * 8, cudaMemcpyHostToDevice);
      cudaMemcpy(B + s * NN, ho.data(), 64 * NN * 8, cudaMemcpyHostToDevice);
    }
    cudaMemset(C, 0, (nsets * NN + 148) * 8);
    std::vector<double> hv((size_t)nsets * kN);
    for (size_t i = 0; i < hv.size(); ++i) hv[i] = 0.5 + (double)(i % 7);
    cudaMemcpy(dv, hv.data(), hv.size() * 8, cudaMemcpyHostToDevice);
    const size_t smem = cta_gemm_doubles(kN, kN) * 8;
    cudaFuncSetAttribute(k_products, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    struct Case {
      const char* name;
      int ta, tb, ks, rs, cs, epi;
      double beta;
    };
    const Case cases[] = {{"push: T Vt_prev", 0, 0, 0, 0, 0, 0, 0.0},
                          {"B1: U_L^T U_R, row/col scalings", 1, 0, 0, 2, 2, 0, 0.0},
                          {"B2: Vt_L Vt_R^T, scalings, beta 1", 0, 1, 0, 3, 3, 0, 1.0},
                          {"B3: W1 U_L^T, k-scaling", 0, 1, 2, 0, 0, 0, 0.0},
                          {"B4: U_R W2, k-scaling, wrap error", 0, 0, 2, 0, 0, 1, 0.0},
                          {"(no transpose) k-scaling only", 0, 0, 2, 0, 0, 0, 0.0},
                          {"(no transpose) wrap error only", 0, 0, 0, 0, 0, 1, 0.0}};
    std::printf("gemm_cta (one 144^3 product per CTA, 8 warps, operands from HBM):\n");
    for (const Case& cs : cases) {
      HqGemmJob j{};
      j.M = j.Nc = j.K = kN;
      j.lda = j.ldb = j.ldc = kN;
      j.ta = cs.ta;
      j.tb = cs.tb;
      j.ks_mode = cs.ks;
      j.rs_mode = cs.rs;
      j.cs_mode = cs.cs;
      j.epi = cs.epi;
      j.alpha = 1.0;
      j.beta = cs.beta;
      j.active = 1;
      const int reps = 20;
      k_products<<<148, HQ_INT_THREADS, smem>>>(A, B, C, dv, nsets, j, 2, clk);
      cudaMemset(clk, 0, 8);
      k_products<<<148, HQ_INT_THREADS, smem>>>(A, B, C, dv, nsets, j, reps, clk);
      const cudaError_t e = cudaDeviceSynchronize();
      unsigned long long c;
      cudaMemcpy(&c, clk, 8, cudaMemcpyDeviceToHost);
      std::printf("  %-36s %7.0f cycles per product (%s)\n", cs.name, (double)c / (148.0 * reps), cudaGetErrorString(e));
    }
  }
  return 0;
}
