// hq_types.h -- data structures shared by the host engine and the sm_100a kernels.
//
// One Markov chain of the attractive-U Hubbard DQMC (the reference's DQMC::Core +
// Model::HubbardAttractiveU state, include/dqmc_core.h:35-112, include/hubbard.h:32-112)
// is described on the device by one HqChain. All matrices are FP64, column-major with
// leading dimension N (the Eigen::MatrixXd layout of the reference), resident in HBM.
#pragma once
#include <stdint.h>

#define HQ_MAX_L 16           // largest linear lattice size of the separable expK path
#define HQ_MAX_N 1024         // largest N = L*L handled by any path
#define HQ_THREADS 512        // threads of the per-chain factorisation kernels (16 warps)
#define HQ_INT_THREADS 256    // threads of the interval kernel (8 warps)

// expK application modes (the reference's is_fft switch, include/dqmc_params.hpp:44)
enum HqExpkMode { HQK_EXPK_DENSE = 0, HQK_EXPK_SEPARABLE = 1 };

// sweep directions (src/dqmc_core.cpp:167, :233, :291)
enum HqDir { HQ_UP = 0, HQ_DOWN = 1, HQ_DYNAMIC = 2 };

// kernel flags
enum HqFlags {
  HQ_F_MEASURE = 1,        // accumulate fused equal-time estimators
  HQ_F_SNAPSHOT = 2,       // store G(tau,tau) per slice (the reference's vecgftt)
  HQ_F_LOG_RATIOS = 4,     // store every acceptance ratio (replay checks)
  HQ_F_PHASE_CLOCKS = 8,   // persistent sweep: accumulate the clock64 cycles of every phase
};

// per-chain accumulators (doubles), laid out at HqChain::acc
enum HqAcc {
  HQ_ACC_FILLING = 0,      // sum over measured slices of 2 - 2 tr G / N
  HQ_ACC_DOCC = 1,         // sum over slices of (1/N) sum_i (1 - G_ii)^2
  HQ_ACC_SWAVE = 2,        // sum over slices of (1/N) sum_ij [(1-G)_ji^2 + G_ij^2]
  HQ_ACC_NSLICE = 3,       // number of slices accumulated
  HQ_ACC_WRAP_TT = 4,      // max signed wrap error, equal-time
  HQ_ACC_WRAP_DYN = 5,     // max signed wrap error, displaced
  HQ_ACC_PROPOSED = 6,     // proposals (as double)
  HQ_ACC_ACCEPTED = 7,     // accepted flips (as double)
  HQ_ACC_STATUS = 8,       // nonzero: a numerical failure was detected (NaN, singular pivot)
  HQ_ACC_DMU = 9,          // log-det adjoint: dt * sum_l tr(1 - G_l)
  HQ_ACC_DALPHA = 10,      // log-det adjoint: sum_l sum_i s_li (1 - G_l)_ii
  HQ_ACC_COUNT = 16
};

struct HqChain {
  // ---- geometry / schedule ----
  int N;            // number of sites = L*L
  int L;            // linear lattice size
  int nt;           // imaginary-time slices
  int pace;         // stabilisation pace
  int n_stab;       // ceil(nt / pace)
  int expk_mode;    // HqExpkMode
  int kmax;         // delay depth of the rank-k Metropolis updates
  int active;       // 0: chain is skipped by every kernel
  // ---- model ----
  double alpha;     // acosh(exp(dt*u/2)) (src/hubbard.cpp:35)
  double dt;
  double delta_p;   // exp(-2 alpha) - 1   (flip of s = +1, src/hubbard.cpp:128)
  double delta_m;   // exp(+2 alpha) - 1   (flip of s = -1)
  double ev_p;      // exp(+alpha)
  double ev_m;      // exp(-alpha)
  double sep_c;     // exp(+dt mu): expK = sep_c * (A (x) A)
  double sep_ci;    // exp(-dt mu): inv_expK = sep_ci * (Ai (x) Ai)
  double sep_a[HQ_MAX_L];   // circulant coefficients of A  = exp(+dt t H_1d)
  double sep_ai[HQ_MAX_L];  // circulant coefficients of Ai = exp(-dt t H_1d)
  const double* expK;       // dense exp(-dt K), N x N (shared by chains of equal parameters)
  const double* inv_expK;   // dense exp(+dt K)
  // ---- state (HBM) ----
  double* G;        // G(tau,tau)
  double* Gt0;      // G(tau,0)
  double* G0t;      // G(0,tau)
  int8_t* fields;   // Ising fields [nt][N]
  uint32_t* rng;    // minstd_rand0 state (1 word)
  double* X;        // B-chain accumulator / factorisation input
  double* stackU;   // [2][n_stab][N*N]  (0: left, 1: right)
  double* stackD;   // [2][n_stab][N]
  double* stackVt;  // [2][n_stab][N*N]  cumulative V^T of each stack level
  double* W0;       // work N x N (factor T of the last decomposition)
  double* W1;       // work N x N
  double* W2;       // work N x N
  double* W3;       // work N x N
  double* W4;       // work N x N
  double* W5;       // work N x N
  double* snap_tt;  // optional [nt][N*N]
  double* snap_t0;  // optional [nt][N*N]
  double* snap_0t;  // optional [nt][N*N]
  double* ratios;   // optional ratio log [capacity]
  long long ratio_cap;
  long long* ratio_count;  // 1 word
  double* acc;      // HQ_ACC_COUNT doubles
  double* dyn_acc;  // [2 + N][nt] : spin, ldos, g(d, tau) for displacements d < N
};

// One job of the batched FP64 GEMM:  C = alpha * op(A) diag(ks) op(B) [scaled] + beta * C
// Vector scalings take a mode: 0 none, 1 multiply by v, 2 multiply by 1/max(v,1),
// 3 multiply by min(v,1) (the dmax / dmin split of include/utils/stable_numerics.hpp:56-64).
struct HqGemmJob {
  const double* A;
  const double* B;
  double* C;
  const double* ks;    // scales the inner index k (applied to A's columns), may be null
  const double* rs;    // scales output rows, may be null
  const double* cs;    // scales output columns, may be null
  int M, Nc, K;
  int lda, ldb, ldc;
  int ta, tb;          // transposes
  int ks_mode, rs_mode, cs_mode;
  double alpha, beta;
  double* err_out;     // epilogue 1: atomically max(C_new - C_old) into *err_out
  int epi;             // 0 plain, 1 wrap error + store
  int active;
};
