// hq_kernels.cu -- the smaller sm_100a kernels of the batched DQMC sweep (FP64) and the
// shared-memory limits of every per-chain kernel. The large kernels have files of their own:
//  hq_interval.cu : k_interval (wrap + Metropolis flips with DMMA-flushed delayed updates)
//  hq_udt.cu      : k_udt (UDV factorisation of a stack push)
//  hq_invert.cu   : k_invert (blocked Gauss-Jordan inverse of the G builders)
//  hq_gemm.cu     : k_gemm (batched DMMA GEMM of the G builders)
// This file holds:
//  k_bchain    : B-matrix chain of one interval applied to U_top*D_top
//                (src/dqmc_core.cpp:190, :251 + the (M*U)*S product of svd_stack.hpp:144).
//  k_measure   : equal-time estimators + snapshot of a freshly built G.
//  k_dyn_*     : time-displaced propagation and estimators (src/dqmc_core.cpp:291-390,
//                include/observable_methods.hpp:84-195).
//  k_adj_*     : adjoint of log|det(1 + B...B)| (no counterpart in the reference).
#include "hq_phases.cuh"

namespace hq {

// ---------------------------------------------------------------------------------
//  k_bchain: X <- (U_top diag(D_top) or 1), then the B products of interval b:
//   up  : X <- B(t) X = e^{V_t} E X, t ascending            (src/dqmc_core.cpp:190)
//   down: X <- B(t)^T X = E e^{V_t} X, t descending           (src/dqmc_core.cpp:251)
//  dir UP pushes onto the left stack, DOWN onto the right stack; that stack holds b
//  entries before the push (top entry b-1, none when b = 0).
//  init: the right stack at initialisation (src/dqmc_core.cpp:67-87) is the down
//  direction without updates.
// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(HQ_INT_THREADS, 1)
k_bchain(const HqChain* __restrict__ chains, int nchains, int dir, int b, int resident) {
  extern __shared__ __align__(16) double smem[];
  __shared__ HqChain ch;
  __shared__ int8_t s[HQ_MAX_N];
  const int c = blockIdx.x;
  if (c >= nchains) return;
  if (threadIdx.x == 0) ch = chains[c];
  __syncthreads();
  if (!ch.active || b >= ch.n_stab) return;
  bchain_body(ch, dir, b, resident != 0, smem, s);
}

// ---------------------------------------------------------------------------------
//  k_measure: estimators + snapshot of G after a stabilisation (slice `lslice`
//  computed from the interval), the last slice of every interval.
// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(HQ_THREADS)
k_measure(const HqChain* __restrict__ chains, int nchains, int dir, int b, int flags) {
  __shared__ HqChain ch;
  __shared__ double red[96];
  const int c = blockIdx.x;
  if (c >= nchains) return;
  if (threadIdx.x == 0) ch = chains[c];
  __syncthreads();
  if (!ch.active || b >= ch.n_stab) return;
  measure_body(ch, dir, b, flags, red);
}

// ---------------------------------------------------------------------------------
//  Dynamic (time-displaced) sweep, src/dqmc_core.cpp:291-390. Per slice t:
//    G(t,t) <- B G B^-1 ; G(t,0) <- B G(t,0) ; G(0,t) <- G(0,t) B^-1
//  k_dyn_slices applies this for the interval's slices to one of the three matrices per
//  CTA (blockIdx.y = 0: G(t,t), 1: G(t,0), 2: G(0,t)), except for the last slice which
//  is rebuilt by the boundary step, and stores the per-slice results.
// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(HQ_INT_THREADS, 1)
k_dyn_slices(const HqChain* __restrict__ chains, int nchains, int b, int flags, int resident) {
  extern __shared__ __align__(16) double smem[];
  __shared__ HqChain ch;
  __shared__ int8_t s[HQ_MAX_N];
  const int c = blockIdx.x, which = blockIdx.y;
  if (c >= nchains) return;
  if (threadIdx.x == 0) ch = chains[c];
  __syncthreads();
  if (!ch.active || b >= ch.n_stab) return;
  const int N = ch.N;
  int t_lo, t_hi;
  interval_range(ch.nt, ch.pace, ch.n_stab, HQ_UP, b, t_lo, t_hi);
  double* src = which == 0 ? ch.G : (which == 1 ? ch.Gt0 : ch.G0t);
  double* snap = which == 0 ? ch.snap_tt : (which == 1 ? ch.snap_t0 : ch.snap_0t);
  double* M;
  int ld;
  double* p = smem;
  if (resident) { M = p; ld = smem_ld(N); p += (size_t)N * ld; load_mat_async(M, ld, src, N, N); }
  else { M = src; ld = N; }
  double* stage = p;
  __syncthreads();
  const int nsl = t_hi - t_lo + 1;
  for (int step = 0; step < nsl; ++step) {
    const int t = t_lo + step;
    const int l = t % ch.nt;
    for (int i = threadIdx.x; i < N; i += blockDim.x) s[i] = ch.fields[(size_t)l * N + i];
    __syncthreads();
    if (which != 2) {  // left multiplication by B(l) = e^V E
      apply_expk(ch, M, ld, 0, false, stage);
      scale_rows(M, ld, N, s, ch.ev_p, ch.ev_m);
      __syncthreads();
    }
    if (which != 1) {  // right multiplication by B(l)^-1 = E^-1 e^-V
      apply_expk(ch, M, ld, 1, true, stage);
      scale_cols(M, ld, N, s, ch.ev_m, ch.ev_p);
      __syncthreads();
    }
    if (step < nsl - 1 && snap) copy_mat(snap + (size_t)l * N * N, N, M, ld, N);
    __syncthreads();
  }
  if (resident) copy_mat(src, N, M, ld, N);
}

// G(t,0) <- G(t,t) and G(0,t) <- G(t,t) - 1 at the start of a dynamic sweep
// (src/dqmc_core.cpp:302-303)
__global__ void k_dyn_start(const HqChain* __restrict__ chains, int nchains) {
  const int c = blockIdx.x;
  if (c >= nchains) return;
  const HqChain& ch = chains[c];
  if (!ch.active) return;
  const int N = ch.N;
  for (int idx = threadIdx.x; idx < N * N; idx += blockDim.x) {
    const int i = idx % N, j = idx / N;
    const double v = ch.G[idx];
    ch.Gt0[idx] = v;
    ch.G0t[idx] = v - (i == j ? 1.0 : 0.0);
  }
}

// dynamic estimators of one slice l from G(t,0), G(0,t) (include/observable_methods.hpp:
// 110-120, 178-195) and the displacement-summed g(d) = sum_i G(t,0)[i+d, i] for G(k,t)
// (:84-103). dyn_acc layout: [0][nt] spin, [1][nt] ldos, [2 + d][nt] g(d) for d < N.
__device__ void dyn_measure(const HqChain& ch, const double* Gt0, const double* G0t, int l, double* red) {
  const int N = ch.N, L = ch.L;
  double sp = 0.0, ld = 0.0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const double a = Gt0[i + (size_t)i * N], b = G0t[i + (size_t)i * N];
    sp -= 2.0 * a * b;
    ld += a;
  }
  sp = block_sum(sp, red);
  ld = block_sum(ld, red);
  if (threadIdx.x == 0) {
    ch.dyn_acc[0 * ch.nt + l] += sp / (2.0 * N);
    ch.dyn_acc[1 * ch.nt + l] += ld / N;
  }
  // g(d): d = dx + L dy, sum over i of G[(xi+dx, yi+dy), i]
  for (int d = threadIdx.x; d < N; d += blockDim.x) {
    const int dx = d % L, dy = d / L;
    double acc = 0.0;
    for (int i = 0; i < N; ++i) {
      const int xi = i % L, yi = i / L;
      const int j = (xi + dx) % L + L * ((yi + dy) % L);
      acc += Gt0[j + (size_t)i * N];
    }
    ch.dyn_acc[(size_t)(2 + d) * ch.nt + l] += acc;
  }
}

// measure the dynamic estimators of every slice of interval b from the snapshots
// (slices of the interval other than the last) or from the fresh G's (the last one).
__global__ void __launch_bounds__(HQ_THREADS)
k_dyn_measure(const HqChain* __restrict__ chains, int nchains, int b, int last_only) {
  __shared__ HqChain ch;
  __shared__ double red[32];
  const int c = blockIdx.x;
  if (c >= nchains) return;
  if (threadIdx.x == 0) ch = chains[c];
  __syncthreads();
  if (!ch.active || b >= ch.n_stab) return;
  const int N = ch.N;
  int t_lo, t_hi;
  interval_range(ch.nt, ch.pace, ch.n_stab, HQ_UP, b, t_lo, t_hi);
  const size_t NN = (size_t)N * N;
  for (int t = last_only ? t_hi : t_lo; t <= t_hi; ++t) {
    const int l = t % ch.nt;
    const double* gt0;
    const double* g0t;
    if (t == t_hi) { gt0 = ch.Gt0; g0t = ch.G0t; }
    else { gt0 = ch.snap_t0 + l * NN; g0t = ch.snap_0t + l * NN; }
    dyn_measure(ch, gt0, g0t, l, red);
    __syncthreads();
  }
}

// at a dynamic boundary: copy the fresh G's into the snapshots of the boundary slice
// with the tau = 0 convention (src/dqmc_core.cpp:379-387)
__global__ void k_dyn_store(const HqChain* __restrict__ chains, int nchains, int b) {
  const int c = blockIdx.x;
  if (c >= nchains) return;
  const HqChain& ch = chains[c];
  if (!ch.active || b >= ch.n_stab) return;
  const int N = ch.N;
  int t_lo, t_hi;
  interval_range(ch.nt, ch.pace, ch.n_stab, HQ_UP, b, t_lo, t_hi);
  const int l = t_hi % ch.nt;
  const size_t NN = (size_t)N * N;
  for (int idx = threadIdx.x; idx < N * N; idx += blockDim.x) {
    const int i = idx % N, j = idx / N;
    const double gtt = ch.G[idx];
    if (ch.snap_tt) ch.snap_tt[l * NN + idx] = gtt;
    if (l == 0) {
      // at tau = beta the stored pair is G(0,0), G(0,0) - 1; the propagated matrices
      // are replaced likewise
      ch.Gt0[idx] = gtt;
      ch.G0t[idx] = gtt - (i == j ? 1.0 : 0.0);
    }
    if (ch.snap_t0) ch.snap_t0[l * NN + idx] = ch.Gt0[idx];
    if (ch.snap_0t) ch.snap_0t[l * NN + idx] = ch.G0t[idx];
  }
}

// commit the freshly built G(t,t), G(t,0), G(0,t) (in W3, W0, W5) after recording the
// signed wrap errors (src/dqmc_core.cpp:334-344)
__global__ void __launch_bounds__(HQ_THREADS) k_dyn_commit(const HqChain* __restrict__ chains, int nchains, int b) {
  __shared__ double red[32];
  const int c = blockIdx.x;
  if (c >= nchains) return;
  const HqChain& ch = chains[c];
  if (!ch.active || b >= ch.n_stab) return;
  const int NN = ch.N * ch.N;
  double ett = -INFINITY, edyn = -INFINITY;
  for (int idx = threadIdx.x; idx < NN; idx += blockDim.x) {
    const double ftt = ch.W3[idx], ft0 = ch.W0[idx], f0t = ch.W4[idx];
    ett = fmax(ett, ftt - ch.G[idx]);
    edyn = fmax(edyn, fmax(ft0 - ch.Gt0[idx], f0t - ch.G0t[idx]));
    ch.G[idx] = ftt;
    ch.Gt0[idx] = ft0;
    ch.G0t[idx] = f0t;
  }
  ett = block_max(ett, red);
  edyn = block_max(edyn, red);
  if (threadIdx.x == 0) {
    ch.acc[HQ_ACC_WRAP_TT] = fmax(ch.acc[HQ_ACC_WRAP_TT], ett);
    ch.acc[HQ_ACC_WRAP_DYN] = fmax(ch.acc[HQ_ACC_WRAP_DYN], edyn);
  }
}

// ---------------------------------------------------------------------------------
//  Adjoint of log|det(1 + B(nt-1)...B(0))| (no counterpart in the reference).
//  With G_l = (1 + B_l..B_1 B_nt..B_{l+1})^-1 the G of the up sweep after slice l:
//    d/dmu    = dt sum_l tr(1 - G_l)
//    d/dalpha = sum_l sum_i s_li (1 - G_l)_ii
//    d/dE     : tr(dE E^-1 D),  D = sum_l e^{-V_l} (1 - G_l) e^{V_l}
//  A no-update up pass wraps G slice by slice and is rebuilt from the stacks every
//  `pace` slices (the checkpoints), so no slice is stored. D accumulates in W4.
// ---------------------------------------------------------------------------------
__device__ void adj_accum(const HqChain& ch, const double* G, int ld, const int8_t* s, double* red) {
  const int N = ch.N;
  double tr = 0.0, sa = 0.0;
  for (int idx = threadIdx.x; idx < N * N; idx += blockDim.x) {
    const int i = idx % N, j = idx / N;
    const double one_m = (i == j ? 1.0 : 0.0) - G[i + (size_t)j * ld];
    const double f = (s[i] > 0 ? ch.ev_m : ch.ev_p) * (s[j] > 0 ? ch.ev_p : ch.ev_m);
    ch.W4[idx] += one_m * f;
    if (i == j) { tr += one_m; sa += (s[i] > 0 ? one_m : -one_m); }
  }
  tr = block_sum(tr, red);
  sa = block_sum(sa, red);
  if (threadIdx.x == 0) {
    ch.acc[HQ_ACC_DMU] += ch.dt * tr;
    ch.acc[HQ_ACC_DALPHA] += sa;
  }
}

__global__ void __launch_bounds__(HQ_INT_THREADS, 1)
k_adj_interval(const HqChain* __restrict__ chains, int nchains, int b, int resident) {
  extern __shared__ __align__(16) double smem[];
  __shared__ HqChain ch;
  __shared__ double red[32];
  __shared__ int8_t s[HQ_MAX_N];
  const int c = blockIdx.x;
  if (c >= nchains) return;
  if (threadIdx.x == 0) ch = chains[c];
  __syncthreads();
  if (!ch.active || b >= ch.n_stab) return;
  const int N = ch.N;
  int t_lo, t_hi;
  interval_range(ch.nt, ch.pace, ch.n_stab, HQ_UP, b, t_lo, t_hi);
  double* G;
  int ld;
  double* p = smem;
  if (resident) { G = p; ld = smem_ld(N); p += (size_t)N * ld; load_mat_async(G, ld, ch.G, N, N); }
  else { G = ch.G; ld = N; }
  double* stage = p;
  __syncthreads();
  const int nsl = t_hi - t_lo + 1;
  for (int step = 0; step < nsl; ++step) {
    const int t = t_lo + step;
    const int l = t % ch.nt;
    for (int i = threadIdx.x; i < N; i += blockDim.x) s[i] = ch.fields[(size_t)l * N + i];
    __syncthreads();
    wrap_slice(ch, G, ld, s, HQ_UP, stage);
    if (step < nsl - 1) adj_accum(ch, G, ld, s, red);
    __syncthreads();
  }
  if (resident) copy_mat(ch.G, N, G, ld, N);
}

// the last slice of interval b, after the boundary rebuilt G
__global__ void __launch_bounds__(HQ_THREADS) k_adj_last(const HqChain* __restrict__ chains, int nchains, int b) {
  __shared__ HqChain ch;
  __shared__ double red[32];
  __shared__ int8_t s[HQ_MAX_N];
  const int c = blockIdx.x;
  if (c >= nchains) return;
  if (threadIdx.x == 0) ch = chains[c];
  __syncthreads();
  if (!ch.active || b >= ch.n_stab) return;
  const int N = ch.N;
  int t_lo, t_hi;
  interval_range(ch.nt, ch.pace, ch.n_stab, HQ_UP, b, t_lo, t_hi);
  const int l = t_hi % ch.nt;
  for (int i = threadIdx.x; i < N; i += blockDim.x) s[i] = ch.fields[(size_t)l * N + i];
  __syncthreads();
  adj_accum(ch, ch.G, N, s, red);
}


}  // namespace hq

// =====================================================================================
//  launch wrappers (host)
// =====================================================================================
namespace hq {

size_t smem_interval_bytes(int Nmax, int kmax, bool resident) {
  return interval_smem_doubles(Nmax, kmax, resident) * sizeof(double);
}
size_t smem_udt_bytes(int Nmax, bool resident) {
  return smem_matrix_bytes(Nmax, resident, 2 * kQB * panel_ld(Nmax) + 2 * kQB * kQB + 3 * Nmax + 64 +
                                               ((Nmax - 1) / kQB) * kQB * kQB);
}
size_t smem_invert_bytes(int Nmax, bool resident) {
  return smem_matrix_bytes(Nmax, resident, 2 * kGJ * panel_ld(Nmax) + 3 * Nmax + 64);
}
size_t smem_matrix_bytes(int Nmax, bool resident, int extra_doubles) {
  const size_t mat = resident ? (size_t)Nmax * smem_ld(Nmax) : 0;
  return (mat + (size_t)extra_doubles) * sizeof(double);
}

// The dynamic shared-memory limit of a kernel is a per-device property of the function
// shared by every context of the process: it is only ever raised, so that preparing a
// context of small chains never lowers the limit an existing context of larger chains
// launches with.
constexpr int kMaxTrackedDevices = 64;
constexpr int kTrackedKernels = 8;
static size_t g_smem_set[kMaxTrackedDevices][kTrackedKernels];

static cudaError_t raise_smem(int slot, const void* fn, size_t bytes) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 0 && dev < kMaxTrackedDevices && g_smem_set[dev][slot] >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess && dev >= 0 && dev < kMaxTrackedDevices) g_smem_set[dev][slot] = bytes;
  return e;
}

// sets the dynamic shared-memory limits of every per-chain kernel (outside any stream
// capture) so that chains of up to Nmax sites can be launched
// dynamic shared memory that kernel fn can take next to its own static shared memory under the
// device's per-block opt-in limit optin
static size_t smem_room(const void* fn, size_t optin) {
  cudaFuncAttributes a;
  const size_t st = cudaFuncGetAttributes(&a, fn) == cudaSuccess ? a.sharedSizeBytes : 16384;  // conservative
  return optin > st ? optin - st : 0;
}

bool interval_fits(int Nmax, int kmax, bool resident, size_t optin) {
  return smem_interval_bytes(Nmax, kmax, resident) <= smem_room(fn_interval(), optin);
}

bool matrices_fit(int Nmax, size_t optin) {
  const size_t mat_stage = smem_matrix_bytes(Nmax, true, 8 * (((Nmax + 15) & ~15) + 4) + 64);
  return interval_fits(Nmax, 4, true, optin) && mat_stage <= smem_room((const void*)k_bchain, optin) &&
         mat_stage <= smem_room((const void*)k_dyn_slices, optin) &&
         mat_stage <= smem_room((const void*)k_adj_interval, optin) &&
         smem_invert_bytes(Nmax, true) <= smem_room(fn_invert(), optin) &&
         smem_udt_bytes(Nmax, true) <= smem_room(fn_udt(), optin);
}

cudaError_t prepare_kernels(int Nmax, int kmax, bool resident) {
  const size_t mat_stage = smem_matrix_bytes(Nmax, resident, 8 * (((Nmax + 15) & ~15) + 4) + 64);
  cudaError_t e;
  if ((e = raise_smem(0, fn_interval(), smem_interval_bytes(Nmax, kmax, resident))) != cudaSuccess) return e;
  if ((e = raise_smem(1, (const void*)k_bchain, mat_stage)) != cudaSuccess) return e;
  if ((e = raise_smem(2, fn_udt(), smem_udt_bytes(Nmax, resident))) != cudaSuccess) return e;
  if ((e = raise_smem(3, fn_invert(), smem_invert_bytes(Nmax, resident))) != cudaSuccess) return e;
  if ((e = raise_smem(4, (const void*)k_dyn_slices, mat_stage)) != cudaSuccess) return e;
  if ((e = raise_smem(5, (const void*)k_adj_interval, mat_stage)) != cudaSuccess) return e;
  return cudaSuccess;
}

cudaError_t prepare_interval_cl() {
  const cudaError_t e = raise_smem(6, fn_interval_cl(), smem_interval_cl_bytes());
  if (e != cudaSuccess) return e;
  return raise_smem(7, fn_bchain_cols(), smem_bchain_cols_bytes());
}

cudaError_t launch_bchain(const HqChain* chains, int n, int dir, int b, int Nmax, bool resident, cudaStream_t st) {
  const size_t bytes = smem_matrix_bytes(Nmax, resident, 8 * (((Nmax + 15) & ~15) + 4) + 64);
  k_bchain<<<n, HQ_INT_THREADS, bytes, st>>>(chains, n, dir, b, resident ? 1 : 0);
  return cudaGetLastError();
}
cudaError_t launch_measure(const HqChain* chains, int n, int dir, int b, int flags, cudaStream_t st) {
  k_measure<<<n, HQ_THREADS, 0, st>>>(chains, n, dir, b, flags);
  return cudaGetLastError();
}
cudaError_t launch_dyn_start(const HqChain* chains, int n, cudaStream_t st) {
  k_dyn_start<<<n, 256, 0, st>>>(chains, n);
  return cudaGetLastError();
}
cudaError_t launch_dyn_slices(const HqChain* chains, int n, int b, int flags, int Nmax, bool resident, cudaStream_t st) {
  const size_t bytes = smem_matrix_bytes(Nmax, resident, 8 * (((Nmax + 15) & ~15) + 4) + 64);
  dim3 grid(n, 3);
  k_dyn_slices<<<grid, HQ_INT_THREADS, bytes, st>>>(chains, n, b, flags, resident ? 1 : 0);
  return cudaGetLastError();
}
cudaError_t launch_dyn_measure(const HqChain* chains, int n, int b, int last_only, cudaStream_t st) {
  k_dyn_measure<<<n, HQ_THREADS, 0, st>>>(chains, n, b, last_only);
  return cudaGetLastError();
}
cudaError_t launch_dyn_store(const HqChain* chains, int n, int b, cudaStream_t st) {
  k_dyn_store<<<n, 256, 0, st>>>(chains, n, b);
  return cudaGetLastError();
}
cudaError_t launch_adj_interval(const HqChain* chains, int n, int b, int Nmax, bool resident, cudaStream_t st) {
  const size_t bytes = smem_matrix_bytes(Nmax, resident, 8 * (((Nmax + 15) & ~15) + 4) + 64);
  k_adj_interval<<<n, HQ_INT_THREADS, bytes, st>>>(chains, n, b, resident ? 1 : 0);
  return cudaGetLastError();
}
cudaError_t launch_adj_last(const HqChain* chains, int n, int b, cudaStream_t st) {
  k_adj_last<<<n, HQ_THREADS, 0, st>>>(chains, n, b);
  return cudaGetLastError();
}
cudaError_t launch_dyn_commit(const HqChain* chains, int n, int b, cudaStream_t st) {
  k_dyn_commit<<<n, HQ_THREADS, 0, st>>>(chains, n, b);
  return cudaGetLastError();
}

// Copies every chain's accumulator block into one chain-major buffer, so that a single
// device-to-host copy reads the estimators of all chains.
__global__ void k_gather_acc(const HqChain* chains, int n, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * HQ_ACC_COUNT) return;
  const int c = i / HQ_ACC_COUNT;
  out[i] = chains[c].acc[i - c * HQ_ACC_COUNT];
}
cudaError_t launch_gather_acc(const HqChain* chains, int n, double* out, cudaStream_t st) {
  const int total = n * HQ_ACC_COUNT;
  k_gather_acc<<<(total + 255) / 256, 256, 0, st>>>(chains, n, out);
  return cudaGetLastError();
}

}  // namespace hq

