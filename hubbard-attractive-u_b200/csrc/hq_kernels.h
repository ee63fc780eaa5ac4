// hq_kernels.h -- host-side launch wrappers of the sm_100a DQMC kernels.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include "hq_types.h"

namespace hq {
size_t smem_interval_bytes(int Nmax, int kmax, bool resident);
size_t smem_matrix_bytes(int Nmax, bool resident, int extra_doubles);
size_t smem_invert_bytes(int Nmax, bool resident);
size_t smem_udt_bytes(int Nmax, bool resident);
// whether the interval kernel's dynamic shared memory for Nmax sites and delay depth kmax fits
// next to its static shared memory under the per-block opt-in limit optin (bytes)
bool interval_fits(int Nmax, int kmax, bool resident, size_t optin);
// whether every per-chain kernel can keep its matrix of Nmax sites in shared memory
bool matrices_fit(int Nmax, size_t optin);
cudaError_t prepare_kernels(int Nmax, int kmax, bool resident);
cudaError_t launch_interval(const HqChain* chains, int n, int dir, int b, int flags, int Nmax, int kmax, bool resident,
                            cudaStream_t st);
cudaError_t launch_bchain(const HqChain* chains, int n, int dir, int b, int Nmax, bool resident, cudaStream_t st);
cudaError_t launch_udt(const HqChain* chains, int n, int side, int b, int Nmax, bool resident, cudaStream_t st);
cudaError_t launch_invert(const HqChain* chains, int n, int b, int which, int Nmax, bool resident, cudaStream_t st);
cudaError_t launch_gemm(const HqGemmJob* jobs, int njobs, int Mmax, int Nmax, cudaStream_t st);
cudaError_t launch_measure(const HqChain* chains, int n, int dir, int b, int flags, cudaStream_t st);
cudaError_t launch_dyn_start(const HqChain* chains, int n, cudaStream_t st);
cudaError_t launch_dyn_slices(const HqChain* chains, int n, int b, int flags, int Nmax, bool resident, cudaStream_t st);
cudaError_t launch_dyn_measure(const HqChain* chains, int n, int b, int last_only, cudaStream_t st);
cudaError_t launch_dyn_store(const HqChain* chains, int n, int b, cudaStream_t st);
cudaError_t launch_dyn_commit(const HqChain* chains, int n, int b, cudaStream_t st);
cudaError_t launch_gather_acc(const HqChain* chains, int n, double* out, cudaStream_t st);
// the per-chain kernels that live in their own translation units (for function attributes)
const void* fn_interval();
const void* fn_udt();
const void* fn_invert();
// the interval kernel on a four-CTA cluster per chain (16 x 16 lattice, separable expK, delay
// depth 16): G spread over the cluster's shared memory
bool interval_cluster_ok(int N, int L, int expk_mode, int kmax);
size_t smem_interval_cl_bytes();
cudaError_t launch_interval_cl(const HqChain* chains, int n, int dir, int b, int flags, cudaStream_t st);
const void* fn_interval_cl();
int interval_cl_max_clusters();
cudaError_t prepare_interval_cl();
// the B chain of the 16 x 16 lattice split over four CTAs per chain by column blocks
size_t smem_bchain_cols_bytes();
cudaError_t launch_bchain_cols(const HqChain* chains, int n, int dir, int b, cudaStream_t st);
const void* fn_bchain_cols();
// the persistent sweep kernel: one launch per up / down sweep, one CTA per SM taking items (the
// next interval of one chain) by longest remaining work (cinfo[c] = {n_stab, cost per interval};
// nitems = the sum of n_stab); lists[(dir * nstab_max + b) * 5 + phase] is the per-chain job list
// of builder phase PH_PUSH..PH_B4; ctl holds sweep_ctl_ints(nchains) ints (counters, progress and
// claim words), zeroed by the launch; clk receives the phase cycles when flags has
// HQ_F_PHASE_CLOCKS
size_t smem_sweep_bytes(int Nmax, int kmax);
size_t sweep_ctl_ints(int nchains);
bool sweep_fits(int Nmax, int kmax, size_t optin);
cudaError_t prepare_sweep(int Nmax, int kmax);
cudaError_t launch_sweep(const HqChain* chains, int nchains, const int2* cinfo, int nitems,
                         const HqGemmJob* const* lists, int nstab_max, int dir, int flags, int* ctl,
                         unsigned long long* clk, int grid, int Nmax, int kmax, cudaStream_t st);
const void* fn_sweep();
cudaError_t launch_adj_interval(const HqChain* chains, int n, int b, int Nmax, bool resident, cudaStream_t st);
cudaError_t launch_adj_last(const HqChain* chains, int n, int b, cudaStream_t st);
}  // namespace hq
