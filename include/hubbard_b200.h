/*
 * hubbard_b200.h -- C ABI of the B200 (sm_100a) DQMC sweep for the attractive-U Hubbard
 * model. A drop-in for the sweep of JefferyWangSH/hubbard-attractive-U: every entry point
 * below replaces a method of the reference's DQMC::Core / Model::HubbardAttractiveU /
 * Utils::SvdStack call surface (cited per function; paths are relative to that project).
 *
 * Conventions
 *   - Every function returns 0 on success and a negative HQ_E* code on failure; the
 *     message of the last failure of the calling thread is available from hq_last_error().
 *     Nothing throws or aborts across this boundary.
 *   - Matrices are FP64, column-major (the reference's Eigen::MatrixXd layout), N = nl*nl.
 *   - Ising fields are int32 arrays [nt][N] with values +1 / -1 (Eigen::ArrayXXi
 *     m_ising_fields(nt, ns) of include/hubbard.h:46).
 *   - A context holds many independent Markov chains (the reference's MPI ranks,
 *     include/dqmc_parser.hpp:94) on one GPU; every call acts on all chains at once
 *     unless it takes a chain index. One host thread per context; all work is issued on
 *     the context's own CUDA stream.
 */
#ifndef HUBBARD_B200_H
#define HUBBARD_B200_H

#include <stddef.h>

#if defined(__GNUC__)
#define HQ_API __attribute__((visibility("default")))
#else
#define HQ_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define HQ_OK 0
#define HQ_E_INVALID (-1)  /* invalid argument / state (reference: std::invalid_argument, assert) */
#define HQ_E_CUDA (-2)     /* CUDA runtime failure */
#define HQ_E_NUMERIC (-3)  /* non-finite value or singular pivot detected on the device */
#define HQ_E_RANGE (-4)    /* index out of range (reference: std::out_of_range) */
#define HQ_E_NOMEM (-5)    /* device allocation failed */

/* sweep directions (src/dqmc_core.cpp:167, :233, :291) */
#define HQ_SWEEP_UP 0      /* DQMC::Core::sweep_from_0_to_beta */
#define HQ_SWEEP_DOWN 1    /* DQMC::Core::sweep_from_beta_to_0 */
#define HQ_SWEEP_DYNAMIC 2 /* DQMC::Core::sweep_for_dynamic_green_functions */

/* sweep flags */
#define HQ_SWEEP_MEASURE 1  /* accumulate the equal-time estimators (filling, double occupancy, s-wave) */
#define HQ_SWEEP_SNAPSHOT 2 /* keep G(tau,tau) of every slice (the reference's vecgftt) */
#define HQ_SWEEP_LOG_RATIOS 4 /* record every Metropolis acceptance ratio (replay checks) */
#define HQ_SWEEP_PHASE_CLOCKS 8 /* persistent sweep: count the cycles of every phase (hq_phase_cycles) */

/* Green's function selectors for hq_get_g (include/dqmc_core.h:76-81) */
#define HQ_G_CURRENT 0 /* current_gftt() */
#define HQ_G_TT 1      /* gftt(t) */
#define HQ_G_T0 2      /* gft0(t) */
#define HQ_G_0T 3      /* gf0t(t) */

/* expK application (the reference's is_fft switch, include/dqmc_params.hpp:44) */
#define HQ_EXPK_DENSE 0      /* dense exp(-dt K) GEMM (the reference's default path) */
#define HQ_EXPK_SEPARABLE 1  /* 2-D lattice transform: exp(-dt K) = e^{dt mu} A (x) A */
#define HQ_EXPK_AUTO (-1)    /* picked by measurement at hq_create */

/* One Markov chain: the keys of the reference's config.toml (include/dqmc_parser.hpp:60-96)
 * plus the chain's seed and the delay depth of the rank-k updates. */
typedef struct hq_chain_params {
  int nl;                 /* [Lattice.SquareLattice] nl */
  double nnt;             /* [Model.HubbardAttractiveU] nnt (hopping t) */
  double u;               /* [Model.HubbardAttractiveU] u (= |U|, >= 0) */
  double mu;              /* [Model.HubbardAttractiveU] mu */
  double beta;            /* [MonteCarlo] beta */
  int nt;                 /* [MonteCarlo] nt */
  int stabilization_pace; /* [MonteCarlo] stabilization_pace */
  int expk_mode;          /* HQ_EXPK_* ([MonteCarlo] is_fft maps to HQ_EXPK_SEPARABLE) */
  long long seed;         /* Utils::Random::set_seed(seed) before set_ising_fields_to_random */
  int delay_depth;        /* sites per submatrix-update block (4, 8 or 16; others round down, min 4); 0 = largest that fits on chip */
  int dynamic;            /* 1: allocate the displaced G's (time-displaced measurements) */
  int snapshots;          /* 1: allocate per-slice G(tau,tau) storage (HQ_SWEEP_SNAPSHOT) */
} hq_chain_params;

typedef struct hq_ctx hq_ctx;

/* Copies the message of the calling thread's last failure into buf (always terminated). */
HQ_API int hq_last_error(char* buf, size_t len);

/* Creates a context of n_chains chains on CUDA device `device`: lattice, K, exp(-dt K),
 * alpha = acosh(exp(dt u / 2)) and the device state of every chain.
 * Replaces: Model::HubbardAttractiveU::initialize (src/hubbard.cpp:25-82),
 *           Lattice::SquareLattice::initialize (src/square_lattice.cpp:14-28),
 *           DQMC::Core::initialize (src/dqmc_core.cpp:20-30). */
HQ_API int hq_create(int device, int n_chains, const hq_chain_params* chains, hq_ctx** out);
HQ_API int hq_destroy(hq_ctx* ctx);

/* Per-bond hopping matrix (N x N, symmetric, column-major) for one chain:
 * K = -hop - mu * 1. Forces the dense expK path for that chain.
 * (Replaces -nnt * lattice.nn_hoppings() at src/hubbard.cpp:41.) */
HQ_API int hq_set_hopping(hq_ctx* ctx, int chain, const double* hop);

/* Replaces: Model::HubbardAttractiveU::set_ising_fields_to_random (src/hubbard.cpp:102-110)
 * with Utils::Random::set_seed(seed) (src/random.cpp:15) -- the same random stream. */
HQ_API int hq_fields_random(hq_ctx* ctx, int chain);
/* Replaces: DQMC::IO::load_ising_fields_configs (include/dqmc_io.hpp:257-290), in memory. */
HQ_API int hq_set_fields(hq_ctx* ctx, int chain, const int* fields);
/* Replaces: DQMC::IO::save_ising_fields_configs (include/dqmc_io.hpp:234-255), in memory. */
HQ_API int hq_get_fields(hq_ctx* ctx, int chain, int* fields);

/* Replaces: DQMC::Core::initialize_svdstacks + initialize_green_functions
 * (src/dqmc_core.cpp:67-97). Leaves every chain at tau = 0. */
HQ_API int hq_init_stacks_and_g(hq_ctx* ctx);

/* One directional sweep of every chain (dir = HQ_SWEEP_*).
 * Replaces: DQMC::Core::sweep_from_0_to_beta / sweep_from_beta_to_0 /
 *           sweep_for_dynamic_green_functions (src/dqmc_core.cpp:167-390). */
HQ_API int hq_sweep(hq_ctx* ctx, int dir, int flags);

/* Waits for the context's stream. */
HQ_API int hq_sync(hq_ctx* ctx);

/* Copies a Green's function of one chain into out (N*N doubles, column-major).
 * Replaces: DQMC::Core::current_gftt / gftt / gft0 / gf0t (include/dqmc_core.h:76-79). */
HQ_API int hq_get_g(hq_ctx* ctx, int chain, int which, int slice, double* out);
/* Overwrites the current G(tau,tau) of one chain (tests and checkpoint restore). */
HQ_API int hq_set_g(hq_ctx* ctx, int chain, const double* in);

/* out[0] = max equal-time wrap error, out[1] = max displaced wrap error (signed maxima).
 * Replaces: DQMC::Core::equaltimeWrapError / dynamicWrapError (include/dqmc_core.h:80-81). */
HQ_API int hq_get_wrap_errors(hq_ctx* ctx, int chain, double* out2);

/* Equal-time estimator sums of one chain since the last reset:
 * out[0] = sum over measured slices of filling, out[1] double occupancy, out[2] s-wave,
 * out[3] number of measured slices, out[4] proposals, out[5] accepted flips.
 * (include/observable_methods.hpp:39-151; divide by out[3] for the per-slice mean.) */
HQ_API int hq_get_estimators(hq_ctx* ctx, int chain, double* out6);
/* The same six sums for every chain at once, chain-major: out[6*chain + k]. One gather
 * launch and one device-to-host copy, instead of one copy per chain. The reference runs one
 * chain per MPI rank and collects the ranks' results with
 * Utils::MPI::gather_measurement_results_from_processors (include/utils/observable_gather.hpp:71);
 * this call is the in-GPU counterpart for the chains of one context. */
HQ_API int hq_get_estimators_all(hq_ctx* ctx, double* out);
/* Displaced estimator sums: spin[nt], ldos[nt] and the displacement-summed
 * g(d, tau) = sum_i G(tau,0)[i+d, i] as gd[N][nt] (include/observable_methods.hpp:84-195);
 * G(k,tau) = (1/N) sum_d cos(k.r_d) g(d,tau). Any pointer may be NULL. */
HQ_API int hq_get_dynamic_estimators(hq_ctx* ctx, int chain, double* spin, double* ldos, double* gd);
/* Zeroes the estimator sums (and with reset_wrap also the wrap errors) of every chain. */
HQ_API int hq_reset_estimators(hq_ctx* ctx, int reset_wrap);

/* Ratio log of one chain (HQ_SWEEP_LOG_RATIOS): copies up to cap ratios in visiting
 * order into out and returns their total count in *count. capacity set at first use. */
HQ_API int hq_ratio_log(hq_ctx* ctx, int chain, long long capacity, double* out, long long cap, long long* count);

/* Gradient of log|det(1 + B(nt-1)...B(0))| of every chain's current fields with respect to
 * mu, alpha and the hopping matrix entries (dK_ij for K = -hop - mu): out per chain is
 * [dmu, dalpha, dK (N*N column-major)] and logdet[chain]. Runs a no-update pass with
 * stabilisation every `pace` slices; state must be at tau = 0 (after init or an up+down pair).
 * No counterpart in the reference (new: adjoint of the log-determinant). */
HQ_API int hq_logdet_adjoint(hq_ctx* ctx, double* out, double* logdet);

/* Records the sequence of one directional sweep into a CUDA graph and replays it
 * (launch-bound inner loops). hq_launch_graph(dir) after hq_capture_graph(dir, flags). */
HQ_API int hq_capture_graph(hq_ctx* ctx, int dir, int flags);
HQ_API int hq_launch_graph(hq_ctx* ctx, int dir);

/* The context's CUDA stream (cudaStream_t), e.g. to time the sweep with CUDA events. */
HQ_API int hq_get_stream(hq_ctx* ctx, void** stream);

/* Per-launch timing: when enabled, every kernel launch of a sweep is bracketed by a pair
 * of CUDA events on the context stream (also inside captured graphs; enabling drops the
 * captured graphs). hq_profile_collect waits for the stream and adds the elapsed time of
 * every launch of the most recent sweep to ms[class] and 1 to counts[class]. Classes:
 * 0 interval (wrap + Metropolis), 1 B chain, 2 UDV factorisation, 3 batched GEMM,
 * 4 inversion, 5 boundary measurement, 6 displaced propagation, 7 log-det adjoint,
 * 8 interval on four-CTA clusters (16 x 16 lattices, G in distributed shared memory),
 * 9 persistent sweep (HQ_SWEEP_PERSISTENT: every phase of every chain in one launch). */
HQ_API int hq_profile_enable(hq_ctx* ctx, int on);
HQ_API int hq_profile_collect(hq_ctx* ctx, double* ms, long long* counts, int nclasses);

/* Per-chain expK mode and delay depth actually in use (after autotuning). */
HQ_API int hq_get_config(hq_ctx* ctx, int chain, int* expk_mode, int* delay_depth);

/* How an up or down sweep is issued (no counterpart in the reference, which updates one chain
 * per MPI rank; this is the batched form of DQMC::Core::sweep_from_0_to_beta /
 * sweep_from_beta_to_0, src/dqmc_core.cpp:167-284):
 *  HQ_SWEEP_LAUNCHES   one kernel launch per phase and stabilisation interval (wrap +
 *                      Metropolis, B chain, UDV, GEMMs, inverse, measurement), the chains split
 *                      into groups on forked streams;
 *  HQ_SWEEP_PERSISTENT one persistent launch per sweep: one CTA per SM takes (chain, interval)
 *                      items from a device queue and runs all the phases of an item; the
 *                      chains' intervals follow each other through device-side progress words.
 * Both give the same G and field trajectories. PERSISTENT needs every chain's matrices to fit
 * in one SM's shared memory (N <= 144 on B200); hq_set_sweep_mode returns HQ_E_RANGE
 * otherwise. Setting a mode drops the captured sweep graphs. hq_autotune picks the faster. */
#define HQ_SWEEP_LAUNCHES 0
#define HQ_SWEEP_PERSISTENT 1
HQ_API int hq_set_sweep_mode(hq_ctx* ctx, int mode);
HQ_API int hq_get_sweep_mode(hq_ctx* ctx, int* mode);

/* Phase cycles of the persistent sweep: for sweeps run with HQ_SWEEP_PHASE_CLOCKS in the
 * persistent mode, the clock64 cycles that the SM running an item spent in each phase, summed
 * over all items since the last reset (no counterpart in the reference; a profiling aid).
 * out[0] waiting for the chain's previous interval, [1] wrap + Metropolis, [2] B chain,
 * [3] UDV factorisation, [4] cumulative V^T, [5] builder products 1-2, [6] inverse,
 * [7] builder products 3-4, [8] measurement, [9] items. Writes min(n, 10) entries; reset != 0
 * zeroes the counters afterwards. Waits for the context stream. */
#define HQ_PHASES 10
HQ_API int hq_phase_cycles(hq_ctx* ctx, unsigned long long* out, int n, int reset);

/* Top of a chain's UDV stack (side 0: left, 1: right), replacing Utils::SvdStack's
 * StackLength / MatrixU / SingularValues / MatrixV (include/utils/svd_stack.hpp:78-103):
 * *length entries; the product of all pushes is U diag(D) V^T (U: N*N column-major, D: N,
 * V: N*N, V = the reference's product V_0 V_1 ...). D holds |diag R| of the pre-pivoted QR
 * that replaces the SVD. Any of U, D, V may be NULL; nothing is written when *length = 0.
 * Between sweeps the stacks are at tau = 0 (left empty) or at tau = beta (right empty). */
HQ_API int hq_get_stack(hq_ctx* ctx, int chain, int side, int* length, double* U, double* D, double* V);

/* State word of a chain's minstd_rand0 engine (Utils::Random, src/random.cpp:14-15). With the
 * fields (hq_get_fields / hq_set_fields) it is a checkpoint: after hq_set_fields,
 * hq_set_rng_state and hq_init_stacks_and_g the chain continues exactly as it would have from
 * tau = 0. The state must lie in [1, 2147483646]. */
HQ_API int hq_get_rng_state(hq_ctx* ctx, int chain, unsigned int* state);
HQ_API int hq_set_rng_state(hq_ctx* ctx, int chain, unsigned int state);

/* One timed candidate of hq_autotune. */
typedef struct {
  int nl;              /* lattice size of the group of chains */
  int expk_mode;       /* HQ_EXPK_SEPARABLE or HQ_EXPK_DENSE */
  int delay_depth;     /* sites per submatrix-update block */
  double ms_per_sweep; /* device time of one directional sweep of the whole context */
  int chosen;          /* 1: the candidate now in use for this lattice size */
  int cluster_size;    /* CTAs per chain of the interval kernel: 4 (G in a cluster's shared memory) or 1 */
  int sweep_mode;      /* HQ_SWEEP_LAUNCHES or HQ_SWEEP_PERSISTENT; nl = 0 marks the entries that
                          time the two modes for the whole context after the per-size choices */
} hq_tune_entry;

/* Picks, per lattice size, the expK application (the is_fft choice of the reference's
 * config, src/hubbard.cpp:38-80, here separable circulant passes vs dense DMMA GEMM), the
 * delay depth and, for the 16 x 16 lattice, the cluster size of the interval kernel (four
 * CTAs with G in distributed shared memory, or one CTA with G in global memory) by timing
 * `sweeps` directional sweeps of the whole context per candidate; then, where the context can
 * run it, the sweep mode (HQ_SWEEP_PERSISTENT or HQ_SWEEP_LAUNCHES) the same way. The device state is
 * restored after each candidate: the Markov chains are unaffected. Captured sweep graphs are
 * dropped (recapture them). Needs hq_init_stacks_and_g; allocates one temporary copy of the
 * context's device state. Writes up to `capacity` entries and the total count to *n_entries. */
HQ_API int hq_autotune(hq_ctx* ctx, int sweeps, hq_tune_entry* entries, int capacity, int* n_entries);

/* Host <-> device copy of the raw device state of all chains' fields (int8, [chain][nt][N])
 * for end-to-end measurements: one cudaMemcpyAsync each on the context stream. */
HQ_API int hq_upload_fields_i8(hq_ctx* ctx, const signed char* fields_all);
HQ_API int hq_download_fields_i8(hq_ctx* ctx, signed char* fields_all);

/* Equal-time G(0,0) = (1 + B(nt-1)...B(0))^-1 of one chain, computed without allocating any
 * device memory. No counterpart in the reference: it serves callers that cannot call
 * cudaMalloc, such as a process that hands out its whole device-memory budget once at start-up
 * and forbids allocations after that, or a long-running service that must never meet an
 * out-of-memory failure in the middle of its work.
 *   fields_dev: device array of nt*N int8 fields (+1/-1, [nt][N]); g_dev: device output,
 *   N*N doubles, column-major; stream: cudaStream_t (NULL = default stream).
 * Limits: N = nl*nl <= 64 and ceil(nt / stabilization_pace) <= 16; larger sizes return
 * HQ_E_RANGE with a message in hq_last_error(). All temporaries live in one 4 MiB device
 * array defined in the library, which every GPU that loads the library keeps until exit.
 * The first call on a device does the set-up: it looks up that array's device address (with
 * the device current) and raises the kernels' shared-memory limits where needed, so make the
 * first call on each device before any stream capture. The address is kept for the life of
 * the device's context: do not call it again on a device after cudaDeviceReset. Every call
 * shares the array and the array keeps the last call's contents: calls that overlap on the
 * GPU race, so serialise them (one stream, or stream ordering). The work is enqueued on
 * `stream`. */
HQ_API int hq_equaltime_g_noalloc(int nl, double nnt, double u, double mu, double beta, int nt,
                                  int stabilization_pace, const signed char* fields_dev, double* g_dev,
                                  void* stream);

#ifdef __cplusplus
}
#endif

#endif /* HUBBARD_B200_H */
