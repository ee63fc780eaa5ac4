// hq_engine.cu -- host engine of the batched B200 DQMC sweep and its C ABI
// (include/hubbard_b200.h).
//
// The engine owns, per context, the device state of many independent Markov chains
// (the reference's MPI ranks) in one HBM arena, precomputes the batched GEMM job lists
// of every stabilisation step, and issues the sweep of src/dqmc_core.cpp:167-390 as a
// fixed sequence of kernel launches on one stream (optionally captured in a CUDA graph).
#include <cuda_runtime.h>
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/hubbard_b200.h"
#include "hq_kernels.h"
#include "hq_types.h"

namespace {

thread_local std::string g_last_error;

struct HqError : std::runtime_error {
  int code;
  HqError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define HQ_CUDA(call)                                                                           \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      throw HqError(HQ_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));             \
  } while (0)

// ---------------------------------------------------------------------------------------
//  Random stream of the reference: std::default_random_engine (minstd_rand0) seeded by
//  Utils::Random::set_seed (src/random.cpp:15) and bernoulli draws through
//  generate_canonical<double, 53> (two engine values per draw).
// ---------------------------------------------------------------------------------------
constexpr uint64_t kA = 16807, kM = 2147483647;

inline uint32_t minstd_seed(long long seed) {
  // linear_congruential_engine::seed: x = s mod m; x = 1 if that is 0 (c = 0)
  const unsigned long s = static_cast<unsigned long>(seed);
  uint32_t x = static_cast<uint32_t>(s % kM);
  return x == 0 ? 1u : x;
}
inline uint32_t minstd_next(uint32_t x) { return static_cast<uint32_t>((kA * x) % kM); }
inline double canonical(uint32_t& x) {
  const uint32_t x1 = minstd_next(x);
  const uint32_t x2 = minstd_next(x1);
  x = x2;
  volatile double R = 2147483646.0;  // keep the IEEE double operation order
  volatile double RR = R * R;
  volatile double t2 = static_cast<double>(x2 - 1u) * R;
  volatile double sum = static_cast<double>(x1 - 1u) + t2;
  double r = sum / RR;
  if (r >= 1.0) r = std::nextafter(1.0, 0.0);
  return r;
}

// ---------------------------------------------------------------------------------------
//  exp(-dt K) for K = -t H_nn - mu 1 on the L x L torus (src/hubbard.cpp:41-47):
//  H_nn = H_1d (x) 1 + 1 (x) H_1d with H_1d[x][x+-1] += 1 (PBC; L = 2 doubles the bond,
//  L = 1 gives the 1 x 1 matrix [2], exactly as src/square_lattice.cpp:48-61 builds it).
//  exp(dt t H_1d) is circulant with a[d] = (1/L) sum_k exp(2 dt t cos(2 pi k/L)) cos(2 pi k d/L).
// ---------------------------------------------------------------------------------------
void circulant_exp(int L, double dt_t, double* a) {
  for (int d = 0; d < L; ++d) {
    long double acc = 0.0L;
    for (int k = 0; k < L; ++k) {
      const long double th = 2.0L * 3.14159265358979323846264338327950288L * k / L;
      acc += std::exp(2.0L * dt_t * std::cos(th)) * std::cos(th * d);
    }
    a[d] = static_cast<double>(acc / L);
  }
}

// cyclic Jacobi eigen-decomposition of a symmetric matrix (host, once per custom K)
void jacobi_eig(int n, std::vector<double> A, std::vector<double>& w, std::vector<double>& Q) {
  Q.assign(size_t(n) * n, 0.0);
  for (int i = 0; i < n; ++i) Q[i + size_t(i) * n] = 1.0;
  auto a = [&](int i, int j) -> double& { return A[i + size_t(j) * n]; };
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < j; ++i) off += a(i, j) * a(i, j);
    if (off < 1e-30) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = a(p, q);
        if (std::fabs(apq) < 1e-300) continue;
        const double theta = (a(q, q) - a(p, p)) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {
          const double akp = a(k, p), akq = a(k, q);
          a(k, p) = c * akp - s * akq;
          a(k, q) = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          const double apk = a(p, k), aqk = a(q, k);
          a(p, k) = c * apk - s * aqk;
          a(q, k) = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double qkp = Q[k + size_t(p) * n], qkq = Q[k + size_t(q) * n];
          Q[k + size_t(p) * n] = c * qkp - s * qkq;
          Q[k + size_t(q) * n] = s * qkp + c * qkq;
        }
      }
  }
  w.resize(n);
  for (int i = 0; i < n; ++i) w[i] = a(i, i);
}

void host_gemm(int n, const double* A, bool ta, const double* B, bool tb, double* C) {
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      long double s = 0.0L;
      for (int k = 0; k < n; ++k) {
        const double av = ta ? A[k + size_t(i) * n] : A[i + size_t(k) * n];
        const double bv = tb ? B[j + size_t(k) * n] : B[k + size_t(j) * n];
        s += (long double)av * bv;
      }
      C[i + size_t(j) * n] = (double)s;
    }
}

struct ChainHost {
  hq_chain_params p;
  int N, n_stab, kmax, expk_mode;
  bool custom_hop = false;
  std::vector<double> hop;     // N x N hopping (custom or nearest neighbour)
  std::vector<double> K;       // N x N
  double alpha, dt;
  uint32_t rng_after_fields = 0;
  bool fields_set = false;
};

inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace

struct hq_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int n = 0;
  std::vector<ChainHost> ch;
  std::vector<HqChain> desc;
  HqChain* d_desc = nullptr;
  // every chain's accumulators gathered chain-major (device) and its pinned host copy
  double* d_acc_all = nullptr;
  double* h_acc_all = nullptr;
  char* arena = nullptr;
  size_t arena_bytes = 0;
  std::vector<void*> extra_allocs;
  int Nmax = 0, kmax_max = 0, ntmax = 0, nstab_max = 0;
  bool resident = true;         // matrices fit in one SM's shared memory
  bool cluster_interval = false;  // the interval kernel may run on four-CTA clusters (16 x 16 lattices)
  bool cluster_capable = false;   // the device can run them (the autotuner may switch them off)
  bool has_dynamic = false;
  // batched GEMM job lists: key (phase, dir, b) -> device pointer + count
  std::map<std::tuple<int, int, int>, std::pair<HqGemmJob*, int>> jobs;
  HqGemmJob* d_jobs = nullptr;
  // identity / ones per N
  std::map<int, std::pair<double*, double*>> ident;
  // CUDA graphs per (dir, flags)
  std::map<std::pair<int, int>, cudaGraphExec_t> graphs;
  std::map<std::pair<int, int>, size_t> graph_prof;  // events recorded by each graph
  // per-launch timing: event pairs recorded around every launch of a sweep (class id)
  bool profiling = false;
  struct ProfEv { int cls; cudaEvent_t e0, e1; };
  std::vector<ProfEv> prof;
  size_t prof_next = 0;
  // chain groups of the up / down sweeps: each group's kernels run on its own stream, so that
  // one group's launches fill the SMs left idle by the other's last wave
  // (two groups when the chains are resident in one SM's shared memory, so that the groups fill
  // the GPU; four for larger chains, whose per-chain phases leave most SMs idle on their own)
  static constexpr int kGroups = 4;
  int ngroups = 1;
  int gbeg[kGroups + 1] = {0, 0, 0, 0, 0};  // first chain of each group (contiguous ranges)
  cudaStream_t gstream[kGroups] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t ev_fork = nullptr, ev_join[kGroups] = {nullptr, nullptr, nullptr, nullptr};
  // the chains and stream the launch helpers currently issue for (default: all, main stream)
  int cur_c0 = 0, cur_n = 0;
  cudaStream_t cur_st = nullptr;
  // persistent sweep (HQ_SWEEP_PERSISTENT): per chain {n_stab, cost of an interval}, the total
  // of the chains' intervals, the per-chain builder job lists of every (direction, interval,
  // phase), the counter / progress / claim words
  bool sweep_capable = false;
  int sweep_mode = HQ_SWEEP_LAUNCHES;
  int2* d_items = nullptr;
  int nitems = 0;
  const HqGemmJob** d_lists = nullptr;
  int* d_ctl = nullptr;
  int nctl = 0;
  unsigned long long* d_clk = nullptr;  // phase cycles (HQ_SWEEP_PHASE_CLOCKS)
  int sweep_grid = 0;
  bool at_zero = false;         // stacks at tau = 0 (left empty, right full)
  bool at_beta = false;         // stacks at tau = beta
  bool initialised = false;

  ~hq_ctx() {
    for (auto& g : graphs) cudaGraphExecDestroy(g.second);
    if (d_jobs) cudaFree(d_jobs);
    if (d_items) cudaFree(d_items);
    if (d_lists) cudaFree(d_lists);
    if (d_ctl) cudaFree(d_ctl);
    if (d_clk) cudaFree(d_clk);
    if (d_desc) cudaFree(d_desc);
    if (d_acc_all) cudaFree(d_acc_all);
    if (h_acc_all) cudaFreeHost(h_acc_all);
    if (arena) cudaFree(arena);
    for (auto* p : extra_allocs) cudaFree(p);
    for (auto& e : prof) { cudaEventDestroy(e.e0); cudaEventDestroy(e.e1); }
    for (int g = 0; g < kGroups; ++g) {
      if (gstream[g] && gstream[g] != stream) cudaStreamDestroy(gstream[g]);
      if (ev_join[g]) cudaEventDestroy(ev_join[g]);
    }
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

enum Phase {
  PH_PUSH = 0,   // Vt_new = T * Vt_prev
  PH_B1, PH_B2, PH_B3, PH_B4,                       // equal-time builder
  PH_D3, PH_D4, PH_D5, PH_D6,  // displaced builder
  PH_LOGDET,
};

// stack views of one chain: top entries (or identity when empty)
struct StackView {
  const double* U;
  const double* D;
  const double* Vt;
};

StackView stack_view(hq_ctx* c, int chain, int side, int top) {
  const HqChain& d = c->desc[chain];
  const size_t NN = size_t(d.N) * d.N;
  if (top < 0) {
    auto& id = c->ident[d.N];
    return {id.first, id.second, id.first};
  }
  return {d.stackU + (size_t(side) * d.n_stab + top) * NN, d.stackD + (size_t(side) * d.n_stab + top) * d.N,
          d.stackVt + (size_t(side) * d.n_stab + top) * NN};
}

HqGemmJob make_job(int N, const double* A, int ta, const double* B, int tb, double* C) {
  HqGemmJob j;
  std::memset(&j, 0, sizeof(j));
  j.A = A; j.B = B; j.C = C;
  j.M = j.Nc = j.K = N;
  j.lda = j.ldb = j.ldc = N;
  j.ta = ta; j.tb = tb;
  j.alpha = 1.0; j.beta = 0.0;
  j.active = 1;
  return j;
}

// dir: 0 up, 1 down, 2 init (right stack build), 3 dynamic
// returns for interval b the (left_top, right_top) after the push/pop of that step
void tops_after(const HqChain& d, int dir, int b, int& lt, int& rt) {
  if (dir == HQ_UP || dir == 3) { lt = b; rt = d.n_stab - 2 - b; }
  else if (dir == HQ_DOWN) { lt = d.n_stab - 2 - b; rt = b; }
  else { lt = -1; rt = b; }
}

void build_jobs(hq_ctx* c) {
  std::vector<HqGemmJob> all;
  std::vector<std::tuple<int, int, int, size_t, int>> index;  // phase, dir, b, offset, count
  auto add_phase = [&](int phase, int dir, int b, const std::vector<HqGemmJob>& js) {
    index.emplace_back(phase, dir, b, all.size(), int(js.size()));
    all.insert(all.end(), js.begin(), js.end());
  };
  for (int dir = 0; dir < 4; ++dir) {
    if (dir == 3 && !c->has_dynamic) continue;
    for (int b = 0; b < c->nstab_max; ++b) {
      std::map<int, std::vector<HqGemmJob>> ph;
      for (int i = 0; i < c->n; ++i) {
        const HqChain& d = c->desc[i];
        const int N = d.N;
        const size_t NN = size_t(N) * N;
        const bool act = b < d.n_stab;
        auto push_job = [&](int phase, HqGemmJob j) {
          j.active = act ? j.active : 0;
          ph[phase].push_back(j);
        };
        // ---- push: Vt_new = T (W0) * Vt_prev ----
        const int side = (dir == HQ_DOWN || dir == 2) ? 1 : 0;
        {
          auto& id = c->ident[N];
          const double* prev = (b == 0) ? id.first : d.stackVt + (size_t(side) * d.n_stab + (b - 1)) * NN;
          double* out = d.stackVt + (size_t(side) * d.n_stab + std::min(b, d.n_stab - 1)) * NN;
          push_job(PH_PUSH, make_job(N, d.W0, 0, prev, 0, out));
        }
        int lt, rt;
        tops_after(d, dir, b, lt, rt);
        const StackView Lv = stack_view(c, i, 0, lt), Rv = stack_view(c, i, 1, rt);
        // ---- builder common part: W1 = dlmax^-1 (U_L^T U_R) drmax^-1 + dlmin (Vt_L Vt_R^T) drmin ----
        {
          HqGemmJob j = make_job(N, Lv.U, 1, Rv.U, 0, d.W1);
          j.rs = Lv.D; j.rs_mode = 2; j.cs = Rv.D; j.cs_mode = 2;
          push_job(PH_B1, j);
          HqGemmJob k = make_job(N, Lv.Vt, 0, Rv.Vt, 1, d.W1);
          k.rs = Lv.D; k.rs_mode = 3; k.cs = Rv.D; k.cs_mode = 3; k.beta = 1.0;
          push_job(PH_B2, k);
        }
        // ---- equal-time: W2 = W1^-1 dlmax^-1 U_L^T ; G = U_R drmax^-1 W2 ----
        {
          HqGemmJob j = make_job(N, d.W1, 0, Lv.U, 1, d.W2);
          j.ks = Lv.D; j.ks_mode = 2;
          push_job(PH_B3, j);
          HqGemmJob k = make_job(N, Rv.U, 0, d.W2, 0, d.G);
          k.ks = Rv.D; k.ks_mode = 2;
          if (dir == HQ_UP || dir == HQ_DOWN) { k.epi = 1; k.err_out = d.acc + HQ_ACC_WRAP_TT; }
          push_job(PH_B4, k);
        }
        if (dir == 3) {
          // G(t,t) fresh -> W3, G(t,0) fresh -> W0, G(0,t) fresh -> W4, with
          // Y = W1^-1 dlmax^-1 U_L^T (W2, from PH_B3) and W1 = T1^-1:
          //   G(t,t) =  U_R drmax^-1 Y
          //   G(t,0) =  U_R drmax^-1 T1^-1 dlmin Vt_L            (stable_numerics.hpp:300-301)
          //   G(0,t) = -B(beta,t) G(t,t) = -Vt_R^T drmin Y         (C = Vt_R^T D_R U_R^T and
          //            D_R drmax^-1 = drmin: no inverse of the V factors is needed)
          HqGemmJob k = make_job(N, Rv.U, 0, d.W2, 0, d.W3);
          k.ks = Rv.D; k.ks_mode = 2;
          push_job(PH_D3, k);
          HqGemmJob j5 = make_job(N, d.W1, 0, Lv.Vt, 0, d.W5);  // T1^-1 dlmin Vt_L
          j5.ks = Lv.D; j5.ks_mode = 3;
          push_job(PH_D4, j5);
          HqGemmJob j6 = make_job(N, Rv.U, 0, d.W5, 0, d.W0);  // U_R drmax^-1 (...)
          j6.ks = Rv.D; j6.ks_mode = 2;
          push_job(PH_D5, j6);
          HqGemmJob j7 = make_job(N, Rv.Vt, 1, d.W2, 0, d.W4);  // -Vt_R^T drmin Y
          j7.ks = Rv.D; j7.ks_mode = 3; j7.alpha = -1.0;
          push_job(PH_D6, j7);
        }
      }
      for (auto& kv : ph) add_phase(kv.first, dir, b, kv.second);
    }
  }
  // log-det matrix: W1 = dmax^-1 U^T + dmin Vt of the left stack at tau = beta (all pushed)
  {
    std::vector<HqGemmJob> js;
    for (int i = 0; i < c->n; ++i) {
      const HqChain& d = c->desc[i];
      const StackView Lv = stack_view(c, i, 0, d.n_stab - 1);
      HqGemmJob j = make_job(d.N, c->ident[d.N].first, 0, Lv.U, 1, d.W1);
      j.rs = Lv.D; j.rs_mode = 2;
      js.push_back(j);
    }
    add_phase(PH_LOGDET, 0, 0, js);
    std::vector<HqGemmJob> js2;
    for (int i = 0; i < c->n; ++i) {
      const HqChain& d = c->desc[i];
      const StackView Lv = stack_view(c, i, 0, d.n_stab - 1);
      HqGemmJob j = make_job(d.N, c->ident[d.N].first, 0, Lv.Vt, 0, d.W1);
      j.rs = Lv.D; j.rs_mode = 3; j.beta = 1.0;
      js2.push_back(j);
    }
    add_phase(PH_LOGDET, 0, 1, js2);
  }
  if (c->d_jobs) cudaFree(c->d_jobs);
  HQ_CUDA(cudaMalloc(&c->d_jobs, std::max<size_t>(1, all.size()) * sizeof(HqGemmJob)));
  HQ_CUDA(cudaMemcpy(c->d_jobs, all.data(), all.size() * sizeof(HqGemmJob), cudaMemcpyHostToDevice));
  c->jobs.clear();
  for (auto& t : index) {
    int phase, dir, b, count;
    size_t off;
    std::tie(phase, dir, b, off, count) = t;
    c->jobs[std::make_tuple(phase, dir, b)] = {c->d_jobs + off, count};
  }
}

// The persistent sweep's scheduling data: per chain {n_stab, estimated cycles of one interval}
// (the kernel claims, among the ready chains, the one with the longest remaining work); the
// per-chain job lists of the five builder phases of every (direction, interval); the counter,
// progress and claim words; the grid (as many CTAs as are resident at once).
int item_cost(const ChainHost& h) {
  // thousands of cycles of one interval, of the measured shape: wrap, flushes, factorisations
  // and products ~ N^3, the walk, reflectors and pivots ~ N sequential steps
  const double N = h.N, pace = h.p.stabilization_pace;
  return int(1e-3 * (N * N * N * (0.074 * pace + 0.54)) + N * (5.0 + 0.3 * pace)) + 1;
}

void setup_sweep(hq_ctx* c) {
  HQ_CUDA(hq::prepare_sweep(c->Nmax, c->kmax_max));
  int sms = 0, per_sm = 0;
  HQ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
  HQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hq::fn_sweep(), HQ_INT_THREADS,
                                                        hq::smem_sweep_bytes(c->Nmax, c->kmax_max)));
  if (per_sm < 1) return;  // not launchable here: the context keeps the launch sequence
  c->sweep_grid = sms * per_sm;
  std::vector<int2> cinfo(c->n);
  c->nitems = 0;
  for (int i = 0; i < c->n; ++i) {
    cinfo[i] = make_int2(c->ch[i].n_stab, item_cost(c->ch[i]));
    c->nitems += c->ch[i].n_stab;
  }
  std::vector<const HqGemmJob*> lists;
  const int phases[5] = {PH_PUSH, PH_B1, PH_B2, PH_B3, PH_B4};
  for (int dir = 0; dir < 2; ++dir)
    for (int b = 0; b < c->nstab_max; ++b)
      for (int ph : phases) {
        auto it = c->jobs.find(std::make_tuple(ph, dir, b));
        if (it == c->jobs.end() || it->second.second != c->n) throw HqError(HQ_E_INVALID, "internal: sweep job list");
        lists.push_back(it->second.first);
      }
  c->nctl = int(hq::sweep_ctl_ints(c->n));
  HQ_CUDA(cudaMalloc(&c->d_items, cinfo.size() * sizeof(int2)));
  HQ_CUDA(cudaMalloc(&c->d_lists, lists.size() * sizeof(HqGemmJob*)));
  HQ_CUDA(cudaMalloc(&c->d_ctl, size_t(c->nctl) * sizeof(int)));
  HQ_CUDA(cudaMemcpy(c->d_items, cinfo.data(), cinfo.size() * sizeof(int2), cudaMemcpyHostToDevice));
  HQ_CUDA(cudaMemcpy(c->d_lists, lists.data(), lists.size() * sizeof(HqGemmJob*), cudaMemcpyHostToDevice));
  HQ_CUDA(cudaMemset(c->d_ctl, 0, size_t(c->nctl) * sizeof(int)));
  HQ_CUDA(cudaMalloc(&c->d_clk, HQ_PHASES * sizeof(unsigned long long)));
  HQ_CUDA(cudaMemset(c->d_clk, 0, HQ_PHASES * sizeof(unsigned long long)));
  c->sweep_capable = true;
}

// launch classes of the per-launch timing (hq_profile_collect)
enum ProfClass { PC_INTERVAL = 0, PC_BCHAIN, PC_UDT, PC_GEMM, PC_INVERT, PC_MEASURE, PC_DYN, PC_ADJ, PC_INTERVAL_CL,
                 PC_SWEEP, PC_COUNT };

struct ProfScope {
  hq_ctx* c;
  size_t idx;
  ProfScope(hq_ctx* c_, int cls) : c(c_), idx(size_t(-1)) {
    if (!c->profiling) return;
    if (c->prof_next == c->prof.size()) {
      hq_ctx::ProfEv e{cls, nullptr, nullptr};
      HQ_CUDA(cudaEventCreate(&e.e0));
      HQ_CUDA(cudaEventCreate(&e.e1));
      c->prof.push_back(e);
    }
    idx = c->prof_next++;
    c->prof[idx].cls = cls;
    // inside a stream capture the records become graph nodes (external events); outside
    // one they are plain records
    st = c->cur_st ? c->cur_st : c->stream;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    HQ_CUDA(cudaStreamIsCapturing(st, &cs));
    capturing = cs == cudaStreamCaptureStatusActive;
    if (capturing) HQ_CUDA(cudaEventRecordWithFlags(c->prof[idx].e0, st, cudaEventRecordExternal));
    else HQ_CUDA(cudaEventRecord(c->prof[idx].e0, st));
  }
  ~ProfScope() {
    if (idx == size_t(-1)) return;
    if (capturing) cudaEventRecordWithFlags(c->prof[idx].e1, st, cudaEventRecordExternal);
    else cudaEventRecord(c->prof[idx].e1, st);
  }
  cudaStream_t st = nullptr;
  bool capturing = false;
};

// the launch range of the current chain group
struct Cur {
  const HqChain* d;
  int n;
  cudaStream_t st;
};
Cur cur(hq_ctx* c) {
  if (!c->cur_st) return {c->d_desc, c->n, c->stream};
  return {c->d_desc + c->cur_c0, c->cur_n, c->cur_st};
}

void run_jobs(hq_ctx* c, int phase, int dir, int b) {
  ProfScope ps(c, PC_GEMM);
  auto it = c->jobs.find(std::make_tuple(phase, dir, b));
  if (it == c->jobs.end()) throw HqError(HQ_E_INVALID, "internal: missing job list");
  if (c->cur_st) {
    // per-chain phases hold one job per chain, in chain order
    if (it->second.second != c->n) throw HqError(HQ_E_INVALID, "internal: job list is not per chain");
    HQ_CUDA(hq::launch_gemm(it->second.first + c->cur_c0, c->cur_n, c->Nmax, c->Nmax, c->cur_st));
  } else {
    HQ_CUDA(hq::launch_gemm(it->second.first, it->second.second, c->Nmax, c->Nmax, c->stream));
  }
}

void upload_desc(hq_ctx* c) {
  HQ_CUDA(cudaStreamSynchronize(c->stream));  // no kernel of the stream may read the old descriptors
  HQ_CUDA(cudaMemcpy(c->d_desc, c->desc.data(), c->desc.size() * sizeof(HqChain), cudaMemcpyHostToDevice));
}

// whether the chains of the current group run their interval kernel on four-CTA clusters (and
// their B chain on four column blocks): every one of them has the 16 x 16 lattice with the
// separable expK and delay depth 16
bool interval_on_clusters(hq_ctx* c) {
  if (!c->cluster_interval) return false;
  const int c0 = c->cur_st ? c->cur_c0 : 0, n = c->cur_st ? c->cur_n : c->n;
  for (int i = c0; i < c0 + n; ++i) {
    const HqChain& d = c->desc[i];
    if (!hq::interval_cluster_ok(d.N, d.L, d.expk_mode, d.kmax)) return false;
  }
  return true;
}

// one stack push of interval b: bchain -> UDV -> cumulative Vt
void push_step(hq_ctx* c, int dir_kernel, int dir_jobs, int b) {
  const Cur g = cur(c);
  {
    ProfScope ps(c, PC_BCHAIN);
    if (interval_on_clusters(c)) HQ_CUDA(hq::launch_bchain_cols(g.d, g.n, dir_kernel, b, g.st));
    else HQ_CUDA(hq::launch_bchain(g.d, g.n, dir_kernel, b, c->Nmax, c->resident, g.st));
  }
  const int side = (dir_kernel == HQ_DOWN) ? 1 : 0;
  { ProfScope ps(c, PC_UDT); HQ_CUDA(hq::launch_udt(g.d, g.n, side, b, c->Nmax, c->resident, g.st)); }
  run_jobs(c, PH_PUSH, dir_jobs, b);
}

void builder_equaltime(hq_ctx* c, int dir_jobs, int b) {
  const Cur g = cur(c);
  run_jobs(c, PH_B1, dir_jobs, b);
  run_jobs(c, PH_B2, dir_jobs, b);
  { ProfScope ps(c, PC_INVERT); HQ_CUDA(hq::launch_invert(g.d, g.n, b, 0, c->Nmax, c->resident, g.st)); }
  run_jobs(c, PH_B3, dir_jobs, b);
  run_jobs(c, PH_B4, dir_jobs, b);
}

// Runs body() once per chain group, each group on its own stream forked from the main
// stream, and joins the groups back into the main stream. One group's launches fill the
// SMs that the other's last wave leaves idle. With one group body() runs on the main stream.
template <class F>
void in_groups(hq_ctx* c, F&& body) {
  const int G = c->ngroups;
  if (G > 1) {
    HQ_CUDA(cudaEventRecord(c->ev_fork, c->stream));
    for (int g = 1; g < G; ++g) HQ_CUDA(cudaStreamWaitEvent(c->gstream[g], c->ev_fork, 0));
  }
  for (int g = 0; g < G; ++g) {
    if (G > 1) {
      c->cur_c0 = c->gbeg[g];
      c->cur_n = c->gbeg[g + 1] - c->gbeg[g];
      c->cur_st = c->gstream[g];
    }
    body();
  }
  c->cur_st = nullptr;
  if (G > 1) {
    for (int g = 1; g < G; ++g) {
      HQ_CUDA(cudaEventRecord(c->ev_join[g], c->gstream[g]));
      HQ_CUDA(cudaStreamWaitEvent(c->stream, c->ev_join[g], 0));
    }
  }
}

void issue_sweep(hq_ctx* c, int dir, int flags) {
  c->prof_next = 0;
  const int kf = flags & (HQ_F_MEASURE | HQ_F_SNAPSHOT | HQ_F_LOG_RATIOS);
  if ((dir == HQ_UP || dir == HQ_DOWN) && c->sweep_mode == HQ_SWEEP_PERSISTENT) {
    ProfScope ps(c, PC_SWEEP);
    HQ_CUDA(hq::launch_sweep(c->d_desc, c->n, c->d_items, c->nitems, c->d_lists, c->nstab_max, dir,
                             kf | (flags & HQ_F_PHASE_CLOCKS), c->d_ctl, c->d_clk, c->sweep_grid, c->Nmax,
                             c->kmax_max, c->stream));
    return;
  }
  if (dir == HQ_UP || dir == HQ_DOWN) {
    in_groups(c, [&] {
      const Cur gr = cur(c);
      for (int b = 0; b < c->nstab_max; ++b) {
        if (interval_on_clusters(c)) {
          ProfScope ps(c, PC_INTERVAL_CL);
          HQ_CUDA(hq::launch_interval_cl(gr.d, gr.n, dir, b, kf, gr.st));
        } else {
          ProfScope ps(c, PC_INTERVAL);
          HQ_CUDA(hq::launch_interval(gr.d, gr.n, dir, b, kf, c->Nmax, c->kmax_max, c->resident, gr.st));
        }
        push_step(c, dir, dir, b);
        builder_equaltime(c, dir, b);
        if (kf & (HQ_F_MEASURE | HQ_F_SNAPSHOT)) { ProfScope ps(c, PC_MEASURE); HQ_CUDA(hq::launch_measure(gr.d, gr.n, dir, b, kf, gr.st)); }
      }
    });
  } else {
    { ProfScope ps(c, PC_DYN); HQ_CUDA(hq::launch_dyn_start(c->d_desc, c->n, c->stream)); }
    for (int b = 0; b < c->nstab_max; ++b) {
      { ProfScope ps(c, PC_DYN); HQ_CUDA(hq::launch_dyn_slices(c->d_desc, c->n, b, kf, c->Nmax, c->resident, c->stream)); }
      push_step(c, HQ_UP, 3, b);
      run_jobs(c, PH_B1, 3, b);
      run_jobs(c, PH_B2, 3, b);
      { ProfScope ps(c, PC_INVERT); HQ_CUDA(hq::launch_invert(c->d_desc, c->n, b, 0, c->Nmax, c->resident, c->stream)); }
      run_jobs(c, PH_B3, 3, b);   // W2 = Y = T1^-1 dlmax^-1 U_L^T
      run_jobs(c, PH_D3, 3, b);   // W3 = G(t,t)
      run_jobs(c, PH_D4, 3, b);   // W5 = T1^-1 dlmin Vt_L
      run_jobs(c, PH_D5, 3, b);   // W0 = G(t,0)
      run_jobs(c, PH_D6, 3, b);   // W4 = G(0,t)
      { ProfScope ps(c, PC_DYN); HQ_CUDA(hq::launch_dyn_commit(c->d_desc, c->n, b, c->stream)); }
      { ProfScope ps(c, PC_DYN); HQ_CUDA(hq::launch_dyn_store(c->d_desc, c->n, b, c->stream)); }
      { ProfScope ps(c, PC_DYN); HQ_CUDA(hq::launch_dyn_measure(c->d_desc, c->n, b, 0, c->stream)); }
    }
  }
}

void check_chain(hq_ctx* c, int chain) {
  if (!c) throw HqError(HQ_E_INVALID, "null context");
  if (chain < 0 || chain >= c->n) throw HqError(HQ_E_RANGE, "chain index out of range");
}

int fail(const HqError& e) {
  g_last_error = e.what();
  return e.code;
}

#define HQ_API_BEGIN try {
#define HQ_API_END                                                     \
  }                                                                    \
  catch (const HqError& e) { return fail(e); }                         \
  catch (const std::bad_alloc&) { g_last_error = "host allocation failed"; return HQ_E_NOMEM; } \
  catch (const std::exception& e) { g_last_error = e.what(); return HQ_E_INVALID; }          \
  return HQ_OK;

}  // namespace

// =======================================================================================
//  C ABI
// =======================================================================================
extern "C" {

int hq_last_error(char* buf, size_t len) {
  if (!buf || len == 0) return HQ_E_INVALID;
  std::snprintf(buf, len, "%s", g_last_error.c_str());
  return HQ_OK;
}

int hq_create(int device, int n_chains, const hq_chain_params* params, hq_ctx** out) {
  HQ_API_BEGIN
  if (!out || !params || n_chains <= 0) throw HqError(HQ_E_INVALID, "hq_create: invalid arguments");
  *out = nullptr;
  auto c = std::make_unique<hq_ctx>();
  c->device = device;
  HQ_CUDA(cudaSetDevice(device));
  HQ_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  c->n = n_chains;
  c->ch.resize(n_chains);
  c->desc.resize(n_chains);
  // ---- validation (include/dqmc_parser.hpp:124-132) and per-chain constants ----
  for (int i = 0; i < n_chains; ++i) {
    const hq_chain_params& p = params[i];
    if (p.u < 0) throw HqError(HQ_E_INVALID, "'u' out of range");
    if (p.nl < 1) throw HqError(HQ_E_INVALID, "'nl' out of range");
    if (p.beta < 0) throw HqError(HQ_E_INVALID, "'beta' out of range");
    if (p.nt < 1) throw HqError(HQ_E_INVALID, "'nt' out of range");
    if (p.stabilization_pace < 1) throw HqError(HQ_E_INVALID, "'stabilization_pace' out of range");
    if (p.nl * p.nl > HQ_MAX_N) throw HqError(HQ_E_INVALID, "lattice too large (N > 1024)");
    ChainHost& h = c->ch[i];
    h.p = p;
    h.N = p.nl * p.nl;
    h.n_stab = (p.nt % p.stabilization_pace == 0) ? p.nt / p.stabilization_pace : p.nt / p.stabilization_pace + 1;
    h.dt = p.beta / p.nt;                        // include/dqmc_parser.hpp:88
    h.alpha = std::acosh(std::exp(0.5 * h.dt * p.u));  // src/hubbard.cpp:35
    h.expk_mode = p.expk_mode;
    if (h.expk_mode == HQ_EXPK_AUTO) h.expk_mode = (p.nl >= 4 && p.nl <= HQ_MAX_L) ? HQ_EXPK_SEPARABLE : HQ_EXPK_DENSE;
    if (p.nl > HQ_MAX_L) h.expk_mode = HQ_EXPK_DENSE;
    c->Nmax = std::max(c->Nmax, h.N);
    c->ntmax = std::max(c->ntmax, p.nt);
    c->nstab_max = std::max(c->nstab_max, h.n_stab);
    if (p.dynamic) c->has_dynamic = true;
  }
  // ---- delay depth and shared-memory residency ----
  int smem_optin = 0;
  HQ_CUDA(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
  const size_t optin = size_t(smem_optin);
  c->resident = hq::matrices_fit(c->Nmax, optin);
  int kfit = 4;
  for (int k : {16, 8, 4})
    if (hq::interval_fits(c->Nmax, k, c->resident, optin)) { kfit = k; break; }
  for (int i = 0; i < n_chains; ++i) {
    ChainHost& h = c->ch[i];
    // the delay depth is the site-block size of the submatrix updates: 4, 8 or 16
    const int want = h.p.delay_depth > 0 ? std::min(h.p.delay_depth, kfit) : kfit;
    h.kmax = want >= 16 ? 16 : (want >= 8 ? 8 : 4);
    c->kmax_max = std::max(c->kmax_max, h.kmax);
  }
  if (!hq::interval_fits(c->Nmax, c->kmax_max, c->resident, optin))
    throw HqError(HQ_E_INVALID, "delay depth does not fit in shared memory");
  // chain groups on forked streams (see in_groups)
  // HQ_CHAIN_GROUPS=1 keeps every launch on the context stream (kernel durations without the
  // other group's kernels beside them, for measurements)
  const char* genv = std::getenv("HQ_CHAIN_GROUPS");
  const bool single_group = genv && std::strcmp(genv, "1") == 0;
  if (n_chains >= 32 && !single_group) {
    c->ngroups = c->resident ? 2 : hq_ctx::kGroups;
    if (n_chains < 16 * c->ngroups) c->ngroups = 2;
    // group boundaries at equal estimated work (nt N^3 per chain: the slices' wraps and
    // flushes and the stabilisations' factorisations and products all scale so), so that
    // uneven chains do not leave one group running alone
    std::vector<double> pre(n_chains + 1, 0.0);
    for (int i = 0; i < n_chains; ++i) {
      const double N = c->ch[i].N;
      pre[i + 1] = pre[i] + double(c->ch[i].p.nt) * N * N * N;
    }
    c->gbeg[0] = 0;
    for (int g = 1; g < c->ngroups; ++g) {
      const double target = pre[n_chains] * g / c->ngroups;
      int k = c->gbeg[g - 1] + 1;
      while (k < n_chains - (c->ngroups - g) && pre[k] < target) ++k;
      c->gbeg[g] = k;
    }
    c->gbeg[c->ngroups] = n_chains;
    c->gstream[0] = c->stream;
    for (int g = 1; g < c->ngroups; ++g) HQ_CUDA(cudaStreamCreateWithFlags(&c->gstream[g], cudaStreamNonBlocking));
    HQ_CUDA(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
    for (int g = 0; g < c->ngroups; ++g) HQ_CUDA(cudaEventCreateWithFlags(&c->ev_join[g], cudaEventDisableTiming));
  }
  // ---- arena layout ----
  struct Off { size_t G, Gt0, G0t, fields, rng, X, sU, sD, sVt, W[6], stt, st0, s0t, acc, dyn, rcount; };
  std::vector<Off> offs(n_chains);
  size_t total = 0;
  auto take = [&](size_t bytes) { const size_t o = total; total += align256(bytes); return o; };
  for (int i = 0; i < n_chains; ++i) {
    const ChainHost& h = c->ch[i];
    const size_t NN = size_t(h.N) * h.N * sizeof(double);
    Off& o = offs[i];
    o.G = take(NN);
    o.Gt0 = h.p.dynamic ? take(NN) : 0;
    o.G0t = h.p.dynamic ? take(NN) : 0;
    o.fields = take(size_t(h.p.nt) * h.N);
    o.rng = take(sizeof(uint32_t));
    o.X = take(NN);
    o.sU = take(2 * size_t(h.n_stab) * NN);
    o.sD = take(2 * size_t(h.n_stab) * h.N * sizeof(double));
    o.sVt = take(2 * size_t(h.n_stab) * NN);
    for (int w = 0; w < 6; ++w) o.W[w] = take(NN);
    o.stt = h.p.snapshots ? take(size_t(h.p.nt) * NN) : 0;
    o.st0 = h.p.dynamic ? take(size_t(h.p.nt) * NN) : 0;
    o.s0t = h.p.dynamic ? take(size_t(h.p.nt) * NN) : 0;
    o.acc = take(HQ_ACC_COUNT * sizeof(double));
    o.dyn = take(size_t(2 + h.N) * h.p.nt * sizeof(double));
    o.rcount = take(sizeof(long long));
  }
  // identity / ones per distinct N
  std::map<int, std::pair<size_t, size_t>> ioffs;
  for (int i = 0; i < n_chains; ++i) {
    const int N = c->ch[i].N;
    if (!ioffs.count(N)) ioffs[N] = {take(size_t(N) * N * sizeof(double)), take(size_t(N) * sizeof(double))};
  }
  // dense expK per distinct parameter set
  std::map<std::tuple<int, double, double, double>, size_t> eoffs;
  for (int i = 0; i < n_chains; ++i) {
    const ChainHost& h = c->ch[i];
    auto key = std::make_tuple(h.p.nl, h.dt, h.p.nnt, h.p.mu);
    if (!eoffs.count(key)) eoffs[key] = take(2 * size_t(h.N) * h.N * sizeof(double));
  }
  c->arena_bytes = total;
  if (cudaMalloc(&c->arena, total) != cudaSuccess) {
    cudaGetLastError();
    throw HqError(HQ_E_NOMEM, "device arena allocation of " + std::to_string(total) + " bytes failed");
  }
  HQ_CUDA(cudaMemsetAsync(c->arena, 0, total, c->stream));
  HQ_CUDA(cudaStreamSynchronize(c->stream));
  char* A = c->arena;
  for (auto& kv : ioffs) {
    const int N = kv.first;
    std::vector<double> I(size_t(N) * N, 0.0), one(N, 1.0);
    for (int k = 0; k < N; ++k) I[k + size_t(k) * N] = 1.0;
    HQ_CUDA(cudaMemcpyAsync(A + kv.second.first, I.data(), I.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    HQ_CUDA(cudaMemcpyAsync(A + kv.second.second, one.data(), N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    c->ident[N] = {reinterpret_cast<double*>(A + kv.second.first), reinterpret_cast<double*>(A + kv.second.second)};
  }
  for (auto& kv : eoffs) {
    int L; double dt, t, mu;
    std::tie(L, dt, t, mu) = kv.first;
    const int N = L * L;
    std::vector<double> a(L), ai(L), E(size_t(N) * N), Ei(size_t(N) * N);
    circulant_exp(L, dt * t, a.data());
    circulant_exp(L, -dt * t, ai.data());
    const double ce = std::exp(dt * mu), cei = std::exp(-dt * mu);
    for (int j = 0; j < N; ++j)
      for (int i = 0; i < N; ++i) {
        const int dx = ((i % L) - (j % L) + L) % L, dy = ((i / L) - (j / L) + L) % L;
        E[i + size_t(j) * N] = ce * a[dx] * a[dy];
        Ei[i + size_t(j) * N] = cei * ai[dx] * ai[dy];
      }
    HQ_CUDA(cudaMemcpy(A + kv.second, E.data(), E.size() * sizeof(double), cudaMemcpyHostToDevice));
    HQ_CUDA(cudaMemcpy(A + kv.second + E.size() * sizeof(double), Ei.data(), Ei.size() * sizeof(double),
                       cudaMemcpyHostToDevice));
  }
  for (int i = 0; i < n_chains; ++i) {
    ChainHost& h = c->ch[i];
    HqChain& d = c->desc[i];
    std::memset(&d, 0, sizeof(d));
    const Off& o = offs[i];
    d.N = h.N; d.L = h.p.nl; d.nt = h.p.nt; d.pace = h.p.stabilization_pace; d.n_stab = h.n_stab;
    d.expk_mode = h.expk_mode; d.kmax = h.kmax; d.active = 1;
    d.alpha = h.alpha; d.dt = h.dt;
    d.delta_p = std::exp(-2 * h.alpha * (+1)) - 1;  // src/hubbard.cpp:128
    d.delta_m = std::exp(-2 * h.alpha * (-1)) - 1;
    d.ev_p = std::exp(h.alpha);
    d.ev_m = std::exp(-h.alpha);
    d.sep_c = std::exp(h.dt * h.p.mu);
    d.sep_ci = std::exp(-h.dt * h.p.mu);
    if (h.p.nl <= HQ_MAX_L) {
      circulant_exp(h.p.nl, h.dt * h.p.nnt, d.sep_a);
      circulant_exp(h.p.nl, -h.dt * h.p.nnt, d.sep_ai);
    }
    const size_t eo = eoffs[std::make_tuple(h.p.nl, h.dt, h.p.nnt, h.p.mu)];
    d.expK = reinterpret_cast<const double*>(A + eo);
    d.inv_expK = reinterpret_cast<const double*>(A + eo) + size_t(h.N) * h.N;
    d.G = reinterpret_cast<double*>(A + o.G);
    d.Gt0 = h.p.dynamic ? reinterpret_cast<double*>(A + o.Gt0) : nullptr;
    d.G0t = h.p.dynamic ? reinterpret_cast<double*>(A + o.G0t) : nullptr;
    d.fields = reinterpret_cast<int8_t*>(A + o.fields);
    d.rng = reinterpret_cast<uint32_t*>(A + o.rng);
    d.X = reinterpret_cast<double*>(A + o.X);
    d.stackU = reinterpret_cast<double*>(A + o.sU);
    d.stackD = reinterpret_cast<double*>(A + o.sD);
    d.stackVt = reinterpret_cast<double*>(A + o.sVt);
    double** W[6] = {&d.W0, &d.W1, &d.W2, &d.W3, &d.W4, &d.W5};
    for (int w = 0; w < 6; ++w) *W[w] = reinterpret_cast<double*>(A + o.W[w]);
    d.snap_tt = h.p.snapshots ? reinterpret_cast<double*>(A + o.stt) : nullptr;
    d.snap_t0 = h.p.dynamic ? reinterpret_cast<double*>(A + o.st0) : nullptr;
    d.snap_0t = h.p.dynamic ? reinterpret_cast<double*>(A + o.s0t) : nullptr;
    d.acc = reinterpret_cast<double*>(A + o.acc);
    d.dyn_acc = reinterpret_cast<double*>(A + o.dyn);
    d.ratio_count = reinterpret_cast<long long*>(A + o.rcount);
    d.ratios = nullptr;
    d.ratio_cap = 0;
    // nearest-neighbour hopping matrix (src/square_lattice.cpp:48-61) and K
    const int L = h.p.nl;
    h.hop.assign(size_t(h.N) * h.N, 0.0);
    for (int s = 0; s < h.N; ++s) {
      const int x = s % L, y = s / L;
      const int xp = (x + 1) % L + L * y, yp = x + L * ((y + 1) % L);
      h.hop[s + size_t(xp) * h.N] += 1.0; h.hop[xp + size_t(s) * h.N] += 1.0;
      h.hop[s + size_t(yp) * h.N] += 1.0; h.hop[yp + size_t(s) * h.N] += 1.0;
    }
    h.K.assign(size_t(h.N) * h.N, 0.0);
    for (size_t k = 0; k < h.K.size(); ++k) h.K[k] = -h.p.nnt * h.hop[k];
    for (int s = 0; s < h.N; ++s) h.K[s + size_t(s) * h.N] -= h.p.mu;
  }
  c->desc.shrink_to_fit();
  HQ_CUDA(hq::prepare_kernels(c->Nmax, c->kmax_max, c->resident));
  // chains too large for one SM: the interval kernel of 16 x 16 lattices runs on four-CTA
  // clusters with G in their distributed shared memory (HQ_INTERVAL_CLUSTER=0 keeps the
  // global-memory path, for comparisons)
  if (!c->resident) {
    const char* env = std::getenv("HQ_INTERVAL_CLUSTER");
    bool any = false;
    for (int i = 0; i < n_chains; ++i) any = any || (c->ch[i].N == 256 && c->ch[i].p.nl == 16);
    if (any && !(env && std::strcmp(env, "0") == 0)) {
      HQ_CUDA(hq::prepare_interval_cl());
      c->cluster_capable = hq::interval_cl_max_clusters() > 0;
      c->cluster_interval = c->cluster_capable;
    }
  }
  HQ_CUDA(cudaMalloc(&c->d_desc, c->desc.size() * sizeof(HqChain)));
  // the gather buffers of hq_get_estimators_all, so that no read allocates
  HQ_CUDA(cudaMalloc(&c->d_acc_all, size_t(c->n) * HQ_ACC_COUNT * sizeof(double)));
  HQ_CUDA(cudaMallocHost(&c->h_acc_all, size_t(c->n) * HQ_ACC_COUNT * sizeof(double)));
  upload_desc(c.get());
  build_jobs(c.get());
  if (c->resident && hq::sweep_fits(c->Nmax, c->kmax_max, optin)) {
    setup_sweep(c.get());
    // HQ_SWEEP_MODE=persistent | launches overrides the default mode (for comparisons)
    const char* m = std::getenv("HQ_SWEEP_MODE");
    if (m && std::strcmp(m, "persistent") == 0) c->sweep_mode = HQ_SWEEP_PERSISTENT;
    if (m && std::strcmp(m, "launches") == 0) c->sweep_mode = HQ_SWEEP_LAUNCHES;
  }
  HQ_CUDA(cudaStreamSynchronize(c->stream));
  *out = c.release();
  HQ_API_END
}

int hq_destroy(hq_ctx* ctx) {
  HQ_API_BEGIN
  delete ctx;
  HQ_API_END
}

int hq_set_hopping(hq_ctx* c, int chain, const double* hop) {
  HQ_API_BEGIN
  check_chain(c, chain);
  if (!hop) throw HqError(HQ_E_INVALID, "null hopping matrix");
  ChainHost& h = c->ch[chain];
  const int N = h.N;
  h.hop.assign(hop, hop + size_t(N) * N);
  h.custom_hop = true;
  h.K.assign(size_t(N) * N, 0.0);
  for (size_t k = 0; k < h.K.size(); ++k) h.K[k] = -h.hop[k];
  for (int s = 0; s < N; ++s) h.K[s + size_t(s) * N] -= h.p.mu;
  // exp(-+dt K) through the eigen-decomposition of the symmetric K
  std::vector<double> w, Q;
  jacobi_eig(N, h.K, w, Q);
  std::vector<double> E(size_t(N) * N), Ei(size_t(N) * N), QE(size_t(N) * N), QEi(size_t(N) * N);
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < N; ++i) {
      QE[i + size_t(j) * N] = Q[i + size_t(j) * N] * std::exp(-h.dt * w[j]);
      QEi[i + size_t(j) * N] = Q[i + size_t(j) * N] * std::exp(h.dt * w[j]);
    }
  host_gemm(N, QE.data(), false, Q.data(), true, E.data());
  host_gemm(N, QEi.data(), false, Q.data(), true, Ei.data());
  double* dE = nullptr;
  HQ_CUDA(cudaMalloc(&dE, 2 * E.size() * sizeof(double)));
  c->extra_allocs.push_back(dE);
  HQ_CUDA(cudaMemcpy(dE, E.data(), E.size() * sizeof(double), cudaMemcpyHostToDevice));
  HQ_CUDA(cudaMemcpy(dE + E.size(), Ei.data(), Ei.size() * sizeof(double), cudaMemcpyHostToDevice));
  HqChain& d = c->desc[chain];
  d.expK = dE;
  d.inv_expK = dE + E.size();
  d.expk_mode = HQ_EXPK_DENSE;
  h.expk_mode = HQ_EXPK_DENSE;
  upload_desc(c);
  for (auto& g : c->graphs) cudaGraphExecDestroy(g.second);
  c->graphs.clear();
  HQ_API_END
}

int hq_fields_random(hq_ctx* c, int chain) {
  HQ_API_BEGIN
  check_chain(c, chain);
  ChainHost& h = c->ch[chain];
  // src/hubbard.cpp:102-110: for t, for i: bernoulli(0.5) ? +1 : -1
  uint32_t x = minstd_seed(h.p.seed);
  std::vector<int8_t> f(size_t(h.p.nt) * h.N);
  for (size_t k = 0; k < f.size(); ++k) f[k] = canonical(x) < 0.5 ? 1 : -1;
  HqChain& d = c->desc[chain];
  HQ_CUDA(cudaMemcpyAsync(d.fields, f.data(), f.size(), cudaMemcpyHostToDevice, c->stream));
  h.rng_after_fields = x;
  HQ_CUDA(cudaMemcpyAsync(d.rng, &h.rng_after_fields, sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream));
  HQ_CUDA(cudaStreamSynchronize(c->stream));
  h.fields_set = true;
  c->initialised = false;
  HQ_API_END
}

int hq_set_fields(hq_ctx* c, int chain, const int* fields) {
  HQ_API_BEGIN
  check_chain(c, chain);
  if (!fields) throw HqError(HQ_E_INVALID, "null fields");
  ChainHost& h = c->ch[chain];
  std::vector<int8_t> f(size_t(h.p.nt) * h.N);
  for (size_t k = 0; k < f.size(); ++k) {
    if (fields[k] != 1 && fields[k] != -1) throw HqError(HQ_E_INVALID, "Ising fields must be +1 or -1");
    f[k] = static_cast<int8_t>(fields[k]);
  }
  HqChain& d = c->desc[chain];
  HQ_CUDA(cudaMemcpyAsync(d.fields, f.data(), f.size(), cudaMemcpyHostToDevice, c->stream));
  if (!h.fields_set) {
    // the engine continues from the seeded stream when fields are loaded from a file
    h.rng_after_fields = minstd_seed(h.p.seed);
    HQ_CUDA(cudaMemcpyAsync(d.rng, &h.rng_after_fields, sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream));
  }
  HQ_CUDA(cudaStreamSynchronize(c->stream));
  h.fields_set = true;
  c->initialised = false;
  HQ_API_END
}

int hq_get_fields(hq_ctx* c, int chain, int* fields) {
  HQ_API_BEGIN
  check_chain(c, chain);
  if (!fields) throw HqError(HQ_E_INVALID, "null fields");
  ChainHost& h = c->ch[chain];
  std::vector<int8_t> f(size_t(h.p.nt) * h.N);
  HQ_CUDA(cudaMemcpyAsync(f.data(), c->desc[chain].fields, f.size(), cudaMemcpyDeviceToHost, c->stream));
  HQ_CUDA(cudaStreamSynchronize(c->stream));
  for (size_t k = 0; k < f.size(); ++k) fields[k] = f[k];
  HQ_API_END
}

// State word of a chain's minstd_rand0 engine (the reference's Utils::Random engine,
// src/random.cpp:14-15): saved with the fields it makes a checkpoint from which the chain
// continues exactly (fields, then this word, then hq_init_stacks_and_g).
int hq_get_rng_state(hq_ctx* c, int chain, unsigned int* state) {
  HQ_API_BEGIN
  check_chain(c, chain);
  if (!state) throw HqError(HQ_E_INVALID, "null state");
  uint32_t v = 0;
  HQ_CUDA(cudaMemcpyAsync(&v, c->desc[chain].rng, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
  HQ_CUDA(cudaStreamSynchronize(c->stream));
  *state = v;
  HQ_API_END
}

int hq_set_rng_state(hq_ctx* c, int chain, unsigned int state) {
  HQ_API_BEGIN
  check_chain(c, chain);
  if (state == 0u || state >= 2147483647u) throw HqError(HQ_E_RANGE, "minstd_rand0 state must be in [1, 2147483646]");
  uint32_t v = state;
  HQ_CUDA(cudaMemcpyAsync(c->desc[chain].rng, &v, sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream));
  HQ_CUDA(cudaStreamSynchronize(c->stream));
  c->ch[chain].rng_after_fields = v;
  HQ_API_END
}

int hq_init_stacks_and_g(hq_ctx* c) {
  HQ_API_BEGIN
  if (!c) throw HqError(HQ_E_INVALID, "null context");
  for (auto& h : c->ch)
    if (!h.fields_set) throw HqError(HQ_E_INVALID, "fields of a chain are not set (hq_fields_random / hq_set_fields)");
  c->prof_next = 0;
  // builder with each chain's full right stack: the dir-2 job list at b = n_stab-1 of each chain.
  // Chains of different n_stab need their own b; issue one launch per distinct n_stab.
  std::vector<int> nstabs;
  for (auto& h : c->ch) nstabs.push_back(h.n_stab);
  std::sort(nstabs.begin(), nstabs.end());
  nstabs.erase(std::unique(nstabs.begin(), nstabs.end()), nstabs.end());
  in_groups(c, [&] {
    // src/dqmc_core.cpp:67-87: right stack from t = nt down to 1 with B^T, push every pace
    for (int b = 0; b < c->nstab_max; ++b) push_step(c, HQ_DOWN, 2, b);
    // src/dqmc_core.cpp:89-97: G(0,0) from (empty left, full right)
    if (nstabs.size() == 1) builder_equaltime(c, 2, nstabs[0] - 1);
  });
  if (nstabs.size() > 1) {
    for (int ns : nstabs) {
      // deactivate chains with other stack lengths for this pass
      std::vector<HqChain> saved = c->desc;
      for (int i = 0; i < c->n; ++i) c->desc[i].active = (c->ch[i].n_stab == ns) ? 1 : 0;
      upload_desc(c);
      builder_equaltime(c, 2, ns - 1);
      HQ_CUDA(cudaStreamSynchronize(c->stream));
      c->desc = saved;
      upload_desc(c);
    }
  }
  HQ_CUDA(cudaStreamSynchronize(c->stream));
  c->at_zero = true;
  c->at_beta = false;
  c->initialised = true;
  HQ_API_END
}

// one directional sweep through its captured graph when there is one
static void dispatch_sweep(hq_ctx* c, int dir, int flags) {
  auto it = c->graphs.find({dir, flags});
  if (it != c->graphs.end()) {
    HQ_CUDA(cudaGraphLaunch(it->second, c->stream));
    c->prof_next = c->graph_prof[{dir, flags}];
  } else {
    issue_sweep(c, dir, flags);
  }
  c->at_zero = (dir == HQ_SWEEP_DOWN);
  c->at_beta = !c->at_zero;
}

int hq_sweep(hq_ctx* c, int dir, int flags) {
  HQ_API_BEGIN
  if (!c) throw HqError(HQ_E_INVALID, "null context");
  if (!c->initialised) throw HqError(HQ_E_INVALID, "hq_sweep: call hq_init_stacks_and_g first");
  if (dir == HQ_SWEEP_UP || dir == HQ_SWEEP_DYNAMIC) {
    if (!c->at_zero) throw HqError(HQ_E_INVALID, "sweep from 0 to beta: stacks are not at tau = 0");
  } else if (dir == HQ_SWEEP_DOWN) {
    if (!c->at_beta) throw HqError(HQ_E_INVALID, "sweep from beta to 0: stacks are not at tau = beta");
  } else {
    throw HqError(HQ_E_INVALID, "unknown sweep direction");
  }
  if (dir == HQ_SWEEP_DYNAMIC && !c->has_dynamic) throw HqError(HQ_E_INVALID, "context created without dynamic storage");
  if (dir == HQ_SWEEP_DYNAMIC) {
    for (auto& h : c->ch)
      if (!h.p.dynamic) throw HqError(HQ_E_INVALID, "every chain needs dynamic storage for a dynamic sweep");
  }
  dispatch_sweep(c, dir, flags);
  HQ_API_END
}

int hq_sync(hq_ctx* c) {
  HQ_API_BEGIN
  if (!c) throw HqError(HQ_E_INVALID, "null context");
  HQ_CUDA(cudaStreamSynchronize(c->stream));
  HQ_API_END
}

int hq_capture_graph(hq_ctx* c, int dir, int flags) {
  HQ_API_BEGIN
  if (!c) throw HqError(HQ_E_INVALID, "null context");
  if (dir < 0 || dir > 2) throw HqError(HQ_E_INVALID, "unknown sweep direction");
  auto it = c->graphs.find({dir, flags});
  if (it != c->graphs.end()) { cudaGraphExecDestroy(it->second); c->graphs.erase(it); }
  cudaGraph_t g;
  HQ_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  try {
    issue_sweep(c, dir, flags);
  } catch (...) {
    cudaStreamEndCapture(c->stream, &g);
    throw;
  }
  HQ_CUDA(cudaStreamEndCapture(c->stream, &g));
  cudaGraphExec_t ex;
  HQ_CUDA(cudaGraphInstantiate(&ex, g, 0));
  cudaGraphDestroy(g);
  c->graphs[{dir, flags}] = ex;
  c->graph_prof[{dir, flags}] = c->prof_next;
  HQ_API_END
}

int hq_launch_graph(hq_ctx* c, int dir) {
  HQ_API_BEGIN
  if (!c) throw HqError(HQ_E_INVALID, "null context");
  for (auto& kv : c->graphs)
    if (kv.first.first == dir) return hq_sweep(c, dir, kv.first.second);
  throw HqError(HQ_E_INVALID, "no graph captured for this direction");
  HQ_API_END
}

int hq_get_g(hq_ctx* c, int chain, int which, int slice, double* out) {
  HQ_API_BEGIN
  check_chain(c, chain);
  if (!out) throw HqError(HQ_E_INVALID, "null output");
  const HqChain& d = c->desc[chain];
  const size_t NN = size_t(d.N) * d.N;
  const double* src = nullptr;
  if (which == HQ_G_CURRENT) src = d.G;
  else {
    if (slice < 0 || slice >= d.nt) throw HqError(HQ_E_RANGE, "slice out of range");
    const double* base = which == HQ_G_TT ? d.snap_tt : which == HQ_G_T0 ? d.snap_t0 : which == HQ_G_0T ? d.snap_0t : nullptr;
    if (!base) throw HqError(HQ_E_INVALID, "requested Green's function storage was not allocated");
    src = base + size_t(slice) * NN;
  }
  HQ_CUDA(cudaMemcpyAsync(out, src, NN * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  HQ_CUDA(cudaStreamSynchronize(c->stream));
  HQ_API_END
}

int hq_set_g(hq_ctx* c, int chain, const double* in) {
  HQ_API_BEGIN
  check_chain(c, chain);
  if (!in) throw HqError(HQ_E_INVALID, "null input");
  const HqChain& d = c->desc[chain];
  HQ_CUDA(cudaMemcpyAsync(d.G, in, size_t(d.N) * d.N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  HQ_CUDA(cudaStreamSynchronize(c->stream));
  HQ_API_END
}

static void read_acc(hq_ctx* c, int chain, double* acc) {
  HQ_CUDA(cudaMemcpyAsync(acc, c->desc[chain].acc, HQ_ACC_COUNT * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  HQ_CUDA(cudaStreamSynchronize(c->stream));
}

int hq_get_wrap_errors(hq_ctx* c, int chain, double* out2) {
  HQ_API_BEGIN
  check_chain(c, chain);
  double acc[HQ_ACC_COUNT];
  read_acc(c, chain, acc);
  if (acc[HQ_ACC_STATUS] != 0.0) throw HqError(HQ_E_NUMERIC, "singular pivot or non-finite value in a G builder");
  out2[0] = acc[HQ_ACC_WRAP_TT];
  out2[1] = acc[HQ_ACC_WRAP_DYN];
  HQ_API_END
}

int hq_get_estimators(hq_ctx* c, int chain, double* out6) {
  HQ_API_BEGIN
  check_chain(c, chain);
  double acc[HQ_ACC_COUNT];
  read_acc(c, chain, acc);
  out6[0] = acc[HQ_ACC_FILLING];
  out6[1] = acc[HQ_ACC_DOCC];
  out6[2] = acc[HQ_ACC_SWAVE];
  out6[3] = acc[HQ_ACC_NSLICE];
  out6[4] = acc[HQ_ACC_PROPOSED];
  out6[5] = acc[HQ_ACC_ACCEPTED];
  HQ_API_END
}

int hq_get_estimators_all(hq_ctx* c, double* out) {
  HQ_API_BEGIN
  if (!c || !out) throw HqError(HQ_E_INVALID, "null argument");
  const size_t cnt = size_t(c->n) * HQ_ACC_COUNT;
  HQ_CUDA(hq::launch_gather_acc(c->d_desc, c->n, c->d_acc_all, c->stream));
  HQ_CUDA(cudaMemcpyAsync(c->h_acc_all, c->d_acc_all, cnt * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  HQ_CUDA(cudaStreamSynchronize(c->stream));
  for (int i = 0; i < c->n; ++i) {
    const double* acc = c->h_acc_all + size_t(i) * HQ_ACC_COUNT;
    double* o = out + size_t(i) * 6;
    o[0] = acc[HQ_ACC_FILLING];
    o[1] = acc[HQ_ACC_DOCC];
    o[2] = acc[HQ_ACC_SWAVE];
    o[3] = acc[HQ_ACC_NSLICE];
    o[4] = acc[HQ_ACC_PROPOSED];
    o[5] = acc[HQ_ACC_ACCEPTED];
  }
  HQ_API_END
}

int hq_get_dynamic_estimators(hq_ctx* c, int chain, double* spin, double* ldos, double* gd) {
  HQ_API_BEGIN
  check_chain(c, chain);
  const HqChain& d = c->desc[chain];
  std::vector<double> buf(size_t(2 + d.N) * d.nt);
  HQ_CUDA(cudaMemcpyAsync(buf.data(), d.dyn_acc, buf.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  HQ_CUDA(cudaStreamSynchronize(c->stream));
  if (spin) std::memcpy(spin, buf.data(), d.nt * sizeof(double));
  if (ldos) std::memcpy(ldos, buf.data() + d.nt, d.nt * sizeof(double));
  if (gd) std::memcpy(gd, buf.data() + 2 * d.nt, size_t(d.N) * d.nt * sizeof(double));
  HQ_API_END
}

int hq_reset_estimators(hq_ctx* c, int reset_wrap) {
  HQ_API_BEGIN
  if (!c) throw HqError(HQ_E_INVALID, "null context");
  for (int i = 0; i < c->n; ++i) {
    const HqChain& d = c->desc[i];
    double acc[HQ_ACC_COUNT];
    read_acc(c, i, acc);
    const double wtt = acc[HQ_ACC_WRAP_TT], wdy = acc[HQ_ACC_WRAP_DYN], st = acc[HQ_ACC_STATUS];
    std::memset(acc, 0, sizeof(acc));
    if (!reset_wrap) { acc[HQ_ACC_WRAP_TT] = wtt; acc[HQ_ACC_WRAP_DYN] = wdy; acc[HQ_ACC_STATUS] = st; }
    HQ_CUDA(cudaMemcpyAsync(d.acc, acc, sizeof(acc), cudaMemcpyHostToDevice, c->stream));
    HQ_CUDA(cudaMemsetAsync(d.dyn_acc, 0, size_t(2 + d.N) * d.nt * sizeof(double), c->stream));
  }
  HQ_CUDA(cudaStreamSynchronize(c->stream));
  HQ_API_END
}

int hq_ratio_log(hq_ctx* c, int chain, long long capacity, double* out, long long cap, long long* count) {
  HQ_API_BEGIN
  check_chain(c, chain);
  HqChain& d = c->desc[chain];
  if (!d.ratios && capacity > 0) {
    double* p = nullptr;
    HQ_CUDA(cudaMalloc(&p, size_t(capacity) * sizeof(double)));
    c->extra_allocs.push_back(p);
    d.ratios = p;
    d.ratio_cap = capacity;
    const long long zero = 0;
    HQ_CUDA(cudaStreamSynchronize(c->stream));
    HQ_CUDA(cudaMemcpy(d.ratio_count, &zero, sizeof(zero), cudaMemcpyHostToDevice));
    upload_desc(c);
    for (auto& g : c->graphs) cudaGraphExecDestroy(g.second);
    c->graphs.clear();
  }
  long long n = 0;
  HQ_CUDA(cudaMemcpyAsync(&n, d.ratio_count, sizeof(n), cudaMemcpyDeviceToHost, c->stream));
  HQ_CUDA(cudaStreamSynchronize(c->stream));
  if (count) *count = n;
  if (out && d.ratios) {
    const long long m = std::min(std::min(n, cap), d.ratio_cap);
    HQ_CUDA(cudaMemcpyAsync(out, d.ratios, size_t(m) * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    HQ_CUDA(cudaStreamSynchronize(c->stream));
  }
  HQ_API_END
}

int hq_get_stream(hq_ctx* c, void** stream) {
  HQ_API_BEGIN
  if (!c || !stream) throw HqError(HQ_E_INVALID, "null argument");
  *stream = reinterpret_cast<void*>(c->stream);
  HQ_API_END
}

int hq_profile_enable(hq_ctx* c, int on) {
  HQ_API_BEGIN
  if (!c) throw HqError(HQ_E_INVALID, "null context");
  HQ_CUDA(cudaStreamSynchronize(c->stream));
  c->profiling = on != 0;
  c->prof_next = 0;
  for (auto& g : c->graphs) cudaGraphExecDestroy(g.second);
  c->graphs.clear();
  HQ_API_END
}

int hq_profile_collect(hq_ctx* c, double* ms, long long* counts, int nclasses) {
  HQ_API_BEGIN
  if (!c || !ms || !counts) throw HqError(HQ_E_INVALID, "null argument");
  HQ_CUDA(cudaStreamSynchronize(c->stream));
  for (size_t k = 0; k < c->prof_next && k < c->prof.size(); ++k) {
    const auto& e = c->prof[k];
    float t = 0.f;
    HQ_CUDA(cudaEventElapsedTime(&t, e.e0, e.e1));
    if (e.cls < nclasses) { ms[e.cls] += t; counts[e.cls] += 1; }
  }
  HQ_API_END
}

int hq_get_config(hq_ctx* c, int chain, int* expk_mode, int* delay_depth) {
  HQ_API_BEGIN
  check_chain(c, chain);
  if (expk_mode) *expk_mode = c->desc[chain].expk_mode;
  if (delay_depth) *delay_depth = c->desc[chain].kmax;
  HQ_API_END
}

// Top entry of a chain's UDV stack, the product U diag(D) V^T of all its pushes: the
// reference's SvdStack::MatrixU / SingularValues / MatrixV (include/utils/svd_stack.hpp:83-103).
// Between whole sweeps the stacks are either at tau = 0 (left empty, right full) or at
// tau = beta (left full, right empty).
int hq_set_sweep_mode(hq_ctx* c, int mode) {
  HQ_API_BEGIN
  if (!c) throw HqError(HQ_E_INVALID, "null context");
  if (mode != HQ_SWEEP_LAUNCHES && mode != HQ_SWEEP_PERSISTENT) throw HqError(HQ_E_INVALID, "unknown sweep mode");
  if (mode == HQ_SWEEP_PERSISTENT && !c->sweep_capable)
    throw HqError(HQ_E_RANGE, "persistent sweep: the chains' matrices do not fit in one SM's shared memory");
  HQ_CUDA(cudaStreamSynchronize(c->stream));
  c->sweep_mode = mode;
  for (auto& g : c->graphs) cudaGraphExecDestroy(g.second);
  c->graphs.clear();
  HQ_API_END
}

int hq_phase_cycles(hq_ctx* c, unsigned long long* out, int n, int reset) {
  HQ_API_BEGIN
  if (!c || (n > 0 && !out)) throw HqError(HQ_E_INVALID, "null argument");
  HQ_CUDA(cudaStreamSynchronize(c->stream));
  unsigned long long h[HQ_PHASES] = {};
  if (c->d_clk) HQ_CUDA(cudaMemcpy(h, c->d_clk, sizeof(h), cudaMemcpyDeviceToHost));
  for (int k = 0; k < n && k < HQ_PHASES; ++k) out[k] = h[k];
  if (reset && c->d_clk) HQ_CUDA(cudaMemset(c->d_clk, 0, sizeof(h)));
  HQ_API_END
}

int hq_get_sweep_mode(hq_ctx* c, int* mode) {
  HQ_API_BEGIN
  if (!c || !mode) throw HqError(HQ_E_INVALID, "null argument");
  *mode = c->sweep_mode;
  HQ_API_END
}

int hq_get_stack(hq_ctx* c, int chain, int side, int* length, double* U, double* D, double* V) {
  HQ_API_BEGIN
  check_chain(c, chain);
  if (side != 0 && side != 1) throw HqError(HQ_E_INVALID, "hq_get_stack: side is 0 (left) or 1 (right)");
  if (!c->initialised) throw HqError(HQ_E_INVALID, "hq_get_stack: call hq_init_stacks_and_g first");
  const HqChain& d = c->desc[chain];
  const int len = (side == 0) ? (c->at_beta ? d.n_stab : 0) : (c->at_zero ? d.n_stab : 0);
  if (length) *length = len;
  if (len > 0 && (U || D || V)) {
    const int N = d.N;
    const size_t NN = size_t(N) * N, e = size_t(side) * d.n_stab + (len - 1);
    HQ_CUDA(cudaStreamSynchronize(c->stream));
    if (U) HQ_CUDA(cudaMemcpy(U, d.stackU + e * NN, NN * sizeof(double), cudaMemcpyDeviceToHost));
    if (D) HQ_CUDA(cudaMemcpy(D, d.stackD + e * N, N * sizeof(double), cudaMemcpyDeviceToHost));
    if (V) {
      std::vector<double> vt(NN);
      HQ_CUDA(cudaMemcpy(vt.data(), d.stackVt + e * NN, NN * sizeof(double), cudaMemcpyDeviceToHost));
      for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) V[i + size_t(j) * N] = vt[j + size_t(i) * N];
    }
  }
  HQ_API_END
}

// Picks each lattice size's expK application (separable circulant passes or dense DMMA GEMM)
// and delay depth (submatrix block size) by timing whole directional sweeps of the context
// with each candidate. The device state is snapshotted before and restored after every
// candidate, so the chains continue exactly as if no tuning had run.
int hq_autotune(hq_ctx* c, int sweeps, hq_tune_entry* entries, int capacity, int* n_entries) {
  HQ_API_BEGIN
  if (!c) throw HqError(HQ_E_INVALID, "null context");
  if (!c->initialised) throw HqError(HQ_E_INVALID, "hq_autotune: call hq_init_stacks_and_g first");
  if (sweeps < 1 || sweeps > 64) throw HqError(HQ_E_RANGE, "hq_autotune: sweeps must be in [1, 64]");
  if (capacity < 0 || (capacity > 0 && !entries)) throw HqError(HQ_E_INVALID, "hq_autotune: bad entries buffer");
  std::map<int, std::vector<int>> groups;  // lattice size -> chains
  for (int i = 0; i < c->n; ++i) groups[c->ch[i].p.nl].push_back(i);
  char* snap = nullptr;
  if (cudaMalloc(&snap, c->arena_bytes) != cudaSuccess) {
    cudaGetLastError();
    throw HqError(HQ_E_NOMEM, "hq_autotune: no room for a snapshot of " + std::to_string(c->arena_bytes) + " bytes");
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  const bool z0 = c->at_zero, b0 = c->at_beta;
  std::vector<hq_tune_entry> out;
  auto run = [&](int n) {
    for (int s = 0; s < n; ++s) dispatch_sweep(c, c->at_zero ? HQ_SWEEP_UP : HQ_SWEEP_DOWN, HQ_SWEEP_MEASURE);
  };
  auto restore = [&]() {
    HQ_CUDA(cudaMemcpyAsync(c->arena, snap, c->arena_bytes, cudaMemcpyDeviceToDevice, c->stream));
    c->at_zero = z0;
    c->at_beta = b0;
  };
  try {
    HQ_CUDA(cudaEventCreate(&e0));
    HQ_CUDA(cudaEventCreate(&e1));
    // the candidates are issued directly: a captured sweep would keep its capture's choices
    HQ_CUDA(cudaStreamSynchronize(c->stream));
    for (auto& gr : c->graphs) cudaGraphExecDestroy(gr.second);
    c->graphs.clear();
    HQ_CUDA(cudaMemcpyAsync(snap, c->arena, c->arena_bytes, cudaMemcpyDeviceToDevice, c->stream));
    for (auto& g : groups) {
      const int nl = g.first;
      bool sep_ok = nl <= HQ_MAX_L;
      for (int i : g.second) sep_ok = sep_ok && !c->ch[i].custom_hop;
      std::vector<int> modes;
      if (sep_ok) modes.push_back(HQ_EXPK_SEPARABLE);
      modes.push_back(HQ_EXPK_DENSE);
      std::vector<int> depths;
      for (int k : {4, 8, 16})
        if (k <= c->kmax_max) depths.push_back(k);
      // cluster sizes: four CTAs per chain (G in distributed shared memory) where the lattice
      // allows it, one CTA with G in global memory otherwise
      std::vector<int> clusters{1};
      if (c->cluster_capable && hq::interval_cluster_ok(nl * nl, nl, HQ_EXPK_SEPARABLE, 16)) clusters = {4, 1};
      double best = 1e300;
      size_t best_at = out.size();
      for (int cl : clusters)
      for (int mode : modes)
        for (int k : depths) {
          if (cl == 4 && !hq::interval_cluster_ok(nl * nl, nl, mode, k)) continue;
          c->cluster_interval = (cl == 4);
          for (int i : g.second) { c->desc[i].expk_mode = mode; c->desc[i].kmax = k; }
          upload_desc(c);
          run(1);  // warm-up
          HQ_CUDA(cudaEventRecord(e0, c->stream));
          run(sweeps);
          HQ_CUDA(cudaEventRecord(e1, c->stream));
          HQ_CUDA(cudaEventSynchronize(e1));
          float ms = 0.f;
          HQ_CUDA(cudaEventElapsedTime(&ms, e0, e1));
          restore();
          hq_tune_entry t;
          t.nl = nl; t.expk_mode = mode; t.delay_depth = k; t.ms_per_sweep = double(ms) / sweeps; t.chosen = 0;
          t.cluster_size = cl;
          t.sweep_mode = c->sweep_mode;
          if (t.ms_per_sweep < best) { best = t.ms_per_sweep; best_at = out.size(); }
          out.push_back(t);
        }
      out[best_at].chosen = 1;
      c->cluster_interval = c->cluster_capable && out[best_at].cluster_size == 4;
      for (int i : g.second) {
        c->desc[i].expk_mode = out[best_at].expk_mode;
        c->desc[i].kmax = out[best_at].delay_depth;
        c->ch[i].expk_mode = out[best_at].expk_mode;
        c->ch[i].kmax = out[best_at].delay_depth;
      }
    }
    upload_desc(c);
    // the sweep mode for the whole context with the per-size choices made above
    if (c->sweep_capable) {
      double best = 1e300;
      size_t best_at = out.size();
      for (int m : {HQ_SWEEP_LAUNCHES, HQ_SWEEP_PERSISTENT}) {
        c->sweep_mode = m;
        run(1);  // warm-up
        HQ_CUDA(cudaEventRecord(e0, c->stream));
        run(sweeps);
        HQ_CUDA(cudaEventRecord(e1, c->stream));
        HQ_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        HQ_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        restore();
        hq_tune_entry t;
        t.nl = 0; t.expk_mode = -1; t.delay_depth = 0; t.cluster_size = 0; t.sweep_mode = m; t.chosen = 0;
        t.ms_per_sweep = double(ms) / sweeps;
        if (t.ms_per_sweep < best) { best = t.ms_per_sweep; best_at = out.size(); }
        out.push_back(t);
      }
      out[best_at].chosen = 1;
      c->sweep_mode = out[best_at].sweep_mode;
    }
    HQ_CUDA(cudaStreamSynchronize(c->stream));
    // captured sweeps hold the kernel choice of their capture
    for (auto& gr : c->graphs) cudaGraphExecDestroy(gr.second);
    c->graphs.clear();
  } catch (...) {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(snap);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(snap);
  for (int k = 0; k < (int)out.size() && k < capacity; ++k) entries[k] = out[k];
  if (n_entries) *n_entries = (int)out.size();
  HQ_API_END
}

int hq_upload_fields_i8(hq_ctx* c, const signed char* all) {
  HQ_API_BEGIN
  if (!c || !all) throw HqError(HQ_E_INVALID, "null argument");
  size_t off = 0;
  for (int i = 0; i < c->n; ++i) {
    const size_t bytes = size_t(c->desc[i].nt) * c->desc[i].N;
    HQ_CUDA(cudaMemcpyAsync(c->desc[i].fields, all + off, bytes, cudaMemcpyHostToDevice, c->stream));
    off += bytes;
  }
  HQ_API_END
}

int hq_download_fields_i8(hq_ctx* c, signed char* all) {
  HQ_API_BEGIN
  if (!c || !all) throw HqError(HQ_E_INVALID, "null argument");
  size_t off = 0;
  for (int i = 0; i < c->n; ++i) {
    const size_t bytes = size_t(c->desc[i].nt) * c->desc[i].N;
    HQ_CUDA(cudaMemcpyAsync(all + off, c->desc[i].fields, bytes, cudaMemcpyDeviceToHost, c->stream));
    off += bytes;
  }
  HQ_API_END
}

int hq_logdet_adjoint(hq_ctx* c, double* out, double* logdet) {
  HQ_API_BEGIN
  if (!c) throw HqError(HQ_E_INVALID, "null context");
  if (!c->initialised || !c->at_zero) throw HqError(HQ_E_INVALID, "hq_logdet_adjoint: stacks must be at tau = 0");
  c->prof_next = 0;
  // zero D (W4) and the scalar accumulators
  for (int i = 0; i < c->n; ++i) {
    const HqChain& d = c->desc[i];
    HQ_CUDA(cudaMemsetAsync(d.W4, 0, size_t(d.N) * d.N * sizeof(double), c->stream));
    HQ_CUDA(cudaMemsetAsync(d.acc + HQ_ACC_DMU, 0, 2 * sizeof(double), c->stream));
  }
  // no-update up pass: wrap slice by slice, rebuild G from the stacks every pace slices
  // (the checkpoints), accumulate the adjoint contractions of every slice
  for (int b = 0; b < c->nstab_max; ++b) {
    { ProfScope ps(c, PC_ADJ); HQ_CUDA(hq::launch_adj_interval(c->d_desc, c->n, b, c->Nmax, c->resident, c->stream)); }
    push_step(c, HQ_UP, HQ_UP, b);
    run_jobs(c, PH_B1, HQ_UP, b);
    run_jobs(c, PH_B2, HQ_UP, b);
    { ProfScope ps(c, PC_INVERT); HQ_CUDA(hq::launch_invert(c->d_desc, c->n, b, 0, c->Nmax, c->resident, c->stream)); }
    run_jobs(c, PH_B3, HQ_UP, b);
    run_jobs(c, PH_B4, HQ_UP, b);
    { ProfScope ps(c, PC_ADJ); HQ_CUDA(hq::launch_adj_last(c->d_desc, c->n, b, c->stream)); }
  }
  // log|det(1 + U D Vt)| = sum log dmax + log|det(dmax^-1 U^T + dmin Vt)| from the full left stack
  run_jobs(c, PH_LOGDET, 0, 0);
  run_jobs(c, PH_LOGDET, 0, 1);
  HQ_CUDA(cudaStreamSynchronize(c->stream));
  size_t off = 0;
  for (int i = 0; i < c->n; ++i) {
    const HqChain& d = c->desc[i];
    ChainHost& h = c->ch[i];
    const int N = d.N;
    const size_t NN = size_t(N) * N;
    std::vector<double> D(NN), Wm(NN), Dl(N);
    double acc[HQ_ACC_COUNT];
    read_acc(c, i, acc);
    HQ_CUDA(cudaMemcpy(D.data(), d.W4, NN * sizeof(double), cudaMemcpyDeviceToHost));
    HQ_CUDA(cudaMemcpy(Wm.data(), d.W1, NN * sizeof(double), cudaMemcpyDeviceToHost));
    HQ_CUDA(cudaMemcpy(Dl.data(), d.stackD + size_t(d.n_stab - 1) * N, N * sizeof(double), cudaMemcpyDeviceToHost));
    // log-determinant (host LU with partial pivoting of the well-conditioned middle matrix)
    double ld = 0.0;
    for (int k = 0; k < N; ++k) ld += std::log(std::max(Dl[k], 1.0));
    {
      std::vector<double> M = Wm;
      for (int k = 0; k < N; ++k) {
        int p = k;
        for (int r = k + 1; r < N; ++r)
          if (std::fabs(M[r + size_t(k) * N]) > std::fabs(M[p + size_t(k) * N])) p = r;
        if (p != k)
          for (int j = 0; j < N; ++j) std::swap(M[k + size_t(j) * N], M[p + size_t(j) * N]);
        const double pv = M[k + size_t(k) * N];
        ld += std::log(std::fabs(pv));
        for (int r = k + 1; r < N; ++r) {
          const double f = M[r + size_t(k) * N] / pv;
          for (int j = k + 1; j < N; ++j) M[r + size_t(j) * N] -= f * M[k + size_t(j) * N];
        }
      }
    }
    if (logdet) logdet[i] = ld;
    // Gamma = Q (Phi o (Q^T E^-1 D Q)^T) Q^T, Phi = divided differences of exp(-dt lambda)
    std::vector<double> w, Q;
    jacobi_eig(N, h.K, w, Q);
    std::vector<double> Einv(NN), M1(NN), M2(NN), Mt(NN), P(NN), G1(NN), Gam(NN);
    for (int j = 0; j < N; ++j)
      for (int i2 = 0; i2 < N; ++i2) M1[i2 + size_t(j) * N] = Q[i2 + size_t(j) * N] * std::exp(h.dt * w[j]);
    host_gemm(N, M1.data(), false, Q.data(), true, Einv.data());  // E^-1 = exp(+dt K)
    host_gemm(N, Einv.data(), false, D.data(), false, M1.data());  // M = E^-1 D
    host_gemm(N, Q.data(), true, M1.data(), false, M2.data());     // Q^T M
    host_gemm(N, M2.data(), false, Q.data(), false, Mt.data());    // Q^T M Q
    for (int j = 0; j < N; ++j)
      for (int i2 = 0; i2 < N; ++i2) {
        const double fi = std::exp(-h.dt * w[i2]), fj = std::exp(-h.dt * w[j]);
        const double dd = std::fabs(w[i2] - w[j]) > 1e-10 ? (fi - fj) / (w[i2] - w[j]) : -h.dt * 0.5 * (fi + fj);
        P[i2 + size_t(j) * N] = dd * Mt[j + size_t(i2) * N];
      }
    host_gemm(N, Q.data(), false, P.data(), false, G1.data());
    host_gemm(N, G1.data(), false, Q.data(), true, Gam.data());
    out[off + 0] = acc[HQ_ACC_DMU];
    out[off + 1] = acc[HQ_ACC_DALPHA];
    std::memcpy(out + off + 2, Gam.data(), NN * sizeof(double));
    off += 2 + NN;
  }
  // the pass left the stacks at tau = beta
  c->at_zero = false;
  c->at_beta = true;
  HQ_API_END
}

}  // extern "C"

// =======================================================================================
//  hq_equaltime_g_noalloc: an entry point that allocates no device memory.
//
//  Some callers cannot call cudaMalloc: a process that hands out its whole device-memory
//  budget once at start-up and forbids allocations after that, or a long-running service
//  that must never meet an out-of-memory failure in the middle of its work. For them,
//  hq_equaltime_g_noalloc computes the equal-time Green's function
//  G(0,0) = (1 + B(nt-1)...B(0))^-1 of one chain from Ising fields already on the device,
//  with every temporary (the UDV stack, the work matrices, the chain descriptor and the GEMM
//  job lists) held in one file-scope device array of fixed size. The work is the kernel
//  sequence of hq_init_stacks_and_g.
// =======================================================================================
namespace {

// Scratch of the no-allocation entry point (hq_equaltime_g_noalloc). Every GPU that loads the library holds these
// bytes until the process exits. Limits: N = nl*nl <= 64 and ceil(nt / pace) <= 16.
constexpr size_t kScratchBytes = size_t(4) << 20;
constexpr int kMaxN = 64;
constexpr int kMaxStab = 16;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
// device address of the scratch, looked up once per device (with that device current) by the
// first call on it; valid for the life of the device's context
std::atomic<void*> g_scratch_addr[kMaxDevices];
std::mutex g_scratch_mutex;

int set_error(int code, const std::string& msg) {
  g_last_error = msg;  // reported by hq_last_error()
  return code;
}

// exp(dt t H_1d) of the L-site periodic chain is circulant:
// a[d] = (1/L) sum_k exp(2 dt t cos(2 pi k / L)) cos(2 pi k d / L)
void circulant(int L, double dt_t, double* a) { circulant_exp(L, dt_t, a); }
size_t up256(size_t b) { return align256(b); }
HqGemmJob job(int N, const double* A, int ta, const double* B, int tb, double* C) { return make_job(N, A, ta, B, tb, C); }

}  // namespace

static int equaltime_g_noalloc(int nl, double nnt, double u, double mu, double beta, int nt, int pace,
                               const signed char* fields_dev, double* g_dev, void* stream) {
  // ---- argument and size checks (include/dqmc_parser.hpp:124-132 plus the scratch limits) ----
  if (!fields_dev || !g_dev) return set_error(HQ_E_INVALID, "hq_equaltime_g_noalloc: null device pointer");
  if (nl < 1 || nt < 1 || pace < 1 || u < 0 || beta < 0)
    return set_error(HQ_E_INVALID, "hq_equaltime_g_noalloc: parameter out of range");
  const int N = nl * nl;
  const int n_stab = (nt % pace == 0) ? nt / pace : nt / pace + 1;
  if (N > kMaxN)
    return set_error(HQ_E_RANGE, "hq_equaltime_g_noalloc: nl*nl = " + std::to_string(N) +
                                     " exceeds the scratch limit of 64 sites");
  if (n_stab > kMaxStab)
    return set_error(HQ_E_RANGE, "hq_equaltime_g_noalloc: ceil(nt/pace) = " + std::to_string(n_stab) +
                                     " exceeds the scratch limit of 16 stack entries");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return set_error(HQ_E_CUDA, "hq_equaltime_g_noalloc: no current CUDA device");
  // ---- set-up, once per device, with that device current: the scratch's device address ----
  void* addr = g_scratch_addr[dev].load(std::memory_order_acquire);
  if (!addr) {
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    addr = g_scratch_addr[dev].load(std::memory_order_relaxed);
    if (!addr) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p)
        return set_error(HQ_E_CUDA, std::string("hq_equaltime_g_noalloc: cudaGetSymbolAddress: ") +
                                        cudaGetErrorString(e));
      g_scratch_addr[dev].store(p, std::memory_order_release);
      addr = p;
    }
  }
  char* base = static_cast<char*>(addr);

  // ---- scratch layout ----
  const size_t NN = size_t(N) * N, mat = NN * sizeof(double);
  size_t off = 0;
  auto take = [&](size_t bytes) { const size_t o = off; off += up256(bytes); return o; };
  const size_t o_desc = take(sizeof(HqChain));
  const int njobs = n_stab + 4;
  const size_t o_jobs = take(sizeof(HqGemmJob) * njobs);
  const size_t o_U = take(2 * size_t(n_stab) * mat);
  const size_t o_D = take(2 * size_t(n_stab) * N * sizeof(double));
  const size_t o_Vt = take(2 * size_t(n_stab) * mat);
  const size_t o_X = take(mat);
  size_t o_W[4];
  for (auto& w : o_W) w = take(mat);
  const size_t o_I = take(mat);
  const size_t o_one = take(N * sizeof(double));
  const size_t o_E = take(2 * mat);
  const size_t o_acc = take(HQ_ACC_COUNT * sizeof(double));
  const size_t o_rng = take(sizeof(uint32_t));
  if (off > kScratchBytes) return set_error(HQ_E_RANGE, "hq_equaltime_g_noalloc: scratch layout exceeds 4 MiB");
  auto ptr = [&](size_t o) { return reinterpret_cast<double*>(base + o); };

  // ---- model constants (src/hubbard.cpp:25-49) ----
  const double dt = beta / nt;
  const double alpha = std::acosh(std::exp(0.5 * dt * u));
  HqChain d;
  std::memset(&d, 0, sizeof(d));
  d.N = N; d.L = nl; d.nt = nt; d.pace = pace; d.n_stab = n_stab;
  d.expk_mode = (nl <= HQ_MAX_L) ? HQK_EXPK_SEPARABLE : HQK_EXPK_DENSE;
  d.kmax = 4; d.active = 1;
  d.alpha = alpha; d.dt = dt;
  d.delta_p = std::exp(-2 * alpha) - 1;
  d.delta_m = std::exp(2 * alpha) - 1;
  d.ev_p = std::exp(alpha);
  d.ev_m = std::exp(-alpha);
  d.sep_c = std::exp(dt * mu);
  d.sep_ci = std::exp(-dt * mu);
  circulant(nl, dt * nnt, d.sep_a);
  circulant(nl, -dt * nnt, d.sep_ai);
  d.expK = ptr(o_E);
  d.inv_expK = ptr(o_E) + NN;
  d.G = g_dev;
  d.fields = reinterpret_cast<int8_t*>(const_cast<signed char*>(fields_dev));
  d.rng = reinterpret_cast<uint32_t*>(base + o_rng);
  d.X = ptr(o_X);
  d.stackU = ptr(o_U);
  d.stackD = ptr(o_D);
  d.stackVt = ptr(o_Vt);
  d.W0 = ptr(o_W[0]); d.W1 = ptr(o_W[1]); d.W2 = ptr(o_W[2]); d.W3 = ptr(o_W[3]);
  d.W4 = d.W3; d.W5 = d.W3;  // not used by this sequence
  d.acc = ptr(o_acc);

  // host images of the constant inputs: dense expK, identity, ones (copied on the caller's
  // stream; pageable sources are consumed before cudaMemcpyAsync returns)
  std::vector<double> a(nl), ai(nl), E(2 * NN), I(NN, 0.0), one(N, 1.0);
  circulant(nl, dt * nnt, a.data());
  circulant(nl, -dt * nnt, ai.data());
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < N; ++i) {
      const int dx = ((i % nl) - (j % nl) + nl) % nl, dy = ((i / nl) - (j / nl) + nl) % nl;
      E[i + size_t(j) * N] = d.sep_c * a[dx] * a[dy];
      E[NN + i + size_t(j) * N] = d.sep_ci * ai[dx] * ai[dy];
    }
  for (int k = 0; k < N; ++k) I[k + size_t(k) * N] = 1.0;

  // ---- batched GEMM jobs: stack pushes, then the builder with an empty left stack ----
  std::vector<HqGemmJob> jobs;
  const double* Iid = ptr(o_I);
  const double* ones = ptr(o_one);
  for (int b = 0; b < n_stab; ++b) {
    const double* prev = (b == 0) ? Iid : d.stackVt + (size_t(n_stab) + (b - 1)) * NN;
    jobs.push_back(job(N, d.W0, 0, prev, 0, d.stackVt + (size_t(n_stab) + b) * NN));
  }
  const double* UR = d.stackU + (size_t(n_stab) + n_stab - 1) * NN;
  const double* DR = d.stackD + (size_t(n_stab) + n_stab - 1) * N;
  const double* VtR = d.stackVt + (size_t(n_stab) + n_stab - 1) * NN;
  HqGemmJob b1 = job(N, Iid, 1, UR, 0, d.W1);
  b1.rs = ones; b1.rs_mode = 2; b1.cs = DR; b1.cs_mode = 2;
  HqGemmJob b2 = job(N, Iid, 0, VtR, 1, d.W1);
  b2.rs = ones; b2.rs_mode = 3; b2.cs = DR; b2.cs_mode = 3; b2.beta = 1.0;
  HqGemmJob b3 = job(N, d.W1, 0, Iid, 1, d.W2);
  b3.ks = ones; b3.ks_mode = 2;
  HqGemmJob b4 = job(N, UR, 0, d.W2, 0, g_dev);
  b4.ks = DR; b4.ks_mode = 2;
  jobs.push_back(b1);
  jobs.push_back(b2);
  jobs.push_back(b3);
  jobs.push_back(b4);

  // ---- upload (no allocation) and launch ----
  cudaError_t e = cudaSuccess;
  HqChain* d_desc = reinterpret_cast<HqChain*>(base + o_desc);
  HqGemmJob* d_jobs = reinterpret_cast<HqGemmJob*>(base + o_jobs);
  if ((e = cudaMemcpyAsync(d_desc, &d, sizeof(d), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
      (e = cudaMemcpyAsync(d_jobs, jobs.data(), jobs.size() * sizeof(HqGemmJob), cudaMemcpyHostToDevice, st)) !=
          cudaSuccess ||
      (e = cudaMemcpyAsync(ptr(o_E), E.data(), E.size() * sizeof(double), cudaMemcpyHostToDevice, st)) !=
          cudaSuccess ||
      (e = cudaMemcpyAsync(ptr(o_I), I.data(), I.size() * sizeof(double), cudaMemcpyHostToDevice, st)) !=
          cudaSuccess ||
      (e = cudaMemcpyAsync(ptr(o_one), one.data(), one.size() * sizeof(double), cudaMemcpyHostToDevice, st)) !=
          cudaSuccess ||
      (e = cudaMemsetAsync(ptr(o_acc), 0, HQ_ACC_COUNT * sizeof(double), st)) != cudaSuccess)
    return set_error(HQ_E_CUDA, std::string("hq_equaltime_g_noalloc: upload: ") + cudaGetErrorString(e));
  // the kernels' shared-memory limits (raised only, and only when an earlier context of
  // smaller chains left them below this size; no allocation)
  if ((e = hq::prepare_kernels(N, 4, true)) != cudaSuccess)
    return set_error(HQ_E_CUDA, std::string("hq_equaltime_g_noalloc: kernel limits: ") + cudaGetErrorString(e));
  for (int b = 0; b < n_stab && e == cudaSuccess; ++b) {
    // src/dqmc_core.cpp:67-87: B^T products from t = nt down to 1, pushed every pace slices
    e = hq::launch_bchain(d_desc, 1, HQ_DOWN, b, N, true, st);
    if (e == cudaSuccess) e = hq::launch_udt(d_desc, 1, 1, b, N, true, st);
    if (e == cudaSuccess) e = hq::launch_gemm(d_jobs + b, 1, N, N, st);
  }
  // src/dqmc_core.cpp:89-97 with stable_numerics.hpp:186-239: G = (1 + right^T)^-1
  const int jb = n_stab;
  if (e == cudaSuccess) e = hq::launch_gemm(d_jobs + jb, 1, N, N, st);
  if (e == cudaSuccess) e = hq::launch_gemm(d_jobs + jb + 1, 1, N, N, st);
  if (e == cudaSuccess) e = hq::launch_invert(d_desc, 1, n_stab - 1, 0, N, true, st);
  if (e == cudaSuccess) e = hq::launch_gemm(d_jobs + jb + 2, 1, N, N, st);
  if (e == cudaSuccess) e = hq::launch_gemm(d_jobs + jb + 3, 1, N, N, st);
  if (e != cudaSuccess) return set_error(HQ_E_CUDA, std::string("hq_equaltime_g_noalloc: launch: ") + cudaGetErrorString(e));
  return HQ_OK;
}

// The C entry point: host-side failures (a std::bad_alloc of the small host vectors, say)
// become status codes instead of crossing the C ABI as exceptions.
extern "C" HQ_API int hq_equaltime_g_noalloc(int nl, double nnt, double u, double mu, double beta, int nt, int pace,
                                             const signed char* fields_dev, double* g_dev, void* stream) {
  try {
    return equaltime_g_noalloc(nl, nnt, u, mu, beta, nt, pace, fields_dev, g_dev, stream);
  } catch (const std::bad_alloc&) {
    return set_error(HQ_E_NOMEM, "hq_equaltime_g_noalloc: host allocation failed");
  } catch (const std::exception& e) {
    return set_error(HQ_E_INVALID, std::string("hq_equaltime_g_noalloc: ") + e.what());
  }
}
