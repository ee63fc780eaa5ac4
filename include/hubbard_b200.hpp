// hubbard_b200.hpp -- header-only C++ facade over the C ABI of hubbard_b200.h that keeps
// the call surface of the reference's DQMC sweep (JefferyWangSH/hubbard-attractive-U):
//   DQMC::Core                (include/dqmc_core.h:35-112)
//   Model::HubbardAttractiveU (include/hubbard.h:32-112)
//   Utils::SvdStack           (include/utils/svd_stack.hpp:51-190, read-only view)
//   DQMC::Params              (include/dqmc_params.hpp:20-45)
// inside namespace hq_b200 so that it can sit next to the reference's own classes. A driver
// written against the reference (src/dqmc_handle.cpp, src/main.cpp) compiles against these
// classes after `using namespace hq_b200;`. Green's functions are returned as column-major
// N x N std::vector<double> (the reference returns Eigen::Ref<Eigen::MatrixXd>, also
// column-major). Failures throw std::runtime_error, as the reference does for its own
// configuration and LAPACK errors.
#pragma once
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "hubbard_b200.h"

namespace hq_b200 {

inline void check(int rc) {
  if (rc != HQ_OK) {
    char buf[1024];
    hq_last_error(buf, sizeof(buf));
    throw std::runtime_error(std::string("hubbard_b200: ") + buf);
  }
}

// One GPU context holding one or more chains.
class Context {
 public:
  Context(int device, const std::vector<hq_chain_params>& chains) {
    hq_ctx* c = nullptr;
    check(hq_create(device, static_cast<int>(chains.size()), chains.data(), &c));
    ctx_.reset(c, [](hq_ctx* p) { hq_destroy(p); });
  }
  hq_ctx* get() const { return ctx_.get(); }
  // HQ_SWEEP_PERSISTENT (one launch per sweep) or HQ_SWEEP_LAUNCHES (one per phase and interval)
  void set_sweep_mode(int mode) { check(hq_set_sweep_mode(get(), mode)); }
  int sweep_mode() const {
    int m = 0;
    check(hq_get_sweep_mode(get(), &m));
    return m;
  }

 private:
  std::shared_ptr<hq_ctx> ctx_;
};

namespace DQMC {

struct Params {  // include/dqmc_params.hpp:20-45 (the sweep's subset)
  int nl{4}, ns{16}, ng{16}, nt{160};
  double dt{0.05}, beta{8.0}, nnt{1.0}, mu{0.0}, u{4.0};
  int stabilization_pace{10};
  bool is_fft{false};
};

}  // namespace DQMC

namespace Model {

// Model::HubbardAttractiveU: owns the Ising fields of one chain.
class HubbardAttractiveU {
 public:
  // src/hubbard.cpp:25-82 (K, exp(-dt K), alpha) -- created on the GPU with the chain
  void initialize(const DQMC::Params& p, long long seed = 0, int device = 0, bool dynamic = true) {
    p_ = p;
    hq_chain_params c{};
    c.nl = p.nl; c.nnt = p.nnt; c.u = p.u; c.mu = p.mu; c.beta = p.beta; c.nt = p.nt;
    c.stabilization_pace = p.stabilization_pace;
    c.expk_mode = p.is_fft ? HQ_EXPK_SEPARABLE : HQ_EXPK_DENSE;
    c.seed = seed;
    c.delay_depth = 0;
    c.dynamic = dynamic ? 1 : 0;
    c.snapshots = 1;
    ctx_ = std::make_shared<Context>(device, std::vector<hq_chain_params>{c});
  }
  // src/hubbard.cpp:102-110
  void set_ising_fields_to_random() { check(hq_fields_random(ctx_->get(), 0)); }
  // include/dqmc_io.hpp:257-290 / :234-255 (in memory, int [nt][ns])
  void load_ising_fields(const std::vector<int>& f) { check(hq_set_fields(ctx_->get(), 0, f.data())); }
  std::vector<int> ising_fields() const {
    std::vector<int> f(static_cast<size_t>(p_.nt) * p_.nl * p_.nl);
    check(hq_get_fields(ctx_->get(), 0, f.data()));
    return f;
  }
  hq_ctx* context() const { return ctx_->get(); }
  const DQMC::Params& params() const { return p_; }

 private:
  DQMC::Params p_;
  std::shared_ptr<Context> ctx_;
};

}  // namespace Model

namespace Utils {

// Utils::SvdStack (include/utils/svd_stack.hpp:51-190): a read-only view of the top of one
// chain's left (side 0) or right (side 1) UDV stack; pushes and pops happen inside the sweeps.
class SvdStack {
 public:
  using Matrix = std::vector<double>;  // column-major N x N
  using Vector = std::vector<double>;
  SvdStack(const Model::HubbardAttractiveU& model, int side) : model_(&model), side_(side) {}
  int MatDim() const { return model_->params().nl * model_->params().nl; }
  int StackLength() const {
    int n = 0;
    check(hq_get_stack(model_->context(), 0, side_, &n, nullptr, nullptr, nullptr));
    return n;
  }
  bool empty() const { return StackLength() == 0; }
  Vector SingularValues() const { Vector d(MatDim()); get(nullptr, d.data(), nullptr); return d; }
  Matrix MatrixU() const { Matrix u(size_t(MatDim()) * MatDim()); get(u.data(), nullptr, nullptr); return u; }
  Matrix MatrixV() const { Matrix v(size_t(MatDim()) * MatDim()); get(nullptr, nullptr, v.data()); return v; }

 private:
  void get(double* u, double* d, double* v) const {
    int n = 0;
    check(hq_get_stack(model_->context(), 0, side_, &n, u, d, v));
    if (n == 0) throw std::runtime_error("Utils::SvdStack: the stack is empty");
  }
  const Model::HubbardAttractiveU* model_;
  int side_;
};

}  // namespace Utils

namespace DQMC {

// DQMC::Core: stacks, Green's functions and the three sweeps of one chain.
class Core {
 public:
  using Hubbard = Model::HubbardAttractiveU;
  using Matrix = std::vector<double>;  // column-major N x N

  void initialize(const Params& p, bool is_equaltime, bool is_dynamic) {  // src/dqmc_core.cpp:20-30
    p_ = p;
    eq_ = is_equaltime;
    dyn_ = is_dynamic;
  }
  void initialize_svdstacks(const Hubbard& model) { model_ = &model; }      // src/dqmc_core.cpp:67-87
  void initialize_green_functions() { check(hq_init_stacks_and_g(ctx())); }  // src/dqmc_core.cpp:89-97
  void set_thermalization(bool on) { thermalization_ = on; }

  void sweep_from_0_to_beta(Hubbard&) { check(hq_sweep(ctx(), HQ_SWEEP_UP, flags())); }    // :167-227
  void sweep_from_beta_to_0(Hubbard&) { check(hq_sweep(ctx(), HQ_SWEEP_DOWN, flags())); }  // :233-284
  void sweep_for_dynamic_green_functions(Hubbard&) {                                          // :291-390
    if (dyn_) check(hq_sweep(ctx(), HQ_SWEEP_DYNAMIC, 0));
  }

  Matrix current_gftt() const { return get(HQ_G_CURRENT, 0); }  // include/dqmc_core.h:76-79
  Matrix gftt(int t) const { return get(HQ_G_TT, t); }
  Matrix gft0(int t) const { return get(HQ_G_T0, t); }
  Matrix gf0t(int t) const { return get(HQ_G_0T, t); }
  double equaltimeWrapError() const { return wrap()[0]; }  // include/dqmc_core.h:80-81
  double dynamicWrapError() const { return wrap()[1]; }

 private:
  hq_ctx* ctx() const {
    if (!model_) throw std::runtime_error("DQMC::Core: initialize_svdstacks(model) first");
    return model_->context();
  }
  int flags() const { return (!thermalization_ && eq_) ? (HQ_SWEEP_MEASURE | HQ_SWEEP_SNAPSHOT) : 0; }
  Matrix get(int which, int t) const {
    const size_t N = static_cast<size_t>(p_.nl) * p_.nl;
    Matrix g(N * N);
    check(hq_get_g(ctx(), 0, which, t, g.data()));
    return g;
  }
  std::vector<double> wrap() const {
    std::vector<double> w(2);
    check(hq_get_wrap_errors(ctx(), 0, w.data()));
    return w;
  }
  Params p_;
  bool eq_{true}, dyn_{false}, thermalization_{false};
  const Hubbard* model_{nullptr};
};

}  // namespace DQMC
}  // namespace hq_b200
