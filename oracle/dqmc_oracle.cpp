// =====================================================================================
//  dqmc_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
//  CPU restatement of the reference DQMC sweep (JefferyWangSH/hubbard-attractive-U),
//  used as the checker of the CUDA path and as the timed CPU baseline. Nothing in the
//  product links or calls this file; only tests/, __graft_entry__.smoke() and bench.py's
//  CPU legs load it.
//
//  Parity status: the reference cannot be compiled in this image (it needs Eigen, MKL,
//  Boost and xtensor), so no bit-level golden vector of the reference exists. This
//  restatement is pinned statistically against the reference's own example run
//  (example/*.out: filling, double occupancy, s-wave pairing at L=4, beta=8, nt=160)
//  and follows every step of the reference listed below, function by function.
//
//  Linear algebra: the reference goes through Eigen+MKL. Here the same operations go
//  through scipy's bundled OpenBLAS (cblas_dgemm, LAPACKE_dgesvd 'S','S',
//  dgetrf/dgetri, dgeqp3, dsyev); differences are at rounding level.
//  RNG: the reference's own generator, std::default_random_engine (libstdc++:
//  minstd_rand0) with std::bernoulli_distribution (src/random.cpp:14-15).
// =====================================================================================
#include <algorithm>
#include <cassert>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

extern "C" {
void scipy_cblas_dgemm(int order, int ta, int tb, int m, int n, int k, double alpha, const double* a, int lda,
                       const double* b, int ldb, double beta, double* c, int ldc);
void scipy_cblas_dtrsm(int order, int side, int uplo, int ta, int diag, int m, int n, double alpha,
                       const double* a, int lda, double* b, int ldb);
int scipy_LAPACKE_dgesvd(int layout, char jobu, char jobvt, int m, int n, double* a, int lda, double* s, double* u,
                         int ldu, double* vt, int ldvt, double* superb);
int scipy_LAPACKE_dgetrf(int layout, int m, int n, double* a, int lda, int* ipiv);
int scipy_LAPACKE_dgetri(int layout, int n, double* a, int lda, const int* ipiv);
int scipy_LAPACKE_dsyev(int layout, char jobz, char uplo, int n, double* a, int lda, double* w);
int scipy_LAPACKE_dgeqp3(int layout, int m, int n, double* a, int lda, int* jpvt, double* tau);
int scipy_LAPACKE_dormqr(int layout, char side, char trans, int m, int n, int k, const double* a, int lda,
                         const double* tau, double* c, int ldc);
void scipy_openblas_set_num_threads(int n);
}

namespace oracle {

constexpr int kColMajor = 102, kNoTrans = 111, kTrans = 112, kLeft = 141, kUpper = 121, kNonUnit = 131;

// Column-major dense matrix, the storage order of Eigen::MatrixXd in the reference
// (include/dqmc_core.h:27).
struct Mat {
  int n = 0;
  std::vector<double> a;
  Mat() = default;
  explicit Mat(int n_) : n(n_), a(size_t(n_) * n_, 0.0) {}
  static Mat Identity(int n_) {
    Mat m(n_);
    for (int i = 0; i < n_; ++i) m(i, i) = 1.0;
    return m;
  }
  double& operator()(int i, int j) { return a[i + size_t(j) * n]; }
  double operator()(int i, int j) const { return a[i + size_t(j) * n]; }
  double* data() { return a.data(); }
  const double* data() const { return a.data(); }
};
using Vec = std::vector<double>;

// C = op(A) * op(B)
static Mat gemm(const Mat& A, bool ta, const Mat& B, bool tb) {
  Mat C(A.n);
  scipy_cblas_dgemm(kColMajor, ta ? kTrans : kNoTrans, tb ? kTrans : kNoTrans, A.n, A.n, A.n, 1.0, A.data(), A.n,
                    B.data(), B.n, 0.0, C.data(), C.n);
  return C;
}
static Mat transpose(const Mat& A) {
  Mat T(A.n);
  for (int j = 0; j < A.n; ++j)
    for (int i = 0; i < A.n; ++i) T(j, i) = A(i, j);
  return T;
}
// Eigen's PartialPivLU inverse (include/utils/stable_numerics.hpp:235) -> dgetrf + dgetri.
static Mat inverse(const Mat& A) {
  Mat B = A;
  std::vector<int> ipiv(A.n);
  if (scipy_LAPACKE_dgetrf(kColMajor, A.n, A.n, B.data(), A.n, ipiv.data()) < 0) throw std::runtime_error("dgetrf");
  if (scipy_LAPACKE_dgetri(kColMajor, A.n, B.data(), A.n, ipiv.data()) < 0) throw std::runtime_error("dgetri");
  return B;
}

// ------------------------------------------------------------------------------------
//  Parameters: include/dqmc_params.hpp:20-45, dt = beta/nt (include/dqmc_parser.hpp:88).
// ------------------------------------------------------------------------------------
struct Params {
  int nl = 4, ns = 16, nt = 160, pace = 10;
  double beta = 8.0, dt = 0.05, nnt = 1.0, mu = 0.0, u = 4.0;
  bool is_equaltime = true, is_dynamic = true;
};

// ------------------------------------------------------------------------------------
//  Square lattice: src/square_lattice.cpp:30-61 (site i = x + L*y, PBC, NN directions
//  0:+x 1:+y 2:-x 3:-y, hopping matrix built with +=, so L=2 doubles the bonds).
// ------------------------------------------------------------------------------------
struct Lattice {
  int nl = 0, ns = 0, nkstars = 0;
  std::vector<int> nn;       // ns x 4
  Mat hop;                   // nn hoppings
  std::vector<int> disp;     // ns x ns displacement table (src/square_lattice.cpp:63-81)
  std::vector<double> kstars;  // nkstars x 2 (src/square_lattice.cpp:83-95)
  std::vector<std::complex<double>> fourier;  // ns x nkstars (src/square_lattice.cpp:120-135)

  void initialize(int L) {
    nl = L;
    ns = L * L;
    nkstars = int((std::floor(L / 2.) + 1) * (std::floor(L / 2.) + 1));
    nn.assign(size_t(ns) * 4, 0);
    for (int i = 0; i < ns; ++i) {
      const int x = i % L, y = i / L;
      nn[i * 4 + 0] = ((x + 1) % L) + L * y;
      nn[i * 4 + 2] = ((x - 1 + L) % L) + L * y;
      nn[i * 4 + 1] = x + L * ((y + 1) % L);
      nn[i * 4 + 3] = x + L * ((y - 1 + L) % L);
    }
    hop = Mat(ns);
    for (int i = 0; i < ns; ++i) {
      const int xp = nn[i * 4 + 0], yp = nn[i * 4 + 1];
      hop(i, xp) += 1.0;
      hop(xp, i) += 1.0;
      hop(i, yp) += 1.0;
      hop(yp, i) += 1.0;
    }
    disp.assign(size_t(ns) * ns, 0);
    for (int i = 0; i < ns; ++i) {
      const int xi = i % L, yi = i / L;
      for (int j = 0; j < ns; ++j) {
        const int xj = j % L, yj = j / L;
        disp[i + size_t(j) * ns] = (xj - xi + L) % L + ((yj - yi + L) % L) * L;
      }
    }
    kstars.assign(size_t(nkstars) * 2, 0.0);
    int n = 0;
    for (double i = std::ceil(L / 2.); i <= L; ++i)
      for (double j = std::ceil(L / 2.); j <= L; ++j) {
        kstars[n * 2 + 0] = i / L * 2 * M_PI - M_PI;
        kstars[n * 2 + 1] = j / L * 2 * M_PI - M_PI;
        ++n;
      }
    fourier.assign(size_t(ns) * nkstars, 0.0);
    for (int i = 0; i < ns; ++i) {
      const int x = i % L, y = i / L;
      for (int k = 0; k < nkstars; ++k) {
        const double kx = kstars[k * 2], ky = kstars[k * 2 + 1];
        fourier[i + size_t(k) * ns] = std::complex<double>(std::cos(x * kx + y * ky), -std::sin(x * kx + y * ky));
      }
    }
  }
};

// Matrix exponential of a symmetric matrix through its eigendecomposition (replaces
// Eigen's MatrixBase::exp() used at src/hubbard.cpp:46-47; K is real symmetric).
static Mat sym_expm(const Mat& K, double scale) {
  const int n = K.n;
  Mat Q = K;
  Vec w(n);
  if (scipy_LAPACKE_dsyev(kColMajor, 'V', 'U', n, Q.data(), n, w.data()) != 0) throw std::runtime_error("dsyev");
  Mat QE(n);
  for (int j = 0; j < n; ++j) {
    const double e = std::exp(scale * w[j]);
    for (int i = 0; i < n; ++i) QE(i, j) = Q(i, j) * e;
  }
  return gemm(QE, false, Q, true);
}

// ------------------------------------------------------------------------------------
//  Model::HubbardAttractiveU: src/hubbard.cpp:25-341.
// ------------------------------------------------------------------------------------
struct Model {
  int nl = 0, ns = 0, nt = 0;
  double dt = 0, nnt = 0, mu = 0, u = 0, alpha = 0;
  std::vector<int> fields;  // (nt, ns), fields[t*ns + i]  (Eigen::ArrayXXi m_ising_fields)
  Mat K, expK, inv_expK;

  int& s(int t, int i) { return fields[size_t(t) * ns + i]; }
  int s(int t, int i) const { return fields[size_t(t) * ns + i]; }

  // src/hubbard.cpp:25-49 (dense path); an optional custom hopping matrix replaces
  // -nnt*H_nn (per-bond hoppings, used by the log-det gradient checks).
  void initialize(const Params& p, const Lattice& lat, const Mat* custom_hop = nullptr) {
    nl = p.nl; ns = p.ns; nt = p.nt; dt = p.dt; nnt = p.nnt; mu = p.mu; u = p.u;
    alpha = std::acosh(std::exp(0.5 * dt * u));  // src/hubbard.cpp:35
    fields.assign(size_t(nt) * ns, 1);
    K = Mat(ns);
    for (int j = 0; j < ns; ++j)
      for (int i = 0; i < ns; ++i) K(i, j) = custom_hop ? -(*custom_hop)(i, j) : -nnt * lat.hop(i, j);
    for (int i = 0; i < ns; ++i) K(i, i) -= mu;  // src/hubbard.cpp:41-42
    expK = sym_expm(K, -dt);
    inv_expK = sym_expm(K, +dt);
  }
  // src/hubbard.cpp:102-110
  void set_fields_random(std::default_random_engine& eng) {
    std::bernoulli_distribution b(0.5);
    for (int t = 0; t < nt; ++t)
      for (int i = 0; i < ns; ++i) s(t, i) = b(eng) ? +1 : -1;
  }
  void left_mult(Mat& g, const Mat& E) const { g = gemm(E, false, g, false); }
  void right_mult(Mat& g, const Mat& E) const { g = gemm(g, false, E, false); }
  void scale_rows(Mat& g, int t, double sign) const {
    for (int i = 0; i < ns; ++i) {
      const double f = std::exp(sign * alpha * s(t, i));
      for (int j = 0; j < ns; ++j) g(i, j) *= f;
    }
  }
  void scale_cols(Mat& g, int t, double sign) const {
    for (int i = 0; i < ns; ++i) {
      const double f = std::exp(sign * alpha * s(t, i));
      for (int j = 0; j < ns; ++j) g(j, i) *= f;
    }
  }
  // src/hubbard.cpp:293-301:  G -> expV(t) * expK * G
  void multiply_B_from_left(Mat& g, int t) const { left_mult(g, expK); scale_rows(g, t, +1); }
  // src/hubbard.cpp:303-311:  G -> G * expV(t) * expK
  void multiply_B_from_right(Mat& g, int t) const { scale_cols(g, t, +1); right_mult(g, expK); }
  // src/hubbard.cpp:313-321:  G -> inv_expK * inv_expV(t) * G
  void multiply_invB_from_left(Mat& g, int t) const { scale_rows(g, t, -1); left_mult(g, inv_expK); }
  // src/hubbard.cpp:323-331:  G -> G * inv_expK * inv_expV(t)
  void multiply_invB_from_right(Mat& g, int t) const { right_mult(g, inv_expK); scale_cols(g, t, -1); }
  // src/hubbard.cpp:333-341:  G -> expK^T * expV(t) * G   (K symmetric)
  void multiply_adjB_from_left(Mat& g, int t) const { scale_rows(g, t, +1); left_mult(g, expK); }

  // src/hubbard.cpp:123-130
  double acceptance_ratio(const Mat& g, int t, int i) const {
    const double delta = std::exp(-2 * alpha * s(t, i)) - 1;
    return std::pow(1 + (1 - g(i, i)) * delta, 2) / (1 + delta);
  }
  // src/hubbard.cpp:132-139: G -= delta/(1+(1-G_ii)delta) * G(:,i) (e_i^T - G(i,:))
  void update_green_function(Mat& g, int t, int i) const {
    const double delta = std::exp(-2 * alpha * s(t, i)) - 1;
    const double coef = delta / (1 + (1 - g(i, i)) * delta);
    Vec col(ns), row(ns);
    for (int k = 0; k < ns; ++k) { col[k] = g(k, i); row[k] = (k == i ? 1.0 : 0.0) - g(i, k); }
    for (int j = 0; j < ns; ++j) {
      const double rj = coef * row[j];
      for (int k = 0; k < ns; ++k) g(k, j) -= col[k] * rj;
    }
  }
};

// ------------------------------------------------------------------------------------
//  Utils::SvdStack<double>: include/utils/svd_stack.hpp:51-188, with
//  LinearAlgebra::mkl_lapack_dgesvd (include/utils/linear_algebra.hpp:46-99):
//  dgesvd('S','S'), V returned (not V^T).
// ------------------------------------------------------------------------------------
struct SvdStack {
  struct Entry { Mat u, v; Vec s; };
  std::vector<Entry> stack;
  int dim = 0, len = 0;
  SvdStack() = default;
  SvdStack(int d, int cap) : dim(d) {
    stack.resize(cap);
    for (auto& e : stack) { e.u = Mat(d); e.v = Mat(d); e.s.assign(d, 0.0); }
  }
  bool empty() const { return len == 0; }
  const Vec& S() const { return stack[len - 1].s; }
  const Mat& U() const { return stack[len - 1].u; }
  // svd_stack.hpp:95-103: V0 * V1 * ... * V_{len-1}
  Mat V() const {
    Mat r = stack[0].v;
    for (int i = 1; i < len; ++i) r = gemm(r, false, stack[i].v, false);
    return r;
  }
  static void dgesvd(const Mat& m, Mat& u, Vec& s, Mat& v) {
    const int n = m.n;
    Mat a = m, vt(n);
    Vec superb(std::max(1, n - 1));
    const int info = scipy_LAPACKE_dgesvd(kColMajor, 'S', 'S', n, n, a.data(), n, s.data(), u.data(), n, vt.data(),
                                          n, superb.data());
    if (info > 0) throw std::runtime_error("dgesvd: the algorithm failed to converge.");
    v = transpose(vt);
  }
  // svd_stack.hpp:107-175 (mixing order (M*U)*S at :144)
  void push(const Mat& m) {
    if (len >= int(stack.size())) throw std::runtime_error("SvdStack overflow");
    if (len == 0) {
      dgesvd(m, stack[0].u, stack[0].s, stack[0].v);
    } else {
      Mat tmp = gemm(m, false, U(), false);
      const Vec& sv = S();
      for (int j = 0; j < dim; ++j)
        for (int i = 0; i < dim; ++i) tmp(i, j) *= sv[j];
      dgesvd(tmp, stack[len].u, stack[len].s, stack[len].v);
    }
    ++len;
  }
  void pop() { assert(len > 0); --len; }
  void clear() { len = 0; }
};

// ------------------------------------------------------------------------------------
//  Utils::StableNumerics: include/utils/stable_numerics.hpp:37-324.
// ------------------------------------------------------------------------------------
// :37-48, signed maximum of (mat1 - mat2)
static double compare_error(const Mat& a, const Mat& b) {
  double e = -INFINITY;
  for (size_t k = 0; k < a.a.size(); ++k) e = std::max(e, a.a[k] - b.a[k]);
  return e;
}
// :56-64
static void div_dvec_max_min(const Vec& d, Vec& dmax, Vec& dmin) {
  dmax.resize(d.size()); dmin.resize(d.size());
  for (size_t i = 0; i < d.size(); ++i) { dmax[i] = std::max(d[i], 1.0); dmin[i] = std::min(d[i], 1.0); }
}
// :71-97  z(j,i) = sum_k v(j,k) u(k,i) / d(k)  (same loop order, scalar accumulator)
static Mat mult_v_invd_u(const Mat& v, const Vec& d, const Mat& u) {
  const int n = v.n;
  Mat z(n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double t = 0.0;
      for (int k = 0; k < n; ++k) t += v(j, k) * u(k, i) / d[k];
      z(j, i) = t;
    }
  return z;
}
// :104-130  z(j,i) = sum_k v(j,k) u(k,i) d(k)
static Mat mult_v_d_u(const Mat& v, const Vec& d, const Mat& u) {
  const int n = v.n;
  Mat z(n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double t = 0.0;
      for (int k = 0; k < n; ++k) t += v(j, k) * u(k, i) * d[k];
      z(j, i) = t;
    }
  return z;
}
// Solve H X = B with column-pivoted Householder QR (stands in for Eigen's
// fullPivHouseholderQr().solve at :154, :179).
static Mat qrp_solve(const Mat& H, const Mat& B) {
  const int n = H.n;
  Mat A = H, Y = B;
  std::vector<int> jpvt(n, 0);
  Vec tau(n);
  if (scipy_LAPACKE_dgeqp3(kColMajor, n, n, A.data(), n, jpvt.data(), tau.data()) != 0) throw std::runtime_error("dgeqp3");
  if (scipy_LAPACKE_dormqr(kColMajor, 'L', 'T', n, n, n, A.data(), n, tau.data(), Y.data(), n) != 0)
    throw std::runtime_error("dormqr");
  scipy_cblas_dtrsm(kColMajor, kLeft, kUpper, kNoTrans, kNonUnit, n, n, 1.0, A.data(), n, Y.data(), n);
  Mat X(n);
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j) X(jpvt[k] - 1, j) = Y(k, j);
  return X;
}
// :136-155  (1 + U S V^T)^-1
static Mat compute_gf_00bb(const Mat& u, const Vec& s, const Mat& v) {
  const int n = u.n;
  Vec sl(n), sr(n);
  for (int i = 0; i < n; ++i) {
    if (s[i] > 1.) { sl[i] = 1. / s[i]; sr[i] = 1.; } else { sl[i] = 1.; sr[i] = s[i]; }
  }
  Mat H(n), R(n);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      H(i, j) = sl[i] * u(j, i) + sr[i] * v(j, i);
      R(i, j) = sl[i] * u(j, i);
    }
  return qrp_solve(H, R);
}
// :186-239
static Mat compute_equaltime_gf(const SvdStack& left, const SvdStack& right) {
  if (left.empty()) return compute_gf_00bb(right.V(), right.S(), right.U());
  if (right.empty()) return compute_gf_00bb(left.U(), left.S(), left.V());
  const int n = left.dim;
  const Mat ul = left.U(), vl = left.V(), ur = right.U(), vr = right.V();
  const Vec dl = left.S(), dr = right.S();
  Vec dlmax, dlmin, drmax, drmin;
  div_dvec_max_min(dl, dlmax, dlmin);
  div_dvec_max_min(dr, drmax, drmin);
  Mat A = gemm(ul, true, ur, false), B = gemm(vl, true, vr, false), T(n);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      A(i, j) = A(i, j) / (dlmax[i] * drmax[j]);
      B(i, j) = B(i, j) * dlmin[i] * drmin[j];
      T(i, j) = A(i, j) + B(i, j);
    }
  Mat tA = mult_v_invd_u(ur, drmax, inverse(T));
  return mult_v_invd_u(tA, dlmax, transpose(ul));
}
// :245-324
static void compute_dynamic_gf(const SvdStack& left, const SvdStack& right, Mat& gt0, Mat& g0t, Mat& gtt) {
  const int n = left.dim;
  if (left.empty()) {
    gtt = compute_gf_00bb(right.V(), right.S(), right.U());
    gt0 = gtt;
    g0t = gtt;
    for (int i = 0; i < n; ++i) g0t(i, i) -= 1.0;  // -(1 - gtt)
    return;
  }
  if (right.empty()) {
    gtt = compute_gf_00bb(left.U(), left.S(), left.V());
    gt0 = Mat(n);
    g0t = Mat(n);
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) { gt0(i, j) = (i == j ? 1.0 : 0.0) - gtt(i, j); g0t(i, j) = -gtt(i, j); }
    return;
  }
  const Mat ul = left.U(), vl = left.V(), ur = right.U(), vr = right.V();
  const Vec dl = left.S(), dr = right.S();
  Vec dlmax, dlmin, drmax, drmin;
  div_dvec_max_min(dl, dlmax, dlmin);
  div_dvec_max_min(dr, drmax, drmin);
  Mat A = gemm(ul, true, ur, false), B = gemm(vl, true, vr, false), T(n);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      A(i, j) = A(i, j) / (dlmax[i] * drmax[j]);
      B(i, j) = B(i, j) * dlmin[i] * drmin[j];
      T(i, j) = A(i, j) + B(i, j);
    }
  Mat tA = mult_v_invd_u(ur, drmax, inverse(T));
  gtt = mult_v_invd_u(tA, dlmax, transpose(ul));
  gt0 = mult_v_d_u(tA, dlmin, transpose(vl));
  Mat C = gemm(vr, true, vl, false), D = gemm(ur, true, ul, false);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      C(i, j) = C(i, j) / (drmax[i] * dlmax[j]);
      D(i, j) = D(i, j) * drmin[i] * dlmin[j];
      T(i, j) = C(i, j) + D(i, j);
    }
  Mat mvl = vl;
  for (auto& x : mvl.a) x = -x;
  Mat tC = mult_v_invd_u(mvl, dlmax, inverse(T));
  g0t = mult_v_d_u(tC, drmin, transpose(ur));
}

// ------------------------------------------------------------------------------------
//  DQMC::Core: src/dqmc_core.cpp:20-390.
// ------------------------------------------------------------------------------------
struct Core {
  int ns = 0, nt = 0, pace = 0;
  bool is_equaltime = false, is_dynamic = false, is_thermalization = false;
  double wrap_err_tt = 0.0, wrap_err_dyn = 0.0;
  int current_t = 0;
  Mat gftt, gft0, gf0t;
  std::vector<Mat> vecgftt, vecgft0, vecgf0t;
  SvdStack left, right;
  std::default_random_engine* eng = nullptr;
  // counters (not in the reference): proposals and acceptances, for acceptance-rate reports
  long long n_proposed = 0, n_accepted = 0;
  // optional replay log: every acceptance ratio in visiting order
  std::vector<double>* ratio_log = nullptr;
  // optional forced trajectory (test infrastructure, not in the reference): when set, site
  // (t, i) flips iff forced[t*ns + i] differs from its current field; the random draw of
  // the reference is still consumed. It replays another implementation's field trajectory
  // so that its G's can be compared at any stabilisation pace.
  const std::vector<int>* forced = nullptr;

  void initialize(const Params& p) {
    ns = p.ns; nt = p.nt; pace = p.pace; is_equaltime = p.is_equaltime; is_dynamic = p.is_dynamic;
  }
  int stack_length() const { return nt % pace == 0 ? nt / pace : nt / pace + 1; }
  int t2index(int t) const { return t % nt; }  // :129-133

  // :67-87
  void initialize_svdstacks(const Model& model) {
    left = SvdStack(ns, nt);
    right = SvdStack(ns, nt);
    Mat stacks = Mat::Identity(ns);
    for (int t = nt; t >= 1; --t) {
      model.multiply_adjB_from_left(stacks, t2index(t));
      if ((t - 1) % pace == 0) { right.push(stacks); stacks = Mat::Identity(ns); }
    }
  }
  // :89-97 (with the allocations of :43-65)
  void initialize_green_functions() {
    gftt = compute_equaltime_gf(left, right);
    if (is_equaltime || is_dynamic) vecgftt.assign(nt, Mat(ns));
    if (is_dynamic) { gft0 = Mat(ns); gf0t = Mat(ns); vecgft0.assign(nt, Mat(ns)); vecgf0t.assign(nt, Mat(ns)); }
  }
  // :102-119
  void metropolis_update(Model& model, int t) {
    for (int i = 0; i < ns; ++i) {
      const double r = model.acceptance_ratio(gftt, t, i);
      if (ratio_log) ratio_log->push_back(r);
      ++n_proposed;
      bool accept = std::bernoulli_distribution(std::min(1.0, std::abs(r)))(*eng);
      if (forced) accept = (*forced)[size_t(t) * ns + i] != model.s(t, i);
      if (accept) {
        model.update_green_function(gftt, t, i);
        model.s(t, i) = -model.s(t, i);  // src/hubbard.cpp:118-121
        ++n_accepted;
      }
    }
  }
  // :142-147
  void wrap_from_0_to_beta(const Model& m, int t) {
    m.multiply_B_from_left(gftt, t2index(t + 1));
    m.multiply_invB_from_right(gftt, t2index(t + 1));
  }
  // :156-161
  void wrap_from_beta_to_0(const Model& m, int t) {
    m.multiply_B_from_right(gftt, t2index(t));
    m.multiply_invB_from_left(gftt, t2index(t));
  }
  void stabilise_equaltime() {
    Mat tmp = compute_equaltime_gf(left, right);
    wrap_err_tt = std::max(wrap_err_tt, compare_error(tmp, gftt));
    gftt = tmp;
  }
  // :167-227
  void sweep_from_0_to_beta(Model& model) {
    if (current_t != 0 || !left.empty() || right.len != stack_length())
      throw std::runtime_error("sweep_from_0_to_beta: stacks not at tau=0");
    Mat stacks = Mat::Identity(ns);
    for (int t = 1; t <= nt; ++t) {
      ++current_t;
      wrap_from_0_to_beta(model, t - 1);
      metropolis_update(model, t2index(t));
      model.multiply_B_from_left(stacks, t2index(t));
      if (t % pace == 0 || t == nt) {
        right.pop();
        left.push(stacks);
        stabilise_equaltime();
        stacks = Mat::Identity(ns);
      }
      if (!is_thermalization && is_equaltime) vecgftt[t2index(t)] = gftt;
    }
  }
  // :233-284
  void sweep_from_beta_to_0(Model& model) {
    if (current_t != nt || !right.empty() || left.len != stack_length())
      throw std::runtime_error("sweep_from_beta_to_0: stacks not at tau=beta");
    Mat stacks = Mat::Identity(ns);
    for (int t = nt; t >= 1; --t) {
      metropolis_update(model, t2index(t));
      model.multiply_adjB_from_left(stacks, t2index(t));
      wrap_from_beta_to_0(model, t);
      if ((t - 1) % pace == 0) {
        left.pop();
        right.push(stacks);
        stabilise_equaltime();
        stacks = Mat::Identity(ns);
      }
      if (!is_thermalization && is_equaltime) vecgftt[t2index(t - 1)] = gftt;
      --current_t;
    }
  }
  // :291-390
  void sweep_for_dynamic_green_functions(Model& model) {
    if (!is_dynamic) return;
    if (current_t != 0 || !left.empty() || right.len != stack_length())
      throw std::runtime_error("sweep_for_dynamic_green_functions: stacks not at tau=0");
    gft0 = gftt;
    gf0t = gftt;
    for (int i = 0; i < ns; ++i) gf0t(i, i) -= 1.0;
    Mat stacks = Mat::Identity(ns);
    for (int t = 1; t <= nt; ++t) {
      ++current_t;
      wrap_from_0_to_beta(model, t - 1);
      model.multiply_B_from_left(gft0, t2index(t));
      model.multiply_invB_from_right(gf0t, t2index(t));
      model.multiply_B_from_left(stacks, t2index(t));
      if (t % pace == 0 || t == nt) {
        right.pop();
        left.push(stacks);
        Mat tt, t0, ot;
        compute_dynamic_gf(left, right, t0, ot, tt);
        wrap_err_tt = std::max(wrap_err_tt, compare_error(tt, gftt));
        wrap_err_dyn = std::max(wrap_err_dyn, std::max(compare_error(t0, gft0), compare_error(ot, gf0t)));
        gftt = tt; gft0 = t0; gf0t = ot;
        stacks = Mat::Identity(ns);
      }
      vecgftt[t2index(t)] = gftt;
      if (t2index(t) != 0) {
        vecgft0[t2index(t)] = gft0;
        vecgf0t[t2index(t)] = gf0t;
      } else {
        vecgft0[0] = gftt;
        vecgf0t[0] = gftt;
        for (int i = 0; i < ns; ++i) vecgf0t[0](i, i) -= 1.0;
      }
    }
  }
};

// ------------------------------------------------------------------------------------
//  Estimators: include/observable_methods.hpp:39-195.
// ------------------------------------------------------------------------------------
static double measure_filling(const Core& c) {  // :39-52
  double f = 0.0;
  for (int t = 0; t < c.nt; ++t) {
    double tr = 0.0;
    for (int i = 0; i < c.ns; ++i) tr += c.vecgftt[t](i, i);
    f += 2. - (tr + tr) / c.ns;
  }
  return f / c.nt;
}
static double measure_double_occupation(const Core& c) {  // :59-74
  double d = 0.0;
  for (int t = 0; t < c.nt; ++t)
    for (int i = 0; i < c.ns; ++i) d += (1. - c.vecgftt[t](i, i)) * (1. - c.vecgftt[t](i, i));
  return d / (c.ns * c.nt);
}
static double measure_swave(const Core& c) {  // :131-151
  double p = 0.0;
  for (int t = 0; t < c.nt; ++t) {
    const Mat& g = c.vecgftt[t];
    for (int i = 0; i < c.ns; ++i)
      for (int j = 0; j < c.ns; ++j) {
        const double gc = (i == j ? 1.0 : 0.0) - g(j, i);
        p += gc * gc + g(i, j) * g(i, j);
      }
  }
  return p / (c.ns * c.nt);
}
static void measure_spin_corr(const Core& c, double* out) {  // :178-195, out[nt] +=
  for (int t = 0; t < c.nt; ++t) {
    double s = 0.0;
    for (int i = 0; i < c.ns; ++i) s -= c.vecgf0t[t](i, i) * c.vecgft0[t](i, i) + c.vecgf0t[t](i, i) * c.vecgft0[t](i, i);
    out[t] += s / (2 * c.ns);
  }
}
static void measure_ldos(const Core& c, double* out) {  // :110-120
  for (int t = 0; t < c.nt; ++t) {
    double tr = 0.0;
    for (int i = 0; i < c.ns; ++i) tr += c.vecgft0[t](i, i);
    out[t] += tr / c.ns;
  }
}
static void measure_dynamic_gf(const Core& c, const Lattice& lat, const std::vector<int>& klist, double* out) {
  // :84-103, out[k*nt + t] +=
  const int nk = int(klist.size());
  for (int t = 0; t < c.nt; ++t) {
    const Mat& g = c.vecgft0[t];
    for (int k = 0; k < nk; ++k) {
      double acc = 0.0;
      for (int i = 0; i < c.ns; ++i)
        for (int j = 0; j < c.ns; ++j) {
          const auto ff = lat.fourier[lat.disp[i + size_t(j) * c.ns] + size_t(klist[k]) * c.ns];
          acc += (ff * g(j, i)).real() / c.ns;
        }
      out[k * c.nt + t] += acc;
    }
  }
}

// ------------------------------------------------------------------------------------
//  One Markov chain: model + core + its own engine (the reference keeps one global
//  engine per MPI rank, src/random.cpp:14; one chain per engine is the same stream).
// ------------------------------------------------------------------------------------
struct Chain {
  Params p;
  Lattice lat;
  Model model;
  Core core;
  std::default_random_engine eng;
};

}  // namespace oracle

using namespace oracle;

// =====================================================================================
//  C ABI for the test harness (ctypes).
// =====================================================================================
extern "C" {

void or_set_num_threads(int n) { scipy_openblas_set_num_threads(n); }

void* or_create(int nl, double nnt, double u, double mu, double beta, int nt, int pace, int is_equaltime,
                int is_dynamic, long long seed, const double* custom_hop) {
  try {
    auto* c = new Chain();
    c->p.nl = nl; c->p.ns = nl * nl; c->p.nt = nt; c->p.pace = pace;
    c->p.beta = beta; c->p.dt = beta / nt; c->p.nnt = nnt; c->p.mu = mu; c->p.u = u;
    c->p.is_equaltime = is_equaltime; c->p.is_dynamic = is_dynamic;
    c->lat.initialize(nl);
    Mat hop;
    if (custom_hop) { hop = Mat(c->p.ns); std::memcpy(hop.data(), custom_hop, sizeof(double) * hop.a.size()); }
    c->model.initialize(c->p, c->lat, custom_hop ? &hop : nullptr);
    c->core.initialize(c->p);
    c->eng.seed(static_cast<std::default_random_engine::result_type>(seed));  // src/random.cpp:15
    c->core.eng = &c->eng;
    return c;
  } catch (...) { return nullptr; }
}
void or_destroy(void* h) {
  auto* c = static_cast<Chain*>(h);
  delete c->core.forced;
  delete c->core.ratio_log;
  delete c;
}
double or_alpha(void* h) { return static_cast<Chain*>(h)->model.alpha; }
void or_get_expk(void* h, double* expk, double* inv_expk) {
  auto* c = static_cast<Chain*>(h);
  std::memcpy(expk, c->model.expK.data(), sizeof(double) * c->model.expK.a.size());
  std::memcpy(inv_expk, c->model.inv_expK.data(), sizeof(double) * c->model.inv_expK.a.size());
}
void or_fields_random(void* h) { auto* c = static_cast<Chain*>(h); c->model.set_fields_random(c->eng); }
void or_set_fields(void* h, const int* f) { auto* c = static_cast<Chain*>(h); std::memcpy(c->model.fields.data(), f, sizeof(int) * c->model.fields.size()); }
void or_get_fields(void* h, int* f) { auto* c = static_cast<Chain*>(h); std::memcpy(f, c->model.fields.data(), sizeof(int) * c->model.fields.size()); }
// raw engine draws (for RNG replay checks)
void or_engine_draws(void* h, long long n, unsigned int* out) {
  auto* c = static_cast<Chain*>(h);
  for (long long k = 0; k < n; ++k) out[k] = static_cast<unsigned int>(c->eng());
}
void or_canonical_draws(void* h, long long n, double* out) {
  auto* c = static_cast<Chain*>(h);
  for (long long k = 0; k < n; ++k) out[k] = std::generate_canonical<double, std::numeric_limits<double>::digits>(c->eng);
}
int or_init(void* h) {
  auto* c = static_cast<Chain*>(h);
  try {
    c->core.initialize_svdstacks(c->model);
    c->core.initialize_green_functions();
    c->core.current_t = 0;
    return 0;
  } catch (...) { return -1; }
}
// forced field trajectory (see Core::forced): target [nt][ns] or NULL to return to Metropolis
void or_set_forced_fields(void* h, const int* target) {
  auto* c = static_cast<Chain*>(h);
  delete c->core.forced;
  c->core.forced = target ? new std::vector<int>(target, target + size_t(c->p.nt) * c->p.ns) : nullptr;
}
void or_set_thermalization(void* h, int on) { static_cast<Chain*>(h)->core.is_thermalization = on; }
int or_sweep(void* h, int dir) {
  auto* c = static_cast<Chain*>(h);
  try {
    if (dir == 0) c->core.sweep_from_0_to_beta(c->model);
    else if (dir == 1) c->core.sweep_from_beta_to_0(c->model);
    else c->core.sweep_for_dynamic_green_functions(c->model);
    return 0;
  } catch (...) { return -1; }
}
void or_current_g(void* h, double* out) { auto* c = static_cast<Chain*>(h); std::memcpy(out, c->core.gftt.data(), sizeof(double) * c->core.gftt.a.size()); }
// which: 0 = gftt, 1 = gft0, 2 = gf0t, slice t in [0, nt)
int or_get_g(void* h, int which, int t, double* out) {
  auto* c = static_cast<Chain*>(h);
  const std::vector<Mat>* v = which == 0 ? &c->core.vecgftt : which == 1 ? &c->core.vecgft0 : &c->core.vecgf0t;
  if (t < 0 || t >= int(v->size())) return -1;
  std::memcpy(out, (*v)[t].data(), sizeof(double) * (*v)[t].a.size());
  return 0;
}
void or_current_dyn(void* h, double* gt0, double* g0t) {
  auto* c = static_cast<Chain*>(h);
  std::memcpy(gt0, c->core.gft0.data(), sizeof(double) * c->core.gft0.a.size());
  std::memcpy(g0t, c->core.gf0t.data(), sizeof(double) * c->core.gf0t.a.size());
}
void or_wrap_errors(void* h, double* out2) { auto* c = static_cast<Chain*>(h); out2[0] = c->core.wrap_err_tt; out2[1] = c->core.wrap_err_dyn; }
void or_counts(void* h, long long* out2) { auto* c = static_cast<Chain*>(h); out2[0] = c->core.n_proposed; out2[1] = c->core.n_accepted; }
void or_set_ratio_log(void* h, int on) {
  auto* c = static_cast<Chain*>(h);
  if (on) { delete c->core.ratio_log; c->core.ratio_log = new std::vector<double>(); } else { delete c->core.ratio_log; c->core.ratio_log = nullptr; }
}
long long or_ratio_log(void* h, double* out, long long cap) {
  auto* c = static_cast<Chain*>(h);
  if (!c->core.ratio_log) return 0;
  const long long n = std::min<long long>(cap, c->core.ratio_log->size());
  if (out) std::memcpy(out, c->core.ratio_log->data(), sizeof(double) * n);
  return (long long)c->core.ratio_log->size();
}
// equal-time estimators from vecgftt: out[0..2] = filling, double occupancy, s-wave
void or_measure_equaltime(void* h, double* out3) {
  auto* c = static_cast<Chain*>(h);
  out3[0] = measure_filling(c->core);
  out3[1] = measure_double_occupation(c->core);
  out3[2] = measure_swave(c->core);
}
// dynamic estimators: spin[nt], ldos[nt], gfk[nk*nt] (accumulated, caller zeroes)
void or_measure_dynamic(void* h, double* spin, double* ldos, const int* klist, int nk, double* gfk) {
  auto* c = static_cast<Chain*>(h);
  measure_spin_corr(c->core, spin);
  measure_ldos(c->core, ldos);
  if (nk > 0) measure_dynamic_gf(c->core, c->lat, std::vector<int>(klist, klist + nk), gfk);
}
int or_nkstars(void* h) { return static_cast<Chain*>(h)->lat.nkstars; }

// -------------------------------------------------------------------------------------
//  Full measurement schedule of DQMC::Handle (src/dqmc_handle.cpp:56-162) for one chain.
//  bins_eq[bin*3 + o] for o in (filling, double occupancy, s-wave);
//  bins_spin[bin*nt + t], bins_ldos[bin*nt + t], bins_gfk[(bin*nk + k)*nt + t].
//  Bin values are normalised by the measurement count (include/observable.hpp:168-177).
// -------------------------------------------------------------------------------------
int or_run_schedule(void* h, int sweeps_warmup, int bin_num, int bin_capacity, int sweeps_between_bins,
                    int measure_eq, int measure_dyn, const int* klist, int nk, double* bins_eq, double* bins_spin,
                    double* bins_ldos, double* bins_gfk) {
  auto* c = static_cast<Chain*>(h);
  Core& core = c->core;
  Model& m = c->model;
  const int nt = c->p.nt;
  try {
    if (sweeps_warmup > 0) {
      core.is_thermalization = true;
      for (int s = 1; s <= int(std::ceil(sweeps_warmup / 2.)); ++s) {
        core.sweep_from_0_to_beta(m);
        core.sweep_from_beta_to_0(m);
      }
    }
    const bool is_eq = measure_eq && bin_num > 0 && bin_capacity > 0;
    const bool is_dyn = measure_dyn && bin_num > 0 && bin_capacity > 0;
    if (!(is_eq || is_dyn)) return 0;
    const int binsize = is_dyn ? bin_capacity : int(std::ceil(bin_capacity / 2.));
    core.is_thermalization = false;
    std::vector<int> kl(klist, klist + nk);
    for (int bin = 0; bin < bin_num; ++bin) {
      for (int s = 1; s <= int(std::ceil(sweeps_between_bins / 2.)); ++s) {
        core.sweep_from_0_to_beta(m);
        core.sweep_from_beta_to_0(m);
      }
      double eq[3] = {0, 0, 0};
      int neq = 0, ndyn = 0;
      std::vector<double> spin(nt, 0.0), ldos(nt, 0.0), gfk(size_t(nk) * nt, 0.0);
      for (int s = 1; s <= binsize; ++s) {
        if (is_dyn) {
          core.sweep_for_dynamic_green_functions(m);
          measure_spin_corr(core, spin.data());
          measure_ldos(core, ldos.data());
          if (nk > 0) measure_dynamic_gf(core, c->lat, kl, gfk.data());
          ++ndyn;
        } else {
          core.sweep_from_0_to_beta(m);
          eq[0] += measure_filling(core); eq[1] += measure_double_occupation(core); eq[2] += measure_swave(core);
          ++neq;
        }
        core.sweep_from_beta_to_0(m);
        if (is_eq) {
          eq[0] += measure_filling(core); eq[1] += measure_double_occupation(core); eq[2] += measure_swave(core);
          ++neq;
        }
      }
      if (is_eq && bins_eq) for (int o = 0; o < 3; ++o) bins_eq[bin * 3 + o] = eq[o] / neq;
      if (is_dyn) {
        for (int t = 0; t < nt; ++t) {
          if (bins_spin) bins_spin[size_t(bin) * nt + t] = spin[t] / ndyn;
          if (bins_ldos) bins_ldos[size_t(bin) * nt + t] = ldos[t] / ndyn;
          for (int k = 0; k < nk; ++k)
            if (bins_gfk) bins_gfk[(size_t(bin) * nk + k) * nt + t] = gfk[size_t(k) * nt + t] / ndyn;
        }
      }
    }
    return 0;
  } catch (...) { return -1; }
}

// top of the left (side 0) or right (side 1) SVD stack as the product U S V^T of all its
// entries (include/utils/svd_stack.hpp:83-103), column-major N x N; returns the stack length
// (checker for hq_get_stack)
int or_stack_top(void* h, int side, double* prod) {
  auto* c = static_cast<Chain*>(h);
  const SvdStack& st = side == 0 ? c->core.left : c->core.right;
  if (st.empty()) return 0;
  Mat us = st.U();
  const Vec& sv = st.S();
  for (int j = 0; j < us.n; ++j)
    for (int i = 0; i < us.n; ++i) us(i, j) *= sv[j];
  const Mat pr = gemm(us, false, st.V(), true);
  std::copy(pr.a.begin(), pr.a.end(), prod);
  return st.len;
}

// -------------------------------------------------------------------------------------
//  log|det(1 + B_nt ... B_1)| of the current fields and its exact gradient identities
//  (no counterpart in the reference; checker for the adjoint kernel).
//  logdet: stable evaluation from the right stack at tau=0 (U S V^T with U, V orthogonal):
//     log|det(1 + U S V^T)| = sum_i log smax_i + log|det(smax^-1 U^T V + smin)|.
// -------------------------------------------------------------------------------------
double or_logdet(void* h) {
  auto* c = static_cast<Chain*>(h);
  // product of the plain B chain X = B(nt-1)...B(0) via an SVD stack of B products,
  // stabilised every `pace` slices.
  const int n = c->p.ns, nt = c->p.nt, pace = c->p.pace;
  SvdStack st(n, nt);
  Mat acc = Mat::Identity(n);
  for (int t = 1; t <= nt; ++t) {
    c->model.multiply_B_from_left(acc, t % nt);
    if (t % pace == 0 || t == nt) { st.push(acc); acc = Mat::Identity(n); }
  }
  const Mat U = st.U(), V = st.V();
  const Vec S = st.S();
  Vec smax, smin;
  div_dvec_max_min(S, smax, smin);
  Mat M = gemm(U, true, V, false);
  double ld = 0.0;
  for (int i = 0; i < n; ++i) ld += std::log(smax[i]);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) M(i, j) = M(i, j) / smax[i] + (i == j ? smin[i] : 0.0);
  std::vector<int> ipiv(n);
  scipy_LAPACKE_dgetrf(kColMajor, n, n, M.data(), n, ipiv.data());
  for (int i = 0; i < n; ++i) ld += std::log(std::abs(M(i, i)));
  // |det U| = |det V| = 1
  return ld;
}

// Gradient identities from the equal-time G at every slice l (G_l after B(l) applied in
// the up direction): d/dmu = dt * sum_l tr(1 - G_l); d/dalpha = sum_l sum_i s_li (1-G_l)_ii;
// d/dK_ij = Gamma_ij with Gamma from the Daleckii-Krein formula. Uses a no-update pass of
// wrapped-and-stabilised G's (state must be at tau = 0 with initialised stacks).
// out: [dmu, dalpha, dK (n*n, column-major)]
int or_logdet_grad(void* h, double* out) {
  auto* c = static_cast<Chain*>(h);
  const int n = c->p.ns, nt = c->p.nt;
  Model& m = c->model;
  // fresh G_l for each slice from stacks (no wrapping shortcuts: the checker favours accuracy)
  double dmu = 0.0, dal = 0.0;
  Mat D(n);  // sum_l exp(-V_l) (1 - G_l) exp(V_l)
  for (int l = 1; l <= nt; ++l) {
    // G_l = (1 + B_l..B_1 B_nt..B_{l+1})^-1 ; build with SVD stacks
    SvdStack L(n, nt), R(n, nt);
    Mat acc = Mat::Identity(n);
    int cnt = 0;
    for (int t = 1; t <= l; ++t) {
      m.multiply_B_from_left(acc, t % nt);
      if (++cnt == c->p.pace || t == l) { L.push(acc); acc = Mat::Identity(n); cnt = 0; }
    }
    acc = Mat::Identity(n);
    cnt = 0;
    for (int t = nt; t >= l + 1; --t) {
      m.multiply_adjB_from_left(acc, t % nt);
      if (++cnt == c->p.pace || t == l + 1) { R.push(acc); acc = Mat::Identity(n); cnt = 0; }
    }
    Mat G = compute_equaltime_gf(L, R);
    const int sl = l % nt;
    for (int i = 0; i < n; ++i) {
      dmu += c->p.dt * (1.0 - G(i, i));
      dal += m.s(sl, i) * (1.0 - G(i, i));
    }
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        const double v = (i == j ? 1.0 : 0.0) - G(i, j);
        D(i, j) += v * std::exp(-m.alpha * m.s(sl, i) + m.alpha * m.s(sl, j));
      }
  }
  // M = E^-1 D ; dlogdet = tr(dE M) ; E = Q diag(f(lam)) Q^T, f = exp(-dt lam)
  Mat Mx = gemm(m.inv_expK, false, D, false);
  Mat Q = m.K;
  Vec w(n);
  scipy_LAPACKE_dsyev(kColMajor, 'V', 'U', n, Q.data(), n, w.data());
  Mat Mt = gemm(gemm(Q, true, Mx, false), false, Q, false);  // Q^T M Q
  Mat Phi(n);
  const double dt = c->p.dt;
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      const double fi = std::exp(-dt * w[i]), fj = std::exp(-dt * w[j]);
      const double dd = std::abs(w[i] - w[j]) > 1e-10 ? (fi - fj) / (w[i] - w[j]) : -dt * 0.5 * (fi + fj);
      Phi(i, j) = dd * Mt(j, i);
    }
  Mat Gam = gemm(gemm(Q, false, Phi, false), false, Q, true);
  out[0] = dmu;
  out[1] = dal;
  std::memcpy(out + 2, Gam.data(), sizeof(double) * n * n);
  return 0;
}

}  // extern "C"
