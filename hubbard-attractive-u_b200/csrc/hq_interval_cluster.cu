// hq_interval_cluster.cu -- k_interval_cl: the interval kernel (wrap + Metropolis flips with
// DMMA-flushed submatrix updates, src/dqmc_core.cpp:102-161) for the 16 x 16 lattice, whose
// G (N = 256, 512 KB) does not fit in one SM's shared memory. One chain runs on a cluster of
// four CTAs; CTA r holds the 64 columns [64 r, 64 r + 64) of G in its shared memory for the
// whole interval, and the CTAs reach each other's columns through distributed shared memory
// (DSMEM: generic loads of cluster-mapped shared addresses, barrier.cluster between phases).
// No TMA multicast and no other GPU's memory are involved.
//
// Per slice:
//  * wrap, separable form exp(-dt K) = c (A (x) A) (the same passes as the one-CTA kernel):
//    the row-side passes and the x-pass of the column side act on local columns only; the
//    y-pass of the column side mixes columns o + 16 e of all four CTAs, so it reads the
//    other CTAs' columns through DSMEM in chunks of 16 rows (reads, cluster barrier, writes);
//  * Metropolis in 16-site blocks: the block's 16 columns live in one CTA (the owner), whose
//    warp 0 walks the block exactly as the one-CTA kernel does; the owner forms the panel X
//    (all N rows, from its own columns); every CTA forms Y for its own columns from the walk's
//    records, copies X from the owner through DSMEM and flushes G[:, own] += X Y by DMMA.
// Each element of G sees the same sequence of floating-point operations as in the one-CTA
// kernel with G in global memory, so both paths give the same G.
#include <cooperative_groups.h>

#include "hq_metropolis.cuh"

namespace cg = cooperative_groups;

namespace hq {

namespace {
constexpr int kCl = 4;          // CTAs per cluster (one chain)
constexpr int kL = 16;          // lattice size of the cluster path
constexpr int kN = kL * kL;     // sites
constexpr int kNC = kN / kCl;   // columns per CTA (a multiple of the 16-site blocks and of L)
constexpr int kLd = interval_ld(kN);       // = 2 (mod 8): conflict-free DMMA accumulator tiles
constexpr int kLdx = panel_ld(kN);         // X panel (N x 16)
constexpr int kLdy = panel_ld(kNC);        // Y panel (16 x NC)
constexpr int kNE = kNC / kL;              // y values (x-fibres) of the column side held per CTA
}  // namespace

__host__ __device__ inline size_t interval_cl_smem_doubles() {
  return (size_t)kNC * kLd + (size_t)kLdx * 16 + (size_t)16 * kLdy + 3 * kNC + kNC / 2 + (kN + kNC + 7) / 8 + 16;
}
size_t smem_interval_cl_bytes() { return interval_cl_smem_doubles() * sizeof(double); }

bool interval_cluster_ok(int N, int L, int expk_mode, int kmax) {
  return N == kN && L == kL && expk_mode == HQK_EXPK_SEPARABLE && kmax == 16;
}

// One local pass of the separable exp(-dt K) on this CTA's columns (side 0: along the rows of
// every local column; side 1, pass 0: along x inside the rows' local y values). The same
// arithmetic as sep_pass (scaling on load / store, L accumulators summed in ascending order).
template <int SIDE, int PASS, int SC>
__device__ __forceinline__ void cl_local_pass(double* Gc, int c0, const double* __restrict__ coef, double cmul,
                                              const int8_t* sf, double rp, double rm, double cp, double cm) {
  static_assert(SIDE == 0 || PASS == 0, "the column-side y-pass exchanges data");
  double a[kL];
#pragma unroll
  for (int d = 0; d < kL; ++d) a[d] = coef[d];
  // side 0: lines = local columns (kNC), fibres per line: kL (o); side 1: lines = rows (kN), o = local y
  constexpr int nfib = (SIDE == 0) ? kNC * kL : kN * kNE;
  for (int f = threadIdx.x; f < nfib; f += blockDim.x) {
    int line, o;
    if (SIDE == 0) { line = f % kNC; o = f / kNC; } else { line = f % kN; o = c0 / kL + f / kN; }
    const int base_site = (SIDE == 0 && PASS == 1) ? o : kL * o;
    const int step_site = (SIDE == 0 && PASS == 1) ? kL : 1;
    double* base;
    size_t stride;
    if (SIDE == 0) { base = Gc + base_site + (size_t)line * kLd; stride = (size_t)step_site; }
    else { base = Gc + line + (size_t)(base_site - c0) * kLd; stride = (size_t)kLd; }
    const int line_site = (SIDE == 0) ? c0 + line : line;
    double lf = 1.0, sp = 1.0, sm = 1.0;
    if (SC) {
      const bool lpos = sf[line_site] > 0;
      lf = (SIDE == 0) ? (lpos ? cp : cm) : (lpos ? rp : rm);
      sp = (SIDE == 0) ? rp : cp;
      sm = (SIDE == 0) ? rm : cm;
    }
    double v[kL];
#pragma unroll
    for (int e = 0; e < kL; ++e) {
      v[e] = base[e * stride];
      if (SC == 1) {
        const double sfac = sf[base_site + e * step_site] > 0 ? sp : sm;
        v[e] *= (SIDE == 0) ? sfac * lf : lf * sfac;
      }
    }
    double acc[kL];
#pragma unroll
    for (int e = 0; e < kL; ++e) acc[e] = 0.0;
#pragma unroll
    for (int e2 = 0; e2 < kL; ++e2) {
#pragma unroll
      for (int e = 0; e < kL; ++e) acc[e] = fma(a[(e - e2 + kL) % kL], v[e2], acc[e]);
    }
#pragma unroll
    for (int e = 0; e < kL; ++e) {
      double out = (PASS == 1) ? acc[e] * cmul : acc[e];
      if (SC == 2) {
        const double sfac = sf[base_site + e * step_site] > 0 ? sp : sm;
        out *= (SIDE == 0) ? sfac * lf : lf * sfac;
      }
      base[e * stride] = out;
    }
  }
}

// The y-pass of the column side (M <- M (1 (x) A) along y, times cmul; SC = 2 scales on store
// by row factor (rp / rm) x column factor (cp / cm)): the fibre of row i and x = o holds the
// columns o + 16 e, e = 0..15, four in each CTA. Rows are taken 16 at a time (one fibre per
// thread): every thread reads its fibre's 16 inputs (12 of them from the other CTAs), the
// cluster barrier lets every CTA finish reading, then each CTA writes its own 4 outputs.
// coef lives in the chain descriptor in shared memory: the rotation by this CTA's e_lo is a
// runtime index, which a register array would turn into a local-memory one.
template <int SC>
__device__ __forceinline__ void cl_exchange_pass(double* Gc, double* const* Gr, int c0, const double* coef, double cmul,
                                                 const int8_t* sf, double rp, double rm, double cp, double cm,
                                                 cg::cluster_group& cluster) {
  constexpr int rows_per_chunk = HQ_INT_THREADS / kL;
  const int o = threadIdx.x % kL;
  const int e_lo = c0 / kL;  // this CTA's outputs: e = e_lo .. e_lo + kNE - 1
  for (int r0 = 0; r0 < kN; r0 += rows_per_chunk) {
    const int i = r0 + threadIdx.x / kL;
    double v[kL];
#pragma unroll
    for (int e2 = 0; e2 < kL; ++e2) {
      // column o + 16 e2 is local column o + 16 (e2 % 4) of CTA e2 / 4
      v[e2] = Gr[e2 / kNE][i + (size_t)(o + kL * (e2 % kNE)) * kLd];
    }
    double acc[kNE];
#pragma unroll
    for (int k = 0; k < kNE; ++k) acc[k] = 0.0;
#pragma unroll
    for (int e2 = 0; e2 < kL; ++e2) {
#pragma unroll
      for (int k = 0; k < kNE; ++k) acc[k] = fma(coef[(e_lo + k - e2 + kL) % kL], v[e2], acc[k]);
    }
    cluster.sync();  // every CTA has read this chunk's rows
    double lf = 1.0;
    if (SC) lf = sf[i] > 0 ? rp : rm;
#pragma unroll
    for (int k = 0; k < kNE; ++k) {
      const int j = o + kL * (e_lo + k);
      double out = acc[k] * cmul;
      if (SC == 2) {
        const double sfac = sf[j] > 0 ? cp : cm;
        out *= lf * sfac;
      }
      Gc[i + (size_t)(j - c0) * kLd] = out;
    }
  }
  __syncthreads();
}

// wrap of this CTA's columns by B(l) (the cluster form of wrap_slice's separable branch)
__device__ __forceinline__ void cl_wrap(const HqChain& ch, double* Gc, double* const* Gr, int c0, const int8_t* s,
                                        int dir, cg::cluster_group& cluster) {
  if (dir == HQ_UP) {
    // G <- e^V E G E^-1 e^-V: E on the rows, E^-1 on the columns with e^V / e^-V on the last pass's stores
    cl_local_pass<0, 0, 0>(Gc, c0, ch.sep_a, ch.sep_c, s, 1.0, 1.0, 1.0, 1.0);
    __syncthreads();
    cl_local_pass<0, 1, 0>(Gc, c0, ch.sep_a, ch.sep_c, s, 1.0, 1.0, 1.0, 1.0);
    __syncthreads();
    cl_local_pass<1, 0, 0>(Gc, c0, ch.sep_ai, ch.sep_ci, s, 1.0, 1.0, 1.0, 1.0);
    cluster.sync();  // the other CTAs' x-pass results are read next
    cl_exchange_pass<2>(Gc, Gr, c0, ch.sep_ai, ch.sep_ci, s, ch.ev_p, ch.ev_m, ch.ev_m, ch.ev_p, cluster);
  } else {
    // G <- E^-1 e^-V G e^V E: the scalings on the first pass's loads
    cl_local_pass<0, 0, 1>(Gc, c0, ch.sep_ai, ch.sep_ci, s, ch.ev_m, ch.ev_p, ch.ev_p, ch.ev_m);
    __syncthreads();
    cl_local_pass<0, 1, 0>(Gc, c0, ch.sep_ai, ch.sep_ci, s, 1.0, 1.0, 1.0, 1.0);
    __syncthreads();
    cl_local_pass<1, 0, 0>(Gc, c0, ch.sep_a, ch.sep_c, s, 1.0, 1.0, 1.0, 1.0);
    cluster.sync();
    cl_exchange_pass<0>(Gc, Gr, c0, ch.sep_a, ch.sep_c, s, 1.0, 1.0, 1.0, 1.0, cluster);
  }
}

// Metropolis over the N sites of the slice (see the one-CTA metropolis_slice_blk): the owner
// of each 16-site block walks it; X by the owner, Y and the flush by every CTA.
__device__ __forceinline__ void cl_metropolis(const HqChain& ch, double* Gc, int rank, int c0, MetroShared& sh,
                                              double* u_l, double* dl_l, int8_t* flip_l, const uint32_t* pw,
                                              double* Xl, double* Yl, uint32_t& rng, double& n_acc, bool log,
                                              cg::cluster_group& cluster) {
  const int tid = threadIdx.x, warp = tid >> 5;
  double* Gs = Gc - (size_t)c0 * kLd;  // absolute column index -> local storage
  for (int q = tid; q < kNC; q += blockDim.x) {
    const uint32_t x1 = minstd_mulmod(pw[q], rng);
    const uint32_t x2 = minstd_mulmod(kMinstdA, x1);
    u_l[q] = canonical_from_pair(x1, x2);
    dl_l[q] = sh.s[c0 + q] > 0 ? ch.delta_p : ch.delta_m;
    flip_l[q] = 0;
  }
  rng = minstd_mulmod(minstd_pow(2ull * kN), rng);
  __syncthreads();
  double acc_count = 0.0;
  for (int b0 = 0, bi = 0; b0 < kN; b0 += 16, ++bi) {
    const int owner = b0 / kNC;
    const int slot = bi & 1;
    if (rank == owner && warp == 0) {
      const bool near = log ? walk_block16<false, true>(ch, Gs, kLd, sh, b0, 16, true, slot)
                            : walk_block16<false, false>(ch, Gs, kLd, sh, b0, 16, false, slot);
      if (near) walk_block16<true>(ch, Gs, kLd, sh, b0, 16, log, slot);
    }
    cluster.sync();  // the walk's records are visible to the cluster
    const int* o_ired = cluster.map_shared_rank(sh.ired, owner);
    const int a = o_ired[slot];
    if (rank == owner && tid == 0) acc_count += a;
    if (a == 0) continue;
    if (rank != owner) {
      const double* oxt = cluster.map_shared_rank(sh.xt, owner);
      const double* oyt = cluster.map_shared_rank(sh.yt, owner);
      const int* oqj = cluster.map_shared_rank(sh.qj, owner);
      const double* oqg = cluster.map_shared_rank(sh.qg, owner);
      for (int k = tid; k < 256; k += blockDim.x) { sh.xt[k] = oxt[k]; sh.yt[k] = oyt[k]; }
      if (tid < 16) { sh.qj[tid] = oqj[tid]; sh.qg[tid] = oqg[tid]; }
      __syncthreads();
    }
    // the owner: X[p, m] = gamma_m (G[p, j_m] + sum_{m'<m} X[p, m'] Y[m', j_m]) for every row p
    if (rank == owner) {
      for (int p = tid; p < kN; p += blockDim.x) {
        double x[16];
#pragma unroll
        for (int m = 0; m < 16; ++m) {
          x[m] = 0.0;
          if (m < a) {
            const int jm = sh.qj[m], sj = jm - b0;
            const double* cy = sh.yt + sj * 16;
            double cx0 = Gs[p + (size_t)jm * kLd], cx1 = 0.0;
#pragma unroll
            for (int m2 = 0; m2 + 1 < m; m2 += 2) {
              const double2 vy = *reinterpret_cast<const double2*>(cy + m2);
              cx0 = fma(x[m2], vy.x, cx0);
              cx1 = fma(x[m2 + 1], vy.y, cx1);
            }
            if (m & 1) cx0 = fma(x[m - 1], cy[m - 1], cx0);
            x[m] = sh.qg[m] * (cx0 + cx1);
          }
        }
#pragma unroll
        for (int m = 0; m < 16; ++m)
          if (m < a) Xl[p + m * kLdx] = x[m];
      }
    }
    // every CTA: Y[m, q] = G[j_m, q] - e_{j_m}(q) + sum_{m'<m} X[j_m, m'] Y[m', q] for its columns
    for (int q = tid; q < kNC; q += blockDim.x) {
      const int pc = c0 + q;
      double y[16];
#pragma unroll
      for (int m = 0; m < 16; ++m) {
        y[m] = 0.0;
        if (m < a) {
          const int jm = sh.qj[m], sj = jm - b0;
          const double* cx = sh.xt + sj * 16;
          double cy0 = Gc[jm + (size_t)q * kLd] - (pc == jm ? 1.0 : 0.0), cy1 = 0.0;
#pragma unroll
          for (int m2 = 0; m2 + 1 < m; m2 += 2) {
            const double2 vx = *reinterpret_cast<const double2*>(cx + m2);
            cy0 = fma(vx.x, y[m2], cy0);
            cy1 = fma(vx.y, y[m2 + 1], cy1);
          }
          if (m & 1) cy0 = fma(cx[m - 1], y[m - 1], cy0);
          y[m] = cy0 + cy1;
        }
      }
#pragma unroll
      for (int m = 0; m < 16; ++m)
        if (m < a) Yl[m * kLdy + q] = y[m];
    }
    cluster.sync();  // X is complete in the owner's shared memory
    if (rank != owner) {
      const double* oX = cluster.map_shared_rank(Xl, owner);
      for (int k = tid; k < kN * a; k += blockDim.x) {
        const int m = k / kN, p = k % kN;
        Xl[p + m * kLdx] = oX[p + m * kLdx];
      }
    }
    __syncthreads();
    rank_update48(Gc, kLd, kN, kNC, Xl, kLdx, Yl, kLdy, a);
    __syncthreads();
  }
  n_acc += acc_count;
  cluster.sync();  // every walk of the slice is done: the flip flags are final
  for (int i = tid; i < kN; i += blockDim.x) {
    const int8_t* of = cluster.map_shared_rank(flip_l, i / kNC);
    if (of[i % kNC]) sh.s[i] = -sh.s[i];
  }
  cluster.sync();  // every CTA has read the flags (they are reset by the next slice)
}

__global__ void __cluster_dims__(kCl, 1, 1) __launch_bounds__(HQ_INT_THREADS, 1)
k_interval_cl(const HqChain* __restrict__ chains, int nchains, int dir, int b, int flags) {
  extern __shared__ __align__(16) double smem[];
  __shared__ HqChain ch;
  __shared__ double red[96];
  __shared__ double part[2][3];  // this CTA's estimator partial sums, double-buffered by step
  __shared__ double acc_part;    // this CTA's accepted flips
  __shared__ int ired[4];
  __shared__ int qj_s[16];
  __shared__ double qg_s[16];
  __shared__ __align__(16) double xt_s[16 * 16];
  __shared__ __align__(16) double yt_s[16 * 16];
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int c = blockIdx.x / kCl;  // every CTA of a cluster serves the same chain
  if (c >= nchains) return;
  if (threadIdx.x == 0) ch = chains[c];
  __syncthreads();
  if (!ch.active || b >= ch.n_stab) return;
  int t_lo, t_hi;
  interval_range(ch.nt, ch.pace, ch.n_stab, dir, b, t_lo, t_hi);
  const int c0 = rank * kNC;

  // shared-memory carve-up
  double* Gc = smem;
  double* p = Gc + (size_t)kNC * kLd;
  double* Xl = p; p += (size_t)kLdx * 16;
  double* Yl = p; p += (size_t)16 * kLdy;
  double* u_l = p; p += kNC;
  double* dl_l = p; p += kNC;
  double* rr_l = p; p += kNC;
  uint32_t* pw = reinterpret_cast<uint32_t*>(p); p += kNC / 2;
  int8_t* s = reinterpret_cast<int8_t*>(p);
  int8_t* flip_l = s + kN;
  // this CTA's columns of G, then the jump-ahead powers of its sites
  for (int q = threadIdx.x >> 5; q < kNC; q += blockDim.x >> 5)
    for (int i = threadIdx.x & 31; i < kN; i += 32) cp_async_8(Gc + i + (size_t)q * kLd, ch.G + i + (size_t)(c0 + q) * kN, true);
  cp_async_commit();
  for (int q = threadIdx.x; q < kNC; q += blockDim.x) pw[q] = minstd_pow(2ull * (c0 + q) + 1);
  double* Gr[kCl];
#pragma unroll
  for (int k = 0; k < kCl; ++k) Gr[k] = (k == rank) ? Gc : cluster.map_shared_rank(Gc, k);
  MetroShared sh;
  sh.dl = dl_l - c0;
  sh.u = u_l - c0;
  sh.rr = rr_l - c0;
  sh.s = s;
  sh.flip = flip_l - c0;
  sh.X = Xl;
  sh.Y = Yl;
  sh.xt = xt_s;
  sh.yt = yt_s;
  sh.ired = ired;
  sh.pw = pw;
  sh.qj = qj_s;
  sh.qg = qg_s;
  uint32_t rng = *ch.rng;
  const bool log = (flags & HQ_F_LOG_RATIOS) && ch.ratios;
  long long log_base = log && ch.ratio_count ? *ch.ratio_count : 0;
  double n_acc = 0.0, n_prop = 0.0;
  cp_async_wait<0>();
  __syncthreads();
  cluster.sync();  // every CTA's columns are in place before the first exchange

  const int nsl = t_hi - t_lo + 1;
  for (int step = 0; step < nsl; ++step) {
    const int t = (dir == HQ_DOWN) ? (t_hi - step) : (t_lo + step);
    const int l = t % ch.nt;
    for (int i = threadIdx.x; i < kN; i += blockDim.x) s[i] = ch.fields[(size_t)l * kN + i];
    __syncthreads();
    if (dir == HQ_UP) {
      cl_wrap(ch, Gc, Gr, c0, s, HQ_UP, cluster);
      cl_metropolis(ch, Gc, rank, c0, sh, u_l, dl_l, flip_l, pw, Xl, Yl, rng, n_acc, log, cluster);
    } else {
      cl_metropolis(ch, Gc, rank, c0, sh, u_l, dl_l, flip_l, pw, Xl, Yl, rng, n_acc, log, cluster);
      cl_wrap(ch, Gc, Gr, c0, s, HQ_DOWN, cluster);
    }
    n_prop += kN;
    for (int q = threadIdx.x; q < kNC; q += blockDim.x) {
      ch.fields[(size_t)l * kN + c0 + q] = s[c0 + q];
      if (log && log_base + c0 + q < ch.ratio_cap) ch.ratios[log_base + c0 + q] = rr_l[q];
    }
    log_base += kN;
    if (step < nsl - 1) {
      const int lm = (dir == HQ_DOWN) ? ((t - 1) % ch.nt) : l;
      if (flags & HQ_F_MEASURE) {
        // estimators of the slice (include/observable_methods.hpp:39-151): partial sums of the
        // local columns, combined in rank order by CTA 0
        double tr = 0.0, dd = 0.0, sq = 0.0;
        for (int q = threadIdx.x >> 5; q < kNC; q += blockDim.x >> 5)
          for (int i = threadIdx.x & 31; i < kN; i += 32) {
            const double v = Gc[i + (size_t)q * kLd];
            sq = fma(v, v, sq);
            if (i == c0 + q) { tr += v; dd += (1.0 - v) * (1.0 - v); }
          }
        block_sum3(tr, dd, sq, red);
        const int pb = step & 1;
        if (threadIdx.x == 0) { part[pb][0] = tr; part[pb][1] = dd; part[pb][2] = sq; }
        cluster.sync();
        if (rank == 0 && threadIdx.x == 0) {
          double T = 0.0, D = 0.0, S = 0.0;
          for (int k = 0; k < kCl; ++k) {
            const double* pk = cluster.map_shared_rank(&part[pb][0], k);
            T += pk[0];
            D += pk[1];
            S += pk[2];
          }
          ch.acc[HQ_ACC_FILLING] += 2.0 - 2.0 * T / kN;
          ch.acc[HQ_ACC_DOCC] += D / kN;
          ch.acc[HQ_ACC_SWAVE] += (2.0 * S - 2.0 * T + kN) / kN;
          ch.acc[HQ_ACC_NSLICE] += 1.0;
        }
      }
      if ((flags & HQ_F_SNAPSHOT) && ch.snap_tt) {
        double* dst = ch.snap_tt + (size_t)lm * kN * kN;
        for (int q = threadIdx.x >> 5; q < kNC; q += blockDim.x >> 5)
          for (int i = threadIdx.x & 31; i < kN; i += 32) dst[i + (size_t)(c0 + q) * kN] = Gc[i + (size_t)q * kLd];
      }
    }
    __syncthreads();
  }
  // write back this CTA's columns; CTA 0 records the chain's counters
  for (int q = threadIdx.x >> 5; q < kNC; q += blockDim.x >> 5)
    for (int i = threadIdx.x & 31; i < kN; i += 32) ch.G[i + (size_t)(c0 + q) * kN] = Gc[i + (size_t)q * kLd];
  if (threadIdx.x == 0) acc_part = n_acc;
  cluster.sync();
  if (rank == 0 && threadIdx.x == 0) {
    double a = 0.0;
    for (int k = 0; k < kCl; ++k) a += *cluster.map_shared_rank(&acc_part, k);
    *ch.rng = rng;
    ch.acc[HQ_ACC_PROPOSED] += n_prop;
    ch.acc[HQ_ACC_ACCEPTED] += a;
    if (log && ch.ratio_count) *ch.ratio_count = log_base;
  }
  cluster.sync();  // no CTA leaves while another may still read its shared memory
}

// ---------------------------------------------------------------------------------
//  k_bchain_cols: the B-matrix chain of one interval for the 16 x 16 lattice (the role of
//  k_bchain, src/dqmc_core.cpp:190, :251 with the (M U) S product of svd_stack.hpp:144).
//  X <- B(t)...(U_top D_top) acts on every column of X on its own, so four CTAs per chain each
//  take 64 columns into shared memory; the one-CTA kernel would keep the 512 KB X in global
//  memory at this size. Same separable passes and arithmetic as k_bchain.
// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(HQ_INT_THREADS, 1)
k_bchain_cols(const HqChain* __restrict__ chains, int nchains, int dir, int b) {
  extern __shared__ __align__(16) double smem[];
  __shared__ HqChain ch;
  __shared__ int8_t s[kN];
  const int c = blockIdx.x / kCl, q = blockIdx.x % kCl;  // chain, column block
  if (c >= nchains) return;
  if (threadIdx.x == 0) ch = chains[c];
  __syncthreads();
  if (!ch.active || b >= ch.n_stab) return;
  int t_lo, t_hi;
  interval_range(ch.nt, ch.pace, ch.n_stab, dir, b, t_lo, t_hi);
  const int side = (dir == HQ_DOWN) ? 1 : 0;
  const int top = b - 1;  // the pushing stack holds b entries before this push
  const int c0 = q * kNC;
  const size_t NN = (size_t)kN * kN;
  double* Xc = smem;                      // kN x kNC, leading dimension kLd
  double* Dc = smem + (size_t)kNC * kLd;  // D of the stack top at the block's columns
  if (top >= 0) {
    const double* U = ch.stackU + ((size_t)side * ch.n_stab + top) * NN;
    const double* D = ch.stackD + ((size_t)side * ch.n_stab + top) * kN;
    for (int k = threadIdx.x; k < kNC; k += blockDim.x) cp_async_8(Dc + k, D + c0 + k, true);
    for (int j = threadIdx.x >> 5; j < kNC; j += blockDim.x >> 5)
      for (int i = threadIdx.x & 31; i < kN; i += 32) cp_async_8(Xc + i + (size_t)j * kLd, U + i + (size_t)(c0 + j) * kN, true);
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    for (int j = threadIdx.x >> 5; j < kNC; j += blockDim.x >> 5)
      for (int i = threadIdx.x & 31; i < kN; i += 32) Xc[i + (size_t)j * kLd] *= Dc[j];
  } else {
    for (int j = threadIdx.x >> 5; j < kNC; j += blockDim.x >> 5)
      for (int i = threadIdx.x & 31; i < kN; i += 32) Xc[i + (size_t)j * kLd] = (i == c0 + j ? 1.0 : 0.0);
  }
  __syncthreads();
  const int nsl = t_hi - t_lo + 1;
  for (int step = 0; step < nsl; ++step) {
    const int t = (dir == HQ_DOWN) ? (t_hi - step) : (t_lo + step);
    const int l = t % ch.nt;
    for (int i = threadIdx.x; i < kN; i += blockDim.x) s[i] = ch.fields[(size_t)l * kN + i];
    __syncthreads();
    // e^{V} rides on the first pass (down: B^T = E e^V) or the last pass (up: B = e^V E)
    if (dir == HQ_DOWN) {
      cl_local_pass<0, 0, 1>(Xc, c0, ch.sep_a, ch.sep_c, s, ch.ev_p, ch.ev_m, 1.0, 1.0);
      __syncthreads();
      cl_local_pass<0, 1, 0>(Xc, c0, ch.sep_a, ch.sep_c, s, 1.0, 1.0, 1.0, 1.0);
    } else {
      cl_local_pass<0, 0, 0>(Xc, c0, ch.sep_a, ch.sep_c, s, 1.0, 1.0, 1.0, 1.0);
      __syncthreads();
      cl_local_pass<0, 1, 2>(Xc, c0, ch.sep_a, ch.sep_c, s, ch.ev_p, ch.ev_m, 1.0, 1.0);
    }
    __syncthreads();
  }
  for (int j = threadIdx.x >> 5; j < kNC; j += blockDim.x >> 5)
    for (int i = threadIdx.x & 31; i < kN; i += 32) ch.X[i + (size_t)(c0 + j) * kN] = Xc[i + (size_t)j * kLd];
}

size_t smem_bchain_cols_bytes() { return ((size_t)kNC * kLd + kNC) * sizeof(double); }
cudaError_t launch_bchain_cols(const HqChain* chains, int n, int dir, int b, cudaStream_t st) {
  k_bchain_cols<<<n * kCl, HQ_INT_THREADS, smem_bchain_cols_bytes(), st>>>(chains, n, dir, b);
  return cudaGetLastError();
}
const void* fn_bchain_cols() { return (const void*)k_bchain_cols; }

cudaError_t launch_interval_cl(const HqChain* chains, int n, int dir, int b, int flags, cudaStream_t st) {
  k_interval_cl<<<n * kCl, HQ_INT_THREADS, smem_interval_cl_bytes(), st>>>(chains, n, dir, b, flags);
  return cudaGetLastError();
}
const void* fn_interval_cl() { return (const void*)k_interval_cl; }

// clusters of the interval kernel that the device can hold at once (0: the cluster path is unusable)
int interval_cl_max_clusters() {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(kCl * 64, 1, 1);
  cfg.blockDim = dim3(HQ_INT_THREADS, 1, 1);
  cfg.dynamicSmemBytes = smem_interval_cl_bytes();
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeClusterDimension;
  attr.val.clusterDim.x = kCl;
  attr.val.clusterDim.y = 1;
  attr.val.clusterDim.z = 1;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, (const void*)k_interval_cl, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

}  // namespace hq
