// Smoothed-aggregation AMG setup on the host (FP64, multithreaded, deterministic).
//
// The reference has no AMG for C3D10 solids; its beam AMG (wnfea/solver/amg_preconditioner.py)
// is the template for the steps: aggregation of nodes (:207-239), tentative prolongator from
// a per-aggregate QR of the rigid-body modes (:30-69, :247-281), Galerkin coarse operator
// R A P with R = P^T, symmetrised (:283-293), dense Cholesky at the coarsest level
// (:309-325).  Differences, all for 3-DOF solid nodes:
//   * strength of connection on 3x3 / 6x6 block Frobenius norms and the three-pass greedy
//     aggregation of Vanek, Mandel & Brezina (1996) instead of beam-edge pairing; nodes with
//     no strong neighbour (fully clamped nodes, identity rows) stay unaggregated;
//   * the near-null space on coarse levels is the R factor of the QR (exact coarse
//     representation of the rigid modes) instead of modes rebuilt from averaged coordinates;
//   * the tentative prolongator is smoothed, P = (I - w/rho D^-1 A) P_tent, w = 4/3;
//   * no diagonal equilibration: D^-1 A, the strength measure and the Galerkin product are
//     invariant to it, and Dirichlet rows (diagonal 1) need no rescaling.
// Every loop that writes shared output is split by rows and sums in a fixed order, so the
// hierarchy is bit-identical for any thread count.
#include "amg_setup.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <functional>
#include <thread>

#include "common.cuh"
#include "pattern.h"

namespace wn {

wn_amg_params amg_default_params() {
  wn_amg_params p;
  p.strength_theta = 0.08;
  p.max_levels = 10;
  p.coarse_size = 1500;
  p.smoother_degree = 1;
  p.cheb_lower = 1.0 / 16.0;
  p.cheb_safety = 1.1;
  p.prolong_omega = 4.0 / 3.0;
  p.smooth_prolongator = 1;
  p.power_iters = 15;
  p.stream_min_mb = 4.0;
  p.setup_on_device = 1;
  p.coarse_block_smoother = 1;
  return p;
}

namespace {

struct View {
  int br, bc;
  int64_t n_rows, n_cols;
  const int32_t* rp;
  const int32_t* ci;
  const double* v;
};

View view(const HostBsr& m) { return View{m.br, m.bc, m.n_rows, m.n_cols, m.rp.data(), m.ci.data(), m.v.data()}; }

void par_rows(int64_t n, const std::function<void(int64_t, int64_t, int)>& fn) {
  const int nth = host_threads();
  if (nth <= 1 || n < 2048) {
    fn(0, n, 0);
    return;
  }
  std::vector<std::thread> th;
  const int64_t chunk = (n + nth - 1) / nth;
  for (int t = 0; t < nth; ++t) {
    const int64_t a = t * chunk, b = std::min(n, a + chunk);
    if (a >= b) break;
    th.emplace_back(fn, a, b, t);
  }
  for (auto& x : th) x.join();
}

// sum_k a[k] b[k] over n terms in a fixed order (four interleaved partial sums, then
// ((s0 + s1) + (s2 + s3)) + tail): vectorisable, and the same result for any thread count
inline double dot_fixed(const double* a, const double* b, int64_t n) {
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  int64_t k = 0;
  for (; k + 4 <= n; k += 4) {
    s0 += a[k] * b[k];
    s1 += a[k + 1] * b[k + 1];
    s2 += a[k + 2] * b[k + 2];
    s3 += a[k + 3] * b[k + 3];
  }
  double s = (s0 + s1) + (s2 + s3);
  for (; k < n; ++k) s += a[k] * b[k];
  return s;
}

// fn(i) for i < n on the host threads, thread t taking i = t, t + nth, ... (for work that
// shrinks or grows with i)
void par_interleaved(int64_t n, const std::function<void(int64_t)>& fn) {
  const int nth = host_threads();
  if (nth <= 1 || n < 64) {
    for (int64_t i = 0; i < n; ++i) fn(i);
    return;
  }
  std::vector<std::thread> th;
  for (int t = 0; t < nth && t < n; ++t)
    th.emplace_back([&, t]() {
      for (int64_t i = t; i < n; i += nth) fn(i);
    });
  for (auto& x : th) x.join();
}

// y = A x (scalar layout), FP64
void spmv(const View& A, const double* x, double* y) {
  par_rows(A.n_rows, [&](int64_t a, int64_t b, int) {
    for (int64_t i = a; i < b; ++i) {
      for (int r = 0; r < A.br; ++r) y[i * A.br + r] = 0.0;
      for (int32_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
        const double* blk = A.v + (int64_t)k * A.br * A.bc;
        const double* xx = x + (int64_t)A.ci[k] * A.bc;
        for (int r = 0; r < A.br; ++r) {
          double s = 0.0;
          for (int c = 0; c < A.bc; ++c) s += blk[r * A.bc + c] * xx[c];
          y[i * A.br + r] += s;
        }
      }
    }
  });
}

std::vector<double> inv_diag(const View& A) {
  std::vector<double> d(A.n_rows * A.br, 1.0);
  par_rows(A.n_rows, [&](int64_t a, int64_t b, int) {
    for (int64_t i = a; i < b; ++i)
      for (int32_t k = A.rp[i]; k < A.rp[i + 1]; ++k)
        if (A.ci[k] == i) {
          const double* blk = A.v + (int64_t)k * A.br * A.bc;
          for (int r = 0; r < A.br; ++r) {
            const double dv = blk[r * A.bc + r];
            d[i * A.br + r] = (dv != 0.0) ? 1.0 / dv : 1.0;
          }
        }
  });
  return d;
}

// largest eigenvalue of D^-1 A by power iteration from a fixed pseudo-random start
double power_rho(const View& A, const std::vector<double>& dinv, int iters) {
  const int64_t n = A.n_rows * A.br;
  std::vector<double> x(n), y(n);
  uint64_t s = 0x9E3779B97F4A7C15ull;
  for (int64_t i = 0; i < n; ++i) {
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    x[i] = 0.5 + (double)(s % 1000003) / 1000003.0;
  }
  double lam = 0.0;
  for (int it = 0; it < std::max(iters, 1); ++it) {
    double nx = 0.0;
    for (int64_t i = 0; i < n; ++i) nx += x[i] * x[i];
    nx = std::sqrt(nx);
    if (nx == 0.0) return 1.0;
    for (int64_t i = 0; i < n; ++i) x[i] /= nx;
    spmv(A, x.data(), y.data());
    double ny = 0.0;
    for (int64_t i = 0; i < n; ++i) {
      y[i] *= dinv[i];
      ny += y[i] * y[i];
    }
    lam = std::sqrt(ny);
    std::swap(x, y);
  }
  return lam;
}

// explicit fused multiply-adds (whatever the compiler's contraction setting), bitwise the device
// builder's ks_block_norms: the aggregation breaks ties between equal norms by order
double block_fro(const double* b, int n) {
  double s = 0.0;
  for (int k = 0; k < n; ++k) s = std::fma(b[k], b[k], s);
  return std::sqrt(s);
}

// three-pass greedy aggregation on the strong block graph
int64_t aggregate(const View& A, double theta, std::vector<int32_t>& agg) {
  const int64_t n = A.n_rows;
  const int bsz = A.br * A.bc;
  std::vector<double> nrm(A.rp[n]);
  par_rows(n, [&](int64_t a, int64_t b, int) {
    for (int64_t i = a; i < b; ++i)
      for (int32_t k = A.rp[i]; k < A.rp[i + 1]; ++k) nrm[k] = block_fro(A.v + (int64_t)k * bsz, bsz);
  });
  return aggregate_norms(n, A.rp, A.ci, nrm.data(), theta, agg);
}

// thin Householder QR of the m x 6 column-major matrix a: Q (m x 6, column-major), R (6x6)
void qr6(int m, std::vector<double>& a, std::vector<double>& q, double r[36]) {
  const int nc = 6;
  std::vector<double> vs((size_t)m * nc, 0.0);
  std::vector<uint8_t> used(nc, 0);
  for (int k = 0; k < nc && k < m; ++k) {
    double nx = 0.0;
    for (int i = k; i < m; ++i) nx += a[(size_t)k * m + i] * a[(size_t)k * m + i];
    nx = std::sqrt(nx);
    if (nx == 0.0) continue;
    const double x0 = a[(size_t)k * m + k];
    const double alpha = x0 >= 0 ? -nx : nx;
    double* v = &vs[(size_t)k * m];
    for (int i = k; i < m; ++i) v[i] = a[(size_t)k * m + i];
    v[k] -= alpha;
    double nv = 0.0;
    for (int i = k; i < m; ++i) nv += v[i] * v[i];
    nv = std::sqrt(nv);
    if (nv == 0.0) continue;
    for (int i = k; i < m; ++i) v[i] /= nv;
    used[k] = 1;
    for (int c = k; c < nc; ++c) {
      double d = 0.0;
      for (int i = k; i < m; ++i) d += v[i] * a[(size_t)c * m + i];
      for (int i = k; i < m; ++i) a[(size_t)c * m + i] -= 2.0 * d * v[i];
    }
  }
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) r[i * 6 + j] = (i <= j && i < m) ? a[(size_t)j * m + i] : 0.0;
  // Q = H_0 ... H_5 applied to the first 6 columns of I (zero columns beyond m)
  q.assign((size_t)m * nc, 0.0);
  for (int c = 0; c < nc && c < m; ++c) q[(size_t)c * m + c] = 1.0;
  for (int k = std::min(nc, m) - 1; k >= 0; --k) {
    if (!used[k]) continue;
    const double* v = &vs[(size_t)k * m];
    for (int c = 0; c < nc; ++c) {
      double d = 0.0;
      for (int i = k; i < m; ++i) d += v[i] * q[(size_t)c * m + i];
      for (int i = k; i < m; ++i) q[(size_t)c * m + i] -= 2.0 * d * v[i];
    }
  }
}

// sparse row accumulator keyed by block column
struct RowAcc {
  std::vector<int32_t> mark;  // column -> slot, -1 if absent
  std::vector<int32_t> cols;
  std::vector<double> vals;
  int bsz = 0;
  void init(int64_t ncols, int block_size) {
    mark.assign(ncols, -1);
    bsz = block_size;
  }
  double* slot(int32_t c) {
    int32_t s = mark[c];
    if (s < 0) {
      s = (int32_t)cols.size();
      mark[c] = s;
      cols.push_back(c);
      vals.resize(vals.size() + bsz, 0.0);
    }
    return &vals[(size_t)s * bsz];
  }
  // emit sorted by column, dropping all-zero blocks; resets the accumulator
  void flush(std::vector<int32_t>& oc, std::vector<double>& ov) {
    std::vector<int32_t> order(cols.size());
    for (size_t k = 0; k < order.size(); ++k) order[k] = (int32_t)k;
    std::sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return cols[x] < cols[y]; });
    for (int32_t s : order) {
      const double* b = &vals[(size_t)s * bsz];
      bool nz = false;
      for (int k = 0; k < bsz && !nz; ++k) nz = b[k] != 0.0;
      if (nz) {
        oc.push_back(cols[s]);
        ov.insert(ov.end(), b, b + bsz);
      }
      mark[cols[s]] = -1;
    }
    cols.clear();
    vals.clear();
  }
};

// out(i, :) rows produced per row in parallel, then concatenated in row order
void rows_to_bsr(int br, int bc, int64_t n_rows, int64_t n_cols, std::vector<std::vector<int32_t>>& rc,
                 std::vector<std::vector<double>>& rv, HostBsr& out) {
  out.br = br;
  out.bc = bc;
  out.n_rows = n_rows;
  out.n_cols = n_cols;
  out.rp.assign(n_rows + 1, 0);
  for (int64_t i = 0; i < n_rows; ++i) out.rp[i + 1] = out.rp[i] + (int32_t)rc[i].size();
  out.ci.resize(out.rp[n_rows]);
  out.v.resize((size_t)out.rp[n_rows] * br * bc);
  par_rows(n_rows, [&](int64_t a, int64_t b, int) {
    for (int64_t i = a; i < b; ++i) {
      std::copy(rc[i].begin(), rc[i].end(), out.ci.begin() + out.rp[i]);
      std::copy(rv[i].begin(), rv[i].end(), out.v.begin() + (size_t)out.rp[i] * br * bc);
      std::vector<int32_t>().swap(rc[i]);
      std::vector<double>().swap(rv[i]);
    }
  });
}

// C = A * B for block-sparse A (AR x AK blocks) and B (AK x BC blocks).  The block shapes
// are compile-time so that the block products unroll and vectorise: the coarse operators of
// 3D meshes reach hundreds of 6x6 blocks per row, and these products are most of the setup.
template <int AR, int AK, int BC>
void spgemm_blocks(const View& A, const View& B, HostBsr& C) {
  std::vector<std::vector<int32_t>> rc(A.n_rows);
  std::vector<std::vector<double>> rv(A.n_rows);
  par_rows(A.n_rows, [&](int64_t a, int64_t b, int) {
    RowAcc acc;
    acc.init(B.n_cols, AR * BC);
    for (int64_t i = a; i < b; ++i) {
      for (int32_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
        const int32_t j = A.ci[k];
        const double* ab = A.v + (size_t)k * AR * AK;
        for (int32_t q = B.rp[j]; q < B.rp[j + 1]; ++q) {
          const double* bb = B.v + (size_t)q * AK * BC;
          double* c = acc.slot(B.ci[q]);
          for (int r = 0; r < AR; ++r)
            for (int s = 0; s < AK; ++s) {
              const double av = ab[r * AK + s];
              for (int t = 0; t < BC; ++t) c[r * BC + t] += av * bb[s * BC + t];
            }
        }
      }
      acc.flush(rc[i], rv[i]);
    }
  });
  rows_to_bsr(AR, BC, A.n_rows, B.n_cols, rc, rv, C);
}

// the shapes of the Galerkin products: A0 P0 (3x3 . 3x6), R0 (A0 P0) (6x3 . 3x6), coarse (6x6)
void spgemm(const View& A, const View& B, HostBsr& C) {
  if (A.br == 3 && A.bc == 3 && B.bc == 6) return spgemm_blocks<3, 3, 6>(A, B, C);
  if (A.br == 6 && A.bc == 3 && B.bc == 6) return spgemm_blocks<6, 3, 6>(A, B, C);
  if (A.br == 6 && A.bc == 6 && B.bc == 6) return spgemm_blocks<6, 6, 6>(A, B, C);
  if (A.br == 3 && A.bc == 3 && B.bc == 3) return spgemm_blocks<3, 3, 3>(A, B, C);
  if (A.br == 6 && A.bc == 6 && B.bc == 3) return spgemm_blocks<6, 6, 3>(A, B, C);
  if (A.br == 3 && A.bc == 6 && B.bc == 6) return spgemm_blocks<3, 6, 6>(A, B, C);
  // no other shape occurs in the hierarchy
  std::fprintf(stderr, "amg_build: unexpected block product %dx%d . %dx%d\n", A.br, A.bc, B.br, B.bc);
  std::abort();
}

// transpose of a block-sparse matrix (blocks transposed too); rows of T in source-row order
void transpose(const View& A, HostBsr& T) {
  T.br = A.bc;
  T.bc = A.br;
  T.n_rows = A.n_cols;
  T.n_cols = A.n_rows;
  T.rp.assign(T.n_rows + 1, 0);
  const int64_t nnz = A.rp[A.n_rows];
  for (int64_t k = 0; k < nnz; ++k) T.rp[A.ci[k] + 1]++;
  for (int64_t i = 0; i < T.n_rows; ++i) T.rp[i + 1] += T.rp[i];
  T.ci.resize(nnz);
  T.v.resize((size_t)nnz * A.br * A.bc);
  std::vector<int32_t> pos(T.rp.begin(), T.rp.end() - 1);
  for (int64_t i = 0; i < A.n_rows; ++i)
    for (int32_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      const int32_t p = pos[A.ci[k]]++;
      T.ci[p] = (int32_t)i;
      const double* s = A.v + (size_t)k * A.br * A.bc;
      double* d = &T.v[(size_t)p * A.br * A.bc];
      for (int r = 0; r < A.br; ++r)
        for (int c = 0; c < A.bc; ++c) d[c * A.br + r] = s[r * A.bc + c];
    }
}

void symmetrize(HostBsr& A) {
  const int b = A.br;
  std::vector<double> out(A.v.size());
  par_rows(A.n_rows, [&](int64_t a, int64_t e, int) {
    for (int64_t i = a; i < e; ++i)
      for (int32_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
        const int32_t j = A.ci[k];
        const int32_t* beg = A.ci.data() + A.rp[j];
        const int32_t* end = A.ci.data() + A.rp[j + 1];
        const int32_t* f = std::lower_bound(beg, end, (int32_t)i);
        const double* x = &A.v[(size_t)k * b * b];
        double* o = &out[(size_t)k * b * b];
        if (f == end || *f != i) {  // structurally unsymmetric entry (not expected): keep
          std::copy(x, x + b * b, o);
          continue;
        }
        const double* y = &A.v[(size_t)(f - A.ci.data()) * b * b];
        for (int r = 0; r < b; ++r)
          for (int c = 0; c < b; ++c) o[r * b + c] = 0.5 * (x[r * b + c] + y[c * b + r]);
      }
  });
  A.v.swap(out);
}

}  // namespace

// Three-pass greedy aggregation (Vanek-Mandel-Brezina) on the strong block graph, given the
// Frobenius norm of every block: (i, j) is strong if |A_ij| >= theta sqrt(|A_ii| |A_jj|).
// Pass 1 makes roots of nodes whose strong neighbourhood is still free; pass 2 joins each left
// node to its strongest aggregated neighbour; pass 3 turns the leftovers with strong links into
// new aggregates.  Nodes without strong links (fully fixed nodes) stay unaggregated (-1).
int64_t aggregate_norms(int64_t n, const int32_t* rp, const int32_t* ci, const double* nrm, double theta,
                        std::vector<int32_t>& agg) {
  std::vector<double> dn(n, 0.0);
  for (int64_t i = 0; i < n; ++i)
    for (int32_t k = rp[i]; k < rp[i + 1]; ++k)
      if (ci[k] == i) dn[i] = nrm[k];
  std::vector<uint8_t> strong(rp[n], 0);
  std::vector<uint8_t> has_strong(n, 0);
  par_rows(n, [&](int64_t a, int64_t b, int) {
    for (int64_t i = a; i < b; ++i)
      for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
        const int32_t j = ci[k];
        if (j != i && nrm[k] > 0.0 && nrm[k] >= theta * std::sqrt(dn[i] * dn[j])) {
          strong[k] = 1;
          has_strong[i] = 1;
        }
      }
  });
  agg.assign(n, -1);
  int64_t na = 0;
  for (int64_t i = 0; i < n; ++i) {  // pass 1: roots whose strong neighbourhood is free
    if (agg[i] >= 0 || !has_strong[i]) continue;
    bool free_all = true;
    for (int32_t k = rp[i]; k < rp[i + 1] && free_all; ++k)
      if (strong[k] && agg[ci[k]] >= 0) free_all = false;
    if (!free_all) continue;
    agg[i] = (int32_t)na;
    for (int32_t k = rp[i]; k < rp[i + 1]; ++k)
      if (strong[k]) agg[ci[k]] = (int32_t)na;
    ++na;
  }
  std::vector<int32_t> pass2(agg);
  for (int64_t i = 0; i < n; ++i) {  // pass 2: join the strongest aggregated neighbour
    if (agg[i] >= 0 || !has_strong[i]) continue;
    double best = -1.0;
    int32_t ba = -1;
    for (int32_t k = rp[i]; k < rp[i + 1]; ++k)
      if (strong[k] && agg[ci[k]] >= 0 && nrm[k] > best) {
        best = nrm[k];
        ba = agg[ci[k]];
      }
    pass2[i] = ba;
  }
  agg.swap(pass2);
  for (int64_t i = 0; i < n; ++i) {  // pass 3: leftovers with strong links form new aggregates
    if (agg[i] >= 0 || !has_strong[i]) continue;
    agg[i] = (int32_t)na;
    for (int32_t k = rp[i]; k < rp[i + 1]; ++k)
      if (strong[k] && agg[ci[k]] < 0) agg[ci[k]] = (int32_t)na;
    ++na;
  }
  return na;
}

// Near-null space of level 0: the 6 rigid-body modes, zero on fixed DOFs.  Rows ux, uy, uz (and
// for 6-DOF nodes rx, ry, rz); columns tx, ty, tz, rx, ry, rz (the layout of
// amg_preconditioner.py:30-69): a rotation w moves a node by w x X and turns it by w.
void near_null_space(int64_t n0, int bs0, const double* coords, const uint8_t* fixed, std::vector<double>& B) {
  B.assign((size_t)n0 * bs0 * 6, 0.0);
  for (int64_t i = 0; i < n0; ++i) {
    const double X = coords[i * 3], Y = coords[i * 3 + 1], Z = coords[i * 3 + 2];
    double* b = &B[(size_t)i * bs0 * 6];
    const double m[6][6] = {{1, 0, 0, 0, Z, -Y}, {0, 1, 0, -Z, 0, X}, {0, 0, 1, Y, -X, 0},
                            {0, 0, 0, 1, 0, 0},  {0, 0, 0, 0, 1, 0},  {0, 0, 0, 0, 0, 1}};
    for (int r = 0; r < bs0; ++r) {
      const bool fx = fixed && fixed[i * bs0 + r];
      for (int c = 0; c < 6; ++c) b[r * 6 + c] = fx ? 0.0 : m[r][c];
    }
  }
}

// Tentative prolongator: per aggregate, a thin QR of its members' near-null-space rows;
// Qnode (n x bs x 6) = each node's block of Q, Bc (n_agg x 36) = the R factors (the coarse
// near-null space).
void tentative_prolongator(int64_t n, int bs, int64_t n_agg, const std::vector<int32_t>& agg,
                           const std::vector<double>& B, std::vector<double>& Qnode, std::vector<double>& Bc) {
  std::vector<int32_t> cnt(n_agg + 1, 0);
  for (int64_t i = 0; i < n; ++i)
    if (agg[i] >= 0) cnt[agg[i] + 1]++;
  for (int64_t a = 0; a < n_agg; ++a) cnt[a + 1] += cnt[a];
  std::vector<int32_t> members(cnt[n_agg]);
  {
    std::vector<int32_t> pos(cnt.begin(), cnt.end() - 1);
    for (int64_t i = 0; i < n; ++i)
      if (agg[i] >= 0) members[pos[agg[i]]++] = (int32_t)i;
  }
  Qnode.assign((size_t)n * bs * 6, 0.0);
  Bc.assign((size_t)n_agg * 36, 0.0);
  par_rows(n_agg, [&](int64_t a0, int64_t a1, int) {
    std::vector<double> mat, q;
    for (int64_t a = a0; a < a1; ++a) {
      const int cntn = cnt[a + 1] - cnt[a];
      const int m = cntn * bs;
      mat.assign((size_t)m * 6, 0.0);
      for (int t = 0; t < cntn; ++t) {
        const int32_t node = members[cnt[a] + t];
        for (int r = 0; r < bs; ++r)
          for (int c = 0; c < 6; ++c) mat[(size_t)c * m + t * bs + r] = B[((size_t)node * bs + r) * 6 + c];
      }
      double R[36];
      qr6(m, mat, q, R);
      for (int t = 0; t < cntn; ++t) {
        const int32_t node = members[cnt[a] + t];
        for (int r = 0; r < bs; ++r)
          for (int c = 0; c < 6; ++c) Qnode[((size_t)node * bs + r) * 6 + c] = q[(size_t)c * m + t * bs + r];
      }
      std::copy(R, R + 36, &Bc[(size_t)a * 36]);
    }
  });
}

// Coarsest level: the n x n block matrix (bs x bs row-major blocks) made dense in FP64, its
// Cholesky factor and the explicit inverse A^-1 = L^-T L^-1 (into out.coarse_A / coarse_inv).
int dense_coarse(int64_t n, int bs, const int32_t* rp, const int32_t* ci, const double* v, HostHierarchy& out) {
  const int64_t nc = n * bs;
  WN_REQUIRE(nc <= 20000, WN_ETOOBIG, "amg_build: coarsest level too large (%lld DOFs); raise max_levels",
             (long long)nc);
  out.n_coarse = nc;
  std::vector<double>& D = out.coarse_A;
  D.assign((size_t)nc * nc, 0.0);
  for (int64_t i = 0; i < n; ++i)
    for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
      const double* blk = v + (size_t)k * bs * bs;
      for (int r = 0; r < bs; ++r)
        for (int c = 0; c < bs; ++c) D[(size_t)(i * bs + r) * nc + ci[k] * bs + c] = blk[r * bs + c];
    }
  // unaggregated-only systems can leave zero rows: give them a unit diagonal
  for (int64_t i = 0; i < nc; ++i) {
    bool any = false;
    for (int64_t j = 0; j < nc && !any; ++j) any = D[(size_t)i * nc + j] != 0.0;
    if (!any) D[(size_t)i * nc + i] = 1.0;
  }
  // Cholesky A = L L^T (left-looking; row-major L, the dot products run over contiguous rows).
  // Column j: the pivot L_jj from row j, then L_ij for every i > j, each from rows i and j only.
  // A team of host threads owns the rows (row i on thread i mod T) and meets once per column;
  // the owner of row j + 1 forms the next pivot right after its L_{j+1,j}.  Every entry is the
  // same fixed-order dot product whatever T is, so L does not depend on the thread count.
  std::vector<double> Lf(D);
  const int nth = (int)std::min<int64_t>(host_threads(), std::max<int64_t>(1, nc / 64));
  std::atomic<int64_t> bad{-1};
  auto pivot = [&](int64_t j) {
    const double* lj = &Lf[(size_t)j * nc];
    const double s = Lf[(size_t)j * nc + j] - dot_fixed(lj, lj, j);
    if (!(s > 0.0 && std::isfinite(s))) {
      int64_t none = -1;
      bad.compare_exchange_strong(none, j);
      return;
    }
    Lf[(size_t)j * nc + j] = std::sqrt(s);
  };
  auto column = [&](int64_t j, int t, int T) {  // L_ij for the rows i > j of thread t
    const double* lj = &Lf[(size_t)j * nc];
    const double ljj = lj[j];
    int64_t i = j + 1 + ((t - (j + 1)) % T + T) % T;
    for (; i < nc; i += T) {
      double* li = &Lf[(size_t)i * nc];
      li[j] = (li[j] - dot_fixed(li, lj, j)) / ljj;
      if (i == j + 1) pivot(i);
    }
  };
  if (nc > 0) pivot(0);
  if (nth <= 1) {
    for (int64_t j = 0; j < nc && bad.load() < 0; ++j) column(j, 0, 1);
  } else if (bad.load() < 0) {
    // sense-counting barrier of the team: a generation counter bumped by the last arrival
    std::atomic<int> arrived{0}, generation{0};
    auto meet = [&]() {
      const int g = generation.load(std::memory_order_acquire);
      if (arrived.fetch_add(1, std::memory_order_acq_rel) + 1 == nth) {
        arrived.store(0, std::memory_order_relaxed);
        generation.fetch_add(1, std::memory_order_acq_rel);
      } else {
        while (generation.load(std::memory_order_acquire) == g) std::this_thread::yield();
      }
    };
    // a failed pivot p is recorded during column p - 1; after the meet that ends column j every
    // thread has seen each failure with p <= j + 1 and stops there, while a failure a faster
    // thread already met in column j + 1 (p = j + 2) is acted on one meet later by all alike
    std::vector<std::thread> team;
    for (int t = 0; t < nth; ++t)
      team.emplace_back([&, t]() {
        for (int64_t j = 0; j < nc; ++j) {
          column(j, t, nth);
          meet();
          const int64_t p = bad.load(std::memory_order_acquire);
          if (p >= 0 && p <= j + 1) break;
        }
      });
    for (auto& x : team) x.join();
  }
  WN_REQUIRE(bad.load() < 0, WN_ENOTSPD, "amg_build: coarsest matrix not SPD (pivot %lld)", (long long)bad.load());
  // Wt = (L^-1)^T, upper triangular, row c = column c of L^-1 (forward substitution on e_c);
  // rows are independent and split over the host threads (interleaved: the work per row falls
  // with c)
  std::vector<double> Wt((size_t)nc * nc, 0.0);
  par_interleaved(nc, [&](int64_t c) {
    double* wc = &Wt[(size_t)c * nc];
    wc[c] = 1.0 / Lf[(size_t)c * nc + c];
    for (int64_t i = c + 1; i < nc; ++i) {
      const double* li = &Lf[(size_t)i * nc];
      wc[i] = -dot_fixed(li + c, wc + c, i - c) / li[i];
    }
  });
  // A^-1 = L^-T L^-1: (A^-1)_ij = sum_{k >= max(i, j)} Wt_ik Wt_jk, the upper half computed and
  // mirrored
  out.coarse_inv.assign((size_t)nc * nc, 0.0);
  par_interleaved(nc, [&](int64_t i) {
    const double* wi = &Wt[(size_t)i * nc];
    for (int64_t j = i; j < nc; ++j) {
      const double* wj = &Wt[(size_t)j * nc];
      out.coarse_inv[(size_t)i * nc + j] = dot_fixed(wi + j, wj + j, nc - j);
    }
  });
  for (int64_t i = 0; i < nc; ++i)
    for (int64_t j = 0; j < i; ++j) out.coarse_inv[(size_t)i * nc + j] = out.coarse_inv[(size_t)j * nc + i];
  return WN_OK;
}

// WN_AMG_TRACE=1 in the environment: phase times of the setup on stderr
struct PhaseTrace {
  bool on;
  std::chrono::steady_clock::time_point t;
  PhaseTrace() : on(std::getenv("WN_AMG_TRACE") != nullptr), t(std::chrono::steady_clock::now()) {}
  void mark(const char* what, int lvl) {
    if (!on) return;
    const auto now = std::chrono::steady_clock::now();
    std::fprintf(stderr, "amg_build: level %d %-12s %8.3f s\n", lvl, what,
                 std::chrono::duration<double>(now - t).count());
    t = now;
  }
};

int amg_build(const wn_amg_params& prm, int64_t n0, int bs0, const int32_t* rp0, const int32_t* ci0,
              const double* v0, const double* coords, const uint8_t* fixed, HostHierarchy& out) {
  PhaseTrace tr;
  out = HostHierarchy();
  out.params = prm;
  WN_REQUIRE(n0 > 0 && rp0 && ci0 && v0 && coords && (bs0 == 3 || bs0 == 6), WN_EINVAL, "amg_build: bad argument");
  std::vector<double> B;
  near_null_space(n0, bs0, coords, fixed, B);
  View A{bs0, bs0, n0, n0, rp0, ci0, v0};
  HostBsr Aown;
  int bs = bs0;
  int64_t n = n0;
  for (int lvl = 0;; ++lvl) {
    const int64_t ndof = n * bs;
    if (ndof <= prm.coarse_size || lvl >= prm.max_levels - 1) break;
    HostLevel L;
    L.bs = bs;
    L.n_nodes = n;
    L.dinv = inv_diag(A);
    L.rho = power_rho(A, L.dinv, prm.power_iters);
    tr.mark("rho", lvl);
    L.n_agg = aggregate(A, prm.strength_theta, L.agg);
    tr.mark("aggregate", lvl);
    if (L.n_agg == 0 || L.n_agg * 6 >= (int64_t)(0.8 * ndof)) break;  // coarsening stalled
    // tentative prolongator: per aggregate QR of its near-null-space rows
    std::vector<double> Qnode, Bc;
    tentative_prolongator(n, bs, L.n_agg, L.agg, B, Qnode, Bc);
    tr.mark("tentative", lvl);
    // (smoothed) prolongator rows
    std::vector<std::vector<int32_t>> rc(n);
    std::vector<std::vector<double>> rv(n);
    const double w = prm.smooth_prolongator ? prm.prolong_omega / L.rho : 0.0;
    par_rows(n, [&](int64_t a0, int64_t a1, int) {
      RowAcc acc;
      acc.init(L.n_agg, bs * 6);
      for (int64_t i = a0; i < a1; ++i) {
        if (L.agg[i] >= 0) {
          double* s = acc.slot(L.agg[i]);
          for (int k = 0; k < bs * 6; ++k) s[k] += Qnode[(size_t)i * bs * 6 + k];
        }
        if (w != 0.0) {
          for (int32_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
            const int32_t j = A.ci[k];
            if (L.agg[j] < 0) continue;
            const double* ab = A.v + (size_t)k * bs * bs;
            const double* qj = &Qnode[(size_t)j * bs * 6];
            double* s = acc.slot(L.agg[j]);
            for (int r = 0; r < bs; ++r) {
              const double f = -w * L.dinv[i * bs + r];
              for (int c = 0; c < bs; ++c) {
                const double av = ab[r * bs + c];
                if (av == 0.0) continue;
                for (int t = 0; t < 6; ++t) s[r * 6 + t] += f * av * qj[c * 6 + t];
              }
            }
          }
        }
        acc.flush(rc[i], rv[i]);
      }
    });
    rows_to_bsr(bs, 6, n, L.n_agg, rc, rv, L.P);
    transpose(view(L.P), L.R);
    tr.mark("prolongator", lvl);
    // Galerkin product A_c = R (A P)
    HostBsr AP, Ac;
    spgemm(A, view(L.P), AP);
    tr.mark("A*P", lvl);
    spgemm(view(L.R), view(AP), Ac);
    tr.mark("R*(AP)", lvl);
    symmetrize(Ac);
    if (lvl > 0) L.A = std::move(Aown);
    out.levels.push_back(std::move(L));
    Aown = std::move(Ac);
    A = view(Aown);
    B.swap(Bc);
    bs = 6;
    n = out.levels.back().n_agg;
  }
  WN_CHECK(dense_coarse(n, bs, A.rp, A.ci, A.v, out));
  tr.mark("coarse", -1);
  // the last coarse matrix (BSR) is kept for tests through coarse_A only
  return WN_OK;
}

}  // namespace wn
