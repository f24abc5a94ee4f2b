// Smoothed-aggregation algebraic multigrid (Vanek, Mandel and Brezina, "Algebraic multigrid by smoothed
// aggregation for second and fourth order elliptic problems", Computing 56 (1996)) as the preconditioner of the
// device GMRES solve of K_con dx = f_con.  It stands in for the reference's ASM/MUMPS preconditioning
// (GMRESLinSolver.cpp:19-96) on one GPU.
//
// Set-up on the host, once per matrix (or reused across Newton iterations): aggregates of mesh nodes from the
// matrix graph, the tentative prolongator from the near-null space (rigid-body modes of the displacement step,
// constants otherwise) orthonormalised per aggregate, one damped-Jacobi smoothing step of it with
// omega = 4 / (3 rho(D^-1 A)), Galerkin coarse matrices R A P with R = P^T, and a dense inverse at the coarsest level.
// Application on the device: one symmetric V-cycle with two damped-Jacobi sweeps before and after the coarse
// correction, all products deterministic (warp-per-row CSR products, fixed summation order).

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "icefem_internal.h"

namespace ifem {

namespace {

struct HostCsr {
  int64_t nrows = 0, ncols = 0;
  std::vector<int64_t> rp{0};
  std::vector<int32_t> ci;
  std::vector<double> v;
};

// Host threads for the set-up: rows are split into contiguous ranges, one per thread; every row's result depends
// only on that row, so the output does not depend on the thread count.
int set_up_threads() {
  const unsigned hw = std::thread::hardware_concurrency();
  return (int)std::max(1u, std::min(hw, 32u));
}

template <class Fn>   // fn(thread, begin, end)
void parallel_rows(int64_t n, Fn fn) {
  // rows of the coarse levels are few but long (the restriction's rows span whole aggregates): split from 64 rows
  const int nt = (int)std::min<int64_t>(set_up_threads(), std::max<int64_t>(1, n / 64));
  if (nt <= 1) { fn(0, (int64_t)0, n); return; }
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t) {
    const int64_t b = n * t / nt, e = n * (t + 1) / nt;
    th.emplace_back([=, &fn] { fn(t, b, e); });
  }
  for (auto& x : th) x.join();
}

// C = A B (rows of A times B), columns sorted; the products of a row are summed in the order of A's columns
HostCsr spgemm(const HostCsr& A, const HostCsr& B) {
  HostCsr C;
  C.nrows = A.nrows; C.ncols = B.ncols;
  C.rp.assign(A.nrows + 1, 0);
  const int nt = set_up_threads();
  std::vector<std::vector<int32_t>> mark(nt);
  // symbolic pass: row lengths
  parallel_rows(A.nrows, [&](int t, int64_t b, int64_t e) {
    auto& mk = mark[t];
    mk.assign(B.ncols, -1);
    for (int64_t i = b; i < e; ++i) {
      int64_t cnt = 0;
      for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k)
        for (int64_t l = B.rp[A.ci[k]]; l < B.rp[A.ci[k] + 1]; ++l)
          if (mk[B.ci[l]] != (int32_t)i) { mk[B.ci[l]] = (int32_t)i; ++cnt; }
      C.rp[i + 1] = cnt;
    }
  });
  for (int64_t i = 0; i < A.nrows; ++i) C.rp[i + 1] += C.rp[i];
  C.ci.resize(C.rp[A.nrows]);
  C.v.resize(C.rp[A.nrows]);
  // numeric pass; the row's columns are known from the symbolic pass, so with few columns (the products with a
  // prolongator) a dense accumulator is read back in column order, with no marks and no sort (the same sums)
  const bool dense = B.ncols <= 4096;
  parallel_rows(A.nrows, [&](int t, int64_t b, int64_t e) {
    if (dense) {
      std::vector<double> acc(B.ncols, 0.0);
      std::vector<char> hit(B.ncols, 0);
      for (int64_t i = b; i < e; ++i) {
        for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
          const int32_t a = A.ci[k];
          const double av = A.v[k];
          for (int64_t l = B.rp[a]; l < B.rp[a + 1]; ++l) {
            acc[B.ci[l]] += av * B.v[l];
            hit[B.ci[l]] = 1;
          }
        }
        int64_t p = C.rp[i];
        for (int32_t j = 0; j < (int32_t)B.ncols; ++j)
          if (hit[j]) { C.ci[p] = j; C.v[p] = acc[j]; ++p; acc[j] = 0.0; hit[j] = 0; }
      }
      return;
    }
    auto& mk = mark[t];
    mk.assign(B.ncols, -1);
    std::vector<double> acc(B.ncols, 0.0);
    std::vector<int32_t> cols;
    for (int64_t i = b; i < e; ++i) {
      cols.clear();
      for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
        const int32_t a = A.ci[k];
        const double av = A.v[k];
        for (int64_t l = B.rp[a]; l < B.rp[a + 1]; ++l) {
          const int32_t j = B.ci[l];
          if (mk[j] != (int32_t)i) { mk[j] = (int32_t)i; acc[j] = 0.0; cols.push_back(j); }
          acc[j] += av * B.v[l];
        }
      }
      std::sort(cols.begin(), cols.end());
      int64_t p = C.rp[i];
      for (int32_t j : cols) { C.ci[p] = j; C.v[p] = acc[j]; ++p; }
    }
  });
  return C;
}

HostCsr transpose(const HostCsr& A) {
  HostCsr T;
  T.nrows = A.ncols; T.ncols = A.nrows;
  T.rp.assign(A.ncols + 1, 0);
  for (int32_t c : A.ci) T.rp[c + 1]++;
  for (int64_t i = 0; i < A.ncols; ++i) T.rp[i + 1] += T.rp[i];
  T.ci.resize(A.ci.size()); T.v.resize(A.v.size());
  std::vector<int64_t> pos(T.rp.begin(), T.rp.end() - 1);
  for (int64_t i = 0; i < A.nrows; ++i)
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      const int64_t p = pos[A.ci[k]]++;
      T.ci[p] = (int32_t)i; T.v[p] = A.v[k];
    }
  return T;
}

std::vector<double> diag_inv(const HostCsr& A) {
  std::vector<double> d(A.nrows, 1.0);
  for (int64_t i = 0; i < A.nrows; ++i)
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (A.ci[k] == i && A.v[k] != 0.0) d[i] = 1.0 / A.v[k];
  return d;
}

// largest eigenvalue of D^-1 A by power iteration (D^-1 A is similar to a symmetric matrix for SPD A)
double spectral_radius(const HostCsr& A, const std::vector<double>& dinv) {
  const int64_t n = A.nrows;
  std::vector<double> x(n), y(n);
  for (int64_t i = 0; i < n; ++i) x[i] = 1.0 + 0.1 * std::sin(0.7 * (double)i);
  double rho = 1.0;
  for (int it = 0; it < 20; ++it) {
    double nx = 0;
    for (double t : x) nx += t * t;
    nx = std::sqrt(nx);
    if (!(nx > 0)) break;
    parallel_rows(n, [&](int, int64_t b, int64_t e) {
      for (int64_t i = b; i < e; ++i) {
        double s = 0;
        for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) s += A.v[k] * x[A.ci[k]];
        y[i] = dinv[i] * s / nx;
      }
    });
    double ny = 0;
    for (double t : y) ny += t * t;
    rho = std::sqrt(ny);
    x.swap(y);
  }
  return rho;
}

}  // namespace

struct AmgLevelDev {
  int64_t n = 0, nnz = 0;
  int64_t* rp = nullptr; int32_t* ci = nullptr; double* v = nullptr; double* dinv = nullptr;
  double omega = 0.0;
  int64_t nc = 0;                          // coarse rows
  int64_t *prp = nullptr, *rrp = nullptr;  // prolongator (n x nc) and restriction R = P^T (nc x n)
  int32_t *pci = nullptr, *rci = nullptr;
  double *pv = nullptr, *rv = nullptr;
  double *x = nullptr, *b = nullptr, *t = nullptr;   // level vectors
};

struct AmgHierarchy {
  std::vector<AmgLevelDev> lv;
  // coarsest level: dense inverse stored as a full CSR
  int64_t nc = 0;
  int64_t* crp = nullptr; int32_t* cci = nullptr; double* cv = nullptr;
  double *cx = nullptr, *cb = nullptr;
  double setup_ms = 0.0;
  int sweeps = 2;
  std::vector<int64_t> sizes, nnzs;
  // the V-cycle between its first level's input and output buffers, captured once as a CUDA graph (about 10
  // launches per level); graph_state 0 not yet captured, 1 captured, -1 capture unavailable (direct launches)
  cudaGraphExec_t graph = nullptr;
  int graph_state = 0;
};


namespace {

// Aggregates of the level's nodes (Vanek et al., sec. 3): a node whose neighbours are all free starts an aggregate
// of itself and its neighbours; remaining nodes join a neighbouring aggregate of the first pass; isolated ones
// form their own.
std::vector<int32_t> aggregate(const HostCsr& A, const std::vector<int32_t>& node, int64_t nnodes, double theta,
                               int64_t& nagg) {
  // strong couplings (Vanek et al., sec. 3): |a_ij| >= theta sqrt(|a_ii a_jj|); theta = 0 keeps the whole graph
  std::vector<double> dabs(A.nrows, 0.0);
  for (int64_t i = 0; i < A.nrows; ++i)
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (A.ci[k] == i) dabs[i] = std::fabs(A.v[k]);
  // rows of each node, then the node graph (sorted neighbour lists), one node per task
  std::vector<int64_t> nrp(nnodes + 1, 0);
  for (int64_t i = 0; i < A.nrows; ++i) nrp[node[i] + 1]++;
  for (int64_t a = 0; a < nnodes; ++a) nrp[a + 1] += nrp[a];
  std::vector<int64_t> nrows(A.nrows), pos(nrp.begin(), nrp.end() - 1);
  for (int64_t i = 0; i < A.nrows; ++i) nrows[pos[node[i]]++] = i;
  std::vector<std::vector<int32_t>> adj(nnodes);
  const int nt = set_up_threads();
  std::vector<std::vector<int32_t>> mark(nt);
  parallel_rows(nnodes, [&](int t, int64_t b, int64_t e) {
    auto& mk = mark[t];
    mk.assign(nnodes, -1);
    for (int64_t a = b; a < e; ++a) {
      auto& v = adj[a];
      for (int64_t r = nrp[a]; r < nrp[a + 1]; ++r) {
        const int64_t i = nrows[r];
        for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
          const int32_t c = node[A.ci[k]];
          if (c == a || mk[c] == (int32_t)a) continue;
          if (theta > 0.0 && std::fabs(A.v[k]) < theta * std::sqrt(dabs[i] * dabs[A.ci[k]])) continue;
          mk[c] = (int32_t)a;
          v.push_back(c);
        }
      }
      std::sort(v.begin(), v.end());
    }
  });
  std::vector<int32_t> agg(nnodes, -1);
  nagg = 0;
  for (int64_t a = 0; a < nnodes; ++a) {
    if (agg[a] >= 0) continue;
    bool free_nb = true;
    for (int32_t b : adj[a]) if (agg[b] >= 0) { free_nb = false; break; }
    if (!free_nb) continue;
    agg[a] = (int32_t)nagg;
    for (int32_t b : adj[a]) agg[b] = (int32_t)nagg;
    ++nagg;
  }
  const std::vector<int32_t> first(agg);
  for (int64_t a = 0; a < nnodes; ++a) {
    if (agg[a] >= 0) continue;
    for (int32_t b : adj[a]) if (first[b] >= 0) { agg[a] = first[b]; break; }
  }
  for (int64_t a = 0; a < nnodes; ++a) if (agg[a] < 0) agg[a] = (int32_t)nagg++;
  return agg;
}

// Tentative prolongator: per aggregate, the near-null-space rows of its dofs orthonormalised by modified
// Gram-Schmidt (columns that vanish are dropped); R gives the coarse near-null space.
void tentative(const std::vector<int32_t>& node, const std::vector<int32_t>& agg, int64_t nagg, const std::vector<double>& B,
               int nm, HostCsr& P0, std::vector<double>& Bc, std::vector<int32_t>& cnode) {
  const int64_t n = (int64_t)node.size();
  std::vector<std::vector<int64_t>> rows(nagg);
  for (int64_t i = 0; i < n; ++i) rows[agg[node[i]]].push_back(i);
  std::vector<int32_t> col0(nagg + 1, 0);
  std::vector<std::vector<double>> Q(nagg);
  std::vector<int> kept(nagg, 0);
  Bc.clear(); cnode.clear();
  for (int64_t g = 0; g < nagg; ++g) {
    const auto& r = rows[g];
    const int64_t m = (int64_t)r.size();
    std::vector<double> q;   // [kept][m]
    std::vector<double> Rg;  // [kept][nm]
    std::vector<double> rrow(nm);
    for (int j = 0; j < nm; ++j) {
      std::vector<double> v(m);
      double n0 = 0;
      for (int64_t i = 0; i < m; ++i) { v[i] = B[r[i] * nm + j]; n0 += v[i] * v[i]; }
      n0 = std::sqrt(n0);
      std::vector<double> coef(kept[g] + 1, 0.0);
      for (int k = 0; k < kept[g]; ++k) {
        double d = 0;
        for (int64_t i = 0; i < m; ++i) d += q[k * m + i] * v[i];
        for (int64_t i = 0; i < m; ++i) v[i] -= d * q[k * m + i];
        coef[k] = d;
      }
      double nv = 0;
      for (double t : v) nv += t * t;
      nv = std::sqrt(nv);
      // R (coarse near-null space) column j: the projections on the kept q's, and the new q's own norm
      if (nv > 1e-10 * n0 && nv > 0) {
        for (int64_t i = 0; i < m; ++i) q.push_back(v[i] / nv);
        coef[kept[g]] = nv;
        kept[g] += 1;
        Rg.resize((size_t)kept[g] * nm, 0.0);
      }
      for (int k = 0; k < kept[g]; ++k) Rg[(size_t)k * nm + j] = coef[k];
    }
    Q[g].swap(q);
    col0[g + 1] = col0[g] + kept[g];
    for (int k = 0; k < kept[g]; ++k) {
      for (int j = 0; j < nm; ++j) Bc.push_back(Rg[(size_t)k * nm + j]);
      cnode.push_back((int32_t)g);
    }
  }
  P0.nrows = n; P0.ncols = col0[nagg];
  P0.rp.assign(n + 1, 0);
  std::vector<int64_t> loc(n);
  for (int64_t g = 0; g < nagg; ++g) for (size_t i = 0; i < rows[g].size(); ++i) loc[rows[g][i]] = (int64_t)i;
  P0.ci.clear(); P0.v.clear();
  for (int64_t i = 0; i < n; ++i) {
    const int32_t g = agg[node[i]];
    const int64_t m = (int64_t)rows[g].size();
    for (int k = 0; k < kept[g]; ++k) { P0.ci.push_back(col0[g] + k); P0.v.push_back(Q[g][(size_t)k * m + loc[i]]); }
    P0.rp[i + 1] = (int64_t)P0.ci.size();
  }
}

// P = (I - omega D^-1 A) P0
HostCsr smooth(const HostCsr& A, const std::vector<double>& dinv, double omega, const HostCsr& P0) {
  HostCsr AP = spgemm(A, P0);
  HostCsr P;
  P.nrows = P0.nrows; P.ncols = P0.ncols;
  P.rp.assign(P.nrows + 1, 0);
  // row i of P merges the sorted rows i of P0 and A P0: count, prefix sum, fill (rows independent)
  auto merge = [&](int64_t i, bool fill) {
    int64_t a = P0.rp[i], b = AP.rp[i], o = fill ? P.rp[i] : 0, cnt = 0;
    while (a < P0.rp[i + 1] || b < AP.rp[i + 1]) {
      const int32_t ca = a < P0.rp[i + 1] ? P0.ci[a] : INT32_MAX, cb = b < AP.rp[i + 1] ? AP.ci[b] : INT32_MAX;
      double val = 0;
      int32_t c;
      if (ca == cb) { c = ca; val = P0.v[a++] - omega * dinv[i] * AP.v[b++]; }
      else if (ca < cb) { c = ca; val = P0.v[a++]; }
      else { c = cb; val = -omega * dinv[i] * AP.v[b++]; }
      if (fill) { P.ci[o + cnt] = c; P.v[o + cnt] = val; }
      ++cnt;
    }
    return cnt;
  };
  parallel_rows(P.nrows, [&](int, int64_t b, int64_t e) { for (int64_t i = b; i < e; ++i) P.rp[i + 1] = merge(i, false); });
  for (int64_t i = 0; i < P.nrows; ++i) P.rp[i + 1] += P.rp[i];
  P.ci.resize(P.rp[P.nrows]);
  P.v.resize(P.rp[P.nrows]);
  parallel_rows(P.nrows, [&](int, int64_t b, int64_t e) { for (int64_t i = b; i < e; ++i) merge(i, true); });
  return P;
}

// dense inverse by LU with partial pivoting (the coarsest level, a few hundred unknowns)
bool dense_inverse(int64_t n, std::vector<double>& A, std::vector<double>& Ainv) {
  std::vector<int64_t> piv(n);
  for (int64_t k = 0; k < n; ++k) {
    int64_t p = k; double best = std::fabs(A[k * n + k]);
    for (int64_t i = k + 1; i < n; ++i) if (std::fabs(A[i * n + k]) > best) { best = std::fabs(A[i * n + k]); p = i; }
    piv[k] = p;
    if (!(best > 0)) return false;
    if (p != k) for (int64_t j = 0; j < n; ++j) std::swap(A[k * n + j], A[p * n + j]);
    const double inv = 1.0 / A[k * n + k];
    for (int64_t i = k + 1; i < n; ++i) {
      const double l = A[i * n + k] * inv;
      A[i * n + k] = l;
      if (l != 0.0) for (int64_t j = k + 1; j < n; ++j) A[i * n + j] -= l * A[k * n + j];
    }
  }
  Ainv.assign((size_t)n * n, 0.0);
  std::vector<double> x(n);
  for (int64_t c = 0; c < n; ++c) {
    for (int64_t i = 0; i < n; ++i) x[i] = (i == c) ? 1.0 : 0.0;
    for (int64_t k = 0; k < n; ++k) if (piv[k] != k) std::swap(x[k], x[piv[k]]);
    for (int64_t i = 1; i < n; ++i) { double s = x[i]; for (int64_t j = 0; j < i; ++j) s -= A[i * n + j] * x[j]; x[i] = s; }
    for (int64_t i = n - 1; i >= 0; --i) { double s = x[i]; for (int64_t j = i + 1; j < n; ++j) s -= A[i * n + j] * x[j]; x[i] = s / A[i * n + i]; }
    for (int64_t i = 0; i < n; ++i) Ainv[(size_t)i * n + c] = x[i];
  }
  return true;
}

template <class T>
T* up(const std::vector<T>& h) {
  T* d = nullptr;
  if (cudaMalloc(&d, std::max<size_t>(1, h.size()) * sizeof(T)) != cudaSuccess) throw Err{IFEM_ERR_NOMEM, "AMG: cudaMalloc"};
  if (!h.empty() && cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
    throw Err{IFEM_ERR_CUDA, "AMG: upload"};
  return d;
}

double* dvec(int64_t n) {
  double* d = nullptr;
  if (cudaMalloc(&d, std::max<int64_t>(1, n) * sizeof(double)) != cudaSuccess) throw Err{IFEM_ERR_NOMEM, "AMG: cudaMalloc"};
  return d;
}

}  // namespace


namespace {

__global__ void k_jacobi(int64_t n, double omega, const double* dinv, const double* b, const double* t, double* x,
                         int first) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (first) x[i] = omega * dinv[i] * b[i];
  else x[i] += omega * dinv[i] * (b[i] - t[i]);
}

__global__ void k_add(int64_t n, const double* t, double* x) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += t[i];
}

__global__ void k_copy(int64_t n, const double* a, double* b) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = a[i];
}

inline unsigned blocks_of(int64_t n) { return (unsigned)((n + 255) / 256); }


}  // namespace

namespace {

struct HostLevel {
  HostCsr A, P, R;
  std::vector<double> dinv;
  double omega = 0.0;
};

// The hierarchy on the host: per level the operator, the smoothed prolongator and its transpose; the last
// matrix is the coarsest one.  node_of_row gives each row's mesh node (level-0 aggregation works on nodes), B the
// near-null space [n][nm].
void plan_hierarchy(HostCsr A, std::vector<int32_t> node, int64_t nn, int nm, std::vector<double> Bl,
                    const AmgOptions& opt, std::vector<HostLevel>& lv, HostCsr& coarse, std::vector<int64_t>& sizes,
                    std::vector<int64_t>& nnzs) {
  for (int level = 0; level < 10; ++level) {
    sizes.push_back(A.nrows); nnzs.push_back((int64_t)A.ci.size());
    if (A.nrows <= 800 || level == 9) break;
    int64_t nagg = 0;
    const std::vector<int32_t> agg = aggregate(A, node, nn, opt.theta * std::ldexp(1.0, -level), nagg);
    HostCsr P0;
    std::vector<double> Bc;
    std::vector<int32_t> cnode;
    tentative(node, agg, nagg, Bl, nm, P0, Bc, cnode);
    if (P0.ncols >= (int64_t)(0.8 * A.nrows) || P0.ncols == 0) break;   // coarsening has stalled
    HostLevel L;
    L.dinv = diag_inv(A);
    const double rho = spectral_radius(A, L.dinv);
    L.omega = 4.0 / (3.0 * rho);
    L.P = smooth(A, L.dinv, L.omega, P0);
    L.R = transpose(L.P);
    HostCsr Ac = spgemm(L.R, spgemm(A, L.P));
    L.A = std::move(A);
    lv.push_back(std::move(L));
    A = std::move(Ac);
    node = std::move(cnode); nn = nagg; Bl = std::move(Bc);
  }
  coarse = std::move(A);
}

}  // namespace

// Hierarchy from the constrained system: planned on the host, then uploaded with a dense inverse of the coarsest
// matrix.
AmgHierarchy* amg_build(int64_t n, const std::vector<int64_t>& rp, const std::vector<int32_t>& ci,
                        const std::vector<double>& v, const std::vector<int32_t>& node_of_row, int64_t nnodes, int nm,
                        const std::vector<double>& B, const AmgOptions& opt) {
  const auto t0 = std::chrono::steady_clock::now();
  AmgHierarchy* h = new AmgHierarchy();
  h->sweeps = opt.sweeps;
  try {
    HostCsr A;
    A.nrows = A.ncols = n; A.rp = rp; A.ci = ci; A.v = v;
    std::vector<HostLevel> lv;
    HostCsr C;
    plan_hierarchy(std::move(A), node_of_row, nnodes, nm, B, opt, lv, C, h->sizes, h->nnzs);
    for (HostLevel& H : lv) {
      AmgLevelDev L;
      L.n = H.A.nrows; L.nnz = (int64_t)H.A.ci.size();
      L.rp = up(H.A.rp); L.ci = up(H.A.ci); L.v = up(H.A.v); L.dinv = up(H.dinv);
      L.omega = H.omega;
      L.nc = H.P.ncols;
      L.prp = up(H.P.rp); L.pci = up(H.P.ci); L.pv = up(H.P.v);
      L.rrp = up(H.R.rp); L.rci = up(H.R.ci); L.rv = up(H.R.v);
      L.x = dvec(L.n); L.b = dvec(L.n); L.t = dvec(L.n);
      h->lv.push_back(L);
      H = HostLevel();   // release the host copies as they go up
    }
    // coarsest level: dense inverse
    const int64_t nc = C.nrows;
    if (nc > 6000) throw Err{IFEM_ERR_UNSUPPORTED, "AMG: coarsening stalled at " + std::to_string(nc) + " rows"};
    std::vector<double> D((size_t)nc * nc, 0.0), Dinv;
    for (int64_t i = 0; i < nc; ++i)
      for (int64_t k = C.rp[i]; k < C.rp[i + 1]; ++k) D[(size_t)i * nc + C.ci[k]] = C.v[k];
    if (!dense_inverse(nc, D, Dinv)) throw Err{IFEM_ERR_NUMERIC, "AMG: singular coarsest matrix"};
    std::vector<int64_t> crp(nc + 1);
    std::vector<int32_t> cci((size_t)nc * nc);
    for (int64_t i = 0; i <= nc; ++i) crp[i] = i * nc;
    for (int64_t i = 0; i < nc; ++i) for (int64_t j = 0; j < nc; ++j) cci[(size_t)i * nc + j] = (int32_t)j;
    h->nc = nc;
    h->crp = up(crp); h->cci = up(cci); h->cv = up(Dinv);
    h->cx = dvec(nc); h->cb = dvec(nc);
  } catch (...) {
    amg_free(h);
    throw;
  }
  h->setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return h;
}

void amg_free(AmgHierarchy* h) {
  if (!h) return;
  auto F = [](void* p) { if (p) cudaFree(p); };
  for (auto& L : h->lv) {
    F(L.rp); F(L.ci); F(L.v); F(L.dinv); F(L.prp); F(L.pci); F(L.pv); F(L.rrp); F(L.rci); F(L.rv);
    F(L.x); F(L.b); F(L.t);
  }
  F(h->crp); F(h->cci); F(h->cv); F(h->cx); F(h->cb);
  if (h->graph) cudaGraphExecDestroy(h->graph);
  delete h;
}

int amg_levels(const AmgHierarchy* h, int64_t* sizes, int max_levels) {
  const int nl = (int)h->sizes.size();
  for (int i = 0; i < nl && i < max_levels; ++i) sizes[i] = h->sizes[i];
  return nl;
}

double amg_setup_ms(const AmgHierarchy* h) { return h->setup_ms; }

namespace {

// lv[0].b -> lv[0].x: one V-cycle from a zero guess on the hierarchy's own buffers
void v_cycle(const AmgHierarchy* h, cudaStream_t s) {
  const int nl = (int)h->lv.size();
  // down: smooth from zero, restrict the residual
  for (int l = 0; l < nl; ++l) {
    const AmgLevelDev& L = h->lv[l];
    k_jacobi<<<blocks_of(L.n), 256, 0, s>>>(L.n, L.omega, L.dinv, L.b, nullptr, L.x, 1);
    for (int k = 1; k < h->sweeps; ++k) {
      launch_spmv(L.n, L.rp, L.ci, L.v, 0, L.x, L.t, s);
      k_jacobi<<<blocks_of(L.n), 256, 0, s>>>(L.n, L.omega, L.dinv, L.b, L.t, L.x, 0);
    }
    launch_spmv(L.n, L.rp, L.ci, L.v, 0, L.x, L.t, s);
    launch_sub(L.n, L.b, L.t, L.t, s);                       // t = b - A x
    double* bc = (l + 1 < nl) ? h->lv[l + 1].b : h->cb;
    launch_spmv(L.nc, L.rrp, L.rci, L.rv, 0, L.t, bc, s);    // b_c = R t
  }
  launch_spmv(h->nc, h->crp, h->cci, h->cv, 0, h->cb, h->cx, s);   // coarsest: dense inverse
  // up: prolong the correction, smooth
  for (int l = nl - 1; l >= 0; --l) {
    const AmgLevelDev& L = h->lv[l];
    const double* xc = (l + 1 < nl) ? h->lv[l + 1].x : h->cx;
    launch_spmv(L.n, L.prp, L.pci, L.pv, 0, xc, L.t, s);
    k_add<<<blocks_of(L.n), 256, 0, s>>>(L.n, L.t, L.x);
    for (int k = 0; k < h->sweeps; ++k) {
      launch_spmv(L.n, L.rp, L.ci, L.v, 0, L.x, L.t, s);
      k_jacobi<<<blocks_of(L.n), 256, 0, s>>>(L.n, L.omega, L.dinv, L.b, L.t, L.x, 0);
    }
  }
}

}  // namespace

// out = M^-1 in, one V-cycle from a zero guess (in and out may alias); the cycle itself replays a CUDA graph
void amg_apply(AmgHierarchy* h, const double* in, double* out, cudaStream_t s) {
  const int nl = (int)h->lv.size();
  if (nl == 0) {
    k_copy<<<blocks_of(h->nc), 256, 0, s>>>(h->nc, in, h->cb);
    launch_spmv(h->nc, h->crp, h->cci, h->cv, 0, h->cb, out, s);
    return;
  }
  k_copy<<<blocks_of(h->lv[0].n), 256, 0, s>>>(h->lv[0].n, in, h->lv[0].b);
  if (h->graph_state == 0) {
    h->graph_state = -1;
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      v_cycle(h, s);
      if (cudaStreamEndCapture(s, &g) == cudaSuccess && g) {
        if (cudaGraphInstantiate(&h->graph, g, 0) == cudaSuccess) h->graph_state = 1;
        cudaGraphDestroy(g);
      }
    }
    cudaGetLastError();   // a refused capture leaves no sticky error; the cycle then runs as direct launches
  }
  if (h->graph_state == 1) {
    if (cudaGraphLaunch(h->graph, s) != cudaSuccess) throw Err{IFEM_ERR_CUDA, "AMG: graph launch"};
  } else {
    v_cycle(h, s);
  }
  k_copy<<<blocks_of(h->lv[0].n), 256, 0, s>>>(h->lv[0].n, h->lv[0].x, out);
}

}  // namespace ifem

// Host-only planning of the hierarchy (no device memory): rows and nonzeros per level, for tests and for sizing.
extern "C" int ifem_multigrid_plan(int64_t n, const int64_t* row_ptr, const int32_t* col_idx, const double* vals,
                                   const int32_t* node_of_row, int64_t n_nodes, int32_t n_modes, const double* modes,
                                   double strength_threshold, int32_t max_levels, int32_t* levels, int64_t* rows_out,
                                   int64_t* nnz_out) {
  using namespace ifem;
  if (n < 0 || !row_ptr || (n > 0 && (!col_idx || !vals || !node_of_row || !modes)) || n_nodes < 0 || n_modes < 1 ||
      !(strength_threshold >= 0.0 && strength_threshold < 1.0) || max_levels < 1 || !levels)
    return IFEM_ERR_INVALID;
  try {
    if (row_ptr[0] != 0) return IFEM_ERR_INVALID;
    for (int64_t i = 0; i < n; ++i)
      if (row_ptr[i + 1] < row_ptr[i] || node_of_row[i] < 0 || node_of_row[i] >= n_nodes) return IFEM_ERR_INVALID;
    const int64_t nnz = row_ptr[n];
    for (int64_t k = 0; k < nnz; ++k)
      if (col_idx[k] < 0 || col_idx[k] >= n) return IFEM_ERR_INVALID;
    HostCsr A;
    A.nrows = A.ncols = n;
    A.rp.assign(row_ptr, row_ptr + n + 1);
    A.ci.assign(col_idx, col_idx + nnz);
    A.v.assign(vals, vals + nnz);
    AmgOptions opt;
    opt.theta = strength_threshold;
    std::vector<HostLevel> lv;
    HostCsr C;
    std::vector<int64_t> sizes, nnzs;
    plan_hierarchy(std::move(A), std::vector<int32_t>(node_of_row, node_of_row + n), n_nodes, n_modes,
                   std::vector<double>(modes, modes + (size_t)n * n_modes), opt, lv, C, sizes, nnzs);
    *levels = (int32_t)sizes.size();
    for (int i = 0; i < (int)sizes.size() && i < max_levels; ++i) {
      if (rows_out) rows_out[i] = sizes[i];
      if (nnz_out) nnz_out[i] = nnzs[i];
    }
    return IFEM_OK;
  } catch (const Err& e) {
    return e.code;
  } catch (const std::bad_alloc&) {
    return IFEM_ERR_NOMEM;
  } catch (...) {
    return IFEM_ERR_INVALID;
  }
}
