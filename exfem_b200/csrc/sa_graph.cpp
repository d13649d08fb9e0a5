// Host graph work of the device smoothed-aggregation set-up: mesh node
// adjacency, rigid-body modes, the tentative prolongator (per-aggregate
// orthonormalisation of the near-null space), the sparsity patterns of P, A P
// and P^T A P, and the coarsest-level inverse.  The numeric products run on the
// device (sa_setup.cu); only index lists and small dense work are done here.
//
// Follows the smoothed-aggregation set-up the reference obtains from
// pyamg.smoothed_aggregation_solver (gfem/linalg.py:103-136): rigid-body modes
// as near-null space (gfem/linalg.py:80-98), standard aggregation on the
// theta = 0 strength graph, tentative prolongator by orthonormalising the
// candidates per aggregate, and a dense coarsest solve by a Cholesky factor
// regularised with 1e-13 max|A| (gfem/linalg.py:122-133).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>

#include "sa.h"

namespace exfem {

namespace {

int nthreads(int64_t work) {
  unsigned t = std::thread::hardware_concurrency();
  if (t == 0) t = 4;
  if (t > 32) t = 32;
  const int64_t per = 1 << 14;  // rows per thread at least
  int64_t m = (work + per - 1) / per;
  if (m < 1) m = 1;
  return (int)std::min<int64_t>(t, m);
}

template <class F>
void parallel_ranges(int64_t n, F f) {
  const int T = nthreads(n);
  if (T == 1) { f(0, (int64_t)0, n); return; }
  std::vector<std::thread> th;
  for (int t = 0; t < T; ++t) {
    const int64_t lo = n * t / T, hi = n * (t + 1) / T;
    th.emplace_back([=]() { f(t, lo, hi); });
  }
  for (auto& x : th) x.join();
}

// Build rows in parallel: fn(row, stamp, out) appends row's sorted list to out;
// stamp is a per-thread marker array of ncols entries (initially -1).
template <class F>
void build_rows(int64_t nrows, int64_t ncols, Rows& R, F fn) {
  const int T = nthreads(nrows);
  std::vector<std::vector<int32_t>> part(T);
  std::vector<std::vector<int64_t>> len(T);
  auto work = [&](int t, int64_t lo, int64_t hi) {
    std::vector<int64_t> stamp((size_t)std::max<int64_t>(ncols, 1), -1);
    auto& out = part[t];
    auto& L = len[t];
    L.reserve(hi - lo);
    for (int64_t i = lo; i < hi; ++i) {
      const size_t before = out.size();
      fn(i, stamp, out);
      std::sort(out.begin() + before, out.end());
      L.push_back((int64_t)(out.size() - before));
    }
  };
  if (T == 1) {
    work(0, 0, nrows);
  } else {
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t) {
      const int64_t lo = nrows * t / T, hi = nrows * (t + 1) / T;
      th.emplace_back(work, t, lo, hi);
    }
    for (auto& x : th) x.join();
  }
  // concatenation: each thread's rows and entries land at offsets known from the
  // part sizes, so the threads write their ranges of ptr and idx side by side
  std::vector<int64_t> row0(T + 1, 0), off(T + 1, 0);
  for (int t = 0; t < T; ++t) {
    row0[t + 1] = row0[t] + (int64_t)len[t].size();
    off[t + 1] = off[t] + (int64_t)part[t].size();
  }
  R.ptr.resize(nrows + 1);
  R.ptr[0] = 0;
  R.idx.resize(off[T]);
  auto place = [&](int t) {
    int64_t o = off[t];
    for (size_t i = 0; i < len[t].size(); ++i) {
      o += len[t][i];
      R.ptr[row0[t] + (int64_t)i + 1] = o;
    }
    if (!part[t].empty()) std::memcpy(R.idx.data() + off[t], part[t].data(), part[t].size() * sizeof(int32_t));
    std::vector<int32_t>().swap(part[t]);
  };
  if (T == 1) {
    place(0);
  } else {
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t) th.emplace_back(place, t);
    for (auto& x : th) x.join();
  }
}

}  // namespace

int host_node_adjacency(int64_t nn, int64_t ne, int nnode, const int32_t* conn, Rows& out) {
  // node -> elements by a counting sort
  std::vector<int64_t> eptr(nn + 1, 0);
  for (int64_t k = 0; k < ne * nnode; ++k) {
    const int32_t n = conn[k];
    if (n < 0 || n >= nn) {
      set_error("connectivity entry %d at slot %lld is outside [0, %lld)", n, (long long)k, (long long)nn);
      return EXFEM_ERR_ARG;
    }
    ++eptr[n + 1];
  }
  for (int64_t n = 0; n < nn; ++n) eptr[n + 1] += eptr[n];
  std::vector<int32_t> elem(eptr[nn]);
  {
    std::vector<int64_t> fill(eptr.begin(), eptr.end() - 1);
    for (int64_t e = 0; e < ne; ++e)
      for (int a = 0; a < nnode; ++a) elem[fill[conn[e * nnode + a]]++] = (int32_t)e;
  }
  build_rows(nn, nn, out, [&](int64_t n, std::vector<int64_t>& stamp, std::vector<int32_t>& o) {
    for (int64_t k = eptr[n]; k < eptr[n + 1]; ++k) {
      const int32_t* c = conn + (int64_t)elem[k] * nnode;
      for (int a = 0; a < nnode; ++a)
        if (stamp[c[a]] != n) { stamp[c[a]] = n; o.push_back(c[a]); }
    }
    if (stamp[n] != n) { stamp[n] = n; o.push_back((int32_t)n); }  // an unused node still lists itself
  });
  return EXFEM_OK;
}

void host_filter_pattern(const Rows& pat, const uint8_t* flag, Rows& S, std::vector<int64_t>& keep) {
  const int64_t nr = pat.nrows();
  S.ptr.assign(nr + 1, 0);
  parallel_ranges(nr, [&](int, int64_t lo, int64_t hi) {
    for (int64_t r = lo; r < hi; ++r) {
      int64_t c = 0;
      for (int64_t q = pat.ptr[r]; q < pat.ptr[r + 1]; ++q) c += flag[q] ? 1 : 0;
      S.ptr[r + 1] = c;
    }
  });
  for (int64_t r = 0; r < nr; ++r) S.ptr[r + 1] += S.ptr[r];
  S.idx.resize(S.ptr[nr]);
  keep.resize(S.ptr[nr]);
  parallel_ranges(nr, [&](int, int64_t lo, int64_t hi) {
    for (int64_t r = lo; r < hi; ++r) {
      int64_t o = S.ptr[r];
      for (int64_t q = pat.ptr[r]; q < pat.ptr[r + 1]; ++q)
        if (flag[q]) {
          S.idx[o] = pat.idx[q];
          keep[o] = q;
          ++o;
        }
    }
  });
}

void host_rigid_body_modes(int64_t nn, const double* X, std::vector<double>& B) {
  double m[3] = {0, 0, 0};
  for (int64_t i = 0; i < nn; ++i)
    for (int d = 0; d < 3; ++d) m[d] += X[3 * i + d];
  for (int d = 0; d < 3; ++d) m[d] /= (double)std::max<int64_t>(nn, 1);
  B.assign((size_t)nn * 3 * 6, 0.0);
  for (int64_t i = 0; i < nn; ++i) {
    const double x = X[3 * i] - m[0], y = X[3 * i + 1] - m[1], z = X[3 * i + 2] - m[2];
    double* r0 = &B[(3 * i + 0) * 6];
    double* r1 = &B[(3 * i + 1) * 6];
    double* r2 = &B[(3 * i + 2) * 6];
    r0[0] = 1; r1[1] = 1; r2[2] = 1;          // translations
    r0[3] = -y; r1[3] = x;                    // rotation about z
    r1[4] = -z; r2[4] = y;                    // rotation about x
    r0[5] = z;  r2[5] = -x;                   // rotation about y
  }
}

void host_fit_candidates(int64_t nb, int bs, int K, const int32_t* agg, int64_t nagg, const double* B,
                         std::vector<double>& Q, std::vector<double>& Bc, double drop) {
  Q.assign((size_t)nb * bs * K, 0.0);
  Bc.assign((size_t)nagg * K * K, 0.0);
  // members of each aggregate in increasing node order
  std::vector<int64_t> aptr(nagg + 1, 0);
  for (int64_t n = 0; n < nb; ++n)
    if (agg[n] >= 0) ++aptr[agg[n] + 1];
  for (int64_t g = 0; g < nagg; ++g) aptr[g + 1] += aptr[g];
  std::vector<int32_t> mem(aptr[nagg]);
  {
    std::vector<int64_t> fill(aptr.begin(), aptr.end() - 1);
    for (int64_t n = 0; n < nb; ++n)
      if (agg[n] >= 0) mem[fill[agg[n]]++] = (int32_t)n;
  }
  parallel_ranges(nagg, [&](int, int64_t lo, int64_t hi) {
    std::vector<double> q, n0(K);
    for (int64_t g = lo; g < hi; ++g) {
      const int64_t nm = aptr[g + 1] - aptr[g];
      const int64_t m = nm * bs;
      q.assign((size_t)m * K, 0.0);
      for (int64_t a = 0; a < nm; ++a) {
        const int64_t node = mem[aptr[g] + a];
        for (int r = 0; r < bs; ++r)
          for (int k = 0; k < K; ++k) q[(a * bs + r) * K + k] = B[(node * bs + r) * K + k];
      }
      for (int k = 0; k < K; ++k) {
        double s = 0;
        for (int64_t i = 0; i < m; ++i) s += q[i * K + k] * q[i * K + k];
        n0[k] = std::sqrt(s) + 1e-300;
      }
      double* R = &Bc[(size_t)g * K * K];
      for (int j = 0; j < K; ++j) {
        for (int i = 0; i < j; ++i) {
          double rij = 0;
          for (int64_t t = 0; t < m; ++t) rij += q[t * K + i] * q[t * K + j];
          R[i * K + j] = rij;
          for (int64_t t = 0; t < m; ++t) q[t * K + j] -= rij * q[t * K + i];
        }
        double s = 0;
        for (int64_t t = 0; t < m; ++t) s += q[t * K + j] * q[t * K + j];
        const double nj = std::sqrt(s);
        const bool ok = nj > drop * n0[j];
        R[j * K + j] = ok ? nj : 0.0;
        for (int64_t t = 0; t < m; ++t) q[t * K + j] = ok ? q[t * K + j] / nj : 0.0;
      }
      for (int64_t a = 0; a < nm; ++a) {
        const int64_t node = mem[aptr[g] + a];
        for (int r = 0; r < bs; ++r)
          for (int k = 0; k < K; ++k) Q[(node * bs + r) * K + k] = q[(a * bs + r) * K + k];
      }
    }
  });
}

void host_p_pattern(const Rows& S, const int32_t* agg, int64_t nagg, Rows& P) {
  build_rows(S.nrows(), nagg, P, [&](int64_t n, std::vector<int64_t>& stamp, std::vector<int32_t>& o) {
    auto add = [&](int32_t g) {
      if (g >= 0 && stamp[g] != n) { stamp[g] = n; o.push_back(g); }
    };
    add(agg[n]);
    for (int64_t k = S.ptr[n]; k < S.ptr[n + 1]; ++k) add(agg[S.idx[k]]);
  });
}

void host_union_pattern(const Rows& outer, const Rows& inner, int64_t ncols, Rows& out) {
  build_rows(outer.nrows(), ncols, out, [&](int64_t i, std::vector<int64_t>& stamp, std::vector<int32_t>& o) {
    for (int64_t k = outer.ptr[i]; k < outer.ptr[i + 1]; ++k) {
      const int32_t j = outer.idx[k];
      for (int64_t l = inner.ptr[j]; l < inner.ptr[j + 1]; ++l) {
        const int32_t c = inner.idx[l];
        if (stamp[c] != i) { stamp[c] = i; o.push_back(c); }
      }
    }
  });
}

void host_transpose_pattern(const Rows& P, int64_t ncols, Rows& PT, std::vector<int32_t>& slot) {
  const int64_t n = P.nrows();
  PT.ptr.assign(ncols + 1, 0);
  for (int32_t g : P.idx) ++PT.ptr[g + 1];
  for (int64_t g = 0; g < ncols; ++g) PT.ptr[g + 1] += PT.ptr[g];
  PT.idx.resize(P.idx.size());
  slot.resize(P.idx.size());
  std::vector<int64_t> fill(PT.ptr.begin(), PT.ptr.end() - 1);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t k = P.ptr[i]; k < P.ptr[i + 1]; ++k) {
      const int64_t d = fill[P.idx[k]]++;
      PT.idx[d] = (int32_t)i;
      slot[d] = (int32_t)(k - P.ptr[i]);
    }
}

int host_coarse_inverse(int64_t n, std::vector<double>& A, std::vector<double>& Ainv) {
  double amax = 0;
  for (int64_t i = 0; i < n; ++i)
    for (int64_t j = 0; j < n; ++j) {
      const double s = 0.5 * (A[i * n + j] + A[j * n + i]);
      A[i * n + j] = s;
      amax = std::max(amax, std::fabs(s));
    }
  std::vector<double> L((size_t)n * n);
  // regularised Cholesky; should rounding leave the matrix indefinite, retry
  // with a larger shift
  for (double reg = 1e-13;; reg *= 100.0) {
    bool ok = true;
    std::fill(L.begin(), L.end(), 0.0);
    for (int64_t j = 0; j < n && ok; ++j) {
      double d = A[j * n + j] + reg * amax;
      for (int64_t k = 0; k < j; ++k) d -= L[j * n + k] * L[j * n + k];
      if (!(d > 0)) { ok = false; break; }
      const double ljj = std::sqrt(d);
      L[j * n + j] = ljj;
      for (int64_t i = j + 1; i < n; ++i) {
        double s = A[i * n + j];
        for (int64_t k = 0; k < j; ++k) s -= L[i * n + k] * L[j * n + k];
        L[i * n + j] = s / ljj;
      }
    }
    if (ok) break;
    if (reg > 1e-3 || amax == 0) {
      set_error("coarsest AMG matrix (%lld rows) is not positive definite", (long long)n);
      return EXFEM_ERR_NONFINITE;
    }
  }
  // Linv = L^-1 (lower triangular), Ainv = Linv^T Linv
  std::vector<double> Li((size_t)n * n, 0.0);
  for (int64_t c = 0; c < n; ++c) {
    Li[c * n + c] = 1.0 / L[c * n + c];
    for (int64_t i = c + 1; i < n; ++i) {
      double s = 0;
      for (int64_t k = c; k < i; ++k) s += L[i * n + k] * Li[k * n + c];
      Li[i * n + c] = -s / L[i * n + i];
    }
  }
  Ainv.assign((size_t)n * n, 0.0);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t j = 0; j < n; ++j) {
      double s = 0;
      for (int64_t k = std::max(i, j); k < n; ++k) s += Li[k * n + i] * Li[k * n + j];
      Ainv[i * n + j] = s;
    }
  return EXFEM_OK;
}

}  // namespace exfem
