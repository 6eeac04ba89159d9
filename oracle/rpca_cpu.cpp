// Multithreaded FP64 C++ restatement of scx's CPU randomized PCA -- TEST AND
// BASELINE INFRASTRUCTURE ONLY.  It is the timed CPU baseline (the reference
// itself is Rust and cannot be built in this environment) and a second
// checker; the product never links it.
//
// Follows scx-accel/src/pca/cpu.rs:
//   randomized_pca_inmemory      :887-952  (loop order, QR of Z only if q > 2)
//   col_sums_and_sum_sq          scx-sparse/src/csr.rs:570-580
//   spmm_forward_into / _row     :1471-1523 (row-parallel, mean correction mc)
//   spmm_transpose_into / block  :1282-1389 (output-partitioned gene blocks,
//                                            each block scans every row's
//                                            sorted sub-range; colblocks.rs)
//   apply_transpose_mean_correction :1253-1267
//   build_pca_result             :1530-1585
// faer's Householder QR (cpu.rs:118-122) is stood in for by FP64 CholeskyQR2
// (same Q up to column signs for a well-conditioned Y) and faer's thin SVD of
// B by an FP64 Jacobi eigendecomposition of B^T B.  Parallelism is std::thread.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <thread>
#include <vector>

namespace {

int g_threads = 1;

void parallel_for(int64_t n, const std::function<void(int64_t, int64_t, int)>& f) {
  int t = (int)std::max<int64_t>(1, std::min<int64_t>(g_threads, n));
  if (t == 1) {
    f(0, n, 0);
    return;
  }
  std::vector<std::thread> ths;
  int64_t per = (n + t - 1) / t;
  for (int i = 0; i < t; ++i) {
    int64_t a = i * per, b = std::min(n, a + per);
    if (a >= b) break;
    ths.emplace_back(f, a, b, i);
  }
  for (auto& th : ths) th.join();
}

struct Csr {
  int64_t n, g;
  const int64_t* indptr;
  const int32_t* idx;
  std::vector<double> val;
};

// Y = (X - mu) M, M row-major g x k
void spmm_forward(const Csr& x, const std::vector<double>& m, int64_t k, const double* mu,
                  std::vector<double>& y) {
  std::vector<double> mc(k, 0.0);
  if (mu)
    for (int64_t v = 0; v < x.g; ++v)
      for (int64_t j = 0; j < k; ++j) mc[j] += mu[v] * m[v * k + j];
  y.assign(x.n * k, 0.0);
  parallel_for(x.n, [&](int64_t a, int64_t b, int) {
    for (int64_t r = a; r < b; ++r) {
      double* yr = &y[r * k];
      for (int64_t p = x.indptr[r]; p < x.indptr[r + 1]; ++p) {
        const double v = x.val[p];
        const double* mr = &m[(int64_t)x.idx[p] * k];
        for (int64_t j = 0; j < k; ++j) yr[j] += v * mr[j];
      }
      if (mu)
        for (int64_t j = 0; j < k; ++j) yr[j] -= mc[j];
    }
  });
}

// Z = (X - mu)^T Q, Q row-major n x k; gene blocks own disjoint output rows.
void spmm_transpose(const Csr& x, const std::vector<double>& q, int64_t k, const double* mu,
                    std::vector<double>& z) {
  z.assign(x.g * k, 0.0);
  int nblocks = std::max(1, g_threads * 2);
  int64_t gb = (x.g + nblocks - 1) / nblocks;
  std::atomic<int> next{0};
  parallel_for(g_threads, [&](int64_t, int64_t, int) {
    for (int b; (b = next.fetch_add(1)) < nblocks;) {
      const int32_t lo = (int32_t)(b * gb), hi = (int32_t)std::min<int64_t>(x.g, (b + 1) * gb);
      if (lo >= hi) continue;
      for (int64_t r = 0; r < x.n; ++r) {
        const int32_t* s = x.idx + x.indptr[r];
        const int32_t* e = x.idx + x.indptr[r + 1];
        const int32_t* p0 = std::lower_bound(s, e, lo);
        const double* qr = &q[r * k];
        for (const int32_t* p = p0; p < e && *p < hi; ++p) {
          const double v = x.val[p - x.idx];
          double* zr = &z[(int64_t)(*p) * k];
          for (int64_t j = 0; j < k; ++j) zr[j] += v * qr[j];
        }
      }
    }
  });
  if (mu) {
    std::vector<double> sq(k, 0.0);
    for (int64_t r = 0; r < x.n; ++r)
      for (int64_t j = 0; j < k; ++j) sq[j] += q[r * k + j];
    for (int64_t v = 0; v < x.g; ++v)
      for (int64_t j = 0; j < k; ++j) z[v * k + j] -= mu[v] * sq[j];
  }
}

// FP64 Gram A^T A of a row-major m x k matrix (thread-partial, then summed).
std::vector<double> gram(const std::vector<double>& a, int64_t m, int64_t k) {
  std::vector<std::vector<double>> part(g_threads, std::vector<double>(k * k, 0.0));
  parallel_for(m, [&](int64_t s, int64_t e, int t) {
    std::vector<double>& g = part[t];
    for (int64_t r = s; r < e; ++r) {
      const double* ar = &a[r * k];
      for (int64_t i = 0; i < k; ++i) {
        const double ai = ar[i];
        double* gi = &g[i * k];
        for (int64_t j = i; j < k; ++j) gi[j] += ai * ar[j];
      }
    }
  });
  std::vector<double> g(k * k, 0.0);
  for (auto& p : part)
    for (int64_t i = 0; i < k * k; ++i) g[i] += p[i];
  for (int64_t i = 0; i < k; ++i)
    for (int64_t j = 0; j < i; ++j) g[i * k + j] = g[j * k + i];
  return g;
}

// In-place CholeskyQR2 of a row-major m x k matrix; returns false on breakdown.
bool cholqr2(std::vector<double>& a, int64_t m, int64_t k) {
  for (int pass = 0; pass < 2; ++pass) {
    std::vector<double> g = gram(a, m, k);
    std::vector<double> r(k * k, 0.0);
    for (int64_t j = 0; j < k; ++j) {
      double d = g[j * k + j];
      for (int64_t l = 0; l < j; ++l) d -= r[l * k + j] * r[l * k + j];
      if (!(d > 0.0)) return false;
      r[j * k + j] = std::sqrt(d);
      for (int64_t c = j + 1; c < k; ++c) {
        double v = g[j * k + c];
        for (int64_t l = 0; l < j; ++l) v -= r[l * k + j] * r[l * k + c];
        r[j * k + c] = v / r[j * k + j];
      }
    }
    // R^{-1} (upper)
    std::vector<double> ri(k * k, 0.0);
    for (int64_t c = 0; c < k; ++c)
      for (int64_t i = c; i >= 0; --i) {
        double v = (i == c) ? 1.0 : 0.0;
        for (int64_t l = i + 1; l <= c; ++l) v -= r[i * k + l] * ri[l * k + c];
        ri[i * k + c] = v / r[i * k + i];
      }
    parallel_for(m, [&](int64_t s, int64_t e, int) {
      std::vector<double> tmp(k);
      for (int64_t row = s; row < e; ++row) {
        double* ar = &a[row * k];
        for (int64_t c = 0; c < k; ++c) {
          double v = 0.0;
          for (int64_t l = 0; l <= c; ++l) v += ar[l] * ri[l * k + c];
          tmp[c] = v;
        }
        memcpy(ar, tmp.data(), sizeof(double) * k);
      }
    });
  }
  return true;
}

// Cyclic Jacobi eigendecomposition of a symmetric k x k matrix (row-major).
void jacobi(std::vector<double> a, int64_t k, std::vector<double>& evals, std::vector<double>& evecs) {
  evecs.assign(k * k, 0.0);
  for (int64_t i = 0; i < k; ++i) evecs[i * k + i] = 1.0;
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int64_t i = 0; i < k; ++i)
      for (int64_t j = 0; j < k; ++j) {
        tot += a[i * k + j] * a[i * k + j];
        if (i != j) off += a[i * k + j] * a[i * k + j];
      }
    if (off <= 1e-30 * tot) break;
    for (int64_t p = 0; p < k - 1; ++p)
      for (int64_t q = p + 1; q < k; ++q) {
        double apq = a[p * k + q];
        if (std::fabs(apq) < 1e-300) continue;
        double theta = (a[q * k + q] - a[p * k + p]) / (2.0 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int64_t r = 0; r < k; ++r) {
          double xp = a[r * k + p], xq = a[r * k + q];
          a[r * k + p] = c * xp - s * xq;
          a[r * k + q] = s * xp + c * xq;
        }
        for (int64_t r = 0; r < k; ++r) {
          double xp = a[p * k + r], xq = a[q * k + r];
          a[p * k + r] = c * xp - s * xq;
          a[q * k + r] = s * xp + c * xq;
        }
        for (int64_t r = 0; r < k; ++r) {
          double xp = evecs[r * k + p], xq = evecs[r * k + q];
          evecs[r * k + p] = c * xp - s * xq;
          evecs[r * k + q] = s * xp + c * xq;
        }
      }
  }
  std::vector<int64_t> order(k);
  for (int64_t i = 0; i < k; ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](int64_t x, int64_t y) { return a[x * k + x] > a[y * k + y]; });
  std::vector<double> ev(k * k);
  evals.resize(k);
  for (int64_t c = 0; c < k; ++c) {
    evals[c] = a[order[c] * k + order[c]];
    for (int64_t r = 0; r < k; ++r) ev[r * k + c] = evecs[r * k + order[c]];
  }
  evecs = ev;
}

}  // namespace

extern "C" {

// Returns 0 on success, 1 on bad input, 2 on a QR breakdown.
// omega: n_vars x k row-major FP64.  Outputs may be null except sigma.
int rpca_cpu_run(int64_t n, int64_t g, const int64_t* indptr, const int32_t* idx, const float* val,
                 int64_t nc, int64_t k, int64_t q, int center, int scale, double clip,
                 const double* omega, int threads, double* sigma, double* comps, float* emb,
                 double* total_var) {
  if (n <= 0 || g <= 0 || nc <= 0 || k < nc || !omega || !sigma) return 1;
  g_threads = std::max(1, threads);
  const int64_t nnz = indptr[n];
  Csr x{n, g, indptr, idx, std::vector<double>(nnz)};
  for (int64_t p = 0; p < nnz; ++p) x.val[p] = val[p];
  auto col_stats = [&](std::vector<double>& s, std::vector<double>& ss) {
    std::vector<std::vector<double>> ps(g_threads, std::vector<double>(2 * g, 0.0));
    parallel_for(nnz, [&](int64_t a, int64_t b, int t) {
      double* acc = ps[t].data();
      for (int64_t p = a; p < b; ++p) {
        acc[x.idx[p]] += x.val[p];
        acc[g + x.idx[p]] += x.val[p] * x.val[p];
      }
    });
    s.assign(g, 0.0);
    ss.assign(g, 0.0);
    for (auto& pp : ps)
      for (int64_t j = 0; j < g; ++j) {
        s[j] += pp[j];
        ss[j] += pp[g + j];
      }
  };
  std::vector<double> s, ss;
  col_stats(s, ss);
  if (scale) {
    std::vector<double> mu(g), is(g), cs(g, 0.0);
    for (int64_t j = 0; j < g; ++j) {
      mu[j] = s[j] / n;
      double var = (ss[j] - n * mu[j] * mu[j]) / std::max<double>(n - 1.0, 1.0);
      double sd = std::sqrt(std::max(var, 0.0));
      if (sd == 0.0) sd = 1.0;
      is[j] = 1.0 / sd;
      if (center) {
        double c = -mu[j] * is[j];
        if (clip > 0) c = std::min(std::max(c, -clip), clip);
        cs[j] = c;
      }
    }
    parallel_for(nnz, [&](int64_t a, int64_t b, int) {
      for (int64_t p = a; p < b; ++p) {
        const int32_t j = x.idx[p];
        double v;
        if (center) {
          v = (x.val[p] - mu[j]) * is[j];
          if (clip > 0) v = std::min(std::max(v, -clip), clip);
          v -= cs[j];
        } else {
          v = x.val[p] * is[j];
          if (clip > 0) v = std::min(v, clip);
        }
        x.val[p] = v;
      }
    });
    col_stats(s, ss);
  }
  std::vector<double> mu(g, 0.0);
  for (int64_t j = 0; j < g; ++j) mu[j] = s[j] / n;
  const double* mup = center ? mu.data() : nullptr;

  std::vector<double> om(omega, omega + g * k), y, z;
  spmm_forward(x, om, k, mup, y);
  if (!cholqr2(y, n, k)) return 2;
  for (int64_t it = 0; it < q; ++it) {
    spmm_transpose(x, y, k, mup, z);
    if (q > 2 && !cholqr2(z, g, k)) return 2;
    spmm_forward(x, z, k, mup, y);
    if (!cholqr2(y, n, k)) return 2;
  }
  spmm_transpose(x, y, k, mup, z);  // B = (X - mu)^T Q, g x k
  std::vector<double> bt = gram(z, g, k), ev, E;
  jacobi(bt, k, ev, E);
  for (int64_t c = 0; c < nc; ++c) sigma[c] = std::sqrt(std::max(ev[c], 0.0));
  if (comps)
    for (int64_t c = 0; c < nc; ++c)
      for (int64_t j = 0; j < g; ++j) {
        double v = 0.0;
        for (int64_t l = 0; l < k; ++l) v += z[j * k + l] * E[l * k + c];
        comps[c * g + j] = sigma[c] > 0 ? v / sigma[c] : 0.0;
      }
  if (emb)
    parallel_for(n, [&](int64_t a, int64_t b, int) {
      for (int64_t r = a; r < b; ++r)
        for (int64_t c = 0; c < nc; ++c) {
          double v = 0.0;
          for (int64_t l = 0; l < k; ++l) v += y[r * k + l] * E[l * k + c];
          emb[r * nc + c] = (float)(v * sigma[c]);
        }
    });
  if (total_var) {
    double t = 0.0;
    for (int64_t j = 0; j < g; ++j) t += center ? ss[j] - n * mu[j] * mu[j] : ss[j];
    *total_var = t / std::max<double>(n - 1.0, 1.0);
  }
  return 0;
}

}  // extern "C"
