// Support code linked into the GCC build of the reference CPU solver (test
// infrastructure: it lets the reference's own fem_solve run here to produce
// parity fixtures; nothing of it is part of the product).
//
// pardiso_64: the calling convention of MKL PARDISO as the reference uses it
// (solver/MG/Elasticity_Matrix.cpp:169-289): real symmetric positive definite
// matrices (mtype 2) given as the upper triangle in 0-based CSR (iparm[34] = 1,
// Build_CSR_Matrix :16-164), double precision, phases 11 (analysis), 22
// (factorization), 33 (solve, one right-hand side) and -1 (release).  The solve
// is exact: a band Cholesky factorization after a reverse Cuthill-McKee
// ordering.  A pivot that is not positive returns error -4, PARDISO's "zero
// pivot" code, which the reference turns into an exception.
//
// ref_free: releases an output blob of the reference's fem_solve (allocated
// with new char[], topo_opt/fem_interface.h:438-441) from a caller that cannot
// call delete[].
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <queue>
#include <vector>

namespace {

struct BandFactor {
  long long n = 0, bw = 0;
  std::vector<long long> perm;   // new index -> old index
  std::vector<long long> iperm;  // old index -> new index
  std::vector<double> L;         // row i holds L(i, i - bw .. i) at [i * (bw + 1) + (j - i + bw)]
  double& at(long long i, long long j) { return L[size_t(i) * size_t(bw + 1) + size_t(j - i + bw)]; }
};

// reverse Cuthill-McKee ordering of the symmetric pattern given by its upper triangle
void rcm(long long n, const long long* ia, const long long* ja, std::vector<long long>& perm) {
  std::vector<std::vector<long long>> adj(static_cast<size_t>(n));
  for (long long i = 0; i < n; ++i)
    for (long long p = ia[i]; p < ia[i + 1]; ++p) {
      const long long j = ja[p];
      if (j == i) continue;
      adj[size_t(i)].push_back(j);
      adj[size_t(j)].push_back(i);
    }
  std::vector<long long> deg(static_cast<size_t>(n));
  for (long long i = 0; i < n; ++i) {
    auto& a = adj[size_t(i)];
    std::sort(a.begin(), a.end());
    a.erase(std::unique(a.begin(), a.end()), a.end());
    deg[size_t(i)] = static_cast<long long>(a.size());
  }
  for (auto& a : adj) std::sort(a.begin(), a.end(), [&](long long x, long long y) { return deg[size_t(x)] < deg[size_t(y)]; });
  std::vector<char> seen(static_cast<size_t>(n), 0);
  perm.clear();
  std::vector<long long> order(static_cast<size_t>(n));
  for (long long i = 0; i < n; ++i) order[size_t(i)] = i;
  std::stable_sort(order.begin(), order.end(), [&](long long x, long long y) { return deg[size_t(x)] < deg[size_t(y)]; });
  for (long long s : order) {
    if (seen[size_t(s)]) continue;
    std::queue<long long> q;
    q.push(s);
    seen[size_t(s)] = 1;
    while (!q.empty()) {
      const long long v = q.front();
      q.pop();
      perm.push_back(v);
      for (long long w : adj[size_t(v)])
        if (!seen[size_t(w)]) {
          seen[size_t(w)] = 1;
          q.push(w);
        }
    }
  }
  std::reverse(perm.begin(), perm.end());
}

}  // namespace

extern "C" void pardiso_64(void* pt, const long long* maxfct, const long long* mnum, const long long* mtype,
                           const long long* phase, const long long* n, const void* a, const long long* ia,
                           const long long* ja, long long* perm, const long long* nrhs, long long* iparm,
                           const long long* msglvl, void* b, void* x, long long* error) {
  (void)maxfct; (void)mnum; (void)perm; (void)msglvl;
  void** handle = static_cast<void**>(pt);
  *error = 0;
  if (*phase == -1) {
    delete static_cast<BandFactor*>(handle[0]);
    handle[0] = nullptr;
    return;
  }
  if (*mtype != 2 || iparm[34] != 1 || iparm[27] != 0 || *nrhs != 1) {
    *error = -1;  // input inconsistent: only what the reference asks for is supported
    return;
  }
  const double* av = static_cast<const double*>(a);
  if (*phase == 11) {
    delete static_cast<BandFactor*>(handle[0]);
    BandFactor* f = new BandFactor();
    handle[0] = f;
    f->n = *n;
    rcm(f->n, ia, ja, f->perm);
    f->iperm.assign(size_t(f->n), 0);
    for (long long i = 0; i < f->n; ++i) f->iperm[size_t(f->perm[size_t(i)])] = i;
    long long bw = 0;
    for (long long i = 0; i < f->n; ++i)
      for (long long p = ia[i]; p < ia[i + 1]; ++p)
        bw = std::max(bw, std::llabs(f->iperm[size_t(i)] - f->iperm[size_t(ja[p])]));
    f->bw = bw;
    iparm[17] = f->n * (bw + 1);  // nonzeros of the factor
    return;
  }
  BandFactor* f = static_cast<BandFactor*>(handle[0]);
  if (!f || f->n != *n) {
    *error = -1;
    return;
  }
  const long long N = f->n, W = f->bw;
  if (*phase == 22) {
    f->L.assign(size_t(N) * size_t(W + 1), 0.0);
    for (long long i = 0; i < N; ++i)
      for (long long p = ia[i]; p < ia[i + 1]; ++p) {
        long long r = f->iperm[size_t(i)], c = f->iperm[size_t(ja[p])];
        if (r < c) std::swap(r, c);
        f->at(r, c) += av[p];
      }
    // row-oriented band Cholesky: L(i, j) for j = i - W .. i
    for (long long i = 0; i < N; ++i) {
      const long long j0 = std::max(0LL, i - W);
      for (long long j = j0; j <= i; ++j) {
        const long long k0 = std::max(j0, j - W);
        double s = f->at(i, j);
        const double* li = &f->at(i, k0);
        const double* lj = &f->at(j, k0);
        for (long long k = 0; k < j - k0; ++k) s -= li[k] * lj[k];
        if (j == i) {
          if (!(s > 0)) {
            *error = -4;
            return;
          }
          f->at(i, i) = std::sqrt(s);
        } else {
          f->at(i, j) = s / f->at(j, j);
        }
      }
    }
    return;
  }
  if (*phase == 33) {
    const double* bv = static_cast<const double*>(b);
    double* xv = static_cast<double*>(x);
    std::vector<double> y(static_cast<size_t>(N));
    for (long long i = 0; i < N; ++i) {
      double s = bv[f->perm[size_t(i)]];
      const long long j0 = std::max(0LL, i - W);
      for (long long j = j0; j < i; ++j) s -= f->at(i, j) * y[size_t(j)];
      y[size_t(i)] = s / f->at(i, i);
    }
    for (long long i = N - 1; i >= 0; --i) {
      y[size_t(i)] /= f->at(i, i);
      const double yi = y[size_t(i)];
      const long long j0 = std::max(0LL, i - W);
      for (long long j = j0; j < i; ++j) y[size_t(j)] -= f->at(i, j) * yi;
    }
    for (long long i = 0; i < N; ++i) xv[f->perm[size_t(i)]] = y[size_t(i)];
    return;
  }
  *error = -1;
}

extern "C" void ref_free(void* blob) { delete[] static_cast<char*>(blob); }
