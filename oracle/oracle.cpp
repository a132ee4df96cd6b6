// ORACLE -- test infrastructure only.  A CPU restatement of the reference's
// hot path (carolc0708/graph-bit-ops) used by tests/ as the parity checker and
// by bench.py's CPU-baseline legs.  Product code never links or calls it.
//
// Each function cites the reference code whose math it restates.  The tile
// layout follows cuSPARSE csr2bsr DIRECTION_ROW (block columns ascending per
// block row, row-major dense tile) followed by ToBit*Col
// (algorithm/bsrbmv.cu:31-235): word r = tile row r, column c at bit b-1-c;
// the COL layout (bsrbmm/csr2bsr_batch.cu:1208) has word c = tile column c.
// Tile words are handed to Python as one uint64 per word.
#include <omp.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <parallel/algorithm>
#include <numeric>
#include <queue>
#include <unordered_set>
#include <vector>

extern "C" {

static const uint32_t INF = 2147483647u;  // algorithm/sssp.cu:140

// --------------------------------------------------------------- packing
// csr2bsr_batch_* (algorithm/csr2bsr_batch_bsrbmv.cu:9-946): tiles of a block
// row = distinct col/b over its b CSR rows, ascending.
long long orc_pack_count(const int* rowptr, const int* colind, int nrows, int b, int* bsr_rowptr) {
  const int nbr = (nrows + b - 1) / b;
  std::vector<int> cnt((size_t)nbr, 0);
#pragma omp parallel for schedule(dynamic, 64)
  for (int R = 0; R < nbr; ++R) {
    std::vector<int> cols;
    for (int r = R * b; r < std::min(nrows, (R + 1) * b); ++r)
      for (int k = rowptr[r]; k < rowptr[r + 1]; ++k) cols.push_back(colind[k] / b);
    std::sort(cols.begin(), cols.end());
    cnt[(size_t)R] = (int)(std::unique(cols.begin(), cols.end()) - cols.begin());
  }
  long long tot = 0;
  bsr_rowptr[0] = 0;
  for (int R = 0; R < nbr; ++R) {
    tot += cnt[(size_t)R];
    bsr_rowptr[R + 1] = (int)tot;
  }
  return tot;
}

void orc_pack_fill(const int* rowptr, const int* colind, int nrows, int b, int layout,
                   const int* bsr_rowptr, int* bsr_colind, uint64_t* words) {
  const int nbr = (nrows + b - 1) / b;
#pragma omp parallel for schedule(dynamic, 64)
  for (int R = 0; R < nbr; ++R) {
    std::vector<int> cols;
    for (int r = R * b; r < std::min(nrows, (R + 1) * b); ++r)
      for (int k = rowptr[r]; k < rowptr[r + 1]; ++k) cols.push_back(colind[k] / b);
    std::sort(cols.begin(), cols.end());
    cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
    const long long base = bsr_rowptr[R];
    for (size_t t = 0; t < cols.size(); ++t) bsr_colind[base + (long long)t] = cols[t];
    memset(words + base * b, 0, sizeof(uint64_t) * (size_t)b * cols.size());
    for (int r = R * b; r < std::min(nrows, (R + 1) * b); ++r)
      for (int k = rowptr[r]; k < rowptr[r + 1]; ++k) {
        const int C = colind[k] / b, c = colind[k] % b, rr = r - R * b;
        const long long t = base + (std::lower_bound(cols.begin(), cols.end(), C) - cols.begin());
        if (layout == 0)
          words[t * b + rr] |= 1ull << (b - 1 - c);  // row word rr, column c at bit b-1-c
        else
          words[t * b + c] |= 1ull << (b - 1 - rr);  // column word c, row rr at bit b-1-rr
      }
  }
}

// ToBit*Row (algorithm/bsrbmv.cu:62-255): element R*b+r -> bit b-1-r of word R.
void orc_pack_vector(const int32_t* x, int n, int b, uint64_t* words) {
  const int nw = (n + b - 1) / b;
  for (int R = 0; R < nw; ++R) {
    uint64_t w = 0;
    for (int r = 0; r < b; ++r) {
      const long long i = (long long)R * b + r;
      if (i < n && x[i] > 0) w |= 1ull << (b - 1 - r);
    }
    words[R] = w;
  }
}

static inline int popc64(uint64_t v) { return __builtin_popcountll(v); }

// bmv{4,8,16,32,64}_sparse (algorithm/bsrbmv.cu:262-474): y[R*b+r] =
// sum over tiles of popc(A_tile[r] & x[colind]).
void orc_bmv_count(const int* brp, const int* bci, const uint64_t* w, int nbr, int b, int nrows,
                   const uint64_t* x, int32_t* y) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int R = 0; R < nbr; ++R)
    for (int r = 0; r < b; ++r) {
      const long long i = (long long)R * b + r;
      if (i >= nrows) break;
      int s = 0;
      for (int t = brp[R]; t < brp[R + 1]; ++t) s += popc64(w[(long long)t * b + r] & x[bci[t]]);
      y[i] = s;
    }
}

// bmv32_sparse_bin_masked_v4 (algorithm/bsrbmv.cu:740-783):
// out[R] = brev(ballot(count > 0)) & ~mask[R].
void orc_bmv_masked(const int* brp, const int* bci, const uint64_t* w, int nbr, int b,
                    const uint64_t* x, const uint64_t* mask, uint64_t* out) {
  const uint64_t full = b == 64 ? ~0ull : ((1ull << b) - 1);
#pragma omp parallel for schedule(dynamic, 64)
  for (int R = 0; R < nbr; ++R) {
    uint64_t o = 0;
    for (int r = 0; r < b; ++r) {
      bool any = false;
      for (int t = brp[R]; t < brp[R + 1] && !any; ++t) any = (w[(long long)t * b + r] & x[bci[t]]) != 0;
      if (any) o |= 1ull << (b - 1 - r);
    }
    out[R] = o & ~(mask ? mask[R] : 0ull) & full;
  }
}

// Min-plus over (P + I) (bmv32_sparse_full_minplus, algorithm/bsrbmv.cu:
// 1083-1138, with the diagonal term always present).
void orc_bmv_minplus(const int* brp, const int* bci, const uint64_t* w, int nbr, int b, int nrows,
                     const uint32_t* x, uint32_t* y) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int R = 0; R < nbr; ++R)
    for (int r = 0; r < b; ++r) {
      const long long i = (long long)R * b + r;
      if (i >= nrows) break;
      uint32_t m = x[i];
      for (int t = brp[R]; t < brp[R + 1]; ++t) {
        const uint64_t word = w[(long long)t * b + r];
        for (int c = 0; c < b; ++c)
          if ((word >> (b - 1 - c)) & 1) {
            const uint32_t d = x[(long long)bci[t] * b + c];
            m = std::min(m, d >= INF ? INF : d + 1);
          }
      }
      y[i] = m;
    }
}

// bmv32_sparse_full (algorithm/bsrbmv.cu:1239-1286) generalised:
// y[i] = alpha * sum_j x[j] * scale[j] + add, accumulated in fp32 in the
// reference's order (tiles ascending, columns ascending).
void orc_bmv_float(const int* brp, const int* bci, const uint64_t* w, int nbr, int b, int nrows,
                   const float* x, const float* scale, float alpha, float add, float* y) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int R = 0; R < nbr; ++R)
    for (int r = 0; r < b; ++r) {
      const long long i = (long long)R * b + r;
      if (i >= nrows) break;
      float s = 0.f;
      for (int t = brp[R]; t < brp[R + 1]; ++t) {
        const uint64_t word = w[(long long)t * b + r];
        for (int c = 0; c < b; ++c)
          if ((word >> (b - 1 - c)) & 1) {
            const long long j = (long long)bci[t] * b + c;
            s += x[j] * (scale ? scale[j] : 1.f);
          }
      }
      y[i] = alpha * s + add;
    }
}

// bmv32_sparse_full_cc (algorithm/bsrbmv.cu:1933-1975): min over set bits.
void orc_bmv_minselect(const int* brp, const int* bci, const uint64_t* w, int nbr, int b, int nrows,
                       const int32_t* x, int32_t* y) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int R = 0; R < nbr; ++R)
    for (int r = 0; r < b; ++r) {
      const long long i = (long long)R * b + r;
      if (i >= nrows) break;
      int32_t m = (int32_t)INF;
      for (int t = brp[R]; t < brp[R + 1]; ++t) {
        const uint64_t word = w[(long long)t * b + r];
        for (int c = 0; c < b; ++c)
          if ((word >> (b - 1 - c)) & 1) m = std::min(m, x[(long long)bci[t] * b + c]);
      }
      y[i] = m;
    }
}

// ------------------------------------------------------------ algorithms
// BFS restating algorithm/bfs.cu:508-564 on B2SR (pull, masked BMV per
// level, stop when the new frontier is empty), emitting levels.  This is
// also the CPU baseline timed by bench.py (OpenMP over block rows).
int orc_bfs_b2sr(const int* brp, const int* bci, const uint64_t* w, int nbr, int b, int nrows,
                 int src, int32_t* level) {
  std::vector<uint64_t> f1((size_t)nbr, 0), f2((size_t)nbr, 0), vis((size_t)nbr, 0);
  for (int i = 0; i < nrows; ++i) level[i] = -1;
  level[src] = 0;
  f1[(size_t)(src / b)] = 1ull << (b - 1 - src % b);
  vis[(size_t)(src / b)] = f1[(size_t)(src / b)];
  int depth = 1;
  for (int L = 0;; ++L) {
    long long succ = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : succ)
    for (int R = 0; R < nbr; ++R) {
      uint64_t o = 0;
      for (int r = 0; r < b; ++r) {
        if ((vis[(size_t)R] >> (b - 1 - r)) & 1) continue;
        for (int t = brp[R]; t < brp[R + 1]; ++t)
          if (w[(long long)t * b + r] & f1[(size_t)bci[t]]) {
            o |= 1ull << (b - 1 - r);
            break;
          }
      }
      f2[(size_t)R] = o;
      if (o) {
        vis[(size_t)R] |= o;
        for (int r = 0; r < b; ++r)
          if ((o >> (b - 1 - r)) & 1) level[(long long)R * b + r] = L + 1;
        succ += popc64(o);
      }
    }
    f1.swap(f2);
    if (succ == 0) break;
    depth = L + 2;
  }
  return depth;
}

// Independent check: queue BFS on the CSR of P (edges j -> i for P[i][j]).
int orc_bfs_csr(const int* rowptr, const int* colind, int n, int src, int32_t* level) {
  // out-adjacency = transpose of P
  std::vector<int> tp((size_t)n + 1, 0), tc((size_t)rowptr[n]);
  for (int k = 0; k < rowptr[n]; ++k) tp[(size_t)colind[k] + 1]++;
  for (int i = 0; i < n; ++i) tp[(size_t)i + 1] += tp[(size_t)i];
  std::vector<int> pos(tp.begin(), tp.end() - 1);
  for (int i = 0; i < n; ++i)
    for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) tc[(size_t)pos[(size_t)colind[k]]++] = i;
  for (int i = 0; i < n; ++i) level[i] = -1;
  std::queue<int> q;
  level[src] = 0;
  q.push(src);
  int depth = 1;
  while (!q.empty()) {
    int u = q.front();
    q.pop();
    for (int k = tp[(size_t)u]; k < tp[(size_t)u + 1]; ++k) {
      int v = tc[(size_t)k];
      if (level[v] < 0) {
        level[v] = level[u] + 1;
        depth = std::max(depth, level[v] + 1);
        q.push(v);
      }
    }
  }
  return depth;
}

// SSSP with unit weights restating algorithm/sssp.cu:420-470: repeated
// min-plus BMV from the improved frontier until nothing improves.
int orc_sssp_b2sr(const int* brp, const int* bci, const uint64_t* w, int nbr, int b, int nrows,
                  int src, uint32_t* dist) {
  std::vector<uint32_t> f1((size_t)nbr * b, INF), f2((size_t)nbr * b, INF);
  for (int i = 0; i < nrows; ++i) dist[i] = INF;
  dist[src] = 0;
  f1[(size_t)src] = 0;
  int iters = 0;
  while (true) {
    ++iters;
    long long succ = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : succ)
    for (int R = 0; R < nbr; ++R)
      for (int r = 0; r < b; ++r) {
        const long long i = (long long)R * b + r;
        uint32_t m = INF;
        if (i < nrows)
          for (int t = brp[R]; t < brp[R + 1]; ++t) {
            const uint64_t word = w[(long long)t * b + r];
            if (!word) continue;
            for (int c = 0; c < b; ++c)
              if ((word >> (b - 1 - c)) & 1) {
                const uint32_t d = f1[(size_t)bci[t] * b + c];
                if (d < INF) m = std::min(m, d + 1);
              }
          }
        if (i < nrows && m < dist[i]) {
          dist[i] = m;
          f2[(size_t)i] = m;
          ++succ;
        } else {
          f2[(size_t)i] = INF;
        }
      }
    f1.swap(f2);
    if (succ == 0) break;
  }
  return iters;
}

// PageRank restating algorithm/pr.cu:449-513 in fp32 (reference term order:
// alpha*p[j]/outdeg[j] summed over tiles and columns ascending) -- returns
// iterations; p has nrows entries.
int orc_pr_b2sr_f32(const int* brp, const int* bci, const uint64_t* w, int nbr, int b, int nrows,
                    const int* outdeg, float alpha, int max_iter, float tol, float* p) {
  std::vector<float> prev((size_t)nrows);
  for (int i = 0; i < nrows; ++i) p[i] = 1.0f / (float)nrows;
  int it = 0;
  float err = 1.0f;
  while (it < max_iter && !(tol >= 0 && err <= tol)) {
    std::copy(p, p + nrows, prev.begin());
    double e2 = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : e2)
    for (int R = 0; R < nbr; ++R)
      for (int r = 0; r < b; ++r) {
        const long long i = (long long)R * b + r;
        if (i >= nrows) break;
        float s = 0.f;
        for (int t = brp[R]; t < brp[R + 1]; ++t) {
          const uint64_t word = w[(long long)t * b + r];
          for (int c = 0; c < b; ++c)
            if ((word >> (b - 1 - c)) & 1) {
              const long long j = (long long)bci[t] * b + c;
              s += alpha * prev[(size_t)j] / (float)outdeg[j];
            }
        }
        p[i] = s + (1.0f - alpha) / (float)nrows;
        const double d = (double)p[i] - (double)prev[(size_t)i];
        e2 += d * d;
      }
    err = (float)std::sqrt(e2);
    ++it;
  }
  return it;
}

// The same recurrence in fp64 on the CSR of P (the PageRank oracle).
int orc_pr_csr_f64(const int* rowptr, const int* colind, int n, const int* outdeg, double alpha,
                   int max_iter, double tol, double* p) {
  std::vector<double> prev((size_t)n);
  for (int i = 0; i < n; ++i) p[i] = 1.0 / n;
  int it = 0;
  double err = 1.0;
  while (it < max_iter && !(tol >= 0 && err <= tol)) {
    std::copy(p, p + n, prev.begin());
    double e2 = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : e2)
    for (int i = 0; i < n; ++i) {
      double s = 0;
      for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) s += prev[(size_t)colind[k]] / outdeg[colind[k]];
      p[i] = alpha * s + (1.0 - alpha) / n;
      e2 += (p[i] - prev[(size_t)i]) * (p[i] - prev[(size_t)i]);
    }
    err = std::sqrt(e2);
    ++it;
  }
  return it;
}

// Personalized PageRank p = alpha P D^-1 p + (1-alpha) v in fp64 until the
// L1 change <= tol (or max_iter), starting from (1-alpha) v.
int orc_ppr_f64(const int* rowptr, const int* colind, int n, const int* outdeg, const double* v,
                double alpha, double tol, int max_iter, double* p) {
  std::vector<double> prev((size_t)n);
  for (int i = 0; i < n; ++i) p[i] = (1 - alpha) * v[i];
  int it = 0;
  while (it < max_iter) {
    std::copy(p, p + n, prev.begin());
    double e1 = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : e1)
    for (int i = 0; i < n; ++i) {
      double s = 0;
      for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) s += prev[(size_t)colind[k]] / outdeg[colind[k]];
      p[i] = alpha * s + (1 - alpha) * v[i];
      e1 += std::fabs(p[i] - prev[(size_t)i]);
    }
    ++it;
    if (tol >= 0 && e1 <= tol) break;
  }
  return it;
}

// Adjoint of the PPR solve for L = dot(w, p): grad_v = (1-alpha) u with
// u = alpha D^-1 P^T u + w, fp64, iterated until the L1 change <= tol.
int orc_ppr_adjoint_f64(const int* rowptr, const int* colind, int n, const int* outdeg,
                        const double* wv, double alpha, double tol, int max_iter, double* grad) {
  std::vector<double> u(wv, wv + n), un((size_t)n);
  int it = 0;
  while (it < max_iter) {
    std::fill(un.begin(), un.end(), 0.0);
    for (int i = 0; i < n; ++i)
      for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) un[(size_t)colind[k]] += u[(size_t)i];
    double e1 = 0;
    for (int j = 0; j < n; ++j) {
      const double nv = wv[j] + (outdeg[j] > 0 ? alpha * un[(size_t)j] / outdeg[j] : 0.0);
      e1 += std::fabs(nv - u[(size_t)j]);
      un[(size_t)j] = nv;
    }
    u.swap(un);
    ++it;
    if (tol >= 0 && e1 <= tol) break;
  }
  for (int j = 0; j < n; ++j) grad[j] = (1 - alpha) * u[(size_t)j];
  return it;
}

// Connected components: label = smallest vertex id of the component (the
// fixed point of algorithm/cc.cu's FastSV loop), by union-find.
void orc_cc(const int* rowptr, const int* colind, int n, int32_t* label) {
  std::vector<int> par((size_t)n);
  std::iota(par.begin(), par.end(), 0);
  auto find = [&](int x) {
    while (par[(size_t)x] != x) {
      par[(size_t)x] = par[(size_t)par[(size_t)x]];
      x = par[(size_t)x];
    }
    return x;
  };
  for (int i = 0; i < n; ++i)
    for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
      int a = find(i), c = find(colind[k]);
      if (a != c) par[(size_t)std::max(a, c)] = std::min(a, c);
    }
  for (int i = 0; i < n; ++i) label[i] = find(i);
}

// SimpleVerifyCc (algorithm/cc.cu:21-60): number of edges whose endpoints
// carry different labels; *ncomp = number of distinct labels.
long long orc_verify_cc(const int* rowptr, const int* colind, int n, const int32_t* label, int* ncomp) {
  long long errors = 0;
  std::unordered_set<int> dict;
  for (int i = 0; i < n; ++i) {
    dict.insert(label[i]);
    for (int k = rowptr[i]; k < rowptr[i + 1]; ++k)
      if (label[colind[k]] != label[i]) ++errors;
  }
  *ncomp = (int)dict.size();
  return errors;
}

// Triangles of a simple undirected graph from its CSR: for every edge (i,k)
// with k < i, |{j < k : j ~ i, j ~ k}| (sorted-list intersection on L).
unsigned long long orc_tc_csr(const int* rowptr, const int* colind, int n) {
  unsigned long long total = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : total)
  for (int i = 0; i < n; ++i) {
    const int* ai = colind + rowptr[i];
    const int li = (int)(std::lower_bound(ai, colind + rowptr[i + 1], i) - ai);  // neighbours < i
    for (int x = 0; x < li; ++x) {
      const int k = ai[x];
      const int* ak = colind + rowptr[k];
      const int lk = (int)(std::lower_bound(ak, colind + rowptr[k + 1], k) - ak);
      int p = 0, q = 0;
      while (p < li && q < lk) {
        if (ai[p] < ak[q]) ++p;
        else if (ai[p] > ak[q]) ++q;
        else {
          if (ai[p] < k) ++total;
          ++p;
          ++q;
        }
      }
    }
  }
  return total;
}

// bmm32_sparse_masked_v5 (bsrbmm/bsrbmm.cu:1214-1265) restated on the row
// layout of L only: sum over mask tiles (I,K), tiles (I,J) and (K,J), of
// sum_r sum_c M[r][c] popc(A_(I,J)[r] & A_(K,J)[c]).
unsigned long long orc_tc_b2sr(const int* brp, const int* bci, const uint64_t* w, int nbr, int b) {
  unsigned long long total = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : total)
  for (int I = 0; I < nbr; ++I)
    for (int m = brp[I]; m < brp[I + 1]; ++m) {
      const int K = bci[m];
      for (int a = brp[I]; a <= m; ++a) {
        const int J = bci[a];
        const int* e = bci + brp[K + 1];
        const int* q = std::lower_bound(bci + brp[K], e, J);
        if (q == e || *q != J) continue;
        const long long tb = q - bci;
        for (int r = 0; r < b; ++r) {
          const uint64_t M = w[(long long)m * b + r];
          if (!M) continue;
          const uint64_t A = w[(long long)a * b + r];
          for (int c = 0; c < b; ++c)
            if ((M >> (b - 1 - c)) & 1) total += popc64(A & w[tb * b + c]);
        }
      }
    }
  return total;
}

// Sparse-output product C = A B over the integers on CSR (the math of
// bmm32_sparse_symbolic/numeric, bsrbmm/bsrbmm.cu:1273-1373): row i of C is
// the multiset union of B's rows m over A's row i, counted per column,
// columns ascending.  Pass 1 (colind == NULL) writes the row lengths into
// rowptr[1..n]; pass 2 fills colind/val at the caller's prefix rowptr.
void orc_spgemm_csr(const int* arp, const int* aci, int n, const int* brp, const int* bci, int m,
                    long long* rowptr, int* colind, int* val) {
#pragma omp parallel
  {
    std::vector<int> acc((size_t)m, 0);
    std::vector<int> touched;
#pragma omp for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
      touched.clear();
      for (int p = arp[i]; p < arp[i + 1]; ++p) {
        const int k = aci[p];
        for (int q = brp[k]; q < brp[k + 1]; ++q) {
          const int j = bci[q];
          if (acc[j]++ == 0) touched.push_back(j);
        }
      }
      std::sort(touched.begin(), touched.end());
      if (!colind) {
        rowptr[i + 1] = (long long)touched.size();
      } else {
        long long o = rowptr[i];
        for (int j : touched) {
          colind[o] = j;
          val[o] = acc[j];
          ++o;
        }
      }
      for (int j : touched) acc[j] = 0;
    }
  }
}

// bmm{4..64}_sparse (bsrbmm/bsrbmm.cu:244-555) restated on tiles: A with row
// words, B with column words (word c = tile column c, row m at bit b-1-m);
// the total over every block row I, A tile (I,K) and B tile (K,C) of
// sum_r sum_c popc(A_IK[r] & B_KC[c]).
unsigned long long orc_bmm_sum_b2sr(const int* arp, const int* aci, const uint64_t* aw, int anbr,
                                    const int* brp, const int* bci, const uint64_t* bw, int b) {
  unsigned long long total = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : total)
  for (int I = 0; I < anbr; ++I)
    for (int ta = arp[I]; ta < arp[I + 1]; ++ta) {
      const int K = aci[ta];
      for (int tb = brp[K]; tb < brp[K + 1]; ++tb)
        for (int r = 0; r < b; ++r) {
          const uint64_t A = aw[(long long)ta * b + r];
          if (!A) continue;
          for (int c = 0; c < b; ++c) total += popc64(A & bw[(long long)tb * b + c]);
        }
    }
  return total;
}

// One pull level of a block-row BFS shard on the CPU, the contract of the
// library's gbo_bfs_shard_level (the masked BMV step of algorithm/bfs.cu:
// 508-564 restricted to the shard's rows): rows [0, nrows) of the shard CSR
// (global column indices), words as one uint64 per b-bit word, `front` the
// whole frontier, `visited` / `level` / `next` the shard's.  Returns the new
// vertices.
unsigned long long orc_bfs_shard_level(const int* rowptr, const int* colind, int nrows, int b,
                                       const uint64_t* front, uint64_t* visited, int32_t* level, int lvl,
                                       uint64_t* next) {
  const int nbr = (nrows + b - 1) / b;
  unsigned long long cnt = 0;
  for (int R = 0; R < nbr; ++R) {
    uint64_t o = 0;
    for (int r = 0; r < b; ++r) {
      const long long i = (long long)R * b + r;
      if (i >= nrows) break;
      if ((visited[R] >> (b - 1 - r)) & 1) continue;
      for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
        const int j = colind[k];
        if ((front[j / b] >> (b - 1 - j % b)) & 1) {
          o |= 1ull << (b - 1 - r);
          break;
        }
      }
    }
    next[R] = o;
    if (o) {
      visited[R] |= o;
      for (int r = 0; r < b; ++r)
        if ((o >> (b - 1 - r)) & 1) level[(long long)R * b + r] = lvl + 1;
      cnt += (unsigned long long)popc64(o);
    }
  }
  return cnt;
}

// ---------------------------------------------------------- generators
// R-MAT (Chakrabarti, Zhan, Faloutsos 2004) with the benchmark's seeding, so
// that the CPU legs build their inputs without the product library: edge k
// draws `scale` uniforms from its own xoshiro256** stream (Blackman & Vigna
// 2018), seeded by four splitmix64 (Steele et al. 2014) outputs started at
// seed ^ (k * 0xD1B54A32D192ED03); a uniform is the top 53 bits of an output
// times 2^-53.  Per level: u < a top-left, < a+b top-right, < a+b+c
// bottom-left, else bottom-right.  The edge list is made symmetric, self
// loops dropped, duplicates removed and each row sorted (both directions
// stored).  Returns the number of stored entries (rowptr[n]); colind must
// hold 2 * 2^scale * edge_factor entries.
static inline uint64_t orc_sm64(uint64_t* s) {
  uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

long long orc_gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                       int* rowptr, int* colind) {
  const long long n = 1ll << scale, m = n * edge_factor;
  std::vector<uint64_t> keys((size_t)(2 * m));
  const double ab = a + b, abc = a + b + c;
#pragma omp parallel for schedule(static)
  for (long long k = 0; k < m; ++k) {
    uint64_t st = seed ^ ((uint64_t)k * 0xD1B54A32D192ED03ull), s[4];
    for (int i = 0; i < 4; ++i) s[i] = orc_sm64(&st);
    uint64_t row = 0, col = 0;
    for (int l = 0; l < scale; ++l) {
      const uint64_t x = s[1] * 5;
      const uint64_t out = ((x << 7) | (x >> 57)) * 9;
      const uint64_t t = s[1] << 17;
      s[2] ^= s[0];
      s[3] ^= s[1];
      s[1] ^= s[2];
      s[0] ^= s[3];
      s[2] ^= t;
      s[3] = (s[3] << 45) | (s[3] >> 19);
      const double u = (double)(out >> 11) * (1.0 / 9007199254740992.0);
      const int down = u >= ab;                           // quadrants c and d
      const int right = (u >= a && u < ab) || u >= abc;   // quadrants b and d
      row = row * 2 + down;
      col = col * 2 + right;
    }
    // both directions; a self loop becomes two copies of a sentinel key
    const uint64_t none = ~0ull;
    keys[(size_t)(2 * k)] = row == col ? none : (row << 32 | col);
    keys[(size_t)(2 * k + 1)] = row == col ? none : (col << 32 | row);
  }
  __gnu_parallel::sort(keys.begin(), keys.end());
  const size_t end = (size_t)(std::unique(keys.begin(), keys.end()) - keys.begin());
  size_t nnz = end;
  if (nnz && keys[nnz - 1] == ~0ull) --nnz;
  for (long long i = 0; i <= n; ++i) rowptr[i] = 0;
  for (size_t e = 0; e < nnz; ++e) {
    rowptr[(keys[e] >> 32) + 1]++;
    colind[e] = (int)(keys[e] & 0xffffffffu);
  }
  for (long long i = 0; i < n; ++i) rowptr[i + 1] += rowptr[i];
  return (long long)nnz;
}

int orc_max_threads(void) { return omp_get_max_threads(); }
void orc_set_threads(int n) { omp_set_num_threads(n); }

}  // extern "C"
