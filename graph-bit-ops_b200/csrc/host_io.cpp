// Host side of the input path: Matrix Market reading with the reference's two
// semantics, CSR utilities and seeded synthetic graph generators.
//
// Replaces readMtx/removeSelfloop/customSort/coo2csr/csr2csc
// (algorithm/readMtx.hpp:150-423) and mmio_data (algorithm/mmio_highlevel.h:
// 139-309).  The reference parses with fscanf and sorts a vector of tuples;
// here the file is read in one block, parsed by hand, and CSR rows are built
// by counting sort + per-row sort (OpenMP), which gives the same CSR.
#include <errno.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <string>
#include <vector>

#include <immintrin.h>

#include "host_common.h"

namespace gbo {

int host_transpose(const int* rowptr, const int* colind, int nrows, int ncols, long long nnz,
                   std::vector<int>* tptr, std::vector<int>* tcol);
int host_degree_relabel(const int* rowptr, const int* colind, int n, long long nnz,
                        std::vector<int>* new_of_old, std::vector<int>* nptr, std::vector<int>* ncol);

namespace {

// ------------------------------------------------------------------ PRNG
inline uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

// xoshiro256** seeded from splitmix64(seed ^ stream * golden-ratio constant).
struct Xoshiro {
  uint64_t s[4];
  Xoshiro(uint64_t seed, uint64_t stream) {
    uint64_t sm = seed ^ (stream * 0xD1B54A32D192ED03ull);
    for (int i = 0; i < 4; ++i) s[i] = splitmix64(sm);
  }
  uint64_t next() {
    const uint64_t result = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return result;
  }
  double uniform() { return (double)(next() >> 11) * 0x1.0p-53; }
  // integer in [0, n)
  uint64_t below(uint64_t n) { return (uint64_t)(((unsigned __int128)next() * n) >> 64); }
};

gbo_csr* new_csr(int nrows, int ncols, long long nnz) {
  if (inject_host_alloc_fails()) return nullptr;
  gbo_csr* c = (gbo_csr*)calloc(1, sizeof(gbo_csr));
  if (!c) return nullptr;
  c->nrows = nrows;
  c->ncols = ncols;
  c->nnz = nnz;
  c->rowptr = (int*)malloc(sizeof(int) * ((size_t)nrows + 1));
  c->colind = (int*)malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
  if (!c->rowptr || !c->colind) {
    free(c->rowptr);
    free(c->colind);
    free(c);
    return nullptr;
  }
  return c;
}

// Build a CSR from (row, col) pairs: rows bucketed, each row sorted, and
// optionally deduplicated.  Self-loops are dropped when drop_self is set.
int csr_from_pairs(const std::vector<int>& rows, const std::vector<int>& cols, int nrows,
                   int ncols, bool dedup, bool drop_self, gbo_csr** out) {
  const long long m = (long long)rows.size();
  std::vector<long long> cnt((size_t)nrows + 1, 0);
  for (long long i = 0; i < m; ++i) {
    if (drop_self && rows[i] == cols[i]) continue;
    cnt[(size_t)rows[i] + 1]++;
  }
  for (int i = 0; i < nrows; ++i) cnt[(size_t)i + 1] += cnt[i];
  std::vector<int> tmp((size_t)cnt[nrows]);
  std::vector<long long> pos(cnt.begin(), cnt.end() - 1);
  for (long long i = 0; i < m; ++i) {
    if (drop_self && rows[i] == cols[i]) continue;
    tmp[(size_t)pos[rows[i]]++] = cols[i];
  }
  std::vector<int> newlen((size_t)nrows, 0);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int r = 0; r < nrows; ++r) {
    int* a = tmp.data() + cnt[r];
    int* e = tmp.data() + cnt[(size_t)r + 1];
    std::sort(a, e);
    if (dedup) e = std::unique(a, e);
    newlen[r] = (int)(e - a);
  }
  long long nnz = 0;
  for (int r = 0; r < nrows; ++r) nnz += newlen[r];
  if (nnz > 2147483647LL) return fail(GBO_ERR_OVERFLOW, "more than 2^31-1 CSR entries");
  gbo_csr* c = new_csr(nrows, ncols, nnz);
  if (!c) return fail(GBO_ERR_NOMEM, "host CSR allocation");
  c->rowptr[0] = 0;
  for (int r = 0; r < nrows; ++r) c->rowptr[r + 1] = c->rowptr[r] + newlen[r];
#pragma omp parallel for schedule(dynamic, 1024)
  for (int r = 0; r < nrows; ++r)
    memcpy(c->colind + c->rowptr[r], tmp.data() + cnt[r], sizeof(int) * (size_t)newlen[r]);
  *out = c;
  return GBO_OK;
}

// --------------------------------------------------------- Matrix Market
bool read_file(const char* path, std::string* data) {
  FILE* f = fopen(path, "rb");
  if (!f) return false;
  fseek(f, 0, SEEK_END);
  long sz = ftell(f);
  fseek(f, 0, SEEK_SET);
  data->resize(sz > 0 ? (size_t)sz : 0);
  size_t got = sz > 0 ? fread(&(*data)[0], 1, (size_t)sz, f) : 0;
  fclose(f);
  return got == data->size();
}

std::string lower(std::string s) {
  for (char& ch : s) ch = (char)tolower((unsigned char)ch);
  return s;
}

}  // namespace

// Banner, comments and size line of a Matrix Market text in [p, end);
// *entries gets the position right after the size line's numbers.
int parse_mtx_header(const char* p, const char* end, MtxHeader* h, const char** entries) {
  // banner
  const char* nl = (const char*)memchr(p, '\n', (size_t)(end - p));
  std::string banner(p, nl ? nl : end);
  std::string b = lower(banner);
  if (b.rfind("%%matrixmarket", 0) != 0) return fail(GBO_ERR_IO, "missing %%MatrixMarket banner");
  if (b.find("coordinate") == std::string::npos)
    return fail(GBO_ERR_IO, "only coordinate Matrix Market files are supported");
  h->pattern = b.find("pattern") != std::string::npos;
  h->real = b.find("real") != std::string::npos;
  h->integer = b.find("integer") != std::string::npos;
  h->complex_ = b.find("complex") != std::string::npos;
  h->skew = b.find("skew-symmetric") != std::string::npos;
  h->hermitian = b.find("hermitian") != std::string::npos;
  h->symmetric = !h->skew && b.find("symmetric") != std::string::npos;
  p = nl ? nl + 1 : end;
  // comments
  while (p < end && (*p == '%' || *p == '\n' || *p == '\r')) {
    const char* q = (const char*)memchr(p, '\n', (size_t)(end - p));
    p = q ? q + 1 : end;
  }
  char* e2 = nullptr;
  long long r = strtoll(p, &e2, 10);
  long long c = strtoll(e2, &e2, 10);
  long long z = strtoll(e2, &e2, 10);
  if (e2 == p || r < 0 || c < 0 || z < 0 || r > 2147483647LL || c > 2147483647LL)
    return fail(GBO_ERR_IO, "bad Matrix Market size line");
  h->nrows = (int)r;
  h->ncols = (int)c;
  h->nnz = z;
  *entries = e2;
  return GBO_OK;
}

bool env_remove_self_loops() {
  // GRB_UTIL_REMOVE_SELFLOOP, default true (readMtx.hpp:155).
  const char* v = getenv("GRB_UTIL_REMOVE_SELFLOOP");
  if (!v) return true;
  return atoi(v) != 0;
}

namespace {

int parse_mtx(const char* path, MtxHeader* h, std::vector<int>* I, std::vector<int>* J) {
  std::string data;
  if (!read_file(path, &data)) return fail(GBO_ERR_IO, std::string("cannot read ") + path);
  const char* p = nullptr;
  const char* end = data.c_str() + data.size();
  GBO_HOST_TRY(parse_mtx_header(data.c_str(), end, h, &p));
  const long long r = h->nrows, c = h->ncols, z = h->nnz;
  I->resize((size_t)z);
  J->resize((size_t)z);
  for (long long k = 0; k < z; ++k) {
    // skip to the next line start, then parse "i j [values]"
    while (p < end && (*p == '\n' || *p == '\r' || *p == ' ' || *p == '\t')) ++p;
    if (p >= end) return fail(GBO_ERR_IO, "fewer entries than the size line promises");
    char* q = nullptr;
    long long i = strtoll(p, &q, 10);
    if (q == p) return fail(GBO_ERR_IO, "malformed entry line");
    long long j = strtoll(q, &q, 10);
    if (i < 1 || j < 1 || i > r || j > c) return fail(GBO_ERR_BOUNDS, "entry index outside the matrix");
    (*I)[(size_t)k] = (int)(i - 1);
    (*J)[(size_t)k] = (int)(j - 1);
    const char* eol = (const char*)memchr(q, '\n', (size_t)(end - q));
    p = eol ? eol + 1 : end;
  }
  return GBO_OK;
}

}  // namespace

int host_transpose(const int* rowptr, const int* colind, int nrows, int ncols, long long nnz,
                   std::vector<int>* tptr, std::vector<int>* tcol) {
  tptr->assign((size_t)ncols + 1, 0);
  tcol->resize((size_t)nnz);
  for (long long k = 0; k < nnz; ++k) {
    int c = colind[k];
    if (c < 0 || c >= ncols) return fail(GBO_ERR_BOUNDS, "CSR column index outside [0, ncols)");
    (*tptr)[(size_t)c + 1]++;
  }
  for (int c = 0; c < ncols; ++c) (*tptr)[(size_t)c + 1] += (*tptr)[c];
  std::vector<int> pos(tptr->begin(), tptr->end() - 1);
  // rows visited in ascending order: every column's row list comes out sorted
  for (int r = 0; r < nrows; ++r)
    for (int k = rowptr[r]; k < rowptr[r + 1]; ++k) (*tcol)[(size_t)pos[colind[k]]++] = r;
  return GBO_OK;
}

// Relabel the vertices of a square CSR by descending degree (ties by id):
// (*new_of_old)[v] is the new label of v; the relabelled CSR comes out with
// every row's columns ascending.
int host_degree_relabel(const int* rowptr, const int* colind, int n, long long nnz,
                        std::vector<int>* new_of_old, std::vector<int>* nptr, std::vector<int>* ncol) {
  std::vector<int> order((size_t)n);
  for (int v = 0; v < n; ++v) order[(size_t)v] = v;
  std::sort(order.begin(), order.end(), [&](int a, int b) {
    const int da = rowptr[a + 1] - rowptr[a], db = rowptr[b + 1] - rowptr[b];
    return da != db ? da > db : a < b;
  });
  new_of_old->resize((size_t)n);
  for (int k = 0; k < n; ++k) (*new_of_old)[(size_t)order[(size_t)k]] = k;
  nptr->assign((size_t)n + 1, 0);
  for (int k = 0; k < n; ++k) {
    const int v = order[(size_t)k];
    (*nptr)[(size_t)k + 1] = (*nptr)[(size_t)k] + (rowptr[v + 1] - rowptr[v]);
  }
  ncol->resize((size_t)nnz);
  std::atomic<int> bad{0};
#pragma omp parallel for schedule(dynamic, 1024)
  for (int k = 0; k < n; ++k) {
    const int v = order[(size_t)k];
    int* dst = ncol->data() + (*nptr)[(size_t)k];
    for (int j = rowptr[v]; j < rowptr[v + 1]; ++j) {
      const int c = colind[j];
      if (c < 0 || c >= n) {
        bad = 1;
        *dst++ = 0;
      } else {
        *dst++ = (*new_of_old)[(size_t)c];
      }
    }
    std::sort(ncol->data() + (*nptr)[(size_t)k], dst);
  }
  if (bad) return fail(GBO_ERR_BOUNDS, "CSR column index outside [0, n)");
  return GBO_OK;
}

}  // namespace gbo

using namespace gbo;

extern "C" int gbo_csr_free(gbo_csr* csr) {
  if (csr) {
    free(csr->rowptr);
    free(csr->colind);
    free(csr);
  }
  return GBO_OK;
}

extern "C" int gbo_read_mtx(const char* path, int mode, int directed, gbo_csr** out) {
  clear_error();
  if (!path || !out) return fail(GBO_ERR_INVALID, "NULL argument");
  *out = nullptr;
  if (mode != GBO_MTX_READMTX && mode != GBO_MTX_MMIO) return fail(GBO_ERR_INVALID, "bad mode");
  MtxHeader h;
  std::vector<int> I, J;
  int st = parse_mtx(path, &h, &I, &J);
  if (st != GBO_OK) return st;
  std::vector<int> rows, cols;
  rows.reserve(I.size() * 2);
  cols.reserve(I.size() * 2);
  if (mode == GBO_MTX_READMTX) {
    // readMtx: undirected if the banner says symmetric or directed == 2,
    // never if directed == 1 (readMtx.hpp:380-384).
    bool undirected = h.symmetric || directed == 2;
    if (directed == 1) undirected = false;
    for (size_t k = 0; k < I.size(); ++k) {
      rows.push_back(I[k]);
      cols.push_back(J[k]);
    }
    if (undirected)
      for (size_t k = 0; k < I.size(); ++k)
        if (I[k] != J[k]) {
          rows.push_back(J[k]);
          cols.push_back(I[k]);
        }
    // sort, drop self-loops (GRB_UTIL_REMOVE_SELFLOOP) and duplicates
    return csr_from_pairs(rows, cols, h.nrows, h.ncols, true, env_remove_self_loops(), out);
  }
  // mmio_data: symmetric or hermitian banners mirror off-diagonal entries;
  // self-loops and duplicates stay (mmio_highlevel.h:213-292).
  const bool mirror = h.symmetric || h.hermitian;
  for (size_t k = 0; k < I.size(); ++k) {
    rows.push_back(I[k]);
    cols.push_back(J[k]);
    if (mirror && I[k] != J[k]) {
      rows.push_back(J[k]);
      cols.push_back(I[k]);
    }
  }
  return csr_from_pairs(rows, cols, h.nrows, h.ncols, false, false, out);
}

extern "C" int gbo_csr_transpose(const gbo_csr* in, gbo_csr** out) {
  clear_error();
  if (!in || !out) return fail(GBO_ERR_INVALID, "NULL argument");
  std::vector<int> tp, tc;
  int st = host_transpose(in->rowptr, in->colind, in->nrows, in->ncols, in->nnz, &tp, &tc);
  if (st != GBO_OK) return st;
  gbo_csr* c = new_csr(in->ncols, in->nrows, in->nnz);
  if (!c) return fail(GBO_ERR_NOMEM, "host CSR allocation");
  memcpy(c->rowptr, tp.data(), sizeof(int) * tp.size());
  if (in->nnz) memcpy(c->colind, tc.data(), sizeof(int) * tc.size());
  *out = c;
  return GBO_OK;
}

extern "C" int gbo_csr_tril(const gbo_csr* in, gbo_csr** out) {
  clear_error();
  if (!in || !out) return fail(GBO_ERR_INVALID, "NULL argument");
  long long nnz = 0;
  for (int r = 0; r < in->nrows; ++r)
    for (int k = in->rowptr[r]; k < in->rowptr[r + 1]; ++k) nnz += in->colind[k] <= r;
  gbo_csr* c = new_csr(in->nrows, in->ncols, nnz);
  if (!c) return fail(GBO_ERR_NOMEM, "host CSR allocation");
  long long p = 0;
  c->rowptr[0] = 0;
  for (int r = 0; r < in->nrows; ++r) {
    for (int k = in->rowptr[r]; k < in->rowptr[r + 1]; ++k)
      if (in->colind[k] <= r) c->colind[p++] = in->colind[k];
    c->rowptr[r + 1] = (int)p;
  }
  *out = c;
  return GBO_OK;
}

extern "C" int gbo_csr_from_edges(const int* src, const int* dst, int64_t nedges, int nvertices,
                                  int symmetrize, int drop_self_loops, gbo_csr** out) {
  clear_error();
  if (!out || nvertices < 0 || nedges < 0 || (nedges > 0 && (!src || !dst)))
    return fail(GBO_ERR_INVALID, "bad argument");
  std::vector<int> rows, cols;
  rows.reserve((size_t)nedges * (symmetrize ? 2 : 1));
  cols.reserve((size_t)nedges * (symmetrize ? 2 : 1));
  for (int64_t k = 0; k < nedges; ++k) {
    if (src[k] < 0 || src[k] >= nvertices || dst[k] < 0 || dst[k] >= nvertices)
      return fail(GBO_ERR_BOUNDS, "edge endpoint outside [0, nvertices)");
    rows.push_back(src[k]);
    cols.push_back(dst[k]);
    if (symmetrize) {
      rows.push_back(dst[k]);
      cols.push_back(src[k]);
    }
  }
  return csr_from_pairs(rows, cols, nvertices, nvertices, true, drop_self_loops != 0, out);
}

// R-MAT (Chakrabarti et al. 2004): each of 2^scale * edge_factor edges picks a
// quadrant per level with probabilities (a, b, c, 1-a-b-c); edge k uses its
// own xoshiro256** stream, so the graph does not depend on the thread count.
// The result is symmetrised, without self-loops, deduplicated and sorted.
extern "C" int gbo_gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                            gbo_csr** out) {
  clear_error();
  if (!out || scale < 1 || scale > 30 || edge_factor < 1 || a < 0 || b < 0 || c < 0 || a + b + c > 1)
    return fail(GBO_ERR_INVALID, "bad R-MAT parameters");
  const int n = 1 << scale;
  const long long m = (long long)n * edge_factor;
  const double ab = a + b, abc = a + b + c;
  // degree counts (both directions, no self-loops)
  std::vector<int> eu((size_t)m), ev((size_t)m);
#pragma omp parallel for schedule(static)
  for (long long k = 0; k < m; ++k) {
    Xoshiro rng(seed, (uint64_t)k);
    int u = 0, v = 0;
    for (int l = 0; l < scale; ++l) {
      double r = rng.uniform();
      int rb = r >= ab ? 1 : 0;                 // quadrants c, d: lower half
      int cb = (r >= a && r < ab) || r >= abc;  // quadrants b, d: right half
      u = (u << 1) | rb;
      v = (v << 1) | cb;
    }
    eu[(size_t)k] = u;
    ev[(size_t)k] = v;
  }
  // counting sort into rows (both directions), then per-row sort + unique
  std::vector<long long> cnt((size_t)n + 1, 0);
  {
    std::vector<std::atomic<long long>> acnt((size_t)n);
    for (auto& x : acnt) x.store(0, std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
    for (long long k = 0; k < m; ++k) {
      int u = eu[(size_t)k], v = ev[(size_t)k];
      if (u == v) continue;
      acnt[(size_t)u].fetch_add(1, std::memory_order_relaxed);
      acnt[(size_t)v].fetch_add(1, std::memory_order_relaxed);
    }
    for (int i = 0; i < n; ++i) cnt[(size_t)i + 1] = cnt[i] + acnt[(size_t)i].load();
  }
  std::vector<int> tmp((size_t)cnt[n]);
  {
    std::vector<std::atomic<long long>> pos((size_t)n);
    for (int i = 0; i < n; ++i) pos[(size_t)i].store(cnt[i], std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
    for (long long k = 0; k < m; ++k) {
      int u = eu[(size_t)k], v = ev[(size_t)k];
      if (u == v) continue;
      tmp[(size_t)pos[(size_t)u].fetch_add(1, std::memory_order_relaxed)] = v;
      tmp[(size_t)pos[(size_t)v].fetch_add(1, std::memory_order_relaxed)] = u;
    }
  }
  std::vector<int>().swap(eu);
  std::vector<int>().swap(ev);
  std::vector<int> len((size_t)n);
#pragma omp parallel for schedule(dynamic, 256)
  for (int r = 0; r < n; ++r) {
    int* p0 = tmp.data() + cnt[r];
    int* p1 = tmp.data() + cnt[(size_t)r + 1];
    std::sort(p0, p1);
    len[(size_t)r] = (int)(std::unique(p0, p1) - p0);
  }
  long long nnz = 0;
  for (int r = 0; r < n; ++r) nnz += len[(size_t)r];
  if (nnz > 2147483647LL) return fail(GBO_ERR_OVERFLOW, "more than 2^31-1 CSR entries");
  gbo_csr* g = new_csr(n, n, nnz);
  if (!g) return fail(GBO_ERR_NOMEM, "host CSR allocation");
  g->rowptr[0] = 0;
  for (int r = 0; r < n; ++r) g->rowptr[r + 1] = g->rowptr[r] + len[(size_t)r];
#pragma omp parallel for schedule(dynamic, 256)
  for (int r = 0; r < n; ++r)
    memcpy(g->colind + g->rowptr[r], tmp.data() + cnt[r], sizeof(int) * (size_t)len[(size_t)r]);
  *out = g;
  return GBO_OK;
}

// G(n, p) with per-row streams and geometric skipping over j > i.
extern "C" int gbo_gen_er(int n, double p, uint64_t seed, gbo_csr** out) {
  clear_error();
  if (!out || n < 0 || p < 0 || p > 1) return fail(GBO_ERR_INVALID, "bad ER parameters");
  std::vector<std::vector<int>> nb((size_t)n);
  if (p > 0) {
    const double lq = p < 1 ? std::log1p(-p) : 0.0;
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
      Xoshiro rng(seed, (uint64_t)i);
      long long j = i;
      while (true) {
        if (p >= 1) {
          j += 1;
        } else {
          double u = rng.uniform();
          j += 1 + (long long)std::floor(std::log1p(-u) / lq);
        }
        if (j >= n) break;
        nb[(size_t)i].push_back((int)j);
      }
    }
  }
  std::vector<int> rows, cols;
  for (int i = 0; i < n; ++i)
    for (int j : nb[(size_t)i]) {
      rows.push_back(i);
      cols.push_back(j);
      rows.push_back(j);
      cols.push_back(i);
    }
  return csr_from_pairs(rows, cols, n, n, true, true, out);
}

// G(n, m) with m = round(n * avg_degree / 2) uniformly drawn pairs.
extern "C" int gbo_gen_er_avgdeg(int n, double avg_degree, uint64_t seed, gbo_csr** out) {
  clear_error();
  if (!out || n < 1 || avg_degree < 0) return fail(GBO_ERR_INVALID, "bad ER parameters");
  const long long m = (long long)std::llround((double)n * avg_degree / 2.0);
  std::vector<int> rows((size_t)m * 2), cols((size_t)m * 2);
#pragma omp parallel for schedule(static)
  for (long long k = 0; k < m; ++k) {
    Xoshiro rng(seed, (uint64_t)k);
    int u = (int)rng.below((uint64_t)n);
    int v = (int)rng.below((uint64_t)n);
    rows[(size_t)(2 * k)] = u;
    cols[(size_t)(2 * k)] = v;
    rows[(size_t)(2 * k + 1)] = v;
    cols[(size_t)(2 * k + 1)] = u;
  }
  return csr_from_pairs(rows, cols, n, n, true, true, out);
}

// side x side king-move mesh, vertex id = r * side + c, 8-neighbourhood.
extern "C" int gbo_gen_king_mesh(int side, gbo_csr** out) {
  clear_error();
  if (!out || side < 1 || (long long)side * side > 2147483647LL) return fail(GBO_ERR_INVALID, "bad side");
  const int n = side * side;
  std::vector<int> deg((size_t)n);
#pragma omp parallel for schedule(static)
  for (int v = 0; v < n; ++v) {
    int r = v / side, c = v % side, d = 0;
    for (int dr = -1; dr <= 1; ++dr)
      for (int dc = -1; dc <= 1; ++dc) {
        if (!dr && !dc) continue;
        int rr = r + dr, cc = c + dc;
        d += rr >= 0 && rr < side && cc >= 0 && cc < side;
      }
    deg[(size_t)v] = d;
  }
  long long nnz = 0;
  for (int v = 0; v < n; ++v) nnz += deg[(size_t)v];
  if (nnz > 2147483647LL) return fail(GBO_ERR_OVERFLOW, "more than 2^31-1 CSR entries");
  gbo_csr* g = new_csr(n, n, nnz);
  if (!g) return fail(GBO_ERR_NOMEM, "host CSR allocation");
  g->rowptr[0] = 0;
  for (int v = 0; v < n; ++v) g->rowptr[v + 1] = g->rowptr[v] + deg[(size_t)v];
#pragma omp parallel for schedule(static)
  for (int v = 0; v < n; ++v) {
    int r = v / side, c = v % side, p = g->rowptr[v];
    for (int dr = -1; dr <= 1; ++dr)
      for (int dc = -1; dc <= 1; ++dc) {
        if (!dr && !dc) continue;
        int rr = r + dr, cc = c + dc;
        if (rr >= 0 && rr < side && cc >= 0 && cc < side) g->colind[p++] = rr * side + cc;
      }
  }
  *out = g;
  return GBO_OK;
}

// A batch of independent G(n, m) graphs as one block-diagonal CSR: graph i
// has n_i vertices, log-uniform in [nmin, nmax] (drawn from stream i of
// `seed`), and round(n_i * avg_degree / 2) uniformly drawn pairs from its own
// seed `seed + 1000 + i`.  offsets (count+1 entries) receives the first vertex
// of every graph.
extern "C" int gbo_gen_er_batch(int count, int nmin, int nmax, double avg_degree, uint64_t seed,
                                gbo_csr** out, int* offsets) {
  clear_error();
  if (!out || !offsets || count < 1 || nmin < 1 || nmax < nmin || avg_degree < 0)
    return fail(GBO_ERR_INVALID, "bad batch parameters");
  std::vector<long long> off((size_t)count + 1, 0);
  const double l0 = std::log((double)nmin), l1 = std::log((double)nmax + 1.0);
  for (int i = 0; i < count; ++i) {
    Xoshiro rng(seed, (uint64_t)i);
    long long n = (long long)std::floor(std::exp(l0 + (l1 - l0) * rng.uniform()));
    if (n < nmin) n = nmin;
    if (n > nmax) n = nmax;
    off[(size_t)i + 1] = off[(size_t)i] + n;
  }
  if (off[(size_t)count] > 2147483647LL) return fail(GBO_ERR_OVERFLOW, "batch has more than 2^31-1 vertices");
  const int N = (int)off[(size_t)count];
  std::vector<std::vector<int>> adj_ptr((size_t)count), adj_col((size_t)count);
  long long total = 0;
  int st_all = GBO_OK;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : total)
  for (int i = 0; i < count; ++i) {
    const int n = (int)(off[(size_t)i + 1] - off[(size_t)i]);
    const long long m = (long long)std::llround((double)n * avg_degree / 2.0);
    std::vector<int> rows((size_t)m * 2), cols((size_t)m * 2);
    for (long long k = 0; k < m; ++k) {
      Xoshiro rng(seed + 1000 + (uint64_t)i, (uint64_t)k);
      int u = (int)rng.below((uint64_t)n), v = (int)rng.below((uint64_t)n);
      rows[(size_t)(2 * k)] = u;
      cols[(size_t)(2 * k)] = v;
      rows[(size_t)(2 * k + 1)] = v;
      cols[(size_t)(2 * k + 1)] = u;
    }
    gbo_csr* c = nullptr;
    if (csr_from_pairs(rows, cols, n, n, true, true, &c) != GBO_OK) {
      st_all = GBO_ERR_NOMEM;
      continue;
    }
    adj_ptr[(size_t)i].assign(c->rowptr, c->rowptr + n + 1);
    adj_col[(size_t)i].assign(c->colind, c->colind + c->nnz);
    total += c->nnz;
    gbo_csr_free(c);
  }
  if (st_all != GBO_OK) return fail(st_all, "batch generation");
  if (total > 2147483647LL) return fail(GBO_ERR_OVERFLOW, "batch has more than 2^31-1 entries");
  gbo_csr* g = new_csr(N, N, total);
  if (!g) return fail(GBO_ERR_NOMEM, "host CSR allocation");
  std::vector<long long> eoff((size_t)count + 1, 0);
  for (int i = 0; i < count; ++i) eoff[(size_t)i + 1] = eoff[(size_t)i] + (long long)adj_col[(size_t)i].size();
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < count; ++i) {
    const int base = (int)off[(size_t)i];
    const int n = (int)(off[(size_t)i + 1] - off[(size_t)i]);
    for (int r = 0; r < n; ++r) g->rowptr[base + r] = (int)(eoff[(size_t)i] + adj_ptr[(size_t)i][(size_t)r]);
    const std::vector<int>& cc = adj_col[(size_t)i];
    for (size_t k = 0; k < cc.size(); ++k) g->colind[eoff[(size_t)i] + (long long)k] = cc[k] + base;
  }
  g->rowptr[N] = (int)total;
  for (int i = 0; i <= count; ++i) offsets[i] = (int)off[(size_t)i];
  *out = g;
  return GBO_OK;
}

// ----------------------------------------------------- result widening
// Served BFS results travel as byte levels (255 = unreachable) and are
// widened to the caller's int32 levels (-1 = unreachable) on the client
// thread.  That pass writes 16 bytes per 4 read per vertex, so it is written
// with AVX2 and non-temporal stores (no read-for-ownership of the 4n-byte
// destination) where the CPU has AVX2.
namespace gbo {
namespace {
__attribute__((target("avx2"))) void widen_levels_avx2(const unsigned char* b8, int* o, long long n) {
  long long i = 0;
  for (; i < n && (reinterpret_cast<uintptr_t>(o + i) & 31); ++i) o[i] = b8[i] == 255 ? -1 : b8[i];
  const __m256i ff = _mm256_set1_epi32(255);
  for (; i + 32 <= n; i += 32) {
    const __m256i v = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(b8 + i));
    const __m128i lo = _mm256_castsi256_si128(v);
    const __m128i hi = _mm256_extracti128_si256(v, 1);
    __m256i q[4] = {_mm256_cvtepu8_epi32(lo), _mm256_cvtepu8_epi32(_mm_srli_si128(lo, 8)),
                    _mm256_cvtepu8_epi32(hi), _mm256_cvtepu8_epi32(_mm_srli_si128(hi, 8))};
    for (int k = 0; k < 4; ++k) {
      q[k] = _mm256_or_si256(q[k], _mm256_cmpeq_epi32(q[k], ff));  // 255 -> all ones = -1
      _mm256_stream_si256(reinterpret_cast<__m256i*>(o + i + 8 * k), q[k]);
    }
  }
  for (; i < n; ++i) o[i] = b8[i] == 255 ? -1 : b8[i];
  _mm_sfence();
}
}  // namespace

void host_widen_levels(const unsigned char* b8, int* o, long long n) {
  static const bool avx2 = __builtin_cpu_supports("avx2");
  if (avx2) {
    widen_levels_avx2(b8, o, n);
    return;
  }
  for (long long i = 0; i < n; ++i) o[i] = (int)b8[i] | -(int)(b8[i] == 255);
}
}  // namespace gbo
