// Matrix Market reader of the bksp API (reference src/read_matrix.c:38-173):
// coordinate real / integer / pattern files, 1-based indices converted to
// 0-based CSR with the entries of each row kept in file order (the
// reference's coo2csr is a stable counting sort by row).  The whole file is
// read at once and its entry lines parsed by several threads.
#include <algorithm>
#include <cctype>
#include <charconv>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/bksp.h"
#include "mmio.h"

namespace {

std::string lower(std::string s) {
  for (char& c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

}  // namespace

namespace bk {

namespace {

const char* skip_blank(const char* p, const char* e) {
  while (p < e && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
  return p;
}

template <typename T>
bool parse_num(const char*& p, const char* e, T& v) {
  p = skip_blank(p, e);
  if (p < e && *p == '+') ++p;
  const auto r = std::from_chars(p, e, v);
  if (r.ec != std::errc()) return false;
  p = r.ptr;
  return true;
}

// Entry lines [b, e): appends coordinates and values; false on a bad line.
bool parse_chunk(const char* b, const char* e, bool pattern, bool cplx,
                 long long M, long long N, std::vector<int>& ri,
                 std::vector<int>& ci, std::vector<double>& vv,
                 std::vector<double>& vi) {
  const char* p = b;
  while (p < e) {
    const char* q = skip_blank(p, e);
    if (q < e && *q == '\n') { p = q + 1; continue; }   // blank line
    if (q >= e) break;
    long long i = 0, j = 0;
    double v = 1.0, w = 0.0;
    if (!parse_num(q, e, i) || !parse_num(q, e, j)) return false;
    if (!pattern && !parse_num(q, e, v)) return false;
    if (cplx && !parse_num(q, e, w)) return false;
    if (i < 1 || i > M || j < 1 || j > N) return false;
    q = skip_blank(q, e);
    if (q < e && *q != '\n') return false;
    ri.push_back((int)(i - 1));
    ci.push_back((int)(j - 1));
    vv.push_back(v);
    if (cplx) vi.push_back(w);
    p = q < e ? q + 1 : e;
  }
  return true;
}

}  // namespace

bool mm_parse(const char* path, MmData& out, bool complex_field) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  std::string buf;
  {
    std::fseek(f, 0, SEEK_END);
    const long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (sz < 0) { std::fclose(f); return false; }
    buf.resize((size_t)sz);
    const size_t got = sz > 0 ? std::fread(&buf[0], 1, (size_t)sz, f) : 0;
    std::fclose(f);
    if (got != (size_t)sz) return false;
  }
  const char* p = buf.data();
  const char* end = p + buf.size();
  auto next_line = [&](std::string& line) {
    if (p >= end) return false;
    const char* q = static_cast<const char*>(std::memchr(p, '\n', (size_t)(end - p)));
    const char* le = q ? q : end;
    line.assign(p, le);
    p = q ? q + 1 : end;
    return true;
  };
  std::string line;
  if (!next_line(line)) return false;
  char b0[64] = {0}, b1[64] = {0}, b2[64] = {0}, b3[64] = {0}, b4[64] = {0};
  if (std::sscanf(line.c_str(), "%63s %63s %63s %63s %63s", b0, b1, b2, b3, b4) != 5 ||
      lower(b0) != "%%matrixmarket" || lower(b1) != "matrix" ||
      lower(b2) != "coordinate")
    return false;
  const std::string field = lower(b3), sym = lower(b4);
  if ((field == "complex") != complex_field) return false;
  const bool pattern = field == "pattern";
  long long M = 0, N = 0, nz = 0;
  for (;;) {
    if (!next_line(line)) return false;
    if (!line.empty() && line[0] == '%') continue;
    if (std::sscanf(line.c_str(), "%lld %lld %lld", &M, &N, &nz) == 3) break;
    for (char c : line)
      if (!std::isspace((unsigned char)c)) return false;
  }
  if (M <= 0 || N <= 0 || nz < 0 || M > 0x7fffffff || N > 0x7fffffff ||
      nz > 0x7fffffff)
    return false;
  // Entry lines: chunks of >= 4 MB split at line ends, one thread each.
  const size_t bytes = (size_t)(end - p);
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t nchunk = std::max<size_t>(1, std::min<size_t>(hw, bytes / (4u << 20)));
  std::vector<const char*> cut(nchunk + 1);
  cut[0] = p;
  cut[nchunk] = end;
  for (size_t c = 1; c < nchunk; ++c) {
    const char* q = p + bytes * c / nchunk;
    if (q < cut[c - 1]) q = cut[c - 1];
    const char* nl = static_cast<const char*>(std::memchr(q, '\n', (size_t)(end - q)));
    cut[c] = nl ? nl + 1 : end;
  }
  std::vector<std::vector<int>> ri(nchunk), ci(nchunk);
  std::vector<std::vector<double>> vv(nchunk), vi(nchunk);
  std::vector<char> ok(nchunk, 0);
  auto work = [&](size_t c) {
    const size_t guess = (size_t)(nz / (long long)nchunk + 16);
    ri[c].reserve(guess);
    ci[c].reserve(guess);
    vv[c].reserve(guess);
    if (complex_field) vi[c].reserve(guess);
    ok[c] = parse_chunk(cut[c], cut[c + 1], pattern, complex_field, M, N, ri[c],
                        ci[c], vv[c], vi[c]);
  };
  std::vector<std::thread> th;
  for (size_t c = 1; c < nchunk; ++c) th.emplace_back(work, c);
  work(0);
  for (auto& t : th) t.join();
  size_t total = 0;
  for (size_t c = 0; c < nchunk; ++c) {
    if (!ok[c]) return false;
    total += ri[c].size();
  }
  if ((long long)total != nz) return false;
  out.rows = M;
  out.cols = N;
  out.symmetric = sym == "symmetric";
  out.ri.clear();
  out.ci.clear();
  out.vv.clear();
  out.vi.clear();
  out.ri.reserve(total);
  out.ci.reserve(total);
  out.vv.reserve(total);
  for (size_t c = 0; c < nchunk; ++c) {
    out.ri.insert(out.ri.end(), ri[c].begin(), ri[c].end());
    out.ci.insert(out.ci.end(), ci[c].begin(), ci[c].end());
    out.vv.insert(out.vv.end(), vv[c].begin(), vv[c].end());
    out.vi.insert(out.vi.end(), vi[c].begin(), vi[c].end());
  }
  return true;
}

}  // namespace bk

extern "C" dspmat* read_matrix_market(char* filename) {
  if (!filename) return nullptr;
  bk::MmData d;
  if (!bk::mm_parse(filename, d)) return nullptr;
  const long long M = d.rows, N = d.cols, nz = (long long)d.ri.size();
  const std::vector<int>& ri = d.ri;
  const std::vector<int>& ci = d.ci;
  const std::vector<double>& vv = d.vv;
  const std::string sym = d.symmetric ? "symmetric" : "general";
  const int n = (int)M;
  dspmat* mat = (dspmat*)std::malloc(sizeof(dspmat));
  int* row_size = (int*)std::malloc(sizeof(int));
  int* col_size = (int*)std::malloc(sizeof(int));
  int* nnzp = (int*)std::malloc(sizeof(int));
  int* row = (int*)std::calloc((size_t)n + 1, sizeof(int));
  int* col = (int*)std::malloc(sizeof(int) * (nz > 0 ? nz : 1));
  double* val = (double*)std::malloc(sizeof(double) * (nz > 0 ? nz : 1));
  if (!mat || !row_size || !col_size || !nnzp || !row || !col || !val) {
    std::free(mat); std::free(row_size); std::free(col_size); std::free(nnzp);
    std::free(row); std::free(col); std::free(val);
    return nullptr;
  }
  for (long long k = 0; k < nz; ++k) row[ri[k] + 1]++;
  for (int i = 0; i < n; ++i) row[i + 1] += row[i];
  std::vector<int> pos(row, row + n);
  for (long long k = 0; k < nz; ++k) {
    const int p = pos[ri[k]]++;
    col[p] = ci[k];
    val[p] = vv[k];
  }
  *row_size = n;
  *col_size = (int)N;
  *nnzp = (int)nz;
  mat->row = row;
  mat->col = col;
  mat->nnz = nnzp;
  mat->row_size = row_size;
  mat->col_size = col_size;
  mat->value = val;
  mat->format = (char*)"csr";
  mat->type = (char*)(sym == "symmetric" ? "symmetric" : "unsymmetric");
  return mat;
}
