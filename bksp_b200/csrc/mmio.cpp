// Matrix Market reader of the bksp API (reference src/read_matrix.c:38-173):
// coordinate real / integer / pattern files, 1-based indices converted to
// 0-based CSR with the entries of each row kept in file order (the
// reference's coo2csr is a stable counting sort by row).  Host file I/O.
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/bksp.h"

namespace {

std::string lower(std::string s) {
  for (char& c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

}  // namespace

extern "C" dspmat* read_matrix_market(char* filename) {
  if (!filename) return nullptr;
  FILE* f = std::fopen(filename, "r");
  if (!f) return nullptr;
  char line[4096];
  if (!std::fgets(line, sizeof(line), f)) { std::fclose(f); return nullptr; }
  char b0[64] = {0}, b1[64] = {0}, b2[64] = {0}, b3[64] = {0}, b4[64] = {0};
  if (std::sscanf(line, "%63s %63s %63s %63s %63s", b0, b1, b2, b3, b4) != 5 ||
      lower(b0) != "%%matrixmarket" || lower(b1) != "matrix" ||
      lower(b2) != "coordinate") {
    std::fclose(f);
    return nullptr;
  }
  const std::string field = lower(b3), sym = lower(b4);
  if (field == "complex") { std::fclose(f); return nullptr; }
  const bool pattern = field == "pattern";
  long long M = 0, N = 0, nz = 0;
  for (;;) {
    if (!std::fgets(line, sizeof(line), f)) { std::fclose(f); return nullptr; }
    if (line[0] == '%') continue;
    if (std::sscanf(line, "%lld %lld %lld", &M, &N, &nz) == 3) break;
    bool blank = true;
    for (char* c = line; *c; ++c) if (!std::isspace((unsigned char)*c)) blank = false;
    if (!blank) { std::fclose(f); return nullptr; }
  }
  if (M <= 0 || N <= 0 || nz < 0 || M > 0x7fffffff || nz > 0x7fffffff) {
    std::fclose(f);
    return nullptr;
  }
  std::vector<int> ri(nz), ci(nz);
  std::vector<double> vv(nz);
  for (long long k = 0; k < nz; ++k) {
    long long i, j;
    double v = 1.0;
    int got = pattern ? std::fscanf(f, "%lld %lld", &i, &j)
                      : std::fscanf(f, "%lld %lld %lf", &i, &j, &v);
    if (got != (pattern ? 2 : 3) || i < 1 || i > M || j < 1 || j > N) {
      std::fclose(f);
      return nullptr;
    }
    ri[k] = (int)(i - 1);
    ci[k] = (int)(j - 1);
    vv[k] = v;
  }
  std::fclose(f);

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
