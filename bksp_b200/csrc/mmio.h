// Matrix Market text parsing shared by the host reader (read_matrix_market)
// and the GPU loader (bksp_gpu_read_matrix_market).
#pragma once

#include <string>
#include <vector>

namespace bk {

struct MmData {
  long long rows = 0, cols = 0;
  bool symmetric = false;      // "symmetric": one triangle stored
  std::vector<int> ri, ci;     // 0-based coordinates, file order
  std::vector<double> vv;      // values (1.0 for "pattern" files; real parts)
  std::vector<double> vi;      // imaginary parts ("complex" files only)
};

// Parses a "matrix coordinate real|integer|pattern general|symmetric" file,
// or, with complex_field, a "matrix coordinate complex ..." file.  The entry
// lines are parsed by several threads (fixed-size chunks split at line ends,
// results concatenated in file order).  False on any error.
bool mm_parse(const char* path, MmData& out, bool complex_field = false);

}  // namespace bk
