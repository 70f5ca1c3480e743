// Host-visible kernel interface: plain structs shared by the CUDA kernels
// (kernels.cu) and the host solver drivers (*.cpp), plus the launch entry
// points.  Nothing here depends on device code.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace bk {

constexpr int kScalars = 8192;    // FP64 scalar slots per solve
constexpr int kGridCap = 148 * 8; // reduction grid cap (= kMaxBlocks)
constexpr int kNotConverged = -1;
constexpr int kDivergence = -2;
constexpr int kLcMaxIn = 24;   // widest linear combination (inputs)
constexpr int kLcMaxOut = 6;   // widest linear combination (outputs)
constexpr int kMaxDotsApi = 8;
constexpr int kPartRows = 64;  // rows of the per-block partials buffer
// Block-kernel reductions run in two levels: the last block of each group
// of kRedGroup blocks sums the group's partials, the last group the
// groups' sums.  Buffer of `per` doubles per block: kGridCap block rows,
// kRedGroups group rows, then kRedGroups unsigned group tickets (zeroed
// once; each group's last block resets its ticket).
constexpr int kRedGroup = 16;
constexpr int kRedGroups = kGridCap / kRedGroup;
constexpr long long red2_doubles(int per) {
  return (long long)per * (kGridCap + kRedGroups) + kRedGroups;
}
constexpr long long red2_ticket_offset(int per) {
  return (long long)per * (kGridCap + kRedGroups);
}
constexpr int kTileNnz = 2048;  // SpMV row block: max stored entries
constexpr int kTileRows = 256;  // SpMV row block: max rows (= threads)

// Coefficient of one linear-combination term (mirrors Cf in dev_common.cuh).
struct CfH {
  signed char op;   // 0 absent, 1 k, 2 k*S[s], 3 k/S[s], 4 k*S[s]/S[s2],
                    // 5 k*S[s]*S[s2]
  unsigned char pad;
  short s, s2;
  short pad2;
  double k;
};
static inline CfH cf_const(double k) { CfH c{}; c.op = 1; c.k = k; return c; }
static inline CfH cf_slot(short s, double k = 1.0) { CfH c{}; c.op = 2; c.s = s; c.k = k; return c; }
static inline CfH cf_inv(short s, double k = 1.0) { CfH c{}; c.op = 3; c.s = s; c.k = k; return c; }
static inline CfH cf_ratio(short s, short s2, double k = 1.0) {
  CfH c{}; c.op = 4; c.s = s; c.s2 = s2; c.k = k; return c;
}
static inline CfH cf_prod(short s, short s2, double k = 1.0) {
  CfH c{}; c.op = 5; c.s = s; c.s2 = s2; c.k = k; return c;
}

struct CtlH {
  int done, iter, ret, max_iter, hist_cap, trips, trip_cap, hist_len;
  double tol;
  double* hist;
  // Conditional IF node of the captured iteration (runtime.h: cond_block):
  // its handle, set by the epilogue that decides the branch (use_cond != 0).
  unsigned long long cond;
  int use_cond;
  int cond_pad;
  // A second conditional node in the same body (a body that holds two
  // iterations); the deciding epilogue picks one by its a1.
  unsigned long long cond_alt;
};

struct RedH {
  double* part;
  unsigned int* ticket;
  double* S;
  CtlH* ctl;
  short out, epi, a0, a1;
  short guard;   // > 0: the kernel runs only while S[guard] != 0
};

// Diagonal form of a CSR operator whose stored entries lie on at most
// kDiaMax diagonals and whose rows list their columns in ascending order
// (k_spmv_dia.cuh).  nd = 0: the operator has no diagonal form.
constexpr int kDiaMax = 8;
struct DiaH {
  const void* val;             // nd x stride values, diagonal-major, 0 where absent
  const unsigned char* mask;   // per row (stride bytes): bit d = entry on diagonal d stored
  long long stride;            // pad64(n)
  int nd;                      // diagonals in use
  int off[kDiaMax];            // their column offsets j - i, ascending
};

// Sliced-ELL copy of a CSR operator (k_spmv_sell.cuh): slices of 32
// consecutive rows; slice s holds width_s = (ptr[s+1] - ptr[s]) / 32 entry
// columns, stored column-major inside the slice (entry k of the slice's row
// r at ptr[s] + 32 k + r) in each row's CSR order, padded with column -1.
// nslice = 0: none.
struct SellH {
  const int* ptr;     // nslice + 1 entry offsets
  const int* col;
  const void* val;    // same precision as CsrH::val
  int nslice;
};

// Device CSR matrix (one value precision).
struct CsrH {
  const int* rowptr;
  const int* col;
  const void* val;
  const int* rb;
  int n;
  int nrb;
  int variant;   // SpMV kernel variant (kernels.cu: spmv_dispatch)
  DiaH dia;
  int nnz;       // stored entries (host-side byte accounting only)
  SellH sell;
};

// One linear-combination launch: out[o] = sum_i c[o][i] * in[i], terms
// evaluated in input order (first term a product, the rest fused
// multiply-adds), repeated `reps` times with operands flagged in the rep
// masks advanced by `stride` elements per repetition.  `nd` dot products
// between any two of [in..., out...] (post-update values) are reduced into
// the scalar slots.  Lengths are padded lengths (multiple of 64).
template <typename T>
struct LcH {
  const T* in[kLcMaxIn];
  T* out[kLcMaxOut];
  CfH c[kLcMaxOut][kLcMaxIn];
  long long n;
  long long stride;
  int nin, nout, reps;
  unsigned in_rep_mask, out_rep_mask;
  int nd;
  unsigned char dot[kMaxDotsApi][2];
};

// All pairwise dots of m <= kGramMax vectors (k_gram_vec).
constexpr int kGramMax = 9;
template <typename T>
struct GramH {
  const T* v[kGramMax];
  long long n;
  int m;
};

template <typename T>
struct SpmvH {
  const T* x;
  T* y;
  T* y2;
  const T* b;
  const T* w0;
  const T* w1;
  int mode;   // 0: y = A x   1: y = b - A x
  int nd;
  unsigned char dot[kMaxDotsApi][2];   // 0 = y, 1 = b, 2 = w0, 3 = w1
  // A + shift I instead of A (the row sum, then + shift x_i); only the
  // diagonal-form and tile kernels take it (the dispatch picks the tile
  // kernel for the others).
  double shift;
};

// Diagonal-form product with its neighbouring vector updates fused in
// (k_spmv_dia_fused): the input is formed on the fly,
//   x = ca xa + cb xb          (xb null: x = ca xa)
// for every element the rows read, so the update of x needs no pass of its
// own; each row's own x is stored to xe, the product to y, and a second
// own-row update fo = c0 f0 + c1 f1 rides along.  Both combinations round as
// a linear-combination launch would (first term a product, then an FMA), so
// a row's stored x equals the value its neighbours used.  Up to three dots
// of the row values: operand 0 = y, 1 = x, 2 = fo.
template <typename T>
struct SpmvFuseH {
  const T* xa;
  const T* xb;
  CfH ca, cb;
  T* xe;
  T* y;
  const T* f0;
  const T* f1;
  T* fo;
  CfH c0, c1;
  int nd;
  unsigned char dot[3][2];
};
// A must have a diagonal form and every vector must be 16-byte aligned
// (else CudaError through the caller's check: spmv_fused_usable).
bool spmv_fused_usable_d(const CsrH& A, const SpmvFuseH<double>& f);
bool spmv_fused_usable_f(const CsrH& A, const SpmvFuseH<float>& f);
void launch_spmv_fused_d(const CsrH& A, const SpmvFuseH<double>& f,
                         const RedH& rd, cudaStream_t st);
void launch_spmv_fused_f(const CsrH& A, const SpmvFuseH<float>& f,
                         const RedH& rd, cudaStream_t st);

// Programmatic dependent launch is kept off for the kernels of a
// conditional node's body and for the first launch after such a node (a
// programmatic edge joins two kernels only): launch_k (launch_util.h)
// honours these per-thread switches.
inline thread_local bool g_plain_scope = false;   // every launch plain
inline thread_local int g_plain_launches = 0;     // the next n launches plain

// ---- launches (kernels.cu) ----
// Kernel launches issued by this thread (graph replays are added by the
// loop runner: captured body kernels x trips).
long long& launch_count();
// Algorithmic DRAM bytes of this thread's launches of the single-vector
// kernels (SpMV, linear combinations, Gram, precision conversions, the
// preconditioner build): every operand counted once per launch, matrix
// bytes as its storage format holds them.  Graph replays are added like
// launch_count; block and shifted-method kernels are not counted.
long long& byte_count();
// SpMV: VT = matrix value type, T = vector/accumulation type.
void launch_spmv_d(const CsrH& A, const SpmvH<double>& io, const RedH& rd,
                   cudaStream_t st);
void launch_spmv_f(const CsrH& A, const SpmvH<float>& io, const RedH& rd,
                   cudaStream_t st);
void launch_lincomb_d(const LcH<double>& d, const RedH& rd, cudaStream_t st);
void launch_lincomb_f(const LcH<float>& d, const RedH& rd, cudaStream_t st);
// Run only a scalar epilogue (one thread).
void launch_epilogue(const RedH& rd, cudaStream_t st);
void launch_gram_d(const GramH<double>& g, const RedH& rd, cudaStream_t st);
void launch_gram_f(const GramH<float>& g, const RedH& rd, cudaStream_t st);
// Element-wise precision conversions / mixed-precision updates.
void launch_convert_d2f(const double* a, float* b, long long n, cudaStream_t st);
void launch_convert_f2d(const float* a, double* b, long long n, cudaStream_t st);
// Structure scan of an uploaded CSR operator (one thread per row, rows with
// valid row pointers): flags |= kScanBadCol (a column outside [0, n)),
// kScanUnsorted (a row whose columns do not strictly ascend), kScanManyOffs
// (more than kScanOffs distinct column offsets j - i), kScanNoDiag (a row
// without a non-zero stored diagonal entry); the distinct offsets (up to
// kScanOffs, unordered, in off[0..noff)); diag[i] = the row's first stored
// diagonal entry (0 when none).
constexpr int kScanOffs = 9;
enum : int { kScanBadCol = 1, kScanUnsorted = 2, kScanManyOffs = 4, kScanNoDiag = 8 };
struct CsrScanH {
  int flags;
  int noff;
  int off[kScanOffs];
};
// scan: device CsrScanH, initialised by the launch.
void launch_csr_scan(const int* rowptr, const int* col, const double* val, int n,
                     double* diag, CsrScanH* scan, cudaStream_t st);
// Matrix Market file -> CSR on the GPU (kernels_mm.cu).  Coordinates are
// 0-based and in file order; with `mirror`, every off-diagonal entry (i, j)
// also goes to row j (one stored triangle of a symmetric file).
// cnt[r] += entries of row r (cnt zero-filled beforehand).
void launch_coo_count(const int* ri, const int* ci, long long nz, int mirror,
                      int* cnt, cudaStream_t st);
// Places the entries in their rows (any order within a row; key = source
// row << 32 | file index); fill zero-filled beforehand.
void launch_coo_scatter(const int* ri, const int* ci, const double* vv,
                        long long nz, int mirror, const int* rowptr, int* fill,
                        int* col, double* val, long long* key, cudaStream_t st);
// Sorts each row by key (file order) or, with by_col, by (column, key).
void launch_row_sort(const int* rowptr, int n, int by_col, int* col, double* val,
                     long long* key, cudaStream_t st);
// Scatter CSR values into the diagonal form (dval zero-filled beforehand);
// mask != nullptr: also write the row masks.
void launch_csr2dia_d(const CsrH& A, const double* val, double* dval,
                      unsigned char* mask, cudaStream_t st);
void launch_csr2dia_f(const CsrH& A, const float* val, float* dval,
                      unsigned char* mask, cudaStream_t st);
// Fill a sliced-ELL copy (SellH) from the CSR arrays (sptr built by the
// host from the row lengths).
void launch_csr2sell_d(const int* rowptr, const int* col, const double* val,
                       int n, int nslice, const int* sptr, int* scol,
                       double* sval, cudaStream_t st);
void launch_csr2sell_f(const int* rowptr, const int* col, const float* val,
                       int n, int nslice, const int* sptr, int* scol,
                       float* sval, cudaStream_t st);
// Mixed precision: o0 (= o1 = o2 when given) = fl32(in), with the dot
// (w, o0) when nd = 1 (w == nullptr: (o0, o0)); and x64 += t32, y32 = 0.
void launch_mx_d2f(const double* in, float* o0, float* o1, float* o2,
                   const float* w, int nd, long long n, const RedH& rd,
                   cudaStream_t st);
void launch_mx_accum(double* x, const float* t, float* y, long long n,
                     const RedH& rd, cudaStream_t st);
// Fused all-shift update of the shifted methods (k_shift.cuh).
struct ShiftArgsH {
  const double* r;
  const double* p;
  double* x;
  double* xs;
  double* ps;
  long long np;
  int ns, l, j, mode;
  float* ps32;   // non-null: the p_k are stored in FP32 here (ps unused)
};
void launch_shift(const ShiftArgsH& a, const RedH& rd, cudaStream_t st);
// Block methods (k_block.cuh): row-major n x s blocks, s <= 16.
// prec 0: FP64 blocks and values; 1: FP32 blocks and values (A's FP32
// copy), the pointers then pointing to floats.  Dots and Gram products
// accumulate in FP64 either way.
struct SpmmH {
  const double* X;
  double* Y;
  const double* C;
  const double* W;
  double alpha;
  int mode, s, nd;   // mode 0: Y = alpha A X; 1: Y = C + alpha A X;
                     // nd dots: (Y, W), (Y, Y)
  int prec;
};
struct BlkH {
  const double* in[4];
  double* out[2];
  CfH c[2][4];
  short mslot[2][4];
  unsigned char trans[2][4];
  int nin, nout, s;
  long long n;
  int ng;
  unsigned char gram[2][2];
  short gslot[2];
  int nd;
  unsigned char dot[2][2];
  int prec;
};
void launch_spmm(const CsrH& A, const SpmmH& a, const RedH& rd, cudaStream_t st);
// Time the diagonal-form and CSR block products for A at width s once
// (outside stream capture) and cache the faster for launch_spmm.
void spmm_autotune(const CsrH& A, int s, int prec, cudaStream_t st);
// This thread's next launch_spmm calls: 0 the diagonal form where usable,
// 1 CSR, -1 the cached choice.
void spmm_force(int kernel);
void launch_block(const BlkH& a, const RedH& rd, cudaStream_t st);
void launch_cm2rm(const double* cm, double* rm, int n, int s, cudaStream_t st);
void launch_rm2cm(const double* rm, double* cm, int n, int s, cudaStream_t st);
// ---- persistent loop (kernels_persist.cu) ----
// One iteration's launches recorded as operations (run_loop in persistent
// mode) and executed for a whole batch of systems by one cooperative
// kernel: phase k runs operation k of every system that is still
// iterating, its work split into units of kPersistUnit rows/elements over
// the whole grid; a grid barrier separates phases.  Reductions are per
// system: each CTA that worked on a system publishes one partial per dot,
// the last of them sums the partials in CTA-slot order and runs the
// system's scalar epilogue.
constexpr int kPersistThreads = 256;   // threads per CTA
constexpr int kPersistUnit = 1024;     // four rows / elements per thread
constexpr int kPersistMaxSys = 512;
enum : int {
  kOpNone = 0,
  kOpSpmvDiaD, kOpSpmvDiaF,   // diagonal-form SpMV (k_spmv_dia's row order)
  kOpSpmvCsrD, kOpSpmvCsrF,   // CSR SpMV, one thread per row (same order)
  kOpLcD, kOpLcF,             // linear combination (k_lincomb)
  kOpGramD, kOpGramF,         // pairwise Gram products, m <= kPersistGramMax
  kOpMxD2f, kOpMxAccum,       // mixed-precision steps
  kOpEpi,                     // scalar epilogue only
};
constexpr int kPersistGramMax = 5;
struct MxD2fH {
  const double* in;
  float* o0;
  float* o1;
  float* o2;
  const float* w;
  long long n;
  int nd;
};
struct MxAccH {
  double* x;
  const float* t;
  float* y;
  long long n;
};
struct alignas(16) ProgOpH {
  int kind;
  int units;   // work units of kPersistUnit
  RedH rd;
  union U {
    struct { CsrH A; SpmvH<double> io; } sd;
    struct { CsrH A; SpmvH<float> io; } sf;
    LcH<double> ld;
    LcH<float> lf;
    GramH<double> gd;
    GramH<float> gf;
    MxD2fH d2f;
    MxAccH acc;
  } u;
};
// Grid-barrier state of one persistent launch (zeroed before the launch).
struct PBarH {
  unsigned count;
  unsigned gen;
  int err;        // 1: a barrier wait ran out of polls
  int err_phase;  // the phase at which it did
};
// What a phase needs to know of an operation before loading it: its units
// and guard slot.
struct OpHdrH {
  int units;
  int guard;
  const double* S;
};
struct PersistH {
  const ProgOpH* ops;   // [nsys][max_ops]
  const OpHdrH* hdr;    // [nsys][max_ops] (units 0: no operation)
  const int* nops;      // operations per system
  CtlH* const* ctl;     // each system's control block
  int nsys, max_ops;
  PBarH* bar;
  long long spin_limit;   // polls per barrier wait before giving up
  int absent_cta;         // test hook: this CTA never arrives (-1: none)
};
// Recording target of this thread's launch wrappers (null: launch).  The
// wrappers append an operation instead of launching; a wrapper without a
// persistent form throws CudaError.
inline thread_local void* g_prog_rec = nullptr;
void prog_push(const ProgOpH& op);           // runtime.cpp
[[noreturn]] void prog_unsupported(const char* what);
// Vector operands of a recorded operation: 16-byte aligned (else the
// operation has no persistent form).
void prog_require_aligned(const void* p);
// Units of kPersistUnit covering n rows / elements (at least one).
inline int prog_units(long long n) {
  const long long u = (n + kPersistUnit - 1) / kPersistUnit;
  return u < 1 ? 1 : (int)u;
}
// Largest grid the persistent kernel may be launched with on the current
// device (all CTAs resident at once).
int persist_max_grid();
// Cooperative launch of the persistent kernel (grid CTAs of kThreads).
cudaError_t launch_persist(const PersistH& p, int grid, cudaStream_t st);

// Solve start: reset control + ticket, optionally preset S[slot] (slot < 0:
// none).  Scalar preset without host synchronisation.
void launch_ctl_init(CtlH* c, unsigned* ticket, double* S, int iter0,
                     int max_iter, double tol, double* hist, int hist_cap,
                     short slot, double value, cudaStream_t st);
void launch_set_scalar(double* S, short slot, double v, cudaStream_t st);
// Graph while-loop control: keep looping while !done and trips < trip_cap.
void launch_loop_control(CtlH* ctl, unsigned long long handle, int use_handle,
                         cudaStream_t st);

}  // namespace bk
