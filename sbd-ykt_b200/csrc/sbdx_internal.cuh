// Internal definitions of the sbdx CUDA library (not part of the C-ABI).
//
// Data layout in HBM (one context = one Hamiltonian + one alpha x beta basis):
//   strings      uint64 per spin string, bit p = spatial orbital p (L <= 64)
//   vectors      D = na*nb elements, alpha-major: index ia*nb + ib, the same
//                order as the reference (chemistry/tpb/mult.h:487-488)
//   integrals    h: L*L FP64; eri: 8-fold packed (pq|rs) FP64 (+FP32 copy);
//                G: (pq|jj) table [npair x L] for the opposite-spin Coulomb
//                term of single excitations
//   connectivity per spin: CSR over bra strings, each row = singles (ascending
//                ket) then doubles (ascending ket), the order of the
//                reference helper lists (chemistry/tpb/helper.h:132-197,
//                367-437). Per entry: ket index, the same-spin part of the
//                matrix element (FP64 and FP32), the opposite-spin sign mask
//                and a packed info word (see below).
#pragma once
#include <cuda_runtime.h>

#include "sbdx.h"
#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>

namespace sbdx {

// ---- info word of a connectivity entry --------------------------------------
//  bit 31      : same-spin sign is negative
//  bit 30      : single excitation (else double)
//  singles     : bits 0-5 hole i (occupied in ket), 6-11 particle a (occupied
//                in bra), 12-23 packed pair index pq(a,i)
//  doubles     : bits 0-5 i, 6-11 j (ket holes, i<j), 12-17 a, 18-23 b
//                (bra particles, a<b)
constexpr uint32_t kInfoNeg = 1u << 31;
constexpr uint32_t kInfoSingle = 1u << 30;

// Balanced SELL-32 of the single-excitation records whose ket index lies in
// [jb0, jb1). A bra string with more than `cap` such singles is split into
// equal parts ("virtual rows") of at most `cap` records; the split parts come
// first, then the unsplit rows longest first. vrow[v]: the bra string;
// vslot[v] = 1 + partial-sum slot of a split part (0 for an unsplit row).
// The parts of split string s occupy slots split_slot[s] .. split_slot[s+1]-1
// and are summed in that order. Record m of lane l of slice s sits at
// sell[soff[s] + 32m + l]; shorter lists are padded with records that have
// bit 41 set.
struct SellPanel {
  uint64_t* sell = nullptr;        // [soff[nslice]]
  // the same records in 32 bits (bits 0-15 position of the ket in the staged
  // rows, Conn::kpos, relative to the panel's first ket; 16-27 pair index,
  // 28 sign, 29 padding, 30 integral
  // copy), read by the packed alpha-beta kernel in blocks of 4 per lane (a
  // padding record repeats the addresses of a real record of its step):
  // record m of lane l of slice s at sell32[soff4[s] + 128*(m/4) + 4*l + m%4],
  // slen4[s] = slen[s] rounded up to a multiple of 4 (padding records)
  uint32_t* sell32 = nullptr;      // [soff4[nslice]]
  uint64_t* soff4 = nullptr;       // [nslice + 1]
  uint32_t* slen4 = nullptr;       // [nslice]
  uint64_t* soff = nullptr;        // [nslice + 1]
  uint32_t* slen = nullptr;        // [nslice]
  uint32_t* vrow = nullptr;        // [nv]
  uint32_t* vslot = nullptr;       // [nv]
  uint32_t* split_row = nullptr;   // [nsplit]
  uint32_t* split_slot = nullptr;  // [nsplit + 1]
  size_t nslice = 0, nv = 0;
  int nsplit = 0, nslot = 0, cap = 0;
  int slices_per_warp = 8;         // 8, 12 or 16: virtual rows per CTA = 1024 * this
  uint32_t jb0 = 0, jb1 = 0;
};

// Bra strings per block of the blocked same-spin kernel, and the determinant
// counts from which the default launch codes use it (FP64, FP32 storage).
constexpr int kBlkRows = 4;
constexpr size_t kBlkMinDets64 = 2000000, kBlkMinDets32 = 1000000;
constexpr uint32_t kNoRow = 0xffffffffu;

// Blocks of the blocked same-spin kernel over the bra strings [row0, row1)
// of one spin. The strings are ordered by their bit-reversed words (strings
// with the same low-orbital holes and different high-orbital particles side
// by side: their double excitations reach largely the same ket strings; at
// 8000 sampled strings per spin the union of four neighbours' double lists
// holds 0.44 of their entries, against 0.74 in ascending order) and cut into
// blocks of kBlkRows. Per block the union of its strings' double-excitation
// kets, ascending, with one signed same-spin value per string of the block
// (zero where that string does not connect). Singles stay in the CSR.
// Work items {block, first union entry, one past the last, 1 + partial slot
// or 0}, longest first; a block with more union entries than the cap is
// split, its first item also does the diagonal and the singles, and the
// parts' kBlkRows partial rows (ypart[(slot * kBlkRows + r) * ldx ..]) are
// summed in slot order by a fix-up kernel.
struct SameBlocks {
  size_t nblk = 0, nu = 0;
  uint4* rows = nullptr;     // [nblk] bra strings (kNoRow: none)
  uint64_t* uoff = nullptr;  // [nblk + 1]
  uint32_t* uket = nullptr;  // [nu]
  double* uval = nullptr;    // [nu * kBlkRows]
  float* uval32 = nullptr;   // [nu * kBlkRows]
  uint4* item = nullptr;     // [n_item]
  size_t n_item = 0;
  uint4* split = nullptr;    // [n_split]: {block, first slot, parts, 0}
  int n_split = 0, n_part = 0, cap = 0;
  double* ypart = nullptr;   // [n_part * kBlkRows * pad8(ncol)]
};

struct Conn {
  size_t n = 0;          // number of bra strings
  size_t total = 0;      // number of entries
  uint32_t* nsing = nullptr;  // [n]
  uint32_t* ndoub = nullptr;  // [n]
  uint64_t* off = nullptr;    // [n+1] row starts
  uint32_t* ket = nullptr;    // [total]
  double* val = nullptr;      // [total] same-spin part of H_IJ (FP64)
  float* val32 = nullptr;     // [total] FP32 copy
  uint64_t* omask = nullptr;  // [total] opposite-spin parity mask
  uint32_t* info = nullptr;   // [total]
  // compact record of single excitations (doubles slots unused), read by the
  // alpha-beta kernels: ket in bits 0-15 and 42-49 (rec_ket), 16-27 pair
  // index pq(a,i), 28-33 lo, 34-39 hi (lo = min(i,a), hi = max(i,a)), bit 40
  // same-spin sign (bit 41 marks a SELL padding record)
  uint64_t* srec = nullptr;   // [total]
  // opposite-spin sign as boundaries of prefix parities: four 7-bit fields
  // (bits 0-6, 7-13, 14-20, 21-27) hold positions x (0..64) with
  // sign = xor_k parity(other & bits[0, x_k)); bit 31 is the same-spin sign,
  // bit 30 marks a single
  uint32_t* spos = nullptr;   // [total]
  uint32_t* order = nullptr;  // [n] bra strings sorted by singles count (desc)
  // single-excitation records in SELL-32 layout over `order`: slice s covers
  // order[32s .. 32s+31]; record m of lane l sits at sell[soff[s] + 32m + l];
  // shorter lists are padded with records that have bit 41 set (no contribution)
  uint64_t* sell = nullptr;   // [soff[nslice]]
  uint64_t* soff = nullptr;   // [nslice + 1]
  uint32_t* slen = nullptr;   // [nslice] records per lane of each slice
  size_t nslice = 0;
  // balanced SELL-32 panels of the single-excitation records (beta spin only),
  // read by the alpha-first alpha-beta kernels: `bal` covers all ket indices;
  // `panels` (empty unless the packed kernel cannot stage a whole ket row in
  // shared memory) split the ket range into slices that it can.
  SellPanel bal;
  std::vector<SellPanel> panels;
  // (beta spin only) position of ket string k in the packed alpha-beta
  // kernel's staged ket rows: a permutation within aligned groups of 8 chosen
  // to spread every bra string's singles over the shared-memory bank slots;
  // the 32-bit records (SellPanel::sell32) hold positions, the 64-bit ones
  // ket indices
  uint32_t* kpos = nullptr;   // [n]
  // work items of the packed alpha-beta kernel (alpha spin only), one CTA
  // each, longest first: {bra alpha string, first single, one past the last
  // single, 1 + partial-row slot or 0}. A string with more singles than the
  // cap is split into items of at most `item_cap` singles (a multiple of 4)
  // whose partial rows (ypart[slot * nb ..], FP64) are added to the output in
  // slot order by a fix-up kernel; the others write the output directly.
  uint4* ab_item = nullptr;    // [n_item]
  size_t n_item = 0;
  uint4* ab_split = nullptr;   // [n_split]: {string, first slot, parts, 0}
  int n_split = 0, n_part = 0, item_cap = 0;
  double* ypart = nullptr;     // [n_part * pad8(nb)]
  // work items of the alpha-first same-spin kernel (either spin), the same
  // scheme over the row's entries (singles then doubles): {bra string, first
  // entry, one past the last entry, 1 + partial-row slot or 0}. Partial rows
  // are [n_same_part * pad8(ncol)] (ncol = the other spin's string count);
  // every part writes all its columns, and the fix-up assigns their sum.
  uint4* same_item = nullptr;
  size_t n_same_item = 0;
  uint4* same_split = nullptr;
  int n_same_split = 0, n_same_part = 0, same_cap = 0;
  double* same_ypart = nullptr;
  // blocks of the blocked same-spin kernel over the same rows as same_item
  SameBlocks blk;
};

// Largest number of partial-sum slots of split rows (shared memory of the
// alpha-first alpha-beta kernel: 8 bytes each).
constexpr int kMaxSplitSlots = 2048;
// Dynamic shared memory the alpha-beta kernels may use per CTA.
constexpr size_t kAbSmemBudget = 227 * 1024 - 1024;
// n rounded up to a multiple of 8 (row strides of padded vectors and tables).
constexpr size_t pad8(size_t n) { return (n + 7) / 8 * 8; }
// The packed alpha-beta kernel stages its integral row twice: copy 0 at pack
// index pq, copy 1 at ab7_epad(npair) + pq with ab7_epad = 4 (mod 8), i.e.
// four 16-byte bank slots further on, so that a record can read whichever
// copy collides less with the other lanes of its quarter-warp (bit 30 of
// the 32-bit record). Packs of both copies: ab7_er_packs.
constexpr size_t ab7_epad(size_t npair) { return (npair + 3) / 8 * 8 + 4; }
constexpr size_t ab7_er_packs(size_t npair) { return ab7_epad(npair) + npair; }

// Stored Hamiltonian (the reference's method 1): off-diagonal elements in CSR
// over determinant rows, basis phases folded into the values (stored.cu).
struct StoredH {
  uint64_t* rowptr = nullptr;  // [D + 1]
  uint32_t* col = nullptr;     // [nnz] determinant index ja*nb + jb
  double* val = nullptr;       // [nnz] H_IJ
  uint64_t nnz = 0;
};

// Launch shape of the sigma kernels. Codes (also the C-ABI encoding):
//   same-spin: 1/2/4/8 = columns per thread of the prefix-parity-table kernel,
//              11/12/14 = 1/2/4 columns of the popcount kernel
//   alpha-beta: 10*variant + staged rows; variant 1 = shared-memory staging,
//              2 = double-buffered TMA staging, 3 = staging with 512-thread CTAs,
//              4 = staging with SELL-32 records, 0 = L1 gathers (rows 1-4)
struct Tune {
  int same_code = 0;  // 0 = built-in default for the precision
  int ab_code = 0;
};

struct Ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  // integrals
  int L = 0;
  double I0 = 0.0;
  size_t npair = 0, neri = 0;
  double* d_h = nullptr;
  double* d_eri = nullptr;
  float* d_eri32 = nullptr;
  double* d_G = nullptr;
  float* d_G32 = nullptr;
  double* d_V = nullptr;    // unpacked (pq|rs) [npair x vstride], row pq contiguous
  float* d_V32 = nullptr;   // same in FP32, row stride vstride32
  size_t vstride = 0, vstride32 = 0;  // row strides padded to 16 bytes
  int* d_err = nullptr;     // device error word (watchdog timeouts), 0 = ok
  std::vector<double> h_h, h_eri;  // host copies (backward / diag host helpers)
  bool have_integrals = false;
  // strings
  size_t na = 0, nb = 0;
  uint64_t* d_a = nullptr;
  uint64_t* d_b = nullptr;
  std::vector<uint64_t> h_a, h_b;
  bool have_strings = false;
  // connectivity (0 = alpha, 1 = beta)
  Conn conn[2];
  bool have_conn = false;   // the full connectivity (everything the sigma reads)
  bool have_lists = false;  // at least the excitation lists (Conn CSR and per-entry data)
  // a shard of the alpha strings: the work items (same-spin and alpha-beta
  // fields of a Conn, nothing else set) of the output rows [range_a0,
  // range_a1) of a row-range sigma (sigma_rows_device)
  Conn range_conn;
  size_t range_a0 = 0, range_a1 = 0;
  bool have_range = false;
  // diagonal
  double* d_hii = nullptr;
  bool have_hii = false;
  // stored Hamiltonian; when present, every FP64 sigma is its sparse product
  StoredH stored;
  // opposite-spin Coulomb term of single excitations in the alpha-first
  // sigma: Db[pq * db_stride + ib] = sum_{q in beta(ib)} (pq|qq) (alpha
  // singles), Da[pq * da_stride + ia] = sum_{p in alpha(ia)} (pq|pp) (beta
  // singles); FP64 and FP32 copies; built with the connectivity
  double *d_Da = nullptr, *d_Db = nullptr;
  float *d_Da32 = nullptr, *d_Db32 = nullptr;
  size_t da_stride = 0, db_stride = 0;
  // sigma scratch (sized for D): transposed input, FP64 partial outputs
  // The alpha-first sigma keeps its vectors with row strides padded to 8
  // elements (xsa >= nb for the alpha-major ones, xsb >= na for the
  // beta-major ones), so every row starts 32-byte aligned and the same-spin
  // kernels load whole vectors of columns whatever na and nb are.
  void* d_xt = nullptr;     // nb x xsb elements of the widest type used (8 B)
  void* d_xp = nullptr;     // na x xsa elements (8 B): phi o C, the input in the alpha-first basis
  double* d_y = nullptr;    // na x xsa FP64: alpha-major partial sigma
  double* d_yt = nullptr;   // nb x xsb FP64: beta-major partial sigma
  size_t xsa = 0, xsb = 0;
  void* d_io_in = nullptr;  // D FP64 staging for host-buffer entry points
  // the host-buffer sigma's pipeline: alpha-row chunks whose host<->device
  // copies run on io_copy beside the chunks' kernels on the context stream
  // (io_chunks_req: 0 automatic, 1 no pipeline, K >= 2 that many chunks)
  int io_chunks_req = 0;
  std::vector<size_t> io_bounds;  // chunk boundaries, multiples of 8
  std::vector<Conn> io_items;     // work items of each chunk's output rows
  cudaStream_t io_copy = nullptr;
  std::vector<cudaEvent_t> io_events;  // per chunk: input copied, output ready; then one for the last copy
  void* d_io_out = nullptr;
  // the wavefunction of the last Davidson solve, resident on the device:
  // wf_roots vectors of D FP64 (root r at d_wf + r*D), kept until the next
  // solve or until the strings change, so the density, RDM, carry-over
  // weights and adjoint run on it without a device-host round trip
  double* d_wf = nullptr;
  int wf_roots = 0;     // vectors the last solve left (0 = none)
  int wf_cap = 0;       // vectors allocated
  // reductions
  double* d_red = nullptr;  // partial sums
  size_t red_cap = 0;
  // launch statistics (kernels launched by this context since reset)
  unsigned long long launches = 0;
  // launch shapes of the sigma kernels per precision (index 0 = FP64, 1 = FP32)
  Tune tune[2];
  // CUDA graphs of whole sigmas, one per (precision, input, output) buffers,
  // captured on first use and replayed when use_graphs is set (needs a
  // non-default stream); cleared whenever the data they read changes
  struct SigmaGraph {
    int precision;
    const void* X;
    void* S;
    cudaGraphExec_t exec;
    unsigned long long kernels;
  };
  bool use_graphs = false;
  // several-root solves (davidson_roots) run the device-driven solver, one
  // CUDA graph per iteration (sbdx_set_graph_steps)
  bool graph_steps = false;
  bool own_stream = false;  // stream created by the library (destroyed with the context)
  // pool of the solvers' stream-ordered scratch. It keeps its memory between
  // allocations (no unmap/map of gigabytes per solve, which stalls the other
  // streams of a batch); a context that owns it trims it after each solve, a
  // batch shares one pool among its subspaces and trims it after the batch.
  cudaMemPool_t pool = nullptr;
  bool own_pool = false;
  std::vector<SigmaGraph> graphs;
  // optional per-phase timing of the sigma (CUDA events on the context stream)
  bool profiling = false;
  cudaEvent_t ev[8] = {};
  double phase_ms[8] = {};
  unsigned long long phase_calls = 0;
};

}  // namespace sbdx

// The opaque handle of the C-ABI.
struct sbdx_ctx {
  sbdx::Ctx c;
};

namespace sbdx {

constexpr int kSigmaPhases = 5;  // alpha same-spin, transpose, beta same-spin, alpha-beta, combine

// ---- error handling -----------------------------------------------------------
bool set_cuda_err(Ctx* c, cudaError_t e, const char* what);
#define SBDX_CUDA(c, call)                                   \
  do {                                                       \
    cudaError_t e_ = (call);                                 \
    if (e_ != cudaSuccess) {                                 \
      set_cuda_err((c), e_, #call);                          \
      return 2;                                              \
    }                                                        \
  } while (0)
#define SBDX_LAUNCHED(c)                                      \
  do {                                                        \
    ++(c)->launches;                                          \
    cudaError_t e_ = cudaGetLastError();                      \
    if (e_ != cudaSuccess) { set_cuda_err((c), e_, "kernel launch"); return 2; } \
  } while (0)

// ---- device helpers ------------------------------------------------------------
// Ket index of a compact single record (Conn::srec and the SELL records):
// bits 0-15 and 42-49, 24 bits in all (at most 16,777,215 strings per spin).
__host__ __device__ __forceinline__ uint32_t rec_ket(uint64_t r) {
  return (uint32_t)(r & 0xffffu) | ((uint32_t)(r >> 26) & 0xff0000u);
}
__host__ __device__ __forceinline__ uint64_t rec_ket_bits(uint32_t k) {
  return (uint64_t)(k & 0xffffu) | ((uint64_t)(k >> 16) << 42);
}
constexpr size_t kMaxStrings = 16777215;  // strings per spin (24-bit record indices)

__host__ __device__ __forceinline__ uint64_t range_mask(int lo, int hi) {
  // bits [lo, hi) for 0 <= lo <= hi <= 64
  uint64_t h = hi >= 64 ? ~0ull : ((1ull << hi) - 1ull);
  uint64_t l = lo >= 64 ? ~0ull : ((1ull << lo) - 1ull);
  return h & ~l;
}

__host__ __device__ __forceinline__ int pair_index(int p, int q) {
  return p > q ? p * (p + 1) / 2 + q : q * (q + 1) / 2 + p;
}

__host__ __device__ __forceinline__ size_t pair2_index(size_t pq, size_t rs) {
  return pq > rs ? pq * (pq + 1) / 2 + rs : rs * (rs + 1) / 2 + pq;
}

__host__ __device__ __forceinline__ size_t eri_index(int p, int q, int r, int s) {
  return pair2_index((size_t)pair_index(p, q), (size_t)pair_index(r, s));
}

__device__ __forceinline__ int popc64(uint64_t x) { return __popcll(x); }

// Flip the sign of v when bit 0 of neg is set (only the high word changes).
__device__ __forceinline__ double flip_sign(double v, uint32_t neg) {
  return __hiloint2double(__double2hiint(v) ^ (int)(neg << 31), __double2loint(v));
}

// Parity bit of popcount(a & b) for 64-bit words split in 32-bit halves.
__device__ __forceinline__ uint32_t and_parity(uint32_t alo, uint32_t ahi, uint32_t blo, uint32_t bhi) {
  return (uint32_t)(__popc(alo & blo) + __popc(ahi & bhi));
}

// Prefix parity word: bit x = parity of popcount(s & bits[0..x]).
__device__ __forceinline__ uint64_t prefix_parity(uint64_t s) {
  s ^= s << 1; s ^= s << 2; s ^= s << 4; s ^= s << 8; s ^= s << 16; s ^= s << 32;
  return s;
}

// Sign of determinant (alpha, beta) of the reference's interleaved ordering
// (alpha p -> spin orbital 2p, beta p -> 2p+1) relative to the alpha-first
// ordering (all alpha spin orbitals before all beta ones): the parity of the
// number of pairs (alpha p, beta q) with q < p, which is
// parity(beta & prefix_parity(alpha)) up to the basis-wide constant
// (-1)^{n_alpha n_beta}. Returns 1 for a minus sign. With C' = phi o C, every
// sign of H in the alpha-first basis is a pure same-spin sign, and
// H C = phi o (H' C').
__device__ __forceinline__ uint32_t basis_phase(uint64_t alpha_prefix_parity, uint64_t beta) {
  return (uint32_t)__popcll(beta & alpha_prefix_parity) & 1u;
}

// Opposite-spin parity mask of one occupied-range term of the reference
// parity() (chemistry/basic/determinants.h:228-279) for a same-spin pair of
// spatial orbitals x < y of spin `spin`: the opposite-spin orbitals whose
// spin-orbital index lies in [2x+spin, 2y+spin).
__host__ __device__ __forceinline__ uint64_t other_range(int spin, int x, int y) {
  return spin == 0 ? range_mask(x, y) : range_mask(x + 1, y + 1);
}

// ---- internal entry points shared between translation units ------------------
// full = false builds the excitation lists only (what the RDM and adjoint
// kernels read); the sigma entry points need (and rebuild) the full form.
int build_connectivity(Ctx* c, bool full = true);
void free_connectivity(Ctx* c);
// Work items of the output rows [a0, a1) (Ctx::range_conn) and their release.
int build_row_range(Ctx* c, size_t a0, size_t a1);
void free_row_range(Ctx* c);
// The work items of rows [a0, a1) into r, and their release.
int build_range_items(Ctx* c, size_t a0, size_t a1, Conn& r);
void free_range_items(Conn& r);
void free_blocks(SameBlocks& b);
// The host-buffer sigma's chunks (their work items, copy stream, events).
void free_io_chunks(Ctx* c);
// S = H C for host buffers (FP64), the copies overlapped with the kernels.
int sigma_host(Ctx* c, const double* hC, double* hS);
// Rows [a0, a1) of S = H X: X the whole vector (na x nb), S the (a1 - a0) x nb
// output rows; a0 a multiple of 8 (or a0 == a1).
int sigma_rows_device(Ctx* c, int precision, const void* X, void* S, size_t a0, size_t a1);
int project_device(Ctx* c, int precision, const void* V, size_t ldv, int m, const void* X, size_t ldx, int nx,
                   size_t D, double* P);
int build_g_table(Ctx* c);
int build_coulomb_tables(Ctx* c);
int diag_terms(Ctx* c);
// sigma: X (na x nb, type by precision: 0 = FP64, 1 = FP32) -> S (same type)
int sigma_device(Ctx* c, int precision, const void* X, void* S);
// Stored Hamiltonian (stored.cu): build (connectivity and diagonal first),
// release, and its product S = H X in FP64.
int build_stored(Ctx* c);
void release_stored(Ctx* c);
int stored_sigma(Ctx* c, const double* X, double* S);
int ensure_sigma_scratch(Ctx* c);
void clear_sigma_graphs(Ctx* c);
int ensure_reduction(Ctx* c, size_t n);
int autotune(Ctx* c);
// Returns 0, or sets c->err and returns SBDX_ERR_CUDA when a kernel recorded a
// watchdog timeout in the device error word (which is then cleared).
int check_device_error(Ctx* c);
// Stream-ordered allocation from the context's pool (created on first use).
cudaError_t pool_alloc(Ctx* c, void** p, size_t bytes);
// Returns the free memory of an owned pool to the device (syncs the stream).
void pool_trim(Ctx* c);
// A pool that keeps its memory, on `device`.
cudaError_t make_pool(int device, cudaMemPool_t* pool);
// Several lowest roots on device vectors (dW: k vectors of na*nb), see davidson.cu.
int davidson_roots(Ctx* c, const sbdx_davidson_params& p, int k, double* dW, double* E, double* res,
                   sbdx_davidson_info& info);
int lowest_diagonal(Ctx* c, int k, std::vector<size_t>& idx);

// Device error codes written to Ctx::d_err.
constexpr int kErrWatchdogAb = 1;  // alpha-beta kernel: TMA completion wait timed out

}  // namespace sbdx
