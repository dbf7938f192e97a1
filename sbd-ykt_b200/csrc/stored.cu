// Stored Hamiltonian: the reference's method 1 (chemistry/tpb/sbdiag.h:275-330).
// The reference builds every non-zero H_IJ of its bra block as (ih, jh, hij)
// triplets per task and thread (makeQCham, chemistry/tpb/qcham.h:10-312) and
// multiplies with them (mult, chemistry/tpb/mult.h:13-123): Wb[ih] += hij *
// T[jh] after Wb += hii * T. Here the matrix lives on the device in CSR form:
//   - row I = ia*nb + ib holds, in this order, the alpha same-spin entries of
//     ia (columns ja*nb + ib), the beta same-spin entries of ib (columns
//     ia*nb + jb) and the alpha single x beta single pairs (columns
//     ja*nb + jb), the same elements the on-the-fly sigma evaluates;
//   - the values carry the determinant phases, H_IJ = phi_I phi_J H'_IJ with
//     H' the alpha-first-basis matrix of the sigma kernels, so the product
//     acts on vectors in determinant order with no phase pass;
//   - the diagonal stays in the context's hii vector;
//   - column indices are 32-bit (at most 2^32 - 1 determinants), values
//     FP64: 12 bytes per stored element.
// Building it costs one count kernel, a device prefix sum and one fill kernel
// (a warp per row, coalesced writes). The product is one warp per row, lanes
// over the row's elements, a fixed-order shuffle sum (deterministic): HBM
// bound on the 12 bytes per element; the vector gathers hit L2 for the
// problem sizes a stored matrix fits.
#include "sbdx.h"
#include "sbdx_internal.cuh"

#include <cub/device/device_scan.cuh>

#include <string>

namespace sbdx {
namespace {

constexpr int kStoredThreads = 256;  // 8 rows (warps) per CTA

__global__ void stored_count_kernel(const uint64_t* __restrict__ a_off, const uint32_t* __restrict__ a_ns,
                                    const uint64_t* __restrict__ b_off, const uint32_t* __restrict__ b_ns, size_t na,
                                    size_t nb, uint64_t* __restrict__ cnt) {
  const size_t D = na * nb;
  for (size_t I = (size_t)blockIdx.x * blockDim.x + threadIdx.x; I <= D; I += (size_t)gridDim.x * blockDim.x) {
    if (I == D) { cnt[D] = 0; continue; }
    const size_t ia = I / nb, ib = I - ia * nb;
    cnt[I] = (a_off[ia + 1] - a_off[ia]) + (b_off[ib + 1] - b_off[ib]) + (uint64_t)a_ns[ia] * b_ns[ib];
  }
}

// Same-spin element of entry e (first `ns` entries of the row are singles):
// sign * (value + opposite-spin Coulomb term of a single, table row pq).
__device__ __forceinline__ double same_element(uint32_t inf, double v, bool single, const double* __restrict__ Dt,
                                               size_t dstride, size_t col) {
  if (single) v += Dt[(size_t)((inf >> 12) & 0xfffu) * dstride + col];
  return (inf >> 31) ? -v : v;
}

__global__ void __launch_bounds__(kStoredThreads)
stored_fill_kernel(size_t na, size_t nb, const uint64_t* __restrict__ astr, const uint64_t* __restrict__ bstr,
                   const uint64_t* __restrict__ a_off, const uint32_t* __restrict__ a_ns,
                   const uint32_t* __restrict__ a_ket, const double* __restrict__ a_val,
                   const uint32_t* __restrict__ a_info, const uint64_t* __restrict__ b_off,
                   const uint32_t* __restrict__ b_ns, const uint32_t* __restrict__ b_ket,
                   const double* __restrict__ b_val, const uint32_t* __restrict__ b_info,
                   const double* __restrict__ Da, size_t da_stride, const double* __restrict__ Db, size_t db_stride,
                   const double* __restrict__ V, size_t vstride, const uint64_t* __restrict__ rowptr,
                   uint32_t* __restrict__ col, double* __restrict__ val) {
  const size_t D = na * nb;
  const int lane = threadIdx.x & 31;
  const size_t warps = (size_t)gridDim.x * (blockDim.x >> 5);
  for (size_t I = (size_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); I < D; I += warps) {
    const size_t ia = I / nb, ib = I - ia * nb;
    const uint64_t ppa = prefix_parity(astr[ia]);
    const uint64_t bI = bstr[ib];
    const uint32_t phI = basis_phase(ppa, bI);
    uint64_t out = rowptr[I];
    // alpha same-spin: (ja, ib)
    const uint64_t a0 = a_off[ia], na_e = a_off[ia + 1] - a0, nas = a_ns[ia];
    for (uint64_t k = lane; k < na_e; k += 32) {
      const uint64_t e = a0 + k;
      const uint32_t ja = a_ket[e];
      double v = same_element(a_info[e], a_val[e], k < nas, Db, db_stride, ib);
      if (phI ^ basis_phase(prefix_parity(astr[ja]), bI)) v = -v;
      col[out + k] = (uint32_t)(ja * nb + ib);
      val[out + k] = v;
    }
    out += na_e;
    // beta same-spin: (ia, jb)
    const uint64_t b0 = b_off[ib], nb_e = b_off[ib + 1] - b0, nbs = b_ns[ib];
    for (uint64_t k = lane; k < nb_e; k += 32) {
      const uint64_t e = b0 + k;
      const uint32_t jb = b_ket[e];
      double v = same_element(b_info[e], b_val[e], k < nbs, Da, da_stride, ia);
      if (phI ^ basis_phase(ppa, bstr[jb])) v = -v;
      col[out + k] = (uint32_t)(ia * nb + jb);
      val[out + k] = v;
    }
    out += nb_e;
    // alpha single x beta single: (ja, jb), s_a s_b (a i|b j)
    const uint64_t npairs = nas * nbs;
    for (uint64_t p = lane; p < npairs; p += 32) {
      const uint64_t ka = p / nbs, kb = p - ka * nbs;
      const uint32_t ia_inf = a_info[a0 + ka], ib_inf = b_info[b0 + kb];
      const uint32_t ja = a_ket[a0 + ka], jb = b_ket[b0 + kb];
      double v = V[(size_t)((ia_inf >> 12) & 0xfffu) * vstride + ((ib_inf >> 12) & 0xfffu)];
      const uint32_t flip = (ia_inf >> 31) ^ (ib_inf >> 31) ^ phI ^ basis_phase(prefix_parity(astr[ja]), bstr[jb]);
      col[out + p] = (uint32_t)(ja * nb + jb);
      val[out + p] = flip ? -v : v;
    }
  }
}

// S = hii o X + H_offdiag X, a warp per row. The matrix streams through in
// chunks of 128 elements (four per lane); the columns and values of the next
// chunk, or of the next row's first chunk, are loaded while the vector
// gathers of the current one are in flight, so the stream always has a chunk
// in flight. Partial sums in fixed lane and chunk order, then a fixed
// shuffle tree (deterministic).
__global__ void __launch_bounds__(kStoredThreads)
stored_spmv_kernel(size_t D, const uint64_t* __restrict__ rowptr, const uint32_t* __restrict__ col,
                   const double* __restrict__ val, const double* __restrict__ hii, const double* __restrict__ X,
                   double* __restrict__ S) {
  const int lane = threadIdx.x & 31;
  const size_t warps = (size_t)gridDim.x * (blockDim.x >> 5);
  size_t I = (size_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (I >= D) return;
  uint64_t k0 = rowptr[I], k1 = rowptr[I + 1];
  // the chunk in hand: columns and values of elements k0 + lane + 32 u
  uint32_t c[4];
  double v[4];
  auto fetch = [&](uint64_t base, uint64_t end, uint32_t* cc, double* vv) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint64_t k = base + lane + 32 * u;
      const bool in = k < end;
      cc[u] = in ? __ldg(col + k) : 0u;
      vv[u] = in ? __ldg(val + k) : 0.0;
    }
  };
  fetch(k0, k1, c, v);
  uint64_t k = k0;
  double a[4] = {0.0, 0.0, 0.0, 0.0};
  for (;;) {
    // the gathers of the chunk in hand first (they need only its columns)
    double x[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) x[u] = k + lane + 32 * u < k1 ? __ldg(X + c[u]) : 0.0;
    // the next chunk: the rest of this row, or the next row of this warp
    uint64_t kn = k + 128, e = k1;
    size_t In = I;
    if (kn >= k1) {
      In = I + warps;
      kn = In < D ? rowptr[In] : 0;
      e = In < D ? rowptr[In + 1] : 0;
    }
    uint32_t cn[4];
    double vn[4];
    fetch(kn, e, cn, vn);
#pragma unroll
    for (int u = 0; u < 4; ++u) a[u] = fma(v[u], x[u], a[u]);  // out-of-range lanes add 0 * 0
    if (In != I) {  // row I complete
      double acc = (a[0] + a[1]) + (a[2] + a[3]);
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
      if (lane == 0) S[I] = fma(hii[I], X[I], acc);
      if (In >= D) return;
      I = In;
      k1 = e;
      a[0] = a[1] = a[2] = a[3] = 0.0;
    }
    k = kn;
#pragma unroll
    for (int u = 0; u < 4; ++u) { c[u] = cn[u]; v[u] = vn[u]; }
  }
}

unsigned grid_for(size_t warps_needed) {
  const size_t ctas = (warps_needed + (kStoredThreads / 32) - 1) / (kStoredThreads / 32);
  return (unsigned)std::min<size_t>(std::max<size_t>(ctas, 1), 148ull * 64);
}

}  // namespace

void release_stored(Ctx* c) {
  cudaFree(c->stored.rowptr);
  cudaFree(c->stored.col);
  cudaFree(c->stored.val);
  c->stored = StoredH{};
}

int build_stored(Ctx* c) {
  if (!c->have_conn) { int rc = build_connectivity(c); if (rc) return rc; }
  if (!c->have_hii) { int rc = diag_terms(c); if (rc) return rc; }
  release_stored(c);
  const size_t na = c->na, nb = c->nb, D = na * nb;
  if (D > (size_t)UINT32_MAX) {  // the columns are 32-bit determinant indices
    c->err = "build_hamiltonian: " + std::to_string(D) +
             " determinants exceed the 32-bit column indices of the stored matrix (at most 4294967295)";
    return SBDX_ERR_ARG;
  }
  const Conn& ca = c->conn[0];
  const Conn& cb = c->conn[1];
  StoredH& H = c->stored;
  SBDX_CUDA(c, cudaMalloc(&H.rowptr, sizeof(uint64_t) * (D + 1)));
  {
    uint64_t* cnt = nullptr;  // row lengths, then their exclusive prefix sum into rowptr
    SBDX_CUDA(c, pool_alloc(c, (void**)&cnt, sizeof(uint64_t) * (D + 1)));
    const unsigned g = (unsigned)std::min<size_t>((D + 256) / 256, 148ull * 32);
    stored_count_kernel<<<g, 256, 0, c->stream>>>(ca.off, ca.nsing, cb.off, cb.nsing, na, nb, cnt);
    SBDX_LAUNCHED(c);
    size_t tmp = 0;
    cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, tmp, cnt, H.rowptr, D + 1, c->stream);
    void* dtmp = nullptr;
    if (e == cudaSuccess) e = pool_alloc(c, &dtmp, tmp);
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(dtmp, tmp, cnt, H.rowptr, D + 1, c->stream);
    if (dtmp) cudaFreeAsync(dtmp, c->stream);
    cudaFreeAsync(cnt, c->stream);
    SBDX_CUDA(c, e);
  }
  uint64_t nnz = 0;
  SBDX_CUDA(c, cudaMemcpyAsync(&nnz, H.rowptr + D, sizeof(uint64_t), cudaMemcpyDeviceToHost, c->stream));
  SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
  const size_t n = nnz ? nnz : 1;
  if (cudaMalloc(&H.col, sizeof(uint32_t) * n) != cudaSuccess || cudaMalloc(&H.val, sizeof(double) * n) != cudaSuccess) {
    cudaGetLastError();
    release_stored(c);
    c->err = "build_hamiltonian: the stored matrix (" + std::to_string(nnz) + " elements, " +
             std::to_string((12.0 * (double)nnz + 8.0 * (double)D) / 1e9) + " GB) does not fit in device memory";
    return SBDX_ERR_NOMEM;
  }
  stored_fill_kernel<<<grid_for(D), kStoredThreads, 0, c->stream>>>(
      na, nb, c->d_a, c->d_b, ca.off, ca.nsing, ca.ket, ca.val, ca.info, cb.off, cb.nsing, cb.ket, cb.val, cb.info,
      c->d_Da, c->da_stride, c->d_Db, c->db_stride, c->d_V, c->vstride, H.rowptr, H.col, H.val);
  SBDX_LAUNCHED(c);
  SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
  H.nnz = nnz;
  clear_sigma_graphs(c);
  return 0;
}

int stored_sigma(Ctx* c, const double* X, double* S) {
  const size_t D = c->na * c->nb;
  stored_spmv_kernel<<<grid_for(D), kStoredThreads, 0, c->stream>>>(D, c->stored.rowptr, c->stored.col,
                                                                    c->stored.val, c->d_hii, X, S);
  SBDX_LAUNCHED(c);
  return 0;
}

}  // namespace sbdx
