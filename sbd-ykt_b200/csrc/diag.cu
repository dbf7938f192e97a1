// Diagonal terms H_II for every determinant of the alpha x beta product basis.
//
// Restates makeQChamDiagTerms / ZeroExcite (reference chemistry/tpb/qcham.h:314-366,
// chemistry/basic/determinants.h:397-421): I0 + sum over occupied spin
// orbitals of h_pp + sum over occupied pairs of [(pp|qq) - delta_spin (pq|qp)].
// The sum separates into E_a(ia) + E_b(ib) + sum_{p in a, q in b} (pp|qq) + I0,
// so two per-string kernels precompute the same-spin energies and, for each
// beta string, the Coulomb row J_b[p] = sum_{q in b} (pp|qq); the determinant
// kernel then needs n_alpha table reads per element and is HBM-write bound
// (8 bytes per determinant).
#include "sbdx_internal.cuh"

#include <algorithm>
#include "sbdx.h"

#include <cstring>
#include <mutex>
#include <string>

namespace sbdx {

namespace {

__global__ void string_energy_kernel(const uint64_t* __restrict__ s, size_t n, int L,
                                     const double* __restrict__ h, const double* __restrict__ eri,
                                     double* __restrict__ E) {
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const uint64_t x = s[k];
  double e = 0.0;
  uint64_t bp = x;
  while (bp) {
    const int p = __ffsll((long long)bp) - 1;
    bp &= bp - 1;
    e += h[(size_t)p * L + p];
    uint64_t bq = bp;  // q > p
    while (bq) {
      const int q = __ffsll((long long)bq) - 1;
      bq &= bq - 1;
      e += eri[eri_index(p, p, q, q)] - eri[eri_index(p, q, q, p)];
    }
  }
  E[k] = e;
}

__global__ void coulomb_row_kernel(const uint64_t* __restrict__ s, size_t n, int L,
                                   const double* __restrict__ eri, double* __restrict__ J) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * (size_t)L) return;
  const size_t k = t / L;
  const int p = (int)(t % L);
  uint64_t bq = s[k];
  double v = 0.0;
  while (bq) {
    const int q = __ffsll((long long)bq) - 1;
    bq &= bq - 1;
    v += eri[eri_index(p, p, q, q)];
  }
  J[t] = v;
}

__global__ void diag_kernel(const uint64_t* __restrict__ a, size_t na, size_t nb, int L, double I0,
                            const double* __restrict__ Ea, const double* __restrict__ Eb,
                            const double* __restrict__ Jb, double* __restrict__ hii) {
  const size_t ib = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ib >= nb) return;
  const double* jrow = Jb + ib * (size_t)L;
  for (size_t ia = blockIdx.y; ia < na; ia += gridDim.y) {  // grid rows stride over the alpha strings
    double v = 0.0;
    uint64_t bp = a[ia];
    while (bp) {
      const int p = __ffsll((long long)bp) - 1;
      bp &= bp - 1;
      v += jrow[p];
    }
    hii[ia * nb + ib] = I0 + Ea[ia] + Eb[ib] + v;
  }
}

}  // namespace

int diag_terms(Ctx* c) {
  if (!c->have_strings || !c->have_integrals) {
    c->err = "diag_terms: set integrals and strings first";
    return 3;
  }
  const size_t na = c->na, nb = c->nb, D = na * nb;
  if (!c->d_hii) SBDX_CUDA(c, cudaMalloc(&c->d_hii, sizeof(double) * D));
  double *Ea = nullptr, *Eb = nullptr, *Jb = nullptr;
  SBDX_CUDA(c, pool_alloc(c, (void**)&Ea, sizeof(double) * na));
  SBDX_CUDA(c, pool_alloc(c, (void**)&Eb, sizeof(double) * nb));
  SBDX_CUDA(c, pool_alloc(c, (void**)&Jb, sizeof(double) * nb * c->L));
  string_energy_kernel<<<(unsigned)((na + 127) / 128), 128, 0, c->stream>>>(c->d_a, na, c->L, c->d_h, c->d_eri, Ea);
  SBDX_LAUNCHED(c);
  string_energy_kernel<<<(unsigned)((nb + 127) / 128), 128, 0, c->stream>>>(c->d_b, nb, c->L, c->d_h, c->d_eri, Eb);
  SBDX_LAUNCHED(c);
  const size_t nj = nb * (size_t)c->L;
  coulomb_row_kernel<<<(unsigned)((nj + 255) / 256), 256, 0, c->stream>>>(c->d_b, nb, c->L, c->d_eri, Jb);
  SBDX_LAUNCHED(c);
  dim3 grid((unsigned)((nb + 255) / 256), (unsigned)std::min<size_t>(na, 65535));  // grid y is at most 65535
  diag_kernel<<<grid, 256, 0, c->stream>>>(c->d_a, na, nb, c->L, c->I0, Ea, Eb, Jb, c->d_hii);
  SBDX_LAUNCHED(c);
  SBDX_CUDA(c, cudaFreeAsync(Ea, c->stream));
  SBDX_CUDA(c, cudaFreeAsync(Eb, c->stream));
  SBDX_CUDA(c, cudaFreeAsync(Jb, c->stream));
  c->have_hii = true;
  return 0;
}

}  // namespace sbdx

// ---- diagonal terms without any device allocation ------------------------------
//
// sbdx_diag_terms_noalloc (include/sbdx.h) computes the same H_II as
// diag_terms() for callers that must not have a library call cudaMalloc or
// cudaFree, for instance code whose device memory all comes from its own
// pre-sized pool. The per-string energies and the beta Coulomb rows that
// diag_terms() puts in stream-ordered pool scratch live instead in the file-scope
// array below, which every GPU that loads the library holds until exit.

namespace sbdx {
namespace {

// Scratch of sbdx_diag_terms_noalloc: E_alpha[na] | E_beta[nb] | J_beta[nb*L].
constexpr size_t kNoAllocScratchDoubles = size_t(1) << 19;  // 4 MiB
static __device__ __align__(256) double g_diag_scratch[kNoAllocScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
double* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_diag_scratch on the current device, looked up once per
// device. On the host the symbol is only a stand-in; kernels must get this
// address.
int scratch_address(int dev, double** out, std::string& err) {
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_diag_scratch);
    if (e != cudaSuccess) {
      err = std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e);
      return SBDX_ERR_CUDA;
    }
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[dev];
  return SBDX_OK;
}

// Variants of the three kernels above that ignore string bits at orbitals >= L
// (the caller's strings are on the device and are not validated on the host).
__global__ void string_energy_masked_kernel(const uint64_t* __restrict__ s, size_t n, int L,
                                            const double* __restrict__ h, const double* __restrict__ eri,
                                            double* __restrict__ E) {
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  uint64_t bp = s[k] & range_mask(0, L);
  double e = 0.0;
  while (bp) {
    const int p = __ffsll((long long)bp) - 1;
    bp &= bp - 1;
    e += h[(size_t)p * L + p];
    uint64_t bq = bp;
    while (bq) {
      const int q = __ffsll((long long)bq) - 1;
      bq &= bq - 1;
      e += eri[eri_index(p, p, q, q)] - eri[eri_index(p, q, q, p)];
    }
  }
  E[k] = e;
}

__global__ void coulomb_row_masked_kernel(const uint64_t* __restrict__ s, size_t n, int L,
                                          const double* __restrict__ eri, double* __restrict__ J) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * (size_t)L) return;
  const int p = (int)(t % L);
  uint64_t bq = s[t / L] & range_mask(0, L);
  double v = 0.0;
  while (bq) {
    const int q = __ffsll((long long)bq) - 1;
    bq &= bq - 1;
    v += eri[eri_index(p, p, q, q)];
  }
  J[t] = v;
}

__global__ void diag_masked_kernel(const uint64_t* __restrict__ a, size_t nb, int L, double I0,
                                   const double* __restrict__ Ea, const double* __restrict__ Eb,
                                   const double* __restrict__ Jb, double* __restrict__ hii) {
  const size_t ia = blockIdx.y;
  const size_t ib = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ib >= nb) return;
  const double* jrow = Jb + ib * (size_t)L;
  double v = 0.0;
  uint64_t bp = a[ia] & range_mask(0, L);
  while (bp) {
    const int p = __ffsll((long long)bp) - 1;
    bp &= bp - 1;
    v += jrow[p];
  }
  hii[ia * nb + ib] = I0 + Ea[ia] + Eb[ib] + v;
}

void put_error(char* buf, size_t len, const std::string& msg) {
  if (!buf || len == 0) return;
  const size_t n = msg.size() < len - 1 ? msg.size() : len - 1;
  std::memcpy(buf, msg.data(), n);
  buf[n] = '\0';
}

}  // namespace
}  // namespace sbdx

extern "C" int sbdx_diag_terms_noalloc(int norb, double I0, const double* d_h, const double* d_eri,
                                       const uint64_t* d_alpha, size_t na, const uint64_t* d_beta, size_t nb,
                                       double* d_hii, void* stream, char* errbuf, size_t errlen) {
  using namespace sbdx;
  try {
    if (norb < 1 || norb > 64) {
      put_error(errbuf, errlen, "diag_terms_noalloc: norb must be in [1, 64]");
      return SBDX_ERR_ARG;
    }
    if (!d_h || !d_eri || !d_alpha || !d_beta || !d_hii) {
      put_error(errbuf, errlen, "diag_terms_noalloc: null pointer");
      return SBDX_ERR_ARG;
    }
    if (na == 0 || nb == 0 || na > 65535) {
      put_error(errbuf, errlen, "diag_terms_noalloc: need 1 <= na <= 65535 and nb >= 1");
      return SBDX_ERR_ARG;
    }
    const size_t need = na + nb + nb * (size_t)norb;
    if (need > kNoAllocScratchDoubles || nb > kNoAllocScratchDoubles) {
      put_error(errbuf, errlen,
                "diag_terms_noalloc: na + nb + nb*norb = " + std::to_string(need) +
                    " exceeds the fixed scratch of " + std::to_string(kNoAllocScratchDoubles) +
                    " doubles; use sbdx_diag_terms");
      return SBDX_ERR_ARG;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
      put_error(errbuf, errlen, "diag_terms_noalloc: no usable current CUDA device");
      return SBDX_ERR_CUDA;
    }
    double* scratch = nullptr;
    std::string err;
    if (scratch_address(dev, &scratch, err) != SBDX_OK) {
      put_error(errbuf, errlen, "diag_terms_noalloc: " + err);
      return SBDX_ERR_CUDA;
    }
    // every scratch word read below is written first in the same call
    double* Ea = scratch;
    double* Eb = Ea + na;
    double* Jb = Eb + nb;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // A launch error that unrelated earlier work left pending on this host
    // thread would otherwise be reported as ours by the check after the
    // launches: clear it first (an error that ruined the context persists and
    // is still reported).
    (void)cudaGetLastError();
    string_energy_masked_kernel<<<(unsigned)((na + 127) / 128), 128, 0, st>>>(d_alpha, na, norb, d_h, d_eri, Ea);
    string_energy_masked_kernel<<<(unsigned)((nb + 127) / 128), 128, 0, st>>>(d_beta, nb, norb, d_h, d_eri, Eb);
    const size_t nj = nb * (size_t)norb;
    coulomb_row_masked_kernel<<<(unsigned)((nj + 255) / 256), 256, 0, st>>>(d_beta, nb, norb, d_eri, Jb);
    dim3 grid((unsigned)((nb + 255) / 256), (unsigned)na);
    diag_masked_kernel<<<grid, 256, 0, st>>>(d_alpha, nb, norb, I0, Ea, Eb, Jb, d_hii);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
      put_error(errbuf, errlen, std::string("diag_terms_noalloc: kernel launch: ") + cudaGetErrorString(e));
      return SBDX_ERR_CUDA;
    }
    return SBDX_OK;
  } catch (...) {
    put_error(errbuf, errlen, "diag_terms_noalloc: unexpected host exception");
    return SBDX_ERR_ARG;
  }
}
