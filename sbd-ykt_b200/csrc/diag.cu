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
  const size_t ia = blockIdx.y;
  const size_t ib = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ib >= nb) return;
  const double* jrow = Jb + ib * (size_t)L;
  double v = 0.0;
  uint64_t bp = a[ia];
  while (bp) {
    const int p = __ffsll((long long)bp) - 1;
    bp &= bp - 1;
    v += jrow[p];
  }
  hii[ia * nb + ib] = I0 + Ea[ia] + Eb[ib] + v;
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
  SBDX_CUDA(c, cudaMallocAsync(&Ea, sizeof(double) * na, c->stream));
  SBDX_CUDA(c, cudaMallocAsync(&Eb, sizeof(double) * nb, c->stream));
  SBDX_CUDA(c, cudaMallocAsync(&Jb, sizeof(double) * nb * c->L, c->stream));
  string_energy_kernel<<<(unsigned)((na + 127) / 128), 128, 0, c->stream>>>(c->d_a, na, c->L, c->d_h, c->d_eri, Ea);
  SBDX_LAUNCHED(c);
  string_energy_kernel<<<(unsigned)((nb + 127) / 128), 128, 0, c->stream>>>(c->d_b, nb, c->L, c->d_h, c->d_eri, Eb);
  SBDX_LAUNCHED(c);
  const size_t nj = nb * (size_t)c->L;
  coulomb_row_kernel<<<(unsigned)((nj + 255) / 256), 256, 0, c->stream>>>(c->d_b, nb, c->L, c->d_eri, Jb);
  SBDX_LAUNCHED(c);
  dim3 grid((unsigned)((nb + 255) / 256), (unsigned)na);
  diag_kernel<<<grid, 256, 0, c->stream>>>(c->d_a, na, nb, c->L, c->I0, Ea, Eb, Jb, c->d_hii);
  SBDX_LAUNCHED(c);
  SBDX_CUDA(c, cudaFreeAsync(Ea, c->stream));
  SBDX_CUDA(c, cudaFreeAsync(Eb, c->stream));
  SBDX_CUDA(c, cudaFreeAsync(Jb, c->stream));
  c->have_hii = true;
  return 0;
}

}  // namespace sbdx
