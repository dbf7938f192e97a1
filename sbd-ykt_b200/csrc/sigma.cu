// Sigma = H * C on the fly (Slater-Condon rules), the hot kernel of the path.
//
// Restates mult (reference chemistry/tpb/mult.h:376-632) at world size 1:
//   S = hii o C                                  (diagonal, :439-444)
//     + sum over alpha singles/doubles, same ib  (task type 2, :484-520)
//     + sum over beta singles/doubles, same ia   (task type 1, :522-556)
//     + sum over alpha single x beta single      (task type 0, :558-578)
// with every matrix element recomputed from the strings, as Hij does
// (chemistry/basic/determinants.h:467-526).
//
// B200 form (one sigma = 5 launches):
//   1. same-spin kernel over alpha rows of C: a CTA owns one bra alpha row ia
//      and a strip of beta columns; it walks the connectivity list of ia
//      (staged in shared memory) and streams the ket rows C[ja, strip]
//      coalesced, so every pair costs one 8/4-byte load, one popcount (the
//      beta-dependent sign) and one FMA; hii o C initialises the accumulator.
//   2. transpose C -> C^T (tiled through shared memory)
//   3. the same kernel over beta rows of C^T (beta excitations become row
//      streams too), writing S^T
//   4. alpha-beta kernel: a CTA owns one bra alpha row ia; for each alpha
//      single ja of ia it stages the whole ket row C[ja, :] and the integral
//      row (ai|..) in shared memory, then every thread sums its bra beta
//      strings' beta singles as shared-memory gathers; the sign splits into an
//      alpha factor (once per thread and ja) and a beta factor (per pair)
//   5. S = S_alpha + S_ab + (S^T)^T, converted to the output precision.
// Accumulation is FP64 in every precision mode ("FP64 per-row accumulation");
// FP32 mode reads FP32 vectors and FP32 matrix elements.
#include "sbdx_internal.cuh"

#include <type_traits>

namespace sbdx {

namespace {

constexpr int kSameThreads = 256;
constexpr int kAbThreads = 512;

template <typename T> struct Prec;
template <> struct Prec<double> { using V = double; };
template <> struct Prec<float> { using V = float; };

template <typename T>
__global__ void __launch_bounds__(kSameThreads)
sigma_same_kernel(const T* __restrict__ X, size_t ncol, const uint64_t* __restrict__ other,
                  const uint64_t* __restrict__ off, const uint32_t* __restrict__ ket,
                  const typename Prec<T>::V* __restrict__ val, const uint64_t* __restrict__ omask,
                  const uint32_t* __restrict__ info, const typename Prec<T>::V* __restrict__ G, int L,
                  const double* __restrict__ hii, double* __restrict__ Y) {
  using V = typename Prec<T>::V;
  const size_t r = blockIdx.y;
  const size_t c = (size_t)blockIdx.x * kSameThreads + threadIdx.x;
  const bool active = c < ncol;
  const uint64_t o = active ? other[c] : 0ull;
  double acc = 0.0;
  if (hii != nullptr && active) acc = hii[r * ncol + c] * (double)X[r * ncol + c];
  __shared__ uint32_t s_ket[kSameThreads], s_info[kSameThreads];
  __shared__ uint64_t s_om[kSameThreads];
  __shared__ V s_val[kSameThreads];
  const uint64_t beg = off[r], end = off[r + 1];
  for (uint64_t base = beg; base < end; base += kSameThreads) {
    const int cnt = (int)min((uint64_t)kSameThreads, end - base);
    __syncthreads();
    if ((int)threadIdx.x < cnt) {
      const uint64_t e = base + threadIdx.x;
      s_ket[threadIdx.x] = ket[e];
      s_info[threadIdx.x] = info[e];
      s_om[threadIdx.x] = omask[e];
      s_val[threadIdx.x] = val[e];
    }
    __syncthreads();
    if (active) {
#pragma unroll 4
      for (int e = 0; e < cnt; ++e) {
        const uint32_t inf = s_info[e];
        double hv = (double)s_val[e];
        if (inf & kInfoSingle) {
          // opposite-spin Coulomb term of OneExcite: sum_{q in other} (ai|qq)
          const V* g = G + (size_t)((inf >> 12) & 0xfffu) * L;
          uint64_t bits = o;
          while (bits) {
            const int q = __ffsll((long long)bits) - 1;
            bits &= bits - 1;
            hv += (double)g[q];
          }
        }
        const uint32_t neg = ((uint32_t)popc64(o & s_om[e]) ^ (inf >> 31)) & 1u;
        const double x = (double)X[(size_t)s_ket[e] * ncol + c];
        acc = fma(neg ? -hv : hv, x, acc);
      }
    }
  }
  if (active) Y[r * ncol + c] = acc;
}

template <typename T>
__global__ void __launch_bounds__(kAbThreads)
sigma_ab_kernel(const T* __restrict__ X, size_t nb, const uint64_t* __restrict__ astr,
                const uint64_t* __restrict__ bstr, const uint64_t* __restrict__ a_off,
                const uint32_t* __restrict__ a_nsing, const uint32_t* __restrict__ a_ket,
                const uint32_t* __restrict__ a_info, const uint64_t* __restrict__ a_omask,
                const uint64_t* __restrict__ b_off, const uint32_t* __restrict__ b_nsing,
                const uint32_t* __restrict__ b_ket, const uint32_t* __restrict__ b_info,
                const typename Prec<T>::V* __restrict__ eri, int npair, int ib_tile,
                double* __restrict__ Y) {
  using V = typename Prec<T>::V;
  extern __shared__ __align__(16) unsigned char smem[];
  double* acc = reinterpret_cast<double*>(smem);                       // [ib_tile]
  T* xs = reinterpret_cast<T*>(smem + sizeof(double) * ib_tile);        // [nb]
  V* erow = reinterpret_cast<V*>(reinterpret_cast<unsigned char*>(xs) +
                                 ((sizeof(T) * nb + 15) & ~(size_t)15));  // [npair]
  const size_t ia = blockIdx.x;
  const size_t ib0 = (size_t)blockIdx.y * ib_tile;
  const size_t ib1 = min(nb, ib0 + (size_t)ib_tile);
  for (size_t t = threadIdx.x; t < ib1 - ib0; t += kAbThreads) acc[t] = 0.0;
  const uint64_t e0 = a_off[ia];
  const uint32_t ns = a_nsing[ia];
  for (uint32_t k = 0; k < ns; ++k) {
    const uint64_t e = e0 + k;
    const size_t ja = a_ket[e];
    const uint32_t inf = a_info[e];
    const uint64_t ma = a_omask[e];
    const size_t pq = (inf >> 12) & 0xfffu;
    __syncthreads();
    const T* xrow = X + ja * nb;
    for (size_t t = threadIdx.x; t < nb; t += kAbThreads) xs[t] = xrow[t];
    for (int t = threadIdx.x; t < npair; t += kAbThreads) erow[t] = eri[pair2_index(pq, (size_t)t)];
    __syncthreads();
    const uint64_t aj = astr[ja];
    const uint32_t sa = inf >> 31;
    for (size_t ib = ib0 + threadIdx.x; ib < ib1; ib += kAbThreads) {
      const uint32_t base = sa ^ ((uint32_t)popc64(bstr[ib] & ma) & 1u);
      const uint64_t m0 = b_off[ib], m1 = m0 + b_nsing[ib];
      double s = 0.0;
      for (uint64_t m = m0; m < m1; ++m) {
        const uint32_t jb = b_ket[m];
        const uint32_t i2 = b_info[m];
        const int j = (int)(i2 & 63u), b = (int)((i2 >> 6) & 63u);
        const int lo = j < b ? j : b, hi = j < b ? b : j;
        const uint32_t neg = (base ^ (i2 >> 31) ^ (uint32_t)popc64(aj & range_mask(lo + 1, hi + 1))) & 1u;
        const double v = (double)erow[(i2 >> 12) & 0xfffu];
        s = fma(neg ? -v : v, (double)xs[jb], s);
      }
      acc[ib - ib0] += s;
    }
  }
  __syncthreads();
  for (size_t t = threadIdx.x; t < ib1 - ib0; t += kAbThreads) Y[ia * nb + ib0 + t] += acc[t];
}

template <typename T>
__global__ void transpose_kernel(const T* __restrict__ in, size_t rows, size_t cols, T* __restrict__ out) {
  __shared__ T tile[32][33];
  const size_t c0 = (size_t)blockIdx.x * 32, r0 = (size_t)blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const size_t r = r0 + k, c = c0 + threadIdx.x;
    if (r < rows && c < cols) tile[k][threadIdx.x] = in[r * cols + c];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const size_t c = c0 + k, r = r0 + threadIdx.x;  // out row = c, out col = r
    if (r < rows && c < cols) out[c * rows + r] = tile[threadIdx.x][k];
  }
}

// S[ia, ib] = Y[ia, ib] + Yt[ib, ia], stored in T.
template <typename T>
__global__ void combine_transpose_kernel(const double* __restrict__ Y, const double* __restrict__ Yt,
                                         size_t na, size_t nb, T* __restrict__ S) {
  __shared__ double tile[32][33];
  const size_t ib0 = (size_t)blockIdx.x * 32, ia0 = (size_t)blockIdx.y * 32;
  // load Yt rows ib0.. (cols ia0..) transposed into tile[ia][ib]
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const size_t ib = ib0 + k, ia = ia0 + threadIdx.x;
    if (ib < nb && ia < na) tile[threadIdx.x][k] = Yt[ib * na + ia];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const size_t ia = ia0 + k, ib = ib0 + threadIdx.x;
    if (ia < na && ib < nb) S[ia * nb + ib] = (T)(Y[ia * nb + ib] + tile[k][threadIdx.x]);
  }
}

__global__ void g_table_kernel(const double* __restrict__ eri, int L, size_t npair, double* __restrict__ G,
                               float* __restrict__ G32) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npair * (size_t)L) return;
  const size_t pq = t / L;
  const int q = (int)(t % L);
  const double v = eri[pair2_index(pq, (size_t)pair_index(q, q))];
  G[t] = v;
  G32[t] = (float)v;
}

size_t ab_smem_bytes(size_t nb, size_t tsz, size_t vsz, size_t npair, size_t tile) {
  return sizeof(double) * tile + ((tsz * nb + 15) & ~(size_t)15) + vsz * npair;
}

template <typename T>
int run_sigma(Ctx* c, const T* X, T* S) {
  using V = typename Prec<T>::V;
  const size_t na = c->na, nb = c->nb;
  const Conn& ca = c->conn[0];
  const Conn& cb = c->conn[1];
  const V* valA = std::is_same<T, double>::value ? (const V*)ca.val : (const V*)ca.val32;
  const V* valB = std::is_same<T, double>::value ? (const V*)cb.val : (const V*)cb.val32;
  const V* G = std::is_same<T, double>::value ? (const V*)c->d_G : (const V*)c->d_G32;
  const V* eri = std::is_same<T, double>::value ? (const V*)c->d_eri : (const V*)c->d_eri32;
  T* xt = reinterpret_cast<T*>(c->d_xt);
  auto mark = [&](int k) {
    if (c->profiling) cudaEventRecord(c->ev[k], c->stream);
  };
  mark(0);
  // 1. alpha excitations + diagonal -> Y
  {
    dim3 grid((unsigned)((nb + kSameThreads - 1) / kSameThreads), (unsigned)na);
    sigma_same_kernel<T><<<grid, kSameThreads, 0, c->stream>>>(X, nb, c->d_b, ca.off, ca.ket, valA, ca.omask,
                                                               ca.info, G, c->L, c->d_hii, c->d_y);
    SBDX_LAUNCHED(c);
  }
  mark(1);
  // 2. C -> C^T
  {
    dim3 grid((unsigned)((nb + 31) / 32), (unsigned)((na + 31) / 32));
    transpose_kernel<T><<<grid, dim3(32, 8), 0, c->stream>>>(X, na, nb, xt);
    SBDX_LAUNCHED(c);
  }
  mark(2);
  // 3. beta excitations on C^T -> Yt
  {
    dim3 grid((unsigned)((na + kSameThreads - 1) / kSameThreads), (unsigned)nb);
    sigma_same_kernel<T><<<grid, kSameThreads, 0, c->stream>>>(xt, na, c->d_a, cb.off, cb.ket, valB, cb.omask,
                                                               cb.info, G, c->L, nullptr, c->d_yt);
    SBDX_LAUNCHED(c);
  }
  mark(3);
  // 4. alpha single x beta single -> Y +=
  {
    const size_t budget = 200 * 1024;
    const size_t fixed = ab_smem_bytes(nb, sizeof(T), sizeof(V), c->npair, 0);
    if (fixed + 8 * 32 > budget) {
      c->err = "sigma: beta dimension too large for the shared-memory ket row";
      return 1;
    }
    size_t tile = (budget - fixed) / sizeof(double);
    if (tile > nb) tile = nb;
    const unsigned ntile = (unsigned)((nb + tile - 1) / tile);
    tile = (nb + ntile - 1) / ntile;
    const size_t smem = ab_smem_bytes(nb, sizeof(T), sizeof(V), c->npair, tile);
    SBDX_CUDA(c, cudaFuncSetAttribute(sigma_ab_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((unsigned)na, ntile);
    sigma_ab_kernel<T><<<grid, kAbThreads, smem, c->stream>>>(X, nb, c->d_a, c->d_b, ca.off, ca.nsing, ca.ket,
                                                              ca.info, ca.omask, cb.off, cb.nsing, cb.ket,
                                                              cb.info, eri, (int)c->npair, (int)tile, c->d_y);
    SBDX_LAUNCHED(c);
  }
  mark(4);
  // 5. S = Y + Yt^T
  {
    dim3 grid((unsigned)((nb + 31) / 32), (unsigned)((na + 31) / 32));
    combine_transpose_kernel<T><<<grid, dim3(32, 8), 0, c->stream>>>(c->d_y, c->d_yt, na, nb, S);
    SBDX_LAUNCHED(c);
  }
  mark(5);
  if (c->profiling) {
    SBDX_CUDA(c, cudaEventSynchronize(c->ev[5]));
    for (int k = 0; k < kSigmaPhases; ++k) {
      float ms = 0.f;
      SBDX_CUDA(c, cudaEventElapsedTime(&ms, c->ev[k], c->ev[k + 1]));
      c->phase_ms[k] += ms;
    }
    ++c->phase_calls;
  }
  return 0;
}

}  // namespace

int build_g_table(Ctx* c) {
  const size_t n = c->npair * (size_t)c->L;
  cudaFree(c->d_G);
  cudaFree(c->d_G32);
  c->d_G = nullptr;
  c->d_G32 = nullptr;
  SBDX_CUDA(c, cudaMalloc(&c->d_G, sizeof(double) * n));
  SBDX_CUDA(c, cudaMalloc(&c->d_G32, sizeof(float) * n));
  g_table_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->d_eri, c->L, c->npair, c->d_G, c->d_G32);
  SBDX_LAUNCHED(c);
  return 0;
}

int ensure_sigma_scratch(Ctx* c) {
  const size_t D = c->na * c->nb;
  if (!c->d_xt) SBDX_CUDA(c, cudaMalloc(&c->d_xt, sizeof(double) * D));
  if (!c->d_y) SBDX_CUDA(c, cudaMalloc(&c->d_y, sizeof(double) * D));
  if (!c->d_yt) SBDX_CUDA(c, cudaMalloc(&c->d_yt, sizeof(double) * D));
  return 0;
}

int sigma_device(Ctx* c, int precision, const void* X, void* S) {
  if (!c->have_conn) {
    int rc = build_connectivity(c);
    if (rc) return rc;
  }
  if (!c->have_hii) {
    int rc = diag_terms(c);
    if (rc) return rc;
  }
  int rc = ensure_sigma_scratch(c);
  if (rc) return rc;
  if (precision == 0) return run_sigma<double>(c, (const double*)X, (double*)S);
  if (precision == 1) return run_sigma<float>(c, (const float*)X, (float*)S);
  c->err = "sigma: precision must be SBDX_FP64 or SBDX_FP32";
  return 1;
}

}  // namespace sbdx
