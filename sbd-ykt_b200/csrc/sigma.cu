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

#include <cstdint>
#include <type_traits>

namespace sbdx {

namespace {

constexpr int kSameThreads = 256;

template <typename T> struct Prec;
template <> struct Prec<double> { using V = double; };
template <> struct Prec<float> { using V = float; };

// ---- v2 kernels ----------------------------------------------------------------

template <typename T, int VEC> struct VecIO;
template <> struct VecIO<double, 1> {
  static __device__ __forceinline__ void load(const double* p, double* o) { o[0] = __ldg(p); }
};
template <> struct VecIO<double, 2> {
  static __device__ __forceinline__ void load(const double* p, double* o) {
    const double2 v = __ldg(reinterpret_cast<const double2*>(p));
    o[0] = v.x; o[1] = v.y;
  }
};
template <> struct VecIO<double, 4> {
  static __device__ __forceinline__ void load(const double* p, double* o) {
    const double2 v = __ldg(reinterpret_cast<const double2*>(p));
    const double2 w = __ldg(reinterpret_cast<const double2*>(p) + 1);
    o[0] = v.x; o[1] = v.y; o[2] = w.x; o[3] = w.y;
  }
};
template <> struct VecIO<float, 1> {
  static __device__ __forceinline__ void load(const float* p, double* o) { o[0] = (double)__ldg(p); }
};
template <> struct VecIO<float, 2> {
  static __device__ __forceinline__ void load(const float* p, double* o) {
    const float2 v = __ldg(reinterpret_cast<const float2*>(p));
    o[0] = v.x; o[1] = v.y;
  }
};
template <> struct VecIO<float, 4> {
  static __device__ __forceinline__ void load(const float* p, double* o) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
  }
};

// Same-spin excitations, VEC consecutive columns per thread. Grid: x = bra
// row (fastest, so the CTAs resident at one time share one column strip of the
// ket rows and the strip stays in L2), y = column strip of kSameThreads*VEC.
// Requires ncol % VEC == 0 (the host picks VEC accordingly).
template <typename T, int VEC>
__global__ void __launch_bounds__(kSameThreads)
sigma_same_v2_kernel(const T* __restrict__ X, size_t ncol, const uint64_t* __restrict__ other,
                     const uint64_t* __restrict__ off, const uint32_t* __restrict__ nsing,
                     const uint32_t* __restrict__ ket, const typename Prec<T>::V* __restrict__ val,
                     const uint64_t* __restrict__ omask, const uint32_t* __restrict__ info,
                     const typename Prec<T>::V* __restrict__ G, int L, const double* __restrict__ hii,
                     double* __restrict__ Y) {
  using V = typename Prec<T>::V;
  const size_t r = blockIdx.x;
  const size_t c0 = ((size_t)blockIdx.y * kSameThreads + threadIdx.x) * VEC;
  const bool active = c0 < ncol;
  uint64_t o[VEC];
  double acc[VEC];
#pragma unroll
  for (int v = 0; v < VEC; ++v) { o[v] = active ? other[c0 + v] : 0ull; acc[v] = 0.0; }
  if (hii != nullptr && active) {
    double x[VEC];
    VecIO<T, VEC>::load(X + r * ncol + c0, x);
#pragma unroll
    for (int v = 0; v < VEC; ++v) acc[v] = hii[r * ncol + c0 + v] * x[v];
  }
  __shared__ uint32_t s_ket[kSameThreads], s_info[kSameThreads];
  __shared__ uint64_t s_om[kSameThreads];
  __shared__ V s_val[kSameThreads];
  const uint64_t beg = off[r], end = off[r + 1], send = beg + nsing[r];
  for (uint64_t base = beg; base < end; base += kSameThreads) {
    const int cnt = (int)min((uint64_t)kSameThreads, end - base);
    const int nsb = send > base ? (int)min((uint64_t)cnt, send - base) : 0;
    __syncthreads();
    if ((int)threadIdx.x < cnt) {
      const uint64_t e = base + threadIdx.x;
      s_ket[threadIdx.x] = ket[e];
      s_info[threadIdx.x] = info[e];
      s_om[threadIdx.x] = omask[e];
      s_val[threadIdx.x] = val[e];
    }
    __syncthreads();
    if (!active) continue;
    // singles: value + opposite-spin Coulomb sum_{q in other} (ai|qq)
    for (int e = 0; e < nsb; ++e) {
      const uint32_t inf = s_info[e];
      const double hv0 = (double)s_val[e];
      const uint64_t om = s_om[e];
      const V* g = G + (size_t)((inf >> 12) & 0xfffu) * L;
      double x[VEC];
      VecIO<T, VEC>::load(X + (size_t)s_ket[e] * ncol + c0, x);
#pragma unroll
      for (int v = 0; v < VEC; ++v) {
        double hv = hv0;
        uint64_t bits = o[v];
        while (bits) {
          const int q = __ffsll((long long)bits) - 1;
          bits &= bits - 1;
          hv += (double)g[q];
        }
        const uint32_t neg = (uint32_t)popc64(o[v] & om) ^ (inf >> 31);
        acc[v] = fma(flip_sign(hv, neg), x[v], acc[v]);
      }
    }
    // doubles: one popcount per pair
#pragma unroll 2
    for (int e = nsb; e < cnt; ++e) {
      const uint32_t sgn = s_info[e] >> 31;
      const double hv = (double)s_val[e];
      const uint64_t om = s_om[e];
      double x[VEC];
      VecIO<T, VEC>::load(X + (size_t)s_ket[e] * ncol + c0, x);
#pragma unroll
      for (int v = 0; v < VEC; ++v) acc[v] = fma(flip_sign(hv, (uint32_t)popc64(o[v] & om) ^ sgn), x[v], acc[v]);
    }
  }
  if (active) {
#pragma unroll
    for (int v = 0; v < VEC; ++v) Y[r * ncol + c0 + v] = acc[v];
  }
}

constexpr int kAb2Threads = 1024;
constexpr int kAb2Slots = 8;  // beta strings per thread per CTA (register accumulators)

// Alpha single x beta single, v2. One CTA per (bra alpha row ia, chunk of the
// beta order). R ket rows C[ja, :] of the alpha singles of ia and their
// integral rows (ai|..) are staged in shared memory per pass; each thread owns
// up to kAb2Slots bra beta strings (taken from the list-length order) and
// walks their beta-single records once per pass, applying each record to all
// R staged rows. Sign: alpha factor s_a (-1)^{|beta(ib) & [lo_a,hi_a)|} per
// (thread, row) and beta factor s_b (-1)^{|alpha(ja) & (lo_b,hi_b]|} per pair,
// the latter from the prefix-parity word of alpha(ja).
template <typename T, int R>
__global__ void __launch_bounds__(kAb2Threads, 1)
sigma_ab_v2_kernel(const T* __restrict__ X, size_t nb, const uint64_t* __restrict__ astr,
                   const uint64_t* __restrict__ bstr, const uint64_t* __restrict__ a_off,
                   const uint32_t* __restrict__ a_nsing, const uint32_t* __restrict__ a_ket,
                   const uint32_t* __restrict__ a_info, const uint64_t* __restrict__ a_omask,
                   const uint64_t* __restrict__ b_off, const uint32_t* __restrict__ b_nsing,
                   const uint64_t* __restrict__ b_rec, const uint32_t* __restrict__ b_order,
                   const typename Prec<T>::V* __restrict__ eri, int npair, size_t xstride,
                   double* __restrict__ Y) {
  using V = typename Prec<T>::V;
  extern __shared__ __align__(16) unsigned char smem[];
  T* xs = reinterpret_cast<T*>(smem);                                  // [R][xstride]
  V* erow = reinterpret_cast<V*>(smem + sizeof(T) * xstride * R);     // [R][npair]
  __shared__ uint64_t s_P[R], s_M[R];
  __shared__ uint32_t s_sa[R];
  const size_t ia = blockIdx.x;
  const size_t chunk0 = (size_t)blockIdx.y * kAb2Threads * kAb2Slots;
  double acc[kAb2Slots];
#pragma unroll
  for (int k = 0; k < kAb2Slots; ++k) acc[k] = 0.0;
  const uint64_t e0 = a_off[ia];
  const int ns = (int)a_nsing[ia];
  for (int k0 = 0; k0 < ns; k0 += R) {
    const int nr = min(R, ns - k0);
    __syncthreads();
    if ((int)threadIdx.x < nr) {
      const uint64_t e = e0 + k0 + threadIdx.x;
      const uint32_t inf = a_info[e];
      s_P[threadIdx.x] = prefix_parity(astr[a_ket[e]]);
      s_M[threadIdx.x] = a_omask[e];
      s_sa[threadIdx.x] = inf >> 31;
    }
    for (int rr = 0; rr < nr; ++rr) {
      const uint64_t e = e0 + k0 + rr;
      const T* xrow = X + (size_t)a_ket[e] * nb;
      T* dst = xs + (size_t)rr * xstride;
      for (size_t t = threadIdx.x; t < nb; t += kAb2Threads) dst[t] = xrow[t];
      const size_t pq = (a_info[e] >> 12) & 0xfffu;
      V* er = erow + (size_t)rr * npair;
      for (int t = threadIdx.x; t < npair; t += kAb2Threads) er[t] = eri[pair2_index(pq, (size_t)t)];
    }
    __syncthreads();
    uint64_t P[R], M[R];
    uint32_t sa[R];
#pragma unroll
    for (int rr = 0; rr < R; ++rr) {
      P[rr] = rr < nr ? s_P[rr] : 0ull;
      M[rr] = rr < nr ? s_M[rr] : 0ull;
      sa[rr] = rr < nr ? s_sa[rr] : 0u;
    }
#pragma unroll
    for (int k = 0; k < kAb2Slots; ++k) {
      const size_t idx = chunk0 + (size_t)k * kAb2Threads + threadIdx.x;
      if (idx >= nb) continue;
      const uint32_t ib = b_order[idx];
      const uint64_t bI = bstr[ib];
      uint32_t base[R];
#pragma unroll
      for (int rr = 0; rr < R; ++rr) base[rr] = sa[rr] ^ (uint32_t)popc64(bI & M[rr]);
      const uint64_t m0 = b_off[ib], m1 = m0 + b_nsing[ib];
      double s = acc[k];
      for (uint64_t m = m0; m < m1; ++m) {
        const uint64_t rec = __ldg(b_rec + m);
        const uint32_t jb = (uint32_t)(rec & 0xffffu);
        const uint32_t pq = (uint32_t)((rec >> 16) & 0xfffu);
        const uint32_t lo = (uint32_t)((rec >> 28) & 63u), hi = (uint32_t)((rec >> 34) & 63u);
        const uint32_t sb = (uint32_t)(rec >> 40);
#pragma unroll
        for (int rr = 0; rr < R; ++rr) {
          if (rr < nr) {
            const uint32_t par = base[rr] ^ sb ^ (uint32_t)((P[rr] >> hi) ^ (P[rr] >> lo));
            const double v = (double)erow[(size_t)rr * npair + pq];
            s = fma(flip_sign(v, par), (double)xs[(size_t)rr * xstride + jb], s);
          }
        }
      }
      acc[k] = s;
    }
  }
#pragma unroll
  for (int k = 0; k < kAb2Slots; ++k) {
    const size_t idx = chunk0 + (size_t)k * kAb2Threads + threadIdx.x;
    if (idx < nb) {
      const uint32_t ib = b_order[idx];
      Y[ia * nb + ib] += acc[k];
    }
  }
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

template <typename T, int VEC>
int launch_same(Ctx* c, const T* X, size_t nrow, size_t ncol, const uint64_t* other, const Conn& cn,
                const typename Prec<T>::V* val, const typename Prec<T>::V* G, const double* hii, double* Y) {
  dim3 grid((unsigned)nrow, (unsigned)((ncol + (size_t)kSameThreads * VEC - 1) / ((size_t)kSameThreads * VEC)));
  sigma_same_v2_kernel<T, VEC><<<grid, kSameThreads, 0, c->stream>>>(X, ncol, other, cn.off, cn.nsing, cn.ket, val,
                                                                      cn.omask, cn.info, G, c->L, hii, Y);
  SBDX_LAUNCHED(c);
  return 0;
}

template <typename T>
int run_same(Ctx* c, const T* X, size_t nrow, size_t ncol, const uint64_t* other, const Conn& cn,
             const typename Prec<T>::V* val, const typename Prec<T>::V* G, const double* hii, double* Y) {
  // widest vector that divides the row length and keeps 16-byte alignment
  constexpr int kWide = sizeof(T) == 8 ? 2 : 4;
  const bool aligned = (reinterpret_cast<uintptr_t>(X) % 16) == 0;
  int vec = c->tune.same_vec > 0 ? c->tune.same_vec : kWide;
  while (vec > 1 && (!aligned || ncol % vec != 0)) vec >>= 1;
  if (vec >= 4) return launch_same<T, 4>(c, X, nrow, ncol, other, cn, val, G, hii, Y);
  if (vec == 2) return launch_same<T, 2>(c, X, nrow, ncol, other, cn, val, G, hii, Y);
  return launch_same<T, 1>(c, X, nrow, ncol, other, cn, val, G, hii, Y);
}

size_t ab2_smem_bytes(size_t nb, size_t tsz, size_t vsz, size_t npair, int R, size_t* stride) {
  const size_t per = 16 / tsz;
  const size_t xstride = (nb + per - 1) / per * per;
  if (stride) *stride = xstride;
  return (size_t)R * (tsz * xstride + vsz * npair);
}

template <typename T, int R>
int launch_ab2(Ctx* c, const T* X, size_t smem, size_t xstride) {
  using V = typename Prec<T>::V;
  const Conn& ca = c->conn[0];
  const Conn& cb = c->conn[1];
  const V* eri = std::is_same<T, double>::value ? (const V*)c->d_eri : (const V*)c->d_eri32;
  SBDX_CUDA(c, cudaFuncSetAttribute(sigma_ab_v2_kernel<T, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const size_t per_cta = (size_t)kAb2Threads * kAb2Slots;
  dim3 grid((unsigned)c->na, (unsigned)((c->nb + per_cta - 1) / per_cta));
  sigma_ab_v2_kernel<T, R><<<grid, kAb2Threads, smem, c->stream>>>(
      X, c->nb, c->d_a, c->d_b, ca.off, ca.nsing, ca.ket, ca.info, ca.omask, cb.off, cb.nsing, cb.srec, cb.order, eri,
      (int)c->npair, xstride, c->d_y);
  SBDX_LAUNCHED(c);
  return 0;
}

template <typename T>
int run_ab(Ctx* c, const T* X) {
  using V = typename Prec<T>::V;
  const size_t budget = 220 * 1024;
  int R = c->tune.ab_rows > 0 ? c->tune.ab_rows : 4;
  size_t stride = 0, smem = 0;
  for (; R >= 1; --R) {
    smem = ab2_smem_bytes(c->nb, sizeof(T), sizeof(V), c->npair, R, &stride);
    if (smem <= budget) break;
  }
  if (R >= 1) {
    if (R >= 4) return launch_ab2<T, 4>(c, X, smem, stride);
    if (R == 3) return launch_ab2<T, 3>(c, X, smem, stride);
    if (R == 2) return launch_ab2<T, 2>(c, X, smem, stride);
    return launch_ab2<T, 1>(c, X, smem, stride);
  }
  c->err = "sigma: beta dimension too large for one shared-memory ket row";
  return 1;
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
  T* xt = reinterpret_cast<T*>(c->d_xt);
  auto mark = [&](int k) {
    if (c->profiling) cudaEventRecord(c->ev[k], c->stream);
  };
  int rc = 0;
  mark(0);
  // 1. alpha excitations + diagonal -> Y
  if ((rc = run_same<T>(c, X, na, nb, c->d_b, ca, valA, G, c->d_hii, c->d_y))) return rc;
  mark(1);
  // 2. C -> C^T
  {
    dim3 grid((unsigned)((nb + 31) / 32), (unsigned)((na + 31) / 32));
    transpose_kernel<T><<<grid, dim3(32, 8), 0, c->stream>>>(X, na, nb, xt);
    SBDX_LAUNCHED(c);
  }
  mark(2);
  // 3. beta excitations on C^T -> Yt
  if ((rc = run_same<T>(c, xt, nb, na, c->d_a, cb, valB, G, nullptr, c->d_yt))) return rc;
  mark(3);
  // 4. alpha single x beta single -> Y +=
  if ((rc = run_ab<T>(c, X))) return rc;
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

// Autotuner: time every candidate (same_vec, ab_rows) on the current problem
// with CUDA events (one warm-up and two timed FP64 sigmas each, on scratch
// vectors) and keep the fastest. The same-spin and alpha-beta choices are
// independent kernels, so they are tuned separately through the phase timers.
int autotune(Ctx* c) {
  int rc = 0;
  if (!c->have_conn && (rc = build_connectivity(c))) return rc;
  if (!c->have_hii && (rc = diag_terms(c))) return rc;
  if ((rc = ensure_sigma_scratch(c))) return rc;
  const size_t D = c->na * c->nb;
  double *X = nullptr, *S = nullptr;
  SBDX_CUDA(c, cudaMallocAsync(&X, sizeof(double) * D, c->stream));
  SBDX_CUDA(c, cudaMallocAsync(&S, sizeof(double) * D, c->stream));
  SBDX_CUDA(c, cudaMemsetAsync(X, 0, sizeof(double) * D, c->stream));
  const bool prof0 = c->profiling;
  const auto saved = c->tune;
  if (!c->ev[0])
    for (auto& e : c->ev) SBDX_CUDA(c, cudaEventCreate(&e));
  c->profiling = true;
  auto measure = [&](int vec, int rows, double* same_ms, double* ab_ms) -> int {
    c->tune.same_vec = vec;
    c->tune.ab_rows = rows;
    int r2 = run_sigma<double>(c, X, S);
    if (r2) return r2;
    for (double& x : c->phase_ms) x = 0.0;
    c->phase_calls = 0;
    for (int k = 0; k < 2; ++k)
      if ((r2 = run_sigma<double>(c, X, S))) return r2;
    *same_ms = c->phase_ms[0] + c->phase_ms[2];
    *ab_ms = c->phase_ms[3];
    return 0;
  };
  int best_vec = 1, best_rows = 1;
  double best_same = 1e300, best_ab = 1e300;
  const int vecs[3] = {1, 2, 4};
  for (int v : vecs) {
    double sm = 0, ab = 0;
    if ((rc = measure(v, 1, &sm, &ab))) break;
    if (sm < best_same) { best_same = sm; best_vec = v; }
  }
  for (int rows = 1; rc == 0 && rows <= 4; ++rows) {
    double sm = 0, ab = 0;
    if ((rc = measure(best_vec, rows, &sm, &ab))) break;
    if (ab < best_ab) { best_ab = ab; best_rows = rows; }
  }
  c->profiling = prof0;
  for (double& x : c->phase_ms) x = 0.0;
  c->phase_calls = 0;
  cudaFreeAsync(X, c->stream);
  cudaFreeAsync(S, c->stream);
  if (rc) { c->tune = saved; return rc; }
  c->tune.same_vec = best_vec;
  c->tune.ab_rows = best_rows;
  SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
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
