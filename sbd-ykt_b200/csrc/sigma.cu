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
  uint32_t olo[VEC], ohi[VEC];
  double acc[VEC];
#pragma unroll
  for (int v = 0; v < VEC; ++v) {
    o[v] = active ? other[c0 + v] : 0ull;
    olo[v] = (uint32_t)o[v];
    ohi[v] = (uint32_t)(o[v] >> 32);
    acc[v] = 0.0;
  }
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
      const uint32_t omlo = (uint32_t)om, omhi = (uint32_t)(om >> 32);
      double x[VEC];
      VecIO<T, VEC>::load(X + (size_t)s_ket[e] * ncol + c0, x);
#pragma unroll
      for (int v = 0; v < VEC; ++v)
        acc[v] = fma(flip_sign(hv, and_parity(olo[v], ohi[v], omlo, omhi) + sgn), x[v], acc[v]);
    }
  }
  if (active) {
#pragma unroll
    for (int v = 0; v < VEC; ++v) Y[r * ncol + c0 + v] = acc[v];
  }
}

template <> struct VecIO<double, 8> {
  static __device__ __forceinline__ void load(const double* p, double* o) {
    const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double2 v = __ldg(q + k);
      o[2 * k] = v.x; o[2 * k + 1] = v.y;
    }
  }
};
template <> struct VecIO<float, 8> {
  static __device__ __forceinline__ void load(const float* p, double* o) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    const float4 w = __ldg(reinterpret_cast<const float4*>(p) + 1);
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w; o[4] = w.x; o[5] = w.y; o[6] = w.z; o[7] = w.w;
  }
};

constexpr int kParityRows = 65;  // prefix-parity positions 0..64

// Same-spin excitations, v4. As v2 (VEC consecutive columns per thread,
// rows-fastest grid) but the opposite-spin sign of an entry is read from a
// per-thread table of prefix parities in shared memory: tab[x][t] bit v =
// parity(other[c0+v] & bits[0,x)); an entry's sign for all VEC columns is the
// xor of four table bytes at its boundary positions (spos). No popcount in
// the inner loop.
template <typename T, int VEC>
__global__ void __launch_bounds__(kSameThreads)
sigma_same_v4_kernel(const T* __restrict__ X, size_t ncol, const uint64_t* __restrict__ other,
                     const uint64_t* __restrict__ off, const uint32_t* __restrict__ nsing,
                     const uint32_t* __restrict__ ket, const typename Prec<T>::V* __restrict__ val,
                     const uint32_t* __restrict__ spos, const uint32_t* __restrict__ info,
                     const typename Prec<T>::V* __restrict__ G, int L, const double* __restrict__ hii,
                     double* __restrict__ Y) {
  static_assert(VEC <= 8, "one byte of parity bits per thread");
  using V = typename Prec<T>::V;
  __shared__ uint8_t tab[kParityRows][kSameThreads];
  __shared__ uint32_t s_ket[kSameThreads], s_pos[kSameThreads];
  __shared__ V s_val[kSameThreads];
  const size_t r = blockIdx.x;
  const size_t c0 = ((size_t)blockIdx.y * kSameThreads + threadIdx.x) * VEC;
  const bool active = c0 < ncol;
  uint64_t o[VEC];
  double acc[VEC];
  {
    uint64_t P[VEC];
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
      o[v] = active ? other[c0 + v] : 0ull;
      P[v] = prefix_parity(o[v]);
      acc[v] = 0.0;
    }
    tab[0][threadIdx.x] = 0;
    for (int x = 1; x < kParityRows; ++x) {
      uint32_t b = 0;
#pragma unroll
      for (int v = 0; v < VEC; ++v) b |= (uint32_t)((P[v] >> (x - 1)) & 1ull) << v;
      tab[x][threadIdx.x] = (uint8_t)b;
    }
  }
  if (hii != nullptr && active) {
    double x[VEC];
    VecIO<T, VEC>::load(X + r * ncol + c0, x);
#pragma unroll
    for (int v = 0; v < VEC; ++v) acc[v] = hii[r * ncol + c0 + v] * x[v];
  }
  const uint64_t beg = off[r], end = off[r + 1], send = beg + nsing[r];
  const unsigned t = threadIdx.x;
  for (uint64_t base = beg; base < end; base += kSameThreads) {
    const int cnt = (int)min((uint64_t)kSameThreads, end - base);
    const int nsb = send > base ? (int)min((uint64_t)cnt, send - base) : 0;
    __syncthreads();
    if ((int)t < cnt) {
      const uint64_t e = base + t;
      s_ket[t] = ket[e];
      s_pos[t] = spos[e];
      s_val[t] = val[e];
    }
    __syncthreads();
    if (!active) continue;
    for (int e = 0; e < nsb; ++e) {
      const uint32_t ps = s_pos[e];
      const uint32_t neg = (uint32_t)tab[ps & 127u][t] ^ (uint32_t)tab[(ps >> 7) & 127u][t] ^ ((ps >> 31) ? 0xffu : 0u);
      const uint32_t inf = info[base + e];
      const V* g = G + (size_t)((inf >> 12) & 0xfffu) * L;
      const double hv0 = (double)s_val[e];
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
        acc[v] = fma(flip_sign(hv, neg >> v), x[v], acc[v]);
      }
    }
#pragma unroll 2
    for (int e = nsb; e < cnt; ++e) {
      const uint32_t ps = s_pos[e];
      const uint32_t neg = (uint32_t)tab[ps & 127u][t] ^ (uint32_t)tab[(ps >> 7) & 127u][t] ^
                           (uint32_t)tab[(ps >> 14) & 127u][t] ^ (uint32_t)tab[(ps >> 21) & 127u][t] ^
                           ((ps >> 31) ? 0xffu : 0u);
      const double hv = (double)s_val[e];
      double x[VEC];
      VecIO<T, VEC>::load(X + (size_t)s_ket[e] * ncol + c0, x);
#pragma unroll
      for (int v = 0; v < VEC; ++v) acc[v] = fma(flip_sign(hv, neg >> v), x[v], acc[v]);
    }
  }
  if (active) {
#pragma unroll
    for (int v = 0; v < VEC; ++v) Y[r * ncol + c0 + v] = acc[v];
  }
}

constexpr int kAb2Threads = 1024;
constexpr int kAb2Slots = 8;  // beta strings per thread per CTA (register accumulators)

// Slot k of thread t takes position k*nthreads + t of the list-length order on
// even k and k*nthreads + (nthreads-1-t) on odd k, so every thread's lists add
// up to about the same length (a plain stride gives warp 0 the longest list of
// every slot).
__device__ __forceinline__ size_t snake_index(size_t chunk0, int k, int nthreads, int t) {
  return chunk0 + (size_t)k * nthreads + (size_t)((k & 1) ? (nthreads - 1 - t) : t);
}

// Alpha single x beta single, v2. One CTA per (bra alpha row ia, chunk of the
// beta order). R ket rows C[ja, :] of the alpha singles of ia and their
// integral rows (ai|..) are staged in shared memory per pass; each thread owns
// up to kAb2Slots bra beta strings (taken from the list-length order) and
// walks their beta-single records once per pass, applying each record to all
// R staged rows. Sign: alpha factor s_a (-1)^{|beta(ib) & [lo_a,hi_a)|} per
// (thread, row) and beta factor s_b (-1)^{|alpha(ja) & (lo_b,hi_b]|} per pair,
// the latter from the prefix-parity word of alpha(ja).
template <typename T, int R, int NT>
__global__ void __launch_bounds__(NT, 1024 / NT)
sigma_ab_v2_kernel(const T* __restrict__ X, size_t nb, const uint64_t* __restrict__ astr,
                   const uint64_t* __restrict__ bstr, const uint64_t* __restrict__ a_off,
                   const uint32_t* __restrict__ a_nsing, const uint32_t* __restrict__ a_ket,
                   const uint32_t* __restrict__ a_info, const uint64_t* __restrict__ a_omask,
                   const uint64_t* __restrict__ b_off, const uint32_t* __restrict__ b_nsing,
                   const uint64_t* __restrict__ b_rec, const uint32_t* __restrict__ b_order,
                   const typename Prec<T>::V* __restrict__ eri, int npair, size_t xstride,
                   double* __restrict__ Y) {
  using V = typename Prec<T>::V;
  constexpr int kSlots = 8192 / NT;
  extern __shared__ __align__(16) unsigned char smem[];
  T* xs = reinterpret_cast<T*>(smem);                                  // [R][xstride]
  V* erow = reinterpret_cast<V*>(smem + sizeof(T) * xstride * R);     // [R][npair]
  __shared__ uint64_t s_P[R], s_M[R];
  __shared__ uint32_t s_sa[R];
  const size_t ia = blockIdx.x;
  const size_t chunk0 = (size_t)blockIdx.y * NT * kSlots;
  double acc[kSlots];
#pragma unroll
  for (int k = 0; k < kSlots; ++k) acc[k] = 0.0;
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
      for (size_t t = threadIdx.x; t < nb; t += NT) dst[t] = xrow[t];
      const size_t pq = (a_info[e] >> 12) & 0xfffu;
      V* er = erow + (size_t)rr * npair;
      for (int t = threadIdx.x; t < npair; t += NT) er[t] = eri[pair2_index(pq, (size_t)t)];
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
    for (int k = 0; k < kSlots; ++k) {
      const size_t idx = snake_index(chunk0, k, NT, threadIdx.x);
      if (idx >= nb) continue;
      const uint32_t ib = b_order[idx];
      const uint64_t bI = bstr[ib];
      uint32_t base[R];
#pragma unroll
      for (int rr = 0; rr < R; ++rr) base[rr] = sa[rr] ^ (uint32_t)popc64(bI & M[rr]);
      const uint64_t m0 = b_off[ib], m1 = m0 + b_nsing[ib];
      double s = acc[k];
      uint64_t next = m0 < m1 ? __ldg(b_rec + m0) : 0ull;
      for (uint64_t m = m0; m < m1; ++m) {
        const uint64_t rec = next;
        if (m + 1 < m1) next = __ldg(b_rec + m + 1);
        const uint32_t jb = rec_ket(rec);
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
  for (int k = 0; k < kSlots; ++k) {
    const size_t idx = snake_index(chunk0, k, NT, threadIdx.x);
    if (idx < nb) {
      const uint32_t ib = b_order[idx];
      Y[ia * nb + ib] += acc[k];
    }
  }
}

// Alpha single x beta single, v5: the v2 staging scheme with the beta-single
// records read in SELL-32 layout. Warp w of the CTA owns slices w, 63-w,
// 64+w, ... (a snake over the length-sorted slices, so warps get equal work);
// lane l of a slice owns bra beta string order[32s+l]. Every record load of a
// warp is one contiguous 256-byte read; padded records contribute zero.
template <typename T, int R, int NT>
__global__ void __launch_bounds__(NT, 1024 / NT)
sigma_ab_v5_kernel(const T* __restrict__ X, size_t nb, const uint64_t* __restrict__ astr,
                   const uint64_t* __restrict__ bstr, const uint64_t* __restrict__ a_off,
                   const uint32_t* __restrict__ a_nsing, const uint32_t* __restrict__ a_ket,
                   const uint32_t* __restrict__ a_info, const uint64_t* __restrict__ a_omask,
                   const uint64_t* __restrict__ sell, const uint64_t* __restrict__ soff,
                   const uint32_t* __restrict__ slen, size_t nslice, const uint32_t* __restrict__ b_order,
                   const typename Prec<T>::V* __restrict__ eri, int npair, size_t xstride,
                   double* __restrict__ Y) {
  using V = typename Prec<T>::V;
  constexpr int kWarps = NT / 32;
  constexpr int kSlices = 8192 / NT;  // slices per warp per CTA (32*kWarps*kSlices = 8192 strings)
  extern __shared__ __align__(16) unsigned char smem[];
  T* xs = reinterpret_cast<T*>(smem);
  V* erow = reinterpret_cast<V*>(smem + sizeof(T) * xstride * R);
  __shared__ uint64_t s_P[R], s_M[R];
  __shared__ uint32_t s_sa[R];
  const size_t ia = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t slice0 = (size_t)blockIdx.y * kWarps * kSlices;
  auto slice_of = [&](int k) -> size_t {
    return slice0 + (size_t)k * kWarps + ((k & 1) ? (kWarps - 1 - warp) : warp);
  };
  uint64_t bI[kSlices];
  double acc[kSlices];
#pragma unroll
  for (int k = 0; k < kSlices; ++k) {
    const size_t sl = slice_of(k);
    const size_t pos = sl * 32 + lane;
    bI[k] = (sl < nslice && pos < nb) ? bstr[b_order[pos]] : 0ull;
    acc[k] = 0.0;
  }
  const uint64_t e0 = a_off[ia];
  const int ns = (int)a_nsing[ia];
  for (int k0 = 0; k0 < ns; k0 += R) {
    const int nr = min(R, ns - k0);
    __syncthreads();
    if ((int)threadIdx.x < nr) {
      const uint64_t e = e0 + k0 + threadIdx.x;
      s_P[threadIdx.x] = prefix_parity(astr[a_ket[e]]);
      s_M[threadIdx.x] = a_omask[e];
      s_sa[threadIdx.x] = a_info[e] >> 31;
    }
    for (int rr = 0; rr < nr; ++rr) {
      const uint64_t e = e0 + k0 + rr;
      const T* xrow = X + (size_t)a_ket[e] * nb;
      T* dst = xs + (size_t)rr * xstride;
      for (size_t t = threadIdx.x; t < nb; t += NT) dst[t] = xrow[t];
      const size_t pq = (a_info[e] >> 12) & 0xfffu;
      V* er = erow + (size_t)rr * npair;
      for (int t = threadIdx.x; t < npair; t += NT) er[t] = eri[pair2_index(pq, (size_t)t)];
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
    for (int k = 0; k < kSlices; ++k) {
      const size_t sl = slice_of(k);
      if (sl >= nslice) continue;
      uint32_t base[R];
#pragma unroll
      for (int rr = 0; rr < R; ++rr) base[rr] = sa[rr] ^ (uint32_t)popc64(bI[k] & M[rr]);
      const uint32_t len = slen[sl];
      const uint64_t* rp = sell + soff[sl] + lane;
      double s = acc[k];
      uint64_t next = len ? __ldg(rp) : 0ull;
      for (uint32_t m = 0; m < len; ++m) {
        const uint64_t rec = next;
        if (m + 1 < len) next = __ldg(rp + 32ull * (m + 1));
        const uint32_t jb = rec_ket(rec);
        const uint32_t pq = (uint32_t)((rec >> 16) & 0xfffu);
        const uint32_t lo = (uint32_t)((rec >> 28) & 63u), hi = (uint32_t)((rec >> 34) & 63u);
        const uint32_t sb = (uint32_t)(rec >> 40);
        const bool pad = (rec >> 41) & 1ull;
#pragma unroll
        for (int rr = 0; rr < R; ++rr) {
          if (rr < nr) {
            const uint32_t par = base[rr] ^ sb ^ (uint32_t)((P[rr] >> hi) ^ (P[rr] >> lo));
            const double v = pad ? 0.0 : (double)erow[(size_t)rr * npair + pq];
            s = fma(flip_sign(v, par), (double)xs[(size_t)rr * xstride + jb], s);
          }
        }
      }
      acc[k] = s;
    }
  }
#pragma unroll
  for (int k = 0; k < kSlices; ++k) {
    const size_t sl = slice_of(k);
    const size_t pos = sl * 32 + lane;
    if (sl < nslice && pos < nb) Y[ia * nb + b_order[pos]] += acc[k];
  }
}

// ---- double-buffered TMA staging ---------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait: gives up when the phase has not completed after `limit_ns`
// nanoseconds of the global timer (or 2^26 polls, whichever comes first).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
  const uint64_t t0 = global_ns();
  for (uint32_t it = 0; it < (1u << 26); ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 255u) == 255u && global_ns() - t0 > limit_ns) return false;
  }
  return false;
}
__device__ __forceinline__ void tma_load_1d(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

constexpr uint64_t kWaitLimit = 2000000000ull;  // 2 s

// Alpha single x beta single, v4: as v2, with the R ket rows and integral
// rows of the next group of alpha singles loaded by TMA (cp.async.bulk, one
// issuing thread) into the second of two shared-memory buffers while the
// current group is computed. Requires 16-byte aligned rows (nb*sizeof(T) % 16
// == 0 and a 16-byte aligned X); the host checks this.
template <typename T, int R>
__global__ void __launch_bounds__(kAb2Threads, 1)
sigma_ab_v4_kernel(const T* __restrict__ X, size_t nb, const uint64_t* __restrict__ astr,
                   const uint64_t* __restrict__ bstr, const uint64_t* __restrict__ a_off,
                   const uint32_t* __restrict__ a_nsing, const uint32_t* __restrict__ a_ket,
                   const uint32_t* __restrict__ a_info, const uint64_t* __restrict__ a_omask,
                   const uint64_t* __restrict__ b_off, const uint32_t* __restrict__ b_nsing,
                   const uint64_t* __restrict__ b_rec, const uint32_t* __restrict__ b_order,
                   const typename Prec<T>::V* __restrict__ Vtab, size_t vstride, int* __restrict__ err,
                   double* __restrict__ Y) {
  using V = typename Prec<T>::V;
  extern __shared__ __align__(128) unsigned char smem[];
  const size_t xbytes = sizeof(T) * nb, vbytes = sizeof(V) * vstride;
  const size_t bufbytes = (size_t)R * (xbytes + vbytes);
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ int s_abort;
  const size_t ia = blockIdx.x;
  const size_t chunk0 = (size_t)blockIdx.y * kAb2Threads * kAb2Slots;
  const uint64_t e0 = a_off[ia];
  const int ns = (int)a_nsing[ia];
  const int ngroups = (ns + R - 1) / R;
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_abort = 0;
  }
  __syncthreads();
  auto issue = [&](int g) {  // thread 0 only
    const int b = g & 1;
    const int nr = min(R, ns - g * R);
    unsigned char* buf = smem + (size_t)b * bufbytes;
    mbar_arrive_expect_tx(&bar[b], (uint32_t)(nr * (xbytes + vbytes)));
    for (int rr = 0; rr < nr; ++rr) {
      const uint64_t e = e0 + (uint64_t)g * R + rr;
      const size_t ja = a_ket[e];
      const size_t pq = (a_info[e] >> 12) & 0xfffu;
      tma_load_1d(buf + (size_t)rr * xbytes, X + ja * nb, (uint32_t)xbytes, &bar[b]);
      tma_load_1d(buf + (size_t)R * xbytes + (size_t)rr * vbytes, Vtab + pq * vstride, (uint32_t)vbytes, &bar[b]);
    }
  };
  if (threadIdx.x == 0) {
    if (ngroups > 0) issue(0);
    if (ngroups > 1) issue(1);
  }
  double acc[kAb2Slots];
#pragma unroll
  for (int k = 0; k < kAb2Slots; ++k) acc[k] = 0.0;
  int g_abort = -1;  // group whose wait timed out (the same in every thread)
  for (int g = 0; g < ngroups; ++g) {
    const int b = g & 1;
    const int nr = min(R, ns - g * R);
    if (!mbar_wait_bounded(&bar[b], (uint32_t)((g >> 1) & 1), kWaitLimit)) {
      atomicExch(err, kErrWatchdogAb);
      s_abort = 1;
    }
    __syncthreads();
    if (s_abort) { g_abort = g; break; }
    const T* xs = reinterpret_cast<const T*>(smem + (size_t)b * bufbytes);
    const V* erow = reinterpret_cast<const V*>(smem + (size_t)b * bufbytes + (size_t)R * xbytes);
    uint64_t P[R], M[R];
    uint32_t sa[R];
#pragma unroll
    for (int rr = 0; rr < R; ++rr) {
      const uint64_t e = e0 + (uint64_t)g * R + (rr < nr ? rr : 0);
      const uint32_t inf = __ldg(a_info + e);
      P[rr] = prefix_parity(__ldg(astr + __ldg(a_ket + e)));
      M[rr] = __ldg(a_omask + e);
      sa[rr] = inf >> 31;
    }
#pragma unroll
    for (int k = 0; k < kAb2Slots; ++k) {
      const size_t idx = snake_index(chunk0, k, kAb2Threads, threadIdx.x);
      if (idx >= nb) continue;
      const uint32_t ib = __ldg(b_order + idx);
      const uint64_t bI = __ldg(bstr + ib);
      uint32_t base[R];
#pragma unroll
      for (int rr = 0; rr < R; ++rr) base[rr] = sa[rr] ^ (uint32_t)popc64(bI & M[rr]);
      const uint64_t m0 = __ldg(b_off + ib), m1 = m0 + __ldg(b_nsing + ib);
      double s = acc[k];
      uint64_t next = m0 < m1 ? __ldg(b_rec + m0) : 0ull;
      for (uint64_t m = m0; m < m1; ++m) {
        const uint64_t rec = next;
        if (m + 1 < m1) next = __ldg(b_rec + m + 1);
        const uint32_t jb = rec_ket(rec);
        const uint32_t pq = (uint32_t)((rec >> 16) & 0xfffu);
        const uint32_t lo = (uint32_t)((rec >> 28) & 63u), hi = (uint32_t)((rec >> 34) & 63u);
        const uint32_t sb = (uint32_t)(rec >> 40);
#pragma unroll
        for (int rr = 0; rr < R; ++rr) {
          if (rr < nr) {
            const uint32_t par = base[rr] ^ sb ^ (uint32_t)((P[rr] >> hi) ^ (P[rr] >> lo));
            const double v = (double)erow[(size_t)rr * vstride + pq];
            s = fma(flip_sign(v, par), (double)xs[(size_t)rr * nb + jb], s);
          }
        }
      }
      acc[k] = s;
    }
    __syncthreads();  // buffer b is free again
    if (threadIdx.x == 0 && g + 2 < ngroups) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(g + 2);
    }
  }
  if (g_abort >= 0) {
    // Leave no bulk copy in flight into this CTA's shared memory. The groups
    // still outstanding are g_abort (its wait timed out) and g_abort + 1 when
    // it was issued; group q completes phase (q >> 1) & 1 of barrier q & 1.
    // Groups before g_abort were all waited for, and g_abort + 2 was never
    // issued (issue(g + 2) follows a completed group g).
    if (threadIdx.x == 0)
      for (int q = g_abort; q < min(g_abort + 2, ngroups); ++q)
        mbar_wait_bounded(&bar[q & 1], (uint32_t)((q >> 1) & 1), kWaitLimit);
    return;
  }
#pragma unroll
  for (int k = 0; k < kAb2Slots; ++k) {
    const size_t idx = snake_index(chunk0, k, kAb2Threads, threadIdx.x);
    if (idx < nb) Y[ia * nb + b_order[idx]] += acc[k];
  }
}

constexpr int kAb3Threads = 256;
constexpr int kAb3Slots = 8;

// Alpha single x beta single, v3: no shared-memory staging and no barriers.
// One CTA per (bra alpha row ia, chunk of kAb3Threads*kAb3Slots beta strings
// of the list-length order). Each thread walks the alpha singles of ia in
// groups of R and, for each of its bra beta strings, the beta-single records;
// the ket values C[ja, jb] and the integrals (ai|bj) (row pq(a,i) of the
// unpacked table) are gathered through L1, where the R rows shared by the CTA
// stay resident.
template <typename T, int R>
__global__ void __launch_bounds__(kAb3Threads)
sigma_ab_v3_kernel(const T* __restrict__ X, size_t nb, const uint64_t* __restrict__ astr,
                   const uint64_t* __restrict__ bstr, const uint64_t* __restrict__ a_off,
                   const uint32_t* __restrict__ a_nsing, const uint32_t* __restrict__ a_ket,
                   const uint32_t* __restrict__ a_info, const uint64_t* __restrict__ a_omask,
                   const uint64_t* __restrict__ b_off, const uint32_t* __restrict__ b_nsing,
                   const uint64_t* __restrict__ b_rec, const uint32_t* __restrict__ b_order,
                   const typename Prec<T>::V* __restrict__ V, int npair, double* __restrict__ Y) {
  using VT = typename Prec<T>::V;
  const size_t ia = blockIdx.x;
  const size_t chunk0 = (size_t)blockIdx.y * kAb3Threads * kAb3Slots;
  uint32_t ibs[kAb3Slots];
  uint32_t bIlo[kAb3Slots], bIhi[kAb3Slots];
  double acc[kAb3Slots];
#pragma unroll
  for (int k = 0; k < kAb3Slots; ++k) {
    const size_t idx = chunk0 + (size_t)k * kAb3Threads + threadIdx.x;
    ibs[k] = idx < nb ? b_order[idx] : 0xffffffffu;
    const uint64_t b = idx < nb ? bstr[ibs[k]] : 0ull;
    bIlo[k] = (uint32_t)b;
    bIhi[k] = (uint32_t)(b >> 32);
    acc[k] = 0.0;
  }
  const uint64_t e0 = a_off[ia];
  const int ns = (int)a_nsing[ia];
  for (int k0 = 0; k0 < ns; k0 += R) {
    const int nr = min(R, ns - k0);
    const T* xr[R];
    const VT* vr[R];
    uint64_t P[R];
    uint32_t Mlo[R], Mhi[R], sa[R];
#pragma unroll
    for (int rr = 0; rr < R; ++rr) {
      const uint64_t e = e0 + k0 + (rr < nr ? rr : 0);
      const uint32_t inf = __ldg(a_info + e);
      const uint32_t ja = __ldg(a_ket + e);
      const uint64_t m = __ldg(a_omask + e);
      xr[rr] = X + (size_t)ja * nb;
      vr[rr] = V + (size_t)((inf >> 12) & 0xfffu) * (size_t)npair;
      P[rr] = prefix_parity(__ldg(astr + ja));
      Mlo[rr] = (uint32_t)m;
      Mhi[rr] = (uint32_t)(m >> 32);
      sa[rr] = inf >> 31;
    }
#pragma unroll
    for (int k = 0; k < kAb3Slots; ++k) {
      if (ibs[k] == 0xffffffffu) continue;
      const uint32_t ib = ibs[k];
      uint32_t base[R];
#pragma unroll
      for (int rr = 0; rr < R; ++rr) base[rr] = sa[rr] + and_parity(bIlo[k], bIhi[k], Mlo[rr], Mhi[rr]);
      const uint64_t m0 = __ldg(b_off + ib), m1 = m0 + __ldg(b_nsing + ib);
      double s = acc[k];
      uint64_t next = m0 < m1 ? __ldg(b_rec + m0) : 0ull;
      for (uint64_t m = m0; m < m1; ++m) {
        const uint64_t rec = next;
        if (m + 1 < m1) next = __ldg(b_rec + m + 1);
        const uint32_t jb = rec_ket(rec);
        const uint32_t pq = (uint32_t)((rec >> 16) & 0xfffu);
        const uint32_t lo = (uint32_t)((rec >> 28) & 63u), hi = (uint32_t)((rec >> 34) & 63u);
        const uint32_t sb = (uint32_t)(rec >> 40);
#pragma unroll
        for (int rr = 0; rr < R; ++rr) {
          if (rr < nr) {
            const uint32_t par = base[rr] + sb + (uint32_t)((P[rr] >> hi) ^ (P[rr] >> lo));
            const double v = (double)__ldg(vr[rr] + pq);
            s = fma(flip_sign(v, par), (double)__ldg(xr[rr] + jb), s);
          }
        }
      }
      acc[k] = s;
    }
  }
#pragma unroll
  for (int k = 0; k < kAb3Slots; ++k)
    if (ibs[k] != 0xffffffffu) Y[ia * nb + ibs[k]] += acc[k];
}

__global__ void unpack_eri_kernel(const double* __restrict__ eri, size_t npair, size_t vs, size_t vs32,
                                  double* __restrict__ V, float* __restrict__ V32) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npair * npair) return;
  const size_t r = t / npair, q = t % npair;
  const double v = eri[pair2_index(r, q)];
  V[r * vs + q] = v;
  V32[r * vs32 + q] = (float)v;
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
                const typename Prec<T>::V* val, const typename Prec<T>::V* G, const double* hii, double* Y,
                int kind) {
  dim3 grid((unsigned)nrow, (unsigned)((ncol + (size_t)kSameThreads * VEC - 1) / ((size_t)kSameThreads * VEC)));
  if (kind == 1) {
    sigma_same_v2_kernel<T, VEC <= 4 ? VEC : 4><<<grid, kSameThreads, 0, c->stream>>>(
        X, ncol, other, cn.off, cn.nsing, cn.ket, val, cn.omask, cn.info, G, c->L, hii, Y);
  } else {
    sigma_same_v4_kernel<T, VEC><<<grid, kSameThreads, 0, c->stream>>>(X, ncol, other, cn.off, cn.nsing, cn.ket, val,
                                                                        cn.spos, cn.info, G, c->L, hii, Y);
  }
  SBDX_LAUNCHED(c);
  return 0;
}

template <typename T>
int run_same(Ctx* c, const T* X, size_t nrow, size_t ncol, const uint64_t* other, const Conn& cn,
             const typename Prec<T>::V* val, const typename Prec<T>::V* G, const double* hii, double* Y) {
  // default: popcount kernel x4 for FP64, parity-table kernel x8 for FP32;
  // narrowed to the widest vector that divides the row and keeps 16-byte alignment
  const int code0 = c->tune[sizeof(T) == 8 ? 0 : 1].same_code;
  const int code = code0 > 0 ? code0 : (sizeof(T) == 8 ? 14 : 8);
  const int kind = code >= 10 ? 1 : 0;
  int vec = code % 10;
  const bool aligned = (reinterpret_cast<uintptr_t>(X) % 16) == 0;
  while (vec > 1 && (!aligned || ncol % vec != 0)) vec >>= 1;
  if (vec >= 8 && kind == 0) return launch_same<T, 8>(c, X, nrow, ncol, other, cn, val, G, hii, Y, kind);
  if (vec >= 4) return launch_same<T, 4>(c, X, nrow, ncol, other, cn, val, G, hii, Y, kind);
  if (vec == 2) return launch_same<T, 2>(c, X, nrow, ncol, other, cn, val, G, hii, Y, kind);
  return launch_same<T, 1>(c, X, nrow, ncol, other, cn, val, G, hii, Y, kind);
}

size_t ab2_smem_bytes(size_t nb, size_t tsz, size_t vsz, size_t npair, int R, size_t* stride) {
  const size_t per = 16 / tsz;
  const size_t xstride = (nb + per - 1) / per * per;
  if (stride) *stride = xstride;
  return (size_t)R * (tsz * xstride + vsz * npair);
}

template <typename T, int R>
int launch_ab2(Ctx* c, const T* X, size_t smem, size_t xstride, int threads) {
  using V = typename Prec<T>::V;
  const Conn& ca = c->conn[0];
  const Conn& cb = c->conn[1];
  const V* eri = std::is_same<T, double>::value ? (const V*)c->d_eri : (const V*)c->d_eri32;
  const size_t per_cta = 8192;
  dim3 grid((unsigned)c->na, (unsigned)((c->nb + per_cta - 1) / per_cta));
  if (threads == 512) {
    SBDX_CUDA(c, cudaFuncSetAttribute(sigma_ab_v2_kernel<T, R, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kAbSmemBudget));
    sigma_ab_v2_kernel<T, R, 512><<<grid, 512, smem, c->stream>>>(
        X, c->nb, c->d_a, c->d_b, ca.off, ca.nsing, ca.ket, ca.info, ca.omask, cb.off, cb.nsing, cb.srec, cb.order,
        eri, (int)c->npair, xstride, c->d_y);
    SBDX_LAUNCHED(c);
    return 0;
  }
  SBDX_CUDA(c, cudaFuncSetAttribute(sigma_ab_v2_kernel<T, R, 1024>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kAbSmemBudget));
  sigma_ab_v2_kernel<T, R, 1024><<<grid, 1024, smem, c->stream>>>(
      X, c->nb, c->d_a, c->d_b, ca.off, ca.nsing, ca.ket, ca.info, ca.omask, cb.off, cb.nsing, cb.srec, cb.order, eri,
      (int)c->npair, xstride, c->d_y);
  SBDX_LAUNCHED(c);
  return 0;
}

template <typename T, int R>
int launch_ab3(Ctx* c, const T* X) {
  using V = typename Prec<T>::V;
  const Conn& ca = c->conn[0];
  const Conn& cb = c->conn[1];
  const V* Vt = std::is_same<T, double>::value ? (const V*)c->d_V : (const V*)c->d_V32;
  const size_t vs = std::is_same<T, double>::value ? c->vstride : c->vstride32;
  const size_t per_cta = (size_t)kAb3Threads * kAb3Slots;
  dim3 grid((unsigned)c->na, (unsigned)((c->nb + per_cta - 1) / per_cta));
  sigma_ab_v3_kernel<T, R><<<grid, kAb3Threads, 0, c->stream>>>(
      X, c->nb, c->d_a, c->d_b, ca.off, ca.nsing, ca.ket, ca.info, ca.omask, cb.off, cb.nsing, cb.srec, cb.order, Vt,
      (int)vs, c->d_y);
  SBDX_LAUNCHED(c);
  return 0;
}

template <typename T, int R>
int launch_ab4(Ctx* c, const T* X, size_t smem) {
  using V = typename Prec<T>::V;
  const Conn& ca = c->conn[0];
  const Conn& cb = c->conn[1];
  const V* Vt = std::is_same<T, double>::value ? (const V*)c->d_V : (const V*)c->d_V32;
  const size_t vs = std::is_same<T, double>::value ? c->vstride : c->vstride32;
  SBDX_CUDA(c, cudaFuncSetAttribute(sigma_ab_v4_kernel<T, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kAbSmemBudget));
  const size_t per_cta = (size_t)kAb2Threads * kAb2Slots;
  dim3 grid((unsigned)c->na, (unsigned)((c->nb + per_cta - 1) / per_cta));
  sigma_ab_v4_kernel<T, R><<<grid, kAb2Threads, smem, c->stream>>>(
      X, c->nb, c->d_a, c->d_b, ca.off, ca.nsing, ca.ket, ca.info, ca.omask, cb.off, cb.nsing, cb.srec, cb.order, Vt,
      vs, c->d_err, c->d_y);
  SBDX_LAUNCHED(c);
  return 0;
}

// Double-buffered TMA variant when rows are 16-byte aligned and two buffers of
// at least one row fit; returns 1 (not launched) otherwise.
template <typename T>
int try_ab4(Ctx* c, const T* X, int rows_req) {
  using V = typename Prec<T>::V;
  const size_t xbytes = sizeof(T) * c->nb;
  const size_t vs = std::is_same<T, double>::value ? c->vstride : c->vstride32;
  const size_t vbytes = sizeof(V) * vs;
  if (xbytes % 16 != 0 || (reinterpret_cast<uintptr_t>(X) % 16) != 0) return 1;
  const size_t budget = 200 * 1024;
  int R = rows_req > 0 ? rows_req : 4;
  for (; R >= 1; --R)
    if (2 * (size_t)R * (xbytes + vbytes) <= budget) break;
  if (R < 1) return 1;
  const size_t smem = 2 * (size_t)R * (xbytes + vbytes);
  int rc;
  if (R >= 4) rc = launch_ab4<T, 4>(c, X, smem);
  else if (R == 3) rc = launch_ab4<T, 3>(c, X, smem);
  else if (R == 2) rc = launch_ab4<T, 2>(c, X, smem);
  else rc = launch_ab4<T, 1>(c, X, smem);
  return rc ? -rc : 0;
}

template <typename T, int R>
int launch_ab5(Ctx* c, const T* X, size_t smem, size_t xstride) {
  using V = typename Prec<T>::V;
  const Conn& ca = c->conn[0];
  const Conn& cb = c->conn[1];
  const V* eri = std::is_same<T, double>::value ? (const V*)c->d_eri : (const V*)c->d_eri32;
  constexpr int NT = 1024;
  SBDX_CUDA(c, cudaFuncSetAttribute(sigma_ab_v5_kernel<T, R, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kAbSmemBudget));
  const size_t slices_per_cta = 8192 / 32;
  dim3 grid((unsigned)c->na, (unsigned)((cb.nslice + slices_per_cta - 1) / slices_per_cta));
  sigma_ab_v5_kernel<T, R, NT><<<grid, NT, smem, c->stream>>>(
      X, c->nb, c->d_a, c->d_b, ca.off, ca.nsing, ca.ket, ca.info, ca.omask, cb.sell, cb.soff, cb.slen, cb.nslice,
      cb.order, eri, (int)c->npair, xstride, c->d_y);
  SBDX_LAUNCHED(c);
  return 0;
}

template <typename T>
int run_ab(Ctx* c, const T* X) {
  using V = typename Prec<T>::V;
  const int code0 = c->tune[sizeof(T) == 8 ? 0 : 1].ab_code;
  const int code = code0 > 0 ? code0 : (sizeof(T) == 8 ? 42 : 13);
  const int variant = code / 10;
  const int rows = code % 10 > 0 ? code % 10 : 2;
  if (variant == 2) {  // double-buffered TMA staging, when rows are 16-byte aligned
    const int rc = try_ab4<T>(c, X, rows);
    if (rc <= 0) return -rc;
  }
  if (variant == 0) {
    if (rows >= 4) return launch_ab3<T, 4>(c, X);
    if (rows == 3) return launch_ab3<T, 3>(c, X);
    if (rows == 2) return launch_ab3<T, 2>(c, X);
    return launch_ab3<T, 1>(c, X);
  }
  const int threads = variant == 3 ? 512 : 1024;
  const size_t budget = threads == 512 ? 110 * 1024 : 220 * 1024;
  int R = rows;
  size_t stride = 0, smem = 0;
  for (; R >= 1; --R) {
    smem = ab2_smem_bytes(c->nb, sizeof(T), sizeof(V), c->npair, R, &stride);
    if (smem <= budget) break;
  }
  if (R < 1) {
    c->err = "sigma: beta dimension too large for one shared-memory ket row";
    return 1;
  }
  if (variant == 4) {
    if (R >= 4) return launch_ab5<T, 4>(c, X, smem, stride);
    if (R == 3) return launch_ab5<T, 3>(c, X, smem, stride);
    if (R == 2) return launch_ab5<T, 2>(c, X, smem, stride);
    return launch_ab5<T, 1>(c, X, smem, stride);
  }
  if (R >= 4) return launch_ab2<T, 4>(c, X, smem, stride, threads);
  if (R == 3) return launch_ab2<T, 3>(c, X, smem, stride, threads);
  if (R == 2) return launch_ab2<T, 2>(c, X, smem, stride, threads);
  return launch_ab2<T, 1>(c, X, smem, stride, threads);
}

// ---- alpha-first sigma (v6) -----------------------------------------------------
//
// The sigma is evaluated in the alpha-first determinant ordering: with the
// +-1 basis phase phi (basis_phase), H C = phi o (H' (phi o C)) where every
// sign of H' is a pure same-spin sign. So the same-spin kernels need no
// opposite-spin parity per pair, and the alpha-beta sign is the product of the
// two same-spin signs stored with the connectivity. The opposite-spin Coulomb
// term of a single excitation, sum_{q in other} (pq|qq), is read from the
// per-string Coulomb tables (Ctx::d_Da / d_Db) instead of being summed per pair.
//   0. Xp = phi o X and Xpt = (phi o X)^T            (phase_split_kernel)
//   1. alpha same-spin + diagonal on Xp -> Y          (sigma_same_v6_kernel)
//   2. beta same-spin on Xpt -> Yt                    (sigma_same_v6_kernel)
//   3. alpha single x beta single on Xp -> Y +=       (sigma_ab_v6_kernel)
//   4. S = phi o (Y + Yt^T)                           (combine_phase_kernel)

template <typename T>
__global__ void phase_split_kernel(const T* __restrict__ X, size_t na, size_t nb, const uint64_t* __restrict__ astr,
                                   const uint64_t* __restrict__ bstr, T* __restrict__ Xp, T* __restrict__ Xpt,
                                   size_t xsa, size_t xsb) {
  __shared__ T tile[32][33];
  __shared__ uint64_t s_pa[32], s_b[32];
  const size_t ib0 = (size_t)blockIdx.x * 32, ia0 = (size_t)blockIdx.y * 32;
  const int tx = threadIdx.x;
  if (threadIdx.y == 0) {
    s_pa[tx] = ia0 + tx < na ? prefix_parity(astr[ia0 + tx]) : 0ull;
    s_b[tx] = ib0 + tx < nb ? bstr[ib0 + tx] : 0ull;
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const size_t ia = ia0 + k, ib = ib0 + tx;
    if (ia < na && ib < nb) {
      T v = X[ia * nb + ib];
      if (basis_phase(s_pa[k], s_b[tx])) v = -v;
      Xp[ia * xsa + ib] = v;
      tile[k][tx] = v;
    }
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const size_t ib = ib0 + k, ia = ia0 + tx;
    if (ia < na && ib < nb) Xpt[ib * xsb + ia] = tile[tx][k];
  }
}

// S[ia, ib] = phi(ia, ib) (Y[ia, ib] + Yt[ib, ia]), stored in T; Y and Yt
// have row strides xsa and xsb.
template <typename T>
__global__ void combine_phase_kernel(const double* __restrict__ Y, const double* __restrict__ Yt, size_t na,
                                     size_t nb, const uint64_t* __restrict__ astr, const uint64_t* __restrict__ bstr,
                                     T* __restrict__ S, size_t xsa, size_t xsb) {
  __shared__ double tile[32][33];
  __shared__ uint64_t s_pa[32], s_b[32];
  const size_t ib0 = (size_t)blockIdx.x * 32, ia0 = (size_t)blockIdx.y * 32;
  const int tx = threadIdx.x;
  if (threadIdx.y == 0) {
    s_pa[tx] = ia0 + tx < na ? prefix_parity(astr[ia0 + tx]) : 0ull;
    s_b[tx] = ib0 + tx < nb ? bstr[ib0 + tx] : 0ull;
  }
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const size_t ib = ib0 + k, ia = ia0 + tx;
    if (ib < nb && ia < na) tile[tx][k] = Yt[ib * xsb + ia];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const size_t ia = ia0 + k, ib = ib0 + tx;
    if (ia < na && ib < nb) {
      const double y = Y[ia * xsa + ib] + tile[k][tx];
      S[ia * nb + ib] = (T)(basis_phase(s_pa[k], s_b[tx]) ? -y : y);
    }
  }
}

// D[pq * stride + k] = sum over the orbitals q < L of string k of (pq|qq).
__global__ void coulomb_table_kernel(const double* __restrict__ G, int L, const uint64_t* __restrict__ s, size_t n,
                                     size_t stride, double* __restrict__ D, float* __restrict__ D32) {
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t pq = blockIdx.y;
  if (k >= n) return;
  const double* g = G + pq * (size_t)L;
  uint64_t bits = s[k] & range_mask(0, L);
  double v = 0.0;
  while (bits) {
    const int q = __ffsll((long long)bits) - 1;
    bits &= bits - 1;
    v += g[q];
  }
  D[pq * stride + k] = v;
  D32[pq * stride + k] = (float)v;
}

// Same-spin excitations in the alpha-first basis, VEC consecutive columns per
// thread; grid x = bra row (fastest: the resident CTAs share one column strip
// of the ket rows, which stays in L2), y = column strip. A CTA stages the
// entries of its row (ket, signed value, signed pair index) in shared memory;
// per pair a double costs one FMA and a single one add (the Coulomb table
// element of its column) and one FMA. X and Y rows have stride ldx, a multiple
// of VEC (padding columns up to ldx are computed and never read); hii has
// stride ncol.
template <typename T, int VEC>
__global__ void __launch_bounds__(kSameThreads)
sigma_same_v6_kernel(const T* __restrict__ X, size_t ncol, size_t ldx, const uint64_t* __restrict__ off,
                     const uint32_t* __restrict__ nsing, const uint32_t* __restrict__ ket,
                     const typename Prec<T>::V* __restrict__ val, const uint32_t* __restrict__ info,
                     const typename Prec<T>::V* __restrict__ Dt, size_t dstride, const double* __restrict__ hii,
                     const uint4* __restrict__ items, double* __restrict__ ypart, double* __restrict__ Y,
                     int accumulate) {
  __shared__ uint32_t s_ket[kSameThreads], s_pq[kSameThreads];
  __shared__ double s_val[kSameThreads];
  const uint4 item = items[blockIdx.x];  // bra string, entry range, output row
  const size_t r = item.x;
  double* __restrict__ Yrow = item.w ? ypart + (size_t)(item.w - 1) * ldx : Y + r * ldx;
  const size_t c0 = ((size_t)blockIdx.y * kSameThreads + threadIdx.x) * VEC;
  const bool active = c0 < ncol;
  double acc[VEC];
#pragma unroll
  for (int v = 0; v < VEC; ++v) acc[v] = 0.0;
  if (hii != nullptr && item.y == 0 && active) {
    double x[VEC];
    VecIO<T, VEC>::load(X + r * ldx + c0, x);
#pragma unroll
    for (int v = 0; v < VEC; ++v) acc[v] = c0 + v < ncol ? hii[r * ncol + c0 + v] * x[v] : 0.0;
  }
  const uint64_t beg = off[r] + item.y, end = off[r] + item.z, send = off[r] + nsing[r];
  const unsigned t = threadIdx.x;
  for (uint64_t base = beg; base < end; base += kSameThreads) {
    const int cnt = (int)min((uint64_t)kSameThreads, end - base);
    const int nsb = send > base ? (int)min((uint64_t)cnt, send - base) : 0;
    __syncthreads();
    if ((int)t < cnt) {
      const uint64_t e = base + t;
      const uint32_t inf = info[e];
      const double v = (double)val[e];
      s_ket[t] = ket[e];
      s_val[t] = (inf >> 31) ? -v : v;
      s_pq[t] = ((inf >> 12) & 0xfffu) | (inf & kInfoNeg);
    }
    __syncthreads();
    if (!active) continue;
    for (int e = 0; e < nsb; ++e) {
      const uint32_t pqs = s_pq[e];
      const double hv = s_val[e];
      double x[VEC], d[VEC];
      VecIO<T, VEC>::load(X + (size_t)s_ket[e] * ldx + c0, x);
      VecIO<T, VEC>::load(Dt + (size_t)(pqs & 0xfffu) * dstride + c0, d);
#pragma unroll
      for (int v = 0; v < VEC; ++v) acc[v] = fma(hv + flip_sign(d[v], pqs >> 31), x[v], acc[v]);
    }
#pragma unroll 4
    for (int e = nsb; e < cnt; ++e) {
      const double hv = s_val[e];
      double x[VEC];
      VecIO<T, VEC>::load(X + (size_t)s_ket[e] * ldx + c0, x);
#pragma unroll
      for (int v = 0; v < VEC; ++v) acc[v] = fma(hv, x[v], acc[v]);
    }
  }
  if (active) {
    if (accumulate && item.w == 0) {  // add to the row (a partial row of a split string is always written)
#pragma unroll
      for (int v = 0; v < VEC; ++v) Yrow[c0 + v] += acc[v];
    } else {
#pragma unroll
      for (int v = 0; v < VEC; ++v) Yrow[c0 + v] = acc[v];
    }
  }
}

// FP32-storage variant of sigma_same_v6_kernel: products and short runs of up
// to kRun entries are summed in FP32, and each run's sum is added to the FP64
// row accumulator (one conversion per run and column instead of one per pair).
constexpr int kRun = 8;

template <int VEC> struct VecF;
template <> struct VecF<1> {
  static __device__ __forceinline__ void load(const float* p, float* o) { o[0] = __ldg(p); }
};
template <> struct VecF<2> {
  static __device__ __forceinline__ void load(const float* p, float* o) {
    const float2 v = __ldg(reinterpret_cast<const float2*>(p));
    o[0] = v.x; o[1] = v.y;
  }
};
template <> struct VecF<4> {
  static __device__ __forceinline__ void load(const float* p, float* o) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
  }
};
template <> struct VecF<8> {
  static __device__ __forceinline__ void load(const float* p, float* o) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    const float4 w = __ldg(reinterpret_cast<const float4*>(p) + 1);
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w; o[4] = w.x; o[5] = w.y; o[6] = w.z; o[7] = w.w;
  }
};

template <int VEC>
__global__ void __launch_bounds__(kSameThreads)
sigma_same_v6f_kernel(const float* __restrict__ X, size_t ncol, size_t ldx, const uint64_t* __restrict__ off,
                      const uint32_t* __restrict__ nsing, const uint32_t* __restrict__ ket,
                      const float* __restrict__ val, const uint32_t* __restrict__ info, const float* __restrict__ Dt,
                      size_t dstride, const double* __restrict__ hii, const uint4* __restrict__ items,
                      double* __restrict__ ypart, double* __restrict__ Y, int accumulate) {
  __shared__ uint32_t s_ket[kSameThreads], s_pq[kSameThreads];
  __shared__ float s_val[kSameThreads];
  const uint4 item = items[blockIdx.x];  // bra string, entry range, output row
  const size_t r = item.x;
  double* __restrict__ Yrow = item.w ? ypart + (size_t)(item.w - 1) * ldx : Y + r * ldx;
  const size_t c0 = ((size_t)blockIdx.y * kSameThreads + threadIdx.x) * VEC;
  const bool active = c0 < ncol;
  double acc[VEC];
#pragma unroll
  for (int v = 0; v < VEC; ++v) acc[v] = 0.0;
  if (hii != nullptr && item.y == 0 && active) {
    float x[VEC];
    VecF<VEC>::load(X + r * ldx + c0, x);
#pragma unroll
    for (int v = 0; v < VEC; ++v) acc[v] = c0 + v < ncol ? hii[r * ncol + c0 + v] * (double)x[v] : 0.0;
  }
  const uint64_t beg = off[r] + item.y, end = off[r] + item.z, send = off[r] + nsing[r];
  const unsigned t = threadIdx.x;
  for (uint64_t base = beg; base < end; base += kSameThreads) {
    const int cnt = (int)min((uint64_t)kSameThreads, end - base);
    const int nsb = send > base ? (int)min((uint64_t)cnt, send - base) : 0;
    __syncthreads();
    if ((int)t < cnt) {
      const uint64_t e = base + t;
      const uint32_t inf = info[e];
      const float v = val[e];
      s_ket[t] = ket[e];
      s_val[t] = (inf >> 31) ? -v : v;
      s_pq[t] = ((inf >> 12) & 0xfffu) | (inf & kInfoNeg);
    }
    __syncthreads();
    if (!active) continue;
    for (int e0 = 0; e0 < nsb; e0 += kRun) {  // singles: value + signed Coulomb-table element
      const int e1 = min(e0 + kRun, nsb);
      float pf[VEC];
#pragma unroll
      for (int v = 0; v < VEC; ++v) pf[v] = 0.f;
      for (int e = e0; e < e1; ++e) {
        const uint32_t pqs = s_pq[e];
        const float hv = s_val[e];
        float x[VEC], d[VEC];
        VecF<VEC>::load(X + (size_t)s_ket[e] * ldx + c0, x);
        VecF<VEC>::load(Dt + (size_t)(pqs & 0xfffu) * dstride + c0, d);
#pragma unroll
        for (int v = 0; v < VEC; ++v) pf[v] = fmaf(hv + ((pqs >> 31) ? -d[v] : d[v]), x[v], pf[v]);
      }
#pragma unroll
      for (int v = 0; v < VEC; ++v) acc[v] += (double)pf[v];
    }
    for (int e0 = nsb; e0 < cnt; e0 += kRun) {  // doubles
      const int e1 = min(e0 + kRun, cnt);
      float pf[VEC];
#pragma unroll
      for (int v = 0; v < VEC; ++v) pf[v] = 0.f;
#pragma unroll 4
      for (int e = e0; e < e1; ++e) {
        const float hv = s_val[e];
        float x[VEC];
        VecF<VEC>::load(X + (size_t)s_ket[e] * ldx + c0, x);
#pragma unroll
        for (int v = 0; v < VEC; ++v) pf[v] = fmaf(hv, x[v], pf[v]);
      }
#pragma unroll
      for (int v = 0; v < VEC; ++v) acc[v] += (double)pf[v];
    }
  }
  if (active) {
    if (accumulate && item.w == 0) {
#pragma unroll
      for (int v = 0; v < VEC; ++v) Yrow[c0 + v] += acc[v];
    } else {
#pragma unroll
      for (int v = 0; v < VEC; ++v) Yrow[c0 + v] = acc[v];
    }
  }
}

// VEC consecutive elements in the storage type.
template <typename T, int VEC> struct LoadT;
template <int VEC> struct LoadT<double, VEC> {
  static __device__ __forceinline__ void load(const double* p, double* o) { VecIO<double, VEC>::load(p, o); }
};
template <int VEC> struct LoadT<float, VEC> {
  static __device__ __forceinline__ void load(const float* p, float* o) { VecF<VEC>::load(p, o); }
};

// Signed same-spin values of one union entry of the blocked kernel, one per
// bra string of the block (kBlkRows = 4).
template <typename V> struct Vals4;
template <> struct Vals4<double> { using P = double4; };
template <> struct Vals4<float> { using P = float4; };

// Resident CTAs per SM the blocked kernel is compiled for (0: no bound; FP32
// storage: three, which caps its registers at 80 with the deeper unroll of
// its union loop), and the union entries summed in FP32 before the FP64 row
// accumulation. Measured at 8000 x 8000 strings: FP64 runs fastest with the
// union loop unrolled 4 deep and no bound (52 registers, 4 CTAs per SM; an
// explicit bound of 1 let it take 96 registers and ran 19% slower), FP32 with
// 8 union entries' ket loads issued ahead.
template <typename T> struct BlkShape { static constexpr int kMinBlocks = 0; };
template <> struct BlkShape<float> { static constexpr int kMinBlocks = 3; };
constexpr int kBlkRun = kRun;

// Blocked same-spin product (codes 31/32/34/38 = columns per thread): one CTA
// per (work item of SameBlocks, strip of kSameThreads*VEC columns). The first
// item of a block adds the diagonal and the singles of its kBlkRows bra
// strings, one string at a time, as sigma_same_v6_kernel does; every item then
// walks its range of the block's union of double-excitation kets: each ket
// row strip is loaded once and applied to all strings of the block with their
// signed values (zero where a string does not connect), so a ket shared by
// several strings of the block costs one load instead of one per string.
// FP32 storage (T = float): products summed in FP32 over runs of kBlkRun union
// entries (or of kRun singles), each run's sum added to the FP64 row
// accumulator.
template <typename T, int VEC>
__global__ void __launch_bounds__(kSameThreads, BlkShape<T>::kMinBlocks)
sigma_same_blk_kernel(const T* __restrict__ X, size_t ncol, size_t ldx, const uint64_t* __restrict__ off,
                      const uint32_t* __restrict__ nsing, const uint32_t* __restrict__ ket,
                      const T* __restrict__ val, const uint32_t* __restrict__ info, const T* __restrict__ Dt,
                      size_t dstride, const double* __restrict__ hii, const uint4* __restrict__ brows,
                      const uint64_t* __restrict__ uoff, const uint32_t* __restrict__ uket,
                      const typename Vals4<T>::P* __restrict__ uval, const uint4* __restrict__ items,
                      double* __restrict__ ypart, double* __restrict__ Y, int accumulate) {
  using P4 = typename Vals4<T>::P;
  constexpr bool kF32 = std::is_same<T, float>::value;
  __shared__ uint32_t s_ket[kSameThreads], s_pq[kSameThreads];
  __shared__ P4 s_val4[kSameThreads];
  __shared__ T s_val[kSameThreads];
  const uint4 item = items[blockIdx.x];  // block, union range, partial slot
  const uint4 rw = brows[item.x];
  const uint32_t rows[kBlkRows] = {rw.x, rw.y, rw.z, rw.w};
  const size_t c0 = ((size_t)blockIdx.y * kSameThreads + threadIdx.x) * VEC;
  const bool active = c0 < ncol;
  const unsigned t = threadIdx.x;
  double acc[kBlkRows][VEC];
#pragma unroll
  for (int k = 0; k < kBlkRows; ++k)
#pragma unroll
    for (int v = 0; v < VEC; ++v) acc[k][v] = 0.0;
  if (item.y == 0) {  // the block's first item: diagonal and singles, string by string
#pragma unroll
    for (int k = 0; k < kBlkRows; ++k) {
      const uint32_t r = rows[k];
      if (r == kNoRow) continue;
      if (hii != nullptr && active) {
        T x[VEC];
        LoadT<T, VEC>::load(X + (size_t)r * ldx + c0, x);
#pragma unroll
        for (int v = 0; v < VEC; ++v) acc[k][v] = c0 + v < ncol ? hii[(size_t)r * ncol + c0 + v] * (double)x[v] : 0.0;
      }
      const uint64_t beg = off[r], end = beg + nsing[r];
      for (uint64_t base = beg; base < end; base += kSameThreads) {
        const int cnt = (int)min((uint64_t)kSameThreads, end - base);
        __syncthreads();
        if ((int)t < cnt) {
          const uint64_t e = base + t;
          const uint32_t inf = info[e];
          const T v = val[e];
          s_ket[t] = ket[e];
          s_val[t] = (inf >> 31) ? -v : v;
          s_pq[t] = ((inf >> 12) & 0xfffu) | (inf & kInfoNeg);
        }
        __syncthreads();
        if (!active) continue;
        for (int e0 = 0; e0 < cnt; e0 += kRun) {
          const int e1 = min(e0 + kRun, cnt);
          T pf[VEC];
#pragma unroll
          for (int v = 0; v < VEC; ++v) pf[v] = (T)0;
          for (int e = e0; e < e1; ++e) {
            const uint32_t pqs = s_pq[e];
            const T hv = s_val[e];
            T x[VEC], d[VEC];
            LoadT<T, VEC>::load(X + (size_t)s_ket[e] * ldx + c0, x);
            LoadT<T, VEC>::load(Dt + (size_t)(pqs & 0xfffu) * dstride + c0, d);
#pragma unroll
            for (int v = 0; v < VEC; ++v) {
              const T dv = (pqs >> 31) ? -d[v] : d[v];
              if constexpr (kF32) pf[v] = fmaf(hv + dv, x[v], pf[v]);
              else acc[k][v] = fma(hv + dv, x[v], acc[k][v]);
            }
          }
          if constexpr (kF32) {
#pragma unroll
            for (int v = 0; v < VEC; ++v) acc[k][v] += (double)pf[v];
          }
        }
      }
    }
  }
  // doubles: the block's union entries [u0, u1)
  const uint64_t ub = uoff[item.x];
  const uint64_t beg = ub + item.y, end = ub + item.z;
  for (uint64_t base = beg; base < end; base += kSameThreads) {
    const int cnt = (int)min((uint64_t)kSameThreads, end - base);
    __syncthreads();
    if ((int)t < cnt) {
      s_ket[t] = uket[base + t];
      s_val4[t] = uval[base + t];
    }
    __syncthreads();
    if (!active) continue;
    for (int e0 = 0; e0 < cnt; e0 += kBlkRun) {
      const int e1 = min(e0 + kBlkRun, cnt);
      T pf[kBlkRows][VEC];
#pragma unroll
      for (int k = 0; k < kBlkRows; ++k)
#pragma unroll
        for (int v = 0; v < VEC; ++v) pf[k][v] = (T)0;
      if constexpr (kF32) {
#pragma unroll 8
        for (int e = e0; e < e1; ++e) {
          T x[VEC];
          LoadT<T, VEC>::load(X + (size_t)s_ket[e] * ldx + c0, x);
          const P4 w = s_val4[e];
          const T wv[kBlkRows] = {w.x, w.y, w.z, w.w};
#pragma unroll
          for (int k = 0; k < kBlkRows; ++k)
#pragma unroll
            for (int v = 0; v < VEC; ++v) pf[k][v] = fmaf(wv[k], x[v], pf[k][v]);
        }
#pragma unroll
        for (int k = 0; k < kBlkRows; ++k)
#pragma unroll
          for (int v = 0; v < VEC; ++v) acc[k][v] += (double)pf[k][v];
      } else {
#pragma unroll 4
        for (int e = e0; e < e1; ++e) {
          T x[VEC];
          LoadT<T, VEC>::load(X + (size_t)s_ket[e] * ldx + c0, x);
          const P4 w = s_val4[e];
          const T wv[kBlkRows] = {w.x, w.y, w.z, w.w};
#pragma unroll
          for (int k = 0; k < kBlkRows; ++k)
#pragma unroll
            for (int v = 0; v < VEC; ++v) acc[k][v] = fma(wv[k], x[v], acc[k][v]);
        }
      }
    }
  }
  if (!active) return;
#pragma unroll
  for (int k = 0; k < kBlkRows; ++k) {
    const uint32_t r = rows[k];
    if (r == kNoRow) continue;
    if (item.w) {  // a part of a split block: its partial row
      double* y = ypart + ((size_t)(item.w - 1) * kBlkRows + k) * ldx + c0;
#pragma unroll
      for (int v = 0; v < VEC; ++v) y[v] = acc[k][v];
    } else {
      double* y = Y + (size_t)r * ldx + c0;
#pragma unroll
      for (int v = 0; v < VEC; ++v) y[v] = accumulate ? y[v] + acc[k][v] : acc[k][v];
    }
  }
}

// Assigns (or, with accumulate, adds) the sums of the partial rows of the
// blocks split over several items of the blocked same-spin kernel, parts in
// slot order; blockIdx.z = string of the block.
__global__ void same_blk_fixup_kernel(const uint4* __restrict__ split, const uint4* __restrict__ brows,
                                      const double* __restrict__ ypart, size_t ncol, size_t ldx,
                                      double* __restrict__ Y, int accumulate) {
  const uint4 sp = split[blockIdx.y];
  const uint4 rw = brows[sp.x];
  const int k = blockIdx.z;
  const uint32_t r = k == 0 ? rw.x : k == 1 ? rw.y : k == 2 ? rw.z : rw.w;
  if (r == kNoRow) return;
  for (size_t col = (size_t)blockIdx.x * blockDim.x + threadIdx.x; col < ncol; col += (size_t)gridDim.x * blockDim.x) {
    double t = 0.0;
    for (uint32_t q = 0; q < sp.z; ++q) t += ypart[((size_t)(sp.y + q) * kBlkRows + k) * ldx + col];
    double* y = Y + (size_t)r * ldx + col;
    *y = accumulate ? *y + t : t;
  }
}

constexpr int kAb6Threads = 1024;

// Alpha single x beta single in the alpha-first basis, balanced. One CTA per
// (bra alpha row ia, chunk of 1024*KS virtual rows of the balanced beta SELL).
// Per group of R alpha singles ja of ia: the ket rows Xp[ja, :] and the
// integral rows (ai|..) of the unpacked table are copied to shared memory with
// 16-byte loads; lane l of a warp owns virtual row 32s+l of slice s and walks
// its records (contiguous 256-byte warp reads), applying each to the R staged
// rows: sign = s_alpha(ia,ja) xor s_beta(ib,jb), both from the connectivity.
// Warp w owns slices w, 2*32-1-w, 2*32+w, ... (a snake over the length-sorted
// slices). Unsplit virtual rows add their sum to Y directly; split parts park
// theirs in shared memory and are added in slot order (deterministic). All
// split parts lie in chunk 0.
template <typename T, int R, int KS>
__global__ void __launch_bounds__(kAb6Threads, 1)
sigma_ab_v6_kernel(const T* __restrict__ Xp, size_t nb, size_t ldx, const uint64_t* __restrict__ a_off,
                   const uint32_t* __restrict__ a_nsing, const uint32_t* __restrict__ a_ket,
                   const uint32_t* __restrict__ a_info, const uint64_t* __restrict__ sell,
                   const uint64_t* __restrict__ soff, const uint32_t* __restrict__ slen, size_t nslice,
                   const uint32_t* __restrict__ vrow, const uint32_t* __restrict__ vslot, size_t nv,
                   const uint32_t* __restrict__ split_row, const uint32_t* __restrict__ split_slot, int nsplit,
                   const typename Prec<T>::V* __restrict__ Vt, size_t vstride, size_t xstride,
                   double* __restrict__ Y) {
  using V = typename Prec<T>::V;
  constexpr int kWarps = kAb6Threads / 32;
  extern __shared__ __align__(16) unsigned char smem[];
  T* xs = reinterpret_cast<T*>(smem);                                               // [R][xstride]
  V* erow = reinterpret_cast<V*>(smem + sizeof(T) * xstride * R);                   // [R][vstride]
  double* part = reinterpret_cast<double*>(smem + sizeof(T) * xstride * R + sizeof(V) * vstride * R);
  __shared__ uint32_t s_sa[R];
  const size_t ia = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t slice0 = (size_t)blockIdx.y * kWarps * KS;
  auto slice_of = [&](int k) -> size_t {
    return slice0 + (size_t)k * kWarps + ((k & 1) ? (kWarps - 1 - warp) : warp);
  };
  double acc[KS];
#pragma unroll
  for (int k = 0; k < KS; ++k) acc[k] = 0.0;
  const uint64_t e0 = a_off[ia];
  const int ns = (int)a_nsing[ia];
  const size_t xv = (nb * sizeof(T) + 15) / 16;  // 16-byte vectors of a ket row (xstride and ldx cover the tail)
  const size_t ev = vstride * sizeof(V) / 16;   // 16-byte vectors of an integral row
  for (int k0 = 0; k0 < ns; k0 += R) {
    const int nr = min(R, ns - k0);
    __syncthreads();
    if ((int)threadIdx.x < nr) s_sa[threadIdx.x] = a_info[e0 + k0 + threadIdx.x] >> 31;
    for (int rr = 0; rr < nr; ++rr) {
      const uint64_t e = e0 + k0 + rr;
      const uint4* s4 = reinterpret_cast<const uint4*>(Xp + (size_t)a_ket[e] * ldx);
      uint4* d4 = reinterpret_cast<uint4*>(xs + (size_t)rr * xstride);
      for (size_t t = threadIdx.x; t < xv; t += kAb6Threads) d4[t] = __ldg(s4 + t);
      const uint4* v4 = reinterpret_cast<const uint4*>(Vt + (size_t)((a_info[e] >> 12) & 0xfffu) * vstride);
      uint4* ed = reinterpret_cast<uint4*>(erow + (size_t)rr * vstride);
      for (size_t t = threadIdx.x; t < ev; t += kAb6Threads) ed[t] = __ldg(v4 + t);
    }
    __syncthreads();
    uint32_t sa[R];
#pragma unroll
    for (int rr = 0; rr < R; ++rr) sa[rr] = rr < nr ? s_sa[rr] : 0u;
#pragma unroll
    for (int k = 0; k < KS; ++k) {
      const size_t sl = slice_of(k);
      if (sl >= nslice) continue;
      const uint32_t len = slen[sl];
      const uint64_t* rp = sell + soff[sl] + lane;
      double s = acc[k];
      uint64_t next = len ? __ldg(rp) : 0ull;
      for (uint32_t m = 0; m < len; ++m) {
        const uint64_t rec = next;
        if (m + 1 < len) next = __ldg(rp + 32ull * (m + 1));
        const uint32_t jb = rec_ket(rec);
        const uint32_t pq = (uint32_t)((rec >> 16) & 0xfffu);
        const uint32_t sb = (uint32_t)(rec >> 40) & 1u;
        const bool pad = (rec >> 41) & 1ull;
#pragma unroll
        for (int rr = 0; rr < R; ++rr) {
          if (rr < nr) {
            const double v = pad ? 0.0 : (double)erow[(size_t)rr * vstride + pq];
            s = fma(flip_sign(v, sa[rr] ^ sb), (double)xs[(size_t)rr * xstride + jb], s);
          }
        }
      }
      acc[k] = s;
    }
  }
#pragma unroll
  for (int k = 0; k < KS; ++k) {
    const size_t sl = slice_of(k);
    const size_t pos = sl * 32 + lane;
    if (sl < nslice && pos < nv) {
      const uint32_t slot1 = vslot[pos];
      if (slot1 == 0) Y[ia * ldx + vrow[pos]] += acc[k];
      else part[slot1 - 1] = acc[k];
    }
  }
  if (blockIdx.y == 0 && nsplit > 0) {
    __syncthreads();
    for (int s = threadIdx.x; s < nsplit; s += kAb6Threads) {
      double t = 0.0;
      for (uint32_t j = split_slot[s]; j < split_slot[s + 1]; ++j) t += part[j];
      Y[ia * ldx + split_row[s]] += t;
    }
  }
}

// 16-byte packs of the staged rows of the alpha-beta kernel v7: element e of
// the pack of ket index jb is C'[ja_e, jb] (and of pair index pq, the signed
// integral s_alpha(ja_e) (a_e i_e|pq)).
template <typename T> struct RowPack;
template <> struct RowPack<double> {
  using P = double2;
  static constexpr int kRows = 2;
  static __device__ __forceinline__ void set(P& p, int e, double v) { if (e == 0) p.x = v; else p.y = v; }
  static __device__ __forceinline__ double dot(const P& a, const P& b) { return fma(a.x, b.x, a.y * b.y); }
};
template <> struct RowPack<float> {
  using P = float4;
  static constexpr int kRows = 4;
  static __device__ __forceinline__ void set(P& p, int e, float v) {
    if (e == 0) p.x = v; else if (e == 1) p.y = v; else if (e == 2) p.z = v; else p.w = v;
  }
  // the 4-term dot of one record in FP32, added to the FP64 row sum by the caller
  static __device__ __forceinline__ double dot(const P& a, const P& b) {
    return (double)fmaf(a.x, b.x, fmaf(a.y, b.y, fmaf(a.z, b.z, a.w * b.w)));
  }
};

// Alpha single x beta single, v7: as v6 (balanced SELL-32, alpha-first signs,
// split beta rows), with the staged rows interleaved into 16-byte packs (2
// FP64 or 4 FP32 rows per group): a record costs two 128-bit shared loads (ket
// pack, integral pack) for all rows of the group, and the alpha sign is
// applied to the integrals when they are staged, so the per-record sign is
// the beta one only. One CTA per (alpha work item, chunk of beta slices): an
// item is a bra alpha string or, for strings with many singles, a range of
// them whose partial row goes to its own slot (Conn::ab_item).
template <typename T, int KS>
__global__ void __launch_bounds__(kAb6Threads, 1)
sigma_ab_v7_kernel(const T* __restrict__ Xp, size_t ldx, const uint64_t* __restrict__ a_off,
                   const uint32_t* __restrict__ a_ket,
                   const uint32_t* __restrict__ a_info, const uint32_t* __restrict__ sell,
                   const uint64_t* __restrict__ soff4, const uint32_t* __restrict__ slen4, size_t nslice,
                   const uint32_t* __restrict__ vrow, const uint32_t* __restrict__ vslot, size_t nv,
                   const uint32_t* __restrict__ split_row, const uint32_t* __restrict__ split_slot, int nsplit,
                   const T* __restrict__ Vt, size_t vstride,
                   int npair, uint32_t epad, uint32_t jb0, size_t nbp, const uint32_t* __restrict__ kpos,
                   const uint4* __restrict__ items, double* __restrict__ ypart, double* __restrict__ Y) {
  using RP = RowPack<T>;
  using P = typename RP::P;
  constexpr int VR = RP::kRows;
  constexpr int kWarps = kAb6Threads / 32;
  extern __shared__ __align__(16) unsigned char smem[];
  P* xs = reinterpret_cast<P*>(smem);   // [nbp]: ket jb at kpos[jb] - jb0 (jb in jb0 .. jb0 + nbp - 1)
  P* er = xs + nbp;                     // [epad + npair]: copy 0 at pq, copy 1 at epad + pq
  double* part = reinterpret_cast<double*>(er + epad + npair);
  // work item: bra alpha string, range of its singles, output row
  const uint4 item = items[blockIdx.x];
  const size_t ia = item.x;
  const int kend = (int)item.z;
  double* __restrict__ Yrow = item.w ? ypart + (size_t)(item.w - 1) * ldx : Y + ia * ldx;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t slice0 = (size_t)blockIdx.y * kWarps * KS;
  auto slice_of = [&](int k) -> size_t {
    return slice0 + (size_t)k * kWarps + ((k & 1) ? (kWarps - 1 - warp) : warp);
  };
  double acc[KS];
#pragma unroll
  for (int k = 0; k < KS; ++k) acc[k] = 0.0;
  const uint64_t e0 = a_off[ia];
  for (int k0 = (int)item.y; k0 < kend; k0 += VR) {
    const int nr = min(VR, kend - k0);
    const T* xrow[VR];
    const T* vrow_p[VR];
    bool neg[VR];
#pragma unroll
    for (int e = 0; e < VR; ++e) {
      const uint64_t ent = e0 + k0 + (e < nr ? e : 0);
      const uint32_t inf = a_info[ent];
      xrow[e] = Xp + (size_t)a_ket[ent] * ldx + jb0;
      vrow_p[e] = Vt + (size_t)((inf >> 12) & 0xfffu) * vstride;
      neg[e] = (inf >> 31) != 0;
    }
    __syncthreads();
    // ket jb goes to position kpos[jb] - jb0, a permutation within aligned
    // groups of 8: the 8 lanes of a quarter-warp store to 8 different slots.
    // Each thread loads kStage packs before it stores them, so as many loads
    // of the ket rows are in flight.
    constexpr int kStage = 4;
    for (size_t t0 = threadIdx.x; t0 < nbp; t0 += (size_t)kStage * kAb6Threads) {
      P p[kStage];
      uint32_t at[kStage];
#pragma unroll
      for (int u = 0; u < kStage; ++u) {
        const size_t t = t0 + (size_t)u * kAb6Threads;
        at[u] = t < nbp ? __ldg(kpos + jb0 + t) - jb0 : 0u;
#pragma unroll
        for (int e = 0; e < VR; ++e) RP::set(p[u], e, (e < nr && t < nbp) ? __ldg(xrow[e] + t) : (T)0);
      }
#pragma unroll
      for (int u = 0; u < kStage; ++u)
        if (t0 + (size_t)u * kAb6Threads < nbp) xs[at[u]] = p[u];
    }
    for (int t = threadIdx.x; t < npair; t += kAb6Threads) {
      P p;
#pragma unroll
      for (int e = 0; e < VR; ++e) {
        const T v = e < nr ? __ldg(vrow_p[e] + t) : (T)0;
        RP::set(p, e, neg[e] ? -v : v);
      }
      er[t] = p;
      er[epad + t] = p;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < KS; ++k) {
      const size_t sl = slice_of(k);
      if (sl >= nslice) continue;
      // 32-bit records (bits 0-15 staged ket position, 16-27 pair, 28 sign, 29 pad, 30 integral
      // copy), four per lane per 16-byte load, the next block in flight
      const uint32_t nblk = slen4[sl] >> 2;
      const uint4* rp = reinterpret_cast<const uint4*>(sell + soff4[sl]) + lane;
      double s = acc[k];
      uint4 cur = nblk ? __ldg(rp) : make_uint4(0u, 0u, 0u, 0u);
      for (uint32_t bk = 0; bk < nblk; ++bk) {
        const uint4 nxt = bk + 1 < nblk ? __ldg(rp + 32ull * (bk + 1)) : cur;
        const uint32_t recs[4] = {cur.x, cur.y, cur.z, cur.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const uint32_t rec = recs[q];
          const P x = xs[rec & 0xffffu];  // panel-relative position; pad records repeat a real record's addresses
          const P ev = er[((rec >> 16) & 0xfffu) + ((rec >> 30) & 1u) * epad];
          double d = RP::dot(ev, x);
          d = ((rec >> 29) & 1u) ? 0.0 : d;
          s += flip_sign(d, (rec >> 28) & 1u);
        }
        cur = nxt;
      }
      acc[k] = s;
    }
  }
#pragma unroll
  for (int k = 0; k < KS; ++k) {
    const size_t sl = slice_of(k);
    const size_t pos = sl * 32 + lane;
    if (sl < nslice && pos < nv) {
      const uint32_t slot1 = vslot[pos];
      if (slot1 == 0) Yrow[vrow[pos]] += acc[k];
      else part[slot1 - 1] = acc[k];
    }
  }
  if (blockIdx.y == 0 && nsplit > 0) {
    __syncthreads();
    for (int s = threadIdx.x; s < nsplit; s += kAb6Threads) {
      double t = 0.0;
      for (uint32_t j = split_slot[s]; j < split_slot[s + 1]; ++j) t += part[j];
      Yrow[split_row[s]] += t;
    }
  }
}

// Shared memory of v7 on one panel: its ket range, the two copies of the
// integral row (ab7_er_packs 16-byte packs) and its split slots. (The kernels' dynamic shared-memory limit is always set
// to the full budget: the attribute is global per kernel, and contexts on
// other host threads launch the same kernel with other sizes.)
size_t ab7_smem_bytes(const Ctx* c, const SellPanel& p) {
  return 16 * ((size_t)(p.jb1 - p.jb0) + ab7_er_packs(c->npair)) + sizeof(double) * (size_t)p.nslot;
}

// The panels v7 runs on: the whole ket range, or the ket-range slices.
const std::vector<SellPanel>* ab7_panels(const Ctx* c, std::vector<SellPanel>& one) {
  const Conn& cb = c->conn[1];
  if (!cb.panels.empty()) return &cb.panels;
  one.assign(1, cb.bal);
  return &one;
}

bool ab7_fits(const Ctx* c) {
  std::vector<SellPanel> one;
  for (const SellPanel& p : *ab7_panels(c, one))
    if (ab7_smem_bytes(c, p) > kAbSmemBudget) return false;
  return true;
}

// `it` supplies the work items: the alpha connectivity itself, or the items
// of a row range (Ctx::range_conn).
template <typename T, int KS>
int launch_ab_v7(Ctx* c, const T* Xp, const SellPanel& bp, const Conn& it) {
  const Conn& ca = c->conn[0];
  const bool f64 = std::is_same<T, double>::value;
  const T* Vt = f64 ? (const T*)c->d_V : (const T*)c->d_V32;
  const size_t vs = f64 ? c->vstride : c->vstride32;
  const size_t smem = ab7_smem_bytes(c, bp);
  SBDX_CUDA(c, cudaFuncSetAttribute(sigma_ab_v7_kernel<T, KS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kAbSmemBudget));
  const size_t per_cta = (size_t)(kAb6Threads / 32) * KS;
  dim3 grid((unsigned)it.n_item, (unsigned)((bp.nslice + per_cta - 1) / per_cta));
  if (grid.y == 0) grid.y = 1;
  sigma_ab_v7_kernel<T, KS><<<grid, kAb6Threads, smem, c->stream>>>(
      Xp, c->xsa, ca.off, ca.ket, ca.info, bp.sell32, bp.soff4, bp.slen4, bp.nslice, bp.vrow, bp.vslot, bp.nv,
      bp.split_row, bp.split_slot, bp.nsplit, Vt, vs, (int)c->npair, (uint32_t)ab7_epad(c->npair), bp.jb0,
      (size_t)(bp.jb1 - bp.jb0), c->conn[1].kpos, it.ab_item, it.ypart, c->d_y);
  SBDX_LAUNCHED(c);
  return 0;
}

// Adds the partial rows of the alpha strings split over several work items to
// the output, parts in slot order (one fixed summation order).
__global__ void ab_split_fixup_kernel(const uint4* __restrict__ split, const double* __restrict__ ypart, size_t nb,
                                      size_t ldx, double* __restrict__ Y) {
  const uint4 sp = split[blockIdx.y];
  const double* part = ypart + (size_t)sp.y * ldx;
  for (size_t ib = (size_t)blockIdx.x * blockDim.x + threadIdx.x; ib < nb; ib += (size_t)gridDim.x * blockDim.x) {
    double t = 0.0;
    for (uint32_t q = 0; q < sp.z; ++q) t += part[(size_t)q * ldx + ib];
    Y[(size_t)sp.x * ldx + ib] += t;
  }
}

template <typename T>
int run_ab_v7(Ctx* c, const T* Xp, const Conn* items = nullptr) {
  const Conn& ca = items ? *items : c->conn[0];
  if (ca.n_item == 0) return 0;  // no alpha string has a single excitation
  if (ca.n_part > 0)
    SBDX_CUDA(c, cudaMemsetAsync(ca.ypart, 0, sizeof(double) * (size_t)ca.n_part * c->xsa, c->stream));
  std::vector<SellPanel> one;
  for (const SellPanel& bp : *ab7_panels(c, one)) {
    int rc;
    if (bp.slices_per_warp >= 16) rc = launch_ab_v7<T, 16>(c, Xp, bp, ca);
    else if (bp.slices_per_warp >= 12) rc = launch_ab_v7<T, 12>(c, Xp, bp, ca);
    else rc = launch_ab_v7<T, 8>(c, Xp, bp, ca);
    if (rc) return rc;
  }
  if (ca.n_split > 0) {
    const unsigned bx = (unsigned)std::min<size_t>((c->nb + 255) / 256, 64);
    ab_split_fixup_kernel<<<dim3(bx, (unsigned)ca.n_split), 256, 0, c->stream>>>(ca.ab_split, ca.ypart, c->nb,
                                                                                  c->xsa, c->d_y);
    SBDX_LAUNCHED(c);
  }
  return 0;
}

// Assigns (or, with accumulate, adds) the sum of the partial rows of the bra
// strings split over several same-spin work items, parts in slot order.
__global__ void same_split_fixup_kernel(const uint4* __restrict__ split, const double* __restrict__ ypart,
                                        size_t ncol, size_t ldx, double* __restrict__ Y, int accumulate) {
  const uint4 sp = split[blockIdx.y];
  const double* part = ypart + (size_t)sp.y * ldx;
  for (size_t col = (size_t)blockIdx.x * blockDim.x + threadIdx.x; col < ncol; col += (size_t)gridDim.x * blockDim.x) {
    double t = 0.0;
    for (uint32_t q = 0; q < sp.z; ++q) t += part[(size_t)q * ldx + col];
    double* y = Y + (size_t)sp.x * ldx + col;
    *y = accumulate ? *y + t : t;
  }
}

template <typename T, int VEC>
int launch_same_v6(Ctx* c, const T* X, size_t nrow, size_t ncol, size_t ldx, const Conn& cn,
                   const typename Prec<T>::V* val, const typename Prec<T>::V* Dt, size_t dstride, const double* hii,
                   double* Y, int accumulate) {
  (void)nrow;
  if (cn.n_same_item > 0) {
    dim3 grid((unsigned)cn.n_same_item,
              (unsigned)((ncol + (size_t)kSameThreads * VEC - 1) / ((size_t)kSameThreads * VEC)));
    if constexpr (std::is_same<T, float>::value) {
      sigma_same_v6f_kernel<VEC><<<grid, kSameThreads, 0, c->stream>>>(X, ncol, ldx, cn.off, cn.nsing, cn.ket, val,
                                                                        cn.info, Dt, dstride, hii, cn.same_item,
                                                                        cn.same_ypart, Y, accumulate);
    } else {
      sigma_same_v6_kernel<T, VEC><<<grid, kSameThreads, 0, c->stream>>>(X, ncol, ldx, cn.off, cn.nsing, cn.ket, val,
                                                                         cn.info, Dt, dstride, hii, cn.same_item,
                                                                         cn.same_ypart, Y, accumulate);
    }
    SBDX_LAUNCHED(c);
  }
  if (cn.n_same_split > 0) {
    const unsigned bx = (unsigned)std::min<size_t>((ncol + 255) / 256, 64);
    same_split_fixup_kernel<<<dim3(bx, (unsigned)cn.n_same_split), 256, 0, c->stream>>>(
        cn.same_split, cn.same_ypart, ncol, ldx, Y, accumulate);
    SBDX_LAUNCHED(c);
  }
  return 0;
}

template <typename T, int VEC>
int launch_same_blk(Ctx* c, const T* X, size_t ncol, size_t ldx, const Conn& cn, const T* val, const T* Dt,
                    size_t dstride, const double* hii, double* Y, int accumulate) {
  const SameBlocks& B = cn.blk;
  using P4 = typename Vals4<T>::P;
  const P4* uval = reinterpret_cast<const P4*>(std::is_same<T, double>::value ? (const void*)B.uval
                                                                              : (const void*)B.uval32);
  if (B.n_item > 0) {
    dim3 grid((unsigned)B.n_item, (unsigned)((ncol + (size_t)kSameThreads * VEC - 1) / ((size_t)kSameThreads * VEC)));
    sigma_same_blk_kernel<T, VEC><<<grid, kSameThreads, 0, c->stream>>>(
        X, ncol, ldx, cn.off, cn.nsing, cn.ket, val, cn.info, Dt, dstride, hii, B.rows, B.uoff, B.uket, uval, B.item,
        B.ypart, Y, accumulate);
    SBDX_LAUNCHED(c);
  }
  if (B.n_split > 0) {
    const unsigned bx = (unsigned)std::min<size_t>((ncol + 255) / 256, 64);
    same_blk_fixup_kernel<<<dim3(bx, (unsigned)B.n_split, kBlkRows), 256, 0, c->stream>>>(B.split, B.rows, B.ypart,
                                                                                         ncol, ldx, Y, accumulate);
    SBDX_LAUNCHED(c);
  }
  return 0;
}

// v6 same-spin codes: 21, 22, 24, 28 = 1, 2, 4, 8 columns per thread, narrowed
// to the widest vector that divides the row stride and keeps 16-byte
// alignment (the internal vectors have strides padded to 8 elements, so only
// a misaligned base narrows).
// Codes 31, 32, 34, 38: the blocked kernel with as many columns per thread.
// accumulate: add to Y's rows instead of writing them (the pipelined
// host-buffer sigma runs the alpha-beta kernel first).
template <typename T>
int run_same_v6(Ctx* c, int code, const T* X, size_t nrow, size_t ncol, size_t ldx, const Conn& cn,
                const typename Prec<T>::V* val, const typename Prec<T>::V* Dt, size_t dstride, const double* hii,
                double* Y, int accumulate = 0) {
  int vec = code % 10;
  const bool aligned = (reinterpret_cast<uintptr_t>(X) % 16) == 0;
  while (vec > 1 && (!aligned || ldx % vec != 0 || dstride % vec != 0)) vec >>= 1;
  if (code / 10 == 3 && cn.blk.nblk > 0) {  // blocked kernel (31, 32, 34, 38)
    if (vec >= 8) return launch_same_blk<T, 8>(c, X, ncol, ldx, cn, val, Dt, dstride, hii, Y, accumulate);
    if (vec >= 4) return launch_same_blk<T, 4>(c, X, ncol, ldx, cn, val, Dt, dstride, hii, Y, accumulate);
    if (vec == 2) return launch_same_blk<T, 2>(c, X, ncol, ldx, cn, val, Dt, dstride, hii, Y, accumulate);
    return launch_same_blk<T, 1>(c, X, ncol, ldx, cn, val, Dt, dstride, hii, Y, accumulate);
  }
  if (vec >= 8) return launch_same_v6<T, 8>(c, X, nrow, ncol, ldx, cn, val, Dt, dstride, hii, Y, accumulate);
  if (vec >= 4) return launch_same_v6<T, 4>(c, X, nrow, ncol, ldx, cn, val, Dt, dstride, hii, Y, accumulate);
  if (vec == 2) return launch_same_v6<T, 2>(c, X, nrow, ncol, ldx, cn, val, Dt, dstride, hii, Y, accumulate);
  return launch_same_v6<T, 1>(c, X, nrow, ncol, ldx, cn, val, Dt, dstride, hii, Y, accumulate);
}

template <typename T, int R, int KS>
int launch_ab_v6(Ctx* c, const T* Xp, size_t smem, size_t xstride) {
  using V = typename Prec<T>::V;
  const Conn& ca = c->conn[0];
  const Conn& cb = c->conn[1];
  const bool f64 = std::is_same<T, double>::value;
  const V* Vt = f64 ? (const V*)c->d_V : (const V*)c->d_V32;
  const size_t vs = f64 ? c->vstride : c->vstride32;
  SBDX_CUDA(c, cudaFuncSetAttribute(sigma_ab_v6_kernel<T, R, KS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kAbSmemBudget));
  const size_t per_cta = (size_t)(kAb6Threads / 32) * KS;  // slices
  const SellPanel& bp = cb.bal;
  dim3 grid((unsigned)c->na, (unsigned)((bp.nslice + per_cta - 1) / per_cta));
  if (grid.y == 0) grid.y = 1;
  sigma_ab_v6_kernel<T, R, KS><<<grid, kAb6Threads, smem, c->stream>>>(
      Xp, c->nb, c->xsa, ca.off, ca.nsing, ca.ket, ca.info, bp.sell, bp.soff, bp.slen, bp.nslice, bp.vrow, bp.vslot,
      bp.nv,
      bp.split_row, bp.split_slot, bp.nsplit, Vt, vs, xstride, c->d_y);
  SBDX_LAUNCHED(c);
  return 0;
}

template <typename T, int R>
int launch_ab_v6_ks(Ctx* c, const T* Xp, size_t smem, size_t xstride) {
  const int ks = c->conn[1].bal.slices_per_warp;
  if (ks >= 16) return launch_ab_v6<T, R, 16>(c, Xp, smem, xstride);
  if (ks >= 12) return launch_ab_v6<T, R, 12>(c, Xp, smem, xstride);
  return launch_ab_v6<T, R, 8>(c, Xp, smem, xstride);
}

// v6 alpha-beta codes: 61-64 = 1-4 staged alpha singles per group, narrowed
// until the ket rows, integral rows and split slots fit in shared memory.
template <typename T>
int run_ab_v6(Ctx* c, int code, const T* Xp) {
  using V = typename Prec<T>::V;
  if (code / 10 == 7) {  // 71: packed rows, on ket-range panels when a whole row does not fit
    if (ab7_fits(c)) return run_ab_v7<T>(c, Xp);
    code = std::is_same<T, double>::value ? 62 : 64;
  }
  const bool f64 = std::is_same<T, double>::value;
  const size_t vs = f64 ? c->vstride : c->vstride32;
  const size_t per = 16 / sizeof(T);
  const size_t xstride = (c->nb + per - 1) / per * per;
  const size_t budget = kAbSmemBudget;  // dynamic part; the static part is a few bytes
  const size_t extra = sizeof(double) * (size_t)c->conn[1].bal.nslot;
  int R = code % 10 > 0 ? code % 10 : 2;
  size_t smem = 0;
  for (; R >= 1; --R) {
    smem = (size_t)R * (sizeof(T) * xstride + sizeof(V) * vs) + extra;
    if (smem <= budget) break;
  }
  if (R < 1) {
    c->err = "sigma: beta dimension too large for one shared-memory ket row";
    return 1;
  }
  if (R >= 4) return launch_ab_v6_ks<T, 4>(c, Xp, smem, xstride);
  if (R == 3) return launch_ab_v6_ks<T, 3>(c, Xp, smem, xstride);
  if (R == 2) return launch_ab_v6_ks<T, 2>(c, Xp, smem, xstride);
  return launch_ab_v6_ks<T, 1>(c, Xp, smem, xstride);
}

bool same_alpha_first(int code) { return (code > 20 && code < 30) || (code > 30 && code < 40); }

bool is_v6(const Tune& t) {
  return same_alpha_first(t.same_code) && ((t.ab_code > 60 && t.ab_code < 70) || t.ab_code == 71);
}

template <typename T>
int run_sigma_v6(Ctx* c, const Tune& tune, const T* X, T* S) {
  using V = typename Prec<T>::V;
  const size_t na = c->na, nb = c->nb;
  const bool f64 = std::is_same<T, double>::value;
  const Conn& ca = c->conn[0];
  const Conn& cb = c->conn[1];
  const V* valA = f64 ? (const V*)ca.val : (const V*)ca.val32;
  const V* valB = f64 ? (const V*)cb.val : (const V*)cb.val32;
  const V* Db = f64 ? (const V*)c->d_Db : (const V*)c->d_Db32;
  const V* Da = f64 ? (const V*)c->d_Da : (const V*)c->d_Da32;
  T* xp = reinterpret_cast<T*>(c->d_xp);
  T* xpt = reinterpret_cast<T*>(c->d_xt);
  auto mark = [&](int k) {
    if (c->profiling) cudaEventRecord(c->ev[k], c->stream);
  };
  int rc = 0;
  mark(0);
  {
    dim3 grid((unsigned)((nb + 31) / 32), (unsigned)((na + 31) / 32));
    phase_split_kernel<T><<<grid, dim3(32, 8), 0, c->stream>>>(X, na, nb, c->d_a, c->d_b, xp, xpt, c->xsa, c->xsb);
    SBDX_LAUNCHED(c);
  }
  mark(1);
  if ((rc = run_same_v6<T>(c, tune.same_code, xp, na, nb, c->xsa, ca, valA, Db, c->db_stride, c->d_hii, c->d_y)))
    return rc;
  mark(2);
  if ((rc = run_same_v6<T>(c, tune.same_code, xpt, nb, na, c->xsb, cb, valB, Da, c->da_stride, nullptr, c->d_yt)))
    return rc;
  mark(3);
  if ((rc = run_ab_v6<T>(c, tune.ab_code, xp))) return rc;
  mark(4);
  {
    dim3 grid((unsigned)((nb + 31) / 32), (unsigned)((na + 31) / 32));
    combine_phase_kernel<T><<<grid, dim3(32, 8), 0, c->stream>>>(c->d_y, c->d_yt, na, nb, c->d_a, c->d_b, S, c->xsa,
                                                                 c->xsb);
    SBDX_LAUNCHED(c);
  }
  mark(5);
  if (c->profiling) {
    // reported in the phase order alpha same-spin, transpose (here the phase
    // split), beta same-spin, alpha-beta, combine
    const int from[kSigmaPhases] = {1, 0, 2, 3, 4};
    SBDX_CUDA(c, cudaEventSynchronize(c->ev[5]));
    for (int k = 0; k < kSigmaPhases; ++k) {
      float ms = 0.f;
      SBDX_CUDA(c, cudaEventElapsedTime(&ms, c->ev[from[k]], c->ev[from[k] + 1]));
      c->phase_ms[k] += ms;
    }
    ++c->phase_calls;
  }
  return 0;
}

template <typename T>
int run_sigma_v5(Ctx* c, const T* X, T* S) {
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

// Default launch codes: the alpha-first kernels; the blocked same-spin kernel
// above a size where its four-strings-per-CTA grid still fills the GPU, the
// one-string-per-CTA kernel below it. Crossovers measured on B200 over the
// 64 subspaces of the batched workload and the 400x400 to 8000x8000
// workloads: FP64 about 2 M determinants (code 32 against 22), FP32 about
// 1 M (code 34 against 24).
Tune default_tune(const Ctx* c, bool f64) {
  const size_t D = c->na * c->nb;
  if (f64) return D >= kBlkMinDets64 ? Tune{32, 71} : Tune{22, 71};
  return D >= kBlkMinDets32 ? Tune{34, 71} : Tune{24, 71};
}

Tune effective_tune(const Ctx* c, bool f64) {
  Tune t = c->tune[f64 ? 0 : 1];
  const Tune d = default_tune(c, f64);
  const bool v6 = same_alpha_first(t.same_code) || (t.ab_code > 60 && t.ab_code < 70) ||
                  t.ab_code == 71 || (t.same_code == 0 && t.ab_code == 0);
  if (v6) {
    if (t.same_code == 0) t.same_code = d.same_code;
    if (t.ab_code == 0) t.ab_code = d.ab_code;
  }
  return t;
}

template <typename T>
int run_sigma(Ctx* c, const T* X, T* S) {
  const Tune t = effective_tune(c, std::is_same<T, double>::value);
  if (is_v6(t)) return run_sigma_v6<T>(c, t, X, S);
  return run_sigma_v5<T>(c, X, S);
}

// Output rows [a0, a1) of the alpha-first sigma (one shard of the alpha
// strings; the reference's bra block of a rank, chemistry/tpb/mult.h:429-432).
// The phase split covers the whole input (every ket row may be read); the
// alpha same-spin and alpha-beta kernels run the range's work items
// (Ctx::range_conn); the beta same-spin kernel runs on the range's columns of
// the transposed input (its output and Coulomb-table columns offset by a0,
// a multiple of 8 so that the vector loads stay aligned); the combine writes
// the range's rows into S, whose row 0 is alpha string a0.
template <typename T>
int run_sigma_rows(Ctx* c, const Tune& tune, const T* X, T* S, size_t a0, size_t a1) {
  using V = typename Prec<T>::V;
  const size_t na = c->na, nb = c->nb, nr = a1 - a0;
  const bool f64 = std::is_same<T, double>::value;
  const Conn& ca = c->conn[0];
  const Conn& cb = c->conn[1];
  const Conn& rc_items = c->range_conn;
  Conn ra = ca;  // the alpha lists with the range's same-spin work items
  ra.blk = rc_items.blk;
  ra.same_item = rc_items.same_item;
  ra.n_same_item = rc_items.n_same_item;
  ra.same_split = rc_items.same_split;
  ra.n_same_split = rc_items.n_same_split;
  ra.n_same_part = rc_items.n_same_part;
  ra.same_ypart = rc_items.same_ypart;
  const V* valA = f64 ? (const V*)ca.val : (const V*)ca.val32;
  const V* valB = f64 ? (const V*)cb.val : (const V*)cb.val32;
  const V* Db = f64 ? (const V*)c->d_Db : (const V*)c->d_Db32;
  const V* Da = f64 ? (const V*)c->d_Da : (const V*)c->d_Da32;
  T* xp = reinterpret_cast<T*>(c->d_xp);
  T* xpt = reinterpret_cast<T*>(c->d_xt);
  auto mark = [&](int k) {
    if (c->profiling) cudaEventRecord(c->ev[k], c->stream);
  };
  int rc = 0;
  mark(0);
  {
    dim3 grid((unsigned)((nb + 31) / 32), (unsigned)((na + 31) / 32));
    phase_split_kernel<T><<<grid, dim3(32, 8), 0, c->stream>>>(X, na, nb, c->d_a, c->d_b, xp, xpt, c->xsa, c->xsb);
    SBDX_LAUNCHED(c);
  }
  mark(1);
  if (nr == 0) return 0;
  if ((rc = run_same_v6<T>(c, tune.same_code, xp, na, nb, c->xsa, ra, valA, Db, c->db_stride, c->d_hii, c->d_y)))
    return rc;
  mark(2);
  if ((rc = run_same_v6<T>(c, tune.same_code, xpt + a0, nb, nr, c->xsb, cb, valB, Da + a0, c->da_stride, nullptr,
                           c->d_yt + a0)))
    return rc;
  mark(3);
  if ((rc = run_ab_v7<T>(c, xp, &rc_items))) return rc;
  mark(4);
  {
    dim3 grid((unsigned)((nb + 31) / 32), (unsigned)((nr + 31) / 32));
    combine_phase_kernel<T><<<grid, dim3(32, 8), 0, c->stream>>>(c->d_y + a0 * c->xsa, c->d_yt + a0, nr, nb,
                                                                 c->d_a + a0, c->d_b, S, c->xsa, c->xsb);
    SBDX_LAUNCHED(c);
  }
  mark(5);
  if (c->profiling) {  // the phase order of run_sigma_v6
    const int from[kSigmaPhases] = {1, 0, 2, 3, 4};
    SBDX_CUDA(c, cudaEventSynchronize(c->ev[5]));
    for (int k = 0; k < kSigmaPhases; ++k) {
      float ms = 0.f;
      SBDX_CUDA(c, cudaEventElapsedTime(&ms, c->ev[from[k]], c->ev[from[k] + 1]));
      c->phase_ms[k] += ms;
    }
    ++c->phase_calls;
  }
  return 0;
}

}  // namespace

int build_coulomb_tables(Ctx* c) {
  cudaFree(c->d_Da); cudaFree(c->d_Db); cudaFree(c->d_Da32); cudaFree(c->d_Db32);
  c->d_Da = c->d_Db = nullptr;
  c->d_Da32 = c->d_Db32 = nullptr;
  c->da_stride = pad8(c->na);
  c->db_stride = pad8(c->nb);
  const size_t na_el = c->npair * c->da_stride, nb_el = c->npair * c->db_stride;
  SBDX_CUDA(c, cudaMalloc(&c->d_Da, sizeof(double) * na_el));
  SBDX_CUDA(c, cudaMalloc(&c->d_Db, sizeof(double) * nb_el));
  SBDX_CUDA(c, cudaMalloc(&c->d_Da32, sizeof(float) * na_el));
  SBDX_CUDA(c, cudaMalloc(&c->d_Db32, sizeof(float) * nb_el));
  SBDX_CUDA(c, cudaMemsetAsync(c->d_Da, 0, sizeof(double) * na_el, c->stream));
  SBDX_CUDA(c, cudaMemsetAsync(c->d_Db, 0, sizeof(double) * nb_el, c->stream));
  SBDX_CUDA(c, cudaMemsetAsync(c->d_Da32, 0, sizeof(float) * na_el, c->stream));
  SBDX_CUDA(c, cudaMemsetAsync(c->d_Db32, 0, sizeof(float) * nb_el, c->stream));
  dim3 ga((unsigned)((c->na + 255) / 256), (unsigned)c->npair);
  coulomb_table_kernel<<<ga, 256, 0, c->stream>>>(c->d_G, c->L, c->d_a, c->na, c->da_stride, c->d_Da, c->d_Da32);
  SBDX_LAUNCHED(c);
  dim3 gb((unsigned)((c->nb + 255) / 256), (unsigned)c->npair);
  coulomb_table_kernel<<<gb, 256, 0, c->stream>>>(c->d_G, c->L, c->d_b, c->nb, c->db_stride, c->d_Db, c->d_Db32);
  SBDX_LAUNCHED(c);
  return 0;
}

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
  const size_t nv = c->npair * c->npair;
  c->vstride = (c->npair + 1) / 2 * 2;
  c->vstride32 = (c->npair + 3) / 4 * 4;
  cudaFree(c->d_V);
  cudaFree(c->d_V32);
  c->d_V = nullptr;
  c->d_V32 = nullptr;
  SBDX_CUDA(c, cudaMalloc(&c->d_V, sizeof(double) * c->npair * c->vstride));
  SBDX_CUDA(c, cudaMalloc(&c->d_V32, sizeof(float) * c->npair * c->vstride32));
  SBDX_CUDA(c, cudaMemsetAsync(c->d_V, 0, sizeof(double) * c->npair * c->vstride, c->stream));
  SBDX_CUDA(c, cudaMemsetAsync(c->d_V32, 0, sizeof(float) * c->npair * c->vstride32, c->stream));
  unpack_eri_kernel<<<(unsigned)((nv + 255) / 256), 256, 0, c->stream>>>(c->d_eri, c->npair, c->vstride,
                                                                           c->vstride32, c->d_V, c->d_V32);
  SBDX_LAUNCHED(c);
  return 0;
}

int ensure_sigma_scratch(Ctx* c) {
  c->xsa = pad8(c->nb);
  c->xsb = pad8(c->na);
  const size_t n = std::max(c->na * c->xsa, c->nb * c->xsb);  // >= D
  auto get = [&](void** p) -> int {
    if (*p) return 0;
    SBDX_CUDA(c, cudaMalloc(p, sizeof(double) * n));
    SBDX_CUDA(c, cudaMemsetAsync(*p, 0, sizeof(double) * n, c->stream));  // padding columns start at zero
    return 0;
  };
  int rc;
  if ((rc = get(&c->d_xt)) || (rc = get(&c->d_xp)) || (rc = get((void**)&c->d_y)) || (rc = get((void**)&c->d_yt)))
    return rc;
  return 0;
}

// Autotuner: for each precision, time the candidate kernel variants and launch
// shapes on the current problem (one warm-up and two timed sigmas each, CUDA
// events between the phases, scratch input vectors) and keep the fastest
// same-spin and alpha-beta choice separately.
int autotune(Ctx* c) {
  int rc = 0;
  clear_sigma_graphs(c);
  if (!c->have_conn && (rc = build_connectivity(c))) return rc;
  if (!c->have_hii && (rc = diag_terms(c))) return rc;
  if ((rc = ensure_sigma_scratch(c))) return rc;
  const size_t D = c->na * c->nb;
  void *X = nullptr, *S = nullptr;
  SBDX_CUDA(c, pool_alloc(c, &X, sizeof(double) * D));
  SBDX_CUDA(c, pool_alloc(c, &S, sizeof(double) * D));
  SBDX_CUDA(c, cudaMemsetAsync(X, 0, sizeof(double) * D, c->stream));
  const bool prof0 = c->profiling;
  if (!c->ev[0])
    for (auto& e : c->ev) SBDX_CUDA(c, cudaEventCreate(&e));
  c->profiling = true;
  const int same_cand[] = {32, 34, 38, 24, 28, 22};
  const int ab_cand[] = {71, 62, 61, 63, 64};
  for (int prec = 0; prec < 2 && rc == 0; ++prec) {
    const Tune saved = c->tune[prec];
    auto measure = [&](int same, int ab, double* same_ms, double* ab_ms) -> int {
      c->tune[prec].same_code = same;
      c->tune[prec].ab_code = ab;
      int r2 = prec == 0 ? run_sigma<double>(c, (const double*)X, (double*)S)
                         : run_sigma<float>(c, (const float*)X, (float*)S);
      if (r2) return r2;
      for (double& x : c->phase_ms) x = 0.0;
      c->phase_calls = 0;
      for (int k = 0; k < 2 && r2 == 0; ++k)
        r2 = prec == 0 ? run_sigma<double>(c, (const double*)X, (double*)S)
                       : run_sigma<float>(c, (const float*)X, (float*)S);
      *same_ms = c->phase_ms[0] + c->phase_ms[2];
      *ab_ms = c->phase_ms[3];
      return r2;
    };
    int best_same = 0, best_ab = 0;
    double t_same = 1e300, t_ab = 1e300;
    for (int sc : same_cand) {
      double sm = 0, ab = 0;
      if ((rc = measure(sc, ab_cand[0], &sm, &ab))) break;
      if (sm < t_same) { t_same = sm; best_same = sc; }
    }
    for (int ac : ab_cand) {
      if (rc) break;
      double sm = 0, ab = 0;
      if ((rc = measure(best_same, ac, &sm, &ab))) break;
      if (ab < t_ab) { t_ab = ab; best_ab = ac; }
    }
    if (rc) { c->tune[prec] = saved; break; }
    c->tune[prec].same_code = best_same;
    c->tune[prec].ab_code = best_ab;
  }
  c->profiling = prof0;
  for (double& x : c->phase_ms) x = 0.0;
  c->phase_calls = 0;
  cudaFreeAsync(X, c->stream);
  cudaFreeAsync(S, c->stream);
  pool_trim(c);
  if (rc) return rc;
  SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
  return 0;
}

void clear_sigma_graphs(Ctx* c) {
  for (auto& g : c->graphs) cudaGraphExecDestroy(g.exec);
  c->graphs.clear();
}

namespace {

int run_sigma_any(Ctx* c, int precision, const void* X, void* S) {
  if (precision == 0) return run_sigma<double>(c, (const double*)X, (double*)S);
  return run_sigma<float>(c, (const float*)X, (float*)S);
}

// Replays the captured graph of this (precision, X, S), capturing it first.
// Returns -1 (nothing launched) when capture is not possible here, so that
// the caller runs the sigma directly.
int sigma_graph(Ctx* c, int precision, const void* X, void* S) {
  for (const auto& g : c->graphs)
    if (g.precision == precision && g.X == X && g.S == S) {
      SBDX_CUDA(c, cudaGraphLaunch(g.exec, c->stream));
      c->launches += g.kernels;
      return 0;
    }
  if (c->graphs.size() >= 96) clear_sigma_graphs(c);
  const unsigned long long before = c->launches;
  if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  const int rc = run_sigma_any(c, precision, X, S);
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
  const unsigned long long kernels = c->launches - before;
  c->launches = before;
  if (rc != 0 || e != cudaSuccess || graph == nullptr) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return rc != 0 ? rc : -1;
  }
  cudaGraphExec_t exec = nullptr;
  const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ei != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  c->graphs.push_back({precision, X, S, exec, kernels});
  SBDX_CUDA(c, cudaGraphLaunch(exec, c->stream));
  c->launches += kernels;
  return 0;
}

}  // namespace

int sigma_rows_device(Ctx* c, int precision, const void* X, void* S, size_t a0, size_t a1) {
  if (a0 > a1 || a1 > c->na) {
    c->err = "sigma_rows: need a0 <= a1 <= na";
    return SBDX_ERR_ARG;
  }
  if (a0 % 8 != 0 && a0 != a1) {
    c->err = "sigma_rows: the first row must be a multiple of 8";
    return SBDX_ERR_ARG;
  }
  if (precision != 0 && precision != 1) {
    c->err = "sigma_rows: precision must be SBDX_FP64 or SBDX_FP32";
    return SBDX_ERR_ARG;
  }
  if (precision == 0 && c->stored.val != nullptr) {
    c->err = "sigma_rows: a row range is evaluated on the fly; release the stored Hamiltonian first";
    return SBDX_ERR_STATE;
  }
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
  const bool f64 = precision == 0;
  Tune t = effective_tune(c, f64);
  if (!is_v6(t)) t = default_tune(c, f64);  // the row range runs the alpha-first kernels
  if (!ab7_fits(c)) {
    c->err = "sigma_rows: the packed alpha-beta kernel cannot stage this problem's rows";
    return SBDX_ERR_ARG;
  }
  if (!c->have_range || c->range_a0 != a0 || c->range_a1 != a1) {
    if ((rc = build_row_range(c, a0, a1))) return rc;
  }
  if (f64) return run_sigma_rows<double>(c, t, static_cast<const double*>(X), static_cast<double*>(S), a0, a1);
  return run_sigma_rows<float>(c, t, static_cast<const float*>(X), static_cast<float*>(S), a0, a1);
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
  if (precision != 0 && precision != 1) {
    c->err = "sigma: precision must be SBDX_FP64 or SBDX_FP32";
    return 1;
  }
  if (precision == 0 && c->stored.val != nullptr)
    return stored_sigma(c, static_cast<const double*>(X), static_cast<double*>(S));
  if (c->use_graphs && !c->profiling && c->stream != nullptr) {
    rc = sigma_graph(c, precision, X, S);
    if (rc >= 0) return rc;
    c->use_graphs = false;  // capture unavailable: plain launches from now on
  }
  return run_sigma_any(c, precision, X, S);
}

// ---- the host-buffer sigma, copies overlapped with the kernels ----------------
//
// S = H C from host C to host S in chunks of alpha rows, each one contiguous
// block of both vectors (alpha-major layout). A copy stream brings chunk i in
// while the context stream runs, for every chunk that has arrived, the phase
// split of its rows and the beta same-spin product on its columns of the
// transpose (which read that chunk only). Once every chunk is in, the context
// stream runs the alpha-beta product of all rows (it reads any ket row), then
// per chunk the alpha same-spin work items of its rows, added to the
// alpha-beta result, and the combine of its rows; the copy stream takes each
// finished chunk out while the next one computes. Exposed: the first chunk's
// copy in, the last chunk's beta same-spin product and the last chunk's copy
// out.

namespace {

constexpr size_t kIoChunkDets = size_t(8) << 20;  // determinants per chunk in automatic mode
constexpr int kIoMaxChunks = 8;

int io_chunk_count(const Ctx* c) {
  if (c->io_chunks_req == 1) return 1;
  const size_t D = c->na * c->nb;
  // automatic: the nearest whole number of kIoChunkDets chunks (64 M
  // determinants: 8 chunks, 40.6 ms end to end against 41.4 ms with 7)
  int k = c->io_chunks_req >= 2 ? c->io_chunks_req
                                : (int)std::min<size_t>(kIoMaxChunks, (D + kIoChunkDets / 2) / kIoChunkDets);
  k = std::min<int>(k, (int)(c->na / 8));  // at least 8 rows per chunk
  return std::max(k, 1);
}

// chunk boundaries for K chunks: equal row counts, multiples of 8
std::vector<size_t> io_bounds_for(const Ctx* c, int K) {
  const size_t na = c->na;
  std::vector<size_t> b{0};
  for (int i = 1; i < K; ++i) {
    const size_t x = na * (size_t)i / (size_t)K / 8 * 8;
    if (x > b.back() && x < na) b.push_back(x);
  }
  b.push_back(na);
  return b;
}

int build_io_chunks(Ctx* c, const std::vector<size_t>& bounds) {
  free_io_chunks(c);
  const size_t n = bounds.size() - 1;
  c->io_items.resize(n);
  for (size_t i = 0; i < n; ++i) {
    const int rc = build_range_items(c, bounds[i], bounds[i + 1], c->io_items[i]);
    if (rc) return rc;
  }
  SBDX_CUDA(c, cudaStreamCreateWithFlags(&c->io_copy, cudaStreamNonBlocking));
  c->io_events.assign(2 * n + 2, nullptr);
  for (auto& e : c->io_events) SBDX_CUDA(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  c->io_bounds = bounds;  // last: a build that failed part way leaves no bounds, so the next call rebuilds
  return 0;
}

}  // namespace

void free_io_chunks(Ctx* c) {
  for (auto& r : c->io_items) free_range_items(r);
  c->io_items.clear();
  c->io_bounds.clear();
  for (auto e : c->io_events)
    if (e) cudaEventDestroy(e);
  c->io_events.clear();
  if (c->io_copy) cudaStreamDestroy(c->io_copy);
  c->io_copy = nullptr;
}

int sigma_host(Ctx* c, const double* hC, double* hS) {
  const size_t na = c->na, nb = c->nb, D = na * nb;
  int rc;
  if (!c->have_conn && (rc = build_connectivity(c))) return rc;
  if (!c->have_hii && (rc = diag_terms(c))) return rc;
  if ((rc = ensure_sigma_scratch(c))) return rc;
  double* din = static_cast<double*>(c->d_io_in);
  double* dout = static_cast<double*>(c->d_io_out);
  const Tune t = effective_tune(c, true);
  const int K = io_chunk_count(c);
  const bool pipe = K >= 2 && c->stored.val == nullptr && is_v6(t) && t.ab_code == 71 && ab7_fits(c) &&
                    !c->profiling;
  if (!pipe) {  // one copy in, the sigma, one copy out
    SBDX_CUDA(c, cudaMemcpyAsync(din, hC, sizeof(double) * D, cudaMemcpyHostToDevice, c->stream));
    if ((rc = sigma_device(c, SBDX_FP64, din, dout))) return rc;
    SBDX_CUDA(c, cudaMemcpyAsync(hS, dout, sizeof(double) * D, cudaMemcpyDeviceToHost, c->stream));
    return 0;
  }
  const std::vector<size_t> want = io_bounds_for(c, K);
  if (want != c->io_bounds) {
    if ((rc = build_io_chunks(c, want))) return rc;
  }
  const size_t n = c->io_bounds.size() - 1;
  const std::vector<size_t>& b = c->io_bounds;
  cudaEvent_t* ev = c->io_events.data();  // [0, n): chunk in; [n, 2n): chunk out ready; 2n: start; 2n + 1: end
  const Conn& ca = c->conn[0];
  const Conn& cb = c->conn[1];
  double* xp = static_cast<double*>(c->d_xp);
  double* xpt = static_cast<double*>(c->d_xt);
  // the copies in follow whatever the context stream was doing
  SBDX_CUDA(c, cudaEventRecord(ev[2 * n], c->stream));
  SBDX_CUDA(c, cudaStreamWaitEvent(c->io_copy, ev[2 * n], 0));
  for (size_t i = 0; i < n; ++i) {
    const size_t off = b[i] * nb, len = (b[i + 1] - b[i]) * nb;
    SBDX_CUDA(c, cudaMemcpyAsync(din + off, hC + off, sizeof(double) * len, cudaMemcpyHostToDevice, c->io_copy));
    SBDX_CUDA(c, cudaEventRecord(ev[i], c->io_copy));
  }
  for (size_t i = 0; i < n; ++i) {  // per arrived chunk: phase split, beta same-spin on its columns
    const size_t a0 = b[i], nr = b[i + 1] - b[i];
    SBDX_CUDA(c, cudaStreamWaitEvent(c->stream, ev[i], 0));
    const dim3 grid((unsigned)((nb + 31) / 32), (unsigned)((nr + 31) / 32));
    phase_split_kernel<double><<<grid, dim3(32, 8), 0, c->stream>>>(din + a0 * nb, nr, nb, c->d_a + a0, c->d_b,
                                                                     xp + a0 * c->xsa, xpt + a0, c->xsa, c->xsb);
    SBDX_LAUNCHED(c);
    if ((rc = run_same_v6<double>(c, t.same_code, xpt + a0, nb, nr, c->xsb, cb, cb.val, c->d_Da + a0, c->da_stride,
                                  nullptr, c->d_yt + a0)))
      return rc;
  }
  // the alpha-beta product of all rows in one launch (its work items keep
  // the whole grid busy, longest first) into a zeroed Y, then per chunk the
  // alpha same-spin items of its rows added to Y, and the combine
  SBDX_CUDA(c, cudaMemsetAsync(c->d_y, 0, sizeof(double) * na * c->xsa, c->stream));
  if ((rc = run_ab_v7<double>(c, xp))) return rc;
  for (size_t i = 0; i < n; ++i) {
    const size_t a0 = b[i], nr = b[i + 1] - b[i];
    const Conn& it = c->io_items[i];
    Conn ra = ca;
    ra.blk = it.blk;
    ra.same_item = it.same_item;
    ra.n_same_item = it.n_same_item;
    ra.same_split = it.same_split;
    ra.n_same_split = it.n_same_split;
    ra.n_same_part = it.n_same_part;
    ra.same_ypart = it.same_ypart;
    if ((rc = run_same_v6<double>(c, t.same_code, xp, na, nb, c->xsa, ra, ca.val, c->d_Db, c->db_stride, c->d_hii,
                                  c->d_y, 1)))
      return rc;
    const dim3 grid((unsigned)((nb + 31) / 32), (unsigned)((nr + 31) / 32));
    combine_phase_kernel<double><<<grid, dim3(32, 8), 0, c->stream>>>(c->d_y + a0 * c->xsa, c->d_yt + a0, nr, nb,
                                                                       c->d_a + a0, c->d_b, dout + a0 * nb, c->xsa,
                                                                       c->xsb);
    SBDX_LAUNCHED(c);
    SBDX_CUDA(c, cudaEventRecord(ev[n + i], c->stream));
  }
  for (size_t i = 0; i < n; ++i) {  // each chunk out as soon as it is ready
    const size_t off = b[i] * nb, len = (b[i + 1] - b[i]) * nb;
    SBDX_CUDA(c, cudaStreamWaitEvent(c->io_copy, ev[n + i], 0));
    SBDX_CUDA(c, cudaMemcpyAsync(hS + off, dout + off, sizeof(double) * len, cudaMemcpyDeviceToHost, c->io_copy));
  }
  SBDX_CUDA(c, cudaEventRecord(ev[2 * n + 1], c->io_copy));
  SBDX_CUDA(c, cudaStreamWaitEvent(c->stream, ev[2 * n + 1], 0));  // the call's work ends on the context stream
  return 0;
}

}  // namespace sbdx
