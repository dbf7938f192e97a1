// 1-/2-particle reduced density matrices, occupation density, alpha-string
// weights and the energy adjoint.
//
// Restates Correlation (reference chemistry/tpb/correlation.h:194-444) with
// ZeroDiffCorrelation (:15-44), OneDiffCorrelation (:49-86) and
// TwoDiffCorrelation (:91-130): the same element indices and signs, summed in
// a different order. The reference accumulates every (bra, ket) pair into a
// per-thread copy of the 4*L^4 array; here the sums are regrouped so that
// global atomics are per connectivity entry, not per determinant pair:
//   - diagonal: per bra row, the row weight sum_c W^2 and the opposite-spin
//     occupation profile sum_c W^2 n_q(c) (one CTA per row), then an L x L
//     finalize;
//   - same-spin singles/doubles: one warp per connectivity entry (r -> k)
//     reduces sum_c W[r,c] W[k,c] (-1)^{opposite-spin parity} over the
//     opposite-spin index c (and, for singles, its n_q-weighted profile);
//     the beta task runs on W^T;
//   - alpha-single x beta-single: one CTA per bra alpha row stages W[ja, :]
//     in shared memory and folds all (ib, jb) pairs of each beta excitation
//     pattern (i_b, a_b) into an L x L shared accumulator before flushing.
// Layout: one[s*L^2 + p + L q], two[(s + 2t)*L^4 + i + L j + L^2 k + L^3 l].
#include "sbdx_internal.cuh"

#include <algorithm>
#include <vector>

namespace sbdx {

int ensure_sigma_scratch(Ctx* c);

namespace {


// Reference parity(det, start, end) (determinants.h:228-279) on the
// interleaved determinant of (alpha, beta): returns the sign bit (1 = -1).
__device__ __forceinline__ uint32_t ref_parity_bit(uint64_t a, uint64_t b, int start, int end) {
  const uint64_t ma = range_mask((start + 1) >> 1, (end + 1) >> 1);
  const uint64_t mb = range_mask(start >> 1, end >> 1);
  const uint64_t sw = (start & 1) ? b : a;
  return (uint32_t)(popc64(a & ma) + popc64(b & mb) + (int)((sw >> (start >> 1)) & 1ull)) & 1u;
}

// Row weights and occupation profiles of one orientation of W (rows x cols),
// without atomics: wrow[r] = sum_c W[r,c]^2 (lane-strided sums, a fixed
// shuffle tree, warps added in order) and, when vq is not null, the row's
// opposite-spin occupation profile vq[r*L + q] = sum_c W[r,c]^2 n_q(s_col[c])
// (per-thread shared accumulators of L doubles, added in thread order).
constexpr int kRowWeightThreads = 64;
__global__ void __launch_bounds__(kRowWeightThreads)
row_weight_kernel(const double* __restrict__ W, size_t cols, const uint64_t* __restrict__ s_col, int L,
                  double* __restrict__ wrow, double* __restrict__ vq) {
  extern __shared__ double acc_q[];  // [thread][L] when vq != null
  __shared__ double red[kRowWeightThreads / 32];
  const size_t r = blockIdx.x;
  double* mine = acc_q + (size_t)threadIdx.x * L;
  if (vq != nullptr)
    for (int q = 0; q < L; ++q) mine[q] = 0.0;
  double s = 0.0;
  for (size_t c = threadIdx.x; c < cols; c += blockDim.x) {
    const double w = W[r * cols + c];
    const double w2 = w * w;
    s += w2;
    if (vq != nullptr && w2 != 0.0) {
      uint64_t bits = s_col[c];
      while (bits) {
        const int q = __ffsll((long long)bits) - 1;
        bits &= bits - 1;
        mine[q] += w2;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kRowWeightThreads / 32; ++w) t += red[w];
    wrow[r] = t;
  }
  if (vq != nullptr)
    for (int q = threadIdx.x; q < L; q += blockDim.x) {
      double v = 0.0;
      for (int t = 0; t < kRowWeightThreads; ++t) v += acc_q[(size_t)t * L + q];
      vq[r * L + q] = v;
    }
}

// P[p][q] = sum_r wrow[r] over the rows whose string holds p and q, and (if X
// is not null) X[p][q] = sum_r vq[r][q] over the rows whose string holds p:
// one thread per (p, q), rows in order.
__global__ void occupation_sums_kernel(size_t rows, const uint64_t* __restrict__ s_row, int L,
                                       const double* __restrict__ wrow, const double* __restrict__ vq,
                                       double* __restrict__ P, double* __restrict__ X) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= L * L) return;
  const int p = t / L, q = t % L;
  double a = 0.0, b = 0.0;
  for (size_t r = 0; r < rows; ++r) {
    const uint64_t own = s_row[r];
    if (!((own >> p) & 1ull)) continue;
    if ((own >> q) & 1ull) a += wrow[r];
    if (X != nullptr) b += vq[r * L + q];
  }
  P[t] = a;
  if (X != nullptr) X[t] = b;
}

// Diagonal (ZeroDiffCorrelation) contributions from P_alpha, P_beta, X.
__global__ void diag_finalize_kernel(int L, const double* __restrict__ Pa, const double* __restrict__ Pb,
                                     const double* __restrict__ X, double* __restrict__ one, double* __restrict__ two) {
  const size_t L2 = (size_t)L * L, L3 = L2 * L, L4 = L3 * L;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= L * L) return;
  const int p = t / L, q = t % L;
  const size_t d = (size_t)p + L * q + L2 * p + L3 * q;   // [p, q, p, q]
  const size_t x = (size_t)p + L * q + L2 * q + L3 * p;   // [p, q, q, p]
  if (p == q) {
    one[(size_t)p + L * p] += Pa[t];
    one[L2 + (size_t)p + L * p] += Pb[t];
  }
  if (two == nullptr) return;  // the 1-RDM alone
  if (p != q) {
    two[0 * L4 + d] += Pa[t];
    two[0 * L4 + x] -= Pa[t];
    two[3 * L4 + d] += Pb[t];
    two[3 * L4 + x] -= Pb[t];
  }
  // opposite spins: alpha p, beta q -> block 2 at [p,q,p,q], block 1 at [q,p,q,p]
  const double v = X[t];
  two[2 * L4 + d] += v;
  two[1 * L4 + (size_t)q + L * p + L2 * q + L3 * p] += v;
}

// Same-spin singles and doubles without atomics. The entries of one spin are
// grouped by excitation pattern on the host (singles: hole, particle;
// doubles: both holes and both particles), each group in ascending bra then
// ket order. Pass 1 (rdm_same_values_kernel, one warp per entry) evaluates the
// entry's value s = sum_c W[r,c] W[k,c] (-1)^{opposite-spin parity} over the
// opposite-spin index c (lane c mod 32, then a fixed shuffle tree) and, for a
// single when the 2-RDM is wanted, its opposite-spin occupation profile
// prof[q] = sum_c (the same terms) n_q(c) (per-lane shared accumulators added
// in lane order). Pass 2 (rdm_singles_finalize_kernel,
// rdm_doubles_finalize_kernel) gives every output element one thread, which
// adds its group's values in group order: the result does not depend on the
// launch. Indices and signs are those of OneDiffCorrelation and
// TwoDiffCorrelation (correlation.h:49-130).
constexpr int kValWarps = 4;

// Dynamic shared memory: kValWarps * 32 * L doubles when profile != 0.
__global__ void __launch_bounds__(kValWarps * 32)
rdm_same_values_kernel(const double* __restrict__ W, size_t cols, const uint64_t* __restrict__ s_row,
                       const uint64_t* __restrict__ s_col, const uint32_t* __restrict__ ket,
                       const uint64_t* __restrict__ omask, const uint32_t* __restrict__ info,
                       const uint32_t* __restrict__ ent, const uint32_t* __restrict__ erow, size_t n, int L,
                       int profile, double* __restrict__ sval, double* __restrict__ prof) {
  extern __shared__ double vq_all[];  // [warp][lane][L]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t t = (size_t)blockIdx.x * kValWarps + warp;
  double* vq = vq_all + ((size_t)warp * 32 + lane) * L;
  if (profile)
    for (int q = 0; q < L; ++q) vq[q] = 0.0;
  if (t >= n) return;
  const size_t e = ent[t], r = erow[t], k = ket[e];
  const uint32_t inf = info[e];
  const uint64_t om = omask[e];
  const uint64_t sr = s_row[r];
  uint32_t sbit;
  if (inf & kInfoSingle) {
    sbit = inf >> 31;
  } else {
    const int i_e = (int)(inf & 63u), j_e = (int)((inf >> 6) & 63u);
    const int a_e = (int)((inf >> 12) & 63u), b_e = (int)((inf >> 18) & 63u);
    // TwoDiffCorrelation sign on the bra: I = a_e, J = b_e (bra-only), A = i_e,
    // B = j_e (ket-only); same-spin part here, opposite-spin part via omask
    int par = 0;
    {
      const int lo = a_e < i_e ? a_e : i_e, hi = a_e < i_e ? i_e : a_e;
      par += popc64(sr & range_mask(lo, hi)) + (int)((sr >> lo) & 1ull);
    }
    {
      const int lo = b_e < j_e ? b_e : j_e, hi = b_e < j_e ? j_e : b_e;
      par += popc64(sr & range_mask(lo, hi)) + (int)((sr >> lo) & 1ull);
    }
    if (i_e > b_e || j_e < a_e) par += 1;
    sbit = (uint32_t)(par & 1);
  }
  double s = 0.0;
  const double* wr = W + r * cols;
  const double* wk = W + k * cols;
  for (size_t c = lane; c < cols; c += 32) {
    const double x = wr[c] * wk[c];
    if (x == 0.0) continue;
    const uint64_t o = s_col[c];
    const double v = ((sbit ^ (uint32_t)popc64(o & om)) & 1u) ? -x : x;
    s += v;
    if (profile) {
      uint64_t bits = o;
      while (bits) {
        const int q = __ffsll((long long)bits) - 1;
        bits &= bits - 1;
        vq[q] += v;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) sval[t] = s;
  if (profile) {
    __syncwarp();
    for (int q = lane; q < L; q += 32) {
      double v = 0.0;
      for (int l = 0; l < 32; ++l) v += vq_all[((size_t)warp * 32 + l) * L + q];
      prof[t * (size_t)L + q] = v;
    }
  }
}

// Singles of spin `spin`, one thread per (group, x): x = 0 the 1-RDM element
// gamma[particle + L hole]; x = 1 + oj (oj < L) the four same-spin 2-RDM
// elements of the bra orbital oj (oj = the particle: they cancel, skipped);
// x = 1 + L + q the two opposite-spin elements of the profile orbital q.
__global__ void rdm_singles_finalize_kernel(int spin, int L, const uint32_t* __restrict__ gkey,
                                            const uint32_t* __restrict__ goff, size_t ngroups,
                                            const uint32_t* __restrict__ erow, const uint64_t* __restrict__ s_row,
                                            const double* __restrict__ sval, const double* __restrict__ prof,
                                            double* __restrict__ one, double* __restrict__ two) {
  const int nx = two ? 1 + 2 * L : 1;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ngroups * nx) return;
  const size_t g = t / nx;
  const int x = (int)(t % nx);
  const uint32_t key = gkey[g];
  const int oa = (int)(key & 63u), oi = (int)((key >> 6) & 63u);  // hole (ket-only), particle (bra-only)
  const size_t L2 = (size_t)L * L, L3 = L2 * L, L4 = L3 * L;
  if (x == 0) {
    double v = 0.0;
    for (uint32_t q = goff[g]; q < goff[g + 1]; ++q) v += sval[q];
    one[(size_t)spin * L2 + oi + (size_t)L * oa] += v;
    return;
  }
  const int ss = 3 * spin;
  if (x <= L) {
    const int oj = x - 1;
    if (oj == oi) return;
    double v = 0.0;
    for (uint32_t q = goff[g]; q < goff[g + 1]; ++q)
      if ((s_row[erow[q]] >> oj) & 1ull) v += sval[q];
    if (v == 0.0) return;
    two[ss * L4 + oa + (size_t)L * oj + L2 * oi + L3 * oj] += v;
    two[ss * L4 + oj + (size_t)L * oa + L2 * oj + L3 * oi] += v;
    two[ss * L4 + oa + (size_t)L * oj + L2 * oj + L3 * oi] -= v;
    two[ss * L4 + oj + (size_t)L * oa + L2 * oi + L3 * oj] -= v;
    return;
  }
  const int qo = x - 1 - L;
  double v = 0.0;
  for (uint32_t q = goff[g]; q < goff[g + 1]; ++q) v += prof[(size_t)q * L + qo];
  if (v == 0.0) return;
  const int so = spin + 2 * (1 - spin), os = (1 - spin) + 2 * spin;
  two[so * L4 + oa + (size_t)L * qo + L2 * oi + L3 * qo] += v;
  two[os * L4 + qo + (size_t)L * oa + L2 * qo + L3 * oi] += v;
}

// Doubles of spin `spin`, one thread per group (i, j ket-only; a, b bra-only).
__global__ void rdm_doubles_finalize_kernel(int spin, int L, const uint32_t* __restrict__ gkey,
                                            const uint32_t* __restrict__ goff, size_t ngroups,
                                            const double* __restrict__ sval, double* __restrict__ two) {
  const size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngroups) return;
  double s = 0.0;
  for (uint32_t q = goff[g]; q < goff[g + 1]; ++q) s += sval[q];
  if (s == 0.0) return;
  const uint32_t key = gkey[g];
  const size_t i_e = key & 63u, j_e = (key >> 6) & 63u, a_e = (key >> 12) & 63u, b_e = (key >> 18) & 63u;
  const size_t L2 = (size_t)L * L, L4 = L2 * L2;
  const int ss = 3 * spin;
  two[ss * L4 + i_e + (size_t)L * j_e + L2 * (a_e + (size_t)L * b_e)] += s;
  two[ss * L4 + j_e + (size_t)L * i_e + L2 * (b_e + (size_t)L * a_e)] += s;
  two[ss * L4 + i_e + (size_t)L * j_e + L2 * (b_e + (size_t)L * a_e)] -= s;
  two[ss * L4 + j_e + (size_t)L * i_e + L2 * (a_e + (size_t)L * b_e)] -= s;
}

// Alpha single x beta single pairs (task type 0). One CTA per bra alpha row.
__global__ void __launch_bounds__(512)
rdm_ab_kernel(const double* __restrict__ W, size_t nb, const uint64_t* __restrict__ astr,
              const uint64_t* __restrict__ bstr, const uint64_t* __restrict__ a_off,
              const uint32_t* __restrict__ a_nsing, const uint32_t* __restrict__ a_ket,
              const uint32_t* __restrict__ a_info, const uint64_t* __restrict__ b_off,
              const uint32_t* __restrict__ b_nsing, const uint32_t* __restrict__ b_ket,
              const uint32_t* __restrict__ b_info, int L, double* __restrict__ two, int staged) {
  extern __shared__ __align__(16) unsigned char smem[];
  double* acc = reinterpret_cast<double*>(smem);  // [L*L] by (i_b, a_b)
  double* ws = acc + (size_t)L * L;               // [nb] when staged
  const size_t ia = blockIdx.x;
  const uint64_t alpha_bra = astr[ia];
  const double* wbra = W + ia * nb;
  const size_t L2 = (size_t)L * L, L3 = L2 * L, L4 = L3 * L;
  const uint32_t ns = a_nsing[ia];
  for (uint32_t k = 0; k < ns; ++k) {
    const uint64_t e = a_off[ia] + k;
    const size_t ja = a_ket[e];
    const uint32_t inf = a_info[e];
    const int ia_h = (int)(inf & 63u);          // alpha ket-only orbital i_a
    const int ia_p = (int)((inf >> 6) & 63u);   // alpha bra-only orbital a_a
    __syncthreads();
    for (int t = threadIdx.x; t < L * L; t += blockDim.x) acc[t] = 0.0;
    // the ket row W[ja, :] in shared memory, or read from global memory
    // (L2) when a beta row does not fit
    const double* wket = staged ? ws : W + ja * nb;
    if (staged)
      for (size_t t = threadIdx.x; t < nb; t += blockDim.x) ws[t] = W[ja * nb + t];
    __syncthreads();
    for (size_t ib = threadIdx.x; ib < nb; ib += blockDim.x) {
      const double wi = wbra[ib];
      if (wi == 0.0) continue;
      const uint64_t beta_bra = bstr[ib];
      const uint64_t m0 = b_off[ib], m1 = m0 + b_nsing[ib];
      for (uint64_t m = m0; m < m1; ++m) {
        const double wj = wket[b_ket[m]];
        if (wj == 0.0) continue;
        const uint32_t i2 = b_info[m];
        const int ib_h = (int)(i2 & 63u), ib_p = (int)((i2 >> 6) & 63u);
        // c = bra-only {2 a_a, 2 a_b + 1}, d = ket-only {2 i_a, 2 i_b + 1}
        const int c0 = 2 * ia_p, c1 = 2 * ib_p + 1, d0 = 2 * ia_h, d1 = 2 * ib_h + 1;
        const int I = c0 < c1 ? c0 : c1, J = c0 < c1 ? c1 : c0;
        const int A = d0 < d1 ? d0 : d1, B = d0 < d1 ? d1 : d0;
        const uint32_t par = ref_parity_bit(alpha_bra, beta_bra, I < A ? I : A, I < A ? A : I) ^
                             ref_parity_bit(alpha_bra, beta_bra, J < B ? J : B, J < B ? B : J);
        const double v = wi * wj;
        atomicAdd(&acc[ib_h * L + ib_p], par ? -v : v);
      }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < L * L; t += blockDim.x) {
      const double v0 = acc[t];
      if (v0 == 0.0) continue;
      const int ib_h = t / L, ib_p = t % L;
      const int c0 = 2 * ia_p, c1 = 2 * ib_p + 1, d0 = 2 * ia_h, d1 = 2 * ib_h + 1;
      const int I = c0 < c1 ? c0 : c1, J = c0 < c1 ? c1 : c0;
      const int A = d0 < d1 ? d0 : d1, B = d0 < d1 ? d1 : d0;
      const double sg = (A > J || B < I) ? -v0 : v0;
      const int oi = I >> 1, si = I & 1, oa = A >> 1, sa = A & 1, oj = J >> 1, sj = J & 1, ob = B >> 1;
      if (si == sa) {
        atomicAdd(&two[(si + 2 * sj) * L4 + oa + (size_t)L * ob + L2 * (oi + (size_t)L * oj)], sg);
        atomicAdd(&two[(sj + 2 * si) * L4 + ob + (size_t)L * oa + L2 * (oj + (size_t)L * oi)], sg);
      } else {
        atomicAdd(&two[(si + 2 * sj) * L4 + oa + (size_t)L * ob + L2 * (oj + (size_t)L * oi)], -sg);
        atomicAdd(&two[(sj + 2 * si) * L4 + ob + (size_t)L * oa + L2 * (oi + (size_t)L * oj)], -sg);
      }
    }
  }
}

// Alpha single x beta single pairs (task type 0), without atomics: the
// singles of each spin are grouped by their excitation pattern (hole, particle),
// and the contribution of a pair depends on the pair of patterns only through
// the two reference parities, which split into an alpha-string part and a
// beta-string part. A CTA takes a chunk of at most kAbChunk alpha singles of
// one alpha pattern; per alpha single (bra ia -> ket ja) it stages the rows
// W[ia, :] and W[ja, :] in shared memory, and warp w sums, for the beta
// patterns w, w + 16, ..., all their beta singles (bra ib -> ket jb) of
// +-W[ia, ib] W[ja, jb] in a fixed lane order and shuffle tree; the warp owns
// those patterns' accumulators, so every sum has one fixed order. The chunk's
// sums go to partial[chunk][beta pattern]; rdm_ab_sum_kernel adds the chunks
// of one alpha pattern in order and rdm_ab_write_kernel writes the 2-RDM
// elements (no other kernel writes them).
constexpr int kAbChunk = 32;
constexpr int kAbDetThreads = 512;

// Combined parity mask of the two reference parity() calls of a pair (one
// per spin of the string): parity(det, s, e) on the interleaved determinant
// counts alpha orbitals in [(s+1)/2, (e+1)/2), beta orbitals in [s/2, e/2) and
// the spin-orbital s itself; the parity of a sum of popcounts is the popcount
// of the XOR of the masks.
__device__ __forceinline__ void pair_parity_masks(int s1, int e1, int s2, int e2, uint64_t& ma, uint64_t& mb) {
  ma = range_mask((s1 + 1) >> 1, (e1 + 1) >> 1) ^ range_mask((s2 + 1) >> 1, (e2 + 1) >> 1);
  mb = range_mask(s1 >> 1, e1 >> 1) ^ range_mask(s2 >> 1, e2 >> 1);
  if (s1 & 1) mb ^= 1ull << (s1 >> 1); else ma ^= 1ull << (s1 >> 1);
  if (s2 & 1) mb ^= 1ull << (s2 >> 1); else ma ^= 1ull << (s2 >> 1);
}

__global__ void __launch_bounds__(kAbDetThreads)
rdm_ab_det_kernel(const double* __restrict__ W, size_t nb, const uint64_t* __restrict__ astr,
                  const uint64_t* __restrict__ bstr, const uint4* __restrict__ chunks,
                  const uint64_t* __restrict__ arec, const uint32_t* __restrict__ bpat_off,
                  const uint32_t* __restrict__ bpat_key, const uint64_t* __restrict__ brec, int npb,
                  double* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char smem[];
  double* wi = reinterpret_cast<double*>(smem);  // [nb] row ia
  double* wj = wi + nb;                          // [nb] row ja
  double* acc = wj + nb;                         // [npb]
  const uint4 ch = chunks[blockIdx.x];           // {alpha pattern key, first single, count, 0}
  const int ia_h = (int)(ch.x >> 6), ia_p = (int)(ch.x & 63u);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int kWarps = kAbDetThreads / 32;
  for (int p = threadIdx.x; p < npb; p += kAbDetThreads) acc[p] = 0.0;
  for (uint32_t q = 0; q < ch.z; ++q) {
    const uint64_t ar = arec[ch.y + q];
    const size_t ia = (uint32_t)ar, ja = ar >> 32;
    __syncthreads();
    for (size_t t = threadIdx.x; t < nb; t += kAbDetThreads) {
      wi[t] = W[ia * nb + t];
      wj[t] = W[ja * nb + t];
    }
    __syncthreads();
    const uint64_t alpha_bra = astr[ia];
    for (int p = warp; p < npb; p += kWarps) {
      const uint32_t key = bpat_key[p];
      const int ib_h = (int)(key >> 6), ib_p = (int)(key & 63u);
      const int c0 = 2 * ia_p, c1 = 2 * ib_p + 1, d0 = 2 * ia_h, d1 = 2 * ib_h + 1;
      const int I = c0 < c1 ? c0 : c1, J = c0 < c1 ? c1 : c0;
      const int A = d0 < d1 ? d0 : d1, B = d0 < d1 ? d1 : d0;
      uint64_t ma, mb;
      pair_parity_masks(I < A ? I : A, I < A ? A : I, J < B ? J : B, J < B ? B : J, ma, mb);
      const uint32_t pa = (uint32_t)popc64(alpha_bra & ma) & 1u;
      double s = 0.0;
      for (uint32_t m = bpat_off[p] + lane; m < bpat_off[p + 1]; m += 32) {
        const uint64_t br = brec[m];
        const uint32_t ib = (uint32_t)br, jb = (uint32_t)(br >> 32);
        const double v = wi[ib] * wj[jb];
        const uint32_t par = (pa + (uint32_t)popc64(bstr[ib] & mb)) & 1u;
        s += par ? -v : v;
      }
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
      if (lane == 0) acc[p] += s;
    }
  }
  __syncthreads();
  for (int p = threadIdx.x; p < npb; p += kAbDetThreads) partial[(size_t)blockIdx.x * npb + p] = acc[p];
}

// Sum of the chunks of each alpha pattern (in chunk order) for every beta
// pattern: G[alpha pattern][beta pattern].
__global__ void rdm_ab_sum_kernel(const uint4* __restrict__ apat, int npa, int npb, const double* __restrict__ partial,
                                  double* __restrict__ G) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)npa * npb) return;
  const int pa = (int)(t / npb), p = (int)(t % npb);
  const uint4 ap = apat[pa];  // {alpha pattern key, first chunk, chunks, 0}
  double v = 0.0;
  for (uint32_t q = 0; q < ap.z; ++q) v += partial[(size_t)(ap.y + q) * npb + p];
  G[t] = v;
}

// The two 2-RDM elements of the pattern pair (alpha hole h1, particle p1;
// beta hole h2, particle p2) and the sign with which its sum enters each: the
// indices and operator-order sign of TwoDiffCorrelation (correlation.h:91-130).
__device__ __forceinline__ void ab_targets(int h1, int p1, int h2, int p2, int L, size_t (&e)[2], double (&sg)[2]) {
  const size_t L2 = (size_t)L * L, L3 = L2 * L, L4 = L3 * L;
  const int c0 = 2 * p1, c1 = 2 * p2 + 1, d0 = 2 * h1, d1 = 2 * h2 + 1;
  const int I = c0 < c1 ? c0 : c1, J = c0 < c1 ? c1 : c0;
  const int A = d0 < d1 ? d0 : d1, B = d0 < d1 ? d1 : d0;
  const double s0 = (A > J || B < I) ? -1.0 : 1.0;
  const int oi = I >> 1, si = I & 1, oa = A >> 1, sa = A & 1, oj = J >> 1, sj = J & 1, ob = B >> 1;
  if (si == sa) {
    e[0] = (si + 2 * sj) * L4 + oa + (size_t)L * ob + L2 * (oi + (size_t)L * oj);
    e[1] = (sj + 2 * si) * L4 + ob + (size_t)L * oa + L2 * (oj + (size_t)L * oi);
    sg[0] = sg[1] = s0;
  } else {
    e[0] = (si + 2 * sj) * L4 + oa + (size_t)L * ob + L2 * (oj + (size_t)L * oi);
    e[1] = (sj + 2 * si) * L4 + ob + (size_t)L * oa + L2 * (oi + (size_t)L * oj);
    sg[0] = sg[1] = -s0;
  }
}

// Writes the alpha-beta 2-RDM elements, one thread per pattern pair. Two
// pattern pairs reach the same element exactly when they differ by exchanging
// the particles (equal holes) or the holes (equal particles) of the two
// spins; the element is then written once, by the pair that comes first in
// (h1, p1, h2, p2) order, as its own term followed by its partner's, so every
// element has one writer and one summation order. amap, bmap: pattern index
// of (hole << 6 | particle), -1 when no single has that pattern.
__global__ void rdm_ab_write_kernel(const uint32_t* __restrict__ akey, int npa, const uint32_t* __restrict__ bkey,
                                    int npb, const int* __restrict__ amap, const int* __restrict__ bmap,
                                    const double* __restrict__ G, int L, double* __restrict__ two) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)npa * npb) return;
  const int pa = (int)(t / npb), p = (int)(t % npb);
  const int h1 = (int)(akey[pa] >> 6), p1 = (int)(akey[pa] & 63u);
  const int h2 = (int)(bkey[p] >> 6), p2 = (int)(bkey[p] & 63u);
  const double v = G[t];
  size_t e[2], ep[2] = {~(size_t)0, ~(size_t)0};
  double sg[2], sgp[2] = {0.0, 0.0};
  ab_targets(h1, p1, h2, p2, L, e, sg);
  int q1 = -1, q2 = -1, x1 = 0, y1 = 0, x2 = 0, y2 = 0;  // partner (alpha x1 -> y1, beta x2 -> y2)
  if (h1 == h2 && p1 != p2) { x1 = h1; y1 = p2; x2 = h2; y2 = p1; }
  else if (p1 == p2 && h1 != h2) { x1 = h2; y1 = p1; x2 = h1; y2 = p2; }
  else x1 = -1;
  double vp = 0.0;
  bool partner_first = false;
  if (x1 >= 0) {
    q1 = amap[(x1 << 6) | y1];
    q2 = bmap[(x2 << 6) | y2];
    if (q1 >= 0 && q2 >= 0) {
      vp = G[(size_t)q1 * npb + q2];
      ab_targets(x1, y1, x2, y2, L, ep, sgp);
      partner_first = x1 < h1 || (x1 == h1 && (y1 < p1 || (y1 == p1 && (x2 < h2 || (x2 == h2 && y2 < p2)))));
    }
  }
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    double val = sg[i] * v;
    bool skip = false;
#pragma unroll
    for (int j = 0; j < 2; ++j)
      if (ep[j] == e[i]) {
        if (partner_first) skip = true;
        else val += sgp[j] * vp;
      }
    if (!skip && val != 0.0) two[e[i]] += val;
  }
}

template <typename T>
__global__ void transpose_d_kernel(const T* __restrict__ in, size_t rows, size_t cols, T* __restrict__ out) {
  __shared__ T tile[32][33];
  const size_t c0 = (size_t)blockIdx.x * 32, r0 = (size_t)blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const size_t r = r0 + k, c = c0 + threadIdx.x;
    if (r < rows && c < cols) tile[k][threadIdx.x] = in[r * cols + c];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const size_t c = c0 + k, r = r0 + threadIdx.x;
    if (r < rows && c < cols) out[c * rows + r] = tile[threadIdx.x][k];
  }
}

// dE/dh and dE/d(pq|rs) from the RDMs: E = I0 + sum_pq h_pq g_pq
//   + 1/2 sum_{io,jo,ia,ja} (io ia|jo ja) sum_s G_s[io + L jo + L^2 ia + L^3 ja]
// (sample main.cc:166-216). One thread per 8-fold class sums its distinct
// index permutations.
__global__ void backward_eri_kernel(int L, const double* __restrict__ two, double* __restrict__ g) {
  const size_t npair = (size_t)L * (L + 1) / 2;
  const size_t neri = npair * (npair + 1) / 2;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= neri) return;
  // decode t -> (pq, rs) with pq >= rs, then pq -> (p >= q), rs -> (r >= s)
  size_t pq = (size_t)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while (pq * (pq + 1) / 2 > t) --pq;
  while ((pq + 1) * (pq + 2) / 2 <= t) ++pq;
  const size_t rs = t - pq * (pq + 1) / 2;
  auto split = [](size_t x, int& a, int& b) {
    size_t p = (size_t)((sqrt(8.0 * (double)x + 1.0) - 1.0) * 0.5);
    while (p * (p + 1) / 2 > x) --p;
    while ((p + 1) * (p + 2) / 2 <= x) ++p;
    a = (int)p;
    b = (int)(x - p * (p + 1) / 2);
  };
  int p, q, r, s;
  split(pq, p, q);
  split(rs, r, s);
  const size_t L2 = (size_t)L * L, L3 = L2 * L, L4 = L3 * L;
  // the 8 index orders (io, ia | jo, ja); keep distinct ones
  int cand[8][4] = {{p, q, r, s}, {q, p, r, s}, {p, q, s, r}, {q, p, s, r},
                    {r, s, p, q}, {s, r, p, q}, {r, s, q, p}, {s, r, q, p}};
  double sum = 0.0;
  for (int k = 0; k < 8; ++k) {
    bool dup = false;
    for (int m = 0; m < k; ++m)
      if (cand[m][0] == cand[k][0] && cand[m][1] == cand[k][1] && cand[m][2] == cand[k][2] && cand[m][3] == cand[k][3])
        dup = true;
    if (dup) continue;
    const int io = cand[k][0], ia = cand[k][1], jo = cand[k][2], ja = cand[k][3];
    const size_t idx = (size_t)io + L * (size_t)jo + L2 * ia + L3 * ja;
    sum += 0.5 * (two[idx] + two[L4 + idx] + two[2 * L4 + idx] + two[3 * L4 + idx]);
  }
  g[t] = sum;
}

struct Scratch {
  double* p = nullptr;
  ~Scratch() { cudaFree(p); }
};

}  // namespace

// Row weights of both orientations: wa[na], wb[nb]; P_a, P_b, X (L*L each).
// (P and X are written, not accumulated; the sums have a fixed order.)
static int weights(Ctx* c, const double* dW, double* wa, double* wb, double* Pa, double* Pb, double* X, double* Wt) {
  const size_t na = c->na, nb = c->nb;
  const int L = c->L;
  Scratch vq;
  if (X) SBDX_CUDA(c, cudaMalloc(&vq.p, sizeof(double) * na * (size_t)L));
  const size_t smem = X ? sizeof(double) * kRowWeightThreads * (size_t)L : 0;
  row_weight_kernel<<<(unsigned)na, kRowWeightThreads, smem, c->stream>>>(dW, nb, c->d_b, L, wa, vq.p);
  SBDX_LAUNCHED(c);
  occupation_sums_kernel<<<(unsigned)((L * L + 127) / 128), 128, 0, c->stream>>>(na, c->d_a, L, wa, vq.p, Pa, X);
  SBDX_LAUNCHED(c);
  if (wb) {
    dim3 grid((unsigned)((nb + 31) / 32), (unsigned)((na + 31) / 32));
    transpose_d_kernel<double><<<grid, dim3(32, 8), 0, c->stream>>>(dW, na, nb, Wt);
    SBDX_LAUNCHED(c);
    row_weight_kernel<<<(unsigned)nb, kRowWeightThreads, 0, c->stream>>>(Wt, na, c->d_a, L, wb, nullptr);
    SBDX_LAUNCHED(c);
    occupation_sums_kernel<<<(unsigned)((L * L + 127) / 128), 128, 0, c->stream>>>(nb, c->d_b, L, wb, nullptr, Pb,
                                                                                  nullptr);
    SBDX_LAUNCHED(c);
  }
  SBDX_CUDA(c, cudaStreamSynchronize(c->stream));  // the profile scratch dies at return
  return 0;
}

// The single excitations of one spin grouped by pattern key = hole << 6 |
// particle (hole: the ket's orbital, particle: the bra's), each group in
// ascending bra then ket order: keys, group offsets and records bra | ket << 32.
static int singles_by_pattern(Ctx* c, int spin, std::vector<uint32_t>& keys, std::vector<uint32_t>& goff,
                              std::vector<uint64_t>& recs) {
  const Conn& cn = c->conn[spin];
  const size_t n = cn.n;
  std::vector<uint64_t> off(n + 1);
  std::vector<uint32_t> ns(n), ket(cn.total ? cn.total : 1), info(cn.total ? cn.total : 1);
  SBDX_CUDA(c, cudaMemcpyAsync(off.data(), cn.off, sizeof(uint64_t) * (n + 1), cudaMemcpyDeviceToHost, c->stream));
  SBDX_CUDA(c, cudaMemcpyAsync(ns.data(), cn.nsing, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, c->stream));
  if (cn.total) {
    SBDX_CUDA(c, cudaMemcpyAsync(ket.data(), cn.ket, sizeof(uint32_t) * cn.total, cudaMemcpyDeviceToHost, c->stream));
    SBDX_CUDA(c, cudaMemcpyAsync(info.data(), cn.info, sizeof(uint32_t) * cn.total, cudaMemcpyDeviceToHost, c->stream));
  }
  SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
  std::vector<uint32_t> count(64 * 64, 0);
  for (size_t r = 0; r < n; ++r)
    for (uint32_t e = 0; e < ns[r]; ++e) ++count[info[off[r] + e] & 0xfffu];
  std::vector<uint32_t> start(64 * 64 + 1, 0), where(64 * 64, 0);
  keys.clear();
  goff.assign(1, 0);
  for (uint32_t k = 0; k < 64 * 64; ++k) {
    start[k + 1] = start[k] + count[k];
    if (count[k]) {
      where[k] = (uint32_t)keys.size();
      // info bits 0-5 hole, 6-11 particle -> key hole << 6 | particle
      keys.push_back(((k & 63u) << 6) | (k >> 6));
      goff.push_back(start[k + 1]);
    }
  }
  recs.assign(start[64 * 64] ? start[64 * 64] : 1, 0);
  std::vector<uint32_t> fill(start.begin(), start.end() - 1);
  for (size_t r = 0; r < n; ++r)
    for (uint32_t e = 0; e < ns[r]; ++e) {
      const uint32_t k = info[off[r] + e] & 0xfffu;
      recs[fill[k]++] = (uint64_t)r | ((uint64_t)ket[off[r] + e] << 32);
    }
  (void)where;
  return 0;
}

// The entries of one spin grouped by pattern, each group in CSR (bra, then
// ket) order: singles by info bits 0-11 (hole, particle), doubles by info
// bits 0-23 (both holes, both particles); per sorted position the entry and
// its bra row.
struct EntryGroups {
  std::vector<uint32_t> key, off, ent, row;
};
static int group_entries(Ctx* c, int spin, EntryGroups& sg, EntryGroups& dg) {
  const Conn& cn = c->conn[spin];
  const size_t n = cn.n;
  std::vector<uint64_t> off(n + 1);
  std::vector<uint32_t> ns(n), info(cn.total ? cn.total : 1);
  SBDX_CUDA(c, cudaMemcpyAsync(off.data(), cn.off, sizeof(uint64_t) * (n + 1), cudaMemcpyDeviceToHost, c->stream));
  SBDX_CUDA(c, cudaMemcpyAsync(ns.data(), cn.nsing, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, c->stream));
  if (cn.total)
    SBDX_CUDA(c, cudaMemcpyAsync(info.data(), cn.info, sizeof(uint32_t) * cn.total, cudaMemcpyDeviceToHost, c->stream));
  SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
  // stable counting sort by 12-bit digits, least significant first (one pass
  // for singles, two for doubles)
  auto sort_by = [&](std::vector<uint32_t> a, int digits, std::vector<uint32_t>& out) {
    std::vector<uint32_t> b(a.size());
    for (int d = 0; d < digits; ++d) {
      std::vector<uint32_t> cnt(4097, 0);
      for (uint32_t e : a) ++cnt[((info[e] >> (12 * d)) & 0xfffu) + 1];
      for (int k = 0; k < 4096; ++k) cnt[k + 1] += cnt[k];
      for (uint32_t e : a) b[cnt[(info[e] >> (12 * d)) & 0xfffu]++] = e;
      a.swap(b);
    }
    out.swap(a);
  };
  std::vector<uint32_t> es, ed, rowof(cn.total ? cn.total : 1);
  for (size_t r = 0; r < n; ++r)
    for (uint64_t e = off[r]; e < off[r + 1]; ++e) {
      rowof[e] = (uint32_t)r;
      (e - off[r] < ns[r] ? es : ed).push_back((uint32_t)e);
    }
  auto finish = [&](const std::vector<uint32_t>& sorted, uint32_t mask, EntryGroups& g) {
    g.ent = sorted;
    g.row.resize(sorted.size());
    g.key.clear();
    g.off.assign(1, 0);
    for (size_t t = 0; t < sorted.size(); ++t) {
      g.row[t] = rowof[sorted[t]];
      const uint32_t k = info[sorted[t]] & mask;
      if (g.key.empty() || k != g.key.back()) {
        if (!g.key.empty()) g.off.push_back((uint32_t)t);
        g.key.push_back(k);
      }
    }
    if (!g.key.empty()) g.off.push_back((uint32_t)sorted.size());
  };
  std::vector<uint32_t> ss, sd;
  sort_by(es, 1, ss);
  sort_by(ed, 2, sd);
  finish(ss, 0xfffu, sg);
  finish(sd, 0xffffffu, dg);
  return 0;
}

// Same-spin 1-/2-RDM contributions of one spin without atomics (two may be
// null: the 1-RDM alone, singles only). Wm: W (spin 0) or W^T (spin 1).
static int rdm_same_deterministic(Ctx* c, int spin, const double* Wm, double* one, double* two) {
  const Conn& cn = c->conn[spin];
  if (cn.total == 0) return 0;
  EntryGroups sg, dg;
  int rc = group_entries(c, spin, sg, dg);
  if (rc) return rc;
  const size_t cols = spin == 0 ? c->nb : c->na;
  const uint64_t* s_row = spin == 0 ? c->d_a : c->d_b;
  const uint64_t* s_col = spin == 0 ? c->d_b : c->d_a;
  const int L = c->L;
  struct Bufs {
    std::vector<void*> p;
    ~Bufs() { for (void* q : p) cudaFree(q); }
  } bufs;
  auto dev = [&](const std::vector<uint32_t>& h, uint32_t** d) -> cudaError_t {
    cudaError_t e = cudaMalloc(d, sizeof(uint32_t) * std::max<size_t>(1, h.size()));
    if (e == cudaSuccess) bufs.p.push_back(*d);
    if (e == cudaSuccess && !h.empty())
      e = cudaMemcpyAsync(*d, h.data(), sizeof(uint32_t) * h.size(), cudaMemcpyHostToDevice, c->stream);
    return e;
  };
  auto run = [&](const EntryGroups& g, bool singles) -> int {
    const size_t n = g.ent.size();
    if (n == 0 || (!singles && two == nullptr)) return 0;
    uint32_t *d_ent = nullptr, *d_row = nullptr, *d_key = nullptr, *d_off = nullptr;
    double *d_val = nullptr, *d_prof = nullptr;
    SBDX_CUDA(c, dev(g.ent, &d_ent));
    SBDX_CUDA(c, dev(g.row, &d_row));
    SBDX_CUDA(c, dev(g.key, &d_key));
    SBDX_CUDA(c, dev(g.off, &d_off));
    SBDX_CUDA(c, cudaMalloc(&d_val, sizeof(double) * n));
    bufs.p.push_back(d_val);
    const int profile = singles && two != nullptr;
    if (profile) {
      SBDX_CUDA(c, cudaMalloc(&d_prof, sizeof(double) * n * (size_t)L));
      bufs.p.push_back(d_prof);
    }
    const size_t smem = profile ? sizeof(double) * kValWarps * 32 * (size_t)L : 0;
    SBDX_CUDA(c, cudaFuncSetAttribute(rdm_same_values_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(sizeof(double) * kValWarps * 32 * 64)));
    rdm_same_values_kernel<<<(unsigned)((n + kValWarps - 1) / kValWarps), kValWarps * 32, smem, c->stream>>>(
        Wm, cols, s_row, s_col, cn.ket, cn.omask, cn.info, d_ent, d_row, n, L, profile, d_val, d_prof);
    SBDX_LAUNCHED(c);
    const size_t ng = g.key.size();
    if (singles) {
      const size_t nt = ng * (two ? 1 + 2 * (size_t)L : 1);
      rdm_singles_finalize_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, c->stream>>>(
          spin, L, d_key, d_off, ng, d_row, s_row, d_val, d_prof, one, two);
    } else {
      rdm_doubles_finalize_kernel<<<(unsigned)((ng + 255) / 256), 256, 0, c->stream>>>(spin, L, d_key, d_off, ng,
                                                                                       d_val, two);
    }
    SBDX_LAUNCHED(c);
    SBDX_CUDA(c, cudaStreamSynchronize(c->stream));  // the host vectors and buffers die at return
    return 0;
  };
  if ((rc = run(sg, true))) return rc;
  return run(dg, false);
}

// The alpha-single x beta-single 2-RDM contributions without atomics
// (rdm_ab_det_kernel, rdm_ab_sum_kernel, rdm_ab_write_kernel); returns 1 when the two staged
// rows do not fit in shared memory (the caller then uses rdm_ab_kernel).
static int rdm_ab_deterministic(Ctx* c, const double* dW, double* two, bool& done) {
  done = false;
  const size_t nb = c->nb;
  std::vector<uint32_t> akeys, agoff, bkeys, bgoff;
  std::vector<uint64_t> arecs, brecs;
  int rc;
  if ((rc = singles_by_pattern(c, 0, akeys, agoff, arecs))) return rc;
  if ((rc = singles_by_pattern(c, 1, bkeys, bgoff, brecs))) return rc;
  const int npb = (int)bkeys.size(), npa = (int)akeys.size();
  const size_t smem = sizeof(double) * (2 * nb + (size_t)npb);
  if (smem > kAbSmemBudget) return 0;
  done = true;
  if (npa == 0 || npb == 0) return 0;
  // chunks of at most kAbChunk alpha singles of one pattern; per pattern its chunk range
  std::vector<uint4> chunks, apat;
  for (int q = 0; q < npa; ++q) {
    const uint32_t first = (uint32_t)chunks.size();
    for (uint32_t b = agoff[q]; b < agoff[q + 1]; b += kAbChunk)
      chunks.push_back(make_uint4(akeys[q], b, std::min<uint32_t>(kAbChunk, agoff[q + 1] - b), 0u));
    apat.push_back(make_uint4(akeys[q], first, (uint32_t)chunks.size() - first, 0u));
  }
  struct Bufs {
    std::vector<void*> p;
    ~Bufs() { for (void* q : p) cudaFree(q); }
  } bufs;
  auto up = [&](const void* h, size_t bytes, void** d) -> cudaError_t {
    cudaError_t e = cudaMalloc(d, bytes ? bytes : 16);
    if (e == cudaSuccess) bufs.p.push_back(*d);
    if (e == cudaSuccess && h && bytes) e = cudaMemcpyAsync(*d, h, bytes, cudaMemcpyHostToDevice, c->stream);
    return e;
  };
  uint4 *d_chunks = nullptr, *d_apat = nullptr;
  uint64_t *d_arec = nullptr, *d_brec = nullptr;
  uint32_t *d_boff = nullptr, *d_bkey = nullptr;
  double* d_part = nullptr;
  SBDX_CUDA(c, up(chunks.data(), sizeof(uint4) * chunks.size(), (void**)&d_chunks));
  SBDX_CUDA(c, up(apat.data(), sizeof(uint4) * apat.size(), (void**)&d_apat));
  SBDX_CUDA(c, up(arecs.data(), sizeof(uint64_t) * arecs.size(), (void**)&d_arec));
  SBDX_CUDA(c, up(bgoff.data(), sizeof(uint32_t) * bgoff.size(), (void**)&d_boff));
  SBDX_CUDA(c, up(bkeys.data(), sizeof(uint32_t) * bkeys.size(), (void**)&d_bkey));
  SBDX_CUDA(c, up(brecs.data(), sizeof(uint64_t) * brecs.size(), (void**)&d_brec));
  SBDX_CUDA(c, up(nullptr, sizeof(double) * chunks.size() * (size_t)npb, (void**)&d_part));
  SBDX_CUDA(c, cudaFuncSetAttribute(rdm_ab_det_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kAbSmemBudget));
  rdm_ab_det_kernel<<<(unsigned)chunks.size(), kAbDetThreads, smem, c->stream>>>(
      dW, nb, c->d_a, c->d_b, d_chunks, d_arec, d_boff, d_bkey, d_brec, npb, d_part);
  SBDX_LAUNCHED(c);
  const size_t npairs = (size_t)npa * npb;
  std::vector<int> amap(64 * 64, -1), bmap(64 * 64, -1);
  for (int q = 0; q < npa; ++q) amap[akeys[q]] = q;
  for (int q = 0; q < npb; ++q) bmap[bkeys[q]] = q;
  std::vector<uint32_t> akey_v(akeys.begin(), akeys.end());
  int *d_amap = nullptr, *d_bmap = nullptr;
  uint32_t* d_akey = nullptr;
  double* d_G = nullptr;
  SBDX_CUDA(c, up(amap.data(), sizeof(int) * amap.size(), (void**)&d_amap));
  SBDX_CUDA(c, up(bmap.data(), sizeof(int) * bmap.size(), (void**)&d_bmap));
  SBDX_CUDA(c, up(akey_v.data(), sizeof(uint32_t) * akey_v.size(), (void**)&d_akey));
  SBDX_CUDA(c, up(nullptr, sizeof(double) * npairs, (void**)&d_G));
  rdm_ab_sum_kernel<<<(unsigned)((npairs + 255) / 256), 256, 0, c->stream>>>(d_apat, npa, npb, d_part, d_G);
  SBDX_LAUNCHED(c);
  rdm_ab_write_kernel<<<(unsigned)((npairs + 255) / 256), 256, 0, c->stream>>>(d_akey, npa, d_bkey, npb, d_amap,
                                                                               d_bmap, d_G, c->L, two);
  SBDX_LAUNCHED(c);
  SBDX_CUDA(c, cudaStreamSynchronize(c->stream));  // the host vectors and buffers die at return
  return 0;
}

int rdm_device(Ctx* c, const double* dW, double* d_one, double* d_two) {
  if (!c->have_lists) { int rc = build_connectivity(c, false); if (rc) return rc; }
  int rc = ensure_sigma_scratch(c);
  if (rc) return rc;
  const size_t na = c->na, nb = c->nb, L = (size_t)c->L, L2 = L * L, L4 = L2 * L2;
  Scratch sc;
  SBDX_CUDA(c, cudaMalloc(&sc.p, sizeof(double) * (na + nb + 3 * L2)));
  double* wa = sc.p;
  double* wb = wa + na;
  double* Pa = wb + nb;
  double* Pb = Pa + L2;
  double* X = Pb + L2;
  double* two = d_two;  // null: the 1-RDM alone
  SBDX_CUDA(c, cudaMemsetAsync(Pa, 0, sizeof(double) * 3 * L2, c->stream));
  SBDX_CUDA(c, cudaMemsetAsync(d_one, 0, sizeof(double) * 2 * L2, c->stream));
  if (two) SBDX_CUDA(c, cudaMemsetAsync(two, 0, sizeof(double) * 4 * L4, c->stream));
  double* Wt = reinterpret_cast<double*>(c->d_xt);
  if ((rc = weights(c, dW, wa, wb, Pa, Pb, X, Wt))) return rc;
  diag_finalize_kernel<<<(unsigned)((L2 + 255) / 256), 256, 0, c->stream>>>(c->L, Pa, Pb, X, d_one, two);
  SBDX_LAUNCHED(c);
  for (int spin = 0; spin < 2; ++spin)
    if ((rc = rdm_same_deterministic(c, spin, spin == 0 ? dW : Wt, d_one, two))) return rc;
  bool done = d_two == nullptr;  // the alpha-beta pairs only add to the 2-RDM
  if (!done && (rc = rdm_ab_deterministic(c, dW, two, done))) return rc;
  if (!done) {
    const int staged = sizeof(double) * (L2 + nb) <= kAbSmemBudget;
    const size_t smem = sizeof(double) * (L2 + (staged ? nb : 0));
    if (smem > kAbSmemBudget) { c->err = "rdm: too many orbitals for the shared-memory accumulator"; return 1; }
    SBDX_CUDA(c, cudaFuncSetAttribute(rdm_ab_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kAbSmemBudget));
    const Conn& ca = c->conn[0];
    const Conn& cb = c->conn[1];
    rdm_ab_kernel<<<(unsigned)na, 512, smem, c->stream>>>(dW, nb, c->d_a, c->d_b, ca.off, ca.nsing, ca.ket, ca.info,
                                                           cb.off, cb.nsing, cb.ket, cb.info, c->L, two, staged);
    SBDX_LAUNCHED(c);
  }
  SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
  return 0;
}

int occupation_device(Ctx* c, const double* dW, double* d_density) {
  int rc = ensure_sigma_scratch(c);
  if (rc) return rc;
  const size_t na = c->na, nb = c->nb, L = (size_t)c->L, L2 = L * L;
  Scratch sc;
  SBDX_CUDA(c, cudaMalloc(&sc.p, sizeof(double) * (na + nb + 3 * L2)));
  double *wa = sc.p, *wb = wa + na, *Pa = wb + nb, *Pb = Pa + L2;  // (the third L2 block is unused here)
  SBDX_CUDA(c, cudaMemsetAsync(Pa, 0, sizeof(double) * 3 * L2, c->stream));
  if ((rc = weights(c, dW, wa, wb, Pa, Pb, nullptr, reinterpret_cast<double*>(c->d_xt)))) return rc;
  // density[2p] = Pa[p][p], density[2p+1] = Pb[p][p]
  std::vector<double> pa(L2), pb(L2), dens(2 * L);
  SBDX_CUDA(c, cudaMemcpyAsync(pa.data(), Pa, sizeof(double) * L2, cudaMemcpyDeviceToHost, c->stream));
  SBDX_CUDA(c, cudaMemcpyAsync(pb.data(), Pb, sizeof(double) * L2, cudaMemcpyDeviceToHost, c->stream));
  SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
  for (size_t p = 0; p < L; ++p) { dens[2 * p] = pa[p * L + p]; dens[2 * p + 1] = pb[p * L + p]; }
  SBDX_CUDA(c, cudaMemcpyAsync(d_density, dens.data(), sizeof(double) * 2 * L, cudaMemcpyHostToDevice, c->stream));
  SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
  return 0;
}

int alpha_weights_device(Ctx* c, const double* dW, double* d_w) {
  const size_t L2 = (size_t)c->L * c->L;
  Scratch sc;
  SBDX_CUDA(c, cudaMalloc(&sc.p, sizeof(double) * L2));
  SBDX_CUDA(c, cudaMemsetAsync(sc.p, 0, sizeof(double) * L2, c->stream));
  return weights(c, dW, d_w, nullptr, sc.p, nullptr, nullptr, nullptr);
}

int backward_device(Ctx* c, const double* dW, double* dE_dh, double* dE_deri) {
  // the excitation lists are rebuilt from the strings; nothing of the forward
  // solve is kept (the sigma's layouts are not needed and not built: a later
  // sigma rebuilds the full connectivity)
  int rc = build_connectivity(c, false);
  if (rc) return rc;
  const size_t L = (size_t)c->L, L2 = L * L, L4 = L2 * L2;
  Scratch sc;
  SBDX_CUDA(c, cudaMalloc(&sc.p, sizeof(double) * (2 * L2 + 4 * L4 + c->neri)));
  double *one = sc.p, *two = one + 2 * L2, *g = two + 4 * L4;
  if ((rc = rdm_device(c, dW, one, two))) return rc;
  backward_eri_kernel<<<(unsigned)((c->neri + 255) / 256), 256, 0, c->stream>>>(c->L, two, g);
  SBDX_LAUNCHED(c);
  std::vector<double> h1(2 * L2);
  SBDX_CUDA(c, cudaMemcpyAsync(h1.data(), one, sizeof(double) * 2 * L2, cudaMemcpyDeviceToHost, c->stream));
  SBDX_CUDA(c, cudaMemcpyAsync(dE_deri, g, sizeof(double) * c->neri, cudaMemcpyDeviceToHost, c->stream));
  SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
  // one FCIDUMP entry (p, q) sets h[p][q] and h[q][p] (makeintegrals.h:108-112)
  for (size_t p = 0; p < L; ++p)
    for (size_t q = 0; q < L; ++q) {
      const double gpq = h1[p + L * q] + h1[L2 + p + L * q];
      const double gqp = h1[q + L * p] + h1[L2 + q + L * p];
      dE_dh[p * L + q] = p == q ? gpq : gpq + gqp;
    }
  return 0;
}

}  // namespace sbdx
