// Excitation-connectivity builder.
//
// Restates GenerateExcitation (reference chemistry/tpb/helper.h:132-197): for
// every bra string r of one spin, the ket strings k with popcount(s_r ^ s_k)
// == 2 (single) or == 4 (double), in ascending k, singles then doubles per
// row (the flattened layout of MakeSmartHelper, helper.h:367-437).
//
// B200 form: one CTA per bra row; pass 1 counts with an XOR-popcount scan, the
// host scans the counts into row offsets, pass 2 re-scans and compacts with a
// warp-ballot prefix so the output order is the ascending scan order. Pass 2
// also evaluates, once per entry, everything of the matrix element that does
// not depend on the opposite-spin string:
//   - the same-spin part of the fermionic sign and the opposite-spin parity
//     mask (the two halves of the reference parity(), determinants.h:228-279,
//     on the interleaved layout alpha p -> 2p, beta p -> 2p+1);
//   - the same-spin part of the value: OneExcite (determinants.h:423-445)
//     without the opposite-spin Coulomb sum, or TwoExcite (:447-465).
// The sigma kernels combine these with the opposite-spin string of each
// determinant in O(1) (a popcount) per pair.
#include "sbdx_internal.cuh"
#include "sbdx.h"

#include <algorithm>
#include <array>
#include <cstdint>
#include <random>
#include <thread>
#include <vector>

namespace sbdx {

namespace {

constexpr int kConnThreads = 256;
// Move budget of the record-order descent, per step of a quarter-warp.
constexpr int kOrderEffort = 3000;

__global__ void __launch_bounds__(kConnThreads)
conn_count_kernel(const uint64_t* __restrict__ s, size_t n, uint32_t* __restrict__ nsing,
                  uint32_t* __restrict__ ndoub) {
  const size_t r = blockIdx.x;
  const uint64_t sr = s[r];
  uint32_t cs = 0, cd = 0;
  for (size_t k = threadIdx.x; k < n; k += blockDim.x) {
    int d = popc64(sr ^ s[k]);
    cs += (d == 2);
    cd += (d == 4);
  }
  for (int o = 16; o > 0; o >>= 1) {
    cs += __shfl_down_sync(0xffffffffu, cs, o);
    cd += __shfl_down_sync(0xffffffffu, cd, o);
  }
  __shared__ uint32_t ws[kConnThreads / 32], wd[kConnThreads / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { ws[warp] = cs; wd[warp] = cd; }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t ts = 0, td = 0;
    for (int w = 0; w < kConnThreads / 32; ++w) { ts += ws[w]; td += wd[w]; }
    nsing[r] = ts;
    ndoub[r] = td;
  }
}

// Same-spin part of <bra|H|ket> for bra string sr, ket string sk of spin `spin`.
__device__ void make_entry(int spin, uint64_t sr, uint64_t sk, int L, const double* __restrict__ h,
                           const double* __restrict__ eri, double& val, uint64_t& om, uint32_t& info) {
  const uint64_t hole = sk & ~sr;  // occupied in ket only
  const uint64_t part = sr & ~sk;  // occupied in bra only
  if (popc64(hole) == 1) {
    const int i = __ffsll((long long)hole) - 1, a = __ffsll((long long)part) - 1;
    const int lo = i < a ? i : a, hi = i < a ? a : i;
    // parity(ket, 2lo+s, 2hi+s): same-spin bits strictly between (the start
    // bit and the [start,end) count cancel on the occupied end), plus the
    // opposite-spin bits of the range.
    const uint32_t neg = (uint32_t)(popc64(sk & range_mask(lo + 1, hi)) & 1);
    om = other_range(spin, lo, hi);
    double v = h[(size_t)a * L + i];
    uint64_t bits = sk;
    while (bits) {
      const int q = __ffsll((long long)bits) - 1;
      v += eri[eri_index(a, i, q, q)] - eri[eri_index(a, q, q, i)];
      bits &= bits - 1;
    }
    val = v;
    info = (neg << 31) | kInfoSingle | (uint32_t)i | ((uint32_t)a << 6) |
           ((uint32_t)pair_index(a, i) << 12);
  } else {
    const int i = __ffsll((long long)hole) - 1;
    const int j = __ffsll((long long)(hole & (hole - 1))) - 1;
    const int a = __ffsll((long long)part) - 1;
    const int b = __ffsll((long long)(part & (part - 1))) - 1;
    int par = 0;
    uint64_t m = 0;
    {
      const int lo = i < a ? i : a, hi = i < a ? a : i;
      par += popc64(sk & range_mask(lo, hi)) + (int)((sk >> lo) & 1ull);
      m ^= other_range(spin, lo, hi);
    }
    {
      const int lo = j < b ? j : b, hi = j < b ? b : j;
      par += popc64(sk & range_mask(lo, hi)) + (int)((sk >> lo) & 1ull);
      m ^= other_range(spin, lo, hi);
    }
    if (a > j || b < i) par += 1;
    om = m;
    val = eri[eri_index(a, i, b, j)] - eri[eri_index(a, j, b, i)];
    info = ((uint32_t)(par & 1) << 31) | (uint32_t)i | ((uint32_t)j << 6) | ((uint32_t)a << 12) |
           ((uint32_t)b << 18);
  }
}

__global__ void __launch_bounds__(kConnThreads)
conn_fill_kernel(int spin, const uint64_t* __restrict__ s, size_t n, const uint64_t* __restrict__ off,
                 const uint32_t* __restrict__ nsing, int L, const double* __restrict__ h,
                 const double* __restrict__ eri, uint32_t* __restrict__ ket, double* __restrict__ val,
                 float* __restrict__ val32, uint64_t* __restrict__ omask, uint32_t* __restrict__ info,
                 uint64_t* __restrict__ srec, uint32_t* __restrict__ spos) {
  const size_t r = blockIdx.x;
  const uint64_t sr = s[r];
  const uint64_t sbase0 = off[r];
  const uint64_t dbase0 = off[r] + nsing[r];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  __shared__ uint32_t ws[kConnThreads / 32], wd[kConnThreads / 32];
  __shared__ uint32_t s_run, d_run;
  if (threadIdx.x == 0) { s_run = 0; d_run = 0; }
  __syncthreads();
  for (size_t k0 = 0; k0 < n; k0 += kConnThreads) {
    const size_t k = k0 + threadIdx.x;
    uint64_t sk = 0;
    int d = 0;
    if (k < n) { sk = s[k]; d = popc64(sr ^ sk); }
    const bool is_s = (k < n) && d == 2, is_d = (k < n) && d == 4;
    const unsigned bs = __ballot_sync(0xffffffffu, is_s), bd = __ballot_sync(0xffffffffu, is_d);
    if (lane == 0) { ws[warp] = __popc(bs); wd[warp] = __popc(bd); }
    __syncthreads();
    uint32_t sp = 0, dp = 0, st = 0, dt = 0;
    for (int w = 0; w < kConnThreads / 32; ++w) {
      if (w < warp) { sp += ws[w]; dp += wd[w]; }
      st += ws[w];
      dt += wd[w];
    }
    if (is_s || is_d) {
      const uint64_t pos = is_s ? sbase0 + s_run + sp + __popc(bs & lt)
                                : dbase0 + d_run + dp + __popc(bd & lt);
      double v;
      uint64_t m;
      uint32_t inf;
      make_entry(spin, sr, sk, L, h, eri, v, m, inf);
      ket[pos] = (uint32_t)k;
      val[pos] = v;
      val32[pos] = (float)v;
      omask[pos] = m;
      info[pos] = inf;
      {
        // boundaries of the opposite-spin ranges: [lo,hi) for alpha
        // excitations, (lo,hi] = [lo+1,hi+1) for beta excitations
        uint32_t p[4] = {0, 0, 0, 0};
        const uint32_t sh = (uint32_t)spin;
        if (is_s) {
          const uint32_t i = inf & 63u, a = (inf >> 6) & 63u;
          p[0] = (i < a ? i : a) + sh;
          p[1] = (i < a ? a : i) + sh;
        } else {
          const uint32_t i = inf & 63u, j = (inf >> 6) & 63u, a = (inf >> 12) & 63u, b = (inf >> 18) & 63u;
          p[0] = (i < a ? i : a) + sh;
          p[1] = (i < a ? a : i) + sh;
          p[2] = (j < b ? j : b) + sh;
          p[3] = (j < b ? b : j) + sh;
        }
        spos[pos] = p[0] | (p[1] << 7) | (p[2] << 14) | (p[3] << 21) | (inf & (kInfoNeg | kInfoSingle));
      }
      if (is_s) {
        const uint32_t i = inf & 63u, a = (inf >> 6) & 63u;
        const uint64_t lo = i < a ? i : a, hi = i < a ? a : i;
        srec[pos] = rec_ket_bits(k) | ((uint64_t)((inf >> 12) & 0xfffu) << 16) | (lo << 28) | (hi << 34) |
                    ((uint64_t)(inf >> 31) << 40);
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) { s_run += st; d_run += dt; }
    __syncthreads();
  }
}

void free_conn(Conn& c) {
  cudaFree(c.nsing); cudaFree(c.ndoub); cudaFree(c.off); cudaFree(c.ket);
  cudaFree(c.val); cudaFree(c.val32); cudaFree(c.omask); cudaFree(c.info);
  cudaFree(c.srec); cudaFree(c.order); cudaFree(c.spos);
  cudaFree(c.sell); cudaFree(c.soff); cudaFree(c.slen); cudaFree(c.kpos);
  auto free_panel = [](SellPanel& p) {
    cudaFree(p.sell); cudaFree(p.sell32); cudaFree(p.soff4); cudaFree(p.slen4);
    cudaFree(p.soff); cudaFree(p.slen); cudaFree(p.vrow); cudaFree(p.vslot);
    cudaFree(p.split_row); cudaFree(p.split_slot);
  };
  free_panel(c.bal);
  for (auto& p : c.panels) free_panel(p);
  cudaFree(c.ab_item); cudaFree(c.ab_split); cudaFree(c.ypart);
  cudaFree(c.same_item); cudaFree(c.same_split); cudaFree(c.same_ypart);
  free_blocks(c.blk);
  c = Conn{};
}

// Splits rows of `len` work units longer than cap into items (see
// Conn::ab_item): {row, first unit, one past the last, 1 + slot or 0},
// longest first; split rows as {row, first slot, parts, 0}. Empty rows get an
// item only with keep_empty (a kernel that assigns its output row).
// Rows are numbered from row0 (len[i] belongs to row row0 + i).
void split_rows(const std::vector<uint32_t>& len, uint32_t cap, bool keep_empty, std::vector<uint4>& items,
                std::vector<uint4>& split, int& nslot, size_t row0 = 0) {
  items.clear();
  split.clear();
  nslot = 0;
  for (size_t i = 0; i < len.size(); ++i) {
    const uint32_t r = (uint32_t)(row0 + i);
    if (len[i] <= cap) {
      if (len[i] || keep_empty) items.push_back(make_uint4(r, 0u, len[i], 0u));
      continue;
    }
    const uint32_t parts = (len[i] + cap - 1) / cap;
    split.push_back(make_uint4(r, (uint32_t)nslot, parts, 0u));
    for (uint32_t q = 0; q < parts; ++q)
      items.push_back(make_uint4(r, q * cap, std::min(len[i], (q + 1) * cap), (uint32_t)(nslot + q + 1)));
    nslot += (int)parts;
  }
  std::stable_sort(items.begin(), items.end(), [](const uint4& x, const uint4& y) { return x.z - x.y > y.z - y.y; });
}

int upload_items(Ctx* c, const std::vector<uint4>& items, const std::vector<uint4>& split, int nslot, size_t ncol,
                 uint4** d_items, uint4** d_split, double** d_part) {
  SBDX_CUDA(c, cudaMalloc(d_items, sizeof(uint4) * std::max<size_t>(1, items.size())));
  SBDX_CUDA(c, cudaMalloc(d_split, sizeof(uint4) * std::max<size_t>(1, split.size())));
  if (!items.empty())
    SBDX_CUDA(c, cudaMemcpyAsync(*d_items, items.data(), sizeof(uint4) * items.size(), cudaMemcpyHostToDevice,
                                 c->stream));
  if (!split.empty()) {
    SBDX_CUDA(c, cudaMemcpyAsync(*d_split, split.data(), sizeof(uint4) * split.size(), cudaMemcpyHostToDevice,
                                 c->stream));
    SBDX_CUDA(c, cudaMalloc(d_part, sizeof(double) * (size_t)nslot * std::max<size_t>(8, pad8(ncol))));
  }
  SBDX_CUDA(c, cudaStreamSynchronize(c->stream));  // host vectors die at return
  return 0;
}

int sm_count(Ctx* c) {
  int nsm = 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess || nsm < 1) nsm = 148;
  return nsm;
}

// Same-spin work items (see Conn::same_item). A CTA handles one item and one
// strip of 1024 columns (4 per thread); an item longer than the mean work of
// a CTA slot (8 resident CTAs per SM) would set the kernel's duration, so
// rows with more entries are split (at least 64 entries per item).
// Rows row0 .. row0 + hs.size() - 1 (all rows, or one shard of them).
int build_same_items(Ctx* c, Conn& cn, const std::vector<uint32_t>& hs, const std::vector<uint32_t>& hd, size_t ncol,
                     size_t row0 = 0) {
  std::vector<uint32_t> len(hs.size());
  uint64_t total = 0;
  for (size_t r = 0; r < hs.size(); ++r) total += (len[r] = hs[r] + hd[r]);
  const uint64_t strips = std::max<uint64_t>(1, (ncol + 1023) / 1024);
  const uint64_t slots = 8ull * sm_count(c);
  const uint32_t cap = (uint32_t)std::max<uint64_t>(64, (total * strips + slots - 1) / slots);
  std::vector<uint4> items, split;
  int nslot = 0;
  split_rows(len, cap, true, items, split, nslot, row0);  // every row's output is assigned
  cn.same_cap = (int)cap;
  cn.n_same_item = items.size();
  cn.n_same_split = (int)split.size();
  cn.n_same_part = nslot;
  return upload_items(c, items, split, nslot, ncol, &cn.same_item, &cn.same_split, &cn.same_ypart);
}

uint64_t bit_reverse64(uint64_t x) {
  x = ((x >> 1) & 0x5555555555555555ull) | ((x & 0x5555555555555555ull) << 1);
  x = ((x >> 2) & 0x3333333333333333ull) | ((x & 0x3333333333333333ull) << 2);
  x = ((x >> 4) & 0x0f0f0f0f0f0f0f0full) | ((x & 0x0f0f0f0f0f0f0f0full) << 4);
  x = ((x >> 8) & 0x00ff00ff00ff00ffull) | ((x & 0x00ff00ff00ff00ffull) << 8);
  x = ((x >> 16) & 0x0000ffff0000ffffull) | ((x & 0x0000ffff0000ffffull) << 16);
  return (x >> 32) | (x << 32);
}

// Blocks of the blocked same-spin kernel (see SameBlocks) over the bra
// strings row0 .. row0 + n - 1 of connectivity cn; hs are their singles
// counts, `strings` all strings of the spin, ncol the other spin's string
// count (partial rows have stride pad8(ncol)). The unions are built on the
// host from a copy of the rows' entries (a merge with one cursor per string
// of a block), blocks split over host threads.
int build_same_blocks(Ctx* c, const Conn& cn, const std::vector<uint64_t>& strings, size_t row0, size_t n,
                      const std::vector<uint32_t>& hs, size_t ncol, SameBlocks& B) {
  free_blocks(B);
  if (n == 0) return 0;
  // the rows' entries (one contiguous range of the CSR)
  std::vector<uint64_t> off(n + 1);
  SBDX_CUDA(c, cudaMemcpyAsync(off.data(), cn.off + row0, sizeof(uint64_t) * (n + 1), cudaMemcpyDeviceToHost,
                               c->stream));
  SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
  const uint64_t e0 = off[0], ne = off[n] - off[0];
  std::vector<uint32_t> ket(ne ? ne : 1), info(ne ? ne : 1);
  std::vector<double> val(ne ? ne : 1);
  std::vector<float> val32(ne ? ne : 1);
  if (ne) {
    SBDX_CUDA(c, cudaMemcpyAsync(ket.data(), cn.ket + e0, sizeof(uint32_t) * ne, cudaMemcpyDeviceToHost, c->stream));
    SBDX_CUDA(c, cudaMemcpyAsync(info.data(), cn.info + e0, sizeof(uint32_t) * ne, cudaMemcpyDeviceToHost, c->stream));
    SBDX_CUDA(c, cudaMemcpyAsync(val.data(), cn.val + e0, sizeof(double) * ne, cudaMemcpyDeviceToHost, c->stream));
    SBDX_CUDA(c, cudaMemcpyAsync(val32.data(), cn.val32 + e0, sizeof(float) * ne, cudaMemcpyDeviceToHost, c->stream));
    SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  // rows in bit-reversed string order, cut into blocks
  std::vector<std::pair<uint64_t, uint32_t>> rkey(n);
  for (size_t i = 0; i < n; ++i) rkey[i] = {bit_reverse64(strings[row0 + i]), (uint32_t)i};
  std::sort(rkey.begin(), rkey.end());
  std::vector<uint32_t> order(n);
  for (size_t i = 0; i < n; ++i) order[i] = rkey[i].second;
  const size_t nblk = (n + kBlkRows - 1) / kBlkRows;
  std::vector<uint4> rows(nblk);
  for (size_t b = 0; b < nblk; ++b) {
    uint32_t r[kBlkRows];
    for (int k = 0; k < kBlkRows; ++k) {
      const size_t i = b * kBlkRows + k;
      r[k] = i < n ? (uint32_t)(row0 + order[i]) : kNoRow;
    }
    rows[b] = make_uint4(r[0], r[1], r[2], r[3]);
  }
  // every row's doubles must be ascending by ket (the builder's scan order);
  // a row that is not gets a sorted index of its doubles
  std::vector<std::vector<uint32_t>> perm(n);
  for (size_t r = 0; r < n; ++r) {
    const uint32_t* k0 = ket.data() + (off[r] - e0 + hs[r]);
    const uint32_t* k1 = ket.data() + (off[r + 1] - e0);
    if (!std::is_sorted(k0, k1)) {
      perm[r].resize(k1 - k0);
      for (uint32_t q = 0; q < perm[r].size(); ++q) perm[r][q] = q;
      std::sort(perm[r].begin(), perm[r].end(), [&](uint32_t x, uint32_t y) { return k0[x] < k0[y]; });
    }
  }
  // per block: a merge of its rows' doubles by ket with one cursor per row;
  // equal kets become one union entry with a value per row
  struct Part {
    std::vector<uint32_t> ket;
    std::vector<double> val;
    std::vector<float> val32;
    std::vector<uint64_t> len;  // union entries per block of the part
  };
  const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  const size_t nth = std::max<size_t>(1, std::min<size_t>(hw, (nblk + 63) / 64));
  std::vector<Part> parts(nth);
  auto work = [&](size_t t) {
    Part& P = parts[t];
    const size_t b0 = nblk * t / nth, b1 = nblk * (t + 1) / nth;
    size_t est = 0;
    for (size_t i = b0 * kBlkRows; i < std::min(n, b1 * kBlkRows); ++i) {
      const size_t r = order[i];
      est += off[r + 1] - off[r] - hs[r];
    }
    P.ket.reserve(est);
    P.val.reserve(est * kBlkRows);
    P.val32.reserve(est * kBlkRows);
    P.len.reserve(b1 - b0);
    for (size_t b = b0; b < b1; ++b) {
      uint64_t base[kBlkRows] = {}, cur[kBlkRows] = {}, len[kBlkRows] = {};
      const uint32_t* pm[kBlkRows] = {};
      for (int k = 0; k < kBlkRows; ++k) {
        const size_t i = b * kBlkRows + k;
        if (i >= n) continue;
        const size_t r = order[i];
        base[k] = off[r] - e0 + hs[r];
        len[k] = off[r + 1] - off[r] - hs[r];
        pm[k] = perm[r].empty() ? nullptr : perm[r].data();
      }
      auto at = [&](int k) -> uint64_t { return base[k] + (pm[k] ? pm[k][cur[k]] : cur[k]); };
      uint64_t cnt = 0;
      while (true) {
        uint32_t m = 0xffffffffu;
        for (int k = 0; k < kBlkRows; ++k)
          if (cur[k] < len[k]) m = std::min(m, ket[at(k)]);
        if (m == 0xffffffffu) break;
        P.ket.push_back(m);
        for (int k = 0; k < kBlkRows; ++k) {
          double v = 0.0;
          float v32 = 0.f;
          if (cur[k] < len[k] && ket[at(k)] == m) {
            const uint64_t e = at(k);
            ++cur[k];
            const bool neg = (info[e] & kInfoNeg) != 0;
            v = neg ? -val[e] : val[e];
            v32 = neg ? -val32[e] : val32[e];
          }
          P.val.push_back(v);
          P.val32.push_back(v32);
        }
        ++cnt;
      }
      P.len.push_back(cnt);
    }
  };
  {
    std::vector<std::thread> th;
    for (size_t t = 1; t < nth; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& x : th) x.join();
  }
  std::vector<uint64_t> uoff(nblk + 1, 0);
  {
    size_t b = 0;
    for (const Part& P : parts)
      for (uint64_t l : P.len) { uoff[b + 1] = uoff[b] + l; ++b; }
  }
  const uint64_t nu = uoff[nblk];
  // work items: union entries plus, for a block's first item, two loads per
  // single; blocks above the cap are split (see build_same_items)
  std::vector<uint64_t> sing(nblk, 0);
  uint64_t total = 0;
  for (size_t b = 0; b < nblk; ++b) {
    for (int k = 0; k < kBlkRows; ++k) {
      const size_t i = b * kBlkRows + k;
      if (i < n) sing[b] += hs[order[i]];
    }
    total += (uoff[b + 1] - uoff[b]) + 2 * sing[b];
  }
  const uint64_t strips = std::max<uint64_t>(1, (ncol + 1023) / 1024);
  const uint64_t slots = 8ull * sm_count(c);
  const uint32_t cap = (uint32_t)std::max<uint64_t>(64, (total * strips + slots - 1) / slots);
  std::vector<uint4> items, split;
  std::vector<uint64_t> weight;
  int nslot = 0;
  for (size_t b = 0; b < nblk; ++b) {
    const uint64_t len = uoff[b + 1] - uoff[b];
    if (len <= cap) {
      items.push_back(make_uint4((uint32_t)b, 0u, (uint32_t)len, 0u));
      weight.push_back(len + 2 * sing[b]);
      continue;
    }
    const uint32_t np = (uint32_t)((len + cap - 1) / cap);
    split.push_back(make_uint4((uint32_t)b, (uint32_t)nslot, np, 0u));
    for (uint32_t q = 0; q < np; ++q) {
      const uint32_t u0 = q * cap, u1 = (uint32_t)std::min<uint64_t>(len, (uint64_t)(q + 1) * cap);
      items.push_back(make_uint4((uint32_t)b, u0, u1, (uint32_t)(nslot + q + 1)));
      weight.push_back((u1 - u0) + (q == 0 ? 2 * sing[b] : 0));
    }
    nslot += (int)np;
  }
  {
    std::vector<size_t> perm(items.size());
    for (size_t i = 0; i < perm.size(); ++i) perm[i] = i;
    std::stable_sort(perm.begin(), perm.end(), [&](size_t x, size_t y) { return weight[x] > weight[y]; });
    std::vector<uint4> sorted(items.size());
    for (size_t i = 0; i < perm.size(); ++i) sorted[i] = items[perm[i]];
    items.swap(sorted);
  }
  // upload
  const size_t nu1 = nu ? nu : 1;
  B.nblk = nblk;
  B.nu = nu;
  B.cap = (int)cap;
  B.n_item = items.size();
  B.n_split = (int)split.size();
  B.n_part = nslot;
  SBDX_CUDA(c, cudaMalloc(&B.rows, sizeof(uint4) * nblk));
  SBDX_CUDA(c, cudaMalloc(&B.uoff, sizeof(uint64_t) * (nblk + 1)));
  SBDX_CUDA(c, cudaMalloc(&B.uket, sizeof(uint32_t) * nu1));
  SBDX_CUDA(c, cudaMalloc(&B.uval, sizeof(double) * kBlkRows * nu1));
  SBDX_CUDA(c, cudaMalloc(&B.uval32, sizeof(float) * kBlkRows * nu1));
  SBDX_CUDA(c, cudaMemcpyAsync(B.rows, rows.data(), sizeof(uint4) * nblk, cudaMemcpyHostToDevice, c->stream));
  SBDX_CUDA(c, cudaMemcpyAsync(B.uoff, uoff.data(), sizeof(uint64_t) * (nblk + 1), cudaMemcpyHostToDevice, c->stream));
  {
    uint64_t at = 0;
    for (const Part& P : parts) {
      const size_t m = P.ket.size();
      if (m) {
        SBDX_CUDA(c, cudaMemcpyAsync(B.uket + at, P.ket.data(), sizeof(uint32_t) * m, cudaMemcpyHostToDevice,
                                     c->stream));
        SBDX_CUDA(c, cudaMemcpyAsync(B.uval + at * kBlkRows, P.val.data(), sizeof(double) * kBlkRows * m,
                                     cudaMemcpyHostToDevice, c->stream));
        SBDX_CUDA(c, cudaMemcpyAsync(B.uval32 + at * kBlkRows, P.val32.data(), sizeof(float) * kBlkRows * m,
                                     cudaMemcpyHostToDevice, c->stream));
      }
      at += m;
    }
  }
  // upload_items synchronises the stream before the host vectors die
  return upload_items(c, items, split, nslot * kBlkRows, ncol, &B.item, &B.split, &B.ypart);
}

// Work items of the packed alpha-beta kernel (see Conn::ab_item; partial rows
// have the padded stride pad8(nb) of the sigma's alpha-major vectors). A CTA
// handles one item and the kernel lasts about as long as the busiest SM, so
// a few strings with many singles (near-Aufbau strings of a small sample
// connect to ten times the mean) would set its duration: strings are split
// into items of at most cap singles, cap = a quarter of the mean work per SM
// (rounded up to a multiple of 4, at least 8), and items run longest first.
// Large samples have many strings per SM and split nothing.
int build_ab_items(Ctx* c, Conn& cn, const std::vector<uint32_t>& hs, size_t nb, size_t row0 = 0) {
  const uint64_t nsm = (uint64_t)sm_count(c);
  uint64_t total = 0;
  for (uint32_t h : hs) total += h;
  const uint64_t quarter = (total + 4 * nsm - 1) / (4 * nsm);
  const uint32_t cap = (uint32_t)std::max<uint64_t>(8, (quarter + 3) & ~3ull);
  std::vector<uint4> items, split;
  int slot = 0;
  split_rows(hs, cap, false, items, split, slot, row0);  // the kernel adds to its output
  cn.item_cap = (int)cap;
  cn.n_item = items.size();
  cn.n_split = (int)split.size();
  cn.n_part = slot;
  return upload_items(c, items, split, slot, nb, &cn.ab_item, &cn.ab_split, &cn.ypart);
}

// Position of each ket string in the packed alpha-beta kernel's staged rows
// (Conn::kpos). A string keeps its aligned group of 8 positions (8*(k/8) ..
// 8*(k/8)+7, a 128-byte row of 16-byte packs) and gets the slot in it that
// spreads the singles of every bra string most evenly over the 8 bank slots:
// a descent on the sum over bra strings of the squared per-slot counts,
// exchanging the slots of two strings of one group. With the singles of each
// bra string spread evenly, every quarter-warp's ket slots are balanced and
// its records can be ordered with few bank conflicts. A quarter-warp's
// staging stores still hit 8 different slots (the group is permuted within
// itself), so staging stays conflict-free.
std::vector<uint32_t> ket_positions(size_t n, const std::vector<uint32_t>& hs, const std::vector<uint64_t>& off,
                                    const std::vector<uint64_t>& rec) {
  std::vector<uint32_t> pos(n);
  for (size_t k = 0; k < n; ++k) pos[k] = (uint32_t)k;
  if (n < 16) return pos;
  // bra strings whose singles include ket k (CSR)
  std::vector<uint64_t> roff(n + 1, 0);
  for (size_t r = 0; r < n; ++r)
    for (uint32_t e = 0; e < hs[r]; ++e) ++roff[rec_ket(rec[off[r] + e]) + 1];
  for (size_t k = 0; k < n; ++k) roff[k + 1] += roff[k];
  std::vector<uint32_t> rows(roff[n]);
  {
    std::vector<uint64_t> fill(roff.begin(), roff.end() - 1);
    for (size_t r = 0; r < n; ++r)
      for (uint32_t e = 0; e < hs[r]; ++e) rows[fill[rec_ket(rec[off[r] + e])]++] = (uint32_t)r;
  }
  std::vector<std::array<int16_t, 8>> h(n);
  for (size_t r = 0; r < n; ++r) {
    h[r].fill(0);
    for (uint32_t e = 0; e < hs[r]; ++e) ++h[r][pos[rec_ket(rec[off[r] + e])] & 7u];
  }
  for (int sweep = 0; sweep < 8; ++sweep) {
    long long gain = 0;
    for (size_t g0 = 0; g0 < n; g0 += 8) {
      const size_t g1 = std::min(n, g0 + 8);
      for (size_t a = g0; a < g1; ++a)
        for (size_t b = a + 1; b < g1; ++b) {
          const uint32_t sa = pos[a] & 7u, sb = pos[b] & 7u;
          long long d = 0;
          // ket a moves from slot sa to sb, ket b from sb to sa
          for (uint64_t t = roff[a]; t < roff[a + 1]; ++t) {
            auto& x = h[rows[t]];
            d += 2 * (x[sb] - x[sa]) + 2;
            --x[sa];
            ++x[sb];
          }
          for (uint64_t t = roff[b]; t < roff[b + 1]; ++t) {
            auto& x = h[rows[t]];
            d += 2 * (x[sa] - x[sb]) + 2;
            --x[sb];
            ++x[sa];
          }
          if (d < 0) {
            std::swap(pos[a], pos[b]);
            gain += d;
          } else {
            for (uint64_t t = roff[b]; t < roff[b + 1]; ++t) { ++h[rows[t]][sb]; --h[rows[t]][sa]; }
            for (uint64_t t = roff[a]; t < roff[a + 1]; ++t) { ++h[rows[t]][sa]; --h[rows[t]][sb]; }
          }
        }
    }
    if (gain == 0) break;
  }
  return pos;
}

// Balanced SELL-32 of the single records (see Conn::bsell). The cap starts at
// twice the mean list length (at least 16), so that no lane of a warp walks a
// list much longer than the others, and doubles until the partial-sum slots
// fit the kernel's shared-memory budget. The slices per warp are the smallest
// of 8, 12, 16 that cover the virtual rows in the fewest CTAs.
int build_balanced_sell(Ctx* c, SellPanel& P, size_t n, const std::vector<uint32_t>& hs_all,
                        const std::vector<uint64_t>& off_all, const std::vector<uint64_t>& rec,
                        const std::vector<uint32_t>& kpos, uint32_t jb0, uint32_t jb1) {
  // the singles of row r are rec[off_all[r] .. off_all[r] + hs_all[r]), ascending
  // ket index: the ones in [jb0, jb1) are a contiguous sub-range
  std::vector<uint32_t> hs(n);
  std::vector<uint64_t> off(n);
  for (size_t r = 0; r < n; ++r) {
    const uint64_t* b = rec.data() + off_all[r];
    const uint64_t* e = b + hs_all[r];
    const uint64_t* lo = std::lower_bound(b, e, jb0, [](uint64_t x, uint32_t v) { return rec_ket(x) < v; });
    const uint64_t* hi = std::lower_bound(lo, e, jb1, [](uint64_t x, uint32_t v) { return rec_ket(x) < v; });
    off[r] = (uint64_t)(lo - rec.data());
    hs[r] = (uint32_t)(hi - lo);
  }
  std::vector<uint32_t> order(n);
  for (size_t r = 0; r < n; ++r) order[r] = (uint32_t)r;
  std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return hs[x] > hs[y]; });
  P.jb0 = jb0;
  P.jb1 = jb1;
  uint64_t total = 0;
  uint32_t mx = 0;
  for (size_t r = 0; r < n; ++r) { total += hs[r]; mx = std::max(mx, hs[r]); }
  uint32_t cap = std::max<uint32_t>(16, 2 * (uint32_t)((total + n - 1) / n));
  std::vector<uint32_t> parts(n);
  int nslot = 0;
  for (;;) {
    nslot = 0;
    for (size_t r = 0; r < n; ++r) {
      parts[r] = hs[r] == 0 ? 0 : (hs[r] + cap - 1) / cap;
      if (parts[r] > 1) nslot += (int)parts[r];
    }
    if (nslot <= kMaxSplitSlots || cap >= mx) break;
    cap *= 2;
  }
  if (nslot > kMaxSplitSlots) {
    c->err = "build_connectivity: too many split beta lists";
    return SBDX_ERR_ARG;
  }
  // virtual rows: (bra string, first record, length, slot + 1 or 0)
  struct VRow { uint32_t r; uint64_t beg; uint32_t len; uint32_t slot1; };
  std::vector<VRow> vr;
  std::vector<uint32_t> split_row, split_slot(1, 0);
  for (uint32_t r : order) {
    if (parts[r] <= 1) continue;
    const uint32_t p = parts[r], base = hs[r] / p, rem = hs[r] % p;
    uint64_t beg = off[r];
    for (uint32_t j = 0; j < p; ++j) {
      const uint32_t len = base + (j < rem ? 1u : 0u);
      vr.push_back({r, beg, len, split_slot.back() + j + 1});
      beg += len;
    }
    split_row.push_back(r);
    split_slot.push_back(split_slot.back() + p);
  }
  for (uint32_t r : order)  // longest first
    if (parts[r] == 1) vr.push_back({r, off[r], hs[r], 0});
  const size_t nv = vr.size();
  int ks = 8;
  {
    size_t best = SIZE_MAX;
    for (int cand : {8, 12, 16}) {
      const size_t chunks = (nv + 1024 * (size_t)cand - 1) / (1024 * (size_t)cand);
      if (chunks < best) { best = chunks; ks = cand; }
    }
  }
  const size_t ns = (nv + 31) / 32;
  std::vector<uint64_t> soff(ns + 1, 0);
  std::vector<uint32_t> slen(ns ? ns : 1, 0);
  for (size_t sl = 0; sl < ns; ++sl) {
    uint32_t m = 0;
    for (size_t l = 0; l < 32 && sl * 32 + l < nv; ++l) m = std::max(m, vr[sl * 32 + l].len);
    slen[sl] = m;
    soff[sl + 1] = soff[sl] + 32ull * m;
  }
  // padding records contribute nothing (bit 41) and point at the panel's first
  // ket index, so the kernels' shared-memory index stays in range
  const uint64_t kPad = (1ull << 41) | rec_ket_bits(jb0);
  std::vector<uint64_t> sell(soff[ns] ? soff[ns] : 1, kPad);
  std::vector<uint32_t> vrow(nv ? nv : 1, 0), vslot(nv ? nv : 1, 0);
  for (size_t v = 0; v < nv; ++v) {
    vrow[v] = vr[v].r;
    vslot[v] = vr[v].slot1;
  }
  // 32-bit records of the packed kernel in blocks of 4 per lane (see
  // SellPanel::sell32); the steps that round a slice up to a multiple of 4
  // are padding at the panel's first staged position
  std::vector<uint64_t> soff4(ns + 1, 0);
  std::vector<uint32_t> slen4(ns ? ns : 1, 0);
  for (size_t sl = 0; sl < ns; ++sl) {
    slen4[sl] = (slen[sl] + 3u) & ~3u;
    soff4[sl + 1] = soff4[sl] + 32ull * slen4[sl];
  }
  const uint32_t kPad32 = 1u << 29;  // position 0 of the panel
  std::vector<uint32_t> sell32(soff4[ns] ? soff4[ns] : 4, kPad32);
  // Record order inside each virtual row is free (it only changes the order
  // of the sum) and decides the bank conflicts of the packed kernel's two
  // 16-byte shared-memory gathers per record. The 8 lanes of a quarter-warp
  // are served together: one 128-byte wavefront when their 16-byte slots
  // differ, one more per further distinct address in a slot. A record's ket
  // slot is kpos[ket] mod 8 (the staged ket rows are permuted within aligned
  // groups of 8, see ket_positions); its integral slot is pq mod 8 or
  // (pq + 4) mod 8 (two staged copies), so the distinct pairs of one class
  // pq mod 4 cost ceil(count / 2) wavefronts. Per quarter: a greedy start
  // (per step, each lane takes the record whose ket slot and pair class are
  // least used in the step, most constrained lane first), then a descent on
  // the quarter's estimate (per step, the largest ket-slot count plus half the
  // largest pair-class count, rounded up) by exchanging the steps of two
  // records of one lane, until the estimate reaches the quarter's lower bound
  // or the move budget runs out. The integral copies then alternate over the
  // distinct pairs of a class in each step, and pad records repeat the
  // addresses of a real record of their step (a broadcast costs nothing).
  // Slices are ordered on several host threads, each slice with its own
  // seeded generator, so the result does not depend on the thread count.
  auto kslot = [&](uint64_t r) { return (uint32_t)(kpos[rec_ket(r)] & 7u); };
  auto pcls = [](uint64_t r) { return (uint32_t)((r >> 16) & 3u); };
  auto order_slice = [&](size_t sl) {
    const size_t l_end = std::min<size_t>(32, nv - sl * 32);
    const uint32_t m_len = slen[sl];
    constexpr uint64_t kEmpty = ~0ull;
    std::vector<uint64_t> grid;
    std::vector<std::vector<uint64_t>> left(8);
    std::vector<std::array<int8_t, 8>> ck;
    std::vector<std::array<int8_t, 4>> cp;
    std::vector<int> sc;
    for (size_t q = 0; q * 8 < l_end; ++q) {
      const int nl = (int)std::min<size_t>(8, l_end - q * 8);
      grid.assign((size_t)m_len * 8, kEmpty);
      uint32_t lmax = 0;
      int deg[8] = {0}, pdeg[4] = {0};
      for (int i = 0; i < nl; ++i) {
        const VRow& w = vr[sl * 32 + q * 8 + i];
        left[i].assign(rec.begin() + w.beg, rec.begin() + w.beg + w.len);
        lmax = std::max(lmax, w.len);
        for (uint64_t r : left[i]) { ++deg[kslot(r)]; ++pdeg[pcls(r)]; }
      }
      // greedy start
      for (uint32_t m = 0; m < m_len; ++m) {
        int lanes[8], n_act = 0;
        for (int i = 0; i < nl; ++i)
          if (!left[i].empty()) lanes[n_act++] = i;
        std::sort(lanes, lanes + n_act, [&](int x, int y) { return left[x].size() < left[y].size(); });
        int cj[8] = {0}, cq[4] = {0};
        for (int a = 0; a < n_act; ++a) {
          std::vector<uint64_t>& lst = left[lanes[a]];
          size_t best = 0;
          int bc = 1 << 30;
          for (size_t t = 0; t < lst.size(); ++t) {
            const int cc = cj[kslot(lst[t])] + cq[pcls(lst[t])];
            if (cc < bc) { bc = cc; best = t; }
          }
          grid[(size_t)m * 8 + lanes[a]] = lst[best];
          ++cj[kslot(lst[best])];
          ++cq[pcls(lst[best])];
          lst.erase(lst.begin() + (std::ptrdiff_t)best);
        }
      }
      // descent
      ck.assign(m_len, std::array<int8_t, 8>{});
      cp.assign(m_len, std::array<int8_t, 4>{});
      for (uint32_t m = 0; m < m_len; ++m)
        for (int i = 0; i < nl; ++i) {
          const uint64_t r = grid[(size_t)m * 8 + i];
          if (r != kEmpty) { ++ck[m][kslot(r)]; ++cp[m][pcls(r)]; }
        }
      auto cost = [&](uint32_t m) {
        int a = 0, b = 0;
        for (int x = 0; x < 8; ++x) a = std::max(a, (int)ck[m][x]);
        for (int x = 0; x < 4; ++x) b = std::max(b, (int)cp[m][x]);
        return a + (b + 1) / 2;
      };
      sc.assign(m_len, 0);
      long long cur = 0;
      for (uint32_t m = 0; m < m_len; ++m) cur += (sc[m] = cost(m));
      const long long lb = (long long)std::max<int>((int)lmax, *std::max_element(deg, deg + 8)) +
                           std::max<int>((int)lmax, (*std::max_element(pdeg, pdeg + 4) + 1) / 2);
      std::mt19937 rng((uint32_t)(sl * 4 + q) * 2654435761u + 12345u);
      const long long budget = (long long)kOrderEffort * m_len;
      for (long long it = 0; it < budget && cur > lb && m_len > 1; ++it) {
        const int i = (int)(rng() % (uint32_t)nl);
        const uint32_t m1 = rng() % m_len, m2 = rng() % m_len;
        if (m1 == m2) continue;
        uint64_t& A = grid[(size_t)m1 * 8 + i];
        uint64_t& B = grid[(size_t)m2 * 8 + i];
        if (A == kEmpty && B == kEmpty) continue;
        auto move = [&](uint64_t r, uint32_t from, uint32_t to) {
          if (r == kEmpty) return;
          --ck[from][kslot(r)]; --cp[from][pcls(r)];
          ++ck[to][kslot(r)]; ++cp[to][pcls(r)];
        };
        move(A, m1, m2);
        move(B, m2, m1);
        const int c1 = cost(m1), c2 = cost(m2);
        const int d = c1 + c2 - sc[m1] - sc[m2];
        if (d <= 0) {
          std::swap(A, B);
          cur += d;
          sc[m1] = c1;
          sc[m2] = c2;
        } else {
          move(A, m2, m1);
          move(B, m1, m2);
        }
      }
      // emit: 64-bit records (original ket index) and 32-bit packed records
      for (uint32_t m = 0; m < m_len; ++m) {
        uint32_t seen[8], seen_copy[8], nseen = 0, cls_count[4] = {0, 0, 0, 0};
        uint32_t src32 = kPad32;
        bool have_src = false;
        for (int i = 0; i < nl; ++i) {
          const uint64_t r = grid[(size_t)m * 8 + i];
          if (r == kEmpty) continue;
          const size_t lane = q * 8 + (size_t)i;
          sell[soff[sl] + 32ull * m + lane] = r;
          const uint32_t pq = (uint32_t)((r >> 16) & 0xfffu);
          uint32_t copy = 0;
          bool dup = false;
          for (uint32_t t = 0; t < nseen; ++t)
            if (seen[t] == pq) { copy = seen_copy[t]; dup = true; }
          if (!dup) {
            // the distinct pairs of class pq mod 4 go alternately to bank
            // slots (pq mod 4) and (pq mod 4) + 4: copy 0 reads slot pq mod 8,
            // copy 1 the slot four further on
            const uint32_t target = (pq & 3u) + 4u * (cls_count[pq & 3u]++ & 1u);
            copy = (pq & 7u) == target ? 0u : 1u;
            seen[nseen] = pq;
            seen_copy[nseen++] = copy;
          }
          const uint32_t w32 = ((kpos[rec_ket(r)] - jb0) & 0xffffu) | (pq << 16) | ((uint32_t)((r >> 40) & 1u) << 28) |
                               (copy << 30);
          sell32[soff4[sl] + 128ull * (m >> 2) + 4 * lane + (m & 3u)] = w32;
          if (!have_src) { src32 = w32 | (1u << 29); have_src = true; }
        }
        for (int i = 0; i < nl; ++i)
          if (grid[(size_t)m * 8 + i] == kEmpty)
            sell32[soff4[sl] + 128ull * (m >> 2) + 4 * (q * 8 + (size_t)i) + (m & 3u)] = src32;
      }
    }
  };
  {
    const unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    const unsigned nt = (unsigned)std::min<size_t>(hw, std::max<size_t>(1, ns));
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nt; ++t)
      pool.emplace_back([&, t]() {
        for (size_t sl = t; sl < ns; sl += nt) order_slice(sl);
      });
    for (auto& th : pool) th.join();
  }
  P.nslice = ns;
  P.nv = nv;
  P.nsplit = (int)split_row.size();
  P.nslot = (int)split_slot.back();
  P.cap = (int)cap;
  P.slices_per_warp = ks;
  if (split_row.empty()) split_row.push_back(0);
  SBDX_CUDA(c, cudaMalloc(&P.sell32, sizeof(uint32_t) * sell32.size()));
  SBDX_CUDA(c, cudaMalloc(&P.soff4, sizeof(uint64_t) * (ns + 1)));
  SBDX_CUDA(c, cudaMalloc(&P.slen4, sizeof(uint32_t) * slen4.size()));
  SBDX_CUDA(c, cudaMemcpyAsync(P.sell32, sell32.data(), sizeof(uint32_t) * sell32.size(), cudaMemcpyHostToDevice,
                               c->stream));
  SBDX_CUDA(c, cudaMemcpyAsync(P.soff4, soff4.data(), sizeof(uint64_t) * (ns + 1), cudaMemcpyHostToDevice,
                               c->stream));
  SBDX_CUDA(c, cudaMemcpyAsync(P.slen4, slen4.data(), sizeof(uint32_t) * slen4.size(), cudaMemcpyHostToDevice,
                               c->stream));
  SBDX_CUDA(c, cudaMalloc(&P.sell, sizeof(uint64_t) * sell.size()));
  SBDX_CUDA(c, cudaMalloc(&P.soff, sizeof(uint64_t) * (ns + 1)));
  SBDX_CUDA(c, cudaMalloc(&P.slen, sizeof(uint32_t) * slen.size()));
  SBDX_CUDA(c, cudaMalloc(&P.vrow, sizeof(uint32_t) * vrow.size()));
  SBDX_CUDA(c, cudaMalloc(&P.vslot, sizeof(uint32_t) * vslot.size()));
  SBDX_CUDA(c, cudaMalloc(&P.split_row, sizeof(uint32_t) * split_row.size()));
  SBDX_CUDA(c, cudaMalloc(&P.split_slot, sizeof(uint32_t) * split_slot.size()));
  SBDX_CUDA(c, cudaMemcpyAsync(P.sell, sell.data(), sizeof(uint64_t) * sell.size(), cudaMemcpyHostToDevice, c->stream));
  SBDX_CUDA(c, cudaMemcpyAsync(P.soff, soff.data(), sizeof(uint64_t) * (ns + 1), cudaMemcpyHostToDevice, c->stream));
  SBDX_CUDA(c, cudaMemcpyAsync(P.slen, slen.data(), sizeof(uint32_t) * slen.size(), cudaMemcpyHostToDevice, c->stream));
  SBDX_CUDA(c, cudaMemcpyAsync(P.vrow, vrow.data(), sizeof(uint32_t) * vrow.size(), cudaMemcpyHostToDevice, c->stream));
  SBDX_CUDA(c, cudaMemcpyAsync(P.vslot, vslot.data(), sizeof(uint32_t) * vslot.size(), cudaMemcpyHostToDevice,
                               c->stream));
  SBDX_CUDA(c, cudaMemcpyAsync(P.split_row, split_row.data(), sizeof(uint32_t) * split_row.size(),
                               cudaMemcpyHostToDevice, c->stream));
  SBDX_CUDA(c, cudaMemcpyAsync(P.split_slot, split_slot.data(), sizeof(uint32_t) * split_slot.size(),
                               cudaMemcpyHostToDevice, c->stream));
  SBDX_CUDA(c, cudaStreamSynchronize(c->stream));  // host vectors die at return
  return 0;
}

// full = false: the lists only (CSR, per-entry values, masks and records),
// without the sigma's work items, SELL layouts, ket positions and blocks.
int build_one(Ctx* c, int spin, bool full) {
  Conn& cn = c->conn[spin];
  free_conn(cn);
  const size_t n = spin == 0 ? c->na : c->nb;
  const uint64_t* s = spin == 0 ? c->d_a : c->d_b;
  cn.n = n;
  SBDX_CUDA(c, cudaMalloc(&cn.nsing, sizeof(uint32_t) * n));
  SBDX_CUDA(c, cudaMalloc(&cn.ndoub, sizeof(uint32_t) * n));
  SBDX_CUDA(c, cudaMalloc(&cn.off, sizeof(uint64_t) * (n + 1)));
  conn_count_kernel<<<(unsigned)n, kConnThreads, 0, c->stream>>>(s, n, cn.nsing, cn.ndoub);
  SBDX_LAUNCHED(c);
  std::vector<uint32_t> hs(n), hd(n);
  SBDX_CUDA(c, cudaMemcpyAsync(hs.data(), cn.nsing, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, c->stream));
  SBDX_CUDA(c, cudaMemcpyAsync(hd.data(), cn.ndoub, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, c->stream));
  SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
  std::vector<uint64_t> off(n + 1, 0);
  for (size_t r = 0; r < n; ++r) off[r + 1] = off[r] + hs[r] + hd[r];
  cn.total = off[n];
  SBDX_CUDA(c, cudaMemcpyAsync(cn.off, off.data(), sizeof(uint64_t) * (n + 1), cudaMemcpyHostToDevice, c->stream));
  const size_t t = cn.total ? cn.total : 1;
  SBDX_CUDA(c, cudaMalloc(&cn.ket, sizeof(uint32_t) * t));
  SBDX_CUDA(c, cudaMalloc(&cn.val, sizeof(double) * t));
  SBDX_CUDA(c, cudaMalloc(&cn.val32, sizeof(float) * t));
  SBDX_CUDA(c, cudaMalloc(&cn.omask, sizeof(uint64_t) * t));
  SBDX_CUDA(c, cudaMalloc(&cn.info, sizeof(uint32_t) * t));
  SBDX_CUDA(c, cudaMalloc(&cn.srec, sizeof(uint64_t) * t));
  SBDX_CUDA(c, cudaMalloc(&cn.spos, sizeof(uint32_t) * t));
  SBDX_CUDA(c, cudaMalloc(&cn.order, sizeof(uint32_t) * n));
  conn_fill_kernel<<<(unsigned)n, kConnThreads, 0, c->stream>>>(spin, s, n, cn.off, cn.nsing, c->L, c->d_h,
                                                                 c->d_eri, cn.ket, cn.val, cn.val32,
                                                                 cn.omask, cn.info, cn.srec, cn.spos);
  SBDX_LAUNCHED(c);
  if (!full) {
    SBDX_CUDA(c, cudaStreamSynchronize(c->stream));  // the host copy of `off` dies at return
    return 0;
  }
  // bra strings ordered by their number of singles (longest first), so the
  // threads of one warp in the alpha-beta kernels walk lists of similar length
  std::vector<uint32_t> order(n);
  for (size_t r = 0; r < n; ++r) order[r] = (uint32_t)r;
  std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return hs[x] > hs[y]; });
  SBDX_CUDA(c, cudaMemcpyAsync(cn.order, order.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, c->stream));
  {
    int rc = build_same_items(c, cn, hs, hd, spin == 0 ? c->nb : c->na);
    if (rc) return rc;
    if ((rc = build_same_blocks(c, cn, spin == 0 ? c->h_a : c->h_b, 0, n, hs, spin == 0 ? c->nb : c->na, cn.blk)))
      return rc;
    if (spin == 0 && (rc = build_ab_items(c, cn, hs, c->nb))) return rc;
  }
  // SELL-32 copy of the single-excitation records in list-length order
  {
    std::vector<uint64_t> rec(cn.total ? cn.total : 1);
    if (cn.total)
      SBDX_CUDA(c, cudaMemcpyAsync(rec.data(), cn.srec, sizeof(uint64_t) * cn.total, cudaMemcpyDeviceToHost, c->stream));
    SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
    const size_t ns = (n + 31) / 32;
    std::vector<uint64_t> soff(ns + 1, 0);
    std::vector<uint32_t> slen(ns, 0);
    for (size_t sl = 0; sl < ns; ++sl) {
      uint32_t mx = 0;
      for (size_t l = 0; l < 32 && sl * 32 + l < n; ++l) mx = std::max(mx, hs[order[sl * 32 + l]]);
      slen[sl] = mx;
      soff[sl + 1] = soff[sl] + 32ull * mx;
    }
    const uint64_t kPad = 1ull << 41;
    std::vector<uint64_t> sell(soff[ns] ? soff[ns] : 1, kPad);
    for (size_t sl = 0; sl < ns; ++sl)
      for (size_t l = 0; l < 32 && sl * 32 + l < n; ++l) {
        const uint32_t r = order[sl * 32 + l];
        for (uint32_t m = 0; m < hs[r]; ++m) sell[soff[sl] + 32ull * m + l] = rec[off[r] + m];
      }
    cn.nslice = ns;
    SBDX_CUDA(c, cudaMalloc(&cn.sell, sizeof(uint64_t) * sell.size()));
    SBDX_CUDA(c, cudaMalloc(&cn.soff, sizeof(uint64_t) * (ns + 1)));
    SBDX_CUDA(c, cudaMalloc(&cn.slen, sizeof(uint32_t) * (ns ? ns : 1)));
    SBDX_CUDA(c, cudaMemcpyAsync(cn.sell, sell.data(), sizeof(uint64_t) * sell.size(), cudaMemcpyHostToDevice, c->stream));
    SBDX_CUDA(c, cudaMemcpyAsync(cn.soff, soff.data(), sizeof(uint64_t) * (ns + 1), cudaMemcpyHostToDevice, c->stream));
    if (ns) SBDX_CUDA(c, cudaMemcpyAsync(cn.slen, slen.data(), sizeof(uint32_t) * ns, cudaMemcpyHostToDevice, c->stream));
    SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
    if (spin == 1) {
      const std::vector<uint32_t> kpos = ket_positions(n, hs, off, rec);
      SBDX_CUDA(c, cudaMalloc(&cn.kpos, sizeof(uint32_t) * n));
      SBDX_CUDA(c, cudaMemcpyAsync(cn.kpos, kpos.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, c->stream));
      int rc = build_balanced_sell(c, cn.bal, n, hs, off, rec, kpos, 0, (uint32_t)n);
      if (rc) return rc;
      // ket-range panels when the packed alpha-beta kernel (16 bytes per ket
      // and per pair index, 8 per split slot) cannot stage a whole ket row
      const size_t er = ab7_er_packs(c->npair);
      const size_t fixed = 16 * er + sizeof(double) * kMaxSplitSlots;
      if (16 * (n + er) + sizeof(double) * (size_t)cn.bal.nslot > kAbSmemBudget && fixed < kAbSmemBudget) {
        // panel widths are multiples of 8: the ket permutation keeps groups of 8
        const size_t width = ((kAbSmemBudget - fixed) / 16) & ~(size_t)7;
        const size_t np = (n + width - 1) / width;
        const size_t w = ((n + np - 1) / np + 7) & ~(size_t)7;
        for (size_t q = 0; q < np && q * w < n; ++q) {
          const uint32_t lo = (uint32_t)(q * w), hi = (uint32_t)std::min(n, (q + 1) * w);
          cn.panels.emplace_back();
          if ((rc = build_balanced_sell(c, cn.panels.back(), n, hs, off, rec, kpos, lo, hi))) return rc;
        }
      }
    }
  }
  // the host copy of `off` must stay alive until the async copy ran
  SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
  return 0;
}

}  // namespace

void free_blocks(SameBlocks& b) {
  cudaFree(b.rows); cudaFree(b.uoff); cudaFree(b.uket); cudaFree(b.uval); cudaFree(b.uval32);
  cudaFree(b.item); cudaFree(b.split); cudaFree(b.ypart);
  b = SameBlocks{};
}

void free_range_items(Conn& r) {
  free_blocks(r.blk);
  cudaFree(r.same_item); cudaFree(r.same_split); cudaFree(r.same_ypart);
  cudaFree(r.ab_item); cudaFree(r.ab_split); cudaFree(r.ypart);
  r.same_item = r.same_split = r.ab_item = r.ab_split = nullptr;
  r.same_ypart = r.ypart = nullptr;
  r.n_same_item = r.n_item = 0;
  r.n_same_split = r.n_same_part = r.n_split = r.n_part = 0;
}

void free_row_range(Ctx* c) {
  free_range_items(c->range_conn);
  c->range_a0 = c->range_a1 = 0;
  c->have_range = false;
}

// Work items of the alpha rows [a0, a1) only, for a sigma that writes those
// output rows (one shard of the alpha strings, or one chunk of a pipelined
// product): the same-spin and alpha-beta items of build_same_items /
// build_ab_items over that range, their caps derived from the range's own
// work.
int build_range_items(Ctx* c, size_t a0, size_t a1, Conn& r) {
  free_range_items(r);
  const Conn& ca = c->conn[0];
  const size_t n = a1 - a0;
  std::vector<uint32_t> hs(n ? n : 1), hd(n ? n : 1);
  if (n) {
    SBDX_CUDA(c, cudaMemcpyAsync(hs.data(), ca.nsing + a0, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, c->stream));
    SBDX_CUDA(c, cudaMemcpyAsync(hd.data(), ca.ndoub + a0, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, c->stream));
    SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  hs.resize(n);
  hd.resize(n);
  int rc = build_same_items(c, r, hs, hd, c->nb, a0);
  if (rc) return rc;
  if ((rc = build_same_blocks(c, ca, c->h_a, a0, n, hs, c->nb, r.blk))) return rc;
  return build_ab_items(c, r, hs, c->nb, a0);
}

int build_row_range(Ctx* c, size_t a0, size_t a1) {
  free_row_range(c);
  const int rc = build_range_items(c, a0, a1, c->range_conn);
  if (rc) return rc;
  c->range_a0 = a0;
  c->range_a1 = a1;
  c->have_range = true;
  return 0;
}

void free_connectivity(Ctx* c) {
  clear_sigma_graphs(c);
  release_stored(c);  // its elements come from the connectivity
  free_row_range(c);
  free_io_chunks(c);
  free_conn(c->conn[0]);
  free_conn(c->conn[1]);
  cudaFree(c->d_Da); cudaFree(c->d_Db); cudaFree(c->d_Da32); cudaFree(c->d_Db32);
  c->d_Da = c->d_Db = nullptr;
  c->d_Da32 = c->d_Db32 = nullptr;
  c->have_conn = false;
  c->have_lists = false;
}

int build_connectivity(Ctx* c, bool full) {
  if (!c->have_strings || !c->have_integrals) {
    c->err = "build_connectivity: set integrals and strings first";
    return 3;
  }
  free_connectivity(c);
  int rc = build_one(c, 0, full);
  if (rc) return rc;
  rc = build_one(c, 1, full);
  if (rc) return rc;
  c->have_lists = true;
  if (!full) return 0;
  rc = build_coulomb_tables(c);
  if (rc) return rc;
  c->have_conn = true;
  return 0;
}

}  // namespace sbdx
