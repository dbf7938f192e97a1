// C-ABI entry points (include/sbdx.h). Validation of every host input happens
// here, before any kernel sees it: sizes, orbital range, equal electron counts
// per spin, finite integrals. No C++ exception crosses the boundary.
#include "sbdx.h"
#include "sbdx_internal.cuh"

#include <cmath>
#include <cstring>
#include <exception>
#include <new>
#include <vector>

namespace sbdx {

bool set_cuda_err(Ctx* c, cudaError_t e, const char* what) {
  c->err = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
  return false;
}

cudaError_t make_pool(int device, cudaMemPool_t* pool) {
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  cudaError_t e = cudaMemPoolCreate(pool, &props);
  if (e != cudaSuccess) {
    *pool = nullptr;
    return e;
  }
  uint64_t keep = UINT64_MAX;
  return cudaMemPoolSetAttribute(*pool, cudaMemPoolAttrReleaseThreshold, &keep);
}

cudaError_t pool_alloc(Ctx* c, void** p, size_t bytes) {
  if (!c->pool) {
    const cudaError_t e = make_pool(c->device, &c->pool);
    if (e != cudaSuccess) return e;
    c->own_pool = true;
  }
  return cudaMallocFromPoolAsync(p, bytes, c->pool, c->stream);
}

void pool_trim(Ctx* c) {
  if (!c->pool || !c->own_pool) return;
  cudaStreamSynchronize(c->stream);
  cudaMemPoolTrimTo(c->pool, 0);
}

int check_device_error(Ctx* c) {
  int h = 0;
  SBDX_CUDA(c, cudaMemcpyAsync(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
  if (h == 0) return 0;
  SBDX_CUDA(c, cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
  c->err = "device watchdog: a bulk-copy completion wait timed out in the alpha-beta sigma kernel (code " +
           std::to_string(h) + ")";
  return SBDX_ERR_CUDA;
}

void free_connectivity(Ctx* c);
int build_g_table(Ctx* c);
int davidson(Ctx* c, const sbdx_davidson_params& p, double* dW, sbdx_davidson_info& info);
int rdm_device(Ctx* c, const double* dW, double* d_one, double* d_two);
int occupation_device(Ctx* c, const double* dW, double* d_density);
int alpha_weights_device(Ctx* c, const double* dW, double* d_w);
int backward_device(Ctx* c, const double* dW, double* dE_dh, double* dE_deri);
int autotune(Ctx* c);

namespace {

void free_vector_state(Ctx* c) {
  sbdx::clear_sigma_graphs(c);
  cudaFree(c->d_hii); c->d_hii = nullptr; c->have_hii = false;
  cudaFree(c->d_xt); c->d_xt = nullptr;
  cudaFree(c->d_xp); c->d_xp = nullptr;
  cudaFree(c->d_y); c->d_y = nullptr;
  cudaFree(c->d_yt); c->d_yt = nullptr;
  cudaFree(c->d_io_in); c->d_io_in = nullptr;
  cudaFree(c->d_io_out); c->d_io_out = nullptr;
  cudaFree(c->d_wf); c->d_wf = nullptr; c->wf_roots = 0; c->wf_cap = 0;
}

// Room for k resident result vectors (contents of earlier solves are dropped).
int ensure_wf(Ctx* c, int k) {
  const size_t D = c->na * c->nb;
  c->wf_roots = 0;
  if (c->wf_cap < k) {
    cudaFree(c->d_wf);
    c->d_wf = nullptr;
    c->wf_cap = 0;
    cudaError_t e = cudaMalloc(&c->d_wf, sizeof(double) * D * (size_t)k);
    if (e != cudaSuccess) {
      cudaGetLastError();
      c->err = "davidson: no device memory for " + std::to_string(k) + " result vector(s) of " + std::to_string(D) +
               " doubles";
      return SBDX_ERR_NOMEM;
    }
    c->wf_cap = k;
  }
  return 0;
}

int ensure_io(Ctx* c) {
  const size_t D = c->na * c->nb;
  if (!c->d_io_in) SBDX_CUDA(c, cudaMalloc(&c->d_io_in, sizeof(double) * D));
  if (!c->d_io_out) SBDX_CUDA(c, cudaMalloc(&c->d_io_out, sizeof(double) * D));
  return 0;
}

int ready(Ctx* c, const char* who) {
  if (!c->have_integrals || !c->have_strings) {
    c->err = std::string(who) + ": set integrals and strings first";
    return SBDX_ERR_STATE;
  }
  if (c->L < 64) {
    const uint64_t lim = 1ull << c->L;
    for (uint64_t x : c->h_a)
      if (x >= lim) { c->err = std::string(who) + ": alpha string has bits beyond norb"; return SBDX_ERR_ARG; }
    for (uint64_t x : c->h_b)
      if (x >= lim) { c->err = std::string(who) + ": beta string has bits beyond norb"; return SBDX_ERR_ARG; }
  }
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) { set_cuda_err(c, e, "cudaSetDevice"); return SBDX_ERR_CUDA; }
  return 0;
}

template <typename F>
int guarded(sbdx_ctx* ctx, F&& f) {
  if (!ctx) return SBDX_ERR_ARG;
  try {
    return f(&ctx->c);
  } catch (const std::bad_alloc&) {
    ctx->c.err = "host allocation failed";
    return SBDX_ERR_NOMEM;
  } catch (const std::exception& ex) {
    ctx->c.err = ex.what();
    return SBDX_ERR_ARG;
  } catch (...) {
    ctx->c.err = "unknown exception";
    return SBDX_ERR_ARG;
  }
}

// map internal 1/2/3/5 codes (already SBDX_*), keep as is
}  // namespace
}  // namespace sbdx

using sbdx::Ctx;

extern "C" {

int sbdx_ctx_create(sbdx_ctx** out, int device) {
  if (!out) return SBDX_ERR_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) return SBDX_ERR_CUDA;
  if (cudaSetDevice(device) != cudaSuccess) return SBDX_ERR_CUDA;
  sbdx_ctx* ctx = new (std::nothrow) sbdx_ctx();
  if (!ctx) return SBDX_ERR_NOMEM;
  ctx->c.device = device;
  if (cudaMalloc(&ctx->c.d_err, sizeof(int)) != cudaSuccess || cudaMemset(ctx->c.d_err, 0, sizeof(int)) != cudaSuccess) {
    delete ctx;
    return SBDX_ERR_CUDA;
  }
  *out = ctx;
  return SBDX_OK;
}

int sbdx_ctx_destroy(sbdx_ctx* ctx) {
  if (!ctx) return SBDX_OK;
  Ctx* c = &ctx->c;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  sbdx::free_connectivity(c);
  sbdx::free_vector_state(c);
  cudaFree(c->d_h); cudaFree(c->d_eri); cudaFree(c->d_eri32); cudaFree(c->d_G); cudaFree(c->d_G32);
  cudaFree(c->d_V); cudaFree(c->d_V32); cudaFree(c->d_err);
  cudaFree(c->d_a); cudaFree(c->d_b); cudaFree(c->d_red);
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  if (c->own_pool && c->pool) cudaMemPoolDestroy(c->pool);
  delete ctx;
  return SBDX_OK;
}

const char* sbdx_last_error(const sbdx_ctx* ctx) { return ctx ? ctx->c.err.c_str() : "null context"; }

unsigned long long sbdx_launch_count(const sbdx_ctx* ctx) { return ctx ? ctx->c.launches : 0ull; }

int sbdx_set_profiling(sbdx_ctx* ctx, int on) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    SBDX_CUDA(c, cudaSetDevice(c->device));
    if (on && !c->ev[0])
      for (auto& e : c->ev) SBDX_CUDA(c, cudaEventCreate(&e));
    for (double& x : c->phase_ms) x = 0.0;
    c->phase_calls = 0;
    c->profiling = on != 0;
    return SBDX_OK;
  });
}

long long sbdx_phase_times(sbdx_ctx* ctx, double* ms, int n) {
  if (!ctx || !ms) return -1;
  for (int k = 0; k < n && k < sbdx::kSigmaPhases; ++k) ms[k] = ctx->c.phase_ms[k];
  return (long long)ctx->c.phase_calls;
}

int sbdx_set_tuning(sbdx_ctx* ctx, int same_code, int ab_code) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    const int v = same_code % 10;
    const bool same_v6 = (same_code > 20 && same_code < 30) || (same_code > 30 && same_code < 40),
               ab_v6 = (ab_code > 60 && ab_code < 70) || ab_code == 71;
    const bool same_ok = same_code == 0 || ((same_code < 10 && (v == 1 || v == 2 || v == 4 || v == 8)) ||
                                            (same_code > 10 && same_code < 20 && (v == 1 || v == 2 || v == 4)) ||
                                            (same_v6 && (v == 1 || v == 2 || v == 4 || v == 8)));
    const bool ab_ok = ab_code == 0 || (ab_code > 0 && ab_code < 50 && ab_code % 10 >= 1 && ab_code % 10 <= 4) ||
                       (ab_v6 && ab_code % 10 >= 1 && ab_code % 10 <= 4);  // 71 included
    // the alpha-first codes (2x, 6x) evaluate the whole sigma in another
    // determinant ordering and cannot be mixed with the interleaved ones
    const bool mixed = (same_v6 && ab_code != 0 && !ab_v6) || (ab_v6 && same_code != 0 && !same_v6) ||
                       (same_code != 0 && !same_v6 && ab_code == 0) || (ab_code != 0 && !ab_v6 && same_code == 0);
    if (!same_ok || !ab_ok || mixed) {
      c->err = "set_tuning: alpha-first codes same in {21,22,24,28,31,32,34,38} with ab in {61..64, 71}, or "
               "interleaved codes "
               "same in {1,2,4,8,11,12,14} with ab = 10*variant + rows (variant 0-4, rows 1-4); 0 = default";
      return SBDX_ERR_ARG;
    }
    for (auto& t : c->tune) {
      t.same_code = same_code;
      t.ab_code = ab_code;
    }
    sbdx::clear_sigma_graphs(c);
    return SBDX_OK;
  });
}

int sbdx_autotune(sbdx_ctx* ctx, int* same_vec, int* ab_rows) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    int rc = sbdx::ready(c, "autotune");
    if (rc) return rc;
    rc = sbdx::autotune(c);
    if (rc) return rc;
    if (same_vec) *same_vec = c->tune[0].same_code;
    if (ab_rows) *ab_rows = c->tune[0].ab_code;
    return SBDX_OK;
  });
}

int sbdx_set_stream(sbdx_ctx* ctx, void* stream) {
  return sbdx::guarded(ctx, [&](Ctx* c) {
    sbdx::clear_sigma_graphs(c);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    c->own_stream = false;
    c->stream = (cudaStream_t)stream;
    return SBDX_OK;
  });
}

int sbdx_set_integrals(sbdx_ctx* ctx, int norb, double I0, const double* h, const double* eri, size_t eri_len) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    if (norb < 1 || norb > 64) { c->err = "set_integrals: norb must be in [1, 64]"; return SBDX_ERR_ARG; }
    if (!h || !eri) { c->err = "set_integrals: null pointer"; return SBDX_ERR_ARG; }
    const size_t npair = (size_t)norb * (norb + 1) / 2, neri = npair * (npair + 1) / 2;
    if (eri_len != neri) {
      c->err = "set_integrals: eri_len must be P*(P+1)/2 with P = norb*(norb+1)/2";
      return SBDX_ERR_ARG;
    }
    if (!std::isfinite(I0)) { c->err = "set_integrals: non-finite I0"; return SBDX_ERR_NUMERIC; }
    for (size_t k = 0; k < (size_t)norb * norb; ++k)
      if (!std::isfinite(h[k])) { c->err = "set_integrals: non-finite one-electron integral"; return SBDX_ERR_NUMERIC; }
    for (size_t k = 0; k < neri; ++k)
      if (!std::isfinite(eri[k])) { c->err = "set_integrals: non-finite two-electron integral"; return SBDX_ERR_NUMERIC; }
    if (cudaSetDevice(c->device) != cudaSuccess) { c->err = "cudaSetDevice failed"; return SBDX_ERR_CUDA; }
    cudaStreamSynchronize(c->stream);
    cudaFree(c->d_h); cudaFree(c->d_eri); cudaFree(c->d_eri32);
    c->d_h = nullptr; c->d_eri = nullptr; c->d_eri32 = nullptr;
    c->L = norb;
    c->I0 = I0;
    c->npair = npair;
    c->neri = neri;
    c->h_h.assign(h, h + (size_t)norb * norb);
    c->h_eri.assign(eri, eri + neri);
    std::vector<float> e32(neri);
    for (size_t k = 0; k < neri; ++k) e32[k] = (float)eri[k];
    SBDX_CUDA(c, cudaMalloc(&c->d_h, sizeof(double) * norb * norb));
    SBDX_CUDA(c, cudaMalloc(&c->d_eri, sizeof(double) * neri));
    SBDX_CUDA(c, cudaMalloc(&c->d_eri32, sizeof(float) * neri));
    SBDX_CUDA(c, cudaMemcpy(c->d_h, h, sizeof(double) * norb * norb, cudaMemcpyHostToDevice));
    SBDX_CUDA(c, cudaMemcpy(c->d_eri, eri, sizeof(double) * neri, cudaMemcpyHostToDevice));
    SBDX_CUDA(c, cudaMemcpy(c->d_eri32, e32.data(), sizeof(float) * neri, cudaMemcpyHostToDevice));
    int rc = sbdx::build_g_table(c);
    if (rc) return rc;
    SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
    c->have_integrals = true;
    // matrix elements cached in the connectivity and the diagonal depend on the integrals
    sbdx::free_connectivity(c);
    cudaFree(c->d_hii); c->d_hii = nullptr; c->have_hii = false;
    return SBDX_OK;
  });
}

int sbdx_set_strings(sbdx_ctx* ctx, const uint64_t* alpha, size_t na, const uint64_t* beta, size_t nb) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    if (!alpha || !beta || na == 0 || nb == 0) { c->err = "set_strings: empty string set"; return SBDX_ERR_ARG; }
    if (na > sbdx::kMaxStrings || nb > sbdx::kMaxStrings) {
      c->err = "set_strings: at most 16777215 strings per spin";
      return SBDX_ERR_ARG;
    }
    const int pa = __builtin_popcountll(alpha[0]), pb = __builtin_popcountll(beta[0]);
    for (size_t k = 0; k < na; ++k)
      if (__builtin_popcountll(alpha[k]) != pa) { c->err = "set_strings: alpha strings differ in electron count"; return SBDX_ERR_ARG; }
    for (size_t k = 0; k < nb; ++k)
      if (__builtin_popcountll(beta[k]) != pb) { c->err = "set_strings: beta strings differ in electron count"; return SBDX_ERR_ARG; }
    if (cudaSetDevice(c->device) != cudaSuccess) { c->err = "cudaSetDevice failed"; return SBDX_ERR_CUDA; }
    cudaStreamSynchronize(c->stream);
    sbdx::free_connectivity(c);
    sbdx::free_vector_state(c);
    cudaFree(c->d_a); cudaFree(c->d_b);
    c->d_a = nullptr; c->d_b = nullptr;
    c->na = na;
    c->nb = nb;
    c->h_a.assign(alpha, alpha + na);
    c->h_b.assign(beta, beta + nb);
    SBDX_CUDA(c, cudaMalloc(&c->d_a, sizeof(uint64_t) * na));
    SBDX_CUDA(c, cudaMalloc(&c->d_b, sizeof(uint64_t) * nb));
    SBDX_CUDA(c, cudaMemcpy(c->d_a, alpha, sizeof(uint64_t) * na, cudaMemcpyHostToDevice));
    SBDX_CUDA(c, cudaMemcpy(c->d_b, beta, sizeof(uint64_t) * nb, cudaMemcpyHostToDevice));
    c->have_strings = true;
    return SBDX_OK;
  });
}

int sbdx_build_connectivity(sbdx_ctx* ctx) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    int rc = sbdx::ready(c, "build_connectivity");
    if (rc) return rc;
    rc = sbdx::build_connectivity(c);
    if (rc) return rc;
    SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
    return SBDX_OK;
  });
}

int sbdx_build_hamiltonian(sbdx_ctx* ctx, uint64_t* nnz) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    int rc = sbdx::ready(c, "build_hamiltonian");
    if (rc) return rc;
    if ((rc = sbdx::build_stored(c))) return rc;
    if (nnz) *nnz = c->stored.nnz;
    return SBDX_OK;
  });
}

int sbdx_release_hamiltonian(sbdx_ctx* ctx) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
    sbdx::release_stored(c);
    sbdx::clear_sigma_graphs(c);
    return SBDX_OK;
  });
}

int sbdx_connectivity_size(sbdx_ctx* ctx, int spin, uint64_t* n_entries) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    if (spin != 0 && spin != 1) { c->err = "connectivity_size: spin must be 0 or 1"; return SBDX_ERR_ARG; }
    if (!n_entries) { c->err = "connectivity_size: null pointer"; return SBDX_ERR_ARG; }
    if (!c->have_lists) { c->err = "connectivity_size: build the connectivity first"; return SBDX_ERR_STATE; }
    *n_entries = c->conn[spin].total;
    return SBDX_OK;
  });
}

int sbdx_get_connectivity(sbdx_ctx* ctx, int spin, uint64_t* slen, uint64_t* dlen, uint64_t* idx) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    if (spin != 0 && spin != 1) { c->err = "get_connectivity: spin must be 0 or 1"; return SBDX_ERR_ARG; }
    if (!c->have_lists) { c->err = "get_connectivity: build the connectivity first"; return SBDX_ERR_STATE; }
    const sbdx::Conn& cn = c->conn[spin];
    std::vector<uint32_t> ns(cn.n), nd(cn.n), ket(cn.total);
    SBDX_CUDA(c, cudaSetDevice(c->device));
    SBDX_CUDA(c, cudaMemcpy(ns.data(), cn.nsing, sizeof(uint32_t) * cn.n, cudaMemcpyDeviceToHost));
    SBDX_CUDA(c, cudaMemcpy(nd.data(), cn.ndoub, sizeof(uint32_t) * cn.n, cudaMemcpyDeviceToHost));
    if (cn.total) SBDX_CUDA(c, cudaMemcpy(ket.data(), cn.ket, sizeof(uint32_t) * cn.total, cudaMemcpyDeviceToHost));
    for (size_t r = 0; r < cn.n; ++r) {
      if (slen) slen[r] = ns[r];
      if (dlen) dlen[r] = nd[r];
    }
    if (idx)
      for (size_t k = 0; k < cn.total; ++k) idx[k] = ket[k];
    return SBDX_OK;
  });
}

int sbdx_diag_terms(sbdx_ctx* ctx, double* hii) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    int rc = sbdx::ready(c, "diag_terms");
    if (rc) return rc;
    rc = sbdx::diag_terms(c);
    if (rc) return rc;
    if (hii) SBDX_CUDA(c, cudaMemcpyAsync(hii, c->d_hii, sizeof(double) * c->na * c->nb, cudaMemcpyDeviceToHost, c->stream));
    SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
    return SBDX_OK;
  });
}

int sbdx_sigma(sbdx_ctx* ctx, const double* C, double* S) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    if (!C || !S) { c->err = "sigma: null pointer"; return SBDX_ERR_ARG; }
    int rc = sbdx::ready(c, "sigma");
    if (rc) return rc;
    if ((rc = sbdx::ensure_io(c))) return rc;
    if ((rc = sbdx::sigma_host(c, C, S))) return rc;
    return sbdx::check_device_error(c);
  });
}

int sbdx_sigma_device(sbdx_ctx* ctx, int precision, const void* dC, void* dS) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    if (!dC || !dS) { c->err = "sigma_device: null pointer"; return SBDX_ERR_ARG; }
    if (dC == dS) { c->err = "sigma_device: input and output must not alias"; return SBDX_ERR_ARG; }
    int rc = sbdx::ready(c, "sigma_device");
    if (rc) return rc;
    return sbdx::sigma_device(c, precision, dC, dS);
  });
}

int sbdx_set_io_chunks(sbdx_ctx* ctx, int chunks) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    if (chunks < 0) { c->err = "set_io_chunks: chunks must be >= 0"; return SBDX_ERR_ARG; }
    cudaStreamSynchronize(c->stream);
    sbdx::free_io_chunks(c);
    c->io_chunks_req = chunks;
    return SBDX_OK;
  });
}

int sbdx_set_graph_steps(sbdx_ctx* ctx, int on) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    c->graph_steps = on != 0;
    return SBDX_OK;
  });
}

int sbdx_sigma_rows_device(sbdx_ctx* ctx, int precision, const void* dC, void* dS, size_t a0, size_t a1) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    if (!dC || (!dS && a1 > a0)) { c->err = "sigma_rows_device: null pointer"; return SBDX_ERR_ARG; }
    int rc = sbdx::ready(c, "sigma_rows_device");
    if (rc) return rc;
    const size_t es = precision == SBDX_FP32 ? sizeof(float) : sizeof(double);
    const char* C0 = static_cast<const char*>(dC);
    const char* S0 = static_cast<const char*>(dS);
    if (S0 && S0 < C0 + es * c->na * c->nb && C0 < S0 + es * (a1 - a0) * c->nb) {
      c->err = "sigma_rows_device: input and output must not overlap";
      return SBDX_ERR_ARG;
    }
    return sbdx::sigma_rows_device(c, precision, dC, dS, a0, a1);
  });
}

int sbdx_project_device(sbdx_ctx* ctx, int precision, const void* dV, size_t ldv, int m, const void* dX, size_t ldx,
                        int nx, size_t D, double* dP) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    if (m < 0 || nx < 1 || nx > 8) { c->err = "project_device: need m >= 0 and 1 <= nx <= 8"; return SBDX_ERR_ARG; }
    if (m > 0 && (!dV || !dX || !dP)) { c->err = "project_device: null pointer"; return SBDX_ERR_ARG; }
    if ((m > 1 && ldv < D) || (nx > 1 && ldx < D)) { c->err = "project_device: stride below D"; return SBDX_ERR_ARG; }
    return sbdx::project_device(c, precision, dV, ldv, m, dX, ldx, nx, D, dP);
  });
}

int sbdx_davidson(sbdx_ctx* ctx, const sbdx_davidson_params* params, int init_from_W, double* W,
                  sbdx_davidson_info* info) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    if (!params || (!W && init_from_W)) { c->err = "davidson: null pointer"; return SBDX_ERR_ARG; }
    int rc = sbdx::ready(c, "davidson");
    if (rc) return rc;
    const size_t D = c->na * c->nb;
    if (init_from_W)
      for (size_t k = 0; k < D; ++k)
        if (!std::isfinite(W[k])) { c->err = "davidson: non-finite start vector"; return SBDX_ERR_NUMERIC; }
    if ((rc = sbdx::ensure_wf(c, 1))) return rc;
    double* dW = c->d_wf;
    if (init_from_W) {
      SBDX_CUDA(c, cudaMemcpyAsync(dW, W, sizeof(double) * D, cudaMemcpyHostToDevice, c->stream));
    } else {
      // BasisInitVector, init == 0 (davidson.h:130-133): W[0] = 1
      SBDX_CUDA(c, cudaMemsetAsync(dW, 0, sizeof(double) * D, c->stream));
      const double one = 1.0;
      SBDX_CUDA(c, cudaMemcpyAsync(dW, &one, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    }
    sbdx_davidson_info inf{};
    rc = sbdx::davidson(c, *params, dW, inf);
    if (rc) return rc;
    if ((rc = sbdx::check_device_error(c))) return rc;
    c->wf_roots = 1;
    if (W) SBDX_CUDA(c, cudaMemcpyAsync(W, dW, sizeof(double) * D, cudaMemcpyDeviceToHost, c->stream));
    SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
    if (info) *info = inf;
    return SBDX_OK;
  });
}

int sbdx_davidson_roots(sbdx_ctx* ctx, const sbdx_davidson_params* params, int nroots, int init_from_W,
                        double* W, double* energies, double* residuals, sbdx_davidson_info* info) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    if (!params || (!W && init_from_W) || !energies) { c->err = "davidson_roots: null pointer"; return SBDX_ERR_ARG; }
    if (nroots < 1 || nroots > 4) { c->err = "davidson_roots: nroots must be in [1, 4]"; return SBDX_ERR_ARG; }
    int rc = sbdx::ready(c, "davidson_roots");
    if (rc) return rc;
    const size_t D = c->na * c->nb;
    if ((size_t)nroots > D) { c->err = "davidson_roots: more roots than determinants"; return SBDX_ERR_ARG; }
    if (init_from_W)
      for (size_t q = 0; q < D * nroots; ++q)
        if (!std::isfinite(W[q])) { c->err = "davidson_roots: non-finite start vector"; return SBDX_ERR_NUMERIC; }
    if ((rc = sbdx::ensure_wf(c, nroots))) return rc;
    double* dW = c->d_wf;
    struct Guard {
      Ctx* c;
      ~Guard() { sbdx::pool_trim(c); }
    } g{c};
    if (init_from_W) {
      SBDX_CUDA(c, cudaMemcpyAsync(dW, W, sizeof(double) * D * nroots, cudaMemcpyHostToDevice, c->stream));
    } else {  // unit vectors on the nroots lowest diagonal elements
      std::vector<size_t> idx;
      if ((rc = sbdx::lowest_diagonal(c, nroots, idx))) return rc;
      SBDX_CUDA(c, cudaMemsetAsync(dW, 0, sizeof(double) * D * nroots, c->stream));
      static const double one = 1.0;
      for (int r = 0; r < nroots; ++r)
        SBDX_CUDA(c, cudaMemcpyAsync(dW + (size_t)r * D + idx[r], &one, sizeof(double), cudaMemcpyHostToDevice,
                                     c->stream));
    }
    std::vector<double> e(nroots), res(nroots);
    sbdx_davidson_info inf{};
    if ((rc = sbdx::davidson_roots(c, *params, nroots, dW, e.data(), res.data(), inf))) return rc;
    if ((rc = sbdx::check_device_error(c))) return rc;
    c->wf_roots = nroots;
    if (W) SBDX_CUDA(c, cudaMemcpyAsync(W, dW, sizeof(double) * D * nroots, cudaMemcpyDeviceToHost, c->stream));
    SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int r = 0; r < nroots; ++r) {
      energies[r] = e[r];
      if (residuals) residuals[r] = res[r];
    }
    if (info) *info = inf;
    return SBDX_OK;
  });
}

int sbdx_rdm(sbdx_ctx* ctx, const double* W, double* one, double* two) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    if (!W || !one) { c->err = "rdm: null pointer"; return SBDX_ERR_ARG; }
    int rc = sbdx::ready(c, "rdm");
    if (rc) return rc;
    if ((rc = sbdx::ensure_io(c))) return rc;
    const size_t D = c->na * c->nb, L = (size_t)c->L, L2 = L * L, L4 = L2 * L2;
    SBDX_CUDA(c, cudaMemcpyAsync(c->d_io_in, W, sizeof(double) * D, cudaMemcpyHostToDevice, c->stream));
    double *d_one = nullptr, *d_two = nullptr;
    SBDX_CUDA(c, cudaMalloc(&d_one, sizeof(double) * 2 * L2));
    if (two) {
      cudaError_t e = cudaMalloc(&d_two, sizeof(double) * 4 * L4);
      if (e != cudaSuccess) { cudaFree(d_one); sbdx::set_cuda_err(c, e, "cudaMalloc(2-RDM)"); return SBDX_ERR_NOMEM; }
    }
    rc = sbdx::rdm_device(c, (const double*)c->d_io_in, d_one, d_two);
    if (!rc) {
      cudaError_t e = cudaMemcpyAsync(one, d_one, sizeof(double) * 2 * L2, cudaMemcpyDeviceToHost, c->stream);
      if (e == cudaSuccess && two) e = cudaMemcpyAsync(two, d_two, sizeof(double) * 4 * L4, cudaMemcpyDeviceToHost, c->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
      if (e != cudaSuccess) { sbdx::set_cuda_err(c, e, "rdm copy-out"); rc = SBDX_ERR_CUDA; }
    }
    cudaFree(d_one);
    cudaFree(d_two);
    return rc;
  });
}

int sbdx_occupation(sbdx_ctx* ctx, const double* W, double* density) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    if (!W || !density) { c->err = "occupation: null pointer"; return SBDX_ERR_ARG; }
    int rc = sbdx::ready(c, "occupation");
    if (rc) return rc;
    if ((rc = sbdx::ensure_io(c))) return rc;
    const size_t D = c->na * c->nb;
    SBDX_CUDA(c, cudaMemcpyAsync(c->d_io_in, W, sizeof(double) * D, cudaMemcpyHostToDevice, c->stream));
    double* d = (double*)c->d_io_out;
    if ((rc = sbdx::occupation_device(c, (const double*)c->d_io_in, d))) return rc;
    SBDX_CUDA(c, cudaMemcpyAsync(density, d, sizeof(double) * 2 * c->L, cudaMemcpyDeviceToHost, c->stream));
    SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
    return SBDX_OK;
  });
}

int sbdx_alpha_weights(sbdx_ctx* ctx, const double* W, double* weights) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    if (!W || !weights) { c->err = "alpha_weights: null pointer"; return SBDX_ERR_ARG; }
    int rc = sbdx::ready(c, "alpha_weights");
    if (rc) return rc;
    if ((rc = sbdx::ensure_io(c))) return rc;
    const size_t D = c->na * c->nb;
    SBDX_CUDA(c, cudaMemcpyAsync(c->d_io_in, W, sizeof(double) * D, cudaMemcpyHostToDevice, c->stream));
    double* d = (double*)c->d_io_out;
    if ((rc = sbdx::alpha_weights_device(c, (const double*)c->d_io_in, d))) return rc;
    SBDX_CUDA(c, cudaMemcpyAsync(weights, d, sizeof(double) * c->na, cudaMemcpyDeviceToHost, c->stream));
    SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
    return SBDX_OK;
  });
}

int sbdx_energy_backward(sbdx_ctx* ctx, const double* W, double* dE_dh, double* dE_deri) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    if (!W || !dE_dh || !dE_deri) { c->err = "energy_backward: null pointer"; return SBDX_ERR_ARG; }
    int rc = sbdx::ready(c, "energy_backward");
    if (rc) return rc;
    if ((rc = sbdx::ensure_io(c))) return rc;
    const size_t D = c->na * c->nb;
    SBDX_CUDA(c, cudaMemcpyAsync(c->d_io_in, W, sizeof(double) * D, cudaMemcpyHostToDevice, c->stream));
    return sbdx::backward_device(c, (const double*)c->d_io_in, dE_dh, dE_deri);
  });
}

// ---- reductions on device-resident vectors ----------------------------------------

int sbdx_wavefunction_device(sbdx_ctx* ctx, int root, const double** dW) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    if (!dW) { c->err = "wavefunction_device: null pointer"; return SBDX_ERR_ARG; }
    if (c->wf_roots == 0) { c->err = "wavefunction_device: no Davidson solve has run on this basis"; return SBDX_ERR_STATE; }
    if (root < 0 || root >= c->wf_roots) {
      c->err = "wavefunction_device: root " + std::to_string(root) + " outside [0, " + std::to_string(c->wf_roots) + ")";
      return SBDX_ERR_ARG;
    }
    *dW = c->d_wf + (size_t)root * c->na * c->nb;
    return SBDX_OK;
  });
}

int sbdx_get_wavefunction(sbdx_ctx* ctx, int root, double* W) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    const double* dW = nullptr;
    int rc = sbdx_wavefunction_device(ctx, root, &dW);
    if (rc) return rc;
    if (!W) { c->err = "get_wavefunction: null pointer"; return SBDX_ERR_ARG; }
    SBDX_CUDA(c, cudaMemcpyAsync(W, dW, sizeof(double) * c->na * c->nb, cudaMemcpyDeviceToHost, c->stream));
    SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
    return SBDX_OK;
  });
}

int sbdx_rdm_device(sbdx_ctx* ctx, const double* dW, double* one, double* two) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    if (!dW || !one) { c->err = "rdm_device: null pointer"; return SBDX_ERR_ARG; }
    int rc = sbdx::ready(c, "rdm_device");
    if (rc) return rc;
    const size_t L = (size_t)c->L, L2 = L * L, L4 = L2 * L2;
    double *d_one = nullptr, *d_two = nullptr;
    SBDX_CUDA(c, cudaMalloc(&d_one, sizeof(double) * 2 * L2));
    if (two) {
      cudaError_t e = cudaMalloc(&d_two, sizeof(double) * 4 * L4);
      if (e != cudaSuccess) { cudaFree(d_one); sbdx::set_cuda_err(c, e, "cudaMalloc(2-RDM)"); return SBDX_ERR_NOMEM; }
    }
    rc = sbdx::rdm_device(c, dW, d_one, d_two);
    if (!rc) {
      cudaError_t e = cudaMemcpyAsync(one, d_one, sizeof(double) * 2 * L2, cudaMemcpyDeviceToHost, c->stream);
      if (e == cudaSuccess && two) e = cudaMemcpyAsync(two, d_two, sizeof(double) * 4 * L4, cudaMemcpyDeviceToHost, c->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
      if (e != cudaSuccess) { sbdx::set_cuda_err(c, e, "rdm copy-out"); rc = SBDX_ERR_CUDA; }
    }
    cudaFree(d_one);
    cudaFree(d_two);
    return rc;
  });
}

int sbdx_occupation_device(sbdx_ctx* ctx, const double* dW, double* density) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    if (!dW || !density) { c->err = "occupation_device: null pointer"; return SBDX_ERR_ARG; }
    int rc = sbdx::ready(c, "occupation_device");
    if (rc) return rc;
    if ((rc = sbdx::ensure_io(c))) return rc;
    double* d = (double*)c->d_io_out;
    if ((rc = sbdx::occupation_device(c, dW, d))) return rc;
    SBDX_CUDA(c, cudaMemcpyAsync(density, d, sizeof(double) * 2 * c->L, cudaMemcpyDeviceToHost, c->stream));
    SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
    return SBDX_OK;
  });
}

int sbdx_alpha_weights_device(sbdx_ctx* ctx, const double* dW, double* weights) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    if (!dW || !weights) { c->err = "alpha_weights_device: null pointer"; return SBDX_ERR_ARG; }
    int rc = sbdx::ready(c, "alpha_weights_device");
    if (rc) return rc;
    if ((rc = sbdx::ensure_io(c))) return rc;
    double* d = (double*)c->d_io_out;
    if ((rc = sbdx::alpha_weights_device(c, dW, d))) return rc;
    SBDX_CUDA(c, cudaMemcpyAsync(weights, d, sizeof(double) * c->na, cudaMemcpyDeviceToHost, c->stream));
    SBDX_CUDA(c, cudaStreamSynchronize(c->stream));
    return SBDX_OK;
  });
}

int sbdx_energy_backward_device(sbdx_ctx* ctx, const double* dW, double* dE_dh, double* dE_deri) {
  return sbdx::guarded(ctx, [&](Ctx* c) -> int {
    if (!dW || !dE_dh || !dE_deri) { c->err = "energy_backward_device: null pointer"; return SBDX_ERR_ARG; }
    int rc = sbdx::ready(c, "energy_backward_device");
    if (rc) return rc;
    return sbdx::backward_device(c, dW, dE_dh, dE_deri);
  });
}

}  // extern "C"
