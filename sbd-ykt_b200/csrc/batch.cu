// Batched solves: many independent sampled subspaces (alpha x beta string
// sets) that share one Hamiltonian, each solved for its lowest roots.
//
// The reference solves one basis per tpb::diag call (chemistry/tpb/sbdiag.h:
// 113-124); a caller with many sampled subspaces (for example the
// configuration-recovery loops of sample-based quantum diagonalisation) calls
// it once per subspace. Here the subspaces of one batch are solved
// concurrently on one GPU:
//   - every subspace has its own context (connectivity, diagonal, Coulomb
//     tables, sigma scratch) on its own non-blocking stream, so the kernels of
//     different subspaces overlap; the small subspaces, whose sigmas are a few
//     microseconds of work, no longer leave the GPU idle between launches;
//   - each subspace's sigma (five kernels) is captured once per (input,
//     output) buffer pair into a CUDA graph and replayed, so a step of a small
//     subspace costs one graph launch instead of five kernel launches;
//   - a pool of host threads drives the Davidson solves, largest subspace
//     first; the solvers allocate stream-ordered from one memory pool of the
//     batch that keeps its memory until the batch is done, so no solve stalls
//     the others with a device-wide synchronisation or a remapping;
//   - the launch shapes of the sigma kernels are tuned once on the largest
//     subspace and applied to all.
#include "sbdx.h"
#include "sbdx_internal.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

struct sbdx_batch {
  int device = 0;
  cudaMemPool_t pool = nullptr;  // shared by the subspaces' contexts
  std::string err;
  int L = 0;
  double I0 = 0.0;
  std::vector<double> h, eri;
  struct Sub {
    sbdx_ctx* ctx = nullptr;
    double* dW = nullptr;  // nroots vectors of the last solve (device)
    int nroots = 0;
  };
  std::vector<Sub> subs;
  bool graph_steps = false;  // the subspaces' solves run one CUDA graph per iteration
};

namespace {

int fail(sbdx_batch* b, int code, const std::string& msg) {
  b->err = msg;
  return code;
}

void release_vectors(sbdx_batch::Sub& s) {
  if (s.dW) cudaFreeAsync(s.dW, s.ctx->c.stream);
  s.dW = nullptr;
  s.nroots = 0;
}

}  // namespace

int sbdx_batch_create(sbdx_batch** out, int device, int norb, double I0, const double* h, const double* eri,
                      size_t eri_len) {
  if (!out) return SBDX_ERR_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) return SBDX_ERR_CUDA;
  if (norb < 1 || norb > 64 || !h || !eri) return SBDX_ERR_ARG;
  const size_t npair = (size_t)norb * (norb + 1) / 2;
  if (eri_len != npair * (npair + 1) / 2) return SBDX_ERR_ARG;
  sbdx_batch* b = new (std::nothrow) sbdx_batch();
  if (!b) return SBDX_ERR_NOMEM;
  b->device = device;
  if (cudaSetDevice(device) != cudaSuccess || sbdx::make_pool(device, &b->pool) != cudaSuccess) {
    if (b->pool) cudaMemPoolDestroy(b->pool);
    delete b;
    return SBDX_ERR_CUDA;
  }
  b->L = norb;
  b->I0 = I0;
  b->h.assign(h, h + (size_t)norb * norb);
  b->eri.assign(eri, eri + eri_len);
  *out = b;
  return SBDX_OK;
}

int sbdx_batch_destroy(sbdx_batch* b) {
  if (!b) return SBDX_OK;
  cudaSetDevice(b->device);
  for (auto& s : b->subs) {
    release_vectors(s);
    sbdx_ctx_destroy(s.ctx);
  }
  if (b->pool) cudaMemPoolDestroy(b->pool);
  delete b;
  return SBDX_OK;
}

const char* sbdx_batch_last_error(const sbdx_batch* b) { return b ? b->err.c_str() : "null batch"; }

int sbdx_batch_size(const sbdx_batch* b) { return b ? (int)b->subs.size() : 0; }

int sbdx_batch_add(sbdx_batch* b, const uint64_t* alpha, size_t na, const uint64_t* beta, size_t nb, int* index) {
  if (!b) return SBDX_ERR_ARG;
  try {
    sbdx_ctx* ctx = nullptr;
    int rc = sbdx_ctx_create(&ctx, b->device);
    if (rc) return fail(b, rc, "batch_add: cannot create a context");
    auto drop = [&](int code) {
      b->err = std::string("batch_add: ") + sbdx_last_error(ctx);
      sbdx_ctx_destroy(ctx);
      return code;
    };
    ctx->c.pool = b->pool;  // not owned: the batch destroys it
    ctx->c.own_pool = false;
    if ((rc = sbdx_set_integrals(ctx, b->L, b->I0, b->h.data(), b->eri.data(), b->eri.size()))) return drop(rc);
    if ((rc = sbdx_set_strings(ctx, alpha, na, beta, nb))) return drop(rc);
    sbdx::Ctx* c = &ctx->c;
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return drop(SBDX_ERR_CUDA);
    c->stream = st;
    c->own_stream = true;
    if ((rc = sbdx_build_connectivity(ctx))) return drop(rc);
    if ((rc = sbdx_diag_terms(ctx, nullptr))) return drop(rc);
    if ((rc = sbdx::ensure_sigma_scratch(c))) return drop(rc);
    c->use_graphs = true;
    c->graph_steps = b->graph_steps;
    b->subs.push_back({ctx, nullptr, 0});
    if (index) *index = (int)b->subs.size() - 1;
    return SBDX_OK;
  } catch (const std::bad_alloc&) {
    return fail(b, SBDX_ERR_NOMEM, "batch_add: host allocation failed");
  } catch (...) {
    return fail(b, SBDX_ERR_ARG, "batch_add: unexpected host exception");
  }
}

int sbdx_batch_set_graph_steps(sbdx_batch* b, int on) {
  if (!b) return SBDX_ERR_ARG;
  for (auto& sub : b->subs) sub.ctx->c.graph_steps = on != 0;
  b->graph_steps = on != 0;
  return SBDX_OK;
}

int sbdx_batch_tune(sbdx_batch* b, int* same_code, int* ab_code) {
  if (!b) return SBDX_ERR_ARG;
  if (b->subs.empty()) return fail(b, SBDX_ERR_STATE, "batch_tune: empty batch");
  size_t big = 0;
  for (size_t i = 1; i < b->subs.size(); ++i)
    if (b->subs[i].ctx->c.na * b->subs[i].ctx->c.nb > b->subs[big].ctx->c.na * b->subs[big].ctx->c.nb) big = i;
  sbdx_ctx* ref = b->subs[big].ctx;
  int s = 0, a = 0;
  int rc = sbdx_autotune(ref, &s, &a);
  if (rc) return fail(b, rc, std::string("batch_tune: ") + sbdx_last_error(ref));
  // the tuned codes go to the subspaces of comparable size; much smaller ones
  // keep the size-dependent defaults (a launch shape that fills the GPU on the
  // largest subspace can leave it half idle on one a few times smaller)
  const size_t dbig = ref->c.na * ref->c.nb;
  for (auto& sub : b->subs) {
    sbdx::Ctx* c = &sub.ctx->c;
    const bool near = 4 * c->na * c->nb >= dbig;
    c->tune[0] = near ? ref->c.tune[0] : sbdx::Tune{};
    c->tune[1] = near ? ref->c.tune[1] : sbdx::Tune{};
    sbdx::clear_sigma_graphs(c);
  }
  if (same_code) *same_code = s;
  if (ab_code) *ab_code = a;
  return SBDX_OK;
}

int sbdx_batch_solve(sbdx_batch* b, const sbdx_davidson_params* params, int nroots, int nthreads,
                     double* energies, double* residuals, sbdx_davidson_info* infos, double* seconds) {
  if (!b) return SBDX_ERR_ARG;
  if (!params || !energies) return fail(b, SBDX_ERR_ARG, "batch_solve: null pointer");
  if (nroots < 1 || nroots > 4) return fail(b, SBDX_ERR_ARG, "batch_solve: nroots must be in [1, 4]");
  const int K = (int)b->subs.size();
  if (K == 0) return fail(b, SBDX_ERR_STATE, "batch_solve: empty batch");
  for (auto& s : b->subs)
    if (s.ctx->c.na * s.ctx->c.nb < (size_t)nroots) return fail(b, SBDX_ERR_ARG, "batch_solve: subspace smaller than nroots");
  if (cudaSetDevice(b->device) != cudaSuccess) return fail(b, SBDX_ERR_CUDA, "batch_solve: cudaSetDevice failed");
  for (auto& s : b->subs) release_vectors(s);
  // largest subspace first, so that the long solves start early
  std::vector<int> order(K);
  for (int i = 0; i < K; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    return b->subs[x].ctx->c.na * b->subs[x].ctx->c.nb > b->subs[y].ctx->c.na * b->subs[y].ctx->c.nb;
  });
  const int T = std::max(1, std::min(nthreads > 0 ? nthreads : 8, K));
  std::atomic<int> next{0};
  std::mutex mu;
  int first_rc = 0;
  std::string first_err;
  const auto t0 = std::chrono::steady_clock::now();
  auto worker = [&]() {
    cudaSetDevice(b->device);
    for (;;) {
      const int slot = next.fetch_add(1);
      if (slot >= K) return;
      {
        std::lock_guard<std::mutex> lk(mu);
        if (first_rc) return;
      }
      const int i = order[slot];
      sbdx_batch::Sub& sub = b->subs[i];
      sbdx::Ctx* c = &sub.ctx->c;
      const size_t D = c->na * c->nb;
      int rc = 0;
      std::string err;
      try {
        double* dW = nullptr;
        if (sbdx::pool_alloc(c, (void**)&dW, sizeof(double) * D * nroots) != cudaSuccess) {
          rc = SBDX_ERR_NOMEM;
          err = "cudaMalloc(start vectors)";
        } else {
          sub.dW = dW;
          sub.nroots = nroots;
          std::vector<size_t> idx;
          rc = sbdx::lowest_diagonal(c, nroots, idx);
          if (!rc && cudaMemsetAsync(dW, 0, sizeof(double) * D * nroots, c->stream) != cudaSuccess) rc = SBDX_ERR_CUDA;
          static const double one = 1.0;
          for (int r = 0; !rc && r < nroots; ++r)
            if (cudaMemcpyAsync(dW + (size_t)r * D + idx[r], &one, sizeof(double), cudaMemcpyHostToDevice,
                                c->stream) != cudaSuccess)
              rc = SBDX_ERR_CUDA;
          std::vector<double> e(nroots), res(nroots);
          sbdx_davidson_info inf{};
          if (!rc) rc = sbdx::davidson_roots(c, *params, nroots, dW, e.data(), res.data(), inf);
          if (!rc) rc = sbdx::check_device_error(c);
          if (!rc) {
            for (int r = 0; r < nroots; ++r) {
              energies[(size_t)i * nroots + r] = e[r];
              if (residuals) residuals[(size_t)i * nroots + r] = res[r];
            }
            if (infos) infos[i] = inf;
          }
          if (rc) err = c->err;
        }
      } catch (...) {
        rc = SBDX_ERR_ARG;
        err = "unexpected host exception";
      }
      if (rc) {
        std::lock_guard<std::mutex> lk(mu);
        if (!first_rc) {
          first_rc = rc;
          first_err = "batch_solve: subspace " + std::to_string(i) + ": " + err;
        }
        return;
      }
    }
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < T; ++t) pool.emplace_back(worker);
  for (auto& th : pool) th.join();
  cudaDeviceSynchronize();
  if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  cudaMemPoolTrimTo(b->pool, 0);  // keeps only the returned Ritz vectors
  if (first_rc) return fail(b, first_rc, first_err);
  return SBDX_OK;
}

int sbdx_batch_vector(sbdx_batch* b, int index, int root, double* W) {
  if (!b || !W) return SBDX_ERR_ARG;
  if (index < 0 || index >= (int)b->subs.size()) return fail(b, SBDX_ERR_ARG, "batch_vector: index out of range");
  const auto& s = b->subs[index];
  if (!s.dW || root < 0 || root >= s.nroots) return fail(b, SBDX_ERR_STATE, "batch_vector: no solved root");
  const size_t D = s.ctx->c.na * s.ctx->c.nb;
  cudaSetDevice(b->device);
  if (cudaMemcpy(W, s.dW + (size_t)root * D, sizeof(double) * D, cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail(b, SBDX_ERR_CUDA, "batch_vector: copy failed");
  return SBDX_OK;
}

int sbdx_batch_dims(const sbdx_batch* b, int index, size_t* na, size_t* nb) {
  if (!b || index < 0 || index >= (int)b->subs.size()) return SBDX_ERR_ARG;
  if (na) *na = b->subs[index].ctx->c.na;
  if (nb) *nb = b->subs[index].ctx->c.nb;
  return SBDX_OK;
}
