// Ensembles of independent replicas and the particle-mesh grid autotuner.
//
// No counterpart in the reference (one system per process).  A batch holds
// contexts of any sizes, flows and strain rates; bd_batch_step_lanczos
// advances all of them by the same number of Krylov Brownian steps with one
// host worker thread per replica, each driving its context's own CUDA
// stream, so the kernels of small replicas run concurrently and fill the GPU
// that one small replica alone would leave idle.  The replicas share no
// device memory and need no synchronisation between them; the call returns
// when every replica has finished, with the first failing replica's status.
//
// bd_autotune_pme_grid picks the particle-mesh grid for a box: among the
// FFT-friendly sizes (2^a 3^b 5^c) from the accuracy bound 1.29 L up to 25 %
// above it, the one whose batched three-component R2C + C2R round trip is
// fastest on this GPU (timed with CUDA events, cached per size and
// precision).
#include <cufft.h>
#include <math.h>

#include <algorithm>
#include <condition_variable>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "bd_ctx.cuh"

struct bd_batch {
  std::vector<bd_ctx*> ctx;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_go, cv_done;
  unsigned long t0 = 0;
  int nsteps = 0, with_hop = 0;
  long long generation = 0;
  int pending = 0;
  bool stop = false;
  std::vector<int> status;
  std::vector<std::string> detail;  // bd_last_error_detail of a failing replica's worker
};

static void worker(bd_batch* b, int r) {
  long long seen = 0;
  bd_ctx* c = b->ctx[r];
  cudaSetDevice(c->device);
  for (;;) {
    unsigned long t0;
    int ns, hop;
    {
      std::unique_lock<std::mutex> lk(b->mu);
      b->cv_go.wait(lk, [&] { return b->stop || b->generation != seen; });
      if (b->stop) return;
      seen = b->generation;
      t0 = b->t0;
      ns = b->nsteps;
      hop = b->with_hop;
    }
    int s = bd_step_lanczos(c, t0, ns, hop);
    {
      std::lock_guard<std::mutex> lk(b->mu);
      b->status[r] = s;
      b->detail[r] = s == BD_ERR_CUDA ? bd_last_error_detail() : "";
      if (--b->pending == 0) b->cv_done.notify_all();
    }
  }
}

extern "C" {

int bd_batch_create(bd_ctx* const* ctxs, int n, bd_batch** out) {
  if (!ctxs || n <= 0 || !out) return BD_ERR_ARG;
  for (int r = 0; r < n; r++)
    if (!ctxs[r]) return BD_ERR_ARG;
  bd_batch* b = new bd_batch();
  b->ctx.assign(ctxs, ctxs + n);
  b->status.assign(n, BD_OK);
  b->detail.assign(n, "");
  for (int r = 0; r < n; r++) b->workers.emplace_back(worker, b, r);
  *out = b;
  return BD_OK;
}

int bd_batch_step_lanczos(bd_batch* b, unsigned long t0, int nsteps, int with_hop) {
  if (!b || nsteps < 0) return BD_ERR_ARG;
  {
    std::lock_guard<std::mutex> lk(b->mu);
    b->t0 = t0;
    b->nsteps = nsteps;
    b->with_hop = with_hop;
    b->pending = (int)b->ctx.size();
    b->generation++;
  }
  b->cv_go.notify_all();
  std::unique_lock<std::mutex> lk(b->mu);
  b->cv_done.wait(lk, [&] { return b->pending == 0; });
  for (size_t r = 0; r < b->status.size(); r++)
    if (b->status[r] != BD_OK) {
      // the failing replica's call site, readable from this thread
      if (b->status[r] == BD_ERR_CUDA)
        bd::set_error_detail(("replica " + std::to_string(r) + ": " + b->detail[r]).c_str());
      return b->status[r];
    }
  return BD_OK;
}

int bd_batch_destroy(bd_batch* b) {
  if (!b) return BD_OK;
  {
    std::lock_guard<std::mutex> lk(b->mu);
    b->stop = true;
  }
  b->cv_go.notify_all();
  for (auto& t : b->workers) t.join();
  delete b;
  return BD_OK;
}

int bd_autotune_pme_grid(double L, int precision, int* K_out) {
  if (!(L > 0) || !K_out || precision < 0 || precision > 1) return BD_ERR_ARG;
  static std::mutex mu;
  static std::map<std::pair<int, int>, float> cache;  // (K, precision) -> ms
  int K0 = (int)ceil(1.29 * L), K1 = (int)ceil(1.25 * K0);
  std::vector<int> cand;
  for (int K = K0; K <= std::max(K1, K0); K++) {
    int r = K;
    for (int f : {2, 3, 5})
      while (r % f == 0) r /= f;
    if (r == 1) cand.push_back(K);
  }
  if (cand.empty()) return BD_ERR_ARG;
  if (cand.back() > 1024) return BD_ERR_ARG;
  std::lock_guard<std::mutex> lk(mu);
  int best = cand[0];
  float best_ms = 1e30f;
  for (int K : cand) {
    auto key = std::make_pair(K, precision);
    auto it = cache.find(key);
    float ms;
    if (it != cache.end()) {
      ms = it->second;
    } else {
      size_t K3 = (size_t)K * K * K, Ks = (size_t)K * K * (K / 2 + 1);
      size_t es = precision ? 4 : 8;
      void *grid = nullptr, *spec = nullptr;
      if (cudaMalloc(&grid, es * 3 * K3) != cudaSuccess) return BD_ERR_OOM;
      if (cudaMalloc(&spec, 2 * es * 3 * Ks) != cudaSuccess) {
        cudaFree(grid);
        return BD_ERR_OOM;
      }
      cudaMemset(grid, 0, es * 3 * K3);
      int dims[3] = {K, K, K};
      cufftHandle f = 0, bk = 0;
      bool okf = cufftPlanMany(&f, 3, dims, nullptr, 1, (int)K3, nullptr, 1, (int)Ks,
                               precision ? CUFFT_R2C : CUFFT_D2Z, 3) == CUFFT_SUCCESS;
      bool okb = okf && cufftPlanMany(&bk, 3, dims, nullptr, 1, (int)Ks, nullptr, 1, (int)K3,
                                      precision ? CUFFT_C2R : CUFFT_Z2D, 3) == CUFFT_SUCCESS;
      if (okf && !okb) cufftDestroy(f);
      bool ok = okf && okb;
      cudaEvent_t e0, e1;
      cudaEventCreate(&e0);
      cudaEventCreate(&e1);
      ms = 1e30f;
      if (ok) {
        for (int rep = 0; rep < 8; rep++) {
          if (rep == 3) cudaEventRecord(e0, 0);
          if (precision) {
            cufftExecR2C(f, (cufftReal*)grid, (cufftComplex*)spec);
            cufftExecC2R(bk, (cufftComplex*)spec, (cufftReal*)grid);
          } else {
            cufftExecD2Z(f, (cufftDoubleReal*)grid, (cufftDoubleComplex*)spec);
            cufftExecZ2D(bk, (cufftDoubleComplex*)spec, (cufftDoubleReal*)grid);
          }
        }
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        ms /= 5;
        cufftDestroy(f);
        cufftDestroy(bk);
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      cudaFree(grid);
      cudaFree(spec);
      if (cudaGetLastError() != cudaSuccess) return BD_ERR_CUDA;
      cache[key] = ms;
    }
    if (ms < best_ms) {
      best_ms = ms;
      best = K;
    }
  }
  *K_out = best;
  return BD_OK;
}

}  // extern "C"
