// Serving loop: continuous batching of arriving solves of uneven sizes.
//
// Requests (A_i X_i = B_i, host buffers) are queued by lm_server_submit and
// admitted as soon as an execution slot and enough of the device arena are
// free; their work overlaps on the device:
//   small requests (n <= small_max_n, nrhs <= 16) go to the device-resident
//     request loop (device_loop): a persistent kernel whose CTAs each claim
//     the next request posted into a ring in device memory, solve it and
//     publish its completion into pinned host memory, so a request starts as
//     soon as its data has arrived; or, with device_loop off, they are
//     gathered into micro-batches: whenever a batch lane is idle it takes
//     every queued small request that fits and runs them as ONE launch of the
//     persistent batch kernel (batch.cu) on its own stream;
//   larger requests each take a worker (own context, stream and pre-grown
//     workspace) and are solved at a padded bucket order, so that the worker
//     replays captured CUDA graphs for orders it has not seen: FP64 LU or
//     Cholesky up to lu_fp64_max_n / chol_fp64_max_n (where the factorisation
//     is bound by its column chain, the same in either precision, and FP64
//     needs no refinement), above that mixed-precision LU with FP64
//     refinement (lm_dgesv_ir) for general and SPD requests alike, then FP64
//     LU (general) or FP64 Cholesky (SPD) when refinement does not converge
//     or the FP32 factor breaks down.
// Admission by HBM footprint: every admitted request holds one block of a
// device arena (its A, B, X, factor and pivots); a request is admitted only
// when its block can be carved from the free space (first fit, coalescing on
// release), and one whose block exceeds the whole arena is rejected at
// submission.  Large requests are admitted in arrival order among themselves;
// small ones never wait behind a large one that does not fit.
// Latency = completion time (X written to the caller's host buffer) minus
// submission time, host steady clock; p50 / p99 over completed requests.
//
// Failure handling is host-side: a request that fails (bad pivot, CUDA error)
// completes with its status; cancel removes a request that is still queued;
// destroy drains admitted work and cancels the rest.  No device-side waits.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

constexpr size_t kAlign = 256;
size_t rup(size_t a) { return (a + kAlign - 1) / kAlign * kAlign; }

// Order a large request is solved at: n rounded up to a multiple of 64 (up to
// 1024), 128 (up to 2048) or 256.  Requests of every order in one of these
// buckets run the same launch sequence on the same worker buffers, so their
// captured CUDA graphs are replayed instead of re-launching every kernel:
// with orders drawn from a continuum almost every request would otherwise be
// a shape never seen before.  At most 6% extra order (from 1024 up; 1024 / n
// below it, where the solves are short).
int padded_order(int n) {
  const int q = n <= 1024 ? 64 : n <= 2048 ? 128 : 256;
  return (n + q - 1) / q * q;
}

// Diagonal of the padding: the system is embedded as [[A, 0], [0, c I]] with
// B padded by zero rows, so the padded unknowns are exactly zero and the first
// n rows of the solution are A's.  c = max_i |a_ii| (1 if that is 0): never
// above ||A||_inf, so ||A_p||_inf = ||A||_inf and the refinement's stopping
// test is the original one, and on A's own scale, so the padded system is no
// worse conditioned than A even when the randomised method mixes the padding
// rows into it.
__global__ void pad_diag_kernel(const double* A, int n, double* c) {
  double m = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, fabs(A[(long long)i * n + i]));
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (int)(blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) *c = (m > 0.0 && m == m) ? m : 1.0;
  }
}

__global__ void embed_kernel(double* Ap, int np, const double* A, int n, const double* c) {
  const long long total = (long long)np * np;
  const double cd = *c;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e / np), j = (int)(e % np);
    Ap[e] = (i < n && j < n) ? A[(long long)i * n + j] : (i == j ? cd : 0.0);
  }
}

// First-fit sub-allocator over one device allocation.
struct Arena {
  char* base = nullptr;
  size_t size = 0, in_use = 0, peak = 0;
  std::map<size_t, size_t> free_;  // offset -> length
  void init(char* b, size_t s) {
    base = b;
    size = s;
    free_.clear();
    free_[0] = s;
  }
  bool alloc(size_t bytes, size_t* off) {
    bytes = rup(bytes);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        *off = it->first;
        const size_t rest = it->second - bytes;
        const size_t noff = it->first + bytes;
        free_.erase(it);
        if (rest) free_[noff] = rest;
        in_use += bytes;
        peak = std::max(peak, in_use);
        return true;
      }
    }
    return false;
  }
  void release(size_t off, size_t bytes) {
    bytes = rup(bytes);
    in_use -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
};

struct Req {
  long long id = 0;
  int n = 0, nrhs = 0, kind = 0;
  const double* A = nullptr;
  const double* B = nullptr;
  double* X = nullptr;
  bool small = false;
  double t_submit = 0, t_admit = 0, t_done = 0;
  // arena block: [A n*n][B n*r][X n*r][F n*n (small only)][ipiv n ints]
  size_t off = 0, bytes = 0, oA = 0, oB = 0, oX = 0, oF = 0, oP = 0;
  int status = 0, iters = 0;
  int ir_method = -1;  // method of a large mixed-precision solve (LM_IR_*), -1 if none
  bool fallback = false, done = false, cancelled = false;
};

size_t layout(Req& r) {
  const size_t nn = (size_t)r.n * r.n * 8, nr = (size_t)r.n * r.nrhs * 8;
  r.oA = 0;
  r.oB = rup(r.oA + nn);
  r.oX = rup(r.oB + nr);
  r.oF = rup(r.oX + nr);
  r.oP = rup(r.oF + (r.small ? nn : 0));
  return rup(r.oP + (size_t)r.n * 4);
}

}  // namespace

struct lm_server;

namespace {

struct Lane {
  lm_server* s = nullptr;
  int idx = 0;
  std::thread th;
  cudaStream_t st = nullptr;
  lm::BatchItem* d_items = nullptr;
  lm::BatchItem* h_items = nullptr;
  int *d_info = nullptr, *d_iters = nullptr, *d_ticket = nullptr;
  double* d_berr = nullptr;
  int *h_info = nullptr, *h_iters = nullptr;
  std::vector<Req*> jobs;
  bool busy = false;
  std::condition_variable cv;
  double busy_s = 0;
  long long batches = 0, solved = 0;
};

struct Worker {
  lm_server* s = nullptr;
  std::thread th;
  lm_ctx* ctx = nullptr;
  Req* job = nullptr;
  bool busy = false;
  std::condition_variable cv;
  double busy_s = 0;
  // fixed operands of the mixed-precision solve (max_n x max_n, max_n x
  // max_nrhs): a request of an order this worker has seen before replays the
  // solve's captured CUDA graphs instead of launching every kernel again
  double *Aw = nullptr, *Bw = nullptr, *Xw = nullptr;
  int* Pw = nullptr;       // pivots of the FP64 LU at the bucket order
  double* cpad = nullptr;  // diagonal of the padding block (device)
};

// Device-resident request loop for the small requests: the feeder thread
// copies each admitted request into its arena block and posts its descriptor
// into a ring in device memory, then advances the ring's tail, all on one copy
// stream (so the device sees the data before the tail that announces it); the
// loop kernel (serve_loop_kernel) claims and solves posted requests and writes
// a completion word into pinned host memory, which the poller thread watches
// before it copies X out and completes the request.  The kernel returns after
// a few milliseconds without work; posting or polling relaunches it.
struct DeviceLoop {
  int cap = 0, ctas = 0;
  size_t smem = 0;
  cudaStream_t feed = nullptr, cons = nullptr, d2h = nullptr;
  lm::BatchItem* d_items = nullptr;
  int* d_ctl = nullptr;  // [0] head, [1] tail, [2] stop
  lm::BatchItem* h_items = nullptr;
  int* h_tail = nullptr;   // per slot: the tail value that posts it
  int* h_info = nullptr;   // mapped: written by the loop
  int* h_done = nullptr;   // mapped: seq + 1 once solved
  cudaEvent_t ev_exit = nullptr;
  std::mutex launch_mu;
  bool running = false;    // a launch was made whose end has not been seen
  long long launches = 0, solved = 0;
  int next_seq = 0;
  std::deque<Req*> to_post;          // admitted, waiting for the feeder
  std::vector<Req*> posted;          // slot -> request (nullptr when free)
  std::vector<int> seq_of;           // slot -> sequence number
  int in_ring = 0;
  std::thread feeder, poller;
  std::condition_variable cv_feed, cv_poll;
};

}  // namespace

struct lm_server {
  int device = 0;
  int num_sms = 0;
  lm_server_config cfg{};
  std::mutex mu;
  std::condition_variable cv_done;
  // queued requests, one FIFO per class: dispatch takes from the fronts, so
  // its cost does not grow with the length of the queue
  std::deque<Req*> pend_small, pend_large;
  size_t pending_count() const { return pend_small.size() + pend_large.size(); }
  std::unordered_map<long long, Req*> live;
  Arena arena;
  std::vector<Lane*> lanes;
  std::vector<Worker*> workers;
  DeviceLoop* loop = nullptr;  // small requests on the device-resident loop (cfg.device_loop)
  std::vector<double> lat_ms;
  long long next_id = 1, completed = 0, rejected = 0, cancelled = 0, fallbacks = 0, failed = 0;
  long long ir_solves = 0, ir_gepp = 0, ir_iterations = 0;
  size_t queue_peak = 0;
  int inflight = 0, inflight_peak = 0;
  bool stopping = false;
  double t_first = 0, t_last = 0;
  double flops_done = 0;
  size_t fixed_bytes = 0;  // pre-grown worker workspaces (outside the arena)
};

namespace {

double req_flops(const Req& r) {
  const double n = r.n;
  return (r.kind == LM_BATCH_GENERAL ? 2.0 / 3.0 : 1.0 / 3.0) * n * n * n + 2.0 * n * n * r.nrhs;
}

void complete(lm_server* s, Req* r) {  // under s->mu
  r->t_done = now_s();
  r->done = true;
  s->arena.release(r->off, r->bytes);
  --s->inflight;
  ++s->completed;
  s->t_last = r->t_done;
  s->lat_ms.push_back((r->t_done - r->t_submit) * 1e3);
  if (r->status < 0) ++s->failed;
  if (r->fallback) ++s->fallbacks;
  if (r->ir_method >= 0) {
    ++s->ir_solves;
    if (r->ir_method == LM_IR_GEPP) ++s->ir_gepp;
    if (r->iters > 0) s->ir_iterations += r->iters;
  }
  s->flops_done += req_flops(*r);
}

bool admit(lm_server* s, Req* r) {  // under s->mu
  if (!s->arena.alloc(r->bytes, &r->off)) return false;
  r->t_admit = now_s();
  ++s->inflight;
  s->inflight_peak = std::max(s->inflight_peak, s->inflight);
  return true;
}

// Hand queued requests to idle lanes / workers.  Under s->mu.
void pump(lm_server* s) {
  // small requests on the device-resident loop: admitted in arrival order
  // while the ring has room
  if (s->loop) {
    DeviceLoop* L = s->loop;
    bool any = false;
    while (!s->pend_small.empty()) {
      Req* r = s->pend_small.front();
      if (L->in_ring + (int)L->to_post.size() >= L->cap || !admit(s, r)) break;
      s->pend_small.pop_front();
      L->to_post.push_back(r);
      any = true;
    }
    if (any) L->cv_feed.notify_one();
  }
  // small requests: one micro-batch per idle lane, in arrival order
  for (Lane* ln : s->lanes) {
    if (ln->busy) continue;
    std::vector<Req*> take;
    while (!s->pend_small.empty() && (int)take.size() < s->cfg.max_batch) {
      Req* r = s->pend_small.front();
      if (!admit(s, r)) break;  // arena full: the rest waits for releases
      s->pend_small.pop_front();
      take.push_back(r);
    }
    if (take.empty()) break;
    ln->jobs = std::move(take);
    ln->busy = true;
    ln->cv.notify_one();
  }
  // large requests: arrival order among themselves
  while (!s->pend_large.empty()) {
    Worker* w = nullptr;
    for (Worker* x : s->workers)
      if (!x->busy) {
        w = x;
        break;
      }
    Req* r = s->pend_large.front();
    if (!w || !admit(s, r)) break;
    s->pend_large.pop_front();
    w->job = r;
    w->busy = true;
    w->cv.notify_one();
  }
}

// ---- batch lane: one persistent-kernel launch per micro-batch -------------------------
void lane_run(Lane* ln) {
  lm_server* s = ln->s;
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    ln->cv.wait(lk, [&] { return ln->busy || s->stopping; });
    if (!ln->busy && s->stopping) return;
    std::vector<Req*> jobs = ln->jobs;
    lk.unlock();
    const double t0 = now_s();
    char* base = s->arena.base;
    int nmax = 1, rmax = 1;
    int nbmax = 1;
    int err = LM_OK;
    const int k = (int)jobs.size();
    for (int i = 0; i < k && err == LM_OK; ++i) {
      Req* r = jobs[i];
      char* blk = base + r->off;
      if (cudaMemcpyAsync(blk + r->oA, r->A, (size_t)r->n * r->n * 8, cudaMemcpyHostToDevice, ln->st) != cudaSuccess ||
          cudaMemcpyAsync(blk + r->oB, r->B, (size_t)r->n * r->nrhs * 8, cudaMemcpyHostToDevice, ln->st) !=
              cudaSuccess)
        err = LM_ERR_CUDA;
      lm::BatchItem& it = ln->h_items[i];
      it.a_off = (long long)((r->off + r->oA) / 8);
      it.b_off = (long long)((r->off + r->oB) / 8);
      it.x_off = (long long)((r->off + r->oX) / 8);
      it.f_off = (long long)((r->off + r->oF) / 8);
      it.p_off = (long long)((r->off + r->oP) / 4);
      it.n = r->n;
      it.nrhs = r->nrhs;
      it.kind = r->kind;
      it.nb = s->cfg.nb[lm::batch_bucket(std::max(r->n, 1))];
      it.index = i;
      nmax = std::max(nmax, r->n);
      rmax = std::max(rmax, r->nrhs);
      nbmax = std::max(nbmax, it.nb);
    }
    // largest first within the micro-batch
    std::sort(ln->h_items, ln->h_items + k, [](const lm::BatchItem& a, const lm::BatchItem& b) {
      return (double)a.n * a.n * a.n > (double)b.n * b.n * b.n;
    });
    if (err == LM_OK && cudaMemcpyAsync(ln->d_items, ln->h_items, sizeof(lm::BatchItem) * k, cudaMemcpyHostToDevice,
                                        ln->st) != cudaSuccess)
      err = LM_ERR_CUDA;
    if (err == LM_OK) {
      lm::BatchArgs g;
      g.items = ln->d_items;
      g.count = k;
      g.prec = s->cfg.small_precision;
      g.nmax = nmax;
      g.rmax = rmax;
      g.nbmax = nbmax;
      g.A = reinterpret_cast<const double*>(base);
      g.B = reinterpret_cast<const double*>(base);
      g.X = reinterpret_cast<double*>(base);
      g.F = reinterpret_cast<double*>(base);
      g.ipiv = reinterpret_cast<int*>(base);
      g.info = ln->d_info;
      g.iters = ln->d_iters;
      g.berr = ln->d_berr;
      g.ticket = ln->d_ticket;
      g.tol = 0.0;
      g.max_iter = 10;
      const size_t smem = lm::batch_smem_bytes(nmax, rmax, nbmax);
      int per_sm = 1;
      err = lm::batch_occupancy(smem, &per_sm);
      const int grid = std::max(1, std::min(k, std::max(per_sm, 1) * s->num_sms));
      if (err == LM_OK) err = lm::batch_launch(g, grid, smem, ln->st);
    }
    for (int i = 0; i < k && err == LM_OK; ++i) {
      Req* r = jobs[i];
      if (cudaMemcpyAsync(r->X, base + r->off + r->oX, (size_t)r->n * r->nrhs * 8, cudaMemcpyDeviceToHost, ln->st) !=
          cudaSuccess)
        err = LM_ERR_CUDA;
    }
    if (err == LM_OK) {
      cudaMemcpyAsync(ln->h_info, ln->d_info, sizeof(int) * k, cudaMemcpyDeviceToHost, ln->st);
      cudaMemcpyAsync(ln->h_iters, ln->d_iters, sizeof(int) * k, cudaMemcpyDeviceToHost, ln->st);
      if (cudaStreamSynchronize(ln->st) != cudaSuccess) err = LM_ERR_CUDA;
    }
    lk.lock();
    for (int i = 0; i < k; ++i) {
      Req* r = jobs[i];
      r->status = err != LM_OK ? err : ln->h_info[i];
      r->iters = err != LM_OK ? 0 : ln->h_iters[i];
      r->fallback = err == LM_OK && ln->h_iters[i] < 0;
      complete(s, r);
    }
    ln->busy_s += now_s() - t0;
    ++ln->batches;
    ln->solved += k;
    ln->jobs.clear();
    ln->busy = false;
    pump(s);
    s->cv_done.notify_all();
  }
}

// ---- worker: one larger request at a time on its own context -------------------------
int worker_solve(lm_server* s, Worker* w, Req* r) {
  char* blk = s->arena.base + r->off;
  double* dA = reinterpret_cast<double*>(blk + r->oA);
  double* dB = reinterpret_cast<double*>(blk + r->oB);
  double* dX = reinterpret_cast<double*>(blk + r->oX);
  int* dP = reinterpret_cast<int*>(blk + r->oP);
  cudaStream_t st = static_cast<cudaStream_t>(lm_ctx_get_stream(w->ctx));
  const size_t nn = (size_t)r->n * r->n * 8, nr = (size_t)r->n * r->nrhs * 8;
  LM_CUDA_TRY(cudaMemcpyAsync(dA, r->A, nn, cudaMemcpyHostToDevice, st));
  LM_CUDA_TRY(cudaMemcpyAsync(dB, r->B, nr, cudaMemcpyHostToDevice, st));
  const bool general = r->kind == LM_BATCH_GENERAL;
  // Both methods run at the bucket order in the worker's fixed buffers, so a
  // request of an order this worker has served before replays captured graphs.
  const int np = padded_order(r->n);
  const long long tot = (long long)np * np;
  pad_diag_kernel<<<1, 256, 0, st>>>(dA, r->n, w->cpad);
  embed_kernel<<<(int)std::min<long long>((tot + 255) / 256, 4096), 256, 0, st>>>(w->Aw, np, dA, r->n, w->cpad);
  lm::count_launch(2);
  LM_CUDA_TRY(cudaGetLastError());
  LM_CUDA_TRY(cudaMemcpyAsync(w->Bw, dB, nr, cudaMemcpyDeviceToDevice, st));
  if (np > r->n)
    LM_CUDA_TRY(cudaMemsetAsync(w->Bw + (size_t)r->n * r->nrhs, 0, sizeof(double) * (size_t)(np - r->n) * r->nrhs, st));
  int info = 0, rc = LM_OK;
  const bool ir = s->cfg.large_precision == LM_PREC_FP32_IR &&
                  r->n > (general ? s->cfg.lu_fp64_max_n : s->cfg.chol_fp64_max_n);
  if (!ir) {
    // FP64 LU or Cholesky of the embedded system, solved in place in Bw: the
    // padding block is decoupled, so the first n rows are A's solution
    rc = general ? lm_dgesv(w->ctx, np, r->nrhs, w->Aw, np, w->Pw, w->Bw, r->nrhs, &info)
                 : lm_dposv(w->ctx, np, r->nrhs, w->Aw, np, w->Bw, r->nrhs, &info);
    if (rc < 0) return rc;
    r->iters = 0;
    LM_CUDA_TRY(cudaMemcpyAsync(r->X, w->Bw, nr, cudaMemcpyDeviceToHost, st));
    LM_CUDA_TRY(cudaStreamSynchronize(st));
    return info;
  }
  int it = 0;
  double be = 0;
  // the stopping test of the original order: 1e-15 n
  rc = lm_dgesv_ir(w->ctx, np, r->nrhs, w->Aw, np, w->Bw, r->nrhs, w->Xw, r->nrhs, 1e-15 * r->n, 30, &it, &be, &info);
  lm_ctx_ir_last_method(w->ctx, &r->ir_method);
  if (rc == LM_OK) {
    r->iters = it;
    LM_CUDA_TRY(cudaMemcpyAsync(r->X, w->Xw, nr, cudaMemcpyDeviceToHost, st));
    LM_CUDA_TRY(cudaStreamSynchronize(st));
    return LM_OK;
  }
  if (rc != LM_ERR_NOT_CONVERGED && rc <= 0) return rc;
  // refinement did not converge (or the FP32 factor broke down): FP64 at the
  // request's own order from the untouched arena copy
  r->fallback = true;
  r->iters = -1;
  LM_CUDA_TRY(cudaMemcpyAsync(dX, dB, nr, cudaMemcpyDeviceToDevice, st));
  rc = general ? lm_dgesv(w->ctx, r->n, r->nrhs, dA, r->n, dP, dX, r->nrhs, &info)
               : lm_dposv(w->ctx, r->n, r->nrhs, dA, r->n, dX, r->nrhs, &info);
  if (rc < 0) return rc;
  LM_CUDA_TRY(cudaMemcpyAsync(r->X, dX, nr, cudaMemcpyDeviceToHost, st));
  LM_CUDA_TRY(cudaStreamSynchronize(st));
  return info;
}

void worker_run(Worker* w) {
  lm_server* s = w->s;
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    w->cv.wait(lk, [&] { return w->busy || s->stopping; });
    if (!w->busy && s->stopping) return;
    Req* r = w->job;
    lk.unlock();
    const double t0 = now_s();
    const int st = worker_solve(s, w, r);
    lk.lock();
    r->status = st;
    complete(s, r);
    w->busy_s += now_s() - t0;
    w->job = nullptr;
    w->busy = false;
    pump(s);
    s->cv_done.notify_all();
  }
}

lm::BatchArgs loop_args(lm_server* s) {
  char* base = s->arena.base;
  lm::BatchArgs g{};
  g.items = nullptr;
  g.count = 0;
  g.prec = LM_PREC_FP64;
  g.nmax = std::max(1, s->cfg.small_max_n);
  g.rmax = 16;
  g.nbmax = 32;
  g.A = reinterpret_cast<const double*>(base);
  g.B = reinterpret_cast<const double*>(base);
  g.X = reinterpret_cast<double*>(base);
  g.F = reinterpret_cast<double*>(base);
  g.ipiv = reinterpret_cast<int*>(base);
  g.tol = 0.0;
  g.max_iter = 0;
  return g;
}

// (Re)launch the loop kernel unless a launch is still running.
int loop_ensure_running(lm_server* s) {
  DeviceLoop* L = s->loop;
  std::lock_guard<std::mutex> lk(L->launch_mu);
  if (L->running) {
    const cudaError_t q = cudaEventQuery(L->ev_exit);
    if (q == cudaErrorNotReady) return LM_OK;
    if (q != cudaSuccess) return LM_ERR_CUDA;
    L->running = false;
  }
  lm::ServeRing rg;
  rg.items = L->d_items;
  rg.cap = L->cap;
  rg.head = L->d_ctl;
  rg.tail = L->d_ctl + 1;
  rg.stop = L->d_ctl + 2;
  rg.h_info = L->h_info;
  rg.h_done = L->h_done;
  LM_TRY(lm::serve_loop_launch(loop_args(s), rg, L->ctas, L->smem, L->cons));
  LM_CUDA_TRY(cudaEventRecord(L->ev_exit, L->cons));
  L->running = true;
  ++L->launches;
  return LM_OK;
}

void loop_feeder(lm_server* s) {
  DeviceLoop* L = s->loop;
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    L->cv_feed.wait(lk, [&] { return !L->to_post.empty() || s->stopping; });
    if (L->to_post.empty() && s->stopping) return;
    std::vector<Req*> batch(L->to_post.begin(), L->to_post.end());
    L->to_post.clear();
    // slots: the next free sequence numbers (the ring has room: pump checked)
    std::vector<int> slots;
    for (Req* r : batch) {
      const int sq = L->next_seq++;
      const int idx = sq % L->cap;
      L->posted[idx] = r;
      L->seq_of[idx] = sq;
      L->h_done[idx] = 0;
      ++L->in_ring;
      slots.push_back(sq);
    }
    lk.unlock();
    char* base = s->arena.base;
    int err = LM_OK;
    for (size_t i = 0; i < batch.size() && err == LM_OK; ++i) {
      Req* r = batch[i];
      const int sq = slots[i], idx = sq % L->cap;
      char* blk = base + r->off;
      lm::BatchItem& it = L->h_items[idx];
      it.a_off = (long long)((r->off + r->oA) / 8);
      it.b_off = (long long)((r->off + r->oB) / 8);
      it.x_off = (long long)((r->off + r->oX) / 8);
      it.f_off = (long long)((r->off + r->oF) / 8);
      it.p_off = (long long)((r->off + r->oP) / 4);
      it.n = r->n;
      it.nrhs = r->nrhs;
      it.kind = r->kind;
      it.nb = s->cfg.nb[lm::batch_bucket(std::max(r->n, 1))];
      it.index = idx;
      L->h_tail[idx] = sq + 1;
      if (cudaMemcpyAsync(blk + r->oA, r->A, (size_t)r->n * r->n * 8, cudaMemcpyHostToDevice, L->feed) != cudaSuccess ||
          cudaMemcpyAsync(blk + r->oB, r->B, (size_t)r->n * r->nrhs * 8, cudaMemcpyHostToDevice, L->feed) !=
              cudaSuccess ||
          cudaMemcpyAsync(L->d_items + idx, &it, sizeof it, cudaMemcpyHostToDevice, L->feed) != cudaSuccess ||
          cudaMemcpyAsync(L->d_ctl + 1, L->h_tail + idx, sizeof(int), cudaMemcpyHostToDevice, L->feed) != cudaSuccess)
        err = LM_ERR_CUDA;
    }
    if (err == LM_OK) err = loop_ensure_running(s);
    lk.lock();
    if (err != LM_OK) {
      // nothing of this batch is in the ring as far as the host is concerned
      for (size_t i = 0; i < batch.size(); ++i) {
        const int idx = slots[i] % L->cap;
        L->posted[idx] = nullptr;
        --L->in_ring;
        batch[i]->status = err;
        complete(s, batch[i]);
      }
      s->cv_done.notify_all();
    }
    L->cv_poll.notify_one();
  }
}

void loop_poller(lm_server* s) {
  DeviceLoop* L = s->loop;
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    L->cv_poll.wait_for(lk, std::chrono::microseconds(200), [&] { return L->in_ring > 0 || s->stopping; });
    if (L->in_ring == 0) {
      if (s->stopping) return;
      continue;
    }
    // requests whose completion word is set
    std::vector<std::pair<Req*, int>> done;
    for (int idx = 0; idx < L->cap && (int)done.size() < L->in_ring; ++idx) {
      Req* r = L->posted[idx];
      if (r && *reinterpret_cast<volatile int*>(L->h_done + idx) == L->seq_of[idx] + 1) done.push_back({r, idx});
    }
    if (done.empty()) {
      lk.unlock();
      loop_ensure_running(s);  // a launch that ran out of idle polls before the post
      std::this_thread::sleep_for(std::chrono::microseconds(20));
      lk.lock();
      continue;
    }
    lk.unlock();
    int err = LM_OK;
    char* base = s->arena.base;
    for (auto& d : done) {
      Req* r = d.first;
      if (cudaMemcpyAsync(r->X, base + r->off + r->oX, (size_t)r->n * r->nrhs * 8, cudaMemcpyDeviceToHost, L->d2h) !=
          cudaSuccess)
        err = LM_ERR_CUDA;
    }
    if (cudaStreamSynchronize(L->d2h) != cudaSuccess) err = LM_ERR_CUDA;
    lk.lock();
    for (auto& d : done) {
      Req* r = d.first;
      L->posted[d.second] = nullptr;
      --L->in_ring;
      r->status = err != LM_OK ? err : L->h_info[d.second];
      r->iters = 0;
      ++L->solved;
      complete(s, r);
    }
    pump(s);
    s->cv_done.notify_all();
  }
}

void server_stop(lm_server* s) {
  {
    std::unique_lock<std::mutex> lk(s->mu);
    // queued requests that never started are cancelled; admitted ones finish
    for (std::deque<Req*>* q : {&s->pend_small, &s->pend_large}) {
      for (Req* r : *q) {
        r->cancelled = true;
        r->done = true;
        r->status = LM_ERR_ARG;
        ++s->cancelled;
      }
      q->clear();
    }
    s->cv_done.wait(lk, [&] { return s->inflight == 0; });
    s->stopping = true;
    for (Lane* ln : s->lanes) ln->cv.notify_all();
    for (Worker* w : s->workers) w->cv.notify_all();
    if (s->loop) {
      s->loop->cv_feed.notify_all();
      s->loop->cv_poll.notify_all();
    }
  }
  if (s->loop) {
    DeviceLoop* L = s->loop;
    if (L->feeder.joinable()) L->feeder.join();
    if (L->poller.joinable()) L->poller.join();
    if (L->d_ctl) {
      const int one = 1;  // end a running loop at once
      cudaMemcpy(L->d_ctl + 2, &one, sizeof one, cudaMemcpyHostToDevice);
      if (L->cons) cudaStreamSynchronize(L->cons);
    }
  }
  for (Lane* ln : s->lanes)
    if (ln->th.joinable()) ln->th.join();
  for (Worker* w : s->workers)
    if (w->th.joinable()) w->th.join();
}

void server_free(lm_server* s) {
  for (Lane* ln : s->lanes) {
    cudaFree(ln->d_items);
    cudaFree(ln->d_info);
    cudaFree(ln->d_iters);
    cudaFree(ln->d_berr);
    cudaFree(ln->d_ticket);
    cudaFreeHost(ln->h_items);
    cudaFreeHost(ln->h_info);
    cudaFreeHost(ln->h_iters);
    if (ln->st) cudaStreamDestroy(ln->st);
    delete ln;
  }
  if (DeviceLoop* L = s->loop) {
    cudaFree(L->d_items);
    cudaFree(L->d_ctl);
    cudaFreeHost(L->h_items);
    cudaFreeHost(L->h_tail);
    cudaFreeHost(L->h_info);
    cudaFreeHost(L->h_done);
    if (L->ev_exit) cudaEventDestroy(L->ev_exit);
    for (cudaStream_t x : {L->feed, L->cons, L->d2h})
      if (x) cudaStreamDestroy(x);
    delete L;
  }
  for (Worker* w : s->workers) {
    if (w->ctx) lm_ctx_destroy(w->ctx);
    cudaFree(w->Aw);
    cudaFree(w->Bw);
    cudaFree(w->Xw);
    cudaFree(w->Pw);
    cudaFree(w->cpad);
    delete w;
  }
  cudaFree(s->arena.base);
  for (auto& kv : s->live) delete kv.second;
  delete s;
}

// Grow a worker context's workspaces to the largest admissible request with
// one solve of each kind (SPD diagonal matrix, so every path succeeds).
int prewarm(lm_server* s, Worker* w) {
  const int n = padded_order(s->cfg.max_n), r = s->cfg.max_nrhs;
  double *A = nullptr, *B = nullptr, *X = nullptr;
  int* P = nullptr;
  const size_t nn = (size_t)n * n * 8, nr = (size_t)n * r * 8;
  LM_CUDA_TRY(cudaMalloc(&A, nn));
  LM_CUDA_TRY(cudaMalloc(&B, nr));
  LM_CUDA_TRY(cudaMalloc(&X, nr));
  LM_CUDA_TRY(cudaMalloc(&P, (size_t)n * 4));
  std::vector<double> h((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) h[(size_t)i * n + i] = 1.0 + i % 7;
  int rc = LM_OK;
  if (cudaMemcpy(A, h.data(), nn, cudaMemcpyHostToDevice) != cudaSuccess || cudaMemset(B, 0, nr) != cudaSuccess)
    rc = LM_ERR_CUDA;
  int it = 0, info = 0;
  double be = 0;
  if (rc == LM_OK && s->cfg.large_precision == LM_PREC_FP32_IR) {
    // both substitution paths: few right-hand sides and many
    for (int rr : {1, r}) {
      rc = lm_dgesv_ir(w->ctx, n, rr, A, n, B, rr, X, rr, 0.0, 30, &it, &be, &info);
      if (rc > 0 || rc == LM_ERR_NOT_CONVERGED) rc = LM_OK;
      if (rc != LM_OK) break;
    }
  }
  if (rc == LM_OK) rc = lm_dgesv(w->ctx, n, r, A, n, P, X, r, &info);
  if (rc == LM_OK) {
    cudaMemcpy(A, h.data(), nn, cudaMemcpyHostToDevice);
    rc = lm_dposv(w->ctx, n, r, A, n, X, r, &info);
  }
  if (rc > 0) rc = LM_OK;
  cudaFree(A);
  cudaFree(B);
  cudaFree(X);
  cudaFree(P);
  return rc;
}

int server_init(lm_server* s) {
  LM_CUDA_TRY(cudaSetDevice(s->device));
  LM_CUDA_TRY(cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, s->device));
  size_t free_b = 0, total_b = 0;
  LM_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
  // workers first (their pre-grown workspaces are fixed overhead)
  for (int i = 0; i < s->cfg.large_workers; ++i) {
    Worker* w = new Worker;
    w->s = s;
    s->workers.push_back(w);
    LM_TRY(lm_ctx_create(&w->ctx, s->device));
    lm::ctx_set_graph_cache(w->ctx, 1024);
    LM_TRY(lm_ctx_set_ir_method(w->ctx, s->cfg.ir_method));
    const size_t np = (size_t)padded_order(s->cfg.max_n);
    const size_t nn = np * np, nr = np * s->cfg.max_nrhs;
    LM_CUDA_TRY(cudaMalloc(&w->Aw, sizeof(double) * nn));
    LM_CUDA_TRY(cudaMalloc(&w->Bw, sizeof(double) * nr));
    LM_CUDA_TRY(cudaMalloc(&w->Xw, sizeof(double) * nr));
    LM_CUDA_TRY(cudaMalloc(&w->Pw, sizeof(int) * np));
    LM_CUDA_TRY(cudaMalloc(&w->cpad, 256));
    LM_TRY(prewarm(s, w));
  }
  size_t free_after = 0;
  LM_CUDA_TRY(cudaMemGetInfo(&free_after, &total_b));
  s->fixed_bytes = free_b > free_after ? free_b - free_after : 0;
  size_t budget = s->cfg.hbm_budget;
  if (budget == 0) budget = free_after / 4;
  budget = rup(budget);
  char* base = nullptr;
  if (cudaMalloc(&base, budget) != cudaSuccess) {
    cudaGetLastError();
    lm::set_last_error("server: arena allocation failed");
    return LM_ERR_NOMEM;
  }
  s->arena.init(base, budget);
  const int mb = s->cfg.max_batch;
  for (int i = 0; i < s->cfg.batch_lanes; ++i) {
    Lane* ln = new Lane;
    ln->s = s;
    ln->idx = i;
    s->lanes.push_back(ln);
    LM_CUDA_TRY(cudaStreamCreateWithFlags(&ln->st, cudaStreamNonBlocking));
    LM_CUDA_TRY(cudaMalloc(&ln->d_items, sizeof(lm::BatchItem) * mb));
    LM_CUDA_TRY(cudaMalloc(&ln->d_info, sizeof(int) * mb));
    LM_CUDA_TRY(cudaMalloc(&ln->d_iters, sizeof(int) * mb));
    LM_CUDA_TRY(cudaMalloc(&ln->d_berr, sizeof(double) * mb));
    LM_CUDA_TRY(cudaMalloc(&ln->d_ticket, sizeof(int) * 4));
    LM_CUDA_TRY(cudaMallocHost(&ln->h_items, sizeof(lm::BatchItem) * mb));
    LM_CUDA_TRY(cudaMallocHost(&ln->h_info, sizeof(int) * mb));
    LM_CUDA_TRY(cudaMallocHost(&ln->h_iters, sizeof(int) * mb));
  }
  // the batch kernel's shared-memory limit for the largest micro-batch shape
  int per_sm = 0;
  LM_TRY(lm::batch_occupancy(lm::batch_smem_bytes(s->cfg.small_max_n, 16, 32), &per_sm));
  if (s->cfg.device_loop) {
    DeviceLoop* L = new DeviceLoop;
    s->loop = L;
    L->cap = 8192;
    L->ctas = std::max(1, std::min(s->cfg.loop_ctas, s->num_sms));
    L->smem = lm::batch_smem_bytes(std::max(1, s->cfg.small_max_n), 16, 32);
    L->posted.assign(L->cap, nullptr);
    L->seq_of.assign(L->cap, -1);
    LM_CUDA_TRY(cudaStreamCreateWithFlags(&L->feed, cudaStreamNonBlocking));
    LM_CUDA_TRY(cudaStreamCreateWithFlags(&L->cons, cudaStreamNonBlocking));
    LM_CUDA_TRY(cudaStreamCreateWithFlags(&L->d2h, cudaStreamNonBlocking));
    LM_CUDA_TRY(cudaEventCreateWithFlags(&L->ev_exit, cudaEventDisableTiming));
    LM_CUDA_TRY(cudaMalloc(&L->d_items, sizeof(lm::BatchItem) * L->cap));
    LM_CUDA_TRY(cudaMalloc(&L->d_ctl, sizeof(int) * 4));
    LM_CUDA_TRY(cudaMemset(L->d_ctl, 0, sizeof(int) * 4));
    LM_CUDA_TRY(cudaMallocHost(&L->h_items, sizeof(lm::BatchItem) * L->cap));
    LM_CUDA_TRY(cudaMallocHost(&L->h_tail, sizeof(int) * L->cap));
    LM_CUDA_TRY(cudaHostAlloc(&L->h_info, sizeof(int) * L->cap, cudaHostAllocMapped));
    LM_CUDA_TRY(cudaHostAlloc(&L->h_done, sizeof(int) * L->cap, cudaHostAllocMapped));
    std::memset(L->h_done, 0, sizeof(int) * L->cap);
    L->feeder = std::thread(loop_feeder, s);
    L->poller = std::thread(loop_poller, s);
  }
  for (Lane* ln : s->lanes) ln->th = std::thread(lane_run, ln);
  for (Worker* w : s->workers) w->th = std::thread(worker_run, w);
  return LM_OK;
}

}  // namespace

extern "C" {

int lm_server_default_config(lm_server_config* c) {
  if (!c) return LM_ERR_ARG;
  std::memset(c, 0, sizeof(*c));
  c->hbm_budget = 0;
  c->large_workers = 8;
  c->batch_lanes = 2;
  c->small_max_n = 256;
  c->small_precision = LM_PREC_FP64;
  c->large_precision = LM_PREC_FP32_IR;
  c->max_batch = 4096;
  c->max_n = 4096;
  c->max_nrhs = 64;
  for (int b = 0; b < 4; ++b) c->nb[b] = 16;
  c->ir_method = LM_IR_GEPP;
  c->device_loop = 1;
  c->loop_ctas = 16;
  c->lu_fp64_max_n = 2048;
  c->chol_fp64_max_n = 4096;
  return LM_OK;
}

int lm_server_create(lm_server** out, int device, const lm_server_config* cfg) {
  if (!out) return LM_ERR_ARG;
  *out = nullptr;
  lm_server_config c;
  if (cfg) {
    c = *cfg;
  } else {
    lm_server_default_config(&c);
  }
  if (c.large_workers < 1 || c.large_workers > 32 || c.batch_lanes < 1 || c.batch_lanes > 8 || c.small_max_n < 0 ||
      c.small_max_n > lm::BatchLimits::kMaxN || c.max_batch < 1 || c.max_n < 1 || c.max_nrhs < 1 ||
      c.max_nrhs > 64 || (c.small_precision != LM_PREC_FP64 && c.small_precision != LM_PREC_FP32_IR) ||
      (c.large_precision != LM_PREC_FP64 && c.large_precision != LM_PREC_FP32_IR) ||
      (c.ir_method != LM_IR_RBT && c.ir_method != LM_IR_GEPP) || (c.device_loop && c.loop_ctas < 1) ||
      (c.device_loop && c.small_precision != LM_PREC_FP64) || c.lu_fp64_max_n < 0 || c.chol_fp64_max_n < 0)
    return LM_ERR_ARG;
  for (int b = 0; b < 4; ++b)
    if (c.nb[b] != 8 && c.nb[b] != 16 && c.nb[b] != 32) return LM_ERR_ARG;
  lm_server* s = new lm_server;
  s->device = device;
  s->cfg = c;
  const int r = server_init(s);
  if (r != LM_OK) {
    server_stop(s);
    server_free(s);
    return r;
  }
  *out = s;
  return LM_OK;
}

int lm_server_submit(lm_server* s, int n, int nrhs, int kind, const double* A, const double* B, double* X,
                     long long* id) {
  if (!s || !id) return LM_ERR_ARG;
  *id = 0;
  if (n < 1 || nrhs < 1 || !A || !B || !X || (kind != LM_BATCH_GENERAL && kind != LM_BATCH_SPD) ||
      n > s->cfg.max_n || nrhs > s->cfg.max_nrhs) {
    std::lock_guard<std::mutex> lk(s->mu);
    ++s->rejected;
    lm::set_last_error("server: request outside the admissible sizes");
    return LM_ERR_ARG;
  }
  Req* r = new Req;
  r->n = n;
  r->nrhs = nrhs;
  r->kind = kind;
  r->A = A;
  r->B = B;
  r->X = X;
  r->small = n <= s->cfg.small_max_n && nrhs <= lm::BatchLimits::kMaxRhs;
  r->bytes = layout(*r);
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stopping) {
    delete r;
    return LM_ERR_ARG;
  }
  if (rup(r->bytes) > s->arena.size) {
    ++s->rejected;
    delete r;
    lm::set_last_error("server: request larger than the whole HBM budget");
    return LM_ERR_NOMEM;
  }
  r->id = s->next_id++;
  r->t_submit = now_s();
  if (s->t_first == 0) s->t_first = r->t_submit;
  s->live[r->id] = r;
  (r->small ? s->pend_small : s->pend_large).push_back(r);
  s->queue_peak = std::max(s->queue_peak, s->pending_count());
  pump(s);
  *id = r->id;
  return LM_OK;
}

int lm_server_test(lm_server* s, long long id, int* done, int* status, double* latency_ms) {
  if (!s || !done) return LM_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->live.find(id);
  if (it == s->live.end()) return LM_ERR_ARG;
  Req* r = it->second;
  *done = r->done ? 1 : 0;
  if (r->done) {
    if (status) *status = r->status;
    if (latency_ms) *latency_ms = r->cancelled ? 0.0 : (r->t_done - r->t_submit) * 1e3;
    s->live.erase(it);
    delete r;
  }
  return LM_OK;
}

int lm_server_wait(lm_server* s, long long id, int* status, double* latency_ms, double timeout_s) {
  if (!s) return LM_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->live.find(id);
  if (it == s->live.end()) return LM_ERR_ARG;
  Req* r = it->second;
  const auto pred = [&] { return r->done; };
  if (timeout_s > 0) {
    if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred)) return LM_ERR_TIMEOUT;
  } else {
    s->cv_done.wait(lk, pred);
  }
  if (status) *status = r->status;
  if (latency_ms) *latency_ms = r->cancelled ? 0.0 : (r->t_done - r->t_submit) * 1e3;
  s->live.erase(id);
  delete r;
  return LM_OK;
}

int lm_server_cancel(lm_server* s, long long id) {
  if (!s) return LM_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->live.find(id);
  if (it == s->live.end()) return LM_ERR_ARG;
  Req* r = it->second;
  std::deque<Req*>& pq = r->small ? s->pend_small : s->pend_large;
  auto q = std::find(pq.begin(), pq.end(), r);
  if (q == pq.end()) return LM_ERR_UNSUPPORTED;  // already admitted (or done)
  pq.erase(q);
  r->cancelled = true;
  r->done = true;
  r->status = LM_ERR_ARG;
  ++s->cancelled;
  s->cv_done.notify_all();
  return LM_OK;
}

int lm_server_drain(lm_server* s, double timeout_s) {
  if (!s) return LM_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  const auto pred = [&] { return s->pending_count() == 0 && s->inflight == 0; };
  if (timeout_s > 0) {
    if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred)) return LM_ERR_TIMEOUT;
  } else {
    s->cv_done.wait(lk, pred);
  }
  return LM_OK;
}

int lm_server_stats(lm_server* s, lm_server_stats_t* o) {
  if (!s || !o) return LM_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(o, 0, sizeof(*o));
  o->completed = s->completed;
  o->rejected = s->rejected;
  o->cancelled = s->cancelled;
  o->failed = s->failed;
  o->fp64_fallbacks = s->fallbacks;
  o->ir_solves = s->ir_solves;
  o->ir_gepp = s->ir_gepp;
  o->ir_iterations = s->ir_iterations;
  o->queue_peak = (long long)s->queue_peak;
  o->inflight_peak = s->inflight_peak;
  o->arena_bytes = s->arena.size;
  o->arena_peak_bytes = s->arena.peak;
  o->fixed_bytes = s->fixed_bytes;
  o->pending = (long long)s->pending_count();
  o->inflight = s->inflight;
  std::vector<double> v = s->lat_ms;
  if (!v.empty()) {
    std::sort(v.begin(), v.end());
    auto pct = [&](double p) {
      const double pos = p * (v.size() - 1);
      const size_t i = (size_t)pos;
      const double f = pos - i;
      return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
    };
    o->p50_ms = pct(0.50);
    o->p99_ms = pct(0.99);
    o->max_ms = v.back();
    double sum = 0;
    for (double x : v) sum += x;
    o->mean_ms = sum / v.size();
  }
  const double span = s->t_last > s->t_first ? s->t_last - s->t_first : 0.0;
  o->span_s = span;
  o->solves_per_s = span > 0 ? s->completed / span : 0.0;
  o->tflops = span > 0 ? s->flops_done / span / 1e12 : 0.0;
  long long batches = 0, small = 0;
  for (Lane* ln : s->lanes) {
    batches += ln->batches;
    small += ln->solved;
  }
  if (s->loop) {
    batches += s->loop->launches;
    small += s->loop->solved;
  }
  o->micro_batches = batches;
  o->small_solved = small;
  return LM_OK;
}

int lm_server_reset_stats(lm_server* s) {
  if (!s) return LM_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  s->lat_ms.clear();
  s->completed = s->rejected = s->cancelled = s->failed = s->fallbacks = 0;
  s->ir_solves = s->ir_gepp = s->ir_iterations = 0;
  s->queue_peak = 0;
  s->inflight_peak = s->inflight;
  s->t_first = s->t_last = 0;
  s->flops_done = 0;
  s->arena.peak = s->arena.in_use;
  for (Lane* ln : s->lanes) ln->batches = ln->solved = 0;
  return LM_OK;
}

int lm_server_destroy(lm_server* s) {
  if (!s) return LM_OK;
  server_stop(s);
  server_free(s);
  return LM_OK;
}

}  // extern "C"
