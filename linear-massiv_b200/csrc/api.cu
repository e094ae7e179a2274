// Context, memory and the extern "C" entry points of lm_b200.h.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cudaTypedefs.h>

#include "common.cuh"
#include "internal.h"

struct lm_ctx;

namespace lm {

struct ProfRec {
  int phase;
  cudaEvent_t a, b;
  double flops, bytes;
};

struct GraphEntry {
  std::string key;
  int stage = 0;  // 1: seen once (eager), 2: captured
  cudaGraphExec_t exec = nullptr;
  long long nlaunch = 0;  // kernels in the graph (for the launch counter)
};

struct Ctx {
  bool graphs = true;         // capture repeated call sequences into CUDA graphs
  std::vector<GraphEntry> gcache;
  long long ws_generation = 0;
  cudaStream_t side = nullptr;  // capture stream when the caller's stream is the legacy default
  cudaStream_t aux = nullptr;   // look-ahead stream of the factorisations (ctx_aux)
  bool allow_aux = true;        // false: the factorisations run without look-ahead
  cudaEvent_t ev_la[2] = {};    // its fork / join events
  void* pinned = nullptr;       // ctx_pinned
  size_t pinned_bytes = 0;
  size_t max_graphs = 16;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  bool prof = false;
  std::vector<ProfRec> recs;
  std::vector<cudaEvent_t> pool;
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int* d_status = nullptr;  // int[4], see common.cuh
  void* ws[kWsSlots] = {};
  size_t ws_bytes[kWsSlots] = {};
  std::mutex mu;
  int ir_method = LM_IR_GEPP;  // lm_ctx_set_ir_method
  int ir_last = -1;           // method of the last mixed-precision result
  std::vector<double> ir_hist;  // worst backward error after each refinement step (ctx_ir_history)
  // batch kernel panel width per precision and size bucket (lm_batch_tune)
  int batch_nb[2][BatchLimits::kBuckets] = {{16, 16, 16, 16}, {16, 16, 16, 16}};
};

namespace {
thread_local std::string g_last_error;
std::atomic<long long> g_launches{0};

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;

int load_encode() {
  std::call_once(g_encode_once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  });
  if (!g_encode) {
    set_last_error("cuTensorMapEncodeTiled is not available from the driver");
    return LM_ERR_CUDA;
  }
  return LM_OK;
}
}  // namespace

void set_last_error(const std::string& msg) { g_last_error = msg; }
void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

namespace {
cudaEvent_t take_event(Ctx& c) {
  if (!c.pool.empty()) {
    cudaEvent_t e = c.pool.back();
    c.pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}
}  // namespace

Prof::Prof(Ctx& cc, int ph, double f, double b, cudaStream_t s) : c(cc), phase(ph), flops(f), bytes(b), st(s) {
  if (c.prof) {
    a = take_event(c);
    cudaEventRecord(a, st);
  }
}

Prof::~Prof() {
  if (a) {
    cudaEvent_t b = take_event(c);
    cudaEventRecord(b, st);
    c.recs.push_back({phase, a, b, flops, bytes});
  }
}

int* ctx_status(Ctx& c) { return c.d_status; }
int ctx_num_sms(Ctx& c) { return c.num_sms; }

std::vector<double>& ctx_ir_history(Ctx& c) { return c.ir_hist; }

int ctx_pinned(Ctx& c, size_t bytes, void** ptr) {
  if (c.pinned_bytes < bytes) {
    if (c.pinned) {
      LM_CUDA_TRY(cudaStreamSynchronize(c.stream));
      cudaFreeHost(c.pinned);
      c.pinned = nullptr;
      c.pinned_bytes = 0;
    }
    // 64 KB holds every user's words (the refinement norms, the GMRES dot
    // products and coefficients), so the buffer normally never moves
    const size_t want = std::max(bytes, (size_t)65536);
    ++c.ws_generation;  // captured graphs that copy into the old buffer are stale
    if (cudaMallocHost(&c.pinned, want) != cudaSuccess) {
      cudaGetLastError();
      set_last_error("pinned host allocation failed");
      return LM_ERR_NOMEM;
    }
    c.pinned_bytes = want;
  }
  *ptr = c.pinned;
  return LM_OK;
}

bool ctx_lookahead(Ctx& c) { return c.allow_aux; }

int ctx_aux(Ctx& c, cudaStream_t* aux, cudaEvent_t* fork, cudaEvent_t* join) {
  if (!c.allow_aux) return LM_ERR_UNSUPPORTED;
  if (!c.aux) {
    int lo = 0, hi = 0;
    LM_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    LM_CUDA_TRY(cudaStreamCreateWithPriority(&c.aux, cudaStreamNonBlocking, hi));
    LM_CUDA_TRY(cudaEventCreateWithFlags(&c.ev_la[0], cudaEventDisableTiming));
    LM_CUDA_TRY(cudaEventCreateWithFlags(&c.ev_la[1], cudaEventDisableTiming));
  }
  *aux = c.aux;
  *fork = c.ev_la[0];
  *join = c.ev_la[1];
  return LM_OK;
}
int ctx_device(Ctx& c) { return c.device; }

int ctx_workspace(Ctx& c, int slot, size_t bytes, void** ptr) {
  if (slot < 0 || slot >= kWsSlots) return LM_ERR_ARG;
  if (c.ws_bytes[slot] < bytes) {
    if (c.ws[slot]) {
      // the old buffer may still be in use by queued work on this stream
      LM_CUDA_TRY(cudaStreamSynchronize(c.stream));
      LM_CUDA_TRY(cudaFree(c.ws[slot]));
      c.ws[slot] = nullptr;
      c.ws_bytes[slot] = 0;
    }
    size_t want = std::max(bytes, (size_t)1 << 20);
    ++c.ws_generation;  // captured graphs that baked in the old buffer are stale
    if (cudaMalloc(&c.ws[slot], want) != cudaSuccess) {
      cudaGetLastError();
      set_last_error("workspace allocation failed");
      return LM_ERR_NOMEM;
    }
    c.ws_bytes[slot] = want;
  }
  *ptr = c.ws[slot];
  return LM_OK;
}

int make_tmap_2d(CUtensorMap* tm, CUtensorMapDataType dt, int elem_bytes, const void* base,
                 long long inner, long long outer, long long ld, int box_inner, int box_outer,
                 CUtensorMapSwizzle swz) {
  LM_TRY(load_encode());
  if (inner <= 0 || outer <= 0) return LM_ERR_ARG;
  cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)outer};
  cuuint64_t strides[1] = {(cuuint64_t)(ld * elem_bytes)};
  cuuint32_t box[2] = {(cuuint32_t)box_inner, (cuuint32_t)box_outer};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = g_encode(tm, dt, 2, const_cast<void*>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_last_error("cuTensorMapEncodeTiled failed with CUresult " + std::to_string((int)r));
    return LM_ERR_CUDA;
  }
  return LM_OK;
}

// Reset the device info word before a factorisation.
int reset_info(Ctx& c) {
  LM_CUDA_TRY(cudaMemsetAsync(c.d_status + 1, 0, sizeof(int), c.stream));
  return LM_OK;
}

// Read back {error, info}; returns the status the ABI reports.
int read_status(Ctx& c, int* info_out) {
  int h[2] = {0, 0};
  LM_CUDA_TRY(cudaMemcpyAsync(h, c.d_status, 2 * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  LM_CUDA_TRY(cudaStreamSynchronize(c.stream));
  if (h[0] != LM_DEVERR_NONE) {
    set_last_error(h[0] == LM_DEVERR_TIMEOUT ? "a bounded device-side wait timed out"
                                              : "a device-side self-check failed");
    int z = 0;
    cudaMemcpy(c.d_status, &z, sizeof(int), cudaMemcpyHostToDevice);
    return LM_ERR_TIMEOUT;
  }
  if (info_out) *info_out = h[1];
  return h[1];
}

// Run `body(stream)` — a fixed sequence of launches — through a cached CUDA
// graph: the first call with a key runs eagerly (sizing workspaces, setting
// kernel attributes), the second is captured and replayed, later calls only
// replay.  Disabled while tracing is on (event timings need eager launches).
template <typename F>
int run_graphed(Ctx& c, const std::string& key0, F&& body) {
  if (!c.graphs || c.prof) return body(c.stream);
  const std::string key = key0 + "|g" + std::to_string(c.ws_generation);
  GraphEntry* e = nullptr;
  for (auto& g : c.gcache)
    if (g.key == key) e = &g;
  if (!e) {
    if (c.gcache.size() >= c.max_graphs) {
      if (c.gcache.front().exec) cudaGraphExecDestroy(c.gcache.front().exec);
      c.gcache.erase(c.gcache.begin());
    }
    c.gcache.push_back(GraphEntry{key, 1, nullptr});
    return body(c.stream);
  }
  // The legacy default stream cannot be captured: use a side stream joined
  // to the caller's stream by events.
  cudaStream_t cs = c.stream;
  const bool via_side = (c.stream == nullptr || c.stream == cudaStreamLegacy || c.stream == cudaStreamPerThread);
  if (via_side) {
    if (!c.side) {
      LM_CUDA_TRY(cudaStreamCreateWithFlags(&c.side, cudaStreamNonBlocking));
      LM_CUDA_TRY(cudaEventCreateWithFlags(&c.ev_in, cudaEventDisableTiming));
      LM_CUDA_TRY(cudaEventCreateWithFlags(&c.ev_out, cudaEventDisableTiming));
    }
    cs = c.side;
  }
  if (e->stage == 1) {
    if (via_side) {
      LM_CUDA_TRY(cudaEventRecord(c.ev_in, c.stream));
      LM_CUDA_TRY(cudaStreamWaitEvent(cs, c.ev_in, 0));
    }
    LM_CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    const long long l0 = g_launches.load();
    int r = body(cs);
    e->nlaunch = g_launches.load() - l0;
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(cs, &g);
    if (r != LM_OK) {
      if (g) cudaGraphDestroy(g);
      return r;
    }
    if (ce != cudaSuccess) {
      cudaGetLastError();
      set_last_error(std::string("graph capture failed: ") + cudaGetErrorString(ce));
      return LM_ERR_CUDA;
    }
    cudaGraphExec_t ex = nullptr;
    ce = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) {
      set_last_error(std::string("graph instantiate failed: ") + cudaGetErrorString(ce));
      return LM_ERR_CUDA;
    }
    e->exec = ex;
    e->stage = 2;
    LM_CUDA_TRY(cudaGraphLaunch(ex, cs));
  } else {
    if (via_side) {
      LM_CUDA_TRY(cudaEventRecord(c.ev_in, c.stream));
      LM_CUDA_TRY(cudaStreamWaitEvent(cs, c.ev_in, 0));
    }
    LM_CUDA_TRY(cudaGraphLaunch(e->exec, cs));
    count_launch((int)e->nlaunch);
  }
  if (via_side) {
    LM_CUDA_TRY(cudaEventRecord(c.ev_out, cs));
    LM_CUDA_TRY(cudaStreamWaitEvent(c.stream, c.ev_out, 0));
  }
  return LM_OK;
}

int dpotrf_borrowed(int device, int num_sms, cudaStream_t st, int n, double* A, long long lda, int* d_status,
                    void* scratch, size_t scratch_bytes) {
  Ctx c;
  c.device = device;
  c.num_sms = num_sms;
  c.stream = st;
  c.graphs = false;
  c.allow_aux = false;  // one stream, no CUDA objects created on the caller's behalf
  c.d_status = d_status;
  c.ws[1] = scratch;  // grow-only workspace that never needs to grow
  c.ws_bytes[1] = scratch_bytes;
  const int r = dpotrf(c, n, A, lda, st);
  c.ws[1] = nullptr;  // borrowed: nothing to free
  return r;
}

std::string gkey(const char* op, std::initializer_list<long long> v) {
  std::string k(op);
  for (long long x : v) k += "," + std::to_string(x);
  return k;
}

}  // namespace lm

struct lm_ctx {
  lm::Ctx c;
};

using lm::Ctx;

namespace lm {
void ctx_set_graphs(lm_ctx* ctx, bool on) {
  if (!ctx) return;
  std::lock_guard<std::mutex> lock(ctx->c.mu);
  ctx->c.graphs = on;
}

void ctx_set_graph_cache(lm_ctx* ctx, int max_graphs) {
  if (!ctx || max_graphs < 1) return;
  std::lock_guard<std::mutex> lock(ctx->c.mu);
  ctx->c.max_graphs = (size_t)max_graphs;
}
}  // namespace lm

namespace {

template <typename F>
int guarded(lm_ctx* ctx, F&& f) {
  if (!ctx) return LM_ERR_ARG;
  std::lock_guard<std::mutex> lock(ctx->c.mu);
  if (cudaSetDevice(ctx->c.device) != cudaSuccess) {
    lm::set_last_error("cudaSetDevice failed");
    return LM_ERR_CUDA;
  }
  return f(ctx->c);
}

inline long long rup(long long a, long long b) { return (a + b - 1) / b * b; }

}  // namespace

extern "C" {

int lm_ctx_create(lm_ctx** out, int device) {
  if (!out) return LM_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  LM_CUDA_TRY(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev || device >= lm::kMaxDevices) return LM_ERR_ARG;
  LM_CUDA_TRY(cudaSetDevice(device));
  cudaDeviceProp prop;
  LM_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) {
    lm::set_last_error("this library is built for sm_100a (B200); device is sm_" +
                       std::to_string(prop.major) + std::to_string(prop.minor));
    return LM_ERR_UNSUPPORTED;
  }
  auto* ctx = new lm_ctx();
  ctx->c.device = device;
  ctx->c.num_sms = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&ctx->c.stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&ctx->c.d_status, 4 * sizeof(int)) != cudaSuccess) {
    lm::set_last_error("context allocation failed");
    delete ctx;
    return LM_ERR_CUDA;
  }
  ctx->c.own_stream = true;
  cudaMemset(ctx->c.d_status, 0, 4 * sizeof(int));
  *out = ctx;
  return LM_OK;
}

int lm_ctx_destroy(lm_ctx* ctx) {
  if (!ctx) return LM_OK;
  {
    std::lock_guard<std::mutex> lock(ctx->c.mu);
    cudaSetDevice(ctx->c.device);
    cudaStreamSynchronize(ctx->c.stream);
    for (int s = 0; s < lm::kWsSlots; ++s)
      if (ctx->c.ws[s]) cudaFree(ctx->c.ws[s]);
    for (auto& r : ctx->c.recs) {
      cudaEventDestroy(r.a);
      cudaEventDestroy(r.b);
    }
    for (auto e : ctx->c.pool) cudaEventDestroy(e);
    for (auto& g : ctx->c.gcache)
      if (g.exec) cudaGraphExecDestroy(g.exec);
    if (ctx->c.side) cudaStreamDestroy(ctx->c.side);
    if (ctx->c.aux) cudaStreamDestroy(ctx->c.aux);
    if (ctx->c.pinned) cudaFreeHost(ctx->c.pinned);
    for (auto e : ctx->c.ev_la)
      if (e) cudaEventDestroy(e);
    if (ctx->c.ev_in) cudaEventDestroy(ctx->c.ev_in);
    if (ctx->c.ev_out) cudaEventDestroy(ctx->c.ev_out);
    if (ctx->c.d_status) cudaFree(ctx->c.d_status);
    if (ctx->c.own_stream) cudaStreamDestroy(ctx->c.stream);
  }
  delete ctx;
  return LM_OK;
}

int lm_ctx_set_stream(lm_ctx* ctx, void* stream) {
  return guarded(ctx, [&](Ctx& c) {
    if (c.own_stream) {
      cudaStreamSynchronize(c.stream);
      cudaStreamDestroy(c.stream);
      c.own_stream = false;
    }
    c.stream = static_cast<cudaStream_t>(stream);
    return LM_OK;
  });
}

void* lm_ctx_get_stream(lm_ctx* ctx) { return ctx ? (void*)ctx->c.stream : nullptr; }

int lm_ctx_synchronize(lm_ctx* ctx) {
  return guarded(ctx, [&](Ctx& c) {
    LM_CUDA_TRY(cudaStreamSynchronize(c.stream));
    return LM_OK;
  });
}

int lm_ctx_check(lm_ctx* ctx) {
  return guarded(ctx, [&](Ctx& c) {
    int r = lm::read_status(c, nullptr);
    return r < 0 ? r : LM_OK;
  });
}

int lm_ctx_set_ir_method(lm_ctx* ctx, int method) {
  return guarded(ctx, [&](Ctx& c) {
    if (method != LM_IR_RBT && method != LM_IR_GEPP) return LM_ERR_ARG;
    c.ir_method = method;
    return LM_OK;
  });
}

int lm_ctx_ir_history(lm_ctx* ctx, double* berr, int max_steps, int* steps) {
  return guarded(ctx, [&](Ctx& c) {
    if (!steps || max_steps < 0 || (max_steps > 0 && !berr)) return LM_ERR_ARG;
    const int k = std::min<int>(max_steps, (int)c.ir_hist.size());
    for (int i = 0; i < k; ++i) berr[i] = c.ir_hist[i];
    *steps = (int)c.ir_hist.size();
    return LM_OK;
  });
}

int lm_ctx_ir_last_method(lm_ctx* ctx, int* method) {
  return guarded(ctx, [&](Ctx& c) {
    if (!method) return LM_ERR_ARG;
    *method = c.ir_last;
    return LM_OK;
  });
}

int lm_ctx_profile(lm_ctx* ctx, int enable) {
  return guarded(ctx, [&](Ctx& c) {
    c.prof = enable != 0;
    return LM_OK;
  });
}

int lm_ctx_profile_read(lm_ctx* ctx, long long* launches, double* ms, double* flops, double* bytes) {
  return guarded(ctx, [&](Ctx& c) {
    LM_CUDA_TRY(cudaStreamSynchronize(c.stream));
    long long L[lm::kNumPhases] = {};
    double M[lm::kNumPhases] = {}, F[lm::kNumPhases] = {}, B[lm::kNumPhases] = {};
    for (auto& r : c.recs) {
      float t = 0.f;
      cudaEventElapsedTime(&t, r.a, r.b);
      L[r.phase] += 1;
      M[r.phase] += t;
      F[r.phase] += r.flops;
      B[r.phase] += r.bytes;
      c.pool.push_back(r.a);
      c.pool.push_back(r.b);
    }
    c.recs.clear();
    for (int i = 0; i < lm::kNumPhases; ++i) {
      if (launches) launches[i] = L[i];
      if (ms) ms[i] = M[i];
      if (flops) flops[i] = F[i];
      if (bytes) bytes[i] = B[i];
    }
    return LM_OK;
  });
}

const char* lm_status_string(int s) {
  switch (s) {
    case LM_OK: return "ok";
    case LM_ERR_ARG: return "invalid argument";
    case LM_ERR_CUDA: return "CUDA error";
    case LM_ERR_UNSUPPORTED: return "unsupported configuration";
    case LM_ERR_TIMEOUT: return "device-side wait timed out";
    case LM_ERR_NOMEM: return "out of memory";
    case LM_ERR_NOT_CONVERGED: return "iterative refinement did not converge";
    default: return s > 0 ? "numerical breakdown (info > 0)" : "unknown error";
  }
}

const char* lm_last_error(void) { return lm::g_last_error.c_str(); }
long long lm_launch_count(void) { return lm::g_launches.load(); }

int lm_dmalloc(lm_ctx* ctx, void** ptr, size_t bytes) {
  return guarded(ctx, [&](Ctx&) {
    if (!ptr) return LM_ERR_ARG;
    if (cudaMalloc(ptr, bytes) != cudaSuccess) {
      cudaGetLastError();
      return LM_ERR_NOMEM;
    }
    return LM_OK;
  });
}

int lm_dfree(lm_ctx* ctx, void* ptr) {
  return guarded(ctx, [&](Ctx& c) {
    LM_CUDA_TRY(cudaStreamSynchronize(c.stream));
    LM_CUDA_TRY(cudaFree(ptr));
    return LM_OK;
  });
}

int lm_h2d(lm_ctx* ctx, void* dst, const void* src, size_t bytes) {
  return guarded(ctx, [&](Ctx& c) {
    LM_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c.stream));
    LM_CUDA_TRY(cudaStreamSynchronize(c.stream));
    return LM_OK;
  });
}

int lm_d2h(lm_ctx* ctx, void* dst, const void* src, size_t bytes) {
  return guarded(ctx, [&](Ctx& c) {
    LM_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c.stream));
    LM_CUDA_TRY(cudaStreamSynchronize(c.stream));
    return LM_OK;
  });
}

int lm_dgemm(lm_ctx* ctx, int m, int n, int k, double alpha, const double* A, int lda,
             const double* B, int ldb, double beta, double* C, int ldc) {
  return guarded(ctx, [&](Ctx& c) {
    if (m < 0 || n < 0 || k < 0 || (m > 0 && n > 0 && !C)) return LM_ERR_ARG;
    if ((k > 0 && m > 0 && (!A || lda < k)) || (k > 0 && n > 0 && (!B || ldb < n)) ||
        (m > 0 && n > 0 && ldc < n))
      return LM_ERR_ARG;
    lm::GemmDesc d;
    d.m = m; d.n = n; d.k = k;
    d.alpha = alpha; d.beta = beta;
    d.A = A; d.lda = lda; d.B = B; d.ldb = ldb; d.C = C; d.ldc = ldc;
    const bool aligned = !((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15) &&
                         !(lda & 1) && !(ldb & 1);
    if (aligned || k == 0 || alpha == 0.0) return lm::dgemm(c, d, c.stream);
    // TMA needs 16-byte aligned rows: stage A and B with even strides.
    const long long lda2 = rup(k, 2), ldb2 = rup(n, 2);
    void* ws = nullptr;
    LM_TRY(lm::ctx_workspace(c, 0, sizeof(double) * ((size_t)m * lda2 + (size_t)k * ldb2), &ws));
    double* A2 = static_cast<double*>(ws);
    double* B2 = A2 + (size_t)m * lda2;
    LM_TRY(lm::copy2d<double>(A2, lda2, A, lda, m, k, c.stream));
    LM_TRY(lm::copy2d<double>(B2, ldb2, B, ldb, k, n, c.stream));
    d.A = A2; d.lda = lda2; d.B = B2; d.ldb = ldb2;
    return lm::dgemm(c, d, c.stream);
  });
}

}  // extern "C"

namespace {

// Run `fn(A2, lda2)` on an even-stride copy of A when lda is odd or A is
// misaligned (TMA rows must start on 16 bytes), copying the result back.
template <typename F>
int with_aligned(Ctx& c, int n, double* A, long long lda, cudaStream_t st, F&& fn) {
  if (!((reinterpret_cast<uintptr_t>(A) & 15) || (lda & 1))) return fn(A, lda);
  const long long lda2 = rup(n, 8);
  void* ws = nullptr;
  LM_TRY(lm::ctx_workspace(c, 0, sizeof(double) * (size_t)n * lda2, &ws));
  double* A2 = static_cast<double*>(ws);
  LM_TRY(lm::copy2d<double>(A2, lda2, A, lda, n, n, st));
  int r = fn(A2, lda2);
  if (r < 0) return r;
  LM_TRY(lm::copy2d<double>(A, lda, A2, lda2, n, n, st));
  return r;
}

int finish_info(Ctx& c, int* info) {
  if (!info) return LM_OK;
  int r = lm::read_status(c, info);
  return r;
}

// Mixed-precision solve with the context's method: partial pivoting
// (LM_IR_GEPP, the default), or the randomised no-pivoting factor first
// (LM_IR_RBT) with partial pivoting when its refinement stalls.  A zero pivot of the randomised factor only triggers the fallback;
// the reported info is that of the method whose result is returned.
int ir_solve(Ctx& c, int n, int nrhs, const double* A, long long lda, const double* B, long long ldb, double* X,
             long long ldx, double tol, int max_iter, int* iters, double* berr, const char* tag) {
  // graph keys: the factor depends on A; a refinement step on every buffer
  auto runner = [&](const char* method) {
    return [&c, n, nrhs, A, lda, B, ldb, X, ldx, tag, method](const char* what,
                                                              const std::function<int(cudaStream_t)>& body) {
      const std::string k = std::string(method) + "_" + tag + "_" + what;
      const std::string key =
          std::strcmp(what, "factor") == 0
              ? lm::gkey(k.c_str(), {n, (long long)A, lda})
              : lm::gkey(k.c_str(), {n, nrhs, (long long)A, lda, (long long)B, ldb, (long long)X, ldx});
      return lm::run_graphed(c, key, body);
    };
  };
  c.ir_hist.clear();
  if (c.ir_method == LM_IR_RBT) {
    int r = lm::dgesv_rbt_ir(c, n, nrhs, A, lda, B, ldb, X, ldx, tol, max_iter, iters, berr, c.stream, runner("rbt"));
    if (r != LM_ERR_NOT_CONVERGED) {
      c.ir_last = LM_IR_RBT;
      return r;
    }
    LM_TRY(lm::reset_info(c));
  }
  c.ir_last = LM_IR_GEPP;
  return lm::dgesv_ir(c, n, nrhs, A, lda, B, ldb, X, ldx, tol, max_iter, iters, berr, c.stream, runner("gepp"));
}

}  // namespace

extern "C" {

int lm_dgetrf(lm_ctx* ctx, int n, double* A, int lda, int* ipiv, int* info) {
  return guarded(ctx, [&](Ctx& c) {
    if (n < 0 || (n > 0 && (!A || !ipiv || lda < n))) return LM_ERR_ARG;
    if (n == 0) {
      if (info) *info = 0;
      return LM_OK;
    }
    LM_TRY(lm::reset_info(c));
    LM_TRY(lm::run_graphed(c, lm::gkey("getrf", {n, (long long)A, lda, (long long)ipiv}), [&](cudaStream_t s) {
      return with_aligned(c, n, A, lda, s, [&](double* A2, long long l2) { return lm::dgetrf(c, n, A2, l2, ipiv, s); });
    }));
    return finish_info(c, info);
  });
}

int lm_dgetrs(lm_ctx* ctx, int n, int nrhs, const double* LU, int lda, const int* ipiv, double* B,
              int ldb) {
  return guarded(ctx, [&](Ctx& c) {
    if (n < 0 || nrhs < 0 || (n > 0 && nrhs > 0 && (!LU || !ipiv || !B || lda < n || ldb < nrhs)))
      return LM_ERR_ARG;
    if (n == 0 || nrhs == 0) return LM_OK;
    return lm::run_graphed(c, lm::gkey("getrs", {n, nrhs, (long long)LU, lda, (long long)ipiv, (long long)B, ldb}),
                           [&](cudaStream_t s) { return lm::dgetrs(c, n, nrhs, LU, lda, ipiv, B, ldb, s); });
  });
}

int lm_dgesv(lm_ctx* ctx, int n, int nrhs, double* A, int lda, int* ipiv, double* B, int ldb,
             int* info) {
  return guarded(ctx, [&](Ctx& c) {
    if (n < 0 || nrhs < 0 || (n > 0 && (!A || !ipiv || lda < n || (nrhs > 0 && (!B || ldb < nrhs)))))
      return LM_ERR_ARG;
    if (n == 0) {
      if (info) *info = 0;
      return LM_OK;
    }
    LM_TRY(lm::reset_info(c));
    LM_TRY(lm::run_graphed(
        c, lm::gkey("gesv", {n, nrhs, (long long)A, lda, (long long)ipiv, (long long)B, ldb}), [&](cudaStream_t s) {
          LM_TRY(with_aligned(c, n, A, lda, s,
                              [&](double* A2, long long l2) { return lm::dgetrf(c, n, A2, l2, ipiv, s); }));
          if (nrhs == 0) return LM_OK;
          return lm::dgetrs(c, n, nrhs, A, lda, ipiv, B, ldb, s);
        }));
    return finish_info(c, info);
  });
}

int lm_dpotrf(lm_ctx* ctx, int n, double* A, int lda, int* info) {
  return guarded(ctx, [&](Ctx& c) {
    if (n < 0 || (n > 0 && (!A || lda < n))) return LM_ERR_ARG;
    if (n == 0) {
      if (info) *info = 0;
      return LM_OK;
    }
    LM_TRY(lm::reset_info(c));
    LM_TRY(lm::run_graphed(c, lm::gkey("potrf", {n, (long long)A, lda}), [&](cudaStream_t s) {
      return with_aligned(c, n, A, lda, s, [&](double* A2, long long l2) { return lm::dpotrf(c, n, A2, l2, s); });
    }));
    return finish_info(c, info);
  });
}

int lm_dpotrs(lm_ctx* ctx, int n, int nrhs, const double* G, int lda, double* B, int ldb) {
  return guarded(ctx, [&](Ctx& c) {
    if (n < 0 || nrhs < 0 || (n > 0 && nrhs > 0 && (!G || !B || lda < n || ldb < nrhs)))
      return LM_ERR_ARG;
    if (n == 0 || nrhs == 0) return LM_OK;
    return lm::run_graphed(c, lm::gkey("potrs", {n, nrhs, (long long)G, lda, (long long)B, ldb}),
                           [&](cudaStream_t s) { return lm::dpotrs(c, n, nrhs, G, lda, B, ldb, s); });
  });
}

int lm_dposv(lm_ctx* ctx, int n, int nrhs, double* A, int lda, double* B, int ldb, int* info) {
  return guarded(ctx, [&](Ctx& c) {
    if (n < 0 || nrhs < 0 || (n > 0 && (!A || lda < n || (nrhs > 0 && (!B || ldb < nrhs))))) return LM_ERR_ARG;
    if (n == 0) {
      if (info) *info = 0;
      return LM_OK;
    }
    LM_TRY(lm::reset_info(c));
    LM_TRY(lm::run_graphed(c, lm::gkey("posv", {n, nrhs, (long long)A, lda, (long long)B, ldb}),
                           [&](cudaStream_t s) {
                             LM_TRY(with_aligned(c, n, A, lda, s, [&](double* A2, long long l2) {
                               return lm::dpotrf(c, n, A2, l2, s);
                             }));
                             if (nrhs == 0) return LM_OK;
                             return lm::dpotrs(c, n, nrhs, A, lda, B, ldb, s);
                           }));
    return finish_info(c, info);
  });
}

int lm_dgesv_ir(lm_ctx* ctx, int n, int nrhs, const double* A, int lda, const double* B, int ldb, double* X,
                int ldx, double tol, int max_iter, int* iters, double* berr, int* info) {
  return guarded(ctx, [&](Ctx& c) {
    if (n < 0 || nrhs < 0 || nrhs > 64 || max_iter < 1) return LM_ERR_ARG;
    if (n == 0 || nrhs == 0) {
      if (iters) *iters = 0;
      if (berr) *berr = 0.0;
      if (info) *info = 0;
      return LM_OK;
    }
    if (!A || !B || !X || lda < n || ldb < nrhs || ldx < nrhs) return LM_ERR_ARG;
    if (tol <= 0) tol = 1e-15 * n;
    LM_TRY(lm::reset_info(c));
    int r = ir_solve(c, n, nrhs, A, lda, B, ldb, X, ldx, tol, max_iter, iters, berr, "dev");
    int inf = 0;
    int s = lm::read_status(c, &inf);
    if (s < 0) return s;
    if (info) *info = inf;
    if (r < 0) return r;
    return inf;
  });
}

int lm_dgesv_ir_prec(lm_ctx* ctx, int n, int nrhs, const double* A, int lda, const double* B, int ldb, double* X,
                     int ldx, int prec, double tol, int max_iter, int* iters, double* berr, int* info) {
  return guarded(ctx, [&](Ctx& c) {
    if (n < 0 || nrhs < 0 || nrhs > 64 || max_iter < 1) return LM_ERR_ARG;
    if (prec != LM_IR_PREC_TF32X3 && prec != LM_IR_PREC_TF32 && prec != LM_IR_PREC_BF16) return LM_ERR_ARG;
    if (n == 0 || nrhs == 0) {
      if (iters) *iters = 0;
      if (berr) *berr = 0.0;
      if (info) *info = 0;
      return LM_OK;
    }
    if (!A || !B || !X || lda < n || ldb < nrhs || ldx < nrhs) return LM_ERR_ARG;
    if (tol <= 0) tol = 1e-15 * n;
    LM_TRY(lm::reset_info(c));
    c.ir_hist.clear();
    c.ir_last = LM_IR_GEPP;
    auto runner = [&c, n, nrhs, A, lda, B, ldb, X, ldx, prec](const char* what,
                                                             const std::function<int(cudaStream_t)>& body) {
      const std::string k = std::string("gepp_p") + std::to_string(prec) + "_" + what;
      const std::string key =
          std::strncmp(what, "factor", 6) == 0
              ? lm::gkey(k.c_str(), {n, (long long)A, lda})
              : lm::gkey(k.c_str(), {n, nrhs, (long long)A, lda, (long long)B, ldb, (long long)X, ldx});
      return lm::run_graphed(c, key, body);
    };
    int r = lm::dgesv_ir(c, n, nrhs, A, lda, B, ldb, X, ldx, tol, max_iter, iters, berr, c.stream, runner, prec);
    int inf = 0;
    int s = lm::read_status(c, &inf);
    if (s < 0) return s;
    if (info) *info = inf;
    if (r < 0) return r;
    return inf;
  });
}

int lm_dresidual(lm_ctx* ctx, int n, int nrhs, const double* A, int lda, const double* X, int ldx,
                 const double* B, int ldb, double* R, int ldr) {
  return guarded(ctx, [&](Ctx& c) {
    if (n < 0 || nrhs < 0) return LM_ERR_ARG;
    if (n == 0 || nrhs == 0) return LM_OK;
    if (!A || !X || !B || !R || lda < n || ldx < nrhs || ldb < nrhs || ldr < nrhs) return LM_ERR_ARG;
    return lm::dresidual(c, n, nrhs, A, lda, X, ldx, B, ldb, R, ldr, c.stream);
  });
}

int lm_dgemv(lm_ctx* ctx, int m, int n, const double* A, int lda, const double* x, double* y) {
  return guarded(ctx, [&](Ctx& c) {
    if (m < 0 || n < 0) return LM_ERR_ARG;
    if (m == 0) return LM_OK;
    if (!y || (n > 0 && (!A || !x || lda < n))) return LM_ERR_ARG;
    return lm::dgemv_exact(m, n, A, lda, x, y, c.stream);
  });
}

int lm_dnorm_inf(lm_ctx* ctx, int m, int n, const double* A, int lda, double* result) {
  return guarded(ctx, [&](Ctx& c) {
    if (m < 0 || n < 0 || !result || (m > 0 && n > 0 && (!A || lda < n))) return LM_ERR_ARG;
    void* ws = nullptr;
    LM_TRY(lm::ctx_workspace(c, 2, 64, &ws));
    unsigned long long* d = static_cast<unsigned long long*>(ws);
    LM_TRY(lm::dnorm_inf_exact(m, n, A, lda, d, c.stream));
    unsigned long long h = 0;
    LM_CUDA_TRY(cudaMemcpyAsync(&h, d, sizeof h, cudaMemcpyDeviceToHost, c.stream));
    LM_CUDA_TRY(cudaStreamSynchronize(c.stream));
    std::memcpy(result, &h, sizeof h);
    return LM_OK;
  });
}

int lm_dgetrf_nopiv(lm_ctx* ctx, int n, double* A, int lda, int* info) {
  return guarded(ctx, [&](Ctx& c) {
    if (n < 0 || (n > 0 && (!A || lda < n))) return LM_ERR_ARG;
    if (n == 0) {
      if (info) *info = 0;
      return LM_OK;
    }
    LM_TRY(lm::reset_info(c));
    LM_TRY(lm::run_graphed(c, lm::gkey("getrf_nopiv", {n, (long long)A, lda}), [&](cudaStream_t s) {
      return with_aligned(c, n, A, lda, s, [&](double* A2, long long l2) { return lm::dgetrf_nopiv(c, n, A2, l2, s); });
    }));
    return finish_info(c, info);
  });
}

int lm_dtridiag_solve(lm_ctx* ctx, int n, const double* diag, const double* supdiag, const double* b, double* x) {
  return guarded(ctx, [&](Ctx& c) {
    if (n < 0 || (n > 0 && (!diag || !b || !x || (n > 1 && !supdiag)))) return LM_ERR_ARG;
    if (n == 0) return LM_OK;
    void* ws = nullptr;
    LM_TRY(lm::ctx_workspace(c, 2, sizeof(double) * 8 * (size_t)n, &ws));
    return lm::dtridiag_pcr(n, diag, n > 1 ? supdiag : diag, b, x, static_cast<double*>(ws), c.stream);
  });
}

int lm_ipiv_to_perm(int n, const int* ipiv, int* perm) {
  if (n < 0 || (n > 0 && (!ipiv || !perm))) return LM_ERR_ARG;
  for (int i = 0; i < n; ++i) perm[i] = i;
  for (int k = 0; k < n; ++k) {
    const int p = ipiv[k];
    if (p < 0 || p >= n) return LM_ERR_ARG;
    std::swap(perm[k], perm[p]);
  }
  return LM_OK;
}

// ---- host-buffer entry points ----------------------------------------------
}  // extern "C"

namespace {

struct HostBufs {
  double* A = nullptr;
  double* B = nullptr;
  int* ipiv = nullptr;
  long long lda = 0, ldb = 0;
};

int host_bufs(Ctx& c, int n, int nrhs, HostBufs& hb) {
  hb.lda = rup(std::max(n, 1), 8);
  hb.ldb = rup(std::max(nrhs, 1), 8);
  const size_t a = sizeof(double) * (size_t)n * hb.lda;
  const size_t b = sizeof(double) * (size_t)n * hb.ldb;
  const size_t p = sizeof(int) * (size_t)rup(std::max(n, 1), 64);
  void* ws = nullptr;
  LM_TRY(lm::ctx_workspace(c, 3, a + b + p, &ws));
  hb.A = static_cast<double*>(ws);
  hb.B = reinterpret_cast<double*>(static_cast<char*>(ws) + a);
  hb.ipiv = reinterpret_cast<int*>(static_cast<char*>(ws) + a + b);
  return LM_OK;
}

int h2d_2d(Ctx& c, double* dst, long long ldd, const double* src, long long lds, int rows, int cols) {
  if (rows == 0 || cols == 0) return LM_OK;
  LM_CUDA_TRY(cudaMemcpy2DAsync(dst, ldd * sizeof(double), src, lds * sizeof(double), cols * sizeof(double),
                                rows, cudaMemcpyHostToDevice, c.stream));
  return LM_OK;
}

int d2h_2d(Ctx& c, double* dst, long long ldd, const double* src, long long lds, int rows, int cols) {
  if (rows == 0 || cols == 0) return LM_OK;
  LM_CUDA_TRY(cudaMemcpy2DAsync(dst, ldd * sizeof(double), src, lds * sizeof(double), cols * sizeof(double),
                                rows, cudaMemcpyDeviceToHost, c.stream));
  return LM_OK;
}

}  // namespace

extern "C" {

int lm_lu_solve_host(lm_ctx* ctx, int n, int nrhs, const double* A, const double* B, double* X,
                     int* info) {
  return guarded(ctx, [&](Ctx& c) {
    if (n < 0 || nrhs < 0 || (n > 0 && (!A || (nrhs > 0 && (!B || !X))))) return LM_ERR_ARG;
    if (n == 0) {
      if (info) *info = 0;
      return LM_OK;
    }
    HostBufs hb;
    LM_TRY(host_bufs(c, n, nrhs, hb));
    LM_TRY(h2d_2d(c, hb.A, hb.lda, A, n, n, n));
    LM_TRY(h2d_2d(c, hb.B, hb.ldb, B, nrhs, n, nrhs));
    LM_TRY(lm::reset_info(c));
    LM_TRY(lm::run_graphed(c, lm::gkey("lu_host", {n, nrhs, (long long)hb.A, hb.lda, (long long)hb.B, hb.ldb}),
                           [&](cudaStream_t s) {
                             LM_TRY(lm::dgetrf(c, n, hb.A, hb.lda, hb.ipiv, s));
                             if (nrhs == 0) return LM_OK;
                             return lm::dgetrs(c, n, nrhs, hb.A, hb.lda, hb.ipiv, hb.B, hb.ldb, s);
                           }));
    LM_TRY(d2h_2d(c, X, nrhs, hb.B, hb.ldb, n, nrhs));
    int inf = 0;
    int r = lm::read_status(c, &inf);
    if (info) *info = inf;
    return r;
  });
}

int lm_chol_solve_host(lm_ctx* ctx, int n, int nrhs, const double* A, const double* B, double* X,
                       int* info) {
  return guarded(ctx, [&](Ctx& c) {
    if (n < 0 || nrhs < 0 || (n > 0 && (!A || (nrhs > 0 && (!B || !X))))) return LM_ERR_ARG;
    if (n == 0) {
      if (info) *info = 0;
      return LM_OK;
    }
    HostBufs hb;
    LM_TRY(host_bufs(c, n, nrhs, hb));
    LM_TRY(h2d_2d(c, hb.A, hb.lda, A, n, n, n));
    LM_TRY(h2d_2d(c, hb.B, hb.ldb, B, nrhs, n, nrhs));
    LM_TRY(lm::reset_info(c));
    LM_TRY(lm::run_graphed(c, lm::gkey("chol_host", {n, nrhs, (long long)hb.A, hb.lda, (long long)hb.B, hb.ldb}),
                           [&](cudaStream_t s) {
                             LM_TRY(lm::dpotrf(c, n, hb.A, hb.lda, s));
                             if (nrhs == 0) return LM_OK;
                             return lm::dpotrs(c, n, nrhs, hb.A, hb.lda, hb.B, hb.ldb, s);
                           }));
    LM_TRY(d2h_2d(c, X, nrhs, hb.B, hb.ldb, n, nrhs));
    int inf = 0;
    int r = lm::read_status(c, &inf);
    if (info) *info = inf;
    return r;
  });
}

int lm_lu_solve_ir_host(lm_ctx* ctx, int n, int nrhs, const double* A, const double* B, double* X, double tol,
                        int max_iter, int* iters, double* berr, int* info) {
  return guarded(ctx, [&](Ctx& c) {
    if (n < 0 || nrhs < 0 || nrhs > 64 || max_iter < 1) return LM_ERR_ARG;
    if (n == 0 || nrhs == 0) {
      if (iters) *iters = 0;
      if (berr) *berr = 0.0;
      if (info) *info = 0;
      return LM_OK;
    }
    if (!A || !B || !X) return LM_ERR_ARG;
    if (tol <= 0) tol = 1e-15 * n;
    HostBufs hb;
    LM_TRY(host_bufs(c, n, 2 * nrhs, hb));  // B and X side by side
    LM_TRY(h2d_2d(c, hb.A, hb.lda, A, n, n, n));
    LM_TRY(h2d_2d(c, hb.B, hb.ldb, B, nrhs, n, nrhs));
    LM_TRY(lm::reset_info(c));
    double* dX = hb.B + nrhs;
    int r = ir_solve(c, n, nrhs, hb.A, hb.lda, hb.B, hb.ldb, dX, hb.ldb, tol, max_iter, iters, berr, "host");
    if (r < 0 && r != LM_ERR_NOT_CONVERGED) return r;
    LM_TRY(d2h_2d(c, X, nrhs, dX, hb.ldb, n, nrhs));
    int inf = 0;
    int s = lm::read_status(c, &inf);
    if (s < 0) return s;
    if (info) *info = inf;
    if (r < 0) return r;
    return inf;
  });
}

int lm_gemm_host(lm_ctx* ctx, int m, int n, int k, double alpha, const double* A, const double* B,
                 double beta, const double* C0, double* C) {
  return guarded(ctx, [&](Ctx& c) {
    if (m < 0 || n < 0 || k < 0) return LM_ERR_ARG;
    if (m == 0 || n == 0) return LM_OK;
    if (!C || (k > 0 && (!A || !B)) || (beta != 0.0 && !C0)) return LM_ERR_ARG;
    const long long lda = rup(std::max(k, 1), 8), ldb = rup(n, 8), ldc = rup(n, 8);
    void* ws = nullptr;
    LM_TRY(lm::ctx_workspace(c, 3, sizeof(double) * ((size_t)m * lda + (size_t)k * ldb + (size_t)m * ldc), &ws));
    double* dA = static_cast<double*>(ws);
    double* dB = dA + (size_t)m * lda;
    double* dC = dB + (size_t)k * ldb;
    LM_TRY(h2d_2d(c, dA, lda, A, k, m, k));
    LM_TRY(h2d_2d(c, dB, ldb, B, n, k, n));
    if (beta != 0.0) LM_TRY(h2d_2d(c, dC, ldc, C0, n, m, n));
    lm::GemmDesc d;
    d.m = m; d.n = n; d.k = k; d.alpha = alpha; d.beta = beta;
    d.A = dA; d.lda = lda; d.B = dB; d.ldb = ldb; d.C = dC; d.ldc = ldc;
    LM_TRY(lm::dgemm(c, d, c.stream));
    LM_TRY(d2h_2d(c, C, n, dC, ldc, m, n));
    int r = lm::read_status(c, nullptr);
    return r < 0 ? r : LM_OK;
  });
}

int lm_matmul_host(lm_ctx* ctx, int m, int n, int k, const double* A, const double* B, double* C) {
  return lm_gemm_host(ctx, m, n, k, 1.0, A, B, 0.0, nullptr, C);
}

int lm_lu_host(lm_ctx* ctx, int n, const double* A, double* LU, int* perm, int* info) {
  return guarded(ctx, [&](Ctx& c) {
    if (n < 0 || (n > 0 && (!A || !LU || !perm))) return LM_ERR_ARG;
    if (n == 0) {
      if (info) *info = 0;
      return LM_OK;
    }
    HostBufs hb;
    LM_TRY(host_bufs(c, n, 0, hb));
    LM_TRY(h2d_2d(c, hb.A, hb.lda, A, n, n, n));
    LM_TRY(lm::reset_info(c));
    LM_TRY(lm::dgetrf(c, n, hb.A, hb.lda, hb.ipiv, c.stream));
    LM_TRY(d2h_2d(c, LU, n, hb.A, hb.lda, n, n));
    std::vector<int> ip(n);
    LM_CUDA_TRY(cudaMemcpyAsync(ip.data(), hb.ipiv, sizeof(int) * n, cudaMemcpyDeviceToHost, c.stream));
    int inf = 0;
    int r = lm::read_status(c, &inf);
    if (r < 0) return r;
    LM_TRY(lm_ipiv_to_perm(n, ip.data(), perm));
    if (info) *info = inf;
    return r;
  });
}

int lm_cholesky_host(lm_ctx* ctx, int n, const double* A, double* G, int* info) {
  return guarded(ctx, [&](Ctx& c) {
    if (n < 0 || (n > 0 && (!A || !G))) return LM_ERR_ARG;
    if (n == 0) {
      if (info) *info = 0;
      return LM_OK;
    }
    HostBufs hb;
    LM_TRY(host_bufs(c, n, 0, hb));
    LM_TRY(h2d_2d(c, hb.A, hb.lda, A, n, n, n));
    LM_TRY(lm::reset_info(c));
    LM_TRY(lm::dpotrf(c, n, hb.A, hb.lda, c.stream));
    LM_TRY(d2h_2d(c, G, n, hb.A, hb.lda, n, n));
    int inf = 0;
    int r = lm::read_status(c, &inf);
    if (info) *info = inf;
    return r;
  });
}

int lm_lu_nopivot_host(lm_ctx* ctx, int n, const double* A, double* LU, int* info) {
  return guarded(ctx, [&](Ctx& c) {
    if (n < 0 || (n > 0 && (!A || !LU))) return LM_ERR_ARG;
    if (n == 0) {
      if (info) *info = 0;
      return LM_OK;
    }
    HostBufs hb;
    LM_TRY(host_bufs(c, n, 0, hb));
    LM_TRY(h2d_2d(c, hb.A, hb.lda, A, n, n, n));
    LM_TRY(lm::reset_info(c));
    LM_TRY(lm::dgetrf_nopiv(c, n, hb.A, hb.lda, c.stream));
    LM_TRY(d2h_2d(c, LU, n, hb.A, hb.lda, n, n));
    int inf = 0;
    int r = lm::read_status(c, &inf);
    if (info) *info = inf;
    return r;
  });
}

int lm_cholesky_gaxpy_host(lm_ctx* ctx, int n, const double* A, double* G, int* info) {
  // choleskyGaxpy computes the same G as cholesky; on the device both are the
  // blocked right-looking factorisation
  return lm_cholesky_host(ctx, n, A, G, info);
}

int lm_matvec_host(lm_ctx* ctx, int m, int n, const double* A, const double* x, double* y) {
  return guarded(ctx, [&](Ctx& c) {
    if (m < 0 || n < 0 || (m > 0 && !y) || (m > 0 && n > 0 && (!A || !x))) return LM_ERR_ARG;
    if (m == 0) return LM_OK;
    const long long lda = rup(std::max(n, 1), 8);
    void* ws = nullptr;
    LM_TRY(lm::ctx_workspace(c, 3, sizeof(double) * ((size_t)m * lda + rup(std::max(n, 1), 8) + rup(m, 8)), &ws));
    double* dA = static_cast<double*>(ws);
    double* dx = dA + (size_t)m * lda;
    double* dy = dx + rup(std::max(n, 1), 8);
    LM_TRY(h2d_2d(c, dA, lda, A, n, m, n));
    if (n > 0) LM_CUDA_TRY(cudaMemcpyAsync(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream));
    LM_TRY(lm::dgemv_exact(m, n, dA, lda, dx, dy, c.stream));
    LM_CUDA_TRY(cudaMemcpyAsync(y, dy, sizeof(double) * m, cudaMemcpyDeviceToHost, c.stream));
    int r = lm::read_status(c, nullptr);
    return r < 0 ? r : LM_OK;
  });
}

int lm_norm_inf_host(lm_ctx* ctx, int m, int n, const double* A, double* result) {
  if (m < 0 || n < 0 || !result || (m > 0 && n > 0 && !A)) return LM_ERR_ARG;
  if (m == 0 || n == 0) {
    *result = 0.0;
    return LM_OK;
  }
  return guarded(ctx, [&](Ctx& c) {
    const long long lda = rup(n, 8);
    void* ws = nullptr;
    LM_TRY(lm::ctx_workspace(c, 3, sizeof(double) * ((size_t)m * lda + 8), &ws));
    double* dA = static_cast<double*>(ws);
    unsigned long long* d = reinterpret_cast<unsigned long long*>(dA + (size_t)m * lda);
    LM_TRY(h2d_2d(c, dA, lda, A, n, m, n));
    LM_TRY(lm::dnorm_inf_exact(m, n, dA, lda, d, c.stream));
    unsigned long long h = 0;
    LM_CUDA_TRY(cudaMemcpyAsync(&h, d, sizeof h, cudaMemcpyDeviceToHost, c.stream));
    LM_CUDA_TRY(cudaStreamSynchronize(c.stream));
    std::memcpy(result, &h, sizeof h);
    return LM_OK;
  });
}

int lm_tridiag_solve_host(lm_ctx* ctx, int n, const double* diag, const double* supdiag, const double* b,
                          double* x) {
  return guarded(ctx, [&](Ctx& c) {
    if (n < 0 || (n > 0 && (!diag || !b || !x || (n > 1 && !supdiag)))) return LM_ERR_ARG;
    if (n == 0) return LM_OK;
    const size_t nn = (size_t)rup(n, 8);
    void* ws = nullptr;
    LM_TRY(lm::ctx_workspace(c, 3, sizeof(double) * 4 * nn, &ws));
    double* d = static_cast<double*>(ws);
    double* sp = d + nn;
    double* rb = sp + nn;
    double* dx = rb + nn;
    void* scr = nullptr;
    LM_TRY(lm::ctx_workspace(c, 2, sizeof(double) * 8 * (size_t)n, &scr));
    LM_CUDA_TRY(cudaMemcpyAsync(d, diag, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream));
    if (n > 1) LM_CUDA_TRY(cudaMemcpyAsync(sp, supdiag, sizeof(double) * (n - 1), cudaMemcpyHostToDevice, c.stream));
    LM_CUDA_TRY(cudaMemcpyAsync(rb, b, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream));
    LM_TRY(lm::dtridiag_pcr(n, d, sp, rb, dx, static_cast<double*>(scr), c.stream));
    LM_CUDA_TRY(cudaMemcpyAsync(x, dx, sizeof(double) * n, cudaMemcpyDeviceToHost, c.stream));
    int r = lm::read_status(c, nullptr);
    return r < 0 ? r : LM_OK;
  });
}

int lm_det_host(lm_ctx* ctx, int n, const double* A, double* det) {
  if (!det || n < 0) return LM_ERR_ARG;
  if (n == 0) {
    *det = 1.0;
    return LM_OK;
  }
  std::vector<double> lu((size_t)n * n);
  std::vector<int> perm(n);
  int info = 0;
  int r = lm_lu_host(ctx, n, A, lu.data(), perm.data(), &info);
  if (r < 0) return r;
  // det (LU.hs:534-545): left fold of the diagonal from 1, then the sign of
  // the permutation counted as in countSwaps (LU.hs:548-557).
  double prod = 1.0;
  for (int i = 0; i < n; ++i) prod = prod * lu[(size_t)i * n + i];
  int swaps = 0;
  for (int i = 0; i < n; ++i) {
    if (perm[i] == i) continue;
    for (int j = i + 1; j < n; ++j)
      if (perm[j] == i) {
        perm[j] = perm[i];
        break;
      }
    ++swaps;
  }
  *det = (swaps % 2 == 0) ? prod : -prod;
  return LM_OK;
}

}  // extern "C"

// ---- batched uneven-size solves ------------------------------------------------
struct lm_batch {
  lm_ctx* ctx = nullptr;
  long long id = 0;  // unique per plan: keys its captured graphs (a freed plan's address can be reused)
  int count = 0, prec = 0;
  int nmax = 0, rmax = 0, nbmax = 0;
  std::vector<long long> a_off, b_off;
  lm::BatchItem* d_items = nullptr;
  double* d_F = nullptr;
  int* d_ipiv = nullptr;
  int* d_info = nullptr;
  int* d_iters = nullptr;
  double* d_berr = nullptr;
  int* d_ticket = nullptr;
  double *hA = nullptr, *hB = nullptr, *hX = nullptr;  // device buffers of the host-buffer entry point
  size_t smem = 0;
  int grid = 0;
};

namespace {

std::atomic<long long> g_plan_ids{0};

// Drop the captured graphs of one plan (their kernels hold its buffers).
void evict_graphs(Ctx& c, const std::string& prefix) {
  for (auto it = c.gcache.begin(); it != c.gcache.end();) {
    if (it->key.compare(0, prefix.size(), prefix) == 0) {
      if (it->exec) cudaGraphExecDestroy(it->exec);
      it = c.gcache.erase(it);
    } else {
      ++it;
    }
  }
}

void batch_free(lm_batch* p) {
  cudaFree(p->d_items);
  cudaFree(p->d_F);
  cudaFree(p->d_ipiv);
  cudaFree(p->d_info);
  cudaFree(p->d_iters);
  cudaFree(p->d_berr);
  cudaFree(p->d_ticket);
  cudaFree(p->hA);
  cudaFree(p->hB);
  cudaFree(p->hX);
}

int batch_build(Ctx& c, lm_batch* p, int count, const int* n, const int* nrhs, const int* kind, int prec) {
  p->count = count;
  p->prec = prec;
  p->a_off.assign(count + 1, 0);
  p->b_off.assign(count + 1, 0);
  std::vector<long long> p_off(count + 1, 0);
  std::vector<lm::BatchItem> items(count);
  for (int i = 0; i < count; ++i) {
    if (n[i] < 0 || n[i] > lm::BatchLimits::kMaxN || nrhs[i] < 0 || nrhs[i] > lm::BatchLimits::kMaxRhs ||
        (kind[i] != LM_BATCH_GENERAL && kind[i] != LM_BATCH_SPD)) {
      lm::set_last_error("batch instance " + std::to_string(i) + ": n must be in [0, 256], nrhs in [0, 16]");
      return LM_ERR_ARG;
    }
    p->a_off[i + 1] = p->a_off[i] + (long long)n[i] * n[i];
    p->b_off[i + 1] = p->b_off[i] + (long long)n[i] * nrhs[i];
    p_off[i + 1] = p_off[i] + n[i];
    lm::BatchItem& it = items[i];
    it.a_off = p->a_off[i];
    it.b_off = p->b_off[i];
    it.x_off = p->b_off[i];
    it.f_off = p->a_off[i];
    it.p_off = p_off[i];
    it.n = n[i];
    it.nrhs = nrhs[i];
    it.kind = kind[i];
    it.nb = c.batch_nb[prec][lm::batch_bucket(std::max(n[i], 1))];
    it.index = i;
    p->nmax = std::max(p->nmax, n[i]);
    p->rmax = std::max(p->rmax, nrhs[i]);
    p->nbmax = std::max(p->nbmax, it.nb);
  }
  p->nmax = std::max(p->nmax, 1);
  p->rmax = std::max(p->rmax, 1);
  p->nbmax = std::max(p->nbmax, 1);
  // longest processing time first: the largest instances are taken first so
  // the small ones fill in behind them
  auto cost = [](const lm::BatchItem& it) {
    const double nn = it.n;
    return (it.kind == LM_BATCH_GENERAL ? 2.0 / 3.0 : 1.0 / 3.0) * nn * nn * nn + 2.0 * nn * nn * it.nrhs +
           64.0 * nn * nn;
  };
  std::stable_sort(items.begin(), items.end(),
                   [&](const lm::BatchItem& a, const lm::BatchItem& b) { return cost(a) > cost(b); });
  const size_t ni = std::max(count, 1);
  LM_CUDA_TRY(cudaMalloc(&p->d_items, sizeof(lm::BatchItem) * ni));
  LM_CUDA_TRY(cudaMalloc(&p->d_F, sizeof(double) * std::max<long long>(p->a_off[count], 1)));
  LM_CUDA_TRY(cudaMalloc(&p->d_ipiv, sizeof(int) * std::max<long long>(p_off[count], 1)));
  LM_CUDA_TRY(cudaMalloc(&p->d_info, sizeof(int) * ni));
  LM_CUDA_TRY(cudaMalloc(&p->d_iters, sizeof(int) * ni));
  LM_CUDA_TRY(cudaMalloc(&p->d_berr, sizeof(double) * ni));
  LM_CUDA_TRY(cudaMalloc(&p->d_ticket, sizeof(int) * 4));
  if (count > 0)
    LM_CUDA_TRY(cudaMemcpy(p->d_items, items.data(), sizeof(lm::BatchItem) * count, cudaMemcpyHostToDevice));
  LM_CUDA_TRY(cudaMemset(p->d_info, 0, sizeof(int) * ni));
  LM_CUDA_TRY(cudaMemset(p->d_iters, 0, sizeof(int) * ni));
  LM_CUDA_TRY(cudaMemset(p->d_berr, 0, sizeof(double) * ni));
  p->smem = lm::batch_smem_bytes(p->nmax, p->rmax, p->nbmax);
  if (p->smem > 200 * 1024) {
    lm::set_last_error("batch: shared memory of the largest instance exceeds 200 KB");
    return LM_ERR_UNSUPPORTED;
  }
  int per_sm = 0;
  LM_TRY(lm::batch_occupancy(p->smem, &per_sm));
  per_sm = std::max(per_sm, 1);
  p->grid = std::max(1, std::min(count, per_sm * c.num_sms));
  return LM_OK;
}

int batch_run(Ctx& c, lm_batch* p, const double* A, const double* B, double* X, double tol, int max_iter) {
  if (p->count == 0) return LM_OK;
  lm::BatchArgs g;
  g.items = p->d_items;
  g.count = p->count;
  g.prec = p->prec;
  g.nmax = p->nmax;
  g.rmax = p->rmax;
  g.nbmax = p->nbmax;
  g.A = A;
  g.B = B;
  g.X = X;
  g.F = p->d_F;
  g.ipiv = p->d_ipiv;
  g.info = p->d_info;
  g.iters = p->d_iters;
  g.berr = p->d_berr;
  g.ticket = p->d_ticket;
  g.tol = tol;
  g.max_iter = max_iter;
  const std::string key = lm::gkey("batch", {p->id, (long long)A, (long long)B, (long long)X,
                                             (long long)(tol * 1e30), max_iter});
  return lm::run_graphed(c, key, [&](cudaStream_t s) { return lm::batch_launch(g, p->grid, p->smem, s); });
}

// Seeded synthetic instances for the tuner: general ones uniform[-1,1], SPD
// ones (R + R^T)/2 + n I (diagonally dominant).
uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
double unif(uint64_t& s) { return (double)(splitmix(s) >> 11) * (2.0 / 9007199254740992.0) - 1.0; }

}  // namespace

extern "C" {

int lm_batch_create(lm_ctx* ctx, lm_batch** plan, int count, const int* n, const int* nrhs, const int* kind,
                    int precision) {
  if (!plan) return LM_ERR_ARG;
  *plan = nullptr;
  return guarded(ctx, [&](Ctx& c) {
    if (count < 0 || (count > 0 && (!n || !nrhs || !kind))) return LM_ERR_ARG;
    if (precision != LM_PREC_FP64 && precision != LM_PREC_FP32_IR) return LM_ERR_ARG;
    lm_batch* p = new lm_batch;
    p->ctx = ctx;
    p->id = ++g_plan_ids;
    const int r = batch_build(c, p, count, n, nrhs, kind, precision);
    if (r != LM_OK) {
      batch_free(p);
      delete p;
      return r;
    }
    *plan = p;
    return LM_OK;
  });
}

int lm_batch_destroy(lm_batch* plan) {
  if (!plan) return LM_OK;
  return guarded(plan->ctx, [&](Ctx& c) {
    cudaStreamSynchronize(c.stream);
    evict_graphs(c, lm::gkey("batch", {plan->id}) + ",");
    batch_free(plan);
    delete plan;
    return LM_OK;
  });
}

int lm_batch_offsets(const lm_batch* plan, long long* a_off, long long* b_off) {
  if (!plan) return LM_ERR_ARG;
  if (a_off) std::copy(plan->a_off.begin(), plan->a_off.end(), a_off);
  if (b_off) std::copy(plan->b_off.begin(), plan->b_off.end(), b_off);
  return LM_OK;
}

int lm_batch_solve(lm_batch* plan, const double* A, const double* B, double* X, double tol, int max_iter) {
  if (!plan) return LM_ERR_ARG;
  return guarded(plan->ctx, [&](Ctx& c) {
    if (plan->count > 0 && (!A || !B || !X)) return LM_ERR_ARG;
    if (max_iter < 1) max_iter = 1;
    return batch_run(c, plan, A, B, X, tol, max_iter);
  });
}

int lm_batch_results(lm_batch* plan, int* info, int* iters, double* berr) {
  if (!plan) return LM_ERR_ARG;
  return guarded(plan->ctx, [&](Ctx& c) {
    const size_t k = plan->count;
    if (k == 0) return LM_OK;
    if (info) LM_CUDA_TRY(cudaMemcpyAsync(info, plan->d_info, sizeof(int) * k, cudaMemcpyDeviceToHost, c.stream));
    if (iters)
      LM_CUDA_TRY(cudaMemcpyAsync(iters, plan->d_iters, sizeof(int) * k, cudaMemcpyDeviceToHost, c.stream));
    if (berr)
      LM_CUDA_TRY(cudaMemcpyAsync(berr, plan->d_berr, sizeof(double) * k, cudaMemcpyDeviceToHost, c.stream));
    LM_CUDA_TRY(cudaStreamSynchronize(c.stream));
    int h[2] = {0, 0};
    LM_CUDA_TRY(cudaMemcpy(h, c.d_status, sizeof(h), cudaMemcpyDeviceToHost));
    return h[0] != 0 ? LM_ERR_TIMEOUT : LM_OK;
  });
}

int lm_batch_factors(const lm_batch* plan, const double** F, const int** ipiv) {
  if (!plan) return LM_ERR_ARG;
  if (F) *F = plan->d_F;
  if (ipiv) *ipiv = plan->d_ipiv;
  return LM_OK;
}

int lm_batch_solve_host(lm_batch* plan, const double* A, const double* B, double* X, double tol, int max_iter) {
  if (!plan) return LM_ERR_ARG;
  return guarded(plan->ctx, [&](Ctx& c) {
    const long long na = plan->a_off.back(), nbv = plan->b_off.back();
    if (plan->count == 0) return LM_OK;
    if (!A || !B || !X) return LM_ERR_ARG;
    if (!plan->hA) {
      LM_CUDA_TRY(cudaMalloc(&plan->hA, sizeof(double) * std::max(na, 1LL)));
      LM_CUDA_TRY(cudaMalloc(&plan->hB, sizeof(double) * std::max(nbv, 1LL)));
      LM_CUDA_TRY(cudaMalloc(&plan->hX, sizeof(double) * std::max(nbv, 1LL)));
    }
    LM_CUDA_TRY(cudaMemcpyAsync(plan->hA, A, sizeof(double) * na, cudaMemcpyHostToDevice, c.stream));
    LM_CUDA_TRY(cudaMemcpyAsync(plan->hB, B, sizeof(double) * nbv, cudaMemcpyHostToDevice, c.stream));
    LM_TRY(batch_run(c, plan, plan->hA, plan->hB, plan->hX, tol, std::max(max_iter, 1)));
    LM_CUDA_TRY(cudaMemcpyAsync(X, plan->hX, sizeof(double) * nbv, cudaMemcpyDeviceToHost, c.stream));
    LM_CUDA_TRY(cudaStreamSynchronize(c.stream));
    return LM_OK;
  });
}

int lm_batch_tune_get(lm_ctx* ctx, int* nb) {
  if (!nb) return LM_ERR_ARG;
  return guarded(ctx, [&](Ctx& c) {
    std::memcpy(nb, c.batch_nb, sizeof(c.batch_nb));
    return LM_OK;
  });
}

int lm_batch_tune_set(lm_ctx* ctx, const int* nb) {
  if (!nb) return LM_ERR_ARG;
  for (int i = 0; i < 2 * lm::BatchLimits::kBuckets; ++i)
    if (nb[i] != 8 && nb[i] != 16 && nb[i] != 32) return LM_ERR_ARG;
  return guarded(ctx, [&](Ctx& c) {
    std::memcpy(c.batch_nb, nb, sizeof(c.batch_nb));
    return LM_OK;
  });
}

int lm_batch_tune(lm_ctx* ctx, int precision, const char* path) {
  if (!ctx || (precision != LM_PREC_FP64 && precision != LM_PREC_FP32_IR)) return LM_ERR_ARG;
  const int lo[4] = {1, 33, 65, 129}, hi[4] = {32, 64, 128, 256};
  const int cands[3] = {8, 16, 32};
  double best_ms[4] = {0, 0, 0, 0};
  int num_sms = 0;
  {
    int r = guarded(ctx, [&](Ctx& c) { num_sms = c.num_sms; return LM_OK; });
    if (r) return r;
  }
  for (int b = 0; b < 4; ++b) {
    const int count = 4 * num_sms;
    std::vector<int> n(count), nrhs(count), kind(count);
    uint64_t seed = 0x5eed0000ULL + b;
    for (int i = 0; i < count; ++i) {
      n[i] = lo[b] + (int)(splitmix(seed) % (uint64_t)(hi[b] - lo[b] + 1));
      nrhs[i] = 1 + (int)(splitmix(seed) % 16);
      kind[i] = i & 1;
    }
    std::vector<long long> ao(count + 1), bo(count + 1);
    for (int i = 0; i < count; ++i) {
      ao[i + 1] = ao[i] + (long long)n[i] * n[i];
      bo[i + 1] = bo[i] + (long long)n[i] * nrhs[i];
    }
    std::vector<double> A(ao[count]), B(bo[count]);
    for (int i = 0; i < count; ++i) {
      double* a = A.data() + ao[i];
      const int m = n[i];
      for (long long e = 0; e < (long long)m * m; ++e) a[e] = unif(seed);
      if (kind[i] == LM_BATCH_SPD)
        for (int r = 0; r < m; ++r) {
          for (int q = 0; q < r; ++q) a[(long long)r * m + q] = a[(long long)q * m + r] = 0.5 * (a[(long long)r * m + q] + a[(long long)q * m + r]);
          a[(long long)r * m + r] += m;
        }
    }
    for (auto& v : B) v = unif(seed);
    double *dA = nullptr, *dB = nullptr, *dX = nullptr;
    if (cudaMalloc(&dA, sizeof(double) * A.size()) != cudaSuccess || cudaMalloc(&dB, sizeof(double) * B.size()) != cudaSuccess ||
        cudaMalloc(&dX, sizeof(double) * B.size()) != cudaSuccess) {
      cudaFree(dA); cudaFree(dB); cudaFree(dX);
      return LM_ERR_NOMEM;
    }
    cudaMemcpy(dA, A.data(), sizeof(double) * A.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(dB, B.data(), sizeof(double) * B.size(), cudaMemcpyHostToDevice);
    int keep = 16;
    double keep_ms = 1e30;
    int saved[2][4];
    lm_batch_tune_get(ctx, &saved[0][0]);
    int rc = LM_OK;
    for (int nb : cands) {
      int t[2][4];
      std::memcpy(t, saved, sizeof(t));
      t[precision][b] = nb;
      lm_batch_tune_set(ctx, &t[0][0]);
      lm_batch* plan = nullptr;
      rc = lm_batch_create(ctx, &plan, count, n.data(), nrhs.data(), kind.data(), precision);
      if (rc) break;
      float ms = 0.f;
      cudaStream_t st = (cudaStream_t)lm_ctx_get_stream(ctx);
      cudaEvent_t e0, e1;
      cudaEventCreate(&e0);
      cudaEventCreate(&e1);
      for (int w = 0; w < 2 && !rc; ++w) rc = lm_batch_solve(plan, dA, dB, dX, 0.0, 10);
      float best = 1e30f;
      for (int rep = 0; rep < 3 && !rc; ++rep) {
        cudaEventRecord(e0, st);
        rc = lm_batch_solve(plan, dA, dB, dX, 0.0, 10);
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        best = std::min(best, ms);
      }
      if (!rc) rc = lm_batch_results(plan, nullptr, nullptr, nullptr);
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      lm_batch_destroy(plan);
      if (rc) break;
      if (best < keep_ms) { keep_ms = best; keep = nb; }
    }
    cudaFree(dA); cudaFree(dB); cudaFree(dX);
    saved[precision][b] = keep;
    lm_batch_tune_set(ctx, &saved[0][0]);
    if (rc) return rc;
    best_ms[b] = keep_ms;
  }
  if (path) {
    FILE* f = std::fopen(path, "w");
    if (!f) return LM_ERR_ARG;
    int t[2][4];
    lm_batch_tune_get(ctx, &t[0][0]);
    std::fprintf(f, "{\"precision\": %d, \"buckets\": [32, 64, 128, 256], \"nb\": [[%d, %d, %d, %d], [%d, %d, %d, %d]], "
                    "\"best_ms\": [%.4f, %.4f, %.4f, %.4f]}\n",
                 precision, t[0][0], t[0][1], t[0][2], t[0][3], t[1][0], t[1][1], t[1][2], t[1][3], best_ms[0],
                 best_ms[1], best_ms[2], best_ms[3]);
    std::fclose(f);
  }
  return LM_OK;
}

}  // extern "C"
