// amg_runtime.cu -- non-template host runtime: errors, device facts, plans, graph
// construction (conditional WHILE node) and execution.
#include <cmath>
#include <tuple>

#include "amg_runtime.cuh"

namespace amg {

thread_local std::string t_err;

[[noreturn]] void fail(amg_status st, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  throw Error{st, std::string(buf)};
}

DevInfo dev_info() {
  static std::mutex m;
  static std::map<int, DevInfo> cache;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(m);
  auto it = cache.find(dev);
  if (it != cache.end()) return it->second;
  DevInfo d;
  CK(cudaDeviceGetAttribute(&d.nsm, cudaDevAttrMultiProcessorCount, dev));
  d.max_ctas = d.nsm * (2048 / kBlock);
  cache[dev] = d;
  return d;
}

bool fuse2_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("AMG_FUSE2");
    return !(e && e[0] == '0');
  }();
  return on;
}

double fuse2_chain() {
  static const double v = [] {
    const char* e = std::getenv("AMG_FUSE2_CHAIN");
    const double x = e ? atof(e) : 400.0;
    return x >= 0.0 ? x : 400.0;
  }();
  return v;
}

double fuse2_work() {
  static const double v = [] {
    const char* e = std::getenv("AMG_FUSE2_WORK");
    const double x = e ? atof(e) : 5e5;
    return x >= 0.0 ? x : 5e5;
  }();
  return v;
}

int fuse2_rows() {
  static const int v = [] {
    const char* e = std::getenv("AMG_FUSE2_ROWS");
    const int x = e ? atoi(e) : 20000;
    return x >= 0 ? x : 20000;
  }();
  return v;
}

bool nvtx_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("AMG_NVTX");
    return e && e[0] == '1';
  }();
  return on;
}

bool pdl_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("AMG_PDL");
    return !(e && e[0] == '0');
  }();
  return on;
}

namespace {
std::mutex g_tune_mu;
std::map<std::tuple<const void*, int64_t, int, int, int, const void*>, int> g_tune;

// Tuning file (AMG_TUNE_FILE=path): one decision per line, "op-type nnz k es kv G".  Read
// once; a decision found there is used without timing, and new decisions are appended.
// The key has no pointers, so a second process (a profiler run, a service restart) reuses
// the first one's layouts; two matrices with the same op, nnz, k and types share a line.
using FileKey = std::tuple<std::string, int64_t, int, int, int>;
std::map<FileKey, int> g_tune_file;
bool g_tune_file_loaded = false;

const char* tune_file_path() {
  const char* p = std::getenv("AMG_TUNE_FILE");
  return (p && p[0]) ? p : nullptr;
}

// A lanes-per-row code the launchers accept: k == 1: G in {1, 2, 4, 8, 16, 32}; k > 1: a
// plain code G in {4, 8, 16, 32}, or a lean / wide / pipelined code (kLeanCode / kWideCode /
// kPipeCode + G) with G
// in {1, 2, 4, 8, 16, 32}.  A stale or edited tuning-file line with any other value would
// otherwise reach a launcher that maps it to a layout covering fewer columns than k.
bool valid_layout_code(int g, int k) {
  auto lanes = [](int v) { return v == 1 || v == 2 || v == 4 || v == 8 || v == 16 || v == 32; };
  if (k == 1) return lanes(g);
  if (g >= kPipe2Code) return pipe_lanes(g - kPipe2Code);
  if (g >= kPipeCode) return pipe_lanes(g - kPipeCode);
  if (g >= kWideCode) return lanes(g - kWideCode);
  if (g >= kLeanCode) return lanes(g - kLeanCode);
  return g == 4 || g == 8 || g == 16 || g == 32;
}

void load_tune_file() {  // g_tune_mu held
  if (g_tune_file_loaded) return;
  g_tune_file_loaded = true;
  const char* path = tune_file_path();
  if (!path) return;
  FILE* f = fopen(path, "r");
  if (!f) return;
  char name[512];
  long long nnz;
  int k, es, kv, g;
  while (fscanf(f, "%511s %lld %d %d %d %d", name, &nnz, &k, &es, &kv, &g) == 6)
    if (valid_layout_code(g, k)) g_tune_file[FileKey(name, nnz, k, es, kv)] = g;  // others: ignored
  fclose(f);
}
}  // namespace

int tuned_g(const void* rowptr, int64_t nnz, int k, int es, int kv, const void* tag) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  const auto key = std::make_tuple(rowptr, nnz, k, es, kv, tag);
  auto it = g_tune.find(key);
  if (it != g_tune.end()) return it->second;
  load_tune_file();
  if (!g_tune_file.empty()) {
    auto ft = g_tune_file.find(FileKey(static_cast<const OpTag*>(tag)->name, nnz, k, es, kv));
    if (ft != g_tune_file.end()) {
      g_tune[key] = ft->second;
      return ft->second;
    }
  }
  return 0;
}

void set_tuned_g(const void* rowptr, int64_t nnz, int k, int es, int kv, const void* tag, int g,
                 bool final) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[std::make_tuple(rowptr, nnz, k, es, kv, tag)] = g;
  if (!final) return;
  const char* path = tune_file_path();
  if (!path) return;
  load_tune_file();
  const char* name = static_cast<const OpTag*>(tag)->name;
  const FileKey fk(name, nnz, k, es, kv);
  if (g_tune_file.count(fk)) return;
  g_tune_file[fk] = g;
  if (FILE* f = fopen(path, "a")) {
    fprintf(f, "%s %lld %d %d %d %d\n", name, (long long)nnz, k, es, kv, g);
    fclose(f);
  }
}

bool tuning_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("AMG_TUNE");
    return !(e && e[0] == '0');
  }();
  return on;
}

int resident_ctas(const void* fn, size_t smem) {
  static std::mutex m;
  static std::map<std::pair<const void*, size_t>, int> cache;
  std::lock_guard<std::mutex> lk(m);
  auto key = std::make_pair(fn, smem);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int nb = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, kBlock, smem));
  nb = std::max(1, std::min(nb, 2048 / kBlock));
  cache[key] = nb;
  return nb;
}

int carveout_pct(const void* fn, size_t smem) {
  static const bool on = [] {
    const char* e = std::getenv("AMG_CARVEOUT");
    return !(e && e[0] == '0');
  }();
  if (!on) return -1;
  static std::mutex m;
  static std::map<std::pair<const void*, size_t>, int> cache;
  {
    std::lock_guard<std::mutex> lk(m);
    auto it = cache.find(std::make_pair(fn, smem));
    if (it != cache.end()) return it->second;
  }
  const int per = resident_ctas(fn, smem);  // with the largest shared-memory share
  cudaFuncAttributes fa{};
  CK(cudaFuncGetAttributes(&fa, fn));
  int dev = 0, sm_bytes = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sm_bytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
  const double need = double(per) * (double(smem) + double(fa.sharedSizeBytes) + 1024.0);
  int pct = sm_bytes > 0 ? int(std::ceil(100.0 * need / double(sm_bytes))) + 2 : -1;
  if (pct > 100) pct = 100;
  std::lock_guard<std::mutex> lk(m);
  cache[std::make_pair(fn, smem)] = pct;
  return pct;
}

void check_csr(const amg_csr& c, const char* what, int lvl) {
  if (c.n_rows < 0 || c.n_cols < 0 || c.nnz < 0)
    fail(AMG_ERR_INVALID_ARG, "level %d %s: negative size", lvl, what);
  if (c.nnz > INT32_MAX) fail(AMG_ERR_UNSUPPORTED, "level %d %s: nnz exceeds int32", lvl, what);
  if (c.n_rows > 0 && (!c.rowptr || (c.nnz > 0 && !c.col)))
    fail(AMG_ERR_INVALID_ARG, "level %d %s: null rowptr/col", lvl, what);
  if (c.nnz > 0 && !c.val64 && !c.val32)
    fail(AMG_ERR_INVALID_ARG, "level %d %s: no values", lvl, what);
}

// ------------------------------------------------------------------ CSR structure check
// Status of the last structure check: [0] error bits, [1] the smallest offending row (bits
// 1, 2, 4) or nonzero (bit 8).  One check runs at a time (g_check_mu).
static __device__ int g_csr_status[2];

enum : int { kBadRow0 = 1, kBadOrder = 2, kBadEnd = 4, kBadCol = 8 };

// Reads rowptr[0 .. n_rows] and col[0 .. nnz), the extents the descriptor declares.
__global__ void csr_check_kernel(const int* __restrict__ rowptr, const int* __restrict__ col, int n_rows,
                                 int n_cols, long long nnz) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  for (long long i = tid; i < n_rows; i += nth) {
    const int a = rowptr[i], b = rowptr[i + 1];
    int bad = 0;
    if (i == 0 && a != 0) bad |= kBadRow0;
    if (b < a) bad |= kBadOrder;
    if (i == n_rows - 1 && (long long)b != nnz) bad |= kBadEnd;
    if (bad) {
      atomicOr(&g_csr_status[0], bad);
      atomicMin(&g_csr_status[1], int(i));
    }
  }
  for (long long e = tid; e < nnz; e += nth) {
    const int c = col[e];
    if (c < 0 || c >= n_cols) {
      atomicOr(&g_csr_status[0], kBadCol);
      atomicMin(&g_csr_status[1], int(e));
    }
  }
}

namespace {
std::mutex g_check_mu;
// Structures already checked, by (rowptr, col, n_rows, n_cols, nnz): the stand-alone kernels
// check a matrix the first time they see it, not on every call.
std::map<std::tuple<const void*, const void*, int, int, int64_t>, bool> g_checked;
}  // namespace

void validate_csr(const amg_csr& c, const char* what, int lvl, cudaStream_t s, bool once) {
  check_csr(c, what, lvl);
  if (c.n_rows == 0) return;
  std::lock_guard<std::mutex> lk(g_check_mu);
  const auto key = std::make_tuple((const void*)c.rowptr, (const void*)c.col, c.n_rows, c.n_cols, c.nnz);
  if (once && g_checked.count(key)) return;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(s, &cap));
  if (cap != cudaStreamCaptureStatusNone) return;  // a capture cannot wait for the verdict
  const int init[2] = {0, INT32_MAX};
  CK(cudaMemcpyToSymbolAsync(g_csr_status, init, sizeof(init), 0, cudaMemcpyHostToDevice, s));
  const long long work = std::max<long long>(c.n_rows, c.nnz);
  const int grid = int(std::max<long long>(1, std::min<long long>((work + 255) / 256, dev_info().max_ctas)));
  csr_check_kernel<<<grid, 256, 0, s>>>(c.rowptr, c.col, c.n_rows, c.n_cols, (long long)c.nnz);
  CK_LAUNCH();
  int st[2] = {0, 0};
  CK(cudaMemcpyFromSymbolAsync(st, g_csr_status, sizeof(st), 0, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (st[0] & kBadRow0) fail(AMG_ERR_BAD_MATRIX, "level %d %s: rowptr[0] is not 0", lvl, what);
  if (st[0] & kBadOrder)
    fail(AMG_ERR_BAD_MATRIX, "level %d %s: rowptr decreases (first at row %d)", lvl, what, st[1]);
  if (st[0] & kBadEnd)
    fail(AMG_ERR_BAD_MATRIX, "level %d %s: rowptr[n_rows] differs from nnz = %lld", lvl, what, (long long)c.nnz);
  if (st[0] & kBadCol)
    fail(AMG_ERR_BAD_MATRIX, "level %d %s: column index out of [0, %d) (first at nonzero %d)", lvl, what,
         c.n_cols, st[1]);
  if (g_checked.size() > 4096) g_checked.clear();
  g_checked[key] = true;
}

// Loop guard: ends each body of the device while-loop.  Sets the loop condition from
// the stop flag and a hard trip bound, so the loop always terminates.
__global__ void loop_guard_kernel(int* stop, int* gcount, int gmax, cudaGraphConditionalHandle h) {
  count_launch();
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    const int g = ++(*gcount);
    const int cont = (*stop == 0) && (g < gmax);
    if (!cont) *stop = 1;
    cudaGraphSetConditional(h, cont ? 1u : 0u);
  }
}

// Host-loop variant of the guard (no conditional node).
__global__ void loop_guard_host_kernel(int* stop, int* gcount, int gmax) {
  count_launch();
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    const int g = ++(*gcount);
    if (!((*stop == 0) && (g < gmax))) *stop = 1;
  }
}

// ------------------------------------------------------------------ plans
static std::string plan_key(int prec, int k, cudaStream_t s) {
  char buf[96];
  snprintf(buf, sizeof(buf), "%d/%d/%p", prec, k, (void*)s);
  return buf;
}

int max_plans() {
  static const int v = [] {
    const char* e = std::getenv("AMG_MAX_PLANS");
    const int x = e ? atoi(e) : 16;
    return x >= 2 ? x : (e ? 2 : 16);
  }();
  return v;
}

Plan* get_plan(amg_hierarchy* h, int prec, int k, cudaStream_t s) {
  const std::string key = plan_key(prec, k, s);
  auto it = h->plans.find(key);
  if (it != h->plans.end()) {
    it->second->last_use = ++h->use_clock;
    return it->second.get();
  }
  if (int(h->plans.size()) >= max_plans()) {  // free the least recently requested plan
    auto lru = h->plans.begin();
    for (auto p = h->plans.begin(); p != h->plans.end(); ++p)
      if (p->second->last_use < lru->second->last_use) lru = p;
    CK(cudaDeviceSynchronize());
    h->plans.erase(lru);
  }
  auto pl = std::make_unique<Plan>();
  pl->last_use = ++h->use_clock;
  pl->prec = prec;
  pl->k = k;
  pl->stream = s;
  CK(cudaGetDevice(&pl->dev));
  pl->csize = (prec == AMG_PREC_F64) ? 8 : 4;
  const size_t osize = (prec == AMG_PREC_F32) ? 4 : 8;
  const int L = int(h->levels.size());
  for (int l = 0; l < L; ++l) {
    const size_t n = size_t(h->levels[l].A.n_rows) * k;
    pl->X.push_back(pl->alloc(n * pl->csize));
    pl->B.push_back(pl->alloc(n * pl->csize));
    pl->W1.push_back(pl->alloc(n * pl->csize));
    pl->W2.push_back(pl->alloc(n * pl->csize));
  }
  const size_t n0 = size_t(h->levels[0].A.n_rows) * k;
  pl->r_out = pl->alloc(n0 * osize);
  pl->p_out = pl->alloc(n0 * osize);
  pl->q_out = pl->alloc(n0 * osize);
  pl->dscal = static_cast<double*>(pl->alloc(sizeof(double) * 7 * k));
  pl->iscal = static_cast<int*>(pl->alloc(sizeof(int) * (2 * k + 4)));
  CK(cudaMemset(pl->iscal, 0, sizeof(int) * (2 * k + 4)));
  pl->partials = static_cast<double*>(
      pl->alloc(sizeof(double) * size_t(dev_info().max_ctas + kRedGroups) * k));
  pl->counter = static_cast<unsigned*>(pl->alloc(sizeof(unsigned) * (1 + kRedGroups)));
  CK(cudaMemset(pl->counter, 0, sizeof(unsigned) * (1 + kRedGroups)));
  CK(cudaHostAlloc(reinterpret_cast<void**>(&pl->h_stop), sizeof(int), cudaHostAllocDefault));
  pl->bar = static_cast<unsigned*>(pl->alloc(sizeof(unsigned) * kBarWords));
  CK(cudaMemset(pl->bar, 0, sizeof(unsigned) * kBarWords));
  Plan* raw = pl.get();
  h->plans[key] = std::move(pl);
  return raw;
}

// ------------------------------------------------------------------ execution
enum ExecMode { EXEC_GRAPH = 0, EXEC_HOSTLOOP = 1, EXEC_EAGER = 2 };

static ExecMode exec_mode() {
  const char* e = std::getenv("AMG_EXEC");
  if (!e) return EXEC_GRAPH;
  if (!strcmp(e, "hostloop")) return EXEC_HOSTLOOP;
  if (!strcmp(e, "eager")) return EXEC_EAGER;
  return EXEC_GRAPH;
}

// A private stream for stream capture (the caller's stream may be the legacy default
// stream, which cannot be captured).
static cudaStream_t capture_stream() {
  static thread_local std::map<int, cudaStream_t> streams;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  auto it = streams.find(dev);
  if (it != streams.end()) return it->second;
  cudaStream_t s;
  CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  streams[dev] = s;
  return s;
}

template <class F>
static cudaGraph_t capture(cudaGraph_t into, const cudaGraphNode_t* deps, size_t ndeps, F&& f) {
  cudaStream_t cs = capture_stream();
  CK(cudaStreamBeginCaptureToGraph(cs, into, deps, nullptr, ndeps, cudaStreamCaptureModeThreadLocal));
  try {
    f(cs);
  } catch (...) {
    cudaGraph_t junk = into;
    cudaStreamEndCapture(cs, &junk);
    throw;
  }
  cudaGraph_t out = into;
  CK(cudaStreamEndCapture(cs, &out));
  return out;
}

static std::vector<cudaGraphNode_t> sinks(cudaGraph_t g) {
  size_t n = 0;
  CK(cudaGraphGetNodes(g, nullptr, &n));
  std::vector<cudaGraphNode_t> nodes(n), out;
  if (n) CK(cudaGraphGetNodes(g, nodes.data(), &n));
  for (auto nd : nodes) {
    size_t d = 0;
    CK(cudaGraphNodeGetDependentNodes(nd, nullptr, &d));
    if (d == 0) out.push_back(nd);
  }
  return out;
}

static int64_t count_nodes(cudaGraph_t g) {
  size_t n = 0;
  CK(cudaGraphGetNodes(g, nullptr, &n));
  return int64_t(n);
}


// Build (or fetch) and run prologue; while(any column active) body; epilogue.
void run_loop(Plan* pl, const std::string& key, cudaStream_t user, const Emit& prologue,
                     const Emit& body, const Emit& epilogue, bool has_loop, int gmax) {
  const ExecMode mode = exec_mode();
  if (mode == EXEC_EAGER) {
    CK(cudaMemsetAsync(pl->bar, 0, sizeof(unsigned) * kBarWords, user));
    prologue(user);
    if (has_loop) {
      for (int trip = 0;; ++trip) {
        body(user);
        launch(loop_guard_host_kernel, 1, 32, 0, user, pl->stop(), pl->gcount(), gmax);
        CK_LAUNCH();
        CK(cudaMemcpyAsync(pl->h_stop, pl->stop(), sizeof(int), cudaMemcpyDeviceToHost, user));
        CK(cudaStreamSynchronize(user));
        if (*pl->h_stop) break;
      }
    }
    epilogue(user);
    CK_LAUNCH();
    return;
  }
  // graph cache lookup (LRU of 8)
  GraphEntry* ge = nullptr;
  for (auto it = pl->graphs.begin(); it != pl->graphs.end(); ++it) {
    if (it->first == key) {
      pl->graphs.splice(pl->graphs.begin(), pl->graphs, it);
      ge = pl->graphs.front().second.get();
      break;
    }
  }
  if (!ge) {
    auto e = std::make_unique<GraphEntry>();
    if (mode == EXEC_GRAPH || !has_loop) {
      cudaGraph_t g;
      CK(cudaGraphCreate(&g, 0));
      e->graph = g;
      capture(g, nullptr, 0, prologue);
      if (has_loop) {
        std::vector<cudaGraphNode_t> dep = sinks(g);
        cudaGraphConditionalHandle hc;
        CK(cudaGraphConditionalHandleCreate(&hc, g, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
        cp.conditional.handle = hc;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t cn;
        CK(cudaGraphAddNode(&cn, g, dep.empty() ? nullptr : dep.data(), dep.size(), &cp));
        cudaGraph_t bg = cp.conditional.phGraph_out[0];
        int* stp = pl->stop();
        int* gc = pl->gcount();
        capture(bg, nullptr, 0, [&](cudaStream_t cs) {
          body(cs);
          launch(loop_guard_kernel, 1, 32, 0, cs, stp, gc, gmax, hc);
          CK_LAUNCH();
        });
        pl->nodes_body = count_nodes(bg);
        capture(g, &cn, 1, epilogue);
      } else {
        pl->nodes_body = 0;
      }
      CK(cudaGraphInstantiate(&e->exec, g, 0));
    } else {  // host loop: prologue+epilogue graph pieces, body graph
      e->host_loop = true;
      cudaGraph_t g;
      CK(cudaGraphCreate(&g, 0));
      e->graph = g;
      capture(g, nullptr, 0, prologue);
      CK(cudaGraphInstantiate(&e->exec, g, 0));
      cudaGraph_t bg;
      CK(cudaGraphCreate(&bg, 0));
      e->body = bg;
      int* stp = pl->stop();
      int* gc = pl->gcount();
      capture(bg, nullptr, 0, [&](cudaStream_t cs) {
        body(cs);
        launch(loop_guard_host_kernel, 1, 32, 0, cs, stp, gc, gmax);
        CK_LAUNCH();
      });
      CK(cudaGraphInstantiate(&e->body_exec, bg, 0));
    }
    pl->graphs.emplace_front(key, std::move(e));
    while (pl->graphs.size() > 8) pl->graphs.pop_back();
    ge = pl->graphs.front().second.get();
  }
  if (pl->used_program)  // barrier count, generation and status start at 0
    CK(cudaMemsetAsync(pl->bar, 0, sizeof(unsigned) * kBarWords, user));
  if (!ge->host_loop) {
    CK(cudaGraphLaunch(ge->exec, user));
  } else {
    CK(cudaGraphLaunch(ge->exec, user));
    for (;;) {
      CK(cudaGraphLaunch(ge->body_exec, user));
      CK(cudaMemcpyAsync(pl->h_stop, pl->stop(), sizeof(int), cudaMemcpyDeviceToHost, user));
      CK(cudaStreamSynchronize(user));
      if (*pl->h_stop) break;
    }
    epilogue(user);  // epilogues are empty or direct launches
    CK_LAUNCH();
  }
}

namespace {
std::mutex g_batch_mu;
std::list<std::pair<std::string, std::unique_ptr<GraphEntry>>> g_batch_graphs;  // LRU of 4
}  // namespace

void run_batch(const std::vector<BatchSys>& systems, const std::string& key, cudaStream_t user) {
  std::lock_guard<std::mutex> lk(g_batch_mu);
  GraphEntry* ge = nullptr;
  for (auto it = g_batch_graphs.begin(); it != g_batch_graphs.end(); ++it) {
    if (it->first == key) {
      g_batch_graphs.splice(g_batch_graphs.begin(), g_batch_graphs, it);
      ge = g_batch_graphs.front().second.get();
      break;
    }
  }
  if (!ge) {
    auto e = std::make_unique<GraphEntry>();
    cudaGraph_t g;
    CK(cudaGraphCreate(&g, 0));
    e->graph = g;
    cudaStream_t cs = capture_stream();
    for (const BatchSys& sy : systems) {
      // prologue as a new root branch; its last nodes come from the capture state
      CK(cudaStreamBeginCaptureToGraph(cs, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
      std::vector<cudaGraphNode_t> dep;
      try {
        sy.pro(cs);
        cudaStreamCaptureStatus st;
        const cudaGraphNode_t* d = nullptr;
        size_t nd = 0;
        CK(cudaStreamGetCaptureInfo(cs, &st, nullptr, nullptr, &d, &nd));
        dep.assign(d, d + nd);
      } catch (...) {
        cudaGraph_t junk = g;
        cudaStreamEndCapture(cs, &junk);
        throw;
      }
      cudaGraph_t g2 = g;
      CK(cudaStreamEndCapture(cs, &g2));
      cudaGraphConditionalHandle hc;
      CK(cudaGraphConditionalHandleCreate(&hc, g, 1, cudaGraphCondAssignDefault));
      cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
      cp.conditional.handle = hc;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      cudaGraphNode_t cn;
      CK(cudaGraphAddNode(&cn, g, dep.empty() ? nullptr : dep.data(), dep.size(), &cp));
      cudaGraph_t bg = cp.conditional.phGraph_out[0];
      int* stp = sy.pl->stop();
      int* gc = sy.pl->gcount();
      const int gmax = sy.gmax;
      capture(bg, nullptr, 0, [&](cudaStream_t c2) {
        sy.body(c2);
        launch(loop_guard_kernel, 1, 32, 0, c2, stp, gc, gmax, hc);
      });
      if (sy.epi) capture(g, &cn, 1, sy.epi);
    }
    CK(cudaGraphInstantiate(&e->exec, g, 0));
    g_batch_graphs.emplace_front(key, std::move(e));
    while (g_batch_graphs.size() > 4) g_batch_graphs.pop_back();
    ge = g_batch_graphs.front().second.get();
  }
  CK(cudaGraphLaunch(ge->exec, user));
}

void read_results(Plan* pl, cudaStream_t s, bool cg, int32_t* iters_out, double* relres_out) {
  if (pl->used_program) {  // a persistent program whose barrier wait ran out gave up
    unsigned st = 0;
    CK(cudaMemcpyAsync(&st, pl->bar + 2, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (st) {
      CK(cudaMemsetAsync(pl->bar, 0, sizeof(unsigned) * kBarWords, s));
      fail(AMG_ERR_TIMEOUT, "a grid barrier of the persistent coarse-level kernel ran out of time "
                            "(AMG_SPIN_LIMIT); the result is not valid");
    }
  }
  if (!iters_out && !relres_out) return;
  const int k = pl->k;
  std::vector<int> it(k);
  std::vector<double> nr(k), nb(k);
  CK(cudaMemcpyAsync(it.data(), pl->iters(), sizeof(int) * k, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(nr.data(), pl->nr(), sizeof(double) * k, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(nb.data(), pl->normb(), sizeof(double) * k, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  for (int c = 0; c < k; ++c) {
    if (iters_out) iters_out[c] = it[c];
    if (relres_out) relres_out[c] = (cg ? std::sqrt(nr[c]) : nr[c]) / nb[c];
  }
}

LoopCtl make_ctl(Plan* pl, int maxiter) {
  LoopCtl c{};
  c.nr = pl->nr();
  c.thresh = pl->thresh();
  c.active = pl->active();
  c.iters = pl->iters();
  c.stop = pl->stop();
  c.maxiter = maxiter;
  c.rmax = pl->rmax();
  c.ru = pl->ru();
  c.delta2 = ru_delta2();
  return c;
}

double ru_delta2() {
  static const double d2 = [] {
    const char* e = std::getenv("AMG_RU_DELTA");
    double d = e ? atof(e) : 3e-3;
    if (!(d > 0.0 && d < 1.0)) d = 3e-3;
    return d * d;
  }();
  return d2;
}

bool is_mixed(int prec) { return prec == AMG_PREC_MIXED || prec == AMG_PREC_MIXED_F64CG; }

Red red_of(Plan* pl) { return Red{pl->partials, pl->counter}; }

char cycle_char(int cycle) {
  if (cycle == AMG_CYCLE_V) return 'V';
  if (cycle == AMG_CYCLE_W) return 'W';
  if (cycle == AMG_CYCLE_F) return 'F';
  fail(AMG_ERR_INVALID_ARG, "Cycle %d not supported. Use 'V', 'W', or 'F'.", cycle);
}

std::string req_key(const char* kind, const Req& q) {
  char buf[320];
  snprintf(buf, sizeof(buf), "%s/%d/%d/%d/%d/%d/%.17g/%.17g/%p/%p/%p/%p/%p/%p", kind, q.prec, q.k,
           q.cycle, q.cpl, q.maxiter, q.tol, q.atol, q.b, (void*)q.x,
           q.A0 ? (const void*)q.A0->rowptr : nullptr, q.A0 ? (const void*)q.A0->col : nullptr,
           q.A0 ? (const void*)q.A0->v64 : nullptr, q.A0 ? (const void*)q.A0->v32 : nullptr);
  return buf;
}

void check_prec_data(amg_hierarchy* h, int prec, const Csr* A0) {
  const int L = int(h->levels.size());
  for (int l = 0; l < L; ++l) {
    const Level& lv = h->levels[l];
    const bool need64 = prec == AMG_PREC_F64;
    auto has = [&](const Csr& M) { return M.nnz == 0 || (need64 ? M.v64 != nullptr : M.v32 != nullptr); };
    const Csr& A = (l == 0 && A0) ? *A0 : lv.A;
    if (!has(A) || (l < L - 1 && (!has(lv.P) || !has(lv.R))))
      fail(AMG_ERR_INVALID_ARG, "level %d lacks %s matrix values", l, need64 ? "FP64" : "FP32");
    if (need64 ? !lv.dinv64 : !lv.dinv32) fail(AMG_ERR_INVALID_ARG, "level %d lacks dinv", l);
  }
  if (is_mixed(prec)) {
    const Csr& A = A0 ? *A0 : h->levels[0].A;
    if (!A.v64) fail(AMG_ERR_INVALID_ARG, "MIXED needs FP64 values of the level-0 operator");
  }
  const Coarse& c = h->coarse;
  const bool need64 = prec == AMG_PREC_F64;
  if (c.kind != AMG_COARSE_JACOBI && (need64 ? !c.m0_64 : !c.m0_32))
    fail(AMG_ERR_INVALID_ARG, "coarse solver data missing for this precision");
  if (c.kind == AMG_COARSE_QR && (need64 ? !c.m1_64 : !c.m1_32))
    fail(AMG_ERR_INVALID_ARG, "coarse QR factor R missing for this precision");
}

Csr override_csr(amg_hierarchy* h, const amg_csr* A0, cudaStream_t s) {
  validate_csr(*A0, "A0", 0, s, false);
  const Csr& A = h->levels[0].A;
  if (A0->n_rows != A.n_rows || A0->n_cols != A.n_cols)
    fail(AMG_ERR_INVALID_ARG, "A0 shape %dx%d does not match level 0 (%dx%d)", A0->n_rows, A0->n_cols,
         A.n_rows, A.n_cols);
  return Csr(*A0);
}

void check_vec(const void* p, const char* name) {
  if (!p) fail(AMG_ERR_INVALID_ARG, "%s is null", name);
}


unsigned long long count_runtime() {
  unsigned long long v = 0;
  cudaMemcpyFromSymbol(&v, g_kernel_count, sizeof(v));
  return v;
}

}  // namespace amg
