// amg_runtime.cuh -- host runtime of the B200 multigrid solve phase (shared by the
// per-precision translation units and the C ABI).
//
// A hierarchy handle wraps caller-owned device CSR arrays.  A "plan" (per precision,
// number of right-hand sides k and stream) owns the per-level work vectors, the
// per-column loop state and the reduction scratch.  Each solve is emitted once as a
// CUDA graph: the cycle's level recursion (V, W, F) is unrolled at capture time into a
// static sequence of fused CSR kernels, and the outer loop is a conditional WHILE node
// whose condition the kernels set on the device, so a whole solve is one graph launch
// with no host round trip.  Graphs are cached per (solve kind, parameters, buffers).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <type_traits>
#include <typeinfo>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/amg_b200.h"
#include "amg_device.cuh"
#include "amg_program.cuh"

namespace amg {

// ------------------------------------------------------------------ errors
extern thread_local std::string t_err;

struct Error {
  amg_status st;
  std::string msg;
};

[[noreturn]] void fail(amg_status st, const char* fmt, ...);

#define CK(call)                                                                        \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      fail(AMG_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
           __LINE__);                                                                   \
  } while (0)

#define CK_LAUNCH() CK(cudaGetLastError())

template <class F>
static amg_status guarded(F&& f) {
  try {
    f();
    t_err.clear();
    return AMG_OK;
  } catch (const Error& e) {
    t_err = e.msg;
    return e.st;
  } catch (const std::exception& e) {
    t_err = e.what();
    return AMG_ERR_CUDA;
  }
}

// ------------------------------------------------------------------ device facts
struct DevInfo {
  int nsm = 148;
  int max_ctas = 148 * 8;
};

DevInfo dev_info();

// ------------------------------------------------------------------ CSR view
struct Csr {
  int n_rows = 0, n_cols = 0;
  int64_t nnz = 0;
  const int* rowptr = nullptr;
  const int* col = nullptr;
  const double* v64 = nullptr;
  const float* v32 = nullptr;
  int g1 = 4;  // threads per row for k == 1

  Csr() = default;
  explicit Csr(const amg_csr& c) {
    n_rows = c.n_rows;
    n_cols = c.n_cols;
    nnz = c.nnz;
    rowptr = c.rowptr;
    col = c.col;
    v64 = c.val64;
    v32 = c.val32;
    const double mean = n_rows > 0 ? double(nnz) / n_rows : 0.0;
    g1 = mean < 1.5 ? 1 : mean < 3 ? 2 : mean < 6 ? 4 : mean < 12 ? 8 : mean < 24 ? 16 : 32;
  }
  template <class T>
  const T* vals() const {
    if constexpr (sizeof(T) == 8) return reinterpret_cast<const T*>(v64);
    else return reinterpret_cast<const T*>(v32);
  }
};

void check_csr(const amg_csr& c, const char* what, int lvl);
// check_csr plus a device pass over the structure on stream s (row pointers start at 0, never
// decrease and end at nnz; every column in [0, n_cols)), waited for: AMG_ERR_BAD_MATRIX
// otherwise.  once: skip a structure already checked (same pointers and sizes).  Skipped
// while s is being captured into a graph.
void validate_csr(const amg_csr& c, const char* what, int lvl, cudaStream_t s, bool once);

// ------------------------------------------------------------------ hierarchy
struct Smooth {
  int kind = AMG_SMOOTH_NONE;
  int iters = 0;
  double omega = 1.0;
  bool on() const { return kind == AMG_SMOOTH_JACOBI && iters > 0; }
};

struct Level {
  Csr A, P, R;
  const double* dinv64 = nullptr;
  const float* dinv32 = nullptr;
  Smooth pre, post;
  template <class T>
  const T* dinv() const {
    if constexpr (sizeof(T) == 8) return reinterpret_cast<const T*>(dinv64);
    else return reinterpret_cast<const T*>(dinv32);
  }
};

struct Coarse {
  int kind = AMG_COARSE_PINV;
  int n = 0;
  const double* m0_64 = nullptr;
  const float* m0_32 = nullptr;
  const double* m1_64 = nullptr;
  const float* m1_32 = nullptr;
  const int* perm = nullptr;
  int iters = 10;
  double omega = 1.0;
  template <class T>
  const T* m0() const {
    if constexpr (sizeof(T) == 8) return reinterpret_cast<const T*>(m0_64);
    else return reinterpret_cast<const T*>(m0_32);
  }
  template <class T>
  const T* m1() const {
    if constexpr (sizeof(T) == 8) return reinterpret_cast<const T*>(m1_64);
    else return reinterpret_cast<const T*>(m1_32);
  }
};

struct GraphEntry {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t body = nullptr;        // host-loop mode
  cudaGraphExec_t body_exec = nullptr;
  bool host_loop = false;
  ~GraphEntry() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (body_exec) cudaGraphExecDestroy(body_exec);
    if (body) cudaGraphDestroy(body);
  }
};

struct Plan {
  int prec = 0, k = 1;
  cudaStream_t stream = nullptr;
  int dev = 0;
  size_t csize = 8;                   // bytes of the cycle's type
  std::vector<void*> X, B, W1, W2;    // per level, cycle type
  void* r_out = nullptr;              // outer residual (outer type)
  void* p_out = nullptr;              // CG direction buffers (outer type): p_out and q_out
  void* q_out = nullptr;              //   alternate as old / new direction per CG step
  void* r_lo = nullptr;               // cycle-type copy of r (MIXED)
  double* dscal = nullptr;            // per-column doubles: thresh, nr, normb, gamma, alpha, beta, rmax
  int* iscal = nullptr;               // per-column ints: active, iters; then stop, gcount, ru[2]
  double* partials = nullptr;
  unsigned* counter = nullptr;
  int* h_stop = nullptr;              // pinned host mirror of the stop flag (host-loop mode)
  unsigned* bar = nullptr;            // persistent-program barrier: count, generation, status
  bool used_program = false;          // some captured solve of this plan runs a program
  std::vector<void*> allocs;
  std::list<std::pair<std::string, std::unique_ptr<GraphEntry>>> graphs;  // LRU
  uint64_t last_use = 0;              // the hierarchy's plan clock at this plan's last request
  int64_t nodes_outside = 0, nodes_body = 0;

  double* thresh() { return dscal; }
  double* nr() { return dscal + k; }
  double* normb() { return dscal + 2 * k; }
  double* gamma() { return dscal + 3 * k; }
  double* alpha() { return dscal + 4 * k; }
  double* beta() { return dscal + 5 * k; }
  double* rmax() { return dscal + 6 * k; }
  int* active() { return iscal; }
  int* iters() { return iscal + k; }
  int* stop() { return iscal + 2 * k; }
  int* gcount() { return iscal + 2 * k + 1; }
  int* ru() { return iscal + 2 * k + 2; }  // [0] true residual due, [1] FP32 increment unfolded

  void* alloc(size_t bytes) {
    void* p = nullptr;
    CK(cudaMalloc(&p, std::max<size_t>(bytes, 256)));
    allocs.push_back(p);
    return p;
  }
  ~Plan() {
    graphs.clear();
    for (void* p : allocs) cudaFree(p);
    if (h_stop) cudaFreeHost(h_stop);
  }
};

}  // namespace amg

namespace amg {
// Staging of amg_pcg_host: two device (B, X) column blocks [n, kc] in FP64, a copy stream
// each way, and the events that order the copies against the block solves.
struct HostStage {
  int dev = -1, n = 0, kc = 0;
  double* b[2] = {nullptr, nullptr};
  double* x[2] = {nullptr, nullptr};
  cudaStream_t h2d = nullptr, d2h = nullptr;
  cudaEvent_t in_done[2] = {}, solved[2] = {}, out_done[2] = {};
  ~HostStage() {
    for (int i = 0; i < 2; ++i) {
      if (b[i]) cudaFree(b[i]);
      if (x[i]) cudaFree(x[i]);
      if (in_done[i]) cudaEventDestroy(in_done[i]);
      if (solved[i]) cudaEventDestroy(solved[i]);
      if (out_done[i]) cudaEventDestroy(out_done[i]);
    }
    if (h2d) cudaStreamDestroy(h2d);
    if (d2h) cudaStreamDestroy(d2h);
  }
};
// Zero-padded staging of requests whose column count is padded (pad_columns in amg_capi.cu):
// right-hand sides and solution [n, kp].
struct PadStage {
  int dev = -1;
  size_t bytes = 0;
  uint64_t last_use = 0;
  void* b = nullptr;
  void* x = nullptr;
  ~PadStage() {
    if (b) cudaFree(b);
    if (x) cudaFree(x);
  }
};
}  // namespace amg

struct amg_hierarchy {
  std::vector<amg::Level> levels;
  amg::Coarse coarse;
  std::mutex mu;
  std::map<std::string, std::unique_ptr<amg::Plan>> plans;  // at most max_plans(), LRU
  uint64_t use_clock = 0;                  // orders plan and padding-stage requests (LRU)
  std::mutex stage_mu;                     // one amg_pcg_host call at a time per hierarchy
  std::unique_ptr<amg::HostStage> stage;
  // padded-request staging per stream (work on one stream is ordered, so a stream's
  // staging is never in use by two requests at once); guarded by mu; at most max_plans(), LRU
  std::map<cudaStream_t, std::unique_ptr<amg::PadStage>> pads;
};

namespace amg {

// ------------------------------------------------------------------ NVTX ranges
// Named host ranges around each level visit of a cycle and each outer-loop stage
// (AMG_NVTX=1; off by default).  They bracket the launches they enclose: in eager mode
// (AMG_EXEC=eager) a profiler attributes every kernel to its level (ncu --nvtx
// --nvtx-include "amg/L1/"); under graph capture they mark only the capture itself.
bool nvtx_enabled();

struct NvtxRange {
  bool on;
  explicit NvtxRange(const char* fmt, ...) : on(nvtx_enabled()) {
    if (!on) return;
    char buf[96];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    nvtxRangePushA(buf);
  }
  ~NvtxRange() {
    if (on) nvtxRangePop();
  }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// ------------------------------------------------------------------ launch helpers
struct Cfg {
  int G = 1, KV = 1, NCH = 1, grid = 1;
  bool lean = false;  // csr_kr (two rows in flight per lane group, NCH == 1)
  bool wide = false;  // csr_kr with 32-byte vectors (KV = 32 / value size)
  bool pipe = false;  // wide, with the row metadata software-pipelined (csr_kp)
  bool pipe2 = false; // csr_kp sized for 2 CTAs per SM
  size_t smem = 0;
};

// A tuned lanes-per-row value of kLeanCode + G selects csr_kr with G lanes; kWideCode + G
// selects csr_kr with G lanes of 32-byte vectors; kPipeCode + G the same layout as csr_kp,
// kPipe2Code + G as csr_kp sized for 2 CTAs per SM (twice the registers, no spills).  The
// pipelined kernels are built for G in {4, 8, 16}.
constexpr int kLeanCode = 64;
constexpr int kWideCode = 128;
constexpr int kPipeCode = 192;
constexpr int kPipe2Code = 256;
inline bool pipe_lanes(int g) { return g == 4 || g == 8 || g == 16; }

// Vector width of the wide kernel when every pointer is 32-byte aligned and k is a
// multiple of it (the row stride is k), else 0.
template <class T>
static int wide_kv(int k, std::initializer_list<const void*> ptrs) {
  const int kv = 32 / int(sizeof(T));
  if (k % kv != 0) return 0;
  for (const void* p : ptrs)
    if (reinterpret_cast<uintptr_t>(p) % 32 != 0) return 0;
  return kv;
}

static int pow2ceil(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

template <class T>
static int pick_kv(int k, std::initializer_list<const void*> ptrs) {
  if (k == 1) return 1;
  int kv = (sizeof(T) == 8) ? 2 : 4;
  while (kv > 1 && (k % kv) != 0) kv >>= 1;
  for (const void* p : ptrs)
    while (kv > 1 && (reinterpret_cast<uintptr_t>(p) % (sizeof(T) * kv)) != 0) kv >>= 1;
  return kv;
}

// Autotuned lanes-per-row for a (matrix, k, value size, vector width, op type): 0 when
// untuned.  op_tag<Op>() is a process-wide unique address per op type; it points at the
// type's name, which keys the optional tuning file (AMG_TUNE_FILE) across processes.
int tuned_g(const void* rowptr, int64_t nnz, int k, int es, int kv, const void* tag);

struct OpTag {
  const char* name;
};

template <class Op>
const void* op_tag() {
  static const OpTag tag{typeid(Op).name()};
  return &tag;
}

// Launches of an op that reduces columns only sometimes (the Jacobi sweep's norm and dot
// are run-time flags) run a different instantiation (its own register budget), so they
// are tuned under their own key; untuned, they fall back to the op's plain key.
template <class Op>
struct ReducingLaunch {};
template <class Op>
const void* op_tag_for(const Op& op) {
  if constexpr (!always_reduces<Op>::value && !never_reduces<Op>::value) {
    if (op.reduces()) return op_tag<ReducingLaunch<Op>>();
  }
  return op_tag<Op>();
}

template <class T>
static Cfg cfg_k(int n_rows, int k, int g1, std::initializer_list<const void*> ptrs,
                 const void* tune_rowptr = nullptr, int64_t tune_nnz = 0, const void* tune_tag = nullptr,
                 const void* fallback_tag = nullptr) {
  Cfg c;
  const DevInfo d = dev_info();
  if (k == 1) {
    c.G = g1;
    c.KV = 1;
    if (tune_rowptr) {  // autotuned lanes per row (1..32), when the tuner has run
      int tg = tuned_g(tune_rowptr, tune_nnz, 1, int(sizeof(T)), 1, tune_tag);
      if (!tg && fallback_tag) tg = tuned_g(tune_rowptr, tune_nnz, 1, int(sizeof(T)), 1, fallback_tag);
      if (tg == 1 || tg == 2 || tg == 4 || tg == 8 || tg == 16 || tg == 32) c.G = tg;
    }
  } else {
    c.KV = pick_kv<T>(k, ptrs);
    const int nch = k / c.KV;
    c.G = std::max(4, std::min(32, pow2ceil(nch)));
    int tg = 0;
    if (tune_rowptr) tg = tuned_g(tune_rowptr, tune_nnz, k, int(sizeof(T)), c.KV, tune_tag);
    if (tune_rowptr && !tg && fallback_tag) tg = tuned_g(tune_rowptr, tune_nnz, k, int(sizeof(T)), c.KV, fallback_tag);
    if (const char* fg = std::getenv("AMG_KB_G")) {  // manual override (experiments)
      const int g = atoi(fg);
      const int gl = g >= kPipe2Code ? g - kPipe2Code : g >= kPipeCode ? g - kPipeCode : g >= kWideCode ? g - kWideCode
                     : g >= kLeanCode ? g - kLeanCode : g;
      if (g >= kPipeCode ? pipe_lanes(gl)
                         : (gl == 4 || gl == 8 || gl == 16 || gl == 32 || (g >= kLeanCode && (gl == 1 || gl == 2))))
        tg = g;
    }
    if (!tune_rowptr && tg >= kLeanCode) tg = 0;  // elementwise passes: no lean / wide kernels
    if (tg >= kWideCode) {
      const bool pipe2 = tg >= kPipe2Code;
      const bool pipe = tg >= kPipeCode;
      tg -= pipe2 ? kPipe2Code : pipe ? kPipeCode : kWideCode;
      const int wk = wide_kv<T>(k, ptrs);
      if (wk && k / wk <= tg) {  // one 32-byte chunk per lane
        c.KV = wk;
        c.wide = true;
        c.pipe = pipe && pipe_lanes(tg);
        c.pipe2 = pipe2 && c.pipe;
      }
      c.lean = true;
    } else if (tg >= kLeanCode) {
      tg -= kLeanCode;
      c.lean = true;
    }
    if (tg) c.G = tg;
    if (c.lean && !c.wide && (k / c.KV + c.G - 1) / c.G > 1) {  // lean needs one chunk per lane
      c.lean = false;
      c.G = std::max(4, std::min(32, pow2ceil(nch)));
    }
    if ((k / c.KV + c.G - 1) / c.G > kMaxCh) {  // a recorded layout too narrow for this k
      c.lean = c.wide = false;
      c.KV = pick_kv<T>(k, ptrs);
      c.G = std::max(4, std::min(32, pow2ceil(k / c.KV)));
    }
    const int per = (k / c.KV + c.G - 1) / c.G;
    if (per > kMaxCh)
      fail(AMG_ERR_UNSUPPORTED, "k=%d exceeds the per-launch column limit (%d)", k, 32 * kMaxCh * c.KV);
    c.NCH = per <= 1 ? 1 : per <= 2 ? 2 : 4;
    if (c.NCH > 1 || c.KV == 1) c.lean = c.wide = c.pipe = c.pipe2 = false;
    if (c.KV == 1 && c.NCH > 1) c.G = 32;
    c.smem = sizeof(double) * std::max<size_t>(size_t(kBlock / c.G) * k, kBlock);
  }
  const int rows_per_cta = kBlock / c.G;
  const int64_t need = (int64_t(n_rows) + rows_per_cta - 1) / rows_per_cta;
  c.grid = int(std::max<int64_t>(1, std::min<int64_t>(need, d.max_ctas)));
  return c;
}

struct Red {
  double* partials = nullptr;
  unsigned* counter = nullptr;
};

// Launch with programmatic stream serialization (PDL): the kernel may start while its
// predecessor on the stream drains; every kernel of this library begins with
// griddepcontrol.wait, so correctness does not depend on it.  AMG_PDL=0 disables.
bool pdl_enabled();
// Two-pass levels for one right-hand side (Cycle::visit): on unless AMG_FUSE2=0, for levels
// of at most AMG_FUSE2_ROWS rows (default 20,000) whose two-hop gathers,
// nnz(R) nnz(A) / n + nnz(A) nnz(P) / n, number at most AMG_FUSE2_WORK (default 500,000).
// Measured at k = 1, PCG mixed, on the Poisson 500² SA hierarchy (levels of 250,000 /
// 41,750 / 4,704 / 532 rows, two-hop gathers 6.2e6 / 2.1e6 / 2.3e5 / 2.4e4): unfused
// 1.288 ms, fused from level 2 1.222 ms, from level 1 1.307 ms, from level 0 1.438 ms; and
// on the 3D 128³ diffusion SA hierarchy (a level of 6,349 rows with 59 nonzeros per row,
// 3.8e6 two-hop gathers) a V-cycle solve took 36.2 ms unfused and 83.6 ms with that level
// fused: recomputing each neighbour's value costs more than the launch it saves unless
// the level's gathers are few.  A coarse row's restriction also walks its two-hop gathers
// in one lane group, so the mean per coarse row, nnz(R) / n_c * nnz(A) / n, must stay at
// most AMG_FUSE2_CHAIN (default 400; Poisson 500² levels 2-4: 212 / 185 / 19; the 128³
// hierarchy's 82-row level, whose two coarse rows hold 76 nonzeros each: 2,830, and fused
// it cost 40.5 vs 36.2 ms).
bool fuse2_enabled();
int fuse2_rows();
double fuse2_work();
double fuse2_chain();
inline bool fuse2_level(const Level& lv, const Csr& A, int k) {
  if (k != 1 || !fuse2_enabled() || A.n_rows == 0 || A.n_rows > fuse2_rows() || lv.R.n_rows == 0) return false;
  const double n = A.n_rows, a = double(A.nnz) / n;
  if (double(lv.R.nnz) / double(lv.R.n_rows) * a > fuse2_chain()) return false;
  return double(lv.R.nnz) * a + double(A.nnz) * (double(lv.P.nnz) / n) <= fuse2_work();
}

// Preferred shared-memory share (percent) of the SM's unified L1 / shared storage for a
// launch of fn with `smem` dynamic bytes: the least that holds the shared memory of the CTAs
// that can be resident (static + dynamic + the 1 KB per CTA the system reserves), so the
// rest serves the gathers as L1.  -1 leaves the driver's choice (AMG_CARVEOUT=0).  Measured
// on the FP32 <p, A p> at N = 250,000, k = 64 (16 KB per CTA, 3 CTAs per SM): 63.3 us with
// the driver's choice, 60.6 us at 25 %, 62.6 us at 50 %, 91.5 us at 100 %; at 0-10 % only one
// CTA fits (142 us).
int carveout_pct(const void* fn, size_t smem);

template <class... Exp, class... Act>
static void launch(void (*kernel)(Exp...), int grid, int block, size_t smem, cudaStream_t s,
                   Act&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[2];
  int na = 0;
  if (pdl_enabled()) {
    attr[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[na].val.programmaticStreamSerializationAllowed = 1;
    ++na;
  }
  const int pct = carveout_pct(reinterpret_cast<const void*>(kernel), smem);
  if (pct >= 0) {
    attr[na].id = cudaLaunchAttributePreferredSharedMemoryCarveout;
    attr[na].val.sharedMemCarveout = static_cast<unsigned>(pct);
    ++na;
  }
  cfg.attrs = attr;
  cfg.numAttrs = na;
  CK(cudaLaunchKernelEx(&cfg, kernel, std::forward<Act>(args)...));
}

// Resident CTAs per SM of one kernel instantiation (cached): grids are capped at
// SMs x this, so a grid-stride kernel runs in a single wave.
int resident_ctas(const void* fn, size_t smem);

template <class K>
static int cap_grid(K* fn, int grid, size_t smem) {
  const int per_sm = resident_ctas(reinterpret_cast<const void*>(fn), smem);
  return std::max(1, std::min(grid, dev_info().nsm * per_sm));
}

template <class Op, int G>
static void launch_k1(const Csr& M, const typename Op::V* vals, const Op& op, const Cfg& c,
                      RedCtx rc, cudaStream_t s) {
  const int grid = cap_grid(csr_k1<Op, G>, c.grid, 0);
  launch(csr_k1<Op, G>, grid, kBlock, 0, s, M.rowptr, M.col, vals, M.n_rows, op, rc);
}

template <class Op, int G, int KV, int NCH>
static void launch_kb(const Csr& M, const typename Op::V* vals, const Op& op, const Cfg& c,
                      RedCtx rc, cudaStream_t s) {
  const size_t smem = op.reduces() ? c.smem : 0;  // the reduction's scratch only
  const int grid = cap_grid(csr_kb<Op, G, KV, NCH>, c.grid, smem);
  launch(csr_kb<Op, G, KV, NCH>, grid, kBlock, smem, s, M.rowptr, M.col, vals, M.n_rows, op, rc);
}

// csr_kr: one column chunk per lane; two rows in flight per lane group with 16-byte
// vectors, one with 32-byte vectors (half the lanes per row, so a warp already holds twice
// the rows; a second row per group would spill).
template <class Op, int G, int KV>
static void launch_kr(const Csr& M, const typename Op::V* vals, const Op& op, const Cfg& c,
                      RedCtx rc, cudaStream_t s) {
  constexpr int R = (KV * sizeof(typename Op::Acc) >= 32) ? 1 : 2;
  if constexpr (!never_reduces<Op>::value) {
    if (op.reduces()) {
      const int grid = cap_grid(csr_kr<Op, G, KV, R, true>, c.grid, c.smem);
      launch(csr_kr<Op, G, KV, R, true>, grid, kBlock, c.smem, s, M.rowptr, M.col, vals, M.n_rows, op, rc);
      return;
    }
  }
  if constexpr (!always_reduces<Op>::value) {
    const int grid = cap_grid(csr_kr<Op, G, KV, R, false>, c.grid, 0);
    launch(csr_kr<Op, G, KV, R, false>, grid, kBlock, 0, s, M.rowptr, M.col, vals, M.n_rows, op, rc);
  }
}

template <class Op, int G, int KV, int MINB_RED, int MINB_PLAIN>
static void launch_kp_t(const Csr& M, const typename Op::V* vals, const Op& op, const Cfg& c,
                        RedCtx rc, cudaStream_t s) {
  if constexpr (!never_reduces<Op>::value) {
    if (op.reduces()) {
      auto* kern = csr_kp<Op, G, KV, true, kPipeB, MINB_RED>;
      const int grid = cap_grid(kern, c.grid, c.smem);
      launch(kern, grid, kBlock, c.smem, s, M.rowptr, M.col, vals, M.n_rows, op, rc);
      return;
    }
  }
  if constexpr (!always_reduces<Op>::value) {
    auto* kern = csr_kp<Op, G, KV, false, kPipeB, MINB_PLAIN>;
    const int grid = cap_grid(kern, c.grid, 0);
    launch(kern, grid, kBlock, 0, s, M.rowptr, M.col, vals, M.n_rows, op, rc);
  }
}

template <class Op, int G, int KV>
static void launch_kp(const Csr& M, const typename Op::V* vals, const Op& op, const Cfg& c,
                      RedCtx rc, cudaStream_t s) {
  if (c.pipe2) launch_kp_t<Op, G, KV, 2, 2>(M, vals, op, c, rc, s);
  else launch_kp_t<Op, G, KV, kr_min_blocks<Op, KV, true>(), kr_min_blocks<Op, KV, false>()>(M, vals, op, c, rc, s);
}

// (G, NCH) pairs: any G in {4, 8, 16, 32} with NCH in {1, 2, 4} for vector widths >= 2;
// scalar columns (odd k) use NCH = 1, or G = 32 with NCH in {2, 4}.
template <class Op, int KV, int G>
static void dispatch_kb_nch(const Csr& M, const typename Op::V* vals, const Op& op, const Cfg& c,
                            RedCtx rc, cudaStream_t s) {
  if constexpr (KV >= 2) {
    if (c.lean) {  // cfg_k sets lean with one chunk per lane only
      launch_kr<Op, G, KV>(M, vals, op, c, rc, s);
      return;
    }
  }
  if (c.NCH == 1) launch_kb<Op, G, KV, 1>(M, vals, op, c, rc, s);
  else if constexpr (KV >= 2 || G == 32) {
    if (c.NCH == 2) launch_kb<Op, G, KV, 2>(M, vals, op, c, rc, s);
    else launch_kb<Op, G, KV, 4>(M, vals, op, c, rc, s);
  } else {
    fail(AMG_ERR_INVALID_ARG, "internal: (G=%d, NCH=%d) not built for scalar columns", G, c.NCH);
  }
}

template <class Op, int KV>
static void dispatch_kb_g(const Csr& M, const typename Op::V* vals, const Op& op, const Cfg& c,
                          RedCtx rc, cudaStream_t s) {
  switch (c.G) {
    case 4: dispatch_kb_nch<Op, KV, 4>(M, vals, op, c, rc, s); break;
    case 8: dispatch_kb_nch<Op, KV, 8>(M, vals, op, c, rc, s); break;
    case 16: dispatch_kb_nch<Op, KV, 16>(M, vals, op, c, rc, s); break;
    default: dispatch_kb_nch<Op, KV, 32>(M, vals, op, c, rc, s); break;
  }
}

// Launch one fused CSR pass of matrix M with epilogue op over k columns.
template <class Op>
static void run_csr(const Csr& M, const Op& op, int k, const Red& red, cudaStream_t s,
                    std::initializer_list<const void*> ptrs) {
  using V = typename Op::V;
  const V* vals = M.template vals<V>();
  if (M.nnz > 0 && !vals) fail(AMG_ERR_INVALID_ARG, "matrix values missing for this precision");
  const Cfg c = cfg_k<typename Op::Acc>(M.n_rows, k, M.g1, ptrs, M.rowptr, M.nnz, op_tag_for(op), op_tag<Op>());
  RedCtx rc{red.partials, red.counter, k};
  if (op.reduces() && !red.partials) fail(AMG_ERR_INVALID_ARG, "reduction scratch missing");
  if constexpr (only_k1<Op>::value) {  // two-hop sources: one right-hand side, csr_k1 only
    if (k != 1) fail(AMG_ERR_INVALID_ARG, "internal: a one-column op with k = %d", k);
    switch (c.G) {
      case 1: launch_k1<Op, 1>(M, vals, op, c, rc, s); break;
      case 2: launch_k1<Op, 2>(M, vals, op, c, rc, s); break;
      case 4: launch_k1<Op, 4>(M, vals, op, c, rc, s); break;
      case 8: launch_k1<Op, 8>(M, vals, op, c, rc, s); break;
      case 16: launch_k1<Op, 16>(M, vals, op, c, rc, s); break;
      default: launch_k1<Op, 32>(M, vals, op, c, rc, s); break;
    }
    CK_LAUNCH();
    return;
  } else {
  if (k == 1) {
    switch (c.G) {
      case 1: launch_k1<Op, 1>(M, vals, op, c, rc, s); break;
      case 2: launch_k1<Op, 2>(M, vals, op, c, rc, s); break;
      case 4: launch_k1<Op, 4>(M, vals, op, c, rc, s); break;
      case 8: launch_k1<Op, 8>(M, vals, op, c, rc, s); break;
      case 16: launch_k1<Op, 16>(M, vals, op, c, rc, s); break;
      default: launch_k1<Op, 32>(M, vals, op, c, rc, s); break;
    }
  } else if (c.wide && c.pipe) {
    constexpr int KW = 32 / int(sizeof(typename Op::Acc));
    switch (c.G) {
      case 4: launch_kp<Op, 4, KW>(M, vals, op, c, rc, s); break;
      case 8: launch_kp<Op, 8, KW>(M, vals, op, c, rc, s); break;
      default: launch_kp<Op, 16, KW>(M, vals, op, c, rc, s); break;
    }
  } else if (c.wide) {
    constexpr int KW = 32 / int(sizeof(typename Op::Acc));
    switch (c.G) {
      case 1: launch_kr<Op, 1, KW>(M, vals, op, c, rc, s); break;
      case 2: launch_kr<Op, 2, KW>(M, vals, op, c, rc, s); break;
      case 4: launch_kr<Op, 4, KW>(M, vals, op, c, rc, s); break;
      case 8: launch_kr<Op, 8, KW>(M, vals, op, c, rc, s); break;
      case 16: launch_kr<Op, 16, KW>(M, vals, op, c, rc, s); break;
      default: launch_kr<Op, 32, KW>(M, vals, op, c, rc, s); break;
    }
  } else if (c.lean && c.G < 4) {  // lean kernel with 1 or 2 lanes per row (few columns)
    if (c.KV == 2) {
      if (c.G == 1) launch_kr<Op, 1, 2>(M, vals, op, c, rc, s);
      else launch_kr<Op, 2, 2>(M, vals, op, c, rc, s);
    } else if constexpr (sizeof(typename Op::Acc) == 4) {
      if (c.G == 1) launch_kr<Op, 1, 4>(M, vals, op, c, rc, s);
      else launch_kr<Op, 2, 4>(M, vals, op, c, rc, s);
    } else {
      fail(AMG_ERR_INVALID_ARG, "internal: lean layout G=%d KV=%d", c.G, c.KV);
    }
  } else {
    if (c.KV == 1) dispatch_kb_g<Op, 1>(M, vals, op, c, rc, s);
    else if (c.KV == 2) dispatch_kb_g<Op, 2>(M, vals, op, c, rc, s);
    else if constexpr (sizeof(typename Op::Acc) == 4) dispatch_kb_g<Op, 4>(M, vals, op, c, rc, s);
    else fail(AMG_ERR_INVALID_ARG, "internal: 4-wide FP64 vectors");
  }
  CK_LAUNCH();
  }
}

// ------------------------------------------------------------------ autotuner
// Record the fastest lanes-per-row for (matrix, k, value size, vector width, op type).
// `final`: the tuner's decision (recorded in AMG_TUNE_FILE when set), not a candidate.
void set_tuned_g(const void* rowptr, int64_t nnz, int k, int es, int kv, const void* tag, int g,
                 bool final = false);
bool tuning_enabled();

// Time one fused CSR op (a fully formed instance on scratch buffers, stop flag off) with
// each candidate lanes-per-row G (each with its chunks per lane) and keep the fastest for
// this (matrix, k, type, op).  Runs outside stream capture, once per key.
// `before` (optional) runs ahead of every launch, outside the timed region: it restores
// state an op's finalisation changes (the CG update freezes the columns that have converged,
// and frozen columns skip their writes, which would flatter later candidates).
template <class Op>
void tune_op(const Csr& M, const Op& op, int k, const Red& red, cudaStream_t s,
             std::initializer_list<const void*> ptrs,
             const std::function<void(cudaStream_t)>& before = {}) {
  using T = typename Op::Acc;
  if (M.n_rows == 0) return;
  if (M.nnz > 0 && !M.template vals<typename Op::V>()) return;
  const int kv = k == 1 ? 1 : pick_kv<T>(k, ptrs);
  if (!tuning_enabled()) return;
  const void* tag = op_tag_for(op);
  if (tuned_g(M.rowptr, M.nnz, k, int(sizeof(T)), kv, tag)) return;
  const int nch = k / kv;
  const int gmax = std::max(4, std::min(32, pow2ceil(nch)));
  std::vector<int> cands;
  if (k == 1)  // csr_k1: lanes sharing a row's nonzeros
    for (int g = 1; g <= 32; g <<= 1) cands.push_back(g);
  for (int g = 4; g <= gmax && k > 1; g <<= 1) {
    const int per = (nch + g - 1) / g;
    if (per <= kMaxCh && (kv > 1 || per == 1 || g == 32)) cands.push_back(g);
  }
  if (kv > 1 && k > 1)  // the lean kernel, one chunk per lane (1 or 2 lanes per row for few columns)
    for (int g = 1; g <= gmax; g <<= 1)
      if (nch <= g && (g >= 4 || kv * int(sizeof(T)) == 16 || kv * int(sizeof(T)) == 8))
        cands.push_back(kLeanCode + g);
  if (const int wk = k > 1 ? wide_kv<T>(k, ptrs) : 0)  // the wide lean kernels, one 32-byte chunk per lane
    for (int g = 1; g <= 32; g <<= 1)
      if (k / wk <= g && g < 2 * std::max(4, pow2ceil(k / wk)) && (g >= 4 || g == pow2ceil(k / wk))) {
        cands.push_back(kWideCode + g);
        if (pipe_lanes(g)) {
          cands.push_back(kPipeCode + g);
          cands.push_back(kPipe2Code + g);
        }
      }
  if (cands.size() <= 1) {
    set_tuned_g(M.rowptr, M.nnz, k, int(sizeof(T)), kv, tag, cands.empty() ? gmax : cands[0], true);
    return;
  }
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  int best = cands.back();
  float best_t = 1e30f;
  for (int g : cands) {
    set_tuned_g(M.rowptr, M.nnz, k, int(sizeof(T)), kv, tag, g);
    if (before) before(s);
    run_csr(M, op, k, red, s, ptrs);
    float tmin = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
      if (before) before(s);
      CK(cudaEventRecord(e0, s));
      run_csr(M, op, k, red, s, ptrs);
      CK(cudaEventRecord(e1, s));
      CK(cudaEventSynchronize(e1));
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, e0, e1));
      tmin = std::min(tmin, ms);
    }
    if (tmin < best_t) {
      best_t = tmin;
      best = g;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  set_tuned_g(M.rowptr, M.nnz, k, int(sizeof(T)), kv, tag, best, true);
  if (std::getenv("AMG_TUNE_LOG"))
    fprintf(stderr, "[amg tune] rows=%d nnz=%lld k=%d es=%d kv=%d op=%p -> G=%d (%.1f us)\n", M.n_rows,
            (long long)M.nnz, k, int(sizeof(T)), kv, tag, best, best_t * 1e3f);
}

// Tune the cycle's ops in type T on every level (Jacobi sweeps, residuals, restriction,
// prolongation) for this plan's k; level 0 uses A0 when given.
template <class T>
void autotune_cycle(amg_hierarchy* h, Plan* pl, int k, const Csr* A0, cudaStream_t s) {
  const int L = int(h->levels.size());
  for (int l = 0; l < L - 1; ++l) {
    const Level& lv = h->levels[l];
    const Csr& A = (l == 0 && A0) ? *A0 : lv.A;
    T* w1 = static_cast<T*>(pl->W1[l]);
    T* w2 = static_cast<T*>(pl->W2[l]);
    T* bl = static_cast<T*>(pl->B[l]);
    T* xc = static_cast<T*>(pl->X[l + 1]);
    T* bc = static_cast<T*>(pl->B[l + 1]);
    const T* dv = lv.template dinv<T>();
    if (!dv) continue;
    {
      OpJacobi<T, XS_PLAIN> op{};
      op.xs = XSource<T, XS_PLAIN>{w1, bl, dv, T(0.5), k};
      op.b = bl; op.dinv = dv; op.omega = T(0.5); op.out = w2; op.ld = k;
      tune_op(A, op, k, Red{}, s, {w1, bl, w2});
    }
    {
      OpJacobi<T, XS_JAC0> op{};
      op.xs = XSource<T, XS_JAC0>{nullptr, bl, dv, T(0.5), k};
      op.b = bl; op.dinv = dv; op.omega = T(0.5); op.out = w2; op.ld = k;
      tune_op(A, op, k, Red{}, s, {bl, w2});
    }
    {
      OpResid<T, T, XS_PLAIN, true, T, false> op{};
      op.xs = XSource<T, XS_PLAIN>{w1, bl, dv, T(0.5), k};
      op.b = bl; op.out = w2; op.ld = k;
      tune_op(A, op, k, Red{}, s, {w1, bl, w2});
    }
    {
      OpResid<T, T, XS_JAC0, true, T, false> op{};
      op.xs = XSource<T, XS_JAC0>{nullptr, bl, dv, T(0.5), k};
      op.b = bl; op.out = w2; op.ld = k;
      tune_op(A, op, k, Red{}, s, {bl, w2});
    }
    {
      OpAxpy<T, XS_ZERO> op{};
      op.x = w2; op.out = bc; op.ld = k;
      tune_op(lv.R, op, k, Red{}, s, {w2, bc});
    }
    {
      OpAxpy<T, XS_PLAIN> op{};
      op.base = XSource<T, XS_PLAIN>{w1, bl, dv, T(0), k};
      op.x = xc; op.out = w2; op.ld = k;
      tune_op(lv.P, op, k, Red{}, s, {w1, xc, w2});
    }
    {
      OpAxpy<T, XS_JAC0> op{};
      op.base = XSource<T, XS_JAC0>{nullptr, bl, dv, T(0.5), k};
      op.x = xc; op.out = w1; op.ld = k;
      tune_op(lv.P, op, k, Red{}, s, {bl, xc, w1});
    }
    if (fuse2_level(lv, A, k)) {  // the two-pass level ops
      OpRestrictX<T, XS_RESJ0> rop{};
      rop.xs = XSource<T, XS_RESJ0>{nullptr, bl, dv, T(0.5), k, A.rowptr, A.col, A.template vals<T>(), nullptr};
      rop.out = bc; rop.ld = k;
      tune_op(lv.R, rop, k, Red{}, s, {bl, bc});
      OpJacobi<T, XS_PROJ0> op{};
      op.xs = XSource<T, XS_PROJ0>{nullptr, bl, dv, T(0.5), k, lv.P.rowptr, lv.P.col, lv.P.template vals<T>(), xc};
      op.b = bl; op.dinv = dv; op.omega = T(0.5); op.out = w2; op.ld = k;
      tune_op(A, op, k, Red{}, s, {bl, w2});
    }
  }
}

template <class Op, int G, int KV, int NCH>
static void launch_elem(int n, const Op& op, const Cfg& c, RedCtx rc, cudaStream_t s) {
  const size_t smem = op.reduces() ? c.smem : 0;  // the reduction's scratch only
  const int grid = cap_grid(elem_kb<Op, G, KV, NCH>, c.grid, smem);
  launch(elem_kb<Op, G, KV, NCH>, grid, kBlock, smem, s, n, op, rc);
}

template <class Op, int KV>
static void dispatch_elem_g(int n, const Op& op, const Cfg& c, RedCtx rc, cudaStream_t s) {
  if (c.NCH == 2) { launch_elem<Op, 32, KV, 2>(n, op, c, rc, s); return; }
  if (c.NCH == 4) { launch_elem<Op, 32, KV, 4>(n, op, c, rc, s); return; }
  switch (c.G) {
    case 1: launch_elem<Op, 1, KV, 1>(n, op, c, rc, s); break;
    case 4: launch_elem<Op, 4, KV, 1>(n, op, c, rc, s); break;
    case 8: launch_elem<Op, 8, KV, 1>(n, op, c, rc, s); break;
    case 16: launch_elem<Op, 16, KV, 1>(n, op, c, rc, s); break;
    default: launch_elem<Op, 32, KV, 1>(n, op, c, rc, s); break;
  }
}

// Elementwise pass over [n, k]; T_align is the narrowest element type the op touches
// (it bounds the vector width).
template <class TA, class Op>
static void run_elem(int n, const Op& op, int k, const Red& red, cudaStream_t s,
                     std::initializer_list<const void*> ptrs) {
  Cfg c = cfg_k<TA>(n, k, 1, ptrs);
  if (k == 1) c.G = 1;
  if (k == 1) {
    const int64_t need = (int64_t(n) + kBlock - 1) / kBlock;
    c.grid = int(std::max<int64_t>(1, std::min<int64_t>(need, dev_info().max_ctas)));
  }
  RedCtx rc{red.partials, red.counter, k};
  if (op.reduces() && !red.partials) fail(AMG_ERR_INVALID_ARG, "reduction scratch missing");
  if (c.KV == 1) dispatch_elem_g<Op, 1>(n, op, c, rc, s);
  else if (c.KV == 2) dispatch_elem_g<Op, 2>(n, op, c, rc, s);
  else if constexpr (sizeof(TA) == 4) dispatch_elem_g<Op, 4>(n, op, c, rc, s);
  else fail(AMG_ERR_INVALID_ARG, "internal: 4-wide FP64 vectors");
  CK_LAUNCH();
}

// ------------------------------------------------------------------ cycle emission
// How the SpMV sees an iterate: a stored vector, one Jacobi sweep from zero computed
// on the fly, or the zero vector.
template <class T>
struct XD {
  int kind = XS_ZERO;
  const T* p = nullptr;
  static XD plain(const T* q) { XD d; d.kind = XS_PLAIN; d.p = q; return d; }
  static XD jac0() { XD d; d.kind = XS_JAC0; return d; }
  static XD zero() { XD d; d.kind = XS_ZERO; return d; }
};

template <class T>
struct Cycle {
  amg_hierarchy* h;
  Plan* pl;
  cudaStream_t s;
  int k;
  const int* stop;         // checked by every cycle kernel (nullable)
  const Csr* A0;           // level-0 operator (override or the hierarchy's)
  const T* b0;             // level-0 right-hand side
  T* x0;                   // level-0 iterate / result
  bool fine_norm = false;  // standalone: fuse ||b - A x|| into the first level-0 sweep
  LoopCtl ctl{};
  bool fine_mask = false;  // write level-0 result only for active columns
  const void* fine_dot = nullptr;  // CG: fuse <r, z> into the last level-0 sweep (outer type)
  bool dot_is_f64 = true;
  Red red;
  int tail_from = -1;                 // levels >= this run as one persistent program (-1: none)
  std::vector<PStep>* rec = nullptr;  // recording a program: steps are appended, not launched

  template <class Op>
  void record(const Op& op, int kind, const Csr& M, const void* x, const void* b, const void* dinv,
              const void* base, void* out, double omega, std::initializer_list<const void*> ptrs) {
    PStep st{};
    st.kind = kind;
    st.n_rows = M.n_rows;
    st.rowptr = M.rowptr;
    st.col = M.col;
    st.val = M.template vals<T>();
    st.x = x; st.b = b; st.dinv = dinv; st.base = base; st.out = out; st.omega = omega;
    st.barrier = 1;
    if (k == 1) {  // the launched kernel's lanes per row (its shuffle order)
      st.g = cfg_k<T>(M.n_rows, 1, M.g1, ptrs, M.rowptr, M.nnz, op_tag_for(op), op_tag<Op>()).G;
      st.kv = 1;
    } else {
      const int kv16 = 16 / int(sizeof(T));
      st.kv = (k % kv16 == 0) ? kv16 : 1;
      st.g = pow2ceil(k / st.kv);
    }
    rec->push_back(st);
  }

  // Run the recorded steps: one cooperative launch per kMaxSteps steps.
  void emit_program(const std::vector<PStep>& steps) {
    const GridBar gb{pl->bar, pl->bar + 1, reinterpret_cast<int*>(pl->bar + 2), pl->bar + 4, spin_limit()};
    for (size_t i0 = 0; i0 < steps.size(); i0 += kMaxSteps) {
      Program p{};
      p.nsteps = int(std::min<size_t>(kMaxSteps, steps.size() - i0));
      for (int j = 0; j < p.nsteps; ++j) p.steps[j] = steps[i0 + size_t(j)];
      launch_program(p, sizeof(T) == 8, k, stop, gb, s);
    }
    pl->used_program = true;
  }

  int L() const { return int(h->levels.size()); }
  const Csr& Aof(int l) const { return (l == 0 && A0) ? *A0 : h->levels[l].A; }
  T* Xb(int l) const { return l == 0 ? x0 : static_cast<T*>(pl->X[l]); }
  const T* Bb(int l) const { return l == 0 ? b0 : static_cast<const T*>(pl->B[l]); }
  T* W1(int l) const { return static_cast<T*>(pl->W1[l]); }
  T* W2(int l) const { return static_cast<T*>(pl->W2[l]); }

  template <int XS>
  XSource<T, XS> xsrc(int l, const T* xp, T omega) const {
    const Level& lv = h->levels[l];
    return XSource<T, XS>{xp, Bb(l), lv.template dinv<T>(), omega, k};
  }

  // One Jacobi sweep in -> out on level l; flags select the fused extras.
  template <int XS>
  void sweep_x(int l, const T* in, T omega, T* out, bool norm, bool mask, bool dot) {
    const Level& lv = h->levels[l];
    if (rec) {
      if (norm || mask || dot) fail(AMG_ERR_INVALID_ARG, "internal: fused extras in a program step");
      OpJacobi<T, XS> op{};
      record(op, XS == XS_PLAIN ? PK_JAC_PLAIN : PK_JAC_J0, Aof(l), in, Bb(l), lv.template dinv<T>(), nullptr, out,
             double(omega), {in, Bb(l), out});
      return;
    }
    OpJacobi<T, XS> op{};
    op.xs = xsrc<XS>(l, in, omega);
    op.b = Bb(l);
    op.dinv = lv.template dinv<T>();
    op.omega = omega;
    op.out = out;
    op.ld = k;
    op.norm = norm ? 1 : 0;
    op.active = mask ? pl->active() : nullptr;
    op.stop = norm ? nullptr : stop;
    op.rdot64 = (dot && dot_is_f64) ? static_cast<const double*>(fine_dot) : nullptr;
    op.rdot32 = (dot && !dot_is_f64) ? static_cast<const float*>(fine_dot) : nullptr;
    op.ctl = ctl;
    op.gamma = pl->gamma();
    op.beta = pl->beta();
    run_csr(Aof(l), op, k, red, s, {in, Bb(l), out, dot ? fine_dot : nullptr});
  }

  void sweep(int l, XD<T> in, T omega, T* out, bool norm, bool mask, bool dot) {
    if (in.kind == XS_PLAIN) sweep_x<XS_PLAIN>(l, in.p, omega, out, norm, mask, dot);
    else if (in.kind == XS_JAC0) sweep_x<XS_JAC0>(l, nullptr, omega, out, norm, mask, dot);
    else fail(AMG_ERR_INVALID_ARG, "internal: sweep from the zero vector");
  }

  // n sweeps starting from `src`; the last writes `dst`, the others alternate between
  // t_a and t_b so that no sweep reads the buffer it writes.  `src` is never written.
  void sweeps(int l, XD<T> src, int n, T omega, T* dst, T* t_a, T* t_b, bool norm_first,
              bool mask_last, bool dot_last) {
    if (n <= 0) return;
    // choose the order of temps so the last intermediate is not dst
    T* ta = t_a;
    T* tb = t_b;
    if (n >= 2) {
      T* last_inter = ((n - 2) % 2 == 0) ? ta : tb;
      if (last_inter == dst) std::swap(ta, tb);
    }
    XD<T> in = src;
    for (int i = 0; i < n; ++i) {
      const bool last = (i == n - 1);
      T* out = last ? dst : ((i % 2 == 0) ? ta : tb);
      if (in.kind == XS_PLAIN && in.p == out) fail(AMG_ERR_INVALID_ARG, "internal: sweep aliasing");
      sweep(l, in, omega, out, norm_first && i == 0, mask_last && last, dot_last && last);
      in = XD<T>::plain(out);
    }
  }

  template <int XS, bool NORM>
  void resid_t(int l, const T* xp, T omega, const T* b, T* out) {
    if (rec) {
      static_assert(!NORM || XS == XS_PLAIN, "");
      if (NORM || b != Bb(l)) fail(AMG_ERR_INVALID_ARG, "internal: residual form not recordable");
      OpResid<T, T, XS, true, T, false> op{};
      record(op, XS == XS_PLAIN ? PK_RES_PLAIN : PK_RES_J0, Aof(l), xp, Bb(l), h->levels[l].template dinv<T>(),
             nullptr, out, double(omega), {xp, Bb(l), b, out});
      return;
    }
    OpResid<T, T, XS, true, T, NORM> op{};
    op.xs = xsrc<XS>(l, xp, omega);
    op.b = b;
    op.out = out;
    op.out_lo = nullptr;
    op.ld = k;
    op.stop = NORM ? nullptr : stop;
    op.ctl = ctl;
    // every array the op reads picks the vector width (a Jacobi-from-zero source reads
    // op.xs.b, which at level 0 may be the caller's right-hand side)
    run_csr(Aof(l), op, k, red, s, {xp, op.xs.b, b, out});
  }

  template <int BS>
  void axpy_t(const Csr& M, const T* base, T omega, int l_base, const T* x, T* out) {
    if (rec) {
      OpAxpy<T, BS> op{};
      const int kind = BS == XS_ZERO ? PK_AXPY_ZERO : BS == XS_PLAIN ? PK_AXPY_PLAIN : PK_AXPY_J0;
      record(op, kind, M, x, Bb(l_base), h->levels[l_base].template dinv<T>(), base, out, double(omega),
             {base, Bb(l_base), x, out});
      return;
    }
    OpAxpy<T, BS> op{};
    op.base = xsrc<BS>(l_base, base, omega);
    op.x = x;
    op.out = out;
    op.ld = k;
    op.stop = stop;
    run_csr(M, op, k, red, s, {base, op.base.b, x, out});
  }

  // Level 0 without a post-smoother but with a mask or a fused CG dot: finish with an
  // elementwise pass dst = src (active columns) that also reduces <r, z>.
  template <class TR, bool DOT>
  void elem_copy_t(int n, const T* src, T* dst, bool mask) {
    OpMaskCopy<T, TR, DOT> op{};
    op.src = src;
    op.dst = dst;
    op.active = mask ? pl->active() : nullptr;
    op.ld = k;
    op.stop = stop;
    op.rdot = static_cast<const TR*>(fine_dot);
    op.gamma = pl->gamma();
    op.beta = pl->beta();
    run_elem<T>(n, op, k, red, s, {src, dst, fine_dot});
  }
  void elem_copy(int n, const T* src, T* dst, bool mask, bool dot) {
    if (!dot) elem_copy_t<double, false>(n, src, dst, mask);
    else if (dot_is_f64) elem_copy_t<double, true>(n, src, dst, mask);
    else elem_copy_t<float, true>(n, src, dst, mask);
  }

  void norm_only(int l, const T* xp) {
    OpResid<T, T, XS_PLAIN, false, T, true> op{};
    op.xs = xsrc<XS_PLAIN>(l, xp, T(1));
    op.b = Bb(l);
    op.out = nullptr;
    op.out_lo = nullptr;
    op.ld = k;
    op.stop = nullptr;
    op.ctl = ctl;
    run_csr(Aof(l), op, k, red, s, {xp, Bb(l)});
  }

  void coarse_solve(const T* b, T* x) {
    const Coarse& c = h->coarse;
    const int l = L() - 1;
    const int n = h->levels[l].A.n_rows;
    const int tot = n * k;
    const int grid = std::max(1, std::min((tot + 127) / 128, dev_info().max_ctas));
    if (rec) {
      if (c.kind != AMG_COARSE_PINV) fail(AMG_ERR_INVALID_ARG, "internal: coarse solver not recordable");
      PStep st{};
      st.kind = PK_GEMV;
      st.n_rows = n;
      st.val = c.template m0<T>();
      st.b = b;
      st.out = x;
      st.barrier = 1;
      rec->push_back(st);
      return;
    }
    if (c.kind == AMG_COARSE_PINV) {
      launch(coarse_gemv<T>, grid, 128, 0, s, c.template m0<T>(), (const T*)b, x, n, k, 0, stop);
    } else if (c.kind == AMG_COARSE_LU) {
      launch(coarse_trsv<T, 0>, (k + 63) / 64, 64, 0, s, c.template m0<T>(), c.perm, (const T*)b, x, n, k, stop);
    } else if (c.kind == AMG_COARSE_QR) {
      launch(coarse_gemv<T>, grid, 128, 0, s, c.template m0<T>(), (const T*)b, x, n, k, 1, stop);
      launch(coarse_trsv<T, 1>, (k + 63) / 64, 64, 0, s, c.template m1<T>(), (const int*)nullptr, (const T*)x, x, n, k, stop);
    } else {  // Jacobi sweeps from zero on the coarsest operator
      const T om = T(c.omega);
      // level l's own right-hand side buffer is b (== B[l]); sweeps read Bb(l)
      if (c.iters <= 0) {
        OpJac0<T> z{b, h->levels[l].template dinv<T>(), T(0), x, k, stop};
        run_elem<T>(n, z, k, red, s, {b, x});
      } else if (c.iters == 1) {
        OpJac0<T> z{b, h->levels[l].template dinv<T>(), om, x, k, stop};
        run_elem<T>(n, z, k, red, s, {b, x});
      } else {
        sweeps(l, XD<T>::jac0(), c.iters - 1, om, x, W1(l), W2(l), false, false, false);
      }
    }
    CK_LAUNCH();
  }

  // One visit of level l (multilevel.py:316-337).  x_zero: the incoming iterate is 0.
  // On return the new iterate is in Xb(l).
  void visit(int l, bool x_zero, char ct, int cpl) {
    NvtxRange nv("amg/L%d/%c", l, ct);
    if (!rec && l > 0 && l == tail_from) {  // this level and all below: one persistent program
      std::vector<PStep> steps;
      rec = &steps;
      try {
        visit(l, x_zero, ct, cpl);
      } catch (...) {
        rec = nullptr;
        throw;
      }
      rec = nullptr;
      emit_program(steps);
      return;
    }
    const Level& lv = h->levels[l];
    const int n = lv.A.n_rows;
    T* X = Xb(l);
    const T* B = Bb(l);
    T* w1 = W1(l);
    T* w2 = W2(l);
    const bool top = (l == 0);

    // ---- one right-hand side on a small level (fuse2_level), iterate zero, one pre- and one
    // post-sweep: two passes per level instead of four (two-hop sources): b_c = R (B - A x1)
    // with x1 = omega D^-1 B evaluated per gathered row, then, after the coarse correction,
    // X = sweep(x1 + P x_c) with x1 + P x_c evaluated per gathered row.
    if (x_zero && !rec && fuse2_level(lv, Aof(l), k) && lv.pre.on() && lv.pre.iters == 1 &&
        lv.post.on() && lv.post.iters == 1 && lv.template dinv<T>()) {
      const T* dv = lv.template dinv<T>();
      const T om_pre = T(lv.pre.omega);
      const Csr& A = Aof(l);
      T* Bc = static_cast<T*>(pl->B[l + 1]);
      T* Xc = static_cast<T*>(pl->X[l + 1]);
      {
        OpRestrictX<T, XS_RESJ0> rop{};
        rop.xs = XSource<T, XS_RESJ0>{nullptr, B, dv, om_pre, k, A.rowptr, A.col, A.template vals<T>(), nullptr};
        rop.out = Bc; rop.ld = k; rop.stop = stop;
        run_csr(lv.R, rop, k, red, s, {B, Bc});
      }
      if (l == L() - 2) coarse_solve(Bc, Xc);
      else if (ct == 'V') visit(l + 1, true, 'V', cpl);
      else if (ct == 'W') { visit(l + 1, true, 'W', cpl); visit(l + 1, false, 'W', cpl); }
      else { visit(l + 1, true, 'F', cpl); for (int i = 0; i < cpl; ++i) visit(l + 1, false, 'V', cpl); }
      const bool mask = top && fine_mask, dot = top && fine_dot != nullptr;
      OpJacobi<T, XS_PROJ0> op{};
      op.xs = XSource<T, XS_PROJ0>{nullptr, B, dv, om_pre, k, lv.P.rowptr, lv.P.col, lv.P.template vals<T>(), Xc};
      op.b = B; op.dinv = dv; op.omega = T(lv.post.omega); op.out = X; op.ld = k;
      op.norm = 0;
      op.active = mask ? pl->active() : nullptr;
      op.stop = stop;
      op.rdot64 = (dot && dot_is_f64) ? static_cast<const double*>(fine_dot) : nullptr;
      op.rdot32 = (dot && !dot_is_f64) ? static_cast<const float*>(fine_dot) : nullptr;
      op.ctl = ctl;
      op.gamma = pl->gamma();
      op.beta = pl->beta();
      run_csr(A, op, k, red, s, {B, X, dot ? fine_dot : nullptr});
      return;
    }

    // ---- pre-smoothing (x1)
    XD<T> x1 = x_zero ? XD<T>::zero() : XD<T>::plain(X);
    const bool fuse_norm = top && fine_norm && !x_zero && lv.pre.on();
    if (top && fine_norm && !fuse_norm) norm_only(0, x_zero ? nullptr : X);
    if (lv.pre.on()) {
      const T om = T(lv.pre.omega);
      if (x_zero) {
        if (lv.pre.iters == 1) x1 = XD<T>::jac0();
        else {
          sweeps(l, XD<T>::jac0(), lv.pre.iters - 1, om, w1, w2, w1, false, false, false);
          x1 = XD<T>::plain(w1);
        }
      } else {
        sweeps(l, XD<T>::plain(X), lv.pre.iters, om, w1, w2, w1, fuse_norm, false, false);
        x1 = XD<T>::plain(w1);
      }
    }
    const T om_pre = T(lv.pre.omega);

    // ---- residual and restriction: b_c = R (b - A x1)
    const T* r = B;
    if (x1.kind != XS_ZERO) {
      if (x1.kind == XS_PLAIN) resid_t<XS_PLAIN, false>(l, x1.p, om_pre, B, w2);
      else resid_t<XS_JAC0, false>(l, nullptr, om_pre, B, w2);
      r = w2;
    }
    T* Bc = static_cast<T*>(pl->B[l + 1]);
    axpy_t<XS_ZERO>(lv.R, nullptr, T(0), l, r, Bc);

    // ---- coarse correction
    T* Xc = static_cast<T*>(pl->X[l + 1]);
    if (l == L() - 2) {
      coarse_solve(Bc, Xc);
    } else if (ct == 'V') {
      visit(l + 1, true, 'V', cpl);
    } else if (ct == 'W') {
      visit(l + 1, true, 'W', cpl);
      visit(l + 1, false, 'W', cpl);
    } else {
      visit(l + 1, true, 'F', cpl);
      for (int i = 0; i < cpl; ++i) visit(l + 1, false, 'V', cpl);
    }

    // ---- prolongation + correction: x2 = x1 + P x_c
    const bool post_on = lv.post.on();
    const bool need_fix = top && (fine_mask || fine_dot) && !post_on;
    T* dst2 = (post_on || need_fix) ? w1 : X;
    if (x1.kind == XS_PLAIN) axpy_t<XS_PLAIN>(lv.P, x1.p, T(0), l, Xc, dst2);
    else if (x1.kind == XS_JAC0) axpy_t<XS_JAC0>(lv.P, nullptr, om_pre, l, Xc, dst2);
    else axpy_t<XS_ZERO>(lv.P, nullptr, T(0), l, Xc, dst2);

    // ---- post-smoothing into X
    if (post_on) {
      sweeps(l, XD<T>::plain(w1), lv.post.iters, T(lv.post.omega), X, w2, w1, false,
             top && fine_mask, top && fine_dot != nullptr);
    } else if (need_fix) {
      elem_copy(n, w1, X, fine_mask, fine_dot != nullptr);
    }
  }
};


// ------------------------------------------------------------------ runtime (amg_runtime.cu)
using Emit = std::function<void(cudaStream_t)>;
Plan* get_plan(amg_hierarchy* h, int prec, int k, cudaStream_t s);
// Plans (and padding stages) a hierarchy keeps: AMG_MAX_PLANS, default 16, at least 2.  A
// request for a new (precision, k, stream) beyond it frees the least recently requested one
// after a device synchronisation (its graphs may still be running on its stream).
int max_plans();
void run_loop(Plan* pl, const std::string& key, cudaStream_t user, const Emit& prologue,
              const Emit& body, const Emit& epilogue, bool has_loop, int gmax);
void read_results(Plan* pl, cudaStream_t s, bool cg, int32_t* iters_out, double* relres_out);
LoopCtl make_ctl(Plan* pl, int maxiter);
Red red_of(Plan* pl);
char cycle_char(int cycle);
void check_prec_data(amg_hierarchy* h, int prec, const Csr* A0);
Csr override_csr(amg_hierarchy* h, const amg_csr* A0, cudaStream_t s);
void check_vec(const void* p, const char* name);

struct Req {
  int prec, k, cycle, cpl, maxiter;
  double tol, atol;
  const void* b;
  void* x;
  const Csr* A0;
  bool program = false;  // the cycle's coarse levels may run as one persistent program
};

// First level of a cycle run as a persistent program, or -1: programs on, allowed for this
// request, at least one level between the finest and the coarsest, a pinv coarse solve, and
// a column layout the program's row loops cover (k = 1, or G = k / KV lanes <= 32 with
// KV = 16 bytes when it divides k, else 1).  AMG_PROGRAM_FROM picks the level (default 1).
template <class T>
int tail_level(const amg_hierarchy* h, int k, bool allowed) {
  if (!allowed || !programs_enabled()) return -1;
  if (h->levels.size() < 3 || h->coarse.kind != AMG_COARSE_PINV) return -1;
  if (k > 1) {
    const int kv16 = 16 / int(sizeof(T));
    const int kv = (k % kv16 == 0) ? kv16 : 1;
    if ((k / kv) > 32) return -1;
  }
  static const int from = [] {
    const char* e = std::getenv("AMG_PROGRAM_FROM");
    const int v = e ? atoi(e) : 1;
    return v >= 1 ? v : 1;
  }();
  return from <= int(h->levels.size()) - 2 ? from : -1;
}

std::string req_key(const char* kind, const Req& q);

template <class T, class TLO, int MODE>
inline void emit_setup(Plan* pl, cudaStream_t cs, int n0, const T* b, T* dst, TLO* dst_lo, T* zero,
                       double tol, double atol, int maxiter) {
  OpSetup<T, TLO, MODE> op{};
  op.src = b;
  op.dst = dst;
  op.dst_lo = dst_lo;
  op.zero = zero;
  op.ld = pl->k;
  op.thresh = pl->thresh();
  op.nr = pl->nr();
  op.normb = pl->normb();
  op.active = pl->active();
  op.iters = pl->iters();
  op.stop = pl->stop();
  op.gcount = pl->gcount();
  op.tol = tol;
  op.atol = atol;
  op.maxiter = maxiter;
  run_elem<TLO>(n0, op, pl->k, red_of(pl), cs, {b, dst, dst_lo, zero});
}

// ------------------------------------------------------------------ drivers
template <class T> void solve_plain(amg_hierarchy* h, Plan* pl, const Req& q, cudaStream_t user);
void solve_mixed(amg_hierarchy* h, Plan* pl, const Req& q, cudaStream_t user);
void solve_mixed_ru(amg_hierarchy* h, Plan* pl, const Req& q, cudaStream_t user);
template <class TO, class TC> void pcg(amg_hierarchy* h, Plan* pl, const Req& q, cudaStream_t user);
template <class TO, class TC>
void pcg_emit(amg_hierarchy* h, Plan* pl, const Req& q, cudaStream_t user, Emit* pro, Emit* bod);
template <class TC>
void pcg_ru_emit(amg_hierarchy* h, Plan* pl, const Req& q, cudaStream_t user, Emit* pro, Emit* bod, Emit* epi);
void pcg_ru(amg_hierarchy* h, Plan* pl, const Req& q, cudaStream_t user);
// Threshold of the reliable-update CG: a true residual is due once the FP32 residual norm
// has dropped by this factor since the last one (AMG_RU_DELTA, default 1e-2); squared.
double ru_delta2();
bool is_mixed(int prec);

// One system of a batch: its plan and its emitters (prologue, loop body).
struct BatchSys {
  Plan* pl;
  Emit pro, body, epi;  // epi: nullable, after the loop
  int gmax;
};
// Capture (once per key) and launch one graph holding every system's loop as an independent
// branch (its own conditional WHILE node), so one launch solves them all concurrently.
void run_batch(const std::vector<BatchSys>& systems, const std::string& key, cudaStream_t user);
template <class T> void precondition(amg_hierarchy* h, Plan* pl, const Req& q, cudaStream_t user);

// per-translation-unit kernel counters (each TU owns a copy of g_kernel_count)
unsigned long long count_f64();
unsigned long long count_f32();
unsigned long long count_mixed();
unsigned long long count_mixed_cg();
unsigned long long count_runtime();
unsigned long long count_capi();
unsigned long long count_program();

}  // namespace amg
