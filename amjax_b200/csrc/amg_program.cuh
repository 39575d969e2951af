// amg_program.cuh -- persistent execution of a cycle's coarse levels.
//
// Below the finest level an AMG cycle is a chain of small dependent CSR passes (residual,
// restriction, coarse solve, prolongation, smoothing on levels of a few thousand rows);
// launched one by one, each costs a kernel launch and a drain of the GPU for a few
// microseconds of work.  A "program" records that chain at capture time as a list of
// steps (one fused CSR pass of one level each, the same epilogue ops as the launched
// kernels), and one cooperative launch runs the list: every CTA takes its share of a
// step's rows, then waits at a grid-wide barrier before the next dependent step.  Steps
// marked without a barrier are independent of the next one (several systems of a batch)
// and run back to back.  The row loops keep the launched kernels' multiply-add order, so
// a program gives bit-identical results to the launches it replaces.
//
// Opt-in (AMG_PROGRAM=1; see programs_enabled).  The barrier wait is bounded (a clock64
// budget, AMG_SPIN_LIMIT cycles, default 2^31, about 1 s): a CTA that runs out sets the
// status word and returns, the others see the status at their next barrier and return too,
// and the host reports AMG_ERR_TIMEOUT.
#pragma once

#include "amg_device.cuh"

namespace amg {

enum PKind : int {
  PK_JAC_PLAIN = 0,  // out = Jacobi sweep of x (OpJacobi, stored x)
  PK_JAC_J0 = 1,     // out = Jacobi sweep of the one-sweep-from-zero iterate (OpJacobi, XS_JAC0)
  PK_RES_PLAIN = 2,  // out = b - A x (OpResid, stored x)
  PK_RES_J0 = 3,     // out = b - A x1, x1 one sweep from zero (OpResid, XS_JAC0)
  PK_AXPY_ZERO = 4,  // out = M x (restriction)
  PK_AXPY_PLAIN = 5, // out = base + M x (prolongation + correction, stored base)
  PK_AXPY_J0 = 6,    // out = x1 + M x, x1 one sweep from zero
  PK_GEMV = 7        // out = M b, M dense n x n row-major (pinv coarse solve)
};

// One step.  Field use per kind, mirroring the launched ops' fields:
//   Jacobi / residual: x = iterate, b = the level's right-hand side, dinv, omega, out;
//   axpy: x = the SpMV operand, base = stored base iterate, b / dinv / omega = the base
//         level's right-hand side, inverse diagonal and damping (XS_JAC0 base), out;
//   gemv: val = the dense matrix, b = right-hand side, out = solution, n_rows = n.
struct PStep {
  int kind;
  int n_rows;
  int g;        // lanes per row (k == 1: lanes sharing a row's nonzeros; k > 1: column lanes)
  int kv;       // vector width (k > 1)
  int barrier;  // a grid barrier follows this step
  const int* rowptr;
  const int* col;
  const void* val;
  const void* x;
  const void* b;
  const void* dinv;
  const void* base;
  void* out;
  double omega;
};

constexpr int kMaxSteps = 64;  // steps per launch (the list travels as a kernel parameter)

struct Program {
  int nsteps;
  PStep steps[kMaxSteps];
};

// Barrier state: a top-level count, the generation, the status word, then one count per
// group of kBarGroup consecutive CTAs, kBarStride words apart (own 128-byte line each).
constexpr int kBarGroup = 8;
constexpr int kBarStride = 32;
constexpr int kBarMaxCtas = 2048;
constexpr int kBarWords = 4 + kBarStride * (kBarMaxCtas / kBarGroup);

struct GridBar {
  unsigned* count;   // groups arrived at the current barrier
  unsigned* gen;     // barrier generation
  int* status;       // nonzero: a wait ran out (the launch gave up)
  unsigned* groups;  // per-group arrival counts
  long long limit;   // clock64 budget of one wait
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier of a cooperative launch (every CTA resident), two levels: the CTAs of
// a group of kBarGroup arrive on the group's own counter, and the last of each group
// arrives on the top-level counter for all of them (one contended atomic per group, not
// per CTA); the last group bumps the generation that every CTA waits on.  Returns false
// when a wait ran out here or in another CTA; the caller then returns.
__device__ __forceinline__ bool grid_sync(const GridBar& gb) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = *reinterpret_cast<volatile int*>(gb.status) == 0;
    if (ok) {
      const unsigned g0 = ld_acquire_u32(gb.gen);
      const unsigned grp = blockIdx.x / kBarGroup;
      const unsigned gsize = min(unsigned(kBarGroup), gridDim.x - grp * kBarGroup);
      const unsigned ngroups = (gridDim.x + kBarGroup - 1) / kBarGroup;
      unsigned* gc = gb.groups + size_t(grp) * kBarStride;
      __threadfence();
      bool last = false;
      if (atomicAdd(gc, 1u) == gsize - 1) {
        atomicExch(gc, 0u);
        __threadfence();
        last = atomicAdd(gb.count, 1u) == ngroups - 1;
      }
      if (last) {
        atomicExch(gb.count, 0u);
        __threadfence();
        atomicAdd(gb.gen, 1u);
      } else {
        const long long t0 = clock64();
        while (ld_acquire_u32(gb.gen) == g0) {
          if (clock64() - t0 > gb.limit || *reinterpret_cast<volatile int*>(gb.status) != 0) {
            atomicOr(gb.status, 1);
            ok = 0;
            break;
          }
          __nanosleep(32);
        }
      }
      __threadfence();
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// k == 1 rows of one step: the csr_k1 mapping with a run-time G (same nonzero split and
// shuffle order as csr_k1<Op, G>).
template <class Op>
__device__ __forceinline__ void prog_rows1(const Op& op, const PStep& st, int gtid, int nth) {
  using A = typename Op::Acc;
  using V = typename Op::V;
  const int G = st.g;
  const int lane = gtid & (G - 1);
  const int wl = threadIdx.x & 31;
  const int grp = gtid / G;
  const int ngrp = nth / G;
  const V* __restrict__ val = static_cast<const V*>(st.val);
  for (int row = grp; row - wl / G < st.n_rows; row += ngrp) {
    A acc = A(0);
    const bool valid = row < st.n_rows;
    if (valid) {
      const int s = __ldg(st.rowptr + row), e = __ldg(st.rowptr + row + 1);
      for (int nz = s + lane; nz < e; nz += G) acc = rfma(static_cast<A>(__ldg(val + nz)), op.x1(__ldg(st.col + nz)), acc);
    }
    for (int off = G >> 1; off > 0; off >>= 1) acc = radd(acc, __shfl_xor_sync(0xffffffffu, acc, off, G));
    if (valid && lane == 0) op.epi1(row, acc);
  }
}

// k > 1 rows of one step: G lanes per row, each one KV-wide column chunk (the lean csr_kr
// mapping with one row in flight; same multiply-add order).
template <class Op, int KV>
__device__ __forceinline__ void prog_rowsk(const Op& op, const PStep& st, int k, int gtid, int nth) {
  using A = typename Op::Acc;
  using V = typename Op::V;
  const int G = st.g;
  const int lane = gtid & (G - 1);
  const int grp = gtid / G;
  const int ngrp = nth / G;
  const int c0 = lane * KV;
  if (c0 >= k) return;
  const V* __restrict__ val = static_cast<const V*>(st.val);
  for (int row = grp; row < st.n_rows; row += ngrp) {
    const int s = __ldg(st.rowptr + row), e = __ldg(st.rowptr + row + 1);
    PreT<A, KV> pre;
    op.template prek<KV>(row, c0, pre);
    A acc[KV];
    if (s < e) {
      const int c1 = __ldg(st.col + s);
      const A a1 = static_cast<A>(__ldg(val + s));
      A xv[KV];
      op.template xk<KV>(c1, c0, xv);
#pragma unroll
      for (int v = 0; v < KV; ++v) acc[v] = fma(a1, xv[v], A(0));
    } else {
#pragma unroll
      for (int v = 0; v < KV; ++v) acc[v] = A(0);
    }
#pragma unroll 4
    for (int nz = s + 1; nz < e; ++nz) {
      const int cj = __ldg(st.col + nz);
      const A a = static_cast<A>(__ldg(val + nz));
      A xv[KV];
      op.template xk<KV>(cj, c0, xv);
#pragma unroll
      for (int v = 0; v < KV; ++v) acc[v] = fma(a, xv[v], acc[v]);
    }
    double unused[KV];
    op.template epik<KV>(row, c0, acc, pre, unused);
  }
}

template <class T, class Op>
__device__ __forceinline__ void prog_run(const Op& op, const PStep& st, int k, int gtid, int nth) {
  if (k == 1) {
    prog_rows1(op, st, gtid, nth);
  } else if (st.kv == 1) {
    prog_rowsk<Op, 1>(op, st, k, gtid, nth);
  } else {
    prog_rowsk<Op, 16 / sizeof(T)>(op, st, k, gtid, nth);
  }
}

template <class T>
__device__ void prog_step(const PStep& st, int k, int gtid, int nth) {
  const T* x = static_cast<const T*>(st.x);
  const T* b = static_cast<const T*>(st.b);
  const T* dv = static_cast<const T*>(st.dinv);
  T* out = static_cast<T*>(st.out);
  const T om = T(st.omega);
  switch (st.kind) {
    case PK_JAC_PLAIN:
    case PK_JAC_J0: {
      if (st.kind == PK_JAC_PLAIN) {
        OpJacobi<T, XS_PLAIN> op{};
        op.xs = XSource<T, XS_PLAIN>{x, b, dv, om, k};
        op.b = b; op.dinv = dv; op.omega = om; op.out = out; op.ld = k;
        prog_run<T>(op, st, k, gtid, nth);
      } else {
        OpJacobi<T, XS_JAC0> op{};
        op.xs = XSource<T, XS_JAC0>{nullptr, b, dv, om, k};
        op.b = b; op.dinv = dv; op.omega = om; op.out = out; op.ld = k;
        prog_run<T>(op, st, k, gtid, nth);
      }
      break;
    }
    case PK_RES_PLAIN: {
      OpResid<T, T, XS_PLAIN, true, T, false> op{};
      op.xs = XSource<T, XS_PLAIN>{x, b, dv, om, k};
      op.b = b; op.out = out; op.out_lo = nullptr; op.ld = k;
      prog_run<T>(op, st, k, gtid, nth);
      break;
    }
    case PK_RES_J0: {
      OpResid<T, T, XS_JAC0, true, T, false> op{};
      op.xs = XSource<T, XS_JAC0>{nullptr, b, dv, om, k};
      op.b = b; op.out = out; op.out_lo = nullptr; op.ld = k;
      prog_run<T>(op, st, k, gtid, nth);
      break;
    }
    case PK_AXPY_ZERO: {
      OpAxpy<T, XS_ZERO> op{};
      op.base = XSource<T, XS_ZERO>{nullptr, b, dv, om, k};
      op.x = x; op.out = out; op.ld = k;
      prog_run<T>(op, st, k, gtid, nth);
      break;
    }
    case PK_AXPY_PLAIN: {
      OpAxpy<T, XS_PLAIN> op{};
      op.base = XSource<T, XS_PLAIN>{static_cast<const T*>(st.base), b, dv, om, k};
      op.x = x; op.out = out; op.ld = k;
      prog_run<T>(op, st, k, gtid, nth);
      break;
    }
    case PK_AXPY_J0: {
      OpAxpy<T, XS_JAC0> op{};
      op.base = XSource<T, XS_JAC0>{nullptr, b, dv, om, k};
      op.x = x; op.out = out; op.ld = k;
      prog_run<T>(op, st, k, gtid, nth);
      break;
    }
    case PK_GEMV: {  // coarse_gemv's order: s += M[i, j] * b[j, c] for j = 0 .. n-1
      const T* M = static_cast<const T*>(st.val);
      const int n = st.n_rows;
      for (int t = gtid; t < n * k; t += nth) {
        const int i = t / k, c = t % k;
        T s = T(0);
        for (int j = 0; j < n; ++j) s = rfma(M[(size_t)i * n + j], b[(size_t)j * k + c], s);
        out[(size_t)i * k + c] = s;
      }
      break;
    }
    default:
      break;
  }
}

// Host side (amg_program.cu).
// Grid of a program launch: every CTA resident (SMs x resident CTAs of the kernel).
int program_grid(bool f64);
// Launch one program (cooperative) on stream s; stop (nullable): the loop's stop flag,
// checked once at the start (the whole program returns when set).
void launch_program(const Program& p, bool f64, int k, const int* stop, const GridBar& gb, cudaStream_t s);
// Clock budget of one barrier wait (AMG_SPIN_LIMIT, default 2^31 cycles).
long long spin_limit();
// Programs on: AMG_PROGRAM=1.  Off by default: measured on B200 at N = 250,000 (k = 1 and
// k = 64, FP64 and mixed), a program step with its grid barrier cost more than the
// graph-launched kernel it replaces (the barrier's serialised L2 round trips across the
// two dies exceed a PDL-overlapped launch), so solves were 12-60 % slower with programs.
bool programs_enabled();
unsigned long long count_program();

}  // namespace amg
