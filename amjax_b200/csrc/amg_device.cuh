// amg_device.cuh -- sm_100a kernels of the multigrid solve phase.
//
// Every SpMV-class kernel is one CSR pass with a fused epilogue ("Op").  Two thread
// mappings cover the two layouts of the right-hand sides:
//   * k == 1 (one RHS): G threads share a row's nonzeros (G = 1..32 picked from the
//     row-length distribution) and reduce with warp shuffles;
//   * k >  1 (X stored [n, k], k contiguous): G lanes split the k columns of a row in
//     KV-wide vectors (16-byte loads), so every gathered x row is read coalesced.
// Column-wise sums (norms, dots) are reduced deterministically: each CTA writes one
// partial per column, and the last CTA to finish (ticket counter) sums them in a fixed
// order and runs the Op's scalar update (step lengths, convergence flags, and the
// condition value of the CUDA-graph while-loop).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace amg {

constexpr int kBlock = 256;     // threads per CTA for every grid kernel
constexpr int kMaxCh = 4;       // column chunks per lane (k <= 32 * kMaxCh * KV)

// Kernels launched (every CTA 0 / thread 0 of every kernel adds one): the launch count
// the benchmark reports is read from here, so it counts what actually ran.
static __device__ unsigned long long g_kernel_count = 0;

// Kernel entry: wait for the preceding grid (programmatic dependent launch: this grid may
// have been launched while its predecessor was still finishing; griddepcontrol.wait
// returns once the predecessor has completed and its memory is visible, and at once when
// there is no programmatic predecessor), then let the next grid start launching, and
// count the launch.
__device__ __forceinline__ void count_launch() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&g_kernel_count, 1ull);
}

// ------------------------------------------------------------------ vector access
// Element offset of (row j, column c) in a [rows, ld] array.  Rows, columns and ld are
// non-negative int32, so one unsigned 32 x 32 -> 64-bit multiply-add forms it (a signed
// 64-bit product costs more instructions per gathered row).
__device__ __forceinline__ size_t voff(int j, int ld, int c) {
  return static_cast<size_t>(static_cast<unsigned long long>(static_cast<unsigned>(j)) * static_cast<unsigned>(ld)) +
         static_cast<unsigned>(c);
}


// Arithmetic with its rounding spelled out.  Every multiply, add and fused multiply-add in
// the ops goes through these, so no kernel's compilation can pick a different contraction
// (a*b + c*d can fuse either product) and every kernel that runs an op -- any lane layout,
// the launched kernels or the persistent program -- rounds it the same way.
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float rfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double rfma(double a, double b, double c) { return __fma_rn(a, b, c); }

// 32-byte accesses (sm_100: one 256-bit load or store per thread), used by the wide lean
// kernel; the address must be 32-byte aligned (the launch configuration checks every
// pointer and the row stride).  The load takes the read-only path: every CSR-op operand
// it serves is either never written by the kernel or read by its owner before it writes it.
__device__ __forceinline__ void ld32(const float* p, float* v) {
  asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
      : "l"(p));
}
__device__ __forceinline__ void ld32(const double* p, double* v) {
  asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3]) : "l"(p));
}
__device__ __forceinline__ void st32(float* p, const float* v) {
  asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "f"(v[0]), "f"(v[1]), "f"(v[2]),
               "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7])
               : "memory");
}
__device__ __forceinline__ void st32(double* p, const double* v) {
  asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(v[0]), "d"(v[1]), "d"(v[2]), "d"(v[3])
               : "memory");
}

template <class T, int KV>
__device__ __forceinline__ void ld_vec(const T* __restrict__ p, T (&v)[KV]) {
  if constexpr (sizeof(T) * KV >= 32 && (sizeof(T) * KV) % 32 == 0) {
    constexpr int n = 32 / sizeof(T);
#pragma unroll
    for (int h = 0; h < KV; h += n) ld32(p + h, v + h);
  } else if constexpr (sizeof(T) * KV == 16) {
    if constexpr (sizeof(T) == 8) {
      double2 t = *reinterpret_cast<const double2*>(p); v[0] = t.x; v[1] = t.y;
    } else {
      float4 t = *reinterpret_cast<const float4*>(p); v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    }
  } else if constexpr (sizeof(T) * KV == 8 && sizeof(T) == 4) {
    float2 t = *reinterpret_cast<const float2*>(p); v[0] = t.x; v[1] = t.y;
  } else {
#pragma unroll
    for (int i = 0; i < KV; ++i) v[i] = p[i];
  }
}

template <class T, int KV>
__device__ __forceinline__ void st_vec(T* __restrict__ p, const T (&v)[KV]) {
  if constexpr (sizeof(T) * KV >= 32 && (sizeof(T) * KV) % 32 == 0) {
    constexpr int n = 32 / sizeof(T);
#pragma unroll
    for (int h = 0; h < KV; h += n) st32(p + h, v + h);
  } else if constexpr (sizeof(T) * KV == 16) {
    if constexpr (sizeof(T) == 8) {
      *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
    } else {
      *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    }
  } else if constexpr (sizeof(T) * KV == 8 && sizeof(T) == 4) {
    *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
  } else {
#pragma unroll
    for (int i = 0; i < KV; ++i) p[i] = v[i];
  }
}

// Load KV values of type S and widen/narrow to T.
template <class T, class S, int KV>
__device__ __forceinline__ void ld_cvt(const S* __restrict__ p, T (&v)[KV]) {
  if constexpr (sizeof(S) == sizeof(T)) {
    ld_vec<T, KV>(reinterpret_cast<const T*>(p), v);
  } else {
    S t[KV];
    ld_vec<S, KV>(p, t);
#pragma unroll
    for (int i = 0; i < KV; ++i) v[i] = static_cast<T>(t[i]);
  }
}

// ------------------------------------------------------------------ reductions
// Epilogue operands of one (row, column-chunk), loaded ahead of the row's gathers so
// their latency overlaps them (fields an op does not use are optimised away).
template <class T, int KV>
struct PreT {
  T x[KV];
  T b[KV];
  T c[KV];
  T d;
};

struct RedCtx {
  double* partials;    // [gridDim.x * k]
  unsigned* counter;   // ticket counter, left at 0 after every kernel
  int k;
};

constexpr int kRedGroups = 16;  // first-level groups of CTAs in the grid reduction

// Sum nparts partial rows (stride k) for every column with all threads of the CTA; the
// per-column order is fixed (deterministic).  Thread (slice sl, column ci) strides over
// parts; slices are combined by a shared-memory tree.  Results for columns cb..cb+kc
// land in sbuf[0..kc).
__device__ __forceinline__ void sum_parts(const double* parts, int nparts, int k, int cb, int kc,
                                          double* sbuf) {
  const int nsl = kBlock / kc;
  const int ci = threadIdx.x % kc, sl = threadIdx.x / kc;
  const int c = cb + ci;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  if (c < k) {
    int b = sl;
    for (; b + 3 * nsl < nparts; b += 4 * nsl) {
      a0 += __ldcg(parts + (size_t)b * k + c);
      a1 += __ldcg(parts + (size_t)(b + nsl) * k + c);
      a2 += __ldcg(parts + (size_t)(b + 2 * nsl) * k + c);
      a3 += __ldcg(parts + (size_t)(b + 3 * nsl) * k + c);
    }
    for (; b < nparts; b += nsl) a0 += __ldcg(parts + (size_t)b * k + c);
  }
  sbuf[threadIdx.x] = (a0 + a1) + (a2 + a3);
  __syncthreads();
  for (int st = nsl >> 1; st > 0; st >>= 1) {
    if (sl < st) sbuf[sl * kc + ci] += sbuf[(sl + st) * kc + ci];
    __syncthreads();
  }
}

// Grid reduction, two levels, deterministic: CTAs are split into kRedGroups contiguous
// groups; the last CTA of a group (ticket counter) sums the group's partials into a
// group row; the last group to finish sums the group rows, then calls
// op.finalize_col(c, sum) for every column and op.finalize_all(any) once.
// partials: [gridDim.x][k] CTA rows followed by [kRedGroups][k] group rows;
// counter: [0] groups done, [1 + g] CTAs done in group g (all left at 0).
template <class Op>
__device__ __forceinline__ void grid_finish(const Op& op, const RedCtx& rc, double* sbuf) {
  __shared__ unsigned s_last;
  const int k = rc.k;
  const int nb = gridDim.x;
  const int ng = nb < kRedGroups ? nb : kRedGroups;
  const int gsz = (nb + ng - 1) / ng;
  const int g = blockIdx.x / gsz;
  const int g0 = g * gsz;
  const int gn = min(gsz, nb - g0);
  const int ngroups = (nb + gsz - 1) / gsz;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(rc.counter + 1 + g, 1u) == (unsigned)(gn - 1)) ? 1u : 0u;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  int kc = 1;
  while (kc < k && kc < kBlock) kc <<= 1;
  double* grow = rc.partials + (size_t)nb * k;
  for (int cb = 0; cb < k; cb += kc) {
    sum_parts(rc.partials + (size_t)g0 * k, gn, k, cb, kc, sbuf);
    if (threadIdx.x < kc && cb + threadIdx.x < k) grow[(size_t)g * k + cb + threadIdx.x] = sbuf[threadIdx.x];
    __syncthreads();
  }
  if (threadIdx.x == 0) rc.counter[1 + g] = 0u;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(rc.counter, 1u) == (unsigned)(ngroups - 1)) ? 1u : 0u;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  int any = 0;
  for (int cb = 0; cb < k; cb += kc) {
    sum_parts(grow, ngroups, k, cb, kc, sbuf);
    if (threadIdx.x < kc && cb + threadIdx.x < k) any |= op.finalize_col(cb + threadIdx.x, sbuf[threadIdx.x]);
    __syncthreads();
  }
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) {
    op.finalize_all(any);
    rc.counter[0] = 0u;
  }
}

// CTA-level reduction of one value per thread (k == 1) -> partials[blockIdx.x].
template <class Op>
__device__ __forceinline__ void block_reduce_1(const Op& op, const RedCtx& rc, double v) {
  __shared__ double sbuf[kBlock];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  if ((threadIdx.x & 31) == 0) sbuf[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kBlock / 32; ++w) s += sbuf[w];
    rc.partials[blockIdx.x] = s;
  }
  __syncthreads();
  grid_finish(op, rc, sbuf);
}

// CTA-level reduction for k > 1: thread (grp, lane) owns columns (lane + j*G)*KV + v.
template <class Op, int G, int KV, int NCH>
__device__ __forceinline__ void block_reduce_k(const Op& op, const RedCtx& rc,
                                               const double (&red)[NCH][KV]) {
  extern __shared__ double dyn[];   // (kBlock / G) * k doubles
  const int k = rc.k;
  const int lane = threadIdx.x % G, grp = threadIdx.x / G;
  const int nchunks = k / KV;
#pragma unroll
  for (int j = 0; j < NCH; ++j) {
    const int ch = lane + j * G;
    if (ch < nchunks) {
#pragma unroll
      for (int v = 0; v < KV; ++v) dyn[grp * k + ch * KV + v] = red[j][v];
    }
  }
  __syncthreads();
  for (int c = threadIdx.x; c < k; c += kBlock) {
    double s = 0.0;
    for (int g = 0; g < kBlock / G; ++g) s += dyn[g * k + c];
    rc.partials[(size_t)blockIdx.x * k + c] = s;
  }
  __syncthreads();
  grid_finish(op, rc, dyn);   // dyn holds >= kBlock doubles (k*kBlock/G >= kBlock)
}

// ------------------------------------------------------------------ CSR kernels
// k == 1: G threads per row split the nonzeros.
template <class Op, int G>
__global__ void __launch_bounds__(kBlock)
csr_k1(const int* __restrict__ rowptr, const int* __restrict__ col,
       const typename Op::V* __restrict__ val, int n_rows, Op op, RedCtx rc) {
  count_launch();
  if (op.stopped()) return;
  using A = typename Op::Acc;
  const int lane = threadIdx.x % G;
  const int wl = threadIdx.x & 31;
  const int grp = (blockIdx.x * kBlock + threadIdx.x) / G;
  const int ngrp = gridDim.x * (kBlock / G);
  double red = 0.0;
  for (int row = grp; row - wl / G < n_rows; row += ngrp) {
    A acc = A(0);
    const bool valid = row < n_rows;
    if (valid) {
      const int s = __ldg(rowptr + row), e = __ldg(rowptr + row + 1);
      for (int nz = s + lane; nz < e; nz += G) acc = rfma(static_cast<A>(__ldg(val + nz)), op.x1(__ldg(col + nz)), acc);
    }
    if constexpr (G > 1) {
#pragma unroll
      for (int off = G >> 1; off > 0; off >>= 1) acc = radd(acc, __shfl_xor_sync(0xffffffffu, acc, off, G));
    }
    if (valid && lane == 0) red += op.epi1(row, acc);
  }
  if (op.reduces()) block_reduce_1(op, rc, red);
}

// k > 1: G lanes per row split the columns in KV-wide vectors (NCH chunks per lane).
// Latency hiding, per row: the G lanes load up to G of the row's (col, val) pairs in one
// coalesced access and broadcast them with shuffles; the gathered x rows are issued up
// to 8 at a time as independent loads, together with the row's epilogue operands and the
// next row's row pointers; the next row's (col, val) are fetched before this row's
// arithmetic, so one memory round trip per row remains exposed instead of five.
template <class Op, int G, int KV, int NCH>
__global__ void __launch_bounds__(kBlock, 4)
csr_kb(const int* __restrict__ rowptr, const int* __restrict__ col,
       const typename Op::V* __restrict__ val, int n_rows, Op op, RedCtx rc) {
  count_launch();
  if (op.stopped()) return;
  using A = typename Op::Acc;
  // gathered x rows in flight per batch: 16-byte vectors 4 at a time, narrower ones 8
  constexpr int kB = (sizeof(A) * KV >= 16) ? 4 : 8;
  const int k = rc.k;
  const int lane = threadIdx.x % G;
  const int grp = (blockIdx.x * kBlock + threadIdx.x) / G;
  const int ngrp = gridDim.x * (kBlock / G);
  const int nchunks = k / KV;
  const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1)));
  double red[NCH][KV];
#pragma unroll
  for (int j = 0; j < NCH; ++j)
#pragma unroll
    for (int v = 0; v < KV; ++v) red[j][v] = 0.0;
  int row = grp;
  int s = 0, e = 0, c_l = 0;
  A v_l = A(0);
  if (row < n_rows) {
    s = __ldg(rowptr + row);
    e = __ldg(rowptr + row + 1);
    if (s + lane < e) {
      c_l = __ldg(col + s + lane);
      v_l = static_cast<A>(__ldg(val + s + lane));
    }
  }
  for (; row < n_rows; row += ngrp) {
    const int nrow = row + ngrp;
    int ns = 0, ne = 0;
    if (nrow < n_rows) {
      ns = __ldg(rowptr + nrow);
      ne = __ldg(rowptr + nrow + 1);
    }
    PreT<A, KV> pre[NCH];
#pragma unroll
    for (int j = 0; j < NCH; ++j)
      if (lane + j * G < nchunks) op.template prek<KV>(row, (lane + j * G) * KV, pre[j]);
    A acc[NCH][KV];
#pragma unroll
    for (int j = 0; j < NCH; ++j)
#pragma unroll
      for (int v = 0; v < KV; ++v) acc[j][v] = A(0);
    for (int base = s; base < e; base += G) {
      if (base != s) {  // rows longer than G: next chunk of (col, val)
        c_l = 0;
        v_l = A(0);
        if (base + lane < e) {
          c_l = __ldg(col + base + lane);
          v_l = static_cast<A>(__ldg(val + base + lane));
        }
      }
      const int cnt = min(G, e - base);
      // One batch of NB gathers: NB independent loads in flight, then their FMAs.  Slots
      // past the row's end gather the batch's first column again (a valid, cached row)
      // with a zero coefficient, so a batch has no per-slot branches; the padded products
      // add exactly zero for finite x.
      auto batch = [&](auto nb, int t) {
        constexpr int NB = decltype(nb)::value;
        int cc[NB];
        A vv[NB];
#pragma unroll
        for (int u = 0; u < NB; ++u) {
          cc[u] = __shfl_sync(gmask, c_l, (t + u) & (G - 1), G);
          vv[u] = __shfl_sync(gmask, v_l, (t + u) & (G - 1), G);
          const bool ok = t + u < cnt;
          vv[u] = ok ? vv[u] : A(0);
          if (u > 0) cc[u] = ok ? cc[u] : cc[0];
        }
#pragma unroll
        for (int j = 0; j < NCH; ++j) {
          const int ch = lane + j * G;
          if (ch < nchunks) {
            A xv[NB][KV];
#pragma unroll
            for (int u = 0; u < NB; ++u) op.template xk<KV>(cc[u], ch * KV, xv[u]);
#pragma unroll
            for (int u = 0; u < NB; ++u)
#pragma unroll
              for (int v = 0; v < KV; ++v) acc[j][v] = fma(vv[u], xv[u][v], acc[j][v]);
          }
        }
      };
      // full batches, then the remainder in the smallest batch that holds it
      int t = 0;
      for (; t + kB <= cnt; t += kB) batch(std::integral_constant<int, kB>{}, t);
      const int rem = cnt - t;
      if (rem > 4) batch(std::integral_constant<int, kB>{}, t);
      else if (rem > 2) batch(std::integral_constant<int, 4>{}, t);
      else if (rem == 2) batch(std::integral_constant<int, 2>{}, t);
      else if (rem == 1) batch(std::integral_constant<int, 1>{}, t);
    }
    // next row's first (col, val) chunk, issued before this row's epilogue
    s = ns;
    e = ne;
    c_l = 0;
    v_l = A(0);
    if (s + lane < e) {
      c_l = __ldg(col + s + lane);
      v_l = static_cast<A>(__ldg(val + s + lane));
    }
#pragma unroll
    for (int j = 0; j < NCH; ++j) {
      const int ch = lane + j * G;
      if (ch < nchunks) op.template epik<KV>(row, ch * KV, acc[j], pre[j], red[j]);
    }
  }
  if (op.reduces()) block_reduce_k<Op, G, KV, NCH>(op, rc, red);
}

// k > 1, lean variant with R independent rows in flight per lane group (rows row0,
// row0 + ngrp, ...; one column chunk per lane, G * KV >= k).  Lanes never exchange data:
// every lane reads the rows' (col, val) itself (same address across the group, one
// broadcast access), the first nonzero of every row is gathered together, and the rest of
// each row runs as a plain loop the compiler unrolls, so its gathers overlap.  No
// shuffles, no padded slots, and lanes without a column chunk skip the row loop at once:
// fewer instructions per nonzero than csr_kb.  Products are accumulated in the row's
// nonzero order with fused multiply-adds, as in csr_kb.
// Ops whose launches always / never reduce columns (a compile-time kReduce); ops without
// one decide per launch (the Jacobi sweep's norm and dot are run-time flags).
template <class Op, class = void>
struct always_reduces : std::false_type {};
template <class Op>
struct always_reduces<Op, std::void_t<decltype(Op::kReduce)>> : std::bool_constant<Op::kReduce> {};
template <class Op, class = void>
struct never_reduces : std::false_type {};
template <class Op>
struct never_reduces<Op, std::void_t<decltype(Op::kReduce)>> : std::bool_constant<!Op::kReduce> {};

// CTAs per SM the registers are sized for: 4 (64 registers), except launches that reduce
// columns with 32-byte vectors: 3 (85 registers), since their row operands and FP64
// column sums spill at 64 (measured at N = 250,000, k = 64: FP64 CG update 139 -> 132 us,
// <p, A p> 110 -> 98 us; the plain sweeps are faster at 4).
template <class Op, int KV, bool RED>
constexpr int kr_min_blocks() {
  return (RED && KV * sizeof(typename Op::Acc) >= 32) ? 3 : 4;
}

// RED: this launch reduces columns (op.reduces(), chosen by the launcher).  The reducing
// row loop carries the FP64 column sums; the plain one sends the epilogue's sums to a dead
// local, so a plain sweep keeps no FP64 accumulators in registers across rows.
template <class Op, int G, int KV, int R, bool RED>
__global__ void __launch_bounds__(kBlock, kr_min_blocks<Op, KV, RED>())
csr_kr(const int* __restrict__ rowptr, const int* __restrict__ col,
       const typename Op::V* __restrict__ val, int n_rows, Op op, RedCtx rc) {
  count_launch();
  if (op.stopped()) return;
  using A = typename Op::Acc;
  const int lane = threadIdx.x % G;
  const int grp = (blockIdx.x * kBlock + threadIdx.x) / G;
  const int ngrp = gridDim.x * (kBlock / G);
  const int c0 = lane * KV;
  double red[1][KV];
#pragma unroll
  for (int v = 0; v < KV; ++v) red[0][v] = 0.0;
  if (c0 < rc.k) {
    // gathers: through the op's per-lane prepared form when it has one (kPrepared)
    Op lop = op;
    if constexpr (Op::kPrepared) lop.template prepare<KV>(c0);
    auto gather = [&](int j, A (&v)[KV]) {
      if constexpr (Op::kPrepared) lop.template xkp<KV>(j, c0, v);
      else op.template xk<KV>(j, c0, v);
    };
    auto rows = [&](auto reducing) {
    for (int row0 = grp; row0 < n_rows; row0 += R * ngrp) {
      int s[R], e[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int row = row0 + r * ngrp;
        s[r] = 0;
        e[r] = 0;
        if (row < n_rows) {
          s[r] = __ldg(rowptr + row);
          e[r] = __ldg(rowptr + row + 1);
        }
      }
      PreT<A, KV> pre[R];
#pragma unroll
      for (int r = 0; r < R; ++r)
        if (row0 + r * ngrp < n_rows) op.template prek<KV>(row0 + r * ngrp, c0, pre[r]);
      // first nonzero of every row, gathered together
      int c1[R];
      A a1[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        c1[r] = 0;
        a1[r] = A(0);
        if (s[r] < e[r]) {
          c1[r] = __ldg(col + s[r]);
          a1[r] = static_cast<A>(__ldg(val + s[r]));
        }
      }
      A acc[R][KV];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        A xv[KV];
        gather(c1[r], xv);
#pragma unroll
        for (int v = 0; v < KV; ++v) acc[r][v] = (s[r] < e[r]) ? fma(a1[r], xv[v], A(0)) : A(0);
      }
      // the rest of every row, then its epilogue
#pragma unroll
      for (int r = 0; r < R; ++r) {
#pragma unroll 4
        for (int nz = s[r] + 1; nz < e[r]; ++nz) {
          const int cj = __ldg(col + nz);
          const A a = static_cast<A>(__ldg(val + nz));
          A xv[KV];
          gather(cj, xv);
#pragma unroll
          for (int v = 0; v < KV; ++v) acc[r][v] = fma(a, xv[v], acc[r][v]);
        }
        if (row0 + r * ngrp < n_rows) {
          if constexpr (decltype(reducing)::value) {
            op.template epik<KV>(row0 + r * ngrp, c0, acc[r], pre[r], red[0]);
          } else {
            double unused[KV];
#pragma unroll
            for (int v = 0; v < KV; ++v) unused[v] = 0.0;
            op.template epik<KV>(row0 + r * ngrp, c0, acc[r], pre[r], unused);
          }
        }
      }
    }
    };
    // RED launches run the reducing loop alone; the others keep both loops behind the
    // run-time test (measured: the plain wide sweep is faster compiled this way, 41.6 vs
    // 44.9 us, with the same 64-register budget).
    if constexpr (RED) {
      rows(std::true_type{});
    } else {
      if (op.reduces()) rows(std::true_type{});
      else rows(std::false_type{});
    }
  }
  if (RED || op.reduces()) block_reduce_k<Op, G, KV, 1>(op, rc, red);
}

// csr_kp: the lean kernel with one row per lane group (the wide 32-byte layout), its row
// metadata software-pipelined.  Per row, csr_kr waits on a chain of loads: row pointers,
// then the first (col, val), then its gather, then the rest of the row's (col, val), then
// their gathers -- ncu on the FP32 CG kernels at N = 250,000, k = 64 showed ~20 stall
// cycles per issued instruction on long scoreboards with 37 % of warp slots active.  Here
// the next row's bounds load at the top of the row and its first (col, val) once those
// bounds are in (mid-row), and the row's remaining (col, val) for up to kPipeB nonzeros
// issue before any gather, so a row mostly waits on its own gathers.  Same multiply-add
// order as csr_kr (fma(a1, x1, 0), then the row's nonzeros in order): bit-identical.
constexpr int kPipeB = 4;

template <class Op, int G, int KV, bool RED, int PB = kPipeB, int MINB = kr_min_blocks<Op, KV, RED>()>
__global__ void __launch_bounds__(kBlock, MINB)
csr_kp(const int* __restrict__ rowptr, const int* __restrict__ col,
       const typename Op::V* __restrict__ val, int n_rows, Op op, RedCtx rc) {
  count_launch();
  if (op.stopped()) return;
  using A = typename Op::Acc;
  const int lane = threadIdx.x % G;
  const int grp = (blockIdx.x * kBlock + threadIdx.x) / G;
  const int ngrp = gridDim.x * (kBlock / G);
  const int c0 = lane * KV;
  double red[1][KV];
#pragma unroll
  for (int v = 0; v < KV; ++v) red[0][v] = 0.0;
  if (c0 < rc.k) {
    Op lop = op;
    if constexpr (Op::kPrepared) lop.template prepare<KV>(c0);
    auto gather = [&](int j, A (&v)[KV]) {
      if constexpr (Op::kPrepared) lop.template xkp<KV>(j, c0, v);
      else op.template xk<KV>(j, c0, v);
    };
    auto rows = [&](auto reducing) {
      int row = grp;
      int s_n = 0, e_n = 0, c_n = 0;
      A a_n = A(0);
      if (row < n_rows) {
        s_n = __ldg(rowptr + row);
        e_n = __ldg(rowptr + row + 1);
        if (s_n < e_n) {
          c_n = __ldg(col + s_n);
          a_n = static_cast<A>(__ldg(val + s_n));
        }
      }
      for (; row < n_rows; row += ngrp) {
        const int s = s_n, e = e_n, c1 = c_n;
        const A a1 = a_n;
        const int nxt = row + ngrp;
        int s2 = 0, e2 = 0;
        if (nxt < n_rows) {
          s2 = __ldg(rowptr + nxt);
          e2 = __ldg(rowptr + nxt + 1);
        }
        PreT<A, KV> pre;
        op.template prek<KV>(row, c0, pre);
        int cr[PB > 0 ? PB : 1];
        A ar[PB > 0 ? PB : 1];
#pragma unroll
        for (int j = 0; j < PB; ++j) {
          cr[j] = c1;
          ar[j] = A(0);
          if (s + 1 + j < e) {
            cr[j] = __ldg(col + s + 1 + j);
            ar[j] = static_cast<A>(__ldg(val + s + 1 + j));
          }
        }
        A acc[KV];
        {
          A xv[KV];
          gather(c1, xv);
#pragma unroll
          for (int v = 0; v < KV; ++v) acc[v] = (s < e) ? fma(a1, xv[v], A(0)) : A(0);
        }
        // the next row's first (col, val): its bounds have arrived by now
        c_n = 0;
        a_n = A(0);
        if (s2 < e2) {
          c_n = __ldg(col + s2);
          a_n = static_cast<A>(__ldg(val + s2));
        }
#pragma unroll
        for (int j = 0; j < PB; ++j) {
          if (s + 1 + j < e) {
            A xv[KV];
            gather(cr[j], xv);
#pragma unroll
            for (int v = 0; v < KV; ++v) acc[v] = fma(ar[j], xv[v], acc[v]);
          }
        }
        for (int nz = s + 1 + PB; nz < e; ++nz) {
          const int cj = __ldg(col + nz);
          const A a = static_cast<A>(__ldg(val + nz));
          A xv[KV];
          gather(cj, xv);
#pragma unroll
          for (int v = 0; v < KV; ++v) acc[v] = fma(a, xv[v], acc[v]);
        }
        if constexpr (decltype(reducing)::value) {
          op.template epik<KV>(row, c0, acc, pre, red[0]);
        } else {
          double unused[KV];
#pragma unroll
          for (int v = 0; v < KV; ++v) unused[v] = 0.0;
          op.template epik<KV>(row, c0, acc, pre, unused);
        }
        s_n = s2;
        e_n = e2;
      }
    };
    if constexpr (RED) {
      rows(std::true_type{});
    } else {
      if (op.reduces()) rows(std::true_type{});
      else rows(std::false_type{});
    }
  }
  if (RED || op.reduces()) block_reduce_k<Op, G, KV, 1>(op, rc, red);
}

// Elementwise over [n_rows, k] with the same (group, lane, KV, NCH) mapping.
template <class Op, int G, int KV, int NCH>
__global__ void __launch_bounds__(kBlock, 4)
elem_kb(int n_rows, Op op, RedCtx rc) {
  count_launch();
  if (op.stopped()) return;
  const int k = rc.k;
  const int lane = threadIdx.x % G;
  const int grp = (blockIdx.x * kBlock + threadIdx.x) / G;
  const int ngrp = gridDim.x * (kBlock / G);
  const int nchunks = k / KV;
  double red[NCH][KV];
#pragma unroll
  for (int j = 0; j < NCH; ++j)
#pragma unroll
    for (int v = 0; v < KV; ++v) red[j][v] = 0.0;
  for (int row = grp; row < n_rows; row += ngrp) {
#pragma unroll
    for (int j = 0; j < NCH; ++j) {
      const int ch = lane + j * G;
      if (ch < nchunks) op.template elem<KV>(row, ch * KV, red[j]);
    }
  }
  if (op.reduces()) {
    if (k == 1) {
      block_reduce_1(op, rc, red[0][0]);
    } else {
      block_reduce_k<Op, G, KV, NCH>(op, rc, red);
    }
  }
}

// ------------------------------------------------------------------ loop control
// Per-column state of a solve loop, in device memory (arrays of length k).
struct LoopCtl {
  double* nr;             // standalone: last ||b - A x||; pcg: last <r, r>
  const double* thresh;   // standalone: tol * ||b|| (0 -> 1 guard); pcg: max(tol^2 <b,b>, atol^2)
  int* active;            // column still iterating
  int* iters;             // cycles / CG steps applied to the column
  int* stop;              // 1 once no column is active (later kernels of the body return)
  int maxiter;

  // Standalone rule (amjax/multilevel.py:414-422): keep cycling while
  // it < maxiter and ||r|| >= tol * ||b||; a column, once stopped, stays stopped.
  __device__ __forceinline__ int standalone_col(int c, double sumsq) const {
    const double n = sqrt(sumsq);
    nr[c] = n;
    const int a = active[c] && iters[c] < maxiter && n >= thresh[c];
    active[c] = a;
    if (a) iters[c] += 1;
    return a;
  }
  // CG rule (jax.scipy.sparse.linalg.cg): continue while <r,r> > atol2 and k < maxiter.
  __device__ __forceinline__ int cg_col(int c, double rr) const {
    nr[c] = rr;
    int a = active[c];
    if (a) {
      iters[c] += 1;
      a = (rr > thresh[c]) && (iters[c] < maxiter);
    }
    active[c] = a;
    return a;
  }
  // No column left: later kernels of this loop trip return at once, and the trip's
  // closing guard kernel ends the loop.
  __device__ __forceinline__ void set_any(int any) const {
    if (!any) *stop = 1;
  }

  // ---- CG with reliable updates (FP32 CG vectors; the FP64 solution and the FP64 true
  // residual are brought up to date on demand).  State besides the above:
  double* rmax = nullptr;  // per column: the largest <r, r> since the last true residual
  int* ru = nullptr;       // ru[0]: a true residual is due; ru[1]: some FP32 increment is unfolded
  double delta2 = 0.0;     // a true residual is due once <r, r> < delta2 * rmax

  // After the FP32 update of an active column: the column always stays active here (only
  // the FP64 true residual may retire it); a true residual is requested when the
  // recursive residual has dropped by delta (the FP32 recurrence has drifted for a while),
  // when it says the column has converged (confirmed in FP64 before stopping), at maxiter,
  // or when it is not a number.
  __device__ __forceinline__ int cg_col_ru(int c, double rr) const {
    nr[c] = rr;
    if (!active[c]) return 0;
    iters[c] += 1;
    ru[1] = 1;
    if (rr <= thresh[c] || iters[c] >= maxiter || rr < delta2 * rmax[c] || !(rr == rr)) ru[0] = 1;
    return 1;
  }
  // After the FP64 true residual: the CG rule on the true <r, r> for the columns still
  // active (frozen columns keep their last values).
  __device__ __forceinline__ int true_col(int c, double rr) const {
    if (!active[c]) return 0;
    nr[c] = rr;
    rmax[c] = rr;
    const int a = (rr > thresh[c]) && (iters[c] < maxiter);
    active[c] = a;
    return a;
  }
  __device__ __forceinline__ void true_all(int any) const {
    ru[0] = 0;
    ru[1] = 0;
    set_any(any);
  }

  // ---- standalone solve with reliable updates (FP32 residual and increment; the rule of
  // amjax/multilevel.py:414-422 decided on the FP64 norm).  thresh = tol * ||b||, nr the
  // last norm; rmax keeps <r, r> (squared) for the delta test.
  __device__ __forceinline__ int sa_col_ru(int c, double rr) const {
    if (!active[c]) return 0;
    iters[c] += 1;
    const double n = sqrt(rr);
    nr[c] = n;
    ru[1] = 1;
    if (n < thresh[c] || iters[c] >= maxiter || rr < delta2 * rmax[c] || !(rr == rr)) ru[0] = 1;
    return 1;
  }
  __device__ __forceinline__ int true_col_sa(int c, double rr) const {
    if (!active[c]) return 0;
    const double n = sqrt(rr);
    nr[c] = n;
    rmax[c] = rr;
    const int a = (n >= thresh[c]) && (iters[c] < maxiter);
    active[c] = a;
    return a;
  }
};

// ------------------------------------------------------------------ x sources
enum XSrc { XS_PLAIN = 0, XS_JAC0 = 1, XS_ZERO = 2, XS_RESJ0 = 3, XS_PROJ0 = 4 };

// x_j as the SpMV sees it: the stored x, or one damped-Jacobi sweep from zero computed
// on the fly, x_j = omega * (dinv_j * b_j) (relaxation.py:94-96 with x = 0: the SpMV of
// the zero vector is exactly zero, so this is bit-identical to running the sweep).
// Two-hop sources, used with one right-hand side (where a cycle is latency-bound and
// recomputing a neighbour's value costs less than a launch), evaluated per gathered row
// from an inner CSR matrix M (mrp / mci / mv):
//   XS_RESJ0: x_j = b_j - sum_m M_jm x1_m, x1 = omega D^-1 b: the residual of the
//             one-sweep-from-zero iterate (M = A): restriction R r without storing r;
//   XS_PROJ0: x_j = x1_j + sum_J M_jJ xc_J (M = P): the prolonged and corrected iterate,
//             so the post-smoothing sweep needs no stored x1 + P xc.
template <class T, int XS>
struct XSource {
  const T* x;
  const T* b;
  const T* dinv;
  T omega;
  int ld;
  const int* mrp = nullptr;
  const int* mci = nullptr;
  const T* mv = nullptr;
  const T* xc = nullptr;
  __device__ __forceinline__ T jac0(int j) const { return rmul(omega, rmul(__ldg(dinv + j), __ldg(b + j))); }
  __device__ __forceinline__ T get1(int j) const {
    if constexpr (XS == XS_PLAIN) return __ldg(x + j);
    else if constexpr (XS == XS_JAC0) return jac0(j);
    else if constexpr (XS == XS_RESJ0) {
      T acc = T(0);
      const int e = __ldg(mrp + j + 1);
      for (int nz = __ldg(mrp + j); nz < e; ++nz) acc = rfma(__ldg(mv + nz), jac0(__ldg(mci + nz)), acc);
      return rsub(__ldg(b + j), acc);
    } else if constexpr (XS == XS_PROJ0) {
      T acc = jac0(j);
      const int e = __ldg(mrp + j + 1);
      for (int nz = __ldg(mrp + j); nz < e; ++nz) acc = rfma(__ldg(mv + nz), __ldg(xc + __ldg(mci + nz)), acc);
      return acc;
    } else {
      return T(0);
    }
  }
  template <int KV>
  __device__ __forceinline__ void getk(int j, int c0, T (&v)[KV]) const {
    static_assert(XS != XS_RESJ0 && XS != XS_PROJ0, "two-hop sources serve one right-hand side");
    if constexpr (XS == XS_PLAIN) {
      ld_vec<T, KV>(x + voff(j, ld, c0), v);
    } else if constexpr (XS == XS_JAC0) {
      T bv[KV];
      ld_vec<T, KV>(b + voff(j, ld, c0), bv);
      const T d = __ldg(dinv + j);
#pragma unroll
      for (int i = 0; i < KV; ++i) v[i] = rmul(omega, rmul(d, bv[i]));
    } else {
#pragma unroll
      for (int i = 0; i < KV; ++i) v[i] = T(0);
    }
  }
};

// ------------------------------------------------------------------ ops
// Damped Jacobi sweep, relaxation.py:94-96:
//   temp = Dinv * (b - A x) + x ;  out = (1 - omega) * x + omega * temp
// Runtime flags (uniform across the grid) select fused extras:
//   norm: also reduce ||b - A x||^2 per column and apply the standalone loop rule;
//   mask: write only columns still active (frozen columns keep their value);
//   rdot64 / rdot32: also reduce <r, out> per column (the CG's gamma = <r, z>).
template <class T, int XS>
struct OpJacobi {
  static constexpr bool kPrepared = false;
  static constexpr bool kOnlyK1 = XS == XS_RESJ0 || XS == XS_PROJ0;
  using V = T;
  using Acc = T;
  XSource<T, XS> xs;
  const T* b;
  const T* dinv;
  T omega;
  T* out;
  int ld;
  int norm;
  const int* active;     // non-null: mask by active columns
  const int* stop;
  const double* rdot64;  // CG dot, FP64 residual
  const float* rdot32;   // CG dot, FP32 residual
  LoopCtl ctl;           // norm
  double* gamma;         // dot: gamma (new) ; beta = gamma_new / gamma_old
  double* beta;

  __host__ __device__ __forceinline__ bool reduces() const { return norm || rdot64 || rdot32; }
  __device__ __forceinline__ bool stopped() const { return stop && *stop; }
  __device__ __forceinline__ T x1(int j) const { return xs.get1(j); }
  template <int KV>
  __device__ __forceinline__ void xk(int j, int c0, T (&v)[KV]) const { xs.template getk<KV>(j, c0, v); }

  __device__ __forceinline__ double epi1(int i, T s) const {
    const T xv = xs.get1(i);
    const T r = rsub(__ldg(b + i), s);
    const T temp = rfma(__ldg(dinv + i), r, xv);
    const T y = rfma(omega, temp, rmul(rsub(T(1), omega), xv));
    if (!active || active[0]) out[i] = y;
    if (norm) return rmul((double)r, (double)r);
    if (rdot64) return rmul(__ldg(rdot64 + i), (double)y);
    if (rdot32) return rmul((double)__ldg(rdot32 + i), (double)y);
    return 0.0;
  }
  template <int KV>
  __device__ __forceinline__ void prek(int i, int c0, PreT<T, KV>& p) const {
    const size_t o = voff(i, ld, c0);
    xs.template getk<KV>(i, c0, p.x);
    ld_vec<T, KV>(b + o, p.b);
    p.d = __ldg(dinv + i);
  }
  template <int KV>
  __device__ __forceinline__ void epik(int i, int c0, const T (&s)[KV], const PreT<T, KV>& p,
                                       double (&red)[KV]) const {
    T y[KV], r[KV];
    const T om1 = rsub(T(1), omega);
#pragma unroll
    for (int v = 0; v < KV; ++v) {
      r[v] = rsub(p.b[v], s[v]);
      const T temp = rfma(p.d, r[v], p.x[v]);
      y[v] = rfma(omega, temp, rmul(om1, p.x[v]));
    }
    const size_t o = voff(i, ld, c0);
    if (!(norm | (rdot64 != nullptr) | (rdot32 != nullptr) | (active != nullptr))) {
      st_vec<T, KV>(out + o, y);  // the plain sweep: one uniform test per row
      return;
    }
    if (norm) {
#pragma unroll
      for (int v = 0; v < KV; ++v) red[v] = rfma((double)r[v], (double)r[v], red[v]);
    } else if (rdot64) {
      double rv[KV];
      ld_vec<double, KV>(rdot64 + o, rv);
#pragma unroll
      for (int v = 0; v < KV; ++v) red[v] = rfma(rv[v], (double)y[v], red[v]);
    } else if (rdot32) {
      float rv[KV];
      bool loaded = false;  // the CG's <r, z> with r the sweep's right-hand side: already in p.b
      if constexpr (std::is_same<T, float>::value) {
        if (rdot32 == b) {
#pragma unroll
          for (int v = 0; v < KV; ++v) rv[v] = p.b[v];
          loaded = true;
        }
      }
      if (!loaded) ld_vec<float, KV>(rdot32 + o, rv);
#pragma unroll
      for (int v = 0; v < KV; ++v) red[v] = rfma((double)rv[v], (double)y[v], red[v]);
    }
    if (active) {
#pragma unroll
      for (int v = 0; v < KV; ++v)
        if (active[c0 + v]) out[o + v] = y[v];
    } else {
      st_vec<T, KV>(out + o, y);
    }
  }
  __device__ __forceinline__ int finalize_col(int c, double s) const {
    if (norm) return ctl.standalone_col(c, s);
    beta[c] = s / gamma[c];
    gamma[c] = s;
    return 1;
  }
  __device__ __forceinline__ void finalize_all(int any) const {
    if (norm) ctl.set_any(any);
  }
};

// r = b - A x (x from an XSource).  RLO: also/instead store a copy in another type.
// NORM: reduce ||r||^2 per column and apply the standalone loop rule (outer loop of the
// mixed-precision refinement), or with `true_rule` the rule of a reliable-update loop on the
// FP64 true residual (1: CG, 2: standalone).  STORE: write r in T.  `gate` (nullable): the
// launch returns at once unless *gate is set (the true residual runs only when one is due).
template <class T, class VT, int XS, bool STORE, class TLO, bool NORM>
struct OpResid {
  static constexpr bool kPrepared = false;
  using V = VT;
  using Acc = T;
  static constexpr bool kReduce = NORM;
  __host__ __device__ __forceinline__ bool reduces() const { return kReduce; }
  XSource<T, XS> xs;
  const T* b;
  T* out;      // STORE
  TLO* out_lo; // nullable: copy of r in the cycle's type
  int ld;
  const int* stop;
  LoopCtl ctl;
  const int* gate = nullptr;
  int true_rule = 0;

  __device__ __forceinline__ bool stopped() const { return (stop && *stop) || (gate && !*gate); }
  __device__ __forceinline__ T x1(int j) const { return xs.get1(j); }
  template <int KV>
  __device__ __forceinline__ void xk(int j, int c0, T (&v)[KV]) const { xs.template getk<KV>(j, c0, v); }
  __device__ __forceinline__ double epi1(int i, T s) const {
    const T r = rsub(__ldg(b + i), s);
    if constexpr (STORE) out[i] = r;
    if (out_lo) out_lo[i] = static_cast<TLO>(r);
    return NORM ? rmul((double)r, (double)r) : 0.0;
  }
  template <int KV>
  __device__ __forceinline__ void prek(int i, int c0, PreT<T, KV>& p) const {
    ld_vec<T, KV>(b + voff(i, ld, c0), p.b);
  }
  template <int KV>
  __device__ __forceinline__ void epik(int i, int c0, const T (&s)[KV], const PreT<T, KV>& p,
                                       double (&red)[KV]) const {
    T r[KV];
#pragma unroll
    for (int v = 0; v < KV; ++v) {
      r[v] = rsub(p.b[v], s[v]);
      if constexpr (NORM) red[v] = rfma((double)r[v], (double)r[v], red[v]);
    }
    if constexpr (STORE) st_vec<T, KV>(out + voff(i, ld, c0), r);
    if (out_lo) {
      TLO rl[KV];
#pragma unroll
      for (int v = 0; v < KV; ++v) rl[v] = static_cast<TLO>(r[v]);
      st_vec<TLO, KV>(out_lo + voff(i, ld, c0), rl);
    }
  }
  __device__ __forceinline__ int finalize_col(int c, double s) const {
    if constexpr (NORM) {
      if (true_rule == 1) return ctl.true_col(c, s);
      if (true_rule == 2) return ctl.true_col_sa(c, s);
      return ctl.standalone_col(c, s);
    }
    return 1;
  }
  __device__ __forceinline__ void finalize_all(int any) const {
    if constexpr (NORM) {
      if (true_rule) ctl.true_all(any);
      else ctl.set_any(any);
    }
  }
};

// out = base + M x  (XS of base: plain (may alias out: each row reads only its own base
// entry before writing it), one Jacobi sweep from zero computed on the fly, or zero).
// With base = zero this is the plain SpMV used for restriction R r.
template <class T, int BS>
struct OpAxpy {
  static constexpr bool kPrepared = false;
  using V = T;
  using Acc = T;
  static constexpr bool kReduce = false;
  __host__ __device__ __forceinline__ bool reduces() const { return kReduce; }
  XSource<T, BS> base;
  const T* x;
  T* out;
  int ld;
  const int* stop;

  __device__ __forceinline__ bool stopped() const { return stop && *stop; }
  __device__ __forceinline__ T x1(int j) const { return __ldg(x + j); }
  template <int KV>
  __device__ __forceinline__ void xk(int j, int c0, T (&v)[KV]) const {
    ld_vec<T, KV>(x + voff(j, ld, c0), v);
  }
  __device__ __forceinline__ double epi1(int i, T s) const {
    out[i] = radd(base.get1(i), s);
    return 0.0;
  }
  template <int KV>
  __device__ __forceinline__ void prek(int i, int c0, PreT<T, KV>& p) const {
    base.template getk<KV>(i, c0, p.x);
  }
  template <int KV>
  __device__ __forceinline__ void epik(int i, int c0, const T (&s)[KV], const PreT<T, KV>& p,
                                       double (&)[KV]) const {
    T y[KV];
#pragma unroll
    for (int v = 0; v < KV; ++v) y[v] = radd(p.x[v], s[v]);
    st_vec<T, KV>(out + voff(i, ld, c0), y);
  }
  __device__ __forceinline__ int finalize_col(int, double) const { return 1; }
  __device__ __forceinline__ void finalize_all(int) const {}
};


// out = M x with x from a (two-hop) x source, one right-hand side: the restriction of the
// residual of the one-sweep-from-zero iterate in one pass (XS_RESJ0).
template <class T, int XS>
struct OpRestrictX {
  static constexpr bool kPrepared = false;
  static constexpr bool kOnlyK1 = true;
  using V = T;
  using Acc = T;
  static constexpr bool kReduce = false;
  __host__ __device__ __forceinline__ bool reduces() const { return kReduce; }
  XSource<T, XS> xs;
  T* out;
  int ld;
  const int* stop;
  __device__ __forceinline__ bool stopped() const { return stop && *stop; }
  __device__ __forceinline__ T x1(int j) const { return xs.get1(j); }
  template <int KV>
  __device__ __forceinline__ void xk(int j, int c0, T (&v)[KV]) const { xs.template getk<KV>(j, c0, v); }
  __device__ __forceinline__ double epi1(int i, T s) const {
    out[i] = s;
    return 0.0;
  }
  template <int KV>
  __device__ __forceinline__ void prek(int, int, PreT<T, KV>&) const {}
  template <int KV>
  __device__ __forceinline__ void epik(int i, int c0, const T (&s)[KV], const PreT<T, KV>&, double (&)[KV]) const {
    st_vec<T, KV>(out + voff(i, ld, c0), s);
  }
  __device__ __forceinline__ int finalize_col(int, double) const { return 1; }
  __device__ __forceinline__ void finalize_all(int) const {}
};

// Ops that serve one right-hand side only (two-hop sources) declare kOnlyK1.
template <class Op, class = void>
struct only_k1 : std::false_type {};
template <class Op>
struct only_k1<Op, std::void_t<decltype(Op::kOnlyK1)>> : std::bool_constant<Op::kOnlyK1> {};

// CG step with the direction update folded in: p_new = z + beta p_old (z in the cycle's
// type, beta per column from the last cycle) is formed on the fly for every gathered row
// and written for the row's own entries into the other direction buffer (other rows
// still gather p_old); <p_new, A p_new> is reduced per column, alpha = gamma / <p, A p>.
// The gathered and the stored p_new come from the same fused multiply-add, so they are
// identical.  This replaces the separate pass p = z + beta p before <p, A p>.
template <class T, class TZ>
struct OpCgQDir {
  static constexpr bool kPrepared = true;
  using V = T;
  using Acc = T;
  static constexpr bool kReduce = true;
  __host__ __device__ __forceinline__ bool reduces() const { return kReduce; }
  const T* p_old;
  const TZ* z;
  T* p_new;
  const double* beta;
  int ld;
  const int* stop;
  const double* gamma;
  double* alpha;
  T bl[8];  // beta of one lane's column chunk, loaded once by prepare() (csr_kr)

  __device__ __forceinline__ bool stopped() const { return stop && *stop; }
  __device__ __forceinline__ T x1(int j) const {
    return fma(static_cast<T>(__ldg(beta)), __ldg(p_old + j), static_cast<T>(__ldg(z + j)));
  }
  // Kernels whose lanes keep one column chunk (csr_kr) load the chunk's beta once per lane
  // and gather through xkp, instead of re-loading beta for every gathered row.
  template <int KV>
  __device__ __forceinline__ void prepare(int c0) {
#pragma unroll
    for (int i = 0; i < KV; ++i) bl[i] = static_cast<T>(__ldg(beta + c0 + i));
  }
  template <int KV>
  __device__ __forceinline__ void xkp(int j, int c0, T (&v)[KV]) const {
    const size_t o = voff(j, ld, c0);
    T pv[KV], zv[KV];
    ld_vec<T, KV>(p_old + o, pv);
    ld_cvt<T, TZ, KV>(z + o, zv);
#pragma unroll
    for (int i = 0; i < KV; ++i) v[i] = fma(bl[i], pv[i], zv[i]);
  }
  template <int KV>
  __device__ __forceinline__ void xk(int j, int c0, T (&v)[KV]) const {
    const size_t o = voff(j, ld, c0);
    T pv[KV], zv[KV];
    ld_vec<T, KV>(p_old + o, pv);
    ld_cvt<T, TZ, KV>(z + o, zv);
#pragma unroll
    for (int i = 0; i < KV; ++i) v[i] = fma(static_cast<T>(__ldg(beta + c0 + i)), pv[i], zv[i]);
  }
  __device__ __forceinline__ double epi1(int i, T s) const {
    const T pn = x1(i);
    p_new[i] = pn;
    return rmul((double)pn, (double)s);
  }
  template <int KV>
  __device__ __forceinline__ void prek(int i, int c0, PreT<T, KV>& pp) const {
    xk<KV>(i, c0, pp.x);
  }
  template <int KV>
  __device__ __forceinline__ void epik(int i, int c0, const T (&s)[KV], const PreT<T, KV>& pp,
                                       double (&red)[KV]) const {
#pragma unroll
    for (int v = 0; v < KV; ++v) red[v] = rfma((double)pp.x[v], (double)s[v], red[v]);
    st_vec<T, KV>(p_new + voff(i, ld, c0), pp.x);
  }
  __device__ __forceinline__ int finalize_col(int c, double s) const {
    alpha[c] = gamma[c] / s;
    return 1;
  }
  __device__ __forceinline__ void finalize_all(int) const {}
};

// CG update with the SpMV recomputed instead of stored: s = A p, then for active columns
// x += alpha p, r -= alpha s; r copied into the cycle's type (r_lo, nullable); reduce
// <r, r> and apply the CG loop rule.
template <class T, class TLO>
struct OpCgUpdA {
  static constexpr bool kPrepared = false;
  using V = T;
  using Acc = T;
  static constexpr bool kReduce = true;
  __host__ __device__ __forceinline__ bool reduces() const { return kReduce; }
  T* x;
  T* r;
  const T* p;
  TLO* r_lo;
  const double* alpha;
  const int* active;
  int ld;
  const int* stop;
  LoopCtl ctl;

  __device__ __forceinline__ bool stopped() const { return stop && *stop; }
  __device__ __forceinline__ T x1(int j) const { return __ldg(p + j); }
  template <int KV>
  __device__ __forceinline__ void xk(int j, int c0, T (&v)[KV]) const {
    ld_vec<T, KV>(p + voff(j, ld, c0), v);
  }
  __device__ __forceinline__ double epi1(int i, T s) const {
    T rv = r[i];
    if (active[0]) {
      const T a = static_cast<T>(alpha[0]);
      x[i] = rfma(a, __ldg(p + i), x[i]);
      rv = rfma(-a, s, rv);
      r[i] = rv;
    }
    if (r_lo) r_lo[i] = static_cast<TLO>(rv);
    return rmul((double)rv, (double)rv);
  }
  template <int KV>
  __device__ __forceinline__ void prek(int i, int c0, PreT<T, KV>& pp) const {
    const size_t o = voff(i, ld, c0);
    ld_vec<T, KV>(p + o, pp.x);
    ld_vec<T, KV>(x + o, pp.b);
    ld_vec<T, KV>(r + o, pp.c);
  }
  template <int KV>
  __device__ __forceinline__ void epik(int i, int c0, const T (&s)[KV], const PreT<T, KV>& pp,
                                       double (&red)[KV]) const {
    const size_t o = voff(i, ld, c0);
    T xv[KV], rv[KV];
    bool any = false;
#pragma unroll
    for (int v = 0; v < KV; ++v) {
      xv[v] = pp.b[v];
      rv[v] = pp.c[v];
      if (active[c0 + v]) {
        const T a = static_cast<T>(alpha[c0 + v]);
        xv[v] = rfma(a, pp.x[v], xv[v]);
        rv[v] = rfma(-a, s[v], rv[v]);
        any = true;
      }
      red[v] = rfma((double)rv[v], (double)rv[v], red[v]);
    }
    if (any) {
      st_vec<T, KV>(x + o, xv);
      st_vec<T, KV>(r + o, rv);
    }
    if (r_lo) {
      TLO rl[KV];
#pragma unroll
      for (int v = 0; v < KV; ++v) rl[v] = static_cast<TLO>(rv[v]);
      st_vec<TLO, KV>(r_lo + o, rl);
    }
  }
  // reliable: the CG of the reliable-update form (x and r are the FP32 increment and
  // residual; retiring columns is left to the FP64 true residual)
  bool reliable = false;
  __device__ __forceinline__ int finalize_col(int c, double s) const {
    return reliable ? ctl.cg_col_ru(c, s) : ctl.cg_col(c, s);
  }
  __device__ __forceinline__ void finalize_all(int any) const {
    if (!reliable) ctl.set_any(any);
  }
};

// Standalone reliable-update step after a cycle e = M r: s = A e; for active columns
// xs += e and r -= s (r stays the residual of x + xs); reduce <r, r> and apply the
// standalone reliable rule (LoopCtl::sa_col_ru).
template <class T>
struct OpResUpd {
  static constexpr bool kPrepared = false;
  using V = T;
  using Acc = T;
  static constexpr bool kReduce = true;
  __host__ __device__ __forceinline__ bool reduces() const { return kReduce; }
  const T* e;
  T* xs;
  T* r;
  const int* active;
  int ld;
  const int* stop;
  LoopCtl ctl;

  __device__ __forceinline__ bool stopped() const { return stop && *stop; }
  __device__ __forceinline__ T x1(int j) const { return __ldg(e + j); }
  template <int KV>
  __device__ __forceinline__ void xk(int j, int c0, T (&v)[KV]) const {
    ld_vec<T, KV>(e + voff(j, ld, c0), v);
  }
  __device__ __forceinline__ double epi1(int i, T s) const {
    T rv = r[i];
    if (active[0]) {
      xs[i] = radd(xs[i], __ldg(e + i));
      rv = rsub(rv, s);
      r[i] = rv;
    }
    return rmul((double)rv, (double)rv);
  }
  template <int KV>
  __device__ __forceinline__ void prek(int i, int c0, PreT<T, KV>& pp) const {
    const size_t o = voff(i, ld, c0);
    ld_vec<T, KV>(e + o, pp.x);
    ld_vec<T, KV>(xs + o, pp.b);
    ld_vec<T, KV>(r + o, pp.c);
  }
  template <int KV>
  __device__ __forceinline__ void epik(int i, int c0, const T (&s)[KV], const PreT<T, KV>& pp,
                                       double (&red)[KV]) const {
    const size_t o = voff(i, ld, c0);
    T xv[KV], rv[KV];
    bool any = false;
#pragma unroll
    for (int v = 0; v < KV; ++v) {
      xv[v] = pp.b[v];
      rv[v] = pp.c[v];
      if (active[c0 + v]) {
        xv[v] = radd(xv[v], pp.x[v]);
        rv[v] = rsub(rv[v], s[v]);
        any = true;
      }
      red[v] = rfma((double)rv[v], (double)rv[v], red[v]);
    }
    if (any) {
      st_vec<T, KV>(xs + o, xv);
      st_vec<T, KV>(r + o, rv);
    }
  }
  __device__ __forceinline__ int finalize_col(int c, double s) const { return ctl.sa_col_ru(c, s); }
  __device__ __forceinline__ void finalize_all(int) const {}
};

// ------------------------------------------------------------------ elementwise ops
// Reliable-update fold: x += xs (FP64 solution += FP32 increment), xs = 0, every column
// (retired columns hold a zero increment).  Runs only when *gate is set.
template <class T, class TS>
struct OpFold {
  static constexpr bool kReduce = false;
  __host__ __device__ __forceinline__ bool reduces() const { return kReduce; }
  T* x;
  TS* xs;
  int ld;
  const int* gate;
  __device__ __forceinline__ bool stopped() const { return !*gate; }
  template <int KV>
  __device__ __forceinline__ void elem(int i, int c0, double (&)[KV]) const {
    const size_t o = voff(i, ld, c0);
    T xv[KV];
    TS sv[KV], zero[KV];
    ld_vec<T, KV>(x + o, xv);
    ld_vec<TS, KV>(xs + o, sv);
#pragma unroll
    for (int v = 0; v < KV; ++v) {
      xv[v] = radd(xv[v], static_cast<T>(sv[v]));
      zero[v] = TS(0);
    }
    st_vec<T, KV>(x + o, xv);
    st_vec<TS, KV>(xs + o, zero);
  }
  __device__ __forceinline__ int finalize_col(int, double) const { return 1; }
  __device__ __forceinline__ void finalize_all(int) const {}
};

// CG update: for active columns x += alpha p, r -= alpha q; copy r into the cycle's
// type (r_lo, nullable); reduce <r, r> and apply the CG loop rule.
template <class T, class TLO>
struct OpCgUpdate {
  static constexpr bool kReduce = true;
  __host__ __device__ __forceinline__ bool reduces() const { return kReduce; }
  T* x;
  T* r;
  const T* p;
  const T* q;
  TLO* r_lo;
  const double* alpha;
  const int* active;
  int ld;
  const int* stop;
  LoopCtl ctl;
  __device__ __forceinline__ bool stopped() const { return stop && *stop; }
  template <int KV>
  __device__ __forceinline__ void elem(int i, int c0, double (&red)[KV]) const {
    T xv[KV], rv[KV], pv[KV], qv[KV];
    const size_t o = voff(i, ld, c0);
    ld_vec<T, KV>(r + o, rv);
    bool any = false;
#pragma unroll
    for (int v = 0; v < KV; ++v) any |= (active[c0 + v] != 0);
    if (any) {
      ld_vec<T, KV>(x + o, xv);
      ld_vec<T, KV>(p + o, pv);
      ld_vec<T, KV>(q + o, qv);
#pragma unroll
      for (int v = 0; v < KV; ++v) {
        if (active[c0 + v]) {
          const T a = static_cast<T>(alpha[c0 + v]);
          xv[v] = rfma(a, pv[v], xv[v]);
          rv[v] = rfma(-a, qv[v], rv[v]);
        }
      }
      st_vec<T, KV>(x + o, xv);
      st_vec<T, KV>(r + o, rv);
    }
#pragma unroll
    for (int v = 0; v < KV; ++v) red[v] = rfma((double)rv[v], (double)rv[v], red[v]);
    if (r_lo) {
      TLO rl[KV];
#pragma unroll
      for (int v = 0; v < KV; ++v) rl[v] = static_cast<TLO>(rv[v]);
      st_vec<TLO, KV>(r_lo + o, rl);
    }
  }
  __device__ __forceinline__ int finalize_col(int c, double s) const { return ctl.cg_col(c, s); }
  __device__ __forceinline__ void finalize_all(int any) const { ctl.set_any(any); }
};


// Mixed-precision refinement update: x += e for active columns (e in the cycle's type).
template <class T, class TE>
struct OpRefine {
  static constexpr bool kReduce = false;
  __host__ __device__ __forceinline__ bool reduces() const { return kReduce; }
  T* x;
  const TE* e;
  const int* active;
  int ld;
  const int* stop;
  __device__ __forceinline__ bool stopped() const { return stop && *stop; }
  template <int KV>
  __device__ __forceinline__ void elem(int i, int c0, double (&)[KV]) const {
    const size_t o = voff(i, ld, c0);
    T xv[KV], ev[KV];
    ld_vec<T, KV>(x + o, xv);
    ld_cvt<T, TE, KV>(e + o, ev);
#pragma unroll
    for (int v = 0; v < KV; ++v)
      if (active[c0 + v]) xv[v] = radd(xv[v], ev[v]);
    st_vec<T, KV>(x + o, xv);
  }
  __device__ __forceinline__ int finalize_col(int, double) const { return 1; }
  __device__ __forceinline__ void finalize_all(int) const {}
};

// One damped-Jacobi sweep from the zero vector, materialised: out = omega*(dinv*b).
template <class T>
struct OpJac0 {
  static constexpr bool kReduce = false;
  __host__ __device__ __forceinline__ bool reduces() const { return kReduce; }
  const T* b;
  const T* dinv;
  T omega;
  T* out;
  int ld;
  const int* stop;
  __device__ __forceinline__ bool stopped() const { return stop && *stop; }
  template <int KV>
  __device__ __forceinline__ void elem(int i, int c0, double (&)[KV]) const {
    const size_t o = voff(i, ld, c0);
    T bv[KV];
    ld_vec<T, KV>(b + o, bv);
    const T d = __ldg(dinv + i);
#pragma unroll
    for (int v = 0; v < KV; ++v) bv[v] = rmul(omega, rmul(d, bv[v]));
    st_vec<T, KV>(out + o, bv);
  }
  __device__ __forceinline__ int finalize_col(int, double) const { return 1; }
  __device__ __forceinline__ void finalize_all(int) const {}
};

// Copy/convert with an optional per-column sum of squares:
//   dst = src (T), dst_lo = src (TLO) ; sums[c] = sum src^2 ; loop set-up.
// MODE 0: store the norm  sqrt(sum) (0 -> 1 guard) * tol into thresh, reset the loop.
// MODE 1: CG set-up: thresh = max(tol^2 sum, atol^2), nr = sum, active = sum > thresh.
// MODE 2: standalone reliable-update set-up: MODE 0's threshold, and the loop's first test
//         ||b|| >= tol ||b|| (x0 = 0) applied here, with rmax = sum.
template <class T, class TLO, int MODE>
struct OpSetup {
  static constexpr bool kReduce = true;
  __host__ __device__ __forceinline__ bool reduces() const { return kReduce; }
  const T* src;
  T* dst;       // nullable
  TLO* dst_lo;  // nullable
  T* zero;      // nullable: zero-filled alongside
  int ld;
  double* thresh;
  double* nr;
  double* normb;
  int* active;
  int* iters;
  int* stop;
  int* gcount;
  double tol, atol;
  int maxiter;
  double* rmax = nullptr;  // reliable-update CG: rmax = <b, b>, no true residual due
  int* ru = nullptr;
  __device__ __forceinline__ bool stopped() const { return false; }
  template <int KV>
  __device__ __forceinline__ void elem(int i, int c0, double (&red)[KV]) const {
    const size_t o = voff(i, ld, c0);
    T v[KV];
    ld_vec<T, KV>(src + o, v);
#pragma unroll
    for (int j = 0; j < KV; ++j) red[j] = rfma((double)v[j], (double)v[j], red[j]);
    if (dst) st_vec<T, KV>(dst + o, v);
    if (dst_lo) {
      TLO l[KV];
#pragma unroll
      for (int j = 0; j < KV; ++j) l[j] = static_cast<TLO>(v[j]);
      st_vec<TLO, KV>(dst_lo + o, l);
    }
    if (zero) {
      T z[KV];
#pragma unroll
      for (int j = 0; j < KV; ++j) z[j] = T(0);
      st_vec<T, KV>(zero + o, z);
    }
  }
  __device__ __forceinline__ int finalize_col(int c, double s) const {
    iters[c] = 0;
    double nb = sqrt(s);
    if (nb == 0.0) nb = 1.0;
    normb[c] = nb;
    if constexpr (MODE == 0) {
      thresh[c] = tol * nb;
      nr[c] = sqrt(s);
      active[c] = 1;
      return 1;
    } else if constexpr (MODE == 2) {
      const double t = tol * nb;
      thresh[c] = t;
      nr[c] = sqrt(s);
      if (rmax) rmax[c] = s;
      const int a = (sqrt(s) >= t) && (maxiter > 0);
      active[c] = a;
      return a;
    } else {
      const double t = fmax(tol * tol * s, atol * atol);
      thresh[c] = t;
      nr[c] = s;
      if (rmax) rmax[c] = s;
      const int a = (s > t) && (maxiter > 0);
      active[c] = a;
      return a;
    }
  }
  __device__ __forceinline__ void finalize_all(int any) const {
    if (gcount) *gcount = 0;
    if (ru) ru[0] = ru[1] = 0;
    *stop = (MODE == 0) ? 0 : (any ? 0 : 1);
  }
};

// dst = src for active columns (all columns when active is null); DOT: also reduce
// <rdot, src> per column and update the CG's gamma / beta.
template <class T, class TR, bool DOT>
struct OpMaskCopy {
  static constexpr bool kReduce = DOT;
  __host__ __device__ __forceinline__ bool reduces() const { return kReduce; }
  const T* src;
  T* dst;
  const int* active;
  int ld;
  const int* stop;
  const TR* rdot;
  double* gamma;
  double* beta;
  __device__ __forceinline__ bool stopped() const { return stop && *stop; }
  template <int KV>
  __device__ __forceinline__ void elem(int i, int c0, double (&red)[KV]) const {
    const size_t o = voff(i, ld, c0);
    T v[KV];
    ld_vec<T, KV>(src + o, v);
    if constexpr (DOT) {
      TR rv[KV];
      ld_vec<TR, KV>(rdot + o, rv);
#pragma unroll
      for (int j = 0; j < KV; ++j) red[j] = rfma((double)rv[j], (double)v[j], red[j]);
    }
    if (active) {
#pragma unroll
      for (int j = 0; j < KV; ++j)
        if (active[c0 + j]) dst[o + j] = v[j];
    } else {
      st_vec<T, KV>(dst + o, v);
    }
  }
  __device__ __forceinline__ int finalize_col(int c, double s) const {
    if constexpr (DOT) {
      beta[c] = s / gamma[c];
      gamma[c] = s;
    }
    return 1;
  }
  __device__ __forceinline__ void finalize_all(int) const {}
};

// ------------------------------------------------------------------ coarse solvers
// Coarse solve of a small dense system for k columns; one thread per (row, column) for
// the products, one thread per column for the triangular solves.  n is small (the
// coarsest level of an AMG hierarchy), so these are latency, not bandwidth, kernels.
template <class T>
__global__ void coarse_gemv(const T* __restrict__ M, const T* __restrict__ b, T* __restrict__ x,
                            int n, int k, int transpose, const int* stop) {
  count_launch();
  if (stop && *stop) return;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n * k; t += gridDim.x * blockDim.x) {
    const int i = t / k, c = t % k;
    T s = T(0);
    if (!transpose) {
      for (int j = 0; j < n; ++j) s = rfma(M[(size_t)i * n + j], b[(size_t)j * k + c], s);
    } else {
      for (int j = 0; j < n; ++j) s = rfma(M[(size_t)j * n + i], b[(size_t)j * k + c], s);
    }
    x[(size_t)i * k + c] = s;
  }
}

// LU (MODE 0: permute, unit-lower forward, upper backward) or QR back-substitution
// (MODE 1: x holds Q^T b on entry, upper backward in place).
template <class T, int MODE>
__global__ void coarse_trsv(const T* __restrict__ LU, const int* __restrict__ perm,
                            const T* __restrict__ b, T* __restrict__ x, int n, int k,
                            const int* stop) {
  count_launch();
  if (stop && *stop) return;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < k; c += gridDim.x * blockDim.x) {
    if (MODE == 0) {
      for (int i = 0; i < n; ++i) x[(size_t)i * k + c] = b[(size_t)perm[i] * k + c];
      for (int i = 0; i < n; ++i) {
        T s = x[(size_t)i * k + c];
        for (int j = 0; j < i; ++j) s = rfma(-LU[(size_t)i * n + j], x[(size_t)j * k + c], s);
        x[(size_t)i * k + c] = s;
      }
    }
    for (int i = n - 1; i >= 0; --i) {
      T s = x[(size_t)i * k + c];
      for (int j = i + 1; j < n; ++j) s = rfma(-LU[(size_t)i * n + j], x[(size_t)j * k + c], s);
      x[(size_t)i * k + c] = s / LU[(size_t)i * n + i];
    }
  }
}

// inverse diagonal (relaxation.py:36-61): d_i = sum of stored (i,i) entries; 1/d or 0.
template <class T>
__global__ void inv_diag_kernel(const int* __restrict__ rowptr, const int* __restrict__ col,
                                const T* __restrict__ val, int n, T* __restrict__ dinv) {
  count_launch();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    T d = T(0);
    for (int nz = rowptr[i]; nz < rowptr[i + 1]; ++nz)
      if (col[nz] == i) d += val[nz];
    dinv[i] = (d != T(0)) ? T(1) / d : T(0);
  }
}

// grad[e] = -sum_c lam[row(e), c] * x[col(e), c]  (sampled -lambda x^T on A's pattern).
static __global__ void sampled_outer_kernel(const int* __restrict__ rowptr, const int* __restrict__ col,
                                     int n_rows, const double* __restrict__ lam,
                                     const double* __restrict__ x, int k, double* __restrict__ grad) {
  count_launch();
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int row = warp; row < n_rows; row += nwarps) {
    const int s = rowptr[row], e = rowptr[row + 1];
    if (k == 1) {
      const double l = lam[row];
      for (int nz = s + lane; nz < e; nz += 32) grad[nz] = -l * x[col[nz]];
    } else {
      for (int nz = s; nz < e; ++nz) {
        const int j = col[nz];
        double acc = 0.0;
        for (int c = lane; c < k; c += 32) acc += lam[(size_t)row * k + c] * x[(size_t)j * k + c];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
        if (lane == 0) grad[nz] = -acc;
      }
    }
  }
}

}  // namespace amg
