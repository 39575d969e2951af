// amg_noalloc.cu -- damped Jacobi sweeps that allocate no device memory.
//
// amg_jacobi needs a second vector for the iterate between sweeps and gets it from
// cudaMallocAsync.  Some callers cannot allocate at the moment they call us: an XLA/JAX
// custom call runs inside memory that XLA has already reserved (it preallocates most of
// the GPU and hands out scratch itself), an application may run on a fixed memory budget
// that forbids new device allocations once its pools are set up, and real-time callers
// cannot afford an allocator call on the solve path.  amg_jacobi_noalloc gives them the
// same sweeps with the intermediate iterate kept in a fixed device array compiled into
// this library (kNoAllocScratchBytes = 16 MiB, held on every GPU that loads the library
// until the process exits).
#include <mutex>
#include <vector>

#include "amg_runtime.cuh"

namespace amg {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;

// The scratch array.  Host code must not pass this name to a kernel: on the host it only
// stands in for the symbol; the device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_scratch_mu;
std::vector<void*> g_scratch_addr;  // device address of g_noalloc_scratch, per device ordinal

// Set-up, once per device, on the current device (the first call on a device does it).
void* scratch_address() {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (int(g_scratch_addr.size()) <= dev) g_scratch_addr.resize(size_t(dev) + 1, nullptr);
  if (g_scratch_addr[size_t(dev)] == nullptr) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      fail(AMG_ERR_CUDA, "cudaGetSymbolAddress of the no-alloc scratch failed on device %d: %s", dev,
           cudaGetErrorString(e));
    g_scratch_addr[size_t(dev)] = p;
  }
  return g_scratch_addr[size_t(dev)];
}

template <class T>
void jacobi_noalloc(const amg_csr* Ad, const void* x, const void* b, const void* dinv, void* out, int k,
                    int iterations, double omega, cudaStream_t s) {
  Csr A(*Ad);
  T* tmp = nullptr;
  if (iterations > 1) {
    const size_t bytes = size_t(A.n_rows) * size_t(k) * sizeof(T);
    if (bytes > kNoAllocScratchBytes)
      fail(AMG_ERR_INVALID_ARG,
           "amg_jacobi_noalloc: %d rows x %d columns need %zu bytes of scratch between sweeps; the "
           "no-alloc variant holds at most %zu bytes (use amg_jacobi, or iterations <= 1)",
           A.n_rows, k, bytes, kNoAllocScratchBytes);
    tmp = static_cast<T*>(scratch_address());
  }
  const T* in = static_cast<const T*>(x);
  for (int i = 0; i < iterations; ++i) {
    // every sweep writes all of its output before the next sweep reads it, so the scratch
    // needs no clearing between calls
    T* o = ((iterations - 1 - i) % 2 == 0) ? static_cast<T*>(out) : tmp;
    OpJacobi<T, XS_PLAIN> op{};
    op.xs = XSource<T, XS_PLAIN>{in, static_cast<const T*>(b), static_cast<const T*>(dinv), T(omega), k};
    op.b = static_cast<const T*>(b);
    op.dinv = static_cast<const T*>(dinv);
    op.omega = T(omega);
    op.out = o;
    op.ld = k;
    run_csr(A, op, k, Red{}, s, {in, b, o});
    in = o;
  }
}

}  // namespace
}  // namespace amg

using namespace amg;

extern "C" amg_status amg_jacobi_noalloc(const amg_csr* A, int32_t dtype, const void* x, const void* b,
                                         const void* dinv, void* out, int32_t k, int32_t iterations,
                                         double omega, void* stream) {
  return guarded([&] {
    if (!A) fail(AMG_ERR_INVALID_ARG, "null matrix");
    check_csr(*A, "A", 0);
    check_vec(x, "x");
    check_vec(b, "b");
    check_vec(dinv, "dinv");
    check_vec(out, "out");
    // every sweep reads x (first sweep), b and dinv while it writes out
    if (x == out || b == out || dinv == out) fail(AMG_ERR_INVALID_ARG, "out may not alias x, b or dinv");
    if (dtype != 0 && dtype != 1) fail(AMG_ERR_INVALID_ARG, "dtype must be 0 (FP64) or 1 (FP32)");
    if (k < 1 || iterations < 0) fail(AMG_ERR_INVALID_ARG, "bad k or iterations");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (iterations == 0) {
      const size_t es = dtype == 0 ? 8 : 4;
      CK(cudaMemcpyAsync(out, x, size_t(A->n_rows) * size_t(k) * es, cudaMemcpyDeviceToDevice, s));
      return;
    }
    if (dtype == 0) jacobi_noalloc<double>(A, x, b, dinv, out, k, iterations, omega, s);
    else if (dtype == 1) jacobi_noalloc<float>(A, x, b, dinv, out, k, iterations, omega, s);
    else fail(AMG_ERR_INVALID_ARG, "dtype must be 0 (FP64) or 1 (FP32)");
  });
}
