// amg_program.cu -- the persistent program kernel (cooperative launch) and its launcher.
#include <cstdlib>
#include <map>
#include <mutex>

#include "amg_runtime.cuh"

namespace amg {

// One cooperative launch runs p.steps in order; a grid barrier follows every step that
// asks for one.  No CTA returns before the last step except on a stop flag (checked once,
// uniformly, before any work) or a barrier that ran out of time.
template <class T>
__global__ void __launch_bounds__(kBlock) program_kernel(const Program p, int k, const int* stop, GridBar gb) {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&g_kernel_count, 1ull);
  if (stop && *stop) return;
  const int gtid = blockIdx.x * kBlock + threadIdx.x;
  const int nth = gridDim.x * kBlock;
  for (int i = 0; i < p.nsteps; ++i) {
    prog_step<T>(p.steps[i], k, gtid, nth);
    if (p.steps[i].barrier && i + 1 < p.nsteps && !grid_sync(gb)) return;
  }
}

int program_grid(bool f64) {
  const void* fn = f64 ? reinterpret_cast<const void*>(program_kernel<double>)
                       : reinterpret_cast<const void*>(program_kernel<float>);
  static const int per_sm_cap = [] {  // AMG_PROGRAM_CTAS: CTAs per SM (default: all that fit)
    const char* e = std::getenv("AMG_PROGRAM_CTAS");
    const int v = e ? atoi(e) : 0;
    return v > 0 ? v : 64;
  }();
  const int per_sm = std::min(resident_ctas(fn, 0), per_sm_cap);
  return std::min(dev_info().nsm * per_sm, kBarMaxCtas);
}

void launch_program(const Program& p, bool f64, int k, const int* stop, const GridBar& gb, cudaStream_t s) {
  if (p.nsteps <= 0) return;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(program_grid(f64));
  cfg.blockDim = dim3(kBlock);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (f64) CK(cudaLaunchKernelEx(&cfg, program_kernel<double>, p, k, stop, gb));
  else CK(cudaLaunchKernelEx(&cfg, program_kernel<float>, p, k, stop, gb));
}

long long spin_limit() {
  static const long long v = [] {
    const char* e = std::getenv("AMG_SPIN_LIMIT");
    const long long d = 1ll << 31;
    if (!e) return d;
    const long long x = atoll(e);
    return x > 0 ? x : d;
  }();
  return v;
}

bool programs_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("AMG_PROGRAM");
    return e && e[0] == '1';
  }();
  return on;
}

unsigned long long count_program() {
  unsigned long long v = 0;
  cudaMemcpyFromSymbol(&v, g_kernel_count, sizeof(v));
  return v;
}

}  // namespace amg
