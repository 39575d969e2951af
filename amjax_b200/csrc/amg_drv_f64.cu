// amg_drv_f64.cu -- FP64 solve drivers (standalone, PCG, preconditioner).
#include "amg_drivers.cuh"

namespace amg {

template void solve_plain<double>(amg_hierarchy*, Plan*, const Req&, cudaStream_t);
template void pcg<double, double>(amg_hierarchy*, Plan*, const Req&, cudaStream_t);
template void pcg_emit<double, double>(amg_hierarchy*, Plan*, const Req&, cudaStream_t, Emit*, Emit*);
template void precondition<double>(amg_hierarchy*, Plan*, const Req&, cudaStream_t);

unsigned long long count_f64() {
  unsigned long long v = 0;
  cudaMemcpyFromSymbol(&v, g_kernel_count, sizeof(v));
  return v;
}

}  // namespace amg
