// amg_drv_f32.cu -- FP32 solve drivers (the reference's dtype=float32 mode; also the FP32 preconditioner).
#include "amg_drivers.cuh"

namespace amg {

template void solve_plain<float>(amg_hierarchy*, Plan*, const Req&, cudaStream_t);
template void pcg<float, float>(amg_hierarchy*, Plan*, const Req&, cudaStream_t);
template void pcg_emit<float, float>(amg_hierarchy*, Plan*, const Req&, cudaStream_t, Emit*, Emit*);
template void precondition<float>(amg_hierarchy*, Plan*, const Req&, cudaStream_t);

unsigned long long count_f32() {
  unsigned long long v = 0;
  cudaMemcpyFromSymbol(&v, g_kernel_count, sizeof(v));
  return v;
}

}  // namespace amg
