// amg_drv_mixed_cg.cu -- mixed-precision PCG drivers: the reliable-update CG (FP32 vectors,
// FP64 refreshes) and the FP64 CG around the FP32 cycle.
#include "amg_drivers.cuh"

namespace amg {

// Mixed-precision PCG in the reliable-update form (FP32 CG, FP64 solution and true
// residual on demand).
void pcg_ru(amg_hierarchy* h, Plan* pl, const Req& q, cudaStream_t user) {
  Emit pro, bod, epi;
  pcg_ru_emit<float>(h, pl, q, user, &pro, &bod, &epi);
  run_loop(pl, req_key("pcg-ru", q), user, pro, bod, epi, true, q.maxiter + 2);
}

template void pcg<double, float>(amg_hierarchy*, Plan*, const Req&, cudaStream_t);
template void pcg_ru_emit<float>(amg_hierarchy*, Plan*, const Req&, cudaStream_t, Emit*, Emit*, Emit*);
template void pcg_emit<double, float>(amg_hierarchy*, Plan*, const Req&, cudaStream_t, Emit*, Emit*);

unsigned long long count_mixed_cg() {
  unsigned long long v = 0;
  cudaMemcpyFromSymbol(&v, g_kernel_count, sizeof(v));
  return v;
}

}  // namespace amg
