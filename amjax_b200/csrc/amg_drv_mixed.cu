// amg_drv_mixed.cu -- mixed-precision drivers: FP32 cycle inside FP64 refinement / FP64 CG.
#include "amg_drivers.cuh"

namespace amg {

// Standalone solve, FP32 cycle inside FP64 iterative refinement (same iterates as the
// plain cycle up to rounding: a linear cycle is x + M (b - A x)).
void solve_mixed(amg_hierarchy* h, Plan* pl, const Req& q, cudaStream_t user) {
  const int n0 = h->levels[0].A.n_rows;
  const double* b = static_cast<const double*>(q.b);
  double* x = static_cast<double*>(q.x);
  float* r32 = static_cast<float*>(pl->B[0]);
  float* e32 = static_cast<float*>(pl->X[0]);
  const char ct = cycle_char(q.cycle);
  const Csr* A0 = q.A0 ? q.A0 : &h->levels[0].A;
  auto prologue = [&](cudaStream_t cs) {
    emit_setup<double, float, 0>(pl, cs, n0, b, nullptr, nullptr, x, q.tol, 0.0, q.maxiter);
  };
  auto body = [&](cudaStream_t cs) {
    OpResid<double, double, XS_PLAIN, false, float, true> rop{};
    rop.xs = XSource<double, XS_PLAIN>{x, b, nullptr, 1.0, q.k};
    rop.b = b;
    rop.out = nullptr;
    rop.out_lo = r32;
    rop.ld = q.k;
    rop.stop = nullptr;
    rop.ctl = make_ctl(pl, q.maxiter);
    run_csr(*A0, rop, q.k, red_of(pl), cs, {x, b, r32});
    Cycle<float> cy{};
    cy.h = h; cy.pl = pl; cy.s = cs; cy.k = q.k; cy.stop = pl->stop(); cy.A0 = A0;
    cy.b0 = r32; cy.x0 = e32; cy.red = red_of(pl);
    cy.tail_from = tail_level<float>(h, q.k, q.program);
    cy.visit(0, true, ct, q.cpl);
    OpRefine<double, float> up{x, e32, pl->active(), q.k, pl->stop()};
    run_elem<float>(n0, up, q.k, red_of(pl), cs, {x, e32});
  };
  autotune_cycle<float>(h, pl, q.k, q.A0, user);
  if (q.k > 1) {  // the outer residual, on scratch (its state is reset by the prologue)
    OpResid<double, double, XS_PLAIN, false, float, true> tr{};
    tr.xs = XSource<double, XS_PLAIN>{static_cast<const double*>(pl->p_out), b, nullptr, 1.0, q.k};
    tr.b = b; tr.out = nullptr; tr.out_lo = r32; tr.ld = q.k; tr.stop = nullptr;
    tr.ctl = make_ctl(pl, q.maxiter);
    tune_op(*A0, tr, q.k, red_of(pl), user, {pl->p_out, b, r32});
  }
  run_loop(pl, req_key("solve", q), user, prologue, body, [](cudaStream_t) {}, true, q.maxiter + 2);
}


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

unsigned long long count_mixed() {
  unsigned long long v = 0;
  cudaMemcpyFromSymbol(&v, g_kernel_count, sizeof(v));
  return v;
}

}  // namespace amg
