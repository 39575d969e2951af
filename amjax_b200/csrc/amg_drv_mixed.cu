// amg_drv_mixed.cu -- mixed-precision drivers: FP32 cycle inside FP64 refinement / FP64 CG.
#include "amg_runtime.cuh"

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

// Preconditioned CG (outer type TO, cycle type TC): tune, then build the prologue (set-up,
// first cycle, p = z) and the loop body (<p, A p>; A p recomputed with the x / r update and
// the stop rule; cycle with the fused <r, z>; p = z + beta p).  The emitters capture by
// value, so they stay valid after this returns (a batch captures many of them at once).
template <class TO, class TC>
void pcg_emit(amg_hierarchy* h, Plan* pl, const Req& q, cudaStream_t user, Emit* pro, Emit* bod) {
  const int n0 = h->levels[0].A.n_rows;
  const TO* b = static_cast<const TO*>(q.b);
  TO* x = static_cast<TO*>(q.x);
  TO* r = static_cast<TO*>(pl->r_out);
  TO* p = static_cast<TO*>(pl->p_out);
  constexpr bool mixed = !std::is_same<TO, TC>::value;
  TC* rc = mixed ? static_cast<TC*>(pl->B[0]) : reinterpret_cast<TC*>(r);
  TC* z = static_cast<TC*>(pl->X[0]);
  const char ct = cycle_char(q.cycle);
  const Csr* A0 = q.A0 ? q.A0 : &h->levels[0].A;
  const int k = q.k, cpl = q.cpl, maxiter = q.maxiter;
  const double tol = q.tol, atol = q.atol;
  auto cycle = [=](cudaStream_t cs) {
    Cycle<TC> cy{};
    cy.h = h; cy.pl = pl; cy.s = cs; cy.k = k; cy.stop = pl->stop(); cy.A0 = nullptr;
    cy.b0 = rc; cy.x0 = z; cy.fine_dot = r; cy.dot_is_f64 = sizeof(TO) == 8;
    cy.red = red_of(pl);
    cy.visit(0, true, ct, cpl);
  };
  *pro = [=](cudaStream_t cs) {
    emit_setup<TO, TC, 1>(pl, cs, n0, b, r, mixed ? rc : nullptr, x, tol, atol, maxiter);
    cycle(cs);
    OpConvert<TO, TC> cp{z, p, k, pl->stop()};
    run_elem<TC>(n0, cp, k, red_of(pl), cs, {z, p});
  };
  *bod = [=](cudaStream_t cs) {
    OpCgQ<TO> qop{p, nullptr, k, pl->stop(), pl->gamma(), pl->alpha()};
    run_csr(*A0, qop, k, red_of(pl), cs, {p});
    OpCgUpdA<TO, TC> up{};
    up.x = x; up.r = r; up.p = p; up.r_lo = mixed ? rc : nullptr;
    up.alpha = pl->alpha(); up.active = pl->active(); up.ld = k; up.stop = pl->stop();
    up.ctl = make_ctl(pl, maxiter);
    run_csr(*A0, up, k, red_of(pl), cs, {x, r, p, up.r_lo});
    cycle(cs);
    OpCgDir<TO, TC> dir{p, z, pl->beta(), k, pl->stop()};
    run_elem<TC>(n0, dir, k, red_of(pl), cs, {p, z});
  };
  autotune_cycle<TC>(h, pl, k, nullptr, user);
  if (k > 1) {  // the outer CG ops, on scratch (the prologue resets every state they touch)
    std::vector<int> ones(size_t(k), 1);
    CK(cudaMemcpy(pl->active(), ones.data(), sizeof(int) * k, cudaMemcpyHostToDevice));
    OpCgQ<TO> tq{p, nullptr, k, nullptr, pl->gamma(), pl->alpha()};
    tune_op(*A0, tq, k, red_of(pl), user, {p});
    OpCgUpdA<TO, TC> tu{};
    tu.x = x; tu.r = r; tu.p = p; tu.r_lo = mixed ? rc : nullptr;
    tu.alpha = pl->alpha(); tu.active = pl->active(); tu.ld = k; tu.stop = nullptr;
    tu.ctl = make_ctl(pl, maxiter);
    tune_op(*A0, tu, k, red_of(pl), user, {x, r, p, tu.r_lo});
  }
}

template <class TO, class TC>
void pcg(amg_hierarchy* h, Plan* pl, const Req& q, cudaStream_t user) {
  Emit pro, bod;
  pcg_emit<TO, TC>(h, pl, q, user, &pro, &bod);
  run_loop(pl, req_key("pcg", q), user, pro, bod, [](cudaStream_t) {}, true, q.maxiter + 2);
}



template void pcg<double, float>(amg_hierarchy*, Plan*, const Req&, cudaStream_t);
template void pcg_emit<double, float>(amg_hierarchy*, Plan*, const Req&, cudaStream_t, Emit*, Emit*);

unsigned long long count_mixed() {
  unsigned long long v = 0;
  cudaMemcpyFromSymbol(&v, g_kernel_count, sizeof(v));
  return v;
}

}  // namespace amg
