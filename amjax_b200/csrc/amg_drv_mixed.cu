// amg_drv_mixed.cu -- mixed-precision standalone drivers: FP32 cycle inside FP64 refinement,
// and the reliable-update standalone solve.
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


// Standalone solve with reliable updates (cycle type float): the FP32 residual r and the
// FP32 increment xs since the last fold are updated after every cycle e = M r in one CSR
// pass (xs += e, r -= A e, <r, r>), and the FP64 solution and FP64 true residual b - A x are
// refreshed when the FP32 norm has dropped by delta since the last refresh, claims
// convergence, reaches maxiter or is not a number.  A column retires only on the FP64 norm
// (the rule of amjax/multilevel.py:414-422: cycle while ||b - A x|| >= tol ||b||).  Per cycle
// this moves one FP32 update pass instead of an FP64 residual pass and an FP64 refinement.
void solve_mixed_ru(amg_hierarchy* h, Plan* pl, const Req& q, cudaStream_t user) {
  const int n0 = h->levels[0].A.n_rows;
  const double* b = static_cast<const double*>(q.b);
  double* x = static_cast<double*>(q.x);
  float* xs = static_cast<float*>(pl->r_out);
  float* rs = static_cast<float*>(pl->B[0]);
  float* e = static_cast<float*>(pl->X[0]);
  const char ct = cycle_char(q.cycle);
  const Csr* A0 = q.A0 ? q.A0 : &h->levels[0].A;
  const int k = q.k;
  const LoopCtl ctl = make_ctl(pl, q.maxiter);
  auto prologue = [&](cudaStream_t cs) {
    OpSetup<double, float, 2> op{};
    op.src = b; op.dst = nullptr; op.dst_lo = rs; op.zero = x; op.ld = k;
    op.thresh = pl->thresh(); op.nr = pl->nr(); op.normb = pl->normb(); op.active = pl->active();
    op.iters = pl->iters(); op.stop = pl->stop(); op.gcount = pl->gcount();
    op.tol = q.tol; op.atol = 0.0; op.maxiter = q.maxiter; op.rmax = pl->rmax(); op.ru = pl->ru();
    run_elem<float>(n0, op, k, red_of(pl), cs, {b, rs, x});
    CK(cudaMemsetAsync(xs, 0, sizeof(float) * size_t(n0) * size_t(k), cs));
  };
  auto body = [&](cudaStream_t cs) {
    Cycle<float> cy{};
    cy.h = h; cy.pl = pl; cy.s = cs; cy.k = k; cy.stop = pl->stop(); cy.A0 = A0;
    cy.b0 = rs; cy.x0 = e; cy.red = red_of(pl);
    cy.tail_from = tail_level<float>(h, k, q.program);
    cy.visit(0, true, ct, q.cpl);
    OpResUpd<float> up{};
    up.e = e; up.xs = xs; up.r = rs; up.active = pl->active(); up.ld = k; up.stop = pl->stop(); up.ctl = ctl;
    run_csr(*A0, up, k, red_of(pl), cs, {e, xs, rs});
    OpFold<double, float> fo{x, xs, k, pl->ru()};
    run_elem<float>(n0, fo, k, red_of(pl), cs, {x, xs});
    OpResid<double, double, XS_PLAIN, false, float, true> tr{};
    tr.xs = XSource<double, XS_PLAIN>{x, b, nullptr, 1.0, k};
    tr.b = b; tr.out = nullptr; tr.out_lo = rs; tr.ld = k; tr.stop = pl->stop();
    tr.ctl = ctl; tr.gate = pl->ru(); tr.true_rule = 2;
    run_csr(*A0, tr, k, red_of(pl), cs, {x, b, rs});
  };
  auto epilogue = [&](cudaStream_t cs) {
    OpFold<double, float> fo{x, xs, k, pl->ru() + 1};
    run_elem<float>(n0, fo, k, red_of(pl), cs, {x, xs});
  };
  autotune_cycle<float>(h, pl, k, q.A0, user);
  {  // the update and the true residual, on scratch (the prologue resets their state)
    std::vector<int> ones(size_t(k), 1);
    auto reset = [&](cudaStream_t ts) {
      CK(cudaMemcpyAsync(pl->active(), ones.data(), sizeof(int) * k, cudaMemcpyHostToDevice, ts));
      CK(cudaStreamSynchronize(ts));
    };
    reset(user);
    float* w1 = static_cast<float*>(pl->W1[0]);
    float* w2 = static_cast<float*>(pl->W2[0]);
    OpResUpd<float> tu{};
    tu.e = e; tu.xs = w1; tu.r = w2; tu.active = pl->active(); tu.ld = k; tu.stop = nullptr; tu.ctl = ctl;
    tune_op(*A0, tu, k, red_of(pl), user, {e, w1, w2}, reset);
    OpResid<double, double, XS_PLAIN, false, float, true> tr{};
    tr.xs = XSource<double, XS_PLAIN>{static_cast<const double*>(pl->q_out), b, nullptr, 1.0, k};
    tr.b = b; tr.out = nullptr; tr.out_lo = rs; tr.ld = k; tr.stop = nullptr; tr.ctl = ctl; tr.true_rule = 2;
    tune_op(*A0, tr, k, red_of(pl), user, {pl->q_out, b, rs}, reset);
  }
  run_loop(pl, req_key("solve-ru", q), user, prologue, body, epilogue, true, q.maxiter + 2);
}

unsigned long long count_mixed() {
  unsigned long long v = 0;
  cudaMemcpyFromSymbol(&v, g_kernel_count, sizeof(v));
  return v;
}

}  // namespace amg
