// amg_pcg.cuh -- the preconditioned CG loop, shared by the FP64, FP32 and mixed drivers.
#pragma once

#include "amg_runtime.cuh"

namespace amg {

// Preconditioned CG (outer type TO, cycle type TC): tune, then build the prologue (set-up,
// first cycle, p = z, beta = 0) and the loop body.  One CG step is
//   <p, A p> with p = z + beta p formed inside the same CSR pass (OpCgQDir, which writes the
//   new direction into the other of two direction buffers); A p recomputed with the x / r
//   update and the stop rule (OpCgUpdA); the cycle with the fused <r, z> (new beta).
// The body holds two steps, the second with the direction buffers swapped, so a captured
// graph needs no pointer swap; when the first step stops the loop, every kernel of the
// second returns at once (stop flag).  The emitters capture by value, so they stay valid
// after this returns (a batch captures many of them at once).
template <class TO, class TC>
void pcg_emit(amg_hierarchy* h, Plan* pl, const Req& q, cudaStream_t user, Emit* pro, Emit* bod) {
  const int n0 = h->levels[0].A.n_rows;
  const TO* b = static_cast<const TO*>(q.b);
  TO* x = static_cast<TO*>(q.x);
  TO* r = static_cast<TO*>(pl->r_out);
  TO* pa = static_cast<TO*>(pl->p_out);
  TO* pb = static_cast<TO*>(pl->q_out);
  constexpr bool mixed = !std::is_same<TO, TC>::value;
  TC* rc = mixed ? static_cast<TC*>(pl->B[0]) : reinterpret_cast<TC*>(r);
  TC* z = static_cast<TC*>(pl->X[0]);
  const char ct = cycle_char(q.cycle);
  const Csr* A0 = q.A0 ? q.A0 : &h->levels[0].A;
  const int k = q.k, cpl = q.cpl, maxiter = q.maxiter;
  const double tol = q.tol, atol = q.atol;
  const int tail = tail_level<TC>(h, k, q.program);
  auto cycle = [=](cudaStream_t cs) {
    Cycle<TC> cy{};
    cy.h = h; cy.pl = pl; cy.s = cs; cy.k = k; cy.stop = pl->stop(); cy.A0 = nullptr;
    cy.b0 = rc; cy.x0 = z; cy.fine_dot = r; cy.dot_is_f64 = sizeof(TO) == 8;
    cy.red = red_of(pl);
    cy.tail_from = tail;
    cy.visit(0, true, ct, cpl);
  };
  auto step = [=](cudaStream_t cs, TO* p_old, TO* p_new) {
    NvtxRange nv("amg/cg-step");
    OpCgQDir<TO, TC> qop{p_old, z, p_new, pl->beta(), k, pl->stop(), pl->gamma(), pl->alpha()};
    run_csr(*A0, qop, k, red_of(pl), cs, {p_old, z, p_new});
    OpCgUpdA<TO, TC> up{};
    up.x = x; up.r = r; up.p = p_new; up.r_lo = mixed ? rc : nullptr;
    up.alpha = pl->alpha(); up.active = pl->active(); up.ld = k; up.stop = pl->stop();
    up.ctl = make_ctl(pl, maxiter);
    run_csr(*A0, up, k, red_of(pl), cs, {x, r, p_new, up.r_lo});
    cycle(cs);
  };
  *pro = [=](cudaStream_t cs) {
    emit_setup<TO, TC, 1>(pl, cs, n0, b, r, mixed ? rc : nullptr, x, tol, atol, maxiter);
    cycle(cs);
    // first direction p = z: p_old = 0 and beta = 0 give fma(0, 0, z) = z (a memset node, not
    // a pass that reads z)
    CK(cudaMemsetAsync(pa, 0, sizeof(TO) * size_t(n0) * size_t(k), cs));
    CK(cudaMemsetAsync(pl->beta(), 0, sizeof(double) * size_t(k), cs));
  };
  *bod = [=](cudaStream_t cs) {
    step(cs, pa, pb);
    step(cs, pb, pa);
  };
  autotune_cycle<TC>(h, pl, k, nullptr, user);
  if (h->levels.size() > 1 && h->levels[0].post.on()) {
    // the fine post-smoothing sweep with the fused <r, z>: a reducing launch, tuned on its
    // own (scratch: W1 -> W2 on level 0; the prologue recomputes gamma and zeroes beta)
    const Level& l0 = h->levels[0];
    if (const TC* dv = l0.template dinv<TC>()) {
      TC* w1 = static_cast<TC*>(pl->W1[0]);
      TC* w2 = static_cast<TC*>(pl->W2[0]);
      const TC om = TC(l0.post.omega);
      OpJacobi<TC, XS_PLAIN> op{};
      op.xs = XSource<TC, XS_PLAIN>{w1, rc, dv, om, k};
      op.b = rc; op.dinv = dv; op.omega = om; op.out = w2; op.ld = k;
      op.rdot64 = sizeof(TO) == 8 ? reinterpret_cast<const double*>(r) : nullptr;
      op.rdot32 = sizeof(TO) == 8 ? nullptr : reinterpret_cast<const float*>(r);
      op.gamma = pl->gamma(); op.beta = pl->beta();
      tune_op(*A0, op, k, red_of(pl), user, {w1, rc, w2, r});
    }
  }
  {  // the outer CG ops, on scratch (the prologue resets every state they touch)
    std::vector<int> ones(size_t(k), 1);
    CK(cudaMemcpy(pl->active(), ones.data(), sizeof(int) * k, cudaMemcpyHostToDevice));
    OpCgQDir<TO, TC> tq{pa, z, pb, pl->beta(), k, nullptr, pl->gamma(), pl->alpha()};
    tune_op(*A0, tq, k, red_of(pl), user, {pa, z, pb});
    OpCgUpdA<TO, TC> tu{};
    tu.x = x; tu.r = r; tu.p = pb; tu.r_lo = mixed ? rc : nullptr;
    tu.alpha = pl->alpha(); tu.active = pl->active(); tu.ld = k; tu.stop = nullptr;
    tu.ctl = make_ctl(pl, maxiter);
    tune_op(*A0, tu, k, red_of(pl), user, {x, r, pb, tu.r_lo}, [&](cudaStream_t ts) {
      CK(cudaMemcpyAsync(pl->active(), ones.data(), sizeof(int) * k, cudaMemcpyHostToDevice, ts));
      CK(cudaStreamSynchronize(ts));
    });
  }
}


// Mixed-precision PCG with reliable updates (cycle type TC = float).  The whole CG runs in
// FP32 vectors (direction, residual, and the solution increment xs accumulated since the
// last fold) with FP64 dot products and step lengths; the FP64 solution x and the FP64 true
// residual b - A x are brought up to date only when one is due: after the FP32 residual has
// dropped by delta since the last true residual, when it reports convergence, at maxiter,
// or on a NaN (LoopCtl::cg_col_ru).  Then x += xs, xs = 0, and the true residual (FP64
// values, FP64 x) replaces the FP32 one; the direction is kept, so CG continues without a
// restart.  Columns retire only on the true residual, so the stop rule
// <r, r> <= max(tol^2 <b, b>, atol^2) is checked in FP64.  One CG step is
//   <p, A p> with p = z + beta p (OpCgQDir, FP32); xs += alpha p, r -= alpha A p with the
//   FP32 residual's <r, r> (OpCgUpdA, reliable rule); fold and true residual (both return
//   at once unless due); the cycle on r with the fused <r, z>.
// The epilogue folds any increment left (the loop ended on its trip bound).
template <class TC>
void pcg_ru_emit(amg_hierarchy* h, Plan* pl, const Req& q, cudaStream_t user, Emit* pro, Emit* bod, Emit* epi) {
  static_assert(sizeof(TC) == 4, "the reliable-update CG runs its vectors in FP32");
  const int n0 = h->levels[0].A.n_rows;
  const double* b = static_cast<const double*>(q.b);
  double* x = static_cast<double*>(q.x);
  TC* xs = static_cast<TC*>(pl->r_out);   // FP32 increment (the plan's outer buffers are FP64-sized)
  TC* pa = static_cast<TC*>(pl->p_out);
  TC* pb = static_cast<TC*>(pl->q_out);
  TC* rs = static_cast<TC*>(pl->B[0]);     // FP32 residual = the cycle's right-hand side
  TC* z = static_cast<TC*>(pl->X[0]);
  const char ct = cycle_char(q.cycle);
  const Csr* A0 = q.A0 ? q.A0 : &h->levels[0].A;
  const int k = q.k, cpl = q.cpl, maxiter = q.maxiter;
  const double tol = q.tol, atol = q.atol;
  const LoopCtl ctl = make_ctl(pl, maxiter);
  const int tail = tail_level<TC>(h, k, q.program);
  auto cycle = [=](cudaStream_t cs) {
    Cycle<TC> cy{};
    cy.h = h; cy.pl = pl; cy.s = cs; cy.k = k; cy.stop = pl->stop(); cy.A0 = nullptr;
    cy.b0 = rs; cy.x0 = z; cy.fine_dot = rs; cy.dot_is_f64 = false;
    cy.red = red_of(pl);
    cy.tail_from = tail;
    cy.visit(0, true, ct, cpl);
  };
  auto true_residual = [=](cudaStream_t cs) {
    NvtxRange nv("amg/true-residual");
    OpFold<double, TC> fo{x, xs, k, pl->ru()};
    run_elem<TC>(n0, fo, k, red_of(pl), cs, {x, xs});
    OpResid<double, double, XS_PLAIN, false, TC, true> tr{};
    tr.xs = XSource<double, XS_PLAIN>{x, b, nullptr, 1.0, k};
    tr.b = b; tr.out = nullptr; tr.out_lo = rs; tr.ld = k; tr.stop = pl->stop();
    tr.ctl = ctl; tr.gate = pl->ru(); tr.true_rule = 1;
    run_csr(*A0, tr, k, red_of(pl), cs, {x, b, rs});
  };
  auto step = [=](cudaStream_t cs, TC* p_old, TC* p_new) {
    NvtxRange nv("amg/cg-step");
    OpCgQDir<TC, TC> qop{p_old, z, p_new, pl->beta(), k, pl->stop(), pl->gamma(), pl->alpha()};
    run_csr(*A0, qop, k, red_of(pl), cs, {p_old, z, p_new});
    OpCgUpdA<TC, TC> up{};
    up.x = xs; up.r = rs; up.p = p_new; up.r_lo = nullptr;
    up.alpha = pl->alpha(); up.active = pl->active(); up.ld = k; up.stop = pl->stop();
    up.ctl = ctl; up.reliable = true;
    run_csr(*A0, up, k, red_of(pl), cs, {xs, rs, p_new});
    true_residual(cs);
    cycle(cs);
  };
  *pro = [=](cudaStream_t cs) {
    OpSetup<double, TC, 1> op{};
    op.src = b; op.dst = nullptr; op.dst_lo = rs; op.zero = x; op.ld = k;
    op.thresh = pl->thresh(); op.nr = pl->nr(); op.normb = pl->normb(); op.active = pl->active();
    op.iters = pl->iters(); op.stop = pl->stop(); op.gcount = pl->gcount();
    op.tol = tol; op.atol = atol; op.maxiter = maxiter; op.rmax = pl->rmax(); op.ru = pl->ru();
    run_elem<TC>(n0, op, k, red_of(pl), cs, {b, rs, x});
    CK(cudaMemsetAsync(xs, 0, sizeof(TC) * size_t(n0) * size_t(k), cs));
    cycle(cs);
    CK(cudaMemsetAsync(pa, 0, sizeof(TC) * size_t(n0) * size_t(k), cs));  // p_old = 0, beta = 0: p = z
    CK(cudaMemsetAsync(pl->beta(), 0, sizeof(double) * size_t(k), cs));
  };
  *bod = [=](cudaStream_t cs) {
    step(cs, pa, pb);
    step(cs, pb, pa);
  };
  *epi = [=](cudaStream_t cs) {
    OpFold<double, TC> fo{x, xs, k, pl->ru() + 1};
    run_elem<TC>(n0, fo, k, red_of(pl), cs, {x, xs});
  };
  // tuning, on scratch (the prologue resets every state these launches touch)
  autotune_cycle<TC>(h, pl, k, nullptr, user);
  if (h->levels.size() > 1 && h->levels[0].post.on()) {
    const Level& l0 = h->levels[0];
    if (const TC* dv = l0.template dinv<TC>()) {
      TC* w1 = static_cast<TC*>(pl->W1[0]);
      TC* w2 = static_cast<TC*>(pl->W2[0]);
      const TC om = TC(l0.post.omega);
      OpJacobi<TC, XS_PLAIN> op{};
      op.xs = XSource<TC, XS_PLAIN>{w1, rs, dv, om, k};
      op.b = rs; op.dinv = dv; op.omega = om; op.out = w2; op.ld = k;
      op.rdot32 = reinterpret_cast<const float*>(rs);
      op.gamma = pl->gamma(); op.beta = pl->beta();
      tune_op(l0.A, op, k, red_of(pl), user, {w1, rs, w2, rs});
    }
  }
  {
    std::vector<int> ones(size_t(k), 1);
    auto reset = [&](cudaStream_t ts) {
      CK(cudaMemcpyAsync(pl->active(), ones.data(), sizeof(int) * k, cudaMemcpyHostToDevice, ts));
      CK(cudaStreamSynchronize(ts));
    };
    CK(cudaMemcpy(pl->active(), ones.data(), sizeof(int) * k, cudaMemcpyHostToDevice));
    OpCgQDir<TC, TC> tq{pa, z, pb, pl->beta(), k, nullptr, pl->gamma(), pl->alpha()};
    tune_op(*A0, tq, k, red_of(pl), user, {pa, z, pb});
    OpCgUpdA<TC, TC> tu{};
    tu.x = xs; tu.r = rs; tu.p = pb; tu.r_lo = nullptr;
    tu.alpha = pl->alpha(); tu.active = pl->active(); tu.ld = k; tu.stop = nullptr;
    tu.ctl = ctl; tu.reliable = true;
    tune_op(*A0, tu, k, red_of(pl), user, {xs, rs, pb}, reset);
    OpResid<double, double, XS_PLAIN, false, TC, true> tr{};
    tr.xs = XSource<double, XS_PLAIN>{static_cast<const double*>(pl->q_out), b, nullptr, 1.0, k};
    tr.b = b; tr.out = nullptr; tr.out_lo = rs; tr.ld = k; tr.stop = nullptr;
    tr.ctl = ctl; tr.true_rule = 1;
    tune_op(*A0, tr, k, red_of(pl), user, {pl->q_out, b, rs}, reset);
  }
}

}  // namespace amg
