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
  auto cycle = [=](cudaStream_t cs) {
    Cycle<TC> cy{};
    cy.h = h; cy.pl = pl; cy.s = cs; cy.k = k; cy.stop = pl->stop(); cy.A0 = nullptr;
    cy.b0 = rc; cy.x0 = z; cy.fine_dot = r; cy.dot_is_f64 = sizeof(TO) == 8;
    cy.red = red_of(pl);
    cy.visit(0, true, ct, cpl);
  };
  auto step = [=](cudaStream_t cs, TO* p_old, TO* p_new) {
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
    // first direction p = z: p_old = z and beta = 0 give z + 0 * z = z exactly
    OpConvert<TO, TC> cp{z, pa, k, pl->stop()};
    run_elem<TC>(n0, cp, k, red_of(pl), cs, {z, pa});
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

}  // namespace amg
