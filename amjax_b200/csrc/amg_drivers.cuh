// amg_drivers.cuh -- the solve drivers shared by the per-precision translation units:
// standalone solve and preconditioner in one precision end to end, and the PCG loop for
// any (outer type, cycle type) pair.  Each .cu file instantiates the types it owns.
#pragma once

#include "amg_pcg.cuh"

namespace amg {

// Standalone solve, one precision end to end (F64 or F32).
template <class T>
void solve_plain(amg_hierarchy* h, Plan* pl, const Req& q, cudaStream_t user) {
  const int n0 = h->levels[0].A.n_rows;
  const T* b = static_cast<const T*>(q.b);
  T* x = static_cast<T*>(q.x);
  const char ct = cycle_char(q.cycle);
  const Csr* A0 = q.A0 ? q.A0 : &h->levels[0].A;
  auto prologue = [&](cudaStream_t cs) {
    emit_setup<T, T, 0>(pl, cs, n0, b, nullptr, nullptr, x, q.tol, 0.0, q.maxiter);
  };
  auto body = [&](cudaStream_t cs) {
    Cycle<T> cy{};
    cy.h = h; cy.pl = pl; cy.s = cs; cy.k = q.k; cy.stop = pl->stop(); cy.A0 = A0;
    cy.b0 = b; cy.x0 = x; cy.fine_norm = true; cy.ctl = make_ctl(pl, q.maxiter);
    cy.fine_mask = q.k > 1; cy.red = red_of(pl);
    cy.tail_from = tail_level<T>(h, q.k, q.program);
    cy.visit(0, false, ct, q.cpl);
  };
  autotune_cycle<T>(h, pl, q.k, A0, user);
  run_loop(pl, req_key("solve", q), user, prologue, body, [](cudaStream_t) {}, true, q.maxiter + 2);
}


template <class TO, class TC>
void pcg(amg_hierarchy* h, Plan* pl, const Req& q, cudaStream_t user) {
  Emit pro, bod;
  pcg_emit<TO, TC>(h, pl, q, user, &pro, &bod);
  run_loop(pl, req_key("pcg", q), user, pro, bod, [](cudaStream_t) {}, true, q.maxiter + 2);
}


template <class T>
void precondition(amg_hierarchy* h, Plan* pl, const Req& q, cudaStream_t user) {
  const char ct = cycle_char(q.cycle);
  auto prologue = [&](cudaStream_t cs) {
    Cycle<T> cy{};
    cy.h = h; cy.pl = pl; cy.s = cs; cy.k = q.k; cy.stop = nullptr; cy.A0 = nullptr;
    cy.b0 = static_cast<const T*>(q.b); cy.x0 = static_cast<T*>(q.x); cy.red = red_of(pl);
    cy.visit(0, true, ct, q.cpl);
  };
  autotune_cycle<T>(h, pl, q.k, nullptr, user);
  run_loop(pl, req_key("prec", q), user, prologue, [](cudaStream_t) {}, [](cudaStream_t) {}, false, 0);
}

}  // namespace amg
