// amg_capi.cu -- the C ABI (include/amg_b200.h) over the runtime.
#include "amg_runtime.cuh"

// ======================================================================= C ABI
using namespace amg;

// Column padding.  A request whose k is above 8 and not a multiple of 8 would run every CSR
// pass with narrow column vectors (KV = 1 or 2 instead of the 32-byte layouts; measured at
// N = 250,000, mixed PCG: k = 21 7.85 ms, k = 24 3.53 ms; k = 43 11.5 ms, k = 48 5.31 ms).
// It runs on kp = ceil(k / 8) * 8 columns instead: the right-hand sides are copied into a
// zero-padded [n, kp] block, the padding columns (zero right-hand side) retire before their
// first iteration, and the first k columns of the solution are copied back.  Columns are
// independent, so the k solved columns are the same solve.
static int padded_k(int k) { return (k > 8 && k % 8 != 0) ? (k + 7) / 8 * 8 : k; }

struct PadReq {  // what a padded request hands to the solve (h->mu held)
  const void* b;
  void* x;
  int k;
};

static PadReq pad_columns(amg_hierarchy* h, const void* b, void* x, int k, size_t es, cudaStream_t s) {
  const int kp = padded_k(k);
  if (kp == k) return PadReq{b, x, k};
  const int n = h->levels[0].A.n_rows;
  const size_t bytes = std::max<size_t>(size_t(n) * kp * es, 256);
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (!h->pads.count(s) && int(h->pads.size()) >= max_plans()) {  // free the least recently used stage
    auto used = [](const std::unique_ptr<PadStage>& st) { return st ? st->last_use : 0; };
    auto lru = h->pads.begin();
    for (auto p = h->pads.begin(); p != h->pads.end(); ++p)
      if (used(p->second) < used(lru->second)) lru = p;
    CK(cudaDeviceSynchronize());
    h->pads.erase(lru);
  }
  std::unique_ptr<PadStage>& slot = h->pads[s];
  if (!slot || slot->dev != dev || slot->bytes < bytes) {
    if (slot) CK(cudaStreamSynchronize(s));  // the old staging may still be read on s
    slot.reset();
    auto p = std::make_unique<PadStage>();
    p->dev = dev;
    p->bytes = bytes;
    CK(cudaMalloc(&p->b, bytes));
    CK(cudaMalloc(&p->x, bytes));
    slot = std::move(p);
  }
  slot->last_use = ++h->use_clock;
  CK(cudaMemcpy2DAsync(slot->b, kp * es, b, k * es, k * es, size_t(n), cudaMemcpyDeviceToDevice, s));
  CK(cudaMemset2DAsync(static_cast<char*>(slot->b) + k * es, kp * es, 0, (kp - k) * es, size_t(n), s));
  return PadReq{slot->b, slot->x, kp};
}

// Copy the first k solution columns back and the per-column results of those columns.
static void unpad_columns(amg_hierarchy* h, const PadReq& r, void* x, int k, size_t es, cudaStream_t s) {
  if (r.k == k) return;
  const int n = h->levels[0].A.n_rows;
  CK(cudaMemcpy2DAsync(x, k * es, r.x, size_t(r.k) * es, k * es, size_t(n), cudaMemcpyDeviceToDevice, s));
}


template <class TO, class TC, bool RU = false>
static void pcg_batch_impl(amg_hierarchy* const* hs, int nsys, int precision, const void* const* b,
                           void* const* x, const int32_t* k, double tol, double atol, int maxiter,
                           int cycle, int cpl, int32_t* iters_out, double* relres_out, cudaStream_t s) {
  std::vector<BatchSys> sys;
  std::vector<Plan*> plans;
  std::vector<PadReq> pads;
  std::string key = "batch";
  const size_t es = sizeof(TO);
  for (int i = 0; i < nsys; ++i) {
    pads.push_back(pad_columns(hs[i], b[i], x[i], k[i], es, s));  // each hierarchy appears once
    const PadReq& pr = pads.back();
    Plan* pl = get_plan(hs[i], precision, pr.k, s);
    Req q{precision, pr.k, cycle, cpl, maxiter, tol, atol, pr.b, pr.x, nullptr};
    BatchSys bs;
    bs.pl = pl;
    bs.gmax = maxiter + 2;
    const bool ru = RU && pr.k > 1;  // MIXED at k = 1 runs the FP64-CG form (faster there)
    if (ru) {
      if constexpr (RU) pcg_ru_emit<TC>(hs[i], pl, q, s, &bs.pro, &bs.body, &bs.epi);
    } else {
      pcg_emit<TO, TC>(hs[i], pl, q, s, &bs.pro, &bs.body);
    }
    sys.push_back(std::move(bs));
    plans.push_back(pl);
    char buf[48];
    snprintf(buf, sizeof(buf), "/%p:", (void*)hs[i]);
    key += buf + req_key(ru ? "pcg-ru" : "pcg", q);
  }
  run_batch(sys, key, s);
  size_t off = 0;
  for (int i = 0; i < nsys; ++i) {
    unpad_columns(hs[i], pads[size_t(i)], x[i], k[i], es, s);
    std::vector<int32_t> it(size_t(pads[size_t(i)].k));
    std::vector<double> rr(size_t(pads[size_t(i)].k));
    read_results(plans[size_t(i)], s, true, iters_out ? it.data() : nullptr, relres_out ? rr.data() : nullptr);
    if (iters_out) std::copy(it.begin(), it.begin() + k[i], iters_out + off);
    if (relres_out) std::copy(rr.begin(), rr.begin() + k[i], relres_out + off);
    off += size_t(k[i]);
  }
}

template <class T>
static void jacobi_impl(const amg_csr* Ad, const void* x, const void* b, const void* dinv, void* out,
                        int k, int iterations, double omega, cudaStream_t s) {
  Csr A(*Ad);
  T* tmp = nullptr;
  const size_t bytes = size_t(A.n_rows) * k * sizeof(T);
  if (iterations > 1) CK(cudaMallocAsync(reinterpret_cast<void**>(&tmp), bytes, s));
  try {
    const T* in = static_cast<const T*>(x);
    {  // pick the layout once per (matrix, k, type); tuning writes only `out`
      OpJacobi<T, XS_PLAIN> top{};
      top.xs = XSource<T, XS_PLAIN>{in, static_cast<const T*>(b), static_cast<const T*>(dinv), T(omega), k};
      top.b = static_cast<const T*>(b);
      top.dinv = static_cast<const T*>(dinv);
      top.omega = T(omega);
      top.out = static_cast<T*>(out);
      top.ld = k;
      tune_op(A, top, k, Red{}, s, {in, b, out});
    }
    for (int i = 0; i < iterations; ++i) {
      T* o = ((iterations - 1 - i) % 2 == 0) ? static_cast<T*>(out) : tmp;
      OpJacobi<T, XS_PLAIN> op{};
      op.xs = XSource<T, XS_PLAIN>{in, static_cast<const T*>(b), static_cast<const T*>(dinv), T(omega), k};
      op.b = static_cast<const T*>(b);
      op.dinv = static_cast<const T*>(dinv);
      op.omega = T(omega);
      op.out = o;
      op.ld = k;
      run_csr(A, op, k, Red{}, s, {in, b, o});
      in = o;
    }
  } catch (...) {
    if (tmp) cudaFreeAsync(tmp, s);
    throw;
  }
  if (tmp) CK(cudaFreeAsync(tmp, s));
}


// Bodies of amg_solve / amg_pcg (also run by amg_adjoint).
static void solve_body(amg_hierarchy* h, int precision, const void* b, void* x, int k, double tol, int maxiter,
                       int cycle, int cycles_per_level, const amg_csr* A0, int32_t* iters_out, double* relres_out,
                       cudaStream_t s) {
  if (!h) fail(AMG_ERR_INVALID_ARG, "null hierarchy");
  check_vec(b, "b");
  check_vec(x, "x");
  if (k < 1) fail(AMG_ERR_INVALID_ARG, "k must be >= 1");
  if (maxiter < 0) fail(AMG_ERR_INVALID_ARG, "maxiter must be >= 0");
  cycle_char(cycle);
  std::lock_guard<std::mutex> lk(h->mu);
  Csr a0;
  const Csr* pa0 = nullptr;
  if (A0) { a0 = override_csr(h, A0, s); pa0 = &a0; }
  check_prec_data(h, precision, pa0);
  if (precision < AMG_PREC_F64 || precision > AMG_PREC_MIXED_F64CG) fail(AMG_ERR_INVALID_ARG, "unknown precision %d", precision);
  const size_t es = precision == AMG_PREC_F32 ? 4 : 8;
  const PadReq pr = pad_columns(h, b, x, k, es, s);
  Plan* pl = get_plan(h, precision, pr.k, s);
  Req q{precision, pr.k, cycle, cycles_per_level, maxiter, tol, 0.0, pr.b, pr.x, pa0};
  q.program = true;
  if (precision == AMG_PREC_F64) solve_plain<double>(h, pl, q, s);
  else if (precision == AMG_PREC_F32) solve_plain<float>(h, pl, q, s);
  else if (precision == AMG_PREC_MIXED && (!pa0 || pa0->v32)) solve_mixed_ru(h, pl, q, s);
  else solve_mixed(h, pl, q, s);  // MIXED_F64CG: FP64 refinement around the FP32 cycle
  unpad_columns(h, pr, x, k, es, s);
  std::vector<int32_t> it(size_t(pr.k));
  std::vector<double> rr(size_t(pr.k));
  read_results(pl, s, false, iters_out ? it.data() : nullptr, relres_out ? rr.data() : nullptr);
  if (iters_out) std::copy(it.begin(), it.begin() + k, iters_out);
  if (relres_out) std::copy(rr.begin(), rr.begin() + k, relres_out);
}

static void pcg_body(amg_hierarchy* h, int precision, const void* b, void* x, int k, double tol, double atol,
                     int maxiter, int cycle, int cycles_per_level, const amg_csr* A0, int32_t* iters_out,
                     double* relres_out, cudaStream_t s) {
  if (!h) fail(AMG_ERR_INVALID_ARG, "null hierarchy");
  check_vec(b, "b");
  check_vec(x, "x");
  if (k < 1) fail(AMG_ERR_INVALID_ARG, "k must be >= 1");
  if (maxiter < 0) fail(AMG_ERR_INVALID_ARG, "maxiter must be >= 0");
  cycle_char(cycle);
  std::lock_guard<std::mutex> lk(h->mu);
  Csr a0;
  const Csr* pa0 = nullptr;
  if (A0) { a0 = override_csr(h, A0, s); pa0 = &a0; }
  check_prec_data(h, precision, nullptr);
  if (pa0 && (precision == AMG_PREC_F32 ? !pa0->v32 : !pa0->v64))
    fail(AMG_ERR_INVALID_ARG, "A0 lacks values for this precision");
  if (precision < AMG_PREC_F64 || precision > AMG_PREC_MIXED_F64CG) fail(AMG_ERR_INVALID_ARG, "unknown precision %d", precision);
  const size_t es = precision == AMG_PREC_F32 ? 4 : 8;
  const PadReq pr = pad_columns(h, b, x, k, es, s);
  Plan* pl = get_plan(h, precision, pr.k, s);
  Req q{precision, pr.k, cycle, cycles_per_level, maxiter, tol, atol, pr.b, pr.x, pa0};
  q.program = true;
  if (precision == AMG_PREC_F64) pcg<double, double>(h, pl, q, s);
  else if (precision == AMG_PREC_F32) pcg<float, float>(h, pl, q, s);
  else if (precision == AMG_PREC_MIXED && pr.k > 1 && (!pa0 || pa0->v32)) pcg_ru(h, pl, q, s);
  else pcg<double, float>(h, pl, q, s);  // MIXED_F64CG; MIXED at k = 1 (faster there)
  unpad_columns(h, pr, x, k, es, s);
  std::vector<int32_t> it(size_t(pr.k));
  std::vector<double> rr(size_t(pr.k));
  read_results(pl, s, true, iters_out ? it.data() : nullptr, relres_out ? rr.data() : nullptr);
  if (iters_out) std::copy(it.begin(), it.begin() + k, iters_out);
  if (relres_out) std::copy(rr.begin(), rr.begin() + k, relres_out);
}


extern "C" {

amg_status amg_hierarchy_create(const amg_level_desc* levels, int32_t n_levels,
                                const amg_coarse_desc* coarse, amg_hierarchy** out) {
  return guarded([&] {
    if (!out || !levels || !coarse) fail(AMG_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    if (n_levels < 2) fail(AMG_ERR_UNSUPPORTED, "a hierarchy needs at least 2 levels (got %d)", n_levels);
    auto h = std::make_unique<amg_hierarchy>();
    for (int l = 0; l < n_levels; ++l) {
      const amg_level_desc& d = levels[l];
      check_csr(d.A, "A", l);
      if (d.A.n_rows != d.A.n_cols) fail(AMG_ERR_INVALID_ARG, "level %d: A is not square", l);
      Level lv;
      lv.A = Csr(d.A);
      if (l < n_levels - 1) {
        check_csr(d.P, "P", l);
        check_csr(d.R, "R", l);
        const int nc = levels[l + 1].A.n_rows;
        if (d.P.n_rows != d.A.n_rows || d.P.n_cols != nc)
          fail(AMG_ERR_INVALID_ARG, "level %d: P is %dx%d, expected %dx%d", l, d.P.n_rows, d.P.n_cols, d.A.n_rows, nc);
        if (d.R.n_rows != nc || d.R.n_cols != d.A.n_rows)
          fail(AMG_ERR_INVALID_ARG, "level %d: R is %dx%d, expected %dx%d", l, d.R.n_rows, d.R.n_cols, nc, d.A.n_rows);
        lv.P = Csr(d.P);
        lv.R = Csr(d.R);
        for (const amg_smoother* sm : {&d.pre, &d.post})
          if (sm->kind != AMG_SMOOTH_NONE && sm->kind != AMG_SMOOTH_JACOBI)
            fail(AMG_ERR_INVALID_ARG, "level %d: unknown smoother kind %d", l, sm->kind);
        lv.pre = Smooth{d.pre.kind, d.pre.iterations, d.pre.omega};
        lv.post = Smooth{d.post.kind, d.post.iterations, d.post.omega};
      }
      lv.dinv64 = d.dinv64;
      lv.dinv32 = d.dinv32;
      h->levels.push_back(lv);
    }
    Coarse c;
    c.kind = coarse->kind;
    c.n = coarse->n;
    c.m0_64 = coarse->m0_64; c.m0_32 = coarse->m0_32;
    c.m1_64 = coarse->m1_64; c.m1_32 = coarse->m1_32;
    c.perm = coarse->perm;
    c.iters = coarse->iterations;
    c.omega = coarse->omega;
    if (c.kind < AMG_COARSE_PINV || c.kind > AMG_COARSE_JACOBI)
      fail(AMG_ERR_INVALID_ARG, "unknown coarse solver kind %d", c.kind);
    if (c.n != h->levels.back().A.n_rows)
      fail(AMG_ERR_INVALID_ARG, "coarse n=%d does not match the coarsest level (%d)", c.n, h->levels.back().A.n_rows);
    if (c.kind == AMG_COARSE_LU && !c.perm) fail(AMG_ERR_INVALID_ARG, "LU coarse solver needs perm");
    // structure of every operator on the device (the arrays may still be filling on another
    // stream: wait for the device first)
    CK(cudaDeviceSynchronize());
    for (int l = 0; l < n_levels; ++l) {
      validate_csr(levels[l].A, "A", l, nullptr, false);
      if (l < n_levels - 1) {
        validate_csr(levels[l].P, "P", l, nullptr, false);
        validate_csr(levels[l].R, "R", l, nullptr, false);
      }
    }
    h->coarse = c;
    *out = h.release();
  });
}

amg_status amg_hierarchy_destroy(amg_hierarchy* h) {
  return guarded([&] { delete h; });
}

amg_status amg_solve(amg_hierarchy* h, int32_t precision, const void* b, void* x, int32_t k,
                     double tol, int32_t maxiter, int32_t cycle, int32_t cycles_per_level,
                     const amg_csr* A0, int32_t* iters_out, double* relres_out, void* stream) {
  return guarded([&] {
    solve_body(h, precision, b, x, k, tol, maxiter, cycle, cycles_per_level, A0, iters_out, relres_out,
               static_cast<cudaStream_t>(stream));
  });
}

amg_status amg_precondition(amg_hierarchy* h, int32_t precision, const void* b, void* x,
                            int32_t k, int32_t cycle, int32_t cycles_per_level, void* stream) {
  return guarded([&] {
    if (!h) fail(AMG_ERR_INVALID_ARG, "null hierarchy");
    check_vec(b, "b");
    check_vec(x, "x");
    if (k < 1) fail(AMG_ERR_INVALID_ARG, "k must be >= 1");
    cycle_char(cycle);
    std::lock_guard<std::mutex> lk(h->mu);
    const int cprec = precision == AMG_PREC_F64 ? AMG_PREC_F64 : AMG_PREC_F32;
    check_prec_data(h, cprec, nullptr);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Plan* pl = get_plan(h, precision, k, s);
    Req q{precision, k, cycle, cycles_per_level, 0, 0.0, 0.0, b, x, nullptr};
    if (precision == AMG_PREC_F64) precondition<double>(h, pl, q, s);
    else if (precision == AMG_PREC_F32 || is_mixed(precision)) precondition<float>(h, pl, q, s);
    else fail(AMG_ERR_INVALID_ARG, "unknown precision %d", precision);
  });
}

amg_status amg_pcg(amg_hierarchy* h, int32_t precision, const void* b, void* x, int32_t k,
                   double tol, double atol, int32_t maxiter, int32_t cycle,
                   int32_t cycles_per_level, const amg_csr* A0, int32_t* iters_out,
                   double* relres_out, void* stream) {
  return guarded([&] {
    pcg_body(h, precision, b, x, k, tol, atol, maxiter, cycle, cycles_per_level, A0, iters_out, relres_out,
             static_cast<cudaStream_t>(stream));
  });
}

amg_status amg_pcg_host(amg_hierarchy* h, int32_t precision, const double* b_host, double* x_host, int32_t k,
                        int32_t blocks, double tol, double atol, int32_t maxiter, int32_t cycle,
                        int32_t cycles_per_level, int32_t* iters_out, double* relres_out, void* stream) {
  return guarded([&] {
    if (!h) fail(AMG_ERR_INVALID_ARG, "null hierarchy");
    if (!b_host || !x_host) fail(AMG_ERR_INVALID_ARG, "null host buffer");
    if (precision == AMG_PREC_F32) fail(AMG_ERR_UNSUPPORTED, "amg_pcg_host moves FP64 vectors: use F64 or a mixed precision");
    if (k < 1 || blocks < 1) fail(AMG_ERR_INVALID_ARG, "k and blocks must be >= 1");
    std::lock_guard<std::mutex> sl(h->stage_mu);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int n = h->levels[0].A.n_rows;
    const int kc = (k + blocks - 1) / blocks;
    const int nb = (k + kc - 1) / kc;
    int dev = 0;
    CK(cudaGetDevice(&dev));
    HostStage* st = h->stage.get();
    if (!st || st->dev != dev || st->n != n || st->kc < kc) {
      h->stage.reset();
      auto ns = std::make_unique<HostStage>();
      ns->dev = dev;
      ns->n = n;
      ns->kc = kc;
      const size_t bytes = std::max<size_t>(size_t(n) * kc * sizeof(double), 256);
      for (int i = 0; i < 2; ++i) {
        CK(cudaMalloc(reinterpret_cast<void**>(&ns->b[i]), bytes));
        CK(cudaMalloc(reinterpret_cast<void**>(&ns->x[i]), bytes));
        CK(cudaEventCreateWithFlags(&ns->in_done[i], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ns->solved[i], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ns->out_done[i], cudaEventDisableTiming));
      }
      CK(cudaStreamCreateWithFlags(&ns->h2d, cudaStreamNonBlocking));
      CK(cudaStreamCreateWithFlags(&ns->d2h, cudaStreamNonBlocking));
      h->stage = std::move(ns);
      st = h->stage.get();
    }
    // the caller's earlier work on s (e.g. writes into the host buffers' device sources)
    // comes first
    cudaEvent_t start;
    CK(cudaEventCreateWithFlags(&start, cudaEventDisableTiming));
    CK(cudaEventRecord(start, s));
    CK(cudaStreamWaitEvent(st->h2d, start, 0));
    cudaEventDestroy(start);
    auto width = [&](int c) { return std::min(kc, k - c * kc); };
    auto copy_in = [&](int c) {  // block c -> slot c % 2, once the solve of block c - 2 is done with it
      const int sl2 = c & 1, w = width(c);
      if (c >= 2) CK(cudaStreamWaitEvent(st->h2d, st->solved[sl2], 0));
      CK(cudaMemcpy2DAsync(st->b[sl2], size_t(w) * 8, b_host + size_t(c) * kc, size_t(k) * 8, size_t(w) * 8, size_t(n),
                           cudaMemcpyHostToDevice, st->h2d));
      CK(cudaEventRecord(st->in_done[sl2], st->h2d));
    };
    copy_in(0);
    if (nb > 1) copy_in(1);
    for (int c = 0; c < nb; ++c) {
      const int sl2 = c & 1, w = width(c);
      CK(cudaStreamWaitEvent(s, st->in_done[sl2], 0));
      if (c >= 2) CK(cudaStreamWaitEvent(s, st->out_done[sl2], 0));  // x slot drained to the host
      pcg_body(h, precision, st->b[sl2], st->x[sl2], w, tol, atol, maxiter, cycle, cycles_per_level, nullptr,
               iters_out ? iters_out + size_t(c) * kc : nullptr, relres_out ? relres_out + size_t(c) * kc : nullptr, s);
      CK(cudaEventRecord(st->solved[sl2], s));
      CK(cudaStreamWaitEvent(st->d2h, st->solved[sl2], 0));
      CK(cudaMemcpy2DAsync(x_host + size_t(c) * kc, size_t(k) * 8, st->x[sl2], size_t(w) * 8, size_t(w) * 8, size_t(n),
                           cudaMemcpyDeviceToHost, st->d2h));
      CK(cudaEventRecord(st->out_done[sl2], st->d2h));
      if (c + 2 < nb) copy_in(c + 2);
    }
    CK(cudaStreamSynchronize(st->d2h));
  });
}

amg_status amg_adjoint(amg_hierarchy* ht, int32_t precision, int32_t method, const void* gx, const double* x,
                       int32_t k, double tol, double atol, int32_t maxiter, int32_t cycle, int32_t cycles_per_level,
                       const amg_csr* At, const amg_csr* pattern, void* lam, double* grad, int32_t* iters_out,
                       double* relres_out, void* stream) {
  return guarded([&] {
    if (precision == AMG_PREC_F32)
      fail(AMG_ERR_UNSUPPORTED, "amg_adjoint returns FP64 gradients: use F64, MIXED or MIXED_F64CG");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (grad) {  // check the gradient's inputs before any solve runs
      if (!pattern) fail(AMG_ERR_INVALID_ARG, "grad needs A's pattern");
      check_vec(x, "x");
      if (!ht) fail(AMG_ERR_INVALID_ARG, "null hierarchy");
      const int n0 = ht->levels[0].A.n_rows;
      if (pattern->n_rows != n0 || pattern->n_cols != n0)
        fail(AMG_ERR_INVALID_ARG, "pattern is %dx%d, expected %dx%d", pattern->n_rows, pattern->n_cols, n0, n0);
      validate_csr(*pattern, "pattern", 0, s, true);
    }
    if (method == 0) {
      solve_body(ht, precision, gx, lam, k, tol, maxiter, cycle, cycles_per_level, At, iters_out, relres_out, s);
    } else if (method == 1) {
      pcg_body(ht, precision, gx, lam, k, tol, atol, maxiter, cycle, cycles_per_level, At, iters_out, relres_out, s);
    } else {
      fail(AMG_ERR_INVALID_ARG, "method must be 0 (standalone solve) or 1 (PCG)");
    }
    if (grad && pattern->n_rows > 0) {
      const int grid = std::max(1, std::min((pattern->n_rows + 7) / 8, dev_info().max_ctas));
      sampled_outer_kernel<<<grid, 256, 0, s>>>(pattern->rowptr, pattern->col, pattern->n_rows,
                                               static_cast<const double*>(lam), x, k, grad);
      CK_LAUNCH();
    }
  });
}

amg_status amg_jacobi(const amg_csr* A, int32_t dtype, const void* x, const void* b,
                      const void* dinv, void* out, int32_t k, int32_t iterations, double omega,
                      void* stream) {
  return guarded([&] {
    if (!A) fail(AMG_ERR_INVALID_ARG, "null matrix");
    validate_csr(*A, "A", 0, static_cast<cudaStream_t>(stream), true);
    check_vec(x, "x"); check_vec(b, "b"); check_vec(dinv, "dinv"); check_vec(out, "out");
    // every sweep reads x (first sweep), b and dinv while it writes out
    if (x == out || b == out || dinv == out) fail(AMG_ERR_INVALID_ARG, "out may not alias x, b or dinv");
    if (dtype != 0 && dtype != 1) fail(AMG_ERR_INVALID_ARG, "dtype must be 0 (FP64) or 1 (FP32)");
    if (k < 1 || iterations < 0) fail(AMG_ERR_INVALID_ARG, "bad k or iterations");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (iterations == 0) {
      const size_t es = dtype == 0 ? 8 : 4;
      CK(cudaMemcpyAsync(out, x, size_t(A->n_rows) * k * es, cudaMemcpyDeviceToDevice, s));
      return;
    }
    if (dtype == 0) jacobi_impl<double>(A, x, b, dinv, out, k, iterations, omega, s);
    else if (dtype == 1) jacobi_impl<float>(A, x, b, dinv, out, k, iterations, omega, s);
    else fail(AMG_ERR_INVALID_ARG, "dtype must be 0 (FP64) or 1 (FP32)");
  });
}

amg_status amg_spmv(const amg_csr* A, int32_t dtype, const void* x, void* y, int32_t k, void* stream) {
  return guarded([&] {
    if (!A) fail(AMG_ERR_INVALID_ARG, "null matrix");
    validate_csr(*A, "A", 0, static_cast<cudaStream_t>(stream), true);
    check_vec(x, "x"); check_vec(y, "y");
    if (k < 1) fail(AMG_ERR_INVALID_ARG, "k must be >= 1");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Csr M(*A);
    if (dtype == 0) {
      OpAxpy<double, XS_ZERO> op{};
      op.x = static_cast<const double*>(x); op.out = static_cast<double*>(y); op.ld = k;
      tune_op(M, op, k, Red{}, s, {x, y});
      run_csr(M, op, k, Red{}, s, {x, y});
    } else if (dtype == 1) {
      OpAxpy<float, XS_ZERO> op{};
      op.x = static_cast<const float*>(x); op.out = static_cast<float*>(y); op.ld = k;
      tune_op(M, op, k, Red{}, s, {x, y});
      run_csr(M, op, k, Red{}, s, {x, y});
    } else {
      fail(AMG_ERR_INVALID_ARG, "dtype must be 0 (FP64) or 1 (FP32)");
    }
  });
}

amg_status amg_inverse_diagonal(const amg_csr* A, int32_t dtype, void* dinv, void* stream) {
  return guarded([&] {
    if (!A) fail(AMG_ERR_INVALID_ARG, "null matrix");
    validate_csr(*A, "A", 0, static_cast<cudaStream_t>(stream), true);
    check_vec(dinv, "dinv");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int grid = std::max(1, std::min((A->n_rows + 255) / 256, dev_info().max_ctas));
    if (dtype == 0) inv_diag_kernel<double><<<grid, 256, 0, s>>>(A->rowptr, A->col, A->val64, A->n_rows, static_cast<double*>(dinv));
    else if (dtype == 1) inv_diag_kernel<float><<<grid, 256, 0, s>>>(A->rowptr, A->col, A->val32, A->n_rows, static_cast<float*>(dinv));
    else fail(AMG_ERR_INVALID_ARG, "dtype must be 0 (FP64) or 1 (FP32)");
    CK_LAUNCH();
  });
}

amg_status amg_sampled_outer(const amg_csr* A, const double* lam, const double* x, int32_t k,
                             double* grad, void* stream) {
  return guarded([&] {
    if (!A) fail(AMG_ERR_INVALID_ARG, "null matrix");
    validate_csr(*A, "A", 0, static_cast<cudaStream_t>(stream), true);
    check_vec(lam, "lam"); check_vec(x, "x"); check_vec(grad, "grad");
    if (k < 1) fail(AMG_ERR_INVALID_ARG, "k must be >= 1");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int grid = std::max(1, std::min((A->n_rows + 7) / 8, dev_info().max_ctas));
    sampled_outer_kernel<<<grid, 256, 0, s>>>(A->rowptr, A->col, A->n_rows, lam, x, k, grad);
    CK_LAUNCH();
  });
}

amg_status amg_pcg_batch(amg_hierarchy* const* hs, int32_t nsys, int32_t precision,
                         const void* const* b, void* const* x, const int32_t* k, double tol,
                         double atol, int32_t maxiter, int32_t cycle, int32_t cycles_per_level,
                         int32_t* iters_out, double* relres_out, void* stream) {
  return guarded([&] {
    if (nsys < 1 || !hs || !b || !x || !k) fail(AMG_ERR_INVALID_ARG, "empty or null batch");
    if (maxiter < 0) fail(AMG_ERR_INVALID_ARG, "maxiter must be >= 0");
    cycle_char(cycle);
    std::vector<amg_hierarchy*> uniq(hs, hs + nsys);
    for (int i = 0; i < nsys; ++i) {
      if (!hs[i]) fail(AMG_ERR_INVALID_ARG, "system %d: null hierarchy", i);
      check_vec(b[i], "b");
      check_vec(x[i], "x");
      if (k[i] < 1) fail(AMG_ERR_INVALID_ARG, "system %d: k must be >= 1", i);
    }
    std::sort(uniq.begin(), uniq.end());
    if (std::adjacent_find(uniq.begin(), uniq.end()) != uniq.end())
      fail(AMG_ERR_INVALID_ARG, "a hierarchy appears twice in one batch");
    std::vector<std::unique_lock<std::mutex>> locks;
    for (amg_hierarchy* hh : uniq) locks.emplace_back(hh->mu);  // address order: no deadlock
    for (int i = 0; i < nsys; ++i) check_prec_data(hs[i], precision, nullptr);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (precision == AMG_PREC_F64)
      pcg_batch_impl<double, double>(hs, nsys, precision, b, x, k, tol, atol, maxiter, cycle, cycles_per_level, iters_out, relres_out, s);
    else if (precision == AMG_PREC_F32)
      pcg_batch_impl<float, float>(hs, nsys, precision, b, x, k, tol, atol, maxiter, cycle, cycles_per_level, iters_out, relres_out, s);
    else if (precision == AMG_PREC_MIXED)
      pcg_batch_impl<double, float, true>(hs, nsys, precision, b, x, k, tol, atol, maxiter, cycle, cycles_per_level, iters_out, relres_out, s);
    else if (precision == AMG_PREC_MIXED_F64CG)
      pcg_batch_impl<double, float>(hs, nsys, precision, b, x, k, tol, atol, maxiter, cycle, cycles_per_level, iters_out, relres_out, s);
    else
      fail(AMG_ERR_INVALID_ARG, "unknown precision %d", precision);
  });
}

int64_t amg_kernel_launch_count(void) {
  if (cudaDeviceSynchronize() != cudaSuccess) return -1;
  unsigned long long mine = 0;
  if (cudaMemcpyFromSymbol(&mine, g_kernel_count, sizeof(mine)) != cudaSuccess) return -1;
  return int64_t(mine + count_f64() + count_f32() + count_mixed() + count_mixed_cg() + count_runtime() + count_program());
}

const char* amg_last_error(void) { return t_err.c_str(); }

const char* amg_version(void) { return "amg_b200 0.1 (sm_100a)"; }

}  // extern "C"
