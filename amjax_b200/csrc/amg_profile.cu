// amg_profile.cu -- diagnostic timing of the fine-level kernels of one mixed-precision
// (reliable-update) PCG step, with the layouts the solve itself uses.
#include <cstring>

#include "amg_runtime.cuh"

using namespace amg;

namespace {

double mpass(const Csr& M, int s) { return double(M.nnz) * (s + 4) + 4.0 * (M.n_rows + 1); }

// Mean device time (microseconds) of `reps` launches, each bracketed by its own events on
// stream s and preceded (outside the events) by a write of `flush_bytes` that evicts L2.
template <class F>
double time_op(F&& launch, int reps, cudaStream_t s, void* flush, size_t flush_bytes) {
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  launch(s);  // warm-up
  double tot = 0.0;
  for (int r = 0; r < reps; ++r) {
    CK(cudaMemsetAsync(flush, r & 1, flush_bytes, s));
    CK(cudaEventRecord(e0, s));
    launch(s);
    CK(cudaEventRecord(e1, s));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    tot += ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return tot / reps * 1e3;
}

}  // namespace

extern "C" amg_status amg_time_pcg_ops(amg_hierarchy* h, int32_t k, int32_t reps, void* stream, int32_t max_ops,
                                       char* names, int32_t name_len, double* us, double* bytes, int32_t* n_ops) {
  return guarded([&] {
    if (!h || !names || !us || !bytes || !n_ops) fail(AMG_ERR_INVALID_ARG, "null argument");
    if (k < 1 || reps < 1 || max_ops < 1 || name_len < 2) fail(AMG_ERR_INVALID_ARG, "bad k, reps or buffer sizes");
    std::lock_guard<std::mutex> lk(h->mu);
    check_prec_data(h, AMG_PREC_MIXED, nullptr);
    if (h->levels.size() < 2) fail(AMG_ERR_UNSUPPORTED, "needs a hierarchy of two or more levels");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Plan* pl = get_plan(h, AMG_PREC_MIXED, k, s);
    const Level& l0 = h->levels[0];
    const Level& l1 = h->levels[1];
    const Csr& A = l0.A;
    const int n = A.n_rows, nc = l1.A.n_rows;
    const double N = n, Nc = nc, K = k;
    float* z = static_cast<float*>(pl->X[0]);
    float* rs = static_cast<float*>(pl->B[0]);
    float* w1 = static_cast<float*>(pl->W1[0]);
    float* w2 = static_cast<float*>(pl->W2[0]);
    float* xs = static_cast<float*>(pl->r_out);
    float* pa = static_cast<float*>(pl->p_out);
    float* pb = static_cast<float*>(pl->q_out);
    const size_t v32 = size_t(n) * k * 4, v64 = size_t(n) * k * 8;
    const size_t flush_bytes = size_t(256) << 20;
    double *x64 = nullptr, *b64 = nullptr;
    void* flush = nullptr;
    CK(cudaMallocAsync(reinterpret_cast<void**>(&x64), v64, s));
    CK(cudaMallocAsync(reinterpret_cast<void**>(&b64), v64, s));
    CK(cudaMallocAsync(&flush, flush_bytes, s));
    struct Row { const char* name; double bytes, us; };
    std::vector<Row> rows;
    try {
      for (void* p : {(void*)z, (void*)rs, (void*)w1, (void*)w2, (void*)xs, (void*)pa, (void*)pb})
        CK(cudaMemsetAsync(p, 0, v32, s));
      CK(cudaMemsetAsync(x64, 0, v64, s));
      CK(cudaMemsetAsync(b64, 0, v64, s));
      for (int l = 1; l < int(h->levels.size()); ++l) {
        const size_t vl = size_t(h->levels[l].A.n_rows) * k * 4;
        CK(cudaMemsetAsync(pl->X[l], 0, vl, s));
        CK(cudaMemsetAsync(pl->B[l], 0, vl, s));
      }
      std::vector<int> ones(size_t(k), 1);
      CK(cudaMemcpyAsync(pl->active(), ones.data(), sizeof(int) * k, cudaMemcpyHostToDevice, s));
      CK(cudaStreamSynchronize(s));
      const Red red = red_of(pl);
      LoopCtl ctl = make_ctl(pl, 1 << 30);
      {
        OpCgQDir<float, float> op{pa, z, pb, pl->beta(), k, nullptr, pl->gamma(), pl->alpha()};
        tune_op(A, op, k, red, s, {pa, z, pb});
        rows.push_back({"cg_direction_pAp", mpass(A, 4) + 4 * K * 3 * N,
                        time_op([&](cudaStream_t c) { run_csr(A, op, k, red, c, {pa, z, pb}); }, reps, s, flush, flush_bytes)});
      }
      {
        OpCgUpdA<float, float> op{};
        op.x = xs; op.r = rs; op.p = pb; op.r_lo = nullptr; op.alpha = pl->alpha(); op.active = pl->active();
        op.ld = k; op.stop = nullptr; op.ctl = ctl; op.reliable = true;
        tune_op(A, op, k, red, s, {xs, rs, pb});
        rows.push_back({"cg_update", mpass(A, 4) + 4 * K * 5 * N,
                        time_op([&](cudaStream_t c) { run_csr(A, op, k, red, c, {xs, rs, pb}); }, reps, s, flush, flush_bytes)});
      }
      const float* dv = l0.template dinv<float>();
      if (l0.post.on() && dv) {
        OpJacobi<float, XS_PLAIN> op{};
        const float om = float(l0.post.omega);
        op.xs = XSource<float, XS_PLAIN>{w1, rs, dv, om, k};
        op.b = rs; op.dinv = dv; op.omega = om; op.out = w2; op.ld = k;
        op.rdot32 = rs; op.gamma = pl->gamma(); op.beta = pl->beta();
        tune_op(A, op, k, red, s, {w1, rs, w2, rs});
        rows.push_back({"post_smooth_with_dot", mpass(A, 4) + 4 * K * 3 * N + 4 * N,
                        time_op([&](cudaStream_t c) { run_csr(A, op, k, red, c, {w1, rs, w2, rs}); }, reps, s, flush, flush_bytes)});
      }
      if (l0.pre.on() && dv) {
        OpResid<float, float, XS_JAC0, true, float, false> op{};
        const float om = float(l0.pre.omega);
        op.xs = XSource<float, XS_JAC0>{nullptr, rs, dv, om, k};
        op.b = rs; op.out = w2; op.out_lo = nullptr; op.ld = k;
        tune_op(A, op, k, Red{}, s, {rs, w2});
        rows.push_back({"residual_presmoothed", mpass(A, 4) + 4 * K * 2 * N + 4 * N,
                        time_op([&](cudaStream_t c) { run_csr(A, op, k, Red{}, c, {rs, w2}); }, reps, s, flush, flush_bytes)});
      }
      {
        OpAxpy<float, XS_ZERO> op{};
        float* bc = static_cast<float*>(pl->B[1]);
        op.x = w2; op.out = bc; op.ld = k;
        tune_op(l0.R, op, k, Red{}, s, {w2, bc});
        rows.push_back({"restriction", mpass(l0.R, 4) + 4 * K * (N + Nc),
                        time_op([&](cudaStream_t c) { run_csr(l0.R, op, k, Red{}, c, {w2, bc}); }, reps, s, flush, flush_bytes)});
      }
      if (l0.pre.on() && dv) {
        OpAxpy<float, XS_JAC0> op{};
        float* xc = static_cast<float*>(pl->X[1]);
        op.base = XSource<float, XS_JAC0>{nullptr, rs, dv, float(l0.pre.omega), k};
        op.x = xc; op.out = w1; op.ld = k;
        tune_op(l0.P, op, k, Red{}, s, {rs, xc, w1});
        rows.push_back({"prolongation_correction", mpass(l0.P, 4) + 4 * K * (2 * N + Nc) + 4 * N,
                        time_op([&](cudaStream_t c) { run_csr(l0.P, op, k, Red{}, c, {rs, xc, w1}); }, reps, s, flush, flush_bytes)});
      }
      {
        OpResid<double, double, XS_PLAIN, false, float, true> op{};
        op.xs = XSource<double, XS_PLAIN>{x64, b64, nullptr, 1.0, k};
        op.b = b64; op.out = nullptr; op.out_lo = rs; op.ld = k; op.stop = nullptr;
        op.ctl = ctl; op.true_rule = true;
        tune_op(A, op, k, red, s, {x64, b64, rs});
        rows.push_back({"true_residual_fp64", mpass(A, 8) + K * (8 * 2 * N + 4 * N),
                        time_op([&](cudaStream_t c) { run_csr(A, op, k, red, c, {x64, b64, rs}); }, reps, s, flush, flush_bytes)});
      }
      {
        OpFold<double, float> op{x64, xs, k, pl->active()};
        rows.push_back({"fold_increment", K * N * (8 + 4) * 2,
                        time_op([&](cudaStream_t c) { run_elem<float>(n, op, k, red, c, {x64, xs}); }, reps, s, flush, flush_bytes)});
      }
    } catch (...) {
      cudaFreeAsync(x64, s);
      cudaFreeAsync(b64, s);
      cudaFreeAsync(flush, s);
      throw;
    }
    CK(cudaFreeAsync(x64, s));
    CK(cudaFreeAsync(b64, s));
    CK(cudaFreeAsync(flush, s));
    CK(cudaStreamSynchronize(s));
    const int m = std::min<int>(max_ops, int(rows.size()));
    for (int i = 0; i < m; ++i) {
      std::strncpy(names + size_t(i) * name_len, rows[size_t(i)].name, size_t(name_len) - 1);
      names[size_t(i) * name_len + name_len - 1] = '\0';
      us[i] = rows[size_t(i)].us;
      bytes[i] = rows[size_t(i)].bytes;
    }
    *n_ops = m;
  });
}
