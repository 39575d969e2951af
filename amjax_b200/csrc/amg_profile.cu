// amg_profile.cu -- diagnostic timing of the fine-level kernels of one mixed-precision
// (reliable-update) PCG step, with the layouts the solve itself uses.
#include <cstring>

#include "amg_runtime.cuh"

using namespace amg;

namespace {

double mpass(const Csr& M, int s) { return double(M.nnz) * (s + 4) + 4.0 * (M.n_rows + 1); }

// Mean device time (microseconds) per launch of `reps` launches issued back to back between
// two CUDA events on stream s, as in a solve (programmatic dependent launch overlaps each
// launch with its predecessor's tail).  Consecutive launches alternate between two
// disjoint buffer sets (launch(set, stream)), so each launch finds its operands evicted
// from L2 by the other set's launch and streams them from DRAM.
template <class F>
double time_op(F&& launch, int reps, cudaStream_t s) {
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  launch(0, s);  // warm-up
  launch(1, s);
  CK(cudaEventRecord(e0, s));
  for (int r = 0; r < reps; ++r) launch(r & 1, s);
  CK(cudaEventRecord(e1, s));
  CK(cudaEventSynchronize(e1));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return double(ms) / reps * 1e3;
}

// One buffer set: the fine level's vectors [n, k] and the coarse level-1 ones [nc, k].
struct Bufs {
  float *z, *rs, *w1, *w2, *xs, *pa, *pb, *bc, *xc;
  double *x64, *b64;
};

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
    const size_t v32 = size_t(n) * k * 4, v64 = size_t(n) * k * 8, c32 = size_t(nc) * k * 4;
    std::vector<void*> owned;
    auto dalloc = [&](size_t bytes) {
      void* p = nullptr;
      CK(cudaMallocAsync(&p, bytes, s));
      owned.push_back(p);
      CK(cudaMemsetAsync(p, 0, bytes, s));
      return p;
    };
    struct Row { const char* name; double bytes, us; };
    std::vector<Row> rows;
    try {
      Bufs set[2];
      for (Bufs& b : set) {
        b.z = static_cast<float*>(dalloc(v32)); b.rs = static_cast<float*>(dalloc(v32));
        b.w1 = static_cast<float*>(dalloc(v32)); b.w2 = static_cast<float*>(dalloc(v32));
        b.xs = static_cast<float*>(dalloc(v32)); b.pa = static_cast<float*>(dalloc(v32));
        b.pb = static_cast<float*>(dalloc(v32)); b.bc = static_cast<float*>(dalloc(c32));
        b.xc = static_cast<float*>(dalloc(c32));
        b.x64 = static_cast<double*>(dalloc(v64)); b.b64 = static_cast<double*>(dalloc(v64));
      }
      int* one = static_cast<int*>(dalloc(sizeof(int) * 2));  // the fold's gate, set to 1
      const int one_h = 1;
      CK(cudaMemcpyAsync(one, &one_h, sizeof(int), cudaMemcpyHostToDevice, s));
      std::vector<int> ones(size_t(k), 1);
      auto all_active = [&]() {
        CK(cudaMemcpyAsync(pl->active(), ones.data(), sizeof(int) * k, cudaMemcpyHostToDevice, s));
        CK(cudaStreamSynchronize(s));
      };
      all_active();
      const Red red = red_of(pl);
      LoopCtl ctl = make_ctl(pl, 1 << 30);
      {
        auto mk = [&](const Bufs& b) {
          return OpCgQDir<float, float>{b.pa, b.z, b.pb, pl->beta(), k, nullptr, pl->gamma(), pl->alpha()};
        };
        tune_op(A, mk(set[0]), k, red, s, {set[0].pa, set[0].z, set[0].pb});
        rows.push_back({"cg_direction_pAp", mpass(A, 4) + 4 * K * 3 * N, time_op([&](int i, cudaStream_t c) {
          run_csr(A, mk(set[i]), k, red, c, {set[i].pa, set[i].z, set[i].pb}); }, reps, s)});
      }
      {
        auto mk = [&](const Bufs& b) {
          OpCgUpdA<float, float> op{};
          op.x = b.xs; op.r = b.rs; op.p = b.pb; op.r_lo = nullptr; op.alpha = pl->alpha(); op.active = pl->active();
          op.ld = k; op.stop = nullptr; op.ctl = ctl; op.reliable = true;
          return op;
        };
        tune_op(A, mk(set[0]), k, red, s, {set[0].xs, set[0].rs, set[0].pb});
        all_active();
        rows.push_back({"cg_update", mpass(A, 4) + 4 * K * 5 * N, time_op([&](int i, cudaStream_t c) {
          run_csr(A, mk(set[i]), k, red, c, {set[i].xs, set[i].rs, set[i].pb}); }, reps, s)});
      }
      const float* dv = l0.template dinv<float>();
      if (l0.post.on() && dv) {
        const float om = float(l0.post.omega);
        auto mk = [&](const Bufs& b) {
          OpJacobi<float, XS_PLAIN> op{};
          op.xs = XSource<float, XS_PLAIN>{b.w1, b.rs, dv, om, k};
          op.b = b.rs; op.dinv = dv; op.omega = om; op.out = b.w2; op.ld = k;
          op.rdot32 = b.rs; op.gamma = pl->gamma(); op.beta = pl->beta();
          return op;
        };
        tune_op(A, mk(set[0]), k, red, s, {set[0].w1, set[0].rs, set[0].w2, set[0].rs});
        rows.push_back({"post_smooth_with_dot", mpass(A, 4) + 4 * K * 3 * N + 4 * N, time_op([&](int i, cudaStream_t c) {
          run_csr(A, mk(set[i]), k, red, c, {set[i].w1, set[i].rs, set[i].w2, set[i].rs}); }, reps, s)});
      }
      if (l0.pre.on() && dv) {
        const float om = float(l0.pre.omega);
        auto mk = [&](const Bufs& b) {
          OpResid<float, float, XS_JAC0, true, float, false> op{};
          op.xs = XSource<float, XS_JAC0>{nullptr, b.rs, dv, om, k};
          op.b = b.rs; op.out = b.w2; op.out_lo = nullptr; op.ld = k;
          return op;
        };
        tune_op(A, mk(set[0]), k, Red{}, s, {set[0].rs, set[0].w2});
        rows.push_back({"residual_presmoothed", mpass(A, 4) + 4 * K * 2 * N + 4 * N, time_op([&](int i, cudaStream_t c) {
          run_csr(A, mk(set[i]), k, Red{}, c, {set[i].rs, set[i].w2}); }, reps, s)});
      }
      {
        auto mk = [&](const Bufs& b) {
          OpAxpy<float, XS_ZERO> op{};
          op.x = b.w2; op.out = b.bc; op.ld = k;
          return op;
        };
        tune_op(l0.R, mk(set[0]), k, Red{}, s, {set[0].w2, set[0].bc});
        rows.push_back({"restriction", mpass(l0.R, 4) + 4 * K * (N + Nc), time_op([&](int i, cudaStream_t c) {
          run_csr(l0.R, mk(set[i]), k, Red{}, c, {set[i].w2, set[i].bc}); }, reps, s)});
      }
      if (l0.pre.on() && dv) {
        const float om = float(l0.pre.omega);
        auto mk = [&](const Bufs& b) {
          OpAxpy<float, XS_JAC0> op{};
          op.base = XSource<float, XS_JAC0>{nullptr, b.rs, dv, om, k};
          op.x = b.xc; op.out = b.w1; op.ld = k;
          return op;
        };
        tune_op(l0.P, mk(set[0]), k, Red{}, s, {set[0].rs, set[0].xc, set[0].w1});
        rows.push_back({"prolongation_correction", mpass(l0.P, 4) + 4 * K * (2 * N + Nc) + 4 * N,
                        time_op([&](int i, cudaStream_t c) {
                          run_csr(l0.P, mk(set[i]), k, Red{}, c, {set[i].rs, set[i].xc, set[i].w1}); }, reps, s)});
      }
      {
        auto mk = [&](const Bufs& b) {
          OpResid<double, double, XS_PLAIN, false, float, true> op{};
          op.xs = XSource<double, XS_PLAIN>{b.x64, b.b64, nullptr, 1.0, k};
          op.b = b.b64; op.out = nullptr; op.out_lo = b.rs; op.ld = k; op.stop = nullptr;
          op.ctl = ctl; op.true_rule = 1;
          return op;
        };
        tune_op(A, mk(set[0]), k, red, s, {set[0].x64, set[0].b64, set[0].rs});
        rows.push_back({"true_residual_fp64", mpass(A, 8) + K * (8 * 2 * N + 4 * N), time_op([&](int i, cudaStream_t c) {
          run_csr(A, mk(set[i]), k, red, c, {set[i].x64, set[i].b64, set[i].rs}); }, reps, s)});
      }
      {
        rows.push_back({"fold_increment", K * N * (8 + 4) * 2, time_op([&](int i, cudaStream_t c) {
          OpFold<double, float> op{set[i].x64, set[i].xs, k, one};
          run_elem<float>(n, op, k, red, c, {set[i].x64, set[i].xs}); }, reps, s)});
      }
    } catch (...) {
      for (void* p : owned) cudaFreeAsync(p, s);
      throw;
    }
    for (void* p : owned) CK(cudaFreeAsync(p, s));
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
