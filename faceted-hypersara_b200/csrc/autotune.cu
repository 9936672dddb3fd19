// Autotuner of the measurement operator's launch shapes.
//
// Two shapes depend on the problem more than on the kernels: how many planes
// one launch of the hand-written real-image FFT passes covers (all planes at
// once fill the GPU best; fewer keep each pass's intermediate -- the half
// spectrum of the forward, the kept image columns of the adjoint -- in L2
// for the pass that reads it next) and how many visibilities one gridding
// work item takes (dense tiles split into more, shorter items balance the
// launch, at the price of partial tiles to sum).  Each candidate is timed on
// the operator itself with CUDA events on its stream, best of 3 after one
// warm-up, and the fastest is kept.  The timed launches write only the
// operator's scratch grids and the solvers' transform buffers, which every
// iteration rewrites before reading.
#include "measop.cuh"

#include <cfloat>

namespace fhs {

namespace {

template <class F>
double best_ms(cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1, F&& run) {
  run();   // warm-up
  double best = DBL_MAX;
  for (int rep = 0; rep < 3; ++rep) {
    FHS_CUDA(cudaEventRecord(e0, s));
    run();
    FHS_CUDA(cudaEventRecord(e1, s));
    FHS_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    FHS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    best = std::min(best, (double)ms);
  }
  return best;
}

struct Events {
  cudaEvent_t a = nullptr, b = nullptr;
  Events() {
    FHS_CUDA(cudaEventCreate(&a));
    FHS_CUDA(cudaEventCreate(&b));
  }
  ~Events() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

}  // namespace

void measop_autotune(MeasOp* op) {
  DeviceGuard g(op->device);
  cudaStream_t s = op->stream;
  measop_enable_r2c(op);
  Events ev;
  op->tune_fft.clear();
  op->tune_grid.clear();
  if (op->own_fft) {
    // the transforms read imgr as their input image and write it back
    FHS_CUDA(cudaMemsetAsync(op->imgr.p, 0, op->imgr.n * sizeof(float), s));
    for (int c : {0, 16, 8, 4}) {
      if (c >= op->L) continue;
      op->fft_chunk = c;
      const double ms = best_ms(s, ev.a, ev.b, [&] {
        solver_fft_forward(op, op->imgr.p, s);
        solver_fft_inverse(op, s);
      });
      op->tune_fft.emplace_back(c, ms);
    }
    auto best = op->tune_fft.front();
    for (const auto& t : op->tune_fft)
      if (t.second < best.second) best = t;
    op->fft_chunk = best.first;
  }
  if (!op->dr && op->Mtot > 0) {
    FHS_CUDA(cudaMemsetAsync(op->zbuf.p, 0, op->zbuf.n * sizeof(float2), s));
    for (int c : {8192, 16384, 32768, 65536}) {
      measop_set_grid_slice(op, c);
      const double ms = best_ms(s, ev.a, ev.b, [&] { launch_grid_plain(op, 0, op->L, op->zbuf.p, s); });
      op->tune_grid.emplace_back(c, ms);
    }
    auto best = op->tune_grid.front();
    for (const auto& t : op->tune_grid)
      if (t.second < best.second) best = t;
    measop_set_grid_slice(op, best.first);
  }
  FHS_CUDA(cudaStreamSynchronize(s));
  op->tuned = true;
  ++op->layout_epoch;
}

}  // namespace fhs
