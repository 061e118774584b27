// Autotuner of the launch shapes (no counterpart in the reference, whose FFTW
// plans are chosen by FFTW's own planner at start-up, src/paw_library.f90,
// LIB_FFTW3 2635-2728).  Four parameters of a handle are picked by timing the
// real operations on its own data, on its own stream:
//   - the FFT plan variant of the plane transforms (values per thread and
//     stage, radix order; grids with compiled lengths) together with
//   - the FFT band batch (bands transformed per launch sequence; the work grid
//     is reallocated when a larger batch wins);
//   - on mixed-precision handles, the tile family of the contractions:
//     split-tf32 tcgen05 tiles (128 x 128 x 8) or FP64 DMMA tiles (64 x 64 x
//     4), timed on the projections, the Gram products and the back-projection
//     (the wide tiles waste most of their columns when there are few bands);
//   - the split-K factor of the projections <p|psi> (FP64 DMMA or tcgen05);
//   - the split-K factor of the plane-wave Gram products.
// The choice is kept in a process-wide table keyed by the shape (precision,
// NGL, NBH, NPRO, grid, SM count), so that further handles of the same shape
// take it without timing.  The tile family changes the arithmetic (FP64
// against split tf32), the split-K factors the summation order: results move
// at the mixed path's precision or at rounding level.  A different split-K factor changes the summation
// order of the contractions: results move at rounding level, which is why the
// tuner runs only when asked.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

#include "cuwaves_internal.cuh"

namespace cuw {
namespace {

using Shape = std::array<long long, 8>;
struct Choice {
  int batch;
  int fft_variant;
  int dmma_tiles;
  double split_proj, split_gram;
  double ms[5];
};
std::mutex g_mu;
std::map<Shape, Choice> g_table;

// best of `reps` timed runs after one untimed run (CUDA events on the handle's
// stream)
template <class F>
int time_best(Handle* h, F&& f, int reps, double* best) {
  cudaEvent_t e0, e1;
  CUW_TRY(cudaEventCreate(&e0));
  CUW_TRY(cudaEventCreate(&e1));
  int rc = f();
  *best = 1e30;
  for (int r = 0; r < reps && rc == CUW_OK; ++r) {
    cudaEventRecord(e0, h->stream);
    rc = f();
    cudaEventRecord(e1, h->stream);
    if (cudaEventSynchronize(e1) != cudaSuccess) rc = h->fail(CUW_ERR_CUDA, "autotune: event");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    *best = std::min(*best, (double)ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

int grid_room(Handle* h, int bands) {
  if (bands <= h->grid_bands) return CUW_OK;
  const size_t es = h->mixed() ? sizeof(float2) : sizeof(double2);
  const size_t per_band = (size_t)h->nzp * h->d.nr1 * h->d.nr2 * es;
  CUW_TRY(cudaStreamSynchronize(h->stream));
  void* p = nullptr;
  if (cudaMalloc(&p, per_band * bands) != cudaSuccess) {
    cudaGetLastError();
    return CUW_ERR_NOMEM;  // candidate skipped
  }
  cudaFree(h->g.grid);
  h->g.grid = reinterpret_cast<decltype(h->g.grid)>(p);
  h->grid_bands = bands;
  h->touch();
  return CUW_OK;
}

}  // namespace

int autotune(Handle* h, double* out, int n) {
  if (!h->have_gset || !h->have_v || !h->have_dh || !h->have_do)
    return h->fail(CUW_ERR_STATE, "autotune needs the G set, V, DH and DO");
  const Shape key{h->d.precision, h->d.ngl, h->d.nbh, h->npro, h->d.nr1, h->d.nr2, h->d.nr3, h->nsm};
  Choice c{};
  bool cached = false;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_table.find(key);
    if (it != g_table.end()) {
      c = it->second;
      cached = true;
    }
  }
  Device& g = h->g;
  h->touch();
  if (cached) {
    CUW_RET(grid_room(h, c.batch));
    CUW_RET(fft_set_variant(h, c.fft_variant));
    h->dmma_tiles = c.dmma_tiles != 0;
  } else {
    CUW_RET(eigr_compute(h, g.r0));
    // FFT band batch: the L2 rule's batch and even splits of the bands
    const size_t es = h->mixed() ? sizeof(float2) : sizeof(double2);
    const size_t per_band = (size_t)h->nzp * h->d.nr1 * h->d.nr2 * es;
    std::vector<int> cand{h->batch};
    for (int k = 1; k <= 8; ++k) cand.push_back(ceil_div(h->d.nbh, k));
    std::sort(cand.begin(), cand.end());
    cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
    c.batch = h->batch;
    c.fft_variant = 0;
    c.ms[0] = 1e30;
    const int nv = fft_variants(h);
    for (int v = 0; v < nv; ++v) {
      CUW_RET(fft_set_variant(h, v));
      for (int b : cand) {
        if (per_band * b > ((size_t)256 << 20) && b != h->batch) continue;
        if (grid_room(h, b) != CUW_OK) continue;
        const int keep = h->batch;
        h->batch = b;
        double ms = 0.0;
        CUW_RET(time_best(h, [&] { return fft_vpsi(h, g.psi0, g.hpsi, true); }, 3, &ms));
        if (ms < c.ms[0]) {
          c.ms[0] = ms;
          c.batch = b;
          c.fft_variant = v;
        }
        h->batch = keep;
      }
    }
    h->batch = c.batch;
    CUW_RET(fft_set_variant(h, c.fft_variant));
    h->have_hpsi = false;
    // tile family of the contractions (mixed precision): projections, Gram
    // products of the plane waves and the back-projection into HPSI, at the
    // default split-K factors
    c.dmma_tiles = h->dmma_tiles ? 1 : 0;
    c.ms[3] = c.ms[4] = 0.0;
    if (h->mixed()) {
      const GramPair pq[3] = {{g.psi0, g.psi0}, {g.psim, g.psi0}, {g.psim, g.psim}};
      h->split_proj = h->split_gram = 1.0;
      for (int fam = 0; fam < 2; ++fam) {
        h->dmma_tiles = fam == 1;
        double ms = 0.0;
        CUW_RET(time_best(h, [&] {
          int rc = proj_compute(h, g.psi0, g.pbuf, nullptr, nullptr);
          if (rc == CUW_OK) rc = gram_planewave(h, pq, 3, g.tmat);
          if (rc == CUW_OK) rc = addpro_run(h, ADDPRO_HPSI, g.hproj, g.oproj);
          return rc;
        }, 3, &ms));
        c.ms[3 + fam] = ms;
      }
      c.dmma_tiles = c.ms[4] < c.ms[3] ? 1 : 0;
      h->dmma_tiles = c.dmma_tiles != 0;
      h->have_hpsi = false;
    }
    // split-K factors
    const double muls[] = {0.5, 1.0, 1.5, 2.0, 3.0};
    c.split_proj = c.split_gram = 1.0;
    c.ms[1] = c.ms[2] = 1e30;
    for (double m : muls) {
      h->split_proj = m;
      double ms = 0.0;
      CUW_RET(time_best(h, [&] { return proj_compute(h, g.psi0, g.pbuf, nullptr, nullptr); }, 3, &ms));
      if (ms < c.ms[1]) {
        c.ms[1] = ms;
        c.split_proj = m;
      }
    }
    const GramPair pp[3] = {{g.psi0, g.psi0}, {g.psim, g.psi0}, {g.psim, g.psim}};
    for (double m : muls) {
      h->split_gram = m;
      double ms = 0.0;
      CUW_RET(time_best(h, [&] { return gram_planewave(h, pp, 3, g.tmat); }, 3, &ms));
      if (ms < c.ms[2]) {
        c.ms[2] = ms;
        c.split_gram = m;
      }
    }
    std::lock_guard<std::mutex> lk(g_mu);
    g_table[key] = c;
  }
  h->batch = c.batch;
  h->split_proj = c.split_proj;
  h->split_gram = c.split_gram;
  h->touch();
  const double v[11] = {(double)c.batch, c.split_proj, c.split_gram, c.ms[0], c.ms[1], c.ms[2], cached ? 1.0 : 0.0,
                        (double)c.fft_variant, (double)c.dmma_tiles, c.ms[3], c.ms[4]};
  for (int i = 0; i < n && i < 11; ++i) out[i] = v[i];
  return h->sync();
}

}  // namespace cuw

extern "C" int cuwaves_autotune(cuw_handle* hp, double* out, int n) {
  if (!hp) return CUW_ERR_ARG;
  cuw::Handle* h = reinterpret_cast<cuw::Handle*>(hp);
  return cuw::autotune(h, out, n);
}
