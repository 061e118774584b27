// Warp-specialised split-precision GEMM pipeline for one 128 x 128 tile of
// C = A * B^T on the tcgen05 tensor cores (sm_100a).
//
//   warps [0, NPW)        producers: fill operand stages in shared memory
//                         (conversion to tf32 hi/lo pairs by the caller's
//                         functor); thread 0 also issues the MMAs
//   warps [NPW, NPW + 8)  drain: read every accumulation run from TMEM and add
//                         it into fp32 registers; drain warp d covers TMEM lanes
//                         32*(d%4).. (tile rows) and columns 64*(d/4)..
//
// A stage holds BKR real K values (BKR/8 MMA steps of K = 8).  Each MMA step
// (its three products hi*hi + hi*lo + lo*hi) is accumulated in a fresh TMEM
// region (four regions of 128 columns in rotation, all of TMEM) and drained on
// its own: the
// tensor core's fp32 accumulation truncates, with a bias that grows with the
// number of products summed into one accumulator, while the register sums of
// the drain warps round to nearest.  The MMAs run up to three steps ahead of
// the drain, and the producers fill later stages meanwhile.
//
// Synchronisation: smem_free[s] (MMA commit -> producers), acc_full[r] (MMA
// commit -> drain), acc_empty[r] (drain arrivals -> MMA thread).  Every wait is
// bounded; a wait that runs out raises the CTA's abort flag and *err, all
// roles leave their loops through votes on named barriers, and TMEM is
// released on the common exit path.
#pragma once

#include "tc_sm100.cuh"

namespace cuw {
namespace tc {

constexpr long long kWaitCycles = 1ll << 31;  // about one second at 2 GHz

template <int BKR, int NSTAGE, int NPW>
struct Pipe {
  static_assert(BKR % 8 == 0, "a stage is a whole number of K=8 MMA steps");
  static_assert(NPW % 4 == 0, "warp roles must keep the TMEM lane quadrants aligned");
  static constexpr int kRows = 128;                 // A rows = TMEM lanes = B rows (N)
  static constexpr int kTile = kRows * BKR;         // floats of one split operand tile
  static constexpr int kStage = 4 * kTile;          // A hi, A lo, B hi, B lo
  static constexpr int kSteps = BKR / 8;            // accumulation runs per stage
  static constexpr int kProducers = 32 * NPW;
  static constexpr int kDrain = 8;                  // drain warps
  static constexpr int kCols = 128 / (kDrain / 4);  // columns per drain thread
  static constexpr int kThreads = 32 * (NPW + kDrain);
  static constexpr int kRegions = 4;                // TMEM accumulators of 128 columns
  static constexpr size_t kSmem = sizeof(float) * NSTAGE * kStage + 1024 + 512;
};

// Element (row, k) of a split operand tile (see tc_sm100.cuh): float4 index of
// the group of four K values starting at k = 4g.
__device__ __forceinline__ int tile_f4(int row, int g) { return g * 128 + row; }

// Splits four FP64 values into tf32 hi/lo float4s and stores them at float4
// index i of the hi and lo tiles.
__device__ __forceinline__ void store_split4(float* hi, float* lo, int i, double x0, double x1, double x2, double x3) {
  float4 h, l;
  split_tf32(x0, h.x, l.x);
  split_tf32(x1, h.y, l.y);
  split_tf32(x2, h.z, l.z);
  split_tf32(x3, h.w, l.w);
  reinterpret_cast<float4*>(hi)[i] = h;
  reinterpret_cast<float4*>(lo)[i] = l;
}

// Start of the (1024-aligned) stage buffers; free for other use once pipe_run
// has returned.
__device__ __forceinline__ float* pipe_stage_base() {
  extern __shared__ __align__(1024) unsigned char pipe_smem[];
  return reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(pipe_smem) + 1023) & ~uintptr_t(1023));
}

// Complex operands in real form.  A complex K index k becomes the real pair
// (2k, 2k+1); a group of four real K values holds two complex ones.
//   A row:                     (Re a, Im a)
//   B rows 2j and 2j+1 for the complex output column j:
//                              (Re c, -Im c)  and  (Im c, Re c)
// so that sum_k A(m,.) B(2j,.) = Re sum_k a c and B(2j+1,.) gives Im: the
// accumulator holds column j's real and imaginary part side by side.
__device__ __forceinline__ void put_a(float* hi, float* lo, int row, int gi, double2 a0, double2 a1) {
  store_split4(hi, lo, tile_f4(row, gi), a0.x, a0.y, a1.x, a1.y);
}
__device__ __forceinline__ void put_b(float* hi, float* lo, int j, int gi, double2 c0, double2 c1) {
  store_split4(hi, lo, tile_f4(2 * j, gi), c0.x, -c0.y, c1.x, -c1.y);
  store_split4(hi, lo, tile_f4(2 * j + 1, gi), c0.y, c0.x, c1.y, c1.x);
}

// produce(c, t, ahi, alo, bhi, blo): producer thread t in [0, 32*NPW) fills its
// share of stage c's operand tiles.  finish(acc, row, col0): a drain thread
// receives the sums of tile row `row` (0..127), columns col0 .. col0+63.
template <int BKR, int NSTAGE, int NPW, class Produce, class Finish>
__device__ __forceinline__ void pipe_run(int nchunk, Produce& produce, Finish& finish, int* err) {
  using P = Pipe<BKR, NSTAGE, NPW>;
  float* st = pipe_stage_base();
  uint64_t* bfree = reinterpret_cast<uint64_t*>(st + NSTAGE * P::kStage);
  constexpr int NR = P::kRegions;
  uint64_t* bfull = bfree + NSTAGE;
  uint64_t* bempty = bfull + NR;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bempty + NR);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < NSTAGE; ++s) mbar_init(&bfree[s], 1);
    for (int r = 0; r < NR; ++r) {
      mbar_init(&bfull[r], 1);
      mbar_init(&bempty[r], 32 * P::kDrain);
    }
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0) {
    tmem_alloc(tslot, 128 * NR);
    tmem_relinquish();
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tslot;
  constexpr uint32_t idesc = idesc_tf32(128, 128);
  constexpr uint32_t lbo = 128 * 16;  // next group of four K values
  const int nrun = nchunk * P::kSteps;
  if (warp < NPW) {
    int last = -1;  // last accumulation run issued (thread 0)
    for (int c = 0; c < nchunk; ++c) {
      const int s = c % NSTAGE;
      bool bad = false;
      if (c >= NSTAGE) bad = !mbar_wait(&bfree[s], ((c / NSTAGE) - 1) & 1, kWaitCycles);
      if (bar_or(1, P::kProducers, bad || *abort_flag != 0)) {
        if (tid == 0) {
          *abort_flag = 1;
          atomicExch(err, 1);
        }
        break;
      }
      float* ahi = st + s * P::kStage;
      float* alo = ahi + P::kTile;
      float* bhi = alo + P::kTile;
      float* blo = bhi + P::kTile;
      produce(c, tid, ahi, alo, bhi, blo);
      fence_async_smem();
      bar_sync(1, P::kProducers);
      if (tid == 0 && !*abort_flag) {
        const uint32_t sa = smem_u32(ahi), sal = smem_u32(alo), sb = smem_u32(bhi), sbl = smem_u32(blo);
        bool ok = true;
#pragma unroll
        for (int ks = 0; ks < P::kSteps; ++ks) {
          const int t = c * P::kSteps + ks, r = t % NR;
          if (t >= NR && !mbar_wait(&bempty[r], ((t / NR) - 1) & 1, kWaitCycles)) {
            ok = false;
            break;
          }
          fence_after_sync();
          const uint32_t d = tmem + (uint32_t)(r * 128);
          const uint32_t off = ks * 2 * lbo;
          mma_tf32(d, sdesc(sal + off, lbo, 128), sdesc(sb + off, lbo, 128), idesc, 0u);
          mma_tf32(d, sdesc(sa + off, lbo, 128), sdesc(sbl + off, lbo, 128), idesc, 1u);
          mma_tf32(d, sdesc(sa + off, lbo, 128), sdesc(sb + off, lbo, 128), idesc, 1u);
          mma_commit(&bfull[r]);
          last = t;
        }
        if (ok) {
          mma_commit(&bfree[s]);
        } else {
          *abort_flag = 1;
          atomicExch(err, 1);
        }
      }
    }
    if (tid == 0 && *abort_flag && last >= 0) {
      // let the MMAs in flight finish before TMEM is released
      mbar_wait(&bfull[last % NR], (last / NR) & 1, kWaitCycles);
    }
  } else {
    const int q = warp & 3, dw = warp - NPW, col0 = P::kCols * (dw / 4);
    const uint32_t lane_base = ((uint32_t)(32 * q) << 16) + (uint32_t)col0;
    float acc[P::kCols];
#pragma unroll
    for (int j = 0; j < P::kCols; ++j) acc[j] = 0.f;
    bool aborted = false;
    for (int t = 0; t < nrun; ++t) {
      const int r = t % NR;
      const bool ok = mbar_wait(&bfull[r], (t / NR) & 1, kWaitCycles);
      if (bar_or(2, 32 * P::kDrain, !ok || *abort_flag != 0)) {
        aborted = true;
        if (warp == NPW && lane == 0) {
          *abort_flag = 1;
          atomicExch(err, 1);
        }
        break;
      }
      fence_after_sync();
      // two loads in flight per wait (register budget of the drain threads)
#pragma unroll
      for (int j = 0; j < P::kCols / 16; j += 2) {
        uint32_t v[2][16];
        tmem_ld16(tmem + lane_base + (uint32_t)(r * 128 + 16 * j), v[0]);
        tmem_ld16(tmem + lane_base + (uint32_t)(r * 128 + 16 * j + 16), v[1]);
        tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          acc[16 * j + i] += __uint_as_float(v[0][i]);
          acc[16 * j + 16 + i] += __uint_as_float(v[1][i]);
        }
      }
      fence_before_sync();
      mbar_arrive(&bempty[r]);
    }
    if (!aborted) finish(acc, 32 * q + lane, col0);
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (warp == 0) tmem_dealloc(tmem, 128 * NR);
}

}  // namespace tc
}  // namespace cuw
