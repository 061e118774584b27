// Warp-specialised split-precision GEMM pipeline for one 128 x 128 tile of
// C = A * B^T on the tcgen05 tensor cores (sm_100a).
//
//   warp 0                MMA issue (one thread) and TMEM allocation
//   warp 1                copies: raw operand data of later chunks from global
//                         to shared memory, contiguous segments as bulk copies
//                         (cp.async.bulk), gathered elements as 16-byte cp.async
//   warps 2..9            converters: split the raw data of the current chunk
//                         into tf32 hi/lo parts, A straight into tensor memory
//                         (tcgen05.st, lane = row), B into shared-memory tiles
//   warps 10..25          drain: read every accumulation run from TMEM and add
//                         it into fp32 registers; drain warp w covers TMEM lanes
//                         32*(w%4).. (tile rows) and 32 of the 128 columns
//
// A chunk holds 16 real K values (two MMA steps of K = 8).  Each MMA step (its
// three products lo*hi + hi*lo + hi*hi) is accumulated in a fresh TMEM region
// (three regions of 128 columns in rotation) and drained on its own: the
// tensor core's fp32 accumulation truncates, with a bias that grows with the
// number of products summed into one accumulator, while the register sums of
// the drain warps round to nearest.  A in tensor memory keeps the tensor
// core's shared-memory reads to the B tiles: shared-memory bandwidth bounds a
// tf32 product of this shape.
//
// TMEM columns: [0, 384) accumulator regions, [384 + 32 s, +32) A of stage s
// (hi: 16 columns, lo: 16 columns).  The copies run up to NRAW chunks ahead of
// the conversion; converted operands sit in NSPLIT stages, so copies,
// conversion, MMAs and drains of different chunks overlap.  Every hand-over is
// an mbarrier: rawfull[slot] (copies landed), rawempty[slot] (converters done
// with the raw slot), sfull[s] (operands converted), sfree[s] (MMAs done with
// stage s), bfull[r] (run r accumulated), bempty[r] (run r drained).  Every
// wait is bounded; a wait that runs out raises the CTA's abort flag and *err,
// every role then leaves its loop (its own waits run out too), copies in
// flight are waited for, and TMEM is released on the common exit path.
#pragma once

#include "tc_sm100.cuh"

namespace cuw {
namespace tc {

constexpr long long kWaitCycles = 1ll << 31;  // about one second at 2 GHz

template <int NSPLIT, int NRAW, int RAWB>
struct Pipe {
  static_assert(NRAW >= 2 && NSPLIT >= 2 && NSPLIT <= 4, "stage counts");
  static_assert(RAWB % 1024 == 0, "raw slots keep the 1024-byte alignment of swizzled TMA boxes");
  static constexpr int kRows = 128;                 // A rows = TMEM lanes = B rows (N)
  static constexpr int kBK = 16;                    // real K values per chunk
  static constexpr int kTile = kRows * kBK;         // floats of one split B tile
  static constexpr int kStage = 2 * kTile;          // B hi, B lo
  static constexpr int kSteps = kBK / 8;            // accumulation runs per chunk
  static constexpr int kConvWarps = 8;              // two per TMEM lane quadrant
  static constexpr int kConv = 32 * kConvWarps;     // converter threads
  static constexpr int kDrain = 16;                 // drain warps
  static constexpr int kCols = 128 / (kDrain / 4);  // columns per drain thread
  static constexpr int kThreads = 32 * (2 + kConvWarps + kDrain);
  static constexpr int kRegions = 3;                // TMEM accumulators of 128 columns
  static constexpr int kACol = 128 * kRegions;      // first TMEM column of the A stages
  static constexpr int kRawBytes = RAWB;
  static constexpr size_t kSplitBytes = sizeof(float) * NSPLIT * kStage;
  static constexpr size_t kSmem = kSplitBytes + (size_t)NRAW * RAWB + 1024 + 512;
};

// Copies of one chunk issued by one lane of the copy warp into a raw slot:
// contiguous segments as bulk copies (16-byte aligned, multiples of 16 bytes),
// single 16-byte elements (gathers) as cp.async.
struct Copier {
  unsigned char* raw;
  uint64_t* bar;
  uint32_t bytes;
  __device__ __forceinline__ void bulk(int off, const void* src, uint32_t n) {
    if (n) {
      bulk_g2s(raw + off, src, n, bar);
      bytes += n;
    }
  }
  __device__ __forceinline__ void el16(int off, const void* src) { cp_async16(raw + off, src, 16); }
  __device__ __forceinline__ void el8(int off, const void* src) { cp_async8(raw + off, src, 8); }
  // one TMA box of `box_bytes` (issued by one lane)
  __device__ __forceinline__ void tensor(int off, const CUtensorMap* tm, int x, int y, uint32_t box_bytes) {
    tma_load_2d(raw + off, tm, x, y, bar);
    bytes += box_bytes;
  }
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
// Start of the (1024-aligned) shared buffers: NSPLIT split stages, then NRAW
// raw slots.  The split stages are free for other use once pipe_run returned.
__device__ __forceinline__ float* pipe_stage_base() {
  extern __shared__ __align__(1024) unsigned char pipe_smem[];
  // pointer arithmetic on the shared array (not an integer round trip) keeps
  // the accesses through this pointer in the shared state space
  const uint32_t off = (1024u - (smem_u32(pipe_smem) & 1023u)) & 1023u;
  return reinterpret_cast<float*>(pipe_smem + off);
}

// Complex operands in real form.  A complex K index k becomes the real pair
// (2k, 2k+1).
//   A row:                     (Re a, Im a)
//   B rows 2j and 2j+1 for the complex output column j:
//                              (Re c, -Im c)  and  (Im c, Re c)
// so that sum_k A(m,.) B(2j,.) = Re sum_k a c and B(2j+1,.) gives Im: the
// accumulator holds column j's real and imaginary part side by side.

// load(c, lane, cp): lane `lane` of the copy warp issues its copies of chunk
// c through `cp` (offsets within the raw slot, at most RAWB bytes).  Rows the
// copies leave out hold stale data: a_row and convert_b mask them.
// a_row(c, raw, row, kh, v): the eight real K values 8kh .. 8kh+7 of A row
// `row` (0..127) of chunk c, from the raw slot.
// convert_b(c, raw, ct, bhi, blo): converter thread ct (0..255) fills its share
// of chunk c's split B tiles.
// finish(acc, row, col0): a drain thread receives the sums of tile row `row`
// (0..127), columns col0 .. col0+31.
template <int NSPLIT, int NRAW, int RAWB, class Load, class ARow, class ConvertB, class Finish>
__device__ __forceinline__ void pipe_run(int nchunk, Load& load, ARow& a_row, ConvertB& convert_b, Finish& finish,
                                         int* err) {
  using P = Pipe<NSPLIT, NRAW, RAWB>;
  float* st = pipe_stage_base();
  unsigned char* raw0 = reinterpret_cast<unsigned char*>(st) + P::kSplitBytes;
  uint64_t* rawfull = reinterpret_cast<uint64_t*>(raw0 + (size_t)NRAW * RAWB);
  constexpr int NR = P::kRegions;
  uint64_t* rawempty = rawfull + NRAW;
  uint64_t* sfull = rawempty + NRAW;
  uint64_t* sfree = sfull + NSPLIT;
  uint64_t* bfull = sfree + NSPLIT;
  uint64_t* bempty = bfull + NR;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bempty + NR);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int i = 0; i < NRAW; ++i) {
      mbar_init(&rawfull[i], 1);
      mbar_init(&rawempty[i], P::kConv);
    }
    for (int i = 0; i < NSPLIT; ++i) {
      mbar_init(&sfull[i], P::kConv);
      mbar_init(&sfree[i], 1);
    }
    for (int r = 0; r < NR; ++r) {
      mbar_init(&bfull[r], 1);
      mbar_init(&bempty[r], 32 * P::kDrain);
    }
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0) {
    tmem_alloc(tslot, 512);
    tmem_relinquish();
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tslot;
  const int nrun = nchunk * P::kSteps;
  auto raise = [&]() {
    *abort_flag = 1;
    atomicExch(err, 1);
  };
  if (warp == 0) {
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_tf32(128, 128);
      constexpr uint32_t lbo = 128 * 16;  // next group of four K values
      int last = -1;                      // last accumulation run issued
      for (int c = 0; c < nchunk && !*abort_flag; ++c) {
        const int s = c % NSPLIT;
        if (!mbar_wait(&sfull[s], (c / NSPLIT) & 1, kWaitCycles)) {
          raise();
          break;
        }
        fence_after_sync();
        const uint32_t sb = smem_u32(st + s * P::kStage), sbl = sb + 4 * P::kTile;
        const uint32_t ta = tmem + (uint32_t)(P::kACol + 32 * s);
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
          const uint32_t ahi = ta + 8 * ks, alo = ahi + 16;
          mma_tf32_ta(d, alo, sdesc(sb + off, lbo, 128), idesc, 0u);
          mma_tf32_ta(d, ahi, sdesc(sbl + off, lbo, 128), idesc, 1u);
          mma_tf32_ta(d, ahi, sdesc(sb + off, lbo, 128), idesc, 1u);
          mma_commit(&bfull[r]);
          last = t;
        }
        if (!ok) {
          raise();
          break;
        }
        mma_commit(&sfree[s]);
      }
      // let the MMAs in flight finish before TMEM is released
      if (last >= 0) mbar_wait(&bfull[last % NR], (last / NR) & 1, kWaitCycles);
    }
  } else if (warp == 1) {
    int issued = 0;
    for (int c = 0; c < nchunk; ++c) {
      const int slot = c % NRAW;
      bool ok = true;
      if (lane == 0) {
        if (c >= NRAW) ok = mbar_wait(&rawempty[slot], ((c / NRAW) - 1) & 1, kWaitCycles);
        ok = ok && !*abort_flag;
      }
      ok = __shfl_sync(0xffffffffu, ok, 0);  // one decision for the whole warp
      if (!ok) {
        if (lane == 0) raise();
        break;
      }
      Copier cp{raw0 + (size_t)slot * RAWB, &rawfull[slot], 0u};
      load(c, lane, cp);
      cp_async_mbar_arrive(&rawfull[slot]);
      __syncwarp();
      const uint32_t total = __reduce_add_sync(0xffffffffu, cp.bytes);
      if (lane == 0) mbar_arrive_expect_tx(&rawfull[slot], total);
      issued = c + 1;
    }
    cp_async_wait_all();
    if (*abort_flag && lane == 0) {
      // copies of chunks nobody consumed complete before the CTA ends
      for (int c = max(0, issued - NRAW); c < issued; ++c)
        mbar_wait(&rawfull[c % NRAW], (c / NRAW) & 1, kWaitCycles);
    }
  } else if (warp < 2 + P::kConvWarps) {
    const int ct = tid - 64;
    // this thread's A row (its TMEM lane) and K half (MMA step)
    const int arow = 32 * (warp & 3) + lane, kh = (warp - 2) >> 2;
    const uint32_t tlane = (uint32_t)(32 * (warp & 3)) << 16;
    for (int c = 0; c < nchunk; ++c) {
      const int s = c % NSPLIT, slot = c % NRAW;
      bool ok = mbar_wait(&rawfull[slot], (c / NRAW) & 1, kWaitCycles);
      if (ok && c >= NSPLIT) ok = mbar_wait(&sfree[s], ((c / NSPLIT) - 1) & 1, kWaitCycles);
      ok = __all_sync(0xffffffffu, ok && !*abort_flag);  // one decision for the whole warp
      if (!ok) {
        if (lane == 0) raise();
        break;
      }
      fence_after_sync();
      const unsigned char* raw = raw0 + (size_t)slot * RAWB;
      float v[8];
      a_row(c, raw, arow, kh, v);
      uint32_t hi[8], lo[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        float h, l;
        split_tf32f(v[i], h, l);
        hi[i] = __float_as_uint(h);
        lo[i] = __float_as_uint(l);
      }
      const uint32_t ta = tmem + tlane + (uint32_t)(P::kACol + 32 * s + 8 * kh);
      tmem_st8(ta, hi);
      tmem_st8(ta + 16, lo);
      float* bhi = st + s * P::kStage;
      convert_b(c, raw, ct, bhi, bhi + P::kTile);
      tmem_wait_st();
      fence_async_smem();
      fence_before_sync();
      mbar_arrive(&sfull[s]);
      mbar_arrive(&rawempty[slot]);
    }
  } else {
    const int q = warp & 3, dw = warp - 2 - P::kConvWarps, col0 = P::kCols * (dw / 4);
    const uint32_t lane_base = ((uint32_t)(32 * q) << 16) + (uint32_t)col0;
    float acc[P::kCols];
#pragma unroll
    for (int j = 0; j < P::kCols; ++j) acc[j] = 0.f;
    bool aborted = false;
    for (int t = 0; t < nrun; ++t) {
      const int r = t % NR;
      const bool got = mbar_wait(&bfull[r], (t / NR) & 1, kWaitCycles);
      const bool ok = __all_sync(0xffffffffu, got && !*abort_flag);  // one decision for the whole warp
      if (!ok) {
        aborted = true;
        if (lane == 0) raise();
        break;
      }
      fence_after_sync();
#pragma unroll
      for (int j = 0; j < P::kCols / 16; j += 2) {
        uint32_t v[2][16];
        tmem_ld16(tmem + lane_base + (uint32_t)(r * 128 + 16 * j), v[0]);
        tmem_ld16(tmem + lane_base + (uint32_t)(r * 128 + 16 * j + 16), v[1]);
        tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 16; i += 2) {
          add2(acc[16 * j + i], acc[16 * j + i + 1], v[0][i], v[0][i + 1]);
          add2(acc[16 * j + 16 + i], acc[16 * j + 17 + i], v[1][i], v[1][i + 1]);
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
  if (warp == 0) {
    __syncwarp();
    tmem_dealloc(tmem, 512);
  }
}

}  // namespace tc
}  // namespace cuw
