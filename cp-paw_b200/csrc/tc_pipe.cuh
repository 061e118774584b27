// Warp-specialised split-precision GEMM pipeline for one 128 x 128 tile of
// C = A * B^T on the tcgen05 tensor cores (sm_100a).
//
//   warp 0                MMA issue (one thread) and TMEM allocation
//   warp 1                copies of raw operand data (TMA boxes, element
//                         copies) of later chunks into raw slots
//   warp 2                bulk copies of pre-split B tiles into their stages
//   warps 3..10           converters, two groups of four warps taking chunks
//                         in turn: split the raw A rows into tf32 hi/lo parts
//                         straight into tensor memory (tcgen05.st, lane = row)
//                         (and, without pre-split B, the B tiles)
//   warps 11..26          drain: read every accumulation region from TMEM and
//                         add it into fp32 registers; drain warp w covers TMEM
//                         lanes 32*(w%4).. (tile rows) and 32 of the 128 columns
//
// A chunk holds 16 real K values (two MMA steps of K = 8).  The products of
// CPR consecutive chunks accumulate in one TMEM region (regions of 128
// columns in rotation), which the drain warps then add into fp32 registers
// (round to nearest).  The tensor core's fp32 accumulation truncates toward
// zero: every add into an accumulator loses on average half a unit in the
// last place of the running sum.  Inside a region all small cross products
// (lo*hi, hi*lo) are issued first and the hi*hi products last, so that each
// MMA step adds one truncation at the size of the result (the cross terms are
// 2^-11 smaller); the drain adds back a quarter unit in the last place of the
// drained value per MMA step (the measured mean loss), which removes that bias.  A in tensor memory
// keeps the tensor core's shared-memory reads to the B tiles:
// shared-memory bandwidth bounds a tf32 product of this shape.
//
// TMEM columns: [0, 128 NREG) accumulator regions, [128 NREG + 32 s, +32) A of
// stage place s (hi: 16 columns, lo: 16 columns).  Chunks move in units of G
// through the copies and the conversion (one raw slot and one stage hold G
// chunks, one hand-over per unit).  Two regions and eight stage places keep
// four regions' worth of chunks in flight: the hand-overs between converters,
// MMA thread and drain each take several hundred cycles, whatever they carry.
// The copies run up to NRAW units ahead of the conversion; converted operands
// sit in NSPLIT stages, so copies, conversion, MMAs and drains of different
// units overlap.  Every hand-over is an mbarrier: rawfull[slot] (copies
// landed), rawempty[slot] (converters done with the raw slot), sfull[s]
// (operands converted), sfree[s] (MMAs done with stage s), bfull[r] (run r
// accumulated), bempty[r] (run r drained).  Every wait is bounded; a wait
// that runs out raises the CTA's abort flag and *err, every role then leaves
// its loop (its own waits run out too), copies in flight are waited for, and
// TMEM is released on the common exit path.
#pragma once

#include "tc_sm100.cuh"

namespace cuw {
namespace tc {

constexpr long long kWaitCycles = 1ll << 31;  // about one second at 2 GHz
// mean loss of the truncating TMEM accumulation per MMA step, in units of
// 2^-23 relative to the binade of the accumulated value
constexpr float kLossPerStep = 0.25f * 1.1920928955078125e-7f;

template <int NSPLIT, int NRAW, int RAWB, bool BPRE = true, int CPR = 2, int NREG = 2, int G = 1>
struct Pipe {
  // G chunks travel together through every hand-over but the drain's: one raw
  // slot holds G chunks' raw data, one stage G chunks' converted operands.
  static_assert(NRAW >= 2 && NSPLIT * G >= 2 * CPR && CPR % G == 0, "stage counts");
  // The two converter groups take alternate chunks.  With an even slot count
  // every raw slot belongs to one group, whose waits on it are never more than
  // one phase ahead of the barrier.  With an odd count a group can wait on
  // phase k+2 of a slot while phase k+1 (the other group's chunk, whose copies
  // may land after later ones) is still open, and the parity wait then passes
  // on phase k.  (Stages need no such rule: the MMAs that free them complete
  // in issue order.)
  static_assert(NRAW % 2 == 0, "raw slot count must be even");
  static_assert(128 * NREG + 32 * G * NSPLIT <= 512, "TMEM: accumulator regions and A stages");
  static_assert(RAWB % 1024 == 0, "raw slots keep the 1024-byte alignment of swizzled TMA boxes");
  static constexpr int kRows = 128;                 // A rows = TMEM lanes = B rows (N)
  static constexpr int kBK = 16;                    // real K values per chunk
  static constexpr int kTile = kRows * kBK;         // floats of one split B tile
  static constexpr int kStage = 2 * kTile;          // B hi, B lo
  static constexpr int kSteps = kBK / 8;            // accumulation runs per chunk
  static constexpr int kConvWarps = 8;              // two groups of one warp per TMEM lane quadrant
  static constexpr int kConv = 32 * kConvWarps;     // converter threads
  static constexpr int kGroup = kConv / 2;          // converter threads of one group (one chunk)
  static constexpr bool kBPre = BPRE;               // B tiles arrive split (bulk copy by the copy warp)
  static constexpr int kBBytes = 4 * 2 * 128 * 16;  // one split B stage: hi and lo tiles
  static constexpr int kDrain = 16;                 // drain warps
  static constexpr int kCols = 128 / (kDrain / 4);  // columns per drain thread
  static constexpr int kThreads = 32 * (3 + kConvWarps + kDrain);
  static constexpr int kRegions = NREG;             // TMEM accumulators of 128 columns
  static constexpr int kCPR = CPR;                  // chunks per accumulation region
  static constexpr int kACol = 128 * kRegions;      // first TMEM column of the A stages
  static constexpr int kRawBytes = RAWB;
  static constexpr int kNRaw = NRAW;
  static constexpr int kNSplit = NSPLIT;
  static constexpr int kG = G;                      // chunks per raw slot and per stage
  static constexpr size_t kSplitBytes = sizeof(float) * NSPLIT * G * kStage;
  static constexpr size_t kSmem = kSplitBytes + (size_t)NRAW * G * RAWB + 1024 + 512;
};

// Copies of one chunk issued by one lane of the copy warp into a raw slot:
// contiguous segments as bulk copies (16-byte aligned, multiples of 16 bytes),
// single 16-byte elements (gathers) as cp.async.
struct Copier {
  unsigned char* raw;
  uint64_t* bar;
  uint32_t bytes;
  bool async = false;  // element copies issued (their completion is tracked on bar)
  __device__ __forceinline__ void bulk(int off, const void* src, uint32_t n) {
    if (n) {
      bulk_g2s(raw + off, src, n, bar);
      bytes += n;
    }
  }
  __device__ __forceinline__ void el16(int off, const void* src) {
    cp_async16(raw + off, src, 16);
    async = true;
  }
  __device__ __forceinline__ void el8(int off, const void* src) {
    cp_async8(raw + off, src, 8);
    async = true;
  }
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

// y + sign(y) * h * 2^e for |y| in [2^e, 2^(e+1)): adds back the expected loss
// of truncating fp32 additions, h units of 2^-23 relative to the binade of y
__device__ __forceinline__ float untruncate(float y, float h) {
  const float binade = __uint_as_float(__float_as_uint(y) & 0xFF800000u);  // sign(y) * 2^e (0 for 0)
  return fmaf(binade, h, y);
}

// load(c, lane, cp): lane `lane` of the copy warp issues its copies of chunk
// c through `cp` (offsets within the chunk's raw space, at most RAWB bytes).
// Rows the copies leave out hold stale data: a_row and convert_b mask them.
// a_row(c, raw, row, kh, v): the eight real K values 8kh .. 8kh+7 of A row
// `row` (0..127) of chunk c, from the raw slot.
// load_b(c, lane, cp) (P::kBPre): lane `lane` issues the bulk copy of chunk
// c's split B tiles (kBBytes, hi then lo, in the tile layout) into the stage.
// convert_b(c, raw, ct, bhi, blo) (otherwise): converter thread ct (0..127 of
// the chunk's group) fills its share of chunk c's split B tiles.
// finish(acc, row, col0): a drain thread receives the sums of tile row `row`
// (0..127), columns col0 .. col0+31.
template <class P, class Load, class LoadB, class ARow, class ConvertB, class Finish>
__device__ __forceinline__ void pipe_run(int nchunk, Load& load, LoadB& load_b, ARow& a_row, ConvertB& convert_b,
                                         Finish& finish, int* err) {
  constexpr int NSPLIT = P::kNSplit;
  constexpr int NRAW = P::kNRaw;
  constexpr int RAWB = P::kRawBytes;
  constexpr int CPR = P::kCPR;
  constexpr int G = P::kG;
  float* st = pipe_stage_base();
  unsigned char* raw0 = reinterpret_cast<unsigned char*>(st) + P::kSplitBytes;
  uint64_t* rawfull = reinterpret_cast<uint64_t*>(raw0 + (size_t)NRAW * G * RAWB);
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
      mbar_init(&rawempty[i], P::kGroup);
    }
    for (int i = 0; i < NSPLIT; ++i) {
      mbar_init(&sfull[i], P::kGroup + (P::kBPre ? 1 : 0));
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
  const int nreg = (nchunk + CPR - 1) / CPR;  // accumulation regions
  const int ngrp = (nchunk + G - 1) / G;      // hand-over units of G chunks
  auto raise = [&]() {
    *abort_flag = 1;
    atomicExch(err, 1);
  };
  if (warp == 0) {
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_tf32(128, 128);
      constexpr uint32_t lbo = 128 * 16;  // next group of four K values
      // The issuing warp shares its scheduler with converter and drain warps:
      // every MMA costs only a few instructions (descriptors differ in their
      // start-address field, address / 16, alone).
      const uint64_t dsc0 = sdesc(0, lbo, 128);
      const uint32_t st0 = smem_u32(st) >> 4;
      constexpr uint32_t kStageU = (uint32_t)(sizeof(float) * P::kStage) >> 4;
      constexpr uint32_t kLoU = (uint32_t)(sizeof(float) * P::kTile) >> 4;
      constexpr uint32_t kOffU = (2 * lbo) >> 4;
      int last = -1;  // last region issued
      for (int u = 0; u < nreg && !*abort_flag; ++u) {
        const int r = u % NR, c0 = u * CPR, nc = min(CPR, nchunk - c0);
        const int q0 = c0 / G, nq = (nc + G - 1) / G;  // the region's hand-over units
        bool ok = u < NR || mbar_wait(&bempty[r], ((u / NR) - 1) & 1, kWaitCycles);
        for (int i = 0; i < nq && ok; ++i) ok = mbar_wait(&sfull[(q0 + i) % NSPLIT], ((q0 + i) / NSPLIT) & 1, kWaitCycles);
        if (!ok) {
          raise();
          break;
        }
        fence_after_sync();
        const uint32_t d = tmem + (uint32_t)(r * 128);
        // cross products of every MMA step of the region, then the hi*hi products
#pragma unroll
        for (int pass = 0; pass < 2; ++pass)
#pragma unroll
          for (int i = 0; i < CPR; ++i) {
            if (i >= nc) continue;
            // stage of chunk c0 + i: sub-stage (c0 + i) % G of unit (c0 + i) / G
            const int s = ((c0 + i) / G) % NSPLIT * G + (c0 + i) % G;
            const uint32_t bu = st0 + (uint32_t)s * kStageU;
            const uint32_t ta = tmem + (uint32_t)(P::kACol + 32 * s);
#pragma unroll
            for (int ks = 0; ks < P::kSteps; ++ks) {
              const uint64_t bhi = dsc0 | (uint64_t)(bu + ks * kOffU), blo = dsc0 | (uint64_t)(bu + kLoU + ks * kOffU);
              const uint32_t ahi = ta + 8 * ks, alo = ahi + 16;
              if (pass == 0) {
                mma_tf32_ta(d, alo, bhi, idesc, (i | ks) ? 1u : 0u);
                mma_tf32_ta(d, ahi, blo, idesc, 1u);
              } else {
                mma_tf32_ta(d, ahi, bhi, idesc, 1u);
              }
            }
          }
        mma_commit(&bfull[r]);
        for (int i = 0; i < nq; ++i) mma_commit(&sfree[(q0 + i) % NSPLIT]);
        last = u;
      }
      // let the MMAs in flight finish before TMEM is released
      if (last >= 0) mbar_wait(&bfull[last % NR], (last / NR) & 1, kWaitCycles);
    }
  } else if (warp == 1) {
    // raw A (and unsplit B) data, up to NRAW units ahead of the converters
    int issued = 0;
    for (int q = 0; q < ngrp; ++q) {
      const int slot = q % NRAW;
      bool ok = true;
      if (lane == 0) {
        if (q >= NRAW) ok = mbar_wait(&rawempty[slot], ((q / NRAW) - 1) & 1, kWaitCycles);
        ok = ok && !*abort_flag;
      }
      ok = __shfl_sync(0xffffffffu, ok, 0);  // one decision for the whole warp
      if (!ok) {
        if (lane == 0) raise();
        break;
      }
      uint32_t bytes = 0;
      bool async = false;
#pragma unroll
      for (int j = 0; j < G; ++j) {
        const int c = q * G + j;
        if (c >= nchunk) break;
        Copier cp{raw0 + (size_t)(slot * G + j) * RAWB, &rawfull[slot], 0u};
        load(c, lane, cp);
        bytes += cp.bytes;
        async = async || cp.async;
      }
      // (an arrival per lane with element copies: many arrivals on one
      // mbarrier serialise, so lanes without any skip it)
      if (async) cp_async_mbar_arrive(&rawfull[slot]);
      __syncwarp();
      const uint32_t total = __reduce_add_sync(0xffffffffu, bytes);
      if (lane == 0) mbar_arrive_expect_tx(&rawfull[slot], total);
      issued = q + 1;
    }
    cp_async_wait_all();
    if (*abort_flag && lane == 0) {
      // copies of units nobody consumed complete before the CTA ends
      for (int q = max(0, issued - NRAW); q < issued; ++q) mbar_wait(&rawfull[q % NRAW], (q / NRAW) & 1, kWaitCycles);
    }
  } else if (warp == 2) {
    // split B tiles straight into their stages, once the MMAs are done with them
    if (P::kBPre) {
      int issued = 0;
      for (int q = 0; q < ngrp; ++q) {
        const int s = q % NSPLIT;
        bool ok = true;
        if (lane == 0) {
          if (q >= NSPLIT) ok = mbar_wait(&sfree[s], ((q / NSPLIT) - 1) & 1, kWaitCycles);
          ok = ok && !*abort_flag;
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);  // one decision for the whole warp
        if (!ok) {
          if (lane == 0) raise();
          break;
        }
        uint32_t bytes = 0;
#pragma unroll
        for (int j = 0; j < G; ++j) {
          const int c = q * G + j;
          if (c >= nchunk) break;
          Copier cb{reinterpret_cast<unsigned char*>(st + (s * G + j) * P::kStage), &sfull[s], 0u};
          load_b(c, lane, cb);
          bytes += cb.bytes;
        }
        const uint32_t tb = __reduce_add_sync(0xffffffffu, bytes);
        if (lane == 0) mbar_arrive_expect_tx(&sfull[s], tb);
        issued = q + 1;
      }
      if (*abort_flag && lane == 0)
        for (int q = max(0, issued - NSPLIT); q < issued; ++q) mbar_wait(&sfull[q % NSPLIT], (q / NSPLIT) & 1, kWaitCycles);
    }
  } else if (warp < 3 + P::kConvWarps) {
    // group grp converts units grp, grp + 2, ...; each thread owns one A row
    // (its TMEM lane) and converts both K halves (MMA steps) of it
    const int grp = (warp - 3) >> 2, gt = tid - 96 - grp * P::kGroup;
    const int arow = 32 * (warp & 3) + lane;
    const uint32_t tlane = (uint32_t)(32 * (warp & 3)) << 16;
    for (int q = grp; q < ngrp; q += 2) {
      const int s = q % NSPLIT, slot = q % NRAW;
      bool ok = mbar_wait(&rawfull[slot], (q / NRAW) & 1, kWaitCycles);
      if (ok && q >= NSPLIT) ok = mbar_wait(&sfree[s], ((q / NSPLIT) - 1) & 1, kWaitCycles);
      ok = __all_sync(0xffffffffu, ok && !*abort_flag);  // one decision for the whole warp
      if (!ok) {
        if (lane == 0) raise();
        break;
      }
      fence_after_sync();
#pragma unroll
      for (int j = 0; j < G; ++j) {
        const int c = q * G + j;
        if (c >= nchunk) break;
        const unsigned char* raw = raw0 + (size_t)(slot * G + j) * RAWB;
#pragma unroll
        for (int kh = 0; kh < 2; ++kh) {
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
          const uint32_t ta = tmem + tlane + (uint32_t)(P::kACol + 32 * (s * G + j) + 8 * kh);
          tmem_st8(ta, hi);
          tmem_st8(ta + 16, lo);
        }
        if (!P::kBPre) {
          float* bhi = st + (s * G + j) * P::kStage;
          convert_b(c, raw, gt, bhi, bhi + P::kTile);
        }
      }
      tmem_wait_st();
      if (!P::kBPre) fence_async_smem();
      fence_before_sync();
      mbar_arrive(&sfull[s]);
      mbar_arrive(&rawempty[slot]);
    }
  } else {
    const int q = warp & 3, dw = warp - 3 - P::kConvWarps, col0 = P::kCols * (dw / 4);
    const uint32_t lane_base = ((uint32_t)(32 * q) << 16) + (uint32_t)col0;
    float acc[P::kCols];
#pragma unroll
    for (int j = 0; j < P::kCols; ++j) acc[j] = 0.f;
    bool aborted = false;
    for (int u = 0; u < nreg; ++u) {
      const int r = u % NR;
      const bool got = mbar_wait(&bfull[r], (u / NR) & 1, kWaitCycles);
      const bool ok = __all_sync(0xffffffffu, got && !*abort_flag);  // one decision for the whole warp
      if (!ok) {
        aborted = true;
        if (lane == 0) raise();
        break;
      }
      fence_after_sync();
      // expected truncation loss of the region: a quarter unit in the last
      // place of the result per MMA step (measured on B200 with the ordering
      // above: the uncorrected signed mean error of four-step regions is
      // -8e-8 of |C|)
      const float half_ulps = kLossPerStep * (float)(P::kSteps * min(CPR, nchunk - u * CPR));
#pragma unroll
      for (int j = 0; j < P::kCols / 16; j += 2) {
        uint32_t v[2][16];
        tmem_ld16(tmem + lane_base + (uint32_t)(r * 128 + 16 * j), v[0]);
        tmem_ld16(tmem + lane_base + (uint32_t)(r * 128 + 16 * j + 16), v[1]);
        tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          v[0][i] = __float_as_uint(untruncate(__uint_as_float(v[0][i]), half_ulps));
          v[1][i] = __float_as_uint(untruncate(__uint_as_float(v[1][i]), half_ulps));
        }
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
