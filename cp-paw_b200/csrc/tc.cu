// Mixed-precision contractions on the 5th-generation tensor cores (tcgen05).
//
// Every product is a real GEMM C = A * B^T whose operands are split into tf32
// pairs (hi + lo) and multiplied as lo*hi + hi*lo + hi*hi with fp32
// accumulation in tensor memory (three-term split precision), drained after
// every K = 8 step into register sums (tc_pipe.cuh).  Complex products use the
// real form of tc_pipe.cuh.  Operand data is staged raw (FP64 wave functions
// and matrices, the fp32 projector table) with cp.async several chunks ahead,
// then split in shared memory by the converter warps.  Every wait is bounded;
// a wait that runs out sets an error flag and the kernel leaves through its
// cleanup path (TMEM released) instead of hanging.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>

#include "cuwaves_internal.cuh"
#include "tc_pipe.cuh"

namespace cuw {
namespace {

// Real K values per chunk: 16 (two MMA steps of K = 8), i.e. eight complex K.
// The accumulation run stays one MMA step: the tensor core's truncating fp32
// accumulation was measured on B200 at a signed mean error of -3.7e-8 /
// -8.7e-8 / -1.8e-7 of |C| for runs of 8 / 16 / 32 real K, and one step keeps
// the energy bias below 1e-6 Ha/atom.
constexpr int kCK = 8, kNSplit = 8;

// Raw slot layouts (bytes) of the A operands.  TMA boxes land row-major; boxes
// whose rows are read down a column by the converters use the 64- or 128-byte
// swizzle, so that eight consecutive rows hit distinct banks.  The B operands
// arrive already split (k_bsplit) as one bulk copy per chunk.
constexpr int kRawProj = 8192;    // Pf 128 p x 8 g (64-byte rows, 64B swizzle)
constexpr int kRawAddpro = 8192;  // Pf 8 p x 128 g (1 KB rows)
constexpr int kRawGram = 16384;   // X, X(-k): 64 rows of 8 k (128B swizzle), or X: 8 rows of 64 (1 KB)
constexpr int kRawAddx = 32768;   // X, second-half X: 8 k x 128 m (2 KB rows) or 128 m x 8 k (128B swizzle)
constexpr int kRawForce = 16384;  // psi0 8 b x 128 g (2 KB rows)
constexpr int kRawGemm = 36864;   // A, B 128 rows x 16 doubles (144-byte rows, element copies)
// Chunks travel in pairs through the copy and conversion hand-overs (the last
// template argument): each hand-over costs several hundred cycles whatever it
// carries, and pairs took 10-20 % off these kernels on B200 (Si64 and Si128
// projections, back-projection, Gram; more raw slots than listed here gained
// nothing).  Stage and slot counts below count pairs.
using ProjPipe = tc::Pipe<4, 4, kRawProj, true, 2, 2, 2>;
using AddproPipe = tc::Pipe<4, 4, kRawAddpro, true, 2, 2, 2>;
using GramPipe = tc::Pipe<4, 2, kRawGram, true, 2, 2, 2>;
using AddxPipe = tc::Pipe<3, 2, kRawAddx, true, 2, 2, 2>;
using ForcePipe = tc::Pipe<4, 2, kRawForce, true, 2, 2, 2>;
using GemmPipe = tc::Pipe<kNSplit, 2, kRawGemm, false>;
constexpr int kThreads = ProjPipe::kThreads;
constexpr int kNC = ProjPipe::kCols / 2;  // complex output columns per drain thread
constexpr int kBTile = 4096;              // floats of one split B chunk (hi and lo tiles)
static_assert(ProjPipe::kSmem <= 232448 && GramPipe::kSmem <= 232448 && AddxPipe::kSmem <= 232448 &&
                  GemmPipe::kSmem <= 232448 && ForcePipe::kSmem <= 232448 && AddproPipe::kSmem <= 232448,
              "shared memory");
// k_tc_force reuses the stage and raw buffers for a 128 x 64 FP64 tile, rows
// padded to an odd number of doubles so that the column stores of a warp (one
// row per lane) spread over the banks
constexpr int kSvLd = 65;
static_assert(ForcePipe::kSplitBytes + ForcePipe::kNRaw * ForcePipe::kG * kRawForce >= sizeof(double) * (128 * kSvLd + 4 * 128 + 4 * 192),
              "stage area too small");

// offset of 16-byte chunk e of row r in a box with 128-byte (64-byte) rows
// under the TMA 128-byte (64-byte) swizzle: chunk bits 4-6 (4-5) of the
// address are XORed with bits 7-9 (7-8)
__device__ __forceinline__ int sw128(int r, int e) { return r * 128 + ((e ^ (r & 7)) << 4); }
__device__ __forceinline__ int sw64(int r, int e) { return r * 64 + ((e ^ ((r >> 1) & 3)) << 4); }

template <class T>
__device__ __forceinline__ T at(const unsigned char* raw, int byte) {
  return *reinterpret_cast<const T*>(raw + byte);
}
__device__ __forceinline__ double2 dz() { return make_double2(0.0, 0.0); }
__device__ __forceinline__ double2 cj(double2 a) { return make_double2(a.x, -a.y); }

// B functors of the pipelines that do not use them
struct NoLoadB {
  __device__ void operator()(int, int, tc::Copier&) const {}
};
struct NoConvertB {
  __device__ void operator()(int, const unsigned char*, int, float*, float*) const {}
};
// bulk copy of the pre-split B chunk (tile, chunk) of a k_bsplit array
__device__ __forceinline__ void load_bsplit(tc::Copier& cp, int lane, const float* bs, int nchk, int tile, int chunk) {
  if (lane == 0) cp.bulk(0, bs + ((size_t)tile * nchk + chunk) * kBTile, 4 * kBTile);
}

// complex value i of an A row as real K values 2i, 2i+1 (conj: -Im)
template <bool CONJ, class C2>
__device__ __forceinline__ void a_put(float (&v)[8], int i, C2 a) {
  v[2 * i] = (float)a.x;
  v[2 * i + 1] = CONJ ? -(float)a.y : (float)a.y;
}

// ---------------------------------------------------------------------------
// Plain real GEMM C(M,N) = A(M,K) * B(N,K)^T, FP64 in and out, row-major with
// K contiguous: the reference product of the split-precision machinery.
// One CTA computes a 128 x 128 tile over the whole K range.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 1)
    k_tf32x3_gemm(int M, int N, int K, const double* __restrict__ A, const double* __restrict__ B,
                  double* __restrict__ C, int* __restrict__ err) {
  const int m0 = blockIdx.x * 128, n0 = blockIdx.y * 128;
  constexpr int RS = 144;  // raw row stride (16 doubles + 16 bytes)
  auto load = [&](int c, int lane, tc::Copier& cp) {
    const int k0 = c * 16;
    for (int it = lane; it < 2 * 128 * 16; it += 32) {
      const int op = it / (128 * 16), r = (it / 16) % 128, kk = it % 16;
      const int row = (op == 0 ? m0 : n0) + r, lim = op == 0 ? M : N;
      if (row < lim && k0 + kk < K) cp.el8(op * 128 * RS + r * RS + kk * 8, (op == 0 ? A : B) + (size_t)row * K + k0 + kk);
    }
  };
  auto a_row = [&](int c, const unsigned char* raw, int row, int kh, float (&v)[8]) {
    const bool rok = m0 + row < M;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int k = c * 16 + 8 * kh + i;
      v[i] = (rok && k < K) ? (float)at<double>(raw, row * RS + (8 * kh + i) * 8) : 0.f;
    }
  };
  auto convert_b = [&](int c, const unsigned char* raw, int ct, float* bhi, float* blo) {
    for (int it = ct; it < 128 * 4; it += GemmPipe::kGroup) {
      const int r = it % 128, g = it / 128;
      double x[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int k = c * 16 + 4 * g + i;
        x[i] = (n0 + r < N && k < K) ? at<double>(raw, 128 * RS + r * RS + (4 * g + i) * 8) : 0.0;
      }
      tc::store_split4(bhi, blo, tc::tile_f4(r, g), x[0], x[1], x[2], x[3]);
    }
  };
  auto finish = [&](const float (&acc)[GemmPipe::kCols], int row, int col0) {
    if (m0 + row >= M) return;
    double* out = C + (size_t)(m0 + row) * N + n0 + col0;
    const int nc = min(GemmPipe::kCols, N - n0 - col0);
#pragma unroll
    for (int j = 0; j < GemmPipe::kCols; ++j)
      if (j < nc) out[j] = (double)acc[j];
  };
  NoLoadB no_b;
  tc::pipe_run<GemmPipe>((K + 15) / 16, load, no_b, a_row, convert_b, finish, err);
}

// out[i] = scale * sum_z part[z*n + i], summed in FP64 in a fixed order
__global__ void k_tc_reduce(const float2* __restrict__ part, int nz, size_t n, double scale,
                            double2* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double sx = 0.0, sy = 0.0;
    int z = 0;
    for (; z + 8 <= nz; z += 8) {  // eight loads in flight, added in split order
      float2 v[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) v[j] = part[(size_t)(z + j) * n + i];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        sx += (double)v[j].x;
        sy += (double)v[j].y;
      }
    }
    for (; z < nz; ++z) {
      const float2 v = part[(size_t)z * n + i];
      sx += (double)v.x;
      sy += (double)v.y;
    }
    out[i] = make_double2(sx * scale, sy * scale);
  }
}

// Projector table of the mixed path: pf[p*ldg + g] = fp32(PRO(g,p)) with
// PRO(g,p) = Y_lm(g) P_ln(|g|) (-i)^l EIGR(g,a) (WAVES_EXPANDPRO,
// src/paw_waves1.f90:6070-6109) evaluated in FP64, zero for g >= NGL.  The
// single rounding to fp32 is the one the split into tf32 pairs starts from.
__global__ void k_pro_f32(int ngl, int ldg, const int* __restrict__ ipro0, const int* __restrict__ nlmn,
                          const ProDesc* __restrict__ pdesc, const double* __restrict__ ylm,
                          const double* __restrict__ pro, const double2* __restrict__ eigr, float2* __restrict__ pf) {
  // one thread per (g, atom): EIGR(g, a) read once for all projectors of the atom
  const int a = blockIdx.y, p0 = ipro0[a], np = nlmn[a];
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ldg; g += gridDim.x * blockDim.x) {
    if (g >= ngl) {
      for (int k = 0; k < np; ++k) pf[(size_t)(p0 + k) * ldg + g] = make_float2(0.f, 0.f);
      continue;
    }
    const double2 e = eigr[(size_t)g + (size_t)ngl * a];
    for (int k = 0; k < np; ++k) {
      const ProDesc d = pdesc[p0 + k];
      const double s = ylm[(size_t)g + (size_t)ngl * d.lm] * pro[(size_t)g + (size_t)ngl * d.ibare];
      const double2 em = cmul(mipow(d.l), e);
      pf[(size_t)(p0 + k) * ldg + g] = make_float2((float)(s * em.x), (float)(s * em.y));
    }
  }
}

// ---------------------------------------------------------------------------
// <p|psi> partial sums (WAVES_PROJECTIONS, src/paw_waves1.f90:5746-5905):
// part[z][p][b] = sum_{g in split z} conj(PRO(g,p)) psi(g,b)   (float2)
// M = 128 projectors (blockIdx.x), N = 64 bands (blockIdx.y), K = g (blockIdx.z)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 1)
    k_tc_proj(const __grid_constant__ CUtensorMap tm_pf, const float* __restrict__ bpsi, int nchk, int ngl, int nbh,
              int npro, int kchunk, float2* __restrict__ part, int* __restrict__ err) {
  const int m0 = blockIdx.x * 128, b0 = blockIdx.y * 64;
  const int gbeg = blockIdx.z * kchunk, gend = min(ngl, gbeg + kchunk);
  // raw slot: Pf box 128 p x 8 g (64-byte rows, 64B swizzle); zeros past NGL
  // and NPRO.  Chunks never straddle a split boundary (kchunk is a multiple of 8).
  auto load = [&](int c, int lane, tc::Copier& cp) {
    if (lane == 0) cp.tensor(0, &tm_pf, 2 * (gbeg + c * kCK), m0, 8192);
  };
  auto load_b = [&](int c, int lane, tc::Copier& cp) { load_bsplit(cp, lane, bpsi, nchk, blockIdx.y, gbeg / kCK + c); };
  auto a_row = [&](int c, const unsigned char* raw, int r, int kh, float (&v)[8]) {  // conj(Pf) row p
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const float4 x = at<float4>(raw, sw64(r, 2 * kh + i));
      v[4 * i] = x.x, v[4 * i + 1] = -x.y, v[4 * i + 2] = x.z, v[4 * i + 3] = -x.w;
    }
  };
  auto finish = [&](const float (&acc)[ProjPipe::kCols], int row, int col0) {
    const int p = m0 + row;
    if (p >= npro) return;
    float2* out = part + ((size_t)blockIdx.z * npro + p) * nbh;
    const int bb = b0 + col0 / 2;
#pragma unroll
    for (int j = 0; j < kNC; ++j)
      if (bb + j < nbh) out[bb + j] = make_float2(acc[2 * j], acc[2 * j + 1]);
  };
  NoConvertB no_cb;
  const int nchunk = gend > gbeg ? (gend - gbeg + kCK - 1) / kCK : 0;
  tc::pipe_run<ProjPipe>(nchunk, load, load_b, a_row, no_cb, finish, err);
}

// ---------------------------------------------------------------------------
// ADDPRO with the step epilogues (WAVES_ADDPRO, src/paw_waves1.f90:5908-6067,
// and the epilogues of the FP64 k_addpro): 128 g x 32 bands per CTA (band
// tile blockIdx.x, G tile blockIdx.y), the tile columns hold C1 (hproj)
// products for the bands, then C2 (oproj) products.
// ---------------------------------------------------------------------------
template <int MODE>
__global__ void __launch_bounds__(kThreads, 1)
    k_tc_addpro(double2* __restrict__ hpsi, double2* __restrict__ opsi, const double2* __restrict__ psi0,
                double2* __restrict__ psim, const double* __restrict__ mpsi, int ldg, int ngl, int nbh, int npro,
                const __grid_constant__ CUtensorMap tm_pf, const float* __restrict__ bc, int nchk, StepCoef sc,
                int* __restrict__ err) {
  constexpr bool USE_H = (MODE != ADDPRO_OPSI);
  constexpr bool USE_O = (MODE != ADDPRO_HPSI);
  // the band tiles of one G tile are consecutive blocks (blockIdx.x), so the
  // second read of the G tile's projector rows comes from L2
  const int g0 = blockIdx.y * 128, b0 = blockIdx.x * 32;
  // raw slot: Pf box 8 p x 128 g (1 KB rows); zeros past NGL and NPRO.  B:
  // [C1 | C2] of bands b0..b0+31, split (k_bsplit, zero where unused)
  auto load = [&](int c, int lane, tc::Copier& cp) {
    if (lane == 0) cp.tensor(0, &tm_pf, 2 * g0, c * kCK, 8192);
  };
  auto load_b = [&](int c, int lane, tc::Copier& cp) { load_bsplit(cp, lane, bc, nchk, blockIdx.x, c); };
  auto a_row = [&](int c, const unsigned char* raw, int r, int kh, float (&v)[8]) {  // Pf(g, p), K = p
#pragma unroll
    for (int i = 0; i < 4; ++i) a_put<false>(v, i, at<float2>(raw, (4 * kh + i) * 1024 + r * 8));
  };
  auto finish = [&](const float (&acc)[AddproPipe::kCols], int row, int col0) {
    const int g = g0 + row;
    if (g >= ngl) return;
    const double rm = 1.0 / mpsi[g];
    const bool hcol = col0 < 64;  // columns 0..63: C1 (H) products, 64..127: C2 (O)
    const int bl0 = (col0 & 63) / 2;
    // columns in groups of kB whose loads are all issued before any store of
    // the group (the arrays may alias as far as the compiler knows, so a load
    // after a store would wait for it: one memory round trip per group, not
    // two per column)
    constexpr int kB = 2;
#pragma unroll
    for (int j0 = 0; j0 < kNC; j0 += kB) {
      double2 hv[kB], p0v[kB], pm[kB];
      size_t k[kB];
      bool ok[kB];
#pragma unroll
      for (int q = 0; q < kB; ++q) {
        const int b = b0 + bl0 + j0 + q;
        ok[q] = b < nbh;
        k[q] = (size_t)g + (size_t)ldg * (ok[q] ? b : 0);
        if (hcol && USE_H) {
          hv[q] = ok[q] ? hpsi[k[q]] : dz();
          if (MODE == ADDPRO_FUSED) {
            p0v[q] = ok[q] ? psi0[k[q]] : dz();
            pm[q] = ok[q] ? psim[k[q]] : dz();
          }
        } else if (!hcol && USE_O) {
          p0v[q] = ok[q] ? psi0[k[q]] : dz();
        }
      }
#pragma unroll
      for (int q = 0; q < kB; ++q) {
        if (!ok[q]) continue;
        const int j = j0 + q;
        const double2 v = make_double2((double)acc[2 * j], (double)acc[2 * j + 1]);
        if (hcol && USE_H) {
          const double2 h2 = cadd(hv[q], v);
          hpsi[k[q]] = h2;
          if (MODE == ADDPRO_FUSED) {
            double a1 = sc.a1, a2 = sc.a2, a3 = sc.a3 * rm;
            if (sc.fr) {  // cell friction ANNEEVEC(G) (src/paw_waves1.f90:6536-6540)
              const double an = 1.0 + sc.fr[g];
              a1 = 2.0 / an;
              a2 = 1.0 - a1;
              a3 = -sc.dt2 / an * rm;
            }
            psim[k[q]] = make_double2(a1 * p0v[q].x + a2 * pm[q].x + a3 * h2.x, a1 * p0v[q].y + a2 * pm[q].y + a3 * h2.y);
          }
        } else if (!hcol && USE_O) {
          const double s = sc.oscale * rm;
          opsi[k[q]] = make_double2((p0v[q].x + v.x) * s, (p0v[q].y + v.y) * s);
        }
      }
    }
  };
  NoConvertB no_cb;
  tc::pipe_run<AddproPipe>((npro + kCK - 1) / kCK, load, load_b, a_row, no_cb, finish, err);
}

// ---------------------------------------------------------------------------
// Gram products (PLANEWAVE$SCALARPRODUCT, src/paw_fft.f90:2344-2422, for
// WAVES_OVERLAP and WAVES_1COVERLAP): for pair (X, Y)
//   T1(m,n) = sum_k conj(X(k,m)) Y(k,n)
//   T2(m,n) = sum_k X(k,m) Y(-k,n) = sum_k X(-k,m) Y(k,n)   (MINUS; the sphere
//             is closed under k -> -k), else sum_k X(k,m) Y(k,n)
// Tile rows 0..63: conj(X) for T1, rows 64..127: X(-k) for T2, sharing the
// Y columns.  Partials part[z][t][m + nm n] (float2), z = split*npair + pair.
// ---------------------------------------------------------------------------
struct TcGramArgs {
  int npair, nk, nm, kchunk, nchk;
  bool kfast;            // X(k, m) contiguous in k (plane waves); else in m (projections)
  const float* ybs[3];   // Y of each pair, split (k_bsplit)
};
// TMA maps of the pairs: X and X(-k) (plane waves with MINUS)
struct TcGramMaps {
  CUtensorMap x[3], xm[3];
};

template <bool MINUS>
__global__ void __launch_bounds__(kThreads, 1)
    k_tc_gram(TcGramArgs a, const __grid_constant__ TcGramMaps tm, float2* __restrict__ part, int* __restrict__ err) {
  const int pair = blockIdx.z % a.npair, split = blockIdx.z / a.npair;
  const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
  const int kbeg = split * a.kchunk, kend = min(a.nk, kbeg + a.kchunk);
  const bool kfast = a.kfast;
  // raw slot: X at 0, X(-k) at 8K (MINUS).  kfast: boxes of 64 rows (m) of
  // eight k (128-byte rows, 128B swizzle); otherwise 8 rows (k) of 64 m (1 KB
  // rows).  Zeros past NK and NM.
  constexpr int XM = 8192;
  const float* ybs = a.ybs[pair];
  auto load = [&](int c, int lane, tc::Copier& cp) {
    if (lane == 0) {
      const int k0 = kbeg + c * kCK;
      if (kfast) {
        cp.tensor(0, &tm.x[pair], 2 * k0, m0, 8192);
        if (MINUS) cp.tensor(XM, &tm.xm[pair], 2 * k0, m0, 8192);
      } else {
        cp.tensor(0, &tm.x[pair], 2 * m0, k0, 8192);
      }
    }
  };
  auto load_b = [&](int c, int lane, tc::Copier& cp) { load_bsplit(cp, lane, ybs, a.nchk, blockIdx.x, kbeg / kCK + c); };
  auto xoff = [&](int r, int e) { return kfast ? sw128(r, e) : e * 1024 + r * 16; };
  auto a_row = [&](int c, const unsigned char* raw, int r, int kh, float (&v)[8]) {
    // rows 0..63 conj X(k), rows 64..127 X(-k) (MINUS) or X(k)
    const int ml = r & 63;
    const int base = (MINUS && r >= 64) ? XM : 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const double2 x = at<double2>(raw, base + xoff(ml, 4 * kh + i));
      if (r < 64) a_put<true>(v, i, x);
      else a_put<false>(v, i, x);
    }
  };
  auto finish = [&](const float (&acc)[GramPipe::kCols], int row, int col0) {
    const int t = row >> 6, m = m0 + (row & 63);
    if (m >= a.nm) return;
    const size_t mn = (size_t)a.nm * a.nm;
    float2* out = part + ((size_t)blockIdx.z * 2 + t) * mn;
    const int nb = n0 + col0 / 2;
#pragma unroll
    for (int j = 0; j < kNC; ++j)
      if (nb + j < a.nm) out[(size_t)m + (size_t)a.nm * (nb + j)] = make_float2(acc[2 * j], acc[2 * j + 1]);
  };
  NoConvertB no_cb;
  const int nchunk = kend > kbeg ? (kend - kbeg + kCK - 1) / kCK : 0;
  tc::pipe_run<GramPipe>(nchunk, load, load_b, a_row, no_cb, finish, err);
}

// ---------------------------------------------------------------------------
// ADDOPSI / ADDOPROJ (src/paw_waves2.f90:547-615, 687-758):
//   out(m,n) += sum_k X(m,k) L1(k,n) + conj(X(m',k)) L2(k,n),
//   m' = minusg[m] (XMINUS) or m.  K runs over both halves (2 nk).
// ---------------------------------------------------------------------------
struct TcAddXArgs {
  double2* out;
  int nm, nn, nk, nchk;
  size_t som, son;
  bool mfast;       // X(m, k) contiguous in m (plane waves); else in k (projections)
  const float* lbs; // [L1; L2], split (k_bsplit)
};
// TMA maps: X for K < NK, the second-half X (conj X(m') for K >= NK)
struct TcAddXMaps {
  CUtensorMap x, x2;
};

__global__ void __launch_bounds__(kThreads, 1)
    k_tc_addx(TcAddXArgs a, const __grid_constant__ TcAddXMaps tm, int* __restrict__ err) {
  const int m0 = blockIdx.x * 128, n0 = blockIdx.y * 64;
  const int ktot = 2 * a.nk;
  const bool mfast = a.mfast;
  (void)n0;
  // raw slot: X at 0 and the second-half X at 16K: mfast boxes of 8 rows (k)
  // of 128 m (2 KB rows), else 128 rows (m) of eight k (128B swizzle).
  // Second-half boxes start at k = kg0 - NK, negative for a chunk that
  // straddles NK: rows or columns outside the arrays read as zero.
  constexpr int X2 = 16384;
  auto load = [&](int c, int lane, tc::Copier& cp) {
    if (lane == 0) {
      const int kg0 = c * kCK, k2 = kg0 - a.nk;
      if (kg0 < a.nk) {
        if (mfast) cp.tensor(0, &tm.x, 2 * m0, kg0, 16384);
        else cp.tensor(0, &tm.x, 2 * kg0, m0, 16384);
      }
      if (kg0 + kCK > a.nk) {
        if (mfast) cp.tensor(X2, &tm.x2, 2 * m0, k2, 16384);
        else cp.tensor(X2, &tm.x2, 2 * k2, m0, 16384);
      }
    }
  };
  auto load_b = [&](int c, int lane, tc::Copier& cp) { load_bsplit(cp, lane, a.lbs, a.nchk, blockIdx.y, c); };
  auto a_row = [&](int c, const unsigned char* raw, int r, int kh, float (&v)[8]) {  // X(m,k) | conj X(m',k)
    const int kg0 = c * kCK + 4 * kh;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int e = 4 * kh + i;
      const bool first = kg0 + i < a.nk;
      const double2 x = (kg0 + i < ktot) ? at<double2>(raw, (first ? 0 : X2) + (mfast ? e * 2048 + r * 16 : sw128(r, e))) : dz();
      if (first) a_put<false>(v, i, x);
      else a_put<true>(v, i, x);
    }
  };
  auto finish = [&](const float (&acc)[AddxPipe::kCols], int row, int col0) {
    const int m = m0 + row;
    if (m >= a.nm) return;
    const int nb = blockIdx.y * 64 + col0 / 2;
    // four columns' loads before their stores (one memory round trip per group)
#pragma unroll
    for (int j0 = 0; j0 < kNC; j0 += 4) {
      double2 o[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int j = j0 + q;
        o[q] = nb + j < a.nn ? a.out[(size_t)m * a.som + (size_t)(nb + j) * a.son] : dz();
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int j = j0 + q;
        if (nb + j < a.nn)
          a.out[(size_t)m * a.som + (size_t)(nb + j) * a.son] =
              make_double2(o[q].x + (double)acc[2 * j], o[q].y + (double)acc[2 * j + 1]);
      }
    }
  };
  NoConvertB no_cb;
  tc::pipe_run<AddxPipe>((ktot + kCK - 1) / kCK, load, load_b, a_row, no_cb, finish, err);
}

// ---------------------------------------------------------------------------
// Forces (WAVES_DEDPRO + WAVES_PROFORCE, src/paw_waves1.f90:5694-5743,
// 6112-6234): D(g,p) = sum_b psi0(g,b) conj(E(b,p)) on the tensor cores for
// 128 g x 64 projectors, then sv(g,p) = Re[i P (-i)^l EIGR conj(D)] Y_lm in the
// drain warps (into the freed stage buffers) and fpart[tile][p][c] =
// sum_g sv(g,p) G_c(g) by the whole CTA.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 1)
    k_tc_force(const __grid_constant__ CUtensorMap tm_psi, const float* __restrict__ be, int nchk, int ngl, int nbh,
               int npro, const ProDesc* __restrict__ pdesc, const double* __restrict__ ylm,
               const double* __restrict__ pro, const double2* __restrict__ eigr, const double* __restrict__ gx,
               const double* __restrict__ gy, const double* __restrict__ gz, double* __restrict__ fpart,
               int* __restrict__ err) {
  const int g0 = blockIdx.x * 128, p0 = blockIdx.y * 64;
  // raw slot: psi0 box 8 b x 128 g (2 KB rows); zeros past NGL and NBH.  B:
  // conj(E) of projectors p0..p0+63, split (k_bsplit)
  auto load = [&](int c, int lane, tc::Copier& cp) {
    if (lane == 0) cp.tensor(0, &tm_psi, 2 * g0, c * kCK, 16384);
  };
  auto load_b = [&](int c, int lane, tc::Copier& cp) { load_bsplit(cp, lane, be, nchk, blockIdx.y, c); };
  auto a_row = [&](int c, const unsigned char* raw, int r, int kh, float (&v)[8]) {  // psi0(g, b), K = b
#pragma unroll
    for (int i = 0; i < 4; ++i) a_put<false>(v, i, at<double2>(raw, (4 * kh + i) * 2048 + r * 16));
  };
  // [128][kSvLd], over the stage and raw buffers: when a drain thread finishes,
  // every chunk has been converted and multiplied and no copy is in flight
  double* sv = reinterpret_cast<double*>(tc::pipe_stage_base());
  auto finish = [&](const float (&acc)[ForcePipe::kCols], int row, int col0) {
    const int g = g0 + row, pb = col0 / 2;
#pragma unroll
    for (int j = 0; j < kNC; ++j) {
      const int p = p0 + pb + j;
      double v = 0.0;
      if (g < ngl && p < npro) {
        const ProDesc d = pdesc[p];
        const double pr = pro[(size_t)g + (size_t)ngl * d.ibare];
        const double y = ylm[(size_t)g + (size_t)ngl * d.lm];
        const double2 cw = cmul(make_double2(0.0, pr), cmul(mipow(d.l), eigr[(size_t)g + (size_t)ngl * d.iat]));
        v = (cw.x * (double)acc[2 * j] + cw.y * (double)acc[2 * j + 1]) * y;
      }
      sv[row * kSvLd + pb + j] = v;
    }
  };
  NoConvertB no_cb;
  tc::pipe_run<ForcePipe>((nbh + kCK - 1) / kCK, load, load_b, a_row, no_cb, finish, err);
  // pipe_run ended with a CTA barrier: sv is complete (if a wait ran out the
  // error flag is set and the caller discards the result).  G components of the
  // tile, then fpart = sum_g sv(g,p) G_c(g) in four row quarters combined in a
  // fixed order
  double* gsh = sv + 128 * kSvLd;  // [128][4]
  double* qsum = gsh + 4 * 128;    // [4][192]
  for (int i = threadIdx.x; i < 3 * 128; i += blockDim.x) {
    const int c = i / 128, r = i % 128, g = g0 + r;
    gsh[4 * r + c] = g < ngl ? (c == 0 ? gx : (c == 1 ? gy : gz))[g] : 0.0;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 4 * 192; i += blockDim.x) {
    const int qr = i / 192, k = i % 192, pl = k / 3, c = k % 3;
    double s = 0.0;
#pragma unroll 8
    for (int r = 32 * qr; r < 32 * qr + 32; ++r) s += sv[r * kSvLd + pl] * gsh[4 * r + c];
    qsum[i] = s;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < 192; k += blockDim.x) {
    const int pl = k / 3, c = k % 3, p = p0 + pl;
    if (p < npro) fpart[((size_t)blockIdx.x * npro + p) * 3 + c] = ((qsum[k] + qsum[192 + k]) + qsum[384 + k]) + qsum[576 + k];
  }
}

// ---------------------------------------------------------------------------
// Forces, persistent form for NBH <= 64 (an even number of K chunks, at most
// eight): the same D(g,p) = sum_b psi0(g,b) conj(E(b,p)) and force sums as
// k_tc_force, but one CTA per SM walks a contiguous run of (g tile, projector
// tile) items.  The split psi0 rows of a g tile (all of K: 8 chunks x 32 TMEM
// columns) stay in tensor memory for every projector tile of that g tile, so
// only the pre-split conj(E) chunks stream.  Each item accumulates in one of
// two TMEM regions (two chunks at a time: cross terms, then hi*hi); the drain
// warps copy the region to registers and release it at once, so the MMAs of
// the next items run while the drains form sv(g,p) = Re[i pf(g,p) conj(D)]
// from the FP32 projector table and the G-weighted column sums of this item.
//   warp 0   TMEM allocation, MMA issue (one thread)
//   warp 1   TMA copies of raw psi0 chunks (two raw slots, one per converter group)
//   warp 2   bulk copies of the split conj(E) chunks into kFNS stages
//   3..10    converters (two groups of four warps, alternate chunks of a g tile)
//   11..26   drains and the per-item force epilogue
// Barriers: rawfull/rawempty (raw psi0 slots), afull[c] (A chunk c of the
// current g tile in TMEM), afree (MMAs of the last item of a g tile done),
// sfull/sfree (B stages), bfull/bempty (accumulation regions, one item each).
// Every wait is bounded; the drain group decides to leave by one vote per item
// (a reduction barrier all 16 drain warps reach), so none of them is left at a
// barrier.  The hand-over protocol is model-checked on the CPU
// (tests/test_pipe_protocol.py).
// ---------------------------------------------------------------------------
constexpr int kFNS = 6;        // B stages (16 KB each)
constexpr int kFMaxChunks = 8; // K chunks of a resident A tile (TMEM columns 256..511)
constexpr size_t kForcePSmem = (size_t)kFNS * 16384 + 2 * 16384 +
                               sizeof(double) * (128 * kSvLd + 4 * 128 + 4 * 192) + 1024 + 512;
static_assert(kForcePSmem <= 232448, "shared memory");

__global__ void __launch_bounds__(kThreads, 1)
    k_tc_force_p(const __grid_constant__ CUtensorMap tm_psi, const float* __restrict__ be, int nchk, int ngl, int npro,
                 int ldg, int tn, int nitems, const float2* __restrict__ pf, const double* __restrict__ gx,
                 const double* __restrict__ gy, const double* __restrict__ gz, double* __restrict__ fpart,
                 int* __restrict__ err) {
  using namespace tc;
  float* st = pipe_stage_base();
  unsigned char* raw0 = reinterpret_cast<unsigned char*>(st) + (size_t)kFNS * 16384;
  double* sv = reinterpret_cast<double*>(raw0 + 2 * 16384);  // [128][kSvLd]
  double* gsh = sv + 128 * kSvLd;                            // [128][4]
  double* qsum = gsh + 4 * 128;                              // [4][192]
  uint64_t* rawfull = reinterpret_cast<uint64_t*>(qsum + 4 * 192);
  uint64_t* rawempty = rawfull + 2;
  uint64_t* sfull = rawempty + 2;
  uint64_t* sfree = sfull + kFNS;
  uint64_t* bfull = sfree + kFNS;
  uint64_t* bempty = bfull + 2;
  uint64_t* afull = bempty + 2;
  uint64_t* afree = afull + kFMaxChunks;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(afree + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long G = gridDim.x;
  const int w0 = (int)((long long)blockIdx.x * nitems / G), w1 = (int)((long long)(blockIdx.x + 1) * nitems / G);
  const int m_first = w0 / tn;
  const int nm = w1 > w0 ? (w1 - 1) / tn - m_first + 1 : 0;  // g tiles of this CTA
  if (tid == 0) {
    for (int i = 0; i < 2; ++i) {
      mbar_init(&rawfull[i], 1);
      mbar_init(&rawempty[i], 128);
      mbar_init(&bfull[i], 1);
      mbar_init(&bempty[i], 512);
    }
    for (int i = 0; i < kFNS; ++i) {
      mbar_init(&sfull[i], 1);
      mbar_init(&sfree[i], 1);
    }
    for (int c = 0; c < kFMaxChunks; ++c) mbar_init(&afull[c], 128);
    mbar_init(afree, 1);
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
  auto raise = [&]() {
    *abort_flag = 1;
    atomicExch(err, 1);
  };
  if (warp == 0) {
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_tf32(128, 128);
      constexpr uint32_t lbo = 128 * 16;
      const uint64_t dsc0 = sdesc(0, lbo, 128);
      const uint32_t st0 = smem_u32(st) >> 4;
      constexpr uint32_t kStageU = 16384u >> 4, kLoU = 8192u >> 4, kOffU = (2 * lbo) >> 4;
      int it = 0, j = 0;
      bool ok = true, pending = false;  // pending: MMAs issued since the last bfull commit
      for (int w = w0; w < w1 && ok && !*abort_flag; ++w, ++it) {
        const int im = w / tn - m_first, r = it & 1;
        const bool first_of_m = (w == w0) || (w % tn == 0), last_of_m = (w == w1 - 1) || ((w + 1) % tn == 0);
        if (it >= 2) ok = mbar_wait(&bempty[r], ((it >> 1) - 1) & 1, kWaitCycles);
        const uint32_t d = tmem + (uint32_t)(r * 128);
        for (int rr = 0; rr < nchk / 2 && ok; ++rr, j += 2) {
          for (int i = 0; i < 2 && ok; ++i) {
            if (first_of_m) ok = mbar_wait(&afull[2 * rr + i], im & 1, kWaitCycles);
            if (ok) ok = mbar_wait(&sfull[(j + i) % kFNS], ((j + i) / kFNS) & 1, kWaitCycles);
          }
          if (!ok) break;
          fence_after_sync();
#pragma unroll
          for (int pass = 0; pass < 2; ++pass)
#pragma unroll
            for (int i = 0; i < 2; ++i) {
              const int c = 2 * rr + i, s = (j + i) % kFNS;
              const uint32_t bu = st0 + (uint32_t)s * kStageU;
              const uint32_t ta = tmem + (uint32_t)(256 + 32 * c);
#pragma unroll
              for (int ks = 0; ks < 2; ++ks) {
                const uint64_t bhi = dsc0 | (uint64_t)(bu + ks * kOffU), blo = dsc0 | (uint64_t)(bu + kLoU + ks * kOffU);
                const uint32_t ahi = ta + 8 * ks, alo = ahi + 16;
                if (pass == 0) {
                  mma_tf32_ta(d, alo, bhi, idesc, (rr | i | ks) ? 1u : 0u);
                  mma_tf32_ta(d, ahi, blo, idesc, 1u);
                } else {
                  mma_tf32_ta(d, ahi, bhi, idesc, 1u);
                }
              }
            }
          mma_commit(&sfree[j % kFNS]);
          mma_commit(&sfree[(j + 1) % kFNS]);
          pending = true;
        }
        if (!ok) break;
        mma_commit(&bfull[r]);
        pending = false;
        if (last_of_m) mma_commit(afree);
      }
      if (!ok) raise();
      // the MMAs in flight finish before TMEM is released (after an abort in
      // the middle of an item, through one more commit on its region)
      if (pending) {
        mma_commit(&bfull[it & 1]);
        mbar_wait(&bfull[it & 1], (it >> 1) & 1, kWaitCycles);
      } else if (it > 0) {
        mbar_wait(&bfull[(it - 1) & 1], ((it - 1) >> 1) & 1, kWaitCycles);
      }
    }
  } else if (warp == 1) {
    // raw psi0 chunks: chunk c of the im-th g tile goes to slot c % 2 (the slot
    // of converter group c % 2)
    int issued = 0;
    const int total = nm * nchk;
    for (int q = 0; q < total; ++q) {
      const int slot = q & 1, m = m_first + q / nchk, c = q % nchk;
      bool ok = true;
      if (lane == 0) {
        if (q >= 2) ok = mbar_wait(&rawempty[slot], ((q >> 1) - 1) & 1, kWaitCycles);
        ok = ok && !*abort_flag;
      }
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) {
        if (lane == 0) raise();
        break;
      }
      if (lane == 0) {
        tma_load_2d(raw0 + slot * 16384, &tm_psi, 2 * 128 * m, c * kCK, &rawfull[slot]);
        mbar_arrive_expect_tx(&rawfull[slot], 16384);
      }
      issued = q + 1;
    }
    if (*abort_flag && lane == 0)
      for (int q = max(0, issued - 2); q < issued; ++q) mbar_wait(&rawfull[q & 1], (q >> 1) & 1, kWaitCycles);
  } else if (warp == 2) {
    int issued = 0;
    int j = 0;
    for (int w = w0; w < w1; ++w) {
      const int n = w % tn;
      bool ok = true;
      for (int c = 0; c < nchk; ++c, ++j) {
        const int s = j % kFNS;
        if (lane == 0) {
          if (j >= kFNS) ok = mbar_wait(&sfree[s], ((j / kFNS) - 1) & 1, kWaitCycles);
          ok = ok && !*abort_flag;
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) break;
        if (lane == 0) {
          bulk_g2s(st + (size_t)s * 4096, be + ((size_t)n * nchk + c) * kBTile, 16384, &sfull[s]);
          mbar_arrive_expect_tx(&sfull[s], 16384);
        }
        issued = j + 1;
      }
      if (!ok) {
        if (lane == 0) raise();
        break;
      }
    }
    if (*abort_flag && lane == 0)
      for (int q = max(0, issued - kFNS); q < issued; ++q) mbar_wait(&sfull[q % kFNS], (q / kFNS) & 1, kWaitCycles);
  } else if (warp < 11) {
    // converters: group grp owns chunks grp, grp + 2, ... of every g tile
    const int grp = (warp - 3) >> 2;
    const int arow = 32 * (warp & 3) + lane;
    const uint32_t tlane = (uint32_t)(32 * (warp & 3)) << 16;
    bool ok = true;
    for (int im = 0; im < nm && ok; ++im) {
      for (int c = grp; c < nchk; c += 2) {
        const int q = im * nchk + c, slot = q & 1;
        bool got = mbar_wait(&rawfull[slot], (q >> 1) & 1, kWaitCycles);
        if (got && c == grp && im >= 1) got = mbar_wait(afree, (im - 1) & 1, kWaitCycles);
        ok = __all_sync(0xffffffffu, got && !*abort_flag);
        if (!ok) {
          if (lane == 0) raise();
          break;
        }
        const unsigned char* raw = raw0 + slot * 16384;
#pragma unroll
        for (int kh = 0; kh < 2; ++kh) {
          uint32_t hi[8], lo[8];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const double2 x = at<double2>(raw, (4 * kh + i) * 2048 + arow * 16);
            float h0, l0, h1, l1;
            split_tf32f((float)x.x, h0, l0);
            split_tf32f((float)x.y, h1, l1);
            hi[2 * i] = __float_as_uint(h0), lo[2 * i] = __float_as_uint(l0);
            hi[2 * i + 1] = __float_as_uint(h1), lo[2 * i + 1] = __float_as_uint(l1);
          }
          const uint32_t ta = tmem + tlane + (uint32_t)(256 + 32 * c + 8 * kh);
          tmem_st8(ta, hi);
          tmem_st8(ta + 16, lo);
        }
        tmem_wait_st();
        fence_before_sync();
        mbar_arrive(&afull[c]);
        mbar_arrive(&rawempty[slot]);
      }
    }
  } else {
    const int q = warp & 3, dw = warp - 11, col0 = 32 * (dw / 4), dt = tid - 11 * 32;
    const uint32_t lane_base = ((uint32_t)(32 * q) << 16) + (uint32_t)col0;
    const int row = 32 * q + lane, pb = col0 / 2;
    // expected truncation loss: a quarter unit in the last place per K=8 step
    const float half_ulps = kLossPerStep * (float)(2 * nchk);
    int it = 0;
    for (int w = w0; w < w1; ++w, ++it) {
      const int m = w / tn, n = w % tn, g = m * 128 + row, r = it & 1;
      bool got = mbar_wait(&bfull[r], (it >> 1) & 1, kWaitCycles);
      got = __all_sync(0xffffffffu, got && !*abort_flag);
      float acc[32];
      if (got) {
        fence_after_sync();
        uint32_t v[2][16];
        tmem_ld16(tmem + lane_base + (uint32_t)(r * 128), v[0]);
        tmem_ld16(tmem + lane_base + (uint32_t)(r * 128 + 16), v[1]);
        tmem_wait_ld();
        fence_before_sync();
        mbar_arrive(&bempty[r]);  // the region is free for the item after next
#pragma unroll
        for (int k = 0; k < 32; ++k) acc[k] = untruncate(__uint_as_float(v[k >> 4][k & 15]), half_ulps);
      }
      // one decision for the whole drain group, reached by all 16 warps
      if (bar_or(1, 512, !got)) {
        if (dt == 0) raise();
        break;
      }
      // G components of the item's g tile ([row][4]: the three components of
      // a row in different banks); sv(g,p) = Re[i pf(g,p) conj(D)], with the
      // sixteen table loads of a thread in flight together
      if (dt < 128) {
        const int gg = m * 128 + dt;
        const bool in = gg < ngl;
        gsh[4 * dt] = in ? gx[gg] : 0.0;
        gsh[4 * dt + 1] = in ? gy[gg] : 0.0;
        gsh[4 * dt + 2] = in ? gz[gg] : 0.0;
      }
      float2 pfv[16];
#pragma unroll
      for (int jx = 0; jx < 16; ++jx) {
        const int p = n * 64 + pb + jx;
        pfv[jx] = (g < ngl && p < npro) ? __ldg(&pf[(size_t)p * ldg + g]) : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int jx = 0; jx < 16; ++jx)
        sv[row * kSvLd + pb + jx] = -(double)pfv[jx].y * (double)acc[2 * jx] + (double)pfv[jx].x * (double)acc[2 * jx + 1];
      bar_sync(1, 512);
      // fpart[m][p][c] = sum_g sv(g,p) G_c(g): four row quarters, fixed order
      for (int t = dt; t < 4 * 192; t += 512) {
        const int qr = t / 192, k = t % 192, pl = k / 3, c = k % 3;
        double sum = 0.0;
#pragma unroll 8
        for (int rw = 32 * qr; rw < 32 * qr + 32; ++rw) sum += sv[rw * kSvLd + pl] * gsh[4 * rw + c];
        qsum[t] = sum;
      }
      bar_sync(1, 512);
      if (dt < 192) {
        const int pl = dt / 3, c = dt % 3, p = n * 64 + pl;
        if (p < npro)
          fpart[((size_t)m * npro + p) * 3 + c] = ((qsum[dt] + qsum[192 + dt]) + qsum[384 + dt]) + qsum[576 + dt];
      }
      bar_sync(1, 512);
    }
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (warp == 0) {
    __syncwarp();
    tmem_dealloc(tmem, 512);
  }
}

// Source of a split B operand: value(row, h) of complex output column `row`
// at complex K index h
//   kind 0: x[h + ld*row]            kind 1: x[row + ld*h]
//   kind 2: conj x[h + ld*row]       kind 3: h < nk1 ? x[h + ld*row] : x2[h - nk1 + ld*row]
//   kind 4: tile of 32 rows of x then 32 rows of x2, each as kind 1 (null: zero)
struct BSplitSrc {
  int kind;
  const double2* x;
  const double2* x2;
  long long ld;
  int nrow, nk, nk1;
};

// B operand in real form, split into tf32 hi/lo tiles in the shared-memory
// layout of the pipeline (tc_pipe.cuh): block (tile, chunk) of 4096 floats =
// hi then lo, element (R, k) of 128 real rows x 16 real K at
// (k/4)*512 + R*4 + k%4; real rows 2j / 2j+1 of complex column j are
// (Re c, -Im c) / (Im c, Re c).  Zero outside the source.
__global__ void k_bsplit(BSplitSrc b, int nchk, float* __restrict__ out) {
  const int tile = blockIdx.y, c = blockIdx.x;
  float* o = out + ((size_t)tile * nchk + c) * kBTile;
  for (int it = threadIdx.x; it < 512; it += blockDim.x) {
    const int R = it & 127, kg = it >> 7, j = R >> 1;
    double2 v[2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int h = c * kCK + 2 * kg + e;
      v[e] = dz();
      if (h >= b.nk) continue;
      if (b.kind == 4) {
        const double2* src = j < 32 ? b.x : b.x2;
        const int row = 32 * tile + (j & 31);
        if (src && row < b.nrow) v[e] = src[(size_t)row + (size_t)b.ld * h];
      } else {
        const int row = 64 * tile + j;
        if (row >= b.nrow) continue;
        if (b.kind == 0) v[e] = b.x[(size_t)h + (size_t)b.ld * row];
        else if (b.kind == 1) v[e] = b.x[(size_t)row + (size_t)b.ld * h];
        else if (b.kind == 2) v[e] = cj(b.x[(size_t)h + (size_t)b.ld * row]);
        else v[e] = h < b.nk1 ? b.x[(size_t)h + (size_t)b.ld * row] : b.x2[(size_t)(h - b.nk1) + (size_t)b.ld * row];
      }
    }
    double w[4];
    if ((R & 1) == 0) w[0] = v[0].x, w[1] = -v[0].y, w[2] = v[1].x, w[3] = -v[1].y;
    else w[0] = v[0].y, w[1] = v[0].x, w[2] = v[1].y, w[3] = v[1].x;
    tc::store_split4(o, o + 2048, kg * 128 + R, w[0], w[1], w[2], w[3]);
  }
}

// dst(g, b) = src(-g, b) for g < NGL, 0 in the padding (ld = ldg)
__global__ void k_minus_copy(const double2* __restrict__ src, double2* __restrict__ dst,
                             const int* __restrict__ minusg, int ngl, int ldg, int nbh) {
  const size_t n = (size_t)ldg * nbh;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int g = (int)(i % ldg);
    dst[i] = g < ngl ? src[(size_t)minusg[g] + (i - g)] : dz();
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// host side of the split-precision contractions
// ---------------------------------------------------------------------------
static int* tc_err(Handle* h) { return h->g.ostatus + 12; }

// number of K splits so that tiles * splits fills the GPU once (one CTA per SM)
static int tc_splits(Handle* h, int tiles, int nk, double mul) {
  // at most mul waves of one CTA per SM (rounded down: a CTA past a whole
  // wave would cost a wave of its own)
  const int want = std::max(1, (int)std::floor(h->nsm * mul / std::max(1, tiles)));
  return std::max(1, std::min(want, ceil_div(nk, 4 * kCK)));
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library links the runtime only)
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiled encode_tiled() {
  static EncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
    cudaGetLastError();
  });
  return fn;
}

// 2-D map of `rows` rows of `inner` real elements (FP64 or fp32), rows `ld`
// elements apart, box bx x by; elements outside read as zero
static int make_map(Handle* h, CUtensorMap* m, const void* base, bool f64, long long inner, long long rows,
                    long long ld, int bx, int by, CUtensorMapSwizzle sw) {
  const EncodeTiled fn = encode_tiled();
  if (!fn) return h->fail(CUW_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  const long long es = f64 ? 8 : 4;
  const cuuint64_t dims[2] = {(cuuint64_t)std::max(1ll, inner), (cuuint64_t)std::max(1ll, rows)};
  const cuuint64_t strides[1] = {(cuuint64_t)(ld * es)};
  const cuuint32_t box[2] = {(cuuint32_t)bx, (cuuint32_t)by};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(m, f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                        const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return h->fail(CUW_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
  return CUW_OK;
}
// complex (ld, cols) array of FP64 pairs: rows = columns of the array
static int map_c(Handle* h, CUtensorMap* m, const double2* base, long long n, long long cols, long long ld, int bx,
                 int by, CUtensorMapSwizzle sw) {
  return make_map(h, m, base, true, 2 * n, cols, 2 * ld, bx, by, sw);
}

int tc_setup(Handle* h) {
  CUW_TRY(smem_allow((const void*)k_tc_proj, (int)ProjPipe::kSmem));
  CUW_TRY(smem_allow((const void*)k_tc_addpro<ADDPRO_HPSI>, (int)AddproPipe::kSmem));
  CUW_TRY(smem_allow((const void*)k_tc_addpro<ADDPRO_OPSI>, (int)AddproPipe::kSmem));
  CUW_TRY(smem_allow((const void*)k_tc_addpro<ADDPRO_FUSED>, (int)AddproPipe::kSmem));
  CUW_TRY(smem_allow((const void*)k_tc_gram<true>, (int)GramPipe::kSmem));
  CUW_TRY(smem_allow((const void*)k_tc_gram<false>, (int)GramPipe::kSmem));
  CUW_TRY(smem_allow((const void*)k_tc_addx, (int)AddxPipe::kSmem));
  CUW_TRY(smem_allow((const void*)k_tc_force, (int)ForcePipe::kSmem));
  CUW_TRY(smem_allow((const void*)k_tc_force_p, (int)kForcePSmem));
  if (!encode_tiled()) return h->fail(CUW_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  auto alloc = [&](void** p, size_t bytes) -> int {
    if (*p) return CUW_OK;
    if (cudaMalloc(p, bytes) != cudaSuccess) {
      cudaGetLastError();
      *p = nullptr;
      return h->fail(CUW_ERR_NOMEM, "cudaMalloc of mixed-path scratch failed");
    }
    CUW_TRY(cudaMemsetAsync(*p, 0, bytes, h->stream));
    return CUW_OK;
  };
  CUW_RET(alloc(reinterpret_cast<void**>(&h->g.pf), sizeof(float2) * (size_t)h->ldg * std::max(1, h->npro)));
  for (int i = 0; i < 2; ++i)
    CUW_RET(alloc(reinterpret_cast<void**>(&h->g.xminus[i]), sizeof(double2) * (size_t)h->ldg * h->d.nbh));
  const size_t psi_split = (size_t)kBTile * ceil_div(h->d.nbh, 64) * ceil_div(h->d.ngl, kCK);
  for (int i = 0; i < 2; ++i) CUW_RET(alloc(reinterpret_cast<void**>(&h->g.bpre[i]), sizeof(float) * psi_split));
  // largest small-matrix operand: [C1 | C2] of ADDPRO, tiles of 32 bands
  const int np = std::max(1, h->npro), nb = h->d.nbh;
  size_t slot = (size_t)ceil_div(nb, 32) * ceil_div(np, kCK);
  slot = std::max(slot, (size_t)ceil_div(np, 64) * ceil_div(nb, kCK));
  slot = std::max(slot, (size_t)ceil_div(nb, 64) * ceil_div(np, kCK));
  slot = std::max(slot, (size_t)ceil_div(nb, 64) * ceil_div(2 * nb, kCK));
  h->g.bsmall_slot = slot * kBTile;
  CUW_RET(alloc(reinterpret_cast<void**>(&h->g.bsmall), sizeof(float) * 3 * h->g.bsmall_slot));
  return CUW_OK;
}

int tc_pro_table(Handle* h) {
  if (h->npro == 0) return CUW_OK;
  const dim3 grid(std::min(ceil_div(h->ldg, 256), 64), h->d.nat);
  k_pro_f32<<<grid, 256, 0, h->stream>>>(h->d.ngl, h->ldg, h->g.t_ipro0, h->g.t_nlmn, h->g.pdesc, h->g.ylm, h->g.pro,
                                         h->g.eigr, h->g.pf);
  CUW_LAUNCH_CHECK("k_pro_f32");
  return CUW_OK;
}

void tc_scope(Handle* h, bool open) {
  h->tc_scope_open = open;
  h->g.bpre_src[0] = h->g.bpre_src[1] = nullptr;
}

static int tc_bsplit(Handle* h, const BSplitSrc& b, int ntile, int nchk, float* out) {
  k_bsplit<<<dim3(nchk, ntile), 256, 0, h->stream>>>(b, nchk, out);
  CUW_LAUNCH_CHECK("k_bsplit");
  return CUW_OK;
}
// split form of wave-function array psi (B operand, rows = bands, K = g)
static int tc_bsplit_psi(Handle* h, const double2* psi, const float** out) {
  Device& g = h->g;
  for (int i = 0; i < 2; ++i)
    if (h->tc_scope_open && g.bpre_src[i] == psi) {
      *out = g.bpre[i];
      return CUW_OK;
    }
  const int i = g.bpre_src[0] ? 1 : 0;
  BSplitSrc b{0, psi, nullptr, (long long)h->ldg, h->d.nbh, h->d.ngl, 0};
  CUW_RET(tc_bsplit(h, b, ceil_div(h->d.nbh, 64), ceil_div(h->d.ngl, kCK), g.bpre[i]));
  if (h->tc_scope_open) g.bpre_src[i] = psi;
  *out = g.bpre[i];
  return CUW_OK;
}
// split form of a small matrix into slot `slot` of h->g.bsmall
static int tc_bsplit_small(Handle* h, const BSplitSrc& b, int ntile, int nchk, int slot, const float** out) {
  if ((size_t)ntile * nchk * kBTile > h->g.bsmall_slot) return h->fail(CUW_ERR_STATE, "split operand scratch too small");
  float* dst = h->g.bsmall + (size_t)slot * h->g.bsmall_slot;
  CUW_RET(tc_bsplit(h, b, ntile, nchk, dst));
  *out = dst;
  return CUW_OK;
}

// X(-G) copy of a wave-function array into scratch slot i
static int tc_minus(Handle* h, const double2* x, int i, const double2** out) {
  const size_t n = (size_t)h->ldg * h->d.nbh;
  const int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)8 * h->nsm);
  k_minus_copy<<<blocks, 256, 0, h->stream>>>(x, h->g.xminus[i], h->g.minusg, h->d.ngl, h->ldg, h->d.nbh);
  CUW_LAUNCH_CHECK("k_minus_copy");
  *out = h->g.xminus[i];
  return CUW_OK;
}

static int tc_reduce(Handle* h, const float2* part, int nz, size_t n, double scale, double2* out) {
  const int rb = (int)std::min<size_t>((n + 255) / 256, (size_t)4 * h->nsm);
  k_tc_reduce<<<rb, 256, 0, h->stream>>>(part, nz, n, scale, out);
  CUW_LAUNCH_CHECK("k_tc_reduce");
  return CUW_OK;
}

int tc_proj(Handle* h, const double2* psi, double2* proj) {
  const int nbh = h->d.nbh, npro = h->npro, ngl = h->d.ngl;
  const int tn = ceil_div(npro, 128), tb = ceil_div(nbh, 64);
  int ks = tc_splits(h, tn * tb, ngl, h->split_proj);
  const int kchunk = ceil_div(ceil_div(ngl, ks), kCK) * kCK;
  ks = ceil_div(ngl, kchunk);
  const size_t n = (size_t)nbh * npro;
  CUW_RET(ensure_part(h, sizeof(float2) * n * ks));
  float2* part = reinterpret_cast<float2*>(h->g.part);
  CUtensorMap tpf;
  CUW_RET(make_map(h, &tpf, h->g.pf, false, 2ll * ngl, npro, 2ll * h->ldg, 16, 128, CU_TENSOR_MAP_SWIZZLE_64B));
  const float* bpsi = nullptr;
  CUW_RET(tc_bsplit_psi(h, psi, &bpsi));
  k_tc_proj<<<dim3(tn, tb, ks), kThreads, ProjPipe::kSmem, h->stream>>>(tpf, bpsi, ceil_div(ngl, kCK), ngl, nbh, npro,
                                                                         kchunk, part, tc_err(h));
  CUW_LAUNCH_CHECK("k_tc_proj");
  return tc_reduce(h, part, ks, n, h->gweight, proj);
}

int tc_addpro(Handle* h, int mode, const double2* hpc, const double2* opc, const StepCoef& sc) {
  const int ngl = h->d.ngl, nbh = h->d.nbh, npro = h->npro;
  const dim3 grid(ceil_div(nbh, 32), ceil_div(ngl, 128));
  Device& g = h->g;
  CUtensorMap tpf;
  CUW_RET(make_map(h, &tpf, g.pf, false, 2ll * ngl, npro, 2ll * h->ldg, 256, 8, CU_TENSOR_MAP_SWIZZLE_NONE));
  const int nchk = ceil_div(npro, kCK);
  const float* bc = nullptr;
  BSplitSrc b{4, mode == ADDPRO_OPSI ? nullptr : hpc, mode == ADDPRO_HPSI ? nullptr : opc, (long long)nbh, nbh, npro, 0};
  CUW_RET(tc_bsplit_small(h, b, ceil_div(nbh, 32), nchk, 0, &bc));
#define TC_ADDPRO(M)                                                                                            \
  k_tc_addpro<M><<<grid, kThreads, AddproPipe::kSmem, h->stream>>>(g.hpsi, g.opsi, g.psi0, g.psim, g.mpsi, h->ldg, \
                                                                   ngl, nbh, npro, tpf, bc, nchk, sc, tc_err(h))
  if (mode == ADDPRO_HPSI) TC_ADDPRO(ADDPRO_HPSI);
  else if (mode == ADDPRO_OPSI) TC_ADDPRO(ADDPRO_OPSI);
  else TC_ADDPRO(ADDPRO_FUSED);
#undef TC_ADDPRO
  CUW_LAUNCH_CHECK("k_tc_addpro");
  return CUW_OK;
}

int tc_gram(Handle* h, const GramPair* pairs, int npair, bool minus, int nk, int nm, size_t sk, size_t sm,
            double scale, double2* dst) {
  if (npair < 1 || npair > 3) return h->fail(CUW_ERR_ARG, "Gram product: one to three pairs");
  TcGramArgs a{};
  a.npair = npair;
  a.nk = nk;
  a.nm = nm;
  a.kfast = sk == 1;
  a.nchk = ceil_div(nk, kCK);
  if (!a.kfast && sm != 1) return h->fail(CUW_ERR_UNSUPPORTED, "Gram product with neither index contiguous");
  if (minus && !a.kfast) return h->fail(CUW_ERR_UNSUPPORTED, "X(-k) Gram product of projections");
  TcGramMaps tm{};
  // X(-k) copies of the distinct X arrays (at most two: PSIBAR and OPSI)
  const double2* src[2] = {nullptr, nullptr};
  const double2* mcopy[2] = {nullptr, nullptr};
  const double2* ydone[3] = {nullptr, nullptr, nullptr};
  int nsmall = 0;
  for (int i = 0; i < npair; ++i) {
    const double2 *x = pairs[i].x, *y = pairs[i].y;
    if (a.kfast) {
      CUW_RET(map_c(h, &tm.x[i], x, nk, nm, (long long)sm, 16, 64, CU_TENSOR_MAP_SWIZZLE_128B));
      CUW_RET(tc_bsplit_psi(h, y, &a.ybs[i]));
    } else {
      CUW_RET(map_c(h, &tm.x[i], x, nm, nk, (long long)sk, 128, 8, CU_TENSOR_MAP_SWIZZLE_NONE));
      int same = -1;
      for (int j = 0; j < i; ++j)
        if (ydone[j] == y) same = j;
      if (same >= 0) {
        a.ybs[i] = a.ybs[same];
      } else {
        BSplitSrc b{1, y, nullptr, (long long)sk, nm, nk, 0};
        CUW_RET(tc_bsplit_small(h, b, ceil_div(nm, 64), a.nchk, nsmall++, &a.ybs[i]));
      }
      ydone[i] = y;
    }
    tm.xm[i] = tm.x[i];
    if (minus) {
      if (sm != (size_t)h->ldg || nk != h->d.ngl || nm != h->d.nbh)
        return h->fail(CUW_ERR_UNSUPPORTED, "X(-k) Gram product of a non wave-function array");
      int slot = -1;
      for (int j = 0; j < 2; ++j)
        if (src[j] == x) slot = j;
      if (slot < 0) {
        slot = src[0] ? 1 : 0;
        if (src[slot]) return h->fail(CUW_ERR_UNSUPPORTED, "more than two X arrays in one Gram call");
        src[slot] = x;
        CUW_RET(tc_minus(h, x, slot, &mcopy[slot]));
      }
      CUW_RET(map_c(h, &tm.xm[i], mcopy[slot], nk, nm, (long long)sm, 16, 64, CU_TENSOR_MAP_SWIZZLE_128B));
    }
  }
  for (int i = npair; i < 3; ++i) {
    tm.x[i] = tm.xm[i] = tm.x[0];
    a.ybs[i] = a.ybs[0];
  }
  const int tiles = ceil_div(nm, 64) * ceil_div(nm, 64) * npair;
  int ks = tc_splits(h, tiles, nk, h->split_gram);
  a.kchunk = ceil_div(ceil_div(nk, ks), kCK) * kCK;
  ks = ceil_div(nk, a.kchunk);
  const size_t mn = (size_t)nm * nm;
  CUW_RET(ensure_part(h, sizeof(float2) * mn * 2 * npair * ks));
  float2* part = reinterpret_cast<float2*>(h->g.part);
  const dim3 grid(ceil_div(nm, 64), ceil_div(nm, 64), ks * npair);
  if (minus) k_tc_gram<true><<<grid, kThreads, GramPipe::kSmem, h->stream>>>(a, tm, part, tc_err(h));
  else k_tc_gram<false><<<grid, kThreads, GramPipe::kSmem, h->stream>>>(a, tm, part, tc_err(h));
  CUW_LAUNCH_CHECK("k_tc_gram");
  return tc_reduce(h, part, ks, mn * 2 * npair, scale, dst);
}

int tc_addx(Handle* h, bool xminus, double2* out, const double2* x, const double2* l1, const double2* l2, int nm,
            int nn, int nk, size_t sxm, size_t sxk, size_t som, size_t son) {
  TcAddXArgs a;
  a.out = out;
  a.nm = nm;
  a.nn = nn;
  a.nk = nk;
  a.som = som;
  a.son = son;
  a.mfast = sxm == 1;
  a.nchk = ceil_div(2 * nk, kCK);
  TcAddXMaps tm;
  if (a.mfast) {
    const double2* x2 = x;
    if (xminus) {
      if (sxk != (size_t)h->ldg || nm != h->d.ngl || nk != h->d.nbh)
        return h->fail(CUW_ERR_UNSUPPORTED, "X(-G) update of a non wave-function array");
      CUW_RET(tc_minus(h, x, 0, &x2));
    }
    CUW_RET(map_c(h, &tm.x, x, nm, nk, (long long)sxk, 256, 8, CU_TENSOR_MAP_SWIZZLE_NONE));
    CUW_RET(map_c(h, &tm.x2, x2, nm, nk, (long long)sxk, 256, 8, CU_TENSOR_MAP_SWIZZLE_NONE));
  } else {
    if (sxk != 1 || xminus) return h->fail(CUW_ERR_UNSUPPORTED, "projection update with gathered rows");
    CUW_RET(map_c(h, &tm.x, x, nk, nm, (long long)sxm, 16, 128, CU_TENSOR_MAP_SWIZZLE_128B));
    tm.x2 = tm.x;
  }
  BSplitSrc b{3, l1, l2, (long long)nk, nn, 2 * nk, nk};
  CUW_RET(tc_bsplit_small(h, b, ceil_div(nn, 64), a.nchk, 0, &a.lbs));
  const dim3 grid(ceil_div(nm, 128), ceil_div(nn, 64));
  k_tc_addx<<<grid, kThreads, AddxPipe::kSmem, h->stream>>>(a, tm, tc_err(h));
  CUW_LAUNCH_CHECK("k_tc_addx");
  return CUW_OK;
}

int tc_force(Handle* h, const double2* ded, double* fpart, int* ntile) {
  const int ngl = h->d.ngl, nbh = h->d.nbh, npro = h->npro;
  const int tm = ceil_div(ngl, 128), tn = ceil_div(npro, 64);
  CUtensorMap tps;
  CUW_RET(map_c(h, &tps, h->g.psi0, ngl, nbh, h->ldg, 256, 8, CU_TENSOR_MAP_SWIZZLE_NONE));
  const int nchk = ceil_div(nbh, kCK);
  const float* be = nullptr;
  BSplitSrc b{2, ded, nullptr, (long long)nbh, npro, nbh, 0};
  CUW_RET(tc_bsplit_small(h, b, tn, nchk, 0, &be));
  if (nchk % 2 == 0 && nchk <= kFMaxChunks) {
    // persistent form: the psi0 tile stays in tensor memory across projector tiles
    const int nitems = tm * tn;
    k_tc_force_p<<<std::min(nitems, h->nsm), kThreads, kForcePSmem, h->stream>>>(
        tps, be, nchk, ngl, npro, h->ldg, tn, nitems, h->g.pf, h->g.gx, h->g.gy, h->g.gz, fpart, tc_err(h));
    CUW_LAUNCH_CHECK("k_tc_force_p");
    *ntile = tm;
    return CUW_OK;
  }
  k_tc_force<<<dim3(tm, tn), kThreads, ForcePipe::kSmem, h->stream>>>(tps, be, nchk, ngl, nbh, npro, h->g.pdesc,
                                                                      h->g.ylm, h->g.pro, h->g.eigr, h->g.gx,
                                                                      h->g.gy, h->g.gz, fpart, tc_err(h));
  CUW_LAUNCH_CHECK("k_tc_force");
  *ntile = tm;
  return CUW_OK;
}

}  // namespace cuw

// Check of the split-precision tensor-core path (no reference counterpart):
// C(M,N) = A(M,K) B(N,K)^T on device buffers, FP64 row-major with K
// contiguous, computed as three tf32 products with fp32 accumulation.
// err (device int) is set to 1 if a bounded wait ran out.
extern "C" int cuwaves_tc_gemm_check(int M, int N, int K, const double* A, const double* B, double* C, int* err,
                                     void* stream) {
  using namespace cuw;
  if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !C || !err) return CUW_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t smem = GemmPipe::kSmem;
  if (smem_allow((const void*)k_tf32x3_gemm, (int)smem) != cudaSuccess) return CUW_ERR_CUDA;
  dim3 grid((M + 127) / 128, (N + 127) / 128);
  k_tf32x3_gemm<<<grid, kThreads, smem, st>>>(M, N, K, A, B, C, err);
  if (cudaGetLastError() != cudaSuccess) return CUW_ERR_CUDA;
  return CUW_OK;
}
