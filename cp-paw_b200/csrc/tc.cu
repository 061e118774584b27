// Mixed-precision contractions on the 5th-generation tensor cores (tcgen05).
//
// Every product is a real GEMM C = A * B^T whose FP64 operands are split on the
// fly into tf32 pairs (hi + lo) and multiplied as hi*hi + hi*lo + lo*hi with
// fp32 accumulation in tensor memory (three-term split precision), drained
// after every K = 8 step into register sums (tc_pipe.cuh).  Complex products
// use the real form of tc_pipe.cuh.  Every wait is bounded; a wait that runs
// out sets an error flag and the kernel leaves through its cleanup path (TMEM
// released) instead of hanging.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "cuwaves_internal.cuh"
#include "tc_pipe.cuh"

namespace cuw {
namespace {

// Real K values per shared-memory stage (four MMA steps of K = 8).  The
// accumulation run stays one MMA step: the tensor core's truncating fp32
// accumulation was measured on B200 at a signed mean error of -3.7e-8 /
// -8.7e-8 / -1.8e-7 of |C| for runs of 8 / 16 / 32 real K, and one step keeps
// the energy bias below 1e-6 Ha/atom.
// Eight producer warps (two per SM sub-partition): the producers' dependent
// table and coefficient loads need more than one warp per scheduler in flight.
constexpr int kBK = 32, kCK = kBK / 2, kStages = 3, kNPW = 8;
using MPipe = tc::Pipe<kBK, kStages, kNPW>;
constexpr int kProd = MPipe::kProducers;
// k_tc_force reuses the stage buffers for a 128 x 64 FP64 tile
static_assert(sizeof(float) * kStages * MPipe::kStage >= sizeof(double) * 128 * 64, "stage area too small");

__device__ __forceinline__ double2 dz() { return make_double2(0.0, 0.0); }

// Producer items per thread and stage: 128 A rows and 64 complex B columns,
// each item covering two complex K values.  Every producer first issues all
// global loads of its items (held in registers), then converts and stores: the
// shared-memory stores would otherwise keep later loads from being hoisted.
constexpr int kItemsA = 128 * (kCK / 2) / kProd;
constexpr int kItemsB = 64 * (kCK / 2) / kProd;
static_assert(128 * (kCK / 2) % kProd == 0 && 64 * (kCK / 2) % kProd == 0, "items must divide evenly");

// ---------------------------------------------------------------------------
// Plain real GEMM C(M,N) = A(M,K) * B(N,K)^T, FP64 in and out, row-major with
// K contiguous: the reference product of the split-precision machinery.
// One CTA computes a 128 x 128 tile over the whole K range.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(MPipe::kThreads, 1)
    k_tf32x3_gemm(int M, int N, int K, const double* __restrict__ A, const double* __restrict__ B,
                  double* __restrict__ C, int* __restrict__ err) {
  const int m0 = blockIdx.x * 128, n0 = blockIdx.y * 128;
  auto produce = [&](int c, int t, float* ahi, float* alo, float* bhi, float* blo) {
    const int k0 = c * kBK;
    for (int it = t; it < 128 * (kBK / 4); it += kProd) {
      const int r = it % 128, g = it / 128, k = k0 + 4 * g;
      double a[4] = {0.0, 0.0, 0.0, 0.0}, b[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (m0 + r < M && k + q < K) a[q] = A[(size_t)(m0 + r) * K + k + q];
        if (n0 + r < N && k + q < K) b[q] = B[(size_t)(n0 + r) * K + k + q];
      }
      tc::store_split4(ahi, alo, tc::tile_f4(r, g), a[0], a[1], a[2], a[3]);
      tc::store_split4(bhi, blo, tc::tile_f4(r, g), b[0], b[1], b[2], b[3]);
    }
  };
  auto finish = [&](const float (&acc)[MPipe::kCols], int row, int col0) {
    if (m0 + row >= M) return;
    double* out = C + (size_t)(m0 + row) * N + n0 + col0;
    const int nc = min(MPipe::kCols, N - n0 - col0);
#pragma unroll
    for (int j = 0; j < MPipe::kCols; ++j)
      if (j < nc) out[j] = (double)acc[j];
  };
  tc::pipe_run<kBK, kStages, kNPW>((K + kBK - 1) / kBK, produce, finish, err);
}

// out[i] = scale * sum_z part[z*n + i], summed in FP64 in a fixed order
__global__ void k_tc_reduce(const float2* __restrict__ part, int nz, size_t n, double scale,
                            double2* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double sx = 0.0, sy = 0.0;
    for (int z = 0; z < nz; ++z) {
      const float2 v = part[(size_t)z * n + i];
      sx += (double)v.x;
      sy += (double)v.y;
    }
    out[i] = make_double2(sx * scale, sy * scale);
  }
}

// ---------------------------------------------------------------------------
// <p|psi> partial sums (WAVES_PROJECTIONS, src/paw_waves1.f90:5746-5905):
// part[z][p][b] = sum_{g in split z} conj(PRO(g,p)) psi(g,b)   (float2)
// M = projectors (blockIdx.x), N = 64 bands (blockIdx.y), K = g (blockIdx.z)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(MPipe::kThreads, 1)
    k_tc_proj(const double2* __restrict__ psi, int ldg, int ngl, int nbh, int npro, int kchunk,
              const ProDesc* __restrict__ pdesc, const double* __restrict__ ylm, const double* __restrict__ pro,
              const double2* __restrict__ eigr, float2* __restrict__ part, int* __restrict__ err) {
  __shared__ ProDesc sd[128];
  const int m0 = blockIdx.x * 128, b0 = blockIdx.y * 64;
  const int gbeg = blockIdx.z * kchunk, gend = min(ngl, gbeg + kchunk);
  for (int t = threadIdx.x; t < 128; t += blockDim.x) sd[t] = m0 + t < npro ? pdesc[m0 + t] : ProDesc{0, 0, 0, -1};
  __syncthreads();
  auto produce = [&](int c, int t, float* ahi, float* alo, float* bhi, float* blo) {
    const int g0 = gbeg + c * kCK;
    double2 av[kItemsA][2], bv[kItemsB][2];
    // eight consecutive lanes cover the stage's 16 g of one row: the table and
    // coefficient reads are contiguous in g
    constexpr int NG = kCK / 2;
#pragma unroll
    for (int q = 0; q < kItemsA; ++q) {
      const int it = t + q * kProd, r = it / NG, g = g0 + 2 * (it % NG);
      const ProDesc d = sd[r];
      av[q][0] = (d.l >= 0 && g < gend) ? pro_value(g, ngl, d, ylm, pro, eigr) : dz();
      av[q][1] = (d.l >= 0 && g + 1 < gend) ? pro_value(g + 1, ngl, d, ylm, pro, eigr) : dz();
    }
#pragma unroll
    for (int q = 0; q < kItemsB; ++q) {
      const int it = t + q * kProd, b = b0 + it / NG, g = g0 + 2 * (it % NG);
      bv[q][0] = (b < nbh && g < gend) ? psi[(size_t)g + (size_t)ldg * b] : dz();
      bv[q][1] = (b < nbh && g + 1 < gend) ? psi[(size_t)g + 1 + (size_t)ldg * b] : dz();
    }
#pragma unroll
    for (int q = 0; q < kItemsA; ++q) {
      const int it = t + q * kProd;
      tc::put_a(ahi, alo, it / NG, it % NG, cconj(av[q][0]), cconj(av[q][1]));
    }
#pragma unroll
    for (int q = 0; q < kItemsB; ++q) {
      const int it = t + q * kProd;
      tc::put_b(bhi, blo, it / NG, it % NG, bv[q][0], bv[q][1]);
    }
  };
  auto finish = [&](const float (&acc)[MPipe::kCols], int row, int col0) {
    const int p = m0 + row;
    if (p >= npro) return;
    float2* out = part + ((size_t)blockIdx.z * npro + p) * nbh;
    const int bb = b0 + col0 / 2;
#pragma unroll
    for (int j = 0; j < 32; ++j)
      if (bb + j < nbh) out[bb + j] = make_float2(acc[2 * j], acc[2 * j + 1]);
  };
  const int nchunk = gend > gbeg ? (gend - gbeg + kCK - 1) / kCK : 0;
  tc::pipe_run<kBK, kStages, kNPW>(nchunk, produce, finish, err);
}

// ---------------------------------------------------------------------------
// ADDPRO with the step epilogues (WAVES_ADDPRO, src/paw_waves1.f90:5908-6067,
// and the epilogues of the FP64 k_addpro): 128 g x 32 bands per CTA, the tile
// columns hold C1 (hproj) products for the bands, then C2 (oproj) products.
// ---------------------------------------------------------------------------
template <int MODE>
__global__ void __launch_bounds__(MPipe::kThreads, 1)
    k_tc_addpro(double2* __restrict__ hpsi, double2* __restrict__ opsi, const double2* __restrict__ psi0,
                double2* __restrict__ psim, const double* __restrict__ mpsi, int ldg, int ngl, int nbh, int npro,
                const double2* __restrict__ c1, const double2* __restrict__ c2, const ProDesc* __restrict__ pdesc,
                const double* __restrict__ ylm, const double* __restrict__ pro, const double2* __restrict__ eigr,
                StepCoef sc, int* __restrict__ err) {
  constexpr bool USE_H = (MODE != ADDPRO_OPSI);
  constexpr bool USE_O = (MODE != ADDPRO_HPSI);
  const int g0 = blockIdx.x * 128, b0 = blockIdx.y * 32;
  auto produce = [&](int c, int t, float* ahi, float* alo, float* bhi, float* blo) {
    const int p0 = c * kCK;
    double2 av[kItemsA][2], bv[kItemsB][2];
#pragma unroll
    for (int q = 0; q < kItemsA; ++q) {
      const int it = t + q * kProd, g = g0 + it % 128, p = p0 + 2 * (it / 128);
      av[q][0] = (g < ngl && p < npro) ? pro_value(g, ngl, pdesc[p], ylm, pro, eigr) : dz();
      av[q][1] = (g < ngl && p + 1 < npro) ? pro_value(g, ngl, pdesc[p + 1], ylm, pro, eigr) : dz();
    }
#pragma unroll
    for (int q = 0; q < kItemsB; ++q) {
      const int it = t + q * kProd, j = it % 64, mt = j / 32, b = b0 + (j % 32), p = p0 + 2 * (it / 64);
      const double2* cm = mt == 0 ? c1 : c2;
      const bool use = (mt == 0 ? USE_H : USE_O) && b < nbh;
      bv[q][0] = (use && p < npro) ? cm[(size_t)b + (size_t)nbh * p] : dz();
      bv[q][1] = (use && p + 1 < npro) ? cm[(size_t)b + (size_t)nbh * (p + 1)] : dz();
    }
#pragma unroll
    for (int q = 0; q < kItemsA; ++q) {
      const int it = t + q * kProd;
      tc::put_a(ahi, alo, it % 128, it / 128, av[q][0], av[q][1]);
    }
#pragma unroll
    for (int q = 0; q < kItemsB; ++q) {
      const int it = t + q * kProd;
      tc::put_b(bhi, blo, it % 64, it / 64, bv[q][0], bv[q][1]);
    }
  };
  auto finish = [&](const float (&acc)[MPipe::kCols], int row, int col0) {
    const int g = g0 + row;
    if (g >= ngl) return;
    const double rm = 1.0 / mpsi[g];
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const int b = b0 + j;
      if (b >= nbh) continue;
      const size_t k = (size_t)g + (size_t)ldg * b;
      const double2 v = make_double2((double)acc[2 * j], (double)acc[2 * j + 1]);
      if (col0 == 0 && USE_H) {
        const double2 hv = cadd(hpsi[k], v);
        hpsi[k] = hv;
        if (MODE == ADDPRO_FUSED) {
          const double2 p0v = psi0[k], pm = psim[k];
          const double a3 = sc.a3 * rm;
          psim[k] = make_double2(sc.a1 * p0v.x + sc.a2 * pm.x + a3 * hv.x, sc.a1 * p0v.y + sc.a2 * pm.y + a3 * hv.y);
        }
      } else if (col0 != 0 && USE_O) {
        const double2 p0v = psi0[k];
        const double s = sc.oscale * rm;
        opsi[k] = make_double2((p0v.x + v.x) * s, (p0v.y + v.y) * s);
      }
    }
  };
  tc::pipe_run<kBK, kStages, kNPW>((npro + kCK - 1) / kCK, produce, finish, err);
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
  GramPair pair[3];
  int npair, nk, nm;
  size_t sk, sm;
  int kchunk;
};

template <bool MINUS>
__global__ void __launch_bounds__(MPipe::kThreads, 1)
    k_tc_gram(TcGramArgs a, const int* __restrict__ minusg, float2* __restrict__ part, int* __restrict__ err) {
  const int pair = blockIdx.z % a.npair, split = blockIdx.z / a.npair;
  const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
  const double2* X = a.pair[pair].x;
  const double2* Y = a.pair[pair].y;
  const int kbeg = split * a.kchunk, kend = min(a.nk, kbeg + a.kchunk);
  auto produce = [&](int c, int t, float* ahi, float* alo, float* bhi, float* blo) {
    const int k0 = kbeg + c * kCK;
    // lanes run along the contiguous index: k when sk == 1 (plane waves), the
    // band otherwise (projections)
    constexpr int NK = kCK / 2;
    const bool kfast = a.sk == 1;
    double2 av[kItemsA][2], bv[kItemsB][2];
#pragma unroll
    for (int q = 0; q < kItemsA; ++q) {
      const int it = t + q * kProd;
      const int r = kfast ? it / NK : it % 128, ki = kfast ? it % NK : it / 128;
      const int k = k0 + 2 * ki, m = m0 + (r & 63);
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        av[q][e] = dz();
        if (m < a.nm && k + e < kend) {
          if (r < 64) {
            av[q][e] = cconj(X[(size_t)(k + e) * a.sk + (size_t)m * a.sm]);
          } else {
            const int kk = MINUS ? minusg[k + e] : k + e;
            av[q][e] = X[(size_t)kk * a.sk + (size_t)m * a.sm];
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < kItemsB; ++q) {
      const int it = t + q * kProd;
      const int j = kfast ? it / NK : it % 64, ki = kfast ? it % NK : it / 64;
      const int n = n0 + j, k = k0 + 2 * ki;
      bv[q][0] = (n < a.nm && k < kend) ? Y[(size_t)k * a.sk + (size_t)n * a.sm] : dz();
      bv[q][1] = (n < a.nm && k + 1 < kend) ? Y[(size_t)(k + 1) * a.sk + (size_t)n * a.sm] : dz();
    }
#pragma unroll
    for (int q = 0; q < kItemsA; ++q) {
      const int it = t + q * kProd;
      tc::put_a(ahi, alo, kfast ? it / NK : it % 128, kfast ? it % NK : it / 128, av[q][0], av[q][1]);
    }
#pragma unroll
    for (int q = 0; q < kItemsB; ++q) {
      const int it = t + q * kProd;
      tc::put_b(bhi, blo, kfast ? it / NK : it % 64, kfast ? it % NK : it / 64, bv[q][0], bv[q][1]);
    }
  };
  auto finish = [&](const float (&acc)[MPipe::kCols], int row, int col0) {
    const int t = row >> 6, m = m0 + (row & 63);
    if (m >= a.nm) return;
    const size_t mn = (size_t)a.nm * a.nm;
    float2* out = part + ((size_t)blockIdx.z * 2 + t) * mn;
    const int nb = n0 + col0 / 2;
#pragma unroll
    for (int j = 0; j < 32; ++j)
      if (nb + j < a.nm) out[(size_t)m + (size_t)a.nm * (nb + j)] = make_float2(acc[2 * j], acc[2 * j + 1]);
  };
  const int nchunk = kend > kbeg ? (kend - kbeg + kCK - 1) / kCK : 0;
  tc::pipe_run<kBK, kStages, kNPW>(nchunk, produce, finish, err);
}

// ---------------------------------------------------------------------------
// ADDOPSI / ADDOPROJ (src/paw_waves2.f90:547-615, 687-758):
//   out(m,n) += sum_k X(m,k) L1(k,n) + conj(X(m',k)) L2(k,n),
//   m' = minusg[m] (XMINUS) or m.  K runs over both halves (2 nk).
// ---------------------------------------------------------------------------
struct TcAddXArgs {
  double2* out;
  const double2* x;
  const double2* l1;
  const double2* l2;
  int nm, nn, nk;
  size_t sxm, sxk, som, son;
};

template <bool XMINUS>
__global__ void __launch_bounds__(MPipe::kThreads, 1)
    k_tc_addx(TcAddXArgs a, const int* __restrict__ minusg, int* __restrict__ err) {
  const int m0 = blockIdx.x * 128, n0 = blockIdx.y * 64;
  const int ktot = 2 * a.nk;
  auto produce = [&](int c, int t, float* ahi, float* alo, float* bhi, float* blo) {
    const int kg0 = c * kCK;
    double2 av[kItemsA][2], bv[kItemsB][2];
#pragma unroll
    for (int q = 0; q < kItemsA; ++q) {
      const int it = t + q * kProd, m = m0 + it % 128;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int kg = kg0 + 2 * (it / 128) + e;
        av[q][e] = dz();
        if (m < a.nm && kg < ktot) {
          if (kg < a.nk) {
            av[q][e] = a.x[(size_t)m * a.sxm + (size_t)kg * a.sxk];
          } else {
            const int mm = XMINUS ? minusg[m] : m;
            av[q][e] = cconj(a.x[(size_t)mm * a.sxm + (size_t)(kg - a.nk) * a.sxk]);
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < kItemsB; ++q) {
      const int it = t + q * kProd, n = n0 + it % 64;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int kg = kg0 + 2 * (it / 64) + e;
        bv[q][e] = dz();
        if (n < a.nn && kg < ktot)
          bv[q][e] = kg < a.nk ? a.l1[(size_t)kg + (size_t)a.nk * n] : a.l2[(size_t)(kg - a.nk) + (size_t)a.nk * n];
      }
    }
#pragma unroll
    for (int q = 0; q < kItemsA; ++q) {
      const int it = t + q * kProd;
      tc::put_a(ahi, alo, it % 128, it / 128, av[q][0], av[q][1]);
    }
#pragma unroll
    for (int q = 0; q < kItemsB; ++q) {
      const int it = t + q * kProd;
      tc::put_b(bhi, blo, it % 64, it / 64, bv[q][0], bv[q][1]);
    }
  };
  auto finish = [&](const float (&acc)[MPipe::kCols], int row, int col0) {
    const int m = m0 + row;
    if (m >= a.nm) return;
    const int nb = n0 + col0 / 2;
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      if (nb + j >= a.nn) continue;
      const size_t k = (size_t)m * a.som + (size_t)(nb + j) * a.son;
      const double2 o = a.out[k];
      a.out[k] = make_double2(o.x + (double)acc[2 * j], o.y + (double)acc[2 * j + 1]);
    }
  };
  tc::pipe_run<kBK, kStages, kNPW>((ktot + kCK - 1) / kCK, produce, finish, err);
}

// ---------------------------------------------------------------------------
// Forces (WAVES_DEDPRO + WAVES_PROFORCE, src/paw_waves1.f90:5694-5743,
// 6112-6234): D(g,p) = sum_b psi0(g,b) conj(E(b,p)) on the tensor cores for
// 128 g x 64 projectors, then sv(g,p) = Re[i P (-i)^l EIGR conj(D)] Y_lm in the
// drain warps (into the freed stage buffers) and fpart[tile][p][c] =
// sum_g sv(g,p) G_c(g) by the whole CTA.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(MPipe::kThreads, 1)
    k_tc_force(const double2* __restrict__ psi0, int ldg, int ngl, int nbh, int npro,
               const double2* __restrict__ ded, const ProDesc* __restrict__ pdesc, const double* __restrict__ ylm,
               const double* __restrict__ pro, const double2* __restrict__ eigr, const double* __restrict__ gx,
               const double* __restrict__ gy, const double* __restrict__ gz, double* __restrict__ fpart,
               int* __restrict__ err) {
  const int g0 = blockIdx.x * 128, p0 = blockIdx.y * 64;
  auto produce = [&](int c, int t, float* ahi, float* alo, float* bhi, float* blo) {
    const int bb = c * kCK;
    double2 av[kItemsA][2], bv[kItemsB][2];
#pragma unroll
    for (int q = 0; q < kItemsA; ++q) {
      const int it = t + q * kProd, g = g0 + it % 128, b = bb + 2 * (it / 128);
      av[q][0] = (g < ngl && b < nbh) ? psi0[(size_t)g + (size_t)ldg * b] : dz();
      av[q][1] = (g < ngl && b + 1 < nbh) ? psi0[(size_t)g + (size_t)ldg * (b + 1)] : dz();
    }
#pragma unroll
    for (int q = 0; q < kItemsB; ++q) {
      const int it = t + q * kProd, p = p0 + it % 64, b = bb + 2 * (it / 64);
      bv[q][0] = (p < npro && b < nbh) ? cconj(ded[(size_t)b + (size_t)nbh * p]) : dz();
      bv[q][1] = (p < npro && b + 1 < nbh) ? cconj(ded[(size_t)b + 1 + (size_t)nbh * p]) : dz();
    }
#pragma unroll
    for (int q = 0; q < kItemsA; ++q) {
      const int it = t + q * kProd;
      tc::put_a(ahi, alo, it % 128, it / 128, av[q][0], av[q][1]);
    }
#pragma unroll
    for (int q = 0; q < kItemsB; ++q) {
      const int it = t + q * kProd;
      tc::put_b(bhi, blo, it % 64, it / 64, bv[q][0], bv[q][1]);
    }
  };
  double* sv = reinterpret_cast<double*>(tc::pipe_stage_base());  // [128][64]
  auto finish = [&](const float (&acc)[MPipe::kCols], int row, int col0) {
    const int g = g0 + row, pb = col0 / 2;
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const int p = p0 + pb + j;
      double v = 0.0;
      if (g < ngl && p < npro) {
        const ProDesc d = pdesc[p];
        const double pr = pro[(size_t)g + (size_t)ngl * d.ibare];
        const double y = ylm[(size_t)g + (size_t)ngl * d.lm];
        const double2 cw = cmul(make_double2(0.0, pr), cmul(mipow(d.l), eigr[(size_t)g + (size_t)ngl * d.iat]));
        v = (cw.x * (double)acc[2 * j] + cw.y * (double)acc[2 * j + 1]) * y;
      }
      sv[row * 64 + pb + j] = v;
    }
  };
  tc::pipe_run<kBK, kStages, kNPW>((nbh + kCK - 1) / kCK, produce, finish, err);
  // pipe_run ended with a CTA barrier: sv is complete (if a wait ran out the
  // error flag is set and the caller discards the result)
  for (int i = threadIdx.x; i < 64 * 3; i += blockDim.x) {
    const int pl = i / 3, c = i % 3, p = p0 + pl;
    if (p >= npro) continue;
    const double* gc = c == 0 ? gx : (c == 1 ? gy : gz);
    double s = 0.0;
    for (int r = 0; r < 128 && g0 + r < ngl; ++r) s += sv[r * 64 + pl] * gc[g0 + r];
    fpart[((size_t)blockIdx.x * npro + p) * 3 + c] = s;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// host side of the split-precision contractions
// ---------------------------------------------------------------------------
static int* tc_err(Handle* h) { return h->g.ostatus + 12; }

// number of K splits so that tiles * splits fills the GPU once (one CTA per SM)
static int tc_splits(Handle* h, int tiles, int nk) {
  const int want = std::max(1, ceil_div(h->nsm, std::max(1, tiles)));
  return std::max(1, std::min(want, ceil_div(nk, 4 * kCK)));
}

int tc_setup(Handle* h) {
  const int sm = (int)MPipe::kSmem;
  CUW_TRY(smem_allow((const void*)k_tc_proj, sm));
  CUW_TRY(smem_allow((const void*)k_tc_addpro<ADDPRO_HPSI>, sm));
  CUW_TRY(smem_allow((const void*)k_tc_addpro<ADDPRO_OPSI>, sm));
  CUW_TRY(smem_allow((const void*)k_tc_addpro<ADDPRO_FUSED>, sm));
  CUW_TRY(smem_allow((const void*)k_tc_gram<true>, sm));
  CUW_TRY(smem_allow((const void*)k_tc_gram<false>, sm));
  CUW_TRY(smem_allow((const void*)k_tc_addx<true>, sm));
  CUW_TRY(smem_allow((const void*)k_tc_addx<false>, sm));
  CUW_TRY(smem_allow((const void*)k_tc_force, sm));
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
  int ks = tc_splits(h, tn * tb, ngl);
  const int kchunk = ceil_div(ceil_div(ngl, ks), kCK) * kCK;
  ks = ceil_div(ngl, kchunk);
  const size_t n = (size_t)nbh * npro;
  CUW_RET(ensure_part(h, sizeof(float2) * n * ks));
  float2* part = reinterpret_cast<float2*>(h->g.part);
  k_tc_proj<<<dim3(tn, tb, ks), MPipe::kThreads, MPipe::kSmem, h->stream>>>(
      psi, h->ldg, ngl, nbh, npro, kchunk, h->g.pdesc, h->g.ylm, h->g.pro, h->g.eigr, part, tc_err(h));
  CUW_LAUNCH_CHECK("k_tc_proj");
  return tc_reduce(h, part, ks, n, h->gweight, proj);
}

int tc_addpro(Handle* h, int mode, const double2* hpc, const double2* opc, const StepCoef& sc) {
  const int ngl = h->d.ngl, nbh = h->d.nbh, npro = h->npro;
  const dim3 grid(ceil_div(ngl, 128), ceil_div(nbh, 32));
  Device& g = h->g;
#define TC_ADDPRO(M)                                                                                         \
  k_tc_addpro<M><<<grid, MPipe::kThreads, MPipe::kSmem, h->stream>>>(g.hpsi, g.opsi, g.psi0, g.psim, g.mpsi, \
                                                                     h->ldg, ngl, nbh, npro, hpc, opc,       \
                                                                     g.pdesc, g.ylm, g.pro, g.eigr, sc,      \
                                                                     tc_err(h))
  if (mode == ADDPRO_HPSI) TC_ADDPRO(ADDPRO_HPSI);
  else if (mode == ADDPRO_OPSI) TC_ADDPRO(ADDPRO_OPSI);
  else TC_ADDPRO(ADDPRO_FUSED);
#undef TC_ADDPRO
  CUW_LAUNCH_CHECK("k_tc_addpro");
  return CUW_OK;
}

int tc_gram(Handle* h, const GramPair* pairs, int npair, bool minus, int nk, int nm, size_t sk, size_t sm,
            double scale, double2* dst) {
  TcGramArgs a;
  for (int i = 0; i < npair; ++i) a.pair[i] = pairs[i];
  a.npair = npair;
  a.nk = nk;
  a.nm = nm;
  a.sk = sk;
  a.sm = sm;
  const int tiles = ceil_div(nm, 64) * ceil_div(nm, 64) * npair;
  int ks = tc_splits(h, tiles, nk);
  a.kchunk = ceil_div(ceil_div(nk, ks), kCK) * kCK;
  ks = ceil_div(nk, a.kchunk);
  const size_t mn = (size_t)nm * nm;
  CUW_RET(ensure_part(h, sizeof(float2) * mn * 2 * npair * ks));
  float2* part = reinterpret_cast<float2*>(h->g.part);
  const dim3 grid(ceil_div(nm, 64), ceil_div(nm, 64), ks * npair);
  if (minus)
    k_tc_gram<true><<<grid, MPipe::kThreads, MPipe::kSmem, h->stream>>>(a, h->g.minusg, part, tc_err(h));
  else
    k_tc_gram<false><<<grid, MPipe::kThreads, MPipe::kSmem, h->stream>>>(a, h->g.minusg, part, tc_err(h));
  CUW_LAUNCH_CHECK("k_tc_gram");
  return tc_reduce(h, part, ks, mn * 2 * npair, scale, dst);
}

int tc_addx(Handle* h, bool xminus, double2* out, const double2* x, const double2* l1, const double2* l2, int nm,
            int nn, int nk, size_t sxm, size_t sxk, size_t som, size_t son) {
  TcAddXArgs a{out, x, l1, l2, nm, nn, nk, sxm, sxk, som, son};
  const dim3 grid(ceil_div(nm, 128), ceil_div(nn, 64));
  if (xminus) k_tc_addx<true><<<grid, MPipe::kThreads, MPipe::kSmem, h->stream>>>(a, h->g.minusg, tc_err(h));
  else k_tc_addx<false><<<grid, MPipe::kThreads, MPipe::kSmem, h->stream>>>(a, h->g.minusg, tc_err(h));
  CUW_LAUNCH_CHECK("k_tc_addx");
  return CUW_OK;
}

int tc_force(Handle* h, const double2* ded, double* fpart, int* ntile) {
  const int ngl = h->d.ngl, nbh = h->d.nbh, npro = h->npro;
  const int tm = ceil_div(ngl, 128), tn = ceil_div(npro, 64);
  k_tc_force<<<dim3(tm, tn), MPipe::kThreads, MPipe::kSmem, h->stream>>>(
      h->g.psi0, h->ldg, ngl, nbh, npro, ded, h->g.pdesc, h->g.ylm, h->g.pro, h->g.eigr, h->g.gx, h->g.gy, h->g.gz,
      fpart, tc_err(h));
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
  const size_t smem = MPipe::kSmem;
  if (smem_allow((const void*)k_tf32x3_gemm, (int)smem) != cudaSuccess)
    return CUW_ERR_CUDA;
  dim3 grid((M + 127) / 128, (N + 127) / 128);
  k_tf32x3_gemm<<<grid, MPipe::kThreads, smem, st>>>(M, N, K, A, B, C, err);
  if (cudaGetLastError() != cudaSuccess) return CUW_ERR_CUDA;
  return CUW_OK;
}
