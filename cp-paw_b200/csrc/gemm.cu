// Complex FP64 contractions of the WAVES path on the FP64 tensor cores
// (mma.sync m8n8k4 f64), with the projector functions generated in the tile
// loaders instead of being stored.
//
// Reference routines and the contraction each kernel replaces:
//   k_proj      WAVES_PROJECTIONS (src/paw_waves1.f90:5746-5905):
//               PROJ(b,p) = Omega sum_G conj(PRO(G,p)) psi(G,b)      [split-K]
//   k_addpro    WAVES_ADDPRO (src/paw_waves1.f90:5908-6067):
//               psi(G,b) += sum_p PRO(G,p) C(p,b)
//               with the epilogues of WAVES$HPSI (:4793-4916), WAVES_OPSI
//               (:5043-5096), the mass scaling of WAVES$ORTHOGONALIZE
//               (src/paw_waves2.f90:140-162) and WAVES$PROPAGATE (:6575-6583)
//   k_gram      PLANEWAVE$SCALARPRODUCT ' '/'='/'-' (src/paw_fft.f90:2344-2422)
//               as used by WAVES_OVERLAP (src/paw_waves2.f90:761-853) and the
//               projector sums of WAVES_1COVERLAP (:856-1022)         [split-K]
//   k_addx      WAVES_ADDOPSI (src/paw_waves2.f90:547-615), WAVES_ADDOPROJ
//               (:687-758) and the PSI update of WAVES_GRAMSCHMIDT (:2131-2136)
//   k_force     WAVES_DEDPRO + WAVES_PROFORCE (src/paw_waves1.f90:5694-5743,
//               6112-6234) fused: the (NGL,NPRO) array DEDPRO is never stored.
//
// PRO(G,p) = Y_lm(G) P_ln(|G|) (-i)^l exp(-iG.R_a)   (WAVES_EXPANDPRO :6070-6109)
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "cuwaves_internal.cuh"

namespace cuw {

namespace {

constexpr int BM = 64, BN = 64, BK = 16, LDS = 20, NT = 256;
constexpr int TILE = BM * LDS;  // doubles of one real or imaginary tile part
constexpr int EPT = BM * BK / NT;  // tile elements per thread and operand (4)

// ---------------------------------------------------------------------------
// warp-level complex MMA over one BK slice held in shared memory:
// As[m][k], Bs[n][k] (real and imaginary parts separately, row stride LDS,
// a pattern free of bank conflicts for the m8n8k4 fragments).
// Warp (wm, wn) in a 2x4 layout owns a 32x16 block: 4 x 2 tiles of 8x8.
// ---------------------------------------------------------------------------
// Complex products by the three-multiplication (Gauss) form: with a = ar + i ai
// and b = br + i bi, the main loops accumulate P1 = sum ar br (in r),
// P2 = sum ai bi (in i) and P3 = sum (ar + ai)(br + bi) (in s), three real MMAs
// per complex product instead of four; finish() turns them into
// Re = P1 - P2 (r) and Im = P3 - P1 - P2 (i).
struct Acc {
  double r[4][2][2];
  double i[4][2][2];
  double s[4][2][2];
  __device__ void zero() {
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        r[a][b][0] = r[a][b][1] = 0.0;
        i[a][b][0] = i[a][b][1] = 0.0;
        s[a][b][0] = s[a][b][1] = 0.0;
      }
  }
  __device__ void finish() {
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const double p1 = r[a][b][e], p2 = i[a][b][e], p3 = s[a][b][e];
          r[a][b][e] = p1 - p2;
          i[a][b][e] = (p3 - p1) - p2;
        }
  }
};

template <bool CONJA>
__device__ __forceinline__ void mma_slice(Acc& acc, const double* Ar, const double* Ai, const double* Br,
                                          const double* Bi, int wm, int wn, int lane) {
  const int r8 = lane >> 2, c4 = lane & 3;
#pragma unroll
  for (int ks = 0; ks < BK / 4; ++ks) {
    double ar[4], ai[4], as[4], br[2], bi[2], bs[2];
#pragma unroll
    for (int mi = 0; mi < 4; ++mi) {
      const int o = (wm * 32 + mi * 8 + r8) * LDS + ks * 4 + c4;
      ar[mi] = Ar[o];
      double t = Ai[o];
      ai[mi] = CONJA ? -t : t;
      as[mi] = ar[mi] + ai[mi];
    }
#pragma unroll
    for (int ni = 0; ni < 2; ++ni) {
      const int o = (wn * 16 + ni * 8 + r8) * LDS + ks * 4 + c4;
      br[ni] = Br[o];
      bi[ni] = Bi[o];
      bs[ni] = br[ni] + bi[ni];
    }
    // three passes over the 8 blocks: the products that add into one
    // accumulator are 24 MMAs apart
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
      for (int ni = 0; ni < 2; ++ni) dmma(acc.r[mi][ni], ar[mi], br[ni]);
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
      for (int ni = 0; ni < 2; ++ni) dmma(acc.i[mi][ni], ai[mi], bi[ni]);
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
      for (int ni = 0; ni < 2; ++ni) dmma(acc.s[mi][ni], as[mi], bs[ni]);
  }
}

// coordinates of accumulator element (mi, ni, e) of this lane
__device__ __forceinline__ void acc_mn(int wm, int wn, int lane, int mi, int ni, int e, int& m, int& n) {
  m = wm * 32 + mi * 8 + (lane >> 2);
  n = wn * 16 + ni * 8 + 2 * (lane & 3) + e;
}

// element e of a thread's share of a 64 x BK tile -> (row, kk)
template <bool KFAST>
__device__ __forceinline__ void tile_rc(int e, int& row, int& kk) {
  if (KFAST) { kk = e % BK; row = e / BK; }
  else { row = e % BM; kk = e / BM; }
}

// Products of the main loop: A0*B0 (+ A1*B0 | + A0*B1 | gram: conj(A0)*B0 and A0*B1)
enum { MP11 = 0, MP21 = 1, MP12 = 2, MPGRAM = 3 };

// Double-buffered main loop over k in [kbeg, kend): the next slice is read from
// global memory into registers while the DMMAs run on the current slice, then
// stored into the other shared-memory stage; one barrier per slice.
// fa0/fa1(row, k) and fb0/fb1(row, k) return the (bounds-checked) operands.
template <int MODE, bool AKF, bool BKF, class FA0, class FA1, class FB0, class FB1>
__device__ __forceinline__ void mainloop(double* sm, int kbeg, int kend, FA0 fa0, FA1 fa1, FB0 fb0, FB1 fb1,
                                         Acc& acc0, Acc& acc1) {
  constexpr int NA = (MODE == MP21) ? 2 : 1;
  constexpr int NBO = (MODE == MP12 || MODE == MPGRAM) ? 2 : 1;
  constexpr int STAGE = 2 * TILE * (NA + NBO);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, wm = warp >> 2, wn = warp & 3;
  double2 ra[NA][EPT], rb[NBO][EPT];
  auto fetch = [&](int k0) {
#pragma unroll
    for (int q = 0; q < EPT; ++q) {
      int row, kk;
      tile_rc<AKF>(tid + q * NT, row, kk);
      ra[0][q] = fa0(row, k0 + kk);
      if (NA == 2) ra[NA - 1][q] = fa1(row, k0 + kk);
      tile_rc<BKF>(tid + q * NT, row, kk);
      rb[0][q] = fb0(row, k0 + kk);
      if (NBO == 2) rb[NBO - 1][q] = fb1(row, k0 + kk);
    }
  };
  auto store = [&](int st) {
    double* base = sm + (size_t)st * STAGE;
#pragma unroll
    for (int q = 0; q < EPT; ++q) {
      int row, kk;
      tile_rc<AKF>(tid + q * NT, row, kk);
#pragma unroll
      for (int x = 0; x < NA; ++x) {
        base[(2 * x) * TILE + row * LDS + kk] = ra[x][q].x;
        base[(2 * x + 1) * TILE + row * LDS + kk] = ra[x][q].y;
      }
      tile_rc<BKF>(tid + q * NT, row, kk);
#pragma unroll
      for (int x = 0; x < NBO; ++x) {
        base[(2 * (NA + x)) * TILE + row * LDS + kk] = rb[x][q].x;
        base[(2 * (NA + x) + 1) * TILE + row * LDS + kk] = rb[x][q].y;
      }
    }
  };
  if (kbeg >= kend) return;
  fetch(kbeg);
  store(0);
  __syncthreads();
  int st = 0;
  for (int k0 = kbeg; k0 < kend; k0 += BK) {
    const bool more = k0 + BK < kend;
    if (more) fetch(k0 + BK);
    const double* base = sm + (size_t)st * STAGE;
    const double* A0r = base;
    const double* A0i = base + TILE;
    const double* B0r = base + 2 * NA * TILE;
    const double* B0i = B0r + TILE;
    if (MODE == MP11) {
      mma_slice<false>(acc0, A0r, A0i, B0r, B0i, wm, wn, lane);
    } else if (MODE == MP21) {
      mma_slice<false>(acc0, A0r, A0i, B0r, B0i, wm, wn, lane);
      mma_slice<false>(acc1, A0r + 2 * TILE, A0i + 2 * TILE, B0r, B0i, wm, wn, lane);
    } else if (MODE == MP12) {
      mma_slice<false>(acc0, A0r, A0i, B0r, B0i, wm, wn, lane);
      mma_slice<false>(acc1, A0r, A0i, B0r + 2 * TILE, B0i + 2 * TILE, wm, wn, lane);
    } else {
      mma_slice<true>(acc0, A0r, A0i, B0r, B0i, wm, wn, lane);
      mma_slice<false>(acc1, A0r, A0i, B0r + 2 * TILE, B0i + 2 * TILE, wm, wn, lane);
    }
    if (more) store(st ^ 1);
    __syncthreads();
    st ^= 1;
  }
  acc0.finish();
  acc1.finish();
}

// ---------------------------------------------------------------------------
// Asynchronous main loop for operands that are plain arrays (or gathers of
// plain elements): every complex element of a K slice goes to shared memory
// by one 16-byte cp.async straight from its address, NS2 slices in flight, so
// no register staging and no load latency in the MMA warps' path.  Tiles
// hold complex elements interleaved, [row][k] at a row stride of LD2 = 20
// (16-byte words), which keeps the m8n8k4 fragment reads free of bank
// conflicts and gives the real and imaginary part of a fragment in one load.
//   pa0/pa1/pb0/pb1(row, k) -> address of the element, or nullptr for zero
//   ca0(k)/ca1(k): conjugate A at global K index k in the product of acc0/acc1
//   CB0/CB1: conjugate B in the product of acc0/acc1
// ---------------------------------------------------------------------------
constexpr int LD2 = 20;
constexpr int LDR = BM + 2;      // [k][row] tiles (row contiguous in global memory)
constexpr int TILE2 = BM * LD2;  // double2 of one operand tile (either layout fits)
static_assert(BK * LDR <= TILE2, "tile layouts");
// offset of element (row, k) of a tile: [row][k] when K is the contiguous
// dimension of the operand in global memory (KF), else [k][row], so that
// consecutive threads' 16-byte copies land in consecutive words either way
template <bool KF>
__device__ __forceinline__ int toff(int row, int k) {
  if constexpr (KF) return row * LD2 + k;
  else return k * LDR + row;
}
constexpr int NS2 = 3;           // K slices in flight

__device__ const double2 g_zero2[1] = {{0.0, 0.0}};

__device__ __forceinline__ void cpa16(double2* dst, const double2* src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src ? src : g_zero2),
               "r"(src ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <bool AKF, bool BKF, bool CB, class CA>
__device__ __forceinline__ void mma_slice2(Acc& acc, const double2* A, const double2* B, int wm, int wn, int lane,
                                           int k0, CA ca) {
  const int r8 = lane >> 2, c4 = lane & 3;
#pragma unroll
  for (int ks = 0; ks < BK / 4; ++ks) {
    const bool cj = ca(k0 + ks * 4 + c4);
    double ar[4], ai[4], as[4], br[2], bi[2], bs[2];
#pragma unroll
    for (int mi = 0; mi < 4; ++mi) {
      const double2 v = A[toff<AKF>(wm * 32 + mi * 8 + r8, ks * 4 + c4)];
      ar[mi] = v.x;
      ai[mi] = cj ? -v.y : v.y;
      as[mi] = ar[mi] + ai[mi];
    }
#pragma unroll
    for (int ni = 0; ni < 2; ++ni) {
      const double2 w = B[toff<BKF>(wn * 16 + ni * 8 + r8, ks * 4 + c4)];
      br[ni] = w.x;
      bi[ni] = CB ? -w.y : w.y;
      bs[ni] = br[ni] + bi[ni];
    }
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
      for (int ni = 0; ni < 2; ++ni) dmma(acc.r[mi][ni], ar[mi], br[ni]);
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
      for (int ni = 0; ni < 2; ++ni) dmma(acc.i[mi][ni], ai[mi], bi[ni]);
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
      for (int ni = 0; ni < 2; ++ni) dmma(acc.s[mi][ni], as[mi], bs[ni]);
  }
}

struct NoConj {
  __device__ __forceinline__ bool operator()(int) const { return false; }
};
struct AllConj {
  __device__ __forceinline__ bool operator()(int) const { return true; }
};

template <int MODE, bool AKF, bool BKF, bool CB0, bool CB1, class PA0, class PA1, class PB0, class PB1, class CA0,
          class CA1>
__device__ __forceinline__ void mainloop2(double2* sm, int kbeg, int kend, PA0 pa0, PA1 pa1, PB0 pb0, PB1 pb1,
                                          CA0 ca0, CA1 ca1, Acc& acc0, Acc& acc1) {
  constexpr int NA = (MODE == MP21) ? 2 : 1;
  constexpr int NBO = (MODE == MP12 || MODE == MPGRAM) ? 2 : 1;
  constexpr int STAGE = TILE2 * (NA + NBO);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, wm = warp >> 2, wn = warp & 3;
  if (kbeg >= kend) return;
  const int nsl = (kend - kbeg + BK - 1) / BK;
  auto issue = [&](int sl) {
    double2* base = sm + (size_t)(sl % NS2) * STAGE;
    const int k0 = kbeg + sl * BK;
#pragma unroll
    for (int q = 0; q < EPT; ++q) {
      int row, kk;
      tile_rc<AKF>(tid + q * NT, row, kk);
      cpa16(base + toff<AKF>(row, kk), pa0(row, k0 + kk));
      if (NA == 2) cpa16(base + TILE2 + toff<AKF>(row, kk), pa1(row, k0 + kk));
      tile_rc<BKF>(tid + q * NT, row, kk);
      cpa16(base + NA * TILE2 + toff<BKF>(row, kk), pb0(row, k0 + kk));
      if (NBO == 2) cpa16(base + (NA + 1) * TILE2 + toff<BKF>(row, kk), pb1(row, k0 + kk));
    }
  };
#pragma unroll
  for (int sl = 0; sl < NS2 - 1; ++sl) {
    if (sl < nsl) issue(sl);
    cpa_commit();
  }
  for (int sl = 0; sl < nsl; ++sl) {
    cpa_wait<NS2 - 2>();
    __syncthreads();
    const double2* base = sm + (size_t)(sl % NS2) * STAGE;
    const int k0 = kbeg + sl * BK;
    const double2* A0 = base;
    const double2* B0 = base + NA * TILE2;
    if (MODE == MP11) {
      mma_slice2<AKF, BKF, CB0>(acc0, A0, B0, wm, wn, lane, k0, ca0);
    } else if (MODE == MP21) {
      mma_slice2<AKF, BKF, CB0>(acc0, A0, B0, wm, wn, lane, k0, ca0);
      mma_slice2<AKF, BKF, CB1>(acc1, A0 + TILE2, B0, wm, wn, lane, k0, ca1);
    } else {
      mma_slice2<AKF, BKF, CB0>(acc0, A0, B0, wm, wn, lane, k0, ca0);
      mma_slice2<AKF, BKF, CB1>(acc1, A0, B0 + TILE2, wm, wn, lane, k0, ca1);
    }
    if (sl + NS2 - 1 < nsl) issue(sl + NS2 - 1);
    cpa_commit();
  }
  cpa_wait<0>();
  __syncthreads();
  acc0.finish();
  acc1.finish();
}

template <int MODE>
constexpr size_t smem2_bytes() {
  return sizeof(double2) * (size_t)NS2 * TILE2 *
         (((MODE == MP21) ? 2 : 1) + ((MODE == MP12 || MODE == MPGRAM) ? 2 : 1));
}

template <int MODE>
constexpr size_t smem_bytes() {
  return sizeof(double) * 2 * 2 * TILE * (((MODE == MP21) ? 2 : 1) + ((MODE == MP12 || MODE == MPGRAM) ? 2 : 1));
}

__device__ __forceinline__ double2 gen_pro(int g, int ngl, const ProDesc& d, const double* __restrict__ ylm,
                                           const double* __restrict__ pro, const double2* __restrict__ eigr) {
  return pro_value(g, ngl, d, ylm, pro, eigr);
}

// ---------------------------------------------------------------------------
// EIGR(g,a) = exp(-i G.R_a)   (PLANEWAVE_STRUCTUREFACTOR, src/paw_fft.f90:1597-1695)
// ---------------------------------------------------------------------------
__global__ void k_eigr(const double* __restrict__ gx, const double* __restrict__ gy, const double* __restrict__ gz,
                       const double* __restrict__ r, int ngl, int nat, double2* __restrict__ eigr) {
  const int a = blockIdx.y;
  const double rx = r[3 * a], ry = r[3 * a + 1], rz = r[3 * a + 2];
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ngl; g += gridDim.x * blockDim.x) {
    double ph = gx[g] * rx + gy[g] * ry + gz[g] * rz;
    double s, c;
    sincos(ph, &s, &c);
    eigr[(size_t)g + (size_t)ngl * a] = make_double2(c, -s);
  }
}

// PRO(g,p) of WAVES_EXPANDPRO for every projector of the present positions
// into prox(LDG, NPRO), zero for NGL <= g < LDG (FP64 handles: the tile
// loaders of the contractions then read whole columns), straight from the
// positions: one thread per (g, atom) forms exp(-iG.R_a) as k_eigr does and
// writes the atom's projectors, so no EIGR array is formed.
__global__ void k_pro_f64_direct(int ngl, int ldg, const double* __restrict__ gx, const double* __restrict__ gy,
                                 const double* __restrict__ gz, const double* __restrict__ r,
                                 const int* __restrict__ ipro0, const int* __restrict__ nlmn,
                                 const ProDesc* __restrict__ pdesc, const double* __restrict__ ylm,
                                 const double* __restrict__ pro, double2* __restrict__ prox) {
  const int a = blockIdx.y;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ldg) return;
  const int p0 = ipro0[a], np = nlmn[a];
  if (g >= ngl) {
    for (int k = 0; k < np; ++k) prox[(size_t)g + (size_t)ldg * (p0 + k)] = make_double2(0.0, 0.0);
    return;
  }
  double sn, cs;
  sincos(gx[g] * r[3 * a] + gy[g] * r[3 * a + 1] + gz[g] * r[3 * a + 2], &sn, &cs);
  const double2 ei = make_double2(cs, -sn);
  for (int k = 0; k < np; ++k) {
    const ProDesc d = pdesc[p0 + k];
    const double sv = ylm[(size_t)g + (size_t)ngl * d.lm] * pro[(size_t)g + (size_t)ngl * d.ibare];
    const double2 e = cmul(mipow(d.l), ei);
    prox[(size_t)g + (size_t)ldg * (p0 + k)] = make_double2(sv * e.x, sv * e.y);
  }
}

__device__ __forceinline__ double2 zero2() { return make_double2(0.0, 0.0); }

// ---------------------------------------------------------------------------
// Projections: part[z][b + nbh*p] = sum_{g in split z} conj(PRO(g,p)) X(g,b)
// for one or two operands X (psiA -> part, psiB -> part + dual_stride).
// M = bands (blockIdx.y), N = projectors (blockIdx.x), K = g (blockIdx.z).
// ---------------------------------------------------------------------------
// TAB: the projector functions come from the expanded table prox(LDG, NPRO)
// of the present positions (FP64 handles) instead of being formed in the loader.
template <bool DUAL, bool TAB>
__global__ void __launch_bounds__(NT, 1) k_proj(const double2* __restrict__ psiA, const double2* __restrict__ psiB,
                                                int ldg, int ngl, int nbh, int npro, int kchunk,
                                                const ProDesc* __restrict__ pdesc, const double* __restrict__ ylm,
                                                const double* __restrict__ pro, const double2* __restrict__ eigr,
                                                double2* __restrict__ part, size_t dual_stride,
                                                const double2* __restrict__ prox = nullptr) {
  extern __shared__ double sm[];
  __shared__ ProDesc sd[BN];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, wm = warp >> 2, wn = warp & 3;
  const int n0 = blockIdx.x * BN, m0 = blockIdx.y * BM;
  const int kbeg = blockIdx.z * kchunk, kend = min(ngl, kbeg + kchunk);
  if (tid < BN) {
    int p = n0 + tid;
    sd[tid] = p < npro ? pdesc[p] : ProDesc{0, 0, 0, 0};
  }
  __syncthreads();
  Acc acc, acc2;
  acc.zero();
  acc2.zero();
  auto fa0 = [&](int row, int g) {
    int b = m0 + row;
    return (g < kend && b < nbh) ? psiA[(size_t)g + (size_t)ldg * b] : zero2();
  };
  auto fa1 = [&](int row, int g) {
    int b = m0 + row;
    return (DUAL && g < kend && b < nbh) ? psiB[(size_t)g + (size_t)ldg * b] : zero2();
  };
  auto fb0 = [&](int row, int g) {
    double2 v = zero2();
    if (g < kend && n0 + row < npro) {
      if constexpr (TAB) v = cconj(prox[(size_t)g + (size_t)ldg * (n0 + row)]);
      else v = cconj(gen_pro(g, ngl, sd[row], ylm, pro, eigr));
    }
    return v;
  };
  if constexpr (TAB) {
    auto pa0 = [&](int row, int g) -> const double2* {
      const int b = m0 + row;
      return (g < kend && b < nbh) ? psiA + (size_t)g + (size_t)ldg * b : nullptr;
    };
    auto pa1 = [&](int row, int g) -> const double2* {
      const int b = m0 + row;
      return (DUAL && g < kend && b < nbh) ? psiB + (size_t)g + (size_t)ldg * b : nullptr;
    };
    auto pb0 = [&](int row, int g) -> const double2* {
      return (g < kend && n0 + row < npro) ? prox + (size_t)g + (size_t)ldg * (n0 + row) : nullptr;
    };
    double2* sm2 = reinterpret_cast<double2*>(sm);
    if (DUAL) mainloop2<MP21, true, true, true, true>(sm2, kbeg, kend, pa0, pa1, pb0, pb0, NoConj(), NoConj(), acc, acc2);
    else mainloop2<MP11, true, true, true, true>(sm2, kbeg, kend, pa0, pa0, pb0, pb0, NoConj(), NoConj(), acc, acc2);
  } else {
    if (DUAL) mainloop<MP21, true, true>(sm, kbeg, kend, fa0, fa1, fb0, fb0, acc, acc2);
    else mainloop<MP11, true, true>(sm, kbeg, kend, fa0, fa0, fb0, fb0, acc, acc2);
  }
  double2* out = part + (size_t)blockIdx.z * nbh * npro;
#pragma unroll
  for (int mi = 0; mi < 4; ++mi)
#pragma unroll
    for (int ni = 0; ni < 2; ++ni)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        int m, n;
        acc_mn(wm, wn, lane, mi, ni, e, m, n);
        int b = m0 + m, p = n0 + n;
        if (b < nbh && p < npro) {
          out[(size_t)b + (size_t)nbh * p] = make_double2(acc.r[mi][ni][e], acc.i[mi][ni][e]);
          if (DUAL) out[dual_stride + (size_t)b + (size_t)nbh * p] = make_double2(acc2.r[mi][ni][e], acc2.i[mi][ni][e]);
        }
      }
}

// out[i] = scale * sum_z part[z*stride + i]   (deterministic order)
__global__ void k_reduce_parts(const double2* __restrict__ part, int nz, size_t stride, size_t n, double scale,
                               double2* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double2 s = make_double2(0.0, 0.0);
    int z = 0;
    for (; z + 8 <= nz; z += 8) {  // eight loads in flight, added in split order
      double2 v[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) v[j] = part[(size_t)(z + j) * stride + i];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        s.x += v[j].x;
        s.y += v[j].y;
      }
    }
    for (; z < nz; ++z) {
      double2 v = part[(size_t)z * stride + i];
      s.x += v.x;
      s.y += v.y;
    }
    out[i] = make_double2(s.x * scale, s.y * scale);
  }
}

// ---------------------------------------------------------------------------
// ADDPRO with the step epilogues.  M = g (blockIdx.x), N = bands (blockIdx.y),
// K = projectors.  Operands C1 (hproj) and/or C2 (oproj), layout (NBH, NPRO).
// mode ADDPRO_HPSI : hpsi += PRO*C1                     (vpsi already in hpsi)
// mode ADDPRO_OPSI : opsi  = (psi0 + PRO*C2) * dt^2/((1+annee) m_G)
// mode ADDPRO_FUSED: both, then psim = a1 psi0 + a2 psim + a3/m_G hpsi
// ---------------------------------------------------------------------------
template <int MODE, bool TAB>
__global__ void __launch_bounds__(NT, 1) k_addpro(double2* __restrict__ hpsi, double2* __restrict__ opsi,
                                                  const double2* __restrict__ psi0, double2* __restrict__ psim,
                                                  const double* __restrict__ mpsi, int ldg, int ngl, int nbh,
                                                  int npro, const double2* __restrict__ c1,
                                                  const double2* __restrict__ c2, const ProDesc* __restrict__ pdesc,
                                                  const double* __restrict__ ylm, const double* __restrict__ pro,
                                                  const double2* __restrict__ eigr, StepCoef sc,
                                                  const double2* __restrict__ prox) {
  constexpr bool USE_H = (MODE != ADDPRO_OPSI);
  constexpr bool USE_O = (MODE != ADDPRO_HPSI);
  extern __shared__ double sm[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, wm = warp >> 2, wn = warp & 3;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  Acc acc, acc2;
  acc.zero();
  acc2.zero();
  auto fa = [&](int row, int p) {
    int g = m0 + row;
    if (!(g < ngl && p < npro)) return zero2();
    if constexpr (TAB) return prox[(size_t)g + (size_t)ldg * p];
    else return gen_pro(g, ngl, pdesc[p], ylm, pro, eigr);
  };
  auto fb1 = [&](int row, int p) {
    int b = n0 + row;
    return (b < nbh && p < npro) ? c1[(size_t)b + (size_t)nbh * p] : zero2();
  };
  auto fb2 = [&](int row, int p) {
    int b = n0 + row;
    return (b < nbh && p < npro) ? c2[(size_t)b + (size_t)nbh * p] : zero2();
  };
  if constexpr (TAB) {
    auto pa = [&](int row, int p) -> const double2* {
      const int g = m0 + row;
      return (g < ngl && p < npro) ? prox + (size_t)g + (size_t)ldg * p : nullptr;
    };
    auto pb1 = [&](int row, int p) -> const double2* {
      const int b = n0 + row;
      return (b < nbh && p < npro) ? c1 + (size_t)b + (size_t)nbh * p : nullptr;
    };
    auto pb2 = [&](int row, int p) -> const double2* {
      const int b = n0 + row;
      return (b < nbh && p < npro) ? c2 + (size_t)b + (size_t)nbh * p : nullptr;
    };
    double2* sm2 = reinterpret_cast<double2*>(sm);
    if (MODE == ADDPRO_FUSED)
      mainloop2<MP12, false, false, false, false>(sm2, 0, npro, pa, pa, pb1, pb2, NoConj(), NoConj(), acc, acc2);
    else if (MODE == ADDPRO_HPSI)
      mainloop2<MP11, false, false, false, false>(sm2, 0, npro, pa, pa, pb1, pb1, NoConj(), NoConj(), acc, acc2);
    else
      mainloop2<MP11, false, false, false, false>(sm2, 0, npro, pa, pa, pb2, pb2, NoConj(), NoConj(), acc2, acc);
  } else {
    if (MODE == ADDPRO_FUSED) mainloop<MP12, false, false>(sm, 0, npro, fa, fa, fb1, fb2, acc, acc2);
    else if (MODE == ADDPRO_HPSI) mainloop<MP11, false, false>(sm, 0, npro, fa, fa, fb1, fb1, acc, acc2);
    else mainloop<MP11, false, false>(sm, 0, npro, fa, fa, fb2, fb2, acc2, acc);
  }
#pragma unroll
  for (int mi = 0; mi < 4; ++mi)
#pragma unroll
    for (int ni = 0; ni < 2; ++ni)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        int m, n;
        acc_mn(wm, wn, lane, mi, ni, e, m, n);
        int g = m0 + m, b = n0 + n;
        if (g >= ngl || b >= nbh) continue;
        size_t k = (size_t)g + (size_t)ldg * b;
        double2 hv = make_double2(0.0, 0.0);
        if (USE_H) {
          hv = hpsi[k];
          hv.x += acc.r[mi][ni][e];
          hv.y += acc.i[mi][ni][e];
          hpsi[k] = hv;
        }
        if (USE_O) {
          double2 p0 = psi0[k];
          double s = sc.oscale / mpsi[g];
          opsi[k] = make_double2((p0.x + acc2.r[mi][ni][e]) * s, (p0.y + acc2.i[mi][ni][e]) * s);
        }
        if (MODE == ADDPRO_FUSED) {
          double2 p0 = psi0[k], pm = psim[k];
          double a1 = sc.a1, a2 = sc.a2, a3 = sc.a3 / mpsi[g];
          if (sc.fr) {  // cell friction ANNEEVEC(G) (src/paw_waves1.f90:6536-6540)
            const double an = 1.0 + sc.fr[g];
            a1 = 2.0 / an;
            a2 = 1.0 - a1;
            a3 = -sc.dt2 / an / mpsi[g];
          }
          psim[k] = make_double2(a1 * p0.x + a2 * pm.x + a3 * hv.x, a1 * p0.y + a2 * pm.y + a3 * hv.y);
        }
      }
}

// ---------------------------------------------------------------------------
// Gram products for one or more (X, Y) pairs (blockIdx.z = split*npair + pair):
//   T1(m,n) = sum_k conj(X(k,m)) Y(k,n)
//   T2(m,n) = sum_k X(k,m) Y(-k,n)    (MINUS: k -> minusg[k])
//           = sum_k X(k,m) Y(k,n)     (otherwise)
// Layout: element (k, m) of an operand at ptr[k*sk + m*sm].
// part[((split*npair + pair)*2 + t)*nm*nn + m + nm*n]
// ---------------------------------------------------------------------------
struct GramArgs {
  GramPair pair[3];
  int npair;
  int nk, nm, nn;   // K, M, N extents
  size_t sk, sm;    // strides of k and of m/n
  int kchunk;
};

template <bool MINUS, bool KFAST>
__global__ void __launch_bounds__(NT, 1) k_gram(GramArgs a, const int* __restrict__ minusg,
                                                double2* __restrict__ part) {
  extern __shared__ double sm[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, wm = warp >> 2, wn = warp & 3;
  const int pair = blockIdx.z % a.npair, split = blockIdx.z / a.npair;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const double2* X = a.pair[pair].x;
  const double2* Y = a.pair[pair].y;
  const int kbeg = split * a.kchunk, kend = min(a.nk, kbeg + a.kchunk);
  Acc t1, t2;
  t1.zero();
  t2.zero();
  auto pa = [&](int row, int k) -> const double2* {
    int m = m0 + row;
    return (k < kend && m < a.nm) ? X + (size_t)k * a.sk + (size_t)m * a.sm : nullptr;
  };
  auto pb = [&](int row, int k) -> const double2* {
    int n = n0 + row;
    return (k < kend && n < a.nn) ? Y + (size_t)k * a.sk + (size_t)n * a.sm : nullptr;
  };
  auto pb2 = [&](int row, int k) -> const double2* {
    int n = n0 + row;
    if (!(k < kend && n < a.nn)) return nullptr;
    int kk = MINUS ? minusg[k] : k;
    return Y + (size_t)kk * a.sk + (size_t)n * a.sm;
  };
  mainloop2<MPGRAM, KFAST, KFAST, false, false>(reinterpret_cast<double2*>(sm), kbeg, kend, pa, pa, pb, pb2,
                                                AllConj(), NoConj(), t1, t2);
  const size_t mn = (size_t)a.nm * a.nn;
  double2* o1 = part + ((size_t)blockIdx.z * 2 + 0) * mn;
  double2* o2 = part + ((size_t)blockIdx.z * 2 + 1) * mn;
#pragma unroll
  for (int mi = 0; mi < 4; ++mi)
#pragma unroll
    for (int ni = 0; ni < 2; ++ni)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        int m, n;
        acc_mn(wm, wn, lane, mi, ni, e, m, n);
        m += m0;
        n += n0;
        if (m < a.nm && n < a.nn) {
          o1[(size_t)m + (size_t)a.nm * n] = make_double2(t1.r[mi][ni][e], t1.i[mi][ni][e]);
          o2[(size_t)m + (size_t)a.nm * n] = make_double2(t2.r[mi][ni][e], t2.i[mi][ni][e]);
        }
      }
}

// ---------------------------------------------------------------------------
//   ADDOPSI form (XMINUS): out(g,n) += sum_k X(g,k) L1(k,n) + conj(X(-g,k)) L2(k,n)
//   ADDOPROJ form       : out(p,n) += sum_k X(p,k) L1(k,n) + conj(X(p,k)) L2(k,n)
// X element (m, k) at X[m*sxm + k*sxk]; out element (m, n) at out[m*som + n*son];
// L1/L2 (nk, nn) column-major complex.  M = blockIdx.x, N = blockIdx.y.
// ---------------------------------------------------------------------------
struct AddXArgs {
  double2* out;
  const double2* x;
  const double2* l1;
  const double2* l2;
  int nm, nn, nk;
  size_t sxm, sxk, som, son;
};

template <bool XMINUS, bool MFAST>
__global__ void __launch_bounds__(NT, 1) k_addx(AddXArgs a, const int* __restrict__ minusg) {
  extern __shared__ double sm[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, wm = warp >> 2, wn = warp & 3;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  Acc acc, dummy;
  acc.zero();
  const int ktot = 2 * a.nk;
  // the second half of K takes conj(X(-g)): conjugated at the fragment read
  auto pa = [&](int row, int kg) -> const double2* {
    int m = m0 + row;
    if (!(m < a.nm && kg < ktot)) return nullptr;
    if (kg < a.nk) return a.x + (size_t)m * a.sxm + (size_t)kg * a.sxk;
    int mm2 = XMINUS ? minusg[m] : m;
    return a.x + (size_t)mm2 * a.sxm + (size_t)(kg - a.nk) * a.sxk;
  };
  auto pb = [&](int row, int kg) -> const double2* {
    int n = n0 + row;
    if (!(n < a.nn && kg < ktot)) return nullptr;
    return kg < a.nk ? a.l1 + (size_t)kg + (size_t)a.nk * n : a.l2 + (size_t)(kg - a.nk) + (size_t)a.nk * n;
  };
  const int nk = a.nk;
  auto second = [nk](int kg) { return kg >= nk; };
  // the outputs' old values (out is not an operand), loaded before the
  // products so that their latency overlaps the MMAs
  double2 old[4][2][2];
#pragma unroll
  for (int mi = 0; mi < 4; ++mi)
#pragma unroll
    for (int ni = 0; ni < 2; ++ni)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        int m, n;
        acc_mn(wm, wn, lane, mi, ni, e, m, n);
        m += m0;
        n += n0;
        old[mi][ni][e] = (m < a.nm && n < a.nn) ? a.out[(size_t)m * a.som + (size_t)n * a.son] : make_double2(0.0, 0.0);
      }
  mainloop2<MP11, !MFAST, true, false, false>(reinterpret_cast<double2*>(sm), 0, ktot, pa, pa, pb, pb, second,
                                              second, acc, dummy);
#pragma unroll
  for (int mi = 0; mi < 4; ++mi)
#pragma unroll
    for (int ni = 0; ni < 2; ++ni)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        int m, n;
        acc_mn(wm, wn, lane, mi, ni, e, m, n);
        m += m0;
        n += n0;
        if (m < a.nm && n < a.nn) {
          size_t k = (size_t)m * a.som + (size_t)n * a.son;
          const double2 o = old[mi][ni][e];
          a.out[k] = make_double2(o.x + acc.r[mi][ni][e], o.y + acc.i[mi][ni][e]);
        }
      }
}

// out(b,p) += sum_k x(k,p) l1(k,b) + conj(x(k,p)) l2(k,b) for (NBH, NPRO)
// arrays with the band index fastest.  A block of 256 threads forms 64 bands
// x 4 projectors, one output per thread with K in order; L1, L2 and x pass
// through shared memory kAopK values of k at a time, copied along k (the
// contiguous index), so that no warp reads L1 or L2 at a stride of NBH.
constexpr int kAopK = 16;
__global__ void k_addoproj(double2* __restrict__ out, const double2* __restrict__ x, const double2* __restrict__ l1,
                           const double2* __restrict__ l2, int npro, int nbh) {
  __shared__ double2 s1[64][kAopK + 1], s2[64][kAopK + 1], sx[4][kAopK];
  const int tb = threadIdx.x & 63, tp = threadIdx.x >> 6;
  const int b0 = blockIdx.y * 64, p0 = blockIdx.x * 4;
  const int b = b0 + tb, p = p0 + tp;
  double sr = 0.0, si = 0.0;
  for (int k0 = 0; k0 < nbh; k0 += kAopK) {
    __syncthreads();  // the previous chunk is consumed
    for (int i = threadIdx.x; i < 64 * kAopK; i += blockDim.x) {
      const int kk = i % kAopK, bb = i / kAopK, k = k0 + kk, bg = b0 + bb;
      const bool ok = k < nbh && bg < nbh;
      s1[bb][kk] = ok ? l1[(size_t)k + (size_t)nbh * bg] : make_double2(0.0, 0.0);
      s2[bb][kk] = ok ? l2[(size_t)k + (size_t)nbh * bg] : make_double2(0.0, 0.0);
    }
    if (threadIdx.x < 4 * kAopK) {
      const int pp = threadIdx.x / kAopK, kk = threadIdx.x % kAopK, k = k0 + kk, pg = p0 + pp;
      sx[pp][kk] = (k < nbh && pg < npro) ? x[(size_t)pg * nbh + k] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    const int kn = min(kAopK, nbh - k0);
    for (int kk = 0; kk < kn; ++kk) {
      const double2 xv = sx[tp][kk], av = s1[tb][kk], cv = s2[tb][kk];
      sr += xv.x * av.x - xv.y * av.y + xv.x * cv.x + xv.y * cv.y;
      si += xv.x * av.y + xv.y * av.x + xv.x * cv.y - xv.y * cv.x;
    }
  }
  if (b < nbh && p < npro) {
    const size_t t = (size_t)b + (size_t)nbh * p;
    const double2 o = out[t];
    out[t] = make_double2(o.x + sr, o.y + si);
  }
}

// ---------------------------------------------------------------------------
// Forces: D(g,p) = sum_b psi0(g,b) conj(E(b,p)); then per projector
//   f_p += Re[ i P(g) (-i)^l EIGR(g) conj(D(g,p)) ] Y_lm(g) G(g)
// reduced over the g tile into fpart[blockIdx.x][p][3].  M = g, N = p, K = b.
// The TINV symmetrisation of WAVES_DEDPRO (src/paw_waves1.f90:5730-5738)
// cancels in this sum (c(-G) = -conj(c(G)) for c = i Y P (-i)^l EIGR over the
// full sphere), so it is not applied.
// ---------------------------------------------------------------------------
template <bool TAB>
__global__ void __launch_bounds__(NT, 1) k_force(const double2* __restrict__ psi0, int ldg, int ngl, int nbh,
                                                 int npro, const double2* __restrict__ ded,
                                                 const ProDesc* __restrict__ pdesc, const double* __restrict__ ylm,
                                                 const double* __restrict__ pro, const double2* __restrict__ eigr,
                                                 const double* __restrict__ gx, const double* __restrict__ gy,
                                                 const double* __restrict__ gz, double* __restrict__ fpart,
                                                 const double2* __restrict__ prox) {
  extern __shared__ double sm[];
  __shared__ double fred[BN][3][2];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, wm = warp >> 2, wn = warp & 3;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  Acc acc, dummy;
  acc.zero();
  auto pa = [&](int row, int b) -> const double2* {
    int g = m0 + row;
    return (g < ngl && b < nbh) ? psi0 + (size_t)g + (size_t)ldg * b : nullptr;
  };
  auto pb = [&](int row, int b) -> const double2* {
    int p = n0 + row;
    return (b < nbh && p < npro) ? ded + (size_t)b + (size_t)nbh * p : nullptr;
  };
  // with the projector table, its values for this tile's outputs are loaded
  // before the products so that their latency overlaps the MMAs
  double2 pvt[4][2][2];
  if constexpr (TAB) {
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
      for (int ni = 0; ni < 2; ++ni)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          int m, n;
          acc_mn(wm, wn, lane, mi, ni, e, m, n);
          const int g = m0 + m, p = n0 + n;
          pvt[mi][ni][e] = (g < ngl && p < npro) ? prox[(size_t)g + (size_t)ldg * p] : make_double2(0.0, 0.0);
        }
  }
  mainloop2<MP11, false, true, true, true>(reinterpret_cast<double2*>(sm), 0, nbh, pa, pa, pb, pb, NoConj(),
                                           NoConj(), acc, dummy);
  // epilogue: per (g, p) contribution, reduced over g
  double f[2][2][3];
#pragma unroll
  for (int ni = 0; ni < 2; ++ni)
#pragma unroll
    for (int e = 0; e < 2; ++e) f[ni][e][0] = f[ni][e][1] = f[ni][e][2] = 0.0;
#pragma unroll
  for (int mi = 0; mi < 4; ++mi)
#pragma unroll
    for (int ni = 0; ni < 2; ++ni)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        int m, n;
        acc_mn(wm, wn, lane, mi, ni, e, m, n);
        int g = m0 + m, p = n0 + n;
        if (g < ngl && p < npro) {
          double2 dd = make_double2(acc.r[mi][ni][e], acc.i[mi][ni][e]);
          double sv;
          if constexpr (TAB) {
            // Re(i PRO(g,p) conj(dd))
            const double2 pv = pvt[mi][ni][e];
            sv = -pv.y * dd.x + pv.x * dd.y;
          } else {
            ProDesc d = pdesc[p];
            double pr = pro[(size_t)g + (size_t)ngl * d.ibare];
            double y = ylm[(size_t)g + (size_t)ngl * d.lm];
            // cw = i * P * (-i)^l * EIGR
            double2 cw = cmul(make_double2(0.0, pr), cmul(mipow(d.l), eigr[(size_t)g + (size_t)ngl * d.iat]));
            sv = (cw.x * dd.x + cw.y * dd.y) * y;  // Re(cw * conj(dd)) * Y
          }
          f[ni][e][0] += sv * gx[g];
          f[ni][e][1] += sv * gy[g];
          f[ni][e][2] += sv * gz[g];
        }
      }
  // reduce across the 8 lanes that share (lane & 3) (different g rows)
#pragma unroll
  for (int ni = 0; ni < 2; ++ni)
#pragma unroll
    for (int e = 0; e < 2; ++e)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double v = f[ni][e][c];
        v += __shfl_xor_sync(0xffffffffu, v, 4);
        v += __shfl_xor_sync(0xffffffffu, v, 8);
        v += __shfl_xor_sync(0xffffffffu, v, 16);
        f[ni][e][c] = v;
      }
  if (lane < 4) {
#pragma unroll
    for (int ni = 0; ni < 2; ++ni)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        int n = wn * 16 + ni * 8 + 2 * lane + e;
#pragma unroll
        for (int c = 0; c < 3; ++c) fred[n][c][wm] = f[ni][e][c];
      }
  }
  __syncthreads();
  for (int i = tid; i < BN * 3; i += NT) {
    int n = i / 3, c = i % 3;
    int p = n0 + n;
    if (p < npro) fpart[((size_t)blockIdx.x * npro + p) * 3 + c] = fred[n][c][0] + fred[n][c][1];
  }
}

// Persistent form of k_force for the projector table and NBH <= 64: the
// force contraction has a short K (the bands), so a CTA per output tile spends
// most of its time filling its pipeline.  Here CTA (gi, pj) keeps the DEDPRO
// tile of projector tile pj (all K) resident in shared memory and walks the G
// tiles gi, gi + gstride, ...: the psi rows of the next G tile are copied
// (16-byte cp.async) while the current one is multiplied and its epilogue
// runs, and the G-weighted sums of every projector accumulate in registers
// over all the CTA's tiles.  fpart(gi, p, c) then holds the CTA's partial sum.
constexpr int kFpSlices = 4;                 // K slices of BK (NBH <= 64)
constexpr int kFpASlice = BK * LDR;          // double2 of one [k][row] psi slice
constexpr size_t kFpSmem = sizeof(double2) * ((size_t)kFpSlices * TILE2 + 2 * (size_t)kFpSlices * kFpASlice);
__global__ void __launch_bounds__(NT, 1) k_force_p(const double2* __restrict__ psi0, int ldg, int ngl, int nbh,
                                                   int npro, const double2* __restrict__ ded,
                                                   const double* __restrict__ gx, const double* __restrict__ gy,
                                                   const double* __restrict__ gz, double* __restrict__ fpart,
                                                   const double2* __restrict__ prox, int gstride) {
  extern __shared__ double sm[];
  __shared__ double fred[BN][3][2];
  double2* bsm = reinterpret_cast<double2*>(sm);  // [slice][TILE2], DEDPRO (row = projector, k = band)
  double2* asm_ = bsm + kFpSlices * TILE2;        // [buffer][slice][kFpASlice], psi (k = band, row = G)
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, wm = warp >> 2, wn = warp & 3;
  const int gi = blockIdx.x, n0 = blockIdx.y * BN;
  const int tm = (ngl + BM - 1) / BM;
  const int nsl = (nbh + BK - 1) / BK;
  // resident DEDPRO tile
  for (int sl = 0; sl < nsl; ++sl)
#pragma unroll
    for (int q = 0; q < EPT; ++q) {
      int row, kk;
      tile_rc<true>(tid + q * NT, row, kk);
      const int b = sl * BK + kk, pr = n0 + row;
      cpa16(bsm + sl * TILE2 + toff<true>(row, kk), (b < nbh && pr < npro) ? ded + b + (size_t)nbh * pr : nullptr);
    }
  auto issue_a = [&](int t, int buf) {
    const int m0 = t * BM;
    for (int sl = 0; sl < nsl; ++sl)
#pragma unroll
      for (int q = 0; q < EPT; ++q) {
        int row, kk;
        tile_rc<false>(tid + q * NT, row, kk);
        const int g = m0 + row, b = sl * BK + kk;
        cpa16(asm_ + ((size_t)buf * kFpSlices + sl) * kFpASlice + toff<false>(row, kk),
              (g < ngl && b < nbh) ? psi0 + (size_t)g + (size_t)ldg * b : nullptr);
      }
  };
  if (gi < tm) issue_a(gi, 0);
  cpa_commit();
  double f[2][2][3];
#pragma unroll
  for (int ni = 0; ni < 2; ++ni)
#pragma unroll
    for (int e = 0; e < 2; ++e) f[ni][e][0] = f[ni][e][1] = f[ni][e][2] = 0.0;
  int buf = 0;
  for (int t = gi; t < tm; t += gstride, buf ^= 1) {
    if (t + gstride < tm) issue_a(t + gstride, buf ^ 1);
    cpa_commit();
    cpa_wait<1>();  // this tile's psi rows (and the DEDPRO tile) have landed
    __syncthreads();
    const int m0 = t * BM;
    // the projector-table values of this tile's outputs, loaded before the
    // products so that their latency overlaps the MMAs
    double2 pvt[4][2][2];
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
      for (int ni = 0; ni < 2; ++ni)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          int m, n;
          acc_mn(wm, wn, lane, mi, ni, e, m, n);
          const int g = m0 + m, p = n0 + n;
          pvt[mi][ni][e] = (g < ngl && p < npro) ? prox[(size_t)g + (size_t)ldg * p] : make_double2(0.0, 0.0);
        }
    Acc acc;
    acc.zero();
    for (int sl = 0; sl < nsl; ++sl)
      mma_slice2<false, true, true>(acc, asm_ + ((size_t)buf * kFpSlices + sl) * kFpASlice, bsm + sl * TILE2, wm,
                                    wn, lane, sl * BK, NoConj());
    acc.finish();
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
      for (int ni = 0; ni < 2; ++ni)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          int m, n;
          acc_mn(wm, wn, lane, mi, ni, e, m, n);
          const int g = m0 + m, p = n0 + n;
          if (g < ngl && p < npro) {
            // Re(i PRO(g,p) conj(dd))
            const double2 pv = pvt[mi][ni][e];
            const double sv = -pv.y * acc.r[mi][ni][e] + pv.x * acc.i[mi][ni][e];
            f[ni][e][0] += sv * gx[g];
            f[ni][e][1] += sv * gy[g];
            f[ni][e][2] += sv * gz[g];
          }
        }
    __syncthreads();  // the buffer is free for the copies of the tile after next
  }
  cpa_wait<0>();
  // reduce across the 8 lanes that share (lane & 3) (different g rows)
#pragma unroll
  for (int ni = 0; ni < 2; ++ni)
#pragma unroll
    for (int e = 0; e < 2; ++e)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double v = f[ni][e][c];
        v += __shfl_xor_sync(0xffffffffu, v, 4);
        v += __shfl_xor_sync(0xffffffffu, v, 8);
        v += __shfl_xor_sync(0xffffffffu, v, 16);
        f[ni][e][c] = v;
      }
  if (lane < 4) {
#pragma unroll
    for (int ni = 0; ni < 2; ++ni)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        int n = wn * 16 + ni * 8 + 2 * lane + e;
#pragma unroll
        for (int c = 0; c < 3; ++c) fred[n][c][wm] = f[ni][e][c];
      }
  }
  __syncthreads();
  for (int i = tid; i < BN * 3; i += NT) {
    int n = i / 3, c = i % 3;
    int p = n0 + n;
    if (p < npro) fpart[((size_t)gi * npro + p) * 3 + c] = fred[n][c][0] + fred[n][c][1];
  }
}

// force(c, iat) = 2 * Omega * sum over g tiles and projectors of atom iat;
// one block per (component, atom), fixed-order tree reduction
__global__ void k_force_final(const double* __restrict__ fpart, int ntile, int npro, const int* __restrict__ ipro0,
                              const int* __restrict__ nlmn, int nat, double gweight, double* __restrict__ force) {
  const int c = blockIdx.x, a = blockIdx.y;
  const int p0 = ipro0[a], np = nlmn[a];
  const int total = ntile * np;
  double s = 0.0;
  for (int k = threadIdx.x; k < total; k += blockDim.x) {
    int t = k / np, p = p0 + k % np;
    s += fpart[((size_t)t * npro + p) * 3 + c];
  }
  __shared__ double red[128];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 64; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) force[3 * a + c] = gweight * 2.0 * red[0];
}

// ---------------------------------------------------------------------------
// one-centre operations on projections (small, one thread per output)
// HPROJ = DH * PROJ per atom (WAVES_HPROJ, src/paw_waves1.f90:4919-4973)
// OPROJ = DO * PROJ per atom (WAVES_OPROJ, src/paw_waves2.f90:497-544)
// ---------------------------------------------------------------------------
// HPROJ(b,p) = sum_l2 DH(l1,l2,atom) PROJ(b, atom's l2) for output i = b + NBH p
__device__ __forceinline__ void hproj_at(size_t i, const double2* __restrict__ proj, const double2* __restrict__ dh,
                                         int lmnxx, const ProDesc* __restrict__ pdesc, const int* __restrict__ ipro0,
                                         const int* __restrict__ nlmn, int nbh, double2* __restrict__ out) {
  int b = (int)(i % nbh), p = (int)(i / nbh);
  int a = pdesc[p].iat;
  int l1 = p - ipro0[a];
  double2 s = make_double2(0.0, 0.0);
  for (int l2 = 0; l2 < nlmn[a]; ++l2) {
    double2 d = dh[(size_t)l1 + (size_t)lmnxx * (l2 + (size_t)lmnxx * a)];
    double2 c = proj[(size_t)b + (size_t)nbh * (ipro0[a] + l2)];
    s = cadd(s, cmul(d, c));
  }
  out[i] = s;
}

__global__ void k_hproj(const double2* __restrict__ proj, const double2* __restrict__ dh, int lmnxx,
                        const ProDesc* __restrict__ pdesc, const int* __restrict__ ipro0,
                        const int* __restrict__ nlmn, int nbh, int npro, double2* __restrict__ out) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= (size_t)nbh * npro) return;
  hproj_at(i, proj, dh, lmnxx, pdesc, ipro0, nlmn, nbh, out);
}

// OPROJ(b,p) = sum over the atom's projectors of equal l and m of DO(ln1,ln2) PROJ
__device__ __forceinline__ void oproj_at(size_t i, const double2* __restrict__ proj, const double* __restrict__ dover,
                                         int lnxx, const ProDesc* __restrict__ pdesc, const int* __restrict__ ipro0,
                                         const int* __restrict__ isp, const int* __restrict__ lnofp,
                                         const int* __restrict__ mofp, const int* __restrict__ lmn0ln,
                                         const int* __restrict__ lox, int maxln, int nbh, double2* __restrict__ out) {
  int b = (int)(i % nbh), p = (int)(i / nbh);
  int a = pdesc[p].iat, s = isp[a];
  int ln1 = lnofp[p], m = mofp[p], l1 = pdesc[p].l;
  double2 acc = make_double2(0.0, 0.0);
  for (int ln2 = 0; ln2 < maxln; ++ln2) {
    int l2 = lox[s * maxln + ln2];
    if (l2 < 0) break;
    if (l2 != l1) continue;
    double dv = dover[(size_t)ln1 + (size_t)lnxx * (ln2 + (size_t)lnxx * s)];
    double2 c = proj[(size_t)b + (size_t)nbh * (ipro0[a] + lmn0ln[s * maxln + ln2] + m)];
    acc.x += dv * c.x;
    acc.y += dv * c.y;
  }
  out[i] = acc;
}

__global__ void k_oproj(const double2* __restrict__ proj, const double* __restrict__ dover, int lnxx,
                        const ProDesc* __restrict__ pdesc, const int* __restrict__ ipro0, const int* __restrict__ isp,
                        const int* __restrict__ lnofp, const int* __restrict__ mofp, const int* __restrict__ lmn0ln,
                        const int* __restrict__ lox, int maxln, int nbh, int npro, double2* __restrict__ out) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= (size_t)nbh * npro) return;
  oproj_at(i, proj, dover, lnxx, pdesc, ipro0, isp, lnofp, mofp, lmn0ln, lox, maxln, nbh, out);
}

// HPROJ and OPROJ of the same PROJ in one launch (the step's back-projection
// needs both)
__global__ void k_hoproj(const double2* __restrict__ proj, const double2* __restrict__ dh, int lmnxx,
                         const double* __restrict__ dover, int lnxx, const ProDesc* __restrict__ pdesc,
                         const int* __restrict__ ipro0, const int* __restrict__ nlmn, const int* __restrict__ isp,
                         const int* __restrict__ lnofp, const int* __restrict__ mofp, const int* __restrict__ lmn0ln,
                         const int* __restrict__ lox, int maxln, int nbh, int npro, double2* __restrict__ hout,
                         double2* __restrict__ oout) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= (size_t)nbh * npro) return;
  hproj_at(i, proj, dh, lmnxx, pdesc, ipro0, nlmn, nbh, hout);
  oproj_at(i, proj, dover, lnxx, pdesc, ipro0, isp, lnofp, mofp, lmn0ln, lox, maxln, nbh, oout);
}

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

int ensure_part(Handle* h, size_t bytes) {
  if (bytes <= h->g.part_bytes) return CUW_OK;
  // (a step being captured into a graph runs again uncaptured instead)
  if (h->capturing) return h->fail(CUW_ERR_STATE, "scratch grows during graph capture");
  h->touch();  // graphs hold the old buffer
  if (h->g.part) cudaFree(h->g.part);
  h->g.part = nullptr;
  h->g.part_bytes = 0;
  CUW_TRY(cudaMalloc(&h->g.part, bytes));
  h->g.part_bytes = bytes;
  return CUW_OK;
}

static int choose_split(Handle* h, int tiles, int nk, int minchunk, double mul) {
  // at most 2 mul waves of one CTA per SM (rounded down: a CTA past a whole
  // wave would cost a wave of its own)
  int want = std::max(1, (int)std::floor(2.0 * h->nsm * mul / std::max(1, tiles)));
  int maxs = std::max(1, ceil_div(nk, minchunk));
  return std::min(want, maxs);
}

int eigr_compute(Handle* h, const double* r_dev) {
  // EIGR (and the fp32 projector table) of the positions in a position buffer
  // stay current until that buffer is written: R(+) of one step is R(0) of the
  // next
  const bool pos = r_dev == h->g.r0 || r_dev == h->g.rp || r_dev == h->g.rm;
  if (pos && r_dev == h->eigr_src) return CUW_OK;
  h->eigr_src = nullptr;
  if (!h->mixed() && h->npro > 0) {
    // FP64 handles: the expanded projector table straight from the positions
    // (the contractions read only the table, so EIGR is not formed)
    if (!h->g.prox) {
      if (h->capturing) return h->fail(CUW_ERR_STATE, "projector table allocated during graph capture");
      h->touch();
      CUW_TRY(cudaMalloc(&h->g.prox, sizeof(double2) * (size_t)h->ldg * h->npro));
    }
    const Device& g = h->g;
    k_pro_f64_direct<<<dim3(ceil_div(h->ldg, 256), h->d.nat), 256, 0, h->stream>>>(
        h->d.ngl, h->ldg, g.gx, g.gy, g.gz, r_dev, g.t_ipro0, g.t_nlmn, g.pdesc, g.ylm, g.pro, g.prox);
    CUW_LAUNCH_CHECK("k_pro_f64_direct");
  } else {
    dim3 grid(std::min(ceil_div(h->d.ngl, 256), 64), h->d.nat);
    k_eigr<<<grid, 256, 0, h->stream>>>(h->g.gx, h->g.gy, h->g.gz, r_dev, h->d.ngl, h->d.nat, h->g.eigr);
    CUW_LAUNCH_CHECK("k_eigr");
    if (h->mixed()) CUW_RET(tc_pro_table(h));
  }
  if (pos) h->eigr_src = r_dev;
  return CUW_OK;
}

// projA = Omega <p|psiA>, projB likewise when psiB != null; uses h->g.eigr
int proj_compute(Handle* h, const double2* psiA, double2* projA, const double2* psiB, double2* projB) {
  if (h->tc_on()) {
    CUW_RET(tc_proj(h, psiA, projA));
    return psiB ? tc_proj(h, psiB, projB) : CUW_OK;
  }
  const int nbh = h->d.nbh, npro = h->npro, ngl = h->d.ngl;
  const int tn = ceil_div(npro, BN), tm = ceil_div(nbh, BM);
  int ks = choose_split(h, tn * tm, ngl, 256, h->split_proj);
  int kchunk = ceil_div(ceil_div(ngl, ks), BK) * BK;
  ks = ceil_div(ngl, kchunk);
  const size_t one = (size_t)ks * nbh * npro;
  const bool dual = (psiB != nullptr);
  CUW_RET(ensure_part(h, sizeof(double2) * one * (dual ? 2 : 1)));
  dim3 grid(tn, tm, ks);
  // FP64 handles read the expanded projector table; the FP64 products of a
  // mixed handle (start-up orthonormalisation, orthonormality test) form it
  const bool tab = !h->mixed() && h->g.prox;
  const Device& g = h->g;
  if (dual && tab)
    k_proj<true, true><<<grid, NT, smem2_bytes<MP21>(), h->stream>>>(psiA, psiB, h->ldg, ngl, nbh, npro, kchunk,
                                                                   g.pdesc, g.ylm, g.pro, g.eigr, g.part, one,
                                                                   g.prox);
  else if (dual)
    k_proj<true, false><<<grid, NT, smem_bytes<MP21>(), h->stream>>>(psiA, psiB, h->ldg, ngl, nbh, npro, kchunk,
                                                                    g.pdesc, g.ylm, g.pro, g.eigr, g.part, one);
  else if (tab)
    k_proj<false, true><<<grid, NT, smem2_bytes<MP11>(), h->stream>>>(psiA, nullptr, h->ldg, ngl, nbh, npro, kchunk,
                                                                    g.pdesc, g.ylm, g.pro, g.eigr, g.part, 0,
                                                                    g.prox);
  else
    k_proj<false, false><<<grid, NT, smem_bytes<MP11>(), h->stream>>>(psiA, nullptr, h->ldg, ngl, nbh, npro, kchunk,
                                                                     g.pdesc, g.ylm, g.pro, g.eigr, g.part, 0);
  CUW_LAUNCH_CHECK("k_proj");
  const size_t n = (size_t)nbh * npro;
  const int rb = std::min(ceil_div((int)std::min<size_t>(n, 1 << 30), 256), 4 * h->nsm);
  k_reduce_parts<<<rb, 256, 0, h->stream>>>(h->g.part, ks, n, n, h->gweight, projA);
  CUW_LAUNCH_CHECK("k_reduce_parts");
  if (dual) {
    k_reduce_parts<<<rb, 256, 0, h->stream>>>(h->g.part + one, ks, n, n, h->gweight, projB);
    CUW_LAUNCH_CHECK("k_reduce_parts");
  }
  return CUW_OK;
}

int addpro_run(Handle* h, int mode, const double2* hpc, const double2* opc) {
  const int ngl = h->d.ngl, nbh = h->d.nbh, npro = h->npro;
  dim3 grid(ceil_div(ngl, BM), ceil_div(nbh, BN));
  StepCoef sc;
  sc.a1 = 2.0 / (1.0 + h->annee);  // WAVES$PROPAGATE (src/paw_waves1.f90:6557-6566)
  sc.a2 = 1.0 - sc.a1;
  sc.a3 = -h->delt * h->delt / (1.0 + h->annee);
  sc.oscale = h->delt * h->delt / (1.0 + h->annee);  // src/paw_waves2.f90:148-156
  sc.fr = h->fric_on ? h->g.anv : nullptr;
  sc.dt2 = h->delt * h->delt;
  if (h->tc_on()) return tc_addpro(h, mode, hpc, opc, sc);
  Device& g = h->g;
  const bool tab = !h->mixed() && g.prox;
#define CUW_ADDPRO(MODE_, MP_)                                                                                  \
  (tab ? k_addpro<MODE_, true><<<grid, NT, smem2_bytes<MP_>(), h->stream>>>(                                      \
             g.hpsi, g.opsi, g.psi0, g.psim, g.mpsi, h->ldg, ngl, nbh, npro, hpc, opc, g.pdesc, g.ylm, g.pro,    \
             g.eigr, sc, g.prox)                                                                                 \
       : k_addpro<MODE_, false><<<grid, NT, smem_bytes<MP_>(), h->stream>>>(                                     \
             g.hpsi, g.opsi, g.psi0, g.psim, g.mpsi, h->ldg, ngl, nbh, npro, hpc, opc, g.pdesc, g.ylm, g.pro,    \
             g.eigr, sc, nullptr))
  switch (mode) {
    case ADDPRO_HPSI: CUW_ADDPRO(ADDPRO_HPSI, MP11); break;
    case ADDPRO_OPSI: CUW_ADDPRO(ADDPRO_OPSI, MP11); break;
    default: CUW_ADDPRO(ADDPRO_FUSED, MP12);
  }
#undef CUW_ADDPRO
  CUW_LAUNCH_CHECK("k_addpro");
  return CUW_OK;
}

// tables of the projector map on the device (Device::t_*)
struct TabView {
  const int *ipro0, *nlmn, *isp, *lnofp, *mofp, *lmn0ln, *lox;
};
static TabView tables(Handle* h) {
  const Device& g = h->g;
  return TabView{g.t_ipro0, g.t_nlmn, g.t_isp, g.t_lnofp, g.t_mofp, g.t_lmn0ln, g.t_lox};
}

// WAVES_DENMAT (src/paw_waves1.f90:3331-3572) for super wave functions (TINV,
// NDIM=1), one block per atom: the one-centre density matrix
//   D(l1,l2) = Re sum_ib P(ib,l1) (s1 conj P(ib,l2) + s2 P(ib,l2)),
//   s1,2 = (f(2ib-1) +- f(2ib))/2                                   (:3384-3412)
// and the energy-weighted E(l1,l2) = Re sum_ib1 conj P(ib1,l1) FUNC_ib1(l2) with
// FUNC_ib1 = sum_ib2 c1 P(ib2,.) + c2 conj P(ib2,.) from LAGR = RLAM0 * OCC
// (:3416-3449); both then Hermitian (:3525-3540, a symmetric average of real
// matrices) and real.  P(ib,l) = PROJ(ib, ipro0 + l).  Sums in band order.
__global__ void k_denmat(const double2* __restrict__ proj, const double2* __restrict__ rlam0,
                         const double* __restrict__ occ, const int* __restrict__ ipro0, const int* __restrict__ nlmn,
                         int nb, int nbh, int lmnxx, double2* __restrict__ denmat, double2* __restrict__ edenmat) {
  extern __shared__ double dsm[];
  const int a = blockIdx.x, lmnx = nlmn[a], p0 = ipro0[a];
  double* d1 = dsm;                   // [lmnx][lmnx]
  double* e1 = dsm + lmnx * lmnx;     // [lmnx][lmnx]
  auto P = [&](int ib, int l) { return proj[(size_t)ib + (size_t)nbh * (p0 + l)]; };
  auto L = [&](int i, int j) {  // LAGR(i,j) = LAMBDA(i,j) OCC(j), 1-based
    const double2 v = rlam0[(size_t)(i - 1) + (size_t)nb * (j - 1)];
    return make_double2(v.x * occ[j - 1], v.y * occ[j - 1]);
  };
  for (int t = threadIdx.x; t < lmnx * lmnx; t += blockDim.x) {
    const int l1 = t % lmnx, l2 = t / lmnx;
    double d = 0.0;
    for (int ib = 0; ib < nbh; ++ib) {
      const double f1 = occ[2 * ib], f2 = 2 * ib + 1 < nb ? occ[2 * ib + 1] : 0.0;
      const double s1 = 0.5 * (f1 + f2), s2 = 0.5 * (f1 - f2);
      const double2 a1 = P(ib, l1), a2 = P(ib, l2);
      // Re[a1 (s1 conj a2 + s2 a2)]
      d += s1 * (a1.x * a2.x + a1.y * a2.y) + s2 * (a1.x * a2.x - a1.y * a2.y);
    }
    double e = 0.0;
    if (edenmat) {
      for (int ib1 = 1; ib1 <= nbh; ++ib1) {
        double2 fu = make_double2(0.0, 0.0);
        for (int ib2 = 1; ib2 <= nbh; ++ib2) {
          const double2 r1 = L(2 * ib1 - 1, 2 * ib2 - 1), r2 = L(2 * ib1, 2 * ib2 - 1);
          const double2 i1 = L(2 * ib1 - 1, 2 * ib2), i2 = L(2 * ib1, 2 * ib2);
          const double2 cr = make_double2(r1.x - r2.y, r1.y + r2.x);  // r1 + i r2
          const double2 ci = make_double2(i1.x - i2.y, i1.y + i2.x);  // i1 + i i2
          // c1 = (cr - i ci)/2, c2 = (cr + i ci)/2
          const double2 c1 = make_double2(0.5 * (cr.x + ci.y), 0.5 * (cr.y - ci.x));
          const double2 c2 = make_double2(0.5 * (cr.x - ci.y), 0.5 * (cr.y + ci.x));
          const double2 p = P(ib2 - 1, l2);
          fu.x += c1.x * p.x - c1.y * p.y + c2.x * p.x + c2.y * p.y;
          fu.y += c1.x * p.y + c1.y * p.x - c2.x * p.y + c2.y * p.x;
        }
        const double2 q = P(ib1 - 1, l1);
        e += q.x * fu.x + q.y * fu.y;  // Re[conj q fu]
      }
    }
    d1[l1 + lmnx * l2] = d;
    e1[l1 + lmnx * l2] = e;
  }
  __syncthreads();
  const size_t per = (size_t)lmnxx * lmnxx;
  for (int t = threadIdx.x; t < lmnxx * lmnxx; t += blockDim.x) {
    const int l1 = t % lmnxx, l2 = t / lmnxx;
    double dv = 0.0, ev = 0.0;
    if (l1 < lmnx && l2 < lmnx) {
      dv = l1 == l2 ? d1[l1 + lmnx * l2] : 0.5 * (d1[l1 + lmnx * l2] + d1[l2 + lmnx * l1]);
      ev = l1 == l2 ? e1[l1 + lmnx * l2] : 0.5 * (e1[l1 + lmnx * l2] + e1[l2 + lmnx * l1]);
    }
    denmat[per * a + t] = make_double2(dv, 0.0);
    if (edenmat) edenmat[per * a + t] = make_double2(ev, 0.0);
  }
}

int denmat_run(Handle* h, int lmnxx, double2* denmat, double2* edenmat) {
  if (h->d.nat == 0) return CUW_OK;
  TabView t = tables(h);
  const size_t smem = sizeof(double) * 2 * (size_t)h->lmnxx * h->lmnxx;
  k_denmat<<<h->d.nat, 128, smem, h->stream>>>(h->g.proj, h->g.rlam0, h->g.occ, t.ipro0, t.nlmn, h->d.nb, h->d.nbh,
                                                lmnxx, denmat, edenmat);
  CUW_LAUNCH_CHECK("k_denmat");
  return CUW_OK;
}

int hproj_compute(Handle* h, const double2* proj, double2* out) {
  TabView t = tables(h);
  size_t n = (size_t)h->d.nbh * h->npro;
  k_hproj<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(proj, h->g.dh, h->lmnxx, h->g.pdesc, t.ipro0, t.nlmn,
                                                              h->d.nbh, h->npro, out);
  CUW_LAUNCH_CHECK("k_hproj");
  return CUW_OK;
}

int hoproj_compute(Handle* h, const double2* proj, double2* hout, double2* oout) {
  TabView t = tables(h);
  size_t n = (size_t)h->d.nbh * h->npro;
  k_hoproj<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(proj, h->g.dh, h->lmnxx, h->g.dover, h->lnxx, h->g.pdesc,
                                                               t.ipro0, t.nlmn, t.isp, t.lnofp, t.mofp, t.lmn0ln, t.lox,
                                                               CUW_MAXLN, h->d.nbh, h->npro, hout, oout);
  CUW_LAUNCH_CHECK("k_hoproj");
  return CUW_OK;
}

int oproj_compute(Handle* h, const double2* proj, double2* out) {
  TabView t = tables(h);
  size_t n = (size_t)h->d.nbh * h->npro;
  k_oproj<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(proj, h->g.dover, h->lnxx, h->g.pdesc, t.ipro0, t.isp,
                                                              t.lnofp, t.mofp, t.lmn0ln, t.lox, CUW_MAXLN, h->d.nbh,
                                                              h->npro, out);
  CUW_LAUNCH_CHECK("k_oproj");
  return CUW_OK;
}

// T(pair) products into h->g.part region [pair][t][nbh*nbh] after reduction at
// offset `dst` (complex), scaled by `scale`.
static int gram_run(Handle* h, const GramPair* pairs, int npair, bool minus, int nk, int nm, size_t sk, size_t sm,
                    double scale, double2* dst) {
  if (h->tc_on()) return tc_gram(h, pairs, npair, minus, nk, nm, sk, sm, scale, dst);
  GramArgs a;
  for (int i = 0; i < npair; ++i) a.pair[i] = pairs[i];
  a.npair = npair;
  a.nk = nk;
  a.nm = nm;
  a.nn = nm;
  a.sk = sk;
  a.sm = sm;
  const int tiles = ceil_div(nm, BM) * ceil_div(nm, BN) * npair;
  int ks = choose_split(h, tiles, nk, 128, h->split_gram);
  a.kchunk = ceil_div(ceil_div(nk, ks), BK) * BK;
  ks = ceil_div(nk, a.kchunk);
  const size_t mn = (size_t)nm * nm;
  CUW_RET(ensure_part(h, sizeof(double2) * mn * 2 * npair * ks));
  dim3 grid(ceil_div(nm, BN), ceil_div(nm, BM), ks * npair);
  if (minus) k_gram<true, true><<<grid, NT, smem2_bytes<MPGRAM>(), h->stream>>>(a, h->g.minusg, h->g.part);
  else k_gram<false, false><<<grid, NT, smem2_bytes<MPGRAM>(), h->stream>>>(a, h->g.minusg, h->g.part);
  CUW_LAUNCH_CHECK("k_gram");
  // reduce over splits: layout part[(split*npair+pair)*2+t] -> dst[(pair*2+t)]
  const size_t n = mn * 2 * npair;
  const int rb = std::min(ceil_div((int)n, 256), 4 * h->nsm);
  k_reduce_parts<<<rb, 256, 0, h->stream>>>(h->g.part, ks, n, n, scale, dst);
  CUW_LAUNCH_CHECK("k_reduce_parts");
  return CUW_OK;
}

int gram_planewave(Handle* h, const GramPair* pairs, int npair, double2* dst) {
  return gram_run(h, pairs, npair, true, h->d.ngl, h->d.nbh, 1, (size_t)h->ldg, h->gweight, dst);
}

int gram_projections(Handle* h, const GramPair* pairs, int npair, double2* dst) {
  return gram_run(h, pairs, npair, false, h->npro, h->d.nbh, (size_t)h->d.nbh, 1, 1.0, dst);
}

int addopsi_run(Handle* h, double2* psibar, const double2* opsi, const double2* l1, const double2* l2) {
  AddXArgs a;
  a.out = psibar;
  a.x = opsi;
  a.l1 = l1;
  a.l2 = l2;
  a.nm = h->d.ngl;
  a.nn = h->d.nbh;
  a.nk = h->d.nbh;
  a.sxm = 1;
  a.sxk = (size_t)h->ldg;
  a.som = 1;
  a.son = (size_t)h->ldg;
  if (h->tc_on()) return tc_addx(h, true, a.out, a.x, a.l1, a.l2, a.nm, a.nn, a.nk, a.sxm, a.sxk, a.som, a.son);
  dim3 grid(ceil_div(a.nm, BM), ceil_div(a.nn, BN));
  k_addx<true, true><<<grid, NT, smem2_bytes<MP11>(), h->stream>>>(a, h->g.minusg);
  CUW_LAUNCH_CHECK("k_addx");
  return CUW_OK;
}

// ADDOPROJ for the (NBH, NPRO) projection arrays (src/paw_waves2.f90:687-758):
// PROJ(b,p) += sum_k OPROJ(k,p) L1(k,b) + conj(OPROJ(k,p)) L2(k,b), in FP64 on
// both paths.  The product is small (NPRO x NBH outputs, K = NBH), so one
// thread per output with K in order beats a tiled GEMM, whose few CTAs
// mostly fill and drain their pipeline.
int addoproj_run(Handle* h, double2* proj, const double2* oproj, const double2* l1, const double2* l2) {
  const int n = h->npro * h->d.nbh;
  if (n == 0) return CUW_OK;
  k_addoproj<<<dim3(ceil_div(h->npro, 4), ceil_div(h->d.nbh, 64)), 256, 0, h->stream>>>(proj, oproj, l1, l2, h->npro,
                                                                                        h->d.nbh);
  CUW_LAUNCH_CHECK("k_addoproj");
  return CUW_OK;
}

int force_gemm(Handle* h, const double2* ded, double* force_dev) {
  const int ngl = h->d.ngl, nbh = h->d.nbh, npro = h->npro;
  int tm = ceil_div(ngl, BM);
  const int tn = ceil_div(npro, BN);
  CUW_RET(ensure_part(h, sizeof(double) * 3 * (size_t)std::max(tm, ceil_div(ngl, 128)) * npro));
  double* fpart = reinterpret_cast<double*>(h->g.part);
  if (h->tc_on()) {
    CUW_RET(tc_force(h, ded, fpart, &tm));
  } else if (!h->mixed() && h->g.prox && nbh <= kFpSlices * BK) {
    // persistent: about one CTA per SM, each walking every gstride-th G tile
    const int gstride = std::max(1, std::min(tm, h->nsm / tn));
    k_force_p<<<dim3(gstride, tn), NT, kFpSmem, h->stream>>>(h->g.psi0, h->ldg, ngl, nbh, npro, ded, h->g.gx,
                                                               h->g.gy, h->g.gz, fpart, h->g.prox, gstride);
    CUW_LAUNCH_CHECK("k_force_p");
    tm = gstride;
  } else {
    if (!h->mixed() && h->g.prox)
      k_force<true><<<dim3(tm, tn), NT, smem2_bytes<MP11>(), h->stream>>>(
          h->g.psi0, h->ldg, ngl, nbh, npro, ded, h->g.pdesc, h->g.ylm, h->g.pro, h->g.eigr, h->g.gx, h->g.gy,
          h->g.gz, fpart, h->g.prox);
    else
      k_force<false><<<dim3(tm, tn), NT, smem2_bytes<MP11>(), h->stream>>>(
          h->g.psi0, h->ldg, ngl, nbh, npro, ded, h->g.pdesc, h->g.ylm, h->g.pro, h->g.eigr, h->g.gx, h->g.gy,
          h->g.gz, fpart, nullptr);
    CUW_LAUNCH_CHECK("k_force");
  }
  TabView t = tables(h);
  k_force_final<<<dim3(3, h->d.nat), 128, 0, h->stream>>>(fpart, tm, npro, t.ipro0, t.nlmn, h->d.nat, h->gweight,
                                                          force_dev);
  CUW_LAUNCH_CHECK("k_force_final");
  return CUW_OK;
}

// dynamic shared memory above 48 KB for the pipelined contraction kernels
int gemm_setup(Handle* h) {
  CUW_TRY(smem_allow((const void*)k_proj<true, false>, (int)smem_bytes<MP21>()));
  CUW_TRY(smem_allow((const void*)k_proj<false, false>, (int)smem_bytes<MP11>()));
  CUW_TRY(smem_allow((const void*)k_proj<true, true>, (int)smem2_bytes<MP21>()));
  CUW_TRY(smem_allow((const void*)k_proj<false, true>, (int)smem2_bytes<MP11>()));
  CUW_TRY(smem_allow((const void*)k_addpro<ADDPRO_HPSI, false>, (int)smem_bytes<MP11>()));
  CUW_TRY(smem_allow((const void*)k_addpro<ADDPRO_OPSI, false>, (int)smem_bytes<MP11>()));
  CUW_TRY(smem_allow((const void*)k_addpro<ADDPRO_FUSED, false>, (int)smem_bytes<MP12>()));
  CUW_TRY(smem_allow((const void*)k_addpro<ADDPRO_HPSI, true>, (int)smem2_bytes<MP11>()));
  CUW_TRY(smem_allow((const void*)k_addpro<ADDPRO_OPSI, true>, (int)smem2_bytes<MP11>()));
  CUW_TRY(smem_allow((const void*)k_addpro<ADDPRO_FUSED, true>, (int)smem2_bytes<MP12>()));
  CUW_TRY(smem_allow((const void*)k_gram<true, true>, (int)smem2_bytes<MPGRAM>()));
  CUW_TRY(smem_allow((const void*)k_gram<false, false>, (int)smem2_bytes<MPGRAM>()));
  CUW_TRY(smem_allow((const void*)k_addx<true, true>, (int)smem2_bytes<MP11>()));
  CUW_TRY(smem_allow((const void*)k_force<false>, (int)smem2_bytes<MP11>()));
  CUW_TRY(smem_allow((const void*)k_force<true>, (int)smem2_bytes<MP11>()));
  CUW_TRY(smem_allow((const void*)k_force_p, (int)kFpSmem));
  return CUW_OK;
}

int small_tables_setup(Handle* h) {
  Device& t = h->g;
  const int nat = h->d.nat, nsp = h->d.nsp, npro = h->npro;
  std::vector<int> ipro0(nat), nlmn(nat), lnofp(npro), mofp(npro), lmn0ln(nsp * CUW_MAXLN, 0),
      lox(nsp * CUW_MAXLN, -1);
  for (int s = 0; s < nsp; ++s) {
    int off = 0;
    for (int ln = 0; ln < h->d.lnx[s]; ++ln) {
      lox[s * CUW_MAXLN + ln] = h->d.lox[s][ln];
      lmn0ln[s * CUW_MAXLN + ln] = off;
      off += 2 * h->d.lox[s][ln] + 1;
    }
  }
  for (int a = 0; a < nat; ++a) {
    ipro0[a] = h->ipro0[a];
    nlmn[a] = h->lmnx[h->isp[a]];
    int s = h->isp[a], p = ipro0[a];
    for (int ln = 0; ln < h->d.lnx[s]; ++ln)
      for (int m = 0; m < 2 * h->d.lox[s][ln] + 1; ++m) {
        lnofp[p] = ln;
        mofp[p] = m;
        ++p;
      }
  }
  auto up = [&](int** dst, const std::vector<int>& src) -> int {
    if (*dst) cudaFree(*dst);
    CUW_TRY(cudaMalloc(dst, sizeof(int) * std::max<size_t>(1, src.size())));
    CUW_TRY(cudaMemcpy(*dst, src.data(), sizeof(int) * src.size(), cudaMemcpyHostToDevice));
    return CUW_OK;
  };
  CUW_RET(up(&t.t_ipro0, ipro0));
  CUW_RET(up(&t.t_nlmn, nlmn));
  CUW_RET(up(&t.t_isp, h->isp));
  CUW_RET(up(&t.t_lnofp, lnofp));
  CUW_RET(up(&t.t_mofp, mofp));
  CUW_RET(up(&t.t_lmn0ln, lmn0ln));
  CUW_RET(up(&t.t_lox, lox));
  return CUW_OK;
}

}  // namespace cuw

// ===========================================================================
// No-allocation projections.
//
// Some callers cannot allocate device memory at all: a host code that hands
// out device memory only from its own pool, a plug-in running inside another
// program's CUDA graph capture or under a memory cap, or a process that must
// not grow its footprint after start-up.  cuwaves_projections_noalloc gives
// them <p|psi> with no cudaMalloc, cudaFree or allocating library call: the
// split-K partial sums live in the file-scope array below.  Every GPU that
// loads this library holds the array (CUW_NOALLOC_SCRATCH_BYTES) until the
// process exits.
// ===========================================================================

#define CUW_NOALLOC_SCRATCH_ELEMS (1u << 18) /* complex doubles: 4 MiB */
static __device__ __align__(256) double2 g_noalloc_scratch[CUW_NOALLOC_SCRATCH_ELEMS];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
double2* g_noalloc_ptr[kMaxDevices] = {nullptr};
}  // namespace

// Device address of the scratch array on the current device; looked up once per
// device (the host-side name of a __device__ array is not a device address).
static int noalloc_scratch(double2** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return CUW_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) return CUW_ERR_CUDA;
    if (cuw::smem_allow((const void*)cuw::k_proj<false, false>, (int)cuw::smem_bytes<cuw::MP11>()) != cudaSuccess)
      return CUW_ERR_CUDA;
    g_noalloc_ptr[dev] = static_cast<double2*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return CUW_OK;
}

extern "C" int cuwaves_projections_noalloc(int ngl, int ldg, int nbh, int nat, int npro, const double* psi,
                                           const int* pdesc, const double* ylm, const double* pro,
                                           const double* eigr, double gweight, double* proj, void* stream) {
  using namespace cuw;
  if (ngl <= 0 || ldg < ngl || nbh <= 0 || nat <= 0 || npro <= 0 || !psi || !pdesc || !ylm || !pro || !eigr ||
      !proj)
    return CUW_ERR_ARG;
  // one split needs nbh*npro complex partial sums
  const size_t per_split = (size_t)nbh * npro;
  if (per_split > CUW_NOALLOC_SCRATCH_ELEMS) return CUW_ERR_ARG;
  double2* scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc != CUW_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // an error the caller left pending belongs to the caller: it is reported as a
  // failure of this call but left in place, and nothing is launched
  if (cudaPeekAtLastError() != cudaSuccess) return CUW_ERR_CUDA;
  int nsm = 148, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int tn = ceil_div(npro, BN), tm = ceil_div(nbh, BM);
  int ks = std::max(1, std::min(ceil_div(2 * nsm, tn * tm), ceil_div(ngl, 256)));
  ks = std::min<int>(ks, (int)(CUW_NOALLOC_SCRATCH_ELEMS / per_split));
  const int kchunk = ceil_div(ceil_div(ngl, ks), BK) * BK;
  ks = ceil_div(ngl, kchunk);
  // every partial sum that the reduction reads is written by k_proj in this
  // call, so nothing in the array has to start at zero; with no error pending
  // before the launches, cudaGetLastError reports only their own failures
  k_proj<false, false><<<dim3(tn, tm, ks), NT, smem_bytes<MP11>(), st>>>(
      reinterpret_cast<const double2*>(psi), nullptr, ldg, ngl, nbh, npro, kchunk,
      reinterpret_cast<const ProDesc*>(pdesc), ylm, pro, reinterpret_cast<const double2*>(eigr), scratch, 0);
  if (cudaGetLastError() != cudaSuccess) return CUW_ERR_CUDA;
  const int rb = std::min(ceil_div((int)per_split, 256), 4 * nsm);
  k_reduce_parts<<<rb, 256, 0, st>>>(scratch, ks, per_split, per_split, gweight, reinterpret_cast<double2*>(proj));
  if (cudaGetLastError() != cudaSuccess) return CUW_ERR_CUDA;
  return CUW_OK;
}
