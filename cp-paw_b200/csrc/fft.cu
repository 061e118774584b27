// Band-batched 3-D FFT with the local potential fused in (WAVES_VPSI).
//
// Reference: WAVES_VPSI (src/paw_waves1.f90:5099-5194) runs, per band, the
// three 1-D passes of PLANEWAVE_FFTGTOR (src/paw_fft.f90:2012-2177), multiplies
// by V(r), and runs the three passes of PLANEWAVE_FFTRTOG (:2180-2341).
// Conventions (src/paw_library.f90:2635-2728): G->r is exp(+iGr) and unscaled;
// r->G is exp(-iGr) with 1/N.  Like the reference, only the z-planes that hold
// G vectors are transformed in x and y (its NR3END1/NR3END2 pruning).
//
// B200 layout: three kernels per band batch.
//   gtor_plane : sphere -> xy-plane in shared memory, x then y transforms,
//                plane written to the work grid (only occupied planes).
//   zcol_v     : z columns of 16 x-points: inverse z transform, V(r) and the
//                1/N scale, forward z transform, in shared memory.
//   rtog_plane : forward y then x transforms of a plane, gathered back onto
//                the sphere with 1/2|G|^2 (+bucket) psi added.
// Each 1-D transform is a mixed-radix Stockham autosort (radix 2,3,4,5,7,8,11)
// whose butterflies run in registers; every stage reads all of its inputs into
// registers before a barrier and writes after it, so it works in place.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "cuwaves_internal.cuh"

namespace cuw {

namespace {

constexpr int kMaxV = 8;   // complex values per thread per stage
// Grids (NR1, NR2, NR3) with kernels compiled for their lengths: the cubic
// grids of the benchmark systems, the grids the reference's rule picks for
// Si8 and Si64 at 60 Ry (28^3, 56^3), and the bulk-Si, water and small-system
// grids of the serving and batched workloads.
#define CUW_FFT_GRIDS                                                                              \
  CUW_FFT_GRID(18, 18, 18) CUW_FFT_GRID(18, 18, 36) CUW_FFT_GRID(24, 24, 24) CUW_FFT_GRID(28, 28, 28) \
  CUW_FFT_GRID(28, 28, 56) CUW_FFT_GRID(28, 56, 56) CUW_FFT_GRID(32, 32, 32) CUW_FFT_GRID(36, 36, 36) \
  CUW_FFT_GRID(48, 48, 48) CUW_FFT_GRID(56, 56, 56) CUW_FFT_GRID(56, 56, 110) CUW_FFT_GRID(64, 64, 64) \
  CUW_FFT_GRID(72, 72, 72) CUW_FFT_GRID(80, 80, 80) CUW_FFT_GRID(96, 96, 96)
constexpr int kPlaneThreads = 256;

// The transforms are written once for double2 (FP64 path) and float2 (the FP32
// FFT of the mixed-precision path).
template <class C>
struct CT;
template <>
struct CT<double2> {
  using R = double;
  __device__ __forceinline__ static double2 mk(double x, double y) { return make_double2(x, y); }
};
template <>
struct CT<float2> {
  using R = float;
  __device__ __forceinline__ static float2 mk(float x, float y) { return make_float2(x, y); }
};

// --- radix butterflies: v <- DFT_R(v) with exp(sign*2*pi*i*q*s/R) -----------
template <class C>
__device__ __forceinline__ C mul_i(C a, typename CT<C>::R sgn) {  // a * (sgn*i)
  return CT<C>::mk(-sgn * a.y, sgn * a.x);
}

template <int R>
struct Bfly;

template <>
struct Bfly<2> {
  template <class C>
  __device__ __forceinline__ static void run(C (&v)[2], typename CT<C>::R, const C*, int) {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <>
struct Bfly<3> {
  template <class C>
  __device__ __forceinline__ static void run(C (&v)[3], typename CT<C>::R sgn, const C*, int) {
    using T = typename CT<C>::R;
    const T h = (T)0.86602540378443864676;  // sqrt(3)/2
    C a = v[0], t = cadd(v[1], v[2]), d = csub(v[1], v[2]);
    C u = mul_i(cscale(d, h), sgn);
    C m = CT<C>::mk(a.x - (T)0.5 * t.x, a.y - (T)0.5 * t.y);
    v[0] = cadd(a, t);
    v[1] = cadd(m, u);
    v[2] = csub(m, u);
  }
};

template <>
struct Bfly<4> {
  template <class C>
  __device__ __forceinline__ static void run(C (&v)[4], typename CT<C>::R sgn, const C*, int) {
    C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    C t2 = cadd(v[1], v[3]), t3 = mul_i(csub(v[1], v[3]), sgn);
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
  }
};

template <>
struct Bfly<5> {
  template <class C>
  __device__ __forceinline__ static void run(C (&v)[5], typename CT<C>::R sgn, const C*, int) {
    using T = typename CT<C>::R;
    const T c1 = (T)0.30901699437494742410, c2 = (T)-0.80901699437494742410;
    const T s1 = (T)0.95105651629515357212, s2 = (T)0.58778525229247312917;
    C a = v[0];
    C p1 = cadd(v[1], v[4]), m1 = csub(v[1], v[4]);
    C p2 = cadd(v[2], v[3]), m2 = csub(v[2], v[3]);
    C r1 = CT<C>::mk(a.x + c1 * p1.x + c2 * p2.x, a.y + c1 * p1.y + c2 * p2.y);
    C r2 = CT<C>::mk(a.x + c2 * p1.x + c1 * p2.x, a.y + c2 * p1.y + c1 * p2.y);
    C i1 = mul_i(CT<C>::mk(s1 * m1.x + s2 * m2.x, s1 * m1.y + s2 * m2.y), sgn);
    C i2 = mul_i(CT<C>::mk(s2 * m1.x - s1 * m2.x, s2 * m1.y - s1 * m2.y), sgn);
    v[0] = CT<C>::mk(a.x + p1.x + p2.x, a.y + p1.y + p2.y);
    v[1] = cadd(r1, i1);
    v[4] = csub(r1, i1);
    v[2] = cadd(r2, i2);
    v[3] = csub(r2, i2);
  }
};

template <>
struct Bfly<8> {
  template <class C>
  __device__ __forceinline__ static void run(C (&v)[8], typename CT<C>::R sgn, const C*, int) {
    using T = typename CT<C>::R;
    const T q = (T)0.70710678118654752440;
    C e[4] = {v[0], v[2], v[4], v[6]};
    C o[4] = {v[1], v[3], v[5], v[7]};
    Bfly<4>::run(e, sgn, (const C*)nullptr, 0);
    Bfly<4>::run(o, sgn, (const C*)nullptr, 0);
    // twiddles W8^k = exp(sgn*i*pi*k/4)
    C w1 = CT<C>::mk(q, sgn * q), w3 = CT<C>::mk(-q, sgn * q);
    C o1 = cmul(o[1], w1), o2 = mul_i(o[2], sgn), o3 = cmul(o[3], w3);
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], o1);
    v[5] = csub(e[1], o1);
    v[2] = cadd(e[2], o2);
    v[6] = csub(e[2], o2);
    v[3] = cadd(e[3], o3);
    v[7] = csub(e[3], o3);
  }
};

// generic prime radix through the twiddle table of the axis (tw[k] = W_N^k)
template <int R>
struct BflyGeneric {
  template <class C>
  __device__ __forceinline__ static void run(C (&v)[R], typename CT<C>::R, const C* tw, int n) {
    C out[R];
    const int step = n / R;
#pragma unroll
    for (int s = 0; s < R; ++s) {
      C acc = v[0];
#pragma unroll
      for (int q = 1; q < R; ++q) acc = cadd(acc, cmul(v[q], tw[((q * s) % R) * step]));
      out[s] = acc;
    }
#pragma unroll
    for (int s = 0; s < R; ++s) v[s] = out[s];
  }
};
template <>
struct Bfly<7> : BflyGeneric<7> {};
template <>
struct Bfly<11> : BflyGeneric<11> {};

// One Stockham stage on lines [line0, line0+nl) of length n held in shared
// memory: element e of line L lives at buf[L*ls + e*es].  tw[k] = exp(sgn*2 pi i k/n).
// jfast selects the thread mapping (consecutive threads -> consecutive j).
// The caller guarantees nl*n/R <= blockDim.x * BPT.
template <int R, class C>
__device__ __noinline__ void stage(C* buf, int n, int ns, int line0, int nl, int ls, int es, bool jfast,
                                      const C* tw, typename CT<C>::R sgn) {
  constexpr int BPT = (kMaxV / R) > 0 ? (kMaxV / R) : 1;
  const int nq = n / R;
  const int total = nl * nq;
  C v[BPT][R];
  int line_[BPT], j_[BPT];
#pragma unroll
  for (int t = 0; t < BPT; ++t) {
    int bf = threadIdx.x + t * blockDim.x;
    line_[t] = -1;
    if (bf < total) {
      int line, j;
      if (jfast) { j = bf % nq; line = bf / nq; }
      else { line = bf % nl; j = bf / nl; }
      line += line0;
      line_[t] = line;
      j_[t] = j;
      const int k = j % ns;
      const int tstep = n / (ns * R);
      C* base = buf + (size_t)line * ls;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        C x = base[(size_t)(j + r * nq) * es];
        if (r && k) x = cmul(x, tw[(r * k * tstep) % n]);
        v[t][r] = x;
      }
      Bfly<R>::run(v[t], sgn, tw, n);
    }
  }
  __syncthreads();
#pragma unroll
  for (int t = 0; t < BPT; ++t) {
    if (line_[t] >= 0) {
      const int j = j_[t], k = j % ns;
      const int idxd = (j / ns) * ns * R + k;
      C* base = buf + (size_t)line_[t] * ls;
#pragma unroll
      for (int r = 0; r < R; ++r) base[(size_t)(idxd + r * ns) * es] = v[t][r];
    }
  }
  __syncthreads();
}

__host__ __device__ constexpr int bpt_of(int r) { return (kMaxV / r) > 0 ? (kMaxV / r) : 1; }

struct AxisArg {
  int n;
  int nstage;
  int radix[8];
};

// ---------------------------------------------------------------------------
// Compile-time specialisation for the common grid lengths: every divisor of
// the index arithmetic is a constant, the stages are inlined and the block
// size is fixed (kPlaneThreads), so the lines per chunk are constant too.
// ---------------------------------------------------------------------------
//
// Plan variants V (chosen per handle by the autotuner, src/paw_library.f90
// LIB_FFTW3 leaves the same choice to FFTW's measured planning):
//   bit 0: 16 instead of 8 complex values per thread and stage (more lines
//          per pass, fewer barrier-separated passes, more registers);
//   bit 1: the radix stages in ascending instead of descending order;
//   bit 2: on 64^3 grids, the z transforms exchange values between the lanes
//          of a column by warp shuffles instead of shared memory (k_zcol_v64).
// Variants 0, 1 and 2 are V = 0, 1, 2; variant 3 is V = 4 (64^3 grids only).
// ---------------------------------------------------------------------------
struct RadixList {
  int n;
  int r[8];
};
__host__ __device__ constexpr RadixList radices_of(int N, int V = 0) {
  RadixList L{0, {0, 0, 0, 0, 0, 0, 0, 0}};
  int m = N;
  const int order[7] = {8, 4, 2, 3, 5, 7, 11};
  for (int i = 0; i < 7; ++i)
    while (m % order[i] == 0 && L.n < 8) {
      L.r[L.n++] = order[i];
      m /= order[i];
    }
  if (V & 2)
    for (int a = 0, b = L.n - 1; a < b; ++a, --b) {
      const int t = L.r[a];
      L.r[a] = L.r[b];
      L.r[b] = t;
    }
  return L;
}
__host__ __device__ constexpr int values_of(int V) { return (V & 1) ? 16 : kMaxV; }
__host__ __device__ constexpr int bpt_v(int r, int mv) { return (mv / r) > 0 ? (mv / r) : 1; }
__host__ __device__ constexpr int chunk_lines(int N, int V = 0) {
  RadixList L = radices_of(N, V);
  int lc = 1 << 30;
  for (int s = 0; s < L.n; ++s) {
    int cap = (kPlaneThreads * bpt_v(L.r[s], values_of(V)) * L.r[s]) / N;
    if (cap < 1) cap = 1;
    lc = lc < cap ? lc : cap;
  }
  return lc;
}
constexpr int kFftVariants = 4;

// Line l of a transform lives at row (row0 + l) mod nrows of the buffer
// (row0 = 0 and nrows above every line index: the identity).
__device__ __forceinline__ int line_row(int l, int row0, int nrows) {
  const int r = row0 + l;
  return r >= nrows ? r - nrows : r;
}

template <int N, int R, int NS, int LC, int MV, class C>
__device__ __forceinline__ void stage_fixed(C* buf, int line0, int nl, int ls, int es, bool jfast, const C* tw,
                                            typename CT<C>::R sgn, int row0, int nrows) {
  constexpr int BPT = bpt_v(R, MV);
  constexpr int NQ = N / R;
  constexpr int TSTEP = N / (NS * R);
  // jfast: index space nl*NQ (line = bf / NQ); otherwise the full chunk LC*NQ
  // decoded modulo LC, with the lines beyond nl masked
  const int total = jfast ? nl * NQ : LC * NQ;
  C v[BPT][R];
  int off_[BPT];
  bool act[BPT];
#pragma unroll
  for (int t = 0; t < BPT; ++t) {
    const int bf = threadIdx.x + t * kPlaneThreads;
    int line, j;
    if (jfast) { j = bf % NQ; line = bf / NQ; }
    else { line = bf % LC; j = bf / LC; }
    act[t] = (bf < total) && (line < nl) && (j < NQ);
    const int k = j % NS;
    off_[t] = line * N + ((j / NS) * NS * R + k);  // (line, destination index) packed
    if (act[t]) {
      C* base = buf + (size_t)line_row(line0 + line, row0, nrows) * ls;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        C x = base[(size_t)(j + r * NQ) * es];
        if (r && k) x = cmul(x, tw[(r * k * TSTEP) % N]);
        v[t][r] = x;
      }
      Bfly<R>::run(v[t], sgn, tw, N);
    }
  }
  __syncthreads();
#pragma unroll
  for (int t = 0; t < BPT; ++t) {
    if (act[t]) {
      const int line = off_[t] / N, idxd = off_[t] % N;
      C* base = buf + (size_t)line_row(line0 + line, row0, nrows) * ls;
#pragma unroll
      for (int r = 0; r < R; ++r) base[(size_t)(idxd + r * NS) * es] = v[t][r];
    }
  }
  __syncthreads();
}

template <int N, int S, int NS, int LC, int V, class C>
__device__ __forceinline__ void stages_fixed(C* buf, int line0, int nl, int ls, int es, bool jfast, const C* tw,
                                             typename CT<C>::R sgn, int row0, int nrows) {
  constexpr RadixList L = radices_of(N, V);
  if constexpr (S < L.n) {
    constexpr int R = L.r[S];
    stage_fixed<N, R, NS, LC, values_of(V)>(buf, line0, nl, ls, es, jfast, tw, sgn, row0, nrows);
    stages_fixed<N, S + 1, NS * R, LC, V>(buf, line0, nl, ls, es, jfast, tw, sgn, row0, nrows);
  }
}

template <int N, int V = 0, class C>
__device__ void transform_fixed(C* buf, int nlines, int ls, int es, bool jfast, const C* tw, typename CT<C>::R sgn,
                                int row0 = 0, int nrows = 1 << 30) {
  constexpr int LC = chunk_lines(N, V);
  for (int l0 = 0; l0 < nlines; l0 += LC) {
    const int nl = min(LC, nlines - l0);
    stages_fixed<N, 0, 1, LC, V>(buf, l0, nl, ls, es, jfast, tw, sgn, row0, nrows);
  }
}

// lines per chunk so that every stage fits one pass of the block
__device__ __forceinline__ int lines_per_chunk(const AxisArg& ax, int nlines) {
  int lc = nlines;
  for (int s = 0; s < ax.nstage; ++s) {
    int r = ax.radix[s];
    int cap = (int)(((long)blockDim.x * bpt_of(r) * r) / ax.n);
    if (cap < 1) cap = 1;
    lc = min(lc, cap);
  }
  return lc;
}

template <class C>
__device__ void transform(C* buf, const AxisArg& ax, int nlines, int ls, int es, bool jfast, const C* tw,
                          typename CT<C>::R sgn) {
  switch (ax.n) {
    case 16: transform_fixed<16>(buf, nlines, ls, es, jfast, tw, sgn); return;
    case 20: transform_fixed<20>(buf, nlines, ls, es, jfast, tw, sgn); return;
    case 24: transform_fixed<24>(buf, nlines, ls, es, jfast, tw, sgn); return;
    case 28: transform_fixed<28>(buf, nlines, ls, es, jfast, tw, sgn); return;
    case 32: transform_fixed<32>(buf, nlines, ls, es, jfast, tw, sgn); return;
    case 36: transform_fixed<36>(buf, nlines, ls, es, jfast, tw, sgn); return;
    case 40: transform_fixed<40>(buf, nlines, ls, es, jfast, tw, sgn); return;
    case 48: transform_fixed<48>(buf, nlines, ls, es, jfast, tw, sgn); return;
    case 56: transform_fixed<56>(buf, nlines, ls, es, jfast, tw, sgn); return;
    case 64: transform_fixed<64>(buf, nlines, ls, es, jfast, tw, sgn); return;
    case 72: transform_fixed<72>(buf, nlines, ls, es, jfast, tw, sgn); return;
    case 80: transform_fixed<80>(buf, nlines, ls, es, jfast, tw, sgn); return;
    case 96: transform_fixed<96>(buf, nlines, ls, es, jfast, tw, sgn); return;
    default: break;
  }
  const int lc = lines_per_chunk(ax, nlines);
  for (int l0 = 0; l0 < nlines; l0 += lc) {
    const int nl = min(lc, nlines - l0);
    int ns = 1;
    for (int s = 0; s < ax.nstage; ++s) {
      switch (ax.radix[s]) {
        case 2: stage<2>(buf, ax.n, ns, l0, nl, ls, es, jfast, tw, sgn); break;
        case 3: stage<3>(buf, ax.n, ns, l0, nl, ls, es, jfast, tw, sgn); break;
        case 4: stage<4>(buf, ax.n, ns, l0, nl, ls, es, jfast, tw, sgn); break;
        case 5: stage<5>(buf, ax.n, ns, l0, nl, ls, es, jfast, tw, sgn); break;
        case 7: stage<7>(buf, ax.n, ns, l0, nl, ls, es, jfast, tw, sgn); break;
        case 8: stage<8>(buf, ax.n, ns, l0, nl, ls, es, jfast, tw, sgn); break;
        case 11: stage<11>(buf, ax.n, ns, l0, nl, ls, es, jfast, tw, sgn); break;
      }
      ns *= ax.radix[s];
    }
  }
}

// N > 0: the transform of compile-time length N, inlined alone into the
// kernel (its registers then fit without spills); N == 0: run-time dispatch.
template <int N, int V = 0, class C>
__device__ __forceinline__ void xform(C* buf, const AxisArg& ax, int nlines, int ls, int es, bool jfast,
                                      const C* tw, typename CT<C>::R sgn) {
  if constexpr (N > 0) transform_fixed<N, V>(buf, nlines, ls, es, jfast, tw, sgn);
  else transform(buf, ax, nlines, ls, es, jfast, tw, sgn);
}

// The x lines of an xy plane restricted to the rows that hold G vectors:
// rows (y0 + l) mod nr2 for l < ny (the plane's rows form one range of signed
// y).  The other rows are zero before the G->R transform and are not read
// after the R->G transform.  Kernels with run-time lengths transform every row.
template <int N, int V = 0, class C>
__device__ __forceinline__ void xform_rows(C* buf, const AxisArg& ax, int y0, int ny, int nr2, int ls,
                                           const C* tw, typename CT<C>::R sgn) {
  if constexpr (N > 0) transform_fixed<N, V>(buf, ny, ls, 1, false, tw, sgn, y0, nr2);
  else transform(buf, ax, nr2, ls, 1, false, tw, sgn);
}

// load twiddles exp(sgn*2 pi i k/n) from the FP64 table exp(+2 pi i k/n)
template <class C>
__device__ void load_tw(C* dst, const double2* src, int n, double sgn) {
  using T = typename CT<C>::R;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    double2 w = src[k];
    dst[k] = CT<C>::mk((T)w.x, (T)(sgn * w.y));
  }
}

template <class C>
__device__ __forceinline__ C from_d2(double2 a) {
  using T = typename CT<C>::R;
  return CT<C>::mk((T)a.x, (T)a.y);
}
__device__ __forceinline__ double2 to_d2(double2 a) { return a; }
__device__ __forceinline__ double2 to_d2(float2 a) { return make_double2((double)a.x, (double)a.y); }

// Shared-memory layout of an xy plane: rows of NR1 elements at a stride of
// NR1+1, and the x lines transformed with consecutive threads on consecutive
// rows.  With the odd stride, the eight (FP64) or sixteen (FP32) threads that
// share a shared-memory wavefront touch eight/sixteen different 16/8-byte bank
// groups in every Stockham stage; with the dense stride NR1 = 2^k, the
// scattered writes of the first radix-8 stage of the x lines (stride 8
// elements) hit one bank group eight times.
__host__ __device__ constexpr int plane_stride(int nr1) { return nr1 + 1; }
// row index of the dense plane offset i (i / NR1, with a constant divisor when
// the kernel is specialised for one length)
template <int N>
__device__ __forceinline__ int row_of(int i, int nr1) {
  if constexpr (N > 0) return i / N;
  else return i / nr1;
}

// ---------------------------------------------------------------------------
// The kernels take the work-grid type C (double2 or float2); the sphere
// coefficients psi/out stay FP64 and are converted at the gather/scatter.
template <class C, int N1, int N2, int V>
__global__ void __launch_bounds__(kPlaneThreads, 2)
    k_gtor_plane(const double2* __restrict__ psi, int ldg, int b0, const int* __restrict__ plane_off,
                 const int* __restrict__ plane_g, const int* __restrict__ plane_pos, const int2* __restrict__ plane_rows,
                 C* __restrict__ grid, int nzp, AxisArg a1, AxisArg a2, const double2* __restrict__ tw1g,
                 const double2* __restrict__ tw2g) {
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  const int nr1 = a1.n, nr2 = a2.n, npl = nr1 * nr2, ps = plane_stride(nr1);
  C* plane = sm;  // [nr2][ps]
  C* tw1 = sm + nr2 * ps;
  C* tw2 = tw1 + nr1;
  const int p = blockIdx.x, bl = blockIdx.y, b = b0 + bl;
  for (int i = threadIdx.x; i < nr2 * ps; i += blockDim.x) plane[i] = CT<C>::mk(0, 0);
  load_tw(tw1, tw1g, nr1, +1.0);
  load_tw(tw2, tw2g, nr2, +1.0);
  __syncthreads();
  const double2* src = psi + (size_t)ldg * b;
  for (int k = plane_off[p] + threadIdx.x; k < plane_off[p + 1]; k += blockDim.x)
    plane[plane_pos[k]] = from_d2<C>(src[plane_g[k]]);
  __syncthreads();
  const int2 rows = plane_rows[p];
  xform_rows<N1, V>(plane, a1, rows.x, rows.y, nr2, ps, tw1, (typename CT<C>::R)1);  // x lines
  xform<N2, V>(plane, a2, nr1, 1, ps, false, tw2, (typename CT<C>::R)1);               // y lines
  C* dst = grid + ((size_t)bl * nzp + p) * npl;
  for (int i = threadIdx.x; i < npl; i += blockDim.x) dst[i] = plane[i + row_of<N1>(i, nr1)];
}

constexpr int kTX = 16;  // x columns per z-column block, generic kernels
// x columns per z-column block of a grid with compile-time lengths: a whole x
// row up to 64 (fewer when the z lines are long, so that two blocks of the FP64
// tile [N3][TX] still fit an SM), which amortises the block's fixed work
// (twiddles, plane map, barriers) over more columns
__host__ __device__ constexpr int tx_of(int n1, int n3) {
  return n1 == 0 ? kTX : (n1 < 64 ? (n3 * n1 * 16 <= 100000 ? n1 : 32) : (n3 * 64 * 16 <= 100000 ? 64 : 56));
}

template <class C, int N, int TX>
__global__ void __launch_bounds__(kPlaneThreads, 2)
    k_zcol_v(C* __restrict__ grid, const double* __restrict__ v, const int* __restrict__ zslot, int nzp, int nr1,
             int nr2, AxisArg a3, const double2* __restrict__ tw3g, double scale) {
  using T = typename CT<C>::R;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  const int nr3 = a3.n;
  C* tile = sm;             // [nr3][TX]
  C* tw = sm + nr3 * TX;
  const int nxb = (nr1 + TX - 1) / TX;
  const int iy = blockIdx.x / nxb, x0 = (blockIdx.x % nxb) * TX;
  const int bl = blockIdx.y;
  const size_t npl = (size_t)nr1 * nr2;
  C* gb = grid + (size_t)bl * nzp * npl;
  load_tw(tw, tw3g, nr3, +1.0);
  for (int i = threadIdx.x; i < nr3 * TX; i += blockDim.x) {
    int iz = i / TX, x = i % TX;
    int s = zslot[iz];
    C val = CT<C>::mk(0, 0);
    if (s >= 0 && x0 + x < nr1) val = gb[(size_t)s * npl + (size_t)iy * nr1 + x0 + x];
    tile[i] = val;
  }
  __syncthreads();
  xform<N>(tile, a3, TX, 1, TX, false, tw, (T)1);
  for (int i = threadIdx.x; i < nr3 * TX; i += blockDim.x) {
    int iz = i / TX, x = i % TX;
    double vv = 0.0;
    if (x0 + x < nr1) vv = v[(size_t)x0 + x + (size_t)nr1 * (iy + (size_t)nr2 * iz)] * scale;
    tile[i] = cscale(tile[i], (T)vv);
  }
  __syncthreads();
  // forward transform: conjugated twiddles
  for (int k = threadIdx.x; k < nr3; k += blockDim.x) tw[k].y = -tw[k].y;
  __syncthreads();
  xform<N>(tile, a3, TX, 1, TX, false, tw, (T)-1);
  for (int i = threadIdx.x; i < nr3 * TX; i += blockDim.x) {
    int iz = i / TX, x = i % TX;
    int s = zslot[iz];
    if (s >= 0 && x0 + x < nr1) gb[(size_t)s * npl + (size_t)iy * nr1 + x0 + x] = tile[i];
  }
}

// z transforms of one y row for a 64^3 grid without block-wide barriers.
// Each x column is transformed by the 8 lanes t = 0..7 of a warp quarter-group
// as 64 = 8 x 8 (Cooley-Tukey): a radix-8 DFT over the lane's strided elements
// x[t + 8r], the twiddles exp(sgn 2 pi i t k1/64), a transpose through the
// column's own 64 shared-memory slots, and a radix-8 DFT across the lanes, which
// leaves X[t + 8 k2] in lane t, the same distribution as the input.  V(r) is
// applied in registers between the G->R and the R->G transforms, so the only
// block barriers are around the coalesced load and store of the tile.
//
// Shared-memory banks: the tile's row stride kZ64Ld = 68 and the rotated slot
// order of the transpose ((t + k1) mod 8) put the lanes of one wavefront
// (8 lanes of 16 bytes, or 16 lanes of 8 bytes) on different bank groups in
// every access.
constexpr int kZ64Ld = 68;
constexpr int kZ64Smem = 64 * kZ64Ld + 2 * 64;  // elements: tile and two twiddle tables
// bytes of shared memory of k_zcol_v64<C>: the elements above and the y row of
// V(r) * scale as [64 z][kZ64Ld] real numbers of the work-grid precision
template <class C>
constexpr int z64_smem_bytes() { return kZ64Smem * (int)sizeof(C) + 64 * kZ64Ld * (int)sizeof(typename CT<C>::R); }

// b[j] = a[(j + sh) & 7] (sh = +-t) for a run-time shift, by three stages of
// selects: the register indices stay compile-time constants
template <class C>
__device__ __forceinline__ void rot8(C (&a)[8], int sh) {
#pragma unroll
  for (int bit = 1; bit < 8; bit <<= 1) {
    const bool on = (sh & bit) != 0;
    C b[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) b[j] = on ? a[(j + bit) & 7] : a[j];
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = b[j];
  }
}
__device__ __forceinline__ float2 shfl_c(float2 v, int src) {
  return make_float2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}
__device__ __forceinline__ double2 shfl_c(double2 v, int src) {
  return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

// on entry a[r] = x[t + 8r]; on exit a[k] = X[t + 8k], X[k] = sum_n x[n] tw[nk mod 64]
// with tw[k] = exp(sgn 2 pi i k/64).  Between the two radix-8 DFTs the 8 x 8
// transpose among the column's lanes (lane t then holds element t of every
// lane): through the column's shared-memory slots col[q * kZ64Ld], or (SHFL)
// by warp shuffles among the 8 lanes, which are `lane0 + 4 t` of the warp:
// round r sends element (t - r) mod 8 to lane (t - r) mod 8 and receives
// element t of lane (t + r) mod 8; the array is rotated by t before and after
// so that every round uses a fixed register.
template <class C, bool SHFL>
__device__ __forceinline__ void z64(C (&a)[8], C* col, int t, const C* tw, typename CT<C>::R sgn) {
  Bfly<8>::run(a, sgn, tw, 64);
#pragma unroll
  for (int k1 = 1; k1 < 8; ++k1) a[k1] = cmul(a[k1], tw[t * k1]);
  if constexpr (SHFL) {
    const int lane = threadIdx.x & 31, l0 = lane & 3;
    rot8(a, t);  // a[j] = old a[(j + t) mod 8]
    C b[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      // send old a[(t - r) mod 8] = rotated a[(-r) mod 8]
      const C v = a[(8 - r) & 7];
      b[r] = shfl_c(v, l0 + 4 * ((t + r) & 7));  // element t of lane (t + r) mod 8
    }
    // b[r] holds element t of lane (t + r) mod 8: a[n1] = b[(n1 - t) mod 8]
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = b[j];
    rot8(a, 8 - t);
  } else {
    __syncwarp();  // the lanes' earlier reads of the slots are done
#pragma unroll
    for (int k1 = 0; k1 < 8; ++k1) col[(k1 * 8 + ((t + k1) & 7)) * kZ64Ld] = a[k1];
    __syncwarp();
#pragma unroll
    for (int n1 = 0; n1 < 8; ++n1) a[n1] = col[(t * 8 + ((n1 + t) & 7)) * kZ64Ld];
  }
  Bfly<8>::run(a, sgn, tw, 64);
}

template <class C, bool SHFL>
__global__ void __launch_bounds__(kPlaneThreads, 2)
    k_zcol_v64(C* __restrict__ grid, const double* __restrict__ v, const int* __restrict__ zslot, int nzp, int nr2,
               const double2* __restrict__ tw3g, double scale) {
  using T = typename CT<C>::R;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  C* tile = sm;               // [64 z][kZ64Ld], x columns 0..63
  C* twp = sm + 64 * kZ64Ld;  // exp(+2 pi i k/64)
  C* twm = twp + 64;          // exp(-2 pi i k/64)
  T* vrow = reinterpret_cast<T*>(twm + 64);  // [64 z][kZ64Ld]: V(x, iy, z) * scale
  const int iy = blockIdx.x, bl = blockIdx.y;
  const size_t npl = (size_t)64 * nr2;
  C* gb = grid + (size_t)bl * nzp * npl;
  load_tw(twp, tw3g, 64, +1.0);
  load_tw(twm, tw3g, 64, -1.0);
  for (int i = threadIdx.x; i < 64 * 64; i += blockDim.x) {
    const int iz = i >> 6, x = i & 63, s = zslot[iz];
    tile[iz * kZ64Ld + x] = s >= 0 ? gb[(size_t)s * npl + (size_t)iy * 64 + x] : CT<C>::mk(0, 0);
    vrow[iz * kZ64Ld + x] = (T)(v[(size_t)x + 64 * ((size_t)iy + (size_t)nr2 * iz)] * scale);
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int t = lane >> 2, l = lane & 3;
  for (int round = 0; round < 2; ++round) {  // 8 warps x 2 rounds x 4 columns
    const int x = warp * 8 + round * 4 + l;
    C* col = tile + x;
    C a[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) a[r] = col[(t + 8 * r) * kZ64Ld];
    z64<C, SHFL>(a, col, t, twp, (T)1);
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = cscale(a[k], vrow[(t + 8 * k) * kZ64Ld + x]);
    z64<C, SHFL>(a, col, t, twm, (T)-1);
    __syncwarp();  // the transpose reads are done before the slots take the result
#pragma unroll
    for (int k = 0; k < 8; ++k) col[(t + 8 * k) * kZ64Ld] = a[k];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 64 * 64; i += blockDim.x) {
    const int iz = i >> 6, x = i & 63, s = zslot[iz];
    if (s >= 0) gb[(size_t)s * npl + (size_t)iy * 64 + x] = tile[iz * kZ64Ld + x];
  }
}

// Pseudo density of WAVES_DENSITY (src/paw_waves1.f90:5377-5500) for super
// wave functions at the Gamma point: after the x/y passes of k_gtor_plane, the
// G->R z transform of kRhoTX x columns of every band of the batch in turn, and
// rho(r) += f1 Re(psi)^2 + f2 Im(psi)^2 (= Re[psi (s1 conj psi + s2 psi)] with
// s1,2 = (f1 +- f2)/2, :5474-5496) in FP64, bands in order, so that the sum is
// deterministic; `first` starts rho from zero, else the batch adds to it.
constexpr int kRhoTX = 16;
template <class C, int N>
__global__ void __launch_bounds__(kPlaneThreads, 2)
    k_zcol_rho(const C* __restrict__ grid, const int* __restrict__ zslot, int nzp, int nr1, int nr2, AxisArg a3,
               const double2* __restrict__ tw3g, const double* __restrict__ occ, int nb, int b0, int nbatch,
               double* __restrict__ rho, int first) {
  using T = typename CT<C>::R;
  constexpr int TX = kRhoTX;
  constexpr int EPT = 8;  // tile elements per thread (nr3 * TX <= EPT * blockDim)
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  const int nr3 = a3.n;
  C* tile = sm;  // [nr3][TX]
  C* tw = sm + nr3 * TX;
  const int nxb = (nr1 + TX - 1) / TX;
  const int iy = blockIdx.x / nxb, x0 = (blockIdx.x % nxb) * TX;
  const size_t npl = (size_t)nr1 * nr2;
  load_tw(tw, tw3g, nr3, +1.0);
  double acc[EPT];
#pragma unroll
  for (int e = 0; e < EPT; ++e) {
    const int i = threadIdx.x + e * blockDim.x, iz = i / TX, x = i % TX;
    const bool in = i < nr3 * TX && x0 + x < nr1;
    acc[e] = (!first && in) ? rho[(size_t)x0 + x + (size_t)nr1 * (iy + (size_t)nr2 * iz)] : 0.0;
  }
  for (int bl = 0; bl < nbatch; ++bl) {
    const int b = b0 + bl;
    const double f1 = occ[2 * b], f2 = 2 * b + 1 < nb ? occ[2 * b + 1] : 0.0;
    if (f1 == 0.0 && f2 == 0.0) continue;  // the same for the whole block
    const C* gb = grid + (size_t)bl * nzp * npl;
    __syncthreads();  // the previous band's reads of the tile are done
    for (int i = threadIdx.x; i < nr3 * TX; i += blockDim.x) {
      const int iz = i / TX, x = i % TX, s = zslot[iz];
      C val = CT<C>::mk(0, 0);
      if (s >= 0 && x0 + x < nr1) val = gb[(size_t)s * npl + (size_t)iy * nr1 + x0 + x];
      tile[i] = val;
    }
    __syncthreads();
    xform<N>(tile, a3, TX, 1, TX, false, tw, (T)1);
#pragma unroll
    for (int e = 0; e < EPT; ++e) {
      const int i = threadIdx.x + e * blockDim.x;
      if (i < nr3 * TX) {
        const double re = (double)tile[i].x, im = (double)tile[i].y;
        acc[e] += f1 * re * re + f2 * im * im;
      }
    }
  }
#pragma unroll
  for (int e = 0; e < EPT; ++e) {
    const int i = threadIdx.x + e * blockDim.x, iz = i / TX, x = i % TX;
    if (i < nr3 * TX && x0 + x < nr1) rho[(size_t)x0 + x + (size_t)nr1 * (iy + (size_t)nr2 * iz)] = acc[e];
  }
}

template <class C, int N1, int N2, int V>
__global__ void __launch_bounds__(kPlaneThreads, 2)
    k_rtog_plane(const C* __restrict__ grid, int nzp, const int* __restrict__ plane_off,
                 const int* __restrict__ plane_g, const int* __restrict__ plane_pos,
                 const int2* __restrict__ plane_rows, double2* __restrict__ out,
                 const double2* __restrict__ psi, int ldg, int b0, const double* __restrict__ g2,
                 const double* __restrict__ bucket, int add_kin, AxisArg a1, AxisArg a2,
                 const double2* __restrict__ tw1g, const double2* __restrict__ tw2g) {
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  const int nr1 = a1.n, nr2 = a2.n, npl = nr1 * nr2, pst = plane_stride(nr1);
  C* plane = sm;  // [nr2][pst]
  C* tw1 = sm + nr2 * pst;
  C* tw2 = tw1 + nr1;
  const int p = blockIdx.x, bl = blockIdx.y, b = b0 + bl;
  const C* srcp = grid + ((size_t)bl * nzp + p) * npl;
  for (int i = threadIdx.x; i < npl; i += blockDim.x) plane[i + row_of<N1>(i, nr1)] = srcp[i];
  load_tw(tw1, tw1g, nr1, -1.0);
  load_tw(tw2, tw2g, nr2, -1.0);
  __syncthreads();
  xform<N2, V>(plane, a2, nr1, 1, pst, false, tw2, (typename CT<C>::R)-1);  // y lines
  const int2 rows = plane_rows[p];
  xform_rows<N1, V>(plane, a1, rows.x, rows.y, nr2, pst, tw1, (typename CT<C>::R)-1);  // x lines
  double2* dst = out + (size_t)ldg * b;
  const double2* ps = psi + (size_t)ldg * b;
  for (int k = plane_off[p] + threadIdx.x; k < plane_off[p + 1]; k += blockDim.x) {
    int g = plane_g[k];
    double2 val = to_d2(plane[plane_pos[k]]);
    if (add_kin) {
      double kin = 0.5 * g2[g] + (bucket ? bucket[g] : 0.0);
      double2 c = ps[g];
      val.x += kin * c.x;
      val.y += kin * c.y;
    }
    dst[g] = val;
  }
}

// One pass of a 3-D transform of a full FP64 complex grid (x fastest), for
// the single real functions of the potential (PLANEWAVE$SUPFFT of
// POTENTIAL$VOFRHO): every block transforms kGridTX lines of one axis in
// shared memory.  x lines are rows (tile [line][x] at a row stride n + 1);
// y and z lines are taken as kGridTX consecutive x columns of one z plane
// (axis 1) or one y row (axis 2), loaded and stored coalesced along x.
constexpr int kGridTX = 16;
__global__ void __launch_bounds__(kPlaneThreads)
    k_grid_lines(double2* __restrict__ grid, int nr1, int nr2, int nr3, int axis, AxisArg ax,
                 const double2* __restrict__ twg, double sgn) {
  extern __shared__ __align__(16) unsigned char smraw[];
  double2* tile = reinterpret_cast<double2*>(smraw);
  const int n = ax.n;
  const int TX = kGridTX;
  double2* tw = tile + (size_t)TX * (n + 1);
  load_tw(tw, twg, n, sgn);
  if (axis == 0) {
    const int nrows = nr2 * nr3, row0 = blockIdx.x * TX, nl = min(TX, nrows - row0);
    for (int i = threadIdx.x; i < nl * n; i += blockDim.x) {
      const int r = i / n, x = i % n;
      tile[r * (n + 1) + x] = grid[(size_t)(row0 + r) * nr1 + x];
    }
    __syncthreads();
    xform<0>(tile, ax, nl, n + 1, 1, false, tw, sgn);
    for (int i = threadIdx.x; i < nl * n; i += blockDim.x) {
      const int r = i / n, x = i % n;
      grid[(size_t)(row0 + r) * nr1 + x] = tile[r * (n + 1) + x];
    }
    return;
  }
  // axis 1: lines along y at fixed z; axis 2: lines along z at fixed y
  const int nxb = (nr1 + TX - 1) / TX;
  const int x0 = (blockIdx.x % nxb) * TX, other = blockIdx.x / nxb;
  const size_t es = axis == 1 ? (size_t)nr1 : (size_t)nr1 * nr2;
  const size_t base = axis == 1 ? (size_t)nr1 * nr2 * other : (size_t)nr1 * other;
  const int nl = min(TX, nr1 - x0);
  for (int i = threadIdx.x; i < n * TX; i += blockDim.x) {
    const int e = i / TX, x = i % TX;
    tile[i] = x < nl ? grid[base + (size_t)e * es + x0 + x] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  xform<0>(tile, ax, TX, 1, TX, false, tw, sgn);
  for (int i = threadIdx.x; i < n * TX; i += blockDim.x) {
    const int e = i / TX, x = i % TX;
    if (x < nl) grid[base + (size_t)e * es + x0 + x] = tile[i];
  }
}

AxisArg make_axis(const AxisPlan& p) {
  AxisArg a;
  a.n = p.n;
  a.nstage = p.nstage;
  for (int i = 0; i < 8; ++i) a.radix[i] = p.radix[i];
  return a;
}

bool plan_axis(int n, AxisPlan& p) {
  p.n = n;
  p.nstage = 0;
  int m = n;
  const int order[] = {8, 4, 2, 3, 5, 7, 11};
  for (int r : order) {
    while (m % r == 0 && p.nstage < 8) {
      p.radix[p.nstage++] = r;
      m /= r;
    }
  }
  // prefer a radix-8 stage over 4*2
  return m == 1;
}

}  // namespace

// out = FFT_RTOG[ V * FFT_GTOR[psi] ] (+ 1/2 G^2 psi + bucket psi when add_kinetic)
template <class C, int N1, int N2, int N3, int V>
static int fft_vpsi_t(Handle* h, const double2* psi, double2* out, bool add_kinetic) {
  constexpr int TX = tx_of(N1, N3);
  const int nr1 = h->d.nr1, nr2 = h->d.nr2, nr3 = h->d.nr3;
  const int smem_plane = (int)(((size_t)nr2 * plane_stride(nr1) + nr1 + nr2) * sizeof(C));
  const int smem_z = (int)(((size_t)nr3 * TX + nr3) * sizeof(C));
  const int tp = kPlaneThreads;
  const int tz = kPlaneThreads;
  AxisArg a1 = make_axis(h->ax[0]), a2 = make_axis(h->ax[1]), a3 = make_axis(h->ax[2]);
  const double scale = 1.0 / ((double)nr1 * nr2 * nr3);
  Device& g = h->g;
  C* grid = reinterpret_cast<C*>(g.grid);
  for (int b0 = 0; b0 < h->d.nbh; b0 += h->batch) {
    const int nb = std::min(h->batch, h->d.nbh - b0);
    k_gtor_plane<C, N1, N2, V><<<dim3(h->nzp, nb), tp, smem_plane, h->stream>>>(psi, h->ldg, b0, g.plane_off, g.plane_g,
                                                                           g.plane_pos, g.plane_rows, grid, h->nzp,
                                                                           a1, a2, g.tw1, g.tw2);
    CUW_LAUNCH_CHECK("k_gtor_plane");
    if constexpr (N1 == 64 && N3 == 64) {
      k_zcol_v64<C, (V & 4) != 0><<<dim3(nr2, nb), tz, z64_smem_bytes<C>(), h->stream>>>(grid, g.v, g.zslot, h->nzp, nr2,
                                                                                 g.tw3, scale);
      CUW_LAUNCH_CHECK("k_zcol_v64");
    } else {
      const int nxb = (nr1 + TX - 1) / TX;
      k_zcol_v<C, N3, TX><<<dim3(nr2 * nxb, nb), tz, smem_z, h->stream>>>(grid, g.v, g.zslot, h->nzp, nr1, nr2, a3,
                                                                       g.tw3, scale);
      CUW_LAUNCH_CHECK("k_zcol_v");
    }
    k_rtog_plane<C, N1, N2, V><<<dim3(h->nzp, nb), tp, smem_plane, h->stream>>>(grid, h->nzp, g.plane_off, g.plane_g,
                                                                      g.plane_pos, g.plane_rows, out, psi, h->ldg, b0, g.g2,
                                                                      g.bucket, add_kinetic ? 1 : 0, a1, a2,
                                                                      g.tw1, g.tw2);
    CUW_LAUNCH_CHECK("k_rtog_plane");
  }
  return CUW_OK;
}


// rho = sum over the bands of this set of f |psi(r)|^2 terms (WAVES_DENSITY
// for TINV at Gamma), batch by batch through the work grid
template <class C, int N1, int N2, int N3, int V>
static int fft_density_t(Handle* h, const double2* psi, double* rho) {
  const int nr1 = h->d.nr1, nr2 = h->d.nr2, nr3 = h->d.nr3;
  if (nr3 * kRhoTX > 8 * kPlaneThreads) return h->fail(CUW_ERR_UNSUPPORTED, "density: NR3 above 128");
  const int smem_plane = (int)(((size_t)nr2 * plane_stride(nr1) + nr1 + nr2) * sizeof(C));
  const int smem_rho = (int)(((size_t)nr3 * kRhoTX + nr3) * sizeof(C));
  AxisArg a1 = make_axis(h->ax[0]), a2 = make_axis(h->ax[1]), a3 = make_axis(h->ax[2]);
  Device& g = h->g;
  C* grid = reinterpret_cast<C*>(g.grid);
  const int nxb = (nr1 + kRhoTX - 1) / kRhoTX;
  for (int b0 = 0; b0 < h->d.nbh; b0 += h->batch) {
    const int nb = std::min(h->batch, h->d.nbh - b0);
    k_gtor_plane<C, N1, N2, V><<<dim3(h->nzp, nb), kPlaneThreads, smem_plane, h->stream>>>(
        psi, h->ldg, b0, g.plane_off, g.plane_g, g.plane_pos, g.plane_rows, grid, h->nzp, a1, a2, g.tw1, g.tw2);
    CUW_LAUNCH_CHECK("k_gtor_plane");
    k_zcol_rho<C, N3><<<nr2 * nxb, kPlaneThreads, smem_rho, h->stream>>>(grid, g.zslot, h->nzp, nr1, nr2, a3, g.tw3,
                                                                       g.occ, h->d.nb, b0, nb, rho, b0 == 0);
    CUW_LAUNCH_CHECK("k_zcol_rho");
  }
  return CUW_OK;
}

// kernels of work-grid type C and length N (0: any length): shared-memory
// limits and the launcher
template <class C, int N1, int N2, int N3, int V>
static int fft_select_v(Handle* h, int smem_plane) {
  constexpr int TX = tx_of(N1, N3);
  const int smem_z = (int)(((size_t)h->d.nr3 * TX + h->d.nr3) * sizeof(C));
  CUW_TRY(smem_allow((const void*)k_gtor_plane<C, N1, N2, V>, smem_plane));
  CUW_TRY(smem_allow((const void*)k_rtog_plane<C, N1, N2, V>, smem_plane));
  if constexpr (N1 == 64 && N3 == 64)
    CUW_TRY(smem_allow((const void*)k_zcol_v64<C, (V & 4) != 0>, z64_smem_bytes<C>()));
  else CUW_TRY(smem_allow((const void*)k_zcol_v<C, N3, TX>, smem_z));
  CUW_TRY(smem_allow((const void*)k_zcol_rho<C, N3>, (int)(((size_t)h->d.nr3 * kRhoTX + h->d.nr3) * sizeof(C))));
  h->fft_run = &fft_vpsi_t<C, N1, N2, N3, V>;
  h->fft_rho = &fft_density_t<C, N1, N2, N3, V>;
  return CUW_OK;
}
// the plan variant h->fft_variant of a grid with compiled lengths (variant 0
// for the kernels with run-time lengths)
template <class C, int N1, int N2, int N3>
static int fft_select(Handle* h, int smem_plane) {
  if constexpr (N1 > 0) {
    switch (h->fft_variant) {
      case 1: return fft_select_v<C, N1, N2, N3, 1>(h, smem_plane);
      case 2: return fft_select_v<C, N1, N2, N3, 2>(h, smem_plane);
      case 3:
        if constexpr (N1 == 64 && N3 == 64) return fft_select_v<C, N1, N2, N3, 4>(h, smem_plane);
        break;
      default: break;
    }
  }
  return fft_select_v<C, N1, N2, N3, 0>(h, smem_plane);
}

// Kernels of the handle's grid and plan variant: grids of the table get
// kernels compiled for their lengths (every index divisor and Stockham stage a
// constant); any other grid takes the kernels with run-time lengths.
static int fft_choose(Handle* h) {
  const int nr1 = h->d.nr1, nr2 = h->d.nr2, nr3 = h->d.nr3;
  const size_t es = h->mixed() ? sizeof(float2) : sizeof(double2);
  const int smem_plane = (int)(((size_t)nr2 * plane_stride(nr1) + nr1 + nr2) * es);
  int rc = CUW_OK;
  bool found = false;
#define CUW_FFT_GRID(A, B, Z)                                                                        \
  if (!found && nr1 == A && nr2 == B && nr3 == Z) {                                                  \
    found = true;                                                                                    \
    rc = h->mixed() ? fft_select<float2, A, B, Z>(h, smem_plane) : fft_select<double2, A, B, Z>(h, smem_plane); \
  }
  CUW_FFT_GRIDS
#undef CUW_FFT_GRID
  h->fft_compiled = found;
  if (!found) {
    h->fft_variant = 0;
    rc = h->mixed() ? fft_select<float2, 0, 0, 0>(h, smem_plane) : fft_select<double2, 0, 0, 0>(h, smem_plane);
  }
  return rc;
}

int fft_setup(Handle* h, const int* igvec) {
  const int nr1 = h->d.nr1, nr2 = h->d.nr2, nr3 = h->d.nr3, ngl = h->d.ngl;
  for (int a = 0; a < 3; ++a) {
    int n = a == 0 ? nr1 : (a == 1 ? nr2 : nr3);
    if (!plan_axis(n, h->ax[a]))
      return h->fail(CUW_ERR_UNSUPPORTED, "FFT length " + std::to_string(n) + " has a prime factor above 11");
  }
  const size_t npl = (size_t)nr1 * nr2;
  // work-grid element: FP64 complex, or FP32 complex on the mixed path
  const size_t es = h->mixed() ? sizeof(float2) : sizeof(double2);
  const size_t plane_elems = (size_t)nr2 * plane_stride(nr1) + nr1 + nr2;
  if (plane_elems * es > (size_t)(220 * 1024) || ((size_t)nr3 * kTX + nr3) * es > 14000 * sizeof(double2))
    return h->fail(CUW_ERR_UNSUPPORTED, "FFT plane too large for shared memory");
  // occupied planes and the per-plane G lists
  std::vector<int> cnt(nr3, 0);
  std::vector<int> iz_of(ngl), pos_of(ngl);
  for (int g = 0; g < ngl; ++g) {
    int i1 = ((igvec[3 * g] % nr1) + nr1) % nr1;
    int i2 = ((igvec[3 * g + 1] % nr2) + nr2) % nr2;
    int i3 = ((igvec[3 * g + 2] % nr3) + nr3) % nr3;
    iz_of[g] = i3;
    pos_of[g] = i1 + plane_stride(nr1) * i2;  // padded shared-memory plane
    cnt[i3]++;
  }
  std::vector<int> zslot(nr3, -1), plane_iz, off(1, 0);
  for (int z = 0; z < nr3; ++z)
    if (cnt[z]) {
      zslot[z] = (int)plane_iz.size();
      plane_iz.push_back(z);
      off.push_back(off.back() + cnt[z]);
    }
  const int nzp = (int)plane_iz.size();
  // signed row range of every occupied plane: rows (y0 + l) mod NR2, l < ny
  std::vector<int> ylo(nzp, 1 << 30), yhi(nzp, -(1 << 30));
  for (int gg = 0; gg < ngl; ++gg) {
    const int s = zslot[iz_of[gg]];
    int y = ((igvec[3 * gg + 1] % nr2) + nr2) % nr2;
    if (y > nr2 / 2) y -= nr2;
    ylo[s] = std::min(ylo[s], y);
    yhi[s] = std::max(yhi[s], y);
  }
  std::vector<int2> rows(nzp);
  for (int s = 0; s < nzp; ++s) {
    int ny = yhi[s] - ylo[s] + 1;
    int y0 = (ylo[s] + nr2) % nr2;
    if (ny > nr2) { ny = nr2; y0 = 0; }
    rows[s] = make_int2(y0, ny);
  }
  std::vector<int> fill(off.begin(), off.end() - 1), pg(ngl), pp(ngl);
  for (int g = 0; g < ngl; ++g) {
    int s = zslot[iz_of[g]];
    int k = fill[s]++;
    pg[k] = g;
    pp[k] = pos_of[g];
  }
  h->nzp = nzp;
  // band batch: keep the work grid near 48 MB so that it stays in L2
  const size_t per_band = (size_t)nzp * npl * es;
  int batch = (int)std::max<size_t>(1, (48u << 20) / per_band);
  batch = std::min(batch, h->d.nbh);
  h->batch = batch;
  Device& g = h->g;
  if (g.plane_off) {
    cudaFree(g.plane_off); cudaFree(g.plane_g); cudaFree(g.plane_pos); cudaFree(g.zslot); cudaFree(g.plane_iz);
    cudaFree(g.plane_rows);
    cudaFree(g.grid); cudaFree(g.tw1); cudaFree(g.tw2); cudaFree(g.tw3);
  }
  CUW_TRY(cudaMalloc(&g.plane_off, sizeof(int) * (nzp + 1)));
  CUW_TRY(cudaMalloc(&g.plane_g, sizeof(int) * ngl));
  CUW_TRY(cudaMalloc(&g.plane_pos, sizeof(int) * ngl));
  CUW_TRY(cudaMalloc(&g.zslot, sizeof(int) * nr3));
  CUW_TRY(cudaMalloc(&g.plane_iz, sizeof(int) * nzp));
  CUW_TRY(cudaMalloc(&g.plane_rows, sizeof(int2) * nzp));
  CUW_TRY(cudaMalloc(&g.grid, per_band * batch));
  h->grid_bands = batch;
  CUW_TRY(cudaMemcpy(g.plane_off, off.data(), sizeof(int) * (nzp + 1), cudaMemcpyHostToDevice));
  CUW_TRY(cudaMemcpy(g.plane_g, pg.data(), sizeof(int) * ngl, cudaMemcpyHostToDevice));
  CUW_TRY(cudaMemcpy(g.plane_pos, pp.data(), sizeof(int) * ngl, cudaMemcpyHostToDevice));
  CUW_TRY(cudaMemcpy(g.zslot, zslot.data(), sizeof(int) * nr3, cudaMemcpyHostToDevice));
  CUW_TRY(cudaMemcpy(g.plane_iz, plane_iz.data(), sizeof(int) * nzp, cudaMemcpyHostToDevice));
  CUW_TRY(cudaMemcpy(g.plane_rows, rows.data(), sizeof(int2) * nzp, cudaMemcpyHostToDevice));
  double2** tws[3] = {&g.tw1, &g.tw2, &g.tw3};
  for (int a = 0; a < 3; ++a) {
    int n = h->ax[a].n;
    std::vector<double2> t(n);
    for (int k = 0; k < n; ++k) {
      double ang = 2.0 * M_PI * (double)k / (double)n;
      t[k] = make_double2(std::cos(ang), std::sin(ang));
    }
    CUW_TRY(cudaMalloc(tws[a], sizeof(double2) * n));
    CUW_TRY(cudaMemcpy(*tws[a], t.data(), sizeof(double2) * n, cudaMemcpyHostToDevice));
  }
  return fft_choose(h);
}

// 3-D transform of a full FP64 complex grid (x fastest), in place and
// unscaled: dir = +1 is G->R (exp(+iGr)), dir = -1 is R->G (exp(-iGr)); the
// caller applies the 1/N of the reference's R->G transform.
int grid_fft(Handle* h, double2* grid, int dir) {
  const int n[3] = {h->d.nr1, h->d.nr2, h->d.nr3};
  const double2* tw[3] = {h->g.tw1, h->g.tw2, h->g.tw3};
  for (int a = 0; a < 3; ++a) {
    const AxisArg ax = make_axis(h->ax[a]);
    const int smem = (int)(((size_t)kGridTX * (n[a] + 1) + n[a]) * sizeof(double2));
    CUW_TRY(smem_allow((const void*)k_grid_lines, smem));
    const int nxb = (n[0] + kGridTX - 1) / kGridTX;
    const int blocks = a == 0 ? ceil_div(n[1] * n[2], kGridTX) : nxb * (a == 1 ? n[2] : n[1]);
    k_grid_lines<<<blocks, kPlaneThreads, smem, h->stream>>>(grid, n[0], n[1], n[2], a, ax, tw[a], (double)dir);
    CUW_LAUNCH_CHECK("k_grid_lines");
  }
  return CUW_OK;
}

// FP64 transforms, or FP32 transforms and V(r) product on the mixed path, with
// the kernels chosen by fft_setup for the grid
int fft_vpsi(Handle* h, const double2* psi, double2* out, bool add_kinetic) {
  if (!h->fft_run) return h->fail(CUW_ERR_STATE, "FFT not set up");
  return h->fft_run(h, psi, out, add_kinetic);
}

int fft_density(Handle* h, const double2* psi, double* rho) {
  if (!h->fft_rho) return h->fail(CUW_ERR_STATE, "FFT not set up");
  return h->fft_rho(h, psi, rho);
}

// plan variant v (0 .. fft_variants()-1) of the compiled kernels; grids with
// run-time lengths have variant 0 only
// the shuffle variant (3) changes only the 64-point z kernel
static bool z64_grid(const Handle* h) { return h->d.nr1 == 64 && h->d.nr2 == 64 && h->d.nr3 == 64; }
int fft_variants(const Handle* h) { return !h->fft_compiled ? 1 : (z64_grid(h) ? kFftVariants : kFftVariants - 1); }
int fft_set_variant(Handle* h, int v) {
  if (!h->fft_run) return h->fail(CUW_ERR_STATE, "FFT not set up");
  if (v < 0 || v >= fft_variants(h)) return CUW_ERR_UNSUPPORTED;
  h->fft_variant = v;
  h->touch();
  return fft_choose(h);
}

}  // namespace cuw
