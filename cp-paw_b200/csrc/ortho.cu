// Orthonormality constraint of the CP step on the device (FP64 throughout).
//
//   k_unravel       WAVES_OVERLAP + WAVES_1COVERLAP unravelling of super wave
//                   functions into real NB x NB matrices (src/paw_waves2.f90:797-848,
//                   999-1020) and their sum (:262-289)
//   k_lambda_init   symmetrisation and occupation scaling of RLAM0 (:295-303, 352-359)
//   k_jacobi        eigenpairs of 0.5*(CHIPSI+CHIPSI^T) (LIB$DIAGR8 -> DSYEV,
//                   src/paw_library.f90:572-631, 1555-1620) by parallel cyclic Jacobi
//   k_ortho_x       the iteration of WAVES_ORTHO_X (src/paw_waves2.f90:1844-2022)
//                   as one thread-block cluster; every wait is a hardware cluster
//                   barrier and the loop is bounded by max_iter
//   k_lambda12      LAMBDA1/LAMBDA2 of WAVES_ADDOPSI (:583-595)
//   k_switch_lambda Lagrange extrapolation of WAVES$SWITCH (:2249-2296)
//   k_ortho_y       WAVES_ORTHO_Y_C (:1025-1338) for WAVES_GRAMSCHMIDT (:2025-2177);
//                   its matrices are real at the Gamma point, so it runs in real
//                   arithmetic
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "cuwaves_internal.cuh"

namespace cg = cooperative_groups;

namespace cuw {

namespace {

// status of k_ortho_x when the Lyapunov fixed point in an earlier eigenbasis
// does not converge fast enough (internal, never returned to the caller)
constexpr int kFixedPointFailed = 100;
// Slots of Device::ostatus used here: [0] status and [1] iterations of the
// last ORTHO_X solve, [4] Jacobi sweeps of the last eigendecomposition, [8]
// Lyapunov sweeps so far, [9] solves redone after a rediagonalisation, [10]
// eigendecompositions so far.
constexpr int kStFallbacks = 9, kStRediag = 10;

// The rediagonalisation after a failed fixed point is enqueued every step and
// decided on the device, so that a step holds no host round trip (and can be
// replayed as a CUDA graph): a gated kernel does nothing unless the ORTHO_X
// status it is given says that the fixed point failed.
__device__ __forceinline__ bool gate_closed(const int* gate) { return gate && *gate != kFixedPointFailed; }

// ---------------------------------------------------------------------------
// T[pair][t] (NBH x NBH complex) -> real (NB x NB) matrices
//   pw : plane-wave part, t=0 <X|Y>, t=1 sum X(G) Y(-G)     (both times Omega)
//   oc : one-centre part, t=0 CMAT1, t=1 CMAT2
// ---------------------------------------------------------------------------
__global__ void k_unravel(const double2* __restrict__ pw, const double2* __restrict__ oc, int npair, int nbh,
                          double* __restrict__ out0, double* __restrict__ out1, double* __restrict__ out2) {
  const int nb = 2 * nbh;
  const size_t mn = (size_t)nbh * nbh;
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  int pair = blockIdx.y;
  if (idx >= (int)mn || pair >= npair) return;
  int i = idx % nbh, j = idx / nbh;
  double* out = pair == 0 ? out0 : (pair == 1 ? out1 : out2);
  double2 t1 = pw[(pair * 2 + 0) * mn + idx], t2 = pw[(pair * 2 + 1) * mn + idx];
  double2 c1 = oc[(pair * 2 + 0) * mn + idx], c2 = oc[(pair * 2 + 1) * mn + idx];
  // one-centre: cs1 = 0.5(C1+C2), cs2 = 0.5(C1-C2)
  double cs1r = 0.5 * (c1.x + c2.x), cs1i = 0.5 * (c1.y + c2.y);
  double cs2r = 0.5 * (c1.x - c2.x), cs2i = 0.5 * (c1.y - c2.y);
  double re = 0.5 * t1.x, im = 0.5 * t1.y, re2 = 0.5 * t2.x, im2 = 0.5 * t2.y;
  const int a = 2 * i, b = 2 * j;
  out[a + (size_t)nb * b] = cs1r + (re + re2);
  out[a + (size_t)nb * (b + 1)] = cs1i + (im + im2);
  out[(a + 1) + (size_t)nb * b] = -cs2i + (-im + im2);
  out[(a + 1) + (size_t)nb * (b + 1)] = cs2r + (re - re2);
}

// Lambda = sym(RLAM0) scaled by 0.5*f_i/(f_i+f_j); real part
__global__ void k_lambda_init(const double2* __restrict__ rlam0, const double* __restrict__ occ, int nb,
                              double* __restrict__ lam) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nb * nb) return;
  int i = idx % nb, j = idx / nb;
  double2 a = rlam0[i + (size_t)nb * j];
  double2 v = a;
  if (i != j) {
    double2 b = rlam0[j + (size_t)nb * i];
    v = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
  }
  double oi = occ[i], oj = occ[j];
  if (oi + oj < 1e-12) oj = 1e-12;
  lam[idx] = v.x * 0.5 * oi / (oi + oj);
}

// 0.5*(A + A^T)
// s = sym(a); with lam non-null also lam0 = lam (the saved Lambda that a
// rediagonalised ORTHO_X restarts from), in the same launch
__global__ void k_symmetrize(const double* __restrict__ a, int n, double* __restrict__ s,
                             const double* __restrict__ lam, double* __restrict__ lam0) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * n) return;
  int i = idx % n, j = idx / n;
  s[idx] = 0.5 * (a[i + (size_t)n * j] + a[j + (size_t)n * i]);
  if (lam) lam0[idx] = lam[idx];
}

// ---------------------------------------------------------------------------
// Parallel cyclic Jacobi on a symmetric n x n matrix (n even), one CTA.
// A is held packed (upper triangle) in shared memory, V (eigenvectors) in
// shared memory when it fits, else in global memory.  Rounds follow the
// round-robin tournament ordering so that the n/2 rotations of a round act on
// disjoint index pairs; each 2x2 block [P,Q] is updated by one thread as
// J_P^T A[P,Q] J_Q.  At most max_sweeps sweeps.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int pk(int i, int j) { return i <= j ? (j * (j + 1)) / 2 + i : (i * (i + 1)) / 2 + j; }

__global__ void __launch_bounds__(1024) k_jacobi(const double* __restrict__ s_in, int n, double* __restrict__ u_out,
                                                 double* __restrict__ e_out, double* __restrict__ vglob,
                                                 int v_in_smem, double* __restrict__ aglob, int max_sweeps,
                                                 int* __restrict__ ost, const int* __restrict__ gate) {
  extern __shared__ double sm[];
  if (gate_closed(gate)) return;
  if (threadIdx.x == 0) {
    ++ost[kStRediag];
    if (gate) ++ost[kStFallbacks];
  }
  int* info = ost + 4;
  const int np = n / 2;
  // packed n(n+1)/2 matrix in shared memory, or in global memory (aglob) when
  // it does not fit (NB above about 200; through L2, slower, used only for
  // the occasional rediagonalisation)
  double* A = aglob ? aglob : sm;
  double* rc = aglob ? sm : A + (size_t)n * (n + 1) / 2;  // np cosines
  double* rs = rc + np;                                  // np sines
  int* pp = reinterpret_cast<int*>(rs + np);             // np
  int* pq = pp + np;                                     // np
  int* flag = pq + np;                                   // 1
  double* V = v_in_smem ? reinterpret_cast<double*>(flag + 2) : vglob;
  // (P, Q) of every 2x2 block, packed P | Q << 16, after V (or after flag)
  int* pqtab = v_in_smem ? reinterpret_cast<int*>(V + (size_t)n * n) : (flag + 2);
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int j = tid; j < n; j += nt)
    for (int i = 0; i <= j; ++i) A[pk(i, j)] = s_in[i + (size_t)n * j];
  __syncthreads();  // V may alias s_in when it lives in global memory
  for (size_t k = tid; k < (size_t)n * n; k += nt) {
    int i = (int)(k % n), j = (int)(k / n);
    V[k] = (i == j) ? 1.0 : 0.0;
  }
  for (int Q = tid; Q < np; Q += nt)
    for (int P = 0; P <= Q; ++P) pqtab[Q * (Q + 1) / 2 + P] = P | (Q << 16);
  __syncthreads();
  int sweep = 0;
  for (; sweep < max_sweeps; ++sweep) {
    if (tid == 0) *flag = 0;
    __syncthreads();
    for (int r = 0; r < n - 1; ++r) {
      if (tid < np) {
        int a, b;
        if (tid == 0) { a = n - 1; b = r; }
        else { a = (r + tid) % (n - 1); b = (r - tid + (n - 1)) % (n - 1); }
        int p = min(a, b), q = max(a, b);
        pp[tid] = p;
        pq[tid] = q;
        double apq = A[pk(p, q)], app = A[pk(p, p)], aqq = A[pk(q, q)];
        double c = 1.0, s = 0.0;
        // rotate unless |apq| <= 1e-14 sqrt(|app aqq|): below that the eigenvectors
        // are exact to ~1e-14, and rounding noise alone keeps |apq| near 1e-16
        if (apq != 0.0 && fabs(apq) > 1e-14 * sqrt(fabs(app * aqq))) {
          double theta = (aqq - app) / (2.0 * apq);
          double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
          c = 1.0 / sqrt(t * t + 1.0);
          s = t * c;
          *flag = 1;
        }
        rc[tid] = c;
        rs[tid] = s;
      }
      __syncthreads();
      // 2x2 blocks between pair P and pair Q (P <= Q), np*(np+1)/2 of them
      const int nblk = np * (np + 1) / 2;
      for (int k = tid; k < nblk; k += nt) {
        const int pqv = pqtab[k];
        const int P = pqv & 0xffff, Q = pqv >> 16;
        int p = pp[P], q = pq[P], r2 = pp[Q], s2 = pq[Q];
        double cP = rc[P], sP = rs[P], cQ = rc[Q], sQ = rs[Q];
        if (P == Q) {
          double apq = A[pk(p, q)], app = A[pk(p, p)], aqq = A[pk(q, q)];
          if (sP != 0.0) {
            double t = sP / cP;
            A[pk(p, p)] = app - t * apq;
            A[pk(q, q)] = aqq + t * apq;
            A[pk(p, q)] = 0.0;
          }
        } else {
          double a_pr = A[pk(p, r2)], a_ps = A[pk(p, s2)], a_qr = A[pk(q, r2)], a_qs = A[pk(q, s2)];
          // rows: J_P^T
          double b_pr = cP * a_pr - sP * a_qr, b_ps = cP * a_ps - sP * a_qs;
          double b_qr = sP * a_pr + cP * a_qr, b_qs = sP * a_ps + cP * a_qs;
          // columns: J_Q
          A[pk(p, r2)] = cQ * b_pr - sQ * b_ps;
          A[pk(p, s2)] = sQ * b_pr + cQ * b_ps;
          A[pk(q, r2)] = cQ * b_qr - sQ * b_qs;
          A[pk(q, s2)] = sQ * b_qr + cQ * b_qs;
        }
      }
      // V <- V J
      for (int k = tid; k < np * n; k += nt) {
        int P = k / n, row = k % n;
        double c = rc[P], s = rs[P];
        if (s == 0.0) continue;
        int p = pp[P], q = pq[P];
        double vp = V[row + (size_t)n * p], vq = V[row + (size_t)n * q];
        V[row + (size_t)n * p] = c * vp - s * vq;
        V[row + (size_t)n * q] = s * vp + c * vq;
      }
      __syncthreads();
    }
    if (*flag == 0) break;
    __syncthreads();
  }
  for (int i = tid; i < n; i += nt) e_out[i] = A[pk(i, i)];
  for (size_t k = tid; k < (size_t)n * n; k += nt) u_out[k] = V[k];
  if (tid == 0) info[0] = sweep;
}

// The same Jacobi iteration as one cluster of kJacCS CTAs for matrices whose
// packed triangle does not fit one CTA's shared memory (A and V in global
// memory, L2 resident).  Every CTA forms the rotations of a round itself (the
// same arithmetic on the same data, so the CTAs agree on them and on the
// convergence flag); a cluster barrier then separates those reads of A from
// the round's updates, which the CTAs share, and a second one ends the round.
constexpr int kJacCS = 8;
__global__ void __launch_bounds__(1024) k_jacobi_cl(const double* __restrict__ s_in, int n, double* __restrict__ u_out,
                                                    double* __restrict__ e_out, double* __restrict__ V,
                                                    double* __restrict__ A, int max_sweeps, int* __restrict__ ost,
                                                    const int* __restrict__ gate) {
  extern __shared__ double sm[];
  if (gate_closed(gate)) return;
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const int tid = threadIdx.x, nt = blockDim.x;
  const int gt = rank * nt + tid, gs = kJacCS * nt;
  if (rank == 0 && tid == 0) {
    ++ost[kStRediag];
    if (gate) ++ost[kStFallbacks];
  }
  int* info = ost + 4;
  const int np = n / 2;
  double* rc = sm;       // np cosines
  double* rs = rc + np;  // np sines
  int* pp = reinterpret_cast<int*>(rs + np);
  int* pq = pp + np;
  int* flag = pq + np;
  int* pqtab = flag + 2;  // (P, Q) of every 2x2 block, P | Q << 16
  for (int j = gt; j < n; j += gs)
    for (int i = 0; i <= j; ++i) A[pk(i, j)] = s_in[i + (size_t)n * j];
  for (int Q = tid; Q < np; Q += nt)
    for (int P = 0; P <= Q; ++P) pqtab[Q * (Q + 1) / 2 + P] = P | (Q << 16);
  cl.sync();  // V may alias s_in
  for (size_t k = gt; k < (size_t)n * n; k += gs) {
    int i = (int)(k % n), j = (int)(k / n);
    V[k] = (i == j) ? 1.0 : 0.0;
  }
  cl.sync();
  const int nblk = np * (np + 1) / 2;
  int sweep = 0;
  for (; sweep < max_sweeps; ++sweep) {
    if (tid == 0) *flag = 0;
    __syncthreads();
    for (int r = 0; r < n - 1; ++r) {
      if (tid < np) {
        int a, b;
        if (tid == 0) { a = n - 1; b = r; }
        else { a = (r + tid) % (n - 1); b = (r - tid + (n - 1)) % (n - 1); }
        int p = min(a, b), q = max(a, b);
        pp[tid] = p;
        pq[tid] = q;
        double apq = A[pk(p, q)], app = A[pk(p, p)], aqq = A[pk(q, q)];
        double c = 1.0, s = 0.0;
        if (apq != 0.0 && fabs(apq) > 1e-14 * sqrt(fabs(app * aqq))) {
          double theta = (aqq - app) / (2.0 * apq);
          double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
          c = 1.0 / sqrt(t * t + 1.0);
          s = t * c;
          *flag = 1;
        }
        rc[tid] = c;
        rs[tid] = s;
      }
      cl.sync();  // every CTA has read the round's pivots before any CTA rotates
      for (int k = gt; k < nblk; k += gs) {
        const int pqv = pqtab[k];
        const int P = pqv & 0xffff, Q = pqv >> 16;
        int p = pp[P], q = pq[P], r2 = pp[Q], s2 = pq[Q];
        double cP = rc[P], sP = rs[P], cQ = rc[Q], sQ = rs[Q];
        if (P == Q) {
          double apq = A[pk(p, q)], app = A[pk(p, p)], aqq = A[pk(q, q)];
          if (sP != 0.0) {
            double t = sP / cP;
            A[pk(p, p)] = app - t * apq;
            A[pk(q, q)] = aqq + t * apq;
            A[pk(p, q)] = 0.0;
          }
        } else {
          double a_pr = A[pk(p, r2)], a_ps = A[pk(p, s2)], a_qr = A[pk(q, r2)], a_qs = A[pk(q, s2)];
          double b_pr = cP * a_pr - sP * a_qr, b_ps = cP * a_ps - sP * a_qs;
          double b_qr = sP * a_pr + cP * a_qr, b_qs = sP * a_ps + cP * a_qs;
          A[pk(p, r2)] = cQ * b_pr - sQ * b_ps;
          A[pk(p, s2)] = sQ * b_pr + cQ * b_ps;
          A[pk(q, r2)] = cQ * b_qr - sQ * b_qs;
          A[pk(q, s2)] = sQ * b_qr + cQ * b_qs;
        }
      }
      for (int k = gt; k < np * n; k += gs) {
        int P = k / n, row = k % n;
        double c = rc[P], s = rs[P];
        if (s == 0.0) continue;
        int p = pp[P], q = pq[P];
        double vp = V[row + (size_t)n * p], vq = V[row + (size_t)n * q];
        V[row + (size_t)n * p] = c * vp - s * vq;
        V[row + (size_t)n * q] = s * vp + c * vq;
      }
      cl.sync();  // the round's rotations are visible to every CTA
    }
    if (*flag == 0) break;
    __syncthreads();  // every thread has read the flag before it is reset
  }
  for (int i = gt; i < n; i += gs) e_out[i] = A[pk(i, i)];
  for (size_t k = gt; k < (size_t)n * n; k += gs) u_out[k] = V[k];
  if (rank == 0 && tid == 0) info[0] = sweep;
}

// ---------------------------------------------------------------------------
// WAVES_ORTHO_X iteration as one cluster of CS CTAs.  All matrices are real,
// column-major n x n, in global memory (L2 resident).  The output tile of every
// product is split into a TRxTC grid of CTA tiles.
// ---------------------------------------------------------------------------
struct OrthoArgs {
  int n;
  const double* chichi;
  const double* psipsi;
  const double* chipsi;
  const double* u;
  const double* e;
  const double* occ;
  double* lam;    // in: start, out: result
  double* lam2;   // second buffer
  double* haux;
  double* gamn;
  double* w;
  double* maxpart;
  int* status;    // [0] status, [1] iterations
  int max_iter;
  double eps;
  int kc;
  // eigenbasis U of an earlier CHIPSI: U^T sym(CHIPSI) U = diag(e) + emat.
  // use_e = 0: emat is zero (U diagonalises the current matrix exactly)
  const double* emat;
  int use_e;
  int max_inner;
  double* gt;     // Gamma in the U basis
  double* xb;     // second buffer of the Lyapunov fixed point
  double* tb;     // E X
  int* inner;     // total inner iterations (diagnostics)
  int fast;       // lyap_fast applies (n <= 128, tiles of at most 32 x 32)
  double lyap_tol;  // relative accuracy of the Lyapunov solve (0: rounding)
  const int* gate;  // gated launch (see gate_closed) or nullptr
  int occ_equal;    // all occupations equal: the Lambda update needs no transpose
};

// C(tile) = op(A) * op(B); op = transpose when tA / tB.  The tile
// [i0,i1) x [j0,j1) has at most RA = 16*MR rows and RB = 16*MC columns.  The K
// extent is staged in chunks of KC (a multiple of 4) into smA[k][row] and
// smB[k][col] with row strides RA+4 / RB+4 doubles, then multiplied on the
// FP64 tensor cores (mma m8n8k4): the tile's 8x8 blocks are spread over the
// warps and the padded strides make the fragment reads free of bank conflicts.
// A and B may have been written by other CTAs of the cluster in the previous
// phase, so they are read through L2 (__ldcg), never through the read-only path.
template <int MR, int MC>
__host__ __device__ constexpr int tile_lda() { return 16 * MR + 4; }
template <int MR, int MC>
__host__ __device__ constexpr int tile_ldb() { return 16 * MC + 4; }

// Number of 8x8 output blocks a warp holds in gemm_acc (8 warps' worth of
// blocks spread over the CTA's warps)
template <int MR, int MC>
__host__ __device__ constexpr int tile_tpw() { return ((16 * MR / 8) * (16 * MC / 8) + 7) / 8; }

// acc += op(A) * op(B) on the tile (see gemm_tile); acc holds this thread's
// elements of its warps' 8x8 blocks
template <int MR, int MC, int KC = 128>
__device__ void gemm_acc(const double* A, bool tA, const double* B, bool tB, int n, int i0, int i1, int j0, int j1,
                         double (&acc)[tile_tpw<MR, MC>()][2], double* smA, double* smB) {
  static_assert(KC % 4 == 0, "the chunk is a whole number of k=4 MMA steps");
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  const int tm = i1 - i0, tn = j1 - j0;
  constexpr int RA = 16 * MR, RB = 16 * MC;
  constexpr int LDA = tile_lda<MR, MC>(), LDB = tile_ldb<MR, MC>();
  constexpr int TR = RA / 8, TC = RB / 8, NTILE = TR * TC;
  constexpr int TPW = (NTILE + 7) / 8;  // 8x8 blocks per warp (8 warps)
  // 16-byte staging needs even offsets of the tile and an even leading dimension
  const bool vec = (n % 2 == 0) && (i0 % 2 == 0) && (j0 % 2 == 0);
  for (int k0 = 0; k0 < n; k0 += KC) {
    const int kk = min(KC, n - k0);
    const int kk4 = (kk + 3) & ~3;
    // stage both operands (the whole chunk, zero past kk) with eight L2 loads in
    // flight per thread: the tile is tiny and the loop is bound by latency;
    // every divisor of the index arithmetic is a compile-time constant
    constexpr int totA = RA * KC, tot = totA + RB * KC;
    if (vec) {
      // pairs of neighbouring elements of the contiguous index (16-byte loads),
      // four pairs in flight per thread; a pair half past the tile or the chunk
      // is loaded alone
      constexpr int totA2 = totA / 2, tot2 = tot / 2;
      for (int base = 0; base < tot2; base += 4 * nt) {
        double2 v[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int t = base + tid + q * nt;
          v[q] = make_double2(0.0, 0.0);
          if (t < totA2) {
            if (!tA) {
              const int ii = 2 * (t % (RA / 2)), k = t / (RA / 2);
              const double* src = &A[(i0 + ii) + (size_t)n * (k0 + k)];
              if (k < kk && ii + 1 < tm) v[q] = __ldcg(reinterpret_cast<const double2*>(src));
              else if (k < kk && ii < tm) v[q].x = __ldcg(src);
            } else {
              const int k = 2 * (t % (KC / 2)), ii = t / (KC / 2);
              const double* src = &A[(k0 + k) + (size_t)n * (i0 + ii)];
              if (ii < tm && k + 1 < kk) v[q] = __ldcg(reinterpret_cast<const double2*>(src));
              else if (ii < tm && k < kk) v[q].x = __ldcg(src);
            }
          } else if (t < tot2) {
            const int u = t - totA2;
            if (!tB) {
              const int k = 2 * (u % (KC / 2)), jj = u / (KC / 2);
              const double* src = &B[(k0 + k) + (size_t)n * (j0 + jj)];
              if (jj < tn && k + 1 < kk) v[q] = __ldcg(reinterpret_cast<const double2*>(src));
              else if (jj < tn && k < kk) v[q].x = __ldcg(src);
            } else {
              const int jj = 2 * (u % (RB / 2)), k = u / (RB / 2);
              const double* src = &B[(j0 + jj) + (size_t)n * (k0 + k)];
              if (k < kk && jj + 1 < tn) v[q] = __ldcg(reinterpret_cast<const double2*>(src));
              else if (k < kk && jj < tn) v[q].x = __ldcg(src);
            }
          }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int t = base + tid + q * nt;
          if (t < totA2) {
            if (!tA) {
              const int ii = 2 * (t % (RA / 2)), k = t / (RA / 2);
              *reinterpret_cast<double2*>(&smA[k * LDA + ii]) = v[q];
            } else {
              const int k = 2 * (t % (KC / 2)), ii = t / (KC / 2);
              smA[k * LDA + ii] = v[q].x;
              smA[(k + 1) * LDA + ii] = v[q].y;
            }
          } else if (t < tot2) {
            const int u = t - totA2;
            if (!tB) {
              const int k = 2 * (u % (KC / 2)), jj = u / (KC / 2);
              smB[k * LDB + jj] = v[q].x;
              smB[(k + 1) * LDB + jj] = v[q].y;
            } else {
              const int jj = 2 * (u % (RB / 2)), k = u / (RB / 2);
              *reinterpret_cast<double2*>(&smB[k * LDB + jj]) = v[q];
            }
          }
        }
      }
    }
    for (int base = vec ? tot : 0; base < tot; base += 8 * nt) {
      double v[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int t = base + tid + q * nt;
        v[q] = 0.0;
        if (t < totA) {
          int ii, k;
          if (!tA) { ii = t % RA; k = t / RA; } else { k = t % KC; ii = t / KC; }
          if (ii < tm && k < kk)
            v[q] = __ldcg(!tA ? &A[(i0 + ii) + (size_t)n * (k0 + k)] : &A[(k0 + k) + (size_t)n * (i0 + ii)]);
        } else if (t < tot) {
          const int u = t - totA;
          int jj, k;
          if (!tB) { k = u % KC; jj = u / KC; } else { jj = u % RB; k = u / RB; }
          if (jj < tn && k < kk)
            v[q] = __ldcg(!tB ? &B[(k0 + k) + (size_t)n * (j0 + jj)] : &B[(j0 + jj) + (size_t)n * (k0 + k)]);
        }
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int t = base + tid + q * nt;
        if (t < totA) {
          int ii, k;
          if (!tA) { ii = t % RA; k = t / RA; } else { k = t % KC; ii = t / KC; }
          smA[k * LDA + ii] = v[q];
        } else if (t < tot) {
          const int u = t - totA;
          int jj, k;
          if (!tB) { k = u % KC; jj = u / KC; } else { jj = u % RB; k = u / RB; }
          smB[k * LDB + jj] = v[q];
        }
      }
    }
    __syncthreads();
    const int fr = lane >> 2, fk = lane & 3;
#pragma unroll
    for (int q = 0; q < TPW; ++q) {
      const int t = warp + q * nw;
      if (t < NTILE) {
        const int r0 = (t % TR) * 8, c0 = (t / TR) * 8;
        // two independent MMA chains (even and odd k steps) to hide the MMA latency
        double a2[2] = {0.0, 0.0};
        for (int k = 0; k < kk4; k += 8) {
          dmma(acc[q], smA[(k + fk) * LDA + r0 + fr], smB[(k + fk) * LDB + c0 + fr]);
          if (k + 4 < kk4) dmma(a2, smA[(k + 4 + fk) * LDA + r0 + fr], smB[(k + 4 + fk) * LDB + c0 + fr]);
        }
        acc[q][0] += a2[0];
        acc[q][1] += a2[1];
      }
    }
    __syncthreads();
  }
}

// calls f(i, j, value) for this thread's elements of the tile
template <int MR, int MC, class F>
__device__ __forceinline__ void tile_each(const double (&acc)[tile_tpw<MR, MC>()][2], int i0, int i1, int j0, int j1,
                                          F&& f) {
  constexpr int TR = 16 * MR / 8, TC = 16 * MC / 8, NTILE = TR * TC, TPW = tile_tpw<MR, MC>();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int tm = i1 - i0, tn = j1 - j0;
#pragma unroll
  for (int q = 0; q < TPW; ++q) {
    const int t = warp + q * nw;
    if (t < NTILE) {
      const int ii = (t % TR) * 8 + (lane >> 2);
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int jj = (t / TR) * 8 + 2 * (lane & 3) + e;
        if (ii < tm && jj < tn) f(i0 + ii, j0 + jj, acc[q][e]);
      }
    }
  }
}

template <int MR, int MC, int KC = 128>
__device__ void gemm_tile(const double* A, bool tA, const double* B, bool tB, int n, int i0, int i1, int j0, int j1,
                          double* C, double* smA, double* smB) {
  double acc[tile_tpw<MR, MC>()][2];
#pragma unroll
  for (int q = 0; q < tile_tpw<MR, MC>(); ++q) acc[q][0] = acc[q][1] = 0.0;
  gemm_acc<MR, MC, KC>(A, tA, B, tB, n, i0, i1, j0, j1, acc, smA, smB);
  tile_each<MR, MC>(acc, i0, i1, j0, j1, [&](int i, int j, double v) { C[i + (size_t)n * j] = v; });
  // callers read the tile back with another thread-to-element map
  __syncthreads();
}

// maxima of (a, b) over the CTA: warp shuffles, then one pass over the warps
// (red holds at least 64 doubles; every thread gets the result)
__device__ __forceinline__ void block_max2(double& a, double& b, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
    b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
  }
  if (lane == 0) {
    red[warp] = a;
    red[32 + warp] = b;
  }
  __syncthreads();
  a = red[0];
  b = red[32];
  for (int w = 1; w < nw; ++w) {
    a = fmax(a, red[w]);
    b = fmax(b, red[32 + w]);
  }
  __syncthreads();
}

// Maxima over the cluster's partials mp[0..cs) and mp[cs..2cs) (cs <= 32):
// one L2 read per lane, then a warp reduction, instead of a chain of reads.
__device__ __forceinline__ void cluster_max2(const double* mp, int cs, double& a, double& b) {
  const int lane = threadIdx.x & 31;
  a = lane < cs ? __ldcg(&mp[lane]) : 0.0;
  b = lane < cs ? __ldcg(&mp[cs + lane]) : 0.0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
    b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
  }
}

// Barrier of the cluster.  Its arrive/wait pair has release/acquire semantics
// at cluster scope, which orders the global-memory writes of every CTA before
// the other CTAs' later reads (all done through L2, __ldcg); no GPU-scope
// fence is needed because every reader is in the cluster.
__device__ __forceinline__ void csync() { cg::this_cluster().sync(); }

// Convergence rule of the Lyapunov fixed point (shared by both loops): true to
// stop; `failed` when the contraction is too slow (the earlier eigenbasis is
// too far from the current one) or there is no convergence within the limit.
__device__ __forceinline__ bool lyap_stop(double gdx, double gxm, double& prev, int it2, int max_inner, double tol,
                                          bool& failed) {
  const double ratio = gdx / prev;
  prev = gdx;
  // requested accuracy reached (the sweep's change bounds the error of a
  // contraction well below one)
  if (gdx <= tol * gxm) return true;
  // converged: change at rounding level, or stalled just above it
  if (gdx <= 4e-16 * gxm || (gdx <= 1e-13 * gxm && ratio > 0.5)) return true;
  if ((it2 >= 4 && ratio > 0.6) || it2 == max_inner - 1 || !(gdx <= 1e200)) {
    failed = true;
    return true;
  }
  return false;
}

// Lyapunov fixed point X <- (GT - E X - X E) / (e_i + e_j) for n <= 128 and
// CTA tiles of at most 32 x 32.  The CTA keeps its slices of the constant E
// in shared memory (rows i0..i1 for E X, columns j0..j1 for X E), stages the
// X slices it needs once per sweep, forms both products of its tile on the
// FP64 tensor cores and updates its X tile in registers; one cluster barrier
// per sweep.  Returns the buffer that holds the last iterate.
template <int MR, int MC>
__device__ double* lyap_fast(const OrthoArgs& a, int cs, int rank, int i0, int i1, int j0, int j1, double* sm,
                             double* red, double* xcur, double* xnext, bool& failed, double& rho_io) {
  constexpr int RA = 16 * MR, RB = 16 * MC, LDA = RA + 4;
  constexpr int TR = RA / 8, TC = RB / 8, NTILE = TR * TC, TPW = (NTILE + 7) / 8;
  // the slices always hold KN = 128 rows of k (zero past n), so that every
  // divisor of the staging index arithmetic is a compile-time constant
  constexpr int KN = 128;
  const int n = a.n, n4 = (n + 3) & ~3;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  const int fr = lane >> 2, fk = lane & 3;
  const int tm = i1 - i0, tn = j1 - j0;
  // Column slices are held column by column ([jj][k], stride LDK = KN + 4):
  // the staging stores run along k and stay free of bank conflicts, and so do
  // the B-fragment reads (LDK = 4 mod 16 doubles).  Row slices are [k][ii].
  constexpr int LDK = KN + 4;
  double* Er = sm;              // Er[k][ii] = E(i0+ii, k)
  double* Ec = Er + LDA * KN;   // Ec[jj][k] = E(k, j0+jj)
  double* Xc = Ec + RB * LDK;   // Xc[jj][k] = X(k, j0+jj)
  double* Xr = Xc + RB * LDK;   // Xr[k][ii] = X(i0+ii, k)
  for (int t = tid; t < KN * RA; t += nt) {
    const int ii = t % RA, k = t / RA;
    Er[k * LDA + ii] = (ii < tm && k < n) ? __ldcg(&a.emat[(i0 + ii) + (size_t)n * k]) : 0.0;
  }
  for (int t = tid; t < KN * RB; t += nt) {
    const int k = t % KN, jj = t / KN;
    Ec[jj * LDK + k] = (jj < tn && k < n) ? __ldcg(&a.emat[k + (size_t)n * (j0 + jj)]) : 0.0;
  }
  // this lane's elements of the tile: right-hand side, denominator, iterate
  // and the iterate before it (Chebyshev recurrence)
  double gtv[TPW][2], den[TPW][2], xp[TPW][2], xq[TPW][2];
  int eidx[TPW][2];
#pragma unroll
  for (int q = 0; q < TPW; ++q) {
    const int t = warp + q * nw;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int ii = (t % TR) * 8 + fr, jj = (t / TR) * 8 + 2 * fk + e;
      const bool ok = t < NTILE && ii < tm && jj < tn;
      eidx[q][e] = ok ? (i0 + ii) + n * (j0 + jj) : -1;
      gtv[q][e] = ok ? __ldcg(&a.gt[eidx[q][e]]) : 0.0;
      den[q][e] = ok ? a.e[i0 + ii] + a.e[j0 + jj] : 1.0;
      xp[q][e] = ok ? __ldcg(&xcur[eidx[q][e]]) : 0.0;
      xq[q][e] = xp[q][e];
    }
  }
  // Chebyshev acceleration: the map X -> -(E X + X E)/(e_i + e_j) is self-adjoint
  // in the inner product weighted by e_i + e_j, so its spectrum is real, in
  // [-rho, rho].  Three plain sweeps estimate rho from the ratio of successive
  // changes (with a margin; an estimate below the true rho still contracts),
  // then x_{k+1} = w (F(x_k) - x_{k-1}) + x_{k-1} with the Chebyshev weights.
  // E and e are the same in every ORTHO_X iteration of a launch, and so is
  // rho: a later solve (rho_io > 0) starts the weights after one plain sweep.
  double prev = INFINITY, rho = rho_io, omega = 1.0;
  const int cheb0 = rho > 0.0 ? 0 : 2;  // sweep after which the weights start
  failed = false;
  for (int it2 = 0; it2 < a.max_inner; ++it2) {
    double* mp = a.maxpart + (it2 & 1) * 2 * cs;
    // stage X(:, j0:j1) and X(i0:i1, :), sixteen loads in flight per thread
    constexpr int totc = KN * RB, tot = totc + KN * RA;
    for (int base = 0; base < tot; base += 16 * nt) {
      double v[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int t = base + tid + q * nt;
        v[q] = 0.0;
        if (t < totc) {
          const int k = t % KN, jj = t / KN;
          if (jj < tn && k < n) v[q] = __ldcg(&xcur[k + (size_t)n * (j0 + jj)]);
        } else if (t < tot) {
          const int u = t - totc, ii = u % RA, k = u / RA;
          if (ii < tm && k < n) v[q] = __ldcg(&xcur[(i0 + ii) + (size_t)n * k]);
        }
      }
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int t = base + tid + q * nt;
        if (t < totc) {
          const int k = t % KN, jj = t / KN;
          Xc[jj * LDK + k] = v[q];
        } else if (t < tot) {
          const int u = t - totc, ii = u % RA, k = u / RA;
          Xr[k * LDA + ii] = v[q];
        }
      }
    }
    __syncthreads();
    double dx = 0.0, xm = 0.0;
#pragma unroll
    for (int q = 0; q < TPW; ++q) {
      const int t = warp + q * nw;
      if (t >= NTILE) continue;
      const int r0 = (t % TR) * 8, c0 = (t / TR) * 8;
      // four independent accumulation chains (two per product, even and odd
      // k steps) to hide the MMA latency
      double ex[2] = {0.0, 0.0}, xe[2] = {0.0, 0.0}, ex1[2] = {0.0, 0.0}, xe1[2] = {0.0, 0.0};
      for (int k = 0; k < n4; k += 8) {
        dmma(ex, Er[(k + fk) * LDA + r0 + fr], Xc[(c0 + fr) * LDK + k + fk]);
        dmma(xe, Xr[(k + fk) * LDA + r0 + fr], Ec[(c0 + fr) * LDK + k + fk]);
        if (k + 4 < n4) {
          dmma(ex1, Er[(k + 4 + fk) * LDA + r0 + fr], Xc[(c0 + fr) * LDK + k + 4 + fk]);
          dmma(xe1, Xr[(k + 4 + fk) * LDA + r0 + fr], Ec[(c0 + fr) * LDK + k + 4 + fk]);
        }
      }
      ex[0] += ex1[0];
      ex[1] += ex1[1];
      xe[0] += xe1[0];
      xe[1] += xe1[1];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        if (eidx[q][e] < 0) continue;
        const double fx = (gtv[q][e] - ex[e] - xe[e]) / den[q][e];
        const double xn = omega * (fx - xq[q][e]) + xq[q][e];
        dx = fmax(dx, fabs(xn - xp[q][e]));
        xm = fmax(xm, fabs(xn));
        xq[q][e] = xp[q][e];
        xp[q][e] = xn;
        xnext[eidx[q][e]] = xn;
      }
    }
    block_max2(dx, xm, red);  // its barriers also end this sweep's reads of Xc / Xr
    if (tid == 0) {
      mp[rank] = dx;
      mp[cs + rank] = xm;
    }
    csync();
    double gdx, gxm;
    cluster_max2(mp, cs, gdx, gxm);
    double* tmpx = xcur;
    xcur = xnext;
    xnext = tmpx;
    if (rank == 0 && tid == 0) a.inner[0] += 1;
    const double ratio = gdx / prev;
    if (lyap_stop(gdx, gxm, prev, it2, a.max_inner, a.lyap_tol, failed)) break;
    if (it2 == cheb0) {
      if (cheb0 == 2) rho_io = rho = fmin(0.9, fmax(0.05, 1.1 * ratio));
      omega = 1.0 / (1.0 - 0.5 * rho * rho);
    } else if (it2 > cheb0) {
      omega = 1.0 / (1.0 - 0.25 * rho * rho * omega);
    }
  }
  return xcur;
}

template <int MR, int MC>
__global__ void __launch_bounds__(512) k_ortho_x(OrthoArgs a) {
  // (a gated launch reads the gate before any CTA of the cluster can reach
  // the status write at the end: every CTA leaves together or none does)
  if (gate_closed(a.gate)) return;
  extern __shared__ double sm[];
  cg::cluster_group cl = cg::this_cluster();
  const int cs = (int)cl.num_blocks(), rank = (int)cl.block_rank();
  const int n = a.n;
  // CTA tile grid: tr x tc
  int tr = 1;
  while (tr * tr < cs) tr *= 2;
  int tc = cs / tr;
  if (tr * tc != cs) { tr = cs; tc = 1; }
  const int ri = rank / tc, ci = rank % tc;
  const int rs = (n + tr - 1) / tr, csz = (n + tc - 1) / tc;
  const int i0 = min(n, ri * rs), i1 = min(n, i0 + rs);
  const int j0 = min(n, ci * csz), j1 = min(n, j0 + csz);
  double* smA = sm;
  double* smB = sm + (size_t)tile_lda<MR, MC>() * a.kc;
  const int tid = threadIdx.x, nt = blockDim.x;
  double* lam = a.lam;
  double* lamn = a.lam2;
  __shared__ double red[256];
  int status = CUW_ERR_NOT_CONVERGED, iters = a.max_iter;
  double rho_known = 0.0;  // contraction of the Lyapunov map, once estimated (lyap_fast)
  for (int iter = 1; iter <= a.max_iter; ++iter) {
    // The reference forms GAMN = LAMBDA^T (CHICHI LAMBDA + 2 CHIPSI) and then
    // W = 0.5 (GAMN + GAMN^T) + PSIPSI - 1 (PSIPSI of the upper triangle).
    // With CHICHI symmetric that is
    //   W = LAMBDA^T (CHICHI LAMBDA + CHIPSI) + CHIPSI^T LAMBDA + PSIPSI - 1,
    // whose tile needs no transposed tile: one product phase and one barrier
    // fewer per iteration (the same matrix to rounding).
    // HAUX = CHICHI * LAMBDA + CHIPSI
    gemm_tile<MR, MC>(a.chichi, false, lam, false, n, i0, i1, j0, j1, a.haux, smA, smB);
    for (int t = tid; t < (i1 - i0) * (j1 - j0); t += nt) {
      int i = i0 + t % (i1 - i0), j = j0 + t / (i1 - i0);
      a.haux[i + (size_t)n * j] = __ldcg(&a.haux[i + (size_t)n * j]) + a.chipsi[i + (size_t)n * j];
    }
    csync();
    // W = LAMBDA^T HAUX + CHIPSI^T LAMBDA + PSIPSI - 1 ; tile max
    double mx = 0.0;
    {
      double acc[tile_tpw<MR, MC>()][2];
#pragma unroll
      for (int q = 0; q < tile_tpw<MR, MC>(); ++q) acc[q][0] = acc[q][1] = 0.0;
      gemm_acc<MR, MC>(lam, true, a.haux, false, n, i0, i1, j0, j1, acc, smA, smB);
      gemm_acc<MR, MC>(a.chipsi, true, lam, false, n, i0, i1, j0, j1, acc, smA, smB);
      tile_each<MR, MC>(acc, i0, i1, j0, j1, [&](int i, int j, double g) {
        double v = g + a.psipsi[min(i, j) + (size_t)n * max(i, j)];
        if (i == j) v -= 1.0;
        a.w[i + (size_t)n * j] = v;
        mx = fmax(mx, fabs(v));
        if (v != v) mx = INFINITY;
      });
    }
    // CTA max (NaN propagates as infinity)
    double unused = 0.0;
    block_max2(mx, unused, red);
    if (tid == 0) a.maxpart[rank] = mx;
    csync();
    double digam, unused2;
    cluster_max2(a.maxpart, cs, digam, unused2);
    if (digam < a.eps) {
      status = CUW_OK;
      iters = iter;
      break;
    }
    if (!(digam <= 1e200)) {
      status = CUW_ERR_DIVERGED;
      iters = iter;
      break;
    }
    // HAUX = U^T W
    gemm_tile<MR, MC>(a.u, true, a.w, false, n, i0, i1, j0, j1, a.haux, smA, smB);
    csync();
    // GT = HAUX U (Gamma in the U basis);  X = GT / (e_i + e_j)
    gemm_tile<MR, MC>(a.haux, false, a.u, false, n, i0, i1, j0, j1, a.gt, smA, smB);
    for (int t = tid; t < (i1 - i0) * (j1 - j0); t += nt) {
      int i = i0 + t % (i1 - i0), j = j0 + t / (i1 - i0);
      a.gamn[i + (size_t)n * j] = __ldcg(&a.gt[i + (size_t)n * j]) / (a.e[i] + a.e[j]);
    }
    csync();
    // When U diagonalises an earlier CHIPSI only, D X + X D = GT - E X - X E is
    // solved by the fixed point X <- (GT - E X - X E)/(e_i + e_j) to rounding
    // level: the same Lyapunov solution as the eigendecomposition of the
    // current matrix.
    double* xcur = a.gamn;
    double* xnext = a.xb;
    bool fp_failed = false;
    if (a.use_e && a.fast) {
      if constexpr (MR <= 2 && MC <= 2)
        xcur = lyap_fast<MR, MC>(a, cs, rank, i0, i1, j0, j1, sm, red, xcur, xnext, fp_failed, rho_known);
    } else if (a.use_e) {
      double prev = INFINITY;
      // one cluster barrier per sweep: E X and X E are both formed on this
      // CTA's tile (X E = (E X)^T would need another CTA's tile), and the
      // convergence partials alternate between two halves of maxpart
      for (int it2 = 0; it2 < a.max_inner; ++it2) {
        double* mp = a.maxpart + (it2 & 1) * 2 * cs;
        gemm_tile<MR, MC>(a.emat, false, xcur, false, n, i0, i1, j0, j1, a.tb, smA, smB);
        gemm_tile<MR, MC>(xcur, false, a.emat, false, n, i0, i1, j0, j1, a.haux, smA, smB);
        double dx = 0.0, xm = 0.0;
        for (int t = tid; t < (i1 - i0) * (j1 - j0); t += nt) {
          int i = i0 + t % (i1 - i0), j = j0 + t / (i1 - i0);
          double xn = (__ldcg(&a.gt[i + (size_t)n * j]) - __ldcg(&a.tb[i + (size_t)n * j]) -
                       __ldcg(&a.haux[i + (size_t)n * j])) / (a.e[i] + a.e[j]);
          dx = fmax(dx, fabs(xn - __ldcg(&xcur[i + (size_t)n * j])));
          xm = fmax(xm, fabs(xn));
          xnext[i + (size_t)n * j] = xn;
        }
        block_max2(dx, xm, red);
        if (tid == 0) {
          mp[rank] = dx;
          mp[cs + rank] = xm;
        }
        csync();
        double gdx, gxm;
        cluster_max2(mp, cs, gdx, gxm);
        double* tmpx = xcur;
        xcur = xnext;
        xnext = tmpx;
        if (rank == 0 && tid == 0) a.inner[0] += 1;
        if (lyap_stop(gdx, gxm, prev, it2, a.max_inner, a.lyap_tol, fp_failed)) break;
      }
    }
    if (fp_failed) {
      status = kFixedPointFailed;
      iters = iter;
      break;
    }
    // HAUX = U X
    gemm_tile<MR, MC>(a.u, false, xcur, false, n, i0, i1, j0, j1, a.haux, smA, smB);
    csync();
    if (a.occ_equal) {
      // equal occupations: LAMBDA(I,J) -= W(I,J) (the weight 2 OCCI/(OCCI+OCCJ)
      // is 1 and the symmetrisation rule never applies), straight from the
      // product tile W = HAUX U^T
      double acc[tile_tpw<MR, MC>()][2];
#pragma unroll
      for (int q = 0; q < tile_tpw<MR, MC>(); ++q) acc[q][0] = acc[q][1] = 0.0;
      gemm_acc<MR, MC>(a.haux, false, a.u, true, n, i0, i1, j0, j1, acc, smA, smB);
      tile_each<MR, MC>(acc, i0, i1, j0, j1, [&](int i, int j, double wv) {
        lamn[i + (size_t)n * j] = __ldcg(&lam[i + (size_t)n * j]) - wv;
      });
      csync();
      double* tmp = lam;
      lam = lamn;
      lamn = tmp;
      continue;
    }
    // W = HAUX U^T
    gemm_tile<MR, MC>(a.haux, false, a.u, true, n, i0, i1, j0, j1, a.w, smA, smB);
    csync();
    // LAMBDA(I,J) -= 2 OCCI/(OCCI+OCCJ) W(I,J); then occupation symmetrisation
    const double dsmall = 1e-12;
    for (int t = tid; t < (i1 - i0) * (j1 - j0); t += nt) {
      int i = i0 + t % (i1 - i0), j = j0 + t / (i1 - i0);
      double oi = a.occ[i], oj = a.occ[j];
      double v;
      if (oi < oj) {
        double occj = oj + dsmall, occi = oi + dsmall;
        double lji = __ldcg(&lam[j + (size_t)n * i]) - 2.0 * occj / (occj + occi) * __ldcg(&a.w[j + (size_t)n * i]);
        v = lji * (oi + dsmall) / (oj + dsmall);
      } else {
        double occi = oi + dsmall, occj = oj + dsmall;
        v = __ldcg(&lam[i + (size_t)n * j]) - 2.0 * occi / (occi + occj) * __ldcg(&a.w[i + (size_t)n * j]);
      }
      lamn[i + (size_t)n * j] = v;
    }
    csync();
    double* tmp = lam;
    lam = lamn;
    lamn = tmp;
  }
  // result into a.lam
  if (lam != a.lam) {
    for (int t = tid; t < (i1 - i0) * (j1 - j0); t += nt) {
      int i = i0 + t % (i1 - i0), j = j0 + t / (i1 - i0);
      a.lam[i + (size_t)n * j] = __ldcg(&lam[i + (size_t)n * j]);
    }
  }
  if (rank == 0 && tid == 0) {
    a.status[0] = status;
    a.status[1] = iters;
  }
  csync();
}

// ---------------------------------------------------------------------------
// ORTHO_X for 64 < n <= 128 with equal occupations, as one cluster of 16 CTAs
// in a 4 x 4 grid: CTA (ri, ci) owns the 32 x 32 tile (ri, ci) of every
// product.  The matrices live in global memory (L2: 128 KB each); a product
// tile op(A) op(B) stages its two operand panels (32 x n and n x 32) into
// shared memory with 16-byte loads of whole column segments, each panel in
// the one of two layouts that keeps the MMA fragment reads free of bank
// conflicts for its orientation:
//   row panel    rows i0..i0+31 of all columns k: [k][r], stride PR = 36
//                (A, or B transposed: column segments of 32 elements)
//   column panel columns j0..j0+31, all rows k:  [c][k], stride PC = 132
//                (B, or A transposed: whole columns)
// then multiplies on the FP64 tensor cores (m8n8k4), each warp one 8 x 8
// block with two accumulation chains.  The elementwise operands of the
// iteration (CHIPSI, PSIPSI, Gamma, the denominators, Lambda) stay in the
// registers of the lanes that own the elements.  One cluster barrier ends
// every phase (its release/acquire orders the global writes of a phase before
// the next phase's reads, all through L2); the maxima of a phase are
// exchanged through shared-memory slots of the cluster.  The arithmetic and
// the phases are those of k_ortho_x with the same stopping rules.
// ---------------------------------------------------------------------------
namespace pnl {
constexpr int T = 32, G = 4, KN = 128;
constexpr int PR = T + 4;    // row panel stride ([k][r])
constexpr int PC = KN + 4;   // column panel stride ([c][k])
constexpr int RSZ = KN * PR, CSZ = T * PC;  // doubles of one row / column panel
// two terms, each an A and a B panel of either kind (sized for the larger)
constexpr int PSZ = RSZ > CSZ ? RSZ : CSZ;
// four staging panels, the two resident panels of E (row panel at i0, column
// panel at j0) and the maxima slots
constexpr size_t kSmemBytes = sizeof(double) * ((size_t)4 * PSZ + RSZ + CSZ + 64);
}  // namespace pnl

// 16-byte asynchronous copy global -> shared through L2 (cp.async.cg: the
// source may have been written by another CTA of the cluster in the previous
// phase); a null source writes zeros.
__device__ const double2 pnl_zero[1] = {{0.0, 0.0}};
__device__ __forceinline__ void pnl_cp16(double* dst, const double* src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d),
               "l"(src ? src : reinterpret_cast<const double*>(pnl_zero)), "r"(src ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void pnl_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void pnl_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Issues the copies that stage op(M) as the A operand (rows i0.. of the
// product, all k) or as the B operand (all k, columns j0..) of a product tile
// into dst.  M is n x n column-major in global memory (n even, so column
// segments are 16-byte aligned); elements outside n x n are zero.  Every
// copy of the panel is in flight before the caller waits for them.
__device__ __forceinline__ void pnl_stage(const double* __restrict__ M, int n, int off, bool row_panel,
                                          double* __restrict__ dst) {
  using namespace pnl;
  const int tid = threadIdx.x, nt = blockDim.x;
  if (row_panel) {
    // rows off..off+31 of every column k: 16 double2 per column
    for (int t = tid; t < KN * (T / 2); t += nt) {
      const int k = t / (T / 2), r2 = (t % (T / 2)) * 2;
      pnl_cp16(dst + k * PR + r2, (k < n && off + r2 < n) ? M + (size_t)n * k + off + r2 : nullptr);
    }
  } else {
    // columns off..off+31, every row k: 64 double2 per column
    for (int t = tid; t < T * (KN / 2); t += nt) {
      const int c = t / (KN / 2), k2 = (t % (KN / 2)) * 2;
      pnl_cp16(dst + c * PC + k2, (off + c < n && k2 < n) ? M + (size_t)n * (off + c) + k2 : nullptr);
    }
  }
}

// One product term op(A) op(B) of a tile: the panels and how to read them.
//   A normal: row panel of A at rows i0      -> element (i, k) at k*PR + i
//   A transposed: column panel of A at cols i0 -> (i, k) = A(k, i) at i*PC + k
//   B normal: column panel of B at cols j0   -> (k, j) at j*PC + k
//   B transposed: row panel of B at rows j0  -> (k, j) = B(j, k) at k*PR + j
struct PnlTerm {
  const double* a;
  bool ta;
  const double* b;
  bool tb;
};

__device__ __forceinline__ void pnl_stage_term(const PnlTerm& t, int n, int i0, int j0, double* sa, double* sb) {
  pnl_stage(t.a, n, i0, !t.ta, sa);
  pnl_stage(t.b, n, j0, t.tb, sb);
}

// acc (two chains) += op(A) op(B) for this warp's 8 x 8 block
__device__ __forceinline__ void pnl_mma(const PnlTerm& t, int nk4, const double* sa, const double* sb, int r0,
                                        int c0, double (&acc)[2], double (&acc2)[2]) {
  using namespace pnl;
  const int lane = threadIdx.x & 31, fr = lane >> 2, fk = lane & 3;
  const double* pa = t.ta ? sa + (r0 + fr) * PC + fk : sa + fk * PR + r0 + fr;
  const int as = t.ta ? 4 : 4 * PR;
  const double* pb = t.tb ? sb + fk * PR + c0 + fr : sb + (c0 + fr) * PC + fk;
  const int bs = t.tb ? 4 * PR : 4;
#pragma unroll 4
  for (int s = 0; s < nk4; s += 2) {
    dmma(acc, pa[s * as], pb[s * bs]);
    if (s + 1 < nk4) dmma(acc2, pa[(s + 1) * as], pb[(s + 1) * bs]);
  }
}

__global__ void __launch_bounds__(512, 1) k_ortho_x_pnl(OrthoArgs a) {
  using namespace pnl;
  if (gate_closed(a.gate)) return;
  extern __shared__ double sm[];
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const int ri = rank / G, ci = rank % G;
  const int n = a.n, nk4 = (n + 3) / 4;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
  const int fr = lane >> 2, fk = lane & 3;
  const int r0 = (warp % 4) * 8, c0 = (warp / 4) * 8;  // this warp's 8 x 8 block of the tile
  const int i0 = ri * T, j0 = ci * T;
  double* sa0 = sm;
  double* sb0 = sm + PSZ;
  double* sa1 = sm + 2 * PSZ;
  double* sb1 = sm + 3 * PSZ;
  double* er = sm + 4 * PSZ;       // E rows i0..i0+31 (row panel), resident
  double* ec = er + RSZ;           // E columns j0..j0+31 (column panel), resident
  double* slotmax = ec + CSZ;      // [2 parities][x: 16 ranks, y: 16 ranks]
  // this lane's two elements (gi, gj0 + e) of the tile
  const int gi = i0 + r0 + fr, gjb = j0 + c0 + 2 * fk;
  bool ok[2];
  size_t gidx[2];
  double cp[2], pp[2], lamv[2], den[2];
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    const int gj = gjb + e;
    ok[e] = gi < n && gj < n;
    gidx[e] = ok[e] ? (size_t)gi + (size_t)n * gj : 0;
    cp[e] = ok[e] ? a.chipsi[gidx[e]] : 0.0;
    pp[e] = ok[e] ? a.psipsi[min(gi, gj) + (size_t)n * max(gi, gj)] : 0.0;
    lamv[e] = ok[e] ? __ldcg(&a.lam[gidx[e]]) : 0.0;
    den[e] = ok[e] ? a.e[gi] + a.e[gj] : 1.0;
  }
  auto put = [&](double* M, const double (&v)[2]) {
#pragma unroll
    for (int e = 0; e < 2; ++e)
      if (ok[e]) M[gidx[e]] = v[e];
  };
  // one product tile: stage both terms (the second may be absent), multiply
  auto product = [&](const PnlTerm& t1, const PnlTerm* t2, double (&out)[2]) {
    pnl_stage_term(t1, n, i0, j0, sa0, sb0);
    pnl_commit();
    if (t2) {
      pnl_stage_term(*t2, n, i0, j0, sa1, sb1);
      pnl_commit();
      pnl_wait<1>();  // the first term's panels; the second's stay in flight
    } else {
      pnl_wait<0>();
    }
    __syncthreads();
    double acc[2] = {0.0, 0.0}, acc2[2] = {0.0, 0.0};
    pnl_mma(t1, nk4, sa0, sb0, r0, c0, acc, acc2);
    out[0] = acc[0] + acc2[0];
    out[1] = acc[1] + acc2[1];
    if (t2) {
      pnl_wait<0>();
      __syncthreads();
      double bcc[2] = {0.0, 0.0}, bcc2[2] = {0.0, 0.0};
      pnl_mma(*t2, nk4, sa1, sb1, r0, c0, bcc, bcc2);
      out[0] += bcc[0] + bcc2[0];
      out[1] += bcc[1] + bcc2[1];
    }
    __syncthreads();  // the panels are free for the next stage
  };
  // Cluster maxima of (x, y).  Warp 0 reduces the CTA's warps and its lanes
  // 0..15 store the CTA's pair into slot [par][rank] of every CTA of the
  // cluster (remote stores, ordered by the barrier's release); after the
  // barrier every CTA reduces its own 16 slots.  A slot of parity par is
  // written again two calls later, after a barrier that every CTA reaches
  // only once it has read it.
  __shared__ double red[64];
  auto cmax2 = [&](double x, double y, int par, double& gx, double& gy) {
    for (int o = 16; o > 0; o >>= 1) {
      x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
      y = fmax(y, __shfl_xor_sync(0xffffffffu, y, o));
    }
    if (lane == 0) {
      red[warp] = x;
      red[32 + warp] = y;
    }
    __syncthreads();
    if (warp == 0) {
      const int nw = nt / 32;
      double bx = lane < nw ? red[lane] : 0.0, by = lane < nw ? red[32 + lane] : 0.0;
      for (int o = 16; o > 0; o >>= 1) {
        bx = fmax(bx, __shfl_xor_sync(0xffffffffu, bx, o));
        by = fmax(by, __shfl_xor_sync(0xffffffffu, by, o));
      }
      if (lane < 16) {
        double* rs = cl.map_shared_rank(slotmax, lane);
        rs[par * 32 + rank] = bx;
        rs[par * 32 + 16 + rank] = by;
      }
    }
    cl.sync();
    double vx = slotmax[par * 32 + (lane & 15)], vy = slotmax[par * 32 + 16 + (lane & 15)];
    for (int o = 8; o > 0; o >>= 1) {
      vx = fmax(vx, __shfl_xor_sync(0xffffffffu, vx, o));
      vy = fmax(vy, __shfl_xor_sync(0xffffffffu, vy, o));
    }
    gx = vx;
    gy = vy;
  };
  // E X + X E for a Lyapunov sweep: the E panels are resident, the X panels
  // staged (both in flight before the first multiply)
  auto sweep_product = [&](const double* x, double (&out)[2]) {
    pnl_stage(x, n, j0, false, sb0);  // X columns j0.. (B of E X)
    pnl_commit();
    pnl_stage(x, n, i0, true, sa1);   // X rows i0.. (A of X E)
    pnl_commit();
    pnl_wait<1>();
    __syncthreads();
    double acc[2] = {0.0, 0.0}, acc2[2] = {0.0, 0.0};
    pnl_mma({a.emat, false, x, false}, nk4, er, sb0, r0, c0, acc, acc2);
    pnl_wait<0>();
    __syncthreads();
    pnl_mma({x, false, a.emat, false}, nk4, sa1, ec, r0, c0, acc, acc2);
    out[0] = acc[0] + acc2[0];
    out[1] = acc[1] + acc2[1];
    __syncthreads();  // the staged panels are free for the next stage
  };
  if (a.use_e) {
    pnl_stage(a.emat, n, i0, true, er);
    pnl_stage(a.emat, n, j0, false, ec);
    pnl_commit();  // waited for with the first product's copies
  }
  int status = CUW_ERR_NOT_CONVERGED, iters = a.max_iter;
  double rho_known = 0.0;
  int par = 0, sweeps = 0;
  for (int iter = 1; iter <= a.max_iter; ++iter) {
    double v[2];
    // HAUX = CHICHI LAMBDA + CHIPSI
    product({a.chichi, false, a.lam, false}, nullptr, v);
    v[0] += cp[0];
    v[1] += cp[1];
    put(a.haux, v);
    cl.sync();
    // W = LAMBDA^T HAUX + CHIPSI^T LAMBDA + PSIPSI - 1, and its maximum
    {
      const PnlTerm t2{a.chipsi, true, a.lam, false};
      product({a.lam, true, a.haux, false}, &t2, v);
    }
    double mx = 0.0;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      double w = v[e] + pp[e];
      if (ok[e] && gi == gjb + e) w -= 1.0;
      if (!ok[e]) w = 0.0;
      v[e] = w;
      mx = fmax(mx, fabs(w));
      if (w != w) mx = INFINITY;
    }
    put(a.w, v);
    double digam, unused;
    cmax2(mx, 0.0, par, digam, unused);
    par ^= 1;
    if (digam < a.eps) {
      status = CUW_OK;
      iters = iter;
      break;
    }
    if (!(digam <= 1e200)) {
      status = CUW_ERR_DIVERGED;
      iters = iter;
      break;
    }
    // HAUX = U^T W
    product({a.u, true, a.w, false}, nullptr, v);
    put(a.haux, v);
    cl.sync();
    // GT = HAUX U ; X = GT / (e_i + e_j)
    double gtv[2], xp[2], xq[2];
    product({a.haux, false, a.u, false}, nullptr, gtv);
#pragma unroll
    for (int e = 0; e < 2; ++e) xp[e] = xq[e] = ok[e] ? gtv[e] / den[e] : 0.0;
    put(a.gamn, xp);
    cl.sync();
    double* xcur = a.gamn;
    double* xnext = a.xb;
    bool fp_failed = false;
    if (a.use_e) {
      // Lyapunov fixed point X <- (GT - E X - X E)/(e_i + e_j), Chebyshev
      // accelerated as in lyap_fast
      double prev = INFINITY, rho = rho_known, omega = 1.0;
      const int cheb0 = rho > 0.0 ? 0 : 2;
      for (int it2 = 0; it2 < a.max_inner; ++it2) {
        double ex[2];
        sweep_product(xcur, ex);
        double dx = 0.0, xm = 0.0, xn[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          xn[e] = 0.0;
          if (ok[e]) {
            const double fx = (gtv[e] - ex[e]) / den[e];
            xn[e] = omega * (fx - xq[e]) + xq[e];
            dx = fmax(dx, fabs(xn[e] - xp[e]));
            xm = fmax(xm, fabs(xn[e]));
          }
          xq[e] = xp[e];
          xp[e] = xn[e];
        }
        put(xnext, xn);
        double gdx, gxm;
        cmax2(dx, xm, par, gdx, gxm);
        par ^= 1;
        double* t = xcur;
        xcur = xnext;
        xnext = t;
        ++sweeps;
        const double ratio = gdx / prev;
        if (lyap_stop(gdx, gxm, prev, it2, a.max_inner, a.lyap_tol, fp_failed)) break;
        if (it2 == cheb0) {
          if (cheb0 == 2) rho_known = rho = fmin(0.9, fmax(0.05, 1.1 * ratio));
          omega = 1.0 / (1.0 - 0.5 * rho * rho);
        } else if (it2 > cheb0) {
          omega = 1.0 / (1.0 - 0.25 * rho * rho * omega);
        }
      }
    }
    if (fp_failed) {
      status = kFixedPointFailed;
      iters = iter;
      break;
    }
    // HAUX = U X
    product({a.u, false, xcur, false}, nullptr, v);
    put(a.haux, v);
    cl.sync();
    // LAMBDA -= HAUX U^T (equal occupations)
    product({a.haux, false, a.u, true}, nullptr, v);
#pragma unroll
    for (int e = 0; e < 2; ++e) lamv[e] -= v[e];
    put(a.lam, lamv);
    cl.sync();
  }
  if (rank == 0 && tid == 0) {
    a.status[0] = status;
    a.status[1] = iters;
    a.inner[0] += sweeps;
  }
  // no CTA leaves while another may still read its shared-memory slots
  cl.sync();
}

// C = op(A) op(B) for n x n matrices, one 32x32 tile per CTA
__global__ void __launch_bounds__(256) k_small_gemm(const double* A, int tA, const double* B, int tB, int n, double* C,
                                                    const int* gate) {
  __shared__ double smA[tile_lda<2, 2>() * 32], smB[tile_ldb<2, 2>() * 32];
  if (gate_closed(gate)) return;
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  gemm_tile<2, 2, 32>(A, tA != 0, B, tB != 0, n, i0, min(n, i0 + 32), j0, min(n, j0 + 32), C, smA, smB);
}

// LAMBDA1/LAMBDA2 (NBH x NBH complex) from real LAMBDA (NB x NB)
__global__ void k_lambda12(const double* __restrict__ lam, int nb, int nbh, double2* __restrict__ l1,
                           double2* __restrict__ l2) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nbh * nbh) return;
  int ibh1 = idx % nbh, ibh2 = idx / nbh;
  int a = 2 * ibh1, b = 2 * ibh1 + 1, c = 2 * ibh2, d = 2 * ibh2 + 1;
  // CSVAR1 = L(a,c) + i L(a,d); CSVAR2 = i L(b,c) - L(b,d)
  double2 s1 = make_double2(lam[a + (size_t)nb * c], lam[a + (size_t)nb * d]);
  double2 s2 = make_double2(-lam[b + (size_t)nb * d], lam[b + (size_t)nb * c]);
  l1[idx] = make_double2(0.5 * (s1.x - s2.x), 0.5 * (s1.y - s2.y));
  l2[idx] = make_double2(0.5 * (s1.x + s2.x), 0.5 * (s1.y + s2.y));
}

// X (real NB x NB) -> X1, X2 of WAVES_GRAMSCHMIDT (src/paw_waves2.f90:2109-2128)
__global__ void k_fold_x(const double* __restrict__ x, int nb, int nbh, double2* __restrict__ x1,
                         double2* __restrict__ x2) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nbh * nbh) return;
  int ibh1 = idx % nbh, ibh2 = idx / nbh;
  int a = 2 * ibh1, b = 2 * ibh1 + 1, c = 2 * ibh2, d = 2 * ibh2 + 1;
  // CSVAR1 = X11 + i X12 ; CSVAR2 = -i X21 + X22
  double2 s1 = make_double2(x[a + (size_t)nb * c], x[a + (size_t)nb * d]);
  double2 s2 = make_double2(x[b + (size_t)nb * d], -x[b + (size_t)nb * c]);
  x1[idx] = make_double2(0.5 * (s1.x + s2.x), 0.5 * (s1.y + s2.y));
  x2[idx] = make_double2(0.5 * (s1.x - s2.x), 0.5 * (s1.y - s2.y));
}

// real LAMBDA -> RLAM0 (complex), and the extrapolation of WAVES$SWITCH
__global__ void k_store_lambda(const double* __restrict__ lam, int n, double2* __restrict__ rlam0) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < n * n) rlam0[idx] = make_double2(lam[idx], 0.0);
}

__global__ void k_switch_lambda(double2* __restrict__ rlam0, double2* __restrict__ rlamm, int n, int have_m) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * n) return;
  double2 l0 = rlam0[idx];
  if (!have_m) {
    rlamm[idx] = l0;  // NLAMBDA=1: RLAMP = RLAM0, RLAMM = RLAM0
  } else {
    double2 lm = rlamm[idx];
    rlam0[idx] = make_double2(2.0 * l0.x - lm.x, 2.0 * l0.y - lm.y);
    rlamm[idx] = l0;
  }
}

// ---------------------------------------------------------------------------
// WAVES_ORTHO_Y_C (src/paw_waves2.f90:1025-1338) for real (Gamma-point)
// PHIPHI, CHIPHI, CHICHI and the state order MAP (identity when map is null),
// as one cluster of kOyCS CTAs (one CTA for NB <= kOySmall, where a cluster
// barrier costs more than a step's updates).  WAVES_GRAMSCHMIDT (:2025-2177)
// passes one matrix S as all three; WAVES$ORTHOGONALIZE with SAFEORTHO = F
// (:361-386) passes MAT, OMAT and OOMAT.  A, B, C, ALPHA and X are n x n in global
// memory (L2).  pos[i] is the place of state i in MAP: "J > N in the order"
// of the reference is pos[j] > nu.  Step nu (pivot N = MAP(nu)) of the
// sequential orthogonalisation has three parts, each ended by a cluster
// barrier:
//   1. CTA 0 forms the step's scalar and the column/row updates of X, A and B
//      along index N (vectors of n, block barriers only);
//   2. every CTA copies what the rank-one updates read into its shared memory
//      (row N of B, columns N of ALPHA and C, row N of C) and forms the two
//      coefficient vectors z1 (from column N of A) and z2 (from column N of
//      B, which part 3 does not change);
//   3. every CTA updates its share of the n x n elements of A, X, B, ALPHA
//      and C from those copies.  The two B updates of an element are applied
//      in the reference's order, the second with row N of B as the first left
//      it; the C update reads the copied row and column instead of a work array.
// The arithmetic of each element is that of the one-CTA form.
// ---------------------------------------------------------------------------
constexpr int kOyCS = 8, kOySmall = 64;
// ostatus[0] of a state order that failed its check (mapped by ortho_result)
constexpr int kStatusOrder = 100;
__global__ void __launch_bounds__(1024) k_ortho_y(const double* __restrict__ s1, const double* __restrict__ s2,
                                                  const double* __restrict__ s3, const int* __restrict__ map,
                                                  int n, double* A, double* B, double* C, double* AL, double* X,
                                                  int* __restrict__ status) {
  extern __shared__ double oysm[];
  double* z1 = oysm;        // coefficients of the phi step
  double* z2 = z1 + n;      // coefficients of the chi step
  double* brow = z2 + n;    // B(nu, j) before part 3
  double* brow2 = brow + n; // B(nu, j) after the first B update
  double* alcol = brow2 + n;  // ALPHA(i, nu)
  double* ccol = alcol + n;   // C(i, nu)
  double* crow = ccol + n;    // C(nu, j)
  int* pos = reinterpret_cast<int*>(crow + n);  // place of each state in MAP
  __shared__ double zn;
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const int tid = threadIdx.x, nt = blockDim.x;
  const size_t gt = (size_t)rank * nt + tid, gstride = (size_t)cl.num_blocks() * nt;
  const double r8small = 1e-10;
  const size_t nn = (size_t)n * n;
  for (size_t k = gt; k < nn; k += gstride) {
    int i = (int)(k % n), j = (int)(k / n);
    A[k] = s1[k] - (i == j ? 1.0 : 0.0);
    B[k] = s2[k];
    C[k] = s3[k];
    X[k] = 0.0;
    AL[k] = (i == j) ? 1.0 : 0.0;
  }
  for (int k = tid; k < n; k += nt) pos[map ? map[k] : k] = k;
  cl.sync();
  auto I = [n](int i, int j) { return (size_t)i + (size_t)n * j; };
  for (int nu = 0; nu < n; ++nu) {
    const int nn0 = map ? map[nu] : nu;
    // ---- part 1: CTA 0
    if (rank == 0) {
      if (tid == 0) {
        double bnn = B[I(nn0, nn0)], ann = A[I(nn0, nn0)], cnn = C[I(nn0, nn0)];
        double svar = bnn * bnn - ann * cnn;
        double svar1 = -bnn, zz;
        if (svar >= 0.0) {
          double svar2 = sqrt(svar);
          zz = (svar1 * svar2 >= 0.0) ? svar1 - svar2 : svar1 + svar2;
        } else {
          zz = svar1;
        }
        zz = zz / (cnn + r8small);
        if (svar != svar) status[0] = CUW_ERR_NAN;
        zn = zz;
      }
      __syncthreads();
      const double zz = zn;
      for (int i = tid; i < n; i += nt) X[I(i, nn0)] += AL[I(i, nn0)] * zz;
      for (int j = tid; j < n; j += nt) A[I(nn0, j)] += zz * B[I(nn0, j)];
      __syncthreads();
      for (int i = tid; i < n; i += nt) A[I(i, nn0)] += B[I(nn0, i)] * zz;
      __syncthreads();
      if (tid == 0) A[I(nn0, nn0)] += zz * C[I(nn0, nn0)] * zz;
      __syncthreads();
      for (int i = tid; i < n; i += nt) B[I(i, nn0)] += C[I(i, nn0)] * zz;
    }
    cl.sync();
    // ---- part 2: every CTA
    const double bnn = B[I(nn0, nn0)] + r8small;
    const double cnn = C[I(nn0, nn0)];
    for (int i = tid; i < n; i += nt) {
      z1[i] = (pos[i] > nu) ? -(A[I(i, nn0)] / bnn) : 0.0;
      z2[i] = (pos[i] > nu) ? -(B[I(i, nn0)] / bnn) : 0.0;
      brow[i] = B[I(nn0, i)];
      alcol[i] = AL[I(i, nn0)];
      ccol[i] = C[I(i, nn0)];
      crow[i] = C[I(nn0, i)];
    }
    __syncthreads();
    for (int j = tid; j < n; j += nt) brow2[j] = (pos[j] > nu) ? brow[j] + ccol[nn0] * z1[j] : brow[j];
    // every CTA has read the columns and rows before any CTA changes them
    cl.sync();
    // ---- part 3: the CTA's share of the n x n elements
    for (size_t k = gt; k < nn; k += gstride) {
      const int i = (int)(k % n), j = (int)(k / n);
      const bool hi = pos[i] > nu, hj = pos[j] > nu;
      // orthogonalise higher phis to this phi
      if (hj) X[k] += alcol[i] * z1[j];
      double add = 0.0;
      if (hi) add += z1[i] * brow[j];
      if (hj) add += brow[i] * z1[j];
      if (hi && hj) add += z1[i] * cnn * z1[j];
      A[k] += add;
      double b = B[k];
      if (hj) b += ccol[i] * z1[j];
      // orthogonalise higher chis to this phi
      if (hj) AL[k] += alcol[i] * z2[j];
      if (hi) b += z2[i] * brow2[j];
      B[k] = b;
      double wv = 0.0;
      if (hi) wv += z2[i] * crow[j];
      if (hj) wv += ccol[i] * z2[j];
      if (hi && hj) wv += z2[i] * cnn * z2[j];
      C[k] += wv;
    }
    cl.sync();
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// host orchestration
// ---------------------------------------------------------------------------

int unravel_run(Handle* h, const double2* pw, const double2* oc, int npair, double* o0, double* o1, double* o2) {
  const int nbh = h->d.nbh;
  dim3 grid(ceil_div(nbh * nbh, 256), npair);
  k_unravel<<<grid, 256, 0, h->stream>>>(pw, oc, npair, nbh, o0, o1, o2);
  CUW_LAUNCH_CHECK("k_unravel");
  return CUW_OK;
}

int lambda12_run(Handle* h, const double* lam_real, double2* l1, double2* l2) {
  const int nbh = h->d.nbh;
  k_lambda12<<<ceil_div(nbh * nbh, 256), 256, 0, h->stream>>>(lam_real, h->d.nb, nbh, l1, l2);
  CUW_LAUNCH_CHECK("k_lambda12");
  return CUW_OK;
}

int jacobi_run(Handle* h, const double* s_dev, double* u, double* e, const int* gate) {
  const int n = h->d.nb;
  const size_t packed = (size_t)n * (n + 1) / 2;
  const size_t tab = sizeof(int) * (size_t)(n / 2) * (n / 2 + 1) / 2;
  const size_t base = sizeof(double) * (packed + n) + sizeof(int) * (n + 2) + 16 + tab;
  size_t smem = base + sizeof(double) * (size_t)n * n;
  int v_in_smem = 1;
  double* aglob = nullptr;
  if (smem > 220 * 1024) {
    v_in_smem = 0;
    smem = base;
  }
  if (smem > 220 * 1024) {
    // the packed matrix goes to global memory too, and the rounds are shared
    // by a cluster of CTAs
    smem = base - sizeof(double) * packed;
    if (smem > 220 * 1024) return h->fail(CUW_ERR_UNSUPPORTED, "NB too large for the eigensolver");
    if (!h->g.jac_a) CUW_TRY(cudaMalloc(&h->g.jac_a, sizeof(double) * packed));
    aglob = h->g.jac_a;
    const size_t smem_cl = sizeof(double) * n + sizeof(int) * (n + 2) + tab;
    CUW_TRY(smem_allow((const void*)k_jacobi_cl, (int)smem_cl));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kJacCS);
    cfg.blockDim = dim3(1024);
    cfg.dynamicSmemBytes = smem_cl;
    cfg.stream = h->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kJacCS;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CUW_TRY(cudaLaunchKernelEx(&cfg, k_jacobi_cl, s_dev, n, u, e, h->g.work, aglob, 40, h->g.ostatus, gate));
    CUW_LAUNCH_CHECK("k_jacobi_cl");
    return CUW_OK;
  }
  CUW_TRY(smem_allow((const void*)k_jacobi, (int)smem));
  k_jacobi<<<1, 1024, smem, h->stream>>>(s_dev, n, u, e, h->g.work, v_in_smem, aglob, 40, h->g.ostatus, gate);
  CUW_LAUNCH_CHECK("k_jacobi");
  return CUW_OK;
}

// diag(B) -> e, B with its diagonal removed -> E
__global__ void k_split_diag(const double* __restrict__ b, int n, double* __restrict__ e, double* __restrict__ emat,
                             const int* gate) {
  if (gate_closed(gate)) return;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n * n; k += gridDim.x * blockDim.x) {
    const int i = k % n, j = k / n;
    const double v = b[k];
    if (i == j) e[i] = v;
    emat[k] = (i == j) ? 0.0 : v;
  }
}

// dst1 = src1 and dst2 = src2 (n elements each) unless the gate is closed
__global__ void k_copy_gated(const double* __restrict__ src1, double* __restrict__ dst1,
                             const double* __restrict__ src2, double* __restrict__ dst2, int n, const int* gate) {
  if (gate_closed(gate)) return;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    dst1[k] = src1[k];
    dst2[k] = src2[k];
  }
}

// One launch of the ORTHO_X iteration (k_ortho_x) with the eigenbasis in
// g.u / g.eig; use_e: g.u diagonalises an earlier CHIPSI only and g.emat holds
// the off-diagonal rest.  Status and iteration count go to g.ostatus[0..1];
// gate: launch gated on the status of an earlier launch (gate_closed).
static int ortho_x_launch(Handle* h, int use_e, int max_iter, double eps, const int* gate) {
  const int n = h->d.nb;
  Device& g = h->g;
  OrthoArgs a;
  a.n = n;
  a.chichi = g.oomat;
  a.psipsi = g.mat;
  a.chipsi = g.omat;
  a.u = g.u;
  a.e = g.eig;
  a.occ = g.occ;
  a.lam = g.lam;
  a.lam2 = g.lam2;
  a.haux = g.haux;
  a.gamn = g.gamn;
  a.w = g.work;
  a.maxpart = g.maxpart;
  a.status = g.ostatus;
  a.max_iter = max_iter;
  a.eps = eps;
  a.emat = g.emat;
  a.use_e = use_e;
  a.max_inner = h->lyap_max_sweeps;
  a.gt = g.gt;
  a.xb = g.xb;
  a.tb = g.tb;
  a.inner = g.ostatus + 8;
  a.lyap_tol = h->lyap_tol;
  a.gate = gate;
  a.occ_equal = 1;
  for (int i = 1; i < n; ++i)
    if (h->occ_h[i] != h->occ_h[0]) a.occ_equal = 0;
  // cluster of 16 CTAs (non-portable size), else 8, 4, ... ; tile rows/cols
  // per CTA are at most 16*MR x 16*MC with MR, MC in {1,2,4}
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  cfg.blockDim = dim3(512);  // 16 warps: one 8x8 block of a 32x32 tile each
  cfg.stream = h->stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  // 64 < NB <= 128 with equal occupations: the panel-staged cluster kernel
  // (k_ortho_x_pnl)
  if (a.occ_equal && n > 64 && n <= 128 && h->ortho_panel) {
    bool ok = true;
    if (!h->capturing && cudaFuncSetAttribute(k_ortho_x_pnl, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                             cudaSuccess) {
      cudaGetLastError();
      ok = false;
    }
    if (ok && smem_allow((const void*)k_ortho_x_pnl, (int)pnl::kSmemBytes) != cudaSuccess) {
      cudaGetLastError();
      ok = false;
    }
    if (ok) {
      cfg.gridDim = dim3(16);
      cfg.dynamicSmemBytes = pnl::kSmemBytes;
      attr[0].val.clusterDim.x = 16;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cudaError_t e = cudaLaunchKernelEx(&cfg, k_ortho_x_pnl, a);
      if (e == cudaSuccess) {
        ++h->launches;
        return CUW_OK;
      }
      cudaGetLastError();
    }
  }
  // NB <= 32: one CTA holds every tile (products of at most 32^3 take it well
  // under a microsecond, less than one cluster barrier), which also leaves the
  // other SMs to the other sets of a batch; larger NB start from 16 CTAs
  int cs = n <= 32 ? 1 : 16;
  cudaError_t e = cudaSuccess;
  bool launched = false;
  for (; cs >= 1 && !launched; cs /= 2) {
    int tr = 1;
    while (tr * tr < cs) tr *= 2;
    int tc = cs / tr;
    if (tr * tc != cs) { tr = cs; tc = 1; }
    const int rs = (n + tr - 1) / tr, csz = (n + tc - 1) / tc;
    const int mr = rs <= 16 ? 1 : (rs <= 32 ? 2 : (rs <= 64 ? 4 : 0));
    const int mc = csz <= 16 ? 1 : (csz <= 32 ? 2 : (csz <= 64 ? 4 : 0));
    if (!mr || !mc) continue;
    a.kc = 128;  // staging chunk of gemm_tile (its default KC)
    a.fast = (n <= 128 && mr <= 2 && mc <= 2) ? 1 : 0;
    const size_t smem = sizeof(double) * (16 * (mr + mc) + 8) * (size_t)std::max(a.kc, a.fast ? 2 * 128 : 0);
    void (*fn)(OrthoArgs) = nullptr;
    if (mr == 1 && mc == 1) fn = k_ortho_x<1, 1>;
    else if (mr == 2 && mc == 2) fn = k_ortho_x<2, 2>;
    else if (mr == 2 && mc == 4) fn = k_ortho_x<2, 4>;
    else if (mr == 4 && mc == 2) fn = k_ortho_x<4, 2>;
    else if (mr == 4 && mc == 4) fn = k_ortho_x<4, 4>;
    else if (mr == 1 && mc == 2) fn = k_ortho_x<1, 2>;
    else if (mr == 2 && mc == 1) fn = k_ortho_x<2, 1>;
    else if (mr == 4 && mc == 1) fn = k_ortho_x<4, 1>;
    else if (mr == 1 && mc == 4) fn = k_ortho_x<1, 4>;
    if (!fn) continue;
    // (set once per kernel, outside any graph capture: a captured step follows
    // an uncaptured one)
    if (cs > 8 && !h->capturing &&
        cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    if (smem_allow((const void*)fn, (int)smem) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    cfg.gridDim = dim3(cs);
    cfg.dynamicSmemBytes = smem;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    e = cudaLaunchKernelEx(&cfg, fn, a);
    if (e == cudaSuccess) launched = true;
    else cudaGetLastError();
  }
  if (!launched) {
    if (e != cudaSuccess && e != cudaErrorInvalidValue && e != cudaErrorInvalidConfiguration &&
        e != cudaErrorInvalidClusterSize && e != cudaErrorLaunchOutOfResources)
      return h->fail(CUW_ERR_CUDA, std::string("k_ortho_x: ") + cudaGetErrorString(e));
    return h->fail(CUW_ERR_UNSUPPORTED, "k_ortho_x: no cluster configuration fits NB");
  }
  ++h->launches;
  return CUW_OK;
}

// B = U^T S U -> g.work, its diagonal -> g.eig and off-diagonal rest -> g.emat
static int rotate_to_basis(Handle* h, const int* gate) {
  const int n = h->d.nb;
  Device& g = h->g;
  const dim3 tg(ceil_div(n, 32), ceil_div(n, 32));
  k_small_gemm<<<tg, 256, 0, h->stream>>>(g.smat, 0, g.u, 0, n, g.haux, gate);
  CUW_LAUNCH_CHECK("k_small_gemm");
  k_small_gemm<<<tg, 256, 0, h->stream>>>(g.u, 1, g.haux, 0, n, g.work, gate);
  CUW_LAUNCH_CHECK("k_small_gemm");
  k_split_diag<<<ceil_div(n * n, 256), 256, 0, h->stream>>>(g.work, n, g.eig, g.emat, gate);
  CUW_LAUNCH_CHECK("k_split_diag");
  return CUW_OK;
}

// WAVES_ORTHO_X with S = sym(CHIPSI).  The reference diagonalises S in every
// call (src/paw_waves2.f90:1905-1915) to solve S X + X S = Gamma.  Here the
// eigenbasis of an earlier call is kept: X is the fixed point of
// X <- (GT - E X - X E) / (e_i + e_j) in that basis (U^T S U = diag(e) + E),
// the same Lyapunov solution to the requested accuracy.  When the fixed point
// contracts too slowly the kernel reports it, and the gated launches after it
// rediagonalise S (Jacobi on U^T S U, U <- U V) and restart the iteration from
// the saved Lambda; they do nothing otherwise.  Only enqueues: ortho_result
// reads the outcome.
int ortho_solve(Handle* h, int max_iter, double eps) {
  const int n = h->d.nb;
  Device& g = h->g;
  const int nn = n * n;
  const dim3 tg(ceil_div(n, 32), ceil_div(n, 32));
  // with an eigenbasis, Lambda is saved to lam0 in the same launch
  k_symmetrize<<<ceil_div(n * n, 256), 256, 0, h->stream>>>(g.omat, n, g.smat, h->have_u ? g.lam : nullptr, g.lam0);
  CUW_LAUNCH_CHECK("k_symmetrize");
  if (h->have_u) {
    const int* gate = g.ostatus;  // status of the first launch
    const int cb = std::min(ceil_div(nn, 256), 2 * h->nsm);
    CUW_RET(rotate_to_basis(h, nullptr));
    CUW_RET(ortho_x_launch(h, 1, max_iter, eps, nullptr));
    CUW_RET(rotate_to_basis(h, gate));  // g.work was overwritten by the iteration
    CUW_RET(jacobi_run(h, g.work, g.wk2, g.eig, gate));
    k_small_gemm<<<tg, 256, 0, h->stream>>>(g.u, 0, g.wk2, 0, n, g.u2, gate);
    CUW_LAUNCH_CHECK("k_small_gemm");
    k_copy_gated<<<cb, 256, 0, h->stream>>>(g.u2, g.u, g.lam0, g.lam, nn, gate);
    CUW_LAUNCH_CHECK("k_copy_gated");
    CUW_RET(ortho_x_launch(h, 0, max_iter, eps, gate));
  } else {
    CUW_RET(jacobi_run(h, g.smat, g.u, g.eig, nullptr));
    h->have_u = true;
    CUW_RET(ortho_x_launch(h, 0, max_iter, eps, nullptr));
  }
  return CUW_OK;
}

// Outcome of the last ortho_solve from its device status st = ostatus[0..1]
// (copied to the host by the caller); the error messages are the reference's
// (src/paw_waves2.f90:1929-1935, 2007-2014).
int ortho_result(Handle* h, const int* st, int* iters) {
  if (iters) *iters = st[1];
  if (st[0] == CUW_ERR_NOT_CONVERGED) return h->fail(st[0], "LOOP FOR ORTHOGONALIZATION IS NOT CONVERGED");
  if (st[0] == CUW_ERR_DIVERGED) return h->fail(st[0], "ITERATION LOOP FOR ORTHOGONALIZATION IS ABOUT TO DIVERGE");
  if (st[0] == CUW_ERR_NAN) return h->fail(st[0], "NAN DETECTED in WAVES_ORTHO_Y_C");
  if (st[0] == kStatusOrder) return h->fail(CUW_ERR_STATE, "STATE ORDERING FAILED");
  if (st[0] != CUW_OK) return h->fail(CUW_ERR_STATE, "orthogonalisation failed");
  return CUW_OK;
}

int lambda_init_run(Handle* h) {
  const int n = h->d.nb;
  k_lambda_init<<<ceil_div(n * n, 256), 256, 0, h->stream>>>(h->g.rlam0, h->g.occ, n, h->g.lam);
  CUW_LAUNCH_CHECK("k_lambda_init");
  return CUW_OK;
}

int store_lambda_run(Handle* h) {
  const int n = h->d.nb;
  k_store_lambda<<<ceil_div(n * n, 256), 256, 0, h->stream>>>(h->g.lam, n, h->g.rlam0);
  CUW_LAUNCH_CHECK("k_store_lambda");
  return CUW_OK;
}

int switch_lambda_run(Handle* h) {
  const int n = h->d.nb;
  k_switch_lambda<<<ceil_div(n * n, 256), 256, 0, h->stream>>>(h->g.rlam0, h->g.rlamm, n, h->have_rlamm ? 1 : 0);
  CUW_LAUNCH_CHECK("k_switch_lambda");
  h->have_rlamm = true;
  return CUW_OK;
}

// WAVES_ORTHO_Y_C of s1 (PHIPHI), s2 (CHIPHI), s3 (CHICHI) in the state order
// map (null: identity) into x; status word ostatus[0] becomes CUW_ERR_NAN on a
// NaN.  clear_status = false keeps a status set earlier in the same solve.
int ortho_y_general(Handle* h, const double* s1, const double* s2, const double* s3, const int* map, double* x,
                    bool clear_status) {
  const int n = h->d.nb;
  if (n > 1024) return h->fail(CUW_ERR_UNSUPPORTED, "WAVES_ORTHO_Y_C supports NB <= 1024");
  Device& g = h->g;
  if (clear_status) CUW_TRY(cudaMemsetAsync(g.ostatus, 0, sizeof(int) * 2, h->stream));
  // A, B, C, ALPHA in NB x NB buffers that ORTHO_X uses only inside its solve
  const int smem = (int)(sizeof(double) * 7 * (size_t)n + sizeof(int) * (size_t)n);
  CUW_TRY(smem_allow((const void*)k_ortho_y, smem));
  cudaLaunchConfig_t cfg = {};
  const int cs = n <= kOySmall ? 1 : kOyCS;
  cfg.gridDim = dim3(cs);
  cfg.blockDim = dim3(1024);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = h->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  CUW_TRY(cudaLaunchKernelEx(&cfg, k_ortho_y, s1, s2, s3, map, n, g.haux, g.gamn, g.work, g.lam2, x, g.ostatus));
  CUW_LAUNCH_CHECK("k_ortho_y");
  return CUW_OK;
}

int ortho_y_run(Handle* h, const double* s, double* x) { return ortho_y_general(h, s, s, s, nullptr, x, true); }

// SMAP of WAVES$ORTHOGONALIZE with SAFEORTHO = F and SWAPSTATES = T
// (src/paw_waves2.f90:306-346): the exchange sort of the states by the real
// diagonal of LAMBDA (that of RLAM0: the hermitisation leaves the diagonal),
// ascending, then the order check ("STATE ORDERING FAILED").  One warp: for
// each place i the inner loop over j > i swaps the running minimum into place
// i; the places where it swaps are those whose value is below every value
// before them (a prefix minimum that keeps the first of equal values), and
// each of them receives the element that held the minimum before it, so a
// chunk of 32 places is done by one warp scan.
static __global__ void k_smap(const double2* __restrict__ rlam0, int n, int* __restrict__ smap,
                              int* __restrict__ status) {
  extern __shared__ double smd[];
  int* s = reinterpret_cast<int*>(smd + n);
  const int lane = threadIdx.x;
  for (int k = lane; k < n; k += 32) {
    smd[k] = rlam0[(size_t)k + (size_t)n * k].x;
    s[k] = k;
  }
  __syncwarp();
  for (int i = 0; i < n; ++i) {
    int cur = s[i];
    double dc = smd[cur];
    for (int j0 = i + 1; j0 < n; j0 += 32) {
      const int j = j0 + lane;
      const bool valid = j < n;
      const int sj = valid ? s[j] : -1;
      const double dj = valid ? smd[sj] : 0.0;
      // inclusive scan over the lanes of (value, element), combine(a, b) =
      // b if b.value < a.value else a (a earlier): the first strict minimum
      double v = dj;
      int e = sj;
      bool has = valid && dj == dj;  // lanes past n and NaN values take no part (never below anything)
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const double vo = __shfl_up_sync(0xffffffffu, v, d);
        const int eo = __shfl_up_sync(0xffffffffu, e, d);
        const bool ho = __shfl_up_sync(0xffffffffu, has, d);
        if (lane >= d && ho) {
          if (!has || !(v < vo)) {
            v = vo;
            e = eo;
          }
          has = true;
        }
      }
      // exclusive value and holder: the running minimum before place j
      double ve = __shfl_up_sync(0xffffffffu, v, 1);
      int ee = __shfl_up_sync(0xffffffffu, e, 1);
      const bool he = __shfl_up_sync(0xffffffffu, has, 1);
      if (lane == 0 || !he || !(ve < dc)) {
        ve = dc;
        ee = cur;
      }
      if (valid && dj < ve) s[j] = ee;
      // running minimum after the chunk (lane 31 holds the chunk's scan)
      const double vl = __shfl_sync(0xffffffffu, v, 31);
      const int el = __shfl_sync(0xffffffffu, e, 31);
      const bool hl = __shfl_sync(0xffffffffu, has, 31);
      if (hl && vl < dc) {
        dc = vl;
        cur = el;
      }
      __syncwarp();
    }
    if (lane == 0) s[i] = cur;
    __syncwarp();
  }
  bool bad = false;
  for (int k = lane; k + 1 < n; k += 32) bad |= smd[s[k]] > smd[s[k + 1]];
  bad = __any_sync(0xffffffffu, bad);
  for (int k = lane; k < n; k += 32) smap[k] = s[k];
  if (lane == 0 && bad) status[0] = kStatusOrder;
}

int smap_run(Handle* h) {
  const int n = h->d.nb;
  Device& g = h->g;
  CUW_TRY(cudaMemsetAsync(g.ostatus, 0, sizeof(int) * 2, h->stream));
  k_smap<<<1, 32, (sizeof(double) + sizeof(int)) * (size_t)n, h->stream>>>(g.rlam0, n, g.smap, g.ostatus);
  CUW_LAUNCH_CHECK("k_smap");
  return CUW_OK;
}

int fold_x_run(Handle* h, const double* x, double2* x1, double2* x2) {
  const int nbh = h->d.nbh;
  k_fold_x<<<ceil_div(nbh * nbh, 256), 256, 0, h->stream>>>(x, h->d.nb, nbh, x1, x2);
  CUW_LAUNCH_CHECK("k_fold_x");
  return CUW_OK;
}

}  // namespace cuw
