// C ABI of the engine (include/cuwaves.h): handle management, data movement
// and the WAVES operations, each a sequence of device kernels on the handle's
// stream.  No operation has a host compute path: results are produced by the
// kernels in fft.cu, gemm.cu and ortho.cu and by the small kernels below.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "cuwaves_internal.cuh"

namespace cuw {

int unravel_run(Handle* h, const double2* pw, const double2* oc, int npair, double* o0, double* o1, double* o2);
int jacobi_run(Handle* h, const double* s_dev, double* u, double* e, const int* gate);
int lambda_init_run(Handle* h);
int store_lambda_run(Handle* h);
int ortho_y_run(Handle* h, const double* s, double* x);
int ortho_y_general(Handle* h, const double* s1, const double* s2, const double* s3, const int* map, double* x,
                    bool clear_status);
int smap_run(Handle* h);
int fold_x_run(Handle* h, const double* x, double2* x1, double2* x2);

namespace {

// ---------------------------------------------------------------------------
// band sums over G (partials per block, deterministic final combination)
// mode 0 (EKIN, src/paw_waves1.f90:2790-2954):
//   q0 = sum g2 |x|^2, q1 = sum g2 Re(conj x(g) conj x(-g)), q2/q3 same with bucket
// mode 1 (WAVEKINETIC, :6713-6847), d = x - y:
//   q0 = sum m |d|^2, q1 = sum m (Re d Re d~ + Im d Im d~), d~ = conj d(-g)
// mode 2 (expectation values, :2094-2123):
//   q0 + i q1 = sum conj(x) y, q2 + i q3 = sum x(g) y(-g)
// ---------------------------------------------------------------------------
constexpr int RB = 256;
constexpr int RG = 2048;  // G values per block at most when blocks are plentiful (sizes g.red)
__device__ void energy_final_block(int mode, const double* __restrict__ part, int nblk, const double* __restrict__ occ,
                                   int nbh, double gweight, double dt2, int tbucket, double* __restrict__ out,
                                   double* __restrict__ scalar, double* sh);
// The last block of a k_band_sums launch to finish (counted on `count`, which
// it resets) forms the scalar results (energy_final_block).
struct BandFinal {
  const double* occ;
  double gweight, dt2;
  int tbucket;
  double* out;
  double* scalar;
  unsigned* count;
};

__global__ void k_band_sums(int mode, const double2* __restrict__ x, const double2* __restrict__ y, int ldg, int ngl,
                            const double* __restrict__ w1, const double* __restrict__ w2,
                            const int* __restrict__ minusg, double* __restrict__ part, int nblk, int rg,
                            BandFinal fin) {
  const int b = blockIdx.y, blk = blockIdx.x;
  const double2* xb = x + (size_t)ldg * b;
  const double2* yb = y ? y + (size_t)ldg * b : nullptr;
  double q[4] = {0.0, 0.0, 0.0, 0.0};
  const int g0 = blk * rg, g1 = min(ngl, g0 + rg);
  for (int g = g0 + threadIdx.x; g < g1; g += RB) {
    int mg = minusg[g];
    if (mode == 0) {
      double2 a = xb[g], c = xb[mg];
      double n2 = a.x * a.x + a.y * a.y;
      double cr = a.x * c.x - a.y * c.y;  // Re(conj(a) conj(c)) = Re(a c)
      q[0] += w1[g] * n2;
      q[1] += w1[g] * cr;
      if (w2) {
        q[2] += w2[g] * n2;
        q[3] += w2[g] * cr;
      }
    } else if (mode == 1) {
      double2 d = csub(xb[g], yb[g]);
      double2 dm = csub(xb[mg], yb[mg]);
      q[0] += w1[g] * (d.x * d.x + d.y * d.y);
      q[1] += w1[g] * (d.x * dm.x - d.y * dm.y);
    } else {
      double2 a = xb[g], hv = yb[g], hm = yb[mg];
      q[0] += a.x * hv.x + a.y * hv.y;
      q[1] += a.x * hv.y - a.y * hv.x;
      q[2] += a.x * hm.x - a.y * hm.y;
      q[3] += a.x * hm.y + a.y * hm.x;
    }
  }
  __shared__ double red[4][RB];
  for (int k = 0; k < 4; ++k) red[k][threadIdx.x] = q[k];
  __syncthreads();
  for (int s = RB / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int k = 0; k < 4; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x < 4) part[((size_t)b * nblk + blk) * 4 + threadIdx.x] = red[threadIdx.x][0];
  if (!fin.count) return;
  __shared__ bool last;
  __threadfence();  // this block's partials before its count
  if (threadIdx.x == 0) last = atomicAdd(fin.count, 1u) == gridDim.x * gridDim.y - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  extern __shared__ double fsh[];
  energy_final_block(mode, part, nblk, fin.occ, gridDim.y, fin.gweight, fin.dt2, fin.tbucket, fin.out, fin.scalar,
                     fsh);
  if (threadIdx.x == 0) *fin.count = 0u;
}

// scalar results from band sums and occupations (the last block of
// k_band_sums): the block sums the block
// partials of every band (the order of the former two-kernel form), forms the
// per-band terms in parallel, and thread 0 adds them in band order
//   out[0] EKIN or WAVEKINETIC energy; out[1 + i] per-band values
//   scalar (when not null) also receives out[0]
// The partials are read through L2: other blocks of the same launch wrote them.
__device__ void energy_final_block(int mode, const double* __restrict__ part, int nblk, const double* __restrict__ occ,
                                   int nbh, double gweight, double dt2, int tbucket, double* __restrict__ out,
                                   double* __restrict__ scalar, double* sh) {
  double* res = sh;            // [4 nbh]
  double* term = sh + 4 * nbh;  // [nbh]
  for (int i = threadIdx.x; i < 4 * nbh; i += blockDim.x) {
    const int b = i / 4, k = i % 4;
    double s = 0.0;
    for (int t = 0; t < nblk; ++t) s += __ldcg(&part[((size_t)b * nblk + t) * 4 + k]);
    res[i] = s;
  }
  __syncthreads();
  for (int b = threadIdx.x; b < nbh; b += blockDim.x) {
    const double f1 = occ[2 * b], f2 = occ[2 * b + 1];
    const double* q = res + 4 * b;
    double e = 0.0;
    if (mode == 0) {
      const double fp = 0.5 * (f1 + f2), fm = 0.5 * (f1 - f2);
      if (!(fp == 0.0 && fm == 0.0)) {
        e = 0.5 * fp * q[0] + (tbucket ? fp * q[2] : 0.0);
        if (fabs(fm) >= 1e-12) e += 0.5 * fm * q[1] + (tbucket ? fm * q[3] : 0.0);
      }
    } else if (mode == 1) {
      double ev1 = 0.0, ev2 = 0.0;
      if (!(f1 == 0.0 && f2 == 0.0)) {
        const double sum = q[0] / dt2;
        ev1 = 0.5 * sum;
        ev2 = 0.5 * sum;
        e = sum * 0.5 * (f1 + f2);
        if (f1 - f2 != 0.0) {
          const double s2 = q[1] / dt2;
          ev1 += 0.5 * s2;
          ev2 -= 0.5 * s2;
          e += s2 * 0.5 * (f1 - f2);
        }
      }
      out[1 + 2 * b] = ev1;
      out[2 + 2 * b] = ev2;
    } else {
      const double tp = q[0] * gweight, tm = q[2] * gweight;
      out[1 + 2 * b] = 0.5 * tp + 0.5 * tm;
      out[2 + 2 * b] = 0.5 * tp - 0.5 * tm;
      e = f1 * out[1 + 2 * b] + f2 * out[2 + 2 * b];
    }
    term[b] = e;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double e = 0.0;
    for (int b = 0; b < nbh; ++b) e += term[b];
    out[0] = (mode == 2) ? e : e * gweight;
    if (scalar) scalar[0] = out[0];
  }
}

// WAVES$PROPAGATE (src/paw_waves1.f90:6575-6583)
__global__ void k_propagate(const double2* __restrict__ psi0, double2* __restrict__ psim,
                            const double2* __restrict__ hpsi, const double* __restrict__ mpsi, int ldg, int ngl,
                            int nbh, double a1, double a2, double a3, const double* __restrict__ fr, double dt2) {
  size_t n = (size_t)ldg * nbh;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int g = (int)(k % ldg);
    if (g >= ngl) continue;
    double b1 = a1, b2 = a2, c = a3 / mpsi[g];
    if (fr) {  // ARR1..ARR3 of ANNEEVEC (src/paw_waves1.f90:6536-6540)
      const double an = 1.0 + fr[g];
      b1 = 2.0 / an;
      b2 = 1.0 - b1;
      c = -dt2 / an / mpsi[g];
    }
    double2 p0 = psi0[k], pm = psim[k], hv = hpsi[k];
    psim[k] = make_double2(b1 * p0.x + b2 * pm.x + c * hv.x, b1 * p0.y + b2 * pm.y + c * hv.y);
  }
}

// ANNEEVEC(G) of WAVES_DMPSI with TSTRESS (src/paw_waves1.f90:6694-6709);
// f = FRICMAT(3,3) in Fortran order
struct Fric {
  double f[9];
};
__global__ void k_anneevec(const double* __restrict__ gx, const double* __restrict__ gy,
                           const double* __restrict__ gz, const double* __restrict__ dbucket, int ngl, Fric fm,
                           double fac1, double fac2, double* __restrict__ anv) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngl) return;
  const double* F = fm.f;
  const double x = gx[g], y = gy[g], z = gz[g];
  const double svar = F[0] * x * x + F[3] * 2.0 * x * y + F[6] * 2.0 * x * z + F[4] * y * y + F[7] * 2.0 * y * z +
                      F[8] * z * z;
  anv[g] = fac1 + fac2 * svar * (1.0 + (dbucket ? dbucket[g] : 0.0));
}

// DEDPROJ = F1 HPROJ + F2 conj(HPROJ) per super wave function (src/paw_waves1.f90:5644-5668)
__global__ void k_dedproj(double2* __restrict__ hp, const double* __restrict__ occ, int nbh, int npro) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= (size_t)nbh * npro) return;
  int b = (int)(i % nbh);
  double f1 = 0.5 * (occ[2 * b] + occ[2 * b + 1]), f2 = 0.5 * (occ[2 * b] - occ[2 * b + 1]);
  double2 c = hp[i];
  hp[i] = make_double2(f1 * c.x + f2 * c.x, f1 * c.y - f2 * c.y);
}

// lambda(i,j) = -Re RLAM0(i,j) * 0.5 (f_i + f_j)   (src/paw_waves1.f90:5673-5680)
__global__ void k_force_lambda(const double2* __restrict__ rlam0, const double* __restrict__ occ, int nb,
                               double* __restrict__ lam) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nb * nb) return;
  int i = idx % nb, j = idx / nb;
  lam[idx] = -rlam0[idx].x * 0.5 * (occ[i] + occ[j]);
}

// R(+) = 2R(0) - R(-) + dt^2 F/M  (ATOMS$PROPAGATE without friction)
__global__ void k_atoms_verlet(const double* __restrict__ r0, const double* __restrict__ rm, double* __restrict__ rp,
                               const double* __restrict__ f, const double* __restrict__ mass, int nat, double dt2) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * nat) return;
  rp[i] = 2.0 * r0[i] - rm[i] + dt2 * f[i] / mass[i / 3];
}

// Ionic kinetic energy from R(+) and R(-), then ATOMS$SWITCH by copies:
// R(-) <- R(0), R(0) <- R(+) (one block; each thread rewrites only the
// coordinates it has read)
__global__ void k_ion_ekin_switch(const double* __restrict__ rp, double* __restrict__ rm, double* __restrict__ r0,
                                  const double* __restrict__ mass, int nat, double dt, double* __restrict__ out) {
  extern __shared__ double term[];  // [3 nat]; summed by thread 0 in index order
  for (int i = threadIdx.x; i < 3 * nat; i += blockDim.x) {
    const double v = (rp[i] - rm[i]) / (2.0 * dt);
    term[i] = 0.5 * mass[i / 3] * v * v;
    rm[i] = r0[i];
    r0[i] = rp[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double e = 0.0;
    for (int i = 0; i < 3 * nat; ++i) e += term[i];
    out[0] = e;
  }
}

// a set's step results into the batch's result slots: the 8 sums and the two
// status words
__global__ void k_batch_out(const double* __restrict__ scal, const int* __restrict__ status, double* __restrict__ res,
                            int* __restrict__ st) {
  const int t = threadIdx.x;
  if (t < 8) res[t] = scal[t];
  if (t < 2) st[t] = status[t];
}

__global__ void k_add_vec(double* __restrict__ a, const double* __restrict__ b, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] += b[i];
}

__global__ void k_copy_psi(const double2* __restrict__ src, double2* __restrict__ dst, size_t n) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    dst[k] = src[k];
}

}  // namespace

// ---------------------------------------------------------------------------
// band reductions: results in h->g.scal (device): [0] energy, [1..nb] per band
// ---------------------------------------------------------------------------
// the band sums of mode over G, then (by the launch's last block) the scalar
// results: out_dev[0] the energy, out_dev[1..] per band, scalar[0] (when not
// null) the energy again
static int band_sums_run(Handle* h, int mode, const double2* x, const double2* y, const double* w1, const double* w2,
                         double* out_dev, double* scalar) {
  const int nmax = ceil_div(h->d.ngl, RG);  // partial slots per band in g.red
  const size_t sm = sizeof(double) * 5 * (size_t)h->d.nbh;
  if (sm > 48 * 1024) CUW_TRY(smem_allow((const void*)k_band_sums, (int)sm));
  if (h->band_bps == 0) {
    int bps = 0;
    CUW_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_band_sums, RB, sm));
    h->band_bps = std::max(1, bps);
  }
  // one wave of blocks on the SMs the set may use (a second, nearly empty
  // wave would double the time): G ranges of a multiple of RB per block
  int nblk = std::min(nmax, std::max(1, h->nsm * h->band_bps / h->d.nbh));
  const int rg = ceil_div(ceil_div(h->d.ngl, nblk), RB) * RB;
  nblk = ceil_div(h->d.ngl, rg);
  Device& g = h->g;
  BandFinal fin{g.occ, h->gweight, h->delt * h->delt, h->tbucket ? 1 : 0, out_dev, scalar,
                reinterpret_cast<unsigned*>(g.red + 4 * (size_t)h->d.nbh * (nmax + 1))};
  k_band_sums<<<dim3(nblk, h->d.nbh), RB, sm, h->stream>>>(mode, x, y, h->ldg, h->d.ngl, w1, w2, g.minusg, g.red,
                                                           nblk, rg, fin);
  CUW_LAUNCH_CHECK("k_band_sums");
  return CUW_OK;
}

// mode: RED_EKIN / RED_WAVEKIN / RED_EXPECT; result vector at out_dev, the
// energy also at scalar (when not null)
static int energy_run(Handle* h, int mode, double* out_dev, double* scalar = nullptr) {
  Device& g = h->g;
  if (mode == RED_EKIN)
    return band_sums_run(h, 0, g.psi0, nullptr, g.g2, h->tbucket ? g.bucket : nullptr, out_dev, scalar);
  if (mode == RED_WAVEKIN) return band_sums_run(h, 1, g.psi0, g.psim, g.mpsi, nullptr, out_dev, scalar);
  return band_sums_run(h, 2, g.psi0, g.hpsi, nullptr, nullptr, out_dev, scalar);
}

cudaError_t smem_allow(const void* fn, int bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, int> limit;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  int& cur = limit[std::make_pair(dev, fn)];
  if (bytes <= cur) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) cur = bytes;
  return e;
}

int band_reduce(Handle* h, int what, double* out_host, double* eig_host) {
  double* out_dev = h->g.scal;
  CUW_RET(energy_run(h, what, out_dev));
  std::vector<double> tmp(1 + h->d.nb);
  CUW_TRY(cudaMemcpyAsync(tmp.data(), out_dev, sizeof(double) * (1 + h->d.nb), cudaMemcpyDeviceToHost, h->stream));
  CUW_TRY(cudaStreamSynchronize(h->stream));
  if (out_host) *out_host = tmp[0];
  if (eig_host) std::memcpy(eig_host, tmp.data() + 1, sizeof(double) * h->d.nb);
  return CUW_OK;
}

// ANNEEVEC of the cell friction for the present ANNEE and G set
static int friction_update(Handle* h) {
  if (!h->fric_on || !h->have_gset) return CUW_OK;
  const double* F = h->fricmat;
  const double fac1 = h->annee - 0.5 * (F[0] + F[4] + F[8]);
  const double fac2 = -0.5 * h->emass * 2.0 * h->emasscg2;
  Fric fm;
  std::memcpy(fm.f, F, sizeof(fm.f));
  k_anneevec<<<ceil_div(h->d.ngl, 256), 256, 0, h->stream>>>(h->g.gx, h->g.gy, h->g.gz,
                                                             h->have_dbucket ? h->g.dbucket : nullptr, h->d.ngl,
                                                             fm, fac1, fac2, h->g.anv);
  CUW_LAUNCH_CHECK("k_anneevec");
  return CUW_OK;
}

int propagate_run(Handle* h) {
  const double a1 = 2.0 / (1.0 + h->annee), a2 = 1.0 - a1, a3 = -h->delt * h->delt / (1.0 + h->annee);
  k_propagate<<<4 * h->nsm, 256, 0, h->stream>>>(h->g.psi0, h->g.psim, h->g.hpsi, h->g.mpsi, h->ldg, h->d.ngl,
                                                 h->d.nbh, a1, a2, a3, h->fric_on ? h->g.anv : nullptr,
                                                 h->delt * h->delt);
  CUW_LAUNCH_CHECK("k_propagate");
  return CUW_OK;
}

// DEDPROJ in h->g.hproj, then forces into force_dev (uses eigr of R(0))
static int force_dev_run(Handle* h, double* force_dev) {
  Device& g = h->g;
  const int nbh = h->d.nbh, npro = h->npro, nb = h->d.nb;
  CUW_RET(hoproj_compute(h, g.proj, g.hproj, g.oproj));
  size_t n = (size_t)nbh * npro;
  k_dedproj<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(g.hproj, g.occ, nbh, npro);
  CUW_LAUNCH_CHECK("k_dedproj");
  k_force_lambda<<<ceil_div(nb * nb, 256), 256, 0, h->stream>>>(g.rlam0, g.occ, nb, g.wk2);
  CUW_LAUNCH_CHECK("k_force_lambda");
  CUW_RET(lambda12_run(h, g.wk2, g.lam1c, g.lam2c));
  CUW_RET(addoproj_run(h, g.hproj, g.oproj, g.lam1c, g.lam2c));
  CUW_RET(force_gemm(h, g.hproj, force_dev));
  return CUW_OK;
}

// the part of WAVES$ORTHOGONALIZE after OPSI is formed (src/paw_waves2.f90:242-490)
static int mark(Handle* h, int phase);
// (enqueues only: the solve's status is read with the step's results)
static int ortho_core(Handle* h, int max_iter, double eps) {
  Device& g = h->g;
  // projections of PSIBAR and OPSI at R(+)
  CUW_RET(mark(h, 1));
  CUW_RET(eigr_compute(h, g.rp));
  CUW_RET(mark(h, 5));
  // PSIBAR and OPSI stay fixed through the Gram products: their split forms
  // are reused (the guard closes the scope on every way out)
  struct ScopeGuard {
    Handle* h;
    ~ScopeGuard() {
      if (h) tc_scope(h, false);
    }
  } guard{h->mixed() ? h : nullptr};
  if (h->mixed()) tc_scope(h, true);
  CUW_RET(proj_compute(h, g.psim, g.proj, g.opsi, g.oproj));
  CUW_RET(mark(h, 6));
  // DO*PROJ and DO*OPROJ
  CUW_RET(oproj_compute(h, g.proj, g.hproj));
  CUW_RET(oproj_compute(h, g.oproj, g.pbuf));
  const size_t mn = (size_t)h->d.nbh * h->d.nbh;
  double2* pw = g.tmat;
  double2* oc = g.tmat + 6 * mn;
  GramPair pc[3] = {{g.proj, g.hproj}, {g.oproj, g.hproj}, {g.oproj, g.pbuf}};
  CUW_RET(gram_projections(h, pc, 3, oc));
  GramPair pp[3] = {{g.psim, g.psim}, {g.opsi, g.psim}, {g.opsi, g.opsi}};
  CUW_RET(gram_planewave(h, pp, 3, pw));
  if (h->mixed()) tc_scope(h, false);
  guard.h = nullptr;
  CUW_RET(unravel_run(h, pw, oc, 3, g.mat, g.omat, g.oomat));
  CUW_RET(mark(h, 7));
  if (h->safeortho) {
    CUW_RET(lambda_init_run(h));
    CUW_RET(ortho_solve(h, max_iter, eps));
  } else {
    // SAFEORTHO = F (src/paw_waves2.f90:306-346, 384-386): WAVES_ORTHO_Y_C of
    // MAT, OMAT, OOMAT gives LAMBDA directly (its X is INTENT(OUT), so the
    // symmetrised and occupation-scaled RLAM0 of the other branch is unused);
    // the state order SMAP follows the RLAM0 diagonal when SWAPSTATES = T
    if (h->swapstates) CUW_RET(smap_run(h));
    CUW_RET(ortho_y_general(h, g.mat, g.omat, g.oomat, h->swapstates ? g.smap : nullptr, g.lam, !h->swapstates));
  }
  CUW_RET(mark(h, 8));
  CUW_RET(lambda12_run(h, g.lam, g.lam1c, g.lam2c));
  CUW_RET(addopsi_run(h, g.psim, g.opsi, g.lam1c, g.lam2c));
  CUW_RET(addoproj_run(h, g.proj, g.oproj, g.lam1c, g.lam2c));
  CUW_RET(store_lambda_run(h));
  h->have_opsi = false;
  return CUW_OK;
}

// phase marks of cuwaves_cp_step (only when timing is enabled)
enum { PH_RED = 0, PH_EIGR, PH_FORCE, PH_FFT, PH_ADDPRO, PH_PROJ, PH_GRAM, PH_ORTHO, PH_ROTATE, PH_MISC, PH_POT };
static int mark(Handle* h, int phase) {
  if (!h->timing) return CUW_OK;
  if (h->nev >= (int)h->ev.size()) {
    cudaEvent_t e;
    CUW_TRY(cudaEventCreate(&e));
    h->ev.push_back(e);
    h->ev_phase.push_back(0);
  }
  h->ev_phase[h->nev] = phase;  // time from this mark to the next is charged to `phase`
  CUW_TRY(cudaEventRecord(h->ev[h->nev], h->stream));
  ++h->nev;
  return CUW_OK;
}
static int collect_marks(Handle* h) {
  if (!h->timing) return CUW_OK;
  for (int i = 0; i + 1 < h->nev; ++i) {
    float ms = 0.f;
    CUW_TRY(cudaEventElapsedTime(&ms, h->ev[i], h->ev[i + 1]));
    h->phase_ms[h->ev_phase[i]] += ms;
  }
  h->nev = 0;
  h->phase_calls++;
  return CUW_OK;
}

}  // namespace cuw

using namespace cuw;

// ---------------------------------------------------------------------------
// extern "C" entry points
// ---------------------------------------------------------------------------
#define H(hp) Handle* h = reinterpret_cast<Handle*>(hp)
#define CUW_BATCH_TRY(expr)                                                                 \
  do {                                                                                      \
    cudaError_t e__ = (expr);                                                               \
    if (e__ != cudaSuccess) return b->fail(CUW_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e__)); \
  } while (0)
#define NEED(cond, code, msg) \
  do {                        \
    if (!(cond)) return h->fail(code, msg); \
  } while (0)

static int dev_alloc(Handle* h, void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
  if (e != cudaSuccess) return h->fail(CUW_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  e = cudaMemset(*p, 0, std::max<size_t>(bytes, 16));
  if (e != cudaSuccess) return h->fail(CUW_ERR_CUDA, cudaGetErrorString(e));
  return CUW_OK;
}
#define ALLOC(ptr, bytes) CUW_RET(dev_alloc(h, reinterpret_cast<void**>(&(ptr)), (bytes)))

static void free_all(Handle* h) {
  Device& g = h->g;
  void* ptrs[] = {g.rho, g.psi0, g.psim, g.hpsi, g.opsi, g.proj, g.oproj, g.hproj, g.pbuf, g.rlam0, g.rlamm, g.igvec,
                  g.minusg, g.gx, g.gy, g.gz, g.g2, g.pro, g.ylm, g.mpsi, g.bucket, g.pdesc, g.plane_iz, g.plane_rows, g.plane_off,
                  g.plane_g, g.plane_pos, g.zslot, g.v, g.grid, g.tw1, g.tw2, g.tw3, g.r0, g.rp, g.rm, g.force, g.mass,
                  g.eigr, g.dh, g.dover, g.occ, g.mat, g.omat, g.oomat, g.lam, g.lam2, g.lam0, g.u, g.u2, g.eig, g.haux, g.gamn,
                  g.work, g.wk2, g.smat, g.emat, g.gt, g.xb, g.tb, g.maxpart, g.ostatus, g.smap, g.lam1c, g.lam2c, g.part, g.red, g.scal, g.tmat, g.t_ipro0,
                  g.t_nlmn, g.t_isp, g.t_lnofp, g.t_mofp, g.t_lmn0ln, g.t_lox, g.pf, g.xminus[0], g.xminus[1], g.bpre[0],
                  g.bpre[1], g.bsmall, g.jac_a, g.r_plus, g.r_minus, g.r_gx, g.r_gy, g.r_gz, g.r_g2, g.r_ylm,
                  g.r_g0, g.r_v0, g.r_pscore, g.r_vbar, g.r_lmrx, g.qlm, g.r_rhog, g.r_vg, g.r_pot, g.r_vtot,
                  g.r_grid, g.r_part, g.fpot, g.vqlm, g.r_out, g.prox, g.anv, g.dbucket};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  h->g = Device();
}

// message of the calling thread's last failed cuwaves_create (its handle is gone)
static thread_local std::string t_create_err;

extern "C" int cuwaves_create(const cuw_dims* dims, cuw_handle** out) {
  auto bad = [](int code, const char* m) {
    t_create_err = m;
    return code;
  };
  if (!dims || !out) return bad(CUW_ERR_ARG, "null argument");
  *out = nullptr;
  const cuw_dims& d = *dims;
  if (d.ngl <= 0 || d.nb <= 0 || d.nat < 0 || d.nsp <= 0 || d.nsp > CUW_MAXSP || d.nr1 <= 0 || d.nr2 <= 0 ||
      d.nr3 <= 0 || d.lmx <= 0 || (d.nat > 0 && !d.isp))
    return bad(CUW_ERR_ARG, "invalid dimensions");
  if (d.ndim != 1 || !d.tinv || (d.nb % 2) || d.nbh != d.nb / 2)
    return bad(CUW_ERR_UNSUPPORTED, "only scalar Gamma-point super wave functions with an even band count");
  if (d.precision != CUW_PREC_FP64 && d.precision != CUW_PREC_MIXED) return bad(CUW_ERR_ARG, "unknown precision");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return bad(CUW_ERR_CUDA, "no CUDA device");
  }
  Handle* h = new Handle();
  h->d = d;
  h->d.isp = nullptr;
  cudaGetDevice(&h->device);
  cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, h->device);
  h->nsm_dev = h->nsm;
  h->isp.resize(d.nat);
  for (int a = 0; a < d.nat; ++a) {
    h->isp[a] = dims->isp[a] - 1;
    if (h->isp[a] < 0 || h->isp[a] >= d.nsp) {
      delete h;
      return bad(CUW_ERR_ARG, "atom species index out of range");
    }
  }
  h->lmnx.resize(d.nsp);
  h->ibpro.resize(d.nsp);
  int nbare = 0;
  for (int s = 0; s < d.nsp; ++s) {
    if (d.lnx[s] <= 0 || d.lnx[s] > CUW_MAXLN) { delete h; return bad(CUW_ERR_ARG, "projector count out of range"); }
    int n = 0;
    for (int ln = 0; ln < d.lnx[s]; ++ln) {
      int l = d.lox[s][ln];
      if (l < 0 || (l + 1) * (l + 1) > d.lmx) { delete h; return bad(CUW_ERR_ARG, "angular momentum above lmx"); }
      n += 2 * l + 1;
    }
    h->lmnx[s] = n;
    h->lmnxx = std::max(h->lmnxx, n);
    h->lnxx = std::max(h->lnxx, d.lnx[s]);
    h->ibpro[s] = nbare;
    nbare += d.lnx[s];
  }
  h->nbarepro = nbare;
  h->ipro0.resize(d.nat);
  for (int a = 0; a < d.nat; ++a) {
    int s = h->isp[a];
    h->ipro0[a] = h->npro;
    for (int ln = 0; ln < d.lnx[s]; ++ln) {
      int l = d.lox[s][ln];
      for (int m = 0; m < 2 * l + 1; ++m) h->pdesc.push_back(ProDesc{a, h->ibpro[s] + ln, l * l + m, l});
    }
    h->npro += h->lmnx[s];
  }
  h->ldg = ceil_div(d.ngl, 32) * 32;
  h->lyap_tol = d.precision == CUW_PREC_MIXED ? 1e-2 : 1e-5;
  h->nr = (size_t)d.nr1 * d.nr2 * d.nr3;
  h->occ_h.assign(d.nb, 0.0);
  int rc = CUW_OK;
  do {
    if (cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking); e != cudaSuccess) {
      rc = h->fail(CUW_ERR_CUDA, std::string("cudaStreamCreateWithFlags: ") + cudaGetErrorString(e));
      break;
    }
    Device& g = h->g;
    const size_t nps = (size_t)h->ldg * d.nbh * sizeof(double2);
    const size_t npj = (size_t)d.nbh * std::max(1, h->npro) * sizeof(double2);
    const size_t nn = (size_t)d.nb * d.nb;
    const size_t mn = (size_t)d.nbh * d.nbh;
#define TRYA(p, b) \
  if ((rc = dev_alloc(h, reinterpret_cast<void**>(&(p)), (b))) != CUW_OK) break
    TRYA(g.psi0, nps); TRYA(g.psim, nps); TRYA(g.hpsi, nps); TRYA(g.opsi, nps);
    TRYA(g.proj, npj); TRYA(g.oproj, npj); TRYA(g.hproj, npj); TRYA(g.pbuf, npj);
    TRYA(g.rlam0, nn * sizeof(double2)); TRYA(g.rlamm, nn * sizeof(double2));
    TRYA(g.igvec, sizeof(int) * 3 * d.ngl); TRYA(g.minusg, sizeof(int) * d.ngl);
    TRYA(g.gx, sizeof(double) * d.ngl); TRYA(g.gy, sizeof(double) * d.ngl); TRYA(g.gz, sizeof(double) * d.ngl);
    TRYA(g.g2, sizeof(double) * d.ngl); TRYA(g.mpsi, sizeof(double) * d.ngl);
    TRYA(g.pro, sizeof(double) * d.ngl * (size_t)nbare); TRYA(g.ylm, sizeof(double) * d.ngl * (size_t)d.lmx);
    TRYA(g.pdesc, sizeof(ProDesc) * std::max(1, h->npro));
    TRYA(g.v, sizeof(double) * h->nr);
    TRYA(g.r0, sizeof(double) * 3 * std::max(1, d.nat)); TRYA(g.rp, sizeof(double) * 3 * std::max(1, d.nat));
    TRYA(g.rm, sizeof(double) * 3 * std::max(1, d.nat)); TRYA(g.force, sizeof(double) * 3 * std::max(1, d.nat));
    TRYA(g.mass, sizeof(double) * std::max(1, d.nat));
    TRYA(g.eigr, sizeof(double2) * d.ngl * (size_t)std::max(1, d.nat));
    TRYA(g.dh, sizeof(double2) * (size_t)h->lmnxx * h->lmnxx * std::max(1, d.nat));
    TRYA(g.dover, sizeof(double) * (size_t)h->lnxx * h->lnxx * d.nsp);
    TRYA(g.occ, sizeof(double) * d.nb);
    TRYA(g.mat, sizeof(double) * nn); TRYA(g.omat, sizeof(double) * nn); TRYA(g.oomat, sizeof(double) * nn);
    TRYA(g.lam, sizeof(double) * nn); TRYA(g.lam2, sizeof(double) * nn); TRYA(g.lam0, sizeof(double) * nn); TRYA(g.u, sizeof(double) * nn);
    TRYA(g.u2, sizeof(double) * nn);
    TRYA(g.eig, sizeof(double) * d.nb); TRYA(g.haux, sizeof(double) * nn); TRYA(g.gamn, sizeof(double) * nn);
    TRYA(g.work, sizeof(double) * nn); TRYA(g.wk2, sizeof(double) * nn);
    TRYA(g.smat, sizeof(double) * nn); TRYA(g.emat, sizeof(double) * nn); TRYA(g.gt, sizeof(double) * nn);
    TRYA(g.xb, sizeof(double) * nn); TRYA(g.tb, sizeof(double) * nn);
    TRYA(g.maxpart, sizeof(double) * 64); TRYA(g.ostatus, sizeof(int) * 16); TRYA(g.smap, sizeof(int) * d.nb);
    TRYA(g.lam1c, sizeof(double2) * mn); TRYA(g.lam2c, sizeof(double2) * mn);
    TRYA(g.tmat, sizeof(double2) * 12 * mn);
    TRYA(g.red, sizeof(double) * (4 * (size_t)d.nbh * (ceil_div(d.ngl, RG) + 1) + 8));
    TRYA(g.scal, sizeof(double) * (size_t)(2 * d.nb + 16));
#undef TRYA
    if (rc != CUW_OK) break;
    if (cudaError_t e = cudaMemcpy(g.pdesc, h->pdesc.data(), sizeof(ProDesc) * h->npro, cudaMemcpyHostToDevice);
        e != cudaSuccess) {
      rc = h->fail(CUW_ERR_CUDA, std::string("cudaMemcpy of the projector table: ") + cudaGetErrorString(e));
      break;
    }
    rc = small_tables_setup(h);
    if (rc == CUW_OK) rc = gemm_setup(h);
    if (rc == CUW_OK && h->mixed()) rc = tc_setup(h);
  } while (0);
  if (rc != CUW_OK) {
    t_create_err = h->err.empty() ? "handle set-up failed" : h->err;
    free_all(h);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return rc;
  }
  *out = reinterpret_cast<cuw_handle*>(h);
  return CUW_OK;
}

extern "C" int cuwaves_destroy(cuw_handle* hp) {
  if (!hp) return CUW_OK;
  H(hp);
  cudaStreamSynchronize(h->stream);
  for (cudaEvent_t e : h->ev) cudaEventDestroy(e);
  h->drop_graphs();
  free_all(h);
  if (h->res_h) cudaFreeHost(h->res_h);
  cudaStreamDestroy(h->stream);
  delete h;
  return CUW_OK;
}

namespace cuw {
// Returns a handle to the state of a freshly created one for the same G set
// (the serving runtime reuses handles of finished requests): no eigenbasis,
// no Lagrange history, no H|psi> or O|psi>, no EIGR, no step graphs.  Buffers
// keep stale data, which every later call writes before it reads.
int handle_recycle(cuw_handle* hp) {
  Handle* h = reinterpret_cast<Handle*>(hp);
  if (!h) return CUW_ERR_ARG;
  CUW_TRY(cudaStreamSynchronize(h->stream));
  // the Lagrange multipliers start from zero as in a new handle (the first
  // ORTHO_X guess and the first forces read RLAM0)
  const size_t nn = (size_t)h->d.nb * h->d.nb;
  CUW_TRY(cudaMemset(h->g.rlam0, 0, sizeof(double2) * nn));
  CUW_TRY(cudaMemset(h->g.rlamm, 0, sizeof(double2) * nn));
  CUW_TRY(cudaMemset(h->g.lam, 0, sizeof(double) * nn));
  h->have_hpsi = h->have_opsi = h->have_u = h->have_rlamm = false;
  h->eigr_src = nullptr;
  h->timing = false;
  h->nev = 0;
  h->scf = false;
  h->drop_graphs();
  h->touch();
  h->err.clear();
  return CUW_OK;
}
}  // namespace cuw

extern "C" int cuwaves_last_error(const cuw_handle* hp, char* buf, int len) {
  if (!buf || len <= 0) return CUW_ERR_ARG;
  const Handle* h = reinterpret_cast<const Handle*>(hp);
  // without a handle: the calling thread's last failed cuwaves_create
  std::snprintf(buf, (size_t)len, "%s", h ? h->err.c_str() : t_create_err.c_str());
  return CUW_OK;
}

extern "C" int cuwaves_set_async(cuw_handle* hp, int async) {
  H(hp);
  h->async = async != 0;
  return CUW_OK;
}

extern "C" int cuwaves_synchronize(cuw_handle* hp) {
  H(hp);
  CUW_TRY(cudaStreamSynchronize(h->stream));
  return CUW_OK;
}

extern "C" int cuwaves_set_gset(cuw_handle* hp, const int* igvec, const int* minusg, const double* gbas,
                                const double* gvec, const double* g2, const double* pro, const double* ylm,
                                const double* mpsi, const double* bucket, double gweight) {
  H(hp);
  CUW_TRY(h->settle());
  h->touch();
  h->eigr_src = nullptr;
  NEED(igvec && minusg && gbas && gvec && g2 && pro && ylm && mpsi, CUW_ERR_ARG, "null argument");
  NEED(gweight > 0.0, CUW_ERR_ARG, "gweight must be the positive cell volume");
  const int ngl = h->d.ngl;
  Device& g = h->g;
  std::vector<int> mg(ngl);
  for (int i = 0; i < ngl; ++i) {
    mg[i] = minusg[i] - 1;
    NEED(mg[i] >= 0 && mg[i] < ngl, CUW_ERR_ARG, "minusg out of range");
    NEED(minusg[mg[i]] - 1 == i, CUW_ERR_ARG, "minusg is not an involution");
  }
  std::vector<double> x(ngl), y(ngl), z(ngl);
  for (int i = 0; i < ngl; ++i) {
    x[i] = gvec[3 * i];
    y[i] = gvec[3 * i + 1];
    z[i] = gvec[3 * i + 2];
  }
  std::memcpy(h->gbas, gbas, sizeof(h->gbas));
  h->gweight = gweight;
  h->igvec_h.assign(igvec, igvec + 3 * (size_t)ngl);
  CUW_TRY(cudaMemcpy(g.igvec, igvec, sizeof(int) * 3 * ngl, cudaMemcpyHostToDevice));
  CUW_TRY(cudaMemcpy(g.minusg, mg.data(), sizeof(int) * ngl, cudaMemcpyHostToDevice));
  CUW_TRY(cudaMemcpy(g.gx, x.data(), sizeof(double) * ngl, cudaMemcpyHostToDevice));
  CUW_TRY(cudaMemcpy(g.gy, y.data(), sizeof(double) * ngl, cudaMemcpyHostToDevice));
  CUW_TRY(cudaMemcpy(g.gz, z.data(), sizeof(double) * ngl, cudaMemcpyHostToDevice));
  CUW_TRY(cudaMemcpy(g.g2, g2, sizeof(double) * ngl, cudaMemcpyHostToDevice));
  CUW_TRY(cudaMemcpy(g.pro, pro, sizeof(double) * ngl * (size_t)h->nbarepro, cudaMemcpyHostToDevice));
  CUW_TRY(cudaMemcpy(g.ylm, ylm, sizeof(double) * ngl * (size_t)h->d.lmx, cudaMemcpyHostToDevice));
  CUW_TRY(cudaMemcpy(g.mpsi, mpsi, sizeof(double) * ngl, cudaMemcpyHostToDevice));
  if (bucket) {
    if (!g.bucket) CUW_TRY(cudaMalloc(&g.bucket, sizeof(double) * ngl));
    CUW_TRY(cudaMemcpy(g.bucket, bucket, sizeof(double) * ngl, cudaMemcpyHostToDevice));
    h->tbucket = true;
  } else {
    h->tbucket = false;
  }
  CUW_RET(fft_setup(h, igvec));
  h->have_gset = true;
  return friction_update(h);
}

extern "C" int cuwaves_set_potential(cuw_handle* hp, const double* v) {
  H(hp);
  NEED(v, CUW_ERR_ARG, "null potential");
  CUW_TRY(h->h2d(h->g.v, v, sizeof(double) * h->nr));
  h->have_v = true;
  return CUW_OK;
}

extern "C" int cuwaves_set_dh(cuw_handle* hp, int lmnxx, const double* dh) {
  H(hp);
  NEED(dh && lmnxx >= h->lmnxx, CUW_ERR_ARG, "DH: lmnxx smaller than the largest LMNX");
  const int L = h->lmnxx, nat = h->d.nat;
  std::vector<double2> t((size_t)L * L * std::max(1, nat));
  for (int a = 0; a < nat; ++a)
    for (int j = 0; j < L; ++j)
      for (int i = 0; i < L; ++i) {
        size_t src = 2 * ((size_t)i + (size_t)lmnxx * (j + (size_t)lmnxx * a));
        t[i + (size_t)L * (j + (size_t)L * a)] = make_double2(dh[src], dh[src + 1]);
      }
  CUW_TRY(h->h2d(h->g.dh, t.data(), sizeof(double2) * t.size()));
  h->have_dh = true;
  return CUW_OK;
}

extern "C" int cuwaves_set_do(cuw_handle* hp, int lnxx, const double* dover) {
  H(hp);
  h->touch();
  NEED(dover && lnxx >= h->lnxx, CUW_ERR_ARG, "DO: lnxx smaller than the largest LNX");
  const int L = h->lnxx, nsp = h->d.nsp;
  std::vector<double> t((size_t)L * L * nsp);
  for (int s = 0; s < nsp; ++s)
    for (int j = 0; j < L; ++j)
      for (int i = 0; i < L; ++i) t[i + (size_t)L * (j + (size_t)L * s)] = dover[i + (size_t)lnxx * (j + (size_t)lnxx * s)];
  CUW_TRY(h->h2d(h->g.dover, t.data(), sizeof(double) * t.size()));
  h->have_do = true;
  return CUW_OK;
}

extern "C" int cuwaves_set_atoms(cuw_handle* hp, const double* r0, const double* rp) {
  H(hp);
  const size_t n = sizeof(double) * 3 * h->d.nat;
  h->eigr_src = nullptr;
  if (r0) CUW_TRY(h->h2d(h->g.r0, r0, n, false));
  if (rp) CUW_TRY(h->h2d(h->g.rp, rp, n, false));
  CUW_TRY(h->h2d_done());
  return CUW_OK;
}

extern "C" int cuwaves_reset_atoms(cuw_handle* hp, const double* r0) {
  H(hp);
  h->touch();
  NEED(r0, CUW_ERR_ARG, "null positions");
  const size_t n = sizeof(double) * 3 * h->d.nat;
  h->eigr_src = nullptr;
  CUW_TRY(h->h2d(h->g.r0, r0, n, false));
  CUW_TRY(h->h2d(h->g.rp, r0, n, false));
  CUW_TRY(h->h2d(h->g.rm, r0, n, false));
  CUW_TRY(h->h2d_done());
  return CUW_OK;
}

extern "C" int cuwaves_get_atoms(cuw_handle* hp, double* rm, double* r0, double* rp) {
  H(hp);
  const size_t n = sizeof(double) * 3 * h->d.nat;
  CUW_TRY(cudaStreamSynchronize(h->stream));
  if (rm) CUW_TRY(cudaMemcpy(rm, h->g.rm, n, cudaMemcpyDeviceToHost));
  if (r0) CUW_TRY(cudaMemcpy(r0, h->g.r0, n, cudaMemcpyDeviceToHost));
  if (rp) CUW_TRY(cudaMemcpy(rp, h->g.rp, n, cudaMemcpyDeviceToHost));
  return CUW_OK;
}

extern "C" int cuwaves_set_occ(cuw_handle* hp, const double* occ) {
  H(hp);
  h->touch();
  NEED(occ, CUW_ERR_ARG, "null occupations");
  h->occ_h.assign(occ, occ + h->d.nb);
  CUW_TRY(h->h2d(h->g.occ, occ, sizeof(double) * h->d.nb));
  return CUW_OK;
}

extern "C" int cuwaves_set_dynamics(cuw_handle* hp, double delt, double annee) {
  H(hp);
  h->touch();
  NEED(delt > 0.0 && annee > -1.0, CUW_ERR_ARG, "DELT must be positive and ANNEE > -1");
  h->delt = delt;
  h->annee = annee;
  return friction_update(h);
}

extern "C" int cuwaves_set_cell_friction(cuw_handle* hp, const double* fricmat, double emass, double emasscg2,
                                         const double* dbucket) {
  H(hp);
  CUW_TRY(h->settle());
  h->touch();
  NEED(h->have_gset, CUW_ERR_STATE, "cuwaves_set_gset first");
  if (!fricmat) {
    h->fric_on = false;
    return CUW_OK;
  }
  for (int i = 0; i < 9; ++i) NEED(std::isfinite(fricmat[i]), CUW_ERR_ARG, "FRICMAT must be finite");
  NEED(std::isfinite(emass) && std::isfinite(emasscg2), CUW_ERR_ARG, "EMASS and EMASSCG2 must be finite");
  Device& g = h->g;
  const size_t nb = sizeof(double) * h->d.ngl;
  if (!g.anv) CUW_TRY(cudaMalloc(&g.anv, nb));
  if (dbucket) {
    if (!g.dbucket) CUW_TRY(cudaMalloc(&g.dbucket, nb));
    CUW_TRY(cudaMemcpy(g.dbucket, dbucket, nb, cudaMemcpyHostToDevice));
  }
  h->have_dbucket = dbucket != nullptr;
  std::memcpy(h->fricmat, fricmat, sizeof(h->fricmat));
  h->emass = emass;
  h->emasscg2 = emasscg2;
  h->fric_on = true;
  return friction_update(h);
}

static double2* psi_ptr(Handle* h, int which) {
  switch (which) {
    case CUW_PSI0: return h->g.psi0;
    case CUW_PSIM: return h->g.psim;
    case CUW_HPSI: return h->g.hpsi;
    case CUW_OPSI: return h->g.opsi;
  }
  return nullptr;
}

extern "C" int cuwaves_upload_psi(cuw_handle* hp, int which, const double* psi) {
  H(hp);
  h->touch();
  double2* d = psi_ptr(h, which);
  NEED(d && psi, CUW_ERR_ARG, "bad wave-function selector or null pointer");
  CUW_TRY(cudaMemcpy2DAsync(d, sizeof(double2) * h->ldg, psi, sizeof(double2) * h->d.ngl,
                            sizeof(double2) * h->d.ngl, h->d.nbh, cudaMemcpyHostToDevice, h->stream));
  if (which == CUW_HPSI) h->have_hpsi = true;
  return h->sync();
}

extern "C" int cuwaves_download_psi(cuw_handle* hp, int which, double* psi) {
  H(hp);
  double2* d = psi_ptr(h, which);
  NEED(d && psi, CUW_ERR_ARG, "bad wave-function selector or null pointer");
  CUW_TRY(cudaMemcpy2DAsync(psi, sizeof(double2) * h->d.ngl, d, sizeof(double2) * h->ldg,
                            sizeof(double2) * h->d.ngl, h->d.nbh, cudaMemcpyDeviceToHost, h->stream));
  CUW_TRY(cudaStreamSynchronize(h->stream));
  return CUW_OK;
}

extern "C" int cuwaves_get_proj(cuw_handle* hp, double* proj) {
  H(hp);
  CUW_TRY(cudaMemcpyAsync(proj, h->g.proj, sizeof(double2) * h->d.nbh * h->npro, cudaMemcpyDeviceToHost, h->stream));
  CUW_TRY(cudaStreamSynchronize(h->stream));
  return CUW_OK;
}

extern "C" int cuwaves_set_proj(cuw_handle* hp, const double* proj) {
  H(hp);
  h->touch();
  CUW_TRY(cudaMemcpyAsync(h->g.proj, proj, sizeof(double2) * h->d.nbh * h->npro, cudaMemcpyHostToDevice, h->stream));
  return h->sync();
}

extern "C" int cuwaves_get_rlam0(cuw_handle* hp, double* r) {
  H(hp);
  CUW_TRY(cudaMemcpyAsync(r, h->g.rlam0, sizeof(double2) * h->d.nb * h->d.nb, cudaMemcpyDeviceToHost, h->stream));
  CUW_TRY(cudaStreamSynchronize(h->stream));
  return CUW_OK;
}

extern "C" int cuwaves_set_rlam0(cuw_handle* hp, const double* r) {
  H(hp);
  h->touch();
  CUW_TRY(cudaMemcpyAsync(h->g.rlam0, r, sizeof(double2) * h->d.nb * h->d.nb, cudaMemcpyHostToDevice, h->stream));
  return h->sync();
}

extern "C" int cuwaves_projections(cuw_handle* hp) {
  H(hp);
  h->touch();
  NEED(h->have_gset, CUW_ERR_STATE, "G set not loaded");
  CUW_RET(eigr_compute(h, h->g.r0));
  CUW_RET(proj_compute(h, h->g.psi0, h->g.proj, nullptr, nullptr));
  return h->sync();
}

extern "C" int cuwaves_hpsi(cuw_handle* hp) {
  H(hp);
  h->touch();
  NEED(h->have_gset && h->have_v && h->have_dh, CUW_ERR_STATE, "G set, potential or DH not loaded");
  CUW_RET(fft_vpsi(h, h->g.psi0, h->g.hpsi, true));
  CUW_RET(hproj_compute(h, h->g.proj, h->g.hproj));
  CUW_RET(eigr_compute(h, h->g.r0));
  CUW_RET(addpro_run(h, ADDPRO_HPSI, h->g.hproj, nullptr));
  h->have_hpsi = true;
  return h->sync();
}

extern "C" int cuwaves_ekin(cuw_handle* hp, double* ekin) {
  H(hp);
  NEED(h->have_gset && ekin, CUW_ERR_STATE, "G set not loaded");
  return band_reduce(h, RED_EKIN, ekin, nullptr);
}

extern "C" int cuwaves_expectation(cuw_handle* hp, double* eig) {
  H(hp);
  NEED(h->have_hpsi, CUW_ERR_STATE, "HPSI NOT AVAILABLE");
  NEED(eig, CUW_ERR_ARG, "null eig");
  return band_reduce(h, RED_EXPECT, nullptr, eig);
}

extern "C" int cuwaves_wavekinetic(cuw_handle* hp, double* ekin, double* eig) {
  H(hp);
  NEED(h->have_gset, CUW_ERR_STATE, "G set not loaded");
  double e = 0.0;
  CUW_RET(band_reduce(h, RED_WAVEKIN, &e, eig));
  if (ekin) *ekin = e;
  return CUW_OK;
}

extern "C" int cuwaves_force(cuw_handle* hp, double* force) {
  H(hp);
  NEED(h->have_gset && h->have_dh && h->have_do, CUW_ERR_STATE, "G set, DH or DO not loaded");
  NEED(force, CUW_ERR_ARG, "null force");
  CUW_RET(eigr_compute(h, h->g.r0));
  CUW_RET(force_dev_run(h, h->g.force));
  CUW_TRY(cudaMemcpyAsync(force, h->g.force, sizeof(double) * 3 * h->d.nat, cudaMemcpyDeviceToHost, h->stream));
  CUW_TRY(cudaStreamSynchronize(h->stream));
  return CUW_OK;
}

// WAVES_DENSITY (src/paw_waves1.f90:5377-5500) of this wave-function set, the
// term WAVES$RHO (:4068-4144) adds per (k-point, spin): rho(NR1*NR2*NR3) on
// the host, x fastest.  PSI0 and the occupations of the handle.
extern "C" int cuwaves_density(cuw_handle* hp, double* rho) {
  H(hp);
  NEED(h->have_gset, CUW_ERR_STATE, "G set not loaded");
  NEED(rho, CUW_ERR_ARG, "null rho");
  if (!h->g.rho) CUW_RET(dev_alloc(h, reinterpret_cast<void**>(&h->g.rho), sizeof(double) * h->nr));
  CUW_RET(fft_density(h, h->g.psi0, h->g.rho));
  CUW_TRY(cudaMemcpyAsync(rho, h->g.rho, sizeof(double) * h->nr, cudaMemcpyDeviceToHost, h->stream));
  return h->sync();
}

// WAVES$DENMAT (src/paw_waves1.f90:2957-3134) of this wave-function set:
// denmat and edenmat (LMNXX,LMNXX,NAT) complex as the reference's DENMAT and
// EDENMAT for one spin (edenmat may be NULL), from PROJ, RLAM0 and the
// occupations.
extern "C" int cuwaves_denmat(cuw_handle* hp, int lmnxx, double* denmat, double* edenmat) {
  H(hp);
  NEED(denmat, CUW_ERR_ARG, "null denmat");
  NEED(lmnxx >= h->lmnxx, CUW_ERR_ARG, "lmnxx smaller than the largest LMNX");
  const size_t n = (size_t)lmnxx * lmnxx * std::max(1, h->d.nat);
  double2 *dd = nullptr, *de = nullptr;
  CUW_TRY(cudaMallocAsync(reinterpret_cast<void**>(&dd), sizeof(double2) * n * 2, h->stream));
  de = dd + n;
  int rc = denmat_run(h, lmnxx, dd, edenmat ? de : nullptr);
  if (rc == CUW_OK) {
    cudaMemcpyAsync(denmat, dd, sizeof(double2) * n, cudaMemcpyDeviceToHost, h->stream);
    if (edenmat) cudaMemcpyAsync(edenmat, de, sizeof(double2) * n, cudaMemcpyDeviceToHost, h->stream);
  }
  cudaFreeAsync(dd, h->stream);
  if (rc != CUW_OK) return rc;
  return h->sync();
}

extern "C" int cuwaves_propagate(cuw_handle* hp) {
  H(hp);
  h->touch();
  NEED(h->have_hpsi, CUW_ERR_STATE, "HPSI NOT AVAILABLE: EITHER WAVES$ETOT HAS NOT BEEN CALLED OR WAVES$PROPAGATE HAS BEEN CALLED PREVIOUSLY");
  CUW_RET(propagate_run(h));
  h->have_hpsi = false;
  return h->sync();
}

extern "C" int cuwaves_orthogonalize(cuw_handle* hp, int max_iter, double eps, int* iters) {
  H(hp);
  h->touch();
  NEED(h->have_gset && h->have_do, CUW_ERR_STATE, "G set or DO not loaded");
  NEED(max_iter > 0 && eps > 0.0, CUW_ERR_ARG, "max_iter and eps must be positive");
  // OPSI = (PSI0 + |p>DO<p|PSI0>) * dt^2/((1+annee) m_G) with PROJ at R(0)
  CUW_RET(oproj_compute(h, h->g.proj, h->g.oproj));
  CUW_RET(eigr_compute(h, h->g.r0));
  CUW_RET(addpro_run(h, ADDPRO_OPSI, nullptr, h->g.oproj));
  CUW_RET(ortho_core(h, max_iter, eps));
  int st[2];
  CUW_TRY(cudaMemcpyAsync(st, h->g.ostatus, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
  CUW_TRY(cudaStreamSynchronize(h->stream));
  CUW_RET(ortho_result(h, st, iters));
  // second part of the fictitious kinetic energy (src/paw_waves2.f90:490)
  double e2 = 0.0;
  CUW_RET(band_reduce(h, RED_WAVEKIN, &e2, nullptr));
  h->waveekin2 = e2;
  return h->sync();
}

extern "C" int cuwaves_switch(cuw_handle* hp) {
  H(hp);
  h->touch();
  std::swap(h->g.psi0, h->g.psim);
  CUW_RET(switch_lambda_run(h));
  h->waveekin1 = h->waveekin2 = 0.0;
  return h->sync();
}

extern "C" int cuwaves_stop(cuw_handle* hp) {
  H(hp);
  h->touch();
  CUW_TRY(cudaMemcpyAsync(h->g.psim, h->g.psi0, sizeof(double2) * h->ldg * h->d.nbh, cudaMemcpyDeviceToDevice,
                          h->stream));
  h->have_rlamm = false;
  return h->sync();
}

extern "C" int cuwaves_gramschmidt(cuw_handle* hp, int which, const double* r) {
  H(hp);
  h->touch();
  NEED(h->have_gset && h->have_do, CUW_ERR_STATE, "G set or DO not loaded");
  NEED(which == CUW_PSI0 || which == CUW_PSIM, CUW_ERR_ARG, "Gram-Schmidt acts on PSI0 or PSIM");
  NEED(r, CUW_ERR_ARG, "null positions");
  Device& g = h->g;
  double2* psi = psi_ptr(h, which);
  // The overlap of arbitrary start vectors can be nearly singular: its
  // contractions run in FP64 on every path (restored on every way out)
  struct Fp64Guard {
    Handle* h;
    ~Fp64Guard() { h->fp64_only = false; }
  } fp64_guard{h};
  h->fp64_only = true;
  // atom positions r -> rm slot is not touched: use force buffer as scratch for r
  double* rd = g.force;
  CUW_TRY(cudaMemcpyAsync(rd, r, sizeof(double) * 3 * h->d.nat, cudaMemcpyHostToDevice, h->stream));
  CUW_RET(eigr_compute(h, rd));
  CUW_RET(proj_compute(h, psi, g.hproj, nullptr, nullptr));
  CUW_RET(oproj_compute(h, g.hproj, g.pbuf));
  const size_t mn = (size_t)h->d.nbh * h->d.nbh;
  double2* pw = g.tmat;
  double2* oc = g.tmat + 6 * mn;
  GramPair pc[1] = {{g.hproj, g.pbuf}};
  CUW_RET(gram_projections(h, pc, 1, oc));
  GramPair pp[1] = {{psi, psi}};
  CUW_RET(gram_planewave(h, pp, 1, pw));
  CUW_RET(unravel_run(h, pw, oc, 1, g.mat, nullptr, nullptr));
  CUW_RET(ortho_y_run(h, g.mat, g.wk2));
  CUW_RET(fold_x_run(h, g.wk2, g.lam1c, g.lam2c));
  // PSIINV = PSI (copy into OPSI), PSI += PSIINV X1 + PSIINV(-) X2
  size_t n = (size_t)h->ldg * h->d.nbh;
  k_copy_psi<<<4 * h->nsm, 256, 0, h->stream>>>(psi, g.opsi, n);
  CUW_LAUNCH_CHECK("k_copy_psi");
  CUW_RET(addopsi_run(h, psi, g.opsi, g.lam1c, g.lam2c));
  int st = 0;
  CUW_TRY(cudaMemcpyAsync(&st, g.ostatus, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CUW_TRY(cudaStreamSynchronize(h->stream));
  if (st != CUW_OK) return h->fail(st, "NAN DETECTED in WAVES_ORTHO_Y_C");
  return CUW_OK;
}

// One CP step (see the header).  Kernel order:
//   EKIN, WAVEKINETIC(1) | EIGR(R0) | forces | FFT V.psi | DH.PROJ, DO.PROJ |
//   fused ADDPRO (HPSI, OPSI, PROPAGATE) | <psi|H|psi> | atoms |
//   ORTHOGONALIZE at R(+) | WAVEKINETIC(2) | SWITCH
// Single-point evaluation at the current wave functions and positions, the
// The orthonormality test of WAVES$ORTHOGONALIZE (TTEST block,
// src/paw_waves2.f90:421-460): MAT = <psi_i|O|psi_j> of PSI0, plane-wave part
// (WAVES_OVERLAP) plus one-centre part (WAVES_1COVERLAP) of projections formed
// afresh at R(0), as the real NB x NB matrix of the Gamma point.  Always FP64,
// whatever the handle's precision, so that it measures the state itself.
// Uses only scratch of the step (PBUF, HPROJ, TMAT, WK2); PROJ is untouched.
extern "C" int cuwaves_overlap_check(cuw_handle* hp, double* mat, double* maxdev) {
  H(hp);
  NEED(h->have_gset && h->have_do, CUW_ERR_STATE, "inputs not loaded");
  NEED(mat || maxdev, CUW_ERR_ARG, "no output");
  Device& g = h->g;
  struct Fp64 {
    Handle* h;
    bool old;
    ~Fp64() { h->fp64_only = old; }
  } fp64{h, h->fp64_only};
  h->fp64_only = true;
  const int nb = h->d.nb, nbh = h->d.nbh;
  const size_t mn = (size_t)nbh * nbh;
  CUW_RET(eigr_compute(h, g.r0));
  CUW_RET(proj_compute(h, g.psi0, g.pbuf, nullptr, nullptr));
  CUW_RET(oproj_compute(h, g.pbuf, g.hproj));
  double2* pw = g.tmat;
  double2* oc = g.tmat + 2 * mn;
  GramPair pc[1] = {{g.pbuf, g.hproj}};
  CUW_RET(gram_projections(h, pc, 1, oc));
  GramPair pp[1] = {{g.psi0, g.psi0}};
  CUW_RET(gram_planewave(h, pp, 1, pw));
  CUW_RET(unravel_run(h, pw, oc, 1, g.wk2, nullptr, nullptr));
  std::vector<double> m((size_t)nb * nb);
  CUW_TRY(cudaMemcpyAsync(m.data(), g.wk2, sizeof(double) * m.size(), cudaMemcpyDeviceToHost, h->stream));
  CUW_TRY(cudaStreamSynchronize(h->stream));
  double dev = 0.0;
  for (int j = 0; j < nb; ++j)
    for (int i = 0; i < nb; ++i) dev = std::max(dev, std::fabs(m[i + (size_t)nb * j] - (i == j ? 1.0 : 0.0)));
  if (mat) std::memcpy(mat, m.data(), sizeof(double) * m.size());
  if (maxdev) *maxdev = dev;
  return CUW_OK;
}

// energy part of WAVES$ETOT (src/paw_waves1.f90:2094-2123 with EKIN and FORCE):
// out[0] = sum_n f_n <psi_n|H|psi_n>, out[1] = kinetic energy; force (3*NAT)
// at R(0).  Leaves H|psi> in HPSI; nothing is propagated.
extern "C" int cuwaves_etot(cuw_handle* hp, double* out, double* force) {
  H(hp);
  h->touch();
  NEED(h->have_gset && h->have_v && h->have_dh && h->have_do, CUW_ERR_STATE, "inputs not loaded");
  NEED(out != nullptr, CUW_ERR_ARG, "null output");
  Device& g = h->g;
  double* sc = g.scal;
  double* tmpv = g.scal + 8;
  h->nev = 0;
  CUW_RET(energy_run(h, RED_EKIN, tmpv, sc + 0));
  CUW_RET(eigr_compute(h, g.r0));
  if (force) CUW_RET(force_dev_run(h, g.force));
  CUW_RET(fft_vpsi(h, g.psi0, g.hpsi, true));
  CUW_RET(hproj_compute(h, g.proj, g.hproj));
  CUW_RET(addpro_run(h, ADDPRO_HPSI, g.hproj, g.oproj));
  h->have_hpsi = true;
  CUW_RET(energy_run(h, RED_EXPECT, tmpv, sc + 1));
  double hs[2];
  CUW_TRY(cudaMemcpyAsync(hs, sc, sizeof(double) * 2, cudaMemcpyDeviceToHost, h->stream));
  if (force) CUW_TRY(cudaMemcpyAsync(force, g.force, sizeof(double) * 3 * h->d.nat, cudaMemcpyDeviceToHost, h->stream));
  CUW_TRY(cudaStreamSynchronize(h->stream));
  CUW_RET(h->tc_status());
  out[0] = hs[1];
  out[1] = hs[0];
  return CUW_OK;
}

// The launches of one CP step (everything between the host inputs and the
// results), in the order of TIMESTEP; also the host-side buffer rotation.
static int step_body(Handle* h, int move_atoms, int max_iter, double eps) {
  Device& g = h->g;
  double* sc = g.scal;  // [0] ekin [1] etot [2] ekin1 [3] ekin2 [4] eion ; per-band scratch after 8
  double* tmpv = g.scal + 8;
  CUW_RET(mark(h, PH_RED));
  CUW_RET(energy_run(h, RED_EKIN, tmpv, sc + 0));
  CUW_RET(energy_run(h, RED_WAVEKIN, tmpv, sc + 2));
  CUW_RET(mark(h, PH_EIGR));
  CUW_RET(eigr_compute(h, g.r0));
  if (h->scf) {
    // self-consistent step: the density of PSI0 and POTENTIAL$VOFRHO give the
    // potential of this step (EHARTREE, EXC, int V rho into sc[5..7])
    CUW_RET(mark(h, PH_POT));
    CUW_RET(fft_density(h, g.psi0, g.rho));
    CUW_RET(vofrho_run(h, g.rho));
  }
  CUW_RET(mark(h, PH_FORCE));
  CUW_RET(force_dev_run(h, g.force));
  if (h->scf) {
    k_add_vec<<<ceil_div(3 * h->d.nat, 128), 128, 0, h->stream>>>(g.force, g.fpot, 3 * h->d.nat);
    CUW_LAUNCH_CHECK("k_add_vec");
  }
  CUW_RET(mark(h, PH_FFT));
  CUW_RET(fft_vpsi(h, g.psi0, g.hpsi, true));
  CUW_RET(mark(h, PH_ADDPRO));
  // OPROJ of this PROJ is still in g.oproj from the forces (which turned
  // g.hproj into DEDPRO): only HPROJ is formed again
  CUW_RET(hproj_compute(h, g.proj, g.hproj));
  CUW_RET(addpro_run(h, ADDPRO_FUSED, g.hproj, g.oproj));
  CUW_RET(mark(h, PH_RED));
  CUW_RET(energy_run(h, RED_EXPECT, tmpv, sc + 1));
  CUW_RET(mark(h, PH_MISC));
  if (move_atoms) {
    if (h->eigr_src == g.rp) h->eigr_src = nullptr;  // R(+) is rewritten
    k_atoms_verlet<<<ceil_div(3 * h->d.nat, 128), 128, 0, h->stream>>>(g.r0, g.rm, g.rp, g.force, g.mass, h->d.nat,
                                                                       h->delt * h->delt);
    CUW_LAUNCH_CHECK("k_atoms_verlet");
  }
  CUW_RET(ortho_core(h, max_iter, eps));
  CUW_RET(mark(h, PH_RED));
  CUW_RET(energy_run(h, RED_WAVEKIN, tmpv, sc + 3));
  CUW_RET(mark(h, PH_MISC));
  if (move_atoms) {
    // ATOMS$SWITCH in the same launch: R(-) <- R(0), R(0) <- R(+) by copies
    // (the buffers keep their roles, so a step's launches see the same
    // pointers every time); R(+) keeps R(0) until the next Verlet step, and
    // EIGR of R(+) is now EIGR of R(0)
    k_ion_ekin_switch<<<1, 128, sizeof(double) * 3 * h->d.nat, h->stream>>>(g.rp, g.rm, g.r0, g.mass, h->d.nat,
                                                                             h->delt, sc + 4);
    CUW_LAUNCH_CHECK("k_ion_ekin_switch");
    h->eigr_src = h->eigr_src == g.rp ? g.r0 : nullptr;
  } else {
    CUW_TRY(cudaMemsetAsync(sc + 4, 0, sizeof(double), h->stream));
  }
  std::swap(g.psi0, g.psim);
  CUW_RET(switch_lambda_run(h));
  h->have_hpsi = false;
  return mark(h, PH_MISC);
}

// The step as a CUDA graph when one was captured for the present host-side
// state (Handle::StepGraph), else captured now; returns false (with nothing
// enqueued and the host state untouched) when the step must run uncaptured.
static bool step_graph(Handle* h, int move_atoms, int max_iter, double eps, int* rc) {
  Device& g = h->g;
  const void* key[6] = {g.psi0, g.psim, g.r0, g.rm, g.rp, h->eigr_src};
  const int rlamm = h->have_rlamm ? 1 : 0;
  for (auto it = h->graphs.begin(); it != h->graphs.end();)  // retire graphs of an earlier epoch
    if (it->epoch != h->epoch) {
      cudaGraphExecDestroy(it->exec);
      it = h->graphs.erase(it);
    } else {
      ++it;
    }
  for (Handle::StepGraph& sg : h->graphs) {
    if (std::memcmp(sg.key, key, sizeof(key)) || sg.move != move_atoms || sg.max_iter != max_iter || sg.eps != eps ||
        sg.rlamm != rlamm)
      continue;
    cudaError_t e = cudaGraphLaunch(sg.exec, h->stream);
    if (e != cudaSuccess) {
      *rc = h->fail(CUW_ERR_CUDA, std::string("cudaGraphLaunch: ") + cudaGetErrorString(e));
      return true;
    }
    // the host side of the captured step
    std::swap(g.psi0, g.psim);
    h->eigr_src = sg.eigr_after;
    h->have_hpsi = false;
    h->have_opsi = false;
    h->have_rlamm = true;
    h->launches += sg.launches;
    ++h->graph_replays;
    *rc = CUW_OK;
    return true;
  }
  // capture; on any failure restore the host state and run uncaptured
  Device saved = g;
  const double* eigr_saved = h->eigr_src;
  const bool hp = h->have_hpsi, ho = h->have_opsi, hr = h->have_rlamm;
  const long long l0 = h->launches, ep = h->epoch;
  if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  h->capturing = true;
  const int brc = step_body(h, move_atoms, max_iter, eps);
  h->capturing = false;
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
  cudaGraphExec_t exec = nullptr;
  if (brc == CUW_OK && e == cudaSuccess && graph && h->epoch == ep)
    e = cudaGraphInstantiate(&exec, graph, 0);
  else if (e == cudaSuccess)
    e = cudaErrorUnknown;
  if (graph) cudaGraphDestroy(graph);
  if (e != cudaSuccess || !exec) {
    cudaGetLastError();
    g = saved;
    h->eigr_src = eigr_saved;
    h->have_hpsi = hp;
    h->have_opsi = ho;
    h->have_rlamm = hr;
    h->launches = l0;
    h->err.clear();
    return false;
  }
  Handle::StepGraph sg;
  std::memcpy(sg.key, key, sizeof(key));
  sg.move = move_atoms;
  sg.max_iter = max_iter;
  sg.eps = eps;
  sg.rlamm = rlamm;
  sg.epoch = h->epoch;
  sg.eigr_after = h->eigr_src;
  sg.launches = h->launches - l0;
  sg.exec = exec;
  if (h->graphs.size() >= 12) h->drop_graphs();
  h->graphs.push_back(sg);
  e = cudaGraphLaunch(exec, h->stream);
  *rc = e == cudaSuccess ? CUW_OK : h->fail(CUW_ERR_CUDA, std::string("cudaGraphLaunch: ") + cudaGetErrorString(e));
  return true;
}

extern "C" int cuwaves_cp_step(cuw_handle* hp, int move_atoms, const double* mass, int max_iter, double eps,
                               double* out, double* force) {
  H(hp);
  NEED(h->have_gset && h->have_v && h->have_dh && h->have_do, CUW_ERR_STATE, "inputs not loaded");
  NEED(!move_atoms || mass, CUW_ERR_ARG, "masses required to move atoms");
  Device& g = h->g;
  h->nev = 0;
  if (move_atoms) CUW_TRY(cudaMemcpyAsync(g.mass, mass, sizeof(double) * h->d.nat, cudaMemcpyHostToDevice, h->stream));
  // graphs once the eigenbasis exists and every step enqueues the same launches
  int rc = CUW_OK;
  const bool graphed = h->use_graphs && !h->timing && h->have_u && h->have_rlamm &&
                       step_graph(h, move_atoms, max_iter, eps, &rc);
  if (!graphed) rc = step_body(h, move_atoms, max_iter, eps);
  if (rc != CUW_OK) return rc;
  // results through one page-locked block: three copies, one wait
  const size_t nf = (size_t)3 * h->d.nat;
  if (!h->res_h) CUW_TRY(cudaMallocHost(&h->res_h, sizeof(double) * (16 + std::max<size_t>(nf, 1))));
  double* hs = h->res_h;
  const int* st = reinterpret_cast<const int*>(h->res_h + 8);  // ostatus[0..15]
  CUW_TRY(cudaMemcpyAsync(h->res_h, g.scal, sizeof(double) * 8, cudaMemcpyDeviceToHost, h->stream));
  CUW_TRY(cudaMemcpyAsync(h->res_h + 8, g.ostatus, sizeof(int) * 16, cudaMemcpyDeviceToHost, h->stream));
  if (force && nf) CUW_TRY(cudaMemcpyAsync(h->res_h + 16, g.force, sizeof(double) * nf, cudaMemcpyDeviceToHost, h->stream));
  CUW_TRY(cudaStreamSynchronize(h->stream));
  if (force && nf) std::memcpy(force, h->res_h + 16, sizeof(double) * nf);
  CUW_RET(h->tc_flag(st[12]));
  int iters = 0;
  CUW_RET(ortho_result(h, st, &iters));
  CUW_RET(collect_marks(h));
  if (out) {
    out[0] = hs[1];
    out[1] = hs[0];
    out[2] = 0.5 * (hs[2] + hs[3]);
    out[3] = hs[4];
    out[4] = iters;
    out[5] = out[6] = out[7] = 0.0;
    if (h->scf) {
      // total energy of the self-consistent step: the band energy without
      // int V rho, plus EHARTREE and EXC
      out[0] = hs[1] - hs[7] + hs[5] + hs[6];
      out[5] = hs[5];
      out[6] = hs[6];
      out[7] = hs[7];
    }
  }
  return CUW_OK;
}

// ---------------------------------------------------------------------------
// Batches: many wave-function sets advanced by one CUDA graph launch.  The
// graph holds two CP steps of every set (after two steps PSI0/PSIM are back in
// their buffers, so the same graph serves every later pair), each set's
// launches on its own stream, forked from and joined to the batch's stream:
// the sets' kernels run concurrently on the device and the host issues one
// launch per pair of steps for all of them.  Every set's launches and their
// order are those of cuwaves_cp_step, so the results are bit-identical to
// stepping each set alone.
// ---------------------------------------------------------------------------
struct cuw_batch {
  std::vector<Handle*> hs;
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t exec = nullptr;
  struct Key {
    const void* k[6];
    long long epoch;
    int rlamm;
  };
  std::vector<Key> keys;                  // host state of each set the graph was captured for
  std::vector<const double*> eigr_after;  // EIGR source buffer of each set after a pair of steps
  std::vector<long long> launches;        // kernels per set in the graph
  int move = -1, max_iter = 0;
  double eps = 0.0;
  double* res = nullptr;  // device: [set][step][8] the outputs of cuwaves_cp_step (sc[0..7])
  int* st = nullptr;      // device: [set][step][2] orthogonalisation status and iterations
  std::string err;
  long long replays = 0;
  int fail(int code, const std::string& m) {
    err = m;
    return code;
  }
};

static cuw_batch::Key batch_key(const Handle* h) {
  cuw_batch::Key k;
  const Device& g = h->g;
  const void* v[6] = {g.psi0, g.psim, g.r0, g.rm, g.rp, h->eigr_src};
  std::memcpy(k.k, v, sizeof(v));
  k.epoch = h->epoch;
  k.rlamm = h->have_rlamm ? 1 : 0;
  return k;
}

// Captures two steps of every set into b->exec; on failure every set's host
// state is as before and nothing is enqueued.
static int batch_capture(cuw_batch* b, int move, int max_iter, double eps) {
  const int n = (int)b->hs.size();
  std::vector<Device> saved(n);
  std::vector<const double*> eigr_saved(n);
  std::vector<long long> l0(n);
  std::vector<cuw_batch::Key> keys(n);
  for (int i = 0; i < n; ++i) {
    Handle* h = b->hs[i];
    saved[i] = h->g;
    eigr_saved[i] = h->eigr_src;
    l0[i] = h->launches;
    keys[i] = batch_key(h);
  }
  if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return b->fail(CUW_ERR_CUDA, "batch: stream capture could not start");
  }
  int rc = CUW_OK;
  cudaError_t e = cudaEventRecord(b->fork, b->stream);
  for (int i = 0; i < n && e == cudaSuccess; ++i) {
    e = cudaStreamWaitEvent(b->hs[i]->stream, b->fork, 0);
    b->hs[i]->capturing = true;
  }
  for (int s = 0; s < 2 && e == cudaSuccess && rc == CUW_OK; ++s)
    for (int i = 0; i < n && rc == CUW_OK; ++i) {
      Handle* h = b->hs[i];
      h->nev = 0;
      rc = step_body(h, move, max_iter, eps);
      if (rc != CUW_OK) {
        b->err = h->err;
        break;
      }
      const size_t slot = (size_t)i * 2 + s;
      k_batch_out<<<1, 32, 0, h->stream>>>(h->g.scal, h->g.ostatus, b->res + slot * 8, b->st + slot * 2);
      ++h->launches;
      e = cudaGetLastError();
      if (e != cudaSuccess) rc = CUW_ERR_CUDA;
    }
  for (int i = 0; i < n; ++i) {
    Handle* h = b->hs[i];
    if (cudaEventRecord(b->join[i], h->stream) == cudaSuccess) cudaStreamWaitEvent(b->stream, b->join[i], 0);
    h->capturing = false;
  }
  cudaGraph_t graph = nullptr;
  cudaError_t ee = cudaStreamEndCapture(b->stream, &graph);
  cudaGraphExec_t exec = nullptr;
  if (rc == CUW_OK && e == cudaSuccess && ee == cudaSuccess && graph) ee = cudaGraphInstantiate(&exec, graph, 0);
  if (graph) cudaGraphDestroy(graph);
  if (rc != CUW_OK || e != cudaSuccess || ee != cudaSuccess || !exec) {
    cudaGetLastError();
    for (int i = 0; i < n; ++i) {
      Handle* h = b->hs[i];
      h->g = saved[i];
      h->eigr_src = eigr_saved[i];
      h->launches = l0[i];
      h->err.clear();
    }
    return b->fail(rc != CUW_OK ? rc : CUW_ERR_CUDA,
                   "batch: the steps could not be captured" + (b->err.empty() ? std::string() : ": " + b->err));
  }
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = exec;
  b->keys = keys;
  b->eigr_after.resize(n);
  b->launches.resize(n);
  for (int i = 0; i < n; ++i) {
    b->eigr_after[i] = b->hs[i]->eigr_src;
    b->launches[i] = b->hs[i]->launches - l0[i];
  }
  b->move = move;
  b->max_iter = max_iter;
  b->eps = eps;
  return CUW_OK;
}

extern "C" int cuwaves_batch_create(cuw_handle* const* handles, int n, cuw_batch** out) {
  if (!handles || n <= 0 || !out) return CUW_ERR_ARG;
  *out = nullptr;
  cuw_batch* b = new cuw_batch();
  for (int i = 0; i < n; ++i) {
    Handle* h = reinterpret_cast<Handle*>(handles[i]);
    if (!h) {
      delete b;
      return CUW_ERR_ARG;
    }
    for (Handle* o : b->hs)
      if (o == h) {
        delete b;
        return CUW_ERR_ARG;  // a set may appear once
      }
    b->hs.push_back(h);
  }
  int dev = b->hs[0]->device;
  bool ok = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess;
  b->join.assign(n, nullptr);
  for (int i = 0; i < n && ok; ++i) {
    ok = b->hs[i]->device == dev && cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming) == cudaSuccess;
  }
  ok = ok && cudaMalloc(&b->res, sizeof(double) * 16 * (size_t)n) == cudaSuccess &&
       cudaMalloc(&b->st, sizeof(int) * 4 * (size_t)n) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    cuwaves_batch_destroy(b);
    return CUW_ERR_CUDA;
  }
  *out = b;
  return CUW_OK;
}

extern "C" int cuwaves_batch_step(cuw_batch* b, int move_atoms, const double* const* mass, int max_iter, double eps,
                                  double* out) {
  if (!b) return CUW_ERR_ARG;
  const int n = (int)b->hs.size();
  if (move_atoms && !mass) return b->fail(CUW_ERR_ARG, "masses required to move atoms");
  for (int i = 0; i < n; ++i) {
    Handle* h = b->hs[i];
    if (!(h->have_gset && h->have_v && h->have_dh && h->have_do))
      return b->fail(CUW_ERR_STATE, "batch: set " + std::to_string(i) + ": inputs not loaded");
    if (!(h->have_u && h->have_rlamm))
      return b->fail(CUW_ERR_STATE, "batch: set " + std::to_string(i) + ": take one cuwaves_cp_step first");
    if (h->timing || h->async) return b->fail(CUW_ERR_STATE, "batch: timing or asynchronous mode is on");
    if (move_atoms && !mass[i]) return b->fail(CUW_ERR_ARG, "batch: masses of set " + std::to_string(i));
  }
  for (int i = 0; i < n; ++i) {
    Handle* h = b->hs[i];
    CUW_BATCH_TRY(cudaStreamSynchronize(h->stream));
    if (move_atoms)
      CUW_BATCH_TRY(cudaMemcpyAsync(h->g.mass, mass[i], sizeof(double) * h->d.nat, cudaMemcpyHostToDevice, b->stream));
  }
  bool same = b->exec && b->move == move_atoms && b->max_iter == max_iter && b->eps == eps &&
              (int)b->keys.size() == n;
  for (int i = 0; i < n && same; ++i) {
    const cuw_batch::Key k = batch_key(b->hs[i]);
    same = std::memcmp(k.k, b->keys[i].k, sizeof(k.k)) == 0 && k.epoch == b->keys[i].epoch &&
           k.rlamm == b->keys[i].rlamm;
  }
  if (same) {
    CUW_BATCH_TRY(cudaGraphLaunch(b->exec, b->stream));
    for (int i = 0; i < n; ++i) {
      Handle* h = b->hs[i];
      h->eigr_src = b->eigr_after[i];  // the PSI0/PSIM swaps of two steps cancel
      h->launches += b->launches[i];
      h->graph_replays += 2;
    }
    ++b->replays;
  } else {
    CUW_BATCH_TRY(cudaStreamSynchronize(b->stream));
    const int rc = batch_capture(b, move_atoms, max_iter, eps);
    if (rc != CUW_OK) return rc;
    CUW_BATCH_TRY(cudaGraphLaunch(b->exec, b->stream));
  }
  for (Handle* h : b->hs) {
    h->have_hpsi = false;
    h->have_opsi = false;
    h->have_rlamm = true;
  }
  std::vector<double> res((size_t)16 * n);
  std::vector<int> st((size_t)4 * n);
  CUW_BATCH_TRY(cudaMemcpyAsync(res.data(), b->res, sizeof(double) * res.size(), cudaMemcpyDeviceToHost, b->stream));
  CUW_BATCH_TRY(cudaMemcpyAsync(st.data(), b->st, sizeof(int) * st.size(), cudaMemcpyDeviceToHost, b->stream));
  CUW_BATCH_TRY(cudaStreamSynchronize(b->stream));
  int rc = CUW_OK;
  for (int i = 0; i < n; ++i) {
    Handle* h = b->hs[i];
    int r = h->tc_status();
    for (int s = 0; s < 2; ++s) {
      const size_t slot = (size_t)i * 2 + s;
      int iters = 0;
      if (r == CUW_OK) r = ortho_result(h, &st[slot * 2], &iters);
      if (out) {
        const double* hs = &res[slot * 8];
        double* o = out + slot * 8;
        o[0] = hs[1];
        o[1] = hs[0];
        o[2] = 0.5 * (hs[2] + hs[3]);
        o[3] = hs[4];
        o[4] = iters;
        o[5] = o[6] = o[7] = 0.0;
        if (h->scf) {
          o[0] = hs[1] - hs[7] + hs[5] + hs[6];
          o[5] = hs[5];
          o[6] = hs[6];
          o[7] = hs[7];
        }
      }
    }
    if (r != CUW_OK && rc == CUW_OK) {
      rc = r;
      b->err = "set " + std::to_string(i) + ": " + h->err;
    }
  }
  return rc;
}

extern "C" int cuwaves_batch_error(const cuw_batch* b, char* buf, int len) {
  if (!b || !buf || len <= 0) return CUW_ERR_ARG;
  std::snprintf(buf, (size_t)len, "%s", b->err.c_str());
  return CUW_OK;
}

extern "C" int cuwaves_batch_destroy(cuw_batch* b) {
  if (!b) return CUW_OK;
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->fork) cudaEventDestroy(b->fork);
  for (cudaEvent_t e : b->join)
    if (e) cudaEventDestroy(e);
  if (b->res) cudaFree(b->res);
  if (b->st) cudaFree(b->st);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return CUW_OK;
}

extern "C" int cuwaves_set_timing(cuw_handle* hp, int enable) {
  H(hp);
  h->timing = enable != 0;
  for (int i = 0; i < Handle::kPhases; ++i) h->phase_ms[i] = 0.0;
  h->phase_calls = 0;
  h->nev = 0;
  return CUW_OK;
}

extern "C" int cuwaves_get_timing(cuw_handle* hp, double* ms, int n, long long* launches, long long* steps) {
  H(hp);
  for (int i = 0; i < n && i < Handle::kPhases; ++i) ms[i] = h->phase_ms[i];
  if (launches) *launches = h->launches;
  if (steps) *steps = h->phase_calls;
  return CUW_OK;
}

extern "C" int cuwaves_get_stream(cuw_handle* hp, void** stream) {
  H(hp);
  if (!stream) return h->fail(CUW_ERR_ARG, "null stream pointer");
  *stream = reinterpret_cast<void*>(h->stream);
  return CUW_OK;
}

extern "C" int cuwaves_get_ortho_stats(cuw_handle* hp, double* out, int n) {
  H(hp);
  if (!out || n < 1) return h->fail(CUW_ERR_ARG, "bad output buffer");
  int st[16] = {0};
  CUW_TRY(cudaMemcpyAsync(st, h->g.ostatus, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
  CUW_TRY(cudaStreamSynchronize(h->stream));
  const double v[5] = {(double)st[10], (double)st[8], (double)st[4], (double)st[1], (double)st[9]};
  for (int i = 0; i < n && i < 5; ++i) out[i] = v[i];
  return CUW_OK;
}

extern "C" int cuwaves_get_graph_stats(cuw_handle* hp, long long* graphs, long long* replays) {
  H(hp);
  if (graphs) *graphs = (long long)h->graphs.size();
  if (replays) *replays = h->graph_replays;
  return CUW_OK;
}

extern "C" int cuwaves_set_option(cuw_handle* hp, int option, double value) {
  H(hp);
  h->touch();
  switch (option) {
    case CUW_OPT_LYAP_TOL:
      if (!(value >= 0.0 && value < 0.1)) return h->fail(CUW_ERR_ARG, "LYAP_TOL must be in [0, 0.1)");
      h->lyap_tol = value;
      return CUW_OK;
    case CUW_OPT_LYAP_MAX_SWEEPS:
      if (!(value >= 1.0 && value <= 1000.0)) return h->fail(CUW_ERR_ARG, "LYAP_MAX_SWEEPS must be in [1, 1000]");
      h->lyap_max_sweeps = (int)value;
      return CUW_OK;
    case CUW_OPT_GRAPHS:
      h->use_graphs = value != 0.0;
      if (!h->use_graphs) h->drop_graphs();
      return CUW_OK;
    case CUW_OPT_FFT_VARIANT: {
      const int v = (int)value;
      if ((double)v != value) return h->fail(CUW_ERR_ARG, "FFT_VARIANT must be an integer");
      const int rc = fft_set_variant(h, v);
      if (rc == CUW_ERR_UNSUPPORTED) return h->fail(rc, "FFT plan variant not available for this grid");
      return rc;
    }
    case CUW_OPT_STREAM_PRIORITY: {
      if (value != 0.0 && value != 1.0) return h->fail(CUW_ERR_ARG, "STREAM_PRIORITY must be 0 or 1");
      const int want = value != 0.0 ? 1 : 0;
      if (want == h->stream_prio) return CUW_OK;
      int least = 0, greatest = 0;
      CUW_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
      cudaStream_t s = nullptr;
      CUW_TRY(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, want ? greatest : least));
      if (cudaError_t e = cudaStreamSynchronize(h->stream); e != cudaSuccess) {
        cudaStreamDestroy(s);
        return h->fail(CUW_ERR_CUDA, std::string("cudaStreamSynchronize: ") + cudaGetErrorString(e));
      }
      cudaStreamDestroy(h->stream);
      h->stream = s;
      h->stream_prio = want;
      h->drop_graphs();
      h->touch();
      return CUW_OK;
    }
    case CUW_OPT_SM_SHARE: {
      const int v = (int)value;
      if ((double)v != value || v < 0) return h->fail(CUW_ERR_ARG, "SM_SHARE must be a non-negative integer");
      h->nsm = v == 0 ? h->nsm_dev : std::min(v, h->nsm_dev);
      h->drop_graphs();
      return CUW_OK;
    }
    case CUW_OPT_CONTRACTION_TILES:
      if (value != 0.0 && value != 1.0) return h->fail(CUW_ERR_ARG, "CONTRACTION_TILES must be 0 or 1");
      if (!h->mixed() && value == 0.0) return h->fail(CUW_ERR_ARG, "FP64 handles have DMMA tiles only");
      h->dmma_tiles = value != 0.0;
      return CUW_OK;
    case CUW_OPT_SAFEORTHO:
      if (value != 0.0 && value != 1.0) return h->fail(CUW_ERR_ARG, "SAFEORTHO must be 0 or 1");
      h->safeortho = value != 0.0;
      return CUW_OK;
    case CUW_OPT_SWAPSTATES:
      if (value != 0.0 && value != 1.0) return h->fail(CUW_ERR_ARG, "SWAPSTATES must be 0 or 1");
      h->swapstates = value != 0.0;
      return CUW_OK;
    case CUW_OPT_SELFCONSISTENT:
      if (value != 0.0 && !(h->have_rhoset && h->have_qlm))
        return h->fail(CUW_ERR_STATE, "self-consistent steps need cuwaves_set_rhoset and cuwaves_set_qlm");
      h->scf = value != 0.0;
      return CUW_OK;
    default:
      return h->fail(CUW_ERR_ARG, "unknown option");
  }
}
