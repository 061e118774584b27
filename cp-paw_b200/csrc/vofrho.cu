// The local potential from the density: POTENTIAL$VOFRHO on the device.
//
// Reference: POTENTIAL$VOFRHO (src/paw_potential.f90:324-485) and
// POTENTIAL_VOFRHO (:487-895) at the Gamma point for one spin, LDA, without
// stress, confining potential, pair potential or isolation:
//   RHOG   = SUPFFT('RTOG', RHOE)                      (:600)
//   RHOG  += pseudo core                 POTENTIAL_ADDCORE (:1038-1066)
//   Hartree energy, potential, forces, VQLM  POTENTIAL_HARTREE (:1069-1336)
//   RHOE   = SUPFFT('GTOR', RHOG)                      (:747)
//   XC energy and potential on the grid    POTENTIAL_XC (:1339-1545), DFT
//   RHOG   = SUPFFT('RTOG', VXC) + VHARTREE            (:778-800)
//   forces on the pseudo core              POTENTIAL_FPSCORE (:897-975)
//   RHOE   = SUPFFT('GTOR', RHOG)  -> the potential    (:890)
//
// B200 layout: every pass is one kernel over the NGLH vectors of the density
// set (one G of each +-G pair) or over the grid; the three transforms of one
// real function run on a full FP64 complex grid (grid_fft, fft.cu).  The
// structure factors exp(-iG.R) are formed in registers (sincos), the sums over
// G are block partials added in a fixed order by one final block, so results
// do not depend on the launch.  All of it stays on the handle's stream and
// enqueues no host round trip (the self-consistent CP step replays it inside
// its CUDA graph).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "cuwaves_internal.cuh"

namespace cuw {

namespace {

constexpr int kVT = 256;     // threads per block of the G and grid passes
constexpr int kLmMax = 25;   // LMRXX limit (l <= 4)
constexpr double kPi = 3.14159265358979323846264338327950288;

// (-i)^l / (2l+1)!! : the CFAC of POTENTIAL_HARTREE (:1143-1152, 1247-1255)
__device__ __forceinline__ double2 cfac_of(int lm) {
  int l = 0;
  while ((l + 1) * (l + 1) <= lm) ++l;
  double d = 1.0;
  for (int k = 1; k <= l; ++k) d /= (double)(2 * k + 1);
  const double2 m = mipow(l);
  return make_double2(m.x * d, m.y * d);
}

__device__ __forceinline__ double2 eigr_of(double gx, double gy, double gz, const double* r) {
  double s, c;
  sincos(gx * r[0] + gy * r[1] + gz * r[2], &s, &c);
  return make_double2(c, -s);
}

// block sum of one value per thread (kVT threads), returned to thread 0
__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < kVT / 32; ++i) t += sh[i];
  return t;
}

// DFT (src/paw_dft.f90:780-967) for functional type 2 (LDA: local exchange,
// EXCHANGE_X1 :2137-2236, plus the Perdew-Wang local correlation of the
// unpolarised gas, PERDEWWANG91L_RHODEP1 :4521-4575, without tables since
// TSAFE is .TRUE.); RHOTMIN = 1e-6 (:62) and the wrap-up of :931-935.
__device__ double dft_lda(double rhot, double* vxc) {
  const double rhotmin = 1e-6;
  const double val = rhot < rhotmin ? rhotmin : rhot;
  const double kffac = pow(3.0 * kPi * kPi, 1.0 / 3.0);
  const double exfac = -3.0 / (4.0 * kPi) * kffac;
  double ex = 0.0, ex_r = 0.0;
  if (fabs(val) >= 1e-50) {
    const double r13 = pow(val, 1.0 / 3.0), r23 = r13 * r13, r43 = r23 * r23;
    ex = exfac * r43;
    ex_r = ex * (4.0 / 3.0) / val;
  }
  const double au = 3.10907e-2, alpha1 = 2.1370e-1, beta1 = 7.5957, beta2 = 3.5876, beta3 = 1.6382,
               beta4 = 4.9294e-1;
  const double rsfac = pow(3.0 / (4.0 * kPi), 1.0 / 3.0);
  const double rs = rsfac / pow(val, 1.0 / 3.0);
  const double sqrs = sqrt(rs), rssqrs = rs * sqrs;
  const double sv1 = -2.0 * au * (1.0 + alpha1 * rs), dsv1 = -2.0 * au * alpha1;
  const double sv2 = 2.0 * au * sqrs * (beta1 + beta2 * sqrs + beta3 * rs + beta4 * rssqrs);
  const double dsv2 = au / sqrs * (beta1 + 2.0 * beta2 * sqrs + 3.0 * beta3 * rs + 4.0 * beta4 * rssqrs);
  const double sv3 = 1.0 + 1.0 / sv2, dsv3 = -dsv2 / (sv2 * sv2);
  const double sv4 = log(sv3), dsv4 = dsv3 / sv3;
  const double ecu = sv1 * sv4;
  const double decu = (dsv1 * sv4 + sv1 * dsv4) * (-(1.0 / 3.0) * rs / val);
  const double ec = val * ecu, dec = val * decu + ecu;
  double exc = ex + ec, dexc = ex_r + dec;
  if (rhot < rhotmin) {
    dexc = exc / rhotmin;
    exc = exc * rhot / rhotmin;
  }
  *vxc = dexc;
  return exc;
}

__global__ void k_vr_load(const double* __restrict__ rho, double2* __restrict__ grid, size_t nr) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nr; i += (size_t)gridDim.x * blockDim.x)
    grid[i] = make_double2(rho[i], 0.0);
}

// PLANEWAVE$SUPFFT('RTOG') unravelling (src/paw_fft.f90:1924-1936):
// out(G) = 0.5 (F(G) + conj F(-G)) * scale (+ add(G))
__global__ void k_vr_gather(const double2* __restrict__ grid, const int* __restrict__ plus,
                            const int* __restrict__ minus, int nglh, double scale, const double2* __restrict__ add,
                            double2* __restrict__ out) {
  const int ig = blockIdx.x * blockDim.x + threadIdx.x;
  if (ig >= nglh) return;
  const double2 f1 = grid[plus[ig]], f2 = grid[minus[ig]];
  double2 v = make_double2(0.5 * (f1.x + f2.x) * scale, 0.5 * (f1.y - f2.y) * scale);
  if (add) v = cadd(v, add[ig]);
  out[ig] = v;
}

// PLANEWAVE$SUPFFT('GTOR') set-up (src/paw_fft.f90:1856-1870) on a zeroed grid:
// F(G) = f, F(-G) = conj f (the second store wins for G = 0, as there)
__global__ void k_vr_scatter(const double2* __restrict__ f, const int* __restrict__ plus,
                             const int* __restrict__ minus, int nglh, double2* __restrict__ grid) {
  const int ig = blockIdx.x * blockDim.x + threadIdx.x;
  if (ig >= nglh) return;
  const double2 v = f[ig];
  grid[plus[ig]] = v;
  grid[minus[ig]] = cconj(v);
}

struct VrSet {
  const double *gx, *gy, *gz, *g2, *ylm, *g0, *v0, *pscore, *vbar, *qlm, *r0;
  const int *lmrx, *isp;
  int nglh, lmrxx, nat, ngamma;
};

// POTENTIAL_ADDCORE (:1038-1066) and the energy part of POTENTIAL_HARTREE
// (:1129-1200) for one G per thread: rhog gains the pseudo core; vg and pot
// (VHARTREE) are formed; RHOB (the thread of G = 0) goes to out[2]; the
// energy terms are summed per block into epart.
__global__ void __launch_bounds__(kVT) k_vr_hartree(VrSet s, double2* __restrict__ rhog, double2* __restrict__ vg,
                                                    double2* __restrict__ pot, double* __restrict__ out,
                                                    double* __restrict__ epart) {
  __shared__ double sh[kVT / 32];
  const int ig = blockIdx.x * blockDim.x + threadIdx.x;
  const double y0 = 1.0 / sqrt(4.0 * kPi);
  double e = 0.0;
  if (ig < s.nglh) {
    const double gx = s.gx[ig], gy = s.gy[ig], gz = s.gz[ig];
    double2 rho = rhog[ig];
    for (int a = 0; a < s.nat; ++a) {
      const int sp = s.isp[a];
      const double2 ei = eigr_of(gx, gy, gz, s.r0 + 3 * a);
      rho = cadd(rho, cscale(ei, s.pscore[ig + (size_t)s.nglh * sp] * y0));
    }
    double2 rho2 = rho, p = make_double2(0.0, 0.0);
    double vb = 0.0;
    const double* y = s.ylm + (size_t)s.lmrxx * ig;
    for (int a = 0; a < s.nat; ++a) {
      const int sp = s.isp[a];
      const double2 ei = eigr_of(gx, gy, gz, s.r0 + 3 * a);
      const double* q = s.qlm + (size_t)s.lmrxx * a;
      if (ig == s.ngamma) vb += q[0] * y0 * s.v0[s.ngamma + (size_t)s.nglh * sp];
      double2 c = make_double2(0.0, 0.0);
      for (int lm = 0; lm < s.lmrx[sp]; ++lm) c = cadd(c, cscale(cfac_of(lm), q[lm] * y[lm]));
      c = cmul(c, ei);
      const size_t k = ig + (size_t)s.nglh * sp;
      rho2 = cadd(rho2, cscale(c, s.g0[k]));
      p = cadd(p, cadd(cscale(c, s.v0[k]), cscale(ei, s.vbar[k] * y0)));
    }
    double2 v;
    if (ig != s.ngamma) {
      v = cscale(rho2, 4.0 * kPi / s.g2[ig]);
      // Re(0.5 conj(rho2) vg + conj(rho) pot)
      e = 0.5 * (rho2.x * v.x + rho2.y * v.y) + (rho.x * p.x + rho.y * p.y);
    } else {
      const double rhob = -rho2.x;
      v = make_double2(-vb, 0.0);
      e = 0.5 * ((rho.x * p.x + rho.y * p.y) + rhob * vb);
      out[2] = rhob;
    }
    rhog[ig] = rho;
    vg[ig] = v;
    pot[ig] = cadd(p, v);
  }
  const double t = block_sum(e, sh);
  if (threadIdx.x == 0) epart[blockIdx.x] = t;
}

// Forces and VQLM of POTENTIAL_HARTREE (:1240-1319) and the forces on the
// pseudo core of POTENTIAL_FPSCORE (:897-975) for atom blockIdx.y over the G
// vectors of block blockIdx.x; per block and atom: part[0..2] Hartree force,
// part[3..5] pseudo-core force, part[6..] VQLM (unscaled sums).
__global__ void __launch_bounds__(kVT) k_vr_forces(VrSet s, const double2* __restrict__ rhog,
                                                   const double2* __restrict__ vg, const double2* __restrict__ vtot,
                                                   const double* __restrict__ out, double* __restrict__ part) {
  __shared__ double sh[kVT / 32];
  const int ig = blockIdx.x * blockDim.x + threadIdx.x, a = blockIdx.y;
  const int sp = s.isp[a];
  const double y0 = 1.0 / sqrt(4.0 * kPi);
  double fh[3] = {0.0, 0.0, 0.0}, fc[3] = {0.0, 0.0, 0.0}, vq[kLmMax];
  for (int lm = 0; lm < kLmMax; ++lm) vq[lm] = 0.0;
  if (ig < s.nglh) {
    const double gv[3] = {s.gx[ig], s.gy[ig], s.gz[ig]};
    const double2 ei = eigr_of(gv[0], gv[1], gv[2], s.r0 + 3 * a);
    const size_t k = ig + (size_t)s.nglh * sp;
    const double g0 = s.g0[k], v0 = s.v0[k];
    const double2 rho = rhog[ig];
    double2 rho2 = rho;
    if (ig == s.ngamma) rho2.x += out[2];  // N_A = RHOTILDE + N_B (:1243-1246)
    const double2 w = vg[ig];
    // AVAL = (G0 conj(VG) + V0 conj(RHO2)) EIGR
    const double2 av0 = make_double2(g0 * w.x + v0 * rho2.x, -(g0 * w.y + v0 * rho2.y));
    const double2 aval = cmul(av0, ei);
    const double* y = s.ylm + (size_t)s.lmrxx * ig;
    const double* q = s.qlm + (size_t)s.lmrxx * a;
    if (ig == s.ngamma) vq[0] -= 0.5 * cmul(cscale(cfac_of(0), y[0]), aval).x;
    double2 cs = make_double2(0.0, 0.0);
    for (int lm = 0; lm < s.lmrx[sp]; ++lm) {
      const double2 c = cscale(cfac_of(lm), y[lm]);
      vq[lm] += cmul(c, aval).x;
      cs = cadd(cs, cscale(c, q[lm]));
    }
    // CVAL = VBAR Y0 EIGR conj(RHO); SVAR = Im(CVAL + CSUM AVAL)
    const double2 cval = cmulc(cscale(ei, s.vbar[k] * y0), rho);
    const double sv = (cval.y + cmul(cs, aval).y);
    // pseudo core: -Im(conj(V) PSCORE EIGR)
    const double2 c2 = cmulc(cscale(ei, s.pscore[k]), vtot[ig]);
    const double svc = -c2.y;
    for (int d = 0; d < 3; ++d) {
      fh[d] = -gv[d] * sv;
      fc[d] = svc * gv[d];
    }
  }
  const int nk = 6 + s.lmrxx;
  double* dst = part + ((size_t)blockIdx.x * s.nat + a) * nk;
  for (int d = 0; d < 3; ++d) {
    const double t = block_sum(fh[d], sh);
    if (threadIdx.x == 0) dst[d] = t;
    const double u = block_sum(fc[d], sh);
    if (threadIdx.x == 0) dst[3 + d] = u;
  }
  for (int lm = 0; lm < s.lmrxx; ++lm) {
    const double t = block_sum(lm < kLmMax ? vq[lm] : 0.0, sh);
    if (threadIdx.x == 0) dst[6 + lm] = t;
  }
}

// POTENTIAL_XC (:1339-1545) for the LDA: RHOT = max(RHO, 1e-8) per grid point,
// EXC summed per block, the potential written back onto the grid
__global__ void __launch_bounds__(kVT) k_vr_xc(double2* __restrict__ grid, size_t nr, double* __restrict__ epart) {
  __shared__ double sh[kVT / 32];
  double e = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nr; i += (size_t)gridDim.x * blockDim.x) {
    const double rhot = fmax(grid[i].x, 1e-8);
    double vt;
    e += dft_lda(rhot, &vt);
    grid[i] = make_double2(vt, 0.0);
  }
  const double t = block_sum(e, sh);
  if (threadIdx.x == 0) epart[blockIdx.x] = t;
}

// the real part of the grid into v; with rho, block sums of v * rho
__global__ void __launch_bounds__(kVT) k_vr_store(const double2* __restrict__ grid, double* __restrict__ v,
                                                  const double* __restrict__ rho, size_t nr,
                                                  double* __restrict__ dpart) {
  __shared__ double sh[kVT / 32];
  double e = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nr; i += (size_t)gridDim.x * blockDim.x) {
    const double x = grid[i].x;
    v[i] = x;
    if (rho) e += x * rho[i];
  }
  const double t = block_sum(e, sh);
  if (rho && threadIdx.x == 0) dpart[blockIdx.x] = t;
}

// the block partials in a fixed order: energies (EHARTREE, EXC, and RHOB or
// int V rho as the third value), forces and VQLM with their weights
__global__ void k_vr_final(const double* __restrict__ ehpart, int neh, const double* __restrict__ xcpart, int nxc,
                           const double* __restrict__ dpart, int nd, const double* __restrict__ fpart, int nfb,
                           int nat, int lmrxx, double cellvol, double nr, const double* __restrict__ out_in,
                           double* __restrict__ eout, double* __restrict__ force, double* __restrict__ vqlm) {
  const double y0 = 1.0 / sqrt(4.0 * kPi);
  const int nk = 6 + lmrxx;
  if (threadIdx.x == 0) {
    double eh = 0.0, ex = 0.0, ed = 0.0;
    for (int i = 0; i < neh; ++i) eh += ehpart[i];
    for (int i = 0; i < nxc; ++i) ex += xcpart[i];
    if (dpart)
      for (int i = 0; i < nd; ++i) ed += dpart[i];
    const double rhob = out_in[2];
    eout[0] = eh * 2.0 * cellvol;
    eout[1] = ex * cellvol / nr;
    eout[2] = dpart ? ed * cellvol / nr : rhob;
  }
  for (int idx = threadIdx.x; idx < nat * nk; idx += blockDim.x) {
    const int a = idx / nk, k = idx % nk;
    double t = 0.0;
    for (int b = 0; b < nfb; ++b) t += fpart[((size_t)b * nat + a) * nk + k];
    if (k < 3) {
      double u = 0.0;
      for (int b = 0; b < nfb; ++b) u += fpart[((size_t)b * nat + a) * nk + 3 + k];
      force[3 * a + k] = t * 2.0 * cellvol + u * y0 * 2.0 * cellvol;
    } else if (k >= 6) {
      vqlm[(k - 6) + (size_t)lmrxx * a] = t * 2.0 * cellvol;
    }
  }
}

int gblocks(int n) { return ceil_div(n, kVT); }
int rblocks(const Handle* h) { return (int)std::min<size_t>((h->nr + kVT - 1) / kVT, (size_t)8 * h->nsm); }

}  // namespace

// POTENTIAL$VOFRHO of the density rho_dev (device, NR) at R(0): the potential
// goes to h->g.v, the Hartree + pseudo-core forces to h->g.fpot, VQLM to
// h->g.vqlm; eout (device, 3 values) receives EHARTREE, EXC and RHOB, or with
// edc, int V rho instead of RHOB.
static int vofrho_enqueue(Handle* h, const double* rho_dev, double* eout, bool edc) {
  Device& g = h->g;
  const int nglh = h->nglh, nat = h->d.nat;
  VrSet s{g.r_gx, g.r_gy, g.r_gz, g.r_g2, g.r_ylm, g.r_g0, g.r_v0, g.r_pscore, g.r_vbar, g.qlm, g.r0,
          g.r_lmrx, g.t_isp, nglh, h->lmrxx, nat, h->ngamma};
  const size_t nr = h->nr;
  const int gb = gblocks(nglh), rb = rblocks(h);
  double* ehpart = g.r_part;
  double* xcpart = ehpart + gb;
  double* dpart = xcpart + rb;
  double* fpart = dpart + rb;
  CUW_TRY(cudaMemsetAsync(g.r_out, 0, sizeof(double) * 4, h->stream));
  // RHOG = SUPFFT('RTOG', rho)
  k_vr_load<<<rb, kVT, 0, h->stream>>>(rho_dev, g.r_grid, nr);
  CUW_LAUNCH_CHECK("k_vr_load");
  CUW_RET(grid_fft(h, g.r_grid, -1));
  k_vr_gather<<<gb, kVT, 0, h->stream>>>(g.r_grid, g.r_plus, g.r_minus, nglh, 1.0 / (double)nr, nullptr, g.r_rhog);
  CUW_LAUNCH_CHECK("k_vr_gather");
  // pseudo core and Hartree
  k_vr_hartree<<<gb, kVT, 0, h->stream>>>(s, g.r_rhog, g.r_vg, g.r_pot, g.r_out, ehpart);
  CUW_LAUNCH_CHECK("k_vr_hartree");
  // total pseudo density on the grid, XC
  CUW_TRY(cudaMemsetAsync(g.r_grid, 0, sizeof(double2) * nr, h->stream));
  k_vr_scatter<<<gb, kVT, 0, h->stream>>>(g.r_rhog, g.r_plus, g.r_minus, nglh, g.r_grid);
  CUW_LAUNCH_CHECK("k_vr_scatter");
  CUW_RET(grid_fft(h, g.r_grid, +1));
  k_vr_xc<<<rb, kVT, 0, h->stream>>>(g.r_grid, nr, xcpart);
  CUW_LAUNCH_CHECK("k_vr_xc");
  // V(G) = SUPFFT('RTOG', VXC) + VHARTREE
  CUW_RET(grid_fft(h, g.r_grid, -1));
  k_vr_gather<<<gb, kVT, 0, h->stream>>>(g.r_grid, g.r_plus, g.r_minus, nglh, 1.0 / (double)nr, g.r_pot, g.r_vtot);
  CUW_LAUNCH_CHECK("k_vr_gather");
  // forces and VQLM
  k_vr_forces<<<dim3(gb, nat), kVT, 0, h->stream>>>(s, g.r_rhog, g.r_vg, g.r_vtot, g.r_out, fpart);
  CUW_LAUNCH_CHECK("k_vr_forces");
  // V(r)
  CUW_TRY(cudaMemsetAsync(g.r_grid, 0, sizeof(double2) * nr, h->stream));
  k_vr_scatter<<<gb, kVT, 0, h->stream>>>(g.r_vtot, g.r_plus, g.r_minus, nglh, g.r_grid);
  CUW_LAUNCH_CHECK("k_vr_scatter");
  CUW_RET(grid_fft(h, g.r_grid, +1));
  k_vr_store<<<rb, kVT, 0, h->stream>>>(g.r_grid, g.v, edc ? rho_dev : nullptr, nr, dpart);
  CUW_LAUNCH_CHECK("k_vr_store");
  k_vr_final<<<1, 256, 0, h->stream>>>(ehpart, gb, xcpart, rb, edc ? dpart : nullptr, edc ? rb : 0, fpart, gb, nat,
                                        h->lmrxx,
                                        h->gweight, (double)nr, g.r_out, eout, g.fpot, g.vqlm);
  CUW_LAUNCH_CHECK("k_vr_final");
  return CUW_OK;
}

int vofrho_run(Handle* h, const double* rho_dev) { return vofrho_enqueue(h, rho_dev, h->g.scal + 5, true); }

}  // namespace cuw

using namespace cuw;

#define H(hp) Handle* h = reinterpret_cast<Handle*>(hp)

extern "C" int cuwaves_set_rhoset(cuw_handle* hp, int nglh, const int* igvec, const double* gvec, const double* g2,
                                  int lmrxx, const int* lmrx, const double* ylm, const double* g0, const double* v0,
                                  const double* pscore, const double* vbar) {
  if (!hp) return CUW_ERR_ARG;
  H(hp);
  if (!h->have_gset) return h->fail(CUW_ERR_STATE, "G set not loaded");
  if (nglh <= 0 || lmrxx <= 0 || lmrxx > kLmMax || !igvec || !gvec || !g2 || !lmrx || !ylm || !g0 || !v0 ||
      !pscore || !vbar)
    return h->fail(CUW_ERR_ARG, "density set: bad arguments (LMRXX at most 25)");
  const int nsp = h->d.nsp, nat = h->d.nat;
  for (int s = 0; s < nsp; ++s)
    if (lmrx[s] < 1 || lmrx[s] > lmrxx) return h->fail(CUW_ERR_ARG, "density set: LMRX out of range");
  const int n[3] = {h->d.nr1, h->d.nr2, h->d.nr3};
  std::vector<int> plus(nglh), minus(nglh);
  int ngamma = -1;
  for (int ig = 0; ig < nglh; ++ig) {
    int p[3], m[3];
    for (int k = 0; k < 3; ++k) {
      const int i = igvec[3 * ig + k];
      if (2 * std::abs(i) >= n[k]) return h->fail(CUW_ERR_ARG, "density G vector outside the FFT grid");
      p[k] = ((i % n[k]) + n[k]) % n[k];
      m[k] = ((-i % n[k]) + n[k]) % n[k];
    }
    plus[ig] = p[0] + n[0] * (p[1] + n[1] * p[2]);
    minus[ig] = m[0] + n[0] * (m[1] + n[1] * m[2]);
    if (igvec[3 * ig] == 0 && igvec[3 * ig + 1] == 0 && igvec[3 * ig + 2] == 0) ngamma = ig;
  }
  h->touch();
  Device& g = h->g;
  void* old[] = {g.r_plus, g.r_minus, g.r_gx, g.r_gy, g.r_gz, g.r_g2, g.r_ylm, g.r_g0, g.r_v0, g.r_pscore, g.r_vbar,
                 g.r_lmrx, g.qlm, g.r_rhog, g.r_vg, g.r_pot, g.r_vtot, g.r_grid, g.r_part, g.fpot, g.vqlm, g.r_out};
  for (void* p : old)
    if (p) cudaFree(p);
  g.r_plus = g.r_minus = g.r_lmrx = nullptr;
  g.r_gx = g.r_gy = g.r_gz = g.r_g2 = g.r_ylm = g.r_g0 = g.r_v0 = g.r_pscore = g.r_vbar = g.qlm = g.r_part =
      g.fpot = g.vqlm = g.r_out = nullptr;
  g.r_rhog = g.r_vg = g.r_pot = g.r_vtot = g.r_grid = nullptr;
  h->have_rhoset = h->have_qlm = h->scf = false;
  std::vector<double> gx(nglh), gy(nglh), gz(nglh);
  for (int ig = 0; ig < nglh; ++ig) {
    gx[ig] = gvec[3 * ig];
    gy[ig] = gvec[3 * ig + 1];
    gz[ig] = gvec[3 * ig + 2];
  }
  const size_t nt = (size_t)nglh * nsp;
  const int gb = gblocks(nglh), rb = rblocks(h);
  const size_t npart = (size_t)gb + 2 * (size_t)rb + (size_t)gb * std::max(1, nat) * (6 + lmrxx);
  auto put = [&](auto** dst, const auto* src, size_t count) -> cudaError_t {
    using T = std::remove_pointer_t<std::remove_pointer_t<decltype(dst)>>;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(dst), sizeof(T) * std::max<size_t>(count, 1));
    if (e == cudaSuccess && src) e = cudaMemcpy(*dst, src, sizeof(T) * count, cudaMemcpyHostToDevice);
    return e;
  };
  CUW_TRY(put(&g.r_plus, plus.data(), nglh));
  CUW_TRY(put(&g.r_minus, minus.data(), nglh));
  CUW_TRY(put(&g.r_gx, gx.data(), nglh));
  CUW_TRY(put(&g.r_gy, gy.data(), nglh));
  CUW_TRY(put(&g.r_gz, gz.data(), nglh));
  CUW_TRY(put(&g.r_g2, g2, nglh));
  CUW_TRY(put(&g.r_ylm, ylm, (size_t)lmrxx * nglh));
  CUW_TRY(put(&g.r_g0, g0, nt));
  CUW_TRY(put(&g.r_v0, v0, nt));
  CUW_TRY(put(&g.r_pscore, pscore, nt));
  CUW_TRY(put(&g.r_vbar, vbar, nt));
  CUW_TRY(put(&g.r_lmrx, lmrx, nsp));
  CUW_TRY(put(&g.qlm, (const double*)nullptr, (size_t)lmrxx * std::max(1, nat)));
  CUW_TRY(put(&g.r_rhog, (const double2*)nullptr, nglh));
  CUW_TRY(put(&g.r_vg, (const double2*)nullptr, nglh));
  CUW_TRY(put(&g.r_pot, (const double2*)nullptr, nglh));
  CUW_TRY(put(&g.r_vtot, (const double2*)nullptr, nglh));
  CUW_TRY(put(&g.r_grid, (const double2*)nullptr, h->nr));
  CUW_TRY(put(&g.r_part, (const double*)nullptr, npart));
  CUW_TRY(put(&g.fpot, (const double*)nullptr, 3 * (size_t)std::max(1, nat)));
  CUW_TRY(put(&g.vqlm, (const double*)nullptr, (size_t)lmrxx * std::max(1, nat)));
  CUW_TRY(put(&g.r_out, (const double*)nullptr, 4));
  CUW_TRY(cudaMemset(g.fpot, 0, sizeof(double) * 3 * std::max(1, nat)));
  if (!g.rho) {
    CUW_TRY(cudaMalloc(&g.rho, sizeof(double) * h->nr));
    CUW_TRY(cudaMemset(g.rho, 0, sizeof(double) * h->nr));
  }
  h->nglh = nglh;
  h->lmrxx = lmrxx;
  h->ngamma = ngamma;
  h->have_rhoset = true;
  return CUW_OK;
}

extern "C" int cuwaves_set_qlm(cuw_handle* hp, const double* qlm) {
  if (!hp) return CUW_ERR_ARG;
  H(hp);
  if (!h->have_rhoset) return h->fail(CUW_ERR_STATE, "density set not loaded");
  if (!qlm) return h->fail(CUW_ERR_ARG, "null QLM");
  CUW_TRY(cudaMemcpyAsync(h->g.qlm, qlm, sizeof(double) * h->lmrxx * h->d.nat, cudaMemcpyHostToDevice, h->stream));
  CUW_TRY(cudaStreamSynchronize(h->stream));
  h->have_qlm = true;
  return CUW_OK;
}

extern "C" int cuwaves_vofrho(cuw_handle* hp, const double* rho, const double* qlm, double* v, double* e,
                              double* force, double* vqlm) {
  if (!hp) return CUW_ERR_ARG;
  H(hp);
  if (!h->have_rhoset) return h->fail(CUW_ERR_STATE, "density set not loaded");
  if (qlm) CUW_RET(cuwaves_set_qlm(hp, qlm));
  if (!h->have_qlm) return h->fail(CUW_ERR_STATE, "QLM not set");
  h->touch();  // the potential changes outside a step
  Device& g = h->g;
  if (rho) CUW_TRY(cudaMemcpyAsync(g.rho, rho, sizeof(double) * h->nr, cudaMemcpyHostToDevice, h->stream));
  else CUW_RET(fft_density(h, g.psi0, g.rho));
  CUW_RET(vofrho_enqueue(h, g.rho, g.r_out, false));
  h->have_v = true;
  double eh[3];
  CUW_TRY(cudaMemcpyAsync(eh, g.r_out, sizeof(eh), cudaMemcpyDeviceToHost, h->stream));
  if (v) CUW_TRY(cudaMemcpyAsync(v, g.v, sizeof(double) * h->nr, cudaMemcpyDeviceToHost, h->stream));
  if (force) CUW_TRY(cudaMemcpyAsync(force, g.fpot, sizeof(double) * 3 * h->d.nat, cudaMemcpyDeviceToHost, h->stream));
  if (vqlm)
    CUW_TRY(cudaMemcpyAsync(vqlm, g.vqlm, sizeof(double) * h->lmrxx * h->d.nat, cudaMemcpyDeviceToHost, h->stream));
  CUW_TRY(cudaStreamSynchronize(h->stream));
  if (e) std::memcpy(e, eh, sizeof(eh));
  return CUW_OK;
}
