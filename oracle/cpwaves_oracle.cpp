// cpwaves_oracle.cpp -- CPU restatement of the CP-PAW wavefunction hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle and the timed CPU
// baseline.  Only tests/, __graft_entry__.smoke() and bench.py's CPU legs load
// it; the product library never links or calls it.
//
// Parity status: PARITY UNPINNED against the reference itself.  The reference
// (Fortran 90 + FFTW3 + BLAS/LAPACK + MPI) cannot be compiled in this image (no
// Fortran compiler, no FFTW/LAPACK), and its own tests hold no golden vectors
// for this path.  What is pinned: the MSLNG random-number known answer
// (seed 1043618065 after 10000 draws, src/paw_generalpurpose.f90:2236-2239),
// which fixes WAVES_INITIALIZERANDOM; the FFT is cross-checked against numpy
// and the symmetric eigensolver against scipy in the CPU tests.
//
// Each routine follows the Fortran routine named in its comment line by line
// (file:line relative to the reference project).  Third-party arithmetic at the
// reference's boundary is restated here:
//   FFTW3 fftw_plan_dft_1d (src/paw_library.f90:2635-2728) -> fft1d() below,
//     same sign/scale convention (GTOR: +i, unscaled; RTOG: -i, 1/LEN);
//   BLAS ZGEMM/ZHERK/DGEMM/DSYRK (src/paw_library.f90:2074-2260) -> ZGEMM of
//     an OpenBLAS loaded at run time by orc_use_blas (the build bundled with
//     scipy; the reference's fast build links a BLAS the same way), else plain
//     loops;
//   LAPACK DSYEV (src/paw_library.f90:1555-1620) -> cyclic Jacobi (jacobi_eig),
//     whose eigenpairs agree with DSYEV up to order and sign; the only consumer
//     (WAVES_ORTHO_X) is invariant under both.
//
// Single task: every MPE$COMBINE / MPE$TRANSPOSE of the reference is the
// identity here (src/paw_mpelib.f90:267 serial build).

#include "../include/cuwaves.h"

#include <dlfcn.h>

#include <algorithm>
#include <cstdint>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cplx;
static const double PI = 3.14159265358979323846264338327950288;
static const cplx CI(0.0, 1.0);

// (-i)**L evaluated exactly, as the Fortran integer power does
static inline cplx mipow(int l) {
  switch (((l % 4) + 4) % 4) {
    case 0: return cplx(1.0, 0.0);
    case 1: return cplx(0.0, -1.0);
    case 2: return cplx(-1.0, 0.0);
    default: return cplx(0.0, 1.0);
  }
}

// ---------------------------------------------------------------------------
// 1-D mixed-radix DFT (stand-in for FFTW's fftw_plan_dft_1d).
// dir=+1: y_k = sum_j x_j exp(+2 pi i jk/n)   (FFTW_BACKWARD, 'GTOR')
// dir=-1: y_k = sum_j x_j exp(-2 pi i jk/n)   (FFTW_FORWARD,  'RTOG', unscaled)
// Iterative self-sorting (Stockham) form over the factors of n: stage s of
// radix R, after the stages whose radices multiply to Ns, takes for every
// j < n/R the R inputs in[j + r n/R], multiplies input r by
// exp(dir 2 pi i r k / (Ns R)) with k = j mod Ns, does an R-point DFT and
// stores output q at (j / Ns) Ns R + k + q Ns.  Twiddles are tabulated per
// stage when the plan is made; radices 2, 3 and 4 have their own butterflies.
// ---------------------------------------------------------------------------
struct FFTPlan {
  int n = 0;
  int dir = 0;
  std::vector<int> factors;
  std::vector<std::vector<cplx>> tw;  // per stage: (Ns, R-1) twiddles
  std::vector<std::vector<cplx>> rt;  // per stage: R-th roots exp(dir 2 pi i q / R)
};

static void factorize(int n, std::vector<int>& f) {
  f.clear();
  int m = n;
  for (int p : {4, 2, 3, 5, 7, 11, 13}) {
    while (m % p == 0) { f.push_back(p); m /= p; }
  }
  for (int p = 17; m > 1; p += 2) {
    while (m % p == 0) { f.push_back(p); m /= p; }
  }
}

static void plan_init(FFTPlan& P, int n, int dir) {
  P.n = n; P.dir = dir;
  factorize(n, P.factors);
  P.tw.clear();
  P.rt.clear();
  int ns = 1;
  for (int r : P.factors) {
    std::vector<cplx> t((size_t)ns * (r - 1)), w(r);
    for (int k = 0; k < ns; ++k)
      for (int q = 1; q < r; ++q) {
        const double a = 2.0 * PI * (double)q * (double)k / ((double)ns * r);
        t[(size_t)k * (r - 1) + q - 1] = cplx(std::cos(a), dir * std::sin(a));
      }
    for (int q = 0; q < r; ++q) {
      const double a = 2.0 * PI * (double)q / (double)r;
      w[q] = cplx(std::cos(a), dir * std::sin(a));
    }
    P.tw.push_back(std::move(t));
    P.rt.push_back(std::move(w));
    ns *= r;
  }
}

static void fft_stages(const FFTPlan& P, cplx* a, cplx* b) {
  const int n = P.n;
  const double sd = (double)P.dir;
  cplx* in = a;
  cplx* out = b;
  int ns = 1;
  for (size_t st = 0; st < P.factors.size(); ++st) {
    const int r = P.factors[st], nr = n / r;
    const cplx* tw = P.tw[st].data();
    const cplx* rt = P.rt[st].data();
    for (int j = 0; j < nr; ++j) {
      const int k = j % ns;
      const size_t o = (size_t)(j / ns) * ns * r + k;
      cplx v[64];
      v[0] = in[j];
      for (int q = 1; q < r; ++q) v[q] = in[j + (size_t)q * nr] * tw[(size_t)k * (r - 1) + q - 1];
      if (r == 2) {
        out[o] = v[0] + v[1];
        out[o + ns] = v[0] - v[1];
      } else if (r == 4) {
        const cplx s0 = v[0] + v[2], s1 = v[0] - v[2], s2 = v[1] + v[3];
        const cplx d = v[1] - v[3];
        const cplx s3(-sd * d.imag(), sd * d.real());  // dir * i * (v1 - v3)
        out[o] = s0 + s2;
        out[o + ns] = s1 + s3;
        out[o + 2 * (size_t)ns] = s0 - s2;
        out[o + 3 * (size_t)ns] = s1 - s3;
      } else if (r == 3) {
        const cplx s = v[1] + v[2], d = v[1] - v[2];
        const cplx m = v[0] - 0.5 * s;
        const double c = sd * 0.86602540378443864676;  // dir * sin(2 pi / 3)
        const cplx id(-c * d.imag(), c * d.real());
        out[o] = v[0] + s;
        out[o + ns] = m + id;
        out[o + 2 * (size_t)ns] = m - id;
      } else {
        for (int q = 0; q < r; ++q) {
          cplx acc = v[0];
          for (int p = 1; p < r; ++p) acc += v[p] * rt[(size_t)(p * q) % r];
          out[o + (size_t)q * ns] = acc;
        }
      }
    }
    std::swap(in, out);
    ns *= r;
  }
  if (in != a) std::copy(in, in + n, a);
}

static void fft1d(const FFTPlan& P, cplx* data, int stride, std::vector<cplx>& work) {
  int n = P.n;
  work.resize(2 * n);
  cplx* a = work.data();
  cplx* b = work.data() + n;
  for (int j = 0; j < n; ++j) a[j] = data[(size_t)j * stride];
  fft_stages(P, a, b);
  for (int j = 0; j < n; ++j) data[(size_t)j * stride] = a[j];
}

// ---------------------------------------------------------------------------
// Symmetric eigensolver (stand-in for LAPACK DSYEV): cyclic Jacobi.
// a(n,n) column-major symmetric (destroyed); e(n) ascending; u(n,n) columns.
// ---------------------------------------------------------------------------
static void jacobi_eig(int n, std::vector<double>& a, std::vector<double>& e,
                       std::vector<double>& u) {
  u.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) u[i + (size_t)n * i] = 1.0;
  auto A = [&](int i, int j) -> double& { return a[i + (size_t)n * j]; };
  for (int sweep = 0; sweep < 60; ++sweep) {
    int nrot = 0;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        double apq = A(p, q);
        double app = A(p, p), aqq = A(q, q);
        if (std::fabs(apq) <= 1e-17 * std::sqrt(std::fabs(app * aqq)) || apq == 0.0) continue;
        ++nrot;
        double theta = (aqq - app) / (2.0 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) /
                   (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {  // columns p,q
          double akp = A(k, p), akq = A(k, q);
          A(k, p) = c * akp - s * akq;
          A(k, q) = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {  // rows p,q
          double apk = A(p, k), aqk = A(q, k);
          A(p, k) = c * apk - s * aqk;
          A(q, k) = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          double ukp = u[k + (size_t)n * p], ukq = u[k + (size_t)n * q];
          u[k + (size_t)n * p] = c * ukp - s * ukq;
          u[k + (size_t)n * q] = s * ukp + c * ukq;
        }
      }
    if (nrot == 0) break;
  }
  e.resize(n);
  for (int i = 0; i < n; ++i) e[i] = A(i, i);
  // ascending order like DSYEV
  std::vector<int> idx(n);
  for (int i = 0; i < n; ++i) idx[i] = i;
  std::sort(idx.begin(), idx.end(), [&](int x, int y) { return e[x] < e[y]; });
  std::vector<double> e2(n), u2((size_t)n * n);
  for (int i = 0; i < n; ++i) {
    e2[i] = e[idx[i]];
    for (int k = 0; k < n; ++k) u2[k + (size_t)n * i] = u[k + (size_t)n * idx[i]];
  }
  e.swap(e2);
  u.swap(u2);
}

// ---------------------------------------------------------------------------
// Oracle state: one WVSET + GSET + MAP (src/paw_waves1.f90:142-193).
// ---------------------------------------------------------------------------
struct orc_handle {
  cuw_dims d{};
  std::vector<int> isp;          // 0-based species of each atom
  std::vector<int> lmnx;         // per species
  std::vector<int> ibpro;        // per species: first bare projector (0-based)
  int npro = 0, nbarepro = 0, lmnxx = 0, lnxx = 0;
  // projector decomposition: per IPRO -> (iat, ln, lm, l)
  std::vector<int> p_iat, p_ln, p_lm, p_l, p_ipro0;  // p_ipro0[iat] first IPRO
  // g-set
  std::vector<int> igvec, minusg;       // minusg 0-based
  std::vector<double> gvec, g2, pro, ylm, mpsi, bucket;
  std::vector<double> gbas;             // 3x3 col-major (reconstructed)
  bool tbucket = false, have_gset = false;
  double gweight = 0.0;
  // FFT stripes (PLANEWAVE$INITIALIZE for one task)
  int nstripe = 0;
  std::vector<int> igtostripe;          // 0-based position in stripe array
  std::vector<int> istripetoyz;         // 1-based I23 = IR2+NR2*(IR3-1)
  FFTPlan p1g, p1r, p2g, p2r, p3g, p3r;
  // potential, one-centre matrices
  std::vector<double> v;
  std::vector<cplx> dh;                 // (lmnxx,lmnxx,nat)
  std::vector<double> dover;            // (lnxx,lnxx,nsp)
  bool have_v = false, have_dh = false, have_do = false;
  // atoms, occupations, dynamics
  std::vector<double> r0, rp, rm;
  std::vector<double> occ;
  double delt = 0.0, annee = 0.0;
  // state
  std::vector<cplx> psi0, psim, hpsi, opsi, proj, rlam0, rlamm;
  bool have_hpsi = false, have_rlamm = false;
  double waveekin1 = 0.0, waveekin2 = 0.0;
  // density G set of the potential (PLANEWAVE 'DENSITY' at the Gamma point:
  // one G of each +-G pair, the NGLH vectors of PLANEWAVE$SUPFFT) with the
  // tables of POTENTIAL_UPDATE (src/paw_potential.f90:250-320)
  int nglh = 0, lmrxx = 0, ngamma = -1;
  std::vector<int> rigvec, rplus, rminus, lmrx;  // grid offsets of +G and -G
  std::vector<double> rgvec, rg2, rylm, rg0, rv0, rpscore, rvbar;
  bool have_rhoset = false;
  std::vector<double> qlm;    // (LMRXX, NAT) multipole moments of the one-centre densities
  bool scf = false;           // cp_step forms V(r) from the density of PSI0 first
  bool safeortho = true, swapstates = false;  // TSAFEORTHO, TSWAPSTATES (waves1:221-222)
  mutable std::vector<cplx> protab;  // work table PRO(G, IPRO) of the ZGEMM path (kept to reuse its pages)
  // cell friction of WAVES$PROPAGATE with TSTRESS (waves1:6524-6543):
  // FRICMAT = CELL 'PSIANNEMAT' (3,3), EMASS, EMASSCG2, GSET%DBUCKET
  bool tstress = false;
  double fricmat[9] = {0};
  double emass = 0.0, emasscg2 = 0.0;
  std::vector<double> dbucket;
  std::string err;
  int nthreads = 0;
};

static int fail(orc_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

#define OCHECK(cond, code, msg) \
  do { if (!(cond)) return fail(h, code, msg); } while (0)

static inline size_t PS(const orc_handle* h, int ig, int ib) {  // PSI(ig,1,ib)
  return (size_t)ig + (size_t)h->d.ngl * ib;
}
static inline size_t PJ(const orc_handle* h, int ib, int ipro) {  // PROJ(1,ib,ipro)
  return (size_t)ib + (size_t)h->d.nbh * ipro;
}

// ZGEMM of the BLAS that LIB$SCALARPRODUCTC8 and LIB$ADDPRODUCTC8 call
// (src/paw_library.f90:2088-2141), through the CBLAS interface of a library
// opened by orc_use_blas; null: the plain loops below.
typedef void (*cblas_zgemm_t)(int order, int ta, int tb, int m, int n, int k, const void* alpha, const void* a,
                              int lda, const void* b, int ldb, const void* beta, void* c, int ldc);
typedef void (*cblas_dgemm_t)(int order, int ta, int tb, int m, int n, int k, double alpha, const double* a, int lda,
                              const double* b, int ldb, double beta, double* c, int ldc);
typedef void (*blas_threads_t)(int);
static cblas_zgemm_t g_zgemm = nullptr;
static cblas_dgemm_t g_dgemm = nullptr;
static blas_threads_t g_blas_threads = nullptr;
static void zgemm(char ta, char tb, int m, int n, int k, cplx alpha, const cplx* a, int lda, const cplx* b, int ldb,
                  cplx beta, cplx* c, int ldc) {
  auto op = [](char t) { return t == 'N' ? 111 : (t == 'T' ? 112 : 113); };  // CblasNoTrans/Trans/ConjTrans
  g_zgemm(102 /* CblasColMajor */, op(ta), op(tb), m, n, k, &alpha, a, lda, b, ldb, &beta, c, ldc);
}

extern "C" {

int orc_set_threads(orc_handle* h, int n) {
  h->nthreads = n;
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#endif
  if (n > 0 && g_blas_threads) g_blas_threads(n);
  return CUW_OK;
}

// Opens a BLAS with a CBLAS ZGEMM (symbols cblas_zgemm or, in scipy's bundled
// OpenBLAS, scipy_cblas_zgemm); 0 when it is in use, else the loops stay.
int orc_use_blas(const char* path) {
  if (!path) {
    g_zgemm = nullptr;
    g_dgemm = nullptr;
    return CUW_OK;
  }
  void* lib = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!lib) return CUW_ERR_ARG;
  void* f = dlsym(lib, "scipy_cblas_zgemm");
  if (!f) f = dlsym(lib, "cblas_zgemm");
  void* t = dlsym(lib, "scipy_openblas_set_num_threads");
  if (!t) t = dlsym(lib, "openblas_set_num_threads");
  void* d = dlsym(lib, "scipy_cblas_dgemm");
  if (!d) d = dlsym(lib, "cblas_dgemm");
  if (!f) return CUW_ERR_ARG;
  g_zgemm = reinterpret_cast<cblas_zgemm_t>(f);
  g_dgemm = reinterpret_cast<cblas_dgemm_t>(d);
  g_blas_threads = reinterpret_cast<blas_threads_t>(t);
  return CUW_OK;
}
int orc_blas_in_use(void) { return g_zgemm ? 1 : 0; }

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

int orc_create(const cuw_dims* dims, orc_handle** out) {
  *out = nullptr;
  orc_handle* h = new orc_handle();
  h->d = *dims;
  const cuw_dims& d = h->d;
  if (d.ngl <= 0 || d.nb <= 0 || d.nat < 0 || d.nsp <= 0 || d.nsp > CUW_MAXSP ||
      d.ndim != 1 || d.nr1 <= 0 || d.nr2 <= 0 || d.nr3 <= 0) {
    delete h;
    return CUW_ERR_ARG;
  }
  if (d.tinv && d.nbh != (d.nb + 1) / 2) { delete h; return CUW_ERR_ARG; }
  if (!d.tinv && d.nbh != d.nb) { delete h; return CUW_ERR_ARG; }
  if (!d.tinv || (d.nb % 2)) { delete h; return CUW_ERR_UNSUPPORTED; }
  h->isp.resize(d.nat);
  for (int i = 0; i < d.nat; ++i) h->isp[i] = dims->isp[i] - 1;
  h->d.isp = nullptr;
  h->lmnx.resize(d.nsp);
  h->ibpro.resize(d.nsp);
  int nbare = 0;
  for (int s = 0; s < d.nsp; ++s) {
    int n = 0;
    h->lnxx = std::max(h->lnxx, d.lnx[s]);
    for (int ln = 0; ln < d.lnx[s]; ++ln) n += 2 * d.lox[s][ln] + 1;
    h->lmnx[s] = n;
    h->lmnxx = std::max(h->lmnxx, n);
    h->ibpro[s] = nbare;
    nbare += d.lnx[s];
  }
  h->nbarepro = nbare;
  h->p_ipro0.resize(d.nat);
  for (int a = 0; a < d.nat; ++a) {
    int s = h->isp[a];
    h->p_ipro0[a] = h->npro;
    for (int ln = 0; ln < d.lnx[s]; ++ln) {
      int l = d.lox[s][ln];
      for (int m = 0; m < 2 * l + 1; ++m) {
        h->p_iat.push_back(a);
        h->p_ln.push_back(ln);
        h->p_lm.push_back(l * l + m);
        h->p_l.push_back(l);
      }
    }
    h->npro += h->lmnx[s];
  }
  size_t nps = (size_t)d.ngl * d.nbh;
  h->psi0.assign(nps, 0.0);
  h->psim.assign(nps, 0.0);
  h->hpsi.assign(nps, 0.0);
  h->opsi.assign(nps, 0.0);
  h->proj.assign((size_t)d.nbh * h->npro, 0.0);
  h->rlam0.assign((size_t)d.nb * d.nb, 0.0);  // waves1:1402-1403
  h->rlamm.assign((size_t)d.nb * d.nb, 0.0);
  h->occ.assign(d.nb, 0.0);
  h->r0.assign(3 * d.nat, 0.0);
  h->rp.assign(3 * d.nat, 0.0);
  h->rm.assign(3 * d.nat, 0.0);
  plan_init(h->p1g, d.nr1, +1); plan_init(h->p1r, d.nr1, -1);
  plan_init(h->p2g, d.nr2, +1); plan_init(h->p2r, d.nr2, -1);
  plan_init(h->p3g, d.nr3, +1); plan_init(h->p3r, d.nr3, -1);
  *out = h;
  return CUW_OK;
}

int orc_destroy(orc_handle* h) { delete h; return CUW_OK; }

int orc_last_error(const orc_handle* h, char* buf, int len) {
  if (!buf || len <= 0) return CUW_ERR_ARG;
  std::snprintf(buf, (size_t)len, "%s", h ? h->err.c_str() : "null handle");
  return CUW_OK;
}

int orc_npro(const orc_handle* h) { return h->npro; }

// PLANEWAVE$INITIALIZE stripe maps for one task (src/paw_fft.f90:960-1068)
static void build_stripes(orc_handle* h) {
  const int nr1 = h->d.nr1, nr2 = h->d.nr2, nr3 = h->d.nr3, ngl = h->d.ngl;
  std::vector<int> task(nr2 * nr3, 0);  // ITASKOFYZ(I2,I3) col-major
  for (int ig = 0; ig < ngl; ++ig) {
    int i2 = ((h->igvec[3 * ig + 1] % nr2) + nr2) % nr2;
    int i3 = ((h->igvec[3 * ig + 2] % nr3) + nr3) % nr3;
    task[i2 + nr2 * i3] = 1;
  }
  // ISTRIPE numbering: DO I2, DO I3 (I3 innermost)  (fft:1043-1068)
  std::vector<int> stripeofyz(nr2 * nr3, 0);
  h->istripetoyz.clear();
  int ns = 0;
  for (int i2 = 0; i2 < nr2; ++i2)
    for (int i3 = 0; i3 < nr3; ++i3)
      if (task[i2 + nr2 * i3]) {
        ++ns;
        stripeofyz[i2 + nr2 * i3] = ns;
        h->istripetoyz.push_back((i2 + 1) + nr2 * i3);
      }
  h->nstripe = ns;
  h->igtostripe.resize(ngl);
  for (int ig = 0; ig < ngl; ++ig) {
    int i1 = ((h->igvec[3 * ig + 0] % nr1) + nr1) % nr1;
    int i2 = ((h->igvec[3 * ig + 1] % nr2) + nr2) % nr2;
    int i3 = ((h->igvec[3 * ig + 2] % nr3) + nr3) % nr3;
    h->igtostripe[ig] = i1 + nr1 * (stripeofyz[i2 + nr2 * i3] - 1);  // 0-based
  }
}

int orc_set_gset(orc_handle* h, const int* igvec, const int* minusg, const double* gbas,
                 const double* gvec, const double* g2, const double* pro, const double* ylm,
                 const double* mpsi, const double* bucket, double gweight) {
  const int ngl = h->d.ngl;
  h->igvec.assign(igvec, igvec + 3 * (size_t)ngl);
  h->minusg.resize(ngl);
  for (int i = 0; i < ngl; ++i) {
    int m = minusg[i] - 1;
    OCHECK(m >= 0 && m < ngl, CUW_ERR_ARG, "minusg out of range");
    h->minusg[i] = m;
  }
  h->gbas.assign(gbas, gbas + 9);
  h->gvec.assign(gvec, gvec + 3 * (size_t)ngl);
  h->g2.assign(g2, g2 + ngl);
  h->pro.assign(pro, pro + (size_t)ngl * h->nbarepro);
  h->ylm.assign(ylm, ylm + (size_t)ngl * h->d.lmx);
  h->mpsi.assign(mpsi, mpsi + ngl);
  h->tbucket = (bucket != nullptr);
  if (bucket) h->bucket.assign(bucket, bucket + ngl);
  else h->bucket.assign(ngl, 0.0);
  h->gweight = gweight;
  build_stripes(h);
  h->have_gset = true;
  return CUW_OK;
}

int orc_set_potential(orc_handle* h, const double* v) {
  h->v.assign(v, v + (size_t)h->d.nr1 * h->d.nr2 * h->d.nr3);
  h->have_v = true;
  return CUW_OK;
}

int orc_set_dh(orc_handle* h, int lmnxx, const double* dh) {
  OCHECK(lmnxx >= h->lmnxx, CUW_ERR_ARG, "lmnxx too small");
  h->dh.assign((size_t)h->lmnxx * h->lmnxx * h->d.nat, 0.0);
  for (int a = 0; a < h->d.nat; ++a)
    for (int j = 0; j < h->lmnxx; ++j)
      for (int i = 0; i < h->lmnxx; ++i) {
        size_t src = 2 * ((size_t)i + (size_t)lmnxx * (j + (size_t)lmnxx * a));
        h->dh[i + (size_t)h->lmnxx * (j + (size_t)h->lmnxx * a)] = cplx(dh[src], dh[src + 1]);
      }
  h->have_dh = true;
  return CUW_OK;
}

int orc_set_do(orc_handle* h, int lnxx, const double* dover) {
  OCHECK(lnxx >= h->lnxx, CUW_ERR_ARG, "lnxx too small");
  h->dover.assign((size_t)h->lnxx * h->lnxx * h->d.nsp, 0.0);
  for (int s = 0; s < h->d.nsp; ++s)
    for (int j = 0; j < h->lnxx; ++j)
      for (int i = 0; i < h->lnxx; ++i)
        h->dover[i + (size_t)h->lnxx * (j + (size_t)h->lnxx * s)] =
            dover[i + (size_t)lnxx * (j + (size_t)lnxx * s)];
  h->have_do = true;
  return CUW_OK;
}

int orc_set_atoms(orc_handle* h, const double* r0, const double* rp) {
  if (r0) h->r0.assign(r0, r0 + 3 * h->d.nat);
  if (rp) h->rp.assign(rp, rp + 3 * h->d.nat);
  return CUW_OK;
}

int orc_reset_atoms(orc_handle* h, const double* r0) {
  h->r0.assign(r0, r0 + 3 * h->d.nat);
  h->rm = h->r0;
  h->rp = h->r0;
  return CUW_OK;
}

int orc_set_occ(orc_handle* h, const double* occ) {
  h->occ.assign(occ, occ + h->d.nb);
  return CUW_OK;
}

int orc_set_dynamics(orc_handle* h, double delt, double annee) {
  h->delt = delt;
  h->annee = annee;
  return CUW_OK;
}

static std::vector<cplx>* which_psi(orc_handle* h, int which) {
  switch (which) {
    case CUW_PSI0: return &h->psi0;
    case CUW_PSIM: return &h->psim;
    case CUW_HPSI: return &h->hpsi;
    case CUW_OPSI: return &h->opsi;
  }
  return nullptr;
}

int orc_upload_psi(orc_handle* h, int which, const double* psi) {
  auto* p = which_psi(h, which);
  OCHECK(p, CUW_ERR_ARG, "bad which");
  std::memcpy((void*)p->data(), psi, p->size() * sizeof(cplx));
  return CUW_OK;
}

int orc_download_psi(orc_handle* h, int which, double* psi) {
  auto* p = which_psi(h, which);
  OCHECK(p, CUW_ERR_ARG, "bad which");
  std::memcpy(psi, p->data(), p->size() * sizeof(cplx));
  return CUW_OK;
}

int orc_get_proj(orc_handle* h, double* proj) {
  std::memcpy(proj, h->proj.data(), h->proj.size() * sizeof(cplx));
  return CUW_OK;
}
int orc_set_proj(orc_handle* h, const double* proj) {
  std::memcpy((void*)h->proj.data(), proj, h->proj.size() * sizeof(cplx));
  return CUW_OK;
}
int orc_get_rlam0(orc_handle* h, double* r) {
  std::memcpy(r, h->rlam0.data(), h->rlam0.size() * sizeof(cplx));
  return CUW_OK;
}
int orc_set_rlam0(orc_handle* h, const double* r) {
  std::memcpy((void*)h->rlam0.data(), r, h->rlam0.size() * sizeof(cplx));
  return CUW_OK;
}

// ---------------------------------------------------------------------------
// PLANEWAVE_FFTGTOR (src/paw_fft.f90:2012-2177), one task.
// fofg(NGL) -> fofr(NR1*NR2*NR3), x fastest.
// ---------------------------------------------------------------------------
static void fft_gtor(const orc_handle* h, const cplx* fofg, cplx* fofr) {
  const int nr1 = h->d.nr1, nr2 = h->d.nr2, nr3 = h->d.nr3;
  const int ns = h->nstripe;
  // work arrays kept per thread (no fresh pages on every transform)
  static thread_local std::vector<cplx> work, fofg1, f;
  fofg1.assign((size_t)nr1 * ns, 0.0);
  for (int ig = 0; ig < h->d.ngl; ++ig) fofg1[h->igtostripe[ig]] = fofg[ig];
  for (int s = 0; s < ns; ++s) fft1d(h->p1g, &fofg1[(size_t)nr1 * s], 1, work);
  // distribute onto FOFR(NR2,NR3,NR1L) (fft:2096-2118)
  f.assign((size_t)nr1 * nr2 * nr3, 0.0);
  const int imid = nr3 / 2;
  int nr3end1 = 1, nr3end2 = nr3;
  const size_t stride2 = (size_t)nr2 * nr3;
  for (int s = 0; s < ns; ++s) {
    int i23 = h->istripetoyz[s];
    for (int ir1 = 0; ir1 < nr1; ++ir1) f[(size_t)(i23 - 1) + stride2 * ir1] = fofg1[(size_t)nr1 * s + ir1];
    int ir3 = 1 + (i23 - 1) / nr2;
    if (ir3 <= imid) nr3end1 = std::max(nr3end1, ir3);
    else nr3end2 = std::min(nr3end2, ir3);
  }
  // y-lines on the occupied z ranges (fft:2123-2131)
  for (int ir1 = 0; ir1 < nr1; ++ir1) {
    for (int ir3 = 1; ir3 <= nr3end1; ++ir3)
      fft1d(h->p2g, &f[(size_t)nr2 * (ir3 - 1) + stride2 * ir1], 1, work);
    for (int ir3 = nr3end2; ir3 <= nr3; ++ir3)
      fft1d(h->p2g, &f[(size_t)nr2 * (ir3 - 1) + stride2 * ir1], 1, work);
  }
  // z-lines (stride NR2 in FOFR(NR2,NR3,NR1)); then transpose to x fastest
  for (int ir1 = 0; ir1 < nr1; ++ir1)
    for (int ir2 = 0; ir2 < nr2; ++ir2) fft1d(h->p3g, &f[(size_t)ir2 + stride2 * ir1], nr2, work);
  for (int ir1 = 0; ir1 < nr1; ++ir1)
    for (int ir3 = 0; ir3 < nr3; ++ir3)
      for (int ir2 = 0; ir2 < nr2; ++ir2)
        fofr[(size_t)ir1 + (size_t)nr1 * (ir2 + (size_t)nr2 * ir3)] =
            f[(size_t)ir2 + (size_t)nr2 * ir3 + stride2 * ir1];
}

// PLANEWAVE_FFTRTOG (src/paw_fft.f90:2180-2341), one task.
static void fft_rtog(const orc_handle* h, const cplx* fofr, cplx* fofg) {
  const int nr1 = h->d.nr1, nr2 = h->d.nr2, nr3 = h->d.nr3;
  const int ns = h->nstripe;
  // work arrays kept per thread (no fresh pages on every transform)
  static thread_local std::vector<cplx> work, f1, f2, fofg1;
  // FOFR1(IR3,IR2,IR1) = FOFR(IR1,IR2,IR3); z-lines
  f1.resize((size_t)nr1 * nr2 * nr3);
  for (int ir1 = 0; ir1 < nr1; ++ir1)
    for (int ir2 = 0; ir2 < nr2; ++ir2)
      for (int ir3 = 0; ir3 < nr3; ++ir3)
        f1[(size_t)ir3 + (size_t)nr3 * (ir2 + (size_t)nr2 * ir1)] =
            fofr[(size_t)ir1 + (size_t)nr1 * (ir2 + (size_t)nr2 * ir3)];
  const double sc3 = 1.0 / nr3, sc2 = 1.0 / nr2, sc1 = 1.0 / nr1;
  for (size_t l = 0; l < (size_t)nr2 * nr1; ++l) {
    fft1d(h->p3r, &f1[(size_t)nr3 * l], 1, work);
    for (int k = 0; k < nr3; ++k) f1[(size_t)nr3 * l + k] *= sc3;
  }
  const int imid = nr3 / 2;
  int nr3end1 = 1, nr3end2 = nr3;
  for (int s = 0; s < ns; ++s) {
    int i23 = h->istripetoyz[s];
    int ir3 = 1 + (i23 - 1) / nr2;
    if (ir3 <= imid) nr3end1 = std::max(nr3end1, ir3);
    else nr3end2 = std::min(nr3end2, ir3);
  }
  if (nr3end1 == nr3end2) nr3end2 = nr3end2 + 1;
  // FOFR2(IR2,IR3,IR1) restricted to occupied z (fft:2262-2280)
  f2.assign((size_t)nr1 * nr2 * nr3, 0.0);
  for (int ir1 = 0; ir1 < nr1; ++ir1)
    for (int ir2 = 0; ir2 < nr2; ++ir2) {
      for (int ir3 = 1; ir3 <= nr3end1; ++ir3)
        f2[(size_t)ir2 + (size_t)nr2 * ((ir3 - 1) + (size_t)nr3 * ir1)] =
            f1[(size_t)(ir3 - 1) + (size_t)nr3 * (ir2 + (size_t)nr2 * ir1)];
      for (int ir3 = nr3end2; ir3 <= nr3; ++ir3)
        f2[(size_t)ir2 + (size_t)nr2 * ((ir3 - 1) + (size_t)nr3 * ir1)] =
            f1[(size_t)(ir3 - 1) + (size_t)nr3 * (ir2 + (size_t)nr2 * ir1)];
    }
  for (int ir1 = 0; ir1 < nr1; ++ir1) {
    for (int ir3 = 1; ir3 <= nr3end1; ++ir3) {
      cplx* p = &f2[(size_t)nr2 * ((ir3 - 1) + (size_t)nr3 * ir1)];
      fft1d(h->p2r, p, 1, work);
      for (int k = 0; k < nr2; ++k) p[k] *= sc2;
    }
    for (int ir3 = nr3end2; ir3 <= nr3; ++ir3) {
      cplx* p = &f2[(size_t)nr2 * ((ir3 - 1) + (size_t)nr3 * ir1)];
      fft1d(h->p2r, p, 1, work);
      for (int k = 0; k < nr2; ++k) p[k] *= sc2;
    }
  }
  fofg1.assign((size_t)nr1 * ns, 0.0);
  for (int s = 0; s < ns; ++s) {
    int i23 = h->istripetoyz[s];
    for (int ir1 = 0; ir1 < nr1; ++ir1)
      fofg1[(size_t)nr1 * s + ir1] = f2[(size_t)(i23 - 1) + (size_t)nr2 * nr3 * ir1];
    fft1d(h->p1r, &fofg1[(size_t)nr1 * s], 1, work);
    for (int k = 0; k < nr1; ++k) fofg1[(size_t)nr1 * s + k] *= sc1;
  }
  for (int ig = 0; ig < h->d.ngl; ++ig) fofg[ig] = fofg1[h->igtostripe[ig]];
}

int orc_fft(orc_handle* h, int dir, int nfft, double* fofg, double* fofr) {
  OCHECK(h->have_gset, CUW_ERR_STATE, "gset not set");
  const size_t nr = (size_t)h->d.nr1 * h->d.nr2 * h->d.nr3;
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < nfft; ++i) {
    cplx* g = reinterpret_cast<cplx*>(fofg) + (size_t)h->d.ngl * i;
    cplx* r = reinterpret_cast<cplx*>(fofr) + nr * i;
    if (dir > 0) fft_gtor(h, g, r);
    else fft_rtog(h, r, g);
  }
  return CUW_OK;
}

// PLANEWAVE_STRUCTUREFACTOR (src/paw_fft.f90:1597-1695): EIGR = exp(-i G R)
static void structurefactor(const orc_handle* h, const double* R, cplx* eigr) {
  const int nr[3] = {h->d.nr1, h->d.nr2, h->d.nr3};
  int nrmax = std::max(nr[0], std::max(nr[1], nr[2]));
  std::vector<cplx> w((size_t)(2 * nrmax + 1) * 3);
  auto W = [&](int i, int dir) -> cplx& { return w[(size_t)(i + nrmax) + (size_t)(2 * nrmax + 1) * dir]; };
  for (int dir = 0; dir < 3; ++dir) {
    double gr = h->gbas[0 + 3 * dir] * R[0] + h->gbas[1 + 3 * dir] * R[1] + h->gbas[2 + 3 * dir] * R[2];
    cplx cfacp(std::cos(gr), -std::sin(gr));
    cplx csvarp(1.0, 0.0);  // Gamma: RK=0
    cplx cfacm = std::conj(cfacp), csvarm = csvarp;
    for (int i = 1; i <= nr[dir]; ++i) {
      W(i - 1, dir) = csvarp;
      csvarp *= cfacp;
      W(-i + 1, dir) = csvarm;
      csvarm *= cfacm;
    }
  }
  for (int ig = 0; ig < h->d.ngl; ++ig)
    eigr[ig] = W(h->igvec[3 * ig], 0) * W(h->igvec[3 * ig + 1], 1) * W(h->igvec[3 * ig + 2], 2);
}

// WAVES_EXPANDPRO (src/paw_waves1.f90:6070-6109) for atom iat: PRO(NGL,LMNX)
static void expandpro(const orc_handle* h, int iat, const cplx* eigr, cplx* pro) {
  const int s = h->isp[iat];
  const int ngl = h->d.ngl;
  int lmn = 0;
  for (int ln = 0; ln < h->d.lnx[s]; ++ln) {
    int l = h->d.lox[s][ln];
    int lm = l * l;
    cplx csvar = mipow(l);
    const double* bare = &h->pro[(size_t)ngl * (h->ibpro[s] + ln)];
    for (int im = 0; im < 2 * l + 1; ++im) {
      const double* y = &h->ylm[(size_t)ngl * (lm + im)];
      for (int ig = 0; ig < ngl; ++ig) pro[(size_t)ngl * lmn + ig] = (y[ig] * bare[ig]) * csvar * eigr[ig];
      ++lmn;
    }
  }
}

// WAVES_PROJECTIONS (src/paw_waves1.f90:5746-5905, unblocked branch):
// PROPSI(1,IB,IPRO) = GWEIGHT * sum_G conj(PRO(G,LMN)) PSI(G,IB)
// PRO(G, IPRO) of every atom at positions R (WAVES_EXPANDPRO per atom)
static void expandpro_all(const orc_handle* h, const double* R, std::vector<cplx>& pro) {
  const int ngl = h->d.ngl;
  if (pro.size() != (size_t)ngl * h->npro) pro.resize((size_t)ngl * h->npro);
#pragma omp parallel
  {
    std::vector<cplx> eigr(ngl);
#pragma omp for schedule(dynamic)
    for (int iat = 0; iat < h->d.nat; ++iat) {
      structurefactor(h, R + 3 * iat, eigr.data());
      expandpro(h, iat, eigr.data(), &pro[(size_t)ngl * h->p_ipro0[iat]]);
    }
  }
}

static void projections(const orc_handle* h, const double* R, const cplx* psi, cplx* propsi) {
  const int ngl = h->d.ngl, nbh = h->d.nbh;
  if (g_zgemm && h->npro > 0) {
    // ZGEMM('C','N') of LIB$SCALARPRODUCTC8 over all atoms at once
    std::vector<cplx>& pro = h->protab;
    std::vector<cplx> c((size_t)h->npro * nbh);
    expandpro_all(h, R, pro);
    zgemm('C', 'N', h->npro, nbh, ngl, h->gweight, pro.data(), ngl, psi, ngl, 0.0, c.data(), h->npro);
    for (int ib = 0; ib < nbh; ++ib)
      for (int ip = 0; ip < h->npro; ++ip) propsi[PJ(h, ib, ip)] = c[ip + (size_t)h->npro * ib];
    return;
  }
#pragma omp parallel
  {
    std::vector<cplx> eigr(ngl), pro((size_t)ngl * h->lmnxx);
#pragma omp for schedule(dynamic)
    for (int iat = 0; iat < h->d.nat; ++iat) {
      structurefactor(h, R + 3 * iat, eigr.data());
      expandpro(h, iat, eigr.data(), pro.data());
      const int s = h->isp[iat];
      const int i0 = h->p_ipro0[iat];
      for (int lmn = 0; lmn < h->lmnx[s]; ++lmn)
        for (int ib = 0; ib < nbh; ++ib) {
          cplx acc = 0.0;
          const cplx* p = &pro[(size_t)ngl * lmn];
          const cplx* f = &psi[PS(h, 0, ib)];
          for (int ig = 0; ig < ngl; ++ig) acc += std::conj(p[ig]) * f[ig];
          propsi[PJ(h, ib, i0 + lmn)] = acc * h->gweight;
        }
    }
  }
}

// WAVES_ADDPRO (src/paw_waves1.f90:5908-6067): PSI(G,IB) += sum PRO(G,LMN) PROPSI(1,IB,IPRO)
static void addpro(const orc_handle* h, const double* R, cplx* psi, const cplx* propsi) {
  const int ngl = h->d.ngl, nbh = h->d.nbh;
  if (g_zgemm && h->npro > 0) {
    // ZGEMM('N','T') of LIB$ADDPRODUCTC8: PSI += PRO * PROPSI^T
    std::vector<cplx>& pro = h->protab;
    expandpro_all(h, R, pro);
    zgemm('N', 'T', ngl, nbh, h->npro, 1.0, pro.data(), ngl, propsi, nbh, 1.0, psi, ngl);
    return;
  }
  std::vector<cplx> eigrall((size_t)ngl * h->d.nat);
#pragma omp parallel for
  for (int iat = 0; iat < h->d.nat; ++iat) structurefactor(h, R + 3 * iat, &eigrall[(size_t)ngl * iat]);
  const int BS = 128;
  const int nblk = (ngl + BS - 1) / BS;
#pragma omp parallel
  {
    std::vector<cplx> pro((size_t)BS * h->lmnxx);
#pragma omp for schedule(dynamic)
    for (int blk = 0; blk < nblk; ++blk) {
      int igb = blk * BS, bs = std::min(BS, ngl - igb);
      for (int iat = 0; iat < h->d.nat; ++iat) {
        const int s = h->isp[iat];
        const cplx* eigr = &eigrall[(size_t)ngl * iat + igb];
        int lmn = 0;
        for (int ln = 0; ln < h->d.lnx[s]; ++ln) {
          int l = h->d.lox[s][ln];
          cplx csvar = mipow(l);
          const double* bare = &h->pro[(size_t)ngl * (h->ibpro[s] + ln) + igb];
          for (int im = 0; im < 2 * l + 1; ++im) {
            const double* y = &h->ylm[(size_t)ngl * (l * l + im) + igb];
            for (int i = 0; i < bs; ++i) pro[(size_t)bs * lmn + i] = (y[i] * bare[i]) * csvar * eigr[i];
            ++lmn;
          }
        }
        const int i0 = h->p_ipro0[iat];
        for (int ib = 0; ib < nbh; ++ib) {
          cplx* f = &psi[PS(h, igb, ib)];
          for (int lmn2 = 0; lmn2 < h->lmnx[s]; ++lmn2) {
            cplx c = propsi[PJ(h, ib, i0 + lmn2)];
            const cplx* p = &pro[(size_t)bs * lmn2];
            for (int i = 0; i < bs; ++i) f[i] += p[i] * c;
          }
        }
      }
    }
  }
}

// WAVES_HPROJ (src/paw_waves1.f90:4919-4973), NDIM=1, all atoms
static void hproj_all(const orc_handle* h, const cplx* proj, cplx* hproj) {
  const int nbh = h->d.nbh;
  std::fill(hproj, hproj + (size_t)nbh * h->npro, cplx(0.0));
  for (int iat = 0; iat < h->d.nat; ++iat) {
    const int s = h->isp[iat], lmnx = h->lmnx[s], i0 = h->p_ipro0[iat];
    for (int l1 = 0; l1 < lmnx; ++l1)
      for (int l2 = 0; l2 < lmnx; ++l2) {
        cplx dhv = h->dh[l1 + (size_t)h->lmnxx * (l2 + (size_t)h->lmnxx * iat)];
        for (int ib = 0; ib < nbh; ++ib) hproj[PJ(h, ib, i0 + l1)] += dhv * proj[PJ(h, ib, i0 + l2)];
      }
  }
}

// WAVES_OPROJ (src/paw_waves2.f90:497-544), all atoms
static void oproj_all(const orc_handle* h, const cplx* proj, cplx* oproj) {
  const int nbh = h->d.nbh;
  std::fill(oproj, oproj + (size_t)nbh * h->npro, cplx(0.0));
  for (int iat = 0; iat < h->d.nat; ++iat) {
    const int s = h->isp[iat], i0 = h->p_ipro0[iat];
    int lmn10 = 0;
    for (int ln1 = 0; ln1 < h->d.lnx[s]; ++ln1) {
      int l1 = h->d.lox[s][ln1];
      int lmn20 = 0;
      for (int ln2 = 0; ln2 < h->d.lnx[s]; ++ln2) {
        int l2 = h->d.lox[s][ln2];
        if (l1 == l2) {
          double dover1 = h->dover[ln1 + (size_t)h->lnxx * (ln2 + (size_t)h->lnxx * s)];
          for (int m = 0; m < 2 * l1 + 1; ++m)
            for (int ib = 0; ib < nbh; ++ib)
              oproj[PJ(h, ib, i0 + lmn10 + m)] += dover1 * proj[PJ(h, ib, i0 + lmn20 + m)];
        }
        lmn20 += 2 * l2 + 1;
      }
      lmn10 += 2 * l1 + 1;
    }
  }
}

// WAVES_VPSI (src/paw_waves1.f90:5099-5194), NDIM=1
static void vpsi(const orc_handle* h, const cplx* psi, cplx* hpsi) {
  const int ngl = h->d.ngl, nbh = h->d.nbh;
  const size_t nr = (size_t)h->d.nr1 * h->d.nr2 * h->d.nr3;
#pragma omp parallel
  {
    std::vector<cplx> psir(nr);
#pragma omp for schedule(dynamic)
    for (int ib = 0; ib < nbh; ++ib) {
      fft_gtor(h, &psi[PS(h, 0, ib)], psir.data());
      for (size_t ir = 0; ir < nr; ++ir) psir[ir] = h->v[ir] * psir[ir];
      fft_rtog(h, psir.data(), &hpsi[PS(h, 0, ib)]);
    }
  }
  for (int ib = 0; ib < nbh; ++ib)
    for (int ig = 0; ig < ngl; ++ig) hpsi[PS(h, ig, ib)] += 0.5 * h->g2[ig] * psi[PS(h, ig, ib)];
  if (h->tbucket)
    for (int ib = 0; ib < nbh; ++ib)
      for (int ig = 0; ig < ngl; ++ig) hpsi[PS(h, ig, ib)] += h->bucket[ig] * psi[PS(h, ig, ib)];
}

int orc_projections(orc_handle* h) {
  OCHECK(h->have_gset, CUW_ERR_STATE, "gset not set");
  projections(h, h->r0.data(), h->psi0.data(), h->proj.data());
  return CUW_OK;
}

// WAVES$HPSI (src/paw_waves1.f90:4793-4916)
int orc_hpsi(orc_handle* h) {
  OCHECK(h->have_gset && h->have_v && h->have_dh, CUW_ERR_STATE, "gset/potential/dh not set");
  vpsi(h, h->psi0.data(), h->hpsi.data());
  std::vector<cplx> hproj((size_t)h->d.nbh * h->npro);
  hproj_all(h, h->proj.data(), hproj.data());
  addpro(h, h->r0.data(), h->hpsi.data(), hproj.data());
  h->have_hpsi = true;
  return CUW_OK;
}

int orc_vpsi_only(orc_handle* h) {
  OCHECK(h->have_gset && h->have_v, CUW_ERR_STATE, "gset/potential not set");
  vpsi(h, h->psi0.data(), h->hpsi.data());
  return CUW_OK;
}

// PLANEWAVE$SCALARPRODUCT (src/paw_fft.f90:2344-2422) for NDIM=1, not super:
// ' '/'=': MAT(I1,I2) = GWEIGHT sum_G conj(F1(G,I1)) F2(G,I2)
// '-'    : MAT(I1,I2) = GWEIGHT sum_G F1(G,I1) F2(-G,I2)
static void scalarproduct(const orc_handle* h, char id, int n1, const cplx* f1, int n2,
                          const cplx* f2, cplx* mat) {
  const int ngl = h->d.ngl;
  if (g_zgemm) {
    if (id == '-') {
      // sum_G F1(G) F2(-G): the gathered F2(-G) as the second operand
      std::vector<cplx> f2m((size_t)ngl * n2);
#pragma omp parallel for schedule(static)
      for (int i2 = 0; i2 < n2; ++i2)
        for (int ig = 0; ig < ngl; ++ig) f2m[ig + (size_t)ngl * i2] = f2[h->minusg[ig] + (size_t)ngl * i2];
      zgemm('T', 'N', n1, n2, ngl, h->gweight, f1, ngl, f2m.data(), ngl, 0.0, mat, n1);
    } else {
      zgemm('C', 'N', n1, n2, ngl, h->gweight, f1, ngl, f2, ngl, 0.0, mat, n1);
    }
    return;
  }
#pragma omp parallel for collapse(2) schedule(static)
  for (int i2 = 0; i2 < n2; ++i2)
    for (int i1 = 0; i1 < n1; ++i1) {
      cplx acc = 0.0;
      const cplx* a = f1 + (size_t)ngl * i1;
      const cplx* b = f2 + (size_t)ngl * i2;
      if (id == '-') {
        // SCALARPRODUCTC8(F1, F2M) with F2M(G)=conj(F2(-G)), then conj
        for (int ig = 0; ig < ngl; ++ig) acc += std::conj(a[ig]) * std::conj(b[h->minusg[ig]]);
        acc = std::conj(acc);
      } else {
        for (int ig = 0; ig < ngl; ++ig) acc += std::conj(a[ig]) * b[ig];
      }
      mat[i1 + (size_t)n1 * i2] = acc * h->gweight;
    }
}

// WAVES_OVERLAP (src/paw_waves2.f90:761-853), TINV branch. MAT(NB,NB) complex.
static void overlap(const orc_handle* h, bool tid, const cplx* psi1, const cplx* psi2, cplx* mat) {
  const int nbh = h->d.nbh, nb = h->d.nb;
  std::vector<cplx> tmat((size_t)nbh * nbh);
  scalarproduct(h, tid ? '=' : ' ', nbh, psi1, nbh, psi2, tmat.data());
  for (int ibh1 = 0; ibh1 < nbh; ++ibh1) {
    int ib1a = 2 * ibh1, ib1b = std::min(2 * ibh1 + 1, nb - 1);
    for (int ibh2 = 0; ibh2 < nbh; ++ibh2) {
      int ib2a = 2 * ibh2, ib2b = std::min(2 * ibh2 + 1, nb - 1);
      double re = 0.5 * tmat[ibh1 + (size_t)nbh * ibh2].real();
      double im = 0.5 * tmat[ibh1 + (size_t)nbh * ibh2].imag();
      double m2[2][2] = {{re, im}, {-im, re}};
      for (int i = ib1a; i <= ib1b; ++i)
        for (int j = ib2a; j <= ib2b; ++j) mat[i + (size_t)nb * j] = m2[i - ib1a][j - ib2a];
    }
  }
  scalarproduct(h, '-', nbh, psi1, nbh, psi2, tmat.data());
  for (int ibh1 = 0; ibh1 < nbh; ++ibh1) {
    int ib1a = 2 * ibh1, ib1b = std::min(2 * ibh1 + 1, nb - 1);
    for (int ibh2 = 0; ibh2 < nbh; ++ibh2) {
      int ib2a = 2 * ibh2, ib2b = std::min(2 * ibh2 + 1, nb - 1);
      double re = 0.5 * tmat[ibh1 + (size_t)nbh * ibh2].real();
      double im = 0.5 * tmat[ibh1 + (size_t)nbh * ibh2].imag();
      double m2[2][2] = {{re, im}, {im, -re}};
      for (int i = ib1a; i <= ib1b; ++i)
        for (int j = ib2a; j <= ib2b; ++j) mat[i + (size_t)nb * j] += m2[i - ib1a][j - ib2a];
    }
  }
}

// WAVES_1COVERLAP (src/paw_waves2.f90:856-1022), one task, TINV
static void onecoverlap(const orc_handle* h, const cplx* proj1, const cplx* proj2, cplx* mat) {
  const int nbh = h->d.nbh, nb = h->d.nb, npro = h->npro;
  std::vector<cplx> proj2a((size_t)nbh * npro, 0.0);
  // PROJ2A = DO*PROJ2 (same as WAVES_OPROJ)
  oproj_all(h, proj2, proj2a.data());
  std::vector<cplx> cmat1((size_t)nbh * nbh, 0.0), cmat2((size_t)nbh * nbh, 0.0);
  for (int ibh1 = 0; ibh1 < nbh; ++ibh1)
    for (int ibh2 = 0; ibh2 < nbh; ++ibh2) {
      cplx c1 = 0.0, c2 = 0.0;
      for (int ip = 0; ip < npro; ++ip) {
        cplx a = proj1[PJ(h, ibh1, ip)], b = proj2a[PJ(h, ibh2, ip)];
        c1 += std::conj(a) * b;
        c2 += a * b;
      }
      cmat1[ibh1 + (size_t)nbh * ibh2] = c1;
      cmat2[ibh1 + (size_t)nbh * ibh2] = c2;
    }
  std::fill(mat, mat + (size_t)nb * nb, cplx(0.0));
  for (int ibh2 = 0; ibh2 < nbh; ++ibh2) {
    int ib2 = 2 * ibh2;
    for (int ibh1 = 0; ibh1 < nbh; ++ibh1) {
      int ib1 = 2 * ibh1;
      cplx cs1 = 0.5 * (cmat1[ibh1 + (size_t)nbh * ibh2] + cmat2[ibh1 + (size_t)nbh * ibh2]);
      cplx cs2 = 0.5 * (cmat1[ibh1 + (size_t)nbh * ibh2] - cmat2[ibh1 + (size_t)nbh * ibh2]);
      mat[ib1 + (size_t)nb * ib2] = cs1.real();
      mat[ib1 + (size_t)nb * (ib2 + 1)] = cs1.imag();
      mat[(ib1 + 1) + (size_t)nb * ib2] = -cs2.imag();
      mat[(ib1 + 1) + (size_t)nb * (ib2 + 1)] = cs2.real();
    }
  }
}

// plain real matrix helpers (column-major n x n)
// LIB$MATMULR8 / LIB$SCALARPRODUCTR8 / LIB$DYADSUMR8 (DGEMM in the reference,
// src/paw_library.f90:2161-2218): the loaded BLAS, else loops
static bool dgemm_nn(char ta, char tb, int n, const double* a, const double* b, double* c) {
  if (!g_dgemm) return false;
  g_dgemm(102, ta == 'T' ? 112 : 111, tb == 'T' ? 112 : 111, n, n, n, 1.0, a, n, b, n, 0.0, c, n);
  return true;
}
static void matmul(int n, const double* a, const double* b, double* c) {  // C = A B
  if (dgemm_nn('N', 'N', n, a, b, c)) return;
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      double s = 0;
      for (int k = 0; k < n; ++k) s += a[i + (size_t)n * k] * b[k + (size_t)n * j];
      c[i + (size_t)n * j] = s;
    }
}
static void matmul_tn(int n, const double* a, const double* b, double* c) {  // C = A^T B
  if (dgemm_nn('T', 'N', n, a, b, c)) return;
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      double s = 0;
      for (int k = 0; k < n; ++k) s += a[k + (size_t)n * i] * b[k + (size_t)n * j];
      c[i + (size_t)n * j] = s;
    }
}
static void matmul_nt(int n, const double* a, const double* b, double* c) {  // C = A B^T
  if (dgemm_nn('N', 'T', n, a, b, c)) return;
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      double s = 0;
      for (int k = 0; k < n; ++k) s += a[i + (size_t)n * k] * b[j + (size_t)n * k];
      c[i + (size_t)n * j] = s;
    }
}

// WAVES_ORTHO_X (src/paw_waves2.f90:1844-2022). Returns iterations or <0 on error.
static int ortho_x(int nb, const double* occ, const double* chichi, const double* psipsi,
                   const double* chipsi, double* lambda, int maxit, double eps, int* status) {
  const double DSMALL = 1e-12;
  const size_t nn = (size_t)nb * nb;
  std::vector<double> gamn(nn), haux(nn), eig, u;
  // LIB$DIAGR8 -> LIB_LAPACK_DSYEV: diagonalise 0.5*(H+H^T)
  std::vector<double> sym(nn);
  for (int j = 0; j < nb; ++j)
    for (int i = 0; i < nb; ++i) sym[i + (size_t)nb * j] = 0.5 * (chipsi[i + (size_t)nb * j] + chipsi[j + (size_t)nb * i]);
  jacobi_eig(nb, sym, eig, u);
  *status = CUW_ERR_NOT_CONVERGED;
  for (int iter = 1; iter <= maxit; ++iter) {
    matmul(nb, chichi, lambda, haux.data());
    for (size_t k = 0; k < nn; ++k) haux[k] += 2.0 * chipsi[k];
    matmul_tn(nb, lambda, haux.data(), gamn.data());
    for (int i = 0; i < nb; ++i) {
      for (int j = i; j < nb; ++j) {
        double svar = 0.5 * (gamn[i + (size_t)nb * j] + gamn[j + (size_t)nb * i]) + psipsi[i + (size_t)nb * j];
        gamn[j + (size_t)nb * i] = svar;
        gamn[i + (size_t)nb * j] = svar;
      }
      gamn[i + (size_t)nb * i] -= 1.0;
    }
    double digam = 0.0;
    for (size_t k = 0; k < nn; ++k) digam = std::max(digam, std::fabs(gamn[k]));
    if (digam < eps) { *status = CUW_OK; return iter; }
    if (!(digam <= 1e200)) { *status = CUW_ERR_DIVERGED; return iter; }
    matmul_tn(nb, u.data(), gamn.data(), haux.data());
    matmul(nb, haux.data(), u.data(), gamn.data());
    for (int i = 0; i < nb; ++i)
      for (int j = 0; j < nb; ++j) gamn[i + (size_t)nb * j] /= (eig[i] + eig[j]);
    matmul(nb, u.data(), gamn.data(), haux.data());
    matmul_nt(nb, haux.data(), u.data(), gamn.data());
    for (int i = 0; i < nb; ++i) {
      double occi = occ[i] + DSMALL;
      for (int j = 0; j < nb; ++j) {
        double occj = occ[j] + DSMALL;
        double svar = 2.0 * occi / (occi + occj);
        lambda[i + (size_t)nb * j] -= svar * gamn[i + (size_t)nb * j];
      }
    }
    for (int i = 0; i < nb; ++i)
      for (int j = 0; j < nb; ++j)
        if (occ[i] < occ[j])
          lambda[i + (size_t)nb * j] = lambda[j + (size_t)nb * i] * (occ[i] + DSMALL) / (occ[j] + DSMALL);
  }
  return maxit;
}

// lambda1/lambda2 of WAVES_ADDOPSI (src/paw_waves2.f90:583-595)
static void lambda12(int nb, int nbh, const cplx* lambda, std::vector<cplx>& l1, std::vector<cplx>& l2) {
  l1.assign((size_t)nbh * nbh, 0.0);
  l2.assign((size_t)nbh * nbh, 0.0);
  for (int ibh1 = 0; ibh1 < nbh; ++ibh1) {
    int ib1a = 2 * ibh1, ib1b = 2 * ibh1 + 1;
    for (int ibh2 = 0; ibh2 < nbh; ++ibh2) {
      int ib2a = 2 * ibh2, ib2b = 2 * ibh2 + 1;
      cplx c1 = lambda[ib1a + (size_t)nb * ib2a] + CI * lambda[ib1a + (size_t)nb * ib2b];
      cplx c2 = CI * lambda[ib1b + (size_t)nb * ib2a] - lambda[ib1b + (size_t)nb * ib2b];
      l1[ibh1 + (size_t)nbh * ibh2] = 0.5 * (c1 - c2);
      l2[ibh1 + (size_t)nbh * ibh2] = 0.5 * (c1 + c2);
    }
  }
}

// WAVES_ADDOPSI (src/paw_waves2.f90:547-615), TINV: PSIBAR += OPSI*L1 + OPSI(-)*L2
static void addopsi(const orc_handle* h, cplx* psibar, const cplx* opsi, const cplx* lambda) {
  const int ngl = h->d.ngl, nbh = h->d.nbh, nb = h->d.nb;
  std::vector<cplx> l1, l2;
  lambda12(nb, nbh, lambda, l1, l2);
  if (g_zgemm) {
    // PSIBAR += OPSI L1 + conj(OPSI(-G)) L2 (two ZGEMMs, waves2:597-610)
    std::vector<cplx> om((size_t)ngl * nbh);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nbh; ++k)
      for (int ig = 0; ig < ngl; ++ig) om[ig + (size_t)ngl * k] = std::conj(opsi[PS(h, h->minusg[ig], k)]);
    zgemm('N', 'N', ngl, nbh, nbh, 1.0, opsi, ngl, l1.data(), nbh, 1.0, psibar, ngl);
    zgemm('N', 'N', ngl, nbh, nbh, 1.0, om.data(), ngl, l2.data(), nbh, 1.0, psibar, ngl);
    return;
  }
#pragma omp parallel for schedule(static)
  for (int ig = 0; ig < ngl; ++ig) {
    int mg = h->minusg[ig];
    for (int j = 0; j < nbh; ++j) {
      cplx acc = 0.0;
      for (int k = 0; k < nbh; ++k) acc += opsi[PS(h, ig, k)] * l1[k + (size_t)nbh * j];
      for (int k = 0; k < nbh; ++k) acc += std::conj(opsi[PS(h, mg, k)]) * l2[k + (size_t)nbh * j];
      psibar[PS(h, ig, j)] += acc;
    }
  }
}

// WAVES_ADDOPROJ (src/paw_waves2.f90:687-758), TINV
static void addoproj(const orc_handle* h, int npro, cplx* proj, const cplx* oproj, const cplx* lambda,
                     int nbproj_stride) {
  const int nbh = h->d.nbh, nb = h->d.nb;
  std::vector<cplx> l1, l2;
  lambda12(nb, nbh, lambda, l1, l2);
  for (int ibh1 = 0; ibh1 < nbh; ++ibh1)
    for (int ibh2 = 0; ibh2 < nbh; ++ibh2) {
      cplx c1 = l1[ibh2 + (size_t)nbh * ibh1], c2 = l2[ibh2 + (size_t)nbh * ibh1];
      for (int ip = 0; ip < npro; ++ip) {
        cplx o = oproj[ibh2 + (size_t)nbproj_stride * ip];
        proj[ibh1 + (size_t)nbproj_stride * ip] += o * c1 + std::conj(o) * c2;
      }
    }
}

// WAVES_WAVEKINETIC (src/paw_waves1.f90:6713-6847), one (k,spin); eig may be null
static double wavekinetic(const orc_handle* h, double* eigout) {
  const int ngl = h->d.ngl, nbh = h->d.nbh, nb = h->d.nb;
  double ekin1 = 0.0;
  std::vector<double> eig(nb, 0.0);
  const double dt2 = h->delt * h->delt;
  for (int ib = 0; ib < nbh; ++ib) {
    int ib1 = 2 * ib, ib2 = 2 * ib + 1;
    double f1 = h->occ[ib1], f2 = h->occ[ib2];
    if (f1 == 0.0 && f2 == 0.0) continue;
    double sum = 0.0;
    for (int ig = 0; ig < ngl; ++ig) {
      cplx c = h->psi0[PS(h, ig, ib)] - h->psim[PS(h, ig, ib)];
      sum += h->mpsi[ig] * (c.real() * c.real() + c.imag() * c.imag());
    }
    sum /= dt2;
    eig[ib1] = 0.5 * sum;
    eig[ib2] = 0.5 * sum;
    ekin1 += sum * 0.5 * (f1 + f2);
    if (f1 - f2 == 0.0) continue;
    sum = 0.0;
    for (int ig = 0; ig < ngl; ++ig) {
      cplx tp = h->psi0[PS(h, ig, ib)] - h->psim[PS(h, ig, ib)];
      int mg = h->minusg[ig];
      cplx tm = std::conj(h->psi0[PS(h, mg, ib)] - h->psim[PS(h, mg, ib)]);
      sum += h->mpsi[ig] * (tp.real() * tm.real() + tp.imag() * tm.imag());
    }
    sum /= dt2;
    eig[ib1] += 0.5 * sum;
    eig[ib2] -= 0.5 * sum;
    ekin1 += sum * 0.5 * (f1 - f2);
  }
  // EKIN=EKIN+EKIN1*CELLVOL
  if (eigout) for (int i = 0; i < nb; ++i) eigout[i] = eig[i];
  return ekin1 * h->gweight;
}

int orc_wavekinetic(orc_handle* h, double* ekin, double* eig) {
  *ekin = wavekinetic(h, eig);
  return CUW_OK;
}

// WAVES_EKIN (src/paw_waves1.f90:2790-2954), no stress
int orc_ekin(orc_handle* h, double* ekin) {
  const int ngl = h->d.ngl, nbh = h->d.nbh;
  std::vector<double> dmat(ngl, 0.0);
  for (int ib = 0; ib < nbh; ++ib) {
    double fp = 0.5 * (h->occ[2 * ib] + h->occ[2 * ib + 1]);
    double fm = 0.5 * (h->occ[2 * ib] - h->occ[2 * ib + 1]);
    if (fp == 0.0 && fm == 0.0) continue;
    for (int ig = 0; ig < ngl; ++ig) dmat[ig] += fp * std::norm(h->psi0[PS(h, ig, ib)]);
    if (std::fabs(fm) < 1e-12) continue;
    for (int ig = 0; ig < ngl; ++ig) {
      cplx p1 = std::conj(h->psi0[PS(h, h->minusg[ig], ib)]);
      dmat[ig] += fm * (std::conj(h->psi0[PS(h, ig, ib)]) * p1).real();
    }
  }
  double e = 0.0;
  for (int ig = 0; ig < ngl; ++ig) e += h->g2[ig] * dmat[ig];
  e *= 0.5;
  if (h->tbucket) {
    double eb = 0.0;
    for (int ig = 0; ig < ngl; ++ig) eb += h->bucket[ig] * dmat[ig];
    e += eb;
  }
  *ekin = e * h->gweight;
  return CUW_OK;
}

// WAVES$ETOT expectation values (src/paw_waves1.f90:2094-2123), TINV
int orc_expectation(orc_handle* h, double* eig) {
  OCHECK(h->have_hpsi, CUW_ERR_STATE, "hpsi not available");
  const int ngl = h->d.ngl, nbh = h->d.nbh;
  for (int ib = 0; ib < nbh; ++ib) {
    // WAVES_OVERLAP(.FALSE.,NGL,NDIM,1,2,PSI0(:,:,IB),HPSI(:,:,IB),HAMILTON)
    cplx tp = 0.0, tm = 0.0;
    const cplx* a = &h->psi0[PS(h, 0, ib)];
    const cplx* b = &h->hpsi[PS(h, 0, ib)];
    for (int ig = 0; ig < ngl; ++ig) tp += std::conj(a[ig]) * b[ig];
    for (int ig = 0; ig < ngl; ++ig) tm += std::conj(a[ig]) * std::conj(b[h->minusg[ig]]);
    tm = std::conj(tm);
    tp *= h->gweight;
    tm *= h->gweight;
    eig[2 * ib] = 0.5 * tp.real() + 0.5 * tm.real();
    eig[2 * ib + 1] = 0.5 * tp.real() - 0.5 * tm.real();
  }
  return CUW_OK;
}

// WAVES$PROPAGATE (src/paw_waves1.f90:6479-6592), no stress
// WAVES_DMPSI (src/paw_waves1.f90:6676-6711): ANNEEVEC(G) = ANNEE without
// TSTRESS, else ANNEE - tr(FRICMAT)/2 - EMASS*EMASSCG2 * G.FRICMAT.G *
// (1 + DBUCKET(G)) (FRICMAT symmetric: its off-diagonal terms counted twice)
static void dmpsi(const orc_handle* h, std::vector<double>& anneevec) {
  const int ngl = h->d.ngl;
  anneevec.assign(ngl, h->annee);
  if (!h->tstress) return;
  const double* F = h->fricmat;  // FRICMAT(i,j) = F[(i-1) + 3*(j-1)]
  const double fac1 = h->annee - 0.5 * (F[0] + F[4] + F[8]);
  const double fac2 = -0.5 * h->emass * 2.0 * h->emasscg2;
  for (int ig = 0; ig < ngl; ++ig) {
    const double* g = &h->gvec[3 * (size_t)ig];
    const double svar = F[0] * g[0] * g[0] + F[3] * 2.0 * g[0] * g[1] + F[6] * 2.0 * g[0] * g[2] +
                        F[4] * g[1] * g[1] + F[7] * 2.0 * g[1] * g[2] + F[8] * g[2] * g[2];
    anneevec[ig] = fac1 + fac2 * svar * (1.0 + (h->dbucket.empty() ? 0.0 : h->dbucket[ig]));
  }
}

int orc_set_cell_friction(orc_handle* h, const double* fricmat, double emass, double emasscg2,
                          const double* dbucket) {
  OCHECK(h->have_gset, CUW_ERR_STATE, "gset not set");
  h->tstress = fricmat != nullptr;
  if (fricmat) std::memcpy(h->fricmat, fricmat, sizeof(h->fricmat));
  h->emass = emass;
  h->emasscg2 = emasscg2;
  if (dbucket) h->dbucket.assign(dbucket, dbucket + h->d.ngl);
  else h->dbucket.clear();
  return CUW_OK;
}

int orc_propagate(orc_handle* h) {
  OCHECK(h->have_hpsi, CUW_ERR_STATE, "HPSI NOT AVAILABLE");
  const int ngl = h->d.ngl, nbh = h->d.nbh;
  if (h->tstress) {
    // ARR1..ARR3 per G from ANNEEVEC (waves1:6536-6540)
    std::vector<double> an, arr1(ngl), arr2(ngl), arr3(ngl);
    dmpsi(h, an);
    for (int ig = 0; ig < ngl; ++ig) {
      arr1[ig] = 2.0 / (1.0 + an[ig]);
      arr2[ig] = 1.0 - arr1[ig];
      arr3[ig] = -h->delt * h->delt / (1.0 + an[ig]) / h->mpsi[ig];
    }
#pragma omp parallel for schedule(static)
    for (int ib = 0; ib < nbh; ++ib)
      for (int ig = 0; ig < ngl; ++ig) {
        size_t k = PS(h, ig, ib);
        h->psim[k] = arr1[ig] * h->psi0[k] + arr2[ig] * h->psim[k] + arr3[ig] * h->hpsi[k];
      }
    h->have_hpsi = false;
    return CUW_OK;
  }
  const double svar1 = 2.0 / (1.0 + h->annee), svar2 = 1.0 - svar1;
  const double svar3 = -h->delt * h->delt / (1.0 + h->annee);
#pragma omp parallel for schedule(static)
  for (int ib = 0; ib < nbh; ++ib)
    for (int ig = 0; ig < ngl; ++ig) {
      double a3 = svar3 / h->mpsi[ig];
      size_t k = PS(h, ig, ib);
      h->psim[k] = svar1 * h->psi0[k] + svar2 * h->psim[k] + a3 * h->hpsi[k];
    }
  h->have_hpsi = false;
  return CUW_OK;
}

// WAVES$ORTHOGONALIZE (src/paw_waves2.f90:11-494), TSAFEORTHO, TINV, no stress
static int ortho_y_c(int nb, const cplx* phiphi, const cplx* chiphi, const cplx* chichi, cplx* x,
                     const int* map = nullptr);

int orc_orthogonalize(orc_handle* h, int maxit, double eps, int* iters) {
  OCHECK(h->have_gset && h->have_do, CUW_ERR_STATE, "gset/do not set");
  const int ngl = h->d.ngl, nbh = h->d.nbh, nb = h->d.nb, npro = h->npro;
  const size_t nps = (size_t)ngl * nbh;
  // OPSI = PSI0 + |p>DO<p|psi0>  (WAVES_OPSI, waves1:5043-5096)
  h->opsi = h->psi0;
  {
    std::vector<cplx> op((size_t)nbh * npro);
    oproj_all(h, h->proj.data(), op.data());
    addpro(h, h->r0.data(), h->opsi.data(), op.data());
  }
  // divide by mass (waves2:140-162)
  {
    const double svar = h->delt * h->delt / (1.0 + h->annee);
    for (size_t k = 0; k < nps; ++k) {
      int ig = (int)(k % ngl);
      h->opsi[k] *= svar / h->mpsi[ig];
    }
  }
  // projections at R(+) (waves2:250-256)
  projections(h, h->rp.data(), h->psim.data(), h->proj.data());
  std::vector<cplx> oproj((size_t)nbh * npro);
  projections(h, h->rp.data(), h->opsi.data(), oproj.data());
  // 1c overlaps (waves2:262-266)
  const size_t nn = (size_t)nb * nb;
  std::vector<cplx> mat(nn), omat(nn), oomat(nn), aux(nn);
  onecoverlap(h, h->proj.data(), h->proj.data(), mat.data());
  onecoverlap(h, oproj.data(), h->proj.data(), omat.data());
  onecoverlap(h, oproj.data(), oproj.data(), oomat.data());
  overlap(h, true, h->psim.data(), h->psim.data(), aux.data());
  for (size_t k = 0; k < nn; ++k) mat[k] += aux[k];
  overlap(h, false, h->opsi.data(), h->psim.data(), aux.data());
  for (size_t k = 0; k < nn; ++k) omat[k] += aux[k];
  overlap(h, true, h->opsi.data(), h->opsi.data(), aux.data());
  for (size_t k = 0; k < nn; ++k) oomat[k] += aux[k];
  // lambda (waves2:295-303, 352-359)
  std::vector<cplx> lambda = h->rlam0;
  for (int i = 0; i < nb; ++i)
    for (int j = i + 1; j < nb; ++j) {
      cplx c = 0.5 * (lambda[i + (size_t)nb * j] + std::conj(lambda[j + (size_t)nb * i]));
      lambda[i + (size_t)nb * j] = c;
      lambda[j + (size_t)nb * i] = std::conj(c);
    }
  // SMAP (waves2:306-346): with SAFEORTHO = F the states are handled in the
  // order MAP; SWAPSTATES = T sorts them by the real diagonal of LAMBDA with
  // the reference's exchange loop, then checks the order
  std::vector<int> smap(nb);
  for (int i = 0; i < nb; ++i) smap[i] = i;
  if (!h->safeortho && h->swapstates) {
    auto dg = [&](int k) { return lambda[k + (size_t)nb * k].real(); };
    for (int i = 0; i < nb; ++i)
      for (int j = i + 1; j < nb; ++j)
        if (dg(smap[j]) < dg(smap[i])) std::swap(smap[i], smap[j]);
    for (int i = 0; i + 1 < nb; ++i)
      OCHECK(!(dg(smap[i]) > dg(smap[i + 1])), CUW_ERR_STATE, "STATE ORDERING FAILED");
  }
  for (int i = 0; i < nb; ++i)
    for (int j = 0; j < nb; ++j) {
      double occi = h->occ[i], occj = h->occ[j];
      if (occi + occj < 1e-12) occj = 1e-12;
      lambda[i + (size_t)nb * j] *= 0.5 * occi / (occi + occj);
    }
  if (!h->safeortho) {
    // WAVES_ORTHO_Y_C(NB, MAT, OMAT, OOMAT, LAMBDA, SMAP) (waves2:384-386)
    OCHECK(ortho_y_c(nb, mat.data(), omat.data(), oomat.data(), lambda.data(), smap.data()) == CUW_OK, CUW_ERR_NAN,
           "NAN DETECTED in WAVES_ORTHO_Y_C");
    if (iters) *iters = 0;
    addopsi(h, h->psim.data(), h->opsi.data(), lambda.data());
    addoproj(h, npro, h->proj.data(), oproj.data(), lambda.data(), nbh);
    h->rlam0 = lambda;
    h->waveekin2 = wavekinetic(h, nullptr);
    return CUW_OK;
  }
  std::vector<double> rmat(nn), romat(nn), roomat(nn), rl(nn);
  for (size_t k = 0; k < nn; ++k) {
    rmat[k] = mat[k].real();
    romat[k] = omat[k].real();
    roomat[k] = oomat[k].real();
    rl[k] = lambda[k].real();
  }
  int status = CUW_OK;
  int it = ortho_x(nb, h->occ.data(), roomat.data(), rmat.data(), romat.data(), rl.data(), maxit, eps, &status);
  if (iters) *iters = it;
  if (status != CUW_OK)
    return fail(h, status, status == CUW_ERR_DIVERGED ? "ITERATION LOOP FOR ORTHOGONALIZATION IS ABOUT TO DIVERGE"
                                                      : "LOOP FOR ORTHOGONALIZATION IS NOT CONVERGED");
  for (size_t k = 0; k < nn; ++k) lambda[k] = cplx(rl[k], 0.0);
  // |psi(+)> = |psibar> + |chi> lambda (waves2:393-399)
  addopsi(h, h->psim.data(), h->opsi.data(), lambda.data());
  addoproj(h, npro, h->proj.data(), oproj.data(), lambda.data(), nbh);
  h->rlam0 = lambda;
  h->waveekin2 = wavekinetic(h, nullptr);
  return CUW_OK;
}

// TTEST block of WAVES$ORTHOGONALIZE (src/paw_waves2.f90:421-460) for PSI0:
// projections at R(0) (waves2:424), WAVES_1COVERLAP (:427) plus WAVES_OVERLAP
// (:438), real part at the Gamma point, and max|MAT - 1|
int orc_overlap_check(orc_handle* h, double* mat, double* maxdev) {
  OCHECK(h->have_gset && h->have_do, CUW_ERR_STATE, "gset/do not set");
  const int nbh = h->d.nbh, nb = h->d.nb, npro = h->npro;
  std::vector<cplx> proj((size_t)nbh * npro);
  projections(h, h->r0.data(), h->psi0.data(), proj.data());
  const size_t nn = (size_t)nb * nb;
  std::vector<cplx> m(nn), aux(nn);
  onecoverlap(h, proj.data(), proj.data(), m.data());
  overlap(h, true, h->psi0.data(), h->psi0.data(), aux.data());
  double dev = 0.0;
  for (int j = 0; j < nb; ++j)
    for (int i = 0; i < nb; ++i) {
      const size_t k = i + (size_t)nb * j;
      const double v = (m[k] + aux[k]).real();
      if (mat) mat[k] = v;
      dev = std::max(dev, std::fabs(v - (i == j ? 1.0 : 0.0)));
    }
  if (maxdev) *maxdev = dev;
  return CUW_OK;
}

// WAVES$SWITCH (src/paw_waves2.f90:2180-2317), NLAMBDAX=2, no stress
int orc_switch(orc_handle* h) {
  std::swap(h->psi0, h->psim);
  const size_t nn = (size_t)h->d.nb * h->d.nb;
  std::vector<cplx> rlamp(nn);
  if (!h->have_rlamm) {  // NLAMBDA=1
    rlamp = h->rlam0;
    h->rlamm = h->rlam0;
    h->have_rlamm = true;
  } else {               // NLAMBDA=2
    for (size_t k = 0; k < nn; ++k) rlamp[k] = 2.0 * h->rlam0[k] - h->rlamm[k];
    h->rlamm = h->rlam0;
  }
  h->rlam0 = rlamp;
  h->waveekin1 = h->waveekin2 = 0.0;
  return CUW_OK;
}

// WAVES$STOP (src/paw_waves1.f90:6445-6476)
int orc_stop(orc_handle* h) {
  h->psim = h->psi0;
  h->have_rlamm = false;
  return CUW_OK;
}

// WAVES_ORTHO_Y_C (src/paw_waves2.f90:1025-1338); map = MAP (0-based), null
// for the identity.  pos[i] is the place of state i in MAP, so "IU = NU+1, NB;
// I = MAP(IU)" of the reference is every i with pos[i] > nu.
static int ortho_y_c(int nb, const cplx* phiphi, const cplx* chiphi, const cplx* chichi, cplx* x, const int* map) {
  std::vector<int> pos(nb);
  for (int k = 0; k < nb; ++k) pos[map ? map[k] : k] = k;
  const size_t nn = (size_t)nb * nb;
  std::vector<cplx> A(nn), B(nn), C(nn), alpha(nn, 0.0), work(nn), z(nb);
  auto I = [nb](int i, int j) { return (size_t)i + (size_t)nb * j; };
  const double r8small = 1e-10;
  for (int i = 0; i < nb; ++i)
    for (int j = 0; j < nb; ++j) {
      A[I(i, j)] = phiphi[I(i, j)];
      B[I(i, j)] = chiphi[I(i, j)];
      C[I(i, j)] = chichi[I(i, j)];
      x[I(i, j)] = 0.0;
    }
  for (int i = 0; i < nb; ++i) {
    A[I(i, i)] -= 1.0;
    alpha[I(i, i)] = 1.0;
  }
  for (int nu = 0; nu < nb; ++nu) {
    const int n = map ? map[nu] : nu;
    double svar = (std::pow(B[I(n, n)].real(), 2) - A[I(n, n)] * C[I(n, n)]).real();
    double svar1 = -B[I(n, n)].real();
    if (svar >= 0.0) {
      double svar2 = std::sqrt(svar);
      z[n] = (svar1 * svar2 >= 0.0) ? svar1 - svar2 : svar1 + svar2;
    } else {
      z[n] = svar1;
    }
    z[n] = z[n] / (C[I(n, n)] + r8small).real();
    if (svar != svar) return CUW_ERR_NAN;
    for (int i = 0; i < nb; ++i) x[I(i, n)] += alpha[I(i, n)] * z[n];
    for (int j = 0; j < nb; ++j) A[I(n, j)] += std::conj(z[n]) * B[I(n, j)];
    for (int i = 0; i < nb; ++i) A[I(i, n)] += std::conj(B[I(n, i)]) * z[n];
    A[I(n, n)] += std::conj(z[n]) * C[I(n, n)] * z[n];
    for (int i = 0; i < nb; ++i) B[I(i, n)] += C[I(i, n)] * z[n];
    // orthogonalise higher phis to this phi
    for (int i = 0; i < nb; ++i) z[i] = pos[i] > nu ? -std::conj(A[I(i, n)] / (B[I(n, n)] + r8small)) : cplx(0.0);
    auto hi = [&](int k) { return pos[k] > nu; };  // JU = NU0..NB, J = MAP(JU)
    for (int j = 0; j < nb; ++j)
      if (hi(j))
        for (int i = 0; i < nb; ++i) x[I(i, j)] += alpha[I(i, n)] * z[j];
    for (int i = 0; i < nb; ++i)
      if (hi(i))
        for (int j = 0; j < nb; ++j) A[I(i, j)] += std::conj(z[i]) * B[I(n, j)];
    for (int i = 0; i < nb; ++i)
      for (int j = 0; j < nb; ++j)
        if (hi(j)) A[I(i, j)] += std::conj(B[I(n, i)]) * z[j];
    for (int i = 0; i < nb; ++i)
      for (int j = 0; j < nb; ++j)
        if (hi(i) && hi(j)) A[I(i, j)] += std::conj(z[i]) * C[I(n, n)] * z[j];
    for (int i = 0; i < nb; ++i)
      for (int j = 0; j < nb; ++j)
        if (hi(j)) B[I(i, j)] += C[I(i, n)] * z[j];
    // orthogonalise higher chis to this phi
    for (int i = 0; i < nb; ++i) z[i] = pos[i] > nu ? -std::conj(B[I(i, n)] / (B[I(n, n)] + r8small)) : cplx(0.0);
    for (int i = 0; i < nb; ++i)
      for (int j = 0; j < nb; ++j)
        if (hi(j)) alpha[I(i, j)] += alpha[I(i, n)] * z[j];
    for (int i = 0; i < nb; ++i)
      if (hi(i))
        for (int j = 0; j < nb; ++j) B[I(i, j)] += std::conj(z[i]) * B[I(n, j)];
    std::fill(work.begin(), work.end(), cplx(0.0));
    for (int i = 0; i < nb; ++i)
      if (hi(i))
        for (int j = 0; j < nb; ++j) work[I(i, j)] += std::conj(z[i]) * C[I(n, j)];
    for (int i = 0; i < nb; ++i)
      for (int j = 0; j < nb; ++j)
        if (hi(j)) work[I(i, j)] += C[I(i, n)] * z[j];
    for (int i = 0; i < nb; ++i)
      for (int j = 0; j < nb; ++j)
        if (hi(i) && hi(j)) work[I(i, j)] += std::conj(z[i]) * C[I(n, n)] * z[j];
    for (size_t k = 0; k < nn; ++k) C[k] += work[k];
  }
  return CUW_OK;
}

// WAVES_GRAMSCHMIDT (src/paw_waves2.f90:2025-2177), TINV
int orc_gramschmidt(orc_handle* h, int which, const double* r) {
  OCHECK(h->have_gset && h->have_do, CUW_ERR_STATE, "gset/do not set");
  auto* pp = which_psi(h, which);
  OCHECK(pp && (which == CUW_PSI0 || which == CUW_PSIM), CUW_ERR_ARG, "bad which");
  std::vector<cplx>& psi = *pp;
  const int ngl = h->d.ngl, nbh = h->d.nbh, nb = h->d.nb, npro = h->npro;
  std::vector<cplx> proj((size_t)nbh * npro);
  projections(h, r, psi.data(), proj.data());
  const size_t nn = (size_t)nb * nb;
  std::vector<cplx> ov(nn), aux(nn), x(nn);
  overlap(h, true, psi.data(), psi.data(), ov.data());
  onecoverlap(h, proj.data(), proj.data(), aux.data());
  for (size_t k = 0; k < nn; ++k) ov[k] += aux[k];
  int st = ortho_y_c(nb, ov.data(), ov.data(), ov.data(), x.data());
  OCHECK(st == CUW_OK, st, "NAN DETECTED in WAVES_ORTHO_Y_C");
  // fold X into X1, X2 (waves2:2109-2128)
  std::vector<cplx> x1((size_t)nbh * nbh), x2((size_t)nbh * nbh);
  for (int ibh1 = 0; ibh1 < nbh; ++ibh1) {
    int ib1a = 2 * ibh1, ib1b = std::min(2 * ibh1 + 1, nb - 1);
    for (int ibh2 = 0; ibh2 < nbh; ++ibh2) {
      int ib2a = 2 * ibh2, ib2b = std::min(2 * ibh2 + 1, nb - 1);
      cplx t[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
      for (int i = ib1a; i <= ib1b; ++i)
        for (int j = ib2a; j <= ib2b; ++j) t[i - ib1a][j - ib2a] = x[i + (size_t)nb * j];
      cplx c1 = t[0][0] + CI * t[0][1];
      cplx c2 = -CI * t[1][0] + t[1][1];
      x1[ibh1 + (size_t)nbh * ibh2] = 0.5 * (c1 + c2);
      x2[ibh1 + (size_t)nbh * ibh2] = 0.5 * (c1 - c2);
    }
  }
  // PSI_I = PSI_I + PSI_J X1_JI + PSIINV_J X2_JI with PSIINV(G) = conj(PSI(-G))
  std::vector<cplx> psiinv = psi;
#pragma omp parallel for schedule(static)
  for (int ig = 0; ig < ngl; ++ig) {
    int mg = h->minusg[ig];
    for (int i = 0; i < nbh; ++i) {
      cplx acc = 0.0;
      for (int j = 0; j < nbh; ++j) acc += psiinv[PS(h, ig, j)] * x1[j + (size_t)nbh * i];
      for (int j = 0; j < nbh; ++j) acc += std::conj(psiinv[PS(h, mg, j)]) * x2[j + (size_t)nbh * i];
      psi[PS(h, ig, i)] += acc;
    }
  }
  return CUW_OK;
}

// WAVES$FORCE (src/paw_waves1.f90:4570-4739) without stress: WAVES_DEDPROJ
// (:5592-5691), WAVES_DEDPRO (:5694-5743), WAVES_PROFORCE (:6112-6234)
int orc_force(orc_handle* h, double* force) {
  OCHECK(h->have_gset && h->have_dh && h->have_do, CUW_ERR_STATE, "gset/dh/do not set");
  const int ngl = h->d.ngl, nbh = h->d.nbh, nb = h->d.nb, nat = h->d.nat;
  std::vector<cplx> hproj((size_t)nbh * h->npro), oproj((size_t)nbh * h->npro);
  hproj_all(h, h->proj.data(), hproj.data());
  oproj_all(h, h->proj.data(), oproj.data());
  // DEDPROJ = DH<P|PSI>F  (TINV: F1*c + F2*conj(c))
  std::vector<cplx> dedproj((size_t)nbh * h->npro);
  for (int ip = 0; ip < h->npro; ++ip)
    for (int ib = 0; ib < nbh; ++ib) {
      double f1 = 0.5 * (h->occ[2 * ib] + h->occ[2 * ib + 1]);
      double f2 = 0.5 * (h->occ[2 * ib] - h->occ[2 * ib + 1]);
      cplx c = hproj[PJ(h, ib, ip)];
      dedproj[PJ(h, ib, ip)] = f1 * c + f2 * std::conj(c);
    }
  // ADD -DO<P|PSI>LAMBDA*(FI+FJ)/2
  std::vector<cplx> lam((size_t)nb * nb);
  for (int i = 0; i < nb; ++i)
    for (int j = 0; j < nb; ++j)
      lam[i + (size_t)nb * j] = -h->rlam0[i + (size_t)nb * j] * 0.5 * (h->occ[i] + h->occ[j]);
  addoproj(h, h->npro, dedproj.data(), oproj.data(), lam.data(), nbh);
  std::fill(force, force + 3 * nat, 0.0);
  // with BLAS: DEDPRO(G,IPRO) = sum_IB PSI(G,IB) conj(DEDPROJ(IB,IPRO)) of all
  // atoms by one ZGEMM (WAVES_DEDPRO, waves1:5694-5745)
  std::vector<cplx>& dall = h->protab;  // the work table of the ZGEMM path
  dall.clear();
  if (g_zgemm && h->npro > 0) {
    std::vector<cplx> dc(dedproj.size());
    for (size_t k = 0; k < dc.size(); ++k) dc[k] = std::conj(dedproj[k]);
    dall.resize((size_t)ngl * h->npro);
    zgemm('N', 'N', ngl, h->npro, nbh, 1.0, h->psi0.data(), ngl, dc.data(), nbh, 0.0, dall.data(), ngl);
  }
#pragma omp parallel
  {
    std::vector<cplx> dedpro((size_t)ngl * h->lmnxx), eigr(ngl), tmp(ngl);
#pragma omp for schedule(dynamic)
    for (int iat = 0; iat < nat; ++iat) {
      const int s = h->isp[iat], lmnx = h->lmnx[s], i0 = h->p_ipro0[iat];
      // DEDPRO(G,LMN) = sum_IB PSI(G,IB) conj(DEDPROJ(IB,LMN)), then TINV symmetrise
      for (int lmn = 0; lmn < lmnx; ++lmn) {
        cplx* d = &dedpro[(size_t)ngl * lmn];
        if (!dall.empty()) {
          std::copy(&dall[(size_t)ngl * (i0 + lmn)], &dall[(size_t)ngl * (i0 + lmn + 1)], d);
        } else {
          for (int ig = 0; ig < ngl; ++ig) d[ig] = 0.0;
          for (int ib = 0; ib < nbh; ++ib) {
            cplx c = std::conj(dedproj[PJ(h, ib, i0 + lmn)]);
            const cplx* p = &h->psi0[PS(h, 0, ib)];
            for (int ig = 0; ig < ngl; ++ig) d[ig] += p[ig] * c;
          }
        }
        for (int ig = 0; ig < ngl; ++ig) tmp[ig] = std::conj(d[h->minusg[ig]]);
        for (int ig = 0; ig < ngl; ++ig) d[ig] = 0.5 * (d[ig] + tmp[ig]);
      }
      structurefactor(h, h->r0.data() + 3 * iat, eigr.data());
      double f[3] = {0, 0, 0};
      int lmn = 0;
      for (int ln = 0; ln < h->d.lnx[s]; ++ln) {
        int l = h->d.lox[s][ln];
        cplx cil = mipow(l);
        const double* bare = &h->pro[(size_t)ngl * (h->ibpro[s] + ln)];
        for (int m = 0; m < 2 * l + 1; ++m) {
          const double* y = &h->ylm[(size_t)ngl * (l * l + m)];
          const cplx* d = &dedpro[(size_t)ngl * lmn];
          for (int ig = 0; ig < ngl; ++ig) {
            cplx cw = CI * bare[ig] * cil * eigr[ig];
            double sv = (cw * std::conj(d[ig])).real() * y[ig];
            f[0] += sv * h->gvec[3 * ig];
            f[1] += sv * h->gvec[3 * ig + 1];
            f[2] += sv * h->gvec[3 * ig + 2];
          }
          ++lmn;
        }
      }
      for (int k = 0; k < 3; ++k) force[3 * iat + k] = h->gweight * 2.0 * f[k];
    }
  }
  return CUW_OK;
}

// One CP step in the order of TIMESTEP (src/paw_driver.f90:280-561) for a fixed
// potential; see cuwaves_cp_step in the C ABI for the meaning of out[].
// Single-point energy and forces at PSI0, R(0): the energy part of WAVES$ETOT
// (src/paw_waves1.f90:2094-2123) with EKIN and FORCE; nothing is propagated.
int orc_etot(orc_handle* h, double* out, double* force) {
  const int nb = h->d.nb, nat = h->d.nat;
  double ekin = 0.0;
  int st = orc_ekin(h, &ekin);
  if (st) return st;
  if (force) {
    std::vector<double> f(3 * nat);
    st = orc_force(h, f.data());
    if (st) return st;
    std::copy(f.begin(), f.end(), force);
  }
  st = orc_hpsi(h);
  if (st) return st;
  std::vector<double> eig(nb);
  orc_expectation(h, eig.data());
  double etot = 0.0;
  for (int i = 0; i < nb; ++i) etot += h->occ[i] * eig[i];
  out[0] = etot;
  out[1] = ekin;
  return CUW_OK;
}

// ===========================================================================
// POTENTIAL$VOFRHO (src/paw_potential.f90:324-485, POTENTIAL_VOFRHO :487-895)
// at the Gamma point for one spin, without gradient corrections (LDA), stress,
// confining potential, pair potential or isolation (those parts do not touch
// the density); restated step by step.
// ===========================================================================
int orc_density(orc_handle* h, double* rho);

// one 3-D transform of the full grid (x fastest): dir = -1 forward with 1/N
// (PLANEWAVE_FFTRTOG), dir = +1 inverse unscaled (PLANEWAVE_FFTGTOR)
static void grid_fft3(const orc_handle* h, std::vector<cplx>& f, int dir) {
  const int n1 = h->d.nr1, n2 = h->d.nr2, n3 = h->d.nr3;
  const FFTPlan& q1 = dir > 0 ? h->p1g : h->p1r;
  const FFTPlan& q2 = dir > 0 ? h->p2g : h->p2r;
  const FFTPlan& q3 = dir > 0 ? h->p3g : h->p3r;
  std::vector<cplx> work;
  for (int k = 0; k < n3; ++k)
    for (int j = 0; j < n2; ++j) fft1d(q1, &f[(size_t)n1 * (j + (size_t)n2 * k)], 1, work);
  for (int k = 0; k < n3; ++k)
    for (int i = 0; i < n1; ++i) fft1d(q2, &f[i + (size_t)n1 * n2 * k], n1, work);
  for (int j = 0; j < n2; ++j)
    for (int i = 0; i < n1; ++i) fft1d(q3, &f[i + (size_t)n1 * j], n1 * n2, work);
  if (dir < 0) {
    const double sc = 1.0 / ((double)n1 * n2 * n3);
    for (cplx& x : f) x *= sc;
  }
}

// PLANEWAVE$SUPFFT('RTOG') of one real function (src/paw_fft.f90:1905-1937):
// FOFG(IGH) = 0.5 (F(G) + conj F(-G))
static void supfft_rtog(const orc_handle* h, const double* fofr, cplx* fofg) {
  const size_t nr = (size_t)h->d.nr1 * h->d.nr2 * h->d.nr3;
  std::vector<cplx> f(nr);
  for (size_t i = 0; i < nr; ++i) f[i] = cplx(fofr[i], 0.0);
  grid_fft3(h, f, -1);
  for (int ig = 0; ig < h->nglh; ++ig) {
    cplx f1 = f[h->rplus[ig]], f2 = std::conj(f[h->rminus[ig]]);
    fofg[ig] = 0.5 * (f1 + f2);
  }
}

// PLANEWAVE$SUPFFT('GTOR') of one real function (src/paw_fft.f90:1851-1886):
// F(G) = FOFG(IGH), F(-G) = conj FOFG(IGH) (the second wins for G = 0)
static void supfft_gtor(const orc_handle* h, const cplx* fofg, double* fofr) {
  const size_t nr = (size_t)h->d.nr1 * h->d.nr2 * h->d.nr3;
  std::vector<cplx> f(nr, cplx(0.0, 0.0));
  for (int ig = 0; ig < h->nglh; ++ig) {
    f[h->rplus[ig]] = fofg[ig];
    f[h->rminus[ig]] = std::conj(fofg[ig]);
  }
  grid_fft3(h, f, +1);
  for (size_t i = 0; i < nr; ++i) fofr[i] = f[i].real();
}

// PLANEWAVE$STRUCTUREFACTOR (src/paw_fft.f90:1597-1695) on the density set
static void rho_structurefactor(const orc_handle* h, const double* R, cplx* eigr) {
  const int nr[3] = {h->d.nr1, h->d.nr2, h->d.nr3};
  int nrmax = std::max(nr[0], std::max(nr[1], nr[2]));
  std::vector<cplx> w((size_t)(2 * nrmax + 1) * 3);
  auto W = [&](int i, int dir) -> cplx& { return w[(size_t)(i + nrmax) + (size_t)(2 * nrmax + 1) * dir]; };
  for (int dir = 0; dir < 3; ++dir) {
    double gr = h->gbas[0 + 3 * dir] * R[0] + h->gbas[1 + 3 * dir] * R[1] + h->gbas[2 + 3 * dir] * R[2];
    cplx cfacp(std::cos(gr), -std::sin(gr));
    cplx csvarp(1.0, 0.0);
    cplx cfacm = std::conj(cfacp), csvarm = csvarp;
    for (int i = 1; i <= nr[dir]; ++i) {
      W(i - 1, dir) = csvarp;
      csvarp *= cfacp;
      W(-i + 1, dir) = csvarm;
      csvarm *= cfacm;
    }
  }
  for (int ig = 0; ig < h->nglh; ++ig)
    eigr[ig] = W(h->rigvec[3 * ig], 0) * W(h->rigvec[3 * ig + 1], 1) * W(h->rigvec[3 * ig + 2], 2);
}

// DFT (src/paw_dft.f90:780-967) for the LDA of functional type 2: local
// exchange (EXCHANGE_X1, :2137-2236, EXFAC of EXCHANGE_INITIALIZE) plus the
// Perdew-Wang local correlation of the unpolarised gas (PERDEWWANG91L$EPSVAL
// with TSAFE, :4718-4834, PERDEWWANG91L_RHODEP1 :4521-4575; TSAFE is a
// parameter .TRUE., :56, so no table is used); RHOTMIN = 1e-6 (:62)
static double dft_lda(double rhot, double* vxc) {
  const double rhotmin = 1e-6;
  double val = rhot < rhotmin ? rhotmin : rhot;
  const double kffac = std::pow(3.0 * PI * PI, 1.0 / 3.0);
  const double exfac = -3.0 / (4.0 * PI) * kffac;
  double ex = 0.0, ex_r = 0.0;
  if (std::fabs(val) >= 1e-50) {
    const double r13 = std::pow(val, 1.0 / 3.0), r23 = r13 * r13, r43 = r23 * r23;
    ex = exfac * r43;
    ex_r = ex * (4.0 / 3.0) / val;
  }
  // PERDEWWANG91L_RHODEP1 with the sigma = 0 parameters
  const double au = 3.10907e-2, alpha1 = 2.1370e-1, beta1 = 7.5957, beta2 = 3.5876, beta3 = 1.6382,
               beta4 = 4.9294e-1;
  const double rsfac = std::pow(3.0 / (4.0 * PI), 1.0 / 3.0);
  const double rs = rsfac / std::pow(val, 1.0 / 3.0);
  const double sqrs = std::sqrt(rs), rssqrs = rs * sqrs;
  const double sv1 = -2.0 * au * (1.0 + alpha1 * rs), dsv1 = -2.0 * au * alpha1;
  const double sv2 = 2.0 * au * sqrs * (beta1 + beta2 * sqrs + beta3 * rs + beta4 * rssqrs);
  const double dsv2 = au / sqrs * (beta1 + 2.0 * beta2 * sqrs + 3.0 * beta3 * rs + 4.0 * beta4 * rssqrs);
  const double sv3 = 1.0 + 1.0 / sv2, dsv3 = -dsv2 / (sv2 * sv2);
  const double sv4 = std::log(sv3), dsv4 = dsv3 / sv3;
  double ecu = sv1 * sv4;
  double decu = dsv1 * sv4 + sv1 * dsv4;
  decu = decu * (-(1.0 / 3.0) * rs / val);
  // PERDEWWANG91L$EVAL1 (:5152-5170)
  const double ec = val * ecu, dec = val * decu + ecu;
  double exc = ex + ec, dexc = ex_r + dec;
  if (rhot < rhotmin) {  // wrap-up of DFT (:931-935)
    dexc = exc / rhotmin;
    exc = exc * rhot / rhotmin;
  }
  *vxc = dexc;
  return exc;
}

// The density G set and its tables.  igvec(3,NGLH), gvec(3,NGLH), g2(NGLH),
// ylm(LMRXX,NGLH) = Y_lm(G)|G|^l (POTENTIAL_YLMOFG, :1548-1616), g0, v0,
// pscore, vbar (NGLH,NSP) as SETUP$GETFOFG gives them (:300-309), lmrx(NSP).
int orc_set_rhoset(orc_handle* h, int nglh, const int* igvec, const double* gvec, const double* g2, int lmrxx,
                   const int* lmrx, const double* ylm, const double* g0, const double* v0, const double* pscore,
                   const double* vbar) {
  OCHECK(h->have_gset, CUW_ERR_STATE, "gset not set");
  OCHECK(nglh > 0 && lmrxx > 0 && igvec && gvec && g2 && lmrx && ylm && g0 && v0 && pscore && vbar, CUW_ERR_ARG,
         "bad density set");
  const int nsp = h->d.nsp;
  const int n[3] = {h->d.nr1, h->d.nr2, h->d.nr3};
  h->nglh = nglh;
  h->lmrxx = lmrxx;
  h->rigvec.assign(igvec, igvec + 3 * (size_t)nglh);
  h->rplus.resize(nglh);
  h->rminus.resize(nglh);
  h->ngamma = -1;
  for (int ig = 0; ig < nglh; ++ig) {
    int p[3], m[3];
    for (int k = 0; k < 3; ++k) {
      const int i = igvec[3 * ig + k];
      OCHECK(2 * std::abs(i) < n[k], CUW_ERR_ARG, "density G vector outside the grid");
      p[k] = ((i % n[k]) + n[k]) % n[k];
      m[k] = ((-i % n[k]) + n[k]) % n[k];
    }
    h->rplus[ig] = p[0] + n[0] * (p[1] + n[1] * p[2]);
    h->rminus[ig] = m[0] + n[0] * (m[1] + n[1] * m[2]);
    if (igvec[3 * ig] == 0 && igvec[3 * ig + 1] == 0 && igvec[3 * ig + 2] == 0) h->ngamma = ig;
  }
  h->rgvec.assign(gvec, gvec + 3 * (size_t)nglh);
  h->rg2.assign(g2, g2 + nglh);
  h->lmrx.assign(lmrx, lmrx + nsp);
  for (int s = 0; s < nsp; ++s) OCHECK(lmrx[s] >= 1 && lmrx[s] <= lmrxx, CUW_ERR_ARG, "LMRX out of range");
  h->rylm.assign(ylm, ylm + (size_t)lmrxx * nglh);
  h->rg0.assign(g0, g0 + (size_t)nglh * nsp);
  h->rv0.assign(v0, v0 + (size_t)nglh * nsp);
  h->rpscore.assign(pscore, pscore + (size_t)nglh * nsp);
  h->rvbar.assign(vbar, vbar + (size_t)nglh * nsp);
  h->have_rhoset = true;
  return CUW_OK;
}

int orc_set_qlm(orc_handle* h, const double* qlm) {
  OCHECK(h->have_rhoset && qlm, CUW_ERR_STATE, "density set not loaded");
  h->qlm.assign(qlm, qlm + (size_t)h->lmrxx * h->d.nat);
  return CUW_OK;
}

int orc_set_option(orc_handle* h, int option, double value) {
  if (option == CUW_OPT_SAFEORTHO) h->safeortho = value != 0.0;
  if (option == CUW_OPT_SWAPSTATES) h->swapstates = value != 0.0;
  if (option == CUW_OPT_SELFCONSISTENT) {
    OCHECK(value == 0.0 || (h->have_rhoset && !h->qlm.empty()), CUW_ERR_STATE, "density set or QLM missing");
    h->scf = value != 0.0;
  }
  return CUW_OK;  // the engine's tuning options do not apply to the oracle
}

// POTENTIAL_VOFRHO for RHOE = rho (pseudo density of the wave functions):
// v = the potential on the grid; e[0] EHARTREE, e[1] EXC, e[2] RHOB;
// force (3,NAT) Hartree + pseudo-core forces; vqlm (LMRXX,NAT)
static int vofrho_core(orc_handle* h, const double* rho, double* v, double* e, double* force, double* vqlm) {
  const int nglh = h->nglh, nat = h->d.nat, lmrxx = h->lmrxx;
  const size_t nr = (size_t)h->d.nr1 * h->d.nr2 * h->d.nr3;
  const double fpi = 4.0 * PI, y0 = 1.0 / std::sqrt(4.0 * PI);
  const double cellvol = h->gweight;
  const int lrxx = (int)std::sqrt((double)(lmrxx - 1) + 1e-5);
  // RHOG = SUPFFT('RTOG', RHOE) (:600)
  std::vector<cplx> rhog(nglh), eigr(nglh);
  supfft_rtog(h, rho, rhog.data());
  // POTENTIAL_ADDCORE (:1038-1066)
  for (int a = 0; a < nat; ++a) {
    const int s = h->isp[a];
    rho_structurefactor(h, &h->r0[3 * a], eigr.data());
    for (int ig = 0; ig < nglh; ++ig) rhog[ig] += h->rpscore[ig + (size_t)nglh * s] * y0 * eigr[ig];
  }
  // POTENTIAL_HARTREE (:1069-1336) without stress
  std::vector<cplx> cfac(lmrxx);
  {
    int lm = 0;
    cplx csvar(0.0, 1.0);
    for (int l = 0; l <= lrxx; ++l) {
      csvar = -csvar * CI / (double)(2 * l + 1);
      for (int m = -l; m <= l; ++m)
        if (lm < lmrxx) cfac[lm++] = csvar;
    }
  }
  std::vector<cplx> rho2(rhog), pot(nglh, cplx(0.0, 0.0)), vg(nglh);
  double vb = 0.0;
  for (int a = 0; a < nat; ++a) {
    const int s = h->isp[a];
    rho_structurefactor(h, &h->r0[3 * a], eigr.data());
    if (h->ngamma >= 0) vb += h->qlm[(size_t)lmrxx * a] * y0 * h->rv0[h->ngamma + (size_t)nglh * s];
    for (int ig = 0; ig < nglh; ++ig) {
      cplx c(0.0, 0.0);
      for (int lm = 0; lm < h->lmrx[s]; ++lm)
        c += cfac[lm] * h->qlm[lm + (size_t)lmrxx * a] * h->rylm[lm + (size_t)lmrxx * ig];
      c *= eigr[ig];
      rho2[ig] += c * h->rg0[ig + (size_t)nglh * s];
      pot[ig] += c * h->rv0[ig + (size_t)nglh * s] + h->rvbar[ig + (size_t)nglh * s] * y0 * eigr[ig];
    }
  }
  double rhob = 0.0;
  if (h->ngamma >= 0) {
    rhob = -rho2[h->ngamma].real();
    rho2[h->ngamma] = 0.0;
  }
  cplx csum(0.0, 0.0);
  for (int ig = 0; ig < nglh; ++ig) {
    if (ig != h->ngamma) {
      vg[ig] = rho2[ig] * fpi / h->rg2[ig];
      csum += 0.5 * std::conj(rho2[ig]) * vg[ig] + std::conj(rhog[ig]) * pot[ig];
      pot[ig] += vg[ig];
    } else {
      vg[ig] = -vb;
      csum += 0.5 * (std::conj(rhog[ig]) * pot[ig] + rhob * vb);
      pot[ig] += vg[ig];
    }
  }
  double ehartree = csum.real();
  // forces and VQLM (:1240-1319)
  for (int ig = 0; ig < nglh; ++ig) rho2[ig] = rhog[ig];
  if (h->ngamma >= 0) rho2[h->ngamma] += rhob;
  std::vector<double> f(3 * (size_t)nat, 0.0), vq((size_t)lmrxx * nat, 0.0);
  for (int a = 0; a < nat; ++a) {
    const int s = h->isp[a];
    rho_structurefactor(h, &h->r0[3 * a], eigr.data());
    for (int ig = 0; ig < nglh; ++ig) {
      const double g0 = h->rg0[ig + (size_t)nglh * s], v0 = h->rv0[ig + (size_t)nglh * s];
      const double* y = &h->rylm[(size_t)lmrxx * ig];
      if (ig == h->ngamma) {
        cplx c0 = g0 * std::conj(vg[ig]) + v0 * std::conj(rho2[ig]);
        cplx c = c0 * cfac[0] * y[0] * eigr[ig];
        vq[(size_t)lmrxx * a] -= 0.5 * c.real();
      }
      cplx aval = (g0 * std::conj(vg[ig]) + v0 * std::conj(rho2[ig])) * eigr[ig];
      cplx cs(0.0, 0.0);
      for (int lm = 0; lm < h->lmrx[s]; ++lm) {
        cplx c = cfac[lm] * y[lm];
        vq[lm + (size_t)lmrxx * a] += (c * aval).real();
        cs += h->qlm[lm + (size_t)lmrxx * a] * c;
      }
      cplx cval = h->rvbar[ig + (size_t)nglh * s] * y0 * eigr[ig] * std::conj(rhog[ig]);
      const double sv = (cval + cs * aval).imag();
      for (int k = 0; k < 3; ++k) f[3 * a + k] -= h->rgvec[3 * ig + k] * sv;
    }
  }
  ehartree *= 2.0 * cellvol;
  for (double& x : vq) x *= 2.0 * cellvol;
  for (double& x : f) x *= 2.0 * cellvol;
  // total pseudo density in real space (:747), XC (POTENTIAL_XC, :1339-1545)
  std::vector<double> rt(nr);
  supfft_gtor(h, rhog.data(), rt.data());
  double sxc = 0.0, ssxc = 0.0;
  for (size_t ir = 0; ir < nr; ++ir) {
    double rhot = std::max(rt[ir], 1e-8);
    double vt = 0.0;
    sxc += dft_lda(rhot, &vt);
    rt[ir] = vt;
    if ((ir + 1) % 100 == 0) {
      ssxc += sxc;
      sxc = 0.0;
    }
  }
  ssxc += sxc;
  const double exc = ssxc * cellvol / (double)nr;
  // V(G) = SUPFFT('RTOG', VXC) + VHARTREE (:778-800)
  std::vector<cplx> vtot(nglh);
  supfft_rtog(h, rt.data(), vtot.data());
  for (int ig = 0; ig < nglh; ++ig) vtot[ig] += pot[ig];
  // POTENTIAL_FPSCORE (:897-975)
  for (int a = 0; a < nat; ++a) {
    const int s = h->isp[a];
    rho_structurefactor(h, &h->r0[3 * a], eigr.data());
    double fa[3] = {0, 0, 0}, f1[3] = {0, 0, 0};
    for (int ig = 0; ig < nglh; ++ig) {
      cplx c = std::conj(vtot[ig]) * h->rpscore[ig + (size_t)nglh * s] * eigr[ig];
      const double sv = -c.imag();
      for (int k = 0; k < 3; ++k) f1[k] += sv * h->rgvec[3 * ig + k];
      if ((ig + 1) % 100 == 0)
        for (int k = 0; k < 3; ++k) {
          fa[k] += f1[k];
          f1[k] = 0.0;
        }
    }
    for (int k = 0; k < 3; ++k) f[3 * a + k] += (fa[k] + f1[k]) * y0 * 2.0 * cellvol;
  }
  // V(r) (:890)
  supfft_gtor(h, vtot.data(), v);
  if (e) {
    e[0] = ehartree;
    e[1] = exc;
    e[2] = rhob;
  }
  if (force) std::memcpy(force, f.data(), sizeof(double) * f.size());
  if (vqlm) std::memcpy(vqlm, vq.data(), sizeof(double) * vq.size());
  return CUW_OK;
}

// POTENTIAL$VOFRHO: the handle's potential becomes V[rho]; rho == NULL takes
// the pseudo density of PSI0 (WAVES_DENSITY); v, e, force, vqlm may be NULL
int orc_vofrho(orc_handle* h, const double* rho, const double* qlm, double* v, double* e, double* force,
               double* vqlm) {
  OCHECK(h->have_rhoset, CUW_ERR_STATE, "density set not loaded");
  if (qlm) h->qlm.assign(qlm, qlm + (size_t)h->lmrxx * h->d.nat);
  OCHECK(!h->qlm.empty(), CUW_ERR_STATE, "QLM not set");
  const size_t nr = (size_t)h->d.nr1 * h->d.nr2 * h->d.nr3;
  std::vector<double> r(nr), vv(nr);
  if (rho) std::memcpy(r.data(), rho, sizeof(double) * nr);
  else {
    int st = orc_density(h, r.data());
    if (st) return st;
  }
  int st = vofrho_core(h, r.data(), vv.data(), e, force, vqlm);
  if (st) return st;
  h->v = vv;
  h->have_v = true;
  if (v) std::memcpy(v, vv.data(), sizeof(double) * nr);
  return CUW_OK;
}

int orc_cp_step(orc_handle* h, int move_atoms, const double* mass, int maxit, double eps,
                double* out, double* force) {
  const int nb = h->d.nb, nat = h->d.nat;
  double ekin = 0.0, ekin1 = 0.0;
  int st = orc_ekin(h, &ekin);
  if (st) return st;
  // self-consistent step: V(r) from the density of PSI0 at R(0) before H|psi>
  // (the order of WAVES$ETOT -> POTENTIAL$VOFRHO -> WAVES$HPSI in TIMESTEP)
  double epot[3] = {0.0, 0.0, 0.0}, edc = 0.0;
  std::vector<double> fpot(3 * (size_t)nat, 0.0);
  if (h->scf) {
    const size_t nr = (size_t)h->d.nr1 * h->d.nr2 * h->d.nr3;
    std::vector<double> rho(nr);
    st = orc_density(h, rho.data());
    if (st) return st;
    st = vofrho_core(h, rho.data(), h->v.data(), epot, fpot.data(), nullptr);
    if (st) return st;
    // sum_n f_n <psi_n|V|psi_n> = int V rho, removed from the band energy
    for (size_t ir = 0; ir < nr; ++ir) edc += h->v[ir] * rho[ir];
    edc *= h->gweight / (double)nr;
  }
  std::vector<double> f(3 * nat);
  st = orc_force(h, f.data());
  if (st) return st;
  for (size_t i = 0; i < f.size(); ++i) f[i] += fpot[i];
  st = orc_hpsi(h);
  if (st) return st;
  std::vector<double> eig(nb);
  orc_expectation(h, eig.data());
  double etot = 0.0;
  for (int i = 0; i < nb; ++i) etot += h->occ[i] * eig[i];
  if (h->scf) etot += epot[0] + epot[1] - edc;
  ekin1 = wavekinetic(h, nullptr);
  double eion = 0.0;
  if (move_atoms) {
    const double dt2 = h->delt * h->delt;
    for (int a = 0; a < nat; ++a)
      for (int k = 0; k < 3; ++k) {
        int i = 3 * a + k;
        h->rp[i] = 2.0 * h->r0[i] - h->rm[i] + dt2 * f[i] / mass[a];
      }
  }
  st = orc_propagate(h);
  if (st) return st;
  int iters = 0;
  st = orc_orthogonalize(h, maxit, eps, &iters);
  if (st) return st;
  double ekin2 = h->waveekin2;
  if (move_atoms) {
    for (int a = 0; a < nat; ++a)
      for (int k = 0; k < 3; ++k) {
        int i = 3 * a + k;
        double vel = (h->rp[i] - h->rm[i]) / (2.0 * h->delt);
        eion += 0.5 * mass[a] * vel * vel;
      }
  }
  orc_switch(h);
  if (move_atoms) {
    h->rm = h->r0;
    h->r0 = h->rp;
  }
  if (out) {
    out[0] = etot;
    out[1] = ekin;
    out[2] = 0.5 * (ekin1 + ekin2);
    out[3] = eion;
    out[4] = iters;
    out[5] = epot[0];
    out[6] = epot[1];
    out[7] = edc;
  }
  if (force) std::memcpy(force, f.data(), sizeof(double) * 3 * nat);
  return CUW_OK;
}

// WAVES_DENSITY (src/paw_waves1.f90:5377-5500) for super wave functions
// (TINV, NDIM=1) at the Gamma point, where EI2KR = 1 (:5466-5470): the pseudo
// density of one wave-function set, rho(r) = sum_ibh Re[psi(r) (s1 conj psi(r)
// + s2 psi(r))] with s1,s2 = (f(2ibh-1) +- f(2ibh))/2 (:5474-5496); the
// G->R transforms of PLANEWAVE$FFT('GTOR') (:5441).  RHOKIN is not formed.
int orc_density(orc_handle* h, double* rho) {
  OCHECK(h->have_gset, CUW_ERR_STATE, "gset not set");
  OCHECK(rho, CUW_ERR_ARG, "null rho");
  const int nb = h->d.nb, nbh = h->d.nbh;
  const size_t nr = (size_t)h->d.nr1 * h->d.nr2 * h->d.nr3;
  std::vector<cplx> psir(nr * nbh);
#pragma omp parallel for schedule(dynamic)
  for (int ib = 0; ib < nbh; ++ib) fft_gtor(h, &h->psi0[PS(h, 0, ib)], &psir[nr * ib]);
  for (size_t ir = 0; ir < nr; ++ir) rho[ir] = 0.0;
  for (int ib = 0; ib < nbh; ++ib) {
    const double f1 = h->occ[2 * ib], f2 = 2 * ib + 1 < nb ? h->occ[2 * ib + 1] : 0.0;
    const double s1 = 0.5 * (f1 + f2), s2 = 0.5 * (f1 - f2);
    if (s1 == 0.0 && s2 == 0.0) continue;
    const cplx* pr = &psir[nr * ib];
#pragma omp parallel for
    for (long long ir = 0; ir < (long long)nr; ++ir) {
      cplx p1 = s1 * std::conj(pr[ir]);
      if (s2 != 0.0) p1 += s2 * pr[ir];
      rho[ir] += std::real(pr[ir] * p1);
    }
  }
  return CUW_OK;
}

// WAVES$DENMAT (src/paw_waves1.f90:2957-3134) for one wave-function set with
// WAVES_DENMAT (:3331-3572) per atom, TINV and NDIM=1: the one-centre density
// matrix D(lmn1,lmn2) = Re sum_ib PROJ(ib,lmn1) (s1 conj PROJ(ib,lmn2) + s2
// PROJ(ib,lmn2)) and the energy-weighted EDENMAT from RLAM0 and the
// occupations (:3438-3472), both made Hermitian (:3525-3540) and real
// (:3551-3554).  denmat, edenmat: (LMNXX,LMNXX,NAT) complex, zero past LMNX.
int orc_denmat(orc_handle* h, int lmnxx, double* denmat, double* edenmat) {
  OCHECK(lmnxx >= h->lmnxx, CUW_ERR_ARG, "lmnxx smaller than the largest LMNX");
  const int nb = h->d.nb, nbh = h->d.nbh, nat = h->d.nat;
  const cplx ci(0.0, 1.0);
  cplx* D = reinterpret_cast<cplx*>(denmat);
  cplx* E = reinterpret_cast<cplx*>(edenmat);
  const size_t per = (size_t)lmnxx * lmnxx;
  if (D) std::fill(D, D + per * nat, cplx(0.0));
  if (E) std::fill(E, E + per * nat, cplx(0.0));
  // LAGR(:,IB2) = LAMBDA(:,IB2) OCC(IB2)
  std::vector<cplx> lagr((size_t)nb * nb);
  for (int j = 0; j < nb; ++j)
    for (int i = 0; i < nb; ++i) lagr[i + (size_t)nb * j] = h->rlam0[i + (size_t)nb * j] * h->occ[j];
  auto L = [&](int i, int j) { return lagr[(size_t)(i - 1) + (size_t)nb * (j - 1)]; };  // 1-based
  for (int a = 0; a < nat; ++a) {
    const int lmnx = h->lmnx[h->isp[a]], p0 = h->p_ipro0[a];
    auto P = [&](int ib, int lmn) { return h->proj[PJ(h, ib, p0 + lmn)]; };
    std::vector<cplx> d1((size_t)lmnx * lmnx, 0.0), e1((size_t)lmnx * lmnx, 0.0), func(lmnx);
    for (int ib = 0; ib < nbh; ++ib) {
      const double f1 = h->occ[2 * ib], f2 = 2 * ib + 1 < nb ? h->occ[2 * ib + 1] : 0.0;
      const double s1 = 0.5 * (f1 + f2), s2 = 0.5 * (f1 - f2);
      for (int l = 0; l < lmnx; ++l) func[l] = s1 * std::conj(P(ib, l)) + s2 * P(ib, l);
      for (int l2 = 0; l2 < lmnx; ++l2)
        for (int l1 = 0; l1 < lmnx; ++l1) d1[l1 + (size_t)lmnx * l2] += P(ib, l1) * func[l2];
    }
    for (auto& x : d1) x = std::real(x);
    for (int ib1 = 1; ib1 <= nbh; ++ib1) {
      std::fill(func.begin(), func.end(), cplx(0.0));
      for (int ib2 = 1; ib2 <= nbh; ++ib2) {
        const cplx cr = L(2 * ib1 - 1, 2 * ib2 - 1) + ci * L(2 * ib1, 2 * ib2 - 1);
        const cplx cim = L(2 * ib1 - 1, 2 * ib2) + ci * L(2 * ib1, 2 * ib2);
        const cplx c1 = 0.5 * (cr - ci * cim), c2 = 0.5 * (cr + ci * cim);
        for (int l = 0; l < lmnx; ++l) func[l] += c1 * P(ib2 - 1, l) + c2 * std::conj(P(ib2 - 1, l));
      }
      for (int l2 = 0; l2 < lmnx; ++l2)
        for (int l1 = 0; l1 < lmnx; ++l1) e1[l1 + (size_t)lmnx * l2] += std::conj(P(ib1 - 1, l1)) * func[l2];
    }
    for (auto& x : e1) x = std::real(x);
    for (int l1 = 0; l1 < lmnx; ++l1)
      for (int l2 = l1 + 1; l2 < lmnx; ++l2) {
        cplx c = 0.5 * (d1[l1 + (size_t)lmnx * l2] + std::conj(d1[l2 + (size_t)lmnx * l1]));
        d1[l1 + (size_t)lmnx * l2] = c;
        d1[l2 + (size_t)lmnx * l1] = std::conj(c);
        c = 0.5 * (e1[l1 + (size_t)lmnx * l2] + std::conj(e1[l2 + (size_t)lmnx * l1]));
        e1[l1 + (size_t)lmnx * l2] = c;
        e1[l2 + (size_t)lmnx * l1] = std::conj(c);
      }
    for (int l2 = 0; l2 < lmnx; ++l2)
      for (int l1 = 0; l1 < lmnx; ++l1) {
        if (D) D[per * a + l1 + (size_t)lmnxx * l2] = std::real(d1[l1 + (size_t)lmnx * l2]);
        if (E) E[per * a + l1 + (size_t)lmnxx * l2] = std::real(e1[l1 + (size_t)lmnx * l2]);
      }
  }
  return CUW_OK;
}

// WAVES$WRITE (src/paw_waves2.f90:3058-3088) for one set: the separator
// (SEPARATOR_TYPE, src/paw_report.f90:108-115) and the records of
// WAVES_WRITEPSI (src/paw_waves2.f90:3216-3326) and WAVES_WRITELAMBDA
// (:3974-4025) for NKPT = NSPIN = NDIM = 1 and a dynamic restart, as
// sequential unformatted Fortran records (4-byte length markers).
}  // extern "C"
static void orc_rec(FILE* f, const std::string& b) {
  const int32_t n = (int32_t)b.size();
  std::fwrite(&n, 4, 1, f);
  std::fwrite(b.data(), 1, b.size(), f);
  std::fwrite(&n, 4, 1, f);
}
template <class T>
static void orc_put(std::string& b, const T* p, size_t n) {
  b.append(reinterpret_cast<const char*>(p), sizeof(T) * n);
}
static void orc_chars(std::string& b, const char* s, size_t w) {
  std::string t(s);
  t.resize(w, ' ');
  b += t;
}

extern "C" {
int orc_write_restart(orc_handle* h, const char* path, const double* rbas_in) {
  OCHECK(h->have_gset && path, CUW_ERR_ARG, "G set or path missing");
  const int ngl = h->d.ngl, nb = h->d.nb, nbh = h->d.nbh;
  double rbas[9];
  if (rbas_in) {
    std::memcpy(rbas, rbas_in, sizeof(rbas));
  } else {  // RBAS = 2 pi GBAS^-T: RBAS(i,j) = 2 pi cofactor(i,j) / det
    auto G = [&](int r, int c) { return h->gbas[r + 3 * c]; };
    auto cof = [&](int i, int j) {
      int r[2], c[2], nr = 0, nc = 0;
      for (int k = 0; k < 3; ++k) {
        if (k != i) r[nr++] = k;
        if (k != j) c[nc++] = k;
      }
      const double m = G(r[0], c[0]) * G(r[1], c[1]) - G(r[0], c[1]) * G(r[1], c[0]);
      return ((i + j) % 2 ? -m : m);
    };
    const double det = G(0, 0) * cof(0, 0) + G(0, 1) * cof(0, 1) + G(0, 2) * cof(0, 2);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) rbas[i + 3 * j] = 2.0 * M_PI * cof(i, j) / det;
  }
  const int32_t nwave = 2, nlambda = h->have_rlamm ? 2 : 1;
  const int32_t nrec = 1 + 2 + nwave * nbh + 1 + nlambda;
  FILE* f = std::fopen(path, "wb");
  OCHECK(f, CUW_ERR_ARG, "cannot open the restart file");
  std::string b;
  orc_put(b, &nrec, 1);
  orc_chars(b, "WAVES", 32); orc_chars(b, "NONE", 32); orc_chars(b, "AUG1996", 64); orc_chars(b, "NONE", 256);
  orc_rec(f, b);
  b.clear();
  const int32_t one = 1;
  orc_put(b, &one, 1); orc_put(b, &one, 1); orc_put(b, rbas, 9); orc_put(b, &nwave, 1);
  orc_rec(f, b);
  b.clear();
  const int32_t hdr[4] = {ngl, 1, nb, 1};
  orc_chars(b, "PSI", 8); orc_put(b, hdr, 4);
  orc_rec(f, b);
  b.clear();
  const double xk[3] = {0, 0, 0};
  orc_put(b, xk, 3); orc_put(b, h->igvec.data(), h->igvec.size());
  orc_rec(f, b);
  for (int w = 0; w < nwave; ++w)
    for (int ib = 0; ib < nbh; ++ib) {
      b.clear();
      orc_put(b, &(w ? h->psim : h->psi0)[PS(h, 0, ib)], (size_t)ngl);
      orc_rec(f, b);
    }
  b.clear();
  const int32_t lh[4] = {nb, 1, 1, nlambda};
  orc_chars(b, "LAMBDA", 8); orc_put(b, lh, 4);
  orc_rec(f, b);
  for (int l = 0; l < nlambda; ++l) {
    b.clear();
    orc_put(b, (l ? h->rlamm : h->rlam0).data(), (size_t)nb * nb);
    orc_rec(f, b);
  }
  std::fclose(f);
  return CUW_OK;
}

// WAVES_READPSI (src/paw_waves2.f90:5147-5513) of a section written for the
// same bands, with the G vectors matched by IGVEC
int orc_read_restart(orc_handle* h, const char* path) {
  OCHECK(h->have_gset && path, CUW_ERR_ARG, "G set or path missing");
  FILE* f = std::fopen(path, "rb");
  OCHECK(f, CUW_ERR_ARG, "cannot open the restart file");
  // one record of exactly `expect` bytes; another length is refused before
  // anything is sized from the file's marker
  auto rd = [&](std::string& b, size_t expect) {
    int32_t n = 0, m = 0;
    if (std::fread(&n, 4, 1, f) != 1 || n < 0 || (size_t)n != expect) return false;
    b.resize(n);
    if (n && std::fread(&b[0], 1, n, f) != (size_t)n) return false;
    return std::fread(&m, 4, 1, f) == 1 && m == n;
  };
  const int ngl = h->d.ngl, nb = h->d.nb, nbh = h->d.nbh;
  std::string b;
  bool ok = rd(b, 388) && b.compare(4, 5, "WAVES") == 0;
  int32_t v4[4];
  ok = ok && rd(b, 84);
  int32_t nwave = 0;
  if (ok) std::memcpy(&nwave, b.data() + 80, 4);
  ok = ok && (nwave == 1 || nwave == 2);
  ok = ok && rd(b, 24) && b.compare(0, 3, "PSI") == 0;
  if (ok) std::memcpy(v4, b.data() + 8, 16);
  // a G-vector count that no record can hold is refused before anything is sized from it
  ok = ok && v4[0] > 0 && (size_t)v4[0] <= ((size_t)INT32_MAX - 24) / 12;
  const int ngg = ok ? v4[0] : 0;
  ok = ok && v4[2] == nb && rd(b, 24 + (size_t)12 * ngg);
  std::vector<int> map(ngg, -1);
  if (ok) {
    std::map<std::vector<int>, int> pos;
    for (int i = 0; i < ngl; ++i) pos[{h->igvec[3 * i], h->igvec[3 * i + 1], h->igvec[3 * i + 2]}] = i;
    for (int i = 0; i < ngg; ++i) {
      int v[3];
      std::memcpy(v, b.data() + 24 + 12 * (size_t)i, 12);
      auto it = pos.find({v[0], v[1], v[2]});
      if (it != pos.end()) map[i] = it->second;
    }
  }
  // G vectors that the file lacks become zero (MAPG(IG)=0, src/paw_waves2.f90:5395-5403)
  // read into copies; the handle changes only once the whole section is valid
  std::vector<cplx> psi0(h->psi0.size(), cplx(0.0, 0.0)), psim(h->psim.size(), cplx(0.0, 0.0));
  std::vector<cplx> rlam0(h->rlam0.size(), cplx(0.0, 0.0)), rlamm(h->rlamm.size(), cplx(0.0, 0.0));
  for (int w = 0; w < nwave && ok; ++w)
    for (int ib = 0; ib < nbh && ok; ++ib) {
      ok = rd(b, 16 * (size_t)ngg);
      for (int i = 0; i < ngg && ok; ++i)
        if (map[i] >= 0) std::memcpy(&(w ? psim : psi0)[PS(h, map[i], ib)], b.data() + 16 * (size_t)i, 16);
    }
  if (ok && nwave == 1) psim = psi0;
  ok = ok && rd(b, 24) && b.compare(0, 6, "LAMBDA") == 0;
  int nlambda = 0;
  if (ok) {
    std::memcpy(v4, b.data() + 8, 16);
    nlambda = v4[3];
    ok = v4[0] == nb && nlambda >= 0 && nlambda <= 4;
  }
  for (int l = 0; l < nlambda && ok; ++l) {
    ok = rd(b, 16 * (size_t)nb * nb);
    if (ok && l < 2) std::memcpy((l ? rlamm : rlam0).data(), b.data(), b.size());
  }
  std::fclose(f);
  OCHECK(ok, CUW_ERR_ARG, "restart file does not hold a WAVES section of this set");
  h->psi0.swap(psi0);
  h->psim.swap(psim);
  h->rlam0.swap(rlam0);
  if (nlambda >= 2) h->rlamm.swap(rlamm);
  h->have_rlamm = nlambda >= 2;
  h->have_hpsi = false;
  return CUW_OK;
}

int orc_get_atoms(orc_handle* h, double* rm, double* r0, double* rp) {
  if (rm) std::memcpy(rm, h->rm.data(), sizeof(double) * 3 * h->d.nat);
  if (r0) std::memcpy(r0, h->r0.data(), sizeof(double) * 3 * h->d.nat);
  if (rp) std::memcpy(rp, h->rp.data(), sizeof(double) * 3 * h->d.nat);
  return CUW_OK;
}

// ---------------------------------------------------------------------------
// Init-time helpers restated for the harness checks.
// ---------------------------------------------------------------------------

// RANDOM_MSLNG (src/paw_generalpurpose.f90:2232-2256), explicit seed state
double orc_mslng(int* seed) {
  const int M = 2147483647, A = 16807, Q = 127773, R = 2836;
  int hi = *seed / Q, lo = *seed % Q;
  int test = A * lo - R * hi;
  *seed = (test > 0) ? test : test + M;
  return (double)(*seed) / (double)M;
}

// WAVES_INITIALIZERANDOM (src/paw_waves2.f90:2372-2492), TDETERMINISTIC branch
int orc_initializerandom(int ng, int ndim, int nb, const double* g, double* psi_out) {
  const int NRAN = 10000;
  std::vector<double> xran(NRAN);
  int seed = 1;
  for (int i = 0; i < NRAN; ++i) xran[i] = orc_mslng(&seed);
  const double GC2 = 3.0;
  const double rsmall = 100.0 * 2.2250738585072014e-308;
  double fac = 2.0 * std::sqrt(PI * GC2);
  fac = fac * fac * fac / (double)ndim * (2.0 / 3.0);
  fac = 1.0 / fac;
  std::vector<double> scale(ng), randarr(ng);
  for (int ig = 0; ig < ng; ++ig) {
    double g2 = g[3 * ig] * g[3 * ig] + g[3 * ig + 1] * g[3 * ig + 1] + g[3 * ig + 2] * g[3 * ig + 2];
    scale[ig] = fac * std::exp(-0.5 * g2 / GC2);
    double svar = 1.0 / std::sqrt(g2 + rsmall);
    double gx = 0.5 * (1.0 + svar * g[3 * ig]);
    double gy = 0.5 * (1.0 + svar * g[3 * ig + 1]);
    double gz = 0.5 * (1.0 + svar * g[3 * ig + 2]);
    double ran = xran[(int)(gx * (double)(NRAN - 1))];
    ran = xran[(int)(ran * gy * (double)(NRAN - 1))];
    ran = xran[(int)(ran * gz * (double)(NRAN - 1))];
    randarr[ig] = ran;
  }
  int ind = 0;  // 1-based index as in the reference
  cplx* psi = reinterpret_cast<cplx*>(psi_out);
  for (int ib = 0; ib < nb; ++ib)
    for (int idim = 0; idim < ndim; ++idim) {
      ind += 2;
      if (ind + 1 > NRAN) ind = 1;
      for (int ig = 0; ig < ng; ++ig) {
        double svar = 0.5 * (xran[ind - 1] * randarr[ig]);
        int isvar = 1 + (int)(svar * (double)NRAN);
        double rec = xran[isvar - 1];
        svar = 0.5 * (xran[ind] * randarr[ig]);
        isvar = 1 + (int)(svar * (double)NRAN);
        double rim = xran[isvar - 1];
        rec = 2.0 * rec - 1.0;
        rim = 2.0 * rim - 1.0;
        psi[(size_t)ig + (size_t)ng * (idim + (size_t)ndim * ib)] = cplx(rec, rim) * scale[ig];
      }
    }
  return CUW_OK;
}

// PLANEWAVE_COUNTG + PLANEWAVE_GETIG (src/paw_fft.f90:1110-1327) at Gamma with
// GBASS/BOXSPH (src/paw_generalpurpose.f90:72-180).  If igvec==NULL only the
// count is returned in *ng.
// WAVES_ORTHO_Y_C (src/paw_waves2.f90:1025-1338) on its own, for the tests:
// complex NB x NB matrices as (re, im) pairs in Fortran order, map = MAP
// (0-based) or null; returns CUW_ERR_NAN where the reference stops on a NaN.
int orc_ortho_y_c(int nb, const double* phiphi, const double* chiphi, const double* chichi, double* x,
                  const int* map) {
  if (nb <= 0 || !phiphi || !chiphi || !chichi || !x) return CUW_ERR_ARG;
  return ortho_y_c(nb, reinterpret_cast<const cplx*>(phiphi), reinterpret_cast<const cplx*>(chiphi),
                   reinterpret_cast<const cplx*>(chichi), reinterpret_cast<cplx*>(x), map);
}

int orc_getig(const double* gbas, double epw, int* ng, int* igvec) {
  // BOXSPH(GBAS,0,0,0,RAD)
  const double* t1 = gbas;      // GBAS(:,1)
  const double* t2 = gbas + 3;  // GBAS(:,2)
  const double* t3 = gbas + 6;  // GBAS(:,3)
  double g1[3], g2v[3], g3[3];
  g1[0] = t2[1] * t3[2] - t2[2] * t3[1];
  g1[1] = t2[2] * t3[0] - t2[0] * t3[2];
  g1[2] = t2[0] * t3[1] - t2[1] * t3[0];
  g2v[0] = t3[1] * t1[2] - t3[2] * t1[1];
  g2v[1] = t3[2] * t1[0] - t3[0] * t1[2];
  g2v[2] = t3[0] * t1[1] - t3[1] * t1[0];
  g3[0] = t1[1] * t2[2] - t1[2] * t2[1];
  g3[1] = t1[2] * t2[0] - t1[0] * t2[2];
  g3[2] = t1[0] * t2[1] - t1[1] * t2[0];
  double det = t1[0] * g1[0] + t1[1] * g1[1] + t1[2] * g1[2];
  for (int i = 0; i < 3; ++i) { g1[i] /= det; g2v[i] /= det; g3[i] /= det; }
  const double rad = std::sqrt(2.0 * epw) + 1e-6;
  double xn1 = std::sqrt(g1[0] * g1[0] + g1[1] * g1[1] + g1[2] * g1[2]) * rad;
  double xn2 = std::sqrt(g2v[0] * g2v[0] + g2v[1] * g2v[1] + g2v[2] * g2v[2]) * rad;
  double xn3 = std::sqrt(g3[0] * g3[0] + g3[1] * g3[1] + g3[2] * g3[2]) * rad;
  const int ibig = 1000000;
  int min1 = (int)(0.0 - xn1 + 1.0 + ibig) - ibig, max1 = (int)(0.0 + xn1 + ibig) - ibig;
  int min2 = (int)(0.0 - xn2 + 1.0 + ibig) - ibig, max2 = (int)(0.0 + xn2 + ibig) - ibig;
  int min3 = (int)(0.0 - xn3 + 1.0 + ibig) - ibig, max3 = (int)(0.0 + xn3 + ibig) - ibig;
  std::vector<int> iv;
  std::vector<double> g2a;
  for (int i = min1; i <= max1; ++i)
    for (int j = min2; j <= max2; ++j)
      for (int k = min3; k <= max3; ++k) {
        double a = (double)i, b = (double)j, c = (double)k;
        double x = gbas[0] * a + gbas[3] * b + gbas[6] * c;
        double y = gbas[1] * a + gbas[4] * b + gbas[7] * c;
        double z = gbas[2] * a + gbas[5] * b + gbas[8] * c;
        double gs = x * x + y * y + z * z;
        if (0.5 * gs > epw) continue;
        iv.push_back(i); iv.push_back(j); iv.push_back(k);
        g2a.push_back(gs);
      }
  const int n = (int)g2a.size();
  if (!igvec) { *ng = n; return CUW_OK; }
  if (*ng != n) return CUW_ERR_ARG;
  // order by increasing G^2 (SORT$), stable
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return g2a[a] < g2a[b]; });
  std::vector<int> ig(3 * (size_t)n);
  std::vector<double> g2s(n);
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) ig[3 * i + k] = iv[3 * order[i] + k];
    g2s[i] = g2a[order[i]];
  }
  // lexicographic order within shells (fft:1290-1325)
  auto swap3 = [&](int a, int b) { for (int k = 0; k < 3; ++k) std::swap(ig[3 * a + k], ig[3 * b + k]); };
  int istart = 0;  // 0-based
  double svar = g2s[istart];
  for (int igx = 1; igx < n; ++igx) {  // IG=2..NG  (1-based igx+1)
    bool last = (igx == n - 1);
    if (std::fabs(g2s[igx] - svar) < 1e-5 && !last) continue;
    int istop = igx - 1;
    if (last) istop = n - 1;
    for (int i = istart; i <= istop; ++i)
      for (int j = i + 1; j <= istop; ++j) {
        if (ig[3 * i] > ig[3 * j]) swap3(i, j);
        else if (ig[3 * i] == ig[3 * j]) {
          if (ig[3 * i + 1] > ig[3 * j + 1]) swap3(i, j);
          else if (ig[3 * i + 1] == ig[3 * j + 1]) {
            if (ig[3 * i + 2] > ig[3 * j + 2]) swap3(i, j);
          }
        }
      }
    if (istop == n - 1) break;
    istart = istop + 1;
    svar = g2s[istart];
  }
  std::memcpy(igvec, ig.data(), sizeof(int) * 3 * (size_t)n);
  return CUW_OK;
}

// PLANEWAVE$MINUSG (src/paw_fft.f90:1157-1208) at Gamma; minusg 1-based
int orc_minusg(int ng, const int* ig, int* minusg) {
  std::fill(minusg, minusg + ng, 0);
  std::map<long long, int> pos;
  auto key = [](int a, int b, int c) {
    return ((long long)(a + 100000) * 200001LL + (b + 100000)) * 200001LL + (c + 100000);
  };
  for (int i = 0; i < ng; ++i) pos[key(ig[3 * i], ig[3 * i + 1], ig[3 * i + 2])] = i;
  for (int i1 = 0; i1 < ng; ++i1) {
    if (minusg[i1] != 0) continue;
    auto it = pos.find(key(-ig[3 * i1], -ig[3 * i1 + 1], -ig[3 * i1 + 2]));
    if (it == pos.end() || it->second < i1) return CUW_ERR_ARG;
    minusg[i1] = it->second + 1;
    minusg[it->second] = i1 + 1;
  }
  return CUW_OK;
}

// LIB$FFTADJUSTGRD (src/paw_library.f90:2336-2393)
int orc_fftadjustgrd(int nr) {
  std::vector<int> ifr;
  for (int h = 1; h <= 25; ++h)
    for (int i = 0; i <= 2; ++i)
      for (int j = 0; j <= 1; ++j)
        for (int k = 0; k <= 1; ++k)
          for (int m = 0; m <= 1; ++m) {
            if ((int)ifr.size() >= 300) goto done;
            double s = std::pow(2.0, h) * std::pow(3.0, i) * std::pow(5.0, j) * std::pow(7.0, k) * std::pow(11.0, m);
            if (s > 37748736.0) continue;
            ifr.push_back((int)std::lround(s));
          }
done:
  std::sort(ifr.begin(), ifr.end());
  for (size_t i = 1; i < ifr.size(); ++i)
    if (ifr[i] >= nr) return ifr[i];
  return -1;
}

// Expose fft1d for the numpy cross-check
int orc_fft1d(int n, int dir, double* data) {
  FFTPlan P;
  plan_init(P, n, dir);
  std::vector<cplx> work;
  fft1d(P, reinterpret_cast<cplx*>(data), 1, work);
  return CUW_OK;
}

// Expose the symmetric eigensolver for the scipy cross-check
int orc_syev(int n, const double* a, double* e, double* u) {
  std::vector<double> aa(a, a + (size_t)n * n), ee, uu;
  jacobi_eig(n, aa, ee, uu);
  std::memcpy(e, ee.data(), sizeof(double) * n);
  std::memcpy(u, uu.data(), sizeof(double) * (size_t)n * n);
  return CUW_OK;
}

}  // extern "C"
