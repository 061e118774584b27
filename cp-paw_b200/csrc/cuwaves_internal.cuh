// Internal state and device helpers of the cuwaves engine (sm_100a).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/cuwaves.h"

namespace cuw {

// ---------------------------------------------------------------------------
// error handling: every CUDA call is checked and turned into a status code
// ---------------------------------------------------------------------------
struct Status {
  int code = CUW_OK;
  std::string msg;
};

#define CUW_TRY(expr)                                              \
  do {                                                             \
    cudaError_t e__ = (expr);                                      \
    if (e__ != cudaSuccess) {                                      \
      return h->fail(CUW_ERR_CUDA, std::string(#expr) + ": " +     \
                                       cudaGetErrorString(e__));   \
    }                                                              \
  } while (0)

#define CUW_LAUNCH_CHECK(name)                                      \
  do {                                                              \
    ++h->launches;                                                  \
    cudaError_t e__ = cudaGetLastError();                           \
    if (e__ != cudaSuccess)                                         \
      return h->fail(CUW_ERR_CUDA, std::string(name) + ": " +       \
                                       cudaGetErrorString(e__));    \
  } while (0)

#define CUW_RET(expr)            \
  do {                           \
    int r__ = (expr);            \
    if (r__ != CUW_OK) return r__; \
  } while (0)

// Projector descriptor: IPRO -> (atom, bare projector column, LM, L)
struct ProDesc {
  int iat;
  int ibare;
  int lm;
  int l;
};

// FFT plan of one grid axis: radix sequence of a Stockham transform
struct AxisPlan {
  int n = 0;
  int nstage = 0;
  int radix[8] = {0};
};

// Device arrays of one wave-function set.
struct Device {
  // wave functions (ld = ldg complex numbers per band)
  double2 *psi0 = nullptr, *psim = nullptr, *hpsi = nullptr, *opsi = nullptr;
  double2 *proj = nullptr;       // (NBH, NPRO)
  double2 *oproj = nullptr;      // (NBH, NPRO) scratch
  double2 *hproj = nullptr;      // (NBH, NPRO) scratch
  double2 *pbuf = nullptr;       // (NBH, NPRO) scratch
  double2 *rlam0 = nullptr;      // (NB, NB) complex, Fortran layout
  double2 *rlamm = nullptr;
  // g-set
  int *igvec = nullptr;          // (3, NGL)
  int *minusg = nullptr;         // (NGL) 0-based
  double *gx = nullptr, *gy = nullptr, *gz = nullptr, *g2 = nullptr;
  double *pro = nullptr;         // (NGL, NBAREPRO)
  double *ylm = nullptr;         // (NGL, LMX)
  double *mpsi = nullptr;        // (NGL)
  double *bucket = nullptr;      // (NGL) or null
  ProDesc *pdesc = nullptr;      // (NPRO)
  // FFT
  int *plane_iz = nullptr;       // (nzp) occupied z planes
  int2 *plane_rows = nullptr;    // (nzp) first row and row count of the plane's G vectors
  int *plane_off = nullptr;      // (nzp+1) CSR offsets of the G lists
  int *plane_g = nullptr;        // (NGL) G index, grouped by plane
  int *plane_pos = nullptr;      // (NGL) ix + NR1*iy of that G
  int *zslot = nullptr;          // (NR3) compact plane index or -1
  double *v = nullptr;           // (NR1*NR2*NR3) local potential
  void *grid = nullptr;          // (batch, nzp, NR2, NR1) work grid, double2 or float2 (mixed)
  double* rho = nullptr;         // (NR) pseudo density of cuwaves_density (allocated on first use)
  double2 *tw1 = nullptr, *tw2 = nullptr, *tw3 = nullptr;  // twiddles exp(+2 pi i k/n)
  // atoms and one-centre data
  double *r0 = nullptr, *rp = nullptr, *rm = nullptr;  // (3, NAT)
  double *force = nullptr;       // (3, NAT)
  double *mass = nullptr;        // (NAT)
  double2 *eigr = nullptr;       // (NGL, NAT) structure factors of the last position set
  float2 *pf = nullptr;          // (LDG, NPRO) mixed path: PRO(g,p) of the last position set in fp32, 0 for g >= NGL
  double2 *prox = nullptr;       // (LDG, NPRO) FP64 path: PRO(g,p) of the last position set, 0 for g >= NGL
  double2 *xminus[2] = {nullptr, nullptr};  // (LDG, NBH) mixed path: X(-G) copies of wave-function arrays
  float *bpre[2] = {nullptr, nullptr};       // mixed path: wave-function arrays split into tf32 B tiles
  const double2 *bpre_src[2] = {nullptr, nullptr};  // arrays they hold (valid inside a solve scope)
  float *bsmall = nullptr;                   // mixed path: small matrices split into tf32 B tiles (3 slots)
  double *jac_a = nullptr;                   // packed matrix of the eigensolver when NB is too large for shared memory
  size_t bsmall_slot = 0;                    // floats per slot
  double2 *dh = nullptr;         // (LMNXX, LMNXX, NAT)
  double *dover = nullptr;       // (LNXX, LNXX, NSP)
  double *occ = nullptr;         // (NB)
  // orthogonalisation (real NB x NB)
  double *mat = nullptr, *omat = nullptr, *oomat = nullptr;
  double *lam = nullptr, *lam2 = nullptr, *lam0 = nullptr;  // lam0: start of a solve that may be redone
  double *u = nullptr, *u2 = nullptr, *eig = nullptr;
  double *haux = nullptr, *gamn = nullptr, *work = nullptr, *wk2 = nullptr;
  double *smat = nullptr, *emat = nullptr, *gt = nullptr, *xb = nullptr, *tb = nullptr;
  double *maxpart = nullptr;
  int *ostatus = nullptr;        // [0] status, [1] iterations
  int *smap = nullptr;           // (NB) state order of WAVES_ORTHO_Y_C (SAFEORTHO = F, SWAPSTATES = T)
  double *anv = nullptr, *dbucket = nullptr;  // (NGL) ANNEEVEC and GSET%DBUCKET of the cell friction
  double2 *lam1c = nullptr, *lam2c = nullptr;  // (NBH, NBH) folded multipliers
  double2 *tmat = nullptr;       // 12 (NBH, NBH) reduced Gram products
  // scratch for split-K partial sums and band reductions
  double2 *part = nullptr;
  size_t part_bytes = 0;
  double *red = nullptr;         // reductions
  double *scal = nullptr;        // small scalar results
  // potential (POTENTIAL$VOFRHO): the density G set (one G of each +-G pair),
  // its tables and work arrays
  int *r_plus = nullptr, *r_minus = nullptr;   // (NGLH) grid offsets of +G and -G
  double *r_gx = nullptr, *r_gy = nullptr, *r_gz = nullptr, *r_g2 = nullptr;  // (NGLH)
  double *r_ylm = nullptr;                     // (LMRXX, NGLH) Y_lm(G) |G|^l
  double *r_g0 = nullptr, *r_v0 = nullptr, *r_pscore = nullptr, *r_vbar = nullptr;  // (NGLH, NSP)
  int *r_lmrx = nullptr;                       // (NSP)
  double *qlm = nullptr;                       // (LMRXX, NAT)
  double2 *r_rhog = nullptr, *r_vg = nullptr, *r_pot = nullptr, *r_vtot = nullptr;  // (NGLH)
  double2 *r_grid = nullptr;                   // (NR1*NR2*NR3) full complex grid
  double *r_part = nullptr;                    // block partial sums
  double *fpot = nullptr;                      // (3, NAT) Hartree and pseudo-core forces
  double *vqlm = nullptr;                      // (LMRXX, NAT)
  double *r_out = nullptr;                     // [0] EHARTREE [1] EXC [2] RHOB of the last cuwaves_vofrho
  // projector-map tables: first IPRO and #LMN per atom, species per atom,
  // (LN, M) of each IPRO, first LMN of each (species, LN), LOX (-1 = none)
  int *t_ipro0 = nullptr, *t_nlmn = nullptr, *t_isp = nullptr, *t_lnofp = nullptr, *t_mofp = nullptr,
      *t_lmn0ln = nullptr, *t_lox = nullptr;
};

struct Handle {
  cuw_dims d{};
  std::vector<int> isp;          // 0-based
  std::vector<int> lmnx, ibpro, ipro0;
  std::vector<ProDesc> pdesc;
  int npro = 0, nbarepro = 0, lmnxx = 0, lnxx = 0;
  int ldg = 0;                   // leading dimension of wave-function arrays
  double gweight = 0.0;
  double gbas[9] = {0};
  std::vector<int> igvec_h;      // IGVEC(3,NGL) of the G set (restart records)
  double delt = 0.0, annee = 0.0;
  bool have_gset = false, have_v = false, have_dh = false, have_do = false;
  bool have_hpsi = false, have_rlamm = false, have_opsi = false, have_u = false;
  bool tbucket = false;
  bool async = false;
  // page-locked host block of cuwaves_cp_step's results (8 sums, the 16 status
  // words, the forces): one copy each and one wait per step
  double* res_h = nullptr;
  int band_bps = 0;  // resident blocks per SM of the band-sum kernel (0: not yet queried)
  int nzp = 0;                   // occupied z planes
  int batch = 0;                 // bands per FFT batch
  int grid_bands = 0;            // bands the FFT work grid has room for
  // split-K factors of the projections and Gram products, as multiples of the
  // default (about two waves of CTAs); set by cuwaves_autotune
  double split_proj = 1.0, split_gram = 1.0;
  AxisPlan ax[3];
  int (*fft_run)(Handle*, const double2*, double2*, bool) = nullptr;  // chosen by fft_setup
  int (*fft_rho)(Handle*, const double2*, double*) = nullptr;          // density, chosen by fft_setup
  int fft_variant = 0;        // plan variant of the compiled FFT kernels (autotuner)
  int stream_prio = 0;        // 1: the stream has the device's highest priority
  bool fft_compiled = false;  // the grid has kernels compiled for its lengths
  size_t nr = 0;
  std::vector<double> occ_h;
  double waveekin1 = 0.0, waveekin2 = 0.0;
  cudaStream_t stream = nullptr;
  // nsm: SMs the launch shapes assume (the device's nsm_dev, or the share of a
  // set that runs beside others, CUW_OPT_SM_SHARE)
  int device = 0, nsm = 148, nsm_dev = 148;
  // CUDA graphs of cuwaves_cp_step.  A step's launches depend on host-side
  // state only through the PSI0/PSIM swap, the buffer EIGR was built from,
  // the Lagrange history flag and the arguments; one graph is kept per such
  // state (two in a run of steps).  `epoch` changes with every call that
  // could change what a step enqueues otherwise (inputs by value, scratch
  // reallocation, set-up routines), which retires the graphs.
  struct StepGraph {
    const void* key[6];
    int move = 0, max_iter = 0, rlamm = 0;
    double eps = 0.0;
    long long epoch = -1;
    const double* eigr_after = nullptr;  // EIGR's source buffer after the step
    long long launches = 0;              // kernels in the graph
    cudaGraphExec_t exec = nullptr;
  };
  std::vector<StepGraph> graphs;
  long long epoch = 0;
  bool use_graphs = true;
  bool capturing = false;
  long long graph_replays = 0;
  void touch() { ++epoch; }
  void drop_graphs() {
    for (StepGraph& sg : graphs)
      if (sg.exec) cudaGraphExecDestroy(sg.exec);
    graphs.clear();
  }
  // measurement: kernel launches, and per-phase device time of cuwaves_cp_step
  long long launches = 0;
  bool timing = false;
  static constexpr int kPhases = 11;
  double phase_ms[kPhases] = {0};
  long long phase_calls = 0;
  std::vector<cudaEvent_t> ev;
  std::vector<int> ev_phase;
  int nev = 0;
  bool mixed() const { return d.precision == CUW_PREC_MIXED; }
  bool fp64_only = false;  // contractions in FP64 even on the mixed path (start-up orthonormalisation)
  // mixed path: the contractions on FP64 DMMA tiles (64 x 64, m8n8k4) instead
  // of the split-tf32 tcgen05 tiles (128 x 128 x 8); set by the autotuner or
  // CUW_OPT_CONTRACTION_TILES
  bool dmma_tiles = false;
  bool tc_on() const { return mixed() && !fp64_only && !dmma_tiles; }
  // relative accuracy to which each ORTHO_X iteration solves its Lyapunov
  // equation (0: to rounding).  Measured on Si64 over 40 CP steps against the
  // solve to rounding: 1e-6 moves the FP64 total energy by 3e-12 Ha and the
  // forces by 1e-13 Ha/bohr with 40% of the sweeps; 1e-2 moves it by 6e-7 Ha
  // (1e-8 Ha/atom) and the forces by 1e-8 Ha/bohr with 16% of the sweeps, far
  // inside the mixed path's own error.
  double lyap_tol = 0.0;
  // WAVES$ORTHOGONALIZE branch (src/paw_waves1.f90:221-222): SAFEORTHO = T runs
  // WAVES_ORTHO_X, F runs WAVES_ORTHO_Y_C, in the order of the RLAM0 diagonal
  // when SWAPSTATES = T
  bool safeortho = true, swapstates = false;
  // cell friction of WAVES$PROPAGATE (cuwaves_set_cell_friction)
  bool fric_on = false, have_dbucket = false;
  double fricmat[9] = {0};
  double emass = 0.0, emasscg2 = 0.0;
  int lyap_max_sweeps = 64;  // sweeps per Lyapunov solve before the fixed point counts as failed
  bool ortho_panel = true;   // ORTHO_X by the panel-staged cluster kernel where it applies (64 < NB <= 128)
  bool tc_scope_open = false;
  const double* eigr_src = nullptr;  // position buffer (r0, rp or rm) that EIGR (and the fp32 table) was built from
  // potential: density G set size, LMRXX, index of G = 0 (-1: none), and
  // whether cuwaves_cp_step forms V(r) from the density first
  int nglh = 0, lmrxx = 0, ngamma = -1;
  bool have_rhoset = false, have_qlm = false, scf = false;
  Device g;
  std::string err;

  int fail(int code, const std::string& m) {
    err = m;
    return code;
  }
  int sync() {
    if (async) return CUW_OK;
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return fail(CUW_ERR_CUDA, std::string("stream: ") + cudaGetErrorString(e));
    return tc_status();
  }
  // error flag of the tensor-core pipelines (a bounded wait that ran out)
  int tc_status() {
    if (!mixed()) return CUW_OK;
    int f = 0;
    cudaError_t e = cudaMemcpy(&f, g.ostatus + 12, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(CUW_ERR_CUDA, std::string("status: ") + cudaGetErrorString(e));
    return tc_flag(f);
  }
  int tc_flag(int f) {
    if (mixed() && f) return fail(CUW_ERR_CUDA, "tensor-core pipeline: a bounded wait ran out");
    return CUW_OK;
  }
  // Copy of n bytes of caller input to the device, ordered on the handle's
  // stream after the work enqueued before it.  Synchronous mode waits for it;
  // asynchronous mode only enqueues (the runtime stages a pageable buffer
  // before the call returns; a page-locked one is read when the stream gets
  // there, so the caller keeps it unchanged until cuwaves_synchronize).
  cudaError_t h2d(void* dst, const void* src, size_t n, bool wait = true) {
    cudaError_t e = cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess && wait && !async) e = cudaStreamSynchronize(stream);
    return e;
  }
  // the wait of synchronous mode after copies enqueued with h2d(..., false)
  cudaError_t h2d_done() { return async ? cudaSuccess : cudaStreamSynchronize(stream); }
  // set-up calls (new G set, new buffers) wait for the work in flight first
  cudaError_t settle() { return async ? cudaStreamSynchronize(stream) : cudaSuccess; }
};

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // a * conj(b)
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// the same for float2 (FP32 transforms of the mixed-precision path)
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

// (-i)^l
__device__ __forceinline__ double2 mipow(int l) {
  switch (l & 3) {
    case 0: return make_double2(1.0, 0.0);
    case 1: return make_double2(0.0, -1.0);
    case 2: return make_double2(-1.0, 0.0);
    default: return make_double2(0.0, 1.0);
  }
}

// PRO(g,p) = Y_lm(g) P_ln(|g|) (-i)^l EIGR(g,a) generated from the tables
// (WAVES_EXPANDPRO, src/paw_waves1.f90:6070-6109)
__device__ __forceinline__ double2 pro_value(int g, int ngl, const ProDesc& d, const double* __restrict__ ylm,
                                             const double* __restrict__ pro, const double2* __restrict__ eigr) {
  double s = ylm[(size_t)g + (size_t)ngl * d.lm] * pro[(size_t)g + (size_t)ngl * d.ibare];
  double2 e = cmul(mipow(d.l), eigr[(size_t)g + (size_t)ngl * d.iat]);
  return make_double2(s * e.x, s * e.y);
}

// coefficients of the fused ADDPRO epilogues (see k_addpro)
struct StepCoef {
  double a1, a2, a3, oscale;
  // G-dependent friction of a moving cell (ANNEEVEC(G), src/paw_waves1.f90:
  // 6536-6540) or null; with it the propagation coefficients are formed per G
  // from fr[g] and dt2 = DELT^2 instead of a1, a2, a3
  const double* fr = nullptr;
  double dt2 = 0.0;
};

// FP64 tensor-core MMA, m8n8k4, A row-major / B column-major fragments:
//   a = A[lane>>2][lane&3], b = B[lane&3][lane>>2],
//   c[0..1] = C[lane>>2][2*(lane&3)+0..1]
__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

// host helpers implemented in the .cu files
int fft_setup(Handle* h, const int* igvec_host);
int fft_vpsi(Handle* h, const double2* psi, double2* out, bool add_kinetic);
int fft_density(Handle* h, const double2* psi, double* rho);
int grid_fft(Handle* h, double2* grid, int dir);  // full-grid FP64 transform, unscaled
int fft_set_variant(Handle* h, int v);  // FFT plan variant of the compiled kernels
int fft_variants(const Handle* h);
int vofrho_run(Handle* h, const double* rho_dev);  // POTENTIAL$VOFRHO on the device
int denmat_run(Handle* h, int lmnxx, double2* denmat, double2* edenmat);
int eigr_compute(Handle* h, const double* r_dev);
int proj_compute(Handle* h, const double2* psiA, double2* projA, const double2* psiB, double2* projB);
int addpro_run(Handle* h, int mode, const double2* hpc, const double2* opc);
int hproj_compute(Handle* h, const double2* proj, double2* out);
int oproj_compute(Handle* h, const double2* proj, double2* out);
int hoproj_compute(Handle* h, const double2* proj, double2* hout, double2* oout);
int gram_overlaps(Handle* h, double2* projP, double2* projO);
int ortho_solve(Handle* h, int max_iter, double eps);
int ortho_result(Handle* h, const int* st, int* iters);
int addopsi_run(Handle* h, double2* psibar, const double2* opsi, const double2* l1, const double2* l2);
int addoproj_run(Handle* h, double2* proj, const double2* oproj, const double2* l1, const double2* l2);
int lambda12_run(Handle* h, const double* lam_real, double2* l1, double2* l2);
int band_reduce(Handle* h, int what, double* out_host, double* eig_host);
int force_run(Handle* h, double* force_host);
int force_gemm(Handle* h, const double2* ded, double* force_dev);
int small_tables_setup(Handle* h);
int gemm_setup(Handle* h);
struct GramPair {
  const double2* x;
  const double2* y;
};
int gram_planewave(Handle* h, const GramPair* pairs, int npair, double2* dst);
int gram_projections(Handle* h, const GramPair* pairs, int npair, double2* dst);
int ensure_part(Handle* h, size_t bytes);  // split-K scratch h->g.part of at least `bytes`
// Raises (never lowers) the dynamic shared-memory limit of kernel fn on the
// current device.  The limit belongs to the function, so it is shared by all
// handles of the process: a handle of a smaller system must not lower the
// limit that a larger one launches with.
cudaError_t smem_allow(const void* fn, int bytes);
// split-precision (tf32 x3) tensor-core versions, used when precision is
// CUW_PREC_MIXED; same arguments and results as the FP64 functions above
int tc_setup(Handle* h);
int tc_pro_table(Handle* h);  // h->g.pf from h->g.eigr (mixed path)
// Split wave-function operands computed inside a scope are reused by later
// contractions of the same scope (the arrays do not change inside it).
void tc_scope(Handle* h, bool open);
int tc_proj(Handle* h, const double2* psi, double2* proj);
int tc_addpro(Handle* h, int mode, const double2* hpc, const double2* opc, const StepCoef& sc);
int tc_gram(Handle* h, const GramPair* pairs, int npair, bool minus, int nk, int nm, size_t sk, size_t sm,
            double scale, double2* dst);
int tc_addx(Handle* h, bool xminus, double2* out, const double2* x, const double2* l1, const double2* l2, int nm,
            int nn, int nk, size_t sxm, size_t sxk, size_t som, size_t son);
int tc_force(Handle* h, const double2* ded, double* fpart, int* ntile);
int propagate_run(Handle* h);
int opsi_scale_run(Handle* h);
int switch_lambda_run(Handle* h);
int gramschmidt_run(Handle* h, double2* psi, const double* r_dev);
int atoms_verlet_run(Handle* h, const double* mass_dev);

enum { ADDPRO_HPSI = 0, ADDPRO_OPSI = 1, ADDPRO_FUSED = 2 };
enum { RED_EKIN = 0, RED_WAVEKIN = 1, RED_EXPECT = 2 };

inline int ceil_div(int a, int b) { return (a + b - 1) / b; }

}  // namespace cuw
