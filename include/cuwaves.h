/*
 * cuwaves.h -- C ABI of the B200 wavefunction engine for the CP-PAW WAVES object.
 *
 * One handle holds the device-resident state of ONE wave-function set of the
 * reference's WAVES_MODULE (one (k-point, spin) pair, src/paw_waves1.f90:176-193
 * WVSET_TYPE) together with its G-set (GSET_TYPE, :156-175) and projector map
 * (MAP_TYPE, :142-154).  The Fortran host selects a handle where the reference
 * calls WAVES_SELECTWV (src/paw_waves1.f90:252-276).
 *
 * Conventions (all identical to the reference's Fortran arrays):
 *  - arrays are column-major; complex numbers are pairs of doubles (COMPLEX(8));
 *  - PSI(NGL,NDIM,NBH), PROJ(NDIM,NBH,NPRO), RLAM0(NB,NB);
 *  - IGVEC(3,NGL) in the order of PLANEWAVE_GETIG (src/paw_fft.f90:1211-1327),
 *    MINUSG(NGL) 1-based (src/paw_fft.f90:1157-1208);
 *  - the real-space grid is x-fastest, NR1*NR2*NR3 (src/paw_fft.f90:2162-2174);
 *  - projector index IPRO runs over atoms, then LN, then M (src/paw_waves1.f90:6070-6109).
 *
 * Every entry point returns CUW_OK (0) or an error code; the message is
 * available from cuwaves_last_error.  The reference stops the program instead
 * (ERROR$STOP, src/paw_error.f90:221); a Fortran shim maps a nonzero status
 * onto ERROR$STOP.  Calls are synchronous on the handle's own CUDA stream
 * unless the handle was put into asynchronous mode with cuwaves_set_async.
 */
#ifndef CUWAVES_H
#define CUWAVES_H

#include <stddef.h> /* size_t */

#ifdef __cplusplus
extern "C" {
#endif

#define CUW_OK                 0
#define CUW_ERR_ARG            1  /* invalid argument or size */
#define CUW_ERR_CUDA           2  /* CUDA runtime error */
#define CUW_ERR_STATE          3  /* call out of order (e.g. propagate before hpsi) */
#define CUW_ERR_NOT_CONVERGED  4  /* orthogonalisation loop not converged */
#define CUW_ERR_DIVERGED       5  /* orthogonalisation loop diverged (max|overlap-1|>1e200) */
#define CUW_ERR_UNSUPPORTED    6  /* configuration outside the implemented path */
#define CUW_ERR_NAN            7  /* non-finite value detected */
#define CUW_ERR_NOMEM          8  /* device allocation failed */

#define CUW_PSI0 0   /* THIS%PSI0 */
#define CUW_PSIM 1   /* THIS%PSIM */
#define CUW_HPSI 2   /* THIS%HPSI */
#define CUW_OPSI 3   /* THIS%OPSI (mass-scaled O|psi0>, valid inside a step) */

#define CUW_PREC_FP64  0  /* every product in FP64 */
#define CUW_PREC_MIXED 1  /* FP32 FFT/V.psi, split-tf32 tensor-core contractions, FP64 solves */

#define CUW_MAXSP 16
#define CUW_MAXLN 8

typedef struct cuw_handle cuw_handle;

/* Sizes and projector map of one wave-function set (MAP_TYPE + WVSET sizes). */
typedef struct cuw_dims {
  int ngl;        /* #G vectors of the full sphere 0.5|G|^2 <= EPWPSI */
  int ndim;       /* spinor components; 1 is implemented */
  int nb;         /* #bands */
  int nbh;        /* #stored functions: (nb+1)/2 with tinv, else nb */
  int tinv;       /* 1: Gamma point, super wave functions (src/paw_fft.f90:35-55) */
  int nr1, nr2, nr3;  /* FFT grid */
  int nat;        /* #atoms */
  int nsp;        /* #species */
  int lmx;        /* #real spherical harmonics in YLM(NGL,LMX) */
  int precision;  /* CUW_PREC_* */
  int lnx[CUW_MAXSP];             /* MAP%LNX */
  int lox[CUW_MAXSP][CUW_MAXLN];  /* MAP%LOX(LN,ISP) stored as lox[isp-1][ln-1] */
  const int* isp;                 /* [nat] MAP%ISP, 1-based */
} cuw_dims;

/* Replaces the WVSET allocation of WAVES$INITIALIZE (src/paw_waves1.f90:1187-1450). */
int cuwaves_create(const cuw_dims* dims, cuw_handle** out);
int cuwaves_destroy(cuw_handle* h);
/* Copies the last error message (NUL-terminated, truncated to len); with
 * h == NULL, the message of the calling thread's last failed cuwaves_create. */
int cuwaves_last_error(const cuw_handle* h, char* buf, int len);
/* 0: every call waits for its work (default); 1: calls only enqueue, input
 * copies included (they run in stream order after the work enqueued before
 * them; a page-locked input buffer is read when the stream gets there, so it
 * stays unchanged until cuwaves_synchronize).  cuwaves_set_gset and
 * cuwaves_set_cell_friction wait for the work in flight in either mode. */
int cuwaves_set_async(cuw_handle* h, int async);
int cuwaves_synchronize(cuw_handle* h);

/* G-set of PLANEWAVE$INITIALIZE + WAVES_UPDATEGSET (src/paw_fft.f90:872-1110;
 * src/paw_waves1.f90:6237-6353): igvec(3,NGL), minusg(NGL) (1-based, required
 * when tinv), gbas(3,3) reciprocal lattice vectors (THIS%GBAS of PLANEWAVE),
 * gvec(3,NGL) and g2(NGL) as PLANEWAVE$GETR8A('GVEC'/'G2'),
 * pro(NGL,NBAREPRO) = GSET%PRO, ylm(NGL,LMX) = GSET%YLM, mpsi(NGL) = GSET%MPSI,
 * bucket(NGL) = GSET%BUCKET or NULL (no bucket potential), gweight = cell volume. */
int cuwaves_set_gset(cuw_handle* h, const int* igvec, const int* minusg,
                     const double* gbas, const double* gvec, const double* g2, const double* pro,
                     const double* ylm, const double* mpsi, const double* bucket,
                     double gweight);
/* Local potential V(r) on the FFT grid (the RHO argument of WAVES$HPSI, src/paw_waves1.f90:4793). */
int cuwaves_set_potential(cuw_handle* h, const double* v);
/* One-centre Hamiltonian DH(LMNXX,LMNXX,NAT) of this spin, complex (WAVES$HPSI argument). */
int cuwaves_set_dh(cuw_handle* h, int lmnxx, const double* dh);
/* One-centre overlap DO(LNXX,LNXX,NSP) as SETUP$GETR8A('DO') per species. */
int cuwaves_set_do(cuw_handle* h, int lnxx, const double* dover);
/* Atomic positions R(0) and R(+) (ATOMLIST 'R(0)', 'R(+)'), each (3,NAT). */
int cuwaves_set_atoms(cuw_handle* h, const double* r0, const double* rp);
/* Positions R(-), R(0), R(+) (each (3,NAT), any may be NULL) as ATOMLIST$GETR8A
 * 'R(-)', 'R(0)', 'R(+)' after the steps this handle has taken. */
int cuwaves_get_atoms(cuw_handle* h, double* rm, double* r0, double* rp);
/* Occupations OCC(NB) of this (k,spin) as WAVES_DYNOCCGETR8A('OCC'). */
int cuwaves_set_occ(cuw_handle* h, const double* occ);
/* DELT and ANNEE (friction) of WAVES_MODULE (src/paw_waves1.f90:216-218). */
int cuwaves_set_dynamics(cuw_handle* h, double delt, double annee);
/* G-dependent friction of WAVES$PROPAGATE for a moving cell (TSTRESS,
 * src/paw_waves1.f90:6524-6543, WAVES_DMPSI :6676-6711): fricmat(3,3) =
 * CELL$GETR8A('PSIANNEMAT'), emass and emasscg2 = EMASS and EMASSCG2 of
 * WAVES_MODULE, dbucket(NGL) = GSET%DBUCKET or NULL (zero).  The propagation
 * (cuwaves_propagate and the one inside cuwaves_cp_step) then uses
 * ANNEEVEC(G) = ANNEE - tr(FRICMAT)/2 - EMASS EMASSCG2 G.FRICMAT.G
 * (1 + DBUCKET(G)) in place of ANNEE, recomputed when ANNEE or the G set
 * change; the mass scaling of O|psi> in cuwaves_orthogonalize keeps ANNEE,
 * as the reference does (src/paw_waves2.f90:148-156).  fricmat = NULL
 * switches it off.  Needs cuwaves_set_gset first. */
int cuwaves_set_cell_friction(cuw_handle* h, const double* fricmat, double emass, double emasscg2,
                              const double* dbucket);

int cuwaves_upload_psi(cuw_handle* h, int which, const double* psi);
int cuwaves_download_psi(cuw_handle* h, int which, double* psi);
int cuwaves_get_proj(cuw_handle* h, double* proj);
int cuwaves_set_proj(cuw_handle* h, const double* proj);
int cuwaves_get_rlam0(cuw_handle* h, double* rlam0);
int cuwaves_set_rlam0(cuw_handle* h, const double* rlam0);

/* WAVES_GRAMSCHMIDT (src/paw_waves2.f90:2025-2177) of PSI0 or PSIM with atoms at r(3,NAT). */
int cuwaves_gramschmidt(cuw_handle* h, int which, const double* r);
/* WAVES$PROJECTIONS('PSI0') (src/paw_waves1.f90:2681-2726): PROJ = <p(R0)|PSI0>. */
int cuwaves_projections(cuw_handle* h);
/* WAVES$HPSI (src/paw_waves1.f90:4793-4916): HPSI = H|PSI0> from V, DH and PROJ. */
int cuwaves_hpsi(cuw_handle* h);
/* WAVES$EKIN without stress (src/paw_waves1.f90:2729-2954). */
int cuwaves_ekin(cuw_handle* h, double* ekin);
/* Expectation values <psi_n|H|psi_n> of WAVES$ETOT (src/paw_waves1.f90:2094-2123), eig(NB). */
int cuwaves_expectation(cuw_handle* h, double* eig);
/* WAVES_WAVEKINETIC (src/paw_waves1.f90:6713-6847); eig(NB) may be NULL. */
int cuwaves_wavekinetic(cuw_handle* h, double* ekin, double* eig);
/* WAVES$FORCE without stress (src/paw_waves1.f90:4570-4739), force(3,NAT). */
int cuwaves_force(cuw_handle* h, double* force);
/* WAVES_DENSITY (src/paw_waves1.f90:5377-5500) of this set at the Gamma point,
 * the term WAVES$RHO (:4068-4144) adds per (k-point, spin): the pseudo density
 * rho(NR1*NR2*NR3), x fastest, from PSI0 and the occupations.  No kinetic-energy
 * density (TRHOKIN). */
int cuwaves_density(cuw_handle* h, double* rho);
/* WAVES$DENMAT (src/paw_waves1.f90:2957-3134) of this set with WAVES_DENMAT
 * (:3331-3572): one-centre density matrix denmat and energy-weighted density
 * matrix edenmat (may be NULL), each (LMNXX,LMNXX,NAT) complex for one spin,
 * from PROJ, RLAM0 and the occupations. */
int cuwaves_denmat(cuw_handle* h, int lmnxx, double* denmat, double* edenmat);
/* The WAVES section of the restart file for this set, as WAVES$WRITE
 * (src/paw_waves2.f90:3058-3088) with WAVES_WRITEPSI (:3168-3357) and
 * WAVES_WRITELAMBDA (:3920-4040) write it for one k-point and spin: the
 * separator record, then NKPT/NSPIN/RBAS/NWAVE, the PSI header, XK and IGVEC,
 * PSI0 and PSIM of every super wave function, the LAMBDA header and RLAM0 (and
 * RLAMM once the handle holds it), as sequential unformatted Fortran records
 * (4-byte length markers).  rbas(3,3) = CELL T(0), or NULL to derive it from
 * the G set's GBAS.  cuwaves_read_restart reads such a section back as
 * WAVES_READPSI (:5147-5513) does for the same bands: G vectors are matched by
 * IGVEC in any order, those the file lacks start at zero; NWAVE = 1 sets
 * PSIM = PSI0.  PROJ is not in the file: call cuwaves_projections after
 * reading, as a run does at its first step.  A file of another band count or
 * layout is refused (CUW_ERR_ARG) before anything on the device changes. */
int cuwaves_write_restart(cuw_handle* h, const char* path, const double* rbas);
int cuwaves_read_restart(cuw_handle* h, const char* path);
/* WAVES$PROPAGATE without cell dynamics (src/paw_waves1.f90:6479-6592). */
int cuwaves_propagate(cuw_handle* h);
/* WAVES$ORTHOGONALIZE with SAFEORTHO=T at the Gamma point (src/paw_waves2.f90:11-494,
 * WAVES_ORTHO_X :1844-2022).  max_iter and eps replace the PARAMETERs MAX=200 and
 * EPS=1e-8; iters (may be NULL) receives the iteration count. */
int cuwaves_orthogonalize(cuw_handle* h, int max_iter, double eps, int* iters);
/* WAVES$SWITCH (src/paw_waves2.f90:2180-2317): PSI0<->PSIM, Lagrange extrapolation. */
int cuwaves_switch(cuw_handle* h);
/* WAVES$STOP (src/paw_waves1.f90:6445-6476): PSIM = PSI0, history of RLAM dropped. */
int cuwaves_stop(cuw_handle* h);

/* One Car-Parrinello time step in the order of TIMESTEP (src/paw_driver.f90:280-561)
 * for a fixed potential: energies and forces at R(0), H|psi>, Verlet propagation,
 * orthogonalisation at R(+), switch.  When move_atoms is nonzero the step also
 * advances the nuclei with the Verlet rule of ATOMS$PROPAGATE without friction,
 * R(+) = 2R(0) - R(-) + dt^2 F/M, using mass(NAT) in electron masses, and keeps
 * R(-), R(0), R(+) on the device; otherwise R(+) is the one last set.  out[8]
 * receives: [0] total energy sum_n f_n <psi_n|H|psi_n>, [1] kinetic energy,
 * [2] fictitious kinetic energy 0.5*(EKIN1+EKIN2), [3] ionic kinetic energy,
 * [4] orthogonalisation iterations, [5..7] zero, or with CUW_OPT_SELFCONSISTENT
 * EHARTREE, EXC and int V rho.  force (3,NAT) may be NULL. */
int cuwaves_cp_step(cuw_handle* h, int move_atoms, const double* mass,
                    int max_iter, double eps, double* out, double* force);
/* Resets the nuclear history so that R(-) = R(0) (start from rest). */
int cuwaves_reset_atoms(cuw_handle* h, const double* r0);
/* Single-point evaluation at PSI0 and R(0), the energy part of WAVES$ETOT
 * (src/paw_waves1.f90:2094-2123) with EKIN (:2790-2954) and FORCE
 * (:4570-4739): out[0] = sum_n f_n <psi_n|H|psi_n>, out[1] = kinetic energy,
 * force (3*NAT, may be NULL).  Nothing is propagated. */
int cuwaves_etot(cuw_handle* h, double* out, double* force);

/* Local potential from the density: POTENTIAL$VOFRHO (src/paw_potential.f90:
 * 324-485 with POTENTIAL_VOFRHO :487-895) at the Gamma point for one spin,
 * LDA (DFT type 2: local exchange + Perdew-Wang local correlation), without
 * stress, confining potential, pair potential or isolation.
 *
 * cuwaves_set_rhoset loads the density G set and the tables of
 * POTENTIAL_UPDATE (:250-320): the NGLH G vectors that PLANEWAVE$SUPFFT keeps
 * (one of each +-G pair, src/paw_fft.f90:1834-1838) as igvec(3,NGLH),
 * gvec(3,NGLH) and g2(NGLH); ylm(LMRXX,NGLH) = Y_lm(G)|G|^l
 * (POTENTIAL_YLMOFG, :1548-1616); g0, v0, pscore, vbar (NGLH,NSP) as
 * SETUP$GETFOFG gives 'G0', 'V0', 'PSCORE', 'VADD' (:300-309); lmrx(NSP).
 * The grid is the handle's FFT grid. */
int cuwaves_set_rhoset(cuw_handle* h, int nglh, const int* igvec, const double* gvec, const double* g2,
                       int lmrxx, const int* lmrx, const double* ylm, const double* g0, const double* v0,
                       const double* pscore, const double* vbar);
/* QLM(LMRXX,NAT): multipole moments of the one-centre densities (the QLM
 * argument of POTENTIAL$VOFRHO), kept for cuwaves_vofrho and the
 * self-consistent step. */
int cuwaves_set_qlm(cuw_handle* h, const double* qlm);
/* POTENTIAL$VOFRHO at R(0): from the pseudo density rho(NR1*NR2*NR3) (x
 * fastest; NULL: the density of PSI0, formed on the device as
 * cuwaves_density does) and QLM (NULL: the one last set), the local
 * potential V(r), which becomes the handle's potential as POTENTIAL$VOFRHO
 * overwrites RHO with it.  Outputs (each may be NULL): v(NR), e[3] =
 * {EHARTREE, EXC, RHOB}, force(3,NAT) the Hartree and pseudo-core forces,
 * vqlm(LMRXX,NAT) = dE/dQLM. */
int cuwaves_vofrho(cuw_handle* h, const double* rho, const double* qlm, double* v, double* e, double* force,
                   double* vqlm);

/* Orthonormality test of WAVES$ORTHOGONALIZE (its TTEST block,
 * src/paw_waves2.f90:421-460) for PSI0 at R(0), e.g. after cuwaves_cp_step:
 * projections of PSI0 formed afresh, mat(NB,NB) = <psi_i|O|psi_j> (plane-wave
 * plus one-centre overlap, real at the Gamma point; may be NULL) and
 * *maxdev = max_ij |mat(i,j) - delta_ij| (may be NULL).  The reference
 * diagonalises the matrix and stops when an eigenvalue is off 1 by more than
 * 1e-4; the caller applies its own bound.  Computed in FP64 on both precision
 * paths; PROJ and the step state are not changed. */
int cuwaves_overlap_check(cuw_handle* h, double* mat, double* maxdev);

/* Serving runtime (no counterpart in the reference, which runs one system per
 * program: PAW_DRIVER's time loop, src/paw_driver.f90:280-561).  A request
 * carries the complete input of one wave-function set, with the meanings and
 * layouts of cuwaves_set_gset, _set_potential, _set_dh, _set_do, _set_occ,
 * _set_dynamics and _upload_psi; the server copies every array at submission
 * unless the request is flagged CUW_REQ_BORROW.
 * nsteps = 0 asks for a single point (cuwaves_etot after Gram-Schmidt of psi at
 * r0); nsteps > 0 for that many cuwaves_cp_step calls starting from rest
 * (PSIM = PSI0), with the nuclei moving when mass (NAT) is given.  Requests are
 * admitted in submission order while the estimated device memory of all
 * admitted sets stays within hbm_budget bytes; nworkers host threads advance
 * the admitted sets one step at a time in round-robin order, each set on its
 * own CUDA stream, so that sets of different sizes share the GPU and a new
 * request starts as soon as memory is free.  A set's result does not depend on
 * what else the server runs (every reduction has a fixed order). */
typedef struct cuw_server cuw_server;
typedef struct cuw_request {
  cuw_dims dims;  /* dims.isp is copied */
  const int* igvec;
  const int* minusg;
  const double* gbas;
  const double* gvec;
  const double* g2;
  const double* pro;
  const double* ylm;
  const double* mpsi;
  double gweight;
  const double* v;
  int lmnxx;
  const double* dh;
  int lnxx;
  const double* dover;
  const double* r0;
  const double* occ;
  const double* psi;   /* starting PSI0 (complex NGL x NBH) */
  double delt, annee;
  int nsteps;
  const double* mass;  /* (NAT) electron masses, or NULL: fixed nuclei */
  int flags;           /* CUW_REQ_* */
} cuw_request;
/* The server reads the request's arrays in place instead of copying them at
 * submission; the caller keeps them unchanged until the request has finished. */
#define CUW_REQ_BORROW 1

int cuwaves_server_create(size_t hbm_budget, int nworkers, cuw_server** out);
/* At most max_active sets are admitted at a time (default 4 * nworkers): the
 * admitted sets share the workers in turn, so the cap trades throughput
 * (overlap on the device) against the latency of the sets already running. */
int cuwaves_server_set_max_active(cuw_server* s, int max_active);
/* CUW_ERR_NOMEM when the request alone exceeds the budget. */
int cuwaves_server_submit(cuw_server* s, const cuw_request* r, long long* id);
/* *done = 1 once the request has finished; then *status is its own CUW_* code,
 * out[8] the last cuwaves_cp_step (or cuwaves_etot: out[0..1]) output, force
 * (3,NAT) the forces of the last step and *latency_ms the time from submission
 * to completion.  Any output pointer may be NULL. */
int cuwaves_server_poll(cuw_server* s, long long id, int* done, int* status, double* out,
                        double* force, double* latency_ms);
int cuwaves_server_error(cuw_server* s, long long id, char* buf, int len);
/* Forgets a finished request. */
int cuwaves_server_release(cuw_server* s, long long id);
/* Blocks until every submitted request has finished; CUW_ERR_STATE if any failed. */
int cuwaves_server_wait_all(cuw_server* s);
/* out[0] completed, [1] failed, [2] p50 and [3] p99 latency in ms, [4] requests
 * completed per second between the first submission and the last completion,
 * [5] peak and [6] current admitted device bytes, [7] requests in the system,
 * [8] mean number of admitted sets, [9] maximum latency in ms.  n values. */
int cuwaves_server_stats(cuw_server* s, double* out, int n);
/* Finishes the steps in flight, releases every set and stops the workers. */
int cuwaves_server_destroy(cuw_server* s);

/* Batches (no counterpart in the reference, which steps one set per program;
 * its loops over sets, src/paw_waves1.f90:252-276 WAVES_SELECTWV, run them one
 * after another): many sets, of any sizes, advanced together by one CUDA
 * graph launch.  cuwaves_batch_step advances every set by TWO CP steps
 * (cuwaves_cp_step with the same arguments; after two steps PSI0 and PSIM are
 * back in their buffers, so one captured graph serves every later pair): each
 * set's launches stay on its own stream, forked from and joined to the batch's
 * stream, so the sets run concurrently on the device; the graph is captured
 * at the first call and again whenever a set's host-side state or inputs
 * changed.  Results are bit-identical to stepping each set alone.  Every set
 * must have taken one cuwaves_cp_step first (the eigenbasis and Lagrange
 * history exist), with timing and asynchronous mode off.  mass: one pointer
 * (NAT masses) per set, or NULL with move_atoms = 0.  out (may be NULL):
 * out[(i*2 + s)*8 + k] = output k of step s of set i, as cuwaves_cp_step.
 * The call returns when both steps of every set are done; on a failed
 * orthogonalisation it returns that set's status (cuwaves_batch_error tells
 * which set).  A set may belong to one batch at a time and must not be used
 * by another thread during cuwaves_batch_step. */
typedef struct cuw_batch cuw_batch;
int cuwaves_batch_create(cuw_handle* const* handles, int n, cuw_batch** out);
int cuwaves_batch_step(cuw_batch* b, int move_atoms, const double* const* mass, int max_iter, double eps,
                       double* out);
int cuwaves_batch_error(const cuw_batch* b, char* buf, int len);
int cuwaves_batch_destroy(cuw_batch* b);

/* Measurement hooks (no counterpart in the reference, whose TIMING$CLOCKON/OFF
 * clocks, src/paw_timing.f90:121-192, play this role on the CPU).
 * cuwaves_set_timing(h, 1) records CUDA events on the handle's stream at the
 * phase boundaries of cuwaves_cp_step and resets the accumulators;
 * cuwaves_get_timing returns the accumulated device time per phase in ms
 * (n <= 11: reductions, structure factors, forces, FFT/V.psi, H and O
 * back-projection with propagation, projections at R(+), Gram products,
 * orthogonality solve, rotation by Lambda, bookkeeping, and the density with
 * POTENTIAL$VOFRHO of a self-consistent step), the number of kernels
 * this handle has launched and the number of timed steps.
 * cuwaves_get_stream returns the handle's cudaStream_t. */
int cuwaves_set_timing(cuw_handle* h, int enable);
int cuwaves_get_timing(cuw_handle* h, double* ms, int n, long long* launches, long long* steps);
int cuwaves_get_stream(cuw_handle* h, void** stream);
/* Diagnostics of the orthonormality solve (no reference counterpart): out[0]
 * eigendecompositions of sym(CHIPSI) so far, out[1] Lyapunov fixed-point sweeps
 * so far, out[2] Jacobi sweeps of the last eigendecomposition, out[3] ORTHO_X
 * iterations of the last solve, out[4] solves whose fixed point in the earlier
 * eigenbasis converged too slowly and were redone after a rediagonalisation.
 * n values (at most 5) are written. */
int cuwaves_get_ortho_stats(cuw_handle* h, double* out, int n);
/* Tuning options (no reference counterpart).
 * CUW_OPT_LYAP_TOL: relative accuracy to which every ORTHO_X iteration solves
 * its Lyapunov equation S X + X S = Gamma (the reference solves it exactly by
 * diagonalising S).  0 = to rounding; default 1e-5 (FP64) and 1e-2 (mixed
 * precision).  The ORTHO_X loop itself still stops on
 * max|<psi|O|psi> - 1| < eps, so a looser inner solve changes the iteration
 * path, not the constraint that the result satisfies. */
#define CUW_OPT_LYAP_TOL 1
/* CUW_OPT_GRAPHS: 1 (default) replays cuwaves_cp_step as CUDA graphs, one for
 * each of the two PSI0/PSIM buffer states of a run of steps, captured on first use and
 * retired by any other call that changes what a step enqueues; 0 launches
 * every kernel from the host.  Results are bit-identical either way. */
#define CUW_OPT_GRAPHS 2
/* CUW_OPT_LYAP_MAX_SWEEPS: sweeps of the Lyapunov fixed point before it counts
 * as failed and the solve is redone after a rediagonalisation (default 64). */
#define CUW_OPT_LYAP_MAX_SWEEPS 3
/* CUW_OPT_SELFCONSISTENT: 1 makes cuwaves_cp_step self-consistent in the order
 * of TIMESTEP (src/paw_driver.f90:280-561): the density of PSI0 and
 * POTENTIAL$VOFRHO (cuwaves_vofrho, with the QLM of cuwaves_set_qlm) give the
 * potential of the step's H|psi> before the forces, which gain the Hartree and
 * pseudo-core terms; out[0] becomes sum_n f_n <psi_n|H|psi_n> - int V rho +
 * EHARTREE + EXC, and out[5..7] = EHARTREE, EXC, int V rho.  Needs
 * cuwaves_set_rhoset and cuwaves_set_qlm first; 0 (default) keeps V fixed. */
#define CUW_OPT_SELFCONSISTENT 4
/* CUW_OPT_FFT_VARIANT: plan variant of the FFT transforms, 0 (default),
 * 1 (16 values per thread and stage), 2 (radix stages in ascending order) or,
 * on 64^3 grids, 3 (the z transforms exchange values between lanes by warp
 * shuffles instead of shared memory); grids without compiled kernels accept 0
 * only (CUW_ERR_UNSUPPORTED).  The autotuner picks it by timing. */
#define CUW_OPT_FFT_VARIANT 5
/* CUW_OPT_STREAM_PRIORITY: 0 (default) or 1: the handle's work runs on a
 * stream of the device's lowest or highest scheduling priority (the stream is
 * replaced after the work in flight; results do not change).  The serving
 * runtime gives its longest requests the high priority. */
#define CUW_OPT_STREAM_PRIORITY 6
/* CUW_OPT_SAFEORTHO: SAFEORTHO of WAVES_MODULE (src/paw_waves1.f90:221, used
 * in WAVES$ORTHOGONALIZE, src/paw_waves2.f90:306-386).  1 (default) solves the
 * constraint with WAVES_ORTHO_X; 0 with WAVES_ORTHO_Y_C (:1025-1338) of the
 * overlap matrices, which orthonormalises the states one after another and
 * needs no iteration (cuwaves_orthogonalize reports 0 iterations).
 * CUW_OPT_SWAPSTATES: SWAPSTATES (:222), 0 (default) or 1; with SAFEORTHO = 0
 * the states are taken in the ascending order of the RLAM0 diagonal.  A NaN in
 * ORTHO_Y_C returns CUW_ERR_NAN ("NAN DETECTED"), a failed state order
 * CUW_ERR_STATE ("STATE ORDERING FAILED"). */
#define CUW_OPT_SAFEORTHO 7
#define CUW_OPT_SWAPSTATES 8
/* CUW_OPT_CONTRACTION_TILES (mixed precision only): tile family of the
 * projector, Gram, rotation and force contractions, 0 (default) = split-tf32
 * tcgen05 tiles of 128 x 128 x 8, 1 = FP64 DMMA tiles of 64 x 64 x 4 (more
 * accurate; wins when few bands leave the wide tiles mostly empty).  The
 * autotuner picks it by timing. */
#define CUW_OPT_CONTRACTION_TILES 9
/* CUW_OPT_SM_SHARE: the number of SMs that this set's launch shapes assume
 * (the split-K factors of the contractions, the persistent force kernel, the
 * grid-stride loops); 0 (default) = every SM of the device.  A set stepped in
 * a batch of k sets can take about (SM count)/k, so that the sets' kernels
 * share the device instead of each launching enough blocks to fill it.  Other
 * split-K factors change summation orders at rounding level; the autotuner
 * keeps its choices per share. */
#define CUW_OPT_SM_SHARE 10
int cuwaves_set_option(cuw_handle* h, int option, double value);
/* Step graphs held now and graph replays so far (CUW_OPT_GRAPHS). */
int cuwaves_get_graph_stats(cuw_handle* h, long long* graphs, long long* replays);
/* Autotuner (no reference counterpart; FFTW's planner picks the reference's
 * FFT plans, src/paw_library.f90:2694-2697): times the FFT plan variant of the
 * plane transforms (values per thread and stage, radix order; grids with
 * compiled lengths) together with the FFT band batch, on mixed-precision
 * handles the tile family of the contractions (CUW_OPT_CONTRACTION_TILES),
 * and the split-K factors of the projections and plane-wave Gram products, on
 * this handle's data (G set, V, DH, DO and PSI0/PSIM loaded) and keeps the
 * fastest, in a process-wide table keyed by the shape so that later handles of
 * the same shape reuse it.  out[0..10] (n values): batch, projection split
 * factor, Gram split factor, their best times in ms, 1 if the choice came from
 * the table, FFT plan variant, tile family (1 = DMMA), the timed contraction
 * set's ms on tcgen05 and on DMMA tiles (0 on FP64 handles).  Results move at
 * rounding level (another summation order) or, with the tile family, at the
 * mixed path's precision. */
int cuwaves_autotune(cuw_handle* h, double* out, int n);
/* Check of the split-precision tensor-core product (no reference
 * counterpart): C(M,N) = A(M,K) * B(N,K)^T on device buffers, FP64 row-major
 * with K contiguous, computed as three tf32 tcgen05 products (hi*hi + hi*lo +
 * lo*hi) with fp32 accumulation.  *err (device int) becomes 1 if a bounded wait
 * inside the kernel ran out.  Work is enqueued on `stream`. */
int cuwaves_tc_gemm_check(int M, int N, int K, const double* A, const double* B, double* C, int* err,
                          void* stream);

/* Projections without any device allocation: PROJ(b,p) = gweight * sum_G
 * conj(PRO(G,p)) psi(G,b), the contraction of cuwaves_projections, for callers
 * that cannot call cudaMalloc (memory handed out only by a host pool, code
 * running under another program's memory cap or inside its stream capture).
 * There is no counterpart in the reference.
 * Every argument is a device pointer the caller owns:
 *   psi(ldg,nbh) complex, pdesc(4,npro) int (0-based atom, column of pro, LM, L
 *   of each projector), ylm(ngl,LMX), pro(ngl,NBAREPRO), eigr(ngl,nat) complex
 *   exp(-iG.R), proj(nbh,npro) complex output; stream is a cudaStream_t (NULL:
 *   the default stream).  Work is only enqueued on `stream`.
 * Its split-K partial sums use one static device array of 4 MiB, so nbh*npro
 * may not exceed 262144 (CUW_ERR_ARG otherwise).  The first call on a device
 * looks the array's address up (cudaGetSymbolAddress), which loads this
 * library's device code there and commits the 4 MiB on that device, where it
 * stays until the process exits: it must fit the caller's memory cap, and that
 * first call should come before any stream capture.  An error already pending
 * on the calling thread is reported (CUW_ERR_CUDA) and left in place.  All
 * calls share the array: calls that overlap on the GPU race. */
int cuwaves_projections_noalloc(int ngl, int ldg, int nbh, int nat, int npro, const double* psi,
                                const int* pdesc, const double* ylm, const double* pro,
                                const double* eigr, double gweight, double* proj, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CUWAVES_H */
