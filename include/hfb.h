/*
 * hfb.h -- C ABI of libhfb, the B200 (sm_100a) implementation of the static
 * Skyrme HF+BCS iteration of jax-hfbfft.
 *
 * Every entry point takes plain device pointers, sizes and scalars, and a
 * CUDA stream (cudaStream_t passed as void*; NULL = legacy default stream).
 * Work is enqueued asynchronously; the return value is an hfb_status for the
 * launch itself.  Errors detected on the device (a Fermi level that is not
 * bracketed, a Jacobi sweep limit, a non-finite energy) are latched in the
 * context and read with hfb_device_status(), which synchronises the stream.
 *
 * Layouts (identical to the reference's arrays, C order):
 *   psi      [nst][2][nx][ny][nz]   complex (interleaved re,im), complex128
 *                                   for HFB_F64, complex64 for HFB_F32;
 *                                   neutron states first (levels.py:54)
 *   fields   [2][nx][ny][nz]        double   (rho, tau, chi, upot, ...)
 *   vectors  [2][3][nx][ny][nz]     double   (current, sdens, sodens, aq, ...)
 *   pot      [2][12][nx][ny][nz]    real of the precision: upot, bmass,
 *                                   v_pair, aq_xyz, spot_xyz, wlspot_xyz
 *                                   (written by hfb_skyrme, read by hfb_hpsi)
 *   matrices [2][nmax][nmax]        complex128, nmax = max(npsi)
 *
 * Grids must be cubic (nx == ny == nz) with n in {8, 16, 24, 32, 40, 48};
 * spacings may differ per axis.
 */
#ifndef HFB_H
#define HFB_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hfb_ctx_s* hfb_ctx_t;

enum hfb_status {
  HFB_OK = 0,
  HFB_ERR_ARG = 1,              /* bad argument / null pointer           */
  HFB_ERR_UNSUPPORTED_GRID = 2, /* grid size not compiled in             */
  HFB_ERR_CUDA = 3,             /* CUDA launch or runtime error          */
  HFB_ERR_NOT_BRACKETED = 4,    /* BCS particle number not bracketed on
                                   [-100, 100] (pairs.py:59 raises)      */
  HFB_ERR_NO_CONVERGENCE = 5,   /* Jacobi or Brent iteration limit       */
  HFB_ERR_NONFINITE = 6,        /* NaN / Inf in an energy or a norm      */
  HFB_ERR_ALLOC = 7,            /* device allocation failed              */
  HFB_ERR_TIMEOUT = 8           /* a bounded device wait ran out         */
};

enum hfb_precision { HFB_F64 = 0, HFB_F32 = 1 };

/* Skyrme force and pairing parameters; the derived b/C coefficients follow
 * forces.py:95-122 and are filled by the host (see hfb/forces.py). */
typedef struct hfb_force {
  double b0, b0p, b1, b1p, b2, b2p, b3, b3p, b4, b4p, power, slate;
  double h2m[2];           /* after the (A-1)/A scaling of static.py:87-88 */
  double h2ma;             /* unscaled 0.5*(h2m_n+h2m_p), forces.py:141   */
  double v0neut, v0prot, rho0pr;
  double Crho0, Crho1, Crho0D, Crho1D, Cdrho0, Cdrho1, Ctau0, Ctau1, CdJ0, CdJ1;
  int ipair;               /* 0 none, 5 VDI, 6 DDDI                        */
  int ex;                  /* Slater exchange on/off                        */
  int zpe;                 /* 1: c.m. correction 17.3/A^0.2                 */
  int pad_;
} hfb_force;

/* ---- set-up ------------------------------------------------------------ */
/* grids.py:66-138, coulomb.py:23-52: grid, dense derivative matrices and the
 * doubled-grid Coulomb Green's function (built on the device).  nstmax sizes
 * the scratch arena. */
int hfb_ctx_create(int nx, int ny, int nz, double dx, double dy, double dz, int periodic,
                   int nstmax, hfb_ctx_t* out);
int hfb_ctx_destroy(hfb_ctx_t ctx);
const char* hfb_status_string(int status);
/* Number of kernels this library has launched in the process. */
unsigned long long hfb_launch_count(void);
/* The CUDA error behind the last HFB_ERR_CUDA returned to this host thread
 * (code in *code when code is not NULL; 0 and "no CUDA error" if none). */
const char* hfb_last_cuda_error(int* code);
/* Latched device-side status (synchronises the stream), then clears it. */
int hfb_device_status(hfb_ctx_t ctx, void* stream, int* status_out);

/* Bound, in SM clock cycles, of any one wait inside the tensor-core kernels
 * (an MMA completion, a copy, another CTA's tile); default 2e9 (about one
 * second).  A wait that runs out latches HFB_ERR_TIMEOUT, the kernel waits
 * for its own MMAs, releases its tensor memory and returns, and the context
 * stays usable.  No counterpart in the reference (JAX has no device waits). */
int hfb_set_wait_limit(hfb_ctx_t ctx, long long cycles);
/* Single-precision hpsi kernel of this context: 0 bf16 three-term operands
 * on the tensor cores (two CTAs per SM), 1 tf32 three-term operands on the
 * tensor cores, 2 FFT line transforms on CUDA cores.  Grids the tensor-core
 * kernels do not serve (n < 24) always use 2.  Read at each launch; for an
 * autotuner choosing per grid and state count (no counterpart in the
 * reference). */
int hfb_set_hpsi_kernel(hfb_ctx_t ctx, int kind);
/* For tests of that path: the next single-precision tensor-core hpsi launch
 * on this context has its first CTA wait, before it takes any work, on a
 * device word nothing writes, so the wait runs out after the wait limit and
 * the launch ends with HFB_ERR_TIMEOUT latched (no counterpart in the
 * reference). */
int hfb_arm_timeout_probe(hfb_ctx_t ctx);

/* ---- levels.py --------------------------------------------------------- */
/* cderv{x,y,z}00 / 01 / 02 (levels.py:132-395) on nsp spinors.
 * kind 0: d1 only; 1: d1 and d2 (Nyquist kept); 2: d1 and d(B d1) with the
 * mean-B Nyquist term; axis 0,1,2 = x,y,z; bfield [nx][ny][nz] (kind 2). */
int hfb_cderv(hfb_ctx_t ctx, int prec, int kind, int axis, int nsp, const void* psin,
              const double* bfield, void* d1, void* d2, void* stream);
/* laplace (levels.py:398-437) on nsp spinors with per-spinor weights
 * wg[nsp], wguv[nsp]; v_pairmax scalar; e0inv = static.e0dmp. */
int hfb_laplace(hfb_ctx_t ctx, int prec, int nsp, const void* psin, const double* wg,
                const double* wguv, double v_pairmax, double e0inv, double h2ma, void* psout,
                void* stream);

/* ---- meanfield.py ------------------------------------------------------ */
/* hpsi01 (meanfield.py:41-159) batched over nst states; state s uses the
 * potentials of isospin (s >= nneut).  Any of pout / pout_mf / pout_del may
 * be NULL except that one of pout / pout_mf is required. */
int hfb_hpsi(hfb_ctx_t ctx, int prec, const void* pot, int nst, int nneut, const void* psi,
             const double* weight, const double* weightuv, void* pout, void* pout_mf,
             void* pout_del, void* stream);
/* skyrme (meanfield.py:164-391): all mean fields from the densities, the
 * Coulomb potential (if tcoul) and ecorrp (device scalar); also packs the
 * hpsi potentials into pot (precision prec). */
int hfb_skyrme(hfb_ctx_t ctx, const hfb_force* f, int tcoul, const double* rho, const double* tau,
               const double* chi, const double* current, const double* sdens, const double* sodens,
               double* upot, double* bmass, double* divaq, double* v_pair, double* aq, double* spot,
               double* wlspot, double* dbmass, double* wcoul, double* ecorrp, int prec, void* pot,
               void* stream);

/* ---- coulomb.py -------------------------------------------------------- */
/* poisson (coulomb.py:54-75): wcoul[nx][ny][nz] from the proton density. */
int hfb_poisson(hfb_ctx_t ctx, const double* rho_p, double* wcoul, void* stream);
/* Same result as hfb_poisson without allocating device memory during the
 * call (no counterpart in the reference), for callers that cannot let the
 * library allocate: applications whose device memory is entirely owned by
 * their own pool allocator, and latency-critical loops where an allocation
 * and the synchronisation it implies would stall.  The work buffer is a
 * fixed 4 MiB array inside the library (64^3 complex doubles), so the
 * Coulomb grid n2 must be at most 64^3: n <= 32 for a non-periodic grid
 * (n2 = 2n); every periodic grid a context accepts (n2 = n <= 48) fits.
 * Larger Coulomb grids return HFB_ERR_UNSUPPORTED_GRID.  Call it with the context's device current
 * (HFB_ERR_ARG otherwise).  The first call on each device looks up the
 * array's device address, so make that first call before any stream
 * capture.  All calls share the one buffer (it keeps the last call's
 * contents; each call rewrites all of it, padding zeros included): calls
 * that overlap on the GPU -- concurrent streams, host threads -- race and
 * must be serialised by the caller. */
int hfb_poisson_noalloc(hfb_ctx_t ctx, const double* rho_p, double* wcoul, void* stream);

/* ---- densities.py / inout.py ------------------------------------------- */
/* add_density (densities.py:177-234) over nst states (neutrons first).
 * If mix < 1, rho/tau/chi are blended as mix*new + (1-mix)*old in place
 * (static.py:1820-1823); current/sdens/sodens are always replaced.
 * sp_kinetic (optional, may be NULL) receives the per-state kinetic energy
 * of inout.py:129-132, computed from the same derivatives; h2m is a HOST
 * array of 2 doubles (neutron, proton). */
int hfb_add_density(hfb_ctx_t ctx, int prec, int nst, int nneut, const void* psi,
                    const double* wocc, const double* wguv, const double* pairwg,
                    const double* wstates, double mix, double* rho, double* chi, double* tau,
                    double* current, double* sdens, double* sodens, const double* h2m,
                    double* sp_kinetic, void* stream);
/* sp_properties kinetic part alone (inout.py:64-150); h2m host array [2]. */
int hfb_sp_kinetic(hfb_ctx_t ctx, int prec, int nst, int nneut, const void* psi,
                   const double* h2m, double* sp_kinetic, void* stream);

/* ---- static.py --------------------------------------------------------- */
/* harmosc (static.py:580-738): state s = Gaussian * x^i y^j z^k in spin
 * component c, normalised; qn is a DEVICE int array [nst][4] = (i, j, k, c).
 */
int hfb_harmosc(hfb_ctx_t ctx, int prec, int nst, const int* qn, double radinx, double radiny,
                double radinz, void* psi, void* stream);

typedef struct hfb_grstep_args {
  int nst, nneut;
  int tbcs;                /* forces.tbcs                                     */
  int use_lagrange;        /* (iteration > 1) and not tbcs  (static.py:99)   */
  int do_fluct;            /* mprint > 0 and iteration % mprint == 0         */
  int pad_;
  double x0dmp, e0dmp, h2ma, wxyz;
  const void* pot;         /* packed potentials [2][12][N]                    */
  const double* v_pair;    /* [2][N] double, for max(v_pair[iq])              */
  void* psi;               /* in/out                                         */
  void* hampsi;            /* out: h psi_old (unweighted)                    */
  void* hmfpsi;            /* out: h psi_new (unweighted); scratch before    */
  void* delpsi;            /* out (optional): v_pair psi_new                 */
  const void* lagrange;
  const double *wocc, *wguv, *pairwg, *wstates;
  double* sp_energy;       /* in: previous; out: <psi_old|h|psi_old>         */
  double* sp_efluct1;      /* in/out                                         */
  double* sp_efluct2;      /* in/out                                         */
  double* sums;            /* out [2]: sum(sp_efluct1), sum(wocc*wstates*denerg) */
  const double* x0dmp_dev; /* optional: a device double read in place of
                              x0dmp (the step size kept on the device by
                              hfb_step_control, so that iterations can be
                              replayed without the host)                  */
} hfb_grstep_args;
/* grstep (static.py:215-259) with grstep_helper / e0dmp_gt_zero / laplace. */
int hfb_grstep(hfb_ctx_t ctx, int prec, const hfb_grstep_args* a, void* stream);

typedef struct hfb_diag_args {
  int npsi[2];
  int nmax;                /* leading dimension of the matrices              */
  int diagonalize;         /* eigh of lambda (static.py:300-303)             */
  int construct;           /* construct_hfb_matrices vs lagrange update      */
  int ipair, tbcs, pad_;
  double wxyz;
  const void* psi;         /* in: states after the gradient step             */
  void* psi_out;           /* out: rotated states psi U (must not alias psi) */
  const void* hampsi;
  const void* hmfpsi;
  void* lagrange;          /* out                                            */
  const double* v_pair;    /* [2][N], delpsi = v_pair * psi_new (static.py:203) */
  const double *wocc, *wguv, *pairwg, *wstates;
  double* sp_norm;         /* out                                            */
  double* sp_energy;       /* out (construct)                                */
  double* deltaf;          /* out (construct, ipair != 0)                    */
  double* hmatrix;         /* complex [2][nmax][nmax]                        */
  double* gapmatrix;
  double* symcond;
  double* lambda_save;     /* in (construct == 0) / out                      */
  double* efluct;          /* out [4]: efluct1q[2], efluct2q[2]              */
} hfb_diag_args;
/* diagstep (static.py:261-461) with loewdin_orthonormalize (463-482) and
 * construct_hfb_matrices (484-577).  Works on both isospins (npsi[0]
 * neutron states first); each isospin block must have at most 166 states
 * (the Jacobi solver holds the packed matrix in one CTA's shared memory). */
int hfb_diagstep(hfb_ctx_t ctx, int prec, const hfb_diag_args* a, void* stream);

/* Building blocks of diagstep, exported for tests:
 * C_a = wxyz * Psi^H X_a for a in the mask (bit0 X=psi, bit1 X=hampsi,
 * bit2 X=hmfpsi, bit3 X=v_pair*psi), states [s0, s0+ns), out complex
 * [4][ns][ns].  Matrices 0, 2 and 3 are Hermitian in the iteration (one set
 * of vectors; h psi and v_pair psi with h, v_pair Hermitian) and are
 * computed on their upper triangle and mirrored. */
int hfb_gram(hfb_ctx_t ctx, int prec, int s0, int ns, int mask, const void* psi,
             const void* hampsi, const void* hmfpsi, const double* v_pair_iq, double wxyz,
             double* out, void* stream);
/* Hermitian eigensolver (cyclic Jacobi, FP64) on nb matrices a[nb][n][lda]
 * using their lower triangle; eigenvalues ascending in w[nb][n],
 * eigenvectors in the columns of v[nb][n][lda]; sweeps (optional device
 * int[nb]) receives the number of Jacobi sweeps each matrix took. */
int hfb_eigh(hfb_ctx_t ctx, int nb, int n, int lda, const double* a, double* w, double* v,
             int* sweeps, void* stream);
/* Hermitian eigensolver for matrices that are close to diagonal (the lambda
 * matrix of a gradient step in the basis of the previous eigenvectors):
 * iterative refinement from X = I with the (near-)degenerate clusters
 * diagonalised exactly, cyclic Jacobi when the refinement does not apply.
 * Same contract as hfb_eigh (lower triangle read, w ascending, columns of v
 * the eigenvectors); lda <= 256.  hfb_diagstep uses it for lambda, the
 * eigh of static.py:300-310 / 397-407. */
int hfb_eigh_near_diagonal(hfb_ctx_t ctx, int nb, int n, int lda, const double* a, double* w,
                           double* v, void* stream);

/* lastdiag (static.py:1072-1168): quasiparticle spectrum of one isospin
 * block after convergence.  hmatrix and gapmatrix are complex [nst][ldh]
 * (the block's corner of static.hmatrix / gapmatrix), wocc the nst BCS
 * occupations of the block's states, eferm one device double (that
 * isospin's Fermi energy), first the index of the block's first state in
 * the whole state array (its parity picks the time-reversal partner in the
 * lower-component coefficients).  Outputs: qp_energy[nst] ascending and
 * qp_norm[nst], the norm of each eigenvector's lower component.  The
 * reference passes nst = nneut / nprot and first = 0 / nneut; the Python
 * mirror passes the isospin's whole block (npsi, npmin) unless asked for the
 * reference's ranges. */
int hfb_lastdiag(hfb_ctx_t ctx, int nst, int ldh, const double* hmatrix, const double* gapmatrix,
                 const double* wocc, const double* eferm, int first, double* qp_energy, double* qp_norm,
                 void* stream);

/* hfb_natural (static.py:920-1070): configuration-space sub-iterations for
 * one isospin block of nst states starting at state index ``start``.
 * Matrices are the complex [2][ld][ld] static.hmatrix, gapmatrix, symcond,
 * lambda_save (block iq); per-state arrays are over all states.  The host
 * runs the reference's loop:
 *   hfb_natural_begin                    cm = I, damping, h and gap at entry
 *   for each sub-iteration:
 *     hfb_natural_step(last)             gradient step on cm, QR (LAPACK
 *                                        conventions), transformed h and gap,
 *                                        sp_energy (and deltaf with pairing)
 *     [BCS solve when pairing is on]
 *     hfb_natural_symcond                (not after the last) new symcond
 *   hfb_natural_end                      psi_out[block] = psi[block] cm,
 *                                        lagrange[block] = psi cm htran, the
 *                                        matrices of the block replaced
 * The work matrices live in the context between these calls: one sequence
 * at a time per context.  nst <= 256. */
typedef struct hfb_natural_args {
  int nst, ld, iq, start;  /* block size, matrix leading dim, isospin, first state */
  int ipair, pad_;
  double delstepbas, e0bas;
  double* hmatrix;         /* complex [2][ld][ld] */
  double* gapmatrix;
  double* symcond;
  double* lambda_save;
  double* sp_energy;       /* [nstmax] */
  double* deltaf;          /* [nstmax], may be NULL without pairing */
  const double* wocc;
  const double* wguv;
  const double* pairwg;
  const double* wstates;
} hfb_natural_args;
int hfb_natural_begin(hfb_ctx_t ctx, const hfb_natural_args* a, void* stream);
int hfb_natural_step(hfb_ctx_t ctx, const hfb_natural_args* a, int last, void* stream);
int hfb_natural_symcond(hfb_ctx_t ctx, const hfb_natural_args* a, void* stream);
int hfb_natural_end(hfb_ctx_t ctx, int prec, const hfb_natural_args* a, const void* psi, void* psi_out,
                    void* lagrange, void* stream);

/* State-vector algebra for the linear-response solver of the sensitivities
 * (no counterpart in the reference, which has no differentiation): sets of
 * nsp two-spinors laid out like psi, precision prec.
 *   hfb_state_dot:       *out (device double) = wxyz sum Re(conj(a) b)
 *   hfb_state_axpby:     y = a x + b y
 *   hfb_state_mul_field: y_s = field x_s, field [nx][ny][nz] double
 *   hfb_state_project:   v_j -= sum_i psi_i wxyz <psi_i | v_j> (np states
 *                        psi, nv states v; np * nv <= 10240)
 *   hfb_state_axpby_diag: y_s = a_s x_s + b y_s, a device double[nsp]
 *   hfb_rms_field:       field = scale (|r - cm|^2 - r0^2) on the centred
 *                        grid (cm host double[3]): the derivative of a point
 *                        rms radius r0 about cm with respect to the density,
 *                        with scale = 1 / (2 N r0) */
int hfb_state_dot(hfb_ctx_t ctx, int prec, int nsp, const void* a, const void* b, double* out, void* stream);
int hfb_state_axpby(hfb_ctx_t ctx, int prec, int nsp, double a, const void* x, double b, void* y, void* stream);
int hfb_state_mul_field(hfb_ctx_t ctx, int prec, int nsp, const double* field, const void* x, void* y,
                        void* stream);
int hfb_state_project(hfb_ctx_t ctx, int prec, int np, const void* psi, int nv, void* v, void* stream);
int hfb_state_axpby_diag(hfb_ctx_t ctx, int prec, int nsp, const double* a, const void* x, double b, void* y,
                         void* stream);
int hfb_rms_field(hfb_ctx_t ctx, const double* cm, double r0, double scale, double* field, void* stream);

/* Vector-Jacobian products of hpsi and of the densities (the reference
 * differentiates meanfield.py:41-159 and densities.py:237-330 with JAX's
 * reverse mode).  The bilinear form <a|h[P]|b> of hpsi is the integral of
 * each potential field times the pair density of (a, b) that hfb_add_density
 * computes (by polarisation), except for the Nyquist term of cderv02
 * (levels.py:314-330), -(pi/d)^2 mean_line(B) x_N / n on the Nyquist bin of
 * each line, x_N = sum_j (-1)^j x_j.  These two calls are that term:
 *   hfb_nyquist_pair:  field[iq][r] += sum_ax (pi/d_ax)^2 / n^2 *
 *                      sum_{s in iq} w[s] sum_spin Re(conj(a_N) b_N) over
 *                      the line through r along ax (the bmass cotangent
 *                      of the term); field device double [2][n^3]
 *   hfb_nyquist_apply: y_s += scale[s] sum_ax c_ax mean_line(field[iq(s)])
 *                      (-1)^j x_N, c_ax = -(pi/d_ax)^2 / n (the term with
 *                      B = field); y must not alias x
 * States s < nneut are neutrons (iq 0); w and scale are device double[nst]. */
int hfb_nyquist_pair(hfb_ctx_t ctx, int prec, int nst, int nneut, const void* a, const void* b, const double* w,
                     double* field, void* stream);
int hfb_nyquist_apply(hfb_ctx_t ctx, int prec, int nst, int nneut, const double* field, const double* scale,
                      const void* x, void* y, void* stream);

/* Step-size control and energy history on the device (the host loop of
 * static.py:1864-1878 moved to one device thread, so that iterations can be
 * replayed without host reads in between; no counterpart in the
 * reference).  After an iteration's energies: hist[*count] = *ehf and
 * *count += 1 while *count < max_hist; with ctl[5] != 0 the reference's
 * adaptation of the step size ctl[0] from E_bind and efluct (device double
 * [4]: efluct1 of each isospin, efluct2 of each isospin), with ctl[1..3] the
 * previous E_bind, efluct1, efluct2 and ctl[4] the minimum step. */
int hfb_step_control(hfb_ctx_t ctx, const double* ehf, const double* efluct, double* ctl, double* hist,
                     int* count, int max_hist, void* stream);

/* ---- pairs.py ---------------------------------------------------------- */
typedef struct hfb_pair_args {
  int npsi[2];
  int nneut, nprot;        /* particle numbers                               */
  int use_const_gap;       /* iteration <= 10 (pairs.py:135)                 */
  int pad_;
  double const_gap;        /* 11.2 / sqrt(A)                                  */
  double pair_cutoff[2], state_cutoff[2], softcut_range;
  const double* sp_energy;
  double *deltaf, *wocc, *wguv, *pairwg, *wstates;   /* in/out */
  double* out;             /* [5][2]: eferm, epair, avdelt, avdeltv2, avg     */
} hfb_pair_args;
/* pair (pairs.py:161-220): gap, Fermi level by Brent's method on [-100,100]
 * with xtol 1e-14 (pairs.py:59), soft cutoffs, v^2, uv and sums. */
int hfb_pair(hfb_ctx_t ctx, const hfb_pair_args* a, void* stream);

/* ---- energies.py / output.py ------------------------------------------- */
/* integ_energy (energies.py:90-306).  out (device) receives HFB_NE doubles
 * in the order of the HFB_E_* indices below (EHF and TKE are left for
 * hfb_sum_energy). */
enum {
  HFB_E_EHFT = 0, HFB_E_EHF0, HFB_E_EHF1, HFB_E_EHF2, HFB_E_EHF3, HFB_E_EHFLS, HFB_E_EHFLSODD,
  HFB_E_EHFC, HFB_E_ECORC, HFB_E_EHFINT, HFB_E_E3CORR, HFB_E_EZPE, HFB_E_EHF, HFB_E_TKE,
  HFB_E_CRHO0, HFB_E_CRHO1, HFB_E_CDRHO0, HFB_E_CDRHO1, HFB_E_CTAU0, HFB_E_CTAU1, HFB_E_CDJ0,
  HFB_E_CDJ1, HFB_E_CJ0, HFB_E_CJ1, HFB_NE
};
int hfb_energies(hfb_ctx_t ctx, const hfb_force* f, int tcoul, double mass_number,
                 const double* rho, const double* tau, const double* current,
                 const double* sdens, const double* sodens, const double* wcoul,
                 const double* epair, double* out, void* stream);
/* sum_energy (energies.py:309-372): out[HFB_E_EHF], out[HFB_E_TKE] from the
 * single-particle sums and out[E3CORR, ECORC, EZPE] of hfb_energies; epair
 * [2] and ecorrp [1] are device arrays. */
int hfb_sum_energy(hfb_ctx_t ctx, int nst, const double* wocc, const double* wstates,
                   const double* sp_kinetic, const double* sp_energy, const double* epair,
                   const double* ecorrp, double* out, void* stream);
/* Explicit derivatives of the integrated functional ehfint (energies.py:
 * 117-258) at fixed densities: out (device) receives HFB_NG doubles,
 * dE/db for the coefficients b0, b0p, b1, b1p, b2, b2p, b3, b3p, b4, b4p
 * (forces.py:95-107) and dE/dpower.  At a self-consistent solution the
 * energy is stationary in the states and occupations, so these (chained
 * with db/dt, db/dx, db/dW0) are the total derivatives of E_bind with
 * respect to the Skyrme couplings: the adjoint of the fixed point vanishes
 * for the energy itself.  No counterpart in the reference (its derivatives
 * would come from jax.grad of the functional). */
enum {
  HFB_G_B0 = 0, HFB_G_B0P, HFB_G_B1, HFB_G_B1P, HFB_G_B2, HFB_G_B2P, HFB_G_B3, HFB_G_B3P,
  HFB_G_B4, HFB_G_B4P, HFB_G_POWER, HFB_NG
};
int hfb_energy_grad(hfb_ctx_t ctx, const hfb_force* f, const double* rho, const double* tau,
                    const double* current, const double* sdens, const double* sodens,
                    double* out, void* stream);
/* Single-particle orbital angular momentum, spin and parity (sp_properties,
 * inout.py:64-150; the kinetic energy is hfb_sp_kinetic): orbital[nst][3],
 * spin[nst][3], parity[nst] FP64 on the device (any may be NULL, not all),
 * the orbital momentum about ``cm`` (host double[3], NULL for the origin),
 * derivatives from the dense spectral matrices (cderv01), FP64 sums for
 * FP64 or FP32 states.  Grids up to 64^3. */
int hfb_sp_properties(hfb_ctx_t ctx, int prec, int nst, const void* psi, const double* cm, double* orbital,
                      double* spin, double* parity, void* stream);
/* Quadrupole / principal-axis constraints (constraint.py:47-342; the
 * reference defines them but does not call them from its driver).  Field
 * kinds (constraint.py:126-184, stacked in this order): Q20 (1 field), Q22
 * (1), principal axes (6: xy, xz, yz, x, y, z).  Fields are masked by
 * 1 / (1 + exp((r - damprad) / dampgamma)), normalised by r0rms^2 A^(5/3),
 * act on both isospins alike and are stored [nc][n^3] FP64 on the device.
 *   hfb_constraint_fields     the fields of ``kinds`` (bitwise or)
 *   hfb_constraint_moments    out[c] = <Q_c> = dV sum Q_c (rho_n + rho_p),
 *                             out[nc + c] = |<Q_c^2> - <Q_c>^2 / N|,
 *                             out[2 nc] = N (device, 2 nc + 1 doubles)
 *   hfb_constraint_potential  upot_q -= sum lambda_c Q_c (FP64 [2][n^3]) and
 *                             the same on field 0 of the packed hpsi
 *                             potentials ``pot`` [2][12][n^3] in ``prec``
 *                             (either may be NULL); lambda: host [nc]
 *   hfb_constraint_correct    psi_s *= exp(wstates_s wocc_s (-sum qcorr_c
 *                             Q_c)) on both spin components; qcorr: host [nc]
 */
enum { HFB_CON_Q20 = 1, HFB_CON_Q22 = 2, HFB_CON_PRINCIPAL = 4, HFB_CON_MAX = 8 };
int hfb_constraint_fields(hfb_ctx_t ctx, int kinds, double mass_number, double r0rms, double damprad,
                          double dampgamma, double* fields, void* stream);
int hfb_constraint_moments(hfb_ctx_t ctx, int nc, const double* fields, const double* rho, double* out,
                           void* stream);
int hfb_constraint_potential(hfb_ctx_t ctx, int prec, int nc, const double* fields, const double* lambda,
                             double* upot, void* pot, void* stream);
int hfb_constraint_correct(hfb_ctx_t ctx, int prec, int nst, int nc, const double* fields, const double* qcorr,
                           const double* wocc, const double* wstates, void* psi, void* stream);
/* Point rms radii (output.py:187-226, 246): out[0..1] particle numbers,
 * out[2..3] rms per isospin, out[4] total rms. */
int hfb_rms(hfb_ctx_t ctx, const double* rho, double* out, void* stream);

/* Density part of the nuclear observables, calculate_complete_observables
 * (output.py:177-276) with calculate_isovector_dipoles (output.py:323-340):
 * particle numbers, centres of mass, summed currents (pcm; zero when
 * current == NULL), point rms radii and second moments about each isospin's
 * own centre of mass, quadrupole tensors Q_ij = sum (3 x_i x_j - delta_ij
 * r^2) rho dV, Q20 / Q22 from their eigenvalues, beta / gamma of the total
 * tensor, the isovector Q20 (q20T1, with the nucleon numbers nneut, nprot)
 * and the isovector dipole.  rho: [2][n^3] FP64; current: [2][3][n^3] FP64
 * or NULL; out: HFB_NOBS doubles on the device, laid out as below
 * (per-isospin arrays iq fastest, as the reference's (3, 2) shapes). */
enum {
  HFB_OBS_PNR = 0,        /* [2]          */
  HFB_OBS_CM = 2,         /* [3][2]       */
  HFB_OBS_PCM = 8,        /* [3][2]       */
  HFB_OBS_RMS = 14,       /* [2]          */
  HFB_OBS_X2M = 16,       /* [3][2]       */
  HFB_OBS_Q20 = 22,       /* [2]          */
  HFB_OBS_Q22 = 24,       /* [2]          */
  HFB_OBS_PNRTOT = 26,
  HFB_OBS_CMTOT = 27,     /* [3]          */
  HFB_OBS_RMSTOT = 30,
  HFB_OBS_X2MTOT = 31,    /* [3]          */
  HFB_OBS_Q20TOT = 34,
  HFB_OBS_Q22TOT = 35,
  HFB_OBS_Q20T1 = 36,
  HFB_OBS_BETA20 = 37,
  HFB_OBS_BETA22 = 38,
  HFB_OBS_BETA = 39,
  HFB_OBS_GAMMA = 40,     /* degrees      */
  HFB_OBS_DIPOLE = 41,    /* [3]          */
  HFB_OBS_QMAT = 44,      /* [3][3][2]    */
  HFB_NOBS = 62
};
int hfb_observables(hfb_ctx_t ctx, const double* rho, const double* current, double nneut, double nprot,
                    double* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* HFB_H */
