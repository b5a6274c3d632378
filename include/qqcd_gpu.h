/* qqcd_gpu.h -- C ABI of the B200 solver library for the qqcd hot path.
 *
 * Every entry point takes plain pointers and sizes, returns an int status (never
 * aborts) and mirrors one routine of the reference Fortran modules diracops,
 * inverters, quark and disconloops.  Array arguments use the reference's own
 * Fortran layouts (column-major, 1-based in the comments below):
 *
 *   Dirac half-vector  g(6, ntotal, 4, 2, 8)   real(8)   Q/diracops.f90:41-59
 *   Gauge field        u(18, ntotal, 4, 2, 16) real(8)   Q/diracops.f90:312-313
 *
 * with nvhalf = nx*ny*nz*nt/32 and ntotal = nvhalf + nbmax (one process, nps = 1,
 * basics.f90:20-31).  Pointers may be host or device memory (detected with
 * cudaPointerGetAttributes); host arrays are staged through the library's own device
 * buffers.  Calls on one context are stream ordered and return after the result is
 * complete.  One context per host thread.
 */
#ifndef QQCD_GPU_H
#define QQCD_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define QQ_OK 0
#define QQ_NOT_CONVERGED 1
#define QQ_NAN 2
#define QQ_BAD_ARG 3
#define QQ_CUDA_ERR 4
#define QQ_ABORTED 5
#define QQ_NO_DEVICE 6
#define QQ_SINGULAR 7

typedef struct qq_ctx qq_ctx;
typedef struct qq_defl qq_defl;

/* Lattice geometry and action coefficients.  Replaces the compile-time latdims
 * (U/latdims.f90:61-70), bc (U/cfgspropsmain.f90:334-337) and the fermion part of
 * coact (G/lattice.f90:426-429): c1[mu] = coact(3,1,mu), c2[mu] = coact(3,2,mu). */
typedef struct qq_geom {
  int nx, ny, nz, nt; /* each a multiple of 4 (latdims.f90:11-13) */
  int bc[4];          /* 1 periodic, -1 antiperiodic, 0 fixed */
  double c1[4];
  double c2[4];
} qq_geom;

/* Per-solve report (replaces the CFGSPROPS.LOG lines of the reference). */
typedef struct qq_solve_info {
  int status;
  int itercount;      /* Krylov iterations, as the reference counts them */
  int mvp;            /* applications of the even-odd operator */
  int ncycles;
  double true_rel;    /* ||phi - A x|| / ||phi|| on the even system, FP64 */
  double seconds;     /* device time of the solve */
  int nhist;          /* per-cycle true relative residuals (gmresdr-norm lines) */
  double hist[1024];
  int hist_mvp[1024];
  int nritz;          /* harmonic Ritz values of the last restart (re, im) */
  double ritz[2 * 512];
  int fallback;       /* qq_fgmres: 1 if plain GMRES-DR took over from a stalled cycle;
                        qq_fermprop_batch: nonzero if the batched BiCGStab stopped short of
                        the tolerance and plain FP64 GMRES-DR(m, k) finished this
                        right-hand side (from the BiCGStab's solution when it is finite and
                        better than zero): 1 a non-finite value, 2 a breakdown (rho,
                        <rhat, v>, ||t|| or omega vanished), 3 a stall (the true residual
                        did not fall 10x within qq_method.stall_window iterations),
                        4 the iteration limit */
  int finished_by;    /* qq_fermprop_batch: what finished this right-hand side -- 0 the batched
                        BiCGStab in the requested precision, 32 the batched FP32 BiCGStab
                        after a 16-bit one stopped short (fallback holds why), 64 plain
                        FP64 GMRES-DR(m, k) */
  int restarts;       /* qq_fermprop_batch: restarts of the batched BiCGStab after a breakdown
                        (the re-inserted residual became the shadow residual) */
} qq_solve_info;

/* ---- context ---- */
int qq_ctx_create(const qq_geom* geom, int device, qq_ctx** out);
int qq_ctx_destroy(qq_ctx* ctx);
/* Reference array sizes: nvhalf and ntotal of basics.f90:23-31. */
int qq_ctx_dims(const qq_ctx* ctx, int* nvhalf, int* ntotal);
/* Text of the last error on this thread. */
const char* qq_last_error(void);
/* Replace coact(3,1,:), coact(3,2,:) (fermpropR's r = -1 flip, Q/quark.f90:921-926). */
int qq_set_coact(qq_ctx* ctx, const double c1[4], const double c2[4]);

/* ---- gauge field ----
 * u_ref: reference u(18,ntotal,4,2,16).  recon: 18, 12, or 0 = choose 12 when every
 * link's third row equals conj(row1 x row2) to 1e-12, else 18.  Also builds the
 * FP32 recon-12 copy used by the mixed-precision solvers. */
int qq_gauge_upload(qq_ctx* ctx, const double* u_ref, int recon);

/* Quenched SU(3) configuration on the GPU: Wilson plaquette action at `beta`,
 * cold start, `nsweeps` Cabibbo-Marinari / Kennedy-Pendleton heatbath sweeps with a
 * counter-based generator seeded by `seed`.  Replaces the configuration-producing
 * part of the reference's generator (G/heatbath.f90 phbup :33-76 driven from
 * C/cfgsprops.f90 sweep :1973-2001); the reference's sequential random stream cannot
 * be reproduced in parallel, so the ensemble is equivalent, not the configuration.
 * Writes u_ref (reference u(18,ntotal,4,2,16), host or device; may be NULL), the
 * average plaquette (1/3) Re Tr U_p into *plaq (may be NULL), and uploads the
 * configuration as the context's gauge field (recon 12). */
int qq_heatbath(qq_ctx* ctx, double beta, int nsweeps, unsigned long long seed, double* u_ref,
                double* plaq);

/* ---- Dirac operator (Q/diracops.f90) ---- */
/* Hsingle :554-599.  gout = H_eo gin (gblclr = 1) or H_oe gin (gblclr = 2).
 * idag = 1 flips the sign of gamma_mu (H^dagger).  gout's halo slots are zeroed;
 * gin's halo slots are neither read nor written. */
int qq_hsingle(qq_ctx* ctx, double* gout, const double* gin, int idag, int gblclr);
/* Hdouble :264-346.  he = (1/kappa^2 - H_eo H_oe) ge. */
int qq_hdouble(qq_ctx* ctx, double* he, const double* ge, int idag, double kappa);
/* Hdbletm :435-550, iflag = -1 (Wilson / twisted mass; the clover branch iflag = -2
 * is out of scope and returns QQ_BAD_ARG).  kappa[0] = kappa, kappa[1] = mu. */
int qq_hdbletm(qq_ctx* ctx, double* he, const double* ge, int idag, const double kappa[2],
               int iflag);
/* twMshift :1863-1995, iflag = -1.  gwhole/hwhole hold the gblclr = 1 half followed
 * by the gblclr = 2 half (each 6*ntotal*64 doubles). */
int qq_twmshift(qq_ctx* ctx, double* hwhole, const double* gwhole, int idag,
                const double kappa[2], int iflag);
/* gamma5mult :1750-1860, iflag = -1: he = -i gamma5 [(1 + 2 i kappa mu gamma5)/kappa^2
 * - H_eo (1 - 2 i kappa mu gamma5) H_oe / (1 + 4 kappa^2 mu^2)] ge / (2 kappa mu),
 * even half in, even half out; kappa[0]*kappa[1] must not be 0. */
int qq_gamma5mult(qq_ctx* ctx, double* he, const double* ge, int idag, const double kappa[2],
                  int iflag);
/* vecdot Q/inverters.f90:13485-13530: adb = sum a^dagger b (FP64). */
int qq_vecdot(qq_ctx* ctx, const double* a, const double* b, double adb[2]);
/* No counterpart in the reference: vecdot for callers that must not allocate device
 * memory (a host code that has committed the device to its own preallocated field
 * arrays, or a solver loop where cudaMalloc/cudaFree would synchronise the device).
 * a and b: reference-layout half-vectors in device memory of this context's device
 * (16-byte aligned; host arrays are rejected, since staging them needs a buffer);
 * adb: host or device memory.  Reduction partials live in a fixed 128 KiB static
 * device array, which bounds the lattice at 4,194,304 sites (QQ_BAD_ARG above that).
 * The first call on a device looks that array up (cudaGetSymbolAddress) and should
 * precede any stream capture.  Calls that overlap on one device race on the array. */
int qq_vecdot_noalloc(qq_ctx* ctx, const double* a, const double* b, double adb[2]);

/* ---- inverters (Q/inverters.f90) ----
 * The deflation handle replaces the module variables of Q/shift.f90 (vtemp, hcnew,
 * beg) and Q/gmresrhs.f90 (isignal) that carry the GMRES-DR eigenvectors to
 * GMRES-Proj. */
int qq_defl_create(qq_ctx* ctx, int nmax, int kmax, qq_defl** out);
int qq_defl_destroy(qq_defl* d);
/* Number k of deflation vectors held (0 before a GMRES-DR solve). */
int qq_defl_size(const qq_defl* d);
/* Deflation vector j (0..k: the first k span the harmonic Ritz vectors of the last
 * restart, the reference's vtemp(:,1:k+1), Q/shift.f90) as a reference-layout even half
 * vector v (host or device).  No counterpart routine in the reference, which keeps them
 * in the shift module; the learned preconditioner trains on these low modes. */
int qq_defl_vector(const qq_defl* d, int j, double* v);

/* gmresdr :2871-3572.  Solves Hdbletm x = phi.  GMRES[0] = n, GMRES[1] = k.
 * x: initial guess on entry, solution on exit.  defl (optional) receives the k+1
 * deflation vectors and the (k+1) x k projected matrix. */
int qq_gmresdr(qq_ctx* ctx, const double* phi, double* x, const int GMRES[2], double resmax,
               int itermin, const double kappa[2], int iflag, qq_defl* defl,
               qq_solve_info* info);
/* gmresproject :7183-8304 with sigma = 0: GMRES(GMRES[0]) cycles, each preceded by
 * a minimum-residual projection over the k = GMRES[1] deflation vectors of defl.
 * The initial guess is zero, as in the reference. */
int qq_gmresproj(qq_ctx* ctx, const double* b, double* x, const int GMRES[2], double resmax,
                 int itermin, const double kappa[2], int iflag, const qq_defl* defl,
                 qq_solve_info* info);
/* psc :4310-4465.  isignal = 1: gmresdr, keeping the deflation space in defl;
 * isignal = 2: gmresproj(n - k, k) to the reference's fixed 1e-8 (resmax unused). */
int qq_psc(qq_ctx* ctx, const double* b, double* x, const int GMRES[2], double resmax,
           int itermin, const double kappa[2], int iflag, int isignal, qq_defl* defl,
           qq_solve_info* info);
/* gmresdrshift :6041-7179 (Darnell, Morgan and Wilcox multi-shift GMRES-DR): solves
 * (A - sigma[s]) x_s = b for s = 0..nshifts-1, A = gamma5mult (qq_gamma5mult), with one
 * Krylov space: GMRES-DR(GMRES[0], GMRES[1]) on A - sigma[0], every other shift kept with a
 * residual collinear to the base residual.  xshift: nshifts consecutive even-half arrays
 * in the reference layout, written on exit (the initial guess is zero for every shift).
 * resid[s] = ||b - (A - sigma[s]) x_s|| (absolute, recursively updated as in the
 * reference); the iteration stops when resid[0] < resmax.  The reference leaves its
 * local sigma unassigned and forms the shifted solutions only when j reaches its
 * compile-time nmaxGMRES; here the shifts are an argument and the solutions are formed
 * at the end of every cycle.  iflag must be -1; kappa[0]*kappa[1] must not be 0.
 * Returns QQ_NOT_CONVERGED after 5000 cycles (kcyclim). */
int qq_gmresdrshift(qq_ctx* ctx, const double* b, double* xshift, int nshifts, const double* sigma,
                    const int GMRES[2], double resmax, int itermin, const double kappa[2], int iflag,
                    double* resid, qq_solve_info* info);
/* bicgstab :302-487.  maxiter <= 0 means no limit beyond the reference's. */
int qq_bicgstab(qq_ctx* ctx, const double* phi, double* x, double resmax, int itermin,
                const double kappa[2], int iflag, int maxiter, qq_solve_info* info);

/* ---- propagators (Q/quark.f90) ---- */
/* fermprop :458-842 for nkappa = -1 (Wilson / twisted-mass Wilson, cSW = 0):
 * source preparation, inverter (0 bicgstab, 5 gmresdr, 6 psc), odd-half
 * reconstruction and, if ntmqcd != 0 and |mu| > 1e-4, the twisted-basis rotation
 * (gamma5vector :3484-3548).  bo is read only.  isignal and defl as for qq_psc. */
int qq_fermprop(qq_ctx* ctx, const double* be, const double* bo, const double kappa[2],
                int inverter, double resmax, int itermin, const int nGMRES[2], double* xe,
                double* xo, int ntmqcd, int isignal, qq_defl* defl, qq_solve_info* info);
/* pointsource :46-108 (src is 1-based global coordinates). */
int qq_pointsource(qq_ctx* ctx, double* be, double* bo, const int src[4], int icsrc, int idsrc);

/* ---- batched mixed-precision propagators (the accelerated method) ----
 * Solves nrhs systems M x = b on the full lattice to the FP64 true residual
 * ||b - M x|| / ||b|| <= tol.  The first right-hand side builds the deflation space
 * with mixed-precision GMRES-DR(m, k) (FP32 Krylov basis and FP32 operator inside
 * FP64 iterative refinement); the others are projected onto it and solved together
 * in blocks with a multi-right-hand-side FP32 (precision = 32) or FP16 (precision =
 * 16) BiCGStab inside FP64 reliable updates.  If that BiCGStab breaks down (a NaN in
 * its recurrences), every unfinished right-hand side of the block is solved again from
 * zero by plain FP64 GMRES-DR(m, k) and reported with fallback = 1.  be/bo/xe/xo: nrhs
 * reference-layout halves each, packed one after the other. */
typedef struct qq_method {
  int m, k;          /* GMRES-DR(m, k) */
  int precision;     /* BiCGStab storage: 64, 32, 16 (FP16) or -16 (BF16); the 16-bit
                        storages keep one FP32 scale per site and compute in FP32; FP64
                        reliable updates in every case */
  int rhs_block;     /* right-hand sides solved together (1..32) */
  double tol;        /* FP64 true full-lattice relative residual target */
  int max_outer;     /* iteration limit in thousands (0: none) */
  int solver;        /* 0: plain FP64 GMRES-DR(m,k) per right-hand side (the reference
                        method); 1: batched BiCGStab */
  int deflate;       /* solver 1: build k deflation vectors with mixed-precision
                        GMRES-DR(m,k) on the first right-hand side and project every
                        residual onto them at each reliable update */
  double defl_tol;   /* relative residual the deflation-building solve stops at */
  int stall_window;  /* solver 1: a right-hand side whose FP64 true residual has not fallen
                        10x within this many BiCGStab iterations stops; a 16-bit one is
                        continued by the batched FP32 BiCGStab, an FP32 one is solved by
                        plain FP64 GMRES-DR(m, k), as after a breakdown (0: 2000, and 400
                        for a 16-bit iteration) */
} qq_method;
int qq_fermprop_batch(qq_ctx* ctx, int nrhs, const double* be, const double* bo,
                      const double kappa[2], const qq_method* method, double* xe, double* xo,
                      qq_solve_info* infos);

/* Uneven batch: propagator solves over several lattices, gauge fields and kappa values
 * in one call (the reference runs them as separate cfgsprops jobs, one fermprop per
 * source: Q/quark.f90:458-842 through C/cfgsprops.f90).  A group is nrhs sources on
 * the lattice and gauge field of its context at one kappa, solved exactly as
 * qq_fermprop_batch solves them (be/bo/xe/xo in that entry point's layout for the
 * group's context; infos: nrhs reports, may be NULL).  concurrent = 1: one host thread
 * per distinct context, its groups in array order, the contexts side by side on their
 * own streams; concurrent = 0: every group in array order on the calling thread.
 * A context must not be used by any other thread during the call.  seconds (may be
 * NULL): wall time of the whole call, every solve synchronised.  Returns the worst
 * status (a hard error stops that context's later groups; QQ_NOT_CONVERGED with every
 * output filled if a solve stopped short). */
typedef struct qq_uneven_group {
  qq_ctx* ctx;
  int nrhs;
  double kappa[2];   /* kappa, twisted mass mu */
  const double* be;
  const double* bo;
  double* xe;
  double* xo;
  qq_solve_info* infos;
} qq_uneven_group;
int qq_fermprop_uneven(int ngroups, const qq_uneven_group* groups, const qq_method* method,
                       int concurrent, double* seconds);

/* ---- noise sources and loop traces (Q/disconloops.f90, G/lagfib.f90) ---- */
/* initlagfib G/lagfib.f90:80-92 (process-global generator state, as the reference). */
int qq_initlagfib(int myid, int iseed);
/* rnds G/lagfib.f90:219-259. */
int qq_rnds(int m, double* rn);
/* z2source :4583-4649 and z4source (active branch) :4518-4570. */
int qq_z2source(qq_ctx* ctx, double* be, double* bo);
int qq_z4source(qq_ctx* ctx, double* be, double* bo);
/* Unsubtracted (level-0) time-slice traces of one noise vector: twAverage
 * (Q/vevbleft.f90:2541-4704) with nsub = 0 and zero momentum, point-split currents of
 * currentCalc2P (:10863-11247, r = +1), scalarCalc (:9261-9299), and the caller's
 * kappa scaling of Q/disconloops.f90:4045-4049.  be/bo: the noise (only its real
 * part enters, as in twAverage); xe/xo: the solution; delta: twist angle (0 for
 * Wilson); dobndry = 1: fixed time boundary (no time current across it).  Uses the
 * context's gauge field.  J(2, nt, 6), host or device: op 1 = J4 point-split time
 * current, 2 = psibar psi, 3..5 = J1..J3 point-split spatial currents,
 * 6 = psibar gamma5 psi, ops other than 2 and 6 multiplied by kappa.  Averaging over
 * noises and the division by nx*ny*nz (:4161-4164) are left to the caller. */
int qq_twaverage_level0(qq_ctx* ctx, const double* be, const double* bo, const double* xe,
                        const double* xo, double kappa, double delta, int dobndry, double* J);
/* Batched disconnected loops at the unsubtracted level: the noise loop of twistdiscon
 * (Q/disconloops.f90:3612-4170).  For each of nnoise noises, in the generator's order
 * (qq_initlagfib first, as the reference): draw Z(noise_kind = 2 or 4) noise, solve,
 * take the level-0 traces of qq_twaverage_level0 and accumulate; J(2, nt, 6) (host or
 * device) receives the sum divided by nnoise and by nx*ny*nz (:4161-4164).
 * method->solver: 0 = plain FP64 GMRES-DR(m, k) per noise to tol; 1 = batched
 * mixed-precision BiCGStab on blocks of rhs_block noises (as qq_fermprop_batch);
 * 2 = the reference's psc sequence (GMRES-DR(m, k) on the first noise keeping its
 * deflation space, GMRES-Proj(m - k, k) to the fixed 1e-8 on the rest).  infos (nnoise
 * entries, may be NULL) receives each solve's report.  Returns QQ_NOT_CONVERGED (with
 * J filled) if any solve stopped short of its tolerance. */
int qq_discon_traces(qq_ctx* ctx, int noise_kind, int nnoise, const double kappa[2],
                     const qq_method* method, double delta, int dobndry, double* J,
                     qq_solve_info* infos);

/* twAverage Q/vevbleft.f90:2541-4704 for one noise: the loop operators of the noise be/bo
 * and its solution xe/xo with the momentum projections imom 2..5 about the origin io
 * (1-based) and Wilson r = ir (+-1: currentCalc2P / currentCalc2M, :10863-11635), into
 * Jave(2, nt, 6, nmom, nop) (Fortran order, host or device), unscaled.
 * The reference's perturbative subtraction inside twAverage is switched off
 * (if (.false.), :2990-3935), so every level it fills -- 1, and 4 (nsub = 4, 6) and 6
 * (nsub = 6) -- holds the unsubtracted traces; every other entry is zero.  kappa enters
 * only that switched-off subtraction.  nmom 1..5, nop >= 6. */
int qq_twaverage(qq_ctx* ctx, const double* be, const double* bo, const double* xe,
                 const double* xo, double kappa, double delta, const int io[3], int dobndry,
                 int ir, int nsub, int nmom, int nop, double* Jave);
/* twistdiscon Q/disconloops.f90:3612-4351 at subtraction levels nsub = 0, 4 or 6, Wilson
 * r = ir (+-1, passed to twvev and twAverage as the reference does):
 * Jtotal = numnoises * Jvev' + sum over noises of Jave' , divided by numnoises and by
 * nx*ny*nz (:4161-4164), where Jvev' is qq_twvev's output with every operator but 2 and
 * 6 times kappa and level 6 combined with level 4 (:3793-3805), and Jave' is qq_twaverage
 * of each noise with the same kappa factor (:4040-4045).  Noises, solves and method as
 * qq_discon_traces (call qq_initlagfib first).  Jtotal(2, nt, 6, nmom, nop), host or
 * device.  Jnoise (may be NULL): every noise's Jtemp = (Jave' + Jvev') / (nx*ny*nz), the
 * per-noise values the reference writes for its error analysis (:4112-4114, :4230-4260),
 * as Jnoise(2, nt, 6, nmom, nop, nnoise).  Returns QQ_NOT_CONVERGED (with the outputs
 * filled) if a solve stopped short. */
int qq_twistdiscon(qq_ctx* ctx, int noise_kind, int nnoise, const double kappa[2],
                   const qq_method* method, double delta, const int io[3], int dobndry, int ir,
                   int nsub, int nmom, int nop, double* Jtotal, double* Jnoise,
                   qq_solve_info* infos);

/* average Q/disconloops.f90:5343-5733 (the Wilson loop driver's operators of one noise):
 * for levels isub = 1..nsub (<= 6), the solution x (isub = 1) or x minus the hopping
 * expansion of the propagator applied to the noise, sum_{n=0}^{isub+1} kappa^n H^n b
 * (isub >= 2), goes through loopops (:7769-7910: point-split currents J1..J4 with the
 * boundary factors, psibar psi with +12 on subtracted levels, local vector currents
 * J5+mu; the complex noise kept whole) and spacesum (:9012-9124) into
 * Jtime(2, nt, nsub, nmom, nop) (Fortran order, host or device, nop >= 9); operators
 * 1..4 are multiplied by kappa.  momfac(nvhalf, 2, 16, nmom-1, >= 5): the caller's
 * momentum factors (host or device; may be NULL when nmom = 1). */
int qq_average(qq_ctx* ctx, const double* be, const double* bo, const double* xe, const double* xo,
               double kappa, int nsub, int nmom, int nop, const double* momfac, double* Jtime);
/* momfacs Q/disconloops.f90:8925-8984 (host memory; no device needed): the momentum
 * factors of the Wilson driver for 4 momenta about the origin io (1-based),
 * momfac(nvhalf, 2, 16, 4, 5), nvhalf = nx*ny*nz*nt/32. */
int qq_momfacs(const int dims[4], const int io[3], double* momfac);

/* smear Q/diracops.f90:712-858: nsmear sweeps of gauge-covariant spatial smearing
 * h <- (1 - 6 asmear) h + asmear sum_{mu=1..3} [U_mu(x) h(x+mu) + U_mu(x-mu)^+ h(x-mu)]
 * (spin diagonal, bc(mu) across the edge) of the reference-layout pair (ge, go) into
 * (he, ho); host or device. */
int qq_smear(qq_ctx* ctx, double* he, double* ho, const double* ge, const double* go, double asmear,
             int nsmear);
/* mesoncorr Q/quark.f90:1297-2137, the correlators of one (q, qbar) propagator pair:
 * q: the 12 propagator columns of a point source src (1-based), column (jc - 1) * 4 +
 * (jd - 1) for source colour jc and spin jd, each the even then the odd reference-layout
 * half (2 * 6 * ntotal * 64 doubles per column; host or device); qbar the same for the
 * antiquark (NULL: q).  corrRe, corrIm(nt, -4:4, -4:4, -4:4, 28) (Fortran order, host or
 * device): per operator pair ii of the reference's table (corrsp set) the slice sums of
 * the contraction times e^{2 pi i p.(x - src)/L}.  channels 0: the pairs the reference
 * evaluates (P->P ii = 2, S->P ii = 11, P->S ii = 22; the rest zero, :1869-1870);
 * 1: all 28.  Sink smearing is qq_smear on each column first; the file handling
 * (FPread of the columns, the MESON.LOG lines) stays with the caller (qq_fpread). */
int qq_mesoncorr(qq_ctx* ctx, const double* q, const double* qbar, const int src[4], int channels,
                 double* corrRe, double* corrIm);

/* vev Q/disconloops.f90:4653-5339: the perturbative vacuum values of the Wilson driver's
 * loop operators from the plaquettes P = U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+ of
 * every plane, summed per time slice with the reference's momentum weights about io
 * (1-based), scaled by 8 kappa^4 and its multiplicities and negated: Jvev(2, nt, 5, 5)
 * (Fortran order, host or device).  plaq (may be NULL): the average plaquette
 * sum Re Tr P / (18 V); psi (may be NULL): the <psibar psi> value it logs. */
int qq_vev(qq_ctx* ctx, double kappa, const int io[3], double* Jvev, double* plaq, double* psi);
/* discon Q/disconloops.f90:3445-3608, one run: Jtotal(2, nt, nsub, nmom, nop) (nop <= 9; the
 * reference uses 5) = (Jvev on levels 2..nsub + the sum over nnoise Z(2) / Z(4) noises of
 * average(nsub, nmom, momfacs about io)) / nnoise / (nx ny nz) -- Jvev divided by the
 * number of noises too, as the reference does.  The noises are solved by the method
 * (the reference uses QMR, inverter 2, which is not on this path).  Jvev (may be NULL)
 * receives qq_vev's output.  Call qq_initlagfib first.  The reference repeats this run
 * numruns = 20 times on one generator stream (20 calls); its numnoises = 0 branch (one
 * given source, no division) is qq_fermprop followed by qq_average. */
int qq_discon(qq_ctx* ctx, int noise_kind, int nnoise, double kappa, const qq_method* method,
              const int io[3], int nsub, int nmom, int nop, double* Jtotal, double* Jvev,
              qq_solve_info* infos);

/* ---- eigenmode subtraction of the Wilson loop driver (testFUNC,
 * Q/disconloops.f90:1980-2569) ----
 * A qq_eig handle holds kept eigenmodes on the device (right vectors R and, for kind 1,
 * left vectors L; both halves of the lattice) and their eigenvalues. */
typedef struct qq_eig qq_eig;
/* kind 1: eigmodesofM Q/disconloops.f90:1593-1937, modes of M = 1 - kappa D.  The Ritz
 * pairs of the even-odd operator Hdbletm (Hdouble when kappa[1] < 1e-8) after ncycles
 * cycles of gmresdrEIGBS Q/working.f90:48-907 (GMRES-DR(nGMRES) whose restart keeps the
 * k = nGMRES[1] harmonic Ritz vectors with the smallest |theta| plus their common
 * residual direction; the reference runs 150 cycles of (200, 160)) from the unit source
 * b(1,1,1,1,1) = 1; se, so are ignored.  Ritz values in conjugate pairs (to 1e-8) are
 * lifted to M, lambda = 1 - sqrt(1 - kappa^2 theta), with odd halves
 * kappa H_oe R_e / sqrt(1 - kappa^2 theta) and left vectors gamma5 times the partner's
 * right vector, R scaled to <R, L> = 1; modes with ||M R - lambda R|| < 1e-8 are kept,
 * sorted by |lambda|.  The reference's sort reads its permutation through the wrong
 * index (ind2(ind(eig)), :1889-1899); the two agree whenever every pair is kept.
 * kind 2: eigmodesofMprime :2573-2875, modes of the Hermitian M gamma5 on the full
 * lattice after ncycles cycles of gmresdr5EIG Q/inverters.f90:1435-2070 (the restart
 * keeps the least-squares residual; the reference allows 5500 cycles) from the start
 * vector (se, so) (the reference draws a Z(4) noise, qq_z4source); unit-norm modes with
 * ||M gamma5 R - Re(theta) R|| < 1e-5 are kept, sorted by |Re theta|, L = R.
 * nGMRES: k < m <= 255.  numEV (may be NULL): modes kept; evals (may be NULL, room for
 * 2 k doubles): their eigenvalues (re, im).  Release with qq_eig_destroy. */
int qq_eigmodes(qq_ctx* ctx, int kind, const int nGMRES[2], int ncycles, const double kappa[2],
                const double* se, const double* so, qq_eig** eig, int* numEV, double* evals);
int qq_eig_destroy(qq_eig* eig);
/* kind, modes kept, cycles run, operator applications, eigenvalues (2 numEV) and the
 * k Ritz values of the last cycle (2 k); any output may be NULL. */
int qq_eig_info(const qq_eig* eig, int* kind, int* numEV, int* cycles, int* mvp, double* evals,
                double* ritz);
/* Mode j (0-based) as reference-layout halves (host or device): R, or L if left != 0. */
int qq_eig_vector(const qq_eig* eig, int j, int left, double* ve, double* vo);
/* xigenerator Q/disconloops.f90:465-838: xiinv(2, 6, numEV) (Fortran order, host or
 * device) = <L_j, S_isub R_j> with S_1 = 0 and S_isub = sum_{n=0}^{isub+1} kappa^n H^n
 * (H = Hsingle on each half), times gamma5 for kind 2 (gammaid = 2). */
int qq_xigenerator(qq_ctx* ctx, const qq_eig* eig, double kappa, double* xiinv);
/* eigaverage Q/disconloops.f90:3239-3342: for each selected mode count j (j = eigstart,
 * every eigstep-th after it, and numEV) the loop operators (loopops, ksub 0; kind 2:
 * eigloopops_original :7919-8038, i.e. of gamma5 x') of the correction
 * x'_j = sum_{i<=j} R_i s_i <L_i, z> against the noise z, summed per time slice;
 * operators 1..4 times kappa; other counts zero.  scal(2, numEV): the multipliers s
 * (1/lambda for the plain estimator, xiinv(:, isub, :) for the combined one).
 * Jtime(2, nt, numEV, 9), Fortran order, host or device: the reference's
 * Jtime(:, :, :, 1, :) (its momentum slots 2..5 stay zero, as its momfac is zero). */
int qq_eigaverage(qq_ctx* ctx, const qq_eig* eig, const double* ze, const double* zo, double kappa,
                  const double* scal, int eigstart, int eigstep, double* Jtime);
/* The least-squares polynomial of ppaverage (p = 5), ppaverage1 (p = 8), ppaverage2
 * (p = 11) and xipolygenerator (p = 8), Q/disconloops.f90:6885-7434, 6290-6883,
 * 5740-6288, 847-1584: co(2, p) (host or device) solving the normal equations
 * sum_b <M^a z, M^b z> co_b = <M^a z, z> (a, b = 1..p) of min || z - sum_b co_b M^b z ||,
 * M = 1 - kappa D on the full lattice, z = (be, bo).  The reference fits these once, on
 * the first noise (psignal, Q/shift.f90:45), and reuses them. */
int qq_ppcoeffs(qq_ctx* ctx, const double* be, const double* bo, double kappa, int p, double* co);
/* ppaverage / ppaverage1 / ppaverage2 (p = 5, 8, 11) at imom = 1: level isub = 1 the
 * solution x, level isub >= 2 x - sub_isub with sub_isub = sum of co_c M^(v-1) b over the
 * terms of levels 2..isub (level 2: c = v = 1..4; then one term per level, c = v = 5, 6,
 * 7 and for p = 11 the four terms 8..11 at level 6; p = 5 reuses c = 5 with v = 6, 7, 8),
 * through loopops (ksub 1 on levels >= 2) and spacesum; operators 1..4 times kappa.
 * Jtime(2, nt, nsub, 9), Fortran order, host or device; nsub <= 6. */
int qq_ppaverage(qq_ctx* ctx, int p, const double* co, const double* be, const double* bo,
                 const double* xe, const double* xo, double kappa, int nsub, double* Jtime);
/* xipolygenerator Q/disconloops.f90:847-1584: xiinv(2, 6, numEV) = <L_j, gamma5 sub_isub R_j>
 * with the p = 8 terms above applied to each mode R_j and coefficients co(2, 8) (the
 * reference fits them on a noise with qq_ppcoeffs for gamma5 modes, and sets them to 1
 * otherwise). */
int qq_xipolygenerator(qq_ctx* ctx, const qq_eig* eig, double kappa, const double* co, double* xiinv);
/* generalaverage Q/disconloops.f90:119-333 for one noise z and its solution x (M x = z):
 * Jave(2, nt, 6, numEV_MAX, 10, 9) (Fortran order, host or device; numEV_MAX the larger
 * mode count) at imom = 1, zero where a style is not defined, with
 *   NS = loopops of x (nsaverage :3079-3143),   PS = -average(z, 0) (qq_average),
 *   ES / HFES = qq_eigaverage of m (1/lambda) / of mp (1/lambda'),
 *   ESPS / HFESPS = qq_eigaverage with xiinv(:, isub, :) of m / mp,
 *   HFESPOLY = qq_eigaverage of mp with qq_xipolygenerator(mp, copoly),
 *   PP, PP4, PP7 = -qq_ppaverage(0) with p = 11 (co11), 5 (co5), 8 (co8):
 * style 1 NS (mode 1, level 1); 2 NS - PS (mode 1); 3 NS - ES (level 1); 4 NS - HFES
 * (level 1); 5 NS - ES - (PS - ESPS); 6 NS - HFES - (PS - HFESPS); 7 NS - PP, 8 NS - PP4,
 * 9 NS - PP7 (mode 1); 10 NS - HFES - (PP7 - HFESPOLY).  m: kind 1, mp: kind 2. */
int qq_generalaverage(qq_ctx* ctx, const qq_eig* m, const qq_eig* mp, const double* ze, const double* zo,
                      const double* xe, const double* xo, double kappa, int eigstart, int eigstep,
                      const double* co11, const double* co8, const double* co5, const double* copoly,
                      double* Jave);

/* ---- file formats (host memory; no device needed) ----
 * Fortran unformatted sequential files, as the reference writes them: every record is
 * framed by its 4-byte length, reals are 8 bytes, integers 4.  nvhalf and ntotal are
 * the reference array sizes (qq_ctx_dims). */
/* GFwrite G/gaugetools.f90:1260-1294: re-unitarises u in place (fixsu3 :1338-1432),
 * then writes rows 1-2 of every link and the trailer (gaction, beta, alat, tad,
 * icfgsave, myid).  The file must not exist (status="new"). */
int qq_gfwrite(const char* path, double* u, int nvhalf, int ntotal, const int gaction[4],
               double beta, const double alat[4], const double tad[4], int icfgsave, int myid);
/* GFread :1298-1334: reads rows 1-2 and the trailer, completes row 3 with fixsu3. */
int qq_gfread(const char* path, double* u, int nvhalf, int ntotal, int gaction[4], double* beta,
              double alat[4], double tad[4], int* icfgsave, int* myid);
/* FPwrite Q/quark.f90:3379-3434 (xe: gblclr = 1 half, xo: gblclr = 2 half) and
 * FPread :3438-3481. */
int qq_fpwrite(const char* path, const double* xe, const double* xo, int nvhalf, int ntotal,
               double kappa, double tmqcd, double cSW, int icsrc, int idsrc, int icfg, int myid);
int qq_fpread(const char* path, double* xe, double* xo, int nvhalf, int ntotal, double* kappa,
              double* tmqcd, double* cSW, int* icsrc, int* idsrc, int* icfg, int* myid);

/* ---- measurement (library-specific; no counterpart in the reference) ---- */
/* The cudaStream_t every call of this context runs on (for event timing). */
int qq_ctx_stream(const qq_ctx* ctx, void** stream);
/* Number of kernels this library has launched in this process so far. */
long long qq_launch_count(void);
/* enable != 0: time every hopping-kernel launch with CUDA events until disabled.
 * qq_profile_hop_read returns the launches, their summed time and their summed
 * algorithmic bytes V/2 * (8 * link bytes + nrhs * (2 or 3) * spinor bytes) since the
 * last enable. */
int qq_profile_hop(qq_ctx* ctx, int enable);
int qq_profile_hop_read(qq_ctx* ctx, long long* launches, double* ms_total, double* bytes_total);
/* The same over the profiled launches of one spinor precision (64, 32, 16; 0: any) and
 * RHS count (0: any), with their algorithmic flops: 1320 per output site and
 * right-hand side (the standard spin-projected count of Q/diracops.f90:554-599). */
int qq_profile_hop_select(qq_ctx* ctx, int precision, int nrhs, long long* launches, double* ms_total,
                          double* bytes_total, double* flops_total);

/* Times `niter` launches of the hopping kernel alone (H_oe of random fields, output
 * parity gblclr = 2) with CUDA events on the library's stream.  precision: 64
 * (links at the uploaded recon), 32, 16 or -16 (BF16) (FP32 recon-12 links); nrhs right-hand
 * sides per launch (1..32; for nrhs > 1 one RHS-interleaved block field, the layout
 * of the batched solver); tps: kernel shape (0 = the autotuned choice the solvers
 * use; 1, 2, 4 direction groups per site; 32-128 threads per block of the staged
 * kernel; 202-204 = block fields with 2-4 right-hand sides per thread, FP32/FP16;
 * 301-303 = FP32 with packed FP32x2 arithmetic, 1-3 right-hand sides per thread;
 * 304 = the same, one right-hand side per thread, loads issued a hop ahead;
 * 305 = 304 with the links staged in shared memory, block fields of >= 8 RHS;
 * 306, 307, 308 = one right-hand side per thread, the neighbour spinors of the next 2,
 * 3, 4 hops in flight as asynchronous copies into a shared-memory ring, the links of
 * neighbour indices and hop matrices of the block's sites built once per block in
 * shared memory, >= 4 RHS recommended; 309, 310 = 306 with its registers capped for 5
 * and 6 resident blocks per SM; 311 = 307 with the hop matrices kept pre-broadcast).
 * flush_l2 != 0 overwrites a 512 MiB buffer between launches so every launch reads
 * its operands from HBM.  ms_per_call: mean kernel time; bytes_per_call:
 * algorithmic bytes of one launch, V/2 * (8 * link bytes + nrhs * 2 * spinor bytes). */
int qq_bench_hsingle(qq_ctx* ctx, int precision, int nrhs, int tps, int niter, int flush_l2,
                     double* ms_per_call, double* bytes_per_call);

/* ---- local meson correlators ----
 * pionrho Q/quark.f90:1033-1212: adds the local pion, rho (third vector component,
 * times rsgn(idsrc) = (1,-1,-1,1)) and pion-decay (fourth axial component) correlators
 * of one propagator column -- the solution xe (gblclr = 1) / xo (gblclr = 2) for source
 * spin idsrc -- to pion[nt], rho[nt], decay[nt] (host or device), as the reference
 * accumulates them over its sources. */
int qq_pionrho(qq_ctx* ctx, const double* xe, const double* xo, int idsrc, double* pion, double* rho,
               double* decay);

/* ---- perturbative vacuum expectation values of the loop operators ----
 * twvev Q/vevbleft.f90:757-2536: the hopping-parameter expansion of the twisted-mass
 * propagator to order kappa^6 from unit sources at every site, colour and spin, with
 * the context's gauge field; no noise.  Fills Jvev(2, nt, 6, nmom, nop) (Fortran order,
 * host or device): level 4 (nsub = 4 or 6) holds orders kappa^3 (currents) and kappa^4
 * (psibar psi, psibar gamma5 psi), plus kappa^1 / kappa^2 when delta /= 0; level 6
 * (nsub = 6) orders kappa^5 / kappa^6; every other entry is zero, as in the reference.
 * Operators iop 1..6: J4 point-split time current, psibar psi, J1..J3 point-split
 * spatial currents, psibar gamma5 psi (momenta imom 2..5: the reference's ffac / fas
 * projections about the origin io, 1-based).  kappa: the hopping parameter, delta: the
 * twist angle; dobndry = 1: fixed time boundary; ir = +-1: the Wilson r.  The caller's
 * kappa scaling and level combination (Q/disconloops.f90:3793-3805) are left to the
 * caller, as in the reference.  nmom 1..5, nop >= 6 (operators past 6 stay zero). */
int qq_twvev(qq_ctx* ctx, double kappa, double delta, const int io[3], int dobndry, int ir,
             int nsub, int nmom, int nop, double* Jvev);

/* ---- learned preconditioner (no counterpart in the reference) ----
 * A gauge-covariant network of linear parallel-transport convolution layers: a layer
 * maps Cin channels to Cout channels (a channel is one colour vector per site of the
 * full lattice) by out_co(x) = sum_p sum_ci W[p][co][ci] (T_p f_ci)(x) over the paths
 * p = 0 (the site itself), 1 + 2 mu (U_mu(x) f(x + mu)) and 2 + 2 mu
 * (U_mu(x - mu)^+ f(x - mu)), with the lattice's boundary factors on wrapping hops.
 * The network maps an even-site (gblclr = 1) Dirac vector, channel = spin, to an
 * even-site vector and is trained to approximate the inverse of Hdbletm; flexible
 * GMRES uses it as a right preconditioner.  Weights are complex, stored
 * [layer][p][co][ci] as (re, im) pairs. */
typedef struct qq_net qq_net;
/* channels[0..nlayers]: 4, then 4, 8 or 16 per hidden layer, then 4.  The network
 * starts near scale * identity (kappa^2 approximates the inverse of Hdbletm's leading
 * term) with small random weights on every other path (seeded). */
int qq_net_create(int nlayers, const int* channels, unsigned long long seed, double scale, qq_net** out);
int qq_net_destroy(qq_net* net);
int qq_net_nweights(const qq_net* net); /* complex weights */
int qq_net_get_weights(const qq_net* net, double* w);
int qq_net_set_weights(qq_net* net, const double* w);
/* out = N(in); reference-layout gblclr = 1 half vectors, host or device. */
int qq_net_apply(qq_ctx* ctx, qq_net* net, const double* in, double* out);
/* Loss l = (1/S) sum_i |N(b_i) - x_i|^2 / |x_i|^2 over nsamples pairs (half vectors
 * back to back) and its gradient dl/d conj(W), same layout as the weights. */
int qq_net_grad(qq_ctx* ctx, qq_net* net, int nsamples, const double* b, const double* x, double* loss,
                double* grad);
/* nsteps Adam steps (learning rate lr) on nsamples pairs (Hdbletm x, x) with Gaussian
 * x drawn from `seed`; losses[step] (may be NULL) receives the loss before each step. */
int qq_net_train(qq_ctx* ctx, qq_net* net, const double kappa[2], int nsamples, int nsteps, double lr,
                 unsigned long long seed, double* losses);
/* The same on the caller's pairs: nsamples sources b and targets x (reference-layout even
 * half vectors back to back, host or device), the network learning N(b) = x -- e.g. the
 * (source, FP64 solution) pairs and the low modes (Hdbletm v, v) of the deflated
 * inverter's own solves. */
int qq_net_train_pairs(qq_ctx* ctx, qq_net* net, int nsamples, const double* b, const double* x, int nsteps,
                       double lr, double* losses);
/* Flexible GMRES(m) on Hdbletm x = phi with the network as right preconditioner (net
 * NULL: none), FP64; converged when ||phi - A x|| / ||phi - A x0|| < resmax, checked
 * once per cycle.  If two consecutive cycles each gain less than a factor 2, plain
 * GMRES-DR(m, m/3) continues from the current x (info->fallback = 1).  x: initial
 * guess in, solution out. */
int qq_fgmres(qq_ctx* ctx, qq_net* net, const double* phi, double* x, int m, double resmax, int max_cycles,
              const double kappa[2], qq_solve_info* info);
/* Flexible GMRES-DR(GMRES[0], GMRES[1]): qq_fgmres with Morgan's deflated restarts
 * (both the Krylov basis and the preconditioned directions are rotated onto the
 * GMRES[1] smallest harmonic Ritz vectors of Hdbletm N), so the low modes the
 * network cannot learn stay deflated.  Same convergence test; the fallback follows three
 * consecutive cycles that each gain less than 10%. */
int qq_fgmresdr(qq_ctx* ctx, qq_net* net, const double* phi, double* x, const int GMRES[2], double resmax,
                int max_cycles, const double kappa[2], qq_solve_info* info);

/* The kernel shape (the codes of qq_bench_hsingle) the autotuner chose for the first
 * hopping launch of Hdbletm (Wilson, else twisted mass, else the second launch) at this
 * precision and RHS count (block fields for nrhs > 1) in this context; QQ_BAD_ARG if
 * no such launch has run yet. */
int qq_hop_tuned_shape(qq_ctx* ctx, int precision, int nrhs, int* shape);

/* The hopping term of qq_hsingle (Hsingle, Q/diracops.f90:554-599) on nrhs half-lattice fields
 * at once, computed in reduced precision the way the batched solver applies it: gin
 * holds nrhs reference-layout input vectors back to back (parity opposite to gblclr),
 * converted to one RHS-interleaved block field of precision 32, 16 or -16 (BF16) (a plain field for
 * nrhs = 1), multiplied by kernel shape `shape` (the codes of qq_bench_hsingle; 0 = the
 * autotuned choice) with FP32 recon-12 links, and written to gout as nrhs FP64
 * reference-layout vectors.  QQ_BAD_ARG when the shape does not support this precision
 * or RHS count. */
int qq_hsingle_block(qq_ctx* ctx, int precision, int nrhs, int shape, double* gout, const double* gin,
                     int idag, int gblclr);

#ifdef __cplusplus
}
#endif
#endif /* QQCD_GPU_H */
