// CPU oracle for the qqcd solver hot path -- TEST INFRASTRUCTURE ONLY.
//
// This is a line-by-line C++ restatement of the BaylorLQCD `qqcd` Fortran-90 routines
// on the solver hot path (Wilson / twisted-mass Dirac operator, GMRES-DR, GMRES-Proj,
// BiCGStab, propagator source preparation / reconstruction, noise sources, lagged
// Fibonacci RNG, loop traces).  Each function cites the reference file:line it follows.
//
// Parity status: UNPINNED against the Fortran itself.  No Fortran compiler exists in
// this environment and the reference ships no golden vectors, known-answer files or
// tests, so the restatement cannot be checked against reference outputs.  It is
// pinned instead against analytic known answers (free-field plane waves, gamma5
// hermiticity, gauge covariance, dense-matrix solves) and against scipy's LAPACK for
// the restated pseudolapack steps.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use this
// library, and only as the checker / timed CPU reference -- never as a product path.
//
// Array layouts are the reference's Fortran column-major layouts, 1-based in the
// comments:
//   Dirac half-vector  g(6, ntotal, 4, 2, 8)   (re/im x colour, site, spin, ieo, ibleo)
//   Gauge field        u(18, ntotal, 4, 2, 16) (3x3 row-major re/im, site, mu, ieo, ibl)
// with nvhalf = V/32 and ntotal = nvhalf + nbmax (one process: nps = 1).
#pragma once
#include <cstdint>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oq_geom oq_geom;

// Build the geometry / index tables of lattice.f90:initlat for one process.
// bc[mu] in {1,-1,0}; c1[mu] = coact(3,1,mu); c2[mu] = coact(3,2,mu).
oq_geom* oq_geom_create(int nx, int ny, int nz, int nt, const int bc[4],
                        const double c1[4], const double c2[4]);
void oq_geom_destroy(oq_geom* g);
int oq_nvhalf(const oq_geom* g);
int oq_ntotal(const oq_geom* g);
int oq_nbmax(const oq_geom* g);
// Copies of the index tables (1-based values, Fortran order):
// lv/lvbc(nvhalf,4,2), ib(nbmax,4,2,2), nms(4), lbd(16,4) as int, iblv(16,4),
// vecbl(2,8), vecblinv(2,16).
void oq_tables(const oq_geom* g, int* lv, int* lvbc, int* ib, int* nms, int* lbd,
               int* iblv, int* vecbl, int* vecblinv);
void oq_set_coact(oq_geom* g, const double c1[4], const double c2[4]);

// ---- map between global 0-based coordinates and the blocked layout ----
// (G/lattice.f90 siteindex/setblk/gblchker; Q/quark.f90:70-105 pointsource)
void oq_site_of_coords(const oq_geom* g, const int x[4], int* isite, int* ieo,
                       int* ibl, int* gblclr, int* ibleo);

// ---- lagged Fibonacci RNG (G/lagfib.f90) ----
void oq_initlagfib(int myid, int iseed);
void oq_rnds(int m, double* rn);
void oq_lagfib_state(int* iw /*521*/, int* jr, int* kr);
void oq_lagfib_set_state(const int* iw, int jr, int kr);

// ---- sources ----
void oq_pointsource(const oq_geom* g, double* be, double* bo, const int src[4],
                    int icsrc, int idsrc);
void oq_z2source(const oq_geom* g, double* be, double* bo);
void oq_z4source(const oq_geom* g, double* be, double* bo);

// ---- Dirac operator (Q/diracops.f90) ----
void oq_hsingle(const oq_geom* g, double* gout, const double* u, double* gin,
                int idag, int gblclr);
void oq_hdouble(const oq_geom* g, double* he, const double* u, double* ge, int idag,
                double kappa);
void oq_hdbletm(const oq_geom* g, double* he, const double* u, double* ge, int idag,
                const double kappa[2]);
void oq_twmshift(const oq_geom* g, double* hwhole, const double* u, double* gwhole,
                 int idag, const double kappa[2]);
void oq_gamma5mult(const oq_geom* g, double* he, const double* u, double* ge, int idag,
                   const double kappa[2]);
void oq_gam5x(const oq_geom* g, double* a);
void oq_gamma5vector(const oq_geom* g, double* a, int ntmqcd);
void oq_vecdot(const oq_geom* g, const double* a, const double* b, double* adb);

// ---- inverters (Q/inverters.f90) ----
// Cycle cap of GMRES-DR / GMRES-Proj (kcyclim, U/latdims.f90:70; default 5000).  A
// small cap times a bounded sample of the reference algorithm.
void oq_set_kcyclim(int n);
typedef struct oq_defl oq_defl;  // replaces module `shift` (vtemp, hcnew, beg)
oq_defl* oq_defl_create(const oq_geom* g, int nmax, int kmax);
void oq_defl_destroy(oq_defl* d);
// k+1 deflation vectors (reference layout) and hcnew((k+1) x k, complex, col-major).
void oq_defl_get(const oq_defl* d, int k, double* vtemp, double* hcnew);

typedef struct oq_solve_log {
  int itercount;
  int mvp;
  int ncycles;
  int nhist;          // entries written into hist (true residual per cycle)
  double hist[4096];
  int hist_mvp[4096];
  int nritz;          // harmonic Ritz values of the last restart (re,im)
  double ritz[2 * 512];
  double final_rel;   // ||phi - A x|| / ||phi|| at exit (even system)
} oq_solve_log;

int oq_gmresdr(const oq_geom* g, const double* phi, double* x, const int GMRES[2],
               double resmax, int itermin, const double* u, const double kappa[2],
               oq_defl* defl, oq_solve_log* log);
// gmresdrshift with explicit shifts sigma[nshifts]: xshift receives nshifts vectors
// (zero initial guess), resid the final ||r_s|| (absolute).
int oq_gmresdrshift(const oq_geom* g, const double* b, double* xshift, int nshifts,
                    const double* sigma, const int GMRES[2], double resmax, int itermin,
                    const double* u, const double kappa[2], double* resid, oq_solve_log* log);
int oq_gmresproject(const oq_geom* g, const double* b, double* x, const int GMRES[2],
                    double resmax, int itermin, const double* u, const double kappa[2],
                    int isignal, oq_defl* defl, oq_solve_log* log);
int oq_psc(const oq_geom* g, const double* b, double* x, const int GMRES[2],
           double resmax, int itermin, const double* u, const double kappa[2],
           int isignal, oq_defl* defl, oq_solve_log* log);
int oq_bicgstab(const oq_geom* g, const double* phi, double* x, double resmax,
                int itermin, const double* u, const double kappa[2], oq_solve_log* log,
                int maxiter);

// ---- propagator driver (Q/quark.f90 fermprop, nkappa = -1 Wilson/twisted mass) ----
int oq_fermprop(const oq_geom* g, const double* be, double* bo, const double kappa[2],
                int inverter, double resmax, int itermin, const int nGMRES[2],
                const double* u, double* xe, double* xo, int ntmqcd, int isignal,
                oq_defl* defl, oq_solve_log* log);

// ---- restated small dense algebra (Q/pseudolapack.f90), exposed for checks ----
// Complex matrices are (2, ld, ncol) Fortran order: re/im interleaved, column-major.
void oq_linearsolver(int n, int nrhs, double* a, int lda, int* ipiv, double* b, int ldb);
void oq_hessenberg(double* a, int lda, int n, int ilo, int ihi, double* tau);
void oq_qgenerator(int n, int ilo, int ihi, double* a, int lda, const double* tau);
void oq_evalues(int ischur, int n, int ilo, int ihi, double* h, int ldh, double* w,
                double* z, int ldz);
void oq_orgschur(const int* select, int n, double* t, int ldt, double* q, int ldq,
                 double* w, int* m);

// ---- loop traces (Q/vevbleft.f90 twAverage, nsub = 0; see loops.cpp) ----
// Per-time-slice traces of one noise solution at the unsubtracted level.
// J is (2, nt, 6) : op 1 = J4 point-split time current, 2 = psibar psi,
// 3..5 = J1..J3 point-split spatial currents, 6 = psibar gamma5 psi; ops other than
// 2 and 6 scaled by kappa.  delta: twist angle (0 for Wilson); dobndry = 1: fixed
// time boundary.
void oq_twaverage_level0(const oq_geom* g, const double* be, const double* bo,
                         const double* xe, const double* xo, const double* u,
                         double kappa, double delta, int dobndry, double* J);
// The same with the momentum projections imom 2..5 about the origin io (1-based) and
// Wilson r = ir (+-1): J(2, nt, nmom, 6), nmom 1..5.
void oq_twaverage_mom(const oq_geom* g, const double* be, const double* bo, const double* xe,
                      const double* xo, const double* u, double kappa, double delta,
                      const int io[3], int dobndry, int nmom, int ir, double* J);

// ---- Wilson loop operators with subtraction levels (Q/disconloops.f90 average,
// loopops, spacesum; see average.cpp) ----
// Jtime(2, nt, nsub, nmom, nop), nop >= 9; momfac(nvhalf, 2, 16, nmom-1, >= 5) as the
// reference's caller builds it (may be NULL when nmom = 1).
void oq_average(const oq_geom* g, const double* u, const double* be, const double* bo,
                const double* xe, const double* xo, double kappa, int nsub, int nmom, int nop,
                const double* momfac, double* Jtime);

// momfacs: momfac(nvhalf, 2, 16, 4, 5) about the origin io (1-based).
void oq_momfacs(const oq_geom* g, const int io[3], double* momfac);

// ---- the Wilson loop driver's vacuum values (Q/disconloops.f90 vev; see vevw.cpp) ----
// Jvev(2, nt, 5, 5), Fortran order (nmom = nop = 5), the average plaquette and
// <psibar psi>.  io: momentum origin (1-based).  Returns 0, or -1 when the reference's
// site enumeration disagrees with the pointsource site map.
int oq_vevw(const oq_geom* g, const double* u, const int io[3], double kappa, double* Jvev, double* plaq,
            double* psi);

// ---- perturbative vacuum expectation values (Q/vevbleft.f90 twvev; see vev.cpp) ----
// Jvev(2, nt, 6, nmom, nop), Fortran order; levels 4 (orders kappa^3 / kappa^4, and
// kappa^1 / kappa^2 when delta /= 0) and 6 (orders kappa^5 / kappa^6, nsub = 6) are
// filled, the other levels are zero.  io: momentum origin (1-based); ir = +-1.
void oq_twvev(const oq_geom* g, const double* u, double kappa, double delta, const int io[3],
              int dobndry, int ir, int nsub, int nmom, int nop, double* Jvev);
// The opertemp contributions of the listed sites (1-based lexicographic):
// opertemp[((isb * 5 + ix) * nt + t) * 12 + op], ix 0..4, op 0..11, isb 0..1.
void oq_twvev_sites(const oq_geom* g, const double* u, double kappa, double delta,
                    const int io[3], int dobndry, int ir, int nsub, const int* sites,
                    int nsites, double* opertemp);

// ---- gauge field helpers ----
// Eigenmode subtraction of the Wilson loop driver (eigen.cpp).  R, L: room for
// nGMRES[1] modes of two reference-layout halves each; evals: 2 nGMRES[1].
int oq_eigmodes(const oq_geom* g, const double* u, int kind, const int nGMRES[2], int ncycles,
                const double kappa[2], const double* se, const double* so, double* R, double* L,
                double* evals, int* cycles);
void oq_xigenerator(const oq_geom* g, const double* u, int numEV, double kappa, const double* R,
                    const double* L, int gammaid, double* xiinv);
void oq_eigaverage(const oq_geom* g, const double* u, int numEV, int eigstart, int eigstep,
                   const double* ze, const double* zo, double kappa, const double* R,
                   const double* L, const double* scal, int eshfes, double* Jtime);

void oq_loop_slices(const oq_geom* g, const double* u, const double* be, const double* bo,
                    const double* ye, const double* yo, int ksub, double kappa, double* J);
void oq_ppcoeffs(const oq_geom* g, const double* u, const double* be, const double* bo, double kappa,
                 int p, double* co);
void oq_ppaverage(const oq_geom* g, const double* u, int p, const double* co, const double* be,
                  const double* bo, const double* xe, const double* xo, double kappa, int nsub,
                  double* Jtime);
void oq_xipolygenerator(const oq_geom* g, const double* u, int numEV, double kappa, const double* R,
                        const double* L, const double* co, double* xiinv);
void oq_generalaverage(const oq_geom* g, const double* u, int n1, const double* R1, const double* L1,
                       const double* ev1, int n2, const double* R2, const double* ev2,
                       const double* ze, const double* zo, const double* xe, const double* xo,
                       double kappa, int eigstart, int eigstep, const double* co11, const double* co8,
                       const double* co5, const double* copoly, double* Jave);

// Sink smearing and the correlators of mesoncorr (meson.cpp).  q, qbar: 12 columns of two
// reference-layout halves; corrRe, corrIm(nt, -4:4, -4:4, -4:4, 28).
void oq_smear(const oq_geom* g, const double* u, double* he, double* ho, const double* ge,
              const double* go, double asmear, int nsmear);
void oq_mesoncorr(const oq_geom* g, const double* q, const double* qbar, const int src[4], int channels,
                  double* corrRe, double* corrIm);

void oq_coldstart(const oq_geom* g, double* u);
// The reference's pseudo-heatbath for the Wilson plaquette action at beta (sweep
// C/cfgsprops.f90:1973-2001, staple G/gaugetools.f90:39-345, phbup / su2up / sprd1
// G/heatbath.f90:33-467), drawing from the lagfib stream; u in place.  plaq (nsweeps
// entries, may be NULL) receives the average plaquette after each sweep.
void oq_heatbath(const oq_geom* g, double* u, double beta, int nsweeps, int nhit, double* plaq);
double oq_aveplaq(const oq_geom* g, const double* u);

#ifdef __cplusplus
}
#endif
