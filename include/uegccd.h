/*
 * uegccd.h -- C ABI of the B200 coupled-cluster path for the uniform electron gas.
 *
 * The entry points replace the Fortran module procedures of the reference
 * (shepherd-group/uegccd) on the MP2 / CCD / dRPA hot path.  They take plain
 * pointers in the reference's own layout so that a Fortran host can bind them
 * with iso_c_binding:
 *
 *   amplitude arrays  T(NOcc, NOcc, NOcc+1:NAO), FP64, column-major, i.e. element
 *                     (i,j,a) (1-based, a > NOcc) at (i-1) + O*(j-1) + O*O*(a-O-1);
 *   nVec              HEGData%nVec(NAO,3), int32, column-major: (p,d) at (p-1) + NAO*(d-1);
 *   Eigen             HEGData%Eigen(NAO), FP64.
 *
 * Every function returns an int status: 0 ok, > 0 not converged, < 0 error
 * (the message is in uegccd_last_error()).  The reference calls Stop or prints
 * "DID NOT CONVERGE" in these places (CCD.f90:107-114, dRPA.f90:100-107); a host
 * shim maps the statuses back to those messages.
 *
 * Calls on one context are serialised on that context's CUDA stream; separate
 * contexts may be used from separate threads.  All device memory a call needs is
 * allocated when the context is created (or grown on first use) and freed by
 * uegccd_ctx_destroy.  There is no CPU fallback: without a CUDA device of compute
 * capability 10.0 every call fails with UEGCCD_ERR_CUDA.
 */
#ifndef UEGCCD_H
#define UEGCCD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    UEGCCD_OK = 0,
    UEGCCD_NOT_CONVERGED = 1,        /* MaxRes > FailRatio*TolMax, or MaxIter reached */
    UEGCCD_ERR_ARG = -1,             /* bad argument (null pointer, size, option)      */
    UEGCCD_ERR_CUDA = -2,            /* CUDA error or no usable device                 */
    UEGCCD_ERR_ALLOC = -3,           /* device or host allocation failed               */
    UEGCCD_ERR_UNSUPPORTED = -4,     /* Input option outside the GPU path (see below)  */
    UEGCCD_ERR_NUMERIC = -5          /* NaN/Inf in the amplitudes or the energy        */
};

/* Precision of the residual contractions. */
enum { UEGCCD_FP64 = 0, UEGCCD_MIXED = 1 };
/* Iteration scheme: REPLAY reproduces the reference iteration (1/2-damped Jacobi,
 * CCD.f90:380, with its DIIS that never extrapolates, DIISCC.f90:110-115);
 * DIIS runs a Pulay extrapolation over ndiis vectors (new in this library). */
enum { UEGCCD_REPLAY = 0, UEGCCD_DIIS = 1 };

/* The plane-wave system, i.e. the fields of HEGDataType / UEGInfoType
 * (Types.f90:7-82) that the hot path reads. */
typedef struct {
    int32_t nocc;            /* UEGInfo%NOcc                                 */
    int32_t nao;             /* UEGInfo%NAO                                  */
    double L;                /* HEGData%L (box length)                       */
    double madelung;         /* HEGData%Madelung; V(q=0) = -Madelung         */
    const double *eigen;     /* HEGData%Eigen(NAO)                           */
    const int32_t *nvec;     /* HEGData%nVec(NAO,3), column-major            */
} UegccdSystem;

/* Run options; uegccd_default_options() fills the reference's values. */
typedef struct {
    int32_t do_ring, do_xring, do_ladder, do_mosaic;   /* Input "Do Rings" ... (IO.f90:170-180)   */
    int32_t core_n;          /* UEGInfo%CoreN: integrals with an orbital <= CoreN are zero (CAS) */
    double gapii;            /* UEGInfo%GapII: integrals above GapII are zero when GapII > 0     */
    int32_t range_flags;     /* sum of |"... Range"| Input values where CasedERI applies them;   */
                             /* non-zero: CCD on the batch's uniform range flag (set_range)      */
    int32_t max_iter;        /* MaxIter, 1000 (CCD.f90:36)                                      */
    double tol;              /* TolMax on max|dT|, 1e-8 (HEG.f90:1078)                          */
    double denom_factor;     /* DenomFactor, 2 (CCD.f90:11)                                     */
    double fail_ratio;       /* FailRatio, 100 for CCD (HEG.f90:1079), 1e4 for dRPA (dRPA.f90:100) */
    int32_t scheme;          /* UEGCCD_REPLAY or UEGCCD_DIIS                                    */
    int32_t ndiis;           /* DIIS vectors for UEGCCD_DIIS (2..16)                            */
    int32_t precision;       /* UEGCCD_FP64 or UEGCCD_MIXED                                     */
    int32_t refine_sweeps;   /* MIXED: FP64 residual sweeps kept at the end                     */
    double *energies;        /* optional: per-iteration energy, as printed to Output            */
    double *dts;             /* optional: per-iteration max|dT|                                 */
    int32_t max_rec;         /* capacity of energies/dts                                        */
} UegccdOptions;

typedef struct {
    double ecorr;            /* Ec(CCD) / Ec(dRPA) (HEGData%ECorr at exit)                      */
    double ecorr_sosex;      /* Ec(SOSEX) (dRPA only)                                           */
    double max_res;          /* max |R| of the final residual (CCD.f90:105)                     */
    double last_dt;          /* max |dT| of the last iteration                                  */
    int32_t niter;           /* NIter at exit                                                   */
    int32_t fail;            /* MaxRes > FailRatio*TolMax                                       */
    int32_t n_recorded;      /* entries written to energies/dts                                 */
    int32_t kernel_launches; /* CUDA kernels this call launched                                 */
    double gpu_ms;           /* device time of the call (CUDA events)                           */
    int32_t status;          /* this solve's status: UEGCCD_OK, UEGCCD_NOT_CONVERGED (MaxIter or  */
                             /* MaxRes > FailRatio*TolMax) or UEGCCD_ERR_NUMERIC (NaN/Inf); a     */
                             /* batch call returns the worst of them                              */
    int32_t ndiis;           /* DIIS vectors used: opt->ndiis, or fewer (down to 2) when device   */
                             /* memory or the library's limit held no more, as SetUpDIISCC steps  */
                             /* its NDIIS down until Allocate succeeds (DIISCC.f90:22-29); 0 for  */
                             /* UEGCCD_REPLAY                                                     */
} UegccdResult;

typedef struct UegccdCtx UegccdCtx;

/* Defaults of FindTol at HEGData%rS = 1 (HEG.f90:1073-1086) and of the Input
 * switches (all terms on). */
void uegccd_default_options(UegccdOptions *opt);

/* Builds the momentum-block plan of one system on the current CUDA device and
 * uploads it.  The context (like a batch) stays on that device: every later call on it
 * runs there, from whichever host thread makes it, and leaves the thread's current device
 * as it found it.  Replaces the per-call FindIndex lookups (HEG.f90:357-404) and the
 * scratch set-up SetUpCCScr (CCScr.f90:9-31). */
int uegccd_ctx_create(const UegccdSystem *sys, UegccdCtx **out);
int uegccd_ctx_destroy(UegccdCtx *ctx);

/* Replaces the eigenvalues (the twist-averaged-eigenvalue solve, Main.f90:243). */
int uegccd_ctx_set_eigen(UegccdCtx *ctx, const double *eigen);

/* Integral options of the non-range-separated ERI routines that SetPointers selects
 * (Main.f90:274-318): core_n = UEGInfo%CoreN zeroes every integral with an orbital
 * <= CoreN (CoreERI, HEG.f90:835-888); gapii = UEGInfo%GapII > 0 zeroes every integral
 * above GapII (GapERI, HEG.f90:890-942); both together are NoCaseERI.  They hold for
 * every later call on the context (MP2, structure factors, G2 terms); uegccd_ccd and
 * uegccd_drpa set them from their options first.  Defaults 0 and 0: the plain integrals.
 * Amplitudes of core pairs (i or j <= CoreN) stay zero, as in the reference; amplitudes
 * passed in are read with their core pairs set to zero. */
int uegccd_ctx_set_integrals(UegccdCtx *ctx, int32_t core_n, double gapii);

/* Range-separated integrals with one flag for every CCD term (CasedERI, HEG.f90:689-774:
 * 1 short range, 2 long range, 3 none), as the reference computes them when all fifteen
 * "... Range" Input values equal flag under CasedERI.  The spin adaptation holds in that
 * case (direct and exchange integrals share the flag).  CCD solves whose options carry
 * range_flags != 0 then use the flag's integrals for every term and the energy (CCD.f90:
 * 216-217, 491-492, 555-556, 620-917); the MP2 start keeps the plain integrals
 * (MP2.f90:61-62).  screening = HEGData%ScreeningDistance (HEG.f90:512).  flag 0 clears.
 * Terms with different flags, and range-separated dRPA, take uegccd_ctx_set_eri below. */
int uegccd_ctx_set_range(UegccdCtx *ctx, int32_t flag, double screening);

/* ---- the two-channel form: per-term integral flags, Do Rings without Do XRings ----------
 * The reference iterates T2abab and T2abba (CCD.f90:18-183) and gives each integral of each
 * CCD term its own range flag, the Max(...) of the term's flags (CCD.f90:620-937).  Once a
 * term's direct and exchange integrals differ, or only one of Do Rings / Do XRings is on,
 * T2abba(i,j,a) = -T2abab(i,j,b) no longer holds.  The two-channel form keeps both arrays as
 * the reference does, in its layout, with per-integral flag tables.
 *
 * The fifteen "... Range" Input values (UEGInfo%IRange*, read in IO.f90), as CasedERI
 * applies them (HEG.f90:689-774): 0 Coulomb, 1 short range, 2 long range, 3 none. */
typedef struct {
    int32_t ring, xring, ladder, mosaic, driver_direct, driver_exchange, energy;
    int32_t lin_rings, quad_rings, direct_rings, exchange_rings;
    int32_t lin_ladders, quad_ladders, direct_ladders, exchange_ladders;
} UegccdRangeTerms;

/* SetPointers in full (Main.f90:274-318): with the options' core_n and gapii, the flags and
 * Safe ERI pick CasedERI (Safe ERI, or flags, GapII and CoreN all set), NoCaseERI, CoreERI,
 * GapERI or BaseERI, and every later uegccd_ccd, uegccd_drpa, uegccd_ccd_g2_2ch and
 * uegccd_drpa_g2 on the context runs the two-channel (dRPA: general-flag) form with them.
 * screening = HEGData%ScreeningDistance (HEG.f90:512), > 0 when a flag is 1 or 2.  Flags
 * outside 0..3 return UEGCCD_ERR_ARG; flags == NULL returns the context to the spin-adapted
 * kernels.  Without this call, uegccd_ccd takes the two-channel form by itself when
 * do_ring != do_xring (with the integrals of core_n and gapii). */
int uegccd_ctx_set_eri(UegccdCtx *ctx, const UegccdRangeTerms *flags, int32_t safe_eri, double screening);

/* TermsWrapper (CCD.f90:146-181) on both channels in the two-channel form, with the
 * integrals of the last uegccd_ctx_set_eri (none: the context's core_n / gapii integrals):
 * G2abab and G2abba of the terms in term_mask (as uegccd_ccd_g2), reference layout. */
int uegccd_ccd_g2_2ch(UegccdCtx *ctx, const double *t_abab, const double *t_abba, int32_t term_mask,
                      double *g_abab, double *g_abba);
/* The dRPA residual G2 (dRPA.f90:339-551: bit0 drivers, bit1 mosaics, bit3 rings) of one
 * amplitude array, with the same integrals. */
int uegccd_drpa_g2(UegccdCtx *ctx, const double *t2, int32_t term_mask, double *g2);

/* DrvMBPT (MP2.f90:11-157): writes the MP2 amplitudes T2aaaa/T2abab/T2abba (each
 * may be NULL) and E(2).  Its structure factor is uegccd_structure_factor of T2abab. */
int uegccd_mp2(UegccdCtx *ctx, double *t_aaaa, double *t_abab, double *t_abba, double *e2);

/* DrvCCD (CCD.f90:18-183): iterates from the amplitudes given (the MP2 guess in
 * Main.f90:85-89) and writes the converged amplitudes back in place.  With do_ring ==
 * do_xring and no uegccd_ctx_set_eri, the library stores the spin-adapted amplitude T2abab
 * alone, with T2abba(i,j,a) = -T2abab(i,j,b) and T2aaaa = T2abab + T2abba, which the
 * reference's equations keep only when rings and crossed rings are both on or both off.
 * Otherwise it runs the two-channel form: t_abba is read as given (NULL: from t_abab by the
 * MP2 relation) and all three arrays are written back. */
int uegccd_ccd(UegccdCtx *ctx, const UegccdOptions *opt, double *t_aaaa, double *t_abab,
               double *t_abba, UegccdResult *res);

/* DrvdRPA (dRPA.f90:23-174) on one amplitude array (the caller passes T2aaaa of
 * the MP2 step, Main.f90:91); returns Ec(dRPA) and Ec(SOSEX).  After uegccd_ctx_set_eri
 * each term takes its own flag; the energy keeps flag 0 (dRPA.f90:206-207). */
int uegccd_drpa(UegccdCtx *ctx, const UegccdOptions *opt, double *t2, UegccdResult *res);

/* One CCD residual G2 of the selected terms (TermsWrapper, CCD.f90:146-181; bit0
 * drivers, bit1 mosaics, bit2 ladders, bit3 rings, bit4 crossed rings) for
 * spin-adapted amplitudes t_abab; writes G2abab in the reference layout. */
int uegccd_ccd_g2(UegccdCtx *ctx, const double *t_abab, int32_t term_mask, double *g_abab);
/* The same in a chosen precision: UEGCCD_MIXED forms the particle-particle ladder on
 * the tensor cores (FP16 operands, FP32 accumulation) from t itself. */
int uegccd_ccd_g2_ex(UegccdCtx *ctx, const double *t_abab, int32_t term_mask, int32_t precision,
                     double *g_abab);

/* ---- structure factors ----------------------------------------------------------
 * The amplitude sums that CCEnergyAndSF (CCD.f90:240-351; fort.80) and DrvMBPT
 * (MP2.f90:86-117; fort.81) accumulate over the momentum transfers q = n_a - n_i,
 * on the reference's grid Sf(-S:S,-S:S,-S:S) with S = uegccd_sf_length(sys)
 * (SfLength of SendForAllocation, HEG.f90:1051-1065).  Column-major like the
 * Fortran array: q = (x,y,z) at (x+S) + W*(y+S) + W*W*(z+S), W = 2S+1.  Each pointer
 * may be NULL; the others receive W^3 doubles:
 *   sum   SfSum:  T2aaaa+T2abab added at q = n_a-n_i, T2aaaa+T2abba subtracted at n_a-n_j
 *   dsum  SfDSum: 2*T2abab added, 2*T2abba subtracted
 *   xsum  SfXSum: T2aaaa-T2abab added, T2aaaa-T2abba subtracted
 *   g     SfG:    |q|*2*pi/L at every q that an allowed amplitude reaches, else 0
 *   v     SfV:    at the same points, the integral of the last amplitude reaching q in
 *                 the reference's loop order: V(q) of BaseERI (HEG.f90:969-976) with the
 *                 GapII filter, or 0 when that amplitude is a core pair; else 0
 * (MP2.f90 fills sum, g and v only.)  sum.v/2 is the correlation energy of the
 * amplitudes.  A transfer outside the grid returns UEGCCD_ERR_ARG. */
typedef struct {
    double *sum, *dsum, *xsum, *g, *v;
} UegccdSfGrid;
/* S = 2*maxval(nVec)+1 (host-only), or < 0 on a bad argument. */
int32_t uegccd_sf_length(const UegccdSystem *sys);
/* The structure factor of spin-adapted amplitudes t_abab (reference layout). */
int uegccd_structure_factor(UegccdCtx *ctx, const double *t_abab, const UegccdSfGrid *out);

/* ---- DIIS for a host-side iteration loop (DIISCC.f90:10-155) -------------------
 * A history of ndiis (T, R) pairs of n amplitudes on the device, one object per
 * amplitude channel (the reference keeps one for T2abab and one for T2abba).
 *   uegccd_diis_create  SetUpDIISCC: t0 (may be NULL) is the newest T until the first push.
 *   uegccd_diis_push    the pair of this iteration: T after the update, R = -G + D.T
 *                       (what CnvrgCC and GetRes store); the oldest pair is dropped.
 *   uegccd_diis_get_t   GetTFromDIIS: the next T into t2.  UEGCCD_REPLAY gives the
 *                       newest T, as the reference's singular solve does
 *                       (DIISCC.f90:110-125); UEGCCD_DIIS extrapolates over the
 *                       pairs held once niter >= ndiis + 5 (the reference's IWait):
 *                       B(i,j) = R(i).R(j), [B 1; 1 0][c; y] = [0; 1], T = sum c(i) T(i);
 *                       a singular B gives the newest T.
 *   uegccd_diis_destroy ShutDownDIISCC.
 * Arrays are host arrays of n doubles (any layout, the same in every call). */
typedef struct UegccdDiis UegccdDiis;
int uegccd_diis_create(int64_t n, int32_t ndiis, int32_t scheme, const double *t0, UegccdDiis **out);
int uegccd_diis_push(UegccdDiis *d, const double *t, const double *r);
int uegccd_diis_get_t(UegccdDiis *d, int32_t niter, double *t2);
int uegccd_diis_destroy(UegccdDiis *d);

/* ---- many independent solves in one launch per residual term ---------------- */
typedef struct UegccdBatch UegccdBatch;

/* A batch of n systems (twists, rs points, basis sizes); each keeps its own
 * momentum blocks.  Amplitudes stay on the device between calls. */
int uegccd_batch_create(const UegccdSystem *systems, int32_t n, UegccdBatch **out);
int uegccd_batch_destroy(UegccdBatch *b);
/* MP2 start + CCD (or dRPA when drpa != 0) of every system; results[n].  CCD with do_ring !=
 * do_xring runs each system in turn in the two-channel form (with the batch's uniform range flag,
 * if any); the batch then holds each solve's T2abab, and uegccd_batch_structure_factor refuses. */
int uegccd_batch_solve(UegccdBatch *b, const UegccdOptions *opt, int32_t drpa, double *e2,
                       UegccdResult *results);
/* An incremental solve, for a serving loop that hands each result back as soon as its solve
 * stops (the reference has no counterpart: Main.f90:112-168 solves one twist after another).
 * uegccd_batch_start runs the MP2 start of every system (e2[n] may be NULL) and opens the
 * iteration with the options of uegccd_batch_solve.  Each uegccd_batch_advance runs up to
 * `rounds` rounds of four iterations of the solves still iterating, then reports every solve
 * that stopped since the previous call -- converged, at MaxIter, or on a NaN: its index in
 * done_ids and its result in done_results (room for n of each), *n_done of them, with its
 * final residual (MaxRes, CCD.f90:103-107) formed at that point.  *n_active counts the solves
 * still iterating; 0 closes the solve.  Converged solves cost nothing more: their kernels
 * return at once.  Each solve's iterations, energy and MaxRes are those of uegccd_batch_solve.
 * FP64 only: UEGCCD_MIXED and range flags return UEGCCD_ERR_UNSUPPORTED. */
int uegccd_batch_start(UegccdBatch *b, const UegccdOptions *opt, int32_t drpa, double *e2);
int uegccd_batch_advance(UegccdBatch *b, int32_t rounds, int32_t *n_active, int32_t *n_done, int32_t *done_ids,
                         UegccdResult *done_results);
/* uegccd_ctx_set_integrals for every system of the batch (uegccd_batch_solve sets
 * them from its options first). */
int uegccd_batch_set_integrals(UegccdBatch *b, int32_t core_n, double gapii);
/* The same for every solve of a batch. */
int uegccd_batch_set_range(UegccdBatch *b, int32_t flag, double screening);
/* DrvMBPT for every system: the MP2 amplitudes stay in the batch (what
 * uegccd_batch_structure_factor and uegccd_batch_get_amplitudes then read); e2[n]
 * may be NULL. */
int uegccd_batch_mp2(UegccdBatch *b, double *e2);
/* The structure factor of solve s from the amplitudes the batch holds: the MP2 ones
 * after uegccd_batch_mp2, the converged ones after a CCD uegccd_batch_solve (not
 * after a dRPA solve, whose amplitude is T2aaaa). */
int uegccd_batch_structure_factor(UegccdBatch *b, int32_t s, const UegccdSfGrid *out);
/* Copies solve s's amplitudes out in the reference layout (T2abab). */
int uegccd_batch_get_amplitudes(UegccdBatch *b, int32_t s, double *t_abab);
/* E(2) of one system with the plain integrals, as uegccd_mp2 computes it, with no device allocation: this
 * entry point has no counterpart in the reference.  It is for callers that cannot
 * allocate device memory when they call: a host whose device memory already belongs
 * to its own pool allocator, or one running other streams that must not be stalled
 * by the device-wide synchronisation a cudaFree brings.  All device storage is one
 * fixed array of 1.05 MB inside the library, so the system must have at most
 * 2048 orbitals and plane-wave components |n_d| <= 31; larger systems return
 * UEGCCD_ERR_ARG.  stream is a cudaStream_t (NULL: the legacy default stream); every
 * call synchronises stream and returns when e2 is written.  Every call on a device shares that array:
 * calls must not overlap on one device (from several streams or threads), or
 * their results are wrong.  The first call on a device looks up the array's
 * address (which may load the library's device code).  The address is kept until the
 * process exits: a cudaDeviceReset invalidates it, so do not use this entry point across one. */
int uegccd_mp2_energy_static(const UegccdSystem *sys, void *stream, double *e2);

/* T2abab of every solve of the batch in the reference layout, solve after solve: solve s
 * fills NOcc_s * NOcc_s * (NAO_s - NOcc_s) doubles (the batched form of
 * uegccd_batch_get_amplitudes: one device-to-host copy for the whole batch).  A
 * page-locked t_abab (cudaHostAlloc / cudaHostRegister) receives the copy directly;
 * pageable memory goes through a cached pinned buffer. */
int uegccd_batch_get_all_amplitudes(UegccdBatch *b, double *t_abab);
/* A destroyed batch leaves its device memory in a per-process cache (at most 32 GiB)
 * that the next batch reuses, and large amplitude downloads keep a pinned host staging
 * buffer; this returns both to the driver. */
int uegccd_trim_cache(void);

/* Solve s's per-iteration energies and biggest changes from the last batch solve (the
 * rows of the reference's iteration table, CCD.f90:76,96 / dRPA.f90:77,92): copies at
 * most max_rec of each (either pointer may be NULL) and sets *n_recorded. */
int uegccd_batch_history(UegccdBatch *b, int32_t s, double *energies, double *dts, int32_t max_rec,
                         int32_t *n_recorded);

/* CTA sizes of the ring kernel's pair classes (by padded pair size: <= 16, 32, 48 rows,
 * larger), as the launch-shape tuner picked them on the batch's first CCD solve (timed
 * on the batch itself, once per batch shape in a process; the CTA size leaves every
 * result bitwise the same).  Writes at most max values; returns how many. */
int32_t uegccd_batch_ring_threads(UegccdBatch *b, int32_t *threads, int32_t max);
/* Every launch shape the tuner picked on the batch's first CCD solve (new; the reference has
 * no launches): the four ring CTA sizes above, the CTA size of the ring staging kernel (64,
 * 128 or 256), the ladder tile order (0: block order, 1: the blocks with the most virtuals
 * first, within each row-tile class), and the column chunk of the hole-hole intermediate (64
 * or 32 virtuals per shared-memory stage).  None changes a result.  Writes at most max values;
 * returns how many. */
int32_t uegccd_batch_launch_shapes(UegccdBatch *b, int32_t *vals, int32_t max);

/* Live kernel timing: when on, every kernel of a batch solve is bracketed by CUDA
 * events on the batch's stream; stats return per-kernel total ms and launches. */
int uegccd_batch_set_profiling(UegccdBatch *b, int32_t on);
int32_t uegccd_batch_kernel_stats(UegccdBatch *b, int32_t max, const char **names, double *ms,
                                  int64_t *launches);

/* Device bytes one system needs inside a batch (tables, amplitudes, DIIS history of
 * ndiis vectors, mixed-precision buffers when mixed != 0) and its number of allowed
 * amplitudes: the admission measure of a serving loop.  Host-only, no device needed. */
int uegccd_footprint(const UegccdSystem *sys, int32_t ndiis, int32_t mixed, int64_t *bytes, int64_t *namp);

/* Device memory.  The library takes its device memory in chunks and keeps the chunks of
 * destroyed objects in a cache (uegccd_trim_cache).  uegccd_set_memory_limit caps the bytes
 * it holds on each device -- live batches and contexts plus that cache -- at `bytes` (0: no
 * cap, the default).  An allocation that would pass the cap first returns the device's cache
 * to the driver; if it still does not fit, the call fails with UEGCCD_ERR_ALLOC and the
 * batch keeps what it held before the call.  The reference has no such cap; its one
 * allocation-failure path is SetUpDIISCC, which steps the DIIS depth down until Allocate
 * succeeds and Stops when none does (DIISCC.f90:22-33): a DIIS solve here likewise takes
 * fewer history vectors (UegccdResult.ndiis) when the cap or the device holds no more.
 * uegccd_memory_info reports, for the current device, the bytes held and the cached part. */
int uegccd_set_memory_limit(int64_t bytes);
int uegccd_memory_info(int64_t *held, int64_t *cached);

/* Host<->device bytes the batch has moved since its creation (its upload included). */
int uegccd_batch_transfer_bytes(UegccdBatch *b, int64_t *h2d, int64_t *d2h);

const char *uegccd_last_error(void);
/* Library version string. */
const char *uegccd_version(void);

#ifdef __cplusplus
}
#endif
#endif
