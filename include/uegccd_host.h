/*
 * uegccd_host.h -- host side of the drop-in: the reference's Input reader and
 * plane-wave set-up, which produce the UegccdSystem that the hot path takes.
 *
 * These replace, on a host without the Fortran build, the set-up the
 * reference's ZCode runs before DrvMBPT/DrvCCD/DrvdRPA: ReadInput (IO.f90:14),
 * init_HEG (HEG.f90:16), change_rs (HEG.f90:494), ChangeTwist (HEG.f90:551)
 * and FindTol (HEG.f90:1073).  A Fortran host keeps its own set-up and calls
 * only include/uegccd.h.
 */
#ifndef UEGCCD_HOST_H
#define UEGCCD_HOST_H

#include <stdint.h>

#include "uegccd.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Input file values (IO.f90:78-121).  range_flags is the sum of |"... Range"|. */
typedef struct {
    int32_t nelectron, maxkpoint;
    double rsmin, rsmax;
    int32_t num_rs_points, safe_eri;
    int32_t do_ring, do_xring, do_ladder, do_mosaic;
    int32_t range_flags;
    double ntwist[3];
    double core_factor;
    int32_t tacalcn, do_calc_ta_ccd, do_drpa_sosex, do_ks;
    double madelung_factor;
    int32_t do_single_calc;
    double gap, fcut, corefcut;
    int32_t fcut2ecut;
    double gapii;
    int32_t do_skip_ta;
    int32_t do_sf_calc_mp2;          /* DoSFCalcMP2: fort.80 block of the start amplitudes in DrvCCD */
    int32_t do_sf_calc_ccd;          /* DoSFCalcCCD: fort.80 block of the converged amplitudes        */
    int32_t do_only_mp2_grid;        /* DoOnlyMP2Grid: stop after the first DrvMBPT (MP2.f90:152-154) */
    int32_t core_factor_set;         /* the Input sets CoreFactor (ReadInput then writes fort.61)    */
    int32_t range_uniform;           /* the value of all fifteen "... Range" flags, -1 if they differ */
    UegccdRangeTerms range_terms;    /* the fifteen "... Range" values themselves                     */
} UegccdInput;

typedef struct {
    int32_t nocc, nao, maxkpoint, cell, core_n;
    double L, omega, madelung, ehf;
    double twist[3];
} UegccdHegInfo;

typedef struct UegccdHeg UegccdHeg;

void uegccd_default_input(UegccdInput *in);
/* ReadInput (IO.f90:14-348).  require_all = 1 enforces "every key set exactly once"
 * (IO.f90:329-335); 0 accepts the older key sets of the benchmark Inputs, with defaults. */
int uegccd_read_input(const char *path, int32_t require_all, UegccdInput *in);
/* init_HEG + change_rs(rSMin) */
int uegccd_heg_create(const UegccdInput *in, UegccdHeg **out);
void uegccd_heg_destroy(UegccdHeg *h);
int uegccd_heg_change_twist(UegccdHeg *h, const double twist[3]);
int uegccd_heg_set_eigen(UegccdHeg *h, const double *eigen);
/* The system view; its arrays stay owned by h (valid until the next change). */
int uegccd_heg_system(const UegccdHeg *h, UegccdSystem *sys);
int uegccd_heg_info(const UegccdHeg *h, UegccdHegInfo *info);
/* ChangeTwist (HEG.f90:551-578) for many twists at once, on the current CUDA device: for
 * each of the ntwist twists (3 doubles each, units of 2 pi/L) the basis SetupBasis picks
 * (HEG.f90:150-324: the |n|^2 <= MaxKPoint candidates stably sorted by |n + k_s|^2, cut by
 * fcut and corefcut), its HF eigenvalues (HEG.f90:581-603) and E_HF (print_HF, as
 * uegccd_heg_info reports it), at h's current rS.  Writes nvec (ntwist x NAO x 3, each
 * twist column-major like HEGData%nVec), eigen (ntwist x NAO) and ehf (ntwist, may be NULL);
 * every value is bit-equal to uegccd_heg_change_twist's.  h is not changed (and writes no
 * fort.60 lines).  At most 4096 candidates. */
int uegccd_heg_twists(const UegccdHeg *h, int32_t ntwist, const double *twists, int32_t *nvec, double *eigen,
                      double *ehf);
void uegccd_find_tol(double rs, double *tolmax, double *failratio, double *denomfactor);
/* print_ex_SF (HEG.f90:617-674): pair counts ExSf and ExV = (1/Omega) 4 pi/|k_l1-k_l2|^2
 * over ordered pairs l1 != l2 of occupied orbitals, on the grid of q = n_l1 - n_l2 with
 * |q_d| <= maxq, column-major from -maxq (side 2*maxq+1).  Sets *maxq; either grid may be
 * NULL (both NULL: only *maxq). */
int uegccd_heg_exchange_sf(const UegccdHeg *h, int32_t *maxq, int32_t *ex_sf, double *ex_v);
const char *uegccd_host_last_error(void);

/* ---- The ZCode program (Main.f90:2-320) ------------------------------------ */

#define UEGCCD_CONN_LIMIT 400   /* ConnectivityLimit, MP2.f90:26 */

/* Connectivity histogram of one basis (MP2.f90:56-87): conn[q-1] counts the allowed
 * excitations ij->ab outside the core (every index >= core_n) with |n_i - n_a|^2 = q,
 * plus those with |n_i - n_b|^2 = q.  conn has UEGCCD_CONN_LIMIT entries. */
int uegccd_connectivity(const UegccdSystem *sys, int32_t core_n, int32_t *conn);
/* Special twist (Main.f90:176,213-231): conn holds ntwists histograms; writes the
 * average histogram (conn_avg, UEGCCD_CONN_LIMIT, may be NULL), each twist's weighted
 * squared distance sum_q ((conn_q - avg_q)/q^2)^2 (diff2, ntwists, may be NULL) and
 * the index of the first twist with the smallest distance. */
int uegccd_special_twist(int32_t ntwists, const int32_t *conn, double *conn_avg, double *diff2, int32_t *best);
/* One REAL(8) item of gfortran list-directed output (write(u,*)), as fort.59 holds
 * them: a blank, then 17 significant digits in a G25 field.  Returns its length. */
int32_t uegccd_list_real(double x, char *buf, int32_t len);
/* The whole program in the working directory: reads input_path (NULL: "Input"),
 * writes Output, fort.58, fort.59, fort.60, fort.61, the structure factors fort.81 (every
 * DrvMBPT) and fort.82 (every print_HF), and fort.80 when DoSFCalcMP2/DoSFCalcCCD
 * are set.  twists_path (may be NULL) lists the twist
 * angles of the average, three numbers per line; missing ones are drawn from a
 * seeded U[-0.5,0.5)^3 stream.  scheme is UEGCCD_REPLAY or UEGCCD_DIIS.  The
 * solves run on the current CUDA device; every twist of the average is one batch. */
int uegccd_zcode(const char *input_path, const char *twists_path, int32_t scheme);
/* The set-up part of the program alone, on the host (no GPU): the fort.60 log that
 * uegccd_zcode writes (the reference's write(60,*) lines of HEG.f90 and Main.f90),
 * into out_path (NULL: "fort.60"). */
int uegccd_zcode_fort60(const char *input_path, const char *twists_path, const char *out_path);
/* The same with the exchange structure factors (fort.82) of the set-up into
 * fort82_path and ReadInput's core/active electron counts (fort.61, IO.f90:233-234,
 * written when the Input sets CoreFactor) into fort61_path as well (NULL: not written). */
int uegccd_zcode_host_logs(const char *input_path, const char *twists_path, const char *fort60_path,
                           const char *fort82_path, const char *fort61_path);
const char *uegccd_zcode_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
