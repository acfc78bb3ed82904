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
    int32_t diagnostics_requested;   /* DoSFCalcMP2/CCD or DoOnlyMP2Grid set (not on the GPU path) */
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
void uegccd_find_tol(double rs, double *tolmax, double *failratio, double *denomfactor);
const char *uegccd_host_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
