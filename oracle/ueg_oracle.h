/*
 * ueg_oracle.h -- CPU oracle for the uegCCD coupled-cluster path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a loop-for-loop C restatement of the
 * reference Fortran (shepherd-group/uegccd, the .f90 files under source).  It is the checker
 * for the CUDA path and the timed CPU baseline; nothing in the product
 * (the uegccd_b200 package and its CUDA library) links, imports or calls it.
 *
 * Parity pin: the restatement reproduces the reference's committed golden
 * outputs (benchmarks/ZRun-dRPA/Output, source/Test/Output, source/Test/fort.59,
 * benchmarks/ZRun-v6-N14/fort.59); see tests/test_oracle_golden.py.
 *
 * Array conventions follow the Fortran: amplitude arrays are
 * T(NOcc,NOcc,NOcc+1:NAO) column-major, i.e. element (i,j,a) (1-based, a>NOcc)
 * sits at (i-1) + O*(j-1) + O*O*(a-O-1).
 */
#ifndef UEG_ORACLE_H
#define UEG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Values of the reference's Input file (IO.f90:78-121, Types.f90:29-82).  */
typedef struct {
    int    nelectron;
    int    maxkpoint;          /* "Momentum Cutoff" (overridden by fcut2ecut) */
    double rsmin, rsmax;
    int    num_rs_points;
    int    safe_eri;
    int    do_ring, do_xring, do_ladder, do_mosaic;
    /* range flags, in the order of Types.f90:36-50 */
    int    irange_ring, irange_xring, irange_ladder, irange_mosaic;
    int    irange_driver_direct, irange_driver_exchange, irange_energy;
    int    irange_lin_rings, irange_quad_rings, irange_direct_rings, irange_exchange_rings;
    int    irange_lin_ladders, irange_quad_ladders, irange_direct_ladders, irange_exchange_ladders;
    double ntwist[3];
    double core_factor;
    int    tacalcn;
    int    do_calc_ta_ccd;
    int    do_drpa_sosex;
    int    do_ks;
    double madelung_factor;
    int    do_single_calc;
    double gap;
    double fcut;
    double corefcut;
    int    fcut2ecut;
    double gapii;
    int    do_skip_ta;
} UoInput;

typedef struct UoCtx UoCtx;

/* Per-solve result of the CCD / dRPA drivers (CCD.f90:18-183, dRPA.f90:23-174). */
typedef struct {
    double ecorr;        /* Ec(CCD) or Ec(dRPA) at exit                     */
    double ecorr_sosex;  /* Ec(SOSEX) (dRPA only, when converged)           */
    double max_res;      /* MaxRes of the final residual check              */
    double last_dt;      /* dT of the last iteration                        */
    int    niter;        /* NIter at exit                                   */
    int    fail;         /* MaxRes > FailRatio*TolMax                        */
    int    n_recorded;   /* number of per-iteration energies written        */
} UoSolveStats;

/* Set-up: ReadInput-derived values (IO.f90) -> init_HEG (HEG.f90:16-43) ->
 * SetPointers (Main.f90:274-318) -> change_rs (HEG.f90:494-533).  NULL on a
 * condition where the reference calls Stop; the message is in uo_last_error(). */
UoCtx *uo_create(const UoInput *in);
void   uo_destroy(UoCtx *c);
const char *uo_last_error(void);

int    uo_nocc(const UoCtx *c);
int    uo_nao(const UoCtx *c);
int    uo_cell(const UoCtx *c);
int    uo_maxkpoint(const UoCtx *c);
/* L, Omega, Madelung, EHF, current twist (3) */
void   uo_scalars(const UoCtx *c, double out[7]);
void   uo_get_eigen(const UoCtx *c, double *eigen);       /* NAO */
void   uo_set_eigen(UoCtx *c, const double *eigen);       /* NAO */
void   uo_get_nvec(const UoCtx *c, int *nvec);            /* NAO x 3, row p = orbital p+1 */
void   uo_get_kvec(const UoCtx *c, double *kvec);         /* NAO x 3 */
/* ChangeTwist (HEG.f90:551-578) to an explicit twist. */
int    uo_change_twist(UoCtx *c, const double twist[3]);

/* DrvMBPT (MP2.f90:11-157) without the structure-factor dump.  conn (400) may be NULL. */
double uo_mp2(UoCtx *c, double *t_aaaa, double *t_abab, double *t_abba, int *conn);
/* DrvCCD (CCD.f90:18-183).  energies/dts (may be NULL) get one entry per printed line. */
int    uo_ccd(UoCtx *c, double *t_aaaa, double *t_abab, double *t_abba,
              int max_iter_override, UoSolveStats *st, double *energies, double *dts, int max_rec);
/* Test hook: TolMax for uo_ccd below the reference's 1e-8 (tight-mode parity); <= 0 restores it. */
void   uo_set_tol_override(double tol);
/* DrvdRPA (dRPA.f90:23-174) on one amplitude array. */
int    uo_drpa(UoCtx *c, double *t2, int max_iter_override, UoSolveStats *st,
               double *energies, double *dts, int max_rec);

/* One CCD residual evaluation, TermsWrapper (CCD.f90:146-181) without GetRes:
 * g_abab/g_abba receive G2 of the terms selected by term_mask
 * (bit0 drivers, bit1 mosaics, bit2 ladders, bit3 rings, bit4 xrings). */
void   uo_ccd_g2(UoCtx *c, const double *t_abab, const double *t_abba, int term_mask,
                 double *g_abab, double *g_abba);
/* dRPA residual G2 (dRPA.f90:144-172), bit0 drivers, bit1 mosaics, bit3 rings. */
void   uo_drpa_g2(UoCtx *c, const double *t2, int term_mask, double *g2);
/* CCEnergy (CCD.f90:186-237) and dRPA CCEnergy (dRPA.f90:181-216). */
double uo_ccd_energy(UoCtx *c, const double *t_aaaa, const double *t_abab, const double *t_abba);
double uo_drpa_energy(UoCtx *c, const double *t2, double csosex);

/* Structure factors.  uo_sf_length: SfLength of SendForAllocation (HEG.f90:1051-1065).
 * uo_structure_factor: the grids of CCEnergyAndSF (CCD.f90:240-351) -- SfSum, SfG, SfV,
 * SfDSum, SfXSum, each (2S+1)^3 column-major from -S, NULL to skip -- whose first
 * three are also DrvMBPT's (MP2.f90:86-117); returns ECorr.  uo_exchange_sf:
 * print_ex_SF (HEG.f90:617-674); returns maxq, grids (2*maxq+1)^3 when non-NULL. */
int    uo_sf_length(const UoCtx *c);
double uo_structure_factor(UoCtx *c, const double *t_aaaa, const double *t_abab, const double *t_abba,
                           double *sf_sum, double *sf_g, double *sf_v, double *sf_dsum, double *sf_xsum,
                           int *oob);
int    uo_exchange_sf(const UoCtx *c, int *ex_sf, double *ex_v);

/* Twist-average driver (Main.f90:99-255) over an explicit twist list.
 * per_twist: ntw x 3 (hf, mp2, ccd).  special: the chosen twist (3).
 * final_st: the special-twist solve (CCD or dRPA by Input). */
int    uo_twist_average(UoCtx *c, int ntw, const double *twists, double *per_twist,
                        double *special, UoSolveStats *final_st, double *final_mp2);

#ifdef __cplusplus
}
#endif
#endif
