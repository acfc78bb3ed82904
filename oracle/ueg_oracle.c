/*
 * ueg_oracle.c -- CPU oracle (test infrastructure, never product code).
 *
 * Loop-for-loop C restatement of the reference Fortran of shepherd-group/uegccd.
 * Every routine cites the reference file:line it restates.  Floating-point
 * expressions keep the Fortran evaluation order (left to right, ** before * /,
 * unary minus after them) so that the set-up values agree with the reference's
 * 16-digit printouts and the energies with its printed 12 digits.
 *
 * Third-party arithmetic restated here:
 *   - LAPACK DGESV (openblas, version unpinned in source/make.sh:75), called at
 *     DIISCC.f90:114 on an (NDIIS+1)^2 matrix.  Restated as LU with partial
 *     pivoting (first maximal |pivot| wins, as IDAMAX) that reports INFO>0 on an
 *     exactly zero pivot, which is the only outcome the reference's matrix allows.
 *   - gfortran rand()/srand() (HEG.f90:543-545, Main.f90:81) is NOT restated; the
 *     twist list is taken explicitly (the goldens list every twist).
 */
#include "ueg_oracle.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define PI 3.1415926535897932384626433833 /* Constants.f90:7 */
#define F12 0.5

static char g_err[512];
const char *uo_last_error(void) { return g_err; }
static void set_err(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

/* ------------------------------------------------------------------ types */

/* UEGInfoType subset (Types.f90:29-82) */
typedef struct {
    int nelectron, nocc, nao, maxkpoint, coren;
    int irange_ring, irange_xring, irange_ladder, irange_mosaic;
    int irange_driver_direct, irange_driver_exchange, irange_energy;
    int irange_lin_rings, irange_quad_rings, irange_direct_rings, irange_exchange_rings;
    int irange_lin_ladders, irange_quad_ladders, irange_direct_ladders, irange_exchange_ladders;
    double rs, exchangefactor, madelungfactor, gap, gapii, fcut, corefcut;
    int safe_eri, do_ring, do_xring, do_ladder, do_mosaic, do_drpa_sosex, do_calc_ta_ccd;
} Info;

/* HEGDataType (Types.f90:7-27) */
typedef struct {
    int nel, cell;
    double L, rS, omega, madelung, density, kf, screening;
    double ntwist[3], this_ntwist[3];
    double xhf, ehf, ecorr;
    double *kvec;   /* kvec(p,d) -> kvec[(p-1)*3+d-1] */
    double *eigen;  /* eigen(p)  -> eigen[p-1]        */
    int *nvec;      /* nvec(p,d) -> nvec[(p-1)*3+d-1] */
    int *kp2bf;     /* kPointToBasisFn(-cell:cell)^3  */
} Heg;

typedef double (*EriFn)(const UoCtx *, int a, int b, int i, int j, int flag);

struct UoCtx {
    Info info;
    Heg heg;
    EriFn eri;
    double denom_factor_ccd;   /* CCD.f90:11 module variable  */
    double denom_factor_drpa;  /* dRPA.f90:16 module variable */
};

#define NV(h, p, d) ((h)->nvec[((p)-1) * 3 + (d)-1])
#define KV(h, p, d) ((h)->kvec[((p)-1) * 3 + (d)-1])

static inline int tix(int O, int i, int j, int a) { return (i - 1) + O * (j - 1) + O * O * (a - O - 1); }

/* ---------------------------------------------------------- HEG.f90 set-up */

/* FcutToBasisFn (HEG.f90:326-342) */
static int fcut_to_basis_fn(double fcut, int nel)
{
    int m = (int)(pow(fcut, 3.0 / 2.0) * nel / 2);
    double target = pow(fcut, 3.0 / 2.0) * nel / 2;
    if (fabs(m - target) > fabs(m + 1 - target)) m = m + 1;
    return m;
}

/* CalcMadelung (HEG.f90:89-148).  Only the l4 = 10 pass survives the reset at
 * the top of each l4 pass, so that pass alone is evaluated (same loop order). */
static double calc_madelung(double omega, double L)
{
    double kappa = 2.8 / pow(omega, 1.0 / 3.0);
    double term2 = -PI / (pow(kappa, 2.0) * pow(L, 3.0));
    double term4 = -2.0 * kappa / sqrt(PI);
    const int l4 = 10;
    double recipsum2 = 0.0;
    for (int l1 = -l4; l1 <= l4; l1++)
        for (int l2 = -l4; l2 <= l4; l2++)
            for (int l3 = -l4; l3 <= l4; l3++) {
                int n2 = l1 * l1 + l2 * l2 + l3 * l3;
                double k2 = (1.0 / pow(L, 2.0)) * (double)n2;
                double ek2 = (1.0 / pow(L, 3.0)) * (1.0 / (PI * k2)) * exp(-(pow(PI, 2.0) * k2) / pow(kappa, 2.0));
                if (n2 != 0) recipsum2 = recipsum2 + ek2;
            }
    double realsum2 = 0.0;
    for (int l1 = -l4; l1 <= l4; l1++)
        for (int l2 = -l4; l2 <= l4; l2++)
            for (int l3 = -l4; l3 <= l4; l3++) {
                double modr = L * sqrt((double)(l1 * l1 + l2 * l2 + l3 * l3));
                if (modr != 0.0) realsum2 = realsum2 + erfc(kappa * modr) / modr;
            }
    return realsum2 + recipsum2 + term2 + term4;
}

typedef struct {
    int n[3];
    int n2;
    double nt[3];
    double nt2;
} G1Entry;

/* eigenvalue loop shared by SetupBasis (HEG.f90:291-304) and change_rs (514-529) */
static void form_eigen(Heg *h, const Info *in, int nbasis)
{
    for (int l1 = 1; l1 <= nbasis; l1++) {
        double e = 0.0;
        e = 0.5 * (KV(h, l1, 1) * KV(h, l1, 1) + KV(h, l1, 2) * KV(h, l1, 2) + KV(h, l1, 3) * KV(h, l1, 3));
        for (int l2 = 1; l2 <= h->nel / 2; l2++) {
            if (l2 != l1) {
                double q1 = KV(h, l1, 1) - KV(h, l2, 1);
                double q2 = KV(h, l1, 2) - KV(h, l2, 2);
                double q3 = KV(h, l1, 3) - KV(h, l2, 3);
                e = e - (1.0 / h->omega) * (4.0 * PI / (q1 * q1 + q2 * q2 + q3 * q3)) * in->exchangefactor;
            } else {
                e = e + h->madelung - in->gap;
            }
        }
        h->eigen[l1 - 1] = e;
    }
}

/* print_HF (HEG.f90:581-615), energy part only */
static void print_hf(Heg *h)
{
    h->ehf = 0.0;
    h->xhf = 0.0;
    for (int l1 = 1; l1 <= h->nel / 2; l1++) {
        h->ehf = h->ehf + 0.5 * (KV(h, l1, 1) * KV(h, l1, 1) + KV(h, l1, 2) * KV(h, l1, 2) + KV(h, l1, 3) * KV(h, l1, 3));
        for (int l2 = 1; l2 <= h->nel / 2; l2++) {
            if (l2 != l1) {
                double q1 = KV(h, l1, 1) - KV(h, l2, 1);
                double q2 = KV(h, l1, 2) - KV(h, l2, 2);
                double q3 = KV(h, l1, 3) - KV(h, l2, 3);
                double qq = q1 * q1 + q2 * q2 + q3 * q3;
                h->ehf = h->ehf - 0.5 * (1.0 / h->omega) * (4.0 * PI / qq);
                h->xhf = h->xhf - 0.5 * (1.0 / h->omega) * (4.0 * PI / qq);
            }
        }
    }
    h->ehf = h->ehf * 2.0;
    h->xhf = h->xhf * 2.0;
    h->ehf = h->ehf + h->madelung * F12 * h->nel;
}

/* SetupBasis (HEG.f90:150-324) */
static int setup_basis(Heg *h, Info *in)
{
    int cell = h->cell, side = 2 * cell + 1;
    G1Entry *g1 = (G1Entry *)calloc((size_t)side * side * side + 1, sizeof(G1Entry));
    if (!g1) { set_err("allocation failed in setup_basis"); return -1; }
    int M = 0;
    for (int l1 = -cell; l1 <= cell; l1++)
        for (int l2 = -cell; l2 <= cell; l2++)
            for (int l3 = -cell; l3 <= cell; l3++) {
                G1Entry *g = &g1[M];
                M = M + 1;
                g->n[0] = l1; g->n[1] = l2; g->n[2] = l3;
                g->n2 = l1 * l1 + l2 * l2 + l3 * l3;
                g->nt[0] = l1 + h->ntwist[0];
                g->nt[1] = l2 + h->ntwist[1];
                g->nt[2] = l3 + h->ntwist[2];
                g->nt2 = g->nt[0] * g->nt[0] + g->nt[1] * g->nt[1] + g->nt[2] * g->nt[2];
                if (g->n2 > in->maxkpoint) M = M - 1;
            }
    int nbasis = M;
    /* bubble sort, ascending twisted |n+k|^2, stable (HEG.f90:206-217) */
    for (;;) {
        int swapped = 0;
        for (int l1 = 1; l1 < nbasis; l1++) {
            if (g1[l1].nt2 < g1[l1 - 1].nt2) {
                G1Entry t = g1[l1 - 1];
                g1[l1 - 1] = g1[l1];
                g1[l1] = t;
                swapped = 1;
            }
        }
        if (!swapped) break;
    }
    int mfcut = (int)(pow(in->fcut, 3.0 / 2.0) * h->nel / 2);
    double mtarget = pow(in->fcut, 3.0 / 2.0) * h->nel / 2;
    if (fabs(mfcut - mtarget) > fabs(mfcut + 1 - mtarget)) mfcut = mfcut + 1;
    if (mfcut < nbasis) { nbasis = mfcut; M = mfcut; }
    if (abs(fcut_to_basis_fn(in->fcut, h->nel) - mfcut) > 0) {
        free(g1);
        set_err("Error in FcutToBasisFn during setup_basis");
        return -1;
    }
    int mcorefcut = fcut_to_basis_fn(in->corefcut, h->nel);
    if ((in->corefcut - 1.0) < 1e-6) {
        if (mcorefcut != h->nel / 2) {
            free(g1);
            set_err("ERROR in setup_basis: corefcut is less than 1 rather than equal to 1");
            return -1;
        }
    }
    nbasis = nbasis - mcorefcut + h->nel / 2;
    M = nbasis;
    in->nao = M;

    free(h->kvec); free(h->eigen); free(h->nvec); free(h->kp2bf);
    h->kvec = (double *)calloc((size_t)M * 3, sizeof(double));
    h->eigen = (double *)calloc((size_t)M, sizeof(double));
    h->nvec = (int *)calloc((size_t)M * 3, sizeof(int));
    h->kp2bf = (int *)calloc((size_t)side * side * side, sizeof(int));
    if (!h->kvec || !h->eigen || !h->nvec || !h->kp2bf) { free(g1); set_err("allocation failed"); return -1; }

    for (int l1 = 1; l1 <= nbasis; l1++) {
        int offset = 0;
        if (l1 > h->nel / 2) offset = mcorefcut - h->nel / 2;
        const G1Entry *g = &g1[l1 + offset - 1];
        for (int d = 1; d <= 3; d++) {
            KV(h, l1, d) = g->nt[d - 1] * (2.0 * PI / h->L);
            NV(h, l1, d) = g->n[d - 1];
        }
    }
    form_eigen(h, in, nbasis);
    for (int l1 = 1; l1 <= nbasis; l1++) {
        int offset = 0;
        if (l1 > h->nel / 2) offset = mcorefcut - h->nel / 2;
        const G1Entry *g = &g1[l1 + offset - 1];
        int x = g->n[0] + cell, y = g->n[1] + cell, z = g->n[2] + cell;
        /* Fortran column-major kPointToBasisFn(n1,n2,n3) */
        h->kp2bf[x + side * (y + side * z)] = l1;
    }
    print_hf(h);
    free(g1);
    return 0;
}

/* FindIndex (HEG.f90:357-404): orbital at n_M + n_N - n_L, or 0 */
static inline int find_index(const Heg *h, int ecut, int nbasis, int m, int n, int l)
{
    int k1 = NV(h, m, 1) + NV(h, n, 1) - NV(h, l, 1);
    int k2 = NV(h, m, 2) + NV(h, n, 2) - NV(h, l, 2);
    int k3 = NV(h, m, 3) + NV(h, n, 3) - NV(h, l, 3);
    int in = 1;
    if (abs(k1) > h->cell) in = 0;
    if (abs(k2) > h->cell) in = 0;
    if (abs(k3) > h->cell) in = 0;
    int e = k1 * k1 + k2 * k2 + k3 * k3;
    if (e > ecut) in = 0;
    if (!in) return 0;
    int side = 2 * h->cell + 1;
    int k = h->kp2bf[(k1 + h->cell) + side * ((k2 + h->cell) + side * (k3 + h->cell))];
    if (k > nbasis) return 0;
    return k;
}
#define FIND(c, m, n, l) find_index(&(c)->heg, (c)->info.maxkpoint, (c)->info.nao, (m), (n), (l))

/* --------------------------------------------------------- ERI variants */

/* CheckMomentumSymmetry (HEG.f90:438-450) */
static inline int check_momentum(const Heg *h, int i, int j, int a, int b)
{
    for (int d = 1; d <= 3; d++) {
        int g1 = -NV(h, i, d) + NV(h, a, d);
        int g2 = -NV(h, j, d) + NV(h, b, d);
        if (g1 != -g2) return 0;
    }
    return 1;
}

static inline double qvec2_of(const Heg *h, int a, int i, int *zero)
{
    int q1 = -NV(h, i, 1) + NV(h, a, 1);
    int q2 = -NV(h, i, 2) + NV(h, a, 2);
    int q3 = -NV(h, i, 3) + NV(h, a, 3);
    *zero = (q1 == 0 && q2 == 0 && q3 == 0);
    return (double)(q1 * q1 + q2 * q2 + q3 * q3);
}

/* BaseERI (HEG.f90:944-978) */
static double base_eri(const UoCtx *c, int a, int b, int i, int j, int flag)
{
    (void)b; (void)j; (void)flag;
    const Heg *h = &c->heg;
    int zero;
    double q2 = qvec2_of(h, a, i, &zero);
    if (zero) return -h->madelung;
    return 1.0 / (h->L * PI * q2);
}

/* CasedERI (HEG.f90:689-774) */
static double cased_eri(const UoCtx *c, int a, int b, int i, int j, int flag)
{
    const Heg *h = &c->heg;
    const Info *in = &c->info;
    double intgrl = 0.0;
    int mn = a; if (b < mn) mn = b; if (i < mn) mn = i; if (j < mn) mn = j;
    if (mn <= 0) return -100.0;
    if (!check_momentum(h, i, j, a, b)) return -100.0;
    int zero;
    double qvec2 = qvec2_of(h, a, i, &zero);
    if (zero) {
        switch (flag) {
        case 0: intgrl = -h->madelung; break;
        case 1: intgrl = (1.0 / pow(h->L, 3.0)) * 4.0 * PI / pow(h->screening, 2.0); break;
        case 2: intgrl = -h->madelung - (1.0 / pow(h->L, 3.0)) * 4.0 * PI / pow(h->screening, 2.0); break;
        case 3: intgrl = 0.0; break;
        default: return -100.0;
        }
    } else {
        double q2s = qvec2 * pow(2.0 * PI / h->L, 2.0);
        switch (flag) {
        case 0: intgrl = 1.0 / (h->L * PI * qvec2); break;
        case 1: intgrl = (1.0 / pow(h->L, 3.0)) * 4.0 * PI / (pow(h->screening, 2.0) + q2s); break;
        case 2:
            intgrl = (1.0 / pow(h->L, 3.0)) * 4.0 * PI / (pow(h->screening, 2.0) + q2s) * pow(h->screening, 2.0) / q2s;
            break;
        case 3: intgrl = 0.0; break;
        default: break; /* intgrl keeps its (undefined in Fortran) value; 0 here */
        }
    }
    if (a <= in->coren || b <= in->coren || i <= in->coren || j <= in->coren) intgrl = 0.0;
    if (intgrl < 0.0) return -100.0;
    if (intgrl > in->gapii && in->gapii > 0.0) intgrl = 0.0;
    return intgrl;
}

/* NoCaseERI (HEG.f90:776-833) */
static double nocase_eri(const UoCtx *c, int a, int b, int i, int j, int flag)
{
    (void)flag;
    const Heg *h = &c->heg;
    const Info *in = &c->info;
    int mn = a; if (b < mn) mn = b; if (i < mn) mn = i; if (j < mn) mn = j;
    if (mn <= 0) return -100.0;
    if (!check_momentum(h, i, j, a, b)) return -100.0;
    int zero;
    double q2 = qvec2_of(h, a, i, &zero);
    double intgrl = zero ? -h->madelung : 1.0 / (h->L * PI * q2);
    if (a <= in->coren || b <= in->coren || i <= in->coren || j <= in->coren) intgrl = 0.0;
    if (intgrl < 0.0) return -100.0;
    if (intgrl > in->gapii && in->gapii > 0.0) intgrl = 0.0;
    return intgrl;
}

/* CoreERI (HEG.f90:835-888) */
static double core_eri(const UoCtx *c, int a, int b, int i, int j, int flag)
{
    (void)flag;
    const Heg *h = &c->heg;
    const Info *in = &c->info;
    int mn = a; if (b < mn) mn = b; if (i < mn) mn = i; if (j < mn) mn = j;
    if (mn <= 0) return -100.0;
    if (!check_momentum(h, i, j, a, b)) return -100.0;
    int zero;
    double q2 = qvec2_of(h, a, i, &zero);
    double intgrl = zero ? -h->madelung : 1.0 / (h->L * PI * q2);
    if (intgrl < 0.0) return -100.0;
    if (a <= in->coren || b <= in->coren || i <= in->coren || j <= in->coren) intgrl = 0.0;
    return intgrl;
}

/* GapERI (HEG.f90:890-942) */
static double gap_eri(const UoCtx *c, int a, int b, int i, int j, int flag)
{
    (void)flag;
    const Heg *h = &c->heg;
    const Info *in = &c->info;
    int mn = a; if (b < mn) mn = b; if (i < mn) mn = i; if (j < mn) mn = j;
    if (mn <= 0) return -100.0;
    if (!check_momentum(h, i, j, a, b)) return -100.0;
    int zero;
    double q2 = qvec2_of(h, a, i, &zero);
    double intgrl = zero ? -h->madelung : 1.0 / (h->L * PI * q2);
    if (intgrl < 0.0) return -100.0;
    if (intgrl > in->gapii && in->gapii > 0.0) intgrl = 0.0;
    return intgrl;
}

/* SetPointers (Main.f90:274-318) */
static void set_pointers(UoCtx *c)
{
    const Info *u = &c->info;
    int s = abs(u->irange_ring) + abs(u->irange_xring) + abs(u->irange_ladder) + abs(u->irange_mosaic) +
            abs(u->irange_driver_direct) + abs(u->irange_driver_exchange) + abs(u->irange_energy) +
            abs(u->irange_lin_rings) + abs(u->irange_quad_rings) + abs(u->irange_direct_rings) +
            abs(u->irange_exchange_rings) + abs(u->irange_lin_ladders) + abs(u->irange_quad_ladders) +
            abs(u->irange_direct_ladders) + abs(u->irange_exchange_ladders);
    if ((s > 0 && u->gapii > 0.0 && u->coren > 0) || u->safe_eri) c->eri = cased_eri;
    else if (u->gapii > 0.0 && u->coren > 0) c->eri = nocase_eri;
    else if (u->coren > 0) c->eri = core_eri;
    else if (u->gapii > 0.0) c->eri = gap_eri;
    else c->eri = base_eri;
}
#define ERI(c, a, b, i, j, f) ((c)->eri((c), (a), (b), (i), (j), (f)))

static inline int imax3(int a, int b, int c) { int m = a > b ? a : b; return m > c ? m : c; }

/* FindTol (HEG.f90:1073-1086) */
static void find_tol(double rs, double *tolmax, double *failratio, double *denomfactor)
{
    *tolmax = 1.0e-8;
    *failratio = 100;
    if (rs > 5.1) *tolmax = 1.0e-6;
    if (rs > 5.1) *denomfactor = 5.0;
    if (rs > 9.9) *tolmax = 1.0e-5;
    if (rs > 80.0) *tolmax = 1.0e-3;
    if (rs < 0.95) *failratio = 1e6;
}

/* ------------------------------------------------------------ public set-up */

UoCtx *uo_create(const UoInput *p)
{
    UoCtx *c = (UoCtx *)calloc(1, sizeof(UoCtx));
    if (!c) return NULL;
    Info *u = &c->info;
    /* ReadInput (IO.f90:148-305) derived values */
    if (p->nelectron < 0) { set_err("Must have positive number of electrons"); free(c); return NULL; }
    if (p->nelectron % 2 == 1) { set_err("Must have closed shell"); free(c); return NULL; }
    if (p->num_rs_points > 1) { set_err("Cannot have more than one rs point"); free(c); return NULL; }
    u->nelectron = p->nelectron;
    u->nocc = p->nelectron / 2;
    u->maxkpoint = p->maxkpoint;
    u->safe_eri = p->safe_eri;
    u->do_ring = p->do_ring; u->do_xring = p->do_xring; u->do_ladder = p->do_ladder; u->do_mosaic = p->do_mosaic;
    u->irange_ring = p->irange_ring; u->irange_xring = p->irange_xring; u->irange_ladder = p->irange_ladder;
    u->irange_mosaic = p->irange_mosaic; u->irange_driver_direct = p->irange_driver_direct;
    u->irange_driver_exchange = p->irange_driver_exchange; u->irange_energy = p->irange_energy;
    u->irange_lin_rings = p->irange_lin_rings; u->irange_quad_rings = p->irange_quad_rings;
    u->irange_direct_rings = p->irange_direct_rings; u->irange_exchange_rings = p->irange_exchange_rings;
    u->irange_lin_ladders = p->irange_lin_ladders; u->irange_quad_ladders = p->irange_quad_ladders;
    u->irange_direct_ladders = p->irange_direct_ladders; u->irange_exchange_ladders = p->irange_exchange_ladders;
    u->coren = (int)(u->nelectron / 2 * p->core_factor);
    u->exchangefactor = p->do_ks ? 0.0 : 1.0;
    u->madelungfactor = p->madelung_factor;
    u->gap = p->gap;
    u->gapii = p->gapii;
    u->fcut = p->fcut;
    u->corefcut = p->corefcut;
    u->do_drpa_sosex = p->do_drpa_sosex;
    u->do_calc_ta_ccd = p->do_calc_ta_ccd;
    if (p->fcut2ecut) {
        double nfermi = pow((double)u->nelectron, 2.0 / 3.0) / 4.0;
        double mult = u->fcut;
        if (u->fcut < 2.0) mult = 2.0;
        u->maxkpoint = (int)(nfermi * mult * 2.0);
        if (nfermi < 10) u->maxkpoint = (int)(10 * mult * 2.0);
    }
    /* init_HEG (HEG.f90:16-43) */
    Heg *h = &c->heg;
    h->ntwist[0] = p->ntwist[0]; h->ntwist[1] = p->ntwist[1]; h->ntwist[2] = p->ntwist[2];
    h->nel = u->nelectron;
    h->rS = 1.0;
    h->L = h->rS * pow(4.0 / 3.0 * PI * h->nel, 1.0 / 3.0);
    h->omega = h->L * h->L * h->L; /* L**3, integer power */
    h->madelung = calc_madelung(h->omega, h->L) * u->madelungfactor;
    h->cell = (int)sqrt((double)u->maxkpoint) + 3;
    h->density = h->nel / pow(h->L, 3.0);
    h->kf = pow(3.0 * pow(PI, 2.0) * h->density, 1.0 / 3.0);
    h->screening = pow(4.0 / PI * h->kf, 0.5);
    if (setup_basis(h, u) != 0) { uo_destroy(c); return NULL; }
    set_pointers(c);
    /* Main.f90:78-79 -> change_rs (HEG.f90:494-533) */
    u->rs = p->rsmin;
    double rescale = u->rs / h->rS;
    h->L = h->L * rescale;
    h->omega = h->omega * pow(rescale, 3.0);
    for (int k = 0; k < u->nao * 3; k++) h->kvec[k] = h->kvec[k] * (1.0 / rescale);
    h->madelung = calc_madelung(h->omega, h->L) * u->madelungfactor;
    h->density = h->nel / pow(h->L, 3.0);
    h->kf = pow(3.0 * pow(PI, 2.0) * h->density, 1.0 / 3.0);
    h->screening = pow(4.0 / PI * h->kf, 0.5);
    form_eigen(h, u, u->nao);
    print_hf(h);
    c->denom_factor_ccd = 2.0;
    c->denom_factor_drpa = 2.0;
    return c;
}

void uo_destroy(UoCtx *c)
{
    if (!c) return;
    free(c->heg.kvec); free(c->heg.eigen); free(c->heg.nvec); free(c->heg.kp2bf);
    free(c);
}

int uo_nocc(const UoCtx *c) { return c->info.nocc; }
int uo_nao(const UoCtx *c) { return c->info.nao; }
int uo_cell(const UoCtx *c) { return c->heg.cell; }
int uo_maxkpoint(const UoCtx *c) { return c->info.maxkpoint; }
void uo_scalars(const UoCtx *c, double out[7])
{
    out[0] = c->heg.L; out[1] = c->heg.omega; out[2] = c->heg.madelung; out[3] = c->heg.ehf;
    out[4] = c->heg.ntwist[0]; out[5] = c->heg.ntwist[1]; out[6] = c->heg.ntwist[2];
}
void uo_get_eigen(const UoCtx *c, double *e) { memcpy(e, c->heg.eigen, sizeof(double) * c->info.nao); }
void uo_set_eigen(UoCtx *c, const double *e) { memcpy(c->heg.eigen, e, sizeof(double) * c->info.nao); }
void uo_get_nvec(const UoCtx *c, int *n) { memcpy(n, c->heg.nvec, sizeof(int) * 3 * c->info.nao); }
void uo_get_kvec(const UoCtx *c, double *k) { memcpy(k, c->heg.kvec, sizeof(double) * 3 * c->info.nao); }

/* ChangeTwist (HEG.f90:551-578) */
int uo_change_twist(UoCtx *c, const double tw[3])
{
    for (int d = 0; d < 3; d++) { c->heg.this_ntwist[d] = tw[d]; c->heg.ntwist[d] = tw[d]; }
    int nao_before = c->info.nao;
    if (setup_basis(&c->heg, &c->info) != 0) return -1;
    if (c->info.nao != nao_before) { set_err("basis size changed with the twist"); return -1; }
    return 0;
}

/* ------------------------------------------------------------------ MP2.f90 */

/* dK2 (HEG.f90:985-1005) with the argument order of its MP2 call sites */
static inline int dk2(const Heg *h, int a, int i)
{
    int q1 = -NV(h, i, 1) + NV(h, a, 1), q2 = -NV(h, i, 2) + NV(h, a, 2), q3 = -NV(h, i, 3) + NV(h, a, 3);
    return q1 * q1 + q2 * q2 + q3 * q3;
}

/* DrvMBPT (MP2.f90:11-157) */
double uo_mp2(UoCtx *c, double *t_aaaa, double *t_abab, double *t_abba, int *conn)
{
    const Info *u = &c->info;
    const Heg *h = &c->heg;
    int O = u->nocc, M = u->nao;
    size_t n = (size_t)O * O * (M - O);
    memset(t_abab, 0, n * sizeof(double));
    memset(t_abba, 0, n * sizeof(double));
    memset(t_aaaa, 0, n * sizeof(double));
    double ecorr = 0.0;
    int connectivity[400];
    memset(connectivity, 0, sizeof connectivity);
    for (int i = 1; i <= O; i++)
        for (int j = 1; j <= O; j++)
            for (int a = O + 1; a <= M; a++) {
                int b = FIND(c, i, j, a);
                if (b <= O) continue;
                double v_ijab = ERI(c, i, j, a, b, 0);
                double v_ijba = ERI(c, i, j, b, a, 0);
                if (fmin(v_ijab, v_ijba) < -80.0) continue;
                double denom = h->eigen[i - 1] + h->eigen[j - 1] - h->eigen[a - 1] - h->eigen[b - 1];
                int x = tix(O, i, j, a);
                t_abab[x] = v_ijab / denom;
                t_abba[x] = -v_ijba / denom;
                t_aaaa[x] = t_abab[x] + t_abba[x];
                ecorr = ecorr + F12 * t_aaaa[x] * (v_ijab - v_ijba) + F12 * t_abab[x] * (v_ijab) -
                        F12 * t_abba[x] * (v_ijba);
                /* connectivity (MP2.f90:75-85); InCore is set by the second call */
                int d_ijab = dk2(h, i, a), d_ijba = dk2(h, i, b);
                int incore = (i <= u->coren) || (j <= u->coren) || (b <= u->coren) || (a <= u->coren);
                if (d_ijab > 400 || d_ijba > 400) { set_err("Connectivity greater than current ConnectivityLimit"); continue; }
                if (!incore) {
                    connectivity[d_ijba - 1] += 1;
                    connectivity[d_ijab - 1] += 1;
                }
            }
    if (conn) memcpy(conn, connectivity, sizeof connectivity);
    c->heg.ecorr = ecorr;
    return ecorr;
}

/* ------------------------------------------------------------------ CCD.f90 */

/* CCEnergy (CCD.f90:186-237) */
double uo_ccd_energy(UoCtx *c, const double *t_aaaa, const double *t_abab, const double *t_abba)
{
    const Info *u = &c->info;
    int O = u->nocc, M = u->nao;
    double ecorr = 0.0;
    for (int i = 1; i <= O; i++)
        for (int j = 1; j <= O; j++)
            for (int a = O + 1; a <= M; a++) {
                int b = FIND(c, i, j, a);
                if (b <= O) continue;
                double v_ijab = ERI(c, a, b, i, j, u->irange_energy);
                double v_ijba = ERI(c, a, b, j, i, u->irange_energy);
                if (fmin(v_ijab, v_ijba) < -80.0) continue;
                int x = tix(O, i, j, a);
                double de = v_ijab * (t_aaaa[x] + t_abab[x]) - v_ijba * (t_aaaa[x] + t_abba[x]);
                ecorr = ecorr + F12 * de;
            }
    c->heg.ecorr = ecorr;
    return ecorr;
}

/* --------------------------------------------------- structure factors */

/* SendForAllocation (HEG.f90:1051-1065): SfLength = maxval(nvec)*2+1 */
int uo_sf_length(const UoCtx *c)
{
    const Heg *h = &c->heg;
    int m = h->nvec[0];
    for (int k = 0; k < 3 * c->info.nao; k++)
        if (h->nvec[k] > m) m = h->nvec[k];
    return m * 2 + 1;
}

/* The structure-factor loop of CCEnergyAndSF (CCD.f90:240-351), whose SfSum/SfG/SfV
 * part is also the loop of DrvMBPT (MP2.f90:86-95).  Grids (2S+1)^3, S = uo_sf_length,
 * column-major from -S; every pointer may be NULL.  Contributions are added in the
 * reference's loop order (I, J, A, A innermost; direct before exchange).  Returns
 * the ECorr the routine computes.  Out-of-grid transfers (the reference writes
 * outside its arrays there) are skipped and counted in *oob. */
double uo_structure_factor(UoCtx *c, const double *t_aaaa, const double *t_abab, const double *t_abba,
                           double *sf_sum, double *sf_g, double *sf_v, double *sf_dsum, double *sf_xsum, int *oob)
{
    const Info *u = &c->info;
    const Heg *h = &c->heg;
    const int O = u->nocc, M = u->nao, S = uo_sf_length(c), W = 2 * S + 1;
    const size_t W3 = (size_t)W * W * W;
    double *grids[5] = {sf_sum, sf_g, sf_v, sf_dsum, sf_xsum};
    for (int k = 0; k < 5; k++)
        if (grids[k]) memset(grids[k], 0, W3 * sizeof(double));
    int bad = 0;
    double ecorr = 0.0;
    const double scale = pow(2.0 * PI / h->L, 2.0);
    for (int i = 1; i <= O; i++)
        for (int j = 1; j <= O; j++)
            for (int a = O + 1; a <= M; a++) {
                int b = FIND(c, i, j, a);
                if (b <= O) continue;
                double v_ijab = ERI(c, a, b, i, j, u->irange_energy);
                double v_ijba = ERI(c, a, b, j, i, u->irange_energy);
                if (fmin(v_ijab, v_ijba) < -80.0) continue;
                int x = tix(O, i, j, a);
                double de = v_ijab * (t_aaaa[x] + t_abab[x]) - v_ijba * (t_aaaa[x] + t_abba[x]);
                ecorr = ecorr + F12 * de;
                for (int pass = 0; pass < 2; pass++) {
                    /* dK(a,b,i,j) = -nvec(i)+nvec(a), then dK(a,b,j,i) */
                    const int o = pass == 0 ? i : j;
                    int q[3];
                    for (int d = 1; d <= 3; d++) q[d - 1] = -NV(h, o, d) + NV(h, a, d);
                    if (abs(q[0]) > S || abs(q[1]) > S || abs(q[2]) > S) { bad++; continue; }
                    size_t g = (size_t)(q[0] + S) + (size_t)W * ((size_t)(q[1] + S) + (size_t)W * (size_t)(q[2] + S));
                    double q2 = (double)(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
                    if (pass == 0) {
                        if (sf_sum) sf_sum[g] = sf_sum[g] + (t_aaaa[x] + t_abab[x]);
                        if (sf_g) sf_g[g] = pow(q2 * scale, 0.5);
                        if (sf_v) sf_v[g] = v_ijab;
                        if (sf_dsum) sf_dsum[g] = sf_dsum[g] + (2.0 * t_abab[x]);
                        if (sf_xsum) sf_xsum[g] = sf_xsum[g] + (t_aaaa[x] - t_abab[x]);
                    } else {
                        if (sf_sum) sf_sum[g] = sf_sum[g] - (t_aaaa[x] + t_abba[x]);
                        if (sf_g) sf_g[g] = pow(q2 * scale, 0.5);
                        if (sf_v) sf_v[g] = v_ijba;
                        if (sf_dsum) sf_dsum[g] = sf_dsum[g] - (2.0 * t_abba[x]);
                        if (sf_xsum) sf_xsum[g] = sf_xsum[g] - (t_aaaa[x] - t_abba[x]);
                    }
                }
            }
    if (oob) *oob = bad;
    return ecorr;
}

/* print_ex_SF (HEG.f90:617-674): the exchange structure factor of the occupied
 * orbitals.  Returns maxq; with ex_sf/ex_v non-NULL fills the (2*maxq+1)^3 grids
 * (column-major from -maxq). */
int uo_exchange_sf(const UoCtx *c, int *ex_sf, double *ex_v)
{
    const Heg *h = &c->heg;
    const int no = h->nel / 2;
    int qmax[3] = {0, 0, 0};
    for (int l1 = 1; l1 <= no; l1++)
        for (int l2 = 1; l2 <= no; l2++)
            if (l2 != l1)
                for (int d = 1; d <= 3; d++) {
                    int q = abs(NV(h, l1, d) - NV(h, l2, d));
                    if (q > qmax[d - 1]) qmax[d - 1] = q;
                }
    const int maxq = imax3(qmax[0], qmax[1], qmax[2]) + 1, W = 2 * maxq + 1;
    if (!ex_sf && !ex_v) return maxq;
    const size_t W3 = (size_t)W * W * W;
    if (ex_sf) memset(ex_sf, 0, W3 * sizeof(int));
    if (ex_v) memset(ex_v, 0, W3 * sizeof(double));
    for (int l1 = 1; l1 <= no; l1++)
        for (int l2 = 1; l2 <= no; l2++) {
            if (l2 == l1) continue;
            int q[3];
            for (int d = 1; d <= 3; d++) q[d - 1] = NV(h, l1, d) - NV(h, l2, d);
            size_t g = (size_t)(q[0] + maxq) + (size_t)W * ((size_t)(q[1] + maxq) + (size_t)W * (size_t)(q[2] + maxq));
            if (ex_sf) ex_sf[g] += 1;
            double k1 = KV(h, l1, 1) - KV(h, l2, 1), k2 = KV(h, l1, 2) - KV(h, l2, 2), k3 = KV(h, l1, 3) - KV(h, l2, 3);
            if (ex_v) ex_v[g] = (1.0 / h->omega) * (4.0 * PI / (k1 * k1 + k2 * k2 + k3 * k3));
        }
    return maxq;
}

/* SolveCC (CCD.f90:354-386; dRPA.f90:223-255) */
static void solve_cc(UoCtx *c, double *t2, const double *g2, double df)
{
    const Info *u = &c->info;
    const double *e = c->heg.eigen;
    int O = u->nocc, M = u->nao;
    for (int i = 1; i <= O; i++)
        for (int j = 1; j <= O; j++)
            for (int a = O + 1; a <= M; a++) {
                int b = FIND(c, i, j, a);
                if (b <= O) continue;
                double denom = e[i - 1] + e[j - 1] - e[a - 1] - e[b - 1];
                int x = tix(O, i, j, a);
                t2[x] = (g2[x] / denom - (1.0 - df) * t2[x]) / df;
            }
}

/* GetRes (CCD.f90:389-424; dRPA.f90:262-297): writes R2(:,:,:,NDIIS) */
static void get_res(UoCtx *c, const double *t2, const double *g2, double *r2_last)
{
    const Info *u = &c->info;
    const double *e = c->heg.eigen;
    int O = u->nocc, M = u->nao;
    for (int i = 1; i <= O; i++)
        for (int j = 1; j <= O; j++)
            for (int a = O + 1; a <= M; a++) {
                int b = FIND(c, i, j, a);
                if (b <= O) continue;
                double denom = e[i - 1] + e[j - 1] - e[a - 1] - e[b - 1];
                int x = tix(O, i, j, a);
                r2_last[x] = -g2[x] + denom * t2[x];
            }
}

/* GetG2Drivers (CCD.f90:465-504) */
static void g2_drivers(UoCtx *c, double *g_abab, double *g_abba)
{
    const Info *u = &c->info;
    int O = u->nocc, M = u->nao;
    size_t n = (size_t)O * O * (M - O);
    memset(g_abab, 0, n * sizeof(double));
    memset(g_abba, 0, n * sizeof(double));
    for (int i = 1; i <= O; i++)
        for (int j = 1; j <= O; j++)
            for (int a = O + 1; a <= M; a++) {
                int b = FIND(c, i, j, a);
                if (b <= O) continue;
                double v_ijab = ERI(c, i, j, a, b, u->irange_driver_direct);
                double v_ijba = ERI(c, i, j, b, a, u->irange_driver_exchange);
                if (fmin(v_ijab, v_ijba) < -80.0) continue;
                int x = tix(O, i, j, a);
                g_abab[x] = v_ijab;
                g_abba[x] = -v_ijba;
            }
}

/* GetG2Mosaics (CCD.f90:507-585) */
static void g2_mosaics(UoCtx *c, double *g_abab, double *g_abba, const double *t_aaaa, const double *t_abab,
                       const double *t_abba)
{
    const Info *u = &c->info;
    int O = u->nocc, M = u->nao;
    double *joo = (double *)calloc((size_t)O, sizeof(double));
    double *jvv = (double *)calloc((size_t)(M - O), sizeof(double)); /* Jvv(c) -> jvv[c-O-1] */
    for (int k = 1; k <= O; k++)
        for (int l = 1; l <= O; l++)
            for (int cc = O + 1; cc <= M; cc++) {
                int d = FIND(c, k, l, cc);
                if (d <= O) continue;
                double v_cdkl = ERI(c, cc, d, k, l, u->irange_mosaic);
                double v_cdlk = ERI(c, cc, d, l, k, u->irange_mosaic);
                if (fmin(v_cdkl, v_cdlk) < -80.0) continue;
                int x = tix(O, k, l, cc);
                jvv[cc - O - 1] = jvv[cc - O - 1] + v_cdkl * (t_aaaa[x] + t_abab[x]) - v_cdlk * (t_aaaa[x] + t_abba[x]);
                joo[k - 1] = joo[k - 1] + v_cdkl * (t_aaaa[x] + t_abab[x]) - v_cdlk * (t_aaaa[x] + t_abba[x]);
            }
    for (int i = 1; i <= O; i++)
        for (int j = 1; j <= O; j++)
            for (int a = O + 1; a <= M; a++) {
                int b = FIND(c, i, j, a);
                if (b <= O) continue;
                int x = tix(O, i, j, a);
                double ja = jvv[a - O - 1], jb = jvv[b - O - 1];
                g_abab[x] = g_abab[x] - F12 * (ja * t_abab[x] + jb * t_abab[x]);
                g_abba[x] = g_abba[x] - F12 * (ja * t_abba[x] + jb * t_abba[x]);
                g_abab[x] = g_abab[x] - F12 * (joo[i - 1] * t_abab[x] + joo[j - 1] * t_abab[x]);
                g_abba[x] = g_abba[x] - F12 * (joo[i - 1] * t_abba[x] + joo[j - 1] * t_abba[x]);
            }
    free(joo);
    free(jvv);
}

/* GetG2Ladders (CCD.f90:588-686) */
static void g2_ladders(UoCtx *c, double *g_abab, double *g_abba, const double *t_abab, const double *t_abba)
{
    const Info *u = &c->info;
    int O = u->nocc, M = u->nao;
    for (int i = 1; i <= O; i++)
        for (int j = 1; j <= O; j++) {
            /* hole-hole ladder */
            for (int k = 1; k <= O; k++) {
                int l = FIND(c, i, j, k);
                if (l > O || l <= 0) continue;
                int f = imax3(u->irange_ladder, u->irange_direct_ladders, u->irange_lin_ladders);
                double j2 = ERI(c, i, j, k, l, f);
                f = imax3(u->irange_ladder, u->irange_exchange_ladders, u->irange_lin_ladders);
                double j3 = -ERI(c, i, j, l, k, f);
                if (fmin(j2, -j3) < -80.0) continue;
                for (int cc = O + 1; cc <= M; cc++) {
                    int d = FIND(c, i, j, cc);
                    if (d <= O) continue;
                    f = imax3(u->irange_ladder, u->irange_direct_ladders, u->irange_quad_ladders);
                    double v_cdkl = ERI(c, cc, d, k, l, f);
                    f = imax3(u->irange_ladder, u->irange_exchange_ladders, u->irange_quad_ladders);
                    double v_cdlk = ERI(c, cc, d, l, k, f);
                    if (fmin(v_cdkl, v_cdlk) < -80.0) continue;
                    int x = tix(O, i, j, cc);
                    j2 = j2 + F12 * (v_cdkl * t_abab[x] - v_cdlk * t_abba[x]);
                    j3 = j3 + F12 * (v_cdkl * t_abba[x] - v_cdlk * t_abab[x]);
                }
                for (int a = O + 1; a <= M; a++) {
                    int b = FIND(c, i, j, a);
                    if (b <= O) continue;
                    int x = tix(O, i, j, a), y = tix(O, k, l, a);
                    g_abab[x] = g_abab[x] + F12 * (j2 * t_abab[y] + j3 * t_abba[y]);
                    g_abba[x] = g_abba[x] + F12 * (j2 * t_abba[y] + j3 * t_abab[y]);
                }
            }
            /* particle-particle ladder */
            for (int a = O + 1; a <= M; a++) {
                int b = FIND(c, i, j, a);
                if (b <= O) continue;
                int x = tix(O, i, j, a);
                for (int cc = O + 1; cc <= M; cc++) {
                    int d = FIND(c, i, j, cc);
                    if (d <= O) continue;
                    int f = imax3(u->irange_ladder, u->irange_direct_ladders, u->irange_lin_ladders);
                    double v_cdab = ERI(c, cc, d, a, b, f);
                    f = imax3(u->irange_ladder, u->irange_exchange_ladders, u->irange_lin_ladders);
                    double v_cdba = ERI(c, cc, d, b, a, f);
                    if (fmin(v_cdab, v_cdba) < -80.0) continue;
                    int y = tix(O, i, j, cc);
                    g_abab[x] = g_abab[x] + F12 * (v_cdab * t_abab[y] - v_cdba * t_abba[y]);
                    g_abba[x] = g_abba[x] + F12 * (v_cdab * t_abba[y] - v_cdba * t_abab[y]);
                }
            }
        }
}

/* GetG2Rings (CCD.f90:689-814) */
static void g2_rings(UoCtx *c, double *g_abab, double *g_abba, const double *t_aaaa, const double *t_abab,
                     const double *t_abba)
{
    const Info *u = &c->info;
    int O = u->nocc, M = u->nao;
    for (int i = 1; i <= O; i++)
        for (int j = 1; j <= O; j++)
            for (int a = O + 1; a <= M; a++) {
                int b = FIND(c, i, j, a);
                if (b <= O) continue;
                int x = tix(O, i, j, a);
                for (int k = 1; k <= O; k++) {
                    int cc = FIND(c, i, k, a);
                    if (cc <= O) continue;
                    int f = imax3(u->irange_ring, u->irange_direct_rings, u->irange_lin_rings);
                    double v_cjkb = ERI(c, cc, j, k, b, f);
                    f = imax3(u->irange_ring, u->irange_exchange_rings, u->irange_lin_rings);
                    double v_cjbk = ERI(c, cc, j, b, k, f);
                    if (fmin(v_cjkb, v_cjbk) < -80.0) continue;
                    int y = tix(O, i, k, a);
                    g_abab[x] = g_abab[x] + (v_cjkb - v_cjbk) * t_abab[y] + v_cjkb * t_aaaa[y];
                    g_abba[x] = g_abba[x] - v_cjbk * t_abba[y];
                }
                for (int k = 1; k <= O; k++) {
                    int cc = FIND(c, j, k, b);
                    if (cc <= O) continue;
                    int f = imax3(u->irange_ring, u->irange_direct_rings, u->irange_lin_rings);
                    double v_cika = ERI(c, cc, i, k, a, f);
                    f = imax3(u->irange_ring, u->irange_exchange_rings, u->irange_lin_rings);
                    double v_ciak = ERI(c, cc, i, a, k, f);
                    if (fmin(v_cika, v_ciak) < -80.0) continue;
                    int y = tix(O, j, k, b);
                    g_abab[x] = g_abab[x] + (v_cika - v_ciak) * t_abab[y] + v_cika * t_aaaa[y];
                    g_abba[x] = g_abba[x] - v_ciak * t_abba[y];
                }
            }
    for (int i = 1; i <= O; i++)
        for (int a = O + 1; a <= M; a++)
            for (int l = 1; l <= O; l++) {
                double j1 = 0.0, j2 = 0.0, j3 = 0.0;
                for (int k = 1; k <= O; k++) {
                    int cc = FIND(c, i, k, a);
                    if (cc <= O) continue;
                    int d = FIND(c, k, l, cc);
                    if (d <= O) continue;
                    int f = imax3(u->irange_ring, u->irange_direct_rings, u->irange_quad_rings);
                    double v_cdkl = ERI(c, cc, d, k, l, f);
                    f = imax3(u->irange_ring, u->irange_exchange_rings, u->irange_quad_rings);
                    double v_cdlk = ERI(c, cc, d, l, k, f);
                    if (fmin(v_cdkl, v_cdlk) < -80.0) continue;
                    int y = tix(O, i, k, a);
                    j1 = j1 + t_aaaa[y] * (v_cdkl - v_cdlk) + t_abab[y] * v_cdkl;
                    j2 = j2 + t_abab[y] * (v_cdkl - v_cdlk) + t_aaaa[y] * v_cdkl;
                    j3 = j3 - t_abba[y] * v_cdlk;
                }
                for (int j = 1; j <= O; j++) {
                    int b = FIND(c, i, j, a);
                    if (b <= O) continue;
                    int d = FIND(c, j, l, b);
                    if (d <= O) continue;
                    int x = tix(O, i, j, a), y = tix(O, l, j, d);
                    g_abab[x] = g_abab[x] + j2 * t_aaaa[y] + j1 * t_abab[y];
                    g_abba[x] = g_abba[x] + j3 * t_abba[y];
                }
            }
}

/* GetG2XRings (CCD.f90:817-940) */
static void g2_xrings(UoCtx *c, double *g_abab, double *g_abba, const double *t_aaaa, const double *t_abab,
                      const double *t_abba)
{
    const Info *u = &c->info;
    int O = u->nocc, M = u->nao;
    for (int i = 1; i <= O; i++)
        for (int j = 1; j <= O; j++)
            for (int a = O + 1; a <= M; a++) {
                int b = FIND(c, i, j, a);
                if (b <= O) continue;
                int x = tix(O, i, j, a);
                for (int k = 1; k <= O; k++) {
                    int cc = FIND(c, k, i, b);
                    if (cc <= O) continue;
                    int f = imax3(u->irange_xring, u->irange_exchange_rings, u->irange_lin_rings);
                    double v_jcka = ERI(c, j, cc, k, a, f);
                    f = imax3(u->irange_xring, u->irange_direct_rings, u->irange_lin_rings);
                    double v_jcak = ERI(c, j, cc, a, k, f);
                    if (fmin(v_jcka, v_jcak) < -80.0) continue;
                    int y = tix(O, k, i, b);
                    g_abab[x] = g_abab[x] - v_jcka * t_abab[y];
                    g_abba[x] = g_abba[x] + (v_jcak - v_jcka) * t_abba[y] + v_jcak * t_aaaa[y];
                }
                for (int k = 1; k <= O; k++) {
                    int cc = FIND(c, k, j, a);
                    if (cc <= O) continue;
                    int f = imax3(u->irange_xring, u->irange_exchange_rings, u->irange_lin_rings);
                    double v_ickb = ERI(c, i, cc, k, b, f);
                    f = imax3(u->irange_xring, u->irange_direct_rings, u->irange_lin_rings);
                    double v_icbk = ERI(c, i, cc, b, k, f);
                    if (fmin(v_ickb, v_icbk) < -80.0) continue;
                    int y = tix(O, k, j, a);
                    g_abab[x] = g_abab[x] - v_ickb * t_abab[y];
                    g_abba[x] = g_abba[x] + (v_icbk - v_ickb) * t_abba[y] + v_icbk * t_aaaa[y];
                }
            }
    for (int i = 1; i <= O; i++)
        for (int b = O + 1; b <= M; b++)
            for (int l = 1; l <= O; l++) {
                double j1 = 0.0, j2 = 0.0, j3 = 0.0;
                for (int k = 1; k <= O; k++) {
                    int cc = FIND(c, i, k, b);
                    if (cc <= O) continue;
                    int d = FIND(c, k, l, cc);
                    if (d <= O) continue;
                    int f = imax3(u->irange_xring, u->irange_direct_rings, u->irange_quad_rings);
                    double v_cdkl = ERI(c, cc, d, k, l, f);
                    f = imax3(u->irange_xring, u->irange_exchange_rings, u->irange_quad_rings);
                    double v_cdlk = ERI(c, cc, d, l, k, f);
                    if (fmin(v_cdkl, v_cdlk) < -80.0) continue;
                    int y = tix(O, k, i, b);
                    j1 = j1 + t_aaaa[y] * (v_cdkl - v_cdlk) + t_abba[y] * v_cdkl;
                    j2 = j2 + t_abba[y] * (v_cdkl - v_cdlk) + t_aaaa[y] * v_cdkl;
                    j3 = j3 + t_abab[y] * v_cdlk;
                }
                for (int j = 1; j <= O; j++) {
                    int a = FIND(c, j, i, b);
                    if (a <= O) continue;
                    int d = FIND(c, l, j, a);
                    if (d <= O) continue;
                    int x = tix(O, i, j, a), y = tix(O, l, j, a);
                    g_abba[x] = g_abba[x] - j1 * t_abba[y] - j2 * t_aaaa[y];
                    g_abab[x] = g_abab[x] + j3 * t_abab[y];
                }
            }
}

void uo_ccd_g2(UoCtx *c, const double *t_abab, const double *t_abba, int mask, double *g_abab, double *g_abba)
{
    int O = c->info.nocc, M = c->info.nao;
    size_t n = (size_t)O * O * (M - O);
    double *t_aaaa = (double *)malloc(n * sizeof(double));
    for (size_t x = 0; x < n; x++) t_aaaa[x] = t_abab[x] + t_abba[x];
    if (mask & 1) g2_drivers(c, g_abab, g_abba);
    else { memset(g_abab, 0, n * sizeof(double)); memset(g_abba, 0, n * sizeof(double)); }
    if (mask & 2) g2_mosaics(c, g_abab, g_abba, t_aaaa, t_abab, t_abba);
    if (mask & 4) g2_ladders(c, g_abab, g_abba, t_abab, t_abba);
    if (mask & 8) g2_rings(c, g_abab, g_abba, t_aaaa, t_abab, t_abba);
    if (mask & 16) g2_xrings(c, g_abab, g_abba, t_aaaa, t_abab, t_abba);
    free(t_aaaa);
}

/* -------------------------------------------------------------- DIISCC.f90 */

/* DGESV restated: LU with partial pivoting; returns INFO (0 ok, k>0 if U(k,k)==0). */
static int small_gesv(int n, double *m /* column-major n x n */, double *v)
{
    int info = 0;
    int piv[64];
    for (int k = 0; k < n; k++) {
        int p = k;
        double best = fabs(m[k + n * k]);
        for (int r = k + 1; r < n; r++)
            if (fabs(m[r + n * k]) > best) { best = fabs(m[r + n * k]); p = r; }
        piv[k] = p;
        if (m[p + n * k] != 0.0) {
            if (p != k)
                for (int cidx = 0; cidx < n; cidx++) {
                    double t = m[k + n * cidx]; m[k + n * cidx] = m[p + n * cidx]; m[p + n * cidx] = t;
                }
            for (int r = k + 1; r < n; r++) m[r + n * k] /= m[k + n * k];
        } else if (info == 0) {
            info = k + 1;
        }
        for (int cidx = k + 1; cidx < n; cidx++)
            for (int r = k + 1; r < n; r++) m[r + n * cidx] -= m[r + n * k] * m[k + n * cidx];
    }
    if (info != 0) return info;
    for (int k = 0; k < n; k++) { int p = piv[k]; if (p != k) { double t = v[k]; v[k] = v[p]; v[p] = t; } }
    for (int k = 0; k < n; k++) for (int r = k + 1; r < n; r++) v[r] -= m[r + n * k] * v[k];
    for (int k = n - 1; k >= 0; k--) { v[k] /= m[k + n * k]; for (int r = 0; r < k; r++) v[r] -= m[r + n * k] * v[k]; }
    return 0;
}

typedef struct {
    int ndiis;
    double *old_abab, *r_abab, *old_abba, *r_abba; /* (O,O,V,NDIIS) */
} Diis;

/* SetUpDIISCC (DIISCC.f90:10-45); NDIIS = 3 (allocation never fails here) */
static int diis_setup(Diis *d, size_t n, const double *t_abab, const double *t_abba)
{
    d->ndiis = 3;
    d->old_abab = (double *)calloc(n * 3, sizeof(double));
    d->r_abab = (double *)calloc(n * 3, sizeof(double));
    d->old_abba = (double *)calloc(n * 3, sizeof(double));
    d->r_abba = (double *)calloc(n * 3, sizeof(double));
    if (!d->old_abab || !d->r_abab || !d->old_abba || !d->r_abba) { set_err("Could not allocate for DIIS"); return -1; }
    memcpy(d->old_abab + n * 2, t_abab, n * sizeof(double));
    memcpy(d->old_abba + n * 2, t_abba, n * sizeof(double));
    return 0;
}
static void diis_free(Diis *d) { free(d->old_abab); free(d->r_abab); free(d->old_abba); free(d->r_abba); }

/* GetTFromDIIS (DIISCC.f90:52-131) */
static void get_t_from_diis(double *t2, const double *old, double *r2, size_t n, int ndiis, int niter)
{
    double cvec[16];
    for (int p = 0; p < ndiis; p++) cvec[p] = 0.0;
    cvec[ndiis - 1] = 1.0;
    if (niter >= ndiis + 5) {
        int nn = ndiis + 1;
        double m[17 * 17], v[17];
        for (int x = 0; x < nn * nn; x++) m[x] = 0.0;
        for (int x = 0; x < nn; x++) v[x] = 0.0;
        for (int p = 0; p < ndiis; p++)
            for (int q = 0; q < ndiis; q++) {
                double s = m[p + nn * q];
                const double *rp = r2 + n * p, *rq = r2 + n * q;
                for (size_t x = 0; x < n; x++) s = s + rp[x] * rq[x];
                m[p + nn * q] = s;
            }
        /* M(1:NDIIS,1:) = One ; M(1,1::NDIIS) = One ; V(NDIIS+1) = One */
        for (int p = 0; p < ndiis; p++)
            for (int q = 0; q < nn; q++) m[p + nn * q] = 1.0;
        for (int q = 0; q < nn; q += ndiis) m[0 + nn * q] = 1.0;
        v[ndiis] = 1.0;
        int info = small_gesv(nn, m, v);
        if (info == 0)
            for (int p = 0; p < ndiis; p++) cvec[p] = v[p];
        for (size_t x = 0; x < n; x++) t2[x] = 0.0;
        for (int p = 0; p < ndiis; p++) {
            const double *op = old + n * p;
            for (size_t x = 0; x < n; x++) t2[x] = t2[x] + cvec[p] * op[x];
        }
    } else {
        memcpy(t2, old + n * (ndiis - 1), n * sizeof(double));
    }
    memmove(r2, r2 + n, n * (ndiis - 1) * sizeof(double));
}

static double maxabs(const double *x, size_t n)
{
    double m = 0.0;
    for (size_t k = 0; k < n; k++) if (fabs(x[k]) > m) m = fabs(x[k]);
    return m;
}

/* CnvrgCC (CCD.f90:427-462) for one channel; returns MaxVal(Abs(T - Old(NDIIS))) */
static double cnvrg_channel(const double *t2, double *old, size_t n, int ndiis)
{
    memmove(old, old + n, n * (ndiis - 1) * sizeof(double));
    double *last = old + n * (ndiis - 1);
    double m = 0.0;
    for (size_t x = 0; x < n; x++) { double d = fabs(t2[x] - last[x]); if (d > m) m = d; }
    memcpy(last, t2, n * sizeof(double));
    return m;
}

/* DrvCCD (CCD.f90:18-183) */
static double g_tol_override = 0.0;
/* Test hook: a TolMax below the reference's (tight-mode parity); <= 0 restores FindTol. */
void uo_set_tol_override(double tol) { g_tol_override = tol; }

int uo_ccd(UoCtx *c, double *t_aaaa, double *t_abab, double *t_abba, int max_iter_override, UoSolveStats *st,
           double *energies, double *dts, int max_rec)
{
    const Info *u = &c->info;
    int O = u->nocc, M = u->nao;
    size_t n = (size_t)O * O * (M - O);
    double tolmax = 1.0e-8, failratio = 100;
    find_tol(c->heg.rS, &tolmax, &failratio, &c->denom_factor_ccd);
    if (g_tol_override > 0.0) tolmax = g_tol_override;
    const int max_iter = max_iter_override > 0 ? max_iter_override : 1000;
    double *g_abab = (double *)calloc(n, sizeof(double));
    double *g_abba = (double *)calloc(n, sizeof(double));
    Diis dd;
    if (!g_abab || !g_abba || diis_setup(&dd, n, t_abab, t_abba) != 0) { free(g_abab); free(g_abba); return -1; }
    int nd = dd.ndiis;
    int niter = 1;
    double dt = fmax(maxabs(t_abab, n), maxabs(t_abba, n));
    double e = uo_ccd_energy(c, t_aaaa, t_abab, t_abba);
    int nrec = 0;
    if (nrec < max_rec) { if (energies) energies[nrec] = e; if (dts) dts[nrec] = dt; nrec++; }
    int mask = 1 | (u->do_mosaic ? 2 : 0) | (u->do_ladder ? 4 : 0) | (u->do_ring ? 8 : 0) | (u->do_xring ? 16 : 0);
    while (dt >= tolmax && niter < max_iter) {
        get_t_from_diis(t_abab, dd.old_abab, dd.r_abab, n, nd, niter);
        get_t_from_diis(t_abba, dd.old_abba, dd.r_abba, n, nd, niter);
        for (size_t x = 0; x < n; x++) t_aaaa[x] = t_abab[x] + t_abba[x];
        uo_ccd_g2(c, t_abab, t_abba, mask, g_abab, g_abba);
        get_res(c, t_abab, g_abab, dd.r_abab + n * (nd - 1));
        get_res(c, t_abba, g_abba, dd.r_abba + n * (nd - 1));
        solve_cc(c, t_abab, g_abab, c->denom_factor_ccd);
        solve_cc(c, t_abba, g_abba, c->denom_factor_ccd);
        for (size_t x = 0; x < n; x++) t_aaaa[x] = t_abab[x] + t_abba[x];
        niter = niter + 1;
        double d1 = cnvrg_channel(t_abab, dd.old_abab, n, nd);
        double d2 = cnvrg_channel(t_abba, dd.old_abba, n, nd);
        dt = fmax(d1, d2);
        e = uo_ccd_energy(c, t_aaaa, t_abab, t_abba);
        if (nrec < max_rec) { if (energies) energies[nrec] = e; if (dts) dts[nrec] = dt; nrec++; }
    }
    /* final residual check (CCD.f90:103-107) */
    uo_ccd_g2(c, t_abab, t_abba, mask, g_abab, g_abba);
    get_res(c, t_abab, g_abab, dd.r_abab + n * (nd - 1));
    get_res(c, t_abba, g_abba, dd.r_abba + n * (nd - 1));
    double maxres = fmax(maxabs(dd.r_abab + n * (nd - 1), n), maxabs(dd.r_abba + n * (nd - 1), n));
    if (st) {
        st->ecorr = c->heg.ecorr;
        st->ecorr_sosex = 0.0;
        st->max_res = maxres;
        st->last_dt = dt;
        st->niter = niter;
        st->fail = maxres > failratio * tolmax;
        st->n_recorded = nrec;
    }
    diis_free(&dd);
    free(g_abab);
    free(g_abba);
    return 0;
}

/* ----------------------------------------------------------------- dRPA.f90 */

/* CCEnergy (dRPA.f90:181-216) */
double uo_drpa_energy(UoCtx *c, const double *t2, double csosex)
{
    const Info *u = &c->info;
    int O = u->nocc, M = u->nao;
    double ecorr = 0.0;
    for (int i = 1; i <= O; i++)
        for (int j = 1; j <= O; j++)
            for (int a = O + 1; a <= M; a++) {
                int b = FIND(c, i, j, a);
                if (b <= O) continue;
                double v_ijab = ERI(c, a, b, i, j, 0);
                double v_ijba = ERI(c, b, a, i, j, 0);
                int x = tix(O, i, j, a);
                double de = v_ijab * t2[x] * 2 - v_ijba * t2[x] * csosex;
                ecorr = ecorr + de;
            }
    c->heg.ecorr = ecorr;
    return ecorr;
}

void uo_drpa_g2(UoCtx *c, const double *t2, int mask, double *g2)
{
    const Info *u = &c->info;
    int O = u->nocc, M = u->nao;
    size_t n = (size_t)O * O * (M - O);
    memset(g2, 0, n * sizeof(double));
    /* GetG2Drivers (dRPA.f90:339-374) */
    if (mask & 1)
        for (int i = 1; i <= O; i++)
            for (int j = 1; j <= O; j++)
                for (int a = O + 1; a <= M; a++) {
                    int b = FIND(c, i, j, a);
                    if (b <= O) continue;
                    double v = ERI(c, i, j, a, b, u->irange_driver_direct);
                    if (v < -80.0) continue;
                    g2[tix(O, i, j, a)] = v;
                }
    /* GetG2Mosaics (dRPA.f90:377-446) */
    if (mask & 2) {
        double *joo = (double *)calloc((size_t)O, sizeof(double));
        double *jvv = (double *)calloc((size_t)(M - O), sizeof(double));
        for (int k = 1; k <= O; k++)
            for (int l = 1; l <= O; l++)
                for (int cc = O + 1; cc <= M; cc++) {
                    int d = FIND(c, k, l, cc);
                    if (d <= O) continue;
                    double v = ERI(c, cc, d, k, l, u->irange_mosaic);
                    if (v < -80.0) continue;
                    int x = tix(O, k, l, cc);
                    jvv[cc - O - 1] = jvv[cc - O - 1] + 2 * v * t2[x];
                    joo[k - 1] = joo[k - 1] + 2 * v * t2[x];
                }
        for (int i = 1; i <= O; i++)
            for (int j = 1; j <= O; j++)
                for (int a = O + 1; a <= M; a++) {
                    int b = FIND(c, i, j, a);
                    if (b <= O) continue;
                    int x = tix(O, i, j, a);
                    g2[x] = g2[x] - F12 * (jvv[a - O - 1] * t2[x] + jvv[b - O - 1] * t2[x]);
                    g2[x] = g2[x] - F12 * (joo[i - 1] * t2[x] + joo[j - 1] * t2[x]);
                }
        free(joo);
        free(jvv);
    }
    /* GetG2Rings (dRPA.f90:453-551) */
    if (mask & 8) {
        for (int i = 1; i <= O; i++)
            for (int j = 1; j <= O; j++)
                for (int a = O + 1; a <= M; a++) {
                    int b = FIND(c, i, j, a);
                    if (b <= O) continue;
                    int x = tix(O, i, j, a);
                    for (int k = 1; k <= O; k++) {
                        int cc = FIND(c, i, k, a);
                        if (cc <= O) continue;
                        int f = imax3(u->irange_ring, u->irange_direct_rings, u->irange_lin_rings);
                        double v = ERI(c, cc, j, k, b, f);
                        if (v < -80.0) continue;
                        g2[x] = g2[x] + 2 * v * t2[tix(O, i, k, a)];
                    }
                    for (int k = 1; k <= O; k++) {
                        int cc = FIND(c, j, k, b);
                        if (cc <= O) continue;
                        int f = imax3(u->irange_ring, u->irange_direct_rings, u->irange_lin_rings);
                        double v = ERI(c, cc, i, k, a, f);
                        if (v < -80.0) continue;
                        g2[x] = g2[x] + 2 * v * t2[tix(O, j, k, b)];
                    }
                }
        for (int i = 1; i <= O; i++)
            for (int a = O + 1; a <= M; a++)
                for (int l = 1; l <= O; l++) {
                    double jj = 0.0;
                    for (int k = 1; k <= O; k++) {
                        int cc = FIND(c, i, k, a);
                        if (cc <= O) continue;
                        int d = FIND(c, k, l, cc);
                        if (d <= O) continue;
                        int f = imax3(u->irange_ring, u->irange_direct_rings, u->irange_quad_rings);
                        double v = ERI(c, cc, d, k, l, f);
                        if (v < -80.0) continue;
                        jj = jj + 2 * t2[tix(O, i, k, a)] * v;
                    }
                    for (int j = 1; j <= O; j++) {
                        int b = FIND(c, i, j, a);
                        if (b <= O) continue;
                        int d = FIND(c, j, l, b);
                        if (d <= O) continue;
                        int x = tix(O, i, j, a);
                        g2[x] = g2[x] + 2 * jj * t2[tix(O, l, j, d)];
                    }
                }
    }
}

/* DrvdRPA (dRPA.f90:23-174) */
int uo_drpa(UoCtx *c, double *t2, int max_iter_override, UoSolveStats *st, double *energies, double *dts, int max_rec)
{
    const Info *u = &c->info;
    int O = u->nocc, M = u->nao;
    size_t n = (size_t)O * O * (M - O);
    double tolmax = 1.0e-8, failratio = 100;
    find_tol(c->heg.rS, &tolmax, &failratio, &c->denom_factor_drpa);
    const int max_iter = max_iter_override > 0 ? max_iter_override : 1000;
    double *g2 = (double *)calloc(n, sizeof(double));
    Diis dd;
    if (!g2 || diis_setup(&dd, n, t2, t2) != 0) { free(g2); return -1; }
    int nd = dd.ndiis;
    int niter = 1;
    double dt = maxabs(t2, n);
    double e = uo_drpa_energy(c, t2, 0.0);
    int nrec = 0;
    if (nrec < max_rec) { if (energies) energies[nrec] = e; if (dts) dts[nrec] = dt; nrec++; }
    int mask = 1 | (u->do_mosaic ? 2 : 0) | (u->do_ring ? 8 : 0);
    while (dt >= tolmax && niter < max_iter) {
        get_t_from_diis(t2, dd.old_abab, dd.r_abab, n, nd, niter);
        uo_drpa_g2(c, t2, mask, g2);
        get_res(c, t2, g2, dd.r_abab + n * (nd - 1));
        solve_cc(c, t2, g2, c->denom_factor_drpa);
        niter = niter + 1;
        dt = cnvrg_channel(t2, dd.old_abab, n, nd);
        e = uo_drpa_energy(c, t2, 0.0);
        if (nrec < max_rec) { if (energies) energies[nrec] = e; if (dts) dts[nrec] = dt; nrec++; }
    }
    uo_drpa_g2(c, t2, mask, g2);
    get_res(c, t2, g2, dd.r_abab + n * (nd - 1));
    double maxres = maxabs(dd.r_abab + n * (nd - 1), n);
    failratio = 10000;
    int fail = maxres > failratio * tolmax;
    double edrpa = c->heg.ecorr, esosex = 0.0;
    if (!fail) esosex = uo_drpa_energy(c, t2, 1.0);
    if (st) {
        st->ecorr = edrpa;
        st->ecorr_sosex = esosex;
        st->max_res = maxres;
        st->last_dt = dt;
        st->niter = niter;
        st->fail = fail;
        st->n_recorded = nrec;
    }
    diis_free(&dd);
    free(g2);
    return 0;
}

/* --------------------------------------------------------- Main.f90 TA loop */

int uo_twist_average(UoCtx *c, int ntw, const double *twists, double *per_twist, double *special,
                     UoSolveStats *final_st, double *final_mp2)
{
    const Info *u = &c->info;
    int O = u->nocc;
    int M = u->nao;
    size_t n = (size_t)O * O * (M - O);
    double *x_aaaa = (double *)calloc(n, sizeof(double)), *x_abab = (double *)calloc(n, sizeof(double));
    double *x_abba = (double *)calloc(n, sizeof(double));
    double *eig_sum = (double *)calloc((size_t)M, sizeof(double));
    int *conn = (int *)calloc((size_t)ntw * 400, sizeof(int));
    int conn_sum[400];
    memset(conn_sum, 0, sizeof conn_sum);
    if (!x_aaaa || !x_abab || !x_abba || !eig_sum || !conn) return -1;
    for (int it = 0; it < ntw; it++) {
        if (uo_change_twist(c, twists + 3 * it) != 0) return -1;
        double mp2 = uo_mp2(c, x_aaaa, x_abab, x_abba, conn + 400 * it);
        double hf = c->heg.ehf;
        double ccd = c->heg.ecorr;
        if (u->do_calc_ta_ccd) {
            UoSolveStats s;
            if (!u->do_drpa_sosex) uo_ccd(c, x_aaaa, x_abab, x_abba, 0, &s, NULL, NULL, 0);
            else uo_drpa(c, x_aaaa, 0, &s, NULL, NULL, 0);
            ccd = c->heg.ecorr;
        }
        per_twist[3 * it + 0] = hf;
        per_twist[3 * it + 1] = mp2;
        per_twist[3 * it + 2] = ccd;
        for (int p = 0; p < 400; p++) conn_sum[p] += conn[400 * it + p];
        for (int p = 0; p < M; p++) eig_sum[p] = eig_sum[p] + c->heg.eigen[p];
    }
    double conn_avg[400];
    for (int p = 0; p < 400; p++) conn_avg[p] = (double)conn_sum[p] / ntw;
    double *eig_avg = (double *)calloc((size_t)M, sizeof(double));
    for (int p = 0; p < M; p++) eig_avg[p] = eig_sum[p] / ntw;
    double best = 1.0 * 100000;
    int best_it = 0;
    for (int it = 0; it < ntw; it++) {
        double s = 0.0;
        for (int p = 0; p < 400; p++) {
            double d = (conn[400 * it + p] - conn_avg[p]) / pow((double)(p + 1), 2.0);
            s = s + d * d;
        }
        if (it == 0) { best = s; best_it = 0; }
        if (s < best) { best = s; best_it = it; }
    }
    for (int d = 0; d < 3; d++) special[d] = twists[3 * best_it + d];
    if (uo_change_twist(c, special) != 0) return -1;
    memcpy(c->heg.eigen, eig_avg, sizeof(double) * M);
    double mp2 = uo_mp2(c, x_aaaa, x_abab, x_abba, NULL);
    if (final_mp2) *final_mp2 = mp2;
    if (!u->do_drpa_sosex) uo_ccd(c, x_aaaa, x_abab, x_abba, 0, final_st, NULL, NULL, 0);
    else uo_drpa(c, x_aaaa, 0, final_st, NULL, NULL, 0);
    free(x_aaaa); free(x_abab); free(x_abba); free(eig_sum); free(eig_avg); free(conn);
    return 0;
}
