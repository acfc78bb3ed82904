// zcode.cpp -- the reference's ZCode program (Main.f90:2-320) as a library
// function, with its hot path on the GPU through include/uegccd.h.
//
// Steps of uegccd_zcode (Main.f90 line ranges):
//   44-48    ReadInput, init_HEG; SetPointers' integrals: CoreN and GapII are
//            served (CoreERI, GapERI, NoCaseERI); one range flag shared by all fifteen
//            "... Range" values is served under CasedERI, different flags are refused,
//            and the flags are ignored where the reference ignores them
//   78-79    change_rs to rSMin
//   83-93    DoSingleCalc: MP2, then CCD or dRPA from the MP2 amplitudes
//   95-97    DoSkipTA: stop after the single calculation
//   112-168  every twist's MP2 (and CCD/dRPA when DoCalcTACCD) -- solved here as
//            ONE GPU batch over all twists; the Output blocks are then written
//            in twist order, as the reference's loop writes them
//   170-231  averages, connectivity histogram, special twist (fort.58, fort.59)
//   233-255  MP2 + CCD/dRPA at the special twist with the twist-averaged
//            eigenvalues, NumRSPoints times
// Structure factors: fort.81 after every DrvMBPT (MP2.f90:98-113), fort.80 in
// DrvCCD when DoSFCalcMP2 / DoSFCalcCCD (CCD.f90:65,109), fort.82 after every
// print_HF (HEG.f90:612); DoOnlyMP2Grid stops after the first DrvMBPT
// (MP2.f90:152-154).
//
// Twists: the reference draws them with gfortran's rand() seeded 86456
// (Main.f90:30,81; HEG.f90:535-549), which is not reproduced here.  The caller
// passes a twist file (three numbers per line, used in order); missing twists
// come from a std::mt19937_64 stream seeded 86456, U[-0.5,0.5)^3.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <random>
#include <string>
#include <vector>

#include "../../include/uegccd.h"
#include "../../include/uegccd_host.h"
#include "listdir.h"

namespace {

using uegccd::ld_int;
using uegccd::ld_real;
using uegccd::ld_str;

thread_local std::string g_zc_error;

int zfail(int code, const std::string &m)
{
    g_zc_error = m;
    return code;
}

// ---- Output blocks (formats of MP2.f90:143-150, CCD.f90:127-140, dRPA.f90:123-138)

const char *kStars = "              **************************************************\n";
const char *kBar = "              *------------------------------------------------*\n";

void write_mp2(FILE *f, double ehf, const double *eig, int nocc, int nao, double e2)
{
    std::fputs(kStars, f);
    std::fprintf(f, "              * E(SCF) is             %18.12f a.u.  *\n", ehf);
    std::fputs(kBar, f);
    std::fprintf(f, "              *                RHF Eigenvalues:                *\n");
    std::fputs(kBar, f);
    for (int i = 0; i < nocc; i++) std::fprintf(f, "              *            %24.16E            *\n", eig[i]);
    std::fprintf(f, "              *            ------------------------            *\n");
    for (int a = nocc; a < nao; a++) std::fprintf(f, "              *            %24.16E            *\n", eig[a]);
    std::fputs(kStars, f);
    std::fprintf(f, "              * E(2) is               %18.12f a.u.  *\n", e2);
    std::fprintf(f, "              * E(SCF) + E(2) is      %18.12f a.u.  *\n", e2 + ehf);
    std::fputs(kStars, f);
}

void write_cc(FILE *f, const UegccdInput &in, int drpa, const UegccdResult &r, const double *en,
              const double *dt, int nrec, double ehf)
{
    std::fprintf(f, drpa ? "              *              dRPA summary follows              *\n"
                         : "              *               CCD summary follows              *\n");
    std::fputs(kBar, f);
    if (in.do_ring) std::fprintf(f, "              * Including ring diagrams...                     *\n");
    if (!drpa && in.do_xring) std::fprintf(f, "              * Including crossed ring diagrams...             *\n");
    if (!drpa && in.do_ladder) std::fprintf(f, "              * Including ladder diagrams...                   *\n");
    if (in.do_mosaic) std::fprintf(f, "              * Including mosaic diagrams...                   *\n");
    std::fputs(kBar, f);
    std::fprintf(f, drpa ? "              * dRPA Energy      Iteration    Biggest change   *\n"
                         : "              *  CCD Energy      Iteration    Biggest change   *\n");
    for (int k = 0; k < nrec; k++)
        std::fprintf(f, "              * %15.10f  %5d       %14.10f    *\n", en[k], k + 1, dt[k]);
    std::fputs(kBar, f);
    if (r.fail) {
        std::fprintf(f, drpa ? "              * Final dRPA Energy is   DID NOT CONVERGE        *\n"
                             : "              * Final CCD Energy is   DID NOT CONVERGE         *\n");
    } else if (!drpa) {
        std::fprintf(f, "              * CCD has converged in %3d iterations            *\n", r.niter);
        std::fprintf(f, "              * Ec(CCD) is           %18.12f a.u.   *\n", r.ecorr);
        std::fprintf(f, "              * Final CCD Energy is  %18.12f a.u.   *\n", r.ecorr + ehf);
    } else {
        std::fprintf(f, "              * dRPA has converged in %3d iterations           *\n", r.niter);
        std::fprintf(f, "              * Ec(dRPA) is          %18.12f a.u.   *\n", r.ecorr);
        std::fprintf(f, "              * Final dRPA Energy is %18.12f a.u.   *\n", r.ecorr + ehf);
        std::fprintf(f, "              * Ec(SOSEX) is         %18.12f a.u.   *\n", r.ecorr_sosex);
        std::fprintf(f, "              * Final SOSEX Energy is%18.12f a.u.   *\n", r.ecorr_sosex + ehf);
    }
    char es[32];
    std::snprintf(es, sizeof es, "%.12E", r.max_res);  // ES18.12
    std::fprintf(f, "              * Max CCD Residual is      %18s    *\n", es);
    std::fputs(kStars, f);
}

constexpr double kPiZ = 3.1415926535897932384626433833;  // Constants.f90:7

// HEGData%ScreeningDistance after change_rs (HEG.f90:509-511)
static double screening_of(const UegccdInput &in, double L)
{
    const double density = in.nelectron / std::pow(L, 3.0);
    const double kf = std::pow(3.0 * std::pow(kPiZ, 2.0) * density, 1.0 / 3.0);
    return std::pow(4.0 / kPiZ * kf, 0.5);
}

// DrvCCD / DrvdRPA options from the Input (FindTol sees rS = 1, HEG.f90:28; the
// dRPA driver's FailRatio is 1e4, dRPA.f90:100)
UegccdOptions options_for(const UegccdInput &in, int32_t scheme)
{
    UegccdOptions o;
    uegccd_default_options(&o);
    double tolmax = 1e-8, failratio = 100, denom = 2.0;
    uegccd_find_tol(1.0, &tolmax, &failratio, &denom);
    o.tol = tolmax;
    o.fail_ratio = in.do_drpa_sosex ? 1.0e4 : failratio;
    o.denom_factor = denom;
    o.do_ring = in.do_ring;
    o.do_xring = in.do_xring;
    o.do_ladder = in.do_ladder;
    o.do_mosaic = in.do_mosaic;
    o.core_n = (int32_t)((in.nelectron / 2) * in.core_factor);
    o.gapii = in.gapii;
    // The range flags act only through CasedERI, which SetPointers (Main.f90:299-302) picks
    // under Safe ERI, or when range flags, GapII and CoreN are all set; any other ERI routine
    // ignores them.
    const bool cased = in.safe_eri || (in.range_flags > 0 && o.gapii > 0.0 && o.core_n > 0);
    o.range_flags = cased ? in.range_flags : 0;
    if (scheme == UEGCCD_DIIS) {
        o.scheme = UEGCCD_DIIS;
        o.ndiis = 6;
        o.denom_factor = 1.0;
    }
    return o;
}

// The two-channel form (uegccd_ctx_set_eri): CCD with only one of rings / crossed rings, or
// with range flags that differ between terms under CasedERI; dRPA with range flags under
// CasedERI.  *eri: CasedERI applies the flags, so the context takes them with set_eri.
bool two_channel_of(const UegccdInput &in, const UegccdOptions &opt, bool *eri)
{
    const bool cased = in.safe_eri || (in.range_flags > 0 && opt.gapii > 0.0 && opt.core_n > 0);
    *eri = cased;
    if (in.do_drpa_sosex) return cased && in.range_flags > 0;
    return in.do_ring != in.do_xring || (cased && in.range_uniform < 0);
}

// ---- structure-factor files (fort.80, fort.81), opened on their first block

struct SfGrids {
    int S = 0;
    std::vector<double> sum, dsum, xsum, g, v;
    UegccdSfGrid view(int32_t S_)
    {
        S = S_;
        const size_t W = 2 * (size_t)S + 1, n = W * W * W;
        for (auto *a : {&sum, &dsum, &xsum, &g, &v}) a->assign(n, 0.0);
        return UegccdSfGrid{sum.data(), dsum.data(), xsum.data(), g.data(), v.data()};
    }
};

// One block: fort.81 (DrvMBPT, MP2.f90:98-113: the points with SfG > 0; q, SfG, SfSum,
// SfV) or fort.80 (CCEnergyAndSF, CCD.f90:263-266,334-342: SfG > 1e-10; also SfDSum,
// SfXSum).  x outermost, z innermost, as the reference's loops run.
std::string sf_block(const SfGrids &f, bool ccd)
{
    std::string o = ld_str("--------") + "\n" + ld_str("Starting a new structure factor") + "\n" +
                    ld_str("--------") + "\n";
    const int S = f.S;
    const size_t W = 2 * (size_t)S + 1;
    for (int x = -S; x <= S; x++)
        for (int y = -S; y <= S; y++)
            for (int z = -S; z <= S; z++) {
                const size_t k = (size_t)(x + S) + W * ((size_t)(y + S) + W * (size_t)(z + S));
                if (!(ccd ? f.g[k] > 1.0e-10 : f.g[k] > 0.0)) continue;
                o += ld_int(x) + ld_int(y) + ld_int(z) + ld_real(f.g[k]) + ld_real(f.sum[k]) + ld_real(f.v[k]);
                if (ccd) o += ld_real(f.dsum[k]) + ld_real(f.xsum[k]);
                o += "\n";
            }
    return o;
}

struct SfFiles {
    FILE *f80 = nullptr, *f81 = nullptr;
    bool mp2_in_cc = false, ccd = false;   // DoSFCalcMP2, DoSFCalcCCD
    SfFiles() = default;
    SfFiles(const SfFiles &) = delete;
    SfFiles &operator=(const SfFiles &) = delete;
    ~SfFiles()
    {
        if (f80) std::fclose(f80);
        if (f81) std::fclose(f81);
    }
    int put(int unit, const std::string &text)
    {
        FILE *&f = unit == 80 ? f80 : f81;
        if (!f) f = std::fopen(unit == 80 ? "fort.80" : "fort.81", "w");
        if (!f) return zfail(UEGCCD_ERR_ARG, unit == 80 ? "cannot write fort.80" : "cannot write fort.81");
        std::fputs(text.c_str(), f);
        return UEGCCD_OK;
    }
};

// fort.81 or fort.80 block of spin-adapted amplitudes on a context
int sf_ctx(UegccdCtx *ctx, const UegccdSystem &sys, const double *t_abab, SfFiles &sf, int unit)
{
    SfGrids g;
    const UegccdSfGrid v = g.view(uegccd_sf_length(&sys));
    if (int rc = uegccd_structure_factor(ctx, t_abab, &v)) return zfail(rc, uegccd_last_error());
    return sf.put(unit, sf_block(g, unit == 80));
}

struct Amps {
    std::vector<double> aaaa, abab, abba;
    explicit Amps(const UegccdSystem &s)
    {
        const size_t n = (size_t)s.nocc * s.nocc * (s.nao - s.nocc);
        aaaa.assign(n, 0.0);
        abab.assign(n, 0.0);
        abba.assign(n, 0.0);
    }
};

// DrvMBPT into x, then DrvCCD/DrvdRPA on t (started from x when copy_start);
// both Output blocks appended, and the structure-factor blocks.  Under DoOnlyMP2Grid
// it returns after the MP2 step (the program ends there).
int mp2_then_cc(const UegccdInput &in, const UegccdSystem &sys, double ehf, const UegccdOptions &opt, Amps &x,
                Amps &t, bool copy_start, UegccdResult *res, SfFiles &sf)
{
    UegccdCtx *ctx = nullptr;
    if (uegccd_ctx_create(&sys, &ctx)) return zfail(UEGCCD_ERR_CUDA, uegccd_last_error());
    double e2 = 0.0;
    int rc = uegccd_ctx_set_integrals(ctx, opt.core_n, opt.gapii);  // the ERI that SetPointers chose
    // one range flag for every term (otherwise the solve refuses range_flags != 0)
    if (!rc && opt.range_flags != 0 && in.range_uniform > 0)
        rc = uegccd_ctx_set_range(ctx, in.range_uniform, screening_of(in, sys.L));
    // the two-channel form: the fifteen flags themselves under CasedERI
    bool eri = false;
    if (!rc && two_channel_of(in, opt, &eri) && eri)
        rc = uegccd_ctx_set_eri(ctx, &in.range_terms, in.safe_eri, screening_of(in, sys.L));
    if (!rc) rc = uegccd_mp2(ctx, x.aaaa.data(), x.abab.data(), x.abba.data(), &e2);
    if (rc) {
        zfail(rc, uegccd_last_error());
        uegccd_ctx_destroy(ctx);
        return rc;
    }
    if ((rc = sf_ctx(ctx, sys, x.abab.data(), sf, 81))) {
        uegccd_ctx_destroy(ctx);
        return rc;
    }
    FILE *f = std::fopen("Output", "a");
    if (!f) {
        uegccd_ctx_destroy(ctx);
        return zfail(UEGCCD_ERR_ARG, "cannot append to Output");
    }
    write_mp2(f, ehf, sys.eigen, sys.nocc, sys.nao, e2);
    if (in.do_only_mp2_grid) {  // "DoOnlyMP2Grid flag is true, so calculation stopping here"
        std::fclose(f);
        uegccd_ctx_destroy(ctx);
        return UEGCCD_OK;
    }
    if (copy_start) t = x;
    UegccdOptions o = opt;
    std::vector<double> en(1100), dt(1100);
    o.energies = en.data();
    o.dts = dt.data();
    o.max_rec = 1100;
    if (!in.do_drpa_sosex && sf.mp2_in_cc && (rc = sf_ctx(ctx, sys, t.abab.data(), sf, 80))) {
        std::fclose(f);
        uegccd_ctx_destroy(ctx);
        return rc;
    }
    rc = in.do_drpa_sosex ? uegccd_drpa(ctx, &o, t.aaaa.data(), res)
                          : uegccd_ccd(ctx, &o, t.aaaa.data(), t.abab.data(), t.abba.data(), res);
    if (rc >= 0) {
        rc = 0;
        if (!in.do_drpa_sosex && sf.ccd) rc = sf_ctx(ctx, sys, t.abab.data(), sf, 80);
        write_cc(f, in, in.do_drpa_sosex, *res, en.data(), dt.data(), res->n_recorded, ehf);
    } else {
        zfail(rc, uegccd_last_error());
    }
    std::fclose(f);
    uegccd_ctx_destroy(ctx);
    return rc;
}

std::vector<std::array<double, 3>> twist_list(const char *path, int count)
{
    std::vector<std::array<double, 3>> tw;
    if (path && *path) {
        std::ifstream f(path);
        double x, y, z;
        while ((int)tw.size() < count && (f >> x >> y >> z)) tw.push_back({x, y, z});
    }
    std::mt19937_64 rng(86456);
    std::uniform_real_distribution<double> u(-0.5, 0.5);
    while ((int)tw.size() < count) {
        const double a = u(rng), b = u(rng), c = u(rng);
        tw.push_back({a, b, c});
    }
    return tw;
}

struct HegGuard {
    UegccdHeg *h = nullptr;
    HegGuard() = default;
    HegGuard(const HegGuard &) = delete;
    HegGuard &operator=(const HegGuard &) = delete;
    ~HegGuard() { uegccd_heg_destroy(h); }
};

}  // namespace

extern "C" {

const char *uegccd_zcode_last_error(void) { return g_zc_error.c_str(); }

int uegccd_connectivity(const UegccdSystem *s, int32_t core_n, int32_t *conn)
{
    if (!s || !conn || !s->nvec || s->nocc <= 0 || s->nao <= s->nocc)
        return zfail(UEGCCD_ERR_ARG, "bad argument");
    const int O = s->nocc, M = s->nao;
    auto n = [&](int p, int d) { return s->nvec[p + (size_t)M * d]; };
    int r = 0;
    for (int p = 0; p < M; p++)
        for (int d = 0; d < 3; d++) r = std::max(r, std::abs(n(p, d)));
    const int side = 4 * r + 1;
    std::vector<int> orb((size_t)side * side * side, -1);
    auto key = [&](int x, int y, int z) {
        return ((size_t)(x + 2 * r) * side + (size_t)(y + 2 * r)) * side + (size_t)(z + 2 * r);
    };
    for (int p = 0; p < M; p++) orb[key(n(p, 0), n(p, 1), n(p, 2))] = p;
    std::fill(conn, conn + UEGCCD_CONN_LIMIT, 0);
    for (int i = 0; i < O; i++)
        for (int j = 0; j < O; j++)
            for (int a = O; a < M; a++) {
                // FindIndex: the virtual b with n_b = n_i + n_j - n_a
                const int x = n(i, 0) + n(j, 0) - n(a, 0), y = n(i, 1) + n(j, 1) - n(a, 1),
                          z = n(i, 2) + n(j, 2) - n(a, 2);
                if (std::abs(x) > 2 * r || std::abs(y) > 2 * r || std::abs(z) > 2 * r) continue;
                const int b = orb[key(x, y, z)];
                if (b < O) continue;
                // dK2(I,J,A,B) = |n_i - n_a|^2, dK2(I,J,B,A) = |n_i - n_b|^2 (HEG.f90:985-1005)
                int qa = 0, qb = 0;
                for (int d = 0; d < 3; d++) {
                    qa += (n(i, d) - n(a, d)) * (n(i, d) - n(a, d));
                    qb += (n(i, d) - n(b, d)) * (n(i, d) - n(b, d));
                }
                if (qa > UEGCCD_CONN_LIMIT || qb > UEGCCD_CONN_LIMIT)
                    return zfail(UEGCCD_ERR_ARG, "Connectivity greater than current ConnectivityLimit");
                if (i < core_n || j < core_n || a < core_n || b < core_n) continue;  // InCore
                conn[qb - 1]++;
                conn[qa - 1]++;
            }
    return UEGCCD_OK;
}

int uegccd_special_twist(int32_t ntw, const int32_t *conn, double *conn_avg, double *diff2, int32_t *best)
{
    if (ntw <= 0 || !conn || !best) return zfail(UEGCCD_ERR_ARG, "bad argument");
    std::vector<long long> sum(UEGCCD_CONN_LIMIT, 0);
    for (int t = 0; t < ntw; t++)
        for (int k = 0; k < UEGCCD_CONN_LIMIT; k++) sum[k] += conn[(size_t)t * UEGCCD_CONN_LIMIT + k];
    std::vector<double> avg(UEGCCD_CONN_LIMIT);
    for (int k = 0; k < UEGCCD_CONN_LIMIT; k++) avg[k] = (double)sum[k] / ntw;
    double best_d = 1.0 * 100000;
    int bt = 0;
    for (int t = 0; t < ntw; t++) {
        double d2 = 0.0;
        for (int k = 0; k < UEGCCD_CONN_LIMIT; k++) {
            const double d = (conn[(size_t)t * UEGCCD_CONN_LIMIT + k] - avg[k]) / std::pow((double)(k + 1), 2.0);
            d2 = d2 + d * d;
        }
        if (t == 0) best_d = d2;
        if (d2 < best_d) {
            best_d = d2;
            bt = t;
        }
        if (diff2) diff2[t] = d2;
    }
    if (conn_avg) std::copy(avg.begin(), avg.end(), conn_avg);
    *best = bt;
    return UEGCCD_OK;
}

int32_t uegccd_list_real(double x, char *buf, int32_t len)
{
    const std::string s = ld_real(x);
    if (!buf || len <= (int32_t)s.size()) return zfail(UEGCCD_ERR_ARG, "buffer too small");
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return (int32_t)s.size();
}

// The program; gpu = false runs only the host set-up (it writes the fort.60 log, and
// fort.82 when f82_path is given).
static int run_zcode(const char *input_path, const char *twists_path, int32_t scheme, bool gpu, const char *log_path,
                     const char *f82_path, const char *f61_path)
{
    UegccdInput in;
    if (uegccd_read_input(input_path ? input_path : "Input", 0, &in))
        return zfail(UEGCCD_ERR_ARG, std::string("ReadInput: ") + uegccd_host_last_error());
    if (f61_path && in.core_factor_set) {
        // ReadInput's CAS counts (IO.f90:232-234)
        const int core_n = (int)((in.nelectron / 2) * in.core_factor);
        FILE *f = std::fopen(f61_path, "w");
        if (!f) return zfail(UEGCCD_ERR_ARG, "cannot write fort.61");
        std::fprintf(f, "%s\n%s\n", (ld_int(core_n * 2) + ld_str("core electrons")).c_str(),
                     (ld_int(in.nelectron - core_n * 2) + ld_str("active electrons")).c_str());
        std::fclose(f);
    }
    // fort.60 (set-up log) and fort.82 (exchange structure factors): collected while the
    // program runs and written at the end
    struct LogFile {
        std::string text;
        std::string path;
        void (*sink)(std::string *);
        LogFile(const char *p, void (*set)(std::string *)) : path(p ? p : ""), sink(set)
        {
            if (!path.empty()) sink(&text);
        }
        ~LogFile()
        {
            if (path.empty()) return;
            sink(nullptr);
            if (FILE *f = std::fopen(path.c_str(), "w")) {
                std::fputs(text.c_str(), f);
                std::fclose(f);
            }
        }
    } log(log_path, uegccd::heg_log_to), log82(f82_path, uegccd::heg_sf_log_to);
    auto logl = [&](const std::string &l) { log.text += l + "\n"; };
    HegGuard h;
    if (uegccd_heg_create(&in, &h.h)) return zfail(UEGCCD_ERR_ARG, std::string("init_HEG: ") + uegccd_host_last_error());
    if (gpu) {
        if (FILE *f = std::fopen("Output", "w")) std::fclose(f);  // Main.f90:61-62
        else return zfail(UEGCCD_ERR_ARG, "cannot create Output");
    }
    SfFiles sf;
    sf.mp2_in_cc = in.do_sf_calc_mp2 != 0;
    sf.ccd = in.do_sf_calc_ccd != 0;
    const UegccdOptions opt = options_for(in, scheme);
    // CCEnergyAndSF takes its integrals with the energy's range flag (CCD.f90:290-291): the
    // structure-factor grids are built on the plain integrals only
    if (opt.range_flags != 0 && (in.do_sf_calc_mp2 || in.do_sf_calc_ccd))
        return zfail(UEGCCD_ERR_UNSUPPORTED, "structure factors of range-separated integrals are outside the GPU path");
    bool two_eri = false;
    const bool two = two_channel_of(in, opt, &two_eri);
    // the structure-factor grids read spin-adapted amplitudes
    if (two && in.do_sf_calc_ccd && !in.do_drpa_sosex)
        return zfail(UEGCCD_ERR_UNSUPPORTED, "structure factors of two-channel CCD amplitudes are outside the GPU path");
    UegccdHegInfo info;
    UegccdSystem sys;
    UegccdResult res;
    int rc = 0;
    if (in.do_single_calc) {
        if (gpu) {
            uegccd_heg_info(h.h, &info);
            uegccd_heg_system(h.h, &sys);
            Amps x(sys), t(sys);
            if ((rc = mp2_then_cc(in, sys, info.ehf, opt, x, t, true, &res, sf))) return rc;
        }
        if (in.do_only_mp2_grid) return UEGCCD_OK;  // stopped in the first DrvMBPT
    }
    if (in.do_skip_ta) return UEGCCD_OK;  // "Finishing calculation after single point calculation"
    const int ntw = in.tacalcn;
    if (ntw <= 0) return UEGCCD_OK;       // no twists to average
    const auto tw = twist_list(twists_path, ntw);

    // every twist's basis, eigenvalues, E_HF and connectivity: ChangeTwist on the one
    // set-up, as the reference's loop does (Main.f90:112-118), the arrays copied out.
    // DoOnlyMP2Grid stops in the first twist's DrvMBPT.
    const int nset = in.do_only_mp2_grid ? 1 : ntw;
    std::vector<UegccdSystem> systems(nset);
    std::vector<std::vector<double>> eigs(nset);
    std::vector<std::vector<int32_t>> nvecs(nset);
    std::vector<double> hf(nset), mp2(nset), cc(nset);
    std::vector<int32_t> conn((size_t)nset * UEGCCD_CONN_LIMIT);
    for (int t = 0; t < nset; t++) {
        logl(ld_int(t + 1) + ld_str("of") + ld_int(ntw));
        logl(ld_str("randomizing twist angle"));  // GenerateTwist (HEG.f90:541-547): here, the listed twist
        logl(ld_str("generated") + ld_real(tw[t][0]) + ld_real(tw[t][1]) + ld_real(tw[t][2]));
        if (uegccd_heg_change_twist(h.h, tw[t].data())) return zfail(UEGCCD_ERR_ARG, uegccd_host_last_error());
        uegccd_heg_info(h.h, &info);
        hf[t] = info.ehf;
        uegccd_heg_system(h.h, &systems[t]);
        if (t == 0) logl(ld_str("EIGEN") + ld_int(systems[t].nao));
        eigs[t].assign(systems[t].eigen, systems[t].eigen + systems[t].nao);
        nvecs[t].assign(systems[t].nvec, systems[t].nvec + 3 * (size_t)systems[t].nao);
        systems[t].eigen = eigs[t].data();
        systems[t].nvec = nvecs[t].data();
        if (systems[t].nao != systems[0].nao) return zfail(UEGCCD_ERR_ARG, "twists give different basis sizes");
        if ((rc = uegccd_connectivity(&systems[t], opt.core_n, &conn[(size_t)t * UEGCCD_CONN_LIMIT]))) return rc;
    }
    const int M = systems[0].nao;
    std::vector<double> cavg(UEGCCD_CONN_LIMIT), diff2(nset);
    int32_t best = 0;
    if (!in.do_only_mp2_grid) uegccd_special_twist(ntw, conn.data(), cavg.data(), diff2.data(), &best);
    if (!gpu) {
        if (in.do_only_mp2_grid) return UEGCCD_OK;
        // the special twist's ChangeTwist ends the set-up log
        return uegccd_heg_change_twist(h.h, tw[best].data()) ? zfail(UEGCCD_ERR_ARG, uegccd_host_last_error())
                                                             : UEGCCD_OK;
    }

    // all twists in one batch: MP2 and its structure factor (fort.81), then CCD/dRPA
    // when DoCalcTACCD (Main.f90:126-139)
    struct BatchGuard {
        UegccdBatch *b = nullptr;
        ~BatchGuard() { uegccd_batch_destroy(b); }
    } bg;
    if (uegccd_batch_create(systems.data(), nset, &bg.b)) return zfail(UEGCCD_ERR_CUDA, uegccd_last_error());
    UegccdBatch *b = bg.b;
    if ((rc = uegccd_batch_set_integrals(b, opt.core_n, opt.gapii)) || (rc = uegccd_batch_mp2(b, mp2.data())))
        return zfail(rc, uegccd_last_error());
    if (opt.range_flags != 0 && in.range_uniform > 0 &&
        (rc = uegccd_batch_set_range(b, in.range_uniform, screening_of(in, systems[0].L))))
        return zfail(rc, uegccd_last_error());
    const bool cc_sf = in.do_calc_ta_ccd && !in.do_drpa_sosex;
    std::vector<std::string> mp2_80(nset);   // DrvCCD's DoSFCalcMP2 blocks, written beside the CCD ones
    for (int t = 0; t < nset; t++) {
        SfGrids g;
        const UegccdSfGrid v = g.view(uegccd_sf_length(&systems[t]));
        if ((rc = uegccd_batch_structure_factor(b, t, &v))) return zfail(rc, uegccd_last_error());
        if ((rc = sf.put(81, sf_block(g, false)))) return rc;
        if (cc_sf && sf.mp2_in_cc) mp2_80[t] = sf_block(g, true);
    }
    std::vector<UegccdResult> br(nset);
    std::vector<std::vector<double>> two_en, two_dt;   // the two-channel solves' iteration tables
    if (in.do_calc_ta_ccd && !in.do_only_mp2_grid) {
        if (two) {
            // one context per twist: the two-channel form runs one system at a time
            two_en.assign(nset, std::vector<double>(1100));
            two_dt.assign(nset, std::vector<double>(1100));
            for (int t = 0; t < nset; t++) {
                Amps x(systems[t]);
                UegccdOptions o = opt;
                o.energies = two_en[t].data();
                o.dts = two_dt[t].data();
                o.max_rec = 1100;
                UegccdCtx *ctx = nullptr;
                if (uegccd_ctx_create(&systems[t], &ctx)) return zfail(UEGCCD_ERR_CUDA, uegccd_last_error());
                double e2 = 0.0;
                rc = uegccd_ctx_set_integrals(ctx, opt.core_n, opt.gapii);
                if (!rc && two_eri)
                    rc = uegccd_ctx_set_eri(ctx, &in.range_terms, in.safe_eri, screening_of(in, systems[t].L));
                if (!rc) rc = uegccd_mp2(ctx, x.aaaa.data(), x.abab.data(), x.abba.data(), &e2);
                if (!rc)
                    rc = in.do_drpa_sosex ? uegccd_drpa(ctx, &o, x.aaaa.data(), &br[t])
                                          : uegccd_ccd(ctx, &o, x.aaaa.data(), x.abab.data(), x.abba.data(), &br[t]);
                if (rc < 0) zfail(rc, uegccd_last_error());
                uegccd_ctx_destroy(ctx);
                if (rc < 0) return rc;
                rc = 0;
            }
        } else {
            rc = uegccd_batch_solve(b, &opt, in.do_drpa_sosex, mp2.data(), br.data());
            if (rc < 0) return zfail(rc, uegccd_last_error());
        }
    }
    FILE *out = std::fopen("Output", "a");
    if (!out) return zfail(UEGCCD_ERR_ARG, "cannot append to Output");
    std::vector<double> en(1100), dt(1100);
    for (int t = 0; t < nset; t++) {
        const UegccdSystem &s = systems[t];
        write_mp2(out, hf[t], s.eigen, s.nocc, s.nao, mp2[t]);
        if (in.do_only_mp2_grid) break;  // "DoOnlyMP2Grid flag is true, so calculation stopping here"
        cc[t] = mp2[t];
        if (in.do_calc_ta_ccd) {
            if (cc_sf && sf.mp2_in_cc) rc = sf.put(80, mp2_80[t]);
            if (!rc && cc_sf && sf.ccd) {
                SfGrids g;
                const UegccdSfGrid v = g.view(uegccd_sf_length(&s));
                rc = uegccd_batch_structure_factor(b, t, &v) ? zfail(UEGCCD_ERR_CUDA, uegccd_last_error())
                                                              : sf.put(80, sf_block(g, true));
            }
            if (rc) {
                std::fclose(out);
                return rc;
            }
            int32_t nrec = 0;
            if (two) {
                nrec = br[t].n_recorded;
                write_cc(out, in, in.do_drpa_sosex, br[t], two_en[t].data(), two_dt[t].data(), nrec, hf[t]);
            } else {
                uegccd_batch_history(b, t, en.data(), dt.data(), 1100, &nrec);
                write_cc(out, in, in.do_drpa_sosex, br[t], en.data(), dt.data(), nrec, hf[t]);
            }
            // HEGData%ECorr after the driver: Ec(SOSEX) for a converged dRPA, else the last energy
            cc[t] = (in.do_drpa_sosex && !br[t].fail) ? br[t].ecorr_sosex : br[t].ecorr;
        }
    }
    std::fclose(out);
    if (in.do_only_mp2_grid) return UEGCCD_OK;
    uegccd_batch_destroy(bg.b);   // before the special-twist solve allocates its own
    bg.b = nullptr;

    // fort.59 per-twist rows and fort.58 connectivity rows (Main.f90:144-153)
    FILE *f59 = std::fopen("fort.59", "w");
    FILE *f58 = std::fopen("fort.58", "w");
    if (!f59 || !f58) {
        if (f59) std::fclose(f59);
        if (f58) std::fclose(f58);
        return zfail(UEGCCD_ERR_ARG, "cannot write fort.58/fort.59");
    }
    int cmax = 0;
    for (int k = UEGCCD_CONN_LIMIT; k >= 1; k--)
        if (conn[k - 1] > 0) {
            cmax = k;
            break;
        }
    std::vector<double> eig_sum(M, 0.0);
    std::array<double, 3> tws{0, 0, 0}, tws2{0, 0, 0};
    double s_hf = 0, s_mp2 = 0, s_cc = 0, s_hf2 = 0, s_mp22 = 0, s_cc2 = 0;
    for (int t = 0; t < ntw; t++) {
        std::string row;
        for (int d = 0; d < 3; d++) row += ld_real(tw[t][d]);
        row += ld_real(hf[t]) + ld_real(mp2[t]) + ld_real(cc[t]);
        std::fprintf(f59, "%s\n", row.c_str());
        row.clear();
        for (int k = 0; k < cmax; k++) row += ld_int(conn[(size_t)t * UEGCCD_CONN_LIMIT + k]);
        std::fprintf(f58, "%s\n", row.c_str());
        s_cc += cc[t];
        s_mp2 += mp2[t];
        s_hf += hf[t];
        for (int d = 0; d < 3; d++) {
            tws[d] += tw[t][d];
            tws2[d] += std::pow(tw[t][d], 2.0);
        }
        for (int p = 0; p < M; p++) eig_sum[p] = eig_sum[p] + systems[t].eigen[p];
        s_cc2 += std::pow(cc[t], 2.0);
        s_mp22 += std::pow(mp2[t], 2.0);
        s_hf2 += std::pow(hf[t], 2.0);
    }
    std::fclose(f58);
    // averages, <x^2>, errors sqrt((<x^2>-<x>^2)/(N-1)) (Main.f90:170-199)
    const double N = ntw;
    auto err = [&](double m2, double m) { return std::pow((m2 - std::pow(m, 2.0)) / (N - 1), 0.5); };
    std::string l1, l2, l3;
    for (int d = 0; d < 3; d++) {
        l1 += ld_real(tws[d] / N);
        l2 += ld_real(tws2[d] / N);
        l3 += ld_real(err(tws2[d] / N, tws[d] / N));
    }
    l1 += ld_real(s_hf / N) + ld_real(s_mp2 / N) + ld_real(s_cc / N) + ld_str("averages");
    l2 += ld_real(s_hf2 / N) + ld_real(s_mp22 / N) + ld_real(s_cc2 / N) + ld_str("squared averages");
    l3 += ld_real(err(s_hf2 / N, s_hf / N)) + ld_real(err(s_mp22 / N, s_mp2 / N)) + ld_real(err(s_cc2 / N, s_cc / N)) +
          ld_str("errors");
    std::fprintf(f59, "%s\n%s\n%s\n", l1.c_str(), l2.c_str(), l3.c_str());
    std::vector<double> eig_avg(M);
    std::string le;
    for (int p = 0; p < M; p++) {
        eig_avg[p] = eig_sum[p] / N;
        le += ld_real(eig_avg[p]);
    }
    std::fprintf(f59, "%s\n", (le + ld_str("eigenvalue averages")).c_str());
    int amax = 0;
    for (int k = UEGCCD_CONN_LIMIT; k >= 1; k--)
        if (cavg[k - 1] > 0) {
            amax = k;
            break;
        }
    std::string lc;
    for (int k = 0; k < amax; k++) lc += ld_real(cavg[k]);
    std::fprintf(f59, "%s\n", (lc + ld_str("conn")).c_str());
    for (int t = 0; t < ntw; t++) std::fprintf(f59, "%s\n", (ld_int(t + 1) + ld_real(diff2[t])).c_str());
    std::fprintf(f59, "%s\n",
                 (ld_str("special twist angle found") + ld_real(tw[best][0]) + ld_real(tw[best][1]) +
                  ld_real(tw[best][2]))
                     .c_str());
    std::fprintf(f59, "%s\n", (ld_str("lowest connectivity diff squared") + ld_real(diff2[best])).c_str());
    std::fclose(f59);

    // the special twist with the twist-averaged eigenvalues (Main.f90:233-255)
    if (uegccd_heg_change_twist(h.h, tw[best].data()) || uegccd_heg_set_eigen(h.h, eig_avg.data()))
        return zfail(UEGCCD_ERR_ARG, uegccd_host_last_error());
    uegccd_heg_info(h.h, &info);
    uegccd_heg_system(h.h, &sys);
    Amps x(sys), t(sys);
    for (int ip = 0; ip < std::max(1, in.num_rs_points); ip++)
        if ((rc = mp2_then_cc(in, sys, info.ehf, opt, x, t, ip == 0, &res, sf))) return rc;
    return UEGCCD_OK;
}

int uegccd_zcode(const char *input_path, const char *twists_path, int32_t scheme)
{
    return run_zcode(input_path, twists_path, scheme, true, "fort.60", "fort.82", "fort.61");
}

int uegccd_zcode_fort60(const char *input_path, const char *twists_path, const char *out_path)
{
    return run_zcode(input_path, twists_path, UEGCCD_REPLAY, false, out_path ? out_path : "fort.60", nullptr, nullptr);
}

int uegccd_zcode_host_logs(const char *input_path, const char *twists_path, const char *fort60_path,
                           const char *fort82_path, const char *fort61_path)
{
    return run_zcode(input_path, twists_path, UEGCCD_REPLAY, false, fort60_path ? fort60_path : "fort.60",
                     fort82_path, fort61_path);
}

}  // extern "C"
