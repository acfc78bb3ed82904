// heg_host.cpp -- host side of the drop-in: the Input file reader and the
// plane-wave set-up that the reference's Fortran host runs before it calls the
// hot path.  Restates IO.f90 ReadInput/ParseLine (IO.f90:14-391) and, from
// HEG.f90, init_HEG (16-43), CalcMadelung (89-148), SetupBasis (150-324),
// FcutToBasisFn (326-342), change_rs (494-533), ChangeTwist (551-578), print_HF
// (581-615), print_ex_SF (617-674) and FindTol (1073-1086).  Floating-point expressions keep the
// Fortran evaluation order, so the eigenvalues equal the reference's printout.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/uegccd.h"
#include "../../include/uegccd_host.h"
#include "heg_device.h"
#include "listdir.h"

namespace {

constexpr double kPi = 3.1415926535897932384626433833;  // Constants.f90:7
thread_local std::string g_host_error;
thread_local std::string *g_log = nullptr;   // fort.60 lines (set by the ZCode program)
thread_local std::string *g_log82 = nullptr; // fort.82 lines (the exchange structure factors)

using uegccd::ld_int;
using uegccd::ld_real;
using uegccd::ld_str;

void log_line(const std::string &l)
{
    if (g_log) *g_log += l + "\n";
}

int herr(int code, const std::string &m)
{
    g_host_error = m;
    return code;
}

struct G1Entry {
    int n[3];
    int n2;
    double nt[3];
    double nt2;
};

}  // namespace

struct UegccdHeg {
    UegccdInput in;
    int nel = 0, nocc = 0, nao = 0, cell = 0, maxkpoint = 0, coren = 0;
    double exchangefactor = 1.0;
    double L = 0, rS = 1.0, omega = 0, madelung = 0, density = 0, kf = 0, screening = 0;
    double ntwist[3] = {0, 0, 0};
    double ehf = 0, xhf = 0;
    std::vector<double> kvec;   // NAO x 3 row-major (p, d)
    std::vector<double> eigen;  // NAO
    std::vector<int32_t> nvec;  // NAO x 3 column-major (Fortran nVec(NAO,3))
};

namespace {

int fcut_to_basis_fn(double fcut, int nel)
{
    int m = (int)(std::pow(fcut, 3.0 / 2.0) * nel / 2);
    double target = std::pow(fcut, 3.0 / 2.0) * nel / 2;
    if (std::fabs(m - target) > std::fabs(m + 1 - target)) m = m + 1;
    return m;
}

// PrintShells (HEG.f90:44-87): cumulative plane-wave counts per |n|^2 < kc^2 (fort.60 only).
void log_shells(int kc)
{
    if (!g_log) return;
    std::vector<int> hist(kc * kc + 1, 0);
    for (int l1 = -kc; l1 <= kc; l1++)
        for (int l2 = -kc; l2 <= kc; l2++)
            for (int l3 = -kc; l3 <= kc; l3++) {
                const int e = l1 * l1 + l2 * l2 + l3 * l3;
                if (e < kc * kc) hist[e]++;
            }
    log_line(ld_str(""));
    log_line(ld_str("--------------------"));
    log_line(ld_str("Basis sets available"));
    log_line(ld_str("--------------------"));
    log_line(ld_str("# ecut k-points M"));
    int culm = 0;
    for (int e = 0; e <= kc * kc; e++)
        if (hist[e] != 0) {
            culm += hist[e];
            log_line(ld_int(e) + ld_int(culm) + ld_int(culm * 2));
        }
}

// CalcMadelung (HEG.f90:89-148).  Each pass of the l4 loop restarts its sum, so the
// result is the l4 = 10 pass; the earlier passes only feed the fort.60 log.
double calc_madelung(double omega, double L)
{
    double kappa = 2.8 / std::pow(omega, 1.0 / 3.0);
    double term2 = -kPi / (std::pow(kappa, 2.0) * std::pow(L, 3.0));
    double term4 = -2.0 * kappa / std::sqrt(kPi);
    if (g_log) {
        log_line(ld_str(""));
        log_line(ld_str("-----------------------------------------------------------"));
        log_line(ld_str("Calculating Madelung Constant - Fraser et al. PRB 53 4 1814"));
        log_line(ld_str("-----------------------------------------------------------"));
        log_line(ld_str("kappa taken from CASINO manual to be") + ld_real(kappa));
        log_line(ld_real(term2) + ld_str("term2"));
        log_line(ld_real(term4) + ld_str("term4"));
    }
    double recip = 0.0;
    for (int l4 = g_log ? 1 : 10; l4 <= 10; l4++) {
        recip = 0.0;
        for (int l1 = -l4; l1 <= l4; l1++)
            for (int l2 = -l4; l2 <= l4; l2++)
                for (int l3 = -l4; l3 <= l4; l3++) {
                    int n2 = l1 * l1 + l2 * l2 + l3 * l3;
                    if (n2 == 0) continue;
                    double k2 = (1.0 / std::pow(L, 2.0)) * (double)n2;
                    double ek2 = (1.0 / std::pow(L, 3.0)) * (1.0 / (kPi * k2)) *
                                 std::exp(-(std::pow(kPi, 2.0) * k2) / std::pow(kappa, 2.0));
                    recip = recip + ek2;
                }
        log_line(ld_int(l4) + ld_real(recip));
    }
    log_line(ld_str("reciprocal space") + ld_real(recip));
    double real = 0.0;
    for (int l4 = g_log ? 1 : 10; l4 <= 10; l4++) {
        real = 0.0;
        for (int l1 = -l4; l1 <= l4; l1++)
            for (int l2 = -l4; l2 <= l4; l2++)
                for (int l3 = -l4; l3 <= l4; l3++) {
                    double modr = L * std::sqrt((double)(l1 * l1 + l2 * l2 + l3 * l3));
                    if (modr != 0.0) real = real + std::erfc(kappa * modr) / modr;
                }
        log_line(ld_int(l4) + ld_real(real));
    }
    log_line(ld_str("real space") + ld_real(real));
    return real + recip + term2 + term4;
}

void form_eigen(UegccdHeg &h)
{
    for (int p = 0; p < h.nao; p++) {
        const double *k = &h.kvec[3 * p];
        double e = 0.5 * (k[0] * k[0] + k[1] * k[1] + k[2] * k[2]);
        for (int q = 0; q < h.nel / 2; q++) {
            if (q != p) {
                const double *kq = &h.kvec[3 * q];
                double q1 = k[0] - kq[0], q2 = k[1] - kq[1], q3 = k[2] - kq[2];
                e = e - (1.0 / h.omega) * (4.0 * kPi / (q1 * q1 + q2 * q2 + q3 * q3)) * h.exchangefactor;
            } else {
                e = e + h.madelung - h.in.gap;
            }
        }
        h.eigen[p] = e;
        log_line(ld_int(p + 1) + ld_int(h.nvec[p]) + ld_int(h.nvec[p + (size_t)h.nao]) +
                 ld_int(h.nvec[p + 2 * (size_t)h.nao]) + ld_real(e));
    }
}

// print_ex_SF (HEG.f90:617-674): ordered pairs of occupied orbitals l1 != l2 counted on
// the grid of q = n_l1 - n_l2 (side 2*maxq+1, column-major from -maxq), with the last
// pair's (1/Omega) 4 pi/|k_l1 - k_l2|^2 at each q.
int exchange_sf(const UegccdHeg &h, std::vector<int32_t> *ex_sf, std::vector<double> *ex_v)
{
    const int no = h.nel / 2;
    auto n = [&](int p, int d) { return h.nvec[p + (size_t)h.nao * d]; };
    int qmax[3] = {0, 0, 0};
    for (int l1 = 0; l1 < no; l1++)
        for (int l2 = 0; l2 < no; l2++)
            if (l2 != l1)
                for (int d = 0; d < 3; d++) qmax[d] = std::max(qmax[d], std::abs(n(l1, d) - n(l2, d)));
    const int maxq = std::max(qmax[0], std::max(qmax[1], qmax[2])) + 1;
    if (!ex_sf && !ex_v) return maxq;
    const size_t W = 2 * maxq + 1;
    if (ex_sf) ex_sf->assign(W * W * W, 0);
    if (ex_v) ex_v->assign(W * W * W, 0.0);
    for (int l1 = 0; l1 < no; l1++)
        for (int l2 = 0; l2 < no; l2++) {
            if (l2 == l1) continue;
            const size_t g = (size_t)(n(l1, 0) - n(l2, 0) + maxq) +
                             W * ((size_t)(n(l1, 1) - n(l2, 1) + maxq) + W * (size_t)(n(l1, 2) - n(l2, 2) + maxq));
            if (ex_sf) (*ex_sf)[g] += 1;
            const double *k = &h.kvec[3 * l1], *kq = &h.kvec[3 * l2];
            const double q1 = k[0] - kq[0], q2 = k[1] - kq[1], q3 = k[2] - kq[2];
            if (ex_v) (*ex_v)[g] = (1.0 / h.omega) * (4.0 * kPi / (q1 * q1 + q2 * q2 + q3 * q3));
        }
    return maxq;
}

// the fort.82 block of one print_ex_SF call
void log_exchange_sf(const UegccdHeg &h)
{
    if (!g_log82) return;
    std::vector<int32_t> cnt;
    std::vector<double> v;
    const int m = exchange_sf(h, &cnt, &v);
    const int W = 2 * m + 1;
    std::string &o = *g_log82;
    o += ld_str("--------") + "\n" + ld_str("Starting a new structure factor") + "\n" + ld_str("--------") + "\n";
    for (int x = -m; x <= m; x++)
        for (int y = -m; y <= m; y++)
            for (int z = -m; z <= m; z++) {
                const size_t g = (size_t)(x + m) + (size_t)W * ((size_t)(y + m) + (size_t)W * (size_t)(z + m));
                if (cnt[g] > 0)  // ExSf > 1e-10
                    o += ld_int(x) + ld_int(y) + ld_int(z) + ld_int(cnt[g]) + ld_real(v[g]) + "\n";
            }
}

void hf_energy(UegccdHeg &h)
{
    double ehf = 0.0, xhf = 0.0;
    for (int p = 0; p < h.nel / 2; p++) {
        const double *k = &h.kvec[3 * p];
        ehf = ehf + 0.5 * (k[0] * k[0] + k[1] * k[1] + k[2] * k[2]);
        for (int q = 0; q < h.nel / 2; q++) {
            if (q == p) continue;
            const double *kq = &h.kvec[3 * q];
            double q1 = k[0] - kq[0], q2 = k[1] - kq[1], q3 = k[2] - kq[2];
            double qq = q1 * q1 + q2 * q2 + q3 * q3;
            ehf = ehf - 0.5 * (1.0 / h.omega) * (4.0 * kPi / qq);
            xhf = xhf - 0.5 * (1.0 / h.omega) * (4.0 * kPi / qq);
        }
    }
    ehf = ehf * 2.0;
    h.xhf = xhf * 2.0;
    // print_HF (HEG.f90:605-610)
    if (g_log) {
        log_line(ld_str("L:") + ld_real(h.L));
        log_line(ld_str("Omega:") + ld_real(h.omega));
        log_line(ld_str("cell:") + ld_int(h.cell));
        log_line(ld_str("HF energy:") + ld_real(ehf / h.nel + h.madelung / 2.0));
        log_line(ld_str("Exchange energy:") + ld_real(h.xhf / h.nel + h.madelung / 2.0));
        log_line(ld_str("Madelung:") + ld_real(h.madelung));
    }
    h.ehf = ehf + h.madelung * 0.5 * h.nel;
    log_exchange_sf(h);
}

int setup_basis(UegccdHeg &h)
{
    const int cell = h.cell;
    log_line(ld_str(""));
    log_line(ld_str("-----------------------------------------------------------"));
    log_line(ld_str("Setting up HEG basis set"));
    log_line(ld_str("-----------------------------------------------------------"));
    log_line(ld_str("G1 memory allocated for") + ld_int((2 * cell + 1) * (2 * cell + 1) * (2 * cell + 1)) +
             ld_str("basis functions"));
    std::vector<G1Entry> g1;
    g1.reserve((size_t)(2 * cell + 1) * (2 * cell + 1) * (2 * cell + 1));
    for (int l1 = -cell; l1 <= cell; l1++)
        for (int l2 = -cell; l2 <= cell; l2++)
            for (int l3 = -cell; l3 <= cell; l3++) {
                G1Entry g;
                g.n[0] = l1; g.n[1] = l2; g.n[2] = l3;
                g.n2 = l1 * l1 + l2 * l2 + l3 * l3;
                g.nt[0] = l1 + h.ntwist[0];
                g.nt[1] = l2 + h.ntwist[1];
                g.nt[2] = l3 + h.ntwist[2];
                g.nt2 = g.nt[0] * g.nt[0] + g.nt[1] * g.nt[1] + g.nt[2] * g.nt[2];
                if (g.n2 <= h.maxkpoint) g1.push_back(g);
            }
    int nbasis = (int)g1.size();
    log_line(ld_str("Actual basis set size") + ld_int(nbasis));
    // stable ascending sort by twisted |n+k|^2 (the reference's bubble sort)
    for (;;) {
        bool swapped = false;
        for (int l1 = 1; l1 < nbasis; l1++)
            if (g1[l1].nt2 < g1[l1 - 1].nt2) {
                std::swap(g1[l1], g1[l1 - 1]);
                swapped = true;
            }
        if (!swapped) break;
    }
    int mfcut = (int)(std::pow(h.in.fcut, 3.0 / 2.0) * h.nel / 2);
    double mtarget = std::pow(h.in.fcut, 3.0 / 2.0) * h.nel / 2;
    if (std::fabs(mfcut - mtarget) > std::fabs(mfcut + 1 - mtarget)) mfcut = mfcut + 1;
    if (mfcut < nbasis) nbasis = mfcut;
    log_line(ld_str("Basis set size after fcut") + ld_int(nbasis));
    int mcore = fcut_to_basis_fn(h.in.corefcut, h.nel);
    if ((h.in.corefcut - 1.0) < 1e-6 && mcore != h.nel / 2)
        return herr(UEGCCD_ERR_ARG, "ERROR in setup_basis: corefcut is less than 1 rather than equal to 1");
    nbasis = nbasis - mcore + h.nel / 2;
    log_line(ld_str("Basis set size after corefcut") + ld_int(nbasis));
    if (nbasis <= h.nel / 2) return herr(UEGCCD_ERR_ARG, "basis has no virtual orbitals");
    h.nao = nbasis;
    h.kvec.assign((size_t)nbasis * 3, 0.0);
    h.eigen.assign(nbasis, 0.0);
    h.nvec.assign((size_t)nbasis * 3, 0);
    for (int p = 0; p < nbasis; p++) {
        int off = (p + 1 > h.nel / 2) ? mcore - h.nel / 2 : 0;
        const G1Entry &g = g1[p + off];
        for (int d = 0; d < 3; d++) {
            h.kvec[3 * p + d] = g.nt[d] * (2.0 * kPi / h.L);
            h.nvec[p + (size_t)nbasis * d] = g.n[d];
        }
    }
    form_eigen(h);
    hf_energy(h);
    return 0;
}

bool parse_bool(const std::string &v)
{
    std::string s;
    for (char c : v)
        if (!isspace((unsigned char)c)) s += (char)toupper((unsigned char)c);
    if (!s.empty() && s[0] == '.') s = s.substr(1);
    return !s.empty() && s[0] == 'T';
}

}  // namespace

namespace uegccd {
void heg_log_to(std::string *sink) { g_log = sink; }
void heg_sf_log_to(std::string *sink) { g_log82 = sink; }
}  // namespace uegccd

namespace uegccd {
// What the device set-up of many twists needs from the host state (heg_device.cu): the
// untwisted candidates of SetupBasis in its loop order, the basis size after fcut and
// corefcut, and the scalars of form_eigen / hf_energy at the current rS.
int heg_twist_setup(const UegccdHeg *h, HegTwistSetup *out)
{
    if (!h || !out) return herr(UEGCCD_ERR_ARG, "null argument");
    const int cell = h->cell;
    out->cand.clear();
    for (int l1 = -cell; l1 <= cell; l1++)
        for (int l2 = -cell; l2 <= cell; l2++)
            for (int l3 = -cell; l3 <= cell; l3++)
                if (l1 * l1 + l2 * l2 + l3 * l3 <= h->maxkpoint) out->cand.push_back({l1, l2, l3});
    const int nbasis0 = (int)out->cand.size();
    int mfcut = (int)(std::pow(h->in.fcut, 3.0 / 2.0) * h->nel / 2);
    double mtarget = std::pow(h->in.fcut, 3.0 / 2.0) * h->nel / 2;
    if (std::fabs(mfcut - mtarget) > std::fabs(mfcut + 1 - mtarget)) mfcut = mfcut + 1;
    const int nbasis = std::min(mfcut, nbasis0);
    const int mcore = fcut_to_basis_fn(h->in.corefcut, h->nel);
    out->nao = nbasis - mcore + h->nel / 2;
    out->mcore = mcore;
    out->nel = h->nel;
    if (out->nao != h->nao) return herr(UEGCCD_ERR_ARG, "basis size differs from the set-up's");
    out->kscale = 2.0 * kPi / h->L;
    out->inv_omega = 1.0 / h->omega;
    out->madelung = h->madelung;
    out->gap = h->in.gap;
    out->exchangefactor = h->exchangefactor;
    out->L = h->L;
    return 0;
}
}  // namespace uegccd

extern "C" {

const char *uegccd_host_last_error(void) { return g_host_error.c_str(); }

void uegccd_default_input(UegccdInput *in)
{
    std::memset(in, 0, sizeof(*in));
    in->nelectron = 14;
    in->maxkpoint = 2;
    in->rsmin = in->rsmax = 1.0;
    in->num_rs_points = 1;
    in->do_ring = in->do_xring = in->do_ladder = in->do_mosaic = 1;
    in->madelung_factor = 1.0;
    in->fcut = 10.0;
    in->corefcut = 1.0;
    in->gapii = -0.01;
    in->do_single_calc = 1;
    // keys newer than an Input file take the behaviour of the code that predates them:
    // without DoSkipTA the twist average always ran
    in->do_skip_ta = 0;
}

// ReadInput (IO.f90:14-348): "Key: Value" lines, '!' comments; every key of the
// reference's list must be set exactly once (IO.f90:329-335); unknown keys stop.
int uegccd_read_input(const char *path, int32_t require_all, UegccdInput *in)
{
    static const char *kNames[] = {
        "# Electrons", "Momentum Cutoff", "rSMin", "rSMax", "# rS Points", "Safe ERI", "Do Rings", "Do XRings",
        "Do Ladders", "Do Mosaics", "Rings Range", "XRings Range", "Ladders Range", "Mosaics Range",
        "DriverDir Range", "DriverEx Range", "Energy Range", "LinRings Range", "QuadRings Range", "DRings Range",
        "ExRings Range", "LinLadd Range", "QuadLadd Range", "DLadders Range", "ExLadders Range", "CoreFactor",
        "TACalcN", "DoCalcTACCD", "DodRPASOSEX", "DoTruncCoulombHF", "DoTruncCoulombAll", "DoKS", "MadelungFactor",
        "DoSingleCalc", "Gap", "fcut", "corefcut", "fcut2ecut", "GapII", "DoSFCalcMP2", "DoSFCalcCCD", "DoSkipTA",
        "DoOnlyMP2Grid", "EndInput"};
    const int nparams = (int)(sizeof(kNames) / sizeof(kNames[0]));
    if (!in || !path) return herr(UEGCCD_ERR_ARG, "null argument");
    uegccd_default_input(in);
    std::ifstream f(path);
    if (!f) return herr(UEGCCD_ERR_ARG, "No Input file");
    std::map<std::string, int> count;
    std::string line;
    int lineno = 0;
    int fcut2ecut = 0;
    std::map<std::string, int> range;   // the "... Range" values read (the others are 0)
    while (std::getline(f, line)) {
        lineno++;
        size_t c = line.find('!');
        if (c != std::string::npos) line = line.substr(0, c);
        for (char &ch : line)
            if ((unsigned char)ch <= 31) ch = ' ';
        if (line.find_first_not_of(' ') == std::string::npos) continue;
        size_t colon = line.find(':');
        std::string key = colon == std::string::npos ? line : line.substr(0, colon);
        std::string val = colon == std::string::npos ? "" : line.substr(colon + 1);
        size_t a = key.find_first_not_of(' '), b = key.find_last_not_of(' ');
        key = (a == std::string::npos) ? "" : key.substr(a, b - a + 1);
        std::istringstream vs(val);
        count[key]++;
        if (key == "# Electrons") {
            vs >> in->nelectron;
            if (in->nelectron < 0) return herr(UEGCCD_ERR_ARG, "Must have positive number of electrons");
            if (in->nelectron % 2 == 1) return herr(UEGCCD_ERR_ARG, "Must have closed shell");
        } else if (key == "Momentum Cutoff") vs >> in->maxkpoint;
        else if (key == "rSMin") vs >> in->rsmin;
        else if (key == "rSMax") vs >> in->rsmax;
        else if (key == "# rS Points") {
            vs >> in->num_rs_points;
            if (in->num_rs_points > 1) return herr(UEGCCD_ERR_ARG, "Cannot have more than one rs point");
        } else if (key == "Safe ERI") in->safe_eri = parse_bool(val);
        else if (key == "Do Rings") in->do_ring = parse_bool(val);
        else if (key == "Do XRings") in->do_xring = parse_bool(val);
        else if (key == "Do Ladders") in->do_ladder = parse_bool(val);
        else if (key == "Do Mosaics") in->do_mosaic = parse_bool(val);
        else if (key.size() > 6 && key.compare(key.size() - 5, 5, "Range") == 0) {
            int r = 0;
            vs >> r;
            in->range_flags += std::abs(r);
            range[key] = r;
        } else if (key == "NTwist") vs >> in->ntwist[0] >> in->ntwist[1] >> in->ntwist[2];
        else if (key == "CoreFactor") {
            vs >> in->core_factor;
            in->core_factor_set = 1;
        }
        else if (key == "TACalcN") vs >> in->tacalcn;
        else if (key == "DoCalcTACCD") in->do_calc_ta_ccd = parse_bool(val);
        else if (key == "DodRPASOSEX") in->do_drpa_sosex = parse_bool(val);
        else if (key == "DoTruncCoulombHF") {
            if (parse_bool(val)) return herr(UEGCCD_ERR_ARG, "Not Implemented");
        } else if (key == "DoTruncCoulombAll") {
            if (parse_bool(val)) return herr(UEGCCD_ERR_ARG, "Not Implemented");
        } else if (key == "DoKS") in->do_ks = parse_bool(val);
        else if (key == "MadelungFactor") vs >> in->madelung_factor;
        else if (key == "DoSingleCalc") in->do_single_calc = parse_bool(val);
        else if (key == "DoSFCalcMP2") in->do_sf_calc_mp2 = parse_bool(val);
        else if (key == "DoSFCalcCCD") in->do_sf_calc_ccd = parse_bool(val);
        else if (key == "DoOnlyMP2Grid") in->do_only_mp2_grid = parse_bool(val);
        else if (key == "DoSkipTA") in->do_skip_ta = parse_bool(val);
        else if (key == "Gap") vs >> in->gap;
        else if (key == "fcut") vs >> in->fcut;
        else if (key == "corefcut") vs >> in->corefcut;
        else if (key == "fcut2ecut") fcut2ecut = parse_bool(val);
        else if (key == "GapII") vs >> in->gapii;
        else if (key == "EndInput") {
            if (!parse_bool(val)) return herr(UEGCCD_ERR_ARG, "EndInput must be T");
        } else {
            return herr(UEGCCD_ERR_ARG, "Error: Line number " + std::to_string(lineno) + " of Input not recognized");
        }
    }
    in->fcut2ecut = fcut2ecut;
    {   // the fifteen range flags (UegccdRangeTerms keeps the Input's order), and one value for
        // all of them, or -1
        int v = 0;
        bool first = true, same = true;
        int32_t *terms = &in->range_terms.ring;
        for (int k = 10; k < 25; k++) {   // kNames[10..24]: the "... Range" keys
            const auto it = range.find(kNames[k]);
            const int r = it == range.end() ? 0 : it->second;
            terms[k - 10] = r;
            if (first) v = r;
            else if (r != v) same = false;
            first = false;
        }
        in->range_uniform = same ? v : -1;
    }
    if (require_all) {
        for (int k = 2; k < nparams; k++)
            if (count[kNames[k]] == 0) return herr(UEGCCD_ERR_ARG, std::string("Error: Parameter ") + kNames[k] + " not set.");
        for (auto &kv : count)
            if (kv.second > 1) return herr(UEGCCD_ERR_ARG, "Error: Parameter " + kv.first + " multiply set.");
    }
    return 0;
}

int uegccd_heg_create(const UegccdInput *in, UegccdHeg **out)
{
    if (!in || !out) return herr(UEGCCD_ERR_ARG, "null argument");
    *out = nullptr;
    auto *h = new UegccdHeg;
    h->in = *in;
    h->nel = in->nelectron;
    h->nocc = in->nelectron / 2;
    h->maxkpoint = in->maxkpoint;
    h->coren = (int)(in->nelectron / 2 * in->core_factor);
    h->exchangefactor = in->do_ks ? 0.0 : 1.0;
    if (in->fcut2ecut) {  // IO.f90:291-300
        double nfermi = std::pow((double)in->nelectron, 2.0 / 3.0) / 4.0;
        double mult = in->fcut < 2.0 ? 2.0 : in->fcut;
        h->maxkpoint = (int)(nfermi * mult * 2.0);
        if (nfermi < 10) h->maxkpoint = (int)(10 * mult * 2.0);
    }
    for (int d = 0; d < 3; d++) h->ntwist[d] = in->ntwist[d];
    // init_HEG at rS = 1
    log_shells(10);
    h->rS = 1.0;
    h->L = h->rS * std::pow(4.0 / 3.0 * kPi * h->nel, 1.0 / 3.0);
    h->omega = h->L * h->L * h->L;
    h->madelung = calc_madelung(h->omega, h->L) * in->madelung_factor;
    h->cell = (int)std::sqrt((double)h->maxkpoint) + 3;
    log_line(ld_str("Madelung constant calculated as") + ld_real(h->madelung));
    int rc = setup_basis(*h);
    if (rc) { delete h; return rc; }
    // change_rs to rSMin (Main.f90:78-79)
    double rescale = in->rsmin / h->rS;
    h->L = h->L * rescale;
    h->omega = h->omega * std::pow(rescale, 3.0);
    for (double &k : h->kvec) k = k * (1.0 / rescale);
    h->madelung = calc_madelung(h->omega, h->L) * in->madelung_factor;
    form_eigen(*h);
    hf_energy(*h);
    *out = h;
    return 0;
}

void uegccd_heg_destroy(UegccdHeg *h) { delete h; }

int uegccd_heg_change_twist(UegccdHeg *h, const double twist[3])
{
    if (!h || !twist) return herr(UEGCCD_ERR_ARG, "null argument");
    int nao = h->nao;
    if (g_log) {  // ChangeTwist (HEG.f90:565)
        std::string l = ld_str("changing twist angle from");
        for (int d = 0; d < 3; d++) l += ld_real(h->ntwist[d]);
        l += ld_str("to");
        for (int d = 0; d < 3; d++) l += ld_real(twist[d]);
        log_line(l);
    }
    for (int d = 0; d < 3; d++) h->ntwist[d] = twist[d];
    int rc = setup_basis(*h);
    if (rc) return rc;
    if (h->nao != nao) return herr(UEGCCD_ERR_ARG, "basis size changed with the twist");
    return 0;
}

int uegccd_heg_set_eigen(UegccdHeg *h, const double *eigen)
{
    if (!h || !eigen) return herr(UEGCCD_ERR_ARG, "null argument");
    h->eigen.assign(eigen, eigen + h->nao);
    return 0;
}

int uegccd_heg_system(const UegccdHeg *h, UegccdSystem *sys)
{
    if (!h || !sys) return herr(UEGCCD_ERR_ARG, "null argument");
    sys->nocc = h->nocc;
    sys->nao = h->nao;
    sys->L = h->L;
    sys->madelung = h->madelung;
    sys->eigen = h->eigen.data();
    sys->nvec = h->nvec.data();
    return 0;
}

int uegccd_heg_info(const UegccdHeg *h, UegccdHegInfo *info)
{
    if (!h || !info) return herr(UEGCCD_ERR_ARG, "null argument");
    info->nocc = h->nocc;
    info->nao = h->nao;
    info->maxkpoint = h->maxkpoint;
    info->cell = h->cell;
    info->core_n = h->coren;
    info->L = h->L;
    info->omega = h->omega;
    info->madelung = h->madelung;
    info->ehf = h->ehf;
    for (int d = 0; d < 3; d++) info->twist[d] = h->ntwist[d];
    return 0;
}

// FindTol (HEG.f90:1073-1086), fed HEGData%rS as the reference does (always 1).
int uegccd_heg_exchange_sf(const UegccdHeg *h, int32_t *maxq, int32_t *ex_sf, double *ex_v)
{
    if (!h || !maxq) return herr(UEGCCD_ERR_ARG, "null argument");
    std::vector<int32_t> c;
    std::vector<double> v;
    *maxq = exchange_sf(*h, ex_sf ? &c : nullptr, ex_v ? &v : nullptr);
    if (ex_sf) std::copy(c.begin(), c.end(), ex_sf);
    if (ex_v) std::copy(v.begin(), v.end(), ex_v);
    return UEGCCD_OK;
}

void uegccd_find_tol(double rs, double *tolmax, double *failratio, double *denomfactor)
{
    *tolmax = 1.0e-8;
    *failratio = 100;
    if (rs > 5.1) *tolmax = 1.0e-6;
    if (rs > 5.1) *denomfactor = 5.0;
    if (rs > 9.9) *tolmax = 1.0e-5;
    if (rs > 80.0) *tolmax = 1.0e-3;
    if (rs < 0.95) *failratio = 1e6;
}

}  // extern "C"
