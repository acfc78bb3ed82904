// two_channel.h -- the two-channel form of the CCD residual and the general-flag dRPA
// residual (two_channel.cu): per-term integral flags and Do Rings without Do XRings.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <vector>

#include "plan.h"
#include "uegccd.h"

namespace uegccd {

// The integral routine SetPointers selects (Main.f90:274-318).
enum TcRoutine { TC_BASE = 0, TC_CORE = 1, TC_GAP = 2, TC_NOCASE = 3, TC_CASED = 4 };

// SetPointers' choice from the fifteen range flags, Safe ERI, CoreN and GapII: CasedERI under
// Safe ERI or with flags, GapII and CoreN all set; NoCaseERI with GapII and CoreN; CoreERI;
// GapERI; BaseERI.
int tc_pick_routine(const UegccdRangeTerms &flags, int safe_eri, int core_n, double gapii);

// Device memory for the two-channel state, carved from the owning context's allocations.
// get returns 0 or an error status; begin/rollback bracket a group of allocations so that a
// failed group leaves nothing behind (the DIIS history steps its depth down on failure).
struct TcAlloc {
    std::function<int(void **, size_t)> get;
    std::function<void()> begin, rollback;
};

// The integral flag of each integral of the terms, after the Max(...) of CCD.f90:620-937.
struct TcFlags {
    int drv_d, drv_x, mosaic, energy;
    int lad_lin_d, lad_lin_x, lad_quad_d, lad_quad_x;
    int ring_lin_d, ring_lin_x, ring_quad_d, ring_quad_x;
    int xr_lin_d, xr_lin_x, xr_quad_d, xr_quad_x;
};

class TwoChannel {
public:
    ~TwoChannel();
    // Device tables of one system (the FindIndex table, plane-wave vectors, work arrays).
    int init(const SystemHost &sys, cudaStream_t stream, TcAlloc alloc);
    // The integrals of every later call: routine (TcRoutine), the fifteen flags, CoreN, GapII
    // and the screening distance of CasedERI.
    int set_integrals(int routine, const UegccdRangeTerms &flags, int core_n, double gapii, double screening);
    // TermsWrapper (CCD.f90:146-181) on both channels, host arrays in the reference layout.
    int ccd_g2(const double *t_abab, const double *t_abba, int mask, double *g_abab, double *g_abba);
    // The dRPA residual (dRPA.f90:339-551) of one channel.
    int drpa_g2(const double *t2, int mask, double *g2);
    // DrvCCD (CCD.f90:18-183) on both channels, or DrvdRPA (dRPA.f90:23-174) on t_abab alone
    // when drpa: iterates in place from the host amplitudes and writes them back.
    int solve(const UegccdOptions &opt, bool drpa, const std::vector<double> &eigen, double *t_aaaa,
              double *t_abab, double *t_abba, UegccdResult &res);
    size_t bytes() const { return bytes_; }

private:
    int O_ = 0, M_ = 0, V_ = 0;
    int64_t n_ = 0;
    int nq_ = 0;
    int core_n_ = 0;
    int routine_ = TC_BASE;
    TcFlags f_{};
    double L_ = 0, madelung_ = 0;
    cudaStream_t st_ = nullptr;
    TcAlloc al_;
    size_t bytes_ = 0;
    // device arrays
    int *F_ = nullptr;          // F[i + O*(j + O*p)] = 1 + FindIndex(i,j,p) (0-based), 0 outside the basis
    int4 *nv_ = nullptr;        // plane-wave vectors
    double *vt_ = nullptr;      // integral tables [core][flag][|q|^2]
    double *eig_ = nullptr;
    double *t_[2] = {nullptr, nullptr}, *g_[2] = {nullptr, nullptr};
    double *jvv_ = nullptr, *joo_ = nullptr;
    double *h_[2] = {nullptr, nullptr};          // hole-hole intermediates, O^3 each
    double *r_[3] = {nullptr, nullptr, nullptr}; // quadratic ring intermediates, O*O*V each
    double *x_[3] = {nullptr, nullptr, nullptr}; // quadratic crossed-ring intermediates
    double *part_ = nullptr, *out_ = nullptr;    // reduction partials and results
    int nblk_ = 0;
    // DIIS history (T after the update, R of the amplitudes before it), per channel
    int ndiis_cap_ = 0;
    double *ht_[2] = {nullptr, nullptr}, *hr_[2] = {nullptr, nullptr};
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    int launches_ = 0;

    int alloc(void **p, size_t bytes);
    int upload_t(const double *h, double *d);
    int residual(bool drpa, int mask);
    int read_out(int k, double *h);
    int diis_alloc(int ndiis);
};

}  // namespace uegccd
