// listdir.h -- gfortran list-directed output (write(u,*)) of the items that the
// reference's fort.58, fort.59, fort.60 and fort.80-82 hold.
//   REAL(8):   a blank, then 17 significant digits in a 25-wide G field: F form
//              (20 wide, then 5 blanks) for 0.1 <= |x| < 1e17, else E form with a
//              three-digit exponent.
//   INTEGER:   a blank, then I11.
//   CHARACTER: a blank, then the text.
#pragma once
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

namespace uegccd {

inline std::string ld_real(double x)
{
    char m[64], f[96], num[64];
    if (!std::isfinite(x)) {
        std::snprintf(f, sizeof f, " %20s     ", std::isnan(x) ? "NaN" : (x > 0 ? "Infinity" : "-Infinity"));
        return f;
    }
    int ex = 0;
    if (x != 0.0) {
        std::snprintf(m, sizeof m, "%.16e", x);  // 17 significant digits, correctly rounded
        ex = std::atoi(std::strchr(m, 'e') + 1);
    }
    if (x == 0.0 || (ex >= -1 && ex < 17)) {
        const int dec = x == 0.0 ? 16 : 16 - ex;
        std::snprintf(num, sizeof num, "%.*f", dec, x);
        std::snprintf(f, sizeof f, " %20s     ", num);
        return f;
    }
    const std::string s(m);
    const size_t e = s.find('e');
    std::snprintf(num, sizeof num, "%sE%c%03d", s.substr(0, e).c_str(), ex < 0 ? '-' : '+', std::abs(ex));
    std::snprintf(f, sizeof f, " %25s", num);
    return f;
}

inline std::string ld_int(long long v)
{
    char f[32];
    std::snprintf(f, sizeof f, " %11lld", v);
    return f;
}

inline std::string ld_str(const char *s) { return std::string(" ") + s; }

// The fort.60 log of the host set-up: lines are appended here while a sink is set
// (per host thread; the ZCode program sets it, nothing else does).
void heg_log_to(std::string *sink);
// The fort.82 lines (exchange structure factor of every print_HF), the same way.
void heg_sf_log_to(std::string *sink);

}  // namespace uegccd
