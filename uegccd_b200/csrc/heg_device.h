// heg_device.h -- the host state the device set-up of many twists reads (heg_host.cpp fills
// it from a UegccdHeg; heg_device.cu runs the set-up).
#pragma once
#include <array>
#include <vector>

struct UegccdHeg;

namespace uegccd {

struct HegTwistSetup {
    std::vector<std::array<int, 3>> cand;   // untwisted n with |n|^2 <= MaxKPoint, SetupBasis loop order
    int nao = 0, mcore = 0, nel = 0;        // basis after fcut and corefcut; its core offset; N
    double kscale = 0;                      // 2 pi / L
    double inv_omega = 0;                   // 1 / Omega
    double madelung = 0, gap = 0, exchangefactor = 1.0, L = 0;
};

int heg_twist_setup(const UegccdHeg *h, HegTwistSetup *out);

}  // namespace uegccd
