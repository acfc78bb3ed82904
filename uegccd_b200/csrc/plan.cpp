// plan.cpp -- momentum-block plan: replaces the FindIndex lookups of every hot
// loop (HEG.f90:357-404) by tables built once per system.
//
// FindIndex(M,N,L) returns the basis orbital at n_M + n_N - n_L (0 when that
// vector lies outside the basis).  An amplitude (i,j,a) is momentum-allowed when
// b = FindIndex(i,j,a) is a virtual (b > NOcc), the test every loop of MP2.f90,
// CCD.f90 and dRPA.f90 makes before touching T(i,j,a).  The blocks group the
// allowed amplitudes by K = n_i + n_j.
#include "plan.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <unordered_map>

namespace uegccd {

namespace {
constexpr double kPi = 3.1415926535897932384626433833;  // Constants.f90:7

struct VecHash {
    size_t operator()(const std::array<int, 3> &v) const {
        return (size_t)((v[0] + 512) * 1048576LL + (v[1] + 512) * 1024LL + (v[2] + 512));
    }
};
}  // namespace

double coulomb_v(double L, double madelung, int q2)
{
    if (q2 == 0) return -madelung;
    return 1.0 / (L * kPi * (double)q2);
}

std::string build_solve_plan(const SystemHost &sys, SolvePlan &p)
{
    const int O = sys.O, M = sys.M, V = M - O;
    if (O <= 0 || V <= 0) return "need NOcc > 0 and NAO > NOcc";
    if (M > 32767) return "NAO too large for 16-bit orbital indices";
    if ((int)sys.n.size() != M || (int)sys.eigen.size() != M) return "nvec/eigen size mismatch";
    p = SolvePlan();
    p.O = O; p.V = V; p.M = M;

    std::unordered_map<std::array<int, 3>, int, VecHash> orb;
    orb.reserve((size_t)M * 2);
    int q2max = 0;
    for (int q = 0; q < M; q++) {
        if (!orb.emplace(sys.n[q], q).second) return "duplicate plane-wave vector in nVec";
    }
    for (int x = 0; x < M; x++)
        for (int y = 0; y < M; y++) {
            int d0 = sys.n[x][0] - sys.n[y][0], d1 = sys.n[x][1] - sys.n[y][1], d2 = sys.n[x][2] - sys.n[y][2];
            q2max = std::max(q2max, d0 * d0 + d1 * d1 + d2 * d2);
        }
    p.q2max = q2max;
    p.vtab.resize((size_t)q2max + 1);
    for (int q2 = 0; q2 <= q2max; q2++) p.vtab[q2] = coulomb_v(sys.L, sys.madelung, q2);

    auto partner = [&](int i, int j, int a) -> int {
        std::array<int, 3> t{sys.n[i][0] + sys.n[j][0] - sys.n[a][0], sys.n[i][1] + sys.n[j][1] - sys.n[a][1],
                             sys.n[i][2] + sys.n[j][2] - sys.n[a][2]};
        auto it = orb.find(t);
        return it == orb.end() ? -1 : it->second;
    };

    // Group ordered occupied pairs by K, keeping first-appearance order (i major).
    std::map<std::array<int, 3>, int> kindex;
    std::vector<std::vector<std::pair<int, int>>> kpairs;
    std::vector<std::array<int, 3>> kvecs;
    for (int i = 0; i < O; i++)
        for (int j = 0; j < O; j++) {
            std::array<int, 3> K{sys.n[i][0] + sys.n[j][0], sys.n[i][1] + sys.n[j][1], sys.n[i][2] + sys.n[j][2]};
            auto it = kindex.find(K);
            int id;
            if (it == kindex.end()) {
                id = (int)kpairs.size();
                kindex.emplace(K, id);
                kpairs.emplace_back();
                kvecs.push_back(K);
            } else {
                id = it->second;
            }
            kpairs[id].emplace_back(i, j);
        }
    p.pos.assign((size_t)O * O * V, -1);
    int64_t t0 = 0;
    for (size_t k = 0; k < kpairs.size(); k++) {
        // virtual columns of block K: a virtual whose partner b = K - a is a virtual
        std::vector<int> cols;
        int i0 = kpairs[k][0].first, j0 = kpairs[k][0].second;
        for (int a = O; a < M; a++) {
            int b = partner(i0, j0, a);
            if (b >= O) cols.push_back(a);
        }
        if (cols.empty()) continue;
        SolvePlan::Block blk;
        blk.o = (int)kpairs[k].size();
        blk.v = (int)cols.size();
        blk.pair0 = (int)p.pair_i.size();
        blk.vir0 = (int)p.vir.size();
        blk.t0 = t0;
        for (auto &pr : kpairs[k]) {
            p.pair_i.push_back((int16_t)pr.first);
            p.pair_j.push_back((int16_t)pr.second);
        }
        for (int a : cols) p.vir.push_back((int16_t)a);
        for (int r = 0; r < blk.o; r++) {
            int i = kpairs[k][r].first, j = kpairs[k][r].second;
            for (int c = 0; c < blk.v; c++) {
                int a = cols[c];
                int b = partner(i, j, a);
                int64_t idx = t0 + (int64_t)r * blk.v + c;
                p.pos[((size_t)i * O + j) * V + (a - O)] = (int32_t)idx;
                p.amps.push_back(AmpInfo{(int16_t)i, (int16_t)j, (int16_t)a, (int16_t)b});
            }
        }
        t0 += (int64_t)blk.o * blk.v;
        p.blocks.push_back(blk);
    }
    p.namp = t0;
    if (p.namp >= (int64_t)1 << 31) return "too many amplitudes for 32-bit packed indices";
    p.ring_entries = (int64_t)O * V * O;

    // particle-hole rows (i,x) grouped by their momentum Q = n_x - n_i
    std::map<std::array<int, 3>, std::vector<std::pair<int, int>>> qrows;
    for (int i = 0; i < O; i++)
        for (int x = O; x < M; x++) {
            std::array<int, 3> Q{sys.n[x][0] - sys.n[i][0], sys.n[x][1] - sys.n[i][1], sys.n[x][2] - sys.n[i][2]};
            qrows[Q].emplace_back(i, x);
        }
    p.phrow_of.assign((size_t)O * V, -1);
    std::map<std::array<int, 3>, int> gidx;
    for (auto &kv : qrows) {
        SolvePlan::PhGroup g{(int)p.ph_i.size(), (int)kv.second.size(), -1};
        gidx[kv.first] = (int)p.groups.size();
        p.groups.push_back(g);
        for (auto &r : kv.second) {
            p.phrow_of[(size_t)r.first * V + (r.second - O)] = (int32_t)p.ph_i.size();
            p.ph_i.push_back((int16_t)r.first);
            p.ph_x.push_back((int16_t)r.second);
        }
    }
    for (auto &kv : qrows) {
        std::array<int, 3> mQ{-kv.first[0], -kv.first[1], -kv.first[2]};
        auto it = gidx.find(mQ);
        if (it != gidx.end()) p.groups[gidx[kv.first]].partner = it->second;
    }
    return "";
}

}  // namespace uegccd
