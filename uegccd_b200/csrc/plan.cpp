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

namespace uegccd {

double coulomb_v(double L, double madelung, int q2)
{
    if (q2 == 0) return -madelung;
    return 1.0 / (L * kPi * (double)q2);
}

namespace {
// Dense lookup over integer lattice vectors with components in [-r, r].
struct Lattice {
    int r = 0, side = 0;
    std::vector<int> idx;
    void init(int radius)
    {
        r = radius;
        side = 2 * r + 1;
        idx.assign((size_t)side * side * side, -1);
    }
    bool inside(int x, int y, int z) const { return std::abs(x) <= r && std::abs(y) <= r && std::abs(z) <= r; }
    int get_inside(int x, int y, int z) const { return idx[((size_t)(x + r) * side + (y + r)) * side + (z + r)]; }
    int &at(int x, int y, int z) { return idx[((size_t)(x + r) * side + (y + r)) * side + (z + r)]; }
    int get(int x, int y, int z) const
    {
        return inside(x, y, z) ? idx[((size_t)(x + r) * side + (y + r)) * side + (z + r)] : -1;
    }
};
}  // namespace

std::string build_solve_plan(const SystemHost &sys, SolvePlan &p)
{
    const int O = sys.O, M = sys.M, V = M - O;
    if (O <= 0 || V <= 0) return "need NOcc > 0 and NAO > NOcc";
    if (M > 32767) return "NAO too large for 16-bit orbital indices";
    if ((int)sys.n.size() != M || (int)sys.eigen.size() != M) return "nvec/eigen size mismatch";
    p = SolvePlan();
    p.O = O; p.V = V; p.M = M;

    int nmax = 0;
    for (int q = 0; q < M; q++)
        for (int d = 0; d < 3; d++) nmax = std::max(nmax, std::abs(sys.n[q][d]));
    if (nmax > 200) return "plane-wave vectors out of range";
    // orbital lookup: n -> orbital (the basis, as FindIndex's kPointToBasisFn, HEG.f90:306-316)
    // radius 3 nmax when small: every K - n_a (|K| <= 2 nmax) then lies inside, and the
    // column scan below needs no bounds test
    Lattice orb;
    const bool orb_wide = nmax <= 8;
    orb.init(orb_wide ? 3 * nmax : nmax);
    for (int q = 0; q < M; q++) {
        int &slot = orb.at(sys.n[q][0], sys.n[q][1], sys.n[q][2]);
        if (slot >= 0) return "duplicate plane-wave vector in nVec";
        slot = q;
    }
    // |q|^2 range of orbital differences: components of n_x - n_y are within [-2 nmax, 2 nmax]
    int q2max = 0;
    {
        // component arrays: the inner loop vectorises
        std::vector<int> nx(M), ny(M), nz(M);
        for (int q = 0; q < M; q++) {
            nx[q] = sys.n[q][0];
            ny[q] = sys.n[q][1];
            nz[q] = sys.n[q][2];
        }
        for (int x = 0; x < M; x++) {
            const int ax = nx[x], ay = ny[x], az = nz[x];
            int m = 0;
            for (int y = x + 1; y < M; y++) {
                const int d0 = ax - nx[y], d1 = ay - ny[y], d2 = az - nz[y];
                m = std::max(m, d0 * d0 + d1 * d1 + d2 * d2);
            }
            q2max = std::max(q2max, m);
        }
    }
    p.q2max = q2max;
    p.vtab.resize((size_t)q2max + 1);
    for (int q2 = 0; q2 <= q2max; q2++) p.vtab[q2] = coulomb_v(sys.L, sys.madelung, q2);

    // Group ordered occupied pairs by K = n_i + n_j, first-appearance order (i major).
    Lattice kid;
    kid.init(2 * nmax);
    std::vector<std::vector<std::pair<int, int>>> kpairs;
    std::vector<std::array<int, 3>> kvecs;
    for (int i = 0; i < O; i++)
        for (int j = 0; j < O; j++) {
            std::array<int, 3> K{sys.n[i][0] + sys.n[j][0], sys.n[i][1] + sys.n[j][1], sys.n[i][2] + sys.n[j][2]};
            int &id = kid.at(K[0], K[1], K[2]);
            if (id < 0) {
                id = (int)kpairs.size();
                kpairs.emplace_back();
                kvecs.push_back(K);
            }
            kpairs[id].emplace_back(i, j);
        }
    // the position map, amplitude list and partner indices are built on the device from
    // the blocks (k_block_tables); the host keeps only the block structure
    int64_t t0 = 0;
    std::vector<int> cols, partner_of_col, col_of(M, -1);
    for (size_t k = 0; k < kpairs.size(); k++) {
        // virtual columns of block K: a virtual whose partner b = K - a is a virtual.  Order:
        // the columns a < b, the column a = b if K = 2 n_a, then the partners b of the first
        // ones in the same order, so column c < nvd has its partner at c + nvd + sd
        cols.clear();
        partner_of_col.clear();
        const auto &K = kvecs[k];
        int nvd = 0, sd = 0;
        auto scan = [&](auto lookup) {
            for (int a = O; a < M; a++) {
                const int b = lookup(K[0] - sys.n[a][0], K[1] - sys.n[a][1], K[2] - sys.n[a][2]);
                if (b > a) {
                    cols.push_back(a);
                    partner_of_col.push_back(b);
                    nvd++;
                }
            }
        };
        if (orb_wide) scan([&](int x, int y, int z) { return orb.get_inside(x, y, z); });
        else scan([&](int x, int y, int z) { return orb.get(x, y, z); });
        // the self-partner a = b has n_a = K / 2
        if (K[0] % 2 == 0 && K[1] % 2 == 0 && K[2] % 2 == 0) {
            const int a = orb.get(K[0] / 2, K[1] / 2, K[2] / 2);
            if (a >= O) {
                cols.push_back(a);
                partner_of_col.push_back(a);
                sd++;
            }
        }
        for (int c = 0; c < nvd; c++) {
            cols.push_back(partner_of_col[c]);
            partner_of_col.push_back(cols[c]);
        }
        if (cols.empty()) continue;
        if (sd > 1) return "virtual block without partner symmetry";
        SolvePlan::Block blk;
        blk.o = (int)kpairs[k].size();
        blk.v = (int)cols.size();
        blk.pair0 = (int)p.pair_i.size();
        blk.vir0 = (int)p.vir.size();
        blk.t0 = t0;
        blk.nvd = nvd;
        blk.sd = sd;
        // rows: pairs i < j, the diagonal pair, then the mirrors (j,i) in the same order
        blk.nd = blk.dg = 0;
        for (auto &pr : kpairs[k])
            if (pr.first < pr.second) {
                p.pair_i.push_back((int16_t)pr.first);
                p.pair_j.push_back((int16_t)pr.second);
                blk.nd++;
            }
        for (auto &pr : kpairs[k])
            if (pr.first == pr.second) {
                p.pair_i.push_back((int16_t)pr.first);
                p.pair_j.push_back((int16_t)pr.second);
                blk.dg++;
            }
        for (int q = 0; q < blk.nd; q++) {
            const int16_t i = p.pair_i[blk.pair0 + q], j = p.pair_j[blk.pair0 + q];
            p.pair_i.push_back(j);
            p.pair_j.push_back(i);
        }
        if (2 * blk.nd + blk.dg != blk.o || blk.dg > 1) return "pair block without mirror symmetry";
        for (int a : cols) p.vir.push_back((int16_t)a);
        for (int c = 0; c < blk.v; c++) col_of[cols[c]] = c;
        for (int c = 0; c < blk.v; c++) p.pcol.push_back((int16_t)col_of[partner_of_col[c]]);
        for (int c = 0; c < blk.v; c++) col_of[cols[c]] = -1;
        t0 += (int64_t)blk.o * blk.v;
        p.blocks.push_back(blk);
    }
    p.namp = t0;
    if (p.namp >= (int64_t)1 << 31) return "too many amplitudes for 32-bit packed indices";
    p.ring_entries = (int64_t)O * V * O;

    // particle-hole rows (i,x) grouped by their momentum Q = n_x - n_i, groups in
    // lexicographic order of Q, rows within a group by i
    Lattice qid;
    qid.init(2 * nmax);
    std::vector<std::array<int, 3>> qvecs;
    std::vector<int> qcount;
    std::vector<int> row_q((size_t)O * V);
    for (int i = 0; i < O; i++)
        for (int x = O; x < M; x++) {
            int q0 = sys.n[x][0] - sys.n[i][0], q1 = sys.n[x][1] - sys.n[i][1], q2 = sys.n[x][2] - sys.n[i][2];
            int &id = qid.at(q0, q1, q2);
            if (id < 0) {
                id = (int)qvecs.size();
                qvecs.push_back({q0, q1, q2});
                qcount.push_back(0);
            }
            qcount[id]++;
            row_q[(size_t)i * V + (x - O)] = id;
        }
    std::vector<int> order(qvecs.size());
    for (size_t g = 0; g < order.size(); g++) order[g] = (int)g;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return qvecs[a] < qvecs[b]; });
    std::vector<int> gpos(qvecs.size()), gstart(qvecs.size());
    int r0 = 0;
    for (size_t g = 0; g < order.size(); g++) {
        gpos[order[g]] = (int)g;
        gstart[order[g]] = r0;
        p.groups.push_back(SolvePlan::PhGroup{r0, qcount[order[g]], -1});
        r0 += qcount[order[g]];
    }
    p.ph_i.assign((size_t)O * V, 0);
    p.ph_x.assign((size_t)O * V, 0);
    std::vector<int> fill(qvecs.size(), 0);
    for (int i = 0; i < O; i++)
        for (int x = O; x < M; x++) {
            int id = row_q[(size_t)i * V + (x - O)];
            int r = gstart[id] + fill[id]++;
            p.ph_i[r] = (int16_t)i;
            p.ph_x[r] = (int16_t)x;
        }
    for (size_t g = 0; g < qvecs.size(); g++) {
        int m = qid.get(-qvecs[g][0], -qvecs[g][1], -qvecs[g][2]);
        if (m >= 0) p.groups[gpos[g]].partner = gpos[m];
    }
    return "";
}

}  // namespace uegccd
