// plan.h -- host-side momentum-block plan of one or many uniform-electron-gas systems.
#pragma once
#include <array>
#include <cstdint>
#include <string>
#include <vector>

#include "uegccd_internal.h"

namespace uegccd {

constexpr double kPi = 3.1415926535897932384626433833;  // Constants.f90:7

// One system as the hot path sees it (HEGData/UEGInfo fields, Types.f90:7-82).
struct SystemHost {
    int O = 0, M = 0;
    double L = 0, madelung = 0;
    std::vector<double> eigen;              // M
    std::vector<std::array<int, 3>> n;      // M integer plane-wave vectors
};

// Plan of one solve: its K blocks and index maps (local indices).
struct SolvePlan {
    int O = 0, V = 0, M = 0;
    int q2max = 0;
    std::vector<double> vtab;               // V(|q|^2), |q|^2 = 0..q2max
    // rows of a block: nd pairs (i,j) with i < j, then the diagonal pair (i,i) if K = 2 n_i
    // (dg = 1), then the mirrors (j,i) of the first nd in the same order: row p < nd has its
    // mirror at p + nd + dg.  Columns likewise: nvd virtuals a < K - a, the virtual a = K - a
    // if any (sd = 1), then the partners: column c < nvd has its partner at c + nvd + sd.
    struct Block { int o, v, pair0, vir0; int64_t t0; int nd, dg, nvd, sd; };
    std::vector<Block> blocks;
    std::vector<int16_t> pair_i, pair_j;    // concatenated pair lists
    std::vector<int16_t> vir;               // concatenated virtual lists (absolute orbital index)
    std::vector<int16_t> pcol;              // beside vir: column of the partner b = K - a in the same block
    int64_t namp = 0;
    int64_t ring_entries = 0;               // O*V*O
    // particle-hole rows (i,x), x virtual, sorted by Q = n_x - n_i
    std::vector<int16_t> ph_i, ph_x;        // row -> (i, x)
    struct PhGroup { int r0, n, partner; }; // partner: index of the -Q group or -1
    std::vector<PhGroup> groups;
};

// Builds the plan of one system.  Returns "" on success, else a message.
std::string build_solve_plan(const SystemHost &sys, SolvePlan &plan);

// Coulomb kernel of the reference for the default Input (BaseERI, HEG.f90:969-976):
// V(q) = 1/(L*pi*|q|^2) for q != 0, and -Madelung at q = 0.
double coulomb_v(double L, double madelung, int q2);

}  // namespace uegccd
