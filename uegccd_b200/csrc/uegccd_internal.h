// uegccd_internal.h -- device data model shared by the host planner and the kernels.
//
// Amplitudes are stored block-packed by total crystal momentum K = n_i + n_j
// (n_p the integer plane-wave vector of orbital p).  Block K holds o_K ordered
// occupied pairs (i,j) as rows and v_K virtuals a (whose partner
// b = K - a is also a virtual of the basis) as columns, row-major, one block
// after another.  Only momentum-allowed amplitudes are stored; the reference's
// dense T(NOcc,NOcc,NOcc+1:NAO) holds the same values with zeros elsewhere.
//
// The stored amplitude is the spin-adapted t(ij,a) = T2abab(i,j,a); the
// reference's other channels follow from it: T2abba(i,j,a) = -t(ij,b) and
// T2aaaa(i,j,a) = t(ij,a) - t(ij,b).
//
// Integral options.  GapII (GapERI, HEG.f90:890-942) zeroes every integral above
// GapII: it is a filter on the |q|^2 table.  CoreN (CoreERI) zeroes every integral
// with a core index.  In every CCD, MP2 and dRPA term each internal occupied index
// appears in the integral and in an amplitude, so for a non-core (i,j) the core
// integrals only ever multiply core amplitudes; and every term of a core (i,j) has
// a core integral or a core amplitude.  With the core amplitudes held at zero the
// unmasked sums are therefore exact: the kernels zero t and G of core pairs only.
//
// Many independent solves (twists, rs values, basis sizes) live in one batch:
// every per-solve array is concatenated and addressed through SolveDev offsets.
#pragma once
#include <cstdint>

namespace uegccd {

constexpr int kChunk = 256;  // amplitudes per element-wise work chunk

struct SolveDev {
    int O, V, M;            // occupied, virtual, orbitals
    int nblk, blk0;         // K blocks of this solve: [blk0, blk0+nblk)
    int orb0;               // offset of this solve's orbitals in nvec/eigen
    int vtab0, q2max;       // Coulomb table: vtab[vtab0 + |q|^2], |q|^2 <= q2max
    int64_t amp0;           // first packed amplitude (global index)
    int32_t namp;           // number of stored amplitudes
    int32_t core_n;         // UEGInfo%CoreN: orbitals p < core_n are core (CoreERI, HEG.f90:835-888)
    int64_t pos0;           // offset of the dense (i,j,a) -> packed map (O*O*V entries)
    int64_t ph0;            // offset of the ring intermediates (O*V*O entries each)
    int32_t jvv0, joo0;     // offsets of the mosaic intermediates (V and O entries)
    double denom_factor;    // SolveCC damping (CCD.f90:380), 2 in the reference
    int64_t phr0;           // offset of the particle-hole row arrays (O*V entries: one per row (i,x))
};

struct BlockDev {
    int solve;              // owning solve
    int o, v;               // o_K rows (ordered occupied pairs), v_K columns (virtuals)
    int pair0;              // offset into pair_i/pair_j
    int vir0;               // offset into vir (absolute orbital indices, local to the solve)
    int64_t t0;             // global packed index of element (row 0, col 0)
    int64_t row0, col0;     // offsets of the block's row and column sums in the mosaic partials
    int nd, dg;             // rows [0, nd) are pairs i < j, row nd the pair (i,i) if dg = 1, and
                            // row p + nd + dg the mirror (j,i) of row p < nd
    int nvd, sd;            // columns likewise: [0, nvd) virtuals a < K - a, column nvd the
                            // virtual a = K - a if sd = 1, column c + nvd + sd the partner of c < nvd
};

// One tile of the particle-particle ladder: rows [p0, p0+P) x columns [a0, a0+A) of block blk.
struct LadderTile {
    int blk, a0, p0, pad;
};

// Mixed precision: where a tensor-core ladder tile finds its FP16 operands, in the MMA's
// canonical K-major layout (32-wide K chunks): the block's Coulomb slab of its 128 virtuals
// (static; woff, in halves) and the scaled d = t - t_ref rows of its row tile (each
// iteration; doff in halves, row scales at soff).
struct TcTileDev {
    int64_t woff, doff;
    int32_t soff, pad;
};
// One FP16 Coulomb slab (block blk, virtuals a0 .. a0+127, every K chunk) to build.
struct WSlabDev {
    int blk, a0;
    int64_t woff;
};
// One row tile (block blk, rows p0 .. p0+np-1) of scaled FP16 d to write each iteration.
struct DTileDev {
    int blk, p0, np, soff;
    int64_t doff;
};

// Per-amplitude record: orbital indices local to the solve (a, b absolute, >= O).
struct AmpInfo {
    int16_t i, j, a, b;
};

// One pair of particle-hole groups {Q, -Q}: rows [r1, r1+n1) have n_x - n_i = Q,
// rows [r2, r2+n2) have -Q (rows local to the solve); group 1 is the smaller one.  All
// ring and crossed-ring products between the two groups are formed by one CTA.
// xy0: where the pair's operands and results start (in doubles) in the batch's
// particle-hole arrays: row a < n1 of group 1 holds 2 round8(n2) doubles -- in xy the
// amplitudes X1[a][b] = t(i_a i_b, x_a) then Y1[a][b] = t(i_b i_a, x_a), in rx the ring G
// of (i_a, i_b, x_a) then the crossed-ring G of (i_a, i_b, x_b), b over group 2.
struct RingPairDev {
    int solve;
    int r1, n1;
    int r2, n2;
    int32_t xy0;
};

struct ChunkDev {
    int solve;
    int32_t start;          // first amplitude of the chunk, local to the solve
};

// A chunk of the amplitudes i <= j (the rows a block keeps; each mirror row follows from
// its pair): [start, end) local to the solve, at most kChunk long, inside one block.
struct HChunkDev {
    int solve;
    int32_t start, end, pad;
};

}  // namespace uegccd
