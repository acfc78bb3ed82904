// kernels.h -- device buffers of a batch and the kernel launch wrappers.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "uegccd_internal.h"

namespace uegccd {

// Raw device pointers of one batch (owned by the Batch object in capi.cu).
constexpr int kVtabSmemEntries = 1024;   // |q|^2 table entries a kernel stages in shared memory at most

struct DevBatch {
    int nsolves = 0, nblocks = 0, ntiles = 0, nchunks = 0, nrchunks = 0, ntargets = 0;
    int max_o = 0;      // largest o_K
    int max_v = 0;      // largest v_K
    // mosaics: block row and column sums, and per target the list of partials to add
    double *mpart = nullptr;
    int32_t *mt_start = nullptr, *mt_list = nullptr;
    size_t mosaic_smem = 0;
    int mosaic_vt = 0;  // |q|^2 table entries k_mosaic_blk stages: the batch's largest, at most kVtabSmemEntries
    int ntile_cls[5] = {0, 0, 0, 0, 0};   // ladder tiles per class: paired 8, then 8, 16, 24, 32 pairs
    int nhtile_cls[5] = {0, 0, 0, 0, 0};  // hole-hole intermediate tiles per class
    int max_occ = 0;    // largest NOcc
    int64_t namp = 0;
    SolveDev *solves = nullptr;
    BlockDev *blocks = nullptr;
    LadderTile *tiles = nullptr;     // particle-particle (+hole-hole apply) tiles; pad = row tile NP (8/16/24/32)
    LadderTile *htiles = nullptr;    // hole-hole intermediate tiles
    int nhtiles = 0;
    ChunkDev *chunks = nullptr;      // amplitude chunks
    ChunkDev *rchunks = nullptr;     // ring-intermediate chunks over (i, x, l)
    int *chunk_begin = nullptr;      // nsolves+1: first chunk of each solve
    HChunkDev *hchunks = nullptr;    // chunks of the amplitudes i <= j (k_update, DIIS, commit)
    int nhchunks = 0;
    int *hchunk_begin = nullptr;     // nsolves+1: first half chunk of each solve
    int2 *targets = nullptr;         // mosaic targets (solve, id)
    int16_t *pair_i = nullptr, *pair_j = nullptr, *vir = nullptr;
    int16_t *pcol = nullptr;          // beside vir: column of the partner d = K - c in the same block
    int32_t *pos = nullptr;          // dense (i,j,a) -> global packed index or -1
    int32_t *partner = nullptr;      // packed -> packed index of (i,j,b)
    int32_t *mirror = nullptr;       // packed (i,j,a): index of (j,i,b) if i < j, -1 if i = j, -2 if i > j
    AmpInfo *amps = nullptr;
    int4 *nv4 = nullptr;
    int *nvp = nullptr;              // the same vectors packed a component per byte (q2p in kernels_fp64.cu)
    double *eigen = nullptr, *vtab = nullptr;
    double *t = nullptr, *t_new = nullptr, *g = nullptr;
    double2 *vcoef = nullptr;         // per amplitude {v(i-a), v(a-j)} (k_vcoef, once per batch)
    double *jvv = nullptr, *joo = nullptr;
    double *J1 = nullptr;             // dRPA ring intermediate (on the first dRPA solve)
    int64_t ph_total = 0;             // O*V*O entries summed over the solves
    int64_t *hh0 = nullptr;          // per block: offset of H_K in hh
    double *hh = nullptr;
    double *part_e = nullptr, *part_dt = nullptr, *part_r = nullptr;
    double *red = nullptr;           // 3 per solve: sum e, max dt, max |r|
    uint8_t *active = nullptr;       // per solve
    // particle-hole form of the ring terms
    int16_t *ph_i = nullptr, *ph_x = nullptr;   // row -> (i, x), rows grouped by Q
    int32_t *ridx_x = nullptr, *ridx_y = nullptr;  // at ph0 + row*O + k: index of t(ik, x), t(ki, x)
    RingPairDev *rpairs = nullptr;              // {Q, -Q} group pairs, by k_rings class
    RingPairDev *spairs = nullptr;              // the same pairs in solve order (k_ring_stage: each
                                                // solve's amplitudes are gathered while in L2)
    // rings in the particle-hole layout (RingPairDev::xy0): xy holds the amplitudes each pair
    // multiplies, row by row (k_ring_stage gathers t into it before every ring launch); rx
    // the ring and crossed-ring G the pair forms, in the same places (k_update reads them).
    // Per (i, x) at phr0 + i*V + x - O: ph_a = the row's offset in xy/rx when (i, x) is in
    // its pair's group 1, else -1; ph_b = round8(n2) of its pair in group 1 (where the Y1 /
    // crossed-ring half of the row starts), its column b in group 2 (-1 without a pair).
    double *xy = nullptr, *rx = nullptr;
    int64_t xy_n = 0;
    int32_t *ph_a = nullptr, *ph_b = nullptr;
    int2 *rpos = nullptr;            // per amplitude i <= j: its ring G and crossed-ring G in rx
    // mixed precision: tensor-core ladder tiles sorted by row tile (16, 32, 64)
    LadderTile *tctiles = nullptr;
    int ntc16 = 0, ntc32 = 0, ntc64 = 0;
    double *t_ref = nullptr, *g_ref = nullptr;  // refresh point of the defect correction
    int *tc_err = nullptr;
    // FP16 operands of the tensor-core ladder (allocated and built on first mixed use)
    TcTileDev *tcx = nullptr;        // beside tctiles
    WSlabDev *wslabs = nullptr;
    DTileDev *dtiles = nullptr;
    int nwslabs = 0, ndtiles = 0;
    int64_t w16_n = 0, d16_n = 0;    // halves
    int nscale = 0;
    void *w16 = nullptr, *d16 = nullptr;   // __half arrays
    float *dscale = nullptr;
    bool w16_valid = false;          // built for the current integral tables
    int nrpairs = 0;
    // ring pair classes, rpairs sorted in this order: k_rings in kRingClasses shared-memory
    // sizes (kRingSmemClass), then k_rings_wide
    int nring[5] = {0, 0, 0, 0, 0};
    size_t ring_smem[5] = {0, 0, 0, 0, 0};
    int ring_threads[4] = {32, 128, 256, 256};  // CTA size per k_rings class: defaults, then tune_rings
    int stage_threads = 128;                    // CTA size of k_ring_stage (tune_rings)
    // ladder tiles in a second order: within each row-tile class the blocks with the most
    // virtuals (the longest c loops) first; ladder_sched picks the order the launches use
    LadderTile *tiles_lpt = nullptr, *htiles_lpt = nullptr;
    int ladder_sched = 0;                       // 0: block order, 1: longest first (tune_rings)
    int hh_kc = 64;                             // the hole-hole intermediate's column chunk: 64 or 32 (tune_rings)
};
// dynamic shared memory of k_rings_wide for NOcc = O and R rows of a group pair
size_t rings_smem_bytes(int O, int R);
// dynamic shared memory of k_mosaic_blk for blocks of at most max_v virtuals
size_t mosaic_smem_bytes(int max_v, int max_o, int vt_n);
void set_mosaic_smem_limit(size_t bytes);
// dynamic shared memory of k_ladder3<np> for blocks of at most max_v virtuals
// row-tile classes: paired 8 (blocks with at most kPairedRows rows i <= j, pad = 4 in
// LadderTile), then 8, 16, 24 and 32 pairs
constexpr int kLadderClasses = 5;
constexpr int kPairedRows = 4;
size_t ladder_smem_bytes(int max_v, int np);
void set_ladder_smem_limit(int max_v);
// dynamic shared memory of k_rings for NOcc = O and groups of n1 and n2 rows
size_t rings_dmma_smem_bytes(int O, int n1, int n2, int q2max);
// k_rings classes by padded pair size N1 + N2 (up to kRingClassRows), each with its
// CTA size (DevBatch::ring_threads); pairs above the last class, or above kRingSmemMax,
// go to k_rings_wide
constexpr int kRingClasses = 4;
constexpr int kRingClassRows[kRingClasses] = {16, 32, 48, 1 << 30};
constexpr size_t kRingSmemMax = 200 * 1024;
void set_rings_smem_limit(int wide, size_t bytes);
// Launch-shape autotuner, on the batch's current amplitudes: times k_rings of every pair
// class with 32, 64, 128 and 256 threads per CTA (d.ring_threads), k_ring_stage with 64,
// 128 and 256 (d.stage_threads), and the particle-particle ladder with its tiles in block
// order and longest first (d.ladder_sched); keeps the fastest of each.  None of these
// changes a sum's order: results are bitwise the same.  Not inside a stream capture.
// Returns a cudaError_t value.
int tune_rings(DevBatch &d, cudaStream_t st);

constexpr int kDiisMax = 16;   // DIIS history capacity (k_update and k_diis_* use the same bound)

// Live per-kernel timing with CUDA events on the launching stream (off unless enabled).
enum KernelId { KID_MP2 = 0, KID_ENERGY, KID_HH_W, KID_LADDER, KID_MOSAIC_S, KID_MOSAIC_RED, KID_RING_INT,
                KID_UPDATE, KID_REDUCE, KID_RINGS, KID_LADDER_TC, KID_RING_STAGE,
                KID_COUNT };
struct KernelTimer {
    bool on = false;
    cudaEvent_t ev[2 * 64];
    int kid[64];
    int n = 0;
    double ms[KID_COUNT] = {};
    long long launches[KID_COUNT] = {};
    void begin(int id, cudaStream_t st)
    {
        if (!on || n >= 64) return;
        kid[n] = id;
        cudaEventRecord(ev[2 * n], st);
    }
    void end(cudaStream_t st)
    {
        if (!on || n >= 64) return;
        cudaEventRecord(ev[2 * n + 1], st);
        n++;
    }
    // call after the stream is synchronised
    void collect()
    {
        for (int k = 0; k < n; k++) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, ev[2 * k], ev[2 * k + 1]) == cudaSuccess) {
                ms[kid[k]] += t;
                launches[kid[k]]++;
            } else {
                cudaGetLastError();  // a missing sample is not an error of the solve
            }
        }
        n = 0;
    }
};
extern const char *kKernelNames[KID_COUNT];

// Per-solve iteration state kept on the device (see k_control).
struct IterState {
    int niter;      // NIter of the reference (1 before the first update)
    int status;     // 0 running, 1 converged, 2 MaxIter reached, 3 non-finite
    double e, dt;   // energy and max|dT| of the latest iteration
};

// Buffers of the device-side iteration control.
struct CtlBuffers {
    IterState *state = nullptr;
    uint8_t *active_next = nullptr;
    int *count = nullptr;
    double *Bm = nullptr, *coef = nullptr, *brow = nullptr, *part = nullptr;
    double *hist_t = nullptr;   // DIIS history: updated amplitudes t' (FP64)
    float *hist_e = nullptr;    // and error vectors e = t' - t (FP32: they only enter the B-matrix dots)
    double *rec_e = nullptr, *rec_dt = nullptr;
    int max_rec = 0;
};

struct TermFlags {
    int do_driver = 1, do_mosaic = 1, do_ladder = 1, do_pp = 1, do_hh = 1, do_ring = 1, do_xring = 1;
    int drpa = 0;
    int mixed = 0;  // particle-particle ladder on the tensor cores (defect correction on t - t_ref)
};

void launch_mp2(const DevBatch &d, cudaStream_t st);
void launch_reduce(const DevBatch &d, cudaStream_t st);
void launch_energy(const DevBatch &d, int kind, double csosex, cudaStream_t st);
// d.t_new = T2aaaa of d.t (t(ij,a) - t(ij,b))
void launch_to_aaaa(const DevBatch &d, cudaStream_t st);
// Residual of the selected terms for d.t; mode 0 also updates into d.t_new.  Returns launches.
struct CtlBuffers;
// diis/ndiis (mode 0 only): fuse the Pulay DIIS push into the update kernel
int launch_residual(const DevBatch &d, const TermFlags &f, int mode, double *g_out, cudaStream_t st,
                    KernelTimer *kt = nullptr, const CtlBuffers *diis = nullptr, int ndiis = 0);
void launch_pack(const DevBatch &d, int s, int namp, const double *dense, cudaStream_t st);
void launch_vcoef(const DevBatch &d, cudaStream_t st);
void launch_unpack_all(const DevBatch &d, const int64_t *dense_off, const double *t, double *out, cudaStream_t st);
// Structure-factor sums of solve `solve` from d.t: groups = its particle-hole groups
// {first row, rows}; grid = 5 arrays of (2S+1)^3 (SfSum, SfDSum, SfXSum, contributions,
// 1 where the reference's last contribution is a core pair), column-major from -S,
// zeroed by the caller; *err = 1 if a transfer falls outside.
void launch_sf(const DevBatch &d, const int2 *groups, int ngroups, int solve, int S, double *grid, int *err,
               cudaStream_t st);
// pos (pre-set to -1), amps, partner, mirror from the block structure; the particle-hole
// tables ph_a, ph_b (pre-set to -1) from the ring pairs; the ring gather indices
void launch_block_tables(const DevBatch &d, cudaStream_t st);
// mt_start / mt_list of the mosaic sums from the blocks (tbase: each solve's first target;
// lbase: its first list entry; smem: (max V + O) ints)
void launch_mosaic_targets(const DevBatch &d, const int *tbase, const int64_t *lbase, size_t smem, cudaStream_t st);
// Mixed precision: FP16 tcgen05 ladder of t - t_ref added to g (plus g_ref); writes the
// scaled FP16 d tiles first (d.w16 must be built)
void launch_ladder_tc(const DevBatch &d, const double *t_ref, const double *g_ref, int *err, cudaStream_t st);
// The static FP16 Coulomb slabs of the tensor-core ladder, from the current |q|^2 tables
void launch_w16_build(const DevBatch &d, cudaStream_t st);
// Refresh point: t_ref <- t and g_ref <- FP64 particle-particle ladder of t_ref
void launch_refresh(const DevBatch &d, cudaStream_t st);
// Device-side iteration control
void launch_control(const DevBatch &d, const CtlBuffers &c, double tol, int max_iter, int ndiis, int init,
                    cudaStream_t st);
void launch_active_swap(const DevBatch &d, const CtlBuffers &c, cudaStream_t st);
int launch_iteration(const DevBatch &d, const CtlBuffers &c, const TermFlags &f, double tol, int max_iter,
                     int ndiis, cudaStream_t st, KernelTimer *kt);
void launch_unpack(const DevBatch &d, int s, int namp, const double *t, double *ab, double *ba, double *aa,
                   cudaStream_t st);

// Makes `dev` the calling thread's current CUDA device for the scope's lifetime and puts the
// previous one back at its end.  Every object of the library (batch, context, DIIS history)
// records the device it was created on, and every call on it runs under one of these, so a
// host thread whose current device differs (a fresh thread starts on device 0) still works on
// the object's own device.  rc is the cudaSetDevice status.
struct DeviceScope {
    int prev = -1, dev = -1;
    cudaError_t rc = cudaSuccess;
    explicit DeviceScope(int d) : dev(d)
    {
        if (d < 0) return;
        rc = cudaGetDevice(&prev);
        if (rc == cudaSuccess && prev != d) rc = cudaSetDevice(d);
        else if (rc == cudaSuccess) prev = -1;   // already current: nothing to restore
    }
    ~DeviceScope()
    {
        if (prev >= 0 && prev != dev) cudaSetDevice(prev);
    }
    DeviceScope(const DeviceScope &) = delete;
    DeviceScope &operator=(const DeviceScope &) = delete;
};

// The current device's index, or 0 when the query fails (for per-device caches).
inline int current_device()
{
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess) d = 0;
    return d;
}
constexpr int kMaxDevices = 64;

}  // namespace uegccd
