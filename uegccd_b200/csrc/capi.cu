// capi.cu -- the C ABI of include/uegccd.h: contexts, batches and the solve drivers.
//
// A context is a batch of one system.  The drivers follow DrvMBPT (MP2.f90:11-157),
// DrvCCD (CCD.f90:18-183) and DrvdRPA (dRPA.f90:23-174): MP2 guess, then
// residual -> update -> convergence -> energy per iteration until max|dT| < TolMax
// or MaxIter, then one final residual for MaxRes.  All amplitudes, index maps
// and intermediates stay on the device for the whole solve; one small
// device-to-host read per iteration carries (E, max|dT|, max|R|) of every solve.
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <deque>
#include <condition_variable>
#include <atomic>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/uegccd.h"
#include "kernels.h"
#include "plan.h"
#include "two_channel.h"
#include "uegccd_internal.h"

using namespace uegccd;

namespace {

thread_local std::string g_last_error;

// A persistent pool of host threads (one per core) for the parallel parts of batch creation
// and downloads: starting threads per call cost more than the work of a small batch.  Several
// callers (the creator threads of a pipelined host) share it.
class HostPool {
public:
    explicit HostPool(int n)
    {
        for (int k = 0; k < n; k++)
            th_.emplace_back([this]() {
                for (;;) {
                    std::function<void()> job;
                    {
                        std::unique_lock<std::mutex> lock(mu_);
                        cv_.wait(lock, [this]() { return stop_ || !q_.empty(); });
                        if (stop_ && q_.empty()) return;
                        job = std::move(q_.front());
                        q_.pop_front();
                    }
                    job();
                }
            });
    }
    ~HostPool()
    {
        {
            std::lock_guard<std::mutex> lock(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &t : th_) t.join();
    }
    void post(std::function<void()> job)
    {
        {
            std::lock_guard<std::mutex> lock(mu_);
            q_.push_back(std::move(job));
        }
        cv_.notify_one();
    }

private:
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<std::function<void()>> q_;
    std::vector<std::thread> th_;
    bool stop_ = false;
};

HostPool &host_pool()
{
    static HostPool pool(std::max(1, (int)std::thread::hardware_concurrency()));
    return pool;
}

// Runs f(0..n-1) on the calling thread and up to nthreads - 1 pool threads; items are taken
// in turn from a shared counter, and each f(i) writes only its own outputs.
template <class F>
void parallel_for(int n, int nthreads, F f)
{
    if (nthreads <= 1 || n <= 1) {
        for (int i = 0; i < n; i++) f(i);
        return;
    }
    struct Shared {
        std::atomic<int> next{0};
        std::mutex mu;
        std::condition_variable cv;
        int finished = 0;
    } sh;
    const int helpers = std::min(nthreads, n) - 1;
    auto body = [&]() {
        for (int i; (i = sh.next.fetch_add(1)) < n;) f(i);
    };
    for (int k = 0; k < helpers; k++)
        host_pool().post([&]() {
            body();
            std::lock_guard<std::mutex> lock(sh.mu);
            if (++sh.finished == helpers) sh.cv.notify_one();
        });
    body();
    std::unique_lock<std::mutex> lock(sh.mu);
    sh.cv.wait(lock, [&]() { return sh.finished == helpers; });
}

int fail(int code, const std::string &msg)
{
    g_last_error = msg;
    return code;
}

#define CU(call)                                                                                       \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return fail(UEGCCD_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_));            \
    } while (0)

int check_device()
{
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
        return fail(UEGCCD_ERR_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
    int dev = 0;
    CU(cudaGetDevice(&dev));
    // one attribute query (cudaGetDeviceProperties reads every property: tens of ms per call)
    int major = 0;
    CU(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
    if (major != 10) {
        cudaDeviceProp p;
        CU(cudaGetDeviceProperties(&p, dev));
        return fail(UEGCCD_ERR_CUDA, std::string("the library is built for sm_100a (B200); device is ") + p.name);
    }
    return 0;
}

}  // namespace

// ----------------------------------------------------------------------------
// Batch: plans + device buffers of n systems
// ----------------------------------------------------------------------------
// Device memory of a batch: carved from chunks of at least kArenaChunk bytes. Chunks
// freed by a destroyed batch are kept in a small per-process cache (up to kPoolCap
// bytes) for the next batch; uegccd_trim_cache returns them to the driver.
namespace {
constexpr size_t kArenaChunk = 64ull << 20;
constexpr size_t kPoolCap = 32ull << 30;   // a 100-twist N=54 batch takes ~3 GB; pipelines keep 3-4 alive
struct DevChunk {
    char *p;
    size_t size;
    int dev;
};
// pinned staging buffer of the batch-wide amplitude download (grown on demand, kept; portable:
// page-locked for every device's context)
constexpr size_t kStageMin = 8ull << 20;
std::mutex g_stage_mu;
char *g_stage = nullptr;
size_t g_stage_bytes = 0;
// g_pool_mu guards the cache, the per-device byte counts and the limit
std::mutex g_pool_mu;
std::vector<DevChunk> g_pool;
size_t g_pool_bytes = 0;
int64_t g_dev_bytes[kMaxDevices] = {};   // bytes the library holds from cudaMalloc per device (live + cached)
int64_t g_mem_limit = 0;                 // uegccd_set_memory_limit; 0: none

// Returns the cache of device dev to the driver (the caller holds no lock; dev is current).
void drop_cached(int dev)
{
    std::vector<DevChunk> drop;
    {
        std::lock_guard<std::mutex> lock(g_pool_mu);
        for (size_t k = 0; k < g_pool.size();)
            if (g_pool[k].dev == dev) {
                drop.push_back(g_pool[k]);
                g_pool_bytes -= g_pool[k].size;
                g_dev_bytes[dev % kMaxDevices] -= (int64_t)g_pool[k].size;
                g_pool.erase(g_pool.begin() + k);
            } else {
                k++;
            }
    }
    for (auto &c : drop) cudaFree(c.p);
}

// True when `need` more bytes on dev stay within the limit (under g_pool_mu).
bool within_limit(int dev, size_t need)
{
    return g_mem_limit <= 0 || g_dev_bytes[dev % kMaxDevices] + (int64_t)need <= g_mem_limit;
}

// A chunk of at least `need` bytes on device dev (current): from the cache, else cudaMalloc.
// Past the memory limit, or when cudaMalloc fails, the device's cache goes back to the driver
// and the request is tried once more; then cudaErrorMemoryAllocation.
cudaError_t chunk_get(size_t need, int dev, DevChunk &out)
{
    bool fits = true;
    {
        std::lock_guard<std::mutex> lock(g_pool_mu);
        int best = -1;
        for (size_t k = 0; k < g_pool.size(); k++)
            if (g_pool[k].dev == dev && g_pool[k].size >= need && g_pool[k].size <= 2 * need + kArenaChunk &&
                (best < 0 || g_pool[k].size < g_pool[best].size))
                best = (int)k;
        if (best >= 0) {
            out = g_pool[best];
            g_pool_bytes -= out.size;
            g_pool.erase(g_pool.begin() + best);
            return cudaSuccess;
        }
        fits = within_limit(dev, need);
    }
    if (!fits) {
        drop_cached(dev);
        std::lock_guard<std::mutex> lock(g_pool_mu);
        if (!within_limit(dev, need)) return cudaErrorMemoryAllocation;
    }
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, need);
    if (e != cudaSuccess) {
        cudaGetLastError();
        drop_cached(dev);
        e = cudaMalloc(&p, need);
    }
    if (e == cudaSuccess) {
        out = DevChunk{(char *)p, need, dev};
        std::lock_guard<std::mutex> lock(g_pool_mu);
        g_dev_bytes[dev % kMaxDevices] += (int64_t)need;
    }
    return e;
}

// Straight back to the driver; c.dev is current.
void chunk_free(const DevChunk &c)
{
    {
        std::lock_guard<std::mutex> lock(g_pool_mu);
        g_dev_bytes[c.dev % kMaxDevices] -= (int64_t)c.size;
    }
    cudaFree(c.p);
}

// Back to the cache, or (past its cap) to the driver; c.dev is current.
void chunk_put(const DevChunk &c)
{
    {
        std::lock_guard<std::mutex> lock(g_pool_mu);
        if (g_pool_bytes + c.size <= kPoolCap) {
            g_pool.push_back(c);
            g_pool_bytes += c.size;
            return;
        }
        g_dev_bytes[c.dev % kMaxDevices] -= (int64_t)c.size;
    }
    cudaFree(c.p);
}
}  // namespace

struct UegccdBatch {
    int dev = -1;                    // the CUDA device the batch lives on (current at creation)
    bool broken = false;             // restoring the plain integral tables failed: calls are refused
    std::vector<SystemHost> sys;
    std::vector<SolvePlan> plans;
    std::vector<SolveDev> hsolves;
    std::vector<int> chunk_begin;
    DevBatch d;
    std::vector<DevChunk> chunks;    // device memory of the batch (see chunk_get): arena chunks
    size_t chunk_used = 0;           // bytes used in the last arena chunk
    std::vector<DevChunk> big;       // chunks of one large array each
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_solve0 = nullptr, ev_solve1 = nullptr;
    std::vector<double> red;         // host copy: 3 per solve
    std::vector<uint8_t> active;     // host copy
    double *dense[3] = {nullptr, nullptr, nullptr};  // reference-layout scratch of the largest solve
    size_t dense_n = 0;
    double *dense_all = nullptr;     // reference layout of every solve, back to back (on first use)
    int64_t *dense_off = nullptr;
    size_t dense_all_n = 0;
    int launches = 0;
    int64_t h2d_bytes = 0, d2h_bytes = 0;   // host<->device traffic of the calls so far
    KernelTimer kt;
    bool kt_events = false;
    // device-side iteration control (allocated on first solve; DIIS history grows on demand)
    CtlBuffers ctl;
    int diis_cap = 0;
    std::vector<int> last_niter;     // iterations of each solve in the last solve call
    // an incremental solve (uegccd_batch_start / _advance): its options and which solves have
    // had their result released
    struct Session {
        bool on = false;
        UegccdOptions opt{};
        int drpa = 0, ndiis = 0, max_rec = 0;
        TermFlags f;
        std::vector<uint8_t> released;
    } ses;
    // CUDA graphs of one iteration: plain and with kernel timers, keyed by the options
    struct GraphKey {
        int do_ring, do_xring, do_ladder, do_mosaic, drpa, ndiis, max_iter, mixed;
        double tol;
        bool operator==(const GraphKey &o) const
        {
            return do_ring == o.do_ring && do_xring == o.do_xring && do_ladder == o.do_ladder &&
                   do_mosaic == o.do_mosaic && drpa == o.drpa && ndiis == o.ndiis && max_iter == o.max_iter &&
                   mixed == o.mixed && tol == o.tol;
        }
    } gkey{};
    bool have_graph = false;
    bool rings_tuned = false;        // k_rings CTA sizes picked (before the first graph capture)
    cudaGraphExec_t gexec = nullptr;
    int g_launches = 0;          // kernels per iteration
    // structure factors (on first use): every solve's particle-hole groups {first row, rows},
    // solve s at [sf_g0[s], sf_g0[s+1]); one grid of the largest solve
    int2 *sf_groups = nullptr;
    std::vector<int> sf_g0;
    // integral options (CoreN, GapII) in force, and the unfiltered |q|^2 tables of all solves
    int core_n = 0;
    double gapii = 0.0;
    std::vector<double> vtab_base;
    // range-separated integrals with one flag for every CCD term (uegccd_*_set_range)
    int range_flag = 0;
    double screening = 0.0;
    // batch solves in the two-channel form (do_ring != do_xring): one two_channel.cu state per
    // system, made on first use; each solve's iteration table; two_channel_amps: the batch's
    // amplitudes hold T2abab of such a solve (the spin relation does not give T2abba)
    std::vector<std::unique_ptr<uegccd::TwoChannel>> tcs;
    std::vector<std::vector<double>> tc_en, tc_dt;
    bool two_channel_amps = false;
    double *sf_grid = nullptr;
    int *sf_err = nullptr;

    ~UegccdBatch()
    {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (kt_events)
            for (auto &e : kt.ev) cudaEventDestroy(e);
        if (stream) cudaStreamSynchronize(stream);
        for (auto &c : chunks) chunk_put(c);
        for (auto &c : big) chunk_put(c);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (ev_solve0) cudaEventDestroy(ev_solve0);
        if (ev_solve1) cudaEventDestroy(ev_solve1);
        if (stream) cudaStreamDestroy(stream);
    }

    template <class T>
    int alloc(T *&p, size_t n)
    {
        p = nullptr;
        if (n == 0) n = 1;
        const size_t bytes = (n * sizeof(T) + 255) & ~(size_t)255;
        if (bytes >= kArenaChunk / 2) {
            // large arrays get a chunk of their own, of exactly the size they need
            DevChunk c;
            cudaError_t e = chunk_get(bytes, dev, c);
            if (e != cudaSuccess)
                return fail(UEGCCD_ERR_ALLOC, std::string("device allocation of ") + std::to_string(bytes) +
                                                  " bytes: " + cudaGetErrorString(e));
            big.push_back(c);
            p = reinterpret_cast<T *>(c.p);
            return 0;
        }
        if (chunks.empty() || chunk_used + bytes > chunks.back().size) {
            DevChunk c;
            cudaError_t e = chunk_get(kArenaChunk, dev, c);
            if (e != cudaSuccess)
                return fail(UEGCCD_ERR_ALLOC, std::string("device allocation of ") + std::to_string(kArenaChunk) +
                                                  " bytes: " + cudaGetErrorString(e));
            chunks.push_back(c);
            chunk_used = 0;
        }
        p = reinterpret_cast<T *>(chunks.back().p + chunk_used);
        chunk_used += bytes;
        return 0;
    }
    // Allocation marks: rollback(mark()) returns every chunk taken since the mark to the driver
    // (not to the cache: a failed group of allocations means memory is short) and the arena
    // space carved since -- the batch is left as it was (arena chunks are only ever appended,
    // so the mark's last one is the last one again).
    struct Mark {
        size_t nchunks, nbig, used;
    };
    Mark mark() const { return Mark{chunks.size(), big.size(), chunk_used}; }
    void rollback(const Mark &m)
    {
        while (big.size() > m.nbig) {
            chunk_free(big.back());
            big.pop_back();
        }
        while (chunks.size() > m.nchunks) {
            chunk_free(chunks.back());
            chunks.pop_back();
        }
        chunk_used = m.used;
    }
    template <class T>
    int upload(T *&p, const std::vector<T> &h)
    {
        int rc = alloc(p, h.size());
        if (rc) return rc;
        if (!h.empty()) CU(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
        h2d_bytes += (int64_t)(h.size() * sizeof(T));
        return 0;
    }
};

struct UegccdCtx {
    std::unique_ptr<UegccdBatch> batch;
    // the two-channel form (two_channel.cu), made on first use, and the integral selection of
    // uegccd_ctx_set_eri
    std::unique_ptr<uegccd::TwoChannel> tc;
    bool eri_set = false;
    UegccdRangeTerms flags{};
    int safe_eri = 0;
    double screening = 0.0;
};

namespace {

int read_system(const UegccdSystem *s, SystemHost &h)
{
    if (!s || !s->eigen || !s->nvec) return fail(UEGCCD_ERR_ARG, "null system or array");
    if (s->nocc <= 0 || s->nao <= s->nocc) return fail(UEGCCD_ERR_ARG, "need 0 < NOcc < NAO");
    if (!(s->L > 0)) return fail(UEGCCD_ERR_ARG, "L must be positive");
    h.O = s->nocc;
    h.M = s->nao;
    h.L = s->L;
    h.madelung = s->madelung;
    h.eigen.assign(s->eigen, s->eigen + s->nao);
    h.n.resize(s->nao);
    for (int p = 0; p < s->nao; p++)
        for (int d = 0; d < 3; d++) h.n[p][d] = s->nvec[p + (size_t)s->nao * d];
    return 0;
}

// UEGCCD_TRACE=1 in the environment: batch creation prints its phase times to stderr.
struct PhaseTrace {
    bool on = false;
    std::chrono::steady_clock::time_point t0, last;
    std::string line;
    PhaseTrace()
    {
        const char *e = std::getenv("UEGCCD_TRACE");
        on = e && e[0] == '1';
        t0 = last = std::chrono::steady_clock::now();
    }
    void mark(const char *what)
    {
        if (!on) return;
        const auto now = std::chrono::steady_clock::now();
        char buf[96];
        std::snprintf(buf, sizeof buf, " %s %.2f", what, std::chrono::duration<double, std::milli>(now - last).count());
        line += buf;
        last = now;
    }
    ~PhaseTrace()
    {
        if (on)
            std::fprintf(stderr, "uegccd batch create (ms):%s total %.2f\n", line.c_str(),
                         std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    }
};

int build_batch(const UegccdSystem *systems, int n, std::unique_ptr<UegccdBatch> &out)
{
    PhaseTrace trace;
    int rc = check_device();
    if (rc) return rc;
    if (n <= 0) return fail(UEGCCD_ERR_ARG, "empty batch");
    auto b = std::make_unique<UegccdBatch>();
    CU(cudaGetDevice(&b->dev));   // the batch lives on the device current now
    b->sys.resize(n);
    b->plans.resize(n);
    for (int s = 0; s < n; s++) {
        rc = read_system(&systems[s], b->sys[s]);
        if (rc) return rc;
    }
    // plans of different systems are independent: build them on parallel host threads
    const int nthreads = std::max(1, std::min(n, (int)std::thread::hardware_concurrency()));
    std::vector<std::string> msgs(n);
    parallel_for(n, nthreads, [&](int s) { msgs[s] = build_solve_plan(b->sys[s], b->plans[s]); });
    for (int s = 0; s < n; s++) {
        if (!msgs[s].empty()) return fail(UEGCCD_ERR_ARG, "system " + std::to_string(s) + ": " + msgs[s]);
        if (b->plans[s].O > 64) return fail(UEGCCD_ERR_UNSUPPORTED, "NOcc > 64 is outside the hole-hole ladder tiling");
        for (const auto &v : b->sys[s].n)
            if (std::abs(v[0]) > 63 || std::abs(v[1]) > 63 || std::abs(v[2]) > 63)
                return fail(UEGCCD_ERR_UNSUPPORTED, "system " + std::to_string(s) +
                                                        ": a plane-wave component beyond +-63 (the kernels take "
                                                        "momentum differences as signed bytes)");
    }
    trace.mark("plans");
    CU(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    CU(cudaEventCreate(&b->ev0));
    CU(cudaEventCreate(&b->ev1));
    CU(cudaEventCreate(&b->ev_solve0));
    CU(cudaEventCreate(&b->ev_solve1));
    trace.mark("stream");

    std::vector<SolveDev> solves(n);
    std::vector<BlockDev> blocks;
    std::vector<LadderTile> tiles, htiles, tc16, tc32, tc64;
    std::vector<TcTileDev> tcx16, tcx32, tcx64;   // beside tc16/32/64: FP16 operand offsets
    std::vector<WSlabDev> wslabs;
    std::vector<DTileDev> dtiles;
    int64_t w16_n = 0, d16_n = 0;
    int nscale = 0;
    // the large host tables live in vectors kept per creating thread between creates: a
    // fresh allocation would page-fault on first touch, which cost more than filling them
    struct HostTables {
        std::vector<ChunkDev> chunks, rchunks;
        std::vector<int2> targets;
        std::vector<int16_t> pair_i, pair_j, vir, pcol, ph_i, ph_x;
        std::vector<int4> nv4;
        std::vector<int> nvp;
        std::vector<double> eigen;
    };
    static thread_local HostTables ht;
    auto &chunks = ht.chunks, &rchunks = ht.rchunks;
    auto &targets = ht.targets;
    auto &pair_i = ht.pair_i, &pair_j = ht.pair_j, &vir = ht.vir;
    auto &pcol = ht.pcol;   // beside vir: the partner's column in the same block
    auto &nv4 = ht.nv4;
    auto &nvp = ht.nvp;     // beside nv4: packed a component per byte
    auto &eigen = ht.eigen;
    auto &ph_i = ht.ph_i, &ph_x = ht.ph_x;
    for (auto *v : {&chunks, &rchunks}) v->clear();
    targets.clear();
    for (auto *v : {&pair_i, &pair_j, &vir, &pcol, &ph_i, &ph_x}) v->clear();
    nv4.clear();
    nvp.clear();
    eigen.clear();
    std::vector<int> chunk_begin(n + 1, 0);
    std::vector<double> vtab;
    std::vector<int64_t> hh0;
    std::vector<RingPairDev> rpairs, spairs;
    int64_t amp0 = 0, pos0 = 0, ph0 = 0, hhoff = 0, phr0 = 0, mrows = 0, mcols = 0;
    std::vector<int> s_t0(n);   // first mosaic target of each solve
    int orb0 = 0, vtab0 = 0, jvv0 = 0, joo0 = 0, max_o = 0, max_v = 0, max_occ = 0;
    // offsets of each solve in the large concatenated arrays (filled in parallel below)
    std::vector<int64_t> s_phr0(n);
    for (int s = 0; s < n; s++) {
        const SolvePlan &P = b->plans[s];
        const SystemHost &H = b->sys[s];
        SolveDev &S = solves[s];
        S.O = P.O; S.V = P.V; S.M = P.M;
        S.nblk = (int)P.blocks.size();
        S.blk0 = (int)blocks.size();
        S.orb0 = orb0;
        S.vtab0 = vtab0;
        S.q2max = P.q2max;
        S.amp0 = amp0;
        S.namp = (int32_t)P.namp;
        S.core_n = 0;
        S.pos0 = pos0;
        S.ph0 = ph0;
        S.jvv0 = jvv0;
        S.joo0 = joo0;
        S.denom_factor = 2.0;
        S.phr0 = phr0;
        max_occ = std::max(max_occ, P.O);
        s_phr0[s] = phr0;
        for (size_t gi = 0; gi < P.groups.size(); gi++) {
            const auto &G = P.groups[gi];
            if (G.partner < 0 || G.partner < (int)gi) continue;  // each {Q, -Q} once
            const auto &H2 = P.groups[G.partner];
            // the smaller group first: k_rings gathers and multiplies from its side
            if (G.n <= H2.n) rpairs.push_back(RingPairDev{s, G.r0, G.n, H2.r0, H2.n, 0});
            else rpairs.push_back(RingPairDev{s, H2.r0, H2.n, G.r0, G.n, 0});
        }
        for (const auto &B : P.blocks) {
            BlockDev bd;
            bd.solve = s; bd.o = B.o; bd.v = B.v;
            bd.pair0 = (int)pair_i.size() + B.pair0;
            bd.vir0 = (int)vir.size() + B.vir0;
            bd.t0 = amp0 + B.t0;
            bd.nd = B.nd;
            bd.dg = B.dg;
            bd.nvd = B.nvd;
            bd.sd = B.sd;
            bd.row0 = mrows;
            bd.col0 = mcols;   // shifted past all rows below
            mrows += B.o;
            mcols += B.v;
            int bi = (int)blocks.size();
            blocks.push_back(bd);
            hh0.push_back(hhoff);
            hhoff += (int64_t)B.o * B.o;
            max_o = std::max(max_o, B.o);
            max_v = std::max(max_v, B.v);
            // FP64 ladder tiles cover the rows up to the diagonal pair (oc = nd + dg); k_ladder3
            // writes each mirror row from its pair (i,j) with the pair symmetry.  Row tiles of 32
            // pairs, the last one the remainder rounded up to 8 (8, 16, 24 or 32): at most 7
            // padded rows per block; columns in tiles of 128 (4 warps x 32)
            // Blocks with at most kPairedRows such rows run paired tiles (pad 4): each 8-wide
            // fragment holds the rows and their partner-column images, over the columns
            // a <= pcol a (mode 0) and the pairs q <= q' (mode 1).
            const int oc = B.nd + B.dg;
            auto row_tile = [&](int p0) { return std::min(32, (oc - p0 + 7) & ~7); };
            if (oc <= kPairedRows) {
                for (int a0 = 0; a0 < B.nvd + B.sd; a0 += 128) tiles.push_back(LadderTile{bi, a0, 0, 4});
                htiles.push_back(LadderTile{bi, 0, 0, 4});
            } else {
                for (int a0 = 0; a0 < B.v; a0 += 128)
                    for (int p0 = 0; p0 < oc; p0 += 32) tiles.push_back(LadderTile{bi, a0, p0, row_tile(p0)});
                for (int q0 = 0; q0 < B.o; q0 += 128)
                    for (int p0 = 0; p0 < oc; p0 += 32) htiles.push_back(LadderTile{bi, q0, p0, row_tile(p0)});
            }
            // tensor-core tiles: 128 virtuals x (16, 32 or 64) rows over the rows i <= j (the
            // update reads G there only); their FP16 operands: one Coulomb slab per 128
            // virtuals, one d tile per row tile, each over all K chunks
            const int ntc = oc <= 16 ? 16 : oc <= 32 ? 32 : 64;
            auto &tl = ntc == 16 ? tc16 : ntc == 32 ? tc32 : tc64;
            auto &tx = ntc == 16 ? tcx16 : ntc == 32 ? tcx32 : tcx64;
            const int64_t nch = (B.v + 31) / 32;
            const int64_t w0 = w16_n, d0 = d16_n;
            const int s0 = nscale;
            for (int a0 = 0; a0 < B.v; a0 += 128) {
                wslabs.push_back(WSlabDev{bi, a0, w16_n});
                w16_n += nch * 128 * 32;
            }
            for (int p0 = 0; p0 < oc; p0 += ntc) {
                dtiles.push_back(DTileDev{bi, p0, ntc, nscale, d16_n});
                d16_n += nch * ntc * 32;
                nscale += ntc;
            }
            for (int a0 = 0; a0 < B.v; a0 += 128)
                for (int p0 = 0; p0 < oc; p0 += ntc) {
                    tl.push_back(LadderTile{bi, a0, p0, ntc});
                    const int it = p0 / ntc;
                    tx.push_back(TcTileDev{w0 + (a0 / 128) * nch * 128 * 32, d0 + it * nch * ntc * 32, s0 + it * ntc, 0});
                }
        }
        pair_i.insert(pair_i.end(), P.pair_i.begin(), P.pair_i.end());
        pair_j.insert(pair_j.end(), P.pair_j.begin(), P.pair_j.end());
        vir.insert(vir.end(), P.vir.begin(), P.vir.end());
        pcol.insert(pcol.end(), P.pcol.begin(), P.pcol.end());
        for (int p = 0; p < P.M; p++) {
            nv4.push_back(make_int4(H.n[p][0], H.n[p][1], H.n[p][2], 0));
            nvp.push_back((H.n[p][0] & 0xff) | ((H.n[p][1] & 0xff) << 8) | ((H.n[p][2] & 0xff) << 16));
        }
        eigen.insert(eigen.end(), H.eigen.begin(), H.eigen.end());
        vtab.insert(vtab.end(), P.vtab.begin(), P.vtab.end());
        chunk_begin[s] = (int)chunks.size();
        for (int64_t st = 0; st < P.namp; st += kChunk) chunks.push_back(ChunkDev{s, (int32_t)st});
        for (int64_t st = 0; st < P.ring_entries; st += kChunk) rchunks.push_back(ChunkDev{s, (int32_t)st});
        s_t0[s] = (int)targets.size();
        for (int x = 0; x < P.V + P.O; x++) targets.push_back(make_int2(s, x));
        amp0 += P.namp;
        pos0 += (int64_t)P.O * P.O * P.V;
        ph0 += P.ring_entries;
        orb0 += P.M;
        vtab0 += P.q2max + 1;
        jvv0 += P.V;
        joo0 += P.O;
        phr0 += (int64_t)P.O * P.V;
        if (amp0 >= ((int64_t)1 << 31)) return fail(UEGCCD_ERR_ARG, "batch too large for 32-bit packed indices");
    }
    chunk_begin[n] = (int)chunks.size();
    // chunks of the amplitudes i <= j: each block's rows up to its diagonal pair
    std::vector<HChunkDev> hchunks;
    std::vector<int> hchunk_begin(n + 1, 0);
    for (int s = 0; s < n; s++) {
        hchunk_begin[s] = (int)hchunks.size();
        for (const auto &B : b->plans[s].blocks) {
            const int64_t lo = B.t0, hi = B.t0 + (int64_t)(B.nd + B.dg) * B.v;
            for (int64_t st = lo; st < hi; st += kChunk)
                hchunks.push_back(HChunkDev{s, (int32_t)st, (int32_t)std::min(st + kChunk, hi), 0});
        }
    }
    hchunk_begin[n] = (int)hchunks.size();
    trace.mark("solve-loop");
    ph_i.resize(phr0);
    ph_x.resize(phr0);
    parallel_for(n, nthreads, [&](int s) {
        const SolvePlan &P = b->plans[s];
        std::copy(P.ph_i.begin(), P.ph_i.end(), ph_i.begin() + s_phr0[s]);
        std::copy(P.ph_x.begin(), P.ph_x.end(), ph_x.begin() + s_phr0[s]);
    });

    // mosaic targets: Jvv(c) adds the column sums of c over the blocks holding it, Joo(k)
    // the row sums of the pairs (k, l); both in block order
    for (auto &bd : blocks) bd.col0 += mrows;
    // the lists themselves are built on the device (k_mosaic_targets); here only each solve's
    // first target and first list entry
    std::vector<int64_t> mt_lbase(n + 1, 0);
    int max_vo = 0;
    for (int s = 0; s < n; s++) {
        int64_t e = 0;
        for (const auto &B : b->plans[s].blocks) e += (int64_t)B.o + B.v;
        mt_lbase[s + 1] = mt_lbase[s] + e;
        max_vo = std::max(max_vo, b->plans[s].V + b->plans[s].O);
    }
    if (mt_lbase[n] >= ((int64_t)1 << 31)) return fail(UEGCCD_ERR_ARG, "batch too large for 32-bit mosaic lists");
    if ((size_t)max_vo * sizeof(int) > 200 * 1024) return fail(UEGCCD_ERR_UNSUPPORTED, "NAO too large for the mosaic lists");
    if (mrows + mcols >= ((int64_t)1 << 31)) return fail(UEGCCD_ERR_ARG, "batch too large for 32-bit mosaic indices");
    trace.mark("ph+mosaic");

    DevBatch &d = b->d;
    d.nsolves = n;
    d.nblocks = (int)blocks.size();
    // ladder tiles by row-tile class (stable: block order within a class)
    auto by_class = [](std::vector<LadderTile> &v, int *cnt) {
        std::vector<LadderTile> out;
        out.reserve(v.size());
        for (int c = 0; c < kLadderClasses; c++) {
            cnt[c] = 0;
            for (const auto &x : v)
                if (x.pad == (c == 0 ? 4 : 8 * c)) {
                    out.push_back(x);
                    cnt[c]++;
                }
        }
        v.swap(out);
    };
    const size_t ntl = tiles.size(), nhtl = htiles.size();
    by_class(tiles, d.ntile_cls);
    by_class(htiles, d.nhtile_cls);
    if (tiles.size() != ntl || htiles.size() != nhtl) return fail(UEGCCD_ERR_UNSUPPORTED, "ladder row tile outside the 4/8/16/24/32 classes");
    d.ntiles = (int)tiles.size();
    d.nhtiles = (int)htiles.size();
    // the second tile order the launch-shape tuner may pick: within each class, the tiles of
    // the blocks with the most virtuals (the longest c loops) first
    auto longest_first = [&](const std::vector<LadderTile> &v, const int *cnt) {
        std::vector<LadderTile> out(v);
        size_t off = 0;
        for (int c = 0; c < kLadderClasses; c++) {
            std::stable_sort(out.begin() + off, out.begin() + off + cnt[c], [&](const LadderTile &x, const LadderTile &y) {
                return blocks[x.blk].v > blocks[y.blk].v;
            });
            off += cnt[c];
        }
        return out;
    };
    const std::vector<LadderTile> tiles_lpt = longest_first(tiles, d.ntile_cls),
                                  htiles_lpt = longest_first(htiles, d.nhtile_cls);
    d.ntc16 = (int)tc16.size();
    d.ntc32 = (int)tc32.size();
    d.ntc64 = (int)tc64.size();
    std::vector<LadderTile> tct;
    tct.insert(tct.end(), tc16.begin(), tc16.end());
    tct.insert(tct.end(), tc32.begin(), tc32.end());
    tct.insert(tct.end(), tc64.begin(), tc64.end());
    std::vector<TcTileDev> tcx;
    tcx.insert(tcx.end(), tcx16.begin(), tcx16.end());
    tcx.insert(tcx.end(), tcx32.begin(), tcx32.end());
    tcx.insert(tcx.end(), tcx64.begin(), tcx64.end());
    d.nwslabs = (int)wslabs.size();
    d.ndtiles = (int)dtiles.size();
    d.w16_n = w16_n;
    d.d16_n = d16_n;
    d.nscale = nscale;
    d.nchunks = (int)chunks.size();
    d.nhchunks = (int)hchunks.size();
    d.nrchunks = (int)rchunks.size();
    d.ntargets = (int)targets.size();
    d.max_o = max_o;
    d.max_v = max_v;
    if (ladder_smem_bytes(max_v, 32) > 227 * 1024) return fail(UEGCCD_ERR_UNSUPPORTED, "ladder block exceeds shared memory");
    set_ladder_smem_limit(max_v);
    {   // the |q|^2 table the mosaic kernel stages: the batch's largest (tables beyond 1024
        // entries stay in global memory)
        int q2m = 0;
        for (const auto &P : b->plans) q2m = std::max(q2m, P.q2max);
        d.mosaic_vt = std::min(q2m + 1, kVtabSmemEntries);
    }
    d.mosaic_smem = mosaic_smem_bytes(max_v, max_o, d.mosaic_vt);
    if (d.mosaic_smem > 227 * 1024) return fail(UEGCCD_ERR_UNSUPPORTED, "mosaic block exceeds shared memory");
    set_mosaic_smem_limit(d.mosaic_smem);
    d.max_occ = max_occ;
    d.namp = amp0;
    // ring pairs by kernel class: k_rings (two shared-memory sizes), then k_rings_wide
    {
        auto cls_of = [&](const RingPairDev &r) {
            const size_t b = rings_dmma_smem_bytes(solves[r.solve].O, r.n1, r.n2, solves[r.solve].q2max);
            if (b > kRingSmemMax) return kRingClasses;
            const int rows = ((r.n1 + 7) & ~7) + ((r.n2 + 7) & ~7);
            for (int c = 0; c < kRingClasses; c++)
                if (rows <= kRingClassRows[c]) return c;
            return kRingClasses;
        };
        // stable counting sort by class
        std::vector<int> cls(rpairs.size());
        std::vector<size_t> start(kRingClasses + 2, 0);
        for (size_t k = 0; k < rpairs.size(); k++) start[(cls[k] = cls_of(rpairs[k])) + 1]++;
        for (int c = 0; c <= kRingClasses; c++) start[c + 1] += start[c];
        std::vector<RingPairDev> sorted(rpairs.size());
        for (size_t k = 0; k < rpairs.size(); k++) sorted[start[cls[k]]++] = rpairs[k];
        rpairs.swap(sorted);
        // each pair's rows in the particle-hole arrays, in launch order: group-1 row a holds
        // 2 round8(n2) doubles (a multiple of 16: every row starts 128-byte aligned)
        int64_t xy_n = 0;
        for (auto &r : rpairs) {
            r.xy0 = (int32_t)xy_n;
            xy_n += (int64_t)r.n1 * 2 * ((r.n2 + 7) & ~7);
            if (xy_n >= ((int64_t)1 << 31)) return fail(UEGCCD_ERR_ARG, "batch too large for 32-bit ring offsets");
        }
        d.xy_n = xy_n;
        // the staging kernel walks the pairs solve by solve (the class sort is stable, so a
        // stable sort by solve restores that order)
        spairs.assign(rpairs.begin(), rpairs.end());
        std::stable_sort(spairs.begin(), spairs.end(),
                         [](const RingPairDev &x, const RingPairDev &y) { return x.solve < y.solve; });
        for (const auto &r : rpairs) {
            const int c = cls_of(r);
            d.nring[c]++;
            const size_t b = c < kRingClasses
                                 ? rings_dmma_smem_bytes(solves[r.solve].O, r.n1, r.n2, solves[r.solve].q2max)
                                 : rings_smem_bytes(solves[r.solve].O, r.n1 + r.n2);
            d.ring_smem[c] = std::max(d.ring_smem[c], b);
        }
    }
    trace.mark("classes");
    d.nrpairs = (int)rpairs.size();
    if (d.ring_smem[kRingClasses] > 227 * 1024)
        return fail(UEGCCD_ERR_UNSUPPORTED, "ring group pair exceeds shared memory");
    set_rings_smem_limit(0, *std::max_element(d.ring_smem, d.ring_smem + kRingClasses));
    set_rings_smem_limit(1, d.ring_smem[kRingClasses]);
    trace.mark("host-tables");
    if ((rc = b->upload(d.solves, solves))) return rc;
    if ((rc = b->upload(d.blocks, blocks))) return rc;
    if ((rc = b->upload(d.tiles, tiles))) return rc;
    if ((rc = b->upload(d.htiles, htiles))) return rc;
    if ((rc = b->upload(d.tiles_lpt, tiles_lpt))) return rc;
    if ((rc = b->upload(d.htiles_lpt, htiles_lpt))) return rc;
    if ((rc = b->upload(d.tctiles, tct))) return rc;
    if ((rc = b->upload(d.tcx, tcx))) return rc;
    if ((rc = b->upload(d.wslabs, wslabs))) return rc;
    if ((rc = b->upload(d.dtiles, dtiles))) return rc;
    if ((rc = b->upload(d.chunks, chunks))) return rc;
    if ((rc = b->upload(d.rchunks, rchunks))) return rc;
    if ((rc = b->upload(d.chunk_begin, chunk_begin))) return rc;
    if ((rc = b->upload(d.hchunks, hchunks))) return rc;
    if ((rc = b->upload(d.hchunk_begin, hchunk_begin))) return rc;
    if ((rc = b->upload(d.targets, targets))) return rc;
    if ((rc = b->upload(d.pcol, pcol))) return rc;
    int *d_tbase = nullptr;
    int64_t *d_lbase = nullptr;
    if ((rc = b->upload(d_tbase, s_t0))) return rc;
    if ((rc = b->upload(d_lbase, mt_lbase))) return rc;
    if ((rc = b->alloc(d.mt_start, targets.size() + 1))) return rc;
    if ((rc = b->alloc(d.mt_list, (size_t)mt_lbase[n]))) return rc;
    if ((rc = b->alloc(d.mpart, mrows + mcols))) return rc;
    if ((rc = b->upload(d.pair_i, pair_i))) return rc;
    if ((rc = b->upload(d.pair_j, pair_j))) return rc;
    if ((rc = b->upload(d.vir, vir))) return rc;
    if ((rc = b->alloc(d.pos, pos0))) return rc;
    if ((rc = b->alloc(d.partner, amp0))) return rc;
    if ((rc = b->alloc(d.mirror, amp0))) return rc;
    if ((rc = b->alloc(d.amps, amp0))) return rc;
    if ((rc = b->upload(d.nv4, nv4))) return rc;
    if ((rc = b->upload(d.nvp, nvp))) return rc;
    if ((rc = b->upload(d.eigen, eigen))) return rc;
    if ((rc = b->upload(d.vtab, vtab))) return rc;
    b->vtab_base = vtab;
    if ((rc = b->upload(d.hh0, hh0))) return rc;
    if ((rc = b->upload(d.rpairs, rpairs))) return rc;
    if ((rc = b->upload(d.spairs, spairs))) return rc;
    if ((rc = b->upload(d.ph_i, ph_i))) return rc;
    if ((rc = b->upload(d.ph_x, ph_x))) return rc;
    if ((rc = b->alloc(d.ridx_x, ph0))) return rc;
    if ((rc = b->alloc(d.ridx_y, ph0))) return rc;
    if ((rc = b->alloc(d.vcoef, amp0))) return rc;
    if ((rc = b->alloc(d.xy, d.xy_n))) return rc;
    if ((rc = b->alloc(d.rx, d.xy_n))) return rc;
    if ((rc = b->alloc(d.ph_a, phr0))) return rc;
    if ((rc = b->alloc(d.ph_b, phr0))) return rc;
    if ((rc = b->alloc(d.rpos, amp0))) return rc;
    if ((rc = b->alloc(d.t, amp0))) return rc;
    if ((rc = b->alloc(d.t_new, amp0))) return rc;
    if ((rc = b->alloc(d.g, amp0))) return rc;
    if ((rc = b->alloc(d.jvv, jvv0))) return rc;
    if ((rc = b->alloc(d.joo, joo0))) return rc;
    d.ph_total = ph0;
    if ((rc = b->alloc(d.hh, hhoff))) return rc;
    const size_t npart = std::max(chunks.size(), hchunks.size());   // per full or half chunk
    if ((rc = b->alloc(d.part_e, npart))) return rc;
    if ((rc = b->alloc(d.part_dt, npart))) return rc;
    if ((rc = b->alloc(d.part_r, npart))) return rc;
    if ((rc = b->alloc(d.red, 3 * (size_t)n))) return rc;
    if ((rc = b->alloc(d.active, n))) return rc;
    b->hsolves = solves;
    b->chunk_begin = chunk_begin;
    b->red.assign(3 * (size_t)n, 0.0);
    b->active.assign(n, 1);
    CU(cudaMemcpyAsync(d.active, b->active.data(), n, cudaMemcpyHostToDevice, b->stream));
    trace.mark("alloc+upload");
    // position map, amplitude list, partners and ring gather indices, from the blocks
    CU(cudaMemsetAsync(d.pos, 0xff, (size_t)pos0 * sizeof(int32_t), b->stream));   // -1: not allowed
    CU(cudaMemsetAsync(d.ph_a, 0xff, (size_t)phr0 * sizeof(int32_t), b->stream));  // -1: no ring pair
    CU(cudaMemsetAsync(d.ph_b, 0xff, (size_t)phr0 * sizeof(int32_t), b->stream));
    CU(cudaMemsetAsync(d.xy, 0, (size_t)d.xy_n * sizeof(double), b->stream));      // padding columns stay 0

    launch_block_tables(d, b->stream);
    launch_mosaic_targets(d, d_tbase, d_lbase, (size_t)max_vo * sizeof(int), b->stream);
    launch_vcoef(d, b->stream);
    size_t dn = 0;
    for (int s = 0; s < n; s++) dn = std::max(dn, (size_t)b->plans[s].O * b->plans[s].O * b->plans[s].V);
    b->dense_n = dn;
    for (int k = 0; k < 3; k++)
        if ((rc = b->alloc(b->dense[k], dn))) return rc;
    trace.mark("device-launch");
    CU(cudaStreamSynchronize(b->stream));
    trace.mark("device-wait");
    out = std::move(b);
    return 0;
}

int set_active_all(UegccdBatch &b, uint8_t v)
{
    std::fill(b.active.begin(), b.active.end(), v);
    CU(cudaMemcpyAsync(b.d.active, b.active.data(), b.active.size(), cudaMemcpyHostToDevice, b.stream));
    b.h2d_bytes += (int64_t)b.active.size();
    return 0;
}

int read_red(UegccdBatch &b)
{
    CU(cudaMemcpyAsync(b.red.data(), b.d.red, b.red.size() * sizeof(double), cudaMemcpyDeviceToHost, b.stream));
    b.d2h_bytes += (int64_t)(b.red.size() * sizeof(double));
    CU(cudaStreamSynchronize(b.stream));
    CU(cudaGetLastError());
    b.kt.collect();
    return 0;
}

// Copies one solve's amplitudes from a host reference-layout array into the packed t.
int pack_from_host(UegccdBatch &b, int s, const double *host_dense)
{
    const SolvePlan &P = b.plans[s];
    size_t n = (size_t)P.O * P.O * P.V;
    CU(cudaMemcpyAsync(b.dense[0], host_dense, n * sizeof(double), cudaMemcpyHostToDevice, b.stream));
    b.h2d_bytes += (int64_t)(n * sizeof(double));
    launch_pack(b.d, s, (int)P.namp, b.dense[0], b.stream);
    b.launches++;
    CU(cudaGetLastError());
    return 0;
}

int unpack_to_host(UegccdBatch &b, int s, const double *t_dev, double *ab, double *ba, double *aa)
{
    const SolvePlan &P = b.plans[s];
    size_t n = (size_t)P.O * P.O * P.V;
    double *h[3] = {ab, ba, aa};
    for (int k = 0; k < 3; k++)
        if (h[k]) CU(cudaMemsetAsync(b.dense[k], 0, n * sizeof(double), b.stream));
    launch_unpack(b.d, s, (int)P.namp, t_dev, ab ? b.dense[0] : nullptr, ba ? b.dense[1] : nullptr,
                  aa ? b.dense[2] : nullptr, b.stream);
    b.launches++;
    CU(cudaGetLastError());
    for (int k = 0; k < 3; k++)
        if (h[k]) {
            CU(cudaMemcpyAsync(h[k], b.dense[k], n * sizeof(double), cudaMemcpyDeviceToHost, b.stream));
            b.d2h_bytes += (int64_t)(n * sizeof(double));
        }
    CU(cudaStreamSynchronize(b.stream));
    return 0;
}

// Integral options for every later call on the batch (SetPointers, Main.f90:274-318, with
// no range flags): GapII > 0 zeroes the integrals above GapII (GapERI, HEG.f90:938-940) --
// the |q|^2 tables are filtered; CoreN > 0 zeroes those with an index p <= CoreN
// (CoreERI, HEG.f90:882-885) -- the kernels hold core pairs at zero.  The per-amplitude
// Coulomb factors are rebuilt from the filtered tables.
// The |q|^2 tables of every solve for an ERI flag (CasedERI, HEG.f90:725-774; flag 0 is
// BaseERI's value), with the reference's "< 0 -> -100" guard and the GapII filter applied in
// its order.  CoreN is not in the tables: the kernels hold core pairs at zero.
std::vector<double> integral_tables(const UegccdBatch &b, int flag, double gapii)
{
    std::vector<double> vt;
    vt.reserve(b.vtab_base.size());
    for (size_t s = 0; s < b.plans.size(); s++) {
        const double L = b.sys[s].L, mad = b.sys[s].madelung, sd = b.screening;
        for (int q2 = 0; q2 <= b.plans[s].q2max; q2++) {
            double v = 0.0;
            if (flag == 0) {
                v = coulomb_v(L, mad, q2);
            } else if (q2 == 0) {
                if (flag == 1) v = (1.0 / std::pow(L, 3.0)) * 4.0 * kPi / std::pow(sd, 2.0);
                else if (flag == 2) v = -mad - (1.0 / std::pow(L, 3.0)) * 4.0 * kPi / std::pow(sd, 2.0);
            } else {
                const double q2s = (double)q2 * std::pow(2.0 * kPi / L, 2.0);
                if (flag == 1) v = (1.0 / std::pow(L, 3.0)) * 4.0 * kPi / (std::pow(sd, 2.0) + q2s);
                else if (flag == 2)
                    v = (1.0 / std::pow(L, 3.0)) * 4.0 * kPi / (std::pow(sd, 2.0) + q2s) * std::pow(sd, 2.0) / q2s;
            }
            if (flag != 0 && v < 0.0) v = -100.0;
            if (gapii > 0.0 && v > gapii) v = 0.0;
            vt.push_back(v);
        }
    }
    return vt;
}

// Uploads the tables of an ERI flag and the Coulomb factors that follow them.
int load_tables(UegccdBatch &b, int flag)
{
    const std::vector<double> vt = integral_tables(b, flag, b.gapii);
    CU(cudaMemcpyAsync(b.d.vtab, vt.data(), vt.size() * sizeof(double), cudaMemcpyHostToDevice, b.stream));
    launch_vcoef(b.d, b.stream);
    b.d.w16_valid = false;   // the FP16 Coulomb slabs follow the tables
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(b.stream));
    b.h2d_bytes += (int64_t)(vt.size() * sizeof(double));
    return 0;
}

int set_integrals(UegccdBatch &b, int core_n, double gapii)
{
    if (core_n < 0) return fail(UEGCCD_ERR_ARG, "CoreN must be >= 0");
    for (const auto &P : b.plans)
        if (core_n > P.O) return fail(UEGCCD_ERR_ARG, "CoreN exceeds NOcc");
    const double g = gapii > 0.0 ? gapii : 0.0;
    if (core_n == b.core_n && g == b.gapii) return 0;
    std::vector<double> vt(b.vtab_base);
    if (g > 0.0)
        for (auto &v : vt)
            if (v > g) v = 0.0;
    CU(cudaMemcpyAsync(b.d.vtab, vt.data(), vt.size() * sizeof(double), cudaMemcpyHostToDevice, b.stream));
    for (auto &S : b.hsolves) S.core_n = core_n;
    CU(cudaMemcpyAsync(b.d.solves, b.hsolves.data(), b.hsolves.size() * sizeof(SolveDev), cudaMemcpyHostToDevice,
                       b.stream));
    launch_vcoef(b.d, b.stream);
    b.d.w16_valid = false;   // the FP16 Coulomb slabs follow the tables
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(b.stream));
    b.h2d_bytes += (int64_t)(vt.size() * sizeof(double) + b.hsolves.size() * sizeof(SolveDev));
    b.core_n = core_n;
    b.gapii = g;
    return 0;
}

// Buffers of the mixed-precision ladder, on first use; the FP16 Coulomb slabs are (re)built
// whenever the integral tables changed since.
int mixed_alloc(UegccdBatch &b)
{
    DevBatch &d = b.d;
    int rc = 0;
    if (!d.t_ref) {
        if ((rc = b.alloc(d.t_ref, d.namp))) return rc;
        if ((rc = b.alloc(d.g_ref, d.namp))) return rc;
        if ((rc = b.alloc(d.tc_err, 1))) return rc;
        uint16_t *w = nullptr, *dd = nullptr;
        if ((rc = b.alloc(w, (size_t)d.w16_n))) return rc;
        if ((rc = b.alloc(dd, (size_t)d.d16_n))) return rc;
        if ((rc = b.alloc(d.dscale, (size_t)d.nscale))) return rc;
        d.w16 = w;
        d.d16 = dd;
    }
    if (!d.w16_valid) {
        launch_w16_build(d, b.stream);
        CU(cudaGetLastError());
        d.w16_valid = true;
    }
    return 0;
}

int validate_options(const UegccdOptions *o, int drpa, const UegccdBatch &b, bool two_channel = false)
{
    if (!o) return fail(UEGCCD_ERR_ARG, "null options");
    if (two_channel) {
        // the two-channel form takes its integrals from uegccd_ctx_set_eri, not range_flags
        if (o->precision != UEGCCD_FP64) return fail(UEGCCD_ERR_UNSUPPORTED, "the two-channel form runs in FP64");
    } else {
        if (o->range_flags != 0 && drpa)
            return fail(UEGCCD_ERR_UNSUPPORTED,
                        "range-separated dRPA takes per-term flags: uegccd_ctx_set_eri on a context");
        if (o->range_flags != 0 && b.range_flag == 0)
            return fail(UEGCCD_ERR_UNSUPPORTED,
                        "range-separated integrals: set one flag for every term with uegccd_*_set_range, or "
                        "per-term flags with uegccd_ctx_set_eri on a context");
        if (!drpa && (o->do_ring != 0) != (o->do_xring != 0))
            return fail(UEGCCD_ERR_UNSUPPORTED,
                        "Do Rings and Do XRings must agree in a batch solve: alone, either breaks the spin "
                        "symmetry of the batched kernels (a context's uegccd_ccd runs the two-channel form)");
    }
    if (o->max_iter <= 0 || !(o->tol > 0) || !(o->denom_factor != 0)) return fail(UEGCCD_ERR_ARG, "bad iteration options");
    if (o->scheme != UEGCCD_REPLAY && o->scheme != UEGCCD_DIIS) return fail(UEGCCD_ERR_ARG, "unknown scheme");
    if (o->scheme == UEGCCD_DIIS && (o->ndiis < 2 || o->ndiis > kDiisMax))
        return fail(UEGCCD_ERR_ARG, "ndiis must be in [2, 16]");
    if (o->precision != UEGCCD_FP64 && o->precision != UEGCCD_MIXED) return fail(UEGCCD_ERR_ARG, "unknown precision");
    return 0;
}

// Buffers of the device-side iteration control, grown on demand.  Each group of arrays is
// allocated as a whole: when one of them fails, the group's memory goes back and the batch
// keeps what it had.
int ctl_alloc(UegccdBatch &b, int ndiis, int max_rec)
{
    CtlBuffers &c = b.ctl;
    const int n = b.d.nsolves;
    int rc = 0;
    if (!c.state) {
        const UegccdBatch::Mark m = b.mark();
        CtlBuffers x = c;
        if ((rc = b.alloc(x.state, n)) || (rc = b.alloc(x.active_next, n)) || (rc = b.alloc(x.count, 1)) ||
            (rc = b.alloc(x.Bm, (size_t)n * kDiisMax * kDiisMax)) || (rc = b.alloc(x.coef, (size_t)n * kDiisMax)) ||
            (rc = b.alloc(x.brow, (size_t)n * kDiisMax)) || (rc = b.alloc(x.part, (size_t)b.d.nhchunks * kDiisMax))) {
            b.rollback(m);
            return rc;
        }
        c = x;
    }
    if (max_rec > c.max_rec) {
        const UegccdBatch::Mark m = b.mark();
        double *re = nullptr, *rd = nullptr;
        if ((rc = b.alloc(re, (size_t)n * max_rec)) || (rc = b.alloc(rd, (size_t)n * max_rec))) {
            b.rollback(m);
            return rc;
        }
        c.rec_e = re;
        c.rec_dt = rd;
        c.max_rec = max_rec;
    }
    if (ndiis > b.diis_cap) {
        const UegccdBatch::Mark m = b.mark();
        double *ht = nullptr;
        float *he = nullptr;
        if ((rc = b.alloc(ht, (size_t)ndiis * b.d.namp)) || (rc = b.alloc(he, (size_t)ndiis * b.d.namp))) {
            b.rollback(m);
            return rc;
        }
        c.hist_t = ht;
        c.hist_e = he;
        b.diis_cap = ndiis;
    }
    return 0;
}

// Captures one iteration as a CUDA graph.
int capture_iteration(UegccdBatch &b, const TermFlags &f, double tol, int max_iter, int ndiis)
{
    UegccdBatch::GraphKey key{f.do_ring, f.do_xring, f.do_ladder, f.do_mosaic, f.drpa, ndiis, max_iter, f.mixed, tol};
    if (b.have_graph && b.gkey == key) return 0;
    if (b.gexec) { cudaGraphExecDestroy(b.gexec); b.gexec = nullptr; }
    cudaGraph_t g = nullptr;
    CU(cudaStreamBeginCapture(b.stream, cudaStreamCaptureModeThreadLocal));
    int nl = launch_iteration(b.d, b.ctl, f, tol, max_iter, ndiis, b.stream, nullptr);
    cudaError_t e = cudaStreamEndCapture(b.stream, &g);
    if (e != cudaSuccess) return fail(UEGCCD_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b.gexec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(UEGCCD_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    b.g_launches = nl;
    b.gkey = key;
    b.have_graph = true;
    return 0;
}

// The launch shapes of a batch (k_rings CTA sizes, k_ring_stage CTA size, ladder tile
// order): measured once per batch shape in this process (the shape: pair count and shared
// memory of every ring class, ladder tiles per class, largest block), on the first CCD
// solve, before the iteration graph is captured.
std::mutex g_tune_mu;
std::map<std::vector<int64_t>, std::array<int, kRingClasses + 3>> g_ring_tuning;

int tune_batch_rings(UegccdBatch &b)
{
    DevBatch &d = b.d;
    std::vector<int64_t> key;
    for (int c = 0; c <= kRingClasses; c++) {
        key.push_back(d.nring[c]);
        key.push_back((int64_t)d.ring_smem[c]);
    }
    for (int c = 0; c < kLadderClasses; c++) {
        key.push_back(d.ntile_cls[c]);
        key.push_back(d.nhtile_cls[c]);
    }
    key.push_back(d.max_v);
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_ring_tuning.find(key);
        if (it != g_ring_tuning.end()) {
            for (int c = 0; c < kRingClasses; c++) d.ring_threads[c] = it->second[c];
            d.stage_threads = it->second[kRingClasses];
            d.ladder_sched = it->second[kRingClasses + 1];
            d.hh_kc = it->second[kRingClasses + 2];
            b.rings_tuned = true;
            return 0;
        }
    }
    const int e = tune_rings(d, b.stream);
    if (e != 0) return fail(UEGCCD_ERR_CUDA, std::string("launch-shape tuning: ") + cudaGetErrorString((cudaError_t)e));
    std::array<int, kRingClasses + 3> th;
    for (int c = 0; c < kRingClasses; c++) th[c] = d.ring_threads[c];
    th[kRingClasses] = d.stage_threads;
    th[kRingClasses + 1] = d.ladder_sched;
    th[kRingClasses + 2] = d.hh_kc;
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_ring_tuning[key] = th;
    b.rings_tuned = true;
    return 0;
}

// Runs the iteration for all solves of the batch from the amplitudes in d.t.
// Iteration control lives on the device; the host replays a captured iteration
// graph kPoll times between polls of the number of active solves.  With kernel
// timing on, the last iteration of each round runs as direct launches between
// CUDA events: that iteration is the sample the per-kernel times come from.
int run_solves(UegccdBatch &b, const UegccdOptions *opt, int drpa, UegccdResult *res)
{
    constexpr int kPoll = 4;
    DevBatch &d = b.d;
    const int n = d.nsolves;
    TermFlags f;
    f.drpa = drpa;
    f.do_driver = 1;
    f.do_mosaic = opt->do_mosaic ? 1 : 0;
    f.do_ladder = (!drpa && opt->do_ladder) ? 1 : 0;
    f.do_ring = opt->do_ring ? 1 : 0;
    f.do_xring = (!drpa && opt->do_xring) ? 1 : 0;
    // range-separated integrals: every CCD term and the energy on the flag's tables (the MP2
    // start before this used the plain ones); the plain tables back on every exit
    struct TableGuard {
        UegccdBatch &b;
        bool on;
        ~TableGuard()
        {
            // a batch left on the range-separated tables would give wrong MP2 and CCD results
            // later: refuse every further call on it instead
            if (on && load_tables(b, 0) != 0) b.broken = true;
        }
    } table_guard{b, false};
    if (opt->range_flags != 0 && b.range_flag != 0) {
        const int rc0 = load_tables(b, b.range_flag);
        if (rc0) return rc0;
        table_guard.on = true;
    }
    const int max_rec = std::min(opt->max_iter, 1100);
    // The DIIS history takes fewer vectors when the device memory (or the library's limit)
    // does not hold ndiis of them, down to 2, as SetUpDIISCC steps Max_N_DIIS down until its
    // Allocate succeeds (DIISCC.f90:22-29); the vectors used are reported per solve.
    int ndiis = opt->scheme == UEGCCD_DIIS ? opt->ndiis : 0;
    int rc = 0;
    while ((rc = ctl_alloc(b, ndiis, max_rec)) == UEGCCD_ERR_ALLOC && ndiis > 2) ndiis--;
    if (rc) return rc;
    for (int s = 0; s < n; s++) b.hsolves[s].denom_factor = opt->denom_factor;
    CU(cudaMemcpyAsync(d.solves, b.hsolves.data(), n * sizeof(SolveDev), cudaMemcpyHostToDevice, b.stream));
    std::vector<IterState> st0(n, IterState{1, 0, 0.0, 0.0});
    CU(cudaMemcpyAsync(b.ctl.state, st0.data(), n * sizeof(IterState), cudaMemcpyHostToDevice, b.stream));
    CU(cudaMemsetAsync(b.ctl.Bm, 0, (size_t)n * kDiisMax * kDiisMax * sizeof(double), b.stream));
    if ((rc = set_active_all(b, 1))) return rc;
    if (opt->precision == UEGCCD_MIXED && (rc = mixed_alloc(b))) return rc;
    if (drpa && !d.J1 && (rc = b.alloc(d.J1, (size_t)d.ph_total))) return rc;
    if (d.tc_err) CU(cudaMemsetAsync(d.tc_err, 0, sizeof(int), b.stream));
    if (!b.rings_tuned && !drpa && (f.do_ring || f.do_xring) && (rc = tune_batch_rings(b))) return rc;
    b.launches = 0;
    CU(cudaEventRecord(b.ev0, b.stream));
    // CCEnergy of the start amplitudes and dT = max|T| (CCD.f90:63-64, dRPA.f90:68-69)
    launch_energy(d, drpa ? 1 : 0, 0.0, b.stream);
    launch_reduce(d, b.stream);
    launch_control(d, b.ctl, opt->tol, opt->max_iter, ndiis, 1, b.stream);
    launch_active_swap(d, b.ctl, b.stream);
    b.launches += 4;
    int count = n, rounds = 0;
    const int max_rounds = opt->max_iter / kPoll + 2;
    // mixed precision: tensor-core ladder of t - t_ref, t_ref refreshed (FP64) each round,
    // then FP64 iterations from where the mixed phase stopped (refinement)
    const bool mixed = opt->precision == UEGCCD_MIXED && f.do_ladder && f.do_pp;
    for (int phase = mixed ? 0 : 1; phase < 2; phase++) {
        f.mixed = phase == 0 ? 1 : 0;
        if (phase == 1 && mixed) {
            // reopen every solve for the FP64 sweeps
            std::vector<IterState> st1(n);
            CU(cudaMemcpyAsync(st1.data(), b.ctl.state, n * sizeof(IterState), cudaMemcpyDeviceToHost, b.stream));
            CU(cudaStreamSynchronize(b.stream));
            for (auto &x : st1) x.status = 0;
            CU(cudaMemcpyAsync(b.ctl.state, st1.data(), n * sizeof(IterState), cudaMemcpyHostToDevice, b.stream));
            if ((rc = set_active_all(b, 1))) return rc;
            count = n;
            rounds = 0;
        }
        if ((rc = capture_iteration(b, f, opt->tol, opt->max_iter, ndiis))) return rc;
        int sweeps = 0;
        while (count > 0 && rounds < max_rounds) {
            if (f.mixed) {
                launch_refresh(d, b.stream);
                b.launches += 2;
            }
            for (int k = 0; k < kPoll; k++) {
                if (b.kt.on && k == kPoll - 1) {
                    // the sampled iteration of the round: direct launches between CUDA events
                    b.launches += launch_iteration(d, b.ctl, f, opt->tol, opt->max_iter, ndiis, b.stream, &b.kt);
                } else {
                    CU(cudaGraphLaunch(b.gexec, b.stream));
                    b.launches += b.g_launches;
                }
            }
            CU(cudaMemcpyAsync(&count, b.ctl.count, sizeof(int), cudaMemcpyDeviceToHost, b.stream));
            b.d2h_bytes += sizeof(int);
            CU(cudaStreamSynchronize(b.stream));
            CU(cudaGetLastError());
            b.kt.collect();
            rounds++;
            if (phase == 1 && mixed && ++sweeps >= std::max(1, opt->refine_sweeps)) break;
        }
    }
    if (mixed) {
        int err = 0;
        CU(cudaMemcpyAsync(&err, d.tc_err, sizeof(int), cudaMemcpyDeviceToHost, b.stream));
        CU(cudaStreamSynchronize(b.stream));
        if (err) return fail(UEGCCD_ERR_CUDA, "tensor-core ladder: an mbarrier wait expired");
    }
    // final residual (CCD.f90:103-107, dRPA.f90:98-101)
    if ((rc = set_active_all(b, 1))) return rc;
    b.launches += launch_residual(d, f, 1, nullptr, b.stream, &b.kt);
    if ((rc = read_red(b))) return rc;
    std::vector<double> rmax(n), esosex(n, 0.0);
    for (int s = 0; s < n; s++) rmax[s] = b.red[3 * s + 2];
    if (drpa) {
        launch_energy(d, 1, 1.0, b.stream);
        launch_reduce(d, b.stream);
        b.launches += 2;
        if ((rc = read_red(b))) return rc;
        for (int s = 0; s < n; s++) esosex[s] = b.red[3 * s];
    }
    std::vector<IterState> st(n);
    CU(cudaMemcpyAsync(st.data(), b.ctl.state, n * sizeof(IterState), cudaMemcpyDeviceToHost, b.stream));
    int nrec = 0;
    if (opt->max_rec > 0 && (opt->energies || opt->dts)) {
        nrec = std::min(std::min(st[0].niter, max_rec), opt->max_rec);
        std::vector<double> re(nrec), rd(nrec);
        CU(cudaMemcpyAsync(re.data(), b.ctl.rec_e, nrec * sizeof(double), cudaMemcpyDeviceToHost, b.stream));
        CU(cudaMemcpyAsync(rd.data(), b.ctl.rec_dt, nrec * sizeof(double), cudaMemcpyDeviceToHost, b.stream));
        CU(cudaStreamSynchronize(b.stream));
        for (int k = 0; k < nrec; k++) {
            if (opt->energies) opt->energies[k] = re[k];
            if (opt->dts) opt->dts[k] = rd[k];
        }
    }
    CU(cudaEventRecord(b.ev1, b.stream));
    CU(cudaEventSynchronize(b.ev1));
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, b.ev0, b.ev1));
    int status = 0;
    b.last_niter.assign(n, 0);
    for (int s = 0; s < n; s++) b.last_niter[s] = std::min(st[s].niter, max_rec);
    for (int s = 0; s < n; s++) {
        UegccdResult &r = res[s];
        r.ecorr = st[s].e;
        r.max_res = rmax[s];
        r.last_dt = st[s].dt;
        r.niter = st[s].niter;
        r.fail = rmax[s] > opt->fail_ratio * opt->tol;
        r.ecorr_sosex = (drpa && !r.fail) ? esosex[s] : 0.0;
        r.n_recorded = (s == 0) ? nrec : 0;
        r.kernel_launches = b.launches;
        r.gpu_ms = ms;
        r.status = st[s].status == 3 ? UEGCCD_ERR_NUMERIC
                   : (r.fail || st[s].status == 2) ? UEGCCD_NOT_CONVERGED : UEGCCD_OK;
        r.ndiis = ndiis;
        if (r.status == UEGCCD_ERR_NUMERIC) status = UEGCCD_ERR_NUMERIC;
        if (status == 0 && r.status == UEGCCD_NOT_CONVERGED) status = UEGCCD_NOT_CONVERGED;
    }
    if (status == UEGCCD_ERR_NUMERIC) fail(status, "non-finite amplitudes or energy");
    return status;
}

// Opens an incremental solve: the set-up of run_solves (control buffers with the DIIS depth
// step-down, start energy and state, the iteration graph), after the MP2 start.
int session_start(UegccdBatch &b, const UegccdOptions *opt, int drpa)
{
    DevBatch &d = b.d;
    const int n = d.nsolves;
    auto &S = b.ses;
    S = UegccdBatch::Session{};
    TermFlags &f = S.f;
    f.drpa = drpa;
    f.do_driver = 1;
    f.do_mosaic = opt->do_mosaic ? 1 : 0;
    f.do_ladder = (!drpa && opt->do_ladder) ? 1 : 0;
    f.do_ring = opt->do_ring ? 1 : 0;
    f.do_xring = (!drpa && opt->do_xring) ? 1 : 0;
    f.mixed = 0;
    S.max_rec = std::min(opt->max_iter, 1100);
    int ndiis = opt->scheme == UEGCCD_DIIS ? opt->ndiis : 0;
    int rc = 0;
    while ((rc = ctl_alloc(b, ndiis, S.max_rec)) == UEGCCD_ERR_ALLOC && ndiis > 2) ndiis--;
    if (rc) return rc;
    for (int s = 0; s < n; s++) b.hsolves[s].denom_factor = opt->denom_factor;
    CU(cudaMemcpyAsync(d.solves, b.hsolves.data(), n * sizeof(SolveDev), cudaMemcpyHostToDevice, b.stream));
    std::vector<IterState> st0(n, IterState{1, 0, 0.0, 0.0});
    CU(cudaMemcpyAsync(b.ctl.state, st0.data(), n * sizeof(IterState), cudaMemcpyHostToDevice, b.stream));
    CU(cudaMemsetAsync(b.ctl.Bm, 0, (size_t)n * kDiisMax * kDiisMax * sizeof(double), b.stream));
    if ((rc = set_active_all(b, 1))) return rc;
    if (drpa && !d.J1 && (rc = b.alloc(d.J1, (size_t)d.ph_total))) return rc;
    if (!b.rings_tuned && !drpa && (f.do_ring || f.do_xring) && (rc = tune_batch_rings(b))) return rc;
    launch_energy(d, drpa ? 1 : 0, 0.0, b.stream);
    launch_reduce(d, b.stream);
    launch_control(d, b.ctl, opt->tol, opt->max_iter, ndiis, 1, b.stream);
    launch_active_swap(d, b.ctl, b.stream);
    b.launches += 4;
    if ((rc = capture_iteration(b, f, opt->tol, opt->max_iter, ndiis))) return rc;
    CU(cudaStreamSynchronize(b.stream));
    S.opt = *opt;
    S.drpa = drpa;
    S.ndiis = ndiis;
    S.released.assign(n, 0);
    S.on = true;
    return 0;
}

// Up to `rounds` poll rounds of the open incremental solve, then the results of every solve
// that stopped since the last call: their final residual (MaxRes, CCD.f90:103-107) is formed
// with only them active, after which the still-running solves are active again.
int session_advance(UegccdBatch &b, int rounds, int *n_active, int *n_done, int *ids, UegccdResult *res)
{
    constexpr int kPoll = 4;
    DevBatch &d = b.d;
    auto &S = b.ses;
    const int n = d.nsolves;
    const UegccdOptions &opt = S.opt;
    int count = 0;
    CU(cudaMemcpyAsync(&count, b.ctl.count, sizeof(int), cudaMemcpyDeviceToHost, b.stream));
    CU(cudaStreamSynchronize(b.stream));
    for (int r = 0; r < rounds && count > 0; r++) {
        for (int k = 0; k < kPoll; k++) {
            CU(cudaGraphLaunch(b.gexec, b.stream));
            b.launches += b.g_launches;
        }
        CU(cudaMemcpyAsync(&count, b.ctl.count, sizeof(int), cudaMemcpyDeviceToHost, b.stream));
        b.d2h_bytes += sizeof(int);
        CU(cudaStreamSynchronize(b.stream));
        CU(cudaGetLastError());
    }
    std::vector<IterState> st(n);
    CU(cudaMemcpyAsync(st.data(), b.ctl.state, n * sizeof(IterState), cudaMemcpyDeviceToHost, b.stream));
    CU(cudaStreamSynchronize(b.stream));
    std::vector<int> fresh;
    for (int s = 0; s < n; s++)
        if (st[s].status != 0 && !S.released[s]) fresh.push_back(s);
    *n_done = (int)fresh.size();
    int running = 0;
    for (int s = 0; s < n; s++) running += st[s].status == 0;
    *n_active = running;
    if (!fresh.empty()) {
        std::fill(b.active.begin(), b.active.end(), 0);
        for (int s : fresh) b.active[s] = 1;
        CU(cudaMemcpyAsync(d.active, b.active.data(), n, cudaMemcpyHostToDevice, b.stream));
        b.h2d_bytes += n;
        b.launches += launch_residual(d, S.f, 1, nullptr, b.stream, nullptr);
        int rc = read_red(b);
        if (rc) return rc;
        std::vector<double> rmax(n), esosex(n, 0.0);
        for (int s = 0; s < n; s++) rmax[s] = b.red[3 * s + 2];
        if (S.drpa) {
            launch_energy(d, 1, 1.0, b.stream);
            launch_reduce(d, b.stream);
            b.launches += 2;
            if ((rc = read_red(b))) return rc;
            for (int s = 0; s < n; s++) esosex[s] = b.red[3 * s];
        }
        for (size_t k = 0; k < fresh.size(); k++) {
            const int s = fresh[k];
            UegccdResult &r = res[k];
            std::memset(&r, 0, sizeof r);
            ids[k] = s;
            r.ecorr = st[s].e;
            r.max_res = rmax[s];
            r.last_dt = st[s].dt;
            r.niter = st[s].niter;
            r.fail = rmax[s] > opt.fail_ratio * opt.tol;
            r.ecorr_sosex = (S.drpa && !r.fail) ? esosex[s] : 0.0;
            r.kernel_launches = b.launches;
            r.status = st[s].status == 3 ? UEGCCD_ERR_NUMERIC
                       : (r.fail || st[s].status == 2) ? UEGCCD_NOT_CONVERGED : UEGCCD_OK;
            r.ndiis = S.ndiis;
            S.released[s] = 1;
        }
        for (int s = 0; s < n; s++) b.active[s] = st[s].status == 0 ? 1 : 0;
        CU(cudaMemcpyAsync(d.active, b.active.data(), n, cudaMemcpyHostToDevice, b.stream));
        b.h2d_bytes += n;
        CU(cudaStreamSynchronize(b.stream));
    }
    if (running == 0) S.on = false;
    return 0;
}

}  // namespace

namespace uegccd {
// The message uegccd_last_error returns, for entry points defined in other files.
int set_last_error(int code, const char *msg) { return fail(code, msg); }
// 0 when a compute-capability-10 device is current, else an error status (message set).
int device_ok() { return check_device(); }
}  // namespace uegccd

// SendForAllocation (HEG.f90:1051-1065): SfLength = maxval(nVec)*2+1
int sf_length(const SystemHost &h)
{
    int m = h.n.empty() ? 0 : h.n[0][0];
    for (const auto &v : h.n) m = std::max(m, std::max(v[0], std::max(v[1], v[2])));
    return m * 2 + 1;
}

// Structure factors of solve s from the batch's amplitudes: the sums on the device
// (k_sf), then SfG and SfV -- functions of q alone -- at the points the sums reached,
// with the reference's expressions: SfG = (|q|^2 (2 pi/L)^2)**0.5 (dK2scaled,
// HEG.f90:1011-1031), SfV = the integral of the last contribution in the reference's
// loop order: BaseERI (HEG.f90:969-976) with the GapII filter, 0 for a core pair.
int structure_factor(UegccdBatch &b, int s, const UegccdSfGrid &out)
{
    DevBatch &d = b.d;
    const int n = d.nsolves;
    int rc = 0;
    if (!b.sf_groups) {
        std::vector<int2> g;
        b.sf_g0.assign(n + 1, 0);
        int64_t w3max = 1;
        for (int k = 0; k < n; k++) {
            for (const auto &G : b.plans[k].groups) g.push_back(make_int2(G.r0, G.n));
            b.sf_g0[k + 1] = (int)g.size();
            const int64_t w = 2 * sf_length(b.sys[k]) + 1;
            w3max = std::max(w3max, w * w * w);
        }
        if ((rc = b.upload(b.sf_groups, g))) return rc;
        if ((rc = b.alloc(b.sf_grid, 5 * (size_t)w3max))) return rc;
        if ((rc = b.alloc(b.sf_err, 1))) return rc;

    }
    const SystemHost &H = b.sys[s];
    const int S = sf_length(H);
    const int64_t W = 2 * S + 1, W3 = W * W * W;
    CU(cudaMemsetAsync(b.sf_grid, 0, 5 * (size_t)W3 * sizeof(double), b.stream));
    CU(cudaMemsetAsync(b.sf_err, 0, sizeof(int), b.stream));
    launch_sf(d, b.sf_groups + b.sf_g0[s], b.sf_g0[s + 1] - b.sf_g0[s], s, S, b.sf_grid, b.sf_err, b.stream);
    b.launches++;
    CU(cudaGetLastError());
    double *dst[3] = {out.sum, out.dsum, out.xsum};
    for (int k = 0; k < 3; k++)
        if (dst[k]) CU(cudaMemcpyAsync(dst[k], b.sf_grid + k * W3, W3 * sizeof(double), cudaMemcpyDeviceToHost, b.stream));
    // contributions, and where the last one is a core pair (read under CoreN only)
    const int ntail = b.core_n > 0 ? 2 : 1;
    std::vector<double> cnt((size_t)ntail * W3);
    CU(cudaMemcpyAsync(cnt.data(), b.sf_grid + 3 * W3, ntail * W3 * sizeof(double), cudaMemcpyDeviceToHost,
                       b.stream));
    int err = 0;
    CU(cudaMemcpyAsync(&err, b.sf_err, sizeof(int), cudaMemcpyDeviceToHost, b.stream));
    CU(cudaStreamSynchronize(b.stream));
    b.d2h_bytes += (int64_t)((3 + ntail) * W3 * sizeof(double));
    if (err) return fail(UEGCCD_ERR_ARG, "a momentum transfer falls outside the structure-factor grid");
    const double c = 2.0 * kPi / H.L, scale = c * c;
    for (int64_t z = 0; z < W; z++)
        for (int64_t y = 0; y < W; y++)
            for (int64_t x = 0; x < W; x++) {
                const int64_t k = x + W * (y + W * z);
                double g = 0.0, v = 0.0;
                if (cnt[k] > 0.0) {
                    const int q2 = (int)((x - S) * (x - S) + (y - S) * (y - S) + (z - S) * (z - S));
                    g = std::pow((double)q2 * scale, 0.5);
                    v = coulomb_v(H.L, H.madelung, q2);
                    if (b.gapii > 0.0 && v > b.gapii) v = 0.0;        // GapERI
                    if (ntail == 2 && cnt[W3 + k] != 0.0) v = 0.0;    // CoreERI of the last pair
                }
                if (out.g) out.g[k] = g;
                if (out.v) out.v[k] = v;
            }
    return UEGCCD_OK;
}

// Every call on a batch or context runs on the device the object was created on (whatever
// device the calling thread has current), and is refused once the batch is unusable.
// The two-channel state of a context, made on first use in the context's batch memory, with
// the integrals of the context's selection (uegccd_ctx_set_eri; none: SetPointers without
// range flags) for CoreN and GapII.
// A two-channel state for system s of a batch, its device memory carved from the batch's.
int make_two_channel(UegccdBatch &b, int s, std::unique_ptr<uegccd::TwoChannel> &out)
{
    struct Arena {
        UegccdBatch *b;
        UegccdBatch::Mark m;
    };
    auto ar = std::make_shared<Arena>(Arena{&b, b.mark()});
    uegccd::TcAlloc al;
    al.get = [ar](void **p, size_t bytes) {
        char *q = nullptr;
        const int rc = ar->b->alloc(q, bytes);
        *p = q;
        return rc;
    };
    al.begin = [ar]() { ar->m = ar->b->mark(); };
    al.rollback = [ar]() { ar->b->rollback(ar->m); };
    auto tc = std::make_unique<uegccd::TwoChannel>();
    const int rc = tc->init(b.sys[s], b.stream, al);
    if (rc) return rc;
    out = std::move(tc);
    return 0;
}

int two_channel_ready(UegccdCtx &c, int core_n, double gapii)
{
    if (!c.tc) {
        const int rc = make_two_channel(*c.batch, 0, c.tc);
        if (rc) return rc;
    }
    UegccdRangeTerms none{};
    const UegccdRangeTerms &fl = c.eri_set ? c.flags : none;
    const int safe = c.eri_set ? c.safe_eri : 0;
    const int routine = uegccd::tc_pick_routine(fl, safe, core_n, gapii);
    return c.tc->set_integrals(routine, fl, core_n, gapii, c.screening);
}

// A batch CCD solve in the two-channel form (do_ring != do_xring): every system in turn from its
// MP2 amplitudes, on a two-channel state of its own; the integrals of the batch's options (and
// its uniform range flag, as CasedERI applies it).  The batch keeps each solve's T2abab (what
// uegccd_batch_get_amplitudes reads) and its iteration table (uegccd_batch_history).
int run_two_channel_solves(UegccdBatch &b, const UegccdOptions *opt, UegccdResult *res)
{
    const int n = b.d.nsolves;
    if (b.tcs.size() != (size_t)n) b.tcs.resize(n);
    b.tc_en.assign(n, {});
    b.tc_dt.assign(n, {});
    UegccdRangeTerms flags{};
    int routine = uegccd::tc_pick_routine(flags, 0, opt->core_n, opt->gapii);
    if (opt->range_flags != 0) {
        int32_t *p = &flags.ring;
        for (int k = 0; k < 15; k++) p[k] = b.range_flag;
        routine = uegccd::TC_CASED;
    }
    const int max_rec = std::min(opt->max_iter, 1100);
    int status = 0;
    for (int s = 0; s < n; s++) {
        const SystemHost &H = b.sys[s];
        const size_t na = (size_t)H.O * H.O * (H.M - H.O);
        std::vector<double> aa(na), ab(na), ba(na);
        int rc = unpack_to_host(b, s, b.d.t, ab.data(), ba.data(), aa.data());
        if (rc) return rc;
        if (!b.tcs[s] && (rc = make_two_channel(b, s, b.tcs[s]))) return rc;
        if ((rc = b.tcs[s]->set_integrals(routine, flags, opt->core_n, opt->gapii, b.screening))) return rc;
        UegccdOptions o = *opt;
        b.tc_en[s].assign(max_rec, 0.0);
        b.tc_dt[s].assign(max_rec, 0.0);
        o.energies = b.tc_en[s].data();
        o.dts = b.tc_dt[s].data();
        o.max_rec = max_rec;
        rc = b.tcs[s]->solve(o, false, H.eigen, aa.data(), ab.data(), ba.data(), res[s]);
        if (rc < 0 && rc != UEGCCD_ERR_NUMERIC) return rc;
        b.tc_en[s].resize(res[s].n_recorded);
        b.tc_dt[s].resize(res[s].n_recorded);
        // the caller's arrays receive solve 0's table, as run_solves gives them
        if (s == 0 && opt->max_rec > 0) {
            const int k = std::min(res[s].n_recorded, opt->max_rec);
            if (opt->energies) std::copy(b.tc_en[s].begin(), b.tc_en[s].begin() + k, opt->energies);
            if (opt->dts) std::copy(b.tc_dt[s].begin(), b.tc_dt[s].begin() + k, opt->dts);
            res[s].n_recorded = k;
        } else {
            res[s].n_recorded = 0;
        }
        if ((rc = pack_from_host(b, s, ab.data()))) return rc;
        if (res[s].status == UEGCCD_ERR_NUMERIC) status = UEGCCD_ERR_NUMERIC;
        if (status == 0 && res[s].status == UEGCCD_NOT_CONVERGED) status = UEGCCD_NOT_CONVERGED;
    }
    b.two_channel_amps = true;
    if (status == UEGCCD_ERR_NUMERIC) fail(status, "non-finite amplitudes or energy");
    return status;
}

#define ENTER_DEVICE(bp)                                                                               \
    DeviceScope dev_scope_((bp)->dev);                                                                 \
    if (dev_scope_.rc != cudaSuccess)                                                                  \
        return fail(UEGCCD_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(dev_scope_.rc))
#define ENTER(bp)                                                                                      \
    ENTER_DEVICE(bp);                                                                                  \
    if ((bp)->broken) return fail(UEGCCD_ERR_CUDA, "batch unusable: restoring its plain integral tables failed")

extern "C" {

const char *uegccd_last_error(void) { return g_last_error.c_str(); }
const char *uegccd_version(void) { return "uegccd_b200 0.1 (sm_100a)"; }

void uegccd_default_options(UegccdOptions *o)
{
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->do_ring = o->do_xring = o->do_ladder = o->do_mosaic = 1;
    o->max_iter = 1000;
    o->tol = 1.0e-8;
    o->denom_factor = 2.0;
    o->fail_ratio = 100.0;
    o->scheme = UEGCCD_REPLAY;
    o->ndiis = 6;
    o->precision = UEGCCD_FP64;
    o->refine_sweeps = 2;
}

int uegccd_ctx_create(const UegccdSystem *sys, UegccdCtx **out)
{
    if (!out) return fail(UEGCCD_ERR_ARG, "null out");
    *out = nullptr;
    std::unique_ptr<UegccdBatch> b;
    int rc = build_batch(sys, 1, b);
    if (rc) return rc;
    auto *c = new UegccdCtx;
    c->batch = std::move(b);
    *out = c;
    return 0;
}

int uegccd_ctx_destroy(UegccdCtx *c)
{
    if (!c) return 0;
    ENTER_DEVICE(c->batch);
    delete c;
    return 0;
}

int uegccd_ctx_set_eigen(UegccdCtx *c, const double *eigen)
{
    if (!c || !eigen) return fail(UEGCCD_ERR_ARG, "null argument");
    ENTER(c->batch);
    UegccdBatch &b = *c->batch;
    b.sys[0].eigen.assign(eigen, eigen + b.sys[0].M);
    CU(cudaMemcpyAsync(b.d.eigen, eigen, b.sys[0].M * sizeof(double), cudaMemcpyHostToDevice, b.stream));
    CU(cudaStreamSynchronize(b.stream));
    return 0;
}

int set_range(UegccdBatch &b, int32_t flag, double screening)
{
    if (flag < 0 || flag > 3) return fail(UEGCCD_ERR_ARG, "range flag must be 0, 1, 2 or 3");
    if (flag != 0 && !(screening > 0.0)) return fail(UEGCCD_ERR_ARG, "screening distance must be > 0");
    b.range_flag = flag;
    b.screening = flag != 0 ? screening : 0.0;
    return 0;
}

int uegccd_ctx_set_range(UegccdCtx *c, int32_t flag, double screening)
{
    if (!c) return fail(UEGCCD_ERR_ARG, "null context");
    return set_range(*c->batch, flag, screening);
}

int uegccd_batch_set_range(UegccdBatch *b, int32_t flag, double screening)
{
    if (!b) return fail(UEGCCD_ERR_ARG, "null batch");
    return set_range(*b, flag, screening);
}

int uegccd_ctx_set_integrals(UegccdCtx *c, int32_t core_n, double gapii)
{
    if (!c) return fail(UEGCCD_ERR_ARG, "null context");
    ENTER(c->batch);
    return set_integrals(*c->batch, core_n, gapii);
}

int uegccd_batch_set_integrals(UegccdBatch *b, int32_t core_n, double gapii)
{
    if (!b) return fail(UEGCCD_ERR_ARG, "null batch");
    ENTER(b);
    return set_integrals(*b, core_n, gapii);
}

int uegccd_mp2(UegccdCtx *c, double *t_aaaa, double *t_abab, double *t_abba, double *e2)
{
    if (!c) return fail(UEGCCD_ERR_ARG, "null context");
    ENTER(c->batch);
    UegccdBatch &b = *c->batch;
    launch_mp2(b.d, b.stream);
    launch_reduce(b.d, b.stream);
    CU(cudaGetLastError());
    int rc = read_red(b);
    if (rc) return rc;
    if (e2) *e2 = b.red[0];
    if (t_aaaa || t_abab || t_abba) {
        rc = unpack_to_host(b, 0, b.d.t, t_abab, t_abba, t_aaaa);
        if (rc) return rc;
    }
    return std::isfinite(b.red[0]) ? 0 : fail(UEGCCD_ERR_NUMERIC, "non-finite MP2 energy");
}

int uegccd_ccd(UegccdCtx *c, const UegccdOptions *opt, double *t_aaaa, double *t_abab, double *t_abba,
               UegccdResult *res)
{
    if (!c || !t_abab || !res) return fail(UEGCCD_ERR_ARG, "null argument");
    ENTER(c->batch);
    UegccdBatch &b = *c->batch;
    const bool two = opt && (c->eri_set || (opt->do_ring != 0) != (opt->do_xring != 0));
    int rc = validate_options(opt, 0, b, two);
    if (rc) return rc;
    if ((rc = set_integrals(b, opt->core_n, opt->gapii))) return rc;
    if (two) {
        if ((rc = two_channel_ready(*c, opt->core_n, opt->gapii))) return rc;
        return c->tc->solve(*opt, false, b.sys[0].eigen, t_aaaa, t_abab, t_abba, *res);
    }
    if ((rc = pack_from_host(b, 0, t_abab))) return rc;
    int st = run_solves(b, opt, 0, res);
    if (st < 0) return st;
    if ((rc = unpack_to_host(b, 0, b.d.t, t_abab, t_abba, t_aaaa))) return rc;
    return st;
}

int uegccd_drpa(UegccdCtx *c, const UegccdOptions *opt, double *t2, UegccdResult *res)
{
    if (!c || !t2 || !res) return fail(UEGCCD_ERR_ARG, "null argument");
    ENTER(c->batch);
    UegccdBatch &b = *c->batch;
    int rc = validate_options(opt, 1, b, c->eri_set);
    if (rc) return rc;
    if ((rc = set_integrals(b, opt->core_n, opt->gapii))) return rc;
    if (c->eri_set) {
        if ((rc = two_channel_ready(*c, opt->core_n, opt->gapii))) return rc;
        return c->tc->solve(*opt, true, b.sys[0].eigen, nullptr, t2, nullptr, *res);
    }
    if ((rc = pack_from_host(b, 0, t2))) return rc;
    int st = run_solves(b, opt, 1, res);
    if (st < 0) return st;
    if ((rc = unpack_to_host(b, 0, b.d.t, t2, nullptr, nullptr))) return rc;
    return st;
}

int uegccd_ccd_g2_ex(UegccdCtx *c, const double *t_abab, int32_t mask, int32_t precision, double *g_abab)
{
    if (!c || !t_abab || !g_abab) return fail(UEGCCD_ERR_ARG, "null argument");
    if (precision != UEGCCD_FP64 && precision != UEGCCD_MIXED) return fail(UEGCCD_ERR_ARG, "unknown precision");
    ENTER(c->batch);
    UegccdBatch &b = *c->batch;
    int rc = pack_from_host(b, 0, t_abab);
    if (rc) return rc;
    if ((rc = set_active_all(b, 1))) return rc;
    TermFlags f;
    f.do_driver = (mask & 1) ? 1 : 0;
    f.do_mosaic = (mask & 2) ? 1 : 0;
    f.do_ladder = (mask & 4) ? 1 : 0;
    f.do_ring = (mask & 8) ? 1 : 0;
    f.do_xring = (mask & 16) ? 1 : 0;
    DevBatch &d = b.d;
    if (precision == UEGCCD_MIXED) {
        // the tensor-core ladder of t itself: refresh point t_ref = 0, g_ref = 0
        if ((rc = mixed_alloc(b))) return rc;
        CU(cudaMemsetAsync(d.t_ref, 0, d.namp * sizeof(double), b.stream));
        CU(cudaMemsetAsync(d.g_ref, 0, d.namp * sizeof(double), b.stream));
        CU(cudaMemsetAsync(d.tc_err, 0, sizeof(int), b.stream));
        f.mixed = 1;
    }
    // g_out reuses t_new (mode 1 does not write the update)
    launch_residual(d, f, 1, d.t_new, b.stream);
    CU(cudaGetLastError());
    if (precision == UEGCCD_MIXED) {
        int err = 0;
        CU(cudaMemcpyAsync(&err, d.tc_err, sizeof(int), cudaMemcpyDeviceToHost, b.stream));
        CU(cudaStreamSynchronize(b.stream));
        if (err) return fail(UEGCCD_ERR_CUDA, "tensor-core ladder: an mbarrier wait expired");
    }
    return unpack_to_host(b, 0, d.t_new, g_abab, nullptr, nullptr);
}

int32_t uegccd_sf_length(const UegccdSystem *sys)
{
    if (!sys || !sys->nvec || sys->nao <= 0) return fail(UEGCCD_ERR_ARG, "bad system");
    int m = sys->nvec[0];
    for (int64_t k = 0; k < 3 * (int64_t)sys->nao; k++) m = std::max(m, (int)sys->nvec[k]);
    return m * 2 + 1;
}

int uegccd_structure_factor(UegccdCtx *c, const double *t_abab, const UegccdSfGrid *out)
{
    if (!c || !t_abab || !out) return fail(UEGCCD_ERR_ARG, "null argument");
    ENTER(c->batch);
    UegccdBatch &b = *c->batch;
    int rc = pack_from_host(b, 0, t_abab);
    if (rc) return rc;
    return structure_factor(b, 0, *out);
}

int uegccd_ccd_g2(UegccdCtx *c, const double *t_abab, int32_t mask, double *g_abab)
{
    return uegccd_ccd_g2_ex(c, t_abab, mask, UEGCCD_FP64, g_abab);
}

int uegccd_ctx_set_eri(UegccdCtx *c, const UegccdRangeTerms *flags, int32_t safe_eri, double screening)
{
    if (!c) return fail(UEGCCD_ERR_ARG, "null context");
    if (!flags) {
        c->eri_set = false;
        return 0;
    }
    const int32_t *p = &flags->ring;
    bool screened = false;
    for (int k = 0; k < 15; k++) {
        if (p[k] < 0 || p[k] > 3) return fail(UEGCCD_ERR_ARG, "range flags must be 0, 1, 2 or 3");
        screened = screened || p[k] == 1 || p[k] == 2;
    }
    if (screened && !(screening > 0.0)) return fail(UEGCCD_ERR_ARG, "screening distance must be > 0");
    c->flags = *flags;
    c->safe_eri = safe_eri ? 1 : 0;
    c->screening = screening;
    c->eri_set = true;
    return 0;
}

int uegccd_ccd_g2_2ch(UegccdCtx *c, const double *t_abab, const double *t_abba, int32_t mask, double *g_abab,
                      double *g_abba)
{
    if (!c || !t_abab || !t_abba || !g_abab || !g_abba) return fail(UEGCCD_ERR_ARG, "null argument");
    ENTER(c->batch);
    int rc = two_channel_ready(*c, c->batch->core_n, c->batch->gapii);
    if (rc) return rc;
    return c->tc->ccd_g2(t_abab, t_abba, mask, g_abab, g_abba);
}

int uegccd_drpa_g2(UegccdCtx *c, const double *t2, int32_t mask, double *g2)
{
    if (!c || !t2 || !g2) return fail(UEGCCD_ERR_ARG, "null argument");
    ENTER(c->batch);
    int rc = two_channel_ready(*c, c->batch->core_n, c->batch->gapii);
    if (rc) return rc;
    return c->tc->drpa_g2(t2, mask, g2);
}

int uegccd_batch_create(const UegccdSystem *systems, int32_t n, UegccdBatch **out)
{
    if (!out || !systems) return fail(UEGCCD_ERR_ARG, "null argument");
    *out = nullptr;
    std::unique_ptr<UegccdBatch> b;
    int rc = build_batch(systems, n, b);
    if (rc) return rc;
    *out = b.release();
    return 0;
}

int uegccd_batch_destroy(UegccdBatch *b)
{
    if (!b) return 0;
    ENTER_DEVICE(b);
    delete b;
    return 0;
}

int uegccd_batch_solve(UegccdBatch *b, const UegccdOptions *opt, int32_t drpa, double *e2, UegccdResult *results)
{
    if (!b || !results) return fail(UEGCCD_ERR_ARG, "null argument");
    ENTER(b);
    b->ses.on = false;   // a full solve ends an open incremental one
    const bool two = opt && !drpa && (opt->do_ring != 0) != (opt->do_xring != 0);
    if (two && opt->range_flags != 0 && b->range_flag == 0)
        return fail(UEGCCD_ERR_UNSUPPORTED, "range-separated integrals: set one flag with uegccd_batch_set_range");
    int rc = validate_options(opt, drpa, *b, two);
    if (rc) return rc;
    if ((rc = set_integrals(*b, opt->core_n, opt->gapii))) return rc;
    b->two_channel_amps = false;
    CU(cudaEventRecord(b->ev_solve0, b->stream));
    b->kt.begin(KID_MP2, b->stream);
    launch_mp2(b->d, b->stream);
    b->kt.end(b->stream);
    launch_reduce(b->d, b->stream);
    if ((rc = read_red(*b))) return rc;
    if (e2)
        for (int s = 0; s < b->d.nsolves; s++) e2[s] = b->red[3 * s];
    if (drpa) {
        // the reference starts dRPA from T2aaaa of the MP2 step (Main.f90:85-91)
        launch_to_aaaa(b->d, b->stream);
        std::swap(b->d.t, b->d.t_new);
    }
    int st = two ? run_two_channel_solves(*b, opt, results) : run_solves(*b, opt, drpa, results);
    if (st < 0) return st;
    CU(cudaEventRecord(b->ev_solve1, b->stream));
    CU(cudaEventSynchronize(b->ev_solve1));
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, b->ev_solve0, b->ev_solve1));
    for (int s = 0; s < b->d.nsolves; s++) results[s].gpu_ms = ms;
    return st;
}

int uegccd_batch_start(UegccdBatch *b, const UegccdOptions *opt, int32_t drpa, double *e2)
{
    if (!b) return fail(UEGCCD_ERR_ARG, "null batch");
    ENTER(b);
    int rc = validate_options(opt, drpa, *b);
    if (rc) return rc;
    if (opt->precision != UEGCCD_FP64)
        return fail(UEGCCD_ERR_UNSUPPORTED, "an incremental solve runs in FP64 (use uegccd_batch_solve for MIXED)");
    if (opt->range_flags != 0)
        return fail(UEGCCD_ERR_UNSUPPORTED, "an incremental solve takes no range flags (use uegccd_batch_solve)");
    if ((rc = set_integrals(*b, opt->core_n, opt->gapii))) return rc;
    b->two_channel_amps = false;
    b->launches = 0;
    launch_mp2(b->d, b->stream);
    launch_reduce(b->d, b->stream);
    b->launches += 2;
    if ((rc = read_red(*b))) return rc;
    if (e2)
        for (int s = 0; s < b->d.nsolves; s++) e2[s] = b->red[3 * s];
    if (drpa) {
        launch_to_aaaa(b->d, b->stream);   // the dRPA start is T2aaaa of the MP2 step (Main.f90:85-91)
        std::swap(b->d.t, b->d.t_new);
        b->launches++;
    }
    return session_start(*b, opt, drpa);
}

int uegccd_batch_advance(UegccdBatch *b, int32_t rounds, int32_t *n_active, int32_t *n_done, int32_t *done_ids,
                         UegccdResult *done_results)
{
    if (!b || !n_active || !n_done || !done_ids || !done_results || rounds < 0)
        return fail(UEGCCD_ERR_ARG, "bad argument");
    ENTER(b);
    *n_active = 0;
    *n_done = 0;
    if (!b->ses.on) return fail(UEGCCD_ERR_ARG, "no incremental solve is open on this batch (uegccd_batch_start)");
    return session_advance(*b, rounds, n_active, n_done, done_ids, done_results);
}

int32_t uegccd_batch_ring_threads(UegccdBatch *b, int32_t *threads, int32_t max)
{
    if (!b || !threads || max <= 0) return fail(UEGCCD_ERR_ARG, "bad argument");
    const int n = std::min<int>(max, kRingClasses);
    for (int c = 0; c < n; c++) threads[c] = b->d.ring_threads[c];
    return n;
}

int32_t uegccd_batch_launch_shapes(UegccdBatch *b, int32_t *vals, int32_t max)
{
    if (!b || !vals || max <= 0) return fail(UEGCCD_ERR_ARG, "bad argument");
    int32_t v[kRingClasses + 3];
    for (int c = 0; c < kRingClasses; c++) v[c] = b->d.ring_threads[c];
    v[kRingClasses] = b->d.stage_threads;
    v[kRingClasses + 1] = b->d.ladder_sched;
    v[kRingClasses + 2] = b->d.hh_kc;
    const int n = std::min<int>(max, kRingClasses + 3);
    for (int k = 0; k < n; k++) vals[k] = v[k];
    return n;
}

int uegccd_batch_set_profiling(UegccdBatch *b, int32_t on)
{
    if (!b) return fail(UEGCCD_ERR_ARG, "null batch");
    ENTER(b);
    if (on && !b->kt_events) {
        for (auto &e : b->kt.ev) CU(cudaEventCreate(&e));
        b->kt_events = true;
    }
    b->kt.on = on != 0;
    for (int k = 0; k < KID_COUNT; k++) { b->kt.ms[k] = 0.0; b->kt.launches[k] = 0; }
    b->have_graph = false;  // re-capture with (or without) the timer events
    return 0;
}

int32_t uegccd_batch_kernel_stats(UegccdBatch *b, int32_t max, const char **names, double *ms, int64_t *launches)
{
    if (!b) return fail(UEGCCD_ERR_ARG, "null batch");
    int n = 0;
    for (int k = 0; k < KID_COUNT && n < max; k++) {
        if (b->kt.launches[k] == 0) continue;
        if (names) names[n] = kKernelNames[k];
        if (ms) ms[n] = b->kt.ms[k];
        if (launches) launches[n] = b->kt.launches[k];
        n++;
    }
    return n;
}

int uegccd_footprint(const UegccdSystem *sys, int32_t ndiis, int32_t mixed, int64_t *bytes, int64_t *namp)
{
    if (!sys || !bytes) return fail(UEGCCD_ERR_ARG, "null argument");
    SystemHost h;
    int rc = read_system(sys, h);
    if (rc) return rc;
    SolvePlan P;
    std::string msg = build_solve_plan(h, P);
    if (!msg.empty()) return fail(UEGCCD_ERR_ARG, msg);
    const int64_t A = P.namp, O = P.O, V = P.V, M = P.M;
    int64_t hh = 0, nblk = (int64_t)P.blocks.size();
    for (const auto &B : P.blocks) hh += (int64_t)B.o * B.o;
    int64_t b = 0;
    int64_t sum_ov = 0;
    for (const auto &B : P.blocks) sum_ov += B.o + B.v;
    b += A * (8 * 3 + 16 + sizeof(AmpInfo) + 4 + 4); // t, t_new, g; Coulomb factors; amps; partner, mirror
    b += sum_ov * (8 + 4) + (V + O + 1) * (4 + 8);   // mosaic partials and target lists
    b += O * O * V * 4;                              // pos
    b += O * V * O * 8;                              // dRPA ring intermediate (allocated for dRPA only)
    b += O * V * 2 * 2;                              // ph rows
    int64_t xy = 0;                                  // particle-hole operands and results of the rings
    for (size_t gi = 0; gi < P.groups.size(); gi++) {
        const auto &G = P.groups[gi];
        if (G.partner < 0 || G.partner < (int)gi) continue;
        const auto &H2 = P.groups[G.partner];
        const int64_t n1 = std::min(G.n, H2.n), n2 = std::max(G.n, H2.n);
        xy += n1 * 2 * ((n2 + 7) & ~7);
    }
    b += xy * 8 * 2 + O * V * 4 * 2;                 // xy, rx; ph_a, ph_b
    b += O * V * O * 4 * 2;                          // ring gather indices
    b += hh * 8 + nblk * (sizeof(BlockDev) + 8) + M * (16 + 8) + (P.q2max + 1) * 8;
    b += A * (8 + 4) * (int64_t)std::max(0, (int)ndiis);  // DIIS history (t' FP64, e FP32)
    if (mixed) {
        b += A * 8 * 2;                              // t_ref, g_ref
        for (const auto &B : P.blocks) {             // FP16 Coulomb slabs and d tiles, row scales
            const int64_t nch = (B.v + 31) / 32, ntc = B.o <= 16 ? 16 : B.o <= 32 ? 32 : 64;
            b += ((B.v + 127) / 128) * nch * 128 * 32 * 2;
            b += ((B.o + ntc - 1) / ntc) * (nch * ntc * 32 * 2 + ntc * 4);
        }
    }
    b += (int64_t)O * O * V * 8 * 3;                 // reference-layout staging (one solve)
    *bytes = b;
    if (namp) *namp = A;
    return 0;
}

int uegccd_batch_transfer_bytes(UegccdBatch *b, int64_t *h2d, int64_t *d2h)
{
    if (!b) return fail(UEGCCD_ERR_ARG, "null batch");
    if (h2d) *h2d = b->h2d_bytes;
    if (d2h) *d2h = b->d2h_bytes;
    return 0;
}

int uegccd_batch_get_amplitudes(UegccdBatch *b, int32_t s, double *t_abab)
{
    if (!b || !t_abab || s < 0 || s >= b->d.nsolves) return fail(UEGCCD_ERR_ARG, "bad argument");
    ENTER(b);
    return unpack_to_host(*b, s, b->d.t, t_abab, nullptr, nullptr);
}

int uegccd_batch_get_all_amplitudes(UegccdBatch *b, double *t_abab)
{
    if (!b || !t_abab) return fail(UEGCCD_ERR_ARG, "bad argument");
    ENTER(b);
    const int n = b->d.nsolves;
    if (!b->dense_all) {
        std::vector<int64_t> off(n + 1, 0);
        for (int s = 0; s < n; s++) off[s + 1] = off[s] + (int64_t)b->plans[s].O * b->plans[s].O * b->plans[s].V;
        int rc = b->upload(b->dense_off, off);
        if (rc) return rc;
        if ((rc = b->alloc(b->dense_all, (size_t)off[n]))) return rc;
        b->dense_all_n = (size_t)off[n];
    }
    CU(cudaMemsetAsync(b->dense_all, 0, b->dense_all_n * sizeof(double), b->stream));
    launch_unpack_all(b->d, b->dense_off, b->d.t, b->dense_all, b->stream);
    b->launches++;
    CU(cudaGetLastError());
    const size_t bytes = b->dense_all_n * sizeof(double);
    b->d2h_bytes += (int64_t)bytes;
    // a page-locked destination takes the copy directly
    cudaPointerAttributes pa;
    const bool pinned = cudaPointerGetAttributes(&pa, t_abab) == cudaSuccess && pa.type == cudaMemoryTypeHost;
    if (!pinned) cudaGetLastError();   // clear the query's status on older drivers
    if (bytes < kStageMin || pinned) {
        CU(cudaMemcpyAsync(t_abab, b->dense_all, bytes, cudaMemcpyDeviceToHost, b->stream));
        CU(cudaStreamSynchronize(b->stream));
        return UEGCCD_OK;
    }
    // large downloads: through a cached pinned buffer, copied out on all host cores
    // (a pageable copy is staged by the driver on one thread)
    std::lock_guard<std::mutex> lock(g_stage_mu);
    if (g_stage_bytes < bytes) {
        if (g_stage) cudaFreeHost(g_stage);
        g_stage = nullptr;
        g_stage_bytes = 0;
        CU(cudaHostAlloc((void **)&g_stage, bytes, cudaHostAllocPortable));
        g_stage_bytes = bytes;
    }
    CU(cudaMemcpyAsync(g_stage, b->dense_all, bytes, cudaMemcpyDeviceToHost, b->stream));
    CU(cudaStreamSynchronize(b->stream));
    const int nth = std::max(1, std::min(16, (int)std::thread::hardware_concurrency()));
    const size_t piece = (bytes + nth - 1) / nth;
    parallel_for(nth, nth, [&](int k) {
        const size_t a = (size_t)k * piece, e = std::min(bytes, a + piece);
        if (a < e) std::memcpy((char *)t_abab + a, g_stage + a, e - a);
    });
    return UEGCCD_OK;
}

int uegccd_batch_mp2(UegccdBatch *b, double *e2)
{
    if (!b) return fail(UEGCCD_ERR_ARG, "null batch");
    ENTER(b);
    b->two_channel_amps = false;
    b->kt.begin(KID_MP2, b->stream);
    launch_mp2(b->d, b->stream);
    b->kt.end(b->stream);
    launch_reduce(b->d, b->stream);
    b->launches += 2;
    int rc = read_red(*b);
    if (rc) return rc;
    int status = UEGCCD_OK;
    for (int s = 0; s < b->d.nsolves; s++) {
        if (e2) e2[s] = b->red[3 * s];
        if (!std::isfinite(b->red[3 * s])) status = fail(UEGCCD_ERR_NUMERIC, "non-finite MP2 energy");
    }
    return status;
}

int uegccd_batch_structure_factor(UegccdBatch *b, int32_t s, const UegccdSfGrid *out)
{
    if (!b || !out || s < 0 || s >= b->d.nsolves) return fail(UEGCCD_ERR_ARG, "bad argument");
    ENTER(b);
    if (b->two_channel_amps)
        return fail(UEGCCD_ERR_UNSUPPORTED, "structure factors of two-channel amplitudes are outside the GPU path");
    return structure_factor(*b, s, *out);
}

int uegccd_trim_cache(void)
{
    {
        std::lock_guard<std::mutex> lock(g_stage_mu);
        if (g_stage) cudaFreeHost(g_stage);
        g_stage = nullptr;
        g_stage_bytes = 0;
    }
    std::vector<DevChunk> drop;
    {
        std::lock_guard<std::mutex> lock(g_pool_mu);
        drop.swap(g_pool);
        g_pool_bytes = 0;
    }
    for (auto &c : drop) {
        DeviceScope on(c.dev);
        cudaFree(c.p);
    }
    {
        std::lock_guard<std::mutex> lock(g_pool_mu);
        for (auto &c : drop) g_dev_bytes[c.dev % kMaxDevices] -= (int64_t)c.size;
    }
    return UEGCCD_OK;
}

int uegccd_set_memory_limit(int64_t bytes)
{
    if (bytes < 0) return fail(UEGCCD_ERR_ARG, "memory limit must be >= 0");
    std::lock_guard<std::mutex> lock(g_pool_mu);
    g_mem_limit = bytes;
    return UEGCCD_OK;
}

int uegccd_memory_info(int64_t *held, int64_t *cached)
{
    const int dev = current_device() % kMaxDevices;
    std::lock_guard<std::mutex> lock(g_pool_mu);
    int64_t c = 0;
    for (const auto &x : g_pool)
        if (x.dev == dev) c += (int64_t)x.size;
    if (held) *held = g_dev_bytes[dev];
    if (cached) *cached = c;
    return UEGCCD_OK;
}

int uegccd_batch_history(UegccdBatch *b, int32_t s, double *energies, double *dts, int32_t max_rec,
                         int32_t *n_recorded)
{
    if (!b || s < 0 || s >= b->d.nsolves || max_rec < 0 || !n_recorded)
        return fail(UEGCCD_ERR_ARG, "bad argument");
    ENTER(b);
    if (b->two_channel_amps) {
        const auto &e = b->tc_en[s], &d = b->tc_dt[s];
        const int n = std::min((int)e.size(), max_rec);
        if (energies) std::copy(e.begin(), e.begin() + n, energies);
        if (dts) std::copy(d.begin(), d.begin() + n, dts);
        *n_recorded = n;
        return UEGCCD_OK;
    }
    if (b->last_niter.size() != (size_t)b->d.nsolves || !b->ctl.rec_e)
        return fail(UEGCCD_ERR_ARG, "no solve has run on this batch");
    const int n = std::min(b->last_niter[s], max_rec);
    const size_t off = (size_t)s * b->ctl.max_rec;
    if (n > 0 && energies)
        CU(cudaMemcpyAsync(energies, b->ctl.rec_e + off, n * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    if (n > 0 && dts)
        CU(cudaMemcpyAsync(dts, b->ctl.rec_dt + off, n * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    CU(cudaStreamSynchronize(b->stream));
    *n_recorded = n;
    return UEGCCD_OK;
}

}  // extern "C"
