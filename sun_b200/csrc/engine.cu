// engine.cu -- host runtime and C ABI of the engine (include/sun_b200.h).
//
// Objects: a context (device, stream, last error, launch shapes), lattices
// (device image + device-resident RNG/sweep counters), groups (device tables
// of same-class lattices that one launch advances), batches (groups of
// mixed classes, optionally replayed from a CUDA graph) and a server
// (continuous batching over a batch).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/sun_b200.h"
#include "sun_ops.h"

using namespace sunb;

namespace {

struct Error : std::runtime_error {
    sun_status st;
    Error(sun_status s, const std::string& m) : std::runtime_error(m), st(s) {}
};

[[noreturn]] void fail(sun_status st, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    throw Error(st, buf);
}

void ck(cudaError_t e, const char* what)
{
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        fail(SUN_ERR_OUT_OF_MEMORY, "%s: %s", what, cudaGetErrorString(e));
    }
    if (e != cudaSuccess) fail(SUN_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// Host-side fault injection (sun_debug_fail_allocations): allocations left
// before every further device allocation reports out-of-memory; -1 = off.
std::atomic<int> g_alloc_budget{-1};

// Device buffer owned by the library.
struct DevBuf {
    void* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    void ensure(size_t bytes)
    {
        if (bytes <= n) return;
        release();
        int left = g_alloc_budget.load();
        while (left > 0 && !g_alloc_budget.compare_exchange_weak(left, left - 1)) {
        }
        if (left == 0) fail(SUN_ERR_OUT_OF_MEMORY, "cudaMalloc: out of memory (injected)");
        ck(cudaMalloc(&p, bytes), "cudaMalloc");
        n = bytes;
    }
};

struct PinnedBuf {
    void* p = nullptr;
    size_t n = 0;
    ~PinnedBuf()
    {
        if (p) cudaFreeHost(p);
    }
    void ensure(size_t bytes)
    {
        if (bytes <= n) return;
        if (p) cudaFreeHost(p);
        p = nullptr;
        ck(cudaMallocHost(&p, bytes), "cudaMallocHost");
        n = bytes;
    }
};

int elems_of(int N, int layout)
{
    if (layout == SUN_SOA12) return 6;
    if (layout == SUN_SOA8) return 4;
    return N * N;
}

double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

}  // namespace

// ---------------------------------------------------------------------------
struct sun_ctx {
    int device = 0;
    int verbosity = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;
    std::recursive_mutex mu;
    DevBuf err;          // device error word (injected-stream overrun)
    size_t hbm_budget = 0;
    // launch shapes (CTA sizes) per kernel family
    int blk_update = 128, blk_sites = 128, blk_links = 256, blk_wilson = 64;
    // update kernel: 0 chosen by size (or by the tuner), 1 always one thread
    // per half-site (k_update), 2 always N lanes per half-site (k_update_rows),
    // 3 the tiled kernel where it applies (k_update_tile: N >= 4, full links).
    // By size: groups of N >= 4, and of SU(3) with FP64 full links, with at
    // most rows_max_halfv half-sites (FP64: half that) take the row-split
    // kernel.  Sweeps measured on B200: SU(6) 8^4 FP32 3.1x and FP64 2.2x
    // faster, 12^4 FP32 1.55x; SU(4) 8^4 16-21 %, 12^4 FP32 10 %; SU(3) FP64
    // 8^4 5 %.  SU(2), SU(3) in FP32 and larger lattices are faster with one
    // thread per half-site.
    int upd_kernel = 0;
    int blk_rows = 128;
    // consecutive update phases launched as programmatic dependents
    // (SUN_B200_PDL=0 turns it off)
    int pdl = 1;
    long long rows_max_halfv = 16384;
    // sun_sweep_measure in one cooperative launch (k_sweeps_resident): -1
    // for SU(3) FP32 lattices of at most resident_max_halfv half-sites, 0
    // never, 1 whenever the lattice and launch shapes allow
    // (SUN_B200_RESIDENT).  Measured on B200, 1 HB + 4 OR with both
    // observables per sweep, us per sweep resident / captured graph: SU(3)
    // FP32 8^4 188 / 200 (full links), 190 / 189 (12-parameter), 12^4
    // 206 / 226; slower for FP64 (SU(3) 8^4 230 / 194, 12^4 297 / 268),
    // SU(2) (8^4 131 / 111), SU(4) (8^4 271 / 224) and from 16^4 up.
    int resident = -1;
    long long resident_max_halfv = 16384;
    unsigned long long barrier_wait_ns = 1000000000ull;  // one grid barrier wait at most
    int skip_arrive = -1;  // test hook (sun_debug_resident_barrier)
    DevBuf res_sync;       // barrier count, generation, status
    DevBuf res_out;        // per-sweep plaquette and Polyakov sums
    // autotuner (tuneLaunch, src/tune.cpp:304): CTA size of the update kernel
    // per (kernel class, total half-volume), timed once, cached in a CSV file
    bool tune = false;
    std::string tune_path;
    std::map<std::string, int> tuned;
};

namespace { struct Group; }

struct sun_lattice {
    sun_ctx* ctx = nullptr;
    sun_lattice_params p{};
    DevBuf links;
    DevBuf state;        // uint32 [heatbath passes, sweeps, advanced, spare]
    size_t bytes = 0;
    LatDev desc{};
    unsigned version = 0;    // bumped when desc changes (device tables re-upload)
    Group* solo = nullptr;   // one-lattice launch table, built on first use
    // one sweep captured as a CUDA graph, replayed by sun_sweep: for (hb, or)
    // passes per sweep at descriptor version graph_version
    cudaGraphExec_t sweep_graph = nullptr;
    int graph_hb = -1, graph_or = -1;
    unsigned graph_version = 0;
    // one sweep plus the plaquette and the Polyakov loop as a CUDA graph,
    // replayed by sun_sweep_measure: the measurement kernels write row *slot
    // of meas (meas_rows rows of plaquettes, then as many of Polyakov loops)
    // and the graph advances slot
    cudaGraphExec_t meas_graph = nullptr;
    int meas_hb = -1, meas_or = -1;
    unsigned meas_version = 0;
    size_t meas_rows = 0;
    // meas_part: the captured measurements' CTA partials, owned by the graph
    // (a shared scratch buffer could be reallocated under it by a later
    // call that needs more partials)
    DevBuf meas, slot, meas_part, meas_cnt;
    ~sun_lattice();
};

namespace {

cudaStream_t S(sun_ctx* c, void* s) { return s ? reinterpret_cast<cudaStream_t>(s) : c->stream; }

int work_of(const LatDev& L, int kind)
{
    switch (kind) {
    case WORK_HALF: return L.halfV;
    case WORK_SITES: return L.V;
    case WORK_SPATIAL: return L.X[0] * L.X[1] * L.X[2];
    case WORK_PLANES: return plaquette_items(L.V);
    case WORK_POLY8: return kPolyLanes * L.X[0] * L.X[1] * L.X[2];
    default: return 4 * L.V;
    }
}

// Same-class lattices advanced by one launch per kernel.
struct Group {
    int N = 0, fp64 = 0, layout = 0;
    std::vector<sun_lattice*> lats;
    DevBuf d_lats;
    struct Begin {
        std::shared_ptr<DevBuf> buf;  // CTA prefix, grows only
        int nblocks = 0;
        bool valid = false;
    };
    std::map<std::pair<int, int>, Begin> begins;
    DevBuf partials, out;
    DevBuf counters;     // per-lattice CTA counters of the fused finalize (kept at zero)
    size_t counters_n = 0;
    PinnedBuf h_out;
    bool dirty = true;
    std::vector<unsigned> versions;

    void sync(cudaStream_t s)
    {
        if (!dirty) {
            for (size_t i = 0; i < lats.size(); ++i)
                if (versions[i] != lats[i]->version) dirty = true;
        }
        if (!dirty) return;
        std::vector<LatDev> h(lats.size());
        versions.resize(lats.size());
        for (size_t i = 0; i < lats.size(); ++i) {
            h[i] = lats[i]->desc;
            versions[i] = lats[i]->version;
        }
        d_lats.ensure(sizeof(LatDev) * std::max<size_t>(1, h.size()));
        if (!h.empty())
            ck(cudaMemcpyAsync(d_lats.p, h.data(), sizeof(LatDev) * h.size(), cudaMemcpyHostToDevice, s),
               "table upload");
        ck(cudaStreamSynchronize(s), "table upload");
        for (auto& kv : begins) kv.second.valid = false;
        dirty = false;
    }
    BatchView view(int kind, int block, cudaStream_t s)
    {
        sync(s);
        Begin& e = begins[std::make_pair(kind, block)];
        if (!e.valid) {
            std::vector<int> b(lats.size() + 1, 0);
            for (size_t i = 0; i < lats.size(); ++i)
                b[i + 1] = b[i] + (work_of(lats[i]->desc, kind) + block - 1) / block;
            if (!e.buf) e.buf = std::make_shared<DevBuf>();
            e.buf->ensure(sizeof(int) * b.size());
            ck(cudaMemcpyAsync(e.buf->p, b.data(), sizeof(int) * b.size(), cudaMemcpyHostToDevice, s), "begin upload");
            ck(cudaStreamSynchronize(s), "begin upload");
            e.nblocks = b.back();
            e.valid = true;
        }
        BatchView v;
        v.lats = reinterpret_cast<const LatDev*>(d_lats.p);
        v.begin = reinterpret_cast<const int*>(e.buf->p);
        v.nlat = (int)lats.size();
        v.nblocks = e.nblocks;
        return v;
    }
};

#define OPS_CALL(N_, FN, ...)                                                      \
    do {                                                                           \
        cudaError_t e_;                                                            \
        switch (N_) {                                                              \
        case 2: e_ = Ops<2>::FN(__VA_ARGS__); break;                               \
        case 3: e_ = Ops<3>::FN(__VA_ARGS__); break;                               \
        case 4: e_ = Ops<4>::FN(__VA_ARGS__); break;                               \
        case 6: e_ = Ops<6>::FN(__VA_ARGS__); break;                               \
        default: fail(SUN_ERR_UNSUPPORTED, "N=%d not built", (int)(N_));          \
        }                                                                          \
        ck(e_, #FN);                                                               \
    } while (0)

// -- sweeps ------------------------------------------------------------------
// Launch shape of the update: cfg > 0 runs k_update with CTAs of cfg threads
// (one per half-site), cfg < 0 runs k_update_rows with CTAs of -cfg threads
// (N lanes per half-site, 32/N half-sites per warp), cfg == kCfgTile runs
// k_update_tile (N warps per 32 half-sites, N >= 4).  All give the same bits.
constexpr int kCfgTile = 1 << 20;
int upd_sites_per_cta(int N, int cfg)
{
    return cfg == kCfgTile ? 32 : (cfg > 0 ? cfg : (-cfg / 32) * (32 / N));
}
bool tile_ok(const Group& g) { return g.N >= 4 && g.layout == SUN_SOA; }

BatchView upd_view(Group& g, int cfg, cudaStream_t s) { return g.view(WORK_HALF, upd_sites_per_cta(g.N, cfg), s); }

// pdl: launch as a programmatic dependent of the previous launch on s, which
// must be the preceding update phase of the same lattices
void launch_update(Group& g, int mode, int cfg, const BatchView& v, int par, int mu, unsigned hb_offset,
                   const InjView& inj, cudaStream_t s, int pdl = 0)
{
    if (cfg == kCfgTile) OPS_CALL(g.N, update_tile, g.fp64, g.layout, mode, v, par, mu, hb_offset, inj, pdl, s);
    else if (cfg > 0) OPS_CALL(g.N, update, g.fp64, g.layout, mode, v, cfg, par, mu, hb_offset, inj, pdl, s);
    else OPS_CALL(g.N, update_rows, g.fp64, g.layout, mode, v, -cfg, par, mu, hb_offset, inj, pdl, s);
}

// Update launch shape for this group and mode.  Without tuning: by the size
// rule of sun_ctx::upd_kernel.  With tuning on, the first use of a (class,
// mode, total half-volume) key times one phase launch per candidate shape on
// the real lattices -- links backed up before and restored after, like
// Tunable::preTune/postTune (include/tune.h:119, monte.h:73-74) -- keeps the
// fastest and appends it to the cache file.
int update_block(sun_ctx* c, Group& g, int mode, cudaStream_t s)
{
    long long work = 0;
    size_t bytes = 0;
    for (auto* l : g.lats) {
        work += l->desc.halfV;
        bytes += l->bytes;
    }
    // by size: SU(6) always tiled (1.6-2x faster than one thread per site
    // from 12^4 up, no spills); small lattices of SU(4) and of SU(3) with
    // FP64 full links row-split; everything else one thread per half-site
    const bool small = work <= (g.fp64 ? c->rows_max_halfv / 2 : c->rows_max_halfv);
    const int fixed = c->upd_kernel == 1   ? c->blk_update
                      : c->upd_kernel == 2 ? -c->blk_rows
                      : (c->upd_kernel == 3 && tile_ok(g)) ? kCfgTile
                      : (g.N == 6 && tile_ok(g))             ? kCfgTile
                      : (small && (g.N >= 4 || (g.N == 3 && g.fp64 && g.layout == SUN_SOA)))
                          ? -c->blk_rows
                          : c->blk_update;
    if (!c->tune) return fixed;
    char key[160];
    snprintf(key, sizeof key, "k_update N=%d %s layout=%d mode=%d halfV=%lld kernel=%d", g.N, g.fp64 ? "f64" : "f32",
             g.layout, mode, work, c->upd_kernel);
    auto it = c->tuned.find(key);
    if (it != c->tuned.end()) return it->second;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) return fixed;
    DevBuf backup;
    backup.ensure(bytes);
    size_t off = 0;
    for (auto* l : g.lats) {
        ck(cudaMemcpyAsync((char*)backup.p + off, l->links.p, l->bytes, cudaMemcpyDeviceToDevice, s), "tune backup");
        off += l->bytes;
    }
    cudaEvent_t e0, e1;
    ck(cudaEventCreate(&e0), "event");
    ck(cudaEventCreate(&e1), "event");
    InjView none{nullptr, 0, nullptr};
    int best = fixed;
    float best_ms = 1e30f;
    for (int blk : {32, 64, 96, 128, -32, -64, -128, kCfgTile}) {
        if (blk == kCfgTile && !tile_ok(g)) continue;
        if (c->upd_kernel != 0 && (blk == kCfgTile) != (c->upd_kernel == 3)) continue;
        if (blk != kCfgTile && ((blk > 0 && c->upd_kernel == 2) || (blk < 0 && c->upd_kernel == 1))) continue;
        BatchView v = upd_view(g, blk, s);
        launch_update(g, mode, blk, v, 0, 0, 0u, none, s);  // warm-up
        ck(cudaEventRecord(e0, s), "event");
        for (int r = 0; r < 3; ++r) launch_update(g, mode, blk, v, 0, 0, 0u, none, s);
        ck(cudaEventRecord(e1, s), "event");
        ck(cudaEventSynchronize(e1), "event");
        float ms = 0;
        ck(cudaEventElapsedTime(&ms, e0, e1), "event");
        if (ms < best_ms) {
            best_ms = ms;
            best = blk;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    off = 0;
    for (auto* l : g.lats) {
        ck(cudaMemcpyAsync(l->links.p, (char*)backup.p + off, l->bytes, cudaMemcpyDeviceToDevice, s), "tune restore");
        off += l->bytes;
    }
    ck(cudaStreamSynchronize(s), "tune restore");
    c->tuned[key] = best;
    if (!c->tune_path.empty()) {
        if (FILE* f = fopen(c->tune_path.c_str(), "a")) {
            fprintf(f, "%s,%d,%.6f\n", key, best, best_ms / 3.0);
            fclose(f);
        }
    }
    return best;
}

// counters_later: the sweep's counter update is left to the launch after
// it (the fused measurement of a sweep-and-measure graph; only without a
// reunitarization, which reads the counters)
void group_sweep(sun_ctx* c, Group& g, int n_hb, int n_or, bool count_sweep, bool reunit, cudaStream_t s,
                 bool counters_later = false)
{
    if (g.lats.empty()) return;
    InjView none{nullptr, 0, nullptr};
    // a shape's table is made only for a mode that runs: inside a graph
    // capture only the tables prepared before it exist.  Every phase after
    // the first is launched as a programmatic dependent of the one before
    // (its launch overlaps the previous phase's drain).
    int pdl = 0;
    if (n_hb > 0) {
        const int bhb = update_block(c, g, MODE_HB, s);
        BatchView vhb = upd_view(g, bhb, s);
        for (int h = 0; h < n_hb; ++h)
            for (int par = 0; par < 2; ++par)
                for (int mu = 0; mu < 4; ++mu, pdl = c->pdl)
                    launch_update(g, MODE_HB, bhb, vhb, par, mu, (unsigned)h, none, s, pdl);
    }
    if (n_or > 0) {
        const int bor = update_block(c, g, MODE_OR, s);
        BatchView vor = upd_view(g, bor, s);
        for (int o = 0; o < n_or; ++o)
            for (int par = 0; par < 2; ++par)
                for (int mu = 0; mu < 4; ++mu, pdl = c->pdl)
                    launch_update(g, MODE_OR, bor, vor, par, mu, 0u, none, s, pdl);
    }
    if ((n_hb > 0 || count_sweep) && !(counters_later && !reunit))
        ck(launch_end_sweep(reinterpret_cast<const LatDev*>(g.d_lats.p), (int)g.lats.size(), (unsigned)n_hb,
                            count_sweep ? 1u : 0u, s),
           "end_sweep");
    // end_sweep above also bumped the sweep counter when count_sweep; the
    // reunitarization kernel checks each lattice's own schedule on device
    if (reunit) {
        BatchView links = g.view(WORK_LINKS, c->blk_links, s);
        OPS_CALL(g.N, reunit, g.fp64, g.layout, links, c->blk_links, 1, s);
    }
}

bool group_needs_reunit(const Group& g)
{
    for (auto* l : g.lats)
        if (l->p.reunit_every > 0) return true;
    return false;
}

// -- measurements --------------------------------------------------------------
// Runs a partial-producing kernel and the deterministic per-lattice finalize;
// returns nvals doubles per lattice in g.h_out.
template <class F> double* group_reduce(Group& g, int kind, int block, int nvals, bool is_max, cudaStream_t s, F launch)
{
    BatchView v = g.view(kind, block, s);
    g.partials.ensure(sizeof(double) * 2 * (size_t)nvals * std::max(1, v.nblocks));
    g.out.ensure(sizeof(double) * (size_t)nvals * g.lats.size());
    g.h_out.ensure(sizeof(double) * (size_t)nvals * g.lats.size());
    launch(v, reinterpret_cast<double*>(g.partials.p));
    if (is_max)
        ck(launch_finalize_max(v, reinterpret_cast<double*>(g.partials.p), reinterpret_cast<double*>(g.out.p), s),
           "finalize");
    else
        ck(launch_finalize_sum(v, reinterpret_cast<double*>(g.partials.p), nvals, reinterpret_cast<double*>(g.out.p),
                               s),
           "finalize");
    ck(cudaMemcpyAsync(g.h_out.p, g.out.p, sizeof(double) * nvals * g.lats.size(), cudaMemcpyDeviceToHost, s),
       "result copy");
    ck(cudaStreamSynchronize(s), "measurement");
    return reinterpret_cast<double*>(g.h_out.p);
}

// The same for kernels that finalize in their last CTA per lattice and write
// the result straight into the pinned host buffer: one launch and a
// synchronisation, no finalize launch and no copy.
template <class F> double* group_reduce_fused(Group& g, int kind, int block, int nvals, cudaStream_t s, F launch)
{
    BatchView v = g.view(kind, block, s);
    g.partials.ensure(sizeof(double) * 2 * (size_t)nvals * std::max(1, v.nblocks));
    g.h_out.ensure(sizeof(double) * (size_t)nvals * g.lats.size());
    if (g.counters_n < g.lats.size()) {
        g.counters.ensure(sizeof(unsigned) * g.lats.size());
        ck(cudaMemsetAsync(g.counters.p, 0, sizeof(unsigned) * g.lats.size(), s), "counters");
        g.counters_n = g.lats.size();
    }
    launch(v, reinterpret_cast<double*>(g.partials.p), reinterpret_cast<double*>(g.h_out.p),
           reinterpret_cast<unsigned*>(g.counters.p));
    ck(cudaStreamSynchronize(s), "measurement");
    return reinterpret_cast<double*>(g.h_out.p);
}

void group_plaquette(sun_ctx* c, Group& g, double* out, cudaStream_t s)
{
    double* r = group_reduce_fused(g, WORK_PLANES, c->blk_sites, 2, s,
                                   [&](const BatchView& v, double* part, double* out, unsigned* cnt) {
                                       OPS_CALL(g.N, plaquette, g.fp64, g.layout, v, c->blk_sites, part, out, cnt, nullptr, s);
                                   });
    for (size_t i = 0; i < g.lats.size(); ++i) {
        const LatDev& L = g.lats[i]->desc;
        double norm = 3.0 * g.N * (double)L.V;
        out[2 * i] = r[2 * i] / norm;
        out[2 * i + 1] = r[2 * i + 1] / norm;
    }
}

void group_polyakov(sun_ctx* c, Group& g, double* out, cudaStream_t s)
{
    double* r = group_reduce_fused(g, WORK_POLY8, c->blk_sites, 2, s,
                                   [&](const BatchView& v, double* part, double* out, unsigned* cnt) {
                                       OPS_CALL(g.N, polyakov, g.fp64, g.layout, v, c->blk_sites, part, out, cnt, nullptr, s);
                                   });
    for (size_t i = 0; i < g.lats.size(); ++i) {
        const LatDev& L = g.lats[i]->desc;
        double norm = (double)g.N * L.X[0] * L.X[1] * L.X[2];
        out[2 * i] = r[2 * i] / norm;
        out[2 * i + 1] = r[2 * i + 1] / norm;
    }
}

// single-lattice group, cached in the lattice (tables and measurement
// scratch persist across calls)
struct Solo {
    Group& g;
    explicit Solo(sun_lattice* l) : g(*make(l)) {}
    static Group* make(sun_lattice* l)
    {
        if (!l->solo) {
            Group* g = new Group();
            g->N = l->p.ncolors;
            g->fp64 = l->p.precision == SUN_F64;
            g->layout = l->p.layout;
            g->lats.push_back(l);
            l->solo = g;
        }
        return l->solo;
    }
};

}  // namespace

sun_lattice::~sun_lattice()
{
    if (sweep_graph) cudaGraphExecDestroy(sweep_graph);
    if (meas_graph) cudaGraphExecDestroy(meas_graph);
    delete solo;
}

namespace {

std::mutex g_err_mu;
std::string g_err;  // errors without a context

sun_status handle(sun_ctx* c, const std::function<void()>& f);

}  // namespace

// ---------------------------------------------------------------------------
// Generic kernels (N-independent)
namespace sunb {

void set_global_error(const char* msg)
{
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_err = msg;
}

struct DDh { double s, c; };
__device__ __forceinline__ DDh ddh_add(DDh a, DDh b)
{
    double s = a.s + b.s;
    double bb = s - a.s;
    double e = (a.s - (s - bb)) + (b.s - bb);
    DDh r;
    r.s = s;
    r.c = (a.c + b.c) + e;
    return r;
}

// one warp per lattice: lane-strided compensated sums over the lattice's
// CTA partials, then a fixed shuffle tree -- identical result whatever else
// shares the launch
__global__ void k_finalize_sum(BatchView bv, const double* partials, int nvals, double* out)
{
    const int l = blockIdx.x;
    const int lane = threadIdx.x;
    const int b0 = bv.begin[l], b1 = bv.begin[l + 1];
    for (int v = 0; v < nvals; ++v) {
        DDh d{0.0, 0.0};
        for (int b = b0 + lane; b < b1; b += 32) {
            DDh t{partials[((size_t)b * nvals + v) * 2], partials[((size_t)b * nvals + v) * 2 + 1]};
            d = ddh_add(d, t);
        }
        for (int o = 16; o > 0; o >>= 1) {
            DDh t{__shfl_down_sync(0xffffffffu, d.s, o), __shfl_down_sync(0xffffffffu, d.c, o)};
            d = ddh_add(d, t);
        }
        if (lane == 0) out[(size_t)l * nvals + v] = d.s + d.c;
    }
}

__global__ void k_finalize_max(BatchView bv, const double* partials, double* out)
{
    const int l = blockIdx.x;
    const int lane = threadIdx.x;
    double m = 0.0;
    for (int b = bv.begin[l] + lane; b < bv.begin[l + 1]; b += 32) m = fmax(m, partials[(size_t)b * 2]);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if (lane == 0) out[l] = m;
}

__global__ void k_end_sweep(const LatDev* lats, int nlat, unsigned n_hb, unsigned inc)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nlat) advance_counters(lats[i], n_hb, inc);
}

cudaError_t launch_finalize_sum(const BatchView& bv, const double* partials, int nvals, double* out, cudaStream_t s)
{
    k_finalize_sum<<<bv.nlat, 32, 0, s>>>(bv, partials, nvals, out);
    return cudaGetLastError();
}
cudaError_t launch_finalize_max(const BatchView& bv, const double* partials, double* out, cudaStream_t s)
{
    k_finalize_max<<<bv.nlat, 32, 0, s>>>(bv, partials, out);
    return cudaGetLastError();
}
__global__ void k_bump(unsigned* slot) { *slot += 1u; }

cudaError_t launch_bump(unsigned* slot, cudaStream_t s)
{
    k_bump<<<1, 1, 0, s>>>(slot);
    return cudaGetLastError();
}

cudaError_t launch_end_sweep(const LatDev* lats, int nlat, unsigned n_hb, unsigned inc, cudaStream_t s)
{
    k_end_sweep<<<(nlat + 127) / 128, 128, 0, s>>>(lats, nlat, n_hb, inc);
    return cudaGetLastError();
}

}  // namespace sunb

namespace {

sun_status handle(sun_ctx* c, const std::function<void()>& f)
{
    try {
        if (c) {
            std::lock_guard<std::recursive_mutex> lk(c->mu);
            f();
        } else {
            f();
        }
        return SUN_OK;
    } catch (const Error& e) {
        if (c) c->last_error = e.what();
        std::lock_guard<std::mutex> lk(g_err_mu);
        g_err = e.what();
        return e.st;
    } catch (const std::bad_alloc&) {
        if (c) c->last_error = "host allocation failed";
        return SUN_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        if (c) c->last_error = e.what();
        return SUN_ERR_CUDA;
    }
}

void validate(const sun_lattice_params* p)
{
    if (!p) fail(SUN_ERR_INVALID_ARG, "null lattice parameters");
    if (p->ncolors != 2 && p->ncolors != 3 && p->ncolors != 4 && p->ncolors != 6)
        fail(SUN_ERR_UNSUPPORTED, "N=%d not supported (built: 2, 3, 4, 6)", p->ncolors);
    for (int d = 0; d < 4; ++d) {
        if (p->dims[d] < 2) fail(SUN_ERR_INVALID_ARG, "dimension %d = %d too small", d, p->dims[d]);
        if (p->dims[d] % 2) fail(SUN_ERR_INVALID_ARG, "dimension %d = %d is odd (even/odd layout needs even)", d, p->dims[d]);
    }
    if (p->layout != SUN_SOA && p->layout != SUN_SOA12 && p->layout != SUN_SOA8)
        fail(SUN_ERR_INVALID_ARG, "unknown layout %d", (int)p->layout);
    if ((p->layout == SUN_SOA12 || p->layout == SUN_SOA8) && p->ncolors != 3)
        fail(SUN_ERR_UNSUPPORTED, "12/8-parameter layouts exist for SU(3) only");
    if (p->order != SUN_EVEN_ODD && p->order != SUN_NORMAL) fail(SUN_ERR_INVALID_ARG, "unknown order");
    if (p->precision != SUN_F32 && p->precision != SUN_F64) fail(SUN_ERR_INVALID_ARG, "unknown precision");
    if (p->reunit_every < 0) fail(SUN_ERR_INVALID_ARG, "reunit_every < 0");
    double V = (double)p->dims[0] * p->dims[1] * p->dims[2] * p->dims[3];
    double maxidx = V * 4.0 * elems_of(p->ncolors, p->layout);
    if (maxidx >= 2147483647.0) fail(SUN_ERR_CAPACITY, "lattice too large for 32-bit element indexing");
}

void need_eo(sun_lattice* l, const char* what)
{
    if (l->p.order != SUN_EVEN_ODD)
        fail(SUN_ERR_UNSUPPORTED, "%s needs an even/odd ordered array (as the reference kernels)", what);
}

}  // namespace

// ===========================================================================
extern "C" {

const char* sun_version(void) { return "sun_b200 0.1 (sm_100a)"; }

sun_status sun_debug_fail_allocations(int after_n)
{
    g_alloc_budget.store(after_n < 0 ? -1 : after_n);
    return SUN_OK;
}

sun_status sun_debug_resident_barrier(sun_ctx* c, long long wait_ns, int skip_cta)
{
    if (!c) return SUN_ERR_INVALID_ARG;
    return handle(c, [&] {
        c->barrier_wait_ns = wait_ns > 0 ? (unsigned long long)wait_ns : 1000000000ull;
        c->skip_arrive = skip_cta < 0 ? -1 : skip_cta;
    });
}

const char* sun_last_error_string(const sun_ctx* c)
{
    if (c) return c->last_error.c_str();
    return g_err.c_str();
}

sun_status sun_init(const sun_config* cfg, sun_ctx** out)
{
    return handle(nullptr, [&] {
        if (!out) fail(SUN_ERR_INVALID_ARG, "null output");
        auto c = std::make_unique<sun_ctx>();
        c->device = cfg ? cfg->device : 0;
        c->tune = cfg && cfg->tune;
        if (cfg && cfg->tune_cache_path) {
            c->tune_path = cfg->tune_cache_path;
            if (FILE* f = fopen(cfg->tune_cache_path, "r")) {  // "key,block,ms" lines
                char line[256];
                while (fgets(line, sizeof line, f)) {
                    char* c1 = strchr(line, ',');
                    if (!c1) continue;
                    *c1 = 0;
                    int blk = atoi(c1 + 1);
                    // k_update CTA sizes, k_update_rows ones as negative
                    // numbers, or the tiled kernel's code
                    const int t = blk < 0 ? -blk : blk;
                    if ((t >= 32 && t <= 128 && t % 32 == 0) || blk == kCfgTile) c->tuned[line] = blk;
                }
                fclose(f);
            }
        }
        c->verbosity = cfg ? cfg->verbosity : 0;
        int n = 0;
        ck(cudaGetDeviceCount(&n), "cudaGetDeviceCount");
        if (c->device < 0 || c->device >= n) fail(SUN_ERR_INVALID_ARG, "device %d not present (%d devices)", c->device, n);
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        ck(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        c->err.ensure(sizeof(int));
        ck(cudaMemset(c->err.p, 0, sizeof(int)), "memset");
        size_t fr = 0, tot = 0;
        ck(cudaMemGetInfo(&fr, &tot), "cudaMemGetInfo");
        c->hbm_budget = (cfg && cfg->hbm_budget_bytes) ? cfg->hbm_budget_bytes : (size_t)(0.9 * (double)fr);
        // launch-shape overrides (CTA sizes, multiples of 32 up to 256)
        auto env_blk = [](const char* name, int& v) {
            if (const char* s = getenv(name)) {
                int b = atoi(s);
                if (b >= 32 && b <= 256 && b % 32 == 0) v = b;
            }
        };
        env_blk("SUN_B200_BLOCK_UPDATE", c->blk_update);
        env_blk("SUN_B200_BLOCK_SITES", c->blk_sites);
        env_blk("SUN_B200_BLOCK_LINKS", c->blk_links);
        env_blk("SUN_B200_BLOCK_ROWS", c->blk_rows);
        if (c->blk_rows > 128) c->blk_rows = 128;
        // update kernel: "sites" (k_update), "rows" (k_update_rows), "tile"
        // (k_update_tile, N >= 4 full links; others by size) or "auto" (by
        // size); SUN_B200_ROWS_MAX_HALFV moves the size threshold
        if (const char* k = getenv("SUN_B200_UPDATE_KERNEL")) {
            if (!strcmp(k, "sites")) c->upd_kernel = 1;
            else if (!strcmp(k, "rows")) c->upd_kernel = 2;
            else if (!strcmp(k, "tile")) c->upd_kernel = 3;
        }
        if (const char* t = getenv("SUN_B200_ROWS_MAX_HALFV")) c->rows_max_halfv = atoll(t);
        if (const char* t = getenv("SUN_B200_RESIDENT")) c->resident = !strcmp(t, "auto") ? -1 : (atoi(t) ? 1 : 0);
        if (const char* t = getenv("SUN_B200_RESIDENT_MAX_HALFV")) c->resident_max_halfv = atoll(t);
        if (const char* t = getenv("SUN_B200_PDL")) c->pdl = atoi(t) ? 1 : 0;
        *out = c.release();
    });
}

sun_status sun_finalize(sun_ctx* c)
{
    if (!c) return SUN_ERR_INVALID_ARG;
    cudaStreamSynchronize(c->stream);
    cudaStreamDestroy(c->stream);
    delete c;
    return SUN_OK;
}

sun_status sun_lattice_create(sun_ctx* c, const sun_lattice_params* p, sun_lattice** out)
{
    return handle(c, [&] {
        if (!c || !out) fail(SUN_ERR_INVALID_ARG, "null argument");
        validate(p);
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        auto l = std::make_unique<sun_lattice>();
        l->ctx = c;
        l->p = *p;
        const int V = p->dims[0] * p->dims[1] * p->dims[2] * p->dims[3];
        const size_t csz = p->precision == SUN_F64 ? 16 : 8;
        l->bytes = csz * (size_t)elems_of(p->ncolors, p->layout) * 4 * (size_t)V;
        l->links.ensure(l->bytes);
        l->state.ensure(4 * sizeof(unsigned));
        ck(cudaMemset(l->state.p, 0, 4 * sizeof(unsigned)), "memset");
        ck(cudaMemset(l->links.p, 0, l->bytes), "memset");
        LatDev& d = l->desc;
        d.links = l->links.p;
        for (int k = 0; k < 4; ++k) d.X[k] = p->dims[k];
        d.V = V;
        d.halfV = V / 2;
        d.beta_over_n = p->beta / p->ncolors;
        d.seed = p->seed;
        d.state = reinterpret_cast<unsigned*>(l->state.p);
        d.reunit_every = p->reunit_every;
        d.evenodd = p->order == SUN_EVEN_ODD;
        *out = l.release();
    });
}

sun_status sun_lattice_destroy(sun_lattice* l)
{
    if (!l) return SUN_ERR_INVALID_ARG;
    delete l;
    return SUN_OK;
}

sun_status sun_lattice_bytes(const sun_lattice* l, size_t* b)
{
    if (!l || !b) return SUN_ERR_INVALID_ARG;
    *b = l->bytes;
    return SUN_OK;
}

sun_status sun_lattice_device_ptr(const sun_lattice* l, void** d)
{
    if (!l || !d) return SUN_ERR_INVALID_ARG;
    *d = l->links.p;
    return SUN_OK;
}

sun_status sun_lattice_init_cold(sun_lattice* l, void* stream)
{
    if (!l) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] {
        // the 8-parameter form is singular at |a1| = 1 (gaugearray.cu:293-297)
        if (l->p.layout == SUN_SOA8) fail(SUN_ERR_UNSUPPORTED, "SOA8 arrays cannot take a cold start");
        cudaStream_t s = S(l->ctx, stream);
        Solo so(l);
        BatchView v = so.g.view(WORK_LINKS, l->ctx->blk_links, s);
        OPS_CALL(l->p.ncolors, cold, so.g.fp64, so.g.layout, v, l->ctx->blk_links, s);
        ck(cudaMemsetAsync(l->state.p, 0, 4 * sizeof(unsigned), s), "memset");
        ck(cudaStreamSynchronize(s), "cold start");
    });
}

sun_status sun_lattice_init_hot(sun_lattice* l, void* stream)
{
    if (!l) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] {
        cudaStream_t s = S(l->ctx, stream);
        Solo so(l);
        BatchView v = so.g.view(WORK_SITES, 128, s);
        OPS_CALL(l->p.ncolors, hot, so.g.fp64, so.g.layout, v, 128, s);
        ck(cudaMemsetAsync(l->state.p, 0, 4 * sizeof(unsigned), s), "memset");
        ck(cudaStreamSynchronize(s), "hot start");
    });
}

static void canon_upload(sun_lattice* l, const void* host, cudaStream_t s, bool host_is_device)
{
    const size_t V = l->desc.V, N = l->p.ncolors;
    const size_t bytes = V * 4 * N * N * 16;
    DevBuf stage;
    const void* src = host;
    if (!host_is_device) {
        stage.ensure(bytes);
        ck(cudaMemcpyAsync(stage.p, host, bytes, cudaMemcpyHostToDevice, s), "upload");
        src = stage.p;
    }
    Solo so(l);
    BatchView v = so.g.view(WORK_LINKS, l->ctx->blk_links, s);
    OPS_CALL(l->p.ncolors, pack, so.g.fp64, so.g.layout, v, l->ctx->blk_links, src, s);
    ck(cudaStreamSynchronize(s), "upload");
}

static void canon_download(sun_lattice* l, void* host, cudaStream_t s)
{
    const size_t V = l->desc.V, N = l->p.ncolors;
    const size_t bytes = V * 4 * N * N * 16;
    DevBuf stage;
    stage.ensure(bytes);
    Solo so(l);
    BatchView v = so.g.view(WORK_LINKS, l->ctx->blk_links, s);
    OPS_CALL(l->p.ncolors, unpack, so.g.fp64, so.g.layout, v, l->ctx->blk_links, stage.p, s);
    ck(cudaMemcpyAsync(host, stage.p, bytes, cudaMemcpyDeviceToHost, s), "download");
    ck(cudaStreamSynchronize(s), "download");
}

sun_status sun_lattice_upload(sun_lattice* l, const void* host, sun_host_format fmt, void* stream)
{
    if (!l || !host) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] {
        cudaStream_t s = S(l->ctx, stream);
        if (fmt == SUN_HOST_IMAGE) {
            ck(cudaMemcpyAsync(l->links.p, host, l->bytes, cudaMemcpyHostToDevice, s), "upload");
            ck(cudaStreamSynchronize(s), "upload");
        } else if (fmt == SUN_HOST_CANONICAL) {
            canon_upload(l, host, s, false);
        } else {
            fail(SUN_ERR_INVALID_ARG, "unknown host format");
        }
    });
}

sun_status sun_lattice_download(sun_lattice* l, void* host, sun_host_format fmt, void* stream)
{
    if (!l || !host) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] {
        cudaStream_t s = S(l->ctx, stream);
        if (fmt == SUN_HOST_IMAGE) {
            ck(cudaMemcpyAsync(host, l->links.p, l->bytes, cudaMemcpyDeviceToHost, s), "download");
            ck(cudaStreamSynchronize(s), "download");
        } else if (fmt == SUN_HOST_CANONICAL) {
            canon_download(l, host, s);
        } else {
            fail(SUN_ERR_INVALID_ARG, "unknown host format");
        }
    });
}

sun_status sun_lattice_upload_async(sun_lattice* l, const void* host_image, void* stream)
{
    if (!l || !host_image) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] {
        ck(cudaMemcpyAsync(l->links.p, host_image, l->bytes, cudaMemcpyHostToDevice, S(l->ctx, stream)), "upload");
    });
}

sun_status sun_lattice_download_async(sun_lattice* l, void* host_image, void* stream)
{
    if (!l || !host_image) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] {
        ck(cudaMemcpyAsync(host_image, l->links.p, l->bytes, cudaMemcpyDeviceToHost, S(l->ctx, stream)), "download");
    });
}

extern "C++" {
namespace {

// dst <- src through the canonical FP64 order (layout, order and precision
// conversion); the RNG counters travel with the links
void copy_links(sun_lattice* dst, sun_lattice* src, cudaStream_t s)
{
    if (dst->p.ncolors != src->p.ncolors) fail(SUN_ERR_INVALID_ARG, "copy between different N");
    for (int k = 0; k < 4; ++k)
        if (dst->p.dims[k] != src->p.dims[k]) fail(SUN_ERR_INVALID_ARG, "copy between different geometries");
    const size_t V = src->desc.V, N = src->p.ncolors;
    DevBuf stage;
    stage.ensure(V * 4 * N * N * 16);
    {
        Solo so(src);
        BatchView v = so.g.view(WORK_LINKS, src->ctx->blk_links, s);
        OPS_CALL(src->p.ncolors, unpack, so.g.fp64, so.g.layout, v, src->ctx->blk_links, stage.p, s);
    }
    {
        Solo so(dst);
        BatchView v = so.g.view(WORK_LINKS, dst->ctx->blk_links, s);
        OPS_CALL(dst->p.ncolors, pack, so.g.fp64, so.g.layout, v, dst->ctx->blk_links, stage.p, s);
    }
    ck(cudaMemcpyAsync(dst->state.p, src->state.p, 2 * sizeof(unsigned), cudaMemcpyDeviceToDevice, s), "copy");
    ck(cudaStreamSynchronize(s), "copy");
}

}  // namespace
}  // extern "C++"

sun_status sun_lattice_copy(sun_lattice* dst, sun_lattice* src, void* stream)
{
    if (!dst || !src) return SUN_ERR_INVALID_ARG;
    return handle(dst->ctx, [&] { copy_links(dst, src, S(dst->ctx, stream)); });
}

sun_status sun_lattice_set_sweep_limit(sun_lattice* l, uint32_t limit)
{
    if (!l) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] {
        if (l->desc.sweep_limit != limit) {
            l->desc.sweep_limit = limit;
            ++l->version;  // device tables and captured sweeps pick it up
        }
    });
}

sun_status sun_ctx_hbm_budget(const sun_ctx* c, size_t* bytes)
{
    if (!c || !bytes) return SUN_ERR_INVALID_ARG;
    *bytes = c->hbm_budget;
    return SUN_OK;
}

sun_status sun_lattice_get_rng(sun_lattice* l, uint64_t* seed, uint32_t* hb, uint32_t* sw)
{
    if (!l) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] {
        unsigned st[2];
        ck(cudaMemcpy(st, l->state.p, sizeof st, cudaMemcpyDeviceToHost), "state read");
        if (seed) *seed = l->p.seed;
        if (hb) *hb = st[0];
        if (sw) *sw = st[1];
    });
}

sun_status sun_lattice_set_rng(sun_lattice* l, uint64_t seed, uint32_t hb, uint32_t sw)
{
    if (!l) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] {
        unsigned st[2] = {hb, sw};
        ck(cudaMemcpy(l->state.p, st, sizeof st, cudaMemcpyHostToDevice), "state write");
        l->p.seed = seed;
        l->desc.seed = seed;
        ++l->version;
    });
}

// One sweep of a lattice as a CUDA graph (captured on first use, kept until
// the passes per sweep or the lattice descriptor change).  A small lattice's
// sweep is 40-odd short launches; replaying them from a graph removes the
// host launch cost between them (SU(3) 8^4 FP64: 380 -> 305 us per sweep).
// The sweep's state (RNG pass and sweep counters, the reunitarization
// schedule) lives on the device, so replays are the same sweeps as direct
// launches.  Returns false, leaving the caller to launch directly, when the
// caller's stream is itself being captured.
static bool solo_sweep_graph(sun_lattice* l, Group& g, int n_hb, int n_or, bool re, cudaStream_t s)
{
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) return false;
    if (l->sweep_graph && l->graph_hb == n_hb && l->graph_or == n_or && l->graph_version == l->version) return true;
    if (l->sweep_graph) cudaGraphExecDestroy(l->sweep_graph);
    l->sweep_graph = nullptr;
    // launch shapes (tuned if tuning is on) and their tables, before capture
    if (n_hb > 0) upd_view(g, update_block(l->ctx, g, MODE_HB, s), s);
    if (n_or > 0) upd_view(g, update_block(l->ctx, g, MODE_OR, s), s);
    if (re) g.view(WORK_LINKS, l->ctx->blk_links, s);
    cudaStream_t cs;
    ck(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "stream");
    cudaGraph_t graph;
    ck(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "capture");
    try {
        group_sweep(l->ctx, g, n_hb, n_or, true, re, cs);
    } catch (...) {
        cudaStreamEndCapture(cs, &graph);
        cudaStreamDestroy(cs);
        throw;
    }
    ck(cudaStreamEndCapture(cs, &graph), "capture end");
    cudaStreamDestroy(cs);
    cudaError_t e = cudaGraphInstantiate(&l->sweep_graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) l->sweep_graph = nullptr;
    ck(e, "graph instantiate");
    l->graph_hb = n_hb;
    l->graph_or = n_or;
    l->graph_version = l->version;
    return true;
}

static void solo_passes(sun_lattice* l, int n_hb, int n_or, int n_sweeps, bool count, cudaStream_t s)
{
    need_eo(l, "the heatbath/overrelaxation update");
    Solo so(l);
    const bool re = count && l->p.reunit_every > 0;
    if (count && n_sweeps > 0 && solo_sweep_graph(l, so.g, n_hb, n_or, re, s)) {
        for (int i = 0; i < n_sweeps; ++i) ck(cudaGraphLaunch(l->sweep_graph, s), "graph launch");
        return;
    }
    for (int i = 0; i < n_sweeps; ++i) group_sweep(l->ctx, so.g, n_hb, n_or, count, re, s);
}

sun_status sun_heatbath(sun_lattice* l, int n, void* stream)
{
    if (!l || n < 0) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] { solo_passes(l, n, 0, 1, false, S(l->ctx, stream)); });
}

sun_status sun_overrelax(sun_lattice* l, int n, void* stream)
{
    if (!l || n < 0) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] { solo_passes(l, 0, n, 1, false, S(l->ctx, stream)); });
}

sun_status sun_sweep(sun_lattice* l, int n_hb, int n_or, int n_sweeps, void* stream)
{
    if (!l || n_hb < 0 || n_or < 0 || n_sweeps < 0) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] { solo_passes(l, n_hb, n_or, n_sweeps, true, S(l->ctx, stream)); });
}

// The graph of sun_sweep_measure for at least `rows` sweeps (captured again
// when the passes per sweep, the lattice descriptor or the row capacity
// change).  Returns false when the caller's stream is being captured.
static bool solo_measure_graph(sun_lattice* l, Group& g, int n_hb, int n_or, size_t rows, cudaStream_t s)
{
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) return false;
    if (l->meas_graph && l->meas_hb == n_hb && l->meas_or == n_or && l->meas_version == l->version &&
        l->meas_rows >= rows)
        return true;
    if (l->meas_graph) cudaGraphExecDestroy(l->meas_graph);
    l->meas_graph = nullptr;
    size_t cap_rows = 64;
    while (cap_rows < rows) cap_rows *= 2;
    l->meas.ensure(sizeof(double) * 4 * cap_rows);
    l->slot.ensure(sizeof(unsigned));
    l->meas_rows = cap_rows;
    sun_ctx* c = l->ctx;
    const bool re = l->p.reunit_every > 0;
    // launch shapes, tables and scratch before the capture
    if (n_hb > 0) upd_view(g, update_block(c, g, MODE_HB, s), s);
    if (n_or > 0) upd_view(g, update_block(c, g, MODE_OR, s), s);
    if (re) g.view(WORK_LINKS, c->blk_links, s);
    BatchView vp = g.view(WORK_PLANES, c->blk_sites, s), vl = g.view(WORK_POLY8, c->blk_sites, s);
    // CTAs of 128 threads: the plaquette and the Polyakov loop in one launch
    // (own partials and counters: the two parts run side by side)
    const bool fused = c->blk_sites == 128;
    l->meas_part.ensure(sizeof(double) * 4 * (size_t)std::max(1, vp.nblocks + vl.nblocks));
    l->meas_cnt.ensure(sizeof(unsigned) * 3);
    ck(cudaMemsetAsync(l->meas_cnt.p, 0, sizeof(unsigned) * 3, s), "counters");
    if (g.counters_n < g.lats.size()) {
        g.counters.ensure(sizeof(unsigned) * g.lats.size());
        ck(cudaMemsetAsync(g.counters.p, 0, sizeof(unsigned) * g.lats.size(), s), "counters");
        g.counters_n = g.lats.size();
    }
    ck(cudaStreamSynchronize(s), "measure graph setup");
    double* part = reinterpret_cast<double*>(l->meas_part.p);
    unsigned* cnt = reinterpret_cast<unsigned*>(g.counters.p);
    unsigned* slot = reinterpret_cast<unsigned*>(l->slot.p);
    double* out_p = reinterpret_cast<double*>(l->meas.p);
    double* out_l = out_p + 2 * cap_rows;
    cudaStream_t cs;
    ck(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "stream");
    cudaGraph_t graph;
    ck(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "capture");
    try {
        group_sweep(c, g, n_hb, n_or, true, re, cs, fused);
        if (fused) {
            unsigned* mc = reinterpret_cast<unsigned*>(l->meas_cnt.p);
            OPS_CALL(g.N, plaq_poly, g.fp64, g.layout, vp, vl, part, part + 4 * (size_t)vp.nblocks, out_p, out_l, mc,
                     mc + 1, slot, mc + 2, re ? -1 : n_hb, cs);
        } else {
            OPS_CALL(g.N, plaquette, g.fp64, g.layout, vp, c->blk_sites, part, out_p, cnt, slot, cs);
            OPS_CALL(g.N, polyakov, g.fp64, g.layout, vl, c->blk_sites, part, out_l, cnt, slot, cs);
            ck(launch_bump(slot, cs), "bump");
        }
    } catch (...) {
        cudaStreamEndCapture(cs, &graph);
        cudaStreamDestroy(cs);
        throw;
    }
    ck(cudaStreamEndCapture(cs, &graph), "capture end");
    cudaStreamDestroy(cs);
    cudaError_t e = cudaGraphInstantiate(&l->meas_graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) l->meas_graph = nullptr;
    ck(e, "graph instantiate");
    l->meas_hb = n_hb;
    l->meas_or = n_or;
    l->meas_version = l->version;
    return true;
}

// sweeps per resident launch at most
constexpr int kResidentChunk = 256;

// sun_sweep_measure in cooperative launches (k_sweeps_resident), for a
// lattice whose launched phases are latency-bound.  Returns false, having
// launched nothing, when the lattice, the launch shapes or the stream do not
// allow it.
static bool resident_sweeps(sun_lattice* l, Group& g, int n_hb, int n_or, int n_sweeps, double* plaq, double* poly,
                            cudaStream_t s)
{
    sun_ctx* c = l->ctx;
    const LatDev& L = l->desc;
    if (c->resident == 0 || L.sweep_limit != 0u || c->blk_sites != 128 || g.N > 4) return false;
    if (c->resident < 0 && (g.N != 3 || g.fp64 || L.halfV > c->resident_max_halfv)) return false;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) return false;
    // the launched path's update shapes: one thread per half-site or the
    // row-split kernel, CTAs of 128 threads, the same for both modes
    const int cfg_hb = n_hb > 0 ? update_block(c, g, MODE_HB, s) : 0;
    const int cfg_or = n_or > 0 ? update_block(c, g, MODE_OR, s) : 0;
    const int cfg = n_hb > 0 ? cfg_hb : cfg_or;
    if ((n_hb > 0 && n_or > 0 && cfg_hb != cfg_or) || (cfg != 128 && cfg != -128)) return false;
    const int rows = cfg < 0;
    int cap_ctas = 0;
    switch (g.N) {
    case 2: cap_ctas = Ops<2>::resident_capacity(g.fp64, g.layout, rows); break;
    case 3: cap_ctas = Ops<3>::resident_capacity(g.fp64, g.layout, rows); break;
    case 4: cap_ctas = Ops<4>::resident_capacity(g.fp64, g.layout, rows); break;
    default: break;
    }
    if (cap_ctas < 2) return false;
    BatchView upd = upd_view(g, cfg, s);
    BatchView vp = g.view(WORK_PLANES, 128, s), vl = g.view(WORK_POLY8, 128, s);
    g.partials.ensure(sizeof(double) * 4 * (size_t)(vp.nblocks + vl.nblocks));
    c->res_sync.ensure(4 * sizeof(unsigned));
    c->res_out.ensure(sizeof(double) * 4 * (size_t)n_sweeps);
    ResidentArgs a{};
    a.upd = upd;
    a.plaq = vp;
    a.poly = vl;
    a.n_hb = n_hb;
    a.n_or = n_or;
    a.partials = reinterpret_cast<double*>(g.partials.p);
    a.bar = reinterpret_cast<unsigned*>(c->res_sync.p);
    a.status = reinterpret_cast<int*>(a.bar + 2);
    a.wait_ns = c->barrier_wait_ns;
    a.skip_arrive = c->skip_arrive;
    // two sets of CTAs that take the phases in turn, each covering the
    // update's CTAs (several per resident CTA when they do not all fit)
    const int grid = 2 * std::max(1, std::min(cap_ctas / 2, upd.nblocks));
    // at most kResidentChunk sweeps per launch, so no launch runs long; each
    // continues from the counters the one before left, and its status is
    // read before the next starts
    double* out_p = reinterpret_cast<double*>(c->res_out.p);
    double* out_l = out_p + 2 * (size_t)n_sweeps;
    for (int done = 0; done < n_sweeps; done += kResidentChunk) {
        ck(cudaMemsetAsync(c->res_sync.p, 0, 4 * sizeof(unsigned), s), "barrier reset");
        a.n_sweeps = std::min(kResidentChunk, n_sweeps - done);
        a.out_plaq = out_p + 2 * (size_t)done;
        a.out_poly = out_l + 2 * (size_t)done;
        OPS_CALL(g.N, sweeps_resident, g.fp64, g.layout, rows, a, grid, s);
        int status = 0;
        ck(cudaMemcpyAsync(&status, a.status, sizeof(int), cudaMemcpyDeviceToHost, s), "status copy");
        ck(cudaStreamSynchronize(s), "resident sweeps");
        if (status)
            fail(SUN_ERR_DEVICE_FLAG, "a grid barrier wait of the resident sweeps ran out (limit %llu ns); the links "
                 "are left part-updated", (unsigned long long)c->barrier_wait_ns);
    }
    std::vector<double> h(4 * (size_t)n_sweeps);
    ck(cudaMemcpyAsync(h.data(), c->res_out.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s), "copy");
    ck(cudaStreamSynchronize(s), "resident sweeps");
    const double np = 3.0 * l->p.ncolors * (double)L.V, nl = (double)l->p.ncolors * L.X[0] * L.X[1] * L.X[2];
    for (int i = 0; i < 2 * n_sweeps; ++i) {
        if (plaq) plaq[i] = h[i] / np;
        if (poly) poly[i] = h[2 * (size_t)n_sweeps + i] / nl;
    }
    return true;
}

sun_status sun_sweep_measure(sun_lattice* l, int n_hb, int n_or, int n_sweeps, double* plaq, double* poly,
                             void* stream)
{
    if (!l || n_hb < 0 || n_or < 0 || n_sweeps < 0) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] {
        need_eo(l, "the heatbath/overrelaxation update");
        cudaStream_t s = S(l->ctx, stream);
        if (n_sweeps == 0) return;
        Solo so(l);
        if (resident_sweeps(l, so.g, n_hb, n_or, n_sweeps, plaq, poly, s)) return;
        if (solo_measure_graph(l, so.g, n_hb, n_or, (size_t)n_sweeps, s)) {
            // n replays back to back, one copy of the observables at the end;
            // normalised on the host as sun_plaquette / sun_polyakov do
            ck(cudaMemsetAsync(l->slot.p, 0, sizeof(unsigned), s), "slot");
            for (int i = 0; i < n_sweeps; ++i) ck(cudaGraphLaunch(l->meas_graph, s), "graph launch");
            std::vector<double> h(4 * (size_t)n_sweeps);
            const double* d = reinterpret_cast<const double*>(l->meas.p);
            ck(cudaMemcpyAsync(h.data(), d, sizeof(double) * 2 * n_sweeps, cudaMemcpyDeviceToHost, s), "copy");
            ck(cudaMemcpyAsync(h.data() + 2 * n_sweeps, d + 2 * l->meas_rows, sizeof(double) * 2 * n_sweeps,
                               cudaMemcpyDeviceToHost, s),
               "copy");
            ck(cudaStreamSynchronize(s), "sweep and measure");
            const LatDev& L = l->desc;
            const double np = 3.0 * l->p.ncolors * (double)L.V, nl = (double)l->p.ncolors * L.X[0] * L.X[1] * L.X[2];
            for (int i = 0; i < 2 * n_sweeps; ++i) {
                if (plaq) plaq[i] = h[i] / np;
                if (poly) poly[i] = h[2 * n_sweeps + i] / nl;
            }
            return;
        }
        double tmp[2];
        for (int i = 0; i < n_sweeps; ++i) {
            solo_passes(l, n_hb, n_or, 1, true, s);
            group_plaquette(l->ctx, so.g, plaq ? plaq + 2 * i : tmp, s);
            group_polyakov(l->ctx, so.g, poly ? poly + 2 * i : tmp, s);
        }
    });
}

sun_status sun_heatbath_injected(sun_lattice* l, const double* u, int stride, void* stream)
{
    if (!l || !u || stride <= 0) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] {
        need_eo(l, "the heatbath update");
        cudaStream_t s = S(l->ctx, stream);
        Solo so(l);
        const int cfg = update_block(l->ctx, so.g, MODE_HB, s);
        BatchView half = upd_view(so.g, cfg, s);
        ck(cudaMemsetAsync(l->ctx->err.p, 0, sizeof(int), s), "memset");
        InjView inj{u, stride, reinterpret_cast<int*>(l->ctx->err.p)};
        for (int par = 0; par < 2; ++par)
            for (int mu = 0; mu < 4; ++mu) launch_update(so.g, MODE_HB_INJECTED, cfg, half, par, mu, 0u, inj, s);
        int flag = 0;
        ck(cudaMemcpyAsync(&flag, l->ctx->err.p, sizeof(int), cudaMemcpyDeviceToHost, s), "flag read");
        ck(cudaStreamSynchronize(s), "heatbath");
        if (flag) fail(SUN_ERR_DEVICE_FLAG, "injected uniform stream ran out (stride %d)", stride);
    });
}

sun_status sun_reunitarize(sun_lattice* l, void* stream)
{
    if (!l) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] {
        cudaStream_t s = S(l->ctx, stream);
        Solo so(l);
        BatchView v = so.g.view(WORK_LINKS, l->ctx->blk_links, s);
        OPS_CALL(l->p.ncolors, reunit, so.g.fp64, so.g.layout, v, l->ctx->blk_links, 0, s);
        ck(cudaStreamSynchronize(s), "reunitarize");
    });
}

sun_status sun_unitarity_violation(sun_lattice* l, double* out, void* stream)
{
    if (!l || !out) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] {
        cudaStream_t s = S(l->ctx, stream);
        Solo so(l);
        double* r = group_reduce(so.g, WORK_LINKS, 256, 1, true, s, [&](const BatchView& v, double* part) {
            OPS_CALL(l->p.ncolors, unitarity, so.g.fp64, so.g.layout, v, 256, part, s);
        });
        *out = r[0];
    });
}

sun_status sun_link_trace_det(sun_lattice* l, double out[4], void* stream)
{
    if (!l || !out) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] {
        cudaStream_t s = S(l->ctx, stream);
        Solo so(l);
        double* r = group_reduce(so.g, WORK_LINKS, 256, 4, false, s, [&](const BatchView& v, double* part) {
            OPS_CALL(l->p.ncolors, linkstats, so.g.fp64, so.g.layout, v, 256, part, s);
        });
        const double nl = 4.0 * (double)l->desc.V;
        out[0] = r[0] / (nl * l->p.ncolors);
        out[1] = r[1] / (nl * l->p.ncolors);
        out[2] = r[2] / nl;
        out[3] = r[3] / nl;
    });
}

sun_status sun_plaquette(sun_lattice* l, double out[2], void* stream)
{
    if (!l || !out) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] {
        Solo so(l);
        group_plaquette(l->ctx, so.g, out, S(l->ctx, stream));
    });
}

sun_status sun_polyakov(sun_lattice* l, double out[2], void* stream)
{
    if (!l || !out) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] {
        Solo so(l);
        group_polyakov(l->ctx, so.g, out, S(l->ctx, stream));
    });
}

sun_status sun_wilson_loops(sun_lattice* l, int R, int T, double* out, void* stream)
{
    if (!l || !out) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] {
        if (R < 0 || T < 0 || R > 8 || T > 8) fail(SUN_ERR_INVALID_ARG, "Wilson loops need 0 <= R, T <= 8");
        for (int d = 0; d < 3; ++d)
            if (R >= l->p.dims[d]) fail(SUN_ERR_INVALID_ARG, "R=%d not below spatial extent %d", R, l->p.dims[d]);
        if (T >= l->p.dims[3]) fail(SUN_ERR_INVALID_ARG, "T=%d not below temporal extent", T);
        cudaStream_t s = S(l->ctx, stream);
        Solo so(l);
        const int nv = 2 * (R + 1) * (T + 1);
        const int blk = l->ctx->blk_wilson;
        double* r = group_reduce(so.g, WORK_SITES, blk, nv, false, s, [&](const BatchView& v, double* part) {
            OPS_CALL(l->p.ncolors, wilson, so.g.fp64, so.g.layout, v, blk, R, T, part, s);
        });
        const double norm = 3.0 * l->p.ncolors * (double)l->desc.V;
        for (int i = 0; i < nv; ++i) out[i] = r[i] / norm;
    });
}

// ---------------------------------------------------------------------------
// Smearing (src/smear/*.cu).  Each step rebuilds the selected directions from
// the unchanged field: the steps alternate between the lattice's image and a
// scratch copy (the unselected directions are equal in both), and an odd
// step count ends with one copy back.
extern "C++" {
namespace {

constexpr int kSmearBlock = 128;  // the smearing kernels' __launch_bounds__

void check_dirmask(int dirmask)
{
    if (dirmask <= 0 || dirmask > 15) fail(SUN_ERR_INVALID_ARG, "direction mask %d not in 1..15", dirmask);
}

template <class F> void smear_steps(sun_lattice* l, int steps, cudaStream_t s, F step)
{
    if (steps <= 0) return;
    DevBuf tmp;
    tmp.ensure(l->bytes);
    ck(cudaMemcpyAsync(tmp.p, l->links.p, l->bytes, cudaMemcpyDeviceToDevice, s), "smear scratch");
    Solo so(l);
    BatchView v = so.g.view(WORK_SITES, kSmearBlock, s);
    void* img[2] = {l->links.p, tmp.p};
    for (int st = 0; st < steps; ++st) step(so.g, v, img[st & 1], img[(st + 1) & 1]);
    if (steps & 1) ck(cudaMemcpyAsync(l->links.p, tmp.p, l->bytes, cudaMemcpyDeviceToDevice, s), "smear copy");
    ck(cudaStreamSynchronize(s), "smearing");
}

void check_pair(sun_lattice* src, sun_lattice* dst)
{
    if (src == dst) fail(SUN_ERR_INVALID_ARG, "multihit needs distinct input and output lattices");
    if (dst->p.ncolors != src->p.ncolors || dst->p.precision != src->p.precision || dst->p.order != src->p.order)
        fail(SUN_ERR_INVALID_ARG, "multihit input and output differ in N, precision or order");
    for (int k = 0; k < 4; ++k)
        if (dst->p.dims[k] != src->p.dims[k]) fail(SUN_ERR_INVALID_ARG, "multihit geometries differ");
    if (dst->p.layout != SUN_SOA) fail(SUN_ERR_INVALID_ARG, "multihit output must use the SOA layout (averages are not SU(N))");
}

}  // namespace
}  // extern "C++"

sun_status sun_smear_ape(sun_lattice* l, double w, int steps, int nhits, double tol, int dirmask, void* stream)
{
    if (!l || steps < 0 || nhits < 0) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] {
        check_dirmask(dirmask);
        cudaStream_t s = S(l->ctx, stream);
        smear_steps(l, steps, s, [&](Group& g, const BatchView& v, const void* src, void* dst) {
            OPS_CALL(g.N, ape, g.fp64, g.layout, v, kSmearBlock, src, dst, dirmask, w, nhits, tol, s);
        });
    });
}

sun_status sun_smear_stout(sun_lattice* l, double w, int steps, int dirmask, void* stream)
{
    if (!l || steps < 0) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] {
        check_dirmask(dirmask);
        if (l->p.ncolors != 3) fail(SUN_ERR_UNSUPPORTED, "stout smearing is defined for SU(3) only");
        cudaStream_t s = S(l->ctx, stream);
        smear_steps(l, steps, s, [&](Group& g, const BatchView& v, const void* src, void* dst) {
            OPS_CALL(g.N, stout, g.fp64, g.layout, v, kSmearBlock, src, dst, dirmask, w, s);
        });
    });
}

sun_status sun_smear_hyp(sun_lattice* l, const double alpha[3], int steps, int nhits, double tol, int dirmask,
                         void* stream)
{
    if (!l || !alpha || steps < 0 || nhits < 0) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] {
        check_dirmask(dirmask);
        cudaStream_t s = S(l->ctx, stream);
        // the reference keeps the three weights as FP32 constants (constants.cu:424-463)
        const double a1 = (float)alpha[0], a2 = (float)alpha[1], a3 = (float)alpha[2];
        const size_t nn = (size_t)l->p.ncolors * l->p.ncolors;
        const size_t slot_bytes = nn * (size_t)l->desc.V * (l->p.precision == SUN_F64 ? 16 : 8);
        DevBuf b1, b2;
        b1.ensure(16 * slot_bytes);
        b2.ensure(16 * slot_bytes);
        smear_steps(l, steps, s, [&](Group& g, const BatchView& v, const void* src, void* dst) {
            OPS_CALL(g.N, hyp, g.fp64, g.layout, v, kSmearBlock, 1, src, b1.p, b2.p, dst, dirmask, a3, nhits, tol, s);
            OPS_CALL(g.N, hyp, g.fp64, g.layout, v, kSmearBlock, 2, src, b1.p, b2.p, dst, dirmask, a2, nhits, tol, s);
            OPS_CALL(g.N, hyp, g.fp64, g.layout, v, kSmearBlock, 3, src, b1.p, b2.p, dst, dirmask, a1, nhits, tol, s);
        });
    });
}

sun_status sun_multihit(sun_lattice* src, sun_lattice* dst, int nhit, uint64_t seed, void* stream)
{
    if (!src || !dst || nhit < 0) return SUN_ERR_INVALID_ARG;
    return handle(dst->ctx, [&] {
        check_pair(src, dst);
        cudaStream_t s = S(dst->ctx, stream);
        copy_links(dst, src, s);
        Solo so(src);
        BatchView v = so.g.view(WORK_SITES, kSmearBlock, s);
        OPS_CALL(src->p.ncolors, multihit, so.g.fp64, so.g.layout, v, kSmearBlock, src->links.p, dst->links.p, nhit,
                 (unsigned long long)seed, 0, s);
        ck(cudaStreamSynchronize(s), "multihit");
    });
}

sun_status sun_multihit_space(sun_lattice* src, sun_lattice* dst, int nhit, void* stream)
{
    if (!src || !dst || nhit <= 0) return SUN_ERR_INVALID_ARG;
    return handle(dst->ctx, [&] {
        check_pair(src, dst);
        cudaStream_t s = S(dst->ctx, stream);
        copy_links(dst, src, s);
        Solo so(src);
        BatchView v = so.g.view(WORK_SITES, kSmearBlock, s);
        OPS_CALL(src->p.ncolors, multihit, so.g.fp64, so.g.layout, v, kSmearBlock, src->links.p, dst->links.p, nhit,
                 0ull, 1, s);
        ck(cudaStreamSynchronize(s), "multihit");
    });
}

// gauge file: header int32 grid[4], beta (leading sizeof(Real) bytes of the
// double), size_t sizeof(RealSave); body = canonical order in RealSave
sun_status sun_save_bin(sun_lattice* l, const char* path, int save_fp64, int with_header)
{
    if (!l || !path) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] {
        const size_t n = (size_t)l->desc.V * 4 * l->p.ncolors * l->p.ncolors * 2;
        std::vector<double> buf(n);
        canon_download(l, buf.data(), S(l->ctx, nullptr));
        FILE* f = fopen(path, "wb");
        if (!f) fail(SUN_ERR_IO, "cannot open %s for writing", path);
        bool ok = true;
        if (with_header) {
            int g[4] = {l->p.dims[0], l->p.dims[1], l->p.dims[2], l->p.dims[3]};
            ok &= fwrite(g, sizeof(int), 4, f) == 4;
            double beta = l->p.beta;
            ok &= fwrite(&beta, l->p.precision == SUN_F64 ? 8 : 4, 1, f) == 1;
            size_t prec = save_fp64 ? 8 : 4;
            ok &= fwrite(&prec, sizeof(size_t), 1, f) == 1;
        }
        if (save_fp64) {
            ok &= fwrite(buf.data(), sizeof(double), n, f) == n;
        } else {
            std::vector<float> t(n);
            for (size_t i = 0; i < n; ++i) t[i] = (float)buf[i];
            ok &= fwrite(t.data(), sizeof(float), n, f) == n;
        }
        ok &= fclose(f) == 0;
        if (!ok) fail(SUN_ERR_IO, "write to %s failed", path);
    });
}

sun_status sun_load_bin(sun_lattice* l, const char* path, int save_fp64, int with_header)
{
    if (!l || !path) return SUN_ERR_INVALID_ARG;
    return handle(l->ctx, [&] {
        const size_t n = (size_t)l->desc.V * 4 * l->p.ncolors * l->p.ncolors * 2;
        FILE* f = fopen(path, "rb");
        if (!f) fail(SUN_ERR_IO, "cannot open %s", path);
        std::unique_ptr<FILE, int (*)(FILE*)> guard(f, fclose);
        if (with_header) {
            int g[4];
            if (fread(g, sizeof(int), 4, f) != 4) fail(SUN_ERR_IO, "%s: short header", path);
            for (int k = 0; k < 4; ++k)
                if (g[k] != l->p.dims[k]) fail(SUN_ERR_INVALID_ARG, "%s: grid mismatch (%d vs %d in dim %d)", path, g[k], l->p.dims[k], k);
            double beta = 0;
            if (fread(&beta, l->p.precision == SUN_F64 ? 8 : 4, 1, f) != 1) fail(SUN_ERR_IO, "%s: short header", path);
            size_t prec = 0;
            if (fread(&prec, sizeof(size_t), 1, f) != 1) fail(SUN_ERR_IO, "%s: short header", path);
            if (prec != (size_t)(save_fp64 ? 8 : 4))
                fail(SUN_ERR_INVALID_ARG, "%s: stored precision %zu does not match %d", path, prec, save_fp64 ? 8 : 4);
        }
        std::vector<double> buf(n);
        if (save_fp64) {
            if (fread(buf.data(), sizeof(double), n, f) != n) fail(SUN_ERR_IO, "%s: truncated body", path);
        } else {
            std::vector<float> t(n);
            if (fread(t.data(), sizeof(float), n, f) != n) fail(SUN_ERR_IO, "%s: truncated body", path);
            for (size_t i = 0; i < n; ++i) buf[i] = t[i];
        }
        canon_upload(l, buf.data(), S(l->ctx, nullptr), false);
    });
}

}  // extern "C"

// ===========================================================================
// Batches
struct sun_batch {
    sun_ctx* ctx = nullptr;
    std::vector<sun_lattice*> order;        // insertion order
    std::vector<std::unique_ptr<Group>> groups;
    cudaGraphExec_t graph = nullptr;
    int graph_hb = -1, graph_or = -1;
    bool dirty = true;
    // one stream and join event per class: in a captured sweep the classes
    // are parallel branches
    std::vector<cudaStream_t> branch;
    std::vector<cudaEvent_t> joined;
    cudaEvent_t forked = nullptr;

    ~sun_batch()
    {
        drop_graph();
        for (auto st : branch) cudaStreamDestroy(st);
        for (auto e : joined) cudaEventDestroy(e);
        if (forked) cudaEventDestroy(forked);
    }
    void ensure_branches(size_t n)
    {
        if (!forked) ck(cudaEventCreateWithFlags(&forked, cudaEventDisableTiming), "event");
        while (branch.size() < n) {
            cudaStream_t st;
            ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
            branch.push_back(st);
            cudaEvent_t e;
            ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
            joined.push_back(e);
        }
    }
    void drop_graph()
    {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
    }
    // Regroup after membership changes.  Groups (and their device tables and
    // scratch, which only grow) are kept per class and refilled, so a server
    // that adds and retires lattices every step does not reallocate them.
    void regroup()
    {
        if (!dirty) return;
        for (auto& g : groups) {
            g->lats.clear();
            g->dirty = true;
        }
        for (auto* l : order) {
            int fp64 = l->p.precision == SUN_F64, lay = l->p.layout;
            Group* g = nullptr;
            for (auto& gg : groups)
                if (gg->N == l->p.ncolors && gg->fp64 == fp64 && gg->layout == lay) g = gg.get();
            if (!g) {
                groups.emplace_back(new Group());
                g = groups.back().get();
                g->N = l->p.ncolors;
                g->fp64 = fp64;
                g->layout = lay;
            }
            g->lats.push_back(l);
        }
        drop_graph();
        dirty = false;
    }
};

namespace {

// One sweep of every class of the batch.  branches: each class on its own
// stream, forked from s and joined back into it (inside a capture: parallel
// branches of the graph, so the classes' launches overlap on the GPU).
void batch_one_sweep(sun_batch* b, int n_hb, int n_or, cudaStream_t s, bool branches = false)
{
    std::vector<Group*> act;
    for (auto& g : b->groups)
        if (!g->lats.empty()) act.push_back(g.get());
    if (!branches || act.size() < 2) {
        for (auto* g : act) group_sweep(b->ctx, *g, n_hb, n_or, true, group_needs_reunit(*g), s);
        return;
    }
    b->ensure_branches(act.size());
    ck(cudaEventRecord(b->forked, s), "fork");
    for (size_t i = 0; i < act.size(); ++i) {
        ck(cudaStreamWaitEvent(b->branch[i], b->forked, 0), "fork");
        group_sweep(b->ctx, *act[i], n_hb, n_or, true, group_needs_reunit(*act[i]), b->branch[i]);
        ck(cudaEventRecord(b->joined[i], b->branch[i]), "join");
    }
    for (size_t i = 0; i < act.size(); ++i) ck(cudaStreamWaitEvent(s, b->joined[i], 0), "join");
}

}  // namespace

extern "C" {

sun_status sun_batch_create(sun_ctx* c, sun_batch** out)
{
    return handle(c, [&] {
        if (!c || !out) fail(SUN_ERR_INVALID_ARG, "null argument");
        auto b = std::make_unique<sun_batch>();
        b->ctx = c;
        *out = b.release();
    });
}

sun_status sun_batch_destroy(sun_batch* b)
{
    if (!b) return SUN_ERR_INVALID_ARG;
    delete b;
    return SUN_OK;
}

sun_status sun_batch_add(sun_batch* b, sun_lattice* l)
{
    if (!b || !l) return SUN_ERR_INVALID_ARG;
    return handle(b->ctx, [&] {
        need_eo(l, "batched sweeps");
        if (std::find(b->order.begin(), b->order.end(), l) != b->order.end())
            fail(SUN_ERR_INVALID_ARG, "lattice already in batch");
        b->order.push_back(l);
        b->dirty = true;
    });
}

sun_status sun_batch_remove(sun_batch* b, sun_lattice* l)
{
    if (!b || !l) return SUN_ERR_INVALID_ARG;
    return handle(b->ctx, [&] {
        auto it = std::find(b->order.begin(), b->order.end(), l);
        if (it == b->order.end()) fail(SUN_ERR_INVALID_ARG, "lattice not in batch");
        b->order.erase(it);
        b->dirty = true;
    });
}

sun_status sun_batch_size(const sun_batch* b, int* n)
{
    if (!b || !n) return SUN_ERR_INVALID_ARG;
    *n = (int)b->order.size();
    return SUN_OK;
}

sun_status sun_batch_sweep(sun_batch* b, int n_hb, int n_or, int n_sweeps, int use_graph, void* stream)
{
    if (!b || n_hb < 0 || n_or < 0 || n_sweeps < 0) return SUN_ERR_INVALID_ARG;
    return handle(b->ctx, [&] {
        b->regroup();
        cudaStream_t s = S(b->ctx, stream);
        if (b->order.empty() || n_sweeps == 0) return;
        const bool wait = !(use_graph & SUN_BATCH_NO_WAIT);
        if (!(use_graph & SUN_BATCH_GRAPH)) {
            // tables first: their uploads synchronise, which a branch stream
            // must not do in the middle of a sweep
            for (auto& g : b->groups) {
                if (g->lats.empty()) continue;
                if (n_hb > 0) upd_view(*g, update_block(b->ctx, *g, MODE_HB, s), s);
                if (n_or > 0) upd_view(*g, update_block(b->ctx, *g, MODE_OR, s), s);
                g->view(WORK_LINKS, b->ctx->blk_links, s);
            }
            for (int i = 0; i < n_sweeps; ++i) batch_one_sweep(b, n_hb, n_or, s, true);
            if (wait) ck(cudaStreamSynchronize(s), "batch sweep");
            return;
        }
        if (!b->graph || b->graph_hb != n_hb || b->graph_or != n_or) {
            b->drop_graph();
            // tables must exist before capture (their uploads synchronise)
            for (auto& g : b->groups) {
                if (g->lats.empty()) continue;
                // launch shapes (tuned if tuning is on) and their tables, before capture
                if (n_hb > 0) upd_view(*g, update_block(b->ctx, *g, MODE_HB, s), s);
                if (n_or > 0) upd_view(*g, update_block(b->ctx, *g, MODE_OR, s), s);
                g->view(WORK_LINKS, b->ctx->blk_links, s);
            }
            cudaStream_t cs;
            ck(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "stream");
            cudaGraph_t graph;
            ck(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "capture");
            b->ensure_branches(b->groups.size());  // streams and events exist before the capture
            try {
                batch_one_sweep(b, n_hb, n_or, cs, true);
            } catch (...) {
                cudaStreamEndCapture(cs, &graph);
                cudaStreamDestroy(cs);
                throw;
            }
            ck(cudaStreamEndCapture(cs, &graph), "capture end");
            cudaStreamDestroy(cs);
            cudaError_t e = cudaGraphInstantiate(&b->graph, graph, 0);
            cudaGraphDestroy(graph);
            ck(e, "graph instantiate");
            b->graph_hb = n_hb;
            b->graph_or = n_or;
        }
        for (int i = 0; i < n_sweeps; ++i) ck(cudaGraphLaunch(b->graph, s), "graph launch");
        if (wait) ck(cudaStreamSynchronize(s), "batch sweep");
    });
}

static sun_status batch_measure(sun_batch* b, double* out, void* stream, bool plaq)
{
    if (!b || !out) return SUN_ERR_INVALID_ARG;
    return handle(b->ctx, [&] {
        b->regroup();
        cudaStream_t s = S(b->ctx, stream);
        for (auto& g : b->groups) {
            if (g->lats.empty()) continue;
            std::vector<double> r(2 * g->lats.size());
            if (plaq) group_plaquette(b->ctx, *g, r.data(), s);
            else group_polyakov(b->ctx, *g, r.data(), s);
            for (size_t i = 0; i < g->lats.size(); ++i) {
                size_t pos = std::find(b->order.begin(), b->order.end(), g->lats[i]) - b->order.begin();
                out[2 * pos] = r[2 * i];
                out[2 * pos + 1] = r[2 * i + 1];
            }
        }
    });
}

sun_status sun_batch_plaquette(sun_batch* b, double* out, void* stream) { return batch_measure(b, out, stream, true); }

sun_status sun_batch_wilson_loops(sun_batch* b, int R, int T, double* out, void* stream)
{
    if (!b || !out) return SUN_ERR_INVALID_ARG;
    return handle(b->ctx, [&] {
        if (R < 0 || T < 0 || R > 8 || T > 8) fail(SUN_ERR_INVALID_ARG, "Wilson loops need 0 <= R, T <= 8");
        for (auto* l : b->order) {
            for (int d = 0; d < 3; ++d)
                if (R >= l->p.dims[d]) fail(SUN_ERR_INVALID_ARG, "R=%d not below spatial extent %d", R, l->p.dims[d]);
            if (T >= l->p.dims[3]) fail(SUN_ERR_INVALID_ARG, "T=%d not below temporal extent", T);
        }
        b->regroup();
        cudaStream_t s = S(b->ctx, stream);
        const int nv = 2 * (R + 1) * (T + 1);
        const int blk = b->ctx->blk_wilson;
        for (auto& g : b->groups) {
            if (g->lats.empty()) continue;
            double* r = group_reduce(*g, WORK_SITES, blk, nv, false, s, [&](const BatchView& v, double* part) {
                OPS_CALL(g->N, wilson, g->fp64, g->layout, v, blk, R, T, part, s);
            });
            for (size_t i = 0; i < g->lats.size(); ++i) {
                const size_t pos = std::find(b->order.begin(), b->order.end(), g->lats[i]) - b->order.begin();
                const double norm = 3.0 * g->N * (double)g->lats[i]->desc.V;
                for (int k = 0; k < nv; ++k) out[pos * nv + k] = r[i * nv + k] / norm;
            }
        }
    });
}
sun_status sun_batch_polyakov(sun_batch* b, double* out, void* stream) { return batch_measure(b, out, stream, false); }

}  // extern "C"
