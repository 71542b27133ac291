// server.cu -- continuous-batching job server over the batch engine.
//
// A job is (N, L^3 x T, beta, sweeps, observables).  Jobs queue FIFO; each
// scheduling step admits queued jobs while a slot is free and their HBM
// footprint fits the budget, advances every active job by up to K sweeps --
// all active lattices of one (n_hb, n_or) kind replayed from one captured
// graph, the (N, precision, layout) classes as parallel branches of it --
// then measures the jobs that finished in one batched launch per class and
// observable and retires them.  Each job's lattice carries its sweep count as
// a device-side limit, so a job that finishes inside a step sits out the
// rest of it unchanged: K only sets how often the host admits and retires
// (K is chosen so a step lasts about step_target_s).  Links and RNG counters
// stay on the device for a job's whole life.  Because the random stream of a
// link is keyed only by (seed, site, direction, heatbath pass) and the
// reductions are per-lattice and fixed-order, a job's result does not depend
// on which other jobs shared its launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <vector>

#include "../../include/sun_b200.h"

namespace {

double clock_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

size_t links_bytes(const sun_job* j)
{
    const size_t V = (size_t)j->dims[0] * j->dims[1] * j->dims[2] * j->dims[3];
    const size_t csz = j->precision == SUN_F64 ? 16 : 8;
    const size_t ne = j->layout == SUN_SOA12 ? 6 : (j->layout == SUN_SOA8 ? 4 : (size_t)j->ncolors * j->ncolors);
    return csz * ne * 4 * V;
}

}  // namespace

extern "C" {

sun_status sun_job_footprint(const sun_job* j, size_t* bytes)
{
    if (!j || !bytes) return SUN_ERR_INVALID_ARG;
    const size_t V = (size_t)j->dims[0] * j->dims[1] * j->dims[2] * j->dims[3];
    size_t scratch = 64 * V / 128 + 4096;  // plaquette / Polyakov partials
    if (j->observables & 4) {
        const size_t nv = 2 * (size_t)(j->wilson_R + 1) * (j->wilson_T + 1);
        scratch += (V / 64 + 1) * nv * 16;
    }
    *bytes = links_bytes(j) + scratch + (1u << 16);
    return SUN_OK;
}

// Admission rule shared by the server and its host-side tests: admit queued
// jobs in FIFO order while a slot is free and the footprint fits; stop at
// the first job that does not fit (no overtaking, so no starvation).
sun_status sun_admit_count(const size_t* footprints, int n_queued, size_t budget, size_t used, int free_slots,
                           int* n_admit)
{
    if (!n_admit || n_queued < 0 || (n_queued > 0 && !footprints)) return SUN_ERR_INVALID_ARG;
    int n = 0;
    while (n < n_queued && n < free_slots && used + footprints[n] <= budget) {
        used += footprints[n];
        ++n;
    }
    *n_admit = n;
    return SUN_OK;
}

}  // extern "C"

struct sun_server {
    struct Pending {
        int64_t id;
        sun_job job;
        double submit_s;
    };
    struct Active {
        int64_t id;
        sun_job job;
        sun_lattice* lat;
        int remaining;
        double submit_s, start_s;
        size_t bytes;
    };
    sun_ctx* ctx = nullptr;
    int max_active = 0;
    size_t budget = 0, used = 0;
    std::deque<Pending> queue;
    std::vector<Active> active;
    std::map<std::pair<int, int>, sun_batch*> batches;
    sun_batch* retiring = nullptr;  // the jobs measured together at a step's end
    std::deque<sun_result> outbox;  // finished results not yet returned
    int64_t next_id = 1;
    double t0 = 0;
    // sweeps per step: about step_target_s of GPU work, at most k_max
    double step_target_s = 0.05, sweep_s = 0.0;
    int k_max = 16;
    // the step's sweeps and measurements run on `work` while new jobs'
    // lattices are set up on `side`; t_sweep brackets the sweeps
    cudaStream_t work = nullptr, side = nullptr;
    cudaEvent_t t_sweep[2] = {nullptr, nullptr};
    std::vector<Active> admitted;  // set up during the last step, not yet in a batch
    sun_server_stats stats{};

    ~sun_server()
    {
        for (auto& a : active) sun_lattice_destroy(a.lat);
        for (auto& a : admitted) sun_lattice_destroy(a.lat);
        for (auto& kv : batches) sun_batch_destroy(kv.second);
        if (retiring) sun_batch_destroy(retiring);
        if (side) cudaStreamDestroy(side);
        if (work) cudaStreamDestroy(work);
        for (auto e : t_sweep)
            if (e) cudaEventDestroy(e);
    }
    double now() const { return clock_s() - t0; }
    sun_batch* batch_for(const sun_job& j)
    {
        auto key = std::make_pair(j.n_hb, j.n_or);
        auto it = batches.find(key);
        if (it != batches.end()) return it->second;
        sun_batch* b = nullptr;
        if (sun_batch_create(ctx, &b) != SUN_OK) return nullptr;
        batches[key] = b;
        return b;
    }
};

namespace {

bool job_valid(const sun_job* j)
{
    if (j->sweeps < 0 || j->n_hb < 0 || j->n_or < 0) return false;
    if (j->observables & 4) {
        if (j->wilson_R < 0 || j->wilson_T < 0 || j->wilson_R > 8 || j->wilson_T > 8) return false;
    }
    return true;
}

sun_result blank_result(int64_t id, sun_status st, double submit)
{
    sun_result r;
    memset(&r, 0, sizeof r);
    r.id = id;
    r.status = st;
    r.submit_s = submit;
    return r;
}

}  // namespace

extern "C" {

sun_status sun_server_create(sun_ctx* ctx, int max_active, sun_server** out)
{
    if (!ctx || !out || max_active <= 0) return SUN_ERR_INVALID_ARG;
    sun_server* s = new sun_server();
    s->ctx = ctx;
    s->max_active = max_active;
    // the context's admission budget (sun_config.hbm_budget_bytes, or 90 %
    // of the free memory at sun_init)
    if (sun_ctx_hbm_budget(ctx, &s->budget) != SUN_OK || sun_batch_create(ctx, &s->retiring) != SUN_OK) {
        delete s;
        return SUN_ERR_INVALID_ARG;
    }
    if (cudaStreamCreateWithFlags(&s->work, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&s->t_sweep[0]) != cudaSuccess || cudaEventCreate(&s->t_sweep[1]) != cudaSuccess) {
        delete s;
        return SUN_ERR_CUDA;
    }
    s->t0 = clock_s();
    *out = s;
    return SUN_OK;
}

sun_status sun_server_set_budget(sun_server* s, size_t bytes)
{
    if (!s) return SUN_ERR_INVALID_ARG;
    s->budget = bytes;
    return SUN_OK;
}

sun_status sun_server_destroy(sun_server* s)
{
    if (!s) return SUN_ERR_INVALID_ARG;
    delete s;
    return SUN_OK;
}

sun_status sun_server_submit(sun_server* s, const sun_job* job, int64_t* id)
{
    if (!s || !job) return SUN_ERR_INVALID_ARG;
    sun_server::Pending p;
    p.id = s->next_id++;
    p.job = *job;
    p.submit_s = s->now();
    if (!job_valid(job)) {
        s->outbox.push_back(blank_result(p.id, SUN_ERR_INVALID_ARG, p.submit_s));
    } else {
        size_t f = 0;
        sun_job_footprint(job, &f);
        if (f > s->budget) s->outbox.push_back(blank_result(p.id, SUN_ERR_CAPACITY, p.submit_s));
        else s->queue.push_back(p);
    }
    if (id) *id = p.id;
    return SUN_OK;
}

sun_status sun_server_pending(const sun_server* s, int* queued, int* active)
{
    if (!s) return SUN_ERR_INVALID_ARG;
    if (queued) *queued = (int)s->queue.size();
    if (active) *active = (int)(s->active.size() + s->admitted.size());
    return SUN_OK;
}

sun_status sun_server_get_stats(const sun_server* s, sun_server_stats* out)
{
    if (!s || !out) return SUN_ERR_INVALID_ARG;
    *out = s->stats;
    return SUN_OK;
}

sun_status sun_server_step(sun_server* s, sun_result* out, int cap, int* n_done)
{
    if (!s || !n_done || (cap > 0 && !out)) return SUN_ERR_INVALID_ARG;
    auto emit = [&](const sun_result& r) { s->outbox.push_back(r); };
    double tick = s->now();
    auto lap = [&](double& acc) {
        const double t = s->now();
        acc += t - tick;
        tick = t;
    };
    // 1. queue up to K sweeps of every active job, batched per (n_hb, n_or),
    // on the work stream without waiting; a job with fewer sweeps left
    // stops at its own count (device-side limit)
    int left_max = 0;
    for (auto& a : s->active) left_max = std::max(left_max, a.remaining);
    int k = 0;
    if (left_max > 0) {
        k = s->sweep_s > 0 ? (int)(s->step_target_s / s->sweep_s + 0.5) : 1;
        k = std::max(1, std::min(std::min(k, s->k_max), left_max));
        cudaEventRecord(s->t_sweep[0], s->work);
        for (auto& kv : s->batches) {
            int n = 0;
            sun_batch_size(kv.second, &n);
            if (n == 0) continue;
            sun_status st = sun_batch_sweep(kv.second, kv.first.first, kv.first.second, k, SUN_BATCH_NO_WAIT, s->work);
            if (st != SUN_OK) return st;
        }
    }
    lap(s->stats.enqueue_s);
    // 2. meanwhile admit queued jobs: their lattices are allocated and
    // initialized on the side stream while the GPU sweeps, and join their
    // batches after this step's sweeps
    {
        std::vector<size_t> fp;
        for (auto& p : s->queue) {
            size_t f = 0;
            sun_job_footprint(&p.job, &f);
            fp.push_back(f);
        }
        int n_admit = 0;
        const int slots = s->max_active - (int)(s->active.size() + s->admitted.size());
        sun_admit_count(fp.data(), (int)fp.size(), s->budget, s->used, slots, &n_admit);
        for (int i = 0; i < n_admit; ++i) {
            sun_server::Pending p = s->queue.front();
            const sun_job& j = p.job;
            sun_lattice_params lp;
            memset(&lp, 0, sizeof lp);
            lp.ncolors = j.ncolors;
            for (int d = 0; d < 4; ++d) lp.dims[d] = j.dims[d];
            lp.beta = j.beta;
            lp.layout = j.layout;
            lp.order = SUN_EVEN_ODD;
            lp.precision = j.precision;
            lp.seed = j.seed;
            lp.reunit_every = j.reunit_every;
            sun_lattice* lat = nullptr;
            sun_status st = sun_lattice_create(s->ctx, &lp, &lat);
            if (st == SUN_ERR_OUT_OF_MEMORY) break;  // retry at the next step
            s->queue.pop_front();
            if (st == SUN_OK) st = j.hot_start ? sun_lattice_init_hot(lat, s->side) : sun_lattice_init_cold(lat, s->side);
            if (st == SUN_OK) st = sun_lattice_set_sweep_limit(lat, (uint32_t)j.sweeps);
            if (st == SUN_OK && j.sweeps > 0 && !s->batch_for(j)) st = SUN_ERR_CUDA;
            if (st != SUN_OK) {
                if (lat) sun_lattice_destroy(lat);
                emit(blank_result(p.id, st, p.submit_s));
                continue;
            }
            sun_server::Active a;
            a.id = p.id;
            a.job = j;
            a.lat = lat;
            a.remaining = j.sweeps;
            a.submit_s = p.submit_s;
            a.start_s = s->now();
            a.bytes = fp[i];
            s->used += a.bytes;
            s->admitted.push_back(a);
        }
    }
    lap(s->stats.admit_s);
    // 3. the sweeps done: seconds per sweep (CUDA events) for the next K
    if (k > 0) {
        cudaEventRecord(s->t_sweep[1], s->work);
        if (cudaEventSynchronize(s->t_sweep[1]) != cudaSuccess) return SUN_ERR_CUDA;
        lap(s->stats.wait_s);
        float ms = 0;
        cudaEventElapsedTime(&ms, s->t_sweep[0], s->t_sweep[1]);
        s->stats.steps += 1;
        s->stats.sweeps += k;
        s->stats.sweep_gpu_s += 1e-3 * ms;
        const double per = 1e-3 * ms / k;
        s->sweep_s = s->sweep_s > 0 ? 0.5 * (s->sweep_s + per) : per;
        for (auto& a : s->active) a.remaining = std::max(0, a.remaining - k);
    }
    // 4. measure the finished jobs together (one launch per class and
    // observable), then retire them
    std::vector<sun_server::Active> keep, fin;
    for (auto& a : s->active) (a.remaining > 0 ? keep : fin).push_back(a);
    if (!fin.empty()) {
        std::vector<sun_result> res(fin.size());
        std::vector<sun_status> stat(fin.size(), SUN_OK);
        for (size_t i = 0; i < fin.size(); ++i) {
            res[i] = blank_result(fin[i].id, SUN_OK, fin[i].submit_s);
            res[i].start_s = fin[i].start_s;
        }
        auto measure = [&](int bit, int R, int T) {
            std::vector<size_t> idx;
            for (size_t i = 0; i < fin.size(); ++i)
                if ((fin[i].job.observables & bit) && stat[i] == SUN_OK &&
                    (bit != 4 || (fin[i].job.wilson_R == R && fin[i].job.wilson_T == T)))
                    idx.push_back(i);
            if (idx.empty()) return;
            for (size_t i : idx) sun_batch_add(s->retiring, fin[i].lat);
            const int nv = bit == 4 ? 2 * (R + 1) * (T + 1) : 2;
            std::vector<double> out(nv * idx.size());
            sun_status st = bit == 1   ? sun_batch_plaquette(s->retiring, out.data(), s->work)
                            : bit == 2 ? sun_batch_polyakov(s->retiring, out.data(), s->work)
                                       : sun_batch_wilson_loops(s->retiring, R, T, out.data(), s->work);
            for (size_t q = 0; q < idx.size(); ++q) {
                const size_t i = idx[q];
                if (st != SUN_OK) stat[i] = st;
                else if (bit == 1) memcpy(res[i].plaquette, &out[2 * q], 2 * sizeof(double));
                else if (bit == 2) memcpy(res[i].polyakov, &out[2 * q], 2 * sizeof(double));
                else memcpy(res[i].wilson, &out[nv * q], nv * sizeof(double));
                sun_batch_remove(s->retiring, fin[i].lat);
            }
        };
        measure(1, 0, 0);
        measure(2, 0, 0);
        std::vector<std::pair<int, int>> rts;
        for (auto& a : fin)
            if ((a.job.observables & 4) &&
                std::find(rts.begin(), rts.end(), std::make_pair(a.job.wilson_R, a.job.wilson_T)) == rts.end())
                rts.emplace_back(a.job.wilson_R, a.job.wilson_T);
        for (auto& rt : rts) measure(4, rt.first, rt.second);
        for (size_t i = 0; i < fin.size(); ++i) {
            sun_server::Active& a = fin[i];
            sun_result& r = res[i];
            r.status = stat[i];
            r.finish_s = s->now();
            const double V = (double)a.job.dims[0] * a.job.dims[1] * a.job.dims[2] * a.job.dims[3];
            r.link_updates = (double)a.job.sweeps * (a.job.n_hb + a.job.n_or) * 4.0 * V;
            if (a.job.sweeps > 0) sun_batch_remove(s->batch_for(a.job), a.lat);
            sun_lattice_destroy(a.lat);
            s->used -= a.bytes;
            emit(r);
        }
    }
    s->active.swap(keep);
    lap(s->stats.retire_s);
    // 5. the jobs admitted during this step join their batches (from the
    // next step on); jobs without sweeps are finished as they stand
    for (auto& a : s->admitted) {
        if (a.job.sweeps > 0 && sun_batch_add(s->batch_for(a.job), a.lat) != SUN_OK) {
            sun_result r = blank_result(a.id, SUN_ERR_CUDA, a.submit_s);
            sun_lattice_destroy(a.lat);
            s->used -= a.bytes;
            emit(r);
            continue;
        }
        s->active.push_back(a);
    }
    s->admitted.clear();
    lap(s->stats.join_s);
    int done = 0;
    while (done < cap && !s->outbox.empty()) {
        out[done++] = s->outbox.front();
        s->outbox.pop_front();
    }
    *n_done = done;
    return SUN_OK;
}

}  // extern "C"
