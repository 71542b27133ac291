// server.cu -- continuous-batching job server over the batch engine.
//
// A job is (N, L^3 x T, beta, sweeps, observables).  Jobs queue FIFO; each
// scheduling step admits queued jobs while a slot is free and their HBM
// footprint fits the budget, advances every active job by one sweep -- all
// active lattices of one (n_hb, n_or) kind in one batched launch per phase --
// then measures and retires the jobs that finished.  Links and RNG counters
// stay on the device for a job's whole life.  Because the random stream of a
// link is keyed only by (seed, site, direction, heatbath pass) and the
// reductions are per-lattice and fixed-order, a job's result does not depend
// on which other jobs shared its launches.
#include <cuda_runtime.h>

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
    std::deque<sun_result> outbox;  // finished results not yet returned
    int64_t next_id = 1;
    double t0 = 0;

    ~sun_server()
    {
        for (auto& a : active) sun_lattice_destroy(a.lat);
        for (auto& kv : batches) sun_batch_destroy(kv.second);
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
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
        delete s;
        return SUN_ERR_CUDA;
    }
    s->budget = (size_t)(0.85 * (double)fr);
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
    if (active) *active = (int)s->active.size();
    return SUN_OK;
}

sun_status sun_server_step(sun_server* s, sun_result* out, int cap, int* n_done)
{
    if (!s || !n_done || (cap > 0 && !out)) return SUN_ERR_INVALID_ARG;
    auto emit = [&](const sun_result& r) { s->outbox.push_back(r); };
    // 1. admission
    {
        std::vector<size_t> fp;
        for (auto& p : s->queue) {
            size_t f = 0;
            sun_job_footprint(&p.job, &f);
            fp.push_back(f);
        }
        int n_admit = 0;
        sun_admit_count(fp.data(), (int)fp.size(), s->budget, s->used, s->max_active - (int)s->active.size(),
                        &n_admit);
        for (int i = 0; i < n_admit; ++i) {
            sun_server::Pending p = s->queue.front();
            const sun_job& j = p.job;
            sun_lattice_params lp;
            memset(&lp, 0, sizeof lp);
            lp.ncolors = j.ncolors;
            for (int k = 0; k < 4; ++k) lp.dims[k] = j.dims[k];
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
            if (st == SUN_OK) st = j.hot_start ? sun_lattice_init_hot(lat, nullptr) : sun_lattice_init_cold(lat, nullptr);
            sun_batch* b = (st == SUN_OK && j.sweeps > 0) ? s->batch_for(j) : nullptr;
            if (st == SUN_OK && j.sweeps > 0 && !b) st = SUN_ERR_CUDA;
            if (st == SUN_OK && b) st = sun_batch_add(b, lat);
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
            s->active.push_back(a);
        }
    }
    // 2. one sweep of every active job, batched per (n_hb, n_or)
    for (auto& kv : s->batches) {
        int n = 0;
        sun_batch_size(kv.second, &n);
        if (n == 0) continue;
        // only lattices with sweeps left are in a batch
        sun_status st = sun_batch_sweep(kv.second, kv.first.first, kv.first.second, 1, 0, nullptr);
        if (st != SUN_OK) return st;
    }
    // 3. retire
    std::vector<sun_server::Active> keep;
    for (auto& a : s->active) {
        if (a.remaining > 0) --a.remaining;
        if (a.remaining > 0) {
            keep.push_back(a);
            continue;
        }
        sun_result r = blank_result(a.id, SUN_OK, a.submit_s);
        r.start_s = a.start_s;
        sun_status st = SUN_OK;
        if (a.job.observables & 1) st = sun_plaquette(a.lat, r.plaquette, nullptr);
        if (st == SUN_OK && (a.job.observables & 2)) st = sun_polyakov(a.lat, r.polyakov, nullptr);
        if (st == SUN_OK && (a.job.observables & 4)) st = sun_wilson_loops(a.lat, a.job.wilson_R, a.job.wilson_T, r.wilson, nullptr);
        r.status = st;
        r.finish_s = s->now();
        const double V = (double)a.job.dims[0] * a.job.dims[1] * a.job.dims[2] * a.job.dims[3];
        r.link_updates = (double)a.job.sweeps * (a.job.n_hb + a.job.n_or) * 4.0 * V;
        if (a.job.sweeps > 0) sun_batch_remove(s->batch_for(a.job), a.lat);
        sun_lattice_destroy(a.lat);
        s->used -= a.bytes;
        emit(r);
    }
    s->active.swap(keep);
    int done = 0;
    while (done < cap && !s->outbox.empty()) {
        out[done++] = s->outbox.front();
        s->outbox.pop_front();
    }
    *n_done = done;
    return SUN_OK;
}

}  // extern "C"
