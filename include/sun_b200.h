/*
 * sun_b200.h -- C ABI of the B200-native SU(N) quenched lattice gauge engine.
 *
 * Drop-in boundary for the hot path of nmrcardoso/sun (CULQCD): gauge-array
 * allocation and layouts, the heatbath / overrelaxation Monte Carlo sweep,
 * reunitarization, and plaquette / Polyakov-loop / Wilson-loop measurements,
 * plus batched many-lattice execution and a continuous-batching server on one
 * GPU.  Each declaration names the reference interface it replaces
 * (paths relative to the reference project root).
 *
 * Conventions
 *  - Every call returns a sun_status; nothing here calls exit() (the
 *    reference's errorCULQCD / CUDA_SAFE_CALL exit the process,
 *    include/comm_mpi.h:102-116, include/cuda_common.h:136-205).
 *    sun_last_error_string() gives the message of the last failure.
 *  - `stream` is a cudaStream_t passed as void* (NULL = the context stream).
 *    Calls that return host values synchronise that stream.
 *  - The library owns all device memory; callers own handles.
 *  - Host lattice buffers: SUN_HOST_CANONICAL is double complex
 *    U[V][4][N][N] with sites in x-fastest lexicographic order, the record
 *    order of the reference gauge file (src/io_gauge.cpp:544-563);
 *    SUN_HOST_IMAGE is the raw device image (layout, order and precision of
 *    the lattice), what a reference `gauge` in Host mode holds.
 */
#ifndef SUN_B200_H
#define SUN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    SUN_OK = 0,
    SUN_ERR_INVALID_ARG = 1,
    SUN_ERR_UNSUPPORTED = 2,
    SUN_ERR_OUT_OF_MEMORY = 3,
    SUN_ERR_CUDA = 4,
    SUN_ERR_IO = 5,
    SUN_ERR_STATE = 6,
    SUN_ERR_CAPACITY = 7,
    SUN_ERR_DEVICE_FLAG = 8
} sun_status;

/* ArrayType (include/modes.h:66-71): SOA = N*N complex, SOA12 = 2 rows (SU(3)),
 * SOA8 = 8 reals (SU(3)).  SOA12A (anti-Hermitian storage for gauge fixing) is
 * out of scope. */
typedef enum { SUN_SOA = 0, SUN_SOA12 = 1, SUN_SOA8 = 2 } sun_layout;
typedef enum { SUN_EVEN_ODD = 0, SUN_NORMAL = 1 } sun_order;
typedef enum { SUN_F32 = 0, SUN_F64 = 1 } sun_precision;
typedef enum { SUN_HOST_CANONICAL = 0, SUN_HOST_IMAGE = 1 } sun_host_format;

typedef struct sun_ctx sun_ctx;
typedef struct sun_lattice sun_lattice;
typedef struct sun_batch sun_batch;
typedef struct sun_server sun_server;

typedef struct {
    int device;            /* CUDA device ordinal (initCULQCD gpuid) */
    int verbosity;         /* 0 silent .. 3 debug (Verbosity, include/modes.h:74-79) */
    int tune;              /* 1: autotune launch shapes (TuneMode) */
    const char *tune_cache_path; /* CSV cache file, NULL: none ($CULQCD_RESOURCE_PATH/tunecache.csv) */
    size_t hbm_budget_bytes;     /* admission budget for the server; 0: 90% of free memory */
} sun_config;

typedef struct {
    int ncolors;           /* N in {2,3,4,6} (the reference's compile-time NCOLORS, Makefile:6) */
    int dims[4];           /* X, Y, Z, T; all even (constants.cu:170-174) */
    double beta;
    sun_layout layout;
    sun_order order;
    sun_precision precision;
    uint64_t seed;         /* Philox key of this lattice */
    int reunit_every;      /* FP64 reunitarization every k sweeps inside sun_sweep (0: never) */
} sun_lattice_params;

/* ---- lifecycle: initCULQCD / EndCULQCD (src/comm_mpi.cpp:107, :186) ---- */
sun_status sun_init(const sun_config *cfg, sun_ctx **out);
sun_status sun_finalize(sun_ctx *ctx);
const char *sun_last_error_string(const sun_ctx *ctx);
/* the context's device-memory admission budget: sun_config.hbm_budget_bytes,
 * or 90% of the free memory at sun_init; servers admit jobs against it */
sun_status sun_ctx_hbm_budget(const sun_ctx *ctx, size_t *bytes);
const char *sun_version(void);
/* host-side fault injection for tests (no reference counterpart): after
 * after_n more device allocations succeed, every further one reports
 * SUN_ERR_OUT_OF_MEMORY without calling the allocator; -1 turns it off */
sun_status sun_debug_fail_allocations(int after_n);
/* test hook of the resident sweeps (no reference counterpart): wait_ns
 * bounds each grid barrier wait of k_sweeps_resident (<= 0: one second);
 * skip_cta >= 0 makes that CTA leave at its first barrier without
 * arriving, so the other CTAs' waits run out and sun_sweep_measure reports
 * SUN_ERR_DEVICE_FLAG with the links part-updated (-1: off) */
sun_status sun_debug_resident_barrier(sun_ctx *ctx, long long wait_ns, int skip_cta);

/* ---- gauge arrays: _gauge<Real>(ArrayType, Device, 4V, evenodd) + Allocate
 * (include/gaugearray.h:139, :603) with SETPARAMS geometry
 * (src/constants.cu:149) made per-lattice. ---- */
sun_status sun_lattice_create(sun_ctx *ctx, const sun_lattice_params *p, sun_lattice **out);
sun_status sun_lattice_destroy(sun_lattice *lat);
sun_status sun_lattice_bytes(const sun_lattice *lat, size_t *bytes);
/* raw device pointer of the image (the reference's gauge::GetPtr) */
sun_status sun_lattice_device_ptr(const sun_lattice *lat, void **dptr);
/* ColdStart / HotStart (src/gaugearray.cu:290, :388); the hot start is Haar */
sun_status sun_lattice_init_cold(sun_lattice *lat, void *stream);
sun_status sun_lattice_init_hot(sun_lattice *lat, void *stream);
/* host <-> device (gauge::Copy + cudaMemcpy of the reference) */
sun_status sun_lattice_upload(sun_lattice *lat, const void *host, sun_host_format fmt, void *stream);
sun_status sun_lattice_download(sun_lattice *lat, void *host, sun_host_format fmt, void *stream);
/* Raw-image transfers that return at once (no reference counterpart: the
 * reference's gauge::Copy is synchronous).  The copy is queued on `stream`
 * and nothing waits for it; `host_image` (SUN_HOST_IMAGE format, sun_lattice_bytes
 * long) must be page-locked for the copy to overlap other work, and must stay
 * valid and untouched until the stream has passed the copy.  Order copies
 * against sweeps on other streams with events. */
sun_status sun_lattice_upload_async(sun_lattice *lat, const void *host_image, void *stream);
sun_status sun_lattice_download_async(sun_lattice *lat, void *host_image, void *stream);
/* layout / order / precision conversion, gauge::Copy (src/gaugearray.cu:130) */
sun_status sun_lattice_copy(sun_lattice *dst, sun_lattice *src, void *stream);
/* Sweep limit (no reference counterpart): once the lattice's sweep counter
 * reaches `limit`, sweeps leave it unchanged -- the update launches skip it,
 * its counters and its reunitarization schedule stop -- so a batch can run
 * more sweeps than some of its lattices need and each still ends after
 * exactly its own count.  0 (the default) means no limit. */
sun_status sun_lattice_set_sweep_limit(sun_lattice *lat, uint32_t limit);
/* RNG state for checkpoint: RNG::Save / RNG::Read (src/random.cu:164, :183);
 * with Philox the state is (seed, heatbath-pass counter, sweep counter) */
sun_status sun_lattice_get_rng(sun_lattice *lat, uint64_t *seed, uint32_t *hb_passes, uint32_t *sweeps);
sun_status sun_lattice_set_rng(sun_lattice *lat, uint64_t seed, uint32_t hb_passes, uint32_t sweeps);

/* ---- Monte Carlo: HeatBath<Real>::Run (src/monte/monte.cu:196),
 * OverRelaxation<Real>::Run (src/monte/ovr.cu:182).  Even/odd arrays only,
 * like the reference kernels. ---- */
sun_status sun_heatbath(sun_lattice *lat, int n_passes, void *stream);
sun_status sun_overrelax(sun_lattice *lat, int n_passes, void *stream);
/* n_sweeps x (n_hb heatbath + n_or overrelaxation); reunitarizes after every
 * reunit_every-th sweep (lattice parameter) */
sun_status sun_sweep(sun_lattice *lat, int n_hb, int n_or, int n_sweeps, void *stream);
/* n_sweeps sweeps of (n_hb heatbath + n_or overrelaxation) with the
 * plaquette and the Polyakov loop measured after every sweep -- the
 * reference driver's loop of HeatBath::Run, OverRelaxation::Run,
 * PlaquetteCUB::Run and OnePolyakovLoop::Run (src/monte/monte.cu:196,
 * src/monte/ovr.cu:182, src/meas/plaquette_cub.cu:226,
 * src/meas/polyakovloop.cu:637) in one call, with the same results as
 * sun_sweep + sun_plaquette + sun_polyakov per sweep.  plaq[2i], plaq[2i+1]:
 * spatial and temporal plaquette after sweep i; poly[2i], poly[2i+1]:
 * Polyakov loop; host arrays of 2 n_sweeps doubles, either may be NULL.
 * A small SU(3) FP32 lattice (at most 16384 half-sites; SUN_B200_RESIDENT=
 * 0|1|auto, SUN_B200_RESIDENT_MAX_HALFV) runs its sweeps in cooperative
 * launches of up to 256 sweeps whose grid barriers replace the launch
 * boundaries, with the same results; a barrier wait that runs out (one second) returns
 * SUN_ERR_DEVICE_FLAG. */
sun_status sun_sweep_measure(sun_lattice *lat, int n_hb, int n_or, int n_sweeps, double *plaq, double *poly,
                             void *stream);
/* one heatbath pass fed caller uniforms (oracle parity): device buffer
 * u[(lex*4 + mu)*stride + k]; running out sets SUN_ERR_DEVICE_FLAG */
sun_status sun_heatbath_injected(sun_lattice *lat, const double *dev_uniforms, int stride, void *stream);

/* Test hook (no reference counterpart): n draws of the SU(2) heatbath
 * element for a fixed alpha on the current device, in the given arithmetic,
 * exactly as the update kernels make them -- the restatement of
 * generate_su2_matrix_milc (include/device_PHB_OVR.h:163-223): Kennedy-Pendleton
 * for alpha > 2, Creutz otherwise, 20 retries.  Draw i reads the Philox
 * stream (seed, i, 0, pass 0).  out: host buffer of 4 n doubles
 * (a0, a1, a2, a3) per draw; 0 < n <= 2^26.  Errors through
 * sun_last_error_string(NULL). */
sun_status sun_debug_su2_draws(sun_precision prec, double alpha, uint64_t seed, int n, double *out);

/* ---- Reunitarize<Real>::Run (src/reunitarize.cu:78), FP64 arithmetic ---- */
sun_status sun_reunitarize(sun_lattice *lat, void *stream);
/* max over links of max_ij |(U^dag U - 1)_ij| */
sun_status sun_unitarity_violation(sun_lattice *lat, double *out, void *stream);
/* link diagnostics: GaugeTraceCUB (src/meas/linktrsum.cu:146, mean tr U / N)
 * and GaugeDetCUB (src/meas/linkdetsum.cu:115, mean det U) in one pass:
 * out = {Re, Im of mean tr U / N, Re, Im of mean det U} */
sun_status sun_link_trace_det(sun_lattice *lat, double out[4], void *stream);

/* ---- measurements (FP64 results, deterministic compensated sums) ----
 * PlaquetteCUB<Real>::Run -> {spatial, temporal} (src/meas/plaquette_cub.cu:226)
 * OnePolyakovLoop<Real>::Run -> {re, im} (src/meas/polyakovloop.cu:637)
 * WilsonLoop<Real>(gauge, res, R, T) -> res[t + r(T+1)] complex
 *   (src/meas/wilsonloop.cu:535); R, T <= 8; any storage order accepted. */
sun_status sun_plaquette(sun_lattice *lat, double out[2], void *stream);
/* The plaquette for callers that cannot allocate device memory (no
 * counterpart in the reference).  sun_plaquette() lets the library
 * cudaMalloc its reduction scratch on first use; applications that own all
 * device memory through their own pool, hosts with a fixed memory budget and
 * loops that cannot afford the synchronisation of a later cudaFree cannot
 * allow that.  This entry point allocates
 * nothing: its scratch is a fixed 2 MiB array compiled into the library
 * (held on every GPU that loads it), so lattices of at most 8,388,608 sites
 * are accepted and larger ones are rejected with SUN_ERR_CAPACITY.
 * d_links: device image with the layout, order and precision given in p
 * (p->beta, p->seed, p->reunit_every are ignored); d_out: device memory for
 * 2 doubles {spatial, temporal}, written asynchronously on `stream`.  The
 * first call on each device looks up the scratch address (no allocation);
 * make that first call before any stream capture.  All calls share the
 * scratch: calls that overlap on the GPU race.  The looked-up address is kept
 * for the process's life: after cudaDeviceReset on a device, do not call this
 * entry point on that device again.  Errors: status code plus
 * sun_last_error_string(NULL). */
sun_status sun_plaquette_noalloc(const void *d_links, const sun_lattice_params *p, double *d_out, void *stream);
sun_status sun_polyakov(sun_lattice *lat, double out[2], void *stream);
sun_status sun_wilson_loops(sun_lattice *lat, int R, int T, double *out, void *stream);

/* ---- smearing and multihit (src/smear/) ----
 * dirmask: bit mu selects direction mu; SUN_SMEAR_SPACE (x, y, z) is the
 * reference's "...inSpace", SUN_SMEAR_TIME its "...inTime".  Each step
 * rebuilds the selected directions from the unchanged field, in place.  Any
 * layout and storage order is accepted (the reference takes normal-order SOA
 * only).  Projections onto SU(N) use Cabibbo-Marinari SU(2) hits:
 * project_link (include/projectlink.h:17) from the unsmeared link, stopping
 * at relative change <= tol, or for SU(3) APE SU3project (projectlink.h:119)
 * from the unit matrix with nhits hits. */
#define SUN_SMEAR_SPACE 7
#define SUN_SMEAR_TIME 8
/* ApplyAPEinSpace / ApplyAPEinTime (src/smear/ape.cu:192, :237):
 * U' = P[(U + w S) / (1 + 6 w)], S the staple over the spatial planes */
sun_status sun_smear_ape(sun_lattice *lat, double w, int steps, int nhits, double tol, int dirmask,
                         void *stream);
/* ApplyStoutinSpace / ApplyStoutinTime (src/smear/stout.cu:687, :734), SU(3)
 * only (SUN_ERR_UNSUPPORTED otherwise): U' = exp(iQ) U, Q the traceless
 * Hermitian part of -i (w S) U^dagger */
sun_status sun_smear_stout(sun_lattice *lat, double w, int steps, int dirmask, void *stream);
/* ApplyHYPinSpace / ApplyHYPinTime (src/smear/hyp.cu:277, :328) with
 * ParamHYP alpha = {alpha1, alpha2, alpha3} (reference default 0.75, 0.6,
 * 0.3), used as FP32 like the reference's constants */
sun_status sun_smear_hyp(sun_lattice *lat, const double alpha[3], int steps, int nhits, double tol, int dirmask,
                         void *stream);
/* ApplyMultiHit (src/smear/multihit.cu:318): dst <- src, then each temporal
 * link of dst is the mean of the link and nhit heatbath updates of it against
 * its staple in src (beta of src).  dst: same N, geometry, precision and
 * order as src, SOA layout.  Random numbers: the Philox stream of link
 * (lex, 3) with purpose 2 under `seed` (the reference's RNG& argument). */
sun_status sun_multihit(sun_lattice *src, sun_lattice *dst, int nhit, uint64_t seed, void *stream);
/* ApplyMultiHitSpace (src/smear/multihitsp.cu:246): dst <- src, then each
 * spatial link of dst is the mean of nhit overrelaxation iterates of it
 * against its spatial staple in src; nhit >= 1 */
sun_status sun_multihit_space(sun_lattice *src, sun_lattice *dst, int nhit, void *stream);

/* ---- gauge file: SaveBin_Gauge<Real,RealSave> / ReadBin_Gauge
 * (src/io_gauge.cpp:429, :605), byte-compatible; save_fp64 selects RealSave,
 * the header's beta field has the lattice's own precision ---- */
sun_status sun_save_bin(sun_lattice *lat, const char *path, int save_fp64, int with_header);
sun_status sun_load_bin(sun_lattice *lat, const char *path, int save_fp64, int with_header);

/* ---- batches: many lattices of any (N, precision, layout) advanced by one
 * launch per (class, phase); no reference counterpart (one lattice per
 * process there) ---- */
sun_status sun_batch_create(sun_ctx *ctx, sun_batch **out);
sun_status sun_batch_destroy(sun_batch *b);
sun_status sun_batch_add(sun_batch *b, sun_lattice *lat);
sun_status sun_batch_remove(sun_batch *b, sun_lattice *lat);
sun_status sun_batch_size(const sun_batch *b, int *n);
/* use_graph: SUN_BATCH_GRAPH captures one sweep into a CUDA graph and replays
 * it (the classes as parallel branches; direct launches fork them onto
 * parallel streams the same way); | SUN_BATCH_NO_WAIT returns once the
 * sweeps are queued on `stream` -- the caller synchronizes it before reading
 * or changing the batch's lattices */
#define SUN_BATCH_GRAPH 1
#define SUN_BATCH_NO_WAIT 2
sun_status sun_batch_sweep(sun_batch *b, int n_hb, int n_or, int n_sweeps, int use_graph, void *stream);
/* out[2*i], out[2*i+1] for the i-th lattice in insertion order */
sun_status sun_batch_plaquette(sun_batch *b, double *out, void *stream);
sun_status sun_batch_polyakov(sun_batch *b, double *out, void *stream);
/* WilsonLoop (src/meas/wilsonloop.cu:535) of every lattice, one launch per
 * class: out[(i (R+1)(T+1) + t + r (T+1)) * 2 + {0, 1}] for the i-th lattice
 * in insertion order; R, T below every lattice's extents, at most 8 */
sun_status sun_batch_wilson_loops(sun_batch *b, int R, int T, double *out, void *stream);

/* ---- continuous-batching server ---- */
typedef struct {
    int ncolors;
    int dims[4];
    double beta;
    int sweeps;            /* sweeps of (n_hb heatbath + n_or overrelaxation) */
    int n_hb, n_or;
    uint64_t seed;
    int hot_start;         /* 1 Haar, 0 cold */
    int observables;       /* bit 0 plaquette, bit 1 Polyakov, bit 2 Wilson loops */
    int wilson_R, wilson_T;
    sun_precision precision;
    sun_layout layout;
    int reunit_every;
} sun_job;

typedef struct {
    int64_t id;
    int status;            /* sun_status of the job */
    double plaquette[2];
    double polyakov[2];
    double wilson[2 * 9 * 9];
    double submit_s, start_s, finish_s;  /* server clock */
    double link_updates;
} sun_result;

sun_status sun_server_create(sun_ctx *ctx, int max_active, sun_server **out);
sun_status sun_server_destroy(sun_server *s);
/* queue a job; the server admits it when its HBM footprint fits */
sun_status sun_server_submit(sun_server *s, const sun_job *job, int64_t *id);
/* run one scheduling step: admit queued jobs, advance every active job by up
 * to K sweeps (K sized so a step is ~50 ms of GPU work, at most 16; each job
 * stops at its own sweep count, sun_lattice_set_sweep_limit), measure the
 * finished jobs in batched launches and retire them; *n_done results are
 * written to out[0..cap) */
sun_status sun_server_step(sun_server *s, sun_result *out, int cap, int *n_done);
sun_status sun_server_pending(const sun_server *s, int *queued, int *active);
/* where the server's steps spent their time (seconds, summed over steps):
 * GPU time of the sweeps (CUDA events), and host time queueing the sweeps
 * (batch graph captures included), admitting jobs (lattice setup),
 * waiting for the sweeps, measuring and retiring finished jobs, and adding
 * admitted jobs to their batches */
typedef struct {
    int64_t steps, sweeps;    /* steps with sweeps; K summed over them */
    double sweep_gpu_s;
    double enqueue_s, admit_s, wait_s, retire_s, join_s;
} sun_server_stats;
sun_status sun_server_get_stats(const sun_server *s, sun_server_stats *out);
/* bytes a job needs on the device (links + measurement scratch) */
sun_status sun_job_footprint(const sun_job *job, size_t *bytes);
/* override the admission budget (default: the context's, sun_ctx_hbm_budget) */
sun_status sun_server_set_budget(sun_server *s, size_t bytes);
/* the admission rule: how many of the queued jobs (FIFO, footprints given)
 * to admit with `free_slots` slots and `used` of `budget` bytes taken */
sun_status sun_admit_count(const size_t *footprints, int n_queued, size_t budget, size_t used, int free_slots,
                           int *n_admit);

#ifdef __cplusplus
}
#endif
#endif
