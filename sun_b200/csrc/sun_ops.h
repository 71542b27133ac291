// sun_ops.h -- host-side launch interface between the C-ABI engine
// (engine.cu) and the per-N kernel translation units (ops_n*.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace sunb {

// One lattice as every kernel sees it (an entry of a device table).
struct LatDev {
    void* links;              // device image, layout/precision of the class
    int X[4];
    int V, halfV;
    double beta_over_n;       // beta / N (constants.cu:443)
    unsigned long long seed;  // Philox key
    unsigned int* state;      // device counters: [0] heatbath passes, [1] sweeps, [2] 1 if the
                              // last counted sweep advanced the lattice (see sweep_limit)
    int reunit_every;         // reunitarize when sweeps % reunit_every == 0 (0: never)
    int evenodd;              // storage order: 1 even/odd, 0 lexicographic
    unsigned sweep_limit;     // 0: none; else the lattice is left unchanged once its sweep
                              // counter reaches the limit (the update kernels skip it, the
                              // counters and the reunitarization schedule stop)
};
// A lattice whose sweep counter reached its limit: update launches skip it.
__host__ __device__ inline bool lat_frozen(const LatDev& L)
{
#ifdef __CUDA_ARCH__
    return L.sweep_limit != 0u && __ldcg(L.state + 1) >= L.sweep_limit;
#else
    (void)L;
    return false;
#endif
}

// The end of a counted sweep: the pass and sweep counters advance by n_hb
// and inc unless the lattice sits at its sweep limit; state[2] records
// whether it advanced.
__device__ inline void advance_counters(const LatDev& L, unsigned n_hb, unsigned inc)
{
    unsigned* st = L.state;
    const unsigned adv = L.sweep_limit == 0u || st[1] < L.sweep_limit;
    if (adv) {
        st[0] += n_hb;
        st[1] += inc;
    }
    st[2] = adv;
}

// A launch over several lattices of one class (same N, precision, layout):
// CTA b works on lattice l with begin[l] <= b < begin[l+1].
struct BatchView {
    const LatDev* lats;
    const int* begin;
    int nlat;
    int nblocks;
};

// Uniforms injected per link for oracle parity: link (lex, mu) reads
// u[(lex*4 + mu)*stride + k], k < stride.
struct InjView {
    const double* u;
    int stride;
    int* err;
};

enum UpdateMode { MODE_HB = 0, MODE_HB_INJECTED = 1, MODE_OR = 2 };


// Work per lattice a launch maps CTAs onto.
// work items per lattice of a launch: half-sites, sites, spatial sites,
// links, (site, plane) pairs of the plaquette (6 V), and 8 lanes per spatial
// site of the Polyakov loop
enum WorkKind { WORK_HALF = 0, WORK_SITES = 1, WORK_SPATIAL = 2, WORK_LINKS = 3, WORK_PLANES = 4, WORK_POLY8 = 5 };
constexpr int kPolyLanes = 8;
// lattices below this volume measure the plaquette with one thread per
// (site, plane), warp-major (a warp: one plane of 32 consecutive sites), the
// others with one thread per site; the choice depends on the lattice alone
constexpr int kPlaneSplitMaxV = 1 << 17;
__host__ __device__ inline int plaquette_items(int V) { return V < kPlaneSplitMaxV ? ((V + 31) / 32) * 192 : V; }

// Many sweeps of one lattice in one cooperative launch (k_sweeps_resident):
// the update phases, the reunitarization and the measurements separated by
// grid barriers instead of launch boundaries.  Every CTA of the launch is
// resident; the kernel walks the launched kernels' CTA decompositions
// (virtual CTAs) so each result has the bits of the launched path.
struct ResidentArgs {
    BatchView upd;            // the update's decomposition (one lattice)
    BatchView plaq, poly;     // k_plaquette's and k_polyakov's (CTAs of 128 threads)
    int n_hb, n_or, n_sweeps;
    double* partials;         // plaquette partials (4 doubles per virtual CTA), then Polyakov ones
    double* out_plaq;         // per sweep: spatial and temporal sums
    double* out_poly;         // per sweep: real and imaginary trace sums
    unsigned* bar;            // arrivals at the grid barriers; zero at launch
    int* status;              // set to 1 when a barrier wait runs out
    unsigned long long wait_ns;  // limit of one barrier wait
    int skip_arrive;          // test hook: CTA that leaves at its first barrier without arriving (-1: none)
};

template <int N> struct Ops {
    // one checkerboard phase (parity, mu) of heatbath or overrelaxation;
    // hb_offset is added to the lattice's pass counter (heatbath pass index
    // inside the current sweep)
    // pdl: launch as a programmatic dependent of the previous launch on the
    // stream, which must be the update phase (parity, mu - 1) or, for mu = 0,
    // (1 - parity, 3); the kernel then waits for it only before the staples
    // of that phase's direction
    static cudaError_t update(int fp64, int layout, int mode, const BatchView& bv, int block,
                              int parity, int mu, unsigned hb_offset, const InjView& inj, int pdl, cudaStream_t s);
    // the same phase with the N lanes of a site sharing its staple products
    // (k_update_rows); block = threads per CTA (a multiple of 32), each warp
    // covering 32/N sites
    static cudaError_t update_rows(int fp64, int layout, int mode, const BatchView& bv, int block,
                                   int parity, int mu, unsigned hb_offset, const InjView& inj, int pdl,
                                   cudaStream_t s);
    // the same phase with a CTA of N warps per 32 half-sites and the staple
    // factors staged in shared memory (k_update_tile; N >= 4, full links);
    // the same bits as update()
    static cudaError_t update_tile(int fp64, int layout, int mode, const BatchView& bv, int parity, int mu,
                                   unsigned hb_offset, const InjView& inj, int pdl, cudaStream_t s);
    // n sweeps of one lattice and their measurements in one cooperative
    // launch of `grid` CTAs of 128 threads (k_sweeps_resident); rows: the
    // row-split update body (k_update_rows) instead of one thread per
    // half-site.  capacity: the most CTAs that can be resident at once.
    static cudaError_t sweeps_resident(int fp64, int layout, int rows, const ResidentArgs& a, int grid,
                                       cudaStream_t s);
    static int resident_capacity(int fp64, int layout, int rows);
    static cudaError_t cold(int fp64, int layout, const BatchView& bv, int block, cudaStream_t s);
    static cudaError_t hot(int fp64, int layout, const BatchView& bv, int block, cudaStream_t s);
    // FP64 reunitarization; only_due: skip lattices whose sweep counter is not
    // a multiple of reunit_every
    static cudaError_t reunit(int fp64, int layout, const BatchView& bv, int block, int only_due,
                              cudaStream_t s);
    // per-CTA partials: plaquette 2 values, polyakov 2, wilson 2(R+1)(T+1),
    // unitarity 1 (max); partial layout [block][value][sum, compensation]
    // plaquette and polyakov: with out non-null, the last CTA of each
    // lattice also finalizes its sums into out[2 l .. 2 l + 1] (counters: one
    // zeroed unsigned per lattice, left at zero); with slot non-null, into
    // row *slot of out (2 nlat doubles per row)
    static cudaError_t plaquette(int fp64, int layout, const BatchView& bv, int block, double* partials,
                                 double* out, unsigned* counters, const unsigned* slot, cudaStream_t s);
    static cudaError_t polyakov(int fp64, int layout, const BatchView& bv, int block, double* partials,
                                double* out, unsigned* counters, const unsigned* slot, cudaStream_t s);
    // both in one launch (k_plaq_poly; CTAs of 128 threads, vp and vl built
    // for 128), the last finalize advancing *slot
    // end_n_hb >= 0: the same launch ends the sweep (advance_counters with
    // n_hb = end_n_hb, one sweep) after the measurements
    static cudaError_t plaq_poly(int fp64, int layout, const BatchView& vp, const BatchView& vl, double* part_p,
                                 double* part_l, double* out_p, double* out_l, unsigned* cnt_p, unsigned* cnt_l,
                                 unsigned* slot, unsigned* joint, int end_n_hb, cudaStream_t s);
    static cudaError_t wilson(int fp64, int layout, const BatchView& bv, int block, int R, int T,
                              double* partials, cudaStream_t s);
    static cudaError_t unitarity(int fp64, int layout, const BatchView& bv, int block, double* partials,
                                 cudaStream_t s);
    // sums of tr U and det U over links: 4 values (Re tr, Im tr, Re det, Im det)
    static cudaError_t linkstats(int fp64, int layout, const BatchView& bv, int block, double* partials,
                                 cudaStream_t s);
    // canonical FP64 host order (site-major, 4 dirs, N*N row-major) <-> image
    static cudaError_t pack(int fp64, int layout, const BatchView& bv, int block, const void* canon,
                            cudaStream_t s);
    static cudaError_t unpack(int fp64, int layout, const BatchView& bv, int block, void* canon,
                              cudaStream_t s);
    // smearing: src and dst are distinct device images of the lattice, the
    // launch rows are the directions in dirmask (bit mu selects mu)
    static cudaError_t ape(int fp64, int layout, const BatchView& bv, int block, const void* src, void* dst,
                           int dirmask, double w, int nhits, double tol, cudaStream_t s);
    static cudaError_t stout(int fp64, int layout, const BatchView& bv, int block, const void* src, void* dst,
                             int dirmask, double w, cudaStream_t s);
    // HYP level 1 (alpha = alpha3), 2 (alpha2) or 3 (alpha1); b1, b2 hold 16
    // N x N slots per site
    static cudaError_t hyp(int fp64, int layout, const BatchView& bv, int block, int level, const void* src,
                           void* b1, void* b2, void* dst, int dirmask, double alpha, int nhits, double tol,
                           cudaStream_t s);
    // heatbath multihit of the temporal links (space = 0) or overrelaxation
    // multihit of the spatial links (space = 1); dst has the SOA layout
    static cudaError_t multihit(int fp64, int layout, const BatchView& bv, int block, const void* src, void* dst,
                                int nhit, unsigned long long seed, int space, cudaStream_t s);
};

extern template struct Ops<2>;
extern template struct Ops<3>;
extern template struct Ops<4>;
extern template struct Ops<6>;

// generic (N-independent) kernels, defined in engine.cu
cudaError_t launch_finalize_sum(const BatchView& bv, const double* partials, int nvals, double* out,
                                cudaStream_t s);
cudaError_t launch_finalize_max(const BatchView& bv, const double* partials, double* out, cudaStream_t s);
cudaError_t launch_end_sweep(const LatDev* lats, int nlat, unsigned n_hb, unsigned inc, cudaStream_t s);
// *slot += 1 (the row counter of replayed measurements)
cudaError_t launch_bump(unsigned* slot, cudaStream_t s);
// message returned by sun_last_error_string(NULL)
void set_global_error(const char* msg);

}  // namespace sunb
