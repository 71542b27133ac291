// noalloc.cu -- the plaquette measurement for callers that cannot allocate
// device memory.
//
// sun_plaquette() keeps its per-CTA partial sums and its result in buffers
// the library allocates with cudaMalloc on first use.  Some callers cannot
// let a library allocate: applications that hand all device memory to their
// own pool or arena and forbid allocations behind their back, embedded and
// real-time hosts with a fixed memory budget set at start-up, and loops that
// cannot afford the device-wide synchronisation a library's later cudaFree
// brings.  sun_plaquette_noalloc() serves them: the same measurement, with
// its scratch in a fixed array compiled into this library.
//
// The scratch is g_plaq_scratch below: 4 doubles per CTA of 128 sites, for
// at most 65536 CTAs (2 MiB, so lattices of at most 8,388,608 sites).  Every
// GPU that loads the library holds this array until the process exits.
// Every call uses the same array: calls whose kernels overlap on the GPU
// (two streams, two host threads) race and must be serialised by the caller.
// Nothing needs clearing between calls: each CTA overwrites its own slot
// before the final reduction reads it, and the reduction reads only the
// slots written in the same call.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/sun_b200.h"
#include "sun_kernels.cuh"

namespace {

constexpr int kBlock = 128;
constexpr int kMaxBlocks = 65536;
constexpr long long kMaxSites = (long long)kBlock * kMaxBlocks;

// (spatial sum, compensation, temporal sum, compensation) per CTA
static __device__ __align__(256) double g_plaq_scratch[4 * kMaxBlocks];

// Host code cannot use g_plaq_scratch's name as a device address (it names a
// host-side stand-in).  The device address is looked up once per device,
// with that device current, and cached here for the life of the process: a
// caller that destroys and re-creates a device's context (cudaDeviceReset)
// must not call this entry point afterwards, since the cached address
// belonged to the old context.
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
double* g_scratch_addr[kMaxDevices] = {};

// Per-site plaquette sum of kernel sunb::k_plaquette, one lattice, partials
// into the caller-supplied (static) scratch.
template <int N, class R, int LAYOUT>
__global__ void __launch_bounds__(kBlock) k_plaquette_noalloc(sunb::LatDev L, double* partials)
{
    using namespace sunb;
    __shared__ DD sh[32];
    const Geom g = geom_of(L);
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    double sp = 0.0, tp = 0.0;
    if (w < g.V) {
        int x[4];
        site_coords(L, g, w, x);
#pragma unroll 1
        for (int mu = 0; mu < 3; ++mu) {
            int xm[4];
            shifted(g, x, mu, 1, xm);
#pragma unroll 1
            for (int nu = mu + 1; nu < 4; ++nu) {
                int xn[4];
                shifted(g, x, nu, 1, xn);
                Mat<N, double> A, B, P, Q;
                load_d<N, R, LAYOUT>(L, g, x, mu, A);
                load_d<N, R, LAYOUT>(L, g, xm, nu, B);
                mmul(A, B, P);
                load_d<N, R, LAYOUT>(L, g, x, nu, A);
                load_d<N, R, LAYOUT>(L, g, xn, mu, B);
                mmul(A, B, Q);
                const double t = mtrace_nd(P, Q).re;
                if (nu == 3) tp += t; else sp += t;
            }
        }
    }
    block_sum(sp, partials + (size_t)blockIdx.x * 4, sh);
    block_sum(tp, partials + (size_t)blockIdx.x * 4 + 2, sh);
}

// one warp: fixed-order compensated sum of the nblocks partials, scaled
__global__ void k_plaquette_noalloc_finalize(const double* partials, int nblocks, double scale, double* out)
{
    using namespace sunb;
    const int lane = threadIdx.x;
    for (int v = 0; v < 2; ++v) {
        DD d;
        d.s = 0.0;
        d.c = 0.0;
        for (int b = lane; b < nblocks; b += 32) {
            DD t;
            t.s = partials[(size_t)b * 4 + 2 * v];
            t.c = partials[(size_t)b * 4 + 2 * v + 1];
            d = dd_add(d, t);
        }
        d = dd_warp(d);
        if (lane == 0) out[v] = (d.s + d.c) * scale;
    }
}

template <int N, class R, int LAYOUT>
cudaError_t launch(const sunb::LatDev& L, int nblocks, double* scratch, double scale, double* out, cudaStream_t s)
{
    k_plaquette_noalloc<N, R, LAYOUT><<<nblocks, kBlock, 0, s>>>(L, scratch);
    k_plaquette_noalloc_finalize<<<1, 32, 0, s>>>(scratch, nblocks, scale, out);
    return cudaGetLastError();
}

template <int N> cudaError_t launch_n(int fp64, int layout, const sunb::LatDev& L, int nb, double* scr, double sc,
                                      double* out, cudaStream_t s)
{
    using namespace sunb;
    if constexpr (N == 3) {
        if (layout == SUN_SOA12) return fp64 ? launch<3, double, L_SOA12>(L, nb, scr, sc, out, s)
                                             : launch<3, float, L_SOA12>(L, nb, scr, sc, out, s);
        if (layout == SUN_SOA8) return fp64 ? launch<3, double, L_SOA8>(L, nb, scr, sc, out, s)
                                            : launch<3, float, L_SOA8>(L, nb, scr, sc, out, s);
    }
    return fp64 ? launch<N, double, L_SOA>(L, nb, scr, sc, out, s) : launch<N, float, L_SOA>(L, nb, scr, sc, out, s);
}

sun_status reject(sun_status st, const char* msg)
{
    sunb::set_global_error(msg);
    return st;
}

}  // namespace

extern "C" sun_status sun_plaquette_noalloc(const void* d_links, const sun_lattice_params* p, double* d_out,
                                            void* stream)
{
    if (!d_links || !p || !d_out) return reject(SUN_ERR_INVALID_ARG, "sun_plaquette_noalloc: null argument");
    const int N = p->ncolors;
    if (N != 2 && N != 3 && N != 4 && N != 6)
        return reject(SUN_ERR_UNSUPPORTED, "sun_plaquette_noalloc: N must be 2, 3, 4 or 6");
    if ((p->layout == SUN_SOA12 || p->layout == SUN_SOA8) && N != 3)
        return reject(SUN_ERR_UNSUPPORTED, "sun_plaquette_noalloc: 12/8-parameter layouts are SU(3) only");
    if (p->layout != SUN_SOA && p->layout != SUN_SOA12 && p->layout != SUN_SOA8)
        return reject(SUN_ERR_INVALID_ARG, "sun_plaquette_noalloc: unknown layout");
    if (p->precision != SUN_F32 && p->precision != SUN_F64)
        return reject(SUN_ERR_INVALID_ARG, "sun_plaquette_noalloc: unknown precision");
    if (p->order != SUN_EVEN_ODD && p->order != SUN_NORMAL)
        return reject(SUN_ERR_INVALID_ARG, "sun_plaquette_noalloc: unknown storage order");
    // the site count, checked against the scratch limit before every
    // multiplication (no overflow whatever the dimensions)
    long long V = 1;
    for (int d = 0; d < 4; ++d) {
        if (p->dims[d] < 2 || p->dims[d] % 2)
            return reject(SUN_ERR_INVALID_ARG, "sun_plaquette_noalloc: every dimension must be even and >= 2");
        if (p->dims[d] > kMaxSites || V > kMaxSites) {
            V = kMaxSites + 1;
            break;
        }
        V *= p->dims[d];
    }
    if (V > kMaxSites) {
        char msg[200];
        snprintf(msg, sizeof msg,
                 "sun_plaquette_noalloc: the lattice's sites exceed the fixed scratch (at most %lld sites); "
                 "use sun_plaquette", kMaxSites);
        return reject(SUN_ERR_CAPACITY, msg);
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return reject(SUN_ERR_CUDA, "sun_plaquette_noalloc: no usable current device");
    double* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_scratch_mu);
        if (!g_scratch_addr[dev]) {
            void* ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&ptr, g_plaq_scratch);
            if (e != cudaSuccess || !ptr) return reject(SUN_ERR_CUDA, "sun_plaquette_noalloc: scratch lookup failed");
            g_scratch_addr[dev] = static_cast<double*>(ptr);
        }
        scratch = g_scratch_addr[dev];
    }
    sunb::LatDev L{};
    L.links = const_cast<void*>(d_links);
    for (int d = 0; d < 4; ++d) L.X[d] = p->dims[d];
    L.V = (int)V;
    L.halfV = (int)(V / 2);
    L.evenodd = p->order == SUN_EVEN_ODD;
    const int nblocks = (int)((V + kBlock - 1) / kBlock);
    const double scale = 1.0 / (3.0 * N * (double)V);
    const int fp64 = p->precision == SUN_F64;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e;
    switch (N) {
    case 2: e = launch_n<2>(fp64, p->layout, L, nblocks, scratch, scale, d_out, s); break;
    case 3: e = launch_n<3>(fp64, p->layout, L, nblocks, scratch, scale, d_out, s); break;
    case 4: e = launch_n<4>(fp64, p->layout, L, nblocks, scratch, scale, d_out, s); break;
    default: e = launch_n<6>(fp64, p->layout, L, nblocks, scratch, scale, d_out, s); break;
    }
    if (e != cudaSuccess) return reject(SUN_ERR_CUDA, cudaGetErrorString(e));
    return SUN_OK;
}
