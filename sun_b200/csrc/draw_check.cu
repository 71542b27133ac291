// draw_check.cu -- test hook: the SU(2) heatbath draw of the update kernels
// (su2_heatbath_draw, the restatement of generate_su2_matrix_milc,
// include/device_PHB_OVR.h:163-223) run on its own for a fixed alpha, so the
// distribution of the FP32 draw -- hardware log/exp/sincos approximations --
// and of the FP64 draw can be tested against the exact density
// sqrt(1 - a0^2) exp(alpha a0) of the SU(2) heatbath.
#include <cuda_runtime.h>

#include <cstdio>

#include "../../include/sun_b200.h"
#include "sun_core.cuh"
#include "sun_ops.h"

namespace {

// sample i: Philox stream (seed, counter word 1 = i, word 2 = 0, pass 0),
// the draw an update kernel makes for link (lex = i, mu = 0) in its first
// heatbath pass
template <class R> __global__ void k_su2_draws(R alpha, unsigned long long seed, int n, double* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    sunb::PhiloxStream<R> st;
    st.init(seed, (uint32_t)i, 0u, 0u);
    R a[4];
    sunb::su2_draw<R>(alpha, st, a);
    for (int k = 0; k < 4; ++k) out[4 * (size_t)i + k] = (double)a[k];
}

sun_status fail(const char* what, cudaError_t e)
{
    char msg[256];
    snprintf(msg, sizeof msg, "sun_debug_su2_draws: %s: %s", what, cudaGetErrorString(e));
    sunb::set_global_error(msg);
    return SUN_ERR_CUDA;
}

}  // namespace

extern "C" sun_status sun_debug_su2_draws(sun_precision prec, double alpha, uint64_t seed, int n, double* out)
{
    if (!out || n <= 0 || n > (1 << 26) || !(alpha > 0.0) || (prec != SUN_F32 && prec != SUN_F64)) {
        sunb::set_global_error("sun_debug_su2_draws: need out != NULL, 0 < n <= 2^26, alpha > 0, a precision");
        return SUN_ERR_INVALID_ARG;
    }
    double* d = nullptr;
    const size_t bytes = sizeof(double) * 4 * (size_t)n;
    cudaError_t e = cudaMalloc(&d, bytes);
    if (e != cudaSuccess) return fail("cudaMalloc", e);
    const int blk = 128, grid = (n + blk - 1) / blk;
    if (prec == SUN_F32) k_su2_draws<float><<<grid, blk>>>((float)alpha, seed, n, d);
    else k_su2_draws<double><<<grid, blk>>>(alpha, seed, n, d);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(out, d, bytes, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? SUN_OK : fail("draw kernel", e);
}
