// ref_link_probe.cu -- runs the reference's per-link device functions
// heatBathSUN (with injected uniforms), overrelaxationSUN and reunit_link
// (include/device_PHB_OVR.h:362, :494; include/reunitlink.h:16) on links
// given in a file, for golden vectors.  TEST INFRASTRUCTURE ONLY, built by
// oracle/ref/Makefile with shim_inject/ first on the include path.
//
// usage: ref_link_probe {hb|or|reunit} IN OUT beta
// IN : int32 nlinks, int32 stride; double U[nlinks][NC*NC][2]; double F[nlinks][NC*NC][2];
//      double u[nlinks][stride]   (F is the staple^dagger the update receives)
// OUT: double U'[nlinks][NC*NC][2]; int32 used[nlinks] (uniforms consumed, -1 overrun)
// NC = NCOLORS of the build (3, or 4 and 6 for the builds of `make ncolors`).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <comm_mpi.h>
#include <complex.h>
#include <constants.h>
#include <device_PHB_OVR.h>
#include <matrixsun.h>
#include <reunitlink.h>

using namespace CULQCD;

template <int MODE>
__global__ void k_link(const double* U, const double* F, const double* u, int stride, int n, double* out, int* used,
                       int* flags)
{
    typedef double Real;
    constexpr int NC = NCOLORS, NE = NCOLORS * NCOLORS;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    msun A, B;
    for (int a = 0; a < NC; ++a)
        for (int b = 0; b < NC; ++b) {
            A.e[a][b] = complex::make_complex(U[(i * NE + a * NC + b) * 2], U[(i * NE + a * NC + b) * 2 + 1]);
            B.e[a][b] = complex::make_complex(F[(i * NE + a * NC + b) * 2], F[(i * NE + a * NC + b) * 2 + 1]);
        }
    cuRNGState st;
    st.u = u + (size_t)i * stride;
    st.pos = 0;
    st.len = stride;
    st.overrun = flags + i;
    if (MODE == 0) heatBathSUN<Real>(A, B, st);
    else if (MODE == 1) overrelaxationSUN<Real>(A, B);
    else reunit_link<Real>(&A);
    for (int a = 0; a < NC; ++a)
        for (int b = 0; b < NC; ++b) {
            out[(i * NE + a * NC + b) * 2] = A.e[a][b].real();
            out[(i * NE + a * NC + b) * 2 + 1] = A.e[a][b].imag();
        }
    used[i] = flags[i] ? -1 : st.pos;
}

int main(int argc, char** argv)
{
    if (argc < 5) {
        fprintf(stderr, "usage: ref_link_probe {hb|or|reunit} IN OUT beta\n");
        return 2;
    }
    initCULQCD(0, SILENT, TUNE_NO);
    SETPARAMS(false, atof(argv[4]), 4, 4, 4, 4, false);  // sets BetaOverNc = beta / N
    FILE* f = fopen(argv[2], "rb");
    if (!f) return 3;
    int n = 0, stride = 0;
    if (fread(&n, 4, 1, f) != 1 || fread(&stride, 4, 1, f) != 1) return 3;
    std::vector<double> U((size_t)n * 2 * NCOLORS * NCOLORS), F((size_t)n * 2 * NCOLORS * NCOLORS), u((size_t)n * stride);
    if (fread(U.data(), 8, U.size(), f) != U.size() || fread(F.data(), 8, F.size(), f) != F.size() ||
        fread(u.data(), 8, u.size(), f) != u.size())
        return 3;
    fclose(f);
    double *dU, *dF, *du, *dout;
    int *dused, *dflags;
    cudaMalloc(&dU, 8 * U.size());
    cudaMalloc(&dF, 8 * F.size());
    cudaMalloc(&du, 8 * (u.size() + 1));
    cudaMalloc(&dout, 8 * U.size());
    cudaMalloc(&dused, 4 * n);
    cudaMalloc(&dflags, 4 * n);
    cudaMemcpy(dU, U.data(), 8 * U.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(dF, F.data(), 8 * F.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(du, u.data(), 8 * u.size(), cudaMemcpyHostToDevice);
    cudaMemset(dflags, 0, 4 * n);
    const std::string m = argv[1];
    const int blocks = (n + 63) / 64;
    if (m == "hb") k_link<0><<<blocks, 64>>>(dU, dF, du, stride, n, dout, dused, dflags);
    else if (m == "or") k_link<1><<<blocks, 64>>>(dU, dF, du, stride, n, dout, dused, dflags);
    else k_link<2><<<blocks, 64>>>(dU, dF, du, stride, n, dout, dused, dflags);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        fprintf(stderr, "%s\n", cudaGetErrorString(e));
        return 4;
    }
    std::vector<double> out(U.size());
    std::vector<int> used(n);
    cudaMemcpy(out.data(), dout, 8 * out.size(), cudaMemcpyDeviceToHost);
    cudaMemcpy(used.data(), dused, 4 * n, cudaMemcpyDeviceToHost);
    FILE* g = fopen(argv[3], "wb");
    if (!g) return 3;
    fwrite(out.data(), 8, out.size(), g);
    fwrite(used.data(), 4, n, g);
    fclose(g);
    cudaFree(dU); cudaFree(dF); cudaFree(du); cudaFree(dout); cudaFree(dused); cudaFree(dflags);
    printf("ok %d links\n", n);
    return 0;
}
