// ref_probe.cu -- driver that runs the reference (nmrcardoso/sun, CULQCD)
// through its own public API to produce golden data for the oracle and the
// reference-build timings.  TEST INFRASTRUCTURE ONLY: built by
// oracle/ref/Makefile into oracle/_ref/ref_probe from the reference sources
// where they lie; the product never calls it.
//
// Every configuration is read and written in the reference's own binary
// format (ReadBin_Gauge / SaveBin_Gauge with header, FP64), even/odd SOA
// arrays as its HeatBath / OverRelaxation require.
//
// usage:
//   ref_probe measure   FILE nx ny nz nt beta R T
//   ref_probe overrelax IN OUT nx ny nz nt beta npass
//   ref_probe reunit    IN OUT nx ny nz nt beta
//   ref_probe ensemble  nx ny nz nt beta seed ntherm nmeas
//   ref_probe timing    nx ny nz nt beta sweeps {f32soa12|f64soa}
//   ref_probe batch     FILE sweeps  (lines 'L T beta': SU(3) L^3 x T lattices, FP32 SOA12,
//                       one after another; prints batch_ms and link_updates)
//   ref_probe plain     nx ny nz nt beta sweeps   (FP64 SOA, cold start, plaquette +
//                       Polyakov loop every sweep; prints plain_ms)
//   ref_probe smear     IN OUT nx ny nz nt beta KIND ARGS
//       KIND ape_space|ape_time w steps nhits tol;  stout_space|stout_time w steps
//       (prints smear_ms: the smearing call's duration, CUDA events)
//            hyp_space|hyp_time steps nhits tol a1 a2 a3;  multihit_space nhit
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include <comm_mpi.h>
#include <complex.h>
#include <constants.h>
#include <cuda_common.h>
#include <gaugearray.h>
#include <io_gauge.h>
#include <matrixsun.h>
#include <meas/plaquette.h>
#include <meas/polyakovloop.h>
#include <meas/wilsonloop.h>
#include <monte/monte.h>
#include <monte/ovr.h>
#include <random.h>
#include <reunitarize.h>
#include <smear/smear.h>

using namespace CULQCD;

static void setup(char** a, int k, bool quiet = true)
{
    int nx = atoi(a[k]), ny = atoi(a[k + 1]), nz = atoi(a[k + 2]), nt = atoi(a[k + 3]);
    double beta = atof(a[k + 4]);
    PARAMS::UseTex = false;
    SETPARAMS(false, beta, nx, ny, nz, nt, !quiet);
}

template <class Real> static int cmd_measure(int argc, char** a)
{
    if (argc < 10) return 2;
    setup(a, 3);
    const int R = atoi(a[8]), T = atoi(a[9]);
    gauge AA(SOA, Device, PARAMS::Volume * 4, true);
    ReadBin_Gauge<Real, double>(AA, a[2], true);
    PlaquetteCUB<Real> plaq(AA);
    complex p = plaq.Run();
    OnePolyakovLoop<Real> poly(AA);
    complex l = poly.Run();
    printf("plaquette %.17g %.17g\n", (double)p.real(), (double)p.imag());
    printf("polyakov %.17g %.17g\n", (double)l.real(), (double)l.imag());
    gauge BB(SOA, Device, PARAMS::Volume * 4, false);
    BB.Copy(AA);
    complex* res = (complex*)malloc(sizeof(complex) * (R + 1) * (T + 1));
    WilsonLoop<Real>(BB, res, R, T);
    for (int r = 0; r <= R; ++r)
        for (int t = 0; t <= T; ++t)
            printf("wilson %d %d %.17g %.17g\n", r, t, (double)res[t + r * (T + 1)].real(),
                   (double)res[t + r * (T + 1)].imag());
    free(res);
    BB.Release();
    AA.Release();
    return 0;
}

template <class Real> static int cmd_overrelax(int argc, char** a)
{
    if (argc < 10) return 2;
    setup(a, 4);
    gauge AA(SOA, Device, PARAMS::Volume * 4, true);
    ReadBin_Gauge<Real, double>(AA, a[2], true);
    OverRelaxation<Real> ovr(AA);
    for (int i = 0; i < atoi(a[9]); ++i) ovr.Run();
    cudaDeviceSynchronize();
    SaveBin_Gauge<Real, double>(AA, a[3], true);
    AA.Release();
    return 0;
}

template <class Real> static int cmd_reunit(int argc, char** a)
{
    if (argc < 9) return 2;
    setup(a, 4);
    gauge AA(SOA, Device, PARAMS::Volume * 4, true);
    ReadBin_Gauge<Real, double>(AA, a[2], true);
    Reunitarize<Real> reu(AA);
    reu.Run();
    cudaDeviceSynchronize();
    SaveBin_Gauge<Real, double>(AA, a[3], true);
    AA.Release();
    return 0;
}

// cold start, then sweeps of 1 heatbath + 4 overrelaxation (reunitarization
// every 10), the plaquette after every measured sweep
template <class Real> static int cmd_ensemble(int argc, char** a)
{
    if (argc < 10) return 2;
    setup(a, 2);
    const unsigned seed = (unsigned)atoi(a[7]);
    const int ntherm = atoi(a[8]), nmeas = atoi(a[9]);
    gauge AA(SOA, Device, PARAMS::Volume * 4, true);
    AA.Init();
    RNG rng;
    rng.Init(seed);
    HeatBath<Real> hb(AA, rng);
    OverRelaxation<Real> ovr(AA);
    Reunitarize<Real> reu(AA);
    PlaquetteCUB<Real> plaq(AA);
    for (int s = 0; s < ntherm + nmeas; ++s) {
        hb.Run();
        for (int k = 0; k < 4; ++k) ovr.Run();
        if ((s + 1) % 10 == 0) reu.Run();
        if (s >= ntherm) {
            complex p = plaq.Run();
            printf("plaq %d %.17g %.17g\n", s, (double)p.real(), (double)p.imag());
        }
    }
    rng.Release();
    AA.Release();
    return 0;
}

template <class Real, ArrayType AT> static int run_timing(char** a)
{
    const int sweeps = atoi(a[7]);
    gauge AA(AT, Device, PARAMS::Volume * 4, true);
    AA.Init();
    RNG rng;
    rng.Init(1234u);
    HeatBath<Real> hb(AA, rng);
    OverRelaxation<Real> ovr(AA);
    for (int w = 0; w < 3; ++w) {  // warm-up (and autotuning)
        hb.Run();
        ovr.Run();
    }
    cudaEvent_t e0, e1, e2;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&e2);
    float ms_hb = 0, ms_or = 0;
    for (int s = 0; s < sweeps; ++s) {
        cudaEventRecord(e0, 0);
        hb.Run();
        cudaEventRecord(e1, 0);
        for (int k = 0; k < 4; ++k) ovr.Run();
        cudaEventRecord(e2, 0);
        cudaEventSynchronize(e2);
        float t1 = 0, t2 = 0;
        cudaEventElapsedTime(&t1, e0, e1);
        cudaEventElapsedTime(&t2, e1, e2);
        ms_hb += t1;
        ms_or += t2;
    }
    const double V = (double)PARAMS::Volume;
    printf("timing hb_ms_per_pass %.6f or_ms_per_pass %.6f sweep_ms %.6f link_updates_per_s %.6e\n", ms_hb / sweeps,
           ms_or / (4.0 * sweeps), (ms_hb + ms_or) / sweeps, 20.0 * V * sweeps / ((ms_hb + ms_or) * 1e-3));
    rng.Release();
    AA.Release();
    return 0;
}

// many lattices the reference's way, one after another (one process-global
// geometry at a time): per lattice SETPARAMS, hot start, 3 untimed sweeps,
// then `sweeps` timed sweeps of 1 HeatBath + 4 OverRelaxation with
// Reunitarize every 10; the timed parts are summed
template <class Real> static int cmd_batch(int argc, char** a)
{
    if (argc < 4) return 2;
    FILE* f = fopen(a[2], "r");
    if (!f) return 2;
    const int sweeps = atoi(a[3]);
    int l, t;
    double beta;
    double ms_total = 0, updates = 0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    unsigned seed = 1234;
    while (fscanf(f, "%d %d %lf", &l, &t, &beta) == 3) {
        PARAMS::UseTex = false;
        SETPARAMS(false, beta, l, l, l, t, false);
        gauge AA(SOA12, Device, PARAMS::Volume * 4, true);
        RNG rng;
        rng.Init(seed++);
        AA.Init(rng);
        HeatBath<Real> hb(AA, rng);
        OverRelaxation<Real> ovr(AA);
        Reunitarize<Real> reu(AA);
        for (int w = 0; w < 3; ++w) {
            hb.Run();
            for (int k = 0; k < 4; ++k) ovr.Run();
        }
        cudaDeviceSynchronize();
        cudaEventRecord(e0, 0);
        for (int s = 0; s < sweeps; ++s) {
            hb.Run();
            for (int k = 0; k < 4; ++k) ovr.Run();
            if ((s + 1) % 10 == 0) reu.Run();
        }
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        ms_total += ms;
        updates += 20.0 * PARAMS::Volume * sweeps;
        rng.Release();
        AA.Release();
    }
    fclose(f);
    printf("batch_ms %.6f link_updates %.6e\n", ms_total, updates);
    return 0;
}

// the plain small case: cold start, sweeps of 1 HeatBath + 4 OverRelaxation
// with PlaquetteCUB and OnePolyakovLoop after every sweep, FP64 full links
template <class Real> static int cmd_plain(int argc, char** a)
{
    if (argc < 8) return 2;
    setup(a, 2);
    const int sweeps = atoi(a[7]);
    gauge AA(SOA, Device, PARAMS::Volume * 4, true);
    AA.Init();
    RNG rng;
    rng.Init(1234u);
    HeatBath<Real> hb(AA, rng);
    OverRelaxation<Real> ovr(AA);
    PlaquetteCUB<Real> plaq(AA);
    OnePolyakovLoop<Real> poly(AA);
    for (int w = 0; w < 3; ++w) {  // warm-up (and autotuning)
        hb.Run();
        ovr.Run();
        plaq.Run();
        poly.Run();
    }
    AA.Init();
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaDeviceSynchronize();
    cudaEventRecord(e0, 0);
    complexd p, l;
    for (int s = 0; s < sweeps; ++s) {
        hb.Run();
        for (int k = 0; k < 4; ++k) ovr.Run();
        p = plaq.Run();
        l = poly.Run();
    }
    cudaEventRecord(e1, 0);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    printf("plain_ms %.6f plaquette %.17g %.17g polyakov %.17g %.17g\n", ms, p.real(), p.imag(), l.real(), l.imag());
    rng.Release();
    AA.Release();
    return 0;
}

static int cmd_timing(int argc, char** a)
{
    if (argc < 9) return 2;
    setup(a, 2);
    if (!strcmp(a[8], "f32soa12")) return run_timing<float, SOA12>(a);
    if (!strcmp(a[8], "f64soa")) return run_timing<double, SOA>(a);
    return 2;
}

// smearing through the reference API on a normal-order SOA copy (the only
// order its smearing accepts); the result is written back in even/odd order
template <class Real> static int cmd_smear(int argc, char** a)
{
    if (argc < 10) return 2;
    setup(a, 4);
    const std::string kind = a[9];
    gauge AA(SOA, Device, PARAMS::Volume * 4, true);
    ReadBin_Gauge<Real, double>(AA, a[2], true);
    gauge BB(SOA, Device, PARAMS::Volume * 4, false);
    BB.Copy(AA);
    int rc = 0;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaDeviceSynchronize();
    cudaEventRecord(t0, 0);
    if ((kind == "ape_space" || kind == "ape_time") && argc >= 14) {
        const Real w = atof(a[10]), tol = atof(a[13]);
        const int steps = atoi(a[11]), nhits = atoi(a[12]);
        if (kind == "ape_space") ApplyAPEinSpace<Real>(BB, w, steps, nhits, tol);
        else ApplyAPEinTime<Real>(BB, w, steps, nhits, tol);
    } else if ((kind == "stout_space" || kind == "stout_time") && argc >= 12) {
        const Real w = atof(a[10]);
        const int steps = atoi(a[11]);
        if (kind == "stout_space") ApplyStoutinSpace<Real>(BB, w, steps);
        else ApplyStoutinTime<Real>(BB, w, steps);
    } else if ((kind == "hyp_space" || kind == "hyp_time") && argc >= 16) {
        const int steps = atoi(a[10]), nhits = atoi(a[11]);
        const Real tol = atof(a[12]);
        ParamHYP hyp((float)atof(a[13]), (float)atof(a[14]), (float)atof(a[15]));
        if (kind == "hyp_space") ApplyHYPinSpace<Real>(BB, steps, nhits, tol, hyp);
        else ApplyHYPinTime<Real>(BB, steps, nhits, tol, hyp);
    } else if (kind == "multihit_space" && argc >= 11) {
        gauge CC(SOA, Device, PARAMS::Volume * 4, false);
        CC.Copy(BB);
        RNG rng;
        rng.Init(1u);
        ApplyMultiHitSpace<Real>(CC, BB, rng, atoi(a[10]));
        rng.Release();
        CC.Release();
    } else {
        rc = 2;
    }
    cudaEventRecord(t1, 0);
    cudaDeviceSynchronize();
    float ms = 0;
    cudaEventElapsedTime(&ms, t0, t1);
    printf("smear_ms %.6f\n", ms);
    if (rc == 0) {
        AA.Copy(BB);
        SaveBin_Gauge<Real, double>(AA, a[3], true);
    }
    BB.Release();
    AA.Release();
    return rc;
}

int main(int argc, char** argv)
{
    if (argc < 2) {
        fprintf(stderr, "usage: see the header of ref_probe.cu\n");
        return 2;
    }
    const bool tune = getenv("SUN_REF_TUNE") != nullptr;
    initCULQCD(0, SILENT, tune ? TUNE_YES : TUNE_NO);
    int rc = 2;
    const std::string c = argv[1];
    if (c == "measure") rc = cmd_measure<double>(argc, argv);
    else if (c == "overrelax") rc = cmd_overrelax<double>(argc, argv);
    else if (c == "reunit") rc = cmd_reunit<double>(argc, argv);
    else if (c == "ensemble") rc = cmd_ensemble<double>(argc, argv);
    else if (c == "timing") rc = cmd_timing(argc, argv);
    else if (c == "plain") rc = cmd_plain<double>(argc, argv);
    else if (c == "batch") rc = cmd_batch<float>(argc, argv);
    else if (c == "smear") rc = cmd_smear<double>(argc, argv);
    fflush(stdout);
    if (rc == 2) fprintf(stderr, "bad arguments\n");
    EndCULQCD(rc);
    return rc;
}
