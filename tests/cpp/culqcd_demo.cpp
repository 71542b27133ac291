// A CULQCD-style program (the reference's entry points and spelling) built
// against include/culqcd_b200.hpp and libsun_b200.so: hot start, three sweeps
// of 1 heatbath + 4 overrelaxation, reunitarization, measurements, save,
// then APE smearing and multihit before a second Wilson loop.
// usage: culqcd_demo OUTFILE
#include <cstdio>

#include "culqcd_b200.hpp"

using namespace CULQCD;

template <class Real> int run(const char* out)
{
    SETPARAMS(false, 6.0, 4, 4, 4, 8, false);
    gauge AA(SOA12, Device, PARAMS::Volume * 4, true);
    RNG rng;
    rng.Init(1234);
    AA.Init(rng);
    HeatBath<Real> hb(AA, rng);
    OverRelaxation<Real> ovr(AA);
    Reunitarize<Real> reu(AA);
    for (int s = 0; s < 3; ++s) {
        hb.Run();
        for (int k = 0; k < 4; ++k) ovr.Run();
    }
    reu.Run();
    PlaquetteCUB<Real> plaq(AA);
    _complex<Real> p = plaq.Run();
    plaq.printValue();
    _complex<Real> l = OnePolyakovLoop<Real>(AA).Run();
    gauge BB(SOA, Device, PARAMS::Volume * 4, false);
    BB.Copy(AA);
    _complex<Real> res[3 * 4];
    WilsonLoop<Real>(BB, res, 2, 3);
    printf("plaquette %.17g %.17g\n", (double)p.real(), (double)p.imag());
    printf("polyakov %.17g %.17g\n", (double)l.real(), (double)l.imag());
    printf("wilson11 %.17g %.17g\n", (double)res[1 * 4 + 1].real(), (double)res[1 * 4 + 1].imag());
    SaveBin_Gauge<Real, double>(AA, out, true);
    // the driver's smearing before Wilson loops (test.cpp:179-219): APE in
    // space, then multihit of the temporal links into BB
    ApplyAPEinSpace<Real>(BB, 0.2, 3, 10, 1.e-10);
    gauge DD(SOA, Device, PARAMS::Volume * 4, false);
    DD.Copy(BB);
    ApplyMultiHit<Real>(DD, BB, rng, 5);
    DD.Release();
    WilsonLoop<Real>(BB, res, 2, 3);
    printf("wilson11_smeared %.17g %.17g\n", (double)res[1 * 4 + 1].real(), (double)res[1 * 4 + 1].imag());
    BB.Release();
    AA.Release();
    return 0;
}

int main(int argc, char** argv)
{
    if (argc < 2) return 2;
    initCULQCD(0, SILENT, TUNE_NO);
    int rc = run<float>(argv[1]);
    EndCULQCD(0);
    return rc;
}
