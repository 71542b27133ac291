// culqcd_b200.hpp -- the reference's C++ entry points (nmrcardoso/sun,
// namespace CULQCD) re-exposed over the C ABI of sun_b200.h, so CULQCD user
// code for the hot path ports by swapping the include:
//
//   initCULQCD(gpuid, SUMMARIZE, TUNE_YES);                 comm_mpi.cpp:107
//   SETPARAMS(usetex, beta, nx, ny, nz, nt, verbose);        constants.cu:149
//   gauge AA(SOA12, Device, PARAMS::Volume * 4, true);       gaugearray.h:139
//   RNG rng; rng.Init(seed); AA.Init(rng);                   random.cu:93, gaugearray.h:781
//   HeatBath<float> hb(AA, rng); hb.Run();                   monte.cu:152, :196
//   OverRelaxation<float> ovr(AA); ovr.Run();                ovr.cu:139, :182
//   Reunitarize<float> reu(AA); reu.Run();                   reunitarize.cu:40, :78
//   complexs p = PlaquetteCUB<float>(AA).Run();              plaquette_cub.cu:226
//   complexs l = OnePolyakovLoop<float>(AA).Run();           polyakovloop.cu:637
//   WilsonLoop<float>(BB, res, R, T);                        wilsonloop.cu:535
//   SaveBin_Gauge<float, double>(AA, file, true);            io_gauge.cpp:429
//   EndCULQCD(0);                                            comm_mpi.cpp:186
//
// Semantics kept: SETPARAMS sets the geometry and beta that subsequently
// constructed arrays take; an array's size argument must be 4 * Volume;
// gauge handles are shallow copies sharing one device array, freed by
// Release() (gaugearray.h:657); errors print a message and exit, like
// errorCULQCD (comm_mpi.h:102-116) -- define CULQCD_B200_THROW before including
// to get a std::runtime_error instead.  Differences: N is a template/runtime
// value (CULQCD_B200_NCOLORS, default 3) instead of the NCOLORS build macro;
// the RNG is the counter-based Philox stream keyed by the seed passed to
// RNG::Init (no state array); EndCULQCD returns instead of exiting.
#ifndef CULQCD_B200_HPP
#define CULQCD_B200_HPP

#include <cstdio>
#include <cstdlib>
#include <memory>
#include <stdexcept>
#include <string>

#include "sun_b200.h"

#ifndef CULQCD_B200_NCOLORS
#define CULQCD_B200_NCOLORS 3
#endif

namespace CULQCD {

typedef enum { SOA = SUN_SOA, SOA12 = SUN_SOA12, SOA8 = SUN_SOA8 } ArrayType;
typedef enum { Host, Device } ReadMode;
typedef enum { SILENT, SUMMARIZE, VERBOSE, DEBUG_VERBOSE } Verbosity;
typedef enum { TUNE_NO, TUNE_YES } TuneMode;

template <class Real> struct _complex {
    Real re, im;
    _complex(Real r = 0, Real i = 0) : re(r), im(i) {}
    Real real() const { return re; }
    Real imag() const { return im; }
};
typedef _complex<float> complexs;
typedef _complex<double> complexd;

namespace detail {
inline sun_ctx*& ctx()
{
    static sun_ctx* c = nullptr;
    return c;
}
inline void check(sun_status st, const char* what)
{
    if (st == SUN_OK) return;
    std::string msg = std::string(what) + ": " + sun_last_error_string(ctx());
#ifdef CULQCD_B200_THROW
    throw std::runtime_error(msg);
#else
    fprintf(stderr, "Error: %s\n", msg.c_str());
    exit(1);
#endif
}
struct Params {
    int grid[4] = {0, 0, 0, 0};
    double beta = 0;
    bool set = false;
};
inline Params& params()
{
    static Params p;
    return p;
}
}  // namespace detail

namespace PARAMS {
inline int Volume = 0;  // set by SETPARAMS (constants.h:53-111)
}  // namespace PARAMS

inline void initCULQCD(int gpuid, Verbosity v = SILENT, TuneMode t = TUNE_NO)
{
    sun_config cfg = {gpuid, (int)v, (int)t, nullptr, 0};
    detail::check(sun_init(&cfg, &detail::ctx()), "initCULQCD");
}

inline void EndCULQCD(int)
{
    if (detail::ctx()) sun_finalize(detail::ctx());
    detail::ctx() = nullptr;
}

inline void SETPARAMS(bool /*usetex*/, double beta, int nx, int ny, int nz, int nt, bool /*verbose*/ = false)
{
    detail::Params& p = detail::params();
    p.grid[0] = nx; p.grid[1] = ny; p.grid[2] = nz; p.grid[3] = nt;
    p.beta = beta;
    p.set = true;
    PARAMS::Volume = nx * ny * nz * nt;
}

class RNG {
public:
    uint64_t seed = 0;
    void Init(unsigned int s) { seed = s; }
    void Release() {}
};

template <class Real> class _gauge {
    struct Handle {
        sun_lattice* lat = nullptr;
        ~Handle()
        {
            if (lat) sun_lattice_destroy(lat);
        }
    };
    std::shared_ptr<Handle> h;
    ArrayType atype;
    bool eo;

public:
    _gauge(ArrayType t, ReadMode /*mode*/, int size, bool evenodd = false) : atype(t), eo(evenodd)
    {
        const detail::Params& p = detail::params();
        if (!p.set) detail::check(SUN_ERR_STATE, "gauge: SETPARAMS not called");
        if (size != 4 * PARAMS::Volume) detail::check(SUN_ERR_INVALID_ARG, "gauge: size must be 4 * Volume");
        sun_lattice_params lp = {CULQCD_B200_NCOLORS, {p.grid[0], p.grid[1], p.grid[2], p.grid[3]}, p.beta,
                                 (sun_layout)t, evenodd ? SUN_EVEN_ODD : SUN_NORMAL,
                                 sizeof(Real) == 8 ? SUN_F64 : SUN_F32, 0, 0};
        h = std::make_shared<Handle>();
        detail::check(sun_lattice_create(detail::ctx(), &lp, &h->lat), "gauge");
    }
    sun_lattice* lat() const { return h->lat; }
    ArrayType Type() const { return atype; }
    bool EvenOdd() const { return eo; }
    void* GetPtr() const
    {
        void* d = nullptr;
        sun_lattice_device_ptr(h->lat, &d);
        return d;
    }
    void Init() { detail::check(sun_lattice_init_cold(h->lat, nullptr), "ColdStart"); }
    void Init(RNG& r)
    {
        detail::check(sun_lattice_set_rng(h->lat, r.seed, 0, 0), "HotStart");
        detail::check(sun_lattice_init_hot(h->lat, nullptr), "HotStart");
    }
    void Copy(const _gauge& src) { detail::check(sun_lattice_copy(h->lat, src.lat(), nullptr), "Copy"); }
    void Release() { h.reset(); }
};

template <class Real> class HeatBath {
    _gauge<Real>& a;

public:
    HeatBath(_gauge<Real>& array, RNG& r) : a(array)
    {
        uint64_t s = 0;
        uint32_t hb = 0, sw = 0;
        detail::check(sun_lattice_get_rng(a.lat(), &s, &hb, &sw), "HeatBath");
        if (s != r.seed) detail::check(sun_lattice_set_rng(a.lat(), r.seed, hb, sw), "HeatBath");
    }
    void Run() { detail::check(sun_heatbath(a.lat(), 1, nullptr), "HeatBath::Run"); }
};

template <class Real> class OverRelaxation {
    _gauge<Real>& a;

public:
    explicit OverRelaxation(_gauge<Real>& array) : a(array) {}
    void Run() { detail::check(sun_overrelax(a.lat(), 1, nullptr), "OverRelaxation::Run"); }
};

template <class Real> class Reunitarize {
    _gauge<Real>& a;

public:
    explicit Reunitarize(_gauge<Real>& array) : a(array) {}
    void Run() { detail::check(sun_reunitarize(a.lat(), nullptr), "Reunitarize::Run"); }
};

template <class Real> class PlaquetteCUB {
    _gauge<Real>& a;
    _complex<Real> v;

public:
    explicit PlaquetteCUB(_gauge<Real>& array) : a(array) {}
    _complex<Real> Run()
    {
        double o[2];
        detail::check(sun_plaquette(a.lat(), o, nullptr), "PlaquetteCUB::Run");
        v = _complex<Real>((Real)o[0], (Real)o[1]);
        return v;
    }
    _complex<Real> Value() const { return v; }
    void printValue() const
    {
        printf("Plaquette: < %.12e : %.12e > :: mean: %.12e\n", (double)v.re, (double)v.im,
               ((double)v.re + (double)v.im) / 2.0);
    }
};

template <class Real> class OnePolyakovLoop {
    _gauge<Real>& a;
    _complex<Real> v;

public:
    explicit OnePolyakovLoop(_gauge<Real>& array) : a(array) {}
    _complex<Real> Run()
    {
        double o[2];
        detail::check(sun_polyakov(a.lat(), o, nullptr), "OnePolyakovLoop::Run");
        v = _complex<Real>((Real)o[0], (Real)o[1]);
        return v;
    }
};

template <class Real> void WilsonLoop(_gauge<Real>& array, _complex<Real>* res, int R, int T)
{
    std::unique_ptr<double[]> o(new double[2 * (R + 1) * (T + 1)]);
    detail::check(sun_wilson_loops(array.lat(), R, T, o.get(), nullptr), "WilsonLoop");
    for (int i = 0; i < (R + 1) * (T + 1); ++i) res[i] = _complex<Real>((Real)o[2 * i], (Real)o[2 * i + 1]);
}

// smearing (include/smear/smear.h): in place on `array`, any layout and order
template <class Real> void ApplyAPEinSpace(_gauge<Real> array, Real w, int steps, int nhits, Real tol)
{
    detail::check(sun_smear_ape(array.lat(), w, steps, nhits, tol, SUN_SMEAR_SPACE, nullptr), "ApplyAPEinSpace");
}
template <class Real> void ApplyAPEinTime(_gauge<Real> array, Real w, int steps, int nhits, Real tol)
{
    detail::check(sun_smear_ape(array.lat(), w, steps, nhits, tol, SUN_SMEAR_TIME, nullptr), "ApplyAPEinTime");
}
template <class Real> void ApplyStoutinSpace(_gauge<Real> array, Real w, int steps)
{
    detail::check(sun_smear_stout(array.lat(), w, steps, SUN_SMEAR_SPACE, nullptr), "ApplyStoutinSpace");
}
template <class Real> void ApplyStoutinTime(_gauge<Real> array, Real w, int steps)
{
    detail::check(sun_smear_stout(array.lat(), w, steps, SUN_SMEAR_TIME, nullptr), "ApplyStoutinTime");
}

// HYP weights (src/smear/hyp.cu:374-398); copyToGPUMem has nothing to do:
// the weights travel with each call
class ParamHYP {
    float alpha1, alpha2, alpha3;

public:
    ParamHYP() { setDefault(); }
    ParamHYP(float a1, float a2, float a3) { set(a1, a2, a3); }
    void setDefault() { set(0.75f, 0.6f, 0.3f); }
    void set(float a1, float a2, float a3)
    {
        alpha1 = a1;
        alpha2 = a2;
        alpha3 = a3;
    }
    void print() const { printf("HYP alpha1 = %g alpha2 = %g alpha3 = %g\n", alpha1, alpha2, alpha3); }
    void copyToGPUMem() const {}
    void get(double a[3]) const
    {
        a[0] = alpha1;
        a[1] = alpha2;
        a[2] = alpha3;
    }
};

template <class Real> void ApplyHYPinSpace(_gauge<Real> array, int steps, int nhits, Real tol, ParamHYP hyp)
{
    double a[3];
    hyp.get(a);
    detail::check(sun_smear_hyp(array.lat(), a, steps, nhits, tol, SUN_SMEAR_SPACE, nullptr), "ApplyHYPinSpace");
}
template <class Real> void ApplyHYPinTime(_gauge<Real> array, int steps, int nhits, Real tol, ParamHYP hyp)
{
    double a[3];
    hyp.get(a);
    detail::check(sun_smear_hyp(array.lat(), a, steps, nhits, tol, SUN_SMEAR_TIME, nullptr), "ApplyHYPinTime");
}
// arrayout: SOA layout; the RNG's seed keys the Philox stream
template <class Real> void ApplyMultiHit(_gauge<Real> array, _gauge<Real> arrayout, RNG& randstates, int nhit)
{
    detail::check(sun_multihit(array.lat(), arrayout.lat(), nhit, randstates.seed, nullptr), "ApplyMultiHit");
}
template <class Real> void ApplyMultiHitSpace(_gauge<Real> array, _gauge<Real> arrayout, RNG& /*randstates*/, int nhit)
{
    detail::check(sun_multihit_space(array.lat(), arrayout.lat(), nhit, nullptr), "ApplyMultiHitSpace");
}

template <class Real, class RealSave>
void SaveBin_Gauge(_gauge<Real>& array, const std::string& file, bool withheader = false)
{
    detail::check(sun_save_bin(array.lat(), file.c_str(), sizeof(RealSave) == 8, withheader), "SaveBin_Gauge");
}

template <class Real, class RealSave>
void ReadBin_Gauge(_gauge<Real>& array, const std::string& file, bool withheader = false)
{
    detail::check(sun_load_bin(array.lat(), file.c_str(), sizeof(RealSave) == 8, withheader), "ReadBin_Gauge");
}

}  // namespace CULQCD

// the reference spells its array type `gauge` (gaugearray.h:468)
#ifndef CULQCD_B200_NO_GAUGE_MACRO
#define gauge _gauge<Real>
#endif

#endif
