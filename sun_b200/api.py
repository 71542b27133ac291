"""Python host API over the C ABI, named after the reference's entry points.

CULQCD user code reads::

    initCULQCD(gpuid, SUMMARIZE, TUNE_YES);                 // comm_mpi.cpp:107
    SETPARAMS(usetex, beta, nx, ny, nz, nt, verbose);        // constants.cu:149
    gauge AA(SOA, Device, PARAMS::Volume * 4, true);         // gaugearray.h:139
    AA.Init(rng);                                            // gaugearray.h:781
    HeatBath<double> hb(AA, rng); hb.Run();                  // monte.cu:152, :196
    OverRelaxation<double> ovr(AA); ovr.Run();               // ovr.cu:139, :182
    Reunitarize<double> reu(AA); reu.Run();                  // reunitarize.cu:40, :78
    PlaquetteCUB<double> plaq(AA); complexd p = plaq.Run();  // plaquette_cub.cu:161, :226
    OnePolyakovLoop<double> pl(AA); complexd l = pl.Run();   // polyakovloop.cu:637
    WilsonLoop<double>(BB, res, R, T);                       // wilsonloop.cu:535
    SaveBin_Gauge<double,double>(AA, file, true);            // io_gauge.cpp:429
    EndCULQCD(0);                                            // comm_mpi.cpp:186

and the same program against this engine reads::

    ctx = initCULQCD(0)
    AA = gauge(ctx, N=3, dims=(nx, ny, nz, nt), beta=beta, atype=SOA, evenodd=True, prec="f64", seed=s)
    AA.Init(hot=True)
    HeatBath(AA).Run(); OverRelaxation(AA).Run(); Reunitarize(AA).Run()
    p = PlaquetteCUB(AA).Run()      # complex(spatial, temporal), like the reference
    l = OnePolyakovLoop(AA).Run()
    w = WilsonLoop(AA, R, T)        # complex array [r, t]
    SaveBin_Gauge(AA, file, True)
    EndCULQCD(ctx)

Differences, all deliberate: geometry and N are per-lattice (no SETPARAMS
globals, no compile-time NCOLORS); errors raise SunError instead of exiting;
the RNG is a counter-based Philox stream owned by the lattice (no RNG object
to allocate); Wilson loops accept even/odd arrays directly.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _native as nat
from ._native import SunError, SunJob, SunLatticeParams, SunResult, check, lib

SOA, SOA12, SOA8 = nat.SOA, nat.SOA12, nat.SOA8
_PREC = {"f32": nat.F32, "f64": nat.F64, "float": nat.F32, "double": nat.F64}


class Context:
    """initCULQCD / EndCULQCD: one device, one default stream."""

    def __init__(self, device: int = 0, verbosity: int = 0, tune: bool = False,
                 hbm_budget_bytes: int = 0, tune_cache_path: Optional[str] = None):
        self._tune_path = tune_cache_path.encode() if tune_cache_path else None
        cfg = nat.SunConfig(device, verbosity, int(tune), self._tune_path, hbm_budget_bytes)
        h = C.c_void_p()
        check(lib().sun_init(C.byref(cfg), C.byref(h)))
        self.h = h

    def close(self) -> None:
        if self.h:
            lib().sun_finalize(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def initCULQCD(gpuid: int = 0, verbosity: int = 0, tune: bool = False) -> Context:
    return Context(gpuid, verbosity, tune)


def EndCULQCD(ctx: Context) -> None:
    ctx.close()


class gauge:
    """A gauge array on the device (``_gauge<Real>``, include/gaugearray.h:88)."""

    def __init__(self, ctx: Context, N: int = 3, dims: Sequence[int] = (4, 4, 4, 4), beta: float = 6.0,
                 atype: int = SOA, evenodd: bool = True, prec: str = "f64", seed: int = 1234,
                 reunit_every: int = 0):
        self.ctx = ctx
        self.N = int(N)
        self.dims = tuple(int(d) for d in dims)
        self.beta = float(beta)
        self.atype = int(atype)
        self.evenodd = bool(evenodd)
        self.prec = prec
        self.seed = int(seed)
        p = SunLatticeParams(self.N, (C.c_int * 4)(*self.dims), self.beta, self.atype,
                             nat.EVEN_ODD if evenodd else nat.NORMAL, _PREC[prec], self.seed, int(reunit_every))
        h = C.c_void_p()
        check(lib().sun_lattice_create(ctx.h, C.byref(p), C.byref(h)), ctx.h)
        self.h = h

    # -- properties ---------------------------------------------------------
    @property
    def volume(self) -> int:
        return int(np.prod(self.dims))

    def Bytes(self) -> int:
        b = C.c_size_t()
        check(lib().sun_lattice_bytes(self.h, C.byref(b)))
        return b.value

    def GetPtr(self) -> int:
        p = C.c_void_p()
        check(lib().sun_lattice_device_ptr(self.h, C.byref(p)))
        return p.value

    def Release(self) -> None:
        if self.h:
            lib().sun_lattice_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.Release()
        except Exception:
            pass

    # -- initialisation -------------------------------------------------------
    def Init(self, hot: bool = False) -> None:
        """Cold (identity) or hot (Haar, Philox-seeded) start."""
        f = lib().sun_lattice_init_hot if hot else lib().sun_lattice_init_cold
        check(f(self.h, None), self.ctx.h)

    # -- host transfer (canonical complex128 [V, 4, N, N], x fastest) --------
    def Set(self, U: np.ndarray) -> None:
        U = np.ascontiguousarray(U, dtype=np.complex128)
        assert U.shape == (self.volume, 4, self.N, self.N)
        check(lib().sun_lattice_upload(self.h, U.ctypes.data, nat.HOST_CANONICAL, None), self.ctx.h)

    def Get(self) -> np.ndarray:
        U = np.empty((self.volume, 4, self.N, self.N), dtype=np.complex128)
        check(lib().sun_lattice_download(self.h, U.ctypes.data, nat.HOST_CANONICAL, None), self.ctx.h)
        return U

    def set_image(self, img: np.ndarray) -> None:
        check(lib().sun_lattice_upload(self.h, img.ctypes.data, nat.HOST_IMAGE, None), self.ctx.h)

    def get_image(self) -> np.ndarray:
        dt = np.complex128 if _PREC[self.prec] == nat.F64 else np.complex64
        img = np.empty(self.Bytes() // np.dtype(dt).itemsize, dtype=dt)
        check(lib().sun_lattice_download(self.h, img.ctypes.data, nat.HOST_IMAGE, None), self.ctx.h)
        return img

    def Copy(self, other: "gauge") -> None:
        """self <- other, converting layout / order / precision (gauge::Copy)."""
        check(lib().sun_lattice_copy(self.h, other.h, None), self.ctx.h)

    # -- RNG checkpoint -------------------------------------------------------
    def rng_state(self):
        s, h, w = C.c_uint64(), C.c_uint32(), C.c_uint32()
        check(lib().sun_lattice_get_rng(self.h, C.byref(s), C.byref(h), C.byref(w)), self.ctx.h)
        return s.value, h.value, w.value

    def set_sweep_limit(self, limit: int) -> None:
        """Sweeps leave the lattice unchanged once its sweep counter reaches
        `limit` (0: no limit)."""
        check(lib().sun_lattice_set_sweep_limit(self.h, int(limit)), self.ctx.h)

    def set_rng_state(self, seed: int, hb_passes: int, sweeps: int) -> None:
        check(lib().sun_lattice_set_rng(self.h, seed, hb_passes, sweeps), self.ctx.h)
        self.seed = seed


class HeatBath:
    """HeatBath<Real>(gauge&, RNG&).Run(): one pass = 2 parities x 4 directions."""

    def __init__(self, g: gauge):
        self.g = g

    def Run(self, n: int = 1) -> None:
        check(lib().sun_heatbath(self.g.h, n, None), self.g.ctx.h)

    def RunInjected(self, dev_uniforms_ptr: int, stride: int) -> None:
        check(lib().sun_heatbath_injected(self.g.h, C.c_void_p(dev_uniforms_ptr), stride, None), self.g.ctx.h)


class OverRelaxation:
    def __init__(self, g: gauge):
        self.g = g

    def Run(self, n: int = 1) -> None:
        check(lib().sun_overrelax(self.g.h, n, None), self.g.ctx.h)


def Sweep(g: gauge, n_hb: int = 1, n_or: int = 4, n_sweeps: int = 1) -> None:
    check(lib().sun_sweep(g.h, n_hb, n_or, n_sweeps, None), g.ctx.h)


def SweepMeasure(g: gauge, n_hb: int = 1, n_or: int = 4, n_sweeps: int = 1):
    """n_sweeps sweeps with the plaquette and Polyakov loop after each:
    returns (plaquette [n_sweeps, 2] {spatial, temporal}, Polyakov loop
    [n_sweeps] complex)."""
    pl = np.zeros(2 * n_sweeps)
    po = np.zeros(2 * n_sweeps)
    dp = C.POINTER(C.c_double)
    check(lib().sun_sweep_measure(g.h, n_hb, n_or, n_sweeps, pl.ctypes.data_as(dp), po.ctypes.data_as(dp), None),
          g.ctx.h)
    return pl.reshape(n_sweeps, 2), po[0::2] + 1j * po[1::2]


class Reunitarize:
    def __init__(self, g: gauge):
        self.g = g

    def Run(self) -> None:
        check(lib().sun_reunitarize(self.g.h, None), self.g.ctx.h)


def unitarity_violation(g: gauge) -> float:
    v = C.c_double()
    check(lib().sun_unitarity_violation(g.h, C.byref(v), None), g.ctx.h)
    return v.value


def link_trace_det(g: gauge):
    """(mean tr U / N, mean det U) as complex numbers -- GaugeTraceCUB and
    GaugeDetCUB (src/meas/linktrsum.cu, src/meas/linkdetsum.cu)."""
    o = (C.c_double * 4)()
    check(lib().sun_link_trace_det(g.h, o, None), g.ctx.h)
    return complex(o[0], o[1]), complex(o[2], o[3])


class PlaquetteCUB:
    """Run() -> complex(spatial, temporal); mean = (re + im) / 2."""

    def __init__(self, g: gauge):
        self.g = g
        self.value = 0j

    def Run(self) -> complex:
        o = (C.c_double * 2)()
        check(lib().sun_plaquette(self.g.h, o, None), self.g.ctx.h)
        self.value = complex(o[0], o[1])
        return self.value

    def mean(self) -> float:
        return (self.value.real + self.value.imag) / 2


class OnePolyakovLoop:
    def __init__(self, g: gauge):
        self.g = g

    def Run(self) -> complex:
        o = (C.c_double * 2)()
        check(lib().sun_polyakov(self.g.h, o, None), self.g.ctx.h)
        return complex(o[0], o[1])


def WilsonLoop(g: gauge, R: int, T: int) -> np.ndarray:
    """res[r, t] complex for r <= R, t <= T (the reference's res[t + r(T+1)])."""
    o = np.zeros(2 * (R + 1) * (T + 1))
    check(lib().sun_wilson_loops(g.h, R, T, o.ctypes.data_as(C.POINTER(C.c_double)), None), g.ctx.h)
    o = o.reshape(R + 1, T + 1, 2)
    return o[..., 0] + 1j * o[..., 1]


# -- smearing and multihit (src/smear/); in place unless an output is given --
SMEAR_SPACE, SMEAR_TIME = 7, 8


def ApplyAPEinSpace(g: gauge, w: float, steps: int, nhits: int, tol: float) -> None:
    """APE smearing of the spatial links (src/smear/ape.cu:192)."""
    check(lib().sun_smear_ape(g.h, w, steps, nhits, tol, SMEAR_SPACE, None), g.ctx.h)


def ApplyAPEinTime(g: gauge, w: float, steps: int, nhits: int, tol: float) -> None:
    """APE smearing of the temporal links (src/smear/ape.cu:237)."""
    check(lib().sun_smear_ape(g.h, w, steps, nhits, tol, SMEAR_TIME, None), g.ctx.h)


def ApplyStoutinSpace(g: gauge, w: float, steps: int) -> None:
    """Stout smearing of the spatial links, SU(3) (src/smear/stout.cu:687)."""
    check(lib().sun_smear_stout(g.h, w, steps, SMEAR_SPACE, None), g.ctx.h)


def ApplyStoutinTime(g: gauge, w: float, steps: int) -> None:
    """Stout smearing of the temporal links, SU(3) (src/smear/stout.cu:734)."""
    check(lib().sun_smear_stout(g.h, w, steps, SMEAR_TIME, None), g.ctx.h)


class ParamHYP:
    """HYP weights alpha1, alpha2, alpha3 (ParamHYP, src/smear/hyp.cu:374-398), FP32."""

    def __init__(self, alpha1: float = 0.75, alpha2: float = 0.6, alpha3: float = 0.3):
        self.set(alpha1, alpha2, alpha3)

    def setDefault(self) -> None:
        self.set(0.75, 0.6, 0.3)

    def set(self, alpha1: float, alpha2: float, alpha3: float) -> None:
        self.alpha = (float(np.float32(alpha1)), float(np.float32(alpha2)), float(np.float32(alpha3)))

    def print(self) -> None:
        print("HYP: alpha1 = %g alpha2 = %g alpha3 = %g" % self.alpha)


def _hyp(g: gauge, steps: int, nhits: int, tol: float, hyp: Optional[ParamHYP], mask: int) -> None:
    a = (C.c_double * 3)(*(hyp or ParamHYP()).alpha)
    check(lib().sun_smear_hyp(g.h, a, steps, nhits, tol, mask, None), g.ctx.h)


def ApplyHYPinSpace(g: gauge, steps: int, nhits: int, tol: float, hyp: Optional[ParamHYP] = None) -> None:
    """HYP smearing of the spatial links (src/smear/hyp.cu:277)."""
    _hyp(g, steps, nhits, tol, hyp, SMEAR_SPACE)


def ApplyHYPinTime(g: gauge, steps: int, nhits: int, tol: float, hyp: Optional[ParamHYP] = None) -> None:
    """HYP smearing of the temporal links (src/smear/hyp.cu:328)."""
    _hyp(g, steps, nhits, tol, hyp, SMEAR_TIME)


def ApplyMultiHit(g: gauge, out: gauge, seed: int, nhit: int) -> None:
    """out <- g with each temporal link replaced by the mean of itself and nhit
    heatbath updates against its staple (src/smear/multihit.cu:318).  `seed`
    keys the Philox stream (the reference takes an RNG&); out uses SOA."""
    check(lib().sun_multihit(g.h, out.h, nhit, seed, None), out.ctx.h)


def ApplyMultiHitSpace(g: gauge, out: gauge, nhit: int) -> None:
    """out <- g with each spatial link replaced by the mean of nhit
    overrelaxation iterates (src/smear/multihitsp.cu:246); out uses SOA."""
    check(lib().sun_multihit_space(g.h, out.h, nhit, None), out.ctx.h)


def SaveBin_Gauge(g: gauge, filename: str, withheader: bool = True, save_fp64: bool = True) -> None:
    check(lib().sun_save_bin(g.h, filename.encode(), int(save_fp64), int(withheader)), g.ctx.h)


def ReadBin_Gauge(g: gauge, filename: str, withheader: bool = True, save_fp64: bool = True) -> None:
    check(lib().sun_load_bin(g.h, filename.encode(), int(save_fp64), int(withheader)), g.ctx.h)


class Batch:
    """Many lattices advanced together (one launch per class and phase)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        h = C.c_void_p()
        check(lib().sun_batch_create(ctx.h, C.byref(h)), ctx.h)
        self.h = h
        self.members = []

    def add(self, g: gauge) -> None:
        check(lib().sun_batch_add(self.h, g.h), self.ctx.h)
        self.members.append(g)

    def remove(self, g: gauge) -> None:
        check(lib().sun_batch_remove(self.h, g.h), self.ctx.h)
        self.members.remove(g)

    def sweep(self, n_hb: int = 1, n_or: int = 4, n_sweeps: int = 1, graph: bool = False) -> None:
        check(lib().sun_batch_sweep(self.h, n_hb, n_or, n_sweeps, int(graph), None), self.ctx.h)

    def plaquette(self) -> np.ndarray:
        o = np.zeros(2 * len(self.members))
        check(lib().sun_batch_plaquette(self.h, o.ctypes.data_as(C.POINTER(C.c_double)), None), self.ctx.h)
        return o.reshape(-1, 2)

    def wilson_loops(self, R: int, T: int) -> np.ndarray:
        """W(r, t) of every lattice: complex [n, R + 1, T + 1]."""
        n = len(self.members)
        out = np.zeros(n * 2 * (R + 1) * (T + 1))
        check(lib().sun_batch_wilson_loops(self.h, R, T, out.ctypes.data_as(C.POINTER(C.c_double)), None), self.ctx.h)
        o = out.reshape(n, R + 1, T + 1, 2)
        return o[..., 0] + 1j * o[..., 1]

    def polyakov(self) -> np.ndarray:
        o = np.zeros(2 * len(self.members))
        check(lib().sun_batch_polyakov(self.h, o.ctypes.data_as(C.POINTER(C.c_double)), None), self.ctx.h)
        return o.reshape(-1, 2)

    def close(self) -> None:
        if self.h:
            lib().sun_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_job(N=3, dims=(8, 8, 8, 8), beta=6.0, sweeps=10, n_hb=1, n_or=4, seed=1, hot=True,
             observables=1, R=0, T=0, prec="f32", layout=SOA, reunit_every=0) -> SunJob:
    return SunJob(N, (C.c_int * 4)(*dims), beta, sweeps, n_hb, n_or, seed, int(hot), observables, R, T,
                  _PREC[prec], layout, reunit_every)


class Server:
    """Continuous-batching job server (sun_server_*)."""

    def __init__(self, ctx: Context, max_active: int = 64, budget_bytes: Optional[int] = None):
        self.ctx = ctx
        h = C.c_void_p()
        check(lib().sun_server_create(ctx.h, max_active, C.byref(h)), ctx.h)
        self.h = h
        if budget_bytes is not None:
            check(lib().sun_server_set_budget(self.h, budget_bytes))
        self.cap = max(256, 4 * max_active)
        self._buf = (SunResult * self.cap)()

    def submit(self, job: SunJob) -> int:
        i = C.c_int64()
        check(lib().sun_server_submit(self.h, C.byref(job), C.byref(i)), self.ctx.h)
        return i.value

    def step(self):
        n = C.c_int()
        check(lib().sun_server_step(self.h, self._buf, self.cap, C.byref(n)), self.ctx.h)
        out = []
        for k in range(n.value):
            r = self._buf[k]
            out.append(dict(id=r.id, status=r.status, plaquette=(r.plaquette[0], r.plaquette[1]),
                            polyakov=(r.polyakov[0], r.polyakov[1]), wilson=list(r.wilson),
                            submit_s=r.submit_s, start_s=r.start_s, finish_s=r.finish_s,
                            link_updates=r.link_updates))
        return out

    def pending(self):
        q, a = C.c_int(), C.c_int()
        check(lib().sun_server_pending(self.h, C.byref(q), C.byref(a)))
        return q.value, a.value

    def stats(self) -> dict:
        """Where the steps spent their time (sun_server_get_stats)."""
        from ._native import SunServerStats
        st = SunServerStats()
        check(lib().sun_server_get_stats(self.h, C.byref(st)))
        return {name: getattr(st, name) for name, _ in SunServerStats._fields_}

    def close(self) -> None:
        if self.h:
            lib().sun_server_destroy(self.h)
            self.h = None


def job_footprint(job: SunJob) -> int:
    b = C.c_size_t()
    check(lib().sun_job_footprint(C.byref(job), C.byref(b)))
    return b.value


def admit_count(footprints, budget: int, used: int, free_slots: int) -> int:
    arr = (C.c_size_t * max(1, len(footprints)))(*footprints)
    n = C.c_int()
    check(lib().sun_admit_count(arr, len(footprints), budget, used, free_slots, C.byref(n)))
    return n.value
