#!/usr/bin/env python
"""Generate golden vectors by running the reference (nmrcardoso/sun) itself.

Runs on a machine with a GPU and the prebuilt reference probes in
oracle/_ref/ (built by `make -C oracle/ref`; the reference sources are only
needed for that build).  Inputs are seeded configurations from the oracle,
written in the reference's own gauge file format; the outputs are what the
reference's public API and device functions return for them:

  * PlaquetteCUB / OnePolyakovLoop / WilsonLoop on fixed configurations
    (src/meas/plaquette_cub.cu:226, polyakovloop.cu:637, wilsonloop.cu:535),
    including a lattice with four different extents;
  * one OverRelaxation::Run pass (src/monte/ovr.cu:182) and
    Reunitarize::Run (src/reunitarize.cu:78), read back with ReadBin_Gauge;
  * per-link heatBathSUN with injected uniforms, overrelaxationSUN and
    reunit_link (include/device_PHB_OVR.h:362, :494; reunitlink.h:16);
  * a beta = 6.0 SU(3) 8^4 ensemble from the reference's own heatbath +
    overrelaxation chain (cuRAND MRG32k3a), plaquette per sweep;
  * the reference build's sweep timings on this GPU (32^4).

Usage: python tests/golden/make_golden.py OUTDIR
Writes OUTDIR/reference_golden.npz and OUTDIR/reference_meta.json.
"""
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

PROBE = os.path.join(ROOT, "oracle", "_ref", "ref_probe")
LINK = os.path.join(ROOT, "oracle", "_ref", "ref_link_probe")

CONFIGS = [  # name, dims (x, y, z, t), beta, seed, oracle sweeps
    ("c4444", (4, 4, 4, 4), 5.8, 11, 2),
    ("c4448", (4, 4, 4, 8), 6.0, 12, 2),
    ("c4648", (4, 6, 4, 8), 5.7, 13, 1),
]


def run(args, timeout=600):
    r = subprocess.run(args, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"{' '.join(args)} failed ({r.returncode}):\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
    return r.stdout


def main(out):
    os.makedirs(out, exist_ok=True)
    tmp = os.path.join(out, "tmp")
    os.makedirs(tmp, exist_ok=True)
    arrays, meta = {}, {"configs": [], "probe": "oracle/_ref/ref_probe", "when": time.strftime("%Y-%m-%dT%H:%M:%SZ")}
    for name, dims, beta, seed, nsw in CONFIGS:
        X = list(dims)
        U = O.hot(3, X, seed)
        O.sweeps(U, X, beta, 1, 1, nsw, seed=seed)
        f = os.path.join(tmp, f"{name}.bin")
        assert O.save_bin(U, X, beta, f) == 0
        args = [str(d) for d in dims] + [repr(beta)]
        R, T = min(2, min(dims[:3]) - 1), min(3, dims[3] - 1)
        txt = run([PROBE, "measure", f] + args + [str(R), str(T)])
        plaq = pol = None
        wl = np.zeros((R + 1, T + 1, 2))
        for line in txt.splitlines():
            p = line.split()
            if p and p[0] == "plaquette":
                plaq = [float(p[1]), float(p[2])]
            elif p and p[0] == "polyakov":
                pol = [float(p[1]), float(p[2])]
            elif p and p[0] == "wilson":
                wl[int(p[1]), int(p[2])] = [float(p[3]), float(p[4])]
        arrays[f"{name}_U"] = U
        arrays[f"{name}_plaquette"] = np.array(plaq)
        arrays[f"{name}_polyakov"] = np.array(pol)
        arrays[f"{name}_wilson"] = wl
        # one overrelaxation pass of the reference
        fo = os.path.join(tmp, f"{name}_or.bin")
        run([PROBE, "overrelax", f, fo] + args + ["1"])
        rc, Uor, g, b = O.load_bin(3, X, fo)
        assert rc == 0 and g == X
        arrays[f"{name}_or1"] = Uor
        # reunitarization of a perturbed configuration
        rng = np.random.default_rng(seed)
        P = U + 1e-3 * (rng.standard_normal(U.shape) + 1j * rng.standard_normal(U.shape))
        fp = os.path.join(tmp, f"{name}_pert.bin")
        assert O.save_bin(P, X, beta, fp) == 0
        fr = os.path.join(tmp, f"{name}_reunit.bin")
        run([PROBE, "reunit", fp, fr] + args)
        rc, Ure, g, b = O.load_bin(3, X, fr)
        assert rc == 0
        arrays[f"{name}_pert"] = P
        arrays[f"{name}_reunit"] = Ure
        meta["configs"].append({"name": name, "dims": list(dims), "beta": beta, "seed": seed, "oracle_sweeps": nsw,
                                "R": R, "T": T})

    # per-link device functions with injected uniforms
    X = [4, 4, 4, 4]
    U = arrays["c4444_U"]
    links, Fs = [], []
    for lex in range(0, O.volume(X), 4):
        for mu in range(4):
            links.append(U[lex, mu])
            Fs.append(O.staple(U, X, lex, mu).conj().T)
    Ul = np.ascontiguousarray(np.array(links)[:128])
    Fl = np.ascontiguousarray(np.array(Fs)[:128])
    stride = 3 * 86
    rng = np.random.default_rng(99)
    uni = (rng.integers(0, 2 ** 53, size=(len(Ul), stride), dtype=np.int64) + 1) / 2.0 ** 53
    for mode, beta in (("hb", 5.8), ("hb_lowbeta", 0.7), ("or", 5.8), ("reunit", 5.8)):
        fi = os.path.join(tmp, f"link_{mode}.in")
        fo = os.path.join(tmp, f"link_{mode}.out")
        Uin = Ul if mode != "reunit" else Ul + 1e-3 * (rng.standard_normal(Ul.shape) + 1j * rng.standard_normal(Ul.shape))
        with open(fi, "wb") as fh:
            np.array([len(Ul), stride], dtype=np.int32).tofile(fh)
            Uin.astype(np.complex128).tofile(fh)
            Fl.astype(np.complex128).tofile(fh)
            uni.astype(np.float64).tofile(fh)
        run([LINK, mode.split("_")[0], fi, fo, repr(beta)])
        raw = open(fo, "rb").read()
        n = len(Ul)
        Uout = np.frombuffer(raw[: n * 9 * 16], dtype=np.complex128).reshape(n, 3, 3)
        used = np.frombuffer(raw[n * 9 * 16:], dtype=np.int32)
        arrays[f"link_{mode}_in"] = Uin
        arrays[f"link_{mode}_out"] = Uout
        arrays[f"link_{mode}_used"] = used
        arrays[f"link_{mode}_beta"] = np.array(beta)
    arrays["link_F"] = Fl
    arrays["link_uniforms"] = uni

    # the reference's own Monte Carlo chain (MRG32k3a): ensemble plaquette
    txt = run([PROBE, "ensemble", "8", "8", "8", "8", "6.0", "1234", "200", "2000"], timeout=1800)
    pl = np.array([[float(v) for v in line.split()[2:4]] for line in txt.splitlines() if line.startswith("plaq ")])
    arrays["ensemble_b6_8x4_plaquette"] = pl
    meta["ensemble"] = {"dims": [8, 8, 8, 8], "beta": 6.0, "seed": 1234, "therm": 200, "meas": 2000,
                        "sweep": "1 HeatBath + 4 OverRelaxation, Reunitarize every 10"}

    # reference-build timings on this GPU
    timings = {}
    env = dict(os.environ, SUN_REF_TUNE="1", CULQCD_RESOURCE_PATH=tmp)
    for kind in ("f32soa12", "f64soa"):
        r = subprocess.run([PROBE, "timing", "32", "32", "32", "32", "6.0", "20", kind], capture_output=True,
                           text=True, timeout=1200, env=env)
        line = [l for l in r.stdout.splitlines() if l.startswith("timing")]
        timings[kind] = line[0] if line else f"failed rc={r.returncode}: {r.stderr[-300:]}"
    meta["timings_32x4"] = timings
    np.savez_compressed(os.path.join(out, "reference_golden.npz"), **arrays)
    with open(os.path.join(out, "reference_meta.json"), "w") as fh:
        json.dump(meta, fh, indent=1)
    print(json.dumps(meta["timings_32x4"], indent=1))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "golden_out")
