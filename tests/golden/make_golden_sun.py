#!/usr/bin/env python
"""Golden vectors for SU(4), SU(6) and for Wilson loops up to 4 x 4, made by
running the reference (nmrcardoso/sun) itself.

The reference fixes N at compile time (NCOLORS); `make -C oracle/ref ncolors`
builds it for N = 4 (oracle/_ref_n4/) and N = 6 (oracle/_ref_n6/), and
`make -C oracle/ref` for N = 3 (oracle/_ref/).  This script runs those probes
on a machine with a GPU.  Every input is regenerated by the oracle from a
seed (Haar hot start and Philox sweeps, bit-reproducible), written in the
reference's own gauge file format, so only the reference's outputs are kept:

  * PlaquetteCUB / OnePolyakovLoop / WilsonLoop (src/meas/plaquette_cub.cu:226,
    polyakovloop.cu:637, wilsonloop.cu:535) with R = T = 4 on 8^4 and
    6^3 x 10 lattices for N = 3, 4, 6, and R = 2, T = 3 on 4^4 for N = 4, 6;
  * one OverRelaxation::Run pass (src/monte/ovr.cu:182) on 4^4 for N = 4, 6
    -- the N != 3 path of overrelaxationSUN (include/device_PHB_OVR.h:557-567);
  * per link, for N = 4, 6: heatBathSUN with injected uniforms (the N != 3
    path M = U F, device_PHB_OVR.h:426-441, and the number of uniforms it
    consumes), overrelaxationSUN, and reunit_link (column Gram-Schmidt with
    the determinant phase, include/reunitlink.h:46-84).

Usage: python tests/golden/make_golden_sun.py OUTDIR
Writes OUTDIR/reference_golden_sun.npz and OUTDIR/reference_meta_sun.json.
The tests rebuild the inputs with `config()` and `link_inputs()` below.
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

PROBES = {3: "_ref", 4: "_ref_n4", 6: "_ref_n6"}

# name, N, dims (x, y, z, t), beta, seed, oracle sweeps (1 HB + 1 OR each), R, T, overrelaxation pass
CONFIGS = [
    ("n3_w8x4", 3, (8, 8, 8, 8), 6.0, 301, 3, 4, 4, False),
    ("n3_w6x10", 3, (6, 6, 6, 10), 5.8, 302, 3, 4, 4, False),
    ("n4_c4444", 4, (4, 4, 4, 4), 11.1, 401, 2, 2, 3, True),
    ("n4_w8x4", 4, (8, 8, 8, 8), 11.1, 402, 3, 4, 4, False),
    ("n4_w6x10", 4, (6, 6, 6, 10), 10.4, 403, 3, 4, 4, False),
    ("n6_c4444", 6, (4, 4, 4, 4), 25.0, 601, 2, 2, 3, True),
    ("n6_w8x4", 6, (8, 8, 8, 8), 25.0, 602, 3, 4, 4, False),
    ("n6_w6x10", 6, (6, 6, 6, 10), 24.0, 603, 3, 4, 4, False),
]
# per-link cases: (mode, beta) for N = 4, 6; the low beta reaches the Creutz branch
LINK_MODES = {4: (("hb", 11.1), ("hb_lowbeta", 1.0), ("or", 11.1), ("reunit", 11.1)),
              6: (("hb", 25.0), ("hb_lowbeta", 2.0), ("or", 25.0), ("reunit", 25.0))}
NLINKS = 64


def config(name, N, dims, beta, seed, nsw):
    """The configuration of a CONFIGS entry (oracle, deterministic)."""
    X = list(dims)
    U = O.hot(N, X, seed)
    O.sweeps(U, X, beta, 1, 1, nsw, seed=seed)
    return U


def link_inputs(N):
    """Links, F = staple^dagger and injected uniforms of the per-link cases:
    NLINKS links of the N's 4^4 configuration, uniforms from the oracle's
    Philox stream (seed 900 + N, one stream per link)."""
    c = [c for c in CONFIGS if c[1] == N and c[2] == (4, 4, 4, 4)][0]
    X = list(c[2])
    U = config(c[0], N, c[2], c[3], c[4], c[5])
    links, Fs = [], []
    for lex in range(0, O.volume(X), 4):
        for mu in range(4):
            links.append(U[lex, mu])
            Fs.append(O.staple(U, X, lex, mu).conj().T)
    Ul = np.ascontiguousarray(np.array(links)[:NLINKS])
    Fl = np.ascontiguousarray(np.array(Fs)[:NLINKS])
    stride = (N * (N - 1) // 2) * 86  # 21 tries of 4 uniforms + 2 per subgroup
    uni = np.stack([O.uniforms(900 + N, i, 0, stride, fp64=True) for i in range(NLINKS)])
    # reunit_link input: the links perturbed by up to 1e-3 per entry (uniforms of seed 950 + N)
    e = np.stack([O.uniforms(950 + N, i, 1, 2 * N * N, fp64=True) for i in range(NLINKS)]) - 0.5
    P = Ul + 2e-3 * (e[:, : N * N] + 1j * e[:, N * N:]).reshape(NLINKS, N, N)
    return Ul, Fl, np.ascontiguousarray(uni), np.ascontiguousarray(P)


def run(args, timeout=900):
    r = subprocess.run(args, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"{' '.join(args)} failed ({r.returncode}):\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
    return r.stdout


def main(out):
    os.makedirs(out, exist_ok=True)
    tmp = os.path.join(out, "tmp_sun")
    os.makedirs(tmp, exist_ok=True)
    arrays, meta = {}, {"configs": [], "link_modes": {}, "when": time.strftime("%Y-%m-%dT%H:%M:%SZ")}
    for name, N, dims, beta, seed, nsw, R, T, do_or in CONFIGS:
        probe = os.path.join(ROOT, "oracle", PROBES[N], "ref_probe")
        X = list(dims)
        U = config(name, N, dims, beta, seed, nsw)
        f = os.path.join(tmp, f"{name}.bin")
        assert O.save_bin(U, X, beta, f) == 0
        args = [str(d) for d in dims] + [repr(beta)]
        txt = run([probe, "measure", f] + args + [str(R), str(T)])
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
        arrays[f"{name}_plaquette"] = np.array(plaq)
        arrays[f"{name}_polyakov"] = np.array(pol)
        arrays[f"{name}_wilson"] = wl
        # a sample of the input, to check that the tests rebuild the same one
        arrays[f"{name}_U_sample"] = U[::97].copy()
        if do_or:
            fo = os.path.join(tmp, f"{name}_or.bin")
            run([probe, "overrelax", f, fo] + args + ["1"])
            rc, Uor, g, b = O.load_bin(N, X, fo)
            assert rc == 0 and g == X
            arrays[f"{name}_or1"] = Uor
        meta["configs"].append({"name": name, "N": N, "dims": list(dims), "beta": beta, "seed": seed,
                                "oracle_sweeps": nsw, "R": R, "T": T, "overrelax": do_or})
    for N, modes in LINK_MODES.items():
        link = os.path.join(ROOT, "oracle", PROBES[N], "ref_link_probe")
        Ul, Fl, uni, P = link_inputs(N)
        for mode, beta in modes:
            fi = os.path.join(tmp, f"n{N}_link_{mode}.in")
            fo = os.path.join(tmp, f"n{N}_link_{mode}.out")
            Uin = P if mode == "reunit" else Ul
            with open(fi, "wb") as fh:
                np.array([len(Ul), uni.shape[1]], dtype=np.int32).tofile(fh)
                Uin.astype(np.complex128).tofile(fh)
                Fl.astype(np.complex128).tofile(fh)
                uni.astype(np.float64).tofile(fh)
            run([link, mode.split("_")[0], fi, fo, repr(beta)])
            raw = open(fo, "rb").read()
            n = len(Ul)
            arrays[f"n{N}_link_{mode}_out"] = np.frombuffer(raw[: n * N * N * 16], dtype=np.complex128).reshape(n, N, N)
            arrays[f"n{N}_link_{mode}_used"] = np.frombuffer(raw[n * N * N * 16:], dtype=np.int32)
            meta["link_modes"][f"n{N}_{mode}"] = beta
    np.savez_compressed(os.path.join(out, "reference_golden_sun.npz"), **arrays)
    with open(os.path.join(out, "reference_meta_sun.json"), "w") as fh:
        json.dump(meta, fh, indent=1)
    print("ok", len(arrays), "arrays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "golden_out")
