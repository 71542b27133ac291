#!/usr/bin/env python
"""Generate golden smearing vectors by running the reference itself.

Runs on a machine with a GPU and the prebuilt reference probe
oracle/_ref/ref_probe (built by `make -C oracle/ref`).  Inputs are seeded,
thermalized SU(3) configurations from the oracle, written in the reference's
gauge file format; each output holds the smeared directions of the
configuration after one call of the reference's smearing API
(src/smear/ape.cu, stout.cu, hyp.cu, multihitsp.cu) on a normal-order SOA
copy, read back with ReadBin_Gauge.

Usage: python tests/golden/make_golden_smear.py OUTDIR
Writes OUTDIR/reference_smear.npz.
"""
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

PROBE = os.path.join(ROOT, "oracle", "_ref", "ref_probe")

CONFIGS = [  # name, dims, beta, seed, oracle sweeps (1 HB + 1 OR each), cases (None: all)
    ("s4448", (4, 4, 4, 8), 6.0, 21, 3, None),
    ("s4646", (4, 6, 4, 6), 5.7, 22, 2, ("ape_space", "stout_space", "hyp_time")),
]
# (kind, probe arguments); the same names key the fixture arrays
CASES = [
    ("ape_space", ["0.2", "2", "10", "1e-10"]),
    ("ape_time", ["0.2", "1", "10", "1e-10"]),
    ("stout_space", ["0.1", "2"]),
    ("stout_time", ["0.15", "1"]),
    ("hyp_space", ["1", "10", "1e-10", "0.75", "0.6", "0.3"]),
    ("hyp_time", ["1", "6", "1e-10", "0.75", "0.6", "0.3"]),
    ("multihit_space", ["5"]),
]


def run(args, timeout=600):
    r = subprocess.run(args, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"{' '.join(args)} failed ({r.returncode}):\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
    return r.stdout


def main(out):
    os.makedirs(out, exist_ok=True)
    tmp = os.path.join(out, "tmp_smear")
    os.makedirs(tmp, exist_ok=True)
    arrays = {}
    for name, dims, beta, seed, nsw, only in CONFIGS:
        X = list(dims)
        U = O.hot(3, X, seed)
        O.sweeps(U, X, beta, 1, 1, nsw, seed=seed)
        f = os.path.join(tmp, f"{name}.bin")
        assert O.save_bin(U, X, beta, f) == 0
        arrays[f"{name}_U"] = U
        arrays[f"{name}_dims"] = np.array(dims)
        arrays[f"{name}_beta"] = np.array(beta)
        for kind, extra in CASES:
            if only and kind not in only:
                continue
            fo = os.path.join(tmp, f"{name}_{kind}.bin")
            run([PROBE, "smear", f, fo] + [str(d) for d in dims] + [repr(beta), kind] + extra)
            rc, Us, g, b = O.load_bin(3, X, fo)
            assert rc == 0 and g == X
            # only the smeared directions are stored (the others are the input's)
            arrays[f"{name}_{kind}"] = Us[:, :3] if kind.endswith("space") else Us[:, 3:]
            arrays[f"{name}_{kind}_args"] = np.array([float(v) for v in extra])
    np.savez_compressed(os.path.join(out, "reference_smear.npz"), **arrays)
    print("wrote", sorted(arrays))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "golden_out")
