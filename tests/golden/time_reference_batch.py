#!/usr/bin/env python
"""Time the reference's own build on the batched ensemble, its way.

The 64 SU(3) lattices of bench.py's batched measurement (the same seeded
draw: L in {8, 12, 16}, T in {L, 2L}, beta in [5.7, 6.4]), FP32 12-parameter
links, run one after another through oracle/_ref/ref_probe (`batch`
command): the reference has one process-global geometry (SETPARAMS), so it
advances one lattice at a time.  Per lattice: hot start, 3 untimed sweeps,
then SWEEPS timed sweeps of 1 HeatBath + 4 OverRelaxation with Reunitarize
every 10; the timed parts are summed (CUDA events, autotuner on).

Usage: python tests/golden/time_reference_batch.py OUTFILE
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
PROBE = os.path.join(ROOT, "oracle", "_ref", "ref_probe")
SWEEPS = 50


def shapes():
    rng = np.random.default_rng(1234)
    out = []
    for _ in range(64):
        l = int(rng.choice([8, 12, 16]))
        t = int(rng.choice([l, 2 * l]))
        beta = float(rng.uniform(5.7, 6.4))
        out.append((l, t, beta))
    return out


def main(out):
    with tempfile.TemporaryDirectory() as tmp:
        f = os.path.join(tmp, "shapes.txt")
        with open(f, "w") as fh:
            for l, t, beta in shapes():
                fh.write(f"{l} {t} {beta!r}\n")
        env = dict(os.environ, SUN_REF_TUNE="1", CULQCD_RESOURCE_PATH=tmp)
        r = subprocess.run([PROBE, "batch", f, str(SWEEPS)], capture_output=True, text=True, timeout=1800, env=env)
    line = [l for l in r.stdout.splitlines() if l.startswith("batch_ms")]
    if r.returncode != 0 or not line:
        res = {"failed": f"rc={r.returncode}: {r.stderr[-300:]}"}
    else:
        p = line[0].split()
        ms, upd = float(p[1]), float(p[3])
        res = {"lattices": 64, "sweeps_each": SWEEPS, "precision": "f32", "layout": "SOA12 even/odd",
               "total_sites": sum(l ** 3 * t for l, t, _ in shapes()), "ms_total": ms,
               "link_updates_per_s": upd / (ms * 1e-3)}
    with open(out, "w") as fh:
        json.dump(res, fh, indent=1)
    print(json.dumps(res, indent=1))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join("golden_out", "reference_timings_batch.json"))
