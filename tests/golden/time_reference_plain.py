#!/usr/bin/env python
"""Time the reference's own build on the plain small case.

SU(3) 8^4, beta = 6.0, FP64 full links, cold start, 200 sweeps of
1 HeatBath + 4 OverRelaxation with PlaquetteCUB and OnePolyakovLoop after
every sweep (their host values end each sweep), through
oracle/_ref/ref_probe (`plain` command, CUDA-event time of the loop, its
autotuner on).  bench.py's `plain_small_fp64` measures the engine on the same
case.

Usage: python tests/golden/time_reference_plain.py OUTFILE
"""
import json
import os
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
PROBE = os.path.join(ROOT, "oracle", "_ref", "ref_probe")
SWEEPS = 200


def main(out):
    with tempfile.TemporaryDirectory() as tmp:
        env = dict(os.environ, SUN_REF_TUNE="1", CULQCD_RESOURCE_PATH=tmp)
        r = subprocess.run([PROBE, "plain", "8", "8", "8", "8", "6.0", str(SWEEPS)], capture_output=True, text=True,
                           timeout=1200, env=env)
    line = [l for l in r.stdout.splitlines() if l.startswith("plain_ms")]
    if r.returncode != 0 or not line:
        res = {"failed": f"rc={r.returncode}: {r.stderr[-300:]}"}
    else:
        p = line[0].split()
        ms = float(p[1])
        res = {"lattice": [8, 8, 8, 8], "precision": "f64", "layout": "SOA even/odd", "start": "cold", "sweeps": SWEEPS,
               "ms_total": ms, "ms_per_sweep": ms / SWEEPS, "link_updates_per_s": 20 * 8 ** 4 * SWEEPS / (ms * 1e-3),
               "final_plaquette": [float(p[3]), float(p[4])], "final_polyakov": [float(p[6]), float(p[7])]}
    with open(out, "w") as fh:
        json.dump(res, fh, indent=1)
    print(json.dumps(res, indent=1))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join("golden_out", "reference_timings_plain.json"))
