#!/usr/bin/env python
"""Time the reference's own build for SU(4) and SU(6) on one GPU.

Runs the probes built by `make -C oracle/ref ncolors` (the reference compiled
with NCOLORS = 4 and 6) on a 24^4 lattice: its autotuner on, 3 warm-up
sweeps, then 20 timed sweeps of 1 HeatBath + 4 OverRelaxation passes on FP32
links (the reference stores SU(N > 3) links as full SOA matrices).  The
probes print their own CUDA-event timings; this script collects them.

Usage: python tests/golden/time_reference_sun.py OUTFILE
"""
import json
import os
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
CASES = [(4, 11.1), (6, 25.0)]  # beta / (2 N^2) fixed, as the engine's SU(N) measurement


def main(out):
    res = {"lattice": [24, 24, 24, 24], "sweep": "1 HeatBath + 4 OverRelaxation, FP32", "autotuner": "on",
           "timed_sweeps": 20, "probe": "oracle/_ref_n{N}/ref_probe timing"}
    with tempfile.TemporaryDirectory() as tmp:
        env = dict(os.environ, SUN_REF_TUNE="1", CULQCD_RESOURCE_PATH=tmp)
        for n, beta in CASES:
            probe = os.path.join(ROOT, "oracle", f"_ref_n{n}", "ref_probe")
            r = subprocess.run([probe, "timing", "24", "24", "24", "24", repr(beta), "20", "f32soa12"],
                               capture_output=True, text=True, timeout=1800, env=env)
            line = [l for l in r.stdout.splitlines() if l.startswith("timing")]
            if not line:
                res[f"su{n}"] = f"failed rc={r.returncode}: {r.stderr[-300:]}"
                continue
            p = line[0].split()
            vals = dict(zip(p[1::2], (float(v) for v in p[2::2])))
            res[f"su{n}"] = dict(beta=beta, **vals)
    with open(out, "w") as fh:
        json.dump(res, fh, indent=1)
    print(json.dumps(res, indent=1))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join("golden_out", "reference_timings_sun.json"))
