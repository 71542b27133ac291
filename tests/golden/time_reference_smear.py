#!/usr/bin/env python
"""Time the reference's own smearing on one GPU.

Runs oracle/_ref/ref_probe (the reference built by `make -C oracle/ref`) on
an SU(3) 24^4 FP64 configuration (seeded hot start written by the oracle in
the reference's file format).  Each case is one call of the reference's
smearing API on a normal-order SOA copy; the probe prints the call's duration
(CUDA events, the reference's per-step array copies included).  Parameters
match bench.py's smearing measurement.

Usage: python tests/golden/time_reference_smear.py OUTFILE
"""
import json
import os
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

PROBE = os.path.join(ROOT, "oracle", "_ref", "ref_probe")
DIMS = [24, 24, 24, 24]
CASES = [  # kind, probe arguments, steps (calls are per step, or per call for multihit)
    ("ape_space", ["0.2", "3", "10", "1e-10"], 3),
    ("stout_space", ["0.1", "3"], 3),
    ("hyp_space", ["1", "10", "1e-10", "0.75", "0.6", "0.3"], 1),
    ("multihit_space", ["10"], 1),
]


def main(out):
    res = {"lattice": DIMS, "precision": "f64", "layout": "SOA, lexicographic order", "probe": "oracle/_ref/ref_probe smear"}
    with tempfile.TemporaryDirectory() as tmp:
        f = os.path.join(tmp, "in.bin")
        U = O.hot(3, DIMS, 1234)
        assert O.save_bin(U, DIMS, 6.0, f) == 0
        for kind, args, steps in CASES:
            fo = os.path.join(tmp, "out.bin")
            r = subprocess.run([PROBE, "smear", f, fo] + [str(d) for d in DIMS] + ["6.0", kind] + args,
                               capture_output=True, text=True, timeout=3600)
            ms = [float(l.split()[1]) for l in r.stdout.splitlines() if l.startswith("smear_ms")]
            if r.returncode != 0 or not ms:
                res[kind] = f"failed rc={r.returncode}: {r.stderr[-300:]}"
                continue
            res[kind] = {"args": args, "ms_total": ms[0], "ms_per_step": ms[0] / steps}
    with open(out, "w") as fh:
        json.dump(res, fh, indent=1)
    print(json.dumps(res, indent=1))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join("golden_out", "reference_timings_smear.json"))
