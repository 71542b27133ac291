#!/usr/bin/env python
"""Benchmark of the SU(N) heatbath/overrelaxation sweep on B200.

Workload (one "step" = one sweep): SU(3) 32^4, beta = 6.0, Haar hot start,
FP32 links in 12-parameter even/odd SoA, 1 heatbath + 4 overrelaxation passes
per sweep, FP64 reunitarization every 10 sweeps.  One sweep is 20 V link
updates.  The metric is link-updates/s, whole job (all ranks).

Multi-GPU: independent lattices per rank ("replicas only": the path does not
shard), max-over-ranks device time.

--impl reference times the reference algorithm's CPU implementation (the
FP64 oracle port, all host threads) on a bounded sample of the same sweep.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DIMS = (32, 32, 32, 32)
BETA = 6.0
N = 3
SEED = 1234
REUNIT = 10
WORKLOAD = ("SU(3) 32^4 beta=6.0 Haar hot start, FP32 SOA12 even/odd links, 1 HB + 4 OR per sweep, "
            "FP64 reunitarization every 10 sweeps")
LINK_RECORD = {"SOA12_f32": 48, "SOA_f64": 144, "SOA_f32": 72}


def measured_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks_dist(x, world, device):
    """Max of a per-rank number over all ranks (the job time of weak-scaled
    replicas is the slowest rank's); identity for one rank."""
    if world == 1:
        return x
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_seed(rank):
    """Each rank advances its own independent lattice (replicas: the sweep
    of one lattice does not shard without a halo exchange)."""
    return SEED + rank


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_sample(nthreads=0, reps=1, lattice=None):
    """Oracle (FP64 C, OpenMP) on 1/8 of a sweep with the sweep's mix: one
    heatbath and four overrelaxation phases of (parity 0, mu 0) on the full
    lattice.  Returns (link-updates/s, threads, seconds)."""
    from oracle import oracle as O
    X = list(DIMS)
    U = lattice if lattice is not None else O.hot(N, X, SEED)
    V = O.volume(X)
    t0 = time.perf_counter()
    for _ in range(reps):
        O.update_phase(U, X, 0, 0, 0, BETA, O.RNG_PHILOX32, SEED, 0, nthreads=nthreads)
        for _ in range(4):
            O.update_phase(U, X, 0, 0, 1, BETA, nthreads=nthreads)
    dt = time.perf_counter() - t0
    threads = nthreads or (os.cpu_count() or 1)
    return reps * 5 * (V // 2) / dt, threads, dt


def lockstep(g, nsweeps, n_hb=1, n_or=4, flip=1e-3):
    """Plaquette error of the engine's sweeps against the FP64 oracle, in
    lockstep: before each sweep the oracle takes the engine's stored links,
    then both run the same sweep with the same Philox draws (24-bit uniforms
    for FP32 lattices), the oracle in FP64 arithmetic.  Per sweep: the signed
    difference of the mean plaquette (engine - oracle) and the number of
    links that differ by more than `flip`: where a heatbath accept/reject
    decision went the other way at the rounding boundary, the following
    overrelaxation passes of the sweep spread the difference over a region
    around that link.  g must have reunit_every = 0.
    The dynamics is chaotic, so only this one-sweep error is a precision
    figure; longer chains agree in distribution, not link by link."""
    import numpy as np
    from oracle import oracle as O
    from sun_b200 import PlaquetteCUB, Sweep
    X = list(g.dims)
    fp32 = g.prec == "f32"
    diffs, off = [], []
    for _ in range(nsweeps):
        U = g.Get()
        seed, hb, _sw = g.rng_state()
        Sweep(g, n_hb, n_or, 1)
        p = PlaquetteCUB(g).Run()
        O.sweeps(U, X, g.beta, n_hb, n_or, 1, mode=O.RNG_PHILOX32 if fp32 else O.RNG_PHILOX64, seed=seed, pass_=hb)
        po = O.plaquette(U, X)
        d = np.abs(g.Get() - U).reshape(U.shape[0] * 4, -1).max(axis=1)
        off.append(int((d > flip).sum()))
        diffs.append(0.5 * (p.real + p.imag) - 0.5 * (po[0] + po[1]))
        del U, d
    a = np.abs(diffs)
    return {"sweeps": nsweeps, "abs_diff_max": float(a.max()), "abs_diff_mean": float(a.mean()),
            "signed_diff_mean": float(np.mean(diffs)), "signed_diffs": [float(v) for v in diffs],
            "links_off_per_sweep": off, "flip_threshold": flip}


def lockstep_copy(g, nsweeps):
    """lockstep() on a copy of g (same links and RNG counters, no
    reunitarization inside the window); g itself is left as it was."""
    from sun_b200 import gauge
    c = gauge(g.ctx, N=g.N, dims=g.dims, beta=g.beta, atype=g.atype, evenodd=True, prec=g.prec, seed=g.seed,
              reunit_every=0)
    c.Copy(g)
    out = lockstep(c, nsweeps)
    c.Release()
    return out


def accuracy_report(ctx, g, stream):
    """Accuracy of the FP32 12-parameter sweep against the FP64 oracle:
    (1) max |U^dagger U - 1| of the benchmarked lattice after its sweeps
    (FP64 reunitarization every 10); (2) its plaquette against the oracle's
    plaquette of the same stored links (both evaluate in FP64); (3) one sweep
    from a Haar start in FP32 on the GPU and in FP64 by the oracle with the
    same Philox draws, then both plaquettes: their difference is what FP32
    storage and arithmetic cost over a sweep."""
    from oracle import oracle as O
    from sun_b200 import PlaquetteCUB, Sweep, gauge, unitarity_violation
    X = list(DIMS)
    stream.synchronize()
    out = {"unitarity_max": unitarity_violation(g)}
    p = PlaquetteCUB(g).Run()
    po = O.plaquette(g.Get(), X)
    out["plaquette"] = [p.real, p.imag]
    out["plaquette_vs_oracle_same_links"] = max(abs(p.real - po[0]), abs(p.imag - po[1]))
    g1 = gauge(ctx, N=N, dims=DIMS, beta=BETA, atype=1, evenodd=True, prec="f32", seed=SEED + 7,
               reunit_every=REUNIT)
    g1.Init(hot=True)
    U = g1.Get()
    Sweep(g1, 1, 4, 1)
    p1 = PlaquetteCUB(g1).Run()
    g1.Release()
    O.sweeps(U, X, BETA, 1, 4, 1, mode=O.RNG_PHILOX32, seed=SEED + 7)
    po1 = O.plaquette(U, X)
    out["one_sweep_from_haar"] = {"plaquette_f32_gpu": [p1.real, p1.imag], "plaquette_f64_oracle": [po1[0], po1[1]],
                                  "abs_diff": max(abs(p1.real - po1[0]), abs(p1.imag - po1[1])),
                                  "draws": "the same Philox stream (24-bit uniforms) on both sides"}
    # lockstep from the benchmarked (thermalized) configuration: a copy with
    # the same links and RNG counters, no reunitarization inside the window
    gl = gauge(ctx, N=N, dims=DIMS, beta=BETA, atype=1, evenodd=True, prec="f32", seed=SEED, reunit_every=0)
    gl.Copy(g)
    out["lockstep"] = lockstep(gl, 10)
    out["lockstep"]["from"] = "the benchmarked configuration after its sweeps (thermalized, beta = 6.0)"
    gl.Release()
    return out


def copy_roofline(torch, nbytes, reps=4):
    """The e2e ceiling: host<->device copy rate with an upload and a download
    of nbytes each in flight at once (pinned host memory, two streams), as the
    e2e pipeline runs them.  Returns GB/s per direction."""
    hs = [torch.empty(nbytes, dtype=torch.uint8, pin_memory=True) for _ in range(2)]
    ds = [torch.empty(nbytes, dtype=torch.uint8, device="cuda") for _ in range(2)]
    s_up, s_dn = torch.cuda.Stream(), torch.cuda.Stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    best = 0.0
    for _ in range(reps):
        torch.cuda.synchronize()
        ev[0].record(s_up)
        s_dn.wait_event(ev[0])
        with torch.cuda.stream(s_up):
            ds[0].copy_(hs[0], non_blocking=True)
        with torch.cuda.stream(s_dn):
            hs[1].copy_(ds[1], non_blocking=True)
        ev[1].record(s_up)
        ev[2].record(s_dn)
        torch.cuda.synchronize()
        t = max(ev[0].elapsed_time(ev[1]), ev[0].elapsed_time(ev[2])) / 1e3
        best = max(best, nbytes / t / 1e9)
    return best


def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    from oracle import oracle as O
    O.build() if not os.path.exists(os.path.join(ROOT, "oracle", "libsun_oracle.so")) else None
    U = O.hot(N, list(DIMS), SEED)
    for _ in range(args.warmup):
        cpu_sample(lattice=U)
    rates, tot = [], 0.0
    for _ in range(args.steps):
        r, threads, dt = cpu_sample(lattice=U)
        rates.append(r)
        tot += dt
    V = O.volume(list(DIMS))
    value = args.steps * 5 * (V // 2) / tot
    line = {
        "metric": "link-updates/s", "value": value, "unit": "link-updates/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Haar hot start)", "impl": "reference",
        "config": {"workload": WORKLOAD, "lattice": list(DIMS), "parallelism": "replicas"},
        "cpu_baseline": {"value": value, "unit": "link-updates/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": "1/8 sweep per step: one heatbath + four overrelaxation phases (parity 0, mu 0) "
                                   "over the full 32^4 lattice, FP64 oracle, OpenMP over sites"},
        "e2e": {"value": value, "unit": "link-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    line["reference_gpu"] = reference_gpu_timing()
    print(json.dumps(line), flush=True)


def reference_gpu_timing(sweeps=20):
    """The reference's own build (oracle/_ref/ref_probe: the reference
    compiled from its sources for sm_100a) timed on this GPU through its
    public API -- HeatBath::Run + 4 x OverRelaxation::Run per sweep, its
    autotuner on, CUDA events -- on the benchmark lattice in the FP32
    12-parameter layout and in FP64 full links, with the SM clocks sampled
    meanwhile.  A report beside the CPU value, not the arm's value."""
    probe = os.path.join(ROOT, "oracle", "_ref", "ref_probe")
    if not os.path.exists(probe):
        return {"unavailable": "oracle/_ref/ref_probe not built (the reference sources were absent at build time)"}
    out = {"what": f"reference build, SU(3) {'x'.join(map(str, DIMS))} beta={BETA}, cold start, 3 untimed sweeps "
                   f"(autotuning), {sweeps} timed sweeps of 1 HB + 4 OR", "sweeps": sweeps}
    with tempfile.TemporaryDirectory() as tmp:
        env = dict(os.environ, SUN_REF_TUNE="1", CULQCD_RESOURCE_PATH=tmp)
        clocks = ClockSampler(0)
        clocks.start()
        for kind in ("f32soa12", "f64soa"):
            try:
                r = subprocess.run([probe, "timing"] + [str(d) for d in DIMS] + [repr(BETA), str(sweeps), kind],
                                   capture_output=True, text=True, timeout=600, env=env)
            except Exception as e:  # noqa: BLE001
                out[kind] = {"unavailable": f"{type(e).__name__}: {e}"}
                continue
            f = [l.split() for l in r.stdout.splitlines() if l.startswith("timing")]
            if r.returncode != 0 or not f:
                out[kind] = {"unavailable": f"rc={r.returncode}: {r.stderr.strip()[-200:]}"}
                continue
            v = dict(zip(f[0][1::2], (float(x) for x in f[0][2::2])))
            out[kind] = {"value": v["link_updates_per_s"], "unit": "link-updates/s", "sweep_ms": v["sweep_ms"],
                         "hb_ms_per_pass": v["hb_ms_per_pass"], "or_ms_per_pass": v["or_ms_per_pass"]}
        out["clocks"] = clocks.stop()
    return out


def e2e_pipeline(torch, L, ctx, g0, host0, steps, barrier, max_over_ranks):
    """Host-resident lattices streamed through the GPU by the C ABI: step k
    uploads lattice k % 4 from its pinned host image, sweeps it once and
    downloads it back; uploads, sweeps and downloads run on three streams
    ordered by events (a slot is re-uploaded only after its last download
    finished).  Returns (steps, seconds)."""
    from sun_b200 import gauge
    from sun_b200._native import check
    nslot = 4
    lats, hosts = [g0], [host0]
    for i in range(1, nslot):
        gi = gauge(ctx, N=N, dims=DIMS, beta=BETA, atype=1, evenodd=True, prec="f32", seed=SEED + 1000 * i,
                   reunit_every=REUNIT)
        gi.Init(hot=True)
        hi = torch.empty(host0.numel(), dtype=torch.uint8, pin_memory=True)
        check(L.sun_lattice_download(gi.h, C.c_void_p(hi.data_ptr()), 1, None), ctx.h)
        lats.append(gi)
        hosts.append(hi)
    check(L.sun_lattice_download(g0.h, C.c_void_p(host0.data_ptr()), 1, None), ctx.h)
    s_up, s_cmp, s_dn = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    p_up, p_cmp, p_dn = (C.c_void_p(s.cuda_stream) for s in (s_up, s_cmp, s_dn))
    ev_up = [torch.cuda.Event() for _ in range(nslot)]
    ev_cmp = [torch.cuda.Event() for _ in range(nslot)]
    ev_dn = [torch.cuda.Event() for _ in range(nslot)]
    for e in ev_dn:
        e.record(s_dn)

    def step(k):
        i = k % nslot
        s_up.wait_event(ev_dn[i])
        check(L.sun_lattice_upload_async(lats[i].h, C.c_void_p(hosts[i].data_ptr()), p_up), ctx.h)
        ev_up[i].record(s_up)
        s_cmp.wait_event(ev_up[i])
        check(L.sun_sweep(lats[i].h, 1, 4, 1, p_cmp), ctx.h)
        ev_cmp[i].record(s_cmp)
        s_dn.wait_event(ev_cmp[i])
        check(L.sun_lattice_download_async(lats[i].h, C.c_void_p(hosts[i].data_ptr()), p_dn), ctx.h)
        ev_dn[i].record(s_dn)

    for k in range(2 * nslot):  # warm-up
        step(k)
    torch.cuda.synchronize()
    barrier()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(s_up)
    for k in range(steps):
        step(k)
    s_dn.wait_stream(s_up)
    s_dn.wait_stream(s_cmp)
    t1.record(s_dn)
    torch.cuda.synchronize()
    barrier()
    t = max_over_ranks(t0.elapsed_time(t1) / 1e3)
    for gi in lats[1:]:
        gi.Release()
    return steps, t


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-extras", action="store_true", help="skip the FP64 and batched side measurements")
    ap.add_argument("--profile-case", default=None,
                    help="run one short workload for a profiler and exit: suN_L (SU(N), L^4, FP32 links, hot "
                         "start, one sweep of 1 HB + 4 OR), e.g. su6_20, or small8 (SU(3) 8^4 FP64, three sweeps)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_case:
        return profile_case(args.profile_case)

    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from sun_b200 import Context, gauge
    from sun_b200._native import check, lib
    L = lib()

    ctx = Context(local)
    stream = torch.cuda.Stream()
    sp = C.c_void_p(stream.cuda_stream)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def max_over_ranks(x):
        return max_over_ranks_dist(x, world, "cuda")

    V = DIMS[0] * DIMS[1] * DIMS[2] * DIMS[3]
    g = gauge(ctx, N=N, dims=DIMS, beta=BETA, atype=1, evenodd=True, prec="f32", seed=replica_seed(rank),
              reunit_every=REUNIT)
    g.Init(hot=True)

    def sweeps(lat, n):
        check(L.sun_sweep(lat.h, 1, 4, n, sp), ctx.h)

    # warm-up
    sweeps(g, args.warmup)
    stream.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sweeps(g, args.steps)
    e1.record(stream)
    stream.synchronize()
    torch.cuda.synchronize()
    barrier()
    t_main = max_over_ranks(e0.elapsed_time(e1) / 1e3)

    # dominant kernel: the overrelaxation phase launch (32 of the 40 update
    # launches of a sweep); 8 launches per pass
    n_or = 10
    e0.record(stream)
    check(L.sun_overrelax(g.h, n_or, sp), ctx.h)
    e1.record(stream)
    stream.synchronize()
    t_or = e0.elapsed_time(e1) / 1e3 / (8 * n_or)
    n_hbp = 4
    e0.record(stream)
    check(L.sun_heatbath(g.h, n_hbp, sp), ctx.h)
    e1.record(stream)
    stream.synchronize()
    t_hb = e0.elapsed_time(e1) / 1e3 / (8 * n_hbp)
    # the spread of single sweeps: p50 / p99 over repeats, each sweep
    # bracketed by its own events
    n_rep = 20
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(n_rep + 1)]
    evs[0].record(stream)
    for i in range(n_rep):
        sweeps(g, 1)
        evs[i + 1].record(stream)
    stream.synchronize()
    per_sweep = sorted(evs[i].elapsed_time(evs[i + 1]) for i in range(n_rep))
    clk = clocks.stop()
    accuracy = None
    if rank == 0 and not args.no_cpu:
        # the accuracy report on the configuration after 500 sweeps (the
        # length of the FP32-against-FP64 run of the 32^4 configuration),
        # besides the 10 overrelaxation and 4 heatbath passes timed above
        done = args.warmup + args.steps + n_rep
        if done < 500:
            sweeps(g, 500 - done)
        accuracy = accuracy_report(ctx, g, stream)
        accuracy["sweeps_before"] = max(500, done)

    # end to end through the C ABI with host buffers.  Serial form: upload the
    # image from pinned memory, one sweep, plaquette to the host, download.
    img_bytes = g.Bytes()
    host = torch.empty(img_bytes, dtype=torch.uint8, pin_memory=True)
    check(L.sun_lattice_download(g.h, C.c_void_p(host.data_ptr()), 1, sp), ctx.h)
    plq = (C.c_double * 2)()
    k_ser = max(3, min(args.steps, 10))
    for _ in range(2):
        check(L.sun_lattice_upload(g.h, C.c_void_p(host.data_ptr()), 1, sp), ctx.h)
        sweeps(g, 1)
        check(L.sun_plaquette(g.h, plq, sp), ctx.h)
        check(L.sun_lattice_download(g.h, C.c_void_p(host.data_ptr()), 1, sp), ctx.h)
    barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(k_ser):
        check(L.sun_lattice_upload(g.h, C.c_void_p(host.data_ptr()), 1, sp), ctx.h)
        sweeps(g, 1)
        check(L.sun_plaquette(g.h, plq, sp), ctx.h)
        check(L.sun_lattice_download(g.h, C.c_void_p(host.data_ptr()), 1, sp), ctx.h)
    e1.record(stream)
    stream.synchronize()
    barrier()
    t_ser = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    # Pipelined form (the headline e2e): host-resident lattices streamed
    # through the GPU.  Step k takes lattice k % 4: its image is uploaded from
    # pinned host memory (the result its previous step downloaded), swept once
    # and downloaded again, on three streams ordered by events, so one
    # lattice's upload and another's download overlap a third's sweep.
    k_e2e, t_e2e = e2e_pipeline(torch, L, ctx, g, host, max(8, min(3 * args.steps, 32)), barrier, max_over_ranks)
    copy_gbs = copy_roofline(torch, int(g.Bytes()))

    extras = {}
    if not args.no_extras:
        # plain single-lattice FP64 full-link sweep (the denominator of the
        # batched-vs-plain target)
        g64 = gauge(ctx, N=N, dims=DIMS, beta=BETA, atype=0, evenodd=True, prec="f64", seed=SEED,
                    reunit_every=REUNIT)
        g64.Init(hot=True)
        sweeps(g64, 3)
        k64 = max(3, args.steps // 3)
        stream.synchronize()
        e0.record(stream)
        sweeps(g64, k64)
        e1.record(stream)
        stream.synchronize()
        t64 = e0.elapsed_time(e1) / 1e3
        extras["fp64_soa_plain"] = {"value": 20 * V * k64 / t64, "unit": "link-updates/s", "sweeps": k64,
                                    "hbm_gbs_model": 20 * V * k64 * 9 * 144 / t64 / 1e9}
        g64.Release()
        extras["batched"] = batched_bench(ctx, L, sp, stream, args, accuracy=rank == 0 and not args.no_cpu)
        extras["plain_small_fp64"] = plain_small_bench(ctx, L, sp, stream)
        extras["sun_n"] = sun_n_bench(ctx, L, sp, stream, accuracy=rank == 0 and not args.no_cpu)
        extras["smearing"] = smear_bench(ctx, L, sp, stream)
        if rank == 0:
            extras["serving"] = serving_bench(ctx)
            # the same job mix at a rate the GPU keeps up with: latency is then
            # service time (jobs overlapping on the device), not queueing
            light = serving_bench(ctx, rate=2.0, window=6.0)
            extras["serving"]["light_load"] = {k: light[k] for k in ("jobs", "completed", "arrival_rate_per_s",
                                                                      "window_s", "p50_latency_s", "p99_latency_s",
                                                                      "link_updates_per_s", "wall_s")}
            if not args.no_cpu:
                extras["serving"]["accuracy"] = serving_accuracy(ctx)

    line = {
        "metric": "link-updates/s",
        "value": world * 20 * V * args.steps / t_main,
        "unit": "link-updates/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * t_main / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded Haar hot start, Philox stream)",
        "config": {"workload": WORKLOAD, "lattice": list(DIMS), "ncolors": N, "beta": BETA, "layout": "SOA12",
                   "precision": "f32", "order": "even/odd", "sweep": "1 HB + 4 OR", "reunit_every": REUNIT,
                   "step": "one sweep = 20 V link updates",
                   "l2": "inputs larger than L2 (201 MB link image vs 126 MB L2)", "parallelism": "replicas"},
        "gpu_launches": args.steps * 42,
        "clocks": clk,
        "sweep_ms": {"p50": per_sweep[n_rep // 2], "p99": per_sweep[-1], "min": per_sweep[0], "repeats": n_rep,
                     "how": "single sweeps after the timed region, CUDA events around each"},
    }
    peak, peak_kind = measured_hbm()
    bytes_or = (V // 2) * 9 * LINK_RECORD["SOA12_f32"]
    ach = bytes_or / t_or / 1e9
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "k_update_or_f32_soa12_32x4.json")) as f:
            traffic = json.load(f).get("dram_bytes_per_launch")
    except Exception:
        pass
    line["roofline"] = {"bound": "hbm", "kernel": "k_update<3,float,SOA12,OR>", "achieved": ach, "peak": peak,
                        "unit": "GB/s", "frac": ach / peak, "traffic": traffic, "peak_kind": peak_kind,
                        "launch_us": t_or * 1e6, "algorithmic_bytes_per_launch": bytes_or,
                        "hb_launch_us": t_hb * 1e6, "hb_achieved_gbs": bytes_or / t_hb / 1e9}
    # the reference's own, larger byte model beside the compulsory one: 20
    # link-records of 12 FP32 reals per update (OverRelaxation::bytes,
    # src/monte/ovr.cu:254-259; the heatbath adds two 48 B cuRAND states,
    # monte.cu:258-262, which a Philox stream does not have)
    bytes_ref = (V // 2) * 20 * 12 * 4
    line["roofline"]["reference_model"] = {
        "bytes_per_update": 20 * 12 * 4, "achieved": bytes_ref / t_or / 1e9, "unit": "GB/s",
        "frac": bytes_ref / t_or / 1e9 / peak,
        "note": "20 link-records per update counted as if every staple load came from DRAM; the compulsory model "
                "above (9 records) is the roofline"}
    line["e2e"] = {"value": world * 20 * V * k_e2e / t_e2e, "unit": "link-updates/s",
                   "h2d_bytes_per_step": img_bytes, "d2h_bytes_per_step": img_bytes,
                   "step": "four host-resident lattices in rotation: upload image (pinned) + 1 sweep + download "
                           "image, C ABI, copies on their own streams overlapping the sweeps",
                   "steps": k_e2e,
                   "roofline": {"bound": "host-device copies", "unit": "GB/s per direction",
                                "achieved": img_bytes * k_e2e / t_e2e / 1e9, "peak": copy_gbs,
                                "frac": img_bytes * k_e2e / t_e2e / 1e9 / copy_gbs,
                                "peak_how": "one upload and one download of the image in flight at once, pinned "
                                            "host memory, best of 4"},
                   "serial": {"value": world * 20 * V * k_ser / t_ser, "unit": "link-updates/s",
                              "h2d_bytes_per_step": img_bytes, "d2h_bytes_per_step": img_bytes + 16,
                              "step": "upload image + 1 sweep + plaquette + download image, one stream"}}
    if accuracy is not None:
        line["accuracy"] = accuracy
    line.update(extras)
    if rank == 0 and world == 1 and not args.no_cpu:
        # about 10 s of CPU work: repeat the 1/8-sweep sample on one lattice
        from oracle import oracle as O
        U = O.hot(N, list(DIMS), SEED)
        _, _, dt1 = cpu_sample(lattice=U)
        reps = max(1, min(60, int(10.0 / max(dt1, 1e-3))))
        rate, threads, dt = cpu_sample(reps=reps, lattice=U)
        line["cpu_baseline"] = {"value": rate, "unit": "link-updates/s", "cores": threads, "kind": "port",
                                "sample": f"{reps} x 1/8 sweep (one heatbath + four overrelaxation phases, parity 0 "
                                          f"mu 0) of the 32^4 lattice, FP64 oracle, {dt:.1f} s"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    g.Release()
    ctx.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def profile_case(case):
    """A short workload for a profiler (ncu): "suN_L" SU(N) on L^4, FP32
    links (the benchmark's 12-parameter layout for SU(3), full links
    otherwise), hot start, one sweep of 1 heatbath + 4 overrelaxation passes
    (8 heatbath then 32 overrelaxation update launches); "small8" the plain
    small case (SU(3) 8^4 FP64 full links, cold start), three such sweeps."""
    import torch
    from sun_b200 import Context, Sweep, gauge
    if case == "small8":
        with Context(0) as ctx:
            g = gauge(ctx, N=3, dims=(8, 8, 8, 8), beta=6.0, atype=0, evenodd=True, prec="f64", seed=SEED)
            g.Init(hot=False)
            Sweep(g, 1, 4, 3)
            torch.cuda.synchronize()
            g.Release()
        print(f"profile case {case}: three sweeps done", flush=True)
        return
    n, l = case[2:].split("_")
    with Context(0) as ctx:
        g = gauge(ctx, N=int(n), dims=(int(l),) * 4, beta={2: 2.5, 3: 6.0, 4: 11.1, 6: 25.0}[int(n)],
                  atype=1 if int(n) == 3 else 0, evenodd=True, prec="f32", seed=SEED)
        g.Init(hot=True)
        Sweep(g, 1, 4, 1)
        torch.cuda.synchronize()
        g.Release()
    print(f"profile case {case}: one sweep done", flush=True)


def serving_jobs(rate=50.0, window=4.0, seed=1234):
    """Poisson arrivals (mean `rate` per second over `window` seconds) of jobs
    with N in {2,3,4}, L^3 x T with L in {8..24} even and T in {L, 2L}, beta
    uniform in a confined-phase range per N, 50..500 sweeps of 1 HB + 4 OR and
    a random non-empty subset of {plaquette, Polyakov loop, Wilson loops up
    to 4x4}; FP32 links (12-parameter for SU(3))."""
    import numpy as np
    rng = np.random.default_rng(seed)
    beta_range = {2: (2.0, 2.3), 3: (5.7, 5.9), 4: (10.2, 10.6)}
    t, jobs = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > window:
            return jobs
        n = int(rng.choice([2, 3, 4]))
        l = int(rng.choice(np.arange(8, 25, 2)))
        tt = int(rng.choice([l, 2 * l]))
        obs = int(rng.integers(1, 8))
        jobs.append(dict(t=t, N=n, dims=(l, l, l, tt), beta=float(rng.uniform(*beta_range[n])),
                         sweeps=int(rng.integers(50, 501)), seed=int(rng.integers(1, 2 ** 62)), observables=obs,
                         R=4 if obs & 4 else 0, T=4 if obs & 4 else 0))


def serving_bench(ctx, rate=50.0, window=3.0, max_active=256):
    """Continuous-batching server under the Poisson stream: jobs are submitted
    at their arrival times while earlier ones run; p50/p99 latency (submit to
    result) and aggregate link-updates/s over the run."""
    import numpy as np
    from sun_b200 import SOA, SOA12, Server, make_job
    jobs = serving_jobs(rate, window)
    srv = Server(ctx, max_active=max_active)
    t0 = time.perf_counter()
    pending, results, nxt = list(jobs), [], 0
    while len(results) < len(jobs):
        now = time.perf_counter() - t0
        while nxt < len(pending) and pending[nxt]["t"] <= now:
            j = pending[nxt]
            srv.submit(make_job(N=j["N"], dims=j["dims"], beta=j["beta"], sweeps=j["sweeps"], seed=j["seed"],
                                observables=j["observables"], R=j["R"], T=j["T"], prec="f32",
                                layout=SOA12 if j["N"] == 3 else SOA, reunit_every=10))
            nxt += 1
        done = srv.step()
        results += done
        if not done and srv.pending() == (0, 0) and nxt < len(pending):
            time.sleep(max(0.0, min(0.01, pending[nxt]["t"] - (time.perf_counter() - t0))))
    wall = time.perf_counter() - t0
    steps = srv.stats()
    srv.close()
    ok = [r for r in results if r["status"] == 0]
    lat = np.array([r["finish_s"] - r["submit_s"] for r in ok])
    upd = sum(r["link_updates"] for r in ok)
    out = {"jobs": len(jobs), "completed": len(ok), "arrival_rate_per_s": rate, "window_s": window,
           "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
           "link_updates_per_s": upd / wall, "wall_s": wall, "max_active": max_active,
           "steps": {k: (round(v, 4) if isinstance(v, float) else v) for k, v in steps.items()},
           "gpu_busy_frac": steps["sweep_gpu_s"] / wall}
    if len(ok) == len(jobs):
        # compulsory bytes: 9 link-records per update (48 B SU(3) 12-parameter,
        # 8 N^2 B full FP32 links)
        byts = sum(20 * int(np.prod(j["dims"])) * j["sweeps"] * 9 * (48 if j["N"] == 3 else 8 * j["N"] ** 2)
                   for j in jobs)
        peak, _ = measured_hbm()
        out["hbm_gbs_model"] = byts / wall / 1e9
        out["hbm_frac"] = byts / wall / 1e9 / peak
    return out


def serving_accuracy(ctx):
    """Plaquette error against the FP64 oracle of one served job per N: the
    first job of each N in the stream is run alone (a job's result does not
    depend on its batch mates), then one lockstep sweep from its final
    configuration."""
    from sun_b200 import SOA, SOA12, Sweep, gauge
    out = {}
    for j in serving_jobs():
        key = f"su{j['N']}"
        if key in out:
            continue
        g = gauge(ctx, N=j["N"], dims=j["dims"], beta=j["beta"], atype=SOA12 if j["N"] == 3 else SOA,
                  evenodd=True, prec="f32", seed=j["seed"], reunit_every=10)
        g.Init(hot=True)
        Sweep(g, 1, 4, j["sweeps"])
        r = lockstep_copy(g, 1)
        out[key] = {"dims": list(j["dims"]), "sweeps": j["sweeps"], "abs_diff": r["abs_diff_max"],
                    "links_off_by_1e-3": r["links_off_per_sweep"][0]}
        g.Release()
    return out


def batched_bench(ctx, L, sp, stream, args, accuracy=False):
    """64 independent SU(3) lattices, L in {8,12,16}, T in {L,2L}, beta in
    [5.7,6.4], FP32 SOA12, advanced together from a captured CUDA graph."""
    import numpy as np
    import torch
    from sun_b200 import Batch, gauge
    from sun_b200._native import check
    rng = np.random.default_rng(1234)
    lats, vol = [], 0
    b = Batch(ctx)
    for i in range(64):
        l = int(rng.choice([8, 12, 16]))
        t = int(rng.choice([l, 2 * l]))
        beta = float(rng.uniform(5.7, 6.4))
        g = gauge(ctx, N=3, dims=(l, l, l, t), beta=beta, atype=1, evenodd=True, prec="f32", seed=1234 + 7919 * i,
                  reunit_every=10)
        g.Init(hot=True)
        b.add(g)
        lats.append(g)
        vol += l ** 3 * t
    check(L.sun_batch_sweep(b.h, 1, 4, 3, 1, sp), ctx.h)
    k = max(5, args.steps)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stream.synchronize()
    e0.record(stream)
    check(L.sun_batch_sweep(b.h, 1, 4, k, 1, sp), ctx.h)
    e1.record(stream)
    stream.synchronize()
    t = e0.elapsed_time(e1) / 1e3
    rate = 20 * vol * k / t
    out = {"value": rate, "unit": "link-updates/s", "lattices": 64, "total_sites": vol, "sweeps": k,
           "hbm_gbs_model": rate * 9 * 48 / 1e9, "graph": True}
    if accuracy:
        # plaquette error against the FP64 oracle, one lockstep sweep from the
        # final configuration of three of the lattices
        out["accuracy"] = []
        for i in (0, 21, 42):
            r = lockstep_copy(lats[i], 1)
            out["accuracy"].append({"lattice": i, "dims": list(lats[i].dims), "abs_diff": r["abs_diff_max"],
                                    "links_off_by_1e-3": r["links_off_per_sweep"][0]})
    b.close()
    for g in lats:
        g.Release()
    return out


def plain_small_bench(ctx, L, sp, stream, sweeps=200):
    """The plain small case: SU(3) 8^4, beta = 6.0, cold start, FP64 full
    links, even/odd, `sweeps` sweeps of 1 HB + 4 OR with the plaquette and the
    Polyakov loop read back to the host after every sweep (the reference's
    PlaquetteCUB / OnePolyakovLoop return host values).  The events bracket
    the whole loop, host round trips included."""
    import torch
    from sun_b200 import gauge
    from sun_b200._native import check
    dims = (8, 8, 8, 8)
    V = 8 ** 4
    g = gauge(ctx, N=3, dims=dims, beta=6.0, atype=0, evenodd=True, prec="f64", seed=SEED)
    g.Init(hot=False)
    pl, po = (C.c_double * 2)(), (C.c_double * 2)()

    def one():
        check(L.sun_sweep(g.h, 1, 4, 1, sp), ctx.h)
        check(L.sun_plaquette(g.h, pl, sp), ctx.h)
        check(L.sun_polyakov(g.h, po, sp), ctx.h)

    for _ in range(3):
        one()
    g.Init(hot=False)
    stream.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(sweeps):
        one()
    e1.record(stream)
    stream.synchronize()
    t = e0.elapsed_time(e1) / 1e3
    out = {"value": 20 * V * sweeps / t, "unit": "link-updates/s", "sweeps": sweeps, "ms_per_sweep": 1e3 * t / sweeps,
           "lattice": list(dims), "precision": "f64", "layout": "SOA", "start": "cold",
           "final_plaquette": [pl[0], pl[1]], "final_polyakov": [po[0], po[1]],
           "measure": "plaquette + Polyakov loop to the host every sweep"}
    # the same sweeps and per-sweep measurements in one call
    # (sun_sweep_measure: one captured graph of sweep + plaquette + Polyakov
    # loop replayed back to back, the observables copied once at the end)
    import numpy as np
    pp, pq = np.zeros(2 * sweeps), np.zeros(2 * sweeps)
    dp = C.POINTER(C.c_double)
    check(L.sun_sweep_measure(g.h, 1, 4, 3, pp.ctypes.data_as(dp), pq.ctypes.data_as(dp), sp), ctx.h)
    g.Init(hot=False)
    stream.synchronize()
    e0.record(stream)
    check(L.sun_sweep_measure(g.h, 1, 4, sweeps, pp.ctypes.data_as(dp), pq.ctypes.data_as(dp), sp), ctx.h)
    e1.record(stream)
    stream.synchronize()
    t1 = e0.elapsed_time(e1) / 1e3
    out["one_call"] = {"value": 20 * V * sweeps / t1, "ms_per_sweep": 1e3 * t1 / sweeps,
                       "final_plaquette": [pp[-2], pp[-1]], "final_polyakov": [pq[-2], pq[-1]],
                       "same_as_per_sweep_calls": bool(pp[-2] == pl[0] and pp[-1] == pl[1] and pq[-2] == po[0])}
    g.Release()
    return out


def sun_n_bench(ctx, L, sp, stream, sweeps=300, accuracy=False):
    """SU(N), N in {2, 4, 6}, on 24^4 with beta/(2 N^2) fixed (2.5, 11.1,
    25.0): FP32 full links, FP64 compensated reductions, hot start; `sweeps`
    timed sweeps of 1 HB + 4 OR (reunitarization every 10) after 2 warm-up
    sweeps, then the plaquette and Wilson loops R x T <= 4 x 4 of the final
    configuration."""
    import torch
    from sun_b200 import WilsonLoop, gauge
    from sun_b200._native import check
    peak, _ = measured_hbm()
    dims = (24, 24, 24, 24)
    V = 24 ** 4
    out = {}
    for n, beta in ((2, 2.5), (4, 11.1), (6, 25.0)):
        g = gauge(ctx, N=n, dims=dims, beta=beta, atype=0, evenodd=True, prec="f32", seed=SEED + n, reunit_every=10)
        g.Init(hot=True)
        check(L.sun_sweep(g.h, 1, 4, 2, sp), ctx.h)
        stream.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        check(L.sun_sweep(g.h, 1, 4, sweeps, sp), ctx.h)
        e1.record(stream)
        stream.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        rate = 20 * V * sweeps / t
        pl = (C.c_double * 2)()
        check(L.sun_plaquette(g.h, pl, sp), ctx.h)
        w = WilsonLoop(g, 4, 4)
        out[f"su{n}"] = {"value": rate, "unit": "link-updates/s", "beta": beta, "sweeps": sweeps,
                         "hbm_frac": rate * 9 * 8 * n * n / 1e9 / peak, "plaquette": [pl[0], pl[1]],
                         "wilson_4x4_re": [[round(float(v), 8) for v in row] for row in w.real]}
        if accuracy:
            r = lockstep_copy(g, 1)
            out[f"su{n}"]["accuracy"] = {"abs_diff": r["abs_diff_max"],
                                         "links_off_by_1e-3": r["links_off_per_sweep"][0],
                                         "how": "one lockstep sweep from the final configuration against the "
                                                "FP64 oracle"}
        g.Release()
    out["lattice"] = list(dims)
    out["bytes_per_update"] = "9 link-records of 8 N^2 B (FP32 full links)"
    return out


def smear_bench(ctx, L, sp, stream):
    """Smearing on SU(3) 24^4 (the step before Wilson loops): per layout, ms
    per step of APE in space (w 0.2, 10 hits), stout in space (w 0.1), HYP
    in space (alpha 0.75/0.6/0.3, 10 hits, tol 1e-10), the heatbath
    multihit of the temporal links and the overrelaxation multihit of the
    spatial links (10 hits each), each after one untimed call.  FP64 full
    links in lexicographic order are the reference's smearing layout; FP32
    12-parameter even/odd is the sweep's."""
    import torch
    from sun_b200 import gauge
    from sun_b200._native import check
    dims = (24, 24, 24, 24)
    out = {"lattice": list(dims)}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    alpha = (C.c_double * 3)(0.75, 0.6, 0.3)

    def timed(f, steps):
        f(1)
        stream.synchronize()
        e0.record(stream)
        f(steps)
        e1.record(stream)
        stream.synchronize()
        return e0.elapsed_time(e1) / steps

    for name, lay, eo, prec in (("f64_soa_lex", 0, False, "f64"), ("f32_soa12_eo", 1, True, "f32")):
        g = gauge(ctx, N=3, dims=dims, beta=6.0, atype=lay, evenodd=eo, prec=prec, seed=SEED)
        g.Init(hot=True)
        o = gauge(ctx, N=3, dims=dims, beta=6.0, atype=0, evenodd=eo, prec=prec, seed=SEED)
        r = {}
        r["ape_ms_per_step"] = timed(lambda n: check(L.sun_smear_ape(g.h, 0.2, n, 10, 1e-10, 7, sp), ctx.h), 3)
        r["stout_ms_per_step"] = timed(lambda n: check(L.sun_smear_stout(g.h, 0.1, n, 7, sp), ctx.h), 3)
        r["hyp_ms_per_step"] = timed(lambda n: check(L.sun_smear_hyp(g.h, alpha, n, 10, 1e-10, 7, sp), ctx.h), 1)
        r["multihit_ms"] = timed(lambda n: [check(L.sun_multihit(g.h, o.h, 10, 99, sp), ctx.h) for _ in range(n)], 2)
        r["multihit_space_ms"] = timed(lambda n: [check(L.sun_multihit_space(g.h, o.h, 10, sp), ctx.h)
                                                  for _ in range(n)], 2)
        out[name] = r
        o.Release()
        g.Release()
    return out


if __name__ == "__main__":
    main()
