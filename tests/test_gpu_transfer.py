"""Asynchronous raw-image transfers (sun_lattice_upload_async /
sun_lattice_download_async): they agree with the synchronous entry points,
and a three-stream pipeline of uploads, sweeps and downloads ordered by
events gives the same lattices as running the same steps one after another."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lat(ctx, seed, dims=(4, 4, 4, 8)):
    from sun_b200 import gauge
    g = gauge(ctx, N=3, dims=dims, beta=6.0, atype=1, evenodd=True, prec="f32", seed=seed, reunit_every=2)
    g.Init(hot=True)
    return g


def test_async_roundtrip(ctx):
    import torch
    from sun_b200._native import check, lib
    L = lib()
    g = _lat(ctx, 5)
    n = g.Bytes()
    src = torch.empty(n, dtype=torch.uint8, pin_memory=True)
    dst = torch.zeros(n, dtype=torch.uint8, pin_memory=True)
    check(L.sun_lattice_download(g.h, C.c_void_p(src.data_ptr()), 1, None), ctx.h)
    ref = src.numpy().copy()
    s = torch.cuda.Stream()
    sp = C.c_void_p(s.cuda_stream)
    g2 = _lat(ctx, 6)
    check(L.sun_lattice_upload_async(g2.h, C.c_void_p(src.data_ptr()), sp), ctx.h)
    check(L.sun_lattice_download_async(g2.h, C.c_void_p(dst.data_ptr()), sp), ctx.h)
    s.synchronize()
    assert np.array_equal(dst.numpy(), ref)
    assert L.sun_lattice_upload_async(g2.h, None, sp) != 0


def test_pipeline_equals_serial(ctx):
    import torch
    from sun_b200._native import check, lib
    L = lib()
    nslot, steps = 3, 9
    lats = [_lat(ctx, 10 + i) for i in range(nslot)]
    n = lats[0].Bytes()
    hosts = [torch.empty(n, dtype=torch.uint8, pin_memory=True) for _ in range(nslot)]
    for g, h in zip(lats, hosts):
        check(L.sun_lattice_download(g.h, C.c_void_p(h.data_ptr()), 1, None), ctx.h)
    start = [h.numpy().copy() for h in hosts]
    s_up, s_cmp, s_dn = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    p_up, p_cmp, p_dn = (C.c_void_p(s.cuda_stream) for s in (s_up, s_cmp, s_dn))
    ev = {k: [torch.cuda.Event() for _ in range(nslot)] for k in ("up", "cmp", "dn")}
    for e in ev["dn"]:
        e.record(s_dn)
    for k in range(steps):
        i = k % nslot
        s_up.wait_event(ev["dn"][i])
        check(L.sun_lattice_upload_async(lats[i].h, C.c_void_p(hosts[i].data_ptr()), p_up), ctx.h)
        ev["up"][i].record(s_up)
        s_cmp.wait_event(ev["up"][i])
        check(L.sun_sweep(lats[i].h, 1, 4, 1, p_cmp), ctx.h)
        ev["cmp"][i].record(s_cmp)
        s_dn.wait_event(ev["cmp"][i])
        check(L.sun_lattice_download_async(lats[i].h, C.c_void_p(hosts[i].data_ptr()), p_dn), ctx.h)
        ev["dn"][i].record(s_dn)
    torch.cuda.synchronize()
    # the same steps, one after another on the default stream
    for i in range(nslot):
        g = _lat(ctx, 10 + i)
        h = torch.empty(n, dtype=torch.uint8, pin_memory=True)
        h.numpy()[:] = start[i]
        for _ in range(steps // nslot):
            check(L.sun_lattice_upload(g.h, C.c_void_p(h.data_ptr()), 1, None), ctx.h)
            check(L.sun_sweep(g.h, 1, 4, 1, None), ctx.h)
            check(L.sun_lattice_download(g.h, C.c_void_p(h.data_ptr()), 1, None), ctx.h)
        assert np.array_equal(h.numpy(), hosts[i].numpy())
