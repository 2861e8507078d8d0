"""Request server (iga_server_*): mixed fan and eigenray requests admitted
concurrently give exactly the results of the same requests run alone, under
a tight device-memory budget too, and the latency statistics are filled in."""
import os
import threading

import numpy as np
import pytest

import infraga_b200 as ig
from infraga_b200 import synth
from tests._cases import GOLDEN, profile_path

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    ig.lib()
    return torch


@pytest.fixture(scope="module")
def workload(dev):
    """A mix over four resident atmospheres: 3D fans (FP64 and FP32C) of
    very different sizes, spherical stratified and range-dependent fans, and
    two eigenray searches."""
    a3 = ig.Atmosphere.load(profile_path(0))
    b3 = ig.Atmosphere.load(profile_path(1))
    s2 = ig.Atmosphere.load(profile_path(2))
    rng = os.path.join(GOLDEN, "rngdep")
    sr = ig.Atmosphere.load_rngdep(os.path.join(rng, "node"), os.path.join(rng, "node_lat.dat"),
                                   os.path.join(rng, "node_lon.dat"), topo_file=os.path.join(rng, "topo.dat"))
    th, ph = synth.fan_angles(0.5, 60.0, 0.5, 0.0, 350.0, 10.0)       # 4320 rays
    reqs = []
    reqs.append(("fan", a3, a3.default_params(bounces=3, rng_max=800.0), th, ph))
    reqs.append(("fan", b3, b3.default_params(bounces=2, precision=ig.FP32C), th[::7], ph[::7]))
    reqs.append(("fan", a3, a3.default_params(bounces=1, calc_amp=0), th[:40], ph[:40]))
    reqs.append(("fan", s2, s2.default_params(geometry=ig.GEOM_SPH, bounces=2), th[::5], ph[::5]))
    p = sr.default_params(geometry=ig.GEOM_SPH, bounces=1)
    reqs.append(("fan", sr, p, th[::97], ph[::97]))
    e4 = ig.Atmosphere.load(profile_path(4))
    reqs.append(("eig", e4, ig.eig_params(e4, bnc_min=0, bnc_max=1), [((0.0, 0.0, 0.0), (330.0, 90.0))], None))
    reqs.append(("eig", a3, ig.eig_params(a3, bnc_min=0, bnc_max=0), [((0.0, 0.0, 0.0), (250.0, 40.0)),
                                                                        ((0.0, 0.0, 0.0), (-200.0, 10.0))], None))
    alone = []
    for kind, atmo, params, x, y in reqs:
        if kind == "fan":
            r = ig.fan_run(atmo, params, x, y)
            alone.append((r["arrivals"], r["ray_index"], r["total_steps"]))
        else:
            r = ig.eig_run(atmo, params, x)
            alone.append((r["eigenrays"], r["pair_index"], r["total_steps"]))
    keep = [a3, b3, s2, sr, e4]
    return reqs, alone, keep


def run_mix(reqs, **cfg):
    with ig.Server(**cfg) as srv:
        ids = [None] * len(reqs)

        def submit(order):
            for i in order:
                kind, atmo, params, x, y = reqs[i]
                ids[i] = srv.submit_fan(atmo, params, x, y) if kind == "fan" else srv.submit_eig(atmo, params, x)

        # two client threads submitting interleaved
        t1 = threading.Thread(target=submit, args=(range(0, len(reqs), 2),))
        t2 = threading.Thread(target=submit, args=(range(1, len(reqs), 2),))
        t1.start(); t2.start(); t1.join(); t2.join()
        out = []
        for rid in ids:
            assert srv.wait(rid, 600.0)
            out.append(srv.fetch(rid))
        return out, srv.stats()


def check(reqs, alone, out):
    for (kind, *_), (rows, idx, steps), got in zip(reqs, alone, out):
        np.testing.assert_array_equal(got["rows"], rows)
        np.testing.assert_array_equal(got["index"], idx)
        assert got["total_steps"] == steps
        assert got["latency_s"] > 0.0


def test_mix_equals_alone(workload):
    reqs, alone, _ = workload
    out, st = run_mix(reqs)
    check(reqs, alone, out)
    assert st["completed"] == len(reqs) and st["pending"] == 0
    assert 0.0 < st["p50_s"] <= st["p99_s"]
    assert st["bytes_in_use"] == 0


def test_mix_under_tight_budget(workload):
    """A budget that holds about one large request at a time still admits
    and completes everything (later small requests pass a waiting large one)."""
    reqs, alone, _ = workload
    out, st = run_mix(reqs, hbm_budget=12 << 20, max_inflight=3, eig_workers=1)
    check(reqs, alone, out)
    assert st["completed"] == len(reqs)


def test_oversized_request_is_refused(dev):
    a = ig.Atmosphere.load(profile_path(0))
    th = np.linspace(1.0, 40.0, 5000)
    with ig.Server(hbm_budget=1 << 20) as srv:
        with pytest.raises(ig.IgaError):
            srv.submit_fan(a, a.default_params(), th, np.full_like(th, 90.0))
