"""The continuous-batching request loop (xpr_serve_*): a request's volume is
bit-identical whether it is served alone or among others arriving while it runs
(tolerance 0 ulp, NaN positions identical), and identical to the same parameters run
through the whole-run entry point (xpr_reconstruct_host, the naive method); admission
keeps the resident requests within the device-memory budget."""
import ctypes as C
import json
import time

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from tests.cases import assert_same_bits  # noqa: E402
from xpulse_recon_b200 import _lib  # noqa: E402
from xpulse_recon_b200.projector import Context  # noqa: E402
from xpulse_recon_b200.serve import DONE, Server  # noqa: E402

pytestmark = pytest.mark.gpu


def _request(i):
    """(params, raw) of request i: mixed grids, sub-iteration counts, offsets and modules."""
    rng = np.random.default_rng(100 + i)
    shapes = [(36, 32, 40), (24, 40, 48), (30, 24, 60), (23, 29, 37), (40, 48, 64), (20, 16, 24)]
    P, H, W = shapes[i % len(shapes)]
    recon = {"method": "naive", "it": 1 + i % 2, "sit": [4, 3, 2, 3, 5, 4][i % 6], "seed": 1000 + i,
             "mlog": True, "weight": 1.0, "weight_factor": 0.9, "normalize": i % 3 == 2}
    det = {"px": 0.1, "rx": [0.0, 1.0, 0.0, -0.7, 0.5, 0.0][i % 6], "sx": [0.0, -0.5, 0.0, 0.0, 1.0, 0.0][i % 6],
           "sy": [0.0, 0.8, 0.0, 0.4, 0.0, 0.0][i % 6]}
    if i % 6 == 2:
        det["module_number"] = 3
        det["modules"] = [{"roll": 1.0, "pitch": -0.5, "yaw": 0.8}, {"roll": 0.0, "pitch": 0.3, "yaw": -1.2},
                          {"roll": -1.5, "pitch": 0.9, "yaw": 0.2}]
    params = {"recon": recon, "geometry": {"so": 100.0, "sd": 1000.0, "angle": 360.0}, "detector": det}
    raw = rng.uniform(0.05, 0.98, (P, H, W)).astype(np.float32)
    return params, raw


@pytest.fixture(scope="module")
def sctx():
    c = Context(0)
    yield c
    c.close()


def _alone(ctx, reqs, storage):
    srv = Server(ctx, storage=storage)
    out = []
    for params, raw in reqs:
        t = srv.submit(params, raw)
        assert srv.wait(t, 60.0).state == DONE
        out.append(srv.result(t).copy())
    srv.close()
    return out


@pytest.mark.parametrize("storage", [_lib.F32, _lib.F16])
def test_alone_equals_mixed(sctx, storage):
    reqs = [_request(i) for i in range(8)]
    alone = _alone(sctx, reqs, storage)
    srv = Server(sctx, storage=storage)
    tickets = []
    for k, (params, raw) in enumerate(reqs):
        tickets.append(srv.submit(params, raw))
        if k % 3 == 1:
            time.sleep(0.002)  # some arrive while others are on the GPU
    infos = [srv.wait(t, 60.0) for t in tickets]
    st = srv.stats()
    for info, t, a in zip(infos, tickets, alone):
        assert info.state == DONE
        assert info.submit_s <= info.admit_s <= info.done_s
        v = srv.result(t)
        assert np.isfinite(v).mean() > 0.5
        assert_same_bits(v, a)
    assert st.completed == len(reqs) and st.failed == 0
    srv.close()


def test_requests_in_flight_share_ticks(sctx):
    """Requests that arrive while others run join the running batch: 4 requests of 100
    short sub-iterations each, submitted back to back, finish in far fewer than 400 ticks."""
    srv = Server(sctx)
    tickets = []
    for i in range(4):
        params, raw = _request(5)  # 20 projections of 16 x 24
        params["recon"].update({"it": 5, "sit": 20, "seed": 500 + i})
        tickets.append(srv.submit(params, raw))
    assert all(srv.wait(t, 60.0).state == DONE for t in tickets)
    st = srv.stats()
    assert st.ticks < 4 * 100, st.ticks
    srv.close()


def test_served_equals_whole_run_entry_point(sctx):
    params, raw = _request(1)
    srv = Server(sctx, arith=_lib.STRICT, storage=_lib.F32)
    t = srv.submit(params, raw)
    assert srv.wait(t, 60.0).state == DONE
    got = srv.result(t)
    srv.close()
    L = _lib.lib()
    L.xpr_reconstruct_host.argtypes = [C.c_char_p, C.c_void_p, C.c_int64, C.c_uint32, C.c_uint32, C.c_void_p,
                                       C.c_uint64, C.POINTER(C.c_double)]
    P, H, W = raw.shape
    exp = np.full(got.size, np.nan, np.float32)
    cfg = json.loads(json.dumps(params))
    cfg["recon"]["arith"] = "strict"
    rc = L.xpr_reconstruct_host(json.dumps(cfg).encode(), raw.ctypes.data, P, W, H, exp.ctypes.data, exp.size,
                                C.byref(C.c_double()))
    assert rc == 0
    assert_same_bits(got, exp)


def test_admission_respects_the_memory_budget(sctx):
    reqs = [_request(i) for i in (0, 1, 4, 5)]
    alone = _alone(sctx, reqs, _lib.F32)
    probe = Server(sctx)
    sizes = []
    for params, raw in reqs:
        t = probe.submit(params, raw)
        sizes.append(probe.wait(t, 60.0).device_bytes)
    probe.close()
    budget = max(sizes) + min(sizes)  # the largest fits, never alongside another large one
    srv = Server(sctx, mem_budget=budget)
    tickets = [srv.submit(p, r) for p, r in reqs]
    for t, a in zip(tickets, alone):
        assert srv.wait(t, 60.0).state == DONE
        assert_same_bits(srv.result(t), a)
    st = srv.stats()
    assert 0 < st.peak_bytes <= budget
    srv.close()


def test_rejections(sctx):
    params, raw = _request(0)
    srv = Server(sctx, mem_budget=4096)  # smaller than any request
    with pytest.raises(_lib.XprError, match="budget"):
        srv.submit(params, raw)
    bad = json.loads(json.dumps(params))
    bad["recon"]["sit"] = 1000  # more sub-iterations than projections
    srv2 = Server(sctx)
    with pytest.raises(_lib.XprError, match="sub-iterations"):
        srv2.submit(bad, raw)
    srv.close()
    srv2.close()
