"""Batched reconstructions (xpr_batch_*): every problem's volume must be bit-identical
to the same reconstruction run alone through xpr_subiteration, whatever the batch's
composition, schedule (projection-run split, backward column length), graph capture or
storage type; and the FP32 form must equal the CPU oracle.  Tolerance: 0 ulp (NaN
positions identical)."""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import oracle as O  # noqa: E402
from tests.cases import assert_same_bits  # noqa: E402
from xpulse_recon_b200 import _lib  # noqa: E402
from xpulse_recon_b200.batch import Batch, Problem  # noqa: E402
from xpulse_recon_b200.projector import Context  # noqa: E402

pytestmark = pytest.mark.gpu

# (geometry, detector (P, H, W), it, sit, seed)
SPECS = [
    (dict(rx=1.0, sx=-0.5, sy=0.8), (36, 32, 40), 2, 4, 11),
    (dict(), (24, 40, 48), 1, 3, 12),
    (dict(module_number=3, mod_rpy=[1.0, -0.5, 0.8, 0.0, 0.3, -1.2, -1.5, 0.9, 0.2]), (20, 24, 60), 2, 2, 13),
    (dict(rx=-0.7, sy=0.4), (23, 29, 37), 1, 3, 14),
]


def _raw(shape, seed):
    return np.random.default_rng(seed).uniform(0.05, 0.98, shape).astype(np.float32)


def _problems(ctx, storage, residual=False):
    return [Problem.from_raw(ctx, _raw(shape, seed), geom, it, sit, seed=seed, storage=storage, residual=residual)
            for geom, shape, it, sit, seed in SPECS]


@pytest.fixture(scope="module")
def bctx():
    c = Context(0)
    yield c
    c.close()


def _alone(ctx, problems, arith, storage):
    out = []
    for p in problems:
        p.run_alone(ctx, arith, storage)
        torch.cuda.synchronize()
        out.append(p.vol.cpu().numpy().copy())
    return out


@pytest.mark.parametrize("storage", [_lib.F32, _lib.BF16, _lib.F16])
def test_batch_equals_each_problem_alone(bctx, storage):
    probs = _problems(bctx, storage)
    alone = _alone(bctx, probs, _lib.FAST, storage)
    b = Batch(bctx, probs, arith=_lib.FAST, storage=storage, use_graph=True, autotune=True)
    assert b.steps == max(p.it * p.sit for p in probs)
    b.run()
    torch.cuda.synchronize()
    for p, a in zip(probs, alone):
        v = p.vol.cpu().numpy()
        assert np.isfinite(v).mean() > 0.5
        assert_same_bits(v, a)
    # the captured run replays to the same volumes
    b.run()
    torch.cuda.synchronize()
    for p, a in zip(probs, alone):
        assert_same_bits(p.vol.cpu().numpy(), a)
    b.close()


@pytest.mark.parametrize("splits,layers,column", [(1, 16, 16), (3, 8, 8), (8, 16, 16), (2, 8, 16)])
def test_schedule_does_not_change_results(bctx, splits, layers, column):
    probs = _problems(bctx, _lib.F32)
    alone = _alone(bctx, probs, _lib.STRICT, _lib.F32)
    b = Batch(bctx, probs, use_graph=False, autotune=False, fwd_splits=splits, bwd_column=column, ctas_per_sm=2,
              fwd_layers=layers)
    sch = b.schedule()
    assert sch["fwd_splits"] == splits and sch["bwd_column"] == column and sch["ctas_per_sm"] <= 2
    assert sch["fwd_layers"] == layers
    for p in probs:  # xpr_batch_step does not initialise the volumes; xpr_batch_run does
        p.vol.fill_(1.0)
    for k in range(b.steps):  # step by step, as a serving loop drives it
        b.step(k)
    torch.cuda.synchronize()
    for p, a in zip(probs, alone):
        assert_same_bits(p.vol.cpu().numpy(), a)
    b.close()


def test_batch_strict_fp32_matches_oracle(bctx):
    geom, shape, it, sit, seed = SPECS[0]
    raw = _raw(shape, seed)
    p = Problem.from_raw(bctx, raw, geom, it, sit, seed=seed)
    b = Batch(bctx, [p], arith=_lib.STRICT, use_graph=True, autotune=False)
    b.run()
    torch.cuda.synchronize()
    imgs = raw.ravel().copy()
    O.lib().orc_preprocess(imgs, imgs.size, 0, 0.0, 0.0, 1)
    P, H, W = shape
    gp = O.geom_params(dwidth=W, dheight=H, projections=P, sit=sit, **geom)
    rp = O.ReconParams(it, sit, 1.0, 0.9, seed, O.STRICT, 0)
    exp = np.zeros(p.vol.numel(), np.float32)
    assert O.lib().orc_recon_naive(C.byref(gp), C.byref(rp), imgs, exp) == 0
    assert_same_bits(p.vol.cpu().numpy(), exp)
    b.close()


def test_batch_residuals_match_alone(bctx):
    probs = _problems(bctx, _lib.F32, residual=True)
    _alone(bctx, probs, _lib.STRICT, _lib.F32)
    ref = [p.residual.cpu().numpy().copy() for p in probs]
    for p in probs:
        p.residual.zero_()
    b = Batch(bctx, probs, use_graph=True, autotune=False)
    b.run()
    torch.cuda.synchronize()
    for p, r in zip(probs, ref):
        got = p.residual.cpu().numpy()
        assert (r > 0).all()
        np.testing.assert_allclose(got, r, rtol=1e-12)  # FP64 sums; the atomic order differs
    b.close()


def test_bad_problem_is_rejected(bctx):
    probs = _problems(bctx, _lib.F32)[:1]
    probs[0].sit = 0
    with pytest.raises(_lib.XprError, match="sit"):
        Batch(bctx, probs)


def test_sixteen_layer_forward_is_strict_only(bctx):
    probs = _problems(bctx, _lib.F32)[:1]
    with pytest.raises(_lib.XprError, match="fwd_layers"):
        Batch(bctx, probs, arith=_lib.FAST, fwd_layers=16)
    with pytest.raises(_lib.XprError, match="fwd_layers"):
        Batch(bctx, probs, arith=_lib.STRICT, fwd_layers=12)
