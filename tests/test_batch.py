"""Batches through the C-ABI: rf_generate_batch / rf_generate_batch_device.

Every request of a batch must give the field it gives alone (the single
call, same precision form) and the FP64 oracle's field within the stated
bounds: relative-L2 <= 2e-3 (BF16, FP16) against the oracle, and the batch
against the single call within the same bound (the two differ only where the
grouped launch takes GEN_TABLE for a Shinozuka grid that the single call runs
with GEN_GRID3, and in the realization blocking).  The mix covers both
generators, 2-D and 3-D, the isotropic method, both marginals, and Nmc from 1
to 128 (realization blocks of the tuner's size and ragged last blocks).
"""
import numpy as np
import pytest

import randomfield_b200 as rf
from oracle import oracle as O
from tests.helpers import errors, grid, uniform_points

pytestmark = pytest.mark.gpu

REL_L2 = 2e-3


def _mix(seed=7):
    rs = np.random.RandomState(seed)
    reqs = []
    # (points, method, Nmc, corrL, marginal, options)
    reqs.append((grid(20, 0.1), 2, 64, (1.0, 1.0, 1.0), "gaussian", dict(k_nstep=(24, 24, 24), seed_start=1)))
    reqs.append((uniform_points(3000, 4.0, seed=2), 2, 5, (1.0, 0.7, 1.5), "lognormal",
                 dict(k_nstep=(16, 16, 16), seed_start=2)))
    reqs.append((uniform_points(5000, 8.0, seed=3), 1, 128, (1.0, 1.0, 1.0), "gaussian",
                 dict(iso_n_radial=32, iso_n_dir=32, seed_start=3)))
    reqs.append((uniform_points(1000, 3.0, nDim=2, seed=4), 2, 1, (0.5, 2.0), "gaussian",
                 dict(k_nstep=(20, 20, 0), seed_start=4)))
    reqs.append((uniform_points(2500, 5.0, seed=5), 2, 100, (2.0, 1.0, 0.5), "gaussian",
                 dict(k_nstep=(24, 24, 24), seed_start=5)))
    reqs.append((uniform_points(700, 6.0, seed=6), 1, 33, (1.0, 1.0, 1.0), "lognormal",
                 dict(iso_n_radial=16, iso_n_dir=16, seed_start=6)))
    return reqs


def _single(x, method, Nmc, corrL, marg, opts, prec):
    avg, var = (1.0, 0.25) if marg == "lognormal" else (0.0, 1.0)
    out = rf.create_standard_gaussian_field_unstruct(x.T, "gaussian", marg, corrL, avg, var, Nmc, method,
                                                     precision=prec, **opts)
    return np.asarray(out)


def _oracle(x, method, Nmc, corrL, marg, opts, rows):
    avg, var = (1.0, 0.25) if marg == "lognormal" else (0.0, 1.0)
    kw = dict(Nmc=Nmc, method=method, corrL=corrL, margiFirst=2 if marg == "lognormal" else 1, fieldAvg=avg,
              fieldVar=var, seedStart=opts.get("seed_start", 0))
    if "k_nstep" in opts:
        kw["kNStep"] = tuple(v for v in opts["k_nstep"][:x.shape[1]])
    if "iso_n_radial" in opts:
        kw["isoNRadial"], kw["isoNDir"] = opts["iso_n_radial"], opts["iso_n_dir"]
    return O.OracleRequest(x, **kw).generate(rows=rows)


def _gauss(f, marg):
    return np.log(f) if marg == "lognormal" else f


@pytest.fixture(scope="module")
def ctx():
    c = rf.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("prec", ["bf16", "fp16"])
def test_batch_matches_single_and_oracle(ctx, prec):
    mix = _mix()
    outs, reqs = [], []
    for (x, method, Nmc, corrL, marg, opts) in mix:
        xf = np.asfortranarray(x.T)
        out = np.full((x.shape[0], Nmc), np.nan, order="F")
        avg, var = (1.0, 0.25) if marg == "lognormal" else (0.0, 1.0)
        reqs.append(rf.make_request(xf, "gaussian", marg, corrL, avg, var, Nmc, method, out, precision=prec, **opts))
        outs.append((xf, out))
    rf.generate_batch(ctx, reqs)
    st = ctx.batch_stats()
    assert st["units"] >= len(mix) and st["work_items"] > 0 and st["stages"] >= 2
    rs = np.random.RandomState(11)
    for (x, method, Nmc, corrL, marg, opts), (_, out) in zip(mix, outs):
        assert np.isfinite(out).all()
        alone = _single(x, method, Nmc, corrL, marg, opts, prec)
        assert errors(_gauss(out, marg), _gauss(alone, marg))[1] <= REL_L2
        rows = rs.choice(x.shape[0], min(64, x.shape[0]), replace=False)
        ref = _oracle(x, method, Nmc, corrL, marg, opts, rows)  # [r, i]
        got = _gauss(out[rows].T, marg)
        # a request of one to three realizations on 64 rows is a per-realization
        # figure, which fluctuates: 1.25x the bound, as in the parity suite
        bound = REL_L2 * (1.25 if Nmc < 4 else 1.0)
        assert errors(got, _gauss(ref, marg))[1] <= bound, (method, Nmc, errors(got, _gauss(ref, marg)))


def test_batch_replays_graph_and_is_repeatable(ctx):
    mix = _mix(seed=9)[:3]
    runs = []
    for rep in range(2):
        reqs, outs = [], []
        for (x, method, Nmc, corrL, marg, opts) in mix:
            xf = np.asfortranarray(x.T)
            out = np.zeros((x.shape[0], Nmc), order="F")
            avg, var = (1.0, 0.25) if marg == "lognormal" else (0.0, 1.0)
            reqs.append(rf.make_request(xf, "gaussian", marg, corrL, avg, var, Nmc, method, out, precision="bf16",
                                        **opts))
            outs.append(out)
        rf.generate_batch(ctx, reqs)
        runs.append(outs)
        if rep == 1:
            assert ctx.batch_stats()["graph_replayed"] == 1
    for a, b in zip(*runs):
        np.testing.assert_array_equal(a, b)  # deterministic: same tables, same schedule


def test_device_batch_equals_host_batch(ctx):
    torch = pytest.importorskip("torch")
    mix = _mix(seed=3)[1:4]
    host, dev, keep = [], [], []
    for (x, method, Nmc, corrL, marg, opts) in mix:
        xf = np.asfortranarray(x.T)
        out = np.zeros((x.shape[0], Nmc), order="F")
        avg, var = (1.0, 0.25) if marg == "lognormal" else (0.0, 1.0)
        host.append((rf.make_request(xf, "gaussian", marg, corrL, avg, var, Nmc, method, out, precision="bf16",
                                     **opts), out))
        dx = torch.from_numpy(np.ascontiguousarray(x)).cuda()
        dout = torch.empty((Nmc, x.shape[0]), dtype=torch.float64, device="cuda")
        keep.append((dx, dout))
        dev.append(rf.make_request(dx, "gaussian", marg, corrL, avg, var, Nmc, method, dout, precision="bf16",
                                   nDim=x.shape[1], n=x.shape[0], **opts))
    rf.generate_batch(ctx, [h for h, _ in host])
    ctx.generate_batch_device(dev)
    ctx.synchronize()
    for (_, out), (_, dout) in zip(host, keep):
        np.testing.assert_array_equal(out, dout.cpu().numpy().T)


def test_batch_rejects_mixed_precision_and_literal(ctx):
    x = np.asfortranarray(uniform_points(200, 2.0).T)
    o1, o2 = np.zeros((200, 2), order="F"), np.zeros((200, 2), order="F")
    a = rf.make_request(x, "gaussian", "gaussian", (1, 1, 1), 0, 1, 2, 2, o1, precision="bf16")
    b = rf.make_request(x, "gaussian", "gaussian", (1, 1, 1), 0, 1, 2, 2, o2, precision="fp16")
    with pytest.raises(rf.RandomFieldError) as e:
        rf.generate_batch(ctx, [a, b])
    assert e.value.code == -9
    c = rf.make_request(x, "gaussian", "gaussian", (1, 1, 1), 0, 1, 2, 2, o2, precision="bf16", literal=True)
    with pytest.raises(rf.RandomFieldError) as e:
        rf.generate_batch(ctx, [a, c])
    assert e.value.code == -10
