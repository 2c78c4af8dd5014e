"""The serving loop (rf_server_*): continuous batching with HBM admission.

Checked through the C-ABI:
  * a request's field is the same alone and in a mix of concurrent requests
    (each request's tables come from its own seed and its tiles are computed
    independently of the others: the fields are bitwise equal), and it
    matches the single call within the BF16 bound (relative-L2 <= 2e-3);
  * requests submitted from several threads while batches run are admitted
    into later batches (more than one batch, all complete);
  * a request whose device footprint exceeds a slot's share of the budget
    fails with RF_ENOMEM_ADMISSION without disturbing the others;
  * latency statistics (p50 <= p99 <= max) are reported.
"""
import threading
import time

import numpy as np
import pytest

import randomfield_b200 as rf
from tests.helpers import errors, grid, uniform_points

pytestmark = pytest.mark.gpu


def _req(x, Nmc, method, seed, marg="gaussian", **opts):
    xf = np.asfortranarray(x.T)
    out = np.full((x.shape[0], Nmc), np.nan, order="F")
    avg, var = (1.0, 0.25) if marg == "lognormal" else (0.0, 1.0)
    if method == 2:
        opts.setdefault("k_nstep", (24, 24, 24)[:x.shape[1]] + (0,) * (3 - x.shape[1]))
    else:
        opts.setdefault("iso_n_radial", 32)
        opts.setdefault("iso_n_dir", 32)
    r = rf.make_request(xf, "gaussian", marg, (1.0, 0.8, 1.3)[:x.shape[1]], avg, var, Nmc, method, out,
                        seed_start=seed, **opts)
    return r, xf, out


def _mix():
    rs = np.random.RandomState(5)
    out = []
    for k in range(12):
        n = int(rs.randint(500, 6000))
        x = uniform_points(n, float(rs.uniform(1, 10)), seed=100 + k)
        out.append((x, int(rs.randint(1, 70)), 1 + (k % 2), 1000 + k, "lognormal" if k % 3 == 0 else "gaussian"))
    return out


def test_same_result_alone_and_in_the_mix():
    srv = rf.Server(precision="bf16")
    try:
        mix = _mix()
        probe = 4
        x, Nmc, method, seed, marg = mix[probe]
        r, xf, alone = _req(x, Nmc, method, seed, marg)
        srv.wait(srv.submit(r, keep=(xf, alone)))
        # the whole mix from two threads with staggered arrivals
        results = {}

        def producer(ids):
            for i in ids:
                x_, Nmc_, m_, s_, mg_ = mix[i]
                rq, xf_, out_ = _req(x_, Nmc_, m_, s_, mg_)
                results[i] = (srv.submit(rq, keep=(xf_, out_)), out_)
                time.sleep(0.002)

        th = [threading.Thread(target=producer, args=(list(range(k, len(mix), 2)),)) for k in range(2)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        for i, (ticket, out) in results.items():
            lat = srv.wait(ticket)
            assert lat > 0 and np.isfinite(out).all(), i
        np.testing.assert_array_equal(results[probe][1], alone)
        single = rf.create_standard_gaussian_field_unstruct(x.T, "gaussian", marg, (1.0, 0.8, 1.3), *(
            (1.0, 0.25) if marg == "lognormal" else (0.0, 1.0)), Nmc, method, precision="bf16",
            seed_start=seed, k_nstep=(24, 24, 24) if method == 2 else (0, 0, 0),
            iso_n_radial=32 if method == 1 else 0, iso_n_dir=32 if method == 1 else 0)
        g = (lambda f: np.log(f)) if marg == "lognormal" else (lambda f: f)
        assert errors(g(alone), g(np.asarray(single)))[1] <= 2e-3
        st = srv.stats()
        assert st["completed"] == len(mix) + 1 and st["failed"] == 0 and st["batches"] >= 2
        assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
        assert st["field_values"] == float(sum(m[0].shape[0] * m[1] for m in mix) + x.shape[0] * Nmc)
    finally:
        srv.close()


def test_admission_rejects_oversized_request():
    # budget of 64 MB: slots of 32 MB; a 200k-point, 64-realization request needs ~110 MB
    srv = rf.Server(precision="bf16", hbm_budget_bytes=64 << 20)
    try:
        big, xb, ob = _req(uniform_points(200000, 10.0, seed=1), 64, 1, 1)
        small, xs, os_ = _req(grid(10, 0.2), 8, 2, 2)
        tb = srv.submit(big, keep=(xb, ob))
        ts = srv.submit(small, keep=(xs, os_))
        with pytest.raises(rf.RandomFieldError) as e:
            srv.wait(tb)
        assert e.value.code == -23
        srv.wait(ts)
        assert np.isfinite(os_).all()
        st = srv.stats()
        assert st["failed"] == 1 and st["completed"] == 1
    finally:
        srv.close()


def test_blended_request_in_the_mix():
    """A localization blend submitted among plain requests gives the field of
    rf_generate_blended alone (FP64 atomic adds make the order of the
    subdomain contributions vary: relative difference <= 1e-12)."""
    grid = rf.BlendGrid.make((21, 21, 21), (0.1, 0.1, 0.1), (2, 2, 2), 0.4)
    ctx = rf.Context(0)
    alone = ctx.generate_blended(grid, "gaussian", "lognormal", (1.0, 1.0, 1.0), 1.0, 0.25, 3, 2, precision="bf16",
                                 seed_start=8, k_nstep=(24, 24, 24))
    ctx.close()
    srv = rf.Server(precision="bf16")
    try:
        tickets = []
        for i, (x, Nmc, method, seed, marg) in enumerate(_mix()[:5]):
            r, xf, out = _req(x, Nmc, method, seed, marg)
            tickets.append(srv.submit(r, keep=(xf, out)))
            if i == 2:
                mixed = np.full(alone.shape, np.nan, order="F")
                tb = srv.submit_blended(grid, "gaussian", "lognormal", (1.0, 1.0, 1.0), 1.0, 0.25, 3, 2, mixed,
                                        seed_start=8, k_nstep=(24, 24, 24))
        srv.wait(tb)
        for t in tickets:
            srv.wait(t)
        assert np.isfinite(mixed).all()
        assert errors(np.log(mixed), np.log(alone))[1] <= 1e-12
    finally:
        srv.close()
