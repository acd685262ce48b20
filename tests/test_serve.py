"""Served ensembles (include/epic_serve.h): each result is the same alone and
in the mix, requests overlap on the device, admission rejects requests that
cannot fit."""
import pytest

from epic_b200 import abi, serve

pytestmark = pytest.mark.gpu

FIXED = dict(use_fixed_dt=1, fixed_dt=0.05)
CASES = [("thermal", (16, 16, 16), 1, (1, 1, 1)), ("beltrami", (16, 16, 16), 0, (1, 1, 1)),
         ("thermal", (32, 32, 16), 5, (1, 1, 1)), ("beltrami", (16, 16, 16), 0, (2, 1, 2)),
         ("thermal", (24, 24, 24), 9, (1, 1, 1)), ("thermal", (16, 16, 16), 2, (1, 1, 1))]


def _alone(glib, req):
    """The same request run directly on a context of its own."""
    ctx = abi.EpicContext(glib, req.cfg)
    ctx.init_state(req.init)
    ctx.init_correction()
    t = req.cfg.t_initial
    for _ in range(req.steps):
        t, info = ctx.step(t)
    out = dict(ke=info.parcel_stats[1], enstrophy=info.parcel_stats[12], n_parcels=info.n_parcels, t_final=t)
    ctx.close()
    return out


@pytest.mark.parametrize("precision", [1, 0])
def test_serve_same_alone_and_in_the_mix(glib, precision):
    reqs = [serve.request(k, n, seed=s, klm=klm, steps=10, precision=precision, lib=glib, **FIXED)
            for k, n, s, klm in CASES]
    with serve.Server(slots=3, lib=glib) as srv:
        ids = [srv.submit(r) for r in reqs]
        mixed = [srv.wait(i) for i in ids]
    for r, m in zip(reqs, mixed):
        assert m["status"] == 0, m["message"]
        a = _alone(glib, r)
        assert m["n_parcels"] == a["n_parcels"]
        assert m["t_final"] == pytest.approx(a["t_final"], rel=1e-14)
        assert abs(m["ke"] - a["ke"]) <= 1e-10 * abs(a["ke"])
        assert abs(m["enstrophy"] - a["enstrophy"]) <= 1e-10 * abs(a["enstrophy"])
    # continuous admission: the runs overlapped in time
    spans = sorted((m["t_start"], m["t_done"]) for m in mixed)
    assert any(spans[k + 1][0] < spans[k][1] for k in range(len(spans) - 1))
    assert len({m["slot"] for m in mixed}) > 1


def test_serve_rejects_request_larger_than_budget(glib):
    big = serve.request("thermal", (16, 16, 16), steps=1, lib=glib, capacity=10 ** 12)
    small = serve.request("thermal", (16, 16, 16), steps=2, lib=glib)
    with serve.Server(slots=2, hbm_fraction=0.5, lib=glib) as srv:
        rb, rs = srv.submit(big), srv.submit(small)
        b, s = srv.wait(rb), srv.wait(rs)
    assert b["status"] == 2 and b["slot"] == -1   # EPIC_ERR_CAPACITY
    assert s["status"] == 0 and s["parcel_steps"] == 2 * 16 ** 3 * 8


def test_serve_reuses_idle_contexts(glib):
    """Requests of one configuration run one after the other on a single slot
    give the same results as fresh contexts (the pooled context is reset)."""
    reqs = [serve.request("thermal", (16, 16, 16), seed=s, steps=5, lib=glib, **FIXED) for s in (3, 4, 3)]
    with serve.Server(slots=1, lib=glib) as srv:
        res = [srv.wait(srv.submit(r)) for r in reqs]
    assert res[0]["ke"] == pytest.approx(res[2]["ke"], rel=1e-12)
    assert res[0]["n_parcels"] == res[2]["n_parcels"]
    a = _alone(glib, reqs[1])
    assert res[1]["ke"] == pytest.approx(a["ke"], rel=1e-10)


@pytest.mark.gpu
def test_serve_results_are_handed_over(glib):
    """A result is handed over by its wait: a second wait on the same id is an
    error instead of blocking."""
    from epic_b200 import abi
    with serve.Server(slots=2, hbm_fraction=0.5, lib=glib) as srv:
        rid = srv.submit(serve.request("thermal", (16, 16, 16), seed=3, steps=2, precision=0, lib=glib))
        assert srv.wait(rid)["status"] == 0
        with pytest.raises(abi.EpicError):
            srv.wait(rid)


@pytest.mark.parametrize("policy", ["shortest-first", "arrival"])
def test_serve_admission_policy(glib, policy):
    """With one slot busy, the two queued requests start in the policy's
    order: the smaller estimated work first under "shortest-first", arrival
    order otherwise; the result is the same as the request run alone."""
    first = serve.request("thermal", (16, 16, 16), seed=1, steps=20, lib=glib, **FIXED)
    big = serve.request("thermal", (32, 32, 16), seed=2, steps=4, lib=glib, **FIXED)
    small = serve.request("thermal", (16, 16, 16), seed=3, steps=2, lib=glib, **FIXED)
    with serve.Server(slots=1, lib=glib, policy=policy) as srv:
        ids = [srv.submit(r) for r in (first, big, small)]
        rf, rb, rs = [srv.wait(i) for i in ids]
    for r in (rf, rb, rs):
        assert r["status"] == 0, r["message"]
    if policy == "shortest-first":
        assert rs["t_start"] < rb["t_start"]
    else:
        assert rb["t_start"] < rs["t_start"]
    a = _alone(glib, small)
    assert rs["n_parcels"] == a["n_parcels"]
    assert abs(rs["ke"] - a["ke"]) <= 1e-10 * abs(a["ke"])


def test_serve_rejects_unknown_policy(glib):
    with pytest.raises(KeyError):
        serve.Server(slots=1, lib=glib, policy="random")
