"""The request server (htrip_server_*): continuous batching over many map
sessions returns, for every request, exactly what the same request returns
alone on a session that saw the same earlier requests (tolerance 0: the
results are integer distances); memory admission and eviction keep that
true; bad requests and sessions that cannot fit are refused on the host."""
import numpy as np
import pytest

from helpers import make_grid
from htrip_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _cfg(b):
    from htrip_b200.minplus_oracle import HierarchyConfig
    return HierarchyConfig(tile_size_b=b, group_w=2, group_h=2)


def _sessions():
    specs = [("street", 64, 8, 1), ("maze", 128, 16, 2), ("rooms", 32, 4, 3), ("street", 128, 16, 4),
             ("maze", 64, 32, 5), ("noise", 64, 8, 6)]
    out = []
    for kind, side, b, seed in specs:
        truth = make_grid(kind, side, side, seed)
        obs, withheld = W.withheld_open(truth, side * side // 8, seed)
        out.append((truth, obs, withheld, b))
    return out


def _replay(sessions, requests, outs):
    """Each session's requests one by one through the plain per-call path."""
    from htrip_b200.minplus_oracle import MinPlusOracle
    devs, grids = [], []
    for truth, obs, withheld, b in sessions:
        d = MinPlusOracle(_cfg(b))
        g = obs.copy()
        assert d.build(g)
        devs.append(d)
        grids.append(g)
    n_q = 0
    for (s, kind, rc), out in zip(requests, outs):
        if kind == 1:
            grids[s][rc[:, 0], rc[:, 1]] = W.FREE
            devs[s].onBatchCellsOpened(rc, grids[s])
        else:
            np.testing.assert_array_equal(out, devs[s].queryAllPairs(rc, grids[s]))
            n_q += 1
    return n_q


def _run(budget, rate, n_req, seed):
    from htrip_b200.minplus_oracle import Server
    sessions = _sessions()
    srv = Server(budget_bytes=budget)
    sids = [srv.add_session(_cfg(b), obs) for _, obs, _, b in sessions]
    reqs, arrival = W.served_trace([(t, w) for t, _, w, _ in sessions], n_req, rate, seed,
                                   k_range=(4, 96), open_range=(1, 48))
    outs, lat, wall = srv.run_trace([(sids[s], k, rc) for s, k, rc in reqs], arrival)
    st = srv.stats()
    srv.close()
    assert (lat >= 0).all()
    assert _replay(sessions, reqs, outs) > 0
    return st, lat


def test_server_each_result_equals_alone(gpu):
    st, lat = _run(0, 20000.0, 600, 7)
    assert st["requests_query"] + st["requests_open"] == 600
    # continuous batching: far fewer launches than requests
    assert st["launches_query"] + st["launches_open"] < 600
    assert st["evictions"] == 0


def test_server_eviction_keeps_results(gpu):
    from htrip_b200.minplus_oracle import estimate_bytes
    sessions = _sessions()
    sizes = [estimate_bytes(_cfg(b), obs.shape[0], obs.shape[1]) for _, obs, _, b in sessions]
    budget = max(sizes) + sorted(sizes)[-2]     # room for about two sessions at a time
    st, lat = _run(budget, 5000.0, 300, 8)
    assert st["evictions"] > 0 and st["restores"] > 0
    assert st["resident_bytes"] <= st["budget_bytes"]


def test_server_refuses_what_cannot_fit_and_bad_requests(gpu):
    from htrip_b200.minplus_oracle import HtripError, Server, estimate_bytes
    grid = make_grid("street", 128, 128, 9)
    need = estimate_bytes(_cfg(8), 128, 128)
    srv = Server(budget_bytes=need // 2)
    with pytest.raises(HtripError) as e:
        srv.add_session(_cfg(8), grid)
    assert e.value.status == 3          # HTRIP_ERR_OOM: admission refused
    with pytest.raises(HtripError) as e:
        srv.submit_query(12345, [[1, 1]])
    assert e.value.status == 1          # unknown session
    srv.close()
    srv = Server()
    sid = srv.add_session(_cfg(8), grid)
    t, out = srv.submit_query(sid, W.sample_free(grid, 10, 1))
    assert srv.wait(t) >= 0
    with pytest.raises(HtripError):
        srv.wait(t)                     # a ticket is consumed once
    srv.remove_session(sid)
    srv.close()


def test_plain_per_call_mode_gives_same_results(gpu):
    """The unbatched baseline mode answers identically (one launch per request)."""
    from htrip_b200.minplus_oracle import Server
    sessions = _sessions()[:3]
    srv = Server(plain=True)
    sids = [srv.add_session(_cfg(b), obs) for _, obs, _, b in sessions]
    reqs, arrival = W.served_trace([(t, w) for t, _, w, _ in sessions], 150, 5000.0, 11,
                                   k_range=(4, 64), open_range=(1, 32))
    outs, lat, wall = srv.run_trace([(sids[s], k, rc) for s, k, rc in reqs], arrival)
    st = srv.stats()
    srv.close()
    assert st["launches_query"] + st["launches_open"] == 150
    _replay(sessions, reqs, outs)


@pytest.mark.parametrize("tight_budget", [False, True])
def test_double_buffered_queries_equal_their_published_state(gpu, tight_budget):
    """Double-buffered sessions (the reference simulator's front / back
    oracle protocol): every query's result equals a replay of exactly the
    openings its reported version includes, versions only move forward, and
    a query submitted after every opening has finished sees them all; with a
    budget for about two sessions the two indexes of a session are offloaded
    and restored together."""
    from htrip_b200.minplus_oracle import MinPlusOracle, Server, estimate_bytes
    sessions = _sessions()[:4]
    budget = 0
    if tight_budget:
        sizes = sorted(2 * estimate_bytes(_cfg(b), o.shape[0], o.shape[1]) for _, o, _, b in sessions)
        budget = sizes[-1] + sizes[-2]
    srv = Server(budget_bytes=budget, double_buffer=True)
    sids = [srv.add_session(_cfg(b), obs) for _, obs, _, b in sessions]
    rng = np.random.default_rng(61)
    batches = [np.array_split(w, 6) for _, _, w, _ in sessions]
    plan = []  # (session index, kind, payload)
    for step in range(6):
        for i in range(len(sessions)):
            plan.append((i, "open", batches[i][step]))
            for _ in range(2):
                plan.append((i, "query", W.sample_free(sessions[i][0], int(rng.integers(4, 40)), int(rng.integers(1 << 30)))))
    tickets = []
    for i, kind, payload in plan:
        if kind == "open":
            tickets.append((i, kind, payload, srv.submit_open(sids[i], payload), None))
        else:
            t, out = srv.submit_query(sids[i], payload)
            tickets.append((i, kind, payload, t, out))
    seen = [[] for _ in sessions]
    for i, kind, payload, t, out in tickets:
        _, version = srv.wait_version(t)
        if kind == "query":
            seen[i].append((version, payload, out))
    for i, (truth, obs0, withheld, b) in enumerate(sessions):
        versions = [v for v, _, _ in seen[i]]
        assert versions == sorted(versions) and 0 <= versions[0] and versions[-1] <= 6
        # replay: the state after v openings, for every version a query saw
        dev = MinPlusOracle(_cfg(b))
        grid = obs0.copy()
        assert dev.build(grid)
        applied = 0
        for v, vps, out in seen[i]:
            while applied < v:
                part = batches[i][applied]
                grid[part[:, 0], part[:, 1]] = W.FREE
                dev.onBatchCellsOpened(part, grid)
                applied += 1
            np.testing.assert_array_equal(out, dev.queryAllPairs(vps, grid), err_msg=f"session {i} version {v}")
        # after every opening has finished, a new query includes them all
        vps = W.sample_free(truth, 24, 100 + i)
        t, out = srv.submit_query(sids[i], vps)
        _, v = srv.wait_version(t)
        assert v == 6
        while applied < 6:
            part = batches[i][applied]
            grid[part[:, 0], part[:, 1]] = W.FREE
            dev.onBatchCellsOpened(part, grid)
            applied += 1
        np.testing.assert_array_equal(out, dev.queryAllPairs(vps, grid))
    st = srv.stats()
    if tight_budget:
        assert st["resident_bytes"] <= st["budget_bytes"]
    srv.close()
