"""The serving loop (ps4_serve_*): continuous batching of subrange and triple queries.

Bar: every query's result in the mix is bit-identical to the same query run alone
(ps4_search_range / ps4_extend_triples) -- lines in order, every counter, the histogram and
the maxima; triple extensions, state and counters.
"""
from __future__ import annotations

import pytest

from conftest import assert_stats_equal
from ps4b200 import Ps4Error, Search, _abi, workloads
from ps4b200.serve import Server, run_stream

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def search():
    with Search(2 * 10 ** 12) as s:
        yield s


def _check_same(search, r, got):
    if r.kind == "range":
        want = search.range(r.lo, r.hi)
        assert got.lines == want.lines, (r.lo, r.hi)
        assert got.six_lines == want.six_lines
        assert_stats_equal(got.stats, want.stats, label=f"[{r.lo},{r.hi})")
    else:
        ext, state, st = search.extend_triples([r.abc], r.dmax)
        assert got == (ext[0], int(state[0]), st), r.abc


def test_mixed_stream_matches_alone(search):
    reqs = workloads.requests(160, seed=31, rate=400.0, wmax=1e8)
    with Server(search, hbm_budget=4 << 30, step_S=1 << 25) as srv:
        rep = run_stream(srv, reqs)
    assert len(rep.results) == len(rep.latency_s) == len(reqs)
    for r in reqs:
        _check_same(search, r, rep.results[r.rid])
    # queries share steps: the steps that carried each query add up to more than the steps run
    assert rep.info["steps"] >= 2
    assert sum(d["steps"] for d in rep.done.values()) > rep.info["steps"]
    assert rep.info["waiting"] == rep.info["active"] == 0 and rep.info["arena_used"] == 0
    assert rep.percentile(50) > 0


def test_admission_by_slots_and_budget(search):
    """Two slots and a small arena: most queries wait, all finish, results unchanged."""
    reqs = workloads.requests(40, seed=32, rate=1e6, wmax=3e7)
    with Server(search, hbm_budget=1 << 30, max_slots=2, step_S=1 << 24, max_step_items=64) as srv:
        for r in reqs:
            if r.kind == "range":
                srv.submit_range(r.rid, r.lo, r.hi)
            else:
                srv.submit_triple(r.rid, r.abc, r.dmax)
        assert srv.info()["waiting"] == len(reqs)
        seen_waiting = 0
        got = {}
        while len(got) < len(reqs):
            for d in srv.progress(5000):
                assert d["status"] == 0, d["message"]
                r = reqs[d["tag"]]
                got[r.rid] = srv.take_range(r.rid) if r.kind == "range" else srv.take_triple(r.rid)
            info = srv.info()
            assert info["active"] <= 2
            seen_waiting = max(seen_waiting, info["waiting"])
    assert seen_waiting > 10
    for r in reqs:
        _check_same(search, r, got[r.rid])


def test_slot_overflow_reruns_the_query(search):
    """A quota far below the query's hits: the query is re-admitted with larger buffers."""
    with Server(search, hits_floor=1, hits_per_1e6_S=1, step_S=1 << 24) as srv:
        srv.submit_range(7, 10 ** 9, 10 ** 9 + 5 * 10 ** 7)
        srv.submit_triple(8, (960000, 1290000, 1600000), 10 ** 12)
        done = []
        while len(done) < 2:
            done += srv.progress(100000)
        d = {x["tag"]: x for x in done}
        assert d[7]["reruns"] >= 1 and d[7]["steps"] >= 3
        got = srv.take_range(7)
        tri = srv.take_triple(8)
    want = search.range(10 ** 9, 10 ** 9 + 5 * 10 ** 7)
    assert len(want.lines) > 100
    assert got.lines == want.lines
    assert_stats_equal(got.stats, want.stats)
    ext, state, st = search.extend_triples([(960000, 1290000, 1600000)], 10 ** 12)
    assert tri == (ext[0], int(state[0]), st)


def test_query_errors_match_alone():
    with Search(10 ** 7, cap_reps=2) as s:
        with pytest.raises(Ps4Error) as alone:
            s.range(1, 10 ** 7)
        with Server(s, hbm_budget=1 << 30, step_S=1 << 22) as srv:
            srv.submit_range(1, 1, 10 ** 7)
            srv.submit_range(2, 5, 5)
            srv.submit_triple(3, (6, 19, 30), 10 ** 6)
            done = {}
            while len(done) < 3:
                for d in srv.progress(100000):
                    done[d["tag"]] = d
            assert done[1]["status"] == alone.value.code == _abi.PS4_ERR_CAP_REPS
            assert done[1]["message"] == alone.value.message
            with pytest.raises(Ps4Error) as e:
                srv.take_range(1)
            assert e.value.message == alone.value.message
            empty = srv.take_range(2)
            assert empty.lines == [] and empty.stats["S_done"] == 0
            ext, state, st = srv.take_triple(3)
        e3, s3, t3 = s.extend_triples([(6, 19, 30)], 10 ** 6)
        assert (ext, state, st) == (e3[0], int(s3[0]), t3)


def test_submit_checks(search):
    with Server(search, hbm_budget=1 << 30, step_S=1 << 22) as srv:
        with pytest.raises(Ps4Error):
            srv.submit_range(1, 10, 3 * 10 ** 12)
        srv.submit_range(1, 10, 20)
        with pytest.raises(Ps4Error):
            srv.submit_range(1, 10, 20)                      # tag in use
        with pytest.raises(Ps4Error):
            srv.submit_triple(2, (1, 2, 3), 2 ** 63)         # dmax too large
        srv.submit_triple(3, (1, 2, 3), 100)                 # not a triple: state 1
        done = []
        while len(done) < 2:
            done += srv.progress(100000)
        assert srv.take_triple(3) == ([], 1, {"triples": 0, "invalid": 1, "ext_cand": 0, "ext_sqrt": 0, "exts": 0})
        r = srv.take_range(1)
        assert r.stats == search.range(10, 20).stats
