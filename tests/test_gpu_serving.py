"""Continuous-batching pool: every request's result is the same alone and in
any mix (bit-identical: per-request reductions never mix), and matches the
one-at-a-time float64 solve within its tolerance."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _engine(**kw):
    from ddg_b200 import serving
    return serving.ServingEngine(degrees=(2, 3, 4), capacity=200_000, max_requests=64, max_request_K=2 * 40 * 40,
                                 pairs=2, **kw)


def test_each_result_same_alone_and_in_the_mix():
    from ddg_b200 import serving
    reqs = serving.make_requests(count=12, seed=3, n_range=(6, 40))
    eng = _engine()
    alone = {}
    for r in reqs[:4]:                                # each alone
        rr = serving.make_requests(count=12, seed=3, n_range=(6, 40))[r.rid]
        alone[r.rid] = eng.run([rr], realtime=False)[0]
    mix = {r.rid: r for r in eng.run(serving.make_requests(count=12, seed=3, n_range=(6, 40)), realtime=False)}
    for rid, a in alone.items():
        b = mix[rid]
        assert a.status == b.status == "converged"
        assert a.iterations == b.iterations
        assert np.array_equal(a.x, b.x)               # bit-identical
    eng.close()


def test_staggered_arrivals_admitted_while_others_iterate():
    from ddg_b200 import serving
    reqs = serving.make_requests(count=24, rate=400.0, seed=5, n_range=(6, 40))
    eng = _engine()
    done = eng.run(reqs, realtime=True)
    assert len(done) == 24 and all(r.status == "converged" for r in done)
    # some request was admitted while an earlier one was still on the GPU
    overlap = any(b.admitted < a.done and b.admitted > a.admitted for a in done for b in done if a is not b)
    assert overlap
    # results agree with the one-at-a-time float64 solve within the tolerance
    base, _ = serving.solve_one_at_a_time(sorted(done, key=lambda r: r.rid)[:6])
    for r, (u, info) in zip(sorted(done, key=lambda r: r.rid)[:6], base):
        assert np.linalg.norm(r.x - u) <= 20 * r.tol * max(np.linalg.norm(u), 1e-30)
    eng.close()


def test_autotuned_tiles_give_identical_results():
    """The autotuner tries every tile shape (threads per block, persistent
    grid, iterations per graph) on live launches and settles per (degree,
    element-count bucket); results are bit-identical to a fixed tile."""
    from ddg_b200 import serving
    from ddg_b200.autotune import CANDIDATES, TileAutotuner
    tuner = TileAutotuner(trials=1)
    eng_t = _engine(autotune=tuner)
    eng_f = _engine(autotune=False)
    tuned = {r.rid: r for r in eng_t.run(serving.make_requests(count=16, seed=7, n_range=(6, 40)),
                                         realtime=False)}
    fixed = {r.rid: r for r in eng_f.run(serving.make_requests(count=16, seed=7, n_range=(6, 40)),
                                         realtime=False)}
    for rid, a in fixed.items():
        b = tuned[rid]
        assert a.status == b.status == "converged" and a.iterations == b.iterations
        assert np.array_equal(a.x, b.x)
    tried = {t for times in tuner._times.values() for t in times}
    assert len(tried) >= len(CANDIDATES) // 2      # exploration covered the candidates
    eng_t.close()
    eng_f.close()


def test_fp32_pool_requests_reach_their_tolerance():
    """Requests with tol 1e-6 run in the float32 pools (float32 vectors,
    float64 reductions); their solutions agree with float64 one-at-a-time
    solves to the tolerance's order, and mixed float32/float64 traffic keeps
    each result identical to its run alone."""
    from ddg_b200 import serving
    reqs = serving.make_requests(count=10, seed=11, n_range=(6, 32), tols=(1e-6,))
    eng = _engine()
    done = sorted(eng.run(reqs, realtime=False), key=lambda r: r.rid)
    assert all(r.status == "converged" for r in done)
    assert all(eng.pools[(r.N, True)] is not None for r in done)
    base, _ = serving.solve_one_at_a_time(done[:5])
    for r, (u, info) in zip(done[:5], base):
        assert np.linalg.norm(r.x - u) <= 50 * r.tol * np.linalg.norm(u)
    alone = eng.run([serving.make_requests(count=10, seed=11, n_range=(6, 32), tols=(1e-6,))[0]],
                    realtime=False)[0]
    assert np.array_equal(alone.x, done[0].x) and alone.iterations == done[0].iterations
    eng.close()
