"""Host logic of the serving tile autotuner (no GPU)."""

from ddg_b200.autotune import CANDIDATES, Tile, TileAutotuner, bucket


def test_bucket():
    assert bucket(1) == 0 and bucket(2) == 1 and bucket(1000) == 10 and bucket(1024) == 10 and bucket(1025) == 11


def test_explores_every_candidate_then_keeps_the_fastest(tmp_path):
    t = TileAutotuner(trials=2)
    seen = []
    fast = Tile(256, 1, 4)
    for _ in range(2 * len(CANDIDATES)):
        c = t.choose("N3", 5000)
        seen.append(c)
        t.record("N3", 5000, c, 1e-6 if c == fast else 2e-6)
    assert set(seen) == set(CANDIDATES)
    assert t.choose("N3", 5000) == fast and t.choose("N3", 6000) == fast      # same bucket
    assert t.choose("N3", 100) in CANDIDATES and ("N3", bucket(100)) not in t.best
    p = tmp_path / "tiles.json"
    t.save(str(p))
    u = TileAutotuner()
    u.load(str(p))
    assert u.choose("N3", 5000) == fast
