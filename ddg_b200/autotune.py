"""Tile-shape autotuner of the serving pools.

Each solve pool (one polynomial degree) runs its block-Jacobi PCG iterations
as captured graphs of element kernels whose tile shape is a free choice:
threads per block (64, 128, 256), one thread per element or a persistent
grid of a few blocks per SM, and how many CG iterations one graph launch
runs (``pairs``: 2 x pairs iterations).  The best shape depends on the
degree and vector precision (registers and work per element) and on how
many elements are packed in the pool, so the tuner keys its choice on (pool
kind, element-count bucket) with power-of-two buckets; a pool kind is a
short string such as ``"N3"`` or ``"N3-fp32"``.

Tuning is online: the first launches of a new key try every candidate
``trials`` times, each timed with CUDA events on the pool's stream and
normalised to seconds per CG iteration; afterwards the fastest (median)
candidate is used for that key.  No candidate changes any arithmetic, so a
request's iterates are the same whatever the tuner picks.  The table can be
saved to and loaded from a JSON file.

Extension: the reference has no serving layer.
"""

from __future__ import annotations

import json
import math
from dataclasses import dataclass


@dataclass(frozen=True)
class Tile:
    threads: int
    persistent: int
    pairs: int


CANDIDATES = tuple(Tile(t, p, k) for t in (64, 128, 256) for p in (0, 1) for k in (2, 4))


def bucket(elements: int) -> int:
    """Power-of-two bucket of a pool's active element count."""
    return max(0, int(math.ceil(math.log2(max(int(elements), 1)))))


class TileAutotuner:
    def __init__(self, candidates=CANDIDATES, trials: int = 2):
        self.candidates = tuple(candidates)
        self.trials = int(trials)
        self._times: dict = {}   # (kind, bucket) -> {Tile: [seconds per iteration]}
        self.best: dict = {}     # (kind, bucket) -> Tile

    def choose(self, kind: str, elements: int) -> Tile:
        key = (str(kind), bucket(elements))
        if key in self.best:
            return self.best[key]
        seen = self._times.setdefault(key, {})
        for c in self.candidates:
            if len(seen.get(c, ())) < self.trials:
                return c
        best = min(self.candidates, key=lambda c: sorted(seen[c])[len(seen[c]) // 2])
        self.best[key] = best
        return best

    def record(self, kind: str, elements: int, tile: Tile, seconds_per_iteration: float) -> None:
        key = (str(kind), bucket(elements))
        if key in self.best:
            return
        self._times.setdefault(key, {}).setdefault(tile, []).append(float(seconds_per_iteration))

    def table(self) -> dict:
        """{"kind/bucket": {"threads", "persistent", "pairs"}} of the settled keys."""
        return {f"{n}/{b}": {"threads": t.threads, "persistent": t.persistent, "pairs": t.pairs}
                for (n, b), t in sorted(self.best.items())}

    def save(self, path: str) -> None:
        with open(path, "w") as f:
            json.dump(self.table(), f, indent=1, sort_keys=True)

    def load(self, path: str) -> None:
        with open(path) as f:
            for k, v in json.load(f).items():
                n, b = k.rsplit("/", 1)
                self.best[(n, int(b))] = Tile(int(v["threads"]), int(v["persistent"]), int(v["pairs"]))
