"""The launch-shape autotuner's search and cache (host logic, no GPU): block
shapes are timed with one particle per thread, then the particle counts at
the winning shape; the winner is applied and cached with its particle count,
and a cache entry without one is re-tuned."""
import pytest

from at_b200 import autotune


@pytest.fixture
def cache(monkeypatch):
    """An in-memory tuning cache (the tests write no file)."""
    store = {}
    monkeypatch.setattr(autotune, "_load_cache", lambda: dict(store))
    monkeypatch.setattr(autotune, "_store_cache", lambda c: store.update(c))
    return store


class FakeEngine:
    def __init__(self):
        self.calls = []
        self.shape = None

    def set_launch(self, threads=0, seg_cap_words=0, particles_per_thread=0, **kw):
        self.shape = (threads, seg_cap_words, particles_per_thread)
        self.calls.append(self.shape)


def _sample(eng, cost):
    def run():
        return cost(*eng.shape)
    return run


def test_two_phase_search_and_cache(cache):
    eng = FakeEngine()

    def cost(t, c, k):              # best block shape 256 x 4096; two per thread better
        return abs(t - 256) / 100 + abs(c - 4096) / 1000 + (0.5 if k == 1 else 0.4)

    t, c, k, timings = autotune.tune(eng, _sample(eng, cost), key="dev|x")
    assert (t, c, k) == (256, 4096, 2)
    assert eng.shape == (256, 4096, 2)
    shapes = {s for s in eng.calls}
    # every block shape once with one particle per thread, then the particle
    # counts at the winner only
    assert {s for s in shapes if s[2] == 1} >= {(tt, cc, 1) for tt in autotune.THREADS
                                                  for cc in autotune.SEG_CAPS}
    assert {s for s in shapes if s[2] == 2} == {(256, 4096, 2)}
    assert len(timings) == len(autotune.THREADS) * len(autotune.SEG_CAPS) + 1
    assert cache["dev|x"]["ppt"] == 2 and cache["dev|x"]["threads"] == 256

    eng2 = FakeEngine()
    t2, c2, k2, info = autotune.tune(eng2, _sample(eng2, cost), key="dev|x")
    assert (t2, c2, k2) == (256, 4096, 2) and info == {"cached": True}
    assert eng2.calls == [(256, 4096, 2)]


def test_cache_entry_without_particle_count_is_retuned(cache):
    cache["dev|y"] = {"threads": 128, "seg_cap": 3072, "seconds": 1.0}
    eng = FakeEngine()
    t, c, k, info = autotune.tune(eng, _sample(eng, lambda t, c, k: t + c + k), key="dev|y")
    assert info != {"cached": True} and (t, c, k) == (128, 3072, 1)


def test_explicit_candidates_and_failures(cache):
    eng = FakeEngine()

    def cost(t, c, k):
        if t == 512:
            raise RuntimeError("launch configuration does not fit on an SM")
        return t

    t, c, k, timings = autotune.tune(eng, _sample(eng, cost), candidates=[(512, 3072),
                                                                          (128, 6144, 2)])
    assert (t, c, k) == (128, 6144, 2) and timings["512x3072x1"] == float("inf")
