"""The autotuner's host logic on the CPU: the coordinate search of tune_batch
over (product chunk, CTAs per SM, work items per claim) with a stand-in for the
CUDA-event timing, and the NTT variant table against the header."""
import os
import re

from lzx_b200 import tune

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


class FakeBatch:
    def __init__(self):
        self.configs = []
        self.checked = 0

    def set_config(self, chunk, ctas, claim):
        self.configs.append((chunk, ctas, claim))

    def check(self):
        self.checked += 1


def run_search(cost, monkeypatch):
    batch = FakeBatch()
    monkeypatch.setattr(tune, "_time_batch", lambda b, reps: cost(b.configs[-1]))
    best, timings = tune.tune_batch(batch)
    return batch, best, timings


def test_search_follows_each_coordinate(monkeypatch):
    # best chunk 4096 at 2 CTAs/SM, then 3 CTAs/SM, then claims of 4
    def cost(cfg):
        chunk, ctas, claim = cfg
        return abs(chunk - 4096) / 1024 + abs(ctas - 3) + (0.5 if claim == 1 else 0.0) + 1.0

    batch, best, timings = run_search(cost, monkeypatch)
    assert best == (4096, 3, 4)
    assert batch.configs[-1] == best and batch.checked == 1  # the winner is left on the batch
    # each configuration timed once: 5 chunks + 3 new CTA counts + 1 new claim size
    assert len(timings) == len(tune.BATCH_CHUNKS) + len(tune.BATCH_CTAS) - 1 + len(tune.BATCH_CLAIMS) - 1
    assert timings["4096/3/4"] == min(timings.values())
    assert all(re.fullmatch(r"\d+/\d/\d", k) for k in timings)


def test_search_keeps_defaults_when_they_win(monkeypatch):
    def cost(cfg):
        return 1.0 if cfg == (1024, 2, 1) else 2.0

    batch, best, _ = run_search(cost, monkeypatch)
    assert best == (1024, 2, 1) and batch.configs[-1] == best


def test_variant_table_matches_header():
    src = open(os.path.join(ROOT, "include", "lattice_cuda.h")).read()
    n = int(re.search(r"#define\s+LC_NTT_NUM_VARIANTS\s+(\d+)", src).group(1))
    assert tune.NUM_VARIANTS == n
    assert sorted(tune.VARIANT_SHAPES) == list(range(n))
