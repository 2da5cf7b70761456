"""The autotuner's host logic on the CPU: the coordinate search of tune_batch
over (product chunk, CTAs per SM, work items per claim) with a stand-in for the
CUDA-event timing (the chunk only for CUDA-core products), and the NTT
variant table against the header."""
import os
import re

from lzx_b200 import tune

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


class FakeBatch:
    PRODUCTS_INT64, PRODUCTS_TENSOR = 0, 1

    def __init__(self, products=0):
        self.configs = []
        self.checked = 0
        self.products = products

    def set_config(self, chunk, ctas, claim):
        self.configs.append((chunk, ctas, claim))

    @property
    def config(self):
        return self.configs[-1] if self.configs else (4096, 2, 1)

    def check(self):
        self.checked += 1


def run_search(cost, monkeypatch, products=0):
    batch = FakeBatch(products)
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


def test_tensor_products_skip_the_chunk_search(monkeypatch):
    """With the products on the tensor cores the chunk shapes nothing, so only
    the CTAs per SM and the claim size are searched, at the current chunk."""
    def cost(cfg):
        chunk, ctas, claim = cfg
        return abs(ctas - 4) + (0.5 if claim == 1 else 0.0) + 1.0

    batch, best, timings = run_search(cost, monkeypatch, products=FakeBatch.PRODUCTS_TENSOR)
    assert best == (4096, 4, 4)
    assert {c[0] for c in batch.configs} == {4096}
    assert len(timings) == len(tune.BATCH_CTAS) + len(tune.BATCH_CLAIMS) - 1
