"""The bench's algorithmic byte count (the roofline's numerator), on CPU."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402

N, NB, V, K = 244_819, 825_618, 11, 10


def test_all_active_count_of_the_large_field():
    # k (89 n + 17 n_b) + n (9 V + 64) + 50 n_b
    assert bench.algorithmic_bytes_per_frame(N, NB, V, K) == 439_430_367


def test_frozen_elements_carry_their_state_over_at_49_bytes_once_per_frame():
    full = bench.algorithmic_bytes_per_frame(N, NB, V, K)
    frozen = bench.algorithmic_bytes_per_frame(N, NB, V, K, n_act=0, nb_act=0)
    assert full - frozen == K * (89 * N + 17 * NB) - 49 * N
    # in place (frames after the first of a call) they carry nothing over
    inplace = bench.algorithmic_bytes_per_frame(N, NB, V, K, n_act=0, nb_act=0, in_place=True)
    assert frozen - inplace == 49 * N
    assert inplace == N * (9 * V + 64) + 50 * NB


def test_active_counts_on_cpu_tensors():
    torch = __import__("torch")
    act = torch.tensor([True, False, False, True, False])
    bi = torch.tensor([0, 1, 2], dtype=torch.int32)
    bj = torch.tensor([1, 2, 4], dtype=torch.int32)
    assert bench.active_counts(act, bi, bj) == (2, 1)


def test_reference_arm_slabs_cover_the_field_once():
    import numpy as np
    sizes = bench.field_slabs(N, 16)
    assert sum(sizes) == N and max(sizes) - min(sizes) <= 1
    order = np.argsort(np.random.default_rng(0).random(N), kind="stable")
    parts = np.array_split(order, 16)
    assert sorted(np.concatenate(parts).tolist()) == list(range(N))


def test_reference_arm_runs_the_whole_small_field_on_cpu():
    """bench.py --impl reference on the small field: every element of the field
    is stepped, as one slab per process, and the line carries the reference
    arm's keys."""
    import argparse
    args = argparse.Namespace(config="small", seed=0, steps=2, warmup=3, horizon=64)
    line = bench.run_reference(args)
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "elem-steps/s"
    cfg = line["config"]
    assert cfg["elements"] == sum(cfg["elements_per_process"]) == bench.load_field("small", 0).n
    assert line["cpu_baseline"]["cores"] == cfg["processes"] and line["e2e"]["h2d_bytes_per_step"] == 0
