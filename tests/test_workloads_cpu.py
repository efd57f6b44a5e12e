"""Host side of the benchmark workloads (no GPU): the seeded uneven problem
set of the batched run and the autotuner's candidate configurations."""
import numpy as np

from charming_b200.batch import default_candidates, uneven_set


def test_uneven_set_is_seeded_and_in_range():
    a, b = uneven_set(), uneven_set()
    assert [(p.nx, p.ny, p.bc) for p in a] == [(p.nx, p.ny, p.bc) for p in b]
    assert len(a) == 64
    sides = np.array([p.nx for p in a])
    assert all(p.nx == p.ny for p in a)
    assert sides.min() >= 64 and sides.max() <= 2048
    assert all(0.0 <= v < 1.0 for p in a for v in p.bc)
    assert all(p.max_sweeps == 500 and p.check_every == 0 for p in a)
    # log-uniform: about half the sides below the geometric mean of 64 and 2048
    assert 20 <= int((sides < np.sqrt(64 * 2048)).sum()) <= 44
    # the set the benchmark reports (seed 0xC3): 56.57 M interior points
    assert int((sides.astype(np.int64) ** 2).sum()) == 56566912
    assert [p.nx for p in uneven_set(seed=1)] != list(sides)


def test_autotune_candidates_are_valid_configs():
    cands = default_candidates()
    assert {c.chare_side for c in cands} == {64, 128, 256}
    assert {c.pes_per_sm for c in cands} == {1, 2, 4}
    for c in cands:
        cfg = c.runtime_config()
        assert cfg["threads_per_pe"] * cfg["pes_per_sm"] == 512
        ring = cfg["ring_bytes"]
        assert ring & (ring - 1) == 0
        assert cfg.get("max_msg_bytes", (1 << 20) + 64) <= ring // 2
