"""Split of batched solves over several GPUs (gp5cu_batch_assign_devices), host side only.

Independent solves shard by index with no data exchanged between devices; the split is
longest-processing-time first by grid sites, so every device gets close to an equal share of
the work and the split is reproducible."""
import numpy as np
import pytest

from gp5_b200 import _abi


def _solves(ns, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(ns):
        n = int(rng.choice([32, 64, 128]))
        out.append(dict(n=n, L=10.0, N=100.0, dt=0.01))
    return out


@pytest.mark.parametrize("ns,ndev", [(1, 1), (5, 2), (64, 2), (64, 4), (63, 8), (3, 8)])
def test_split_is_a_balanced_deterministic_partition(ns, ndev):
    solves = _solves(ns, ns * 10 + ndev)
    pos = _abi.assign_devices(solves, ndev)
    assert pos == _abi.assign_devices(solves, ndev)
    assert len(pos) == ns and all(0 <= p < ndev for p in pos)
    load = np.zeros(ndev)
    for sd, p in zip(solves, pos):
        load[p] += sd["n"] ** 3
    biggest = max(sd["n"] ** 3 for sd in solves)
    if ns >= ndev:
        # LPT: no device carries more than the lightest one plus the largest single solve
        assert load.max() - load.min() <= biggest
    else:
        assert sorted(pos) == list(range(ns))  # one solve per device


def test_split_follows_the_lpt_rule():
    solves = [dict(n=n, L=8.0, N=50.0, dt=0.01) for n in (32, 128, 64, 128, 32, 64)]
    # order by sites: 128 (1), 128 (3), 64 (2), 64 (5), 32 (0), 32 (4); each to the lightest
    # device, ties to the lower position: 1->0, 3->1, 2->0, 5->1, 0->0, 4->1
    assert _abi.assign_devices(solves, 2) == [0, 0, 0, 1, 1, 1]


def test_split_rejects_bad_arguments():
    solves = _solves(4, 1)
    with pytest.raises(_abi.Gp5Error) as e:
        _abi.assign_devices(solves, 0)
    assert e.value.status == _abi.GP5_ERR_ARG
