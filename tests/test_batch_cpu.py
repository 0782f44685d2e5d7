"""Host-side tests of the uneven batch: the workload generator is
deterministic and spans the stated ranges, and xs_batch_create (host only)
groups items by generated kernel, sending lattices beyond shared memory to
the streaming path."""
import collections

import pytest

from xspde_matlab_b200 import batch


def test_uneven_instances_deterministic_and_in_range():
    a = batch.uneven_instances(64, seed=1)
    b = batch.uneven_instances(64, seed=1)
    c = batch.uneven_instances(64, seed=2)
    assert a == b and a != c
    full = batch.uneven_instances()
    assert len(full) == 512
    for inp in full:
        dim = inp["dimensions"] - 1
        N = inp["points"][1]
        assert dim in (1, 2)
        assert N in ((32, 64, 128, 256, 512, 1024) if dim == 1 else (32, 64, 128, 256))
        assert 0.001 <= inp["g"] <= 0.1
        assert 64 <= inp["ensembles"][0] <= 1024 and inp["ensembles"][0] % 64 == 0
        assert 50 // 4 <= inp["steps"] <= 2000 // 4 + 1
    kinds = collections.Counter((i["dimensions"], i["drift"]) for i in full)
    assert len(kinds) == 4 and min(kinds.values()) > 80


def test_batch_grouping_host_only():
    items = batch.uneven_instances(40, seed=3)
    b = batch.Batch(items, skip_unsupported=True)
    s = b.summary()
    assert s["items"] == len(b) == 40 - len(b.skipped)
    # every skipped item is a 2D 128 x 128 lattice (neither path covers it)
    assert all(items[k]["points"][1:] == [128, 128] for k in b.skipped)
    names = collections.defaultdict(set)
    for i in range(len(b)):
        inf = b.info(i)
        inp = items[b.index[i]]
        if inp["points"][1:] == [256, 256]:
            assert inf["path"] == 2
        else:
            assert inf["path"] == 1
            names[inf["variant"]].add(inp["name"])
    # one variant per (drift, dimension, lattice)
    assert all(len(v) == 1 for v in names.values())
    assert len(names) == len({items[b.index[i]]["name"] for i in range(len(b)) if b.info(i)["path"] == 1})


def test_batch_checks_and_block_rules():
    """checks = 1 items are accepted (both passes run in the graph; two pass
    results per item), checks > 1 and several ensemble blocks are refused."""
    from xspde_matlab_b200 import _lib
    items = batch.uneven_instances(2, seed=1)
    one = batch.Batch([items[0]])
    two = batch.Batch([dict(items[0], checks=1)])
    L = _lib.lib()
    assert L.xs_batch_av_doubles(two.h, 0) == 2 * L.xs_batch_av_doubles(one.h, 0) > 0
    bad = dict(items[0], checks=2)
    with pytest.raises(_lib.XsError, match="checks"):
        batch.Batch([bad])
    bad = dict(items[0], ensembles=[64, 2, 1])
    with pytest.raises(_lib.XsError, match="ensemble block"):
        batch.Batch([bad])
