"""start(nodeList, edgeList, part_init): the reference's Python entry point
(LouvainCPP.cpp:808-951) over liblvg -- id mapping and argument checks on the
CPU, the returned partition against the oracle on the GPU."""
import numpy as np
import pytest

from louvaingpu_b200 import compat


def dict_lists(n, s, d, w, ids):
    nodes = [{"id": int(ids[i])} for i in range(n)]
    edges = [{"source": int(ids[a]), "target": int(ids[b]), "weight": float(x)} for a, b, x in zip(s, d, w)]
    return nodes, edges


def arbitrary_ids(n, seed=4):
    rng = np.random.default_rng(seed)
    return rng.permutation(np.arange(n) * 7 + 1000)


def test_lists_to_arrays_maps_ids_in_list_order(gen):
    n, s, d, w = gen.sbm(300, 3, 0.1, 0.01, 1, 4, seed=1)
    ids = arbitrary_ids(n)
    nodes, edges = dict_lists(n, s, d, w, ids)
    got_ids, gs, gd, gw = compat.lists_to_arrays(nodes, edges)
    np.testing.assert_array_equal(got_ids, ids)
    np.testing.assert_array_equal(gs, s)
    np.testing.assert_array_equal(gd, d)
    np.testing.assert_array_equal(gw, w)


def test_lists_to_arrays_rejects_what_the_reference_reads_wrong():
    with pytest.raises(ValueError, match="listed twice"):
        compat.lists_to_arrays([{"id": 5}, {"id": 5}], [])
    with pytest.raises(ValueError, match="not in nodeList"):
        compat.lists_to_arrays([{"id": 5}, {"id": 6}], [{"source": 5, "target": 9, "weight": 1.0}])
    with pytest.raises(KeyError):
        compat.lists_to_arrays([{"id": 5}, {"id": 6}], [{"source": 5, "weight": 1.0}])
    with pytest.raises(KeyError):
        compat.lists_to_arrays([{"name": 5}], [])


def test_part_init_is_checked_and_renumbered_like_the_reference():
    got = compat.check_part_init([{"node": 3, "community": 40, "weight": 1.0}, {"node": 4, "community": 9, "weight": 2},
                                  {"node": 5, "community": 40, "weight": 0.5}])
    assert got == {3: (0, 1.0), 4: (1, 2.0), 5: (0, 0.5)}
    with pytest.raises(KeyError):
        compat.check_part_init([{"node": 3, "weight": 1.0}])


@pytest.mark.gpu
@pytest.mark.parametrize("quirk", [True, False])
def test_start_matches_the_oracle(gen, oracle, quirk):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from louvaingpu_b200 import start
    n, s, d, w = gen.sbm(3000, 30, 0.05, 0.002, 1, 4, seed=2)
    ids = arbitrary_ids(n)
    nodes, edges = dict_lists(n, s, d, w, ids)
    part_init = [{"node": int(ids[i]), "community": int(i % 5), "weight": 1.0} for i in range(n)]
    out = start(nodes, edges, part_init, reference_quirk=quirk)
    r = oracle.Run(n, s, d, w)
    assert len(r.levels) > 2          # the quirk and the last level differ here
    level = 1 if quirk else len(r.levels) - 1
    exp = r.partition(level)
    assert out["size"] == int(exp.max()) + 1
    assert [out[int(v)] for v in ids] == exp.tolist()
    assert [nd["cluster"] for nd in nodes] == exp.tolist()
    assert [nd["my_community"] for nd in nodes] == exp.tolist()


@pytest.mark.gpu
def test_start_without_edges_returns_singletons():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from louvaingpu_b200 import start
    nodes = [{"id": 10}, {"id": 20}, {"id": 30}]
    out = start(nodes, [], [])
    assert out == {"size": 3, 10: 0, 20: 1, 30: 2}
