"""Constructor (cbm_mkl_cpp.init / cbm_build) against the oracle's restatement of
cbm_init_ (cbm/cbm_extensions.cpp:60-345).  CPU only.

Pinned, for every case:
  * the candidate list: the tree uses only candidate edges of the reference's
    rules, and the prefix-filtered search equals the exhaustive one;
  * optimality: the tree's cost equals the optimum found by an independent
    Chu-Liu/Edmonds over the oracle's candidate list;
  * the six output arrays equal, bit for bit, the oracle's BFS emission for the
    same tree (children visited in candidate order);
  * the delta matrix plus tree reconstructs A exactly.
"""
import numpy as np
import pytest
import torch

from conftest import chain_graph, near_dup_graph, random_graph


def _check_structure(edge_index, n, alpha, oracle_mod, exhaustive_too=True):
    from cbm import cbm_mkl_cpp

    s = cbm_mkl_cpp.build(edge_index[0], edge_index[1], n, alpha)
    parent = s.parent
    (dr, dc, dv, br, src, dst), (f, t, w) = oracle_mod.reference_structure(edge_index, n, alpha, parent)
    np.testing.assert_array_equal(s.delta_row, dr)
    np.testing.assert_array_equal(s.delta_col, dc)
    np.testing.assert_array_equal(s.delta_val, dv)
    np.testing.assert_array_equal(s.branches, br)
    np.testing.assert_array_equal(s.src, src)
    np.testing.assert_array_equal(s.dst, dst)
    # candidates without the n virtual edges
    assert s.n_candidates == f.size - n
    # optimality
    opt = oracle_mod.arborescence_cost(n + 1, n, f, t, w)
    assert s.tree_cost == opt
    assert s.tree_cost == s.delta_val.size  # edge weight = delta entries of the child
    # exact reconstruction: CBM product with integer X equals A X in fp64
    ptr, idx = oracle_mod.csr_from_edges(edge_index, n)
    rng = np.random.default_rng(0)
    x = rng.integers(-3, 4, size=(n, 3)).astype(np.float64)
    y = np.zeros((n, 3))
    np.add.at(y, s.delta_row, s.delta_val[:, None].astype(np.float64) * x[s.delta_col])
    for u, v in zip(s.src, s.dst):
        y[v] += y[u]
    np.testing.assert_array_equal(y, oracle_mod.dense_f64(ptr, idx, n, x))
    if exhaustive_too:
        s2 = cbm_mkl_cpp.build(edge_index[0], edge_index[1], n, alpha, exhaustive=True)
        for f_ in ("delta_row", "delta_col", "delta_val", "branches", "src", "dst"):
            np.testing.assert_array_equal(getattr(s, f_), getattr(s2, f_))
    return s


@pytest.mark.parametrize("alpha", [0, 2, 8, -3])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_random_symmetric(alpha, seed, oracle_mod):
    ei = random_graph(300, 6, seed)
    _check_structure(ei, 300, alpha, oracle_mod)


@pytest.mark.parametrize("alpha", [0, 4])
def test_near_duplicates(alpha, oracle_mod):
    ei = near_dup_graph(400, seed=5, deg=12)
    s = _check_structure(ei, 400, alpha, oracle_mod)
    assert s.src.size > 50  # the copies hang below their templates


def test_directed_with_isolated_and_self_loops(oracle_mod):
    ei = random_graph(250, 5, 7, symmetric=False, self_loops=True, isolated=20)
    n = 250
    _check_structure(ei, n, 0, oracle_mod)


def test_chain(oracle_mod):
    ei, n = chain_graph(40)
    s = _check_structure(ei, n, 0, oracle_mod)
    # one branch, a chain 0 -> 1 -> ... -> 39
    assert s.branches.tolist() == [0, 39]
    assert s.src.tolist() == list(range(39))
    assert s.dst.tolist() == list(range(1, 40))


def test_community_4096_matches_oracle(oracle_mod):
    from cbm.synthetic import workload

    ei, n, spec = workload("community-4096")
    # brute-force candidates over 4096 rows are still quick in C
    _check_structure(ei, n, spec["alpha"], oracle_mod, exhaustive_too=True)


def test_hand_checked_example():
    """Rows 0 and 1 are identical, row 2 is row 0 plus one column.

    A (4 x 4, no self loops):  0: {2, 3}   1: {2, 3}   2: {0, 1, 3}   3: {0, 1, 2}
    syrk pairs: (0,1) o=2 h=0 -> both directions; (0,2) o=1 h=3; (0,3) o=1 h=3;
    (1,2),(1,3) o=1 h=3; (2,3) o=2 h=2.  With alpha = 0 the candidates are
    (1->0, 0), (0->1, 0), (3->2, 2), (2->3, 2) (h=3 fails h < nnz - alpha for
    nnz 2, and for nnz 3 h != nnz fails).  G order (virtual edges first per row):
      0:(4->0,2) 1:(1->0,0) 2:(0->1,0) 3:(4->1,2) 4:(4->2,3) 5:(3->2,2) 6:(2->3,2) 7:(4->3,3)
    Optimum 2 + 0 + 3 + 2 = 7 with ties: 0 root + 0->1, or 1 root + 1->0 (the
    contraction of the 2-cycle {0, 1} picks its entering edge 4->0 (index 0)
    before 4->1 (index 3): ties go to the lower candidate index); likewise {2,3}:
    4->2 (index 4, weight 3) or 4->3 (index 7, weight 3) -> 4->2.
    Tree: roots 0 and 2; edges 0->1 and 2->3; branches [0, 1, 2].
    Delta: row 0 = {2, 3} (+1), row 2 = {0, 1, 3} (+1), row 1 = A1 - A0 = {},
    row 3 = A3 - A2: +2, -3.
    """
    from cbm import cbm_mkl_cpp

    ei = torch.tensor([[0, 0, 1, 1, 2, 2, 2, 3, 3, 3], [2, 3, 2, 3, 0, 1, 3, 0, 1, 2]], dtype=torch.int32)
    out = cbm_mkl_cpp.init(ei[0], ei[1], torch.ones(10), 4, 0)
    dr, dc, dv, br, src, dst = [o.tolist() for o in out]
    assert dr == [0, 0, 2, 2, 2, 3, 3]
    assert dc == [2, 3, 0, 1, 3, 2, 3]
    assert dv == [1, 1, 1, 1, 1, 1, -1]
    assert br == [0, 1, 2]
    assert src == [0, 2]
    assert dst == [1, 3]
    assert [o.dtype for o in out] == [torch.int32, torch.int32, torch.float32, torch.int32, torch.int32,
                                      torch.int32]


def test_init_dtype_checks():
    from cbm import cbm_mkl_cpp

    ei = torch.tensor([[0, 1], [1, 0]], dtype=torch.int64)
    with pytest.raises(RuntimeError):
        cbm_mkl_cpp.init(ei[0], ei[1], torch.ones(2), 2, 0)
    ei = ei.to(torch.int32)
    with pytest.raises(RuntimeError):
        cbm_mkl_cpp.init(ei[0], ei[1], torch.ones(2, dtype=torch.float64), 2, 0)
    out = cbm_mkl_cpp.init(ei[0], ei[1], torch.ones(2), 2, 0)
    assert len(out) == 6


def test_out_of_range_index_rejected():
    from cbm import cbm_mkl_cpp

    ei = torch.tensor([[0, 5], [1, 0]], dtype=torch.int32)
    with pytest.raises(RuntimeError, match="index out of range"):
        cbm_mkl_cpp.init(ei[0], ei[1], torch.ones(2), 3, 0)


def test_duplicate_edges_are_merged(oracle_mod):
    ei = random_graph(100, 4, 3)
    dup = np.concatenate([ei, ei[:, :50]], axis=1)
    from cbm import cbm_mkl_cpp

    a = cbm_mkl_cpp.build(ei[0], ei[1], 100, 0)
    b = cbm_mkl_cpp.build(dup[0], dup[1], 100, 0)
    np.testing.assert_array_equal(a.delta_col, b.delta_col)
    np.testing.assert_array_equal(a.src, b.src)


def test_empty_rows_only():
    from cbm import cbm_mkl_cpp

    # one edge, the rest of the rows empty
    s = cbm_mkl_cpp.build(np.array([0], np.int32), np.array([3], np.int32), 6, 0)
    assert s.delta_row.tolist() == [0] and s.delta_col.tolist() == [3]
    assert s.src.size == 0 and s.branches.tolist() == [0]
    assert s.csr_ptr.tolist() == [0, 1, 1, 1, 1, 1, 1]


def test_csr_form_is_coalesced_coo():
    """The CSR arrays equal what torch's coalesce + to_sparse_csr gives (cbm/cbm4mm.py:26-37)."""
    from cbm import cbm_mkl_cpp

    ei = near_dup_graph(300, seed=2)
    s = cbm_mkl_cpp.build(ei[0], ei[1], 300, 0)
    coo = torch.sparse_coo_tensor(torch.from_numpy(np.stack([s.delta_row, s.delta_col])),
                                  torch.from_numpy(s.delta_val), (300, 300)).coalesce().to_sparse_csr()
    np.testing.assert_array_equal(coo.crow_indices().numpy(), s.csr_ptr)
    np.testing.assert_array_equal(coo.col_indices().numpy(), s.csr_col)
    np.testing.assert_array_equal(coo.values().numpy(), s.csr_val)


@pytest.mark.parametrize("threads", [1, 3])
def test_thread_count_does_not_change_output(threads):
    from cbm import cbm_mkl_cpp

    ei = near_dup_graph(500, seed=9)
    a = cbm_mkl_cpp.build(ei[0], ei[1], 500, 2, n_threads=threads)
    b = cbm_mkl_cpp.build(ei[0], ei[1], 500, 2, n_threads=0)
    for f in ("delta_row", "delta_col", "delta_val", "branches", "src", "dst"):
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f))


def test_structure_cache_round_trip(tmp_path):
    """The on-disk structure cache returns exactly what the constructor built,
    keyed by the edge list and alpha."""
    from cbm import cbm_mkl_cpp
    from conftest import near_dup_graph

    ei = near_dup_graph(700, seed=9)
    s0 = cbm_mkl_cpp.build(ei[0], ei[1], 700, 2)
    s1 = cbm_mkl_cpp.build_cached(ei[0], ei[1], 700, 2, cache_dir=str(tmp_path))
    s2 = cbm_mkl_cpp.build_cached(ei[0], ei[1], 700, 2, cache_dir=str(tmp_path))  # from the file
    files = list(tmp_path.iterdir())
    assert len(files) == 1
    for s in (s1, s2):
        for f in ("delta_row", "delta_col", "delta_val", "branches", "src", "dst", "parent", "csr_ptr", "csr_col",
                  "csr_val"):
            np.testing.assert_array_equal(getattr(s, f), getattr(s0, f))
        assert (s.n, s.tree_cost, s.nnz_a, s.n_candidates) == (s0.n, s0.tree_cost, s0.nnz_a, s0.n_candidates)
    # another alpha is another entry
    s3 = cbm_mkl_cpp.build_cached(ei[0], ei[1], 700, 0, cache_dir=str(tmp_path))
    assert len(list(tmp_path.iterdir())) == 2
    np.testing.assert_array_equal(s3.csr_col, cbm_mkl_cpp.build(ei[0], ei[1], 700, 0).csr_col)
    # a file of another format or key is ignored
    assert cbm_mkl_cpp.load_structure(str(files[0]), key="other") is None


def test_coalesced_and_shuffled_inputs_give_the_same_structure():
    """Coalesced COO takes the constructor's direct CSR path; the same edges
    shuffled (and with duplicates) take the sorting path: same structure."""
    from cbm import cbm_mkl_cpp
    from conftest import near_dup_graph

    ei = near_dup_graph(900, seed=14)
    s0 = cbm_mkl_cpp.build(ei[0], ei[1], 900, 3)
    perm = np.random.default_rng(0).permutation(ei.shape[1])
    dup = np.concatenate([perm, perm[:200]])
    s1 = cbm_mkl_cpp.build(np.ascontiguousarray(ei[0][dup]), np.ascontiguousarray(ei[1][dup]), 900, 3)
    for f in ("csr_ptr", "csr_col", "csr_val", "branches", "src", "dst", "parent"):
        np.testing.assert_array_equal(getattr(s0, f), getattr(s1, f))
    assert s0.nnz_a == s1.nnz_a == ei.shape[1]
