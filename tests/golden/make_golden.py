"""Generates tests/golden/reference_products.npz: outputs of the reference's own
GPU product path on small seeded graphs -- TEST INFRASTRUCTURE ONLY.

The products come from the reference modules compiled by oracle/build_ref.py
from the reference sources (cbm/cbm.cu: cusparseCBM.matmul_AX_ADX and
matmul_DAX_DADX; cbm/csr.cu: cusparseCSR.matmul) into oracle/_ref/.  Run on a
machine with a GPU:

    python oracle/build_ref.py            # once, where the reference sources are
    python tests/golden/make_golden.py [output.npz]

The reference constructor (cbm/cbm_extensions.cpp:60-345) needs Intel MKL and
the arbok submodule, neither available, so the structure handed to the
reference product is the one this library's constructor emits under the same
rules (cbm_mkl_cpp.build).  The fixture stores that structure, the inputs and
the reference's outputs, so the checks in tests/test_golden.py need neither a
GPU nor a rebuild:

* <case>/ei, n, alpha        edge list (int32 [2, nnz]), node count, alpha
* <case>/crow, col, sign     delta CSR (int32, int32, fp32 +-1)
* <case>/branches, src, dst  tree: branch offsets, BFS (parent, child) edges
* <case>/D                   d^-1/2, d = A 1 through the reference product
                             (cbm/cbm4ad.py:11-19)
* <case>/val_ad, val_dad     values as cbm4ad / cbm4dad prepare them
                             (cbm/cbm4ad.py:21-25, cbm/cbm4dad.py:21-34)
* <case>/x                   fp32 U(0,1) input (benchmark/compare_matmul_cuda.py:43)
* <case>/y_ax, y_adx, y_dadx reference CBM products of the three forms
* <case>/y_csr               reference CSR product A x (cusparseCSR)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(REPO, "cbm-gpu_b200"), REPO):
    if p not in sys.path:
        sys.path.insert(0, p)

# (name, builder, alpha, columns, scaled forms recorded)
def _cases():
    from cbm import synthetic

    def community():
        return synthetic.community_graph(512, 32, 10, 3, seed=11), 512

    def near_dup():
        rng = np.random.Generator(np.random.PCG64(12))
        ei = synthetic.community_graph(800, 32, 12, 2, rng=rng)
        return synthetic.near_duplicates(ei, 800, 0.4, 0.1, rng=rng), 800

    def powerlaw():
        return synthetic._w_powerlaw(1500, 2.1, 12.0, 0.3, 0.1, 13), 1500

    def isolated():
        # a near-duplicate graph whose ids 100..139 have no edges
        rng = np.random.Generator(np.random.PCG64(14))
        ei = synthetic.community_graph(560, 28, 10, 2, rng=rng)
        ei = synthetic.near_duplicates(ei, 560, 0.4, 0.1, rng=rng)
        return np.where(ei >= 100, ei + 40, ei).astype(np.int32), 600

    def chain():
        # row i = columns {n..n+i}: one long chain in the tree
        n = 64
        rows = np.concatenate([np.full(i + 1, i) for i in range(n)])
        cols = np.concatenate([np.arange(n, n + i + 1) for i in range(n)])
        return np.stack([rows, cols]).astype(np.int32), 2 * n

    # the chain's columns n..2n-1 are empty rows (degree 0, D = inf), so only
    # its unscaled product is recorded
    return [("community", community, 0, 8, True), ("near_dup", near_dup, 0, 12, True),
            ("near_dup_a4", near_dup, 4, 8, True), ("powerlaw", powerlaw, 2, 8, True),
            ("isolated", isolated, 0, 8, True), ("chain", chain, 0, 8, False)]


def generate(out_path):
    import torch

    from cbm import cbm_mkl_cpp
    from oracle import build_ref

    cbm_ref = build_ref.load("cbm_cusparse_ref")
    csr_ref = build_ref.load("csr_cusparse_ref")
    if cbm_ref is None or csr_ref is None:
        raise SystemExit("reference modules missing: run python oracle/build_ref.py first")
    dev = torch.device("cuda")
    out = {}
    for case, (name, builder, alpha, cols, scaled) in enumerate(_cases()):
        ei, n = builder()
        order = np.lexsort((ei[1], ei[0]))
        ei = np.ascontiguousarray(ei[:, order], dtype=np.int32)
        s = cbm_mkl_cpp.build(ei[0], ei[1], n, alpha)
        crow = torch.from_numpy(s.csr_ptr.astype(np.int32)).to(dev)
        col = torch.from_numpy(s.csr_col.astype(np.int32)).to(dev)
        sign = torch.from_numpy(s.csr_val.astype(np.float32)).to(dev)
        br = torch.from_numpy(s.branches.astype(np.int32)).to(dev)
        # the reference's update kernels read mca_branches one element past its
        # end; give that read an empty range (a view of a longer buffer)
        br_pad = torch.cat([br, br[-1:]])[: br.numel()]
        src = torch.from_numpy(s.src.astype(np.int32)).to(dev)
        dst = torch.from_numpy(s.dst.astype(np.int32)).to(dev)
        empty = torch.empty(0, device=dev)

        plain = cbm_ref.cusparseCBM(torch.sparse_csr_tensor(crow, col, sign, (n, n)), br_pad, src, dst, empty)
        d = torch.zeros(n, 1, device=dev)
        plain.matmul_AX_ADX(torch.ones(n, 1, device=dev), d)
        D = (d ** (-1 / 2)).view(-1)
        val_ad = sign * D[col.long()]
        rows = torch.repeat_interleave(torch.arange(n, device=dev), (crow[1:] - crow[:-1]).long())
        val_dad = val_ad * D[rows]

        g = torch.Generator(device=dev).manual_seed(1000 + case)
        x = torch.rand(n, cols, device=dev, generator=g)
        y_ax, y_adx, y_dadx, y_csr = (torch.empty(n, cols, device=dev) for _ in range(4))
        plain.matmul_AX_ADX(x, y_ax)
        ad = dad = None
        if scaled:
            ad = cbm_ref.cusparseCBM(torch.sparse_csr_tensor(crow, col, val_ad, (n, n)), br_pad, src, dst, empty)
            ad.matmul_AX_ADX(x, y_adx)
            dad = cbm_ref.cusparseCBM(torch.sparse_csr_tensor(crow, col, val_dad, (n, n)), br_pad, src, dst, D)
            dad.matmul_DAX_DADX(x, y_dadx)
        a_ptr = np.zeros(n + 1, np.int64)
        np.add.at(a_ptr, ei[0].astype(np.int64) + 1, 1)
        a_csr = torch.sparse_csr_tensor(torch.from_numpy(np.cumsum(a_ptr).astype(np.int32)).to(dev),
                                        torch.from_numpy(ei[1]).to(dev), torch.ones(ei.shape[1], device=dev), (n, n))
        csr = csr_ref.cusparseCSR(a_csr)
        csr.matmul(x, y_csr)
        torch.cuda.synchronize()
        arrays = dict(ei=ei, n=np.int64(n), alpha=np.int64(alpha), crow=crow, col=col, sign=sign, branches=br,
                      src=src, dst=dst, x=x, y_ax=y_ax, y_csr=y_csr)
        if scaled:
            arrays.update(D=D, val_ad=val_ad, val_dad=val_dad, y_adx=y_adx, y_dadx=y_dadx)
        for k, v in arrays.items():
            out[f"{name}/{k}"] = v.cpu().numpy() if torch.is_tensor(v) else v
        print(f"{name}: n={n} nnz={ei.shape[1]} Z={s.csr_col.size} E={s.src.size} B={s.branches.size - 1} C={cols}")
        del plain, ad, dad, csr
    os.makedirs(os.path.dirname(os.path.abspath(out_path)), exist_ok=True)
    np.savez_compressed(out_path, **out)
    print("wrote", out_path)


if __name__ == "__main__":
    generate(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "reference_products.npz"))
