"""Patch assembly tables (ensc_batch_prepare / ensc_prepared_patch_tables),
checked on the host against the mesh they were built from: the stored order
is a permutation; every (element, local slot) incidence belongs to exactly
one partial, and that partial is the one of the element's patch and node;
a partial lists its incidences in slot order; each node adds its partials in
patch order, one per patch that touches it.  On a structured block whose
sides are multiples of four the patches are 4x4x4 bricks (125 nodes each).
No GPU: the host part makes no CUDA call."""
import numpy as np
import pytest

from enscdynamics_b200 import capi
from enscdynamics_b200 import workloads as W


def tables(p, precision=capi.MIXED, assembly=capi.ASSEMBLY_PATCH):
    pr = capi.Prepared(p.mesh.x0, p.mesh.conn, p.v0, material=p.material, controls=p.controls,
                       precision=precision, assembly=assembly)
    try:
        info = pr.assembly
        t = pr.patch_tables() if info["assembly"] == capi.ASSEMBLY_PATCH else None
    finally:
        pr.close()
    return info, t


def check(p, t):
    conn = np.asarray(p.mesh.conn, dtype=np.int64)
    ne, nn = conn.shape[0], p.mesh.n_nodes
    stored = t["stored"]
    assert np.array_equal(np.sort(stored), np.arange(ne))
    order = np.empty(ne, dtype=np.int64)
    order[stored] = np.arange(ne)                      # stored position -> element
    pf, incf, inc = t["patch_first"], t["inc_first"], t["inc"]
    nfirst, nparts = t["node_first"], t["node_partials"]
    npatch = (ne + 63) // 64
    assert len(pf) == npatch + 1 and pf[0] == 0 and np.all(np.diff(pf) > 0)
    nq = pf[-1]
    assert incf[0] == 0 and incf[-1] == 8 * ne and np.all(np.diff(incf) > 0)
    # partial -> node, from the node lists
    assert nfirst[0] == 0 and nfirst[-1] == nq and len(nparts) == nq
    node_of = np.full(nq, -1, dtype=np.int64)
    for n in range(nn):
        qs = nparts[nfirst[n]:nfirst[n + 1]]
        assert np.all(np.diff(qs) > 0)                 # patch order
        node_of[qs] = n
    assert np.all(node_of >= 0)
    seen = np.zeros((ne, 8), dtype=np.int32)
    for pch in range(npatch):
        for q in range(pf[pch], pf[pch + 1]):
            ent = inc[incf[q]:incf[q + 1]].astype(np.int64)
            el, k = ent >> 3, ent & 7
            assert np.all(np.diff(k) > 0)              # slot order, one element per slot
            e = order[64 * pch + el]
            assert np.all(conn[e, k] == node_of[q])
            seen[e, k] += 1
    assert np.all(seen == 1)
    # one partial per (patch, node) pair
    patch_of = np.repeat(np.arange(npatch), np.diff(pf))
    pairs = set(zip(patch_of.tolist(), node_of.tolist()))
    assert len(pairs) == nq


def test_structured_block_patches_are_bricks():
    p = W.block(16, 8, 8, 0.16, 0.08, 0.08)
    info, t = tables(p)
    assert info["assembly"] == capi.ASSEMBLY_PATCH
    assert info["patches"] == 16 * 8 * 8 // 64
    check(p, t)
    assert np.all(np.diff(t["patch_first"]) == 125)


@pytest.mark.parametrize("dims", [(7, 5, 3), (13, 6, 9), (1, 1, 1)])
def test_uneven_blocks(dims):
    nx, ny, nz = dims
    p = W.block(nx, ny, nz, 0.01 * nx, 0.01 * ny, 0.01 * nz)
    info, t = tables(p)
    assert info["assembly"] == capi.ASSEMBLY_PATCH
    check(p, t)


def test_sweep_instance_and_unstructured_order():
    p = W.sweep_instance(3, seed=3, ne_min=150, ne_max=3000, cycles=10)
    info, t = tables(p)
    check(p, t)
    # a shuffled element numbering gives the same patches, up to the order
    rng = np.random.default_rng(1)
    perm = rng.permutation(p.mesh.n_elements)
    p2 = W.block(12, 6, 5, 0.12, 0.06, 0.05)
    base_info, _ = tables(p2)
    p2.mesh.conn = p2.mesh.conn[rng.permutation(p2.mesh.n_elements)]
    info2, t2 = tables(p2)
    check(p2, t2)
    assert info2["partials"] == base_info["partials"]
    del perm


def test_slot_assembly_where_patches_do_not_apply():
    p = W.block(4, 4, 4, 0.04, 0.04, 0.04)
    assert tables(p, precision=capi.FP64, assembly=capi.ASSEMBLY_AUTO)[0]["assembly"] == capi.ASSEMBLY_SLOT
    assert tables(p, assembly=capi.ASSEMBLY_AUTO)[0]["assembly"] == capi.ASSEMBLY_SLOT
    assert tables(p, assembly=capi.ASSEMBLY_SLOT)[0]["assembly"] == capi.ASSEMBLY_SLOT
    with pytest.raises(capi.EnscError, match="patch assembly"):
        tables(p, precision=capi.FP64, assembly=capi.ASSEMBLY_PATCH)
    with pytest.raises(capi.EnscError, match="assembly"):
        tables(p, assembly=7)


def test_prepared_tables_do_not_depend_on_the_mesh_arrays_afterwards():
    # the prepared instance copies what it needs: overwriting and dropping the
    # mesh arrays after ensc_batch_prepare leaves its tables unchanged
    p = W.block(8, 8, 8, 0.08, 0.08, 0.08, plastic=True)
    x0, conn, v0 = p.mesh.x0.copy(), p.mesh.conn.copy(), p.v0.copy()
    pr = capi.Prepared(x0, conn, v0, material=p.material, controls=p.controls, precision=capi.MIXED,
                       assembly=capi.ASSEMBLY_PATCH)
    try:
        x0[:] = np.nan
        conn[:] = 0
        v0[:] = np.nan
        del x0, conn, v0
        got = pr.patch_tables()
        nbytes = pr.device_bytes
    finally:
        pr.close()
    _, ref = tables(p)
    for k in ref:
        assert np.array_equal(got[k], ref[k]), k
    ref_pr = capi.Prepared(p.mesh.x0, p.mesh.conn, p.v0, material=p.material, controls=p.controls,
                           precision=capi.MIXED, assembly=capi.ASSEMBLY_PATCH)
    try:
        assert ref_pr.device_bytes == nbytes
    finally:
        ref_pr.close()
