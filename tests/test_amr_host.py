"""The adaptive-mesh bookkeeping on the host (z4c_b200.amr) against the
reference's own adaptive run (fixture amr_bbh_amr.npz, made by
tests/golden/make_golden.py with the reference build): Mesh::Initialize's
refinement loop, then for every cycle the Linf_box_in_box flags of every
MeshBlock, the derefinement counters, UpdateMeshBlockTree and the
MeshBlockTree refine/derefine rules.  The puncture-tracker positions the
reference's flags saw each cycle are stored in the fixture bit for bit, so
the block list of every cycle must come out identical, gid order included.
No GPU: the device run is tests/test_gpu_amr.py."""
import json
import os

import numpy as np
import pytest

from z4c_testlib import GOLDEN

from z4c_b200 import amr as A

FIX = os.path.join(GOLDEN, "amr_bbh_amr.npz")


@pytest.fixture(scope="module")
def fx():
    return np.load(FIX)


def refinement(fx):
    mesh = json.loads(str(fx["mesh"]))
    amr = json.loads(str(fx["amr"]))
    prob = json.loads(str(fx["problem"]))
    return A.Refinement(mesh["nb"], mesh["nx"], mesh["xmin"], mesh["xmax"], mesh["bc"],
                        amr["numlevel"], amr["derefine_count"], prob["par_b"])


def start_points(fx):
    ex = json.loads(str(fx["extra"]))
    return [tuple(ex[f"bh_{n}_{c}"] for c in "xyz") for n in range(ex["npunct"])]


def ref_list(fx, cycle):
    b = fx["blocks"]
    rows = b[b[:, 0] == cycle]
    assert np.array_equal(rows[:, 1], np.arange(len(rows))), "gid order"
    return rows[:, 2:6].astype(np.int64)


def test_block_lists_of_every_cycle_match_the_reference(fx):
    ref = refinement(fx)
    start = start_points(fx)
    trk = fx["trackers"]
    # the trackers have not moved before the first cycle
    assert np.array_equal(trk[0], np.array(start))
    gen = ref.build_initial(start)
    assert gen is None
    assert np.array_equal(ref.locs(), ref_list(fx, 0))
    nlim = int(fx["nlim"])
    changes = []
    for c in range(nlim):
        flags = ref.flags([tuple(p) for p in trk[c]])
        if ref.update(flags):
            changes.append(c + 1)
        assert np.array_equal(ref.locs(), ref_list(fx, c + 1)), f"cycle {c + 1}"
    # the run refines once and derefines once
    assert len(changes) == 2, changes
    counts = [len(ref_list(fx, c)) for c in (0, changes[0], changes[1])]
    assert counts[1] > counts[0] and counts[2] < counts[1], counts


def test_tree_balance_and_coverage(fx):
    """Every list the replay produces tiles the root grid exactly and keeps
    neighbouring blocks within one level (2:1), faces, edges and corners."""
    ref = refinement(fx)
    ref.build_initial(start_points(fx))
    trk = fx["trackers"]
    for c in range(int(fx["nlim"])):
        ref.update(ref.flags([tuple(p) for p in trk[c]]))
        leaves = ref.tree.leaves
        r0, nb = ref.tree.r0, ref.tree.nb
        maxlev = max(b[0] for b in leaves)
        fine = {}
        for b in leaves:
            s = 1 << (maxlev - b[0])
            for k in range(b[3] * s, (b[3] + 1) * s):
                for j in range(b[2] * s, (b[2] + 1) * s):
                    for i in range(b[1] * s, (b[1] + 1) * s):
                        assert (i, j, k) not in fine
                        fine[(i, j, k)] = b[0]
        n = [nb[a] << (maxlev - r0) for a in range(3)]
        assert len(fine) == n[0] * n[1] * n[2]
        lev = np.zeros(n, dtype=int)
        for (i, j, k), lv in fine.items():
            lev[i, j, k] = lv
        for ax in range(3):
            d = np.abs(np.diff(lev, axis=ax))
            assert d.max() <= 1
        # diagonal neighbours too
        for sh in [(1, 1, 0), (1, 0, 1), (0, 1, 1), (1, 1, 1), (1, -1, 0), (1, 0, -1),
                   (0, 1, -1), (1, -1, 1), (1, 1, -1), (1, -1, -1)]:
            a = lev[max(0, sh[0]):n[0] + min(0, sh[0]), max(0, sh[1]):n[1] + min(0, sh[1]),
                    max(0, sh[2]):n[2] + min(0, sh[2])]
            b = lev[max(0, -sh[0]):n[0] + min(0, -sh[0]), max(0, -sh[1]):n[1] + min(0, -sh[1]),
                    max(0, -sh[2]):n[2] + min(0, -sh[2])]
            assert np.abs(a - b).max() <= 1


def test_box_in_box_criterion_levels():
    """Linf_box_in_box on a hand-checked case: mesh [-8, 8]^3, par_b 1.5
    (L = 6.5), one puncture at the origin.  A root block (level 0) whose
    inner-box vertex nearest the origin is 2 away in L-infinity wants level
    floor(log2(3.25)) = 1; a block 16 away wants to derefine."""
    import z4c_b200 as Z
    mesh = Z.Mesh((2, 2, 2), (8, 8, 8), (-8.0,) * 3, (8.0,) * 3, "outflow")
    # root block [0, 8]^3: inner box vertices at 3 and 5 per axis
    assert A.linf_box_in_box(mesh, (1, 1, 1, 1), [(0.0, 0.0, 0.0)], 1.5) == 1
    # the same block at level 1 of the tree (lx = 2: [0, 4]^3, vertices 1.5
    # and 2.5): d = 1.5, floor(log2(6.5 / 1.5)) = 2 > 1
    assert A.linf_box_in_box(mesh, (2, 2, 2, 2), [(0.0, 0.0, 0.0)], 1.5) == 1
    # puncture far outside: ratio < 1
    assert A.linf_box_in_box(mesh, (2, 2, 2, 2), [(40.0, 0.0, 0.0)], 1.5) == -1
    # d = 0 (puncture on an inner-box vertex): refine
    assert A.linf_box_in_box(mesh, (1, 1, 1, 1), [(3.0, 3.0, 3.0)], 1.5) == 1


def test_vectorised_criterion_equals_the_scalar_one():
    """The array form used per cycle gives the scalar restatement's flags
    on every block of a deep tree, for punctures on and off block corners."""
    import z4c_b200 as Z
    mesh = Z.Mesh((8, 8, 8), (16, 16, 16), (-512.0,) * 3, (512.0,) * 3, "outflow")
    ref = A.Refinement((8, 8, 8), (16, 16, 16), (-512.0,) * 3, (512.0,) * 3, mesh.bc, 7, 10, 3.0)
    trk = [(3.0, 0.023, 0.013), (-3.0, -0.023, -0.013)]
    ref.build_initial(trk)
    order = ref.order()
    assert len(order) > 1000
    rng = np.random.default_rng(1)
    for pts in (trk, [(0.0, 0.0, 0.0)], [tuple(rng.uniform(-600, 600, 3)) for _ in range(3)],
                [(256.0, 128.0, 64.0)]):
        vec = A.linf_box_in_box_all(ref.root, order, pts, 3.0)
        scal = [A.linf_box_in_box(ref.root, b, pts, 3.0) for b in order]
        assert vec.tolist() == scal
