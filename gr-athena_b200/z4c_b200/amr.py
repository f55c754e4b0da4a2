"""Adaptive mesh refinement driven from the host.

The block-tree bookkeeping is the reference's, restated over sets of logical
locations (level, lx1, lx2, lx3):

  MeshBlockTree::Refine / AddMeshBlock   mesh/meshblock_tree.cpp:108-230
  MeshBlockTree::Derefine                mesh/meshblock_tree.cpp:253-302
  MeshBlockTree::FindNeighbor            mesh/meshblock_tree.cpp:400-499
  MeshRefinement::CheckRefinementCondition  mesh/mesh_refinement.cpp:381-462
  Mesh::UpdateMeshBlockTree              mesh/amr_loadbalance.cpp:225-410
  Z4c_AMR::LinfBoxInBox                  z4c/z4c_amr.cpp:407-516

and the time loop follows the reference's order (main.cpp:156-333): the
refinement flags of a cycle are taken on its last RK stage, with the puncture
trackers where the previous cycle left them (the trackers move after the
task list, main.hpp:1078-1082); the tree is updated after the step, the state
is carried to the new block list on the device (z4c_regrid, the Main AMR
group transfer of RedistributeAndRefineMeshBlocks) and its ghosts finalised
(FinalizeZ4cADMGhosts), the constraints are re-evaluated on the new mesh
(CalculateZ4cInitDiagnostics), and dt becomes min(2 dt, new dt)
(Mesh::NewTimeStep, mesh/mesh.cpp:1753-1800).  The initial mesh is built the
way Mesh::Initialize does (mesh/mesh.cpp:2148-2416): initial data, flags,
tree update, repeated until the block count stops changing.
"""
import math
import sys

import numpy as np

from . import BC_NAMES, Mesh, Z4c, _mesh_gen_x

DBL_MAX = sys.float_info.max
_OFFSETS = [(ox, oy, oz) for oz in (-1, 0, 1) for oy in (-1, 0, 1) for ox in (-1, 0, 1)
            if (ox, oy, oz) != (0, 0, 0)]


def morton_order(locs):
    """Leaves in the order of the tree's depth-first walk (children n = i +
    2 j + 4 k): Morton order of their corners on the finest level."""
    if not locs:
        return []
    maxlev = max(b[0] for b in locs)

    def key(b):
        sh = maxlev - b[0]
        x, y, z = (v << sh for v in b[1:])
        k = 0
        for bit in range(maxlev + 1):
            k |= (((x >> bit) & 1) << (3 * bit)) | (((y >> bit) & 1) << (3 * bit + 1)) \
                | (((z >> bit) & 1) << (3 * bit + 2))
        return k
    return sorted(locs, key=key)


class BlockTree:
    """The leaves and interior nodes of the MeshBlock tree of a root grid of
    nb blocks per axis, with the reference's refine and derefine rules."""

    def __init__(self, nb, bc, locs=None):
        self.nb = tuple(int(v) for v in nb)
        self.r0 = max(0, (max(self.nb) - 1).bit_length())
        self.periodic = [int(bc[2 * a]) == BC_NAMES["periodic"] for a in range(3)]
        self.leaves = set()
        self.internal = set()
        if locs is None:
            locs = [(self.r0, i, j, k) for k in range(self.nb[2]) for j in range(self.nb[1])
                    for i in range(self.nb[0])]
        for b in locs:
            b = tuple(int(v) for v in b)
            self.leaves.add(b)
            for lv in range(self.r0, b[0]):
                self.internal.add((lv, *[x >> (b[0] - lv) for x in b[1:]]))

    def nblocks_at(self, level, a):
        return self.nb[a] << (level - self.r0)

    def wrap(self, level, l):
        """Location l on `level` with periodic wrapping; None outside a
        non-periodic face (FindNeighbor's and Refine's boundary rule)."""
        out = []
        for a in range(3):
            n = self.nblocks_at(level, a)
            x = l[a]
            if x < 0 or x >= n:
                if not self.periodic[a]:
                    return None
                x %= n
            out.append(x)
        return (level, *out)

    def order(self):
        return morton_order(list(self.leaves))

    def refine(self, node):
        """MeshBlockTree::Refine: eight children, then every same-level
        neighbour made to exist (AddMeshBlock from the root)."""
        if node in self.internal:
            return
        lev, l = node[0], node[1:]
        self.leaves.discard(node)
        self.internal.add(node)
        for c in range(8):
            self.leaves.add((lev + 1, 2 * l[0] + (c & 1), 2 * l[1] + ((c >> 1) & 1),
                             2 * l[2] + ((c >> 2) & 1)))
        for ox, oy, oz in _OFFSETS:
            nloc = self.wrap(lev, (l[0] + ox, l[1] + oy, l[2] + oz))
            if nloc is not None:
                self.add_block(nloc)

    def add_block(self, loc):
        """MeshBlockTree::AddMeshBlock: refine every leaf on the way down to
        loc."""
        lev = loc[0]
        for lv in range(self.r0, lev):
            anc = (lv, *[x >> (lev - lv) for x in loc[1:]])
            if anc in self.leaves:
                self.refine(anc)

    def finer_neighbour(self, loc):
        """True when a neighbour of the leaf loc is finer than it (the
        neighbor_level test of CheckRefinementCondition): the same-level
        node at some offset has children."""
        for ox, oy, oz in _OFFSETS:
            nloc = self.wrap(loc[0], (loc[1] + ox, loc[2] + oy, loc[3] + oz))
            if nloc is not None and nloc in self.internal:
                return True
        return False

    def derefine(self, node):
        """MeshBlockTree::Derefine: make the interior node a leaf unless a
        neighbour (itself included) has a child next to it that has children
        of its own.  Returns whether it derefined."""
        lev, l = node[0], node[1:]
        for oz in (-1, 0, 1):
            for oy in (-1, 0, 1):
                for ox in (-1, 0, 1):
                    nb = self.wrap(lev, (l[0] + ox, l[1] + oy, l[2] + oz))
                    if nb is None or nb not in self.internal:
                        continue
                    rng = [(1,) if o == -1 else (0,) if o == 1 else (0, 1) for o in (ox, oy, oz)]
                    for lk in rng[2]:
                        for lj in rng[1]:
                            for li in rng[0]:
                                ch = (lev + 1, 2 * nb[1] + li, 2 * nb[2] + lj, 2 * nb[3] + lk)
                                if ch in self.internal:
                                    return False
        for c in range(8):
            self.leaves.discard((lev + 1, 2 * l[0] + (c & 1), 2 * l[1] + ((c >> 1) & 1),
                                 2 * l[2] + ((c >> 2) & 1)))
        self.internal.discard(node)
        self.leaves.add(node)
        return True


def block_bounds(mesh, loc):
    """block_size.x?min/x?max of the block at loc (Mesh::
    SetBlockSizeAndBoundaries, mesh/mesh.cpp:2517-2600)."""
    lo, hi = [], []
    r0 = mesh.root_level
    for a in range(3):
        n = mesh.nb[a] << (loc[0] - r0)
        lx = int(loc[1 + a])
        lo.append(mesh.xmin[a] if lx == 0 else _mesh_gen_x(lx, n, mesh.xmin[a], mesh.xmax[a]))
        hi.append(mesh.xmax[a] if lx == n - 1 else
                  _mesh_gen_x(lx + 1, n, mesh.xmin[a], mesh.xmax[a]))
    return lo, hi


def linf_box_in_box(mesh, loc, trackers, par_b):
    """Z4c_AMR::LinfBoxInBox of the block at loc: 1 refine, -1 derefine,
    0 keep.  L = half the mesh's x1 extent minus par_b; d = the L-infinity
    distance from the nearest puncture to the nearest of the eight vertices
    of the box of the block's centre and 1/4 its size; the block wants level
    floor(log2(L / d)) above the root."""
    level = int(loc[0]) - mesh.root_level
    L = (mesh.xmax[0] - mesh.xmin[0]) / 2. - par_b
    lo, hi = block_bounds(mesh, loc)
    sup = [(5 * hi[a] + 3 * lo[a]) / 8. for a in range(3)]
    inf = [(3 * hi[a] + 5 * lo[a]) / 8. for a in range(3)]
    verts = [(sx[0], sy[1], sz[2]) for sx in (sup, inf) for sy in (sup, inf) for sz in (sup, inf)]
    d = DBL_MAX
    for p in trackers:
        dmin = DBL_MAX
        for v in verts:
            norm = -1.0
            for a in range(3):
                diff = abs(p[a] - v[a])
                if diff > norm:
                    norm = diff
            if dmin > norm:
                dmin = norm
        if d > dmin:
            d = dmin
    ratio = L / d if d != 0.0 else math.inf
    if ratio < 1:
        return -1
    th = math.floor(math.log2(ratio)) if math.isfinite(ratio) else math.inf
    if th > level:
        return 1
    if th < level:
        return -1
    return 0


def _gen_x(index, nrange, x0, x1):
    """_mesh_gen_x over integer arrays (the same IEEE operations)."""
    rx = (2 * index - nrange).astype(np.float64) / (2 * nrange).astype(np.float64)
    return 0.5 * (x0 + x1) + (rx * x1 - rx * x0)


def linf_box_in_box_all(mesh, locs, trackers, par_b):
    """linf_box_in_box of every block of locs (rows level, lx1, lx2, lx3),
    with the same floating-point operations in the same order."""
    locs = np.asarray(locs, dtype=np.int64).reshape(-1, 4)
    level = locs[:, 0] - mesh.root_level
    L = (mesh.xmax[0] - mesh.xmin[0]) / 2. - par_b
    sup, inf = [], []
    for a in range(3):
        n = np.left_shift(np.int64(mesh.nb[a]), level)
        lx = locs[:, 1 + a]
        lo = np.where(lx == 0, mesh.xmin[a], _gen_x(lx, n, mesh.xmin[a], mesh.xmax[a]))
        hi = np.where(lx == n - 1, mesh.xmax[a], _gen_x(lx + 1, n, mesh.xmin[a], mesh.xmax[a]))
        sup.append((5 * hi + 3 * lo) / 8.)
        inf.append((3 * hi + 5 * lo) / 8.)
    d = np.full(len(locs), DBL_MAX)
    for p in trackers:
        # the L-infinity distance to the nearest vertex factorises per axis
        dmin = np.full(len(locs), DBL_MAX)
        for sx in (sup, inf):
            for sy in (sup, inf):
                for sz in (sup, inf):
                    norm = np.maximum(np.maximum(np.abs(p[0] - sx[0]), np.abs(p[1] - sy[1])),
                                      np.abs(p[2] - sz[2]))
                    dmin = np.minimum(dmin, norm)
        d = np.minimum(d, dmin)
    with np.errstate(divide="ignore"):
        ratio = L / d
    out = np.zeros(len(locs), dtype=np.int64)
    for b, r in enumerate(ratio.tolist()):
        if r < 1:
            out[b] = -1
            continue
        th = math.floor(math.log2(r)) if math.isfinite(r) else math.inf
        out[b] = 1 if th > level[b] else (-1 if th < level[b] else 0)
    return out


class Refinement:
    """Refinement state of an adaptive mesh: the tree, each block's
    derefinement counter, and the flag and update steps."""

    def __init__(self, nb, nx, xmin, xmax, bc, numlevel, derefine_count=10, par_b=1.0,
                 locs=None):
        self.root = Mesh(nb, nx, xmin, xmax, bc)
        self.tree = BlockTree(nb, self.root.bc, locs)
        self.max_level = int(numlevel) + self.tree.r0 - 1
        self.threshold = int(derefine_count)
        self.par_b = float(par_b)
        self.deref_count = {b: 0 for b in self.tree.leaves}
        self._order = None

    def order(self):
        if self._order is None:
            self._order = self.tree.order()
        return self._order

    def locs(self):
        return np.array(self.order(), dtype=np.int64).reshape(-1, 4)

    def root_with(self, locs):
        m = Mesh(self.root.nb, self.root.nx, self.root.xmin, self.root.xmax, self.root.bc)
        m.locs = np.asarray(locs, dtype=np.int64).reshape(-1, 4)
        return m

    def mesh(self):
        return self.root_with(self.locs())

    def build_initial(self, trackers):
        """Mesh::Initialize's refinement loop (mesh/mesh.cpp:2157-2416):
        flags and a tree update until the count of MeshBlocks stops
        changing.  Returns None, or the block list the initial data are made
        on when the last update changed the blocks at an unchanged count
        (the state then reaches the final list by a regrid)."""
        while True:
            onb = len(self.tree.leaves)
            prev = self.locs()
            changed = self.update(self.flags(trackers))
            if len(self.tree.leaves) == onb:
                return prev if changed else None

    def flags(self, trackers):
        """CheckRefinementCondition on every block (gid order): the flag
        list, with the derefinement counters advanced."""
        out = []
        order = self.order()
        crit = linf_box_in_box_all(self.root, order, trackers, self.par_b)
        for loc, ret in zip(order, crit.tolist()):
            aret = max(-1, ret)
            flag = 0
            if aret >= 0:
                self.deref_count[loc] = 0
            if aret > 0:
                flag = 0 if loc[0] == self.max_level else 1
            elif aret < 0:
                if loc[0] == self.tree.r0:
                    self.deref_count[loc] = 0
                else:
                    self.deref_count[loc] += 1
                    if not self.tree.finer_neighbour(loc) and \
                            self.deref_count[loc] >= self.threshold:
                        flag = -1
            out.append((loc, flag))
        return out

    def update(self, flags):
        """UpdateMeshBlockTree: refine every block flagged 1, then derefine
        each complete octet of siblings flagged -1 (finest level first).
        Returns whether the tree changed."""
        lref = [loc for loc, f in flags if f == 1]
        lder = [loc for loc, f in flags if f == -1]
        if not lref and len(lder) < 8:
            return False
        parents = []
        if len(lder) >= 8:
            for n, a in enumerate(lder):
                if a[1] & 1 or a[2] & 1 or a[3] & 1:
                    continue
                r, rr = n, 0
                for k in (0, 1):
                    for j in (0, 1):
                        for i in (0, 1):
                            if r < len(lder):
                                if lder[r] == (a[0], a[1] + i, a[2] + j, a[3] + k):
                                    rr += 1
                                r += 1
                if rr == 8:
                    parents.append((a[0] - 1, a[1] >> 1, a[2] >> 1, a[3] >> 1))
        parents.sort(key=lambda p: -p[0])
        before = set(self.tree.leaves)
        for loc in lref:
            self.tree.refine(loc)
        for p in parents:
            self.tree.derefine(p)
        changed = self.tree.leaves != before
        self._order = None
        self.deref_count = {b: (self.deref_count[b] if b in before else 0)
                            for b in self.tree.leaves}
        return changed


class AdaptiveEvolution:
    """A Z4c evolution on an adaptive mesh: one device context per block
    list, regridded after every cycle whose flags change the tree.

    initial(mesh) -> ADM state (gid order) of the problem generator;
    trackers: starting points of the puncture trackers (the refinement
    criterion's punctures).  `tile`, when set (point_threads,
    column_threads, column_slabs, e.g. an autotuner's pick), is the launch
    shape of every context the run creates, `point_regs` and `contract`
    their register budget and right-hand-side path (see Z4c.set_point_regs,
    Z4c.set_contract).  `initial` may instead be a
    callable load(ctx) that fills the first context's Z4c state itself
    (pass load=True)."""

    def __init__(self, refinement, params, integrator, initial, trackers, cfl=0.25,
                 history=True, stream=None, load=False):
        from . import initial_data as ID
        self.ref = refinement
        self.params = params
        self.integrator = integrator
        self.cfl = float(cfl)
        self.history = history
        self.stream = stream
        self.tile = None
        self.point_regs = 0
        self.contract = False
        self.start = [tuple(float(v) for v in p) for p in trackers]
        self.ncycle = 0
        self.nregrid = 0
        self.log = []  # (ncycle, nblocks) after each regrid
        # Mesh::Initialize: the initial data go on the mesh the loop ends with
        # (or on the one before it, carried over, when the last update
        # changed the blocks but not their count)
        gen = self.ref.build_initial(self.start)
        mesh = self.ref.mesh() if gen is None else self.ref.root_with(gen)
        self.ctx = self._context(mesh)
        if load:
            initial(self.ctx)
        else:
            ID.load_adm(self.ctx, initial(mesh))
        if gen is not None:
            self._regrid()
        for p in self.start:
            self.ctx.add_tracker(p)
        if history:
            self.ctx.constraints()
        self.mesh_dt = self.ctx.mesh.new_dt(self.cfl)
        self.dt = self.mesh_dt

    def _context(self, mesh):
        ctx = Z4c(mesh, self.params, self.integrator)
        if self.stream is not None:
            ctx.set_stream(self.stream)
        if self.tile is not None:
            ctx.set_tile(*self.tile)
        ctx.set_point_regs(self.point_regs)
        ctx.set_contract(self.contract)
        return ctx

    def _regrid(self):
        new = self._context(self.ref.mesh())
        new.regrid_from(self.ctx)
        self.ctx.close()
        self.ctx = new
        self.mesh_dt = new.mesh.new_dt(self.cfl)
        self.nregrid += 1
        self.log.append((self.ncycle, new.nblocks))

    @property
    def mesh(self):
        return self.ctx.mesh

    def trackers(self):
        return [self.ctx.tracker(i)[0] for i in range(len(self.start))]

    def step(self):
        """One cycle: the RK step, the flags with the trackers where they
        stood before it, the regrid, the new dt.  Returns whether it
        regridded."""
        pos = self.trackers()
        self.ctx.evolve(self.dt, 1, with_constraints=self.history)
        self.ncycle += 1
        flags = self.ref.flags(pos)
        regridded = False
        if self.ref.update(flags):
            self._regrid()
            if self.history:
                self.ctx.constraints()
            regridded = True
        self.dt = min(2.0 * self.dt, self.mesh_dt)
        return regridded

    def close(self):
        if self.ctx is not None:
            self.ctx.close()
            self.ctx = None
