"""Host-side mesh generation: creat_mesh with its static block refinement
(src/mesh.F90:9-47, 49-197, 262-303, 421-461).

The reference refines the background grid at creat_mesh when lvlBlock > 0:
Block_refi refines every leaf whose centre lies in the box Block_size to
lvlBlock, BlockDis_refi refines a leaf at level l < lvlBlock whose distance
to the box (miblock) is within refinesize(i) = BufferLayerLVL*h/2**(i-1) for
some i > l, and lvlBlock-1 passes of gridmodify then refine every face
neighbour more than one level coarser than a leaf.  The passes are
order-dependent (a neighbour refined ahead of the traversal is visited in the
same pass, one behind it is not), so this follows the reference's pointer
walk: roots in order, sons 1, 2, 3, 4, the four neighbours of a leaf taken
before any of them is refined.  Cells are never solid (gridsort is
identically 0, src/mesh.F90:81-87).

The result is a leaf set (keys in key order) for fdm_upload_leaves: the tree
crosses the C-ABI as keys, so mesh generation stays host code as in the
reference.
"""
from __future__ import annotations

import numpy as np

from . import params as P

_SP_TO_Q = {1: 0, 2: 1, 3: 3, 4: 2}   # sp -> quadrant bits of the key path


class _Cell:
    __slots__ = ("num0", "num1", "lvl", "sp", "father", "sons", "cx", "cy", "root", "path")

    def __init__(self, num0, num1, lvl, sp, father, cx, cy, root, path):
        self.num0, self.num1, self.lvl, self.sp = num0, num1, lvl, sp
        self.father, self.sons = father, None
        self.cx, self.cy = cx, cy
        self.root, self.path = root, path


class _Tree:
    def __init__(self, cfg: P.Config):
        p = cfg.params
        self.m, self.n = cfg.m, cfg.n
        self.h, self.xf = p.h, p.x_factor
        self.cells = []
        for i in range(1, self.m * self.n + 1):          # creat_mesh, src/mesh.F90:15-37
            ni = (i - 1) // self.m + 1
            nj = i - self.m * (ni - 1)
            cx = 0.5 * (2.0 * nj - 1.0) * p.x_factor * p.h + p.xmin
            cy = (ni - 0.5) * p.h + p.ymin
            self.cells.append(_Cell(ni, nj, 0, 0, None, cx, cy, i - 1, 0))

    # Refine_cell, src/mesh.F90:199-260 (child centres by the same operations)
    def refine(self, c: _Cell):
        qx = self.xf * self.h / float(1 << (c.lvl + 2))
        qy = self.h / float(1 << (c.lvl + 2))
        sons = []
        for sp, sx, sy in ((1, c.cx - qx, c.cy - qy), (2, c.cx + qx, c.cy - qy),
                           (3, c.cx + qx, c.cy + qy), (4, c.cx - qx, c.cy + qy)):
            lvl = c.lvl + 1
            path = c.path | (_SP_TO_Q[sp] << (2 * (15 - lvl)))
            sons.append(_Cell(c.num0, c.num1, lvl, sp, c, sx, sy, c.root, path))
        c.sons = sons

    # up/down/left/right_neighbor, src/neighbor.F90:6-196
    def up(self, c):
        f = c.father
        if f is None:
            return None if c.num0 == self.n else self.cells[c.num0 * self.m + c.num1 - 1]
        if c.sp == 1:
            return f.sons[3]
        if c.sp == 2:
            return f.sons[2]
        fn = self.up(f)
        if fn is not None:
            if fn.sons is None:
                return fn
            return fn.sons[0] if c.sp == 4 else fn.sons[1]
        return None

    def down(self, c):
        f = c.father
        if f is None:
            return None if c.num0 == 1 else self.cells[(c.num0 - 2) * self.m + c.num1 - 1]
        if c.sp == 4:
            return f.sons[0]
        if c.sp == 3:
            return f.sons[1]
        fn = self.down(f)
        if fn is not None:
            if fn.sons is None:
                return fn
            return fn.sons[3] if c.sp == 1 else fn.sons[2]
        return None

    def left(self, c):
        f = c.father
        if f is None:
            return None if c.num1 == 1 else self.cells[(c.num0 - 1) * self.m + c.num1 - 2]
        if c.sp == 2:
            return f.sons[0]
        if c.sp == 3:
            return f.sons[3]
        fn = self.left(f)
        if fn is not None:
            if fn.sons is None:
                return fn
            return fn.sons[2] if c.sp == 4 else fn.sons[1]
        return None

    def right(self, c):
        f = c.father
        if f is None:
            return None if c.num1 == self.m else self.cells[(c.num0 - 1) * self.m + c.num1]
        if c.sp == 1:
            return f.sons[1]
        if c.sp == 4:
            return f.sons[2]
        fn = self.right(f)
        if fn is not None:
            if fn.sons is None:
                return fn
            return fn.sons[0] if c.sp == 2 else fn.sons[3]
        return None

    def leaves(self):
        out = []
        stack = []
        for c in reversed(self.cells):
            stack.append(c)
        while stack:
            c = stack.pop()
            if c.sons is None:
                out.append((c.root << 34) | (c.path << 4) | c.lvl)
            else:
                stack.extend(reversed(c.sons))
        return np.array(sorted(out), dtype=np.uint64)


def _miblock(bs, c) -> float:                          # src/mesh.F90:421-461
    xo, yo = c.cx, c.cy
    if xo > bs[1]:
        if yo > bs[3]:
            return float(np.sqrt((xo - bs[1]) * (xo - bs[1]) + (yo - bs[3]) * (yo - bs[3])))
        if yo < bs[2]:
            return float(np.sqrt((xo - bs[1]) * (xo - bs[1]) + (yo - bs[2]) * (yo - bs[2])))
        return xo - bs[1]
    if xo < bs[0]:
        if yo > bs[3]:
            return float(np.sqrt((xo - bs[0]) * (xo - bs[0]) + (yo - bs[3]) * (yo - bs[3])))
        if yo < bs[2]:
            return float(np.sqrt((xo - bs[0]) * (xo - bs[0]) + (yo - bs[2]) * (yo - bs[2])))
        return bs[0] - xo
    if yo > bs[3]:
        return yo - bs[3]
    if yo < bs[2]:
        return bs[2] - yo
    return 0.0


def block_refined_keys(cfg: P.Config) -> np.ndarray:
    """Leaf keys after creat_mesh (with Block_refine when cfg.block is set),
    in key order."""
    t = _Tree(cfg)
    if not cfg.block:
        return t.leaves()
    lvlblock, bs, buf = cfg.block
    refinesize = [0.0] + [float(buf) * t.h / float(1 << (i - 1)) for i in range(1, lvlblock + 1)]

    def block_refi(c):                                  # src/mesh.F90:176-197
        if c.lvl >= lvlblock:
            return
        if c.sons is None:
            if c.cx < bs[0] or c.cx > bs[1] or c.cy < bs[2] or c.cy > bs[3]:
                return
            t.refine(c)
        for s in c.sons:
            block_refi(s)

    def blockdis_refi(c):                               # src/mesh.F90:144-174
        if c.lvl >= lvlblock:
            return
        if c.sons is not None:
            for s in c.sons:
                blockdis_refi(s)
            return
        dis = _miblock(bs, c)
        for i in range(1, lvlblock + 1):
            if dis <= refinesize[i] and c.lvl < i:
                t.refine(c)
                for s in c.sons:
                    blockdis_refi(s)
                break

    def gridmodify(c):                                  # src/mesh.F90:262-303
        if c.sons is not None:
            for s in c.sons:
                gridmodify(s)
            return
        nbs = (t.up(c), t.down(c), t.left(c), t.right(c))
        for nb in nbs:
            if nb is not None and c.lvl - nb.lvl > 1:
                t.refine(nb)

    for c in t.cells:
        block_refi(c)
    for c in t.cells:
        blockdis_refi(c)
    for _ in range(lvlblock - 1):
        for c in t.cells:
            if c.sons is not None:
                gridmodify(c)
    return t.leaves()
