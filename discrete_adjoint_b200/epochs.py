"""Forward and adjoint across mesh adaptation: a horizon split into mesh epochs.

The reference adapts its mesh during the forward run (H_adapt / unrefine, hpfem.C:243-267) and its
dual solver follows the recorded meshes backward, moving the adjoint between fathers and sons
(dualmesh.C:700-712, 980-995).  Here a horizon is a list of epochs, each a mesh and a step count;
between two epochs the state moves to the next mesh by the reference's transfer (element2.C:223-252,
520-532): a son takes its father's state (``myfractionoffather`` = 1), a father the mean of its four
sons, summed from zero in son order (SW, SE, NE, NW) with weight 0.25.  The forward runs each epoch
on the device; the adjoint runs the epochs backward, each reverse sweep starting from the later
epoch's lambda^0 carried back through the transpose of the transfer (a father receives the sum of
its sons' adjoints, each son a quarter of its father's), exactly the reference's dual-mesh rules.

Meshes of consecutive epochs must differ by at most one level in each cell (one refinement or one
unrefinement, as one adapt pass does).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _ffi
from .mesh import Mesh
from .solver import GeoflowContext, Gradient, MatProps, TimeProps, adjoint_run, adjoint_run_seeded, set_dt_replay

# son order of the reference (gen_my_sons_key, element2.C:4392-4399): SW, SE, NE, NW
_SONS = ((0, 0), (1, 0), (1, 1), (0, 1))


def _keys(level, ix, iy) -> np.ndarray:
    return (np.asarray(level, np.int64) << 58) | (np.asarray(ix, np.int64) << 29) | np.asarray(iy, np.int64)


@dataclass
class Transfer:
    """U_new = T U_old, row by row: new cell c takes sum_k w[k][c] U_old[src[k][c]] (src -1 unused);
    a row with one source of weight 1 is a copy."""
    src: np.ndarray  # [4][n_new]
    w: np.ndarray    # [4][n_new]
    n_old: int

    @property
    def n_new(self) -> int:
        return self.src.shape[1]

    def apply(self, u_old: np.ndarray) -> np.ndarray:
        """The forward transfer of one field, in the reference's order of operations."""
        u_old = np.asarray(u_old, dtype=np.float64)
        copy = (self.src[1] < 0) & (self.w[0] == 1.0)
        out = np.zeros(self.n_new)
        out[copy] = u_old[self.src[0][copy]]
        avg = ~copy
        for k in range(4):
            sel = avg & (self.src[k] >= 0)
            out[sel] = out[sel] + u_old[self.src[k][sel]] * self.w[k][sel]
        return out

    def adjoint(self, lam_new: np.ndarray) -> np.ndarray:
        """The transpose: lam_old[j] = sum over rows c naming j of w lam_new[c]."""
        lam_new = np.asarray(lam_new, dtype=np.float64)
        out = np.zeros(self.n_old)
        for k in range(4):
            sel = self.src[k] >= 0
            np.add.at(out, self.src[k][sel], self.w[k][sel] * lam_new[sel])
        return out


def transfer_between(old: Mesh, new: Mesh) -> Transfer:
    """The state transfer from mesh old to mesh new (same base grid, levels within one of each
    other in every cell): the same cell is copied, a son copies its father, a father averages its
    four sons."""
    ko = _keys(old.level, old.ix, old.iy)
    order = np.argsort(ko)
    ks = ko[order]

    def find(level, ix, iy):
        q = _keys(level, ix, iy)
        pos = np.minimum(np.searchsorted(ks, q), len(ks) - 1)
        hit = ks[pos] == q
        return np.where(hit, order[pos], -1)

    n = new.n
    src = np.full((4, n), -1, dtype=np.int64)
    w = np.zeros((4, n))
    same = find(new.level, new.ix, new.iy)
    src[0] = same
    w[0] = np.where(same >= 0, 1.0, 0.0)
    rest = same < 0
    father = np.full(n, -1, dtype=np.int64)
    father[rest] = find(new.level[rest] - 1, new.ix[rest] >> 1, new.iy[rest] >> 1)
    ref = rest & (father >= 0)
    src[0][ref] = father[ref]
    w[0][ref] = 1.0
    unr = rest & (father < 0)
    for k, (a, b) in enumerate(_SONS):
        s = find(new.level[unr] + 1, 2 * new.ix[unr] + a, 2 * new.iy[unr] + b)
        if np.any(s < 0):
            raise ValueError("meshes of consecutive epochs must differ by at most one level in each cell")
        src[k][unr] = s
        w[k][unr] = 0.25
    return Transfer(src, w, old.n)


@dataclass
class Epoch:
    mesh: Mesh
    nsteps: int


def _ctx(mat, precision, mesh, state, time, it, dts):
    c = GeoflowContext(mat, TimeProps(), precision=precision)
    c.upload_mesh(mesh)
    c.set_state(*state)
    c.set_time(time, it)
    if dts is not None:
        set_dt_replay(c, dts, it)
    return c


def forward(mat: MatProps, epochs: list, state0, precision: int = _ffi.DA_PREC_FP64, dts: list | None = None):
    """Runs the epochs from state0 (on the first mesh).  Returns (the state at the start of each
    epoch, the time and iteration there, the final state, the dt of every step per epoch)."""
    starts, clocks, steps = [], [], []
    state = [np.asarray(v, dtype=np.float64) for v in state0]
    time, it = 0.0, 0
    for k, ep in enumerate(epochs):
        if k:
            T = transfer_between(epochs[k - 1].mesh, ep.mesh)
            state = [T.apply(v) for v in state]
        starts.append(state)
        clocks.append((time, it))
        with _ctx(mat, precision, ep.mesh, state, time, it, None if dts is None else dts[k]) as c:
            d = []
            for _ in range(ep.nsteps):
                s = c.step()
                d.append(s.dt)
            time, it = s.time, s.iter
            state = list(c.get_state())
        steps.append(d)
    return starts, clocks, state, steps


def adjoint(mat: MatProps, epochs: list, state0, box, nsnapshots: int, dh0_dpile=None,
            precision: int = _ffi.DA_PREC_FP64, dts: list | None = None) -> Gradient:
    """J = sum h^2 dx dy over box at the end of the last epoch and its gradient with respect to the
    friction angles and (through state0 on the first mesh) the pile heights.  dts: the dt of every
    step per epoch to replay (else each epoch's CFL dt)."""
    starts, clocks, _, steps = forward(mat, epochs, state0, precision, dts)
    replay = steps if dts is None else dts
    K = len(epochs) - 1
    total = None
    lam_next = None
    for k in range(K, -1, -1):
        ep = epochs[k]
        time, it = clocks[k]
        with _ctx(mat, precision, ep.mesh, starts[k], time, it, replay[k]) as c:
            dh = dh0_dpile if k == 0 else None
            if k == K:
                g = adjoint_run(c, box, ep.nsteps, nsnapshots, dh, want_lambda0=True)
            else:
                g = adjoint_run_seeded(c, lam_next, ep.nsteps, nsnapshots, dh)
        if total is None:
            total = g
        else:
            total.dJ_dbedfrict = [a + b for a, b in zip(total.dJ_dbedfrict, g.dJ_dbedfrict)]
            total.dJ_dintfrict += g.dJ_dintfrict
            total.forward_steps += g.forward_steps
            total.device_ms += g.device_ms
        if k == 0:
            total.dJ_dpile = list(g.dJ_dpile)
            total.lambda0 = g.lambda0
        else:
            T = transfer_between(epochs[k - 1].mesh, ep.mesh)
            lam_next = np.stack([T.adjoint(g.lambda0[v]) for v in range(3)])
    return total
