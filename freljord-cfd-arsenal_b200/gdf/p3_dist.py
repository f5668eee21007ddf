"""Block decomposition of the k = 3 variant over several devices.

MPI_BalsaraP3/main.f90 runs one MPI rank per block of an Nx_process x
Ny_process grid of blocks (main.f90:8-11, :494-501): every rank holds its
block with one ghost layer, set_bc exchanges the ghost layers with the
neighbouring ranks (x columns, then y rows that carry the fresh x ghosts,
main.f90:1574-1867), and calculate_dt takes the maximum speed over the ranks
(:1492-1538). Here a block is a P3Solver handle driven stage by stage
(gdf_p3_step_speeds / _step_begin / _stage_lh / _stage_limit); between the
stages the ghost layers of its device arrays are filled by a transport:

* LocalTransport: every block in this process (one device or several),
  tensor copies between the blocks' arrays;
* DistTransport: one block per rank, torch.distributed point-to-point
  exchanges (NCCL between GPUs, gloo on the host) and an all-reduce(max)
  of the speeds.

Because every ghost value equals the one set_bc gives the undivided grid
and every other value is computed from the block's own cells, a decomposed
run equals the single-block run value for value.
"""
from __future__ import annotations

import numpy as np

from . import p3
from .p3 import GdfP3Config, NB3, P3Solver

NS3 = 84
BC_PERIODIC = 1


class BlockGrid:
    """px x py equal blocks of a grid (the reference's Nx = Nx0/Nx_process)."""

    def __init__(self, cfg: GdfP3Config, px: int, py: int):
        if cfg.nx % px or cfg.ny % py:
            raise ValueError(f"{cfg.nx} x {cfg.ny} cells do not split into {px} x {py} equal blocks")
        self.cfg = cfg.copy()
        self.px, self.py = px, py
        self.nxb, self.nyb = cfg.nx // px, cfg.ny // py

    def blocks(self):
        return [(bi, bj) for bj in range(self.py) for bi in range(self.px)]

    def rank_of(self, bi: int, bj: int) -> int:
        """main.f90:494-501: myid1 = myidx + Nx_process*(myidy - 1)."""
        return bi + self.px * bj

    def block_of(self, rank: int):
        return rank % self.px, rank // self.px

    def block_config(self) -> GdfP3Config:
        c = self.cfg.copy()
        c.nx, c.ny = self.nxb, self.nyb
        c.nx_global, c.ny_global = self.cfg.nx, self.cfg.ny
        return c

    # host arrays in the reference layouts: uh (8, 15, NY+2, NX+2),
    # Bx (4, NY+2, NX+1), By (4, NY+1, NX+2)
    def split(self, uh, bx, by, bi: int, bj: int):
        x0, y0 = bi * self.nxb, bj * self.nyb
        return (np.ascontiguousarray(uh[:, :, y0:y0 + self.nyb + 2, x0:x0 + self.nxb + 2]),
                np.ascontiguousarray(bx[:, y0:y0 + self.nyb + 2, x0:x0 + self.nxb + 1]),
                np.ascontiguousarray(by[:, y0:y0 + self.nyb + 1, x0:x0 + self.nxb + 2]))

    def join(self, parts: dict):
        """Whole-grid arrays from the blocks' (uh, bx, by): interior cells and
        every face (ghost cells and ghost face rows/columns zero)."""
        uh, bx, by = p3.p3_new_state(self.cfg.nx, self.cfg.ny)
        for (bi, bj), (u, x, y) in parts.items():
            x0, y0 = bi * self.nxb, bj * self.nyb
            uh[:, :, y0 + 1:y0 + self.nyb + 1, x0 + 1:x0 + self.nxb + 1] = u[:, :, 1:-1, 1:-1]
            bx[:, y0 + 1:y0 + self.nyb + 1, x0:x0 + self.nxb + 1] = x[:, 1:-1, :]
            by[:, y0:y0 + self.nyb + 1, x0 + 1:x0 + self.nxb + 1] = y[:, :, 1:-1]
        return uh, bx, by

    def neighbour(self, bi: int, bj: int, side: str):
        """The block across `side` (l, r, d, u), or None at an outflow edge."""
        c = self.cfg
        if side == "l":
            return (bi - 1, bj) if bi > 0 else ((self.px - 1, bj) if c.bc_l == BC_PERIODIC else None)
        if side == "r":
            return (bi + 1, bj) if bi < self.px - 1 else ((0, bj) if c.bc_r == BC_PERIODIC else None)
        if side == "d":
            return (bi, bj - 1) if bj > 0 else ((bi, self.py - 1) if c.bc_d == BC_PERIODIC else None)
        return (bi, bj + 1) if bj < self.py - 1 else ((bi, 0) if c.bc_u == BC_PERIODIC else None)


# -------------------------------------------------------- ghost layers ----
# A block's arrays as (torch) views: cells (S, nyb+2, nxb+2), Bx faces
# (4, nyb+2, nxb+1), By faces (4, nyb+1, nxb+2). The four edge strips of a
# phase: x phase columns (full height), y phase rows (full width).

class LocalTransport:
    """All blocks in this process: the x phase, then the y phase, as tensor
    copies (a block on a periodic edge of a one-block-wide grid is its own
    neighbour)."""

    def __init__(self, grid: BlockGrid):
        self.grid = grid

    def fill(self, views: dict, kind: str) -> None:
        """views[(bi, bj)] = cell tensor (kind 'cells'), or (bx, by) face
        tensors (kind 'faces')."""
        g = self.grid
        nxb, nyb = g.nxb, g.nyb
        if kind == "cells":
            for phase in ("x", "y"):
                for b, a in views.items():
                    for side in (("l", "r") if phase == "x" else ("d", "u")):
                        nb = g.neighbour(*b, side)
                        src = views[nb] if nb is not None else a
                        if phase == "x":
                            if side == "l":
                                a[:, :, 0] = src[:, :, nxb] if nb is not None else a[:, :, 1]
                            else:
                                a[:, :, nxb + 1] = src[:, :, 1] if nb is not None else a[:, :, nxb]
                        else:
                            if side == "d":
                                a[:, 0, :] = src[:, nyb, :] if nb is not None else a[:, 1, :]
                            else:
                                a[:, nyb + 1, :] = src[:, 1, :] if nb is not None else a[:, nyb, :]
            return
        # faces: Bx ghost rows from the y neighbours, By ghost columns from the x neighbours
        for b, (fx, fy) in views.items():
            nd, nu = g.neighbour(*b, "d"), g.neighbour(*b, "u")
            fx[:, 0, :] = views[nd][0][:, nyb, :] if nd is not None else fx[:, 1, :]
            fx[:, nyb + 1, :] = views[nu][0][:, 1, :] if nu is not None else fx[:, nyb, :]
            nl, nr = g.neighbour(*b, "l"), g.neighbour(*b, "r")
            fy[:, :, 0] = views[nl][1][:, :, nxb] if nl is not None else fy[:, :, 1]
            fy[:, :, nxb + 1] = views[nr][1][:, :, 1] if nr is not None else fy[:, :, nxb]

    def max_speeds(self, speeds):
        return max(s[0] for s in speeds), max(s[1] for s in speeds)


class DistTransport:
    """One block per rank of a torch.distributed group (rank r holds block
    grid.block_of(r)); point-to-point exchanges of the edge strips."""

    def __init__(self, grid: BlockGrid, dist, group=None):
        self.grid = grid
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.block = grid.block_of(self.rank)

    def _phase(self, lo, hi, a_lo, a_hi, g_lo, g_hi):
        """One phase along an axis: lo/hi = neighbour blocks below/above (None
        at an outflow edge); a_lo/a_hi = my first/last interior strips; g_lo/
        g_hi = my ghost strips. Sends go up first (my last strip to hi, my
        low ghost from lo), then down, so that two ranks that are each
        other's neighbour on both sides (a periodic axis of two blocks) match
        their messages in posting order."""
        import torch
        ops, posts = [], []

        def post(peer, send, target, self_src, outflow_src):
            if peer is None:
                target.copy_(outflow_src)
                return
            pr = self.grid.rank_of(*peer)
            if pr == self.rank:
                target.copy_(self_src)
                return
            if send is not None:
                ops.append(self.dist.P2POp(self.dist.isend, send.contiguous(), pr, self.group))
            if target is not None:
                buf = torch.empty_like(target.contiguous())
                ops.append(self.dist.P2POp(self.dist.irecv, buf, pr, self.group))
                posts.append((target, buf))

        # upward: my last strip to hi; my low ghost from lo
        if hi is not None and self.grid.rank_of(*hi) != self.rank:
            post(hi, a_hi, None, None, None)
        post(lo, None, g_lo, a_hi, a_lo)
        # downward: my first strip to lo; my high ghost from hi
        if lo is not None and self.grid.rank_of(*lo) != self.rank:
            post(lo, a_lo, None, None, None)
        post(hi, None, g_hi, a_lo, a_hi)
        if ops:
            for r in self.dist.batch_isend_irecv(ops):
                r.wait()
        for target, buf in posts:
            target.copy_(buf)

    def fill(self, views: dict, kind: str) -> None:
        g = self.grid
        nxb, nyb = g.nxb, g.nyb
        b = self.block
        nl, nr, nd, nu = (g.neighbour(*b, s) for s in ("l", "r", "d", "u"))
        if kind == "cells":
            a = views[b]
            self._phase(nl, nr, a[:, :, 1], a[:, :, nxb], a[:, :, 0], a[:, :, nxb + 1])
            self._phase(nd, nu, a[:, 1, :], a[:, nyb, :], a[:, 0, :], a[:, nyb + 1, :])
            return
        fx, fy = views[b]
        self._phase(nd, nu, fx[:, 1, :], fx[:, nyb, :], fx[:, 0, :], fx[:, nyb + 1, :])
        self._phase(nl, nr, fy[:, :, 1], fy[:, :, nxb], fy[:, :, 0], fy[:, :, nxb + 1])

    def max_speeds(self, speeds):
        import torch
        v = torch.tensor([speeds[0][0], speeds[0][1]], dtype=torch.float64)
        if self.dist.get_backend(self.group) == "nccl":
            v = v.cuda()
        self.dist.all_reduce(v, op=self.dist.ReduceOp.MAX, group=self.group)
        return float(v[0]), float(v[1])


# ------------------------------------------------- decomposed stepping --

class _DeviceArray:
    """A raw device pointer as an object torch.as_tensor can view."""

    def __init__(self, ptr: int, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f8", "data": (ptr, False),
                                         "version": 3, "strides": None}


class P3Decomposed:
    """The k = 3 solver over the blocks this process owns (all of them for
    LocalTransport, one for DistTransport)."""

    def __init__(self, grid: BlockGrid, transport, blocks=None, devices=None, exact: bool = True):
        import torch
        self.grid = grid
        self.tr = transport
        self.blocks = list(blocks if blocks is not None else grid.blocks())
        self.solvers = {}
        self.views = {}
        bc = grid.block_config()
        for k, b in enumerate(self.blocks):
            if devices is not None:
                p3._lib(exact).gdf_set_device(devices[k % len(devices)])
            s = P3Solver(bc, exact=exact)
            self.solvers[b] = s
        self.torch = torch
        self.t = 0.0

    def _views(self, b):
        torch = self.torch
        s = self.solvers[b]
        arr = s.block_arrays()
        g = self.grid
        n2x, n2y = g.nxb + 2, g.nyb + 2
        dev = None

        def view(name, shape):
            return torch.as_tensor(_DeviceArray(arr[name], shape), device=dev)

        return {"U": view("U", (NS3, n2y, n2x)), "T": view("T", (NS3, n2y, n2x)),
                "BX": view("BX", (NB3, n2y, g.nxb + 1)), "BY": view("BY", (NB3, g.nyb + 1, n2x)),
                "BXT": view("BXT", (NB3, n2y, g.nxb + 1)), "BYT": view("BYT", (NB3, g.nyb + 1, n2x))}

    def upload(self, uh, bx, by) -> None:
        for b, s in self.solvers.items():
            s.upload(*self.grid.split(uh, bx, by, *b))
            self.views[b] = self._views(b)
        self.t = 0.0

    def download(self):
        return self.grid.join({b: s.download() for b, s in self.solvers.items()})

    def _sync(self):
        # the blocks' kernels run on their handles' streams; the ghost
        # copies on torch's: the whole device is the simplest fence
        self.torch.cuda.synchronize()

    def _fill(self, which: str) -> None:
        self._sync()
        if which == "U":
            self.tr.fill({b: v["U"] for b, v in self.views.items()}, "cells")
        else:
            self.tr.fill({b: v["T"] for b, v in self.views.items()}, "cells")
            self.tr.fill({b: (v["BXT"], v["BYT"]) for b, v in self.views.items()}, "faces")
        self.torch.cuda.synchronize()

    def prepare(self) -> None:
        """RK4's start on every block (gdf_p3_prepare of the whole grid)."""
        for s in self.solvers.values():
            s.stage_load_t()
        self._fill("T")
        for s in self.solvers.values():
            s.stage_limit()
        self._sync()

    def step(self, tend: float):
        speeds = [s.step_speeds() for s in self.solvers.values()]
        ax, ay = self.tr.max_speeds(speeds)
        for s in self.solvers.values():
            t, dt = s.step_begin(ax, ay, tend)
        self.t = t
        for stage in range(1, 11):
            self._fill("U")
            for s in self.solvers.values():
                s.stage_lh(stage)
            if stage != 5:
                self._fill("T")
                for s in self.solvers.values():
                    s.stage_limit()
        self._sync()
        return t, dt
