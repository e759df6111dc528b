"""Horizontal domain decomposition of one FastEddy domain over px x py slabs.

FastEddy runs one MPI rank per GPU on a numProcsX x numProcsY grid of subdomains
(fempi.c:98-160: rank r sits at rx = r % numProcsX, ry = r / numProcsX; periodic neighbours
fempi.c:226-245) and exchanges 3-cell halos of every prognostic field at the start of each RK
stage (cuda_hydroCoreDevice.cu:276-314 calling fecuda_SendRecvWestEast/EastWest/SouthNorth/
NorthSouth, fecuda_Utils.cu:205-418).

Here the exchange is part of the commit: each slab's RK-stage kernel writes its cells within 3
of a slab edge into the neighbouring slabs' halos as peer stores (the same stores that write
an undecomposed domain's periodic images), and a stage barrier orders the stages. Two forms:

  SlabGroup        all slabs on one device in this process (fe_slab_group_create); the
                   stages of the slabs run as parallel graph branches joined per stage.
  DistributedSlab  one slab per process and GPU under torch.distributed: the slabs' state
                   arenas are shared by CUDA IPC handles (exchanged with all_gather_object),
                   the barrier is a one-element NCCL all-reduce per stage in the engine.

The host-side pieces (rank grid, slab inputs, reassembly, handle tables) are plain functions
so they can be checked without a GPU.
"""
from __future__ import annotations

import copy
import ctypes
from typing import Optional

import numpy as np

from .runtime import Domain, FeConfig, FeError, _check, load


class RankGrid:
    """The px x py rank grid of fempi.c:98-160 with periodic neighbours (fempi.c:226-245)."""

    def __init__(self, px: int, py: int) -> None:
        if px < 1 or py < 1:
            raise ValueError("slab counts must be >= 1")
        self.px, self.py = px, py
        self.size = px * py

    def coords(self, rank: int) -> tuple[int, int]:
        return rank % self.px, rank // self.px

    def rank(self, rx: int, ry: int) -> int:
        return (ry % self.py) * self.px + (rx % self.px)

    def neighbour(self, rank: int, dx: int, dy: int) -> int:
        rx, ry = self.coords(rank)
        return self.rank(rx + dx, ry + dy)

    def neighbours(self, rank: int) -> list[int]:
        """The 9 ranks around `rank` (itself included) in the engine's order (dx+1)*3 + (dy+1)."""
        return [self.neighbour(rank, dx, dy) for dx in (-1, 0, 1) for dy in (-1, 0, 1)]


def slab_config(cfg: FeConfig, px: int, py: int) -> FeConfig:
    """The configuration of one slab: Nx/px x Ny/py columns of the global domain."""
    if cfg.Nx % px or cfg.Ny % py:
        raise FeError(f"Nx={cfg.Nx}, Ny={cfg.Ny} do not divide into {px} x {py} slabs")
    c = copy.copy(cfg)
    c.Nx, c.Ny = cfg.Nx // px, cfg.Ny // py
    return c


def _xy_axes(a: np.ndarray) -> tuple[int, int]:
    # reference layout: (x, y) planes, (x, y, z) fields, (field, x, y, z) field sets
    return (0, 1) if a.ndim <= 3 else (1, 2)


# prognostic fields: an undecomposed domain's initial boundary pass replaces their horizontal
# halo columns by the periodic images of its own cells (the inputs' halo values are not used)
STATE_KEYS = ("hydroFlds", "sgstke", "moist")


def periodic_halos(a: np.ndarray) -> np.ndarray:
    """A copy of a halo-inclusive array whose 3-cell x and y halo columns are the periodic
    images of its own cells (all levels)."""
    ax, ay = _xy_axes(a)
    out = a.copy()
    for axis in (ax, ay):
        n = out.shape[axis] - 6
        idx = (np.arange(out.shape[axis]) - 3) % n + 3
        out = np.take(out, idx, axis=axis)
    return out


def split_inputs(inp: dict, px: int, py: int, rank: int) -> dict:
    """Rank `rank`'s slab of halo-inclusive global inputs (the arrays Host.inputs() returns):
    its cells plus a 3-cell halo on every side, which holds the neighbouring slabs' cells (or,
    at the global edges, what the undecomposed domain holds there: the periodic images for the
    prognostic fields, the given values for the grid, base state and surface planes)."""
    g = RankGrid(px, py)
    rx, ry = g.coords(rank)
    out = {}
    for k, a in inp.items():
        if a is None:
            out[k] = None
            continue
        if k in STATE_KEYS:
            a = periodic_halos(a)
        ax, ay = _xy_axes(a)
        nx, ny = (a.shape[ax] - 6) // px, (a.shape[ay] - 6) // py
        sl = [slice(None)] * a.ndim
        sl[ax] = slice(rx * nx, rx * nx + nx + 6)
        sl[ay] = slice(ry * ny, ry * ny + ny + 6)
        out[k] = np.ascontiguousarray(a[tuple(sl)])
    return out


def gather(parts: list[Optional[np.ndarray]], px: int, py: int) -> Optional[np.ndarray]:
    """Reassemble one halo-inclusive global array from the slabs' arrays (rank order): every
    slab's own cells, and the global halo from the slabs on the global edges."""
    if parts[0] is None:
        return None
    g = RankGrid(px, py)
    a0 = parts[0]
    ax, ay = _xy_axes(a0)
    nx, ny = a0.shape[ax] - 6, a0.shape[ay] - 6
    shape = list(a0.shape)
    shape[ax], shape[ay] = nx * px + 6, ny * py + 6
    out = np.empty(shape, a0.dtype)
    for r, a in enumerate(parts):
        rx, ry = g.coords(r)
        # x range of the slab's array kept: own cells, plus the halo on a global edge
        xs = slice(0 if rx == 0 else 3, nx + 6 if rx == px - 1 else nx + 3)
        ys = slice(0 if ry == 0 else 3, ny + 6 if ry == py - 1 else ny + 3)
        src = [slice(None)] * a.ndim
        dst = [slice(None)] * a.ndim
        src[ax], src[ay] = xs, ys
        dst[ax] = slice(rx * nx + xs.start, rx * nx + xs.stop)
        dst[ay] = slice(ry * ny + ys.start, ry * ny + ys.stop)
        out[tuple(dst)] = a[tuple(src)]
    return out


def gather_state(states: list[dict], px: int, py: int) -> dict:
    return {k: gather([s[k] for s in states], px, py) for k in states[0]}


def handle_table(grid: RankGrid, rank: int, handles: list[bytes]) -> list[Optional[bytes]]:
    """The engine's 9-entry neighbour table of `rank`: each neighbour's arena handle, None where
    the neighbour is the rank itself."""
    return [None if nb == rank else handles[nb] for nb in grid.neighbours(rank)]


def exchange_handles(local: bytes, group=None) -> list[bytes]:
    """Every rank's arena handle, in rank order (torch.distributed all_gather_object)."""
    import torch.distributed as dist

    out: list = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, local, group=group)
    return out


def _set_peers(dom: Domain, px: int, py: int, table: list[Optional[bytes]]) -> None:
    bufs = [None if h is None else ctypes.create_string_buffer(h, len(h)) for h in table]
    arr = (ctypes.c_void_p * 9)(*[None if b is None else ctypes.addressof(b) for b in bufs])
    _check(dom.e.fe_set_halo_peers(dom.h, px, py, arr), "fe_set_halo_peers")


class SlabGroup:
    """A decomposed domain whose px x py slabs all live on one device of this process."""

    def __init__(self, cfg: FeConfig, inputs: dict, px: int, py: int, device: int = 0, simTime: float = 0.0,
                 simTime_it: int = 0) -> None:
        self.px, self.py = px, py
        scfg = slab_config(cfg, px, py)
        self.slabs = [Domain(scfg, device) for _ in range(px * py)]
        self.e = load()["engine"]
        arr = (ctypes.c_void_p * len(self.slabs))(*[s.h.value for s in self.slabs])
        h = ctypes.c_void_p()
        _check(self.e.fe_slab_group_create(arr, px, py, ctypes.byref(h)), "fe_slab_group_create")
        self.h = h
        for r, s in enumerate(self.slabs):
            s.set_inputs(split_inputs(inputs, px, py, r), simTime, simTime_it)

    def advance(self, nsteps: int, sync: bool = True) -> None:
        _check(self.e.fe_ensemble_advance(self.h, nsteps), "fe_ensemble_advance")
        if sync:
            _check(self.e.fe_ensemble_sync(self.h), "fe_ensemble_sync")

    def get_state(self) -> dict:
        return gather_state([s.get_state() for s in self.slabs], self.px, self.py)

    def close(self) -> None:
        if self.h:
            self.e.fe_ensemble_destroy(self.h)
            self.h = ctypes.c_void_p()
        for s in self.slabs:
            s.close()


class DistributedSlab:
    """This process's slab of a domain decomposed over all ranks of a torch.distributed group
    (one GPU per rank; px * py must equal the group size). Every rank constructs it with the
    same global configuration and inputs and advances the same number of steps."""

    def __init__(self, cfg: FeConfig, inputs: dict, px: int, py: int, device: int, group=None, simTime: float = 0.0,
                 simTime_it: int = 0) -> None:
        import torch.distributed as dist

        self.grid = RankGrid(px, py)
        self.rank = dist.get_rank(group)
        if dist.get_world_size(group) != self.grid.size:
            raise FeError(f"{px} x {py} slabs need {self.grid.size} ranks, the group has {dist.get_world_size(group)}")
        self.group = group
        self.domain = Domain(slab_config(cfg, px, py), device)
        e = self.domain.e
        hb = ctypes.create_string_buffer(int(e.fe_ipc_handle_bytes()))
        _check(e.fe_arena_ipc_handle(self.domain.h, hb, len(hb)), "fe_arena_ipc_handle")
        handles = exchange_handles(hb.raw, group)
        _set_peers(self.domain, px, py, handle_table(self.grid, self.rank, handles))
        uid = None
        if self.rank == 0:
            ub = ctypes.create_string_buffer(int(e.fe_comm_unique_id_bytes()))
            _check(e.fe_comm_unique_id(ub, len(ub)), "fe_comm_unique_id")
            uid = ub.raw
        box = [uid]
        dist.broadcast_object_list(box, src=dist.get_global_rank(group, 0) if group is not None else 0, group=group)
        ub = ctypes.create_string_buffer(box[0], len(box[0]))
        c = ctypes.c_void_p()
        _check(e.fe_comm_create(ub, self.grid.size, self.rank, device, ctypes.byref(c)), "fe_comm_create")
        self.comm = c
        _check(e.fe_set_halo_comm(self.domain.h, c), "fe_set_halo_comm")
        self.domain.set_inputs(split_inputs(inputs, px, py, self.rank), simTime, simTime_it)
        # no slab's first commit may reach a neighbour whose buffers are still being set up
        dist.barrier(group)

    def advance(self, nsteps: int, sync: bool = True) -> None:
        self.domain.advance(nsteps, sync)

    def get_state(self) -> dict:
        return self.domain.get_state()

    def close(self) -> None:
        import torch.distributed as dist

        if self.domain.h:
            e = self.domain.e
            self.domain.sync()
            dist.barrier(self.group)  # no neighbour still writes into this slab's arena
            e.fe_clear_halo_peers(self.domain.h)  # unmap the neighbours' arenas
            e.fe_set_halo_comm(self.domain.h, None)
            e.fe_comm_destroy(self.comm)
            dist.barrier(self.group)  # every mapping of this slab's arena is closed
            self.domain.close()
