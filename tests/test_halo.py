"""Horizontal domain decomposition (fempi.c rank grid, per-stage halo exchange of
cuda_hydroCoreDevice.cu:276-314) on the CPU: the rank grid and neighbour table, the slab
inputs and their reassembly, the handle exchange over gloo, and -- with the FP64 oracle as the
per-slab model -- that slabs which exchange 3-cell halos before every RK stage reproduce the
undecomposed domain bit for bit (world size 2 over gloo, x and y decompositions)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _spawn(target, world: int, *args):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, q, *args)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in procs), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    return res


def _init(rank: int, world: int, port: int):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    return dist


def test_rank_grid_follows_the_reference_topology(fe):
    """rx = r % px, ry = r / px (fempi.c:113-114); neighbours across a global edge wrap
    periodically (fempi.c:226-245)."""
    g = fe.halo.RankGrid(3, 2)
    assert [g.coords(r) for r in range(6)] == [(0, 0), (1, 0), (2, 0), (0, 1), (1, 1), (2, 1)]
    assert g.neighbour(0, -1, 0) == 2 and g.neighbour(2, 1, 0) == 0  # x wraps within the row
    assert g.neighbour(1, 0, -1) == 4 and g.neighbour(4, 0, 1) == 1  # y wraps within the column
    assert g.neighbour(0, -1, -1) == 5
    nb = g.neighbours(4)
    assert nb[4] == 4 and nb[1] == 3 and nb[7] == 5 and nb[3] == 1 and nb[5] == 1
    t = fe.halo.handle_table(fe.halo.RankGrid(2, 1), 0, [b"h0", b"h1"])
    assert t == [b"h1", b"h1", b"h1", None, None, None, b"h1", b"h1", b"h1"]


@pytest.mark.parametrize("px,py", [(2, 1), (1, 2), (2, 3), (4, 2)])
def test_split_and_gather_round_trip(fe, px, py):
    rng = np.random.default_rng(px * 10 + py)
    nx, ny, nz = 8 * px, 6 * py, 5
    g = {"a4": rng.random((3, nx + 6, ny + 6, nz + 6)).astype(np.float32),
         "a3": rng.random((nx + 6, ny + 6, nz + 6)).astype(np.float32),
         "a2": rng.random((nx + 6, ny + 6)).astype(np.float32), "none": None}
    parts = [fe.halo.split_inputs(g, px, py, r) for r in range(px * py)]
    assert parts[0]["a4"].shape == (3, 14, 12, 11) and parts[0]["a2"].shape == (14, 12)
    # a slab's x halo holds its neighbour's cells
    if px > 1:
        np.testing.assert_array_equal(parts[0]["a3"][-3:], parts[1]["a3"][3:6])
    back = fe.halo.gather_state(parts, px, py)
    for k, a in g.items():
        if a is None:
            assert back[k] is None
        else:
            np.testing.assert_array_equal(back[k], a)
    # prognostic fields: the global halos are replaced by periodic images (the undecomposed
    # domain's initial boundary pass), on every slab on the global edge
    g["hydroFlds"] = g.pop("a4")
    parts = [fe.halo.split_inputs(g, px, py, r) for r in range(px * py)]
    back = fe.halo.gather([p["hydroFlds"] for p in parts], px, py)
    np.testing.assert_array_equal(back[:, 3:-3, 3:-3], g["hydroFlds"][:, 3:-3, 3:-3])
    np.testing.assert_array_equal(back[:, :3, 3:-3], g["hydroFlds"][:, -6:-3, 3:-3])
    np.testing.assert_array_equal(back[:, 3:-3, -3:], g["hydroFlds"][:, 3:-3, 3:6])
    np.testing.assert_array_equal(back[:, :3, :3], g["hydroFlds"][:, -6:-3, -6:-3])
    with pytest.raises(fe.FeError, match="divide"):
        fe.halo.slab_config(fe.cases.setup_host("cbl_dry", 10, 6, 6).config(), 3, 1)


def _handles_worker(rank, world, port, q):
    dist = _init(rank, world, port)
    import importlib

    fe = importlib.import_module("fasteddy-model_b200")
    hs = fe.halo.exchange_handles(bytes([rank]) * 64)
    table = fe.halo.handle_table(fe.halo.RankGrid(world, 1), rank, hs)
    q.put((rank, [h[:1] if h else None for h in hs], [t[:1] if t else None for t in table]))
    dist.destroy_process_group()


def test_handle_exchange_over_gloo():
    res = _spawn(_handles_worker, 2)
    for rank, hs, table in res:
        assert hs == [b"\x00", b"\x01"]
        other = bytes([1 - rank])
        assert table == [other, other, other, None, None, None, other, other, other]


def _exchange(dist, fld: np.ndarray, axis: int, n: int, other: int) -> None:
    """Two-slab halo exchange along `axis` (both neighbours are the other rank): my first 3
    cells go to its high halo, my last 3 to its low halo."""
    import torch

    def plane(a, s):
        sl = [slice(None)] * a.ndim
        sl[axis] = s
        return tuple(sl)

    lo = torch.from_numpy(np.ascontiguousarray(fld[plane(fld, slice(3, 6))]))
    hi = torch.from_numpy(np.ascontiguousarray(fld[plane(fld, slice(n, n + 3))]))
    got_hi, got_lo = torch.empty_like(lo), torch.empty_like(hi)
    reqs = [dist.isend(lo, other, tag=1), dist.isend(hi, other, tag=2)]
    dist.recv(got_hi, other, tag=1)
    dist.recv(got_lo, other, tag=2)
    for r in reqs:
        r.wait()
    fld[plane(fld, slice(n + 3, n + 6))] = got_hi.numpy()
    fld[plane(fld, slice(0, 3))] = got_lo.numpy()


def _oracle_slab_worker(rank, world, port, q, px, py, nsteps):
    dist = _init(rank, world, port)
    import importlib

    from oracle.pyoracle import Oracle

    fe = importlib.import_module("fasteddy-model_b200")
    host = fe.cases.setup_host("cbl_moist_hill", 16, 12, 8, hill_halfwidth=60.0, hill_height=12.0, qv=(24.0, 8.0, 300.0))
    cfg, inp = host.config(), host.inputs()
    o = Oracle(fe.halo.slab_config(cfg, px, py))
    o.set_decomposition(px > 1, py > 1)
    o.set_inputs(fe.halo.split_inputs(inp, px, py, rank))
    # x first (own rows), then y over the whole x range, halos included: the corners arrive with it
    # (with two slabs per direction both neighbours along a direction are the same rank)
    dirs = ([(1, cfg.Nx // px, rank ^ 1)] if px > 1 else []) + ([(2, cfg.Ny // py, rank ^ px)] if py > 1 else [])
    t, it = np.float32(0.0), 0
    for _ in range(nsteps):
        for stage in range(3):
            s = o.get_state()
            for key in ("hydroFlds", "sgstke", "moist"):
                if s[key] is not None:
                    for axis, n, other in dirs:
                        _exchange(dist, s[key], axis, n, other)
            o.set_state_f64(s["hydroFlds"], s["sgstke"], s["moist"])
            o.rk_stage(stage)
        t, it = np.float32(t + np.float32(cfg.dt)), it + 1  # the clock rule of ora_step
        o.set_clock(float(t), it)
    part = o.get_state()
    parts = [None] * world
    dist.all_gather_object(parts, part)
    res = None
    if rank == 0:
        whole = fe.halo.gather_state(parts, px, py)
        ref = Oracle(cfg)
        ref.set_inputs(inp)
        ref.step(nsteps)
        r = ref.get_state()
        res = {k: (None if r[k] is None else float(np.abs(whole[k][..., 3:-3, 3:-3, 3:-3] - r[k][..., 3:-3, 3:-3, 3:-3]).max()))
               for k in ("hydroFlds", "sgstke", "moist", "pres")}
    q.put((rank, res))
    dist.destroy_process_group()
    host.cleanup()


@pytest.mark.parametrize("px,py", [(2, 1), (1, 2), (2, 2)])
def test_slabs_with_per_stage_halo_exchange_equal_the_whole_domain(px, py):
    """Moist CBL over a hill, 16 x 12 x 8, 3 RK3 steps: oracle slabs (two, or four with corner
    neighbours) exchanging their halos over gloo before each stage give the single-domain state
    exactly."""
    res = _spawn(_oracle_slab_worker, px * py, px, py, 3)
    diffs = res[0][1]
    for k, v in diffs.items():
        if v is not None:
            assert v == 0.0, (k, v)


def _distributed_slab_worker(rank, world, port, q):
    """DistributedSlab's set-up and tear-down on a stand-in engine that records its calls."""
    dist = _init(rank, world, port)
    import ctypes
    import importlib

    fe = importlib.import_module("fasteddy-model_b200")
    log = []

    class Engine:
        def fe_ipc_handle_bytes(self):
            return 64

        def fe_arena_ipc_handle(self, h, buf, n):
            ctypes.memmove(buf, bytes([0xA0 + rank]) * 64, 64)
            return 0

        def fe_set_halo_peers(self, h, px, py, arr):
            log.append(("peers", px, py, [None if arr[t] is None else ctypes.string_at(arr[t], 64) for t in range(9)]))
            return 0

        def fe_comm_unique_id_bytes(self):
            return 128

        def fe_comm_unique_id(self, buf, n):
            ctypes.memmove(buf, b"U" * 128, 128)
            return 0

        def fe_comm_create(self, uid, n, r, dev, out):
            log.append(("comm", uid.raw, n, r, dev))
            out._obj.value = 7
            return 0

        def fe_set_halo_comm(self, h, c):
            log.append(("set_comm", None if c is None else c.value))
            return 0

        def fe_clear_halo_peers(self, h):
            log.append(("clear_peers",))
            return 0

        def fe_comm_destroy(self, c):
            log.append(("destroy_comm", c.value))
            return 0

    class Domain:
        def __init__(self, cfg, device):
            self.h, self.e = ctypes.c_void_p(1), Engine()
            log.append(("domain", cfg.Nx, cfg.Ny, device))

        def set_inputs(self, inp, simTime, simTime_it):
            log.append(("inputs", inp["hydroFlds"].shape))

        def sync(self):
            log.append(("sync",))

        def close(self):
            log.append(("close",))
            self.h = ctypes.c_void_p()

    fe.halo.Domain = Domain
    host = fe.cases.setup_host("cbl_dry", 16, 12, 8)
    slab = fe.halo.DistributedSlab(host.config(), host.inputs(), 2, 1, device=rank)
    slab.close()
    host.cleanup()
    q.put((rank, log))
    dist.destroy_process_group()


def test_distributed_slab_set_up_and_tear_down_over_gloo():
    """Two ranks, 2 x 1 slabs: each makes an 8 x 12 slab, gets the other rank's arena handle for
    its x neighbours (itself for y), the communicator of rank 0's unique id with its own rank and
    device, its slab of the inputs; on close, the peers are unmapped and the communicator
    released before the slab."""
    res = _spawn(_distributed_slab_worker, 2)
    for rank, log in res:
        other = bytes([0xA0 + 1 - rank]) * 64
        kinds = [e[0] for e in log]
        assert kinds == ["domain", "peers", "comm", "set_comm", "inputs", "sync", "clear_peers", "set_comm",
                         "destroy_comm", "close"]
        assert log[0] == ("domain", 8, 12, rank)
        assert log[1] == ("peers", 2, 1, [other, other, other, None, None, None, other, other, other])
        assert log[2] == ("comm", b"U" * 128, 2, rank, rank)
        assert log[3] == ("set_comm", 7) and log[7] == ("set_comm", None) and log[8] == ("destroy_comm", 7)
        assert log[4] == ("inputs", (5, 14, 18, 14))
