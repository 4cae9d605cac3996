"""The partition plan and the halo exchange of pdcuda/halo.py on CPU (no GPU): the reference's
decomposition (distribute_equally, decomposition.jl:32-58), halo rows and exchange lists
checked against the body's bond lists, and two gloo ranks (127.0.0.1) stepping a bond-based
plate through HaloExchange with the FP64 oracle as the force, bit-identical to the undivided
body. The device side of the same path is tests/test_gpu_halo.py."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import pdcuda as pd
from pdcuda.halo import (HaloExchange, candidate_rows, distribute_equally, link_partitions,
                         owner_of, part_body, recv_blocks, send_rows)
from helpers import oracle_body, plate_body


def test_distribute_equally_matches_reference():
    # decomposition.jl:32-58 (1-based ranges 1:4, 5:7, 8:10 there)
    assert distribute_equally(10, 3) == [(0, 4), (4, 7), (7, 10)]
    assert distribute_equally(9, 3) == [(0, 3), (3, 6), (6, 9)]
    assert distribute_equally(5, 5) == [(k, k + 1) for k in range(5)]
    # fewer elements than chunks: one element each, the rest empty
    r = distribute_equally(2, 4)
    assert r[:2] == [(0, 1), (1, 2)] and all(a == b for a, b in r[2:])
    assert owner_of(distribute_equally(10, 3), [0, 3, 4, 6, 7, 9]).tolist() == [0, 0, 1, 1, 2, 2]


def small_plate():
    body = plate_body(pd.BBMaterial(), nx=16, ny=8, nz=3, v=0.5, Gc=50.0)
    return body


def exact_rows(ob, o0, o1):
    """Owned points and every point bonded to one of them (from the oracle's bond lists)."""
    nb = set(range(o0, o1))
    for i in range(o0, o1):
        nb.update(ob.nbr[ob.off[i]:ob.off[i + 1]].tolist())
    return np.array(sorted(nb))


@pytest.mark.parametrize("n_parts", [2, 3, 5])
def test_plan_rows_and_exchange_lists(n_parts):
    body = small_plate()
    ob = oracle_body(body)
    ranges = distribute_equally(body.n_points, n_parts)
    plans = []
    for p, (o0, o1) in enumerate(ranges):
        rows = exact_rows(ob, o0, o1)
        assert set(rows) <= set(candidate_rows(body, o0, o1))
        owned = ((rows >= o0) & (rows < o1)).astype(np.uint8)
        recv = recv_blocks(rows, owned, ranges)
        # every halo row is received once, from its owner, in a contiguous block
        got = np.sort(np.concatenate([g for _, g in recv.values()])) if recv else np.array([])
        assert np.array_equal(got, rows[owned == 0])
        for src, (row0, gids) in recv.items():
            assert np.array_equal(rows[row0:row0 + len(gids)], gids)
            assert all(ranges[src][0] <= g < ranges[src][1] for g in gids)
        plans.append((rows, owned, recv, int(np.searchsorted(rows, o0))))
    requests = [{s: g for s, (_, g) in recv.items()} for _, _, recv, _ in plans]
    for p, (rows, owned, recv, own0) in enumerate(plans):
        for dst, srows in send_rows(p, ranges, own0, requests).items():
            # the rows p sends to dst are the points dst holds as halo rows from p, in order
            assert np.array_equal(rows[srows], plans[dst][2][p][1])
            assert owned[srows].all()


def test_part_body_restricts_conditions_to_owned_rows():
    body = small_plate()
    ob = oracle_body(body)
    o0, o1 = distribute_equally(body.n_points, 2)[1]
    rows = exact_rows(ob, o0, o1)
    owned = ((rows >= o0) & (rows < o1)).astype(np.uint8)
    sub = part_body(body, rows, owned)
    top = body.point_sets["top"]
    assert np.array_equal(rows[sub.point_sets["top"]], top[(top >= o0) & (top < o1)])
    # the pre-crack sets keep their halo rows
    a, b, filt = sub.point_sets_precracks[0]
    ga = body.point_sets["crack_a"]
    assert np.array_equal(np.sort(rows[sub.point_sets[a]]), np.sort(ga[np.isin(ga, rows)]))
    assert filt


# -- two gloo ranks --------------------------------------------------------------------------
class OraclePart:
    """A partition whose force is the FP64 oracle on its rows (halo rows bonded to all rows
    in reach: only the owned rows' forces are used)."""

    def __init__(self, body, ranges, part, ob_body):
        import torch
        o0, o1 = ranges[part]
        self.part, self.n_parts, self.ranges = part, len(ranges), ranges
        self.rows = exact_rows(ob_body, o0, o1)
        self.owned = ((self.rows >= o0) & (self.rows < o1)).astype(np.uint8)
        self.sub = part_body(body, self.rows, self.owned)
        self.ob = oracle_body(self.sub)
        self.own_row0 = int(np.searchsorted(self.rows, o0))
        self.n_owned = o1 - o0
        self.recv = recv_blocks(self.rows, self.owned, ranges)
        self.torch = torch

    def requests(self):
        return {s: g for s, (_, g) in self.recv.items()}

    def link(self, requests):
        self.send = send_rows(self.part, self.ranges, self.own_row0, requests)
        t = self.torch
        self.send_bufs = {0: {d: (t.from_numpy(r), t.empty(len(r) * 24, dtype=t.uint8))
                              for d, r in self.send.items()}}
        self.recv_bufs = {0: {s: t.empty(len(g) * 24, dtype=t.uint8) for s, (_, g) in self.recv.items()}}

    def pack(self, kind):
        for d, (rows, buf) in self.send_bufs[kind].items():
            buf.numpy().view(np.float64)[:] = self.ob.pos[rows.numpy()].ravel()

    def unpack(self, kind):
        for s, buf in self.recv_bufs[kind].items():
            row0, g = self.recv[s]
            self.ob.pos[row0:row0 + len(g)] = buf.numpy().view(np.float64).reshape(-1, 3)


def vv_steps(ob, sets, n, dt, v, exchange=None):
    """Velocity Verlet (velocity_verlet.jl:239-295) in numpy around the oracle's force: the
    top / bottom rows held at +-v in y."""
    rho = np.array([ob.params_list[k].rho for k in ob.pid])[:, None]
    for step in range(1, n + 1):
        ob.vh[:] = ob.v + 0.5 * dt * ob.a
        ob.vh[sets["top"], 1] = v
        ob.vh[sets["bottom"], 1] = -v
        du = ob.vh * dt
        ob.u += du
        ob.pos += du
        if exchange is not None:
            exchange(0)
        ob.force_density(step * dt, dt)
        ob.a[:] = (ob.b_int + ob.b_ext) / rho
        ob.v[:] = ob.vh + 0.5 * dt * ob.a


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        body = small_plate()
        gob = oracle_body(body)
        ranges = distribute_equally(body.n_points, world)
        part = OraclePart(body, ranges, rank, gob)
        link_partitions([part], dist)
        # calc_stable_timestep: the minimum over the ranks is the body's step
        import torch
        t = torch.tensor([part.ob.stable_timestep(0.7)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        dt = float(t.item())
        ex = HaloExchange([part], dist)
        ex(0)
        part.ob.force_density(0.0, dt)
        vv_steps(part.ob, part.sub.point_sets, 40, dt, 0.5, exchange=ex)
        sl = slice(part.own_row0, part.own_row0 + part.n_owned)
        nn = np.diff(part.ob.off)
        off = np.concatenate(([0], np.cumsum(nn)))
        bonds = part.ob.bond_active[off[part.own_row0]:off[part.own_row0 + part.n_owned]]
        out = (rank, dt, part.ob.u[sl].copy(), part.ob.v[sl].copy(), bonds.copy())
        gathered = [None] * world
        dist.all_gather_object(gathered, out)
        if rank == 0:
            q.put(gathered)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(180)
def test_two_gloo_ranks_step_like_the_undivided_body():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=150), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    body = small_plate()
    ob = oracle_body(body)
    dt = ob.stable_timestep(0.7)
    assert all(r[1] == dt for r in res)
    ob.force_density(0.0, dt)
    vv_steps(ob, body.point_sets, 40, dt, 0.5)
    u = np.concatenate([r[2] for r in res])
    v = np.concatenate([r[3] for r in res])
    bonds = np.concatenate([r[4] for r in res])
    assert np.array_equal(u, ob.u) and np.array_equal(v, ob.v)
    assert np.array_equal(bonds, ob.bond_active[:ob.n_bonds])
    assert np.count_nonzero(bonds == 0) > 0      # bonds failed during the run
