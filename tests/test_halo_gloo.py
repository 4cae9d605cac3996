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
from pdcuda.halo import (HaloExchange, bond_segments, candidate_rows, decompose,
                         distribute_equally, link_partitions, owner_of, part_body, recv_lists,
                         send_rows)
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


def exact_rows(ob, owned_points):
    """Owned points and every point bonded to one of them (from the oracle's bond lists)."""
    nb = set(int(i) for i in owned_points)
    for i in owned_points:
        nb.update(ob.nbr[ob.off[i]:ob.off[i + 1]].tolist())
    return np.array(sorted(nb))


def test_decompositions():
    body = small_plate()
    owner = decompose(body, 3, "index")
    assert [np.nonzero(owner == p)[0].tolist() for p in range(3)] == \
        [list(range(a, b)) for a, b in distribute_equally(body.n_points, 3)]
    owner = decompose(body, 4, "slabs")          # the plate is longest along x
    x = body._pos[:, 0]
    counts = np.bincount(owner, minlength=4)
    assert counts.max() - counts.min() <= 1
    for p in range(3):
        assert x[owner == p].max() <= x[owner == p + 1].min()


@pytest.mark.parametrize("how,n_parts", [("index", 2), ("index", 3), ("index", 5), ("slabs", 3)])
def test_plan_rows_and_exchange_lists(how, n_parts):
    body = small_plate()
    ob = oracle_body(body)
    owner = decompose(body, n_parts, how)
    plans = []
    for p in range(n_parts):
        own_pts = np.nonzero(owner == p)[0]
        rows = exact_rows(ob, own_pts)
        assert set(rows) <= set(candidate_rows(body, own_pts))
        owned = (owner[rows] == p).astype(np.uint8)
        recv = recv_lists(rows, owned, owner)
        # every halo row is received once, from its owner
        got = np.sort(np.concatenate([g for _, g in recv.values()])) if recv else np.array([])
        assert np.array_equal(got, rows[owned == 0])
        for src, (r, gids) in recv.items():
            assert np.array_equal(rows[r], gids) and (owner[gids] == src).all()
            if how == "index":     # contiguous point ranges: one block of rows per source
                assert r[-1] - r[0] + 1 == len(r)
        plans.append((rows, owned, recv))
    requests = [{s: g for s, (_, g) in recv.items()} for _, _, recv in plans]
    for p, (rows, owned, recv) in enumerate(plans):
        for dst, srows in send_rows(p, rows, requests).items():
            # the rows p sends to dst are the points dst holds as halo rows from p, in order
            assert np.array_equal(rows[srows], plans[dst][2][p][1])
            assert owned[srows].all()


def test_bond_segments():
    nn = np.array([2, 0, 3, 1])
    assert bond_segments(nn, [0, 2]).tolist() == [0, 1, 2, 3, 4]
    assert bond_segments(nn, [3, 1, 0]).tolist() == [5, 0, 1]
    assert bond_segments(nn, []).tolist() == []


def test_part_body_restricts_conditions_to_owned_rows():
    body = small_plate()
    ob = oracle_body(body)
    o0, o1 = distribute_equally(body.n_points, 2)[1]
    rows = exact_rows(ob, np.arange(o0, o1))
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

    def __init__(self, body, owner, part, ob_body):
        import torch
        self.part, self.n_parts = part, int(owner.max()) + 1
        self.rows = exact_rows(ob_body, np.nonzero(owner == part)[0])
        self.owned = (owner[self.rows] == part).astype(np.uint8)
        self.owned_rows = np.nonzero(self.owned)[0]
        self.sub = part_body(body, self.rows, self.owned)
        self.ob = oracle_body(self.sub)
        self.recv = recv_lists(self.rows, self.owned, owner)
        self.torch = torch

    def requests(self):
        return {s: g for s, (_, g) in self.recv.items()}

    def link(self, requests):
        self.send = send_rows(self.part, self.rows, requests)
        t = self.torch
        self.send_bufs = {0: {d: (t.from_numpy(r), t.empty(len(r) * 24, dtype=t.uint8))
                              for d, r in self.send.items()}}
        self.recv_bufs = {0: {s: t.empty(len(g) * 24, dtype=t.uint8) for s, (_, g) in self.recv.items()}}

    def pack(self, kind):
        for d, (rows, buf) in self.send_bufs[kind].items():
            buf.numpy().view(np.float64)[:] = self.ob.pos[rows.numpy()].ravel()

    def unpack(self, kind):
        for s, buf in self.recv_bufs[kind].items():
            rows, _ = self.recv[s]
            self.ob.pos[rows] = buf.numpy().view(np.float64).reshape(-1, 3)


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


def _rank(rank, world, port, how, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        body = small_plate()
        gob = oracle_body(body)
        owner = decompose(body, world, how)
        part = OraclePart(body, owner, rank, gob)
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
        own = part.owned_rows
        nn = np.diff(part.ob.off)
        bonds = part.ob.bond_active[bond_segments(nn, own)]
        out = (rank, dt, part.rows[own], part.ob.u[own].copy(), part.ob.v[own].copy(),
               bonds.copy(), nn[own])
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
@pytest.mark.parametrize("how", ["index", "slabs"])
def test_two_gloo_ranks_step_like_the_undivided_body(how):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, how, q)) for r in range(2)]
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
    u = np.empty_like(ob.u)
    v = np.empty_like(ob.v)
    nn = np.zeros(body.n_points, np.int64)
    for _, _, gids, uu, vv, _, n_nb in res:
        u[gids], v[gids], nn[gids] = uu, vv, n_nb
    bonds = np.empty(int(nn.sum()), np.uint8)
    for _, _, gids, _, _, b, _ in res:
        bonds[bond_segments(nn, gids)] = b
    assert np.array_equal(u, ob.u) and np.array_equal(v, ob.v)
    assert np.array_equal(nn, np.diff(ob.off))
    assert np.array_equal(bonds, ob.bond_active[:ob.n_bonds])
    assert np.count_nonzero(bonds == 0) > 0      # bonds failed during the run
