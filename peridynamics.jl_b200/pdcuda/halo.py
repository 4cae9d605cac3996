"""Partitioned bodies: one partition per GPU, halo exchange between the stages of a step.

The reference's MPI data handler (src/core/mpi_body_data_handler.jl) re-expressed for GPUs:

- the body's points are cut into contiguous index ranges, one per rank (PointDecomposition /
  distribute_equally, src/discretization/decomposition.jl:32-63; mpi_data_handler :81-100),
  or, as an option, into slabs of equal point counts along the body's longest extent, which
  cross the body where it is thinnest (fewer halo points when the point order runs along a
  short side);
- a partition holds its owned points and the halo points bonded to them, in the body's point
  order (chop_body_mpi :102-109, get_halo_infos :111-125). Halo rows carry only their bonds to
  owned points (pd_create_partition), so every owned point keeps the bond list and the
  summation order of the undivided body;
- before every force evaluation the owners' point state is copied into the halo rows
  (exchange_loc_to_halo!, :239-318). The reference scatters the force contributions of its
  state-based materials into halo rows and adds them back afterwards (exchange_halo_to_loc!,
  :320-398); these kernels gather instead, so their second exchange runs in the same
  direction as the first: the per-point state of the first force kernel (OSB: weighted volume
  and dilatation terms; CMat: F and P K^-1, killed flag) into the halo rows before the second.

Transfers are torch.distributed point-to-point operations (NCCL between GPUs, gloo between
CPU processes) issued on the partitions' stream, or device copies when one process holds
several partitions of a body on one GPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .body import Body, Condition
from .materials import BBMaterial, EnergySurfaceCorrection


def torch_int32():
    import torch
    return torch.int32


def distribute_equally(n_elems, n_chunks):
    """distribute_equally (decomposition.jl:32-58) as 0-based half-open (start, stop) ranges;
    with fewer elements than chunks the chunks past the last element are empty."""
    if n_chunks < 1:
        raise ValueError("n_chunks must be >= 1")
    if n_elems >= n_chunks:
        size, rem = divmod(n_elems, n_chunks)
        sidx = [i * size + min(i, rem) for i in range(n_chunks + 1)]
        return [(sidx[i], sidx[i + 1]) for i in range(n_chunks)]
    return [(i, i + 1) if i < n_elems else (n_elems, n_elems) for i in range(n_chunks)]


def owner_of(ranges, points):
    """Index of the range that holds each point number."""
    stops = np.array([r[1] for r in ranges])
    return np.searchsorted(stops, np.asarray(points), side="right")


def decompose(body, n_parts, how="index"):
    """The partition that owns every point. "index": the reference's PointDecomposition,
    contiguous ranges of point numbers (distribute_equally); "slabs": the same counts taken
    along the body's longest extent (points ordered by that coordinate, then by number), so
    that the cuts cross the body where it is thinnest."""
    n = body.n_points
    ranges = distribute_equally(n, n_parts)
    owner = np.empty(n, np.int32)
    if how == "index":
        order = np.arange(n)
    elif how == "slabs":
        X = body._pos
        axis = int(np.argmax(X.max(axis=0) - X.min(axis=0)))
        order = np.lexsort((np.arange(n), X[:, axis]))
    else:
        raise ValueError('decomposition must be "index" or "slabs"')
    for p, (a, b) in enumerate(ranges):
        owner[order[a:b]] = p
    return owner


def candidate_rows(body, owned_points):
    """The owned points and every point inside their bounding box grown by the largest
    horizon: a superset of the halo (a bond is never longer than its owner's horizon)."""
    X = body._pos
    dmax = max(p.delta for p in body.point_params)
    own = X[owned_points]
    lo = own.min(axis=0) - dmax * (1 + 1e-12)
    hi = own.max(axis=0) + dmax * (1 + 1e-12)
    inside = np.all((X >= lo) & (X <= hi), axis=1)
    inside[owned_points] = True
    return np.nonzero(inside)[0]


def recv_lists(rows, owned, owner):
    """{source partition: (rows (int32), point numbers)} of the halo rows, by owner."""
    halo_rows = np.nonzero(~np.asarray(owned, bool))[0]
    halo = rows[halo_rows]
    src_of = owner[halo]
    out = {}
    for src in np.unique(src_of):
        idx = np.nonzero(src_of == src)[0]
        out[int(src)] = (np.ascontiguousarray(halo_rows[idx], np.int32), halo[idx])
    return out


def send_rows(part, rows, requests):
    """{destination partition: rows (int32)} this partition sends: requests[r] is partition
    r's {source: point numbers} of its halo rows; rows are this partition's point numbers."""
    out = {}
    for r, req in enumerate(requests):
        if r != part and part in req:
            gids = np.asarray(req[part])
            idx = np.searchsorted(rows, gids)
            if not np.array_equal(rows[np.minimum(idx, len(rows) - 1)], gids):
                raise AssertionError(f"partition {r} asks partition {part} for points it does not hold")
            out[r] = np.ascontiguousarray(idx, np.int32)
    return out


def bond_segments(nn, rows):
    """Flat indices of the bonds of the given rows in a CSR with bond counts nn."""
    rows = np.asarray(rows)
    if len(rows) == 0:
        return np.zeros(0, np.int64)
    off = np.concatenate(([0], np.cumsum(nn)))
    cnt = nn[rows]
    starts = np.repeat(off[rows] - np.concatenate(([0], np.cumsum(cnt)[:-1])), cnt)
    return starts + np.arange(int(cnt.sum()))


def part_body(body, rows, owned):
    """The partition's Body over `rows` (sorted point numbers of body). Point sets hold only
    owned rows, so conditions and initial conditions act on owned points; pre-crack sets also
    keep their halo rows, so bonds between owned and halo points are cut as in the body."""
    owned = np.asarray(owned, bool)
    sub = Body(body.mat, body._pos[rows].T, body.volume[rows])
    sub.point_params = body.point_params
    sub.params_map = body.params_map[rows].copy()
    sub.fail_permit = body.fail_permit[rows].copy()
    local = np.full(body.n_points, -1, np.int64)
    local[rows] = np.arange(len(rows))
    sub.point_sets = {}
    for name, pts in body.point_sets.items():
        r = local[pts]
        r = r[r >= 0]
        sub.point_sets[name] = r[owned[r]]
    for k, (a, b, filt) in enumerate(body.point_sets_precracks):
        names = []
        for tag, s in (("a", a), ("b", b)):
            r = local[body.point_sets[s]]
            name = f"__partition_crack_{k}_{tag}"
            sub.point_sets[name] = r[r >= 0]
            names.append(name)
        sub.point_sets_precracks.append((names[0], names[1], filt))
    sub.single_dim_bcs = list(body.single_dim_bcs)
    sub.posdep_single_dim_bcs = list(body.posdep_single_dim_bcs)
    sub.pos_single_dim_bcs = list(body.pos_single_dim_bcs)
    sub.data_bcs = [Condition(c.kind, c.fun, c.field, c.point_set, c.dim, data=c.data[:, rows])
                    for c in body.data_bcs]
    sub.single_dim_ics = list(body.single_dim_ics)
    sub.posdep_single_dim_ics = list(body.posdep_single_dim_ics)
    return sub


class Partition:
    """Partition `part` of `n_parts` of a body on one device (chop_body_mpi): a DeviceBody over
    its owned and halo rows (in the body's point order), and the rows it receives and sends.
    owner: the partition of every point (decompose; computed from `decomposition` if None)."""

    def __init__(self, body, n_parts, part, precision="fp64", device=0, decomposition="index",
                 owner=None):
        from .solver import DeviceBody
        self.body, self.n_parts, self.part = body, n_parts, part
        self.precision, self.device = precision, device
        self.owner = decompose(body, n_parts, decomposition) if owner is None else owner
        owned_points = np.nonzero(self.owner == part)[0]
        if len(owned_points) == 0:
            raise ValueError(f"partition {part} of {n_parts} has no points")
        rows = candidate_rows(body, owned_points)
        owned = (self.owner[rows] == part).astype(np.uint8)
        dev = DeviceBody(part_body(body, rows, owned), precision, device, owned=owned)
        keep = owned.astype(bool) | (dev.field("n_neighbors") > 0)
        if not keep.all():  # candidates without a bond to an owned point
            dev.close()
            rows = rows[keep]
            owned = owned[keep]
            dev = DeviceBody(part_body(body, rows, owned), precision, device, owned=owned)
        self.dev, self.rows, self.owned = dev, rows, owned
        self.owned_rows = np.nonzero(owned)[0]
        self.n_owned = len(self.owned_rows)
        self.recv = recv_lists(rows, owned, self.owner)
        self.send = {}

    def requests(self):
        return {src: gids for src, (_, gids) in self.recv.items()}

    def link(self, requests):
        self.send = send_rows(self.part, self.rows, requests)

    def break_random_pairs(self, fraction, seed):
        """pd_break_random_pairs on the body's point numbers: the same pairs as the body."""
        ids = np.ascontiguousarray(self.rows, np.int64)
        L.check(L.lib().pd_break_random_pairs_ids(self.dev.h, float(fraction), int(seed), L.ptr(ids)),
                "pd_break_random_pairs_ids")

    def owned_field(self, name):
        """A point field of the owned rows (3 x n_owned or n_owned, in the body's point order);
        bond_active: the bonds of the owned rows, which are the body's bonds of these points."""
        if name == "bond_active":
            nn = self.dev.field("n_neighbors")
            return self.dev.field("bond_active")[bond_segments(nn, self.owned_rows)]
        f = self.dev.field(name)
        return f[..., self.owned_rows] if f.ndim == 2 else f[self.owned_rows]

    # -- halo data on the device -----------------------------------------------------------
    def alloc_buffers(self, kinds, torch_device):
        import torch
        self.send_bufs, self.recv_bufs, self.row_bytes = {}, {}, {}
        for kind in kinds:
            rb = C.c_int64()
            L.check(L.lib().pd_halo_row_bytes(self.dev.h, kind, C.byref(rb)), "pd_halo_row_bytes")
            rb = self.row_bytes[kind] = rb.value
            self.send_bufs[kind] = {
                dst: (torch.from_numpy(rows).to(torch_device),
                      torch.empty(len(rows) * rb, dtype=torch.uint8, device=torch_device))
                for dst, rows in self.send.items()}
            self.recv_bufs[kind] = {
                src: torch.empty(len(gids) * rb, dtype=torch.uint8, device=torch_device)
                for src, (_, gids) in self.recv.items()}
        self.recv_rows = {src: torch.from_numpy(rows).to(torch_device)
                          for src, (rows, _) in self.recv.items()}

    def _check_buffer(self, kind, rows, buf):
        # the kernels write rows x row bytes: the buffer must hold exactly that
        if buf.numel() != len(rows) * self.row_bytes[kind] or rows.dtype != torch_int32():
            raise ValueError("halo buffer does not match its row list")

    def pack(self, kind):
        for dst, (rows, buf) in self.send_bufs[kind].items():
            self._check_buffer(kind, rows, buf)
            L.check(L.lib().pd_halo_pack(self.dev.h, kind, C.c_void_p(rows.data_ptr()), len(rows),
                                         C.c_void_p(buf.data_ptr())), "pd_halo_pack")

    def unpack(self, kind):
        for src, buf in self.recv_bufs[kind].items():
            rows = self.recv_rows[src]
            self._check_buffer(kind, rows, buf)
            L.check(L.lib().pd_halo_unpack(self.dev.h, kind, C.c_void_p(rows.data_ptr()), len(rows),
                                           C.c_void_p(buf.data_ptr())), "pd_halo_unpack")

    def close(self):
        self.dev.close()


class HaloExchange:
    """Moves one kind of halo data between the partitions: every partition packs the rows its
    neighbours need, the buffers travel (torch.distributed point-to-point operations, or
    in-process copies when dist is None and this process holds all partitions), and every
    partition unpacks into its halo rows. Partitions provide send_bufs[kind] = {dst: (rows,
    buffer)}, recv_bufs[kind] = {src: buffer}, pack(kind) and unpack(kind)."""

    def __init__(self, parts, dist=None):
        self.parts, self.dist = parts, dist

    def __call__(self, kind):
        for p in self.parts:
            p.pack(kind)
        self.transfer(kind)
        for p in self.parts:
            p.unpack(kind)

    def transfer(self, kind):
        if self.dist is None:
            by = {p.part: p for p in self.parts}
            for p in self.parts:
                for src, buf in p.recv_bufs[kind].items():
                    buf.copy_(by[src].send_bufs[kind][p.part][1])
            return
        ops = []
        for p in self.parts:
            for dst, (_, buf) in sorted(p.send_bufs[kind].items()):
                ops.append(self.dist.P2POp(self.dist.isend, buf, dst))
            for src, buf in sorted(p.recv_bufs[kind].items()):
                ops.append(self.dist.P2POp(self.dist.irecv, buf, src))
        if ops:
            for w in self.dist.batch_isend_irecv(ops):
                w.wait()


def link_partitions(parts, dist=None):
    """Every partition learns which of its rows the others hold as halo rows
    (find_halo_exchanges, :142-162): gathered over the ranks when dist is given."""
    reqs = {p.part: p.requests() for p in parts}
    if dist is not None:
        gathered = [None] * dist.get_world_size()
        dist.all_gather_object(gathered, reqs)
        reqs = {}
        for g in gathered:
            reqs.update(g)
    n_parts = parts[0].n_parts
    requests = [reqs.get(r, {}) for r in range(n_parts)]
    for p in parts:
        p.link(requests)


class PartitionedBody:
    """The partitions of a body that this process holds (all of them on one device when
    dist is None; its own one per rank otherwise), stepping together: the Velocity Verlet
    stages of every partition with the halo exchanges between them, on one stream."""

    def __init__(self, parts, dist=None, device=0):
        import torch
        self.parts, self.dist, self.device = parts, dist, device
        link_partitions(parts, dist)
        self.torch_device = torch.device("cuda", device)
        self.stream = torch.cuda.Stream(device=self.torch_device)
        for p in parts:
            L.check(L.lib().pd_set_stream(p.dev.h, C.c_void_p(self.stream.cuda_stream)), "pd_set_stream")
        self.state_based = not isinstance(parts[0].body.mat, BBMaterial)
        self.kinds = (0, 1) if self.state_based else (0,)
        esc = isinstance(getattr(parts[0].body.mat, "correction", None), EnergySurfaceCorrection)
        for p in parts:
            p.alloc_buffers(self.kinds + ((2,) if esc else ()), self.torch_device)
        self.exchange = HaloExchange(parts, dist)
        if esc:
            # initialize! of the correction (bond_system_corrections.jl:86-94): the owners'
            # multiplication factors reach the halo rows before the bond factors are formed
            import torch
            with torch.cuda.stream(self.stream):
                for p in parts:
                    L.check(L.lib().pd_esc_init(p.dev.h, 1), "pd_esc_init")
                self.exchange(2)
                for p in parts:
                    L.check(L.lib().pd_esc_init(p.dev.h, 2), "pd_esc_init")

    # -- reductions over ranks (MPI.Allreduce of the reference) -----------------------------
    def _reduce(self, x, op):
        if self.dist is None:
            return x
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.torch_device)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def stable_timestep(self, safety_factor=0.7):
        """calc_stable_timestep (velocity_verlet.jl:149-153): the minimum over the partitions."""
        dt = min(p.dev.stable_timestep(safety_factor) for p in self.parts)
        return self._reduce(dt, self.dist.ReduceOp.MIN if self.dist else None)

    def _finish(self, statuses, t, dt):
        nan = max((1.0 if st == L.PD_ERR_NAN else 0.0) for st in statuses)
        nan = self._reduce(nan, self.dist.ReduceOp.MAX if self.dist else None)
        for st in statuses:
            if st not in (L.PD_OK, L.PD_ERR_NAN):
                L.check(st, "partitioned step")
        if nan:
            raise L.NaNError(t, -1)

    def force(self, t, dt):
        """initialize! (calc_force_density!(dh, 0, Δt), mpi_body_data_handler.jl:400-409)."""
        import torch
        lib = L.lib()
        with torch.cuda.stream(self.stream):
            self.exchange(0)
            for p in self.parts:
                L.check(lib.pd_force_phase(p.dev.h, 1, t, dt), "pd_force_phase")
            if self.state_based:
                self.exchange(1)
            statuses = [lib.pd_force_phase(p.dev.h, 2, t, dt) for p in self.parts]
        self._finish(statuses, t, dt)

    def run(self, first_step, n_steps, dt, timed=False):
        """n_steps Velocity Verlet steps from first_step (verlet_timestep!, velocity_verlet.jl:
        226-237, on every partition). timed: CUDA events on the partitions' stream at every
        stage boundary; returns milliseconds {total, integrate, halo_0, force_a, halo_1,
        force_b} summed over the steps."""
        import torch
        lib = L.lib()
        for p in self.parts:
            p.dev.tabulate_bcs(first_step, n_steps, dt)
            L.check(lib.pd_vv_begin(p.dev.h, first_step, n_steps, dt), "pd_vv_begin")
        ev = []

        def mark():
            if timed:
                e = torch.cuda.Event(enable_timing=True)
                e.record(self.stream)
                ev.append(e)

        with torch.cuda.stream(self.stream):
            for k in range(n_steps):
                mark()
                for p in self.parts:
                    L.check(lib.pd_vv_stage(p.dev.h, 0, k), "pd_vv_stage")
                mark()
                self.exchange(0)
                mark()
                for p in self.parts:
                    L.check(lib.pd_vv_stage(p.dev.h, 1, k), "pd_vv_stage")
                mark()
                if self.state_based:
                    self.exchange(1)
                    mark()
                    for p in self.parts:
                        L.check(lib.pd_vv_stage(p.dev.h, 2, k), "pd_vv_stage")
                    mark()
            mark()
            statuses = [lib.pd_vv_end(p.dev.h) for p in self.parts]
            mark()
        self._finish(statuses, (first_step + n_steps - 1) * dt, dt)
        if not timed:
            return None
        self.stream.synchronize()
        per = 6 if self.state_based else 4
        names = ("integrate", "halo_0", "force_a", "halo_1", "force_b")[:per - 1]
        out = dict.fromkeys(names, 0.0)
        for k in range(n_steps):
            base = k * per
            for j, nm in enumerate(names):
                out[nm] += ev[base + j].elapsed_time(ev[base + j + 1])
        out["integrate"] += ev[-2].elapsed_time(ev[-1])
        out["total"] = ev[0].elapsed_time(ev[-1])
        return out

    def field(self, name):
        """A field of the whole body assembled from the owned rows (all partitions held by
        this process); bond_active in the body's bond order."""
        if len(self.parts) != self.parts[0].n_parts:
            raise ValueError("field() needs every partition in this process (dist is None)")
        n = self.parts[0].body.n_points
        if name == "bond_active":
            nn = np.zeros(n, np.int64)
            for p in self.parts:
                nn[p.rows[p.owned_rows]] = p.dev.field("n_neighbors")[p.owned_rows]
            out = np.empty(int(nn.sum()), np.uint8)
            for p in self.parts:
                out[bond_segments(nn, p.rows[p.owned_rows])] = p.owned_field(name)
            return out
        out = None
        for p in self.parts:
            v = p.owned_field(name)
            if out is None:
                out = np.empty(v.shape[:-1] + (n,), v.dtype)
            out[..., p.rows[p.owned_rows]] = v
        return out

    def close(self):
        for p in self.parts:
            p.close()
