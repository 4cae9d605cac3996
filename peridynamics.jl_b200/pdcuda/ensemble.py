"""Ensembles of independent specimens advanced together on one device.

The reference runs parameter studies one job after the other (``Study`` / ``submit!``,
src/core/study.jl:68-283), each job with its own CFL step (velocity_verlet.jl:136-142). Here
the specimens are concatenated into device bodies: their bond graphs are disjoint (the
specimens are laid out apart), every specimen keeps its own parameter set and its own time
step (``pd_set_param_timesteps``), and every boundary condition is evaluated at the time of
its specimen.

Size classes: with ``classes=k`` the specimens are sorted by point count and cut into k
classes of (nearly) equal specimen counts, smallest first; every class is one device body with
its own point-to-lane mapping (``autotune`` chooses it per class), and one CUDA graph advances
all classes (``pd_group_run_vv``: each class's launches on its own stream). ``classes=1`` is
one body holding every specimen.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .body import Body, Condition
from .solver import DeviceBody


def _concat(bodies):
    """One body holding every given specimen; for the neighbour search the specimens are
    shifted apart along x by more than a horizon."""
    pos, vol = [], []
    x0 = 0.0
    for b in bodies:
        p = b._pos.copy()
        gap = 3.0 * max(q.delta for q in b.point_params)
        p[:, 0] += x0 - p[:, 0].min()
        x0 = p[:, 0].max() + gap
        pos.append(p)
        vol.append(b.volume)
    offsets = np.cumsum([0] + [b.n_points for b in bodies])
    P = np.concatenate([b._pos for b in bodies])
    body = Body(bodies[0].mat, P.T, np.concatenate(vol))
    # the device keeps every specimen's own coordinates (their bond vectors then round
    # exactly as in a run of the specimen alone); the neighbour search runs on the copy
    # shifted apart, so no bond joins two specimens
    body._search_pos = np.ascontiguousarray(np.concatenate(pos))
    for k, b in enumerate(bodies):
        o = offsets[k]
        body.point_params.append(b.point_params[0])
        body.params_map[o:o + b.n_points] = k + 1
        body.fail_permit[o:o + b.n_points] = b.fail_permit
        for name, pts in b.point_sets.items():
            body.point_sets[f"s{k}:{name}"] = np.asarray(pts) + o
        ren = lambda c, k=k: Condition(c.kind, c.fun, c.field, f"s{k}:{c.point_set}", c.dim, c.data)
        body.single_dim_bcs += [ren(c) for c in b.single_dim_bcs]
        body.posdep_single_dim_bcs += [ren(c) for c in b.posdep_single_dim_bcs]
        for c in b.data_bcs:
            # DataBC matrices cover the points of one specimen: widen to all points
            cc = ren(c)
            cc.data = np.full((c.data.shape[0], offsets[-1]), np.nan)
            cc.data[:, o:o + b.n_points] = c.data
            body.data_bcs.append(cc)
        body.single_dim_ics += [ren(c) for c in b.single_dim_ics]
        body.posdep_single_dim_ics += [ren(c) for c in b.posdep_single_dim_ics]
    # pre-cracks: the c-th crack of every specimen (of one mode) becomes one crack of the
    # ensemble. No bond joins two specimens, so the union of the a-sets against the union
    # of the b-sets selects exactly the bonds each specimen's own crack selects.
    for mode in (True, False):
        per = [[(a, c) for a, c, f in b.point_sets_precracks if f == mode] for b in bodies]
        for c in range(max((len(p) for p in per), default=0)):
            sa, sb = [], []
            for k, p in enumerate(per):
                if c < len(p):
                    o = offsets[k]
                    sa.append(np.asarray(bodies[k].point_sets[p[c][0]]) + o)
                    sb.append(np.asarray(bodies[k].point_sets[p[c][1]]) + o)
            tag = "filter" if mode else "damage"
            body.point_sets[f"{tag}{c}:a"] = np.concatenate(sa)
            body.point_sets[f"{tag}{c}:b"] = np.concatenate(sb)
            body.point_sets_precracks.append((f"{tag}{c}:a", f"{tag}{c}:b", mode))
    return body, offsets


class Ensemble:
    """Specimens (Body objects of one material type, one parameter set each) on one device,
    in `classes` size classes."""

    def __init__(self, bodies, precision="fp32", device=0, graph_steps=0, safety_factor=0.7,
                 classes=1):
        if not bodies:
            raise ValueError("an ensemble needs at least one body")
        mat_t = type(bodies[0].mat)
        for b in bodies:
            if type(b.mat) is not mat_t:
                raise ValueError("all specimens of an ensemble must use the same material type")
            if len(b.point_params) != 1:
                raise ValueError("every specimen of an ensemble has exactly one parameter set")
            if np.any(b.params_map == 0):
                raise ValueError("not all points have material parameters: use material!")
        self.bodies = list(bodies)
        n_cls = max(1, min(int(classes), len(self.bodies)))
        order = np.argsort([b.n_points for b in self.bodies], kind="stable")
        cut = [len(order) * c // n_cls for c in range(n_cls + 1)]
        # members of every class in specimen order (one class: all specimens, as given)
        self.members = [sorted(int(k) for k in order[cut[c]:cut[c + 1]]) for c in range(n_cls)]
        self.devs, self.offsets, self.where = [], [], {}
        self.dt = np.empty(len(self.bodies))
        self.graph_steps = int(graph_steps)
        for c, mem in enumerate(self.members):
            combined, offsets = _concat([self.bodies[k] for k in mem])
            dev = DeviceBody(combined, precision=precision, device=device, independent_params=True)
            _, dts = dev.stable_timestep(safety_factor, per_param=True)
            dev.set_param_timesteps(dts.copy())
            if graph_steps and n_cls == 1:
                dev.set_graph(graph_steps)
            for q, k in enumerate(mem):
                self.where[k] = (c, q)
                self.dt[k] = dts[q]
            self.devs.append(dev)
            self.offsets.append(offsets)
        # one class: the device body of every specimen
        self.dev = self.devs[0] if n_cls == 1 else None
        self._group = None
        if n_cls > 1:
            hs = (C.c_void_p * n_cls)(*[d.h.value for d in self.devs])
            g = C.c_void_p()
            L.check(L.lib().pd_group_create(hs, n_cls, C.byref(g)), "pd_group_create")
            self._group = g

    # -- per class ----------------------------------------------------------------------------
    def autotune(self):
        """Chooses every class's mapping by timing the candidates on it; returns
        [(lanes per point, block size, bond-stream variant)] per class."""
        for d in self.devs:
            d.autotune()
        return self.mappings()

    def mappings(self):
        return [d.mapping() for d in self.devs]

    def set_mapping(self, group, block=256):
        for d in self.devs:
            d.set_mapping(group, block)

    def info(self):
        """(points, bonds) of the whole ensemble."""
        n = nb = 0
        for d in self.devs:
            a, b, _ = d.info()
            n += a
            nb += b
        return n, nb

    def class_info(self):
        """Per class: specimens, points, bonds, mapping."""
        out = []
        for c, d in enumerate(self.devs):
            n, nb, _ = d.info()
            g, b, p = d.mapping()
            out.append({"specimens": len(self.members[c]), "points": int(n), "bonds": int(nb),
                        "point_range": [int(min(self.bodies[k].n_points for k in self.members[c])),
                                        int(max(self.bodies[k].n_points for k in self.members[c]))],
                        "mapping": {"group": g, "block": b, "pipe": p}})
        return out

    def launch_count(self):
        return sum(d.launch_count() for d in self.devs)

    # -- stepping ------------------------------------------------------------------------------
    def run(self, n_steps, first_step=1):
        """Velocity Verlet steps of every specimen with its own time step (the reference's
        initialize! force evaluation happens before the first block)."""
        if first_step == 1:
            for d in self.devs:
                d.force(0.0, float(self.dt.min()))
        if self._group is None:
            self.dev.run(first_step, n_steps, -1.0)
        else:
            self._run_group(first_step, n_steps, None)

    def _run_group(self, first_step, n_steps, ms):
        for d in self.devs:
            d.tabulate_bcs(first_step, n_steps, -1.0)
        st = L.lib().pd_group_run_vv(self._group, first_step, n_steps, -1.0, self.graph_steps,
                                     None if ms is None else C.byref(ms))
        if st == L.PD_ERR_NAN:
            for d in self.devs:
                s = C.c_int64()
                L.lib().pd_nan_step(d.h, C.byref(s))
                if s.value >= 0:
                    raise L.NaNError(float("nan"), s.value)
        L.check(st, "pd_group_run_vv")

    def run_timed(self, first_step, n_steps, phases=True):
        """run() timed on the device. phases=True (one class): (total, force phase A, phase B,
        integration) ms with events around every kernel; phases=False: the steps as run()
        issues them (graphs), total ms."""
        if self._group is None:
            return self.dev.run_timed(first_step, n_steps, -1.0, phases=phases)
        if phases:
            raise ValueError("per-phase times of several classes: use class_phase_times")
        ms = C.c_double()
        self._run_group(first_step, n_steps, ms)
        return ms.value

    def class_phase_times(self, first_step, n_steps):
        """Every class alone for the same steps, eagerly with events around every kernel:
        [(total, phase A, phase B, integration) ms] per class (advances every class)."""
        return [d.run_timed(first_step, n_steps, -1.0) for d in self.devs]

    def field(self, name, k):
        """Storage field of specimen k: 3 x n_k (9 x n_k) point vectors (tensors), n_k point
        scalars, or the bond_active bytes of its bonds."""
        c, q = self.where[k]
        dev, offsets = self.devs[c], self.offsets[c]
        f = dev.field(name)
        o, m = offsets[q], self.bodies[k].n_points
        if name == "bond_active":
            nn = np.concatenate([[0], np.cumsum(dev.field("n_neighbors"))])
            return f[nn[o]:nn[o + m]]
        return f[..., o:o + m]

    def close(self):
        if self._group is not None:
            L.lib().pd_group_destroy(self._group)
            self._group = None
        for d in self.devs:
            d.close()
