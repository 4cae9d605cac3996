"""Ensembles of independent specimens advanced together on one device.

The reference runs parameter studies one job after the other (``Study`` / ``submit!``,
src/core/study.jl:68-283), each job with its own CFL step (velocity_verlet.jl:136-142). Here
the specimens are concatenated into one device body: their bond graphs are disjoint (the
specimens are laid out apart), every specimen keeps its own parameter set and its own time
step (``pd_set_param_timesteps``), and every boundary condition is evaluated at the time of
its specimen. One launch sequence (CUDA-graph captured when requested) advances all of them.
"""
from __future__ import annotations

import numpy as np

from .body import Body, Condition
from .solver import DeviceBody


class Ensemble:
    """Specimens (Body objects of one material type, one parameter set each) on one device."""

    def __init__(self, bodies, precision="fp32", device=0, graph_steps=0, safety_factor=0.7):
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
        self.offsets = np.cumsum([0] + [b.n_points for b in bodies])
        self.combined = self._concat()
        self.dev = DeviceBody(self.combined, precision=precision, device=device,
                              independent_params=True)
        if graph_steps:
            self.dev.set_graph(graph_steps)
        _, dts = self.dev.stable_timestep(safety_factor, per_param=True)
        self.dt = dts.copy()
        self.dev.set_param_timesteps(self.dt)

    def _concat(self):
        """One body holding every specimen; for the neighbour search the specimens are shifted
        apart along x by more than a horizon."""
        pos, vol = [], []
        x0 = 0.0
        for b in self.bodies:
            p = b._pos.copy()
            gap = 3.0 * max(q.delta for q in b.point_params)
            p[:, 0] += x0 - p[:, 0].min()
            x0 = p[:, 0].max() + gap
            pos.append(p)
            vol.append(b.volume)
        P = np.concatenate([b._pos for b in self.bodies])
        body = Body(self.bodies[0].mat, P.T, np.concatenate(vol))
        # the device keeps every specimen's own coordinates (their bond vectors then round
        # exactly as in a run of the specimen alone); the neighbour search runs on the copy
        # shifted apart, so no bond joins two specimens
        body._search_pos = np.ascontiguousarray(np.concatenate(pos))
        for k, b in enumerate(self.bodies):
            o = self.offsets[k]
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
                cc.data = np.full((c.data.shape[0], self.offsets[-1]), np.nan)
                cc.data[:, o:o + b.n_points] = c.data
                body.data_bcs.append(cc)
            body.single_dim_ics += [ren(c) for c in b.single_dim_ics]
            body.posdep_single_dim_ics += [ren(c) for c in b.posdep_single_dim_ics]
        # pre-cracks: the c-th crack of every specimen (of one mode) becomes one crack of the
        # ensemble. No bond joins two specimens, so the union of the a-sets against the union
        # of the b-sets selects exactly the bonds each specimen's own crack selects.
        for mode in (True, False):
            per = [[(a, c) for a, c, f in b.point_sets_precracks if f == mode] for b in self.bodies]
            for c in range(max((len(p) for p in per), default=0)):
                sa, sb = [], []
                for k, p in enumerate(per):
                    if c < len(p):
                        o = self.offsets[k]
                        sa.append(np.asarray(self.bodies[k].point_sets[p[c][0]]) + o)
                        sb.append(np.asarray(self.bodies[k].point_sets[p[c][1]]) + o)
                tag = "filter" if mode else "damage"
                body.point_sets[f"{tag}{c}:a"] = np.concatenate(sa)
                body.point_sets[f"{tag}{c}:b"] = np.concatenate(sb)
                body.point_sets_precracks.append((f"{tag}{c}:a", f"{tag}{c}:b", mode))
        return body

    def run(self, n_steps, first_step=1):
        """Velocity Verlet steps of every specimen with its own time step (the reference's
        initialize! force evaluation happens before the first block)."""
        if first_step == 1:
            self.dev.force(0.0, float(self.dt.min()))
        self.dev.run(first_step, n_steps, -1.0)

    def run_timed(self, first_step, n_steps):
        """run() with CUDA events: (total, force phase A, phase B, integration) ms."""
        return self.dev.run_timed(first_step, n_steps, -1.0)

    def field(self, name, k):
        """Storage field of specimen k: 3 x n_k (9 x n_k) point vectors (tensors), n_k point
        scalars, or the bond_active bytes of its bonds."""
        f = self.dev.field(name)
        o, m = self.offsets[k], self.bodies[k].n_points
        if name == "bond_active":
            nn = np.concatenate([[0], np.cumsum(self.dev.field("n_neighbors"))])
            return f[nn[o]:nn[o + m]]
        return f[..., o:o + m]

    def close(self):
        self.dev.close()
