"""Ensembles of independent ice-sheet members of uneven grid sizes.

Each member is an `IceDynamics` on its own hierarchy (own device arena, own
captured V-cycle graphs).  `Ensemble` drives them concurrently: members are
dealt to a fixed pool of host workers, each worker owns a CUDA stream and
always serves the same members (handles are single-threaded), and the C-ABI
calls release the interpreter lock, so the GPU runs kernels of many members
at once.  A member's convergence checks synchronise only its own stream.

`Ensemble.autotune` picks, per size class, the fastest of a few solver
schedules and FASCD launch shapes (resident Vanka-sweep blocks per SM) by
timing a step of the class's first member from a warm state: the member is
first advanced one step, trials run from that state, and the member's
original state is restored afterwards.

With `grouped=True` the members' cycles run in grouped launches
(glide_b200.group): one forward solve and one adjoint solve cover the group
members -- each kind of launch of a cycle issued once for all of them, the
cycle one CUDA graph, each member's convergence test and Newton decisions on
the device -- while members above `group_max_cells` solve on the worker
streams meanwhile.  Members run the same cycles either way.

No counterpart in the reference (its models run one grid at a time); the
members themselves are the reference-compatible `IceDynamics`.
"""
from __future__ import annotations

import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass

import numpy as np
import torch

from .group import HierarchyGroup
from .model import IceDynamics

STATE = ("u", "v", "H", "H_prev", "phi", "mask")


class _Streams:
    """CUDA streams of the ensemble's own, one per host worker and grouped
    job.  torch.cuda.Stream() hands out streams round-robin from a fixed pool
    (32 per priority), so many workers would share some -- and a stream that
    one thread drives while another captures a graph on it breaks the
    capture.  Created non-blocking, destroyed by close()."""

    def __init__(self):
        self._raw = []

    def new(self) -> torch.cuda.Stream:
        from cuda.bindings import runtime as rt
        err, s = rt.cudaStreamCreateWithFlags(rt.cudaStreamNonBlocking)
        if err != rt.cudaError_t.cudaSuccess:
            raise RuntimeError(f"cudaStreamCreateWithFlags: {err}")
        self._raw.append(s)
        return torch.cuda.ExternalStream(int(s))

    def close(self):
        from cuda.bindings import runtime as rt
        if self._raw:
            torch.cuda.synchronize()
        for s in self._raw:
            rt.cudaStreamDestroy(s)
        self._raw = []


def levels_for(n: int, min_coarse: int = 16, max_levels: int = 8) -> int:
    """Most levels such that n halves exactly down to a coarsest grid of at
    least `min_coarse` cells."""
    levels = 1
    while levels < max_levels and n % (2 ** levels) == 0 and n // (2 ** levels) >= min_coarse:
        levels += 1
    return levels


@dataclass
class MemberSpec:
    n: int
    dx: float
    levels: int
    radius: float
    seed: int
    lapse: float


def member_specs(n_members: int, seed: int = 0, sizes=(128, 192, 256, 384, 512, 768), dx: float = 1500.0,
                 radius=(200e3, 600e3), lapse=(1e-3, 3e-3), min_coarse: int = 16) -> list[MemberSpec]:
    """Seeded uneven ensemble: sizes drawn from `sizes`, dome radius and smb
    lapse rate drawn uniformly, levels down to a coarsest grid >= min_coarse."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_members):
        n = int(rng.choice(sizes))
        R = float(rng.uniform(*radius))
        # the dome must fit the domain
        R = min(R, 0.45 * n * dx)
        out.append(MemberSpec(n=n, dx=dx, levels=levels_for(n, min_coarse), radius=R,
                              seed=int(rng.integers(1 << 30)), lapse=float(rng.uniform(*lapse))))
    return out


# solver schedules the autotuner chooses among (applied through the options
# API); blocks: resident Vanka-sweep blocks per SM of the FASCD smoother
CANDIDATES = {
    "fast": dict(quirks=False, schedule=(4, 4, 0, 50), newton_steps=3, method="newton", switch=0,
                 tangent=(4, 4, 0, 10), blocks=2),
    "fascd": dict(quirks=False, schedule=(4, 4, 0, 50), newton_steps=3, method="fascd", switch=None,
                  tangent=None, blocks=2),
    "fascd/1": dict(quirks=False, schedule=(4, 4, 0, 50), newton_steps=3, method="fascd", switch=None,
                    tangent=None, blocks=1),
    "classic": dict(quirks=False, schedule=(10, 20, 50, 200), newton_steps=30, method="fascd", switch=None,
                    tangent=None, blocks=2),
    # guarded Newton whose fallback cycles are the classic schedule
    "newton/classic": dict(quirks=False, schedule=(10, 20, 50, 200), newton_steps=30, method="newton",
                           switch=0, tangent=(4, 4, 0, 10), blocks=2),
}
FALLBACK = "classic"


def _converged(model: IceDynamics, st: dict) -> bool:
    """The forward solve met its relative or absolute tolerance."""
    c = model.forward_solver._fas_config
    return st["final_norm"] <= max(c.relative_tolerance * st["initial_norm"], c.absolute_tolerance)


def apply_schedule(model: IceDynamics, cfg: dict):
    h = model.mg.hierarchy
    h.set_reference_quirks(cfg["quirks"])
    pre, post, fin, coarse = cfg["schedule"]
    h.set_fas(False, pre_steps=pre, post_steps=post, finest_steps=fin, coarsest_steps=coarse)
    h.set_vanka(False, -1, newton_steps=cfg["newton_steps"])
    h.set_tuning(forward_method=cfg["method"], newton_switch_exp10=cfg["switch"],
                 sweep_blocks_per_sm=cfg.get("blocks", 2))
    if cfg["tangent"]:
        pre, post, fin, coarse = cfg["tangent"]
        h.set_fas(2, pre_steps=pre, post_steps=post, finest_steps=fin, coarsest_steps=coarse)


class Ensemble:
    """Concurrent driver of independent members (see the module text)."""

    def __init__(self, members: list[IceDynamics], workers: int | None = None, grouped: bool = False,
                 group_max_cells: int | None = None, group_by: str = "class", group_size: int | None = None,
                 group_waves: int | None = None):
        self.members = list(members)
        n = len(self.members)
        self.workers = max(1, min(workers or min(n, 16), n))
        # members dealt round-robin, largest first, so workers get even loads
        order = sorted(range(n), key=lambda k: -self.members[k].mg.hierarchy.shapes[0][0] ** 2)
        self._groups = [[] for _ in range(self.workers)]
        for r, k in enumerate(order):
            self._groups[r % self.workers].append(k)
        self._pool = ThreadPoolExecutor(max_workers=self.workers)
        self._own = _Streams()
        self._streams = [None] * self.workers
        self.schedules: dict[int, str] = {}
        self.retries = 0  # forward solves repeated under another schedule
        # autotune trials per size class: name -> {"ms": warm step, "vcycles", "converged",
        # "history": the residual norms relative to the first}
        self.trials: dict[int, dict[str, dict]] = {}
        self.grouped = grouped
        # grouped mode: members of at most this many cells join the groups (None: every member);
        # group_by "class": one group per grid size, each on its own stream; "all": one group
        self.group_max_cells = group_max_cells
        if group_by not in ("class", "all"):
            raise ValueError("group_by must be 'class' or 'all'")
        self.group_by = group_by
        self.group_size = group_size  # at most this many members per group (None: no limit)
        self.group_waves = group_waves  # launch shape of the grouped launches (None: the default)
        self._groups_of: dict[tuple[str, tuple[int, ...]], HierarchyGroup] = {}
        self._fwd_keys: tuple[int, ...] = ()
        self._adj_keys: tuple[int, ...] = ()
        self._side = ThreadPoolExecutor(max_workers=max(self.workers, 8)) if grouped else None
        self._side_streams: list = []
        self._parts_now: list[tuple[int, ...]] = []

    def close(self):
        self._pool.shutdown(wait=True)
        if self._side is not None:
            self._side.shutdown(wait=True)
        for g in self._groups_of.values():
            g.close()
        self._groups_of = {}
        self._own.close()

    def groups(self, kind: str) -> list[tuple[tuple[int, ...], HierarchyGroup]]:
        """The current groups of the forward ("fwd") or adjoint ("adj") solves
        and their members."""
        return [(keys, g) for (kd, keys), g in self._groups_of.items() if kd == kind]

    def _parts(self, keys: tuple[int, ...]) -> list[tuple[int, ...]]:
        if self.group_by == "all":
            parts = [list(keys)] if keys else []
        else:
            by: dict[int, list[int]] = {}
            for k in keys:
                by.setdefault(self.members[k].mg.hierarchy.shapes[0][0], []).append(k)
            parts = [v for _, v in sorted(by.items())]
        q = self.group_size or max(len(keys), 1)
        return [tuple(p[i:i + q]) for p in parts for i in range(0, len(p), q)]

    def _group(self, kind: str, keys: tuple[int, ...]) -> HierarchyGroup:
        """The group of these members for `kind`; groups of that kind over
        other member sets are closed."""
        for key in [q for q in self._groups_of if q[0] == kind and q[1] not in self._parts_now]:
            self._groups_of.pop(key).close()
        g = self._groups_of.get((kind, keys))
        if g is None:
            g = self._groups_of[(kind, keys)] = HierarchyGroup([self.members[k].mg.hierarchy for k in keys])
            g.set_tuning(waves=self.group_waves)
        return g

    def _grouped_jobs(self, kind: str, keys: tuple[int, ...], call):
        """One side job per group of `keys`: call(group) on its own stream."""
        self._parts_now = self._parts(keys)
        return [(part, (lambda g=self._group(kind, part): call(g))) for part in self._parts_now]

    def _run(self, fn, keys=None, sides=()):
        """fn(k, model) for the members `keys` (every member by default), each
        worker on its own stream; every callable in `sides` runs meanwhile on
        a stream of its own.  Returns the results in member order and the
        sides' results."""
        res = [None] * len(self.members)
        keys = set(range(len(self.members))) if keys is None else set(keys)
        caller = torch.cuda.current_stream()
        start = torch.cuda.Event()
        start.record(caller)

        def work(w):
            if self._streams[w] is None:
                self._streams[w] = self._own.new()
            s = self._streams[w]
            s.wait_event(start)
            with torch.cuda.stream(s):
                for k in self._groups[w]:
                    if k in keys:
                        res[k] = fn(k, self.members[k])
            done = torch.cuda.Event()
            done.record(s)
            return done

        while len(self._side_streams) < len(sides):
            self._side_streams.append(self._own.new())

        def side_job(q):
            s = self._side_streams[q]
            s.wait_event(start)
            with torch.cuda.stream(s):
                out = sides[q]()
            done = torch.cuda.Event()
            done.record(s)
            return out, done

        futs = [self._side.submit(side_job, q) for q in range(len(sides))]
        events = list(self._pool.map(work, range(self.workers)))
        side_out = []
        for f in futs:
            out, e = f.result()
            side_out.append(out)
            events.append(e)
        for e in events:
            caller.wait_event(e)
        return res, side_out

    def _in_groups(self, k: int) -> bool:
        """Member k joins the grouped solves: binary64 or binary32, solved
        from its top level, within the size limit."""
        m = self.members[k]
        ny, nx, _ = m.mg.hierarchy.shapes[0]
        return (m.mg.hierarchy.precision != "mixed" and m.top_level == 0
                and (self.group_max_cells is None or ny * nx <= self.group_max_cells))

    def _groupable(self, k: int) -> bool:
        """Member k's forward solve runs in the grouped solve: a group member
        with a schedule (FASCD or guarded Newton)."""
        return self._in_groups(k) and self.schedules.get(k) in CANDIDATES

    def forward(self, t: float, dt: float, update_geometry: bool = True, retry: bool = True):
        """One forward step of every member.  With `retry`, a member whose
        solve stops short of its tolerance (cycle cap reached) is solved again
        from its current iterate under the other candidate schedules in turn,
        each aiming at the first solve's target (relative tolerance times its
        initial residual, or the absolute tolerance); the first that gets
        there becomes that member's schedule.  The returned statistics span
        all attempts.  The geometry update and post-forward hooks run once,
        after the last solve."""
        def one(k, m, st=None):
            if st is None:
                st = m.forward_solver.solve(dt, start_level=m.top_level, report_norms=False)
            else:  # the grouped solve's result, recorded as the member's own solve records it
                m.forward_solver.dt, m.forward_solver.last_stats = float(dt), st
            if retry and not _converged(m, st):
                c = m.forward_solver._fas_config
                rtol, atol = c.relative_tolerance, c.absolute_tolerance
                target = max(rtol * st["initial_norm"], atol)
                first, cycles = st, st["vcycles"]
                m.forward_solver.fas_options.set(relative_tolerance=0.0, absolute_tolerance=target)
                tried = {self.schedules.get(k)}
                try:
                    for name in list(CANDIDATES) + [FALLBACK]:
                        if name in tried:
                            continue
                        tried.add(name)
                        apply_schedule(m, CANDIDATES[name])
                        st = m.forward_solver.solve(dt, start_level=m.top_level, report_norms=False)
                        cycles += st["vcycles"]
                        self.retries += 1
                        if st["final_norm"] <= target:
                            self.schedules[k] = name
                            break
                finally:
                    m.forward_solver.fas_options.set(relative_tolerance=rtol, absolute_tolerance=atol)
                    if self.schedules.get(k) in CANDIDATES:
                        apply_schedule(m, CANDIDATES[self.schedules[k]])
                st = dict(st, initial_norm=first["initial_norm"], vcycles=cycles)
            if update_geometry:
                lev = m.mg.levels[m.top_level]
                lev.state.H_prev.data.copy_(lev.state.H.data)
            for hook in m._post_forward_hooks:
                hook(t + dt)
            return st
        if not self.grouped:
            return self._run(one)[0]
        n = len(self.members)
        gk = tuple(k for k in range(n) if self._groupable(k))
        solo = [k for k in range(n) if k not in gk]
        if not gk:
            return self._run(one)[0]
        jobs = self._grouped_jobs("fwd", gk, lambda g: g.forward(dt))
        self._fwd_keys = gk
        res, outs = self._run(one, keys=solo, sides=[job for _, job in jobs])
        # retries, geometry update and hooks of the grouped members, on the workers
        first = {k: st for (part, _), gst in zip(jobs, outs) for k, st in zip(part, gst)}
        done, _ = self._run(lambda k, m: one(k, m, first[k]), keys=gk)
        for k in gk:
            res[k] = done[k]
        return res

    def backward(self, t: float, dt: float, dJ):
        """dJ(k, model) -> (dJdu, dJdv, dJdH) per member; returns the adjoint
        stats.  Grouped: the group members' adjoint solves in one grouped
        solve, the others on the worker streams meanwhile."""
        def one(k, m):
            du, dv, dH = dJ(k, m)
            return m.backward(t, dt, dJdu=du, dJdv=dv, dJdH=dH)
        gk = tuple(k for k in range(len(self.members)) if self.grouped and self._in_groups(k))
        if not gk:
            return self._run(one)[0]
        masks = set()
        for k in gk:
            m = self.members[k]
            du, dv, dH = dJ(k, m)
            masks.add(m.prepare_backward(dJdu=du, dJdv=dv, dJdH=dH))
        if len(masks) != 1:
            raise ValueError("grouped adjoint solves need one gradient mask for every member")
        mask = masks.pop()
        jobs = self._grouped_jobs("adj", gk, lambda g: g.backward(dt, mask=mask))
        self._adj_keys = gk
        solo = [k for k in range(len(self.members)) if k not in gk]
        res, outs = self._run(one, keys=solo, sides=[job for _, job in jobs])
        for (part, _), gst in zip(jobs, outs):
            for k, s in zip(part, gst):
                self.members[k].adjoint_solver.dt, self.members[k].adjoint_solver.last_stats = float(dt), s
                res[k] = s
        return res

    def autotune(self, dt: float, candidates: dict | None = None, warm: bool = True) -> dict[int, str]:
        """Per size class: time one forward step of the class's first member
        with every candidate schedule, keep the fastest that converges for the
        whole class.  With `warm`, the member is first advanced one step (the
        "fast" schedule, the others in turn if it stops short), so the trials
        time the warm-started steps a run is made of rather than its cold
        first step; every trial starts from that state and the member's
        original state is restored at the end."""
        candidates = candidates or CANDIDATES
        classes: dict[int, list[int]] = {}
        for k, m in enumerate(self.members):
            classes.setdefault(m.mg.hierarchy.shapes[0][0], []).append(k)
        chosen = {}
        for n, ks in sorted(classes.items()):
            m = self.members[ks[0]]
            h = m.mg.hierarchy
            original = {f: h.get(f, 0) for f in STATE}
            saved = original
            if warm:
                for name in list(candidates) + [FALLBACK]:
                    for f, v in original.items():
                        h.set(f, 0, v, restrict_down=True)
                    apply_schedule(m, candidates.get(name, CANDIDATES[FALLBACK]))
                    st = m.forward(0.0, dt, update_geometry=False)
                    if _converged(m, st):
                        break
                saved = {f: h.get(f, 0) for f in STATE}
                saved["H_prev"] = saved["H"].clone()  # the next step starts from the solved geometry
            best, best_t = None, float("inf")
            for name, cfg in candidates.items():
                apply_schedule(m, cfg)
                for trial in range(2):  # the first run captures the V-cycle graphs
                    for f, v in saved.items():
                        h.set(f, 0, v, restrict_down=True)
                    torch.cuda.synchronize()
                    t0 = time.perf_counter()
                    st = m.forward(0.0, dt, update_geometry=False)
                    torch.cuda.synchronize()
                    el = time.perf_counter() - t0
                ok = st["final_norm"] <= max(h.get_fas(False)["relative_tolerance"] * st["initial_norm"],
                                             h.get_fas(False)["absolute_tolerance"])
                h0 = st["history"][0] if st["history"] and st["history"][0] > 0 else 1.0
                self.trials.setdefault(n, {})[name] = {
                    "ms": el * 1e3, "vcycles": int(st["vcycles"]), "converged": bool(ok),
                    "history": [float(f"{x / h0:.2e}") for x in st["history"][:12]]}
                if ok and el < best_t:
                    best, best_t = name, el
            best = best or FALLBACK
            for f, v in original.items():
                h.set(f, 0, v, restrict_down=True)
            for k in ks:
                apply_schedule(self.members[k], candidates[best])
                self.schedules[k] = best
            chosen[n] = best
        return chosen

