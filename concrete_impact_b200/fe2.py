"""Explicit FE^2 impact dynamics on the GPU: macro Hex8 bar, velocity Verlet, RVE or RNO points.

Restates the reference's explicit material dynamics (solve_material_explicit,
src/fem/dynamics/material.py:89-297: lumped row-sum mass, velocity Verlet, homogeneous
Dirichlet DOFs, material update without tangent each step), its CFL bound
(src/fem/dynamics/stability.py:34-48), the half-sine pressure pulse
(src/concrete_impact/benchmarks/dynamic_viscoplastic.py:147-170) and the uniform boundary
pressure (src/fem/assembly/load.py:40-77), with the macro kernels of ``csrc/hex8.cu`` and
``csrc/fe2.cu``.  The macro material at the integration points is either

* ``DirectRVEPoints`` -- one periodic RVE per macro point, all solved in device batches
  (the reference's RVEHomogenizedMaterial), or
* ``RNOPoints`` -- the recurrent surrogate with one latent state per point, behind an error
  gate: a point whose surrogate input leaves the training envelope falls back to a direct
  RVE solve (fallback pool of RVEs; its RVE starts with a catch-up step that loads it
  proportionally to the current macro strain over the elapsed time), and optionally a
  runtime judge (``SurrogateJudge``): direct FP64 RVEs at a seeded sample of points follow
  the run's macro strains, measure the error of the delivered stress against the direct
  solve, and escalate a sampled point whose error passes a threshold to the fallback pool
  with its direct RVE history.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native
from .assembly import MaterialAssemblyCache, build_hex8_material_assembly_cache
from .materials import MaterialPointRequest, MaterialState, MaterialUpdateSettings
from .rno import RNOSurrogate
from .rve import RS_SIGMA, RVEBatch, StructuredHex8RVE, build_structured_hex8_box, solve_batch_step


@dataclass
class MacroBar:
    """Structured macro Hex8 bar with the left face fixed and a pressure on the right face."""

    nodes: np.ndarray
    elements: np.ndarray
    divisions: tuple[int, int, int]
    lengths: tuple[float, float, float]
    density: float
    fixed: torch.Tensor  # (3N,) uint8
    unit_force: torch.Tensor  # (3N,) nodal force of a unit pressure
    mass: torch.Tensor  # (3N,) lumped row-sum mass
    cache: MaterialAssemblyCache = field(repr=False)

    @property
    def points(self) -> int:
        return 8 * int(self.elements.shape[0])

    @property
    def min_edge(self) -> float:
        return float(min(l / n for l, n in zip(self.lengths, self.divisions)))


def build_macro_bar(divisions=(64, 16, 16), lengths=(0.64, 0.16, 0.16), density: float = 2400.0) -> MacroBar:
    """Bar with x the long axis: x = 0 face fixed, unit pressure on the x = L face."""
    dev = _native.require_cuda()
    nodes, elements = build_structured_hex8_box(tuple(lengths), tuple(divisions))
    n = nodes.shape[0]
    left = np.isclose(nodes[:, 0], 0.0)
    right = np.isclose(nodes[:, 0], lengths[0])
    fixed = np.zeros(3 * n, dtype=np.uint8)
    fixed[(3 * np.flatnonzero(left)[:, None] + np.arange(3)).ravel()] = 1
    # uniform traction -p * outward normal (+x) split equally over the 4 nodes of each face quad
    ny, nz = divisions[1], divisions[2]
    face_area = (lengths[1] / ny) * (lengths[2] / nz)
    count = np.zeros(n)
    jr = np.rint(nodes[:, 1] / (lengths[1] / ny)).astype(int)
    kr = np.rint(nodes[:, 2] / (lengths[2] / nz)).astype(int)
    inner_y = np.where((jr == 0) | (jr == ny), 1, 2)
    inner_z = np.where((kr == 0) | (kr == nz), 1, 2)
    count[right] = (inner_y * inner_z)[right]
    unit = np.zeros(3 * n)
    unit[3 * np.flatnonzero(right)] = -face_area / 4.0 * count[right]
    vol = float(np.prod([l / d for l, d in zip(lengths, divisions)]))
    mass_node = np.zeros(n)
    np.add.at(mass_node, elements.reshape(-1), density * vol / 8.0)
    cache = build_hex8_material_assembly_cache(nodes, elements)
    t = lambda a, dt=torch.float64: torch.as_tensor(a, dtype=dt, device=dev)  # noqa: E731
    return MacroBar(nodes, elements, tuple(divisions), tuple(lengths), density, t(fixed, torch.uint8), t(unit),
                    t(np.repeat(mass_node, 3)), cache)  # fmt: skip


def half_sine_pressure(time: float, amplitude: float = 50.0e6, duration: float = 50.0e-6) -> float:
    """Half-sine pulse amplitude * sin(pi t / duration) for 0 <= t <= duration, else 0."""
    return amplitude * math.sin(math.pi * time / duration) if 0.0 <= time <= duration else 0.0


def stable_time_step(bar: MacroBar, wave_speed: float, safety: float = 0.5) -> float:
    """CFL bound safety * h_min / c_p."""
    return safety * bar.min_edge / wave_speed


# --------------------------------------------------------------------------------------
# Macro materials.


class MaterialPoints:
    """A material model of the point protocol (J2, linear elastic, phased) at every macro
    point, with its state on the device; the reference's solve_material_explicit with a
    plain constitutive law."""

    def __init__(self, material, n_points: int, update_settings: MaterialUpdateSettings) -> None:
        dev = _native.require_cuda()
        self.material = material
        self.settings = update_settings
        init = material.initialize_state(n_points)
        self.state = MaterialState({k: torch.as_tensor(v, device=dev) for k, v in init.variables.items()})
        self.trial = self.state

    def stress(self, strain: torch.Tensor, rate: torch.Tensor, dt: float) -> torch.Tensor:
        req = MaterialPointRequest(strain, rate, dt, "three_dimensional", self.settings)
        resp = self.material.update(req, self.state)
        self.trial = resp.state
        return resp.stresses

    def commit(self) -> None:
        self.state = self.trial


class DirectRVEPoints:
    """One RVE per macro point, solved in device batches of at most ``chunk`` RVEs."""

    def __init__(self, model: StructuredHex8RVE, n_points: int, update_settings: MaterialUpdateSettings,
                 precision: int = 32, chunk: int = 16384) -> None:  # fmt: skip
        self.model = model
        self.n = n_points
        self.settings = update_settings
        self.batches = [RVEBatch([model] * min(chunk, n_points - s), precision=precision, device_control=True)
                        for s in range(0, n_points, chunk)]  # fmt: skip
        self.starts = list(range(0, n_points, chunk))
        self.volume = float(self.batches[0].volumes[0])
        self.newton_iterations = 0

    def stress(self, strain: torch.Tensor, rate: torch.Tensor, dt: float) -> torch.Tensor:
        out = torch.empty((self.n, 6), dtype=torch.float64, device=strain.device)
        for s, b in zip(self.starts, self.batches):
            sl = slice(s, s + b.nrve)
            b.macro.copy_(strain[sl])
            b.dt.fill_(dt)
            res = solve_batch_step(b, self.model.newton_settings, self.settings, False)
            self.newton_iterations = max(self.newton_iterations, int(res.newton_iterations.max()))
            b.response(b.batch_struct(self.settings), b.w, None, None)
            out[sl] = b.sums[:, RS_SIGMA : RS_SIGMA + 6] / self.volume
        return out

    def commit(self) -> None:
        for b in self.batches:
            b.commit()


def _pool_solver(model: StructuredHex8RVE):
    """PCG controls of the small same-size RVE batches of the fallback pool and the judge:
    a few hundred RVEs at most, so each system gets a cluster of CTAs (8 for an 8^3 RVE:
    about 2.8x faster per solve than one CTA) instead of the size rule's one CTA."""
    from .rve import LinearSolverOptions

    nz = int(model.divisions[2])
    return LinearSolverOptions(cluster=8 if nz >= 8 else (4 if nz >= 4 else 1))


class SurrogateJudge:
    """Direct RVE solves that judge the surrogate's error during an FE^2 run.

    A seeded sample of ``sample`` macro points carries its own direct RVEs (``precision``
    64: the reference's precision), advanced along the surrogate run's macro strains every
    ``every`` macro steps (one RVE step over the elapsed interval).  At each judge step the
    stress delivered at those points (surrogate, or fallback where a point was flagged) is
    compared with the direct homogenised stress; the judge keeps the squared errors and
    squared reference stresses per point, so ``error`` is the relative Frobenius error of
    the homogenised stress over the sampled points and judge steps.  A sampled point whose
    own error exceeds ``threshold`` relative to its reference stress, or to
    ``stress_floor`` where that is larger (so that the arrival of a wave front, when the
    stress is still near zero, is not judged relative to nothing), is escalated: it leaves
    the surrogate for the fallback pool, which takes over the judge's RVE state of that
    point (its exact history).  ``threshold`` None only measures.  One host read per judge
    step decides the escalations.
    """

    def __init__(self, model: StructuredHex8RVE, n_points: int, update_settings: MaterialUpdateSettings,
                 sample: int = 256, every: int = 1, threshold: float | None = 0.05, stress_floor: float = 1.0e6,
                 seed: int = 0, precision: int = 64) -> None:  # fmt: skip
        rng = np.random.default_rng(seed)
        pts = np.sort(rng.choice(n_points, size=min(sample, n_points), replace=False))
        self.model = model
        self.settings = update_settings
        self.every = max(int(every), 1)
        self.threshold = None if threshold is None else float(threshold)
        self.floor2 = float(stress_floor) ** 2
        self.batch = RVEBatch([model] * pts.size, precision=precision, device_control=True,
                              linear_solver=_pool_solver(model))  # fmt: skip
        dev = self.batch.device
        self.points = torch.as_tensor(pts, device=dev)
        self.volume = float(self.batch.volumes[0])
        self.sq_err = torch.zeros(pts.size, dtype=torch.float64, device=dev)
        self.sq_ref = torch.zeros(pts.size, dtype=torch.float64, device=dev)
        self.sq_den = torch.zeros(pts.size, dtype=torch.float64, device=dev)  # sum of max(|ref|^2, floor^2)
        self.escalated = torch.zeros(pts.size, dtype=torch.bool, device=dev)
        self.count = 0
        self.elapsed = 0.0
        self.judge_steps = 0
        self.history: list[tuple[int, float, float]] = []  # (macro step, running error, worst point error)

    @property
    def error(self) -> float:
        ref = float(self.sq_ref.sum())
        return math.sqrt(float(self.sq_err.sum()) / ref) if ref > 0.0 else 0.0

    def observe(self, strain: torch.Tensor, delivered: torch.Tensor, dt: float) -> torch.Tensor | None:
        """After a macro step's material update: every ``every`` steps solve the sampled
        RVEs and compare.  Returns the sample slots to escalate (or None)."""
        self.count += 1
        self.elapsed += dt
        if self.count % self.every:
            return None
        b = self.batch
        b.macro.copy_(strain[self.points])
        b.dt.fill_(self.elapsed)
        self.elapsed = 0.0
        solve_batch_step(b, self.model.newton_settings, self.settings, False)
        b.response(b.batch_struct(self.settings), b.w, None, None)
        ref = b.sums[:, RS_SIGMA : RS_SIGMA + 6] / self.volume
        b.commit()
        self.reference = ref
        diff = delivered[self.points] - ref
        ref2 = (ref * ref).sum(dim=1)
        self.sq_err += (diff * diff).sum(dim=1)
        self.sq_ref += ref2
        self.sq_den += ref2.clamp(min=self.floor2)
        self.judge_steps += 1
        point_err2 = self.sq_err / self.sq_den
        worst = float(point_err2.max().sqrt())
        self.history.append((self.count, self.error, worst))
        if self.threshold is None:
            return None
        bad = (point_err2 > self.threshold**2) & ~self.escalated
        slots = torch.nonzero(bad).flatten()
        if slots.numel() == 0:
            return None
        self.escalated[slots] = True
        return slots


class RNOPoints:
    """The surrogate at every macro point, with an input-envelope gate and a direct fallback.

    ``envelope`` = (max |normalised strain|, max |normalised rate|) seen in training, each a
    scalar or a 6-vector of per-component maxima; a point any of whose input components
    exceeds ``envelope_factor`` times its limit is flagged and solved by a fallback RVE from
    then on (at most ``fallback_capacity`` points).  A point whose surrogate answer is not
    finite is flagged the same way.
    """

    def __init__(self, rno: RNOSurrogate, n_points: int, envelope: tuple[float, float],
                 model: StructuredHex8RVE | None = None, update_settings: MaterialUpdateSettings | None = None,
                 envelope_factor: float = 1.05, fallback_capacity: int = 2048, precision: int = 32,
                 judge: SurrogateJudge | None = None) -> None:  # fmt: skip
        self.rno = rno
        self.judge = judge
        self.escalations = 0
        self.n = n_points
        dev = rno.device
        self.z = torch.zeros((n_points, 6), dtype=torch.float32, device=dev)
        self.z_next = self.z
        self.envelope = envelope
        self.factor = envelope_factor
        self._lim = None
        self.model = model
        self.settings = update_settings
        self.buffers = None
        self.flagged = torch.zeros(n_points, dtype=torch.bool, device=dev)
        self.slot_of = torch.full((n_points,), -1, dtype=torch.int64, device=dev)
        self.slots_used = 0
        self.pool = (RVEBatch([model] * fallback_capacity, precision=precision, device_control=True,
                              linear_solver=_pool_solver(model))
                     if model is not None else None)  # fmt: skip
        self.capacity = fallback_capacity if model is not None else 0
        self.pool_points = torch.full((self.capacity,), -1, dtype=torch.int64, device=dev)
        self.time = 0.0
        self.fallback_steps = 0
        self._catch_up: tuple[int, int] | None = None  # slots whose next solve covers the elapsed time
        self.lib = _native.load_library()
        if rno.fused:  # device buffers of the fused gate (two launches around the surrogate per step)
            f32 = torch.float32
            self.zbuf = torch.zeros((2, n_points, 6), dtype=f32, device=dev)  # current / next latent
            self.xn = torch.empty((n_points, 6), dtype=f32, device=dev)
            self.rn = torch.empty((n_points, 6), dtype=f32, device=dev)
            self.cf = torch.empty(n_points, dtype=f32, device=dev)
            self.sn = torch.empty((n_points, 6), dtype=f32, device=dev)
            self.out = torch.empty((n_points, 6), dtype=torch.float64, device=dev)
            self.fresh = torch.zeros(n_points, dtype=torch.uint8, device=dev)
            self.flag8 = torch.zeros(n_points, dtype=torch.uint8, device=dev)
            self.count = torch.zeros(1, dtype=torch.int32, device=dev)

    def stress(self, strain: torch.Tensor, rate: torch.Tensor, dt: float) -> torch.Tensor:
        stress = self._stress(strain, rate, dt)
        if self.judge is not None:
            slots = self.judge.observe(strain, stress, dt)
            if slots is not None:
                stress = stress.clone()
                self._escalate(slots, stress)
        return stress

    def _escalate(self, slots: torch.Tensor, stress: torch.Tensor) -> None:
        """Move judged points whose error passed the threshold to the fallback pool with
        the judge's RVE state; their stress of this step is the judge's."""
        judge = self.judge
        pts = judge.points[slots]
        keep = ~self.flagged[pts]
        slots, pts = slots[keep], pts[keep]
        if pts.numel() == 0:
            return
        room = self.capacity - self.slots_used
        if pts.numel() > room:
            raise RuntimeError(f"the judge escalated more points than the fallback pool holds ({self.capacity}).")
        a, b = self.slots_used, self.slots_used + int(pts.numel())
        p, j = self.pool, judge.batch
        E = int(p.elem_counts[0])
        for k, (slot, pt) in enumerate(zip(range(a, b), slots.tolist())):
            g0, g1, h0, h1 = 8 * E * slot, 8 * E * (slot + 1), 8 * E * pt, 8 * E * (pt + 1)
            # committed and trial state alike: the step's commit copies trial -> committed
            for dst, src in ((p.ep_n, j.ep_n), (p.ep, j.ep_n)):
                dst[:, g0:g1] = src[:, h0:h1].to(dst.dtype)
            for dst in (p.q_n, p.q):
                dst[g0:g1] = j.q_n[h0:h1]
            for dst in (p.vpm_n, p.vpm):
                dst[g0:g1] = j.vpm_n[h0:h1]
            for dst in (p.w_n, p.w):
                dst[3 * E * slot : 3 * E * (slot + 1)] = j.w_n[3 * E * pt : 3 * E * (pt + 1)]
            p.macro_n[slot] = j.macro_n[pt]
            p.macro[slot] = j.macro_n[pt]
        self.pool_points[a:b] = pts
        self.flagged[pts] = True
        if self.rno.fused:
            self.flag8[pts] = 1
        self.slot_of[pts] = torch.arange(a, b, device=pts.device)
        self.slots_used = b
        stress[pts] = judge.reference[slots]
        self.escalations += int(pts.numel())

    def _stress(self, strain: torch.Tensor, rate: torch.Tensor, dt: float) -> torch.Tensor:
        if self.rno.fused and self.pool is not None:
            return self._stress_fused(strain, rate, dt)
        s = self.rno.scales
        coef = torch.full((self.n,), dt / self.rno.config.tau_ref, dtype=torch.float32, device=strain.device)
        out, z_next, self.buffers = self.rno.predict(strain, rate, self.z, coef, self.buffers)
        self.z_next = z_next
        stress = out.double()
        if self.pool is None:
            return stress
        lim_e, lim_r = self._limits(strain.device)
        over = ((strain.abs() / s.strain) > lim_e).any(dim=1) | ((rate.abs() / s.rate) > lim_r).any(dim=1)
        over |= ~torch.isfinite(stress).all(dim=1) | ~torch.isfinite(strain).all(dim=1)  # never trust a non-finite answer
        new = over & ~self.flagged
        if bool(new.any()):
            self._admit(torch.nonzero(new).flatten(), strain)
        if self.slots_used:
            self._solve_pool(stress, strain, dt)
        return stress

    def _solve_pool(self, stress: torch.Tensor, strain: torch.Tensor, dt: float) -> None:
        """Direct RVE solves of the flagged points; their rows of ``stress`` are replaced."""
        used = slice(0, self.slots_used)
        pts = self.pool_points[used]
        self.pool.macro[used] = strain[pts]
        self.pool.dt[used] = dt
        if self._catch_up is not None:
            a, b = self._catch_up
            self.pool.dt[a:b] = max(self.time + dt, dt)
            self._catch_up = None
        mask = np.zeros(self.capacity, dtype=bool)
        mask[: self.slots_used] = True
        solve_batch_step(self.pool, self.model.newton_settings, self.settings, False, live_mask=mask)
        self.pool.response(self.pool.batch_struct(self.settings), self.pool.w, None, None)
        vol = float(self.pool.volumes[0])
        stress[pts] = self.pool.sums[used, RS_SIGMA : RS_SIGMA + 6] / vol
        self.fallback_steps += 1

    def _stress_fused(self, strain: torch.Tensor, rate: torch.Tensor, dt: float) -> torch.Tensor:
        """The gate in two kernels around the fused surrogate step: normalise and test the
        inputs, run the surrogate, scale and test its answers; one read of the count of
        newly flagged points decides whether the fallback pool is needed."""
        s = self.rno.scales
        lim_e, lim_r = self._limits(strain.device)
        if not hasattr(self, "_lim12"):
            self._lim12 = torch.cat([lim_e.expand(6), lim_r.expand(6)]).contiguous()
        strain, rate = strain.contiguous(), rate.contiguous()
        sp = _native.stream_ptr()
        self.count.zero_()
        _native.check(self.lib.cib_rno_gate_prepare(
            self.n, strain.data_ptr(), rate.data_ptr(), s.strain, s.rate, self._lim12.data_ptr(),
            dt / self.rno.config.tau_ref, self.flag8.data_ptr(), self.xn.data_ptr(), self.rn.data_ptr(),
            self.cf.data_ptr(), self.fresh.data_ptr(), self.count.data_ptr(), sp), "cib_rno_gate_prepare")  # fmt: skip
        self.rno.predict_normalized(self.xn, self.rn, self.cf, self.zbuf, self.sn)
        _native.check(self.lib.cib_rno_gate_finish(
            self.n, self.sn.data_ptr(), s.stress, self.flag8.data_ptr(), self.fresh.data_ptr(), self.count.data_ptr(),
            self.out.data_ptr(), sp), "cib_rno_gate_finish")  # fmt: skip
        stress = self.out
        if int(self.count.item()) > 0:
            new = torch.nonzero(self.fresh).flatten()
            self.flag8[new] = 1
            self._admit(new, strain)
        if self.slots_used:
            stress = stress.clone()
            self._solve_pool(stress, strain, dt)
        return stress

    def _limits(self, device) -> tuple[torch.Tensor, torch.Tensor]:
        """Gate limits per component (scalars broadcast to all six)."""
        if self._lim is None:
            e = torch.as_tensor(self.envelope[0], dtype=torch.float64, device=device).reshape(-1)
            r = torch.as_tensor(self.envelope[1], dtype=torch.float64, device=device).reshape(-1)
            self._lim = (self.factor * e, self.factor * r)
        return self._lim

    def _admit(self, points: torch.Tensor, strain: torch.Tensor) -> None:
        """Give newly flagged points a fallback RVE from the zero state; the first solve of
        the slot is a catch-up step over the elapsed time."""
        room = self.capacity - self.slots_used
        if points.numel() > room:
            raise RuntimeError(f"RNO error gate flagged more points than the fallback pool holds ({self.capacity}).")
        a, b = self.slots_used, self.slots_used + int(points.numel())
        self.pool_points[a:b] = points
        self.flagged[points] = True
        self.slot_of[points] = torch.arange(a, b, device=points.device)
        p = self.pool
        E = int(p.elem_counts[0])
        g0, g1 = 8 * E * a, 8 * E * b
        p.ep_n[:, g0:g1] = 0
        p.q_n[g0:g1] = 0
        p.vpm_n[g0:g1] = 0
        p.w_n[3 * E * a : 3 * E * b] = 0
        p.macro_n[a:b] = 0
        self.slots_used = b
        self._catch_up = (a, b) if self._catch_up is None else (self._catch_up[0], b)

    def commit(self) -> None:
        if self.rno.fused and self.pool is not None:
            self.zbuf[0].copy_(self.zbuf[1])
        else:
            self.z = self.z_next.clone()
        if self.slots_used:
            self.pool.commit()

    def advance_time(self, dt: float) -> None:
        self.time += dt


class ExplicitFE2:
    """Velocity-Verlet macro dynamics with a macro-point material (direct RVEs or RNO)."""

    def __init__(self, bar: MacroBar, material, dt: float, pressure=half_sine_pressure) -> None:
        self.bar = bar
        self.material = material
        self.dt = float(dt)
        self.pressure = pressure
        self.lib = _native.load_library()
        dev = bar.fixed.device
        n3 = bar.fixed.numel()
        z = lambda: torch.zeros(n3, dtype=torch.float64, device=dev)  # noqa: E731
        self.u, self.v, self.a = z(), z(), z()
        self.u_next, self.v_next, self.a_next = z(), z(), z()
        npts = bar.points
        self.strain = torch.zeros((npts, 6), dtype=torch.float64, device=dev)
        self.rate = torch.zeros((npts, 6), dtype=torch.float64, device=dev)
        self.fe = torch.empty(npts * 3, dtype=torch.float64, device=dev)
        self.f_int = z()
        self.time = 0.0
        self.step_count = 0
        self.last_stress: torch.Tensor | None = None

    def _strains(self, u: torch.Tensor, u_prev: torch.Tensor) -> None:
        c = self.bar.cache
        code = self.lib.cib_hex8_strains(int(c.elements.shape[0]), c.elements.data_ptr(), c.grads.data_ptr(),
                                         u.data_ptr(), u_prev.data_ptr(), self.dt, self.strain.data_ptr(),
                                         self.rate.data_ptr(), _native.stream_ptr())  # fmt: skip
        _native.check(code, "cib_hex8_strains")

    def _internal_force(self, stress: torch.Tensor) -> None:
        c = self.bar.cache
        code = self.lib.cib_hex8_internal_force(int(c.elements.shape[0]), c.node_count, c.grads.data_ptr(),
                                                c.jw.data_ptr(), stress.data_ptr(), c.node_ptr.data_ptr(),
                                                c.node_list.data_ptr(), self.fe.data_ptr(), self.f_int.data_ptr(),
                                                _native.stream_ptr())  # fmt: skip
        _native.check(code, "cib_hex8_internal_force")

    def step(self) -> None:
        """One velocity-Verlet step (material.py:195-219)."""
        sp = _native.stream_ptr()
        n = self.u.numel()
        _native.check(self.lib.cib_verlet_predict(n, self.u.data_ptr(), self.v.data_ptr(), self.a.data_ptr(),
                                                  self.bar.fixed.data_ptr(), self.dt, self.u_next.data_ptr(), sp),
                      "cib_verlet_predict")  # fmt: skip
        self._strains(self.u_next, self.u)
        stress = self.material.stress(self.strain, self.rate, self.dt).contiguous()
        self._internal_force(stress)
        t1 = self.time + self.dt
        _native.check(self.lib.cib_verlet_correct(n, self.bar.unit_force.data_ptr(), float(self.pressure(t1)),
                                                  self.f_int.data_ptr(), self.bar.mass.data_ptr(),
                                                  self.bar.fixed.data_ptr(), self.dt, self.a.data_ptr(),
                                                  self.v.data_ptr(), self.a_next.data_ptr(), self.v_next.data_ptr(), sp),
                      "cib_verlet_correct")  # fmt: skip
        self.material.commit()
        if hasattr(self.material, "advance_time"):
            self.material.advance_time(self.dt)
        self.u, self.u_next = self.u_next, self.u
        self.v, self.v_next = self.v_next, self.v
        self.a, self.a_next = self.a_next, self.a
        self.time = t1
        self.step_count += 1
        self.last_stress = stress

    def run(self, steps: int) -> None:
        for _ in range(steps):
            self.step()
