"""Differentiable Gaussian heat source on the GPU.

    -Δu = Q exp(-|x - x0|^2 / sigma^2)  in the domain,   u = g on the boundary,

with g given per mesh vertex (interpolated at the nearest boundary point).
:class:`HeatProblem` binds a :class:`~walk_on_spheres_b200.solver.Solver`
(mesh already uploaded), a set of probe points and the walk settings;
``forward`` estimates the probe values (``wos_heat_forward``) and ``adjoint``
replays the same walks from their seeds to return gradients
(``wos_heat_adjoint``).  :func:`heat_probe_values` wraps both in a
``torch.autograd.Function`` so that probe values enter torch graphs with
gradients for Q, x0, sigma and every vertex value:

    heat = HeatProblem(solver, probes, N_walks=2048, epsilon=1e-5, seed=7)
    Q = torch.tensor(1e3, dtype=torch.float64, requires_grad=True)
    u = heat_probe_values(heat, Q, x0, sigma, g)      # (n_probes,)
    loss = (u ** 2).sum(); loss.backward()            # Q.grad, x0.grad, ...

Because a walk's geometry does not depend on (Q, x0, sigma, g), repeated
forward calls with the same HeatProblem use common random numbers: central
differences of ``forward`` and the adjoint's derivatives estimate the same
per-walk quantities.  The reference has no gradients and no 3D Gaussian
source; the estimator is its Poisson walk (include/wos/wos.hpp:54-138).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .solver import METHODS, SOURCE_MODES, Solver, _enum, _ptr

PARAMETERS = ("Q", "x0.x", "x0.y", "x0.z", "sigma")


@dataclass
class HeatValues:
    mean: np.ndarray
    variance: np.ndarray
    standard_error: np.ndarray
    mean_steps: np.ndarray
    location: np.ndarray
    counters: dict = field(default_factory=dict)


@dataclass
class HeatGradients:
    grad_source: np.ndarray         # (5,) sum_p w_p du_p/d(Q, x0.x, x0.y, x0.z, sigma)
    grad_vertex_values: np.ndarray  # (n_verts,) sum_p w_p du_p/dg_v
    jacobian: np.ndarray            # (n, 5) per-probe du_p/dtheta
    jacobian_se: np.ndarray         # (n, 5) standard errors of the above
    replayed_mean: np.ndarray       # (n,) probe values of the replay (== forward mean)
    counters: dict = field(default_factory=dict)


class HeatProblem:
    """Probe points and walk settings of one differentiable heat solve."""

    def __init__(self, solver: Solver, probes, N_walks: int = 2048, epsilon: float = 1e-5,
                 max_steps: int = 100000, max_ray_attempts: int = 12, seed: int = 0,
                 source_mode="green", method="fast", point_index=None,
                 mis_green_probability: float = 0.5, proposal=None):
        """source_mode "uniform", "green" or "mis"; for "mis", each step takes a
        Green sample with probability mis_green_probability, else a sample of the
        proposal N(x0p, sigmap^2/2 I), proposal = (x0p, sigmap) held fixed across calls
        (None: each call's own x0 and sigma)."""
        self.solver = solver
        self.mis_green_probability = float(mis_green_probability)
        self.proposal = proposal
        self.probes = np.ascontiguousarray(probes, dtype=np.float64).reshape(-1, solver.dim)
        self.n = self.probes.shape[0]
        self.point_index = (None if point_index is None
                            else np.ascontiguousarray(point_index, dtype=np.uint64))
        p = _lib.Params()
        p.equation = 1
        p.source_mode = _enum(source_mode, SOURCE_MODES, "source mode")
        p.alpha = 0.0
        p.N_walks = int(N_walks)
        p.epsilon = float(epsilon)
        p.max_steps = int(max_steps)
        p.max_ray_attempts = int(max_ray_attempts)
        p.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        p.method = _enum(method, METHODS, "method")
        self.params = p
        nv = C.c_int()
        solver._check(solver._L.wos_mesh_vertex_count(solver._ctx, C.byref(nv)))
        self.n_verts = nv.value

    def _source(self, Q, x0, sigma) -> _lib.GaussianSource:
        s = _lib.GaussianSource()
        s.Q = float(Q)
        xs = [float(v) for v in np.asarray(x0, dtype=np.float64).ravel()] + [0.0, 0.0, 0.0]
        s.x0 = (C.c_double * 3)(*xs[:3])
        s.sigma = float(sigma)
        s.mis_green_probability = self.mis_green_probability
        if self.proposal is not None:
            px = [float(v) for v in np.asarray(self.proposal[0], np.float64).ravel()] + [0.0] * 3
            s.proposal_x0 = (C.c_double * 3)(*px[:3])
            s.proposal_sigma = float(self.proposal[1])
        return s

    def _values(self, vertex_values):
        if vertex_values is None:
            return None
        g = np.ascontiguousarray(vertex_values, dtype=np.float64).ravel()
        if g.shape[0] != self.n_verts:
            raise ValueError(f"vertex_values has {g.shape[0]} entries; the mesh has "
                             f"{self.n_verts} vertices")
        return g

    def forward(self, Q, x0, sigma, vertex_values=None) -> HeatValues:
        n = self.n
        out = HeatValues(np.empty(n), np.empty(n), np.empty(n), np.empty(n),
                         np.empty(n, dtype=np.uint8))
        src = self._source(Q, x0, sigma)
        g = self._values(vertex_values)
        c = _lib.Counters()
        s = self.solver
        s._check(s._L.wos_heat_forward(s._ctx, C.byref(self.params), C.byref(src), _ptr(g),
                                       _ptr(self.probes), _ptr(self.point_index), n,
                                       _ptr(out.mean), _ptr(out.variance),
                                       _ptr(out.standard_error), _ptr(out.mean_steps),
                                       _ptr(out.location), C.byref(c)))
        out.counters = c.as_dict()
        return out

    def adjoint(self, Q, x0, sigma, vertex_values=None, grad_u=None) -> HeatGradients:
        n = self.n
        src = self._source(Q, x0, sigma)
        g = self._values(vertex_values)
        w = None if grad_u is None else np.ascontiguousarray(grad_u, dtype=np.float64).ravel()
        if w is not None and w.shape[0] != n:
            raise ValueError("grad_u must have one entry per probe")
        out = HeatGradients(np.zeros(5), np.zeros(self.n_verts), np.empty((n, 5)),
                            np.empty((n, 5)), np.empty(n))
        c = _lib.Counters()
        s = self.solver
        s._check(s._L.wos_heat_adjoint(s._ctx, C.byref(self.params), C.byref(src), _ptr(g),
                                       _ptr(self.probes), _ptr(self.point_index), n, _ptr(w),
                                       _ptr(out.grad_source), _ptr(out.grad_vertex_values),
                                       _ptr(out.jacobian), _ptr(out.jacobian_se),
                                       _ptr(out.replayed_mean), C.byref(c)))
        out.counters = c.as_dict()
        return out


def _autograd_function():
    import torch

    class GaussianHeatFunction(torch.autograd.Function):
        """Probe values of the heat problem as a differentiable torch op; the backward
        pass is the adjoint replay (no walk paths are stored)."""

        @staticmethod
        def forward(ctx, heat: HeatProblem, Q, x0, sigma, vertex_values):
            dev = Q.device
            g = None if vertex_values is None else vertex_values.detach().double().cpu().numpy()
            r = heat.forward(float(Q), x0.detach().double().cpu().numpy(), float(sigma), g)
            ctx.heat = heat
            ctx.args = (float(Q), x0.detach().double().cpu().numpy(), float(sigma), g)
            ctx.dims = x0.numel()
            ctx.has_values = vertex_values is not None
            ctx.device = dev
            return torch.from_numpy(r.mean).to(dev)

        @staticmethod
        def backward(ctx, grad_u):
            w = grad_u.detach().double().cpu().numpy()
            w = np.where(np.isfinite(w), w, 0.0)
            r = ctx.heat.adjoint(*ctx.args, grad_u=w)
            gs = torch.from_numpy(r.grad_source).to(ctx.device)
            gQ = gs[0]
            gx0 = gs[1:1 + ctx.dims]
            gsig = gs[4]
            gv = (torch.from_numpy(r.grad_vertex_values).to(ctx.device) if ctx.has_values
                  else None)
            return None, gQ, gx0, gsig, gv

    return GaussianHeatFunction


_FN = None


def heat_probe_values(heat: HeatProblem, Q, x0, sigma, vertex_values=None):
    """Differentiable probe values (float64 tensor of shape (n_probes,)) for torch tensors
    Q (scalar), x0 (dim), sigma (scalar) and vertex_values (n_verts, optional)."""
    global _FN
    if _FN is None:
        _FN = _autograd_function()
    return _FN.apply(heat, Q, x0, sigma, vertex_values)
