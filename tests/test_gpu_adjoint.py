"""The rollout adjoint (mps_adjoint_record / mps_adjoint_backward, adjoint.rollout).

Gradients with respect to the viscosity and the initial fluid velocities are checked
against central finite differences, tolerance 1e-3 relative:
  * of the FP64 GPU forward (the same step the adjoint differentiates);
  * of the CPU oracle in FP64 (an independent restatement of the reference's step), on a
    scene small enough for it.
Two losses: a random linear functional of the final positions and velocities (every
particle contributes), and the dam-break loss of the adjoint workload (squared error of
the fluid centroid and of the mean height beyond x = 0.7 m against the rollout at
nu = 2e-6). Differences are summed with exact rounding (math.fsum): the viscosity signal
of the centroid loss is a few hundred ulps of a centroid coordinate.

Step sizes. The viscosity is perturbed by the relative step 1e-4. The rollout is only
piecewise smooth in the initial velocities: a collision starts (kernel.cu:1193-1275) in
the step in which a pair first comes closer than 0.9 l0, and pressures are clamped at 0
at the free surface. Once the random initial velocities bring pairs together (after about
50 steps at the adjoint workload), a relative velocity step of 1e-4 moves such onsets by
a step and the central difference measures the jump, not the derivative. So the velocity
direction is checked at the step where the difference has stopped crossing them: 1e-6 on
the small scene (30 steps), 1e-8 on the 48 000-particle scene (200 steps) for a random
direction. The dam-break loss (a few hundred ulps of signal) is checked along a uniform
shift of all initial velocities in x, which moves the centroid without changing any
relative velocity, at the relative step 1e-7.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from mps_cuda_b200 import SceneDesc, configs, select_device
from mps_cuda_b200 import _lib as L
from mps_cuda_b200.adjoint import (RolloutProblem, dambreak_loss, loss_target, rollout,
                                   rollout_loss)

pytestmark = pytest.mark.gpu

RTOL = 1e-3   # finite differences vs adjoint
REL_STEP = 1e-4       # viscosity
VEL_STEP_SMALL = 1e-6  # initial velocities, small scene
VEL_STEP_LARGE = 1e-8  # initial velocities, adjoint workload, random direction
VEL_STEP_SHIFT = 1e-7  # initial velocities, adjoint workload, uniform shift


def small_problem():
    desc = SceneDesc(0.02, (0.4, 0.2, 0.4), (8, 6, 10), seed=3, vel_sigma=0.05, vel_seed=1)
    return RolloutProblem(desc, dt=2e-4, steps=30, every=10)


def config_problem():
    desc, dt, steps = configs.WORKLOADS["adjoint_l0.01_48k"]
    return RolloutProblem(desc, dt=dt, steps=steps, every=20)


def fsum_dot(a, b):
    return math.fsum((np.asarray(a, np.float64) * np.asarray(b, np.float64)).ravel())


def linear_value(st, fluid, a, b):
    return fsum_dot(a, st["pos"][:, fluid]) + fsum_dot(b, st["vel"][:, fluid])


def rel(a, b):
    return abs(a - b) / max(abs(a), abs(b), 1e-300)


def adjoint_of_linear(problem, a, b, nu):
    """Adjoint gradients of sum a.pos + b.vel; backward twice on one recording."""
    n, f = problem.typ.shape[0], problem.fluid
    lam_pos = np.zeros((3, n)); lam_pos[:, f] = a
    lam_vel = np.zeros((3, n)); lam_vel[:, f] = b
    h = problem.solver(nu, problem.vel[:, f])
    try:
        h.adjoint_record(problem.steps, problem.every)
        end = h.state()
        _, gv, gnu = h.adjoint_backward(lam_pos, lam_vel)
        _, gv2, gnu2 = h.adjoint_backward(lam_pos, lam_vel)
        again = h.state()
    finally:
        h.close()
    # repeatable up to the order of the double atomic adds (mirror -> owner terms), and
    # the handle is left at the end of the rollout
    gv, gv2 = gv[:, f], gv2[:, f]
    assert np.max(np.abs(gv - gv2)) <= 1e-8 * np.max(np.abs(gv)), np.max(np.abs(gv - gv2))
    assert rel(gnu, gnu2) < 1e-8
    for k in ("pos", "vel", "typ"):
        assert np.array_equal(end[k], again[k]), k
    return gv, gnu


def check_linear(problem, run, seed, vel_step):
    f = problem.fluid
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((3, f.size))
    b = rng.standard_normal((3, f.size))
    nu = configs.NU
    v0 = problem.vel[:, f].copy()
    gv, gnu = adjoint_of_linear(problem, a, b, nu)
    h = REL_STEP * nu
    fd_nu = (linear_value(run(nu + h, v0), f, a, b) - linear_value(run(nu - h, v0), f, a, b)) / (2 * h)
    d = rng.standard_normal(v0.shape)
    eps = vel_step * float(np.sqrt(np.mean(v0 ** 2)))
    fd_v = (linear_value(run(nu, v0 + eps * d), f, a, b)
            - linear_value(run(nu, v0 - eps * d), f, a, b)) / (2 * eps)
    return (gnu, fd_nu), (fsum_dot(gv, d), fd_v)


def gpu_run(problem):
    return lambda nu, v0: problem.run(nu, v0)


def oracle_run(problem):
    from oracle.oracle import Oracle, params_from

    def run(nu, v0):
        p = problem.params
        p.knm_vsc = float(nu)
        vel = problem.vel.copy()
        vel[:, problem.fluid] = v0
        o = Oracle(params_from(p), problem.typ, problem.pos, vel, problem.nrm)
        try:
            o.step(problem.steps)
            return o.state()
        finally:
            o.close()
            p.knm_vsc = configs.NU
    return run


@pytest.fixture(scope="module", autouse=True)
def _device():
    select_device(0)


def test_linear_functional_small_scene_vs_gpu_differences():
    pr = small_problem()
    (gnu, fd_nu), (ad_v, fd_v) = check_linear(pr, gpu_run(pr), seed=11, vel_step=VEL_STEP_SMALL)
    assert rel(gnu, fd_nu) < RTOL, (gnu, fd_nu)
    assert rel(ad_v, fd_v) < RTOL, (ad_v, fd_v)


def test_linear_functional_small_scene_vs_oracle_differences():
    """The FP64 reference gradient: finite differences of the CPU oracle's rollouts."""
    pr = small_problem()
    (gnu, fd_nu), (ad_v, fd_v) = check_linear(pr, oracle_run(pr), seed=12, vel_step=VEL_STEP_SMALL)
    assert rel(gnu, fd_nu) < RTOL, (gnu, fd_nu)
    assert rel(ad_v, fd_v) < RTOL, (ad_v, fd_v)


def test_linear_functional_adjoint_workload():
    pr = config_problem()
    (gnu, fd_nu), (ad_v, fd_v) = check_linear(pr, gpu_run(pr), seed=13, vel_step=VEL_STEP_LARGE)
    assert rel(gnu, fd_nu) < RTOL, (gnu, fd_nu)
    assert rel(ad_v, fd_v) < RTOL, (ad_v, fd_v)


def exact_loss(problem, nu, v0, target):
    return rollout_loss(problem, nu, v0, target)


def test_dambreak_loss_through_torch_autograd():
    import torch
    pr = config_problem()
    f = pr.fluid
    v0 = pr.vel[:, f].copy()
    target = loss_target(pr, 2e-6, v0)
    nu_t = torch.tensor(configs.NU, dtype=torch.float64, requires_grad=True)
    vel_t = torch.tensor(v0, dtype=torch.float64, requires_grad=True)
    pos, vel, alive = rollout(nu_t, vel_t, pr)
    loss = dambreak_loss(pos, alive, torch.tensor(target))
    loss.backward()
    assert float(loss.detach()) > 0
    gnu, gv = float(nu_t.grad), vel_t.grad.numpy()
    assert np.isfinite(gnu) and np.all(np.isfinite(gv))
    nu = configs.NU
    h = REL_STEP * nu
    fd_nu = (exact_loss(pr, nu + h, v0, target) - exact_loss(pr, nu - h, v0, target)) / (2 * h)
    d = np.zeros(v0.shape)
    d[0] = 1.0  # every initial velocity shifted in x
    eps = VEL_STEP_SHIFT * float(np.sqrt(np.mean(v0 ** 2)))
    fd_v = (exact_loss(pr, nu, v0 + eps * d, target) - exact_loss(pr, nu, v0 - eps * d, target)) / (2 * eps)
    assert rel(gnu, fd_nu) < RTOL, (gnu, fd_nu)
    assert rel(fsum_dot(gv, d), fd_v) < RTOL, (fsum_dot(gv, d), fd_v)


def test_backward_before_record_is_a_state_error():
    pr = small_problem()
    h = pr.solver(configs.NU, pr.vel[:, pr.fluid])
    try:
        with pytest.raises(L.MPSError) as e:
            h.adjoint_backward()
        assert e.value.code == L.MPS_ERR_STATE
    finally:
        h.close()
