"""GPU adjoint of the permeability: vs the FP64 reference adjoint, vs central finite differences,
FP32 vs FP64, checkpoint independence, and the torch.autograd wrapper."""

import numpy as np
import pytest
import torch

from oracle import psc_adjoint as adj

pytestmark = pytest.mark.gpu

PARTS = np.array([[4.3, 5.1, 4.8, 2.2] + [0.0] * 6,
                  [7.9, 3.2, 6.1, 1.7] + [0.0] * 6,
                  [2.0, 8.5, 1.0, 1.9] + [0.0] * 6])
N, S, EPS, TAU, F, STEPS = 10, 2, 0.05, 0.8, (1e-4, 0.0, 0.0), 25


def problem(precision="fp64", every=7, steps=STEPS):
    from particuology_hydraulic_penalty_b200.adjoint import PermeabilityProblem

    return PermeabilityProblem(N, tau=TAU, force=F, subsamples=S, eps=EPS, steps=steps, checkpoint_every=every,
                               precision=precision)


def test_gpu_fp64_adjoint_matches_reference_adjoint():
    Kref, gref, _ = adj.gradient(PARTS, N, S, EPS, TAU, F, STEPS)
    pr = problem("fp64")
    K = pr.forward(PARTS)
    g = pr.backward()
    assert abs(K - Kref) <= 1e-12 * abs(Kref)
    assert np.linalg.norm(g - gref) <= 1e-9 * np.linalg.norm(gref)


def test_gpu_adjoint_matches_central_differences():
    pr = problem("fp64")
    pr.forward(PARTS)
    g = pr.backward()
    h = 1e-3
    worst = 0.0
    for p in range(len(PARTS)):
        for k in range(4):
            pp = PARTS.copy()
            pp[p, k] += h
            pm = PARTS.copy()
            pm[p, k] -= h
            fd = (problem("fp64").forward(pp) - problem("fp64").forward(pm)) / (2 * h)
            worst = max(worst, abs(fd - g[p, k]) / abs(fd))
    assert worst <= 1e-3


def test_fp32_adjoint_close_to_fp64():
    p64 = problem("fp64")
    p64.forward(PARTS)
    g64 = p64.backward()
    p32 = problem("fp32")
    p32.forward(PARTS)
    g32 = p32.backward()
    assert np.linalg.norm(g32 - g64) <= 1e-3 * np.linalg.norm(g64)


def test_checkpoint_interval_does_not_change_gradient():
    a = problem("fp64", every=7)
    a.forward(PARTS)
    b = problem("fp64", every=STEPS)
    b.forward(PARTS)
    assert np.array_equal(a.backward(), b.backward())


def test_autograd_function():
    from particuology_hydraulic_penalty_b200.adjoint import permeability

    pr = problem("fp64")
    centres = torch.tensor(PARTS[:, 0:3], dtype=torch.float64, requires_grad=True)
    radii = torch.tensor(PARTS[:, 3], dtype=torch.float64, requires_grad=True)
    K = permeability(centres, radii, pr, template=PARTS)
    (2.0 * K).backward()
    ref = problem("fp64")
    ref.forward(PARTS)
    g = ref.backward()
    assert np.allclose(centres.grad.numpy(), 2.0 * g[:, 0:3], rtol=1e-12, atol=0)
    assert np.allclose(radii.grad.numpy(), 2.0 * g[:, 3], rtol=1e-12, atol=0)


def test_native_adjoint_handle_matches_python_problem():
    """The C++ adjoint handle (psc_adjoint_*) runs the same algorithm as PermeabilityProblem."""
    from particuology_hydraulic_penalty_b200 import _native as nat
    from particuology_hydraulic_penalty_b200 import windows as wgen
    from particuology_hydraulic_penalty_b200.adjoint import PermeabilityProblem
    from particuology_hydraulic_penalty_b200.handle import AdjointHandle, make_config

    w = wgen.make_window(24, "preloaded", 21)
    prob = PermeabilityProblem(24, tau=0.8, force=(1e-6, 0.0, 0.0), subsamples=4, eps=0.05, steps=120,
                               checkpoint_every=25, precision="fp32")
    K_py = prob.forward(w.particles)
    g_py = prob.backward()
    h = AdjointHandle(make_config((24, 24, 24), tau=0.8, force=(1e-6, 0.0, 0.0), subsamples=4,
                                  store=nat.STORE_F32), smooth_eps=0.05, steps=120, checkpoint_every=25)
    K_c = h.forward(w.particles)
    g_c = h.backward()
    assert abs(K_c - K_py) <= 1e-12 * abs(K_py)
    assert np.abs(g_c - g_py).max() <= 1e-12 * np.abs(g_py).max()
    # a second run on the same handle gives the same answer
    assert h.forward(w.particles) == K_c
    assert np.array_equal(h.backward(), g_c)


def test_full_size_adjoint_case_gradient_and_cost():
    """The adjoint sensitivity case at its stated size: a preloaded 96^3 window with 64 fines (radius
    0.15x the skeleton's), 2000 forward steps checkpointed every 100, FP32 populations with FP64
    reductions.  On 8 seeded fines the FP64 adjoint matches FP64 central differences of K (step
    1e-3 lu) to 1e-3 relative in every (x, y, z, r) component, the FP32 adjoint the FP64 one to
    1e-3, and forward + backward costs at most 4x the forward pass (CUDA events)."""
    from particuology_hydraulic_penalty_b200 import validation

    r = validation.adjoint_check(n=96, n_fines=64, steps=2000, every=100, n_check=8)
    assert r["n_fines"] == 64
    assert r["fd_vs_adjoint_fp64_max_rel"] <= 1e-3, r["fd_vs_adjoint_fp64_max_rel"]
    assert r["adjoint_fp32_vs_fp64_norm_rel"] <= 1e-3, r["adjoint_fp32_vs_fp64_norm_rel"]
    assert r["adjoint_plus_forward_over_forward"] <= 4.0, r["adjoint_plus_forward_over_forward"]
    assert abs(r["K_fp32"] - r["K_fp64"]) <= 1e-4 * abs(r["K_fp64"])
