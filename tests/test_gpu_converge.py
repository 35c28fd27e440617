"""lbm_converge (coupling_sync/couple_psc_liggghts.py:284-296) run natively with the criterion on the
device, against the reference's per-step loop over collide_stream_psc() on the same solver class.

check_every = 1 must give the same iterations, residual, convergence flag, final populations,
diagnostics and particle loads as the loop; check_every = k stops on a multiple of k in the state a
plain run of that many steps reaches."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


class _PerStepLoop:
    """Only the reference's interface: coupling.lbm_converge runs its per-step Python loop."""

    def __init__(self, solver):
        self.solver = solver

    def collide_stream_psc(self):
        return self.solver.collide_stream_psc()


def _bed(precision, n=24):
    from particuology_hydraulic_penalty_b200 import Particle3D, SparsePscD3Q19

    parts = [Particle3D(6.0, 7.0, 8.0, 3.2), Particle3D(15.5, 14.0, 12.5, 4.1), Particle3D(9.0, 18.0, 19.0, 2.6),
             Particle3D(20.0, 5.0, 3.0, 1.3)]
    return SparsePscD3Q19(n=n, particles=parts, tau=0.8, subsamples=3, body_force_z=1.0e-5, static_geometry=False,
                          precision=precision)


@pytest.mark.parametrize("precision", ["fp64-exact", "fp32"])
@pytest.mark.parametrize("tol,max_steps", [(1.0e-6, 5000), (1.0e-12, 40)])
def test_native_converge_matches_reference_loop(precision, tol, max_steps):
    from particuology_hydraulic_penalty_b200 import coupling

    a = _bed(precision)
    b = _bed(precision)
    ia, ra, ca, da = coupling.lbm_converge(_PerStepLoop(a), residual_tol=tol, min_steps=3, max_steps=max_steps)
    ib, rb, cb, db = coupling.lbm_converge(b, residual_tol=tol, min_steps=3, max_steps=max_steps)
    assert (ib, cb) == (ia, ca)
    assert rb == ra
    assert ca == (max_steps == 5000)  # the loose tolerance converges, the tight one runs out of steps
    assert db == da
    assert np.array_equal(b.f, a.f)
    assert np.array_equal(b.uz, a.uz)
    assert np.array_equal(b.hydro_forces, a.hydro_forces)
    assert np.array_equal(b.hydro_torques, a.hydro_torques)


@pytest.mark.parametrize("k", [7, 50])
def test_check_every_k_stops_on_a_multiple_in_the_plain_state(k):
    from particuology_hydraulic_penalty_b200 import coupling

    s = _bed("fp32")
    it, res, conv, d = coupling.lbm_converge(s, residual_tol=1.0e-6, min_steps=1, max_steps=5000, check_every=k)
    assert conv and it % k == 0 and res < 1.0e-6
    ref = _bed("fp32")
    means = [ref.collide_stream_psc()["mean_uz"] for _ in range(it)]
    assert np.array_equal(s.f, ref.f)
    assert d["mean_uz"] == means[-1]
    # the criterion on the stopping pair of steps, recomputed from the per-step run's mean u_z
    m0, m1 = means[-2], means[-1]
    assert abs(res - abs(m1 - m0) / abs(m1)) <= 1e-9 * res


def test_converge_then_continue_and_particle_change():
    """After a native convergence the solver keeps stepping from the stopping state, and a new particle
    state (the coupled driver's next macro step) is taken by the next call."""
    from particuology_hydraulic_penalty_b200 import coupling

    a = _bed("fp64-exact")
    b = _bed("fp64-exact")
    it, _, conv, _ = coupling.lbm_converge(a, residual_tol=1.0e-5, min_steps=1, max_steps=5000)
    assert conv
    for _ in range(it):
        b.collide_stream_psc()
    assert np.array_equal(a.f, b.f)
    for s in (a, b):
        s.particles[0].x += 0.4  # moved in place, as the driver's update does
        s.collide_stream_psc()
    assert np.array_equal(a.f, b.f)
    assert np.array_equal(a.hydro_forces, b.hydro_forces)
