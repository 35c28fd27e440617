"""BatchHandle.set_particles_all marshals the particle arrays' addresses into ctypes arrays; it
reuses them while the caller passes the same float64 C-contiguous array objects, and builds them
afresh for new objects or for inputs it has to convert (a converted copy must not be reused, the
caller's array may change).  Checked on the host with a stand-in for the library call."""

import numpy as np

from particuology_hydraulic_penalty_b200 import handle as H


class _Lib:
    def __init__(self):
        self.calls = []

    def psc_batch_set_particles_all(self, h, ptrs, counts):
        self.calls.append(([ptrs[k] for k in range(len(counts))], list(counts), ptrs))
        return 0


def _handle(nwin):
    h = H.BatchHandle.__new__(H.BatchHandle)
    h.nwin = nwin
    h._staged = None
    h._h = None
    h._lib = _Lib()
    return h


def test_pointer_arrays_reused_only_for_the_same_objects():
    rng = np.random.default_rng(0)
    arrays = [rng.random((5, 10)), rng.random((3, 10)), np.zeros((0, 10))]
    h = _handle(3)
    h.set_particles_all(arrays)
    h.set_particles_all(arrays)
    first, second = h._lib.calls
    assert second[2] is first[2]  # the same ctypes pointer array
    assert first[0][0] == arrays[0].__array_interface__["data"][0] and first[0][2] is None
    assert h.P == [5, 3, 0]
    # a new object in one slot: built afresh
    arrays2 = [arrays[0], arrays[1].copy(), arrays[2]]
    h.set_particles_all(arrays2)
    third = h._lib.calls[-1]
    assert third[2] is not first[2]
    assert third[0][1] == arrays2[1].__array_interface__["data"][0]


def test_converted_inputs_are_not_reused():
    base = np.arange(40, dtype=np.float64).reshape(4, 10)
    arrays = [base[:, ::1].T.copy().T, np.arange(20, dtype=np.int64).reshape(2, 10)]  # Fortran order, ints
    h = _handle(2)
    h.set_particles_all(arrays)
    assert h._staged is None
    h.set_particles_all(arrays)
    a, b = h._lib.calls
    assert b[2] is not a[2]
    assert h.P == [4, 2]
