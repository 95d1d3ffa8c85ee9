"""Edge cases at the limits: the largest states one B200 holds (34 qubits
complex64 and 33 qubits complex128, 128 GiB each), the creation limits of
the C ABI, empty circuits and one-qubit states (the reference's state tests,
lib.rs:2533-2600, start from one and two qubits)."""
import numpy as np
import pytest

from nqpu_b200 import _lib
from nqpu_b200.state import Circuit, StateVector

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,dtype", [(34, "c64"), (33, "c128")])
def test_largest_state_uniform_superposition(n, dtype):
    sv = StateVector(n, dtype)
    try:
        c = Circuit(n, [("h", (q,), ()) for q in range(n)] + [("z", (n - 1,), ()), ("h", (n - 1,), ())])
        c.execute(sv, "tiled")
        # H on every qubit, then HZH = X on the top qubit: <Z_i> = 0 except <Z_top> = -1
        z = sv.expectation_z_all()
        tol = 1e-5 if dtype == "c64" else 1e-10
        assert np.abs(z[:-1]).max() < tol
        assert abs(z[-1] + 1.0) < tol
        assert abs(sv.norm() - 1.0) < tol
        shots = sv.sample(256)
        assert np.all((shots >> np.uint64(n - 1)) & np.uint64(1) == 1)
        assert shots.max() < (1 << n)
    finally:
        sv.close()


def test_creation_limits():
    lib = _lib.load()
    assert not lib.nqpu_state_create_ex(35, 1)
    assert not lib.nqpu_state_create_ex(0, 0)
    assert not lib.nqpu_state_create(31)  # the reference's C FFI cap (c_ffi.rs:789)
    h = lib.nqpu_state_create(30)
    assert h
    lib.nqpu_state_destroy(h)


@pytest.mark.parametrize("dtype", ["c64", "c128"])
def test_empty_circuit_and_one_qubit(dtype):
    with StateVector(1, dtype) as sv:
        Circuit(1, []).execute(sv)
        np.testing.assert_allclose(sv.amplitudes(), [1.0, 0.0], atol=0)
        Circuit(1, [("ry", (0,), (0.5,)), ("rz", (0,), (0.3,))]).execute(sv)
        a = sv.amplitudes()
        assert abs(np.vdot(a, a).real - 1.0) < 1e-6
    with StateVector(20, dtype) as sv:
        Circuit(20, []).execute(sv, "tiled")
        assert abs(sv.amplitude(0) - 1.0) == 0.0
