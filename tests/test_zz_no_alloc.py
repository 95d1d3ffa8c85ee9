"""The no-allocation all-<Z_i> entry point against the regular one.

nqpu_expectation_z_all_noalloc is for callers that cannot allocate device
memory: plugins whose host runtime owns the device memory pool, and real-time
loops that must not wait on the allocator.  The caller owns the amplitude and output
buffers; the entry point takes its scratch from a fixed device array of the
library, so its size is capped (complex64 up to 28 qubits, complex128 up to 27)
and the cases at those caps fill the array.  This file is collected last so
that a run stopping at the first failure has run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

from nqpu_b200 import _lib, circuits
from nqpu_b200.state import Circuit, StateVector

pytestmark = pytest.mark.gpu

C128, C64 = 0, 1


def _random_state(n, dtype, seed):
    rng = np.random.default_rng(seed)
    a = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    a /= np.linalg.norm(a)
    return a.astype(np.complex64 if dtype == "c64" else np.complex128)


@pytest.mark.parametrize("n,dtype", [(3, "c128"), (10, "c128"), (20, "c128"), (7, "c64"), (14, "c64"), (22, "c64")])
def test_noalloc_matches_regular_entry_point_twice(n, dtype):
    import torch

    lib = _lib.load()
    amps = _random_state(n, dtype, seed=n)
    # regular entry point on an engine-owned state holding the same amplitudes
    sv = StateVector(n, dtype)
    sv.set_amplitudes(amps.astype(np.complex128))
    expected = sv.expectation_z_all()

    # caller-owned device buffers (allocated by the caller, not by the library)
    real = np.ascontiguousarray(amps).view(np.float32 if dtype == "c64" else np.float64)
    d_amp = torch.from_numpy(real.copy()).cuda()
    d_out = torch.empty(n, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    code = C64 if dtype == "c64" else C128
    for _ in range(2):  # two calls in a row share the library's scratch array
        d_out.fill_(float("nan"))
        err = lib.nqpu_expectation_z_all_noalloc(C.c_void_p(d_amp.data_ptr()), n, code,
                                                 C.cast(C.c_void_p(d_out.data_ptr()), C.POINTER(C.c_double)),
                                                 C.c_void_p(stream.cuda_stream))
        assert err == 0
        torch.cuda.synchronize()
        got = d_out.cpu().numpy()
        np.testing.assert_allclose(got, expected, atol=1e-12, rtol=0)
    sv.close()


@pytest.mark.parametrize("n,dtype", [(28, "c64"), (27, "c128")])
def test_noalloc_at_its_documented_limits(n, dtype):
    # the largest states the fixed scratch array serves: the per-segment
    # partials fill it up to the region that holds the n+1 sums
    import torch

    lib = _lib.load()
    sv = StateVector(n, dtype)
    Circuit(n, circuits.brickwork(n, 2, seed=n)).execute(sv, "tiled")
    expected = sv.expectation_z_all()
    amps = sv.amplitudes()  # complex128 on the host
    sv.close()
    host = amps.astype(np.complex64) if dtype == "c64" else amps
    del amps
    real = host.view(np.float32 if dtype == "c64" else np.float64)
    d_amp = torch.from_numpy(real).cuda()
    del host, real
    d_out = torch.empty(n, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    code = C64 if dtype == "c64" else C128
    for _ in range(2):
        d_out.fill_(float("nan"))
        err = lib.nqpu_expectation_z_all_noalloc(C.c_void_p(d_amp.data_ptr()), n, code,
                                                 C.cast(C.c_void_p(d_out.data_ptr()), C.POINTER(C.c_double)),
                                                 C.c_void_p(stream.cuda_stream))
        assert err == 0
        torch.cuda.synchronize()
        np.testing.assert_allclose(d_out.cpu().numpy(), expected, atol=1e-12, rtol=0)
    del d_amp
    torch.cuda.empty_cache()


def test_noalloc_rejects_states_beyond_its_fixed_scratch():
    lib = _lib.load()
    fake = C.c_void_p(256)  # never dereferenced: the size check comes first
    out = C.cast(C.c_void_p(256), C.POINTER(C.c_double))
    assert lib.nqpu_expectation_z_all_noalloc(fake, 29, C64, out, None) == 2  # NQPU_INVALID_PARAMETER
    assert lib.nqpu_expectation_z_all_noalloc(fake, 28, C128, out, None) == 2
    assert lib.nqpu_expectation_z_all_noalloc(None, 10, C64, out, None) == 5  # NQPU_NULL_POINTER
