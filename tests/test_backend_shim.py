"""The backend's array namespace under the reference's own solvers, on CPU.

The reference solvers (installed unmodified in ``baseline/_ref``) only touch
the backend through ``xp`` and a few ``Backend`` methods.  Run over torch CPU
tensors (the same namespace class the B200 backend uses on the GPU) and an
oracle-backed operator, they must produce the run they produce over NumPy:
this pins ``copy()`` on namespace arrays and NumPy complex scalars times
tensors (``numpy.complex64`` is not read correctly by torch itself).
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

from conftest import ROOT, golden, rel_err

REF = os.path.join(ROOT, "baseline", "_ref")


def _reference():
    if not os.path.isdir(os.path.join(REF, "em3d")):
        pytest.skip("the reference is not installed in baseline/_ref")
    if REF not in sys.path:
        sys.path.insert(0, REF)
    import em3d

    return em3d


class _OracleOperator:
    """matvec / rmatvec of the oracle on host arrays, wrapped for a backend."""

    def __init__(self, backend, chi, N, L, k, precision, torch_arrays):
        from oracle import em as oem

        self.backend = backend
        self._chi = chi
        self._N = N
        self._kh = oem.kernel_hat(N, L, k, precision)
        self._torch = torch_arrays

    def _wrap(self, y):
        if not self._torch:
            return y
        import torch

        from em3d_b200.backend import as_device_array

        return as_device_array(torch.as_tensor(y))

    def _host(self, x):
        return x.numpy() if hasattr(x, "numpy") else np.asarray(x)

    def matvec(self, x):
        from oracle import em as oem

        return self._wrap(oem.matvec(self._chi, self._host(x), self._kh, self._N))

    def rmatvec(self, x):
        from oracle import em as oem

        return self._wrap(oem.rmatvec(self._chi, self._host(x), self._N, khat=self._kh))


@pytest.mark.parametrize("prec", ["double", "single"])
@pytest.mark.parametrize("solver", ["BiCGStab", "TwoStep"])
def test_reference_solver_on_torch_namespace_matches_numpy_run(solver, prec):
    import torch

    from em3d_b200.backend import Backend, Precision, TorchNamespace

    em3d = _reference()
    g = golden("em_aniso12.npz")
    N, L, k = tuple(int(v) for v in g["N"]), tuple(float(v) for v in g["L"]), float(g["k"])
    chi, wave = g[f"chi_{prec}"], g[f"wave_{prec}"]
    rtol = 1e-8 if prec == "double" else 1e-5
    cfg = em3d.SolverConfig(max_iter=60, rtol=rtol)

    np_be = em3d.Backend.numpy(em3d.Precision.DOUBLE if prec == "double" else em3d.Precision.SINGLE)
    ref = getattr(em3d, solver)(cfg).solve(_OracleOperator(np_be, chi, N, L, k, prec, False), wave)

    t_be = Backend(xp=TorchNamespace(torch.device("cpu")), device="cuda",
                   precision=Precision.DOUBLE if prec == "double" else Precision.SINGLE)
    got = getattr(em3d, solver)(cfg).solve(_OracleOperator(t_be, chi, N, L, k, prec, True), torch.as_tensor(wave))

    assert got.status == ref.status
    assert got.iterations == ref.iterations
    assert got.matvec_count == ref.matvec_count
    # torch and NumPy sum the inner products in different orders; BiCGStab
    # amplifies that round-off as the residual falls, and TwoStep's history is
    # chaotic in it after about twenty updates (its early history is compared)
    if solver == "BiCGStab":
        np.testing.assert_allclose(got.residual_history, ref.residual_history,
                                   rtol=1e-4 if prec == "double" else 5e-2)
        sol_tol = 1e-10 if prec == "double" else 1e-4
    else:
        n = 15 if prec == "double" else 10
        np.testing.assert_allclose(got.residual_history[:n], ref.residual_history[:n],
                                   rtol=1e-9 if prec == "double" else 1e-3)
        sol_tol = 1e-3
    u = t_be.to_host(got.u)
    assert u.dtype == ref.u.dtype
    assert rel_err(u, ref.u) < sol_tol


def test_namespace_arrays_copy_and_complex64_scalars():
    import torch

    from em3d_b200.backend import TorchNamespace

    xp = TorchNamespace(torch.device("cpu"))
    x = xp.asarray(np.arange(4, dtype=np.complex64))
    y = x.copy()
    y[0] = 7.0
    assert float(x[0].real) == 0.0
    z = np.complex64(1 + 2j) * x
    assert z.dtype == torch.complex64
    np.testing.assert_array_equal(z.numpy(), np.complex64(1 + 2j) * np.arange(4, dtype=np.complex64))
    w = x - np.complex64(0.5 - 1j) * x
    np.testing.assert_array_equal(w.numpy(), np.arange(4, dtype=np.complex64)
                                  - np.complex64(0.5 - 1j) * np.arange(4, dtype=np.complex64))
