"""The CPU restatement (oracle/) against the golden fixtures produced by the
compiled reference (tests/golden/make_golden.py). Bit-exact: the assembled
FP64 system, iteration counts, pressure and projected velocities."""
import numpy as np
import pytest

from conftest import GoldenScene
from oracle import oracle


def test_oracle_matches_reference_golden(golden):
    name, g = golden
    sc = GoldenScene(g)
    res = oracle.project(sc, mic0=True)
    S = res.system
    assert S.n == len(g["rhs"])
    np.testing.assert_array_equal(S.indptr, g["indptr"])
    np.testing.assert_array_equal(S.indices, g["indices"])
    np.testing.assert_array_equal(S.data, g["data"])
    np.testing.assert_array_equal(S.rhs, g["rhs"])
    assert res.iterations == int(g["iterations_mic0"])
    assert res.reresid == float(g["reresid_mic0"])
    np.testing.assert_array_equal(res.pressure, g["pressure"])
    np.testing.assert_array_equal(res.pressure_active, g["pressure_active"])
    for d, k in enumerate("uvw"):
        np.testing.assert_array_equal(res.velocity[d], g[k])
        np.testing.assert_array_equal(res.velocity_active[d], g[k + "_active"])


def test_oracle_shipped_mode_is_plain_cg(golden):
    """The shipped solver discards its MIC(0) result (pcg_solver.h:379-384):
    the oracle's identity-preconditioned run reproduces its iteration count."""
    name, g = golden
    sc = GoldenScene(g)
    res = oracle.project(sc, mic0=False)
    assert res.iterations == int(g["iterations_shipped"])
    np.testing.assert_array_equal(res.pressure, g["pressure_shipped"])


def test_system_is_symmetric_m_matrix(golden):
    _, g = golden
    sc = GoldenScene(g)
    area, rho = oracle.fractions(sc)
    S = oracle.assemble(sc, area, rho)
    A = S.matrix()
    assert abs(A - A.T).max() == 0.0
    d = A.diagonal()
    assert (d > 0).all()
    off = A - np.diag(d) if A.shape[0] < 2000 else None
    assert (A.data[A.indices != np.repeat(np.arange(S.n), np.diff(S.indptr))] < 0).all()


def test_get_area_and_fraction_cases():
    import ctypes
    L = oracle.lib()
    def area(v00, v10, v11, v01):
        q = (ctypes.c_double * 4)(v00, v01, v10, v11)  # iso[i][j] row-major: [0][0],[0][1],[1][0],[1][1]
        return L.shkzo_get_area(q)
    assert area(1, 1, 1, 1) == 0.0
    assert area(-1, -1, -1, -1) == 1.0
    assert abs(area(-1, 1, 1, -1) - 0.5) < 1e-15
    assert L.shkzo_fraction(-1.0, 1.0) == 0.5
    assert L.shkzo_fraction(-1.0, -2.0) == 1.0
    assert L.shkzo_fraction(1.0, 2.0) == 0.0


def test_mic0_reduces_iterations_vs_shipped(golden):
    _, g = golden
    assert int(g["iterations_mic0"]) < int(g["iterations_shipped"])
