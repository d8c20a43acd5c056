"""lbm_field_diagnostics_static: the diagnostics without any device allocation.

It is meant for callers that cannot allocate device memory at the point
where they need the numbers (all of it handed to a pool, or an allocation
would synchronise the device), so it reduces caller-owned device arrays
through the library's file-scope scratch array.  Checked against
lbm_diagnostics on the same state, on two calls in a row (the scratch keeps
the previous call's contents), within the FP64 summation-order tolerance of
the other diagnostics tests.  Collected last so that a stop-at-first-failure
run has executed every other test before this one.
"""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O

pkg = O.pkg
pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def _static(torch, den, prev, ux, uy, uz):
    out = np.zeros(8, np.float64)
    torch.cuda.synchronize()
    p = [C.c_void_p(t.data_ptr()) if t is not None else None for t in (den, prev, ux, uy, uz)]
    pkg.check(pkg.lib().lbm_field_diagnostics_static(*p, C.c_longlong(den.numel()),
                                                     out.ctypes.data_as(C.c_void_p), None))
    return out


def test_static_diagnostics_match_lbm_diagnostics_twice():
    torch = pytest.importorskip("torch")
    iv = pkg.make_inputval(40, 36, 44, casetype=pkg.CAVITY, re=150.0, u=0.1, mrt=True, les=True,
                           cs=0.1, h=40)
    dom = pkg.Domain(iv, pkg.default_options(init_kind=pkg.INIT_DENSITY_NOISE, noise_amp=1e-4))
    results = []
    for _ in range(2):
        dom.run(7)
        prev = dom.macroscopic()[0]
        dom.run(1)
        den, ux, uy, uz = dom.macroscopic()
        want = dom.diagnostics()
        got = _static(torch, _dev(torch, den), _dev(torch, prev), _dev(torch, ux),
                      _dev(torch, uy), _dev(torch, uz))
        for k in (0, 1, 2, 3, 4, 5):
            assert abs(got[k] - want[k]) <= 1e-12 * max(1.0, abs(want[k])), (k, got[k], want[k])
        assert got[6] == want[6] and got[7] == want[7] == 0
        results.append(got)
    assert not np.array_equal(results[0], results[1])  # the state moved on between calls
    dom.close()


def test_static_diagnostics_without_previous_density_and_size_limit():
    torch = pytest.importorskip("torch")
    n = 1000
    den = torch.ones(n, device="cuda")
    u = torch.zeros(n, device="cuda")
    out = _static(torch, den, None, u, u, u)
    assert out[0] == n and out[4] == 0.0 and out[7] == 0
    big = np.zeros(8, np.float64)
    rc = pkg.lib().lbm_field_diagnostics_static(C.c_void_p(den.data_ptr()), None,
                                                C.c_void_p(u.data_ptr()), C.c_void_p(u.data_ptr()),
                                                C.c_void_p(u.data_ptr()),
                                                C.c_longlong(67108864 + 1),
                                                big.ctypes.data_as(C.c_void_p), None)
    assert rc == pkg.LBM_ERR_INVALID
    assert b"capacity" in pkg.lib().lbm_last_error()


def test_static_diagnostics_on_the_256_cube_cavity_fields():
    """The 256^3 MRT+LES cavity (Cs 0.1, Re 5000): 16,777,216 nodes, i.e.
    1,024 partial-sum blocks reduced by the fixed-order final pass, checked
    against lbm_diagnostics on the same state, twice in a row."""
    torch = pytest.importorskip("torch")
    iv = pkg.make_inputval(256, casetype=pkg.CAVITY, re=5000.0, u=0.1, mrt=True, les=True,
                           cs=0.1)
    dom = pkg.Domain(iv, pkg.default_options(init_kind=pkg.INIT_DENSITY_NOISE, noise_amp=1e-6))
    assert 256 ** 3 // (256 * 64) == 1024
    for _ in range(2):
        dom.run(4)
        prev = dom.macroscopic()[0]
        dom.run(1)
        den, ux, uy, uz = dom.macroscopic()
        want = dom.diagnostics()
        got = _static(torch, _dev(torch, den), _dev(torch, prev), _dev(torch, ux),
                      _dev(torch, uy), _dev(torch, uz))
        for k in (0, 1, 2, 3, 4, 5):
            assert abs(got[k] - want[k]) <= 1e-12 * max(1.0, abs(want[k])), (k, got[k], want[k])
        assert got[6] == want[6] and got[7] == want[7] == 0
    dom.close()
