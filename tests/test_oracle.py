"""The oracle itself: pinned to the reference before it is trusted.

- bit-exact against the golden fixtures produced by the reference's own
  lbm_codelets.cpp (tests/golden/make_golden.py);
- bit-exact against the reference codelets run live, when oracle/_ref was
  built here (the reference tree is only present at build time);
- invariants the reference's physics guarantees (mass conservation of the
  closed cavity, rest state, tile-count invariance, FP32 vs FP64).
"""
import glob
import os

import numpy as np
import pytest

import oracle_lib as O

pkg = O.pkg
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def cavity(n, re=None, tau=None, cs=0.0, mrt=True, les=True, u=0.1):
    return pkg.make_inputval(n, casetype=pkg.CAVITY, re=re, tau=tau, u=u, mrt=mrt, les=les,
                             cs=cs, h=n)


def golden_files(prefix="cavity"):
    return sorted(glob.glob(os.path.join(GOLDEN, prefix + "*.npz")))


def iv_from_golden(g):
    n = int(g["nx"])
    iv = cavity(n, tau=float(g["tau"]), cs=float(g["cs"]), mrt=bool(g["mrt"]), les=bool(g["les"]),
                u=float(g["u"]))
    assert np.float32(iv.m_dTau) == g["tau"]
    return iv


@pytest.mark.parametrize("path", golden_files("cavity"), ids=os.path.basename)
def test_port_reproduces_reference_golden_bit_exact(path):
    g = np.load(path)
    iv = iv_from_golden(g)
    r = O.Run(iv, init_kind=int(g["init_kind"]), seed=int(g["seed"]), amp=float(g["noise_amp"]))
    r.step(int(g["steps"]))
    f = r.fields()
    for k in ("den", "ux", "uy", "uz"):
        np.testing.assert_array_equal(f[k].astype(np.float32), g[k], err_msg=k)
    if "arF" in g:
        np.testing.assert_array_equal(f["arF"].astype(np.float32), g["arF"])
        np.testing.assert_array_equal(f["arF"][:, 2, :, 9].astype(np.float32),
                                      g["printout_dir9_k2"])


def test_golden_fixtures_present():
    names = [os.path.basename(p) for p in golden_files("cavity")]
    assert "cavity10_mrtles_cs0.npz" in names and "cavity10_mrtles_cs01.npz" in names


def test_shipped_config_les_is_inactive_and_cs01_active():
    # F8: main.cpp never assigns m_dSmagorinsky, so tau_eddy = 0 in the shipped run
    r0 = O.Run(cavity(10, re=1000.0, cs=0.0))
    r0.step(5)
    assert np.abs(r0.fields()["tau_e"]).max() < 1e-6
    r1 = O.Run(cavity(10, re=1000.0, cs=0.1))
    r1.step(5)
    assert np.abs(r1.fields()["tau_e"]).max() > 1e-4


needs_ref = pytest.mark.skipif(O.poplar_ref_lib() is None,
                               reason="reference codelets not built here")


@needs_ref
@pytest.mark.parametrize("shape,steps,cs,kind", [
    ((10, 10, 10), 199, 0.1, 0),
    ((12, 9, 7), 30, 0.1, 1),
    ((17, 13, 11), 20, 0.2, 1),
])
def test_port_matches_reference_codelets_live(shape, steps, cs, kind):
    nx, ny, nz = shape
    iv = pkg.make_inputval(nx, ny, nz, casetype=pkg.CAVITY, re=300.0, u=0.1, mrt=True,
                           les=True, cs=cs, h=nx)
    a = O.Run(iv, init_kind=kind, amp=1e-6)
    b = O.Run(iv, init_kind=kind, amp=1e-6, which="ref")
    a.step(steps)
    b.step(steps)
    fa, fb = a.fields(), b.fields()
    for k in ("arF", "den", "ux", "uy", "uz", "pden", "tau_e", "ntype", "dstate"):
        np.testing.assert_array_equal(fa[k], fb[k], err_msg=k)


def test_tile_count_invariance():
    iv = cavity(14, re=200.0, cs=0.1)
    a = O.Run(iv, init_kind=1, amp=1e-6, split=1)
    b = O.Run(iv, init_kind=1, amp=1e-6, split=5)
    a.step(25)
    b.step(25)
    fa, fb = a.fields(), b.fields()
    for k in ("arF", "den", "ux"):
        np.testing.assert_array_equal(fa[k], fb[k])


@pytest.mark.parametrize("mrt,les", [(False, False), (True, True)])
def test_closed_cavity_conserves_mass_fp64(mrt, les):
    iv = cavity(12, re=100.0, cs=0.1, mrt=mrt, les=les)
    r = O.Run(iv, init_kind=1, amp=1e-4, double=True)
    m0 = r.fields()["arF"].sum()
    r.step(100)
    m1 = r.fields()["arF"].sum()
    assert abs(m1 - m0) / m0 < 1e-12


def test_rest_state_is_stationary():
    iv = cavity(9, tau=0.8, mrt=True, les=True, cs=0.1, u=0.0)
    r = O.Run(iv)
    f0 = r.fields()["arF"].copy()
    r.step(50)
    f1 = r.fields()["arF"]
    assert np.abs(f1 - f0).max() < 1e-7


def test_fp32_tracks_fp64():
    iv = cavity(12, re=200.0, cs=0.1)
    a = O.Run(iv, init_kind=1, amp=1e-6)
    b = O.Run(iv, init_kind=1, amp=1e-6, double=True)
    a.step(100)
    b.step(100)
    fa, fb = a.fields(), b.fields()
    assert O.rel_field_err(fa["den"], fb["den"]) < 1e-5
    assert O.rel_vel_err((fa["ux"], fa["uy"], fa["uz"]), (fb["ux"], fb["uy"], fb["uz"])) < 1e-5


def test_channel_oracle_runs_and_inlet_profile():
    iv = pkg.make_inputval(24, 10, 12, casetype=pkg.CHANNEL, tau=0.7, u=0.05, mrt=True, les=True,
                           cs=0.1)
    r = O.Run(iv, init_kind=pkg.INIT_CHANNEL, amp=0.01)
    f = r.fields()
    t = f["ntype"]
    assert (t[:, :, 0][1:-1, 1:-1] == pkg.NODE_INLET).all()
    assert (t[:, :, -1][1:-1, 1:-1] == pkg.NODE_OUTLET).all()
    assert (t[0] == pkg.NODE_FIXEDWALL).all() and (t[:, 0] == pkg.NODE_FIXEDWALL).all()
    r.step(60)
    f = r.fields()
    assert np.isfinite(f["arF"]).all()
    # the flow is driven through the channel: mean u_x positive in the core
    assert f["ux"][3:-3, 3:-3, 5:-5].mean() > 0.005


def test_noise_and_profile_are_fixed():
    L = O.oracle_lib()
    v = [L.orc_noise(1, n, 0) for n in range(1000)]
    assert min(v) >= -1.0 and max(v) < 1.0 and abs(np.mean(v)) < 0.1
    # deterministic: exact values of the counter hash (24-bit grid)
    assert all((x + 1.0) * 2 ** 23 == int((x + 1.0) * 2 ** 23) for x in v)
    assert L.orc_profile(0.05, 0, 5, 11, 11) == 0.0
    assert abs(L.orc_profile(0.05, 5, 5, 11, 11) - 0.05) < 1e-7


def test_inverse_mrt_port_is_reference_and_exact_transpose():
    L = O.oracle_lib()
    M = np.zeros((19, 19), np.float32)
    L.orc_tables(None, None, None, O._p(M))
    inv = np.zeros((19, 19), np.float32)
    assert L.orc_inverse_mrt(O._p(M), O._p(inv)) == 0
    n2 = (M.astype(np.float64) ** 2).sum(axis=1)
    exact = M.T.astype(np.float64) / n2[None, :]
    assert np.abs(inv - exact).max() < 1e-6
    R = O.poplar_ref_lib()
    if R is not None:
        inv_ref = np.zeros((19, 19), np.float32)
        R.ref_inverse_mrt(O._p(M), O._p(inv_ref))
        np.testing.assert_array_equal(inv, inv_ref)


@pytest.mark.parametrize("path", golden_files("kernelcu"), ids=os.path.basename)
def test_port_matches_kernelcu_golden(path):
    """SRT (and SRT + LES) exist only in the reference's kernel.cu; these
    fixtures were produced by that code itself on a B200
    (tests/golden/make_golden.py --kernelcu).  The port differs from it only
    by rounding (FP64 literals and FMA contraction on the GPU)."""
    g = np.load(path)
    iv = iv_from_golden(g)
    r = O.Run(iv, init_kind=int(g["init_kind"]), seed=int(g["seed"]), amp=float(g["noise_amp"]))
    r.step(int(g["steps"]))
    f = r.fields()
    assert O.rel_field_err(f["den"], g["den"]) <= 1e-5
    assert O.rel_vel_err((f["ux"], f["uy"], f["uz"]), (g["ux"], g["uy"], g["uz"])) <= 1e-5
