"""AA-pattern streaming (one lattice, in place) against the pull (A/B) form
and the oracle, for cavities and channels (inlet / outlet rules applied when
the natural layout is read).

The AA steps evaluate the same node arithmetic on the same populations.  The
first step after the initial state gives the same bits as the pull form;
later steps differ by FP32 rounding (the two kernels may fuse a
multiply-add differently; ~1e-7 after a few steps, ~1e-6 after a hundred), so
they are compared at the 1e-5 parity tolerance, which both also meet against
the oracle.  The 16-bit
forms also round the lid's bounce-back value at a different point and are
compared within the 16-bit tolerance."""
import numpy as np
import pytest

import oracle_lib as O

pkg = O.pkg
pytestmark = pytest.mark.gpu
CLOSE = 1e-5


def cavity(nx, ny, nz, re=400.0, mrt=True, les=True):
    return pkg.make_inputval(nx, ny, nz, casetype=pkg.CAVITY, re=re, u=0.1, mrt=mrt, les=les,
                             cs=0.1, h=nx)


def channel(nx, ny, nz, tau=0.56, mrt=True, les=True):
    return pkg.make_inputval(nx, ny, nz, casetype=pkg.CHANNEL, tau=tau, u=0.05, mrt=mrt, les=les,
                             cs=0.1)


def pair(iv, storage=pkg.STORE_F32):
    if iv.casetype == pkg.CHANNEL:
        o = dict(storage=storage, init_kind=pkg.INIT_CHANNEL, noise_amp=0.01)
    else:
        o = dict(storage=storage, init_kind=pkg.INIT_DENSITY_NOISE, noise_amp=1e-6)
    return (pkg.Domain(iv, pkg.default_options(stream_mode=pkg.STREAM_AA, **o)),
            pkg.Domain(iv, pkg.default_options(stream_mode=pkg.STREAM_AB, **o)))


@pytest.mark.parametrize("case", ["cavity", "channel"])
@pytest.mark.parametrize("mrt,les", [(True, True), (False, False), (True, False)])
def test_aa_matches_pull(case, mrt, les):
    iv = cavity(34, 21, 19, mrt=mrt, les=les) if case == "cavity" else \
        channel(34, 13, 15, mrt=mrt, les=les)
    aa, ab = pair(iv)
    np.testing.assert_array_equal(aa.export_arF(), ab.export_arF())  # initial state
    aa.run(1)
    ab.run(1)
    np.testing.assert_array_equal(aa.export_arF(), ab.export_arF())  # first step: same bits
    for steps in (1, 2, 37, 70, 3):  # odd and even totals; 70 uses graph chunks
        aa.run(steps)
        ab.run(steps)
        assert aa.steps() == ab.steps()
        assert O.rel_field_err(aa.export_arF(), ab.export_arF()) <= CLOSE
        pa, pb = aa.export_arF(padded=True), ab.export_arF(padded=True)
        assert O.rel_field_err(pa, pb) <= CLOSE
        assert not pa[0].any() and not pa[:, 0].any()  # ghost layer
        den_a, *u_a = aa.macroscopic()
        den_b, *u_b = ab.macroscopic()
        assert O.rel_field_err(den_a, den_b) <= CLOSE
        assert O.rel_vel_err(u_a, u_b) <= CLOSE
        da, db = aa.diagnostics(), ab.diagnostics()
        assert abs(da[0] - db[0]) <= 1e-6 * abs(db[0])  # mass
        assert da[7] == db[7] == 0


@pytest.mark.parametrize("case", ["cavity", "channel"])
def test_aa_import_and_checkpoint_continue(tmp_path, case):
    mk = (lambda: cavity(24, 20, 22)) if case == "cavity" else (lambda: channel(30, 12, 14))
    aa, ab = pair(mk())
    ab.run(41)
    arF = ab.export_arF(padded=True)
    aa.import_arF(arF, padded=True)
    np.testing.assert_array_equal(aa.export_arF(padded=True), arF)  # complete layout
    ab2 = pkg.Domain(mk())
    ab2.import_arF(arF, padded=True)
    for steps in (1, 1, 65):  # from the complete layout, then pending / swapped
        aa.run(steps)
        ab2.run(steps)
        assert O.rel_field_err(aa.export_arF(), ab2.export_arF()) <= CLOSE
        den_a, *u_a = aa.macroscopic()
        den_b, *u_b = ab2.macroscopic()
        assert O.rel_field_err(den_a, den_b) <= CLOSE
        assert O.rel_vel_err(u_a, u_b) <= CLOSE
    aa.save_checkpoint(tmp_path / "aa.bin")  # odd step count: swapped layout
    c = pkg.Domain(mk(), pkg.default_options(stream_mode=pkg.STREAM_AA))
    c.load_checkpoint(tmp_path / "aa.bin")
    c.run(10)
    aa.run(10)
    # the restart begins with a local step where the continued run takes a
    # neighbour step: the same arithmetic in another kernel, rounding apart
    assert O.rel_field_err(c.export_arF(), aa.export_arF()) <= CLOSE


@pytest.mark.parametrize("case", ["cavity", "channel"])
@pytest.mark.parametrize("storage", [pkg.STORE_F16_SHIFT, pkg.STORE_BF16_SHIFT])
def test_aa_16bit_close_to_pull(storage, case):
    aa, ab = pair(cavity(40, 32, 28) if case == "cavity" else channel(48, 16, 18), storage)
    aa.run(150)
    ab.run(150)
    ua = np.stack(aa.macroscopic()[1:])
    ub = np.stack(ab.macroscopic()[1:])
    tol = 1e-3 if storage == pkg.STORE_F16_SHIFT else 1e-2
    assert np.abs(ua - ub).max() / np.abs(ub).max() <= tol


@pytest.mark.parametrize("case,steps", [("cavity", 101), ("channel", 250), ("channel", 251)])
def test_aa_vs_oracle(case, steps):
    if case == "cavity":
        iv, kind, amp = cavity(30, 26, 22), 1, 1e-6
    else:
        iv, kind, amp = channel(40, 14, 18, tau=0.6), pkg.INIT_CHANNEL, 0.01
    aa = pkg.Domain(iv, pkg.default_options(stream_mode=pkg.STREAM_AA, init_kind=kind,
                                            noise_amp=amp))
    ref = O.Run(iv, init_kind=kind, amp=amp)
    aa.run(steps)
    ref.step(steps)
    r = ref.fields()
    den, ux, uy, uz = aa.macroscopic()
    assert O.rel_field_err(den, r["den"]) <= 1e-5
    assert O.rel_vel_err((ux, uy, uz), (r["ux"], r["uy"], r["uz"])) <= 1e-5


def test_aa_halves_the_lattice_memory_and_rejects_struct_geometries():
    iv = cavity(64, 64, 64)
    aa, ab = pair(iv)
    lat = 19 * 64 * 64 * 64 * 4
    assert ab.device_bytes() - aa.device_bytes() >= lat
    pipe = pkg.make_inputval(32, 16, 16, casetype=pkg.POISEUILLE, tau=0.6, u=0.05)
    with pytest.raises(pkg.LbmError):
        pkg.Domain(pipe, pkg.default_options(stream_mode=pkg.STREAM_AA))
    with pytest.raises(pkg.LbmError):
        aa.set_solid_mask(np.ones((64, 64, 64), bool))

