"""The TMA-staged step kernel (LBM_KERNEL_TMA) against the oracle.

Same tolerance as the other FP32 paths (1e-5 on rho and on u relative to
max |u|); the 16-bit formats against the FP64 build.  The tiles are
128 x 4 nodes, so the shapes below include partial tiles in x and z and
tiles that touch every face.
"""
import numpy as np
import pytest

import oracle_lib as O

pkg = O.pkg
pytestmark = pytest.mark.gpu
TOL = 1e-5


def run(iv, steps, storage=pkg.STORE_F32, kernel=pkg.KERNEL_TMA, kind=1, amp=1e-6):
    d = pkg.Domain(iv, pkg.default_options(storage=storage, kernel=kernel, init_kind=kind,
                                           noise_amp=amp))
    d.run(steps)
    return d


@pytest.mark.parametrize("shape", [(48, 20, 18), (130, 9, 11), (256, 24, 7), (131, 10, 9),
                                   (5, 6, 7), (3, 4, 5)])
@pytest.mark.parametrize("mrt,les", [(True, True), (False, False)])
def test_tma_cavity_vs_oracle(shape, mrt, les):
    # the tiny boxes (every node on a face) run at a lower Re: at tau ~ 0.5045
    # SRT rounding differences of 1 ulp grow past the tolerance in 120 steps
    re = 200.0 if min(shape) >= 7 else 20.0
    iv = pkg.make_inputval(*shape, casetype=pkg.CAVITY, re=re, u=0.1, mrt=mrt, les=les, cs=0.1,
                           h=shape[0])
    d = run(iv, 120)
    ref = O.Run(iv, init_kind=1, amp=1e-6)
    ref.step(120)
    r = ref.fields()
    den, ux, uy, uz = d.macroscopic()
    assert O.rel_field_err(den, r["den"]) <= TOL
    assert O.rel_vel_err((ux, uy, uz), (r["ux"], r["uy"], r["uz"])) <= TOL
    assert O.rel_field_err(d.export_arF(), r["arF"]) <= TOL
    d.sync()


def test_tma_channel_vs_oracle():
    iv = pkg.make_inputval(140, 14, 18, casetype=pkg.CHANNEL, tau=0.6, u=0.05, mrt=True, les=True,
                           cs=0.1)
    d = run(iv, 150, kind=pkg.INIT_CHANNEL, amp=0.01)
    ref = O.Run(iv, init_kind=pkg.INIT_CHANNEL, amp=0.01)
    ref.step(150)
    r = ref.fields()
    den, ux, uy, uz = d.macroscopic()
    assert O.rel_field_err(den, r["den"]) <= TOL
    assert O.rel_vel_err((ux, uy, uz), (r["ux"], r["uy"], r["uz"])) <= TOL


@pytest.mark.parametrize("storage,tol", [(pkg.STORE_F16_SHIFT, 1e-3), (pkg.STORE_BF16_SHIFT, 3e-2)])
def test_tma_16bit_vs_fp64(storage, tol):
    iv = pkg.make_inputval(64, 40, 36, casetype=pkg.CAVITY, re=400.0, u=0.1, mrt=True, les=True,
                           cs=0.1, h=64)
    lo = run(iv, 300, storage=storage)
    hi = run(iv, 300, storage=pkg.STORE_F64, kernel=pkg.KERNEL_SCALAR)
    ul = np.stack(lo.macroscopic()[1:])
    uh = np.stack(hi.macroscopic()[1:])
    assert np.abs(ul - uh).max() / np.abs(uh).max() <= tol


def test_tma_matches_scalar_kernel_closely():
    iv = pkg.make_inputval(128, 64, 64, casetype=pkg.CAVITY, re=1000.0, u=0.1, mrt=True, les=True,
                           cs=0.1, h=128)
    a = run(iv, 200)
    b = run(iv, 200, kernel=pkg.KERNEL_SCALAR)
    fa, fb = a.export_arF(), b.export_arF()
    assert O.rel_field_err(fa, fb) <= 1e-6


def test_bounded_wait_gives_up_with_timeout_and_the_device_stays_usable():
    """The failure path of the TMA kernel's bounded mbarrier waits: with
    wait_test the producer withholds the copies of one tile (a barrier that
    nothing completes) and the waits give up after ~1 ms; the step reports
    LBM_ERR_TIMEOUT at the next synchronising call instead of hanging, and a
    fresh domain on the same device then steps normally."""
    iv = pkg.make_inputval(64, 32, 32, casetype=pkg.CAVITY, re=100.0, u=0.1, mrt=True, les=True,
                           cs=0.1, h=64)
    d = pkg.Domain(iv, pkg.default_options(kernel=pkg.KERNEL_TMA, wait_test=3))
    d.run(1)
    with pytest.raises(pkg.LbmError) as e:
        d.sync()
    assert e.value.code == pkg.LBM_ERR_TIMEOUT
    d.close()
    good = pkg.Domain(iv, pkg.default_options(kernel=pkg.KERNEL_TMA))
    good.run(5)
    good.sync()
    plain = pkg.Domain(iv, pkg.default_options(kernel=pkg.KERNEL_SCALAR))
    plain.run(5)
    a, b = good.macroscopic(), plain.macroscopic()
    good.close()
    plain.close()
    assert O.rel_field_err(a[0], b[0]) <= 1e-6
    with pytest.raises(pkg.LbmError) as e:
        pkg.Domain(iv, pkg.default_options(kernel=pkg.KERNEL_SCALAR, wait_test=1))
    assert e.value.code == pkg.LBM_ERR_INVALID
