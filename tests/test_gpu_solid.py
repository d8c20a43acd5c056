"""Solid voxel masks (lbm_set_solid_mask) on the GPU against the oracle and,
in the POISEUILLE case where the reference runs keBoundaryStruct, against
the reference's kernel.cu itself."""
import numpy as np
import pytest

import oracle_lib as O
from test_solid_mask_oracle import sphere

pkg = O.pkg
pytestmark = pytest.mark.gpu
TOL = 1e-5


def compare(d, r):
    den, ux, uy, uz = d.macroscopic()
    assert O.rel_field_err(den, r["den"]) <= TOL
    assert O.rel_vel_err((ux, uy, uz), (r["ux"], r["uy"], r["uz"])) <= TOL
    assert O.rel_field_err(d.export_arF(), r["arF"]) <= TOL


@pytest.mark.parametrize("mrt,les", [(True, True), (False, False)])
def test_cavity_with_obstacle_vs_oracle(mrt, les):
    nx, ny, nz = 30, 26, 22
    iv = pkg.make_inputval(nx, ny, nz, casetype=pkg.CAVITY, re=200.0, u=0.1, mrt=mrt, les=les,
                           cs=0.1, h=nx)
    m = sphere(nx, ny, nz, 14, 13, 10, 5.5)
    m[20:24, 3:9, 2:6] = True  # a box touching nothing else
    m[0:3, 10:14, 0:4] = True  # a block merged into two walls
    o = pkg.default_options(init_kind=pkg.INIT_DENSITY_NOISE, noise_amp=1e-6)
    d = pkg.Domain(iv, o)
    d.set_solid_mask(m)
    ref = O.Run(iv, init_kind=1, amp=1e-6)
    ref.set_solid(m)
    t, _ = d.node_info()
    np.testing.assert_array_equal(t, ref.fields()["ntype"])
    for steps in (1, 80):
        d.run(steps)
        ref.step(steps)
        r = ref.fields()
        compare(d, r)
        assert not d.export_arF()[m].any()


def test_channel_with_cylinder_vs_oracle():
    nx, ny, nz = 64, 24, 20
    iv = pkg.make_inputval(nx, ny, nz, casetype=pkg.CHANNEL, tau=0.6, u=0.05, mrt=True, les=True,
                           cs=0.1)
    y, z, x = np.meshgrid(np.arange(ny), np.arange(nz), np.arange(nx), indexing="ij")
    m = (x - 20) ** 2 + (y - 12) ** 2 <= 16
    o = pkg.default_options(init_kind=pkg.INIT_CHANNEL, noise_amp=0.01)
    d = pkg.Domain(iv, o)
    d.set_solid_mask(m)
    ref = O.Run(iv, init_kind=pkg.INIT_CHANNEL, amp=0.01)
    ref.set_solid(m)
    d.run(100)
    ref.step(100)
    compare(d, ref.fields())


@pytest.mark.skipif(O.kernelcu_ref_lib() is None, reason="reference kernel.cu not built")
def test_pipe_with_obstacle_vs_reference_kernelcu():
    nx, ny, nz = 26, 50, 50
    iv = pkg.make_inputval(nx, ny, nz, casetype=pkg.POISEUILLE, tau=0.7, u=0.03)
    m = sphere(nx, ny, nz, 12, 25, 25, 6)
    k = O.kernelcu_run(iv, 60, init_kind=1, amp=1e-6, solid=m)
    d = pkg.Domain(iv, pkg.default_options(init_kind=pkg.INIT_DENSITY_NOISE, noise_amp=1e-6))
    d.set_solid_mask(m)
    d.run(60)
    den, ux, uy, uz = d.macroscopic()
    assert O.rel_field_err(den, k["den"]) <= TOL
    assert O.rel_vel_err((ux, uy, uz), (k["ux"], k["uy"], k["uz"])) <= TOL
    ref = O.Run(iv, init_kind=1, amp=1e-6)
    ref.set_solid(m)
    ref.step(60)
    compare(d, ref.fields())


def test_removing_the_mask_restores_the_plain_case():
    iv = pkg.make_inputval(20, 18, 16, casetype=pkg.CAVITY, re=100.0, u=0.1, mrt=True, les=True,
                           cs=0.1, h=20)
    o = pkg.default_options(init_kind=pkg.INIT_DENSITY_NOISE, noise_amp=1e-6)
    a = pkg.Domain(iv, o)
    a.set_solid_mask(sphere(20, 18, 16, 10, 9, 8, 3))
    a.run(10)
    a.set_solid_mask(None)
    a.run(25)
    b = pkg.Domain(iv, o)
    b.run(25)
    np.testing.assert_array_equal(a.export_arF(), b.export_arF())


@pytest.mark.parametrize("storage", [pkg.STORE_F16_SHIFT, pkg.STORE_BF16_SHIFT])
def test_mask_with_16bit_storage_close_to_fp64(storage):
    iv = pkg.make_inputval(32, 28, 24, casetype=pkg.CAVITY, re=300.0, u=0.1, mrt=True, les=True,
                           cs=0.1, h=32)
    m = sphere(32, 28, 24, 16, 14, 12, 6)
    lo = pkg.Domain(iv, pkg.default_options(storage=storage))
    hi = pkg.Domain(iv, pkg.default_options(storage=pkg.STORE_F64, kernel=pkg.KERNEL_SCALAR))
    for d in (lo, hi):
        d.set_solid_mask(m)
        d.run(200)
    ul = np.stack(lo.macroscopic()[1:])
    uh = np.stack(hi.macroscopic()[1:])
    assert np.abs(ul - uh).max() / np.abs(uh).max() <= (1e-3 if storage == pkg.STORE_F16_SHIFT
                                                       else 3e-2)


def test_batch_members_take_no_mask():
    iv = pkg.make_inputval(16, casetype=pkg.CAVITY, tau=0.6, u=0.1)
    b = pkg.Batch(hbm_budget=64 << 20)
    i = b.add(iv, None, 4)
    with pytest.raises(pkg.LbmError):
        b.member(i).set_solid_mask(np.zeros((16, 16, 16), bool))
    b.close()
