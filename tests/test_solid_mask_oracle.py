"""Solid voxel masks in the oracle (CPU): the STRUCT rules of the reference
(keStreaming skips STRUCT donors, keBoundaryStruct half-way bounce-back for
FLUID nodes, kernel.cu:489-516, 659-697) on arbitrary obstacles."""
import numpy as np

import oracle_lib as O

pkg = O.pkg


def sphere(nx, ny, nz, cx, cy, cz, r):
    y, z, x = np.meshgrid(np.arange(ny), np.arange(nz), np.arange(nx), indexing="ij")
    return ((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2) <= r * r


def test_mask_nodes_are_struct_and_stay_zero():
    iv = pkg.make_inputval(14, 12, 10, casetype=pkg.CAVITY, re=100.0, u=0.1, mrt=True, les=True,
                           cs=0.1, h=14)
    r = O.Run(iv, init_kind=1, amp=1e-6)
    m = sphere(14, 12, 10, 7, 5, 5, 2.5)
    r.set_solid(m)
    r.step(30)
    f = r.fields()
    assert (f["ntype"][m] == pkg.NODE_STRUCT).all()
    assert not f["arF"][m].any()
    assert np.isfinite(f["arF"]).all()
    # no population of a fluid node facing the obstacle is left at zero
    fl = f["ntype"] == pkg.NODE_FLUID
    assert (f["arF"][fl] > 0).all()


def test_empty_mask_is_the_plain_case():
    iv = pkg.make_inputval(12, 10, 9, casetype=pkg.CAVITY, re=100.0, u=0.1, mrt=True, les=True,
                           cs=0.1, h=12)
    a = O.Run(iv, init_kind=1, amp=1e-6)
    b = O.Run(iv, init_kind=1, amp=1e-6)
    b.set_solid(np.zeros((10, 9, 12), bool))
    a.step(20)
    b.step(20)
    np.testing.assert_array_equal(a.fields()["arF"], b.fields()["arF"])


def test_mask_on_the_pipe_adds_to_the_pipe_wall():
    iv = pkg.make_inputval(20, 50, 50, casetype=pkg.POISEUILLE, tau=0.8, u=0.02)
    r = O.Run(iv, init_kind=1, amp=1e-6)
    m = sphere(20, 50, 50, 10, 25, 25, 4)
    r.set_solid(m)
    t = r.fields()["ntype"]
    y, z = np.meshgrid(np.arange(50), np.arange(50), indexing="ij")
    pipe_wall = ((y - 25) ** 2 + (z - 25) ** 2 > 400)[:, :, None]
    assert ((t == pkg.NODE_STRUCT) == (m | np.broadcast_to(pipe_wall, m.shape))).all()
