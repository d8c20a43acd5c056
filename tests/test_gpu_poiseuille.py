"""The POISEUILLE case of kernel.cu (kernel.cu:1078-1094): inlet x=0,
outlet x=nx-1, STRUCT outside the circle of radius 20 about (y,z)=(25,25),
half-way bounce-back next to STRUCT (keBoundaryStruct), donors that are
STRUCT never stream, and populations that no rule writes keep their initial
value.  Against the oracle port and the reference's own kernel.cu."""
import numpy as np
import pytest

import oracle_lib as O

pkg = O.pkg
pytestmark = pytest.mark.gpu
TOL = 1e-5


def pipe(nx, ny, nz, mrt=False, les=False, u=0.02, tau=0.8):
    return pkg.make_inputval(nx, ny, nz, casetype=pkg.POISEUILLE, tau=tau, u=u, mrt=mrt, les=les,
                             cs=0.1)


def errs(d, r):
    den, ux, uy, uz = d.macroscopic()
    return (O.rel_field_err(den, r["den"]),
            O.rel_vel_err((ux, uy, uz), (r["ux"], r["uy"], r["uz"])))


@pytest.mark.parametrize("shape", [(30, 52, 52), (24, 30, 34)], ids=["full", "cut"])
@pytest.mark.parametrize("mrt,les", [(False, False), (True, True)])
def test_poiseuille_vs_oracle(shape, mrt, les):
    iv = pipe(*shape, mrt=mrt, les=les)
    d = pkg.Domain(iv, pkg.default_options(init_kind=pkg.INIT_DENSITY_NOISE, noise_amp=1e-6))
    ref = O.Run(iv, init_kind=1, amp=1e-6)
    for steps in (1, 60):
        d.run(steps)
        ref.step(steps)
        r = ref.fields()
        e_den, e_u = errs(d, r)
        assert e_den <= TOL and e_u <= TOL, (steps, e_den, e_u)
        f = d.export_arF()
        assert O.rel_field_err(f, r["arF"]) <= TOL
        struct = r["ntype"] == pkg.NODE_STRUCT
        assert struct.any()
        assert not f[struct].any()  # STRUCT nodes stay at zero


def test_poiseuille_node_info_and_batch_member():
    iv = pipe(20, 50, 50)
    o = pkg.default_options(init_kind=pkg.INIT_DENSITY_NOISE, noise_amp=1e-6)
    d = pkg.Domain(iv, o)
    t, s = d.node_info()
    r = O.Run(iv).fields()
    np.testing.assert_array_equal(t, r["ntype"])
    np.testing.assert_array_equal(s, r["dstate"])
    d.run(25)
    alone = d.export_arF()
    b = pkg.Batch(hbm_budget=256 << 20, chunk_steps=8)
    i = b.add(iv, o, 25)
    b.step(25)
    b.sync()
    np.testing.assert_array_equal(b.member(i).export_arF(), alone)
    b.close()


@pytest.mark.skipif(O.kernelcu_ref_lib() is None, reason="reference kernel.cu not built")
def test_poiseuille_vs_reference_kernelcu():
    iv = pipe(26, 50, 50, u=0.03, tau=0.7)
    k = O.kernelcu_run(iv, 80, init_kind=1, amp=1e-6)
    ref = O.Run(iv, init_kind=1, amp=1e-6)
    ref.step(80)
    r = ref.fields()
    assert O.rel_field_err(r["den"], k["den"]) <= TOL
    assert O.rel_vel_err((r["ux"], r["uy"], r["uz"]), (k["ux"], k["uy"], k["uz"])) <= TOL
    d = pkg.Domain(iv, pkg.default_options(init_kind=pkg.INIT_DENSITY_NOISE, noise_amp=1e-6))
    d.run(80)
    e_den, e_u = errs(d, k)
    assert e_den <= TOL and e_u <= TOL
