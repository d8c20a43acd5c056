"""Paired rows (LBM_KERNEL_PAIRED, the default of the 16-bit pull form).

The paired layout stores word w of every row as the node pair (w, w + px/2)
and steps two nodes per thread with packed FP32 arithmetic; the per-node
kernel steps the plain layout one node per thread.  Both run the same node
arithmetic without multiply-add contraction, so a domain must give the same
bits either way: after any number of steps the exported arF (which undoes
the layout) and the macroscopic fields are compared for equality, over
shapes that exercise the seam between the two halves, rows whose pitch is
padded (nx not a multiple of 8), tiny rows with no main words, both
collision models, the channel's inlet/outlet rules, the POISEUILLE struct
geometry and solid masks, imports, checkpoints and the batch.
"""
import numpy as np
import pytest

import oracle_lib as O

pkg = O.pkg
pytestmark = pytest.mark.gpu

STORES = [pkg.STORE_F16_SHIFT, pkg.STORE_BF16_SHIFT]


def cavity(nx, ny, nz, mrt=True, les=True, re=300.0):
    return pkg.make_inputval(nx, ny, nz, casetype=pkg.CAVITY, re=re, u=0.1, mrt=mrt, les=les,
                             cs=0.1 if les else 0.0, h=nx)


def channel(nx, ny, nz, mrt=True, les=True):
    return pkg.make_inputval(nx, ny, nz, casetype=pkg.CHANNEL, tau=0.56, u=0.05, mrt=mrt, les=les,
                             cs=0.1 if les else 0.0)


def opts(storage, kernel, kind=pkg.INIT_DENSITY_NOISE, amp=1e-4):
    return pkg.default_options(storage=storage, kernel=kernel, init_kind=kind, noise_amp=amp,
                               seed=7)


def both(iv, storage, steps, kind=pkg.INIT_DENSITY_NOISE, amp=1e-4, mask=None):
    out = []
    for kern in (pkg.KERNEL_PAIRED, pkg.KERNEL_SCALAR):
        d = pkg.Domain(iv, opts(storage, kern, kind, amp))
        if mask is not None:
            d.set_solid_mask(mask)
        d.run(steps)
        out.append((d.export_arF(), d.macroscopic()))
        d.close()
    return out


def assert_same(a, b):
    np.testing.assert_array_equal(a[0], b[0])
    for x, y in zip(a[1], b[1]):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("storage", STORES)
@pytest.mark.parametrize("shape", [(64, 20, 18), (256, 6, 5), (130, 9, 11), (131, 10, 7),
                                   (9, 8, 7), (5, 6, 7), (3, 4, 5), (17, 16, 3)])
@pytest.mark.parametrize("steps", [1, 2, 37])
def test_paired_equals_per_node_cavity(storage, shape, steps):
    a, b = both(cavity(*shape), storage, steps)
    assert_same(a, b)
    assert np.isfinite(a[0]).all()


@pytest.mark.parametrize("storage", STORES)
@pytest.mark.parametrize("mrt,les", [(True, True), (False, False), (False, True), (True, False)])
def test_paired_equals_per_node_models(storage, mrt, les):
    a, b = both(cavity(48, 14, 12, mrt=mrt, les=les), storage, 70)
    assert_same(a, b)


@pytest.mark.parametrize("storage", STORES)
@pytest.mark.parametrize("shape", [(48, 12, 14), (41, 9, 10)])
def test_paired_equals_per_node_channel(storage, shape):
    a, b = both(channel(*shape), storage, 66, kind=pkg.INIT_CHANNEL, amp=0.01)
    assert_same(a, b)


@pytest.mark.parametrize("storage", STORES)
def test_paired_equals_per_node_poiseuille_and_mask(storage):
    iv = pkg.make_inputval(24, 52, 52, casetype=pkg.POISEUILLE, tau=0.7, u=0.02)
    a, b = both(iv, storage, 20, kind=pkg.INIT_REFERENCE, amp=0.0)
    assert_same(a, b)
    iv = cavity(40, 16, 18)
    mask = np.zeros((16, 18, 40), np.uint8)
    mask[5:10, 6:12, 15:22] = 1
    a, b = both(iv, storage, 30, mask=mask)
    assert_same(a, b)


@pytest.mark.parametrize("storage", STORES)
def test_paired_import_export_and_checkpoint(storage, tmp_path):
    """Import, export and a checkpoint round trip give the same bits with
    either layout.  The AoS FP32 round trip itself is not exact for 16-bit
    storage (g -> w + g -> g loses the bits of g below the FP32 ulp of w),
    so a continuation after a checkpoint load is compared with never
    stopping to within the storage quantum, not bit for bit."""
    iv = cavity(34, 12, 10)
    src = pkg.Domain(iv, opts(pkg.STORE_F32, pkg.KERNEL_SCALAR))
    src.run(9)
    arF = src.export_arF(padded=True)
    src.close()
    res = []
    for kern in (pkg.KERNEL_PAIRED, pkg.KERNEL_SCALAR):
        d = pkg.Domain(iv, opts(storage, kern))
        d.import_arF(arF, padded=True)
        first = d.export_arF(padded=True)
        path = str(tmp_path / f"k{kern}.ckpt")
        d.run(5)
        d.save_checkpoint(path)
        d.run(6)
        a1 = d.export_arF()
        d.load_checkpoint(path)
        d.run(6)
        a2 = d.export_arF()
        d.close()
        res.append((first, a1, a2))
    for x, y in zip(*res):
        np.testing.assert_array_equal(x, y)
    # the import holds arF to within the storage quantum
    tol = 2e-5 if storage == pkg.STORE_F16_SHIFT else 2e-4
    assert np.abs(res[0][0] - arF).max() <= tol
    assert np.abs(res[0][1] - res[0][2]).max() <= 2 * tol


def test_paired_is_the_16bit_default_and_batch_members_match_it():
    iv = cavity(40, 18, 16)
    o_auto = opts(pkg.STORE_F16_SHIFT, pkg.KERNEL_AUTO)
    d = pkg.Domain(iv, o_auto)
    d.run(40)
    want = d.export_arF()
    d.close()
    b = pkg.Batch(hbm_budget=256 << 20, chunk_steps=8)
    i = b.add(iv, o_auto, 40)
    b.step(40)
    b.sync()
    np.testing.assert_array_equal(b.member(i).export_arF(), want)
    b.close()


def test_paired_option_rejected_where_it_does_not_apply():
    iv = cavity(16, 12, 10)
    for o in (pkg.default_options(storage=pkg.STORE_F32, kernel=pkg.KERNEL_PAIRED),
              pkg.default_options(storage=pkg.STORE_F16_SHIFT, kernel=pkg.KERNEL_PAIRED,
                                  stream_mode=pkg.STREAM_AA)):
        with pytest.raises(pkg.LbmError) as e:
            pkg.Domain(iv, o)
        assert e.value.code == pkg.LBM_ERR_INVALID


# ---------------------------------------------------------------------------
# Stochastic rounding (LBM_ROUND_STOCHASTIC): the random bits of a store
# depend on the node's pair word, the step and the seed only, and cvt.rs
# rounds each element of a 16x2 conversion with its own bits, so the paired
# kernel (both elements real) and the per-node kernel over plain rows (the
# other element 0) give the same bits.
# ---------------------------------------------------------------------------
def sr_opts(storage, kernel, kind=pkg.INIT_DENSITY_NOISE, amp=1e-4, seed=7):
    return pkg.default_options(storage=storage, kernel=kernel, init_kind=kind, noise_amp=amp,
                               seed=seed, rounding=pkg.ROUND_STOCHASTIC)


def run_arF(iv, o, steps, mask=None):
    d = pkg.Domain(iv, o)
    if mask is not None:
        d.set_solid_mask(mask)
    d.run(steps)
    out = (d.export_arF(), d.macroscopic())
    d.close()
    return out


@pytest.mark.parametrize("storage", STORES)
@pytest.mark.parametrize("shape", [(64, 20, 18), (130, 9, 11), (17, 16, 3), (9, 8, 7)])
def test_stochastic_rounding_same_bits_paired_and_per_node(storage, shape):
    iv = cavity(*shape)
    a = run_arF(iv, sr_opts(storage, pkg.KERNEL_PAIRED), 70)
    b = run_arF(iv, sr_opts(storage, pkg.KERNEL_SCALAR), 70)
    assert_same(a, b)


@pytest.mark.parametrize("storage", STORES)
def test_stochastic_rounding_channel_and_mask(storage):
    iv = channel(48, 12, 14)
    a = run_arF(iv, sr_opts(storage, pkg.KERNEL_PAIRED, pkg.INIT_CHANNEL, 0.01), 66)
    b = run_arF(iv, sr_opts(storage, pkg.KERNEL_SCALAR, pkg.INIT_CHANNEL, 0.01), 66)
    assert_same(a, b)
    iv = cavity(40, 16, 18)
    mask = np.zeros((16, 18, 40), np.uint8)
    mask[5:10, 6:12, 15:22] = 1
    a = run_arF(iv, sr_opts(storage, pkg.KERNEL_PAIRED), 30, mask)
    b = run_arF(iv, sr_opts(storage, pkg.KERNEL_SCALAR), 30, mask)
    assert_same(a, b)


def test_stochastic_rounding_is_reproducible_and_seeded():
    iv = cavity(48, 14, 12)
    st = pkg.STORE_F16_SHIFT
    a = run_arF(iv, sr_opts(st, pkg.KERNEL_AUTO), 70)   # graph chunks + single steps
    b = run_arF(iv, sr_opts(st, pkg.KERNEL_AUTO), 70)
    assert_same(a, b)
    c = run_arF(iv, sr_opts(st, pkg.KERNEL_AUTO, seed=8), 70)
    n = run_arF(iv, opts(st, pkg.KERNEL_AUTO), 70)
    assert not np.array_equal(a[0], c[0]) and not np.array_equal(a[0], n[0])
    # the same physics: every variant within a few storage quanta of the others
    assert np.abs(a[0] - n[0]).max() < 2e-4
    # 70 steps in one call equal 33 + 37 steps (the step counter carries over)
    d = pkg.Domain(iv, sr_opts(st, pkg.KERNEL_AUTO))
    d.run(33)
    d.run(37)
    np.testing.assert_array_equal(d.export_arF(), a[0])
    d.close()


def test_stochastic_rounding_rejected_where_not_built():
    iv = cavity(16, 12, 10)
    for o in (pkg.default_options(storage=pkg.STORE_F32, rounding=pkg.ROUND_STOCHASTIC),
              # AA on plain rows (the per-node AA step has no stochastic rounding)
              pkg.default_options(storage=pkg.STORE_F16_SHIFT, rounding=pkg.ROUND_STOCHASTIC,
                                  stream_mode=pkg.STREAM_AA, kernel=pkg.KERNEL_SCALAR),
              pkg.default_options(storage=pkg.STORE_F16_SHIFT, rounding=pkg.ROUND_STOCHASTIC,
                                  kernel=pkg.KERNEL_TMA),
              pkg.default_options(storage=pkg.STORE_F16_SHIFT, rounding=5)):
        with pytest.raises(pkg.LbmError) as e:
            pkg.Domain(iv, o)
        assert e.value.code == pkg.LBM_ERR_INVALID
    # AA rows that are not quad rows (nx not a multiple of 8)
    with pytest.raises(pkg.LbmError):
        pkg.Domain(cavity(20, 12, 10),
                   pkg.default_options(storage=pkg.STORE_F16_SHIFT, rounding=pkg.ROUND_STOCHASTIC,
                                       stream_mode=pkg.STREAM_AA))
    b = pkg.Batch(hbm_budget=64 << 20)
    with pytest.raises(pkg.LbmError):
        b.add(iv, pkg.default_options(storage=pkg.STORE_F16_SHIFT,
                                      rounding=pkg.ROUND_STOCHASTIC), 4)
    b.close()


@pytest.mark.parametrize("storage", STORES)
@pytest.mark.parametrize("shape", [(0, 0, 256, 2), (1, 1, 128, 1), (0, 1, 128, 16),
                                   (1, 0, 256, 3), (2, 0, 128, 2)])
def test_batch_members_in_paired_rows_match_alone(storage, shape):
    """16-bit A/B batch members keep the paired rows (the batched kernel
    steps their words), except where the paired step does not apply (tiny
    rows: plain rows); a mix of both, of both collision models and of the
    channel, against each domain alone, over warp tiles that wrap rows."""
    sched, regs, block, npt = shape
    cases = [(cavity(64, 20, 18), pkg.INIT_DENSITY_NOISE, 1e-4),
             (cavity(9, 8, 7), pkg.INIT_DENSITY_NOISE, 1e-4),
             (cavity(130, 9, 11, mrt=False, les=False), pkg.INIT_DENSITY_NOISE, 1e-4),
             (channel(48, 12, 14), pkg.INIT_CHANNEL, 0.01),
             (cavity(41, 10, 7, mrt=True, les=False), pkg.INIT_DENSITY_NOISE, 1e-4)]
    kerns = [pkg.KERNEL_AUTO, pkg.KERNEL_AUTO, pkg.KERNEL_PAIRED, pkg.KERNEL_AUTO,
             pkg.KERNEL_SCALAR]
    want = []
    for (iv, kind, amp), k in zip(cases, kerns):
        d = pkg.Domain(iv, opts(storage, k, kind, amp))
        d.run(45)
        want.append((d.export_arF(), d.macroscopic()))
        d.close()
    b = pkg.Batch(hbm_budget=256 << 20, chunk_steps=16, schedule=sched, regs=regs, block=block,
                  nodes_per_thread=npt)
    ids = [b.add(iv, opts(storage, k, kind, amp), 45)
           for (iv, kind, amp), k in zip(cases, kerns)]
    b.step(45)
    b.sync()
    for i, w in zip(ids, want):
        m = b.member(i)
        assert_same((m.export_arF(), m.macroscopic()), w)
    b.close()
