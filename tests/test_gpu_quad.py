"""The word AA step of the 16-bit forms over quad rows (LBM_KERNEL_QUAD, the
default of FP16/BF16 shifted storage with LBM_STREAM_AA).

Quad rows store the 8-byte word w of every row as the nodes w, w + nx/2,
w + nx/4, w + 3nx/4 and step four nodes per thread (two F2 halves of packed
FP32 arithmetic); the per-node AA step (LBM_KERNEL_SCALAR) steps plain rows
one node per thread.  Both run the same node arithmetic without multiply-add
contraction, so a domain must give the same bits either way: after any
number of steps (ending on either AA layout, across CUDA-graph chunks) the
exported arF, which undoes the layout, and the macroscopic fields are
compared for equality over shapes that exercise the seams between the row
quarters (the smallest rows of four words, rows of one partial warp, rows
of several warps), both collision models with and without LES, the
channel's inlet/outlet rules, imports and checkpoints.
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


def opts(storage, kernel, kind=pkg.INIT_DENSITY_NOISE, amp=1e-4, rounding=pkg.ROUND_NEAREST,
         seed=7):
    return pkg.default_options(storage=storage, kernel=kernel, stream_mode=pkg.STREAM_AA,
                               init_kind=kind, noise_amp=amp, seed=seed, rounding=rounding)


def run(iv, o, steps):
    d = pkg.Domain(iv, o)
    d.run(steps)
    out = (d.export_arF(), d.macroscopic())
    d.close()
    return out


WORDS = [pkg.KERNEL_QUAD]


def both(iv, storage, steps, kind=pkg.INIT_DENSITY_NOISE, amp=1e-4, kernel=pkg.KERNEL_QUAD):
    return [run(iv, opts(storage, k, kind, amp), steps) for k in (kernel, pkg.KERNEL_SCALAR)]


def assert_same(a, b):
    np.testing.assert_array_equal(a[0], b[0])
    for x, y in zip(a[1], b[1]):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("kernel", WORDS)
@pytest.mark.parametrize("storage", STORES)
@pytest.mark.parametrize("shape", [(64, 20, 18), (16, 9, 7), (32, 6, 5), (256, 6, 5),
                                   (136, 10, 9)])
@pytest.mark.parametrize("steps", [1, 2, 37, 70])
def test_words_equal_per_node_cavity(kernel, storage, shape, steps):
    a, b = both(cavity(*shape), storage, steps, kernel=kernel)
    assert_same(a, b)
    assert np.isfinite(a[0]).all()


@pytest.mark.parametrize("kernel", WORDS)
@pytest.mark.parametrize("storage", STORES)
@pytest.mark.parametrize("mrt,les", [(True, True), (False, False), (False, True), (True, False)])
def test_words_equal_per_node_models(kernel, storage, mrt, les):
    a, b = both(cavity(48, 14, 12, mrt=mrt, les=les), storage, 71, kernel=kernel)
    assert_same(a, b)


@pytest.mark.parametrize("kernel", WORDS)
@pytest.mark.parametrize("storage", STORES)
@pytest.mark.parametrize("shape", [(48, 12, 14), (64, 9, 10), (16, 8, 9)])
@pytest.mark.parametrize("steps", [66, 67])
def test_words_equal_per_node_channel(kernel, storage, shape, steps):
    a, b = both(channel(*shape), storage, steps, kind=pkg.INIT_CHANNEL, amp=0.01, kernel=kernel)
    assert_same(a, b)


@pytest.mark.parametrize("storage", STORES)
def test_quad_import_export_and_checkpoint(storage, tmp_path):
    """Import (the first step then leaves a complete natural layout), export
    in both layouts and a checkpoint round trip give the same bits with quad
    and plain rows."""
    iv = cavity(40, 12, 10)
    src = pkg.Domain(iv, pkg.default_options(init_kind=pkg.INIT_DENSITY_NOISE, noise_amp=1e-4,
                                             seed=3))
    src.run(9)
    arF = src.export_arF(padded=True)
    src.close()
    res = []
    for kern in (pkg.KERNEL_QUAD, pkg.KERNEL_SCALAR):
        d = pkg.Domain(iv, opts(storage, kern))
        d.import_arF(arF, padded=True)
        first = d.export_arF(padded=True)
        d.run(3)
        odd = d.export_arF()
        path = str(tmp_path / f"k{kern}.ckpt")
        d.run(2)
        d.save_checkpoint(path)
        d.run(6)
        a1 = d.export_arF()
        d.load_checkpoint(path)
        d.run(6)
        a2 = d.export_arF()
        den = d.macroscopic()[0]
        d.close()
        res.append((first, odd, a1, a2, den))
    for other in res[1:]:
        for x, y in zip(res[0], other):
            np.testing.assert_array_equal(x, y)


def test_quad_is_the_16bit_aa_default_and_fallbacks():
    """AUTO picks quad rows where they fit (same bits as KERNEL_QUAD), plain
    rows otherwise (nx not a multiple of 8); KERNEL_QUAD is refused where
    quad rows do not fit and outside the 16-bit AA form."""
    iv = cavity(40, 18, 16)
    st = pkg.STORE_F16_SHIFT
    assert_same(run(iv, opts(st, pkg.KERNEL_AUTO), 33), run(iv, opts(st, pkg.KERNEL_QUAD), 33))
    iv2 = cavity(36, 10, 9)
    assert_same(run(iv2, opts(st, pkg.KERNEL_AUTO), 33),
                run(iv2, opts(st, pkg.KERNEL_SCALAR), 33))
    with pytest.raises(pkg.LbmError):
        pkg.Domain(iv2, opts(st, pkg.KERNEL_QUAD))
    with pytest.raises(pkg.LbmError):
        pkg.Domain(iv, opts(st, pkg.KERNEL_PAIRED))  # paired rows: the pull form
    with pytest.raises(pkg.LbmError):
        pkg.Domain(iv, pkg.default_options(storage=st, kernel=pkg.KERNEL_QUAD))  # pull form
    with pytest.raises(pkg.LbmError):
        pkg.Domain(iv, pkg.default_options(kernel=pkg.KERNEL_QUAD, stream_mode=pkg.STREAM_AA))


@pytest.mark.parametrize("kernel", WORDS)
@pytest.mark.parametrize("storage", STORES)
def test_words_stochastic_rounding(kernel, storage):
    """Stochastic rounding on quad rows: reproducible for a seed, different
    for another seed, and within a few storage quanta of round-to-nearest
    after a few steps (deviations g ~ 1e-3 here: the FP16 quantum of g is
    ~5e-7, the BF16 one ~4e-6)."""
    iv = cavity(64, 20, 18)
    sr = lambda seed: run(iv, opts(storage, kernel, rounding=pkg.ROUND_STOCHASTIC, seed=seed), 6)
    a, b, c = sr(7), sr(7), sr(8)
    rn = run(iv, opts(storage, kernel, seed=7), 6)
    assert_same(a, b)
    assert not np.array_equal(a[0], c[0])
    d = np.abs(a[0].astype(np.float64) - rn[0]).max()
    assert 0 < d < (1e-4 if storage == pkg.STORE_F16_SHIFT else 1e-3), d


@pytest.mark.parametrize("kernel", WORDS)
@pytest.mark.parametrize("storage", STORES)
def test_words_equal_per_node_precision_channel(kernel, storage):
    """The shortened precision channel (128x32x32, MRT + LES, tau 0.5192):
    word rows and plain rows agree bit for bit over 130 steps."""
    nu = (0.5192 - 0.5) / 3.0
    iv = pkg.make_inputval(128, 32, 32, casetype=pkg.CHANNEL, tau=3.0 * nu + 0.5, u=0.05,
                           mrt=True, les=True, cs=0.1)
    a, b = both(iv, storage, 130, kind=pkg.INIT_CHANNEL, amp=0.01, kernel=kernel)
    assert_same(a, b)
