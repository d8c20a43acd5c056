"""Result files of a live domain (snapshot -> asynchronous host copy ->
writer) and the residual-based convergence stop (kernel.cu:203-248)."""
import os
import struct

import numpy as np
import pytest

import oracle_lib as O

pkg = O.pkg
pytestmark = pytest.mark.gpu


def cavity(n=24, re=100.0, mrt=True, les=True):
    return pkg.make_inputval(n, n - 4, n + 2, casetype=pkg.CAVITY, re=re, u=0.1, mrt=mrt, les=les,
                             cs=0.1, h=n)


def test_save_file_csv_equals_writer_on_macroscopic(tmp_path):
    iv = cavity()
    d = pkg.Domain(iv, pkg.default_options(init_kind=pkg.INIT_DENSITY_NOISE, noise_amp=1e-6))
    d.run(40)
    d.save_file(pkg.SAVE_CSV, tmp_path / "gpu")
    pkg.write_csv(tmp_path / "r.csv", tmp_path / "s.csv", *d.macroscopic())
    assert (tmp_path / "gpu" / "result.csv").read_bytes() == (tmp_path / "r.csv").read_bytes()
    assert (tmp_path / "gpu" / "section.csv").read_bytes() == (tmp_path / "s.csv").read_bytes()
    d.close()


def test_snapshot_is_the_state_when_taken_while_stepping_continues(tmp_path):
    iv = cavity(32)
    d = pkg.Domain(iv, pkg.default_options(init_kind=pkg.INIT_DENSITY_NOISE, noise_amp=1e-6))
    d.run(20)
    before = d.macroscopic()
    d.snapshot()
    d.run(30)  # overlaps the snapshot's host copy
    after = d.macroscopic()
    d.save_snapshot(pkg.SAVE_VTU, tmp_path, index=3)
    raw = (tmp_path / "Output000003.vtu").read_bytes()
    rest = raw.split(b'<AppendedData encoding="raw">\n_', 1)[1]
    blocks, pos = [], 0
    for _ in range(12):
        n = struct.unpack_from("<Q", rest, pos)[0]
        blocks.append(rest[pos + 8: pos + 8 + n])
        pos += 8 + n
    den = np.frombuffer(blocks[5], np.float64).reshape(before[0].shape)
    np.testing.assert_array_equal(den, before[0].astype(np.float64))
    assert not np.array_equal(before[0], after[0])
    t, _ = d.node_info()
    for k, bit in enumerate([pkg.NODE_FLUID, pkg.NODE_FIXEDWALL, pkg.NODE_MOVINGWALL,
                             pkg.NODE_INLET, pkg.NODE_OUTLET, pkg.NODE_STRUCT]):
        flags = np.frombuffer(blocks[6 + k], np.int32).reshape(t.shape)
        np.testing.assert_array_equal(flags, ((t & bit) != 0).astype(np.int32))
    d.close()


def test_save_errors(tmp_path):
    iv = cavity(12)
    d = pkg.Domain(iv)
    (tmp_path / "a_file").write_text("x")
    bad = tmp_path / "a_file" / "sub"  # cannot be created
    with pytest.raises(pkg.LbmError) as e:
        d.save_snapshot(pkg.SAVE_CSV, bad)
    assert e.value.code == pkg.LBM_ERR_STATE  # no snapshot yet
    d.snapshot()
    with pytest.raises(pkg.LbmError) as e:
        d.save_snapshot(pkg.SAVE_CSV, bad)
    assert e.value.code == pkg.LBM_ERR_IO
    with pytest.raises(pkg.LbmError):
        d.save_snapshot(7, "/tmp")
    d.close()


def test_run_until_converged_stops_on_the_residual():
    iv = cavity(20, re=20.0, les=False)
    o = pkg.default_options(init_kind=pkg.INIT_DENSITY_NOISE, noise_amp=1e-6)
    probe = pkg.Domain(iv, o)
    probe.run(100)
    tol = probe.diagnostics()[4] / 50  # fifty-fold decay of the start-up residual
    probe.close()
    d = pkg.Domain(iv, o)
    n, r = d.run_until_converged(max_steps=20000, check_every=100, tol=tol)
    assert 100 < n < 20000 and n % 100 == 0
    assert r <= tol
    assert d.diagnostics()[4] == r
    assert d.steps() == n
    # the same number of plain steps gives the same state
    e = pkg.Domain(iv, o)
    e.run(n)
    np.testing.assert_array_equal(d.export_arF(), e.export_arF())
    # a budget that ends first reports the last residual, above tol
    f = pkg.Domain(iv, o)
    n2, r2 = f.run_until_converged(max_steps=150, check_every=100, tol=tol)
    assert n2 == 150 and r2 > tol
    for h in (d, e, f):
        h.close()


def test_checkpoint_restart_continues_bit_for_bit(tmp_path):
    iv = cavity(24, re=300.0)
    o = pkg.default_options(init_kind=pkg.INIT_DENSITY_NOISE, noise_amp=1e-6)
    a = pkg.Domain(iv, o)
    a.run(70)
    a.save_checkpoint(tmp_path / "ck.bin")
    a.run(55)
    b = pkg.Domain(iv, o)
    assert b.load_checkpoint(tmp_path / "ck.bin") == 70
    b.run(55)
    np.testing.assert_array_equal(a.export_arF(), b.export_arF())
    for x, y in zip(a.macroscopic(), b.macroscopic()):
        np.testing.assert_array_equal(x, y)
    # wrong extents and non-checkpoint files are errors
    c = pkg.Domain(cavity(16), o)
    with pytest.raises(pkg.LbmError):
        c.load_checkpoint(tmp_path / "ck.bin")
    (tmp_path / "junk.bin").write_bytes(b"not a checkpoint" * 8)
    with pytest.raises(pkg.LbmError):
        b.load_checkpoint(tmp_path / "junk.bin")
    for h in (a, b, c):
        h.close()
