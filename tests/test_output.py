"""Result files (kernel.cu:699-1018 saveFile) written by lbm_write_csv /
lbm_write_vtu, against the reference's own saveFile (oracle/_ref, host code
of kernel.cu) and against committed fixtures made by it.

CSV: byte for byte.  VTU: same document (element order, names, attribute
text, appended UInt64-prefixed blocks); the reference's Float64 blocks hold
the bytes of two neighbouring floats (it writes 8 bytes from each 4-byte
value) and its cell list is padded with all-zero cells up to nx*ny*nz, so
those are compared as documented differences: our Float64 blocks must equal
the float fields, our cells must equal the reference's non-padding cells.
"""
import os
import re
import struct

import numpy as np
import pytest

import oracle_lib as O

pkg = O.pkg
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "savefile")
FLAGS = [pkg.NODE_FLUID, pkg.NODE_FIXEDWALL, pkg.NODE_MOVINGWALL, pkg.NODE_INLET,
         pkg.NODE_OUTLET, pkg.NODE_STRUCT]


def fields(nx, ny, nz, seed):
    """Seeded fields [ny][nz][nx] with the value ranges of a run."""
    rng = np.random.default_rng(seed)
    sh = (ny, nz, nx)
    den = (1.0 + 0.01 * rng.standard_normal(sh)).astype(np.float32)
    u = [(0.05 * rng.standard_normal(sh)).astype(np.float32) for _ in range(3)]
    t = rng.choice(np.array(FLAGS, np.int32), size=sh)
    return den, u, t


def ref_save(tmp, nx, ny, nz, den, u, t, savetype, index=0):
    L = O.kernelcu_ref_lib()
    iv = pkg.make_inputval(nx, ny, nz, tau=0.6)
    os.makedirs(tmp, exist_ok=True)
    rc = L.kref_save_file(O.C.byref(iv), O._p(den), *[O._p(a) for a in u], O._p(t), savetype,
                          index, os.fsencode(tmp))
    assert rc == 0


def parse_vtu(path):
    raw = open(path, "rb").read()
    head, rest = raw.split(b'<AppendedData encoding="raw">\n_', 1)
    blocks = []
    pos = 0
    for _ in range(12):
        n = struct.unpack_from("<Q", rest, pos)[0]
        blocks.append(rest[pos + 8: pos + 8 + n])
        pos += 8 + n
    assert rest[pos:] == b"</AppendedData>\n</VTKFile>"
    return head.decode(), blocks


needs_ref = pytest.mark.skipif(O.kernelcu_ref_lib() is None,
                               reason="reference kernel.cu not built (oracle/_ref)")


@needs_ref
@pytest.mark.parametrize("shape,seed", [((7, 5, 6), 1), ((52, 4, 51), 2), ((3, 3, 3), 3)])
def test_csv_byte_for_byte_with_reference(tmp_path, shape, seed):
    nx, ny, nz = shape
    den, u, t = fields(nx, ny, nz, seed)
    ref_save(str(tmp_path / "ref"), nx, ny, nz, den, u, t, pkg.SAVE_CSV)
    pkg.write_csv(tmp_path / "result.csv", tmp_path / "section.csv", den, *u)
    for name in ("result.csv", "section.csv"):
        assert (tmp_path / name).read_bytes() == (tmp_path / "ref" / name).read_bytes(), name


def test_csv_matches_committed_fixtures(tmp_path):
    for (nx, ny, nz), seed in (((7, 5, 6), 1), ((52, 4, 51), 2)):
        den, u, t = fields(nx, ny, nz, seed)
        pkg.write_csv(tmp_path / "result.csv", tmp_path / "section.csv", den, *u)
        for name in ("result.csv", "section.csv"):
            path = os.path.join(GOLDEN, f"{nx}x{ny}x{nz}_{name}")
            if not os.path.exists(path):  # only the section line is kept for 52x4x51
                continue
            want = open(path, "rb").read()
            assert (tmp_path / name).read_bytes() == want, (nx, ny, nz, name)


@needs_ref
@pytest.mark.parametrize("shape,seed", [((6, 5, 4), 4), ((9, 3, 7), 5)])
def test_vtu_document_matches_reference(tmp_path, shape, seed):
    nx, ny, nz = shape
    den, u, t = fields(nx, ny, nz, seed)
    ref_save(str(tmp_path / "ref"), nx, ny, nz, den, u, t, pkg.SAVE_VTU, index=7)
    ref_path = tmp_path / "ref" / "result" / "Output000007.vtu"
    pkg.write_vtu(tmp_path / "ours.vtu", den, *u, t)
    h_ref, b_ref = parse_vtu(ref_path)
    h_our, b_our = parse_vtu(tmp_path / "ours.vtu")
    N = nx * ny * nz
    cells = (nx - 1) * (ny - 1) * (nz - 1)
    # header: identical once the cell count and the block offsets that follow
    # the (shorter) cell blocks are masked
    mask = lambda h: re.sub(r'(NumberOfCells|offset)="\d+"', r'\1="#"', h)
    assert mask(h_our) == mask(h_ref)
    assert f'NumberOfCells="{N}"' in h_ref and f'NumberOfCells="{cells}"' in h_our
    conn_ref = np.frombuffer(b_ref[1], np.int32)
    conn_our = np.frombuffer(b_our[1], np.int32)
    np.testing.assert_array_equal(conn_our, conn_ref[: cells * 8])
    assert not conn_ref[cells * 8:].any()  # the reference's padding cells
    np.testing.assert_array_equal(np.frombuffer(b_our[2], np.int32),
                                  np.frombuffer(b_ref[2], np.int32)[:cells])
    assert b_our[3] == b_ref[3][:cells] and set(b_our[3]) == {12}
    for k in range(6):  # Int32 flag blocks: identical
        assert b_our[6 + k] == b_ref[6 + k]
    # Float64 blocks: ours hold the fields themselves
    pts = np.frombuffer(b_our[0], np.float64).reshape(ny, nz, nx, 3)
    yy, zz, xx = np.meshgrid(np.arange(ny), np.arange(nz), np.arange(nx), indexing="ij")
    np.testing.assert_array_equal(pts, np.stack([xx, yy, zz], -1).astype(np.float64))
    vel = np.frombuffer(b_our[4], np.float64).reshape(ny, nz, nx, 3)
    np.testing.assert_array_equal(vel, np.stack(u, -1).astype(np.float64))
    np.testing.assert_array_equal(np.frombuffer(b_our[5], np.float64).reshape(ny, nz, nx),
                                  den.astype(np.float64))


def test_writer_errors_are_status_codes(tmp_path):
    den, u, t = fields(4, 4, 4, 0)
    with pytest.raises(pkg.LbmError) as e:
        pkg.write_csv(tmp_path / "missing_dir" / "r.csv", None, den, *u)
    assert e.value.code == pkg.LBM_ERR_IO
    with pytest.raises(pkg.LbmError) as e:
        pkg.write_vtu(tmp_path / "missing_dir" / "a.vtu", den, *u, t)
    assert e.value.code == pkg.LBM_ERR_IO
    L = pkg.lib()
    assert L.lbm_write_vtu(b"x.vtu", 4, 4, 4, None, None, None, None, None) == pkg.LBM_ERR_INVALID
