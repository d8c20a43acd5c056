"""The C ABI without a GPU: the library loads, exports every declared symbol,
and its host-side surface (decomposition, set_move_decomp, slice_chunk,
inverseMRT, tables, argument checking) matches the reference."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import oracle_lib as O

pkg = O.pkg
ROOT = O.ROOT
HEADERS = [os.path.join(ROOT, "include", h) for h in os.listdir(os.path.join(ROOT, "include"))
           if h.endswith(".h")]


def declared_symbols():
    names = set()
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[\w\s\*]+?\b(lbm_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_loads_and_exports_every_declared_symbol():
    L = pkg.lib()
    syms = declared_symbols()
    assert len(syms) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", pkg.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    missing = [s for s in syms if s not in exported]
    assert not missing, missing
    for s in syms:
        getattr(L, s)


def test_version_string():
    assert b"sm_100a" in pkg.lib().lbm_version()


@pytest.mark.parametrize("shape", [(10, 10, 10), (64, 64, 64), (7, 5, 3), (2, 9, 31), (256, 128, 128)])
def test_decomposition_matches_reference(shape):
    iv = pkg.make_inputval(*shape, tau=0.6)
    got = pkg.decomposition(iv)
    L = O.oracle_lib()
    want = np.zeros((pkg.TILE_NUM, 3, 2), np.int32)
    n = L.orc_decomposition(C.byref(iv), O._p(want))
    np.testing.assert_array_equal(got, want[:n])
    R = O.poplar_ref_lib()
    if R is not None:
        ref = np.zeros((pkg.TILE_NUM, 3, 2), np.int32)
        n2 = R.ref_decomposition(C.byref(iv), O._p(ref))
        np.testing.assert_array_equal(got, ref[:n2])
        mv_ref = np.zeros((n2, 19), np.int32)
        R.ref_set_move_decomp(n2, O._p(ref), O._p(mv_ref))
        np.testing.assert_array_equal(pkg.set_move_decomp(got), mv_ref)
    # slice_chunk: 1 for empty tiles, chunk sizes otherwise
    L2 = pkg.lib()
    for t in range(len(got)):
        v = [C.c_int() for _ in range(10)]
        rc = L2.lbm_slice_chunk(t, O._p(got), *[C.byref(x) for x in v])
        dx, dy, dz = (got[t, m, 1] - got[t, m, 0] for m in range(3))
        assert rc == (1 if min(dx, dy, dz) < 1 else 0)
        assert [x.value for x in v[6:]] == [dx, dy, dz, dx * dy * dz]


def test_move_table_is_neighbour_offset():
    iv = pkg.make_inputval(9, 6, 12, tau=0.6)
    sl = pkg.decomposition(iv)
    mv = pkg.set_move_decomp(sl)
    d, _, _, _ = pkg.d3q19_tables()
    for t in range(len(sl)):
        px = sl[t, 0, 1] - sl[t, 0, 0] + 2
        pz = sl[t, 2, 1] - sl[t, 2, 0] + 2
        for q in range(19):
            cx, cz, cy = int(d[0 * 19 + q]), int(d[1 * 19 + q]), int(d[2 * 19 + q])
            assert mv[t, q] == (cx + 1) + (cy + 1) * px * pz + (cz + 1) * px


def test_inverse_mrt_bit_exact_with_reference():
    _, _, _, M = pkg.d3q19_tables()
    inv = pkg.inverse_mrt(M)
    L = O.oracle_lib()
    want = np.zeros((19, 19), np.float32)
    L.orc_inverse_mrt(O._p(M), O._p(want))
    np.testing.assert_array_equal(inv, want)
    R = O.poplar_ref_lib()
    if R is not None:
        ref = np.zeros((19, 19), np.float32)
        R.ref_inverse_mrt(O._p(M), O._p(ref))
        np.testing.assert_array_equal(inv, ref)
    assert np.abs(inv.astype(np.float64) @ M - np.eye(19)).max() < 1e-5


def test_inverse_mrt_singular_is_an_error_not_exit():
    M = np.ones((19, 19), np.float32)
    with pytest.raises(pkg.LbmError) as e:
        pkg.inverse_mrt(M)
    assert e.value.code == pkg.LBM_ERR_SINGULAR
    assert b"singular" in pkg.lib().lbm_last_error()


def test_tables_match_reference_main_cpp():
    d, o, w, M = pkg.d3q19_tables()
    L = O.oracle_lib()
    d2, o2, w2, M2 = (np.zeros(57, np.float32), np.zeros(19, np.int32), np.zeros(19, np.float32),
                      np.zeros((19, 19), np.float32))
    L.orc_tables(O._p(d2), O._p(o2), O._p(w2), O._p(M2))
    for a, b in ((d, d2), (o, o2), (w, w2), (M, M2)):
        np.testing.assert_array_equal(a, b)
    assert abs(w.sum() - 1.0) < 1e-6
    # rows of M are orthogonal (so M^-1 = M^T diag(1/|row|^2))
    G = M.astype(np.float64) @ M.T.astype(np.float64)
    assert np.abs(G - np.diag(np.diag(G))).max() == 0


def test_argument_errors_are_status_codes():
    L = pkg.lib()
    h = C.c_void_p()
    assert L.lbm_create(None, None, C.byref(h)) == pkg.LBM_ERR_INVALID
    assert b"NULL" in L.lbm_last_error()
    iv = pkg.make_inputval(2, 8, 8, tau=0.6)
    assert L.lbm_create(C.byref(iv), None, C.byref(h)) == pkg.LBM_ERR_INVALID
    iv = pkg.make_inputval(8, tau=0.6, casetype=7)
    assert L.lbm_create(C.byref(iv), None, C.byref(h)) == pkg.LBM_ERR_INVALID
    iv = pkg.make_inputval(8, tau=float("nan"))
    assert L.lbm_create(C.byref(iv), None, C.byref(h)) == pkg.LBM_ERR_INVALID
    iv = pkg.make_inputval(8, tau=0.6)
    bad = pkg.default_options(storage=7)
    assert L.lbm_create(C.byref(iv), C.byref(bad), C.byref(h)) == pkg.LBM_ERR_INVALID
    bad = pkg.default_options(kernel=9)
    assert L.lbm_create(C.byref(iv), C.byref(bad), C.byref(h)) == pkg.LBM_ERR_INVALID
    assert b"kernel" in L.lbm_last_error()
    for fn in ("lbm_initialize", "lbm_sync", "lbm_destroy"):
        assert getattr(L, fn)(None) == pkg.LBM_ERR_INVALID
    assert L.lbm_run_simulation(None, 1) == pkg.LBM_ERR_INVALID


def test_estimate_bytes():
    iv = pkg.make_inputval(256, tau=0.6)
    b = C.c_size_t()
    assert pkg.lib().lbm_estimate_bytes(C.byref(iv), None, C.byref(b)) == 0
    lat = 2 * 19 * 256 ** 3 * 4
    assert lat <= b.value <= lat * 1.2
    o = pkg.default_options(storage=pkg.STORE_F16_SHIFT)
    b2 = C.c_size_t()
    assert pkg.lib().lbm_estimate_bytes(C.byref(iv), C.byref(o), C.byref(b2)) == 0
    assert b2.value < b.value * 0.6


def test_aa_streaming_cases_and_footprint():
    """AA streaming: cavities and channels pass validation, POISEUILLE (STRUCT
    geometry) does not; the footprint (single domain and batch member) drops
    by one population lattice."""
    L = pkg.lib()
    h = C.c_void_p()
    aa = pkg.default_options(stream_mode=pkg.STREAM_AA)
    pipe = pkg.make_inputval(32, 16, 16, casetype=pkg.POISEUILLE, tau=0.6, u=0.05)
    assert L.lbm_create(C.byref(pipe), C.byref(aa), C.byref(h)) == pkg.LBM_ERR_INVALID
    assert b"AA streaming" in L.lbm_last_error()
    for case in (pkg.CAVITY, pkg.CHANNEL):
        iv = pkg.make_inputval(64, 32, 32, casetype=case, tau=0.6, u=0.05)
        for st, size in ((pkg.STORE_F32, 4), (pkg.STORE_F16_SHIFT, 2)):
            ab_o = pkg.default_options(storage=st, stream_mode=pkg.STREAM_AB)
            aa_o = pkg.default_options(storage=st, stream_mode=pkg.STREAM_AA)
            lattice = 19 * 64 * 32 * 32 * size
            b_ab, b_aa = C.c_size_t(), C.c_size_t()
            assert L.lbm_estimate_bytes(C.byref(iv), C.byref(ab_o), C.byref(b_ab)) == 0
            assert L.lbm_estimate_bytes(C.byref(iv), C.byref(aa_o), C.byref(b_aa)) == 0
            assert b_ab.value - b_aa.value >= lattice
            assert pkg.batch_domain_bytes(iv, ab_o) - pkg.batch_domain_bytes(iv, aa_o) >= lattice
    with pytest.raises(pkg.LbmError):
        pkg.batch_domain_bytes(pipe, aa)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU path")
def test_no_device_is_reported_not_faked():
    iv = pkg.make_inputval(8, tau=0.6)
    with pytest.raises(pkg.LbmError) as e:
        pkg.Domain(iv)
    assert e.value.code in (pkg.LBM_ERR_NO_DEVICE, pkg.LBM_ERR_CUDA)


def test_pattern_ceiling_rejects_bad_arguments():
    """Argument checks of lbm_pattern_ceiling happen before any device call."""
    m, g = C.c_double(), C.c_double()
    L = pkg.lib()
    for args in ((99, pkg.STORE_F32, 64, 2), (pkg.PATTERN_PULL, pkg.STORE_F64, 64, 2),
                 (pkg.PATTERN_PULL_PAIRED, pkg.STORE_F32, 64, 2), (pkg.PATTERN_PULL, pkg.STORE_F32, 48, 2),
                 (pkg.PATTERN_PULL, pkg.STORE_F32, 1024, 2), (pkg.PATTERN_PULL, pkg.STORE_F32, 64, 0)):
        assert L.lbm_pattern_ceiling(*args, C.byref(m), C.byref(g)) == pkg.LBM_ERR_INVALID, args
    assert L.lbm_pattern_ceiling(pkg.PATTERN_PULL, pkg.STORE_F32, 64, 2, None, None) == \
        pkg.LBM_ERR_INVALID


def test_compat_header_compiles_and_runs_the_host_functions(tmp_path):
    """include/lbm_b200_compat.hpp compiled by a C++ caller that uses the
    reference's spelling: LBMSolver's tables, decomposition, inverseMRT
    (host numerics only, no device needed)."""
    src = tmp_path / "caller.cpp"
    src.write_text(r'''
#include <cstdio>
#include "lbm_b200_compat.hpp"
int main() {
  LBMSolver s;
  Inputval in{};
  in.h = in.nx = in.ny = in.nz = 10;
  static int Slice[TILE_NUM][DIMENSION][2];
  int n = decomposition(&in, Slice);
  std::vector<std::vector<float>> m(DIRECTION_SIZE, std::vector<float>(DIRECTION_SIZE)), inv;
  float M[DIRECTION_SIZE * DIRECTION_SIZE];
  lbm_d3q19_tables(nullptr, nullptr, nullptr, M);
  for (int i = 0; i < DIRECTION_SIZE; ++i)
    for (int j = 0; j < DIRECTION_SIZE; ++j) m[i][j] = M[i * DIRECTION_SIZE + j];
  inverseMRT(m, inv);
  double e = 0;
  for (int i = 0; i < DIRECTION_SIZE; ++i)
    for (int j = 0; j < DIRECTION_SIZE; ++j) {
      double acc = 0;
      for (int k = 0; k < DIRECTION_SIZE; ++k) acc += m[i][k] * inv[k][j];
      e += acc - (i == j);
    }
  std::printf("%d %d %.6f %.6f %d %g\n", n, s.m_HostOppIndex[7], s.m_HostW[0], s.m_HostW[18],
              s.m_pDomain == nullptr, e);
  return 0;
}
''')
    exe = tmp_path / "caller"
    pkgdir = os.path.join(O.ROOT if hasattr(O, "ROOT") else os.path.dirname(os.path.dirname(
        os.path.abspath(__file__))), "nflow-red-poplar_b200")
    inc = os.path.join(os.path.dirname(pkgdir), "include")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", inc, str(src), "-L", pkgdir, "-llbm_b200",
                    "-Wl,-rpath," + pkgdir, "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    assert out[0] == "27" and out[1] == "10"
    assert abs(float(out[2]) - 1 / 3) < 1e-6 and abs(float(out[3]) - 1 / 36) < 1e-6
    assert out[4] == "1" and abs(float(out[5])) < 1e-3


def test_server_rejects_bad_options_before_any_device_call():
    """lbm_server_create checks the policy and the residual-check spacing
    (a positive multiple of the batch chunk) before it creates the batch."""
    L = pkg.lib()
    for policy, every, chunk in ((7, 256, 32), (pkg.SERVE_FIFO, 33, 32), (pkg.SERVE_FIFO, 0, 32),
                                 (pkg.SERVE_SHORTEST, 48, 32), (pkg.SERVE_FIFO, 16, 32)):
        o = pkg.ServerOptions()
        L.lbm_server_default_options(C.byref(o))
        o.policy, o.check_every, o.batch.chunk_steps = policy, every, chunk
        h = C.c_void_p()
        assert L.lbm_server_create(C.byref(o), C.byref(h)) == pkg.LBM_ERR_INVALID
        assert not h.value
    o = pkg.ServerOptions()
    L.lbm_server_default_options(C.byref(o))
    assert o.policy == pkg.SERVE_FIFO and o.check_every == 256
    assert L.lbm_server_create(C.byref(o), None) == pkg.LBM_ERR_INVALID
