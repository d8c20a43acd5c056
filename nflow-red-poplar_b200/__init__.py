"""ctypes binding of the B200 D3Q19 lattice-Boltzmann library (liblbm_b200.so).

The library exposes the C ABI declared in include/lbm_b200.h; this module is
a thin Python view of it used by the tests and bench.py.  The directory name
contains dashes, so it is loaded by path (see ``load_package`` in
tests/conftest.py and bench.py) rather than imported by name.

Nothing here computes: every numeric call goes to the CUDA library, and a
missing library raises instead of falling back to anything else.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("LBM_B200_LIB") or os.path.join(HERE, "liblbm_b200.so")

DIRECTION_SIZE = 19
DIMENSION = 3
XDIM, ZDIM, YDIM = 0, 1, 2
XDECOMP = YDECOMP = ZDECOMP = 3
TILE_NUM = 1471
CAVITY, POISEUILLE, CHANNEL = 1, 0, 2
NODE_FLUID, NODE_FIXEDWALL, NODE_MOVINGWALL = 1 << 1, 1 << 2, 1 << 3
NODE_INLET, NODE_OUTLET, NODE_STRUCT = 1 << 4, 1 << 5, 1 << 6

LBM_OK = 0
LBM_ERR_INVALID = -1
LBM_ERR_CUDA = -2
LBM_ERR_OOM = -3
LBM_ERR_SINGULAR = -4
LBM_ERR_STATE = -5
LBM_ERR_TIMEOUT = -6
LBM_ERR_BUDGET = -7
LBM_ERR_NOT_FINITE = -8
LBM_ERR_NO_DEVICE = -9
LBM_ERR_IO = -10
SAVE_VTU, SAVE_CSV = 0, 1

STORE_F32, STORE_F16_SHIFT, STORE_BF16_SHIFT, STORE_F64 = 0, 1, 2, 3
INIT_REFERENCE, INIT_DENSITY_NOISE, INIT_CHANNEL = 0, 1, 2
STREAM_AB, STREAM_AA = 0, 1
KERNEL_AUTO, KERNEL_SCALAR, KERNEL_PACKED, KERNEL_TMA, KERNEL_PAIRED, KERNEL_QUAD = 0, 1, 2, 3, 4, 5
ROUND_NEAREST, ROUND_STOCHASTIC = 0, 1
(PATTERN_COPY, PATTERN_PULL, PATTERN_PULL_PAIRED, PATTERN_AA_LOCAL, PATTERN_AA_NEIGHBOR,
 PATTERN_AA_LOCAL_V8, PATTERN_AA_LOCAL_V16, PATTERN_AA_PAIRED_LOCAL, PATTERN_AA_PAIRED_NEIGHBOR,
 PATTERN_PULL_QUAD, PATTERN_AA_QUAD_LOCAL, PATTERN_AA_QUAD_NEIGHBOR) = range(12)
SERVE_FIFO, SERVE_SHORTEST = 0, 1
REQ_QUEUED, REQ_RESIDENT, REQ_DONE = 0, 1, 2


class Inputval(C.Structure):
    """struct.h:78-100 of the reference, field for field."""

    _fields_ = [
        ("h", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("ngrid", C.c_int), ("maxitr", C.c_int), ("nwrite", C.c_int),
        ("irestart", C.c_int), ("irst", C.c_int), ("icycle", C.c_int),
        ("m_dSmagorinsky", C.c_float), ("Re", C.c_float), ("length", C.c_float),
        ("nu", C.c_float), ("m_dRefViscosity", C.c_float), ("m_dRefDen", C.c_float),
        ("m_dTau", C.c_float), ("m_dRefVelx", C.c_float), ("m_dRefVely", C.c_float),
        ("m_dRefVelz", C.c_float), ("dWeps", C.c_float), ("dWepsj", C.c_float),
        ("dWXX", C.c_float), ("bEnableMRT", C.c_bool), ("bEnableLES", C.c_bool),
        ("savetype", C.c_int), ("casetype", C.c_int),
    ]


class Options(C.Structure):
    _fields_ = [
        ("storage", C.c_int), ("init_kind", C.c_int), ("seed", C.c_uint64),
        ("noise_amp", C.c_float), ("store_scale", C.c_float), ("stream_mode", C.c_int),
        ("device", C.c_int), ("kernel", C.c_int), ("rounding", C.c_int),
        ("wait_test", C.c_int), ("reserved", C.c_int * 5),
    ]


class BatchOptions(C.Structure):
    _fields_ = [
        ("device", C.c_int), ("hbm_budget", C.c_size_t), ("chunk_steps", C.c_int),
        ("block", C.c_int), ("nodes_per_thread", C.c_int), ("ctas_per_sm", C.c_int),
        ("schedule", C.c_int), ("regs", C.c_int), ("own_set_ctas", C.c_int),
        ("reserved", C.c_int * 5),
    ]


class ServerOptions(C.Structure):
    _fields_ = [
        ("batch", BatchOptions), ("policy", C.c_int), ("check_every", C.c_int),
        ("backlog_horizon_s", C.c_double), ("nominal_mlups", C.c_double),
        ("reserved", C.c_int * 6),
    ]


class ServerRequest(C.Structure):
    _fields_ = [
        ("state", C.c_int), ("converged", C.c_int), ("steps_done", C.c_longlong),
        ("residual", C.c_double), ("t_arrive", C.c_double), ("t_admit", C.c_double),
        ("t_done", C.c_double),
    ]


class ServerSummary(C.Structure):
    _fields_ = [
        ("submitted", C.c_longlong), ("admitted", C.c_longlong), ("completed", C.c_longlong),
        ("converged", C.c_longlong), ("queued", C.c_longlong), ("resident", C.c_longlong),
        ("elapsed_s", C.c_double), ("tts_p50_s", C.c_double), ("tts_p99_s", C.c_double),
        ("service_p50_s", C.c_double), ("service_p99_s", C.c_double),
        ("executed_lups", C.c_double), ("completed_lups", C.c_double),
        ("aggregate_mlups", C.c_double), ("pool_used_bytes", C.c_size_t),
    ]


def make_inputval(nx, ny=None, nz=None, *, casetype=CAVITY, tau=None, re=None, u=0.1,
                  mrt=False, les=False, cs=0.0, rho0=1.0, h=None):
    """Fill an Inputval the way main.cpp:59-85 does.

    tau is taken as given, or derived from Re as main.cpp:81 does
    (tau = 3*u*h/Re + 0.5 with h the grid size).
    """
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    iv = Inputval()
    iv.h = h if h is not None else nx
    iv.nx, iv.ny, iv.nz = nx, ny, nz
    iv.maxitr = 0
    iv.bEnableMRT = bool(mrt)
    iv.bEnableLES = bool(les)
    iv.m_dRefDen = rho0
    iv.m_dRefVelx, iv.m_dRefVely, iv.m_dRefVelz = u, 0.0, 0.0
    iv.length = float(nx * ny * nz)
    if tau is None:
        if re is None:
            raise ValueError("give tau or re")
        iv.Re = re
        iv.nu = np.float32(u) * np.float32(iv.h) / np.float32(re)
        tau = np.float32(3.0) * np.float32(u) * np.float32(iv.h) / np.float32(re) + np.float32(0.5)
    iv.m_dTau = tau
    iv.m_dSmagorinsky = cs
    iv.dWeps, iv.dWepsj, iv.dWXX = 3.0, -5.5, -0.5
    iv.nwrite = 10000
    iv.savetype = 1
    iv.casetype = casetype
    return iv


_lib = None


def lib():
    """The loaded liblbm_b200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run __graft_entry__.build() first")
        L = C.CDLL(LIB_PATH)
        vp, i32, ip = C.c_void_p, C.c_int, C.POINTER(C.c_int)
        L.lbm_last_error.restype = C.c_char_p
        L.lbm_version.restype = C.c_char_p
        L.lbm_default_options.argtypes = [C.POINTER(Options)]
        L.lbm_decomposition.argtypes = [C.POINTER(Inputval), vp]
        L.lbm_set_move_decomp.argtypes = [i32, vp, vp]
        L.lbm_slice_chunk.argtypes = [C.c_uint, vp] + [ip] * 10
        L.lbm_inverse_mrt.argtypes = [vp, vp]
        L.lbm_d3q19_tables.argtypes = [vp, vp, vp, vp]
        L.lbm_create.argtypes = [C.POINTER(Inputval), C.POINTER(Options), C.POINTER(vp)]
        L.lbm_destroy.argtypes = [vp]
        L.lbm_set_stream.argtypes = [vp, vp]
        L.lbm_get_stream.argtypes = [vp]
        L.lbm_get_stream.restype = vp
        L.lbm_initialize.argtypes = [vp]
        L.lbm_run_simulation.argtypes = [vp, i32]
        L.lbm_steps_done.argtypes = [vp, C.POINTER(C.c_longlong)]
        L.lbm_import_arF.argtypes = [vp, vp, i32]
        L.lbm_export_arF.argtypes = [vp, vp, i32]
        L.lbm_get_macroscopic.argtypes = [vp, vp, vp, vp, vp]
        L.lbm_get_node_info.argtypes = [vp, vp, vp]
        L.lbm_diagnostics.argtypes = [vp, vp]
        L.lbm_sync.argtypes = [vp]
        L.lbm_device_bytes.argtypes = [vp, C.POINTER(C.c_size_t)]
        L.lbm_estimate_bytes.argtypes = [C.POINTER(Inputval), C.POINTER(Options),
                                         C.POINTER(C.c_size_t)]
        L.lbm_last_run_ms.argtypes = [vp, C.POINTER(C.c_float)]
        L.lbm_field_diagnostics_static.argtypes = [vp, vp, vp, vp, vp, C.c_longlong, vp, vp]
        L.lbm_run_until_converged.argtypes = [vp, i32, i32, C.c_double, ip,
                                              C.POINTER(C.c_double)]
        L.lbm_write_vtu.argtypes = [C.c_char_p, i32, i32, i32, vp, vp, vp, vp, vp]
        L.lbm_write_csv.argtypes = [C.c_char_p, C.c_char_p, i32, i32, i32, vp, vp, vp, vp]
        L.lbm_snapshot.argtypes = [vp]
        L.lbm_save_snapshot.argtypes = [vp, i32, C.c_char_p, i32]
        L.lbm_save_file.argtypes = [vp, i32, C.c_char_p, i32]
        L.lbm_save_checkpoint.argtypes = [vp, C.c_char_p]
        L.lbm_set_solid_mask.argtypes = [vp, vp]
        L.lbm_load_checkpoint.argtypes = [vp, C.c_char_p, C.POINTER(C.c_longlong)]
        L.lbm_batch_default_options.argtypes = [C.POINTER(BatchOptions)]
        L.lbm_batch_create.argtypes = [C.POINTER(BatchOptions), C.POINTER(vp)]
        L.lbm_batch_destroy.argtypes = [vp]
        L.lbm_batch_add.argtypes = [vp, C.POINTER(Inputval), C.POINTER(Options), C.c_longlong,
                                    C.POINTER(C.c_int)]
        L.lbm_batch_step.argtypes = [vp, i32]
        L.lbm_batch_poll.argtypes = [vp, vp, i32, C.POINTER(C.c_int)]
        L.lbm_batch_domain.argtypes = [vp, i32, C.POINTER(vp)]
        L.lbm_batch_remove.argtypes = [vp, i32]
        L.lbm_batch_fetch.argtypes = [vp, i32, vp, vp, vp, vp]
        L.lbm_batch_sync.argtypes = [vp]
        L.lbm_batch_usage.argtypes = [vp, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t),
                                      C.POINTER(C.c_int)]
        L.lbm_batch_domain_bytes.argtypes = [C.POINTER(Inputval), C.POINTER(Options),
                                             C.POINTER(C.c_size_t)]
        L.lbm_batch_autotune.argtypes = [vp, i32, C.POINTER(BatchOptions)]
        L.lbm_batch_last_step_ms.argtypes = [vp, C.POINTER(C.c_float), C.POINTER(C.c_longlong)]
        L.lbm_pattern_ceiling.argtypes = [i32, i32, i32, i32, C.POINTER(C.c_double),
                                          C.POINTER(C.c_double)]
        L.lbm_device_fields.argtypes = [vp] + [C.POINTER(vp)] * 5
        L.lbm_server_default_options.argtypes = [C.POINTER(ServerOptions)]
        L.lbm_server_create.argtypes = [C.POINTER(ServerOptions), C.POINTER(vp)]
        L.lbm_server_destroy.argtypes = [vp]
        L.lbm_server_submit.argtypes = [vp, C.POINTER(Inputval), C.POINTER(Options),
                                        C.c_longlong, C.c_double, C.POINTER(C.c_int)]
        L.lbm_server_progress.argtypes = [vp, C.POINTER(C.c_int)]
        L.lbm_server_wait.argtypes = [vp, i32]
        L.lbm_server_result.argtypes = [vp, i32, vp, vp, vp, vp, C.POINTER(ServerRequest)]
        L.lbm_server_release.argtypes = [vp, i32]
        L.lbm_server_stats.argtypes = [vp, C.POINTER(ServerSummary)]
        L.lbm_server_batch.argtypes = [vp, C.POINTER(vp)]
        _lib = L
    return _lib


class LbmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def check(rc):
    if rc < 0:
        raise LbmError(rc, lib().lbm_last_error().decode())
    return rc


def pattern_ceiling(pattern, storage, n=256, iters=20):
    """(MLUPS, GB/s) of a bare memory pattern of the step (lbm_pattern_ceiling)."""
    m, g = C.c_double(), C.c_double()
    check(lib().lbm_pattern_ceiling(int(pattern), int(storage), int(n), int(iters), C.byref(m),
                                    C.byref(g)))
    return m.value, g.value


def default_options(**kw):
    o = Options()
    lib().lbm_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class Domain:
    """One resident D3Q19 domain on a GPU (owns its device memory)."""

    def __init__(self, inputval, options=None, initialize=True):
        self.iv = inputval
        self.opt = options if options is not None else default_options()
        h = C.c_void_p()
        check(lib().lbm_create(C.byref(self.iv), C.byref(self.opt), C.byref(h)))
        self.h = h
        self.shape = (inputval.ny, inputval.nz, inputval.nx)
        if initialize:
            self.initialize()

    def close(self):
        if self.h:
            check(lib().lbm_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def initialize(self):
        check(lib().lbm_initialize(self.h))

    def run(self, nsteps):
        check(lib().lbm_run_simulation(self.h, int(nsteps)))

    def sync(self):
        check(lib().lbm_sync(self.h))

    def set_stream(self, stream_ptr):
        check(lib().lbm_set_stream(self.h, C.c_void_p(stream_ptr) if stream_ptr else None))

    def steps(self):
        s = C.c_longlong()
        check(lib().lbm_steps_done(self.h, C.byref(s)))
        return s.value

    def export_arF(self, padded=False, out=None):
        ny, nz, nx = self.shape
        shp = (ny + 2, nz + 2, nx + 2, 19) if padded else (ny, nz, nx, 19)
        if out is None:
            out = np.empty(shp, np.float32)
        assert out.shape == shp and out.dtype == np.float32 and out.flags.c_contiguous
        check(lib().lbm_export_arF(self.h, _ptr(out), 1 if padded else 0))
        return out

    def import_arF(self, arF, padded=False):
        arF = np.ascontiguousarray(arF, dtype=np.float32)
        check(lib().lbm_import_arF(self.h, _ptr(arF), 1 if padded else 0))

    def macroscopic(self):
        out = [np.empty(self.shape, np.float32) for _ in range(4)]
        check(lib().lbm_get_macroscopic(self.h, *[_ptr(a) for a in out]))
        return out  # den, ux, uy, uz

    def node_info(self):
        t = np.empty(self.shape, np.int32)
        s = np.empty(self.shape, np.int32)
        check(lib().lbm_get_node_info(self.h, _ptr(t), _ptr(s)))
        return t, s

    def diagnostics(self):
        out = np.zeros(8, np.float64)
        check(lib().lbm_diagnostics(self.h, _ptr(out)))
        return out

    def run_until_converged(self, max_steps, check_every, tol):
        """Step until the residual sum|rho_k - rho_(k-1)| <= tol (checked every
        check_every steps) or max_steps; returns (steps taken, residual)."""
        n, r = C.c_int(), C.c_double()
        check(lib().lbm_run_until_converged(self.h, int(max_steps), int(check_every), float(tol),
                                            C.byref(n), C.byref(r)))
        return n.value, r.value

    def set_solid_mask(self, mask):
        """Solid voxels [ny][nz][nx] (nonzero = solid), or None; restarts
        the domain from its initial state."""
        if mask is None:
            check(lib().lbm_set_solid_mask(self.h, None))
            return
        m = np.ascontiguousarray(np.asarray(mask) != 0, dtype=np.uint8)
        assert m.shape == (self.iv.ny, self.iv.nz, self.iv.nx), m.shape
        check(lib().lbm_set_solid_mask(self.h, _ptr(m)))

    def save_checkpoint(self, path):
        check(lib().lbm_save_checkpoint(self.h, os.fsencode(path)))

    def load_checkpoint(self, path):
        """Restart from a checkpoint file; returns the step count stored in it."""
        k = C.c_longlong()
        check(lib().lbm_load_checkpoint(self.h, os.fsencode(path), C.byref(k)))
        return k.value

    def snapshot(self):
        check(lib().lbm_snapshot(self.h))

    def save_snapshot(self, savetype, directory=None, index=0):
        d = None if directory is None else os.fsencode(directory)
        check(lib().lbm_save_snapshot(self.h, int(savetype), d, int(index)))

    def save_file(self, savetype, directory=None, index=0):
        d = None if directory is None else os.fsencode(directory)
        check(lib().lbm_save_file(self.h, int(savetype), d, int(index)))

    def device_bytes(self):
        b = C.c_size_t()
        check(lib().lbm_device_bytes(self.h, C.byref(b)))
        return b.value

    def last_run_ms(self):
        v = C.c_float()
        check(lib().lbm_last_run_ms(self.h, C.byref(v)))
        return v.value


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def write_vtu(path, den, ux, uy, uz, node_type):
    """kernel.cu's BINARYTYPE file from host fields shaped [ny][nz][nx]."""
    ny, nz, nx = np.shape(den)
    f = [_f32(a) for a in (den, ux, uy, uz)]
    t = np.ascontiguousarray(node_type, dtype=np.int32)
    check(lib().lbm_write_vtu(os.fsencode(path), nx, ny, nz, *[_ptr(a) for a in f], _ptr(t)))


def write_csv(result_path, section_path, den, ux, uy, uz):
    """kernel.cu's CSVTYPE files (result.csv, section.csv); a path may be None."""
    ny, nz, nx = np.shape(den)
    f = [_f32(a) for a in (den, ux, uy, uz)]
    rp = None if result_path is None else os.fsencode(result_path)
    sp = None if section_path is None else os.fsencode(section_path)
    check(lib().lbm_write_csv(rp, sp, nx, ny, nz, *[_ptr(a) for a in f]))


def decomposition(iv):
    sl = np.zeros((TILE_NUM, 3, 2), np.int32)
    n = check(lib().lbm_decomposition(C.byref(iv), _ptr(sl)))
    return sl[:n]


def set_move_decomp(slices):
    slices = np.ascontiguousarray(slices, np.int32)
    mv = np.zeros((len(slices), 19), np.int32)
    check(lib().lbm_set_move_decomp(len(slices), _ptr(slices), _ptr(mv)))
    return mv


def inverse_mrt(mat):
    mat = np.ascontiguousarray(mat, np.float32)
    inv = np.zeros((19, 19), np.float32)
    check(lib().lbm_inverse_mrt(_ptr(mat), _ptr(inv)))
    return inv


def d3q19_tables():
    d = np.zeros(57, np.float32)
    o = np.zeros(19, np.int32)
    w = np.zeros(19, np.float32)
    m = np.zeros((19, 19), np.float32)
    lib().lbm_d3q19_tables(_ptr(d), _ptr(o), _ptr(w), _ptr(m))
    return d, o, w, m


class _Member(Domain):
    """View of a batch member through the single-domain calls (owned by the batch)."""

    def __init__(self, handle, inputval):
        self.iv = inputval
        self.h = handle
        self.shape = (inputval.ny, inputval.nz, inputval.nx)

    def close(self):
        self.h = None

    def run(self, nsteps):
        raise RuntimeError("batch members are stepped by Batch.step")


class Batch:
    """Many resident domains stepped together (continuous batching)."""

    def __init__(self, hbm_budget=1 << 30, device=0, chunk_steps=32, block=0,
                 nodes_per_thread=0, ctas_per_sm=0, schedule=2, regs=0, own_set_ctas=0):
        o = BatchOptions()
        lib().lbm_batch_default_options(C.byref(o))
        o.device, o.hbm_budget, o.chunk_steps = device, hbm_budget, chunk_steps
        if block:
            o.block = block
        if nodes_per_thread:
            o.nodes_per_thread = nodes_per_thread
        o.ctas_per_sm = ctas_per_sm
        o.schedule, o.regs, o.own_set_ctas = schedule, regs, own_set_ctas
        h = C.c_void_p()
        check(lib().lbm_batch_create(C.byref(o), C.byref(h)))
        self.h = h
        self.ivs = {}

    def close(self):
        if self.h:
            check(lib().lbm_batch_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, inputval, options=None, steps=0):
        opt = options if options is not None else default_options()
        i = C.c_int()
        check(lib().lbm_batch_add(self.h, C.byref(inputval), C.byref(opt), int(steps),
                                  C.byref(i)))
        self.ivs[i.value] = inputval
        return i.value

    def step(self, steps):
        check(lib().lbm_batch_step(self.h, int(steps)))

    def poll(self, max_ids=4096):
        ids = np.zeros(max_ids, np.int32)
        n = C.c_int()
        check(lib().lbm_batch_poll(self.h, _ptr(ids), max_ids, C.byref(n)))
        return [int(v) for v in ids[:n.value]]

    def member(self, i):
        h = C.c_void_p()
        check(lib().lbm_batch_domain(self.h, int(i), C.byref(h)))
        return _Member(h, self.ivs[i])

    def fetch(self, i):
        """rho, ux, uy, uz [ny][nz][nx] of a member that reached its target,
        without waiting for the chunks queued behind its last one."""
        iv = self.ivs[i]
        out = [np.empty((iv.ny, iv.nz, iv.nx), np.float32) for _ in range(4)]
        check(lib().lbm_batch_fetch(self.h, int(i), *[_ptr(a) for a in out]))
        return tuple(out)

    def remove(self, i):
        check(lib().lbm_batch_remove(self.h, int(i)))
        self.ivs.pop(i, None)

    def sync(self):
        check(lib().lbm_batch_sync(self.h))

    def usage(self):
        u, f, n = C.c_size_t(), C.c_size_t(), C.c_int()
        check(lib().lbm_batch_usage(self.h, C.byref(u), C.byref(f), C.byref(n)))
        return u.value, f.value, n.value

    def autotune(self, trial_steps=32):
        o = BatchOptions()
        check(lib().lbm_batch_autotune(self.h, int(trial_steps), C.byref(o)))
        return dict(block=o.block, nodes_per_thread=o.nodes_per_thread, ctas_per_sm=o.ctas_per_sm,
                    schedule=o.schedule, regs=o.regs, own_set_ctas=o.own_set_ctas)

    def last_step_ms(self):
        ms, lups = C.c_float(), C.c_longlong()
        check(lib().lbm_batch_last_step_ms(self.h, C.byref(ms), C.byref(lups)))
        return ms.value, lups.value


class Server:
    """A request queue over one batch: admission into the HBM pool, one chunk
    of steps per progress() turn, residual checks and early retirement; the
    loop itself is the C++ library's (lbm_server_*)."""

    def __init__(self, hbm_budget=1 << 30, device=0, chunk_steps=32, policy=SERVE_FIFO,
                 check_every=256, backlog_horizon_s=0.0, nominal_mlups=0.0, **batch_kw):
        o = ServerOptions()
        lib().lbm_server_default_options(C.byref(o))
        o.batch.device, o.batch.hbm_budget, o.batch.chunk_steps = device, hbm_budget, chunk_steps
        for k, v in batch_kw.items():
            setattr(o.batch, k, v)
        o.policy, o.check_every = policy, check_every
        o.backlog_horizon_s, o.nominal_mlups = backlog_horizon_s, nominal_mlups
        h = C.c_void_p()
        check(lib().lbm_server_create(C.byref(o), C.byref(h)))
        self.h = h
        self.ivs = {}

    def close(self):
        if self.h:
            check(lib().lbm_server_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, inputval, options=None, steps=1, tol=0.0):
        opt = options if options is not None else default_options()
        i = C.c_int()
        check(lib().lbm_server_submit(self.h, C.byref(inputval), C.byref(opt), int(steps),
                                      float(tol), C.byref(i)))
        self.ivs[i.value] = inputval
        return i.value

    def progress(self):
        n = C.c_int()
        check(lib().lbm_server_progress(self.h, C.byref(n)))
        return n.value

    def wait(self, i):
        check(lib().lbm_server_wait(self.h, int(i)))

    def info(self, i):
        r = ServerRequest()
        check(lib().lbm_server_result(self.h, int(i), None, None, None, None, C.byref(r)))
        return {k: getattr(r, k) for k, _ in ServerRequest._fields_}

    def result(self, i):
        """rho, ux, uy, uz [ny][nz][nx] of a done request."""
        if i not in self.ivs:  # the library reports the unknown id
            check(lib().lbm_server_result(self.h, int(i), None, None, None, None, None))
        iv = self.ivs[i]
        out = [np.empty((iv.ny, iv.nz, iv.nx), np.float32) for _ in range(4)]
        check(lib().lbm_server_result(self.h, int(i), *[_ptr(a) for a in out], None))
        return tuple(out)

    def release(self, i):
        check(lib().lbm_server_release(self.h, int(i)))
        self.ivs.pop(i, None)

    def stats(self):
        st = ServerSummary()
        check(lib().lbm_server_stats(self.h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerSummary._fields_}


def batch_domain_bytes(inputval, options=None):
    opt = options if options is not None else default_options()
    b = C.c_size_t()
    check(lib().lbm_batch_domain_bytes(C.byref(inputval), C.byref(opt), C.byref(b)))
    return b.value
