"""Generate the golden fixtures of tests/golden from the reference itself.

Runs the reference's own lbm_codelets.cpp (compiled from the reference tree
into oracle/_ref/libpoplar_ref.so by oracle/Makefile and driven by
oracle/ref_poplar_emu.cpp) on the cavity cases below and stores the results
as small .npz files.  Needs the reference tree at build time; the fixtures
are committed so that the tests run without it.

    python tests/golden/make_golden.py            # cavity fixtures (CPU)
    python tests/golden/make_golden.py --kernelcu # kernel.cu fixtures (GPU)
    python tests/golden/make_golden.py --savefile # saveFile CSV fixtures (CPU)

Cases
  cavity10_mrtles_cs0   main.cpp:59-85 as shipped: h=10, Re=1000, u_lid=0.1,
                        MRT+LES, m_dSmagorinsky never assigned (= 0),
                        Initialize then 199 steps (main.cpp:287-291)
  cavity10_mrtles_cs01  the same with Cs = 0.1 (LES active)
  cavity16_noise_cs01   16^3, Re=100, Cs=0.1, seeded density noise 1e-6, 50 steps
  kernelcu_srt32        kernel.cu SRT cavity 32^3, tau=0.6, noise 1e-6, 200 steps
  kernelcu_srtles24     kernel.cu SRT+LES cavity 24^3, Re=200, Cs=0.1, 100 steps
  savefile/<nx>x<ny>x<nz>_result.csv, _section.csv
                        the reference's saveFile (kernel.cu:973-1018, host
                        code of the kernel.cu build, no GPU) on the seeded
                        fields of tests/test_output.py:fields()
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import oracle_lib as O  # noqa: E402

pkg = O.pkg


def cavity(n, re=None, tau=None, cs=0.0, mrt=True, les=True):
    return pkg.make_inputval(n, casetype=pkg.CAVITY, re=re, tau=tau, u=0.1, mrt=mrt, les=les,
                             cs=cs, h=n)


OUTDIR = HERE


def save(name, fields, iv, steps, extra=None):
    out = dict(den=fields["den"].astype(np.float32), ux=fields["ux"].astype(np.float32),
               uy=fields["uy"].astype(np.float32), uz=fields["uz"].astype(np.float32),
               steps=np.int32(steps), nx=np.int32(iv.nx), ny=np.int32(iv.ny), nz=np.int32(iv.nz),
               tau=np.float32(iv.m_dTau), cs=np.float32(iv.m_dSmagorinsky),
               u=np.float32(iv.m_dRefVelx), mrt=np.int32(iv.bEnableMRT),
               les=np.int32(iv.bEnableLES))
    if extra:
        out.update(extra)
    path = os.path.join(OUTDIR, name + ".npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def poplar_cases():
    if O.poplar_ref_lib() is None:
        raise SystemExit("oracle/_ref/libpoplar_ref.so missing (needs the reference tree)")
    for name, iv, kind, amp, steps in (
        ("cavity10_mrtles_cs0", cavity(10, re=1000.0, cs=0.0), 0, 0.0, 199),
        ("cavity10_mrtles_cs01", cavity(10, re=1000.0, cs=0.1), 0, 0.0, 199),
        ("cavity16_noise_cs01", cavity(16, re=100.0, cs=0.1), 1, 1e-6, 50),
    ):
        r = O.Run(iv, init_kind=kind, seed=1, amp=amp, which="ref")
        r.step(steps)
        f = r.fields()
        extra = dict(init_kind=np.int32(kind), noise_amp=np.float32(amp), seed=np.int32(1))
        if iv.nx == 10:
            extra["arF"] = f["arF"].astype(np.float32)
            # main.cpp:321-347 prints direction 9 at k=2 for all (j, i)
            extra["printout_dir9_k2"] = f["arF"][:, 2, :, 9].astype(np.float32)
        save(name, f, iv, steps, extra)


def kernelcu_cases():
    for name, iv, steps in (
        ("kernelcu_srt32", cavity(32, tau=0.6, mrt=False, les=False), 200),
        ("kernelcu_srtles24", cavity(24, re=200.0, cs=0.1, mrt=False, les=True), 100),
    ):
        f = O.kernelcu_run(iv, steps, init_kind=1, seed=1, amp=1e-6)
        save(name, f, iv, steps, dict(init_kind=np.int32(1), noise_amp=np.float32(1e-6),
                                      seed=np.int32(1)))


def savefile_cases():
    import shutil
    import tempfile
    from test_output import fields, ref_save
    out = os.path.join(OUTDIR, "savefile")
    os.makedirs(out, exist_ok=True)
    for (nx, ny, nz), seed in (((7, 5, 6), 1), ((52, 4, 51), 2)):
        den, u, t = fields(nx, ny, nz, seed)
        tmp = tempfile.mkdtemp()
        ref_save(tmp, nx, ny, nz, den, u, t, pkg.SAVE_CSV)
        # the 52x4x51 case is kept for its section line only (small files)
        names = ("result.csv", "section.csv") if nx < 49 else ("section.csv",)
        for name in names:
            shutil.copy(os.path.join(tmp, name), os.path.join(out, f"{nx}x{ny}x{nz}_{name}"))
        shutil.rmtree(tmp)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--kernelcu", action="store_true")
    ap.add_argument("--savefile", action="store_true")
    ap.add_argument("--outdir", default=HERE)
    a = ap.parse_args()
    OUTDIR = a.outdir
    os.makedirs(OUTDIR, exist_ok=True)
    if a.kernelcu:
        kernelcu_cases()
    elif a.savefile:
        savefile_cases()
    else:
        poplar_cases()
