#!/usr/bin/env python
"""Throughput of the fused D3Q19 step on B200 (MLUPS and HBM roofline).

Default workload: 256^3 lid-driven cavity, MRT + Smagorinsky LES (Cs=0.1),
Re=5000 (tau = 3*u*N/Re + 0.5 = 0.51536), FP32 populations, seeded density
noise 1e-6, synthetic.  A "step" is one lattice time step over the whole
domain (one fused kernel launch).  Both lattices (2 x 1.27 GB) are far larger
than the 126 MB L2, so no L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun) every rank steps its own 256^3 domain (independent
replicas, no collective on the data path): weak scaling, value = all
lattice updates / max-over-ranks time.

--impl reference times the reference's own CPU implementation of the step
(its lbm_codelets.cpp bodies, built as OpenMP C++ in oracle/_ref) on the host
cores, on rank 0 only.
"""
import argparse
import importlib.util
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
BYTES = {"f32": 4, "f16_shift": 2, "bf16_shift": 2, "f64": 8, "f16_shift_sr": 2,
         "bf16_shift_sr": 2}


def load_package():
    name = "nflow_red_poplar_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(
        name, os.path.join(ROOT, "nflow-red-poplar_b200", "__init__.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


WORKLOADS = {
    # the headline workload: 256^3 lid-driven cavity, MRT + LES, Re 5000
    "cavity256_mrt_les": dict(nx=256, ny=256, nz=256, case="cavity", re=5000.0, u=0.1, cs=0.1,
                              mrt=True, les=True, init=1, amp=1e-6),
    # the small SRT cavity the reference's CPU path runs in seconds
    "cavity64_srt": dict(nx=64, ny=64, nz=64, case="cavity", tau=0.6, u=0.1, cs=0.0, mrt=False,
                         les=False, init=1, amp=1e-6),
    # channel, Re = u_max*ny/nu = 1000 (precision comparison)
    "channel512x128x128_mrt_les": dict(nx=512, ny=128, nz=128, case="channel", re_ch=1000.0,
                                       u=0.05, cs=0.1, mrt=True, les=True, init=2, amp=0.01),
}


def KERNELS(pkg):
    return {"auto": pkg.KERNEL_AUTO, "scalar": pkg.KERNEL_SCALAR, "packed": pkg.KERNEL_PACKED,
            "tma": pkg.KERNEL_TMA, "paired": pkg.KERNEL_PAIRED, "quad": pkg.KERNEL_QUAD}


def make_case(pkg, w, size=None):
    nx, ny, nz = w["nx"], w["ny"], w["nz"]
    if size:
        f = size / nx
        nx, ny, nz = size, max(3, int(ny * f)), max(3, int(nz * f))
    if w["case"] == "cavity":
        if "tau" in w:
            iv = pkg.make_inputval(nx, ny, nz, casetype=pkg.CAVITY, tau=w["tau"], u=w["u"],
                                   mrt=w["mrt"], les=w["les"], cs=w["cs"], h=nx)
        else:
            iv = pkg.make_inputval(nx, ny, nz, casetype=pkg.CAVITY, re=w["re"], u=w["u"],
                                   mrt=w["mrt"], les=w["les"], cs=w["cs"], h=nx)
    else:
        nu = w["u"] * ny / w["re_ch"]
        iv = pkg.make_inputval(nx, ny, nz, casetype=pkg.CHANNEL, tau=3.0 * nu + 0.5, u=w["u"],
                               mrt=w["mrt"], les=w["les"], cs=w["cs"])
    return iv


def max_over_ranks(value, world):
    """max of a float over all ranks (the timing rule: the slowest rank).

    Uses the process group's backend: NCCL on a CUDA tensor for GPU runs,
    gloo on a CPU tensor otherwise."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_mlups(nodes_per_rank, steps, max_ms, world):
    """Whole-job MLUPS of `world` independent replicas (weak scaling): all
    lattice updates over the slowest rank's time."""
    return world * nodes_per_rank * steps / (max_ms / 1e3) / 1e6


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_from_profile(workload, storage, streaming="ab"):
    """dram bytes per launch of the step kernel from the committed ncu summary."""
    kern = "k_aa_step" if streaming == "aa" else "k_step"
    path = os.path.join(ROOT, "profiles", f"{kern}_{storage}_{workload}.txt")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_launch:"):
                return int(float(line.split(":", 1)[1].split()[0]))
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, local_rank):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        ident = str(local_rank)
        if vis:
            ids = [v.strip() for v in vis.split(",") if v.strip()]
            if local_rank < len(ids):
                ident = ids[local_rank]
        q = ("clocks.sm,clocks.max.sm,power.draw,utilization.gpu,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--id={ident}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except Exception:
            self.p.kill()
            out = ""
        rows = []
        for ln in out.splitlines():
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                rows.append(dict(sm=float(parts[0]), smax=float(parts[1]), util=float(parts[3]),
                                 hw=parts[4], hwt=parts[5], swt=parts[6], pc=parts[7]))
            except ValueError:
                continue
        if not rows:
            return None
        load = [r for r in rows if r["util"] > 0] or rows
        reasons = set()
        for r in load:
            for k, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"),
                            ("swt", "sw_thermal_slowdown"), ("pc", "sw_power_cap")):
                if r[k].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in load),
                "sm_max_mhz": max(r["smax"] for r in load), "reasons": sorted(reasons),
                "samples": len(load)}


def cpu_baseline(pkg, w, budget_s=20.0):
    """The reference's own codelets (oracle/_ref) on the host cores, or the
    oracle port if the reference build is absent: one warm-up step, then as
    many full-size steps as fit in the budget."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O

    cores = os.cpu_count() or 1
    which = "ref" if O.poplar_ref_lib() is not None and w["case"] == "cavity" and w["mrt"] else "orc"
    iv = make_case(pkg, w)
    split = max(1, math.ceil(2 * cores / 27))
    r = O.Run(iv, init_kind=w["init"], amp=w["amp"], split=split, threads=cores, which=which)
    t0 = time.perf_counter()
    r.step(1)
    t1 = time.perf_counter()
    per = t1 - t0
    n = max(1, min(50, int(budget_s / max(per, 1e-3))))
    t0 = time.perf_counter()
    r.step(n)
    dt = time.perf_counter() - t0
    r.close()
    cells = iv.nx * iv.ny * iv.nz
    return dict(value=cells * n / dt / 1e6, unit="MLUPS", cores=cores,
                kind="reference" if which == "ref" else "port",
                sample=f"{n} full steps of {iv.nx}x{iv.ny}x{iv.nz} after 1 warm-up step, "
                       f"{27 * split} tiles, {cores} OpenMP threads, {dt:.1f} s")


def run_reference_arm(args, pkg, w):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O

    cores = os.cpu_count() or 1
    which = "ref" if O.poplar_ref_lib() is not None and w["case"] == "cavity" and w["mrt"] else "orc"
    iv = make_case(pkg, w)
    split = max(1, math.ceil(2 * cores / 27))
    r = O.Run(iv, init_kind=w["init"], amp=w["amp"], split=split, threads=cores, which=which)
    t0 = time.perf_counter()
    r.step(1)
    per = time.perf_counter() - t0
    # each step is a bounded sample: the whole run stays within ~2-3 minutes
    total = args.steps + args.warmup
    nz_s = iv.nz
    if per * total > 150.0:
        nz_s = max(4, int(iv.nz * 150.0 / (per * total)))
        r.close()
        iv = pkg.make_inputval(iv.nx, iv.ny, nz_s, casetype=iv.casetype, tau=iv.m_dTau,
                               u=iv.m_dRefVelx, mrt=iv.bEnableMRT, les=iv.bEnableLES,
                               cs=iv.m_dSmagorinsky, h=iv.h)
        r = O.Run(iv, init_kind=w["init"], amp=w["amp"], split=split, threads=cores, which=which)
    if args.warmup:
        r.step(args.warmup)
    t0 = time.perf_counter()
    r.step(args.steps)
    dt = time.perf_counter() - t0
    cells = iv.nx * iv.ny * iv.nz
    v = cells * args.steps / dt / 1e6
    sample = (f"each step one full step of {iv.nx}x{iv.ny}x{iv.nz}"
              + ("" if nz_s == w["nz"] else f" (z cut from {w['nz']} to bound the run)")
              + f", {27 * split} tiles, {cores} OpenMP threads")
    line = {
        "impl": "reference", "metric": "MLUPS", "value": v, "unit": "MLUPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": args.workload, "nx": w["nx"], "ny": w["ny"], "nz": w["nz"],
                   "collision": "MRT" if iv.bEnableMRT else "SRT", "les": bool(iv.bEnableLES),
                   "cs": round(float(iv.m_dSmagorinsky), 6), "tau": round(float(iv.m_dTau), 6),
                   "storage": "f32", "device": "host CPU",
                   "implementation": ("reference lbm_codelets.cpp (OpenMP over the decomposition "
                                      "tiles)" if which == "ref" else "oracle port"),
                   "parallelism": "host threads"},
        "cpu_baseline": {"value": v, "unit": "MLUPS", "cores": cores,
                         "kind": "reference" if which == "ref" else "port", "sample": sample},
        "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# Further forms (run with --report): precision (FP16/BF16 vs FP32 storage on
# the 512x128x128 channel), batched (256 mixed domains) and serving (Poisson
# arrivals).  Each prints one JSON line.
# --------------------------------------------------------------------------
def _enstrophy(ux, uy, uz):
    """0.5 * sum |curl u|^2 over the interior, central differences, FP64.
    Arrays are [y][z][x]."""
    ux, uy, uz = (np.asarray(a, np.float64) for a in (ux, uy, uz))

    def d(a, axis):
        return 0.5 * (np.roll(a, -1, axis) - np.roll(a, 1, axis))
    wx = d(uz, 0) - d(uy, 1)   # dw/dy - dv/dz
    wy = d(ux, 1) - d(uz, 2)   # du/dz - dw/dx
    wz = d(uy, 2) - d(ux, 0)   # dv/dx - du/dy
    w2 = (wx * wx + wy * wy + wz * wz)[1:-1, 1:-1, 1:-1]
    return 0.5 * float(w2.sum())


def precision_c3(pkg, steps, kernel, size=None, warmup=0, re=None):
    """Channel 512x128x128 MRT+LES, parabolic inlet u_max=0.05, outlet rho=1,
    walls, 1 % seeded velocity perturbation, Re = u_max ny / nu = 1000; the
    same run with FP16-shift, BF16-shift and FP32 storage against the FP64
    build of the same kernels.  Errors of rho, u (max over nodes, rms and
    relative L2 norm ||u - u64|| / ||u64||), kinetic energy and enstrophy."""
    import torch
    w = dict(WORKLOADS["channel512x128x128_mrt_les"])
    if re:
        w["re_ch"] = float(re)
    iv = make_case(pkg, w, size)
    out = {"workload": "channel512x128x128_mrt_les", "steps": steps,
           "nx": iv.nx, "ny": iv.ny, "nz": iv.nz, "re": w["re_ch"], "tau": float(iv.m_dTau),
           "data": "synthetic", "forms": {}}

    def run(storage, kern, rounding=0, streaming=None):
        o = pkg.default_options(storage=storage, init_kind=w["init"], noise_amp=w["amp"], seed=1,
                                kernel=kern, rounding=rounding,
                                stream_mode=pkg.STREAM_AB if streaming == "ab" else
                                pkg.STREAM_AA)
        d = pkg.Domain(iv, o)
        d.run(warmup)
        d.sync()
        t0 = time.perf_counter()
        d.run(steps - warmup)
        d.sync()
        dt = time.perf_counter() - t0
        den, ux, uy, uz = d.macroscopic()
        diag = d.diagnostics()
        d.close()
        torch.cuda.synchronize()
        return dict(den=den, ux=ux, uy=uy, uz=uz, ke=float(diag[5]),
                    mlups=iv.nx * iv.ny * iv.nz * (steps - warmup) / dt / 1e6,
                    nonfinite=int(diag[7]))

    ref = run(pkg.STORE_F64, pkg.KERNEL_SCALAR, streaming="ab")
    ens_ref = _enstrophy(ref["ux"], ref["uy"], ref["uz"])
    u2_ref = (ref["ux"].astype(np.float64) ** 2 + ref["uy"].astype(np.float64) ** 2 +
              ref["uz"].astype(np.float64) ** 2)
    umax = float(np.sqrt(u2_ref.max()))
    out["fp64"] = {"MLUPS": ref["mlups"], "kinetic_energy": ref["ke"], "enstrophy": ens_ref,
                   "max_u": umax}
    # every form in the AA scheme (FP32: one node per thread; 16-bit: quad
    # rows), and the 16-bit stochastic-rounding forms also in the pull
    # scheme (paired rows)
    for name, st, rnd, sm in (("f32", pkg.STORE_F32, 0, "aa"),
                              ("f16_shift", pkg.STORE_F16_SHIFT, 0, "aa"),
                              ("bf16_shift", pkg.STORE_BF16_SHIFT, 0, "aa"),
                              ("f16_shift_sr", pkg.STORE_F16_SHIFT, pkg.ROUND_STOCHASTIC, "aa"),
                              ("bf16_shift_sr", pkg.STORE_BF16_SHIFT, pkg.ROUND_STOCHASTIC, "aa"),
                              ("f16_shift_sr_ab", pkg.STORE_F16_SHIFT, pkg.ROUND_STOCHASTIC,
                               "ab"),
                              ("bf16_shift_sr_ab", pkg.STORE_BF16_SHIFT, pkg.ROUND_STOCHASTIC,
                               "ab")):
        r = run(st, kernel, rnd, sm)
        d2 = sum((r[k].astype(np.float64) - ref[k].astype(np.float64)) ** 2
                 for k in ("ux", "uy", "uz"))
        ens = _enstrophy(r["ux"], r["uy"], r["uz"])
        out["forms"][name] = {
            "MLUPS": r["mlups"],
            "rho_max_abs_err": float(np.abs(r["den"].astype(np.float64) - ref["den"]).max()),
            "u_max_err_rel_umax": float(np.sqrt(d2.max())) / umax,
            "u_rms_err_rel_umax": float(np.sqrt(d2.mean())) / umax,
            "u_rel_l2_err": float(np.sqrt(d2.sum() / u2_ref.sum())),
            "kinetic_energy_rel_err": abs(r["ke"] - ref["ke"]) / abs(ref["ke"]),
            "enstrophy_rel_err": abs(ens - ens_ref) / abs(ens_ref),
            "nonfinite_nodes": r["nonfinite"], "streaming": sm}
    f32 = out["forms"]["f32"]["MLUPS"]
    for name in out["forms"]:
        if name != "f32":
            out["forms"][name]["speedup_vs_f32"] = out["forms"][name]["MLUPS"] / f32
    return out


def report_precision(args, pkg):
    """--report precision: precision_c3 with --steps steps as one JSON line."""
    kern = KERNELS(pkg)[args.kernel]
    out = precision_c3(pkg, args.steps, kern, args.size or None, args.warmup, args.re or None)
    out["report"] = "precision"
    print(json.dumps(out), flush=True)


def pattern_ceilings(pkg, n=256, iters=20):
    """MLUPS / GB/s of the bare memory patterns of the step forms on an n^3
    box (lbm_pattern_ceiling): the upper bound of any kernel with that
    memory pattern."""
    out = {}
    for name, pat, st in (
            ("copy_f32", pkg.PATTERN_COPY, pkg.STORE_F32),
            ("copy_f16", pkg.PATTERN_COPY, pkg.STORE_F16_SHIFT),
            ("pull_f32", pkg.PATTERN_PULL, pkg.STORE_F32),
            ("pull_f16", pkg.PATTERN_PULL, pkg.STORE_F16_SHIFT),
            ("pull_paired_f16", pkg.PATTERN_PULL_PAIRED, pkg.STORE_F16_SHIFT),
            ("aa_local_f32", pkg.PATTERN_AA_LOCAL, pkg.STORE_F32),
            ("aa_neighbor_f32", pkg.PATTERN_AA_NEIGHBOR, pkg.STORE_F32),
            ("aa_local_f16", pkg.PATTERN_AA_LOCAL, pkg.STORE_F16_SHIFT),
            ("aa_neighbor_f16", pkg.PATTERN_AA_NEIGHBOR, pkg.STORE_F16_SHIFT),
            ("aa_local_v8_f16", pkg.PATTERN_AA_LOCAL_V8, pkg.STORE_F16_SHIFT),
            ("aa_local_v16_f16", pkg.PATTERN_AA_LOCAL_V16, pkg.STORE_F16_SHIFT),
            ("aa_local_v16_f32", pkg.PATTERN_AA_LOCAL_V16, pkg.STORE_F32),
            ("aa_paired_local_f16", pkg.PATTERN_AA_PAIRED_LOCAL, pkg.STORE_F16_SHIFT),
            ("aa_paired_neighbor_f16", pkg.PATTERN_AA_PAIRED_NEIGHBOR, pkg.STORE_F16_SHIFT),
            ("pull_quad_f16", pkg.PATTERN_PULL_QUAD, pkg.STORE_F16_SHIFT),
            ("aa_quad_local_f16", pkg.PATTERN_AA_QUAD_LOCAL, pkg.STORE_F16_SHIFT),
            ("aa_quad_neighbor_f16", pkg.PATTERN_AA_QUAD_NEIGHBOR, pkg.STORE_F16_SHIFT)):
        m, g = pkg.pattern_ceiling(pat, st, n, iters)
        out[name] = {"MLUPS": round(m, 1), "GB_s": round(g, 1)}
    out["box"] = f"{n}^3, {iters} timed launches after 3, CUDA events"
    return out


def _c4_domains(seed, n, storage):
    """Mixed domains: edge from {32,48,64,96,128}; 50 % cavities e^3 (lid 0.1),
    50 % channels 4e x e x e (u_max 0.05); Re log-uniform in [100, 5000]
    (nu = u e / Re, tau = 3 nu + 0.5); 50 % SRT, 50 % MRT+LES (Cs 0.1)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        e = int(rng.choice([32, 48, 64, 96, 128]))
        cav = bool(rng.random() < 0.5)
        re = float(np.exp(rng.uniform(np.log(100.0), np.log(5000.0))))
        mrt = bool(rng.random() < 0.5)
        out.append(dict(e=e, cavity=cav, re=re, mrt=mrt, storage=storage))
    return out


def _case_iv(pkg, c):
    e = c["e"]
    if c["cavity"]:
        u = 0.1
        tau = 3.0 * u * e / c["re"] + 0.5
        return pkg.make_inputval(e, casetype=pkg.CAVITY, tau=tau, u=u, mrt=c["mrt"], les=c["mrt"],
                                 cs=0.1, h=e), 1, 1e-6
    u = 0.05
    tau = 3.0 * u * e / c["re"] + 0.5
    return (pkg.make_inputval(4 * e, e, e, casetype=pkg.CHANNEL, tau=tau, u=u, mrt=c["mrt"],
                              les=c["mrt"], cs=0.1), pkg.INIT_CHANNEL, 0.01)


def batch_c4(pkg, ndom=256, steps=64, warmup=4, streaming="ab", batch_shape="",
             storages=("f32", "f16_shift")):
    """256 independent domains in one persistent launch per step
    (CUDA-graph chunks, autotuned launch shape) vs each domain launched
    alone, for FP32 and FP16-shift storage; streaming "aa" keeps every
    domain in one lattice (AA pattern), "ab" in two (pull).  Batched MLUPS
    are device time (CUDA events on the batch stream) of `steps` steps;
    alone MLUPS sum the device time of each domain's own `steps` steps."""
    mode = pkg.STREAM_AA if streaming == "aa" else pkg.STREAM_AB
    sid = {"f32": pkg.STORE_F32, "f16_shift": pkg.STORE_F16_SHIFT}
    res = {"domains": ndom, "steps": steps, "data": "synthetic (seeded)",
           "streaming": streaming, "forms": {}}
    for sname in storages:
        st = sid[sname]
        cases = _c4_domains(7, ndom, st)
        ivs = [_case_iv(pkg, c) for c in cases]
        opts = [pkg.default_options(storage=st, init_kind=k, noise_amp=a, seed=i + 1,
                                    stream_mode=mode)
                for i, (iv, k, a) in enumerate(ivs)]
        need = sum(pkg.batch_domain_bytes(iv, o) for (iv, _, _), o in zip(ivs, opts))
        shape = {}
        if batch_shape:  # fixed launch shape, no autotuning (profiling)
            v = [int(x) for x in batch_shape.split(",")]
            shape = dict(schedule=v[0], regs=v[1], block=v[2], nodes_per_thread=v[3])
            if len(v) > 4:
                shape["own_set_ctas"] = v[4]
        b = pkg.Batch(hbm_budget=int(need * 1.02) + (64 << 20), chunk_steps=32, **shape)
        t0 = time.perf_counter()
        for (iv, _, _), o in zip(ivs, opts):
            b.add(iv, o, 10 ** 9)
        b.sync()
        t_admit = time.perf_counter() - t0
        cfg = b.autotune(trial_steps=32) if not shape else dict(shape, fixed=True)
        b.step(warmup)
        b.sync()
        b.step(steps)
        ms, lups = b.last_step_ms()
        nodes = sum(iv.nx * iv.ny * iv.nz for iv, _, _ in ivs)
        batched = lups / (ms * steps / 1e3) / 1e6
        nonfinite = 0
        steps_done = []
        for i in list(b.ivs):
            m = b.member(i)
            nonfinite += int(m.diagnostics()[7] > 0)
            steps_done.append(m.steps())
        b.close()
        # each domain alone (same kernels, one launch per step, graph chunks)
        t_alone = 0.0
        nonfinite_alone = 0
        for ((iv, _, _), o), sd in zip(zip(ivs, opts), steps_done):
            d = pkg.Domain(iv, o)
            d.run(warmup)
            d.run(steps)
            t_alone += d.last_run_ms() * steps / 1e3
            # the same step count as in the batch (autotuner trials included)
            d.run(max(0, sd - warmup - steps))
            nonfinite_alone += int(d.diagnostics()[7] > 0)
            d.close()
        alone = nodes * steps / t_alone / 1e6
        bpl = 2 * 19 * BYTES[sname]
        peak, _ = measured_peak()
        res["forms"][sname] = {"batched_MLUPS": batched, "alone_MLUPS": alone,
                               "batched_over_alone": batched / alone, "nodes": nodes,
                               "pool_GB": need / 1e9, "admit_s": t_admit, "autotuned": cfg,
                               "batched_GB_s": batched * 1e6 * bpl / 1e9,
                               "batched_frac_of_hbm": batched * 1e6 * bpl / 1e9 / peak,
                               "domains_nonfinite": nonfinite,
                               "domains_nonfinite_alone": nonfinite_alone}
    return res


def report_batch(args, pkg):
    out = batch_c4(pkg, args.domains, args.steps, args.warmup, args.streaming, args.batch_shape)
    out["report"] = "batch"
    print(json.dumps(out), flush=True)


def serving_c5(pkg, rate=200.0, window=20.0, budget_gb=150.0, policy="shortest", tol=0.0,
               streaming="ab", horizon=0.0, nominal_mlups=30000.0, nreq=20000, seed=11):
    """Seeded Poisson arrivals (mean `rate` req/s, up to `nreq` requests) of
    cavity/channel solves with edge 32-192, steps U[500, 5000], Re
    log-U[100, 5000], FP16-shift or FP32 storage per request (MRT+LES).  This
    function only generates the stream: each request is handed to the
    library's serving loop (pkg.Server: lbm_server_submit at its arrival
    time, lbm_server_progress turns in between), which admits by HBM budget
    (and the backlog horizon), steps by continuous batching, checks residuals
    and retires.  Over a bounded wall-clock window; the time stamps and
    percentiles are the library's (lbm_server_stats)."""
    budget = int(min(150e9, budget_gb * 1e9))
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, nreq))
    reqs = []
    for i in range(nreq):
        e = int(rng.integers(32, 193))
        cav = bool(rng.random() < 0.5)
        re = float(np.exp(rng.uniform(np.log(100.0), np.log(5000.0))))
        steps = int(rng.integers(500, 5001))
        st = pkg.STORE_F16_SHIFT if rng.random() < 0.5 else pkg.STORE_F32
        reqs.append(dict(t=float(arrivals[i]), e=e, cavity=cav, re=re, steps=steps, storage=st))
    mode = pkg.STREAM_AA if streaming == "aa" else pkg.STREAM_AB
    pol = {"fifo": pkg.SERVE_FIFO, "shortest": pkg.SERVE_SHORTEST}[policy]
    srv = pkg.Server(hbm_budget=budget, chunk_steps=32, policy=pol, check_every=256,
                     backlog_horizon_s=horizon, nominal_mlups=nominal_mlups if horizon else 0.0)
    nxt = 0
    t0 = time.perf_counter()
    while True:
        now = time.perf_counter() - t0
        if now > window:
            break
        while nxt < nreq and reqs[nxt]["t"] <= now:
            r = reqs[nxt]
            iv, k, a = _case_iv(pkg, dict(e=r["e"], cavity=r["cavity"], re=r["re"], mrt=True))
            o = pkg.default_options(storage=r["storage"], init_kind=k, noise_amp=a,
                                    seed=nxt + 1, stream_mode=mode)
            srv.submit(iv, o, steps=r["steps"], tol=tol)
            nxt += 1
        st = srv.stats()
        if st["queued"] == 0 and st["resident"] == 0:
            if nxt < nreq:
                time.sleep(max(0.0, min(reqs[nxt]["t"] - now, window - now)))
            continue
        srv.progress()
    st = srv.stats()
    srv.close()
    return {
        "rate_req_s": rate, "window_s": window, "budget_GB": budget / 1e9, "policy": policy,
        "residual_tol": tol, "streaming": streaming,
        "arrived": nxt, "admitted": st["admitted"], "completed": st["completed"],
        "converged_early": st["converged"], "queued_at_end": st["queued"],
        "resident_at_end": st["resident"],
        "tts_p50_s": st["tts_p50_s"], "tts_p99_s": st["tts_p99_s"],
        "service_p50_s": st["service_p50_s"], "service_p99_s": st["service_p99_s"],
        "completed_MLUPS": st["completed_lups"] / st["elapsed_s"] / 1e6,
        "aggregate_MLUPS": st["executed_lups"] / st["elapsed_s"] / 1e6,
        "admission": {"hbm_budget_GB": budget / 1e9, "backlog_horizon_s": horizon,
                      "nominal_MLUPS": nominal_mlups},
        "offered_LUPS": float(np.mean([(r["e"] ** 3 if r["cavity"] else 4 * r["e"] ** 3) *
                                       r["steps"] for r in reqs]) * rate),
        "loop": "lbm_server_* (C++ library); bench.py only generates the arrival stream",
        "data": "synthetic (seeded Poisson stream)"}


def report_serving(args, pkg):
    out = serving_c5(pkg, args.rate, args.window, args.budget_gb, args.policy, args.tol,
                     args.streaming, args.horizon, args.nominal_mlups)
    out["report"] = "serving"
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cavity256_mrt_les", choices=sorted(WORKLOADS))
    ap.add_argument("--storage", default="f32",
                    choices=["f32", "f16_shift", "bf16_shift", "f64", "f16_shift_sr",
                             "bf16_shift_sr"])
    ap.add_argument("--size", type=int, default=0, help="scale the workload to this nx (profiling)")
    ap.add_argument("--kernel", default="auto",
                    choices=["auto", "scalar", "packed", "tma", "paired", "quad"])
    ap.add_argument("--streaming", default=None, choices=["ab", "aa"],
                    help="ab: pull between two lattices; aa: AA pattern in one lattice "
                         "(default: aa for the step line, the 256^3 configuration's scheme; "
                         "ab for the batch and serving reports)")
    ap.add_argument("--report", default="", choices=["", "precision", "batch", "serving"])
    ap.add_argument("--domains", type=int, default=256,
                    help="batch: number of seeded domains (256 = the batched workload; fewer "
                         "for a small profiling case)")
    ap.add_argument("--batch-shape", default="",
                    help="batch: fixed launch shape 'schedule,regs,block,nodes_per_thread"
                         "[,own_set_ctas]' instead of autotuning")
    ap.add_argument("--rate", type=float, default=200.0, help="serving: arrivals per second")
    ap.add_argument("--window", type=float, default=20.0, help="serving: wall-clock window (s)")
    ap.add_argument("--policy", default="shortest", choices=["fifo", "shortest"],
                    help="serving: admission order")
    ap.add_argument("--tol", type=float, default=0.0,
                    help="serving: residual tolerance for early retirement (0 = full budget)")
    ap.add_argument("--c4-steps", type=int, default=64,
                    help="timed steps of the batched comparison the default run reports")
    ap.add_argument("--c5-window", type=float, default=20.0,
                    help="wall-clock window of the serving run the default run reports")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="serving: HBM budget")
    ap.add_argument("--horizon", type=float, default=2.0,
                    help="serving: admit while the resident backlog is below this many seconds "
                         "of work at --nominal-mlups (0 = HBM budget only)")
    ap.add_argument("--nominal-mlups", type=float, default=30000.0,
                    help="serving: throughput the backlog horizon is converted with")
    ap.add_argument("--re", type=float, default=0.0,
                    help="precision report: Reynolds number of the channel (0 = 1000)")
    ap.add_argument("--c3-steps", type=int, default=20000,
                    help="steps of the precision comparison on the 512x128x128 channel that the "
                         "default run reports (precision_c3)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip cpu baseline, e2e and storage forms (profiling runs)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    pkg = load_package()
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        run_reference_arm(args, pkg, w)
        return
    if args.report:
        args.streaming = args.streaming or "ab"
        {"precision": report_precision, "batch": report_batch,
         "serving": report_serving}[args.report](args, pkg)
        return
    args.streaming = args.streaming or "aa"

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    def allmax(v):
        return max_over_ranks(v, world)

    storage_id = {"f32": pkg.STORE_F32, "f16_shift": pkg.STORE_F16_SHIFT,
                  "bf16_shift": pkg.STORE_BF16_SHIFT, "f64": pkg.STORE_F64,
                  "f16_shift_sr": pkg.STORE_F16_SHIFT, "bf16_shift_sr": pkg.STORE_BF16_SHIFT}
    iv = make_case(pkg, w, args.size or None)
    cells = iv.nx * iv.ny * iv.nz
    # a dedicated stream: the library launches on it and the CUDA events
    # below are recorded on it
    stream = torch.cuda.Stream()

    def timed_steps(storage, k, warm, sampler=None, streaming=None):
        streaming = streaming or args.streaming
        opt = pkg.default_options(storage=storage_id[storage], init_kind=w["init"],
                                  noise_amp=w["amp"], seed=1, device=local,
                                  kernel=KERNELS(pkg)[args.kernel],
                                  stream_mode=pkg.STREAM_AA if streaming == "aa"
                                  else pkg.STREAM_AB,
                                  rounding=pkg.ROUND_STOCHASTIC if storage.endswith("_sr")
                                  else pkg.ROUND_NEAREST)
        dom = pkg.Domain(iv, opt)
        dom.set_stream(stream.cuda_stream)
        dom.run(warm)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        dom.run(k)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        return dom, ms

    # pre-roll under the clock sampler so that short timed regions still see
    # several samples under load
    sampler = None if args.no_extras else ClockSampler(local)
    if sampler is not None:
        dom0, _ = timed_steps(args.storage, 800, args.warmup)
        dom0.close()
    dom, ms = timed_steps(args.storage, args.steps, args.warmup)
    clocks = sampler.stop() if sampler is not None else None
    ms_max = allmax(ms)
    per_launch_ms = ms / args.steps
    value = aggregate_mlups(cells, args.steps, ms_max, world)

    peak, peak_kind = measured_peak()
    bpl = 2 * 19 * BYTES[args.storage]
    alg_bytes = bpl * cells
    achieved = alg_bytes / (per_launch_ms / 1e3) / 1e9
    traffic = traffic_from_profile(args.workload, args.storage, args.streaming)

    line = {
        "metric": "MLUPS", "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": args.storage, "data": "synthetic",
        "config": {"workload": args.workload, "nx": iv.nx, "ny": iv.ny, "nz": iv.nz,
                   "collision": "MRT" if iv.bEnableMRT else "SRT", "les": bool(iv.bEnableLES),
                   "cs": round(float(iv.m_dSmagorinsky), 6), "tau": round(float(iv.m_dTau), 6),
                   "storage": args.storage,
                   "streaming": ("AA pattern, one lattice in place, fused boundaries"
                                 if args.streaming == "aa" else "pull A/B, fused boundaries"),
                   "kernel": args.kernel,
                   "l2": "inputs larger than L2 (%d lattice(s) of %.2f GB vs 126 MB)" %
                         (1 if args.streaming == "aa" else 2,
                          19 * BYTES[args.storage] * cells / 1e9),
                   "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": alg_bytes,
                     "bytes_per_lattice_update": bpl},
        "gpu_launches": args.steps,
        "clocks": clocks,
    }

    if not args.no_extras:
        # end to end through the C ABI with pinned host buffers: import the
        # padded arF (H2D), K steps, export the padded arF (D2H)
        shp = (iv.ny + 2, iv.nz + 2, iv.nx + 2, 19)
        h_in = torch.empty(shp, dtype=torch.float32, pin_memory=True).numpy()
        h_out = torch.empty(shp, dtype=torch.float32, pin_memory=True).numpy()
        dom.export_arF(padded=True, out=h_in)
        dom.import_arF(h_in, padded=True)  # warm the staging buffer
        dom.run(args.warmup)
        dom.export_arF(padded=True, out=h_out)
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        dom.import_arF(h_in, padded=True)
        dom.run(args.steps)
        dom.export_arF(padded=True, out=h_out)
        dt = time.perf_counter() - t0
        barrier()
        dt = allmax(dt)
        nbytes = h_in.nbytes
        line["e2e"] = {"value": world * cells * args.steps / dt / 1e6, "unit": "MLUPS",
                       "h2d_bytes_per_step": nbytes / args.steps,
                       "d2h_bytes_per_step": nbytes / args.steps,
                       "what": "lbm_import_arF(padded host AoS) + lbm_run_simulation(K) + "
                               "lbm_export_arF(padded host AoS), pinned host memory"}
        dom.close()
        # storage forms of the same workload (precision form: throughput),
        # each with both streaming schemes (16-bit: paired rows for pull,
        # quad rows for AA)
        forms = {}
        for st in ("f32", "f16_shift", "bf16_shift", "f16_shift_sr", "bf16_shift_sr"):
            f = {}
            for sm in ("ab", "aa"):
                d2, ms2 = timed_steps(st, args.steps, args.warmup, streaming=sm)
                d2.close()
                ms2 = allmax(ms2)
                f[sm + "_MLUPS"] = world * cells * args.steps / (ms2 / 1e3) / 1e6
            best = max(("ab", "aa"), key=lambda k: f.get(k + "_MLUPS", 0.0))
            f["MLUPS"] = f[best + "_MLUPS"]
            f["streaming"] = best
            f["GB_s"] = 2 * 19 * BYTES[st] * f["MLUPS"] * 1e6 / world / 1e9
            forms[st] = f
        for st in forms:
            forms[st]["vs_f32"] = forms[st]["MLUPS"] / forms["f32"]["MLUPS"]
        line["storage_forms"] = forms
        # the same workload with the other streaming scheme
        other = "ab" if args.streaming == "aa" else "aa"
        if args.storage in ("f32", "f16_shift", "bf16_shift"):
            v = forms[args.storage][other + "_MLUPS"]
            line["pull_ab" if other == "ab" else "aa_pattern"] = {
                "value": v, "unit": "MLUPS",
                "roofline_frac": bpl * v * 1e6 / world / 1e9 / peak}
        if rank == 0 and world == 1:
            line["cpu_baseline"] = cpu_baseline(pkg, w)
            line["pattern_ceilings"] = pattern_ceilings(pkg)
            line["precision_c3"] = precision_c3(pkg, args.c3_steps, pkg.KERNEL_AUTO)
            line["batch_c4"] = batch_c4(pkg, 256, args.c4_steps, 4)
            line["serving_c5"] = serving_c5(pkg, 200.0, args.c5_window, 150.0, "shortest",
                                            0.0, "ab", args.horizon, args.nominal_mlups)
    else:
        dom.close()

    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
