#!/usr/bin/env python
"""bench.py -- particle-steps/s of the polar-grid particle-mesh step on B200.

Default workload (N=1): the 3D cylindrical polar grid of 128 rings x 256
spokes x 125 planes (dz = 0.04, harmonics m = 0..16, Plummer softening 0.1,
log-spaced rings r = 0.05 .. 5) with 10M particles of a seeded
Kuzmin-Toomre disc (sech^2 layer z0 = 0.1), dt = 0.02.  One step = findf
(azimuthal + doubled-grid vertical transforms, radial contraction with the
resident Green table, synthesis, polcat) + the fused particle pass (grdacc,
stpgrp, new cell keys) + the row radix sort + the deterministic deposit
(massgn, scaled).  Inputs are larger than L2 (particle store 240 MB, Green
table 411 MB per step), so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the CPU restatement of the same step (the oracle
port; the Fortran reference cannot be built without a Fortran compiler) on the host
cores, on a bounded sample of the same workload.
Under torchrun (N > 1) each rank owns its own particles (weak scaling) and
the ranks sum their mass grids every step (the reference's MPI design).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s on 1 B200 vs plain FP64 GPU path at force rel-err <=1e-5"
UNIT = "particle-steps/s"

WORKLOADS = {
    # 3D polar grid, the configuration the metric is quoted on
    "polar3d-128x256x125-10M": dict(ndim=3, nr=128, na=256, ngz=125, dzg=0.04, ng=17,
                                    softl=0.1, n=10_000_000, dt=0.02, z0=0.1, disk_rmax=4.8,
                                    r0=0.05, r1=5.0),
    # 2D polar grid, the CPU-runnable case
    "polar2d-64x128-100k": dict(ndim=2, nr=64, na=128, ngz=1, dzg=0.0, ng=9, softl=0.1,
                                n=100_000, dt=0.025, z0=0.0, disk_rmax=4.8, r0=0.05, r1=5.0),
}
DEFAULT = "polar3d-128x256x125-10M"


def make_cfg(w, precision):
    from galaxy_b200 import make_config, GX_RMAP_LOG
    a = float(np.log(w["r1"] / w["r0"]) / (w["nr"] - 1))
    return make_config(w["ndim"], w["nr"], w["na"], ngz=w["ngz"], dzg=w["dzg"], ng=w["ng"],
                       rmap=GX_RMAP_LOG, rmap_a=a, rmap_r0=w["r0"], softl=w["softl"], tsoft=1,
                       precision=precision)


def make_ic(w, n, seed):
    from galaxy_b200.disk import kt_disk
    return kt_disk(n, seed=seed, rmax=w["disk_rmax"], ndim=w["ndim"], z0=w["z0"] or 0.1,
                   dt=w["dt"])


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clock, power and clock-event reasons of one GPU, polled through
    NVML from a thread every ~0.5 ms (the timed region of the step is only
    tens of milliseconds long).  Start it before the warm-up; window(t0, t1)
    marks the timed region in host time, and summary() reports the samples
    inside it (the whole sampling span if none fell inside)."""

    def __init__(self, index, period=0.0005):
        self.index = index
        self.period = period
        self.rows = []      # (t, sm_mhz, reasons bitmask, power W)
        self.max_mhz = None
        self.stop = threading.Event()
        self.t = None
        self.win = None
        self.err = None

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            self.nv = nv
            self.h = nv.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM))
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
        except Exception as e:  # no NVML: the line says the clocks were unsampled
            self.err = str(e)
        return self

    def _poll(self):
        nv, h = self.nv, self.h
        while not self.stop.is_set():
            try:
                t = time.perf_counter()
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                self.rows.append((t, float(sm), int(rs), pw))
            except Exception as e:
                self.err = str(e)
                return
            time.sleep(self.period)

    def window(self, t0, t1):
        self.win = (t0, t1)

    def __exit__(self, *a):
        self.stop.set()
        if self.t is not None:
            self.t.join(timeout=5)

    def summary(self):
        rows = self.rows
        where = "timed region"
        if self.win is not None:
            inside = [r for r in rows if self.win[0] <= r[0] <= self.win[1]]
            if inside:
                rows = inside
            else:
                where = "warm-up and timed region (no sample inside the timed region)"
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"],
                    "error": self.err}
        nv = self.nv
        names = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                 "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                 "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                 "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        reasons = sorted({k for r in rows for k, b in names.items() if r[2] & b})
        return {"sm_mhz": float(np.median([r[1] for r in rows])), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(rows), "power_w_max": max(r[3] for r in rows),
                "where": where, "how": "NVML polled every 0.5 ms from a host thread"}


# ---------------------------------------------------------------------------
# algorithmic bytes per launch of each phase (the figures roofline.achieved
# is built from; the per-step formula of the measurement plan is
# N * 2 * 2d * 4 + Green bytes + mesh * 4 * (2 + 2F))
def green_counts(cfg, geo, lpot=False):
    """(m, kz) pairs the radial contraction reads for each field type."""
    act = [m for m in range(geo.ng) if not geo.lg[m]]
    nkz = geo.ngz + 1 if cfg.ndim == 3 else 1
    n_fr = len(act) * nkz
    n_ft = len([m for m in act if 1 <= m <= min(geo.ng, geo.mmax - 1) - 1]) * nkz
    n_fz = len(act) * (geo.ngz - 1) if cfg.ndim == 3 else 0
    return n_fr + n_ft + n_fz + (n_fr if lpot else 0), len(act), nkz


def phase_bytes(cfg, geo, n):
    d = cfg.ndim
    mesh = geo.mesh
    npairs, nact, nkz = green_counts(cfg, geo)
    spec = nact * nkz * geo.nr * 16
    ntypes = 3 if d == 3 else 2
    return {
        # the fused pass: phase space read + written, the mass it deposits
        "push": n * 2 * 2 * d * 4 + mesh * 4,
        "conv": npairs * geo.nr * geo.nr * 4 + spec * (1 + ntypes),
        "syn": spec * ntypes + mesh * 16,                 # spectra in, float4 field out
        "fwd": mesh * 4 + spec,
        "sort": (geo.nr * geo.ngz + 1) * 4 * 6,           # the plan: row tables in and out
        "combine": mesh * (8 + 4),                        # fixed-point mass in, mass out
    }


def step_bytes(cfg, geo, n):
    npairs, _, _ = green_counts(cfg, geo)
    nf = cfg.ndim  # Cartesian field components
    return n * 2 * 2 * cfg.ndim * 4 + npairs * geo.nr * geo.nr * 4 + geo.mesh * 4 * (2 + 2 * nf)


KERNEL_OF = {"push": "k_push_bkt", "conv": "k_conv_bulk", "syn": "k_synz_tc+k_synaz",
             "fwd": "k_fwd_az+k_fwd_z", "sort": "k_bk_plan", "combine": "k_mass_convert"}


def ncu_traffic(workload):
    """dram bytes per launch per kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return {}
    d = json.load(open(p))
    return d.get(workload, {})


# ---------------------------------------------------------------------------
def run_ours(args, w, rank, world, comm):
    import galaxy_b200 as gb
    from galaxy_b200 import Galaxy, GX_PREC_MIXED, GX_PREC_FP64
    n = args.n or w["n"]
    rec, pm = make_ic(w, n, seed=12345 + rank)
    out = {}
    cfg = make_cfg(w, GX_PREC_MIXED)
    cfg.flags = args.flags
    cfg.pmass = pm / world          # the ranks' discs together carry the disc mass
    cfg.device = int(os.environ.get("LOCAL_RANK", 0))
    gal = Galaxy(cfg)
    geo = gal.geo
    if comm is not None:
        comm.attach(gal)
    gal.greenm()
    gal.loadup(rec)
    gal.masset()
    gal.findf(True)
    gal.tmcent(True)
    with ClockSampler(cfg.device) as clk:
        gal.step(args.warmup)
        if comm is not None:
            comm.barrier()
        t0 = time.perf_counter()
        gal.step(args.steps)
        clk.window(t0, time.perf_counter())
    ms = gal.last_step_ms()
    launches = gal.last_launch_count()
    ms_max = comm.max(ms) if comm is not None else ms
    out["ms_total"] = ms_max
    out["ms_per_step"] = ms_max / args.steps
    out["value"] = n * world * args.steps / (ms_max * 1e-3)
    out["gpu_launches"] = launches
    out["clocks"] = clk.summary()
    # phase timing pass (separate from the timed region)
    gal.set_profile(True)
    kp = 3
    gal.step(kp)
    ph = gal.phase_ms()
    gal.set_profile(False)
    pb = phase_bytes(cfg, geo, n)
    peak, src = peaks()
    traffic = ncu_traffic(args.workload)
    phases = {}
    for k, (t, c) in ph.items():
        per = t / max(c, 1)
        gbs = pb.get(k, 0) / (per * 1e-3) / 1e9 if per > 0 else 0.0
        phases[k] = {"ms": round(per, 4), "GB_s": round(gbs, 1)}
    top = max(ph, key=lambda k: ph[k][0])
    per = ph[top][0] / max(ph[top][1], 1)
    ach = pb[top] / (per * 1e-3) / 1e9
    tr = traffic.get(KERNEL_OF.get(top, top))
    out["roofline"] = {"kernel": KERNEL_OF.get(top, top), "bound": "hbm",
                       "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                       "frac": round(ach / peak, 4), "traffic": tr,
                       "algorithmic_bytes": pb[top], "peak_source": src}
    sb = step_bytes(cfg, geo, n)
    out["step_roofline"] = {"bytes": sb, "achieved": round(sb / (out["ms_per_step"] * 1e-3) / 1e9, 1),
                            "frac": round(sb / (out["ms_per_step"] * 1e-3) / 1e9 / peak, 4)}
    out["phases"] = phases
    # the same step with the compensated position update (GX_FLAG_COMPENSATED)
    if rank == 0 and world == 1 and not args.no_fp64:
        from galaxy_b200 import GX_FLAG_COMPENSATED
        cfgc = make_cfg(w, GX_PREC_MIXED)
        cfgc.pmass = pm / world
        cfgc.device = cfg.device
        cfgc.flags = GX_FLAG_COMPENSATED
        with Galaxy(cfgc) as gc:
            gc.greenm()
            gc.loadup(rec)
            gc.masset()
            gc.findf(False)
            gc.tmcent(True)
            gc.step(3)
            kc = 50
            gc.step(kc)
            msc = gc.last_step_ms() / kc
        out["compensated_step"] = {"ms_per_step": round(msc, 4), "value": n / (msc * 1e-3),
                                   "what": "GX_FLAG_COMPENSATED: two-float positions (+12 B per particle per step)"}
    # accuracy at the evolved state of this run (after the warm-up, timed and
    # profile steps): the mixed path's forces and potentials against the plain
    # FP64 GPU path on the same positions and against the FP64 oracle on a
    # sample of them; then the FP64 path's own step rate
    if rank == 0 and world == 1 and not args.no_fp64:
        out.update(accuracy_and_fp64_rate(args, w, gal, cfg, pm))
    gal.close()
    return out, rec, pm, cfg


def accuracy_and_fp64_rate(args, w, gal, cfg, pm, n_sample=200_000, k64=20):
    """Force and potential relative errors of the mixed path at the current
    state of gal (L2 over particles): against the plain FP64 GPU path on all
    particles, and against the FP64 oracle (masset, findf, grdacc on the
    host) on a seeded sample of them.  Then the FP64 path's step rate over
    k64 single steps after two warm-up steps: median and spread."""
    from galaxy_b200 import Galaxy, GX_PREC_FP64
    from oracle import oracle as ox
    gal.findf(True)
    a32, p32 = gal.getacc()
    pos = gal.unload()
    n = pos.shape[0]
    cfg64 = make_cfg(w, GX_PREC_FP64)
    cfg64.pmass = cfg.pmass
    cfg64.device = cfg.device
    res = {}
    with Galaxy(cfg64) as g64:
        g64.greenm()
        g64.loadup(pos)
        g64.masset()
        g64.findf(True)
        a64, p64 = g64.getacc()
        g64.step(2)
        ms = []
        for _ in range(k64):
            g64.step(1)
            ms.append(g64.last_step_ms())
    ms = np.array(ms)
    med = float(np.median(ms))
    res["fp64_path"] = {"value": n * 1e3 / med, "ms_per_step": round(med, 3),
                        "ms_min": round(float(ms.min()), 3), "ms_max": round(float(ms.max()), 3),
                        "steps": k64, "what": "median of single timed steps (CUDA events) after "
                                              "2 warm-up steps; solve scratch allocated once per context"}
    res["force_rel_err"] = float(np.linalg.norm(a32 - a64) / np.linalg.norm(a64))
    res["pot_rel_err"] = float(np.linalg.norm(p32 - p64) / np.linalg.norm(p64))
    # the FP64 oracle on a sample
    ox.set_threads(os.cpu_count() or 1)
    t0 = time.perf_counter()
    c_or = make_cfg(w, GX_PREC_FP64)
    c_or.pmass = cfg.pmass
    G = ox.green(c_or, 64)
    pos64 = pos.astype(np.float64)
    mass, jrk = ox.masset(c_or, pos64, prec=64)
    f = ox.findf(c_or, G, mass, lpot=True, jrk=jrk, prec=64, polar=False)
    idx = np.sort(np.random.default_rng(4321).choice(n, size=min(n, n_sample), replace=False))
    acc_o, pot_o = ox.grdacc(c_or, pos64[idx], f, phys=True, prec=64)
    ox.set_threads(1)
    def rel(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))
    res["vs_oracle"] = {
        "sample": f"{idx.size} of {n} particles (seed 4321) at the evolved state, "
                  f"oracle masset/findf over all {n}",
        "force_rel_err_vs_oracle": rel(a32[idx].astype(np.float64), acc_o),
        "pot_rel_err_vs_oracle": rel(p32[idx].astype(np.float64), pot_o),
        "fp64_path_force_rel_err_vs_oracle": rel(a64[idx].astype(np.float64), acc_o),
        "fp64_path_pot_rel_err_vs_oracle": rel(p64[idx].astype(np.float64), pot_o),
        "oracle_s": round(time.perf_counter() - t0, 1)}
    return res


def run_e2e(args, w, rec, pm, cfg_dev):
    """The same run through the public C ABI with host buffers: loadup (H2D
    from pinned host memory), masset, K steps, unload (D2H), wall clock."""
    from galaxy_b200 import Galaxy, GX_PREC_MIXED, PinnedArray
    pin_in = PinnedArray(rec.shape)
    pin_in.array[...] = rec
    pin_out = PinnedArray(rec.shape)
    src, dst, pinned = pin_in.ptr, pin_out.ptr, True
    cfg = make_cfg(w, GX_PREC_MIXED)
    cfg.pmass = pm
    cfg.device = cfg_dev
    gal = Galaxy(cfg)
    gal.greenm()
    gal.loadup_ptr(src, rec.shape[0])      # warm the allocation
    gal.masset()
    gal.step(1)
    n = rec.shape[0]
    # best of two runs: the wall clock includes host-side copies whose speed
    # varies with what else the host is doing
    best = None
    for _ in range(2):
        t0 = time.perf_counter()
        gal.loadup_ptr(src, n)
        gal.masset()
        gal.step(args.steps)
        gal.unload_ptr(dst)
        t1 = time.perf_counter()
        best = (t1 - t0) if best is None else min(best, t1 - t0)
    ok = bool(np.isfinite(pin_out.array).all())
    gal.close()
    pin_in.free()
    pin_out.free()
    nbytes = n * rec.shape[1] * 4
    return {"value": n * args.steps / best, "unit": UNIT,
            "h2d_bytes_per_step": nbytes / args.steps, "d2h_bytes_per_step": nbytes / args.steps,
            "pinned": pinned, "finite": ok, "what": "gx_loadup + gx_masset + gx_step(K) + gx_unload, wall clock, best of 2"}


def run_small2d(steps=200):
    """The 2D CPU-runnable configuration (64 x 128 log rings x spokes, m =
    0..8, 100k particles, dt = 0.025) stepped on the GPU: the size of the
    reference's own p2d examples, where a step takes tens of microseconds."""
    from galaxy_b200 import Galaxy, GX_PREC_MIXED
    w = WORKLOADS["polar2d-64x128-100k"]
    rec, pm = make_ic(w, w["n"], seed=12345)
    cfg = make_cfg(w, GX_PREC_MIXED)
    cfg.pmass = pm
    with Galaxy(cfg) as gal:
        gal.greenm()
        gal.loadup(rec)
        gal.masset()
        gal.findf(True)
        gal.tmcent(True)
        gal.step(10)
        gal.step(steps)
        ms = gal.last_step_ms() / steps
    return {"workload": "polar2d-64x128-100k", "steps": steps, "ms_per_step": round(ms, 4),
            "particle_steps_per_s": w["n"] / (ms * 1e-3)}


def run_sfp(n=20_000_000, reps=5):
    """The SFP coefficient sum of the 2D Abel-Jacobi configuration: 20M
    particles of an exponential disc (scale 1, truncated at r = 6), k = 7,
    n = 0..19, m = 0..8, maxr = 6; tensor-core path against the FP64 path."""
    from galaxy_b200.disk import exp_disk
    from galaxy_b200.sfp import Basis, Sfp
    basis = Basis.from_json(os.path.join(ROOT, "tests", "golden", "aj07.json"), maxm=8, maxn=19)
    pos = exp_disk(n, seed=12345)
    out = {"workload": f"sfp2d-aj07-m0..8-n0..19-{n // 1_000_000}M"}
    with Sfp(basis, 6.0) as s:
        s.load(pos)
        s.sum(1.0 / n, 0)
        t = []
        for _ in range(reps):
            c32 = s.sum(1.0 / n, 0)
            t.append(s.last_ms()[0])
        c64 = s.sum(1.0 / n, 1)
        t64 = s.last_ms()[0]
        s.sum(1.0 / n, 2)
        t5 = []
        for _ in range(reps):
            c5 = s.sum(1.0 / n, 2)
            t5.append(s.last_ms()[0])
        # the SFP-driven time loop (sum + force + kick/drift per step, one
        # host round trip per step for the coefficients), wall clock
        s.step(2, 0.01, pmass=1.0 / n)
        t0 = time.perf_counter()
        s.step(10, 0.01, pmass=1.0 / n)
        step_ms = (time.perf_counter() - t0) * 1e3 / 10
    ms = float(np.median(t))
    peak, src = peaks()
    nbytes = n * 8
    out.update({"ms": round(ms, 4), "particles_per_s": n / (ms * 1e-3),
                "ms_fp64_path": round(t64, 3), "speedup_vs_fp64_path": round(t64 / ms, 2),
                "coeff_rel_err_vs_fp64": float(np.linalg.norm(c32 - c64) / np.linalg.norm(c64)),
                "tcgen05_path": {"ms": round(float(np.median(t5)), 4),
                                 "coeff_rel_err_vs_fp64": float(np.linalg.norm(c5 - c64) / np.linalg.norm(c64)),
                                 "what": "tcgen05.mma M=128 N=48 K=16 per 16 particles, FP16 hi/lo operands MN-major in shared memory, TMEM accumulator"},
                "sfp_step": {"ms_per_step": round(step_ms, 4), "particle_steps_per_s": n / (step_ms * 1e-3),
                             "what": "gx_sfp_step: coefficients (mma.sync path), force and leapfrog per step, wall clock"},
                "hbm_GB_s": round(nbytes / (ms * 1e-3) / 1e9, 1),
                "hbm_frac": round(nbytes / (ms * 1e-3) / 1e9 / peak, 4),
                "useful_tflops": round(2 * n * 340 / (ms * 1e-3) / 1e12, 3)})
    return out


def run_ensemble(ndisc=64, steps=1000, loop_steps=20, seed=12345):
    """Batched ensemble: ndisc seeded Kuzmin-Toomre discs (seeds 0..ndisc-1),
    particle counts log-uniform in [2e4, 2e6], each on its own 64 x 128 2D
    grid (log rings 0.05..5, m = 0..8, Plummer 0.1), dt = 0.025; one
    persistent launch per step under a CUDA graph after the autotuner.
    Against the plain per-run loop (one single-disc context per disc, the
    same arithmetic), timed over loop_steps steps per disc."""
    from galaxy_b200 import Galaxy, make_config, GX_RMAP_LOG
    from galaxy_b200.disk import kt_disk
    from galaxy_b200.ensemble import Ensemble
    rng = np.random.default_rng(seed)
    counts = np.round(np.exp(rng.uniform(np.log(2e4), np.log(2e6), ndisc))).astype(np.int64)

    def cfg():
        return make_config(2, 64, 128, ng=9, rmap=GX_RMAP_LOG, rmap_a=float(np.log(100.0) / 63),
                           rmap_r0=0.05, softl=0.1, tsoft=1, pmass=1.0)
    recs, pms = [], []
    for d in range(ndisc):
        r, pm = kt_disk(int(counts[d]), seed=d, rmax=4.8, ndim=2, dt=0.025)
        recs.append(r.astype(np.float32))
        pms.append(pm)
    ntot = int(counts.sum())
    ens = Ensemble(cfg(), recs, np.array(pms, np.float32), max_steps=loop_steps + 16 + steps)
    threads, chunk = ens.tune()
    ens.step(loop_steps)
    p_ens = ens.unload()
    ens.step(16)
    ens.step(steps)
    ms, launches = ens.last_ms()
    conf = ens.config()
    a2 = ens.a2()
    ens.close()
    # plain per-run loop
    t_loop = 0.0
    err = 0.0
    for d in range(ndisc):
        c = cfg()
        c.pmass = float(pms[d])
        with Galaxy(c) as gal:
            gal.greenm()
            gal.loadup(recs[d])
            gal.masset()
            gal.step(loop_steps)
            t_loop += gal.last_step_ms()
            pos = gal.unload()
        ref = pos[:, :2].astype(np.float64)
        err = max(err, float(np.abs(p_ens[d][:, :2] - ref).max() / np.abs(ref).max()))
    rate = ntot * steps / (ms * 1e-3)
    rate_loop = ntot * loop_steps / (t_loop * 1e-3)
    # algorithmic bytes of one ensemble step: every particle's phase space read
    # and written (2 x 2 x 2 x 4 B) and each disc's mass and (fx, fy) grids
    # written and read once (64 x 128 cells x 4 B x (2 + 2 x 2))
    peak, src = peaks()
    eb = 32 * ntot + ndisc * 64 * 128 * 4 * 6
    ach = eb / (ms / steps * 1e-3) / 1e9
    return {"workload": f"ensemble2d-{ndisc}x64x128-{ntot}", "discs": ndisc, "particles": ntot,
            "steps": steps, "ms_per_step": round(ms / steps, 4), "particle_steps_per_s": rate,
            "launches_per_step": launches / steps, "cuda_graph": conf["graph"],
            "tuned": {"threads": threads, "chunk": chunk, "ctas": conf["grid"]},
            "per_run_loop": {"particle_steps_per_s": rate_loop, "steps": loop_steps,
                             "ms_per_step_all_discs": round(t_loop / loop_steps, 4)},
            "speedup_vs_per_run_loop": round(rate / rate_loop, 2),
            "max_pos_rel_diff_vs_per_run_loop": err,
            "a2_final_abs_mean": float(np.abs(a2[-1]).mean()),
            "roofline": {"kernel": "k_ens_step", "bound": "hbm", "achieved": round(ach, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(ach / peak, 4), "algorithmic_bytes": eb,
                         "peak_source": src}}


def run_adjoint(n=1_000_000, steps=400, ckpt=50, n_check=20_000, steps_check=50):
    """Differentiable 2D PM: n particles of a seeded Kuzmin-Toomre disc in a
    cored isothermal halo (r_c = 1, v0 = 0.7), 128 x 256 grid (log rings
    0.05..5, m = 0..8, Plummer 0.1), dt = 0.025, steps leapfrog steps;
    gradient of |A2(t_final)| by the adjoint with checkpoints every ckpt
    steps, against the forward run alone.  Accuracy on a companion case
    (n_check particles, steps_check steps) against the FP64 oracle gradient."""
    from galaxy_b200 import Galaxy, make_config, GX_RMAP_LOG
    from galaxy_b200.disk import kt_disk
    dt, v0, rc = 0.025, 0.7, 1.0

    def cfg(pm):
        return make_config(2, 128, 256, ng=9, rmap=GX_RMAP_LOG, rmap_a=float(np.log(100.0) / 127),
                           rmap_r0=0.05, softl=0.1, tsoft=1, pmass=pm, halo=1,
                           halo_v2=v0 * v0 * dt * dt, halo_rc=rc)
    rec, pm = kt_disk(n, seed=12345, rmax=4.8, ndim=2, dt=dt, halo_v2=v0 * v0, halo_rc=rc)
    with Galaxy(cfg(pm)) as gal:
        gal.greenm()
        gal.loadup(rec)
        gal.masset()
        gal.step(3)
        gal.loadup(rec)
        gal.masset()
        gal.step(steps)
        t_fwd = gal.last_step_ms()
        gal.loadup(rec)
        gal.masset()
        J, grad, dth, drift = gal.adjoint(steps, ckpt)
        t_adj = gal.last_step_ms()
    out = {"workload": f"adjoint2d-128x256-{n}-{steps}steps", "particles": n, "steps": steps,
           "checkpoint_every": ckpt, "J_abs_A2": J, "ms_adjoint": round(t_adj, 2),
           "ms_forward_only": round(t_fwd, 2), "adjoint_over_forward": round(t_adj / t_fwd, 2),
           "gradient_particle_steps_per_s": n * steps / (t_adj * 1e-3),
           "dJ_drc": float(dth[0]), "dJ_dv0": float(dth[1] * 2 * v0 * dt * dt),
           "reversal_drift_max_abs": drift, "grad_finite": bool(np.isfinite(grad).all())}
    # accuracy on the companion case
    try:
        sys.path.insert(0, ROOT)
        from oracle import oracle as ox
        r2, pm2 = kt_disk(n_check, seed=777, rmax=4.8, ndim=2, dt=dt, halo_v2=v0 * v0, halo_rc=rc)
        c2 = cfg(pm2)
        ox.set_threads(os.cpu_count() or 1)
        J_ref, g_ref, th_ref = ox.adj_gradient(c2, ox.green(c2, 64), r2.astype(np.float64), steps_check)
        with Galaxy(c2) as gal:
            gal.greenm()
            gal.loadup(r2)
            gal.masset()
            J2, g2, th2, _ = gal.adjoint(steps_check, ckpt)
        out["check"] = {"particles": n_check, "steps": steps_check,
                        "J_rel_err_vs_fp64": abs(J2 - J_ref) / J_ref,
                        "grad_rel_err_vs_fp64": float(np.linalg.norm(g2 - g_ref) / np.linalg.norm(g_ref)),
                        "dtheta_rel_err_vs_fp64": [float(abs(a - b) / abs(b)) for a, b in zip(th2, th_ref)]}
    except Exception as e:  # the oracle is test infrastructure: report, do not fail
        out["check"] = {"error": str(e)}
    return out


def cpu_rate(w, rec, pm, steps, warmup, threads):
    """CPU restatement of the step (the oracle's FP32 mirror of the
    reference routines) on the host cores, over ALL particles of the
    workload: per step findf on the full grid, then the particle loop
    (grdacc, stpgrp, weight, massgn, scaled) over every particle.  The Green
    table is built once beforehand and timed separately, as the reference
    builds it once per run.  Returns a dict."""
    from oracle import oracle as ox
    from galaxy_b200 import GX_PREC_MIXED
    ox.set_threads(threads)
    cfg = make_cfg(w, GX_PREC_MIXED)
    cfg.pmass = pm
    n = rec.shape[0]
    t0 = time.perf_counter()
    G = ox.green(cfg, 32)
    t_green = time.perf_counter() - t0
    pos = np.array(rec, dtype=np.float32, copy=True, order="C")
    mass, jrk = ox.masset(cfg, pos, prec=32)
    times = []
    for s in range(warmup + steps):
        t0 = time.perf_counter()
        f = ox.findf(cfg, G, mass, lpot=False, jrk=jrk, prec=32, polar=False)
        mass, jrk = ox.particle_pass(cfg, pos, f, prec=32)
        if s >= warmup:
            times.append(time.perf_counter() - t0)
    ox.set_threads(1)
    t_tot = float(np.sum(times))
    return {"value": n * steps / t_tot, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": (f"{steps} full steps (after {warmup} untimed) of all {n} particles on the "
                       f"{w['nr']}x{w['na']}x{w['ngz']} grid: findf + the particle loop "
                       f"(grdacc, stpgrp, weight, massgn); step times "
                       f"{min(times):.3f}..{max(times):.3f} s; Green table built separately "
                       f"in {t_green:.1f} s"),
            "t_step_s": t_tot / steps, "steps_timed": len(times)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT, choices=sorted(WORKLOADS))
    ap.add_argument("--n", type=int, default=0, help="particles per GPU (default: workload)")
    ap.add_argument("--flags", type=int, default=0,
                    help="context flags GX_FLAG_* of the timed context (e.g. 8: the sorted deposit)")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-sfp", action="store_true")
    ap.add_argument("--no-ens", action="store_true")
    ap.add_argument("--no-adj", action="store_true")
    ap.add_argument("--sfp-only", action="store_true",
                    help="run only the SFP coefficient sum and print its JSON (profiling)")
    ap.add_argument("--sfp-n", type=int, default=20_000_000, help="particles of the SFP sum")
    ap.add_argument("--ens-only", action="store_true",
                    help="run only the batched ensemble and print its JSON (profiling)")
    ap.add_argument("--ens-steps", type=int, default=1000, help="steps of the batched ensemble")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.sfp_only:
        print(json.dumps(run_sfp(args.sfp_n)))
        return
    if args.ens_only:
        print(json.dumps(run_ensemble(steps=args.ens_steps)))
        return
    w = WORKLOADS[args.workload]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    n = args.n or w["n"]
    wcfg = {"workload": args.workload, "grid": [w["nr"], w["na"], w["ngz"]],
            "harmonics": f"0..{w['ng'] - 1}", "particles_per_gpu": n, "dt": w["dt"],
            "softening": w["softl"], "rings": f"log-spaced {w['r0']}..{w['r1']}",
            "l2": "inputs larger than L2 (no flush)"}
    if args.flags:
        wcfg["flags"] = args.flags
    if args.impl == "reference":
        if rank != 0:
            return
        rec, pm = make_ic(w, n, seed=12345)
        threads = os.cpu_count() or 1
        r = cpu_rate(w, rec, pm, args.steps, args.warmup, threads)
        line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["t_step_s"] * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic", "config": wcfg, "impl": "reference",
                "cpu_baseline": {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0},
                "note": "CPU restatement of the reference step (Fortran reference not buildable "
                        "here: no Fortran compiler)"}
        print(json.dumps(line))
        return
    comm = None
    if world > 1:
        import torch
        import torch.distributed as dist
        import datetime
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        from galaxy_b200.dist import RankComm
        comm = RankComm()
    out, rec, pm, cfg = run_ours(args, w, rank, world, comm)
    if comm is not None:
        comm.barrier()
    if rank == 0:
        e2e = run_e2e(args, w, rec, pm, cfg.device) if world == 1 else None
        small2d = run_small2d() if world == 1 else None
        sfp = run_sfp() if (world == 1 and not args.no_sfp) else None
        ens = run_ensemble() if (world == 1 and not args.no_ens) else None
        adj = run_adjoint() if (world == 1 and not args.no_adj) else None
        cpu = None
        if world == 1 and not args.no_cpu:
            cpu = cpu_rate(w, rec, pm, 3, 1, os.cpu_count() or 1)
            cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        line = {"metric": METRIC, "value": out["value"], "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": out["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic", "config": wcfg,
                "roofline": out["roofline"], "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": out["gpu_launches"], "clocks": out["clocks"],
                "fp64_path": out.get("fp64_path"),
                "speedup_vs_fp64_path": (round(out["value"] / out["fp64_path"]["value"], 2)
                                         if out.get("fp64_path") else None),
                "force_rel_err": out.get("force_rel_err"),
                "pot_rel_err": out.get("pot_rel_err"),
                "accuracy_vs_oracle": out.get("vs_oracle"),
                "compensated_step": out.get("compensated_step"),
                "step_roofline": out["step_roofline"], "phases": out["phases"], "small2d": small2d, "sfp": sfp,
                "ensemble": ens, "adjoint": adj}
        print(json.dumps(line))
    if comm is not None:
        comm.dist.destroy_process_group()


if __name__ == "__main__":
    main()
