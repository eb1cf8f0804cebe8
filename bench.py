"""Benchmark: DOF-stage updates/s of the SDDC drop-in on one or more B200s.

Workload: the cylinder case on the 256 radial x 512 circumferential O-grid
with p = 4 (N = 5; 131,072 cells, 3,276,800 solution points x 9 variables),
RK_S5P3 at CFL 0.3.  One step = one RK3 step = 5 fused stage launches over
every cell.  The state registers (236 MB each) are larger than the 126 MB L2,
so no flush is needed between steps.

Arms:
* default (ours): the mixed form is the headline ``value``; the FP64 and the
  FP64-exact forms are timed on the same workload beside it.  ``e2e`` runs the
  same steps through the C ABI with host buffers (state in, step, state and
  monitor out, every step).  ``cpu_baseline`` times the CPU oracle (the
  restatement of the reference's FP64 path) on the host cores.
* ``--impl reference``: the reference's own path on the CPU, i.e. the oracle
  restatement (the Fortran reference cannot be built here), all host cores.

Blocks beside the headline, at N = 1 only (a flag skips each):
* ``accuracy``: the mixed and FP64 forms against the exact form (bit-equal
  to the oracle) over 2000 steps, per variable, with ||divB|| and mass drift;
* ``ensemble``: 64 cylinder cases of uneven size batched in one launch per
  stage, against one case per context in the mixed form and in both FP64
  forms (the FP64 drop-in), with the batch's error against the exact form;
* ``adjoint``: the discrete adjoint's cost ratio, J, dJ/dMs, dJ/dMA and
  central differences;
* ``output``: the stepping time with restart and Tecplot output every 100
  steps, against none.

Multi-GPU (torchrun): every rank runs an independent replica of the
workload (the drop-in is single-GPU; the case does not shard), timing is the
max over ranks and ``value`` is the total over ranks.
"""
from __future__ import annotations

import argparse
import math
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "DOF-stage updates/s (mixed vs FP64, same B200, rel-L2≤1e-6); adjoint cost ratio"
UNIT = "DOF-stage updates/s"
NR, NT, NPTS = 256, 512, 5
# The configured Ms = 1.5 drives the reference's algorithm (its AV coefficients
# are hard-coded to zero, getrusanov.f90:326,328) to negative pressure after 4
# RK3 steps and a non-finite state after 6 (tests/test_configured_mach.py, on
# the oracle; tests/test_gpu_configured.py follows it on the GPU), so the
# benchmark runs Ms = 0.5
MS, MA = 0.5, 2.0


# Operations (+, -, *, / and square roots) on state-dependent values per
# DOF-stage of RK_S5P3 at N = 5 with mu = eta0 = 0: the reference's FP64
# arithmetic, counted by the oracle's operation-count build on the cylinder
# (1568.1 at 128x256, 1568.6 at 64x128; tests/test_oracle_counts.py pins the
# count).  The FP64 side of the roofline.
REF_OPS_PER_DOF_STAGE_N5 = 1568.0


def bytes_per_dof_stage(N: int) -> float:
    """Algorithmic HBM bytes per DOF-stage: 3*9*8 (state in, state out, RK
    register traffic averaged over RK_S5P3) + 8 (Jac) + 32(N+1)/N (the four
    metric normals at the 2N(N+1) flux points)."""
    return 3 * 9 * 8 + 8 + 32.0 * (N + 1) / N


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def bench_config(c, dt, world: int) -> dict:
    """The workload description both arms print (the same case, built by
    build_case, for the reference arm and ours)."""
    return {
        "workload": f"cylinder O-grid {NR}x{NT}, p={NPTS - 1} (N={NPTS}), RK_S5P3, CFL 0.3",
        "ncell": c.mesh.ncell, "N": c.N, "dof": c.mesh.ncell * c.N * c.N, "dt": dt,
        "physics": f"ideal MHD gamma=5/3, Ms={MS}, MA={MA}, seeded U(+-1e-6) noise",
        "l2": "inputs larger than L2 (236 MB per state register)",
        "parallelism": "replicas" if world > 1 else "single GPU",
    }


def build_case():
    from sddc_b200 import cases, host

    c = cases.cylinder_case(NR, NT, NPTS, ms=MS, ma=MA, seed=0, noise=1e-6)
    t = host.build_tables(c.mesh, c.N)
    Q0 = c.initial_state(t)
    dt = cases.cfl_dt(c.mesh, Q0, c.N, 0.3)
    return c, t, Q0, dt


class Clocks:
    """nvidia-smi clock samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "samples": len(sm), "reasons": sorted(reasons)}


TILES = {}
FIXED_TILE = 0


def time_form(torch, solver_mod, t, ph, Q0, dt, precision, steps, warmup):
    """Device time of `steps` RK3 steps (state resident), CUDA events on the
    context's stream; the tile is picked by the autotuner first (untimed)."""
    from sddc_b200 import autotune

    if FIXED_TILE:
        cpb, times = FIXED_TILE, None
    else:
        cpb, times = autotune.tune(t, ph, Q0, dt, precision)
    TILES[precision] = {"cells_per_cta": cpb, "tuning_s_per_step": times}
    s = solver_mod.Solver(t, ph, precision=precision, cells_per_cta=cpb)
    s.set_state(Q0)
    s.rk_s5p3(dt, warmup)
    stream = torch.cuda.ExternalStream(s.stream_handle())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    s.rk_s5p3(dt, steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    return s, ms


def max_over_ranks(dist, x: float, device: str = "cuda") -> float:
    """The largest of every rank's x (identity on one process).  Every rank
    must call it at the same point: it is a collective."""
    if dist is None:
        return x
    import torch

    m = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(m, op=dist.ReduceOp.MAX)
    return float(m.item())


def run_ours(args):
    import torch

    from sddc_b200 import solver as solver_mod

    rank, world = int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    c, t, Q0, dt = build_case()
    ph = c.physics
    dof = c.mesh.ncell * c.N * c.N
    steps, warm = args.steps, args.warmup

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    if args.only:
        # one form only, no e2e or baselines: the command profiled under ncu
        s, ms = time_form(torch, solver_mod, t, ph, Q0, dt, args.only, steps, warm)
        s.close()
        if rank == 0:
            print(json.dumps({"profile_run": args.only, "steps": steps, "ms_per_step": ms / steps,
                              "dof_stage_per_s": dof * 5 * steps / (ms / 1e3)}))
        if dist:
            dist.destroy_process_group()
        return
    results = {}
    states = {}
    try:
        gpu_index = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        gpu_index = str(local)
    clocks = None
    for prec in ("mixed", "fp64", "fp64_exact"):
        barrier()
        if prec == "mixed":
            with Clocks(gpu_index) as ck:
                s, ms = time_form(torch, solver_mod, t, ph, Q0, dt, prec, steps, warm)
            clocks = ck.summary()
        else:
            s, ms = time_form(torch, solver_mod, t, ph, Q0, dt, prec, steps, warm)
        ms = max_over_ranks(dist, ms)
        results[prec] = ms
        states[prec] = s.state()["Q"]
        s.close()
    barrier()
    # end-to-end through the C ABI with host buffers, every step:
    # state host->device, one RK3 step, state and monitor device->host
    s = solver_mod.Solver(t, ph, precision="mixed", cells_per_cta=TILES["mixed"]["cells_per_cta"])
    q_host =torch.empty(Q0.size, dtype=torch.float64, pin_memory=True).numpy().reshape(Q0.shape, order="F")
    q_host[...] = Q0
    out_host = torch.empty(Q0.size, dtype=torch.float64, pin_memory=True).numpy().reshape(Q0.shape, order="F")
    s.set_state(q_host)
    s.rk_s5p3(dt, 1)
    e2e_steps = max(3, min(steps, 20))
    stream = torch.cuda.ExternalStream(s.stream_handle())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    for _ in range(e2e_steps):
        s.set_state(q_host)
        s.rk_s5p3(dt, 1)
        s.state(out=out_host)
        s.monitor()
        q_host, out_host = out_host, q_host
    e1.record(stream)
    e1.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    s.close()
    e2e_ms = max_over_ranks(dist, e2e_ms)
    if rank != 0:
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    ref = states["fp64_exact"]
    acc = {
        "mixed_vs_fp64_exact_rel_l2": float(np.linalg.norm(states["mixed"] - ref) / np.linalg.norm(ref)),
        "fp64_vs_fp64_exact_rel_l2": float(np.linalg.norm(states["fp64"] - ref) / np.linalg.norm(ref)),
        "after_steps": steps + warm,
        "note": "fp64_exact is bit-equal to the CPU oracle (tests/test_gpu_parity.py, test_gpu_fullsize.py)",
    }
    # the single-GPU diagnostic blocks run at N = 1 only (replicas repeat them)
    single = world == 1
    if args.accuracy_steps and single:
        acc["long_run"] = accuracy_run(solver_mod, t, ph, Q0, dt, dof, args.accuracy_steps)
    units = dof * 5 * steps
    val = {k: world * units / (v / 1e3) for k, v in results.items()}
    peak, peak_kind = measured_peaks()
    bpd = bytes_per_dof_stage(c.N)
    launch_ms = results["mixed"] / (5 * steps)
    achieved = dof * bpd / (launch_ms / 1e3) / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(prof):
        traffic = json.load(open(prof)).get("mixed_n5_bytes_per_launch")
    cpu = cpu_baseline(t, ph, Q0, dt, dof) if not args.no_cpu_baseline and single else None
    e2e_units = dof * 5 * e2e_steps * world
    line = {
        "metric": METRIC,
        "value": val["mixed"],
        "unit": UNIT,
        "n_gpus": world,
        "steps": steps,
        "warmup": warm,
        "ms_per_step": results["mixed"] / steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 flux/f64 state",
        "data": "synthetic",
        "config": bench_config(c, dt, world),
        "tiles": TILES,
        "fp64": {"value": val["fp64"], "ms_per_step": results["fp64"] / steps},
        "fp64_exact": {"value": val["fp64_exact"], "ms_per_step": results["fp64_exact"] / steps},
        "mixed_over_fp64": val["mixed"] / val["fp64"],
        "accuracy": acc,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "traffic_note": "mean DRAM bytes per stage launch over the 5 stages of a step (ncu, "
                                     "profiles/traffic.json); algorithmic bytes per launch: "
                                     f"{dof * bpd:.4g}",
                     "bytes_per_dof_stage": bpd, "kernel": f"stage_kernel<{c.N},{TILES['mixed']['cells_per_cta']},float> (mixed)",
                     "fp64_side": {"ref_ops_per_dof_stage": REF_OPS_PER_DOF_STAGE_N5,
                                   "ref_ops_per_byte": REF_OPS_PER_DOF_STAGE_N5 / bpd,
                                   "fp64_form_ref_ops_per_s": val["fp64"] * REF_OPS_PER_DOF_STAGE_N5,
                                   "fp64_exact_ref_ops_per_s": val["fp64_exact"] * REF_OPS_PER_DOF_STAGE_N5,
                                   "note": "the reference's FP64 +,-,*,/,sqrt per DOF-stage (oracle count); "
                                           "a division or root is one operation here, an FMA sequence on the GPU"}},
        "cpu_baseline": cpu,
        "clocks": clocks,
        "e2e": {"value": e2e_units / (e2e_ms / 1e3), "unit": UNIT,
                "h2d_bytes_per_step": int(Q0.nbytes), "d2h_bytes_per_step": int(Q0.nbytes) + 32,
                "steps": e2e_steps, "path": "sddc_set_state + sddc_rk_step + sddc_get_state + sddc_monitor"},
        "gpu_launches": 5 * steps,
        "ensemble": ensemble_run(torch, gpu_index) if not args.no_ensemble and single else None,
        "adjoint": adjoint_bench(torch, nsteps=args.adjoint_steps, n1=args.adjoint_steps * 5 // 6,
                                 n2=args.adjoint_steps) if args.adjoint_steps and single else None,
        "output": output_bench(torch, solver_mod, c.mesh, t, ph, Q0, dt, TILES["mixed"]["cells_per_cta"])
        if single and not args.no_output else None,
    }
    print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def accuracy_run(solver_mod, t, ph, Q0, dt, dof, nsteps):
    """The mixed and FP64 forms against the FP64-exact form (bit-equal to
    the CPU oracle) after `nsteps` RK3 steps: rel-L2 of each variable, the
    divB L2 norm and the change of the integrated density."""
    out = {}
    for prec in ("fp64_exact", "fp64", "mixed"):
        s = solver_mod.Solver(t, ph, precision=prec, cells_per_cta=TILES.get(prec, {}).get("cells_per_cta", 0))
        s.set_state(Q0)
        m0 = s.monitor()["mass"]
        s.rk_s5p3(dt, nsteps)
        mon = s.monitor()
        out[prec] = (s.state()["Q"], m0, mon)
        s.close()
    ref, m0, mref = out["fp64_exact"]
    res = {"steps": nsteps, "t_end": nsteps * dt, "finite": bool(np.isfinite(ref).all()),
           "divB_l2_fp64_exact": float(np.sqrt(mref["divbsum"] / dof)),
           "mass_change_fp64_exact": (mref["mass"] - m0) / m0}
    names = ["rho", "rhou", "rhov", "rhow", "E", "Bx", "By", "Bz", "psi"]
    for prec in ("fp64", "mixed"):
        q, m0p, mon = out[prec]
        res[prec] = {
            "rel_l2_all": float(np.linalg.norm(q - ref) / np.linalg.norm(ref)),
            "rel_l2_per_var": {n: float(np.linalg.norm(q[k] - ref[k]) / max(np.linalg.norm(ref[k]), 1e-300))
                               for k, n in enumerate(names)},
            "divB_l2": float(np.sqrt(mon["divbsum"] / dof)),
            "mass_change_minus_exact": (mon["mass"] - m0p) / m0p - res["mass_change_fp64_exact"],
        }
    return res


def orszag_tang_run(torch, n=1024, t_end=0.5, chunk=200, max_steps=0, forms=("fp64_exact", "fp64", "mixed")):
    """The Orszag-Tang vortex on a periodic 1024^2 mesh, p = 3, to t = 0.5
    (dt fixed from CFL 0.3 of the initial state): each form from the same
    seeded initial state, its DOF-stage/s (CUDA events on the context's
    stream), and the mixed and FP64 forms' error against the exact FP64 form
    (bit-equal to the CPU oracle) at the end: per-variable rel-L2, ||divB||,
    mass drift.  A form that faults numerically reports the time reached.
    max_steps > 0 stops after that many steps (the short runs profiled under
    ncu); forms selects the forms run."""
    from sddc_b200 import cases, host
    from sddc_b200.solver import NumericalFault, Solver

    c = cases.config3(n)
    t = host.build_tables(c.mesh, c.N)
    Q0 = c.initial_state(t)
    dt = cases.cfl_dt(c.mesh, Q0, c.N)
    nsteps = int(math.ceil(t_end / dt))
    if max_steps:
        nsteps = min(nsteps, max_steps)
    dof = c.mesh.ncell * c.N * c.N
    out, res = {}, {"workload": f"Orszag-Tang {n}x{n} periodic, p=3 (N=4), RK_S5P3, CFL 0.3, t_end={t_end}",
                    "dof": dof, "dt": dt, "steps": nsteps}
    from sddc_b200 import autotune

    for prec in forms:
        cpb, _ = autotune.tune(t, c.physics, Q0, dt, prec, steps=2)
        res.setdefault("cells_per_cta", {})[prec] = cpb
        s = Solver(t, c.physics, precision=prec, cells_per_cta=cpb)
        s.set_state(Q0)
        m0 = s.monitor()["mass"]
        st = torch.cuda.ExternalStream(s.stream_handle())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        done, fault, ms = 0, None, 0.0
        while done < nsteps:
            k = min(chunk, nsteps - done)
            e0.record(st)
            try:
                s.rk_s5p3(dt, k)
            except NumericalFault as e:
                fault = str(e)
                break
            e1.record(st)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
            done += k
        mon = s.monitor() if fault is None else None
        out[prec] = (s.state()["Q"] if fault is None else None, m0, mon)
        res[prec] = {"steps_done": done, "t_reached": done * dt, "fault": fault,
                     "value": dof * 5 * done / (ms / 1e3) if ms > 0 else None, "unit": UNIT}
        s.close()
    ref, m0, mref = out.get("fp64_exact", (None, None, None))
    names = ["rho", "rhou", "rhov", "rhow", "E", "Bx", "By", "Bz", "psi"]
    if ref is not None:
        res["fp64_exact"].update(divB_l2=float(np.sqrt(mref["divbsum"] / dof)),
                                 mass_change=(mref["mass"] - m0) / m0)
        for prec in ("fp64", "mixed"):
            q, m0p, mon = out.get(prec, (None, None, None))
            if q is None:
                continue
            res[prec].update(
                rel_l2_all=float(np.linalg.norm(q - ref) / np.linalg.norm(ref)),
                rel_l2_per_var={nm: float(np.linalg.norm(q[k] - ref[k]) / max(np.linalg.norm(ref[k]), 1e-300))
                                for k, nm in enumerate(names)},
                divB_l2=float(np.sqrt(mon["divbsum"] / dof)),
                mass_change_minus_exact=(mon["mass"] - m0p) / m0p - res["fp64_exact"]["mass_change"])
    return res


def ensemble_run(torch, gpu_index=None, ncase=64, steps=1000, warmup=3, seed=0):
    """64 cylinder cases (p = 3, mixed, sizes uniform over 16x32..128x256,
    per-case CFL time steps), 1000 RK3 steps, in one launch per stage: one
    CTA per tile, and persistent (as many CTAs as are resident, each walking
    the tile table largest case first); against the same cases run one
    after another, each on its own context."""
    from sddc_b200 import autotune, ensemble

    members = ensemble.build_members(ensemble.make_cases(ncase, seed=seed))
    dof_total = sum(m.tables.ncell * m.tables.N ** 2 for m in members)

    def timed(run, stream_handle):
        st = torch.cuda.ExternalStream(stream_handle)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        run()
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3

    # tile for the batch (untimed tuning on the batch itself)
    best, best_t = 4, None
    for cpb in autotune.CANDIDATES:
        b = ensemble.Batch(members, precision="mixed", cells_per_cta=cpb)
        b.reset()
        b.step(2)
        tt = timed(lambda: b.step(3), b.solver.stream_handle())
        if best_t is None or tt < best_t:
            best, best_t = cpb, tt
        b.close()
    launches = {}
    clocks = {}
    for mode in ("per_tile", "persistent"):
        b = ensemble.Batch(members, precision="mixed", cells_per_cta=best, persistent=mode == "persistent")
        b.reset()
        b.step(warmup)
        # the clocks of the batched runs (after the runs before them, a
        # power cap may hold the SM clock below its maximum)
        with Clocks(gpu_index if gpu_index is not None else "0") as ck:
            t = timed(lambda: b.step(steps), b.solver.stream_handle())
        clocks[mode] = ck.summary()
        q = b.solver.state()["Q"]
        launches[mode] = (t, q, bool(np.isfinite(q).all()))
        b.close()
    assert np.array_equal(launches["per_tile"][1], launches["persistent"][1]), "launch modes differ"
    mode_best = min(launches, key=lambda k: launches[k][0])
    t_batch, qb, finite = launches[mode_best]
    from sddc_b200.solver import Solver

    # each case on its own context, one after another: the mixed form, and
    # the FP64 drop-in in both FP64 forms; the exact form's final states (bit
    # for bit the oracle's) are the reference of the batch's accuracy
    t_seq = {"mixed": 0.0, "fp64": 0.0, "fp64_exact": 0.0}
    errs = []
    off = 0
    for m in members:
        nq = m.Q0.size
        for prec in t_seq:
            cpb, _ = autotune.tune(m.tables, m.case.physics, m.Q0, m.dt, prec, steps=2)
            s = Solver(m.tables, m.case.physics, precision=prec, cells_per_cta=cpb)
            s.set_state(m.Q0)
            s.rk_s5p3(m.dt, warmup)
            t_seq[prec] += timed(lambda: s.rk_s5p3(m.dt, steps), s.stream_handle())
            if prec == "fp64_exact":
                ref = s.state()["Q"].ravel(order="F")
                got = qb.ravel(order="F")[off:off + nq]
                errs.append(float(np.linalg.norm(got - ref) / np.linalg.norm(ref)))
            s.close()
        off += nq
    units = dof_total * 5 * steps
    sizes = {}
    for m in members:
        key = f"{m.case.mesh.ncell}"
        sizes[key] = sizes.get(key, 0) + 1
    return {"cases": ncase, "dof_total": dof_total, "cells_by_case_size": sizes, "steps": steps,
            "form": "mixed", "cells_per_cta": best, "finite": finite,
            "batched": {"value": units / t_batch, "unit": UNIT, "s_per_step": t_batch / steps,
                        "launch": mode_best},
            "batched_by_launch": {k: {"value": units / v[0], "unit": UNIT, "s_per_step": v[0] / steps,
                                      "clocks": clocks[k]}
                                  for k, v in launches.items()},
            "sequential": {"value": units / t_seq["mixed"], "unit": UNIT, "s_per_step": t_seq["mixed"] / steps},
            "batched_over_sequential": t_seq["mixed"] / t_batch,
            "fp64_dropin": {f: {"value": units / t_seq[f], "unit": UNIT, "s_per_step": t_seq[f] / steps}
                            for f in ("fp64", "fp64_exact")},
            "batched_mixed_over_fp64_dropin": t_seq["fp64"] / t_batch,
            "batched_mixed_over_fp64_exact_dropin": t_seq["fp64_exact"] / t_batch,
            "batched_mixed_rel_l2_vs_exact": {"max": max(errs), "median": float(np.median(errs)),
                                              "after_steps": warmup + steps,
                                              "note": "per case, against the exact form (bit-equal to the oracle)"}}


def output_bench(torch, solver_mod, mesh, t, ph, Q0, dt, cpb, steps=200, nwrite=100, nre=4):
    """Restart + Tecplot output every nwrite steps (iterations.f90:77-80)
    while stepping: the stepping stream's time with and without output, the
    stream time each write call adds (state snapshot, plot-node kernel) and
    the background writer's wall time for the files."""
    import shutil

    from sddc_b200 import host

    pm = host.plot_mesh(mesh, nre)
    out = tempfile.mkdtemp(prefix="sddc_out_")
    s = solver_mod.Solver(t, ph, precision="mixed", cells_per_cta=cpb)
    s.set_plot(pm)
    stream = torch.cuda.ExternalStream(s.stream_handle())
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def run(with_output):
        s.set_state(Q0)
        s.rk_s5p3(dt, 3)
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        call_ms = []
        e0.record(stream)
        for it in range(1, steps + 1):
            s.rk_s5p3(dt, 1)
            if with_output and (it % nwrite == 1 or it == steps):
                a, b = ev(), ev()
                a.record(stream)
                s.write_restart(os.path.join(out, host.restart_filename(it)), it)
                s.write_tecplot(os.path.join(out, f"TEC{it:07d}.plt"))
                b.record(stream)
                call_ms.append((a, b))
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        w0 = time.perf_counter()
        s.output_wait()
        drain = time.perf_counter() - w0
        return ms, [a.elapsed_time(b) for a, b in call_ms], drain

    # one output first, untimed: the restart snapshot and its pinned buffer
    # are allocated by the first write
    s.set_state(Q0)
    s.write_restart(os.path.join(out, "warm.dat"), 0)
    s.output_wait()
    base_ms, _, _ = run(False)
    t0 = time.perf_counter()
    out_ms, call_ms, drain_s = run(True)
    wall = time.perf_counter() - t0
    # the synchronous alternative: read the state back and write on the host
    w0 = time.perf_counter()
    q = s.state()["Q"]
    host.restart_write(os.path.join(out, "sync.dat"), q, steps, 0.0)
    sync_restart_s = time.perf_counter() - w0
    nfiles = len(call_ms)
    rbytes = os.path.getsize(os.path.join(out, host.restart_filename(steps)))
    tbytes = os.path.getsize(os.path.join(out, f"TEC{steps:07d}.plt"))
    s.close()
    shutil.rmtree(out, ignore_errors=True)
    return {
        "workload": f"{steps} mixed RK_S5P3 steps, restart + Tecplot (nre={nre}) after steps 1, 101, .., {steps}",
        "plotnodes": pm.plotnodes, "plotcells": pm.plotcells,
        "restart_bytes": rbytes, "tecplot_bytes": tbytes, "outputs": nfiles,
        "ms_per_step_no_output": base_ms / steps, "ms_per_step_with_output": out_ms / steps,
        "stream_ms_per_output": statistics.median(call_ms) if call_ms else None,
        "writer_drain_s_after_last_step": drain_s, "wall_s_with_output": wall,
        "sync_restart_write_s": sync_restart_s,
        "note": "write calls queue a snapshot on the stepping stream; the files are written by a host thread",
    }


def adjoint_bench(torch, nsteps=1200, n1=1000, n2=1200, fd_dirs=16, seed=0):
    """The discrete adjoint on the cylinder 128x256, p = 3 (N = 4): the
    objective is C_D averaged over the states after n1..n2 exact RK_S5P3
    steps; gradients with respect to the initial field and the inflow sonic
    and Alfven Mach numbers (through the boundary states and the initial
    field), checkpoints every 20 steps.  Cost ratio: the reverse sweep
    (recomputation and VJPs) over the plain exact forward run of the same
    steps, both timed with CUDA events on the context's stream.  Central
    differences of J in 16 seeded random directions of the initial field, at
    h = 1e-6 and at h = 1e-9, check the gradient."""
    from sddc_b200 import adjoint, cases, host, mesh
    from sddc_b200.solver import Solver

    m = mesh.cylinder_ogrid(128, 256)
    t = host.build_tables(m, 4)
    ph = cases.cylinder_physics(ms=MS, ma=MA)
    Q0 = cases.freestream_state(ph, 4, m.ncell, noise=1e-6, seed=seed)
    dt = cases.cfl_dt(m, Q0, 4)
    from sddc_b200 import autotune

    cpb, _ = autotune.tune(t, ph, Q0, dt, "fp64_exact", steps=2)
    free0 = torch.cuda.mem_get_info()[0]
    prob = adjoint.DragLiftProblem(t, dt, nsteps, n1, n2, w_drag=1.0, w_lift=0.0, checkpoint_every=20,
                                   cells_per_cta=cpb)
    fs0 = np.array([ph.rinf, ph.pinf, ph.uinf, ph.vinf, ph.bxinf, ph.byinf])
    s = prob.solver(fs0)
    ctx_bytes = free0 - torch.cuda.mem_get_info()[0]
    # the plain forward of the same steps (exact form, graph-launched)
    s.set_state(Q0)
    s.rk_s5p3(dt, 3)
    s.set_state(Q0)
    st = torch.cuda.ExternalStream(s.stream_handle())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    s.rk_s5p3(dt, nsteps)
    e1.record(st)
    e1.synchronize()
    fwd_ms = e0.elapsed_time(e1)
    # objective and gradients (Mach numbers through the boundary states and Q0)
    fs_base = adjoint.cylinder_freestream(MS, MA).numpy()
    Qbase = adjoint.freestream_field(torch.from_numpy(fs_base), 4, m.ncell).numpy()
    noise = Q0 - Qbase
    J, dms, dma, qbar = adjoint.mach_gradients(prob, MS, MA, noise)
    r = prob.last
    # central differences of J in random directions of the initial field; the
    # running max behind c_h makes J piecewise smooth, so a step that moves
    # the argmax of one of the thousands of raised maxima averages the
    # one-sided slopes: both a 1e-6 and a 1e-9 step are reported
    rng = np.random.default_rng(seed + 1)
    scale = np.abs(Q0).max(axis=(1, 2, 3), keepdims=True)
    errs = {1e-6: [], 1e-9: []}
    Q0b = Qbase + noise
    for _ in range(fd_dirs):
        V = rng.uniform(-1.0, 1.0, Q0.shape) * scale
        ad = float(np.vdot(qbar, V))
        for h in errs:
            jp = prob.run(Q0b + h * V, fs_base, gradient=False)["J"]
            jm = prob.run(Q0b - h * V, fs_base, gradient=False)["J"]
            errs[h].append(abs((jp - jm) / (2 * h) - ad) / max(abs(ad), 1e-300))
    prob.close()
    stats = r["stats"]
    return {"workload": "cylinder O-grid 128x256, p=3 (N=4), exact FP64 RK_S5P3, "
                        f"{nsteps} steps, J = mean C_D over steps {n1}..{n2}, checkpoints every 20 steps",
            "cells_per_cta": cpb,
            "J": J, "cd": r["cd"], "cl": r["cl"], "dJ_dMs": dms, "dJ_dMA": dma,
            "dJ_dQ0_l2": float(np.linalg.norm(qbar)),
            "forward_ms": fwd_ms, "recording_forward_ms": stats["forward_ms"], "reverse_ms": stats["reverse_ms"],
            "cost_ratio": stats["reverse_ms"] / fwd_ms,
            "cost_ratio_with_recording": (stats["forward_ms"] + stats["reverse_ms"]) / fwd_ms,
            "owner_stages": stats["owner_stages"], "stages": 5 * nsteps,
            "device_bytes_run": stats["device_bytes"], "device_bytes_context": int(ctx_bytes),
            "fd_check": {"directions": fd_dirs,
                         "h1e-6": {"max_rel_err": max(errs[1e-6]), "median_rel_err": float(np.median(errs[1e-6]))}
                         if fd_dirs else None,
                         "h1e-9": {"max_rel_err": max(errs[1e-9]), "median_rel_err": float(np.median(errs[1e-9]))}
                         if fd_dirs else None,
                         "bar_1e-6_at_h1e-6_met": bool(fd_dirs and max(errs[1e-6]) <= 1e-6),
                         "note": "the 1e-6 bar at h=1e-6 is not met: J is piecewise smooth (the running-max "
                                 "c_h has thousands of kinks over 1200 steps) and a 1e-6 step moves argmaxes, so "
                                 "the quotient averages one-sided slopes; at h=1e-9 the rounding of J over "
                                 "1200 steps limits the quotient to ~1e-5. The adjoint equals the complex-step "
                                 "FP64 tangent to 1e-12"},
            "tangent_check": "tests/test_gpu_adjoint.py: adjoint = complex-step FP64 CPU tangent to 1e-12 "
                             "(24x48 cells, 200 steps, 600 raised maxima)"}


def cpu_baseline(t, ph, Q0, dt, dof, steps=1):
    """The CPU oracle on all host threads, one RK3 step of the full mesh."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import sddc_oracle as O

    n = os.cpu_count() or 1
    O.set_threads(n)
    o = O.Oracle(t, ph)
    o.set_state(Q0)
    t0 = time.perf_counter()
    o.rk_s5p3(dt, steps)
    el = time.perf_counter() - t0
    return {"value": dof * 5 * steps / el, "unit": UNIT, "cores": n, "kind": "port",
            "sample": f"{steps} RK3 step of the {NR}x{NT} p={NPTS - 1} cylinder ({dof} DOF, 5 stages), FP64"}


def run_reference(args):
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    c, t, Q0, dt = build_case()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import sddc_oracle as O

    n = os.cpu_count() or 1
    O.set_threads(n)
    o = O.Oracle(t, c.physics)
    o.set_state(Q0)
    dof = c.mesh.ncell * c.N * c.N
    o.rk_s5p3(dt, args.warmup)
    t0 = time.perf_counter()
    o.rk_s5p3(dt, args.steps)
    el = time.perf_counter() - t0
    v = dof * 5 * args.steps / el
    line = {
        "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": int(os.environ.get("WORLD_SIZE", 1)),
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": bench_config(c, dt, int(os.environ.get("WORLD_SIZE", 1))),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": n, "kind": "port",
                         "sample": f"{args.steps} full RK3 steps of the {NR}x{NT} p={NPTS - 1} cylinder; the "
                                   "Fortran reference cannot be compiled here (no Fortran compiler), so this is "
                                   "the C restatement of its FP64 path, OpenMP over cells and faces"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 64-case batched ensemble block")
    ap.add_argument("--no-output", action="store_true", help="skip the restart / Tecplot output block")
    ap.add_argument("--only", choices=["mixed", "fp64", "fp64_exact"], default=None,
                    help="time one form only (the command used for ncu captures)")
    ap.add_argument("--accuracy-steps", type=int, default=2000,
                    help="RK3 steps of the mixed/FP64 vs FP64-exact comparison (0: skip)")
    ap.add_argument("--adjoint-steps", type=int, default=1200,
                    help="RK3 steps of the discrete-adjoint block (objective over the last sixth; 0: skip)")
    ap.add_argument("--tile", type=int, default=0, choices=[0, 4, 6, 8, 16],
                    help="cells per CTA; 0 lets the autotuner choose")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="run only the discrete-adjoint block (with --adjoint-steps; the command profiled under ncu)")
    ap.add_argument("--orszag-tang", action="store_true",
                    help="run only the Orszag-Tang 1024^2 comparison (mixed/FP64 vs exact FP64 to t = 0.5)")
    ap.add_argument("--ot-n", type=int, default=1024, help="Orszag-Tang cells per side")
    ap.add_argument("--ot-steps", type=int, default=0, help="Orszag-Tang: stop after this many steps (0: t = 0.5)")
    args = ap.parse_args()
    global FIXED_TILE
    FIXED_TILE = args.tile
    if args.warmup < 3:
        args.warmup = 3
    if args.adjoint_only:
        import torch

        n = args.adjoint_steps
        print(json.dumps({"adjoint": adjoint_bench(torch, nsteps=n, n1=n * 5 // 6, n2=n,
                                                   fd_dirs=16 if n >= 100 else 0)}))
        return
    if args.orszag_tang:
        import torch

        forms = (args.only,) if args.only else ("fp64_exact", "fp64", "mixed")
        print(json.dumps({"orszag_tang": orszag_tang_run(torch, n=args.ot_n, max_steps=args.ot_steps, forms=forms)}))
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
