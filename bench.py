#!/usr/bin/env python
"""Throughput of the RK3 fractional-step core on one vortex ring.

Workload (the configuration the headline metric is quoted on): a Gaussian-core
vortex ring (R = 1, sigma = 0.2, Gamma = 1, z0 = 3, seeded noise 1e-4) on the
cylindrical staggered grid Nr x Ntheta x Nz = 256 x 128 x 512, r in [0, 4],
z in [0, 12], Re = 3000, dt = 5e-4, free slip at r = 4 (slip = 1), the
reference's z boundaries (wall + convective outflow) and the discrete theta
wavenumber in the Poisson solve (max |div u| at round-off), with 1,048,576
tracer particles uniform in area over r in [0.3, 1.7], z in [2, 4] (seed 0).
One step = one RK3 time step: the particle advance (iter_part, nsubdt Euler
substeps) and the three field substeps.  FP64.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs one independent replica per GPU (a single ring does not shard at
this size); value = cells x steps of all ranks / max-over-ranks time.
--impl reference times the CPU restatement of the same path (OpenMP over all
host cores) on the same configuration.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-RK3-steps/s at 256×128×512, mixed vs FP64 on B200 at max|div u|≤1e-9"
UNIT = "Mcell-RK3-steps/s"
NTH, NR, NZ = 128, 256, 512
RMAX, ZMAX, DT, RE, SLIP = 4.0, 12.0, 5e-4, 3000.0, 1.0
NPART, PART_CLASS, PART_MODE = 1048576, 8, 1  # tracers (u_p = u(x_p)), class 8: nsubdt 5
PART_R, PART_Z = (0.3, 1.7), (2.0, 4.0)
WORKLOAD = ("vortex ring, Nr x Ntheta x Nz = 256 x 128 x 512, r<=4, z<=12, Re 3000, dt 5e-4, "
            "free slip, reference z boundaries, discrete theta wavenumber, 1,048,576 tracer "
            "particles (5 Euler substeps per step), FP64")
# algorithmic 8-byte words per interior cell and substep, by kernel family
# (each field word read or written once per logical phase of the reference):
#   A rhs 15 | B theta 6, r 7, z 8 | C divq 4 | D fft 4, dct 4, radial 2 | E upsol 7 | F uppres 9
WORDS = {"rhs": 15, "tsweep": 6, "rsweep": 7, "zsweep": 8, "divq": 4, "fft": 4, "dct": 4,
         "radial": 2, "upsol": 7, "uppres": 9}
WORDS_PER_CELL_STEP = 3 * sum(WORDS.values())  # 198 words = 1584 B


def family_words(fam, prof):
    """Algorithmic words per cell and substep of a timed kernel family, with the
    phases fused into it: the fused right-hand side also solves the theta
    lines (tsweep), the fused pressure update also runs upsol, the forward
    theta transform of the fused substep also takes divq."""
    if fam in SLAB_WORDS:
        return SLAB_WORDS[fam]
    w = WORDS[fam]
    if fam == "rhs" and "tsweep" not in prof:
        w += WORDS["tsweep"]
    if fam == "uppres" and "upsol" not in prof:
        w += WORDS["upsol"]
    if fam == "fft" and "divq" not in prof:
        w += WORDS["divq"]
    return w


# the slab cluster kernels of the fused substep: divq + the forward theta and
# z transforms, and the two inverse transforms
SLAB_WORDS = {"pois_fwd": WORDS["divq"] + (WORDS["fft"] + WORDS["dct"]) // 2,
              "pois_bwd": (WORDS["fft"] + WORDS["dct"]) // 2}


def roofline(prof, steps, ncell, peak, peak_kind, traffic_tab, ms_per_step):
    """Roofline of the dominant field family (largest event time among the
    families with algorithmic words): algorithmic bytes per launch over its
    mean launch time, against the HBM peak; traffic is the family's DRAM
    bytes per launch from the committed ncu summaries; step_frac compares the
    whole step with the HBM floor of all 198 words per cell-step."""
    fam = max((k for k in prof if k in WORDS or k in SLAB_WORDS), key=lambda k: prof[k][0])
    tot_ms, nl = prof[fam]
    per_sub = nl / (3 * steps)  # launches of this family per substep
    bytes_per_launch = family_words(fam, prof) / per_sub * ncell * 8
    achieved = bytes_per_launch / (tot_ms / nl / 1e3) / 1e9
    step_ideal_ms = WORDS_PER_CELL_STEP * 8 * ncell / (peak * 1e9) * 1e3
    return {"bound": "hbm", "kernel": fam, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind,
            "algorithmic_bytes_per_launch": bytes_per_launch, "traffic": traffic_tab.get(fam),
            "traffic_source": traffic_tab.get("_note") if traffic_tab.get(fam) is not None else None,
            "step_frac": step_ideal_ms / ms_per_step}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_table():
    """DRAM bytes per launch from the committed ncu summaries (None if absent)."""
    p = os.path.join(ROOT, "profiles", "dram_traffic.json")
    try:
        return json.load(open(p))
    except Exception:
        return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [l.split(",") for l in open(self.f.name).read().strip().splitlines() if l.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for n, v in zip(names, r[5:9]):
                    if v.strip() == "Active":
                        reasons.add(n)
            except Exception:
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "samples": len(sm),
                "reasons": sorted(reasons)}


def bench_config(world=1):
    """The config dict both arms print (identical keys and values)."""
    return {"workload": WORKLOAD, "grid_nr_ntheta_nz": [NR, NTH, NZ], "particles": NPART,
            "parallelism": "replicas" if world > 1 else "single GPU",
            "l2": "working set ~2.7 GB per replica, every field 137 MB > 126 MB L2"}


def ring_state():
    from vring_b200.synthetic import ring_fields
    return ring_fields(NTH, NR, NZ, RMAX, ZMAX, R=1.0, sigma=0.2, gamma=1.0, z0=3.0, noise=1e-4, seed=0)


def particle_state(n, seed=0):
    """u(n, 117), v(n, 3) of n particles injected at rest (injc_part layout)."""
    import numpy as np
    from vring_b200.synthetic import annulus_particles
    x, y, z = annulus_particles(n, PART_R[0], PART_R[1], PART_Z[0], PART_Z[1], seed=seed)
    u = np.zeros((n, 117), order="F")
    v = np.zeros((n, 3), order="F")
    u[:, 0], u[:, 1], u[:, 2] = x, y, z
    u[:, 6] = u[:, 10] = u[:, 14] = 1.0
    return u, v


def cpu_reference(steps, budget_s, q=None, part_sample=None):
    """The CPU restatement on the same workload, all host threads: full-size
    field steps and the particle advance of all NPART particles (part_sample
    smaller than NPART advances the first part_sample of the same cloud and
    scales their time).  Steps stop early once budget_s has passed.  Returns
    (Mcell-steps/s, steps timed, threads, sample text)."""
    from oracle import oracle as O
    q = q if q is not None else ring_state()
    o = O.Oracle(NTH, NR, NZ, RMAX, ZMAX, DT, RE, 1.0, SLIP, 1, 0, 0)
    for n, a in zip(("q1", "q2", "q3"), q):
        o.field(n)[...] = a
    pu, pv = particle_state(NPART)
    part_sample = NPART if part_sample is None else min(part_sample, NPART)
    op = O.OraclePart(o, PART_CLASS, part_sample, PART_MODE)
    op.u[...] = pu[:part_sample]
    op.v[...] = pv[:part_sample]
    op._s.nlast = op._s.npart = part_sample
    done, t_field, t_part, t0 = 0, 0.0, 0.0, time.perf_counter()
    while done < steps:
        ta = time.perf_counter()
        op.iter_part(1)
        tb = time.perf_counter()
        o.iterate(1)
        tc = time.perf_counter()
        t_part += tb - ta
        t_field += tc - tb
        done += 1
        if tc - t0 > budget_s:
            break
    step_s = (t_field + t_part * NPART / part_sample) / done
    if part_sample == NPART:
        sample = ("%d RK3 steps of the full %dx%dx%d workload with all %d particles (CPU FP64 "
                  "restatement, OpenMP, %d threads)" % (done, NR, NTH, NZ, NPART, os.cpu_count()))
    else:
        sample = ("%d RK3 steps of the full %dx%dx%d field workload plus the particle advance of "
                  "%d of the %d particles scaled by %.3g (CPU FP64 restatement, OpenMP, %d threads)"
                  % (done, NR, NTH, NZ, part_sample, NPART, NPART / part_sample, os.cpu_count()))
    return NTH * NR * NZ / step_s / 1e6, done, os.cpu_count(), sample


def particle_alone_ms(run, stream, e0, e1, pid, mode, order, calls=3):
    """ms per iter_part call of NPART particles of class pid on the run's
    current field, walked in cell order (order 1) or slot order (0); the
    first, untimed call builds the order.  Returns (ms, particle class)."""
    import vring_b200 as V
    run.set_stream(stream.cuda_stream)
    p = V.Part(run, pid, NPART, mode)
    p.set_order(order)
    pu, pv = particle_state(NPART)
    p.set_state(pu, pv, None, NPART)
    del pu, pv
    p.iter_part(1)
    run.sync()
    e0.record(stream)
    for _ in range(calls):
        p.iter_part(1)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / calls
    live = p.counts["npart"]
    nsub = p.nsubdt
    p.close()
    return ms, nsub, live


def inertial_bench(run, stream, e0, e1, calls=3):
    ms, nsub, live = particle_alone_ms(run, stream, e0, e1, 1, 0, 0, calls)
    ms_cell, _, _ = particle_alone_ms(run, stream, e0, e1, 1, 0, 1, calls)
    return {"n": NPART, "mode": "inertial", "class": 1, "nsubdt": nsub, "ms_per_step": ms,
            "value": NPART / (ms / 1e3), "unit": "particle-steps/s (iter_part alone, CUDA events)",
            "substeps_per_s": NPART * nsub / (ms / 1e3), "live_after": live,
            "cell_order_ms_per_step": ms_cell}


def ensemble_bench(local, steps):
    """The ensemble workload (64 rings drawn from seed 1, 65,536 tracers each,
    mixed form): the rings stepped as one ensemble (one graph launch per RK
    substep, sweep tiles from the autotuner) against the same rings stepped
    one context after another.  Host wall time around K steps with the device
    synchronised on both sides (the ensemble's streams are internal)."""
    import vring_b200 as V
    from vring_b200 import ensemble as E
    specs = E.ensemble_specs(64, seed=1)
    rings = [E.make_ring(s, device=local) for s in specs]
    runs = [r for r, _ in rings]
    ncell = sum(E.cells(s) for s in specs)
    # per-context loop (each ring's own substep graphs, rings in turn)
    for r in runs:
        r.iterate(1)
    for r in runs:
        r.sync()
    t0 = time.perf_counter()
    for _ in range(steps):
        for r in runs:
            r.iterate(1)
    for r in runs:
        r.sync()
    t_loop = time.perf_counter() - t0
    ens = V.Ensemble(runs)
    ens.autotune()
    tiles = sorted({(s["nth"], s["nr"], s["nz"]): V.autotune(r) for s, r in zip(specs, runs)}.items())
    ens.iterate(1)
    ens.sync()
    n0 = ens.launch_count
    t0 = time.perf_counter()
    ens.iterate(steps)
    ens.sync()
    t_ens = time.perf_counter() - t0
    kernels = (ens.launch_count - n0) / steps
    maxdiv = max(r.max_divergence() for r in runs)
    out = {"rings": len(specs), "particles_per_ring": E.NPART, "cells": ncell, "steps": steps,
           "precision": "mixed", "value": ncell * steps / t_ens / 1e6, "unit": UNIT,
           "per_context_loop": ncell * steps / t_loop / 1e6,
           "speedup_vs_loop": t_loop / t_ens, "graph_launches_per_step": 3,
           "field_kernels_per_step": kernels, "max_div_u": maxdiv,
           "tiles_r_z_by_grid": [[list(k), list(v)] for k, v in tiles],
           "timing": "host wall time of K steps, device synchronised on both sides"}
    ens.close()
    for r, p in rings:
        p.attach(False)
        p.close()
        r.close()
    return out


def vr2d_bench():
    """The VR2D axisymmetric pressure solve (512 x 1024, tanh-stretched radial
    grid) on one triple of seed 2: iterations and device time of plain CG,
    Jacobi CG, the flexible CG with the Jacobi steps alone and with the
    committed trained network between them, each to 1e-10 from the previous
    step's pressure; and the agreement of each answer with the direct solve."""
    import numpy as np
    from vring_b200 import learned as Lr
    import os as _os
    if not _os.path.exists(Lr.WEIGHTS):
        return None
    k = Lr.make_solver()
    net = Lr.make_net()
    Lr.load_weights(net)
    seq = Lr.RingSequence(2, k.faces, Lr.NZ, Lr.ZMAX)
    f, p_prev, p = Lr.triple(k, seq, 500)
    Lr.compare(k, net, f, x0=p_prev, maxit=200)  # capture the graphs outside the timing
    res = Lr.compare(k, net, f, x0=p_prev)
    out = {"grid_nr_nz": [Lr.NR, Lr.NZ], "tol": 1e-10, "start": "previous step's pressure",
           "params": net.nparams, "pool": net.pool}
    for m, (it, rr, ms, x) in res.items():
        out[m] = {"iterations": it, "relres": rr, "ms": ms,
                  "max_err_vs_direct": float(np.abs(x - p).max() / np.abs(p).max())}
    out["iterations_cg_over_learned"] = res["cg"][0] / max(1, res["learned"][0])
    out["iterations_fcg_jacobi_over_learned"] = res["fcg_jacobi"][0] / max(1, res["learned"][0])
    net.close()
    k.close()
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    q = ring_state()
    # untimed warm-up bounded to one step, then a bounded timed sample
    if args.warmup > 0:
        cpu_reference(1, 1e9, q)
    val, done, cores, sample = cpu_reference(args.steps, 150.0, q)
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(1),
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=30)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision timing")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 64-ring ensemble timing")
    ap.add_argument("--grid", type=int, nargs=3, metavar=("NR", "NTHETA", "NZ"), default=None,
                    help="smaller grid for profiling captures (not the benchmark workload)")
    ap.add_argument("--nparticles", type=int, default=None,
                    help="particle count for profiling captures (not the benchmark workload)")
    ap.add_argument("--no-graphs", action="store_true",
                    help="issue the warm-up substeps launch by launch instead of replaying CUDA graphs "
                         "(the same kernels in the same order; for profiler launch lists)")
    ap.add_argument("--no-vr2d", action="store_true", help="skip the VR2D Krylov solves")
    ap.add_argument("--no-particles-alone", action="store_true",
                    help="skip the particle classes timed alone (inertial class, walk orders)")
    ap.add_argument("--step-only", action="store_true",
                    help="the headline step alone: implies --no-cpu-baseline --no-mixed --no-ensemble "
                         "--no-vr2d --no-particles-alone --e2e-steps 0 (for profiler launch lists)")
    args = ap.parse_args()
    if args.step_only:
        args.no_cpu_baseline = args.no_mixed = args.no_ensemble = True
        args.no_vr2d = args.no_particles_alone = True
        args.e2e_steps = 0
    global NR, NTH, NZ, NPART, WORKLOAD
    if args.grid is not None or args.nparticles is not None:
        if args.grid is not None:
            NR, NTH, NZ = args.grid
        if args.nparticles is not None:
            NPART = args.nparticles
        WORKLOAD = ("REDUCED profiling case (not the benchmark): vortex ring, Nr x Ntheta x Nz = "
                    "%d x %d x %d, %d tracer particles, FP64" % (NR, NTH, NZ, NPART))
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import vring_b200 as V
    from vring_b200 import replicas

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    rep = replicas.init("nccl", timeout_s=300.0)
    rank, world = rep.rank, rep.world
    barrier, max_over_ranks = rep.barrier, rep.max_over_ranks

    q = ring_state()
    run = V.Run(NTH, NR, NZ, RMAX, ZMAX, DT, RE, 1.0, SLIP, theta_wavenumber="modified", device=local)
    for n, a in zip(("q1", "q2", "q3"), q):
        run.set(n, a)
    part = V.Part(run, PART_CLASS, NPART, PART_MODE)
    pu, pv = particle_state(NPART)
    part.set_state(pu, pv, None, NPART)
    del pu, pv
    part.attach(True)  # advanced by vr_iterate before substep 1 of every step
    # a dedicated (non-default) stream shared by the library and the events
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    run.set_stream(stream.cuda_stream)
    if args.no_graphs:
        run.set_graphs(False)
    ncell = NTH * NR * NZ
    # the sweep tile shapes the autotuner picks for this grid (state restored);
    # a profiler launch list (--step-only) keeps the default shapes, so that
    # it holds the step's launches only
    tiles = (0, 0) if args.step_only else V.autotune(run)

    for _ in range(args.warmup):
        run.iterate(1)
    torch.cuda.synchronize()

    # ---- timed region: K steps, inputs resident in HBM ---------------------
    clocks = ClockSampler(local)
    run.profile(True)
    n0 = run.launch_count
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        run.iterate(1)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    launches = run.launch_count - n0
    prof = run.profile_read()
    run.profile(False)
    clk = clocks.stop()
    ms_max = max_over_ranks(ms)
    value = replicas.throughput(ncell * args.steps, world, ms_max / 1e3) / 1e6
    maxdiv = run.max_divergence()
    nonfinite = run.count_nonfinite()
    # the FP64 state after warm-up + timed steps, for the mixed form's per-field error
    ref_fields = None
    if not args.no_mixed:
        ref_fields = {n: run.get(n) for n in ("q1", "q2", "q3", "pres")}
        ref_fields["xyz"] = part.state()[0][:, 0:3].copy()

    # ---- end to end: per step, velocity in from pinned host memory, one step
    # through the C ABI, velocity back to pinned host memory ------------------
    e2e = None
    if args.e2e_steps > 0:
        def pinned(arrs):
            out = [torch.empty(a.size, dtype=torch.float64, pin_memory=True) for a in arrs]
            for p, a in zip(out, arrs):
                p.numpy()[:] = a.ravel(order="F")
            return out

        names = ("q1", "q2", "q3")
        # two input states the host holds ahead of time (the ring and the
        # ring one step later), used alternately, and two result buffers
        run.set_stream(0)
        pin_in = [pinned(q)]
        for p, n in zip(pin_in[0], names):
            run.set_ptr(n, p.data_ptr())
        run.iterate(1)
        pin_in.append(pinned([run.get(n) for n in names]))
        pin_out = [pinned(q), pinned(q)]
        run.sync()
        h2d, d2h = torch.cuda.Stream(), torch.cuda.Stream()

        def e2e_run(round_trip):
            """seconds for args.e2e_steps steps; round_trip: every step's
            input is the previous step's result, in the same host buffers"""
            barrier()
            t0 = time.perf_counter()
            for st in range(args.e2e_steps):
                src = pin_out[0] if round_trip else pin_in[st % 2]
                dst = pin_out[0] if round_trip else pin_out[st % 2]
                for p, n in zip(src, names):
                    run.set_async(n, p.data_ptr(), h2d.cuda_stream)
                run.iterate(1)
                for p, n in zip(dst, names):
                    run.get_async(n, p.data_ptr(), d2h.cuda_stream)
            d2h.synchronize()
            run.sync()
            return max_over_ranks(time.perf_counter() - t0)

        e2e_run(False)  # the staging buffers are allocated on first use
        e2e_s = e2e_run(False)

        def copies_only_s(reps=5):
            """the same bytes each way with no step: both directions at once,
            in 4 pieces per field on the same two streams (the link's floor)"""
            dst = [torch.empty(p.numel(), dtype=torch.float64, device="cuda") for p in pin_in[0]]
            src = [torch.zeros(p.numel(), dtype=torch.float64, device="cuda") for p in pin_in[0]]
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(reps):
                for p_in, p_out, d, sd in zip(pin_in[0], pin_out[1], dst, src):
                    m = p_in.numel()
                    for q_ in range(4):
                        b_, e_ = m * q_ // 4, m * (q_ + 1) // 4
                        with torch.cuda.stream(h2d):
                            d[b_:e_].copy_(p_in[b_:e_], non_blocking=True)
                        with torch.cuda.stream(d2h):
                            p_out[b_:e_].copy_(sd[b_:e_], non_blocking=True)
            torch.cuda.synchronize()
            return (time.perf_counter() - t0) / reps

        copy_s = copies_only_s()
        for p, src in zip(pin_out[0], pin_in[0]):
            p.copy_(src)
        rt_s = e2e_run(True)
        bytes_q = sum(p.numel() for p in pin_in[0]) * 8
        e2e = {"value": replicas.throughput(ncell * args.e2e_steps, world, e2e_s) / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": bytes_q, "d2h_bytes_per_step": bytes_q, "steps": args.e2e_steps,
               "what": "per step: q1,q2,q3 host->device from pinned memory (two input states the "
                       "host holds ahead of time, used alternately), vr_iterate(1) (particles "
                       "included), q1,q2,q3 device->host into pinned result buffers "
                       "(vr_set_field_async / vr_get_field_async, one copy stream per direction, "
                       "through the library's staging buffers, so the copies of neighbouring steps "
                       "overlap the step); pressure, RK history and particle state stay resident; "
                       "host wall clock, device synchronised at both ends",
               "copies_alone": {
                   "ms_per_step": copy_s * 1e3,
                   "value_if_the_step_were_free": replicas.throughput(ncell, world, copy_s) / 1e6,
                   "gb_s_per_direction": bytes_q / copy_s / 1e9,
                   "what": "the same host<->device bytes with no step, both directions at once: the "
                           "PCIe floor of the end-to-end loop"},
               "round_trip": {
                   "value": replicas.throughput(ncell * args.e2e_steps, world, rt_s) / 1e6, "unit": UNIT,
                   "what": "the same, with every step's input the previous step's result in the same "
                           "host buffers: each set waits for the get before it, piece by piece"}}

    # ---- the mixed form on the same workload ---------------------------------
    mixed = None
    if not args.no_mixed:
        rm_ = V.Run(NTH, NR, NZ, RMAX, ZMAX, DT, RE, 1.0, SLIP, precision="mixed",
                    theta_wavenumber="modified", device=local)
        for n, a in zip(("q1", "q2", "q3"), q):
            rm_.set(n, a)
        pm = V.Part(rm_, PART_CLASS, NPART, PART_MODE)
        pu, pv = particle_state(NPART)
        pm.set_state(pu, pv, None, NPART)
        del pu, pv
        pm.attach(True)
        rm_.set_stream(stream.cuda_stream)
        if args.no_graphs:
            rm_.set_graphs(False)
        tiles_m = V.autotune(rm_)
        for _ in range(args.warmup):
            rm_.iterate(1)
        torch.cuda.synchronize()
        clocks_m = ClockSampler(local)
        rm_.profile(True)
        barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            rm_.iterate(1)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms_m = max_over_ranks(e0.elapsed_time(e1))
        prof_m = rm_.profile_read()
        rm_.profile(False)
        clk_m = clocks_m.stop()
        # error per field against the FP64 form after the same steps (the FP64
        # form matches the oracle to 1e-13 per step at this size)
        import numpy as np
        uscale = max(float(np.abs(ref_fields[n]).max()) for n in ("q1", "q2", "q3"))
        field_err = {
            "velocity": max(float(np.abs(rm_.get(n) - ref_fields[n]).max()) for n in ("q1", "q2", "q3")) / uscale,
            "pressure": float(np.abs(rm_.get("pres") - ref_fields["pres"]).max() / np.abs(ref_fields["pres"]).max()),
            "particle_positions": float(np.abs(pm.state()[0][:, 0:3] - ref_fields["xyz"]).max() / ZMAX),
            "after_steps": args.warmup + args.steps,
            "norm": "max |mixed - fp64| / max |fp64| per field; positions over the domain length"}
        max_div_m = rm_.max_divergence()
        # the FP64 form's divergence-free velocity rounded to float: what an
        # FP32-stored velocity would give whatever the solver did
        for n in ("q1", "q2", "q3"):
            rm_.set(n, ref_fields[n].astype(np.float32).astype(np.float64))
        div_f32 = rm_.max_divergence()
        del ref_fields
        value_m = replicas.throughput(ncell * args.steps, world, ms_m / 1e3) / 1e6
        mixed = {"value": value_m, "unit": UNIT, "ms_per_step": ms_m / args.steps,
                 "vs_fp64": value_m / value, "max_div_u": max_div_m,
                 "max_div_u_of_fp64_velocity_rounded_to_fp32": div_f32,
                 "storage": "float: dq, ru, prg, pres; double: q, sweep work arrays, Poisson "
                            "right-hand side, transforms, dph",
                 "tolerance": "max|u_mixed - u_fp64| <= 2e-6 max|u| after 5 steps (tests/test_gpu_mixed.py)",
                 "error_vs_fp64": field_err, "sweep_tiles_r_z": list(tiles_m),
                 "kernel_ms_per_step": {k: v[0] / args.steps for k, v in sorted(prof_m.items())},
                 "clocks": clk_m}
        pm.close()
        rm_.close()

    # the committed DRAM traffic belongs to the benchmark size; a reduced run reports none
    reduced = args.grid is not None or args.nparticles is not None
    # ---- the 64-ring ensemble workload -----------------------------------------
    ensemble = None
    if not args.no_ensemble and not reduced and world == 1:
        ensemble = ensemble_bench(local, 5)
    vr2d = vr2d_bench() if not reduced and world == 1 and not args.no_vr2d else None

    # ---- roofline of the dominant kernel family -------------------------------
    peak, peak_kind = peaks()
    roof = roofline(prof, args.steps, ncell, peak, peak_kind, {} if reduced else traffic_table(),
                    ms_max / args.steps)

    part_ms = prof.get("part", (0.0, 0))[0]
    counts = part.counts
    particles = {"n": NPART, "mode": "tracer", "class": PART_CLASS, "nsubdt": part.nsubdt,
                 "live_after": counts["npart"], "ms_per_step": part_ms / args.steps,
                 "share_of_step": part_ms / ms if ms > 0 else None,
                 "value": NPART * args.steps / (part_ms / 1e3) if part_ms > 0 else None,
                 "unit": "particle-steps/s (particle kernel time)",
                 "substeps_per_s": NPART * part.nsubdt * args.steps / (part_ms / 1e3) if part_ms > 0 else None}
    # the reference's inertial particles (class 1: Stokes drag, the 117-word
    # state with Jacobian and Hessian rates; part_tools.F90:241-251, 847-870)
    # on the same field and cloud, timed alone over a few iter_part calls
    if not reduced and not args.no_particles_alone:
        particles["inertial"] = inertial_bench(run, stream, e0, e1)
        # the tracers alone, walked in slot order (the default) and in cell order
        particles["alone_ms_per_step"] = {
            "cell_order": particle_alone_ms(run, stream, e0, e1, PART_CLASS, PART_MODE, 1)[0],
            "slot_order": particle_alone_ms(run, stream, e0, e1, PART_CLASS, PART_MODE, 0)[0]}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(world),
            "max_div_u": maxdiv, "nonfinite": nonfinite, "particles": particles, "mixed": mixed,
            "ensemble": ensemble, "vr2d_krylov": vr2d,
            "e2e": e2e,
            "gpu_launches": launches,
            "roofline": roof,
            "kernel_ms_per_step": {k: v[0] / args.steps for k, v in sorted(prof.items())},
            "sweep_tiles_r_z": list(tiles),
            "clocks": clk}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        val, done, cores, sample = cpu_reference(3, 20.0, q)
        line["cpu_baseline"] = {"value": val, "unit": UNIT, "cores": cores, "kind": "port",
                                "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    part.close()
    run.close()
    rep.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
