"""Benchmark of the force path: atom-force-evaluations per second.

Workload (default, --workload eam_cuni_256k): fcc Cu-Ni random 50/50 alloy,
40x40x40 cubic cells = 256,000 atoms, a = 3.58 A, Gaussian displacements
sigma = 0.08 A, Zhou (2004) alloy EAM, mixed precision (float32 pair terms,
float64 wrap / rho-bar / embedding argument / accumulation).  Synthetic, seeded
data in the shape of the reference's benchmarks/bench_force.py generator.

A step is one energy + force + virial evaluation of the whole structure with
a prebuilt device neighbour list (the reference's call_nl_s methodology,
benchmarks/bench_force.py:372-409).  value = atoms / step time on the device
(CUDA events, L2 flushed between steps outside the events), whole job over all
ranks; e2e = the same through the public force_fn API with host numpy arrays
(host->device positions + species, device->host forces, energy, stress inside
the timed region).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With --gpus N > 1 (torchrun), every rank evaluates its own replica of the
structure ("replicas only": one structure does not shard) and the time is the
max over ranks.

--workload batched_si512: 512 independent periodic Si structures (diamond
supercells of {1..4}^3 cell multiples, symmetric strain entries uniform
+-3 %, Gaussian displacements 0.1 A); one step evaluates every structure
with Tersoff (1988 Si(C)) and with Stillinger-Weber, replayed as one CUDA
graph with the autotuned lanes-per-atom.  value counts atoms of the original
structures (thin cells are evaluated as replicated supercells; the replicas
are overhead, not counted).  With N ranks every rank takes 512 / N
structures ("weak": a fixed share per rank would be 512 each; here the set is
split, "strong").
"""
import argparse
import gc
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "atom-force-evals/s"

from akitsushima_b200.workloads import (make_cuni, make_gesn, make_ni3al_set, make_si,  # noqa: E402
                                        make_si_set, make_sic_set)


def _ncu_traffic(kernel, workload, precision):
    """DRAM bytes per launch of `kernel` from the committed ncu capture of
    this workload (profiles/ncu_traffic.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            rec = json.load(f).get(kernel)
    except (OSError, ValueError):
        return None
    if not rec or rec.get("workload") != workload or rec.get("precision") != precision:
        return None
    return {"bytes_per_launch": rec["dram_bytes_per_launch"], "source": rec["source"]}


def _ncu_issue(kernel, workload, precision):
    """The instruction-issue view of `kernel` from the same committed ncu
    capture: the fraction of issue slots used (the bound of an issue-limited
    kernel) and the warp instructions per launch, or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            rec = json.load(f).get(kernel)
    except (OSError, ValueError):
        return None
    if not rec or rec.get("workload") != workload or rec.get("precision") != precision \
            or "issue_active_pct" not in rec:
        return None
    return {"frac": rec["issue_active_pct"] / 100.0, "metric": "smsp__issue_active.avg.pct_of_peak_sustained_active",
            "warp_inst_per_launch": rec["warp_inst_per_launch"],
            "threads_per_warp_inst": rec["threads_per_warp_inst"], "source": rec["source"]}


def cpu_count():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


class ClockSampler:
    """SM clock and clock-event reasons sampled through NVML every few
    milliseconds on a background thread while the timed region runs (read
    only; no setting of the GPU is touched)."""

    NAMES = {"applications_clocks_setting": 0x2, "sw_power_cap": 0x4, "hw_slowdown": 0x8,
             "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
             "hw_power_brake_slowdown": 0x80}

    def __init__(self, gpu_index, period_s=0.002):
        import threading
        self.samples, self.reasons, self.max_mhz, self.err = [], set(), None, None
        self._stop = threading.Event()
        self._period = period_s
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(gpu_index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM))
        except Exception as exc:  # no NVML: report it instead of a number
            self._nv = None
            self.err = f"nvml unavailable: {exc}"
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                self.samples.append(float(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM)))
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                for name, b in self.NAMES.items():
                    if bits & b:
                        self.reasons.add(name)
            except Exception as exc:
                self.err = str(exc)
                return
            self._stop.wait(self._period)

    def __enter__(self):
        if self._nv is not None:
            self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._nv is not None:
            self._t.join(timeout=2)

    def summary(self):
        out = {"sm_mhz": float(np.median(self.samples)) if self.samples else None,
               "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
               "samples": len(self.samples), "source": "NVML, 2 ms period, during the timed steps"}
        if self.err:
            out["note"] = self.err
        return out


def emit(args, line):
    """Print the JSON line, or keep it when the caller collects sub-records."""
    if getattr(args, "collect", None) is not None:
        args.collect.append(line)
    else:
        print(json.dumps(line), flush=True)


def time_reference(lat, pos, ids, steps, warmup, result=None):
    """The CPU port of the reference's numba path (oracle/): numpy prep and
    C kernels under OpenMP with every host thread, prebuilt neighbour list.
    ``result`` (a list) receives the last call's (E, F, S)."""
    import oracle
    from akitsushima_b200.published_parameters import ZHOU_2004
    threads = cpu_count()
    oracle.set_threads(threads)
    spec = oracle.zhou_spec({s: ZHOU_2004[s] for s in ("Cu", "Ni")}, ["Cu", "Ni"])
    types = np.array(["Cu", "Ni"])[ids]
    i, j, _, _ = oracle.nl_build(lat, pos, spec.r_cut, 0.3)
    for _ in range(max(1, warmup)):
        oracle.eam(spec, lat, pos, types, (i, j))
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        out = oracle.eam(spec, lat, pos, types, (i, j))
        ts.append(time.perf_counter() - t0)
    if result is not None:
        result.append(out)
    return float(np.mean(ts)), threads

def time_reference_batched(structs, n_sample):
    """The oracle port of the reference's Tersoff and SW numba paths over the
    first n_sample structures (thin cells as the same replicated
    supercells), every host thread, prebuilt pair lists; seconds per
    structure-pair-of-evaluations and the atoms counted."""
    import oracle
    from akitsushima_b200.published_parameters import SW_SI_1985, TERSOFF_SI_1988
    from akitsushima_b200.system import replicate_thin
    threads = cpu_count()
    oracle.set_threads(threads)
    rc_t = TERSOFF_SI_1988["R"] + TERSOFF_SI_1988["D"]
    rc_s = SW_SI_1985["a"] * SW_SI_1985["sigma"]
    work = []
    for lat, pos, _ in structs[:n_sample]:
        z = np.zeros(len(pos), np.int32)
        lt, pt, _, _ = replicate_thin(lat, pos, z, rc_t + 0.3)
        ls, ps, _, _ = replicate_thin(lat, pos, z, rc_s + 0.3)
        work.append((len(pos), lt, pt, oracle.nl_build(lt, pt, rc_t, 0.3)[:2],
                     ls, ps, oracle.nl_build(ls, ps, rc_s, 0.3)[:2]))
    t0 = time.perf_counter()
    atoms = 0
    for n, lt, pt, pr_t, ls, ps, pr_s in work:
        oracle.tersoff_single(TERSOFF_SI_1988, lt, pt, pr_t)
        oracle.sw_single(SW_SI_1985, ls, ps, pr_s)
        atoms += 2 * n
    return time.perf_counter() - t0, atoms, threads


def run_batched(args, world, rank, local):
    n_struct = 512
    structs = make_si_set(n_struct)
    cfg = {"workload": "batched_si512_tersoff_sw", "n_structures": n_struct,
           "sizes": "diamond {1..4}^3 cell multiples, 8-512 atoms", "strain": 0.03,
           "sigma": 0.1, "skin": 0.3, "precision": args.precision,
           "potentials": ["Tersoff 1988 Si(C)", "Stillinger-Weber 1985 Si"],
           "l2": "256 MB scratch write between steps, outside the timed events",
           "parallelism": f"split{world}"}
    if args.impl == "reference":
        if rank != 0:
            return 0
        import oracle  # noqa: F401  (built by __graft_entry__.build)
        per = []
        for _ in range(max(1, args.warmup) if args.steps > 0 else 0):
            time_reference_batched(structs, 8)
        for _ in range(args.steps):
            t, atoms, threads = time_reference_batched(structs, 128)
            per.append(atoms / t)
        v = float(np.mean(per))
        line = {"metric": METRIC, "value": v, "unit": "atoms/s", "impl": "reference",
                "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": None, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": dict(cfg, precision="fp64"),
                "cpu_baseline": {"value": v, "unit": "atoms/s", "cores": threads, "kind": "port",
                                 "sample": "per step: Tersoff + SW force calls of the first 128 "
                                           "of the 512 structures, prebuilt pair lists"},
                "e2e": {"value": v, "unit": "atoms/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    import torch
    import akitsushima_b200 as ak
    from akitsushima_b200 import _lib

    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())
    from akitsushima_b200.fit import shard_structures
    mine = [structs[q] for q in shard_structures([len(p) for _, p, _ in structs], world)[rank]]
    n_atoms = sum(len(p) for _, p, _ in mine)
    pots = [ak.TersoffPotential(ak.TERSOFF_SI_1988, species=["Si"], precision=args.precision),
            ak.StillingerWeberPotential(ak.SW_SI_1985, species=["Si"], precision=args.precision)]
    evs = [ak.BatchedEvaluator(p, mine, skin=0.3, device=dev) for p in pots]
    tuned = [ev.autotune(candidates=(4, 8, 16), reps=5) for ev in evs]
    for ev in evs:
        ev.run()
    torch.cuda.synchronize()
    side = torch.cuda.Stream(dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        for ev in evs:
            ev._eval()
    torch.cuda.current_stream(dev).wait_stream(side)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        for ev in evs:
            ev._eval()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        graph.replay()
    torch.cuda.synchronize()

    ev_t = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.zero_()
            ev_t[k][0].record()
            graph.replay()
            ev_t[k][1].record()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
    ms = sum(a.elapsed_time(b) for a, b in ev_t) / args.steps
    if dist:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    total_atoms = sum(len(p) for _, p, _ in structs)
    value = 2 * total_atoms / (ms * 1e-3)

    # per-kernel breakdown (eager, same launches as the graph)
    _lib.profile_begin()
    for _ in range(args.steps):
        for ev in evs:
            ev._eval()
    prof = _lib.profile_end()
    launches = sum(c for c, _ in prof.values()) / args.steps

    # the same work as per-structure launches (one list + one call each)
    singles = []
    for lat, pos, types in ([] if args.skip_singles else mine):
        row = []
        for p in pots:
            b = ak.Batch.single(*_replicated(lat, pos, p.r_cut + 0.3), device=dev)
            dl = ak.DeviceNeighbourList(p.r_cut + 0.3).build(b)
            row.append((p, b, dl))
        singles.append(row)
    for row in singles:
        for p, b, dl in row:
            p.evaluate(b, dl)
    torch.cuda.synchronize()
    a, b_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for row in singles:
        for p, b, dl in row:
            p.evaluate(b, dl)
    b_.record()
    torch.cuda.synchronize()
    ms_single = a.elapsed_time(b_) if singles else float("nan")

    # end to end: host positions in (pinned staging), per-structure forces,
    # energies and stresses out, through the evaluator's public calls
    host_pos = [np.ascontiguousarray(ev.batch.pos.cpu().numpy()) for ev in evs]
    for ev in evs:
        ev.capture()               # results() then replays the evaluator's graph
    for _ in range(args.warmup):   # the staging and result blocks are allocated on first use
        for ev, hp in zip(evs, host_pos):
            ev.batch.set_positions(hp)
            ev.results()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        res = []
        for ev, hp in zip(evs, host_pos):
            ev.batch.set_positions(hp)
            res.append(ev.results())
    t_e2e = (time.perf_counter() - t0) / args.e2e_steps
    if dist:
        t = torch.tensor([t_e2e, ms_single], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_e2e, ms_single = float(t[0].item()), float(t[1].item())
    h2d = sum(ev.batch.n_atoms * 24 for ev in evs)
    d2h = sum(ev.n_atoms * 24 + ev.n_structures * (8 + 72) for ev in evs)
    e2e = {"value": 2 * total_atoms / t_e2e, "unit": "atoms/s", "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h, "ms_per_step": t_e2e * 1e3,
           "path": "BatchedEvaluator (captured): batch.set_positions(numpy) + results() -> numpy, "
                   "Tersoff and SW"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        t_cpu, atoms, threads = time_reference_batched(structs, 32)
        cpu = {"value": atoms / t_cpu, "unit": "atoms/s", "cores": threads, "kind": "port",
               "sample": "Tersoff + SW force calls of the first 32 of the 512 structures, "
                         "oracle port of the reference's numba paths, prebuilt pair lists"}
    clocks = clk.summary()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": METRIC, "value": value, "unit": "atoms/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32+f64" if args.precision == "mixed" else "f64", "data": "synthetic",
            "config": cfg, "structures_per_s": 2 * n_struct / (ms * 1e-3),
            "gpu_launches": int(round(launches * args.steps)), "gpu_launches_per_step": launches,
            "clocks": clocks, "autotune": tuned,
            "per_structure_launches": None if not singles else
            {"ms_per_step": ms_single, "value": 2 * total_atoms / (ms_single * 1e-3),
             "speedup_of_batched": ms_single / ms},
            "kernels": {k: {"launches": c, "ms_per_launch": t / c} for k, (c, t) in prof.items()},
            "e2e": e2e, "cpu_baseline": cpu, "roofline": None}
    emit(args, line)
    return 0

MD_WORKLOADS = {
    # name: (potential, cells, sigma, precision, MD steps per bench step)
    "md_tersoff_si4096": ("tersoff", 8, 0.05, "fp64", 10),
    "md_sw_si64k": ("sw", 20, 0.1, "mixed", 10),
}


def _md_potential(kind, precision):
    import akitsushima_b200 as ak
    if kind == "tersoff":
        return ak.TersoffPotential(ak.TERSOFF_SI_1988, species=["Si"], precision=precision)
    return ak.StillingerWeberPotential(ak.SW_SI_1985, species=["Si"], precision=precision)


def time_reference_md(kind, lat, pos, types, n_steps):
    """The oracle port of the reference's NVE loop and force call
    (solvers/molecular_dynamics.py:1969-2000), every host thread, the pair
    list rebuilt every 10 steps; seconds per MD step."""
    import oracle
    from akitsushima_b200.published_parameters import SW_SI_1985, TERSOFF_SI_1988
    threads = cpu_count()
    oracle.set_threads(threads)
    m = np.full(len(pos), 28.086)
    v0 = oracle.init_velocities_mb(300.0, m, np.random.default_rng(0))
    rc = TERSOFF_SI_1988["R"] + TERSOFF_SI_1988["D"] if kind == "tersoff" else \
        SW_SI_1985["a"] * SW_SI_1985["sigma"]
    state = {"k": 0, "pairs": None}

    def force(r):
        if state["k"] % 10 == 0:
            state["pairs"] = oracle.nl_build(lat, r, rc, 0.3)[:2]
        state["k"] += 1
        if kind == "tersoff":
            e, f, _ = oracle.tersoff_single(TERSOFF_SI_1988, lat, r, state["pairs"])
        else:
            e, f, _ = oracle.sw_single(SW_SI_1985, lat, r, state["pairs"])
        return e, f

    force(pos)
    t0 = time.perf_counter()
    oracle.nve(force, lat, pos, m, v0, 1.0, n_steps)
    return (time.perf_counter() - t0) / n_steps, threads


def run_md(args, world, rank, local):
    kind, n_cells, sigma, precision, per_step = MD_WORKLOADS[args.workload]
    if args.precision_given:
        precision = args.precision
    lat, pos, types = make_si(n_cells, sigma=sigma)
    n_atoms = len(pos)
    cfg = {"workload": args.workload, "potential": "Tersoff 1988 Si(C)" if kind == "tersoff"
           else "Stillinger-Weber 1985 Si", "n_atoms": n_atoms, "a": 5.431, "sigma": sigma,
           "ensemble": "NVE velocity Verlet, dt 1 fs, Maxwell-Boltzmann 300 K (seed 0)",
           "skin": 0.3, "rebuild": "the reference's displacement criterion (2 max|dr| >= skin), "
                                   "checked on the device every step; the rebuild is a CUDA-graph "
                                   "IF branch", "md_steps_per_bench_step": per_step,
           "precision": precision, "l2": "256 MB scratch write between bench steps (each a "
                                         "10-MD-step graph replay), outside the timed events",
           "parallelism": f"replicas{world}"}
    if args.impl == "reference":
        if rank != 0:
            return 0
        n = 3 if n_atoms > 10000 else 10
        t, threads = time_reference_md(kind, lat, pos, types, n)
        v = n_atoms / t
        line = {"metric": METRIC, "value": v, "unit": "atoms/s", "impl": "reference", "n_gpus": 0,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3 * per_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": dict(cfg, precision="fp64"),
                "cpu_baseline": {"value": v, "unit": "atoms/s", "cores": threads, "kind": "port",
                                 "sample": f"{n} NVE steps of the {n_atoms}-atom structure (oracle port "
                                           "of the reference loop and force call)"},
                "e2e": {"value": v, "unit": "atoms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    import torch
    from akitsushima_b200 import _lib, md

    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())
    pot = _md_potential(kind, precision)
    sim = md.NVE(pot, lat, pos, types, temperature=300.0, seed=0, steps_per_graph=per_step, device=dev)
    sim.capture()
    for _ in range(args.warmup):
        sim.run(per_step)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record()
            sim.run(per_step)
            ev[k][1].record()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
    ms = sum(a.elapsed_time(b) for a, b in ev) / args.steps
    if dist:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    res = sim.results()
    value = world * n_atoms * per_step / (ms * 1e-3)

    # per-kernel breakdown: one interval of eager launches under the profiler
    _lib.profile_begin()
    sim.run(per_step, graph=False)
    prof = _lib.profile_end()
    launches = sum(c for c, _ in prof.values())

    # end to end through the public API: host arrays in, NVE built (list,
    # MB start, first forces), 10 x per_step steps, positions and thermo out
    # (the whole job three times: its mean, and each job's time)
    torch.cuda.synchronize()
    n_e2e = 10 * per_step
    jobs = []
    for _ in range(3):
        t0 = time.perf_counter()
        s2 = md.NVE(pot, lat, pos, types, temperature=300.0, seed=0, steps_per_graph=per_step, device=dev)
        s2.run(n_e2e)
        r2 = s2.results()
        p2 = s2.positions
        jobs.append(time.perf_counter() - t0)
        del s2
    t_e2e = float(np.mean(jobs)) / n_e2e
    e2e = {"value": world * n_atoms / t_e2e, "unit": "atoms/s",
           "h2d_bytes_per_step": (n_atoms * (24 + 24 + 4 + 8)) / n_e2e,
           "d2h_bytes_per_step": (n_atoms * 24 + len(r2["e_pot"]) * 16) / n_e2e,
           "ms_per_step": t_e2e * 1e3,
           "job_ms": [round(1e3 * j, 3) for j in jobs],
           "path": f"md.NVE(numpy in) + run({n_e2e}) + results() + positions (graph captured inside), "
                   "mean of 3 jobs"}
    # energy conservation over drift_ps picoseconds (dt 1 fs) in both
    # precisions: the slope of E_tot per atom against time, against the
    # reference's bar for a mixed-precision GPU path (<= 1e-5 eV/atom/ps over
    # 10 ps, docs/adr/0016-gpu-support.md:115-123)
    drift_rec = None
    if getattr(args, "drift_ps", 0) > 0:
        n_dr = int(round(args.drift_ps * 1000))
        drift_rec = {"ps": args.drift_ps, "steps": n_dr, "bar_mixed_eV_per_atom_per_ps": 1e-5}
        for prec in ("mixed", "fp64"):
            s3 = md.NVE(_md_potential(kind, prec), lat, pos, types, temperature=300.0, seed=0,
                        steps_per_graph=50, device=dev)
            s3.run(n_dr)
            r3 = s3.results()
            t_ps = np.arange(1, len(r3["e_tot"]) + 1) * 1e-3
            slope = float(np.polyfit(t_ps, r3["e_tot"] / n_atoms, 1)[0])
            drift_rec[prec] = {"drift_eV_per_atom_per_ps": slope,
                               "max_abs_deviation_eV_per_atom": float(np.abs(r3["drift"]).max() / n_atoms),
                               "rebuilds": int(r3["rebuilds"])}
            del s3
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        n = 3 if n_atoms > 10000 else 10
        t_cpu, threads = time_reference_md(kind, lat, pos, types, n)
        cpu = {"value": n_atoms / t_cpu, "unit": "atoms/s", "cores": threads, "kind": "port",
               "sample": f"{n} NVE steps of the same structure, oracle port of the reference's "
                         "loop and numba force call"}
    clocks = clk.summary()
    drift = res["drift"]
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": METRIC, "value": value, "unit": "atoms/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "ms_per_md_step": ms / per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64" if precision == "mixed" else "f64",
            "data": "synthetic", "config": cfg, "gpu_launches": int(launches * args.steps),
            "gpu_launches_per_step": launches, "clocks": clocks,
            "kernels": {k: {"launches": c, "ms_per_launch": t / c} for k, (c, t) in prof.items()},
            "energy": {"md_steps": int(len(drift)), "max_abs_drift_ev_per_atom":
                       float(np.abs(drift).max() / n_atoms),
                       "final_drift_ev_per_atom": float(drift[-1] / n_atoms),
                       "max_skin_displacement": float(res["skin_displacement"].max()),
                       "rebuilds": int(res["rebuilds"])},
            "nve_drift": drift_rec,
            "e2e": e2e, "cpu_baseline": cpu, "roofline": None}
    emit(args, line)
    return 0


def _fit_setup():
    """The Tersoff-1989 Si-C parameter set (fitting/registry.py:724-730) and
    its target parameters theta * U(0.95, 1.05) (seeded), as x vectors."""
    from akitsushima_b200 import fit
    from akitsushima_b200.published_parameters import TERSOFF_1989
    species = ["Si", "C"]
    el = {s: dict(TERSOFF_1989["elements"][s]) for s in species}
    ps = fit.Tersoff1989ParameterSet(el, {"Si-C": TERSOFF_1989["chi"]["C-Si"]}, species)
    x0 = ps.x0
    u = np.random.default_rng(7).uniform(0.95, 1.05, len(x0))
    xt = np.array([np.log(np.exp(x) * f) if key in ps._LOG_KEYS else x * f
                   for x, f, (_, key, _) in zip(x0, u, ps.variables)])
    return ps, x0, xt


def _fit_setup_multi():
    """The multi-species Si-C record set (fitting/parameter_sets.py:1068-1203;
    A, B, lambda1, lambda2 per unordered pair and c, d, h per (i, j, k)
    record: every species triplet) at the Tersoff-1989 Si-C values, and its
    target parameters theta * U(0.95, 1.05) (seeded), as x vectors."""
    from akitsushima_b200 import fit
    from akitsushima_b200.published_parameters import TERSOFF_1989
    from akitsushima_b200.tersoff import tersoff1989_to_triplets
    species = ["Si", "C"]
    el = {s: dict(TERSOFF_1989["elements"][s]) for s in species}
    recs = tersoff1989_to_triplets(el, {"Si-C": TERSOFF_1989["chi"]["C-Si"]}, species)
    ps = fit.MultiSpeciesTersoffParameterSet(recs, species)
    x0 = ps.x0
    u = np.random.default_rng(7).uniform(0.95, 1.05, len(x0))
    xt = np.array([np.log(np.exp(x) * f) if key in ps._LOG_KEYS else x * f
                   for x, f, (_, key, _) in zip(x0, u, ps.variables)])
    return ps, x0, xt


def _fit_setup_zhou():
    """The Zhou (2004) Al-Ni parameter set (ZhouEAMParameterSet defaults:
    A B alpha beta Fn2 Fn3 F2 F3 eta per element) and its target
    parameters theta * U(0.97, 1.03) (seeded), as x vectors."""
    from akitsushima_b200 import fit
    from akitsushima_b200.published_parameters import ZHOU_2004
    species = ["Al", "Ni"]
    ps = fit.ZhouEAMParameterSet({s: dict(ZHOU_2004[s]) for s in species}, species)
    x0 = ps.x0
    u = np.random.default_rng(7).uniform(0.97, 1.03, len(x0))
    xt = np.array([np.log(np.exp(x) * f) if key in ps._LOG_KEYS else x * f
                   for x, f, (_, key, _) in zip(x0, u, ps.variables)])
    return ps, x0, xt


FIT_WORKLOADS = {
    # name: (structure set, parameter set, loss weights, config)
    "fit_sic256": (lambda: make_sic_set(256), _fit_setup_multi, {"energy": 1.0, "forces": 1.0, "stress": 0.1},
                   {"workload": "fit_sic256_multispecies",
                    "sizes": "zincblende SiC 2^3 / 3^3 cells (64 / 216 atoms)", "a": 4.36, "strain": 0.02,
                    "sigma": 0.1,
                    "parameter_set": "MultiSpeciesTersoffParameterSet (A B lambda1 lambda2 per pair, c d h per "
                                     "(i, j, k) record), Tersoff-1989 Si-C start",
                    "targets": "float64 E/F/S at theta * U(0.95, 1.05)",
                    "loss": "w_E 1, w_F 1, w_S 0.1, r0 1, eps0 1 (squared)"}),
    "fit_sic256_t1989": (lambda: make_sic_set(256), _fit_setup, {"energy": 1.0, "forces": 1.0, "stress": 0.1},
                   {"workload": "fit_sic256_tersoff1989",
                    "sizes": "zincblende SiC 2^3 / 3^3 cells (64 / 216 atoms)", "a": 4.36, "strain": 0.02,
                    "sigma": 0.1, "parameter_set": "Tersoff1989ParameterSet (A B lambda mu c d h per element, chi)",
                    "targets": "float64 E/F/S at theta * U(0.95, 1.05)",
                    "loss": "w_E 1, w_F 1, w_S 0.1, r0 1, eps0 1 (squared)"}),
    "fit_ni3al256_zhou": (lambda: make_ni3al_set(256), _fit_setup_zhou,
                          {"energy": 1.0, "forces": 1.0, "stress": 1.0, "r0": 0.1, "eps0": 0.01},
                          {"workload": "fit_ni3al256_zhou2004",
                           "sizes": "L1_2 Ni3Al 4^3 / 5^3 cells (256 / 500 atoms)", "a": 3.57, "strain": 0.02,
                           "sigma": 0.08,
                           "parameter_set": "ZhouEAMParameterSet (A B alpha beta Fn2 Fn3 F2 F3 eta per element)",
                           "targets": "float64 E/F/S at theta * U(0.97, 1.03)",
                           "loss": "w_E 1, w_F 1, w_S 1, r0 0.1, eps0 0.01 (squared)"}),
}


def _fit_structs(raw, efs):
    out = []
    for (lat, pos, types), (e, f, s) in zip(raw, efs):
        out.append({"lattice": lat, "positions": pos, "atom_types": types, "natoms": len(pos),
                    "ref_energy": e / len(pos), "ref_forces": f, "ref_stress": s})
    return out


def time_reference_fit(raw, ps, x0, xt, n_sample, w):
    """The reference's gradient: forward differences of the loss, one loss
    evaluation per variable plus one (fitting/driver.py:802-816), each a
    loop of force calls (fitting/loss.py:184-242) -- the oracle port under
    OpenMP with every host thread, on the first n_sample structures;
    seconds per gradient of the whole set, scaled by atoms."""
    import oracle
    threads = cpu_count()
    oracle.set_threads(threads)
    sample = raw[:n_sample]
    if "eam" in ps.decode(x0):
        def force_of(x):
            d = ps.decode(x)["eam"]
            return oracle.zhou_force(d["elements"], ps.species, d["r_cut"], d["chi"])
        r_list = ps.r_cut + 0.3
    else:
        def force_of(x):
            rec = ps.decode(x)["tersoff"]
            return lambda L, P, T, pairs: oracle.tersoff_multi(rec, ps.species, L, P, T, pairs)
        r_list = 3.0 + 0.3
    pairs = [oracle.nl_build(L, P, r_list - 0.3, 0.3)[:2] for L, P, _ in sample]
    ft = force_of(xt)
    efs = [ft(L, P, T, pq) for (L, P, T), pq in zip(sample, pairs)]
    st = _fit_structs(sample, efs)
    f0 = force_of(x0)
    oracle.fit_loss(None, ps.species, st, w, pairs, force=f0)
    t0 = time.perf_counter()
    oracle.fit_loss(None, ps.species, st, w, pairs, force=f0)
    t_loss = time.perf_counter() - t0
    atoms_sample = sum(len(p) for _, p, _ in sample)
    atoms_all = sum(len(p) for _, p, _ in raw)
    return t_loss * (len(x0) + 1) * atoms_all / atoms_sample, threads


def run_fit(args, world, rank, local):
    make_set, setup, weights, cfg0 = FIT_WORKLOADS[args.workload]
    raw = make_set()
    n_struct = len(raw)
    n_atoms = sum(len(p) for _, p, _ in raw)
    cfg = dict(cfg0, n_structures=n_struct, n_atoms=n_atoms, precision="fp64",
               l2="256 MB scratch write between steps, outside the timed events", parallelism=f"split{world}")
    n_sample = 4 if "zhou" in args.workload else 16
    from akitsushima_b200 import fit
    ps, x0, xt = setup()
    n_var = len(x0)
    if args.impl == "reference":
        if rank != 0:
            return 0
        per = []
        for _ in range(max(1, args.steps)):
            t, threads = time_reference_fit(raw, ps, x0, xt, n_sample, weights)
            per.append(1.0 / t)
        v = float(np.mean(per))
        line = {"metric": "fit grads/s", "value": v, "unit": "gradients/s", "impl": "reference",
                "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / v,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": cfg,
                "cpu_baseline": {"value": v, "unit": "gradients/s", "cores": threads, "kind": "port",
                                 "sample": f"one loss over the first {n_sample} structures, scaled by atoms to "
                                           f"the {n_struct} and by {n_var + 1} (forward differences)"},
                "e2e": {"value": v, "unit": "gradients/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    import torch

    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())
    from akitsushima_b200 import _lib
    # targets: float64 evaluation of every structure at the target parameters
    tgt = fit.PotentialFit(ps, [{"lattice": L, "positions": P, "atom_types": T, "natoms": len(P),
                                 "ref_energy": 0.0} for L, P, T in raw], device=dev)
    with torch.no_grad():
        E, F, W = tgt.model.efs(torch.as_tensor(xt), tgt.ev)
    E, F, W = E.cpu().numpy(), F.cpu().numpy(), W.cpu().numpy()
    off = tgt.ev.batch.offsets
    vols = tgt.ev.batch.volumes
    efs = [(E[q], F[off[q]:off[q + 1]], W[q].reshape(3, 3) / vols[q]) for q in range(n_struct)]
    structs = _fit_structs(raw, efs)
    del tgt
    f = fit.PotentialFit(ps, structs, weights, device=dev, rank=rank, world=world)
    # x, its tables and their x-Jacobians live on the host (a few dozen
    # scalars); the batch, the evaluation, the fused loss and the adjoint on
    # the device; the step ends with the loss and the table gradients on the
    # device (their sum over ranks is the whole set's)

    def device_step():
        loss, d, _ = f.device_step(x0, True)
        return torch.cat([loss] + [t.reshape(-1) for t in d])

    for _ in range(args.warmup):
        device_step()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record()
            vec = device_step()
            fit.allreduce_sum(vec, world)
            ev[k][1].record()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
    ms = sum(a.elapsed_time(b) for a, b in ev) / args.steps
    if dist:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = 1e3 / ms
    _lib.profile_begin()
    device_step()
    torch.cuda.synchronize()
    prof = _lib.profile_end()
    launches = sum(c for c, _ in prof.values())
    # end to end: numpy x in, (loss, numpy gradient) out, every rank
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        loss, grad = f.loss_and_grad(x0)
    t_e2e = (time.perf_counter() - t0) / args.e2e_steps
    if dist:
        t = torch.tensor([t_e2e], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_e2e = float(t.item())
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        t_cpu, threads = time_reference_fit(raw, ps, x0, xt, n_sample, weights)
        cpu = {"value": 1.0 / t_cpu, "unit": "gradients/s", "cores": threads, "kind": "port",
               "sample": f"one loss over the first {n_sample} structures (oracle port), scaled by atoms to the "
                         f"{n_struct} and by {n_var + 1}: the reference's forward-difference gradient"}
    clocks = clk.summary()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": "fit grads/s", "value": value, "unit": "gradients/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
            "atom_force_evals_per_s": n_atoms / (ms * 1e-3), "n_variables": n_var,
            "gpu_launches": int(launches * args.steps), "gpu_launches_per_step": launches, "clocks": clocks,
            "kernels": {k: {"launches": c, "ms_per_launch": t / c} for k, (c, t) in prof.items()},
            "e2e": {"value": 1.0 / t_e2e, "unit": "gradients/s", "h2d_bytes_per_step": 8 * n_var,
                    "d2h_bytes_per_step": 8 * (n_var + 2), "ms_per_step": t_e2e * 1e3,
                    "path": "PotentialFit.loss_and_grad(numpy x) -> (loss, numpy gradient)"},
            "check": {"loss": float(loss), "grad_norm": float(np.linalg.norm(grad))},
            "cpu_baseline": cpu, "roofline": None}
    emit(args, line)
    return 0


def _perf_case(name, precision):
    """(lattice, positions, species names, potential, oracle evaluator) of a
    performance-path workload."""
    import oracle
    import akitsushima_b200 as ak
    from akitsushima_b200 import eam as eam_mod
    from akitsushima_b200.published_parameters import SW_GESN_TOMITA_2018, ZHOU_2004
    if name == "eam_setfl_cuni_256k":
        lat, pos, ids = make_cuni(40)
        types = list(np.array(["Cu", "Ni"])[ids])
        zp = ak.zhou_eam({s: ZHOU_2004[s] for s in ("Cu", "Ni")}, ["Cu", "Ni"])
        pot = eam_mod.tabulate(zp, precision=precision)
        sp = ["Cu", "Ni"]
        specs = ([pot.rho_spec[s] for s in sp] + [pot.F_spec[s] for s in sp]
                 + [pot.phi_spec[frozenset(k)] for k in (("Cu",), ("Cu", "Ni"), ("Ni",))])
        ospec = oracle.EAMSpec(sp, specs, [0, 1], [2, 3], np.array([[4, 5], [5, 6]]), pot.r_cut)

        def ref(L, P, T, pairs):
            return oracle.eam(ospec, L, P, T, pairs)
        desc = "Zhou 2004 Cu-Ni as setfl cubic splines (2000 r and rho knots), fcc 40^3"
    else:
        lat, pos, types = make_gesn()
        pot = ak.StillingerWeberPotential(SW_GESN_TOMITA_2018, species=["Ge", "Sn"], precision=precision)
        recs = {(r["i"], r["j"], r["k"]): {k: v for k, v in r.items() if k not in "ijk"}
                for r in SW_GESN_TOMITA_2018}

        def ref(L, P, T, pairs):
            return oracle.sw_multi(recs, ["Ge", "Sn"], L, P, T, pairs)
        desc = "Tomita 2018 Ge-Sn Stillinger-Weber, diamond 20^3 (a 5.762 A), 25 % Sn at random"
    return lat, pos, types, pot, ref, desc


def run_perf_path(args, world, rank, local):
    """One evaluation of a large structure through the spline-EAM or the
    multi-species SW path (the performance paths beside the headline)."""
    import oracle
    lat, pos, types, pot, ref, desc = _perf_case(args.workload, args.precision)
    n_atoms = len(pos)
    cfg = {"workload": args.workload, "potential": desc, "n_atoms": n_atoms, "skin": 0.3,
           "precision": args.precision, "l2": "256 MB scratch write between steps, outside the timed events",
           "parallelism": f"replicas{world}"}

    def cpu_time(n):
        threads = cpu_count()
        oracle.set_threads(threads)
        pairs = oracle.nl_build(lat, pos, float(pot.r_cut), 0.3)[:2]
        ref(lat, pos, types, pairs)
        t0 = time.perf_counter()
        for _ in range(n):
            ref(lat, pos, types, pairs)
        return (time.perf_counter() - t0) / n, threads

    if args.impl == "reference":
        if rank != 0:
            return 0
        t, threads = cpu_time(max(1, min(args.steps, 3)))
        v = n_atoms / t
        line = {"metric": METRIC, "value": v, "unit": "atoms/s", "impl": "reference", "n_gpus": 0,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": dict(cfg, precision="fp64"),
                "cpu_baseline": {"value": v, "unit": "atoms/s", "cores": threads, "kind": "port",
                                 "sample": "force calls of the whole structure, prebuilt pair list"},
                "e2e": {"value": v, "unit": "atoms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    import torch
    import akitsushima_b200 as ak
    from akitsushima_b200 import _lib
    from akitsushima_b200.system import species_ids
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())
    batch = ak.Batch.single(lat, pos, species_ids(types, pot.species), device=dev)
    dnl = ak.DeviceNeighbourList(float(pot.r_cut) + 0.3).build(batch)
    tuned = pot.autotune_lanes(batch, dnl)
    out = pot.evaluate(batch, dnl)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        pot.evaluate(batch, dnl, out=out)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record()
            pot.evaluate(batch, dnl, out=out)
            ev[k][1].record()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
    ms = sum(a.elapsed_time(b) for a, b in ev) / args.steps
    if dist:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    _lib.profile_begin()
    pot.evaluate(batch, dnl, out=out)
    prof = _lib.profile_end()
    nl = ak.NeighbourList(float(pot.r_cut), skin_width=0.3, device=dev)
    nl.build_batch(batch)
    fn = ak.make_force_fn(pot)
    for _ in range(args.warmup):
        fn(lat, pos, types, nl)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        fn(lat, pos, types, nl)
    t_e2e = (time.perf_counter() - t0) / args.e2e_steps
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        t_cpu, threads = cpu_time(1)
        cpu = {"value": n_atoms / t_cpu, "unit": "atoms/s", "cores": threads, "kind": "port",
               "sample": "one force call of the whole structure (oracle port), prebuilt pair list"}
    clocks = clk.summary()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": METRIC, "value": world * n_atoms / (ms * 1e-3), "unit": "atoms/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if args.precision == "mixed" else "f64",
            "data": "synthetic", "config": cfg, "autotune": tuned,
            "gpu_launches": int(sum(c for c, _ in prof.values()) * args.steps),
            "kernels": {k: {"launches": c, "ms_per_launch": t / c} for k, (c, t) in prof.items()},
            "clocks": clocks,
            "e2e": {"value": world * n_atoms / t_e2e, "unit": "atoms/s", "h2d_bytes_per_step": n_atoms * 28,
                    "d2h_bytes_per_step": n_atoms * 24 + 80, "ms_per_step": t_e2e * 1e3,
                    "path": "force_fn(lattice, numpy positions, species names, NeighbourList) -> numpy"},
            "cpu_baseline": cpu, "roofline": None}
    emit(args, line)
    return 0


def _replicated(lat, pos, r_list):
    from akitsushima_b200.system import replicate_thin
    L2, P2, T2, _ = replicate_thin(lat, pos, np.zeros(len(pos), np.int32), r_list)
    return L2, P2, T2


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--cells", type=int, default=40)
    ap.add_argument("--lanes", type=int, default=4, help="EAM lanes per atom (1, 2, 4 or 8)")
    ap.add_argument("--drift-ps", type=float, default=0.0,
                    help="MD workloads: also run this many ps (dt 1 fs) in both precisions for the drift")
    ap.add_argument("--no-sub-records", action="store_true",
                    help="default workload: skip the other configurations' sub-records")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=200)
    ap.add_argument("--skip-singles", action="store_true",
                    help="batched workload: skip the per-structure-launch comparison (profiling runs)")
    ap.add_argument("--workload", default="eam_cuni_256k",
                    choices=["eam_cuni_256k", "batched_si512", "eam_setfl_cuni_256k",
                             "sw_gesn_64k"] + sorted(FIT_WORKLOADS) + sorted(MD_WORKLOADS))
    args = ap.parse_args()
    args.precision_given = "--precision" in sys.argv
    args.warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload == "batched_si512":
        return run_batched(args, world, rank, local)
    if args.workload in MD_WORKLOADS:
        return run_md(args, world, rank, local)
    if args.workload in FIT_WORKLOADS:
        return run_fit(args, world, rank, local)
    if args.workload in ("eam_setfl_cuni_256k", "sw_gesn_64k"):
        return run_perf_path(args, world, rank, local)
    if world > 1 and args.impl != "reference":
        return run_eam_spatial(args, world, rank, local)
    lat, pos, ids = make_cuni(args.cells)
    n_atoms = len(pos)
    workload = f"eam_zhou_cuni_fcc{args.cells}^3_{n_atoms}_atoms"
    cfg = {"workload": workload, "potential": "Zhou 2004 EAM Cu-Ni", "n_atoms": n_atoms,
           "a": 3.58, "sigma": 0.08, "skin": 0.3, "precision": args.precision,
           "l2": "256 MB scratch write between steps, outside the timed events",
           "parallelism": f"replicas{world}"}

    if args.impl == "reference":
        if rank != 0:
            return 0
        t, threads = time_reference(lat, pos, ids, args.steps, args.warmup)
        v = n_atoms / t
        line = {"metric": METRIC, "value": v, "unit": "atoms/s", "impl": "reference",
                "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": dict(cfg, precision="fp64"),
                "cpu_baseline": {"value": v, "unit": "atoms/s", "cores": threads, "kind": "port",
                                 "sample": f"{args.steps} full force calls of the {n_atoms}-atom "
                                           "structure, prebuilt neighbour list"},
                "e2e": {"value": v, "unit": "atoms/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    import torch
    import akitsushima_b200 as ak
    from akitsushima_b200 import _lib, roofline

    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())

    fn = ak.force_fn_from_config({"type": "EAM", "form": "zhou2004", "elements": ["Cu", "Ni"]},
                                 precision=args.precision)
    pot = fn.engine.potentials[0]
    pot.lanes_per_atom = args.lanes
    batch = ak.Batch.single(lat, pos, ids, device=dev)
    dnl = ak.DeviceNeighbourList(pot.r_cut + 0.3).build(batch)
    out = pot.evaluate(batch, dnl)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        pot.evaluate(batch, dnl, out=out)
    torch.cuda.synchronize()

    # timed region
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record()
            pot.evaluate(batch, dnl, out=out)
            ev[k][1].record()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
    clocks = clk.summary()
    ms = sum(a.elapsed_time(b) for a, b in ev) / args.steps
    if dist:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * n_atoms / (ms * 1e-3)
    res_main = (float(out.energy[0]), out.forces.cpu().numpy(), out.virial[0].cpu().numpy())

    # the other precision on the same inputs and list (the float64 GPU path
    # the mixed one is measured against), timed the same way after the
    # timed region
    other = "fp64" if args.precision == "mixed" else "mixed"
    out_o = pot.evaluate(batch, dnl, precision=other)
    for _ in range(3):
        pot.evaluate(batch, dnl, precision=other, out=out_o)
    n_o = max(3, min(args.steps, 10))
    ev_o = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n_o)]
    for k in range(n_o):
        flush.zero_()
        ev_o[k][0].record()
        pot.evaluate(batch, dnl, precision=other, out=out_o)
        ev_o[k][1].record()
    torch.cuda.synchronize()
    ms_o = sum(a.elapsed_time(b) for a, b in ev_o) / n_o
    res_other = (float(out_o.energy[0]), out_o.forces.cpu().numpy(), out_o.virial[0].cpu().numpy())

    # per-kernel breakdown: a second identical pass under the launch profiler
    _lib.profile_begin()
    for k in range(args.steps):
        flush.zero_()
        pot.evaluate(batch, dnl, out=out)
    prof = _lib.profile_end()
    launches_per_step = sum(c for c, _ in prof.values()) / args.steps

    # the neighbour-list build timed apart (a fresh list each time, after one
    # warm build), and build + evaluation as one atoms/s figure
    ak.DeviceNeighbourList(pot.r_cut + 0.3).build(batch)
    t_build = []
    for _ in range(3):
        flush.zero_()
        b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        b0.record()
        ak.DeviceNeighbourList(pot.r_cut + 0.3).build(batch)
        b1.record()
        b1.synchronize()
        t_build.append(b0.elapsed_time(b1))
    nl_build = {"ms": float(np.mean(t_build)), "r_list": pot.r_cut + 0.3,
                "atoms_per_s_build_plus_call": n_atoms / ((float(np.mean(t_build)) + ms) * 1e-3),
                "note": "CUDA events around DeviceNeighbourList.build (it reads the slot count back to "
                        "size the rows), mean of 3 after one warm build"}

    # algorithmic work of the dominant kernel (the force pass)
    pi, pj = dnl.half_pairs()
    pi, pj = pi.long(), pj.long()
    d = batch.pos[pj] - batch.pos[pi]
    cell = torch.as_tensor(lat, device=dev)
    s = d @ torch.linalg.inv(cell)
    s -= torch.round(s)
    r = torch.linalg.norm(s @ cell, dim=1)
    inside = (r < pot.r_cut) & (r > 1e-12)
    tp = batch.types
    cross = (tp[pi] != tp[pj]) & inside
    n_in = int(inside.sum().item())
    n_cross = int(cross.sum().item())
    del pi, pj, d, s, r, inside, cross
    force_flops = roofline.eam_force_flops(n_in - n_cross, n_cross)
    force_bytes = roofline.eam_force_bytes(n_atoms, dnl.n_slots)
    dom = "eam_force"
    cnt, tot = prof.get(dom, (1, float("nan")))
    t_dom = tot / cnt * 1e-3
    scratch = torch.empty(148 * 8 * 256 * 8 * 4, dtype=torch.uint8, device=dev)
    peak = _lib._d(0.0)
    pcode = _lib.MBF_MIXED if args.precision == "mixed" else _lib.MBF_FP64
    _lib.check(_lib.lib().mbf_peak_probe(pcode, _lib.ptr(scratch), scratch.numel(), peak,
                                         torch.cuda.current_stream().cuda_stream), "peak probe")
    peak_tf = peak.value / 1e12
    ach_tf = force_flops / t_dom / 1e12
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            hbm_peak = float(json.load(f)["hbm_gbs"])
            hbm_src = "MEASURED_PEAKS.json"
    except (OSError, KeyError, ValueError):
        hbm_peak, hbm_src = 6650.0, "fallback"
    ach_gbs = force_bytes / t_dom / 1e9
    dens_flops = roofline.eam_density_flops(n_in, n_atoms)
    t_all = sum(t for _, t in prof.values()) / args.steps * 1e-3
    roof = {"kernel": dom, "bound": "fp32" if args.precision == "mixed" else "fp64",
            "achieved": ach_tf, "peak": peak_tf, "unit": "TFLOP/s", "frac": ach_tf / peak_tf,
            "peak_source": "measured live on this GPU: mbf_peak_probe FMA chains",
            "algorithmic_flops_per_launch": force_flops, "launch_ms": t_dom * 1e3,
            "traffic": _ncu_traffic(dom, workload, args.precision),
            "issue_view": _ncu_issue(dom, workload, args.precision),
            "hbm_view": {"achieved": ach_gbs, "peak": hbm_peak, "unit": "GB/s",
                         "frac": ach_gbs / hbm_peak, "peak_source": hbm_src,
                         "algorithmic_bytes_per_launch": force_bytes},
            "whole_step": {"algorithmic_flops": force_flops + dens_flops,
                           "kernels_ms": t_all * 1e3,
                           "frac": (force_flops + dens_flops) / t_all / 1e12 / peak_tf,
                           "note": "density + force algorithmic FLOPs over the sum of the step's kernel "
                                   "times, against the same FMA peak"},
            "kernels": {k: {"launches": c, "ms_per_launch": t / c} for k, (c, t) in prof.items()}}

    # end to end through the public API in the reference's call form: host
    # lattice and positions, atom_types a list of species names (the same
    # list object every call, as the reference's solvers pass it), host
    # (E, F (N, 3), stress) back
    nl = ak.NeighbourList(fn.r_cut, skin_width=0.3)
    nl.build_batch(batch)
    pos_host = np.ascontiguousarray(pos)
    names = [("Cu", "Ni")[t] for t in ids.tolist()]

    def e2e_loop(types, n):
        for _ in range(args.warmup):   # the same warm-up as the device-timed steps
            fn(lat, pos_host, types, nl)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        calls = []
        t0 = time.perf_counter()
        for _ in range(n):
            c0 = time.perf_counter()
            r_ = fn(lat, pos_host, types, nl)
            calls.append(time.perf_counter() - c0)
        t_ = (time.perf_counter() - t0) / n
        if dist:
            tt = torch.tensor([t_], device=dev, dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t_ = float(tt.item())
        return t_, calls, r_

    t_e2e, calls, (e, f, st) = e2e_loop(names, args.e2e_steps)
    t_ids, calls_ids, _ = e2e_loop(ids, args.e2e_steps)
    # per call: positions in (the species ids are uploaded once: an
    # unchanged list maps to the same ids and is not sent again; the lattice
    # is compared on the host), forces out plus one copy of energy, virial
    # and the two device status words
    e2e = {"value": world * n_atoms / t_e2e, "unit": "atoms/s",
           "h2d_bytes_per_step": n_atoms * 24, "d2h_bytes_per_step": n_atoms * 24 + 8 * (1 + 9 + 2),
           "ms_per_step": t_e2e * 1e3,
           "ms_per_call_min_median_max": [round(1e3 * float(np.min(calls)), 4),
                                          round(1e3 * float(np.median(calls)), 4),
                                          round(1e3 * float(np.max(calls)), 4)],
           "path": "force_fn(lattice, numpy positions, list of species names, NeighbourList) -> numpy "
                   "(the reference's call form)",
           "with_int_ids": {"value": world * n_atoms / t_ids, "ms_per_step": t_ids * 1e3,
                            "path": "the same call with an int32 species-id array"}}

    cpu = None
    oracle_res = []
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        t_cpu, threads = time_reference(lat, pos, ids, steps=2, warmup=1, result=oracle_res)
        cpu = {"value": n_atoms / t_cpu, "unit": "atoms/s", "cores": threads, "kind": "port",
               "sample": "2 full force calls of the same structure (after 1 warm-up), oracle port "
                         "of the reference's numba EAM path, prebuilt neighbour list"}

    # each result's error: against the float64 oracle (the CPU port, same
    # pairs) when it ran, and mixed against the float64 GPU path always
    vol = abs(float(np.linalg.det(lat)))

    def err(a, b):
        return {"max_force_eVA": float(np.abs(a[1] - b[1]).max()),
                "energy_per_atom_eV": abs(a[0] - b[0]) / n_atoms,
                "stress_eVA3": float(np.abs(np.asarray(a[2]).reshape(-1) - np.asarray(b[2]).reshape(-1)).max()) / vol}

    res = {args.precision: res_main, other: res_other}
    errors = {"tolerance": {"max_force_eVA": 1e-5, "energy_per_atom_eV": 1e-6, "stress_eVA3": 1e-5,
                            "fp64_relative": 1e-10},
              "mixed_vs_fp64_gpu": err(res["mixed"], res["fp64"])}
    if oracle_res:
        e0, f0, s0 = oracle_res[0]
        ref = (e0, f0, np.asarray(s0) * vol)   # the oracle's stress is already / V
        errors["mixed_vs_fp64_oracle"] = err(res["mixed"], ref)
        errors["fp64_gpu_vs_fp64_oracle"] = err(res["fp64"], ref)
    ms64 = ms if args.precision == "fp64" else ms_o
    fp64_gpu = {"ms_per_step": ms64, "value": world * n_atoms / (ms64 * 1e-3),
                "mixed_speedup": (ms_o / ms) if args.precision == "mixed" else (ms / ms_o),
                "note": "the float64 GPU path on the same inputs and list, CUDA events, L2 flushed"}

    subs = None
    if world == 1 and not args.no_sub_records:
        subs = sub_records(args)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": METRIC, "value": value, "unit": "atoms/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if args.precision == "mixed" else "f64", "data": "synthetic",
            "config": cfg, "gpu_launches": int(round(launches_per_step * args.steps)),
            "gpu_launches_per_step": launches_per_step, "clocks": clocks, "roofline": roof, "nl_build": nl_build,
            "fp64_gpu": fp64_gpu, "errors": errors, "e2e": e2e, "cpu_baseline": cpu,
            "check": {"energy_per_atom": e / n_atoms, "max_abs_force_sum": float(np.abs(f.sum(0)).max())},
            "configs": subs}
    print(json.dumps(line), flush=True)
    return 0


def run_eam_spatial(args, world, rank, local):
    """The headline alloy on N GPUs, weak scaling: fcc Cu-Ni of 40 x 40 x
    40 N cells (256,000 N atoms, the same generator), one slab of 256,000
    atoms per rank along z with a halo of one list radius.  A step is one
    distributed evaluation: the embedding pass, the exchange of the halo
    atoms' F'(rho-bar) (an NCCL all-gather of each rank's boundary block),
    the force pass and gather, and the all-reduce of energy and virial; the
    forces stay with their owners, as they would in a spatially split MD
    run.  Timed with CUDA events, max over ranks."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    import akitsushima_b200 as ak
    from akitsushima_b200 import _lib
    from akitsushima_b200.spatial import SlabState, exchange_fprime
    backend = os.environ.get("MBF_BENCH_BACKEND", "nccl")
    n_dev = torch.cuda.device_count()
    torch.cuda.set_device(local % n_dev)
    dist.init_process_group(backend, timeout=timedelta(seconds=120))
    dev = torch.device("cuda", torch.cuda.current_device())
    rng = np.random.default_rng(0)
    a, c = 3.58, args.cells
    frac = (np.asarray([[0, 0, 0], [0, 0.5, 0.5], [0.5, 0, 0.5], [0.5, 0.5, 0]], float)[None]
            + np.stack(np.meshgrid(np.arange(c), np.arange(c), np.arange(c * world), indexing="ij"),
                       -1).reshape(-1, 3)[:, None]).reshape(-1, 3)
    pos = frac * a + rng.normal(0.0, 0.08, frac.shape)
    ids = np.random.default_rng(1).integers(0, 2, len(pos)).astype(np.int32)
    lat = np.diag([a * c, a * c, a * c * world])
    n_atoms = len(pos)
    fn = ak.force_fn_from_config({"type": "EAM", "form": "zhou2004", "elements": ["Cu", "Ni"]},
                                 precision=args.precision)
    pot = fn.engine.potentials[0]
    pot.lanes_per_atom = args.lanes
    st = SlabState(pot, lat, pos, ids, rank, world, 0.3, dev)
    st.batch.set_positions(pos[st.local], check=False)
    out = None
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    ew = torch.zeros(10, dtype=torch.float64, device=dev)

    def step():
        nonlocal out
        fp = pot.embedding(st.batch, st.dlist, ws=st.ws)
        fp = exchange_fprime(fp, st.plan)
        out = pot.forces_from_embedding(st.batch, st.dlist, fp, ws=st.ws, out=out)
        ew[0] = out.energy[0]
        ew[1:] = out.virial[0]
        dist.all_reduce(ew)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    _lib.profile_begin()
    step()
    prof = _lib.profile_end()
    with ClockSampler(local % n_dev) as clk:
        dist.barrier()
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record()
            step()
            ev[k][1].record()
        torch.cuda.synchronize()
        dist.barrier()
    ms = sum(x.elapsed_time(y) for x, y in ev) / args.steps
    t = torch.tensor([ms], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    e_total = float(ew[0].item())
    # end to end: host arrays in, every rank the whole result back
    sfn = ak.SpatialForceFn(pot, skin=0.3, device=dev)
    types = [("Cu", "Ni")[k] for k in ids.tolist()]
    sfn(lat, pos, types)
    dist.barrier()
    t0 = time.perf_counter()
    n_e2e = max(1, min(args.e2e_steps, 10))
    for _ in range(n_e2e):
        e_, F_, s_ = sfn(lat, pos, types)
    t_e2e = (time.perf_counter() - t0) / n_e2e
    tt = torch.tensor([t_e2e], device=dev, dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    t_e2e = float(tt.item())
    clocks = clk.summary()
    n_local = len(st.local)
    dist.barrier()
    del st, sfn
    dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": METRIC, "value": n_atoms / (ms * 1e-3), "unit": "atoms/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if args.precision == "mixed" else "f64",
            "data": "synthetic",
            "config": {"workload": f"eam_zhou_cuni_fcc{c}x{c}x{c * world}_{n_atoms}_atoms_spatial",
                       "potential": "Zhou 2004 EAM Cu-Ni", "n_atoms": n_atoms, "atoms_per_gpu": n_atoms // world,
                       "a": a, "sigma": 0.08, "skin": 0.3, "precision": args.precision,
                       "l2": "256 MB scratch write between steps, outside the timed events",
                       "parallelism": f"spatial{world}: z slabs, halo of one list radius, F' all-gather "
                                      f"({backend}), energy / virial all-reduce"},
            "gpu_launches": int(sum(c_ for c_, _ in prof.values()) * args.steps),
            "kernels": {k: {"launches": c_, "ms_per_launch": t_ / c_} for k, (c_, t_) in prof.items()},
            "halo": {"local_atoms_rank0": n_local, "owned_atoms_rank0": n_atoms // world},
            "clocks": clocks, "check": {"energy_per_atom": e_total / n_atoms},
            "e2e": {"value": n_atoms / t_e2e, "unit": "atoms/s", "h2d_bytes_per_step": n_atoms * 24,
                    "d2h_bytes_per_step": n_atoms * 24 + 80, "ms_per_step": t_e2e * 1e3,
                    "path": "SpatialForceFn(lattice, numpy positions, species names) on every rank -> "
                            "the whole (E, F, stress) on every rank"},
            "cpu_baseline": None, "roofline": None}
    print(json.dumps(line), flush=True)
    return 0


# The other configurations, measured inside the default run and attached to
# its line (steps kept small so the whole run stays within a few minutes).
SUB_RECORDS = (
    ("fit_sic256", {"steps": 10, "warmup": 3, "e2e_steps": 10}),
    ("batched_si512", {"steps": 10, "warmup": 3, "e2e_steps": 20}),
    ("md_tersoff_si4096", {"steps": 10, "warmup": 3, "e2e_steps": 1, "drift_ps": 10.0}),
    ("md_sw_si64k", {"steps": 5, "warmup": 3, "e2e_steps": 1, "drift_ps": 10.0}),
)


def _summary(line):
    keep = ("metric", "value", "unit", "ms_per_step", "ms_per_md_step", "dtype", "structures_per_s",
            "per_structure_launches", "gpu_launches_per_step", "energy", "atom_force_evals_per_s",
            "n_variables", "check", "nve_drift")
    out = {k: line[k] for k in keep if k in line}
    out["workload"] = line["config"].get("workload")
    e = line.get("e2e") or {}
    out["e2e"] = {k: e.get(k) for k in ("value", "unit", "ms_per_step", "h2d_bytes_per_step",
                                          "d2h_bytes_per_step", "path")}
    c = line.get("cpu_baseline")
    if c:
        out["cpu_baseline"] = c
        out["vs_cpu_port"] = line["value"] / c["value"]
    return out


def sub_records(args):
    out = {}
    for wl, over in SUB_RECORDS:
        a = argparse.Namespace(**vars(args))
        a.workload, a.collect, a.precision, a.precision_given = wl, [], "mixed", False
        a.skip_singles = False
        for k, v in over.items():
            setattr(a, k, v)
        # the earlier workloads' objects (the 256k species-name lists among
        # them) out of the collector's way: each record times its own calls
        gc.collect()
        gc.freeze()
        t0 = time.perf_counter()
        try:
            fn = run_fit if wl in FIT_WORKLOADS else run_md if wl in MD_WORKLOADS else run_batched
            fn(a, 1, 0, 0)
            out[wl] = _summary(a.collect[0])
        except Exception as exc:  # a failed sub-record is reported, not fatal
            out[wl] = {"error": f"{type(exc).__name__}: {exc}"}
        out[wl]["wall_s"] = round(time.perf_counter() - t0, 2)
    return out


if __name__ == "__main__":
    sys.exit(main())
