"""Benchmark: bond-force updates/s of the per-step force path on B200.

One bench "step" is one full specimen run: ``--sim-steps`` velocity-Verlet
time steps (default: the workload's configured count) starting from the
same initial state, i.e. one pass of the hot path over one batch of
synthetic input.

  value     device time with the state resident in HBM (CUDA events on the
            library's stream), state/bond reset and an L2 flush between
            iterations (outside the timed region).
  e2e       the same run through the public API with host buffers: upload
            of y, v from pinned memory, the run, download of y, v and damage,
            all inside the timed region.
  roofline  algorithmic bytes of one step (per intact directed bond 4.125 B:
            a 4-byte neighbour index and one intact bit; per particle the
            state one step must stream: 84 B bond-based FP32C, 168 B FP64;
            state-based blocks sweep the bonds twice and add 8 B per
            particle) over the device time of one step, measured in the
            timed runs themselves: CUDA events on the library's stream
            around every replay of a captured multi-step graph and around
            the bond kernels of every directly launched step.

Default workload: 256 independent bond-based cuboids (edges U{12..32} per
axis, 2.8 M particles, 290 M bonds), 2000 steps in FP32C -- the largest
single-GPU configuration, larger than L2.

``--impl reference`` times the CPU restatement of the reference loop
(oracle/, OpenMP over particles on all host cores) on a bounded sample of
the same workload (for the batched workload: its first specimens).

Launch: python bench.py [--gpus N --steps K --warmup W]; for N > 1 under
torch.distributed.run, one rank per GPU, each rank advancing its own
specimen (independent specimens: weak scaling, no data-path collective).
"""
import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from peridyn_b200 import replicas  # noqa: E402  (host logic only; no library load)

METRIC = "bond-force updates/s"
UNIT = "bond-updates/s"


def build_workload(name, args):
    from peridyn_b200 import configs

    if name == "lps_bar":
        return configs.lps_bar()
    if name == "pmb_cube":
        return configs.pmb_cube()
    if name == "batched":
        return configs.batched_cubes(nspec=args.nspec, cubes=args.cubes)
    if name == "disk_impact":
        return configs.disk_impact()
    if name == "elasto_plastic":
        return configs.ep_bar()
    raise SystemExit(f"unknown workload {name}")


def step_bytes(intact_bonds, particles, precision, lps):
    """Algorithmic bytes of one step: per intact directed bond a 4-byte
    neighbour index plus its intact bit (4.125 B), counted once per bond
    sweep (twice for state-based blocks: dilatation and force); per
    particle the state a step streams -- FP32C bond-based: x, u read, u
    written (3 x 12 B) plus the FP64 position accumulator read and written
    (2 x 24 B) = 84 B; FP64: x 24 + y, v, a read and written (6 x 24) =
    168 B; state-based blocks add the dilatation written and read (8 B)."""
    sweeps = 2 if lps else 1
    per_particle = (84 if precision == "fp32c" else 168) + (8 if lps else 0)
    return sweeps * 4.125 * intact_bonds + per_particle * particles


# The layout's own byte count of one bond-force launch: the bond storage the
# walk must read (one intact bit per bond slot plus the neighbour-index
# array: one int32 per (slot, particle) in explicit slices, one per slot in
# stencil slices) and per particle the state the kernel streams (listed per
# precision below).
def bond_bytes(layout, ep=False):
    # elasto-plastic: per slot the plastic strain read and written (8 + 8)
    # plus, in the throughput modes, the reverse slot's index and strain (4 + 8)
    return layout["slots"] / 8.0 + 4.0 * layout["index_entries"] + (28.0 * layout["slots"] if ep else 0.0)


def particle_bytes(precision, lps):
    if precision == "fp64_serial":
        return 104 + (16 if lps else 0)  # x4 32 + y 32 + f 32 + cnt/tinfo 8 (+ m,theta 16)
    if precision == "fp64":
        # x4 32, u 32 read + 32 write, v 32 + 32, cnt/tinfo 8, 1/rho 8 (+ theta/m, 1/m 16)
        return 176 + (16 if lps else 0)
    # fp32c: x 16, u32 16 read + 16 write, FP64 accumulator 24 + 24, v 16 + 16,
    # cnt/tinfo 8, 1/rho 4, BC flags 1 (+ theta/m, 1/m 8)
    return 141 + (8 if lps else 0)


NEIGH_EVERY = 100  # contact neighbour update cadence (run!'s neigh_update_freq)


def advance(env, work, nsteps):
    """nsteps velocity-Verlet steps; with contacts the contact neighbours
    are rebuilt every NEIGH_EVERY steps, as run! does (solvers.jl:176-178)."""
    from peridyn_b200 import _abi

    L = _abi.lib()
    if not work["contacts"]:
        _abi.check(L.pd_env_vv_steps(env._h, nsteps))
        return
    done = 0
    while done < nsteps:
        k = min(NEIGH_EVERY, nsteps - done)
        _abi.check(L.pd_env_vv_steps(env._h, k))
        done += k
        if done < nsteps:
            _abi.check(L.pd_env_update_neighs(env._h, 30))


def accuracy_vs_serial(work, precision, sim_steps, env_fast, device):
    """Error of a throughput-mode run against the serial-order FP64 path
    (bit-identical to the CPU oracle) over the same run; for the contact
    workload and workloads above 200 k particles, whose serial runs would
    take minutes, against the one-pass FP64 GPU path (within 1e-10 of the
    oracle in the tests)."""
    import peridyn_b200 as pb

    big = sum(m.general.n for m in work["materials"]) > 200000
    ref_prec = "fp64" if (work["contacts"] or big) else "fp64_serial"
    ref = pb.Env(1, work["materials"], work["contacts"], work["bcs"], work["dt"], precision=ref_prec,
                 device=device)
    if work["bcs"]:
        pb.apply_bc_at0(ref, 0)
    pb.update_neighs(ref)
    pb.update_acc(ref)
    advance(ref, work, sim_steps)
    yr, vr, _, _ = ref.get_state()
    yf, vf, _, _ = env_fast.get_state()
    dr, df = pb.cal_damage(ref), pb.cal_damage(env_fast)
    x = np.hstack([m.general.x for m in work["materials"]])
    mism = 0
    broken = 0
    for b in range(len(work["materials"])):
        fr, ir = ref._family(b)
        _, i_f = env_fast._family(b)
        mism += int((ir != i_f).sum())
        broken += int((fr > 0).sum() - ir.sum())
    ref.close()
    l2 = lambda a, b: float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    vs = ("fp64 one-pass GPU path" if ref_prec == "fp64" else
          "fp64_serial GPU path (bit-identical to the CPU oracle)")
    return {"vs": vs, "vv_steps": int(sim_steps),
            "displacement_rel_l2": l2(yf - x, yr - x), "velocity_rel_l2": l2(vf, vr),
            "damage_rel_l2": l2(df, dr), "broken_bonds_fp64": broken, "broken_bond_mismatch": mism}


class ClockSampler:
    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def cpu_threads(work):
    """Host threads the oracle uses for this workload: all cores, except
    the elasto-plastic restatement, which is single-threaded."""
    if any(m.specific.kind == 3 for m in work["materials"]):
        return 1
    return os.cpu_count() or 1


def cpu_sample(work, seconds, nthreads):
    """Oracle (CPU restatement of the reference loop) on a bounded sample."""
    from oracle import oracle

    ora = oracle.OracleEnv(work["materials"], work["contacts"], work["bcs"], work["dt"], nthreads=nthreads)
    ora.apply_bc_at0()
    bonds0 = sum(int(B.intact.sum()) for B in ora.blocks)
    t0 = time.perf_counter()
    ora.vv_step()
    one = time.perf_counter() - t0
    nsteps = max(1, min(10000, int(seconds / max(one, 1e-6))))
    t0 = time.perf_counter()
    for _ in range(nsteps):
        ora.vv_step()
    dt = time.perf_counter() - t0
    bonds1 = sum(int(B.intact.sum()) for B in ora.blocks)
    rate = 0.5 * (bonds0 + bonds1) * nsteps / dt
    return rate, nsteps, dt


def traffic_for(workload, precision):
    """Per-launch DRAM bytes of the bond kernel from a committed ncu
    summary (profiles/roofline_traffic.json), or None."""
    p = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    try:
        d = json.load(open(p))
        return d.get(f"{workload}/{precision}")
    except (OSError, ValueError):
        return None


def time_precision(work, precision, sim_steps, device, flush, dist):
    """The same workload on another precision path: 1 warm-up and 2 timed
    runs, timed like the main measurement."""
    import torch

    import peridyn_b200 as pb
    from peridyn_b200 import _abi

    env = pb.Env(1, work["materials"], work["contacts"], work["bcs"], work["dt"], precision=precision,
                 device=device)
    L = _abi.lib()
    sp = ctypes_void()
    _abi.check(L.pd_env_stream(env._h, ctypes.byref(sp)))
    stream = torch.cuda.ExternalStream(sp.value, device=torch.device("cuda", device))
    y0, v0, _, _ = env.get_state()
    t_total, bonds = 0.0, 0.0
    for k in range(3):
        env.set_state(y=y0, v=v0, f=np.zeros_like(y0))
        _abi.check(L.pd_env_reset_bonds(env._h))
        _abi.check(L.pd_env_reset_deformed(env._h))
        env.time_step = 0
        if work["bcs"]:
            pb.apply_bc_at0(env, 0)
        pb.update_neighs(env)
        pb.update_acc(env)
        b0 = env.num_bonds()
        flush.zero_()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        advance(env, work, sim_steps)
        e1.record(stream)
        torch.cuda.synchronize()
        if k > 0:
            t_total += e0.elapsed_time(e1) / 1e3
            bonds += 0.5 * (b0 + env.num_bonds()) * sim_steps
    env.close()
    t_total, bonds = replicas.reduce_timing(t_total, bonds, dist, "cuda")
    return {"precision": precision, "value": bonds / t_total, "unit": UNIT, "ms_per_step": 1e3 * t_total / 2,
            "steps": 2, "warmup": 1}


def run_serving(args, rank, world, local):
    """Serving stream: Poisson arrivals of mixed PMB / state-based jobs
    submitted to a pd_server at their arrival times; aggregate bond-updates/s
    over the stream's wall time and p50/p99 job latency (submit to result),
    FP32C beside the plain FP64 GPU path.  One bench step = one stream."""
    import torch

    import peridyn_b200 as pb
    from peridyn_b200 import configs

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    # each rank serves its own stream (seeded by rank): independent jobs, no collective on the data path
    out = {}
    for precision in ("fp32c", "fp64"):
        # one global stream of jobs x world, dealt to the ranks by footprint
        jobs, arrivals = configs.serving_jobs(args.jobs * world, seed=5, precision=precision)
        mine = replicas.shard_by_footprint([w["materials"][0].general.n for w in jobs], world)[rank]
        jobs, arrivals = [jobs[i] for i in mine], [arrivals[i] for i in mine]
        warm, warm_arr = configs.serving_jobs(4, seed=99, n_lo=5e3, n_hi=2e4, steps_lo=100, steps_hi=200,
                                              precision=precision)
        with pb.Server(device=local, max_active=args.max_active) as srv:
            pb.serve_stream(srv, warm, [0.0] * len(warm))
            runs = []
            for _ in range(args.steps):
                if dist is not None:
                    dist.barrier()
                recs, summary = pb.serve_stream(srv, jobs, arrivals)
                runs.append(summary)
        wall, bonds = replicas.reduce_timing(max(r["wall_s"] for r in runs),
                                             sum(r["bond_updates"] for r in runs) / len(runs), dist, "cuda")
        out[precision] = {"value": bonds / wall, "wall_s": wall,
                          "latency_ms": runs[-1]["latency_ms"], "jobs": runs[-1]["jobs"]}
    if rank == 0:
        main = out["fp32c"]
        line = {"metric": METRIC, "value": main["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": 1, "ms_per_step": 1e3 * main["wall_s"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32 (f64 position accumulator)", "data": "synthetic",
                "config": {"workload": f"serving_{args.jobs}_jobs_poisson50", "max_active": args.max_active,
                           "sizes": "log-uniform 5e3..5e5 particles", "steps": "U{500..5000}",
                           "parallelism": f"one server per GPU x{world}" if world > 1 else "1 GPU"},
                "latency_ms": main["latency_ms"], "fp64_compare": out["fp64"],
                "e2e": {"value": main["value"], "unit": UNIT, "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                        "note": "serving is end to end: host job description in, host results out"}}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def cpu_workload(work, max_particles=120000):
    """The bounded sample of a workload the CPU arms time: the batched
    workload's first specimens up to about max_particles particles (the
    specimens are independent, so its per-bond rate is the workload's);
    other workloads whole."""
    mats = work["materials"]
    if not work["workload"].startswith("batched") or len(mats) <= 1:
        return work, work["workload"]
    n, k = 0, 0
    while k < len(mats) and (k == 0 or n + mats[k].general.n <= max_particles):
        n += mats[k].general.n
        k += 1
    sub = dict(work)
    sub["materials"] = mats[:k]
    return sub, f"first {k} of {len(mats)} specimens ({n} particles) of {work['workload']}"


def run_reference(args, rank, world):
    if rank != 0:
        return
    work, sample = cpu_workload(build_workload(args.workload, args))
    nthreads = cpu_threads(work)
    per_step = max(2.0, min(20.0, 150.0 / max(1, args.steps + args.warmup)))
    vals = []
    samples = []
    for k in range(args.warmup + args.steps):
        rate, n, dt = cpu_sample(work, per_step, nthreads)
        if k >= args.warmup:
            vals.append(rate)
            samples.append((n, dt))
    value = float(np.median(vals))
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": build_workload(args.workload, args)["workload"], "precision": "fp64",
                       "particles": None},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port",
                             "sample": f"{samples[0][0]} velocity-Verlet steps per bench step of {sample} "
                                       + ("(OpenMP, atomic scatter)" if nthreads > 1 else "(single thread)")},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batched",
                    choices=["lps_bar", "pmb_cube", "batched", "disk_impact", "elasto_plastic", "serving"])
    ap.add_argument("--jobs", type=int, default=48, help="serving: jobs per stream")
    ap.add_argument("--max-active", type=int, default=16, help="serving: most jobs resident at once")
    ap.add_argument("--no-pipe-peaks", action="store_true",
                    help="skip measuring the FP32 and MUFU pipe rates for the compute roofline")
    ap.add_argument("--precision", default="fp32c", choices=["fp64_serial", "fp64", "fp32c"])
    ap.add_argument("--no-fp64-compare", action="store_true",
                    help="skip timing the plain FP64 GPU path beside an FP32C run")
    ap.add_argument("--sim-steps", type=int, default=0, help="VV steps per bench step (default: workload's)")
    ap.add_argument("--nspec", type=int, default=256)
    ap.add_argument("--cubes", action="store_true",
                    help="batched: one drawn edge per specimen (cubes) instead of one per axis")
    ap.add_argument("--cpu-sample-s", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--no-serving", action="store_true",
                    help="skip the serving stream measured after the timed runs")
    ap.add_argument("--persist", action="store_true",
                    help="run flip-free stretches as one persistent cooperative launch (PD_PERSIST=1)")
    args = ap.parse_args()
    if args.persist:
        os.environ["PD_PERSIST"] = "1"
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "serving":
        run_serving(args, rank, world, local)
        return

    import torch

    import peridyn_b200 as pb
    from peridyn_b200 import _abi

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    work = build_workload(args.workload, args)
    sim_steps = args.sim_steps or work["steps"]
    t_setup = time.perf_counter()
    env = pb.Env(1, work["materials"], work["contacts"], work["bcs"], work["dt"], precision=args.precision,
                 device=local)
    setup_s = time.perf_counter() - t_setup  # assembly + finalize (families, layout, weighted volumes)
    L = _abi.lib()
    stream_ptr = ctypes_void()
    _abi.check(L.pd_env_stream(env._h, ctypes.byref(stream_ptr)))
    stream = torch.cuda.ExternalStream(stream_ptr.value, device=torch.device("cuda", local))
    lps = any(m.specific.kind in (1, 3) for m in work["materials"])
    ep = any(m.specific.kind == 3 for m in work["materials"])
    y0, v0, _, _ = env.get_state()
    # pinned host copies for the end-to-end arm
    hy = torch.from_numpy(np.ascontiguousarray(y0.T)).pin_memory()
    hv = torch.from_numpy(np.ascontiguousarray(v0.T)).pin_memory()
    out_y = torch.empty_like(hy).pin_memory()
    out_v = torch.empty_like(hv).pin_memory()
    out_d = torch.empty(env.N, dtype=torch.float64).pin_memory()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2

    def reset():
        env.set_state(y=y0, v=v0, f=np.zeros_like(y0))
        _abi.check(L.pd_env_reset_bonds(env._h))
        _abi.check(L.pd_env_reset_deformed(env._h))
        env.time_step = 0
        if work["bcs"]:
            pb.apply_bc_at0(env, 0)
        pb.update_neighs(env)
        pb.update_acc(env)  # the run's initial force evaluation (save_state! at t0)

    def one_run():
        advance(env, work, sim_steps)

    bonds_start = None
    # warm-up
    for _ in range(args.warmup):
        reset()
        one_run()
    # timed: device-resident; CUDA events on the library's stream bracket
    # every graph replay / direct step inside the run (pd_env_profile), which
    # times the bond kernels in the launch path the run takes
    times = []
    bonds = []
    prof_total_ms, prof_steps = 0.0, 0
    prof_ms = ctypes_double()
    prof_n = ctypes_i64()
    launches0 = _abi.kernel_launches()
    with ClockSampler(local) as clocks:
        for k in range(args.steps):
            reset()
            b0 = env.num_bonds()
            flush.zero_()
            _abi.check(L.pd_env_profile(env._h, 1))
            torch.cuda.synchronize()
            if dist is not None:
                dist.barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            one_run()
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
            _abi.check(L.pd_env_profile_read(env._h, ctypes.byref(prof_ms), ctypes.byref(prof_n)))
            _abi.check(L.pd_env_profile(env._h, 0))
            prof_total_ms += prof_ms.value
            prof_steps += prof_n.value
            b1 = env.num_bonds()
            bonds.append(0.5 * (b0 + b1) * sim_steps)
            bonds_start = b0
    launches = _abi.kernel_launches() - launches0
    t_total, total_bonds = replicas.reduce_timing(sum(times), sum(bonds), dist, "cuda")
    value = total_bonds / t_total
    # end-to-end through the public API with host buffers
    h2d = hy.numel() * 8 + hv.numel() * 8
    d2h = out_y.numel() * 8 + out_v.numel() * 8 + out_d.numel() * 8
    e2e_times = []
    for _ in range(args.steps):
        _abi.check(L.pd_env_reset_bonds(env._h))
        _abi.check(L.pd_env_reset_deformed(env._h))
        env.time_step = 0
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        yv = hy.numpy().T
        vv = hv.numpy().T
        _abi.check(L.pd_env_set_state(env._h, _abi.dptr(np.asfortranarray(yv)), _abi.dptr(np.asfortranarray(vv)),
                                      None))
        if work["bcs"]:
            pb.apply_bc_at0(env, 0)
        pb.update_neighs(env)
        pb.update_acc(env)
        one_run()
        ybuf = out_y.numpy()
        vbuf = out_v.numpy()
        _abi.check(L.pd_env_get_state(env._h, ybuf.ctypes.data_as(_abi.c_dp), vbuf.ctypes.data_as(_abi.c_dp),
                                      None, None))
        _abi.check(L.pd_env_damage(env._h, out_d.numpy().ctypes.data_as(_abi.c_dp)))
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_times.append(e0.elapsed_time(e1) / 1e3)
    e2e_t, _ = replicas.reduce_timing(sum(e2e_times), 0.0, dist, "cuda")
    e2e_value = total_bonds / e2e_t
    # the state now holds one complete run from the initial state
    accuracy = None
    if args.precision != "fp64_serial" and rank == 0 and not args.no_accuracy:
        accuracy = accuracy_vs_serial(work, args.precision, sim_steps, env, local)
    # roofline of one step (bond-based: the fused k_step launch)
    n_real = sum(m.general.n for m in work["materials"])
    n_int = sum(((m.general.n + 31) // 32) * 32 for m in work["materials"])
    layout = env.layout()
    shape = env.kernel_shape()
    mean_bonds = sum(bonds) / max(1, len(bonds)) / sim_steps
    bytes_step = step_bytes(mean_bonds, n_real, args.precision, lps)
    bytes_layout = bond_bytes(layout, ep) + n_int * particle_bytes(args.precision, lps)
    avg_ms = prof_total_ms / max(1, prof_steps)
    achieved = bytes_step / (avg_ms * 1e-3) / 1e9 if avg_ms > 0 else None
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    traffic = traffic_for(work["workload"], args.precision)
    clk = clocks.summary()
    fp64_cmp = None
    if args.precision == "fp32c" and not args.no_fp64_compare:  # every rank: it holds collectives
        fp64_cmp = time_precision(work, "fp64", sim_steps, local, flush, dist)
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": {"fp64_serial": "f64", "fp64": "f64", "fp32c": "f32 (f64 position accumulator)"}[args.precision],
        "data": "synthetic",
        "config": {"workload": work["workload"], "precision": args.precision, "particles": int(env.N),
                   "intact_bonds": int(bonds_start), "vv_steps_per_step": int(sim_steps), "dt": work["dt"],
                   "l2": "256 MB buffer written between timed iterations",
                   "parallelism": f"specimen replicas x{world}" if world > 1 else "1 GPU"},
        "hbm_gbs_algorithmic": bytes_step * sim_steps * args.steps / t_total / 1e9,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "kernel": ("k_force_serial" if args.precision == "fp64_serial" else
                                "k_theta + k_step (dilatation, fused bond force + velocity-Verlet)" if lps else
                                "k_step (fused bond force + velocity-Verlet), one launch per step"),
                     "bytes_per_launch": bytes_step,
                     "byte_model": "per step: 4.125 B per intact directed bond per bond sweep + "
                                   + ("84" if args.precision == "fp32c" else "168")
                                   + (" + 8" if lps else "") + " B per particle",
                     "layout_bytes_per_launch": bytes_layout,
                     "avg_launch_ms": avg_ms, "launches_timed": int(prof_steps),
                     "launch_timing": "CUDA events on the library's stream around every graph replay and "
                                      "every directly launched step of the timed runs",
                     "peak_source": f"{peak_src} MEASURED_PEAKS.json hbm_gbs" if peak_src == "measured"
                     else "fallback 6650 GB/s"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "clocks": clk,
        "accuracy": accuracy,
    }
    line["config"]["bond_layout"] = layout
    line["config"]["slot_efficiency"] = float(bonds_start) / max(1, layout["slots"])
    # the same over the slots the kernels walk (without each slice's padding
    # of its slot list to a multiple of 32)
    line["config"]["slot_efficiency_walked"] = float(bonds_start) / max(1, layout["walked_slots"])
    line["config"]["setup_s"] = setup_s
    line["config"]["kernel_shape"] = {"warps_per_slice": shape[0], "unroll": shape[1], "chosen_by":
                                      "PD_KERNEL_SHAPE" if os.environ.get("PD_KERNEL_SHAPE") else "autotuner"}
    line["config"]["launch_path"] = ("persistent cooperative kernel over flip-free runs" if args.persist else
                                     "CUDA graphs of 32 steps" if not work["contacts"] else
                                     "CUDA graphs of 32 steps between contact neighbour updates")
    if args.precision == "fp32c" and not lps and not args.no_pipe_peaks:
        line["compute"] = compute_roofline(layout["walked_slots"], avg_ms, local)
    if fp64_cmp is not None:
        line["fp64_compare"] = fp64_cmp
    if world == 1 and not args.no_cpu_baseline:
        sub, sample = cpu_workload(work)
        nth = cpu_threads(sub)
        rate, n, dt = cpu_sample(sub, args.cpu_sample_s, nth)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": nth, "kind": "port",
                                "sample": f"{n} velocity-Verlet steps of {sample} in {dt:.1f} s "
                                          + ("(OpenMP over particles, atomic scatter)" if nth > 1 else
                                             "(single thread)")}
    env.close()
    if world == 1 and not args.no_serving:
        line["serving"] = serving_sample(args, local)
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def serving_sample(args, device):
    """One serving stream after the timed runs (outside the timed region):
    args.jobs FP32C jobs of mixed size and kind (log-uniform 5e3..5e5
    particles, U{500..5000} steps, PMB and state-based) submitted to a
    pd_server at Poisson arrival times (50 jobs/s, seed 5), after a warm-up
    stream of 4 small jobs; p50/p99 latency from submission to result and
    the aggregate bond-updates/s over the stream's wall time."""
    import peridyn_b200 as pb
    from peridyn_b200 import configs

    jobs, arrivals = configs.serving_jobs(args.jobs, seed=5, precision="fp32c")
    warm, _ = configs.serving_jobs(4, seed=99, n_lo=5e3, n_hi=2e4, steps_lo=100, steps_hi=200, precision="fp32c")
    with pb.Server(device=device, max_active=args.max_active) as srv:
        pb.serve_stream(srv, warm, [0.0] * len(warm))
        _, summary = pb.serve_stream(srv, jobs, arrivals)
    return {"workload": f"serving_{args.jobs}_jobs_poisson50", "precision": "fp32c", "max_active": args.max_active,
            "jobs": summary["jobs"], "wall_s": summary["wall_s"], "latency_ms": summary["latency_ms"],
            "aggregate_bond_updates_per_s": summary["bond_updates_per_s"],
            "timing": "wall clock from the first submission to the last result, after the timed runs"}


# Per slot of the FP32C bond-based stencil walk (one lane, one bond slot),
# counted from the walk's source: FP32-pipe lane operations, a multiply-add
# counting once -- bond vector 3, displacement difference 3, deformed bond 3,
# 2 xi + eta 3, |xi|^2 4, numerator e.(2 xi + e) 4, |Y|^2 1, (|Y|+|xi|)|xi| 1,
# critical-stretch test 1, 1/(dl |Y|) operand 1, c V num 1, coefficient 1,
# force accumulation 3 -- and MUFU operations: sqrt.approx twice,
# rcp.approx once.
FP32_OPS_PER_SLOT = 29
MUFU_OPS_PER_SLOT = 3


def compute_roofline(slots, avg_ms, device):
    """The bond walk's compute side against the GPU's measured pipe rates
    (pd_pipe_peaks): lane operations of one step's slots divided by the
    measured step time, as fractions of the FP32 FMA pipe and of the MUFU
    pipe."""
    from peridyn_b200 import _abi

    peaks = _abi.pipe_peaks(device)
    if not avg_ms or avg_ms <= 0:
        return {"pipe_peaks": peaks}
    t = avg_ms * 1e-3
    fp32 = FP32_OPS_PER_SLOT * slots / t
    mufu = MUFU_OPS_PER_SLOT * slots / t
    mufu_peak = min(peaks["sqrt_approx_lane_ops_per_s"], peaks["rcp_approx_lane_ops_per_s"])
    return {"slots_per_launch": int(slots), "fp32_ops_per_slot": FP32_OPS_PER_SLOT,
            "mufu_ops_per_slot": MUFU_OPS_PER_SLOT,
            "fp32_achieved": fp32, "fp32_peak": peaks["ffma_lane_ops_per_s"],
            "fp32_frac": fp32 / peaks["ffma_lane_ops_per_s"],
            "mufu_achieved": mufu, "mufu_peak": mufu_peak, "mufu_frac": mufu / mufu_peak,
            "unit": "lane ops/s", "pipe_peaks": peaks,
            "peak_source": "measured in this run (pd_pipe_peaks)"}


def ctypes_void():
    import ctypes

    return ctypes.c_void_p()


def ctypes_double():
    import ctypes

    return ctypes.c_double()


def ctypes_i64():
    import ctypes

    return ctypes.c_int64()


if __name__ == "__main__":
    main()
