"""Solvers and the run loop mirroring src/solvers/*.jl.

Every call dispatches to the device (libperidyn_b200.so); the host only
sequences the calls with the reference's cadence (solvers.jl:97-187).
"""
import ctypes

import numpy as np

from . import _abi
from .environment import GeneralEnvironment


class Solver:
    pass


class DSVelocityVerlet(Solver):
    """velocity_verlet.jl:9-10."""


class QSDrag(Solver):
    """minimize.jl:25-56: ``QSDrag(step_size, drag; max_iter=1000,
    x_tol=1e-3, f_tol=1e-3)``."""

    def __init__(self, step_size, drag, max_iter=1000, x_tol=1.0e-3, f_tol=1.0e-3):
        self.step_size = float(step_size)
        self.drag = float(drag)
        self.max_iter = int(max_iter)
        self.x_tol = float(x_tol)
        self.f_tol = float(f_tol)
        self.last_iterations = 0


SOLVERS = {"vv": DSVelocityVerlet, "qs": QSDrag}


def update_acc(env):
    """solvers.jl:320-336 ``update_acc!``."""
    _abi.check(_abi.lib().pd_env_update_acc(env._h))


def velocity_verlet_step(env, solver=None, nsteps=1):
    """velocity_verlet.jl:57-89 ``velocity_verlet_step!`` (nsteps times)."""
    _abi.check(_abi.lib().pd_env_vv_steps(env._h, int(nsteps)))


def minimize(env, solver):
    """minimize.jl:105-231 ``minimize!``; returns the iteration count."""
    it = ctypes.c_int64()
    _abi.check(_abi.lib().pd_env_qsdrag(env._h, solver.step_size, solver.drag, solver.max_iter, solver.x_tol,
                                        solver.f_tol, ctypes.byref(it)))
    solver.last_iterations = int(it.value)
    return int(it.value)


def apply_solver(env, solver):
    """``apply_solver!`` (velocity_verlet.jl:27, minimize.jl:74)."""
    if isinstance(solver, DSVelocityVerlet):
        velocity_verlet_step(env, solver)
    elif isinstance(solver, QSDrag):
        minimize(env, solver)
    else:
        raise TypeError(f"unknown solver {solver!r}")


def apply_bc_at0(env, start_at):
    """solvers.jl:200-206."""
    if start_at == 0:
        _abi.check(_abi.lib().pd_env_apply_bc_at0(env._h))


def update_neighs(envs, max_part=30):
    """solvers.jl:351-361 ``update_neighs!``."""
    if isinstance(envs, GeneralEnvironment):
        envs = [envs]
    for env in envs:
        if env.state == 2 and env.short_range_contact:
            _abi.check(_abi.lib().pd_env_update_neighs(env._h, int(max_part)))


def cal_damage(env):
    """peri.jl:587-594."""
    d = np.zeros(env.N)
    _abi.check(_abi.lib().pd_env_damage(env._h, _abi.dptr(d)))
    return d


def printdata(env):
    """environment.jl:308-320: the logged quantities as a dict."""
    out = np.zeros(8)
    _abi.check(_abi.lib().pd_env_diagnostics(env._h, _abi.dptr(out)))
    return {"envID": env.id, "time": env.time_step * env.dt, "px": out[0], "py": out[1], "pz": out[2],
            "Fx": out[3], "Fy": out[4], "Fz": out[5], "damage": out[6]}


def save_state(env, writer=None, filename=None):
    """io.jl:44-54 ``save_state!``: update_acc!, damage, then hand the
    arrays to ``writer(filename, data)`` (file formats stay with the host)."""
    update_acc(env)
    damage = cal_damage(env)
    if writer is not None:
        y, v, f, _ = env.get_state()
        writer(filename, {"id": np.arange(1, env.N + 1), "type": env.type, "position": y, "velocity": v,
                          "acceleration": f, "mass": env.mass, "volume": env.volume, "damage": damage})
    return damage


class _StagedWriter:
    """save_state! through the output staging slots: the snapshot is
    copied to pinned memory while the next steps run, and the writer is
    called for it just before its slot is needed again (or at the end)."""

    def __init__(self, writer):
        self.writer = writer
        self.pending = {}  # id(env) -> list of (slot, filename, env)
        self.next_slot = {}

    def save(self, env, filename):
        update_acc(env)
        q = self.pending.setdefault(id(env), [])
        slot = self.next_slot.get(id(env), 0)
        for item in [p for p in q if p[0] == slot]:
            self._emit(item)
            q.remove(item)
        env.stage_state(slot)
        q.append((slot, filename, env))
        self.next_slot[id(env)] = 1 - slot

    def _emit(self, item):
        slot, filename, env = item
        d = env.read_stage(slot)
        self.writer(filename, {"id": np.arange(1, env.N + 1), "type": env.type, "position": d["position"],
                               "velocity": d["velocity"], "acceleration": d["acceleration"], "mass": env.mass,
                               "volume": env.volume, "damage": d["damage"]})

    def flush(self):
        for q in self.pending.values():
            for item in q:  # in the order they were taken
                self._emit(item)
            q.clear()


def _print_data_file(envs, step, writer, ext):
    for env in envs:
        name = f"env_{env.id}_step_{step}.{ext}"
        if isinstance(writer, _StagedWriter):
            writer.save(env, name)
        else:
            save_state(env, writer, name)


def run(envs, N, solver, filewrite_freq=10, neigh_update_freq=1, average_prop_freq=1, out_dir="datafile",
        start_at=0, write_from=0, ext="jld", max_part=30, writer=None, logger=None, staged_io=True):
    """solvers.jl:97-187 ``run!`` with the reference's cadence: a force
    evaluation at every file write (including the initial two), contact
    neighbour updates every ``neigh_update_freq`` steps, diagnostics every
    ``average_prop_freq`` steps.  Consecutive velocity-Verlet steps with no
    event between them are issued as one device call."""
    if isinstance(envs, GeneralEnvironment):
        envs = [envs]
    # with staged_io the snapshots reach the writer through pinned staging
    # buffers, overlapping the copies with the next steps
    if writer is not None and staged_io:
        writer = _StagedWriter(writer)
    _print_data_file(envs, "start_with", writer, ext)
    update_neighs(envs, max_part)
    for env in envs:
        if env.state == 2:
            apply_bc_at0(env, start_at)
    _print_data_file(envs, 0 + write_from, writer, ext)
    last = N + start_at
    i = 1 + start_at

    def event(k):
        return ((k % average_prop_freq == 0 or (k == 1 and write_from == 0)) and logger is not None) or \
               (k % filewrite_freq == 0 or (k == 1 and write_from == 0)) or (k % neigh_update_freq == 0)

    while i <= last:
        chunk = 1
        if isinstance(solver, DSVelocityVerlet) and all(e.Collect is None for e in envs):
            while i + chunk - 1 < last and not event(i + chunk - 1):
                chunk += 1
        for env in envs:
            if env.state == 2:
                if isinstance(solver, DSVelocityVerlet):
                    velocity_verlet_step(env, solver, nsteps=chunk)
                else:
                    apply_solver(env, solver)
                if env.Collect is not None:
                    env.Collect(env, i)
        i += chunk - 1
        if logger is not None and (i % average_prop_freq == 0 or (i == 1 and write_from == 0)):
            logger({"Step": i, "envs": [printdata(env) for env in envs]})
        if i % filewrite_freq == 0 or (i == 1 and write_from == 0):
            _print_data_file(envs, i + write_from, writer, ext)
        if i % neigh_update_freq == 0:
            update_neighs(envs, max_part)
        i += 1
    _print_data_file(envs, "end_with", writer, ext)
    if isinstance(writer, _StagedWriter):
        writer.flush()


def simulate(*args, out_dir="datafile", append_date=True, **kwargs):
    """solvers.jl:62-68."""
    return run(*args, out_dir=out_dir, **kwargs)
