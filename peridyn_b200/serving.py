"""Serving: continuous batching of simulation jobs on one GPU
(``pd_server_*`` of libperidyn_b200.so).

A job is a complete simulation -- materials, contacts, boundary conditions,
dt, a step count and a precision -- run the way ``run!`` starts one
(solvers.jl:97-187: BC snapshot, force evaluation at t0, then velocity-
Verlet steps).  The server admits queued jobs while their estimated HBM
footprints fit the budget, keeps admitted jobs resident and advances each on
its own stream in chunks, so jobs that arrive while others run share the
device.  Results come back in the environment's particle order.
"""
import ctypes
import time

import numpy as np

from . import _abi
from .environment import GeneralEnvironment


class Server:
    def __init__(self, device=0, hbm_budget=0, max_active=16, chunk_steps=128):
        h = ctypes.c_void_p()
        _abi.check(_abi.lib().pd_server_create(ctypes.byref(h), int(device), int(hbm_budget), int(max_active),
                                               int(chunk_steps)))
        self._h = h
        self.device = int(device)
        self._n = {}

    def submit(self, materials, short_range_contact, boundary_conds, dt, nsteps, precision="fp32c"):
        """Queue a job; returns its id."""
        env = GeneralEnvironment(1, materials, short_range_contact, boundary_conds, dt, precision=precision,
                                 device=self.device, finalize=False)
        n = env.N
        handle = env._detach()
        job = ctypes.c_int64()
        st = _abi.lib().pd_server_submit(self._h, handle, int(nsteps), ctypes.byref(job))
        if st != _abi.PD_OK:
            _abi.lib().pd_env_destroy(handle)
            _abi.check(st)
        self._n[job.value] = n
        return int(job.value)

    @staticmethod
    def _info(info):
        return {"state": _abi.JOB_STATES.get(info.state, str(info.state)), "status": int(info.status),
                "steps_done": int(info.steps_done), "particles": int(info.particles),
                "footprint_bytes": int(info.footprint_bytes), "bond_updates": int(info.bond_updates),
                "queue_ms": float(info.queue_ms), "latency_ms": float(info.latency_ms)}

    def poll(self, job):
        info = _abi.JobInfo()
        _abi.check(_abi.lib().pd_server_poll(self._h, int(job), ctypes.byref(info)))
        return self._info(info)

    def poll_state(self, job):
        """The job's state name; does not raise for a failed job."""
        info = _abi.JobInfo()
        _abi.lib().pd_server_poll(self._h, int(job), ctypes.byref(info))
        return _abi.JOB_STATES.get(info.state, str(info.state))

    def wait(self, job, timeout=600.0):
        info = _abi.JobInfo()
        _abi.check(_abi.lib().pd_server_wait(self._h, int(job), float(timeout), ctypes.byref(info)))
        return self._info(info)

    def result(self, job):
        """(y, v, damage) of a finished job; releases the job's record."""
        n = self._n.pop(int(job))
        y = np.zeros((3, n), order="F")
        v = np.zeros((3, n), order="F")
        d = np.zeros(n)
        _abi.check(_abi.lib().pd_server_result(self._h, int(job), _abi.dptr(y), _abi.dptr(v), _abi.dptr(d)))
        return y, v, d

    def cancel(self, job):
        _abi.check(_abi.lib().pd_server_cancel(self._h, int(job)))

    def close(self):
        if getattr(self, "_h", None):
            _abi.lib().pd_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def percentile(values, q):
    """q-th percentile (0..100) by linear interpolation between order statistics."""
    a = np.sort(np.asarray(values, dtype=np.float64))
    if a.size == 0:
        return float("nan")
    pos = (a.size - 1) * q / 100.0
    lo = int(np.floor(pos))
    hi = min(lo + 1, a.size - 1)
    return float(a[lo] + (a[hi] - a[lo]) * (pos - lo))


def serve_stream(server, jobs, arrivals):
    """Submit ``jobs`` (dicts with materials, contacts, bcs, dt, nsteps,
    precision) at the ``arrivals`` times (seconds from now), wait for all,
    and return per-job records and the stream's summary: p50/p99 latency and
    the aggregate bond-updates/s over the wall time of the stream."""
    t0 = time.perf_counter()
    ids = []
    for w, ta in zip(jobs, arrivals):
        delay = ta - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        ids.append(server.submit(w["materials"], w["contacts"], w["bcs"], w["dt"], w["nsteps"],
                                 precision=w.get("precision", "fp32c")))
    recs = [server.wait(j) for j in ids]
    wall = time.perf_counter() - t0
    for j in ids:
        server.result(j)
    lat = [r["latency_ms"] for r in recs]
    bonds = sum(r["bond_updates"] for r in recs)
    return recs, {"jobs": len(recs), "wall_s": wall, "latency_ms": {"p50": percentile(lat, 50),
                                                                      "p99": percentile(lat, 99),
                                                                      "max": max(lat) if lat else None},
                  "bond_updates": int(bonds), "bond_updates_per_s": bonds / wall if wall > 0 else None}
