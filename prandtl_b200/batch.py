"""Batches of independent DGSEM solves and the serving loop over them.

``Batch`` wraps ``prandtl_batch_*``: many solves of uneven meshes, orders and
physics constants stay resident in one device arena and advance together.
Per RK stage, each (dim, order, physics) class runs one persistent lifting
launch and one persistent RHS + stage-update launch over all its solves.  The
step is captured once in a CUDA graph and replayed.  ``Server`` wraps
``prandtl_serve_*``: a native worker thread admits submitted solves as arena
room frees up and batches their stages with the resident ones (continuous
batching).

Every call goes to the CUDA kernels; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .mesh import Mesh
from .operator import MeshArrays, _ptr, make_config

_SCHEMES = {"RK3SSP": _lib.RK3SSP, "LSRK45": _lib.LSRK45}
_PREC = {"fp64": 0, "fp32": 1}


def _batch_config(precision, scheme, arena_bytes, max_solves, steps_per_graph, use_graph, timeout_s):
    L = _lib.load()
    c = _lib.BatchConfig()
    L.prandtl_batch_config_default(C.byref(c))
    if precision not in _PREC:
        raise ValueError("precision must be 'fp64' or 'fp32'")
    if scheme not in _SCHEMES:
        raise ValueError("scheme must be 'LSRK45' or 'RK3SSP'")
    c.precision = _PREC[precision]
    c.scheme = _SCHEMES[scheme]
    c.arena_bytes = int(arena_bytes)
    c.max_solves = int(max_solves)
    c.steps_per_graph = int(steps_per_graph)
    c.use_graph = int(bool(use_graph))
    c.timeout_s = float(timeout_s)
    return c


def _solve_desc(mesh: Mesh, dt, nsteps, cfl, hmin, t_final=0.0):
    return _lib.SolveDesc(float(dt), float(cfl), float(mesh.hmin if hmin is None else hmin), int(nsteps),
                          float(t_final))


class Batch:
    """Resident solves advanced together (see module docstring)."""

    def __init__(self, precision="fp32", scheme="LSRK45", *, arena_bytes=0, max_solves=4096,
                 steps_per_graph=4, use_graph=True, timeout_s=120.0):
        self._L = L = _lib.load()
        c = _batch_config(precision, scheme, arena_bytes, max_solves, steps_per_graph, use_graph, timeout_s)
        h = C.c_void_p()
        _lib.check(L.prandtl_batch_create(C.byref(c), C.byref(h)), None, "prandtl_batch_last_error")
        self._h = h
        self.precision, self.scheme = precision, scheme
        self._shape = {}
        self._nf = {}

    def _check(self, st):
        _lib.check(st, self._h, "prandtl_batch_last_error")

    def footprint(self, mesh: Mesh, **phys) -> int:
        arr = MeshArrays(mesh)
        cfg = make_config(**phys)
        n = C.c_size_t()
        self._check(self._L.prandtl_batch_footprint(self._h, C.byref(arr.desc), C.byref(cfg), C.byref(n)))
        return n.value

    def add(self, mesh: Mesh, u0, *, dt, nsteps, cfl=0.0, hmin=None, t_final=0.0, **phys) -> int:
        """Admit a solve; raises PrandtlError(ENOMEM) when the arena has no room.
        cfl > 0 updates dt from each step's lambda_max; t_final > 0 stops the
        solve at that time (the last step shortened to reach it)."""
        arr = MeshArrays(mesh)
        cfg = make_config(**phys)
        p, flag = _ptr(u0)
        sd = _solve_desc(mesh, dt, nsteps, cfl, hmin, t_final)
        sid = C.c_int(-1)
        self._check(self._L.prandtl_batch_add(self._h, C.byref(arr.desc), C.byref(cfg), p, flag,
                                              C.byref(sd), C.byref(sid)))
        self._shape[sid.value] = (mesh.num_fields * mesh.ndof,)
        self._nf[sid.value] = mesh.num_fields
        return sid.value

    def advance(self, nsteps: int):
        self._check(self._L.prandtl_batch_advance(self._h, int(nsteps)))

    def sync(self):
        self._check(self._L.prandtl_batch_sync(self._h))

    def finished(self) -> list:
        cap = max(1, len(self._shape))
        ids = (C.c_int * cap)()
        n = C.c_int()
        self._check(self._L.prandtl_batch_finished(self._h, ids, cap, C.byref(n)))
        return list(ids[: min(n.value, cap)])

    def query(self, sid: int) -> dict:
        left, done = C.c_int(), C.c_int()
        dt, lam = C.c_double(), C.c_double()
        self._check(self._L.prandtl_batch_query(self._h, int(sid), C.byref(left), C.byref(done),
                                                C.byref(dt), C.byref(lam)))
        return {"steps_left": left.value, "steps_done": done.value, "dt": dt.value, "lambda_max": lam.value}

    def time(self, sid: int) -> float:
        """Simulated time of the solve (the sum of its steps' dt)."""
        t = C.c_double()
        self._check(self._L.prandtl_batch_time(self._h, int(sid), C.byref(t)))
        return t.value

    def add_many(self, solves) -> list:
        """Admit several solves at once (prandtl_batch_add_many): `solves` holds
        (mesh, u0, dict(dt=..., nsteps=..., [cfl, hmin, t_final,] **phys)) items;
        their mesh checks and tables are prepared on several host threads.  All
        u0 are host arrays or all device tensors.  Raises PrandtlError for the
        first solve that fails; the ones before it stay admitted."""
        n = len(solves)
        keep, descs, cfgs, ptrs, flags = [], [], [], [], set()
        sds = (_lib.SolveDesc * max(n, 1))()
        for k, (mesh, u0, kw) in enumerate(solves):
            kw = dict(kw)
            dt, nsteps = kw.pop("dt"), kw.pop("nsteps")
            cfl, hmin, t_final = kw.pop("cfl", 0.0), kw.pop("hmin", None), kw.pop("t_final", 0.0)
            arr = MeshArrays(mesh)
            cfg = make_config(**kw)
            p, flag = _ptr(u0)
            keep += [arr, cfg, u0]
            descs.append(C.addressof(arr.desc))
            cfgs.append(C.addressof(cfg))
            ptrs.append(p)
            flags.add(flag)
            sds[k] = _solve_desc(mesh, dt, nsteps, cfl, hmin, t_final)
        if len(flags) > 1:
            raise ValueError("add_many takes host or device initial states, not both")
        ids = (C.c_int * max(n, 1))()
        st = self._L.prandtl_batch_add_many(self._h, n, (C.c_void_p * max(n, 1))(*descs),
                                            (C.c_void_p * max(n, 1))(*cfgs), (C.c_void_p * max(n, 1))(*ptrs),
                                            flags.pop() if flags else 0, sds, ids)
        out = [int(ids[k]) for k in range(n)]
        for k, (mesh, _, _) in enumerate(solves):
            if out[k] >= 0:
                self._shape[out[k]] = (mesh.num_fields * mesh.ndof,)
                self._nf[out[k]] = mesh.num_fields
        self._check(st)
        return out

    def read(self, sid: int, out=None):
        if out is None:
            out = np.empty(self._shape[sid], dtype=np.float64)
        p, flag = _ptr(out)
        self._check(self._L.prandtl_batch_read(self._h, int(sid), p, flag))
        return out

    def read_many(self, sids, outs=None):
        """States of several solves with two waits in all (prandtl_batch_read_many);
        outs: arrays or tensors of one kind (host or device), one per id."""
        sids = [int(x) for x in sids]
        if outs is None:
            outs = [np.empty(self._shape[x], dtype=np.float64) for x in sids]
        ptrs = [_ptr(o) for o in outs]
        flags = {f for _, f in ptrs}
        if len(flags) > 1:
            raise ValueError("read_many takes host or device outputs, not both")
        ids = (C.c_int * len(sids))(*sids)
        arr = (C.c_void_p * len(sids))(*[p for p, _ in ptrs])
        self._check(self._L.prandtl_batch_read_many(self._h, len(sids), ids, arr, flags.pop() if flags else 0))
        return outs

    def budgets(self, sid: int) -> dict:
        """FP64 integrals of the solve's resident state, reduced on the device:
        the conserved fields and the entropy function."""
        nf = self._nf[sid]
        out = np.zeros(nf + 1)
        self._check(self._L.prandtl_batch_budgets(self._h, int(sid), out.ctypes.data))
        return {"conserved": out[:nf].copy(), "entropy": float(out[nf])}

    def remove(self, sid: int):
        self._check(self._L.prandtl_batch_remove(self._h, int(sid)))
        self._shape.pop(sid, None)

    def tune(self, reps: int = 3):
        self._check(self._L.prandtl_batch_tune(self._h, int(reps)))

    def tune_in_steps(self):
        """Tune inside the next advances: their first n_variants steps run every
        class with one RHS launch shape each, timed by CUDA events, and the
        fastest shape is kept (the host waits for each of those steps)."""
        self._check(self._L.prandtl_batch_tune_in_steps(self._h))

    def class_info(self, dim: int, order: int, parabolic: bool):
        """(chosen RHS launch shape, tuned ms per RHS launch of each shape, tuned ms per lifting launch)."""
        v, n = C.c_int(), C.c_int()
        ms = (C.c_double * 8)()
        lift = C.c_double(-1.0)
        self._check(self._L.prandtl_batch_class_info(self._h, dim, order, int(parabolic), C.byref(v),
                                                     C.byref(n), ms, C.byref(lift)))
        return v.value, list(ms[: n.value]), lift.value

    @property
    def stream(self) -> int:
        """cudaStream_t of the batch (for torch.cuda.ExternalStream and event timing)."""
        return self._L.prandtl_batch_stream(self._h) or 0

    @property
    def device_bytes(self) -> int:
        return self._L.prandtl_batch_device_bytes(self._h)

    @property
    def kernel_launches(self) -> int:
        return self._L.prandtl_batch_kernel_launches(self._h)

    def close(self):
        if getattr(self, "_h", None):
            self._L.prandtl_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching request loop (see module docstring)."""

    def __init__(self, precision="fp32", scheme="LSRK45", *, steps_per_tick=4, arena_bytes=0,
                 max_solves=4096, steps_per_graph=4, use_graph=True, timeout_s=120.0):
        self._L = L = _lib.load()
        c = _batch_config(precision, scheme, arena_bytes, max_solves, steps_per_graph, use_graph, timeout_s)
        h = C.c_void_p()
        st = L.prandtl_serve_create(C.byref(c), int(steps_per_tick), C.byref(h))
        if st != _lib.PRANDTL_OK:
            raise _lib.PrandtlError(st, L.prandtl_batch_last_error(None).decode(errors="replace"))
        self._h = h
        self._out = {}

    def submit(self, mesh: Mesh, u0: np.ndarray, *, dt, nsteps, cfl=0.0, hmin=None, **phys) -> int:
        arr = MeshArrays(mesh)
        cfg = make_config(**phys)
        u0 = np.ascontiguousarray(u0, dtype=np.float64)
        out = np.empty_like(u0)
        sd = _solve_desc(mesh, dt, nsteps, cfl, hmin)
        t = C.c_longlong()
        st = self._L.prandtl_serve_submit(self._h, C.byref(arr.desc), C.byref(cfg), u0.ctypes.data, C.byref(sd),
                                          out.ctypes.data, C.byref(t))
        if st != _lib.PRANDTL_OK:
            raise _lib.PrandtlError(st, self._L.prandtl_serve_last_error(self._h).decode(errors="replace"))
        self._out[t.value] = out
        return t.value

    def poll(self, ticket: int):
        done, sec = C.c_int(), C.c_double()
        st = self._L.prandtl_serve_poll(self._h, ticket, C.byref(done), C.byref(sec))
        if st != _lib.PRANDTL_OK:
            raise _lib.PrandtlError(st, f"request {ticket} failed")
        return bool(done.value), sec.value

    def wait(self, ticket: int, timeout_s: float = 0.0):
        """(final state, submit-to-result seconds); the state buffer is released to the caller."""
        sec = C.c_double()
        st = self._L.prandtl_serve_wait(self._h, ticket, float(timeout_s), C.byref(sec))
        if st != _lib.PRANDTL_OK:
            raise _lib.PrandtlError(st, f"request {ticket}: " +
                                    self._L.prandtl_serve_last_error(self._h).decode(errors="replace"))
        return self._out.pop(ticket), sec.value

    def stats(self) -> dict:
        s = _lib.ServeStats()
        _lib.check(self._L.prandtl_serve_stats_get(self._h, C.byref(s)), None, "prandtl_serve_last_error")
        return {k: getattr(s, k) for k, _ in _lib.ServeStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            self._L.prandtl_serve_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
