"""Host-side mirror of the reference's projection interface.

``Projection`` owns one ``mf3d_ctx`` (device hierarchy for a fixed block
layout) and exposes the reference's entry points by name:

* ``newsolv_mg(fields, dt, alfapr)`` - newsolv_mg.for:2-102 on host arrays
  (the drop-in; host<->device copies inside the call);
* ``newsolv_mg_device(fields, dt, alfapr)`` - the same on device arrays
  (``torch.Tensor`` on the context's GPU);
* ``mgkcyc_device(su, pp)`` - one V-cycle, mgsolver.for:224-369.

Return values mirror the reference's module variables: ``rmax`` and
``iter``, plus the per-iteration rmax history the reference does not log.
Negative library statuses raise; ``NOT_CONVERGED`` / ``DIVERGED`` are
returned in ``info.status`` (the reference prints and continues / stops).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import abi

_dp = C.POINTER(C.c_double)


@dataclass
class SolveResult:
    status: int
    rmax: float
    rmax0: float
    iter: int
    ms_device: float
    history: np.ndarray


class Projection:
    def __init__(self, descriptors, params: abi.Params, lib=None):
        self.lib = lib or abi.load()
        self.nblocks = len(descriptors)
        self.desc = descriptors
        self.params = params
        ctx = C.c_void_p()
        st = self.lib.mf3d_create(descriptors, self.nblocks, C.byref(params), C.byref(ctx))
        abi.check(self.lib, st, "mf3d_create")
        self.ctx = ctx

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.mf3d_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _run(self, fn, fields_arr, dt, alfapr) -> SolveResult:
        cap = max(self.params.maxcy, 1)
        hist = np.zeros(cap)
        info = abi.SolveInfo()
        st = fn(self.ctx, fields_arr, C.c_double(dt), C.c_double(alfapr), C.byref(info),
                hist.ctypes.data_as(_dp), cap)
        abi.check(self.lib, st, fn.__name__)
        return SolveResult(st, info.rmax, info.rmax0, info.iter, info.ms_device, hist[:info.iter].copy())

    def newsolv_mg(self, blocks, dt=1.0, alfapr=1.0) -> SolveResult:
        """Host arrays (numpy, ttc layout) per block, updated in place."""
        from .problems import fields_struct
        return self._run(self.lib.mf3d_newsolv_mg, fields_struct(blocks), dt, alfapr)

    def newsolv_mg_device(self, blocks, dt=1.0, alfapr=1.0) -> SolveResult:
        """Device arrays (torch float64 CUDA tensors, ttc layout) per block."""
        arr = (abi.Fields * len(blocks))()
        for b, f in enumerate(blocks):
            for k in ("ustar", "vstar", "wstar", "u", "v", "w", "p", "su", "dens"):
                t = f.get(k)
                setattr(arr[b], k, C.cast(C.c_void_p(t.data_ptr()), _dp) if t is not None else None)
        return self._run(self.lib.mf3d_newsolv_mg_device, arr, dt, alfapr)

    def mgkcyc_device(self, su_list, pp_list):
        su = (_dp * len(su_list))(*[C.cast(C.c_void_p(t.data_ptr()), _dp) for t in su_list])
        pp = (_dp * len(pp_list))(*[C.cast(C.c_void_p(t.data_ptr()), _dp) for t in pp_list])
        abi.check(self.lib, self.lib.mf3d_mgkcyc_device(self.ctx, su, pp), "mf3d_mgkcyc_device")

    def profile(self, kind: int):
        """Start timing one kernel class (abi.MF3D_PROF_*; 0 = off)."""
        abi.check(self.lib, self.lib.mf3d_profile(self.ctx, kind), "mf3d_profile")

    def profile_read(self):
        """(total device ms, launches, algorithmic bytes) since profile()."""
        ms, n, by = C.c_double(), C.c_longlong(), C.c_double()
        abi.check(self.lib, self.lib.mf3d_profile_read(self.ctx, C.byref(ms), C.byref(n), C.byref(by)),
                  "mf3d_profile_read")
        return ms.value, n.value, by.value

    @property
    def launches(self) -> int:
        return int(self.lib.mf3d_last_launch_count(self.ctx))

    def set_inlet(self, block_id: int, code: int, values, uprof_sem: int = 0):
        """The inlet values of a west face of code 7 or 8 (mf3d_set_inlet):
        ``values`` as ``read_inlet_file`` returns them."""
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        abi.check(self.lib, self.lib.mf3d_set_inlet(self.ctx, int(block_id), int(code), int(uprof_sem),
                                                    v.ctypes.data_as(_dp), v.size), "mf3d_set_inlet")

    def bind_old_velocity(self, blocks=None):
        """uoo, voo, woo (device tensors, one dict per block) for the
        convective outflow of the solve's bounds (mf3d_bind_old_velocity);
        None unbinds.  The tensors stay borrowed until the next call."""
        if blocks is None:
            self._oo = None
            abi.check(self.lib, self.lib.mf3d_bind_old_velocity(self.ctx, None), "mf3d_bind_old_velocity")
            return
        arr = (abi.RkFields * len(blocks))()
        for b, f in enumerate(blocks):
            for k in ("uoo", "voo", "woo"):
                setattr(arr[b], k, C.cast(C.c_void_p(f[k].data_ptr()), _dp))
        self._oo = (arr, blocks)
        abi.check(self.lib, self.lib.mf3d_bind_old_velocity(self.ctx, arr), "mf3d_bind_old_velocity")

    def set_wall_model(self, re: float, fric: float = 0.0):
        """Re and fric of the wall functions (mf3d_set_wall_model)."""
        abi.check(self.lib, self.lib.mf3d_set_wall_model(self.ctx, float(re), float(fric)), "mf3d_set_wall_model")

    def bounds_device(self, blocks, dt=1.0, alfapr=1.0, alfabc=1):
        """boundu/v/w alone on device arrays (mf3d_bounds_device)."""
        abi.check(self.lib, self.lib.mf3d_bounds_device(self.ctx, _dev_fields(blocks), float(dt), float(alfapr),
                                                        int(alfabc)), "mf3d_bounds_device")

    def tuning(self, level: int) -> dict:
        """Launch shapes chosen for one level (mf3d_tuning)."""
        v = [C.c_int() for _ in range(4)]
        abi.check(self.lib, self.lib.mf3d_tuning(self.ctx, level, *[C.byref(x) for x in v]), "mf3d_tuning")
        return dict(zip(("sweep_schedule", "small_sweep", "restrict_planes", "cluster_ctas"), (x.value for x in v)))


def read_inlet_file(path: str, code: int) -> np.ndarray:
    """The numbers boundu/v/w read from an inlet file (bounds.for:55-103,
    397-438, 686-730): code 7 (Inlet/Inlet_<dom>_<n>.dat) one value per line,
    u's lines then v's then w's, returned in file order; code 8
    (inflow/Inlet_<dom>_<n>.dat) two header lines, then "up v w" per line,
    returned as an (lines, 3) array.  ``inlet_values`` turns them into what
    ``Projection.set_inlet`` takes."""
    with open(path) as f:
        lines = f.read().splitlines()
    conv = lambda x: float(x.replace("D", "E").replace("d", "e"))
    if code == 7:
        return np.array([conv(ln.split()[0]) for ln in lines if ln.strip()])
    if code == 8:
        return np.array([[conv(x) for x in ln.split()[:3]] for ln in lines[2:] if ln.strip()])
    raise ValueError("inlet files exist for the west codes 7 and 8")


def inlet_counts(desc, code: int):
    """Values of u, v, w a west inlet of code 7 or 8 reads for block ``desc``:
    each component over its own rows and planes (v one row short of a north
    wall, w one plane short of a top wall), code 7 with both ghost rows,
    code 8 with the low one only (bounds.for:84-86)."""
    out = []
    for c in range(3):
        je = desc.ny - (1 if c == 1 and desc.jnext < 0 and desc.bc_north != 5 else 0)
        ke = desc.nz - (1 if c == 2 and desc.knext < 0 and desc.bc_top != 5 else 0)
        out.append((je + 2) * (ke + 2) if code == 7 else (je + 1) * (ke + 1))
    return out


def inlet_values(desc, code: int, data, data_vw=None) -> np.ndarray:
    """The values of ``Projection.set_inlet`` from ``read_inlet_file``'s
    output: code 7 the file's numbers as they stand; code 8 the first column
    for u and the second and third for v and w (``data_vw``: the file boundv
    and boundw open, when it is another one)."""
    nu, nv, nw = inlet_counts(desc, code)
    if code == 7:
        return np.asarray(data, dtype=np.float64)[:nu + nv + nw]
    vw = data if data_vw is None else data_vw
    return np.concatenate([data[:nu, 0], vw[:nv, 1], vw[:nw, 2]])


def _dev_fields(blocks):
    arr = (abi.Fields * len(blocks))()
    for b, f in enumerate(blocks):
        for k in ("ustar", "vstar", "wstar", "u", "v", "w", "p", "su"):
            t = f.get(k)
            setattr(arr[b], k, C.cast(C.c_void_p(t.data_ptr()), _dp) if t is not None else None)
    return arr


class Batch:
    """Many independent single-block domains solved by one set of launches
    (``mf3d_batch_create`` / ``mf3d_batch_solve_device``).  Each domain runs
    its own V-cycles and stops on its own test; results equal solo solves."""

    def __init__(self, domains, params: abi.Params, lib=None):
        self.lib = lib or abi.load()
        self.n = len(domains)
        arr = (abi.DomainDesc * self.n)(*domains)
        self._arr = arr
        self.params = params
        ctx = C.c_void_p()
        abi.check(self.lib, self.lib.mf3d_batch_create(arr, self.n, C.byref(params), C.byref(ctx)),
                  "mf3d_batch_create")
        self.ctx = ctx

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.mf3d_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve_device(self, fields, dt=None, alfapr=None):
        """fields: one dict of CUDA float64 tensors per domain.  Returns a
        list of SolveResult and the batch's worst status."""
        dt = np.asarray(dt if dt is not None else np.ones(self.n), dtype=np.float64)
        al = np.asarray(alfapr if alfapr is not None else np.ones(self.n), dtype=np.float64)
        cap = max(self.params.maxcy, 1)
        hist = np.zeros((self.n, cap))
        infos = (abi.SolveInfo * self.n)()
        st = self.lib.mf3d_batch_solve_device(self.ctx, _dev_fields(fields), dt.ctypes.data_as(_dp),
                                              al.ctypes.data_as(_dp), infos, hist.ctypes.data_as(_dp), cap)
        abi.check(self.lib, st, "mf3d_batch_solve_device")
        out = [SolveResult(infos[d].status, infos[d].rmax, infos[d].rmax0, infos[d].iter, infos[d].ms_device,
                           hist[d, :infos[d].iter].copy()) for d in range(self.n)]
        return out, st

    @property
    def launches(self) -> int:
        return int(self.lib.mf3d_last_launch_count(self.ctx))


class Server:
    """The request loop (``mf3d_server_*``): submit single-block solves as
    they arrive; worker threads in the library (one per size lane) admit
    them by memory, keep their hierarchies resident and advance all resident
    requests by one outer iteration per cycle.  ``fields`` are device
    tensors (ttc layout) borrowed until the request finishes; their contents
    must be complete on the device at submit (synchronise the producing
    stream first)."""

    def __init__(self, params: abi.Params, mem_cap_bytes: float = 150e9, max_resident: int = 256, lib=None):
        self.lib = lib or abi.load()
        self.params = params
        ctx = C.c_void_p()
        abi.check(self.lib, self.lib.mf3d_server_create(C.byref(params), float(mem_cap_bytes), int(max_resident),
                                                        C.byref(ctx)), "mf3d_server_create")
        self.ctx = ctx
        self._keep = {}

    def submit(self, domain: abi.DomainDesc, fields: dict, dt: float = 1.0, alfapr: float = 1.0) -> int:
        arr = _dev_fields([fields])
        t = C.c_longlong()
        abi.check(self.lib, self.lib.mf3d_server_submit(self.ctx, C.byref(domain), arr, dt, alfapr, C.byref(t)),
                  "mf3d_server_submit")
        self._keep[t.value] = (domain, arr, fields)
        return t.value

    def poll(self, ticket: int, wait_ms: int = 0):
        """(status, RequestInfo) once finished, else (MF3D_PENDING, None)."""
        info = abi.RequestInfo()
        st = self.lib.mf3d_server_poll(self.ctx, ticket, C.byref(info), int(wait_ms))
        if st == abi.MF3D_PENDING:
            return st, None
        self._keep.pop(ticket, None)
        if st == abi.MF3D_E_INVALID and info.t_submit == 0.0:
            abi.check(self.lib, st, "mf3d_server_poll")
        return st, info

    def stats(self) -> dict:
        v = [C.c_longlong() for _ in range(4)] + [C.c_double(), C.c_longlong()]
        abi.check(self.lib, self.lib.mf3d_server_stats(self.ctx, *[C.byref(x) for x in v]), "mf3d_server_stats")
        keys = ("submitted", "completed", "resident", "queued", "resident_bytes", "cycles")
        return {k: x.value for k, x in zip(keys, v)}

    def clock(self) -> float:
        return self.lib.mf3d_server_clock()

    def profile(self) -> dict:
        v = [C.c_double() for _ in range(4)] + [C.c_longlong() for _ in range(2)]
        abi.check(self.lib, self.lib.mf3d_server_profile(self.ctx, *[C.byref(x) for x in v]), "mf3d_server_profile")
        keys = ("build_s", "rebuild_s", "cycle_s", "finish_s", "builds", "rebuilds")
        return {k: x.value for k, x in zip(keys, v)}

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.mf3d_server_destroy(self.ctx)
            self.ctx = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
