"""ctypes binding of libdisco_gpu.so (the C ABI in include/disco_gpu.h).

Python is a thin caller here: every numerical step runs in the library's CUDA
kernels.  Loading fails loudly when the shared library has not been built.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import configs

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libdisco_gpu.so")

OK = 0
ERR_NAMES = {-1: "ARG", -2: "PARFILE", -3: "UNSUPPORTED", -4: "CUDA", -5: "FACE_OVERFLOW",
             -6: "NUMERIC", -7: "NOMEM", -8: "IO"}

# Every symbol the header declares, with its ctypes signature.
_P, _I, _D = C.c_void_p, C.c_int, C.c_double
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
SIGNATURES = {
    "dgpu_sim_from_parfile": (_I, [C.c_char_p, C.POINTER(_P)]),
    "dgpu_sim_from_text": (_I, [C.c_char_p, C.POINTER(_P)]),
    "dgpu_sim_destroy": (None, [_P]),
    "dgpu_sim_num_annuli": (_I, [_P]),
    "dgpu_sim_num_cells": (_I, [_P]),
    "dgpu_sim_grid": (_I, [_P, _ip, _dp]),
    "dgpu_sim_param": (_I, [_P, C.c_char_p, _dp]),
    "dgpu_sim_initial_state": (_I, [_P, _dp, _dp, _dp, _dp]),
    "dgpu_create": (_I, [C.POINTER(_P), _I, _I, _P, C.POINTER(_P)]),
    "dgpu_destroy": (None, [_P]),
    "dgpu_last_error": (C.c_char_p, [_P]),
    "dgpu_num_instances": (_I, [_P]),
    "dgpu_init_state": (_I, [_P, _I]),
    "dgpu_set_state": (_I, [_P, _I, _dp, _dp, _dp]),
    "dgpu_get_state": (_I, [_P, _I, _dp, _dp, _dp, _dp]),
    "dgpu_set_gravmass": (_I, [_P, _I, _dp]),
    "dgpu_get_gravmass": (_I, [_P, _I, _dp]),
    "dgpu_get_time": (_I, [_P, _I, _dp, _dp]),
    "dgpu_set_time": (_I, [_P, _I, _D]),
    "dgpu_step_rk2": (_I, [_P, _I]),
    "dgpu_synchronize": (_I, [_P]),
    "dgpu_step_rk2_timed": (_I, [_P, _I, _dp]),
    "dgpu_set_fused": (_I, [_P, _I]),
    "dgpu_fused": (_I, [_P]),
    "dgpu_stage": (_I, [_P, _I]),
    "dgpu_get_stage_data": (_I, [_P, _I, _dp, _dp, _dp, _dp, _dp]),
    "dgpu_face_list": (_I, [_P, _I, _I, _ip, _ip, _ip, _dp, _dp, _dp, _dp, _dp, _dp, _ip]),
    "dgpu_face_list_z": (_I, [_P, _I, _I, _ip, _ip, _ip, _dp, _dp, _dp, _dp, _dp, _dp, _ip]),
    "dgpu_torque": (_I, [_P, _I, _dp]),
    "dgpu_face_list_noalloc": (_I, [_P, _P, _P, _I, _P, _P, _P, _P, _P, _P, _ip, _P]),
    "dgpu_autotune": (_I, [_P, _I, _ip]),
    "dgpu_diagnostics": (_I, [_P, _I, _dp, _dp, _dp, _dp]),
    "dgpu_objective": (_I, [_P, _I, _I, _dp, _dp, _dp]),
    "dgpu_tangent": (_I, [_P, _I, _I, _D, _D, _dp, _dp, _dp]),
    "dgpu_adjoint": (_I, [_P, _I, _I, _I, _dp, _dp, _dp, _dp, _dp]),
    "dgpu_hdf5_out": (_I, [C.c_char_p, _D, _dp, _dp, C.c_longlong, _I]),
    "dgpu_hdf5_dims": (_I, [C.c_char_p, C.POINTER(C.c_longlong), _ip]),
    "dgpu_hdf5_dataset": (_I, [C.c_char_p, C.c_char_p, _ip, C.POINTER(C.c_longlong), _dp]),
    "dgpu_hdf5_in": (_I, [C.c_char_p, C.c_longlong, C.c_longlong, _I, _dp, _dp, _dp]),
    "dgpu_sim_restart_state": (_I, [_P, C.c_char_p, _dp, _dp, _dp, _dp, _dp]),
    "dgpu_checkpoint_out": (_I, [_P, _I, C.c_char_p]),
    "dgpu_checkpoint_in": (_I, [_P, _I, C.c_char_p]),
}

_lib = None


class DiscoError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load the library (once).  Raises if it is missing: there is no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m disco2_b200.build`")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _dptr(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _iptr(a):
    return None if a is None else a.ctypes.data_as(_ip)


class Sim:
    """Host-side Sim built from a parfile (text, path or parameter dict)."""

    def __init__(self, par):
        lib = load()
        h = _P()
        if isinstance(par, dict):
            rc = lib.dgpu_sim_from_text(configs.parfile_text(par).encode(), C.byref(h))
        elif isinstance(par, str) and "\n" in par:
            rc = lib.dgpu_sim_from_text(par.encode(), C.byref(h))
        else:
            rc = lib.dgpu_sim_from_parfile(os.fsencode(par), C.byref(h))
        if rc != OK:
            raise DiscoError(rc, lib.dgpu_last_error(None).decode())
        self._h = h
        self.num_annuli = lib.dgpu_sim_num_annuli(h)
        self.num_cells = lib.dgpu_sim_num_cells(h)
        # NUM_Q: the five hydro variables and the passive scalars (NUM_N)
        self.num_q = 5 + int(self.param("NUM_N"))

    def grid(self):
        N_p = np.zeros(self.num_annuli, np.int32)
        rf = np.zeros(self.num_annuli + 1, np.float64)
        load().dgpu_sim_grid(self._h, _iptr(N_p), _dptr(rf))
        return N_p, rf

    def param(self, key: str) -> float:
        v = C.c_double()
        rc = load().dgpu_sim_param(self._h, key.encode(), C.byref(v))
        if rc != OK:
            raise KeyError(key)
        return v.value

    def initial_state(self) -> dict:
        """Host-computed initial state (what Context.init_state uploads)."""
        n = self.num_cells
        out = {"prim": np.zeros((n, self.num_q)), "tiph": np.zeros(n), "dphi": np.zeros(n),
               "gm": np.zeros((2, 6))}
        rc = load().dgpu_sim_initial_state(self._h, _dptr(out["prim"]), _dptr(out["tiph"]),
                                          _dptr(out["dphi"]), _dptr(out["gm"]))
        if rc != OK:
            raise DiscoError(rc, load().dgpu_last_error(None).decode())
        return out

    def restart_state(self, path) -> dict:
        """Host-computed restart state from a checkpoint file (what
        Context.checkpoint_in uploads): prim, tiph, dphi, gm and t."""
        n = self.num_cells
        out = {"prim": np.zeros((n, self.num_q)), "tiph": np.zeros(n), "dphi": np.zeros(n),
               "gm": np.zeros((2, 6))}
        t = C.c_double(0.0)
        rc = load().dgpu_sim_restart_state(self._h, os.fsencode(path), _dptr(out["prim"]), _dptr(out["tiph"]),
                                          _dptr(out["dphi"]), _dptr(out["gm"]), C.byref(t))
        if rc != OK:
            raise DiscoError(rc, load().dgpu_last_error(None).decode())
        out["t"] = t.value
        return out

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.dgpu_sim_destroy(self._h)
            self._h = None


class Context:
    """Device state of one or more independent disks."""

    def __init__(self, sims, device: int = 0, stream: int | None = None):
        lib = load()
        if isinstance(sims, Sim):
            sims = [sims]
        self.sims = list(sims)
        arr = (_P * len(self.sims))(*[s._h for s in self.sims])
        h = _P()
        rc = lib.dgpu_create(arr, len(self.sims), device, _P(stream) if stream else None, C.byref(h))
        if rc != OK:
            raise DiscoError(rc, lib.dgpu_last_error(None).decode())
        self._h = h

    def _ck(self, rc):
        if rc != OK:
            raise DiscoError(rc, load().dgpu_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            load().dgpu_destroy(self._h)
            self._h = None

    def __del__(self):
        if _lib is not None:
            self.close()

    def init_state(self, inst: int = 0):
        self._ck(load().dgpu_init_state(self._h, inst))

    def set_state(self, inst, prim, tiph, dphi):
        prim = np.ascontiguousarray(prim, np.float64)
        tiph = np.ascontiguousarray(tiph, np.float64)
        dphi = np.ascontiguousarray(dphi, np.float64)
        n = self.sims[inst].num_cells
        assert prim.shape == (n, self.sims[inst].num_q) and tiph.shape == (n,) and dphi.shape == (n,)
        self._ck(load().dgpu_set_state(self._h, inst, _dptr(prim), _dptr(tiph), _dptr(dphi)))
        self._ck(load().dgpu_synchronize(self._h))

    def checkpoint_out(self, path, inst: int = 0) -> None:
        """Write disk inst as a checkpoint file in the reference's layout."""
        self._ck(load().dgpu_checkpoint_out(self._h, inst, os.fsencode(path)))

    def checkpoint_in(self, path, inst: int = 0) -> None:
        """Restart disk inst from a checkpoint file (the reference's restart set-up)."""
        self._ck(load().dgpu_checkpoint_in(self._h, inst, os.fsencode(path)))

    def get_state(self, inst: int = 0) -> dict:
        n, nq = self.sims[inst].num_cells, self.sims[inst].num_q
        prim = np.zeros((n, nq))
        cons = np.zeros((n, nq))
        tiph = np.zeros(n)
        dphi = np.zeros(n)
        self._ck(load().dgpu_get_state(self._h, inst, _dptr(prim), _dptr(cons), _dptr(tiph), _dptr(dphi)))
        return {"prim": prim, "cons": cons, "tiph": tiph, "dphi": dphi}

    def stage_data(self, inst: int = 0) -> dict:
        n, nq = self.sims[inst].num_cells, self.sims[inst].num_q
        out = {"grad": np.zeros((n, nq)), "gradp": np.zeros((n, nq)), "wiph": np.zeros(n),
               "RKcons": np.zeros((n, nq)), "RKtiph": np.zeros(n)}
        self._ck(load().dgpu_get_stage_data(self._h, inst, _dptr(out["grad"]), _dptr(out["gradp"]),
                                            _dptr(out["wiph"]), _dptr(out["RKcons"]),
                                            _dptr(out["RKtiph"])))
        return out

    def set_gravmass(self, inst, gm):
        gm = np.ascontiguousarray(gm, np.float64).reshape(12)
        self._ck(load().dgpu_set_gravmass(self._h, inst, _dptr(gm)))

    def gravmass(self, inst: int = 0) -> np.ndarray:
        gm = np.zeros(12)
        self._ck(load().dgpu_get_gravmass(self._h, inst, _dptr(gm)))
        return gm.reshape(2, 6)

    def time(self, inst: int = 0):
        t, dt = C.c_double(), C.c_double()
        self._ck(load().dgpu_get_time(self._h, inst, C.byref(t), C.byref(dt)))
        return t.value, dt.value

    def set_time(self, inst, t):
        self._ck(load().dgpu_set_time(self._h, inst, float(t)))

    def step(self, nsteps: int = 1, sync: bool = True):
        self._ck(load().dgpu_step_rk2(self._h, nsteps))
        if sync:
            self.synchronize()

    KERNELS = ("cellprep", "merge", "rslope", "plm_r", "source", "flux_phi", "flux_r", "update")
    FUSED_KERNELS = ("prep", "sweep")

    @property
    def fused(self) -> bool:
        """True when a substep is the two fused kernels (k_prep, k_sweep)."""
        return bool(load().dgpu_fused(self._h))

    def set_fused(self, on: bool):
        self._ck(load().dgpu_set_fused(self._h, 1 if on else 0))

    @property
    def kernels(self) -> tuple:
        return self.FUSED_KERNELS if self.fused else self.KERNELS

    def step_timed(self, nsteps: int = 1) -> dict:
        """Device milliseconds per launch of each kernel of the step, summed
        over nsteps: {kernel: (substep 1, substep 2)}."""
        ms = np.zeros(16)
        self._ck(load().dgpu_step_rk2_timed(self._h, nsteps, _dptr(ms)))
        return {k: (ms[i], ms[8 + i]) for i, k in enumerate(self.kernels)}

    @property
    def handle(self):
        return self._h

    def synchronize(self):
        self._ck(load().dgpu_synchronize(self._h))

    def stage(self, phase: int):
        self._ck(load().dgpu_stage(self._h, phase))

    def face_list(self, inst: int = 0, z: bool = False) -> dict:
        """The r-face list (z: the z-face list of a 3-D disk) in the
        reference's order; "nri" holds the pair offsets."""
        lib = load()
        s = self.sims[inst]
        fn = lib.dgpu_face_list_z if z else lib.dgpu_face_list
        nf = C.c_int()
        fn(self._h, inst, 0, None, None, None, None, None, None, None, None, None, C.byref(nf))
        n = nf.value
        npairs = int(s.param("NZ" if z else "NR"))
        out = {"nri": np.zeros(npairs, np.int32), "L": np.zeros(n, np.int32),
               "R": np.zeros(n, np.int32)}
        for k in ("r", "dphi", "dA", "deltaL", "deltaR", "cm"):
            out[k] = np.zeros(n)
        self._ck(fn(self._h, inst, n, _iptr(out["nri"]), _iptr(out["L"]),
                    _iptr(out["R"]), _dptr(out["r"]), _dptr(out["dphi"]),
                    _dptr(out["dA"]), _dptr(out["deltaL"]), _dptr(out["deltaR"]),
                    _dptr(out["cm"]), C.byref(nf)))
        return out

    def torque(self, inst: int = 0) -> float:
        v = C.c_double()
        self._ck(load().dgpu_torque(self._h, inst, C.byref(v)))
        return v.value

    def diagnostics(self, inst: int = 0) -> dict:
        """diagnostics_set's reductions of the current state (before dtout)."""
        s = self.sims[inst]
        nr = int(s.param("NumR"))
        N_p, _ = s.grid()
        ncell = int(sum(N_p[1:1 + nr]))  # one inner ghost annulus (sim_alloc_arr, single rank)
        out = {"vector": np.zeros((nr, 17)), "scalar": np.zeros(16), "equat": np.zeros((ncell, 18)),
               "extra": np.zeros(14)}
        self._ck(load().dgpu_diagnostics(self._h, inst, _dptr(out["vector"]), _dptr(out["scalar"]),
                                         _dptr(out["equat"]), _dptr(out["extra"])))
        return out

    TUNED = ("plm_r", "flux_phi", "flux_r", "source", "update", "sweep")

    def autotune(self, steps: int = 3, choice=None) -> dict:
        """Time each launch shape of the heavy kernels on this context's disks
        and keep the fastest (steps == 0: apply `choice`); returns the blocks
        per SM chosen for each tuned kernel."""
        ch = (C.c_int * 6)(*(list(choice) + [0] * (6 - len(choice)) if choice is not None else [0] * 6))
        self._ck(load().dgpu_autotune(self._h, steps, ch))
        return dict(zip(self.TUNED, list(ch)))

    # ---- differentiation (one disk per context) ----
    def objective(self, nsteps: int, window_start: int, dt=None, return_dt: bool = False):
        """J = (mean torque, mean accretion rate) over steps window_start+1..nsteps;
        dt (nsteps values) freezes the dt schedule instead of the CFL dt."""
        J = np.zeros(2)
        dt_out = np.zeros(nsteps)
        dt_in = None
        if dt is not None:
            dt = np.ascontiguousarray(dt, dtype=np.float64)
            assert dt.shape == (nsteps,)
            dt_in = _dptr(dt)
        self._ck(load().dgpu_objective(self._h, nsteps, window_start, dt_in, _dptr(dt_out), _dptr(J)))
        return (J, dt_out) if return_dt else J

    def tangent(self, nsteps: int, window_start: int, dq: float = 0.0, dalpha: float = 0.0,
                dprim: np.ndarray | None = None) -> tuple[np.ndarray, np.ndarray]:
        """(J, dJ/de) along dq/de, dalpha/de and d prim_0/de ([N][5] or None)."""
        J, dJ = np.zeros(2), np.zeros(2)
        dp = None
        if dprim is not None:
            dprim = np.ascontiguousarray(dprim, dtype=np.float64)
            dp = _dptr(dprim)
        self._ck(load().dgpu_tangent(self._h, nsteps, window_start, float(dq), float(dalpha), dp,
                                     _dptr(J), _dptr(dJ)))
        return J, dJ

    def adjoint(self, nsteps: int, window_start: int, ckpt_every: int = 25,
                weights=(1.0, 0.0)) -> dict:
        """Gradient of weights . J with respect to q, alpha and the initial prims."""
        w = np.asarray(weights, dtype=np.float64)
        J = np.zeros(2)
        dq, da = C.c_double(), C.c_double()
        n = self.sims[0].num_cells
        dprim = np.zeros((n, 5))
        self._ck(load().dgpu_adjoint(self._h, nsteps, window_start, ckpt_every, _dptr(w), _dptr(J),
                                     C.byref(dq), C.byref(da), _dptr(dprim)))
        return {"J": J, "dq": dq.value, "dalpha": da.value, "dprim": dprim}


def hdf5_out(path, t: float, gravmass, data) -> None:
    """Write a checkpoint file: T = t, GravMass [2][4], Data [rows][cols]."""
    gravmass = np.ascontiguousarray(gravmass, np.float64)
    data = np.ascontiguousarray(data, np.float64)
    assert gravmass.shape == (2, 4) and data.ndim == 2
    rc = load().dgpu_hdf5_out(os.fsencode(path), float(t), _dptr(gravmass), _dptr(data), data.shape[0], data.shape[1])
    if rc != OK:
        raise DiscoError(rc, load().dgpu_last_error(None).decode())


def hdf5_in(path, row0: int = 0, nrows: int | None = None) -> dict:
    """Read a checkpoint file: t, gravmass [2][4] and rows of Data."""
    lib = load()
    rows, cols = C.c_longlong(0), C.c_int(0)
    rc = lib.dgpu_hdf5_dims(os.fsencode(path), C.byref(rows), C.byref(cols))
    if rc != OK:
        raise DiscoError(rc, lib.dgpu_last_error(None).decode())
    if nrows is None:
        nrows = rows.value - row0
    data = np.zeros((max(nrows, 0), cols.value))
    gm = np.zeros((2, 4))
    t = C.c_double(0.0)
    rc = lib.dgpu_hdf5_in(os.fsencode(path), row0, nrows, cols.value, C.byref(t), _dptr(gm), _dptr(data))
    if rc != OK:
        raise DiscoError(rc, lib.dgpu_last_error(None).decode())
    return {"t": t.value, "gravmass": gm, "data": data}


def hdf5_dataset(path, name: str) -> np.ndarray:
    """One 64-bit float dataset of an HDF5 file's root group."""
    lib = load()
    rank = C.c_int(0)
    dims = (C.c_longlong * 2)()
    rc = lib.dgpu_hdf5_dataset(os.fsencode(path), name.encode(), C.byref(rank), dims, None)
    if rc != OK:
        raise DiscoError(rc, lib.dgpu_last_error(None).decode())
    out = np.zeros(tuple(int(d) for d in dims[:rank.value]))
    rc = lib.dgpu_hdf5_dataset(os.fsencode(path), name.encode(), C.byref(rank), dims, _dptr(out))
    if rc != OK:
        raise DiscoError(rc, lib.dgpu_last_error(None).decode())
    return out
