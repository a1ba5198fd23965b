"""Helpers that run and read the CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  It runs either the reference build (_ref/disco_ref, compiled
from the reference's own sources by oracle/Makefile) or the C restatement
(_build/disco_port, compiled from oracle/port/), both with the same command
line and the same dump formats (documented in ref_driver.c).
"""
from __future__ import annotations

import os
import subprocess
import tempfile
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(HERE, "_ref", "disco_ref")
PORT_BIN = os.path.join(HERE, "_build", "disco_port")
PORT_LIB = os.path.join(HERE, "_build", "libdisco_port.so")
# the restatement built with every libm result in the step moved by one ulp
# (the sensitivity of a case to last-ulp differences; tests only)
PORT_ULP_BIN = os.path.join(HERE, "_build", "disco_port_ulp")
# the reference's main loop stepping through the B200 library (binding/)
BINDING_BIN = os.path.join(HERE, "_ref", "disco_gpu_main")
GPU_LIB = os.path.join(os.path.dirname(HERE), "disco2_b200", "_lib", "libdisco_gpu.so")
# the reference tree where it is mounted (override with DISCO_REFSRC)
REFSRC = os.environ.get("DISCO_REFSRC", "/root/reference/src")


def build(ref: bool | None = None, port: bool = True) -> None:
    """Compile the oracle.  The reference build needs the reference sources,
    which exist only where they were mounted; the restatement builds anywhere."""
    if ref is None:
        ref = os.path.isdir(REFSRC)
    port = port and os.path.exists(os.path.join(HERE, "port", "disco_port.c"))
    targets = (["ref"] if ref else []) + (["port"] if port else [])
    if ref and os.path.exists(GPU_LIB):
        targets.append("binding")
    if targets:
        subprocess.run(["make", "-s", "-C", HERE, "-j8", *targets], check=True)


def have_ref() -> bool:
    return os.path.exists(REF_BIN)


def have_port() -> bool:
    return os.path.exists(PORT_BIN)


def _exe(impl: str) -> str:
    return {"ref": REF_BIN, "port": PORT_BIN, "port_ulp": PORT_ULP_BIN}[impl]


def build_port_ulp() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "port-ulp"], check=True)


@dataclass
class State:
    NR: int
    NZ: int
    NQ: int
    N: int
    t: float
    dt: float
    gm: np.ndarray          # [2, 6]: r phi M omega Mdot Macc
    N_p: np.ndarray         # [NR] int32
    r_faces: np.ndarray     # [NR+1]
    prim: np.ndarray        # [N, NQ]
    cons: np.ndarray        # [N, NQ]
    tiph: np.ndarray        # [N]
    dphi: np.ndarray        # [N]
    ext: dict = field(default_factory=dict)

    @property
    def cell_off(self) -> np.ndarray:
        return np.concatenate([[0], np.cumsum(self.N_p.astype(np.int64))])


def read_state(path: str) -> State:
    with open(path, "rb") as f:
        buf = f.read()
    assert buf[:8] == b"DSTATE1\0", path
    o = 8
    NR, NZ, NQ, N, ext = np.frombuffer(buf, np.int32, 5, o); o += 20
    t, dt = np.frombuffer(buf, np.float64, 2, o); o += 16
    gm = np.frombuffer(buf, np.float64, 12, o).reshape(2, 6).copy(); o += 96

    def take(dtype, n):
        nonlocal o
        a = np.frombuffer(buf, dtype, n, o).copy()
        o += a.nbytes
        return a

    N_p = take(np.int32, NR)
    r_faces = take(np.float64, NR + 1)
    prim = take(np.float64, N * NQ).reshape(N, NQ)
    cons = take(np.float64, N * NQ).reshape(N, NQ)
    tiph = take(np.float64, N)
    dphi = take(np.float64, N)
    st = State(int(NR), int(NZ), int(NQ), int(N), float(t), float(dt), gm, N_p, r_faces,
               prim, cons, tiph, dphi)
    if ext:
        st.ext["grad"] = take(np.float64, N * NQ).reshape(N, NQ)
        st.ext["gradp"] = take(np.float64, N * NQ).reshape(N, NQ)
        st.ext["wiph"] = take(np.float64, N)
        st.ext["RKcons"] = take(np.float64, N * NQ).reshape(N, NQ)
        st.ext["RKtiph"] = take(np.float64, N)
    return st


def write_state(path: str, st: State) -> None:
    """Write a state file in the driver's format (for --load)."""
    with open(path, "wb") as f:
        f.write(b"DSTATE1\0")
        f.write(np.array([st.NR, st.NZ, st.NQ, st.N, 0], np.int32).tobytes())
        f.write(np.array([st.t, st.dt], np.float64).tobytes())
        f.write(np.asarray(st.gm, np.float64).reshape(12).tobytes())
        f.write(np.asarray(st.N_p, np.int32).tobytes())
        f.write(np.asarray(st.r_faces, np.float64).tobytes())
        f.write(np.ascontiguousarray(st.prim, np.float64).tobytes())
        f.write(np.ascontiguousarray(st.cons, np.float64).tobytes())
        f.write(np.ascontiguousarray(st.tiph, np.float64).tobytes())
        f.write(np.ascontiguousarray(st.dphi, np.float64).tobytes())


@dataclass
class Faces:
    nri: np.ndarray
    L: np.ndarray
    R: np.ndarray
    r: np.ndarray
    dphi: np.ndarray
    dA: np.ndarray
    deltaL: np.ndarray
    deltaR: np.ndarray
    cm: np.ndarray


def read_faces(path: str) -> Faces:
    with open(path, "rb") as f:
        buf = f.read()
    assert buf[:8] == b"DFACES1\0", path
    o = 8
    NR, Nf = np.frombuffer(buf, np.int32, 2, o); o += 8
    nri = np.frombuffer(buf, np.int32, NR, o).copy(); o += 4 * NR
    L = np.frombuffer(buf, np.int32, Nf, o).copy(); o += 4 * Nf
    R = np.frombuffer(buf, np.int32, Nf, o).copy(); o += 4 * Nf
    arrs = []
    for _ in range(6):
        arrs.append(np.frombuffer(buf, np.float64, Nf, o).copy())
        o += 8 * Nf
    return Faces(nri, L, R, *arrs)


def read_ckpt(path: str) -> dict:
    """A checkpoint buffer dump (ref_driver.c, dump_ckpt): t, gravmass [2][4]
    and data [nrows][ncols] as io_setbuf fills them."""
    with open(path, "rb") as f:
        b = f.read()
    assert b[:8] == b"DCKPT1\0\0", path
    nrows, ncols = np.frombuffer(b, "<i4", 2, 8)
    t = float(np.frombuffer(b, "<f8", 1, 16)[0])
    gm = np.frombuffer(b, "<f8", 8, 24).reshape(2, 4).copy()
    data = np.frombuffer(b, "<f8", int(nrows) * int(ncols), 88).reshape(int(nrows), int(ncols)).copy()
    return {"t": t, "gravmass": gm, "data": data}


def write_ckpt(path: str, ck: dict) -> None:
    """The inverse of read_ckpt (the driver's --restart input)."""
    data = np.ascontiguousarray(ck["data"], "<f8")
    with open(path, "wb") as f:
        f.write(b"DCKPT1\0\0")
        f.write(np.array(data.shape, "<i4").tobytes())
        f.write(np.array([ck["t"]], "<f8").tobytes())
        f.write(np.ascontiguousarray(ck["gravmass"], "<f8").tobytes())
        f.write(data.tobytes())


def checkpoint(parfile: str, nsteps: int, *, load: State | None = None, restart: dict | None = None) -> dict:
    """Reference build: run `nsteps` RK2 steps and return the checkpoint
    buffer that io_setbuf fills (src/IO/io_buffer.c:26-58)."""
    exe = _exe("ref")
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "ck.bin")
        cmd = [exe, "checkpoint", parfile, str(nsteps), out]
        if load is not None:
            lp = os.path.join(td, "in.bin")
            write_state(lp, load)
            cmd += ["--load", lp]
        if restart is not None:
            rp = os.path.join(td, "restart.bin")
            write_ckpt(rp, restart)
            cmd += ["--restart", rp]
        subprocess.run(cmd, check=True, stderr=subprocess.PIPE)
        return read_ckpt(out)


def run(parfile: str, nsteps: int, *, impl: str = "ref", load: State | None = None,
        faces: bool = False, dtlog: bool = False, workdir: str | None = None, zfaces: bool = False,
        restart: dict | None = None):
    """Run `nsteps` RK2 steps; returns (final State, Faces|None, dt log array|None).
    zfaces (reference build, 3-D disks): the Faces are the z faces.  restart
    (reference build): a checkpoint (t, gravmass, data) to start from instead
    of the initial data, through the reference's restart branch."""
    exe = _exe(impl)
    if not os.path.exists(exe):
        raise FileNotFoundError(f"oracle binary missing: {exe} (run oracle.build())")
    with tempfile.TemporaryDirectory(dir=workdir) as td:
        out = os.path.join(td, "out.bin")
        cmd = [exe, "run", parfile, str(nsteps), out]
        if load is not None:
            lp = os.path.join(td, "in.bin")
            write_state(lp, load)
            cmd += ["--load", lp]
        if restart is not None:
            rp = os.path.join(td, "restart.bin")
            write_ckpt(rp, restart)
            cmd += ["--restart", rp]
        fp = os.path.join(td, "faces.bin")
        if faces:
            cmd += ["--zfaces" if zfaces else "--faces", fp]
        lg = os.path.join(td, "dt.log")
        if dtlog:
            cmd += ["--dtlog", lg]
        subprocess.run(cmd, check=True, stderr=subprocess.PIPE)
        st = read_state(out)
        fc = read_faces(fp) if faces else None
        log = np.loadtxt(lg, ndmin=2) if dtlog else None
    return st, fc, log


def stage(parfile: str, phase: int, *, impl: str = "ref", load: State | None = None) -> State:
    """Run the prologue of one RK2 step and the first substep up to `phase`
    (0-7), or all of the first substep and the second up to `phase` - 8
    (8-15)."""
    exe = _exe(impl)
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "out.bin")
        cmd = [exe, "stage", parfile, str(phase), out]
        if load is not None:
            lp = os.path.join(td, "in.bin")
            write_state(lp, load)
            cmd += ["--load", lp]
        subprocess.run(cmd, check=True, stderr=subprocess.PIPE)
        return read_state(out)
