"""The allocation-free face list (dgpu_face_list_noalloc) through the C ABI.

It exists for callers that cannot allocate device memory (code inside another
framework's memory pool or a fixed arena): inputs and outputs are the
caller's device buffers, and the only working memory is a static device array
sized for DGPU_NOALLOC_MAX_ANNULI annuli.  Its output must equal the face list
of the context entry point (dgpu_face_list) bit for bit -- the tolerance all
face-list tests use -- on two calls in a row, since every call reuses the
same static array.  Collected last (file name) so a failure here stops a run
only after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

from disco2_b200 import configs, lib

pytestmark = pytest.mark.gpu

ERR_ARG = -1


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _call(L, sim, tiph, dphi, cap, out, nf):
    return L.dgpu_face_list_noalloc(sim._h, _ptr(tiph), _ptr(dphi), cap, _ptr(out["nri"]),
                                    _ptr(out["L"]), _ptr(out["R"]), _ptr(out["dphi"]),
                                    _ptr(out["dA"]), _ptr(out["cm"]), C.byref(nf), None)


@pytest.mark.parametrize("make,steps", [(configs.circumbinary, 3), (configs.gresho, 2)])
def test_noalloc_face_list_matches_context_entry_point_twice(make, steps):
    import torch

    L = lib.load()
    sim = lib.Sim(make())
    ctx = lib.Context(sim)
    ctx.init_state(0)
    ctx.step(steps)
    want = ctx.face_list(0)
    st = ctx.get_state(0)
    ctx.close()
    dev = torch.device("cuda", 0)
    tiph = torch.tensor(st["tiph"], dtype=torch.float64, device=dev)
    dphi = torch.tensor(st["dphi"], dtype=torch.float64, device=dev)
    nf_want = len(want["L"])
    cap = nf_want + 64
    out = {"nri": torch.empty(sim.num_annuli, dtype=torch.int32, device=dev),
           "L": torch.empty(cap, dtype=torch.int32, device=dev),
           "R": torch.empty(cap, dtype=torch.int32, device=dev),
           "dphi": torch.empty(cap, dtype=torch.float64, device=dev),
           "dA": torch.empty(cap, dtype=torch.float64, device=dev),
           "cm": torch.empty(cap, dtype=torch.float64, device=dev)}
    torch.cuda.synchronize()
    free_after = []
    for call in range(2):
        for k, v in out.items():
            v.fill_(-7 if v.dtype == torch.int32 else float("nan"))
        torch.cuda.synchronize()
        nf = C.c_int(-1)
        rc = _call(L, sim, tiph, dphi, cap, out, nf)
        assert rc == 0, (call, rc)
        # device memory in use does not grow from one call to the next
        free_after.append(torch.cuda.mem_get_info(0)[0])
        assert nf.value == nf_want
        got = {k: v.cpu().numpy() for k, v in out.items()}
        assert np.array_equal(got["nri"], want["nri"]), call
        for k in ("L", "R", "dphi", "dA", "cm"):
            assert np.array_equal(got[k][:nf_want], want[k]), (call, k)
    assert free_after[1] == free_after[0], free_after


def test_noalloc_rejects_sizes_beyond_its_limits():
    import torch

    L = lib.load()
    dev = torch.device("cuda", 0)
    # more annuli than the static scratch holds: refused before any device work
    big = lib.Sim(configs.gresho(num_r=4200))
    assert big.num_annuli > 4096
    t = torch.zeros(8, dtype=torch.float64, device=dev)
    i = torch.zeros(8, dtype=torch.int32, device=dev)
    nf = C.c_int(-1)
    rc = L.dgpu_face_list_noalloc(big._h, _ptr(t), _ptr(t), 8, _ptr(i), _ptr(i), _ptr(i), _ptr(t),
                                  _ptr(t), _ptr(t), C.byref(nf), None)
    assert rc == ERR_ARG
    # a face count above cap: refused, count reported, nothing written past cap
    sim = lib.Sim(configs.gresho(num_r=16))
    h = sim.initial_state()
    tiph = torch.tensor(h["tiph"], device=dev)
    dphi = torch.tensor(h["dphi"], device=dev)
    cap = 10
    out = {k: torch.full((cap + 8,), -7, dtype=torch.int32, device=dev) for k in ("L", "R")}
    out.update({k: torch.full((cap + 8,), 0.5, dtype=torch.float64, device=dev)
                for k in ("dphi", "dA", "cm")})
    out["nri"] = torch.empty(sim.num_annuli, dtype=torch.int32, device=dev)
    rc = _call(L, sim, tiph, dphi, cap, out, nf)
    assert rc == ERR_ARG and nf.value > cap
    assert torch.all(out["L"] == -7) and torch.all(out["dA"] == 0.5)
