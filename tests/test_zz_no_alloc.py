"""nc_mass_sum_noalloc: the mass sum for callers that may not allocate device
memory (a framework's caching allocator or custom-call context).  It takes the
caller's device arrays and keeps its partial sums in a fixed device array of
the library instead of allocating; it adds the same terms in the same order as
nc_mass_sums, so its result must equal that of a handle holding the same state
bit for bit, on consecutive calls.

Kept in a file of its own that pytest collects last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float64)).cuda()


def test_noalloc_mass_sum_matches_handle(pkg, golden):
    import torch
    geo, st = golden
    lib = pkg.load_library()
    core = pkg.NicamCuda(geo, graph=False)
    try:
        core.upload(st["state2"], st["state2_pl"])
        want = core.mass_sums()
    finally:
        core.close()
    G, K, L = int(geo["gall_1d"]), int(geo["kall"]), int(geo["lall"])
    kmin, kmax = int(geo["kmin"]), int(geo["kmax"])
    reg = lambda a: _dev(torch, np.transpose(a, (3, 2, 1, 0)))      # (i,j,k,l) -> device (l,k,j,i)
    s, sp = st["state2"], st["state2_pl"]
    rhog, rhogq = reg(s[..., 0]), reg(s[..., 6])
    gs, vol = reg(geo["VMTR_GSGAM2"]), reg(geo["VMTR_VOLUME"])
    rhog_pl, rhogq_pl = _dev(torch, sp[..., 0]), _dev(torch, sp[..., 6])
    gs_pl, vol_pl = _dev(torch, geo["VMTR_GSGAM2_pl"]), _dev(torch, geo["VMTR_VOLUME_pl"])
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    p = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None

    def call(num, num_pl):
        rc = lib.nc_mass_sum_noalloc(p(rhog), p(num), p(gs), p(vol), p(rhog_pl), p(num_pl), p(gs_pl), p(vol_pl),
                                     G, L, K, kmin, kmax, p(out), ctypes.c_void_p(stream))
        assert rc == 0, lib.nc_last_error().decode()
        torch.cuda.synchronize()
        return float(out.item())

    for _ in range(2):                       # two calls in a row of each kind
        air = call(None, None)
        trc = call(rhogq, rhogq_pl)
        assert air == want[0]
        assert trc == want[1]


def test_noalloc_mass_sum_rejects_oversize_grid(pkg):
    import torch
    lib = pkg.load_library()
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(x.data_ptr())
    rc = lib.nc_mass_sum_noalloc(p, None, p, p, p, None, p, p, 1026, 1000, 42, 1, 40, p, None)
    assert rc != 0
    assert "scratch limit" in lib.nc_last_error().decode()
    rc = lib.nc_mass_sum_noalloc(p, None, p, p, p, None, p, p, 34, 40, 200, 1, 40, p, None)
    assert rc != 0                           # kall beyond the library's 128 levels
    assert "bad sizes" in lib.nc_last_error().decode()
