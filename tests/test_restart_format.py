"""Restart files (fio "ADVANCED") against files the reference wrote itself
(tests/golden/make_restart.py), on the CPU: the header bytes this package
writes, the payload layout the device swaps into, and the read semantics the
device follows (fio_read's dummy-level repair, COMM_var's pole-centre fill,
then the halo exchange) restated with numpy and the oracle's exchange."""
import gzip
import importlib
import os

import numpy as np
import pytest

from oracle import nicam_step as O

R = importlib.import_module("pynicam-dc_b200.restart")


@pytest.fixture(scope="module")
def rs(tmp_path_factory):
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "gl03_z10_restart.npz"))
    d = tmp_path_factory.mktemp("restart")
    files = {}
    for k in ("write", "read"):
        p = str(d / f"{k}.pe000000")
        with open(p, "wb") as f:
            f.write(gzip.decompress(z[f"{k}_file_gz"].tobytes()))
        files[k] = p
    return z, files


def test_headers_match_reference(rs, golden):
    z, files = rs
    meta, items = R.parse(files["write"])
    assert meta["header"] == "INITIAL/RESTART_data_of_prognostic_variables"
    assert [it["varname"] for it in items] == list(z["names"])
    with open(files["write"], "rb") as f:
        b = f.read()
    head = R.file_header(meta["header"], "", 0, 2, 0, int(z["glevel"]), int(z["rlevel"]), z["rgnid"])
    assert b.startswith(head + len(items).to_bytes(4, "big"))
    K = golden[1]["state1"].shape[2]
    for it, nm, lb, un in zip(items, z["names"], z["labels"], z["units"]):
        ih = R.item_header(str(nm), str(lb), str(un), str(z["layername"]), it["datasize"], R.F8, K, 1,
                           int(z["ctime"]), int(z["ctime"]))
        assert b[it["offset"] - len(ih):it["offset"]] == ih, nm


def test_payload_is_device_layout_big_endian(rs, golden):
    """each variable's data: the (l, k, j, i) array, big-endian float64"""
    z, files = rs
    _, st = golden
    _, items = R.parse(files["write"])
    with open(files["write"], "rb") as f:
        b = f.read()
    for v, it in enumerate(items):
        want = np.ascontiguousarray(st["state1"][..., v].transpose(3, 2, 1, 0)).astype(">f8").tobytes()
        assert b[it["offset"]:it["offset"] + it["datasize"]] == want, it["varname"]


def test_read_semantics_vs_reference(rs, golden):
    z, files = rs
    geo, st = golden
    g = O.Geo(geo)
    _, items = R.parse(files["read"])
    G, K, L = st["state1"].shape[0], st["state1"].shape[2], st["state1"].shape[3]
    var = np.zeros(st["state1"].shape)
    for v, it in enumerate(items):
        a = np.fromfile(files["read"], dtype=">f8", count=it["datasize"] // 8, offset=it["offset"])
        a = a.reshape(L, K, G, G).astype(np.float64)
        for kd, ks in ((K - 1, K - 2), (0, 1)):
            bad = ~np.isfinite(a[:, kd])
            a[:, kd][bad] = a[:, ks][bad]
        var[..., v] = a.transpose(3, 2, 1, 0)
    assert not np.all(np.isfinite(np.fromfile(files["read"], dtype=">f8", count=items[1]["datasize"] // 8,
                                              offset=items[1]["offset"])))
    var_pl = np.full(st["state1_pl"].shape, np.nan)
    for pg, pl, i, j, l in z["pole_src"]:
        var_pl[pg, :, pl, :] = var[i, j, :, l, :]
    O.comm(g, var, var_pl)
    assert np.array_equal(var, z["read_state"])
    assert np.array_equal(var_pl, z["read_state_pl"])


def test_pole_centre_sources(rs, golden):
    """backend.pole_centre_sources on the reference's copy lists with the rl01
    region table (region ids = local indices on one process; regions 2 and 21
    are the first whose north / south vertex is a pole, RGNMNG_rgn4pl,
    share/mod_adm.py:267-278): the rows the reference's COMM_var used"""
    from types import SimpleNamespace as NS
    B = importlib.import_module("pynicam-dc_b200.backend")
    z, _ = rs
    geo, _ = golden
    cl = np.asarray(geo["copy_p2r"])
    L = int(np.asarray(geo["lall"]))
    adm = NS(RGNMNG_lp2r=np.arange(L).reshape(L, 1), RGNMNG_rgn4pl=np.array([2, 21]), I_NPL=0, I_SPL=1)
    comm = NS(Copy_list_p2r=cl, Copy_info_p2r=np.array([cl.shape[1], 0, 0]), I_size=0, I_prc_to=2,
              I_gridi_from=0, I_gridj_from=1, I_l_from=2, I_gridi_to=3, I_gridj_to=4, I_l_to=5)
    got = B.pole_centre_sources(NS(adm=adm, comm=comm))
    assert np.array_equal(got, z["pole_src"])


class _FakeCore:
    """records what restart.read hands to the device (host logic only)"""

    def __init__(self, shape):
        self.shape = shape
        self.unpacked, self.finished = {}, None

    def restart_unpack(self, var, buf):
        self.unpacked[var] = np.array(buf, copy=True)

    def restart_finish(self, pole_src):
        self.finished = np.asarray(pole_src)


def test_read_host_logic(rs, golden):
    """restart.read without a device: each named variable's payload goes to its
    device index unchanged (big-endian bytes, swapped on the device), a missing
    tracer is zero only when allowed, and COMM_var gets the pole sources"""
    z, files = rs
    _, st = golden
    names = [str(n) for n in z["names"]]
    core = _FakeCore(st["state1"].shape)
    R.read(core, files["write"], names, z["pole_src"])
    _, items = R.parse(files["write"])
    for v, it in enumerate(items):
        raw = np.fromfile(files["write"], dtype=np.uint64, count=it["datasize"] // 8, offset=it["offset"])
        assert np.array_equal(core.unpacked[v], raw), names[v]
    assert np.array_equal(core.finished, z["pole_src"])
    with pytest.raises(KeyError):
        R.read(_FakeCore(st["state1"].shape), files["write"], names[:6] + ["rhogqx"], z["pole_src"])
    c2 = _FakeCore(st["state1"].shape)
    R.read(c2, files["write"], names[:6] + ["rhogqx"], z["pole_src"], allow_missingq=True)
    assert not np.any(c2.unpacked[6])
    with pytest.raises(KeyError):   # a missing prognostic is never zero-filled
        R.read(_FakeCore(st["state1"].shape), files["write"], ["rhogx"] + names[1:], z["pole_src"],
               allow_missingq=True)
    bad = list(st["state1"].shape)
    bad[2] += 1
    with pytest.raises(ValueError):   # payload size does not match the device grid
        R.read(_FakeCore(tuple(bad)), files["write"], names, z["pole_src"])


class _PackCore:
    """hands restart.write the payload the device's byte swap produces for a
    state: (l, k, j, i) big-endian"""

    def __init__(self, state):
        self.shape = state.shape
        self.state = state

    def restart_pack(self, var, buf):
        be = np.ascontiguousarray(self.state[..., var].transpose(3, 2, 1, 0)).astype(">f8")
        buf[:] = be.reshape(-1).view(np.uint64)


def test_writer_host_logic_matches_reference_file(rs, golden, tmp_path):
    """restart.write with the device payload emulated: the whole file equals the
    one the reference's restart_output wrote, byte for byte; and through
    CudaDyn.restart_output with the reference's own item list"""
    z, files = rs
    _, st = golden
    items = [(str(n), str(lb), str(u), v) for v, (n, lb, u) in enumerate(zip(z["names"], z["labels"], z["units"]))]
    out = str(tmp_path / "w.pe000000")
    R.write(_PackCore(st["state1"]), out, items, str(z["layername"]), z["rgnid"], int(z["glevel"]),
            int(z["rlevel"]), int(z["ctime"]))
    with open(out, "rb") as f, open(files["write"], "rb") as g:
        assert f.read() == g.read()
    from types import SimpleNamespace as NS
    B = importlib.import_module("pynicam-dc_b200.backend")
    d = object.__new__(B.CudaDyn)
    d.core, d._device_valid, d._host_stale, d._forced = _PackCore(st["state1"]), True, True, False
    L = len(z["rgnid"])
    prgv = NS(output_io_mode="ADVANCED", output_diagnostics=False, layername=str(z["layername"]),
              _restart_output_items=lambda rcnf: [(n, lb, u, None, v) for (n, lb, u, v) in items])
    msc = NS(prgv=prgv, rcnf=None, adm=NS(RGNMNG_lp2r=np.asarray(z["rgnid"]).reshape(L, 1), ADM_prc_me=0,
                                          ADM_lall=L, ADM_glevel=int(z["glevel"]), ADM_rlevel=int(z["rlevel"])))
    d.restart_output(msc, str(tmp_path / "d.pe"), ctime=int(z["ctime"]))
    with open(str(tmp_path / "d.pe000000"), "rb") as f, open(files["write"], "rb") as g:
        assert f.read() == g.read()


def test_restart_input_host_logic(rs, golden):
    """CudaDyn.restart_input: the reference's variable names (PRG_name, then
    'rhog' + TRC_name), the <basename>000000 file, the pole-centre sources from
    the copy lists; the device state is then the handle's and the host copy stale"""
    from types import SimpleNamespace as NS
    B = importlib.import_module("pynicam-dc_b200.backend")
    z, files = rs
    geo, st = golden
    d = object.__new__(B.CudaDyn)
    d.core, d._device_valid, d._host_stale, d._forced = _FakeCore(st["state1"].shape), False, False, False
    cl = np.asarray(geo["copy_p2r"])
    L = int(np.asarray(geo["lall"]))
    names = [str(n) for n in z["names"]]
    msc = NS(prgv=NS(input_io_mode="ADVANCED", input_diagnostics=False, allow_missingq=False,
                     restart_input_basename=files["read"][:-6]),
             rcnf=NS(PRG_name=names[:6], PRG_vmax0=6, TRC_name=["qv"], TRC_vmax=1),
             adm=NS(RGNMNG_lp2r=np.arange(L).reshape(L, 1), RGNMNG_rgn4pl=np.array([2, 21]), I_NPL=0, I_SPL=1),
             comm=NS(Copy_list_p2r=cl, Copy_info_p2r=np.array([cl.shape[1], 0, 0]), I_size=0, I_prc_to=2,
                     I_gridi_from=0, I_gridj_from=1, I_l_from=2, I_gridi_to=3, I_gridj_to=4, I_l_to=5))
    d.restart_input(msc)
    assert sorted(d.core.unpacked) == list(range(7))
    assert np.array_equal(d.core.finished, z["pole_src"])
    assert d._device_valid and d._host_stale
    msc.prgv.input_io_mode = "npz"
    with pytest.raises(NotImplementedError):
        d.restart_input(msc)
