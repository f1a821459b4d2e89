"""Restart files written and read by the device (nc_restart_pack /
nc_restart_unpack / nc_restart_finish through restart.py) against the files
and the state the reference's own restart writer and reader produced
(tests/golden/make_restart.py): byte-for-byte and bit-for-bit."""
import gzip

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rs(tmp_path_factory):
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "gl03_z10_restart.npz"))
    d = tmp_path_factory.mktemp("restart_gpu")
    files = {}
    for k in ("write", "read"):
        p = str(d / f"{k}.pe000000")
        with open(p, "wb") as f:
            f.write(gzip.decompress(z[f"{k}_file_gz"].tobytes()))
        files[k] = p
    return z, files, d


def test_device_write_matches_reference_bytes(pkg, golden, rs):
    geo, st = golden
    z, files, d = rs
    core = pkg.NicamCuda(geo)
    core.upload(st["state1"], st["state1_pl"])
    items = [(str(n), str(lb), str(u), v) for v, (n, lb, u) in enumerate(zip(z["names"], z["labels"], z["units"]))]
    out = str(d / "dev_write.pe000000")
    pkg.restart.write(core, out, items, str(z["layername"]), z["rgnid"], int(z["glevel"]), int(z["rlevel"]),
                      int(z["ctime"]))
    with open(out, "rb") as f, open(files["write"], "rb") as g:
        assert f.read() == g.read()


def test_device_read_matches_reference_state(pkg, golden, rs):
    """dummy-level repair, pole-centre fill and halo exchange as the
    reference's restart_input; the pole state before the read is NaN, so every
    pole value must come from the read"""
    geo, st = golden
    z, files, _ = rs
    core = pkg.NicamCuda(geo)
    core.upload(st["state0"], np.full(st["state0_pl"].shape, np.nan))
    pkg.restart.read(core, files["read"], [str(n) for n in z["names"]], z["pole_src"])
    got, got_pl = core.download()
    assert np.array_equal(got, z["read_state"])
    assert np.array_equal(got_pl, z["read_state_pl"])


def test_device_round_trip_then_step(pkg, golden, rs):
    """write the state after step 1, read it into a fresh handle, step: the
    reference's state after step 2"""
    geo, st = golden
    z, _, d = rs
    a = pkg.NicamCuda(geo)
    a.upload(st["state1"], st["state1_pl"])
    items = [(str(n), "", "", v) for v, n in enumerate(z["names"])]
    p = str(d / "rt.pe000000")
    pkg.restart.write(a, p, items, "L", z["rgnid"], int(z["glevel"]), int(z["rlevel"]))
    b = pkg.NicamCuda(geo)
    pkg.restart.read(b, p, [str(n) for n in z["names"]], z["pole_src"])
    s1, s1p = b.download()
    assert np.array_equal(s1, st["state1"]) and np.array_equal(s1p, st["state1_pl"])
    b.step(1)
    s2, s2p = b.download()
    assert np.array_equal(s2, st["state2"]) and np.array_equal(s2p, st["state2_pl"])


def test_missing_variable_is_an_error(pkg, golden, rs):
    geo, _ = golden
    z, files, _ = rs
    core = pkg.NicamCuda(geo)
    names = [str(n) for n in z["names"]]
    with pytest.raises(KeyError):
        pkg.restart.read(core, files["read"], names[:6] + ["rhogqx"], z["pole_src"])
    pkg.restart.read(core, files["read"], names[:6] + ["rhogqx"], z["pole_src"], allow_missingq=True)
    got, _ = core.download()
    assert not np.any(got[..., 6])


def test_restart_argument_checks(pkg, golden):
    """no state to write, a variable index outside the state, a payload of the
    wrong size: refused before any device work"""
    geo, st = golden
    core = pkg.NicamCuda(geo)
    n = int(np.prod(st["state0"].shape[:4]))
    with pytest.raises(pkg.NicamError):
        core.restart_pack(0, np.empty(n, np.uint64))
    with pytest.raises(pkg.NicamError):
        core.restart_unpack(99, np.zeros(n, np.uint64))
    with pytest.raises(ValueError):
        core.restart_unpack(0, np.zeros(n - 1, np.uint64))
