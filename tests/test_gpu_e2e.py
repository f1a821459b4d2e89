"""The marshal paths a driver uses around the step, checked against the
reference's golden states bit for bit, and the non-finite status.

* pinned host buffers with the asynchronous download (the bench's end-to-end
  sequence): upload -> step -> download_async per step, copies overlapping the
  neighbouring steps, two steps queued before one join/sync;
* device tensors (torch) with the device-pointer marshal;
* NC_ERR_NONFINITE from nc_check_finite and nc_download_state for a state
  seeded with a NaN.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def core(pkg, golden):
    geo, _ = golden
    c = pkg.NicamCuda(geo, graph=True)
    yield c
    c.close()


def _pinned(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory()


def test_pipelined_pinned_marshal_equals_reference(core, golden):
    """two steps queued with their uploads and asynchronous downloads before
    any wait: the second upload must not overwrite the staging buffer before
    the first unpack, the second download must not overwrite the first copy"""
    import torch
    _, st = golden
    a0, a0p = _pinned(torch, st["state0"]), _pinned(torch, st["state0_pl"])
    a1, a1p = _pinned(torch, st["state1"]), _pinned(torch, st["state1_pl"])
    outs = [(torch.empty_like(a0).pin_memory(), torch.empty_like(a0p).pin_memory()) for _ in range(3)]
    # step 1 from state0 -> outs[0]; step 1 from state1 -> outs[1]; step 1 from state0 again -> outs[2]
    for (src, srcp), (dst, dstp) in zip(((a0, a0p), (a1, a1p), (a0, a0p)), outs):
        core.upload_ptr(src.data_ptr(), srcp.data_ptr())
        core.step(1)
        core.download_ptr_async(dst.data_ptr(), dstp.data_ptr())
    core.join_copies()
    core.sync()
    for (dst, dstp), want in zip(outs, ("state1", "state2", "state1")):
        assert np.array_equal(dst.numpy(), st[want]), f"regional state, expected {want}"
        assert np.array_equal(dstp.numpy(), st[want + "_pl"]), f"pole state, expected {want}"
    # the synchronous download of the same device state equals the last asynchronous one
    out, out_pl = core.download()
    assert np.array_equal(out, outs[2][0].numpy()) and np.array_equal(out_pl, outs[2][1].numpy())


def test_chained_pinned_marshal_two_steps(core, golden):
    """each step's output is the next step's input (alternating buffers)"""
    import torch
    _, st = golden
    bufs = [(_pinned(torch, st["state0"]), _pinned(torch, st["state0_pl"])),
            (_pinned(torch, np.zeros_like(st["state0"])), _pinned(torch, np.zeros_like(st["state0_pl"])))]
    for s in range(2):
        src, dst = bufs[s % 2], bufs[(s + 1) % 2]
        core.upload_ptr(src[0].data_ptr(), src[1].data_ptr())
        core.step(1)
        core.download_ptr_async(dst[0].data_ptr(), dst[1].data_ptr())
        core.join_copies()
        core.sync()
    out = bufs[0]
    assert np.array_equal(out[0].numpy(), st["state2"]) and np.array_equal(out[1].numpy(), st["state2_pl"])


def test_device_tensor_marshal(core, golden):
    import torch
    _, st = golden
    s0 = torch.from_numpy(st["state0"]).cuda()
    s0p = torch.from_numpy(st["state0_pl"]).cuda()
    core.upload_tensor(s0, s0p)
    del s0, s0p                     # ordered on torch's stream: freeing the inputs is safe
    core.step(2)
    out, out_pl = core.download_tensor()
    torch.cuda.current_stream().synchronize()
    assert np.array_equal(out.cpu().numpy(), st["state2"])
    assert np.array_equal(out_pl.cpu().numpy(), st["state2_pl"])
    with pytest.raises(ValueError):
        core.upload_tensor(out.float(), out_pl)


def test_nonfinite_state_is_reported(pkg, core, golden):
    _, st = golden
    bad = st["state0"].copy()
    bad[3, 4, 5, 7, 5] = np.nan                        # RHOGE of one interior cell
    core.upload(bad, st["state0_pl"])
    with pytest.raises(pkg.NonFiniteStateError, match="variable 5"):
        core.check_finite()
    buf = np.zeros_like(bad)
    buf_pl = np.zeros_like(st["state0_pl"])
    with pytest.raises(pkg.NonFiniteStateError):
        core.download(buf, buf_pl)
    assert np.isnan(buf[3, 4, 5, 7, 5])                # the arrays are filled all the same
    bad_pl = st["state0_pl"].copy()
    bad_pl[0, 5, 1, 6] = np.inf                         # the tracer at a pole point
    core.upload(st["state0"], bad_pl)
    with pytest.raises(pkg.NonFiniteStateError, match="variable 6"):
        core.check_finite()
    core.upload(st["state0"], st["state0_pl"])
    core.check_finite()                                 # a clean state passes
    core.step(1)
    core.check_finite()
    out, _ = core.download()
    assert np.array_equal(out, st["state1"])
