"""Rate control and Tier-2 on the GPU: on Tier-1 frames from the reference CPU encoder, the
device path (hull, slope histogram, size measurements and packets computed on the device)
must give the same codestream, passes and lambda as the host codec, which itself equals
the reference's allocateRate + buildCodestream (checked here too)."""
import numpy as np
import pytest

from libgail_b200 import codestream as CS
from libgail_b200 import plugin as P
from libgail_b200 import synth
from oracle.oracle import RefEncoder, Reference, _ref_bind, have_reference, ref_codestream

pytestmark = pytest.mark.skipif(not have_reference(), reason="reference CPU build (oracle/_ref) not present")

PROFILES = [(1998, 1080, 0), (2048, 858, 0), (3996, 2160, 1), (4096, 1716, 1)]


@pytest.fixture(scope="module")
def frames():
    ref = Reference()
    _ref_bind(ref.lib)
    out = {}
    for W, H, fk in PROFILES:
        enc = RefEncoder(ref, W, H, fk)
        out[(W, H, fk)] = enc.encode(synth.xyz12_to_rgb48(synth.xyz12_planes(W, H, seed=11 + W)))
        enc.close()
    return ref, out


@pytest.mark.gpu
@pytest.mark.parametrize("prof", PROFILES)
@pytest.mark.parametrize("mbps,comp", [(230.0, 200.0), (90.0, 200.0), (230.0, 60.0)])
def test_device_rate_and_build_equals_host(frames, prof, mbps, comp):
    ref, fr = frames
    W, H, fk = prof
    t1 = fr[prof]
    lay = P.LayoutHolder(W, H, fk)
    want = CS.rate_and_build(lay, t1, fps=24.0, max_mbps=mbps, comp_mbps=comp, tag="cuda13.0")
    got = CS.device_rate_and_build(lay, t1, fps=24.0, max_mbps=mbps, comp_mbps=comp, tag="cuda13.0")
    assert np.array_equal(got[1], want[1]), "passes differ"
    assert got[2] == want[2], "lambda differs"
    assert got[0] == want[0], "codestream differs"
    ok, msg = CS.check_dci(got[0])
    assert ok or comp < 200.0, msg
    if comp == 200.0:
        rcs, rpasses, rlam, _ = ref_codestream(ref, W, H, fk, t1, fps=24.0, mbps=mbps, tag=b"cuda13.0")
        assert got[0] == rcs and got[2] == rlam


@pytest.mark.gpu
@pytest.mark.parametrize("prof", [(1998, 1080, 0), (3996, 2160, 1)])
@pytest.mark.parametrize("fps", [48.0, 25.0])
def test_device_rate_other_frame_rates(frames, prof, fps):
    """At 48 and 25 frames/s (a smaller per-frame budget): the device path's codestream,
    passes and lambda equal the host codec's and the reference's."""
    ref, fr = frames
    W, H, fk = prof
    t1 = fr[prof]
    lay = P.LayoutHolder(W, H, fk)
    want = CS.rate_and_build(lay, t1, fps=fps, tag="cuda13.0")
    got = CS.device_rate_and_build(lay, t1, fps=fps, tag="cuda13.0")
    assert got[0] == want[0] and np.array_equal(got[1], want[1]) and got[2] == want[2]
    rcs, _, rlam, _ = ref_codestream(ref, W, H, fk, t1, fps=fps, tag=b"cuda13.0")
    assert got[0] == rcs and got[2] == rlam
    ok, msg = CS.check_dci(got[0], fps)
    assert ok, msg


@pytest.mark.gpu
def test_device_rate_control_flat_and_repeated(frames):
    """A nearly empty frame (flat picture: few passes) and the same frame twice in a row
    through the cached device rate control."""
    ref, _ = frames
    W, H, fk = 1998, 1080, 0
    planes = np.full((3, H, W), 2048, np.uint16)
    planes[:, :, : W // 2] += 3  # one edge
    flat = synth.xyz12_to_rgb48(planes)
    enc = RefEncoder(ref, W, H, fk)
    t1 = enc.encode(flat)
    enc.close()
    lay = P.LayoutHolder(W, H, fk)
    want = CS.rate_and_build(lay, t1)
    for _ in range(2):
        got = CS.device_rate_and_build(lay, t1)
        assert got[0] == want[0] and np.array_equal(got[1], want[1]) and got[2] == want[2]
