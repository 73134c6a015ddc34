"""The split pyramid's level-0 blend divides each frame's weight by the
weight sum through Markstein's refinement from the sum's correctly rounded
reciprocal (formed once per pixel for all frames).  It must be the IEEE
division bit for bit, as the reference divides (src/fuse/pyramid.zig:303-316):
checked through the library's own division routine on 2^26 pairs of the
normalisation's ranges (weights as float bit patterns in [2^-20, 2) and
zeros, weight sums in [1e-12, 512], divisors with all-ones and zero
significands among them) against torch's float32 division on the device."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from __graft_entry__ import load_package  # noqa: E402

fsb = load_package()
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    if not t.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return t


def test_blend_division_is_the_ieee_division(torch):
    dev = "cuda:0"
    g = torch.Generator(device=dev)
    g.manual_seed(5)
    n = 1 << 26
    wb = torch.randint(0x35800000, 0x40000000, (n,), device=dev, generator=g, dtype=torch.int64).to(torch.int32)
    nb = torch.randint(0x2B8CBCCC, 0x44000000, (n,), device=dev, generator=g, dtype=torch.int64).to(torch.int32)
    nb[0::16] |= 0x007FFFFF  # all-ones significands
    nb[1::16] &= -0x00800000  # powers of two
    wb[2::7] = 0
    w, d = wb.view(torch.float32), nb.view(torch.float32)
    out = torch.empty_like(w)
    with fsb.Context(0) as ctx:
        fsb.check_normalise(ctx, w, d, out)
    ref = w / d
    assert torch.equal(out.view(torch.int32), ref.view(torch.int32)), int((out != ref).sum())
