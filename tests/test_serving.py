"""Serving form on the device: a mixed request stream admitted against a
small HBM budget, stacks in flight on several contexts; every result must be
the same alone and in the mix (bit-identical: each stack's kernels see only
its own state, whatever else runs beside it)."""
import numpy as np
import pytest

from __graft_entry__ import load_package

fsb = load_package()
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    if not t.cuda.is_available():
        pytest.skip("no CUDA device")
    return t


def test_mixed_stream_same_alone_and_in_the_mix(torch):
    sizes = ((320, 240), (640, 480), (800, 600))
    ctx = fsb.Context(0)
    pool = fsb.serving.SynthFramePool(ctx, torch, 0, seed=5, sizes=sizes, depth={s: 8 for s in sizes},
                                      scene=fsb.SCENE_SMALL)
    rng = np.random.default_rng(2)
    reqs, t = [], 0.0
    for i in range(12):
        t += float(rng.exponential(0.01))
        w, h = sizes[int(rng.integers(0, len(sizes)))]
        reqs.append(fsb.serving.StackRequest(i, t, w, h, int(rng.integers(3, 9)), frame_interval_s=0.001))
    # a budget that holds about two of the larger stacks at once
    roi_big = pool.roi(fsb.serving.StackRequest(0, 0, 800, 600, 8))
    big = fsb.stack_footprint(fsb.stack_desc(800, 600, 8, roi_big), 1 << 50)[0]
    budget = int(2.2 * big)
    with fsb.serving.StackServer(0, hbm_budget_bytes=budget, workers=3, max_stack_fraction=0.5) as srv:
        rep = srv.serve(reqs, pool.roi, pool.frame, torch, keep_outputs=True)
    s = rep.summary()
    assert s["requests"] == len(reqs)
    assert rep.peak_reserved_bytes <= budget
    assert s["p50_latency_ms"] <= s["p99_latency_ms"]
    for r in rep.results:
        assert r.done_s >= r.admitted_s >= r.arrival_s
    # alone: the same frames through a fresh context, one stack at a time, in
    # the pass-2 mode the server ran the request in (cache and resident give
    # the same bytes; laps rounds level 0 in its own order)
    alone_ctx = fsb.Context(0)
    for req, res in zip(sorted(reqs, key=lambda r: r.arrival_s), rep.results):
        roi = pool.roi(req)
        st = fsb.PyramidContrastStack(alone_ctx, req.width, req.height, req.frames, roi=roi, pass2_mode=res.pass2)
        for i in range(req.frames):
            buf, stride, pose = pool.frame(req, i)
            st.add_frame_device(buf, stride, pose)
        out = st.finish()
        st.close()
        assert np.array_equal(out, res.output), req
    alone_ctx.close()
    ctx.close()
