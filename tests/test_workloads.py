"""Seeded workload generators (CPU): served-registration traces and bundle-adjustment pairs."""
import numpy as np

from kd_slam2_b200 import ba, streams


def test_trace_orders_and_seeds():
    poi = streams.make_trace(11, num_streams=3, scans_per_stream=4, rate_hz=10.0, beam_mix=(16, 32), map_scans=1)
    sat = streams.saturated(poi)
    again = streams.make_trace(11, num_streams=3, scans_per_stream=4, rate_hz=10.0, beam_mix=(16, 32), map_scans=1)
    assert len(poi.requests) == len(sat.requests) == 12
    arr = [r.arrival for r in poi.requests]
    assert arr == sorted(arr) and arr[0] > 0.0
    assert all(r.arrival == 0.0 for r in sat.requests)
    # saturated: round-robin by scan index
    assert [(r.seq, r.stream) for r in sat.requests] == sorted((r.seq, r.stream) for r in sat.requests)
    # per stream, requests keep their order; the scans are the same in both traces and reproducible
    for s in range(3):
        seqs = [r.seq for r in poi.requests if r.stream == s]
        assert seqs == sorted(seqs)
    key = {(r.stream, r.seq): r for r in poi.requests}
    for r in sat.requests:
        assert np.array_equal(r.xyz, key[(r.stream, r.seq)].xyz)
    for a, b in zip(poi.requests, again.requests):
        assert np.array_equal(a.xyz, b.xyz) and np.array_equal(a.X0, b.X0) and a.kind == b.kind
    # stream layout: beams 16 / 32, max points from the layout
    assert [st.beams for st in poi.streams] == [16, 32, 16]
    assert all(len(r.xyz) <= poi.streams[r.stream].max_points for r in poi.requests)


def test_trace_motion_model():
    tr = streams.make_trace(3, num_streams=1, scans_per_stream=3, beam_mix=(16,), map_scans=1)
    rs = sorted(tr.requests, key=lambda r: r.seq)
    v = tr.streams[0].vel
    for a, b in zip(rs, rs[1:]):
        want = streams.compose(a.X_true, streams.motion(v, 0.1))
        assert np.allclose(b.X_true, want, atol=1e-12)


def test_ba_pairs_within_radius():
    wl = ba.make_workload(seed=2, num_keyframes=8, min_pts=2000, max_pts=5000, beams=16, cols=512, threads=4)
    assert len(wl.keyframes) == 8
    n = [len(k.xyz) for k in wl.keyframes]
    assert min(n) >= 1000 and max(n) <= 5000
    P = np.array([k.X[:2, 3] for k in wl.keyframes])
    pairs = {(p.i, p.j) for p in wl.pairs}
    for i in range(8):
        for j in range(i + 1, 8):
            assert ((i, j) in pairs) == (np.linalg.norm(P[i] - P[j]) < 30.0)
    assert sorted({p.kind for p in wl.pairs}) == [0, 1]
    for p in wl.pairs:
        Xj = streams.compose(wl.keyframes[p.i].X, p.X_true)
        assert np.allclose(Xj, wl.keyframes[p.j].X, atol=1e-9)


def test_track_is_closed_and_continuous():
    s = np.linspace(0.0, ba.LOOP_LEN, 4001)
    pts = np.array([ba.track_pose(x)[0] for x in s])
    steps = np.linalg.norm(np.diff(pts, axis=0), axis=1)
    assert steps.max() < 1.01 * ba.LOOP_LEN / 4000
    assert np.allclose(pts[0], pts[-1], atol=1e-6)
