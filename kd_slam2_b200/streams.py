"""Seeded multi-stream registration traces for the served form.

Each sensor stream moves through one shared box scene with its own constant body
velocity (forward speed and yaw rate); scan i starts where scan i-1 ended, as in
the CT model's end pose X * [R(w T), t T].  A stream brings an initial local map
(the union of a few static scans taken before its trajectory, in the world frame),
then one request per scan: the scan in the sensor frame with per-point stamps, an
initial guess perturbed from the true start pose, and an arrival time.  The beam
mix is 16/32/64/128 beams (16k-262k rays), 70% of the requests are CT-ICP and 30%
rigid ICP, and arrivals are Poisson at a given rate per stream.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import synth

BEAM_MIX = (16, 32, 64, 128)


def beam_layout(beams: int):
    """(cols, elevation range) of a scan with this many beams."""
    cols = 2048 if beams >= 128 else 1024
    elev = (-15.0, 15.0) if beams <= 32 else (-22.5, 22.5)
    return cols, elev


def rodrigues(w):
    w = np.asarray(w, np.float64)
    a = np.linalg.norm(w)
    if a < 1e-15:
        return np.eye(3)
    k = w / a
    K = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
    return np.eye(3) + np.sin(a) * K + (1 - np.cos(a)) * (K @ K)


def compose(A, B):
    A = np.asarray(A, np.float64).reshape(3, 4)
    B = np.asarray(B, np.float64).reshape(3, 4)
    C = np.zeros((3, 4))
    C[:, :3] = A[:, :3] @ B[:, :3]
    C[:, 3] = A[:, :3] @ B[:, 3] + A[:, 3]
    return C


def motion(v, T):
    """[R(w T) | t T]: the pose change over T seconds at body velocity v = [t; w]."""
    M = np.zeros((3, 4))
    M[:, :3] = rodrigues(np.asarray(v[3:], np.float64) * T)
    M[:, 3] = np.asarray(v[:3], np.float64) * T
    return M


@dataclass
class StreamTrace:
    beams: int
    max_points: int
    map_xyz: np.ndarray
    vel: np.ndarray


@dataclass
class RequestTrace:
    stream: int
    seq: int
    kind: int          # 0 ICP, 1 CT-ICP
    xyz: np.ndarray
    stamps: np.ndarray
    X_true: np.ndarray
    X0: np.ndarray
    v0: np.ndarray
    arrival: float


@dataclass
class Trace:
    streams: list = field(default_factory=list)
    requests: list = field(default_factory=list)  # submission order (non-decreasing arrival)


def make_trace(seed: int, num_streams: int = 16, scans_per_stream: int = 20, rate_hz: float = 10.0,
               saturate: bool = False, ct_fraction: float = 0.7, map_scans: int = 5, beam_mix=BEAM_MIX,
               scene_seed: int = 1005, guess_t: float = 0.1, guess_deg: float = 1.0, threads: int = 8,
               map_layout=None) -> Trace:
    """A served-registration trace.  saturate=True makes every request arrive at 0
    (submitted round-robin by scan index); otherwise arrivals are Poisson at rate_hz
    per stream.  map_layout = (beams, cols, elevation range) of the initial maps' static
    scans (default: the stream's own layout)."""
    rng = np.random.default_rng(seed)
    boxes = synth.scene(scene_seed)
    tr = Trace()
    per_stream = []
    for s in range(num_streams):
        beams = beam_mix[s % len(beam_mix)]
        cols, elev = beam_layout(beams)
        yaw = rng.uniform(-np.pi, np.pi)
        start = synth.pose((rng.uniform(-15, 15), rng.uniform(-15, 15), 1.8), (0.0, 0.0, yaw))
        vel = np.array([rng.uniform(6.0, 12.0), 0.0, 0.0, 0.0, 0.0, np.deg2rad(rng.uniform(-20.0, 20.0))])
        # initial map: static scans at the poses of the map_scans scans before the start
        back = motion(-vel, 0.1)
        poses_back = []
        X = start
        for _ in range(map_scans):
            X = compose(X, back)
            poses_back.append(X)
        pts = []
        mb, mc, me = (beams, cols, elev) if map_layout is None else map_layout
        for k, Xm in enumerate(poses_back):
            xyz, _ = synth.scan(boxes, Xm, None, beams=mb, cols=mc, elev=me,
                                seed=seed * 100003 + s * 1009 + 500 + k, threads=threads)
            pts.append(synth.transform(xyz, Xm))
        tr.streams.append(StreamTrace(beams=beams, max_points=beams * cols,
                                      map_xyz=np.ascontiguousarray(np.concatenate(pts)), vel=vel))
        # requests
        reqs = []
        X = start
        t_arr = 0.0
        for i in range(scans_per_stream):
            xyz, st = synth.scan(boxes, X, vel, beams=beams, cols=cols, elev=elev, t_start=0.1 * i,
                                 seed=seed * 100003 + s * 1009 + i, threads=threads)
            d = rng.normal(size=3)
            d /= np.linalg.norm(d)
            a = rng.normal(size=3)
            a /= np.linalg.norm(a)
            P = synth.pose(guess_t * rng.uniform(0.5, 1.0) * d, np.deg2rad(guess_deg) * rng.uniform(0.5, 1.0) * a)
            X0 = compose(X, P)
            kind = 1 if rng.uniform() < ct_fraction else 0
            v0 = vel * (1.0 + 0.05 * rng.normal(size=6)) if kind == 1 else np.zeros(6)
            t_arr += rng.exponential(1.0 / rate_hz)
            reqs.append(RequestTrace(stream=s, seq=i, kind=kind, xyz=xyz, stamps=st, X_true=X, X0=X0, v0=v0,
                                     arrival=t_arr))
            X = compose(X, motion(vel, 0.1))
        per_stream.append(reqs)
    allr = [r for rs in per_stream for r in rs]
    allr.sort(key=lambda r: (r.arrival, r.stream))
    tr.requests = allr
    return saturated(tr) if saturate else tr


def saturated(tr: Trace) -> Trace:
    """The same requests all arriving at 0, submitted round-robin by scan index."""
    from dataclasses import replace
    order = sorted(tr.requests, key=lambda r: (r.seq, r.stream))
    return Trace(streams=tr.streams, requests=[replace(r, arrival=0.0) for r in order])


def serve(trace: Trace, serial: bool = False, tree=None, icp=None, ct=None, inputs=None, timeout: float = 600.0,
          **server_params):
    """Runs a trace through a kds Server; returns (results in trace order, stats, seconds).
    inputs: optional list of (xyz, stamps) per request to submit in place of the trace's
    arrays (torch tensors in device or page-locked host memory)."""
    import time

    from . import Server
    srv = Server(tree=tree, icp=icp, ct=ct, serial=1 if serial else 0, **server_params)
    try:
        for st in trace.streams:
            srv.add_stream(st.map_xyz, st.max_points)
        tickets = []
        for k, r in enumerate(trace.requests):
            xyz, stamps = (r.xyz, r.stamps) if inputs is None else inputs[k]
            tickets.append(srv.submit(r.stream, r.kind, xyz, stamps, r.X0, r.v0, r.arrival))
        t0 = time.perf_counter()
        srv.start()
        srv.drain(timeout)
        secs = time.perf_counter() - t0
        results = [srv.result(t) for t in tickets]
        stats = srv.stats()
    finally:
        srv.free()
    return results, stats, secs
