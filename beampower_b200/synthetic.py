"""Seeded synthetic workloads with the shapes of the beamforming benchmarks.

No public dataset is involved: the reference's tutorial data (IRIS waveforms,
an eikonal travel-time table) is not available, so every workload here is
generated from a fixed recipe with ``numpy.random.default_rng(seed)`` and a
fixed draw order (stations -> grid -> noise -> events):

* stations at seeded uniform (x, y) in a square, depth 0;
* a regular source grid spanning the square and a depth range, flattened
  with depth slowest and x fastest (``meshgrid(..., indexing="ij")`` over
  (depth, y, x), the order the reference tutorial uses for its travel-time
  grid, notebooks/2_travel_times.ipynb cell 24);
* ``time_delays = rint(fs * hypocentral_distance / v)`` with v_P = 6.0 km/s
  and v_S = 3.46 km/s, minus each source's minimum P delay;
* three channels (Z, N, E); features are |N(0, 1)| (or |Student-t|) noise
  smoothed by a 25-sample moving average, plus Gaussian pulses
  (sigma = 5 samples, amplitude 5) for injected events: P on Z, S on N and E;
* ``weights_phases``: Z -> P = 1 and N/E -> S = 1, everything else 0.
"""
from __future__ import annotations

import hashlib
from dataclasses import dataclass, field

import numpy as np

V_P = 6.0
V_S = 3.46
PULSE_SIGMA = 5.0
PULSE_AMPLITUDE = 5.0
SMOOTH = 25


@dataclass(frozen=True)
class NetworkSpec:
    """Recipe of one synthetic beamforming workload."""

    name: str
    n_stations: int
    square_km: float
    fs: float
    n_samples: int
    grid: tuple  # (nx, ny, nz)
    depth_km: float
    n_events: int
    max_epicentral_km: float | None = None  # weights 0 beyond this distance
    noise: str = "normal"  # "normal" or "student_t3"
    seed: int = 0
    extra: dict = field(default_factory=dict)

    @property
    def n_sources(self) -> int:
        return int(np.prod(self.grid))


# Plain beamform at tutorial scale: 4,000 sources, 20 stations, 2 phases.
SMALL = NetworkSpec("small-4k-src-20-sta-6000-samples", 20, 50.0, 25.0, 6000,
                    (20, 20, 10), 20.0, 3)
# The plain method at scale: 400,000 sources, 60 stations, 1 h at 50 Hz.
LARGE = NetworkSpec("large-400k-src-60-sta-180000-samples", 60, 150.0, 50.0,
                    180_000, (100, 100, 40), 40.0, 30, max_epicentral_km=100.0)
# The small network with heavy-tailed noise (precision stress case).
SMALL_HEAVY = NetworkSpec("small-heavy-tailed", 20, 50.0, 25.0, 6000,
                          (20, 20, 10), 20.0, 3, noise="student_t3")

# A regional network: 64,000 sources ~10 km apart over 800 x 800 km, 100 Hz,
# so that a tile's delay windows span 1,000-2,000 samples (wider than the
# 16-bit default kernel shape holds).
REGIONAL = NetworkSpec("regional-64k-src-60-sta-120000-samples", 60, 800.0, 100.0,
                       120_000, (80, 80, 10), 40.0, 5)

SPECS = {s.name: s for s in (SMALL, LARGE, SMALL_HEAVY, REGIONAL)}


def _smooth(x: np.ndarray, width: int) -> np.ndarray:
    """Centred moving average along the last axis (zero padded), float32."""
    pad_l = width // 2
    pad_r = width - 1 - pad_l
    xp = np.pad(x.astype(np.float64), [(0, 0)] * (x.ndim - 1) + [(pad_l, pad_r)])
    c = np.cumsum(xp, axis=-1)
    c = np.concatenate([np.zeros(c.shape[:-1] + (1,)), c], axis=-1)
    return ((c[..., width:] - c[..., :-width]) / width).astype(np.float32)


def source_grid(spec: NetworkSpec) -> np.ndarray:
    """(n_sources, 3) source coordinates (x, y, z) in km, x fastest."""
    nx, ny, nz = spec.grid
    xs = np.linspace(0.0, spec.square_km, nx)
    ys = np.linspace(0.0, spec.square_km, ny)
    zs = np.linspace(0.0, spec.depth_km, nz)
    zg, yg, xg = np.meshgrid(zs, ys, xs, indexing="ij")
    return np.stack([xg.ravel(), yg.ravel(), zg.ravel()], axis=1)


def travel_time_delays(stations: np.ndarray, sources: np.ndarray, fs: float,
                       chunk: int = 65536) -> np.ndarray:
    """int32 (n_sources, n_stations, 2) delays in samples, P then S, each
    source shifted so that its earliest P arrival is at delay 0."""
    n_src = sources.shape[0]
    out = np.empty((n_src, stations.shape[0], 2), dtype=np.int32)
    for a in range(0, n_src, chunk):
        src = sources[a:a + chunk]
        dx = src[:, None, 0] - stations[None, :, 0]
        dy = src[:, None, 1] - stations[None, :, 1]
        dz = src[:, None, 2] - stations[None, :, 2]
        dist = np.sqrt(dx * dx + dy * dy + dz * dz)
        tp = np.rint(fs * dist / V_P).astype(np.int64)
        ts = np.rint(fs * dist / V_S).astype(np.int64)
        ref = tp.min(axis=1, keepdims=True)
        out[a:a + chunk, :, 0] = tp - ref
        out[a:a + chunk, :, 1] = ts - ref
    return out


def make_workload(spec: NetworkSpec):
    """Return a dict with the four ``beamform`` inputs plus ground truth.

    Keys: waveform_features (S, 3, T) f32, time_delays (N, S, 2) i32,
    weights_phases (S, 3, 2) f32, weights_sources (N, S) f32,
    events [(source, origin_sample)], stations (S, 3), sources (N, 3).
    """
    rng = np.random.default_rng(spec.seed)
    S, T = spec.n_stations, spec.n_samples
    # stations
    stations = np.zeros((S, 3))
    stations[:, :2] = rng.uniform(0.0, spec.square_km, size=(S, 2))
    # grid and delays
    sources = source_grid(spec)
    delays = travel_time_delays(stations, sources, spec.fs)
    if spec.max_epicentral_km is None:
        weights_sources = np.ones((sources.shape[0], S), dtype=np.float32)
    else:
        weights_sources = np.empty((sources.shape[0], S), dtype=np.float32)
        for a in range(0, sources.shape[0], 65536):
            src = sources[a:a + 65536]
            epi = np.hypot(src[:, None, 0] - stations[None, :, 0],
                           src[:, None, 1] - stations[None, :, 1])
            weights_sources[a:a + 65536] = (epi <= spec.max_epicentral_km)
    # noise
    if spec.noise == "normal":
        raw = np.abs(rng.standard_normal((S, 3, T), dtype=np.float32))
    elif spec.noise == "student_t3":
        raw = np.abs(rng.standard_t(3.0, size=(S, 3, T))).astype(np.float32)
    else:
        raise ValueError(f"unknown noise model {spec.noise!r}")
    features = _smooth(raw, SMOOTH)
    # events: P pulse on Z (channel 0), S pulse on N and E (channels 1, 2)
    events = []
    half = int(np.ceil(6 * PULSE_SIGMA))
    taps = np.arange(-half, half + 1)
    pulse = (PULSE_AMPLITUDE * np.exp(-0.5 * (taps / PULSE_SIGMA) ** 2)).astype(np.float32)
    for _ in range(spec.n_events):
        src = int(rng.integers(0, sources.shape[0]))
        dmax = int(delays[src].max())
        t0 = int(rng.integers(half, max(half + 1, T - dmax - half - 1)))
        events.append((src, t0))
        for s in range(S):
            for ch, ph in ((0, 0), (1, 1), (2, 1)):
                c = t0 + int(delays[src, s, ph])
                lo, hi = c - half, c + half + 1
                a, b = max(lo, 0), min(hi, T)
                if a < b:
                    features[s, ch, a:b] += pulse[a - lo:b - lo]
    weights_phases = np.zeros((S, 3, 2), dtype=np.float32)
    weights_phases[:, 0, 0] = 1.0
    weights_phases[:, 1:, 1] = 1.0
    return {
        "waveform_features": features,
        "time_delays": delays,
        "weights_phases": weights_phases,
        "weights_sources": weights_sources,
        "events": events,
        "stations": stations,
        "sources": sources,
        "spec": spec,
    }


def digest(*arrays: np.ndarray) -> str:
    """sha256 over the raw bytes of the given arrays (shape-tagged)."""
    h = hashlib.sha256()
    for a in arrays:
        a = np.ascontiguousarray(a)
        h.update(str((a.dtype.str, a.shape)).encode())
        h.update(a.tobytes())
    return h.hexdigest()


def nominal_terms(n_sources: int, n_samples: int, n_stations: int, n_phases: int) -> int:
    """Beam terms of one call: sources x samples x stations x phases."""
    return int(n_sources) * int(n_samples) * int(n_stations) * int(n_phases)


# ---------------------------------------------------------------------------
# Batching workload: many detection windows over one 100-station network and
# two source grids (400,000 and 50,000 points).  Each window has a seeded
# length of 1-30 min at 50 Hz, a station subset of 20-80 stations (applied
# as zero weights / a station mask) and 1-5 injected events.
# ---------------------------------------------------------------------------
@dataclass(frozen=True)
class BatchSpec:
    name: str = "batch-128-windows-100-sta-400k-and-50k-src"
    n_stations: int = 100
    square_km: float = 150.0
    fs: float = 50.0
    grids: tuple = ((100, 100, 40, 40.0), (50, 50, 20, 20.0))  # (nx, ny, nz, depth_km)
    n_windows: int = 128
    t_range: tuple = (3000, 90000)
    subset: tuple = (20, 80)
    events: tuple = (1, 5)
    seed: int = 0


BATCH = BatchSpec()


def make_batch_workload(spec: BatchSpec = BATCH, n_windows: int | None = None):
    """Stations, per-grid (delays, weights) and the window list.

    Windows are dicts {table, n_samples, stations (sorted list), events
    [(source, origin)], seed}; their features are drawn by
    ``window_features`` (numpy) or ``window_features_torch`` (device)."""
    rng = np.random.default_rng(spec.seed)
    S = spec.n_stations
    stations = np.zeros((S, 3))
    stations[:, :2] = rng.uniform(0.0, spec.square_km, size=(S, 2))
    grids = []
    for nx, ny, nz, depth in spec.grids:
        g = NetworkSpec("grid", S, spec.square_km, spec.fs, 1, (nx, ny, nz), depth, 0)
        src = source_grid(g)
        D = travel_time_delays(stations, src, spec.fs)
        W = np.ones((src.shape[0], S), dtype=np.float32)
        grids.append((D, W))
    alpha = np.zeros((S, 3, 2), dtype=np.float32)
    alpha[:, 0, 0] = 1.0
    alpha[:, 1:, 1] = 1.0
    windows = []
    n = spec.n_windows if n_windows is None else n_windows
    for i in range(n):
        table = int(rng.integers(0, len(grids)))
        T = int(rng.integers(spec.t_range[0], spec.t_range[1] + 1))
        k = int(rng.integers(spec.subset[0], spec.subset[1] + 1))
        st = sorted(int(s) for s in rng.choice(S, size=k, replace=False))
        D = grids[table][0]
        evs = []
        for _ in range(int(rng.integers(spec.events[0], spec.events[1] + 1))):
            src = int(rng.integers(0, D.shape[0]))
            dmax = int(D[src].max())
            if T - dmax - 40 > 40:
                evs.append((src, int(rng.integers(40, T - dmax - 40))))
        windows.append({"table": table, "n_samples": T, "stations": st, "events": evs,
                        "seed": int(rng.integers(0, 2**31 - 1))})
    return {"stations": stations, "grids": grids, "weights_phases": alpha,
            "windows": windows, "spec": spec}


def window_features(wl, i):
    """(S, 3, T) float32 features of window i (numpy)."""
    w = wl["windows"][i]
    S = wl["spec"].n_stations
    rng = np.random.default_rng(w["seed"])
    F = _smooth(np.abs(rng.standard_normal((S, 3, w["n_samples"]), dtype=np.float32)), SMOOTH)
    _inject(F, wl["grids"][w["table"]][0], w["events"])
    return F


def window_features_torch(wl, i, device):
    """(S, 3, T) float32 features of window i drawn on the device (seeded,
    not bit-identical to ``window_features``)."""
    import torch
    w = wl["windows"][i]
    S = wl["spec"].n_stations
    g = torch.Generator(device=device)
    g.manual_seed(w["seed"])
    x = torch.randn((S * 3, 1, w["n_samples"]), generator=g, device=device).abs_()
    k = torch.full((1, 1, SMOOTH), 1.0 / SMOOTH, device=device)
    F = torch.nn.functional.conv1d(x, k, padding=SMOOTH // 2)[:, 0, :w["n_samples"]]
    F = F.reshape(S, 3, w["n_samples"]).contiguous()
    D = wl["grids"][w["table"]][0]
    half = int(np.ceil(6 * PULSE_SIGMA))
    taps = torch.arange(-half, half + 1, device=device, dtype=torch.float32)
    pulse = PULSE_AMPLITUDE * torch.exp(-0.5 * (taps / PULSE_SIGMA) ** 2)
    for src, t0 in w["events"]:
        for s in range(S):
            for ch, ph in ((0, 0), (1, 1), (2, 1)):
                c = t0 + int(D[src, s, ph])
                lo, hi = c - half, c + half + 1
                a, b = max(lo, 0), min(hi, w["n_samples"])
                if a < b:
                    F[s, ch, a:b] += pulse[a - lo:b - lo]
    return F


def _inject(F, D, events):
    S, _, T = F.shape
    half = int(np.ceil(6 * PULSE_SIGMA))
    taps = np.arange(-half, half + 1)
    pulse = (PULSE_AMPLITUDE * np.exp(-0.5 * (taps / PULSE_SIGMA) ** 2)).astype(np.float32)
    for src, t0 in events:
        for s in range(S):
            for ch, ph in ((0, 0), (1, 1), (2, 1)):
                c = t0 + int(D[src, s, ph])
                lo, hi = c - half, c + half + 1
                a, b = max(lo, 0), min(hi, T)
                if a < b:
                    F[s, ch, a:b] += pulse[a - lo:b - lo]


# ---------------------------------------------------------------------------
# Serving workload: 8 networks of 30-100 stations, grids of 50,000-400,000
# sources, sampling rates of 20, 50 or 100 Hz, 60 s chunks arriving as
# Poisson processes that total ~200 chunks/s, events at 0.1 per minute.
# ---------------------------------------------------------------------------
@dataclass(frozen=True)
class ServingSpec:
    name: str = "serving-8-networks-60s-chunks"
    n_networks: int = 8
    stations: tuple = (30, 100)
    grids: tuple = ((50, 50, 20), (100, 50, 20), (100, 100, 20), (100, 100, 40))
    fs: tuple = (20.0, 50.0, 100.0)
    chunk_s: float = 60.0
    total_rate: float = 200.0  # chunks / s over all networks
    events_per_min: float = 0.1
    square_km: float = 150.0
    depth_km: float = 40.0
    seed: int = 0


SERVING = ServingSpec()


def make_serving_networks(spec: ServingSpec = SERVING):
    """Per network: name, stations, fs, chunk length, delays (N, S, 2),
    weights (N, S), weights_phases and its Poisson rate (chunks / s)."""
    rng = np.random.default_rng(spec.seed)
    rates = rng.uniform(0.5, 1.5, size=spec.n_networks)
    rates *= spec.total_rate / rates.sum()
    nets = []
    for i in range(spec.n_networks):
        S = int(rng.integers(spec.stations[0], spec.stations[1] + 1))
        fs = float(spec.fs[int(rng.integers(0, len(spec.fs)))])
        nx, ny, nz = spec.grids[int(rng.integers(0, len(spec.grids)))]
        st = np.zeros((S, 3))
        st[:, :2] = rng.uniform(0.0, spec.square_km, size=(S, 2))
        g = NetworkSpec("grid", S, spec.square_km, fs, 1, (nx, ny, nz), spec.depth_km, 0)
        D = travel_time_delays(st, source_grid(g), fs)
        W = np.ones((D.shape[0], S), dtype=np.float32)
        A = np.zeros((S, 3, 2), dtype=np.float32)
        A[:, 0, 0] = 1.0
        A[:, 1:, 1] = 1.0
        nets.append({"name": f"net{i}", "n_stations": S, "fs": fs,
                     "chunk": int(round(spec.chunk_s * fs)), "delays": D, "weights": W,
                     "weights_phases": A, "rate": float(rates[i]),
                     "seed": int(rng.integers(0, 2**31 - 1))})
    return nets


def serving_record(net, n_chunks, events_per_min=SERVING.events_per_min):
    """A continuous (S, 3, n_chunks * chunk) record for one network with
    Poisson events, to be cut into chunks."""
    rng = np.random.default_rng(net["seed"])
    S, L = net["n_stations"], net["chunk"]
    T = n_chunks * L
    F = _smooth(np.abs(rng.standard_normal((S, 3, T), dtype=np.float32)), SMOOTH)
    n_ev = rng.poisson(events_per_min * T / net["fs"] / 60.0)
    D = net["delays"]
    evs = []
    for _ in range(int(n_ev)):
        src = int(rng.integers(0, D.shape[0]))
        dmax = int(D[src].max())
        if T - dmax - 40 > 40:
            evs.append((src, int(rng.integers(40, T - dmax - 40))))
    _inject(F, D, evs)
    return F, evs
