"""Seeded synthetic scenarios in the reference's data model.

A ``Scenario`` holds what the reference builds in triton_init.h from a .cfg and
its input files: padded rows x cols fields (ghost ring included, row 0 =
north, Manning squared, closed walls as DEM ghost 1e6), the flattened forcing
tables and the loop parameters.  It can be loaded into a ``Domain`` and it can
be written out as a reference-format case (``write_case``: .cfg, ASCII
rasters, .hyg/.roff/.src/.extbc/.obs files) so the reference executable runs
the same inputs.

Workloads (all synthetic; no dataset is shipped or needed):
  dambreak   circular dam break on a flat frictionless bed (512x512, dx 1 m)
  thacker    planar oscillation in a paraboloid bowl (Thacker 1981), 2048x2048
  watershed  fractal terrain with a carved valley, rain, inflows and an open
             outflow edge (8192x8192 at full size)
  mixed      small random case exercising every forcing path (tests)
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

G = 9.81
WALL = 1e6  # closed-boundary DEM ghost value (matrix.h:929-945)


@dataclass
class Scenario:
    name: str
    dx: float
    z: np.ndarray            # padded DEM
    h: np.ndarray            # padded initial depth
    qx: np.ndarray
    qy: np.ndarray
    n2: np.ndarray           # padded Manning squared
    courant: float = 0.5
    hextra: float = 0.001
    open_boundaries: int = 0
    sim_duration: float = 1.0
    print_interval: float = 1.0
    print_observation: float = 0.0
    time_series: int = 0
    it_print: int = 10000
    time_step: float = 0.01
    xll: float = 0.0
    yll: float = 0.0
    # forcing, as flattened reference tables
    runoff: dict | None = None   # zone (padded int32), times[s], rates[zone*nrows+row] (m/s), nzones
    sources: dict | None = None  # cells (padded idx), times[s], flows[row*nsrc+src] (m3/s)
    extbc: dict | None = None    # cells, types, start, nrows, var1, var2
    obs_cells: np.ndarray | None = None
    meta: dict = field(default_factory=dict)

    @property
    def rows(self):
        return self.z.shape[0]

    @property
    def cols(self):
        return self.z.shape[1]

    @property
    def interior_cells(self):
        return (self.rows - 2) * (self.cols - 2)

    def init_dt(self):
        """compute_init_dt (triton_simulate.h:163-187)."""
        v = min(self.print_observation, self.print_interval) if self.time_series else self.print_interval
        if self.runoff is not None:
            v = min(v, self.runoff["times"][1] - self.runoff["times"][0])
        if self.sources is not None and len(self.sources["cells"]):
            v = min(v, self.sources["times"][1] - self.sources["times"][0])
        return v * 0.01

    def clock(self):
        return dict(simtime=0.0, sim_duration=self.sim_duration, print_interval=self.print_interval,
                    print_observation=self.print_observation if self.time_series else self.print_interval,
                    last_obs_time=0.0, init_dt=self.init_dt(), time_step=self.time_step, print_id=0,
                    it_count=0, it_print=self.it_print, time_series=self.time_series, time_increment_fixed=0,
                    runoff_row=self.runoff_row0(), src_idx_low=0)

    def runoff_row0(self):
        """process_runoff's initial row for simtime 0 (triton_init.h:1300-1310)."""
        return 0

    def to_domain(self, precision="fp64", stream=None):
        from .domain import Domain
        d = Domain(self.rows, self.cols, self.dx, self.courant, self.hextra, self.open_boundaries, precision,
                   stream=stream)
        d.set_state(self.h, self.qx, self.qy, self.z, self.n2)
        if self.runoff is not None:
            d.set_runoff(self.runoff["zone"], self.runoff["times"], self.runoff["rates"], self.runoff["nzones"])
        if self.sources is not None and len(self.sources["cells"]):
            d.set_sources(self.sources["cells"], self.sources["times"], self.sources["flows"])
        if self.extbc is not None and len(self.extbc["cells"]):
            e = self.extbc
            d.set_extbc(e["cells"], e["types"], e["start"], e["nrows"], e["var1"], e["var2"])
        if self.obs_cells is not None and len(self.obs_cells):
            d.set_observations(self.obs_cells)
        d.set_clock(**self.clock())
        return d


def _pad(interior, ghost=0.0):
    r, c = interior.shape
    out = np.full((r + 2, c + 2), ghost, dtype=np.float64)
    out[1:-1, 1:-1] = interior
    return out


def _walls(z_int, open_boundaries=0):
    z = _pad(z_int, WALL)
    if open_boundaries:
        z = _copy_ghosts(z)
    return z


def _copy_ghosts(a):
    """matrix<T>::copy_value_into_ghost_cells (matrix.h:848-865)."""
    a = a.copy()
    a[:, 0] = a[:, 1]
    a[:, -1] = a[:, -2]
    a[0, :] = a[1, :]
    a[-1, :] = a[-2, :]
    return a


def _centres(n_rows, n_cols, dx, xll=0.0, yll=0.0):
    """Cell-centre coordinates of the interior, row 0 = north (calc_src_row,
    triton_init.h:1602-1605)."""
    x = xll + (np.arange(n_cols) + 0.5) * dx
    y = yll + (n_rows - np.arange(n_rows) - 0.5) * dx
    return np.meshgrid(x, y)


# ---------------------------------------------------------------------------
def dambreak(n=512, dx=1.0, radius=50.0, depth=10.0, duration=5.0):
    """Circular dam break: flat frictionless bed, `depth` m inside a circle of
    `radius` m centred on the grid, dry outside, closed walls, CFL 0.5."""
    X, Y = _centres(n, n, dx)
    xc = yc = n * dx / 2
    inside = (X - xc) ** 2 + (Y - yc) ** 2 <= radius ** 2
    h = _pad(np.where(inside, depth, 0.0))
    zero = np.zeros_like(h)
    return Scenario("dambreak", dx, _walls(np.zeros((n, n))), h, zero.copy(), zero.copy(), zero.copy(),
                    courant=0.5, hextra=0.001, sim_duration=duration, print_interval=duration,
                    meta=dict(n=n, radius=radius, depth=depth))


def thacker_state(X, Y, t, h0, a, eta, xc, yc):
    """Planar-surface solution of Thacker (1981) in the bowl z = h0 r^2/a^2.

    omega = sqrt(2 g h0)/a; the free surface stays a tilted plane,
        w = h0 + (eta h0 / a^2) (2 x' cos(wt) + 2 y' sin(wt) - eta),
    h = max(w - z, 0), u = -eta omega sin(wt), v = eta omega cos(wt), with
    x', y' measured from the bowl centre.  eta is the horizontal shoreline
    excursion; the surface amplitude at the rim (r = a) is A = 2 eta h0 / a."""
    om = math.sqrt(2 * G * h0) / a
    xp, yp = X - xc, Y - yc
    z = h0 * (xp ** 2 + yp ** 2) / a ** 2
    w = h0 + (eta * h0 / a ** 2) * (2 * xp * math.cos(om * t) + 2 * yp * math.sin(om * t) - eta)
    h = np.maximum(w - z, 0.0)
    u = -eta * om * math.sin(om * t) * np.ones_like(h)
    v = eta * om * math.cos(om * t) * np.ones_like(h)
    return z, h, h * u, h * v, om


def thacker(n=2048, dx=4.0, h0=10.0, a=3000.0, amplitude=0.5, periods=2.0, hextra=0.001):
    """Thacker planar oscillation; `amplitude` is the rim surface amplitude
    A = 2 eta h0 / a (0.5 m -> eta = 75 m for h0 = 10 m, a = 3000 m)."""
    eta = amplitude * a / (2 * h0)
    X, Y = _centres(n, n, dx)
    xc = yc = n * dx / 2
    z, h, qx, qy, om = thacker_state(X, Y, 0.0, h0, a, eta, xc, yc)
    period = 2 * math.pi / om
    dur = periods * period
    sc = Scenario("thacker", dx, _walls(z), _pad(h), _pad(qx), _pad(qy), np.zeros((n + 2, n + 2)),
                  courant=0.5, hextra=hextra, sim_duration=dur, print_interval=dur,
                  meta=dict(n=n, h0=h0, a=a, eta=eta, omega=om, period=period, xc=xc, yc=yc))
    return sc


# ---------------------------------------------------------------------------
def _value_noise(rng, n_rows, n_cols, octaves=8, hurst=0.8):
    """Sum of bilinear value-noise octaves, octave k amplitude 2^(-hurst k)."""
    out = np.zeros((n_rows, n_cols))
    for k in range(octaves):
        cells = 2 ** (k + 1)
        g = rng.standard_normal((cells + 2, cells + 2))
        yi = np.linspace(0, cells, n_rows)
        xi = np.linspace(0, cells, n_cols)
        y0 = np.floor(yi).astype(int)
        x0 = np.floor(xi).astype(int)
        fy = (yi - y0)[:, None]
        fx = (xi - x0)[None, :]
        v = (g[y0][:, x0] * (1 - fy) * (1 - fx) + g[y0 + 1][:, x0] * fy * (1 - fx) +
             g[y0][:, x0 + 1] * (1 - fy) * fx + g[y0 + 1][:, x0 + 1] * fy * fx)
        out += v * 2.0 ** (-hurst * k)
    return out


def _value_noise_torch(seed, n_rows, n_cols, octaves=8, hurst=0.8):
    """_value_noise drawn on the GPU with torch (same octave lattices and
    bilinear interpolation, torch's generator): seconds become milliseconds
    on 4096^2 grids.  Returns a float64 numpy array."""
    import torch
    import torch.nn.functional as F
    g = torch.Generator(device="cuda")
    g.manual_seed(int(seed))
    out = torch.zeros((n_rows, n_cols), dtype=torch.float64, device="cuda")
    for k in range(octaves):
        cells = 2 ** (k + 1)
        lat = torch.randn((1, 1, cells + 1, cells + 1), generator=g, device="cuda", dtype=torch.float64)
        out += F.interpolate(lat, size=(n_rows, n_cols), mode="bilinear", align_corners=True)[0, 0] * \
            2.0 ** (-hurst * k)
    return out.cpu().numpy()


def watershed(n=8192, dx=10.0, seed=1234, duration=6 * 3600.0, rain_mm_h=50.0, rain_hours=1.0,
              manning_median=0.035, manning_sigma=0.3, relief=300.0, valley_depth=40.0, peak_flow=500.0,
              nsrc=3, print_interval=None, gpu_noise=False):
    """Fractal watershed: value-noise DEM rescaled to 0..relief m with a carved
    meandering valley draining to the southern (lowest) edge, log-normal
    Manning, `nsrc` triangular inflow hydrographs (0 -> peak at 2 h -> 0 at
    4 h), uniform rain for `rain_hours`, and an open (extbc type 0) outflow
    along the southern edge."""
    rng = np.random.default_rng(seed)
    if gpu_noise:  # same recipe, terrain and roughness drawn on the GPU
        dem = _value_noise_torch(rng.integers(1 << 31), n, n)
    else:
        dem = _value_noise(np.random.default_rng(rng.integers(1 << 31)), n, n)
    dem = (dem - dem.min()) / max(dem.max() - dem.min(), 1e-12) * relief
    # tilt toward the south edge so it is the lowest
    rows = np.arange(n)[:, None]
    dem = dem * 0.7 + relief * 0.3 * (1 - rows / (n - 1))
    # meandering valley: centre column x_c(row) = n/2 + A sin(2 pi row / L)
    cols = np.arange(n)[None, :]
    xc = n / 2 + 0.15 * n * np.sin(2 * np.pi * rows / (0.6 * n))
    halfw = max(n / 64, 3.0)
    dist = np.abs(cols - xc) / halfw
    carve = valley_depth * np.exp(-dist ** 2)
    dem = np.maximum(dem - carve, 0.0)
    if gpu_noise:
        import torch
        gm = torch.Generator(device="cuda")
        gm.manual_seed(int(rng.integers(1 << 31)))
        mann = torch.exp(np.log(manning_median) + manning_sigma * torch.randn(
            (n, n), generator=gm, device="cuda", dtype=torch.float64)).cpu().numpy()
    else:
        mann = np.exp(np.log(manning_median) + manning_sigma * np.random.default_rng(rng.integers(1 << 31))
                      .standard_normal((n, n)))
    z = _walls(dem)
    n2 = _copy_ghosts(_pad(mann)) ** 2
    zero = np.zeros_like(z)
    pi = print_interval or duration
    sc = Scenario("watershed", dx, z, zero.copy(), zero.copy(), zero.copy(), n2, courant=0.5, hextra=0.001,
                  sim_duration=duration, print_interval=pi, meta=dict(n=n, seed=seed, mann=mann))
    # inflows along the valley in the northern half: 0 -> peak at 2 h -> 0 at 4 h
    if nsrc > 0:
        src_rows = np.linspace(n * 0.1, n * 0.45, nsrc).astype(int)
        src_cols = (n / 2 + 0.15 * n * np.sin(2 * np.pi * src_rows / (0.6 * n))).astype(int)
        flows = np.zeros((4, nsrc))
        flows[1, :] = peak_flow
        sources_table(sc, list(zip(src_rows.tolist(), src_cols.tolist())), [0.0, 2.0, 4.0, 1000.0], flows)
    # uniform rain on one zone: (0 h, rain), (rain_hours, 0), (end, 0)
    end_h = max(duration / 3600.0, rain_hours + 1.0)
    runoff_table(sc, np.zeros((n, n), dtype=np.int32), [0.0, rain_hours, end_h], [[rain_mm_h], [0.0], [0.0]])
    # open outflow (type 0) along the southern edge, the lowest one
    extbc_segments(sc, [(0, (n - 1, 0), (n - 1, n - 1), None)])
    return sc


def ensemble(members=256, seed=2024, side_min=256, side_max=2048, dx_range=(5.0, 20.0), duration=3 * 3600.0,
             rain_range=(10.0, 100.0), rain_hours=1.0, manning_spread=0.3, max_side=None, gpu_noise=False):
    """Ensemble of rain-on-grid watershed members of uneven sizes: per member
    a side drawn log-uniformly in [side_min, side_max] (capped at max_side),
    a cell size in dx_range, a rain intensity in rain_range (mm/h) for
    rain_hours, the Manning median 0.035 perturbed uniformly by
    +/- manning_spread (relative) and its own terrain seed.  Members carry no point sources."""
    return list(ensemble_iter(members, seed, side_min, side_max, dx_range, duration, rain_range, rain_hours,
                              manning_spread, max_side, gpu_noise))


def ensemble_iter(members=256, seed=2024, side_min=256, side_max=2048, dx_range=(5.0, 20.0),
                  duration=3 * 3600.0, rain_range=(10.0, 100.0), rain_hours=1.0, manning_spread=0.3, max_side=None,
                  gpu_noise=False):
    """The members of ensemble(), built one at a time (a caller that loads
    each into a domain holds one member's host arrays at a time)."""
    rng = np.random.default_rng(seed)
    for i in range(members):
        side = int(np.exp(rng.uniform(np.log(side_min), np.log(side_max))))
        if max_side is not None:
            side = min(side, max_side)
        dx = float(rng.uniform(*dx_range))
        rain = float(rng.uniform(*rain_range))
        mann = 0.035 * (1.0 + float(rng.uniform(-manning_spread, manning_spread)))
        sc = watershed(n=side, dx=dx, seed=int(rng.integers(1 << 31)), duration=duration, rain_mm_h=rain,
                       rain_hours=rain_hours, manning_median=mann, nsrc=0, gpu_noise=gpu_noise)
        sc.name = f"member{i:03d}"
        yield sc


def extbc_segments(sc, segments):
    """Builds the external-boundary tables the reference derives from an
    .extbc file (process_boundary_condition, triton_init.h:869-1055) and
    applies its ghost-cell preprocessing (matrix.h:869-926 for the DEM and
    triton_init.h:1250-1289 for DEM/h/qx/qy).

    segments: list of (type, (row1, col1), (row2, col2), value) in interior
    0-based cell coordinates along one edge; value is the Froude number
    (type 3), the slope (type 2), ignored for type 0, or for type 1 a list of
    (hours, water level) rows.  Cells are listed from the lower to the higher
    row/column index, segment by segment, as create_involved_cells does."""
    R, C = sc.rows - 2, sc.cols - 2
    Cp = sc.cols
    cells, types, start, nrows, var1, var2 = [], [], [], [], [], []
    for bt, (r1, c1), (r2, c2), val in segments:
        if c1 == c2:
            loc = 0 if c1 == 0 else 2
            pts = [(r, c1) for r in range(min(r1, r2), max(r1, r2) + 1)]
        elif r1 == r2:
            loc = 1 if r1 == 0 else 3
            pts = [(r1, c) for c in range(min(c1, c2), max(c1, c2) + 1)]
        else:
            raise ValueError("segment must follow one edge")
        if bt == 1:
            rows_h = [(float(t), float(v)) for t, v in val]
            t_s = [t * 3600.0 for t, _ in rows_h]  # extBC::convert_to_secs
            lv = [v for _, v in rows_h]
        else:
            t_s = [float(val or 0.0)]
            lv = [float(val or 0.0)]
        s0 = len(var1)
        var1 += t_s
        var2 += lv
        for r, c in pts:
            cells.append((r + 1) * Cp + c + 1)
            types.append(bt)
            start.append(s0)
            nrows.append(len(t_s))
        # DEM ghosts next to the segment (copy_value_into_ghost_cells_location)
        z = sc.z
        for r, c in pts:
            ix, iy = r + 1, c + 1
            if loc == 0:
                z[ix, iy - 1] = z[ix, iy]
            if loc == 2:
                z[ix, iy + 1] = z[ix, iy]
            if loc == 1:
                z[ix - 1, iy] = z[ix, iy]
            if loc == 3:
                z[ix + 1, iy] = z[ix, iy]
            v = z[ix, iy]
            if r == 0 and c == 0:
                z[0, 0] = z[0, 1] = z[1, 0] = v
            if r == 0 and c == C - 1:
                z[0, Cp - 2] = z[0, Cp - 1] = z[1, Cp - 1] = v
            if r == R - 1 and c == 0:
                z[sc.rows - 2, 0] = z[sc.rows - 1, 0] = z[sc.rows - 1, 1] = v
            if r == R - 1 and c == C - 1:
                z[sc.rows - 2, Cp - 1] = z[sc.rows - 1, Cp - 2] = z[sc.rows - 1, Cp - 1] = v
        if not hasattr(sc, "_segments"):
            sc._segments = []
        sc._segments.append((bt, (r1, c1), (r2, c2), val))
    # per-cell ghost copies of DEM, h, qx, qy (triton_init.h:1250-1289)
    for ii in cells:
        ix, iy = divmod(ii, Cp)
        nb = []
        if iy == 1:
            nb.append(ii - 1)
        if iy == Cp - 2:
            nb.append(ii + 1)
        if ix == 1:
            nb.append(ii - Cp)
        if ix == sc.rows - 2:
            nb.append(ii + Cp)
        for g in nb:
            for a in (sc.z, sc.h, sc.qx, sc.qy):
                a.flat[g] = a.flat[ii]
    sc.extbc = dict(cells=np.array(cells, np.int32), types=np.array(types, np.int32),
                    start=np.array(start, np.int32), nrows=np.array(nrows, np.int32),
                    var1=np.array(var1, dtype=np.float64), var2=np.array(var2, dtype=np.float64))
    return sc


def sources_table(sc, cells_rc, times_h, flows):
    """Point sources at interior cells (row, col) with a hydrograph given in
    hours and m3/s (hydrograph::convert_time_hr_to_secs, inflow.h:260-272)."""
    Cp = sc.cols
    times_h = np.asarray(times_h, dtype=np.float64)
    flows = np.asarray(flows, dtype=np.float64).reshape(times_h.size, len(cells_rc))
    sc.sources = dict(cells=np.array([(r + 1) * Cp + c + 1 for r, c in cells_rc], np.int32),
                      times=times_h * 3600.0, flows=flows.reshape(-1), times_h=times_h, flows_rows=flows,
                      cells_rc=list(cells_rc))
    return sc


def runoff_table(sc, zone_interior, times_h, rates_mm_h):
    """Runoff zones with rates in mm/h per zone (columns) and time rows in
    hours, converted as read_inflows does (triton_init.h:155-162:
    hours->s, then /3600, then *0.001)."""
    times_h = np.asarray(times_h, dtype=np.float64)
    mm = np.asarray(rates_mm_h, dtype=np.float64).reshape(times_h.size, -1)
    nz = mm.shape[1]
    zone = np.zeros((sc.rows, sc.cols), dtype=np.int32)
    zone[1:-1, 1:-1] = zone_interior
    si = (mm / 3600.0) * 0.001
    sc.runoff = dict(zone=zone, times=times_h * 3600.0, rates=np.ascontiguousarray(si.T).reshape(-1), nzones=nz,
                     times_h=times_h, rates_mm_h=mm)
    return sc


def mixed(rows=37, cols=53, dx=5.0, seed=7, open_boundaries=0, friction=True, with_sources=True,
          with_runoff=True, with_extbc=True, duration=30.0, wet_fraction=0.5):
    """Small random case that drives every forcing path of the step: rough
    terrain with partly wet cells, friction, two sources sharing a cell,
    zoned runoff, external boundary cells of types 0-3 (segments sharing
    corners) and optional open boundaries."""
    rng = np.random.default_rng(seed)
    R, C = rows, cols
    dem = _value_noise(rng, R, C, octaves=4) * 2.0 + 5.0
    h = np.where(rng.random((R, C)) < wet_fraction, rng.random((R, C)) * 1.5, 0.0)
    h[rng.random((R, C)) < 0.1] = 0.0005  # below hextra
    qx = np.where(h > 0.01, rng.standard_normal((R, C)) * 0.3, 0.0)
    qy = np.where(h > 0.01, rng.standard_normal((R, C)) * 0.3, 0.0)
    mann = np.full((R, C), 0.03) + rng.random((R, C)) * 0.02 if friction else np.zeros((R, C))
    z = _walls(dem, open_boundaries)
    hp, qxp, qyp = _pad(h), _pad(qx), _pad(qy)
    if open_boundaries:
        hp, qxp, qyp = _copy_ghosts(hp), _copy_ghosts(qxp), _copy_ghosts(qyp)
    n2 = _copy_ghosts(_pad(mann)) ** 2
    sc = Scenario("mixed", dx, z, hp, qxp, qyp, n2, courant=0.5, hextra=0.001, open_boundaries=open_boundaries,
                  sim_duration=duration, print_interval=duration / 3, print_observation=duration / 7,
                  time_series=1, it_print=25)
    sc.meta["mann"] = mann
    if with_runoff:
        nz = 3
        t_h = np.array([0.0, 0.001, 0.0025, 0.004, 30.0])
        mm = np.round(rng.random((t_h.size, nz)) * 40.0 - 5.0, 3)  # includes small negative rates
        runoff_table(sc, rng.integers(0, nz, (R, C)), t_h, mm)
    if with_sources:
        cells_rc = [(R // 3, C // 4), (2 * R // 3, C // 2), (R // 3, C // 4)]
        t_h = np.array([0.0, 0.0015, 0.003, 0.006, 30.0])
        flows = np.round(rng.random((t_h.size, len(cells_rc))) * 2.0, 4)
        sources_table(sc, cells_rc, t_h, flows)
    if with_extbc:
        # east column: type 1 water level series; north row: type 3 (Froude)
        # sharing the NE corner, then type 2 (normal slope); west column:
        # type 2; south row: type 0 (open copy)
        extbc_segments(sc, [
            (1, (0, C - 1), (R - 1, C - 1), [(0.0, 6.0), (0.0017, 7.0), (0.0039, 6.5), (30.0, 6.5)]),
            (3, (0, C // 2), (0, C - 1), 0.8),
            (2, (0, 0), (0, C // 2 - 1), 0.002),
            (2, (1, 0), (R - 1, 0), 0.002),
            (0, (R - 1, 1), (R - 1, C - 2), None),
        ])
    Cp = C + 2
    sc.obs_cells = np.array([(R // 2 + 1) * Cp + C // 2 + 1, (2 + 1) * Cp + 3, (R) * Cp + C], dtype=np.int32)
    sc.meta["obs_rc"] = [(R // 2, C // 2), (2, 2), (R - 1, C - 1)]
    return sc


# ---------------------------------------------------------------------------
def _write_raster(path, a, fmt, dem_header=None, dtype=np.float64):
    """Interior raster in the reference's formats: ASCII rows separated by
    single spaces (matrix_io.h:77-149; the DEM adds a 6-line header,
    dem_utils.h:163-228) or binary (a header of 2 values, rows and cols, or
    6 DEM header values, in the raster's type, then row-major data,
    matrix_io.h:225-286)."""
    if fmt == "BIN":
        if dem_header is not None:
            hdr = np.array(dem_header, dtype=dtype)
        else:
            hdr = np.array([a.shape[0], a.shape[1]], dtype=dtype)
        with open(path, "wb") as f:
            hdr.tofile(f)
            np.ascontiguousarray(a, dtype=dtype).tofile(f)
    else:
        with open(path, "w") as f:
            if dem_header is not None:
                names = ["ncols", "nrows", "xllcorner", "yllcorner", "cellsize", "NODATA_value"]
                for k, v in zip(names, dem_header):
                    f.write(f"{k} {v!r}\n" if isinstance(v, float) else f"{k} {v}\n")
            for row in a:
                if dtype == np.int32:
                    f.write(" ".join(str(int(v)) for v in row) + "\n")
                else:  # repr keeps the double exactly; a '.' marks it as floating point
                    f.write(" ".join(_fmt(v) for v in row) + "\n")


def _fmt(v):
    s = repr(float(v))
    if "." not in s:
        if "e" in s or "E" in s:
            m, e = s.lower().split("e")
            s = f"{m}.0e{e}"
        else:
            s += ".0"
    return s


def _write_parts(base, suffix, a, fmt, parts, dtype=np.float64):
    """Partitioned raster (input_option=PAR): `parts` files <base>_NN<suffix>
    holding row slabs split as the reference splits rows among ranks
    (create_local_dims, mpi_utils.h:73-89), each without a DEM header; a
    binary file starts with its slab's rows and cols."""
    R = a.shape[0]
    r0 = 0
    for p in range(parts):
        rows = R // parts + (1 if p < R % parts else 0)
        _write_raster(f"{base}_{p:02d}{suffix}", a[r0:r0 + rows], fmt, dtype=dtype)
        r0 += rows


def write_case(sc, directory, fmt="BIN", output_format="BIN", output_folder="output", name=None,
               max_value_print="", partitions=0):
    """Writes `sc` as a reference-format case (cfg + inputs) into `directory`
    and returns the cfg path.  Paths inside the cfg are absolute.  The
    reference recovers the same padded arrays and tables from these files
    (initial fields, walls, Manning squared, forcing unit conversions, cell
    coordinates -> indices via calc_src_col/row).  partitions > 0 writes the
    rasters partitioned (input_option=PAR): an ASCII header file and one file
    per partition and field (triton_init.h:359-717)."""
    os.makedirs(directory, exist_ok=True)
    name = name or sc.name
    R, C = sc.rows - 2, sc.cols - 2
    dx = sc.dx
    P = lambda f: os.path.abspath(os.path.join(directory, f))
    ext = "bin" if fmt == "BIN" else "asc"
    mann = sc.meta.get("mann")
    if mann is None:
        mann = np.sqrt(sc.n2[1:-1, 1:-1])
    if partitions > 0:
        with open(P(f"{name}.header"), "w") as f:
            f.write(f"ncols {C}\nnrows {R}\nxllcorner {sc.xll!r}\nyllcorner {sc.yll!r}\ncellsize {dx!r}\n"
                    f"NODATA_value -9999\n")
        names = {k: P(f"{name}_{k}") for k in ("dem", "h", "qx", "qy", "mann")}
        _write_parts(names["dem"], ".dem", sc.z[1:-1, 1:-1], fmt, partitions)
        _write_parts(names["h"], ".out", sc.h[1:-1, 1:-1], fmt, partitions)
        _write_parts(names["qx"], ".out", sc.qx[1:-1, 1:-1], fmt, partitions)
        _write_parts(names["qy"], ".out", sc.qy[1:-1, 1:-1], fmt, partitions)
        _write_parts(names["mann"], ".mann", mann, fmt, partitions)
    else:
        names = {k: P(f"{name}.{k}.{ext}") for k in ("dem", "h", "qx", "qy", "mann")}
        _write_raster(names["dem"], sc.z[1:-1, 1:-1], fmt,
                      dem_header=[float(C), float(R), sc.xll, sc.yll, dx, -9999.0] if fmt == "BIN" else
                      [C, R, sc.xll, sc.yll, dx, -9999])
        _write_raster(names["h"], sc.h[1:-1, 1:-1], fmt)
        _write_raster(names["qx"], sc.qx[1:-1, 1:-1], fmt)
        _write_raster(names["qy"], sc.qy[1:-1, 1:-1], fmt)
        _write_raster(names["mann"], mann, fmt)

    def xy(r, c):
        return sc.xll + (c + 0.5) * dx, sc.yll + (R - r - 0.5) * dx

    cfg = {
        "dem_filename": names["dem"], "input_format": fmt, "input_option": "PAR" if partitions > 0 else "SEQ",
        "outfile_pattern": "%s/%s/%s_%02d_%02d", "output_format": output_format, "output_option": "SEQ",
        "output_folder": output_folder, "n_infile": names["mann"], "const_mann": "0.0",
        "h_infile": names["h"], "qx_infile": names["qx"], "qy_infile": names["qy"],
        "num_sources": "0", "num_runoffs": "0", "num_extbc": "0", "time_series_flag": str(int(sc.time_series)),
        "print_option": "huv", "sim_start_time": "0", "sim_duration": repr(float(sc.sim_duration)),
        "checkpoint_id": "0", "time_increment_fixed": "0", "time_step": repr(float(sc.time_step)),
        "print_interval": repr(float(sc.print_interval)), "it_print": str(int(sc.it_print)), "it_count": "0",
        "courant": repr(float(sc.courant)), "hextra": repr(float(sc.hextra)), "gpu_direct_flag": "0",
        "domain_decomposition": "static", "factor_interval_domain_decomposition": "2",
        "open_boundaries": str(int(sc.open_boundaries)),
    }
    if max_value_print:  # the reference's cfg parser needs a value after '=' (config_utils.h:216-219)
        cfg["max_value_print_option"] = max_value_print
    if sc.time_series:
        cfg["print_observation"] = repr(float(sc.print_observation))
        rc = sc.meta.get("obs_rc")
        if rc is None:
            rc = [divmod(int(i), sc.cols) for i in sc.obs_cells]
            rc = [(r - 1, c - 1) for r, c in rc]
        with open(P(f"{name}.obs"), "w") as f:
            f.write("%X-Location,Y-Location\n")
            for r, c in rc:
                x, y = xy(r, c)
                f.write(f"{x!r},{y!r}\n")
        cfg["observation_loc_file"] = P(f"{name}.obs")
    if sc.sources is not None and len(sc.sources["cells"]):
        s = sc.sources
        rcs = s.get("cells_rc") or [((int(i) // sc.cols) - 1, (int(i) % sc.cols) - 1) for i in s["cells"]]
        with open(P(f"{name}.src"), "w") as f:
            f.write("%X-Location,Y-Location\n")
            for r, c in rcs:
                x, y = xy(r, c)
                f.write(f"{x!r},{y!r}\n")
        with open(P(f"{name}.hyg"), "w") as f:
            f.write("% Time(hr), Discharge(cms)\n")
            for t, row in zip(s["times_h"], s["flows_rows"]):
                f.write(",".join([repr(float(t))] + [repr(float(v)) for v in row]) + "\n")
        cfg.update(num_sources=str(len(rcs)), src_loc_file=P(f"{name}.src"), hydrograph_filename=P(f"{name}.hyg"))
    if partitions > 0:
        cfg["header_filename"] = P(f"{name}.header")
    if sc.runoff is not None:
        r = sc.runoff
        if partitions > 0:
            rmap = P(f"{name}_rmap")
            _write_parts(rmap, ".rmap", r["zone"][1:-1, 1:-1], fmt, partitions, dtype=np.int32)
        else:
            rmap = P(f"{name}.rmap.{ext}")
            _write_raster(rmap, r["zone"][1:-1, 1:-1], fmt, dtype=np.int32)
        with open(P(f"{name}.roff"), "w") as f:
            f.write("% Time(hr), Rate(mm/hr)\n")
            for t, row in zip(r["times_h"], r["rates_mm_h"]):
                f.write(",".join([repr(float(t))] + [repr(float(v)) for v in np.atleast_1d(row)]) + "\n")
        cfg.update(num_runoffs=str(int(r["nzones"])), runoff_filename=P(f"{name}.roff"), runoff_map=rmap)
    segs = getattr(sc, "_segments", None)
    if segs:
        lines = ["% BC Type, X1, Y1, X2, Y2, BC"]
        for k, (bt, (r1, c1), (r2, c2), val) in enumerate(segs):
            x1, y1 = xy(r1, c1)
            x2, y2 = xy(r2, c2)
            if bt == 1:
                fn = f"{name}_bc{k}.txt"
                with open(P(fn), "w") as f:
                    f.write("% Time(hr), WSE(m)\n")
                    for t, v in val:
                        f.write(f"{float(t)!r},{float(v)!r}\n")
                tail = fn
            elif bt == 0:
                tail = "0"
            else:
                tail = repr(float(val))
            lines.append(f"{bt},{x1!r},{y1!r},{x2!r},{y2!r},{tail}")
        with open(P(f"{name}.extbc"), "w") as f:
            f.write("\n".join(lines) + "\n")
        cfg.update(num_extbc=str(len(segs)), extbc_file=P(f"{name}.extbc"), extbc_dir=os.path.abspath(directory))
    path = P(f"{name}.cfg")
    with open(path, "w") as f:
        for k, v in cfg.items():
            f.write(f"{k}={v}\n")
    return path
