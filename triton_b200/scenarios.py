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


def watershed(n=8192, dx=10.0, seed=1234, duration=6 * 3600.0, rain_mm_h=50.0, rain_hours=1.0,
              manning_median=0.035, manning_sigma=0.3, relief=300.0, valley_depth=40.0, peak_flow=500.0,
              nsrc=3, print_interval=None):
    """Fractal watershed: value-noise DEM rescaled to 0..relief m with a carved
    meandering valley draining to the southern (lowest) edge, log-normal
    Manning, `nsrc` triangular inflow hydrographs (0 -> peak at 2 h -> 0 at
    4 h), uniform rain for `rain_hours`, and an open (extbc type 0) outflow
    along the southern edge."""
    rng = np.random.default_rng(seed)
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
    mann = np.exp(np.log(manning_median) + manning_sigma * np.random.default_rng(rng.integers(1 << 31))
                  .standard_normal((n, n)))
    z = _walls(dem)
    n2 = _copy_ghosts(_pad(mann)) ** 2
    zero = np.zeros_like(z)
    # sources along the valley in the northern half
    src_rows = np.linspace(n * 0.1, n * 0.45, nsrc).astype(int)
    src_cols = (n / 2 + 0.15 * n * np.sin(2 * np.pi * src_rows / (0.6 * n))).astype(int)
    cells = ((src_rows + 1) * (n + 2) + src_cols + 1).astype(np.int32)
    times_h = np.array([0.0, 2.0, 4.0, 1000.0])
    flows = np.zeros((4, nsrc))
    flows[1, :] = peak_flow
    sources = dict(cells=cells, times=times_h * 3600.0, flows=flows.reshape(-1), times_h=times_h,
                   flows_rows=flows)
    # uniform rain: one zone, rows (h, mm/h): (0, rain), (rain_hours, 0), (duration_h, 0)
    rt_h = np.array([0.0, rain_hours, max(duration / 3600.0, rain_hours + 1.0)])
    rr_mm = np.array([rain_mm_h, 0.0, 0.0])
    runoff = dict(zone=np.zeros((n + 2, n + 2), dtype=np.int32), times=rt_h * 3600.0,
                  rates=rr_mm / 3600.0 * 0.001, nzones=1, times_h=rt_h, rates_mm_h=rr_mm[:, None])
    # open outflow along the southern edge (last interior row), type 0
    bc_cells = ((n) * (n + 2) + np.arange(1, n + 1)).astype(np.int32)
    extbc = dict(cells=bc_cells, types=np.zeros(n, np.int32), start=np.zeros(n, np.int32),
                 nrows=np.ones(n, np.int32), var1=np.zeros(1), var2=np.zeros(1),
                 segments=[(0, 0.0, dx * 0.5, n * dx - dx * 0.5, dx * 0.5, None)])
    pi = print_interval or duration
    return Scenario("watershed", dx, z, zero.copy(), zero.copy(), zero.copy(), n2, courant=0.5, hextra=0.001,
                    sim_duration=duration, print_interval=pi, runoff=runoff, sources=sources, extbc=extbc,
                    meta=dict(n=n, seed=seed))


def mixed(rows=37, cols=53, dx=5.0, seed=7, open_boundaries=0, friction=True, with_sources=True,
          with_runoff=True, with_extbc=True, duration=30.0, wet_fraction=0.5):
    """Small random case that drives every forcing path of the step: rough
    terrain with partly wet cells, friction, two sources sharing a cell,
    zoned runoff, external boundary cells of types 0-3 (two segments sharing
    a corner) and optional open boundaries."""
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
    Cp = C + 2
    if with_runoff:
        nz = 3
        zone = np.zeros((R + 2, C + 2), dtype=np.int32)
        zone[1:-1, 1:-1] = rng.integers(0, nz, (R, C))
        t = np.array([0.0, 4.0, 9.0, 15.0, 1e5])
        rates = (rng.random((nz, t.size)) * 40.0 - 5.0) / 3600.0 * 0.001  # includes small negative rates
        sc.runoff = dict(zone=zone, times=t, rates=rates.reshape(-1), nzones=nz)
    if with_sources:
        cells = np.array([(R // 3 + 1) * Cp + C // 4 + 1, (2 * R // 3 + 1) * Cp + C // 2 + 1,
                          (R // 3 + 1) * Cp + C // 4 + 1], dtype=np.int32)
        t = np.array([0.0, 5.0, 12.0, 20.0, 1e5])
        flows = rng.random((t.size, cells.size)) * 2.0
        sc.sources = dict(cells=cells, times=t, flows=flows.reshape(-1))
    if with_extbc:
        # east column: type 1 level series; north row: type 3 (Froude) from the
        # NE corner it shares with the east segment, then type 2 (normal
        # slope); west column: type 2; south row: type 0 (open copy)
        cells, types, start, nrows = [], [], [], []
        var1, var2 = [], []
        t1 = [0.0, 6.0, 14.0, 1e5]
        l1 = [6.0, 7.0, 6.5, 6.5]
        s1 = len(var1)
        var1 += t1
        var2 += l1
        for r in range(1, R + 1):
            cells.append(r * Cp + C); types.append(1); start.append(s1); nrows.append(len(t1))
        s3 = len(var1)
        var1 += [0.8]
        var2 += [0.8]
        for c in range(C, C // 2, -1):
            cells.append(1 * Cp + c); types.append(3); start.append(s3); nrows.append(1)
        s2 = len(var1)
        var1 += [0.002]
        var2 += [0.002]
        for c in range(C // 2, 0, -1):
            cells.append(1 * Cp + c); types.append(2); start.append(s2); nrows.append(1)
        for r in range(2, R + 1):
            cells.append(r * Cp + 1); types.append(2); start.append(s2); nrows.append(1)
        s0 = len(var1)
        var1 += [0.0]
        var2 += [0.0]
        for c in range(2, C):
            cells.append(R * Cp + c); types.append(0); start.append(s0); nrows.append(1)
        sc.extbc = dict(cells=np.array(cells, np.int32), types=np.array(types, np.int32),
                        start=np.array(start, np.int32), nrows=np.array(nrows, np.int32),
                        var1=np.array(var1), var2=np.array(var2))
    sc.obs_cells = np.array([(R // 2 + 1) * Cp + C // 2 + 1, (2 + 1) * Cp + 3, (R) * Cp + C], dtype=np.int32)
    return sc
