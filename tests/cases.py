"""Seeded problem definitions shared by the parity tests, smoke() and bench.py.

Each case is built identically on the CPU oracle (oracle/oracle.py) and on the
CUDA library (gdfv.Simulation), so the two can be compared cell by cell.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "gdtk-rmhd_b200")
if PKG not in sys.path:
    sys.path.insert(0, PKG)

R_AIR_CHICKEN = 287.1
R_AIR_EILMER = 8.31451 / 28.96e-3   # ideal-air-gas-model.lua via species-database/air.lua
R_HE = 8.31451 / 4.0026020e-3       # species-database/He.lua


class Case:
    """A problem: config, gas, blocks (dims, spacing, origin, BCs) and initial rhoT fields."""

    def __init__(self, name, config, R, gamma):
        self.name = name
        self.config = dict(config)
        self.R = R
        self.gamma = gamma
        self.blocks = []

    def add_block(self, n, d, origin, bcs, rho, vel, T, B=None, psi=None, vertices=None):
        """vertices: (xv, yv, zv) of a graded (rectilinear) block; d and origin are then
        those of its first cell."""
        self.blocks.append(dict(n=n, d=d, origin=origin, bcs=bcs, rho=rho, vel=vel, T=T, B=B, psi=psi,
                                vertices=vertices))
        return len(self.blocks) - 1

    @property
    def mhd(self):
        return bool(self.config.get("MHD", False))

    @property
    def nq(self):
        return 10 if self.mhd else 5

    def total_cells(self):
        return sum(int(np.prod(b["n"])) for b in self.blocks)


def _noisy_rho(rng, rho, shape, amp=0.01):
    return rho * (1.0 + amp * rng.standard_normal(shape))


def c1_shock_box(n=32, seed=1234):
    """32^3 cells of 1 mm, ideal air (R=287.1, gamma=1.4), ausmdv, PC, CFL 0.5;
    x < 16 mm: p=1e5 T=300, else p=1e4 T=300; u=0; density noise 1%; extrapolate BCs."""
    c = Case("c1", dict(flux_calculator="ausmdv"), R_AIR_CHICKEN, 1.4)
    rng = np.random.default_rng(seed)
    dx = 1.0e-3
    x = (np.arange(n) + 0.5) * dx
    p = np.where(x < 0.5 * n * dx, 1.0e5, 1.0e4)
    T = 300.0
    rho0 = np.broadcast_to(p / (R_AIR_CHICKEN * T), (n, n, n))
    rho = _noisy_rho(rng, rho0, (n, n, n))
    bcs = {f: ("outflow_simple_extrapolate", dict(x_order=0)) for f in
           ("west", "east", "south", "north", "bottom", "top")}
    c.add_block((n, n, n), (dx, dx, dx), (0, 0, 0), bcs, rho, (0.0, 0.0, 0.0), T)
    return c


def inflow_state_m3():
    """M=3 ideal air, p=5e3 Pa, T=220 K."""
    T = 220.0
    a = np.sqrt(1.4 * R_AIR_CHICKEN * T)
    return dict(p=5.0e3, T=T, vel=(3.0 * a, 0.0, 0.0))


def c2_inflow_box(n=(256, 256, 256), flux="ausmdv", seed=4321, precision="fp64", noise_all=False, d=1e-3):
    """Single block, M=3 inflow on x-min, extrapolate outflow on x-max, slip walls
    on y and z faces, inflow state everywhere plus 1% density noise (dx = 1 mm).
    noise_all: also 1% noise on T and on the velocity components, so that no
    reconstructed field is exactly uniform (limiters away from their kinks)."""
    c = Case("c2", dict(flux_calculator=flux, flux_precision=precision), R_AIR_CHICKEN, 1.4)
    rng = np.random.default_rng(seed)
    inf = inflow_state_m3()
    nic, njc, nkc = n
    shp = (nkc, njc, nic)
    rho_inf = inf["p"] / (R_AIR_CHICKEN * inf["T"])
    rho = _noisy_rho(rng, rho_inf, shp)
    T, vel = inf["T"], inf["vel"]
    if noise_all:
        T = inf["T"] * (1.0 + 0.01 * rng.standard_normal(shp))
        u = inf["vel"][0]
        vel = (u * (1.0 + 0.01 * rng.standard_normal(shp)), 0.01 * u * rng.standard_normal(shp),
               0.01 * u * rng.standard_normal(shp))
    bcs = {"west": ("inflow_supersonic", dict(inflow=inf)),
           "east": ("outflow_simple_extrapolate", dict(x_order=0)),
           "south": ("wall_with_slip", {}), "north": ("wall_with_slip", {}),
           "bottom": ("wall_with_slip", {}), "top": ("wall_with_slip", {})}
    c.add_block(n, (d, d, d), (0, 0, 0), bcs, rho, vel, T)
    return c


def multiblock_lattice(nb=(2, 2, 2), sizes=(16, 24, 32), seed=77, flux="ausmdv", precision="fp64", choices=None):
    """Blocks on an nb lattice joined by full-face exchange; per-axis sizes drawn
    from `sizes` by seed (chicken's lattice model: faces always match).  M=3 inflow
    on the outer x-min faces, extrapolate on x-max, slip walls elsewhere."""
    c = Case("multiblock", dict(flux_calculator=flux, flux_precision=precision), R_AIR_CHICKEN, 1.4)
    rng = np.random.default_rng(seed)
    sz = [rng.choice(sizes, nb[a]) if choices is None else np.array(choices[a]) for a in range(3)]
    inf = inflow_state_m3()
    rho_inf = inf["p"] / (R_AIR_CHICKEN * inf["T"])
    dx = 1e-3
    idx = {}
    for bk in range(nb[2]):
        for bj in range(nb[1]):
            for bi in range(nb[0]):
                idx[(bi, bj, bk)] = len(idx)
    for bk in range(nb[2]):
        for bj in range(nb[1]):
            for bi in range(nb[0]):
                n = (int(sz[0][bi]), int(sz[1][bj]), int(sz[2][bk]))
                origin = (dx * sum(sz[0][:bi]), dx * sum(sz[1][:bj]), dx * sum(sz[2][:bk]))
                bcs = {}
                pos = (bi, bj, bk)
                for a, (fm, fp) in enumerate((("west", "east"), ("south", "north"), ("bottom", "top"))):
                    lo = list(pos); lo[a] -= 1
                    hi = list(pos); hi[a] += 1
                    if pos[a] > 0:
                        bcs[fm] = ("exchange_over_full_face", dict(other=idx[tuple(lo)], other_face=fp))
                    elif a == 0:
                        bcs[fm] = ("inflow_supersonic", dict(inflow=inf))
                    else:
                        bcs[fm] = ("wall_with_slip", {})
                    if pos[a] < nb[a] - 1:
                        bcs[fp] = ("exchange_over_full_face", dict(other=idx[tuple(hi)], other_face=fm))
                    elif a == 0:
                        bcs[fp] = ("outflow_simple_extrapolate", dict(x_order=0))
                    else:
                        bcs[fp] = ("wall_with_slip", {})
                rho = _noisy_rho(rng, rho_inf, (n[2], n[1], n[0]))
                c.add_block(n, (dx, dx, dx), origin, bcs, rho, inf["vel"], inf["T"])
    return c


def sod_eilmer(nic=100):
    """examples/eilmer/3D/sod-shock-tube/sg/sod.lua: 1 m x 0.1 m x 0.1 m, 100x2x2,
    ideal air, ausmdv, slip walls everywhere (the default BC), max_time 0.6 ms."""
    c = Case("sod", dict(flux_calculator="ausmdv"), R_AIR_EILMER, 1.4)
    dx = 1.0 / nic
    x = (np.arange(nic) + 0.5) * dx
    p = np.where(x < 0.5, 1.0e5, 1.0e4)
    T = np.where(x < 0.5, 348.4, 278.8)
    rho = np.broadcast_to(p / (R_AIR_EILMER * T), (2, 2, nic))
    T3 = np.broadcast_to(T, (2, 2, nic))
    c.add_block((nic, 2, 2), (dx, 0.05, 0.05), (0, 0, 0), {}, rho, (0.0, 0.0, 0.0), T3)
    return c


def mhd_shock_tube(N=512, noise=0.0, seed=5):
    """examples/eilmer/2D/MHDShockTube/MHDShockTube.lua (Dai & Woodward problem 3):
    2D, two 256x3 blocks, hlle MHD without cleaning, stringent CFL, ideal He.
    noise > 0 multiplies rho, T and every velocity and B component cell by cell by
    (1 + noise * N(0, 1)): a state off the piecewise residual's switch points, where
    the uniform regions would otherwise meet the disturbed ones one ulp apart."""
    rng = np.random.default_rng(seed)
    c = Case("mhd_tube", dict(flux_calculator="hlle", MHD=1, divergence_cleaning=0, dimensions=2,
                              stringent_cfl=1, cfl_value=0.5, dt_init=1e-5), R_HE, 5.0 / 3.0)
    nic, njc = N // 2, 3
    dx, dy = 0.5 / nic, 0.5 / 3
    Bx = 5 / np.sqrt(4 * np.pi)
    s4 = 1 / np.sqrt(4 * np.pi)
    for side in (0, 1):
        vel = (11.7106, -0.312542, -0.495260) if side == 0 else (-11.7106, 0.312542, -0.495260)
        B = (Bx, s4, -s4) if side == 0 else (Bx, s4, s4)
        rho, p = 1.0, 1.0
        T = p / (rho * R_HE)
        if noise > 0.0:
            shp = (1, njc, nic)
            jit = lambda x: x * (1.0 + noise * rng.standard_normal(shp))
            rho, T = jit(rho), jit(T)
            vel, B = tuple(jit(x) for x in vel), tuple(jit(x) for x in B)
        bcs = {"north": ("exchange_over_full_face", dict(other=side, other_face="south")),
               "south": ("exchange_over_full_face", dict(other=side, other_face="north"))}
        if side == 0:
            bcs["west"] = ("outflow_simple_extrapolate", dict(x_order=1))
            bcs["east"] = ("exchange_over_full_face", dict(other=1, other_face="west"))
        else:
            bcs["east"] = ("outflow_simple_extrapolate", dict(x_order=1))
            bcs["west"] = ("exchange_over_full_face", dict(other=0, other_face="east"))
        c.add_block((nic, njc, 1), (dx, dy, 1.0), (0.5 * side, 0, 0), bcs, rho, vel, T, B=B)
    return c


def orszag_tang(n=(512, 512, 4), seed=99, precision="fp64", cleaning=True):
    """Ideal MHD Orszag-Tang vortex on [0,1]^2 x [0, 4/512], periodic on all faces,
    gamma=5/3, rho=25/(36 pi), p=5/(12 pi), v=(-sin 2 pi y, sin 2 pi x, 0),
    B=(-sin 2 pi y, sin 4 pi x, 0)/sqrt(4 pi), 1% density noise; hlle with GLM."""
    R = 1.0
    c = Case("orszag_tang", dict(flux_calculator="hlle", MHD=1, divergence_cleaning=int(cleaning),
                                 stringent_cfl=1, flux_precision=precision, dt_init=1e-3, dt_max=1e-3),
             R, 5.0 / 3.0)
    nic, njc, nkc = n
    dx, dy = 1.0 / nic, 1.0 / njc
    dz = dx
    rng = np.random.default_rng(seed)
    x = (np.arange(nic) + 0.5) * dx
    y = (np.arange(njc) + 0.5) * dy
    X = np.broadcast_to(x[None, None, :], (nkc, njc, nic))
    Y = np.broadcast_to(y[None, :, None], (nkc, njc, nic))
    rho0 = 25.0 / (36.0 * np.pi)
    p0 = 5.0 / (12.0 * np.pi)
    rho = _noisy_rho(rng, rho0, (nkc, njc, nic))
    T = p0 / (rho * R)
    vel = (-np.sin(2 * np.pi * Y), np.sin(2 * np.pi * X), np.zeros_like(X))
    B = (-np.sin(2 * np.pi * Y) / np.sqrt(4 * np.pi), np.sin(4 * np.pi * X) / np.sqrt(4 * np.pi), np.zeros_like(X))
    bcs = {"west": ("exchange_over_full_face", dict(other=0, other_face="east")),
           "east": ("exchange_over_full_face", dict(other=0, other_face="west")),
           "south": ("exchange_over_full_face", dict(other=0, other_face="north")),
           "north": ("exchange_over_full_face", dict(other=0, other_face="south")),
           "bottom": ("exchange_over_full_face", dict(other=0, other_face="top")),
           "top": ("exchange_over_full_face", dict(other=0, other_face="bottom"))}
    c.add_block(n, (dx, dy, dz), (0, 0, 0), bcs, rho, vel, T, B=B)
    return c


def mhd_slip_dipole(n=(64, 48, 4), seed=31, precision="fp64"):
    """Ideal MHD (hlle + GLM, gamma 5/3, R 1) in x in [-0.5, 0.5], y in [0.45, 1.2],
    z in [0, 4/64]: slip walls on the y and z faces, periodic in x.  Every wall ghost
    with |x| < 0.4136 takes the dipole field of internal_copy_then_reflect.d:140-143
    (the y-min wall sits at r >= 0.45 from the dipole, so the field stays moderate).
    Uniform rho 1, p 1 with 1% density noise, v = (0.2, 0.05 sin 2 pi x, 0),
    B = (0.1, 0.05 cos 2 pi x, 0.02)."""
    R = 1.0
    c = Case("mhd_slip_dipole", dict(flux_calculator="hlle", MHD=1, divergence_cleaning=1, stringent_cfl=1,
                                     flux_precision=precision, dt_init=2e-3, dt_max=5e-3), R, 5.0 / 3.0)
    nic, njc, nkc = n
    dx, dy = 1.0 / nic, 0.75 / njc
    dz = dx
    x0, y0 = -0.5, 0.45
    rng = np.random.default_rng(seed)
    x = x0 + (np.arange(nic) + 0.5) * dx
    X = np.broadcast_to(x[None, None, :], (nkc, njc, nic))
    rho = _noisy_rho(rng, 1.0, (nkc, njc, nic))
    T = 1.0 / (rho * R)
    vel = (np.full(X.shape, 0.2), 0.05 * np.sin(2 * np.pi * X), np.zeros(X.shape))
    B = (np.full(X.shape, 0.1), 0.05 * np.cos(2 * np.pi * X), np.full(X.shape, 0.02))
    bcs = {"west": ("exchange_over_full_face", dict(other=0, other_face="east")),
           "east": ("exchange_over_full_face", dict(other=0, other_face="west")),
           "south": ("wall_with_slip", {}), "north": ("wall_with_slip", {}),
           "bottom": ("wall_with_slip", {}), "top": ("wall_with_slip", {})}
    c.add_block(n, (dx, dy, dz), (x0, y0, 0.0), bcs, rho, vel, T, B=B)
    return c


def stretched(n, d0, ratio, x0=0.0):
    """n+1 vertex coordinates from x0 with first cell d0 and cell-to-cell growth ratio."""
    return x0 + np.concatenate([[0.0], np.cumsum(d0 * ratio ** np.arange(n))])


def graded_inflow_box(n=(40, 28, 20), seed=17, precision="fp64", flux="ausmdv", uniform=False):
    """The M=3 inflow box on a stretched rectilinear grid: cells growing by 3% along x from
    0.8 mm, shrinking by 2% along y from 1.2 mm, 1 mm along z; inflow on x-min, extrapolation on x-max, slip
    walls on y and z, 1% density noise.  uniform=True: 1/1024 m everywhere (vertices i/1024
    are exact, so the cell lengths are too), built as a graded block."""
    c = Case("graded_box", dict(flux_calculator=flux, flux_precision=precision), R_AIR_CHICKEN, 1.4)
    rng = np.random.default_rng(seed)
    inf = inflow_state_m3()
    nic, njc, nkc = n
    if uniform:
        verts = tuple(np.arange(m + 1) / 1024.0 for m in n)
    else:
        verts = (stretched(nic, 0.8e-3, 1.03), stretched(njc, 1.2e-3, 0.98), np.arange(nkc + 1) * 1e-3)
    rho = _noisy_rho(rng, inf["p"] / (R_AIR_CHICKEN * inf["T"]), (nkc, njc, nic))
    bcs = {"west": ("inflow_supersonic", dict(inflow=inf)),
           "east": ("outflow_simple_extrapolate", dict(x_order=0)),
           "south": ("wall_with_slip", {}), "north": ("wall_with_slip", {}),
           "bottom": ("wall_with_slip", {}), "top": ("wall_with_slip", {})}
    d = tuple(float(v[1] - v[0]) for v in verts)
    c.add_block(n, d, tuple(float(v[0]) for v in verts), bcs, rho, inf["vel"], inf["T"], vertices=verts)
    return c


def graded_lattice(seed=23, precision="fp64"):
    """2 x 2 x 1 blocks of stretched grids joined by full-face exchange (the ghost cells
    across an exchange take the partner's cell lengths), a shock-box state (x < mid:
    p 1e5, else 1e4; T 300) with 1% density noise, extrapolation on the outer x faces,
    slip walls elsewhere."""
    c = Case("graded_lattice", dict(flux_calculator="ausmdv", flux_precision=precision), R_AIR_CHICKEN, 1.4)
    rng = np.random.default_rng(seed)
    xs = [stretched(20, 1.0e-3, 1.04), None]
    xs[1] = stretched(24, 0.7e-3, 0.99, x0=xs[0][-1])
    ys = [stretched(18, 1.1e-3, 0.97), None]
    ys[1] = stretched(16, 0.9e-3, 1.05, x0=ys[0][-1])
    zv = stretched(12, 1.0e-3, 1.02)
    xmid = 0.5 * (xs[0][0] + xs[1][-1])
    idx = {(bi, bj): bi + 2 * bj for bj in range(2) for bi in range(2)}
    for bj in range(2):
        for bi in range(2):
            xv, yv = xs[bi], ys[bj]
            n = (len(xv) - 1, len(yv) - 1, len(zv) - 1)
            xc = 0.5 * (xv[1:] + xv[:-1])
            p = np.where(xc < xmid, 1.0e5, 1.0e4)
            rho = _noisy_rho(rng, np.broadcast_to(p / (R_AIR_CHICKEN * 300.0), (n[2], n[1], n[0])), (n[2], n[1], n[0]))
            bcs = {}
            bcs["west"] = ("exchange_over_full_face", dict(other=idx[(0, bj)], other_face="east")) if bi == 1 else \
                ("outflow_simple_extrapolate", dict(x_order=0))
            bcs["east"] = ("exchange_over_full_face", dict(other=idx[(1, bj)], other_face="west")) if bi == 0 else \
                ("outflow_simple_extrapolate", dict(x_order=0))
            if bj == 1:
                bcs["south"] = ("exchange_over_full_face", dict(other=idx[(bi, 0)], other_face="north"))
            else:
                bcs["north"] = ("exchange_over_full_face", dict(other=idx[(bi, 1)], other_face="south"))
            d = (float(xv[1] - xv[0]), float(yv[1] - yv[0]), float(zv[1] - zv[0]))
            c.add_block(n, d, (float(xv[0]), float(yv[0]), float(zv[0])), bcs, rho, (0.0, 0.0, 0.0), 300.0,
                        vertices=(xv, yv, zv))
    return c


R90 = (0.0, -1.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0)    # +90 degrees about z: (x, y) -> (-y, x)
R270 = (0.0, 1.0, 0.0, -1.0, 0.0, 0.0, 0.0, 0.0, 1.0)   # -90 degrees about z


def exchange_pair(orientation, precision="fp64", seed=41, graded=False):
    """Two blocks joined by a full-face exchange between block 0's east face and block
    1's north face, both ways with the same orientation 0..3 (the map of one direction
    is then the inverse of the other's; full_face_copy.d:680-1409).  The faces are 16 x 16
    cells, so every orientation fits.  The library's blocks are axis-aligned, so the join
    is not geometric: the case tests the ghost map on a flow that stays valid, a
    two-state box (p 1e5 / 3e4, T 300 / 350) with 1% noise on density and on all three
    velocity components about (40, -25, 30) m/s, extrapolation on the other faces.
    graded: block 1 stretched along j (the normal of its exchange face), so the ghosts
    of block 0's east face take block 1's j lengths."""
    c = Case(f"exchange_pair_o{orientation}", dict(flux_calculator="ausmdv", flux_precision=precision),
             R_AIR_CHICKEN, 1.4)
    rng = np.random.default_rng(seed + orientation)
    d = 1.0e-3
    ext = {f: ("outflow_simple_extrapolate", dict(x_order=0)) for f in
           ("west", "east", "south", "north", "bottom", "top")}
    for blk, (n, origin, p, T, face, other_face) in enumerate(
            [((20, 16, 16), (0.0, 0.0, 0.0), 1.0e5, 300.0, "east", "north"),
             ((16, 12, 16), (0.03, 0.0, 0.0), 3.0e4, 350.0, "north", "east")]):
        shp = (n[2], n[1], n[0])
        rho = _noisy_rho(rng, p / (R_AIR_CHICKEN * T), shp)
        vel = tuple(v * (1.0 + 0.01 * rng.standard_normal(shp)) for v in (40.0, -25.0, 30.0))
        bcs = dict(ext)
        bcs[face] = ("exchange_over_full_face", dict(other=1 - blk, other_face=other_face, orientation=orientation))
        vertices = None
        if graded and blk == 1:
            vertices = (origin[0] + d * np.arange(n[0] + 1), stretched(n[1], 0.8e-3, 1.05),
                        d * np.arange(n[2] + 1))
        c.add_block(n, (d, d, d), origin, bcs, rho, vel, T, vertices=vertices)
    return c


def quarter_rotational(n=(24, 24, 4), precision="fp64", mhd=False, seed=None):
    """The quadrant x, y >= 0 of a flow with four-fold rotational symmetry about the z
    axis: the ghosts beyond x = 0 copy the cells inside y = 0 turned by +90 degrees, and
    the ghosts beyond y = 0 the cells inside x = 0 turned by -90 degrees (ExchangeBC_FullFace
    west <-> south with reorient_vector_quantities; the vectors turn with the cells).
    Euler: air, a density and pressure bump of 30% and a swirl of up to 80 m/s about the
    axis, slip walls at x = L, y = L and on the z faces.  mhd: hlle + GLM (gamma 5/3, R 1)
    with an azimuthal magnetic field on top of a uniform B_z, extrapolation at x = L and
    y = L and periodic in z (this fork's MHD slip-wall ghosts carry a dipole field for
    |x| < 0.4136, internal_copy_then_reflect.d:140-143, which walls through the axis would
    meet at its singular point).  seed: 1% density noise (breaks the symmetry; the parity
    tests), None: the smooth field."""
    nic, njc, nkc = n
    if mhd:
        c = Case("quarter_rotational_mhd", dict(flux_calculator="hlle", MHD=1, divergence_cleaning=1, stringent_cfl=1,
                                                flux_precision=precision, dt_init=2e-3, dt_max=1e-2), 1.0, 5.0 / 3.0)
        L = 1.0
    else:
        c = Case("quarter_rotational", dict(flux_calculator="ausmdv", flux_precision=precision), R_AIR_CHICKEN, 1.4)
        L = 0.024
    dx = L / nic
    x = (np.arange(nic) + 0.5) * dx
    y = (np.arange(njc) + 0.5) * dx
    X = np.broadcast_to(x[None, None, :], (nkc, njc, nic))
    Y = np.broadcast_to(y[None, :, None], (nkc, njc, nic))
    g = np.exp(-(X * X + Y * Y) / (0.4 * L) ** 2)
    if mhd:
        rho = 1.0 + 0.3 * g
        T = (1.0 + 0.3 * g) / rho
        w = 0.5 * g / L
        B = (-0.2 * g * Y / L, 0.2 * g * X / L, np.full(X.shape, 0.1))
    else:
        rho = 1.2 * (1.0 + 0.3 * g)
        T = 300.0 * (1.0 + 0.1 * g)
        w = 80.0 * g / L
        B = None
    if seed is not None:
        rho = _noisy_rho(np.random.default_rng(seed), rho, rho.shape)
    vel = (-w * Y, w * X, np.zeros(X.shape))
    bcs = {"west": ("exchange_over_full_face", dict(other=0, other_face="south", Rmatrix=R90)),
           "south": ("exchange_over_full_face", dict(other=0, other_face="west", Rmatrix=R270)),
           "east": ("wall_with_slip", {}), "north": ("wall_with_slip", {}),
           "bottom": ("wall_with_slip", {}), "top": ("wall_with_slip", {})}
    if mhd:
        bcs.update(east=("outflow_simple_extrapolate", dict(x_order=0)),
                   north=("outflow_simple_extrapolate", dict(x_order=0)),
                   bottom=("exchange_over_full_face", dict(other=0, other_face="top")),
                   top=("exchange_over_full_face", dict(other=0, other_face="bottom")))
    c.add_block(n, (dx, dx, dx), (0.0, 0.0, 0.0), bcs, rho, vel, T, B=B)
    return c


def full_rotational(n=(24, 24, 4)):
    """quarter_rotational's Euler flow (smooth) on the whole square [-L, L]^2 as one block,
    slip walls all round: its quadrant x, y >= 0 is the quarter case."""
    nic, njc, nkc = n
    c = Case("full_rotational", dict(flux_calculator="ausmdv"), R_AIR_CHICKEN, 1.4)
    L = 0.024
    dx = L / nic
    x = (np.arange(2 * nic) + 0.5) * dx - L
    y = (np.arange(2 * njc) + 0.5) * dx - L
    X = np.broadcast_to(x[None, None, :], (nkc, 2 * njc, 2 * nic))
    Y = np.broadcast_to(y[None, :, None], (nkc, 2 * njc, 2 * nic))
    g = np.exp(-(X * X + Y * Y) / (0.4 * L) ** 2)
    rho = 1.2 * (1.0 + 0.3 * g)
    T = 300.0 * (1.0 + 0.1 * g)
    w = 80.0 * g / L
    bcs = {f: ("wall_with_slip", {}) for f in ("west", "east", "south", "north", "bottom", "top")}
    c.add_block((2 * nic, 2 * njc, nkc), (dx, dx, dx), (-L, -L, 0.0), bcs, rho, (-w * Y, w * X, np.zeros(X.shape)), T)
    return c


# ---------------------------------------------------------------- builders
_ORACLE_BC = {"wall_with_slip": "wall_with_slip", "outflow_simple_extrapolate": "extrapolate",
              "inflow_supersonic": "inflow_supersonic", "exchange_over_full_face": "exchange",
              "outflow_fixed_p": "fixed_p", "outflow_fixed_p_and_t": "fixed_pt", "outflow_simple_flux": "simple_flux"}


def build_oracle(case):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import OracleSim
    # the oracle takes the flow-state limits under their GlobalConfig field names
    cfg = {k.replace("flowstate_limits_", ""): v for k, v in case.config.items() if k != "flux_precision"}
    s = OracleSim(R=case.R, gamma=case.gamma, **cfg)
    for b in case.blocks:
        if b.get("vertices") is not None:
            s.add_block_graded(*b["vertices"])
        else:
            s.add_block(*b["n"], *b["d"], *b["origin"])
    for bi, b in enumerate(case.blocks):
        for face, (kind, kw) in b["bcs"].items():
            inflow = kw.get("inflow")
            if kind in ("outflow_fixed_p", "outflow_fixed_p_and_t"):
                inflow = dict(p=kw["p_outside"], T=kw.get("T_outside", 0.0))
            if kind == "exchange_over_full_face":
                s.set_exchange(bi, face, kw["other"], kw["other_face"], kw.get("orientation", 0), kw.get("Rmatrix"))
                continue
            s.set_bc(bi, face, _ORACLE_BC[kind], x_order=kw.get("x_order", 0),
                     other_block=kw.get("other", -1), other_face=kw.get("other_face", -1), inflow=inflow)
        s.set_flow_rhoT(bi, b["rho"], b["vel"], b["T"], B=b["B"])
    s.init()
    return s


def build_gpu(case, **extra_config):
    import gdfv
    cfg = gdfv.Config(**{**case.config, **extra_config})
    sim = gdfv.Simulation(cfg, gas=gdfv.IdealGas(R=case.R, gamma=case.gamma))
    for b in case.blocks:
        if b.get("vertices") is not None:
            sim.add_block_graded(*b["vertices"])
        else:
            sim.add_block(*b["n"], *b["d"], *b["origin"])
    for bi, b in enumerate(case.blocks):
        for face, (kind, kw) in b["bcs"].items():
            if kind == "wall_with_slip":
                bc = gdfv.WallBC_WithSlip()
            elif kind == "outflow_simple_extrapolate":
                bc = gdfv.OutFlowBC_SimpleExtrapolate(xOrder=kw.get("x_order", 0))
            elif kind == "outflow_simple_flux":
                bc = gdfv.OutFlowBC_SimpleFlux()
            elif kind == "outflow_fixed_p":
                bc = gdfv.OutFlowBC_FixedP(kw["p_outside"])
            elif kind == "outflow_fixed_p_and_t":
                bc = gdfv.OutFlowBC_FixedPT(kw["p_outside"], kw["T_outside"])
            elif kind == "inflow_supersonic":
                inf = kw["inflow"]
                bc = gdfv.InFlowBC_Supersonic(gdfv.FlowState(p=inf["p"], T=inf["T"], velx=inf["vel"][0],
                                                             vely=inf["vel"][1], velz=inf["vel"][2]))
            elif kw.get("Rmatrix") is not None:
                bc = gdfv.ExchangeBC_FullFace(kw["other"], kw["other_face"], orientation=kw.get("orientation", 0),
                                              reorient_vector_quantities=True, Rmatrix=kw["Rmatrix"])
            else:
                bc = gdfv.ExchangeBC_FullFace(kw["other"], kw["other_face"], orientation=kw.get("orientation", 0))
            sim.set_bc(bi, face, bc)
    sim.prepare()
    for bi, b in enumerate(case.blocks):
        sim.set_flow_rhoT(bi, b["rho"], b["vel"], b["T"], B=b["B"])
    return sim


def build_pair(case, **extra_config):
    """Oracle and GPU simulation started from the same conserved state: the oracle
    encodes the rhoT initial state (e4/fvcell.d:511-583), both sides then decode
    that U0, so the comparison starts from identical inputs."""
    orc = build_oracle(case)
    sim = build_gpu(case, **extra_config)
    for b in range(len(case.blocks)):
        U0 = orc.get_U(b)
        assert orc.set_U(b, U0) == 0
        sim.set_conserved(b, U0)
    return orc, sim


def rel_err_per_cell(x, ref):
    """max over cells of |x - ref| / max(|ref|, scale), scale = max |ref| of the variable
    times 1e-3 (a floor for variables that pass through zero, e.g. momentum)."""
    scale = np.max(np.abs(ref)) * 1e-3 + 1e-300
    return float(np.max(np.abs(x - ref) / np.maximum(np.abs(ref), scale)))


def cell_errors(U, Uref, mhd):
    """Per-cell relative errors of the conserved vector, by group:
    mass and total energy per cell; momentum and B as vectors per cell (|dm|/|m|),
    with a floor of 1e-3 of the field maximum of the group's magnitude for cells
    where it passes through zero; psi likewise.  Returns {group: max over cells}."""
    out = {}

    def vec(a, b):
        d = np.sqrt(np.sum((a - b) ** 2, axis=0))
        m = np.sqrt(np.sum(b ** 2, axis=0))
        floor = 1e-3 * np.max(m) + 1e-300
        return float(np.max(d / np.maximum(m, floor)))

    out["mass"] = float(np.max(np.abs(U[0] - Uref[0]) / np.abs(Uref[0])))
    out["momentum"] = vec(U[1:4], Uref[1:4])
    out["energy"] = float(np.max(np.abs(U[4] - Uref[4]) / np.abs(Uref[4])))
    if mhd:
        out["B"] = vec(U[5:8], Uref[5:8])
        out["psi"] = vec(U[8:9], Uref[8:9])
    return out


def rel_l2(x, ref):
    return float(np.linalg.norm(x - ref) / (np.linalg.norm(ref) + 1e-300))
