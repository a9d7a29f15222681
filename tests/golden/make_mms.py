"""Generate tests/golden/mms_euler_16.npz: the manufactured solution of the reference's
2D Euler MMS smoke test, sampled where the oracle needs it (run from the repository
root; needs sympy).

The reference case (examples/eilmer/2D/manufactured-solution/sg/smoke-tests/,
case-euler.txt: case 1, ausmdv, x_order 2, 2x2 blocks, 16x16 cells on the unit square)
prescribes the steady fields of Roy, Nelson, Smith and Ober (2004), Appendix A, in its
analytic_solution.py (supersonic set, S = 1):

    phi(x, y) = phi0 + phix f(a_phix pi x / L) + phiy g(a_phiy pi y / L)   (+ xy term, zero here)

with sin/cos as written there for rho, u, v, p, and derives the source terms that make
them steady with sympy (make_lua_files.py): for the Euler case mu = k = 0,

    fmass = d(rho u)/dx + d(rho v)/dy
    fxmom = d(rho u u + p)/dx + d(rho u v)/dy
    fymom = d(rho v u)/dx + d(rho v v + p)/dy
    fe    = d(rho u et + p u)/dx + d(rho v et + p v)/dy,   et = p/(rho (gamma-1)) + (u^2+v^2)/2

with Rgas = 287, gamma = 1.4 (constants.txt).  The same derivation is done here with
sympy and evaluated in double precision at:
  centres   the 16 x 16 cell centres ((i + 1/2)/16, (j + 1/2)/16): source terms and the
            exact density the norms are taken against (ref-soln-template.lua);
  west      the two ghost layers beyond x = 0: x = -1/32, -3/32 at the row centres;
  south     the two ghost layers beyond y = 0: y = -1/32, -3/32 at the column centres;
            ghost states are p, T = p/(rho Rgas), vel.x, vel.y, as udf-bc-template.lua
            returns them for UserDefinedGhostCell.
"""
import os

import numpy as np
import sympy as sp

HERE = os.path.dirname(os.path.abspath(__file__))

L = 1.0
RGAS, GAMMA = 287.0, 1.4
N = 16


def fields():
    x, y = sp.symbols("x y")
    pi = sp.pi
    rho0, rhox, rhoy, arhox, arhoy = 1.0, 0.15, -0.1, 1.0, 0.5
    u0, ux, uy, aux, auy = 800.0, 50.0, -30.0, 1.5, 0.6
    v0, vx, vy, avx, avy = 800.0, -75.0, 40.0, 0.5, 2.0 / 3
    p0, px, py, apx, apy = 1.0e5, 0.2e5, 0.5e5, 2.0, 1.0
    rho = rho0 + rhox * sp.sin(arhox * pi * x / L) + rhoy * sp.cos(arhoy * pi * y / L)
    u = u0 + ux * sp.sin(aux * pi * x / L) + uy * sp.cos(auy * pi * y / L)
    v = v0 + vx * sp.cos(avx * pi * x / L) + vy * sp.sin(avy * pi * y / L)
    p = p0 + px * sp.cos(apx * pi * x / L) + py * sp.sin(apy * pi * y / L)
    et = p / rho / (GAMMA - 1) + u * u / 2 + v * v / 2
    fmass = sp.diff(rho * u, x) + sp.diff(rho * v, y)
    fxmom = sp.diff(rho * u * u + p, x) + sp.diff(rho * u * v, y)
    fymom = sp.diff(rho * v * u, x) + sp.diff(rho * v * v + p, y)
    fe = sp.diff(rho * u * et + p * u, x) + sp.diff(rho * v * et + p * v, y)
    f = lambda e: sp.lambdify((x, y), e, "numpy")
    return dict(rho=f(rho), u=f(u), v=f(v), p=f(p), fmass=f(fmass), fxmom=f(fxmom), fymom=f(fymom), fe=f(fe))


def sample(F, X, Y):
    X, Y = np.asarray(X, float), np.asarray(Y, float)
    one = np.ones_like(X)
    return {k: fn(X, Y) * one for k, fn in F.items()}


def main():
    F = fields()
    c = (np.arange(N) + 0.5) / N
    X, Y = np.meshgrid(c, c)            # [j][i]
    cen = sample(F, X, Y)
    g = np.array([-0.5, -1.5]) / N      # ghost-layer centres beyond the minus faces
    west = sample(F, g[:, None] * np.ones((2, N)), np.ones((2, 1)) * c[None, :])    # [layer][j]
    south = sample(F, np.ones((2, 1)) * c[None, :], g[:, None] * np.ones((2, N)))   # [layer][i]

    def ghost(s):
        return np.stack([s["p"], s["p"] / (s["rho"] * RGAS), s["u"], s["v"], np.zeros_like(s["p"])], axis=-1)

    out = dict(
        rho_exact=cen["rho"],
        Q=np.stack([cen["fmass"], cen["fxmom"], cen["fymom"], np.zeros_like(cen["fe"]), cen["fe"]]),
        ghost_west=ghost(west), ghost_south=ghost(south),
        R=np.float64(RGAS), gamma=np.float64(GAMMA))
    np.savez_compressed(os.path.join(HERE, "mms_euler_16.npz"), **out)


if __name__ == "__main__":
    main()
