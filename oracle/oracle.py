"""ctypes front end of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY.  The oracle restates the Eilmer-4 explicit
structured-grid update on the CPU (see fv_oracle.hpp / fv_oracle.cpp for the
reference file:line of every function).  Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline leg may load it, and only as the checker.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

FLUX = {"ausmdv": 0, "hllc": 1, "hlle": 2}
SCHEME = {"euler": 0, "pc": 1, "predictor_corrector": 1, "tvd_rk3": 2}
BC = {"wall_with_slip": 0, "extrapolate": 1, "inflow_supersonic": 2, "exchange": 3, "fixed_p": 4, "fixed_pt": 5, "simple_flux": 6}
FACES = {"west": 0, "east": 1, "south": 2, "north": 3, "bottom": 4, "top": 5}


def build():
    """Compile liboracle.so in place (g++ with OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        L.orc_new.restype = ctypes.c_int
        L.orc_set_int.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
        L.orc_set_double.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_double]
        L.orc_add_block.argtypes = [ctypes.c_int] + [ctypes.c_int] * 3 + [ctypes.c_double] * 6
        L.orc_set_bc.argtypes = [ctypes.c_int] * 7 + [dp]
        L.orc_set_flow_rhoT.argtypes = [ctypes.c_int, ctypes.c_int, dp]
        L.orc_run.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double]
        L.orc_get_time.argtypes = [ctypes.c_int, dp, ctypes.POINTER(ctypes.c_int)]
        L.orc_get_U.argtypes = [ctypes.c_int, ctypes.c_int, dp]
        L.orc_set_U.argtypes = [ctypes.c_int, ctypes.c_int, dp]
        L.orc_get_flow.argtypes = [ctypes.c_int, ctypes.c_int, dp]
        L.orc_residual.argtypes = [ctypes.c_int, dp, dp]
        L.orc_jvp_complex.argtypes = [ctypes.c_int, dp, dp, ctypes.c_double, dp]
        L.orc_jvp_real.argtypes = [ctypes.c_int, dp, dp, ctypes.c_double, dp, dp]
        L.orc_face_flux.argtypes = [ctypes.c_int, ctypes.c_int, dp, ctypes.c_double, dp]
        L.orc_last_error.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
        L.orc_set_ghost_states.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]
        L.orc_set_source.argtypes = [ctypes.c_int, ctypes.c_int, dp]
        L.orc_add_block_graded.argtypes = [ctypes.c_int] * 4 + [dp] * 3
        L.orc_set_exchange.argtypes = [ctypes.c_int] * 6 + [dp]
        ip = ctypes.POINTER(ctypes.c_int)
        L.orc_exchange_source.argtypes = [ctypes.c_int] * 4 + [ip] * 4
        _LIB = L
    return _LIB


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class OracleSim:
    """One oracle simulation: a set of uniform Cartesian blocks."""

    INT_KEYS = {"dimensions", "MHD", "divergence_cleaning", "apply_limiter", "extrema_clipping",
                "apply_entropy_fix", "glm_reference_indexing", "stringent_cfl", "cfl_count",
                "max_attempts_for_step", "max_invalid_cells", "chicken_compat", "lmr_epsilon"}

    def __init__(self, **cfg):
        self.L = lib()
        self.h = self.L.orc_new()
        self.blocks = []
        self.mhd = bool(cfg.get("MHD", False))
        for k, v in cfg.items():
            self.set(k, v)

    def set(self, key, value):
        if key == "flux_calculator":
            rc = self.L.orc_set_int(self.h, b"flux_calculator", FLUX[value])
        elif key == "gasdynamic_update_scheme":
            rc = self.L.orc_set_int(self.h, b"update_scheme", SCHEME[value.replace("-", "_")])
        elif key == "van_albada_variant":   # "e4" (default) or "lmr"
            if value not in ("e4", "lmr"):
                raise KeyError(value)
            rc = self.L.orc_set_int(self.h, b"lmr_epsilon", int(value == "lmr"))
        elif key in self.INT_KEYS:
            rc = self.L.orc_set_int(self.h, key.encode(), int(value))
        else:
            rc = self.L.orc_set_double(self.h, key.encode(), float(value))
        if rc != 0:
            raise KeyError(key)

    @property
    def nq(self):
        return 10 if self.mhd else 5

    def add_block(self, nic, njc, nkc, dx, dy, dz, x0=0.0, y0=0.0, z0=0.0):
        b = self.L.orc_add_block(self.h, nic, njc, nkc, dx, dy, dz, x0, y0, z0)
        self.blocks.append((nic, njc, nkc))
        self.geometry = getattr(self, "geometry", []) + [((dx, dy, dz), (x0, y0, z0))]
        return b

    def add_block_graded(self, xv, yv, zv):
        """A rectilinear block from vertex coordinates along each axis (n+1 each)."""
        xv, yv, zv = (np.ascontiguousarray(v, dtype=np.float64) for v in (xv, yv, zv))
        n = (len(xv) - 1, len(yv) - 1, len(zv) - 1)
        b = self.L.orc_add_block_graded(self.h, *n, _p(xv), _p(yv), _p(zv))
        if b < 0:
            raise ValueError(self.last_error())
        self.blocks.append(n)
        self.geometry = getattr(self, "geometry", []) + [((xv[1] - xv[0], yv[1] - yv[0], zv[1] - zv[0]),
                                                          (xv[0], yv[0], zv[0]))]
        return b

    def ghost_positions(self, blk, face):
        """Centres of the two ghost layers beyond a face, [layer][q][p] x (x, y, z), in
        the face's (p, q) order: p along axis (d+1)%3, q along (d+2)%3 (d the face's axis)."""
        f = FACES[face] if isinstance(face, str) else face
        d, plus = f // 2, f % 2
        n = self.blocks[blk]
        (ln, org) = self.geometry[blk]
        a1, a2 = (d + 1) % 3, (d + 2) % 3
        out = np.zeros((2, n[a2], n[a1], 3))
        for layer in range(2):
            idx = n[d] + layer if plus else -1 - layer
            for q in range(n[a2]):
                for p in range(n[a1]):
                    ijk = [0, 0, 0]
                    ijk[d], ijk[a1], ijk[a2] = idx, p, q
                    out[layer, q, p] = [org[c] + (ijk[c] + 0.5) * ln[c] for c in range(3)]
        return out

    def set_ghost_states(self, blk, face, pTv):
        """Ghost states of a face given by the caller (as UserDefinedGhostCell supplies
        them): pTv [2][q][p][5] = p, T, vel.x, vel.y, vel.z, positions as ghost_positions."""
        f = FACES[face] if isinstance(face, str) else face
        arr = np.ascontiguousarray(pTv, dtype=np.float64)
        if self.L.orc_set_ghost_states(self.h, blk, f, _p(arr)) != 0:
            raise ValueError("bad ghost states")

    def set_source(self, blk, Q):
        """Fixed per-cell source term [nq][ncells] added to dU/dt (user-defined source)."""
        arr = np.ascontiguousarray(Q, dtype=np.float64)
        if self.L.orc_set_source(self.h, blk, _p(arr)) != 0:
            raise ValueError("bad source")

    def set_bc(self, blk, face, kind, x_order=0, other_block=-1, other_face=-1, inflow=None):
        """inflow: dict with p, T, vel=(3,), B=(3,), psi (FlowState:new{p=,T=,...})."""
        arr = np.zeros(9)
        if inflow is not None:
            arr[0] = inflow["p"]
            arr[1] = inflow.get("T", 0.0)
            arr[2:5] = inflow.get("vel", (0.0, 0.0, 0.0))
            arr[5:8] = inflow.get("B", (0.0, 0.0, 0.0))
            arr[8] = inflow.get("psi", 0.0)
        f = FACES[face] if isinstance(face, str) else face
        of = FACES[other_face] if isinstance(other_face, str) else other_face
        rc = self.L.orc_set_bc(self.h, blk, f, BC[kind], x_order, other_block, of, _p(arr))
        if rc != 0:
            raise ValueError("set_bc failed")

    def set_exchange(self, blk, face, other_block, other_face, orientation=0, Rmatrix=None):
        """ExchangeBC_FullFace{otherBlock, otherFace, orientation, reorient_vector_quantities,
        Rmatrix} (bc.lua:1603-1625); Rmatrix: 9 numbers, row major, or None."""
        f = FACES[face] if isinstance(face, str) else face
        of = FACES[other_face] if isinstance(other_face, str) else other_face
        R = None if Rmatrix is None else np.ascontiguousarray(Rmatrix, dtype=np.float64).reshape(9)
        rc = self.L.orc_set_exchange(self.h, blk, f, other_block, of, orientation, None if R is None else _p(R))
        if rc != 0:
            raise ValueError("set_exchange failed")

    def set_flow_rhoT(self, blk, rho, vel, T, B=None, psi=None):
        """Arrays shaped (nkc, njc, nic) (i fastest); vel (3, ...)."""
        nic, njc, nkc = self.blocks[blk]
        n = nic * njc * nkc
        prim = np.zeros((9, n))
        prim[0] = np.broadcast_to(rho, (nkc, njc, nic)).ravel()
        for c in range(3):
            prim[1 + c] = np.broadcast_to(vel[c], (nkc, njc, nic)).ravel()
        prim[4] = np.broadcast_to(T, (nkc, njc, nic)).ravel()
        if B is not None:
            for c in range(3):
                prim[5 + c] = np.broadcast_to(B[c], (nkc, njc, nic)).ravel()
        if psi is not None:
            prim[8] = np.broadcast_to(psi, (nkc, njc, nic)).ravel()
        prim = np.ascontiguousarray(prim)
        if self.L.orc_set_flow_rhoT(self.h, blk, _p(prim)) != 0:
            raise ValueError("bad initial state")

    def init(self):
        self.L.orc_init(self.h)

    def run(self, nsteps, max_time=0.0, fixed_dt=None):
        rc = self.L.orc_run(self.h, int(nsteps), float(max_time), 1 if fixed_dt else 0,
                            float(fixed_dt or 0.0))
        return rc

    def time(self):
        out = np.zeros(5)
        st = ctypes.c_int(0)
        self.L.orc_get_time(self.h, _p(out), ctypes.byref(st))
        return dict(time=out[0], dt=out[1], c_h=out[2], cfl_max=out[3], dt_allow=out[4], step=st.value)

    def get_U(self, blk):
        nic, njc, nkc = self.blocks[blk]
        out = np.zeros((self.nq, nic * njc * nkc))
        self.L.orc_get_U(self.h, blk, _p(out))
        return out

    def set_U(self, blk, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        return self.L.orc_set_U(self.h, blk, _p(U))

    def get_flow(self, blk):
        nic, njc, nkc = self.blocks[blk]
        out = np.zeros((12, nic * njc * nkc))
        self.L.orc_get_flow(self.h, blk, _p(out))
        names = ["rho", "vx", "vy", "vz", "u", "p", "T", "a", "Bx", "By", "Bz", "psi"]
        return {k: out[q] for q, k in enumerate(names)}

    def all_U(self):
        return np.concatenate([self.get_U(b).ravel() for b in range(len(self.blocks))])

    def residual(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        R = np.zeros_like(U)
        rc = self.L.orc_residual(self.h, _p(U), _p(R))
        if rc != 0:
            raise ValueError("residual failed")
        return R

    def jvp_complex(self, U, v, sigma=1.0e-30):
        U = np.ascontiguousarray(U, dtype=np.float64)
        v = np.ascontiguousarray(v, dtype=np.float64)
        Jv = np.zeros_like(U)
        if self.L.orc_jvp_complex(self.h, _p(U), _p(v), sigma, _p(Jv)) != 0:
            raise ValueError("jvp failed")
        return Jv

    def jvp_real(self, U, v, sigma=0.0):
        U = np.ascontiguousarray(U, dtype=np.float64)
        v = np.ascontiguousarray(v, dtype=np.float64)
        Jv = np.zeros_like(U)
        used = np.zeros(1)
        if self.L.orc_jvp_real(self.h, _p(U), _p(v), sigma, _p(Jv), _p(used)) != 0:
            raise ValueError("jvp failed")
        return Jv, used[0]

    def face_flux(self, d, cells, length):
        cells = np.ascontiguousarray(cells, dtype=np.float64).reshape(4, 12)
        F = np.zeros(self.nq)
        self.L.orc_face_flux(self.h, d, _p(cells), float(length), _p(F))
        return F

    def last_error(self):
        buf = ctypes.create_string_buffer(512)
        self.L.orc_last_error(self.h, buf, 512)
        return buf.value.decode()

    def __del__(self):
        try:
            self.L.orc_free(self.h)
        except Exception:
            pass


def exchange_source(dims, face, other_face, orientation, n, n_other, ijk):
    """The partner cell (i, j, k) that the exchange ghost ijk copies (full_face_copy.d:680-1409),
    or None for a ghost the map does not place inside the partner."""
    L = lib()
    arr = lambda v: (ctypes.c_int * 3)(*[int(x) for x in v])
    src = (ctypes.c_int * 3)()
    rc = L.orc_exchange_source(dims, face, other_face, orientation, arr(n), arr(n_other), arr(ijk), src)
    return None if rc != 0 else tuple(src)

