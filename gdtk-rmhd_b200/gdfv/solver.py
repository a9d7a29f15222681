"""Host-side solver API over libgdfv, in the vocabulary of the reference's
job scripts (e4/prep.lua, e4/configoptions.lua, e4/bc.lua, e4/fluidblock.lua):

    cfg = Config(flux_calculator="ausmdv")          # config.flux_calculator = "ausmdv"
    sim = Simulation(cfg, gas=IdealGas(R=287.1, gamma=1.4))
    inflow = FlowState(p=5e3, T=220.0, velx=891.8)   # FlowState:new{p=,T=,velx=}
    blk = sim.add_block(nic, njc, nkc, dx, dy, dz,
                        bcList={"west": InFlowBC_Supersonic(inflow),
                                "east": OutFlowBC_SimpleExtrapolate()})
    sim.set_flow_rhoT(blk, rho, vel, T)
    sim.run(max_time=..., max_step=...)

Option names and accepted values are the reference's (e4/globalconfig.d:1858-2004),
boundary-condition classes keep the reference's names.  Every call goes through
the C ABI in include/gdfv.h.
"""
import numpy as np

from ._lib import GDFV_OK, GdfvError, check, ffi, lib

FACE_INDEX = {"west": 0, "iminus": 0, "east": 1, "iplus": 1, "south": 2, "jminus": 2,
              "north": 3, "jplus": 3, "bottom": 4, "kminus": 4, "top": 5, "kplus": 5}
FACE_NAMES = ["west", "east", "south", "north", "bottom", "top"]

_STR_KEYS = ("flux_calculator", "gasdynamic_update_scheme", "thermo_interpolator", "flux_precision",
             "van_albada_variant")
_INT_KEYS = ("interpolation_order", "dimensions", "MHD", "divergence_cleaning", "apply_limiter",
             "extrema_clipping", "apply_entropy_fix", "interpolate_in_local_frame", "stringent_cfl",
             "cfl_count", "max_attempts_for_step", "max_invalid_cells", "fixed_time_step",
             "n_ghost_cell_layers", "glm_reference_indexing", "tile_kchunk", "persistent", "tile_width",
             "autotune")
_DBL_KEYS = ("cfl_value", "dt_init", "dt_max", "epsilon_van_albada", "divB_damping_length",
             "flowstate_limits_max_velocity", "flowstate_limits_max_temp", "flowstate_limits_min_temp")


class Config:
    """Solver options.  Defaults are the reference's (e4/globalconfig.d:927-1299)
    except flux_calculator, whose reference default (adaptive_hanel_ausmdv) is not
    on this path; ausmdv is used instead."""

    def __init__(self, **kw):
        self.flux_calculator = "ausmdv"
        self.gasdynamic_update_scheme = "predictor_corrector"
        self.thermo_interpolator = "rhou"
        self.flux_precision = "fp64"
        self.van_albada_variant = "e4"   # "lmr": epsilon scaled per face as Eilmer 5 (lmr) does
        self.interpolation_order = 2
        self.dimensions = 3
        self.MHD = False
        self.divergence_cleaning = False
        self.apply_limiter = True
        self.extrema_clipping = True
        self.apply_entropy_fix = True
        self.interpolate_in_local_frame = True
        self.stringent_cfl = False
        self.cfl_count = 10
        self.max_attempts_for_step = 3
        self.max_invalid_cells = 0
        self.fixed_time_step = False
        self.n_ghost_cell_layers = 2
        self.glm_reference_indexing = True
        self.tile_kchunk = 0          # planes per tile (0: the block's nkc up to 32)
        self.persistent = False       # True: stage kernels as a resident grid over the tile queue
        self.tile_width = 32          # float Euler kernel: tiles 32 or 16 cells wide
        self.autotune = False         # time tile shapes and launch forms on the first run
        self.cfl_value = 0.5
        self.dt_init = 1.0e-3
        self.dt_max = 1.0e-3
        self.epsilon_van_albada = 1.0e-12
        self.divB_damping_length = 1.0
        self.flowstate_limits_max_velocity = 30000.0
        self.flowstate_limits_max_temp = 50000.0
        self.flowstate_limits_min_temp = 0.0
        for k, v in kw.items():
            if not hasattr(self, k):
                raise KeyError(f"unknown config option {k}")
            setattr(self, k, v)


class IdealGas:
    """Ideal gas (src/gas/ideal_gas.d): R = R_universal / mMass."""

    R_UNIVERSAL = 8.31451  # src/gas/physical_constants.d:13

    def __init__(self, R=None, gamma=1.4, mMass=None):
        if R is None:
            if mMass is None:
                raise ValueError("give R or mMass")
            R = self.R_UNIVERSAL / mMass
        self.R = float(R)
        self.gamma = float(gamma)
        self.Cv = self.R / (self.gamma - 1.0)


class FlowState:
    """Uniform flow state given by p and T (FlowState:new{p=,T=,velx=,...})."""

    def __init__(self, p, T, velx=0.0, vely=0.0, velz=0.0, Bx=0.0, By=0.0, Bz=0.0, psi=0.0):
        self.p, self.T = float(p), float(T)
        self.vel = (float(velx), float(vely), float(velz))
        self.B = (float(Bx), float(By), float(Bz))
        self.psi = float(psi)

    def as_array(self):
        return np.array([self.p, self.T, *self.vel, *self.B, self.psi], dtype=np.float64)


class WallBC_WithSlip:
    name = "wall_with_slip"


class OutFlowBC_SimpleExtrapolate:
    name = "outflow_simple_extrapolate"

    def __init__(self, xOrder=0):
        self.xOrder = int(xOrder)


class OutFlowBC_SimpleFlux:
    """bc.lua:1532-1556: ghost cells by ExtrapolateCopy (xOrder 0) and the boundary
    face's flux from the interior cell (boundary_flux_effect.d:504-645)."""
    name = "outflow_simple_flux"


class OutFlowBC_FixedP:
    """bc.lua:1558-1578: ghost cells copy the interior cells with the pressure fixed
    at p_outside (fixed_p.d)."""
    name = "outflow_fixed_p"

    def __init__(self, p_outside, xOrder=0):
        self.p_outside = float(p_outside)
        self.xOrder = int(xOrder)


class OutFlowBC_FixedPT:
    """bc.lua:1580-1600: ghost cells copy the interior cells' velocity with pressure
    and temperature fixed at p_outside, T_outside (fixed_pt.d)."""
    name = "outflow_fixed_p_and_t"

    def __init__(self, p_outside, T_outside, xOrder=0):
        self.p_outside = float(p_outside)
        self.T_outside = float(T_outside)
        self.xOrder = int(xOrder)


class InFlowBC_Supersonic:
    name = "inflow_supersonic"

    def __init__(self, flowState):
        self.flowState = flowState


class ExchangeBC_FullFace:
    """bc.lua:1603-1625: the ghost cells copy the partner block's cells inside face
    otherFace, placed by the face pair and orientation (full_face_copy.d:680-1409); with
    reorient_vector_quantities their velocity and magnetic field are multiplied by the
    row-major 3x3 Rmatrix (flowstate.d:393-400)."""
    name = "exchange_over_full_face"

    def __init__(self, otherBlock, otherFace, orientation=0, reorient_vector_quantities=False,
                 Rmatrix=(1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0)):
        self.otherBlock = int(otherBlock)
        self.otherFace = FACE_INDEX[otherFace] if isinstance(otherFace, str) else int(otherFace)
        self.orientation = int(orientation)
        self.reorient_vector_quantities = bool(reorient_vector_quantities)
        self.Rmatrix = np.asarray(Rmatrix, dtype=np.float64).reshape(9)


class Simulation:
    """One libgdfv context: configuration, blocks, and the time-marching state."""

    def __init__(self, config=None, gas=None):
        self.config = config or Config()
        self.gas = gas or IdealGas(R=287.1, gamma=1.4)
        self.L = lib()
        self.ctx = self.L.gdfv_context_new()
        if self.ctx < 0:
            raise GdfvError(self.ctx, "could not create a context")
        self.blocks = []
        self._bcs = []
        self._prepared = False
        self._inflow = {}   # (block, face) -> state array of a supersonic-inflow face

    # ---------------------------------------------------------------- setup
    def _apply_config(self):
        c = self.config
        L, h = self.L, self.ctx
        for k in _STR_KEYS:
            check(h, L.gdfv_config_set_str(h, k.encode(), str(getattr(c, k)).encode()))
        for k in _INT_KEYS:
            check(h, L.gdfv_config_set_int(h, k.encode(), int(getattr(c, k))))
        for k in _DBL_KEYS:
            check(h, L.gdfv_config_set_double(h, k.encode(), float(getattr(c, k))))
        check(h, L.gdfv_config_set_double(h, b"R", self.gas.R))
        check(h, L.gdfv_config_set_double(h, b"gamma", self.gas.gamma))

    @property
    def nq(self):
        return 10 if self.config.MHD else 5

    def add_block(self, nic, njc, nkc, dx, dy, dz, x0=0.0, y0=0.0, z0=0.0, bcList=None):
        """A uniform Cartesian block; bcList maps face names to BC objects
        (faces not listed are slip walls, as in e4/fluidblock.lua:102)."""
        b = self.L.gdfv_block_new(self.ctx, nic, njc, nkc, dx, dy, dz, x0, y0, z0)
        if b < 0:
            check(self.ctx, b)
        self.blocks.append((nic, njc, nkc))
        self._bcs.append({})
        for face, bc in (bcList or {}).items():
            self.set_bc(b, face, bc)
        return b

    def inflow_states(self):
        """State arrays {p, T, vel.x, vel.y, vel.z, B.x, B.y, B.z, psi} of the
        supersonic-inflow faces in the order the library numbers them (by block, then
        face; faces beyond the active ones of a 2D run carry none)."""
        nfaces = 6 if int(self.config.dimensions) == 3 else 4
        return [self._inflow[k] for k in sorted(self._inflow) if k[1] < nfaces]

    @property
    def n_inflow(self):
        return len(self.inflow_states())

    def set_inflow(self, index, flowState):
        """Replace the state of supersonic-inflow face `index` (inflow_states order)
        after preparation; the next step uses it."""
        self.prepare()
        arr = np.ascontiguousarray(flowState.as_array() if hasattr(flowState, "as_array") else flowState,
                                   dtype=np.float64)
        check(self.ctx, self.L.gdfv_set_inflow(self.ctx, int(index), ffi.cast("double*", arr.ctypes.data)))
        self.inflow_states()[index][:] = arr

    def last_bad_cell(self):
        """(block, (i, j, k), (x, y, z)) of the cell the last failed step reported."""
        blk = ffi.new("int*")
        ijk = ffi.new("int[3]")
        pos = ffi.new("double[3]")
        check(self.ctx, self.L.gdfv_last_bad_cell(self.ctx, blk, ijk, pos))
        return blk[0], (ijk[0], ijk[1], ijk[2]), (pos[0], pos[1], pos[2])

    def add_block_graded(self, xv, yv, zv, bcList=None):
        """A rectilinear block from its vertex coordinates along each axis (stretched
        grids): cell (i, j, k) spans [xv[i], xv[i+1]] x [yv[j], yv[j+1]] x [zv[k], zv[k+1]]."""
        xv, yv, zv = (np.ascontiguousarray(v, dtype=np.float64) for v in (xv, yv, zv))
        n = (len(xv) - 1, len(yv) - 1, len(zv) - 1)
        p = lambda a: ffi.cast("double*", a.ctypes.data)
        b = self.L.gdfv_block_new_graded(self.ctx, *n, p(xv), p(yv), p(zv))
        if b < 0:
            check(self.ctx, b)
        self.blocks.append(n)
        self._bcs.append({})
        for face, bc in (bcList or {}).items():
            self.set_bc(b, face, bc)
        return b

    def set_bc(self, blk, face, bc):
        f = FACE_INDEX[face] if isinstance(face, str) else int(face)
        x_order, other, other_face = 0, -1, -1
        inflow = ffi.NULL
        self._inflow.pop((blk, f), None)
        if isinstance(bc, OutFlowBC_SimpleExtrapolate):
            x_order = bc.xOrder
        elif isinstance(bc, ExchangeBC_FullFace):
            R = ffi.NULL
            if bc.reorient_vector_quantities:
                arr = np.ascontiguousarray(bc.Rmatrix, dtype=np.float64)
                self._bcs[blk][f] = arr
                R = ffi.cast("double*", arr.ctypes.data)
            check(self.ctx, self.L.gdfv_block_set_exchange(self.ctx, blk, f, bc.otherBlock, bc.otherFace,
                                                            bc.orientation, R))
            return
        elif isinstance(bc, InFlowBC_Supersonic):
            arr = np.array(bc.flowState.as_array(), dtype=np.float64)
            self._bcs[blk][f] = arr  # keep alive
            inflow = ffi.cast("double*", arr.ctypes.data)
            self._inflow[(blk, f)] = arr
        elif isinstance(bc, (OutFlowBC_FixedP, OutFlowBC_FixedPT)):
            arr = np.zeros(9)
            arr[0] = bc.p_outside
            arr[1] = getattr(bc, "T_outside", 0.0)
            self._bcs[blk][f] = arr
            inflow = ffi.cast("double*", arr.ctypes.data)
            x_order = bc.xOrder
        check(self.ctx, self.L.gdfv_block_set_bc(self.ctx, blk, f, bc.name.encode(), x_order, other,
                                                  other_face, inflow))

    def prepare(self):
        if not self._prepared:
            self._apply_config()
            check(self.ctx, self.L.gdfv_prepare(self.ctx))
            self._prepared = True

    def ncells(self, blk):
        nic, njc, nkc = self.blocks[blk]
        return nic * njc * nkc

    # ---------------------------------------------------------------- state
    def set_flow_rhoT(self, blk, rho, vel, T, B=None, psi=None):
        """Cell states from density, velocity and temperature (arrays shaped
        (nkc, njc, nic) or broadcastable)."""
        self.prepare()
        nic, njc, nkc = self.blocks[blk]
        shp = (nkc, njc, nic)
        prim = np.zeros((9, nic * njc * nkc))
        prim[0] = np.broadcast_to(rho, shp).ravel()
        for c in range(3):
            prim[1 + c] = np.broadcast_to(vel[c], shp).ravel()
        prim[4] = np.broadcast_to(T, shp).ravel()
        if B is not None:
            for c in range(3):
                prim[5 + c] = np.broadcast_to(B[c], shp).ravel()
        if psi is not None:
            prim[8] = np.broadcast_to(psi, shp).ravel()
        prim = np.ascontiguousarray(prim)
        check(self.ctx, self.L.gdfv_block_set_flow_rhoT(self.ctx, blk, ffi.cast("double*", prim.ctypes.data)))

    def set_flowstate(self, blk, fs):
        """Uniform initial state from a p,T FlowState."""
        rho = fs.p / (fs.T * self.gas.R)
        self.set_flow_rhoT(blk, rho, fs.vel, fs.T, B=fs.B, psi=fs.psi)

    def get_conserved(self, blk, out=None):
        """Conserved state of block blk as (nq, ncells) float64.  `out` (C-contiguous
        float64 of that shape, e.g. a view of pinned host memory) is filled in place
        and returned; without it a new array is allocated."""
        self.prepare()
        shape = (self.nq, self.ncells(blk))
        if out is None:
            out = np.empty(shape)
        elif out.shape != shape or out.dtype != np.float64 or not out.flags["C_CONTIGUOUS"]:
            raise ValueError(f"out must be a C-contiguous float64 array of shape {shape}")
        check(self.ctx, self.L.gdfv_block_get_conserved(self.ctx, blk, ffi.cast("double*", out.ctypes.data)))
        return out

    def set_conserved(self, blk, U):
        self.prepare()
        U = np.ascontiguousarray(U, dtype=np.float64)
        check(self.ctx, self.L.gdfv_block_set_conserved(self.ctx, blk, ffi.cast("double*", U.ctypes.data)))

    def get_flow(self, blk):
        self.prepare()
        out = np.zeros((12, self.ncells(blk)))
        check(self.ctx, self.L.gdfv_block_get_flow(self.ctx, blk, ffi.cast("double*", out.ctypes.data)))
        names = ["rho", "vx", "vy", "vz", "u", "p", "T", "a", "Bx", "By", "Bz", "psi"]
        return {k: out[q] for q, k in enumerate(names)}

    # ---------------------------------------------------------------- marching
    def run(self, max_step=1, max_time=0.0):
        """Advance until max_step more steps or time >= max_time; returns steps taken."""
        self.prepare()
        taken = ffi.new("int*")
        check(self.ctx, self.L.gdfv_run(self.ctx, int(max_step), float(max_time), taken))
        return taken[0]

    def time(self):
        out = ffi.new("double[5]")
        st = ffi.new("int*")
        check(self.ctx, self.L.gdfv_get_time(self.ctx, out, st))
        return dict(time=out[0], dt=out[1], c_h=out[2], cfl_max=out[3], dt_allow=out[4], step=st[0])

    def set_time(self, time, step, dt_global):
        check(self.ctx, self.L.gdfv_set_time(self.ctx, float(time), int(step), float(dt_global)))

    def total_cells(self):
        return int(self.L.gdfv_total_cells(self.ctx))

    def residual(self, U_ptr, R_ptr):
        """R(U) on device arrays [nq][total] given as integer device addresses."""
        check(self.ctx, self.L.gdfv_residual(self.ctx, ffi.cast("double*", U_ptr), ffi.cast("double*", R_ptr)))

    def state_ptr(self):
        p = ffi.new("double**")
        check(self.ctx, self.L.gdfv_state_device_ptr(self.ctx, p))
        return int(ffi.cast("uintptr_t", p[0]))

    def set_stream(self, stream_handle):
        check(self.ctx, self.L.gdfv_set_stream(self.ctx, ffi.cast("void*", stream_handle)))

    def residual_norms(self):
        """(Linf[nq], L2) of dU/dt of the last step's predictor stage, the figures the
        reference writes with report_residuals (e4/simcore.d:1193-1212)."""
        self.prepare()
        linf = ffi.new("double[]", self.nq)
        l2 = ffi.new("double*")
        check(self.ctx, self.L.gdfv_residual_norms(self.ctx, linf, l2))
        return np.array([linf[q] for q in range(self.nq)]), float(l2[0])

    def time_stages(self, reps=10):
        ms = ffi.new("double[2]")
        check(self.ctx, self.L.gdfv_time_stages(self.ctx, int(reps), ms))
        return ms[0], ms[1]

    def option(self, key):
        """Current value of a numeric option as the library holds it (after an
        autotuned run: tile_kchunk, persistent, tile_width and autotune_stage_ms)."""
        v = ffi.new("double*")
        check(self.ctx, self.L.gdfv_config_get_double(self.ctx, key.encode(), v))
        return v[0]

    def close(self):
        if getattr(self, "ctx", -1) >= 0:
            self.L.gdfv_context_free(self.ctx)
            self.ctx = -1

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
