"""CPU checks of the boundary: libgdfv.so loads, exports every entry point the
header declares, and takes the reference's option and BC names (no GPU needed
for configuration calls); the oracle library loads; the multi-rank timing
reduction works over gloo with two ranks."""
import ctypes
import os

import pytest

import gdfv
from gdfv._lib import GDFV_ERR_ARG, GDFV_OK, LIBPATH, check, ffi, last_error


def test_library_exports_every_declared_symbol():
    syms = gdfv.exported_symbols()
    assert len(syms) >= 20
    raw = ctypes.CDLL(LIBPATH)
    for s in syms:
        assert hasattr(raw, s), s          # dlsym
        getattr(gdfv.lib(), s)             # and the cffi binding


def test_config_accepts_reference_names_and_rejects_others():
    L = gdfv.lib()
    h = L.gdfv_context_new()
    assert h >= 0
    for key, val in (("flux_calculator", "ausmdv"), ("flux_calculator", "hllc"), ("flux_calculator", "hlle"),
                     ("gasdynamic_update_scheme", "predictor-corrector"), ("gasdynamic_update_scheme", "pc"),
                     ("thermo_interpolator", "rhou"), ("flux_precision", "fp32")):
        assert L.gdfv_config_set_str(h, key.encode(), val.encode()) == GDFV_OK, (key, val)
    for key, val in (("flux_calculator", "roe"), ("gasdynamic_update_scheme", "tvd_rk3"),
                     ("thermo_interpolator", "pT"), ("no_such_option", "x")):
        assert L.gdfv_config_set_str(h, key.encode(), val.encode()) == GDFV_ERR_ARG
        assert len(last_error(h)) > 0
    for key, val in (("interpolation_order", 2), ("MHD", 1), ("divergence_cleaning", 1), ("cfl_count", 10),
                     ("max_attempts_for_step", 3), ("n_ghost_cell_layers", 2), ("dimensions", 3)):
        assert L.gdfv_config_set_int(h, key.encode(), val) == GDFV_OK, key
    for key, val in (("tile_kchunk", 16), ("persistent", 0), ("autotune", 1)):
        assert L.gdfv_config_set_int(h, key.encode(), val) == GDFV_OK, key
        check(h, L.gdfv_config_get_double(h, key.encode(), v := ffi.new("double*")))
        assert v[0] == val
    assert L.gdfv_config_set_int(h, b"tile_kchunk", -1) == GDFV_ERR_ARG
    assert L.gdfv_config_set_int(h, b"interpolation_order", 3) == GDFV_ERR_ARG
    assert L.gdfv_config_set_int(h, b"cfl_count", 0) == GDFV_ERR_ARG
    for key in ("cfl_value", "dt_init", "dt_max", "epsilon_van_albada", "R", "gamma", "divB_damping_length"):
        assert L.gdfv_config_set_double(h, key.encode(), 0.5) == GDFV_OK, key
    v = ffi.new("double*")
    check(h, L.gdfv_config_get_double(h, b"cfl_value", v))
    assert v[0] == 0.5
    assert L.gdfv_context_free(h) == GDFV_OK
    assert L.gdfv_context_free(h) == GDFV_ERR_ARG


def test_blocks_and_boundary_names():
    L = gdfv.lib()
    h = L.gdfv_context_new()
    assert L.gdfv_block_new(h, 0, 4, 4, 1.0, 1.0, 1.0, 0, 0, 0) < 0
    b = L.gdfv_block_new(h, 8, 4, 4, 1e-3, 1e-3, 1e-3, 0, 0, 0)
    assert b == 0
    inflow = ffi.new("double[9]", [5e3, 220.0, 890.0, 0, 0, 0, 0, 0, 0])
    for face, name in ((0, b"inflow_supersonic"), (1, b"outflow_simple_extrapolate"), (2, b"wall_with_slip"),
                       (3, b"exchange_over_full_face")):
        assert L.gdfv_block_set_bc(h, b, face, name, 0, 0, 2, inflow) == GDFV_OK
    assert L.gdfv_block_set_bc(h, b, 4, b"wall_no_slip_fixed_t", 0, -1, -1, ffi.NULL) == GDFV_ERR_ARG
    assert L.gdfv_block_set_bc(h, b, 7, b"wall_with_slip", 0, -1, -1, ffi.NULL) == GDFV_ERR_ARG
    assert L.gdfv_block_ncells(h, b) == 128
    assert L.gdfv_total_cells(h) == 128
    L.gdfv_context_free(h)


def test_oracle_library_loads():
    from oracle import lib as orc_lib
    L = orc_lib()
    assert L.orc_new() >= 0


def _ranks_worker(rank, world, port, q):
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    q.put((rank, bench.max_over_ranks(10.0 + rank)))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    import socket
    import sys
    import torch.multiprocessing as mp
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in sys.path:
        sys.path.insert(0, root)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_ranks_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert res == {0: 11.0, 1: 11.0}


def _ctx_with_block(L, n, dims=3, flux=b"ausmdv"):
    h = L.gdfv_context_new()
    assert L.gdfv_config_set_int(h, b"dimensions", dims) == GDFV_OK
    assert L.gdfv_config_set_str(h, b"flux_calculator", flux) == GDFV_OK
    b = L.gdfv_block_new(h, n[0], n[1], n[2], 1e-3, 1e-3, 1e-3, 0, 0, 0)
    return h, b


def test_prepare_rejects_invalid_layouts_before_touching_the_device():
    """Layout errors come back from gdfv_prepare as status codes with a message, like
    the reference's C wrappers (src/gas/gas_cwrap.d:423-446), and before any device
    allocation (this test runs without a GPU)."""
    from gdfv._lib import GDFV_ERR_STATE
    L = gdfv.lib()
    h = L.gdfv_context_new()
    assert L.gdfv_prepare(h) == GDFV_ERR_STATE          # no blocks
    assert "no blocks" in last_error(h)
    assert L.gdfv_block_new(h, 1 << 12, 1 << 12, 1 << 11, 1e-3, 1e-3, 1e-3, 0, 0, 0) == GDFV_ERR_ARG
    L.gdfv_context_free(h)
    # the kernels index a block's cells and faces in 32-bit arithmetic
    h, b = _ctx_with_block(L, (1300, 1300, 1300))
    assert b == 0
    assert L.gdfv_prepare(h) == GDFV_ERR_ARG
    assert "2^31" in last_error(h)
    L.gdfv_context_free(h)
    h, _ = _ctx_with_block(L, (16, 1, 16))                # one cell thick in an active direction
    assert L.gdfv_prepare(h) == GDFV_ERR_ARG
    L.gdfv_context_free(h)
    h, _ = _ctx_with_block(L, (16, 16, 2), dims=2)        # 2D blocks have nkc = 1
    assert L.gdfv_prepare(h) == GDFV_ERR_ARG
    L.gdfv_context_free(h)
    h, _ = _ctx_with_block(L, (16, 16, 16), flux=b"hlle")  # hlle is the MHD flux
    assert L.gdfv_prepare(h) == GDFV_ERR_ARG
    assert "MHD" in last_error(h)
    L.gdfv_context_free(h)
    # exchange across faces of different sizes, and onto the same face
    h, b0 = _ctx_with_block(L, (16, 16, 16))
    b1 = L.gdfv_block_new(h, 16, 8, 16, 1e-3, 1e-3, 1e-3, 0.016, 0, 0)
    assert L.gdfv_block_set_bc(h, b0, 1, b"exchange_over_full_face", 0, b1, 0, ffi.NULL) == GDFV_OK
    assert L.gdfv_block_set_bc(h, b1, 0, b"exchange_over_full_face", 0, b0, 1, ffi.NULL) == GDFV_OK
    assert L.gdfv_prepare(h) == GDFV_ERR_ARG
    assert "differ in size" in last_error(h)
    L.gdfv_context_free(h)
    # east onto north: the partner's i runs along this face's j (orientation 0) or along
    # its k (orientation 1); a 16 x 8 x 16 partner fits the first, an 8 x 16 x 12 one neither
    for nb1, orientation, ok in (((16, 8, 16), 0, True), ((8, 16, 12), 0, False), ((8, 16, 12), 1, False)):
        h, b0 = _ctx_with_block(L, (16, 16, 16))
        b1 = L.gdfv_block_new(h, *nb1, 1e-3, 1e-3, 1e-3, 0.016, 0, 0)
        assert L.gdfv_block_set_exchange(h, b0, 1, b1, 3, orientation, ffi.NULL) == GDFV_OK
        assert L.gdfv_block_set_exchange(h, b1, 3, b0, 1, orientation, ffi.NULL) == GDFV_OK
        if ok:
            assert L.gdfv_prepare(h) != GDFV_ERR_ARG   # valid: no GPU here, so it fails later
        else:
            assert L.gdfv_prepare(h) == GDFV_ERR_ARG
            assert "differ in size" in last_error(h)
        L.gdfv_context_free(h)
    h, b0 = _ctx_with_block(L, (16, 16, 16))
    assert L.gdfv_block_set_exchange(h, b0, 1, b0, 0, 4, ffi.NULL) == GDFV_ERR_ARG
    bad = ffi.new("double[9]", [1.0, 0.0, 0.0, 0.0, float("nan"), 0.0, 0.0, 0.0, 1.0])
    assert L.gdfv_block_set_exchange(h, b0, 1, b0, 0, 0, bad) == GDFV_ERR_ARG
    assert L.gdfv_block_set_exchange(h, b0, 1, 5, 0, 0, ffi.NULL) == GDFV_OK
    assert L.gdfv_prepare(h) == GDFV_ERR_ARG                     # no block 5
    L.gdfv_context_free(h)


def test_block_size_limits():
    """The largest blocks: the kernels index a block's cells and faces in 32-bit
    arithmetic, so gdfv_prepare refuses a block whose faces of some direction (bounded
    by (nic+1)(njc+1)(nkc+1)) pass 2^31 - 1, before any device allocation; 1289^3 cells
    pass that check, 1290 x 1290 x 1289 do not.  gdfv_block_new refuses more than 2^34
    cells outright."""
    L = gdfv.lib()
    h = L.gdfv_context_new()
    assert L.gdfv_block_new(h, 4096, 4096, 1025, 1e-3, 1e-3, 1e-3, 0, 0, 0) == GDFV_ERR_ARG
    assert "too large" in last_error(h)
    L.gdfv_context_free(h)
    import torch
    # on a machine with a GPU the valid case would go on to allocate 3 x 86 GB
    cases_ = [((1290, 1290, 1289), False)] + ([] if torch.cuda.is_available() else [((1289, 1289, 1289), True)])
    for n, ok in cases_:
        h, b = _ctx_with_block(L, n)
        rc = L.gdfv_prepare(h)
        if ok:
            assert rc != GDFV_ERR_ARG, last_error(h)   # valid: no GPU here, so it fails later
        else:
            assert rc == GDFV_ERR_ARG and "2^31 - 1" in last_error(h)
        L.gdfv_context_free(h)


def test_exchange_map_is_the_reference_map():
    """gdfv_exchange_source (the map the kernels evaluate, from the same rule) against
    the reference's own map of every face pair and orientation
    (full_face_copy.d:680-1409, tests/golden/exchange_map.json), every ghost."""
    import test_oracle_pins as pins
    L = gdfv.lib()
    maps = pins.exchange_maps()
    src = ffi.new("int[3]")
    for rec in maps:
        for n, on, ijk, want in pins.exchange_ghosts(rec):
            rc = L.gdfv_exchange_source(rec["dims"], rec["face"], rec["other_face"], rec["orientation"],
                                        ffi.new("int[3]", n), ffi.new("int[3]", on), ffi.new("int[3]", ijk), src)
            assert rc == GDFV_OK and tuple(src) == want, (rec, ijk)
    n, on = ffi.new("int[3]", [3, 4, 5]), ffi.new("int[3]", [4, 6, 5])
    assert L.gdfv_exchange_source(3, 1, 3, 0, n, on, ffi.new("int[3]", [5, 0, 0]), src) == GDFV_ERR_ARG   # depth 2
    assert L.gdfv_exchange_source(3, 1, 3, 1, n, on, ffi.new("int[3]", [3, 3, 4]), src) == GDFV_ERR_ARG   # too small
    assert L.gdfv_exchange_source(2, 4, 3, 0, n, on, ffi.new("int[3]", [0, 0, -1]), src) == GDFV_ERR_ARG  # 2D k face
