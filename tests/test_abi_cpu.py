"""C-ABI checks that need no GPU: the library loads, exports every symbol the
header declares, and rejects bad arguments before touching the device."""

import ctypes as C

import pytest

from pelephysics_b200 import _lib


def test_library_exports_header_symbols():
    L = _lib.lib()
    names = _lib.header_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_mechanism_info_and_names():
    assert _lib.mechanism_info("LiDryer") == (9, 21)
    assert _lib.mechanism_info("drm19") == (21, 84)
    assert _lib.mechanism_info("dodecane_lu") == (53, 268)
    assert _lib.mechanism_info("heptane_lu_88sk") == (88, 729)
    assert _lib.species_names("LiDryer")[:3] == ["H2", "O2", "H2O"]
    with pytest.raises(_lib.EngineError) as e:
        _lib.mechanism_info("nope")
    assert e.value.code == _lib.PPB_E_MECH


def test_default_options_match_reference_defaults():
    o = _lib.default_options()
    assert (o.rtol, o.atol, o.max_order, o.max_steps, o.max_nls_iters) == (1e-6, 1e-10, 2, 10000, 3)
    assert (o.rk64_nsubsteps_guess, o.rk64_nsubsteps_min, o.rk64_nsubsteps_max) == (10, 5, 500)
    # engine tuning: the block rendezvous before each right-hand side is on,
    # its bound picked by block size
    assert o.rendezvous_cycles == -1 and o.cost_order == 1
    assert o.arkode_barrier_us == 20000000


def test_rendezvous_and_block_size_bounds_checked_without_device():
    L = _lib.lib()
    h = C.c_void_p()
    assert L.ppb_create(b"drm19", b"ReactorCvode", C.byref(h)) == 0
    for field, bad, msg in (("rendezvous_cycles", -2, b"rendezvous_cycles"),
                            ("rendezvous_cycles", 10000001, b"rendezvous_cycles"),
                            ("warps_per_block", 17, b"warps_per_block"),
                            ("arkode_barrier_us", -1, b"arkode_barrier_us"),
                            ("arkode_barrier_us", 60000001, b"arkode_barrier_us")):
        o = _lib.default_options()
        setattr(o, field, bad)
        assert L.ppb_init(h, 1, 10, C.byref(o)) == _lib.PPB_E_ARG
        assert msg in L.ppb_last_error()
    L.ppb_destroy(h)


def test_bad_arguments_rejected_without_device():
    L = _lib.lib()
    h = C.c_void_p()
    assert L.ppb_create(b"drm19", b"NoSuchReactor", C.byref(h)) == _lib.PPB_E_ARG
    assert L.ppb_create(b"nope", b"ReactorCvode", C.byref(h)) == _lib.PPB_E_MECH
    assert L.ppb_create(b"drm19", b"ReactorCvode", C.byref(h)) == 0
    o = _lib.default_options()
    # ReactorTypes::check_reactor_type message
    assert L.ppb_init(h, 3, 10, C.byref(o)) == _lib.PPB_E_ARG
    assert b"Wrong reactor type" in L.ppb_last_error()
    o.max_order = 6
    assert L.ppb_init(h, 1, 10, C.byref(o)) == _lib.PPB_E_ARG
    dt = C.c_double(1e-5)
    t = C.c_double(0.0)
    cost = C.c_long()
    assert L.ppb_react_flat(h, None, None, None, None, C.byref(dt), C.byref(t), 4, None, C.byref(cost)) == \
        _lib.PPB_E_STATE
    L.ppb_destroy(h)
