"""C ABI checks that need no GPU: the library loads, exports every entry point
the header declares, its struct layout and defaults agree with the Python
mirror, and invalid configurations are rejected with an error code (never an
exit) before any device work."""
import ctypes as C
import os
import re

import pytest

from mpulse_b200 import abi, runtime

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "mpulse_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mp_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = runtime.lib()
    names = declared_functions()
    assert names, "no declarations found"
    for n in names:
        assert hasattr(L, n), f"{n} declared in include/mpulse_b200.h but not exported"
    assert set(names) == set(runtime.EXPORTED)


def test_defaults_match_python_mirror():
    a = bytes(runtime.library_defaults())
    b = bytes(abi.default_config())
    assert len(a) == C.sizeof(abi.Config)
    assert a == b


def _create_error(cfg):
    L = runtime.lib()
    h = C.c_void_p()
    rc = L.mp_create(C.byref(cfg), C.byref(h))
    return rc, L.mp_create_error().decode()


@pytest.mark.parametrize("mutate,code,text", [
    (lambda c: setattr(c, "abi_version", 99), abi.MP_ERR_INVALID, "abi_version"),
    (lambda c: setattr(c, "nx", 1), abi.MP_ERR_INVALID, "at least 2"),
    (lambda c: setattr(c, "dt", 0.0), abi.MP_ERR_INVALID, "positive"),
    (lambda c: setattr(c.poles[1], "om2", 0.0), abi.MP_ERR_INVALID, "Omega should not be zero"),
    (lambda c: (setattr(c.poles[0], "delta", 2.0), setattr(c.poles[0], "om2", 1.0)), abi.MP_ERR_INVALID, "om2 > delta"),
    (lambda c: (setattr(c, "cpml", abi.MP_CPML_ALL), setattr(c, "cpml_d", 40)), abi.MP_ERR_INVALID, "thicker"),
    (lambda c: (setattr(c, "cpml", abi.MP_CPML_Z), setattr(c, "cpml_sigma_max", 0.0), setattr(c, "cpml_a_max", 0.0)),
     abi.MP_ERR_INVALID, "0/0"),
    (lambda c: (setattr(c, "solver", abi.MP_SOLVER_PLAIN), setattr(c, "cpml", abi.MP_CPML_Z)), abi.MP_ERR_INVALID,
     "cannot be used"),
    (lambda c: (setattr(c, "n_sources", 1), setattr(c.sources[0], "kind", abi.MP_SOURCE_PLANE_GAUSS),
                setattr(c.sources[0], "distance", 0)), abi.MP_ERR_INVALID, "distance"),
    (lambda c: setattr(c, "solver", 9), abi.MP_ERR_INVALID, "unknown solver"),
])
def test_invalid_configs_are_rejected(mutate, code, text):
    cfg = abi.default_config()
    mutate(cfg)
    rc, msg = _create_error(cfg)
    assert rc == code
    assert text in msg


def test_null_arguments():
    L = runtime.lib()
    assert L.mp_create(None, None) == abi.MP_ERR_INVALID
    assert L.mp_step(None, 1) == abi.MP_ERR_INVALID
    assert L.mp_launch_count(None) == -1


def test_tma_staging_needs_tile_multiples():
    cfg = abi.default_config()
    cfg.nx, cfg.ny, cfg.nz = 20, 16, 8
    cfg.staging = abi.MP_STAGING_TMA
    rc, msg = _create_error(cfg)
    assert rc == abi.MP_ERR_UNSUPPORTED and "multiple of 32" in msg


def header_constants():
    """NAME = value enumerators and #define NAME value constants of the header."""
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {m.group(1): int(m.group(2)) for m in re.finditer(r"\b(MP_[A-Z0-9_]+)\s*=\s*(-?\d+)", text)}
    out.update({m.group(1): int(m.group(2)) for m in re.finditer(r"#define\s+(MP_[A-Z0-9_]+)\s+(-?\d+)", text)})
    return out


def test_header_constants_match_python_mirror():
    consts = header_constants()
    assert "MP_ERR_BOUNDS" in consts and "MP_SOLVER_PLRC_NONLIN" in consts
    for name, value in consts.items():
        if hasattr(abi, name):
            assert getattr(abi, name) == value, name
    # every status code has a name in the Python mirror
    for name, value in consts.items():
        if name.startswith("MP_ERR_") or name == "MP_OK":
            assert getattr(abi, name) == value, name


def test_checked_library_exports_the_same_symbols():
    """libmpulse_b200_checked.so (MPB_CHECKED=1) is the same ABI."""
    from mpulse_b200 import build
    assert os.path.exists(build.LIB_CHECKED), "build the checked library: python -m mpulse_b200.build --checked"
    L = C.CDLL(build.LIB_CHECKED)
    for n in declared_functions():
        assert hasattr(L, n), n
