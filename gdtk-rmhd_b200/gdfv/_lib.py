"""cffi binding of libgdfv.so, in the style of the reference's loadable
libraries (src/lib/gdtk/gas.py:12-126: ffi.cdef of the C header, then
ffi.dlopen of the shared object).

The CUDA library is the only implementation: importing this module fails
loudly if libgdfv.so is absent; there is no CPU fallback.
"""
import os
import re

from cffi import FFI

_HERE = os.path.dirname(os.path.abspath(__file__))
_REPO = os.path.dirname(os.path.dirname(_HERE))
HEADER = os.path.join(_REPO, "include", "gdfv.h")
# GDFV_LIBRARY selects another build of the same library (e.g. other tile sizes)
LIBPATH = os.environ.get("GDFV_LIBRARY") or os.path.join(_HERE, "libgdfv.so")

GDFV_OK = 0
GDFV_ERR_ARG = -1
GDFV_ERR_BAD_CELLS = -2
GDFV_ERR_STEP_FAILED = -3
GDFV_ERR_CUDA = -4
GDFV_ERR_STATE = -5


def _cdef_source():
    with open(HEADER) as f:
        src = f.read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    lines = []
    for line in src.splitlines():
        s = line.strip()
        if not s or s.startswith("#") or s.startswith("extern \"C\"") or s == "}":
            continue
        lines.append(line)
    return "\n".join(lines)


ffi = FFI()
ffi.cdef(_cdef_source())

_lib = None


class GdfvError(RuntimeError):
    """Raised when a libgdfv entry point returns a nonzero status."""

    def __init__(self, code, msg):
        super().__init__(f"gdfv error {code}: {msg}")
        self.code = code


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise ImportError(
                f"libgdfv.so not found at {LIBPATH}; build it with `make -C gdtk-rmhd_b200` "
                "(the CUDA library is required; there is no CPU path)")
        _lib = ffi.dlopen(LIBPATH)
    return _lib


def last_error(ctx):
    buf = ffi.new("char[1024]")
    lib().gdfv_last_error(ctx, buf, 1024)
    return ffi.string(buf).decode(errors="replace")


def check(ctx, rc):
    if rc != GDFV_OK:
        raise GdfvError(rc, last_error(ctx))
    return rc


def exported_symbols():
    """Function names the header declares (for the ABI check)."""
    with open(HEADER) as f:
        src = re.sub(r"/\*.*?\*/", "", f.read(), flags=re.S)
    return re.findall(r"\b(gdfv_[a-z_0-9]+)\s*\(", src)
