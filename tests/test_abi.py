"""The C-ABI library loads and exports every function include/cells.h declares (CPU only: no
compute calls)."""
import ctypes
import os
import re

from cells_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(cells\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_solver_api():
    names = declared_functions()
    for must in ("cells3d_create", "cells3d_step", "cells3d_read_forces", "cells3d_read_macro", "cells3d_set_sdf",
                 "cells2d_create", "cells2d_step", "cells2d_read_forces", "cells2d_read_macro", "cells2d_set_sdf",
                 "cells2d_update", "cells2d_brush", "cells2d_batch_create", "cells2d_batch_step",
                 "cells2d_batch_autotune", "cells3d_sample_slice", "cells3d_advect_tracers"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert missing == []


def test_copy_roofline_rejects_bad_arguments_without_a_device():
    lib = _lib.lib()
    ms = ctypes.c_double()
    for args in ((0, 5, 19, 100, 10, 0), (0, 0, 0, 100, 10, 0), (0, 1, 19, 101, 10, 0), (0, 0, 19, 100, 0, 0)):
        assert lib.cells_copy_roofline(*args, ctypes.byref(ms)) == _lib.CELLS_E_INVALID
