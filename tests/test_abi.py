"""The C-ABI library loads and exports every function include/colvillea_b200.h
declares (no device calls: this runs without a GPU)."""
import ctypes
import re

from colvillea_b200 import _native


def declared_functions():
    text = open(_native.HEADER).read()
    return sorted(set(re.findall(r"\b(?:cl_status|void)\s+(cl_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for required in ("cl_integrator_create", "cl_integrator_destroy", "cl_build_meshes", "cl_build_instances",
                     "cl_build_materials", "cl_build_emitters", "cl_update_camera", "cl_render", "cl_readback_film",
                     "cl_readback_film_stats", "cl_resize", "cl_reset_iteration", "cl_get_stats", "cl_last_error"):
        assert required in names


def test_library_exports_every_declared_symbol(native):
    L = ctypes.CDLL(native.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    assert set(declared_functions()) == set(native._SIGS), "ctypes signatures out of sync with the header"


def test_library_is_built_for_sm100a():
    """The build compiles SASS for sm_100a only; the GPU tests also check the
    loaded kernels' binaryVersion through cl_unit_binary_version."""
    from colvillea_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_errors_without_crashing(native):
    L = native.lib()
    # invalid arguments are reported, never fatal
    assert L.cl_render(None, 1) == native.CL_ERR_INVALID_ARG
    assert "null" in native.last_error()
    h = ctypes.c_void_p()
    assert L.cl_integrator_create(99, 4, 4, None, ctypes.byref(h)) == native.CL_ERR_INVALID_ARG
    assert L.cl_unit_bsdf_eval(7, None, None, None, None, 1) == native.CL_ERR_INVALID_ARG
