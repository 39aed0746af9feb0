"""The C-ABI library: it loads, exports every function include/*.h declares,
its structures have the reference's layouts, and its host-side argument
checks behave like the reference's — all without touching a GPU."""
import ctypes as C
import glob
import os
import re

import pytest

import n_body_sim_pro_b200 as nb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        for m in re.finditer(r"N_BODY_SIM_PRO_CUDA_API\s+[^;{]*?\b(n_body_sim_pro_\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_the_plugin_functions():
    names = declared_functions()
    assert "n_body_sim_pro_gravity_compute_acceleration_cuda" in names
    assert "n_body_sim_pro_barnes_hut_compute_acceleration_cuda" in names
    assert len(names) >= 19


def test_library_loads_and_exports_every_declared_symbol():
    L = nb.library()
    for name in declared_functions():
        assert hasattr(L, name), name
    assert set(nb.EXPORTS) <= set(declared_functions())


def test_library_is_built_for_sm_100a_only():
    assert nb.library().n_body_sim_pro_cuda_architecture() == b"sm_100a"


def test_structure_layouts_match_the_reference():
    # include/n_body_sim_pro/core/particle_system.h:38-50 : size_t + 10 pointers
    assert C.sizeof(nb.View) == 8 + 10 * 8
    assert nb.View.masses.offset == 80
    # status.h:30-35 : enum, pointer, int, char[256]
    assert C.sizeof(nb.Error) == 4 + 4 + 8 + 4 + 256 + 4
    assert nb.Error.message.offset == 20
    assert C.sizeof(nb.Gravity) == 24
    assert C.sizeof(nb.BarnesHutStats) == 8 * 8
    assert C.sizeof(nb.DiagnosticsQuantities) == 11 * 8


def test_null_arguments_are_rejected_like_the_reference():
    """gravity.c:19-23 / barnes_hut.c:642-646: NULL view or gravity -> INVALID_ARGUMENT,
    checked before any device work."""
    L = nb.library()
    err = nb.Error()
    g = nb.gravity_init(1.0, 0.01)
    for fn in (L.n_body_sim_pro_gravity_compute_acceleration_cuda,
               L.n_body_sim_pro_barnes_hut_compute_acceleration_cuda):
        assert fn(None, C.byref(g), None, C.byref(err)) == nb.Status.INVALID_ARGUMENT
        assert b"must not be null" in err.message
        v = nb.View()
        assert fn(C.byref(v), None, None, None) == nb.Status.INVALID_ARGUMENT


def test_empty_barnes_hut_is_rejected():
    """barnes_hut.c:446-451: an empty system has no tree."""
    L = nb.library()
    err = nb.Error()
    v = nb.View()
    g = nb.gravity_init(1.0, 0.01)
    rc = L.n_body_sim_pro_barnes_hut_compute_acceleration_cuda(C.byref(v), C.byref(g), None,
                                                              C.byref(err))
    assert rc == nb.Status.INVALID_ARGUMENT
    assert b"empty system" in err.message


def test_invalid_gravity_is_rejected():
    L = nb.library()
    err = nb.Error()
    v = nb.View()
    g = nb.Gravity(1.0, 0.1, -1.0)
    rc = L.n_body_sim_pro_gravity_compute_acceleration_cuda(C.byref(v), C.byref(g), None,
                                                           C.byref(err))
    assert rc == nb.Status.INVALID_ARGUMENT


def test_context_setters_validate_without_a_device():
    L = nb.library()
    err = nb.Error()
    assert L.n_body_sim_pro_cuda_context_set_multipole_order(None, 1, C.byref(err)) == \
        nb.Status.INVALID_ARGUMENT
    assert L.n_body_sim_pro_cuda_context_set_opening(None, 1, C.byref(err)) == \
        nb.Status.INVALID_ARGUMENT
    assert L.n_body_sim_pro_cuda_context_set_relative_opening(None, 0.01, C.byref(err)) == \
        nb.Status.INVALID_ARGUMENT
    assert L.n_body_sim_pro_cuda_context_set_relative_source(None, 1, C.byref(err)) == \
        nb.Status.INVALID_ARGUMENT
    assert L.n_body_sim_pro_cuda_context_stats(None, None) != 0
    assert L.n_body_sim_pro_cuda_context_theta(None) == 0.0


@pytest.mark.skipif(os.path.exists("/dev/nvidia0"), reason="a GPU is present")
def test_no_cpu_fallback_without_a_gpu():
    """No device -> UNSUPPORTED_PLATFORM, never a silent CPU computation."""
    with pytest.raises(nb.CudaError) as e:
        nb.CudaContext()
    assert e.value.status == nb.Status.UNSUPPORTED_PLATFORM
    s = nb.ParticleSystem.zeros(4)
    s.m[:] = 1.0
    s.x[:] = [0, 1, 2, 3]
    with pytest.raises(nb.CudaError) as e:
        nb.n_body_sim_pro_gravity_compute_acceleration_cuda(s, nb.gravity_init(1.0, 0.01))
    assert e.value.status == nb.Status.UNSUPPORTED_PLATFORM
