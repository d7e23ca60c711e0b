"""The C ABI: every entry point declared in include/pdgpu.h is exported by
the built library and bound by peridem_b200.api with a signature; no
compute call is made (no GPU needed)."""
import ctypes
import os
import re

import pytest

from peridem_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "pdgpu.h")).read()
    return sorted(set(re.findall(r"PDGPU_API\s+(?:int|void)\s+(pdgpu_\w+)\s*\(", text)))


def test_header_declares_the_abi():
    names = _declared()
    assert len(names) >= 30
    assert "pdgpu_step" in names and "pdgpu_create" in names


def test_binding_covers_every_declared_entry_point():
    assert sorted(api.SIGNATURES) == _declared()


@pytest.mark.skipif(not os.path.exists(api.LIB_PATH), reason="libpdgpu.so not built")
def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(api.LIB_PATH)
    for name in _declared():
        assert hasattr(lib, name), name


@pytest.mark.skipif(not os.path.exists(api.LIB_PATH), reason="libpdgpu.so not built")
def test_create_fails_loudly_without_a_b200():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    from peridem_b200 import scene as scn
    from peridem_b200.model import GpuDEMModel
    sc = scn.build_scene(scn.two_particle(h_div=4, nt=10))
    with pytest.raises(api.PdgpuError):
        GpuDEMModel(sc)


def test_struct_layouts_match_header():
    # sizes of the ABI structs as the C compiler lays them out
    assert ctypes.sizeof(api.Particle) == 3 * 8 + 6 * 4 + 6 * 8 + 6 * 8
    assert ctypes.sizeof(api.BcSet) == 4 * 4 + 6 * 8


def _null_args(argtypes):
    out = []
    for t in argtypes:
        if t in (ctypes.c_float, ctypes.c_double):
            out.append(t(0.0))
        elif t in (ctypes.c_int32, ctypes.c_int64, ctypes.c_uint8, ctypes.c_size_t, ctypes.c_int,
                   ctypes.c_uint32, ctypes.c_uint64):
            out.append(t(0))
        else:  # every pointer: NULL
            out.append(None)
    return out


@pytest.mark.skipif(not os.path.exists(api.LIB_PATH), reason="libpdgpu.so not built")
def test_every_entry_point_rejects_null_arguments_before_device_work():
    """The error behaviour of the interface: a NULL context or NULL buffer is
    PDGPU_ERR_ARG, returned before any CUDA call (so this runs without a
    GPU); pdgpu_destroy(NULL) is a no-op."""
    L = api.lib()
    skip = {"pdgpu_device_check"}  # reports on the device, takes no pointer it needs
    for name, argtypes in sorted(api.SIGNATURES.items()):
        if name in skip:
            continue
        rc = getattr(L, name)(*_null_args(argtypes))
        if name == "pdgpu_destroy":
            assert rc is None
        else:
            assert rc == -1, (name, rc)  # PDGPU_ERR_ARG


@pytest.mark.skipif(not os.path.exists(api.LIB_PATH), reason="libpdgpu.so not built")
def test_device_check_reports_no_device_without_a_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    L = api.lib()
    buf = ctypes.create_string_buffer(128)
    assert L.pdgpu_device_check(0, buf, 128) == -7  # PDGPU_ERR_NODEVICE
    assert buf.value
