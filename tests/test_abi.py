"""The C-ABI library: it loads, exports every entry point include/gg_step.h
declares, parses parameters.xml, and fails cleanly without a GPU."""
import ctypes
import os
import re

import pytest

from gragles2d_b200 import build, gg

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
HEADER = os.path.join(ROOT, "include", "gg_step.h")
GOLDEN = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def lib():
    build.build()
    return gg.load_library()


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(gg_\w+)\s*\(", text, re.M)))


def test_header_declares_the_python_export_list():
    assert declared_functions() == sorted(gg.EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_params_default_and_xml(lib):
    s = gg.Settings(os.path.join(GOLDEN, "mob_v30", "mob_v30.xml"))
    assert s.p.struct_size == ctypes.sizeof(gg.Params)
    assert s.p.microstructure_gen_mode == 4
    assert s.p.number_of_timesteps == 20
    assert s.p.domain_border_size == 7
    assert s.p.is_isotropic_network == 0
    assert s.p.use_mobility_model == 1
    assert s.p.triple_point_drag == 5.0
    assert s.p.read_from_filename == b"mob_v30.bin"
    assert s.p.theta_ref_deg == 15.0 and s.p.gamma_hagb == 1.0 and s.p.m_hagb == 1.0


def test_params_xml_missing_file(lib):
    p = gg.Params()
    assert lib.gg_params_from_xml(b"/nonexistent/parameters.xml", ctypes.byref(p)) == 3


def test_create_rejects_unsupported_settings(lib):
    s = gg.Settings(os.path.join(GOLDEN, "iso_v20", "iso_v20.xml"), convolution_mode=0)
    with pytest.raises(gg.GGError) as e:
        gg.GrainHandler(s)
    assert e.value.code == 1 and "Gaussian" in str(e.value)


def test_stage_calls_before_load_fail_with_state_error(lib):
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("covered on the GPU")
    except ImportError:
        pass
    s = gg.Settings(os.path.join(GOLDEN, "iso_v20", "iso_v20.xml"))
    with pytest.raises(gg.GGError) as e:
        gg.GrainHandler(s)  # no device here: a clean CUDA error, no crash
    assert e.value.code == 2
