"""The C ABI library: it loads, exports every entry point the header declares,
its structs match the header, and it fails loudly without a GPU."""
import ctypes as C
import os
import re
import subprocess

import pytest

from matter_tests_b200 import abi, gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "matter_gpu.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mtr_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(gpu.LIB_PATH):
        from matter_tests_b200 import build
        build.build()
    return gpu.load_library()


def test_header_declarations_match_binding():
    assert declared_functions() == sorted(gpu.EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", gpu.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (mtr_\w+)", out))
    missing = [f for f in declared_functions() if f not in exported]
    assert not missing, missing


def test_struct_layouts_match_the_c_compiler(tmp_path):
    prog = tmp_path / "sz.c"
    prog.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "matter_gpu.h"\n'
                    'int main(void){printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(mtr_params), sizeof(mtr_plate),'
                    ' sizeof(mtr_object), sizeof(mtr_clock), offsetof(mtr_params, fps), offsetof(mtr_params, mu_2),'
                    ' offsetof(mtr_plate, load_factor)); return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(prog), "-o", str(exe)], check=True)
    vals = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert vals == [C.sizeof(abi.MtrParams), C.sizeof(abi.MtrPlate), C.sizeof(abi.MtrObject), C.sizeof(abi.MtrClock),
                    abi.MtrParams.fps.offset, abi.MtrParams.mu_2.offset, abi.MtrPlate.load_factor.offset]


def test_enums_follow_reference_numbering():
    # tools.hpp:53-57
    assert (abi.PlateType.top, abi.PlateType.back) == (0, 5)
    assert (abi.PlasticModel.NoPlasticity, abi.PlasticModel.DPMui, abi.PlasticModel.Snow) == (0, 8, 10)
    assert (abi.HardeningLaw.NoHard, abi.HardeningLaw.SinhImpl) == (0, 4)
    assert (abi.BC.NoSlip, abi.BC.SlipStick, abi.BC.SlipFree) == (0, 1, 2)


def test_invalid_parameters_are_rejected(lib):
    p = abi.default_params(3, 2)
    h = C.c_void_p()
    p.dim = 4
    assert lib.mtr_ctx_create(C.byref(p), 0, C.byref(h)) == abi.MTR_ERR_INVALID
    p = abi.default_params(3, 2)
    p.elastic_model = abi.ElasticModel.NeoHookean
    p.plastic_model = abi.PlasticModel.DP  # simulation.cpp:80-84 refuses this combination
    assert lib.mtr_ctx_create(C.byref(p), 0, C.byref(h)) == abi.MTR_ERR_INVALID
    assert b"Hencky" in lib.mtr_last_error()
    p = abi.default_params(3, 2)
    p.pbc, p.use_mibf = 1, 1  # pbc.cpp copies x, v, F, B only: no friction field for the copies
    assert lib.mtr_ctx_create(C.byref(p), 0, C.byref(h)) == abi.MTR_ERR_INVALID
    p = abi.default_params(3, 2)
    p.pbc, p.L[2] = 1, 0.0
    assert lib.mtr_ctx_create(C.byref(p), 0, C.byref(h)) == abi.MTR_ERR_INVALID


def test_null_and_state_errors(lib):
    assert lib.mtr_step(None, 1) == abi.MTR_ERR_INVALID
    assert lib.mtr_download(None, None, None, None, None, None) == abi.MTR_ERR_STATE
    lib.mtr_ctx_destroy(None)


def test_no_device_fails_loudly(lib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is visible")
    except ImportError:
        pass
    p = abi.default_params(3, 2)
    p.dx, p.particle_mass, p.particle_volume = 0.01, 1e-3, 1e-6
    h = C.c_void_p()
    assert lib.mtr_ctx_create(C.byref(p), 0, C.byref(h)) == abi.MTR_ERR_NO_DEVICE
    with pytest.raises(gpu.MtrFailure):
        gpu.GpuSim(p)
