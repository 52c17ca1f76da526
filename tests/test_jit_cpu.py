"""The run-time compiled rescoring module (no GPU needed): the embedded source is the header the
library build compiles, and it compiles under NVRTC for sm_100a with each entry point's
geometry constants, as the library does at its first learned call for a geometry."""
import ctypes
import ctypes.util

import pytest

from conftest import REPO

CSRC = REPO / "pseudoctimaging_b200" / "csrc"
INC = REPO / "pseudoctimaging_b200" / "_build" / "pct_rescore_src.inc"


def _nvrtc():
    for name in ("libnvrtc.so.12", "libnvrtc.so", ctypes.util.find_library("nvrtc")):
        if not name:
            continue
        try:
            return ctypes.CDLL(name)
        except OSError:
            continue
    pytest.skip("NVRTC not installed")


def _compile(lib, src: bytes, opts: list[bytes]) -> tuple[int, str, int]:
    prog = ctypes.c_void_p()
    assert lib.nvrtcCreateProgram(ctypes.byref(prog), src, b"pct_rescore.cuh", 0, None, None) == 0
    arr = (ctypes.c_char_p * len(opts))(*opts)
    rc = lib.nvrtcCompileProgram(prog, len(opts), arr)
    size = ctypes.c_size_t()
    lib.nvrtcGetProgramLogSize(prog, ctypes.byref(size))
    log = ctypes.create_string_buffer(max(size.value, 1))
    lib.nvrtcGetProgramLog(prog, log)
    cubin = ctypes.c_size_t(0)
    if rc == 0:
        assert lib.nvrtcGetCUBINSize(prog, ctypes.byref(cubin)) == 0
    lib.nvrtcDestroyProgram(ctypes.byref(prog))
    return rc, log.value.decode(errors="replace"), cubin.value


def test_embedded_source_is_the_header():
    text = (CSRC / "pct_rescore.cuh").read_text()
    inc = INC.read_text()
    start = inc.index('R"pct_src(') + len('R"pct_src(')
    end = inc.rindex(')pct_src"')
    assert inc[start:end] == text


@pytest.mark.parametrize("nx,pitch,hw", [(222, 222, 5), (222, 224, 5), (64, 64, 4), (17, 20, 3)])
def test_rescore_module_compiles_for_sm100a(nx, pitch, hw):
    lib = _nvrtc()
    src = (CSRC / "pct_rescore.cuh").read_bytes()
    opts = [b"-DPCT_RS_JIT", b"-DPCT_RS_NX=%d" % nx, b"-DPCT_RS_PITCH=%d" % pitch,
            b"-DPCT_RS_HW=%d" % hw, b"--gpu-architecture=sm_100a", b"-std=c++17"]
    rc, log, cubin = _compile(lib, src, opts)
    assert rc == 0, log
    assert cubin > 0
