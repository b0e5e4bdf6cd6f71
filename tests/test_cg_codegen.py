"""The model-specialised CG kernel is generated and NVRTC-compiled for sm_100a
at model load (no GPU needed to compile)."""
import ctypes

from sus2sh import _lib


def _info(path, use_float):
    lib = _lib.load()
    info = (ctypes.c_int * 5)()
    txt = ctypes.create_string_buffer(8192)
    rc = lib.sus2sh_cg_kernel_info(path.encode(), use_float, info, txt, 8192)
    return rc, list(info), txt.value.decode()


def test_l3k3_cg_kernel_compiles_without_spills(l3k3_path):
    rc, info, log = _info(l3k3_path, 1)
    assert rc == 0, log
    regs, spill, terms, ms, cubin = info
    assert 0 < regs <= 255 and spill == 0, log
    # 806 products: 606 forward terms + 200 fused terminal terms (x2) + 606 back terms (x2)
    assert terms == 606 + 2 * 200 + 2 * 606
    assert cubin > 0


def test_large_graph_stays_on_the_interpreter(l4k4_path):
    rc, info, log = _info(l4k4_path, 1)
    assert rc == -1
    assert "interpreter" in _lib.load().sus2sh_last_error().decode()
