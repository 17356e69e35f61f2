"""The C-ABI library on a machine without a GPU.

The library must load, export every entry point include/g6b200.h declares,
answer g6_npipes_() without touching a device (kira asks during
configuration, kira_config.C:62), and fail loudly -- never fall back to a
CPU computation -- when no GPU is present.
"""
import ctypes
import os
import re
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
HEADER = os.path.join(REPO, "include", "g6b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*([a-z_0-9]+)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if n.startswith(("g6", "g6b200"))))


def test_header_declares_the_reference_abi():
    names = declared_functions()
    # include/grape6.h:16-104 of the reference
    ref = ["g6_set_tunit_", "g6_set_xunit_", "g6_open_", "g6_close_", "g6_open_special",
           "g6_open_special2", "g6_reset_", "g6_reset_fofpga_", "g6_npipes_", "g6_set_ti_",
           "g6_set_j_particle_", "g6calc_firsthalf_", "g6calc_lasthalf_", "g6calc_lasthalf2_",
           "g6_read_neighbour_list_", "g6_read_neighbour_list_old_", "g6_get_neighbour_list_",
           "g6_initialize_jp_buffer_", "g6_flush_jp_buffer_"]
    for r in ref:
        assert r in names, r


def test_library_exports_every_declared_symbol():
    from starlab_b200 import LIB_PATH
    lib = ctypes.CDLL(LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], stdout=subprocess.PIPE, text=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if " T " in l)
    assert set(declared_functions()) <= exported


def test_library_is_sm100a_only():
    from starlab_b200 import LIB_PATH
    out = subprocess.run(["cuobjdump", "--list-elf", LIB_PATH], stdout=subprocess.PIPE,
                         stderr=subprocess.STDOUT, text=True).stdout
    assert "sm_100a" in out
    assert not re.search(r"sm_(?!100a)\d+", out), out


def test_npipes_without_device():
    code = ("import ctypes,sys; lib=ctypes.CDLL(sys.argv[1]); print(lib.g6_npipes_())")
    from starlab_b200 import LIB_PATH
    env = dict(os.environ, G6B200_NPIPES="300")
    r = subprocess.run([sys.executable, "-c", code, LIB_PATH], env=env, stdout=subprocess.PIPE, text=True)
    assert r.stdout.strip() == "300"
    env.pop("G6B200_NPIPES")
    r = subprocess.run([sys.executable, "-c", code, LIB_PATH], env=env, stdout=subprocess.PIPE, text=True)
    assert r.stdout.strip() == "256"


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU behaviour")
def test_fails_loudly_without_gpu():
    from starlab_b200 import G6Engine, G6Error
    eng = G6Engine(cluster_id=900)
    with pytest.raises(G6Error):
        eng.open()
    with pytest.raises(G6Error):
        eng.set_j_particles(0.0, np.ones(4), np.zeros((4, 3)), np.zeros((4, 3)), np.zeros((4, 3)),
                            np.eye(4, 3))
    eng.calc_firsthalf(4, np.arange(4), np.eye(4, 3), np.zeros((4, 3)), 1e-4)
    with pytest.raises(G6Error):
        eng.calc_lasthalf2()


def test_config_validation():
    from starlab_b200 import G6Engine
    eng = G6Engine(cluster_id=901)
    eng.set_config(32, 2, 8, 1, 4)
    for bad in [(16, 1, 8, 1, 1), (8, 2, 8, 1, 1), (32, 1, 3, 1, 1), (32, 1, 8, 3, 1), (32, 1, 8, 1, 0)]:
        with pytest.raises(ValueError):
            eng.set_config(*bad)
    eng.set_config(0)


def test_precision_and_npipes_setters():
    from starlab_b200 import G6Engine
    eng = G6Engine(cluster_id=902, precision="mixed", npipes=1024)
    assert eng.precision() == 1 and eng.npipes() == 1024
    eng.set_precision("fp64")
    assert eng.precision() == 0
    with pytest.raises(ValueError):
        eng.set_npipes(0)
