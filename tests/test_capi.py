"""The C-ABI library without a GPU: it loads, exports every function that
include/*.h declares, validates configurations, lays out the coefficient
buffer as otbl_layout.h says, and refuses to create a context when no CUDA
device is usable (no CPU fallback)."""
import ctypes
import os
import re

import numpy as np
import pytest

from opentbl_b200 import config, native, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


def _declared():
    names = set()
    for h in sorted(os.listdir(INCLUDE)):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, h)).read()
        text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
        text = re.sub(r"#define[^\n]*(\\\n[^\n]*)*", " ", text)
        for m in re.finditer(r"\b(otbl_[a-z0-9_]+)\s*\(", text):
            start = text.rfind("\n", 0, m.start())
            line = text[start + 1:m.start()]
            if line.strip().startswith(("static", "return")):
                continue
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_function():
    L = native.lib()
    decl = _declared()
    assert len(decl) >= 25, decl
    missing = [n for n in sorted(decl) if not hasattr(L, n)]
    assert not missing, missing


def test_library_is_built_for_sm100a_only():
    """The product library is compiled for sm_100a and nothing else."""
    from opentbl_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert os.path.exists(native.LIB_PATH)


def test_config_check():
    L = native.lib()
    good = native.make_config(config.TINY, 300.0, 10)
    assert L.otbl_config_check(ctypes.byref(good)) == 0
    for field, bad in (("nx", 3), ("ny", 2), ("nz", 2), ("xout", 0), ("xout", 99), ("re", -1.0),
                       ("precision", 2), ("precision", -1)):
        c = native.make_config(config.TINY, 300.0, 10)
        setattr(c, field, bad)
        assert L.otbl_config_check(ctypes.byref(c)) == 2, field
    mixed = native.make_config(config.TINY, 300.0, 10)
    mixed.precision = 1
    assert L.otbl_config_check(ctypes.byref(mixed)) == 0
    mixed.xpose_round = 1  # REAL4 transposes are an FP64-path mode
    assert L.otbl_config_check(ctypes.byref(mixed)) == 2
    assert L.otbl_config_check(None) == 1


def test_coefficient_layout_matches_header():
    """Offsets follow OTBL_COEF_LIST: each block starts where the previous
    one ends, with the lengths of include/otbl_layout.h."""
    cfg = config.C1
    off = native.coef_offsets(cfg)
    NX, NY, NZ2 = cfg.nx, cfg.ny, cfg.nz2
    text = open(os.path.join(INCLUDE, "otbl_layout.h")).read()
    block = text[text.index("#define OTBL_COEF_LIST"):text.index("/* scalar slots")]
    entries = re.findall(r"X\((\w+),\s*([^)]+(?:\)[^X\\]*?)?)\)", block)
    lengths = [(n, eval(l.strip(), {}, {"NX": NX, "NY": NY, "NZ2": NZ2})) for n, l in entries]
    assert [n for n, _ in lengths] == list(native.COEF_NAMES)
    cur = 0
    for n, ln in lengths:
        assert off[n] == cur, n
        cur += ln
    assert off["TOTAL"] == cur
    assert native.lib().otbl_coef_count(cfg.nx, cfg.ny, cfg.nz) == cur


def test_no_device_means_no_context():
    """Without a usable CUDA device the context is refused with
    OTBL_ERR_NODEV: nothing runs on the CPU instead."""
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    cfg = config.TINY
    init = synth.make_initial(cfg)
    coef = native.coef_compute(cfg, init["re"], init["xout"], init["y"], init["u0"])
    c = native.make_config(cfg, init["re"], init["xout"])
    h = ctypes.c_void_p()
    st = native.lib().otbl_ctx_create(ctypes.byref(c), native.dptr(coef), 0, ctypes.byref(h))
    assert st == 6 and not h.value
    from opentbl_b200 import Box
    from opentbl_b200.native import OtblError
    with pytest.raises(OtblError):
        Box(cfg, init, coef)


def test_null_context_is_an_argument_error():
    L = native.lib()
    for name in ("otbl_rhsp", "otbl_substep"):
        assert getattr(L, name)(None, 1, 1) == 1
    for name in ("otbl_outflow_correction", "otbl_boun", "otbl_genflu", "otbl_sync"):
        assert getattr(L, name)(None) == 1
    assert L.otbl_pois(None, 1) == 1
    assert L.otbl_advance(None, 1) == 1
    assert L.otbl_launch_count(None) == 0
    assert L.otbl_last_error(None) == b"null context"


def test_coefficients_are_host_only_and_deterministic():
    cfg = config.SMALL
    init = synth.make_initial(cfg)
    a = native.coef_compute(cfg, init["re"], init["xout"], init["y"], init["u0"])
    b = native.coef_compute(cfg, init["re"], init["xout"], init["y"], init["u0"])
    assert np.array_equal(a, b) and np.isfinite(a).all()


def _driver():
    from opentbl_b200 import build
    if not os.path.exists(build.DRIVER):
        build.build_driver()
    return build.DRIVER


def test_c_driver_without_gpu():
    """csrc/otbl_driver.c drives the time loop through include/otbl.h alone.
    Here (no GPU) it computes the coefficients and stops at context creation
    with OTBL_ERR_NODEV (exit status 3): no CPU fallback."""
    import subprocess
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present: the GPU test runs the driver")
    r = subprocess.run([_driver()], capture_output=True, text=True, timeout=120)
    assert r.returncode == 3, (r.returncode, r.stdout, r.stderr)
    assert "OTBL_ERR_NODEV" in r.stdout


@pytest.mark.gpu
def test_c_driver_on_gpu():
    """The C driver on the GPU: three RK3 steps through the context API and
    through the array surface on caller-owned arrays, bit-identical."""
    import subprocess
    r = subprocess.run([_driver(), "33", "41", "32", "3"], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert "bit-identical" in r.stdout
    steps = [ln for ln in r.stdout.splitlines() if ln.startswith("step ")]
    assert len(steps) == 3
