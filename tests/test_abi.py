"""The C-ABI library loads and exports every entry point include/dimgpu.h
declares (no device work: this runs on CPU-only machines)."""
from __future__ import annotations

import ctypes as C
import os
import re

import pytest

from diffuse_vs_gfm_mms_b200 import abi, native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "dimgpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dimgpu_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(native.LIB_PATH):
        from diffuse_vs_gfm_mms_b200 import build
        build.build()
    return native.lib()


def test_header_declares_the_api():
    syms = declared_symbols()
    for s in ("dimgpu_create", "dimgpu_step", "dimgpu_steps", "dimgpu_compute_dt_cfl",
              "dimgpu_sweep_direction", "dimgpu_apply_boundary_conditions", "dimgpu_advance_one_step"):
        assert s in syms


def test_library_exports_every_declared_symbol(lib):
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_signatures_cover_the_header():
    assert set(declared_symbols()) <= set(native.SIGNATURES)


def test_struct_layout_matches_header(tmp_path):
    """ctypes offsets == the C compiler's offsets for every descriptor field."""
    import subprocess
    fields = [f for f, _ in abi.Desc._fields_]
    src = tmp_path / "layout.c"
    body = "".join(f'printf("%zu ", offsetof(dimgpu_desc, {f}));' for f in fields)
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "dimgpu.h"\n'
                   f'int main(void){{ {body} printf("%zu %zu", sizeof(dimgpu_desc), sizeof(dimgpu_material));'
                   ' return 0; }\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", f"-I{os.path.join(ROOT, 'include')}", str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    want = [getattr(abi.Desc, f).offset for f in fields] + [C.sizeof(abi.Desc), C.sizeof(abi.Material)]
    assert got == want


def test_components():
    d = abi.make_desc(3, [4, 4, 4], [1, 1, 1], [("ideal_gas", 1.4, 0), ("ideal_gas", 1.6, 0)])
    assert d.nvar == 7 and d.ncell == 64


def test_slab_creator_refusals(lib):
    """dimgpu_slabs_create refuses, before touching a device, what the slab
    decomposition does not cover: 1D grids, the unsplit update, the Euler
    model, and slabs thinner than three planes."""
    import ctypes as C

    def create(d, n):
        h = C.c_void_p()
        devs = (C.c_int * n)(*([0] * n))
        return lib.dimgpu_slabs_create(C.byref(d), n, devs, C.byref(h)), h

    mats = [("ideal_gas", 1.4, 0), ("stiffened_gas", 4.4, 6e8)]
    rc, h = create(abi.make_desc(1, [64], [1 / 64], mats), 2)
    assert rc == abi.E_UNSUPPORTED and not h.value
    d = abi.make_desc(2, [16, 16], [1 / 16, 1 / 16], mats)
    d.time_update = abi.TIME_UNSPLIT
    assert create(d, 2)[0] == abi.E_UNSUPPORTED
    d = abi.make_desc(2, [16, 16], [1 / 16, 1 / 16], mats)
    d.model = abi.MODEL_EULER
    assert create(d, 2)[0] == abi.E_UNSUPPORTED
    d = abi.make_desc(3, [8, 8, 11], [1 / 8] * 3, mats)
    assert create(d, 4)[0] == abi.E_INVALID_ARG
    assert create(d, 0)[0] == abi.E_INVALID_ARG


def test_every_struct_layout_matches_header(tmp_path):
    """ctypes field offsets and sizes == the C compiler's for every struct
    the header passes by pointer (server configuration and counters,
    initial-condition parameters, phase times)."""
    import subprocess
    pairs = [(abi.PhaseTimes, "dimgpu_phase_times"), (abi.ServerConfig, "dimgpu_server_config"),
             (abi.ServerCounters, "dimgpu_server_counters"), (abi.ShockBubbleIC, "dimgpu_ic_shock_bubble"),
             (abi.BubbleIC, "dimgpu_ic_bubble"), (abi.BubbleCloudIC, "dimgpu_ic_bubble_cloud")]
    body, want = "", []
    for cls, cname in pairs:
        for f, _ in cls._fields_:
            body += f'printf("%zu ", offsetof({cname}, {f}));'
            want.append(getattr(cls, f).offset)
        body += f'printf("%zu ", sizeof({cname}));'
        want.append(C.sizeof(cls))
    src = tmp_path / "layout2.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "dimgpu.h"\n'
                   f'int main(void){{ {body} return 0; }}\n')
    exe = tmp_path / "layout2"
    subprocess.run(["gcc", f"-I{os.path.join(ROOT, 'include')}", str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert got == want
