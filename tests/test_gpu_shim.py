"""The C++ drop-in header (include/dimgpu_reference_shim.hpp) inside the
reference's own time loop: oracle/_ref/shim_parity runs dim::advance_one_step
and dimgpu::advance_one_step / dimgpu::ResidentDim side by side in one
process and exits 0 only if every double of every step agrees."""
from __future__ import annotations

import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

EXE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "shim_parity")


@pytest.mark.skipif(not os.path.exists(EXE), reason="shim_parity is built only where the reference sources exist")
def test_reference_time_loop_with_drop_in_header():
    out = subprocess.run([EXE], capture_output=True, text=True, timeout=600)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "identical" in out.stdout


SM_EXE = os.path.join(os.path.dirname(EXE), "sm_shim_parity")


@pytest.mark.skipif(not os.path.exists(SM_EXE), reason="sm_shim_parity is built only where the reference sources exist")
def test_reference_single_material_step_with_drop_in_header():
    """advance_one_step<DIM, EOS> (no level set, one material) against
    dimgpu::sm_advance_one_step from include/dimgpu_sm_shim.hpp."""
    out = subprocess.run([SM_EXE], capture_output=True, text=True, timeout=600)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "identical" in out.stdout
