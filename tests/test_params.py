"""Driver derivations of src/MAIN.cpp:174-318 (host logic, no GPU)."""
import os

import pytest

from spns_b200.params import read_params, derive_hit_args, ParamsError
from qa_util import GOLDEN


def test_cubic_dns():
    a = derive_hit_args(read_params(os.path.join(GOLDEN, "TEST_1_DHIT_DNS", "params")))
    assert (a.Nx, a.Mx, a.Lx, a.isNotCubic, a.isLES, a.isReLambda) == (32, 48, 1, False, False, False)
    assert a.isInitialFieldFromASCIIFile and a.C_At == 0.5 and a.nu == 3.283e-4


def test_noncubic_expansion():
    # Lx,Ly,Lz = 1,2,3 -> lcm 6 -> factors (6,3,2); N and M expanded (src/MAIN.cpp:216-253)
    a = derive_hit_args(read_params(os.path.join(GOLDEN, "TEST_7_DHIT_DNS_NONCUBIC", "params")))
    assert (a.Lx, a.Ly, a.Lz) == (6, 3, 2)
    assert (a.Nx, a.Ny, a.Nz) == (192, 96, 64)
    assert (a.Mx, a.My, a.Mz) == (288, 144, 96)
    assert a.isNotCubic


def test_les_rotating_relambda():
    a = derive_hit_args(read_params(os.path.join(GOLDEN, "TEST_8_DHIT_SMAGORINSKY_ROTATING_NONCUBIC", "params")))
    assert a.isLES and a.isRotating and a.isReLambda and a.isReLambda_iter and a.ReLambda_Freq == 1
    assert (a.omega_x, a.omega_y, a.omega_z) == (1.5, -2.1, 3.0)


def test_both_nu_and_relambda_rejected(tmp_path):
    p = tmp_path / "params"
    p.write_text("Nx 32\nNy 32\nNz 32\nnu 1e-3\nReynolds_lambda 100\nFinal_Time 1\n")
    with pytest.raises(ParamsError):
        derive_hit_args(read_params(str(p)))


def test_missing_required(tmp_path):
    p = tmp_path / "params"
    p.write_text("Nx 32\nNy 32\nnu 1e-3\nFinal_Time 1\n")
    with pytest.raises(ParamsError):
        read_params(str(p))
