"""The reference solver itself as a second checker of the oracle.

oracle/Makefile, target `ref`, compiles src/*.cpp of adalbal/SpNS unchanged where
they lie, against the single-process MPI and FFTW stand-ins of oracle/ref_shim/
(whose transforms are the oracle's FFT), into oracle/_ref/.  Then:

- its QA build reproduces the reference's own logged runs that start from a file
  (QA TEST_1 and TEST_2): the Final lines identical and every per-step line within
  the digits printed.  The other QA cases start from K41 fields drawn per rank of a
  4-rank MPI run, which a one-process build draws differently;
- the fields it writes after the same steps equal the oracle's to 1e-12 (relative
  L2) in all nine QA configurations (DNS, LES, spectrum forcing, rotation, the
  self-adaptive step, conjugate correction, non-cubic boxes, Re_lambda control) and
  one combination of their options: the oracle is pinned to the reference code
  itself, beyond the 7 digits of the logs.

Skipped where oracle/_ref/ was not built (no reference checkout at build time).
"""
import os
import re
import subprocess

import numpy as np
import pytest

from test_gpu_dropin import CASES, _parse, _set_param, _stage
from qa_util import load_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_QA = os.path.join(ROOT, "oracle", "_ref", "spns_ref_qa")
REF = os.path.join(ROOT, "oracle", "_ref", "spns_ref")

needs_ref = pytest.mark.skipif(not (os.path.exists(REF) and os.path.exists(REF_QA)),
                               reason="oracle/_ref not built (make -C oracle ref REF=<reference>/src)")


def _run(exe, cwd, params="params"):
    env = dict(os.environ, OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "4"))
    r = subprocess.run([exe, params], cwd=cwd, env=env, capture_output=True, timeout=600)
    out = r.stdout.decode(errors="replace") + r.stderr.decode(errors="replace")
    assert r.returncode == 0, out[-3000:]
    return out


@needs_ref
@pytest.mark.parametrize("name", ["TEST_1_DHIT_DNS", "TEST_2_DHIT_SMAGORINSKY"])
def test_reference_build_reproduces_its_logs(name, tmp_path):
    _stage(name, str(tmp_path))
    _run(REF_QA, str(tmp_path))
    with open(os.path.join(str(tmp_path), "stdout.0"), errors="replace") as fh:
        steps, final = _parse(fh.read())
    _, _, ref = load_case(name)
    for k in ("Final time-steps", "Final time", "Final energy", "Final ReLambda"):
        assert final.get(k) == ref["final"][k], k
    assert len(steps) == len(ref["steps"])
    for g, e in zip(steps, ref["steps"]):
        assert g[1] == e[1]
        assert abs(g[0] - e[0]) <= 1.5e-6
        for i in (2, 3, 4):
            assert abs(g[i] - e[i]) <= 1.5e-6 * abs(e[i])
        assert abs(g[5] - e[5]) <= 1.5e-3


def _actual(m, L):
    """Grid points of the true box along one axis (src/HIT_LES.h:31-36)."""
    return m // L if m % 2 == 0 else (m - 1) // L + 1


VARIANTS = {name: (name, ()) for name in CASES}
VARIANTS["TEST_1+rotating-selfadaptive-conj"] = ("TEST_1_DHIT_DNS", (
    ("omega_x", 1.5), ("omega_y", -2.1), ("omega_z", 3.0), ("SelfAdaptiveTimestep", 1), ("ComplexConjugateCorrection", 1)))


@needs_ref
@pytest.mark.parametrize("variant", list(VARIANTS))
def test_oracle_matches_reference_fields(variant, tmp_path, oracle_lib):
    """All nine QA configurations (and one combination of their options), shortened to
    Final_Time 0.03 (0.012 for the non-cubic boxes): 2 to 8 steps.  A K41 initial field is drawn by the one process as the oracle draws
    it with one rank.  The reference writes its physical field (the true box of a
    non-cubic domain, src/HIT_LES_output.cpp:66-115) and its spectrum after the loop."""
    import oracle as O
    from gpu_util import rel_l2
    from spns_b200 import driver
    from spns_b200.params import derive_hit_args, read_params
    name, extra = VARIANTS[variant]
    _stage(name, str(tmp_path))
    p = tmp_path / "params"
    txt = p.read_text()
    final_time = "0.012" if "NONCUBIC" in name else "0.03"      # the non-cubic grids are 288 x 144 x 96
    for k, v in (("Final_Time", final_time), ("Velocity_Physical", 1), ("Energy_Cascade", 1),
                 ("Spectra_Folder", "OUTPUT")) + extra:
        txt = _set_param(txt, k, v)
    p.write_text(txt)
    out = _run(REF, str(tmp_path))
    nsteps = int(re.search(r"Final time-steps:\s*(\d+)", out).group(1))
    assert nsteps >= 2

    args = derive_hit_args(read_params(str(p)), base_dir=str(tmp_path))
    _, uvw, _ = load_case(name)
    h = O.OracleHIT(args, uvw, k41_ranks=1)
    done = []
    driver.run(h, args, qa_report=False, on_step=done.append)
    assert len(done) == nsteps
    assert abs(h.gettime() - float(re.search(r"Final time:\s*(\S+)", out).group(1))) < 1e-6
    h.Recalculate_Velocity_Antitransform()
    Po = h.get_physical()
    Eo = h.Recalculate_Energy_Cascade()
    am = (_actual(args.Mx, args.Lx), _actual(args.My, args.Ly), _actual(args.Mz, args.Lz))
    Po = Po[:, :am[0], :am[1], :am[2]]
    od = tmp_path / "OUTPUT"
    Pf = np.fromfile(od / "Velocity.bin", dtype="<f8").reshape(Po.shape)
    err = rel_l2(Pf, Po)
    print(f"{variant}: {nsteps} steps, physical field rel L2 {err:.2e}")
    assert err < 1e-12
    rows = np.loadtxt(od / "Energy_Cascade.dat")
    assert rows.shape == (Eo.size, 2)
    m = Eo > 1e-12 * Eo.max()
    assert np.max(np.abs(rows[m, 1] - Eo[m]) / Eo[m]) < 1e-5        # 6 printed digits
