"""The reference driver (src/MAIN.cpp, parser, util of adalbal/SpNS, compiled
unchanged) linked against libspns through the HIT forwarding unit, run on the
nine QA configurations of the reference.

Bar: the reference's own QA check (QA/check.sh) -- the "Final ..." lines of
stdout.0 identical to those of its 4-rank FFTW run -- plus every per-step report
line within the rounding of its printed digits.  The K41 tests build their
initial field as the 4-rank run does (SPNS_K41_RANKS=4).
"""
import glob
import json
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "spns_b200", "dropin", "_build", "spns_hit_qa")
QA = os.path.join(ROOT, "tests", "golden", "qa")
STEP_RE = re.compile(r"Time:\s*([-+0-9.eE]+),\s*iter:\s*(\d+),\s*Dt:\s*([-+0-9.eE]+),\s*Ek:\s*([-+0-9.eE]+),"
                     r"\s*Om:\s*([-+0-9.eE]+),\s*ReLambda:\s*([-+0-9.eE]+)")


def _stage(name, dst):
    """Working directory of one QA case: params plus its DATA files rebuilt from the fixtures."""
    src = os.path.join(QA, name)
    shutil.copyfile(os.path.join(src, "params"), os.path.join(dst, "params"))
    os.makedirs(os.path.join(dst, "DATA"), exist_ok=True)
    os.makedirs(os.path.join(dst, "OUTPUT"), exist_ok=True)
    params = open(os.path.join(src, "params")).read()
    for key in ("ASCII_Input_Filename", "Binary_Input_Filename"):
        m = re.search(rf"^{key}\s+(\S+)", params, re.M)
        if m:
            uvw = np.load(os.path.join(src, "init_uvw.npy"))
            path = os.path.join(dst, m.group(1))
            if key.startswith("ASCII"):
                rows = uvw.reshape(3, -1).T
                np.savetxt(path, rows, fmt="%.17g")
            else:
                uvw.astype("<f8").tofile(path)
    m = re.search(r"^InputEkFilename\s+(\S+)", params, re.M)
    if m:
        shutil.copyfile(os.path.join(src, "Forced_Energy_Cascade.dat"), os.path.join(dst, m.group(1)))


def _parse(stdout0):
    steps, final = [], {}
    for line in stdout0.splitlines():
        m = STEP_RE.search(line)
        if m:
            t, it, dt, ek, om, rl = m.groups()
            steps.append([float(t), int(it), float(dt), float(ek), float(om), float(rl)])
        elif line.startswith("Final "):
            k, v = line.split(":", 1)
            final[k.strip()] = v.strip()
    return steps, final


CASES = sorted(os.path.basename(p) for p in glob.glob(os.path.join(QA, "TEST_*")))


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_reference_driver_qa(name, tmp_path):
    if not os.path.exists(EXE):
        pytest.fail("drop-in driver not built (make -C spns_b200/dropin)")
    _stage(name, str(tmp_path))
    env = dict(os.environ, SPNS_K41_RANKS="4")
    r = subprocess.run([EXE, "params"], cwd=str(tmp_path), env=env, capture_output=True, timeout=120)
    out = r.stdout.decode(errors="replace") + r.stderr.decode(errors="replace")
    assert r.returncode == 0, out[-3000:]
    with open(os.path.join(str(tmp_path), "stdout.0"), errors="replace") as fh:
        steps, final = _parse(fh.read())
    ref = json.load(open(os.path.join(QA, name, "ref_steps.json")))
    ref_final = {k: v for k, v in ref["final"].items() if k in ("Final time-steps", "Final time", "Final energy", "Final ReLambda")}
    got_final = {k: final.get(k) for k in ref_final}
    assert got_final == ref_final
    assert len(steps) == len(ref["steps"])
    for g, e in zip(steps, ref["steps"]):
        assert g[1] == e[1]
        assert abs(g[0] - e[0]) <= 1.5e-6                       # Time %f
        for i in (2, 3, 4):                                     # Dt, Ek, Om %e (7 digits)
            assert abs(g[i] - e[i]) <= 1.5e-6 * abs(e[i]) + 1e-300
        assert abs(g[5] - e[5]) <= 1.5e-3                       # ReLambda %8.3f


@pytest.mark.gpu
def test_reference_driver_writes_invariant_spectra(tmp_path):
    """VelGradInv_Spectra 1 with an output frequency: the unchanged driver writes the
    per-frequency and final QG/QS/RG/RS/V2 files (src/MAIN.cpp:460-469, 497-503);
    the final ones equal the oracle's spectra after the same steps to the 6 digits
    the reference's writer prints."""
    import oracle as O
    from qa_util import load_case
    if not os.path.exists(EXE):
        pytest.fail("drop-in driver not built (make -C spns_b200/dropin)")
    name = "TEST_1_DHIT_DNS"
    _stage(name, str(tmp_path))
    p = tmp_path / "params"
    txt = re.sub(r"^Final_Time\s+\S+", "Final_Time\t0.1", p.read_text(), flags=re.M)
    p.write_text(txt + "\nVelGradInv_Spectra\t1\nVelGradInv_Spectra_Freq\t2\nSpectra_Folder\tOUTPUT\n")
    r = subprocess.run([EXE, "params"], cwd=str(tmp_path), capture_output=True, timeout=120)
    out = r.stdout.decode(errors="replace") + r.stderr.decode(errors="replace")
    assert r.returncode == 0, out[-3000:]
    with open(os.path.join(str(tmp_path), "stdout.0"), errors="replace") as fh:
        _, final = _parse(fh.read())
    nsteps = int(final["Final time-steps"])
    names = ("QG", "QS", "RG", "RS", "V2")
    for i in range(nsteps // 2):
        for nm in names:
            assert (tmp_path / "OUTPUT" / f"{nm}_{i:08d}.dat").exists()
    args, uvw, _ = load_case(name)
    ref = O.OracleHIT(args, file_uvw=uvw)
    for _ in range(nsteps):
        ref.New_Fractional_Step_Method()
    sp = ref.Recalculate_Invariants_Distribution()
    for c, nm in enumerate(names):
        rows = np.loadtxt(tmp_path / "OUTPUT" / f"{nm}.dat")
        assert rows.shape == (sp.shape[1], 2) and np.array_equal(rows[:, 0], np.arange(sp.shape[1]))
        m = np.abs(sp[c]) > 1e-6 * np.abs(sp[c]).max()
        assert np.max(np.abs(rows[m, 1] - sp[c][m]) / np.abs(sp[c][m])) < 2e-5, nm
