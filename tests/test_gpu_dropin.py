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


def _set_param(txt, key, value):
    """Sets `key value` in a parameters file text (uncommenting or appending the line)."""
    pat = re.compile(rf"^#?\s*{key}\s+\S+.*$", re.M)
    if pat.search(txt):
        return pat.sub(f"{key}\t{value}", txt, count=1)
    return txt + f"\n{key}\t{value}\n"


@pytest.mark.gpu
def test_reference_driver_writes_fields_and_spectra(tmp_path):
    """Velocity_Physical / Velocity_Fourier / Energy_Cascade outputs of the unchanged driver
    (src/MAIN.cpp:452-484, 492-515; writers src/HIT_LES_output.cpp:8-115 and the
    "K<TAB>Ek" file of src/HIT_LES.cpp:1180-1187), against the oracle after the same
    steps; then the written physical field is read back as an initial field
    (Binary_Input_Filename, src/HIT_LES.cpp:618-686, 738-763) and reproduces the state."""
    import oracle as O
    from qa_util import load_case
    from gpu_util import rel_l2
    from spns_b200.params import read_params, derive_hit_args
    if not os.path.exists(EXE):
        pytest.fail("drop-in driver not built (make -C spns_b200/dropin)")
    name = "TEST_1_DHIT_DNS"
    _stage(name, str(tmp_path))
    p = tmp_path / "params"
    txt = p.read_text()
    for k, v in (("Final_Time", "0.05"), ("Velocity_Physical", 1), ("Velocity_Fourier", 1), ("Energy_Cascade", 1),
                 ("Velocity_Phys_Freq", 2), ("Velocity_Four_Freq", 2), ("Energy_Cascade_Freq", 2),
                 ("Spectra_Folder", "OUTPUT")):
        txt = _set_param(txt, k, v)
    p.write_text(txt)
    r = subprocess.run([EXE, "params"], cwd=str(tmp_path), capture_output=True, timeout=120)
    out = r.stdout.decode(errors="replace") + r.stderr.decode(errors="replace")
    assert r.returncode == 0, out[-3000:]
    with open(os.path.join(str(tmp_path), "stdout.0"), errors="replace") as fh:
        _, final = _parse(fh.read())
    nsteps = int(final["Final time-steps"])
    assert nsteps >= 3
    od = tmp_path / "OUTPUT"
    # per-frequency files after step n (the driver's counter, src/MAIN.cpp:436): physical when
    # n % 2 == 0, Fourier and spectra when (n+1) % 2 == 0
    assert len(list(od.glob("Velocity_0*.bin"))) == nsteps // 2
    assert len(list(od.glob("Velocity_Fourier_0*.bin"))) == (nsteps + 1) // 2
    assert len(list(od.glob("Energy_Cascade_0*.dat"))) == (nsteps + 1) // 2

    args, uvw, _ = load_case(name)
    ref = O.OracleHIT(args, file_uvw=uvw)
    for _ in range(nsteps):
        ref.New_Fractional_Step_Method()
    Uo = ref.get_compact()
    ref.Recalculate_Velocity_Antitransform()
    Po = ref.get_physical()
    Eo = ref.Recalculate_Energy_Cascade()

    Uf = np.fromfile(od / "Velocity_Fourier.bin", dtype="<f8").view(np.complex128).reshape(Uo.shape)
    assert rel_l2(Uf, Uo) < 1e-12
    Pf = np.fromfile(od / "Velocity.bin", dtype="<f8").reshape(Po.shape)
    assert rel_l2(Pf, Po) < 1e-12
    rows = np.loadtxt(od / "Energy_Cascade.dat")
    assert rows.shape == (Eo.size, 2) and np.array_equal(rows[:, 0], np.arange(Eo.size))
    m = Eo > 1e-12 * Eo.max()
    assert np.max(np.abs(rows[m, 1] - Eo[m]) / Eo[m]) < 1e-5        # 6 printed digits
    assert np.all(np.abs(rows[~m, 1]) <= 1e-10 * Eo.max())

    # the physical field read back as an initial field (M^3 file: every retained mode survives the truncation)
    M = Po.shape[1]
    (tmp_path / "DATA").mkdir(exist_ok=True)
    Pf.astype("<f8").tofile(tmp_path / "DATA" / "restart.bin")
    txt2 = re.sub(r"^ASCII_Input_Filename.*$", "#", txt, flags=re.M)
    for k, v in (("Binary_Input_Filename", "DATA/restart.bin"), ("Nx_file", M), ("Ny_file", M), ("Nz_file", M)):
        txt2 = _set_param(txt2, k, v)
    p2 = tmp_path / "params_restart"
    p2.write_text(txt2)
    a2 = derive_hit_args(read_params(str(p2)), base_dir=str(tmp_path))
    ref2 = O.OracleHIT(a2, file_uvw=Pf)
    assert rel_l2(ref2.get_compact(), Uo) < 1e-13
    from spns_b200.hit import HIT
    gpu2 = HIT(a2, file_uvw=Pf)
    assert rel_l2(gpu2.get_compact(), Uo) < 1e-13
    gpu2.close()
    r = subprocess.run([EXE, "params_restart"], cwd=str(tmp_path), capture_output=True, timeout=120)
    out = r.stdout.decode(errors="replace") + r.stderr.decode(errors="replace")
    assert r.returncode == 0, out[-3000:]
