"""Regenerate the QA golden fixtures from the reference tree (run in a container that has it).

Reads the reference's own regression data -- QA/TEST_*/params*, the per-step
report lines of QA/TEST_*/REF/stdout.0 (4-rank reference run linked against
FFTW 3) and the initial-field / forced-spectrum files under QA/TEST_*/DATA -- and
writes them under tests/golden/qa/ so that the tests need no reference tree at
run time.  Initial velocity files are stored as float64 .npy arrays of shape
[3, Nx_file, Ny_file, Nz_file], parsed exactly as src/HIT_LES.cpp:604-709 reads
them (ASCII rows ``u v w``; binary float64 components one after another).

Usage:  python tests/golden/make_fixtures.py [/path/to/SpNS]
"""
import glob
import json
import os
import re
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from spns_b200.params import read_params, derive_hit_args, read_initial_field  # noqa: E402

STEP_RE = re.compile(r"Time:\s*([-+0-9.eE]+),\s*iter:\s*(\d+),\s*Dt:\s*([-+0-9.eE]+),\s*Ek:\s*([-+0-9.eE]+),"
                     r"\s*Om:\s*([-+0-9.eE]+),\s*ReLambda:\s*([-+0-9.eE]+)")


def main(ref_root):
    out_root = os.path.join(HERE, "qa")
    os.makedirs(out_root, exist_ok=True)
    for tdir in sorted(glob.glob(os.path.join(ref_root, "QA", "TEST_*"))):
        name = os.path.basename(tdir)
        dst = os.path.join(out_root, name)
        os.makedirs(dst, exist_ok=True)
        pfile = glob.glob(os.path.join(tdir, "params*"))[0]
        shutil.copyfile(pfile, os.path.join(dst, "params"))
        steps, final = [], {}
        with open(os.path.join(tdir, "REF", "stdout.0"), errors="replace") as fh:
            for line in fh:
                m = STEP_RE.search(line)
                if m:
                    t, it, dt, ek, om, rl = m.groups()
                    steps.append([float(t), int(it), float(dt), float(ek), float(om), float(rl)])
                elif line.startswith("Final "):
                    k, v = line.split(":", 1)
                    final[k.strip()] = v.strip()
        with open(os.path.join(dst, "ref_steps.json"), "w") as fh:
            json.dump({"source": f"QA/{name}/REF/stdout.0", "steps": steps, "final": final}, fh, indent=0)
        P = read_params(os.path.join(dst, "params"))
        args = derive_hit_args(P, base_dir=tdir)
        if args.is_file_init:
            uvw = read_initial_field(args)
            np.save(os.path.join(dst, "init_uvw.npy"), uvw)
        if args.isForcedEk:
            shutil.copyfile(args.EkFilename, os.path.join(dst, "Forced_Energy_Cascade.dat"))
        print(name, len(steps), "steps", "file-init" if args.is_file_init else "K41")


if __name__ == "__main__":
    # the reference checkout: first argument, else $SPNS_REFERENCE
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SPNS_REFERENCE", "")
    if not src:
        sys.exit("usage: make_fixtures.py <reference checkout>  (or set SPNS_REFERENCE)")
    main(src)
