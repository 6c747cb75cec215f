"""Helpers shared by the QA golden tests (reference QA/TEST_* logs)."""
import json
import os

import numpy as np

from spns_b200.params import read_params, derive_hit_args

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "qa")
QA_TESTS = sorted(d for d in os.listdir(GOLDEN) if d.startswith("TEST_"))


def load_case(name):
    d = os.path.join(GOLDEN, name)
    args = derive_hit_args(read_params(os.path.join(d, "params")), base_dir=d)
    if args.isForcedEk:
        args.EkFilename = os.path.join(d, "Forced_Energy_Cascade.dat")
    uvw = np.load(os.path.join(d, "init_uvw.npy")) if args.is_file_init else None
    with open(os.path.join(d, "ref_steps.json")) as fh:
        ref = json.load(fh)
    return args, uvw, ref


def compare_records(records, ref_steps):
    """Golden lines hold Time %f, Dt/Ek/Om %e (7 digits) and ReLambda %8.3f."""
    assert len(records) == len(ref_steps), (len(records), len(ref_steps))
    worst = 0.0
    for r, g in zip(records, ref_steps):
        t, it, dt, ek, om, rl = g
        assert r.iter == it
        assert abs(r.time - t) <= 1.5e-6, (it, r.time, t)
        for a, b in ((r.dt, dt), (r.ek, ek), (r.om, om)):
            rel = abs(a - b) / abs(b)
            worst = max(worst, rel)
            assert rel <= 1.0e-6, (it, a, b, rel)
        assert abs(r.relambda - rl) <= 1.5e-3, (it, r.relambda, rl)
    return worst
