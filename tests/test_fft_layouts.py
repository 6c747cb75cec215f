"""The exchange-layout table of the FFT engine (spns_b200/csrc/fft_layouts.h)
is what its generator produces, and its model agrees with hand-counted cases."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "spns_b200", "csrc")


def test_layout_table_is_current():
    r = subprocess.run([sys.executable, os.path.join(CSRC, "gen_layouts.py"), "--check"], timeout=300)
    assert r.returncode == 0, "fft_layouts.h is stale: run python spns_b200/csrc/gen_layouts.py"


def test_wavefront_model_hand_counts():
    sys.path.insert(0, CSRC)
    import gen_layouts as G
    # 8-byte elements, 32 consecutive rows: two half-warp phases of one wavefront each
    assert G.wavefronts([2 * i for i in range(32)], 2) == 2
    # stride of 16 rows (128 bytes): the 16 lanes of a phase share two banks
    assert G.wavefronts([32 * i for i in range(32)], 2) == 32
    # 16-byte elements, consecutive rows: four quarter-warp phases
    assert G.wavefronts([4 * i for i in range(32)], 4) == 4
    # radix-12 first stage, length 768: a pad of one row per 12 removes the stride conflicts
    rs = G.plan(768, 12, False)
    assert G.cost(768, 12, rs, 0, 1, 0, 2) < G.cost(768, 12, rs, 0, 0, 0, 2)
    # every padded layout keeps each butterfly's writes inside its block of X rows
    for L in G.LENGTHS:
        for inv in (True, False):
            rs = G.plan(L, 12, inv)
            for S in range(len(rs) - 1):
                X = 1
                for r in rs[:S + 1]:
                    X *= r
                assert (L // rs[S + 1]) % X == 0
