"""The CPU oracle reproduces the reference's own QA golden logs (all 9 tests).

K41-initialised tests are reproduced by emulating the 4-rank K41 draw of the
reference run (each rank reseeds rand() with 0 for its ky slab).
"""
import pytest

from spns_b200 import driver
from qa_util import QA_TESTS, load_case, compare_records


@pytest.mark.parametrize("name", QA_TESTS)
def test_oracle_matches_reference_qa_log(name, oracle_lib):
    import oracle as O
    args, uvw, ref = load_case(name)
    h = O.OracleHIT(args, uvw, k41_ranks=4)
    recs = driver.run(h, args)
    worst = compare_records(recs, ref["steps"])
    assert worst < 1e-6
    final = ref["final"]
    assert int(final["Final time-steps"]) == len(recs)
    assert abs(float(final["Final energy"]) - recs[-1].ek) < 1.5e-6


def test_oracle_parseval_invariant(oracle_lib):
    """Check_PhysFour_Energy (src/HIT_LES.cpp:1216-1252) holds on the oracle."""
    import oracle as O
    args, uvw, ref = load_case("TEST_1_DHIT_DNS")
    h = O.OracleHIT(args, uvw)
    for _ in range(3):
        h.New_Fractional_Step_Method()
    ok, d1, d2 = h.Check_PhysFour_Energy(1e-13)
    assert ok, (d1, d2)
