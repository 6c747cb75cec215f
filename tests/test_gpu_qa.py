"""The reference's QA regression suite run through the GPU solver and the restated driver loop.

Same comparison as QA/check.sh but on every per-step line (Dt, Ek, Om at 7
significant digits, ReLambda at 3 decimals), not only the Final lines.
"""
import pytest

from spns_b200 import driver
from qa_util import QA_TESTS, load_case, compare_records

pytestmark = pytest.mark.gpu



@pytest.mark.parametrize("name", QA_TESTS)
def test_gpu_matches_reference_qa_log(name):
    from spns_b200.hit import HIT
    args, uvw, ref = load_case(name)
    h = HIT(args, uvw, k41_ranks=4)
    # a wrong time step would make the Final_Time loop run on: cap it well above the reference's count
    recs = driver.run(h, args, max_steps=2 * len(ref["steps"]) + 10)
    compare_records(recs, ref["steps"])
