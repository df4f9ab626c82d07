"""The oracle's sort against Teide itself (CPU): stable order by the encoded
keys, F64 NaN / signed-zero placement, SYM by string, two keys, HEAD over a
sort (Teide's heap top-N path, unique keys), and a sorted group-by result."""
import pytest

import sort_cases


@pytest.mark.parametrize("case", sort_cases.ALL, ids=lambda c: c.__name__)
def test_sort_oracle_matches_reference(ref, case):
    got, want = case(ref)
    sort_cases.same(got, want)
