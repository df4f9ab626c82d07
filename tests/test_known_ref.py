"""Teide's own known answers, run on Teide itself (CPU).  Pins the td.h
translations in known_cases.py before they are used to check the GPU library."""
import pytest

import known_cases


@pytest.mark.parametrize("case", known_cases.ALL, ids=lambda c: c.__name__)
def test_known_answer_on_reference(ref, case):
    case(ref)
