"""Teide's own known answers through td_execute on libteide_b200.so (GPU)."""
import pytest

import known_cases


@pytest.mark.gpu
@pytest.mark.parametrize("case", known_cases.ALL, ids=lambda c: c.__name__)
def test_known_answer_on_gpu(gpu, case):
    case(gpu)
