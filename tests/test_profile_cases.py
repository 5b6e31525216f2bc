"""The ncu profiling cases: the module imports without a GPU, names its
cases, and refuses unknown ones (and runs nothing without a CUDA device)."""
import torch

from ct_laboratory_b200 import profile_cases


def test_cases_and_usage():
    assert set(profile_cases.CASES) == {"static512-v24", "batch64"}
    assert profile_cases.main([]) == 2
    assert profile_cases.main(["nope"]) == 2
    if not torch.cuda.is_available():
        assert profile_cases.main(["batch64"]) == 1
