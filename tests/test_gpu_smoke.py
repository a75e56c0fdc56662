"""The package's own smoke check (one small FP64 run on cuda:0 against the
oracle) as a GPU test."""
import pytest

pytestmark = pytest.mark.gpu


def test_smoke(gpu):
    import __graft_entry__
    __graft_entry__.smoke()
