"""The C-ABI library loads without a GPU and exports every symbol that
include/mgk.h declares; host-only entry points give the oracle's answers."""
import os
import re

import numpy as np
import pytest

import mgpukde_tiled_b200 as mk
import oracle_py as o
from golden_cases import CASES, load

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(REPO, "include", "mgk.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mgk_[a-z0-9_]+)\s*\(", src)))


def test_every_declared_symbol_is_exported():
    L = mk.lib()
    names = declared_symbols()
    assert len(names) >= 25
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(mk.EXPORTS)


@pytest.mark.parametrize("case", CASES)
def test_rule_of_thumb_bit_exact(case):
    d = load(case)
    assert mk.rule_of_thumb(d["x"], d["y"], d["w"]) == o.rule_of_thumb(d["x"], d["y"], d["w"])


def test_context_without_gpu_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(mk.MgkError) as e:
        mk.Context(0)
    assert e.value.status == -4


def test_status_strings():
    L = mk.lib()
    assert L.mgk_status_string(0) == b"ok"
    assert L.mgk_status_string(-3) == b"HBM budget exceeded"
