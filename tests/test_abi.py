"""CPU checks of the drop-in boundary: the C-ABI library loads without a GPU
and exports every function that include/hj.h declares; calls fail cleanly
(an error status, never a crash) when no device is present."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hj.h")


def declared_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"HJ_API\s+[\w\s\*]+?\b(hj_\w+)\s*\(", src)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("hj_self_join_count", "hj_join_count", "hj_self_join_count_f32", "hj_join_count_f32",
                 "hj_test_ego_loop3_macro", "hj_test_ego_loop3_noself", "hj_ego_sort", "hj_server_create",
                 "hj_submit", "hj_poll", "hj_wait", "hj_set_upload", "hj_self_join_pairs", "hj_join_pairs",
                 "hj_self_join_pairs_f32", "hj_join_pairs_f32"):
        assert must in names


def test_library_exports_every_declared_symbol():
    import hilbertjoin_b200 as hj
    L = hj.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    assert hj.version().startswith("hj ")


def test_no_device_gives_status_not_crash():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    import numpy as np
    import hilbertjoin_b200 as hj
    with pytest.raises(hj.HJError) as e:
        hj.self_join_count(np.zeros((10, 3)), 0.1)
    assert e.value.status in (3, 6)


def test_status_strings():
    import hilbertjoin_b200 as hj
    L = hj.lib()
    for s in range(11):
        assert L.hj_status_str(s)
