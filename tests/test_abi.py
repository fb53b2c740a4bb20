"""The C-ABI library loads and exports exactly what include/ecsg_b200.h declares.
No compute call runs here (CPU host): only loading, symbol checks and the
loud failure of ecsg_create without a device."""
import ctypes
import os
import re

import pytest

import ecsg_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ecsg_b200.h")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ecsg_\w+)\s*\(", text)))


def test_library_is_built_for_sm100a():
    assert os.path.exists(ecsg_b200.LIB_PATH)
    ecsg_b200.lib()


def test_exports_every_declared_symbol():
    L = ctypes.CDLL(ecsg_b200.LIB_PATH)
    names = declared()
    assert len(names) >= 25
    for n in names:
        assert hasattr(L, n), n


def test_python_mirror_binds_every_declared_symbol():
    bound = {s[0] for s in ecsg_b200.SIGNATURES}
    assert bound == set(declared())


def test_create_fails_loudly_without_device():
    if ecsg_b200.lib().ecsg_device_count() > 0:
        pytest.skip("a device is present")
    from ecsg_b200.workloads import random_case
    with pytest.raises(ecsg_b200.EcsgError):
        ecsg_b200.Simulation(random_case(0))


def test_product_does_not_import_the_oracle():
    pkg = os.path.join(ROOT, "ecsg_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".cpp", ".h")):
                text = open(os.path.join(dirpath, f)).read()
                assert "import oracle" not in text and "from oracle" not in text, f
                assert "ecsg_oracle" not in text, f


def test_shots_entry_rejects_bad_arguments_without_a_device():
    """ecsg_shots_misfit_gradient checks its arguments before touching a
    device: no instances, or more than 16 shots, is ECSG_ERR_INVALID."""
    L = ecsg_b200.lib()
    assert L.ecsg_shots_misfit_gradient(None, 1, 10, None, 5, 0, None) == -1
    handles = (ctypes.c_void_p * 1)(None)
    assert L.ecsg_shots_misfit_gradient(handles, 1, 10, None, 5, 0, None) == -1
