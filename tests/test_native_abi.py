"""CPU-side checks of the C ABI: the library loads and exports every function declared in
include/clothstep.h; on a machine without a usable device the product path fails loudly."""
import os
import re

import pytest

from clothsimulator_b200 import native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "clothstep.h")).read()
    return sorted(set(re.findall(r"^\s*(?:cs_status|const char\*)\s+(cs_\w+)\s*\(", text, re.M)))


def test_header_matches_binding_list():
    assert declared_functions() == sorted(native.EXPORTED)


def test_library_exports_every_declared_symbol():
    lib = native.load_library()
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_create_without_device_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(native.ClothStepError) as e:
        native.Context(0)
    assert e.value.status == native.CS_ERR_NO_DEVICE
