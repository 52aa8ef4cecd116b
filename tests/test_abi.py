"""The C-ABI library loads without a GPU and exports every entry point that
include/mdn.h declares; without a device it refuses to run instead of
falling back to a CPU path."""
import ctypes as C
import os
import re

import pytest

from md_nucleation_b200 import abi, build, engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mdn_[a-z_0-9]+)\s*\(", src)))


@pytest.fixture(scope="module")
def libmdn():
    build.build()
    return C.CDLL(engine.LIB_PATH)


def test_every_declared_symbol_is_exported(libmdn):
    names = declared("mdn.h")
    assert len(names) >= 20
    for n in names:
        assert hasattr(libmdn, n), f"{n} declared in include/mdn.h but not exported"


def test_abi_version_and_struct_sizes(libmdn):
    assert libmdn.mdn_abi_version() == abi.ABI_VERSION
    # sizes the C compiler sees must match the ctypes mirror (checked through
    # offsets of the last fields: a mismatch shows up as a wrong default)
    o = abi.Options()
    libmdn.mdn_default_options(C.byref(o))
    assert o.quirks == abi.Q_ALL and o.threads == 512 and o.capacity_factor == 1.5


def test_no_device_is_an_error_not_a_fallback(libmdn):
    n = C.c_int(-1)
    libmdn.mdn_device_count(C.byref(n))
    if n.value > 0:
        pytest.skip("a CUDA device is present")
    from md_nucleation_b200 import generate as g
    with pytest.raises(engine.MdnError) as e:
        engine.Engine([g.small_system(n_gas=50, n_vap=2)])
    assert e.value.code == abi.ERR_NO_DEVICE


def test_descriptor_validation_rejects_bad_topology(libmdn):
    """Bad descriptors fail with MDN_ERR_ARG before any device work; on a
    CPU-only machine the device check comes first."""
    from md_nucleation_b200 import generate as g
    s = g.small_system(n_gas=50, n_vap=2)
    s.ion.bonds = s.ion.bonds.copy()
    if len(s.ion.bonds) == 0:
        import numpy as np
        s.ion.bonds = np.array([[0, 99, 0]], np.int32)
    else:
        s.ion.bonds[0, 1] = 10_000
    with pytest.raises(engine.MdnError) as e:
        engine.Engine([s])
    assert e.value.code in (abi.ERR_ARG, abi.ERR_NO_DEVICE)
