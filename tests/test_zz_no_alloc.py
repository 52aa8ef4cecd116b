"""mdn_snapshot_noalloc (the snapshot staged in the library's fixed device
array, no allocation) against mdn_snapshot (staging allocated on its first
call), through the C ABI.

Both entry points run the same gather kernels over the same resident state,
so the rows must agree exactly: the tolerance is 0, inside every position
and velocity tolerance the parity tests use.  The file is collected last, so
it runs both alone and after every other GPU test in one process.
"""
import ctypes as C

import numpy as np
import pytest

from md_nucleation_b200 import abi
from md_nucleation_b200 import generate as g
from tests import systems
from tests.gpu_helpers import need_gpu

pytestmark = pytest.mark.gpu

MAX_ROWS = 65536      # MDN_NOALLOC_MAX_ROWS
XTOL = 0.0            # identical kernels on identical state
ERR_CAPACITY = -4     # MDN_ERR_CAPACITY


@pytest.fixture(scope="module")
def eng():
    return need_gpu()


def _fn(L):
    f = L.mdn_snapshot_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.POINTER(C.c_longlong), C.c_longlong, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.POINTER(C.c_double)]
    return f


def noalloc(e, cap):
    off = np.zeros(e.n + 1, np.int64)
    t = np.zeros(max(cap, 1), np.int32)
    x = np.zeros((max(cap, 1), 3))
    v = np.zeros((max(cap, 1), 3))
    U = np.zeros((e.n, 8))
    rc = _fn(e.L)(e.h, abi.ptr(off, C.c_longlong), cap, t.ctypes.data_as(C.c_void_p),
                  x.ctypes.data_as(C.c_void_p), v.ctypes.data_as(C.c_void_p), abi.ptr(U))
    return rc, off, t, x, v, U


def reference_snapshot(eng, e, cap):
    buf = eng.SnapshotBuffer(e.n, cap, pinned=False)
    e.snapshot(buf, energies=True)
    return buf


def same(got, buf):
    rc, off, t, x, v, U = got
    assert rc == 0, f"mdn_snapshot_noalloc returned {rc}"
    n = int(buf.offset[-1])
    assert 0 < n <= MAX_ROWS
    assert np.array_equal(off, buf.offset)
    assert np.array_equal(t[:n], buf.type[:n])
    assert np.abs(x[:n] - buf.x[:n]).max() <= XTOL
    assert np.abs(v[:n] - buf.v[:n]).max() <= XTOL
    assert np.array_equal(U, buf.U)


def test_noalloc_allocates_no_device_memory(eng):
    """The point of the entry point: on a handle that never took a
    mdn_snapshot, neither the first nor the second call takes device memory
    (the fixed array and the snapshot kernels are loaded by mdn_create).
    Free device memory is read with cudaMemGetInfo through torch."""
    import torch
    torch.cuda.init()
    e = eng.Engine([systems.make("chain_he_water"), systems.make("nacl_n2_meoh")])
    e.step(4, energy_mode=1)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    first = noalloc(e, MAX_ROWS)
    free1, _ = torch.cuda.mem_get_info(0)
    second = noalloc(e, MAX_ROWS)
    free2, _ = torch.cuda.mem_get_info(0)
    assert first[0] == 0 and second[0] == 0
    assert free1 >= free0, f"the first call took {free0 - free1} bytes of device memory"
    assert free2 >= free0, f"the second call took {free0 - free2} bytes of device memory"
    assert np.array_equal(first[1], second[1]) and np.array_equal(first[3], second[3])


def test_noalloc_matches_snapshot_twice_in_a_row(eng):
    specs = [systems.make(n) for n in ("nacl_n2_meoh", "chain_he_water", "nacl_n2mono_meoh")]
    e = eng.Engine(specs)
    e.step(5, energy_mode=1)
    cap = MAX_ROWS
    ref = reference_snapshot(eng, e, cap)
    same(noalloc(e, cap), ref)
    same(noalloc(e, cap), ref)          # the second call of a pair, same state
    e.step(10, energy_mode=1)
    ref = reference_snapshot(eng, e, cap)
    same(noalloc(e, cap), ref)
    # a smaller batch after a larger one: rows left in the array by the
    # earlier calls are never returned
    e1 = eng.Engine([systems.make("nacl_n2rigid_water")])
    e1.step(3, energy_mode=1)
    ref1 = reference_snapshot(eng, e1, cap)
    assert ref1.offset[-1] < ref.offset[-1]
    same(noalloc(e1, cap), ref1)
    same(noalloc(e1, cap), ref1)


def test_noalloc_rejects_more_rows_than_it_holds(eng):
    """Five replicas of 20,000 dense N2 molecules: about 70,000 in-domain
    atoms, beyond the 65,536 rows of the fixed array."""
    specs = [g.small_system(seed=40 + k, gas="N2", vapor="methanol", ion="nacl", n_gas=20000, n_vap=10,
                            box=250.0) for k in range(5)]
    e = eng.Engine(specs)
    rc, off, *_ = noalloc(e, MAX_ROWS)
    if off[-1] <= MAX_ROWS:
        pytest.fail(f"the oversize case holds only {off[-1]} rows")
    assert rc == ERR_CAPACITY
    assert "MDN_NOALLOC_MAX_ROWS" in eng.lib().mdn_last_error().decode()
    # offsets are still those of mdn_snapshot, and a later call that fits works
    ref = reference_snapshot(eng, e, int(off[-1]))
    assert np.array_equal(off, ref.offset)
    small = eng.Engine([systems.make("nacl_n2_meoh")])
    small.step(2, energy_mode=1)
    same(noalloc(small, MAX_ROWS), reference_snapshot(eng, small, MAX_ROWS))


def test_noalloc_reports_a_small_host_buffer(eng):
    e = eng.Engine([systems.make("nacl_n2_meoh")])
    rc, off, *_ = noalloc(e, 10)
    assert rc == ERR_CAPACITY and off[-1] > 10
