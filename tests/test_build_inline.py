"""The step kernel keeps its per-CTA context (struct Ctx: the replica's
parameters, the shared-memory core arrays) in registers, which needs every
device function of advance.cu that takes it by reference inlined into
mdn_advance.  An outlined one forces the context into local memory: every
access to it becomes a local load, and the core sums' atomics, whose shared
address space the compiler can no longer see, become generic atomics (the
step measured 20-25 % slower that way).  ptxas lists a "Function properties"
block for each function it compiles on its own, so only the kernel (and
libdevice's internal slow paths) may appear."""
import re
import shutil

import pytest

from md_nucleation_b200 import build


def _have_nvcc():
    try:
        build.nvcc()
        return True
    except RuntimeError:
        return shutil.which("nvcc") is not None


@pytest.mark.skipif(not _have_nvcc(), reason="nvcc not available")
def test_step_kernel_fully_inlined():
    rep = build.ptxas_report()
    funcs = re.findall(r"Function properties for (\S+)", rep)
    assert "mdn_advance" in funcs, rep[-2000:]
    outlined = [f for f in funcs if f != "mdn_advance" and not f.startswith("__internal_")]
    assert not outlined, outlined
