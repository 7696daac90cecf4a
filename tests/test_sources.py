"""Source conventions the GPU code relies on, checked without a GPU.

Every kernel of the solve path is launched with programmatic stream
serialization (kutta_b200/csrc/cuda/common.cuh: pdl), which lets a kernel
start before its predecessor has finished; that is only correct because each
such kernel's first statement waits for the predecessor (pdl_entry). A kernel
added without that wait, or launched with <<<>>> in these files, would break
the ordering or bypass the convention, so both are checked here."""
import pathlib
import re

import pytest

CUDA = pathlib.Path(__file__).resolve().parent.parent / "kutta_b200" / "csrc" / "cuda"
PDL_FILES = ["exact_kernels.cu", "mixed_kernels.cu", "tail_cycle.cu"]


@pytest.mark.parametrize("name", PDL_FILES)
def test_every_solve_path_kernel_waits_for_its_predecessor_first(name):
    text = (CUDA / name).read_text()
    kernels = 0
    for m in re.finditer(r"__global__", text):
        body = text.index("{", m.end())
        first = text[body + 1:].lstrip().split(";", 1)[0]
        assert first in ("pdl_entry()", "dev::pdl_entry()"), (name, text[m.start():body + 80])
        kernels += 1
    assert kernels > 0


@pytest.mark.parametrize("name", PDL_FILES)
def test_solve_path_kernels_launch_through_the_pdl_helper(name):
    text = (CUDA / name).read_text()
    assert "<<<" not in text
