"""jfg_assemble_values_noalloc: K's values with no device allocation (gpu).

Some callers cannot let the library call cudaMalloc between solves: their
device memory belongs to another framework's caching pool, or other streams
must not be stalled by a device-wide allocation.  For them the library keeps
the element matrices of this one entry point in a fixed 16 MiB device array.
These tests call it through the C ABI, twice in a row, and check the values
against the regular jfg_assemble path (jfg_get_values): the same kernels run,
so the values must be bit-identical.  They check that a call leaves the
device's free memory unchanged, the size limit and the not-ready error.
The file is named so that pytest collects it last.
"""
import numpy as np
import pytest

from jf_2026_05_25_b200 import build as jbuild
from jf_2026_05_25_b200 import lib
from jf_2026_05_25_b200 import model as M

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    jbuild.build()
    c = lib.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("make", [lambda: M.flat_plate(nx=20, ny=20),
                                  lambda: M.quad8_plate(nx=8, ny=6, skew=0.2, tilt_deg=30.0),
                                  lambda: M.solid_block(n=2, n_cases=1)],
                         ids=["cquad4_plate", "cquad8_plate", "ctetra10_block"])
def test_noalloc_matches_assemble_twice(ctx, make):
    """Same element and gather kernels as jfg_assemble, so the values must be
    bit-identical; after the first call (which looks the array up and, with
    lazy module loading, brings it onto the device) a call allocates no
    device memory: the device's free bytes are unchanged across it."""
    import torch
    dm = lib.DeviceModel(ctx, make())
    dm.assemble()
    ref = dm.values()
    out = torch.full((len(ref),), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    dm.assemble_values_noalloc(out.data_ptr())          # set-up call
    assert np.array_equal(out.cpu().numpy(), ref)
    for _ in range(2):
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        dm.assemble_values_noalloc(out.data_ptr())
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0, f"device free bytes changed by {free0 - free1} across the call"
        got = out.cpu().numpy()
        assert np.array_equal(got, ref)
    dm.close()


def test_noalloc_rejects_models_over_the_scratch_limit(ctx):
    import torch
    # 64 x 64 CQUAD4 need 4096 * 576 * 8 bytes > 16 MiB of element storage
    dm = lib.DeviceModel(ctx, M.flat_plate(nx=64, ny=64))
    dm.assemble()
    out = torch.zeros(dm.sizes()[1], dtype=torch.float64, device="cuda")
    with pytest.raises(lib.JfgError) as ei:
        dm.assemble_values_noalloc(out.data_ptr())
    assert ei.value.status_name == "BAD_INPUT"
    assert "16777216" in str(ei.value)
    dm.close()


def test_noalloc_needs_the_pattern(ctx):
    import torch
    dm = lib.DeviceModel(ctx, M.flat_plate(nx=4, ny=4))
    out = torch.zeros(16, dtype=torch.float64, device="cuda")
    with pytest.raises(lib.JfgError) as ei:
        dm.assemble_values_noalloc(out.data_ptr())
    assert ei.value.status_name == "NOT_READY"
    dm.close()
