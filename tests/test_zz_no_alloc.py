"""jfg_assemble_values_noalloc: K's values with no device allocation (gpu).

Some callers cannot let the library call cudaMalloc between solves: their
device memory belongs to another framework's caching pool, or other streams
must not be stalled by a device-wide allocation.  For them the library keeps
the element matrices of this one entry point in a fixed 16 MiB device array.
These tests call it through the C ABI, twice in a row, and check the values
against the regular jfg_assemble path (jfg_get_values) within the element
tolerance of the parity tests; they also check the size limit and the
not-ready error.  The file is named so that pytest collects it last.
"""
import numpy as np
import pytest

from jf_2026_05_25_b200 import build as jbuild
from jf_2026_05_25_b200 import lib
from jf_2026_05_25_b200 import model as M

pytestmark = pytest.mark.gpu

ELEM_RTOL = 1e-12


@pytest.fixture(scope="module")
def ctx():
    jbuild.build()
    c = lib.Context(0)
    yield c
    c.close()


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("make", [lambda: M.flat_plate(nx=20, ny=20),
                                  lambda: M.solid_block(n=2, n_cases=1)],
                         ids=["cquad4_plate", "ctetra10_block"])
def test_noalloc_matches_assemble_twice(ctx, make):
    import torch
    dm = lib.DeviceModel(ctx, make())
    dm.assemble()
    ref = dm.values()
    out = torch.full((len(ref),), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    for _ in range(2):
        dm.assemble_values_noalloc(out.data_ptr())
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert _rel(got, ref) <= ELEM_RTOL
        out.fill_(float("nan"))
        torch.cuda.synchronize()
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
