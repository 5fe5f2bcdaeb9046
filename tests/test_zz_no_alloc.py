"""The allocation-free entry point cf_q_device_noalloc, called through the C ABI.

Some callers cannot let a library allocate device memory: a host whose device memory all belongs
to its own allocator, or code that is about to record its work into a stream capture.  For them
cf_q_device_noalloc runs the batched contraction with its scratch in a fixed array inside the
library (CF_NOALLOC_SCRATCH_BYTES, 64 MiB per device, held until exit).  This test checks it
against the allocating entry point cf_q_device, on two calls in a row, with the tolerance of the
other FP64 parity tests, and checks that it rejects a batch too large for the array.

The file is named to be collected last, so that a run stopping at the first failure has already run
every other test.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import GOLDEN, per_cell_err

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12


def test_noalloc_matches_cf_q_device_on_two_calls(cuda_available):
    import torch

    import cf_b200
    from cf_b200 import _lib, geometry, workloads

    L, K, B = 8, 8, 1000
    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    R = np.load(GOLDEN / "R_hs_k7_l8_pad20.npy")
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    f = torch.from_numpy(workloads.maxwellian_cells(K, L, B, seed=77)).cuda()
    ref = op.q(f).cpu().numpy()  # cf_q_device: scratch allocated inside the plan

    lib = _lib.load()
    stream = torch.cuda.current_stream()
    free_after_first = None
    for call in range(2):
        out = torch.zeros_like(f)
        torch.cuda.synchronize()
        st = lib.cf_q_device_noalloc(op._h, out.data_ptr(), f.data_ptr(), B, _lib.FORM_AF, stream.cuda_stream)
        assert st == 0, lib.cf_last_error().decode()
        torch.cuda.synchronize()
        err = per_cell_err(out.cpu().numpy(), ref)
        assert err <= TOL_FP64, f"call {call}: {err:.3e}"
        free_now = torch.cuda.mem_get_info()[0]
        if call == 0:
            free_after_first = free_now
        else:
            assert free_now == free_after_first, "the second call changed the free device memory"

    # accumulates like the other entry points (out += Q(f))
    out = torch.from_numpy(ref.copy()).cuda()
    st = lib.cf_q_device_noalloc(op._h, out.data_ptr(), f.data_ptr(), B, _lib.FORM_AF, stream.cuda_stream)
    assert st == 0
    torch.cuda.synchronize()
    assert per_cell_err(out.cpu().numpy(), 2.0 * ref) <= 1e-14

    # a batch larger than the fixed scratch array is rejected, not run.  The smallest such batch is
    # derived from the header's limit (2 tiled copies of 32-cell tiles), and the buffers passed are
    # sized for it, so the call stays in bounds even if the check were missing.
    scratch = 64 << 20  # CF_NOALLOC_SCRATCH_BYTES
    M = geo.n_q * K
    big = (scratch // (2 * 8 * M) // 32 + 1) * 32
    assert 2 * 8 * M * big > scratch
    f_big = torch.zeros((big, K, geo.n_q), dtype=torch.float64, device="cuda")
    out_big = torch.zeros_like(f_big)
    st = lib.cf_q_device_noalloc(op._h, out_big.data_ptr(), f_big.data_ptr(), big, _lib.FORM_AF, stream.cuda_stream)
    assert st == 2
    assert b"scratch" in lib.cf_last_error()
    # the largest batch that fits runs (on zeros: Q stays zero)
    fit = (scratch // (2 * 8 * M) // 32) * 32
    st = lib.cf_q_device_noalloc(op._h, out_big.data_ptr(), f_big.data_ptr(), fit, _lib.FORM_AF, stream.cuda_stream)
    assert st == 0, lib.cf_last_error().decode()
    torch.cuda.synchronize()
    assert float(out_big.abs().max()) == 0.0
    op.close()


def test_noalloc_folded_form_needs_its_operator_built_first(cuda_available):
    """The folded form runs on the plan's folded operator, whose first use builds it with
    allocations; the allocation-free call refuses it until then, and afterwards matches cf_q_device
    on two calls in a row, allocating nothing."""
    import torch

    import cf_b200
    from cf_b200 import _lib, geometry, workloads

    L, K, B = 8, 8, 700
    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    R = np.load(GOLDEN / "R_hs_k7_l8_pad20.npy")
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    f = torch.from_numpy(workloads.maxwellian_cells(K, L, B, seed=78)).cuda()
    lib = _lib.load()
    stream = torch.cuda.current_stream()
    out = torch.zeros_like(f)
    st = lib.cf_q_device_noalloc(op._h, out.data_ptr(), f.data_ptr(), B, _lib.FORM_AF_SYM, stream.cuda_stream)
    assert st == 1 and b"folded operator is not built" in lib.cf_last_error()
    ref = op.q(f, form="af_sym").cpu().numpy()  # builds the folded operator
    free_after_first = None
    for call in range(2):
        out = torch.zeros_like(f)
        torch.cuda.synchronize()
        st = lib.cf_q_device_noalloc(op._h, out.data_ptr(), f.data_ptr(), B, _lib.FORM_AF_SYM, stream.cuda_stream)
        assert st == 0, lib.cf_last_error().decode()
        torch.cuda.synchronize()
        assert per_cell_err(out.cpu().numpy(), ref) <= TOL_FP64, f"call {call}"
        free_now = torch.cuda.mem_get_info()[0]
        if call == 0:
            free_after_first = free_now
        else:
            assert free_now == free_after_first
    op.close()
