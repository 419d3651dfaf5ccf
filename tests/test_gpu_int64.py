"""64-bit rating positions: the engine must address ratings past 2^32.

The largest rating matrices the engine is sized for (50,082,604 x 39,781 with
about 3.1 billion ratings) have row pointers beyond the int32 range, which the
reference cannot represent (its CSR is int32, als/src/cuda/als.h:96-103). This
test places a small matrix's CSR and CSC at position 2^32 + 2^20 + 3 of
17 GB index and rating arrays, so every row pointer is above 2^32, and checks
that each form gives the same bits as the same matrix stored from position 0.

The offset is chosen so that a position truncated to 32 bits (signed or
unsigned) would still land inside the arrays, in the zero-filled region in
front of the data: a truncation shows up as wrong results, never as an
out-of-bounds access.
"""
import numpy as np
import pytest
import torch

import als_b200 as A

pytestmark = pytest.mark.gpu

BASE = (1 << 32) + (1 << 20) + 3


@pytest.fixture(scope="module")
def big_arrays():
    r = A.synth(A.scaled_config("netflix", 0.05), seed=12)
    nnz = r.nnz
    gap = 1 << 12
    length = BASE + 2 * nnz + 2 * gap
    col = torch.zeros(length, dtype=torch.int32, device="cuda")
    val = torch.zeros(length, dtype=torch.float32, device="cuda")
    b_csr, b_csc = BASE, BASE + nnz + gap
    col[b_csr:b_csr + nnz] = torch.from_numpy(r.csr_col).cuda()
    val[b_csr:b_csr + nnz] = torch.from_numpy(r.csr_val).cuda()
    col[b_csc:b_csc + nnz] = torch.from_numpy(r.csc_row).cuda()
    val[b_csc:b_csc + nnz] = torch.from_numpy(r.csc_val).cuda()
    csr_ptr = torch.from_numpy(r.csr_ptr + b_csr).cuda()
    csc_ptr = torch.from_numpy(r.csc_ptr + b_csc).cuda()
    arrays = (csr_ptr, col, val, csc_ptr, col, val)
    test = [torch.from_numpy(a).cuda() for a in (r.test_u, r.test_i, r.test_r)]
    yield r, arrays, test
    del arrays, col, val, csr_ptr, csc_ptr, test
    torch.cuda.empty_cache()  # hand the 34 GB back before the later tests run


FORMS = [
    ("fp32-cholesky", 32, dict()),
    ("bf16-cg", 100, dict(precision=A.PREC_BF16, solver=A.SOLVER_CG,
                          warm_start=A.WARM_PREVIOUS, solver_groups=2)),
    ("bf16-cholesky", 64, dict(precision=A.PREC_BF16, solver=A.SOLVER_CHOLESKY, solver_groups=3)),
    ("fp16-cg-f128", 128, dict(precision=A.PREC_FP16, solver=A.SOLVER_CG,
                               warm_start=A.WARM_PREVIOUS)),
]


@pytest.mark.parametrize("name,f,kw", FORMS, ids=[x[0] for x in FORMS])
def test_positions_above_2_32_give_identical_bits(big_arrays, name, f, kw):
    r, arrays, test = big_arrays
    assert int(arrays[0][0]) > (1 << 32) and int(arrays[3][-1]) > (1 << 32)
    # the matrix has rows long enough to be split across CTAs
    assert np.diff(r.csc_ptr).max() > 8192
    th = A.init_factors(r.n, f, 5)
    ref = A.Model(r, f, A.options(**kw), theta0=th)
    off = A.Model.from_device(r.m, r.n, f, r.nnz, arrays, test, A.options(**kw), theta0=th)
    ref.iterate(0.05, 2)
    off.iterate(0.05, 2)
    for a, b in zip(ref.factors(), off.factors()):
        a, b = a.cpu(), b.cpu()
        assert torch.isfinite(a).all()
        assert torch.equal(a, b), name
    assert ref.rmse() == off.rmse()
    s_ref, s_off = ref.stats(), off.stats()
    assert s_off["kernel_errors"] == 0 and s_ref["kernel_errors"] == 0
    assert s_off["rows_solved"] == s_ref["rows_solved"] == 2 * (r.m + r.n)
    ref.close()
    off.close()
