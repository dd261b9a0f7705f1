"""The pressure solve that allocates nothing (cfd_pcg_solve_noalloc).

It exists for callers that may not allocate or free device memory while they
solve: cudaFree synchronizes the whole device, and some host codes reserve all
of their device memory up front in their own pool.  The caller owns every
input and output buffer; the work vectors live in a fixed static array, so
the system size is limited to CFD_NOALLOC_MAX_N rows.

Checked here through the C ABI against the context's own solve
(cfd_pressure_solve) on two calls in a row, with the tolerance the other
pressure-solve tests use.  This file is collected last on purpose.
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

SOLVE_TOL = 1e-7   # relative L2, as the Pdot checks of test_gpu_parity.py


def test_noalloc_solve_matches_context_solve(decks):
    import torch
    import cfdfs
    s = cfdfs.Solver(device=0)
    s.load(decks["graded"])
    s.step0()
    rp, col, zval = s.matrix("Z")
    n = len(rp) - 1
    diag = np.array([zval[rp[i]:rp[i + 1]][col[rp[i]:rp[i + 1]] == i][0] for i in range(n)])
    dev = torch.device("cuda:0")
    rp_t = torch.from_numpy(rp).to(dev)
    col_t = torch.from_numpy(col).to(dev)
    val_t = torch.from_numpy(zval).to(dev)
    dinv_t = torch.from_numpy(1.0 / diag).to(dev)
    x_t = torch.zeros(n, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rng = np.random.default_rng(11)
    for call in range(2):                                   # two calls in a row
        b = rng.standard_normal(n)
        b_t = torch.from_numpy(b).to(dev)
        x_t.fill_(123.0)                                    # output is fully overwritten
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(0)[0]
        reserved_before = torch.cuda.memory_reserved(0)
        rc, info, msg = cfdfs.pcg_solve_noalloc(rp_t.data_ptr(), col_t.data_ptr(), val_t.data_ptr(),
                                                dinv_t.data_ptr(), b_t.data_ptr(), x_t.data_ptr(), n,
                                                1e-8, 1000, stream)
        assert rc == cfdfs.CFD_OK, msg
        torch.cuda.synchronize()
        # the property the entry point exists for: once its static array is
        # on the device (the first call puts it there), a call allocates no
        # device memory, neither through CUDA nor through torch's allocator
        if call == 1:
            assert torch.cuda.mem_get_info(0)[0] == free_before
            assert torch.cuda.memory_reserved(0) == reserved_before
        x_ref, st = s.pressure_solve(b)
        assert st.status == 0
        assert rel_l2(x_t.cpu().numpy(), x_ref) < SOLVE_TOL, call
        assert abs(int(info[0]) - st.iterations) <= 2
        assert info[1] <= 1e-8
    # sizes beyond the static work array are refused with a message
    rc, info, msg = cfdfs.pcg_solve_noalloc(rp_t.data_ptr(), col_t.data_ptr(), val_t.data_ptr(),
                                            dinv_t.data_ptr(), b_t.data_ptr(), x_t.data_ptr(),
                                            cfdfs.NOALLOC_MAX_N + 1, 1e-8, 1000, stream)
    assert rc == cfdfs.CFD_E_BADARG and "524288" in msg
    s.close()
