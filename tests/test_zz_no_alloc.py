"""vvm_gpu_poisson_solve_noalloc: the elliptic solve on caller-owned device
buffers, with no context and no device allocation.

It is checked through the C ABI against vvm_gpu_poisson_solve_device (the
context's multigrid-PCG solve of the same system) on two calls in a row with
different right-hand sides, both solved to a relative residual of 1e-12. The
solutions then agree to within cond(A) * 1e-12; the test allows 1e-8. The
solve's own residual report is not trusted alone: each solution's true
residual ||b - A W|| / ||b|| is recomputed on the host with the C
restatement's copy of the reference's matrix (src/PoissonSolver.cpp:760-796)
and must stay within 10x the tolerance. This file sorts last so that it also
runs after every other GPU test.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2

TOL = 1e-12
AGREE = 1e-8


def _lib():
    from vvm_b200 import build, gpu as G
    build.build()
    return G


def test_noalloc_rejects_oversize_problem():
    """The size check runs before any CUDA call, so this needs no GPU."""
    G = _lib()
    NX, NZ = 1024, 257                       # 1024 * 256 unknowns > VVM_NOALLOC_MAX_UNKNOWNS
    prof = np.ones(NZ + 2)
    with pytest.raises(G.VVMGpuError) as e:
        G.poisson_solve_noalloc(NX, NZ, prof, prof, 16, 16, tol=TOL)
    assert e.value.code == 1 and "exceeds its static scratch" in str(e.value)


@pytest.mark.gpu
@pytest.mark.parametrize("NX,NZ,d", [(128, 64, 200.0), (512, 256, 100.0)])
def test_noalloc_matches_context_solve(NX, NZ, d, port_lib):
    import torch
    from vvm_b200.initial_state import warm_bubble
    G = _lib()
    st = warm_bubble(NX, NZ, d, d)
    n = NX * (NZ - 1)
    assert n <= 131072
    rng = np.random.default_rng(11)
    rhs = [rng.standard_normal(n), np.sin(np.arange(n) * 0.37) + 0.5 * rng.standard_normal(n)]

    g = G.VVMGpu(st.grid, warm_start=False)
    g.upload(st)
    A = port_lib.PortModel(st.grid)
    A.load(st)
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev)
    d_b = torch.empty(n, dtype=torch.float64, device=dev)
    d_W = torch.empty(n, dtype=torch.float64, device=dev)
    d_Wc = torch.empty(n, dtype=torch.float64, device=dev)
    rhou, rhow = st.prof["rhou"], st.prof["rhow"]

    # set-up call (looks up the scratch array's address on this device)
    d_b.copy_(torch.from_numpy(rhs[0]))
    torch.cuda.synchronize()
    G.poisson_solve_noalloc(NX, NZ, rhou, rhow, d_b.data_ptr(), d_W.data_ptr(), tol=TOL, maxit=20000,
                            stream=stream.cuda_stream)
    torch.cuda.synchronize()

    for b in rhs:   # two calls in a row
        d_b.copy_(torch.from_numpy(b))
        d_W.fill_(float("nan"))                  # the incoming W must be ignored
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info(dev)[0]
        it, rel = G.poisson_solve_noalloc(NX, NZ, rhou, rhow, d_b.data_ptr(), d_W.data_ptr(), tol=TOL,
                                          maxit=20000, stream=stream.cuda_stream)
        free1 = torch.cuda.mem_get_info(dev)[0]
        assert free1 == free0, "the call changed the device's free memory"
        assert it > 0 and rel <= TOL
        W_na = d_W.cpu().numpy()
        true_rel = np.linalg.norm(b - A.apply_A(W_na)) / np.linalg.norm(b)
        assert true_rel <= 10 * TOL, true_rel

        g.synchronize()
        itc, relc = g.poisson_solve_device(d_b.data_ptr(), d_Wc.data_ptr(), tol=TOL)
        g.synchronize()
        assert relc <= TOL
        W_ctx = d_Wc.cpu().numpy()
        assert np.isfinite(W_na).all()
        assert rel_l2(W_na, W_ctx) <= AGREE
    g.close()
    A.close()
