"""lica_gpu_trdiag3_noalloc_device: TRDIAG3 for callers that cannot allocate device
memory (their memory comes from a fixed pool, or they cannot afford the device-wide
synchronisation or the out-of-memory risk of cudaMalloc inside a solver loop).

It must give the same solution as the allocating entry point lica_gpu_trdiag3_device
(same kernel, so the tolerance is exact), on consecutive calls that reuse its fixed
scratch, and must refuse systems larger than that scratch.  This file is collected
last so that a run stopping at the first failure has run every other test first.
"""
import numpy as np
import pytest

from lica_boiling1d_b200 import native

pytestmark = pytest.mark.gpu


def _system(rng, ld, n):
    A = rng.uniform(-1, 1, (ld, n))
    C = rng.uniform(-1, 1, (ld, n))
    B = rng.uniform(-1, 1, (ld, n)) + np.sign(rng.uniform(-1, 1, (ld, n))) * 3.0
    R = rng.standard_normal((ld, n))
    return A, B, C, R


def _dev(a):
    import torch
    # a Fortran (ld, n) array is a C-contiguous (n, ld) tensor
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda()


def test_noalloc_matches_allocating_entry_on_two_calls():
    import torch
    lib = native.lib()
    rng = np.random.default_rng(2024)
    stream = torch.cuda.current_stream().cuda_stream
    for call, (ld, n, l1, l2, ll1, ll2) in enumerate([(300, 129, 2, 128, 1, 297), (512, 512, 1, 512, 3, 512)]):
        A, B, C, R = _system(rng, ld, n)
        dA, dB, dC = _dev(A), _dev(B), _dev(C)
        R_ref, U_ref = _dev(R), torch.zeros((n, ld), dtype=torch.float64, device="cuda")
        R_new, U_new = _dev(R), torch.zeros((n, ld), dtype=torch.float64, device="cuda")
        native.check(lib.lica_gpu_trdiag3_device(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), R_ref.data_ptr(),
                                                 U_ref.data_ptr(), l1, l2, ll1, ll2, ld, stream), "trdiag3_device")
        native.check(lib.lica_gpu_trdiag3_noalloc_device(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(),
                                                         R_new.data_ptr(), U_new.data_ptr(), l1, l2, ll1, ll2, ld,
                                                         stream), "trdiag3_noalloc_device")
        torch.cuda.synchronize()
        assert torch.equal(U_new, U_ref), f"call {call}: solutions differ"
        assert torch.equal(R_new, R_ref), f"call {call}: R differs"
        # and the solution solves every line's system (lines ll1..ll2, unknowns l1..l2)
        Ucpu = U_new.cpu().numpy().T
        i = np.arange(ll1 - 1, ll2)[:, None]
        j = np.arange(l1 - 1, l2)[None, :]
        res = B[i, j] * Ucpu[i, j] - R[i, j]
        res[:, 1:] += A[i, j[:, 1:]] * Ucpu[i, j[:, :-1]]
        res[:, :-1] += C[i, j[:, :-1]] * Ucpu[i, j[:, 1:]]
        assert np.abs(res).max() < 1e-10 * max(1.0, np.abs(R).max())


def test_noalloc_rejects_systems_larger_than_its_scratch():
    import torch
    lib = native.lib()
    ld, n = 1024, 257   # ld * l2 = 263168 > 262144 doubles
    t = torch.zeros((n, ld), dtype=torch.float64, device="cuda")
    code = lib.lica_gpu_trdiag3_noalloc_device(t.data_ptr(), t.data_ptr(), t.data_ptr(), t.data_ptr(), t.data_ptr(),
                                               1, n, 1, ld, ld, torch.cuda.current_stream().cuda_stream)
    assert code == 4
    assert b"262144" in lib.lica_last_error()
