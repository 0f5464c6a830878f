"""qs_sample_noalloc: the allocation-free sampling entry point.

It serves callers that cannot allocate device memory (their device memory is
already handed to a pool allocator, or they are plain C / FFI callers that own
only the state, the uniforms and the output).  This test calls it through the
C-ABI and checks that it returns exactly the indices of the workspace-based
entry points (qs_sample_prepare + qs_sample), on two calls in a row: the
second call reuses the shared static tree the first one left behind.  The file
is named so pytest collects it last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _state(n, seed, dtype):
    import torch
    rng = np.random.default_rng(seed)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    v /= np.linalg.norm(v)
    return torch.from_numpy(v.astype(dtype)).cuda()


def _density(n, seed, dtype):
    """A random n-qubit density matrix (PSD, trace 1) as a 2^n x 2^n device array."""
    import torch
    rng = np.random.default_rng(seed)
    a = rng.normal(size=(1 << n, 1 << n)) + 1j * rng.normal(size=(1 << n, 1 << n))
    rho = a @ a.conj().T
    rho /= np.trace(rho).real
    return torch.from_numpy(np.ascontiguousarray(rho.astype(dtype))).cuda()


def _with_workspace(lib, N, vec, n, dt, u, shots, mode, src=None):
    import torch
    src = N.QS_SRC_SV if src is None else src
    wsb = lib.qs_sample_ws_bytes(n)
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    out = torch.empty(shots, dtype=torch.int64, device="cuda")
    N.call("qs_sample_prepare", C.c_void_p(vec.data_ptr()), n, dt, src, C.c_void_p(ws.data_ptr()), wsb, None)
    N.call("qs_sample", C.c_void_p(vec.data_ptr()), n, dt, src, C.c_void_p(ws.data_ptr()), wsb,
           C.c_void_p(u.data_ptr()), shots, mode, C.c_void_p(out.data_ptr()), None)
    return out


def _no_alloc(N, vec, n, dt, u, shots, mode, src=None):
    import torch
    src = N.QS_SRC_SV if src is None else src
    out = torch.empty(shots, dtype=torch.int64, device="cuda")
    N.call("qs_sample_noalloc", C.c_void_p(vec.data_ptr()), n, dt, src, C.c_void_p(u.data_ptr()), shots,
           mode, C.c_void_p(out.data_ptr()), None)
    return out


def test_noalloc_sampling_matches_workspace_entry_point_twice(cuda_ok):
    import torch
    from quict_b200 import _native as N
    lib = N.load()
    # two calls in a row with different sizes, precisions and modes: the second
    # call must not see anything of the first one's tree
    cases = [(20, np.complex128, N.QS_C128, N.QS_SAMPLE_CDF, 4096, 1),
             (13, np.complex64, N.QS_C64, N.QS_SAMPLE_SEQ, 1024, 2)]
    for n, npdt, dt, mode, shots, seed in cases:
        vec = _state(n, seed, npdt)
        per = 1 if mode == N.QS_SAMPLE_CDF else n
        u = torch.from_numpy(np.random.default_rng(seed + 10).random(shots * per)).cuda()
        want = _with_workspace(lib, N, vec, n, dt, u, shots, mode)
        got = _no_alloc(N, vec, n, dt, u, shots, mode)
        torch.cuda.synchronize()
        assert torch.equal(got, want)


def test_noalloc_at_its_largest_size_and_on_a_density_matrix(cuda_ok):
    """n = 26 fills the static tree exactly (2 * 2^16 doubles); a density
    matrix source reads the diagonal of a 2^n x 2^n array."""
    import torch
    from quict_b200 import _native as N
    lib = N.load()
    n = N.QS_NOALLOC_SAMPLE_MAX_QUBITS
    vec = _state(n, 3, np.complex64)
    u = torch.from_numpy(np.random.default_rng(13).random(8192)).cuda()
    want = _with_workspace(lib, N, vec, n, N.QS_C64, u, 8192, N.QS_SAMPLE_CDF)
    got = _no_alloc(N, vec, n, N.QS_C64, u, 8192, N.QS_SAMPLE_CDF)
    torch.cuda.synchronize()
    assert torch.equal(got, want)
    del vec
    for mode, per in ((N.QS_SAMPLE_CDF, 1), (N.QS_SAMPLE_SEQ, 8)):
        rho = _density(8, 4, np.complex128)
        u = torch.from_numpy(np.random.default_rng(14).random(2048 * per)).cuda()
        want = _with_workspace(lib, N, rho, 8, N.QS_C128, u, 2048, mode, N.QS_SRC_DM)
        got = _no_alloc(N, rho, 8, N.QS_C128, u, 2048, mode, N.QS_SRC_DM)
        torch.cuda.synchronize()
        assert torch.equal(got, want)


def test_noalloc_rejects_sizes_beyond_its_limit(cuda_ok):
    import torch
    from quict_b200 import _native as N
    lib = N.load()
    fake = C.c_void_p(0x1000)  # never dereferenced: the size check comes first
    rc = lib.qs_sample_noalloc(fake, 27, N.QS_C64, N.QS_SRC_SV, fake, 1,
                               N.QS_SAMPLE_CDF, fake, None)
    assert rc == N.QS_EINVAL and b"limit" in lib.qs_last_error()
