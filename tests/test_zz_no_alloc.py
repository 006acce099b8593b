"""The allocation-free entry point gfix_theta_functional_noalloc.

Callers that cannot allocate device memory when they call in -- codes that
hand all of HBM to their own arena allocator, and stream-ordered pipelines in
which a cudaMalloc would synchronise the device -- use this variant: its only
scratch is a fixed device array inside the library.  Its results must equal
those of the ordinary, allocating entry point (gfix_observables) on repeated
calls, the second of which reuses the scratch left by the first.  This file
is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from glu_b200 import _lib, gfix  # noqa: E402


@pytest.mark.parametrize("side_stream", [False, True])
@pytest.mark.parametrize("case", ["lat400", "hb8"])
def test_noalloc_matches_allocating_entry_point(case, side_stream, request):
    """Two calls in a row on the caller's stream (the default one, or a
    side stream that the links were written on) give the allocating entry
    point's values."""
    g = request.getfixturevalue(case)
    dims = tuple(int(d) for d in g["dims"])
    lib = _lib.load()
    ref = gfix.observables(g["links"], dims)[:2]
    U = np.ascontiguousarray(g["links"], dtype=np.complex128)
    host = torch.from_numpy(U.view(np.float64).reshape(-1)).pin_memory()
    stream = torch.cuda.Stream() if side_stream else torch.cuda.current_stream()
    cd = (C.c_size_t * 4)(*dims)
    with torch.cuda.stream(stream):
        # the links arrive by an asynchronous copy on the same stream: the
        # call is ordered after it without any synchronisation
        d_links = host.to("cuda", non_blocking=True)
        for _ in range(2):
            d_out = torch.full((2,), float("nan"), dtype=torch.float64,
                               device="cuda")
            rc = lib.gfix_theta_functional_noalloc(
                d_links.data_ptr(), cd, d_out.data_ptr(), stream.cuda_stream)
            assert rc == 0, lib.gfix_noalloc_error()
            got = d_out.cpu().numpy()  # waits for this stream's work
            assert abs(got[0] - ref[0]) <= 1e-12 * abs(ref[0])
            assert abs(got[1] - ref[1]) <= 1e-14


@pytest.mark.parametrize("dims", [(64, 64, 64, 128),
                                  # the product wraps around 2^64 to 2^24
                                  ((1 << 40) + 1, 1 << 22, 2, 2)])
def test_noalloc_rejects_lattices_beyond_its_scratch(dims):
    lib = _lib.load()
    d = torch.zeros(16, dtype=torch.float64, device="cuda")
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    cd = (C.c_size_t * 4)(*dims)
    assert lib.gfix_theta_functional_noalloc(d.data_ptr(), cd,
                                             out.data_ptr(), None) == -1
    assert b"16777216" in lib.gfix_noalloc_error()
