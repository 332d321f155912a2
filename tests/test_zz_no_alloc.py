"""The gridding entry point that allocates nothing
(mlg_gridder_n2u_leight_noalloc), for callers that cannot allocate device
memory while they run: a program that reserved the GPU's memory for its own
pool, or an embedding that forbids allocation after start-up.  The caller
owns every input and output buffer (here: torch CUDA tensors); the entry
point takes its scratch from the library's fixed device array.  Its results
must match the allocating entry point's (mlg_gridder_n2u_leight, the
cell-binned gather) within the gridder's tolerance (relative L2 1e-5: the
two forms sum each cell's samples in different orders), on two calls in a
row -- the second call reuses the scratch left by the first -- and the
second call must leave the device's free memory unchanged.

Kept in a file of its own that pytest collects last."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def test_noalloc_gridder_matches_allocating_gridder_twice():
    import torch

    from monalisa_b200 import _native as N

    rng = np.random.default_rng(404)
    imDim, Nn, nCh, nPt, nWin = 3, 32, 4, 60000, 3
    # half the samples crowd the centre so that bins are split into chunks
    # and partial tiles (the scratch's largest users) are exercised
    t = np.concatenate([rng.normal(Nn / 2 + 1, 1.5, (imDim, nPt // 2)),
                        rng.uniform(0.5, Nn + 0.5, (imDim, nPt - nPt // 2))], 1).astype(np.float32)
    aR = rng.standard_normal((nPt, nCh)).astype(np.float32)  # [nCh, nPt] column-major
    aI = rng.standard_normal((nPt, nCh)).astype(np.float32)
    Dn = rng.uniform(0.1, 1.0, nPt).astype(np.float32)
    nu = Nn ** imDim
    refR = np.zeros((nu, nCh), np.float32)
    refI = np.zeros((nu, nCh), np.float32)
    ts = [np.ascontiguousarray(t[d]) for d in range(imDim)]
    N.call("mlg_gridder_n2u_leight", imDim, N.fptr(aR), N.fptr(aI), N.fptr(ts[0]), N.fptr(ts[1]), N.fptr(ts[2]),
           N.fptr(Dn), nCh, nPt, Nn, Nn, Nn, nWin, 0.61, 10.0, N.fptr(refR), N.fptr(refI))

    dev = torch.device("cuda", 0)
    d_in = [torch.from_numpy(v).to(dev) for v in (aR, aI, ts[0], ts[1], ts[2], Dn)]
    bR = torch.empty((nu, nCh), dtype=torch.float32, device=dev)
    bI = torch.empty((nu, nCh), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    for call in range(2):
        bR.fill_(float("nan"))  # every output cell must be written by the call
        bI.fill_(float("nan"))
        torch.cuda.synchronize(dev)
        free_before = torch.cuda.mem_get_info(dev)[0]
        N.call("mlg_gridder_n2u_leight_noalloc", imDim, *[ctypes.c_void_p(x.data_ptr()) for x in d_in], nCh, nPt,
               Nn, Nn, Nn, nWin, 0.61, 10.0, ctypes.c_void_p(bR.data_ptr()), ctypes.c_void_p(bI.data_ptr()),
               ctypes.c_void_p(stream.cuda_stream))
        torch.cuda.synchronize(dev)
        if call == 1:  # the first call may load the library's kernels; the second takes no memory
            assert torch.cuda.mem_get_info(dev)[0] == free_before, "the call changed the device's free memory"
        gotR, gotI = bR.cpu().numpy(), bI.cpu().numpy()
        assert np.isfinite(gotR).all() and np.isfinite(gotI).all(), f"call {call}: unwritten output cells"
        assert _rel(gotR + 1j * gotI, refR + 1j * refI) <= 1e-5, f"call {call}"


def test_noalloc_gridder_rejects_problems_beyond_its_scratch():
    import torch

    from monalisa_b200 import _native as N

    out = torch.empty(2, dtype=torch.float32, device="cuda")
    # a 1536 x 1024 x 1024 grid needs more tile counters than the fixed
    # scratch holds: refused before anything is launched
    with pytest.raises(N.MonalisaError, match="no-allocation scratch"):
        N.call("mlg_gridder_n2u_leight_noalloc", 3, None, None, None, None, None, None, 1, 0, 1536, 1024, 1024, 3,
               0.61, 10.0, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(out.data_ptr()), None)


def test_noalloc_gridder_rejects_too_many_tile_pairs():
    import torch

    from monalisa_b200 import _native as N

    buf = torch.zeros(4, dtype=torch.float32, device="cuda")
    p = ctypes.c_void_p(buf.data_ptr())
    # 2^28 samples on a 64^3 grid with 8 coils: each window may meet 2 x 2 x 2
    # tiles, so the 32-bit bin offsets could overflow -- refused before any
    # launch (the pointers are never read)
    with pytest.raises(N.MonalisaError, match="pairs"):
        N.call("mlg_gridder_n2u_leight_noalloc", 3, p, p, p, p, p, p, 8, 1 << 28, 64, 64, 64, 3, 0.61, 10.0, p, p,
               None)
