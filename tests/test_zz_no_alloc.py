"""The allocation-free refinement entry point, gsj_refine_pairs_noalloc, through the C ABI.

It exists for callers that cannot allocate device memory while they run (a server that reserved its device
memory budget up front, or a request path that cannot take cudaMalloc's implicit synchronisation): they pass
device buffers, and the refinement's scratch comes from one static device array. Its results must equal those
of the ordinary entry point gsj_refine_pairs bit for bit (the tolerance all parity tests here use), call after
call, since every call reuses the same static array. Collected last so a failure here cannot hide other tests.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    import torch

    import gsj
    from gsj import gen
    eng = gsj.Engine(0)
    # multipolygons and holes give pairs larger than the shared-memory lists, so both paths see big edge lists
    P = eng.upload_polygons(gen.layer_parcels(20000, (-118.3, 33.95, -118.1, 34.15), seed=5))
    Q = eng.upload_polygons(gen.layer_parcels(15000, (-118.3, 33.95, -118.1, 34.15), seed=6))
    yield eng, P, Q, torch, gsj
    P.free(); Q.free(); eng.close()


def call_noalloc(gsj, torch, eng, A, B, pairs, rel):
    n = len(pairs)
    dev = torch.device("cuda", 0)
    d_pairs = torch.from_numpy(np.ascontiguousarray(pairs, dtype=np.uint32).view(np.int32)).to(dev)
    d_flag = torch.full((n,), 7, dtype=torch.uint8, device=dev)          # garbage the call must overwrite
    d_area = torch.full((n,), -1.0, dtype=torch.float64, device=dev)
    d_ev = torch.full((n, 4), -1.0, dtype=torch.float64, device=dev) if rel else None
    d_evb = torch.full((n,), -1, dtype=torch.int32, device=dev) if rel else None
    torch.cuda.synchronize()
    rp = gsj.refine_params(want_area=True, want_relate=rel)
    rc = gsj.lib().gsj_refine_pairs_noalloc(eng.ctx, A.h, B.h, ctypes.c_void_p(d_pairs.data_ptr()), n, ctypes.byref(rp),
                                            ctypes.c_void_p(d_flag.data_ptr()), ctypes.c_void_p(d_area.data_ptr()),
                                            ctypes.c_void_p(d_ev.data_ptr()) if rel else None,
                                            ctypes.c_void_p(d_evb.data_ptr()) if rel else None)
    assert rc == 0, gsj.lib().gsj_last_error(eng.ctx)
    out = [d_flag.cpu().numpy(), d_area.cpu().numpy()]
    if rel:
        out += [d_ev.cpu().numpy(), d_evb.cpu().numpy().view(np.uint32)]
    return out


@pytest.mark.parametrize("rel", [False, True])
def test_noalloc_matches_refine_pairs_twice(setup, rel):
    eng, P, Q, torch, gsj = setup
    for A, B, upper in ((P, P, True), (P, Q, False)):
        pairs = eng.candidates(A, B, upper=upper)
        f, a, e, b = eng.refine_pairs(A, B, pairs, want_area=True, want_relate=rel)
        for _ in range(2):                      # two calls in a row share the static array
            got = call_noalloc(gsj, torch, eng, A, B, pairs, rel)
            assert np.array_equal(got[0], f)
            assert np.array_equal(got[1], a)
            if rel:
                assert np.array_equal(got[2], e) and np.array_equal(got[3], b)
        assert (f == 1).sum() > 1000


def test_noalloc_rejects_oversized_geometry(setup):
    """One polygon of 600k edges needs a larger per-warp slab than the static array: a clear error, no launch."""
    eng, P, Q, torch, gsj = setup
    from gsj.gen import PolygonSet
    t = np.linspace(0, 2 * np.pi, 600001)
    ring = np.stack([-118.2 + 0.01 * np.cos(t), 34.05 + 0.01 * np.sin(t)], 1)
    ring[-1] = ring[0]
    big = eng.upload_polygons(PolygonSet(np.array([0, 1], np.uint64), np.array([0, len(ring)], np.uint64), ring))
    d_pairs = torch.zeros(2, dtype=torch.int32, device="cuda")
    d_flag = torch.zeros(1, dtype=torch.uint8, device="cuda")
    rc = gsj.lib().gsj_refine_pairs_noalloc(eng.ctx, big.h, big.h, ctypes.c_void_p(d_pairs.data_ptr()), 1, None,
                                            ctypes.c_void_p(d_flag.data_ptr()), None, None, None)
    assert rc == 1 and b"static scratch" in gsj.lib().gsj_last_error(eng.ctx)
    big.free()
