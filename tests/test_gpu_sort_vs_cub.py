"""gs_stage_sort against the library sort the reference calls: CUB's
DeviceRadixSort::SortPairs as sortTileList runs it (core/gaussian_render.cu:
591-632, built into oracle/_ref/libgsref.so), on identical pairs and key
widths.  Both are stable LSD radix sorts, so the sorted keys and the values
carried with them must be identical, ties included."""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def ref():
    import oracle
    if not os.path.exists(oracle.REF_LIB):
        pytest.skip("reference harness not built")
    return oracle.Ref()


@pytest.mark.parametrize("n,bits", [(1, 44), (4097, 44), (2_600_000, 44), (3_000_001, 51), (500_000, 64)])
def test_sort_identical_to_cub(gs, ref, n, bits):
    rng = np.random.default_rng(n + bits)
    if bits == 64:
        keys = rng.integers(0, 2 ** 63, n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, n, dtype=np.uint64)
    else:
        hi = rng.integers(0, 1 << (bits - 32), n).astype(np.uint64)
        lo = rng.integers(0, 1 << 14, n).astype(np.uint64)  # many equal keys
        keys = (hi << np.uint64(32)) | lo
    vals = rng.permutation(n).astype(np.int32)
    src_k = torch.from_numpy(keys.view(np.int64).copy()).cuda()
    src_v = torch.from_numpy(vals).cuda()
    k0, k1 = torch.empty_like(src_k), torch.empty_like(src_k)
    v0, v1 = torch.empty_like(src_v), torch.empty_like(src_v)
    sel = ctypes.c_int(0)
    ms = ref.lib.gsref_cub_sort_timed(n, bits, src_k.data_ptr(), src_v.data_ptr(), k0.data_ptr(), k1.data_ptr(),
                                      v0.data_ptr(), v1.data_ptr(), 2, ctypes.byref(sel))
    torch.cuda.synchronize()
    assert ms >= 0
    cub_k = (k1 if sel.value else k0).cpu().numpy().view(np.uint64)
    cub_v = (v1 if sel.value else v0).cpu().numpy()
    ctx = gs.Context(0)
    k0.copy_(src_k)
    v0.copy_(src_v)
    s = gs.stage_sort(ctx, n, bits, k0, v0, k1, v1)
    torch.cuda.synchronize()
    ours_k = (k1 if s else k0).cpu().numpy().view(np.uint64)
    ours_v = (v1 if s else v0).cpu().numpy()
    ctx.close()
    assert np.array_equal(ours_k, cub_k)
    assert np.array_equal(ours_v, cub_v)
