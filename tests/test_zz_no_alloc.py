"""tgb_partition_noalloc: the partition entry point for callers that cannot allocate
device memory (its scratch is a fixed device array inside the library).

It must give exactly what tgb_partition (caller-provided workspace) gives, call after
call, although every call reuses the same library-owned scratch.  This file is
collected last so that a failure here does not hide the other tests in a run that
stops at the first failure.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _p(t):
    return C.c_void_p(t.data_ptr())


def _with_workspace(L, codes, stride, rows, n_rows, feat, thr, ml):
    out = torch.full((max(1, n_rows),), -1, dtype=torch.int32, device="cuda")
    nl = torch.zeros(1, dtype=torch.int32, device="cuda")
    wsb = L.tgb_partition_workspace_bytes(n_rows)
    ws = torch.zeros(wsb, dtype=torch.uint8, device="cuda")
    rc = L.tgb_partition(_p(codes), stride, _p(rows), n_rows, feat, thr, ml, _p(out), _p(nl), _p(ws), wsb, None)
    assert rc == 0, L.tgb_last_error()
    torch.cuda.synchronize()
    return out.cpu().numpy()[:n_rows], int(nl.item())


def _without_workspace(L, codes, stride, rows, n_rows, feat, thr, ml):
    out = torch.full((max(1, n_rows),), -1, dtype=torch.int32, device="cuda")
    nl = torch.full((1,), -7, dtype=torch.int32, device="cuda")
    rc = L.tgb_partition_noalloc(_p(codes), stride, _p(rows), n_rows, feat, thr, ml, _p(out), _p(nl), None)
    assert rc == 0, L.tgb_last_error()
    torch.cuda.synchronize()
    return out.cpu().numpy()[:n_rows], int(nl.item())


def _expected(codes_h, rows_h, feat, thr, ml):
    """The stable partition as numpy states it: left rows in order, then right rows."""
    b = codes_h[rows_h, feat].astype(int)
    left = np.where(b == 0, ml == 1, b <= thr)
    return np.concatenate([rows_h[left], rows_h[~left]]), int(left.sum())


def test_partition_noalloc_matches_workspace_version_twice(native):
    L = native.lib()
    rng = np.random.default_rng(123)
    n, stride = 3_200_000, 32
    codes_h = np.zeros((n, stride), np.uint8)
    codes_h[:, :24] = rng.integers(0, 256, size=(n, 24))
    codes = torch.from_numpy(codes_h).cuda()
    # Calls in a row with different sizes and splits: each must be unaffected by the
    # previous call's leftovers in the shared scratch.  3,000,000 rows are 1,465 tiles, more
    # than the 1,184 CTAs of a launch, so the grid-stride tile loop and the running prefix
    # over the shared tile counts run too; 0 rows must report no left rows.
    cases = [(3_000_000, 9, 200, 1), (250_001, 5, 120, 1), (70_000, 17, 30, 0), (0, 3, 10, 1)]
    for n_rows, feat, thr, ml in cases:
        rows_h = np.sort(rng.choice(n, n_rows, replace=False)).astype(np.int32)
        rows = torch.from_numpy(rows_h if n_rows else np.zeros(1, np.int32)).cuda()
        a, na = _with_workspace(L, codes, stride, rows, n_rows, feat, thr, ml)
        b, nb = _without_workspace(L, codes, stride, rows, n_rows, feat, thr, ml)
        exp, n_left = _expected(codes_h, rows_h, feat, thr, ml)
        assert na == nb == n_left
        assert np.array_equal(b, exp)
        assert np.array_equal(a, b)


def test_partition_noalloc_rejects_oversize(native):
    L = native.lib()
    dummy = torch.zeros(16, dtype=torch.int32, device="cuda")
    rc = L.tgb_partition_noalloc(_p(dummy), 16, _p(dummy), (1 << 24) + 1, 0, 0, 1, _p(dummy), _p(dummy), None)
    assert rc == -1
    assert "n_rows" in L.tgb_last_error().decode()
