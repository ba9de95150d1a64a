"""The allocation-free Verlet-list entry point, amlp_nlist_build_noalloc.

It exists for callers that may not allocate device memory at all, not even
a workspace. One example is a plug-in inside a host program that owns every
GPU buffer under a fixed memory budget. Such a caller can still use this entry
point, because its scratch is a fixed array inside the library. This file
checks, through the C ABI, that the entry point returns exactly the list of
the ordinary entry point (which takes a caller workspace). It checks two calls
in a row with different inputs, so that contents the shared array keeps from
the first call cannot leak into the second. It also checks that sizes beyond
the array's limit are refused.

It is collected last on purpose, and it passes both alone and after the other tests.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from amlp import _lib  # noqa: E402
from amlp.configs import make_state  # noqa: E402

DEV = torch.device("cuda:0")


def _workspace_list(pos_t, n, L, r):
    ws = torch.empty(_lib.size_query("amlp_nlist_workspace_bytes", n, L, r), dtype=torch.uint8, device=DEV)
    cnt = torch.zeros(1, dtype=torch.int64, device=DEV)
    cap = n * 128
    out = torch.empty(cap, 2, dtype=torch.int32, device=DEV)
    _lib.call("amlp_nlist_build", pos_t.data_ptr(), n, L, r, out.data_ptr(), cap, cnt.data_ptr(), ws.data_ptr(),
              ws.numel(), torch.cuda.current_stream().cuda_stream)
    k = int(cnt.item())
    assert k <= cap
    return out[:k].cpu().numpy()


def _noalloc_list(pos_t, n, L, r):
    cnt = torch.full((1,), -1, dtype=torch.int64, device=DEV)
    cap = n * 128
    out = torch.full((cap, 2), -7, dtype=torch.int32, device=DEV)
    _lib.call("amlp_nlist_build_noalloc", pos_t.data_ptr(), n, L, r, out.data_ptr(), cap, cnt.data_ptr(),
              torch.cuda.current_stream().cuda_stream)
    k = int(cnt.item())
    assert k <= cap
    return out[:k].cpu().numpy()


def test_noalloc_matches_workspace_entry_point_twice():
    # two different systems one after the other: the second call must not see the first one's scratch
    cases = [make_state(20000, "cube26", 0.45, seed=21), make_state(3000, "cyl24", 0.30, seed=22)]
    for s in cases:
        _check_same_list(s.pos, s.L)


def test_noalloc_box_beyond_its_cell_limit():
    # a box of 230 at radius 4.5 would take 51 cells per edge; the entry point caps them at 48
    # (larger cells, the same list)
    L = np.float32(230.0)
    assert L / 4.5 > 48
    pos = (np.random.default_rng(23).random((40000, 3)) * L - L / 2).astype(np.float32)
    _check_same_list(pos, float(L))


def _check_same_list(pos, L):
    pos_t = torch.tensor(pos, device=DEV)
    ref = _workspace_list(pos_t, len(pos), L, 4.5)
    got = _noalloc_list(pos_t, len(pos), L, 4.5)
    assert len(ref) > 0
    assert np.array_equal(got, ref)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    n = 262144 + 1
    pos_t = torch.zeros(n, 3, device=DEV)
    cnt = torch.zeros(1, dtype=torch.int64, device=DEV)
    out = torch.empty(16, 2, dtype=torch.int32, device=DEV)
    st = _lib.call_status("amlp_nlist_build_noalloc", pos_t.data_ptr(), n, 100.0, 4.5, out.data_ptr(), 16,
                          cnt.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert st == 6 and "scratch" in _lib.status_string(st)
