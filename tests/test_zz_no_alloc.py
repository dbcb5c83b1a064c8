"""The allocation-free reduction fm_reduce_static, checked against fm_reduce.

fm_reduce_static is there for callers that cannot call cudaMalloc -- an
application that reserved its device memory up front in its own pool, or code
running where an allocation would stall the device or break an asynchronous
pipeline.  It sums buffers the caller owns and keeps its intermediate sums in
a static device array instead of allocating.

The GPU test copies a lattice's state into caller-owned device buffers (a
plane stride wider than the lattice's own) and checks two consecutive calls of
the static entry point against the lattice's fm_reduce, within the domain-sum
tolerance the parity tests use.  The file is named to be collected last, so a
failure here comes after every other test has run.
"""
import numpy as np
import pytest

from fluidmaxxer_b200 import _abi

SUM_TOL = 1e-6          # relative, as for the domain sums in test_gpu_parity.py
MAX_CELLS = 134_217_728


def test_static_reduce_rejects_sizes_beyond_its_scratch():
    lib = _abi.lib()
    out = np.zeros(3)
    # rejected before any device work: no GPU needed
    rc = lib.fm_reduce_static(None, None, None, MAX_CELLS + 1, MAX_CELLS + 1, out.ctypes.data, None)
    assert rc == _abi.FM_ERR_ARG
    assert b"134217728" in lib.fm_last_error()
    assert lib.fm_reduce_static(None, None, None, 10, 20, out.ctypes.data, None) == _abi.FM_ERR_ARG
    assert lib.fm_reduce_static(None, None, None, 10, 10, None, None) == _abi.FM_ERR_ARG
    assert lib.fm_reduce_static(None, None, None, 10, -1, out.ctypes.data, None) == _abi.FM_ERR_ARG


@pytest.mark.gpu
def test_static_reduce_matches_fm_reduce_on_two_calls():
    import torch

    from fluidmaxxer_b200 import lattice, problems

    p = problems.channel_small(nx=48, ny=24, nz=20, steps=60)
    L = lattice.from_problem(p, "f32")
    L.step(p.steps)
    ref = L.reduce()
    st = L.get_state()
    L.close()

    n = p.n_cells
    ns = (n + 31) // 32 * 32 + 64
    dev = torch.device("cuda:0")
    f = torch.zeros(19, ns, dtype=torch.float32, device=dev)
    f[:, :n] = torch.from_numpy(st["f"].astype(np.float32)).to(dev)
    phi = torch.from_numpy(st["phi"].astype(np.float32)).to(dev)
    q = torch.from_numpy(st["q"].astype(np.float32)).to(dev)
    torch.cuda.synchronize()

    lib = _abi.lib()
    for call in range(2):
        out = np.full(3, np.nan)
        rc = lib.fm_reduce_static(f.data_ptr(), phi.data_ptr(), q.data_ptr(), ns, n, out.ctypes.data, None)
        assert rc == 0, lib.fm_last_error()
        for i in range(3):
            assert abs(out[i] - ref[i]) <= SUM_TOL * max(abs(ref[i]), 1e-30), (call, i, out[i], ref[i])
