"""pf_sort_particles_static, the sort that takes no workspace, against
pf_sort_particles through the C ABI.

The sort is integer work, so the tolerance is zero: keys, permutation, cell
offsets and both particle streams must match bit for bit.  Every case calls
the static variant twice in a row on different inputs, so that state left in
its static scratch by one call cannot reach the next unnoticed.  This file is
collected last so that it also runs after every other GPU test has used the
library on the same device.
"""

import ctypes as C
import zlib

import numpy as np
import pytest
import torch

from oracle import oracle as O
from pfflip import Config, scenes
from pfflip import _native as N

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _inputs(pos, vel):
    n = len(pos)
    p4 = torch.zeros((max(n, 1), 4), dtype=torch.float32, device=DEV)
    v4 = torch.zeros((max(n, 1), 4), dtype=torch.float32, device=DEV)
    if n:
        p4[:n, :3] = torch.from_numpy(pos).to(DEV)
        v4[:n, :3] = torch.from_numpy(vel).to(DEV)
        v4.view(torch.int32)[:n, 3] = torch.arange(n, dtype=torch.int32, device=DEV)
    return p4, v4


def _outputs(n, res):
    po = torch.full((max(n, 1), 4), np.nan, dtype=torch.float32, device=DEV)
    vo = torch.full((max(n, 1), 4), np.nan, dtype=torch.float32, device=DEV)
    keys = torch.full((max(n, 1),), -7, dtype=torch.int32, device=DEV)
    perm = torch.full((max(n, 1),), -7, dtype=torch.int32, device=DEV)
    start = torch.full((int(np.prod(res)) + 1,), -7, dtype=torch.int32, device=DEV)
    return po, vo, keys, perm, start


def _host(n, po, vo, keys, perm, start):
    torch.cuda.synchronize()
    return (keys[:n].cpu().numpy(), perm[:n].cpu().numpy(), start.cpu().numpy(),
            po[:n].cpu().numpy(), vo[:n].cpu().numpy())


def sort_with_workspace(pos, vel, res, dx):
    n = len(pos)
    g = N.grid(res, np.float32(dx))
    p4, v4 = _inputs(pos, vel)
    po, vo, keys, perm, start = _outputs(n, res)
    ws = torch.empty(int(N.lib().pf_sort_workspace_bytes(C.byref(g), n)), dtype=torch.uint8, device=DEV)
    N.call("pf_sort_particles", C.byref(g), n, p4.data_ptr(), v4.data_ptr(), po.data_ptr(), vo.data_ptr(),
           keys.data_ptr(), perm.data_ptr(), start.data_ptr(), ws.data_ptr(), ws.numel(), N.stream())
    return _host(n, po, vo, keys, perm, start)


def sort_static(pos, vel, res, dx):
    n = len(pos)
    g = N.grid(res, np.float32(dx))
    p4, v4 = _inputs(pos, vel)
    po, vo, keys, perm, start = _outputs(n, res)
    N.call("pf_sort_particles_static", C.byref(g), n, p4.data_ptr(), v4.data_ptr(), po.data_ptr(), vo.data_ptr(),
           keys.data_ptr(), perm.data_ptr(), start.data_ptr(), N.stream())
    return _host(n, po, vo, keys, perm, start)


def _case(name):
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    if name == "dam_break_128":
        cfg = Config(res=(128,) * 3, dx=1 / 128, ppc=8)
        pos, _, _ = scenes.dam_break(cfg)
        res, dx = cfg.res, np.float32(cfg.dx)
        pos = pos[rng.permutation(len(pos))]
    elif name == "random_ragged":  # 17,280 cells: five scan tiles, the last one partial
        res, dx = (24, 20, 36), np.float32(1 / 24)
        L = np.array(res, np.float64) * float(dx)
        pos = (rng.random((200_003, 3)) * L).astype(np.float32)
    elif name == "clustered":  # cells with more than 32 particles
        res, dx = (24, 20, 36), np.float32(1 / 24)
        L = np.array(res, np.float64) * float(dx)
        base = (rng.random((300, 3)) * L).astype(np.float32)
        pos = np.repeat(base, 150, axis=0) + (rng.random((45000, 3)) * 1e-3 * float(dx)).astype(np.float32)
        pos = pos[rng.permutation(len(pos))]
    elif name == "walls":  # on and outside the walls: keys clamp
        res, dx = (16, 16, 16), np.float32(1 / 16)
        pos = (rng.random((5000, 3))).astype(np.float32)
        pos[:500] = 0.0
        pos[500:1000] = 1.0
        pos[1000:1500] = -0.5
        pos[1500:2000] = 7.0
    elif name == "empty":
        res, dx = (8, 8, 8), np.float32(1 / 8)
        pos = np.zeros((0, 3), np.float32)
    elif name == "max_cells":  # 512^3 = the largest grid the static scratch covers
        res, dx = (512, 512, 512), np.float32(1 / 512)
        pos = rng.random((100_000, 3)).astype(np.float32)
    else:
        raise ValueError(name)
    vel = rng.standard_normal(pos.shape).astype(np.float32)
    return pos, vel, res, dx


def _assert_same(a, b):
    for x, y, what in zip(a, b, ("keys", "perm", "cell_start", "pos4", "vel4")):
        assert x.shape == y.shape, what
        assert np.array_equal(x.view(np.int32), y.view(np.int32)), what


@pytest.mark.parametrize("first,second", [
    ("dam_break_128", "random_ragged"),
    ("random_ragged", "random_ragged"),
    ("clustered", "walls"),
    ("walls", "empty"),
    ("empty", "dam_break_128"),
    ("max_cells", "clustered"),
])
def test_static_sort_matches_workspace_sort_on_two_calls(first, second):
    cases = [_case(first), _case(second)]
    got = [sort_static(*c) for c in cases]  # two calls in a row
    for c, g in zip(cases, got):
        _assert_same(g, sort_with_workspace(*c))


@pytest.mark.parametrize("name", ["random_ragged", "clustered", "walls"])
def test_static_sort_matches_the_oracle(name):
    """Directly against the oracle's stable CPU sort of the binary32 keys."""
    pos, vel, res, dx = _case(name)
    keys, perm, start, po, vo = sort_static(pos, vel, res, dx)
    k_ref, p_ref, s_ref = O.sort_by_cell(pos, dx, res)
    assert np.array_equal(start, s_ref)
    assert np.array_equal(perm, p_ref)
    assert np.array_equal(keys, k_ref[p_ref])
    assert np.array_equal(po[:, :3], pos[p_ref]) and np.array_equal(vo[:, :3], vel[p_ref])
    assert np.array_equal(vo[:, 3].view(np.int32), p_ref)


def test_static_sort_leaves_free_device_memory_unchanged():
    """The property the entry point exists for: after one warm-up call (which
    loads the kernels), further calls change no device allocation."""
    pos, vel, res, dx = _case("random_ragged")
    n = len(pos)
    g = N.grid(res, np.float32(dx))
    p4, v4 = _inputs(pos, vel)
    po, vo, keys, perm, start = _outputs(n, res)
    args = (C.byref(g), n, p4.data_ptr(), v4.data_ptr(), po.data_ptr(), vo.data_ptr(), keys.data_ptr(),
            perm.data_ptr(), start.data_ptr(), N.stream())
    N.call("pf_sort_particles_static", *args)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        N.call("pf_sort_particles_static", *args)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_static_sort_rejects_overlapping_scratch():
    """pos4_out holds the keys and ranks for the whole call: an output that
    shares bytes with it (or with an input) is refused before any launch."""
    pos, vel, res, dx = _case("walls")
    n = len(pos)
    g = N.grid(res, np.float32(dx))
    p4, v4 = _inputs(pos, vel)
    po, vo, keys, perm, start = _outputs(n, res)
    big = torch.zeros((2 * n, 4), dtype=torch.float32, device=DEV)
    before = N.launch_count()
    # perm_out inside pos4_out's bytes
    rc = N.lib().pf_sort_particles_static(C.byref(g), n, p4.data_ptr(), v4.data_ptr(), big.data_ptr(),
                                         vo.data_ptr(), keys.data_ptr(), big.data_ptr() + 16 * n - 64,
                                         start.data_ptr(), N.stream())
    assert rc == N.PF_ERR_ARG and "overlaps" in N.last_error()
    # vel4_out overlapping vel4_in by one particle
    vv = torch.zeros((2 * n, 4), dtype=torch.float32, device=DEV)
    vv[:n] = v4[:n]
    rc = N.lib().pf_sort_particles_static(C.byref(g), n, p4.data_ptr(), vv.data_ptr(), po.data_ptr(),
                                         vv.data_ptr() + 16 * (n - 1), keys.data_ptr(), perm.data_ptr(),
                                         start.data_ptr(), N.stream())
    assert rc == N.PF_ERR_ARG and "overlaps" in N.last_error()
    assert N.launch_count() == before


def test_static_sort_rejects_grid_beyond_its_scratch():
    res = (512, 512, 513)
    g = N.grid(res, np.float32(1 / 512))
    p4, v4 = _inputs(np.zeros((4, 3), np.float32), np.zeros((4, 3), np.float32))
    po, vo = torch.empty_like(p4), torch.empty_like(v4)
    keys = torch.zeros(4, dtype=torch.int32, device=DEV)
    perm = torch.zeros(4, dtype=torch.int32, device=DEV)
    # sized for the whole grid, so the call would stay in bounds even if it were not rejected
    start = torch.zeros(int(np.prod(res)) + 1, dtype=torch.int32, device=DEV)
    before = N.launch_count()
    rc = N.lib().pf_sort_particles_static(C.byref(g), 4, p4.data_ptr(), v4.data_ptr(), po.data_ptr(), vo.data_ptr(),
                                         keys.data_ptr(), perm.data_ptr(), start.data_ptr(), N.stream())
    assert rc == N.PF_ERR_ARG
    assert "512^3" in N.last_error()
    assert N.launch_count() == before
    assert int(np.prod(res)) > N.PF_SORT_STATIC_MAX_CELLS
