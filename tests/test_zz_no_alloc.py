"""The allocation-free colouring entry point (avbd_colour_graph_noalloc), called through
the C ABI, against the colouring the regular step computes (avbd_read_colours).

It serves callers that cannot allocate device memory (allocator-managed hosts, real-time
loops, fully reserved GPUs); all its scratch lives in an array built into the library.
The comparison is exact: colours are integers."""
import ctypes

import numpy as np
import pytest

from avbd_demo3d_b200 import World, _lib, scenes

pytestmark = pytest.mark.gpu


def constraint_graph(w: World):
    """Vertex flags and neighbour CSR of the constraint graph of the last step, rebuilt on
    the host from the world's readback (manifolds, joints, springs, ignore pairs)."""
    n = w.n
    pairs = [tuple(x) for x in w.manifolds()["ab"]] + [tuple(x) for x in w.joints()["ab"]]
    pairs += [tuple(x) for x in w._force_arrays["s_ab"]]
    ignores = [tuple(x) for x in w._force_arrays["i_ab"]]
    deg = np.zeros(n, np.int64)
    nbr = [[] for _ in range(n)]
    for a, b in pairs + ignores:
        if a >= 0:
            deg[a] += 1
        deg[b] += 1
    for a, b in pairs:
        if a >= 0:
            nbr[a].append(b)
            nbr[b].append(a)
    vertex = ((w.props["mass"] > 0) & (deg > 0)).astype(np.int32)
    start = np.zeros(n + 1, np.int32)
    start[1:] = np.cumsum([len(x) for x in nbr])
    other = np.array([u for x in nbr for u in x] or [0], np.int32)
    return vertex, start, other


def colour_noalloc(n, vertex, start, other, mode):
    import torch

    lib = _lib.load()
    dv = torch.from_numpy(vertex).cuda()
    ds = torch.from_numpy(start).cuda()
    do = torch.from_numpy(other).cuda()
    out = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    nc = ctypes.c_int32(-1)
    torch.cuda.synchronize()
    rc = lib.avbd_colour_graph_noalloc(n, dv.data_ptr(), ds.data_ptr(), do.data_ptr(), mode, out.data_ptr(),
                                       ctypes.byref(nc), None)
    return rc, out.cpu().numpy(), nc.value


def test_noalloc_colouring_matches_the_step(gpu):
    sc = scenes.mixed_drop(3000, 20, 12, 0.05, extent=(30, 30, 20), seed=5)
    w = World(sc)
    for call, (steps, mode) in enumerate(((12, 0), (9, 1))):
        w.set_colouring(mode)
        w.step(steps)
        expected, n_expected = w.colours()
        vertex, start, other = constraint_graph(w)
        rc, got, n_got = colour_noalloc(w.n, vertex, start, other, mode)
        assert rc == _lib.AVBD_OK, (call, rc)
        assert n_got == n_expected, (call, n_got, n_expected)
        assert np.array_equal(got, expected), call
    w.close()


def test_noalloc_calls_leave_free_device_memory_unchanged(gpu):
    """The point of the entry point: once the first call on the device has placed the
    library's scratch array, further calls take no device memory. Inputs for graphs of
    three sizes are allocated up front; the device's free-memory count (cudaMemGetInfo)
    is read after a warm-up call and again after six more calls, which must colour
    exactly like the warm-up calls."""
    import torch

    lib = _lib.load()
    sc = scenes.mixed_drop(3000, 20, 12, 0.05, extent=(30, 30, 20), seed=5)
    w = World(sc)
    w.step(12)
    vertex, start, other = constraint_graph(w)
    w.close()
    cases = []
    for n in (w.n, w.n // 2, 257):
        # a prefix of the bodies: neighbours at n or above are skipped by the entry point
        dv = torch.from_numpy(np.ascontiguousarray(vertex[:n])).cuda()
        ds = torch.from_numpy(np.ascontiguousarray(start[:n + 1])).cuda()
        do = torch.from_numpy(other).cuda()
        out = torch.full((n,), -7, dtype=torch.int32, device="cuda")
        cases.append((n, dv, ds, do, out))
    nc = ctypes.c_int32(-1)

    def call(case, mode):
        n, dv, ds, do, out = case
        rc = lib.avbd_colour_graph_noalloc(n, dv.data_ptr(), ds.data_ptr(), do.data_ptr(), mode, out.data_ptr(),
                                           ctypes.byref(nc), None)
        assert rc == _lib.AVBD_OK, (n, rc)
        return out.cpu().numpy().copy(), nc.value

    first = [call(c, 0) for c in cases]
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    again = [call(c, m) for m in (0, 1) for c in cases]
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before, (free_before, free_after)
    for (c0, n0), (c1, n1) in zip(first, again[:3]):
        assert n0 == n1 and np.array_equal(c0, c1)


def test_noalloc_rejects_oversize_and_bad_arguments(gpu):
    lib = _lib.load()
    nc = ctypes.c_int32()
    too_many = (1 << 20) + 1
    assert lib.avbd_colour_graph_noalloc(too_many, None, None, None, 0, None, ctypes.byref(nc), None) == -3
    assert lib.avbd_colour_graph_noalloc(10, None, None, None, 0, None, ctypes.byref(nc), None) == -1
    assert lib.avbd_colour_graph_noalloc(10, None, None, None, 7, None, ctypes.byref(nc), None) == -1
