"""ms_build_atom_index_noalloc: the atom index without device allocation.

Callers whose memory manager owns all device memory, or that cannot afford
cudaMalloc's device synchronisation, pass their own device buffers; the
library's scratch is a fixed device array.
This test drives the entry point through the C ABI on device buffers owned by
the caller (allocated here with PyTorch, as such a host application would with
its own allocator) and requires its index to equal, bit for bit, the index of
the allocating entry point ms_upload_binned_atoms, on two calls in a row with
different structures (the shared scratch must not leak from one call into the
next).  It also checks that oversized requests are refused with a message."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _box(x, y, z):
    # LoadAtomFile's padded box in FP32 (U.cu:1350-1355)
    f = np.float32
    return np.array([f(x.max()) + f(2), f(x.min()) - f(2), f(y.max()) + f(2), f(y.min()) - f(2),
                     f(z.max()) + f(2), f(z.min()) - f(2)], np.float32)


def _reference_index(atoms):
    from cudamultislice_b200 import ManagedMultisliceSimulation

    sim = ManagedMultisliceSimulation()
    sim.SetAtoms(*atoms)
    sim.UploadBinnedAtoms()
    out = sim.Binned()
    sim.close()
    return out


def _noalloc_index(L, atoms):
    import torch

    Z, x, y, z = atoms
    n = len(Z)
    box = _box(x, y, z)
    nz = int(np.ceil(box[4] - box[5]))
    nz += nz == 0
    dev = torch.device("cuda", 0)
    dZ = torch.from_numpy(np.ascontiguousarray(Z, np.int32)).to(dev)
    dx, dy, dzz = (torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev) for a in (x, y, z))
    d_atoms = torch.empty(4 * n, dtype=torch.float32, device=dev)
    d_off = torch.full((nz * 2500 + 1,), -7, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    nz_out = C.c_int(-1)
    rc = L.ms_build_atom_index_noalloc(dZ.data_ptr(), dx.data_ptr(), dy.data_ptr(), dzz.data_ptr(), n,
                                       box.ctypes.data_as(C.c_void_p), d_atoms.data_ptr(), d_off.data_ptr(),
                                       d_off.numel(), C.byref(nz_out), None)
    assert rc == 0, L.ms_last_error(None).decode()
    torch.cuda.synchronize()
    assert nz_out.value == nz
    at = d_atoms.cpu().numpy().reshape(n, 4)
    return (d_off.cpu().numpy(), at[:, 3].copy().view(np.int32), at[:, 0].copy(), at[:, 1].copy(),
            at[:, 2].copy())


def test_noalloc_index_matches_allocating_entry_point():
    from cudamultislice_b200 import _lib, structures

    L = _lib.lib()
    first = structures.random_atoms(30000, size=(41.0, 37.0, 60.0), Zs=(6, 8, 14, 38, 79), seed=101)
    second = structures.srtio3(4, 4, 20)
    for atoms in (first, second):  # two calls in a row through the shared scratch
        got = _noalloc_index(L, atoms)
        want = _reference_index(atoms)
        for g, w in zip(got, want):
            assert g.dtype == w.dtype and g.shape == w.shape
            assert np.array_equal(g, w)


def test_noalloc_refuses_oversized_requests():
    from cudamultislice_b200 import _lib

    L = _lib.lib()
    box = np.array([10, 0, 10, 0, 10, 0], np.float32)
    nz = C.c_int()
    fake = C.c_void_p(256)  # never dereferenced: the size checks come first
    rc = L.ms_build_atom_index_noalloc(fake, fake, fake, fake, 131073, box.ctypes.data_as(C.c_void_p), fake, fake,
                                       1 << 20, C.byref(nz), None)
    assert rc == 1 and b"131072" in L.ms_last_error(None)
    deep = np.array([10, 0, 10, 0, 500, 0], np.float32)  # 500 z-bins > 209
    rc = L.ms_build_atom_index_noalloc(fake, fake, fake, fake, 10, deep.ctypes.data_as(C.c_void_p), fake, fake,
                                       1 << 22, C.byref(nz), None)
    assert rc == 1 and b"z-bins" in L.ms_last_error(None)
    # a non-finite box, and a finite one whose depth would overflow an int bin
    # count, are refused before any launch
    for bad in ([10, 0, 10, 0, np.inf, 0], [10, 0, 10, 0, 10, -np.inf], [10, 0, 10, 0, 1e10, 0],
                [np.nan, 0, 10, 0, 10, 0]):
        b = np.array(bad, np.float32)
        rc = L.ms_build_atom_index_noalloc(fake, fake, fake, fake, 10, b.ctypes.data_as(C.c_void_p), fake, fake,
                                           1 << 22, C.byref(nz), None)
        assert rc == 1, bad


def test_noalloc_index_in_graph_capture():
    """The entry point enqueues into a CUDA graph: after one warm-up call (which
    looks up the scratch array's device address outside any capture), a call
    captured on a non-default stream records the index build, and each replay
    of the graph rebuilds the index of ms_upload_binned_atoms bit for bit."""
    import torch
    from cudamultislice_b200 import _lib, structures

    L = _lib.lib()
    atoms = structures.random_atoms(20000, size=(31.0, 29.0, 40.0), Zs=(6, 8, 38), seed=7)
    _noalloc_index(L, atoms)  # warm-up, outside capture
    want = _reference_index(atoms)
    Z, x, y, z = atoms
    n = len(Z)
    box = _box(x, y, z)
    nz = int(np.ceil(box[4] - box[5]))
    nz += nz == 0
    dev = torch.device("cuda", 0)
    dZ = torch.from_numpy(np.ascontiguousarray(Z, np.int32)).to(dev)
    dx, dy, dzz = (torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev) for a in (x, y, z))
    d_atoms = torch.zeros(4 * n, dtype=torch.float32, device=dev)
    d_off = torch.zeros(nz * 2500 + 1, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    stream = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    nz_out = C.c_int(-1)
    with torch.cuda.graph(graph, stream=stream):
        rc = L.ms_build_atom_index_noalloc(dZ.data_ptr(), dx.data_ptr(), dy.data_ptr(), dzz.data_ptr(), n,
                                           box.ctypes.data_as(C.c_void_p), d_atoms.data_ptr(), d_off.data_ptr(),
                                           d_off.numel(), C.byref(nz_out), C.c_void_p(stream.cuda_stream))
    assert rc == 0, L.ms_last_error(None).decode()
    assert nz_out.value == nz
    for _ in range(2):  # the captured work, not the capture, fills the buffers
        d_off.fill_(-7)
        d_atoms.zero_()
        graph.replay()
        torch.cuda.synchronize()
        at = d_atoms.cpu().numpy().reshape(n, 4)
        got = (d_off.cpu().numpy(), at[:, 3].copy().view(np.int32), at[:, 0].copy(), at[:, 1].copy(),
               at[:, 2].copy())
        for g, w in zip(got, want):
            assert g.dtype == w.dtype and g.shape == w.shape
            assert np.array_equal(g, w)
    del graph
