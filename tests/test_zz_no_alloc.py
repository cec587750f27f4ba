"""The allocation-free RDF loss entry point, against the handle-based one.

revsim_rdf_loss_grad_noalloc serves callers that cannot let the library allocate
device memory -- a host whose own pool allocator owns the device memory and hands out
pointers, a loop that must not take the device-wide synchronisation of
cudaMalloc/cudaFree, a service whose memory is fixed before it starts.  It works on
the caller's device buffers and keeps its scratch in a fixed array inside the library.
These tests call it through the C ABI on device buffers the test owns and compare
loss and dL/dx with revsim_loss_grad (Engine.loss_grad) on the same positions, twice
in a row, since every call reuses the same scratch.  The file sorts last so that a
run stopping at the first failure has already run every other test.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    import build
    build.build()
    import torch
    from revsim import Engine, _lib, constants as C, systems
    from revsim.engine import RdfTerm
    from revsim.loss import reference_rdf_terms

    L = _lib.load()
    n_mol, box = 400, 2.6
    x = systems.water_coords(n_mol, box, seed=11)
    rng = np.random.default_rng(12)
    x = x + rng.normal(scale=0.003, size=x.shape)
    x -= np.floor(x / box) * box
    v = np.zeros_like(x)
    terms = [RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, rng.uniform(0, 2, 200), 2, 1.0)]
    terms += reference_rdf_terms(rng.uniform(0, 2, 248), rng.uniform(0, 2, 281))
    # the largest grid the scratch holds (8,192 points, 0.0005 nm apart): above 6,144 points
    # the histogram kernel sums in global memory instead of shared memory, and the
    # normaliser sits right after the last histogram entry, next to dL/dh
    terms.append(RdfTerm(0, 0, 0.0005, 0.0005, 0.0005, 0.04, 8192, 0, 1, rng.uniform(0, 2, 8192), 2, 1.0))
    refs = []
    for t in terms:
        e = Engine(n_mol, box)
        e.set_params(C.default_params())
        e.set_state(x, v)
        e.set_loss([t])
        refs.append(e.loss_grad())
        e.close()
    return L, torch, n_mol, box, x, terms, refs


def _call(L, torch, n_mol, box, dx, t, dtarget, dloss, dgrad):
    from revsim import _lib
    term = _lib.RdfTermC(t.sel1, t.sel2, t.x_min, t.step, t.width, t.exp_cutoff, t.n_grid,
                         t.slice_start, t.slice_stride, len(t.target), t.norm, t.weight)
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.revsim_rdf_loss_grad_noalloc(dx.data_ptr(), n_mol, box, ctypes.byref(term),
                                        dtarget.data_ptr(), dloss.data_ptr(), dgrad.data_ptr(),
                                        stream)
    torch.cuda.synchronize()
    return rc


@pytest.mark.parametrize("which", [0, 1, 2, 3])
def test_noalloc_matches_handle_loss_twice(setup, which):
    L, torch, n_mol, box, x, terms, refs = setup
    t = terms[which]
    lref, gref = refs[which]
    dx = torch.tensor(x, dtype=torch.float64, device="cuda")
    dtarget = torch.tensor(np.asarray(t.target, dtype=np.float64), device="cuda")
    for _ in range(2):   # the second call reuses the scratch the first one left behind
        dloss = torch.full((1,), 123.0, dtype=torch.float64, device="cuda")
        dgrad = torch.full_like(dx, 7.0)
        assert _call(L, torch, n_mol, box, dx, t, dtarget, dloss, dgrad) == 0
        loss = dloss.cpu().numpy()[0]
        grad = dgrad.cpu().numpy()
        assert abs(loss - lref[0]) <= 1e-10 * abs(lref[0])
        assert np.linalg.norm(grad - gref) <= 1e-10 * np.linalg.norm(gref)


def test_noalloc_rejects_grid_beyond_scratch(setup):
    L, torch, n_mol, box, x, terms, refs = setup
    from revsim.engine import RdfTerm
    dx = torch.tensor(x, dtype=torch.float64, device="cuda")
    big = RdfTerm(0, 0, 0.0005, 0.0005, 0.0005, 0.04, 8193, 0, 1, np.zeros(10), 2, 1.0)
    dtarget = torch.zeros(10, dtype=torch.float64, device="cuda")
    dloss = torch.zeros(1, dtype=torch.float64, device="cuda")
    dgrad = torch.zeros_like(dx)
    assert _call(L, torch, n_mol, box, dx, big, dtarget, dloss, dgrad) == -1
    # a width so small against the grid step that the Gaussian recurrence would overflow
    thin = RdfTerm(0, 0, 0.005, 0.005, 1e-7, 0.04, 200, 0, 1, np.zeros(10), 2, 1.0)
    assert _call(L, torch, n_mol, box, dx, thin, dtarget, dloss, dgrad) == -1
