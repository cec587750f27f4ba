"""CUDA-graph mode (revsim_set_graph_mode): forward and reverse passes captured once and
replayed give the same trajectories (bit for bit) as plain launches, across new seeds, host
noise, a parameter change (recapture) and batched replicas; passes with a host decision
inside (gradient clipping) still run, as plain launches.  The losses and gradients agree to
1e-12 relative: the smoothed-RDF histogram sums with FP64 atomics, whose order varies from
run to run in the last bits, in either mode."""

import numpy as np
import pytest

from conftest import relaxed_water
from oracle import orc
from revsim import Engine, RdfTerm, constants as C, systems

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    import build
    build.build()


def _target(x, n_mol, box):
    s = orc.make_system(n_mol, box)
    t0 = orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, np.zeros(200), 2, 1.0)
    return 0.9 * orc.rdf(s, t0, x) + 0.05


def _same(a, b):
    """Trajectories bit for bit; losses and gradients to the RDF atomics' rounding."""
    lf, xf, vf, lr, g, x0, v0 = a
    lf2, xf2, vf2, lr2, g2, x02, v02 = b
    for u, w in ((xf, xf2), (vf, vf2), (x0, x02), (v0, v02)):
        np.testing.assert_array_equal(u, w)
    for u, w in ((lf, lf2), (lr, lr2), (g, g2)):
        np.testing.assert_allclose(u, w, rtol=1e-12, atol=1e-12 * np.abs(w).max())


def _run(e, x, v, seeds, p, n=60, nl=30, tr=20, noise=None, clip=np.inf):
    e.set_params(p)
    e.set_state(x, v)
    lf = e.forward(seeds, 1.0, n, nl, 0.001, noise=noise)
    xf, vf = e.get_state()
    lr, g = e.reverse(seeds, 1.0, n, nl, tr, 0.001, clip=clip, noise=noise)
    x0, v0 = e.get_state()
    return [lf, xf, vf, lr, g, x0, v0]


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_graph_replays_match_plain_launches(small_water, prec):
    n_mol, box, x, v = small_water
    terms = [RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, _target(x, n_mol, box), 2, 1.0)]
    p0 = np.array(C.default_params())
    p1 = p0.copy()
    p1[0] *= 1.01
    plain = Engine(n_mol, box, precision=prec, n_steps_log=30)
    graph = Engine(n_mol, box, precision=prec, n_steps_log=30)
    for e in (plain, graph):
        e.set_params(p0)
        e.set_loss(terms)
    graph.set_graph_mode(True)
    cases = [(systems.noise_seeds(60, seed=s), p) for s, p in ((1, p0), (2, p0), (3, p1), (4, p1))]
    for seeds, p in cases:
        _same(_run(plain, x, v, seeds, p), _run(graph, x, v, seeds, p))
    captures, replays = graph.graph_stats()
    # forward + reverse captured for p0 and again for p1; every pass launched as a graph
    assert captures == 4 and replays == 8, (captures, replays)
    assert plain.graph_stats() == (0, 0)
    # host noise through the graph, and a clipped reverse pass (plain launches)
    xi = np.stack([plain.noise([sd]) for sd in cases[0][0]])
    _same(_run(plain, x, v, None, p0, noise=xi), _run(graph, x, v, None, p0, noise=xi))
    _same(_run(plain, x, v, cases[0][0], p0, clip=1e-3), _run(graph, x, v, cases[0][0], p0, clip=1e-3))


def test_graph_mode_with_replicas():
    sizes, boxes, temps = [150, 90], [2.6, 2.5], [285.0, 310.0]
    xs, vs = zip(*[relaxed_water(m, b, seed=60 + i, steps=10) for i, (m, b) in enumerate(zip(sizes, boxes))])
    target = np.stack([_target(xs[r], sizes[r], boxes[r]) for r in range(2)])
    out = []
    for mode in (False, True):
        e = Engine(sizes, boxes, temp=temps, precision="mixed")
        e.set_params(C.default_params())
        e.set_loss([RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, target, 2, 1.0)])
        e.set_graph_mode(mode)
        seeds = np.stack([systems.noise_seeds(40, seed=70 + r) for r in range(2)], axis=1)
        res = []
        for _ in range(2):
            res.append(_run(e, np.concatenate(xs), np.concatenate(vs), seeds, np.array(C.default_params()),
                            n=40, nl=40, tr=40))
        out.append(res)
        e.close()
    for ra, rb in zip(*out):
        _same(ra, rb)
