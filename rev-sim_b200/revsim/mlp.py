"""The learned pair correction of the water model: parameter layout, seeded initialisation
and the Adam training loop driven by the reversible-simulation gradient.

No reference counterpart: the reference's learned terms are MACE-OFF / DimeNet++ through
PyTorch / JAX hooks (water_maceoff.jl:147-163, diamond.jl:1699-1755); the engine's term is a
per element pair MLP (O-O, O-H, H-H; 16 Gaussian radial basis functions on 0-1 nm, width
0.05 nm -> 64 -> 64 SiLU -> scalar, times a cosine cutoff) evaluated by librevsim.so
(include/revsim.h, ``mlp`` in the system description).  Its parameters follow the classical
ones in the parameter vector.  The training loop follows the reference's (water.jl:1682-1696:
one gradient per update, Adam).
"""

import numpy as np

NRBF, H, NT = 16, 64, 3
PER_TYPE = H * NRBF + H + H * H + H + H + 1
N_PARAMS = NT * PER_TYPE


def _splitmix_uniform(seed, n):
    """n uniforms in [0, 1) from a splitmix64 stream (the engine's seeded initialisation)."""
    out = np.empty(n)
    s = np.uint64(seed)
    with np.errstate(over="ignore"):
        for i in range(n):
            s = s + np.uint64(0x9E3779B97F4A7C15)
            z = s
            z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
            z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
            z = z ^ (z >> np.uint64(31))
            out[i] = float(int(z) >> 11) * (1.0 / 9007199254740992.0)
    return out


def init_params(seed=3):
    """Xavier-uniform W1 and W2, w3 Xavier-uniform times 0.01, zero biases (per type)."""
    theta = np.zeros(N_PARAMS)
    u = _splitmix_uniform(seed, NT * (H * NRBF + H * H + H))
    k = 0
    for t in range(NT):
        p = theta[t * PER_TYPE:(t + 1) * PER_TYPE]
        a1, a2, a3 = np.sqrt(6.0 / (NRBF + H)), np.sqrt(6.0 / (2 * H)), np.sqrt(6.0 / (H + 1))
        p[:H * NRBF] = a1 * (2.0 * u[k:k + H * NRBF] - 1.0)
        k += H * NRBF
        o = H * NRBF + H
        p[o:o + H * H] = a2 * (2.0 * u[k:k + H * H] - 1.0)
        k += H * H
        o2 = o + H * H + H
        p[o2:o2 + H] = 0.01 * a3 * (2.0 * u[k:k + H] - 1.0)
        k += H
    return theta


class Adam:
    """Adam (Kingma & Ba) on a flat parameter vector; `mask` selects the trained entries and
    the step size may be a scalar or one value per parameter."""

    def __init__(self, n, lr=1e-3, betas=(0.9, 0.999), eps=1e-8, mask=None):
        self.lr, self.b1, self.b2, self.eps = lr, betas[0], betas[1], eps
        self.m = np.zeros(n)
        self.v = np.zeros(n)
        self.t = 0
        self.mask = np.ones(n, dtype=bool) if mask is None else np.asarray(mask, dtype=bool)

    def step(self, theta, grad, lr=None):
        lr = self.lr if lr is None else lr
        g = np.where(self.mask, grad, 0.0)
        self.t += 1
        self.m = self.b1 * self.m + (1 - self.b1) * g
        self.v = self.b2 * self.v + (1 - self.b2) * g * g
        mh = self.m / (1 - self.b1 ** self.t)
        vh = self.v / (1 - self.b2 ** self.t)
        return theta - np.where(self.mask, lr * mh / (np.sqrt(vh) + self.eps), 0.0)


def train(engine, theta0, x0, v0, seeds_fn, n_updates, n_steps, n_steps_loss, dt=0.001,
          gamma=1.0, lr_classical=1e-3, lr_mlp=1e-3, train_classical=True, train_mlp=True,
          callback=None):
    """Reversible-simulation training: per update one forward + reverse pass from (x0, v0)
    with seeds_fn(update) as noise seeds, then one Adam step.  The learning rate of each
    classical parameter is lr_classical times its initial magnitude (the parameters span
    eight decades).  Returns (theta, losses)."""
    theta = np.array(theta0, dtype=np.float64)
    nc = len(theta) - (N_PARAMS if engine.mlp else 0)
    mask = np.zeros(len(theta), dtype=bool)
    if train_classical:
        mask[:nc] = True
    if engine.mlp and train_mlp:
        mask[nc:] = True
    scale = np.ones(len(theta))
    scale[:nc] = np.maximum(np.abs(theta[:nc]), 1e-3) * lr_classical
    scale[nc:] = lr_mlp
    opt = Adam(len(theta), lr=scale, mask=mask)
    losses = []
    for u in range(n_updates):
        engine.set_params(theta)
        engine.set_state(x0, v0)
        seeds = seeds_fn(u)
        lf = engine.forward(seeds, gamma, n_steps, n_steps_loss, dt)
        _, g = engine.reverse(seeds, gamma, n_steps, n_steps_loss, n_steps_loss, dt)
        g = g.mean(axis=0)
        losses.append(float(np.mean(lf)))
        if callback:
            callback(u, theta, float(np.mean(lf)), g)
        theta = opt.step(theta, g)
    return theta, losses
