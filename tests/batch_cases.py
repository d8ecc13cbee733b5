"""Batched-instance definitions for the FP32 batch tests."""
import numpy as np

from oracle.wigner2d import WignerParams, wigner_harmonic_oscillator


def random_batch(sizes, seed=0, steps_dt=0.005, damp=True):
    """Instances on the given square grids: V = a x^4 + b x^2, a ~ U[0.01, 0.1],
    b ~ U[-1, 0.5], gamma ~ U[0, 0.2] (D_theta = 2 gamma m kT, kT = 0.5), coherent
    state at x0 ~ U[-2, 2], p0 ~ U[-1, 1], amplitudes 10, dt 0.005."""
    rng = np.random.default_rng(seed)
    out = []
    for n in sizes:
        a, b = rng.uniform(0.01, 0.1), rng.uniform(-1., 0.5)
        g = rng.uniform(0., 0.2) if damp else 0.
        x0, p0 = rng.uniform(-2., 2.), rng.uniform(-1., 1.)
        out.append(dict(n=int(n), a=a, b=b, gamma=g, x0=x0, p0=p0))
    return out


def to_instance(c, dt=0.005):
    from pywignercuda_b200.batch import instance
    return instance(c['n'], x_amplitude=10., dt=dt, gamma=c['gamma'], d_theta=c['gamma'], v4=c['a'],
                    v2=c['b'])


def to_params(c, dt=0.005):
    return WignerParams(c['n'], c['n'], 10., 10., dt, potential='%r*pow(x,4) + %r*pow(x,2)' % (c['a'], c['b']),
                        dpotential='4*%r*pow(x,3) + 2*%r*x' % (c['a'], c['b']), gamma=c['gamma'],
                        d_theta=c['gamma'], damping='CaldeiraLeggett', fp_damping='fabs(p)', constants='exact')


def initial_state(c):
    prm = to_params(c)
    return np.ascontiguousarray(wigner_harmonic_oscillator(prm, 0, 1., c['x0'], c['p0']))


def config3_cases(seed=0, count=64):
    """The 64-instance mixed-grid batch: square grids from {128, 256, 512, 1024},
    a ~ U[0.01, 0.1], b ~ U[-1, 0.5], gamma ~ U[0, 0.2], D_theta = 2 gamma m kT
    (kT = 0.5), coherent states at x0 ~ U[-2, 2], p0 ~ U[-1, 1], in the draw order
    of numpy default_rng(seed) that the benchmark uses."""
    rng = np.random.default_rng(seed)
    sizes = rng.choice([128, 256, 512, 1024], size=count)
    a = rng.uniform(0.01, 0.1, count)
    b = rng.uniform(-1., 0.5, count)
    g = rng.uniform(0., 0.2, count)
    x0 = rng.uniform(-2., 2., count)
    p0 = rng.uniform(-1., 1., count)
    return [dict(n=int(sizes[i]), a=float(a[i]), b=float(b[i]), gamma=float(g[i]), d_theta=float(g[i]),
                 x0=float(x0[i]), p0=float(p0[i])) for i in range(count)]
