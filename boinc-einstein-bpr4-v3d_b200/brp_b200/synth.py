"""Seeded synthetic workloads of the search path.

No public dataset is involved: the reference's real BRP4 workunits and
orbital banks are not part of its snapshot.  Every series is seeded white
Gaussian noise (mean 0, variance 1) plus binary pulsars: a pulse train of spin
frequency f with `harmonics` Fourier harmonics of a rectangular pulse of duty
cycle `duty`, Doppler-delayed by a circular orbit,

    x(t) = A * sum_h sinc(h duty) cos(2 pi h f (t + tau (sin(Omega t + psi) - sin psi)))

which the resampler's map r[i] = x[i - offset(i)] (src/science.cpp:36-40,
:75-85) turns back into a strictly periodic signal for the matching template.
Templates are drawn as the reference's banks are described: P_orb
log-uniform, tau uniform, psi uniform in [0, 2 pi).
"""
from dataclasses import dataclass, field

import numpy as np

from .host import parameters, search_parameters

DT = 128e-6          # sample time (s)
SAMPLE_US = 128.0


@dataclass
class Pulsar:
    f: float            # spin frequency (Hz)
    period: float       # orbital period (s)
    tau: float          # projected semi-major axis (light-s)
    psi: float          # orbital phase (rad)
    amplitude: float = 0.05
    harmonics: int = 5
    duty: float = 0.1


@dataclass
class Workload:
    name: str
    series: list                     # float32 arrays (unpadded samples)
    n: list                          # padded length per series
    templates: list                  # Params
    series_of: np.ndarray            # series index per template
    orbits: list                     # (period, tau, psi) per template
    pulsars: list = field(default_factory=list)
    meta: dict = field(default_factory=dict)


def pulsar_signal(samples, p: Pulsar, dt=DT):
    t = np.arange(samples, dtype=np.float64) * dt
    delay = p.tau * (np.sin(2 * np.pi / p.period * t + p.psi) - np.sin(p.psi))
    phase = 2 * np.pi * p.f * (t + delay)
    s = np.zeros(samples)
    for h in range(1, p.harmonics + 1):
        s += np.sinc(h * p.duty) * np.cos(h * phase)
    return p.amplitude * s


def make_series(samples, seed, pulsars=(), dt=DT):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(samples)
    for p in pulsars:
        x += pulsar_signal(samples, p, dt)
    return x.astype(np.float32)


def random_pulsars(rng, count, fmin=50.0, fmax=700.0, pmin_h=1.0, pmax_h=24.0, tmin=0.1, tmax=3.0, amplitude=0.02,
                   harmonics=8):
    out = []
    for _ in range(count):
        out.append(Pulsar(f=float(rng.uniform(fmin, fmax)), period=float(rng.uniform(pmin_h, pmax_h) * 3600),
                          tau=float(rng.uniform(tmin, tmax)), psi=float(rng.uniform(0, 2 * np.pi)),
                          amplitude=amplitude, harmonics=harmonics, duty=0.1))
    return out


def random_orbits(rng, count, pmin_h=1.0, pmax_h=24.0, tau_max=3.0):
    P = np.exp(rng.uniform(np.log(pmin_h * 3600), np.log(pmax_h * 3600), count))
    tau = rng.uniform(0, tau_max, count)
    psi = rng.uniform(0, 2 * np.pi, count)
    return [(float(a), float(b), float(c)) for a, b, c in zip(P, tau, psi)]


def sigma_false_alarm(n, sigma):
    """False-alarm rate whose per-bin probability (src/workload.cpp:120) is the
    one-sided Gaussian tail of `sigma`."""
    from math import erfc, sqrt
    p = 0.5 * erfc(sigma / sqrt(2.0))
    return float(-np.expm1((n // 2 + 1) * np.log1p(-p)))


# ---------------------------------------------------------------- configs
def config_single(n, unpadded, pulsar: Pulsar, seed, production=False):
    """One template equal to the injected orbit, bench-mode constants
    (src/science.cpp:46-65), optionally production FMA arithmetic."""
    from .host import production as prod
    x = make_series(unpadded, seed, [pulsar])
    p = parameters(n, unpadded, pulsar.tau, pulsar.period, pulsar.psi, DT)
    if production:
        p = prod(p)
    return Workload("single", [x], [n], [p], np.zeros(1, np.uint32), [(pulsar.period, pulsar.tau, pulsar.psi)],
                    [pulsar])


def config1():
    """N = 65536, 137.5 Hz, 5 harmonics, duty 0.1, A = 0.05, P = 3600 s, tau = 0.3 s, psi = 1.1."""
    return config_single(65536, 65536 - 17, Pulsar(137.5, 3600.0, 0.3, 1.1, 0.05, 5, 0.1), seed=1)


def config2():
    """N = 2^22, 421.3 Hz, 8 harmonics, P = 11 h, tau = 1.7 s, psi = 0.4."""
    n = 1 << 22
    return config_single(n, n - 17, Pulsar(421.3, 11 * 3600.0, 1.7, 0.4, 0.02, 8, 0.1), seed=2)


def bank_workload(name, lengths, counts, pulsars_per_series, seed, f0=800.0, false_alarm=0.08, window=1000,
                  sigmas=None, include_truth=True, search=None):
    """Series of the given lengths (no padding: samples = n) with injected
    pulsars, `counts[s]` production templates (src/workload.cpp:108-125) per
    series.  With `sigmas`, templates alternate between per-bin false-alarm
    levels of those Gaussian sigmas.  `search` computes a template's
    constants (the signature of search_parameters); by default this package's
    host code, which is byte-identical to the reference's."""
    search = search or search_parameters
    rng = np.random.default_rng(seed)
    series, pulsars, templates, series_of, orbits = [], [], [], [], []
    for s, (n, count, npul) in enumerate(zip(lengths, counts, pulsars_per_series)):
        pul = random_pulsars(rng, npul)
        pulsars.append(pul)
        series.append(make_series(n, seed * 1000 + s, pul))
        orb = random_orbits(rng, count)
        if include_truth:
            for k, p in enumerate(pul[:count]):
                orb[k * max(1, count // max(1, len(pul)))] = (p.period, p.tau, p.psi)
        for k, (P, tau, psi) in enumerate(orb):
            fa = false_alarm if sigmas is None else sigma_false_alarm(n, sigmas[k % len(sigmas)])
            templates.append(search(n, n, SAMPLE_US, P, tau, psi, f0, fa, window))
            series_of.append(s)
            orbits.append((P, tau, psi))
    return Workload(name, series, list(lengths), templates, np.asarray(series_of, np.uint32), orbits, pulsars,
                    dict(f0=f0, false_alarm=false_alarm, window=window, sigmas=sigmas))


def config3(templates=512):
    """One N = 2^22 series, 3 pulsars, 512 templates."""
    return bank_workload("bank-2^22", [1 << 22], [templates], [3], seed=3)


def config4(templates=128):
    """N = 3*2^21, 2 pulsars, 128 templates."""
    return bank_workload("bank-3x2^21", [3 << 21], [templates], [2], seed=4)


def config5(total=1024):
    """1024 templates over N in {2^20, 3*2^20, 2^22} in ratio 4:2:1, 0-2 pulsars
    per series, thresholds at 5 and 7 sigma-equivalent."""
    c1 = round(total * 4 / 7)
    c2 = round(total * 2 / 7)
    c3 = total - c1 - c2
    return bank_workload("uneven", [1 << 20, 3 << 20, 1 << 22], [c1, c2, c3], [2, 1, 0], seed=5, sigmas=(5.0, 7.0))
