"""Compact fingerprints of large vectors, for fixtures at the workloads' full sizes.

A field of a 32^4 lattice is 134 MB, too large for a fixture.  A digest keeps what a parity
check needs: the norm, three weighted sums over every entry (weights cos(0.1 i),
sin(0.37 i + 0.5) and 1, fixed formulas so no random generator is involved), and the entries
at 4096 fixed positions (i * 7919 + 13 mod n, distinct for every n coprime to 7919).  A wrong
entry anywhere moves a weighted sum; a systematic error moves the norm and the samples.
"""
from __future__ import annotations

import numpy as np

NSAMPLES = 4096


def sample_index(n: int) -> np.ndarray:
    k = min(NSAMPLES, n)
    return (np.arange(k, dtype=np.int64) * 7919 + 13) % n


def _weights(n: int):
    i = np.arange(n, dtype=np.float64)
    return np.cos(0.1 * i), np.sin(0.37 * i + 0.5), np.ones(n)


def digest(y: np.ndarray) -> dict:
    y = np.asarray(y, dtype=np.float64).ravel()
    n = y.size
    return {"n": np.array(n), "norm": np.array(np.linalg.norm(y)),
            "wsum": np.array([float(w @ y) for w in _weights(n)]),
            "samples": y[sample_index(n)]}


def store(out: dict, prefix: str, y: np.ndarray) -> None:
    """Adds the digest of y to a fixture dictionary under prefix_*."""
    for k, v in digest(y).items():
        out[f"{prefix}_{k}"] = v


def check(y: np.ndarray, fx, prefix: str, rtol: float) -> dict:
    """Compares y with the digest stored under prefix in fixture fx.

    Every quantity is compared relative to the vector's scale: the norm to rtol * norm, each
    weighted sum to rtol * |w| * norm (its Cauchy-Schwarz bound), each sample to
    rtol * max |sample|.  Returns the worst relative deviation of each kind; asserts they are
    within rtol.
    """
    y = np.asarray(y, dtype=np.float64).ravel()
    n = int(fx[f"{prefix}_n"])
    assert y.size == n, (y.size, n)
    norm = float(fx[f"{prefix}_norm"])
    got = digest(y)
    dev = {"norm": abs(float(got["norm"]) - norm) / norm}
    wn = [np.linalg.norm(w) for w in _weights(n)]
    dev["wsum"] = max(abs(a - b) / (w * norm) for a, b, w in
                      zip(got["wsum"], fx[f"{prefix}_wsum"], wn))
    s = fx[f"{prefix}_samples"]
    dev["samples"] = float(np.max(np.abs(got["samples"] - s)) / np.max(np.abs(s)))
    for k, v in dev.items():
        assert v <= rtol, f"{prefix} {k}: {v:.3e} > {rtol:.1e}"
    return dev
