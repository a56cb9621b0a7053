"""Shared test inputs and error measures."""
import numpy as np


def relerr(a, b):
    """max |a - b| / max |b| (absolute when b is identically zero)."""
    den = np.abs(b).max()
    num = np.abs(a - b).max()
    return num / den if den > 0 else num


def generic_state(X, Y, Z, seed=3, amp=1.0):
    """A smooth non-trivial BSSN state: every field varies, the shift takes
    both signs, the metric stays near the identity and chi+1 in [0.5, 0.9]."""
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(Z, Y, X, indexing="ij")
    st = np.empty((24,) + x.shape)
    base = {0: -0.3, 17: -0.25}
    scale = {0: 0.1, 1: 0.05, 2: 0.05, 3: 0.02, 4: 0.02, 5: 0.05, 6: 0.02, 7: 0.05, 17: 0.1}
    for f in range(24):
        a, b, c = rng.uniform(0.3, 0.9, 3)
        ph = rng.uniform(0, 2 * np.pi, 3)
        s = scale.get(f, 0.03 if f < 14 else 0.08)
        st[f] = base.get(f, 0.0) + amp * s * np.sin(a * x + ph[0]) * np.cos(b * y + ph[1]) * np.sin(c * z + ph[2] + 0.3)
    return st
