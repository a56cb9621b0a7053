"""Initial states of a hierarchy: puncture data (get_lousto_nbhs on the GPU,
bssn_class.C:1028-1240 calls it block by block) plus seeded noise.

The noise of a cell depends only on (seed, level, field, global cell index),
so every copy of a cell -- its owner, a neighbour's ghost cell, a buffer cell --
starts with the same value, as a single-resolution field would.
"""
import numpy as np

from . import dropin


def grid_noise(level, field, gi, gj, gk, seed):
    """Uniform values in [-1, 1) for global cell indices (gi, gj, gk) of a
    level: the splitmix64 finaliser (Steele, Lea, Flood 2014) of a key packing
    seed, level, field and the 16 low bits of each index."""
    with np.errstate(over="ignore"):   # 64-bit wrap-around is part of the hash
        key = (np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15)
               ^ (np.uint64(level) << np.uint64(56)) ^ (np.uint64(field) << np.uint64(48))
               ^ ((gk.astype(np.uint64) & np.uint64(0xFFFF)) << np.uint64(32))
               ^ ((gj.astype(np.uint64) & np.uint64(0xFFFF)) << np.uint64(16))
               ^ (gi.astype(np.uint64) & np.uint64(0xFFFF)))
        z = key + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (2.0 / 2.0 ** 53) - 1.0


def initial_state(H, masses, positions, noise=0.0, seed=1, nf=24, momenta=None, spins=None):
    """One (nf, ez, ey, ex) state per block of H: puncture data plus
    noise * grid_noise on every field.  nf = 25 appends the Z4c Theta field
    (zero before the noise)."""
    out = []
    with np.errstate(over="ignore"):
        for b in H.blocks:
            X, Y, Z = H.coords(b)
            st = dropin.get_lousto_nbhs(X, Y, Z, masses, positions, momenta, spins)
            if nf == 25:
                st = np.concatenate([st, np.zeros((1,) + st.shape[1:])])
            if noise > 0:
                gk, gj, gi = np.meshgrid(np.arange(b.ex[2]) + b.org[2], np.arange(b.ex[1]) + b.org[1],
                                         np.arange(b.ex[0]) + b.org[0], indexing="ij")
                for f in range(nf):
                    st[f] += noise * grid_noise(b.level, f, gi, gj, gk, seed)
            out.append(st)
    return out


def single_block_state(n_interior, lo, hi, ghosts, masses, positions, noise=0.0, seed=1):
    """A uniform cell-centred block of n_interior^3 cells on [lo, hi]^3 plus
    `ghosts` cells each side (one level-0 patch): (X, state, bbox, h), with
    seeded uniform noise U(-noise, noise) drawn by numpy.random.default_rng(seed)
    field by field in state order."""
    h = (hi - lo) / n_interior
    n = n_interior + 2 * ghosts
    a_lo, a_hi = lo - ghosts * h, hi + ghosts * h
    ha = (a_hi - a_lo) / n
    X = a_lo + (np.arange(n) + 0.5) * ha
    st = dropin.get_lousto_nbhs(X, X, X, masses, positions)
    if noise > 0:
        rng = np.random.default_rng(seed)
        for f in range(24):
            st[f] += rng.uniform(-noise, noise, size=st[f].shape)
    return X, st, (a_lo, a_lo, a_lo, a_hi, a_hi, a_hi), h


def gaussian(X, Y, Z, amplitude, width, centre):
    """amplitude * exp(-|x - centre|^2 / width^2) on the cell centres."""
    z, y, x = np.meshgrid(Z, Y, X, indexing="ij")
    r2 = (x - centre[0]) ** 2 + (y - centre[1]) ** 2 + (z - centre[2]) ** 2
    return amplitude * np.exp(-r2 / width ** 2)
