"""Octree leaf lists for grid_type = 'amr'.

The library reads the generic text leaf list of read_generic_amr.f90:60-81:
a header line "nleaf boxlen", then one row "x y z level nH" per leaf, with
coordinates centred on the box (the box spans [-boxlen/2, boxlen/2]^3) and
level 0 the whole box.  This module writes such lists:

* `build_leaves` refines an octree level by level from a complete base
  level with a caller's refinement test and density, and returns the leaves
  in Morton order (depth first, octant index ix + 2 iy + 4 iz as in
  amr_build_tree, octree_mod.f90:342-432), so leaves that are neighbours in
  space are mostly neighbours in memory;
* `lognormal_field` is a seeded Gaussian random field with power spectrum
  P(k) ~ k^slope, exponentiated to a log-normal density of given mean and
  dispersion of ln n;
* `clumpy_nebula` is the dusty clumpy nebula workload: the log-normal field
  sampled on 256^3, an octree with base level 6 refined towards level 10
  where the density exceeds a threshold that rises by a fixed factor per
  level.
"""
import numpy as np


def _morton(ix, iy, iz, bits):
    key = np.zeros(ix.shape, dtype=np.uint64)
    for b in range(bits):
        key |= ((ix >> b) & 1).astype(np.uint64) << np.uint64(3 * b)
        key |= ((iy >> b) & 1).astype(np.uint64) << np.uint64(3 * b + 1)
        key |= ((iz >> b) & 1).astype(np.uint64) << np.uint64(3 * b + 2)
    return key


def build_leaves(boxlen, base_level, max_level, refine, density):
    """Leaves of an octree over [-boxlen/2, boxlen/2]^3.

    refine(x, y, z, level) -> bool array: whether the cells with these
    centres at this level split (asked for levels base_level..max_level-1);
    density(x, y, z, level) -> n_H of the leaves.  Returns (x, y, z, level,
    nH) arrays in Morton order.
    """
    if not (0 <= base_level <= max_level <= 20):
        raise ValueError("need 0 <= base_level <= max_level <= 20")
    half = 0.5 * boxlen
    n0 = 1 << base_level
    i = np.arange(n0, dtype=np.int64)
    iz, iy, ix = np.meshgrid(i, i, i, indexing="ij")
    cells = [ix.ravel(), iy.ravel(), iz.ravel()]
    out = []
    for lev in range(base_level, max_level + 1):
        h = boxlen / (1 << lev)
        cx, cy, cz = (-half + (c + 0.5) * h for c in cells)
        split = np.zeros(cx.shape, bool) if lev == max_level else np.asarray(refine(cx, cy, cz, lev), bool)
        keep = ~split
        if keep.any():
            out.append((cells[0][keep], cells[1][keep], cells[2][keep], lev))
        if not split.any():
            break
        sx, sy, sz = (c[split] for c in cells)
        nxt = [[], [], []]
        for o in range(8):   # children in octant order
            nxt[0].append(2 * sx + (o & 1))
            nxt[1].append(2 * sy + ((o >> 1) & 1))
            nxt[2].append(2 * sz + ((o >> 2) & 1))
        cells = [np.concatenate(a) for a in nxt]
    lx, ly, lz, lv, key = [], [], [], [], []
    for ix, iy, iz, lev in out:
        sh = max_level - lev   # lower corner on the finest lattice
        key.append(_morton(ix << sh, iy << sh, iz << sh, max_level))
        h = boxlen / (1 << lev)
        lx.append(-half + (ix + 0.5) * h)
        ly.append(-half + (iy + 0.5) * h)
        lz.append(-half + (iz + 0.5) * h)
        lv.append(np.full(ix.shape, lev, dtype=np.int64))
    key = np.concatenate(key)
    order = np.argsort(key, kind="stable")
    x, y, z, lev = (np.concatenate(a)[order] for a in (lx, ly, lz, lv))
    nH = np.asarray(density(x, y, z, lev), dtype=float)
    return x, y, z, lev, nH


def write_leaf_list(path, boxlen, x, y, z, lev, nH):
    """The generic text leaf list (read_generic_amr.f90:60-81)."""
    n = len(x)
    with open(path, "w") as f:
        f.write(f"{n} {boxlen!r}\n")
        f.writelines(f"{a!r} {b!r} {c!r} {int(l)} {d!r}\n" for a, b, c, l, d in
                     zip(x.tolist(), y.tolist(), z.tolist(), lev.tolist(), nH.tolist()))


def lognormal_field(n=256, mean=30.0, sigma_ln=1.0, slope=-11.0 / 3.0, seed=2024):
    """Periodic log-normal density on an n^3 lattice: a unit-variance Gaussian
    field g with P(k) ~ k^slope (seeded white noise shaped in Fourier space),
    n_H = mean exp(sigma_ln g - sigma_ln^2 / 2) (mean preserving)."""
    rng = np.random.default_rng(seed)
    k = np.fft.fftfreq(n)
    kr = np.fft.rfftfreq(n)
    k2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + kr[None, None, :] ** 2
    amp = np.zeros_like(k2)
    nz = k2 > 0
    amp[nz] = k2[nz] ** (slope / 4.0)   # |g_k| ~ sqrt(P(k)) = k^(slope/2)
    w = rng.standard_normal((n, n, n))
    g = np.fft.irfftn(np.fft.rfftn(w) * amp, s=(n, n, n), axes=(0, 1, 2))
    g = (g - g.mean()) / g.std()
    return mean * np.exp(sigma_ln * g - 0.5 * sigma_ln * sigma_ln)


def clumpy_nebula(boxlen, field, base_level=6, max_level=10, threshold=120.0, growth=1.47):
    """Octree over a density lattice (field[iz, iy, ix], n^3, n a power of
    two covering the box): a cell at level L splits while the mean density
    of the lattice voxels it covers (below the lattice spacing, the voxel's
    own density) exceeds threshold * growth^(L - base_level).  Leaves take
    that density.

    With a fixed threshold (growth = 1) a steep spectrum refines almost every
    dense base cell down to max_level: 4 <n> on the 256^3 log-normal field
    with sigma_ln n = 1 gives 3.5e7 leaves.  The threshold that rises by
    growth per level keeps 4 <n> at the base and reaches level 10 in the
    densest clumps; growth = 1.47 gives about 3e6 leaves."""
    n = field.shape[0]
    lvl = int(round(np.log2(n)))
    if 1 << lvl != n or field.shape != (n, n, n):
        raise ValueError("field must be a cube of side 2^k")
    half = 0.5 * boxlen
    means = {lvl: field}
    for L in range(lvl - 1, -1, -1):   # block means of the coarser levels
        f = means[L + 1]
        m = f.shape[0] // 2
        means[L] = f.reshape(m, 2, m, 2, m, 2).mean(axis=(1, 3, 5))

    def dens(x, y, z, lev):
        lev = np.broadcast_to(np.asarray(lev), np.shape(x))
        out = np.empty(np.shape(x))
        for L in np.unique(lev):
            s = lev == L
            Lc = min(int(L), lvl)
            m = 1 << Lc
            idx = [np.clip(((np.asarray(c)[s] + half) / boxlen * m).astype(np.int64), 0, m - 1) for c in (x, y, z)]
            out[s] = means[Lc][idx[2], idx[1], idx[0]]
        return out

    return build_leaves(boxlen, base_level, max_level,
                        lambda x, y, z, L: dens(x, y, z, L) > threshold * growth ** (L - base_level), dens)
