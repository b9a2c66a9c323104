"""Seeded synthetic inputs for the particle workloads (host numpy arrays).

The reference measures on synthetic particle sets only (its performance
harness draws uniform random particles, e.g.
Vector/performance/vector_dist_performance_common.hpp:141-198); these
generators produce the benchmark shapes of this project:

* ``lj_lattice``   -- simple-cubic lattice + uniform jitter, Gaussian velocities
                      (16^3 at spacing 1.0 in a 16 box; 160^3 at 1.1 in a 176 box)
* ``lj_clustered`` -- Gaussian clusters with a minimum-distance rejection
* ``sph_dam``      -- dam-break fluid block plus fixed wall layers
* ``serving_sizes``-- log-uniform system sizes for the serving stream
"""
import numpy as np


def maxwell_velocities(n, temperature, mass, rng):
    v = rng.normal(0.0, np.sqrt(temperature / mass), size=(n, 3))
    v -= v.mean(axis=0, keepdims=True)
    return v


def lj_lattice(n_side, spacing, jitter, seed=1, temperature=1.0, mass=1.0):
    """n_side^3 particles on a simple-cubic lattice (cell centres), jitter
    U(-jitter, jitter) per coordinate, box [0, n_side*spacing)^3.
    Returns (x[N,3] f64, v[N,3] f64, L)."""
    rng = np.random.default_rng(seed)
    L = n_side * spacing
    k = (np.arange(n_side) + 0.5) * spacing
    z, y, x = np.meshgrid(k, k, k, indexing="ij")
    pos = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    pos += rng.uniform(-jitter, jitter, size=pos.shape)
    pos = np.mod(pos, L)
    pos[pos >= L] = 0.0
    v = maxwell_velocities(pos.shape[0], temperature, mass, rng)
    return pos, v, L


def lj_clustered(n, L, n_clusters=64, sigma_c=8.0, min_dist=0.8, seed=4, temperature=1.0, mass=1.0,
                 max_tries=64):
    """n particles in n_clusters Gaussian clusters (std sigma_c per axis) at
    uniform centres in a periodic box of side L.  A candidate closer than
    min_dist (minimum image) to an accepted particle is redrawn, up to
    max_tries times per particle; after that its cluster centre is redrawn.
    Returns (x, v, L)."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0, L, size=(n_clusters, 3))
    cell = min_dist
    nc = max(1, int(L // cell))
    cell = L / nc
    grid = {}
    out = np.empty((n, 3))
    md2 = min_dist * min_dist
    per = n // n_clusters
    cid = np.minimum(np.arange(n) // max(per, 1), n_clusters - 1)
    batch = 1 << 14
    cand = None
    ci = 0
    for i in range(n):
        tries = 0
        while True:
            if cand is None or ci >= cand.shape[0]:
                cand = rng.normal(0.0, sigma_c, size=(batch, 3))
                ci = 0
            p = np.mod(centres[cid[i]] + cand[ci], L)
            ci += 1
            key = tuple((p // cell).astype(np.int64) % nc)
            ok = True
            for dz in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dx in (-1, 0, 1):
                        kk = ((key[0] + dx) % nc, (key[1] + dy) % nc, (key[2] + dz) % nc)
                        lst = grid.get(kk)
                        if not lst:
                            continue
                        q = out[lst]
                        d = p - q
                        d -= L * np.round(d / L)
                        if np.any((d * d).sum(axis=1) < md2):
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                break
            tries += 1
            if tries >= max_tries:
                centres[cid[i]] = rng.uniform(0, L, size=3)
                tries = 0
        out[i] = p
        grid.setdefault(key, []).append(i)
    out[out >= L] = 0.0
    v = maxwell_velocities(n, temperature, mass, rng)
    return out, v, L


def sph_dam(dp, fluid=(0.4, 1.0, 0.6), box=(1.0, 1.0, 1.0), wall_layers=3, rho0=1000.0, seed=5):
    """Dam-break block [0,fx]x[0,fy]x[0,fz] of fluid on a lattice of spacing dp
    inside a tank [0,bx]x[0,by]x[0,bz] whose floor and four sides carry
    ``wall_layers`` layers of fixed wall particles (outside the tank).
    Returns (x[N,3], type[N] int32 (0 fluid, 1 wall), mass, domain_lo, domain_hi)."""
    fx, fy, fz = fluid
    bx, by, bz = box
    nfx, nfy, nfz = int(round(fx / dp)), int(round(fy / dp)), int(round(fz / dp))
    i = (np.arange(nfx) + 0.5) * dp
    j = (np.arange(nfy) + 0.5) * dp
    k = (np.arange(nfz) + 0.5) * dp
    z, y, x = np.meshgrid(k, j, i, indexing="ij")
    flu = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    nbx, nby, nbz = int(round(bx / dp)), int(round(by / dp)), int(round(bz / dp))
    wi = (np.arange(-wall_layers, nbx + wall_layers) + 0.5) * dp
    wj = (np.arange(-wall_layers, nby + wall_layers) + 0.5) * dp
    wk = (np.arange(-wall_layers, nbz) + 0.5) * dp
    z, y, x = np.meshgrid(wk, wj, wi, indexing="ij")
    w = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    inside = (w[:, 0] > 0) & (w[:, 0] < bx) & (w[:, 1] > 0) & (w[:, 1] < by) & (w[:, 2] > 0)
    w = w[~inside]
    pos = np.concatenate([flu, w])
    typ = np.concatenate([np.zeros(flu.shape[0], np.int32), np.ones(w.shape[0], np.int32)])
    mass = rho0 * dp ** 3
    lo = np.array([-(wall_layers + 1) * dp, -(wall_layers + 1) * dp, -(wall_layers + 1) * dp])
    hi = np.array([bx + (wall_layers + 1) * dp, by + (wall_layers + 1) * dp, bz + (wall_layers + 1) * dp])
    return pos, typ, mass, lo, hi


def serving_sizes(count, lo=512, hi=262144, seed=6):
    """System sizes N = round(exp(U(ln lo, ln hi)))."""
    rng = np.random.default_rng(seed)
    return np.rint(np.exp(rng.uniform(np.log(lo), np.log(hi), size=count))).astype(np.int64)


def serving_system(n, density=0.8, seed=0, temperature=1.0):
    """A jittered cubic lattice of about n particles at the given number density
    (box L = (n/density)^(1/3)); returns exactly n particles (x, v, L)."""
    rng = np.random.default_rng(seed)
    L = (n / density) ** (1.0 / 3.0)
    side = int(np.ceil(n ** (1.0 / 3.0)))
    sp = L / side
    k = (np.arange(side) + 0.5) * sp
    z, y, x = np.meshgrid(k, k, k, indexing="ij")
    pos = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    sel = rng.permutation(pos.shape[0])[:n]
    pos = pos[np.sort(sel)]
    pos += rng.uniform(-0.05 * sp, 0.05 * sp, size=pos.shape)
    pos = np.mod(pos, L)
    pos[pos >= L] = 0.0
    v = maxwell_velocities(n, temperature, 1.0, rng)
    return pos, v, L
