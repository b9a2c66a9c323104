"""Spatial decomposition of one system over ranks: slabs, particle migration
(map) and halo exchange (ghost_get) over torch.distributed.

The reference splits the box into sub-domains (`Decomposition/CartDecomposition.hpp`),
sends every particle to the sub-domain that owns its position
(`vector_dist_comm.hpp:1957-2014`, `map`) and copies to each neighbouring
sub-domain the particles within the ghost width of it, shifted by the box
length where the halo crosses a periodic face (`vector_dist_comm.hpp:1398-1596`,
`ghost_get`).  Here a sub-domain is a slab of the box along one axis (the
longest unless given), one slab per rank; a slab is at least as wide as the
ghost, so halos come from the two neighbouring slabs only.  Both exchanges are
two all-to-alls (counts, then rows of float64 columns), NCCL between GPUs or
gloo on the host, on tensors of any device.

Forces of a rank's particles come from the single-GPU library on the rank's
extended slab: its own particles followed by the received halo, the slab's
axis non-periodic and widened by the ghost on both sides, the other axes as
the global box (the library adds their periodic images).  Only the rank's own
particles' forces are kept.
"""
import numpy as np
import torch
import torch.distributed as dist


class SlabDecomposition:
    """Slabs [edges[r], edges[r+1]) of the box along `axis`, one per rank."""

    def __init__(self, lo, hi, bc, ghost, nranks, axis=None):
        self.lo = np.asarray(lo, np.float64).reshape(3)
        self.hi = np.asarray(hi, np.float64).reshape(3)
        self.bc = np.asarray(bc, np.int32).reshape(3)
        self.g = float(np.max(ghost))
        self.P = int(nranks)
        if self.P < 1:
            raise ValueError("at least one rank")
        ext = self.hi - self.lo
        self.axis = int(np.argmax(ext)) if axis is None else int(axis)
        a = self.axis
        self.L = float(ext[a])
        self.width = self.L / self.P
        if self.P > 1 and self.width < self.g:
            raise ValueError("a slab (%g) is narrower than the ghost (%g)" % (self.width, self.g))
        self.edges = self.lo[a] + self.width * np.arange(self.P + 1)
        self.edges[-1] = self.hi[a]
        self.periodic = bool(self.bc[a] == 1)

    def wrap(self, x):
        """Positions folded into the box along the periodic axes."""
        x = x.clone()
        for d in range(3):
            if self.bc[d] == 1:
                L = float(self.hi[d] - self.lo[d])
                x[:, d] = self.lo[d] + torch.remainder(x[:, d] - self.lo[d], L)
        return x

    def owner(self, x):
        """Rank owning each position (int64 tensor on x's device)."""
        r = torch.floor((x[:, self.axis] - self.lo[self.axis]) / self.width).to(torch.int64)
        return r.clamp_(0, self.P - 1)

    def local_box(self, rank):
        """(lo, hi, bc) of the rank's extended slab for the single-GPU library."""
        lo, hi, bc = self.lo.copy(), self.hi.copy(), self.bc.copy()
        if self.P > 1:
            a = self.axis
            lo[a] = self.edges[rank] - self.g
            hi[a] = self.edges[rank + 1] + self.g
            bc[a] = 0
        return lo, hi, bc

    def halo_sends(self, rank, x):
        """[(destination, indices, shift along the axis)] of the rank's particles
        within the ghost of a neighbouring slab.  One rank: none (the library's
        periodic images cover the box)."""
        if self.P == 1:
            return []
        a = self.axis
        lo_thr, hi_thr = self.edges[rank] + self.g, self.edges[rank + 1] - self.g
        native = None
        if x.is_cuda and x.dtype == torch.float64:
            from . import pd  # the library's selection kernel (same comparisons, ascending indices)
            native = pd.slab_halo(x, a, lo_thr, hi_thr)
        out = []
        for side in (+1, -1):
            dest, shift = rank + side, 0.0
            if dest == self.P or dest == -1:
                if not self.periodic:
                    continue
                dest = dest % self.P
                shift = -self.L if side > 0 else self.L
            if native is not None:
                out.append((dest, native[1] if side > 0 else native[0], shift))
                continue
            sel = x[:, a] >= hi_thr if side > 0 else x[:, a] < lo_thr
            out.append((dest, torch.nonzero(sel).flatten(), shift))
        return out


def _pack(x, props):
    cols = [x.to(torch.float64)]
    meta = []
    for p in props:
        if p.dtype not in (torch.float64, torch.float32, torch.int32):
            raise TypeError("properties must be float64, float32 or int32 (packed exactly as float64)")
        k = int(np.prod(p.shape[1:], dtype=np.int64)) if p.dim() > 1 else 1
        q = p.reshape(p.shape[0], k)
        meta.append((p.dtype, tuple(p.shape[1:]), k))
        cols.append(q.to(torch.float64))
    return torch.cat(cols, dim=1), meta


def _unpack(rows, meta):
    x = rows[:, :3].contiguous()
    props, c = [], 3
    for dt, shp, k in meta:
        props.append(rows[:, c:c + k].to(dt).reshape((rows.shape[0],) + shp))
        c += k
    return x, props


class DistParticles:
    """map / ghost_get of one system decomposed in slabs over the ranks of `group`."""

    def __init__(self, dec, group=None):
        self.dec = dec
        self.group = group
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        world = dist.get_world_size(group) if dist.is_initialized() else 1
        if world != dec.P:
            raise ValueError("the decomposition has %d slabs for %d ranks" % (dec.P, world))

    def _exchange(self, rows, dest):
        """Rows sent to their destination ranks; the rows received, in rank order."""
        P = self.dec.P
        order = torch.argsort(dest, stable=True)
        rows = rows[order].contiguous()
        sc = torch.bincount(dest, minlength=P).to(torch.int64)
        if P == 1:
            return rows
        rc = torch.empty_like(sc)
        dist.all_to_all_single(rc, sc, group=self.group)
        out = torch.empty((int(rc.sum()), rows.shape[1]), dtype=rows.dtype, device=rows.device)
        dist.all_to_all_single(out, rows, output_split_sizes=rc.tolist(), input_split_sizes=sc.tolist(),
                               group=self.group)
        return out

    def map(self, x, props=()):
        """Every particle to the rank owning its (wrapped) position: (x, props) held here."""
        x = self.dec.wrap(x)
        rows, meta = _pack(x, props)
        return _unpack(self._exchange(rows, self.dec.owner(x)), meta)

    def ghost_get(self, x, props=()):
        """Halo received from the neighbouring slabs (positions shifted across
        periodic faces): (x, props) to append after this rank's particles."""
        sends = self.dec.halo_sends(self.rank, x)
        rows, meta = _pack(x, props)
        parts, dests = [], []
        for dest, idx, shift in sends:
            r = rows[idx].clone()
            r[:, self.dec.axis] += shift
            parts.append(r)
            dests.append(torch.full((idx.shape[0],), dest, dtype=torch.int64, device=x.device))
        if parts:
            send = torch.cat(parts)
            dest = torch.cat(dests)
        else:
            send = rows[:0]
            dest = torch.zeros(0, dtype=torch.int64, device=x.device)
        return _unpack(self._exchange(send, dest), meta)


def lj_forces_library(x, lo, hi, bc, r_cut=2.5, eps=1.0, sigma=1.0):
    """LJ forces of the particles x [n, 3] (float64; a host array, or a CUDA
    tensor kept on the GPU) in the box (lo, hi, bc), computed by the single-GPU
    library (cell list of side r_cut, periodic images of the periodic axes)."""
    from . import pd
    on_gpu = isinstance(x, torch.Tensor) and x.is_cuda
    if not on_gpu:
        x = np.ascontiguousarray(np.asarray(x, np.float64))
    n = x.shape[0]
    vd = pd.VectorDist(n, lo, hi, np.asarray(bc, np.int32), r_cut, dtype=np.float64, props=[(pd.PD_F64, 3)])
    vd.hostToDevicePos(x)
    vd.ghost_get()
    cl = vd.getCellListGPU(r_cut)
    vd.updateCellListGPU(cl)
    vd.lj_forces(0, cl=cl, eps=eps, sigma=sigma, r_cut=r_cut)
    return vd.deviceToHostProp(0, count=n, device=on_gpu)


def lj_forces_distributed(dp, x, force_fn=lj_forces_library, **kw):
    """Forces of this rank's particles x (after `map`): halo exchange, then the
    single-GPU forces on the extended slab; `force_fn(x_all, lo, hi, bc, **kw)`.
    CUDA tensors stay on the GPU (the library reads and writes them in place of
    host arrays); host tensors go through numpy."""
    xh, _ = dp.ghost_get(x)
    lo, hi, bc = dp.dec.local_box(dp.rank)
    allx = torch.cat([x, xh])
    if allx.is_cuda and force_fn is lj_forces_library:
        return force_fn(allx.contiguous(), lo, hi, bc, **kw)[: x.shape[0]]
    f = force_fn(allx.cpu().numpy(), lo, hi, bc, **kw)
    return torch.from_numpy(np.ascontiguousarray(f[: x.shape[0]])).to(x.device)


def md_distributed(dp, x, v, steps, props=(), dt=0.005, mass=1.0, force_fn=lj_forces_library, **kw):
    """Velocity-Verlet steps of the decomposed system (x, v and `props` of this
    rank's particles after `map`): each step kicks, drifts, migrates the
    particles to their owners (`map`, carrying v and props) and exchanges the
    halo for the new forces.  Returns (x, v, props) held here at the end."""
    h = 0.5 * dt / mass
    props = list(props)
    f = lj_forces_distributed(dp, x, force_fn, **kw)
    for _ in range(steps):
        v = v + h * f
        x = x + dt * v
        x, moved = dp.map(x, [v] + props)
        v, props = moved[0], moved[1:]
        f = lj_forces_distributed(dp, x, force_fn, **kw)
        v = v + h * f
    return x, v, props
