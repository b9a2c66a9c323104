"""Spatial decomposition of one system over ranks: slabs, particle migration
(map) and halo exchange (ghost_get).

The reference splits the box into sub-domains (`Decomposition/CartDecomposition.hpp`),
sends every particle to the sub-domain that owns its position
(`vector_dist_comm.hpp:1957-2014`, `map`) and copies to each neighbouring
sub-domain the particles within the ghost width of it, shifted by the box
length where the halo crosses a periodic face (`vector_dist_comm.hpp:1398-1596`,
`ghost_get`).  Here a sub-domain is a slab of the box along one axis (the
longest unless given), one slab per rank; a slab is at least as wide as the
ghost, so halos come from the two neighbouring slabs only.

The device work is the library's (`pd_slab_*`): labelling (owners, halo
selection, rows grouped by destination rank), packing into a device buffer of
rows that keep every property's type, and unpacking.  This module only moves
the packed bytes between ranks with two all-to-alls of torch.distributed
(counts, then rows): over NCCL the buffers stay on the GPU, over gloo they pass
through host memory.

Each rank's vector holds its slab with the split axis non-periodic; its own
periodic images (ghost_get of the library) cover the other axes, and the halo
from the neighbouring slabs is appended after them.  Pair kernels of the
library then run over the rank's particles with all of these as neighbours.
"""
import numpy as np
import torch
import torch.distributed as dist

from . import pd


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

    def slab_t(self):
        """The decomposition as the library's pd_slab_t."""
        return pd.SlabT(self.axis, self.P, int(self.periodic), float(self.lo[self.axis]), float(self.hi[self.axis]),
                        self.g)

    def owner(self, x):
        """Rank owning each position (host arrays; the library labels on the device)."""
        x = np.asarray(x, np.float64)
        r = np.floor((x[:, self.axis] - self.lo[self.axis]) / self.width).astype(np.int64)
        return np.clip(r, 0, self.P - 1)

    def local_box(self, rank):
        """(lo, hi, bc) of the rank's vector: its slab along the axis, non-periodic
        there; one rank keeps the global box."""
        lo, hi, bc = self.lo.copy(), self.hi.copy(), self.bc.copy()
        if self.P > 1:
            a = self.axis
            lo[a] = self.edges[rank]
            hi[a] = self.edges[rank + 1]
            bc[a] = 0
        return lo, hi, bc


def exchange_rows(send, send_counts, row_bytes, group=None):
    """All-to-all of packed rows.  `send` is a uint8 tensor of rows grouped by
    destination rank (send_counts[d] rows to rank d, ranks ascending); returns
    (received uint8 tensor on send's device, rows received from each rank)."""
    P = dist.get_world_size(group) if dist.is_initialized() else 1
    if P == 1:
        return send, list(send_counts)
    dev = send.device if dist.get_backend(group) == "nccl" else torch.device("cpu")
    sc = torch.tensor([int(c) for c in send_counts], dtype=torch.int64, device=dev)
    rc = torch.empty_like(sc)
    dist.all_to_all_single(rc, sc, group=group)
    rcl = [int(c) for c in rc.tolist()]
    out = torch.empty(sum(rcl) * row_bytes, dtype=torch.uint8, device=dev)
    dist.all_to_all_single(out, send.to(dev), output_split_sizes=[c * row_bytes for c in rcl],
                           input_split_sizes=[int(c) * row_bytes for c in send_counts], group=group)
    return out.to(send.device), rcl


class DistVector:
    """This rank's slab of a decomposed system: a library vector (`self.vd`) with
    map and ghost_get between ranks.  `props` as for pd.VectorDist."""

    def __init__(self, dec, props=(), dtype=np.float64, group=None):
        self.dec = dec
        self.group = group
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        world = dist.get_world_size(group) if dist.is_initialized() else 1
        if world != dec.P:
            raise ValueError("the decomposition has %d slabs for %d ranks" % (dec.P, world))
        lo, hi, bc = dec.local_box(self.rank)
        self.vd = pd.VectorDist(0, lo, hi, bc, dec.g, dtype=dtype, props=props)
        self.slab = dec.slab_t()
        self.all_props = (1 << len(props)) - 1

    def map(self, props=None):
        """Every particle to the rank owning its (wrapped) position, with the
        properties in `props` (all when None); the ghost is dropped."""
        mask = self.all_props if props is None else sum(1 << p for p in props)
        counts = self.vd.slab_map_label(self.slab)
        rb = self.vd.slab_row_bytes(mask)
        send = self.vd.slab_pack(mask, sum(counts))
        recv, rc = exchange_rows(send, counts, rb, self.group)
        self.vd.slab_map_unpack(mask, recv, sum(rc))

    def ghost_get(self, props=None):
        """The rank's periodic images, then the halo of the neighbouring slabs
        (shifted across periodic faces) with the properties in `props`."""
        mask = self.all_props if props is None else sum(1 << p for p in props)
        self.vd.ghost_get(props)
        counts = self.vd.slab_halo_label(self.slab, self.rank)
        rb = self.vd.slab_row_bytes(mask)
        send = self.vd.slab_pack(mask, sum(counts))
        recv, rc = exchange_rows(send, counts, rb, self.group)
        self.vd.slab_halo_unpack(mask, recv, sum(rc))


def lj_forces_distributed(dv, force_prop, r_cut=2.5, eps=1.0, sigma=1.0, ghost_props=()):
    """LJ forces of this rank's particles into property `force_prop`: ghost_get
    (positions and `ghost_props`), the library's cell list over the rank's
    particles, images and halo, and its pair kernel.  Returns (PE, virial) of the
    rank's particles."""
    dv.ghost_get(list(ghost_props))
    cl = dv.vd.getCellListGPU(r_cut)
    dv.vd.updateCellListGPU(cl)
    return dv.vd.lj_forces(force_prop, cl=cl, eps=eps, sigma=sigma, r_cut=r_cut)


def md_distributed(dv, steps, vel_prop, force_prop, dt=0.005, mass=1.0, **lj):
    """Velocity-Verlet steps of the decomposed system held by `dv`: each step
    kicks, drifts, migrates the particles to their owners (map, every property)
    and exchanges the halo for the new forces.  The elementwise updates run on
    the GPU through torch on the vector's data."""
    h = 0.5 * dt / mass
    vd = dv.vd
    lj_forces_distributed(dv, force_prop, **lj)
    for _ in range(steps):
        n = vd.size_local()
        x = vd.deviceToHostPos(count=n, device=True)
        v = vd.deviceToHostProp(vel_prop, count=n, device=True)
        f = vd.deviceToHostProp(force_prop, count=n, device=True)
        v = v + h * f
        vd.hostToDevicePos(x + dt * v)
        vd.hostToDeviceProp(vel_prop, v)
        dv.map()
        lj_forces_distributed(dv, force_prop, **lj)
        n = vd.size_local()
        v = vd.deviceToHostProp(vel_prop, count=n, device=True)
        f = vd.deviceToHostProp(force_prop, count=n, device=True)
        vd.hostToDeviceProp(vel_prop, v + h * f)
