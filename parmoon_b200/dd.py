"""Domain decomposition of a structured hierarchy into z-slabs, one per rank,
and the transport of pmg_solve_dd over torch.distributed.

The reference's parallel mode (src/Parallel/ParFECommunicator3D.C:218-346)
keeps, per rank, the cells of its subdomain plus the neighbouring cells, the
dofs it owns ("master") and copies of the neighbours' dofs on the shared cells,
updated by CommUpdate.  Here a rank's subdomain at every level is the slab
z in [r/R, (r+1)/R) of the unit cube (R ranks; the slabs follow coarse cell
layers, so they are nested across the levels) plus one layer of cells on
either side.  The local numbering puts the rank's active owned dofs first,
then its own Dirichlet dofs, then the ghost dofs (owned by the neighbouring
ranks); the local problem treats every row past the active ones as a
Dirichlet row.  A dof on a slab face belongs to the slab above it (the top
face of the cube to the last slab).

`local_hierarchy` gives, per level, the arrays pmg_set_level_* take (local
cell order = global cell order restricted), the local prolongation, the
lattice row colours, the map local -> global dof, and on the finest level the
halo: the owned dofs each neighbour needs (sorted by global dof) and the ghost
rows filled from each neighbour (sorted by global dof).  `TorchComm` moves the
packed halo buffers and sums the inner products through torch.distributed
(NCCL for device tensors on one GPU per rank, or gloo through host copies).
"""
import ctypes

import numpy as np

from . import Q1_HEX, Q2_HEX, struct_hierarchy


def _cell_layer(elem, cell_vert, n):
    """z layer (0..n-1) of every cell of a level with n cells per direction (by centroid)."""
    v = np.asarray(cell_vert).reshape(-1, 8, 3)
    nv = 8 if elem in (Q1_HEX, Q2_HEX) else 4
    zc = v[:, :nv, 2].mean(axis=1)
    return np.clip(np.floor(zc * n).astype(np.int64), 0, n - 1)


def owner_of(z, n_ranks):
    """Owning rank of a dof at height z (slab [r/R, (r+1)/R); z = 1 to the last)."""
    return np.minimum(np.floor(np.asarray(z) * n_ranks + 1e-9).astype(np.int64), n_ranks - 1)


def local_level(L, n_ranks, rank):
    """The subdomain of one level: local arrays and the local <-> global dof maps."""
    n = L["n"]
    if n % n_ranks:
        raise ValueError("the cells per direction of every level must be a multiple of the rank count")
    layer = _cell_layer(L["elem"], L["cell_vert"], n)
    lo, hi = rank * n // n_ranks, (rank + 1) * n // n_ranks
    cells = np.nonzero((layer >= lo - 1) & (layer <= hi))[0]
    nloc = L["elem_dof"].size // L["n_cells"]
    ed_g = L["elem_dof"].reshape(-1, nloc)[cells]
    dofs = np.unique(ed_g)
    z = L["dof_xyz"][dofs, 2]
    own = owner_of(z, n_ranks) == rank
    active_g = dofs < L["active_bound"]
    order = np.concatenate([dofs[own & active_g], dofs[own & ~active_g], dofs[~own]])
    na = int(np.count_nonzero(own & active_g))
    n_own = int(np.count_nonzero(own))
    g2l = np.full(L["N"], -1, dtype=np.int64)
    g2l[order] = np.arange(order.size)
    ed_l = g2l[ed_g].astype(np.int32).ravel()
    cv_l = L["cell_vert"].reshape(-1, 24)[cells].ravel()
    return dict(elem=L["elem"], n=n, cells=cells, glob=order, g2l=g2l, N=int(order.size), active_bound=na,
                n_owned=n_own, elem_dof=ed_l, cell_vert=cv_l, dof_xyz=L["dof_xyz"][order],
                colors=L["colors"][order].astype(np.int32), n_colors=L["n_colors"],
                owner=owner_of(L["dof_xyz"][order, 2], n_ranks))


def local_hierarchy(elem, n_fine, n_levels, n_ranks, rank):
    """Per-level subdomains of struct_hierarchy(elem, n_fine, n_levels) for `rank`, with local
    prolongations and, on the finest level, the halo (send / receive lists per neighbour)."""
    glob = struct_hierarchy(elem, n_fine, n_levels)
    loc = [local_level(L, n_ranks, rank) for L in glob]
    for l in range(1, n_levels):
        prp, pcol, pval = glob[l]["P"]
        F, C = loc[l], loc[l - 1]
        rows = F["glob"]
        starts, ends = prp[rows], prp[rows + 1]
        cnt = (ends - starts).astype(np.int64)
        rp = np.zeros(rows.size + 1, dtype=np.int32)
        rp[1:] = np.cumsum(cnt)
        idx = np.concatenate([np.arange(s, e) for s, e in zip(starts, ends)]) if rows.size else np.zeros(0, int)
        col = C["g2l"][pcol[idx]]
        if np.any(col < 0):
            raise RuntimeError("a fine dof of the subdomain has a coarse dof outside the coarse subdomain")
        F["P"] = (rp, col.astype(np.int32), pval[idx].copy())
    F = loc[-1]
    neighbours = [q for q in (rank - 1, rank + 1) if 0 <= q < n_ranks]
    recv, send = {}, {}
    for q in neighbours:
        # ghosts of this rank owned by q, and owned dofs of this rank that are ghosts of q
        recv[q] = np.nonzero(F["owner"] == q)[0]
        Fq = local_level(glob[-1], n_ranks, q)
        theirs = Fq["glob"][Fq["owner"] == rank]
        send[q] = np.sort(F["g2l"][theirs])
        if np.any(send[q] < 0):
            raise RuntimeError("a ghost of a neighbour is not in this subdomain")
    # both sides order a segment by global dof
    for q in neighbours:
        recv[q] = recv[q][np.argsort(F["glob"][recv[q]], kind="stable")]
        send[q] = send[q][np.argsort(F["glob"][send[q]], kind="stable")]
    F["neighbours"] = neighbours
    F["recv"] = recv
    F["send"] = send
    return glob, loc


class TorchComm:
    """pmg_comm over torch.distributed: the halo segments of the finest level
    go to / come from the slab neighbours, the sums are all-reduces.  With the
    NCCL backend the device buffers are sent as they are; with gloo they go
    through host copies."""

    ALLREDUCE = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int)
    EXCHANGE = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                ctypes.c_int)

    def __init__(self, dist, F, device="cuda"):
        import torch
        self.dist, self.torch = dist, torch
        self.nccl = dist.get_backend() == "nccl"
        self.neighbours = F["neighbours"]
        self.send_idx = np.concatenate([F["send"][q] for q in self.neighbours] or [np.zeros(0, int)]).astype(np.int32)
        self.recv_idx = np.concatenate([F["recv"][q] for q in self.neighbours] or [np.zeros(0, int)]).astype(np.int32)
        self.send_len = [len(F["send"][q]) for q in self.neighbours]
        self.recv_len = [len(F["recv"][q]) for q in self.neighbours]
        self.send_buf = torch.zeros(max(1, self.send_idx.size), dtype=torch.float64, device=device)
        self.recv_buf = torch.zeros(max(1, self.recv_idx.size), dtype=torch.float64, device=device)
        self._allreduce = self.ALLREDUCE(self._allreduce_sum)
        self._exchange = self.EXCHANGE(self._exchange_cb)

    def _allreduce_sum(self, ctx, v, n):
        try:
            torch = self.torch
            a = np.ctypeslib.as_array(v, shape=(n,))
            t = torch.from_numpy(a.copy())
            if self.nccl:
                t = t.cuda()
            self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
            a[:] = t.cpu().numpy()
            return 0
        except Exception:
            return 1

    def _exchange_cb(self, ctx, send_dev, n_send, recv_dev, n_recv):
        try:
            torch = self.torch
            dist = self.dist
            ops, bufs = [], []
            so = ro = 0
            for q, ns, nr in zip(self.neighbours, self.send_len, self.recv_len):
                s = self.send_buf[so:so + ns]
                r = self.recv_buf[ro:ro + nr]
                if not self.nccl:
                    s, r = s.cpu(), torch.empty(nr, dtype=torch.float64)
                ops.append(dist.P2POp(dist.isend, s, q))
                ops.append(dist.P2POp(dist.irecv, r, q))
                bufs.append((r, ro, nr))
                so += ns
                ro += nr
            if ops:
                for req in dist.batch_isend_irecv(ops):
                    req.wait()
            if not self.nccl:
                for r, o, nr in bufs:
                    self.recv_buf[o:o + nr].copy_(r)
            torch.cuda.synchronize()
            return 0
        except Exception:
            return 1

    def struct(self, lib):
        class PmgComm(ctypes.Structure):
            _fields_ = [("ctx", ctypes.c_void_p), ("allreduce_sum", self.ALLREDUCE), ("exchange", self.EXCHANGE)]
        self._c = PmgComm(None, self._allreduce, self._exchange)
        return self._c


def load_subdomain(h, loc, dirichlet=None):
    """Hand a rank's local hierarchy to its Handle: patterns built on the device, meshes,
    colours, local prolongations, Dirichlet values (ghost rows 0: they are filled from the
    neighbours)."""
    for l, L in enumerate(loc):
        nloc = L["elem_dof"].size // L["cells"].size
        h.build_level_csr(l, L["elem_dof"], nloc, L["N"], L["active_bound"])
        h.set_level_mesh(l, L["elem"], L["elem_dof"], L["cell_vert"], brick=L["elem"] in (Q1_HEX, Q2_HEX))
        h.set_row_colors(l, L["colors"], L["n_colors"])
        if l > 0:
            rp, col, val = L["P"]
            h.set_transfer(l, rp, col, val, loc[l - 1]["N"])
        Na = L["active_bound"]
        xyz = L["dof_xyz"][Na:]
        vals = np.zeros(len(xyz)) if dirichlet is None else dirichlet(xyz[:, 0], xyz[:, 1], xyz[:, 2])
        vals[L["n_owned"] - Na:] = 0.0
        h.set_dirichlet_values(l, vals)


def exchange_host(dist, F, x):
    """The halo protocol of TorchComm on a host vector (local numbering of the
    finest level): the neighbours' values of the ghost rows, in place."""
    import torch
    ops, bufs = [], []
    for q in F["neighbours"]:
        s = torch.from_numpy(np.ascontiguousarray(x[F["send"][q]], dtype=np.float64))
        r = torch.empty(len(F["recv"][q]), dtype=torch.float64)
        ops += [dist.P2POp(dist.isend, s, q), dist.P2POp(dist.irecv, r, q)]
        bufs.append((q, r))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    for q, r in bufs:
        x[F["recv"][q]] = r.numpy()
    return x
