"""Domain-decomposed R+K assembly over ranks (one process per GPU).

The reference assembles per MPI rank over its own elements: entries of rows
the rank owns go into its block of the parallel matrix, entries of rows owned
by other ranks are collected per peer (PLoc_Sparse's Lk[proc],
src/PLoc_Sparse.cc:143-170) and summed into the owners' rows by the
post / send / assemble_nonlocal exchange of ISIR_SparseComm
(src/communication/ISIR_SparseComm.cc:119-200), with the elements on the
partition boundary assembled first so that the exchange overlaps the interior
(src/stiffmat_fd.cc:863-983).  Here:

* partition: contiguous slabs of the element order; with the reference's
  first-visit DOF numbering (src/generate_dof_ids.cc:306-412) the DOFs first
  visited by slab p are one contiguous id range, which is the block of rows
  rank p owns (blocked row distribution);
* each rank assembles two pieces -- its boundary elements (touching a row
  another rank owns) and its interior elements -- each a mesh of its own with
  local DOF ids (the global ids renumbered in order) and its own CSR pattern
  (Psparse_ApAi of the piece), so any assembly backend runs it unchanged (a
  device context of this library, or the CPU oracle in tests);
* the piece entries of rows owned elsewhere are sent to their owners as one
  buffer per peer (point-to-point sends posted after the boundary piece,
  waited for after the interior piece); every rank adds its own entries and
  the received ones into its owned rows at positions fixed at set-up (each
  sender's positions are sent once, at set-up);
* the status word (counts of inverted elements, non-converged points, bad
  diagonals, other) is reduced with MAX over the ranks;
* u of the rows a rank does not own (ghosts) comes from the owners through the
  reverse exchange (gather_ghosts).

Element state stays with the rank that owns the element; nothing else moves.
The exchange runs on torch.distributed (NCCL over NVLink between GPUs, gloo on
CPU).
"""
import numpy as np

import pgfem_gpu as pg


def slab_bounds(ne, nparts):
    """Element ranges [b[p], b[p+1]) of the slabs (equal sizes, the last one
    takes the remainder)."""
    return np.array([(ne * p) // nparts for p in range(nparts + 1)], dtype=np.int64)


def row_bounds(conn, ids, ndof, ebounds):
    """Owned row ranges [r[p], r[p+1]): the DOFs first visited by slab p.  With
    first-visit numbering these are contiguous; checked here."""
    nparts = len(ebounds) - 1
    r = np.zeros(nparts + 1, dtype=np.int64)
    seen = 0
    for p in range(nparts):
        e0, e1 = ebounds[p], ebounds[p + 1]
        d = ids[conn[e0:e1].ravel()].ravel()
        d = d[d > 0]
        mx = int(d.max()) if d.size else 0
        seen = max(seen, mx)
        r[p + 1] = seen
    r[nparts] = ndof
    # contiguity: every DOF first visited in slab p lies in (r[p], r[p+1]]
    first = np.full(ndof + 1, -1, dtype=np.int64)
    for p in range(nparts):
        d = ids[conn[ebounds[p]:ebounds[p + 1]].ravel()].ravel()
        d = np.unique(d[d > 0])
        new = d[first[d] < 0]
        first[new] = p
        if new.size and (new.min() <= r[p] or new.max() > r[p + 1]):
            raise ValueError("DOF numbering is not first-visit over the element order")
    return r


class Piece:
    """A subset of one rank's elements as a mesh of its own: nodes, local DOF
    ids (global free ids renumbered in order; fixed 0 and prescribed ids kept),
    the piece's CSR pattern, and for every R / K entry its global row and its
    position in the global CSR."""

    def __init__(self, X, conn, ids, elems, Ap, Ai, ndof):
        self.elems = np.asarray(elems, dtype=np.int64)
        c = conn[self.elems]
        nodes, inv = np.unique(c.ravel(), return_inverse=True)
        self.nodes = nodes
        self.X = X[nodes]
        self.conn = inv.reshape(c.shape).astype(np.int32)
        gids = ids[nodes]
        free = np.unique(gids[gids > 0])
        self.gdof = free - 1                      # local row -> global row (0-based)
        loc = np.zeros(ndof + 1, dtype=np.int64)
        loc[free] = np.arange(1, len(free) + 1)
        self.ids = np.where(gids > 0, loc[np.maximum(gids, 0)], gids)
        self.ndof = len(free)
        if self.ndof:
            self.Ap, self.Ai = pg.psparse_apai(self.conn, self.ids, self.ndof)
        else:
            self.Ap, self.Ai = np.zeros(1, dtype=np.int32), np.zeros(0, dtype=np.int32)
        rows = np.repeat(np.arange(self.ndof), np.diff(self.Ap))
        self.krow = self.gdof[rows]               # global row of each K entry
        gcol = self.gdof[self.Ai]
        # position of (row, col) in the global CSR: one sorted key per entry
        # of the global rows the piece spans, (row - rmin) * (ndof + 1) + col
        self.kpos = np.zeros(0, dtype=np.int64)
        if len(self.krow):
            rmin, rmax = int(self.krow.min()), int(self.krow.max())
            a0, a1 = int(Ap[rmin]), int(Ap[rmax + 1])
            seg_rows = np.repeat(np.arange(rmin, rmax + 1, dtype=np.int64), np.diff(Ap[rmin:rmax + 2]))
            keys = (seg_rows - rmin) * (ndof + 1) + np.asarray(Ai[a0:a1], dtype=np.int64)
            q = (self.krow - rmin) * (ndof + 1) + gcol
            j = np.searchsorted(keys, q)
            if np.any(j >= len(keys)) or np.any(keys[np.minimum(j, len(keys) - 1)] != q):
                raise ValueError("piece pattern not inside the global pattern")
            self.kpos = a0 + j

    def local_u(self, u_global):
        return np.asarray(u_global)[self.gdof]


class RankPlan:
    """One rank's share of a partitioned assembly: its boundary and interior
    pieces, its owned rows, and the exchange lists."""

    def __init__(self, X, conn, ids, ndof, Ap, Ai, nparts, rank):
        conn = np.asarray(conn)
        ids = np.asarray(ids)
        Ap = np.asarray(Ap).astype(np.int64)
        Ai = np.asarray(Ai)
        self.nparts, self.rank, self.ndof = nparts, rank, ndof
        self.eb = slab_bounds(conn.shape[0], nparts)
        self.rb = row_bounds(conn, ids, ndof, self.eb)
        self.row0, self.row1 = int(self.rb[rank]), int(self.rb[rank + 1])
        self.k0, self.k1 = int(Ap[self.row0]), int(Ap[self.row1])
        # the owned block of the global pattern
        self.Ap_owned = (Ap[self.row0:self.row1 + 1] - self.k0).astype(np.int32)
        self.Ai_owned = Ai[self.k0:self.k1]
        elems = np.arange(self.eb[rank], self.eb[rank + 1])
        d = ids[conn[elems]]
        owner_of = self.owner
        foreign = np.zeros(len(elems), dtype=bool)
        for a in range(conn.shape[1]):
            for j in range(3):
                g = d[:, a, j]
                m = g > 0
                foreign[m] |= owner_of(g[m] - 1) != rank
        self.boundary = Piece(X, conn, ids, elems[foreign], Ap, Ai, ndof) if foreign.any() else None
        self.interior = Piece(X, conn, ids, elems[~foreign], Ap, Ai, ndof) if (~foreign).any() else None
        self.pieces = [p for p in (self.boundary, self.interior) if p is not None]
        self.Ap = Ap
        # own entries: (piece index, R local idx, R owned idx, K local idx, K owned idx)
        # send[q]: (R local idx, K local idx) of the boundary piece's entries owned by q
        self.own, self.send = [], {}
        for ip, pc in enumerate(self.pieces):
            r_own = owner_of(pc.gdof)
            k_own = owner_of(pc.krow)
            rl, kl = np.nonzero(r_own == rank)[0], np.nonzero(k_own == rank)[0]
            self.own.append((ip, rl, pc.gdof[rl] - self.row0, kl, pc.kpos[kl] - self.k0))
            if pc is self.interior:
                assert rl.size == pc.ndof and kl.size == len(pc.krow)  # interior rows are all owned here
                continue
            for q in range(nparts):
                if q != rank:
                    rq, kq = np.nonzero(r_own == q)[0], np.nonzero(k_own == q)[0]
                    if rq.size or kq.size:
                        self.send[q] = (rq, kq)

    def owner(self, grow):
        return np.searchsorted(self.rb, np.asarray(grow), side="right") - 1

    def send_positions(self, q):
        """Owned-block positions at rank q (R rows, K entries) of the values
        this rank sends it, in send order."""
        if q not in self.send:
            return np.zeros(0, np.int64), np.zeros(0, np.int64)
        rq, kq = self.send[q]
        pc = self.boundary
        return pc.gdof[rq] - self.rb[q], pc.kpos[kq] - self.Ap[self.rb[q]]


class DistributedAssembly:
    """Partitioned R+K assembly of one rank.

    backend(piece, u_local, u_presc) -> (R_local, K_local, status(4)) assembles
    one piece (a device context of this library, or the CPU oracle in tests).
    assemble_RK(u_owned_and_ghosts) returns this rank's owned rows (R over
    [row0, row1), K over the owned block of the global pattern) and the status
    word reduced with MAX over the ranks.
    """

    def __init__(self, X, conn, ids, ndof, Ap, Ai, backend, group=None):
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        # NCCL moves device buffers, gloo host buffers
        self.dev = (torch.device("cuda", torch.cuda.current_device())
                    if dist.get_backend(group) == "nccl" else torch.device("cpu"))
        nparts = dist.get_world_size(group)
        rank = dist.get_rank(group)
        self.plan = RankPlan(X, conn, ids, ndof, Ap, Ai, nparts, rank)
        self.backend = backend
        # exchange the receive positions once: every rank tells every peer the
        # owned-block positions of what it will send
        sendpos = [self.plan.send_positions(q) if q != rank else (np.zeros(0, np.int64),) * 2
                   for q in range(nparts)]
        allpos = [None] * nparts
        dist.all_gather_object(allpos, sendpos, group=group)
        self.recv = {q: allpos[q][rank] for q in range(nparts)
                     if q != rank and (allpos[q][rank][0].size or allpos[q][rank][1].size)}

    @property
    def owned_rows(self):
        return self.plan.row0, self.plan.row1

    def gather_ghosts(self, u_owned):
        """The displacement of every row each piece touches, from this rank's
        owned values and the owners' (reverse exchange)."""
        import torch
        p = self.plan
        dist = self.dist
        nparts, rank = p.nparts, p.rank
        need = {}
        for ip, pc in enumerate(p.pieces):
            o = p.owner(pc.gdof)
            for q in range(nparts):
                if q != rank:
                    m = np.nonzero(o == q)[0]
                    if m.size:
                        need.setdefault(q, []).append((ip, m, pc.gdof[m]))
        req = [None] * nparts
        req[rank] = {q: np.concatenate([g for _, _, g in v]) for q, v in need.items()}
        allreq = [None] * nparts
        dist.all_gather_object(allreq, req[rank], group=self.group)
        ops, bufs = [], {}
        u_owned = np.asarray(u_owned, dtype=np.float64)
        for q in range(nparts):
            if q == rank:
                continue
            want = allreq[q].get(rank)
            if want is not None and want.size:
                t = torch.from_numpy(np.ascontiguousarray(u_owned[want - p.row0])).to(self.dev)
                ops.append(dist.P2POp(dist.isend, t, q, group=self.group))
            if q in need:
                bufs[q] = torch.zeros(sum(len(m) for _, m, _ in need[q]), dtype=torch.float64, device=self.dev)
                ops.append(dist.P2POp(dist.irecv, bufs[q], q, group=self.group))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        out = []
        for ip, pc in enumerate(p.pieces):
            ul = np.zeros(pc.ndof)
            mine = p.owner(pc.gdof) == rank
            ul[mine] = u_owned[pc.gdof[mine] - p.row0]
            out.append(ul)
        for q, lst in need.items():
            v = bufs[q].cpu().numpy()
            o = 0
            for ip, m, _ in lst:
                out[ip][m] = v[o:o + len(m)]
                o += len(m)
        return out

    def assemble_RK(self, u_pieces, u_presc=None):
        """u_pieces: the local displacement of each piece (gather_ghosts).
        Boundary piece, then the exchange posted, interior piece, own entries,
        then the received partial rows."""
        import torch
        p = self.plan
        dist = self.dist
        R = np.zeros(p.row1 - p.row0)
        K = np.zeros(p.k1 - p.k0)
        status = np.zeros(4, dtype=np.int64)
        results = [None] * len(p.pieces)
        ops, keep = [], []
        recvbufs = {}
        for q, (rpos, kpos) in self.recv.items():
            recvbufs[q] = torch.zeros(len(rpos) + len(kpos), dtype=torch.float64, device=self.dev)
            ops.append(dist.P2POp(dist.irecv, recvbufs[q], q, group=self.group))
        works = []
        for ip, pc in enumerate(p.pieces):
            Rl, Kl, st = self.backend(pc, u_pieces[ip], u_presc)
            results[ip] = (np.asarray(Rl), np.asarray(Kl))
            status = np.maximum(status, np.asarray(st, dtype=np.int64))
            if ip == 0:  # after the first piece (the boundary piece when there is one)
                for q, (rq, kq) in p.send.items():
                    b = torch.from_numpy(np.ascontiguousarray(np.concatenate([results[0][0][rq],
                                                                              results[0][1][kq]]))).to(self.dev)
                    keep.append(b)
                    ops.append(dist.P2POp(dist.isend, b, q, group=self.group))
                if ops:
                    works = dist.batch_isend_irecv(ops)
        for ip, rl, ro, kl, ko in p.own:
            Rl, Kl = results[ip]
            np.add.at(R, ro, Rl[rl])
            np.add.at(K, ko, Kl[kl])
        for w in works:
            w.wait()
        for q, (rpos, kpos) in self.recv.items():
            v = recvbufs[q].cpu().numpy()
            np.add.at(R, rpos, v[:len(rpos)])
            np.add.at(K, kpos, v[len(rpos):])
        st = torch.from_numpy(status.copy()).to(self.dev)
        dist.all_reduce(st, op=dist.ReduceOp.MAX, group=self.group)
        return R, K, st.cpu().numpy()


class DeviceBackend:
    """Piece assembly on this library's device contexts: one context per
    piece (created at its first call), the piece's element state taken from the
    global per-point state array, R and K of the piece from
    pgfem_gpu_assemble_RK."""

    def __init__(self, mat, state=None, nint=1, npres=0, dt=0.0, R_cp=None):
        self.mat, self.state, self.nint, self.npres, self.dt, self.R_cp = mat, state, nint, npres, dt, R_cp
        self.ctx = {}

    def context(self, pc):
        c = self.ctx.get(id(pc))
        if c is None:
            Rcp = None if self.R_cp is None else self.R_cp[pc.elems]
            c = pg.Context(pc.X, pc.conn, pc.ids, pc.ndof, pc.Ap, pc.Ai, self.mat, npres=self.npres, R_cp=Rcp)
            if self.state is not None:
                rows = (pc.elems[:, None] * self.nint + np.arange(self.nint)).ravel()
                c.set_state(self.state[rows])
            self.ctx[id(pc)] = c
        return c

    def __call__(self, pc, u_local, u_presc):
        R, K, st = self.context(pc).assemble_RK(u_local, u_presc, dt=self.dt)
        return R, K, np.array([st.inverted, st.nonconverged, st.bad_diagonal, st.other], dtype=np.int64)

    def close(self):
        for c in self.ctx.values():
            c.close()
        self.ctx = {}
