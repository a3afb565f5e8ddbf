"""One mesh over several GPUs: an element partition, the nodes on the cuts
shared by the parts, and every step the sum of their residual between the
element loop and the nodal update -- the reference's rhsmod ->
pararr('SLX') exchange of interface nodes (sld_matrix.f90:274-281) -- with
their lumped mass summed once at set-up.

The parts run in this process (``PartitionedSolid(prob, nparts)``: every
part on ``device``, or one device each) or one per rank under
torch.distributed (``PartitionedSolid(prob, group=...)``).  Each part's
elements are ordered interface first (the elements touching a shared node);
under torch.distributed a step runs the interface elements, gathers the
shared rows, and sends each neighbouring part the rows of the nodes the two
share (NCCL send/recv on a communication stream, the reference's
PAR_INTERFACE_NODE_EXCHANGE with MPI_Isend/Irecv) while the interior
elements compute; the received rows are added and written back before the
nodal update.  Steps use the context's sma_step_prologue /
sma_step_elements(_range) / sma_step_nodes, the same kernels as
sma_explicit_step without its graphs."""
import ctypes as C

import numpy as np

from . import problem as P


def partition_elements(prob, nparts):
    """Element ids of each part (sorted): the elements ordered by centroid
    along the mesh's longest extent, cut into nparts runs of equal count."""
    if nparts < 1 or nparts > prob.nelem:
        raise ValueError(f"nparts must be in [1, {prob.nelem}]")
    cent = prob.coord[prob.lnods].mean(axis=1)
    ax = int(np.argmax(prob.coord.max(axis=0) - prob.coord.min(axis=0)))
    order = np.argsort(cent[:, ax], kind="stable")
    cuts = [prob.nelem * k // nparts for k in range(nparts + 1)]
    return [np.sort(order[cuts[k]:cuts[k + 1]]) for k in range(nparts)]


def sub_problem(prob, elems, load_owner):
    """The part of ``prob`` made of ``elems``: its nodes renumbered in
    increasing global order (returned as the second value).  Nodal loads
    stay only where ``load_owner[node]`` is true, so a shared node's load is
    applied by one part."""
    nodes = np.unique(prob.lnods[elems])
    remap = -np.ones(prob.npoin, np.int64)
    remap[nodes] = np.arange(nodes.size)
    fext = None
    if prob.fext is not None:
        fext = prob.fext[nodes] * load_owner[nodes][:, None]
    q = P.Problem(coord=prob.coord[nodes], lnods=remap[prob.lnods[elems]].astype(np.int32),
                  props=prob.props, e_mart=prob.e_mart, densi=prob.densi,
                  fixno=prob.fixno[nodes], bcfun=prob.bcfun[nodes], fun_npts=prob.fun_npts,
                  fun_smooth=prob.fun_smooth, fun_tab=prob.fun_tab,
                  lmate=None if prob.lmate is None else prob.lmate[elems],
                  tempe=None if prob.tempe is None else prob.tempe[elems],
                  fext=fext, dampi=prob.dampi, load_fun=prob.load_fun, dtime=prob.dtime,
                  nsteps=prob.nsteps, name=f"{prob.name}[part]")
    return q, nodes


def layout(prob, parts):
    """The partition's bookkeeping: per part its global node ids, and for the
    nodes shared by several parts their slot in 0..nshared-1 and, per part,
    the local indices of its shared nodes with their slots."""
    node_sets = [np.unique(prob.lnods[e]) for e in parts]
    count = np.zeros(prob.npoin, np.int32)
    for g in node_sets:
        count[g] += 1
    shared = np.nonzero(count > 1)[0]
    slot = -np.ones(prob.npoin, np.int64)
    slot[shared] = np.arange(shared.size)
    owner = -np.ones(prob.npoin, np.int64)                # lowest part holding the node
    for k in range(len(parts) - 1, -1, -1):
        owner[node_sets[k]] = k
    local = []
    for g in node_sets:
        loc = np.nonzero(count[g] > 1)[0]
        local.append((loc.astype(np.int32), slot[g[loc]]))
    return node_sets, shared, owner, local


def interface_first(prob, elems, shared_mask):
    """The part's elements with those touching a shared node first (both
    runs in increasing global order), and the number of interface ones."""
    touch = shared_mask[prob.lnods[elems]].any(axis=1)
    return np.concatenate([elems[touch], elems[~touch]]), int(touch.sum())


def neighbour_plan(node_sets, local):
    """Per part k: [(j, positions)] for every other part j sharing nodes with
    k, positions indexing k's shared rows (ordered by global node id, as
    ``layout`` lists them) of the nodes k and j share, in increasing global
    id -- the same nodes in the same order on both sides."""
    plans = []
    for k, g in enumerate(node_sets):
        loc, _ = local[k]
        gk = g[loc]                                      # global ids of k's shared nodes, increasing
        plan = []
        for j, h in enumerate(node_sets):
            if j == k:
                continue
            pos = np.nonzero(np.isin(gk, h, assume_unique=True))[0]
            if pos.size:
                plan.append((j, pos.astype(np.int64)))
        plans.append(plan)
    return plans


def exchange_neighbours(rows, plan, group=None):
    """The shared rows (n, 3) of this rank summed with its neighbours': the
    rows of the nodes shared with each neighbour go to it and its rows of
    the same nodes come back (point-to-point, all posted before any wait),
    then are added.  NCCL for CUDA tensors; with gloo (host tensors only for
    point-to-point) CUDA rows are staged through host memory."""
    import torch
    import torch.distributed as dist
    if not plan:
        return rows.clone()
    host = rows.is_cuda and dist.get_backend(group) != "nccl"
    src = rows.cpu() if host else rows
    ops, bufs = [], []
    for j, pos in plan:
        pt = torch.as_tensor(pos, device=src.device)
        send = src.index_select(0, pt).contiguous()
        recv = torch.empty_like(send)
        peer = dist.get_global_rank(group, j) if group is not None else j
        ops += [dist.P2POp(dist.isend, send, peer, group), dist.P2POp(dist.irecv, recv, peer, group)]
        bufs.append((pt, recv, send))
    for r in dist.batch_isend_irecv(ops):
        r.wait()
    out = src.clone()
    for pt, recv, _ in bufs:
        out.index_add_(0, pt, recv)
    return out.to(rows.device) if host else out


def reduce_shared(rows, slots, nshared, group=None):
    """Sum the rows (n, 3) a rank holds for shared nodes with every other
    rank's rows of the same nodes: each rank places its rows at their slots
    of a (nshared, 3) buffer, all-reduce SUM, and reads its slots back.
    Works for CUDA tensors (NCCL) and CPU tensors (gloo)."""
    import torch
    import torch.distributed as dist
    buf = torch.zeros((nshared, 3), dtype=rows.dtype, device=rows.device)
    buf.index_put_((slots,), rows, accumulate=True)
    dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    return buf.index_select(0, slots)


class PartitionedSolid:
    """A mesh split into parts, each an ExplicitSolid, advanced together.

    Local mode (``group`` None): all ``nparts`` parts live in this process,
    on ``device`` or on ``devices[k]``; the shared rows are summed on the
    first part's device.  Distributed mode (``group`` a torch.distributed
    process group, one part per rank): this rank builds part ``rank`` only.
    ``get`` returns the global field (local mode) or this part's rows with
    their global node ids (distributed mode)."""

    def __init__(self, prob, nparts=None, precision="fp64", scatter="atomic", device=0, devices=None,
                 group=None, block=0, scheme="cd", phitw=0.0):
        import torch
        from . import ExplicitSolid, _check, lib
        self._check, self._lib = _check, lib
        self.prob = prob
        self.group = group
        if group is not None:
            import torch.distributed as dist
            self.rank, nparts = dist.get_rank(group), dist.get_world_size(group)
        else:
            self.rank = None
            nparts = nparts or 1
        self.parts = partition_elements(prob, nparts)
        self.node_sets, self.shared, owner, self.local = layout(prob, self.parts)
        self.nshared = int(self.shared.size)
        shared_mask = np.zeros(prob.npoin, bool)
        shared_mask[self.shared] = True
        self.n_iface = {}
        for k in range(nparts):
            self.parts[k], self.n_iface[k] = interface_first(prob, self.parts[k], shared_mask)
        self.plan = neighbour_plan(self.node_sets, self.local)
        mine = range(nparts) if group is None else [self.rank]
        self.solids, self.idx, self.slots = {}, {}, {}
        self._comm = None
        for k in mine:
            dev = device if devices is None else devices[k]
            q, _ = sub_problem(prob, self.parts[k], owner == k)
            self.solids[k] = ExplicitSolid(q, precision=precision, scatter=scatter, device=dev,
                                           block=block, scheme=scheme, phitw=phitw)
            loc, sl = self.local[k]
            self.idx[k] = torch.as_tensor(loc, dtype=torch.int32, device=f"cuda:{dev}")
            self.slots[k] = torch.as_tensor(sl, dtype=torch.int64, device=f"cuda:{dev}")
        self._sum_mass()

    # -- shared nodes -------------------------------------------------------
    def _sum_mass(self):
        import torch
        if self.nshared == 0:
            return
        vms = {k: s.get("vmass") for k, s in self.solids.items()}
        if self.group is None:
            total = np.zeros(self.nshared)
            for k in self.solids:
                loc, sl = self.local[k]
                np.add.at(total, sl, vms[k][loc])
            for k in self.solids:
                loc, sl = self.local[k]
                vms[k][loc] = total[sl]
        else:
            k = self.rank
            loc, _ = self.local[k]
            rows = torch.zeros((loc.size, 3), dtype=torch.float64, device=self.idx[k].device)
            rows[:, 0] = torch.as_tensor(vms[k][loc], device=rows.device)
            vms[k][loc] = reduce_shared(rows, self.slots[k], self.nshared, self.group)[:, 0].cpu().numpy()
        for k, s in self.solids.items():
            s.set("vmass", vms[k])

    def _exchange(self):
        import torch
        if self.nshared == 0:
            return
        L = self._lib()
        if self.group is not None:
            k = self.rank
            s = self.solids[k]
            n = self.idx[k].numel()
            with torch.cuda.stream(torch.cuda.ExternalStream(s.stream)):   # ordered with the part's kernels
                rows = torch.empty((n, 3), dtype=torch.float64, device=self.idx[k].device)
                self._check(L.sma_gather_residual(s._ctx, n, self.idx[k].data_ptr(), rows.data_ptr()))
                back = exchange_neighbours(rows, self.plan[k], self.group).contiguous()
                self._check(L.sma_scatter_residual(s._ctx, n, self.idx[k].data_ptr(), back.data_ptr()))
                self._keep = back                     # alive until the stream has used it
            return
        # local parts: gather on each part's stream, sum on the first part's
        # device, scatter back (host-synchronised between the three stages)
        rows = {}
        for k, s in self.solids.items():
            n = self.idx[k].numel()
            rows[k] = torch.empty((n, 3), dtype=torch.float64, device=self.idx[k].device)
            self._check(L.sma_gather_residual(s._ctx, n, self.idx[k].data_ptr(), rows[k].data_ptr()))
        for s in self.solids.values():
            torch.cuda.ExternalStream(s.stream).synchronize()
        dev = self.idx[next(iter(self.solids))].device
        total = torch.zeros((self.nshared, 3), dtype=torch.float64, device=dev)
        for k in self.solids:
            total.index_add_(0, self.slots[k].to(dev), rows[k].to(dev))
        back = {k: total.index_select(0, self.slots[k].to(dev)).to(self.idx[k].device).contiguous()
                for k in self.solids}
        for k in self.solids:
            torch.cuda.synchronize(self.idx[k].device)
        for k, s in self.solids.items():
            self._check(L.sma_scatter_residual(s._ctx, self.idx[k].numel(), self.idx[k].data_ptr(),
                                               back[k].data_ptr()))
        for s in self.solids.values():
            torch.cuda.ExternalStream(s.stream).synchronize()

    # -- stepping -----------------------------------------------------------
    def _step_overlapped(self, nsteps):
        """Distributed steps: interface elements, shared rows gathered and
        exchanged with the neighbours on a communication stream while the
        interior elements compute, sums written back, nodal update."""
        import torch
        L = self._lib()
        k = self.rank
        s = self.solids[k]
        idx = self.idx[k]
        dev = idx.device
        n, ni, ne = idx.numel(), self.n_iface[k], s.nelem
        st = torch.cuda.ExternalStream(s.stream)
        if self._comm is None:
            self._comm = torch.cuda.Stream(device=dev)
        comm = self._comm
        self._check(L.sma_step_prologue(s._ctx))
        for step in range(nsteps):
            self._check(L.sma_step_elements_range(s._ctx, 0, ni, 1, 0))
            with torch.cuda.stream(st):
                rows = torch.empty((n, 3), dtype=torch.float64, device=dev)
            self._check(L.sma_gather_residual(s._ctx, n, idx.data_ptr(), rows.data_ptr()))
            ready = torch.cuda.Event()
            ready.record(st)
            comm.wait_event(ready)
            with torch.cuda.stream(comm):
                summed = exchange_neighbours(rows, [(j, pos) for j, pos in self.plan[k]], self.group)
            rows.record_stream(comm)
            self._check(L.sma_step_elements_range(s._ctx, ni, ne, 0, 1))     # interior, meanwhile
            done = torch.cuda.Event()
            done.record(comm)
            st.wait_event(done)
            summed.record_stream(st)
            self._check(L.sma_scatter_residual(s._ctx, n, idx.data_ptr(), summed.data_ptr()))
            self._check(L.sma_step_nodes(s._ctx, C.c_int32(int(step == nsteps - 1))))

    def step(self, nsteps):
        """nsteps explicit steps of the whole mesh (sma_explicit_step's
        sequence on every part, shared residual summed every step)."""
        if nsteps <= 0:
            return
        if self.group is not None and self.nshared > 0:
            return self._step_overlapped(nsteps)
        L = self._lib()
        for s in self.solids.values():
            self._check(L.sma_step_prologue(s._ctx))
        for n in range(nsteps):
            for s in self.solids.values():
                self._check(L.sma_step_elements(s._ctx))
            self._exchange()
            for s in self.solids.values():
                self._check(L.sma_step_nodes(s._ctx, C.c_int32(int(n == nsteps - 1))))

    def set(self, field, values):
        """Set a global nodal field (npoin, 3) on every part."""
        for k, s in self.solids.items():
            s.set(field, np.asarray(values)[self.node_sets[k]])

    def get(self, field):
        """The global field (npoin, ...) in local mode; in distributed mode
        this part's rows and their global node ids."""
        if self.group is not None:
            k = self.rank
            return self.solids[k].get(field), self.node_sets[k]
        out = None
        for k, s in self.solids.items():
            v = s.get(field)
            if out is None:
                out = np.zeros((self.prob.npoin,) + v.shape[1:], dtype=v.dtype)
            out[self.node_sets[k]] = v
        return out

    def counters(self):
        """Counters summed over this process's parts."""
        tot = {}
        for s in self.solids.values():
            for key, v in s.counters().items():
                if key in ("gpdet_min", "ielem_min"):
                    continue
                tot[key] = tot.get(key, 0) + v
        return tot

    def close(self):
        for s in self.solids.values():
            s.close()
