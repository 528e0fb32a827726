"""One 2D domain cut into x-slabs, one slab per GPU.

nest splits a domain into patches with subspace() (include/nest/core.hpp:
183-199: the first `total % parts` pieces get one extra cell) and fills each
patch's halo from its neighbours' edge cells before every RK stage
(execute_all_exchanges, include/nest/patch.hpp:153-190, called from
examples/sod2d/sod2d.cpp:331-362).  Here a patch is a whole x-slab (rows
x0 .. x0+n of the global domain, all columns) on one device:

* the two ghost rows on each cut side come from the neighbour slab's edge
  rows, moved by NCCL send/recv (torch.distributed) -- two swaps per step,
  one before each stage; columns (y ghosts) stay with the slab's own kernel;
* the CFL step needs the global maxima of |u|+c and |v|+c: the two words of
  each slab's speed slot (bit patterns of non-negative doubles, which order
  like the doubles) are max-all-reduced before stage 1, so every slab derives
  the same dt, and a sharded run equals the one-domain run bit for bit.

The slab objects only need: ``speed_words()`` (int64 tensor of 2, in place),
``edges(buf)`` (send/receive row views of the state, buf 0, or the stage
buffer, buf 1), ``stage(which, cfl, t_final)`` and ``stream()`` (a context
for the copies and collectives, ordered with the slab's kernels).  GPUSlab
is the device implementation; a process may also hold several slabs of one
domain (copies between them replace the messages), which is how one device
runs a multi-slab domain.
"""
from __future__ import annotations

import contextlib
from dataclasses import dataclass

import numpy as np

from . import _capi as A


def slab_range(total: int, parts: int, part: int) -> tuple[int, int]:
    """(offset, length) of piece `part` of `parts`: subspace(), include/nest/core.hpp:183-199."""
    base, extra = divmod(total, parts)
    return part * base + min(part, extra), base + (1 if part < extra else 0)


@dataclass
class Edges:
    """Row views (nvars, 2, row length) of one buffer of a slab."""
    send_lo: object   # first two interior rows
    send_hi: object   # last two interior rows
    recv_lo: object   # ghost rows -2, -1
    recv_hi: object   # ghost rows n, n+1


class _DevArray:
    """Zero-copy device view handed to torch.as_tensor."""

    def __init__(self, ptr: int, shape, strides, typestr: str):
        self.__cuda_array_interface__ = {"data": (ptr, False), "shape": tuple(shape),
                                         "strides": tuple(strides), "typestr": typestr, "version": 3}


class GPUSlab:
    """One slab held by a Solver on the current device."""

    def __init__(self, nx_local: int, ny: int, dx: float, dy: float, bc: int, precision: int,
                 xlo_exchange: bool, xhi_exchange: bool, gamma: float = 1.4, flags: int = 0, stream=None):
        import torch
        from .solver import Solver
        if nx_local < 2:
            raise ValueError("every slab needs at least two rows (the stencil's halo)")
        self.torch = torch
        self.stream_obj = stream if stream is not None else torch.cuda.Stream()
        self.solver = Solver(2, nx_local, ny, dx=dx, dy=dy, gamma=gamma, bc=bc, precision=precision,
                             flags=flags, stream=self.stream_obj.cuda_stream)
        if xlo_exchange or xhi_exchange:
            self.solver.set_exchange_sides(xlo_exchange, xhi_exchange)
        self.n = nx_local
        _, self.pitch, self.vstride = self.solver.state_ptr()
        self.esize = 8 if precision == A.F64 else 4
        self._edges, self._speed = {}, {}

    def stream(self):
        return self.torch.cuda.stream(self.stream_obj)

    def _rows(self, base: int, first: int):
        es = self.esize
        arr = _DevArray(base + (first + 2) * self.pitch * es, (4, 2, self.pitch),
                        (self.vstride * es, self.pitch * es, es), "<f8" if es == 8 else "<f4")
        return self.torch.as_tensor(arr, device="cuda")

    def edges(self, buf: int) -> Edges:
        if buf not in self._edges:
            base = self.solver.state_ptr()[0] if buf == 0 else self.solver.stage_ptr()
            self._edges[buf] = Edges(self._rows(base, 0), self._rows(base, self.n - 2),
                                     self._rows(base, -2), self._rows(base, self.n))
        return self._edges[buf]

    def speed_words(self):
        ptr = self.solver.speed_slot_ptr()   # alternates between the two step slots
        t = self._speed.get(ptr)
        if t is None:
            t = self._speed[ptr] = self.torch.as_tensor(_DevArray(ptr, (2,), (8,), "<i8"), device="cuda")
        return t

    def stage(self, which: int, cfl: float, t_final: float):
        self.solver.stage(which, cfl, t_final)


class SlabDomain:
    """Steps one domain held as x-slabs by one or several processes.

    slabs: the slab objects this process holds; ids: their slab indices;
    nslabs: slabs in the domain; periodic: x wraps around; group: a
    torch.distributed group when other processes hold slabs (slab k lives on
    rank owner[k]), else None.
    """

    TAG_UP, TAG_DOWN = 0, 1   # hi rows travel to the hi neighbour, lo rows to the lo one

    def __init__(self, slabs, ids, nslabs: int, periodic: bool, group=None, owner=None):
        self.slabs, self.ids, self.nslabs, self.periodic = list(slabs), list(ids), nslabs, periodic
        self.group = group
        self.local = {k: s for k, s in zip(self.ids, self.slabs)}
        self.owner = owner if owner is not None else list(range(nslabs))
        self._bufs = {}

    def peers(self, k: int):
        lo, hi = k - 1, k + 1
        if self.periodic:
            lo, hi = lo % self.nslabs, hi % self.nslabs
        return (lo if lo >= 0 else None), (hi if hi < self.nslabs else None)

    def _ctx(self):
        return self.slabs[0].stream() if self.slabs else contextlib.nullcontext()

    def reduce_speeds(self):
        """Max of every slab's two speed words, written back to each."""
        import torch
        words = [s.speed_words() for s in self.slabs]
        m = words[0].clone()
        for w in words[1:]:
            torch.maximum(m, w, out=m)
        if self.group is not None:
            import torch.distributed as dist
            dist.all_reduce(m, op=dist.ReduceOp.MAX, group=self.group)
        for w in words:
            w.copy_(m)

    def _buf(self, key, like):
        import torch
        b = self._bufs.get(key)
        if b is None or b.shape != like.shape or b.dtype != like.dtype or b.device != like.device:
            b = torch.empty(like.shape, dtype=like.dtype, device=like.device)
            self._bufs[key] = b
        return b

    def exchange(self, buf: int):
        """Fill the cut sides' ghost rows of buffer `buf` (0 state, 1 stage)."""
        if self.nslabs == 1:
            return
        ops, unpack = [], []
        for s, k in zip(self.slabs, self.ids):
            e = s.edges(buf)
            lo, hi = self.peers(k)
            # posting order per slab: up-send, down-send, receive-from-lo, receive-from-hi;
            # with two slabs both neighbours are the same rank and messages match in this order
            sends, recvs = [], []
            if hi is not None and hi not in self.local:
                sb = self._buf((k, buf, "su"), e.send_hi)
                sb.copy_(e.send_hi)
                sends.append((sb, hi, self.TAG_UP))
            if lo is not None and lo not in self.local:
                sb = self._buf((k, buf, "sd"), e.send_lo)
                sb.copy_(e.send_lo)
                sends.append((sb, lo, self.TAG_DOWN))
            if lo is not None:
                if lo in self.local:
                    e.recv_lo.copy_(self.local[lo].edges(buf).send_hi)
                else:
                    rb = self._buf((k, buf, "rl"), e.recv_lo)
                    recvs.append((rb, lo, self.TAG_UP))
                    unpack.append((e.recv_lo, rb))
            if hi is not None:
                if hi in self.local:
                    e.recv_hi.copy_(self.local[hi].edges(buf).send_lo)
                else:
                    rb = self._buf((k, buf, "rh"), e.recv_hi)
                    recvs.append((rb, hi, self.TAG_DOWN))
                    unpack.append((e.recv_hi, rb))
            ops.extend(("send",) + x for x in sends)
            ops.extend(("recv",) + x for x in recvs)
        if ops:
            import torch.distributed as dist
            p2p = [dist.P2POp(dist.isend if kind == "send" else dist.irecv, t, self.owner[peer],
                              group=self.group, tag=tag) for kind, t, peer, tag in ops]
            for r in dist.batch_isend_irecv(p2p):
                r.wait()
        for dst, src in unpack:
            dst.copy_(src)

    def step(self, nsteps: int, cfl: float, t_final: float = 0.0):
        """nsteps RK2 steps of every slab (steps at or past t_final are no-ops)."""
        with self._ctx():
            for _ in range(nsteps):
                self.reduce_speeds()
                self.exchange(0)
                for s in self.slabs:
                    s.stage(1, cfl, t_final)
                self.exchange(1)
                for s in self.slabs:
                    s.stage(2, cfl, t_final)


def native_peers(k: int, nslabs: int, periodic: bool) -> tuple[int, int]:
    """Neighbour ranks (lo, hi) of slab k for the native driver, -1 at a
    domain boundary; a periodic one-slab domain is its own neighbour."""
    if periodic:
        return (k - 1) % nslabs, (k + 1) % nslabs
    return (k - 1 if k > 0 else -1), (k + 1 if k < nslabs - 1 else -1)


class NativeSlabDomain:
    """This rank's x-slab stepped by the C++ driver (nest_slab_step): the
    speed all-reduce and the ghost-row exchanges go through NCCL on the
    solver's stream and runs of 16 steps replay from CUDA graphs, so no
    Python runs per step.  Same interface as SlabDomain for one slab."""

    def __init__(self, slab: GPUSlab, k: int, nslabs: int, periodic: bool, group=None):
        import ctypes as C
        import torch
        from ._capi import check, lib
        A.bind({
            "nest_slab_comm_id": (C.c_int, [C.c_char_p]),
            "nest_slab_comm_create": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
            "nest_slab_comm_destroy": (C.c_int, [C.c_void_p]),
            "nest_slab_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double]),
        })
        self.slabs, self.ids, self.nslabs = [slab], [k], nslabs
        idbuf = C.create_string_buffer(128)
        if group is None or k == 0:
            check(lib.nest_slab_comm_id(idbuf), "nest_slab_comm_id")
        if group is not None:
            import torch.distributed as dist
            obj = [bytes(idbuf.raw)]
            dist.broadcast_object_list(obj, src=dist.get_global_rank(group, 0) if group is not dist.group.WORLD else 0,
                                       group=group)
            idbuf = C.create_string_buffer(obj[0], 128)
        h = C.c_void_p()
        torch.cuda.synchronize()
        check(lib.nest_slab_comm_create(idbuf, nslabs, k, C.byref(h)), "nest_slab_comm_create")
        self._comm = h
        self.lo, self.hi = native_peers(k, nslabs, periodic)
        self._lib, self._check = lib, check

    def step(self, nsteps: int, cfl: float, t_final: float = 0.0):
        self._check(self._lib.nest_slab_step(self.slabs[0].solver._h, self._comm, self.lo, self.hi, nsteps, cfl,
                                             t_final), "nest_slab_step")

    def close(self):
        """Release the solvers' graphs, then the communicator."""
        if getattr(self, "_comm", None):
            for s in self.slabs:
                s.solver.close()
            self._lib.nest_slab_comm_destroy(self._comm)
            self._comm = None


def gpu_domain(nx: int, ny: int, *, bc: int = A.BC_PERIODIC, precision: int = A.F64, gamma: float = 1.4,
               flags: int = 0, group=None, local_slabs: int = 1, native: bool = False, nslabs: int | None = None):
    """Slabs of an nx x ny domain on [0,1]^2 for this process.

    With a torch.distributed group of W ranks, rank r holds slab r of W
    (one per device, the caller sets the current device); without one the
    process holds `local_slabs` slabs on the current device, sharing one
    stream.  native=True: this process's single slab is stepped by the C++
    NCCL driver (NativeSlabDomain); without a group that is a one-rank
    domain whose periodic neighbour is itself.  Returns (domain,
    [(x0, n) per held slab])."""
    import torch
    if group is not None:
        import torch.distributed as dist
        W, r = dist.get_world_size(group), dist.get_rank(group)
        ids = [r]
        owner = [dist.get_global_rank(group, k) for k in range(W)] if group is not dist.group.WORLD else None
    else:
        W, ids, owner = local_slabs, list(range(local_slabs)), None
    periodic = bc == A.BC_PERIODIC
    stream = torch.cuda.Stream()
    slabs, ranges = [], []
    for k in ids:
        x0, n = slab_range(nx, W, k)
        if native:  # exchange sides are the sides with a neighbour rank
            lo, hi = native_peers(k, W, periodic)
            lo_ex, hi_ex = lo >= 0, hi >= 0
        else:
            lo_ex = W > 1 and (periodic or k > 0)
            hi_ex = W > 1 and (periodic or k < W - 1)
        slabs.append(GPUSlab(n, ny, 1.0 / nx, 1.0 / ny, bc, precision, lo_ex, hi_ex, gamma, flags, stream))
        ranges.append((x0, n))
    if native:
        if len(slabs) != 1:
            raise ValueError("the native driver steps one slab per process")
        return NativeSlabDomain(slabs[0], ids[0], W, periodic, group), ranges
    return SlabDomain(slabs, ids, W, periodic, group, owner), ranges


def slab_rows(U_global: np.ndarray, x0: int, n: int) -> np.ndarray:
    """Rows of slab (x0, n) of an extended global array [nv][nx+4][ny+4], ghosts included."""
    return np.ascontiguousarray(U_global[:, x0:x0 + n + 4, :])
