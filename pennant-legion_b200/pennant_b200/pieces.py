"""Multi-piece runs: one piece of a mesh per rank of a torch.distributed
group (the reference's numpcs decomposition, Mesh.cc:211-241, with its halo
sums of corner force and mass, Hydro.cc:571-574 and 766-769, and its dt
reductions, Hydro.cc:961-970).

The library does every piece's arithmetic (pnt_hydro_piece_forces /
advance / finish, include/pennant_b200.h); this module moves, every cycle,

* the corner mass and force of the sides at shared points to the
  neighbours that hold those points (one message pair per neighbour), into
  their halo slots, and
* the four per-piece scalars {dtnew, -dvovmax, inverted sides in pass A,
  in pass C}: minimum of the first two, sum of the last two.

With the NCCL backend the transfers run on device buffers, ordered on the
hydro object's own stream (no host round trip); with gloo they are staged
through host memory (CPU-only groups, or several ranks sharing one GPU).
Every piece ends each cycle with exactly the single-piece values of its
zones and points.
"""
from __future__ import annotations

import ctypes as C

import torch
import torch.distributed as dist

from . import Hydro, Mesh, PieceBuffers, check, lib

_TAG_CMASS, _TAG_CFORCE = 11, 12


class _DeviceBytes:
    """A byte range of library device memory, for a zero-copy torch view."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (int(nbytes),), "typestr": "|u1",
                                         "data": (int(ptr), False), "version": 3, "strides": None}


def device_bytes(ptr: int, nbytes: int, device: torch.device) -> torch.Tensor:
    if nbytes == 0:
        return torch.empty(0, dtype=torch.uint8, device=device)
    return torch.as_tensor(_DeviceBytes(ptr, nbytes), device=device)


class HaloExchange:
    """The per-cycle halo exchange of one piece, given its exchange lists
    (Mesh.piece_info) and the byte layout of its buffers: `send` holds the
    corner masses of the send lists, then their corner forces from byte
    `foff`; `halo_m` / `halo_f` are the halo slots' corner masses / forces.
    Works on CPU or CUDA byte tensors; CUDA tensors on a gloo group go
    through host copies."""

    def __init__(self, info: dict, cmass_bytes: int, cforce_bytes: int, foff: int, group=None):
        # pieces are numbered by rank within the group; point-to-point
        # operations address global ranks
        self.nbr = [int(q) if group is None else dist.get_global_rank(group, int(q)) for q in info["nbr"]]
        self.send_off = [int(v) for v in info["send_off"]]
        self.recv_off = [int(v) for v in info["recv_off"]]
        self.cmb, self.cfb, self.foff = cmass_bytes, cforce_bytes, foff
        self.group = group

    def _ranges(self, j: int):
        a, b = self.send_off[j], self.send_off[j + 1]
        ra, rb = self.recv_off[j], self.recv_off[j + 1]
        return ((a * self.cmb, b * self.cmb), (self.foff + a * self.cfb, self.foff + b * self.cfb),
                (ra * self.cmb, rb * self.cmb), (ra * self.cfb, rb * self.cfb))

    def exchange(self, send: torch.Tensor, halo_m: torch.Tensor, halo_f: torch.Tensor) -> None:
        backend = dist.get_backend(self.group)
        staged = send.is_cuda and backend != "nccl"
        if staged:
            send_x, halo_m_x, halo_f_x = send.cpu(), torch.empty(halo_m.shape, dtype=torch.uint8), \
                torch.empty(halo_f.shape, dtype=torch.uint8)
        else:
            send_x, halo_m_x, halo_f_x = send, halo_m, halo_f
        if backend == "nccl":
            ops = []
            for j, q in enumerate(self.nbr):
                (sm0, sm1), (sf0, sf1), (rm0, rm1), (rf0, rf1) = self._ranges(j)
                ops += [dist.P2POp(dist.isend, send_x[sm0:sm1], q, self.group),
                        dist.P2POp(dist.isend, send_x[sf0:sf1], q, self.group),
                        dist.P2POp(dist.irecv, halo_m_x[rm0:rm1], q, self.group),
                        dist.P2POp(dist.irecv, halo_f_x[rf0:rf1], q, self.group)]
            reqs = dist.batch_isend_irecv(ops) if ops else []
        else:
            reqs = []
            for j, q in enumerate(self.nbr):
                (sm0, sm1), (sf0, sf1), (rm0, rm1), (rf0, rf1) = self._ranges(j)
                reqs += [dist.isend(send_x[sm0:sm1].contiguous(), q, self.group, tag=_TAG_CMASS),
                         dist.isend(send_x[sf0:sf1].contiguous(), q, self.group, tag=_TAG_CFORCE)]
                reqs += [dist.irecv(halo_m_x[rm0:rm1], q, self.group, tag=_TAG_CMASS),
                         dist.irecv(halo_f_x[rf0:rf1], q, self.group, tag=_TAG_CFORCE)]
        for r in reqs:
            r.wait()
        if staged:
            halo_m.copy_(halo_m_x, non_blocking=False)
            halo_f.copy_(halo_f_x, non_blocking=False)


def reduce_scalars(red: torch.Tensor, group=None) -> None:
    """red = [dtnew, -dvovmax, badA, badC] of this piece -> over all pieces:
    minimum of the first two, sum of the last two (exact in any order)."""
    staged = red.is_cuda and dist.get_backend(group) != "nccl"
    x = red.cpu() if staged else red
    lo, hi = x[0:2].clone(), x[2:4].clone()
    dist.all_reduce(lo, op=dist.ReduceOp.MIN, group=group)
    dist.all_reduce(hi, op=dist.ReduceOp.SUM, group=group)
    x[0:2] = lo
    x[2:4] = hi
    if staged:
        red.copy_(x)


class PieceHydro:
    """This rank's piece of `mesh` (rank r of the group's size), stepped in
    lockstep with the other ranks' pieces.  fields() gives the piece's
    zone fields (global zones zone0 ..) and point fields (global points
    gpoint)."""

    def __init__(self, mesh: Mesh, params, group=None, device: int = 0, closure=None, closure_mode: int = 0):
        self.group = group
        size, rank = dist.get_world_size(group), dist.get_rank(group)
        self.mesh = mesh.piece(size, rank)
        self.info = self.mesh.piece_info()
        self.hydro = Hydro(self.mesh, params, device)
        if closure is not None:
            self.hydro.set_closure(closure, closure_mode)
        b = PieceBuffers()
        check(lib.pnt_hydro_piece_buffers(self.hydro.h, C.byref(b)))
        self.device = torch.device("cuda", device)
        self.stream = torch.cuda.ExternalStream(b.stream, device=self.device)
        nsend, nhalo = int(self.info["send_off"][-1]), int(self.info["nhalo"])
        self.send = device_bytes(b.send, b.send_cforce_offset + nsend * b.cforce_bytes, self.device)
        self.halo_m = device_bytes(b.halo_cmass, nhalo * b.cmass_bytes, self.device)
        self.halo_f = device_bytes(b.halo_cforce, nhalo * b.cforce_bytes, self.device)
        self.red = device_bytes(b.red, 32, self.device).view(torch.float64)
        self.halo = HaloExchange(self.info, b.cmass_bytes, b.cforce_bytes, b.send_cforce_offset, group)

    def cycle(self) -> None:
        """One cycle of every piece (all ranks call it together)."""
        with torch.cuda.stream(self.stream):
            self._cycle_ops()

    def _cycle_ops(self) -> None:
        h = self.hydro.h
        nccl = dist.get_backend(self.group) == "nccl"
        check(lib.pnt_hydro_piece_forces(h))
        if not nccl:
            self.stream.synchronize()
        self.halo.exchange(self.send, self.halo_m, self.halo_f)
        check(lib.pnt_hydro_piece_advance(h))
        if not nccl:
            self.stream.synchronize()
        reduce_scalars(self.red, self.group)
        check(lib.pnt_hydro_piece_finish(h))

    def capture(self, ncycles: int) -> None:
        """Records `ncycles` whole cycles -- the library's kernels, the NCCL
        halo sends and receives and both reductions -- in one CUDA graph on
        the piece's stream (NCCL groups only; every rank captures the same
        count).  replay() then runs them with one launch from the host, the
        analogue of the reference's traced cycle loop (Driver.cc:113-145).
        close() releases the graph, which must happen before the process
        group is destroyed."""
        if dist.get_backend(self.group) != "nccl":
            raise RuntimeError("graph capture needs the NCCL backend (gloo transfers go through the host)")
        self.release_graph()
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=self.stream, capture_error_mode="thread_local"):
            for _ in range(ncycles):
                self._cycle_ops()
        self.graph, self.graph_cycles = g, ncycles

    def replay(self) -> None:
        """One launch of the captured cycles on the piece's stream."""
        with torch.cuda.stream(self.stream):
            self.graph.replay()

    def release_graph(self) -> None:
        if getattr(self, "graph", None) is not None:
            torch.cuda.synchronize(self.device)
            self.graph.reset()
            self.graph = None

    def run(self, max_cycles: int = 0, check_every: int = 16) -> dict:
        """Cycles until the run is done (or max_cycles); identical on every
        rank, since every piece ends each cycle from the same reduced
        scalars."""
        n = 0
        while True:
            for _ in range(check_every):
                self.cycle()
                n += 1
                if max_cycles and n >= max_cycles:
                    break
            s = self.hydro.scalars()
            if s["done"] or (max_cycles and n >= max_cycles):
                return s

    def scalars(self) -> dict:
        return self.hydro.scalars()

    def fields(self, names=("px", "pu", "zr", "ze", "zetot", "zvol", "zwrate")) -> dict:
        return {k: self.hydro.download(k) for k in names}

    def close(self) -> None:
        self.release_graph()
        self.hydro.close()
