"""One box over several GPUs: the slab decomposition of the reference's FFTW-MPI plans.

The reference splits physical space in x planes (``local_n0``) and spectral space in
ky rows (``local_n1``) and transposes between them inside every 3-D transform
(``fftw_mpi_local_size_3d_transposed`` and the TRANSPOSED_OUT/IN plans,
src/FFTW_package.cpp:47-56, src/FFTW_package.h:60-64).  Here each rank (one
process per GPU) holds the ky rows ``[y0, y0+ny)`` of the compact state, runs the
x passes and the spectral sweep on them, and between the inverse and the forward
y pass holds the x planes ``[x0, x0+nx)`` (y and z passes).  One step is

    phase A (x inverse, pack) -> all-to-all -> [sum of the forced shells' energy]
    phase B (y inverse, z pass, y forward, pack) -> all-to-all -> [max of the CFL words]
    phase C (x forward, sweep, time step)

with both splits FFTW-MPI's default block (``ceil(n/ranks)`` per rank).  The
kernels and the pack/unpack reorders live in libspns (``spns_slab_*``); this
module moves the staging arrays between ranks and reduces the scalars:

* ``TorchTransport``: one rank per process over ``torch.distributed`` (NCCL on
  GPUs, ordered on each rank's CUDA stream; gloo on CPU tensors);
* ``LocalTransport``: several ranks driven by one process on one device, the
  all-to-all as device-to-device copies (no kernel waits on another).

``SlabHIT`` gives the group of ranks a process drives the ``HIT`` stepping
interface.  Its arithmetic is the advective form (or LES) of the one-GPU solver,
so a box stepped on slabs equals the same box stepped on one GPU to rounding.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np

from .hit import SPNS_FP64, SpnsError, _dp, lib, make_args_c
from .params import HitArgs

PH_VEL_A, PH_VEL_B, PH_DT, PH_A, PH_B, PH_C = range(6)


def block(n: int, nranks: int, rank: int):
    """(start, count) of rank's block when n items are split over nranks (ceil(n/nranks) per rank)."""
    blk = -(-n // nranks)
    s = min(n, rank * blk)
    return s, min(n, s + blk) - s


def exchange_counts(Ky: int, Mx: int, Kz: int, nranks: int, rank: int, nf: int, back: bool):
    """Complex values sent to / received from every rank (the counts of spns_slab_counts)."""
    L = lib()
    send = (C.c_longlong * nranks)()
    recv = (C.c_longlong * nranks)()
    st = L.spns_slab_counts(Ky, Mx, Kz, nranks, rank, nf, int(back), send, recv)
    if st != 0:
        raise SpnsError(st, "spns_slab_counts")
    return list(send), list(recv)


class _DeviceArray:
    """Device memory of libspns as a CUDA array (read by torch.as_tensor)."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3}


class SlabRank:
    """One rank's libspns slab handle."""

    def __init__(self, args: HitArgs, nranks: int, rank: int, *, precision: int = SPNS_FP64, device: int = 0,
                 fixed_dt: float = 0.0, eps_forcing: float = 0.0, eps_kmin: int = 1, eps_kmax: int = 2):
        L = lib()
        a = make_args_c(args, precision=precision, device=device, fixed_dt=fixed_dt, eps_forcing=eps_forcing,
                        eps_kmin=eps_kmin, eps_kmax=eps_kmax, nonlinear_form=2)
        h = C.c_void_p()
        st = L.spns_slab_create(C.byref(a), int(nranks), int(rank), C.byref(h))
        if st != 0:
            raise SpnsError(st, L.spns_last_error(None).decode())
        self._L, self._h = L, h
        self.args, self.nranks, self.rank, self.device, self.precision = args, nranks, rank, device, precision
        y0, ny, x0, nx = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        self._ck(L.spns_slab_layout(h, C.byref(y0), C.byref(ny), C.byref(x0), C.byref(nx)))
        self.y0, self.ny, self.x0, self.nx = y0.value, ny.value, x0.value, nx.value
        kx, ky, kz = C.c_int(), C.c_int(), C.c_int()
        L.spns_spectral_dims(h, C.byref(kx), C.byref(ky), C.byref(kz))
        self.local_shape = (3, ky.value, kx.value, kz.value)
        send, recv, scal = C.c_void_p(), C.c_void_p(), C.c_void_p()
        elems = C.c_size_t()
        off = (C.c_size_t * 3)()
        self._ck(L.spns_slab_buffers(h, C.byref(send), C.byref(recv), C.byref(elems), C.byref(scal), off))
        self.send_ptr, self.recv_ptr, self.elems = send.value, recv.value, int(elems.value)
        self.scalars_ptr, self.off_max, self.off_nonfinite, self.off_ef = scal.value, off[0], off[1], off[2]
        p = C.c_void_p()
        self._ck(L.spns_stream(h, C.byref(p)))
        self.stream_ptr = p.value or 0

    def _ck(self, st):
        if st != 0:
            raise SpnsError(st, self._L.spns_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._L.spns_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def phase(self, p: int):
        self._ck(self._L.spns_slab_phase(self._h, int(p)))

    def counts(self, p: int):
        send = (C.c_longlong * self.nranks)()
        recv = (C.c_longlong * self.nranks)()
        self._ck(self._L.spns_slab_exchange(self._h, int(p), send, recv))
        return list(send), list(recv)

    def set_rows(self, U_rows):
        buf = np.ascontiguousarray(U_rows, dtype=np.complex128)
        if buf.shape != self.local_shape:
            raise SpnsError(-1, f"slab state shape {buf.shape} != {self.local_shape}")
        self._ck(self._L.spns_set_spectral(self._h, _dp(buf.view(np.float64))))

    def get_rows(self) -> np.ndarray:
        out = np.zeros(self.local_shape, dtype=np.complex128)
        self._ck(self._L.spns_get_spectral(self._h, _dp(out.view(np.float64))))
        return out

    def energy_cascade_rows(self) -> np.ndarray:
        """E(K) of this rank's rows (the shell sums of src/HIT_LES.cpp:1137-1214 over its modes)."""
        s = self.scalars()
        ek = np.zeros(int(s.last_rad_max) + 1)
        tot = C.c_double()
        self._ck(self._L.spns_recalculate_energy_cascade(self._h, _dp(ek), C.byref(tot)))
        return ek

    def scalars(self):
        from .hit import ScalarsC
        s = ScalarsC()
        self._ck(self._L.spns_get_scalars(self._h, C.byref(s)))
        return s

    # device views for a transport
    def tensors(self):
        import torch
        word = np.dtype(np.float64 if self.precision == SPNS_FP64 else np.float32)
        ts = "<f8" if word.itemsize == 8 else "<f4"
        dev = torch.device("cuda", self.device)
        send = torch.as_tensor(_DeviceArray(self.send_ptr, 2 * self.elems, ts), device=dev)
        recv = torch.as_tensor(_DeviceArray(self.recv_ptr, 2 * self.elems, ts), device=dev)
        mx = torch.as_tensor(_DeviceArray(self.scalars_ptr + self.off_max, 4, "<i8"), device=dev)
        nf = torch.as_tensor(_DeviceArray(self.scalars_ptr + self.off_nonfinite, 1, "<i4"), device=dev)
        ef = torch.as_tensor(_DeviceArray(self.scalars_ptr + self.off_ef, 1, "<f8"), device=dev)
        return send, recv, mx, nf, ef


class LocalTransport:
    """All ranks in this process on one device: the all-to-all as device-to-device copies."""

    def exchange(self, ranks: Sequence[SlabRank], p: int):
        import torch
        torch.cuda.synchronize()
        views = [r.tensors() for r in ranks]
        counts = [r.counts(p) for r in ranks]
        for r, rr in enumerate(ranks):
            send_off = np.concatenate([[0], np.cumsum(counts[r][0])])
            for s, rs in enumerate(ranks):
                recv_off = np.concatenate([[0], np.cumsum(counts[s][1])])
                n = counts[r][0][s]
                assert n == counts[s][1][r]
                dst = views[s][1][2 * recv_off[r]:2 * (recv_off[r] + n)]
                dst.copy_(views[r][0][2 * send_off[s]:2 * (send_off[s] + n)])
        torch.cuda.synchronize()

    def reduce(self, ranks: Sequence[SlabRank], what: str):
        import torch
        torch.cuda.synchronize()
        views = [r.tensors() for r in ranks]
        if what == "ef":
            tot = views[0][4].clone()
            for v in views[1:]:
                tot += v[4]
            for v in views:
                v[4].copy_(tot)
        else:
            mx = views[0][2].clone()
            nf = views[0][3].clone()
            for v in views[1:]:
                mx = torch.maximum(mx, v[2])
                nf = torch.maximum(nf, v[3])
            for v in views:
                v[2].copy_(mx)
                v[3].copy_(nf)
        torch.cuda.synchronize()


class TorchTransport:
    """One rank per process over torch.distributed, ordered on the rank's CUDA stream."""

    def __init__(self, group=None):
        self.group = group

    def _stream(self, rank: SlabRank):
        import torch
        return torch.cuda.stream(torch.cuda.ExternalStream(rank.stream_ptr, device=torch.device("cuda", rank.device)))

    def exchange(self, ranks: Sequence[SlabRank], p: int):
        import torch.distributed as dist
        (r,) = ranks
        send_c, recv_c = r.counts(p)
        send, recv, *_ = r.tensors()
        with self._stream(r):
            dist.all_to_all_single(recv[:2 * sum(recv_c)], send[:2 * sum(send_c)], [2 * c for c in recv_c],
                                   [2 * c for c in send_c], group=self.group)

    def reduce(self, ranks: Sequence[SlabRank], what: str):
        import torch.distributed as dist
        (r,) = ranks
        _, _, mx, nf, ef = r.tensors()
        with self._stream(r):
            if what == "ef":
                dist.all_reduce(ef, op=dist.ReduceOp.SUM, group=self.group)
            else:
                dist.all_reduce(mx, op=dist.ReduceOp.MAX, group=self.group)
                dist.all_reduce(nf, op=dist.ReduceOp.MAX, group=self.group)


class SlabHIT:
    """The ranks one process drives (all of them with LocalTransport, its own with
    TorchTransport), stepped together with the HIT interface of the one-GPU solver."""

    def __init__(self, args: HitArgs, nranks: int, transport, ranks: Optional[List[int]] = None, **options):
        self.args, self.nranks, self.transport = args, nranks, transport
        self.eps = options.get("eps_forcing", 0.0) > 0.0
        self.ranks = [SlabRank(args, nranks, r, **options) for r in (ranks if ranks is not None else range(nranks))]

    def close(self):
        for r in self.ranks:
            r.close()

    def _all(self, p: int):
        for r in self.ranks:
            r.phase(p)

    def set_compact(self, U):
        """The whole box's compact state [3][Ky][Kx][Kz]; each rank takes its rows."""
        for r in self.ranks:
            r.set_rows(U[:, r.y0:r.y0 + r.ny])

    def get_compact(self) -> np.ndarray:
        """The rows of the ranks this process drives, in order (the whole box with LocalTransport)."""
        return np.concatenate([r.get_rows() for r in self.ranks], axis=1)

    def Recalculate_Velocity_Antitransform(self):
        self._all(PH_VEL_A)
        self.transport.exchange(self.ranks, PH_VEL_A)
        self._all(PH_VEL_B)
        self.transport.reduce(self.ranks, "max")

    def Recalculate_TimeStep(self):
        self._all(PH_DT)

    def New_Fractional_Step_Method(self, nsteps: int = 1):
        for _ in range(nsteps):
            self._all(PH_A)
            self.transport.exchange(self.ranks, PH_A)
            if self.eps:
                self.transport.reduce(self.ranks, "ef")
            self._all(PH_B)
            self.transport.exchange(self.ranks, PH_B)
            self.transport.reduce(self.ranks, "max")
            self._all(PH_C)

    def Recalculate_Energy_Cascade_rows(self) -> np.ndarray:
        """E(K) summed over the ranks this process drives."""
        return sum(r.energy_cascade_rows() for r in self.ranks)

    def gettime(self) -> float:
        return self.ranks[0].scalars().time

    def getAt(self) -> float:
        return self.ranks[0].scalars().At
