"""Regular force and potential of one cluster split over ranks.

This is the multi-rank form of the regular block in the reference's parallel
build (``intgrt.F:942-1100``).  Every rank holds the whole predicted state and
sends the whole j set to its own GPU (``intgrt.F:875-882``); the active list
is cut into contiguous pieces, one per rank (``intgrt.F:955-968``); each rank
evaluates its piece (``CALC_REG_ON_GPU(IREG,istart,iend)``, ``intgrt.F:992``);
then the per-particle results travel to every rank (the ``MPI_SENDRECV`` ring
of ``intgrt.F:1046-1095``), so that each rank ends the block with the results
of the whole active list.

Here the exchange is one all-gather per result kind over ``torch.distributed``
(NCCL between GPUs, gloo between host processes): the FP64 rows
(acc, jrk, pot) and the neighbour-list rows (``lmax`` ints each).  The pieces
are padded to the largest piece so that every rank contributes the same
number of rows.  Every rank takes the same collective steps in the same
order, including ranks whose piece is empty; a block with no active
particles takes none on any rank, since the active count is the same
everywhere.

The force itself goes through :class:`nb6b200.abi.ForceLib` (``gpunb_regf_``
of ``libnb6b200.so``) in calls of at most 1024 particles, the reference's
per-call limit (``util_gpu.F:7``).  Results are those of a single-rank call
over the whole list, row for row: each particle's force is computed
independently of how the list is cut.

The potential follows the reference's parallel ENERGY (``energy_mpi.F``):
a set of more than 5e4 bodies is cut the same way (``energy_mpi.F:59-77``),
each rank evaluates the potential of its own range against all bodies
(``GPUPOT(rank,istart,NN,...)``, ``energy_mpi.F:101``), and the potentials
travel to every rank (``energy_mpi.F:179-181``); a smaller set is evaluated
whole on every rank (``energy_mpi.F:216``).

The irregular force follows the parallel irregular step
(``intgrt.F:600-720``): every rank keeps the whole irregular state
(``IRR_SIMD_SET_JP`` / ``SET_LIST`` for all bodies), the block's active list
is cut the same way, each rank evaluates its piece
(``IRR_SIMD_FIRR_VEC(TIME,NPART_LEN,NXTLST_MPI(istart_lst),...)``,
``intgrt.F:648``), and the rows travel to every rank (``intgrt.F:690-720``).
"""
from __future__ import annotations

import numpy as np

NIMAX = 1024  # particles per gpunb_regf_ call (util_gpu.F:7)
NREC = 7      # FP64 values per result row: acc[3], jrk[3], pot
POT_SPLIT_MIN = 50000  # bodies above which the potential is split (energy_mpi.F:60)


def _device_view(ptr: int, shape, typestr: str, device):
    """A torch tensor over device memory the library owns (no copy)."""
    import torch

    class _Buf:
        __cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (ptr, False),
                                    "version": 3, "strides": None}
    return torch.as_tensor(_Buf(), device=device)


def active_split(nl: int, size: int) -> tuple[list[int], list[int]]:
    """Contiguous pieces of an active list of ``nl`` particles over ``size``
    ranks, as ``intgrt.F:955-968`` cuts it: each rank gets ``nl // size``
    and the first ``nl % size`` ranks one more.  Returns (start, count) per
    rank, starts 0-based (the Fortran ``ista`` minus one)."""
    if size < 1 or nl < 0:
        raise ValueError(f"active_split: nl={nl}, size={size}")
    inl, idiff = divmod(nl, size)
    start, count, run = [], [], 0
    for r in range(size):
        n = inl + (1 if r < idiff else 0)
        start.append(run)
        count.append(n)
        run += n
    return start, count


class RankSplit:
    """Regular force (``regf``), potential (``gpupot``) and irregular force
    (``firr``) of one cluster over the ranks of a process group, each split
    into one piece of its particle list per rank.

    ``lib`` is this rank's :class:`ForceLib`, already opened on this rank's
    GPU (``gpunb_open``; ``irr_open`` with every body's state set, for
    ``firr``).  ``group`` is a ``torch.distributed`` process group (None: the
    default group; no initialised group: one rank, no exchange).  ``chunk``
    is the largest ``gpunb_regf_`` call.
    """

    def __init__(self, lib, group=None, chunk: int = NIMAX):
        if not 1 <= chunk <= NIMAX:
            raise ValueError(f"chunk={chunk} outside [1, {NIMAX}]")
        self.lib = lib
        self.chunk = chunk
        self.group = group
        self.rank, self.size = 0, 1
        self.dist = None
        try:
            import torch.distributed as dist
            if dist.is_available() and dist.is_initialized():
                self.dist = dist
                self.rank = dist.get_rank(group)
                self.size = dist.get_world_size(group)
        except ImportError:
            pass
        self.device = None
        if self.dist is not None:
            import torch
            if self.dist.get_backend(group) == "nccl":
                # NCCL buffers live on the GPU the library opened on
                # (gpunb_open_ picks irank modulo the visible devices).
                dev = -1
                query = getattr(getattr(lib, "lib", None), "nb6_device_", None)
                if query is not None:
                    dev = int(query())
                if dev < 0:
                    dev = torch.cuda.current_device()
                torch.cuda.set_device(dev)
                self.device = torch.device("cuda", dev)
            else:
                self.device = torch.device("cpu")

    def send(self, m, x, v) -> None:
        """Every rank sends the whole predicted j set to its own GPU
        (``intgrt.F:882``); list ids are then the same on every rank."""
        self.lib.gpunb_send(m, x, v)

    def piece(self, nl: int) -> tuple[int, int]:
        """(start, count) of this rank's piece of an ``nl``-particle list."""
        start, count = active_split(nl, self.size)
        return start[self.rank], count[self.rank]

    def _own(self, h2, dtr, xi, vi, lmax, nnbmax, m_flag, s, n):
        rec = np.zeros((n, NREC))
        lst = np.zeros((n, lmax), dtype=np.int32)
        for a in range(0, n, self.chunk):
            b = min(n, a + self.chunk)
            acc, jrk, pot, l = self.lib.gpunb_regf(h2[s + a:s + b], dtr[s + a:s + b], xi[s + a:s + b],
                                                   vi[s + a:s + b], lmax, nnbmax, m_flag)
            rec[a:b, 0:3] = acc
            rec[a:b, 3:6] = jrk
            rec[a:b, 6] = pot
            lst[a:b] = l
        return rec, lst

    def _gather(self, rows: np.ndarray, width: int, counts: list[int]) -> np.ndarray:
        """All-gather of each rank's first ``counts[rank]`` rows, padded to
        ``counts[0]`` (the largest piece); returns the rows in rank order."""
        import torch
        pad = counts[0]
        buf = np.zeros((pad, width), dtype=rows.dtype)
        buf[:rows.shape[0]] = rows
        src = torch.from_numpy(buf).to(self.device)
        out = torch.empty((self.size * pad, width), dtype=src.dtype, device=self.device)
        self.dist.all_gather_into_tensor(out, src, group=self.group)
        full = out.cpu().numpy().reshape(self.size, pad, width)
        return np.concatenate([full[r, :counts[r]] for r in range(self.size)], axis=0)

    def regf(self, h2, dtr, xi, vi, lmax: int, nnbmax: int, m_flag: int = 0):
        """Regular force of the whole active list (``gpunb_regf_`` semantics:
        acc, jrk, pot exclude neighbours; list rows ``[nnb, ids...]`` or
        ``-nnb`` on overflow).  Every rank passes the same list and gets every
        particle's results back; it evaluates only its own piece."""
        h2 = np.ascontiguousarray(h2, dtype=np.float64)
        nl = h2.shape[0]
        dtr = np.ascontiguousarray(dtr, dtype=np.float64).reshape(nl)
        xi = np.ascontiguousarray(xi, dtype=np.float64).reshape(nl, 3)
        vi = np.ascontiguousarray(vi, dtype=np.float64).reshape(nl, 3)
        start, count = active_split(nl, self.size)
        s, n = start[self.rank], count[self.rank]
        rec, lst = self._own(h2, dtr, xi, vi, lmax, nnbmax, m_flag, s, n)
        if self.dist is not None and self.size > 1 and nl > 0:
            rec = self._gather(rec, NREC, count)
            lst = self._gather(lst, lmax, count)
        return rec[:, 0:3].copy(), rec[:, 3:6].copy(), rec[:, 6].copy(), lst

    # ------------------------------------------------ device-resident form
    def _own_device(self, d_h2, d_dtr, d_xi, d_vi, lmax, nnbmax, m_flag, s, n, pad):
        """This rank's piece [s, s + n) of device-resident i data through
        nb6_regf_device_ in calls of at most ``chunk``, each call's output
        rows copied on the library's stream into (pad, 7) FP64 and (pad, W)
        int32 device tensors (rows past n stay zero)."""
        import ctypes as C
        import torch
        raw = self.lib.lib
        W = max(0, min(nnbmax, lmax - 1)) + 1
        dev = self.device
        rec = torch.zeros((pad, NREC), dtype=torch.float64, device=dev)
        lst = torch.zeros((pad, W), dtype=torch.int32, device=dev)
        stream = torch.cuda.ExternalStream(raw.nb6_stream_(), device=dev)
        ci = C.c_int
        po, pl = C.POINTER(C.c_double)(), C.POINTER(C.c_int)()
        with torch.cuda.stream(stream):
            for a in range(0, n, self.chunk):
                b = min(n, a + self.chunk)
                k = s + a
                raw.nb6_regf_device_(C.byref(ci(b - a)), C.c_void_p(d_h2.data_ptr() + 8 * k),
                                     C.c_void_p(d_dtr.data_ptr() + 8 * k),
                                     C.c_void_p(d_xi.data_ptr() + 24 * k),
                                     C.c_void_p(d_vi.data_ptr() + 24 * k),
                                     C.byref(ci(lmax)), C.byref(ci(nnbmax)), C.byref(ci(m_flag)))
                raw.nb6_regf_outputs_(C.byref(po), C.byref(pl))
                outf = _device_view(C.cast(po, C.c_void_p).value, (b - a, 8), "<f8", dev)
                outl = _device_view(C.cast(pl, C.c_void_p).value, (b - a, W), "<i4", dev)
                rec[a:b].copy_(outf[:, :NREC])
                lst[a:b].copy_(outl)
        return rec, lst, stream

    def regf_device(self, d_h2, d_dtr, d_xi, d_vi, lmax: int, nnbmax: int, m_flag: int = 0):
        """``regf`` with the i data and the results on the device: d_h2,
        d_dtr (nl,), d_xi, d_vi (nl, 3) FP64 CUDA tensors on this rank's
        GPU, the same on every rank.  Returns (rec, lst): (nl, 7) FP64 rows
        (acc, jrk, pot) and (nl, W) int32 list rows (W = min(nnbmax,
        lmax-1) + 1) of the whole list, on the device: each rank's rows go
        from the library's output buffers into the all-gather's send buffer
        and come back from NCCL without touching the host."""
        import contextlib
        import torch
        nl = int(d_h2.shape[0])
        start, count = active_split(nl, self.size)
        s, n = start[self.rank], count[self.rank]
        pad = count[0] if nl else 0
        rec, lst, stream = self._own_device(d_h2, d_dtr, d_xi, d_vi, lmax, nnbmax, m_flag, s, n, pad)
        if self.dist is not None and self.size > 1 and nl > 0:
            # the collective follows the library's work in stream order
            with torch.cuda.stream(stream) if stream is not None else contextlib.nullcontext():
                rec = self._gather_device(rec, count)
                lst = self._gather_device(lst, count)
        else:
            rec, lst = rec[:n], lst[:n]
        if stream is not None:
            torch.cuda.current_stream(self.device).wait_stream(stream)
        return rec, lst

    def _gather_device(self, rows, counts: list[int]):
        """All-gather of every rank's (counts[0], width) padded tensor on
        its device; the first counts[r] rows of rank r, in rank order."""
        import torch
        pad = rows.shape[0]
        out = torch.empty((self.size * pad,) + tuple(rows.shape[1:]), dtype=rows.dtype, device=rows.device)
        self.dist.all_gather_into_tensor(out, rows.contiguous(), group=self.group)
        out = out.view(self.size, pad, *rows.shape[1:])
        return torch.cat([out[r, :counts[r]] for r in range(self.size)], dim=0)

    def gpupot(self, m, x, split_min: int = POT_SPLIT_MIN) -> np.ndarray:
        """Potential of every body against all bodies (``gpupot_``
        semantics: positive, self excluded).  Every rank passes the whole set
        and gets every body's potential back; above ``split_min`` bodies each
        rank evaluates only its own range."""
        m = np.ascontiguousarray(m, dtype=np.float64)
        n = m.shape[0]
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(n, 3)
        if self.dist is None or self.size == 1 or n <= split_min:
            return self.lib.gpupot(m, x, 1, n, self.rank) if n else np.zeros(0)
        start, count = active_split(n, self.size)
        s, c = start[self.rank], count[self.rank]
        own = self.lib.gpupot(m, x, s + 1, c, self.rank) if c else np.zeros(0)
        return self._gather(own.reshape(c, 1), 1, count).reshape(n)

    def firr(self, ti: float, addr):
        """Irregular force of the whole active list ``addr`` (1-based
        addresses, ``irr_simd_firr_vec_`` semantics): acc, jrk over each
        body's neighbour list and ``nnbid``, the 1-based nearest neighbour.
        Every rank passes the same list and gets every body's results back;
        it evaluates only its own piece."""
        addr = np.ascontiguousarray(addr, dtype=np.int32)
        nl = addr.shape[0]
        start, count = active_split(nl, self.size)
        s, c = start[self.rank], count[self.rank]
        rec = np.zeros((c, NREC))
        if c:
            acc, jrk, nnbid = self.lib.irr_firr_vec(ti, addr[s:s + c])
            rec[:, 0:3] = acc
            rec[:, 3:6] = jrk
            rec[:, 6] = nnbid  # int32 ids are exact in FP64
        if self.dist is not None and self.size > 1 and nl > 0:
            rec = self._gather(rec, NREC, count)
        return rec[:, 0:3].copy(), rec[:, 3:6].copy(), rec[:, 6].astype(np.int32)
