"""One 1-D transform spread over the ranks of a process group (one process
per GPU): the four-step decomposition with its transposes as all-to-all
exchanges, for lengths beyond one device's memory.

The reference has no distributed transform; its single-process four-step
(internal/kernels/sixstep.go:29-178) sets the index maps used here.  With
N = N1 * N2, n = N2*n1 + n2 and k = k1 + N1*k2:

    X[k1 + N1 k2] = sum_n2 W_N^(n2 k1) [sum_n1 x[N2 n1 + n2] W_N1^(n1 k1)] W_N2^(n2 k2)

Rank r of P holds the contiguous slab x[r N/P, (r+1) N/P), i.e. rows
n1 in [r N1/P, (r+1) N1/P) of x viewed as N1 x N2.  Forward:
  1. exchange: rank r receives columns n2 in [r N2/P, (r+1) N2/P) of every
     row; N2/P transforms of length N1 (over n1);
  2. times W_N^(n2 k1) (the rank's own n2, every k1; FP64 table rounded to
     the element type, built at plan creation);
  3. exchange: rank r receives rows k1 in [r N1/P, (r+1) N1/P) for every
     n2; N1/P transforms of length N2 (over n2);
  4. exchange back to natural order: the owner of X[k] (k // (N/P)) depends
     on k2 only, so rank r receives k2 in [r N2/P, (r+1) N2/P) for every k1
     and holds X[r N/P, (r+1) N/P) again.  With natural_order=False the
     output stays after step 3: rank r holds X[k1 + N1 k2] for its k1 rows,
     row-major (k1 local, k2), and Inverse takes that layout as its input.
The inverse runs the same steps with the inverse local transforms (each
scaled by 1/N1 and 1/N2, so 1/N in all) and the conjugate twiddle.

Every exchange moves N/P elements per rank (all but 1/P of them across
ranks); the local transforms are batched device transforms of the library.
Requires N1 and N2 divisible by P.  Every rank calls Forward/Inverse in the
same order (each call makes the same collectives on every rank).
"""
from __future__ import annotations

import math


def _split(n: int, world: int) -> tuple[int, int]:
    """N1 x N2 with both divisible by `world` and N1 <= N2 as close to
    sqrt(N) as the divisors allow; raises ValueError if none exists."""
    best = None
    for n1 in range(1, math.isqrt(n) + 1):
        if n % n1 == 0 and n1 % world == 0 and (n // n1) % world == 0:
            best = n1
    if best is None:
        raise ValueError(f"length {n} has no split N1 x N2 with both factors divisible by {world} ranks")
    return best, n // best


class PlanDistributed:
    """A length-n complex transform over the ranks of `group` (default: the
    world group).  Each rank passes its slab of n / world elements as a 1-D
    tensor on its device.  `local_fft(x, inverse)` computes the transforms of
    the rows of a contiguous (count, length) tensor, scaling the inverse by
    1/length; by default it runs the library's batched plans on the tensor's
    device."""

    def __init__(self, n: int, precision=None, group=None, local_fft=None, device=None):
        import torch
        import torch.distributed as dist
        from .plan import COMPLEX64, COMPLEX128
        if precision is None:
            precision = COMPLEX64
        if precision not in (COMPLEX64, COMPLEX128):
            raise ValueError("precision must be COMPLEX64 or COMPLEX128")
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.n = int(n)
        self.n1, self.n2 = _split(self.n, self.world)
        self.dtype = torch.complex64 if precision == COMPLEX64 else torch.complex128
        self.precision = precision
        self.device = torch.device(device) if device is not None else torch.device("cpu")
        self._plans = {}
        self._local_fft = local_fft or self._device_fft
        # W_N^(n2 k1) for this rank's columns n2 and every k1, (N2/P, N1),
        # from the exact integer product reduced mod N, evaluated in FP64
        p2 = self.n2 // self.world
        n2 = torch.arange(self.rank * p2, (self.rank + 1) * p2, dtype=torch.int64)
        k1 = torch.arange(self.n1, dtype=torch.int64)
        m = (n2[:, None] * k1[None, :]) % self.n
        ang = m.to(torch.float64) * (-2.0 * math.pi / self.n)
        self.twiddle = torch.polar(torch.ones_like(ang), ang).to(self.dtype).to(self.device)

    def _tw(self, device, inverse: bool):
        """The twiddle table on the slabs' device (moved there once)."""
        if self.twiddle.device != device:
            self.twiddle = self.twiddle.to(device)
        return self.twiddle.conj() if inverse else self.twiddle

    # -- local pieces --------------------------------------------------------

    def _device_fft(self, x, inverse: bool):
        """The library's batched transform of the rows of x, by a plan on x's
        own device (one plan per (length, device))."""
        from .plan import Plan, PlanOptions
        import torch
        if not x.is_cuda:
            raise ValueError("the default local transform needs slabs on a CUDA device")
        count, length = x.shape
        dev = x.device.index if x.device.index is not None else torch.cuda.current_device()
        key = (length, dev)
        if key not in self._plans:
            self._plans[key] = Plan(length, self.precision, PlanOptions(Device=dev))
        out = torch.empty_like(x)
        p = self._plans[key]
        (p.InverseBatch if inverse else p.ForwardBatch)(out, x, count)
        return out

    def _exchange(self, blocks):
        """blocks: (P, a, b) contiguous, block q for rank q; returns (P, a, b)
        with block q received from rank q."""
        import torch
        import torch.distributed as dist
        blocks = blocks.contiguous()
        out = torch.empty_like(blocks)
        dist.all_to_all_single(torch.view_as_real(out).reshape(-1), torch.view_as_real(blocks).reshape(-1),
                               group=self.group)
        return out

    # -- transforms ----------------------------------------------------------

    def _check(self, x):
        if x.numel() != self.n // self.world:
            raise ValueError(f"rank slab must hold {self.n // self.world} elements, got {x.numel()}")
        if x.dtype != self.dtype:
            raise TypeError(f"slab dtype {x.dtype} does not match the plan's {self.dtype}")

    def _natural(self, x, inverse: bool, natural_out: bool):
        """Steps 1-4 from this rank's natural slab."""
        P, N1, N2 = self.world, self.n1, self.n2
        r1, r2 = N1 // P, N2 // P
        tw = self._tw(x.device, inverse)
        # rows n1 of this rank (r1 x N2) -> columns n2 of this rank (N1 x r2)
        a = x.reshape(r1, P, r2).permute(1, 0, 2)
        cols = self._exchange(a).reshape(N1, r2)
        y = self._local_fft(cols.t().contiguous(), inverse)                # (r2 n2, N1 k1): over n1
        y = y * tw                                                         # W_N^(n2 k1)
        # -> rows k1 of this rank for every n2: (N2, r1)
        b = y.reshape(r2, P, r1).permute(1, 0, 2)
        rows = self._exchange(b).reshape(N2, r1)
        z = self._local_fft(rows.t().contiguous(), inverse)                # (r1 k1, N2 k2)
        if not natural_out:
            return z.reshape(-1)
        c = z.reshape(r1, P, r2).permute(1, 0, 2)                          # block q: k2 of rank q
        back = self._exchange(c).reshape(N1, r2)                           # (k1 all, k2 local)
        return back.t().contiguous().reshape(-1)                           # k = k1 + N1 k2

    def _transposed_inverse(self, z):
        """Inverse from the forward's step-3 layout (rows k1 of this rank, all
        k2): x[N2 n1 + n2] = (1/N) sum_k1 W_N1^(-n1 k1) W_N^(-n2 k1)
        sum_k2 X[k1 + N1 k2] W_N2^(-n2 k2), ending in natural order."""
        P, N1, N2 = self.world, self.n1, self.n2
        r1, r2 = N1 // P, N2 // P
        inverse = True
        tw = self._tw(z.device, True)
        # transforms over k2 of the rank's k1 rows
        y = self._local_fft(z.contiguous(), inverse)                           # (r1 k1, N2 n2)
        b = y.reshape(r1, P, r2).permute(1, 0, 2)                              # block q: n2 of rank q
        cols = self._exchange(b).reshape(N1, r2).t().contiguous()              # (r2 n2, N1 k1)
        cols = cols * tw
        u = self._local_fft(cols, inverse)                                     # (r2 n2, N1 n1)
        a = u.reshape(r2, P, r1).permute(1, 0, 2)                              # block q: n1 of rank q
        rows = self._exchange(a).reshape(N2, r1)                               # (n2 all, n1 local)
        return rows.t().contiguous().reshape(-1)                               # n = N2 n1 + n2

    def Forward(self, x, natural_order: bool = True):
        """The rank's slab of the transform of the distributed vector whose
        slab x this rank holds (natural_order=False: the layout after step 3,
        one exchange fewer)."""
        self._check(x)
        return self._natural(x, False, natural_order)

    def Inverse(self, x, natural_order: bool = True):
        """Inverse (scaled by 1/n), ending in natural order.
        natural_order=False: x is in the layout Forward(natural_order=False)
        returns, which saves one exchange."""
        self._check(x)
        if natural_order:
            return self._natural(x, True, True)
        return self._transposed_inverse(x.reshape(self.n1 // self.world, self.n2))

    def Len(self) -> int:
        return self.n

    def Close(self):
        for p in self._plans.values():
            p.Close()
        self._plans.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.Close()
