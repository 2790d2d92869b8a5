"""Row-sharded Gibbs chains: one chain over several ranks (one process per GPU).

Within a half-sweep of MacauX::run (macau.cpp:110-147) the rows of a mode are sampled
independently given the other mode's latents and the hyperparameters (the OpenMP row loop of
latentprior.cpp:69-77).  So each rank samples a contiguous range of the mode's rows, balanced by
entries, and after the half-sweep the ranks all-gather the new rows: every rank then holds the
whole latent matrix.  The hyperparameter updates need no collective: every rank computes them from
the same latents with the same kernels and the same keyed draws, so all ranks hold the same
values, and the N-rank chain is the 1-rank chain (draws are keyed by the global row index, and a
long row is split by the whole mode's threshold).  The only exchange per half-sweep is the
all-gather of the new latent block (N_mode x K values).

The driver runs over a backend with four operations (the CUDA library through its C ABI, or, in
tests, the CPU oracle), and a torch.distributed process group (NCCL on GPUs, gloo on CPUs):

    sample_rows(mode, it)     sample this rank's rows of `mode` with the draws of sweep `it`
    latent_view(mode)         torch tensor (N_mode x stride) holding the mode's latents
    latents_written(mode)     the view's rows were written by the gather
    update_prior(mode, it)    hyperparameter update of `mode` from the (whole) latents
"""
import numpy as np


def balanced_row_ranges(row_lengths, world):
    """Contiguous row ranges [lo, hi) for `world` ranks with about equal entries each: range r
    ends at the first row where the running entry count reaches (r + 1) / world of the total."""
    lengths = np.asarray(row_lengths, dtype=np.int64)
    n = len(lengths)
    if world < 1:
        raise ValueError("world must be >= 1")
    csum = np.concatenate([[0], np.cumsum(lengths)])
    total = csum[-1]
    cuts = [0]
    for r in range(1, world):
        target = total * r / world
        cut = int(np.searchsorted(csum, target, side="left"))
        cuts.append(min(max(cut, cuts[-1]), n))
    cuts.append(n)
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def gather_rows(dist, view, ranges, rank, group=None):
    """All-gather of row blocks in place: rank r contributes rows ranges[r] of `view` (a torch
    tensor of N x stride values on the process group's device), and afterwards every rank's
    `view` holds every block.  Blocks are padded to the longest so that the collective moves
    equal-sized pieces."""
    import torch
    width = max(hi - lo for lo, hi in ranges)
    lo, hi = ranges[rank]
    send = torch.zeros((width,) + tuple(view.shape[1:]), dtype=view.dtype, device=view.device)
    send[:hi - lo] = view[lo:hi]
    recv = [torch.empty_like(send) for _ in ranges]
    dist.all_gather(recv, send, group=group)
    for r, (a, b) in enumerate(ranges):
        if r != rank and b > a:
            view[a:b] = recv[r][:b - a]


class ShardedChain:
    """One Gibbs chain over the ranks of a process group: rows of each mode split by
    balanced_row_ranges, an all-gather after each half-sweep, local hyperparameter updates."""

    def __init__(self, backend, dist, rank, world, row_lengths, group=None):
        self.backend = backend
        self.dist = dist
        self.rank = rank
        self.world = world
        self.group = group
        self.ranges = [balanced_row_ranges(row_lengths[m], world) for m in (0, 1)]
        for m in (0, 1):
            backend.set_rows(m, *self.ranges[m][rank])

    def half_sweep(self, mode, it):
        self.backend.sample_rows(mode, it)
        if self.world > 1:
            with self.backend.collective_stream():
                gather_rows(self.dist, self.backend.latent_view(mode), self.ranges[mode],
                            self.rank, self.group)
            self.backend.latents_written(mode)

    def sweep(self, it):
        for mode in (0, 1):
            self.half_sweep(mode, it)
        for mode in (0, 1):
            self.backend.update_prior(mode, it)


class _CudaArray:
    """__cuda_array_interface__ over a device buffer the library owns (no copy)."""

    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr,
                                         "data": (ptr, False), "version": 3, "strides": None}


class LibraryBackend:
    """The CUDA library as a ShardedChain backend: a Sampler (macau_b200._lib) whose context
    samples this rank's row range; the latent views are torch tensors over the library's own
    device buffers, and collectives run on the library's stream."""

    def __init__(self, sampler, device):
        self.s = sampler
        self.device = device

    def set_rows(self, mode, lo, hi):
        self.s.set_row_range(mode, lo, hi)

    def sample_rows(self, mode, it):
        self.s.sample_latents(mode, it)

    def latent_view(self, mode):
        import torch
        ptr, stride, eb = self.s.latents_device(mode)
        n = self.s.dims[mode]
        arr = _CudaArray(ptr, (n, stride), "<f4" if eb == 4 else "<f8")
        return torch.as_tensor(arr, device=self.device)

    def latents_written(self, mode):
        self.s.latents_changed(mode)

    def collective_stream(self):
        import torch
        return torch.cuda.stream(torch.cuda.ExternalStream(self.s.stream(), device=self.device))

    def update_prior(self, mode, it):
        self.s.update_prior(mode, it)


class OracleBackend:
    """The CPU oracle (test infrastructure) as a ShardedChain backend, for checking the
    partition, the exchange and the local updates against a single oracle chain."""

    def __init__(self, model):
        self.m = model
        self.rows = [None, None]
        self._views = [None, None]

    def set_rows(self, mode, lo, hi):
        self.rows[mode] = (lo, hi)

    def sample_rows(self, mode, it):
        lo, hi = self.rows[mode]
        if self.m.sample_rows(mode, it, lo, hi) != 0:
            raise RuntimeError("oracle row sampler failed")

    def latent_view(self, mode):
        import torch
        self._views[mode] = torch.from_numpy(np.ascontiguousarray(self.m.latents(mode)))
        return self._views[mode]

    def latents_written(self, mode):
        self.m.set("latents", mode, self._views[mode].numpy())

    def collective_stream(self):
        import contextlib
        return contextlib.nullcontext()

    def update_prior(self, mode, it):
        if self.m.update_prior(mode, it) != 0:
            raise RuntimeError("oracle prior update failed")
