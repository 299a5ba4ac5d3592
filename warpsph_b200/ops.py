"""Torch-tensor wrappers of the C ABI (one function per entry point).

Every function takes CUDA float32 / int32 tensors, allocates its outputs with torch
on the same device, and enqueues the CUDA kernels on the current torch stream.
Errors from the library raise RuntimeError; there is no CPU path.
"""
from __future__ import annotations

import contextlib
import ctypes as C
from typing import Optional

import torch

from . import _capi
from ._capi import check, fptr, iptr, ptr, stream_ptr
from .core import AdjacencyList, CRKState, SupportScheme


class KernelTimer:
    """Records CUDA events around selected library calls on the launching stream.

    ``names`` is the set of wrapper names to time (None = all).  Durations are read
    with ``summary()`` after a synchronize."""

    def __init__(self, names=None):
        self.names = None if names is None else set(names)
        self.events = []

    def wants(self, name: str) -> bool:
        return self.names is None or name in self.names

    def summary(self) -> dict:
        out = {}
        for name, a, b in self.events:
            t = out.setdefault(name, [0, 0.0])
            t[0] += 1
            t[1] += a.elapsed_time(b)
        return {k: {"launches": v[0], "total_ms": v[1], "avg_ms": v[1] / max(v[0], 1)} for k, v in out.items()}


TIMER: Optional[KernelTimer] = None


class _timed:
    def __init__(self, name: str):
        self.name = name

    def __enter__(self):
        t = TIMER
        self.ev = None
        if t is not None and t.wants(self.name):
            self.ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            self.ev[0].record()
        return self

    def __exit__(self, *exc):
        if self.ev is not None:
            self.ev[1].record()
            TIMER.events.append((self.name, self.ev[0], self.ev[1]))
        return False


_SUPPORT = {SupportScheme.Gather: 0, SupportScheme.Scatter: 1, SupportScheme.Symmetric: 2,
            SupportScheme.SuperSymmetric: 3, SupportScheme.KernelMeanSymmetric: 4}


def _p(params) -> C.c_void_p:
    return C.cast(C.pointer(params), C.c_void_p)


def _f32(t: torch.Tensor) -> torch.Tensor:
    if not t.is_cuda:
        raise RuntimeError("warpsph_b200 operates on CUDA tensors only (no CPU fallback)")
    if t.dtype != torch.float32:
        raise RuntimeError(f"expected float32 tensor, got {t.dtype}")
    return t.contiguous()


def _empty(shape, like: torch.Tensor, dtype=torch.float32) -> torch.Tensor:
    return torch.empty(shape, device=like.device, dtype=dtype)


_dt_cache: dict = {}


def dt_tensor(dt, device) -> torch.Tensor:
    """Device float32 scalar (shape [1]) holding dt; accepts floats or tensors."""
    if isinstance(dt, torch.Tensor):
        t = dt.reshape(-1)[:1]
        if t.device != torch.device(device) or t.dtype != torch.float32:
            t = t.to(device=device, dtype=torch.float32)
        return t.contiguous()
    key = (str(device), float(dt))
    t = _dt_cache.get(key)
    if t is None:
        if len(_dt_cache) > 64:
            _dt_cache.clear()
        t = torch.tensor([float(dt)], device=device, dtype=torch.float32)
        _dt_cache[key] = t
    return t


# ------------------------------------------------------------------ neighbour search
def _version(t: torch.Tensor) -> tuple:
    return (id(t), t._version, t.data_ptr(), tuple(t.shape))


class _NbCache:
    def __init__(self):
        self.ws = {}
        self.cap_hint = {}


_nb_cache = _NbCache()


def cell_capacity_for(n: int, dim: int) -> int:
    want = max(1024, n * (1 << dim))
    cap = 1
    while cap < want:
        cap <<= 1
    return min(cap, 1 << 24)


# Reuse still-valid prior lists (sph_neighbors_refresh) instead of rebuilding them.
REUSE_PRIOR = True


_LIST_GRANULE = 1 << 22   # entries (16 MB)


def _list_capacity(entries: int) -> int:
    """List capacity rounded up to a whole number of granules.  Rebuilds then request the
    same few sizes, and the caching allocator reuses the freed blocks instead of going to
    cudaMalloc, which synchronises the device."""
    return max(-(-int(entries) // _LIST_GRANULE) * _LIST_GRANULE, _LIST_GRANULE)


def _pair_empty(nnz: int, d: int, like: torch.Tensor) -> torch.Tensor:
    """An uninitialised per-entry array of nnz rows (d columns, or a vector for d = 0) cut
    from storage rounded up to whole list granules, so that successive steps request the
    same few sizes from the caching allocator."""
    cap = _list_capacity(nnz)
    base = torch.empty((cap, d) if d else cap, dtype=like.dtype, device=like.device)
    return base[:nnz]


def speculative_refresh(x: torch.Tensor, H: torch.Tensor, params, verletScale: float, prior: Optional[AdjacencyList]):
    """Launches the validity check of `prior`'s Verlet rows for (x, H) (sph_neighbors_refresh,
    verdict only) and returns (the list kept for (x, H), its device status word) without
    reading the verdict, or None when `prior` cannot be kept whatever the verdict (none,
    another size, scale, device or dimension).  The kept list is only valid once
    verdicts_stale() says it is not stale; it filters its interacting rows on first use."""
    x = _f32(x)
    H = _f32(H)
    n = int(H.shape[0])
    dim = int(params.dim)
    dev = x.device
    if _DEVICE_LISTS[0]:   # the device-decided update below keeps or rebuilds the rows itself
        return None
    if not (REUSE_PRIOR and prior is not None and prior._x0 is not None and prior.numRows == n and
            prior.verletScale == float(verletScale) and prior._x0.device == dev and prior._dim == dim):
        return None
    params.verlet_scale = float(verletScale)
    flags = torch.zeros(4, dtype=torch.int64, device=dev)   # [-, status (low half), scratch (2 words)]
    with _timed("neighbors_refresh"):
        check(_capi.lib().sph_neighbors_refresh(_p(params), n, ptr(x), ptr(H), ptr(prior._x0), ptr(prior._h0), None, None, None,
                                                None, None, flags.data_ptr() + 16, None, flags.data_ptr() + 8, stream_ptr(dev)),
              "sph_neighbors_refresh")
    adj = AdjacencyList(neighborOffsets=prior.neighborOffsets, numNeighbors=prior.numNeighbors,
                        neighborList=prior.neighborList, numRows=n, numCols=n, nnz=prior.nnz, sortIndex=prior.sortIndex,
                        sortedKeys=prior.sortedKeys, grid=prior.grid, queryPositions=x, querySupports=H,
                        verletScale=float(verletScale))
    adj._x_version, adj._h_version = _version(x), _version(H)
    adj._x0, adj._h0, adj._dim = prior._x0, prior._h0, dim
    adj._pending = _capi.SphParams.from_buffer_copy(params)   # interacting sublist filtered on first use
    return adj, flags


def verdicts_stale(flags_list) -> list:
    """Reads the verdicts of several speculative_refresh calls in one host read: True where
    the kept list is stale (a particle left the Verlet skin) and must be rebuilt."""
    words = flags_list[0][1:2] if len(flags_list) == 1 else torch.stack([f[1] for f in flags_list])
    return [bool((int(w) & 0xffffffff) & _capi.STATUS_LIST_STALE) for w in words.cpu().tolist()]


def buildVerletList(x: torch.Tensor, H: torch.Tensor, params, verletScale: float,
                    priorNeighborhood: Optional[AdjacencyList] = None, keep_sort: bool = True) -> AdjacencyList:
    """Replaces warpSPHCore buildVerletList (schemes/crkSPH.py:54-58).

    An unchanged prior list (same position and support tensors, same version) is
    returned as is.  A prior list that is still valid for the new positions and
    supports (sph_neighbors_refresh: no particle moved or grew its support far enough
    to leave the Verlet skin) keeps its Verlet rows and gets a fresh interacting
    sublist; otherwise the list is rebuilt on the GPU."""
    x = _f32(x)
    H = _f32(H)
    if priorNeighborhood is not None and priorNeighborhood._x_version == _version(x) and \
            priorNeighborhood._h_version == _version(H) and priorNeighborhood.verletScale == float(verletScale):
        return priorNeighborhood
    if _DEVICE_LISTS[0]:
        return device_lists_for(x, H, params, verletScale).update(x, H, params)
    n = int(H.shape[0])
    dim = int(params.dim)
    params.verlet_scale = float(verletScale)
    dev = x.device
    L = _capi.lib()
    prior = priorNeighborhood
    spec = speculative_refresh(x, H, params, verletScale, prior)
    if spec is not None:
        adj, flags = spec
        if not verdicts_stale([flags])[0]:
            return adj
    cap = cell_capacity_for(n, dim)
    wsb = C.c_int64(0)
    check(L.sph_neighbors_workspace_size(_p(params), n, cap, C.byref(wsb)), "sph_neighbors_workspace_size")
    key = (dev.index, wsb.value)
    ws = _nb_cache.ws.get(key)
    if ws is None:
        _nb_cache.ws.clear()
        ws = torch.empty(wsb.value, dtype=torch.uint8, device=dev)
        _nb_cache.ws[key] = ws
    offs = torch.empty(n, dtype=torch.int32, device=dev)
    cnt = torch.empty(n, dtype=torch.int32, device=dev)
    si = torch.empty(n, dtype=torch.int32, device=dev)
    sk = torch.empty(n, dtype=torch.int32, device=dev)
    cb = torch.empty(cap, dtype=torch.int32, device=dev)
    ce = torch.empty(cap, dtype=torch.int32, device=dev)
    grid = torch.empty(8, dtype=torch.int32, device=dev)
    icnt = torch.empty(n, dtype=torch.int32, device=dev)
    flags = torch.zeros(3, dtype=torch.int64, device=dev)   # [nnz, status (int32 in the low half), interacting nnz]
    hint = _nb_cache.cap_hint.get((dev.index, n, dim))
    list_cap = hint if hint is not None else _list_capacity(n * 64)
    for attempt in range(2):
        lst = torch.empty(max(list_cap, 1), dtype=torch.int32, device=dev)
        flags.zero_()
        with _timed("neighbors_build"):
            rc = L.sph_neighbors_build(_p(params), n, ptr(x), ptr(H), ptr(ws), wsb.value, cap, ptr(si), ptr(sk), ptr(cb), ptr(ce),
                                       ptr(grid), ptr(offs), ptr(cnt), ptr(lst), list_cap, flags.data_ptr(),
                                       ptr(icnt), flags.data_ptr() + 16, flags.data_ptr() + 8, stream_ptr(dev))
        check(rc, "sph_neighbors_build")
        f = flags.cpu()
        nnz, status, innz = int(f[0]), int(f[1]) & 0xffffffff, int(f[2])
        if status & _capi.STATUS_NONFINITE:
            raise RuntimeError("buildVerletList: supports must be finite and positive")
        if status & _capi.STATUS_LIST_OVERFLOW:
            list_cap = max(list_cap, _list_capacity(int(nnz * 1.15) + 1024))
            continue
        break
    else:  # pragma: no cover
        raise RuntimeError("buildVerletList: list capacity could not be satisfied")
    _nb_cache.cap_hint[(dev.index, n, dim)] = max(_list_capacity(int(nnz * 1.15) + 1024), hint or 0)
    adj = AdjacencyList(neighborOffsets=offs, numNeighbors=cnt, neighborList=lst[:nnz], numRows=n, numCols=n, nnz=nnz,
                        sortIndex=si if keep_sort else None, sortedKeys=sk if keep_sort else None, grid=grid,
                        queryPositions=x, querySupports=H, verletScale=float(verletScale),
                        interCounts=icnt, interNnz=innz)
    adj._x_version = _version(x)
    adj._h_version = _version(H)
    adj._x0, adj._h0, adj._dim = x.clone(), H.clone(), dim   # build-time state for the validity check
    return adj


def expand_adjacency(adj: AdjacencyList):
    dev = adj.neighborList.device
    nnz = list_entries(adj)
    i = torch.empty(nnz, dtype=torch.int64, device=dev)
    j = torch.empty(nnz, dtype=torch.int64, device=dev)
    check(_capi.lib().sph_neighbors_expand(adj.numRows, ptr(adj.neighborOffsets), ptr(adj.numNeighbors),
                                           ptr(adj.neighborList), nnz, ptr(i), ptr(j), stream_ptr(dev)),
          "sph_neighbors_expand")
    return i, j


def _csr(adj: AdjacencyList):
    return iptr(adj.neighborOffsets), iptr(adj.numNeighbors), iptr(adj.neighborList)


def _materialize_inter(adj: AdjacencyList, V_out: Optional[torch.Tensor] = None) -> None:
    """Rewrites the rows of a kept prior list with the interacting entries for the
    current positions first (sph_neighbors_refresh).  The rows go to a new tensor:
    earlier stages keep the old order their pairwise arrays are indexed by.  With V_out
    the CRK volumes of the rewritten rows are computed in the same pass."""
    if isinstance(adj._pending, _DevicePending):
        adj._pending.rewrite(adj, V_out)
        return
    params = adj._pending
    n, dev = adj.numRows, adj.neighborList.device
    icnt = torch.empty(n, dtype=torch.int32, device=dev)
    lst = torch.empty(_list_capacity(adj.nnz), dtype=torch.int32, device=dev)
    flags = torch.zeros(4, dtype=torch.int64, device=dev)   # [inter nnz, status (low half), scratch (2 words)]
    args = (_p(params), n, ptr(adj.queryPositions), ptr(adj.querySupports), ptr(adj._x0), ptr(adj._h0), ptr(adj.neighborOffsets),
            ptr(adj.numNeighbors), ptr(adj.neighborList), ptr(lst), ptr(icnt), flags.data_ptr() + 16, flags.data_ptr(),
            flags.data_ptr() + 8)
    with _timed("neighbors_refresh"):
        if V_out is None:
            check(_capi.lib().sph_neighbors_refresh(*args, stream_ptr(dev)), "sph_neighbors_refresh")
        else:   # the rewrite fused with the CRK volume sum of the rewritten rows
            check(_capi.lib().sph_neighbors_refresh_volume(*args, fptr(V_out), stream_ptr(dev)), "sph_neighbors_refresh_volume")
    adj.neighborList, adj.interCounts = lst[: adj.nnz], icnt
    adj._ij = None
    adj._inter_nnz_dev = flags[:1]
    adj._pending = None


# ------------------------------------------------------------------ device-decided lists
# A stepping loop that must not read the device (a CUDA graph replays it, or the host runs
# ahead of the GPU) keeps its Verlet rows in fixed buffers and lets the GPU decide between
# keeping and rebuilding them (sph_neighbors_update); pair passes walk per-call rewrites of
# the rows (sph_neighbors_rewrite).  Lists then report their capacity as nnz (per-entry
# arrays are allocated that long; entries past the rows are never read) and
# ``list_entries`` reads the true count.
_DEVICE_LISTS = [0]
_device_lists: dict = {}
DEVICE_LIST_HEADROOM = 1.3   # list capacity over the entries of the sizing build


@contextlib.contextmanager
def device_decided_lists():
    """Within this context buildVerletList neither reads the device nor allocates its rows:
    see DeviceLists."""
    _DEVICE_LISTS[0] += 1
    try:
        yield
    finally:
        _DEVICE_LISTS[0] -= 1


class DeviceLists:
    """The kept Verlet rows of one particle set (n, dim, verlet scale, device) for
    device-decided updates.  The list capacity is DEVICE_LIST_HEADROOM times the entries of
    one ordinary build at creation; a rebuild that needs more sets the overflow bit of the
    status word, which ``check()`` (one host read) turns into an error."""

    def __init__(self, x: torch.Tensor, H: torch.Tensor, params, verletScale: float):
        n, dim, dev = int(H.shape[0]), int(params.dim), x.device
        self.n, self.dim, self.verletScale = n, dim, float(verletScale)
        sizing = _capi.SphParams.from_buffer_copy(params)
        with _suspend_device_lists():
            probe = buildVerletList(x, H, sizing, verletScale, None, keep_sort=False)
        self.capacity = int(probe.nnz * DEVICE_LIST_HEADROOM) + 4096
        self.cell_capacity = cell_capacity_for(n, dim)
        wsb = C.c_int64(0)
        check(_capi.lib().sph_neighbors_workspace_size(_p(sizing), n, self.cell_capacity, C.byref(wsb)), "sph_neighbors_workspace_size")
        self.ws_bytes = wsb.value
        self.ws = torch.empty(self.ws_bytes, dtype=torch.uint8, device=dev)
        i32 = dict(dtype=torch.int32, device=dev)
        self.sort_index, self.sorted_keys = torch.empty(n, **i32), torch.empty(n, **i32)
        self.cell_begin, self.cell_end = torch.empty(self.cell_capacity, **i32), torch.empty(self.cell_capacity, **i32)
        self.grid = torch.zeros(8, **i32)
        self.offsets, self.counts = torch.zeros(n, **i32), torch.zeros(n, **i32)
        self.rows = torch.zeros(self.capacity, **i32)     # zero-filled: a cut row never names a bad index
        self.nnz = torch.zeros(1, dtype=torch.int64, device=dev)
        # zero build-time supports fail every validity check: the first update builds
        self.x0 = x.detach().clone()
        self.h0 = torch.zeros_like(H)
        self.verdict = torch.zeros(4, **i32)
        self.status = torch.zeros(1, **i32)
        self.rebuilds = torch.zeros(1, dtype=torch.int64, device=dev)   # counted on the device
        self.generation = 0

    def update(self, x: torch.Tensor, H: torch.Tensor, params) -> AdjacencyList:
        x, H = _f32(x), _f32(H)
        params.verlet_scale = self.verletScale
        with _timed("neighbors_update"):
            check(_capi.lib().sph_neighbors_update(_p(params), self.n, ptr(x), ptr(H), ptr(self.x0), ptr(self.h0), ptr(self.ws),
                                                   self.ws_bytes, self.cell_capacity, ptr(self.sort_index), ptr(self.sorted_keys),
                                                   ptr(self.cell_begin), ptr(self.cell_end), ptr(self.grid), ptr(self.offsets),
                                                   ptr(self.counts), ptr(self.rows), self.capacity, ptr(self.nnz), ptr(self.verdict),
                                                   ptr(self.status), ptr(self.rebuilds), stream_ptr(x.device)), "sph_neighbors_update")
        self.generation += 1
        adj = AdjacencyList(neighborOffsets=self.offsets, numNeighbors=self.counts, neighborList=self.rows, numRows=self.n,
                            numCols=self.n, nnz=self.capacity, grid=self.grid, queryPositions=x, querySupports=H,
                            verletScale=self.verletScale)
        adj._x_version, adj._h_version, adj._dim = _version(x), _version(H), self.dim
        adj._pending = _DevicePending(self, _capi.SphParams.from_buffer_copy(params), self.generation)
        adj._device_rows = True
        return adj

    def check(self) -> None:
        """Raises when a rebuild since creation overflowed the list or met a non-finite or
        non-positive support (one host read)."""
        st = int(self.status.item()) & 0xffffffff
        if st & _capi.STATUS_NONFINITE:
            raise RuntimeError("device-decided neighbour list: supports must be finite and positive")
        if st & _capi.STATUS_LIST_OVERFLOW:
            raise RuntimeError(f"device-decided neighbour list: a rebuild needed more than {self.capacity} entries; "
                               "raise DEVICE_LIST_HEADROOM and start again from a saved state")


class _DevicePending:
    """The interacting rewrite of a device-decided list, done on first use."""

    def __init__(self, lists: DeviceLists, params, generation: int):
        self.lists, self.params, self.generation = lists, params, generation

    def rewrite(self, adj: AdjacencyList, V_out: Optional[torch.Tensor]) -> None:
        nb = self.lists
        if nb.generation != self.generation:
            raise RuntimeError("a device-decided list was used after a later update of the same rows")
        n, dev = nb.n, nb.rows.device
        lst = torch.empty(nb.capacity, dtype=torch.int32, device=dev)
        offs, cnt, icnt = (torch.empty(n, dtype=torch.int32, device=dev) for _ in range(3))
        innz = torch.empty(1, dtype=torch.int64, device=dev)
        with _timed("neighbors_rewrite"):
            check(_capi.lib().sph_neighbors_rewrite(_p(self.params), n, ptr(adj.queryPositions), ptr(adj.querySupports),
                                                    ptr(nb.offsets), ptr(nb.counts), ptr(nb.rows), ptr(lst), ptr(offs), ptr(cnt),
                                                    ptr(icnt), ptr(innz), fptr(V_out) if V_out is not None else None,
                                                    ptr(nb.status), stream_ptr(dev)), "sph_neighbors_rewrite")
        adj.neighborOffsets, adj.numNeighbors, adj.neighborList, adj.interCounts = offs, cnt, lst, icnt
        adj._inter_nnz_dev = innz
        adj._ij = None
        adj._pending = None


@contextlib.contextmanager
def _suspend_device_lists():
    saved = _DEVICE_LISTS[0]
    _DEVICE_LISTS[0] = 0
    try:
        yield
    finally:
        _DEVICE_LISTS[0] = saved


def device_lists_for(x: torch.Tensor, H: torch.Tensor, params, verletScale: float) -> DeviceLists:
    """The DeviceLists of this particle set, created (with one sizing build) on first use."""
    key = (x.device.index, int(H.shape[0]), int(params.dim), float(verletScale))
    nb = _device_lists.get(key)
    if nb is None:
        nb = DeviceLists(x, H, params, verletScale)
        _device_lists[key] = nb
    return nb


def release_device_lists() -> None:
    """Drops every DeviceLists (their buffers return to the caching allocator)."""
    _device_lists.clear()


def list_entries(adj: AdjacencyList) -> int:
    """Entries in the rows of `adj`: its nnz, or for a device-decided list (whose nnz is the
    capacity) the true count, read from the device."""
    if not getattr(adj, "_device_rows", False) or adj.numRows == 0:
        return adj.nnz
    return int((adj.neighborOffsets[-1].long() + adj.numNeighbors[-1].long()).item())


def _lists(params, adj: AdjacencyList, interacting: bool):
    """Selects the rows a pass walks: the interacting prefixes (r < max(H_i, H_j)) when
    available and sufficient, else the whole Verlet rows.  A kept prior list has its
    rows reordered here, on first use."""
    params.list_stride = 1
    if interacting and adj._pending is not None:
        _materialize_inter(adj)
    if interacting and adj.interCounts is not None:
        return iptr(adj.neighborOffsets), iptr(adj.interCounts), iptr(adj.neighborList)
    return _csr(adj)


# ------------------------------------------------------------------ pair operations
def density(params, x, H, m, adj: AdjacencyList, supportMode: SupportScheme = SupportScheme.Gather) -> torch.Tensor:
    n = H.shape[0]
    rho = _empty(n, H)
    with _timed("density"):
        check(_capi.lib().sph_density_gather(_p(params), n, _SUPPORT[supportMode], fptr(x), fptr(H), fptr(m), *_lists(params, adj, True), ptr(rho),
                                             stream_ptr(H.device)), "sph_density_gather")
    return rho


def minmax(a: torch.Tensor) -> torch.Tensor:
    out = _empty(2, a)
    with _timed("minmax"):
        check(_capi.lib().sph_minmax(a.shape[0], fptr(a), ptr(out), stream_ptr(a.device)), "sph_minmax")
    return out


def owen_iter(params, x, H, adj: AdjacencyList, lut_nh: torch.Tensor, lut_psiH: torch.Tensor, target_nh: float,
              hbounds: torch.Tensor, want_psi0: bool = False):
    """One Owen support iteration (psi0 pair sums, table lookup, update): (psiH, H_new,
    ratio), and psi0 last when ``want_psi0``."""
    n = H.shape[0]
    psiH, Hn, ratio = _empty(n, H), _empty(n, H), _empty(n, H)
    psi0 = _empty(n, H) if want_psi0 else None
    if lut_nh.dtype != torch.float64 or lut_psiH.dtype != torch.float64:
        raise RuntimeError("the Owen table is FP64")
    with _timed("owen_iter"):
        check(_capi.lib().sph_owen_iter(_p(params), n, fptr(x), fptr(H), *_lists(params, adj, True), ptr(lut_nh), ptr(lut_psiH),
                                        int(lut_nh.shape[0]), float(target_nh), fptr(hbounds), ptr(psi0), ptr(psiH), ptr(Hn),
                                        ptr(ratio), stream_ptr(H.device)), "sph_owen_iter")
    return (psiH, Hn, ratio, psi0) if want_psi0 else (psiH, Hn, ratio)


def adaptive_h_iter(params, x, H, m, adj: AdjacencyList, hbounds: torch.Tensor):
    n = H.shape[0]
    rho, Hn, ratio = _empty(n, H), _empty(n, H), _empty(n, H)
    with _timed("adaptive_h_iter"):
        # the supports change right after this pass: a kept list that has not filtered its
        # interacting subset yet is walked over its Verlet rows (W = 0 beyond the support)
        check(_capi.lib().sph_adaptive_h_iter(_p(params), n, 0, fptr(x), fptr(H), fptr(m), *_lists(params, adj, adj._pending is None),
                                              fptr(hbounds), ptr(rho), ptr(Hn),
                                              ptr(ratio), stream_ptr(H.device)), "sph_adaptive_h_iter")
    return rho, Hn, ratio


def crk_volume(params, x, H, adj: AdjacencyList) -> torch.Tensor:
    """V_i = 1 / sum_j W(r_ij, H_j).  A kept list whose rows still await their rewrite for
    (x, H) gets it here, fused with the volume sum (sph_neighbors_refresh_volume)."""
    n = H.shape[0]
    V = _empty(n, H)
    if adj is not None and adj._pending is not None and adj.queryPositions is x and adj.querySupports is H:
        _materialize_inter(adj, V_out=V)
        return V
    with _timed("crk_volume"):
        check(_capi.lib().sph_crk_volume(_p(params), n, fptr(x), fptr(H), *_lists(params, adj, True), ptr(V), stream_ptr(H.device)), "sph_crk_volume")
    return V


def crk_factors(params, x, H, m, V, adj: AdjacencyList):
    n, d = H.shape[0], int(params.dim)
    A, B, gA, gB, rho = _empty(n, H), _empty((n, d), H), _empty((n, d), H), _empty((n, d, d), H), _empty(n, H)
    with _timed("crk_factors"):
        check(_capi.lib().sph_crk_factors(_p(params), n, fptr(x), fptr(H), fptr(m), fptr(V), *_lists(params, adj, True), ptr(A), ptr(B), ptr(gA), ptr(gB),
                                          ptr(rho), stream_ptr(H.device)), "sph_crk_factors")
    return CRKState(A=A, B=B, gradA=gA, gradB=gB), rho


def crk_factors_eos(params, x, H, m, V, adj: AdjacencyList, u):
    """crk_factors with the ideal-gas EOS of the CRK density in the same pass
    (sph_crk_factors_eos): (crk, rho, entropy, P, c)."""
    n, d = H.shape[0], int(params.dim)
    A, B, gA, gB, rho = _empty(n, H), _empty((n, d), H), _empty((n, d), H), _empty((n, d, d), H), _empty(n, H)
    Ae, P, c = _empty(n, H), _empty(n, H), _empty(n, H)
    with _timed("crk_factors"):
        check(_capi.lib().sph_crk_factors_eos(_p(params), n, fptr(x), fptr(H), fptr(m), fptr(V), *_lists(params, adj, True), ptr(A), ptr(B),
                                              ptr(gA), ptr(gB), ptr(rho), fptr(u), ptr(Ae), ptr(P), ptr(c), stream_ptr(H.device)),
              "sph_crk_factors_eos")
    return CRKState(A=A, B=B, gradA=gA, gradB=gB), rho, Ae, P, c


def eos_ideal_gas(params, u, rho):
    n = u.shape[0]
    A, P, c = _empty(n, u), _empty(n, u), _empty(n, u)
    with _timed("eos_ideal_gas"):
        check(_capi.lib().sph_eos_ideal_gas(_p(params), n, fptr(u), fptr(rho), ptr(A), ptr(P), ptr(c), stream_ptr(u.device)),
              "sph_eos_ideal_gas")
    return A, P, c


def grad_v(params, x, H, m, rho, V, crk: CRKState, v, c, adj: AdjacencyList, cullen: bool, want_vsig: bool = False):
    """CRK velocity gradient (+ the Cullen divergence when `cullen`).  v_sig needs the
    Verlet set; the step computes it in the Cullen pass, tests may ask for it here."""
    n, d = H.shape[0], int(params.dim)
    G, drho = _empty((n, d, d), H), _empty(n, H)
    div = _empty(n, H) if cullen else None
    vs = _empty(n, H) if want_vsig else None
    with _timed("grad_v"):
        check(_capi.lib().sph_grad_v(_p(params), n, fptr(x), fptr(H), fptr(m), fptr(rho), fptr(V), fptr(crk.A), fptr(crk.B), fptr(crk.gradA),
                                     fptr(crk.gradB), fptr(v), fptr(c), *_lists(params, adj, not want_vsig), ptr(G), ptr(drho), ptr(div),
                                     ptr(vs), stream_ptr(H.device)), "sph_grad_v")
    return G, drho, div, vs


def switch_cullen(params, x, H, m, rho, div, div_prev, vsig, alpha0, dt, adj: AdjacencyList, want_R: bool = False,
                  v=None, c=None, want_vsig: bool = False):
    """Cullen-Dehnen switch.  With vsig=None the signal velocity is computed in the same
    pass from v and c over the Verlet list (returned third when want_vsig)."""
    n = H.shape[0]
    al = _empty(n, H)
    R = _empty(n, H) if want_R else None
    vs_out = _empty(n, H) if (vsig is None and want_vsig) else None
    with _timed("switch_cullen"):
        check(_capi.lib().sph_switch_cullen(_p(params), n, fptr(x), fptr(H), fptr(m), fptr(rho), fptr(div), fptr(_f32(div_prev)),
                                            fptr(vsig), fptr(v), fptr(c), fptr(_f32(alpha0)), fptr(dt_tensor(dt, H.device)),
                                            *_lists(params, adj, vsig is not None), ptr(al), ptr(R), ptr(vs_out),
                                            stream_ptr(H.device)), "sph_switch_cullen")
    return al, R, vs_out


def switch_hopkins_terms(params, x, H, m, rho, v, alpha0, adj: AdjacencyList):
    """Cullen-Hopkins switch terms: (alphas, div, |S|^2, R)."""
    n = H.shape[0]
    al, div, s2, R = _empty(n, H), _empty(n, H), _empty(n, H), _empty(n, H)
    with _timed("switch_hopkins_terms"):
        check(_capi.lib().sph_switch_hopkins_terms(_p(params), n, fptr(x), fptr(H), fptr(m), fptr(rho), fptr(v), fptr(_f32(alpha0)),
                                                   *_lists(params, adj, True), ptr(div), ptr(s2), ptr(al), ptr(R),
                                                   stream_ptr(H.device)), "sph_switch_hopkins_terms")
    return al, div, s2, R


def surface_color_field(params, x, H, m, rho, adj: AdjacencyList):
    """Colour field c_i = sum_j m_j/rho_j W(r_ij, H_i) (colorFieldCompute.py:11-31)."""
    c = _empty(H.shape[0], H)
    with _timed("surface_color_field"):
        check(_capi.lib().sph_surface_color_field(_p(params), H.shape[0], fptr(x), fptr(H), fptr(m), fptr(rho),
                                                  *_lists(params, adj, True), ptr(c), stream_ptr(H.device)),
              "sph_surface_color_field")
    return c


def surface_detect_color_field(params, x, H, m, rho, color, adj: AdjacencyList, neighbor_limit: float, normal_sign: float = -1.0):
    """detectFreeSurfaceColorField (colorFieldDetection.py:16-73): (mask, normals, counts)."""
    n, d = H.shape[0], x.shape[1]
    fs, nn = _empty(n, H), _empty(n, H)
    normals = torch.empty((n, d), device=H.device, dtype=torch.float32)
    with _timed("surface_detect"):
        check(_capi.lib().sph_surface_detect_color_field(_p(params), n, fptr(x), fptr(H), fptr(m), fptr(rho), fptr(color),
                                                         *_lists(params, adj, True), float(neighbor_limit), float(normal_sign),
                                                         ptr(fs), ptr(normals), ptr(nn), stream_ptr(H.device)),
              "sph_surface_detect_color_field")
    return fs, normals, nn


def surface_dilate(params, x, H, fs, adj: AdjacencyList):
    """One dilation iteration (wp_dilate.py:14-89): the sum of fs_j over the super-symmetric pairs."""
    out = _empty(H.shape[0], H)
    with _timed("surface_dilate"):
        check(_capi.lib().sph_surface_dilate(_p(params), H.shape[0], fptr(x), fptr(H), fptr(_f32(fs)),
                                             *_lists(params, adj, True), ptr(out), stream_ptr(H.device)), "sph_surface_dilate")
    return out


def surface_barecasco(params, x, H, adj: AdjacencyList, threshold: float):
    """Barecasco detection (wp_barecasco.py, barecascoDetection.py): (mask, normalised cover
    vectors, cone counts)."""
    n, d = H.shape[0], x.shape[1]
    fs, cnt = _empty(n, H), _empty(n, H)
    normals = torch.empty((n, d), device=H.device, dtype=torch.float32)
    with _timed("surface_barecasco"):
        check(_capi.lib().sph_surface_barecasco(_p(params), n, fptr(x), fptr(H), *_lists(params, adj, True), float(threshold),
                                                ptr(fs), ptr(normals), ptr(cnt), stream_ptr(H.device)), "sph_surface_barecasco")
    return fs, normals, cnt


def surface_maronne(params, x, H, normals, adj: AdjacencyList):
    """Maronne detection with the given normals (wp_maronne.py, maronneDetection.py): (mask, counts)."""
    n = H.shape[0]
    fs, cnt = _empty(n, H), _empty(n, H)
    with _timed("surface_maronne"):
        check(_capi.lib().sph_surface_maronne(_p(params), n, fptr(x), fptr(H), fptr(normals), *_lists(params, adj, True), ptr(fs),
                                              ptr(cnt), stream_ptr(H.device)), "sph_surface_maronne")
    return fs, cnt


def surface_detect_color_gradient(params, x, H, m, rho, color, adj: AdjacencyList, threshold: float):
    """Colour-field-gradient detection (colorFieldGradientDetection.py): (mask, normals)."""
    n, d = H.shape[0], x.shape[1]
    fs = _empty(n, H)
    normals = torch.empty((n, d), device=H.device, dtype=torch.float32)
    with _timed("surface_detect"):
        check(_capi.lib().sph_surface_detect_color_gradient(_p(params), n, fptr(x), fptr(H), fptr(m), fptr(rho), fptr(color),
                                                            *_lists(params, adj, True), float(threshold), ptr(fs), ptr(normals),
                                                            stream_ptr(H.device)), "sph_surface_detect_color_gradient")
    return fs, normals


def surface_renormalization(params, x, H, m, rho, adj: AdjacencyList):
    """Renormalisation matrices L = pinv(M) [n, d, d] and the smallest |eigenvalue| of M [n]."""
    n, d = H.shape[0], x.shape[1]
    L = torch.empty((n, d, d), device=H.device, dtype=torch.float32)
    lam = _empty(n, H)
    with _timed("surface_renormalization"):
        check(_capi.lib().sph_surface_renormalization(_p(params), n, fptr(x), fptr(H), fptr(m), fptr(rho), *_lists(params, adj, True),
                                                      ptr(L), ptr(lam), stream_ptr(H.device)), "sph_surface_renormalization")
    return L, lam


def surface_renormalized_normals(params, mode: int, x, H, m, rho, L, lambdas, adj: AdjacencyList, want_grad: bool = False):
    """Normals from the renormalised lambda gradient (mode 0) or Maronne's (mode 1); with
    ``want_grad`` also the renormalised gradient."""
    n, d = H.shape[0], x.shape[1]
    normals = torch.empty((n, d), device=H.device, dtype=torch.float32)
    g = torch.empty((n, d), device=H.device, dtype=torch.float32) if want_grad else None
    with _timed("surface_normals"):
        check(_capi.lib().sph_surface_renormalized_normals(_p(params), n, int(mode), fptr(x), fptr(H), fptr(m), fptr(rho), fptr(L),
                                                           fptr(lambdas) if lambdas is not None else None,
                                                           *_lists(params, adj, True), ptr(normals), ptr(g), stream_ptr(H.device)),
              "sph_surface_renormalized_normals")
    return (normals, g) if want_grad else normals


def switch_hopkins_update(params, x, H, v, c, div, div_prev, alpha0, dt, adj: AdjacencyList, want_vsig: bool = False):
    """Cullen-Hopkins alpha0 update (v_sig over the Verlet rows); (alpha0, v_sig or None)."""
    n = H.shape[0]
    a0 = _empty(n, H)
    vs = _empty(n, H) if want_vsig else None
    with _timed("switch_hopkins_update"):
        check(_capi.lib().sph_switch_hopkins_update(_p(params), n, fptr(x), fptr(H), fptr(v), fptr(c), fptr(div), fptr(_f32(div_prev)),
                                                    fptr(_f32(alpha0)), fptr(dt_tensor(dt, H.device)), *_lists(params, adj, False),
                                                    ptr(a0), ptr(vs), stream_ptr(H.device)), "sph_switch_hopkins_update")
    return a0, vs


def switch_balsara(params, DvDx, c):
    n = c.shape[0]
    al = _empty(n, c)
    check(_capi.lib().sph_switch_balsara(_p(params), n, fptr(DvDx), fptr(c), ptr(al), stream_ptr(c.device)), "sph_switch_balsara")
    return al


def crk_accel_dudt(params, x, H, m, rho, V, crk: CRKState, v, c, P, DvDx, adj: AdjacencyList, pair_arrays: bool = True,
                   want_dEdt: bool = False, reference_layout: bool = True):
    """Fused CRK momentum and energy RHS over the interacting prefixes, gathering each
    neighbour from a packed per-particle record (sph_crk_accel_dudt_packed).  The
    pairwise accelerations are returned in Verlet-entry order.  With
    ``reference_layout`` the rest of each row is written as zeros, the reference's
    layout; without it only the interacting prefix is written and the rest is left
    unspecified (what the library's own readers of these arrays need: the energy
    partition and the compatible-energy finalize read the prefix only).
    Returns (dvdt, dudt, ap, av), and dE/dt last when ``want_dEdt``."""
    n, d = H.shape[0], int(params.dim)
    dvdt, dudt = _empty((n, d), H), _empty(n, H)
    dEdt = _empty(n, H) if want_dEdt else None
    ap = _pair_empty(adj.nnz, d, H) if pair_arrays else None
    av = _pair_empty(adj.nnz, d, H) if pair_arrays else None
    recs = _empty(n * crk_record_floats(d), H)
    with _timed("crk_accel_dudt"):
        rows = _lists(params, adj, True)
        check(_capi.lib().sph_crk_accel_dudt_packed(_p(params), n, fptr(x), fptr(H), fptr(m), fptr(rho), fptr(V), fptr(crk.A),
                                                    fptr(crk.B), fptr(crk.gradA), fptr(crk.gradB), fptr(v), fptr(c), fptr(P),
                                                    fptr(DvDx), *rows, iptr(adj.numNeighbors) if reference_layout else None,
                                                    ptr(dvdt), ptr(dudt), ptr(dEdt), ptr(ap), ptr(av), ptr(recs),
                                                    stream_ptr(H.device)), "sph_crk_accel_dudt_packed")
    return (dvdt, dudt, ap, av, dEdt) if want_dEdt else (dvdt, dudt, ap, av)


def crk_record_floats(dim: int) -> int:
    """Floats per particle of the packed record of the CRK accel pass."""
    return int(_capi.lib().sph_crk_record_floats(int(dim)))


def pair_reference_layout(adj: AdjacencyList, *arrays):
    """Copies of per-entry arrays with the entries past each row's interacting prefix set
    to zero: the reference's layout of ap_ij / av_ij, for arrays written over the
    prefixes only.  Arrays of lists without interacting prefixes are returned as is."""
    if adj is None or adj.interCounts is None or getattr(adj, "_pending", None) is not None:
        return arrays
    n = adj.numRows
    nnz = list_entries(adj)
    dev = adj.neighborOffsets.device
    rows = torch.repeat_interleave(torch.arange(n, device=dev), adj.numNeighbors.long(), output_size=nnz)
    pos = torch.arange(nnz, device=dev) - adj.neighborOffsets.long()[rows]
    tail = pos >= adj.interCounts.long()[rows]
    out = []
    for a in arrays:
        if a is None:
            out.append(None)
            continue
        b = a[:nnz].clone()
        b[tail] = 0
        out.append(b)
    return tuple(out)


def compsph_prep(params, x, H, m, rho, v, adj: AdjacencyList, grad_h: bool = True, want_div: bool = True,
                 want_drhodt: bool = True):
    """Grad-h Omega, the super-symmetric velocity divergence and the consistent
    continuity d rho/dt from one pass (each None when not requested)."""
    n = H.shape[0]
    om = _empty(n, H) if grad_h else None
    div = _empty(n, H) if want_div else None
    dr = _empty(n, H) if want_drhodt else None
    with _timed("compsph_prep"):
        check(_capi.lib().sph_compsph_prep(_p(params), n, fptr(x), fptr(H), fptr(m), fptr(rho), fptr(v), *_lists(params, adj, True),
                                           ptr(om), ptr(div), ptr(dr), stream_ptr(H.device)), "sph_compsph_prep")
    return om, div, dr


def compsph_accel_dudt(params, x, H, m, rho, v, c, alpha, P, omega, adj: AdjacencyList, pair_arrays: bool = True,
                       want_dEdt: bool = True, reference_layout: bool = True):
    """Fused CompSPH momentum and energy RHS over packed particle records
    (sph_compsph_accel_dudt_packed); returns (dvdt, dudt, dEdt, ap_ij, av_ij) with
    the pairwise accelerations in Verlet-entry order: zeros beyond the support with
    ``reference_layout``, else written over the interacting prefixes only (as
    crk_accel_dudt)."""
    n, d = H.shape[0], int(params.dim)
    dvdt, dudt = _empty((n, d), H), _empty(n, H)
    dEdt = _empty(n, H) if want_dEdt else None
    ap = _pair_empty(adj.nnz, d, H) if pair_arrays else None
    av = _pair_empty(adj.nnz, d, H) if pair_arrays else None
    recs = _empty(n * int(_capi.lib().sph_compsph_record_floats(d)), H)
    with _timed("compsph_accel_dudt"):
        rows = _lists(params, adj, True)
        check(_capi.lib().sph_compsph_accel_dudt_packed(_p(params), n, fptr(x), fptr(H), fptr(m), fptr(rho), fptr(v), fptr(c),
                                                        fptr(alpha), fptr(P), fptr(omega), *rows,
                                                        iptr(adj.numNeighbors) if reference_layout else None, ptr(dvdt), ptr(dudt),
                                                        ptr(dEdt), ptr(ap), ptr(av), ptr(recs), stream_ptr(H.device)),
              "sph_compsph_accel_dudt_packed")
    return dvdt, dudt, dEdt, ap, av


def monaghan_rhs(params, x, H, m, rho, v, u, c, alpha, P, omega, adj: AdjacencyList, terms: bool = False):
    """Monaghan-scheme RHS: (dvdt, dudt, dEdt, parts) with parts = dict(pressure, viscosity,
    pdv, conductivity, heating) when `terms`, else None."""
    n, d = H.shape[0], int(params.dim)
    dvdt, dudt, dEdt = _empty((n, d), H), _empty(n, H), _empty(n, H)
    parts = None
    if terms:
        parts = dict(pressure=_empty((n, d), H), viscosity=_empty((n, d), H), pdv=_empty(n, H), conductivity=_empty(n, H),
                     heating=_empty(n, H))
    q = parts or {}
    with _timed("monaghan_rhs"):
        check(_capi.lib().sph_monaghan_rhs(_p(params), n, fptr(x), fptr(H), fptr(m), fptr(rho), fptr(v), fptr(u), fptr(c), fptr(alpha),
                                           fptr(P), fptr(omega), *_lists(params, adj, True), ptr(dvdt), ptr(dudt), ptr(dEdt),
                                           ptr(q.get("pressure")), ptr(q.get("viscosity")), ptr(q.get("pdv")),
                                           ptr(q.get("conductivity")), ptr(q.get("heating")), stream_ptr(H.device)), "sph_monaghan_rhs")
    return dvdt, dudt, dEdt, parts


def compsph_balance(params, m, rho, P, u, v, dvdt, dt, adj: AdjacencyList, ap, av):
    """Energy partition f_ij for every Verlet entry."""
    n, d = m.shape[0], int(params.dim)
    f = _pair_empty(adj.nnz, 0, m)
    scratch = _empty(n * (d + 1), m)
    with _timed("compsph_balance"):
        check(_capi.lib().sph_compsph_balance(_p(params), n, fptr(m), fptr(rho), fptr(P), fptr(u), fptr(v), fptr(dvdt),
                                              fptr(dt_tensor(dt, m.device)), *_lists(params, adj, False),
                                              iptr(adj.interCounts) if adj._pending is None else None, fptr(ap), fptr(av),
                                              ptr(scratch), ptr(f), stream_ptr(m.device)), "sph_compsph_balance")
    return f


def cfl_dt(params, H, u, rho=None, dt_prev=None) -> torch.Tensor:
    """Device-side CFL time step (returns a [1] float32 tensor; no host sync)."""
    buf = _empty(4, H)
    prev = None if dt_prev is None else dt_tensor(dt_prev, H.device)
    with _timed("cfl_dt"):
        check(_capi.lib().sph_cfl_dt(_p(params), H.shape[0], fptr(H), fptr(u), None, ptr(prev), ptr(buf), stream_ptr(H.device)),
              "sph_cfl_dt")
    return buf[:1]


def rk_combine(params, y0: torch.Tensor, ks, weights, dt, wrap_dim: int = 0, out: Optional[torch.Tensor] = None) -> torch.Tensor:
    y0 = _f32(y0)
    y = torch.empty_like(y0) if out is None else out
    kp = [fptr(_f32(k)) for k in ks]
    arr = _capi.ptr_array(kp) if kp else None
    w = _capi.double_array(weights) if kp else None
    with _timed("rk_combine"):
        check(_capi.lib().sph_rk_combine(_p(params), y0.numel(), ptr(y0), len(kp), C.cast(arr, C.c_void_p) if arr is not None else None,
                                         C.cast(w, C.c_void_p) if w is not None else None, fptr(dt_tensor(dt, y0.device)), wrap_dim,
                                         ptr(y), stream_ptr(y0.device)), "sph_rk_combine")
    return y


def rk_combine_fields(params, fields, weights, dt):
    """rk_combine over up to 4 fields in one launch (sph_rk_combine_fields).  fields: list of
    (y0, [K_1..K_nk], wrap_dim); returns the new arrays in order."""
    if not fields:
        return []
    if len(fields) > 4:
        raise ValueError("rk_combine_fields: at most 4 fields per launch")
    nk = len(weights)
    y0s = [_f32(y0) for y0, _, _ in fields]
    outs = [torch.empty_like(y) for y in y0s]
    ks = []
    for (_, kf, _), y in zip(fields, y0s):
        if len(kf) != nk:
            raise ValueError("rk_combine_fields: every field needs one derivative per weight")
        ks += [fptr(_f32(k)) for k in kf]
    counts = (C.c_int64 * len(fields))(*[y.numel() for y in y0s])
    wraps = (C.c_int32 * len(fields))(*[int(w) for _, _, w in fields])
    karr = _capi.ptr_array(ks) if ks else None
    w = _capi.double_array(weights) if nk else None
    dev = y0s[0].device
    with _timed("rk_combine"):
        check(_capi.lib().sph_rk_combine_fields(_p(params), len(fields), C.cast(counts, C.c_void_p),
                                                C.cast(_capi.ptr_array([ptr(y) for y in y0s]), C.c_void_p),
                                                C.cast(_capi.ptr_array([ptr(y) for y in outs]), C.c_void_p),
                                                C.cast(wraps, C.c_void_p), nk,
                                                C.cast(karr, C.c_void_p) if karr is not None else None,
                                                C.cast(w, C.c_void_p) if w is not None else None,
                                                fptr(dt_tensor(dt, dev)), stream_ptr(dev)), "sph_rk_combine_fields")
    return outs


def finalize_compatible_energy(params, weights, dt, v0, u0, stages):
    """stages: list of (dvdt, adjacency, f_ij, ap_ij, av_ij)."""
    n, d = u0.shape[0], int(params.dim)
    u = _empty(n, u0)
    scratch = _empty(n * (1 + d), u0)
    ns = len(stages)
    # a stage whose list has interacting prefixes is walked over them (its pairwise
    # arrays carry no interaction past them, and may be left unwritten there)
    inter = [s[1].interCounts is not None and s[1]._pending is None for s in stages]
    params.list_stride = 1
    arrs = [_capi.ptr_array([fptr(s[0]) for s in stages]),
            _capi.ptr_array([iptr(s[1].neighborOffsets) for s in stages]),
            _capi.ptr_array([iptr(s[1].interCounts if it else s[1].numNeighbors) for s, it in zip(stages, inter)]),
            _capi.ptr_array([iptr(s[1].neighborList) for s in stages]),
            _capi.ptr_array([fptr(s[2]) for s in stages]),
            _capi.ptr_array([fptr(s[3]) for s in stages]),
            _capi.ptr_array([fptr(s[4]) for s in stages])]
    w = _capi.double_array(weights)
    with _timed("finalize_compatible_energy"):
        check(_capi.lib().sph_finalize_compatible_energy(_p(params), n, ns, C.cast(w, C.c_void_p), fptr(dt_tensor(dt, u0.device)),
                                                         fptr(_f32(v0)), fptr(_f32(u0)), *[C.cast(a, C.c_void_p) for a in arrs],
                                                         ptr(u), ptr(scratch), stream_ptr(u0.device)), "sph_finalize_compatible_energy")
    return u, scratch[:n]


def conservation_sums(params, m, v, u) -> torch.Tensor:
    out = torch.empty(7, device=m.device, dtype=torch.float64)
    check(_capi.lib().sph_conservation_sums(_p(params), m.shape[0], fptr(m), fptr(v), fptr(u), ptr(out), stream_ptr(m.device)),
          "sph_conservation_sums")
    return out


# ------------------------------------------------------------------ incompressible (DFSPH)
def dfsph_alpha(params, x, H, m, rho, adj: AdjacencyList) -> torch.Tensor:
    """computeAlpha (modules/incompressible/wp_alpha.py:294-313): the negative DFSPH diagonal."""
    out = _empty(m.shape[0], m)
    with _timed("dfsph_alpha"):
        check(_capi.lib().sph_dfsph_alpha(_p(params), m.shape[0], fptr(x), fptr(H), fptr(m), fptr(rho), *_lists(params, adj, True),
                                          ptr(out), stream_ptr(m.device)), "sph_dfsph_alpha")
    return out


def incompressible_divergence(params, rho0, x, H, m, rho, v, adj: AdjacencyList, dvdt=None, dt=None) -> torch.Tensor:
    """computeMomentumIncompressible (modules/momentum/incompressible.py:9-34) of v + dt*dvdt."""
    out = _empty(m.shape[0], m)
    dtt = None if dvdt is None else dt_tensor(dt, m.device)
    with _timed("incompressible_divergence"):
        check(_capi.lib().sph_incompressible_divergence(_p(params), m.shape[0], float(rho0), fptr(x), fptr(H), fptr(m), fptr(rho),
                                                        fptr(v), fptr(dvdt), ptr(dtt), *_lists(params, adj, True), ptr(out),
                                                        stream_ptr(m.device)), "sph_incompressible_divergence")
    return out


def pressure_accel_iisph(params, x, H, m, rho, pressure, adj: AdjacencyList) -> torch.Tensor:
    """computePressureAccelIISPH (modules/pressure/iisph.py:7-24)."""
    out = _empty((m.shape[0], int(params.dim)), m)
    with _timed("pressure_accel_iisph"):
        check(_capi.lib().sph_pressure_accel_iisph(_p(params), m.shape[0], fptr(x), fptr(H), fptr(m), fptr(rho), fptr(pressure),
                                                   *_lists(params, adj, True), ptr(out), stream_ptr(m.device)),
              "sph_pressure_accel_iisph")
    return out


def pressure_shift_iisph(params, x, H, m, rho, accel, adj: AdjacencyList) -> torch.Tensor:
    """computePressureShiftIISPH (modules/incompressible/drift.py:38-57)."""
    out = _empty(m.shape[0], m)
    with _timed("pressure_shift_iisph"):
        check(_capi.lib().sph_pressure_shift_iisph(_p(params), m.shape[0], fptr(x), fptr(H), fptr(m), fptr(rho), fptr(accel),
                                                   *_lists(params, adj, True), ptr(out), stream_ptr(m.device)),
              "sph_pressure_shift_iisph")
    return out


_jacobi_ws: dict = {}

DIVERGENCE_FREE = 0
DENSITY = 1


def jacobi_solve(params, mode: int, cfg, x, H, m, rho, v, dvdt, p_init, dt, adj: AdjacencyList):
    """One persistent-kernel relaxed Jacobi solve (mode DIVERGENCE_FREE or DENSITY).

    cfg is a _capi.SphJacobiConfig.  Returns device tensors
    (pressure [n], accel [n, dim], history [max_iterations, 4], iterations [1] int32,
    status [1] int32); nothing is synchronised."""
    n, d = m.shape[0], int(params.dim)
    ws = _jacobi_workspace(n, d, m.device)
    pr = _empty(n, m)
    acc = _empty((n, d), m)
    hist = torch.zeros((max(int(cfg.max_iterations), 1), 4), device=m.device, dtype=torch.float32)
    flags = torch.zeros(2, device=m.device, dtype=torch.int32)
    fn = _capi.lib().sph_dfsph_div_solve if mode == DIVERGENCE_FREE else _capi.lib().sph_dfsph_density_solve
    with _timed("dfsph_div_solve" if mode == DIVERGENCE_FREE else "dfsph_density_solve"):
        check(fn(_p(params), C.cast(C.pointer(cfg), C.c_void_p), n, fptr(x), fptr(H), fptr(m), fptr(rho), fptr(v), fptr(dvdt),
                 fptr(p_init), ptr(dt_tensor(dt, m.device)), *_lists(params, adj, True), ptr(ws), int(ws.numel()), ptr(pr), ptr(acc),
                 ptr(hist), ptr(flags), ptr(flags[1:]), stream_ptr(m.device)), "jacobi solve")
    return pr, acc, hist, flags[:1], flags[1:]


def _jacobi_workspace(n: int, d: int, device) -> torch.Tensor:
    key = (device.index, n)
    ws = _jacobi_ws.get(key)
    need = int(_capi.lib().sph_dfsph_workspace_size(n, d))
    if ws is None or ws.numel() < need:
        if len(_jacobi_ws) > 8:
            _jacobi_ws.clear()
        ws = torch.empty(need, dtype=torch.uint8, device=device)
        _jacobi_ws[key] = ws
    return ws


# ------------------------------------------------------------------ learned warm start
def dfsph_features(params, mode: int, cfg, x, H, m, rho, v, dvdt, p_prev, dt, adj: AdjacencyList):
    """The eight warm-start features of solve `mode` and the pressure scale P
    (feats [n, 8], scale [1]; device tensors, no sync)."""
    n, d = m.shape[0], int(params.dim)
    ws = _jacobi_workspace(n, d, m.device)
    feats = torch.empty((n, 8), device=m.device, dtype=torch.float32)
    scale = torch.empty(1, device=m.device, dtype=torch.float32)
    with _timed("dfsph_features"):
        check(_capi.lib().sph_dfsph_features(_p(params), C.cast(C.pointer(cfg), C.c_void_p), int(mode), n, fptr(x), fptr(H), fptr(m),
                                             fptr(rho), fptr(v), fptr(dvdt), fptr(p_prev), ptr(dt_tensor(dt, m.device)),
                                             *_lists(params, adj, True), ptr(ws), int(ws.numel()), ptr(feats), ptr(scale),
                                             stream_ptr(m.device)), "sph_dfsph_features")
    return feats, scale


_mlp_suspect: set = set()
_mlp_status: dict = {}


def mlp_status(device) -> torch.Tensor:
    """The device int32 word into which sph_mlp_forward_tc and sph_mlp_grad_tc or SPH_STATUS_TIMEOUT."""
    dev = torch.device(device)
    st = _mlp_status.get(dev.index)
    if st is None:
        st = torch.zeros(1, dtype=torch.int32, device=dev)
        _mlp_status[dev.index] = st
    return st


def check_mlp_status(device) -> None:
    """Reads the tcgen05 forward's status word (one host read).  A timeout means an MMA
    chain did not complete in about a second: its outputs are NaN and the device context is
    suspect, so this device's tensor-core forward refuses further launches (RuntimeError)."""
    dev = torch.device(device)
    if int(mlp_status(dev).item()) & 0x8:
        _mlp_suspect.add(dev.index)
        raise RuntimeError(f"tcgen05 MLP forward timed out on {dev}: the CUDA context is suspect; restart the process")


def mlp_forward(theta, feats, scale=None, tensor_cores: str = "tcgen05") -> torch.Tensor:
    """MLP(feats) * scale.  tensor_cores "tcgen05" runs sph_mlp_forward_tc (TMEM
    accumulators, 128-sample tiles); "mma" runs sph_mlp_forward (warp-level mma.sync)."""
    out = torch.empty(feats.shape[0], device=feats.device, dtype=torch.float32)
    f = feats.contiguous()
    if tensor_cores == "tcgen05":
        if f.device.index in _mlp_suspect:
            raise RuntimeError(f"tcgen05 MLP forward on {f.device}: an earlier launch timed out; the context is suspect")
        if f.data_ptr() % 16:
            f = f.clone()
        with _timed("mlp_forward"):
            check(_capi.lib().sph_mlp_forward_tc(fptr(theta), f.shape[0], fptr(f), ptr(scale), ptr(out), ptr(mlp_status(f.device)),
                                                 stream_ptr(f.device)), "sph_mlp_forward_tc")
    elif tensor_cores == "mma":
        with _timed("mlp_forward"):
            check(_capi.lib().sph_mlp_forward(fptr(theta), f.shape[0], fptr(f), ptr(scale), ptr(out), stream_ptr(f.device)),
                  "sph_mlp_forward")
    else:
        raise ValueError(f"tensor_cores must be 'tcgen05' or 'mma', not {tensor_cores!r}")
    return out


def mlp_grad(theta, feats, target, tensor_cores: str = "tcgen05"):
    """(grad [P] float32, loss [1] float64 = sum of squared errors) of the MSE.
    tensor_cores "tcgen05" runs sph_mlp_grad_tc (every GEMM on tcgen05, the weight
    gradients accumulated in TMEM); "mma" runs sph_mlp_grad (warp-level mma.sync)."""
    g = torch.empty_like(theta)
    loss = torch.empty(1, device=theta.device, dtype=torch.float64)
    f = feats.contiguous()
    t = target.contiguous()
    if tensor_cores == "tcgen05":
        if f.device.index in _mlp_suspect:
            raise RuntimeError(f"tcgen05 MLP gradient on {f.device}: an earlier launch timed out; the context is suspect")
        if f.data_ptr() % 16:
            f = f.clone()
        with _timed("mlp_grad"):
            check(_capi.lib().sph_mlp_grad_tc(fptr(theta), f.shape[0], fptr(f), fptr(t), ptr(g), ptr(loss), ptr(mlp_status(f.device)),
                                              stream_ptr(theta.device)), "sph_mlp_grad_tc")
    elif tensor_cores == "mma":
        with _timed("mlp_grad"):
            check(_capi.lib().sph_mlp_grad(fptr(theta), f.shape[0], fptr(f), fptr(t), ptr(g), ptr(loss), stream_ptr(theta.device)),
                  "sph_mlp_grad")
    else:
        raise ValueError(f"tensor_cores must be 'tcgen05' or 'mma', not {tensor_cores!r}")
    return g, loss


def mlp_adam(theta, grad, m1, m2, step: int, lr: float, beta1=0.9, beta2=0.999, eps=1e-8):
    check(_capi.lib().sph_mlp_adam(fptr(theta), fptr(grad), fptr(m1), fptr(m2), theta.numel(), float(lr), float(beta1),
                                   float(beta2), float(eps), int(step), stream_ptr(theta.device)), "sph_mlp_adam")


# ------------------------------------------------------------------ weakly compressible delta-SPH
def deltasph_rhs(params, wc, x, H, m, rho, v, adj: AdjacencyList, surface_mask=None):
    """One delta-SPH right-hand side: (dvdt [n, dim], drhodt [n], gradRhoL [n, dim], P [n]).
    surface_mask: the int32 free-surface indicators (None: no free surface)."""
    n, d = m.shape[0], int(params.dim)
    scratch = _empty(n * (d + 1), m)
    dvdt, drhodt = _empty((n, d), m), _empty(n, m)
    sm = None if surface_mask is None else surface_mask.to(torch.int32).contiguous()
    with _timed("deltasph_rhs"):
        check(_capi.lib().sph_deltasph_rhs(_p(params), C.cast(C.pointer(wc), C.c_void_p), n, fptr(x), fptr(H), fptr(m), fptr(rho),
                                           fptr(v), iptr(sm), *_lists(params, adj, True), ptr(scratch), ptr(dvdt), ptr(drhodt),
                                           stream_ptr(m.device)), "sph_deltasph_rhs")
    return dvdt, drhodt, scratch[: n * d].view(n, d), scratch[n * d:]


def wc_visc_continuity(params, wc, x, H, m, rho, v, adj: AdjacencyList):
    """Velocity diffusion and continuity of the DFSPH step: (dvdt_diss [n, dim], drhodt [n])."""
    n, d = m.shape[0], int(params.dim)
    dvdt, drhodt = _empty((n, d), m), _empty(n, m)
    with _timed("wc_visc_continuity"):
        check(_capi.lib().sph_wc_visc_continuity(_p(params), C.cast(C.pointer(wc), C.c_void_p), n, fptr(x), fptr(H), fptr(m), fptr(rho),
                                                 fptr(v), *_lists(params, adj, True), ptr(dvdt), ptr(drhodt), stream_ptr(m.device)),
              "sph_wc_visc_continuity")
    return dvdt, drhodt


def delta_shift(params, x, H, m, rho, v, kinds, adj: AdjacencyList, cfl: float, c0: float, R: float = 0.25, nexp: int = 4,
                rho0: float = 1.0) -> torch.Tensor:
    """One delta-plus shift [n, dim] (zero for kinds != 0; kinds may be None)."""
    n, d = m.shape[0], int(params.dim)
    out = _empty((n, d), m)
    scratch = torch.empty(2, dtype=torch.int32, device=m.device)
    k = None if kinds is None else kinds.to(torch.int32).contiguous()
    with _timed("delta_shift"):
        check(_capi.lib().sph_delta_shift(_p(params), n, fptr(x), fptr(H), fptr(m), fptr(rho), fptr(_f32(v)), iptr(k),
                                          *_lists(params, adj, True), float(cfl), float(c0), float(R), int(nexp), float(rho0),
                                          ptr(scratch), ptr(out), stream_ptr(m.device)), "sph_delta_shift")
    return out


def wc_eos(wc, rho) -> torch.Tensor:
    out = torch.empty_like(rho)
    check(_capi.lib().sph_wc_eos(C.cast(C.pointer(wc), C.c_void_p), rho.shape[0], fptr(rho), ptr(out), stream_ptr(rho.device)),
          "sph_wc_eos")
    return out


# ------------------------------------------------------------------ mDBC wall particles
def mdbc_density(params, x, H, m, rho, kinds, ghost_indices, ghost_offsets, adj: AdjacencyList, rest_density: float,
                 sound_speed: float, gravity=None, want_neighbors: bool = False):
    """computeMdbcDensity on the GPU: the densities with the wall particles' replaced
    (sph_mdbc_density).  adj is a list over every particle, ghosts included.  Returns the
    densities, and the ghosts' neighbour counts with want_neighbors."""
    n = m.shape[0]
    out = _empty(n, m)
    nb = torch.zeros(n, dtype=torch.int32, device=m.device) if want_neighbors else None
    g = None
    if gravity is not None:
        gv = [float(a) for a in gravity] + [0.0] * (3 - len(gravity))
        g = (C.c_double * 3)(*gv[:3])
    with _timed("mdbc_density"):
        check(_capi.lib().sph_mdbc_density(_p(params), n, fptr(x), fptr(H), fptr(m), fptr(rho), iptr(kinds.to(torch.int32).contiguous()),
                                           iptr(ghost_indices.to(torch.int32).contiguous()), fptr(_f32(ghost_offsets)),
                                           *_csr(adj), float(rest_density), float(sound_speed),
                                           None if g is None else C.cast(g, C.c_void_p), ptr(out), ptr(nb), stream_ptr(m.device)),
              "sph_mdbc_density")
    return (out, nb) if want_neighbors else out


def mdbc_nopen_shift(params, x, H, m, v, kinds, ghost_offsets, adj: AdjacencyList) -> torch.Tensor:
    """computeMdbcNoPenShift on the GPU: the no-penetration shift [n, dim] (zero for non-fluid)."""
    n, d = m.shape[0], int(params.dim)
    out = _empty((n, d), m)
    with _timed("mdbc_nopen_shift"):
        check(_capi.lib().sph_mdbc_nopen_shift(_p(params), n, fptr(x), fptr(H), fptr(m), fptr(_f32(v)), iptr(kinds.to(torch.int32).contiguous()),
                                               fptr(_f32(ghost_offsets)), *_csr(adj), ptr(out), stream_ptr(m.device)),
              "sph_mdbc_nopen_shift")
    return out
