"""Order 1 on the B200: grouped pencils of spectral elements.

Reference: the grouped order 1 of ``transport_prompt`` (``prompt.py:1020-1258``)
as the shower route calls it (``shower/api.py:36-44``: fused bands, pixel face
96, 192 ring nodes). Stage A (``compress``, ``prompt.py:1317-1402``) builds the
pencil table from the elements; stage B (``grouped_pencils_order1``,
``_prompt_numba.py:1750-2086``) evaluates the OMs. Both run in
``liblh_b200.so``; the host forms the small static tables (band constants,
acceptance monomials, ``exp(kappa edges)`` and ``interval_table``) once.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import _lib

__all__ = ["PromptSettings", "Order1Tables", "order1", "interval_table", "acceptance_monomials"]

GAUSS_NODES = 48


@dataclass(frozen=True)
class PromptSettings:
    """The fields of the reference's ``PromptConfig`` (``prompt.py:154-196``) the
    grouped order 1 reads, with the shower route's values."""
    cell_m: float = 0.5
    pixel_face: int = 96
    ring_nodes: int = 192
    path_step: float = 0.1
    path_step_tail: float = 0.25
    tail_exponent: float = 25.0
    direct_bins: int = 4
    max_path_nodes: int = 2048
    smoothing_factor: float = 6.0
    merge_theta_min: float = 2e-3
    merge_theta_ratio: float = 0.08
    merge_tau_ns: float = 0.5
    merge_log_r: float = 0.02
    screen: bool = False      # the coarse charge screen (compress_screen / screen_order1)
    parent_face: int = 0      # the screen's parent pixels per face edge

    @classmethod
    def of(cls, config, *, fused=True):
        """From a reference ``PromptConfig`` (fused units use the fused pixel/ring)."""
        return cls(cell_m=config.cell_m,
                   pixel_face=config.fused_pixel_face if fused else config.pixel_face,
                   ring_nodes=config.fused_ring_nodes if fused else config.ring_nodes,
                   path_step=config.path_step, path_step_tail=config.path_step_tail,
                   tail_exponent=config.tail_exponent, direct_bins=config.direct_bins,
                   max_path_nodes=config.max_path_nodes,
                   smoothing_factor=config.smoothing_factor,
                   merge_theta_min=config.merge_theta_min,
                   merge_theta_ratio=config.merge_theta_ratio,
                   merge_tau_ns=config.merge_tau_ns, merge_log_r=config.merge_log_r)

    def coarse(self):
        """The coarse charge screen (``prompt.py:1155-1160``, ``compress_screen``
        and ``screen_order1``, ``_prompt_screen.py:91-503``): 2 m cells, 24 ring
        nodes, 32-pixel faces under 8-pixel parents refined near each OM, merge
        ratio 0.3 and 2 ns, one path step inside and beyond the window."""
        from dataclasses import replace
        return replace(self, cell_m=2.0, pixel_face=32, ring_nodes=24, merge_theta_ratio=0.3,
                       merge_tau_ns=2.0, path_step_tail=self.path_step, screen=True,
                       parent_face=8)


def _ifuncs(z):
    """``I_k(z) = int_0^1 x^k e^{z x} dx``, k = 0, 1, 2 (``_prompt_numba.py:139-154``)."""
    if abs(z) < 1.0:
        out = []
        for j in range(3):
            value = 0.0
            for n in range(23, -1, -1):
                value = value * z + 1.0 / (math.factorial(n) * (n + j + 1.0))
            out.append(value)
        return out
    ez = math.exp(z)
    return [(ez - 1.0) / z, (ez * (z - 1.0) + 1.0) / (z * z),
            (ez * (z * z - 2.0 * z + 2.0) - 2.0) / (z * z * z)]


def interval_table(edges, kappa):
    """``I_k(kappa * width)`` per band and bin (``_prompt_numba.py:635-644``)."""
    width = np.diff(np.asarray(edges, float))
    return np.array([[_ifuncs(k * w) for w in width] for k in np.asarray(kappa, float)])


def acceptance_monomials(alpha):
    """``(coef, ipow, jpow, degree)`` of the Legendre acceptance (``prompt.py:380-399``)."""
    from math import comb
    alpha = np.asarray(alpha, float)
    series = alpha * (2 * np.arange(len(alpha)) + 1) / (4 * np.pi)
    power = np.polynomial.legendre.leg2poly(series)
    degree = len(power) - 1
    coef, ipow, jpow = [], [], []
    for k in range(degree + 1):
        for i in range(k + 1):
            coef.append(power[k] * comb(k, i))
            ipow.append(i)
            jpow.append(k - i)
    return np.asarray(coef, float), np.asarray(ipow), np.asarray(jpow), int(degree)


class Order1Tables:
    """Band constants, acceptance monomials, OMs and bin tables on the device."""

    def __init__(self, bands, g, monomials, positions_m, looks, areas_m2, edges, *,
                 settings=PromptSettings(), group_capacity=8192, compute_bins=True,
                 device="cuda"):
        import torch
        self.device = torch.device(device)
        dev = self.device
        self.settings = s = settings
        coef, ipow, jpow, degree = monomials
        positions = np.ascontiguousarray(np.atleast_2d(positions_m), float)
        self.n_om = n = len(positions)
        mus, mut, speed = (np.asarray(bands[k], float) for k in ("mus", "mut", "speed"))
        s0w, s2w = np.asarray(bands["s0w"], float), np.asarray(bands["s2w"], float)
        self.edges = edges = np.asarray(edges, float)
        kappa = -mut * speed
        eedge = np.exp(np.outer(kappa, edges))
        itab = interval_table(edges, kappa)
        gx, gw = np.polynomial.legendre.leggauss(GAUSS_NODES)
        gauss_tau, gauss_w = 0.25 * math.pi * (gx + 1.0), 0.25 * math.pi * gw
        self.theta_bins = 2 + int(math.log(math.pi / s.merge_theta_min)
                                  / math.log(1.0 + s.merge_theta_ratio))
        if not s.merge_log_r >= 710.0 / ((1 << 20) - 2):
            raise ValueError("grouped radius/angular resolution exceeds integer key range")

        def f64(x):
            return torch.tensor(np.ascontiguousarray(x, float), dtype=torch.float64, device=dev)

        def i32(x):
            return torch.tensor(np.ascontiguousarray(x, np.int32), dtype=torch.int32, device=dev)

        self._t = t = dict(
            pos=f64(positions), look=f64(np.atleast_2d(looks)),
            area=f64(np.broadcast_to(np.asarray(areas_m2, float), (n,))),
            mus=f64(mus), mut=f64(mut), speed=f64(speed), s0w=f64(s0w), s2w=f64(s2w),
            coef=f64(coef), ipow=i32(ipow), jpow=i32(jpow), edges=f64(edges), eedge=f64(eedge),
            itab=f64(itab), gauss_tau=f64(gauss_tau), gauss_w=f64(gauss_w))
        self.struct = _lib.Order1Config(
            n, t["pos"].data_ptr(), t["look"].data_ptr(), t["area"].data_ptr(), len(mus),
            t["mus"].data_ptr(), t["mut"].data_ptr(), t["speed"].data_ptr(), t["s0w"].data_ptr(),
            t["s2w"].data_ptr(), float(g), len(coef), t["coef"].data_ptr(), t["ipow"].data_ptr(),
            t["jpow"].data_ptr(), int(degree), len(edges), t["edges"].data_ptr(),
            t["eedge"].data_ptr(), t["itab"].data_ptr(), int(bool(compute_bins)),
            float(s.cell_m), int(s.pixel_face),
            int(s.ring_nodes), float(s.path_step), float(s.path_step_tail),
            float(s.tail_exponent), int(s.direct_bins), int(s.max_path_nodes),
            float(s.smoothing_factor), float(s.merge_theta_min), float(s.merge_theta_ratio),
            float(s.merge_tau_ns), float(s.merge_log_r), self.theta_bins, float(np.max(speed)),
            GAUSS_NODES, t["gauss_tau"].data_ptr(), t["gauss_w"].data_ptr(), int(group_capacity),
            int(bool(s.screen)), int(s.parent_face))
        self.compute_bins = bool(compute_bins)
        self._workspace = None

    def widened(self, group_capacity):
        """These tables with ``group_capacity`` group slots per OM (a power of two
        up to 2^20) and their own workspace: for steps whose pencils mix times
        (delayed light), which multiply the (tau, r, theta) groups per OM."""
        import copy
        view = copy.copy(self)
        st = _lib.Order1Config()
        _C.pointer(st)[0] = self.struct
        st.group_capacity = int(group_capacity)
        view.struct = st
        view._workspace = None
        return view

    def pencil_table(self, capacity):
        """A pencil table over this object's pooled buffer (grown when needed). Tables
        from the pool are valid until the next stage-A call on the same stream."""
        import torch
        need = int(capacity) * PencilTable.ROW
        if getattr(self, "_pencil_pool", None) is None or self._pencil_pool.numel() < need:
            self._pencil_pool = torch.empty(max(need, 1 << 22), dtype=torch.float64,
                                            device=self.device)
        cached = getattr(self, "_pool_table", None)
        if (cached is not None and cached.capacity == int(capacity)
                and cached._buffer.data_ptr() == self._pencil_pool.data_ptr()):
            return cached  # the same views of the same pool: no new table object
        table = PencilTable(capacity, self.device, self._pencil_pool[:need],
                            screen=self.settings.screen)
        table.pooled = True
        self._pool_table = table
        return table

    def workspace(self, n_subseg, n_work):
        import torch
        need = int(_lib.load().lh_order1_workspace_bytes(self.struct, int(n_subseg), int(n_work)))
        if need == 0:
            raise ValueError("order-1 configuration rejected by the device library")
        if self._workspace is None or self._workspace.numel() < need:
            self._workspace = torch.empty(need, dtype=torch.uint8, device=self.device)
        return self._workspace


class PencilTable:
    """Device pencil table (stage A output), one float64 buffer cut into its fields."""

    FIELDS = (("position", 3), ("direction", 3), ("w0", 1), ("w2", 1), ("time", 1),
              ("major", 3), ("var_major", 1), ("var_minor", 1), ("pos_cov", 6))
    ROW = sum(c for _, c in FIELDS)

    def __init__(self, capacity, device, buffer=None, *, screen=False):
        import torch
        self.capacity = int(capacity)
        if buffer is None:
            buffer = torch.empty(self.capacity * self.ROW, dtype=torch.float64, device=device)
        self.pooled = buffer is not None and buffer.numel() != self.capacity * self.ROW
        self.t = {}
        pos = 0
        for k, c in self.FIELDS:
            view = buffer[pos:pos + self.capacity * c]
            self.t[k] = view.view(self.capacity, c) if c > 1 else view
            pos += self.capacity * c
        self._buffer = buffer
        self.count = torch.zeros(1, dtype=torch.int32, device=device)
        # the screen's parent row of every child (-1 for parents)
        self.parent = (torch.empty(self.capacity, dtype=torch.int32, device=device) if screen
                       else None)
        self.struct = _lib.Order1PencilTable(self.capacity,
                                             *[self.t[k].data_ptr() for k, _ in self.FIELDS],
                                             self.parent.data_ptr() if screen else None)

    def host(self, n=None):
        n = int(self.count.item()) if n is None else n
        return {k: v[:n].cpu().numpy() for k, v in self.t.items()}

    @classmethod
    def from_host(cls, pencils, device):
        import torch
        n = len(pencils["w0"])
        table = cls(max(n, 1), device)
        for k, _ in cls.FIELDS:
            table.t[k][:n] = torch.as_tensor(np.asarray(pencils[k], float), device=device)
        table.count.fill_(n)
        return table, n


def _element(source, name):
    return source[name] if isinstance(source, dict) else getattr(source, name)


def element_box(elements):
    """Per-coordinate minima and maxima of the element starts and ends
    ``start + length * direction`` (``compress``'s cell grid, ``prompt.py:1317-1402``):
    ``(low, high)``, in one host pass of the library (minima and maxima are
    exact in any order)."""
    start = np.ascontiguousarray(_element(elements, "start_m"), float)
    direction = np.ascontiguousarray(_element(elements, "direction"), float)
    length = np.ascontiguousarray(_element(elements, "length_m"), float)
    if len(length) == 0:
        raise ValueError("element_box of no elements")
    low, high = np.empty(3), np.empty(3)
    _lib.check(_lib.load().lh_element_box(len(length), start.ctypes.data, direction.ctypes.data,
                                          length.ctypes.data, low.ctypes.data, high.ctypes.data),
               "lh_element_box")
    return low, high


def pencils(tables: Order1Tables, elements, cone_cos, *, stream=None, status=None,
            device_elements=None, capacity_full=False, box=None):
    """Stage A: ``compress`` of the elements with frozen cone cosines.

    ``device_elements``: the same elements already on the device (dict of
    tensors with the reference field names), read instead of uploading.
    ``box``: ``element_box(elements)`` when the caller has it already.
    """
    import torch
    dev = tables.device
    s = tables.settings
    start = np.ascontiguousarray(_element(elements, "start_m"), float)
    direction = np.ascontiguousarray(_element(elements, "direction"), float)
    length = np.asarray(_element(elements, "length_m"), float)
    n_el = len(length)
    a_step = 0.5 * s.cell_m
    # max(1, ceil(length / a_step)) sub-segments per element, their running totals
    offsets = np.empty(n_el + 1, np.int64)
    n_total = np.zeros(1, np.int64)
    length = np.ascontiguousarray(length, float)
    if _lib.load().lh_subsegment_offsets(n_el, length.ctypes.data, a_step, offsets.ctypes.data,
                                         n_total.ctypes.data):
        raise ValueError("element lengths must be finite and non-negative")
    n_sub = int(n_total[0])
    if n_el:
        lo_box, hi_box = element_box(elements) if box is None else box
        low = lo_box - s.cell_m
        high = hi_box + s.cell_m
        dims = np.ceil((high - low) / s.cell_m).astype(np.int64) + 1
    else:
        low, dims = np.zeros(3), np.ones(3, np.int64)
    if float(np.prod(dims.astype(float))) * 6 * s.pixel_face ** 2 >= 2.0 ** 62:
        raise ValueError("cell grid too large for 64-bit pencil keys; increase cell_m")

    def f64(x):
        return _lib.upload(x, torch.float64, dev)

    d = device_elements
    if d is None:
        keep = dict(start=f64(start), direction=f64(direction), length=f64(length),
                    c0=f64(_element(elements, "coefficient0")),
                    c2=f64(_element(elements, "coefficient2")),
                    t0=f64(_element(elements, "start_ns")), t1=f64(_element(elements, "end_ns")))
    else:
        keep = dict(start=d["start_m"], direction=d["direction"], length=d["length_m"],
                    c0=d["coefficient0"], c2=d["coefficient2"], t0=d["start_ns"],
                    t1=d["end_ns"])
    keep["cone"] = (cone_cos if isinstance(cone_cos, torch.Tensor) else f64(cone_cos)).contiguous()
    keep["off"] = _lib.upload(offsets, torch.int64, dev)
    el = _lib.Order1Elements(n_el, n_sub, keep["off"].data_ptr(), keep["start"].data_ptr(),
                             keep["direction"].data_ptr(), keep["length"].data_ptr(),
                             keep["c0"].data_ptr(), keep["c2"].data_ptr(), keep["cone"].data_ptr(),
                             keep["t0"].data_ptr(), keep["t1"].data_ptr(),
                             (C_DOUBLE3)(*low), (C_INT64_3)(*dims))
    nodes = max(n_sub * s.ring_nodes, 1)
    # Pencils are distinct (cell, pixel) keys: far fewer than ring nodes when many
    # elements share cells. A table that overflows is redone at the full bound.
    if s.screen:  # parents and children
        nodes *= 2
    # pooled tables in powers of two, so that showers of similar size reuse one
    capacity = (nodes if capacity_full
                else min(nodes, max(1 << 17, 1 << int(nodes // 4 - 1).bit_length())))
    table = (PencilTable(capacity, dev, screen=s.screen) if capacity_full
             else tables.pencil_table(capacity))
    if n_sub == 0:
        table.count.zero_()  # stage A writes no count for no elements (a reused table)
    ws = tables.workspace(n_sub, 0)
    st = status if status is not None else torch.zeros(1, dtype=torch.int32, device=dev)
    sp = _lib.stream_ptr(stream or torch.cuda.current_stream(dev))
    _lib.check(_lib.load().lh_order1_pencils(tables.struct, el, table.struct,
                                             table.count.data_ptr(), ws.data_ptr(), ws.numel(),
                                             st.data_ptr(), sp), "lh_order1_pencils")
    table._keep = keep
    table.nodes = nodes
    if status is None:
        flags = int(st.item())
        if flags & _lib.LH_STATUS_OVERFLOW and capacity < nodes:
            return pencils(tables, elements, cone_cos, stream=stream,
                           device_elements=device_elements, capacity_full=True, box=box)
        _raise(flags)
    return table


def grouped(tables: Order1Tables, table: "PencilTable", work, origins, *, n_pencils=None,
            stream=None, status=None):
    """Stage B: ``grouped_pencils_order1`` for the OMs ``work``: charge, bins (device)."""
    import torch
    dev = tables.device
    n = tables.n_om
    work = np.asarray(work, np.int32)
    # the count stays on the device unless the caller passes it
    n_p = table.capacity if n_pencils is None else min(int(n_pencils), table.capacity)
    count_ptr = table.count.data_ptr() if n_pencils is None else None
    if len(work) and (work.min() < 0 or work.max() >= n):
        raise ValueError("work lists OMs outside the detector")
    if np.shape(origins) != (n,):
        raise ValueError("time origins must hold one value per OM")
    work_t = _lib.upload(work, torch.int32, dev)
    origins_t = (origins.to(dev, torch.float64).contiguous() if isinstance(origins, torch.Tensor)
                 else _lib.upload(origins, torch.float64, dev))
    charge = torch.empty(n, dtype=torch.float64, device=dev)
    bins = (torch.empty((n, len(tables.edges) - 1), dtype=torch.float64, device=dev)
            if tables.compute_bins else None)
    ws = tables.workspace(0, len(work))
    st = status if status is not None else torch.zeros(1, dtype=torch.int32, device=dev)
    sp = _lib.stream_ptr(stream or torch.cuda.current_stream(dev))
    _lib.check(_lib.load().lh_order1_grouped(tables.struct, table.struct, n_p, count_ptr,
                                             work_t.data_ptr(), len(work), origins_t.data_ptr(),
                                             charge.data_ptr(),
                                             bins.data_ptr() if bins is not None else None,
                                             ws.data_ptr(),
                                             ws.numel(), st.data_ptr(), sp),
               "lh_order1_grouped")
    if status is None:
        _raise(int(st.item()))
    return charge, bins


MAX_GROUP_CAPACITY = 1 << 20


def grouped_widening(tables: Order1Tables, table, work, origins):
    """``grouped`` that retries with 4x larger group tables while they overflow
    (up to 2^20 slots per OM)."""
    capacity = int(tables.struct.group_capacity)
    current = tables
    while True:
        try:
            return grouped(current, table, work, origins)
        except MemoryError:
            capacity *= 4
            if capacity > MAX_GROUP_CAPACITY:
                raise
            current = tables.widened(capacity)


def order1(tables: Order1Tables, elements, cone_cos, origins, work=None):
    """Fine grouped order 1 (charge (OM,), bins (OM, bins)) of one element set."""
    table = pencils(tables, elements, cone_cos)
    work = np.arange(tables.n_om) if work is None else work
    return grouped(tables, table, work, origins)


def _raise(flags):
    if flags & _lib.LH_STATUS_OVERFLOW:
        raise MemoryError("order-1 tables overflowed their device capacity "
                          "(pencils, groups per OM or batch size)")


import ctypes as _C  # noqa: E402

C_DOUBLE3 = _C.c_double * 3
C_INT64_3 = _C.c_int64 * 3
