"""ctypes binding of ``liblh_b200.so`` (declarations in ``include/lighthit_b200.h``).

The library is the only compute path: there is no CPU fallback. Loading fails
loudly when it is missing; ``lighthit_b200.build`` compiles it in-tree.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "liblh_b200.so"

LH_OK, LH_EINVAL, LH_ECUDA, LH_ENOMEM, LH_ETIMEDOUT, LH_EUNSUPPORTED = 0, 1, 2, 3, 4, 5
LH_STATUS_COINCIDENT, LH_STATUS_UNSAFE, LH_STATUS_TIMEOUT = 1, 2, 4
LH_STATUS_ON_TRACK, LH_STATUS_INSIDE_GLASS, LH_STATUS_NEGATIVE_ACCEPTANCE = 8, 16, 32
LH_STATUS_OVERFLOW = 64
LH_MODE_PLAIN_FP32, LH_MODE_SPLIT_BF16, LH_MODE_BF16 = 0, 1, 2
MODES = {"fp32": LH_MODE_PLAIN_FP32, "split-bf16": LH_MODE_SPLIT_BF16, "bf16": LH_MODE_BF16}

_ERRORS = {LH_EINVAL: "invalid argument", LH_ECUDA: "CUDA launch failed",
           LH_ENOMEM: "workspace too small", LH_ETIMEDOUT: "device wait timed out",
           LH_EUNSUPPORTED: "unsupported shape"}

P = C.c_void_p


class ReadoutOperator(C.Structure):
    _fields_ = [("n_bins", C.c_int32), ("k_pad", C.c_int32), ("n_tile", C.c_int32),
                ("n_tiles", C.c_int32), ("b_fp32", P), ("b_hi", P), ("b_lo", P)]


class FlashProblem(C.Structure):
    _fields_ = [("n_om", C.c_int32), ("om_pos", P), ("om_look", P), ("om_area", P),
                ("acc_top", C.c_int32), ("alpha", P), ("efficiency", C.c_double),
                ("n_omega", C.c_int32), ("omega", P), ("n_radii", C.c_int32), ("log_r", P),
                ("coef", P), ("mu_a", C.c_double), ("mu_t", C.c_double), ("speed", C.c_double),
                ("origin_speed", C.c_double), ("r_low", C.c_double), ("r_high", C.c_double),
                ("threshold", C.c_double), ("n_edges", C.c_int32), ("edges", P)]


class FlashBatch(C.Structure):
    _fields_ = [("n_flash", C.c_int32), ("pos", P), ("photons", P), ("time_ns", P),
                ("spectrum", P), ("components", P), ("charge", P), ("origin", P),
                ("active", P), ("status", P), ("n_flash_device", P),
                ("block_threads", C.c_int32)]


class FlashNodes(C.Structure):
    _fields_ = [("n_nodes", C.c_int32), ("spectrum", P * 8), ("components", P * 8),
                ("charge", P * 8), ("photons", P * 8), ("efficiency", C.c_double * 8),
                ("absorption", C.c_double * 8)]


class Ge2Table(C.Structure):
    _fields_ = [("n_bands", C.c_int32), ("n_intervals", C.c_int32), ("degree", C.c_int32),
                ("acc_degree", C.c_int32), ("max_m", C.c_int32), ("n_pairs", C.c_int32),
                ("nch", C.c_int32), ("n_omega", C.c_int32), ("coef", P), ("log_r", P),
                ("absorption", P), ("speed", P), ("omega", P), ("pair_lambda", P),
                ("pair_mu", P), ("alpha", P), ("starts", P), ("start_norm", P),
                ("jmax", C.c_int32), ("flight", C.c_int32)]


class Ge2Problem(C.Structure):
    _fields_ = [("n_points", C.c_int32), ("points", P), ("channels", P),
                ("n_omega_channels", C.c_int32), ("n_omega", C.c_int32), ("n_om", C.c_int32),
                ("receivers", P), ("looks", P), ("out_scale", P), ("radial_low", C.c_double),
                ("radial_high", C.c_double), ("reference_ns", C.c_double), ("result", P)]


class WindowEvent(C.Structure):
    _fields_ = [("n_points", C.c_int32 * 8), ("capacity", C.c_int32), ("points", P),
                ("channels", P), ("channel_stride", C.c_int32), ("centre", C.c_double * 3),
                ("axis", C.c_double * 3), ("first", C.c_double * 3), ("second", C.c_double * 3)]


class RadialWindowProblem(C.Structure):
    _fields_ = [("n_om", C.c_int32), ("n_bands", C.c_int32), ("om_pos", P),
                ("radial_low", C.c_double), ("radial_high", C.c_double), ("n_att", C.c_int32),
                ("att_radius", P), ("att_log", P), ("photon_scale", C.c_double),
                ("efficiency", C.c_double * 8), ("n_near", P), ("n_far", P), ("far_sum", P)]


class Order0Optics(C.Structure):
    _fields_ = [("n_om", C.c_int32), ("om_pos", P), ("om_look", P), ("om_area", P),
                ("om_radius", P), ("n_alpha", C.c_int32), ("alpha", P),
                ("n_panel_edges", C.c_int32), ("panel_edges", P), ("phase", P), ("group", P),
                ("extinction", P), ("eff_cols", C.c_int32), ("efficiency", P),
                ("order", C.c_int32), ("gauss_x", P), ("gauss_w", P),
                ("check_order", C.c_int32), ("check_x", P), ("check_w", P)]


class Order0Batch(C.Structure):
    _fields_ = [("n_events", C.c_int32), ("element_offset", P), ("n_elements", C.c_int64),
                ("start", P), ("direction", P), ("length", P),
                ("c0", P), ("c2", P), ("beta", P), ("t0", P), ("t1", P), ("origins", P),
                ("n_edges", C.c_int32), ("edges", P), ("charge", P), ("bins", P),
                ("status", P), ("workspace", P), ("workspace_bytes", C.c_size_t),
                ("charge_check", P)]


class Order1Config(C.Structure):
    _fields_ = [("n_om", C.c_int32), ("om_pos", P), ("om_look", P), ("om_area", P),
                ("n_bands", C.c_int32), ("mus", P), ("mut", P), ("speed", P), ("s0w", P),
                ("s2w", P), ("g", C.c_double), ("n_mono", C.c_int32), ("coef", P), ("ipow", P),
                ("jpow", P), ("max_power", C.c_int32), ("n_edges", C.c_int32), ("edges", P),
                ("eedge", P), ("itab", P), ("compute_bins", C.c_int32), ("cell_m", C.c_double),
                ("pixel_face", C.c_int32), ("ring_nodes", C.c_int32), ("path_step", C.c_double),
                ("path_step_tail", C.c_double), ("tail_exponent", C.c_double),
                ("direct_bins", C.c_int32), ("max_path_nodes", C.c_int32),
                ("smoothing_factor", C.c_double), ("theta_lo", C.c_double),
                ("theta_ratio", C.c_double), ("tau_step", C.c_double), ("log_r_step", C.c_double),
                ("theta_bins", C.c_int32), ("speed_ref", C.c_double), ("n_gauss", C.c_int32),
                ("gauss_tau", P), ("gauss_w", P), ("group_capacity", C.c_int32),
                ("screen", C.c_int32), ("parent_face", C.c_int32)]


class Order1Elements(C.Structure):
    _fields_ = [("n_el", C.c_int32), ("n_subseg", C.c_int64), ("subseg_offset", P),
                ("start", P), ("direction", P), ("length", P), ("c0", P), ("c2", P),
                ("cone_cos", P), ("t0", P), ("t1", P), ("grid_origin", C.c_double * 3),
                ("grid_dims", C.c_int64 * 3)]


class Order1PencilTable(C.Structure):
    _fields_ = [("capacity", C.c_int32), ("position", P), ("direction", P), ("w0", P), ("w2", P),
                ("time", P), ("major", P), ("var_major", P), ("var_minor", P), ("pos_cov", P),
                ("parent", P)]


class SourceProblem(C.Structure):
    _fields_ = [("n_el", C.c_int32), ("start", P), ("direction", P), ("length", P), ("c0", P),
                ("c2", P), ("beta", P), ("t0", P), ("t1", P), ("n_bands", C.c_int32),
                ("band_s0", C.c_double * 8), ("band_s2", C.c_double * 8),
                ("band_phase", C.c_double * 8), ("band_scale", C.c_double * 8),
                ("centre", C.c_double * 3), ("first", C.c_double * 3), ("second", C.c_double * 3),
                ("axis", C.c_double * 3), ("degree", C.c_int32), ("max_m", C.c_int32),
                ("nch", C.c_int32), ("starts", C.c_int32 * 18), ("channel_degree", C.c_int32 * 153),
                ("aa", C.c_double * 85), ("bb", C.c_double * 85), ("element_order", C.c_int32),
                ("node_fraction", C.c_double * 2), ("node_weight", C.c_double * 2),
                ("cell_m", C.c_double), ("stencil_m", C.c_double),
                ("stencil_threshold_m", C.c_double), ("time_step_ns", C.c_double),
                ("reference_ns", C.c_double), ("z_origin", C.c_double), ("n_slices", C.c_int64),
                ("kmax", C.c_int64), ("n_omega", C.c_int32), ("omega", P)]


class SourceOutput(C.Structure):
    _fields_ = [("capacity", C.c_int64), ("points", P), ("channels", P), ("n_points", P)]


class OmGeometry(C.Structure):
    _fields_ = [("n_om", C.c_int32), ("om_pos", P), ("n_events", C.c_int32),
                ("element_offset", P), ("start", P), ("direction", P), ("length", P),
                ("start_ns", P), ("group_index", C.c_double), ("min_distance", P),
                ("earliest_ns", P)]


class NearTable(C.Structure):
    _fields_ = [("n_lambda", C.c_int32), ("degree", C.c_int32), ("acc_degree", C.c_int32),
                ("n_pairs", C.c_int32), ("n_omega", C.c_int32), ("coef", P),
                ("log_r0", C.c_double), ("log_r1", C.c_double), ("radial_high", C.c_double),
                ("absorption", P), ("speed", P), ("omega", P), ("pair_lambda", P),
                ("pair_mu", P), ("alpha", P), ("start_norm", P), ("flight", C.c_int32),
                ("wavelength_nm", P), ("phase_index", P), ("spectral_weight", P),
                ("gauss_order", C.c_int32), ("gauss_x", P), ("gauss_w", P),
                ("panel_m", C.c_double)]


class NearProblem(C.Structure):
    _fields_ = [("n_om", C.c_int32), ("om_pos", P), ("om_look", P), ("om_area", P),
                ("time_origin_ns", P), ("n_elements", C.c_int32), ("start_m", P),
                ("direction", P), ("length_m", P), ("coefficient0", P), ("coefficient2", P),
                ("beta", P), ("start_ns", P), ("end_ns", P), ("radius_m", C.c_double),
                ("spectrum", P), ("charge", P), ("portions", P)]


# name -> (restype, argtypes); every symbol the header declares
SIGNATURES = {
    "lh_version": (C.c_char_p, []),
    "lh_readout_packed_bytes": (C.c_size_t, [C.POINTER(ReadoutOperator), C.c_int, C.c_int64]),
    "lh_readout_pack": (C.c_int, [C.POINTER(ReadoutOperator), C.c_int, P, C.c_int32, C.c_int64,
                                  P, P]),
    "lh_readout_rows": (C.c_int, [C.POINTER(ReadoutOperator), C.c_int, P, C.c_int64, P,
                                  C.c_int64, P, P]),
    "lh_flash_workspace_bytes": (C.c_size_t, [C.POINTER(FlashProblem),
                                              C.POINTER(ReadoutOperator), C.c_int, C.c_int32]),
    "lh_flash_transport": (C.c_int, [C.POINTER(FlashProblem), C.POINTER(ReadoutOperator), C.c_int,
                                     C.POINTER(FlashBatch), P, C.c_size_t, P]),
    "lh_flash_transport_noalloc": (C.c_int, [C.POINTER(FlashProblem), C.POINTER(ReadoutOperator),
                                             C.POINTER(FlashBatch), P]),
    "lh_kernel_timing": (C.c_int, [C.c_int]),
    "lh_kernel_timing_read": (C.c_int, [C.c_int32, P, P]),
    "lh_kernel_units_read": (C.c_int, [C.c_int32, P]),
    "lh_axis_frame_sums": (C.c_int, [C.c_int64, P, P, P, P, P, P]),
    "lh_element_box": (C.c_int, [C.c_int64, P, P, P, P, P]),
    "lh_element_delays": (C.c_int, [C.c_int64, P, P, C.c_int64, C.c_double, P, P]),
    "lh_subsegment_offsets": (C.c_int, [C.c_int64, P, C.c_double, P, P]),
    "lh_flash_combine": (C.c_int, [C.POINTER(FlashProblem), C.POINTER(FlashNodes),
                                   C.POINTER(FlashBatch), P]),
    "lh_ge2_workspace_bytes": (C.c_size_t, [C.POINTER(Ge2Table), C.POINTER(Ge2Problem)]),
    "lh_ge2_apply": (C.c_int, [C.POINTER(Ge2Table), C.POINTER(Ge2Problem), P, C.c_size_t, P]),
    "lh_window_slot_bytes": (C.c_size_t, [C.c_int32]),
    "lh_radial_window": (C.c_int, [C.POINTER(RadialWindowProblem), C.POINTER(WindowEvent),
                                   C.c_int32, P, C.c_size_t, P]),
    "lh_ge2_batch_workspace_bytes": (C.c_size_t, [C.POINTER(Ge2Table), C.POINTER(Ge2Problem),
                                                  C.c_int32]),
    "lh_ge2_batch_slot_bytes": (C.c_size_t, [C.c_int32]),
    "lh_ge2_apply_batch": (C.c_int, [C.POINTER(Ge2Table), C.POINTER(Ge2Problem), C.c_int32, P,
                                     C.c_size_t, P, P]),
    "lh_ge2_tc_pack_bytes": (C.c_size_t, [C.POINTER(Ge2Table)]),
    "lh_ge2_tc_pack": (C.c_int, [C.POINTER(Ge2Table), P, C.c_size_t, P]),
    "lh_ge2_tc_workspace_bytes": (C.c_size_t, [C.POINTER(Ge2Table), C.POINTER(Ge2Problem),
                                               C.c_int32]),
    "lh_ge2_apply_batch_tc": (C.c_int, [C.POINTER(Ge2Table), C.POINTER(Ge2Problem), C.c_int32,
                                        C.c_int32, P, P, C.c_size_t, P, P, P]),
    "lh_order0_workspace_bytes": (C.c_size_t, [C.POINTER(Order0Optics), C.POINTER(Order0Batch)]),
    "lh_order0": (C.c_int, [C.POINTER(Order0Optics), C.POINTER(Order0Batch), P]),
    "lh_order1_workspace_bytes": (C.c_size_t, [C.POINTER(Order1Config), C.c_int64, C.c_int32]),
    "lh_order1_pencils": (C.c_int, [C.POINTER(Order1Config), C.POINTER(Order1Elements),
                                    C.POINTER(Order1PencilTable), P, P, C.c_size_t, P, P]),
    "lh_order1_grouped": (C.c_int, [C.POINTER(Order1Config), C.POINTER(Order1PencilTable),
                                    C.c_int32, P, P, C.c_int32, P, P, P, P, C.c_size_t, P, P]),
    "lh_om_geometry": (C.c_int, [C.POINTER(OmGeometry), P]),
    "lh_source_workspace_bytes": (C.c_size_t, [C.POINTER(SourceProblem)]),
    "lh_source_compile": (C.c_int, [C.POINTER(SourceProblem), C.POINTER(SourceOutput), P,
                                    C.c_size_t, P, P]),
    "lh_near_workspace_bytes": (C.c_size_t, [C.POINTER(NearTable), C.POINTER(NearProblem)]),
    "lh_near_field": (C.c_int, [C.POINTER(NearTable), C.POINTER(NearProblem), P, C.c_size_t, P]),
    "lh_wait_selftest": (C.c_int, [P, C.c_int64, P]),
}
LH_ESCRATCH = 6
# kernel ids of lh_kernel_timing_read
TIMED_KERNELS = ("order0_kernel", "o1_ring_kernel", "o1_group_kernel", "o1_batch_kernel",
                 "ge2_apply_batch_kernel", "src_group_kernel", "src_transform_kernel",
                 "readout_tc_kernel", "flash_tc_kernel", "ge2_tc_kernel")

_lib = None


def load():
    """Load the library once and bind every declared symbol."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with "
                               "`python -m lighthit_b200.build` (nvcc, sm_100a)")
        lib = C.CDLL(str(LIB_PATH))
        for name, (restype, argtypes) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
    return _lib


def check(rc, what):
    if rc != LH_OK:
        raise RuntimeError(f"{what}: {_ERRORS.get(rc, 'error')} (code {rc})")


def ptr(tensor):
    """Device address of a contiguous torch tensor (None -> NULL)."""
    if tensor is None:
        return None
    if not tensor.is_contiguous():
        raise ValueError("tensor must be contiguous")
    return C.c_void_p(tensor.data_ptr())


def upload(array, dtype, device):
    """Host array -> device tensor without waiting for the device: staged through
    pinned memory and copied asynchronously on the current stream (a pageable copy
    would first drain every kernel queued on the stream)."""
    import numpy as np
    import torch
    np_dtype = {torch.float64: np.float64, torch.int32: np.int32, torch.int64: np.int64,
                torch.complex128: np.complex128, torch.complex64: np.complex64,
                torch.float32: np.float32}[dtype]
    if torch.device(device).type != "cuda":
        return torch.from_numpy(np.array(array, dtype=np_dtype, copy=True)).to(device)
    array = np.asarray(array)
    host = torch.empty(array.shape, dtype=dtype, pin_memory=True)
    host.numpy()[...] = array  # one conversion copy straight into pinned memory
    return host.to(device, non_blocking=True)


def upload_parts(parts, dtype, device):
    """Several host arrays -> one flat device tensor (their raveled concatenation)
    through one pinned buffer and one asynchronous copy; returns it and the offsets."""
    import numpy as np
    import torch
    sizes = [int(np.size(a)) for a in parts]
    offsets = np.zeros(len(parts) + 1, np.int64)
    offsets[1:] = np.cumsum(sizes)
    host = torch.empty(int(offsets[-1]), dtype=dtype, pin_memory=torch.device(device).type == "cuda")
    flat = host.numpy()
    for a, lo, hi in zip(parts, offsets[:-1], offsets[1:]):
        flat[lo:hi] = np.ravel(a)
    return host.to(device, non_blocking=True), offsets


def fetch(tensors):
    """Device tensors -> host NumPy arrays with one wait: each is copied into
    pinned memory asynchronously on the current stream, then the stream is
    synchronised once (instead of one blocking read per tensor)."""
    import torch
    hosts = []
    for t in tensors:
        h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
        h.copy_(t, non_blocking=True)
        hosts.append(h)
    if hosts:
        torch.cuda.current_stream(tensors[0].device).synchronize()
    return [h.numpy() for h in hosts]


def stream_ptr(stream):
    return C.c_void_p(stream.cuda_stream) if stream is not None else None


def kernel_timing(enable=True):
    """Start (clearing the record) or stop the library's kernel timing."""
    check(load().lh_kernel_timing(int(bool(enable))), "lh_kernel_timing")


def kernel_times():
    """``{kernel: (launches, total_ms)}`` of the timed launches since the last read."""
    import numpy as np
    n = len(TIMED_KERNELS)
    launches = np.zeros(n, np.int64)
    total = np.zeros(n)
    check(load().lh_kernel_timing_read(n, launches.ctypes.data, total.ctypes.data),
          "lh_kernel_timing_read")
    return {name: (int(launches[k]), float(total[k])) for k, name in enumerate(TIMED_KERNELS)
            if launches[k]}


def kernel_units():
    """``{kernel: units}`` of algorithmic work counted on the device since the
    timing was last started ((OM, pencil) evaluations of ``o1_group_kernel``,
    integrand nodes of ``order0_kernel``, in-window (OM, point) pairs of the
    tensor-core >=2 contraction)."""
    import numpy as np
    n = len(TIMED_KERNELS)
    units = np.zeros(n, np.int64)
    check(load().lh_kernel_units_read(n, units.ctypes.data), "lh_kernel_units_read")
    return {name: int(units[k]) for k, name in enumerate(TIMED_KERNELS) if units[k]}
