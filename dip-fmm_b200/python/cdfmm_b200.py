"""ctypes binding of the B200 evaluator's C ABI (include/cdfmm_b200.h).

This is the thin FFI a host program uses when it talks to the evaluator
without the C++ layer (the pybind11 `cdfmm` module goes through
libcdfmm.so -> libcdfmm_b200.so instead).  Arrays are numpy (host memory) or
anything exposing `data_ptr()` (e.g. torch CUDA tensors, device memory).

The library must have been built (`make -C dip-fmm_b200`); importing this
module raises if it is missing -- there is no fallback implementation.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, "..", "lib", "libcdfmm_b200.so")

OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_RUNTIME = 2
ERR_OUT_OF_MEMORY = 3
ERR_LOGIC = 4
ERR_NO_DEVICE = 5
ERR_TIMEOUT = 6

OUTPUT_POTENTIAL = 1
OUTPUT_FIELD = 2
M2L_AUTO, M2L_FP32, M2L_BF16X3 = 0, 1, 2
MOMENTS_ON_HOST = 1
RESULTS_ON_HOST = 2
LAYOUT_SEPARATE = 0
LAYOUT_INTERLEAVED = 1
SCHEDULE_AUTO, SCHEDULE_SEPARATE, SCHEDULE_CORUN = 0, 1, 2
NEAR_AUTO, NEAR_FP32, NEAR_TF32X3 = 0, 1, 2

EXPORTED = (
    "cdfmm_b200_device_count", "cdfmm_b200_device_info", "cdfmm_b200_plan_create",
    "cdfmm_b200_plan_destroy", "cdfmm_b200_set_self_indices", "cdfmm_b200_evaluate",
    "cdfmm_b200_read_expansions", "cdfmm_b200_set_timing", "cdfmm_b200_get_stats",
    "cdfmm_b200_direct_fp64", "cdfmm_b200_m2l_matrix", "cdfmm_b200_last_error",
    "cdfmm_b200_evaluate_noalloc", "cdfmm_b200_backward", "cdfmm_b200_batch_create",
    "cdfmm_b200_batch_launch", "cdfmm_b200_batch_destroy", "cdfmm_b200_direct_grad_fp64",
    "cdfmm_b200_selftest_bounded_wait", "cdfmm_b200_m2l_shapes", "cdfmm_b200_set_m2l_shape",
    "cdfmm_b200_poll_status", "cdfmm_b200_set_wait_limit", "cdfmm_b200_set_schedule", "cdfmm_b200_batch_groups",
    "cdfmm_b200_plan_create_from_points", "cdfmm_b200_plan_tree", "cdfmm_b200_m2l_stencil",
    "cdfmm_b200_set_source_cuboids", "cdfmm_b200_set_near_mode", "cdfmm_b200_m2l_traceless",
)

ROOT_CENTRE, ROOT_HALF_WIDTH = 1, 2

# Scratch capacity of cdfmm_b200_evaluate_noalloc (bytes).
NOALLOC_SCRATCH_BYTES = 64 << 20


class PlanDesc(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_int32), ("n_sources", ctypes.c_int32), ("n_targets", ctypes.c_int32),
        ("order", ctypes.c_int32), ("depth", ctypes.c_int32), ("max_states", ctypes.c_int32),
        ("m2l_mode", ctypes.c_int32), ("device", ctypes.c_int32),
        ("root_centre", ctypes.c_double * 3), ("root_half_width", ctypes.c_double),
        ("sorted_source_positions", ctypes.c_void_p), ("sorted_target_positions", ctypes.c_void_p),
        ("source_permutation", ctypes.c_void_p), ("target_permutation", ctypes.c_void_p),
        ("leaf_source_offsets", ctypes.c_void_p), ("leaf_target_offsets", ctypes.c_void_p),
    ]


class PointsDesc(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_int32), ("n_sources", ctypes.c_int32), ("n_targets", ctypes.c_int32),
        ("order", ctypes.c_int32), ("depth", ctypes.c_int32), ("max_states", ctypes.c_int32),
        ("m2l_mode", ctypes.c_int32), ("device", ctypes.c_int32), ("root_flags", ctypes.c_int32),
        ("positions_on_host", ctypes.c_int32),
        ("root_centre", ctypes.c_double * 3), ("root_half_width", ctypes.c_double),
        ("source_positions", ctypes.c_void_p), ("target_positions", ctypes.c_void_p),
        ("self_map", ctypes.c_int32), ("reserved0", ctypes.c_int32),
    ]


class EvalArgs(ctypes.Structure):
    _fields_ = [
        ("moments", ctypes.c_void_p), ("moments_dtype", ctypes.c_int32), ("n_states", ctypes.c_int32),
        ("output", ctypes.c_uint32), ("layout", ctypes.c_int32), ("field", ctypes.c_void_p),
        ("potential", ctypes.c_void_p), ("memory", ctypes.c_uint32), ("stream", ctypes.c_void_p),
        ("synchronize", ctypes.c_int32),
    ]


class BackwardArgs(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_int32), ("n_states", ctypes.c_int32), ("grad_field", ctypes.c_void_p),
        ("moments", ctypes.c_void_p), ("moments_dtype", ctypes.c_int32), ("grad_moments", ctypes.c_void_p),
        ("grad_target_positions", ctypes.c_void_p), ("memory", ctypes.c_uint32), ("stream", ctypes.c_void_p),
        ("synchronize", ctypes.c_int32), ("forward_evaluation", ctypes.c_uint64),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("persistent_device_bytes", ctypes.c_uint64), ("setup_h2d_bytes", ctypes.c_uint64),
        ("evaluation_h2d_bytes", ctypes.c_uint64), ("evaluation_d2h_bytes", ctypes.c_uint64),
        ("evaluation_h2d_calls", ctypes.c_uint64), ("evaluation_d2h_calls", ctypes.c_uint64),
        ("evaluations", ctypes.c_uint64), ("m2l_classes", ctypes.c_uint64),
        ("m2l_interactions", ctypes.c_uint64), ("m2l_matrix_bytes", ctypes.c_uint64),
        ("p2p_pairs", ctypes.c_uint64), ("kernel_launches_last", ctypes.c_uint64),
        ("m2l_mode_resolved", ctypes.c_int32), ("timing_enabled", ctypes.c_int32),
        ("m2l_tc_m_tiles", ctypes.c_int32), ("m2l_tc_stages", ctypes.c_int32),
        ("backward_reused_forward", ctypes.c_int32), ("m2l_tc_fused", ctypes.c_int32),
        ("ms_gather", ctypes.c_double), ("ms_p2m", ctypes.c_double), ("ms_m2m", ctypes.c_double),
        ("ms_m2l", ctypes.c_double), ("ms_l2l", ctypes.c_double), ("ms_l2p", ctypes.c_double),
        ("ms_p2p", ctypes.c_double), ("ms_total", ctypes.c_double),
        ("trace_p2p_begin", ctypes.c_double), ("trace_p2p_end", ctypes.c_double),
        ("trace_far_begin", ctypes.c_double), ("trace_m2l_begin", ctypes.c_double),
        ("trace_far_end", ctypes.c_double), ("trace_end", ctypes.c_double),
        ("schedule_last", ctypes.c_int32), ("near_tc_last", ctypes.c_int32),
        ("setup_ms_tree", ctypes.c_double), ("setup_ms_geometry", ctypes.c_double),
        ("setup_ms_near", ctypes.c_double), ("setup_ms_operators", ctypes.c_double),
        ("setup_ms_statistics", ctypes.c_double), ("setup_ms_buffers", ctypes.c_double),
        ("setup_ms_m2l", ctypes.c_double), ("setup_ms_total", ctypes.c_double),
        ("near_tc_k_cols", ctypes.c_uint64),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class CdfmmError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"[{code}] {message}")
        self.code = code


_lib = None


def library() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    path = os.path.abspath(LIBRARY_PATH)
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `make -C dip-fmm_b200`")
    lib = ctypes.CDLL(path)
    vp, i32, u64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_size_t
    lib.cdfmm_b200_device_count.argtypes = [ctypes.POINTER(i32)]
    lib.cdfmm_b200_device_info.argtypes = [i32, ctypes.c_char_p, u64, ctypes.POINTER(i32), ctypes.POINTER(i32)]
    lib.cdfmm_b200_plan_create.argtypes = [ctypes.POINTER(PlanDesc), ctypes.POINTER(vp)]
    lib.cdfmm_b200_plan_create_from_points.argtypes = [ctypes.POINTER(PointsDesc), ctypes.POINTER(vp)]
    lib.cdfmm_b200_plan_tree.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp]
    lib.cdfmm_b200_m2l_stencil.argtypes = [i32, vp, u64, ctypes.POINTER(i32)]
    lib.cdfmm_b200_m2l_traceless.argtypes = [i32, vp, vp, vp, vp, vp, vp, vp]
    lib.cdfmm_b200_set_source_cuboids.argtypes = [vp, vp, i32, i32]
    lib.cdfmm_b200_plan_destroy.argtypes = [vp]
    lib.cdfmm_b200_plan_destroy.restype = None
    lib.cdfmm_b200_set_self_indices.argtypes = [vp, vp]
    lib.cdfmm_b200_evaluate.argtypes = [vp, ctypes.POINTER(EvalArgs)]
    lib.cdfmm_b200_evaluate_noalloc.argtypes = [vp, ctypes.POINTER(EvalArgs)]
    lib.cdfmm_b200_backward.argtypes = [vp, ctypes.POINTER(BackwardArgs)]
    lib.cdfmm_b200_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(EvalArgs), i32, ctypes.POINTER(vp)]
    lib.cdfmm_b200_batch_launch.argtypes = [vp, vp, i32]
    lib.cdfmm_b200_batch_groups.argtypes = [vp, ctypes.POINTER(i32), i32]
    lib.cdfmm_b200_batch_destroy.argtypes = [vp]
    lib.cdfmm_b200_batch_destroy.restype = None
    lib.cdfmm_b200_read_expansions.argtypes = [vp, i32, i32, vp, u64]
    lib.cdfmm_b200_set_timing.argtypes = [vp, i32]
    lib.cdfmm_b200_set_schedule.argtypes = [vp, i32]
    lib.cdfmm_b200_set_near_mode.argtypes = [vp, i32]
    lib.cdfmm_b200_m2l_shapes.argtypes = [vp, ctypes.POINTER(i32), i32]
    lib.cdfmm_b200_set_m2l_shape.argtypes = [vp, i32, i32, i32]
    lib.cdfmm_b200_get_stats.argtypes = [vp, ctypes.POINTER(Stats)]
    lib.cdfmm_b200_direct_fp64.argtypes = [i32, i32, vp, vp, i32, vp, vp, vp, vp]
    lib.cdfmm_b200_direct_grad_fp64.argtypes = [i32, i32, vp, vp, i32, vp, vp, vp, vp]
    lib.cdfmm_b200_selftest_bounded_wait.argtypes = [i32]
    lib.cdfmm_b200_poll_status.argtypes = [vp]
    lib.cdfmm_b200_set_wait_limit.argtypes = [vp, ctypes.c_int64]
    lib.cdfmm_b200_m2l_matrix.argtypes = [i32, vp, vp, u64]
    lib.cdfmm_b200_last_error.argtypes = [vp]
    lib.cdfmm_b200_last_error.restype = ctypes.c_char_p
    _lib = lib
    return lib


def _check(code, plan=None):
    if code != OK:
        msg = library().cdfmm_b200_last_error(plan).decode()
        if code == ERR_INVALID_ARGUMENT:
            raise ValueError(msg)
        raise CdfmmError(code, msg)


def _ptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return ctypes.c_void_p(a.ctypes.data)


def device_count() -> int:
    c = ctypes.c_int32(0)
    _check(library().cdfmm_b200_device_count(ctypes.byref(c)))
    return int(c.value)


def m2l_matrix(order: int, R) -> np.ndarray:
    """(n, n) FP64 matrix [beta, alpha] = D^{alpha+beta} G(R), as generated by the plan."""
    n = (order + 1) * (order + 2) * (order + 3) // 6
    out = np.zeros(n * n)
    Rv = np.ascontiguousarray(R, dtype=np.float64)
    _check(library().cdfmm_b200_m2l_matrix(order, _ptr(Rv), _ptr(out), out.size))
    return out.reshape(n, n).T.copy()


STENCIL_COMPUTED, STENCIL_PROCESS, STENCIL_DISK = 0, 1, 2


def m2l_stencil(order: int):
    """The 343 normalised M2L matrices of `order` as plans use them,
    (343, n, n) FP64, and where they came from (STENCIL_*): computed, this
    process's cache, or the CDFMM_B200_OPERATOR_CACHE directory."""
    n = (order + 1) * (order + 2) * (order + 3) // 6
    out = np.zeros((343, n, n))
    src = ctypes.c_int32(-1)
    _check(library().cdfmm_b200_m2l_stencil(order, _ptr(out), out.size, ctypes.byref(src)))
    return out, src.value


def m2l_traceless(order: int) -> dict:
    """The traceless reduction the M2L applies at `order`
    (cdfmm_b200_m2l_traceless): full ranks of the folded moments ("in") and
    of the computed locals ("out"), the fold as CSR ("fold_offsets",
    "fold_ranks", "fold_coefficients") and the derived locals as rows
    (d, s1, s2) with L_d = -(L_s1 + L_s2), in evaluation order."""
    counts = np.zeros(4, dtype=np.int32)
    _check(library().cdfmm_b200_m2l_traceless(order, _ptr(counts), None, None, None, None, None, None))
    n_in, n_out, nnz, nd = (int(c) for c in counts)
    out = {"in": np.zeros(n_in, np.int32), "out": np.zeros(n_out, np.int32),
           "fold_offsets": np.zeros(n_in + 1, np.int32), "fold_ranks": np.zeros(max(nnz, 1), np.int32),
           "fold_coefficients": np.zeros(max(nnz, 1), np.int32), "derived": np.zeros((max(nd, 1), 3), np.int32)}
    _check(library().cdfmm_b200_m2l_traceless(order, _ptr(counts), _ptr(out["in"]), _ptr(out["out"]),
                                              _ptr(out["fold_offsets"]), _ptr(out["fold_ranks"]),
                                              _ptr(out["fold_coefficients"]), _ptr(out["derived"])))
    out["fold_ranks"] = out["fold_ranks"][:nnz]
    out["fold_coefficients"] = out["fold_coefficients"][:nnz]
    out["derived"] = out["derived"][:nd]
    return out


def direct_fp64(sources, moments, targets, self_indices=None, device=0):
    """FP64 direct sum on the device; returns (phi, H)."""
    s = np.ascontiguousarray(sources, dtype=np.float64).reshape(-1, 3)
    m = np.ascontiguousarray(moments, dtype=np.float64).reshape(-1, 3)
    t = np.ascontiguousarray(targets, dtype=np.float64).reshape(-1, 3)
    ids = None if self_indices is None else np.ascontiguousarray(self_indices, dtype=np.int32)
    phi = np.zeros(len(t))
    H = np.zeros((len(t), 3))
    _check(library().cdfmm_b200_direct_fp64(device, len(s), _ptr(s), _ptr(m), len(t), _ptr(t), _ptr(ids),
                                            _ptr(phi), _ptr(H)))
    return phi, H


def direct_grad_fp64(sources, moments, targets, weights, self_indices=None, device=0):
    """FP64 direct position gradient d/dx_i (w_i . H_i) on the device; (nt, 3)."""
    s = np.ascontiguousarray(sources, dtype=np.float64).reshape(-1, 3)
    m = np.ascontiguousarray(moments, dtype=np.float64).reshape(-1, 3)
    t = np.ascontiguousarray(targets, dtype=np.float64).reshape(-1, 3)
    w = np.ascontiguousarray(weights, dtype=np.float64).reshape(-1, 3)
    ids = None if self_indices is None else np.ascontiguousarray(self_indices, dtype=np.int32)
    g = np.zeros((len(t), 3))
    _check(library().cdfmm_b200_direct_grad_fp64(device, len(s), _ptr(s), _ptr(m), len(t), _ptr(t), _ptr(ids),
                                                 _ptr(w), _ptr(g)))
    return g


class DevicePlan:
    """One fixed geometry on the device (cdfmm_b200_plan)."""

    def __init__(self, sorted_sources, sorted_targets, source_permutation, target_permutation,
                 leaf_source_offsets, leaf_target_offsets, root_centre, root_half_width, order, depth,
                 max_states=1, m2l_mode=M2L_AUTO, device=0):
        lib = library()
        self._keep = [np.ascontiguousarray(sorted_sources, dtype=np.float64).reshape(-1, 3),
                      np.ascontiguousarray(sorted_targets, dtype=np.float64).reshape(-1, 3),
                      np.ascontiguousarray(source_permutation, dtype=np.int32),
                      np.ascontiguousarray(target_permutation, dtype=np.int32),
                      np.ascontiguousarray(leaf_source_offsets, dtype=np.int32),
                      np.ascontiguousarray(leaf_target_offsets, dtype=np.int32)]
        d = PlanDesc()
        d.struct_size = ctypes.sizeof(PlanDesc)
        d.n_sources = len(self._keep[0])
        d.n_targets = len(self._keep[1])
        d.order = order
        d.depth = depth
        d.max_states = max_states
        d.m2l_mode = m2l_mode
        d.device = device
        for a in range(3):
            d.root_centre[a] = float(root_centre[a])
        d.root_half_width = float(root_half_width)
        (d.sorted_source_positions, d.sorted_target_positions, d.source_permutation,
         d.target_permutation, d.leaf_source_offsets, d.leaf_target_offsets) = [a.ctypes.data for a in self._keep]
        handle = ctypes.c_void_p()
        _check(lib.cdfmm_b200_plan_create(ctypes.byref(d), ctypes.byref(handle)))
        self._h = handle
        self.n_sources, self.n_targets, self.order, self.depth = d.n_sources, d.n_targets, order, depth
        self.n_coefficients = (order + 1) * (order + 2) * (order + 3) // 6
        self.n_nodes = ((1 << (3 * (depth + 1))) - 1) // 7
        self.max_states = max_states
        self._keep = None

    @classmethod
    def from_tree(cls, tree, order, **kw):
        """Builds the descriptor from a cdfmm.UniformTree (the host tree)."""
        depth = tree.max_level
        soff = np.asarray(tree.leaf_source_offsets(), dtype=np.int32)
        toff = np.asarray(tree.leaf_target_offsets(), dtype=np.int32)
        rc = tree.root_centre
        return cls(tree.sorted_source_positions(), tree.sorted_target_positions(), tree.source_permutation,
                   tree.target_permutation, soff, toff, (rc.x, rc.y, rc.z), tree.root_half_width, order, depth, **kw)

    @classmethod
    def from_points(cls, sources, order, depth, targets=None, root_centre=None, root_half_width=None,
                    self_map=None, max_states=1, m2l_mode=M2L_AUTO, device=0):
        """Builds the uniform octree on the device from user-order FP64
        positions ((n, 3) numpy array, or a contiguous float64 CUDA tensor
        with any array interface exposing data_ptr()) and the plan on it
        (cdfmm_b200_plan_create_from_points).  targets None: the targets are
        the sources, and self_map (default True then) excludes each point's
        own source from its near field.  The tree equals cdfmm.UniformTree's
        for the same points and options."""
        lib = library()

        def view(a):
            if hasattr(a, "data_ptr"):
                if a.dtype.__repr__() != "torch.float64" or not a.is_contiguous() or a.dim() != 2 or a.shape[1] != 3:
                    raise ValueError("device positions must be a contiguous (n, 3) float64 tensor")
                return a, a.data_ptr(), int(a.shape[0]), 0
            h = np.ascontiguousarray(a, dtype=np.float64).reshape(-1, 3)
            return h, h.ctypes.data, len(h), 1

        ks, sp, ns, host_s = view(sources)
        d = PointsDesc()
        d.struct_size = ctypes.sizeof(PointsDesc)
        d.n_sources = ns
        d.order, d.depth, d.max_states, d.m2l_mode, d.device = order, depth, max_states, m2l_mode, device
        d.positions_on_host = host_s
        d.source_positions = sp
        keep = [ks]
        if targets is not None:
            kt, tp, nt, host_t = view(targets)
            if host_t != host_s:
                raise ValueError("sources and targets must both be host arrays or both device arrays")
            keep.append(kt)
            d.n_targets, d.target_positions = nt, tp
            if self_map:
                raise ValueError("self_map needs targets=None (targets are the sources)")
        else:
            d.n_targets = ns
            d.self_map = 1 if self_map in (None, True) else 0
        flags = 0
        if root_centre is not None:
            flags |= ROOT_CENTRE
            for a in range(3):
                d.root_centre[a] = float(root_centre[a])
        if root_half_width is not None:
            flags |= ROOT_HALF_WIDTH
            d.root_half_width = float(root_half_width)
        d.root_flags = flags
        handle = ctypes.c_void_p()
        _check(lib.cdfmm_b200_plan_create_from_points(ctypes.byref(d), ctypes.byref(handle)))
        self = cls.__new__(cls)
        self._h = handle
        self.n_sources, self.n_targets, self.order, self.depth = ns, d.n_targets, order, depth
        self.n_coefficients = (order + 1) * (order + 2) * (order + 3) // 6
        self.n_nodes = ((1 << (3 * (depth + 1))) - 1) // 7
        self.max_states = max_states
        self._keep = None
        return self

    def tree(self) -> dict:
        """The plan's tree (cdfmm_b200_plan_tree): root centre and half
        width, permutations, leaf offsets and Morton-sorted positions."""
        nl = (1 << (3 * self.depth)) + 1
        root = np.zeros(4)
        sp = np.zeros(self.n_sources, dtype=np.int32)
        tp = np.zeros(self.n_targets, dtype=np.int32)
        so = np.zeros(nl, dtype=np.int32)
        to = np.zeros(nl, dtype=np.int32)
        sx = np.zeros((self.n_sources, 3))
        tx = np.zeros((self.n_targets, 3))
        _check(library().cdfmm_b200_plan_tree(self._h, *[a.ctypes.data for a in (root, sp, tp, so, to, sx, tx)]),
               self._h)
        return {"root_centre": root[:3].copy(), "root_half_width": float(root[3]), "source_permutation": sp,
                "target_permutation": tp, "leaf_source_offsets": so, "leaf_target_offsets": to,
                "sorted_source_positions": sx, "sorted_target_positions": tx}

    def close(self):
        if getattr(self, "_h", None):
            library().cdfmm_b200_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_source_cuboids(self, sizes, cuboid_p2m=True):
        """Uniformly magnetised cuboid sources (cdfmm_b200_set_source_cuboids):
        sizes (n_sources, 3) or (3,) / (1, 3) side lengths in user order;
        None returns to point dipoles."""
        if sizes is None:
            _check(library().cdfmm_b200_set_source_cuboids(self._h, None, 0, 0), self._h)
            return
        a = np.ascontiguousarray(sizes, dtype=np.float64).reshape(-1, 3)
        _check(library().cdfmm_b200_set_source_cuboids(self._h, _ptr(a), len(a), 1 if cuboid_p2m else 0), self._h)

    def set_self_indices(self, sorted_self):
        if sorted_self is None:
            _check(library().cdfmm_b200_set_self_indices(self._h, None), self._h)
            return
        a = np.ascontiguousarray(sorted_self, dtype=np.int32)
        if a.shape != (self.n_targets,):
            raise ValueError("sorted_self must have one entry per target")
        _check(library().cdfmm_b200_set_self_indices(self._h, _ptr(a)), self._h)

    def set_timing(self, enabled=True):
        """True / 1: per-stage times (stages serialised); 2: trace of the
        concurrent schedule; False / 0: off."""
        _check(library().cdfmm_b200_set_timing(self._h, int(enabled)), self._h)

    def set_schedule(self, schedule):
        """Near/far schedule of K > 1 evaluations (SCHEDULE_*)."""
        _check(library().cdfmm_b200_set_schedule(self._h, int(schedule)), self._h)

    def set_near_mode(self, mode):
        """Near-field arithmetic of evaluations of 8..128 states: NEAR_AUTO
        (tensor cores where supported), NEAR_FP32 or NEAR_TF32X3."""
        _check(library().cdfmm_b200_set_near_mode(self._h, int(mode)), self._h)

    def m2l_shapes(self) -> list:
        """Tensor-core M2L pipeline shapes of this plan as (accumulators per
        CTA, stages, fused) tuples (empty without the tensor-core M2L)."""
        lib = library()
        n = lib.cdfmm_b200_m2l_shapes(self._h, None, 0)
        if n < 0:
            _check(n, self._h)
        buf = (ctypes.c_int32 * (3 * max(n, 1)))()
        lib.cdfmm_b200_m2l_shapes(self._h, buf, n)
        return [(buf[3 * i], buf[3 * i + 1], bool(buf[3 * i + 2])) for i in range(n)]

    def set_m2l_shape(self, m_tiles, stages=0, fused=False):
        """Pins one of m2l_shapes() (no autotuning, run-to-run identical
        results); m_tiles = 0 returns to autotuning."""
        _check(library().cdfmm_b200_set_m2l_shape(self._h, int(m_tiles), int(stages), 1 if fused else 0), self._h)

    def poll_status(self):
        """Raises CdfmmError (ERR_TIMEOUT) if the completed work of an earlier
        call on this plan recorded an expired bounded wait not yet reported
        (cdfmm_b200_poll_status); does not wait for work in flight."""
        _check(library().cdfmm_b200_poll_status(self._h), self._h)

    def set_wait_limit(self, iterations):
        """Failure injection for tests: polls per tensor-core M2L progress
        wait before it expires (0: at once; negative: the default)."""
        _check(library().cdfmm_b200_set_wait_limit(self._h, int(iterations)), self._h)

    def stats(self) -> dict:
        s = Stats()
        _check(library().cdfmm_b200_get_stats(self._h, ctypes.byref(s)), self._h)
        return s.as_dict()

    def evaluate(self, moments, output="field", layout=LAYOUT_SEPARATE, field=None, potential=None,
                 stream=None, synchronize=True, memory=None):
        """Evaluates K states.

        moments: (K, n_sources, 3) or (n_sources, 3) host numpy (float32 or
        float64) or a tensor with data_ptr().  numpy inputs give numpy host
        results (allocated here when not supplied).  For tensors the caller
        supplies `field` / `potential` and `memory` defaults to "device" for
        CUDA tensors and "host" (pinned, ideally) for CPU tensors.
        """
        flags = {"field": OUTPUT_FIELD, "potential": OUTPUT_POTENTIAL, "both": OUTPUT_FIELD | OUTPUT_POTENTIAL}[output]
        is_tensor = hasattr(moments, "data_ptr")
        if is_tensor:
            K = int(moments.shape[0]) if len(moments.shape) == 3 else 1
            dtype = 1 if str(moments.dtype).endswith("float64") else 0
            if memory is None:
                memory = 0 if getattr(moments, "is_cuda", False) else MOMENTS_ON_HOST | RESULTS_ON_HOST
        else:
            moments = np.ascontiguousarray(moments)
            if moments.dtype not in (np.float32, np.float64):
                moments = moments.astype(np.float64)
            K = moments.shape[0] if moments.ndim == 3 else 1
            dtype = 1 if moments.dtype == np.float64 else 0
            memory = MOMENTS_ON_HOST | RESULTS_ON_HOST
            width = 4 if layout == LAYOUT_INTERLEAVED else 3
            if field is None and (flags & OUTPUT_FIELD or layout == LAYOUT_INTERLEAVED):
                field = np.zeros((K, self.n_targets, width), dtype=np.float32)
            if potential is None and flags & OUTPUT_POTENTIAL and layout == LAYOUT_SEPARATE:
                potential = np.zeros((K, self.n_targets), dtype=np.float32)
        a = EvalArgs()
        a.moments = _ptr(moments).value if moments is not None else None
        a.moments_dtype = dtype
        a.n_states = K
        a.output = flags
        a.layout = layout
        a.field = _ptr(field).value if field is not None else None
        a.potential = _ptr(potential).value if potential is not None else None
        a.memory = memory
        a.stream = stream
        a.synchronize = 1 if synchronize else 0
        _check(library().cdfmm_b200_evaluate(self._h, ctypes.byref(a)), self._h)
        return {"H": field, "phi": potential}

    def evaluate_noalloc(self, moments, field, potential=None, output="field", layout=LAYOUT_SEPARATE,
                         stream=None, synchronize=True):
        """Allocation-free evaluation (cdfmm_b200_evaluate_noalloc) on
        device-resident tensors; scratch comes from the library's fixed
        64 MiB device array instead of the plan."""
        flags = {"field": OUTPUT_FIELD, "potential": OUTPUT_POTENTIAL, "both": OUTPUT_FIELD | OUTPUT_POTENTIAL}[output]
        a = EvalArgs()
        a.moments = _ptr(moments).value
        a.moments_dtype = 1 if str(moments.dtype).endswith("float64") else 0
        a.n_states = int(moments.shape[0]) if len(moments.shape) == 3 else 1
        a.output = flags
        a.layout = layout
        a.field = _ptr(field).value if field is not None else None
        a.potential = _ptr(potential).value if potential is not None else None
        a.memory = 0
        a.stream = stream
        a.synchronize = 1 if synchronize else 0
        _check(library().cdfmm_b200_evaluate_noalloc(self._h, ctypes.byref(a)), self._h)

    def backward(self, grad_field, moments=None, grad_moments=None, grad_target_positions=None,
                 want_moments=True, want_positions=False, stream=None, synchronize=True, memory=None,
                 forward_evaluation=0):
        """Reverse mode of `evaluate` for L = sum w . H with w = grad_field
        (K, n_targets, 3) float32: returns {"moments": dL/dm (K, n_sources, 3),
        "positions": dL/dx_target (n_targets, 3), summed over states}.
        `moments` (the forward ones) are needed for the position gradient.
        numpy inputs give numpy outputs; for tensors the caller supplies the
        outputs it asks for."""
        is_tensor = hasattr(grad_field, "data_ptr")
        if is_tensor:
            K = int(grad_field.shape[0]) if len(grad_field.shape) == 3 else 1
            if memory is None:
                memory = 0 if getattr(grad_field, "is_cuda", False) else MOMENTS_ON_HOST | RESULTS_ON_HOST
        else:
            grad_field = np.ascontiguousarray(grad_field, dtype=np.float32)
            K = grad_field.shape[0] if grad_field.ndim == 3 else 1
            memory = MOMENTS_ON_HOST | RESULTS_ON_HOST
            if moments is not None:
                moments = np.ascontiguousarray(moments)
                if moments.dtype not in (np.float32, np.float64):
                    moments = moments.astype(np.float64)
            if want_moments and grad_moments is None:
                grad_moments = np.zeros((K, self.n_sources, 3), dtype=np.float32)
            if want_positions and grad_target_positions is None:
                grad_target_positions = np.zeros((self.n_targets, 3), dtype=np.float32)
        a = BackwardArgs()
        a.struct_size = ctypes.sizeof(BackwardArgs)
        a.n_states = K
        a.grad_field = _ptr(grad_field).value
        a.moments = _ptr(moments).value if moments is not None else None
        a.moments_dtype = 1 if moments is not None and str(moments.dtype).endswith("float64") else 0
        a.grad_moments = _ptr(grad_moments).value if (want_moments and grad_moments is not None) else None
        a.grad_target_positions = (_ptr(grad_target_positions).value
                                   if (want_positions and grad_target_positions is not None) else None)
        a.memory = memory
        a.stream = stream
        a.synchronize = 1 if synchronize else 0
        a.forward_evaluation = int(forward_evaluation)
        _check(library().cdfmm_b200_backward(self._h, ctypes.byref(a)), self._h)
        return {"moments": grad_moments if want_moments else None,
                "positions": grad_target_positions if want_positions else None}

    def read_expansions(self, which="multipole", state=0) -> np.ndarray:
        out = np.zeros(self.n_nodes * self.n_coefficients, dtype=np.float32)
        w = 0 if which == "multipole" else 1
        _check(library().cdfmm_b200_read_expansions(self._h, w, state, _ptr(out), out.size), self._h)
        return out.reshape(self.n_nodes, self.n_coefficients)


class Batch:
    """Several plans (independent geometries) evaluated by one CUDA graph
    launch (cdfmm_b200_batch_*).  `items` is a list of (plan, moments,
    field, potential) with device tensors (moments (K, ns, 3); field
    (K, nt, 3); potential (K, nt) or None); arguments are fixed here."""

    def __init__(self, items, output="field", layout=LAYOUT_SEPARATE):
        flags = {"field": OUTPUT_FIELD, "potential": OUTPUT_POTENTIAL, "both": OUTPUT_FIELD | OUTPUT_POTENTIAL}[output]
        n = len(items)
        plans = (ctypes.c_void_p * n)()
        args = (EvalArgs * n)()
        self._keep = []
        for i, (plan, moments, field, potential) in enumerate(items):
            plans[i] = plan._h.value if isinstance(plan._h, ctypes.c_void_p) else plan._h
            a = args[i]
            a.moments = _ptr(moments).value
            a.moments_dtype = 1 if str(moments.dtype).endswith("float64") else 0
            a.n_states = int(moments.shape[0]) if len(moments.shape) == 3 else 1
            a.output = flags
            a.layout = layout
            a.field = _ptr(field).value if field is not None else None
            a.potential = _ptr(potential).value if potential is not None else None
            a.memory = 0
            a.stream = None
            a.synchronize = 0
            self._keep.append((plan, moments, field, potential))
        handle = ctypes.c_void_p()
        _check(library().cdfmm_b200_batch_create(plans, args, n, ctypes.byref(handle)))
        self._h = handle

    def launch(self, stream=None, synchronize=True):
        _check(library().cdfmm_b200_batch_launch(self._h, stream, 1 if synchronize else 0))

    def groups(self) -> list:
        """Stacked-M2L group of each plan (-1: evaluated on its own)."""
        n = len(self._keep)
        buf = (ctypes.c_int32 * max(n, 1))()
        got = library().cdfmm_b200_batch_groups(self._h, buf, n)
        if got < 0:
            _check(got)
        return [int(buf[i]) for i in range(n)]

    def close(self):
        if getattr(self, "_h", None):
            library().cdfmm_b200_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def dipole_field(plan: DevicePlan, moments, target_positions=None):
    """Differentiable field H = FMM(moments) on `plan`'s fixed geometry.

    moments: CUDA float32 tensor (K, n_sources, 3) (or (n_sources, 3));
    target_positions: optional CUDA tensor (n_targets, 3) holding the plan's
    target positions (user order).  It is not read -- the geometry is the
    plan's -- but gradients flow to it: dL/dx = sum over states of the
    position gradient.  Returns (K, n_targets, 3) float32 (squeezed like the
    input).  torch.autograd.Function wrapper of cdfmm_b200_evaluate /
    cdfmm_b200_backward, on the current CUDA stream, no host copies.
    """
    import torch

    class _DipoleField(torch.autograd.Function):
        @staticmethod
        def forward(ctx, m, x):
            squeeze = m.dim() == 2
            m3 = (m.unsqueeze(0) if squeeze else m).contiguous()
            if m3.dtype != torch.float32:
                m3 = m3.float()
            H = torch.empty((m3.shape[0], plan.n_targets, 3), dtype=torch.float32, device=m3.device)
            plan.evaluate(m3, output="field", field=H, stream=torch.cuda.current_stream(m3.device).cuda_stream,
                          synchronize=False)
            ctx.save_for_backward(m3)
            ctx.squeeze = squeeze
            # lets the backward reuse this evaluation's moments and locals if
            # nothing else evaluates on the plan in between
            ctx.evaluation = plan.stats()["evaluations"]
            return H.squeeze(0) if squeeze else H

        @staticmethod
        def backward(ctx, gH):
            (m3,) = ctx.saved_tensors
            g3 = (gH.unsqueeze(0) if ctx.squeeze else gH).contiguous().float()
            want_m = ctx.needs_input_grad[0]
            want_x = ctx.needs_input_grad[1]
            gm = torch.empty_like(m3) if want_m else None
            gx = torch.empty((plan.n_targets, 3), dtype=torch.float32, device=m3.device) if want_x else None
            if want_m or want_x:
                plan.backward(g3, moments=m3, grad_moments=gm, grad_target_positions=gx, want_moments=want_m,
                              want_positions=want_x, stream=torch.cuda.current_stream(m3.device).cuda_stream,
                              synchronize=False, forward_evaluation=ctx.evaluation)
            if gm is not None and ctx.squeeze:
                gm = gm.squeeze(0)
            return gm, gx

    return _DipoleField.apply(moments, target_positions)
